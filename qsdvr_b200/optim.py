"""Fused grid optimizer (qsdvr_adam_step): torch.optim.Adam's update for grid parameters
in one HBM pass, with the gradient zeroed and the bf16 storage copy refreshed in the same
pass.  Replaces ``optimizer.step(); optimizer.zero_grad()`` of the reference's training
loop (test.py:34-35) for the grids."""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import I32, P, U32, U64, call

ZERO_GRAD = 1
SKIP_ZERO_GRAD = 2
GRAD_BF16 = 4
SDF_CELLS = 8
STATE_BF16 = 16


class AdamArgs(ctypes.Structure):
    """qsdvr_adam_args (include/qsdvr_b200.h)."""
    _fields_ = [("param", P), ("grad", P), ("exp_avg", P), ("exp_avg_sq", P), ("param_bf16", P), ("count", U64),
                ("lr", ctypes.c_double), ("beta1", ctypes.c_double), ("beta2", ctypes.c_double),
                ("eps", ctypes.c_double), ("step", U32), ("flags", I32)]


_lib.extra_signatures({"qsdvr_adam_step": [ctypes.POINTER(AdamArgs), P]})


def adam_step(param, grad, exp_avg, exp_avg_sq, step, lr, betas=(0.9, 0.999), eps=1e-8, param_bf16=None,
              zero_grad=True, skip_zero_grad=False, sdf_cells=False):
    """One fused Adam step.  ``sdf_cells``: ``param`` is a quadric cell grid [R^3,8] and its
    bf16 copy is written in the compensated cell form (``fused.sdf_cells_bf16``).  bfloat16
    moments (both) are updated in fp32 and stochastically rounded back."""
    if not param.is_cuda or param.dtype != torch.float32 or not param.is_contiguous():
        raise ValueError("param must be a contiguous CUDA float32 tensor")
    state_bf16 = exp_avg.dtype == torch.bfloat16
    for t, nm in ((exp_avg, "exp_avg"), (exp_avg_sq, "exp_avg_sq")):
        if (not t.is_cuda or t.dtype != exp_avg.dtype or t.dtype not in (torch.float32, torch.bfloat16)
                or not t.is_contiguous() or t.numel() != param.numel()):
            raise ValueError(f"{nm} must be a contiguous CUDA float32 (or, both moments, bfloat16) tensor shaped "
                             "like param")
    if (not grad.is_cuda or grad.dtype not in (torch.float32, torch.bfloat16) or not grad.is_contiguous()
            or grad.numel() != param.numel()):
        raise ValueError("grad must be a contiguous CUDA float32 or bfloat16 tensor shaped like param")
    if param_bf16 is not None and (param_bf16.dtype != torch.bfloat16 or param_bf16.numel() != param.numel()):
        raise ValueError("param_bf16 must be a bfloat16 tensor shaped like param")
    a = AdamArgs()
    a.param, a.grad, a.exp_avg, a.exp_avg_sq = param.data_ptr(), grad.data_ptr(), exp_avg.data_ptr(), exp_avg_sq.data_ptr()
    a.param_bf16 = param_bf16.data_ptr() if param_bf16 is not None else None
    a.count = param.numel()
    a.lr, a.beta1, a.beta2, a.eps = float(lr), float(betas[0]), float(betas[1]), float(eps)
    a.step = int(step)
    a.flags = ((ZERO_GRAD if zero_grad else 0) | (SKIP_ZERO_GRAD if skip_zero_grad else 0)
               | (GRAD_BF16 if grad.dtype == torch.bfloat16 else 0) | (SDF_CELLS if sdf_cells else 0)
               | (STATE_BF16 if state_bf16 else 0))
    with torch.cuda.device(param.device):
        call("qsdvr_adam_step", ctypes.byref(a), ctypes.c_void_p(torch.cuda.current_stream(param.device).cuda_stream))


class FusedGridAdam(torch.optim.Optimizer):
    """Adam for grid parameters using the fused kernel.  ``step()`` also zeroes the
    gradients (so ``zero_grad()`` is a no-op) and, for parameters registered with a bf16
    copy via ``bf16_copies={param: copy}``, refreshes the copy.  ``grads={param: tensor}``
    names a gradient buffer to use instead of ``param.grad`` (e.g. a bf16 one, which torch
    does not allow as the .grad of an fp32 parameter).  Parameters in ``sdf_cells`` are
    quadric cell grids [R^3,8]: their bf16 copies take the compensated cell form.
    ``state_dtype=torch.bfloat16`` keeps the moments in bf16 (stochastic rounding; 24 instead
    of 32 bytes of traffic per parameter and step).  ``skip_zero_grad`` leaves elements whose
    gradient is exactly 0 untouched (their moments do not decay that step, unlike torch's)."""

    def __init__(self, params, lr=1e-2, betas=(0.9, 0.999), eps=1e-8, bf16_copies=None, skip_zero_grad=False,
                 grads=None, sdf_cells=(), state_dtype=torch.float32):
        super().__init__(params, dict(lr=lr, betas=betas, eps=eps))
        self.state_dtype = state_dtype
        self.bf16_copies = bf16_copies or {}
        self.skip_zero_grad = skip_zero_grad
        self.grads = grads or {}
        self.sdf_cells = {id(p) for p in sdf_cells}

    def zero_grad(self, set_to_none: bool = False):
        pass  # step() already wrote zeros over the gradients it consumed

    @torch.no_grad()
    def step(self, closure=None):
        for group in self.param_groups:
            for p in group["params"]:
                grad = self.grads.get(p, p.grad)
                if grad is None:
                    continue
                st = self.state[p]
                if not st:
                    st["step"] = 0
                    st["exp_avg"] = torch.zeros_like(p, dtype=self.state_dtype, memory_format=torch.contiguous_format)
                    st["exp_avg_sq"] = torch.zeros_like(p, dtype=self.state_dtype,
                                                        memory_format=torch.contiguous_format)
                st["step"] += 1
                adam_step(p.data, grad, st["exp_avg"], st["exp_avg_sq"], st["step"], group["lr"], group["betas"],
                          group["eps"], self.bf16_copies.get(p), True, self.skip_zero_grad,
                          sdf_cells=id(p) in self.sdf_cells)
