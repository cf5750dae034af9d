"""Central finite-difference check of the fused backward against an FP64 forward on the
GPU (qsdvr_render_loss_f64), in fixed mode, where the backward is the exact gradient.

The FD derivative of L(theta) = mean |color - target|^2 for entry j is
(L(theta + h e_j) - L(theta - h e_j)) / 2h with h = 1e-3 in double precision."""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import F32, P, U32, call

_lib.extra_signatures({"qsdvr_render_loss_f64": [P, P, P, U32, U32, F32, ctypes.c_double, P, P, P, P, P]})


def loss_f64(rays, origin, direction, sdf_grid64, data64, reso, interval, k, target64) -> float:
    """Mean squared error of the FP64 render (mean over rays x 3)."""
    n = rays.shape[0]
    out = torch.empty(n, dtype=torch.float64, device=rays.device)
    call("qsdvr_render_loss_f64", ctypes.c_void_p(rays.data_ptr()), ctypes.c_void_p(origin.data_ptr()),
         ctypes.c_void_p(direction.data_ptr()), n, int(reso), float(interval), float(k),
         ctypes.c_void_p(sdf_grid64.data_ptr()), ctypes.c_void_p(data64.data_ptr()), ctypes.c_void_p(target64.data_ptr()),
         ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(torch.cuda.current_stream(rays.device).cuda_stream))
    return float(out.sum()) / (3 * n)


def finite_differences(rays, origin, direction, sdf_grid, data, reso, interval, k, target, sdf_entries, data_entries,
                       h: float = 1e-3):
    """FD gradients (double) of the mean-squared loss at the given flat entries of the
    [R^3,8] SDF grid and the [(R+1)^3,32] appearance grid."""
    g64 = sdf_grid.double().contiguous().clone()
    d64 = data.double().contiguous().clone()
    t64 = target.double().contiguous()
    out = []
    for grid, entries in ((g64, sdf_entries), (d64, data_entries)):
        flat = grid.view(-1)
        fd = torch.empty(len(entries), dtype=torch.float64)
        for i, e in enumerate(entries.tolist()):
            v = flat[e].item()
            flat[e] = v + h
            lp = loss_f64(rays, origin, direction, g64, d64, reso, interval, k, t64)
            flat[e] = v - h
            lm = loss_f64(rays, origin, direction, g64, d64, reso, interval, k, t64)
            flat[e] = v
            fd[i] = (lp - lm) / (2 * h)
        out.append(fd)
    return out
