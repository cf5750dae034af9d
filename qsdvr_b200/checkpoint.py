"""Checkpoint and resume of a training run: the fp32 master grids, the fused Adam state, the
proposal network with its Adam state, the step count and the state of the ray-batch random
generator.  The reference writes only images (test.py:41-44); a run resumed from a checkpoint
draws the same ray batches as the uninterrupted run.

    save(path, model, optimizer, net=None, step=0, generator=None)
    step = load(path, model, optimizer, net=None, generator=None)

``load`` restores into existing objects in place, so references held elsewhere (the
optimizer's bf16 storage copies, CUDA tensors passed to kernels) stay valid.
"""
from __future__ import annotations

import torch

FORMAT = 1


def _config(model) -> dict:
    return {"reso": model.reso, "interval": model.interval, "mode": model.mode, "storage": model.storage,
            "transmittance": model.transmittance, "logisticCoef": model.logisticCoef,
            "channels": int(model.renderData.shape[1])}


def save(path, model, optimizer=None, net=None, step: int = 0, generator=None) -> None:
    """Write the training state to ``path`` (torch.save; tensors are stored on the CPU)."""
    state = {
        "format": FORMAT,
        "config": _config(model),
        "model": {k: v.detach().cpu() for k, v in model.state_dict().items()},
        "optimizer": None,
        "proposal": None,
        "step": int(step),
        "generator": generator.get_state() if generator is not None else None,
    }
    if optimizer is not None:
        opt = optimizer.state_dict()
        opt["state"] = {i: {k: (v.detach().cpu() if torch.is_tensor(v) else v) for k, v in s.items()}
                        for i, s in opt["state"].items()}
        state["optimizer"] = opt
    if net is not None:
        state["proposal"] = {"params": net.params.detach().cpu(), "m": net.m.detach().cpu(),
                             "v": net.v.detach().cpu(), "step_count": int(net.step_count), "lr": float(net.lr),
                             "under_weight": float(net.under_weight)}
    torch.save(state, path)


def load(path, model, optimizer=None, net=None, generator=None) -> int:
    """Restore the state saved by ``save`` into ``model`` (and the optimizer, proposal network
    and generator when given); returns the saved step.  The model's configuration must
    match the saved one."""
    state = torch.load(path, map_location="cpu", weights_only=True)
    if state.get("format") != FORMAT:
        raise ValueError(f"{path}: not a qsdvr_b200 checkpoint (format {state.get('format')})")
    want, have = state["config"], _config(model)
    if want != have:
        raise ValueError(f"{path}: checkpoint configuration {want} does not match the model's {have}")
    with torch.no_grad():
        params = dict(model.named_parameters())
        for k, v in state["model"].items():
            params[k].copy_(v)
        if model.storage == "bf16" and model._copies is not None:
            model.sync_storage()
    if optimizer is not None:
        if state["optimizer"] is None:
            raise ValueError(f"{path}: the checkpoint holds no optimizer state")
        optimizer.load_state_dict(state["optimizer"])
    if net is not None:
        p = state["proposal"]
        if p is None:
            raise ValueError(f"{path}: the checkpoint holds no proposal network")
        with torch.no_grad():
            net.params.copy_(p["params"])
            net.params_bf16.copy_(net.params.to(torch.bfloat16))
            net.m.copy_(p["m"])
            net.v.copy_(p["v"])
        net.step_count, net.lr, net.under_weight = p["step_count"], p["lr"], p["under_weight"]
    if generator is not None and state["generator"] is not None:
        generator.set_state(state["generator"])
    return int(state["step"])
