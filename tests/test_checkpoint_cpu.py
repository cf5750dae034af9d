"""Checkpoint round trip on the CPU: the master grids, the fused Adam state, the proposal
network with its Adam state, the step and the ray-batch generator come back exactly, into
the existing objects (the optimizer's bf16 copies stay the same tensors)."""
import pytest
import torch


def _setup(seed, storage="bf16"):
    from qsdvr_b200.fused import DenseRenderGrid
    from qsdvr_b200.optim import FusedGridAdam
    from qsdvr_b200.proposal import ProposalNet

    g = torch.Generator().manual_seed(seed)
    model = DenseRenderGrid(8, 5.0, 4.0 / 64, mode="fixed", storage=storage, device="cpu")
    with torch.no_grad():
        model.sdfGrid.add_(torch.rand(model.sdfGrid.shape, generator=g))
        model.renderData.add_(torch.rand(model.renderData.shape, generator=g))
    model.sync_storage()
    copies = dict(zip((model.sdfGrid, model.renderData), model._copies)) if storage == "bf16" else None
    opt = FusedGridAdam(model.parameters(), lr=1e-2, bf16_copies=copies)
    for p in model.parameters():  # Adam state as the fused step leaves it (that step needs a GPU)
        opt.state[p] = {"step": 7, "exp_avg": torch.rand(p.shape, generator=g),
                        "exp_avg_sq": torch.rand(p.shape, generator=g)}
    net = ProposalNet("cpu", seed=seed)
    with torch.no_grad():
        net.params.add_(torch.rand(net.params.shape, generator=g))
        net.params_bf16.copy_(net.params.to(torch.bfloat16))
        net.m.copy_(torch.rand(net.m.shape, generator=g))
        net.v.copy_(torch.rand(net.v.shape, generator=g))
    net.step_count = 11
    gen = torch.Generator().manual_seed(seed + 1)
    torch.randint(0, 100, (5,), generator=gen)
    return model, opt, net, gen


def test_checkpoint_round_trip(tmp_path):
    from qsdvr_b200 import checkpoint

    model, opt, net, gen = _setup(0)
    path = str(tmp_path / "ck.pt")
    checkpoint.save(path, model, opt, net, step=42, generator=gen)
    m2, o2, n2, g2 = _setup(1)
    copy_ids = [id(c) for c in m2._copies]
    assert checkpoint.load(path, m2, o2, n2, g2) == 42
    assert torch.equal(m2.sdfGrid, model.sdfGrid) and torch.equal(m2.renderData, model.renderData)
    assert [id(c) for c in m2._copies] == copy_ids
    assert torch.equal(m2._copies[1], model.renderData.detach().to(torch.bfloat16))
    for p, q in zip(model.parameters(), m2.parameters()):
        a, b = opt.state[p], o2.state[q]
        assert a["step"] == b["step"] and torch.equal(a["exp_avg"], b["exp_avg"])
        assert torch.equal(a["exp_avg_sq"], b["exp_avg_sq"])
    for k in ("params", "params_bf16", "m", "v"):
        assert torch.equal(getattr(n2, k), getattr(net, k))
    assert n2.step_count == 11
    assert torch.equal(torch.randint(0, 100, (8,), generator=g2), torch.randint(0, 100, (8,), generator=gen))


def test_checkpoint_rejects_other_configuration(tmp_path):
    from qsdvr_b200 import checkpoint
    from qsdvr_b200.fused import DenseRenderGrid

    model, opt, net, gen = _setup(0)
    path = str(tmp_path / "ck.pt")
    checkpoint.save(path, model, opt)
    other = DenseRenderGrid(16, 5.0, 4.0 / 64, mode="fixed", storage="bf16", device="cpu")
    with pytest.raises(ValueError):
        checkpoint.load(path, other)
    with pytest.raises(ValueError):
        checkpoint.load(path, model, opt, net)  # saved without a proposal network
