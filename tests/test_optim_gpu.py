"""Fused grid Adam (qsdvr_adam_step) against torch.optim.Adam."""
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = "cuda"


@pytest.mark.parametrize("n", [4096 * 33 + 3, 1 << 20])
def test_fused_adam_matches_torch_adam(n):
    from qsdvr_b200.optim import FusedGridAdam

    gen = torch.Generator(device=DEV).manual_seed(0)
    p0 = torch.randn(n, generator=gen, device=DEV)
    a = torch.nn.Parameter(p0.clone())
    b = torch.nn.Parameter(p0.clone())
    copy = torch.empty(n, dtype=torch.bfloat16, device=DEV)
    ref = torch.optim.Adam([a], lr=1e-2, betas=(0.9, 0.999), eps=1e-8)
    ours = FusedGridAdam([b], lr=1e-2, betas=(0.9, 0.999), eps=1e-8, bf16_copies={b: copy})
    for step in range(5):
        g = torch.randn(n, generator=gen, device=DEV) * (0.1 + step)
        a.grad = g.clone()
        b.grad = g.clone()
        ref.step()
        ours.step()
        assert torch.count_nonzero(b.grad) == 0  # zeroed by the fused step
        err = (a.detach() - b.detach()).abs().max().item() / a.detach().abs().max().item()
        assert err < 1e-6, (step, err)
    assert torch.equal(copy, b.detach().to(torch.bfloat16))
    sa, sb = ref.state[a], ours.state[b]
    assert (sa["exp_avg"] - sb["exp_avg"]).abs().max().item() < 1e-6
    assert (sa["exp_avg_sq"] - sb["exp_avg_sq"]).abs().max().item() < 1e-6


def test_skip_zero_grad_leaves_untouched_entries():
    from qsdvr_b200.optim import adam_step

    n = 1 << 16
    p = torch.randn(n, device=DEV)
    g = torch.randn(n, device=DEV)
    g[::3] = 0.0
    m, v = torch.zeros_like(p), torch.zeros_like(p)
    m[::3] = 0.5
    v[::3] = 0.25
    p0, m0, v0 = p.clone(), m.clone(), v.clone()
    adam_step(p, g, m, v, 7, 1e-2, skip_zero_grad=True)
    assert torch.equal(p[::3], p0[::3]) and torch.equal(m[::3], m0[::3]) and torch.equal(v[::3], v0[::3])
    touched = torch.ones(n, dtype=torch.bool, device=DEV)
    touched[::3] = False
    assert (p[touched] != p0[touched]).all()


@pytest.mark.parametrize("n", [4096 * 33 + 3, 1 << 20])
def test_bf16_gradient_adam_matches_fp32(n):
    """QSDVR_ADAM_GRAD_BF16: the fused step reads a bf16 gradient exactly as the same values in
    fp32 (parameters, moments and the bf16 copy identical) and zeroes it."""
    from qsdvr_b200.optim import adam_step

    gen = torch.Generator(device=DEV).manual_seed(3)
    p0 = torch.randn(n, generator=gen, device=DEV)
    g16 = (torch.randn(n, generator=gen, device=DEV) * 0.3).to(torch.bfloat16)
    outs = []
    for grad in (g16.clone(), g16.float()):
        p, m, v = p0.clone(), torch.zeros_like(p0), torch.zeros_like(p0)
        copy = torch.empty(n, dtype=torch.bfloat16, device=DEV)
        adam_step(p, grad, m, v, 1, 1e-2, param_bf16=copy)
        assert torch.count_nonzero(grad) == 0
        outs.append((p, m, v, copy))
    for a, b in zip(*outs):
        assert torch.equal(a, b)


def test_sdf_cells_adam_and_bf16_form():
    """QSDVR_ADAM_SDF_CELLS: the same fp32 update as the element-wise step, and the bf16 copy in
    the compensated cell form, bit-identical with qsdvr_sdf_cells_bf16 on the updated masters
    and with the oracle's float32 restatement; the kernels read a6 as slot 6 + slot 7."""
    import numpy as np

    import oracle.oracle as O
    from qsdvr_b200 import fused, scenes
    from qsdvr_b200.optim import adam_step

    R = 24
    grid8 = fused.pad_grid7(scenes.procedural_grid(R, seed=3).reshape(-1, 7)).to(DEV)
    enc = fused.sdf_cells_bf16(grid8)
    want = O.sdf_cells_bf16(grid8.cpu().numpy())
    assert np.array_equal(enc.cpu().view(torch.int16).numpy().view(np.uint16), want)
    gen = torch.Generator(device=DEV).manual_seed(4)
    g = torch.randn(grid8.shape, generator=gen, device=DEV) * 1e-3
    g[::5] = 0.0  # whole cells without gradient keep their copy under skip_zero_grad
    outs = []
    for cells in (False, True):
        p, m, v = grid8.clone(), torch.zeros_like(grid8), torch.zeros_like(grid8)
        copy = torch.zeros(grid8.shape, dtype=torch.bfloat16, device=DEV)
        adam_step(p, g.clone(), m, v, 1, 1e-2, param_bf16=copy, sdf_cells=cells, skip_zero_grad=True)
        outs.append((p, m, v, copy))
    (p0, m0, v0, c0), (p1, m1, v1, c1) = outs
    assert torch.equal(p0, p1) and torch.equal(m0, m1) and torch.equal(v0, v1)
    touched = g.abs().sum(1) != 0
    assert torch.equal(c1[touched], fused.sdf_cells_bf16(p1)[touched])
    assert torch.count_nonzero(c1[~touched]) == 0  # untouched cells were not rewritten
    assert torch.equal(c0[touched], p0[touched].to(torch.bfloat16))


def test_bf16_state_adam_tracks_fp32_state():
    """QSDVR_ADAM_STATE_BF16: the moments live in bf16, updated in fp32 and stochastically
    rounded back.  After one step each stored moment is one of the two bf16 neighbours of the
    fp32-state value, unbiased on average, and the farther one a quarter of the time (as
    stochastic rounding of uniformly placed values gives); after 5 steps the parameters stay
    within 0.1 of one step's size of the fp32-state run."""
    from qsdvr_b200.optim import adam_step

    n = (1 << 20) + 3  # with a tail of 3 elements
    gen = torch.Generator(device=DEV).manual_seed(5)
    p0 = torch.randn(n, generator=gen, device=DEV)
    grads = [torch.randn(n, generator=gen, device=DEV) * (0.2 + s) for s in range(5)]
    lr = 1e-2
    runs = {}
    for dt in (torch.float32, torch.bfloat16):
        p, m, v = p0.clone(), torch.zeros(n, dtype=dt, device=DEV), torch.zeros(n, dtype=dt, device=DEV)
        for step, g in enumerate(grads, 1):
            adam_step(p, g.clone(), m, v, step, lr)
            if step == 1:
                runs[(dt, "m1")], runs[(dt, "v1")] = m.float().clone(), v.float().clone()
        runs[dt] = p
    for key in ("m1", "v1"):
        exact, got = runs[(torch.float32, key)], runs[(torch.bfloat16, key)]
        lo = exact.to(torch.bfloat16).float()
        ulp = (torch.nextafter(exact.to(torch.bfloat16), torch.full_like(lo, float("inf")).to(torch.bfloat16)).float()
               - lo).abs()
        assert ((got - exact).abs() <= 2 * ulp).all(), key
        rel = (got - exact) / ulp.clamp_min(1e-30)
        assert abs(float(rel.mean())) < 5e-3, key  # unbiased
        # stochastic, not nearest: a quarter of the values go to the farther neighbour
        far = float((rel.abs() > 0.5).float().mean())
        assert 0.2 < far < 0.3, (key, far)
    err = float((runs[torch.bfloat16] - runs[torch.float32]).abs().max())
    assert err < 0.1 * lr, err  # 5 steps of ~lr each, moments within 2^-8
