"""Resume on the GPU: training 3 steps, saving, and resuming to 6 ends where 6 uninterrupted
steps end (same ray batches through the restored generator, same Adam and proposal-network
state).  The gradient REDs sum in launch order, so the two runs agree to float rounding, not
bit for bit: grids within 1e-4 relative (max-abs error over max-abs value)."""
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _args(tmp, steps, **kw):
    from qsdvr_b200 import train

    a = train.parser().parse_args([])
    a.reso, a.views, a.size, a.rays, a.steps, a.log_every = 32, 3, 48, 2048, steps, 10 ** 9
    a.interval, a.proposal, a.proposal_warmup, a.proposal_rays, a.proposal_points = 4.0 / 96, True, 1, 512, 4096
    for k, v in kw.items():
        setattr(a, k, v)
    return a


def test_resume_matches_uninterrupted_run(tmp_path):
    from qsdvr_b200 import _lib, train

    _lib.lib()
    dev = torch.device("cuda", 0)
    a0 = _args(tmp_path, 6)
    data = train.build(a0.reso, a0.views, a0.size, 1111.1 * a0.size / 800, 4.03, a0.interval, a0.k, a0.seed, dev)
    _, m_full, n_full = train.run(a0, data, quiet=True, return_state=True)
    ck = str(tmp_path / "ck.pt")
    train.run(_args(tmp_path, 3, save=ck), data, quiet=True)
    out, m_res, n_res = train.run(_args(tmp_path, 6, resume=ck), data, quiet=True, return_state=True)
    assert out["first_step"] == 4
    assert rel_err(m_res.sdfGrid.detach().cpu(), m_full.sdfGrid.detach().cpu()) < 1e-4
    assert rel_err(m_res.renderData.detach().cpu(), m_full.renderData.detach().cpu()) < 1e-4
    assert n_res.step_count == n_full.step_count == 6
    assert rel_err(n_res.params.cpu(), n_full.params.cpu()) < 1e-4
    assert _lib.device_error() == 0
