"""vg_sht_analysis_noalloc (device buffers, static device scratch, no
allocation) against vg_sht_analysis on the same fields, two calls in a row
with different inputs, then a batch of two and a request over the scratch
limit. Kept in its own file, collected last, so it runs alone or after the
rest of the GPU suite."""
import ctypes as C

import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib

pytestmark = pytest.mark.gpu

SCRATCH_DOUBLES = 1 << 19  # VG_NOALLOC_SCRATCH_DOUBLES


def model(lmax):
    p = vlib.default_params()
    p.lmax, p.nlat, p.nphi = lmax, lmax + 1, 2 * (lmax + 1)
    return vlib.Model(p)


def noalloc(m, d_f, d_q, batch):
    import torch

    torch.cuda.synchronize()
    rc = vlib.lib().vg_sht_analysis_noalloc(m.h, C.c_void_p(d_f.data_ptr()), C.c_void_p(d_q.data_ptr()), batch)
    torch.cuda.synchronize()
    return rc


def test_noalloc_analysis_matches_existing_entry_point():
    import torch

    m = model(64)
    rng = np.random.default_rng(3)
    d_q = torch.empty(2 * m.nlm, dtype=torch.float64, device="cuda")
    for _ in range(2):  # two calls in a row, fresh input each time
        f = rng.standard_normal(m.ng)
        d_f = torch.from_numpy(f).cuda()
        assert noalloc(m, d_f, d_q, 1) == 0, vlib.lib().vg_last_error(m.h).decode()
        q_new = d_q.cpu().numpy()
        q_old = m.analysis(f)
        q_old = np.stack([q_old.real, q_old.imag], axis=1).reshape(-1)
        assert np.abs(q_new - q_old).max() <= 1e-13 * np.abs(q_old).max()


def test_noalloc_batch_and_limit():
    import torch

    m = model(32)
    rng = np.random.default_rng(4)
    fs = [rng.standard_normal(m.ng) for _ in range(2)]
    d_f = torch.from_numpy(np.concatenate(fs)).cuda()
    d_q = torch.empty(2 * 2 * m.nlm, dtype=torch.float64, device="cuda")
    assert noalloc(m, d_f, d_q, 2) == 0, vlib.lib().vg_last_error(m.h).decode()
    q = d_q.cpu().numpy().reshape(2, -1)
    for b in range(2):
        ref = m.analysis(fs[b])
        ref = np.stack([ref.real, ref.imag], axis=1).reshape(-1)
        assert np.abs(q[b] - ref).max() <= 1e-13 * np.abs(ref).max()
    too_many = SCRATCH_DOUBLES // (2 * (m.p.lmax + 1) * m.p.nlat) + 1
    assert noalloc(m, d_f, d_q, too_many) != 0
    assert "scratch" in vlib.lib().vg_last_error(m.h).decode()
