"""Ensemble batching through vg_update_batch: independent instances with their
own lmax, earth, viscosity and precision, advanced together, give exactly the
results of advancing them one after the other; a failing instance is reported
by index without disturbing the others; bad arguments are refused."""
import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth

pytestmark = pytest.mark.gpu


def members():
    return [
        synth.EnsembleMember("a", 16, 20, 70.0, 3e20, 4e21, True, 11),
        synth.EnsembleMember("b", 24, 24, 100.0, 8e20, 2e22, False, 12),
        synth.EnsembleMember("c", 32, 30, 55.0, 1.5e20, 1e21, True, 13),
        synth.EnsembleMember("d", 20, 16, 90.0, 5e20, 5e22, True, 14),
    ]


def make(mb, precision):
    p = mb.params(vlib.default_params)
    p.visc3d_precision = precision if mb.visc3d else 0
    m = vlib.Model(p)
    zb, hi = mb.reference()
    m.set_reference(zb, hi)
    if mb.visc3d:
        m.enable_visc3d(mb.pert(m.p))
    return m


@pytest.mark.parametrize("on_device", [False, True])
def test_batch_equals_sequential(on_device):
    import torch

    ms = members()
    precisions = [0, 0, 1, 0]  # split tensor-core and FP64 3-D instances side by side
    batched = [make(mb, pr) for mb, pr in zip(ms, precisions)]
    single = [make(mb, pr) for mb, pr in zip(ms, precisions)]
    for step in range(1, 4):
        ices = [mb.ice_at(step * 300) for mb in ms]
        if on_device:
            dev = [torch.tensor(x, device="cuda") for x in ices]
            vlib.update_batch(batched, [d.data_ptr() for d in dev], 50.0, on_device=True, nthreads=3)
            torch.cuda.synchronize()
        else:
            vlib.update_batch(batched, ices, 50.0)
        for m, x in zip(single, ices):
            m.update(x, 50.0)
    for a, b in zip(batched, single):
        fa, fb = a.fields(), b.fields()
        assert np.array_equal(fa[0], fb[0])
        assert np.array_equal(fa[1], fb[1])
        (sa, ta), (sb, tb) = a.state(), b.state()
        assert ta == tb
        for x, y in zip(sa, sb):
            assert np.array_equal(x, y)


def test_batch_reports_the_failing_instance():
    ms = members()[:3]
    models = [make(mb, 0) for mb in ms]
    p = ms[1].params(vlib.default_params)
    models[1] = vlib.Model(p)  # no reference set: its update must fail
    with pytest.raises(vlib.VilmaError, match=r"instance 1: .*vg_set_reference"):
        vlib.update_batch(models, [mb.ice_at(300) for mb in ms], 50.0)
    # the other instances advanced
    assert models[0].info().time_yr == pytest.approx(50.0)
    assert models[2].info().time_yr == pytest.approx(50.0)


def test_batch_refuses_a_repeated_handle():
    mb = members()[0]
    m = make(mb, 0)
    with pytest.raises(vlib.VilmaError, match="appears twice"):
        vlib.update_batch([m, m], [mb.ice_at(300)] * 2, 50.0)
