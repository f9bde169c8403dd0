"""The oracle's results do not depend on its OpenMP thread count (its
parallel loops run over independent degrees, slots and 3-D elements, and
every reduction is taken in a fixed order), so the parity tests and the CPU
baseline mean the same thing on hosts with different core counts: three
coupled updates of a small 3-D sea-level model on 1 and on 8 threads agree
bit for bit in rsl, z_bed, the ocean function and the memory state."""
import os

import numpy as np

from fastearth3d_b200 import synth
from oracle import orc


def run(threads):
    orc.set_threads(threads)
    w = synth.Workload("threads", 32, 40, 50.0, 1000, 4, "sawtooth", sle=True, visc3d=True, seed=9)
    o = orc.Oracle(w.params(orc.default_params))
    o.set_reference(*w.reference())
    o.enable_visc3d(w.pert(o.p))
    for s in (100, 101, 102):
        o.update(w.ice_at(s), w.dt_yr)
    return o.fields()[:3], o.state()[0]


def test_oracle_is_thread_count_independent():
    try:
        f1, s1 = run(1)
        f8, s8 = run(8)
    finally:
        orc.set_threads(os.cpu_count() or 1)
    for a, b in zip(f1, f8):
        assert np.array_equal(a, b)
    for a, b in zip(s1, s8):
        assert np.array_equal(a, b)
