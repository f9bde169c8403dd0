"""vg_enable_visc3d_from_nodes (response_enable_lateral_visc_from_nodes,
src/vilma_response.f90:1120-1169) on the GPU: the same model updates as the
oracle's from-nodes path (1e-10) and, bit for bit, as vg_enable_visc3d with
the perturbation restated in tests/test_oracle_visc_nodes.py; with and
without the lithosphere-lid rule."""
import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth
from oracle import orc

from test_oracle_visc_nodes import node_field, restated_pert

pytestmark = pytest.mark.gpu


def test_from_nodes_parity():
    w = synth.Workload("n", 12, 16, 100.0, 2, 2, "sawtooth", sle=True, visc3d=True, seed=6)
    rng = np.random.default_rng(4)
    zb, hi = w.reference()
    for lid in ((0.0, 0.0, 0.0), (400e3, 21.0, 24.0)):
        o = orc.Oracle(w.params(orc.default_params))
        g, g2 = vlib.Model(w.params(vlib.default_params)), vlib.Model(w.params(vlib.default_params))
        vn, r, lay = node_field(w, o, rng)
        for m in (o, g, g2):
            m.set_reference(zb, hi)
        o.enable_visc3d_from_nodes(vn.reshape(-1), *lid)
        g.enable_visc3d_from_nodes(vn.reshape(-1), *lid)
        g2.enable_visc3d(restated_pert(o, vn, r, lay, *lid).reshape(-1))
        for step in (1, 2):
            for m in (o, g, g2):
                m.update(w.ice_at(step * 300), w.dt_yr)
        rg, ro = g.fields()[0], o.fields()[0]
        assert np.abs(rg - ro).max() <= 1e-10 * np.abs(ro).max()
        assert np.array_equal(rg, g2.fields()[0])
