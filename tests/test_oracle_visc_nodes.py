"""Lateral viscosity from absolute nodal log10 viscosities
(response_enable_lateral_visc_from_nodes, src/vilma_response.f90:1120-1169) in
the oracle: the conversion equals its plain restatement here (element =
log10-mean of its two nodes, capped above lid_log10max inside the lid,
minus log10 of the radial viscosity; elastic and fluid elements untouched),
checked through identical model updates."""
import numpy as np

from fastearth3d_b200 import synth
from fastearth3d_b200.abi import VG_RHEOL_MAXWELL
from oracle import orc


def node_field(w, o, rng):
    r, lay = o.mesh()
    ng = w.nlat * w.nphi
    base = np.log10(np.array([o.p.eta[k] if o.p.rheology[k] == VG_RHEOL_MAXWELL else 1e23 for k in range(4)]))
    node_lay = np.concatenate([lay, [lay[-1]]])
    return base[node_lay][:, None] + 0.5 * rng.standard_normal((len(r), ng)), r, lay


def restated_pert(o, vn, r, lay, lid_depth, lid_max, cap):
    ne = len(lay)
    pert = np.zeros((ne, vn.shape[1]))
    r_lid = r[-1] - lid_depth if lid_depth > 0 else np.inf
    for e in range(ne):
        L = lay[e]
        if o.p.rheology[L] != VG_RHEOL_MAXWELL:
            continue
        v = 0.5 * (vn[e] + vn[e + 1])
        if r[e] >= r_lid - 1e-6 * r[-1]:
            v = np.where(v > lid_max, cap, v)
        pert[e] = v - np.log10(o.p.eta[L])
    return pert


def test_from_nodes_equals_restatement():
    w = synth.Workload("n", 12, 16, 100.0, 2, 2, "sawtooth", sle=True, visc3d=True, seed=6)
    rng = np.random.default_rng(4)
    zb, hi = w.reference()
    for lid in ((0.0, 0.0, 0.0), (400e3, 21.0, 24.0)):
        a, b = orc.Oracle(w.params(orc.default_params)), orc.Oracle(w.params(orc.default_params))
        vn, r, lay = node_field(w, a, rng)
        for m in (a, b):
            m.set_reference(zb, hi)
        a.enable_visc3d_from_nodes(vn.reshape(-1), *lid)
        b.enable_visc3d(restated_pert(b, vn, r, lay, *lid).reshape(-1))
        assert a.info().ne3d == b.info().ne3d > 0
        for step in (1, 2):
            for m in (a, b):
                m.update(w.ice_at(step * 300), w.dt_yr)
        assert np.array_equal(a.fields()[0], b.fields()[0])
