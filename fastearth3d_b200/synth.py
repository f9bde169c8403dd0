"""Seeded synthetic inputs standing in for the benchmark workloads.

The reference quotes its performance on real-data runs (GLAC-1D ice, RTopo
bathymetry, Bagge-2021 3-D viscosity); no dataset is named for these
workloads and none is available offline, so seeded fields with the stated
shapes, sizes and value distributions are used:

* Earth: 4-layer incompressible Maxwell sphere, 6371 km; elastic lithosphere
  70 km (rho 3300, mu 0.7e11); upper mantle to 670 km (rho 3450, mu 0.9e11,
  eta 5e20); lower mantle (rho 4900, mu 2.0e11, eta 2e21); fluid core below
  3480 km (rho 10900).
* Ice: N Gaussian caps, centres uniform on the sphere, half-width at half
  maximum U(5, 15) deg, peak U(1000, 3000) m, profile H exp(-ln2 (d/w)^2).
* Topography: random spherical-harmonic field with coefficient variance
  proportional to l^-2 (l >= 1), rescaled to std 2500 m and mean -1500 m.
* 3-D viscosity: log10 perturbation = random SH field (lmax 32, l^-2), std 0.4,
  clipped to +/- 1 dex, the same lateral pattern in every Maxwell element.
"""
import numpy as np

from .abi import VG_RHEOL_ELASTIC, VG_RHEOL_FLUID, VG_RHEOL_MAXWELL, set_layers

SEC_PER_YEAR = 31556926.0

EARTH4 = [
    (6301.0e3, 6371.0e3, 3300.0, 0.7e11, 1e300, VG_RHEOL_ELASTIC),
    (5701.0e3, 6301.0e3, 3450.0, 0.9e11, 5e20, VG_RHEOL_MAXWELL),
    (3480.0e3, 5701.0e3, 4900.0, 2.0e11, 2e21, VG_RHEOL_MAXWELL),
    (0.0, 3480.0e3, 10900.0, 0.0, 0.0, VG_RHEOL_FLUID),
]
# element counts the reference depth rule gives this earth (5/10/40 km targets)
NATIVE_COUNTS = [14, 60, 56, 87]


def element_counts(n_total):
    """Split n_total radial elements over the 4 layers in proportion to the
    reference-native counts (largest remainder)."""
    tot = sum(NATIVE_COUNTS)
    raw = [n_total * c / tot for c in NATIVE_COUNTS]
    out = [int(np.floor(x)) for x in raw]
    rem = sorted(range(4), key=lambda i: -(raw[i] - out[i]))
    for i in rem[: n_total - sum(out)]:
        out[i] += 1
    return out


def gauss_grid(nlat, nphi):
    x, w = np.polynomial.legendre.leggauss(nlat)
    order = np.argsort(-x)  # north first
    x, w = x[order], w[order]
    colat = np.arccos(x)
    lon = 2 * np.pi * np.arange(nphi) / nphi
    return colat, lon, w


def lmidx(lmax, l, m):
    return m * (lmax + 1) - m * (m - 1) // 2 + (l - m)


def alf_table(lmax, x):
    """Orthonormal associated Legendre functions (no Condon-Shortley phase),
    shape (nlm, nlat), m-major order."""
    nlm = (lmax + 1) * (lmax + 2) // 2
    P = np.zeros((nlm, x.size))
    st = np.sqrt((1 - x) * (1 + x))
    pmm = np.full(x.size, 1 / np.sqrt(4 * np.pi))
    for m in range(lmax + 1):
        if m > 0:
            pmm = pmm * np.sqrt((2 * m + 1) / (2 * m)) * st
        p2, p1 = np.zeros_like(x), pmm.copy()
        P[lmidx(lmax, m, m)] = pmm
        for l in range(m + 1, lmax + 1):
            a = np.sqrt((4 * l * l - 1) / (l * l - m * m))
            b = np.sqrt(((l - 1) ** 2 - m * m) / (4 * (l - 1) ** 2 - 1))
            p = a * (x * p1 - b * p2)
            P[lmidx(lmax, l, m)] = p
            p2, p1 = p1, p
    return P


def synthesize(q, lmax, nlat, nphi):
    """Real field on the Gauss grid (nlat, nphi) from m-major coefficients q."""
    colat, lon, _ = gauss_grid(nlat, nphi)
    P = alf_table(lmax, np.cos(colat))
    f = np.zeros((nlat, nphi))
    for m in range(lmax + 1):
        i0 = lmidx(lmax, m, m)
        G = q[i0 : i0 + lmax + 1 - m] @ P[i0 : i0 + lmax + 1 - m]  # (nlat,)
        fac = 1.0 if m == 0 else 2.0
        f += fac * (np.outer(G.real, np.cos(m * lon)) - np.outer(G.imag, np.sin(m * lon)))
    return f


def random_sh_field(seed, lmax_field, lmax, nlat, nphi, std, mean):
    rng = np.random.default_rng(seed)
    nlm = (lmax + 1) * (lmax + 2) // 2
    q = np.zeros(nlm, complex)
    lmax_field = min(lmax_field, lmax)
    for m in range(lmax_field + 1):
        for l in range(max(m, 1), lmax_field + 1):
            s = l ** -1.0  # amplitude ~ l^-1 -> variance ~ l^-2
            q[lmidx(lmax, l, m)] = s * (rng.standard_normal() + (1j * rng.standard_normal() if m > 0 else 0))
    f = synthesize(q, lmax, nlat, nphi)
    f = (f - f.mean()) / f.std()
    return std * f + mean


def ice_caps(seed, n_caps, nlat, nphi):
    rng = np.random.default_rng(seed)
    colat, lon, _ = gauss_grid(nlat, nphi)
    th, ph = np.meshgrid(colat, lon, indexing="ij")
    ice = np.zeros((nlat, nphi))
    for _ in range(n_caps):
        z = rng.uniform(-1, 1)
        phc = rng.uniform(0, 2 * np.pi)
        thc = np.arccos(z)
        w = np.deg2rad(rng.uniform(5, 15))
        H = rng.uniform(1000, 3000)
        cosd = np.cos(th) * np.cos(thc) + np.sin(th) * np.sin(thc) * np.cos(ph - phc)
        d = np.arccos(np.clip(cosd, -1, 1))
        ice += H * np.exp(-np.log(2) * (d / w) ** 2)
    return ice


def ramp(t_yr, t_ramp=20000.0):
    return np.clip(t_yr / t_ramp, 0.0, 1.0)


def sawtooth(t_yr, period=100000.0, grow=90000.0):
    tau = np.mod(t_yr, period)
    return np.where(tau < grow, tau / grow, 1.0 - (tau - grow) / (period - grow))


class Workload:
    """One benchmark configuration: params, reference fields, ice history."""

    def __init__(self, name, lmax, n_elem, dt_yr, n_steps, n_caps, history, sle, visc3d, seed=1234, rotation=False):
        self.name, self.lmax, self.n_elem = name, lmax, n_elem
        self.rotation = rotation
        self.nlat, self.nphi = lmax + 1, 2 * (lmax + 1)
        self.dt_yr, self.n_steps, self.history, self.sle, self.visc3d = dt_yr, n_steps, history, sle, visc3d
        self.seed = seed
        self.ice_full = ice_caps(seed, n_caps, self.nlat, self.nphi)
        if sle:
            self.topo = random_sh_field(seed + 1, lmax, lmax, self.nlat, self.nphi, 2500.0, -1500.0)
        else:
            # no ocean anywhere: the sea-level equation exits at C_int <= 0
            self.topo = np.full((self.nlat, self.nphi), 1000.0)
        self.pert2d = None
        if visc3d:
            f = random_sh_field(seed + 2, 32, lmax, self.nlat, self.nphi, 0.4, 0.0)
            self.pert2d = np.clip(f, -1.0, 1.0)

    def params(self, default_params):
        p = default_params()
        p.lmax, p.nlat, p.nphi = self.lmax, self.nlat, self.nphi
        set_layers(p, EARTH4)
        for i, c in enumerate(element_counts(self.n_elem)):
            p.ne_layer[i] = c
        p.rotation = 1 if self.rotation else 0
        return p

    def ice_at(self, step):
        t = step * self.dt_yr
        f = ramp(t) if self.history == "ramp" else sawtooth(t)
        return np.ascontiguousarray((self.ice_full * f).reshape(-1))

    def reference(self):
        zb = np.ascontiguousarray(self.topo.reshape(-1))
        return zb, np.zeros(self.nlat * self.nphi)

    def pert(self, p):
        """(ne, nlat, nphi) log10-viscosity perturbation for the params `p`
        (explicit per-layer element counts): the lateral pattern in every
        Maxwell element, zero elsewhere. Elements run bottom-up, layers are
        surface-first."""
        elem_layers = []
        for i in range(p.n_layer - 1, -1, -1):
            elem_layers += [i] * p.ne_layer[i]
        out = np.zeros((len(elem_layers), self.nlat, self.nphi))
        for e, L in enumerate(elem_layers):
            if p.rheology[L] == VG_RHEOL_MAXWELL:
                out[e] = self.pert2d
        return out


class EnsembleMember(Workload):
    """One instance of the batched ensemble: its own lmax, lithosphere
    thickness and mantle viscosities on the 4-layer earth above (radii,
    densities and shear moduli kept), seeded ice and topography, and, for
    half the instances, the lateral viscosity field of the 3-D workload."""

    def __init__(self, name, lmax, n_elem, litho_km, eta_um, eta_lm, visc3d, seed):
        self.litho_km, self.eta_um, self.eta_lm = litho_km, eta_um, eta_lm
        super().__init__(name, lmax, n_elem, 50.0, 2000, 6, "sawtooth", sle=True, visc3d=visc3d, seed=seed)

    def layers(self):
        rl = 6371.0e3 - self.litho_km * 1e3
        (_, _, r0, m0, e0, h0), (_, _, r1, m1, _, h1), (_, _, r2, m2, _, h2), core = EARTH4
        return [(rl, 6371.0e3, r0, m0, e0, h0), (5701.0e3, rl, r1, m1, self.eta_um, h1),
                (3480.0e3, 5701.0e3, r2, m2, self.eta_lm, h2), core]

    def params(self, default_params):
        p = super().params(default_params)
        set_layers(p, self.layers())
        return p


def ensemble(n=32, seed=2024):
    """The batched-ensemble workload: n instances, lmax drawn from
    {64, 96, 128, 192, 256}, upper-mantle eta log-uniform in [1e20, 1e21] Pa s,
    lower-mantle eta log-uniform in [1e21, 1e23] Pa s, lithosphere 50-120 km,
    every other instance with 3-D viscosity; 60, 80 and 100 radial elements
    for lmax 64, 96 and >= 128."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        lmax = int(rng.choice([64, 96, 128, 192, 256]))
        n_elem = {64: 60, 96: 80}.get(lmax, 100)
        out.append(EnsembleMember(f"e{i}_l{lmax}", lmax, n_elem, float(rng.uniform(50.0, 120.0)),
                                  float(10 ** rng.uniform(20.0, 21.0)), float(10 ** rng.uniform(21.0, 23.0)),
                                  i % 2 == 0, seed + 17 * i))
    return out


def workloads():
    return {
        "c1_1d_l64": Workload("c1_1d_l64", 64, 60, 50.0, 400, 3, "ramp", sle=False, visc3d=False),
        "c2_1d_sle_l128": Workload("c2_1d_sle_l128", 128, 100, 100.0, 1000, 6, "sawtooth", sle=True, visc3d=False,
                                   rotation=True),
        "c3_3d_l128": Workload("c3_3d_l128", 128, 100, 50.0, 2000, 6, "sawtooth", sle=True, visc3d=True),
    }
