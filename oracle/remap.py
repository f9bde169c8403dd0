"""CPU ORACLE — test infrastructure only (see orc.hpp).

Host lon-lat <-> Gauss-grid remap of the coupling layer (src/vilma_remap.f90:
56-166, used by src/vilma_coupling.f90:172-176, 355-359, 436-447, 631-641),
restated with dense per-axis overlap tables at small sizes:

* remap_init (:56-99): cell boundaries from axis midpoints for both grids (the
  outermost ones half a spacing beyond the last centre; latitudes clamped to
  +/-90), the Gauss grid taken south first. The weights come from the
  fesm-utils `coords` library (map_init method "con" and "bilinear", not
  present in the reference tree); this restates their published meaning:
  first-order conservative weights = the spherical area of each source /
  target cell overlap, and bilinear interpolation between the four
  surrounding target nodes.
* remap_to_gauss (:101-136): stat "mean" (the overlap-area-weighted mean of
  the source cells), rows flipped to north first, then the optional global
  rescale so the Gauss quadrature integral equals the source area integral
  (sum f area / sum area * 4 pi).
* remap_to_ll (:138-164): bilinear from the Gauss grid; poleward of the
  outermost Gauss row the outermost row is used.

The overlap of two lon-lat rectangles on the unit sphere is
(lon overlap, radians) x (sin lat_top - sin lat_bot overlap), with the
longitude intervals compared modulo 360 degrees; the full cell-pair matrix is
the Kronecker product of the two per-axis tables.
"""
import numpy as np
from scipy import sparse


def bounds(x, lo=None, hi=None):
    """Cell boundaries from the axis midpoints, the ends half a spacing out."""
    x = np.asarray(x, dtype=np.float64)
    b = np.empty(len(x) + 1)
    b[1:-1] = 0.5 * (x[1:] + x[:-1])
    b[0] = x[0] - 0.5 * (x[1] - x[0])
    b[-1] = x[-1] + 0.5 * (x[-1] - x[-2])
    if lo is not None:
        b = np.clip(b, lo, hi)
    return b


def lon_overlap(a0, a1, b0, b1):
    """Length (degrees) of [a0, a1) intersect [b0, b1) on the circle."""
    tot = 0.0
    for k in (-2, -1, 0, 1, 2):
        lo = max(a0, b0 + 360.0 * k)
        hi = min(a1, b1 + 360.0 * k)
        if hi > lo:
            tot += hi - lo
    return tot


class Remap:
    def __init__(self, lon_src, lat_src, colat_gauss, nphi):
        self.lon_s = np.asarray(lon_src, dtype=np.float64)
        self.lat_s = np.asarray(lat_src, dtype=np.float64)
        self.nlon, self.nlat_s = len(self.lon_s), len(self.lat_s)
        self.nphi, self.nlat = nphi, len(colat_gauss)
        self.lat_g = 90.0 - np.degrees(np.asarray(colat_gauss))[::-1]  # south first
        self.lon_g = 360.0 * np.arange(nphi) / nphi
        lb_s, pb_s = bounds(self.lon_s), bounds(self.lat_s, -90.0, 90.0)
        lb_g, pb_g = bounds(self.lon_g), bounds(self.lat_g, -90.0, 90.0)
        ss, sg = np.sin(np.radians(pb_s)), np.sin(np.radians(pb_g))
        # source cell areas (steradians)
        self.area_s = np.outer(ss[1:] - ss[:-1], np.radians(lb_s[1:] - lb_s[:-1]))
        # overlap areas A[target (j asc, i), source (r, c)]: a lon-lat rectangle
        # overlap is its sin-latitude overlap times its longitude overlap
        Z = np.zeros((self.nlat, self.nlat_s))
        for j in range(self.nlat):
            for r in range(self.nlat_s):
                Z[j, r] = max(0.0, min(sg[j + 1], ss[r + 1]) - max(sg[j], ss[r]))
        L = np.zeros((self.nphi, self.nlon))
        for i in range(self.nphi):
            for c in range(self.nlon):
                L[i, c] = np.radians(lon_overlap(lb_g[i], lb_g[i + 1], lb_s[c], lb_s[c + 1]))
        self.A = sparse.csr_matrix(sparse.kron(sparse.csr_matrix(Z), sparse.csr_matrix(L)))

    def to_gauss(self, f_ll, wts, conserve_mass):
        """f_ll (nlat_s, nlon), south first -> (nlat, nphi), north first."""
        f = np.asarray(f_ll, dtype=np.float64).reshape(-1)
        cover = np.asarray(self.A.sum(axis=1)).reshape(-1)
        g = np.where(cover > 0.0, (self.A @ f) / np.where(cover > 0.0, cover, 1.0), 0.0)
        g = g.reshape(self.nlat, self.nphi)[::-1].copy()
        if conserve_mass:
            src = (np.asarray(f_ll) * self.area_s).sum() / self.area_s.sum() * 4.0 * np.pi
            gi = (2.0 * np.pi / self.nphi) * (g.sum(axis=1) * wts).sum()
            if abs(gi) > np.finfo(float).tiny:
                g = g * (src / gi)
        return g

    def to_ll(self, f_gauss):
        """f_gauss (nlat, nphi), north first -> (nlat_s, nlon), south first."""
        g = np.asarray(f_gauss, dtype=np.float64)[::-1]  # south first
        out = np.zeros((self.nlat_s, self.nlon))
        for r in range(self.nlat_s):
            y = self.lat_s[r]
            if y <= self.lat_g[0]:
                j0, j1, a = 0, 0, 0.0
            elif y >= self.lat_g[-1]:
                j0, j1, a = self.nlat - 1, self.nlat - 1, 0.0
            else:
                j0 = int(np.searchsorted(self.lat_g, y, side="right")) - 1
                j1 = j0 + 1
                a = (y - self.lat_g[j0]) / (self.lat_g[j1] - self.lat_g[j0])
            for c in range(self.nlon):
                x = self.lon_s[c] % 360.0
                dlon = 360.0 / self.nphi
                i0 = int(np.floor(x / dlon)) % self.nphi
                i1 = (i0 + 1) % self.nphi
                b = (x - i0 * dlon) / dlon
                out[r, c] = (1 - a) * ((1 - b) * g[j0, i0] + b * g[j0, i1]) + a * ((1 - b) * g[j1, i0] + b * g[j1, i1])
        return out
