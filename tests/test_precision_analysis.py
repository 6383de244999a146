"""Why the mixed-precision path forms the pair offset, distance and overlap in FP64 and only the
force arithmetic in FP32 (CPU, numpy emulation of both forms of the pair geometry).

The alternative -- positions stored as FP32 offsets from their cell's origin, the pair offset
(c_i - c_j) h + (o_i - o_j) and everything after it in FP32 -- rounds the centre distance to the
FP32 spacing of the cell size (h ~ 2.5 mm: about 2e-10 m).  The Hertz force depends on the
overlap r_i + r_j - |x_ij| to the power 1.5, so a distance error e becomes a force error of
1.5 e / overlap: in the emulation below, the 99th percentile of the relative force error is
1.8e-3 at 0.3 um of overlap, 1.3e-4 at 3 um, 1.2e-5 at 30 um, against 1e-5.  The workloads' contacts
are mostly that small (the 200k-disk dam break: overlaps of 0.1-30 um; the 2M lattice's
contacts: grazing).  With the offset formed in FP64 from the FP64 positions and then rounded
to FP32, the distance error is 2^-24 of the distance itself, and the overlap r_i + r_j - |x_ij|
is still formed in FP64: the force error is FP32 rounding of the force arithmetic alone."""
import numpy as np

TOL = 1e-5


def _contacts(rng, n, overlaps, h=2.5e-3):
    """n sphere pairs with radii U[0.8, 1.2] mm at the given overlaps, random directions, centres
    at random places in a 0.27 m box, each on its cell grid of size h."""
    ri = rng.uniform(0.8e-3, 1.2e-3, n)
    rj = rng.uniform(0.8e-3, 1.2e-3, n)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    xi = rng.uniform(0.0, 0.27, size=(n, 3))
    xj = xi - v * (ri + rj - overlaps)[:, None]
    return xi, xj, ri, rj, h


def _force64(xi, xj, ri, rj):
    d = xi - xj
    ov = ri + rj - np.sqrt((d * d).sum(axis=1))
    return ov * np.sqrt(ov)          # kn cancels in a relative error


def _force_cell32(xi, xj, ri, rj, h):
    ci, cj = np.floor(xi / h), np.floor(xj / h)
    oi = (xi - ci * h).astype(np.float32)
    oj = (xj - cj * h).astype(np.float32)
    d = (ci - cj).astype(np.float32) * np.float32(h) + (oi - oj)
    dist = np.sqrt((d * d).sum(axis=1, dtype=np.float32), dtype=np.float32)
    ov = (ri.astype(np.float32) + rj.astype(np.float32)) - dist
    ov = np.maximum(ov, np.float32(0))
    return (ov * np.sqrt(ov)).astype(np.float64)


def _force_offset64(xi, xj, ri, rj):
    # this build: offset, distance and overlap in FP64, the force arithmetic in FP32
    d = xi - xj
    ov = (ri + rj - np.sqrt((d * d).sum(axis=1))).astype(np.float32)
    return (ov * np.sqrt(ov)).astype(np.float64)


def test_fp32_cell_relative_offsets_miss_the_force_bound_for_small_overlaps():
    rng = np.random.default_rng(1)
    for ov_um, expect_fail in ((0.3, True), (3.0, True), (30.0, False)):
        ov = np.full(20000, ov_um * 1e-6)
        xi, xj, ri, rj, h = _contacts(rng, len(ov), ov)
        f64 = _force64(xi, xj, ri, rj)
        e_cell = np.abs(_force_cell32(xi, xj, ri, rj, h) - f64) / f64
        e_ours = np.abs(_force_offset64(xi, xj, ri, rj) - f64) / f64
        assert e_ours.max() <= TOL, (ov_um, e_ours.max())
        if expect_fail:     # one contact in a hundred is off by ten times the bound or more
            assert np.quantile(e_cell, 0.99) > 10 * TOL, (ov_um, np.quantile(e_cell, 0.99))
        else:
            assert np.quantile(e_cell, 0.99) < 10 * TOL, (ov_um, np.quantile(e_cell, 0.99))
