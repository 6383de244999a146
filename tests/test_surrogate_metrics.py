"""The observables the surrogate is judged by (cabanadem_b200/surrogate.py), on inputs with
known answers (CPU): the runout front of a block, the deposit depth and height of a hexagonal
disk packing, and the acceleration scale of a uniformly accelerating trajectory."""
import math

import numpy as np
import torch

from cabanadem_b200 import surrogate as SG


def _hex_block(ncol=40, nrow=20, r=1e-3):
    """Touching disks of radius r on a hexagonal lattice: ncol per row, nrow rows, x >= 0,
    y >= 0; packing fraction pi / (2 sqrt 3)."""
    pts = [((2 * i + (j % 2)) * r + r, j * math.sqrt(3.0) * r + r) for j in range(nrow) for i in range(ncol)]
    x = np.zeros((len(pts), 3))
    x[:, :2] = pts
    return x, np.full(len(pts), r)


def test_runout_front_is_the_far_edge():
    x, _ = _hex_block(ncol=100, nrow=20)                 # 2,000 disks, x up to 0.2 m
    assert abs(SG.runout_front(x, q=1.0) - x[:, 0].max()) < 1e-15
    x_out = np.vstack([x, [[1.0, 0.0, 0.0]]])           # one stray particle far downstream
    assert SG.runout_front(x_out) <= x[:, 0].max()       # the 0.999 quantile of 2,001 ignores it


def test_depth_and_height_of_a_hex_block():
    r, ncol, nrow = 1e-3, 40, 20
    x, rad = _hex_block(ncol, nrow, r)
    width = (2 * ncol + 1) * r
    top = (nrow - 1) * math.sqrt(3.0) * r + 2 * r
    bins = 20
    depth = SG.depth_profile(x, rad, width, bins=bins)
    inner = depth[2:-2]
    # mass / (column width x 0.85): the hexagonal packing fraction over 0.85, times the height
    expect = (math.pi / (2 * math.sqrt(3.0))) / 0.85 * (nrow * math.sqrt(3.0) * r)
    assert np.all(np.abs(inner / expect - 1.0) < 0.06), inner / expect
    h = SG.pile_profile(x, rad, width, bins=bins)
    assert np.allclose(h[1:-1], top, rtol=0, atol=1e-12)


def test_sigma_a_of_uniform_acceleration():
    """Frames of x = a k^2 / 2 (k the frame): every second difference is a, so the RMS is |a|
    over the in-plane components (z is not used)."""
    k = torch.arange(6, dtype=torch.float64)[:, None, None]
    a = torch.tensor([3e-6, -4e-6, 9.0], dtype=torch.float64)
    traj = (0.5 * a * k * k).expand(6, 10, 3).contiguous()
    got = SG.sigma_a_of([(traj, torch.ones(10))])
    assert abs(got - math.sqrt((3e-6 ** 2 + 4e-6 ** 2) / 2.0)) < 1e-18
