"""Particle snapshots written by the C++ interface's Particles::output (particles_<k>.csv).

The reference writes particles_<k>.h5 through Cabana's HDF5 writer with one dataset per
slice label and a Time attribute (src/CabanaDEM_Particles.hpp:299-326); no HDF5 library is
in this image, so each snapshot is a CSV file: a "# time <t>" line, a header of slice labels
with a component suffix (positions_0 ... total_no_tangential_contacts) and one row per
particle.  `read` returns the datasets under the reference's names with the reference's
shapes, so post-processing written against the HDF5 files (automate.py:133-135, :315, :447,
:531) indexes them the same way.
"""
from __future__ import annotations

import os
import re

import numpy as np

_VEC = ("positions", "velocities", "omega", "forces")
_SCALAR = ("mass", "density", "radius", "total_no_tangential_contacts")


def files(folder: str) -> list[str]:
    """particles_<k>.csv in `folder`, sorted by k (automate.py:64-80 does the same for .h5)."""
    pat = re.compile(r"^particles_(\d+)\.csv$")
    found = [(int(m.group(1)), f) for f in os.listdir(folder) if (m := pat.match(f))]
    return [os.path.join(folder, f) for _, f in sorted(found)]


def read(path: str) -> dict:
    """One snapshot -> {"time": t, "positions": (n, 3), ..., "total_no_tangential_contacts": (n,)}."""
    with open(path) as fh:
        first = fh.readline().split()
        if len(first) != 3 or first[:2] != ["#", "time"]:
            raise ValueError("%s: not a particle snapshot" % path)
        head = fh.readline().strip().split(",")
    data = np.loadtxt(path, delimiter=",", skiprows=2, ndmin=2)
    col = {h: i for i, h in enumerate(head)}
    out = {"time": float(first[2])}
    for name in _VEC:
        out[name] = data[:, [col["%s_%d" % (name, d)] for d in range(3)]].copy()
    for name in _SCALAR:
        out[name] = data[:, col[name]].copy()
    out["total_no_tangential_contacts"] = out["total_no_tangential_contacts"].astype(np.int32)
    return out
