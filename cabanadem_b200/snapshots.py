"""Particle snapshots written by the C++ interface's Particles::output (particles_<k>.csv, or
particles_<k>.xmf with its particles_<k>.bin).

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


def files(folder: str, ext: str = ".csv") -> list[str]:
    """particles_<k><ext> in `folder` (".csv" or ".xmf"), sorted by k (automate.py:64-80 does
    the same for .h5)."""
    pat = re.compile(r"^particles_(\d+)" + re.escape(ext) + "$")
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


_XDMF_TYPES = {("Float", "8"): "<f8", ("Float", "4"): "<f4", ("Int", "4"): "<i4", ("Int", "8"): "<i8"}


def read_xdmf(path: str) -> dict:
    """One XDMF snapshot (Particles::output with the "xdmf" format: a Polyvertex grid whose
    Format="Binary" data items point into particles_<k>.bin) -> the same dictionary as read()."""
    import xml.etree.ElementTree as ET
    grid = ET.parse(path).getroot().find("Domain/Grid")
    if grid is None:
        raise ValueError("%s: no Domain/Grid" % path)
    folder = os.path.dirname(path)

    def load(item):
        if item.get("Format") != "Binary" or item.get("Endian", "Little") != "Little":
            raise ValueError("%s: only little-endian Binary data items are read" % path)
        dims = [int(d) for d in item.get("Dimensions").split()]
        dt = np.dtype(_XDMF_TYPES[(item.get("NumberType", "Float"), item.get("Precision", "4"))])
        count = int(np.prod(dims))
        a = np.fromfile(os.path.join(folder, item.text.strip()), dtype=dt, count=count,
                        offset=int(item.get("Seek", "0")))
        if a.size != count:
            raise ValueError("%s: %s holds fewer than %d values" % (path, item.text.strip(), count))
        return a.reshape(dims).astype(dt.newbyteorder("="))

    out = {"time": float(grid.find("Time").get("Value")), "positions": load(grid.find("Geometry/DataItem"))}
    for att in grid.findall("Attribute"):
        out[att.get("Name")] = load(att.find("DataItem"))
    missing = [k for k in _VEC + _SCALAR if k not in out]
    if missing:
        raise ValueError("%s: missing datasets %s" % (path, missing))
    return out
