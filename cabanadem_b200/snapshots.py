"""Particle snapshots as the C++ interface's Particles::output writes them (particles_<k>.csv,
or particles_<k>.xmf with its particles_<k>.bin): readers, and writers of the same files for
Python callers (a ParticleState, e.g. from api.Particles.download()).

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


# dataset name (the reference's slice label) -> ParticleState field
_FIELDS = (("positions", "x"), ("velocities", "u"), ("omega", "omega"), ("forces", "force"), ("mass", "m"),
           ("density", "rho"), ("radius", "rad"), ("total_no_tangential_contacts", "tng_count"))


def write_csv(folder: str, step: int, time: float, state) -> str:
    """particles_<step>.csv of a ParticleState, byte for byte as Particles::output writes it
    (every double with 17 significant digits, so read() gives back the same bits)."""
    path = os.path.join(folder, "particles_%d.csv" % step)
    cols = [getattr(state, f) for _, f in _FIELDS]
    with open(path, "w") as fh:
        fh.write("# time %.17g\n" % time)
        fh.write("id," + ",".join("%s_%d" % (n, d) for n in _VEC for d in range(3)) + "," + ",".join(_SCALAR) + "\n")
        for i in range(state.n):
            vals = [("%.17g" % v) for c in cols[:4] for v in c[i]] + [("%.17g" % c[i]) for c in cols[4:7]]
            fh.write("%d,%s,%d\n" % (i, ",".join(vals), int(cols[7][i])))
    return path


def write_xdmf(folder: str, step: int, time: float, state) -> str:
    """particles_<step>.xmf and .bin of a ParticleState, byte for byte as the C++ interface's
    writeXdmfSnapshot writes them; returns the .xmf path."""
    stem = "particles_%d" % step
    n, seek, at = state.n, [], 0
    with open(os.path.join(folder, stem + ".bin"), "wb") as fb:
        for name, f in _FIELDS:
            a = np.ascontiguousarray(getattr(state, f), dtype="<i4" if name == _SCALAR[-1] else "<f8")
            seek.append(at)
            fb.write(a.tobytes())
            at += a.nbytes
    lines = ['<?xml version="1.0" ?>', '<!DOCTYPE Xdmf SYSTEM "Xdmf.dtd" []>', '<Xdmf Version="2.0">',
             '  <Domain>', '    <Grid Name="particles" GridType="Uniform">', '      <Time Value="%.17g"/>' % time,
             '      <Topology TopologyType="Polyvertex" NumberOfElements="%d" NodesPerElement="1"/>' % n]

    def item(k, name):
        vec, is_int = name in _VEC, name == _SCALAR[-1]
        return ('        <DataItem Dimensions="%d%s" NumberType="%s" Precision="%d" Format="Binary" Endian="Little" '
                'Seek="%d">%s.bin</DataItem>' % (n, " 3" if vec else "", "Int" if is_int else "Float",
                                                 4 if is_int else 8, seek[k], stem))
    lines += ['      <Geometry GeometryType="XYZ">', item(0, "positions"), '      </Geometry>']
    for k, (name, _) in enumerate(_FIELDS[1:], start=1):
        lines += ['      <Attribute Name="%s" AttributeType="%s" Center="Node">' % (name, "Vector" if name in _VEC
                                                                                       else "Scalar"),
                  item(k, name), '      </Attribute>']
    lines += ['    </Grid>', '  </Domain>', '</Xdmf>']
    path = os.path.join(folder, stem + ".xmf")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return path
