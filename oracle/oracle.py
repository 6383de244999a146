"""ctypes wrapper of the CPU oracle (liboracle.so).  TEST INFRASTRUCTURE ONLY.

Used by tests/, the smoke check and bench.py's CPU-baseline leg as the checker; the
product (cabanadem_b200) never imports it.  The C++ functions it wraps cite the
reference file:line they restate (dem_oracle.cpp).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")

Q1_VELJ_USES_UI = 0x01
Q2_ETA_T_ZERO = 0x02
Q3_NO_PP_TORQUE = 0x04
Q4_UNIT_HISTORY = 0x08
Q5_WALL_FT_TYPO = 0x10
Q6_WALL_STATIC = 0x20
REF_COMPAT = 0x3F
POW_LIBM = 0
POW_SQRT = 1
BQ10_INDEX_BY_J = 0x01
BQ11_HARDCODED_K = 0x02
BQ1_VELJ_USES_UI = 0x04
BOND_REF_COMPAT = 0x07

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_up = C.POINTER(C.c_ubyte)


class _Particles(C.Structure):
    _fields_ = [("n", C.c_int), ("max_cnts", C.c_int), ("max_walls", C.c_int)] + \
               [(f, _dp) for f in ("x", "u", "omega", "force", "torque", "m", "rad", "I", "E", "nu", "G")] + \
               [("tng_idx", _ip), ("tng_ss_x", _dp), ("tng_ss_y", _dp), ("tng_ss_z", _dp),
                ("tng_count", _ip), ("tng_sw_x", _dp), ("tng_sw_y", _dp), ("tng_sw_z", _dp)]


class _Walls(C.Structure):
    _fields_ = [("n", C.c_int), ("x", _dp), ("normal", _dp), ("E", _dp), ("nu", _dp), ("G", _dp), ("u", _dp)]


class _ForceParams(C.Structure):
    _fields_ = [("cor_pp", C.c_double), ("cor_pw", C.c_double), ("mu_pp", C.c_double), ("mu_pw", C.c_double),
                ("quirks", C.c_uint), ("pow_mode", C.c_int)]


class _Mesh(C.Structure):
    _fields_ = [("nt", C.c_int), ("tri", _dp), ("E", C.c_double), ("nu", C.c_double), ("G", C.c_double),
                ("u", C.c_double * 3), ("D", C.c_double * 3), ("max_contacts", C.c_int), ("tid", _ip),
                ("th_x", _dp), ("th_y", _dp), ("th_z", _dp), ("cnt", _ip)]


class _Hooks(C.Structure):
    _fields_ = [("gravity", C.c_double * 3), ("ext_force", _dp), ("fix_flags", _up), ("mesh", C.POINTER(_Mesh))]


class _Bonds(C.Structure):
    _fields_ = [("n", C.c_int), ("max_bonds", C.c_int), ("idx", _ip), ("init_len", _dp), ("count", _ip)] + \
               [(f, _dp) for f in ("fn_x", "fn_y", "fn_z", "ft_x", "ft_y", "ft_z",
                                   "mn_x", "mn_y", "mn_z", "mt_x", "mt_y", "mt_z")] + [("broken", _up)]


class _BondParams(C.Structure):
    _fields_ = [("quirks", C.c_uint), ("beta", C.c_double), ("radius_factor", C.c_double), ("kn", C.c_double),
                ("kt", C.c_double), ("break_strain", C.c_double), ("pow_mode", C.c_int)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        L.orc_nlist_create.restype = C.c_void_p
        L.orc_nlist_destroy.argtypes = [C.c_void_p]
        L.orc_nlist_build.argtypes = [C.c_void_p, C.POINTER(_Particles), C.c_double, C.c_double]
        L.orc_nlist_total.restype = C.c_long
        L.orc_nlist_total.argtypes = [C.c_void_p]
        L.orc_nlist_copy.argtypes = [C.c_void_p, _ip, _ip]
        L.orc_run.argtypes = [C.POINTER(_Particles), C.POINTER(_Walls), C.POINTER(_ForceParams),
                              C.POINTER(_Hooks), C.c_double, C.c_int, C.c_double, C.c_double]
        L.orc_step.argtypes = [C.POINTER(_Particles), C.POINTER(_Walls), C.POINTER(_ForceParams),
                               C.POINTER(_Hooks), C.c_void_p, C.c_double, C.c_double, C.c_double]
        L.orc_force_pp.argtypes = [C.POINTER(_Particles), C.c_void_p, C.POINTER(_ForceParams), C.c_double]
        L.orc_force_wall.argtypes = [C.POINTER(_Particles), C.POINTER(_Walls), C.POINTER(_ForceParams), C.c_double]
        for f in ("orc_stage1", "orc_stage2", "orc_stage3"):
            getattr(L, f).argtypes = [C.POINTER(_Particles), C.c_double]
        L.orc_zero_force.argtypes = [C.POINTER(_Particles)]
        L.orc_update_tangential_contacts.argtypes = [C.POINTER(_Particles)]
        L.orc_kinetic_energy.restype = C.c_double
        L.orc_kinetic_energy.argtypes = [C.POINTER(_Particles)]
        L.orc_elastic_energy.restype = None
        L.orc_elastic_energy.argtypes = [C.POINTER(_Particles), C.POINTER(_Walls), C.POINTER(C.c_double)]
        L.orc_setup_bonds.argtypes = [C.POINTER(_Bonds), C.POINTER(_Particles), C.c_double, C.c_double]
        L.orc_bonded_force.argtypes = [C.POINTER(_Particles), C.POINTER(_Bonds), C.POINTER(_BondParams), C.c_double]
        L.orc_bonded_step.argtypes = [C.POINTER(_Particles), C.POINTER(_Bonds), C.POINTER(_BondParams),
                                      C.POINTER(_Hooks), C.c_double]
        _lib = L
    return _lib


def _ptr(a, t):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(t)


def _particles(s):
    for k, v in s.arrays().items():
        assert v.flags["C_CONTIGUOUS"], k
    p = _Particles()
    p.n, p.max_cnts, p.max_walls = s.n, s.max_cnts, s.tng_sw_x.shape[1]
    for f in ("x", "u", "omega", "force", "torque", "m", "rad", "I", "E", "nu", "G",
              "tng_ss_x", "tng_ss_y", "tng_ss_z", "tng_sw_x", "tng_sw_y", "tng_sw_z"):
        setattr(p, f, _ptr(getattr(s, f), _dp))
    p.tng_idx = _ptr(s.tng_idx, _ip)
    p.tng_count = _ptr(s.tng_count, _ip)
    return p


def _walls(w):
    c = _Walls()
    if w is None:
        c.n = 0
        return c
    c.n = w.n
    c.x, c.normal = _ptr(w.x, _dp), _ptr(w.normal, _dp)
    c.E, c.nu, c.G = _ptr(w.E, _dp), _ptr(w.nu, _dp), _ptr(w.G, _dp)
    c.u = _ptr(w.u, _dp)   # velocity: used with Q6 clear; x is then advanced in place
    return c


def _fp(params, pow_mode):
    return _ForceParams(params["cor_pp"], params["cor_pw"], params["mu_pp"], params["mu_pw"],
                        int(params.get("quirks", REF_COMPAT)), pow_mode)


class _HookHolder:
    def __init__(self, gravity=(0.0, 0.0, 0.0), ext_force=None, fix_flags=None, mesh=None):
        self.h = _Hooks()
        self.h.gravity = (C.c_double * 3)(*gravity)
        self._ext = None if ext_force is None else np.ascontiguousarray(ext_force, dtype=np.float64)
        self._fix = None if fix_flags is None else np.ascontiguousarray(fix_flags, dtype=np.uint8)
        self.h.ext_force = _ptr(self._ext, _dp) if self._ext is not None else None
        self.h.fix_flags = _ptr(self._fix, _up) if self._fix is not None else None
        self.mesh = mesh
        if mesh is not None:
            self._m = _Mesh()
            self._tri = np.ascontiguousarray(mesh.tri, dtype=np.float64)
            self._m.nt = mesh.nt
            self._m.tri = _ptr(self._tri, _dp)
            self._m.E, self._m.nu, self._m.G = mesh.E, mesh.nu, mesh.G
            self._m.u = (C.c_double * 3)(*mesh.u)
            self._m.D = (C.c_double * 3)(*mesh.D)
            self._m.max_contacts = mesh.max_contacts
            self._m.tid = _ptr(mesh.tid, _ip)
            self._m.th_x, self._m.th_y, self._m.th_z = _ptr(mesh.th_x, _dp), _ptr(mesh.th_y, _dp), _ptr(mesh.th_z, _dp)
            self._m.cnt = _ptr(mesh.cnt, _ip)
            self.h.mesh = C.pointer(self._m)

    def done(self):
        """Copy the mesh translation back into the MeshState (the arrays are shared)."""
        if self.mesh is not None:
            self.mesh.D[:] = list(self._m.D)


def run(state, walls, params, dt, nsteps, delta=0.0, skin=0.0, gravity=(0.0, 0.0, 0.0), ext_force=None,
        fix_flags=None, pow_mode=POW_LIBM, mesh=None):
    """Advance `state` in place by nsteps reference steps (Solver.hpp:81-94).
    Neighbour cutoff is `delta` when > 0, else rad_i + rad_j + skin; rebuilt every step.
    `mesh` (a MeshState) adds a triangle-mesh wall after the plane walls; its contact
    history and translation are updated in place."""
    p, w, fp = _particles(state), _walls(walls), _fp(params, pow_mode)
    h = _HookHolder(gravity, ext_force, fix_flags, mesh)
    st = lib().orc_run(C.byref(p), C.byref(w), C.byref(fp), C.byref(h.h), dt, int(nsteps), float(delta), float(skin))
    h.done()
    return st


def neighbor_list(state, delta=0.0, skin=0.0):
    L = lib()
    nl = L.orc_nlist_create()
    try:
        p = _particles(state)
        L.orc_nlist_build(nl, C.byref(p), float(delta), float(skin))
        tot = L.orc_nlist_total(nl)
        off = np.zeros(state.n + 1, dtype=np.int32)
        idx = np.zeros(max(tot, 1), dtype=np.int32)
        L.orc_nlist_copy(nl, _ptr(off, _ip), _ptr(idx, _ip))
        return off, idx[:tot]
    finally:
        L.orc_nlist_destroy(nl)


def kinetic_energy(state):
    p = _particles(state)
    return lib().orc_kinetic_energy(C.byref(p))


def elastic_energy(state, walls):
    """Hertz elastic energy (pairs, walls) of a state: 2/5 kn overlap^2.5 per overlap."""
    p = _particles(state)
    w = _walls(walls)
    out = (C.c_double * 2)()
    lib().orc_elastic_energy(C.byref(p), C.byref(w), out)
    return float(out[0]), float(out[1])


def _bonds(b):
    c = _Bonds()
    c.n, c.max_bonds = b.n, b.max_bonds
    c.idx, c.init_len, c.count = _ptr(b.idx, _ip), _ptr(b.init_len, _dp), _ptr(b.count, _ip)
    for k, v in b.hist.items():
        setattr(c, k, _ptr(v, _dp))
    c.broken = _ptr(b.broken, _up)
    return c


def _bp(bparams, pow_mode=POW_LIBM):
    return _BondParams(int(bparams.get("quirks", BOND_REF_COMPAT)), float(bparams.get("beta", 0.1)),
                       float(bparams.get("radius_factor", 1.0)), float(bparams.get("kn", 0.0)),
                       float(bparams.get("kt", 0.0)), float(bparams.get("break_strain", 0.0)), int(pow_mode))


def setup_bonds(bonds, state, factor, search_cutoff=0.0):
    return lib().orc_setup_bonds(C.byref(_bonds(bonds)), C.byref(_particles(state)), float(factor),
                                 float(search_cutoff))


def bonded_run(state, bonds, bparams, dt, nsteps, gravity=(0.0, 0.0, 0.0), ext_force=None, fix_flags=None,
               pow_mode=POW_LIBM):
    p, b, bp = _particles(state), _bonds(bonds), _bp(bparams, pow_mode)
    h = _HookHolder(gravity, ext_force, fix_flags)
    st = 0
    L = lib()
    for _ in range(int(nsteps)):
        st |= L.orc_bonded_step(C.byref(p), C.byref(b), C.byref(bp), C.byref(h.h), dt)
    return st
