"""Host-side particle / wall / bond state in the reference's array layout.

These containers hold exactly the per-particle properties that
``CabanaDEM::Particles`` (src/CabanaDEM_Particles.hpp:349-370), ``CabanaDEM::Wall``
(src/CabanaDEM_Wall.hpp) and ``CabanaBondedDEM::ParticlesBondedDEM``
(src/CabanaBondedDEM_Particles.hpp:29-293) expose through their ``slice*()``
accessors, as C-contiguous numpy arrays in the reference's index order: vectors are
``[n][3]``, tangential history ``[n][MaxCnts]``, wall history ``[n][MaxNoWalls]``.
They are the staging format for the device library's ``dem_particles_set/get``.
"""
from __future__ import annotations

from dataclasses import dataclass, field, fields

import numpy as np

VEC_FIELDS = ("x", "u", "omega", "force", "torque")
SCALAR_FIELDS = ("m", "rho", "rad", "I", "E", "nu", "G")


@dataclass
class ParticleState:
    n: int
    max_cnts: int
    max_walls: int
    x: np.ndarray = field(repr=False, default=None)
    u: np.ndarray = field(repr=False, default=None)
    omega: np.ndarray = field(repr=False, default=None)
    force: np.ndarray = field(repr=False, default=None)
    torque: np.ndarray = field(repr=False, default=None)
    m: np.ndarray = field(repr=False, default=None)
    rho: np.ndarray = field(repr=False, default=None)
    rad: np.ndarray = field(repr=False, default=None)
    I: np.ndarray = field(repr=False, default=None)
    E: np.ndarray = field(repr=False, default=None)
    nu: np.ndarray = field(repr=False, default=None)
    G: np.ndarray = field(repr=False, default=None)
    tng_idx: np.ndarray = field(repr=False, default=None)
    tng_ss_x: np.ndarray = field(repr=False, default=None)
    tng_ss_y: np.ndarray = field(repr=False, default=None)
    tng_ss_z: np.ndarray = field(repr=False, default=None)
    tng_count: np.ndarray = field(repr=False, default=None)
    tng_sw_x: np.ndarray = field(repr=False, default=None)
    tng_sw_y: np.ndarray = field(repr=False, default=None)
    tng_sw_z: np.ndarray = field(repr=False, default=None)

    @classmethod
    def create(cls, n: int, max_cnts: int = 16, max_walls: int = 6) -> "ParticleState":
        s = cls(n=n, max_cnts=max_cnts, max_walls=max_walls)
        for f in VEC_FIELDS:
            setattr(s, f, np.zeros((n, 3)))
        for f in SCALAR_FIELDS:
            setattr(s, f, np.zeros(n))
        s.tng_idx = np.full((n, max_cnts), -1, dtype=np.int32)
        for c in "xyz":
            setattr(s, "tng_ss_" + c, np.zeros((n, max_cnts)))
            setattr(s, "tng_sw_" + c, np.zeros((n, max(max_walls, 1))))
        s.tng_count = np.zeros(n, dtype=np.int32)
        return s

    def arrays(self):
        return {f.name: getattr(self, f.name) for f in fields(self) if isinstance(getattr(self, f.name), np.ndarray)}

    def copy(self) -> "ParticleState":
        s = ParticleState(n=self.n, max_cnts=self.max_cnts, max_walls=self.max_walls)
        for k, v in self.arrays().items():
            setattr(s, k, np.ascontiguousarray(v).copy())
        return s

    def resized(self, n: int) -> "ParticleState":
        """A copy with n particles (Particles::resize, src/CabanaDEM_Particles.hpp:273-297): the
        first min(n, self.n) keep their values; added particles are zeroed, with empty contact
        slots (tangential index -1)."""
        out = ParticleState.create(n, self.max_cnts, self.tng_sw_x.shape[1])
        k = min(n, self.n)
        for name, a in self.arrays().items():
            getattr(out, name)[:k] = a[:k]
        return out

    def set_sphere_mass(self):
        """m = 4/3 pi r^3 rho and I = 2/5 m r^2, in the reference examples' order (e.g.
        examples/01_elastic_normal_impact_of_two_identical_particles.cpp:106-107)."""
        r = self.rad
        self.m[:] = 4.0 / 3.0 * np.pi * r * r * r * self.rho
        self.I[:] = 2.0 / 5.0 * self.m * r * r

    def contact_pairs(self):
        """Tracked tangential contacts as {(i, j): (hx, hy, hz)} (slot order dropped)."""
        out = {}
        for i in range(self.n):
            for k in range(int(self.tng_count[i])):
                j = int(self.tng_idx[i, k])
                out[(i, j)] = (self.tng_ss_x[i, k], self.tng_ss_y[i, k], self.tng_ss_z[i, k])
        return out


@dataclass
class WallState:
    n: int
    x: np.ndarray = field(repr=False, default=None)
    u: np.ndarray = field(repr=False, default=None)
    omega: np.ndarray = field(repr=False, default=None)
    normal: np.ndarray = field(repr=False, default=None)
    E: np.ndarray = field(repr=False, default=None)
    nu: np.ndarray = field(repr=False, default=None)
    G: np.ndarray = field(repr=False, default=None)

    @classmethod
    def create(cls, n: int) -> "WallState":
        w = cls(n=n)
        for f in ("x", "u", "omega", "normal"):
            setattr(w, f, np.zeros((n, 3)))
        for f in ("E", "nu", "G"):
            setattr(w, f, np.zeros(n))
        return w

    def copy(self) -> "WallState":
        w = WallState(n=self.n)
        for f in ("x", "u", "omega", "normal", "E", "nu", "G"):
            setattr(w, f, getattr(self, f).copy())
        return w


@dataclass
class MeshState:
    """A triangle-mesh wall: vertices [nt, 3, 3] at translation D, one material, translation
    velocity u (the mesh moves only when the force's Q6 bit is clear), and the per-particle
    tracked triangle contacts (triangle id, tangential history, count) for n particles."""
    tri: np.ndarray = field(repr=False, default=None)
    E: float = 0.0
    nu: float = 0.0
    G: float = 0.0
    u: np.ndarray = field(repr=False, default=None)
    D: np.ndarray = field(repr=False, default=None)
    max_contacts: int = 8
    tid: np.ndarray = field(repr=False, default=None)
    th_x: np.ndarray = field(repr=False, default=None)
    th_y: np.ndarray = field(repr=False, default=None)
    th_z: np.ndarray = field(repr=False, default=None)
    cnt: np.ndarray = field(repr=False, default=None)

    @classmethod
    def create(cls, tri, n: int, E: float, nu: float, G: float, u=(0.0, 0.0, 0.0), max_contacts: int = 8):
        m = cls(tri=np.ascontiguousarray(tri, dtype=np.float64).reshape(-1, 3, 3), E=float(E), nu=float(nu),
                G=float(G), u=np.array(u, dtype=np.float64), D=np.zeros(3), max_contacts=int(max_contacts))
        m.tid = np.full((n, m.max_contacts), -1, dtype=np.int32)
        for f in ("th_x", "th_y", "th_z"):
            setattr(m, f, np.zeros((n, m.max_contacts)))
        m.cnt = np.zeros(n, dtype=np.int32)
        return m

    @property
    def nt(self) -> int:
        return self.tri.shape[0]

    def copy(self) -> "MeshState":
        m = MeshState(tri=self.tri.copy(), E=self.E, nu=self.nu, G=self.G, u=self.u.copy(), D=self.D.copy(),
                      max_contacts=self.max_contacts)
        for f in ("tid", "th_x", "th_y", "th_z", "cnt"):
            setattr(m, f, getattr(self, f).copy())
        return m


BOND_HIST = ("fn_x", "fn_y", "fn_z", "ft_x", "ft_y", "ft_z", "mn_x", "mn_y", "mn_z", "mt_x", "mt_y", "mt_z")


@dataclass
class BondState:
    """Bond slots of ``ParticlesBondedDEM`` (src/CabanaBondedDEM_Particles.hpp:187-201)."""
    n: int
    max_bonds: int
    idx: np.ndarray = field(repr=False, default=None)
    init_len: np.ndarray = field(repr=False, default=None)
    count: np.ndarray = field(repr=False, default=None)
    broken: np.ndarray = field(repr=False, default=None)
    hist: dict = field(repr=False, default=None)

    @classmethod
    def create(cls, n: int, max_bonds: int) -> "BondState":
        b = cls(n=n, max_bonds=max_bonds)
        b.idx = np.full((n, max_bonds), -1, dtype=np.int32)
        b.init_len = np.zeros((n, max_bonds))
        b.count = np.zeros(n, dtype=np.int32)
        b.broken = np.zeros((n, max_bonds), dtype=np.uint8)
        b.hist = {k: np.zeros((n, max_bonds)) for k in BOND_HIST}
        return b

    def copy(self) -> "BondState":
        b = BondState(n=self.n, max_bonds=self.max_bonds)
        b.idx, b.init_len, b.count, b.broken = (self.idx.copy(), self.init_len.copy(), self.count.copy(),
                                                self.broken.copy())
        b.hist = {k: v.copy() for k, v in self.hist.items()}
        return b

    def broken_bonds(self) -> int:
        """Broken bonds, each counted once (both ends of a bond break together)."""
        return int(self.broken.sum()) // 2
