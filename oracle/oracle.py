"""ORACLE — test infrastructure only (the checker, never the product).

ctypes access to the two CPU libraries that oracle/Makefile builds:

* ``Oracle``: liboracle.so, the serial restatement of the reference's hot path (oracle/md_oracle.cpp);
* ``Reference``: oracle/_ref/libmdref.so, the reference's own sources compiled unmodified, driven through
  oracle/ref_harness.cpp (strict IEEE build, for parity); ``stock_reference_path()`` names the same sources built
  with the reference's release flags, for timing.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs import this module.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmdref.so")
REF_MD_SIM = os.path.join(HERE, "_ref", "md_sim")
REF_STOCK = {"v4": os.path.join(HERE, "_ref", "libmdref_stock_v4.so"),
             "v3": os.path.join(HERE, "_ref", "libmdref_stock_v3.so")}
_V4_FLAGS = {"avx512f", "avx512dq", "avx512cd", "avx512bw", "avx512vl"}


def stock_reference_path() -> tuple[str, str]:
    """The reference built with its release flags (-O3, FMA contraction on; CMakeLists.txt:12) for the ISA level
    this host runs -- x86-64-v4 (AVX-512) when /proc/cpuinfo lists its flags, else x86-64-v3 -- standing in for
    -march=native. Falls back to the strict parity build when neither was built. Returns (path, description)."""
    flags = set()
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    break
    except OSError:
        pass
    level = "v4" if _V4_FLAGS <= flags else "v3"
    for lv in ([level, "v3"] if level == "v4" else ["v3"]):
        if os.path.exists(REF_STOCK[lv]):
            return REF_STOCK[lv], f"reference sources, release flags (-O3, FMA contraction on, -march=x86-64-{lv})"
    return REF_SO, "reference sources, strict parity build (-O3 -march=x86-64-v3 -ffp-contract=off)"

_P = C.c_void_p
_D = C.c_double
_I = C.c_int
_I64 = C.c_int64
_U64 = C.c_uint64
_PD = C.POINTER(C.c_double)
_PI = C.POINTER(C.c_int)
_PU64 = C.POINTER(C.c_uint64)


def _pd(a):
    return None if a is None else a.ctypes.data_as(_PD)


def _pu(a):
    return None if a is None else a.ctypes.data_as(_PU64)


def _pi(a):
    return None if a is None else a.ctypes.data_as(_PI)


def fcc_box(cells: int, density: float) -> tuple[float, float]:
    """Lattice constant and box length of md_sim's FCC start (src/main.cpp:164-166), via the C library's
    cbrt so the bits match the reference's std::cbrt."""
    a, box = C.c_double(0), C.c_double(0)
    Oracle().lib.orc_fcc_box(cells, density, C.byref(a), C.byref(box))
    return a.value, box.value


@dataclass
class State:
    """Host copy of a System: pos is (n, 4) packed x, y, z, pad; vel/force are (3, n) component arrays."""

    pos: np.ndarray
    vel: np.ndarray
    force: np.ndarray
    mass: np.ndarray
    ids: np.ndarray
    box: float

    @property
    def n(self) -> int:
        return self.pos.shape[0]

    def copy(self) -> "State":
        return State(self.pos.copy(), self.vel.copy(), self.force.copy(), self.mass.copy(), self.ids.copy(),
                     self.box)


def state_hash(pos: np.ndarray, vel: np.ndarray) -> int:
    """FNV-1a over the bytes of (x, vx, y, vy, z, vz) per particle (src/System.cpp:85-105), vectorised."""
    n = pos.shape[0]
    inter = np.empty((n, 6), dtype=np.float64)
    inter[:, 0::2] = pos[:, :3]
    inter[:, 1::2] = vel.T
    data = inter.reshape(-1).view(np.uint8)
    h = 14695981039346656037
    prime = 1099511628211
    mask = (1 << 64) - 1
    for b in data.tobytes():
        h = ((h ^ b) * prime) & mask
    return h


class _Lib:
    def __init__(self, path: str):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)


class Oracle(_Lib):
    """The serial C++ restatement (liboracle.so)."""

    def __init__(self, path: str = ORACLE_SO):
        super().__init__(path)
        L = self.lib
        L.orc_last_error.restype = C.c_char_p
        L.orc_fcc.argtypes = [_I, _D, _PD]
        L.orc_fcc_box.argtypes = [_I, _D, _PD, _PD]
        L.orc_sys_create.restype = _P
        L.orc_sys_create.argtypes = [_I64, _D, _PD, _PD, _PD, _PD]
        L.orc_sys_destroy.argtypes = [_P]
        L.orc_sys_get.argtypes = [_P, _PD, _PD, _PD, _PD, _PU64]
        L.orc_sys_set.argtypes = [_P, _PD, _PD, _PD]
        L.orc_sys_reorder.argtypes = [_P, _PU64]
        for f in ("orc_kinetic", "orc_temperature"):
            getattr(L, f).restype = _D
            getattr(L, f).argtypes = [_P]
        L.orc_hash.restype = _U64
        L.orc_hash.argtypes = [_P]
        L.orc_scale.argtypes = [_P, _D]
        L.orc_rescale.argtypes = [_P, _D]
        L.orc_init_velocities.argtypes = [_P, _D, C.c_uint32]
        L.orc_bussi_factor.restype = _D
        L.orc_bussi_factor.argtypes = [_D, _I64, _D, _D, _D, _D]
        L.orc_bussi_apply.argtypes = [_P, _D, _D, _D, _D]
        L.orc_bussi_noise.argtypes = [_U64, _I64, _I64, _PD, _PD]
        L.orc_cells_per_side.restype = _I
        L.orc_cells_per_side.argtypes = [_D, _D]
        L.orc_cells_build.restype = _I
        L.orc_cells_build.argtypes = [_P, _D, _PI, _PU64, _PU64]
        L.orc_neighbour_cells.argtypes = [_I, _I, _PI]
        L.orc_nl_create.restype = _P
        L.orc_nl_create.argtypes = [_D, _D, _I]
        L.orc_nl_destroy.argtypes = [_P]
        L.orc_nl_build.restype = _I
        L.orc_nl_build.argtypes = [_P, _P]
        L.orc_nl_update.restype = _I
        L.orc_nl_update.argtypes = [_P, _P, _PI]
        L.orc_nl_pairs.restype = _U64
        L.orc_nl_pairs.argtypes = [_P]
        L.orc_nl_rebuilds.restype = _I
        L.orc_nl_rebuilds.argtypes = [_P]
        L.orc_nl_cells_per_side.restype = _I
        L.orc_nl_cells_per_side.argtypes = [_P]
        L.orc_nl_get.argtypes = [_P, _PU64, _PU64, _PU64, _PU64, _PI, _PU64]
        L.orc_ff_create.restype = _P
        L.orc_ff_create.argtypes = [_D, _D, _D]
        L.orc_ff_destroy.argtypes = [_P]
        for f in ("orc_ff_shift", "orc_ff_virial", "orc_ff_inside"):
            getattr(L, f).restype = _D
            getattr(L, f).argtypes = [_P]
        L.orc_ff_forces.restype = _I
        L.orc_ff_forces.argtypes = [_P, _P, _P, _I, _PD]
        L.orc_step.restype = _I
        L.orc_step.argtypes = [_P, _P, _P, _D, _I, _PD]
        L.orc_rdf_sample.argtypes = [_P, _P, _D, _I, _PD]
        L.orc_rdf_values.argtypes = [_PD, _I, _D, _I, _D, _D, _PD]
        L.orc_adj_create.restype = _P
        L.orc_adj_create.argtypes = [_I64, _D, _PD, _PD, _PD, _D, _D, _D, _D, _D, _I, _I]
        L.orc_adj_destroy.argtypes = [_P]
        L.orc_adj_forward.argtypes = [_P, _PD, _PD, _PD, _PD, _PD]
        L.orc_adj_backward.argtypes = [_P, _D, _D, _PD, _PD, _PD, _PD]

    def error(self) -> str:
        return self.lib.orc_last_error().decode()

    def fcc(self, cells: int, a: float) -> np.ndarray:
        pos = np.zeros((4 * cells ** 3, 4))
        self.lib.orc_fcc(cells, a, _pd(pos))
        return pos

    def system(self, pos, box, vel=None, force=None, mass=None) -> "OSystem":
        return OSystem(self, pos, box, vel, force, mass)

    def fcc_system(self, cells: int, density: float, temperature: float, seed: int = 42) -> "OSystem":
        a, box = fcc_box(cells, density)
        s = self.system(self.fcc(cells, a), box)
        self.lib.orc_init_velocities(s.h, temperature, seed)
        return s

    def cells_build(self, s: "OSystem", min_cell: float):
        ncps = self.lib.orc_cells_per_side(s.box, min_cell)
        cell = np.zeros(s.n, dtype=np.int32)
        start = np.zeros(ncps ** 3 + 1, dtype=np.uint64)
        parts = np.zeros(s.n, dtype=np.uint64)
        self.lib.orc_cells_build(s.h, min_cell, _pi(cell), _pu(start), _pu(parts))
        return ncps, cell, start, parts

    def neighbour_cells(self, ncps: int, cell: int) -> np.ndarray:
        out = np.zeros(27, dtype=np.int32)
        self.lib.orc_neighbour_cells(ncps, cell, _pi(out))
        return out

    def bussi_factor(self, kinetic, n, temperature, c, r1, chi2) -> float:
        return self.lib.orc_bussi_factor(kinetic, n, temperature, c, r1, chi2)

    def bussi_noise(self, seed: int, n: int, count: int) -> tuple[np.ndarray, np.ndarray]:
        r1 = np.zeros(count)
        chi2 = np.zeros(count)
        self.lib.orc_bussi_noise(seed, n, count, _pd(r1), _pd(chi2))
        return r1, chi2

    def rdf_values(self, hist, rmax, samples, particles, box) -> np.ndarray:
        g = np.zeros(len(hist))
        h = np.ascontiguousarray(hist, dtype=np.float64)
        self.lib.orc_rdf_values(_pd(h), len(h), rmax, samples, float(particles), box, _pd(g))
        return g


class OSystem:
    def __init__(self, o: Oracle, pos, box, vel=None, force=None, mass=None):
        self.o = o
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        if pos.shape[1] == 3:
            pos = np.concatenate([pos, np.zeros((pos.shape[0], 1))], axis=1)
        n = pos.shape[0]
        vel = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64)
        force = None if force is None else np.ascontiguousarray(force, dtype=np.float64)
        mass = None if mass is None else np.ascontiguousarray(mass, dtype=np.float64)
        self.n = n
        self.box = float(box)
        self.h = o.lib.orc_sys_create(n, self.box, _pd(pos), _pd(vel), _pd(force), _pd(mass))

    def __del__(self):
        try:
            self.o.lib.orc_sys_destroy(self.h)
        except Exception:
            pass

    def state(self) -> State:
        n = self.n
        pos = np.zeros((n, 4))
        vel = np.zeros((3, n))
        force = np.zeros((3, n))
        mass = np.zeros(n)
        ids = np.zeros(n, dtype=np.uint64)
        self.o.lib.orc_sys_get(self.h, _pd(pos), _pd(vel), _pd(force), _pd(mass), _pu(ids))
        return State(pos, vel, force, mass, ids, self.box)

    def set(self, pos=None, vel=None, force=None):
        self.o.lib.orc_sys_set(self.h, _pd(None if pos is None else np.ascontiguousarray(pos, np.float64)),
                               _pd(None if vel is None else np.ascontiguousarray(vel, np.float64)),
                               _pd(None if force is None else np.ascontiguousarray(force, np.float64)))

    def reorder(self, order):
        o = np.ascontiguousarray(order, dtype=np.uint64)
        self.o.lib.orc_sys_reorder(self.h, _pu(o))

    def kinetic(self) -> float:
        return self.o.lib.orc_kinetic(self.h)

    def temperature(self) -> float:
        return self.o.lib.orc_temperature(self.h)

    def hash(self) -> int:
        return self.o.lib.orc_hash(self.h)

    def scale(self, s: float):
        self.o.lib.orc_scale(self.h, s)

    def rescale(self, t: float):
        self.o.lib.orc_rescale(self.h, t)

    def bussi(self, temperature, c, r1, chi2):
        self.o.lib.orc_bussi_apply(self.h, temperature, c, r1, chi2)


class ONeighbourList:
    def __init__(self, o: Oracle, rc: float, skin: float, reverse: bool = False):
        self.o = o
        self.reverse = reverse
        self.h = o.lib.orc_nl_create(rc, skin, int(reverse))

    def __del__(self):
        try:
            self.o.lib.orc_nl_destroy(self.h)
        except Exception:
            pass

    def build(self, s: OSystem):
        if self.o.lib.orc_nl_build(self.h, s.h) != 0:
            raise RuntimeError(self.o.error())

    def update(self, s: OSystem) -> bool:
        r = C.c_int(0)
        if self.o.lib.orc_nl_update(self.h, s.h, C.byref(r)) != 0:
            raise RuntimeError(self.o.error())
        return bool(r.value)

    @property
    def pairs(self) -> int:
        return self.o.lib.orc_nl_pairs(self.h)

    @property
    def rebuilds(self) -> int:
        return self.o.lib.orc_nl_rebuilds(self.h)

    def get(self, n: int):
        P = self.pairs
        ncps = self.o.lib.orc_nl_cells_per_side(self.h)
        off = np.zeros(n + 1, dtype=np.uint64)
        nb = np.zeros(P, dtype=np.uint64)
        roff = np.zeros(n + 1, dtype=np.uint64) if self.reverse else None
        rp = np.zeros(P, dtype=np.uint64) if self.reverse else None
        cell = np.zeros(n, dtype=np.int32)
        start = np.zeros(ncps ** 3 + 1, dtype=np.uint64)
        self.o.lib.orc_nl_get(self.h, _pu(off), _pu(nb), _pu(roff), _pu(rp), _pi(cell), _pu(start))
        return dict(offsets=off, neighbours=nb, rev_offsets=roff, rev_pairs=rp, cell=cell, cell_start=start,
                    ncps=ncps)


MODE_DEFAULT, MODE_DETERMINISTIC, MODE_MIXED, MODE_ALL_PAIRS = 0, 1, 2, 3


class OForceField:
    def __init__(self, o: Oracle, eps: float, sigma: float, rc: float):
        self.o = o
        self.h = o.lib.orc_ff_create(eps, sigma, rc)

    def __del__(self):
        try:
            self.o.lib.orc_ff_destroy(self.h)
        except Exception:
            pass

    def forces(self, s: OSystem, nl: ONeighbourList | None, mode: int = MODE_DETERMINISTIC) -> float:
        pe = C.c_double(0)
        if self.o.lib.orc_ff_forces(self.h, s.h, None if nl is None else nl.h, mode, C.byref(pe)) != 0:
            raise RuntimeError(self.o.error())
        return pe.value

    def step(self, s: OSystem, nl: ONeighbourList | None, dt: float, mode: int = MODE_DETERMINISTIC) -> float:
        pe = C.c_double(0)
        if self.o.lib.orc_step(s.h, self.h, None if nl is None else nl.h, dt, mode, C.byref(pe)) != 0:
            raise RuntimeError(self.o.error())
        return pe.value

    @property
    def shift(self):
        return self.o.lib.orc_ff_shift(self.h)

    @property
    def virial(self):
        return self.o.lib.orc_ff_virial(self.h)

    @property
    def inside(self):
        return self.o.lib.orc_ff_inside(self.h)


def rdf_sample(o: Oracle, s: OSystem, nl: ONeighbourList, rmax: float, bins: int, hist: np.ndarray):
    o.lib.orc_rdf_sample(s.h, nl.h, rmax, bins, _pd(hist))


class OAdjoint:
    """The FP64 CPU adjoint of the trajectory (md_adjoint.cpp): J = g_pe mean U + g_p mean P over `steps` steps."""

    def __init__(self, o: Oracle, pos, box, vel, mass=None, eps=1.0, sigma=1.0, rc=2.5, skin=0.3, dt=0.005,
                 steps=200, every=20):
        self.o = o
        self.n = len(pos)
        self.steps = steps
        p = np.ascontiguousarray(pos, dtype=np.float64)
        v = np.ascontiguousarray(vel, dtype=np.float64)
        m = None if mass is None else np.ascontiguousarray(mass, dtype=np.float64)
        self.h = o.lib.orc_adj_create(self.n, box, _pd(p), _pd(v), _pd(m), eps, sigma, rc, skin, dt, steps, every)

    def __del__(self):
        try:
            self.o.lib.orc_adj_destroy(self.h)
        except Exception:
            pass

    def forward(self):
        """(mean U, mean P, U_k, W_k, KE_k)"""
        mu, mp = C.c_double(), C.c_double()
        u, w, k = np.zeros(self.steps), np.zeros(self.steps), np.zeros(self.steps)
        self.o.lib.orc_adj_forward(self.h, C.byref(mu), C.byref(mp), _pd(u), _pd(w), _pd(k))
        return mu.value, mp.value, u, w, k

    def backward(self, g_pe, g_p):
        de, ds = C.c_double(), C.c_double()
        dp, dv = np.zeros((3, self.n)), np.zeros((3, self.n))
        self.o.lib.orc_adj_backward(self.h, g_pe, g_p, C.byref(de), C.byref(ds), _pd(dp), _pd(dv))
        return dict(d_epsilon=de.value, d_sigma=ds.value, d_pos=dp, d_vel=dv)


class Reference(_Lib):
    """The reference's own classes (oracle/_ref/libmdref.so, built from its unmodified sources)."""

    def __init__(self, path: str = REF_SO):
        super().__init__(path)
        L = self.lib
        L.ref_last_error.restype = C.c_char_p
        L.ref_set_threads.argtypes = [_I]
        L.ref_max_threads.restype = _I
        L.ref_sys_create_fcc.restype = _P
        L.ref_sys_create_fcc.argtypes = [_I, _D, _D, C.c_uint]
        L.ref_sys_create.restype = _P
        L.ref_sys_create.argtypes = [_I64, _D, _PD, _PD, _PD]
        L.ref_sys_clone.restype = _P
        L.ref_sys_clone.argtypes = [_P]
        L.ref_sys_destroy.argtypes = [_P]
        L.ref_sys_size.restype = _I64
        L.ref_sys_size.argtypes = [_P]
        L.ref_sys_box.restype = _D
        L.ref_sys_box.argtypes = [_P]
        L.ref_sys_get.argtypes = [_P, _PD, _PD, _PD, _PD, _PU64]
        L.ref_sys_set_velocity.argtypes = [_P, _PD]
        for f in ("ref_kinetic", "ref_temperature"):
            getattr(L, f).restype = _D
            getattr(L, f).argtypes = [_P]
        L.ref_hash.restype = _U64
        L.ref_hash.argtypes = [_P]
        L.ref_rescale.argtypes = [_P, _D]
        L.ref_cells_build.restype = _I
        L.ref_cells_build.argtypes = [_P, _D, _PI, _PU64, _PU64]
        L.ref_nl_create.restype = _P
        L.ref_nl_create.argtypes = [_D, _D, _I]
        L.ref_nl_destroy.argtypes = [_P]
        L.ref_nl_build.restype = _I
        L.ref_nl_build.argtypes = [_P, _P]
        L.ref_nl_update.restype = _I
        L.ref_nl_update.argtypes = [_P, _P, _PI]
        L.ref_nl_pairs.restype = _U64
        L.ref_nl_pairs.argtypes = [_P]
        L.ref_nl_rebuilds.restype = _I
        L.ref_nl_rebuilds.argtypes = [_P]
        L.ref_nl_get.argtypes = [_P, _I64, _PU64, _PU64, _PU64, _PU64]
        L.ref_ff_create.restype = _P
        L.ref_ff_create.argtypes = [_D, _D, _D]
        L.ref_ff_destroy.argtypes = [_P]
        L.ref_ff_set.argtypes = [_P, _I, _I]
        for f in ("ref_ff_shift", "ref_ff_virial", "ref_ff_inside"):
            getattr(L, f).restype = _D
            getattr(L, f).argtypes = [_P]
        L.ref_ff_forces_list.restype = _I
        L.ref_ff_forces_list.argtypes = [_P, _P, _P, _PD]
        L.ref_ff_forces_all.restype = _I
        L.ref_ff_forces_all.argtypes = [_P, _P, _PD]
        L.ref_run.restype = _I
        L.ref_run.argtypes = [_P, _P, _P, _D, _I, _I, _D, _PD, _PD]
        L.ref_run_observables.restype = _I
        L.ref_run_observables.argtypes = [_P, _P, _P, _D, _I, _PD, _PD, _PD]
        L.ref_bussi_create.restype = _P
        L.ref_bussi_create.argtypes = [_D, _D, _U64]
        L.ref_bussi_destroy.argtypes = [_P]
        L.ref_bussi_apply.argtypes = [_P, _P, _D]
        L.ref_rdf_create.restype = _P
        L.ref_rdf_create.argtypes = [_D, _I]
        L.ref_rdf_destroy.argtypes = [_P]
        L.ref_rdf_sample.argtypes = [_P, _P, _P]
        L.ref_rdf_values.argtypes = [_P, _PD, _PD]

    def error(self) -> str:
        return self.lib.ref_last_error().decode()

    def set_threads(self, n: int):
        self.lib.ref_set_threads(n)

    def max_threads(self) -> int:
        return self.lib.ref_max_threads()

    def fcc_system(self, cells, density, temperature, seed=42) -> "RSystem":
        return RSystem(self, self.lib.ref_sys_create_fcc(cells, density, temperature, seed))

    def system(self, pos, box, vel=None, mass=None) -> "RSystem":
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        if pos.shape[1] == 3:
            pos = np.concatenate([pos, np.zeros((pos.shape[0], 1))], axis=1)
        v = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64)
        m = None if mass is None else np.ascontiguousarray(mass, dtype=np.float64)
        return RSystem(self, self.lib.ref_sys_create(pos.shape[0], box, _pd(pos), _pd(v), _pd(m)))


class RSystem:
    def __init__(self, r: Reference, h):
        self.r = r
        self.h = h

    def __del__(self):
        try:
            self.r.lib.ref_sys_destroy(self.h)
        except Exception:
            pass

    @property
    def n(self) -> int:
        return self.r.lib.ref_sys_size(self.h)

    @property
    def box(self) -> float:
        return self.r.lib.ref_sys_box(self.h)

    def clone(self) -> "RSystem":
        return RSystem(self.r, self.r.lib.ref_sys_clone(self.h))

    def state(self) -> State:
        n = self.n
        pos = np.zeros((n, 4))
        vel = np.zeros((3, n))
        force = np.zeros((3, n))
        mass = np.zeros(n)
        ids = np.zeros(n, dtype=np.uint64)
        self.r.lib.ref_sys_get(self.h, _pd(pos), _pd(vel), _pd(force), _pd(mass), _pu(ids))
        return State(pos, vel, force, mass, ids, self.box)

    def set_velocity(self, vel):
        self.r.lib.ref_sys_set_velocity(self.h, _pd(np.ascontiguousarray(vel, np.float64)))

    def kinetic(self):
        return self.r.lib.ref_kinetic(self.h)

    def temperature(self):
        return self.r.lib.ref_temperature(self.h)

    def hash(self) -> int:
        return self.r.lib.ref_hash(self.h)

    def rescale(self, t):
        self.r.lib.ref_rescale(self.h, t)

    def cells_build(self, min_cell):
        from math import floor
        ncps = max(1, int(floor(self.box / min_cell)))
        n = self.n
        cell = np.zeros(n, dtype=np.int32)
        start = np.zeros(ncps ** 3 + 1, dtype=np.uint64)
        parts = np.zeros(n, dtype=np.uint64)
        got = self.r.lib.ref_cells_build(self.h, min_cell, _pi(cell), _pu(start), _pu(parts))
        assert got == ncps
        return ncps, cell, start, parts


class RNeighbourList:
    def __init__(self, r: Reference, rc, skin, reverse=False):
        self.r = r
        self.reverse = reverse
        self.h = r.lib.ref_nl_create(rc, skin, int(reverse))

    def __del__(self):
        try:
            self.r.lib.ref_nl_destroy(self.h)
        except Exception:
            pass

    def build(self, s: RSystem):
        if self.r.lib.ref_nl_build(self.h, s.h) != 0:
            raise RuntimeError(self.r.error())

    def update(self, s: RSystem) -> bool:
        x = C.c_int(0)
        if self.r.lib.ref_nl_update(self.h, s.h, C.byref(x)) != 0:
            raise RuntimeError(self.r.error())
        return bool(x.value)

    @property
    def pairs(self):
        return self.r.lib.ref_nl_pairs(self.h)

    @property
    def rebuilds(self):
        return self.r.lib.ref_nl_rebuilds(self.h)

    def get(self, n):
        P = self.pairs
        off = np.zeros(n + 1, dtype=np.uint64)
        nb = np.zeros(P, dtype=np.uint64)
        roff = np.zeros(n + 1, dtype=np.uint64) if self.reverse else None
        rp = np.zeros(P, dtype=np.uint64) if self.reverse else None
        self.r.lib.ref_nl_get(self.h, n, _pu(off), _pu(nb), _pu(roff), _pu(rp))
        return dict(offsets=off, neighbours=nb, rev_offsets=roff, rev_pairs=rp)


class RForceField:
    def __init__(self, r: Reference, eps, sigma, rc, deterministic=False, mixed=False):
        self.r = r
        self.h = r.lib.ref_ff_create(eps, sigma, rc)
        r.lib.ref_ff_set(self.h, int(deterministic), int(mixed))

    def __del__(self):
        try:
            self.r.lib.ref_ff_destroy(self.h)
        except Exception:
            pass

    def set(self, deterministic=False, mixed=False):
        self.r.lib.ref_ff_set(self.h, int(deterministic), int(mixed))

    def forces(self, s: RSystem, nl: RNeighbourList | None) -> float:
        pe = C.c_double(0)
        if nl is None:
            rc = self.r.lib.ref_ff_forces_all(self.h, s.h, C.byref(pe))
        else:
            rc = self.r.lib.ref_ff_forces_list(self.h, s.h, nl.h, C.byref(pe))
        if rc != 0:
            raise RuntimeError(self.r.error())
        return pe.value

    def run(self, s: RSystem, nl: RNeighbourList | None, dt: float, steps: int, rescale_every=0, rescale_t=0.0,
            record=False):
        pe = np.zeros(steps) if record else None
        ke = np.zeros(steps) if record else None
        if self.r.lib.ref_run(s.h, self.h, None if nl is None else nl.h, dt, steps, rescale_every, rescale_t,
                              _pd(pe), _pd(ke)) != 0:
            raise RuntimeError(self.r.error())
        return pe, ke

    def observables(self, s: RSystem, nl: RNeighbourList, dt: float, steps: int):
        """`steps` NVE steps through the reference's integrator: per-step (PE, virial, KE)."""
        pe, w, ke = np.zeros(steps), np.zeros(steps), np.zeros(steps)
        if self.r.lib.ref_run_observables(s.h, self.h, nl.h, dt, steps, _pd(pe), _pd(w), _pd(ke)) != 0:
            raise RuntimeError(self.r.error())
        return pe, w, ke

    @property
    def shift(self):
        return self.r.lib.ref_ff_shift(self.h)

    @property
    def virial(self):
        return self.r.lib.ref_ff_virial(self.h)

    @property
    def inside(self):
        return self.r.lib.ref_ff_inside(self.h)


class RBussi:
    def __init__(self, r: Reference, temperature, tau, seed):
        self.r = r
        self.h = r.lib.ref_bussi_create(temperature, tau, seed)

    def __del__(self):
        try:
            self.r.lib.ref_bussi_destroy(self.h)
        except Exception:
            pass

    def apply(self, s: RSystem, dt):
        self.r.lib.ref_bussi_apply(self.h, s.h, dt)


class RRdf:
    def __init__(self, r: Reference, rmax, bins):
        self.r = r
        self.bins = bins
        self.h = r.lib.ref_rdf_create(rmax, bins)

    def __del__(self):
        try:
            self.r.lib.ref_rdf_destroy(self.h)
        except Exception:
            pass

    def sample(self, s: RSystem, nl: RNeighbourList):
        self.r.lib.ref_rdf_sample(self.h, s.h, nl.h)

    def values(self):
        radii = np.zeros(self.bins)
        g = np.zeros(self.bins)
        self.r.lib.ref_rdf_values(self.h, _pd(radii), _pd(g))
        return radii, g
