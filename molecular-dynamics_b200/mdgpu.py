"""Python mirror of the reference's hot-path classes over libmdgpu.so's C-ABI (include/md_b200.h).

The names and argument meanings follow nhantran1711/molecular-dynamics (include/System.hpp,
include/CellList.hpp, include/NeighbourList.hpp, include/Forcefield.hpp, include/Integrator.hpp,
include/Thermostat.hpp, include/RadialDistribution.hpp); the errors the reference throws as
std::runtime_error are raised as RuntimeError with the same messages. Every computation runs in the CUDA
library: this module only moves arrays and calls entry points. It raises at import time when the library has
not been built, and every device call fails loudly when no GPU is present.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmdgpu.so")

PREC_FP64, PREC_FP32FX, PREC_FP32, PREC_FX64, PREC_FX32 = 0, 1, 2, 3, 4
GRAPH_TEST_RERUN = 1  # md_system_set_graph test flag
_ERRORS = {1: "MD_ERR_INVALID", 2: "MD_ERR_CUTOFF", 3: "MD_ERR_LIST_RADIUS", 4: "MD_ERR_NO_REVERSE_INDEX",
           5: "MD_ERR_CAPACITY", 6: "MD_ERR_CUDA", 7: "MD_ERR_NO_DEVICE", 8: "MD_ERR_STATE", 9: "MD_ERR_TIMEOUT"}

_P, _D, _I, _I64, _U64 = C.c_void_p, C.c_double, C.c_int, C.c_int64, C.c_uint64
_PD, _PI, _PU64, _PP = C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_uint64), C.POINTER(C.c_void_p)


class MDError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code
        self.name = _ERRORS.get(code, str(code))


class md_run_options(C.Structure):
    _fields_ = [("thermostat", C.c_int), ("rescale_every", C.c_int), ("rescale_temperature", C.c_double),
                ("melt_until", C.c_int), ("melt_temperature", C.c_double), ("bussi_temperature", C.c_double),
                ("bussi_tau", C.c_double), ("bussi_r1", _PD), ("bussi_chi2", _PD), ("rdf", C.c_void_p),
                ("rdf_every", C.c_int), ("first_step", C.c_int64)]


class md_batch_options(C.Structure):
    _fields_ = [("epsilon", C.c_double), ("sigma", C.c_double), ("cutoff", C.c_double), ("skin", C.c_double),
                ("dt", C.c_double), ("precision", C.c_int), ("thermostat", C.c_int), ("rescale_every", C.c_int),
                ("bussi_tau", C.c_double), ("energy_every", C.c_int), ("chunk_steps", C.c_int),
                ("initial_capacity", C.c_int)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = C.CDLL(LIB_PATH)
    sig = {
        "md_last_error": (C.c_char_p, []), "md_version": (C.c_char_p, []), "md_device_count": (_I, []),
        "md_system_create": (_I, [_I64, _D, _I, _PP]), "md_system_destroy": (_I, [_P]),
        "md_system_size": (_I, [_P, C.POINTER(C.c_int64), _PD]),
        "md_system_upload": (_I, [_P, _PD, _PD, _PD, _PD, _PU64]),
        "md_system_download": (_I, [_P, _PD, _PD, _PD, _PD, _PU64]),
        "md_system_reorder": (_I, [_P, _PU64]), "md_kinetic_energy": (_I, [_P, _PD]),
        "md_temperature": (_I, [_P, _PD]), "md_state_hash": (_I, [_P, _PU64]),
        "md_scale_velocities": (_I, [_P, _D]), "md_rescale_velocities": (_I, [_P, _D]),
        "md_bussi_apply": (_I, [_P, _D, _D, _D, _D, _D]), "md_bussi_noise": (_I, [_U64, _I64, _I64, _PD, _PD]),
        "md_cells_create": (_I, [_D, _PP]), "md_cells_destroy": (_I, [_P]), "md_cells_build": (_I, [_P, _P, _PI]),
        "md_cells_download": (_I, [_P, _PI, _PU64, _PU64]),
        "md_nlist_create": (_I, [_D, _D, _I, _PP]), "md_nlist_destroy": (_I, [_P]),
        "md_nlist_build": (_I, [_P, _P]), "md_nlist_update": (_I, [_P, _P, _PI]),
        "md_nlist_info": (_I, [_P, _PU64, _PI, _PI, _PI]),
        "md_nlist_layout": (_I, [_P, _PI, _PI, _PI, _PI, _PI]),
        "md_nlist_set_force_variant": (_I, [_P, _I, _I]), "md_nlist_force_variant": (_I, [_P, _I, _PI]),
        "md_nlist_set_build_variant": (_I, [_P, _I]), "md_nlist_build_variant": (_I, [_P, _PI]),
        "md_nlist_download": (_I, [_P, _PU64, _PU64, _PU64, _PU64]),
        "md_nlist_fx32_rows": (_I, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), _PI, _PD]),
        "md_forcefield_create": (_I, [_D, _D, _D, _PP]), "md_forcefield_destroy": (_I, [_P]),
        "md_forcefield_shift": (_I, [_P, _PD]), "md_forcefield_set_precision": (_I, [_P, _I]),
        "md_forcefield_set_deterministic": (_I, [_P, _I]),
        "md_forces_list": (_I, [_P, _P, _P, _PD, _PD, _PD]), "md_forces_all_pairs": (_I, [_P, _P, _PD, _PD, _PD]),
        "md_step_list": (_I, [_P, _P, _P, _D, _PD, _PI]), "md_step_all_pairs": (_I, [_P, _P, _D, _PD]),
        "md_run": (_I, [_P, _P, _P, _D, _I64, C.POINTER(md_run_options), _PD, _PD, _PD]),
        "md_run_prepare": (_I, [_P, _P, _P, _D, _I64, C.POINTER(md_run_options), _I]),
        "md_system_set_graph": (_I, [_P, _I, _I]),
        "md_system_graph_info": (_I, [_P, C.POINTER(_I), _PU64, _PU64, _PU64]),
        "md_rdf_create": (_I, [_D, _I, _PP]), "md_rdf_destroy": (_I, [_P]), "md_rdf_sample": (_I, [_P, _P, _P]),
        "md_rdf_values": (_I, [_P, _PD, _PD, _PI]), "md_rdf_histogram": (_I, [_P, _PD]),
        "md_fcc_lattice": (_I, [_I, _D, _PD]), "md_initialize_velocities": (_I, [_P, _D, C.c_uint32]),
        "md_system_stream": (_I, [_P, _PP]), "md_system_synchronize": (_I, [_P]),
        "md_system_launch_count": (_I, [_P, _PU64]), "md_profile_enable": (_I, [_P, _I]),
        "md_profile_read": (_I, [_P, _PD, C.POINTER(C.c_int64)]),
        "md_forcefield_results": (_I, [_P, _PD, _PD]),
        "md_system_frame_by_id": (_I, [_P, _PD, _I]), "md_system_frame_wait": (_I, [_P]),
        "md_batch_create": (_I, [_I, _I, C.POINTER(C.c_int64), _PD, _PD, _PU64, _PD, _PD, _PD,
                                 C.POINTER(md_batch_options), _PP]),
        "md_batch_destroy": (_I, [_P]), "md_batch_info": (_I, [_P, _PI, C.POINTER(C.c_int64), _PI, _PU64]),
        "md_batch_stream": (_I, [_P, _PP]), "md_batch_run": (_I, [_P, _I64, _PD, _PD, _PD]),
        "md_batch_run_records": (_I, [_P, _I64, _PD, _PD, _PD, _PD]),
        "md_batch_set_thermostat": (_I, [_P, _I, _I, _D, _PD, _PU64]),
        "md_batch_energy": (_I, [_P, _PD, _PD, _PD, _PD]),
        "md_batch_download": (_I, [_P, _I, _PD, _PD, _PD, _PD, _PU64]),
        "md_batch_state_hash": (_I, [_P, _PU64]), "md_batch_rebuilds": (_I, [_P, _PU64]),
        "md_batch_set_force_variant": (_I, [_P, _I]), "md_batch_force_variant": (_I, [_P, _PI, _PI, _PI, _PI]),
        "md_batch_time_forces": (_I, [_P, _I, _PD]),
        "md_adjoint_create": (_I, [_I, _I64, _D, _PD, _PD, _PD, _D, _D, _D, _D, _D, _I, _I, _PP]),
        "md_adjoint_destroy": (_I, [_P]), "md_adjoint_set_parameters": (_I, [_P, _D, _D]),
        "md_adjoint_set_state": (_I, [_P, _PD, _PD]),
        "md_adjoint_forward": (_I, [_P, _PD, _PD, _PD, _PD, _PD]),
        "md_adjoint_backward": (_I, [_P, _D, _D, _PD, _PD, _PD, _PD]),
        "md_adjoint_info": (_I, [_P, C.POINTER(C.c_int64), _PI, _PI, _PI, _PU64]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


LIB = _load()


def _pd(a):
    return None if a is None else a.ctypes.data_as(_PD)


def _pu(a):
    return None if a is None else a.ctypes.data_as(_PU64)


def _pi(a):
    return None if a is None else a.ctypes.data_as(_PI)


def _check(code: int):
    if code != 0:
        raise MDError(code, LIB.md_last_error().decode())


def device_count() -> int:
    return LIB.md_device_count()


def bussi_noise(seed: int, n: int, count: int) -> tuple[np.ndarray, np.ndarray]:
    """The (r1, chi2) draws of `count` successive BussiThermostat::apply calls (src/Thermostat.cpp:48-51)."""
    r1 = np.zeros(count)
    chi2 = np.zeros(count)
    _check(LIB.md_bussi_noise(seed, n, count, _pd(r1), _pd(chi2)))
    return r1, chi2


def lattice_constant(density: float) -> float:
    """a = cbrt(4 / density), the FCC lattice constant md_sim uses (src/main.cpp:164-166)."""
    import math

    return math.cbrt(4.0 / density)


def fcc_lattice(cells: int, lattice_constant: float) -> np.ndarray:
    """createFCCLattice (src/Initialisation.cpp:7-44): (4 cells^3, 4) packed positions."""
    pos = np.zeros((4 * cells ** 3, 4))
    _check(LIB.md_fcc_lattice(cells, lattice_constant, _pd(pos)))
    return pos


def fcc_system(cells: int, density: float, temperature: float, seed: int = 42, device: int = 0) -> "System":
    """The FCC lattice of md_sim with seeded Maxwell-Boltzmann velocities (src/main.cpp:164-170)."""
    a = lattice_constant(density)
    s = System.from_arrays(fcc_lattice(cells, a), cells * a, device=device)
    s.initialize_velocities(temperature, seed)
    return s


class System:
    """System (include/System.hpp:12-136) resident on one GPU. pos is (n, 4): x, y, z, pad; vel/force are
    (3, n) component arrays, as the reference stores them."""

    def __init__(self, n: int, box_length: float, device: int = 0):
        h = C.c_void_p()
        _check(LIB.md_system_create(n, box_length, device, C.byref(h)))
        self.h = h
        self.n = n
        self.box = float(box_length)

    @classmethod
    def from_arrays(cls, pos, box_length, vel=None, mass=None, force=None, ids=None, device=0) -> "System":
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        if pos.ndim == 2 and pos.shape[1] == 3:
            pos = np.concatenate([pos, np.zeros((pos.shape[0], 1))], axis=1)
        s = cls(pos.shape[0], box_length, device)
        s.upload(pos=pos, vel=vel, mass=mass, force=force, ids=ids)
        return s

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            LIB.md_system_destroy(h)
            self.h = None

    def upload(self, pos=None, vel=None, force=None, mass=None, ids=None):
        def f64(a, shape):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float64)
            assert a.size == int(np.prod(shape)), (a.shape, shape)
            return a
        pos, vel, force, mass = f64(pos, (self.n, 4)), f64(vel, (3, self.n)), f64(force, (3, self.n)), f64(mass, (self.n,))
        ids = None if ids is None else np.ascontiguousarray(ids, dtype=np.uint64)
        _check(LIB.md_system_upload(self.h, _pd(pos), _pd(vel), _pd(force), _pd(mass), _pu(ids)))

    def frame_by_id(self) -> np.ndarray:
        """(n, 6) array of (x, y, z, vx, vy, vz) in id order, gathered on the device (writeXyzFrame's data)."""
        out = np.zeros((self.n, 6))
        _check(LIB.md_system_frame_by_id(self.h, _pd(out), 1))
        return out

    def download(self):
        pos = np.zeros((self.n, 4))
        vel = np.zeros((3, self.n))
        force = np.zeros((3, self.n))
        mass = np.zeros(self.n)
        ids = np.zeros(self.n, dtype=np.uint64)
        _check(LIB.md_system_download(self.h, _pd(pos), _pd(vel), _pd(force), _pd(mass), _pu(ids)))
        return dict(pos=pos, vel=vel, force=force, mass=mass, ids=ids)

    def positions(self) -> np.ndarray:
        pos = np.zeros((self.n, 4))
        _check(LIB.md_system_download(self.h, _pd(pos), None, None, None, None))
        return pos

    def velocities(self) -> np.ndarray:
        vel = np.zeros((3, self.n))
        _check(LIB.md_system_download(self.h, None, _pd(vel), None, None, None))
        return vel

    def forces(self) -> np.ndarray:
        f = np.zeros((3, self.n))
        _check(LIB.md_system_download(self.h, None, None, _pd(f), None, None))
        return f

    def ids(self) -> np.ndarray:
        ids = np.zeros(self.n, dtype=np.uint64)
        _check(LIB.md_system_download(self.h, None, None, None, None, _pu(ids)))
        return ids

    def reorder(self, order):
        o = np.ascontiguousarray(order, dtype=np.uint64)
        _check(LIB.md_system_reorder(self.h, _pu(o)))

    def kinetic_energy(self) -> float:
        x = C.c_double()
        _check(LIB.md_kinetic_energy(self.h, C.byref(x)))
        return x.value

    def temperature(self) -> float:
        x = C.c_double()
        _check(LIB.md_temperature(self.h, C.byref(x)))
        return x.value

    def state_hash(self) -> int:
        x = C.c_uint64()
        _check(LIB.md_state_hash(self.h, C.byref(x)))
        return x.value

    def scale_velocities(self, scale: float):
        _check(LIB.md_scale_velocities(self.h, scale))

    def rescale_velocities(self, target: float):
        """rescaleVelocities (src/Thermostat.cpp:17-30)."""
        _check(LIB.md_rescale_velocities(self.h, target))

    def initialize_velocities(self, temperature: float, seed: int):
        """initializeVelocities (src/Initialisation.cpp:47-76)."""
        _check(LIB.md_initialize_velocities(self.h, temperature, seed))

    @property
    def stream(self) -> int:
        """The cudaStream_t (as an integer) all of this system's work is queued on."""
        p = C.c_void_p()
        _check(LIB.md_system_stream(self.h, C.byref(p)))
        return p.value or 0

    def synchronize(self):
        _check(LIB.md_system_synchronize(self.h))

    @property
    def launch_count(self) -> int:
        x = C.c_uint64()
        _check(LIB.md_system_launch_count(self.h, C.byref(x)))
        return x.value

    def set_graph(self, chunk_steps: int, test_rerun: bool = False):
        """md_run's CUDA-graph chunk length (0: every step from the host); test_rerun is a test switch that makes
        every device rebuild report an overflow, so chunks with rebuilds rerun on the host path
        (md_system_set_graph)."""
        _check(LIB.md_system_set_graph(self.h, chunk_steps, GRAPH_TEST_RERUN if test_rerun else 0))

    def graph_info(self) -> dict:
        c, g, l, r = C.c_int(), C.c_uint64(), C.c_uint64(), C.c_uint64()
        _check(LIB.md_system_graph_info(self.h, C.byref(c), C.byref(g), C.byref(l), C.byref(r)))
        return {"chunk_steps": c.value, "graphs": g.value, "launches": l.value, "recoveries": r.value}

    def profile(self, enable: bool):
        _check(LIB.md_profile_enable(self.h, int(enable)))

    def profile_read(self) -> tuple[float, int]:
        """(total ms, launches) of the list force kernel since profile(True)."""
        ms, k = C.c_double(), C.c_int64()
        _check(LIB.md_profile_read(self.h, C.byref(ms), C.byref(k)))
        return ms.value, k.value

    def bussi_apply(self, temperature: float, tau: float, dt: float, r1: float, chi2: float):
        """BussiThermostat::apply (src/Thermostat.cpp:36-58) with the draws given (see bussi_noise)."""
        _check(LIB.md_bussi_apply(self.h, temperature, tau, dt, r1, chi2))


class CellList:
    """CellList (include/CellList.hpp:11-50)."""

    def __init__(self, min_cell_size: float):
        h = C.c_void_p()
        _check(LIB.md_cells_create(min_cell_size, C.byref(h)))
        self.h = h
        self.ncps = 0
        self.n = 0

    def __del__(self):
        if getattr(self, "h", None):
            LIB.md_cells_destroy(self.h)
            self.h = None

    def build(self, system: System) -> int:
        x = C.c_int()
        _check(LIB.md_cells_build(self.h, system.h, C.byref(x)))
        self.ncps = x.value
        self.n = system.n
        return self.ncps

    def download(self):
        cell = np.zeros(self.n, dtype=np.int32)
        start = np.zeros(self.ncps ** 3 + 1, dtype=np.uint64)
        parts = np.zeros(self.n, dtype=np.uint64)
        _check(LIB.md_cells_download(self.h, _pi(cell), _pu(start), _pu(parts)))
        return cell, start, parts


class NeighbourList:
    """NeighbourList (include/NeighbourList.hpp:10-76)."""

    def __init__(self, cutoff: float, skin: float, reverse_index: bool = False):
        h = C.c_void_p()
        _check(LIB.md_nlist_create(cutoff, skin, int(reverse_index), C.byref(h)))
        self.h = h
        self.reverse_index = reverse_index
        self.n = 0

    def __del__(self):
        if getattr(self, "h", None):
            LIB.md_nlist_destroy(self.h)
            self.h = None

    def build(self, system: System):
        _check(LIB.md_nlist_build(self.h, system.h))
        self.n = system.n

    def update(self, system: System) -> bool:
        r = C.c_int()
        _check(LIB.md_nlist_update(self.h, system.h, C.byref(r)))
        self.n = system.n
        return bool(r.value)

    def _info(self):
        p, rb, nc, rv = C.c_uint64(), C.c_int(), C.c_int(), C.c_int()
        _check(LIB.md_nlist_info(self.h, C.byref(p), C.byref(rb), C.byref(nc), C.byref(rv)))
        return p.value, rb.value, nc.value, bool(rv.value)

    @property
    def pair_count(self) -> int:
        return self._info()[0]

    @property
    def rebuild_count(self) -> int:
        return self._info()[1]

    @property
    def cells_per_side(self) -> int:
        return self._info()[2]

    def set_force_variant(self, precision: int, variant: int):
        """-1 autotunes the list force kernel; 0 pins global gathers; 1 pins the shared-memory tile kernel; 2 pins
        prefetching global gathers (FP64: branch-free quads); for the float modes 3 pins variant 2 with capped
        registers and 4 the same on a resident grid. Every variant gives the same bits."""
        _check(LIB.md_nlist_set_force_variant(self.h, precision, variant))

    def force_variant(self, precision: int) -> int:
        v = C.c_int()
        _check(LIB.md_nlist_force_variant(self.h, precision, C.byref(v)))
        return v.value

    def set_build_variant(self, variant: int):
        """-1 uses the tile build where the list has tiles; 0 pins one thread per particle, 1 the tiles."""
        _check(LIB.md_nlist_set_build_variant(self.h, variant))

    def build_variant(self) -> int:
        v = C.c_int()
        _check(LIB.md_nlist_build_variant(self.h, C.byref(v)))
        return v.value

    def layout(self) -> dict:
        """Tile geometry and row capacity of the last build (diagnostics)."""
        v = [C.c_int() for _ in range(5)]
        _check(LIB.md_nlist_layout(self.h, *[C.byref(x) for x in v]))
        return dict(zip(("use_tiles", "segment_cells", "segments_per_column", "max_staged", "row_capacity"),
                        (x.value for x in v)))

    def download(self):
        P, _, _, rev = self._info()
        n = self.n
        off = np.zeros(n + 1, dtype=np.uint64)
        nb = np.zeros(P, dtype=np.uint64)
        roff = np.zeros(n + 1, dtype=np.uint64) if rev else None
        rp = np.zeros(P, dtype=np.uint64) if rev else None
        _check(LIB.md_nlist_download(self.h, _pu(off), _pu(nb), _pu(roff), _pu(rp)))
        return dict(offsets=off, neighbours=nb, rev_offsets=roff, rev_pairs=rp)

    def fx32_rows(self):
        """MD_PREC_FX32's near and far rows of the last build (diagnostics): entries j | code << 27 per row in
        order (near: 16 slots, far: row_capacity slots), (near groups, far groups) per particle and the squared
        radius that classified them. Raises until MD_PREC_FX32 forces were computed on this build."""
        n, cap = self.n, self.layout()["row_capacity"]
        near = np.zeros((n, 16), dtype=np.uint32)
        far = np.zeros((n, cap), dtype=np.uint32)
        groups = np.zeros((n, 2), dtype=np.int32)
        near2 = C.c_double()
        u32 = C.POINTER(C.c_uint32)
        _check(LIB.md_nlist_fx32_rows(self.h, near.ctypes.data_as(u32), far.ctypes.data_as(u32), _pi(groups),
                                      C.byref(near2)))
        return dict(near=near, far=far, groups=groups, near2=near2.value)


class LennardJonesForceField:
    """LennardJonesForceField (include/Forcefield.hpp:6-78)."""

    def __init__(self, epsilon: float, sigma: float, cutoff: float, precision: int = PREC_FP64):
        h = C.c_void_p()
        _check(LIB.md_forcefield_create(epsilon, sigma, cutoff, C.byref(h)))
        self.h = h
        self.virial = 0.0
        self.inside_pairs = 0.0
        self.set_precision(precision)

    def __del__(self):
        if getattr(self, "h", None):
            LIB.md_forcefield_destroy(self.h)
            self.h = None

    @property
    def energy_shift(self) -> float:
        x = C.c_double()
        _check(LIB.md_forcefield_shift(self.h, C.byref(x)))
        return x.value

    def set_precision(self, precision: int):
        _check(LIB.md_forcefield_set_precision(self.h, precision))

    def set_mixed_precision(self, mixed: bool):
        """setMixedPrecision (include/Forcefield.hpp:39-41): float pair arithmetic, fixed-point accumulation."""
        self.set_precision(PREC_FP32FX if mixed else PREC_FP64)

    def set_deterministic(self, deterministic: bool):
        _check(LIB.md_forcefield_set_deterministic(self.h, int(deterministic)))

    def fetch_results(self):
        """getVirial / getInsidePairs of the last evaluation, steps included (md_forcefield_results)."""
        w, ins = C.c_double(), C.c_double()
        _check(LIB.md_forcefield_results(self.h, C.byref(w), C.byref(ins)))
        self.virial, self.inside_pairs = w.value, ins.value

    def compute_forces(self, system: System, neighbour_list: NeighbourList | None = None) -> float:
        pe, w, ins = C.c_double(), C.c_double(), C.c_double()
        if neighbour_list is None:
            _check(LIB.md_forces_all_pairs(self.h, system.h, C.byref(pe), C.byref(w), C.byref(ins)))
        else:
            _check(LIB.md_forces_list(self.h, system.h, neighbour_list.h, C.byref(pe), C.byref(w), C.byref(ins)))
        self.virial, self.inside_pairs = w.value, ins.value
        return pe.value


class RadialDistribution:
    """RadialDistribution (include/RadialDistribution.hpp:8-29)."""

    def __init__(self, r_max: float, bins: int):
        h = C.c_void_p()
        _check(LIB.md_rdf_create(r_max, bins, C.byref(h)))
        self.h = h
        self.bins = bins

    def __del__(self):
        if getattr(self, "h", None):
            LIB.md_rdf_destroy(self.h)
            self.h = None

    def sample(self, system: System, neighbour_list: NeighbourList):
        _check(LIB.md_rdf_sample(self.h, system.h, neighbour_list.h))

    def radii(self) -> np.ndarray:
        r = np.zeros(self.bins)
        _check(LIB.md_rdf_values(self.h, _pd(r), None, None))
        return r

    def values(self) -> np.ndarray:
        g = np.zeros(self.bins)
        _check(LIB.md_rdf_values(self.h, None, _pd(g), None))
        return g

    def histogram(self) -> np.ndarray:
        h = np.zeros(self.bins)
        _check(LIB.md_rdf_histogram(self.h, _pd(h)))
        return h


class VelocityVerletIntegrator:
    """VelocityVerletIntegrator (include/Integrator.hpp:7-29)."""

    def __init__(self, dt: float):
        self.dt = dt
        self.last_rebuilt = False

    def step(self, system: System, force_field: LennardJonesForceField,
             neighbour_list: NeighbourList | None = None) -> float:
        pe = C.c_double()
        if neighbour_list is None:
            _check(LIB.md_step_all_pairs(system.h, force_field.h, self.dt, C.byref(pe)))
        else:
            r = C.c_int()
            _check(LIB.md_step_list(system.h, force_field.h, neighbour_list.h, self.dt, C.byref(pe), C.byref(r)))
            self.last_rebuilt = bool(r.value)
            neighbour_list.n = system.n
        force_field.fetch_results()
        return pe.value

    def run(self, system: System, force_field: LennardJonesForceField, neighbour_list: NeighbourList, n_steps: int,
            thermostat: str = "none", rescale_every: int = 10, rescale_temperature: float = 0.0,
            melt_until: int = 0, melt_temperature: float = 2.0, bussi_temperature: float = 0.0,
            bussi_tau: float = 0.5, bussi_r1=None, bussi_chi2=None, rdf: RadialDistribution | None = None,
            rdf_every: int = 10, first_step: int = 1, record: bool = True):
        """n_steps device-resident steps (md_run). Returns per-step (pe, ke, virial) arrays when record."""
        o, keep = self._options(thermostat, rescale_every, rescale_temperature, melt_until, melt_temperature,
                                bussi_temperature, bussi_tau, bussi_r1, bussi_chi2, rdf, rdf_every, first_step)
        pe = np.zeros(n_steps) if record else None
        ke = np.zeros(n_steps) if record else None
        w = np.zeros(n_steps) if record else None
        _check(LIB.md_run(system.h, force_field.h, neighbour_list.h, self.dt, n_steps, C.byref(o), _pd(pe), _pd(ke),
                          _pd(w)))
        neighbour_list.n = system.n
        return pe, ke, w

    def prepare(self, system: System, force_field: LennardJonesForceField, neighbour_list: NeighbourList,
                n_steps: int, thermostat: str = "none", rescale_every: int = 10, rescale_temperature: float = 0.0,
                melt_until: int = 0, melt_temperature: float = 2.0, bussi_temperature: float = 0.0,
                bussi_tau: float = 0.5, rdf: RadialDistribution | None = None, rdf_every: int = 10,
                first_step: int = 1, record: bool = True):
        """Capture the CUDA graphs run() would launch with these arguments, without running (md_run_prepare)."""
        r1 = np.zeros(max(n_steps, 1))
        o, keep = self._options(thermostat, rescale_every, rescale_temperature, melt_until, melt_temperature,
                                bussi_temperature, bussi_tau, r1, r1, rdf, rdf_every, first_step)
        _check(LIB.md_run_prepare(system.h, force_field.h, neighbour_list.h, self.dt, n_steps, C.byref(o),
                                  3 if record else 0))

    @staticmethod
    def _options(thermostat, rescale_every, rescale_temperature, melt_until, melt_temperature, bussi_temperature,
                 bussi_tau, bussi_r1, bussi_chi2, rdf, rdf_every, first_step):
        o = md_run_options()
        o.thermostat = {"none": 0, "rescale": 1, "bussi": 2}[thermostat]
        o.rescale_every = rescale_every
        o.rescale_temperature = rescale_temperature
        o.melt_until = melt_until
        o.melt_temperature = melt_temperature
        o.bussi_temperature = bussi_temperature
        o.bussi_tau = bussi_tau
        keep = []
        if thermostat == "bussi":
            r1 = np.ascontiguousarray(bussi_r1, dtype=np.float64)
            chi2 = np.ascontiguousarray(bussi_chi2, dtype=np.float64)
            keep += [r1, chi2]
            o.bussi_r1, o.bussi_chi2 = _pd(r1), _pd(chi2)
        o.rdf = rdf.h if rdf is not None else None
        o.rdf_every = rdf_every
        o.first_step = first_step
        return o, keep


class Batch:
    """Many independent replicas advanced together (md_batch_*): each replica is the reference's System with
    NeighbourList(cutoff, skin, True), a deterministic LennardJonesForceField and VelocityVerletIntegrator, plus
    an optional thermostat per replica; the reference has no batched class, so this stands for a loop over
    systems. `systems` is a list of (pos (n, 4), box_length, vel (3, n) or None, mass (n,) or None) tuples."""

    def __init__(self, systems, cutoff=2.5, skin=0.3, dt=0.005, epsilon=1.0, sigma=1.0, precision=PREC_FP64,
                 thermostat="none", temperatures=None, seeds=None, rescale_every=10, bussi_tau=0.1,
                 energy_every=0, chunk_steps=0, initial_capacity=0, device=0):
        self.replicas = len(systems)
        n = np.array([len(p) for p, *_ in systems], dtype=np.int64)
        box = np.array([float(b) for _, b, *_ in systems])
        pos = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.float64).reshape(-1, 4) for p, *_ in systems]))
        vel = np.ascontiguousarray(np.concatenate([
            (np.zeros(3 * len(p)) if v is None else np.asarray(v, dtype=np.float64).reshape(-1))
            for p, _, v, *_ in systems]))
        mass = np.ascontiguousarray(np.concatenate([
            (np.ones(len(p)) if m is None else np.asarray(m, dtype=np.float64)) for p, _, _, m in systems]))
        o = md_batch_options()
        o.epsilon, o.sigma, o.cutoff, o.skin, o.dt = epsilon, sigma, cutoff, skin, dt
        o.precision = precision
        o.thermostat = {"none": 0, "rescale": 1, "bussi": 2}[thermostat]
        o.rescale_every, o.bussi_tau = rescale_every, bussi_tau
        o.energy_every, o.chunk_steps, o.initial_capacity = energy_every, chunk_steps, initial_capacity
        temps = None if temperatures is None else np.ascontiguousarray(temperatures, dtype=np.float64)
        sd = None if seeds is None else np.ascontiguousarray(seeds, dtype=np.uint64)
        h = C.c_void_p()
        _check(LIB.md_batch_create(device, self.replicas, n.ctypes.data_as(C.POINTER(C.c_int64)), _pd(box),
                                   _pd(temps), _pu(sd), _pd(pos), _pd(vel), _pd(mass), C.byref(o), C.byref(h)))
        self.h = h
        self.n = n
        self.box = box
        self.energy_every = energy_every

    def __del__(self):
        if getattr(self, "h", None):
            LIB.md_batch_destroy(self.h)
            self.h = None

    def info(self) -> dict:
        r, cap = C.c_int(), C.c_int()
        atoms, launches = C.c_int64(), C.c_uint64()
        _check(LIB.md_batch_info(self.h, C.byref(r), C.byref(atoms), C.byref(cap), C.byref(launches)))
        return dict(replicas=r.value, atoms=atoms.value, capacity=cap.value, launches=launches.value)

    def run(self, n_steps: int, record: bool = True, inside: bool = False):
        """n_steps steps of every replica; returns (pe, virial, ke) arrays of shape (n_steps // energy_every,
        replicas) when energy_every > 0 and record, plus the inside-cutoff pair counts with inside, else None."""
        rows = n_steps // self.energy_every if self.energy_every > 0 and record else 0
        if rows == 0:
            _check(LIB.md_batch_run(self.h, n_steps, None, None, None))
            return None
        pe, w, ke, ins = (np.zeros((rows, self.replicas)) for _ in range(4))
        _check(LIB.md_batch_run_records(self.h, n_steps, _pd(pe), _pd(w), _pd(ke), _pd(ins) if inside else None))
        return (pe, w, ke, ins) if inside else (pe, w, ke)

    def set_thermostat(self, thermostat: str, temperatures=None, rescale_every: int = 10, bussi_tau: float = 0.5,
                       seeds=None):
        """Switch the thermostat between runs (md_batch_set_thermostat): "none", "rescale" (every rescale_every
        steps to temperatures[r]) or "bussi" (coupling time bussi_tau, generators started afresh from seeds)."""
        temps = None if temperatures is None else np.ascontiguousarray(temperatures, dtype=np.float64)
        sd = None if seeds is None else np.ascontiguousarray(seeds, dtype=np.uint64)
        self.thermostat = thermostat
        _check(LIB.md_batch_set_thermostat(self.h, {"none": 0, "rescale": 1, "bussi": 2}[thermostat], rescale_every,
                                           bussi_tau, _pd(temps), _pu(sd)))

    def energy(self):
        """(pe, virial, ke, inside) arrays over replicas for the current state."""
        out = [np.zeros(self.replicas) for _ in range(4)]
        _check(LIB.md_batch_energy(self.h, *(_pd(a) for a in out)))
        return tuple(out)

    def download(self, replica: int) -> dict:
        k = int(self.n[replica])
        pos, vel, force, mass = np.zeros((k, 4)), np.zeros((3, k)), np.zeros((3, k)), np.zeros(k)
        ids = np.zeros(k, dtype=np.uint64)
        _check(LIB.md_batch_download(self.h, replica, _pd(pos), _pd(vel), _pd(force), _pd(mass), _pu(ids)))
        return dict(pos=pos, vel=vel, force=force, mass=mass, ids=ids)

    def state_hashes(self) -> np.ndarray:
        h = np.zeros(self.replicas, dtype=np.uint64)
        _check(LIB.md_batch_state_hash(self.h, _pu(h)))
        return h

    def rebuilds(self) -> np.ndarray:
        r = np.zeros(self.replicas, dtype=np.uint64)
        _check(LIB.md_batch_rebuilds(self.h, _pu(r)))
        return r

    def set_force_variant(self, variant: int):
        _check(LIB.md_batch_set_force_variant(self.h, variant))

    def force_variant(self) -> dict:
        v, c, apb, tpa = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _check(LIB.md_batch_force_variant(self.h, C.byref(v), C.byref(c), C.byref(apb), C.byref(tpa)))
        return dict(variant=v.value, count=c.value, particles_per_block=apb.value, threads_per_particle=tpa.value)

    def time_forces(self, reps: int = 10) -> float:
        ms = C.c_double()
        _check(LIB.md_batch_time_forces(self.h, reps, C.byref(ms)))
        return ms.value

    def stream(self) -> int:
        p = C.c_void_p()
        _check(LIB.md_batch_stream(self.h, C.byref(p)))
        return p.value or 0


class Adjoint:
    """Trajectory adjoint (md_adjoint_*): J = g_pe * mean U + g_pressure * mean P over `steps` NVE steps of the
    system (pos (n, 4), box, vel (3, n), mass (n,) or None), differentiated with respect to epsilon, sigma and
    the initial positions and velocities. forward() -> (mean U, mean P); backward(g_pe, g_pressure) -> dict of
    gradients (d_pos and d_vel as (3, n) component arrays, like the velocities)."""

    def __init__(self, pos, box, vel, mass=None, epsilon=1.0, sigma=1.0, cutoff=2.5, skin=0.3, dt=0.005, steps=200,
                 checkpoint_every=20, device=0):
        p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 4)
        v = np.ascontiguousarray(vel, dtype=np.float64).reshape(3, -1)
        m = None if mass is None else np.ascontiguousarray(mass, dtype=np.float64)
        self.n, self.box, self.steps = len(p), float(box), steps
        h = C.c_void_p()
        _check(LIB.md_adjoint_create(device, self.n, self.box, _pd(p), _pd(v), _pd(m), epsilon, sigma, cutoff, skin,
                                     dt, steps, checkpoint_every, C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            LIB.md_adjoint_destroy(self.h)
            self.h = None

    def set_parameters(self, epsilon: float, sigma: float):
        _check(LIB.md_adjoint_set_parameters(self.h, float(epsilon), float(sigma)))

    def set_state(self, pos=None, vel=None):
        p = None if pos is None else np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 4)
        v = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64).reshape(3, -1)
        _check(LIB.md_adjoint_set_state(self.h, _pd(p), _pd(v)))

    def forward(self, record: bool = False):
        mu, mp = C.c_double(), C.c_double()
        if not record:
            _check(LIB.md_adjoint_forward(self.h, C.byref(mu), C.byref(mp), None, None, None))
            return mu.value, mp.value
        u, w, k = np.zeros(self.steps), np.zeros(self.steps), np.zeros(self.steps)
        _check(LIB.md_adjoint_forward(self.h, C.byref(mu), C.byref(mp), _pd(u), _pd(w), _pd(k)))
        return mu.value, mp.value, u, w, k

    def backward(self, g_pe: float, g_pressure: float) -> dict:
        de, ds = C.c_double(), C.c_double()
        dp, dv = np.zeros((3, self.n)), np.zeros((3, self.n))
        _check(LIB.md_adjoint_backward(self.h, float(g_pe), float(g_pressure), C.byref(de), C.byref(ds), _pd(dp),
                                       _pd(dv)))
        return dict(d_epsilon=de.value, d_sigma=ds.value, d_pos=dp, d_vel=dv)

    def info(self) -> dict:
        n, st, ev, rb, la = C.c_int64(), C.c_int(), C.c_int(), C.c_int(), C.c_uint64()
        _check(LIB.md_adjoint_info(self.h, C.byref(n), C.byref(st), C.byref(ev), C.byref(rb), C.byref(la)))
        return dict(n=n.value, steps=st.value, checkpoint_every=ev.value, rebuilds=rb.value, launches=la.value)


def trajectory_observables(epsilon, sigma, pos, engine: Adjoint):
    """torch.autograd.Function over an Adjoint engine: (epsilon, sigma, pos (n, 3)) tensors in float64 ->
    tensor([mean U, mean P]); backward returns the engine's gradients. The initial velocities are the engine's."""
    import torch

    class _TrajectoryObservables(torch.autograd.Function):
        @staticmethod
        def forward(ctx, eps, sig, p):
            engine.set_parameters(float(eps), float(sig))
            p4 = np.zeros((engine.n, 4))
            p4[:, :3] = p.detach().cpu().numpy()
            engine.set_state(pos=p4)
            u, pr = engine.forward()
            return torch.tensor([u, pr], dtype=torch.float64)

        @staticmethod
        def backward(ctx, g):
            r = engine.backward(float(g[0]), float(g[1]))
            return (torch.tensor(r["d_epsilon"], dtype=torch.float64), torch.tensor(r["d_sigma"], dtype=torch.float64),
                    torch.from_numpy(np.ascontiguousarray(r["d_pos"].T)))

    return _TrajectoryObservables.apply(epsilon, sigma, pos)

