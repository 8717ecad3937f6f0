"""CPU-side checks of the C-ABI library (no GPU needed): it loads, exports every entry point that
include/md_b200.h declares, its host-only entry points match the oracle bit for bit, and device entry
points fail loudly (an error code, never a silent CPU result) when no GPU is present."""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include")))
           if f.endswith(".h")]
LIB = os.path.join(ROOT, "molecular-dynamics_b200", "libmdgpu.so")


def declared_functions():
    names = []
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(md_[a-z0-9_]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "md_system_create" in names and "md_run" in names and len(names) > 40


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_library_is_sm100a_only():
    out = open(os.path.join(ROOT, "molecular-dynamics_b200", "csrc", "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in out


def test_host_entry_points_match_oracle(oracle):
    import mdgpu

    a = mdgpu.lattice_constant(0.8442)
    from oracle.oracle import fcc_box
    a_o, _ = fcc_box(6, 0.8442)
    assert a == a_o
    assert np.array_equal(mdgpu.fcc_lattice(6, a), oracle.fcc(6, a))
    r1, chi2 = mdgpu.bussi_noise(7, 500, 64)
    r1o, chi2o = oracle.bussi_noise(7, 500, 64)
    assert np.array_equal(r1, r1o) and np.array_equal(chi2, chi2o)


def test_device_calls_fail_loudly_without_gpu():
    import mdgpu

    if mdgpu.device_count() > 0:
        pytest.skip("a GPU is present; this checks the CPU-only host")
    with pytest.raises(mdgpu.MDError) as e:
        mdgpu.System(10, 5.0)
    assert e.value.name == "MD_ERR_NO_DEVICE"


def test_argument_errors_are_reported():
    import mdgpu

    with pytest.raises(mdgpu.MDError) as e:
        mdgpu.NeighbourList(-1.0, 0.3)
    assert e.value.name == "MD_ERR_INVALID"
    with pytest.raises(mdgpu.MDError):
        mdgpu.RadialDistribution(1.0, 0)
    # force variants: 0-4 for the float modes, 0-2 for FP64, 0 for FX64, -1 autotunes
    nl = mdgpu.NeighbourList(2.5, 0.3)
    for prec, v in ((mdgpu.PREC_FP32FX, 5), (mdgpu.PREC_FP32, -2), (mdgpu.PREC_FP64, 3), (mdgpu.PREC_FX64, 1)):
        with pytest.raises(mdgpu.MDError) as e:
            nl.set_force_variant(prec, v)
        assert e.value.name == "MD_ERR_INVALID"
    for prec, v in ((mdgpu.PREC_FP32FX, 4), (mdgpu.PREC_FP32, 3), (mdgpu.PREC_FP64, 2), (mdgpu.PREC_FX64, 0),
                    (mdgpu.PREC_FP32FX, -1)):
        nl.set_force_variant(prec, v)


def test_batch_geometry_and_option_errors():
    """md_batch_create validates every replica before touching a device: the reference's geometry errors
    (src/Forcefield.cpp:18-22, src/NeighbourList.cpp:57-59) per replica, then bad options."""
    import mdgpu

    a = mdgpu.lattice_constant(0.8442)
    ok = (mdgpu.fcc_lattice(6, a), 6 * a, None, None)
    small = (mdgpu.fcc_lattice(3, a), 3 * a, None, None)  # L = 5.04 < 2 (r_c + skin)
    with pytest.raises(mdgpu.MDError) as e:
        mdgpu.Batch([ok, small], cutoff=2.5, skin=0.3)
    assert e.value.name == "MD_ERR_LIST_RADIUS" and "replica 1" in str(e.value)
    with pytest.raises(mdgpu.MDError) as e:
        mdgpu.Batch([small], cutoff=2.6, skin=0.1)
    assert e.value.name == "MD_ERR_CUTOFF"
    with pytest.raises(mdgpu.MDError) as e:
        mdgpu.Batch([ok], thermostat="bussi", temperatures=[1.0])  # no seeds
    assert e.value.name == "MD_ERR_INVALID"
    if mdgpu.device_count() == 0:
        with pytest.raises(mdgpu.MDError) as e:
            mdgpu.Batch([ok])
        assert e.value.name == "MD_ERR_NO_DEVICE"
