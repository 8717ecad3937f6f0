"""The list path at the headline size, N = 4,000,000 (FCC 100^3 x 4, density 0.8442), through properties that do
not need the oracle to run at that size: every force-kernel variant and both list builds give the same bits, the
FP64 forces sum to zero (tests/test_forcefield.cpp:103-119), and the reduced-precision modes stay within their
error bounds of the FP64 path (FX64 and FX32: every particle within 1e-6 of the rms force and 99 % of particles
within 1e-6 of their own force; FP32FX: the reference's mixed-precision tolerance,
tests/test_forcefield.cpp:123-149). The state is a liquid: 60 steps of the bench's
melt/rescale schedule from the lattice.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RC, SKIN = 2.5, 0.3


@pytest.fixture(scope="module")
def liquid_4m(md):
    s = md.fcc_system(100, 0.8442, 0.71, seed=42)
    nl = md.NeighbourList(RC, SKIN)
    nl.build(s)
    ff = md.LennardJonesForceField(1.0, 1.0, RC, precision=md.PREC_FP32FX)
    ff.compute_forces(s, nl)
    md.VelocityVerletIntegrator(0.005).run(s, ff, nl, 60, thermostat="rescale", rescale_every=10,
                                           rescale_temperature=0.71, melt_until=30, melt_temperature=2.0,
                                           record=False)
    st = s.download()
    assert s.n == 4_000_000
    return st, s.box


def forces(md, state, precision, variant=-1, build_variant=-1):
    """Forces, PE, virial and inside count of `state` after a fresh list build (the build's reorder gives every
    call the same storage order)."""
    st, box = state
    s = md.System.from_arrays(st["pos"], box, vel=st["vel"])
    nl = md.NeighbourList(RC, SKIN, reverse_index=precision == md.PREC_FP64)
    nl.set_build_variant(build_variant)
    if variant >= 0:
        nl.set_force_variant(precision, variant)
    nl.build(s)
    ff = md.LennardJonesForceField(1.0, 1.0, RC, precision=precision)
    if precision == md.PREC_FP64:
        ff.set_deterministic(True)
    pe = ff.compute_forces(s, nl)
    if variant >= 0:
        assert nl.force_variant(precision) == variant
    return s.forces(), pe, ff.virial, ff.inside_pairs, nl.pair_count


def test_fp64_variants_bit_identical_and_total_force_zero(md, liquid_4m):
    f0, pe0, w0, in0, p0 = forces(md, liquid_4m, md.PREC_FP64, 0)
    f2, pe2, w2, in2, p2 = forces(md, liquid_4m, md.PREC_FP64, 2)
    assert np.array_equal(f0, f2) and pe0 == pe2 and w0 == w2 and in0 == in2 and p0 == p2
    assert np.abs(f0.sum(axis=1)).max() < 1e-6
    assert 35.0 < p0 / f0.shape[1] < 42.0  # about 37.5 half-list pairs per atom in the liquid at r_l = 2.8


def test_float_variants_and_builds_bit_identical(md, liquid_4m):
    ref = forces(md, liquid_4m, md.PREC_FP32FX, 2)
    for variant, build in ((4, -1), (0, -1), (3, -1), (4, 0)):
        f, pe, w, ins, p = forces(md, liquid_4m, md.PREC_FP32FX, variant, build)
        assert np.array_equal(f, ref[0]), (variant, build)
        assert (pe, w, ins, p) == ref[1:], (variant, build)


def test_reduced_precision_within_bounds_of_fp64(md, liquid_4m):
    f64, pe64, w64, in64, _ = forces(md, liquid_4m, md.PREC_FP64)
    rms = float(np.sqrt((f64 ** 2).sum(axis=0).mean()))
    fx, pex, wx, inx, _ = forces(md, liquid_4m, md.PREC_FX64)
    dfx = np.sqrt(((fx - f64) ** 2).sum(axis=0))
    assert dfx.max() < 1e-6 * rms, dfx.max() / rms
    # the virial cancels (terms of both signs), so its relative error runs higher than the energy's
    assert abs(pex - pe64) < 1e-8 * abs(pe64) and abs(wx - w64) < 1e-5 * abs(w64) and inx == in64
    f32, pe32, w32, in32, _ = forces(md, liquid_4m, md.PREC_FP32FX)
    assert np.abs(f32 - f64).max() < 1e-5 * np.abs(f64).max()
    assert abs(pe32 - pe64) < 1e-5 * abs(pe64) and abs(w32 - w64) < 1e-4 * abs(w64) and in32 == in64


def test_fx32_meets_the_per_particle_bound_at_4m(md, liquid_4m):
    """MD_PREC_FX32 at the headline size: max |dF_i| <= 1e-6 rms |F| and >= 99 % of particles with
    |dF_i| <= 1e-6 |F_i| against the FP64 path, PE within 1e-6 and the virial within 1e-5 relative, the same
    inside count, and a bit-identical repeat."""
    f64, pe64, w64, in64, _ = forces(md, liquid_4m, md.PREC_FP64)
    f, pe, w, ins, _ = forces(md, liquid_4m, md.PREC_FX32)
    d = np.sqrt(((f - f64) ** 2).sum(axis=0))
    mag = np.sqrt((f64 ** 2).sum(axis=0))
    rms = float(np.sqrt((mag ** 2).mean()))
    frac = float((d <= 1e-6 * mag).mean())
    print("fx32 4M: max|dF|/rms", d.max() / rms, "frac<=1e-6", frac, "pe", abs(pe - pe64) / abs(pe64),
          "w", abs(w - w64) / abs(w64))
    assert d.max() <= 1e-6 * rms and frac >= 0.99
    assert abs(pe - pe64) < 1e-6 * abs(pe64) and abs(w - w64) < 1e-5 * abs(w64) and ins == in64
    f2, pe2, w2, ins2, _ = forces(md, liquid_4m, md.PREC_FX32)
    assert np.array_equal(f, f2) and (pe2, w2, ins2) == (pe, w, ins)
