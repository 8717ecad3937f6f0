"""Precision sweep on the 256,000-atom FCC start (40^3 x 4) over densities {0.5, 0.8442, 1.0} and
T* in {0.71, 1.5, 3.0}: FP32 fixed-point, FP32 float-accumulate, FX64 and FX32 against FP64 — per-particle force error,
energy drift, virial pressure and g(r), each a mean over replicas with its standard error. The full-length sweep
(10,000 steps, 4 replicas) is `bench.py --sweep precision`; here 400 steps per run and 2 replicas keep the test to
a few minutes, with the tolerances stated below."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


def test_precision_sweep_short(md):
    import bench

    for pt in bench.precision_sweep(steps=400, equil=100, replicas=2):
        tag = (pt["density"], pt["temperature"])
        for prec in ("fp32fx", "fp32"):
            e = pt["force_error_vs_fp64"][prec]
            # float pair arithmetic: rms force error a few 1e-6 of rms |F|; the cutoff test is exact, so the
            # largest error is rounding of the strongest pairs, well under the reference's mixed-precision
            # bound of 1e-5 max |F| (tests/test_forcefield.cpp:123-149)
            assert e["rms_dF_over_rms_F"] < 1e-5, (tag, prec, e)
            assert e["max_abs_dF_over_max_F"] < 1e-5, (tag, prec, e)
            assert e["pe_rel"] < 1e-6, (tag, prec, e)
            run, ref = pt[prec], pt["fp64"]
            # NVE drift stays within the reference's bound (3e-4) and within 10x of the FP64 run's
            assert run["max_drift"] < max(3e-4, 10 * ref["max_drift"]), (tag, prec, run, ref)
            # the same state point: the trajectories separate chaotically, so only averages are compared —
            # pressure within 2 % (+0.01 absolute near P = 0) and g(r) within 0.1 of the FP64 run's
            assert abs(run["pressure"] - ref["pressure"]) <= 0.02 * abs(ref["pressure"]) + 0.01, (tag, prec)
            assert run["max_dg_vs_fp64"] < 0.1, (tag, prec, run["max_dg_vs_fp64"])
        assert pt["fp64"]["max_drift"] < 3e-4, (tag, pt["fp64"])
        # replica error bars: every float mode reports its paired pressure difference from FP64 with an error
        for prec in ("fp32fx", "fp32", "fx64", "fx32"):
            assert pt[prec]["dp_vs_fp64_err"] is not None and pt[prec]["pressure_err"] is not None, (tag, prec)
        # FX64 (exact separations, double pair terms) and FX32 (the same separations, double terms for the close
        # pairs only) meet the 1e-6 per-particle bound
        for prec in ("fx64", "fx32"):
            e = pt["force_error_vs_fp64"][prec]
            assert e["max_particle_dF_over_rms_F"] <= 1e-6 and e["frac_particles_rel_le_1e-6"] >= 0.99, (tag, prec, e)
            run, ref = pt[prec], pt["fp64"]
            assert run["max_drift"] < max(3e-4, 10 * ref["max_drift"]), (tag, prec, run, ref)
            assert abs(run["pressure"] - ref["pressure"]) <= 0.02 * abs(ref["pressure"]) + 0.01, (tag, prec)
