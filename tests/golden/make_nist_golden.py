"""Generate tests/golden/nist_analysis.json from the reference's own validation code (bench/validate.py of
nhantran1711/molecular-dynamics): its tail corrections, energy shift, block error, per-replica series with the
unshifted-energy convention, replica statistics and z-scores, evaluated on synthetic replica records.

validate.py imports its plotting helpers from bench/benchmark.py; those are replaced by stubs here, and its file
reader (read_rows) by one that serves the synthetic records, so only the analysis code runs. The fixture it
writes is committed and is all the tests read.

    python tests/golden/make_nist_golden.py [REFERENCE_ROOT]
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys
import types

import numpy as np

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "nist_analysis.json")


def load_validate(reference: str):
    stub = types.ModuleType("benchmark")
    for name in ("BINARY", "RESULTS", "SERIES", "SURFACE", "TEXT_SECONDARY"):
        setattr(stub, name, None)
    for name in ("figure", "read_rows", "save", "style", "write_rows"):
        setattr(stub, name, lambda *a, **k: None)
    sys.modules["benchmark"] = stub
    spec = importlib.util.spec_from_file_location("ref_validate", os.path.join(reference, "bench", "validate.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def synthetic_records(rng, replicas, steps, n=500):
    """Per replica: production rows (pe_per_particle, inside_pairs, pressure) plus a few equilibration rows that
    the analysis must skip"""
    recs = []
    for _ in range(replicas):
        pe = -5.6 + 0.02 * rng.standard_normal(steps)
        inside = np.round(n * 44 + 30 * rng.standard_normal(steps))
        p = 0.3 + 0.05 * rng.standard_normal(steps)
        rows = [{"phase": "equilibration", "pe_per_particle": 9.0, "inside_pairs": 1.0, "pressure": 9.0}] * 3
        rows += [{"phase": "production", "pe_per_particle": float(pe[k]), "inside_pairs": float(inside[k]),
                  "pressure": float(p[k])} for k in range(steps)]
        recs.append(rows)
    return recs


def main():
    reference = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    v = load_validate(reference)
    rng = np.random.default_rng(2024)
    out = {"cutoff": v.CUTOFF, "replicas": v.REPLICAS, "nist_md": v.NIST_MD, "nist_mc": v.NIST_MC,
           "shift_energy": v.shift_energy(v.CUTOFF), "tail": [], "block_error": [], "analyse": []}
    for _, rho, *_ in v.NIST_MD + v.NIST_MC:
        out["tail"].append({"rho": rho, "energy": v.tail_energy(rho, v.CUTOFF), "pressure": v.tail_pressure(rho, v.CUTOFF)})
    series = list(0.1 * rng.standard_normal(1024).cumsum() / 64)
    for b in (1, 4, 16, 64):
        out["block_error"].append({"block_len": b, "error": v.block_error(series, b)})
    out["block_series"] = series
    for t, rho in ((0.85, 0.776), (0.90, 0.9)):
        recs = synthetic_records(rng, v.REPLICAS, 50)
        v.read_rows = lambda path, recs=recs, t=t, rho=rho: recs[int(str(path).rsplit("_r", 1)[1].split(".")[0])]
        v.run_path = lambda temperature, density, replica: f"validate_T{temperature}_rho{density}_r{replica}.csv"
        a = v.analyse(t, rho)
        ref = next(r for r in v.NIST_MC if r[0] == t and r[1] == rho)
        zu = (a["u"] - ref[2]) / np.hypot(a["u_err"], ref[3])
        zp = (a["p"] - ref[4]) / np.hypot(a["p_err"], ref[5])
        prod = [[{k: r[k] for k in ("pe_per_particle", "inside_pairs", "pressure")} for r in rows
                 if r["phase"] == "production"] for rows in recs]
        out["analyse"].append({"T": t, "rho": rho, "records": prod, "result": a, "z_u": zu, "z_p": zp})
    with open(OUT, "w") as f:
        json.dump(out, f)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
