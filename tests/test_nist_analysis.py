"""The NIST validation analysis (molecular-dynamics_b200/nist.py) against the reference's own analysis code,
bench/validate.py, as evaluated by tests/golden/make_nist_golden.py: the tables, the energy shift, the tail
corrections, block errors, the per-replica series with the unshifted-energy convention, replica statistics and
z-scores. CPU only."""
from __future__ import annotations

import json
import os

import pytest

import nist

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "nist_analysis.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def test_tables_and_protocol(golden):
    assert [list(r) for r in nist.NIST_MD] == golden["nist_md"]
    assert [list(r) for r in nist.NIST_MC] == golden["nist_mc"]
    assert nist.CUTOFF == golden["cutoff"] and nist.REPLICAS == golden["replicas"]
    assert len(nist.state_points()) == 16


def test_shift_and_tail_corrections(golden):
    assert nist.shift_energy(nist.CUTOFF) == golden["shift_energy"]
    for row in golden["tail"]:
        assert nist.tail_energy(row["rho"], nist.CUTOFF) == row["energy"]
        assert nist.tail_pressure(row["rho"], nist.CUTOFF) == row["pressure"]


def test_block_error(golden):
    for row in golden["block_error"]:
        assert nist.block_error(golden["block_series"], row["block_len"]) == pytest.approx(row["error"], rel=1e-12)


def test_replica_statistics_and_z_scores(golden):
    for case in golden["analyse"]:
        us, ps = [], []
        for recs in case["records"]:
            u, p = nist.replica_series([r["pe_per_particle"] for r in recs], [r["inside_pairs"] for r in recs],
                                       [r["pressure"] for r in recs], 500, case["rho"])
            us.append(u)
            ps.append(p)
        a = nist.analyse(us, ps)
        for k in ("u", "u_err", "p", "p_err"):
            assert a[k] == pytest.approx(case["result"][k], rel=1e-12, abs=1e-15), k
        ref = next(r for r in nist.NIST_MC if r[0] == case["T"] and r[1] == case["rho"])
        zu, zp = nist.z_scores(a, ref)
        assert zu == pytest.approx(case["z_u"], rel=1e-10) and zp == pytest.approx(case["z_p"], rel=1e-10)
