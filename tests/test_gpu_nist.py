"""The NIST validation protocol through the batched engine (molecular-dynamics_b200/nist.py, the reference's
bench/validate.py): phases switched with md_batch_set_thermostat (melt, cool, Bussi NVT production) and the
inside-cutoff counts recorded per step for the unshifted-energy convention.

1. The phase protocol is the single-system protocol: each replica equals the same system run alone through
   md_run with the same rescale/melt schedule and then Bussi draws from the replica's seed, bit for bit (FP64).
2. A reduced validation (2 state points x 4 replicas, 1,500 + 1,500 steps instead of 10,000 + 20,000) lands near
   NIST's Monte Carlo values; the full protocol is `bench.py --nist`."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_phase_protocol_equals_single_runs(md):
    import nist

    cases = [(5, 0.776, 0.85, 1001), (5, 0.9, 0.9, 1002), (4, 0.84, 0.85, 1003)]
    systems, temps, seeds = [], [], []
    for cells, rho, t, seed in cases:
        s = md.fcc_system(cells, rho, t, seed=seed)
        d = s.download()
        systems.append((d["pos"], s.box, d["vel"], None))
        temps.append(t)
        seeds.append(seed)
    b = md.Batch(systems, cutoff=nist.CUTOFF, skin=nist.SKIN, dt=nist.DT, precision=md.PREC_FP64,
                 thermostat="rescale", temperatures=np.full(3, 2.0), rescale_every=10, energy_every=1, chunk_steps=50)
    b.run(30, record=False)
    b.set_thermostat("rescale", temperatures=temps, rescale_every=10)
    b.run(60, record=False)
    b.set_thermostat("bussi", temperatures=temps, bussi_tau=0.5, seeds=seeds)
    pe, w, ke, inside = b.run(90, inside=True)
    hashes = b.state_hashes()
    integ = md.VelocityVerletIntegrator(nist.DT)
    for r, (cells, rho, t, seed) in enumerate(cases):
        s = md.fcc_system(cells, rho, t, seed=seed)
        nl = md.NeighbourList(nist.CUTOFF, nist.SKIN, True)
        ff = md.LennardJonesForceField(1.0, 1.0, nist.CUTOFF)
        ff.set_deterministic(True)
        nl.build(s)
        ff.compute_forces(s, nl)
        integ.run(s, ff, nl, 90, thermostat="rescale", rescale_every=10, rescale_temperature=t, melt_until=30,
                  melt_temperature=2.0, record=False)
        r1, chi2 = md.bussi_noise(seed, s.n, 90)
        spe, ske, sw = integ.run(s, ff, nl, 90, thermostat="bussi", bussi_temperature=t, bussi_tau=0.5, bussi_r1=r1,
                                 bussi_chi2=chi2)
        assert int(hashes[r]) == s.state_hash(), r
        assert np.array_equal(pe[:, r], spe) and np.array_equal(ke[:, r], ske) and np.array_equal(w[:, r], sw), r
        # the last step's inside count is the force field's getInsidePairs after the run
        ff.fetch_results()
        assert inside[-1, r] == ff.inside_pairs, r


def test_reduced_validation_near_nist(md):
    import nist

    states = [(0.85, 0.776), (0.9, 0.9)]
    rows, _ = nist.run(md, states=states, replicas=4, equil=1500, prod=1500)
    for row in rows:
        ref = row["nist_mc"]
        print(row["T"], row["rho"], "U", row["u"], "+-", row["u_err"], "NIST", ref[2], "z", row["z_u_mc"],
              "P", row["p"], "+-", row["p_err"], "NIST", ref[4], "z", row["z_p_mc"])
        assert row["u_err"] > 0 and row["p_err"] > 0
        # short runs of 500 atoms: within a few hundredths of NIST's energy and a few tenths of its pressure
        assert abs(row["u"] - ref[2]) < 0.05 and abs(row["p"] - ref[4]) < 0.3
