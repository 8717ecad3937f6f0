"""Batched replicas (md_batch_*) against the same systems run one at a time.

Every replica of a batch follows the reference's single-system step on its own box, so its trajectory must be
bit-identical to that system run alone: through the oracle (FP64, the reference's deterministic arithmetic) and
through the single-system GPU path (md_run) in every precision. The batch makes its rebuild decisions on the
device inside CUDA graphs of `chunk_steps` steps; the cases below use chunks that do not divide the run, boxes
under 3 cells per side (the all-pairs candidate fallback, src/NeighbourList.cpp:69) and boxes with cells.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle.oracle import MODE_DETERMINISTIC, ONeighbourList, OForceField

pytestmark = pytest.mark.gpu

RC, SKIN, DT, TAU = 2.5, 0.3, 0.005, 0.1
# (FCC cells per side, density, temperature, seed): n = 4 and 5 fall back to all-pairs candidates
CASES = [(4, 0.80, 1.2, 11), (6, 0.75, 2.0, 13), (5, 0.95, 0.7, 12), (7, 0.85, 1.0, 14), (4, 0.93, 1.6, 15),
         (6, 0.90, 0.9, 16)]


def make_batch(md, cases, precision, steps_every=10, chunk=40, thermostat="bussi", capacity=0):
    systems, temps, seeds = [], [], []
    for cells, rho, temp, seed in cases:
        s = md.fcc_system(cells, rho, temp, seed=seed)
        d = s.download()
        systems.append((d["pos"], s.box, d["vel"], None))
        temps.append(temp)
        seeds.append(seed)
    return md.Batch(systems, cutoff=RC, skin=SKIN, dt=DT, precision=precision, thermostat=thermostat,
                    temperatures=temps, seeds=seeds, bussi_tau=TAU, energy_every=steps_every, chunk_steps=chunk,
                    initial_capacity=capacity)


def single_run(md, case, precision, steps, thermostat="bussi"):
    cells, rho, temp, seed = case
    s = md.fcc_system(cells, rho, temp, seed=seed)
    nl = md.NeighbourList(RC, SKIN, True)
    ff = md.LennardJonesForceField(1.0, 1.0, RC, precision=precision)
    ff.set_deterministic(True)
    nl.build(s)
    ff.compute_forces(s, nl)
    integ = md.VelocityVerletIntegrator(DT)
    kw = {}
    if thermostat == "bussi":
        r1, chi2 = md.bussi_noise(seed, s.n, steps)
        kw = dict(bussi_temperature=temp, bussi_tau=TAU, bussi_r1=r1, bussi_chi2=chi2)
    pe, ke, w = integ.run(s, ff, nl, steps, thermostat=thermostat, **kw)
    return s, nl, pe, ke, w


@pytest.mark.parametrize("precision", [0, 1, 2], ids=["fp64", "fp32fx", "fp32"])
def test_batch_replicas_bit_identical_to_single_runs(md, precision):
    steps = 150
    b = make_batch(md, CASES, precision)
    pe, w, ke = b.run(steps)
    hashes = b.state_hashes()
    rebuilds = b.rebuilds()
    for r, case in enumerate(CASES):
        s, nl, spe, ske, sw = single_run(md, case, precision, steps)
        assert int(hashes[r]) == s.state_hash(), (r, case)
        assert int(rebuilds[r]) == nl.rebuild_count, (r, case)
        assert np.array_equal(pe[:, r], spe[9::10]), (r, case)
        assert np.array_equal(w[:, r], sw[9::10]), (r, case)
        assert np.array_equal(ke[:, r], ske[9::10]), (r, case)
        d = b.download(r)
        got = s.download()
        assert np.array_equal(d["ids"], got["ids"]) and np.array_equal(d["force"], got["force"])


def test_batch_fp64_matches_oracle(md, oracle):
    """FP64 replicas against the oracle's restatement of the reference (deterministic forces, Bussi)."""
    steps = 120
    cases = CASES[:3]
    b = make_batch(md, cases, 0, chunk=50)
    pe, w, ke = b.run(steps)
    hashes = b.state_hashes()
    for r, (cells, rho, temp, seed) in enumerate(cases):
        s = oracle.fcc_system(cells, rho, temp, seed)
        nl = ONeighbourList(oracle, RC, SKIN, True)
        ff = OForceField(oracle, 1.0, 1.0, RC)
        nl.build(s)
        ff.forces(s, nl, MODE_DETERMINISTIC)
        r1, chi2 = oracle.bussi_noise(seed, s.n, steps)
        c = math.exp(-DT / TAU)
        opes = []
        for k in range(steps):
            opes.append(ff.step(s, nl, DT, MODE_DETERMINISTIC))
            s.bussi(temp, c, r1[k], chi2[k])
        assert int(hashes[r]) == s.hash(), (r, cells, rho, temp)
        assert np.array_equal(pe[:, r], np.array(opes)[9::10])
        assert int(b.rebuilds()[r]) == nl.rebuilds


def test_batch_force_variants_same_bits(md):
    b = make_batch(md, CASES, 1)
    b.run(30)
    info = b.force_variant()
    assert info["count"] > 1
    ref = None
    for v in range(info["count"]):
        b.set_force_variant(v)
        pe, w, ke, ins = b.energy()
        forces = [b.download(r)["force"] for r in range(len(CASES))]
        cur = (pe, w, ins, forces)
        if ref is None:
            ref = cur
        else:
            assert np.array_equal(cur[0], ref[0]) and np.array_equal(cur[1], ref[1]) and np.array_equal(cur[2], ref[2])
            for f, g in zip(cur[3], ref[3]):
                assert np.array_equal(f, g), v
    b.set_force_variant(-1)
    assert 0 <= b.force_variant()["variant"] < info["count"]


def test_batch_row_capacity_regrowth_keeps_trajectory(md):
    """Rows of 80 fit the FCC lattice at density 0.8442 (78 neighbours within r_c + skin); the hot liquid
    outgrows them inside a chunk, which is then restored and run again with a larger capacity."""
    cases = [(6, 0.8442, 2.0, 21), (7, 0.8442, 1.8, 22)]
    small = make_batch(md, cases, 0, capacity=80, thermostat="none", chunk=25)
    assert small.info()["capacity"] == 80
    big = make_batch(md, cases, 0, thermostat="none", chunk=25)
    a = small.run(100)
    c = big.run(100)
    assert small.info()["capacity"] > 80
    assert np.array_equal(small.state_hashes(), big.state_hashes())
    assert all(np.array_equal(x, y) for x, y in zip(a, c))


def test_batch_rescale_thermostat_matches_single(md):
    cases = CASES[1:3]
    b = make_batch(md, cases, 0, thermostat="rescale", chunk=30)
    b.run(60)
    for r, (cells, rho, temp, seed) in enumerate(cases):
        s = md.fcc_system(cells, rho, temp, seed=seed)
        nl = md.NeighbourList(RC, SKIN, True)
        ff = md.LennardJonesForceField(1.0, 1.0, RC)
        ff.set_deterministic(True)
        nl.build(s)
        ff.compute_forces(s, nl)
        md.VelocityVerletIntegrator(DT).run(s, ff, nl, 60, thermostat="rescale", rescale_every=10,
                                            rescale_temperature=temp, record=False)
        assert int(b.state_hashes()[r]) == s.state_hash()


def test_batch_nve_conserves_energy(md):
    cases = [(6, 0.8442, 0.71, 31), (8, 0.8442, 0.71, 32)]
    b = make_batch(md, cases, 1, thermostat="none", steps_every=10, chunk=100)
    pe0, w0, ke0, _ = b.energy()
    pe, w, ke = b.run(1000)
    e0 = pe0 + ke0
    drift = np.abs((pe + ke - e0) / e0).max(axis=0)
    assert (drift < 3e-4).all(), drift  # tests/test_dynamics.cpp:40-56 bound
