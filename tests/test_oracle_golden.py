"""Pins the oracle (oracle/md_oracle.cpp) to golden vectors recorded from the reference itself.

The reference's tests cannot be built here (GoogleTest is fetched at configure time), so the known answers
they hold are restated: analytic two-body forces (tests/test_forcefield.cpp:28-63), virial
(tests/test_observables.cpp:6-19), cell membership (tests/test_neighbourlist.cpp:85-129), list contents
(:38-57). The golden files come from tests/golden/make_golden.py, which runs the reference compiled from its
own sources with strict IEEE double arithmetic.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle.oracle import (MODE_ALL_PAIRS, MODE_DEFAULT, MODE_DETERMINISTIC, MODE_MIXED, ONeighbourList,
                           OForceField, fcc_box, rdf_sample, state_hash)

C1 = dict(cells=8, density=0.8442, temperature=0.71, seed=42, rc=2.5, skin=0.3, dt=0.005)


def lj_force(r):
    return 24.0 * (2.0 * r ** -13 - r ** -7)


def lj_energy(r, rc):
    v = lambda x: 4.0 * (x ** -12 - x ** -6)  # noqa: E731
    return v(r) - v(rc)


def pair_system(oracle, x0, x1, box):
    pos = np.array([[x0, 5.0, 5.0, 0.0], [x1, 5.0, 5.0, 0.0]])
    return oracle.system(pos, box)


@pytest.mark.parametrize("r", [0.95, 1.12, 1.5, 2.0, 2.45])
def test_two_particle_analytic(oracle, r):
    # tests/test_forcefield.cpp:28-40
    s = pair_system(oracle, 5.0, 5.0 + r, 20.0)
    ff = OForceField(oracle, 1.0, 1.0, 2.5)
    pe = ff.forces(s, None, MODE_ALL_PAIRS)
    f = s.state().force
    assert abs(f[0, 0] + lj_force(r)) < 1e-10
    assert abs(f[0, 1] - lj_force(r)) < 1e-10
    assert abs(f[1, 0]) < 1e-12
    assert abs(pe - lj_energy(r, 2.5)) < 1e-12


def test_zero_force_at_minimum_and_cutoff_and_pbc(oracle):
    ff = OForceField(oracle, 1.0, 1.0, 2.5)
    s = pair_system(oracle, 5.0, 5.0 + 2.0 ** (1.0 / 6.0), 20.0)
    ff.forces(s, None, MODE_ALL_PAIRS)
    assert abs(s.state().force[0, 0]) < 1e-12
    s = pair_system(oracle, 5.0, 5.0 + 2.5 + 1e-9, 20.0)
    assert ff.forces(s, None, MODE_ALL_PAIRS) == 0.0
    s = pair_system(oracle, 0.5, 19.5, 20.0)
    pe = ff.forces(s, None, MODE_ALL_PAIRS)
    assert abs(s.state().force[0, 0] - lj_force(1.0)) < 1e-10
    assert abs(pe - lj_energy(1.0, 2.5)) < 1e-12
    s = pair_system(oracle, 1.0, 2.0, 4.0)
    with pytest.raises(RuntimeError, match="half the box"):
        ff.forces(s, None, MODE_ALL_PAIRS)


def test_two_particle_virial(oracle):
    # tests/test_observables.cpp:6-19
    s = pair_system(oracle, 5.0, 6.3, 20.0)
    ff = OForceField(oracle, 1.0, 1.0, 2.5)
    ff.forces(s, None, MODE_ALL_PAIRS)
    assert abs(ff.virial - 1.3 * lj_force(1.3)) < 1e-12
    assert ff.inside == 1.0


def test_config1_init_and_cells(oracle, golden):
    g = golden("config1")
    s = oracle.fcc_system(C1["cells"], C1["density"], C1["temperature"], C1["seed"])
    st = s.state()
    assert st.box == float(g["box"])
    assert np.array_equal(st.pos, g["init_pos"])
    assert np.array_equal(st.vel, g["init_vel"])
    ncps, cell, start, parts = oracle.cells_build(s, C1["rc"] + C1["skin"])
    assert ncps == int(g["cells_ncps"])
    assert np.array_equal(cell, g["cells_cell"])
    assert np.array_equal(start, g["cells_start"])
    assert np.array_equal(parts, g["cells_particles"])


def test_config1_allpairs_build_and_deterministic_forces(oracle, golden):
    g = golden("config1")
    s = oracle.fcc_system(C1["cells"], C1["density"], C1["temperature"], C1["seed"])
    ff = OForceField(oracle, 1.0, 1.0, C1["rc"])
    pe = ff.forces(s, None, MODE_ALL_PAIRS)
    assert pe == float(g["allpairs_pe"]) and ff.virial == float(g["allpairs_virial"])
    assert ff.inside == float(g["allpairs_inside"])
    assert np.array_equal(s.state().force, g["allpairs_force"])
    nl = ONeighbourList(oracle, C1["rc"], C1["skin"], reverse=True)
    nl.build(s)
    st = s.state()
    assert np.array_equal(st.pos, g["build_pos"]) and np.array_equal(st.vel, g["build_vel"])
    assert np.array_equal(st.force, g["build_force"]) and np.array_equal(st.ids, g["build_ids"])
    L = nl.get(s.n)
    for k in ("offsets", "neighbours", "rev_offsets", "rev_pairs"):
        assert np.array_equal(L[k], g["nl_" + k]), k
    pe = ff.forces(s, nl, MODE_DETERMINISTIC)
    assert pe == float(g["det_pe"]) and ff.virial == float(g["det_virial"])
    assert ff.inside == float(g["det_inside"])
    assert np.array_equal(s.state().force, g["det_force"])


def test_config1_trajectory_bit_exact(oracle, golden):
    """md_sim 8 --deterministic --skin 0.3 --temperature 0.71 --equil 0 --steps 1000: every per-step PE and
    KE, the checkpoint hashes and g(r) (200 bins to 5 sigma) equal the reference's bit for bit."""
    g = golden("config1")
    s = oracle.fcc_system(C1["cells"], C1["density"], C1["temperature"], C1["seed"])
    ff = OForceField(oracle, 1.0, 1.0, C1["rc"])
    ff.forces(s, None, MODE_ALL_PAIRS)
    nl = ONeighbourList(oracle, C1["rc"], C1["skin"], reverse=True)
    nl.build(s)
    want = dict(zip(g["hash_steps"].tolist(), g["hash_values"].tolist()))
    hist = np.zeros(200)
    samples = 0
    for step in range(1, 1001):
        pe = ff.step(s, nl, C1["dt"], MODE_DETERMINISTIC)
        assert pe == g["pe"][step - 1], step
        assert s.kinetic() == g["ke"][step - 1], step
        if step in want:
            assert s.hash() == want[step], step
        if step % 100 == 0:
            clone = oracle.system(s.state().pos, s.box, s.state().vel)
            big = ONeighbourList(oracle, 4.7, 0.3)
            big.build(clone)
            rdf_sample(oracle, clone, big, 5.0, 200, hist)
            samples += 1
    assert nl.rebuilds == int(g["rebuilds"])
    st = s.state()
    assert np.array_equal(st.pos, g["final_pos"]) and np.array_equal(st.vel, g["final_vel"])
    assert np.array_equal(st.ids, g["final_ids"])
    assert state_hash(st.pos, st.vel) == want[1000]
    gr = oracle.rdf_values(hist, 5.0, samples, s.n, s.box)
    assert np.array_equal(gr, g["rdf_g"])


def test_small_box_fallback(oracle, golden):
    g = golden("small_box")
    s = oracle.fcc_system(4, 0.8442, 0.728, 42)
    ff = OForceField(oracle, 1.0, 1.0, 2.5)
    nl = ONeighbourList(oracle, 2.5, 0.2, reverse=True)
    nl.build(s)
    ff.forces(s, nl, MODE_DETERMINISTIC)
    for k in range(1, 61):
        ff.step(s, nl, 0.005, MODE_DETERMINISTIC)
        if k % 10 == 0:
            s.rescale(0.728)
    assert s.hash() == int(g["hash"]) and nl.rebuilds == int(g["rebuilds"])
    L = nl.get(s.n)
    for k in ("offsets", "neighbours", "rev_offsets", "rev_pairs"):
        assert np.array_equal(L[k], g["nl_" + k]), k
    pe = ff.forces(s, nl, MODE_DETERMINISTIC)
    assert pe == float(g["det_pe"]) and ff.virial == float(g["det_virial"])
    assert np.array_equal(s.state().force, g["det_force"])


def test_bussi_noise_and_scaling(oracle, golden):
    g = golden("bussi")
    s = oracle.fcc_system(5, 0.8442, 0.728, 42)
    assert s.kinetic() == float(g["ke0"])
    r1, chi2 = oracle.bussi_noise(7, s.n, 50)
    c = math.exp(-0.005 / 0.05)
    for k in range(50):
        s.bussi(0.85, c, r1[k], chi2[k])
        assert s.kinetic() == g["ke"][k], k
    assert s.hash() == int(g["hash"])


def test_default_and_mixed_paths_match_deterministic(oracle, golden):
    """List forces (default and mixed precision) against the deterministic path, with the reference's own
    tolerances (tests/test_forcefield.cpp:73-149)."""
    g = golden("config1")
    # the state after 1000 steps is a liquid (on the lattice every net force is ~0 and relative bounds mislead)
    s = oracle.system(g["final_pos"], float(g["box"]), g["final_vel"])
    nl = ONeighbourList(oracle, C1["rc"], C1["skin"], reverse=True)
    nl.build(s)
    ff = OForceField(oracle, 1.0, 1.0, C1["rc"])
    pe_det = ff.forces(s, nl, MODE_DETERMINISTIC)
    f_det = s.state().force
    pe_def = ff.forces(s, nl, MODE_DEFAULT)
    assert abs(pe_def - pe_det) < 1e-9 * abs(pe_det)
    assert np.abs(s.state().force - f_det).max() < 1e-11
    pe_mix = ff.forces(s, nl, MODE_MIXED)
    assert abs(pe_mix - pe_det) < 1e-5 * abs(pe_det)
    assert np.abs(s.state().force - f_det).max() < 1e-5 * np.abs(f_det).max()
    pe_all = ff.forces(s, None, MODE_ALL_PAIRS)
    assert abs(pe_all - pe_det) < 1e-9 * abs(pe_det)
    assert np.abs(s.state().force - f_det).max() < 1e-11


def test_fcc_box_matches_md_sim(golden):
    a, box = fcc_box(8, 0.8442)
    assert box == float(golden("config1")["box"])
