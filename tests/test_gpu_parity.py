"""GPU parity: libmdgpu through its C-ABI against golden vectors recorded from the reference and against the
oracle. Integer/index results (cells, sort order, lists) and every FP64 result are compared bit for bit;
the float force modes are compared with stated tolerances.

The checks restate the reference's own tests where they apply: tests/test_forcefield.cpp,
tests/test_neighbourlist.cpp, tests/test_dynamics.cpp, tests/test_determinism.cpp,
tests/test_observables.cpp, tests/test_system.cpp.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle.oracle import MODE_ALL_PAIRS, MODE_DETERMINISTIC, ONeighbourList, OForceField, fcc_box

pytestmark = pytest.mark.gpu

C1 = dict(cells=8, density=0.8442, temperature=0.71, seed=42, rc=2.5, skin=0.3, dt=0.005)


def lj_force(r):
    return 24.0 * (2.0 * r ** -13 - r ** -7)


def lj_energy(r, rc):
    v = lambda x: 4.0 * (x ** -12 - x ** -6)  # noqa: E731
    return v(r) - v(rc)


def config1_system(md, g):
    return md.System.from_arrays(g["init_pos"], float(g["box"]), vel=g["init_vel"])


def test_cell_list_bit_exact(md, golden):
    g = golden("config1")
    s = config1_system(md, g)
    cl = md.CellList(C1["rc"] + C1["skin"])
    assert cl.build(s) == int(g["cells_ncps"])
    cell, start, parts = cl.download()
    assert np.array_equal(cell, g["cells_cell"])
    assert np.array_equal(start, g["cells_start"])
    assert np.array_equal(parts, g["cells_particles"])


def test_all_pairs_build_and_deterministic_forces_bit_exact(md, golden):
    g = golden("config1")
    s = config1_system(md, g)
    ff = md.LennardJonesForceField(1.0, 1.0, C1["rc"])
    ff.set_deterministic(True)
    pe = ff.compute_forces(s)
    assert pe == float(g["allpairs_pe"])
    assert ff.virial == float(g["allpairs_virial"]) and ff.inside_pairs == float(g["allpairs_inside"])
    assert np.array_equal(s.forces(), g["allpairs_force"])
    nl = md.NeighbourList(C1["rc"], C1["skin"], reverse_index=True)
    nl.build(s)
    st = s.download()
    assert np.array_equal(st["pos"], g["build_pos"]) and np.array_equal(st["vel"], g["build_vel"])
    assert np.array_equal(st["force"], g["build_force"]) and np.array_equal(st["ids"], g["build_ids"])
    L = nl.download()
    for k in ("offsets", "neighbours", "rev_offsets", "rev_pairs"):
        assert np.array_equal(L[k], g["nl_" + k]), k
    assert nl.pair_count == len(g["nl_neighbours"])
    pe = ff.compute_forces(s, nl)
    assert pe == float(g["det_pe"])
    assert ff.virial == float(g["det_virial"]) and ff.inside_pairs == float(g["det_inside"])
    assert np.array_equal(s.forces(), g["det_force"])


def test_trajectory_bit_exact_1000_steps(md, golden):
    """md_sim 8 --deterministic --skin 0.3 --temperature 0.71 --equil 0 --steps 1000 on the device: every
    step's PE and KE, the checkpoint state hashes, the rebuild count, the final state and g(r) equal the
    reference's bit for bit."""
    g = golden("config1")
    s = config1_system(md, g)
    ff = md.LennardJonesForceField(1.0, 1.0, C1["rc"])
    ff.set_deterministic(True)
    ff.compute_forces(s)
    nl = md.NeighbourList(C1["rc"], C1["skin"], reverse_index=True)
    nl.build(s)
    integ = md.VelocityVerletIntegrator(C1["dt"])
    want = dict(zip(g["hash_steps"].tolist(), g["hash_values"].tolist()))
    rdf = md.RadialDistribution(5.0, 200)
    # step 1 through the single-step API, the rest through the device-resident loop
    pe1 = integ.step(s, ff, nl)
    assert pe1 == g["pe"][0]
    assert s.kinetic_energy() == g["ke"][0]
    assert s.state_hash() == want[1]
    st = s.download()
    assert np.array_equal(st["force"], g["step1_force"]) and np.array_equal(st["ids"], g["step1_ids"])
    done = 1
    for target in sorted(want):
        if target <= done:
            continue
        pe, ke, _ = integ.run(s, ff, nl, target - done, first_step=done + 1)
        assert np.array_equal(pe, g["pe"][done:target]), (done, target)
        assert np.array_equal(ke, g["ke"][done:target]), (done, target)
        done = target
        assert s.state_hash() == want[target], target
        if target % 100 == 0:
            st = s.download()
            clone = md.System.from_arrays(st["pos"], s.box, vel=st["vel"])
            big = md.NeighbourList(4.7, 0.3)
            big.build(clone)
            rdf.sample(clone, big)
    assert nl.rebuild_count == int(g["rebuilds"])
    st = s.download()
    assert np.array_equal(st["pos"], g["final_pos"]) and np.array_equal(st["vel"], g["final_vel"])
    assert np.array_equal(st["ids"], g["final_ids"])
    assert np.array_equal(rdf.values(), g["rdf_g"])
    assert np.array_equal(rdf.radii(), g["rdf_radii"])


def test_small_box_fallback_bit_exact(md, golden):
    g = golden("small_box")
    o_pos = None
    from oracle.oracle import Oracle
    o = Oracle()
    os_ = o.fcc_system(4, 0.8442, 0.728, 42)
    st = os_.state()
    s = md.System.from_arrays(st.pos, st.box, vel=st.vel)
    ff = md.LennardJonesForceField(1.0, 1.0, 2.5)
    ff.set_deterministic(True)
    nl = md.NeighbourList(2.5, 0.2, reverse_index=True)
    nl.build(s)
    assert nl.cells_per_side == 2
    ff.compute_forces(s, nl)
    integ = md.VelocityVerletIntegrator(0.005)
    integ.run(s, ff, nl, 60, thermostat="rescale", rescale_every=10, rescale_temperature=0.728, record=False)
    assert s.state_hash() == int(g["hash"]) and nl.rebuild_count == int(g["rebuilds"])
    L = nl.download()
    for k in ("offsets", "neighbours", "rev_offsets", "rev_pairs"):
        assert np.array_equal(L[k], g["nl_" + k]), k
    pe = ff.compute_forces(s, nl)
    assert pe == float(g["det_pe"]) and ff.virial == float(g["det_virial"])
    assert np.array_equal(s.forces(), g["det_force"])
    del o_pos


def test_bussi_noise_and_thermostat_bit_exact(md, oracle, golden):
    g = golden("bussi")
    os_ = oracle.fcc_system(5, 0.8442, 0.728, 42)
    st = os_.state()
    s = md.System.from_arrays(st.pos, st.box, vel=st.vel)
    assert s.kinetic_energy() == float(g["ke0"])
    r1, chi2 = md.bussi_noise(7, s.n, 50)
    r1o, chi2o = oracle.bussi_noise(7, s.n, 50)
    assert np.array_equal(r1, r1o) and np.array_equal(chi2, chi2o)
    for k in range(50):
        s.bussi_apply(0.85, 0.05, 0.005, r1[k], chi2[k])
        assert s.kinetic_energy() == g["ke"][k], k
    assert s.state_hash() == int(g["hash"])


@pytest.mark.parametrize("r", [0.95, 1.12, 1.5, 2.0, 2.45])
def test_two_particles_analytic(md, r):
    # tests/test_forcefield.cpp:28-40
    s = md.System.from_arrays(np.array([[5.0, 5.0, 5.0], [5.0 + r, 5.0, 5.0]]), 20.0)
    ff = md.LennardJonesForceField(1.0, 1.0, 2.5)
    pe = ff.compute_forces(s)
    f = s.forces()
    assert abs(f[0, 0] + lj_force(r)) < 1e-10 and abs(f[0, 1] - lj_force(r)) < 1e-10
    assert abs(f[1, 0]) < 1e-12
    assert abs(pe - lj_energy(r, 2.5)) < 1e-12


def test_pbc_cutoff_and_errors(md):
    ff = md.LennardJonesForceField(1.0, 1.0, 2.5)
    s = md.System.from_arrays(np.array([[0.5, 5.0, 5.0], [19.5, 5.0, 5.0]]), 20.0)
    pe = ff.compute_forces(s)
    assert abs(s.forces()[0, 0] - lj_force(1.0)) < 1e-10 and abs(pe - lj_energy(1.0, 2.5)) < 1e-12
    s = md.System.from_arrays(np.array([[5.0, 5.0, 5.0], [5.0 + 2.5 + 1e-9, 5.0, 5.0]]), 20.0)
    assert ff.compute_forces(s) == 0.0 and s.forces()[0, 0] == 0.0
    s = md.System.from_arrays(np.array([[5.0, 5.0, 5.0], [6.3, 5.0, 5.0]]), 20.0)
    ff.compute_forces(s)
    assert abs(ff.virial - 1.3 * lj_force(1.3)) < 1e-12 and ff.inside_pairs == 1.0
    # tests/test_forcefield.cpp:65-69, tests/test_neighbourlist.cpp:79-83, tests/test_determinism.cpp:84-91
    s = md.System.from_arrays(np.array([[1.0, 2.0, 2.0], [2.0, 2.0, 2.0]]), 4.0)
    with pytest.raises(RuntimeError, match="Cutoff must be less than half the box length"):
        ff.compute_forces(s)
    nl = md.NeighbourList(2.5, 0.2)
    with pytest.raises(RuntimeError, match="Cutoff \\+ skin must be less than half the box length"):
        nl.build(md.System.from_arrays(np.random.default_rng(0).uniform(0, 5.0, (108, 3)), 5.0))
    s = md.System.from_arrays(np.random.default_rng(1).uniform(0, 10.0, (400, 3)), 10.0)
    nl.build(s)
    ffd = md.LennardJonesForceField(1.0, 1.0, 2.5)
    ffd.set_deterministic(True)
    with pytest.raises(RuntimeError, match="reverseIndex = true"):
        ffd.compute_forces(s, nl)


def liquid(md, golden):
    """The config-1 state after 1000 steps: a liquid, cell-sorted and with its list current."""
    g = golden("config1")
    s = md.System.from_arrays(g["final_pos"], float(g["box"]), vel=g["final_vel"])
    nl = md.NeighbourList(C1["rc"], C1["skin"], reverse_index=True)
    nl.build(s)
    return s, nl


def test_float_modes_against_fp64(md, golden):
    """FP32 pair arithmetic against the FP64 path on a liquid: the reference's mixed-precision tolerance
    (tests/test_forcefield.cpp:123-149: max |dF| < 1e-5 max |F|, PE within 1e-5 relative), the same inside
    count, and bit-identical forces when repeated (fixed-point accumulation is order independent)."""
    s, nl = liquid(md, golden)
    ff = md.LennardJonesForceField(1.0, 1.0, C1["rc"])
    pe64 = ff.compute_forces(s, nl)
    f64, w64, ins64 = s.forces(), ff.virial, ff.inside_pairs
    for prec in (md.PREC_FP32FX, md.PREC_FP32):
        ff.set_precision(prec)
        pe = ff.compute_forces(s, nl)
        f = s.forces()
        assert abs(pe - pe64) < 1e-5 * abs(pe64), prec
        assert abs(ff.virial - w64) < 1e-5 * abs(w64), prec
        assert ff.inside_pairs == ins64
        assert np.abs(f - f64).max() < 1e-5 * np.abs(f64).max(), prec
        rel = np.linalg.norm(f - f64) / np.linalg.norm(f64)
        assert rel < 2e-6, (prec, rel)
        pe2 = ff.compute_forces(s, nl)
        assert pe2 == pe and np.array_equal(s.forces(), f), prec


def test_total_force_and_momentum(md, golden):
    # tests/test_forcefield.cpp:103-119 and tests/test_dynamics.cpp:59-73
    s, nl = liquid(md, golden)
    ff = md.LennardJonesForceField(1.0, 1.0, C1["rc"])
    ff.compute_forces(s, nl)
    assert np.all(np.abs(s.forces().sum(axis=1)) < 1e-10)
    integ = md.VelocityVerletIntegrator(C1["dt"])
    integ.run(s, ff, nl, 1000, record=False)
    st = s.download()
    p = (st["mass"][None, :] * st["vel"]).sum(axis=1)
    assert np.all(np.abs(p) < 1e-10)


@pytest.mark.parametrize("prec", ["PREC_FX64", "PREC_FX32"])
@pytest.mark.parametrize("cells,density", [(8, 0.8442), (6, 0.5), (20, 1.0), (10, 1.3)])
def test_fixed_point_modes_per_particle_force_error(md, golden, cells, density, prec):
    """MD_PREC_FX64 (exact fixed-point separations, double pair terms) and MD_PREC_FX32 (the same separations,
    float pair terms except for the close pairs, which are double): every particle's force within 1e-6 of the rms
    force of the FP64 path, 99 % of particles within 1e-6 of their own force, PE and virial close to FP64's
    (FX64 within 5e-8 relative; FX32 within 1e-6 and 1e-5: its float pair energies round at ~6e-8 each), the same
    inside count, bit-identical repeats. Melted liquid states (config 1's after 1000 steps, and melted boxes), and a
    compressed solid (rho = 1.3: 18 neighbours within 1.5 sigma, so FX32's rows hold more close entries than its
    double groups and take the closest 16)."""
    if cells == 8:
        s, nl = liquid(md, golden)
    else:
        s = md.fcc_system(cells, density, 2.0, seed=5)
        nl = md.NeighbourList(2.5, 0.3)
        nl.build(s)
        warm = md.LennardJonesForceField(1.0, 1.0, 2.5)
        warm.compute_forces(s, nl)
        md.VelocityVerletIntegrator(0.005).run(s, warm, nl, 300, record=False)
    ff = md.LennardJonesForceField(1.0, 1.0, 2.5)
    pe64 = ff.compute_forces(s, nl)
    f64, w64, ins64 = s.forces(), ff.virial, ff.inside_pairs
    ff.set_precision(getattr(md, prec))
    pe = ff.compute_forces(s, nl)
    f = s.forces()
    d = np.linalg.norm(f - f64, axis=0)
    mag = np.linalg.norm(f64, axis=0)
    rms = np.sqrt((mag ** 2).mean())
    print(prec, cells, density, "max|dF|/rms", d.max() / rms, "frac<=1e-6", (d <= 1e-6 * mag).mean(),
          "pe", abs(pe - pe64) / abs(pe64), "w", abs(ff.virial - w64) / abs(w64))
    assert d.max() <= 1e-6 * rms, d.max() / rms
    assert (d <= 1e-6 * mag).mean() >= 0.99, (d <= 1e-6 * mag).mean()
    if prec == "PREC_FX64":
        # frames quantised to 2^-28 put ~4e-9 on each separation: PE and virial agree to a few 1e-9 relative
        assert abs(pe - pe64) <= 5e-8 * abs(pe64) and abs(ff.virial - w64) <= 5e-8 * abs(w64)
    else:
        assert abs(pe - pe64) <= 1e-6 * abs(pe64) and abs(ff.virial - w64) <= 1e-5 * abs(w64)
    assert ff.inside_pairs == ins64
    assert ff.compute_forces(s, nl) == pe and np.array_equal(s.forces(), f)


@pytest.mark.parametrize("prec", ["fp64", "fp32fx", "fp32", "fx64", "fx32"])
def test_nve_energy_drift(md, golden, prec):
    """tests/test_dynamics.cpp:40-56 and tests/test_forcefield.cpp:151-167: |dE/E0| < 3e-4 over 2000 steps
    with more than one rebuild, starting from a melted liquid."""
    s, nl = liquid(md, golden)
    ff = md.LennardJonesForceField(1.0, 1.0, C1["rc"],
                                   precision={"fp64": md.PREC_FP64, "fp32fx": md.PREC_FP32FX, "fp32": md.PREC_FP32,
                                              "fx64": md.PREC_FX64, "fx32": md.PREC_FX32}[prec])
    pe0 = ff.compute_forces(s, nl)
    e0 = s.kinetic_energy() + pe0
    integ = md.VelocityVerletIntegrator(C1["dt"])
    rb0 = nl.rebuild_count
    pe, ke, _ = integ.run(s, ff, nl, 2000)
    drift = np.abs((pe + ke - e0) / e0).max()
    assert drift < 3e-4, drift
    assert nl.rebuild_count - rb0 > 1


def test_time_reversibility_all_pairs(md, oracle):
    # tests/test_dynamics.cpp:77-108 (4 cells, all-pairs path)
    o = oracle.fcc_system(4, 0.8442, 0.728, 42)
    st = o.state()
    s = md.System.from_arrays(st.pos, st.box, vel=st.vel)
    ff = md.LennardJonesForceField(1.0, 1.0, 2.5)
    ff.compute_forces(s)
    start = s.positions()[:, :3].copy()
    integ = md.VelocityVerletIntegrator(0.005)
    for _ in range(100):
        integ.step(s, ff)
    st = s.download()
    s.upload(vel=-st["vel"])
    for _ in range(100):
        integ.step(s, ff)
    d = s.positions()[:, :3] - start
    d -= s.box * np.round(d / s.box)
    assert np.abs(d).max() < 1e-8


def test_all_pairs_step_matches_oracle(md, oracle):
    """The O(N^2) step overload (src/Integrator.cpp:7-16) reproduces the oracle bit for bit."""
    o = oracle.fcc_system(4, 0.8442, 0.728, 42)
    off = OForceField(oracle, 1.0, 1.0, 2.5)
    off.forces(o, None, MODE_ALL_PAIRS)
    st = o.state()
    s = md.System.from_arrays(st.pos, st.box, vel=st.vel, force=st.force)
    ff = md.LennardJonesForceField(1.0, 1.0, 2.5)
    integ = md.VelocityVerletIntegrator(0.005)
    for _ in range(20):
        pe_o = off.step(o, None, 0.005, MODE_ALL_PAIRS)
        pe = integ.step(s, ff)
        assert pe == pe_o
    assert s.state_hash() == o.hash()


def test_rebuild_only_after_half_skin(md, golden):
    # tests/test_neighbourlist.cpp:59-77
    s, nl = liquid(md, golden)
    builds = nl.rebuild_count
    pos = s.positions()
    r = pos[0, :3].copy()
    r[0] += 0.4 * C1["skin"]
    r -= s.box * np.floor(r / s.box)
    pos[0, :3] = r
    s.upload(pos=pos)
    assert not nl.update(s) and nl.rebuild_count == builds
    r[0] += 0.2 * C1["skin"]
    r -= s.box * np.floor(r / s.box)
    pos = s.positions()
    pos[0, :3] = r
    s.upload(pos=pos)
    assert nl.update(s) and nl.rebuild_count == builds + 1


def test_reorder_kinetic_rescale(md, oracle):
    # tests/test_system.cpp:61-88, tests/test_dynamics.cpp:33-37
    o = oracle.fcc_system(5, 0.8442, 0.728, 42)
    st = o.state()
    s = md.System.from_arrays(st.pos, st.box, vel=st.vel)
    assert s.kinetic_energy() == o.kinetic() and s.temperature() == o.temperature()
    s.rescale_velocities(1.7)
    o.rescale(1.7)
    assert s.state_hash() == o.hash()
    assert abs(s.temperature() - 1.7) < 1e-12
    order = np.random.default_rng(3).permutation(s.n).astype(np.uint64)
    s.reorder(order)
    o.reorder(order)
    assert s.state_hash() == o.hash()
    assert np.array_equal(s.ids(), o.state().ids)


def test_ideal_gas_rdf(md):
    # tests/test_observables.cpp:71-96
    rng = np.random.default_rng(3)
    rdf = md.RadialDistribution(2.5, 25)
    for _ in range(40):
        s = md.System.from_arrays(rng.uniform(0.0, 12.0, (2000, 3)), 12.0)
        nl = md.NeighbourList(2.5, 0.2)
        nl.build(s)
        rdf.sample(s, nl)
    r, gr = rdf.radii(), rdf.values()
    assert np.all(np.abs(gr[r > 1.0] - 1.0) < 0.06)


@pytest.mark.parametrize("cells,density", [(20, 0.8442), (12, 0.5), (10, 1.0)])
def test_larger_systems_match_oracle(md, oracle, cells, density):
    """Lists and 50 deterministic steps on larger boxes (N = 32,000 / 6,912 / 4,000) equal the oracle's."""
    o = oracle.fcc_system(cells, density, 0.71, 42)
    off = OForceField(oracle, 1.0, 1.0, 2.5)
    onl = ONeighbourList(oracle, 2.5, 0.3, reverse=True)
    onl.build(o)
    off.forces(o, onl, MODE_DETERMINISTIC)
    st = o.state()
    s = md.System.from_arrays(st.pos, st.box, vel=st.vel, force=st.force)
    nl = md.NeighbourList(2.5, 0.3, reverse_index=True)
    nl.build(s)
    L, Lo = nl.download(), onl.get(o.n)
    for k in ("offsets", "neighbours", "rev_offsets", "rev_pairs"):
        assert np.array_equal(L[k], Lo[k]), k
    ff = md.LennardJonesForceField(1.0, 1.0, 2.5)
    ff.set_deterministic(True)
    integ = md.VelocityVerletIntegrator(0.005)
    pe, ke, _ = integ.run(s, ff, nl, 50)
    for k in range(50):
        assert off.step(o, onl, 0.005, MODE_DETERMINISTIC) == pe[k], k
        assert o.kinetic() == ke[k]
    assert s.state_hash() == o.hash()
    assert nl.rebuild_count == onl.rebuilds


def ragged_start(oracle, kind):
    """Non-uniform starts with empty cells and ragged rows (seeded): 'sparse' keeps 5 % of an FCC 12^3 lattice
    (rows of 0 to about 10 entries, some particles without neighbours); 'blob' is an FCC 8^3 liquid-density
    block in a 30-sigma box of vacuum (rows far above the capacity estimated from the mean density, so the
    build regrows them); 'slab' is the bottom third of an FCC 12^3 lattice; 'no_pairs' is 27 particles 4 sigma
    apart (every row empty, zero pairs)."""
    rng = np.random.default_rng({"sparse": 1, "blob": 2, "slab": 3, "no_pairs": 4}[kind])
    if kind == "sparse":
        a, box = fcc_box(12, 0.8442)
        pos = oracle.fcc(12, a)
        pos = pos[rng.random(len(pos)) < 0.05]
    elif kind == "blob":
        a, _ = fcc_box(8, 0.8442)
        pos = oracle.fcc(8, a)
        pos[:, :3] += 5.0
        box = 30.0
    elif kind == "slab":
        a, box = fcc_box(12, 0.8442)
        pos = oracle.fcc(12, a)
        pos = pos[pos[:, 2] < box / 3.0]
    else:
        g = np.arange(3) * 4.0 + 1.0
        pos = np.array([(x, y, z, 0.0) for x in g for y in g for z in g])
        box = 12.0
    vel = rng.normal(0.0, 1.0, (3, len(pos)))
    return np.ascontiguousarray(pos), float(box), vel


@pytest.mark.parametrize("kind", ["sparse", "blob", "slab", "no_pairs"])
def test_ragged_and_empty_rows_match_oracle(md, oracle, kind):
    """Empty cells, ragged and empty rows, zero pairs and row-capacity regrowth: both list builds write the
    reference's lists (src/NeighbourList.cpp:55-134), the deterministic forces, energy, virial and inside count
    and 30 steps equal the oracle's bit for bit, and the float modes stay within their error bounds of them."""
    pos, box, vel = ragged_start(oracle, kind)
    o = oracle.system(pos, box, vel=vel)
    off = OForceField(oracle, 1.0, 1.0, 2.5)
    onl = ONeighbourList(oracle, 2.5, 0.3, reverse=True)
    onl.build(o)
    pe0 = off.forces(o, onl, MODE_DETERMINISTIC)
    w0, in0 = off.virial, off.inside
    st = o.state()
    Lo = onl.get(o.n)
    if kind == "no_pairs":
        assert len(Lo["neighbours"]) == 0 and pe0 == 0.0
    for variant in (0, 1):
        s = md.System.from_arrays(pos, box, vel=vel)
        nl = md.NeighbourList(2.5, 0.3, reverse_index=True)
        nl.set_build_variant(variant)
        nl.build(s)
        assert nl.build_variant() == variant or (variant == 1 and not nl.layout()["use_tiles"])
        L = nl.download()
        for k in ("offsets", "neighbours", "rev_offsets", "rev_pairs"):
            assert np.array_equal(L[k], Lo[k]), (variant, k)
        ff = md.LennardJonesForceField(1.0, 1.0, 2.5)
        ff.set_deterministic(True)
        assert ff.compute_forces(s, nl) == pe0
        assert ff.virial == w0 and ff.inside_pairs == in0
        assert np.array_equal(s.forces(), st.force), variant
    # the float modes from the same start (the build gives the same storage order)
    rms = float(np.sqrt((st.force ** 2).sum(axis=0).mean()))
    for prec, bound in ((md.PREC_FP32FX, 2e-4), (md.PREC_FP32, 2e-4), (md.PREC_FX64, 2e-6)):
        s = md.System.from_arrays(pos, box, vel=vel)
        nl = md.NeighbourList(2.5, 0.3)
        nl.build(s)
        ff = md.LennardJonesForceField(1.0, 1.0, 2.5, precision=prec)
        pe = ff.compute_forces(s, nl)
        dF = np.sqrt(((s.forces() - st.force) ** 2).sum(axis=0))
        if kind == "no_pairs":
            assert pe == 0.0 and not s.forces().any(), prec
        else:
            assert dF.max() <= bound * rms, (prec, dF.max() / rms)
            assert abs(pe - pe0) <= 1e-5 * abs(pe0), prec
    # 30 deterministic steps (rebuilds included) against the oracle's
    s = md.System.from_arrays(pos, box, vel=vel)
    nl = md.NeighbourList(2.5, 0.3, reverse_index=True)
    nl.build(s)
    ff = md.LennardJonesForceField(1.0, 1.0, 2.5)
    ff.set_deterministic(True)
    ff.compute_forces(s, nl)
    pe, ke, _ = md.VelocityVerletIntegrator(0.005).run(s, ff, nl, 30)
    for k in range(30):
        assert off.step(o, onl, 0.005, MODE_DETERMINISTIC) == pe[k], k
        assert o.kinetic() == ke[k], k
    assert s.state_hash() == o.hash()
    assert nl.rebuild_count == onl.rebuilds


@pytest.mark.parametrize("cells,density", [(8, 0.8442), (40, 0.8442), (40, 1.0)])
def test_force_kernel_variants_agree_bit_for_bit(md, cells, density):
    """The autotuner may pick the global-gather, the shared-memory tile or a prefetching global-gather force
    kernel; all (and the fused kick) give the same bits in every precision, so the choice never changes a
    trajectory."""
    import numpy as np

    base = md.fcc_system(cells, density, 1.2, seed=7)
    nl0 = md.NeighbourList(2.5, 0.3)
    nl0.build(base)
    md.VelocityVerletIntegrator(0.005).run(base, md.LennardJonesForceField(1.0, 1.0, 2.5), nl0, 30, record=False)
    st = base.download()
    for prec in (md.PREC_FP64, md.PREC_FP32FX, md.PREC_FP32):
        results = []
        for variant in ((0, 1, 2) if prec == md.PREC_FP64 else (0, 1, 2, 3, 4)):
            s = md.System.from_arrays(st["pos"], base.box, vel=st["vel"], force=st["force"])
            nl = md.NeighbourList(2.5, 0.3)
            nl.set_force_variant(prec, variant)
            nl.build(s)
            ff = md.LennardJonesForceField(1.0, 1.0, 2.5, precision=prec)
            pe, ke, w = md.VelocityVerletIntegrator(0.005).run(s, ff, nl, 20)
            if nl.layout()["use_tiles"] or variant != 1:
                assert nl.force_variant(prec) == variant
            results.append((pe, ke, w, s.download()))
        pa, ka, wa, sa = results[0]
        for pb, kb, wb, sb in results[1:]:
            assert np.array_equal(pa, pb) and np.array_equal(ka, kb) and np.array_equal(wa, wb), prec
            for k in ("pos", "vel", "force"):
                assert np.array_equal(sa[k], sb[k]), (prec, k)


@pytest.mark.parametrize("cells,density,temperature,skin", [
    (6, 0.8442, 1.2, 0.3),   # 3 cells per side: every neighbour cell wraps
    (10, 1.0, 2.0, 0.3),
    (12, 0.5, 1.2, 0.3),
    (20, 0.8442, 0.71, 0.3),
    (12, 1.2, 1.5, 0.3),     # dense: cells above 32 particles
    (12, 0.8442, 1.2, 1.5),  # long list radius: about 55 particles per cell, two lanes' chunks per cell
])
def test_list_build_variants_agree(md, cells, density, temperature, skin):
    """The shared-memory tile build and the thread-per-particle build write the same rows: the same neighbours,
    reverse pairs and cell codes (checked through FP32FX trajectories, whose separations use the codes)."""
    base = md.fcc_system(cells, density, temperature, seed=11)
    nl0 = md.NeighbourList(2.5, skin)
    nl0.build(base)
    md.VelocityVerletIntegrator(0.005).run(base, md.LennardJonesForceField(1.0, 1.0, 2.5), nl0, 40, record=False)
    st = base.download()
    out = []
    for variant in (0, 1):
        s = md.System.from_arrays(st["pos"], base.box, vel=st["vel"], force=st["force"])
        nl = md.NeighbourList(2.5, skin, reverse_index=True)
        nl.set_build_variant(variant)
        nl.build(s)
        assert nl.build_variant() == variant or (variant == 1 and not nl.layout()["use_tiles"])
        L = nl.download()
        ff = md.LennardJonesForceField(1.0, 1.0, 2.5, precision=md.PREC_FP32FX)
        pe, ke, w = md.VelocityVerletIntegrator(0.005).run(s, ff, nl, 10)
        out.append((L, pe, w, s.download()))
    for L, pe, w, d in out[1:]:
        for k in ("offsets", "neighbours", "rev_offsets", "rev_pairs"):
            assert np.array_equal(L[k], out[0][0][k]), k
        assert np.array_equal(pe, out[0][1]) and np.array_equal(w, out[0][2])
        for k in ("pos", "vel", "force"):
            assert np.array_equal(d[k], out[0][3][k]), k


@pytest.mark.parametrize("prec", ["PREC_FP32FX", "PREC_FP32", "PREC_FX64", "PREC_FX32"])
def test_fused_next_drift_matches_separate_steps(md, prec):
    """md_run fuses each NVE step's closing kick with the next step's opening kick and drift in the float and FX64
    force kernels (new positions and frames into spare buffers, the half-skin test alongside). The trajectory, its
    energies and its rebuilds equal stepping one md_step_list at a time (separate drift kernel) bit for bit; a
    rescale step in between breaks the fusion for that step and nothing else changes."""
    p = getattr(md, prec)
    base = md.fcc_system(12, 0.8442, 1.3, seed=5)
    st = base.download()
    runs = []
    for fused in (True, False):
        s = md.System.from_arrays(st["pos"], base.box, vel=st["vel"])
        nl = md.NeighbourList(2.5, 0.3)
        ff = md.LennardJonesForceField(1.0, 1.0, 2.5, precision=p)
        nl.build(s)
        ff.compute_forces(s, nl)
        integ = md.VelocityVerletIntegrator(0.005)
        if fused:
            pe, _, _ = integ.run(s, ff, nl, 120)
            pe = list(pe)
        else:
            pe = [integ.step(s, ff, nl) for _ in range(120)]
        runs.append((np.array(pe), s.download(), nl.rebuild_count, s.state_hash()))
    (pa, sa, ra, ha), (pb, sb, rb, hb) = runs
    assert ra == rb and ra > 2
    assert np.array_equal(pa, pb)
    for k in ("pos", "vel", "force"):
        assert np.array_equal(sa[k], sb[k]), k
    assert ha == hb
    # with a rescale every 7 steps, one md_run of 49 steps equals 49 one-step runs (nothing to fuse across)
    out = []
    for one_step_calls in (False, True):
        s = md.System.from_arrays(st["pos"], base.box, vel=st["vel"])
        nl = md.NeighbourList(2.5, 0.3)
        ff = md.LennardJonesForceField(1.0, 1.0, 2.5, precision=p)
        nl.build(s)
        ff.compute_forces(s, nl)
        integ = md.VelocityVerletIntegrator(0.005)
        if one_step_calls:
            for k in range(1, 50):
                integ.run(s, ff, nl, 1, thermostat="rescale", rescale_every=7, rescale_temperature=1.0,
                          first_step=k, record=False)
        else:
            integ.run(s, ff, nl, 49, thermostat="rescale", rescale_every=7, rescale_temperature=1.0, record=False)
        out.append(s.download())
    for k in ("pos", "vel"):
        assert np.array_equal(out[0][k], out[1][k]), k


def test_frame_by_id_inverts_the_list_permutation(md):
    """md_system_frame_by_id (writeXyzFrame's data, src/Trajectory.cpp:4-25): after rebuilds have reordered
    the particles, the device gather through the ids equals the host-side inverse permutation."""
    s = md.fcc_system(8, 0.8442, 1.5, seed=3)
    nl = md.NeighbourList(2.5, 0.3)
    nl.build(s)
    ff = md.LennardJonesForceField(1.0, 1.0, 2.5)
    ff.compute_forces(s, nl)
    md.VelocityVerletIntegrator(0.005).run(s, ff, nl, 100, record=False)
    assert nl.rebuild_count > 1
    st = s.download()
    frame = s.frame_by_id()
    where = np.empty(s.n, dtype=np.int64)
    where[st["ids"].astype(np.int64)] = np.arange(s.n)
    assert np.array_equal(frame[:, :3], st["pos"][where, :3])
    assert np.array_equal(frame[:, 3:], st["vel"][:, where].T)
    assert np.array_equal(s.frame_by_id(), frame)
