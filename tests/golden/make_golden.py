"""Generate the golden vectors in tests/golden/ by running the reference itself.

The reference (nhantran1711/molecular-dynamics) is compiled unmodified from its own sources by
``make -C oracle ref`` into oracle/_ref/ (strict IEEE double arithmetic: -ffp-contract=off). This script
drives its classes through oracle/ref_harness.cpp and its md_sim binary, and writes compressed .npz files.
It needs the reference sources only to build oracle/_ref; the fixtures it writes are committed and are
all that the tests read.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import gzip
import hashlib
import json
import os
import re
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import REF_MD_SIM, RBussi, Reference, RForceField, RNeighbourList, RRdf  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# Config 1 of the workload: FCC 8x8x8 cells x 4 = 2048 atoms, density 0.8442, T* = 0.71, seed 42, r_c = 2.5,
# skin = 0.3, dt = 0.005, deterministic FP64 forces
C1 = dict(cells=8, density=0.8442, temperature=0.71, seed=42, rc=2.5, skin=0.3, dt=0.005)


def md_sim_hash(steps: int) -> str:
    out = subprocess.run([REF_MD_SIM, "8", "--deterministic", "--skin", "0.3", "--temperature", "0.71", "--equil",
                          "0", "--steps", str(steps), "--quiet"], capture_output=True, text=True, check=True,
                         env=dict(os.environ, OMP_NUM_THREADS="4")).stdout
    return re.search(r"state_hash=([0-9a-f]+)", out).group(1)


def u32(a):
    a = np.asarray(a)
    assert a.max(initial=0) < 2 ** 32
    return a.astype(np.uint32)


def config1(r: Reference):
    c = C1
    s = r.fcc_system(c["cells"], c["density"], c["temperature"], c["seed"])
    init = s.state()
    out = dict(box=init.box, init_pos=init.pos, init_vel=init.vel)

    # CellList(r_c + skin) on the unsorted lattice (src/CellList.cpp:9-52)
    ncps, cell, start, parts = s.cells_build(c["rc"] + c["skin"])
    out.update(cells_ncps=ncps, cells_cell=cell, cells_start=u32(start), cells_particles=u32(parts))

    # md_sim's start: O(N^2) forces on the lattice (src/main.cpp:190), then the first list build (:191)
    ff = RForceField(r, 1.0, 1.0, c["rc"], deterministic=True)
    out["allpairs_pe"] = ff.forces(s, None)
    out["allpairs_virial"] = ff.virial
    out["allpairs_inside"] = ff.inside
    out["allpairs_force"] = s.state().force
    nl = RNeighbourList(r, c["rc"], c["skin"], reverse=True)
    nl.build(s)
    st = s.state()
    g = nl.get(s.n)
    out.update(build_pos=st.pos, build_vel=st.vel, build_force=st.force, build_ids=st.ids,
               nl_offsets=u32(g["offsets"]), nl_neighbours=u32(g["neighbours"]),
               nl_rev_offsets=u32(g["rev_offsets"]), nl_rev_pairs=u32(g["rev_pairs"]))

    # Deterministic list forces on the sorted lattice (src/Forcefield.cpp:214-326), on a clone so the
    # trajectory below keeps md_sim's all-pairs starting forces
    s2 = s.clone()
    out["det_pe"] = ff.forces(s2, nl)
    out["det_virial"] = ff.virial
    out["det_inside"] = ff.inside
    out["det_force"] = s2.state().force

    # 1000 NVE steps from md_sim's start, recording per-step PE and KE, hashes at checkpoints, and g(r) from
    # RadialDistribution(5.0, 200) over a clone with its own NeighbourList(4.7, 0.3) every 100 steps
    rdf = RRdf(r, 5.0, 200)
    pe_all, ke_all, hashes = [], [], {}
    done = 0
    for target in (1, 10, 100, 200, 300, 400, 500, 600, 700, 800, 900, 1000):
        pe, ke = ff.run(s, nl, c["dt"], target - done, record=True)
        pe_all.append(pe)
        ke_all.append(ke)
        done = target
        hashes[target] = s.hash()
        if target % 100 == 0:
            clone = s.clone()
            big = RNeighbourList(r, 4.7, 0.3)
            big.build(clone)
            rdf.sample(clone, big)
        if target == 1:
            st1 = s.state()
            out.update(step1_pos=st1.pos, step1_vel=st1.vel, step1_force=st1.force, step1_ids=st1.ids)
    st = s.state()
    radii, gr = rdf.values()
    out.update(pe=np.concatenate(pe_all), ke=np.concatenate(ke_all), final_pos=st.pos, final_vel=st.vel,
               final_ids=st.ids, rebuilds=nl.rebuilds, rdf_radii=radii, rdf_g=gr,
               hash_steps=np.array(sorted(hashes), dtype=np.int64),
               hash_values=np.array([hashes[k] for k in sorted(hashes)], dtype=np.uint64))
    for steps in (1, 1000):
        h = md_sim_hash(steps)
        assert int(h, 16) == hashes[steps], (steps, h, hex(hashes[steps]))
    out["md_sim_hash_1"] = int(md_sim_hash(1), 16)
    return out


def small_box(r: Reference):
    """makeLiquid(4)-style 256 atoms: 2 cells per side, so the list falls back to all pairs
    (src/NeighbourList.cpp:69 and :38-52)."""
    s = r.fcc_system(4, 0.8442, 0.728, 42)
    ff = RForceField(r, 1.0, 1.0, 2.5, deterministic=True)
    nl = RNeighbourList(r, 2.5, 0.2, reverse=True)
    nl.build(s)
    ff.forces(s, nl)
    ff.run(s, nl, 0.005, 60, rescale_every=10, rescale_t=0.728)
    st = s.state()
    g = nl.get(s.n)
    s2 = s.clone()
    pe = ff.forces(s2, nl)
    return dict(box=st.box, pos=st.pos, vel=st.vel, ids=st.ids, rebuilds=nl.rebuilds, nl_offsets=u32(g["offsets"]),
                nl_neighbours=u32(g["neighbours"]), nl_rev_offsets=u32(g["rev_offsets"]),
                nl_rev_pairs=u32(g["rev_pairs"]), det_force=s2.state().force, det_pe=pe, det_virial=ff.virial,
                det_inside=ff.inside, hash=s.hash())


def bussi(r: Reference):
    """BussiThermostat(0.85, 0.05, seed 7) applied 50 times to the 500-atom lattice with no forces
    (the set-up of tests/test_observables.cpp:42-68); records the kinetic energy after each call."""
    s = r.fcc_system(5, 0.8442, 0.728, 42)
    b = RBussi(r, 0.85, 0.05, 7)
    ke0 = s.kinetic()
    ke = []
    for _ in range(50):
        b.apply(s, 0.005)
        ke.append(s.kinetic())
    st = s.state()
    return dict(ke0=ke0, ke=np.array(ke), final_vel=st.vel, hash=s.hash())


# md_sim command lines whose outputs the GPU md_sim must reproduce byte for byte (FP64, --deterministic) or
# within tolerance (the default and --mixed force paths)
MD_SIM_CASES = {
    "nve_rescale": ["8", "--deterministic", "--skin", "0.3", "--temperature", "0.71", "--equil", "100", "--steps",
                    "300", "--xyz-every", "100"],
    "nvt_melt_rdf": ["6", "--deterministic", "--nvt", "--melt", "--seed", "7", "--equil", "60", "--steps", "200",
                     "--density", "0.9", "--temperature", "1.2"],
    "brute": ["5", "--brute", "--deterministic", "--equil", "20", "--steps", "60", "--dt", "0.004"],
    "default_list": ["8", "--skin", "0.3", "--temperature", "0.71", "--equil", "50", "--steps", "200"],
    "mixed": ["8", "--mixed", "--skin", "0.3", "--temperature", "0.71", "--equil", "50", "--steps", "200"],
}


def md_sim_case(binary: str, args: list[str], workdir: str) -> dict:
    """Runs one md_sim command line with --csv/--rdf/--xyz outputs under `workdir`; returns its stdout (timing and
    thread-count lines dropped), the RESULT fields that do not depend on timing, and the output files' text."""
    files = {"csv": os.path.join(workdir, "run.csv"), "xyz": os.path.join(workdir, "run.xyz")}
    extra = ["--csv", files["csv"], "--xyz", files["xyz"]]
    if "--brute" not in args:
        files["rdf"] = os.path.join(workdir, "run.rdf")
        extra += ["--rdf", files["rdf"]]
    out = subprocess.run([binary, *args, *extra], capture_output=True, text=True, check=True,
                         env=dict(os.environ, OMP_NUM_THREADS="4")).stdout
    result = dict(kv.split("=", 1) for kv in re.search(r"^RESULT (.*)$", out, re.M).group(1).split())
    for k in ("threads", "seconds", "ms_per_step"):
        result.pop(k)
    table = [ln for ln in out.splitlines() if not ln.startswith(("N = ", "Production took", "RESULT"))]
    texts = {k: open(f).read() for k, f in files.items()}
    # The trajectory is kept as its digest and the head of its first frame
    xyz = texts.pop("xyz")
    texts["xyz_sha256"] = hashlib.sha256(xyz.encode()).hexdigest()
    texts["xyz_head"] = "".join(xyz.splitlines(keepends=True)[:102])
    return dict(stdout=table, result=result, files=texts)


def md_sim_golden() -> dict:
    import tempfile

    with tempfile.TemporaryDirectory() as d:
        return {name: dict(args=args, **md_sim_case(REF_MD_SIM, args, d)) for name, args in MD_SIM_CASES.items()}


def main():
    r = Reference()
    r.set_threads(4)
    np.savez_compressed(os.path.join(OUT, "config1.npz"), **config1(r))
    np.savez_compressed(os.path.join(OUT, "small_box.npz"), **small_box(r))
    np.savez_compressed(os.path.join(OUT, "bussi.npz"), **bussi(r))
    with gzip.open(os.path.join(OUT, "md_sim.json.gz"), "wt") as f:
        json.dump(md_sim_golden(), f)
    for f in sorted(os.listdir(OUT)):
        if f.endswith((".npz", ".gz")):
            print(f, os.path.getsize(os.path.join(OUT, f)))


if __name__ == "__main__":
    main()
