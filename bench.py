#!/usr/bin/env python
"""Throughput of the Lennard-Jones hot path on B200: atom-steps/s of NVE velocity-Verlet steps (cell list,
neighbour list at its natural rebuild rate, LJ forces, integration) on the 4,000,000-atom FCC fluid.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (the large single system of the benchmark): FCC 100^3 x 4 = 4,000,000 atoms, density 0.8442,
T* = 0.71 after a 200-step rescale equilibration from a T = 2 melt (md_sim's --melt schedule), r_c = 2.5
truncated and shifted, skin 0.3, dt 0.005, NVE. The headline precision is MD_PREC_FX32 (FP32 pair arithmetic
with 64-bit fixed-point force accumulation, the close pairs in double on exact fixed-point separations), the
mode that keeps every particle's force within 1e-6 of the FP64 path; the FP64 path (bit-identical to the
reference's deterministic mode) is timed beside it on the same state, and FP32FX (float for every pair) and
the other modes beside that. Inputs are synthetic (seeded lattice and velocities) and the working set
(~1.4 GB) is far larger than the 126 MB L2.

One rank per GPU (torchrun); ranks run independent replicas (seed 42 + rank), so scaling is weak and no
collective touches the data path. `value` is atom-steps/s summed over ranks, timed with CUDA events on the
library's stream and taken as the max over ranks.

--impl reference times the reference's own OpenMP CPU code (compiled from its sources into oracle/_ref) on
this host's cores for a bounded sample of the same workload; rank 0 alone runs it.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "molecular-dynamics_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "atom-steps/s at N=4M, FP32+fixed-pt vs FP64 GPU at <=1e-6 rel force err; %roofline"
FALLBACK_HBM_GBS = 6650.0
# precision name -> (md_precision value, arithmetic of the pair path)
PRECISIONS = {"fp32fx": (1, "f32+i64"), "fp32": (2, "f32"), "fp64": (0, "f64"), "fx64": (3, "i32+f64+i64"),
              "fx32": (4, "i32+f32+i64 (f64 for close pairs)")}


def args_parse():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2000)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--cells", type=int, default=100, help="FCC cells per side (N = 4 cells^3)")
    p.add_argument("--density", type=float, default=0.8442)
    p.add_argument("--temperature", type=float, default=0.71)
    p.add_argument("--equil", type=int, default=200)
    p.add_argument("--precision", choices=list(PRECISIONS), default="fx32")
    p.add_argument("--fp64-steps", type=int, default=None,
                   help="steps of the FP64 comparison run from the headline's starting state (default: --steps; 0: skip)")
    p.add_argument("--side-steps", type=int, default=300,
                   help="steps of the runs of the other float precisions on the same state (0: skip)")
    p.add_argument("--cpu-steps", type=int, default=None,
                   help="timed reference steps of the CPU samples (default: --steps, capped at 200; 0: skip the "
                        "cpu_baseline leg); the untimed steps are --warmup, capped at 20")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--sweep", choices=["precision"], default=None,
                   help="instead of the headline line: the N=256,000 precision sweep over densities {0.5, 0.8442, 1.0} "
                        "x T {0.71, 1.5, 3.0} (one JSON line per state point; --steps NVE steps each)")
    p.add_argument("--sweep-replicas", type=int, default=4,
                   help="replicas per state point of the precision sweep (error bars from their spread)")
    p.add_argument("--nist", action="store_true",
                   help="instead of the headline line: the reference's NIST validation (bench/validate.py: 16 state "
                        "points x 8 replicas of 500 atoms, 10,000 + 20,000 steps) in one md_batch, one JSON line per "
                        "state point with U, P, replica error bars and z-scores against the NIST tables")
    p.add_argument("--nist-precision", choices=["fp64", "fp32fx", "fp32"], default="fp64")
    p.add_argument("--replica-steps", type=int, default=5000,
                   help="steps of the batched-replica workload (512 replicas; 0: skip)")
    p.add_argument("--replicas", type=int, default=512)
    p.add_argument("--replica-precision", choices=["fp64", "fp32fx", "fp32"], default=None,
                   help="precision of the batched-replica workload (default: the headline precision where the batch "
                        "engine has it, else fp32fx)")
    p.add_argument("--adjoint-steps", type=int, default=200,
                   help="trajectory length of the differentiation workload (N = 32,000; 0: skip)")
    p.add_argument("--force-variant", type=int, default=-1,
                   help="list force kernel of the headline run: -1 autotunes, 0-4 pin one (md_nlist_set_force_variant)")
    p.add_argument("--graph-chunk", type=int, default=64,
                   help="md_run's CUDA-graph chunk length (md_system_set_graph); 0 runs every step from the host, as "
                        "profilers need (ncu cannot profile kernels in graphs with conditional nodes)")
    p.add_argument("--profile-region", action="store_true",
                   help="bracket the timed steps with cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    return p.parse_args()


def workload(a) -> dict:
    n = 4 * a.cells ** 3
    return {"workload": f"lj_fcc{a.cells}_n{n}_rho{a.density}_T{a.temperature}_rc2.5_skin0.3_dt0.005_nve",
            "n_atoms": n, "density": a.density, "temperature": a.temperature, "cutoff": 2.5, "skin": 0.3,
            "dt": 0.005, "equilibration": f"{a.equil} steps, rescale every 10 to T=2 then T={a.temperature}",
            "precision": a.precision, "l2": "inputs larger than L2 (no flush needed)"}


# ---- reference CPU path --------------------------------------------------------------------------------------

REF_MAX_STEPS = 200  # cap of the CPU samples (about 0.6 s per 4M-atom step on 16 host threads)
REF_MAX_WARMUP = 20


def cpu_sample_shape(a) -> tuple[int, int]:
    """Timed and untimed steps of a CPU sample: the run's own --steps/--warmup, capped so the sample stays
    within a few minutes. Both CPU legs (the GPU arm's cpu_baseline and the reference arm) use this."""
    steps = a.cpu_steps if a.cpu_steps is not None else a.steps
    return max(1, min(steps, REF_MAX_STEPS)), min(a.warmup, REF_MAX_WARMUP)


def reference_sample(a, steps: int, warmup: int) -> dict:
    """Time the reference's OpenMP path on all host cores: the same 4M-atom FCC start, list build and list
    forces, then `warmup` untimed and `steps` timed NVE steps of the default (non-deterministic) force path, as
    md_sim runs without --deterministic, with list rebuilds at their natural rate inside the timed steps. The
    library timed is the reference's unmodified sources built with its release flags (oracle/_ref/
    libmdref_stock_*.so); the strict parity build is used only where those were not built."""
    from oracle.oracle import Oracle, Reference, RForceField, RNeighbourList, stock_reference_path

    threads = os.cpu_count() or 1
    path, build = stock_reference_path()
    if os.path.exists(path):
        r = Reference(path)
        r.set_threads(threads)
        t0 = time.perf_counter()
        s = r.fcc_system(a.cells, a.density, a.temperature, 42)
        nl = RNeighbourList(r, 2.5, 0.3)
        nl.build(s)
        ff = RForceField(r, 1.0, 1.0, 2.5)
        ff.forces(s, nl)
        setup = time.perf_counter() - t0
        if warmup:
            ff.run(s, nl, 0.005, warmup)
        rb0 = nl.rebuilds
        t0 = time.perf_counter()
        ff.run(s, nl, 0.005, steps)
        dt = time.perf_counter() - t0
        kind, cores, rebuilds = "reference", r.max_threads(), nl.rebuilds - rb0
    else:  # the oracle's serial restatement, when the reference could not be built on this machine
        from oracle.oracle import MODE_DEFAULT, OForceField, ONeighbourList
        build = "the oracle's serial restatement"
        o = Oracle()
        t0 = time.perf_counter()
        s = o.fcc_system(a.cells, a.density, a.temperature, 42)
        nl = ONeighbourList(o, 2.5, 0.3)
        nl.build(s)
        ff = OForceField(o, 1.0, 1.0, 2.5)
        ff.forces(s, nl, MODE_DEFAULT)
        setup = time.perf_counter() - t0
        for _ in range(warmup):
            ff.step(s, nl, 0.005, MODE_DEFAULT)
        rb0 = nl.rebuilds
        t0 = time.perf_counter()
        for _ in range(steps):
            ff.step(s, nl, 0.005, MODE_DEFAULT)
        dt = time.perf_counter() - t0
        kind, cores, rebuilds = "port", 1, nl.rebuilds - rb0
    n = 4 * a.cells ** 3
    return {"value": n * steps / dt, "unit": "atom-steps/s", "cores": cores, "kind": kind,
            "sample": f"{steps} timed NVE steps (after {warmup} untimed) of the same {n}-atom FCC start, "
                      f"list start, FP64 default force path, {rebuilds} list rebuilds inside the timed steps; "
                      f"{build}; setup {setup:.1f} s untimed",
            "ms_per_step": 1e3 * dt / steps, "steps": steps, "warmup": warmup, "rebuilds": rebuilds}


def run_reference_arm(a):
    if int(os.environ.get("RANK", "0")) != 0:
        return  # rank 0 alone runs the CPU reference
    steps, warm = cpu_sample_shape(a)
    cb = reference_sample(a, steps, warm)
    line = {"metric": METRIC, "value": cb["value"], "unit": "atom-steps/s", "impl": "reference",
            "n_gpus": a.gpus, "steps": steps, "warmup": warm, "ms_per_step": cb["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload(a),
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---- clocks ------------------------------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi every 200 ms on one GPU during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self) -> dict:
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.strip() == "Active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---- ranks -------------------------------------------------------------------------------------------------

def max_over_ranks(x: float) -> float:
    """Max of a per-rank time over all ranks of the default process group (NCCL on GPUs, gloo on CPUs)."""
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world: int, n_atoms: int, steps: int, max_ms: float) -> float:
    """Whole-job atom-steps/s of `world` independent replicas, timed by the slowest rank."""
    return world * n_atoms * steps / (max_ms / 1e3)


# ---- GPU arm ------------------------------------------------------------------------------------------------

def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, copy)"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback 6.65 TB/s"


def ncu_traffic_per_atom(precision: str):
    """DRAM bytes per atom of the precision's force kernel from the committed ncu summary, or None."""
    try:
        with open(os.path.join(ROOT, "profiles", f"force_{precision}_traffic.json")) as f:
            d = json.load(f)
        return float(d["dram_bytes_per_launch"]) / float(d["n_atoms"])
    except (OSError, KeyError, ValueError):
        return None


def force_errors(md, s, nl) -> dict:
    """Per-particle force error of the float modes against the FP64 path on the same state."""
    import numpy as np

    ff64 = md.LennardJonesForceField(1.0, 1.0, 2.5, precision=md.PREC_FP64)
    pe64 = ff64.compute_forces(s, nl)
    w64 = ff64.virial
    f64 = s.forces()
    out = {}
    for name in ("fp32fx", "fp32", "fx64", "fx32"):
        ff = md.LennardJonesForceField(1.0, 1.0, 2.5, precision=PRECISIONS[name][0])
        pe = ff.compute_forces(s, nl)
        f = s.forces()
        d = np.linalg.norm(f - f64, axis=0)
        mag = np.linalg.norm(f64, axis=0)
        rel = d / np.maximum(mag, 1e-300)
        rms = float(np.sqrt((mag ** 2).mean()))
        out[name] = {"max_abs_dF_over_max_F": float(np.abs(f - f64).max() / np.abs(f64).max()),
                     "rms_dF_over_rms_F": float(np.sqrt((d ** 2).mean()) / rms),
                     "max_particle_dF_over_rms_F": float(d.max() / rms),
                     "per_particle_rel_p50": float(np.percentile(rel, 50)),
                     "per_particle_rel_p99": float(np.percentile(rel, 99)),
                     "per_particle_rel_max": float(rel.max()),
                     "frac_particles_rel_le_1e-6": float((rel <= 1e-6).mean()),
                     "pe_rel": float(abs(pe - pe64) / abs(pe64)), "virial_rel": float(abs(ff.virial - w64) / abs(w64))}
    ff = md.LennardJonesForceField(1.0, 1.0, 2.5, precision=md.PREC_FP32FX)
    ff.compute_forces(s, nl)
    return out


def block_error(x, blocks: int = 10):
    """Mean and its standard error from `blocks` block averages of the rows of x (samples x replicas)."""
    import numpy as np

    m = (x.shape[0] // blocks) * blocks
    b = x[:m].reshape(blocks, m // blocks, *x.shape[1:]).mean(axis=1)
    return b.mean(axis=0), b.std(axis=0, ddof=1) / np.sqrt(blocks)


def replica_workload(md, a, device: int) -> dict:
    """The batched-replica workload: `a.replicas` independent LJ systems, N = 4 n^3 with n uniform in [4, 20],
    density uniform in [0.7, 0.95], T* uniform in [0.7, 2.0] (all drawn from one generator with a fixed seed),
    seeded FCC starts, Bussi NVT with tau = 0.1, dt = 0.005, r_c = 2.5, skin 0.3, in one md_batch (CUDA graphs of
    100 steps, per-replica device-side rebuilds). Aggregate atom-steps/s over `a.replica_steps` steps after 100
    untimed ones, and per-replica means with block-averaged error bars of PE/N and the virial pressure."""
    import numpy as np
    import torch

    rng = np.random.default_rng(20240611)
    R = a.replicas
    cells = rng.integers(4, 21, size=R)
    rho = rng.uniform(0.7, 0.95, size=R)
    temp = rng.uniform(0.7, 2.0, size=R)
    systems = []
    for k in range(R):
        s = md.fcc_system(int(cells[k]), float(rho[k]), float(temp[k]), seed=1000 + k, device=device)
        d = s.download()
        systems.append((d["pos"], s.box, d["vel"], None))
        del s
    name = a.replica_precision or (a.precision if a.precision in ("fp64", "fp32fx", "fp32") else "fp32fx")
    b = md.Batch(systems, precision=PRECISIONS[name][0], thermostat="bussi", temperatures=temp, seeds=1000 + np.arange(R),
                 bussi_tau=0.1, energy_every=10, chunk_steps=100, device=device)
    info = b.info()
    b.run(100)
    stream = torch.cuda.ExternalStream(b.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    l0 = b.info()["launches"]
    e0.record(stream)
    pe, w, ke = b.run(a.replica_steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    n = np.array([len(p) for p, *_ in systems], dtype=np.float64)
    vol = np.array([bx ** 3 for _, bx, *_ in systems])
    keep = pe.shape[0] // 5  # the first fifth of the samples is equilibration
    pe_n, pe_err = block_error(pe[keep:] / n)
    p_mean, p_err = block_error((2 * ke[keep:] + w[keep:]) / (3 * vol))
    t_mean = (2 * ke[keep:] / (3 * n - 3)).mean(axis=0)
    return {"workload": f"{R} replicas, n~U[4,20] (N 256-32000), rho~U[0.7,0.95], T~U[0.7,2.0], Bussi tau=0.1, "
                        f"dt=0.005, rc=2.5, skin=0.3, {a.replica_steps} steps",
            "atoms": info["atoms"], "value": info["atoms"] * a.replica_steps / (ms / 1e3), "unit": "atom-steps/s",
            "ms_per_step": ms / a.replica_steps, "precision": name,
            "force_variant": b.force_variant(), "gpu_launches": b.info()["launches"] - l0,
            "rebuilds_per_replica_mean": float(b.rebuilds().mean()),
            "pe_per_atom_stderr": {"median": float(np.median(pe_err)), "max": float(pe_err.max())},
            "pressure_stderr": {"median": float(np.median(p_err)), "max": float(p_err.max())},
            "mean_T_rel_dev_from_target": {"median": float(np.median(np.abs(t_mean / temp - 1))),
                                           "max": float(np.abs(t_mean / temp - 1).max())},
            "examples": [{"n": int(n[k]), "rho": float(rho[k]), "T": float(temp[k]),
                          "pe_per_atom": [float(pe_n[k]), float(pe_err[k])], "pressure": [float(p_mean[k]), float(p_err[k])]}
                         for k in range(3)]}


def adjoint_workload(md, a, device: int) -> dict:
    """The differentiation workload: N = 32,000 (FCC 20^3 x 4), density 0.8442, T* = 1.0, `a.adjoint_steps` NVE
    steps of dt = 0.005, checkpoints every 20; timings of forward and backward, and the gradients of mean U with
    respect to epsilon, sigma and the initial positions (along one random unit direction) against central
    differences at h = 1e-4 (the workload's nominal step: the cutoff's force jump enters the stencil), 1e-7 and
    1e-8 (relative error per step size)."""
    import numpy as np
    import torch

    s = md.fcc_system(20, 0.8442, 1.0, seed=42, device=device)
    d = s.download()
    eng = md.Adjoint(d["pos"], s.box, d["vel"], steps=a.adjoint_steps, checkpoint_every=20, device=device)
    eng.forward()  # untimed forward and backward: module loading and first-use allocations stay out of the timings
    eng.backward(1.0, 0.0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    mu, mp = eng.forward()
    t1 = time.perf_counter()
    g = eng.backward(1.0, 0.0)
    t2 = time.perf_counter()
    pos0 = d["pos"]
    rng = np.random.default_rng(3)
    u = np.zeros_like(pos0)
    u[:, :3] = rng.standard_normal((len(pos0), 3))
    u /= np.linalg.norm(u)

    def J(eps=1.0, sig=1.0, pos=pos0):
        eng.set_parameters(eps, sig)
        eng.set_state(pos=pos)
        return eng.forward()[0]

    checks = {"epsilon": (g["d_epsilon"], lambda h: J(eps=1.0 + h)),
              "sigma": (g["d_sigma"], lambda h: J(sig=1.0 + h)),
              "positions": (float((g["d_pos"].T * u[:, :3]).sum()), lambda h: J(pos=pos0 + h * u))}
    fd = {}
    for name, (adj, f) in checks.items():
        fd[name] = {str(h): abs((f(h) - f(-h)) / (2 * h) - adj) / abs(adj) for h in (1e-4, 1e-7, 1e-8)}
    J()
    n = s.n
    return {"workload": f"N={n} FCC 20^3x4, rho=0.8442, T=1.0, {a.adjoint_steps} NVE steps, checkpoints every 20",
            "mean_pe": mu, "mean_pressure": mp, "forward_s": t1 - t0, "backward_s": t2 - t1,
            "forward_atom_steps_per_s": n * a.adjoint_steps / (t1 - t0),
            "d_mean_pe_d_epsilon": g["d_epsilon"], "d_mean_pe_d_sigma": g["d_sigma"],
            "fd_rel_err": fd,
            "fd_note": "central differences of mean U; h = 1e-4 puts pairs across the cutoff's force jump inside the "
                       "stencil, so the clean figures are the smaller h (the GPU gradients equal the FP64 CPU "
                       "adjoint's bit for bit)",
            "rebuilds": eng.info()["rebuilds"]}


def run_gpu_arm(a):
    import numpy as np
    import torch

    rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    import mdgpu as md

    prec = PRECISIONS[a.precision][0]
    n = 4 * a.cells ** 3
    dt = 0.005
    s = md.fcc_system(a.cells, a.density, a.temperature, seed=42 + rank, device=local)
    s.set_graph(a.graph_chunk)
    nl = md.NeighbourList(2.5, 0.3)
    if a.force_variant >= 0:
        nl.set_force_variant(prec, a.force_variant)
    ff = md.LennardJonesForceField(1.0, 1.0, 2.5, precision=prec)
    integ = md.VelocityVerletIntegrator(dt)
    nl.build(s)
    ff.compute_forces(s, nl)
    if a.equil:
        integ.run(s, ff, nl, a.equil, thermostat="rescale", rescale_every=10, rescale_temperature=a.temperature,
                  melt_until=a.equil // 3, melt_temperature=2.0, record=False)
    errors = force_errors(md, s, nl) if rank == 0 else None
    if a.warmup:
        integ.run(s, ff, nl, a.warmup, first_step=a.equil + 1)

    # the state the timed steps start from: the FP64 and other-precision runs below start from it too
    start = s.download() if rank == 0 and (a.fp64_steps != 0 or a.side_steps) else None
    stream = torch.cuda.ExternalStream(s.stream)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    # the force-kernel events are recorded inside md_run's CUDA graphs; the graphs of the timed run are captured
    # here, before the timed region (md_run_prepare)
    s.profile(True)
    integ.prepare(s, ff, nl, a.steps, first_step=a.equil + a.warmup + 1)
    torch.cuda.synchronize()
    s.synchronize()
    rb0, l0 = nl.rebuild_count, s.launch_count
    if a.profile_region:
        torch.cuda.profiler.start()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        pe, ke, _ = integ.run(s, ff, nl, a.steps, first_step=a.equil + a.warmup + 1)
        ev1.record(stream)
        ev1.synchronize()
    if a.profile_region:
        torch.cuda.profiler.stop()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    force_ms, force_n = s.profile_read()
    s.profile(False)
    launches = s.launch_count - l0
    variant = nl.force_variant(prec)
    rebuilds = nl.rebuild_count - rb0
    pairs = nl.pair_count
    if dist:
        ms = max_over_ranks(ms)
        dist.barrier()
    e0 = pe[0] + ke[0]
    drift = float(np.abs((pe + ke - e0) / e0).max())

    # The FP64 path (bit-identical to the reference's deterministic mode) and the other precisions, each from the
    # state the timed steps started from: list build, forces (the first force call tunes the kernel), then the
    # steps timed with CUDA events and their energy drift, max |E_k - E_1| / |E_1| as for the headline run
    def side_run(precision: int, steps: int) -> dict:
        s2 = md.System.from_arrays(start["pos"], s.box, vel=start["vel"], force=start["force"], device=local)
        nl2 = md.NeighbourList(2.5, 0.3)
        nl2.build(s2)
        ff2 = md.LennardJonesForceField(1.0, 1.0, 2.5, precision=precision)
        ff2.compute_forces(s2, nl2)
        st2 = torch.cuda.ExternalStream(s2.stream)
        e0_, e1_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s2.profile(True)
        integ.prepare(s2, ff2, nl2, steps)
        s2.synchronize()
        rb = nl2.rebuild_count
        e0_.record(st2)
        pe2, ke2, _ = integ.run(s2, ff2, nl2, steps)
        e1_.record(st2)
        e1_.synchronize()
        ms2 = e0_.elapsed_time(e1_)
        f_ms, f_n = s2.profile_read()
        return {"value": n * steps / (ms2 / 1e3), "steps": steps, "ms_per_step": ms2 / steps,
                "force_kernel_ms": f_ms / max(f_n, 1), "rebuilds": nl2.rebuild_count - rb,
                "max_drift": float(np.abs((pe2 + ke2 - pe2[0] - ke2[0]) / (pe2[0] + ke2[0])).max()),
                "start": "the state the headline's timed steps started from"}

    fp64_steps = a.steps if a.fp64_steps is None else a.fp64_steps
    fp64 = side_run(md.PREC_FP64, fp64_steps) if fp64_steps and rank == 0 else None
    others = {}
    if a.side_steps and rank == 0:
        for name in ("fx32", "fp32fx", "fx64", "fp32"):
            if name != a.precision:
                others[name] = side_run(PRECISIONS[name][0], a.side_steps)

    # End to end through the public C-ABI with host buffers: pinned host state -> device, list build,
    # initial forces, K steps returning per-step PE/KE/virial, final positions and velocities -> host.
    e2e = None
    if not a.no_e2e:
        st = s.download()
        h_pos = torch.empty((n, 4), dtype=torch.float64, pin_memory=True)
        h_vel = torch.empty((3, n), dtype=torch.float64, pin_memory=True)
        h_mass = torch.empty((n,), dtype=torch.float64, pin_memory=True)
        h_pos.numpy()[:] = st["pos"]
        h_vel.numpy()[:] = st["vel"]
        h_mass.numpy()[:] = st["mass"]
        out_pos = torch.empty((n, 4), dtype=torch.float64, pin_memory=True)
        out_vel = torch.empty((3, n), dtype=torch.float64, pin_memory=True)
        s2 = md.System(n, s.box, device=local)
        nl2 = md.NeighbourList(2.5, 0.3)
        ff2 = md.LennardJonesForceField(1.0, 1.0, 2.5, precision=prec)
        st2 = torch.cuda.ExternalStream(s2.stream)
        x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        # one untimed pass, as a caller's first call: it allocates the system's, list's and force field's device
        # buffers and captures the run's graphs, which later calls reuse
        s2.upload(pos=h_pos.numpy(), vel=h_vel.numpy(), mass=h_mass.numpy())
        nl2.build(s2)
        ff2.compute_forces(s2, nl2)
        integ.prepare(s2, ff2, nl2, a.steps)
        if dist:
            dist.barrier()
        s2.synchronize()
        x0.record(st2)
        s2.upload(pos=h_pos.numpy(), vel=h_vel.numpy(), mass=h_mass.numpy())
        nl2.build(s2)
        ff2.compute_forces(s2, nl2)
        pe2, ke2, w2 = integ.run(s2, ff2, nl2, a.steps)
        import ctypes
        md._check(md.LIB.md_system_download(s2.h, ctypes.cast(out_pos.data_ptr(), md._PD),
                                            ctypes.cast(out_vel.data_ptr(), md._PD), None, None, None))
        x1.record(st2)
        x1.synchronize()
        ems = x0.elapsed_time(x1)
        if dist:
            ems = max_over_ranks(ems)
        h2d = n * (32 + 24 + 8)
        d2h = n * (32 + 24) + a.steps * 3 * 8
        e2e = {"value": replica_throughput(world, n, a.steps, ems), "unit": "atom-steps/s",
               "h2d_bytes_per_step": h2d / a.steps, "d2h_bytes_per_step": d2h / a.steps,
               "includes": "pinned H2D of positions/velocities/masses, list build, initial forces, all steps with "
                           "per-step PE/KE/virial read back, D2H of final positions/velocities (after one untimed "
                           "pass that allocated the device buffers and captured the run's graphs)"}
        del s2, nl2, ff2

    replicas = replica_workload(md, a, local) if rank == 0 and a.replica_steps > 0 else None
    adjoint = adjoint_workload(md, a, local) if rank == 0 and a.adjoint_steps > 0 else None

    cpu = None
    if rank == 0 and world == 1 and a.cpu_steps != 0:
        cb = reference_sample(a, *cpu_sample_shape(a))
        cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    peak, peak_src = measured_peak()
    kernel_s = (force_ms / max(force_n, 1)) / 1e3
    # DRAM bytes per atom of one force launch: the particle's own coordinates, its force, the full-list int32
    # indices (neighbour coordinates are gathered through L1/L2 and counted once, in the own term), the fused
    # closing kick (velocity read and write, mass) and, in the float modes, the fused next kick and drift
    # (position in and out, reference position, build cell, new float frame); FP64 adds its own-pair r^2
    # records for the ordered energy sums.
    own = 32 if a.precision == "fp64" else 16
    bytes_per_atom = own + 24 + 4 * 2 * pairs / n + 56
    if a.precision in ("fp32fx", "fp32", "fx32", "fx64"):
        bytes_per_atom += 32 + 32 + 4 + 32 + 16
    if a.precision == "fp64":
        bytes_per_atom += 8 * pairs / n
    achieved = bytes_per_atom * n / kernel_s / 1e9
    if a.precision == "fx32":
        bytes_per_atom += 32  # the own fixed-point frame read and the next one written, beside the float frames
    tpa = ncu_traffic_per_atom(a.precision)
    # the FP32-pipe side of the roofline (the force kernel sits between the two): 23 flop per ordered pair of
    # the full list (separation, r^2, reciprocal, F/r, three accumulating FMAs) and 6 per unordered pair for the
    # energy and virial, against the nominal FP32 peak (SMs x 128 lanes x 2 flop x the max SM clock sampled)
    clocks = clk.summary()
    flops_per_atom = 23 * 2 * pairs / n + 6 * pairs / n
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    fp32_peak = sms * 128 * 2 * clocks.get("sm_max_mhz", 1965.0) * 1e6 / 1e12 if clocks.get("sm_max_mhz") else None
    fp32_achieved = flops_per_atom * n / kernel_s / 1e12
    value = replica_throughput(world, n, a.steps, ms)
    line = {"metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": PRECISIONS[a.precision][1],
            "data": "synthetic", "config": workload(a),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None if tpa is None else tpa * n,
                         "kernel": {"fp64": "k_force_fp64", "fx64": "k_force_fx64_rows",
                                    "fx32": "k_force_fx32"}.get(a.precision, "k_force_fp32"),
                         "force_variant": {0: "global gathers", 1: "shared-memory tiles",
                                           2: ("global gathers, branch-free quads" if a.precision == "fp64"
                                               else "global gathers, rows prefetched"),
                                           3: "global gathers, rows prefetched, registers capped",
                                           4: "global gathers, rows prefetched, resident grid"}.get(variant, str(variant)),
                         "kernel_ms": kernel_s * 1e3,
                         "algorithmic_bytes_per_atom": bytes_per_atom, "peak_source": peak_src,
                         "fp32": {"flops_per_atom": flops_per_atom, "achieved_tflops": fp32_achieved,
                                  "nominal_peak_tflops": fp32_peak,
                                  "frac": None if not fp32_peak else fp32_achieved / fp32_peak}},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
            "rebuilds": rebuilds, "half_list_pairs": pairs, "max_energy_drift": drift,
            "fp64": fp64, "speedup_vs_fp64": None if fp64 is None else value / world / fp64["value"],
            "other_precisions": others,
            "force_error_vs_fp64": errors, "replicas": replicas, "adjoint": adjoint}
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


# ---- precision sweep (the N = 256,000 density x temperature grid) -------------------------------------------

def precision_sweep(cells=40, densities=(0.5, 0.8442, 1.0), temperatures=(0.71, 1.5, 3.0), steps=10000,
                    equil=200, rdf_every=100, device=0, replicas=4):
    """For each state point and each of `replicas` replicas (FCC start with velocities from seed 42 + r): the
    melt/rescale equilibration in FP64 (T = 2 for the first third, then T, every 10 steps), then `steps` NVE steps
    from that replica's equilibrated state in each precision. Force errors of the float modes against FP64 are
    taken on replica 0's equilibrated state. Yields one dict per state point; per precision the replica means and
    standard errors of the energy drift (max |E - E0| / |E0| and the per-step slope), the mean virial pressure
    P = (2K + W) / 3V and atom-steps/s, g(r) from the run's list pairs to r_c every `rdf_every` steps, and against
    FP64, replica by replica (each pair of runs starts from the same state): the mean pressure difference with its
    standard error and z-score, and the largest g(r) difference of the replica-mean g(r) in units of the replica
    standard error of that bin."""
    import numpy as np

    import mdgpu as md

    names = ("fp64", "fp32fx", "fp32", "fx64", "fx32")
    for rho in densities:
        for temp in temperatures:
            runs = {name: [] for name in names}
            errors = None
            n_atoms = 0
            for rep in range(replicas):
                s = md.fcc_system(cells, rho, temp, seed=42 + rep, device=device)
                nl = md.NeighbourList(2.5, 0.3)
                ff = md.LennardJonesForceField(1.0, 1.0, 2.5, precision=md.PREC_FP64)
                integ = md.VelocityVerletIntegrator(0.005)
                nl.build(s)
                ff.compute_forces(s, nl)
                integ.run(s, ff, nl, equil, thermostat="rescale", rescale_every=10, rescale_temperature=temp,
                          melt_until=equil // 3, melt_temperature=2.0, record=False)
                if rep == 0:
                    errors = force_errors(md, s, nl)
                start = s.download()
                vol = s.box ** 3
                n_atoms = s.n
                for name in names:
                    prec = PRECISIONS[name][0]
                    r = md.System.from_arrays(start["pos"], s.box, vel=start["vel"], force=start["force"],
                                              device=device)
                    rl = md.NeighbourList(2.5, 0.3)
                    rf = md.LennardJonesForceField(1.0, 1.0, 2.5, precision=prec)
                    rl.build(r)
                    pe0 = rf.compute_forces(r, rl)
                    e0 = r.kinetic_energy() + pe0
                    rdf = md.RadialDistribution(2.5, 100)
                    t0 = time.perf_counter()
                    pe, ke, w = integ.run(r, rf, rl, steps, rdf=rdf, rdf_every=rdf_every)
                    dt = time.perf_counter() - t0
                    e = pe + ke
                    dev = np.abs((e - e0) / e0)
                    slope = float(np.polyfit(np.arange(1, steps + 1), (e - e0) / abs(e0), 1)[0])
                    runs[name].append({"max_drift": float(dev.max()), "drift_per_step": slope,
                                       "pressure": float(np.mean((2.0 * ke + w) / (3.0 * vol))), "g": rdf.values(),
                                       "atom_steps_per_s": r.n * steps / dt, "rebuilds": rl.rebuild_count})
            out = {"density": rho, "temperature": temp, "n_atoms": n_atoms, "steps": steps, "replicas": replicas,
                   "force_error_vs_fp64": errors}

            def mean_se(x):
                x = np.asarray(x, dtype=np.float64)
                return float(x.mean()), (float(x.std(ddof=1) / np.sqrt(len(x))) if len(x) > 1 else None)

            g_ref = np.array([r["g"] for r in runs["fp64"]])
            for name in names:
                rr = runs[name]
                row = {}
                for key in ("max_drift", "drift_per_step", "pressure", "atom_steps_per_s", "rebuilds"):
                    row[key], row[key + "_err"] = mean_se([r[key] for r in rr])
                g = np.array([r["g"] for r in rr])
                row["max_dg_vs_fp64"] = float(np.abs(g.mean(axis=0) - g_ref.mean(axis=0)).max())
                if replicas > 1 and name != "fp64":
                    dp = [a["pressure"] - b["pressure"] for a, b in zip(rr, runs["fp64"])]
                    m, se = mean_se(dp)
                    row["dp_vs_fp64"], row["dp_vs_fp64_err"] = m, se
                    row["z_pressure_vs_fp64"] = m / se if se else None
                    dg = g - g_ref
                    se_g = dg.std(axis=0, ddof=1) / np.sqrt(replicas)
                    mask = se_g > 0
                    row["max_abs_z_g_vs_fp64"] = (float(np.abs(dg.mean(axis=0)[mask] / se_g[mask]).max())
                                                  if mask.any() else None)
                    dd = [a["max_drift"] - b["max_drift"] for a, b in zip(rr, runs["fp64"])]
                    row["d_drift_vs_fp64"], row["d_drift_vs_fp64_err"] = mean_se(dd)
                out[name] = row
            yield out


def main():
    a = args_parse()
    if a.impl == "reference":
        run_reference_arm(a)
    elif a.nist:
        import mdgpu as md
        import nist

        t0 = time.perf_counter()
        rows, b = nist.run(md, precision=PRECISIONS[a.nist_precision][0])
        wall = time.perf_counter() - t0
        info = b.info()
        for row in rows:
            row.update({"precision": a.nist_precision, "replicas": nist.REPLICAS, "equil_steps": nist.EQUIL_STEPS,
                        "prod_steps": nist.PROD_STEPS, "batch_atoms": info["atoms"], "wall_s": wall})
            print(json.dumps(row), flush=True)
    elif a.sweep == "precision":
        for line in precision_sweep(steps=a.steps, replicas=a.sweep_replicas):
            print(json.dumps(line), flush=True)
    else:
        run_gpu_arm(a)


if __name__ == "__main__":
    main()
