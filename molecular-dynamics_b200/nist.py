"""NIST Lennard-Jones validation through the batched replica engine (md_batch_*): the reference's physics check,
bench/validate.py of nhantran1711/molecular-dynamics, with all replicas of all state points in one batch.

The reference runs md_sim once per replica: N = 500 (FCC 5^3 x 4), r_c = 3 sigma, dt = 0.005, skin 0.2 (md_sim's
default), a lattice melted at T = 2 for the first third of 10,000 equilibration steps (velocities rescaled every
10 steps, src/main.cpp:219-227), then cooled to T, then 20,000 production steps under the Bussi thermostat
(tau = 0.5, src/main.cpp:242, 275-277), each replica with its own seed (bench/validate.py:96-111). Energies are
reported with NIST's conventions: the truncated, unshifted energy plus the standard tail corrections
(bench/validate.py:65-75, 114-120). The error bar of a state point is the standard error of its replica means
(bench/validate.py:123-134), and each comparison with the NIST tables is a z-score (bench/validate.py:137-150).

The tables are NIST's published values for this system as the reference's validate.py lists them
(bench/validate.py:41-62; NIST Standard Reference Simulation Website, LJ_PURE md.htm and mc.htm).
"""
from __future__ import annotations

import math
import statistics

import numpy as np

CUTOFF = 3.0
SKIN = 0.2
DT = 0.005
CELLS = 5                  # N = 4 * 5^3 = 500
EQUIL_STEPS = 10000
PROD_STEPS = 20000
REPLICAS = 8
RESCALE_EVERY = 10
MELT_TEMPERATURE = 2.0
BUSSI_TAU = 0.5

# NIST NVE MD: (T measured, rho, U per particle, sigma U, P, sigma P) — bench/validate.py:41-48
NIST_MD = [
    (0.851, 0.776, -5.517, 0.001, 0.030, 0.006),
    (0.853, 0.780, -5.533, 0.001, 0.072, 0.005),
    (0.852, 0.820, -5.803, 0.001, 0.573, 0.005),
    (0.851, 0.840, -5.909, 0.001, 0.910, 0.006),
    (0.849, 0.860, -6.027, 0.001, 1.282, 0.005),
    (0.851, 0.900, -6.234, 0.001, 2.544, 0.006),
]

# NIST NVT Monte Carlo at liquid densities: (T, rho, U, sigma U, P, sigma P) — bench/validate.py:50-62
NIST_MC = [
    (0.85, 0.776, -5.5121, 4.55e-4, 6.7714e-3, 1.77e-3),
    (0.85, 0.780, -5.5386, 7.26e-4, 4.7924e-2, 3.18e-3),
    (0.85, 0.820, -5.7947, 6.03e-4, 5.5355e-1, 4.13e-3),
    (0.85, 0.860, -6.0305, 2.38e-3, 1.2660, 1.36e-2),
    (0.85, 0.900, -6.2391, 5.27e-3, 2.2314, 2.72e-2),
    (0.90, 0.776, -5.4689, 4.20e-4, 2.4056e-1, 2.74e-3),
    (0.90, 0.780, -5.4956, 7.86e-4, 2.7851e-1, 2.97e-3),
    (0.90, 0.820, -5.7456, 7.51e-4, 8.2386e-1, 2.85e-3),
    (0.90, 0.860, -5.9753, 5.53e-4, 1.5781, 3.29e-3),
    (0.90, 0.900, -6.1773, 1.57e-3, 2.5848, 9.54e-3),
]


def state_points() -> list[tuple[float, float]]:
    """Every (T, rho) of both tables, sorted (bench/validate.py:206): 16 state points"""
    return sorted({(t, rho) for t, rho, *_ in NIST_MD + NIST_MC})


def shift_energy(rc: float) -> float:
    """4 (rc^-12 - rc^-6): the energy shift of the truncated-shifted potential at sigma = eps = 1"""
    return 4.0 * (rc ** -12 - rc ** -6)


def tail_energy(rho: float, rc: float) -> float:
    """Long-range correction to U per particle for g(r) = 1 beyond the cutoff: (8/3) pi rho (rc^-9 / 3 - rc^-3)"""
    return 8.0 / 3.0 * math.pi * rho * (rc ** -9 / 3.0 - rc ** -3)


def tail_pressure(rho: float, rc: float) -> float:
    """Long-range correction to the pressure: (16/3) pi rho^2 ((2/3) rc^-9 - rc^-3)"""
    return 16.0 / 3.0 * math.pi * rho ** 2 * (2.0 / 3.0 * rc ** -9 - rc ** -3)


def block_error(series, block_len: int) -> float:
    """Standard error of the mean from non-overlapping blocks of block_len samples (bench/validate.py:78-85)"""
    blocks = len(series) // block_len
    means = [sum(series[b * block_len:(b + 1) * block_len]) / block_len for b in range(blocks)]
    mean = sum(means) / blocks
    var = sum((m - mean) ** 2 for m in means) / (blocks - 1)
    return math.sqrt(var / blocks)


def replica_series(pe_per_particle, inside_pairs, pressure, n: int, rho: float, rc: float = CUTOFF):
    """U per particle and P per step with NIST's conventions: the shifted energy made unshifted again (each pair
    inside the cutoff gets its shift back) plus the tail corrections (bench/validate.py:114-120)"""
    shift = shift_energy(rc)
    u = [pe_per_particle[k] + inside_pairs[k] * shift / n + tail_energy(rho, rc) for k in range(len(pe_per_particle))]
    p = [pressure[k] + tail_pressure(rho, rc) for k in range(len(pressure))]
    return u, p


def analyse(u_series: list, p_series: list) -> dict:
    """Mean over replicas of the replicas' time averages, with the standard error from their spread
    (bench/validate.py:123-134)"""
    u_means = [sum(u) / len(u) for u in u_series]
    p_means = [sum(p) / len(p) for p in p_series]
    k = len(u_means)
    return {"u": statistics.mean(u_means), "u_err": statistics.stdev(u_means) / math.sqrt(k),
            "p": statistics.mean(p_means), "p_err": statistics.stdev(p_means) / math.sqrt(k)}


def z_scores(result: dict, reference: tuple) -> tuple[float, float]:
    """(U, P) z-scores against one NIST row: the difference over both error bars in quadrature
    (bench/validate.py:142-143)"""
    _, _, u_ref, u_ref_err, p_ref, p_ref_err = reference
    zu = (result["u"] - u_ref) / math.hypot(result["u_err"], u_ref_err)
    zp = (result["p"] - p_ref) / math.hypot(result["p_err"], p_ref_err)
    return zu, zp


def run(md, states=None, replicas: int = REPLICAS, equil: int = EQUIL_STEPS, prod: int = PROD_STEPS,
        precision: int | None = None, device: int = 0, chunk_steps: int = 100):
    """Every replica of every state point in one md_batch: the lattice melted at T = 2 for the first third of the
    equilibration (rescaled every 10 steps), then rescaled to each state point's T, then NVT production under the
    Bussi thermostat, recording the potential energy, virial, kinetic energy and inside-cutoff pairs of every
    production step. Replica r of the s-th state point (1-based, in state_points() order) has seed
    1000 s + r + 1 for its velocities and its thermostat (bench/validate.py:104). Returns one dict per state
    point: T, rho, the analysis (U, P and their errors) and the per-replica means."""
    states = state_points() if states is None else states
    precision = md.PREC_FP64 if precision is None else precision
    all_points = state_points()
    systems, temps, seeds, meta = [], [], [], []
    for t, rho in states:
        s_index = all_points.index((t, rho)) + 1
        for r in range(replicas):
            seed = 1000 * s_index + r + 1
            s = md.fcc_system(CELLS, rho, t, seed=seed, device=device)
            d = s.download()
            systems.append((d["pos"], s.box, d["vel"], None))
            temps.append(t)
            seeds.append(seed)
            meta.append((t, rho, s.n, s.box))
            del s
    melt = equil // 3 // RESCALE_EVERY * RESCALE_EVERY  # rescales at steps <= equil / 3 use T = 2
    b = md.Batch(systems, cutoff=CUTOFF, skin=SKIN, dt=DT, precision=precision, thermostat="rescale",
                 temperatures=np.full(len(systems), MELT_TEMPERATURE), rescale_every=RESCALE_EVERY, energy_every=1,
                 chunk_steps=chunk_steps, device=device)
    if melt:
        b.run(melt, record=False)
    b.set_thermostat("rescale", temperatures=temps, rescale_every=RESCALE_EVERY)
    if equil - melt:
        b.run(equil - melt, record=False)
    b.set_thermostat("bussi", temperatures=temps, bussi_tau=BUSSI_TAU, seeds=seeds)
    pe, w, ke, inside = b.run(prod, inside=True)
    out = []
    for si, (t, rho) in enumerate(states):
        us, ps = [], []
        for r in range(replicas):
            k = si * replicas + r
            _, _, n, box = meta[k]
            vol = box ** 3
            pressure = (2.0 * ke[:, k] + w[:, k]) / (3.0 * vol)  # src/main.cpp:210-211
            u, p = replica_series(pe[:, k] / n, inside[:, k], pressure, n, rho)
            us.append(u)
            ps.append(p)
        a = analyse(us, ps)
        row = {"T": t, "rho": rho, **a, "replica_u": [float(np.mean(u)) for u in us],
               "replica_p": [float(np.mean(p)) for p in ps]}
        # each state point is one row of one table (the state points are the tables' own (T, rho) pairs)
        for label, table in (("md", NIST_MD), ("mc", NIST_MC)):
            ref = [r for r in table if r[0] == t and r[1] == rho]
            if ref:
                row[f"nist_{label}"] = ref[0]
                row[f"z_u_{label}"], row[f"z_p_{label}"] = z_scores(a, ref[0])
        out.append(row)
    return out, b
