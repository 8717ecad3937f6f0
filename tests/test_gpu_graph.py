"""md_run as CUDA graphs (every precision on a tiled list): every step of a chunk, the list rebuild decided on the
device in a conditional node, the thermostat and the g(r) sample included. The graph path must give the host
loop's trajectory bit for bit (the host loop is md_system_set_graph(s, 0), and md_step_list one step at a time),
also when a device rebuild outgrows the recorded tile and the chunk reruns on the host path."""
from __future__ import annotations

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PRECS = ["PREC_FP32FX", "PREC_FP32", "PREC_FX64", "PREC_FX32", "PREC_FP64"]


def start(md, cells=12, temperature=1.3, seed=5):
    base = md.fcc_system(cells, 0.8442, temperature, seed=seed)
    return base.download(), base.box


def make(md, st, box, prec):
    s = md.System.from_arrays(st["pos"], box, vel=st["vel"])
    nl = md.NeighbourList(2.5, 0.3)
    ff = md.LennardJonesForceField(1.0, 1.0, 2.5, precision=prec)
    nl.build(s)
    ff.compute_forces(s, nl)
    return s, nl, ff


@pytest.mark.parametrize("prec", PRECS)
def test_graph_run_matches_step_list(md, prec):
    """150 NVE steps (three chunks of 64, 64 and 22) against 150 md_step_list calls."""
    p = getattr(md, prec)
    st, box = start(md)
    integ = md.VelocityVerletIntegrator(0.005)
    s, nl, ff = make(md, st, box, p)
    pe_g, ke_g, w_g = integ.run(s, ff, nl, 150)
    info = s.graph_info()
    assert info["launches"] == 3 and info["recoveries"] == 0, info
    r, rl, rf = make(md, st, box, p)
    pe_h = np.array([integ.step(r, rf, rl) for _ in range(150)])
    assert np.array_equal(pe_g, pe_h)
    assert nl.rebuild_count == rl.rebuild_count and nl.rebuild_count > 5
    a, b = s.download(), r.download()
    for k in ("pos", "vel", "force", "ids"):
        assert np.array_equal(a[k], b[k]), k
    assert s.state_hash() == r.state_hash()


@pytest.mark.parametrize("prec", ["PREC_FP32FX", "PREC_FX32", "PREC_FP64"])
@pytest.mark.parametrize("thermostat", ["rescale", "bussi"])
def test_graph_run_with_thermostat_and_rdf_matches_host_loop(md, prec, thermostat):
    """Rescale (melt schedule, every 7 steps) or Bussi NVT, with a g(r) sample every 5 steps: per-step PE, KE and
    virial, the final state, the rebuilds and the histogram equal the host loop's."""
    p = getattr(md, prec)
    st, box = start(md, temperature=1.0)
    integ = md.VelocityVerletIntegrator(0.005)
    n = 140
    r1, chi2 = md.bussi_noise(11, 4 * 12 ** 3, n)
    kw = dict(thermostat=thermostat, rescale_every=7, rescale_temperature=0.9, melt_until=30, melt_temperature=1.6,
              bussi_temperature=0.9, bussi_tau=0.1, bussi_r1=r1, bussi_chi2=chi2, rdf_every=5, first_step=3)
    out = []
    for chunk in (32, 0):
        s, nl, ff = make(md, st, box, p)
        s.set_graph(chunk)
        rdf = md.RadialDistribution(2.5, 50)
        pe, ke, w = integ.run(s, ff, nl, n, rdf=rdf, **kw)
        out.append((pe, ke, w, s.download(), nl.rebuild_count, rdf.histogram(), s.graph_info()))
    (pa, ka, wa, sa, ra, ha, ia), (pb, kb, wb, sb, rb, hb, ib) = out
    assert ia["launches"] == 5 and ib["launches"] == 0
    assert np.array_equal(pa, pb) and np.array_equal(ka, kb) and np.array_equal(wa, wb)
    assert ra == rb and ra > 3
    assert np.array_equal(ha, hb) and ha.sum() > 0
    for k in ("pos", "vel", "force"):
        assert np.array_equal(sa[k], sb[k]), k


@pytest.mark.parametrize("prec", ["PREC_FP32FX", "PREC_FX32", "PREC_FP64"])
def test_graph_overflow_reruns_chunk_on_host_path(md, prec):
    """With the test flag, every device rebuild reports an overflow (as a row past the capacity or a cell past the
    recorded tile would); each chunk that rebuilds starts again from its snapshot on the host path. The trajectory
    still equals the host loop's."""
    p = getattr(md, prec)
    st, box = start(md, cells=14, temperature=1.5, seed=9)
    integ = md.VelocityVerletIntegrator(0.005)
    out = []
    for chunk, rerun in ((16, True), (0, False)):
        s, nl, ff = make(md, st, box, p)
        s.set_graph(chunk, test_rerun=rerun)
        pe, ke, _ = integ.run(s, ff, nl, 200)
        out.append((pe, ke, s.download(), nl.rebuild_count, s.graph_info()))
    (pa, ka, sa, ra, ia), (pb, kb, sb, rb, ib) = out
    assert ia["recoveries"] > 0 and ia["launches"] >= ia["recoveries"], ia
    assert np.array_equal(pa, pb) and np.array_equal(ka, kb) and ra == rb
    for k in ("pos", "vel", "force", "ids"):
        assert np.array_equal(sa[k], sb[k]), k


def test_graph_run_is_faster_at_small_n(md):
    """N = 2,048 (config 1's box): the graph path against the host loop, per step, FP32FX NVE."""
    import torch

    st, box = start(md, cells=8, temperature=0.71, seed=42)
    integ = md.VelocityVerletIntegrator(0.005)
    us = {}
    for chunk in (64, 0):
        s, nl, ff = make(md, st, box, md.PREC_FP32FX)
        s.set_graph(chunk)
        integ.run(s, ff, nl, 200)
        integ.prepare(s, ff, nl, 2000)
        stream = torch.cuda.ExternalStream(s.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.synchronize()
        e0.record(stream)
        integ.run(s, ff, nl, 2000)
        e1.record(stream)
        e1.synchronize()
        us[chunk] = 1e3 * e0.elapsed_time(e1) / 2000
    print("N=2048 FP32FX us/step: graph", us[64], "host", us[0])
    assert us[64] < 0.8 * us[0], us
