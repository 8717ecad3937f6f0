"""The FP64 CPU adjoint (oracle/md_adjoint.cpp), the checker of the GPU adjoint, against central finite
differences of its own trajectory and against the reference's own trajectory (oracle/_ref, when built).

The truncated potential's force jumps by |F(r_c)| at the cutoff, so a finite-difference stencil that moves a
pair across r_c at some step adds a jump the derivative does not have. The derivative is therefore checked at
the steps h where the stencil straddles no crossing: the smallest relative error over h in H must be tiny, and
the errors at h = 1e-4 (the usual choice) are reported beside it."""
from __future__ import annotations

import os

import numpy as np
import pytest

from oracle.oracle import REF_SO, OAdjoint

H = (1e-4, 1e-5, 1e-6, 1e-7)
CASES = [(4, 0.8442, 1.0, 50, 20), (6, 0.8442, 1.0, 60, 25)]  # all-pairs candidates, then cells


def central(f, x, d, h):
    return (f(x + h * d) - f(x - h * d)) / (2 * h)


@pytest.mark.parametrize("cells,density,temperature,steps,every", CASES)
@pytest.mark.parametrize("g_pe,g_p", [(1.0, 0.0), (0.0, 1.0), (0.7, -2.0)])
def test_cpu_adjoint_against_central_differences(oracle, cells, density, temperature, steps, every, g_pe, g_p):
    s = oracle.fcc_system(cells, density, temperature, 42)
    st = s.state()
    pos, vel, box = st.pos, st.vel, st.box

    def J(eps=1.0, sig=1.0, p=pos, v=vel):
        mu, mp, *_ = OAdjoint(oracle, p, box, v, eps=eps, sigma=sig, steps=steps, every=every).forward()
        return g_pe * mu + g_p * mp

    a = OAdjoint(oracle, pos, box, vel, steps=steps, every=every)
    a.forward()
    g = a.backward(g_pe, g_p)
    rng = np.random.default_rng(cells)
    dp = np.zeros_like(pos)
    dp[:, :3] = rng.standard_normal((len(pos), 3))
    dp /= np.linalg.norm(dp)
    dv = rng.standard_normal(vel.shape)
    dv /= np.linalg.norm(dv)
    checks = {
        "epsilon": (g["d_epsilon"], lambda h: central(lambda e: J(eps=e), 1.0, 1.0, h)),
        "sigma": (g["d_sigma"], lambda h: central(lambda x: J(sig=x), 1.0, 1.0, h)),
        "positions": (float((g["d_pos"].T * dp[:, :3]).sum()), lambda h: central(lambda p: J(p=p), pos, dp, h)),
        "velocities": (float((g["d_vel"] * dv).sum()), lambda h: central(lambda v: J(v=v), vel, dv, h)),
    }
    for name, (adj, fd) in checks.items():
        errs = [abs(fd(h) - adj) / abs(adj) for h in H]
        # below ~1e-6 the difference quotient of J (|J| up to ~1e4) is limited by its own rounding
        assert min(errs) < 1e-6, (name, adj, errs)


def test_adjoint_trajectory_is_the_reference_trajectory(oracle):
    """mean U and mean P of the adjoint's forward pass equal those of the reference's own integrator
    (src/Integrator.cpp:18-30, deterministic forces) to rounding: the particles are not reordered and the
    sums run in another order, nothing else differs."""
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref is not built (make -C oracle ref)")
    from oracle.oracle import Reference, RForceField, RNeighbourList

    r = Reference()
    for cells, steps in ((4, 50), (6, 80)):
        rs = r.fcc_system(cells, 0.8442, 1.0, 42)
        nl = RNeighbourList(r, 2.5, 0.3, True)
        ff = RForceField(r, 1.0, 1.0, 2.5, deterministic=True)
        nl.build(rs)
        ff.forces(rs, nl)
        pe, w, ke = ff.observables(rs, nl, 0.005, steps)
        s = oracle.fcc_system(cells, 0.8442, 1.0, 42)
        st = s.state()
        mu, mp, u, ww, k = OAdjoint(oracle, st.pos, st.box, st.vel, steps=steps, every=20).forward()
        assert np.allclose(u, pe, rtol=1e-12, atol=0) and np.allclose(ww, w, rtol=1e-10, atol=1e-10)
        assert np.allclose(k, ke, rtol=1e-12, atol=0)
        assert abs(mu - pe.mean()) <= 1e-12 * abs(mu)
        V = st.box ** 3
        assert abs(mp - ((2 * ke + w) / (3 * V)).mean()) <= 1e-10 * abs(mp)
