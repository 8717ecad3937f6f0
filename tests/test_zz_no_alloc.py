"""md_kinetic_energy_noalloc: the kinetic energy for callers that may not allocate device memory (a host
runtime that owns every device buffer, or one that must not call cudaMalloc/cudaFree while it runs). The
caller passes its own device buffers; the library keeps its block partial sums in a fixed device array.

Checked through the C-ABI against md_kinetic_energy on the same velocities and masses, on two calls in a
row (the second smaller, so partials left by the first call would show), on the legacy default stream
(stream = NULL) and for n = 0; that after one warm-up call further calls change neither the device's free
memory (cudaMemGetInfo) nor torch's allocator; and the size limit. This file is named to run last so a
failure here cannot hide the rest of the suite.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_PARTICLES = 16384 * 1024


def _entry(md):
    f = md.LIB.md_kinetic_energy_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    return f


def test_noalloc_kinetic_energy_matches_md_kinetic_energy(md):
    import torch

    f = _entry(md)
    rng = np.random.default_rng(11)
    stream = torch.cuda.current_stream()
    for n in (300_000, 5_000):
        vel = rng.normal(0.0, 1.0, size=(3, n))
        mass = rng.uniform(0.5, 2.0, size=n)
        pos = np.zeros((n, 4))
        s = md.System.from_arrays(pos, 10.0, vel=vel, mass=mass)
        want = s.kinetic_energy()
        d_vel = torch.from_numpy(np.ascontiguousarray(vel)).cuda()
        d_mass = torch.from_numpy(mass).cuda()
        out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        rc = f(d_vel.data_ptr(), d_mass.data_ptr(), n, out.data_ptr(), stream.cuda_stream)
        assert rc == 0, md.LIB.md_last_error().decode()
        torch.cuda.synchronize()
        # the same blocked summation order as md_kinetic_energy: bit-identical doubles
        assert out.item() == want, (n, out.item(), want)


def test_noalloc_kinetic_energy_rejects_oversize(md):
    import torch

    f = _entry(md)
    buf = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = f(buf.data_ptr(), buf.data_ptr(), MAX_PARTICLES + 1, buf.data_ptr(), None)
    assert rc == 1  # MD_ERR_INVALID
    assert "exceeds the maximum" in md.LIB.md_last_error().decode()


def test_noalloc_kinetic_energy_null_stream_and_empty(md):
    import torch

    f = _entry(md)
    rng = np.random.default_rng(12)
    n = 70_001
    vel = rng.normal(0.0, 1.0, size=(3, n))
    mass = rng.uniform(0.5, 2.0, size=n)
    want = md.System.from_arrays(np.zeros((n, 4)), 10.0, vel=vel, mass=mass).kinetic_energy()
    d_vel = torch.from_numpy(np.ascontiguousarray(vel)).cuda()
    d_mass = torch.from_numpy(mass).cuda()
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert f(d_vel.data_ptr(), d_mass.data_ptr(), n, out.data_ptr(), None) == 0, md.LIB.md_last_error().decode()
    torch.cuda.synchronize()
    assert out.item() == want
    # n = 0: no particles, a kinetic energy of exactly zero (the pointers may be NULL)
    assert f(None, None, 0, out.data_ptr(), None) == 0, md.LIB.md_last_error().decode()
    torch.cuda.synchronize()
    assert out.item() == 0.0


def test_noalloc_kinetic_energy_allocates_nothing_after_warmup(md):
    import torch

    f = _entry(md)
    rng = np.random.default_rng(13)
    n = 1_000_003
    d_vel = torch.from_numpy(rng.normal(0.0, 1.0, size=(3, n))).cuda()
    d_mass = torch.from_numpy(rng.uniform(0.5, 2.0, size=n)).cuda()
    outs = torch.zeros(8, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    # one warm-up call: it may load the library's device code and look the scratch array up
    assert f(d_vel.data_ptr(), d_mass.data_ptr(), n, outs.data_ptr(), stream.cuda_stream) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    stats0 = torch.cuda.memory_stats()
    for k in range(8):
        assert f(d_vel.data_ptr(), d_mass.data_ptr(), n - 1000 * k, outs[k:].data_ptr(), stream.cuda_stream) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    stats1 = torch.cuda.memory_stats()
    assert free1 == free0, (free0, free1)
    for key in ("allocation.all.allocated", "segment.all.allocated", "reserved_bytes.all.current"):
        assert stats1.get(key, 0) == stats0.get(key, 0), key
