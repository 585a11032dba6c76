"""fg_energy_noalloc: the field energy of caller-owned device arrays, for callers that cannot
allocate device memory at that point (an operator callback that runs while a host framework's
caching allocator owns the device memory, or a loop that must not take the device-wide
synchronisation of cudaMalloc/cudaFree). Its per-block sums sit in a fixed per-device array
instead of an allocation.

The tests fill device arrays themselves (torch owns them) and check, on two calls in a row, that
the entry point returns the energy the session's own check (fg_session_energy) reports for the
same fields and a host f64 sum of the same values; a second case spans many blocks with a ragged
tail, and an empty array gives 0. This file is named to be collected last; it also passes alone
in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from fieldgrid_b200 import _lib, fdtd
from fieldgrid_b200 import workloads as W

pytestmark = pytest.mark.gpu

REL = 1e-10  # both are f64 sums of the same f32 values, in different orders


def _host_energy(e, h):
    e = np.asarray(e, np.float64)
    h = np.asarray(h, np.float64) * 376.73
    return float(np.sum(e * e) + np.sum(h * h))


def _energy_noalloc(e, h):
    import torch
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    L = _lib.lib()
    code = L.fg_energy_noalloc(C.c_void_p(e.data_ptr()), C.c_void_p(h.data_ptr()), e.numel(),
                               C.c_void_p(out.data_ptr()), None)
    assert code == 0, L.fg_last_error().decode()
    torch.cuda.synchronize()
    return float(out.item())


def test_energy_without_allocation_matches_the_session_energy(gpu):
    import torch
    sc = W.spheres(48, pml=6, count=10, rmin=3, rmax=10, steps=200, fused=True)
    sim = fdtd.Sim.try_new(*sc.args())
    s = fdtd.Session(gpu, sim, 0, sc.pulse, sc.extras)
    nn = int(np.prod(sc.grid.dims()))
    results = []
    for steps in (40, 75):  # two calls in a row, on different fields
        s.step(steps - s.steps)
        want = s.energy()
        e_host, h_host = s.read("e", 3 * nn), s.read("h", 3 * nn)
        e = torch.from_numpy(e_host).cuda()
        h = torch.from_numpy(h_host).cuda()
        got = _energy_noalloc(e, h)
        again = _energy_noalloc(e, h)  # the shared array keeps the last call's sums; no effect
        assert want > 0
        assert abs(got - want) <= REL * want, (steps, got, want)
        host = _host_energy(e_host, h_host)
        assert abs(got - host) <= REL * host, (steps, got, host)
        assert again == got
        results.append(got)
    assert results[0] != results[1]
    s.close()


def test_energy_without_allocation_over_many_blocks(gpu):
    import torch
    g = torch.Generator().manual_seed(7)
    n = 3 * (1 << 20) + 12345   # many blocks, the last one partial
    results = []
    for scale in (1.0, 0.25):   # two calls in a row on different values
        e_host = (torch.rand(n, generator=g) * 2 - 1) * scale
        h_host = (torch.rand(n, generator=g) * 2 - 1) * (scale / 376.73)
        got = _energy_noalloc(e_host.cuda(), h_host.cuda())
        want = _host_energy(e_host.numpy(), h_host.numpy())
        assert abs(got - want) <= 1e-9 * want, (n, got, want)
        results.append(got)
    assert results[0] != results[1]
    empty = torch.zeros(0, dtype=torch.float32, device="cuda")
    assert _energy_noalloc(empty, empty) == 0.0


def test_energy_without_allocation_refuses_oversized_input(gpu):
    import torch
    L = _lib.lib()
    e = torch.zeros(4, dtype=torch.float32, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    too_many = 4096 * (1 << 20) + 1
    code = L.fg_energy_noalloc(C.c_void_p(e.data_ptr()), C.c_void_p(e.data_ptr()), too_many,
                               C.c_void_p(out.data_ptr()), None)
    assert code == 1
    assert "exceed the maximum" in L.fg_last_error().decode()
