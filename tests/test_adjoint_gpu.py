"""The flux-objective adjoint (fg_flux_gradient) against central finite differences of an FP64
forward (the oracle's f64 run), on a small version of the adjoint workload; checkpointed and
stored-history sweeps agree bit for bit; the torch.autograd wrapper hands back the same gradient."""
import numpy as np
import pytest

from fieldgrid_b200 import fdtd
from fieldgrid_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

H = 1e-4           # central-difference step, as for the full-size check
FD_TOL = 1e-3      # |adjoint - FD| / |FD| per parameter


def dual(line):
    """Node spacings dd of one axis (sim.rs:29-57)."""
    d = np.diff(line)
    dd = np.empty(len(line))
    dd[0], dd[-1] = d[0], d[-1]
    dd[1:-1] = 0.5 * (line[2:] - line[:-2])
    return dd


def flux_f64(sc, spec):
    """J of the scene from the oracle's FP64 run, with the objective's definition."""
    rec = O.run_cpu(O.OracleSim(*sc.args(), bits=64), 0, sc.pulse, sc.extras)
    n = sc.grid.dims()
    pml = sc.grid.pml
    p = rec.plane.reshape(n[0], n[1], 10)
    z = p[..., 0::2] + 1j * p[..., 1::2]           # Ex, Ey, Ez, Hx, Hy
    da = np.outer(dual(sc.grid.x), dual(sc.grid.y))
    w = (slice(pml, n[0] - pml), slice(pml, n[1] - pml))
    F = np.sum(da[w] * (z[w][..., 0] * np.conj(z[w][..., 4]) - z[w][..., 1] * np.conj(z[w][..., 3])))
    return abs(F) ** 2


@pytest.fixture(scope="module")
def small():
    scene, spec, eps0, sig0 = W.flux_design(24, 24, 24, pml=4, design=(4, 4, 3), steps=400, checkpoints=0)
    return scene, spec, eps0, sig0


def test_the_objective_matches_the_fp64_forward(gpu, small):
    scene, spec, eps0, sig0 = small
    sc = scene()
    r = fdtd.flux_gradient(gpu, fdtd.Sim.try_new(*sc.args()), 0, sc.pulse, spec, grad=False)
    ref = flux_f64(sc, spec)
    assert ref > 0
    assert abs(r.objective - ref) <= 1e-4 * ref, (r.objective, ref)


def test_the_adjoint_gradient_matches_central_differences(gpu, small):
    scene, spec, eps0, sig0 = small
    sc = scene()
    r = fdtd.flux_gradient(gpu, fdtd.Sim.try_new(*sc.args()), 0, sc.pulse, spec)
    assert r.grad_eps.shape == spec.shape() and r.design_edges > 0
    rng = W.SplitMix64(5)
    scale = max(np.abs(r.grad_eps).max(), 1e-300)
    for q in range(6):
        at = tuple(rng.integer(0, s - 1) for s in spec.shape())
        which = "eps" if q % 2 == 0 else "sig"
        base = eps0 if which == "eps" else sig0
        up, dn = base.copy(), base.copy()
        up[at] = np.float32(base[at] + H)
        dn[at] = np.float32(base[at] - H)
        h_eff = 0.5 * (float(up[at]) - float(dn[at]))    # the step the f32 materials carry
        args = (up, sig0) if which == "eps" else (eps0, up)
        jp = flux_f64(scene(*args), spec)
        args = (dn, sig0) if which == "eps" else (eps0, dn)
        jm = flux_f64(scene(*args), spec)
        fd = (jp - jm) / (2 * h_eff)
        adj = (r.grad_eps if which == "eps" else r.grad_sigma)[at]
        print(which, at, adj, fd)
        floor = 1e-6 * scale if which == "eps" else 0.0
        assert abs(adj - fd) <= FD_TOL * max(abs(fd), floor), (which, at, adj, fd)


def fp64(spec):
    return fdtd.FluxSpec(spec.design_lo, spec.design_hi, spec.plane_k, spec.freq, spec.steps, precision=64)


def test_the_fp64_device_forward_matches_the_fp64_oracle(gpu, small):
    """The device's FP64 forward (the full-size FD reference) against the oracle's f64 run; they
    differ only where setup overrode an edge (the port), kept at its f32 value on the device."""
    scene, spec, eps0, sig0 = small
    sc = scene()
    r = fdtd.flux_gradient(gpu, fdtd.Sim.try_new(*sc.args()), 0, sc.pulse, fp64(spec), grad=False)
    ref = flux_f64(sc, spec)
    assert abs(r.objective - ref) <= 1e-5 * ref, (r.objective, ref)


def test_the_adjoint_matches_differences_of_the_device_fp64_forward(gpu, small):
    scene, spec, eps0, sig0 = small
    sc = scene()
    r = fdtd.flux_gradient(gpu, fdtd.Sim.try_new(*sc.args()), 0, sc.pulse, spec)
    rng = W.SplitMix64(7)
    for q in range(4):
        at = tuple(rng.integer(0, s - 1) for s in spec.shape())
        which = "eps" if q % 2 == 0 else "sig"
        base = eps0 if which == "eps" else sig0
        up, dn = base.copy(), base.copy()
        up[at] = np.float32(base[at] + H)
        dn[at] = np.float32(base[at] - H)
        h_eff = 0.5 * (float(up[at]) - float(dn[at]))
        j = []
        for arr in (up, dn):
            s2 = scene(*((arr, sig0) if which == "eps" else (eps0, arr)))
            j.append(fdtd.flux_gradient(gpu, fdtd.Sim.try_new(*s2.args()), 0, s2.pulse, fp64(spec), grad=False).objective)
        fd = (j[0] - j[1]) / (2 * h_eff)
        adj = (r.grad_eps if which == "eps" else r.grad_sigma)[at]
        assert abs(adj - fd) <= FD_TOL * abs(fd), (which, at, adj, fd)


@pytest.fixture(scope="module")
def small_debye():
    return W.flux_design(24, 24, 24, pml=4, design=(4, 4, 3), steps=400, checkpoints=0, debye=True)


def test_the_adjoint_through_debye_media_matches_central_differences(gpu, small_debye):
    """The Debye ADE transposed in the sweep: a one-pole slab beside the design block."""
    scene, spec, eps0, sig0 = small_debye
    sc = scene()
    sim = fdtd.Sim.try_new(*sc.args())
    r = fdtd.flux_gradient(gpu, sim, 0, sc.pulse, spec)
    rng = W.SplitMix64(9)
    for q in range(4):
        at = tuple(rng.integer(0, s - 1) for s in spec.shape())
        which = "eps" if q % 2 == 0 else "sig"
        base = eps0 if which == "eps" else sig0
        up, dn = base.copy(), base.copy()
        up[at] = np.float32(base[at] + H)
        dn[at] = np.float32(base[at] - H)
        h_eff = 0.5 * (float(up[at]) - float(dn[at]))
        jp = flux_f64(scene(*((up, sig0) if which == "eps" else (eps0, up))), spec)
        jm = flux_f64(scene(*((dn, sig0) if which == "eps" else (eps0, dn))), spec)
        fd = (jp - jm) / (2 * h_eff)
        adj = (r.grad_eps if which == "eps" else r.grad_sigma)[at]
        assert abs(adj - fd) <= FD_TOL * abs(fd), (which, at, adj, fd)
    # checkpoints restore the Debye state: the same gradient bit for bit
    spec4 = fdtd.FluxSpec(spec.design_lo, spec.design_hi, spec.plane_k, spec.freq, spec.steps, checkpoints=5)
    b = fdtd.flux_gradient(gpu, sim, 0, sc.pulse, spec4)
    assert np.array_equal(r.grad_eps, b.grad_eps) and np.array_equal(r.grad_sigma, b.grad_sigma)


def test_cone_reruns_reproduce_the_tma_march_history(gpu):
    """On a grid the forward marches with the TMA kernel (k-layer tiles, CPML shell), re-runs that
    march only the dependency cone with the direct-load kernel record the same history: the
    checkpointed gradient equals the stored-history one bit for bit, with Debye media present."""
    scene, spec, _, _ = W.flux_design(64, 60, 72, pml=8, design=(8, 6, 4), steps=160, checkpoints=0, debye=True)
    sc = scene()
    sim = fdtd.Sim.try_new(*sc.args())
    s = fdtd.Session(gpu, sim, 0, sc.pulse, sc.extras)
    assert "TMA" in s.variant
    s.close()
    a = fdtd.flux_gradient(gpu, sim, 0, sc.pulse, spec)
    ck = fdtd.FluxSpec(spec.design_lo, spec.design_hi, spec.plane_k, spec.freq, spec.steps, checkpoints=6)
    b = fdtd.flux_gradient(gpu, sim, 0, sc.pulse, ck)
    assert b.segments > 2 and np.abs(a.grad_eps).max() > 0
    assert np.array_equal(a.grad_eps, b.grad_eps)
    assert np.array_equal(a.grad_sigma, b.grad_sigma)


def test_checkpointed_sweep_equals_stored_history(gpu, small):
    scene, spec, eps0, sig0 = small
    sc = scene()
    sim = fdtd.Sim.try_new(*sc.args())
    a = fdtd.flux_gradient(gpu, sim, 0, sc.pulse, spec)
    spec4 = fdtd.FluxSpec(spec.design_lo, spec.design_hi, spec.plane_k, spec.freq, spec.steps, checkpoints=5)
    b = fdtd.flux_gradient(gpu, sim, 0, sc.pulse, spec4)
    assert b.segments > 1 and b.segment_len % 2 == 0
    assert a.objective == b.objective
    assert np.array_equal(a.grad_eps, b.grad_eps)
    assert np.array_equal(a.grad_sigma, b.grad_sigma)


@pytest.mark.parametrize("dims,debye", [((24, 24, 24), False), ((40, 44, 70), False), ((70, 37, 33), False),
                                        ((40, 44, 70), True)])
def test_the_fused_adjoint_step_equals_the_separate_transposes(gpu, dims, debye):
    """One fused launch per adjoint step against the E and H transposes as two launches, on grids
    whose (j, k) extents leave partial (30, 14) tiles and whose x extent spans several segments."""
    scene, spec, _, _ = W.flux_design(*dims, pml=4, design=(4, 4, 3), steps=120, checkpoints=3, debye=debye)
    sc = scene()
    sim = fdtd.Sim.try_new(*sc.args())
    a = fdtd.flux_gradient(gpu, sim, 0, sc.pulse, spec)
    sep = fdtd.FluxSpec(spec.design_lo, spec.design_hi, spec.plane_k, spec.freq, spec.steps,
                        checkpoints=spec.checkpoints, transposes=1)
    b = fdtd.flux_gradient(gpu, sim, 0, sc.pulse, sep)
    assert np.abs(a.grad_eps).max() > 0
    assert np.array_equal(a.grad_eps, b.grad_eps)
    assert np.array_equal(a.grad_sigma, b.grad_sigma)


def test_the_autograd_function_returns_the_adjoint_gradient(gpu, small):
    import torch
    from fieldgrid_b200.autograd import FluxObjective
    scene, spec, eps0, sig0 = small
    eps = torch.tensor(eps0, dtype=torch.float64, requires_grad=True)
    sig = torch.tensor(sig0, dtype=torch.float64, requires_grad=True)
    J = FluxObjective.apply(eps, sig, gpu, scene, spec, 0)
    (2.0 * J).backward()
    sc = scene()
    r = fdtd.flux_gradient(gpu, fdtd.Sim.try_new(*sc.args()), 0, sc.pulse, spec)
    assert float(J.detach()) == r.objective
    assert np.allclose(eps.grad.numpy(), 2.0 * r.grad_eps, rtol=0, atol=0)
    assert np.allclose(sig.grad.numpy(), 2.0 * r.grad_sigma, rtol=0, atol=0)


def test_unsupported_media_are_refused(gpu):
    sc = W.everything(steps=20, fused=True)   # Debye slab, inductor, thin wires, sheets
    spec = fdtd.FluxSpec((8, 8, 8), (10, 10, 10), 12, 10e9, 20)
    with pytest.raises(fdtd.FdtdError, match="no inductor"):
        fdtd.flux_gradient(gpu, fdtd.Sim.try_new(*sc.args()), 0, sc.pulse, spec)
    scene, spec, _, _ = W.flux_design(24, 24, 24, pml=4, design=(4, 4, 3), steps=20)
    edge = fdtd.FluxSpec((0, 10, 10), (4, 14, 13), spec.plane_k, spec.freq, 20)
    sc = scene()
    with pytest.raises(fdtd.FdtdError, match="grid boundary"):
        fdtd.flux_gradient(gpu, fdtd.Sim.try_new(*sc.args()), 0, sc.pulse, edge)


def test_a_batch_of_flux_gradients_equals_running_each_alone(gpu):
    """fg_flux_gradient_batch: uneven grids with Debye spheres, in groups of 3 (two groups); every
    run's objective and gradients equal flux_gradient of that run alone, bit for bit."""
    jobs = W.batch_flux(count=5, lo=32, hi=48, pml=4, steps=120, checkpoints=4, design=8)
    scenes = [j[0]() for j in jobs]
    sims = [fdtd.Sim.try_new(*sc.args()) for sc in scenes]
    specs = [j[1] for j in jobs]
    got = fdtd.flux_gradient_batch(gpu, sims, [sc.pulse for sc in scenes], specs, group=3)
    assert len(got) == 5
    for sc, sim, spec, r in zip(scenes, sims, specs, got):
        a = fdtd.flux_gradient(gpu, sim, 0, sc.pulse, spec)
        assert r.objective == a.objective and r.objective > 0
        assert np.array_equal(r.grad_eps, a.grad_eps) and np.abs(a.grad_eps).max() > 0
        assert np.array_equal(r.grad_sigma, a.grad_sigma)


def test_a_batch_names_the_run_it_refuses(gpu):
    jobs = W.batch_flux(count=2, lo=32, hi=48, pml=4, steps=20, checkpoints=2, design=8)
    scenes = [j[0]() for j in jobs]
    sims = [fdtd.Sim.try_new(*sc.args()) for sc in scenes]
    bad = fdtd.FluxSpec((0, 10, 10), (4, 14, 13), jobs[1][1].plane_k, 10e9, 20)
    with pytest.raises(fdtd.FdtdError, match="job 1: the design box touches the grid boundary"):
        fdtd.flux_gradient_batch(gpu, sims, [sc.pulse for sc in scenes], [jobs[0][1], bad])
