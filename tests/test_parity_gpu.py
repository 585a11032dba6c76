"""Parity of the CUDA engine with the oracle (the CPU restatement of sims-field's own CPU FDTD),
through the C ABI. Tolerances: the reference's `worst` measure below 1e-5 for its every-feature
scene (tests/fdtd.rs:163-173), relative L2 at most 1e-4 for fields, probe series, plane DFT,
NTFF accumulators and far fields elsewhere (the float parity bar of this port)."""
import math

import numpy as np
import pytest

from conftest import rel_l2, worst
from fieldgrid_b200 import fdtd
from fieldgrid_b200 import workloads as W
from fieldgrid_b200.fdtd import C0
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _with_ntff(scene, sim, inset):
    scene.extras.ntff = fdtd.patches(sim, inset).gpu
    return scene


@pytest.fixture(scope="module")
def every():
    sc = W.everything(steps=1500)
    sim = fdtd.Sim.try_new(*sc.args())
    _with_ntff(sc, sim, 2)
    osim = O.OracleSim(*sc.args(), bits=32)
    return sc, sim, osim


def _agree(a, b, limit, what):
    assert a.steps == b.steps, what
    for name in ("series", "plane", "ntff"):
        x, y = getattr(a, name), getattr(b, name)
        w = worst(x, y)
        print(f"{what} {name}: {w:.2e}")
        assert w < limit, (what, name, w)


def test_every_feature_steps_the_same_on_the_cpu_and_the_gpu(gpu, every):
    """tests/fdtd.rs:147-174: CPU vs separate GPU, separate vs fused, and the second port."""
    sc, sim, osim = every
    cpu = O.run_cpu(osim, 0, sc.pulse, sc.extras)
    assert np.all(np.isfinite(cpu.series))
    sc.extras.fused_e = False
    apart = fdtd.run(gpu, sim, 0, sc.pulse, sc.extras)
    _agree(cpu, apart, 1e-5, "cpu against gpu")
    sc.extras.fused_e = True
    fused = fdtd.run(gpu, sim, 0, sc.pulse, sc.extras)
    _agree(apart, fused, 1e-5, "separate against fused")
    sc.extras.fused_e = False
    other = fdtd.run(gpu, sim, 1, sc.pulse, sc.extras)
    cpu_other = O.run_cpu(osim, 1, sc.pulse, sc.extras)
    _agree(cpu_other, other, 1e-5, "second port")
    sc.extras.fused_e = True
    other_fused = fdtd.run(gpu, sim, 1, sc.pulse, sc.extras)
    _agree(cpu_other, other_fused, 1e-5, "second port fused")


@pytest.fixture(scope="module")
def box():
    sc = W.dielectric_box(64)
    o32 = O.run_cpu(O.OracleSim(*sc.args(), bits=32), 0, sc.pulse, sc.extras, keep_fields=True)
    o64 = O.run_cpu(O.OracleSim(*sc.args(), bits=64), 0, sc.pulse, sc.extras, keep_fields=True)
    return sc, o32, o64


@pytest.mark.parametrize("fused", [True, False])
def test_plain_fdtd_64_cubed_matches_after_1000_steps(gpu, box, fused):
    """64^3 cells, dielectric box, soft Ez source, 4 probes, 1000 steps: final E/H and the probe
    series within 1e-4 relative L2 of the oracle; both stated against the FP64 run."""
    sc, o32, o64 = box
    sc.extras.fused_e = fused
    sim = fdtd.Sim.try_new(*sc.args())
    rec = fdtd.run(gpu, sim, 0, sc.pulse, sc.extras, keep_fields=True)
    assert rec.steps == 1000
    for name in ("e", "h", "series"):
        g, c32, c64 = getattr(rec, name), getattr(o32, name), getattr(o64, name)
        e_gpu, e_cpu, e_64 = rel_l2(g, c32), rel_l2(g, c64), rel_l2(c32, c64)
        print(f"{name}: gpu vs oracle f32 {e_gpu:.2e}, gpu vs f64 {e_cpu:.2e}, oracle f32 vs f64 {e_64:.2e}")
        assert e_gpu <= TOL, (name, e_gpu)
    # each probe on its own
    for p in range(rec.ports):
        assert rel_l2(rec.series[2 * p::2 * rec.ports], o32.series[2 * p::2 * rec.ports]) <= TOL


@pytest.mark.parametrize("fused", [True, False])
def test_debye_spheres_match(gpu, fused):
    """Random sigma/eps spheres with a shared one-pole Debye model and CPML."""
    sc = W.spheres(56, pml=6, count=14, rmin=3, rmax=12, steps=500, fused=fused)
    sim = fdtd.Sim.try_new(*sc.args())
    assert sim.count("debye_edges") > 0
    o32 = O.run_cpu(O.OracleSim(*sc.args(), bits=32), 0, sc.pulse, sc.extras, keep_fields=True)
    rec = fdtd.run(gpu, sim, 0, sc.pulse, sc.extras, keep_fields=True)
    for name in ("e", "h", "series"):
        err = rel_l2(getattr(rec, name), getattr(o32, name))
        print(name, err)
        assert err <= TOL, (name, err)


def test_wide_class_ids_match(gpu):
    """Per-cell random permittivity: more than 65536 node classes, so 32-bit class ids."""
    sc = W.dielectric_box(44, pml=4, steps=300)
    rng = np.random.default_rng(3)
    sc.mats.eps[:] = rng.uniform(1.0, 8.0, sc.mats.eps.size).astype(np.float32)
    sim = fdtd.Sim.try_new(*sc.args())
    assert sim.coef_classes() > 65536
    o32 = O.run_cpu(O.OracleSim(*sc.args(), bits=32), 0, sc.pulse, sc.extras, keep_fields=True)
    rec = fdtd.run(gpu, sim, 0, sc.pulse, sc.extras, keep_fields=True)
    for name in ("e", "h", "series"):
        assert rel_l2(getattr(rec, name), getattr(o32, name)) <= TOL


@pytest.fixture(scope="module")
def patch():
    sc = W.patch_antenna(64, 64, 48, pml=8, patch=(14, 10), steps=1200)
    sim = fdtd.Sim.try_new(*sc.args())
    _with_ntff(sc, sim, 3)
    sc.extras.plane_k = sc.info["kg"] + 4
    o32 = O.run_cpu(O.OracleSim(*sc.args(), bits=32), 0, sc.pulse, sc.extras)
    return sc, sim, o32


def test_patch_antenna_dft_ntff_and_far_field_match(gpu, patch):
    sc, sim, o32 = patch
    rec = fdtd.run(gpu, sim, 0, sc.pulse, sc.extras)
    for name in ("series", "plane", "ntff"):
        err = rel_l2(getattr(rec, name), getattr(o32, name))
        print(name, err)
        assert err <= TOL, (name, err)
    p = fdtd.patches(sim, 3)
    th = np.radians(np.arange(0, 181, 15))
    ph = np.radians(np.arange(0, 360, 30))
    T, P = np.meshgrid(th, ph, indexing="ij")
    dirs = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], -1).reshape(-1, 3)
    for k, f in enumerate(sc.extras.freqs):
        far_gpu = fdtd.Far.load(p, rec.ntff, 3, k, f, gpu=gpu)
        want_f, want_u = O.far_eval(p.pos, p.area, o32.ntff.astype(np.float32), 3, k, f, dirs)
        got_u = far_gpu.intensities(dirs)
        err = rel_l2(got_u, want_u)
        print("far", f, err)
        assert err <= TOL
        # the device transform and the host transform agree to f64 rounding on the same input
        far_host = fdtd.Far.load(p, rec.ntff, 3, k, f)
        a, b = far_gpu.fields(dirs), far_host.fields(dirs)
        assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max()


def test_an_empty_cavity_rings_at_its_analytic_modes_on_the_gpu(gpu):
    """tests/fdtd.rs:189-236 through the CUDA engine."""
    sc = W.cavity()
    sc.extras.fused_e = True
    sim = fdtd.Sim.try_new(*sc.args())
    rec = fdtd.run(gpu, sim, 0, sc.pulse, sc.extras)
    v = rec.series[0::2].astype(np.float64)
    a, b, d = sc.info["a"], sc.info["b"], sc.info["d"]
    s = np.arange(len(v))
    for m, n_, p in [(1, 1, 0), (2, 1, 0), (1, 1, 1)]:
        fa = C0 / 2.0 * math.sqrt((m / a) ** 2 + (n_ / b) ** 2 + (p / d) ** 2)
        cands = [fa * (0.97 + 0.06 * q / 400.0) for q in range(401)]
        mags = [abs(np.sum(v * np.exp(-1j * 2 * math.pi * f * sim.dt * s))) for f in cands]
        peak = cands[int(np.argmax(mags))]
        assert abs(peak / fa - 1.0) < 0.004, (m, n_, p, peak, fa)


def test_a_run_stops_when_progress_says_so(gpu, every):
    sc, sim, _ = every
    sc.extras.max_steps = 5000
    calls = []

    def progress(steps, decay):
        calls.append(steps)
        return len(calls) < 2

    with pytest.raises(fdtd.FdtdError) as e:
        fdtd.run(gpu, sim, 0, sc.pulse, sc.extras, progress)
    sc.extras.max_steps = 1500
    assert str(e.value) == "cancelled"
    assert len(calls) == 2 and calls == [250, 500]


def test_an_unstable_run_is_reported(gpu):
    """A non-finite material makes non-finite fields: the first energy check returns the
    reference's error (run.rs:734-738)."""
    sc = W.dielectric_box(16, pml=3, steps=300)
    sc.mats.eps[100] = np.float32("nan")
    sim = fdtd.Sim.try_new(*sc.args())
    with pytest.raises(fdtd.FdtdError) as e:
        fdtd.run(gpu, sim, 0, sc.pulse, sc.extras)
    assert str(e.value) == "the FDTD run went unstable"


def test_a_run_stops_once_the_energy_has_decayed(gpu):
    """run.rs:745-747: past the pulse and min_steps, a decay of decay_db ends the run early."""
    sc = W.dielectric_box(24, pml=6, steps=20000)
    sc.extras.decay_db = 30.0
    sc.extras.check_every = 200
    sim = fdtd.Sim.try_new(*sc.args())
    rec = fdtd.run(gpu, sim, 0, sc.pulse, sc.extras)
    o = O.run_cpu(O.OracleSim(*sc.args(), bits=32), 0, sc.pulse, sc.extras)
    assert rec.steps < 20000 and rec.steps == o.steps
    assert rec.decay_db >= 30.0
    assert rel_l2(rec.series, o.series) <= TOL


@pytest.mark.parametrize("fused", [True, False])
def test_stepping_in_odd_chunks_is_the_same_as_one_run(gpu, fused):
    """The session's graph replays (blocks of 32, pairs, singles of either parity) give the same
    fields as one run."""
    sc = W.spheres(40, pml=5, count=8, rmin=3, rmax=8, steps=101, fused=fused)
    sim = fdtd.Sim.try_new(*sc.args())
    rec = fdtd.run(gpu, sim, 0, sc.pulse, sc.extras, keep_fields=True)
    s = fdtd.Session(gpu, sim, 0, sc.pulse, sc.extras)
    for k in (1, 33, 2, 1, 64):
        s.step(k)
    assert s.steps == 101
    nn = int(np.prod(sc.grid.dims()))
    assert np.array_equal(s.read("e", 3 * nn), rec.e)
    assert np.array_equal(s.read("h", 3 * nn), rec.h)
    assert np.array_equal(s.read("series", 101 * 2), rec.series)
    s.close()


def test_the_pipelines_are_the_cuda_kernels(gpu):
    # a grid with room for a clean box inside its CPML: the TMA march plus the two shell kernels
    sc = W.dielectric_box(48, pml=6, steps=4)
    sim = fdtd.Sim.try_new(*sc.args())
    s = fdtd.Session(gpu, sim, 0, sc.pulse, sc.extras)
    assert "TMA" in s.variant and "CPML shell" in s.variant, s.variant
    assert s.launches_per_step >= 4
    assert s.stream != 0
    s.close()
    # 11 nodes with a 4-cell CPML: a one-node clean box whose only tile reaches the k layer
    sc = W.spheres(10, pml=4, count=2, rmin=1, rmax=2, steps=30, fused=True)
    sim = fdtd.Sim.try_new(*sc.args())
    s = fdtd.Session(gpu, sim, 0, sc.pulse, sc.extras)
    assert "TMA" in s.variant and "(1 reaching the k layer)" in s.variant, s.variant
    s.close()
    rec = fdtd.run(gpu, sim, 0, sc.pulse, sc.extras)
    ref = O.run_cpu(O.OracleSim(*sc.args(), bits=32), 0, sc.pulse, sc.extras)
    assert rel_l2(rec.series, ref.series) <= 1e-4


def test_the_tma_step_and_the_direct_march_agree_bit_for_bit(gpu, monkeypatch):
    """The TMA-fed fused step and the direct-load fused march do the same arithmetic."""
    sc = W.spheres(72, pml=6, count=16, rmin=3, rmax=14, steps=120, fused=True)
    sim = fdtd.Sim.try_new(*sc.args())
    s = fdtd.Session(gpu, sim, 0, sc.pulse, sc.extras)
    assert s.variant.startswith("TMA"), s.variant
    s.close()
    a = fdtd.run(gpu, sim, 0, sc.pulse, sc.extras, keep_fields=True)
    monkeypatch.setenv("FIELDGRID_NO_TMA", "1")
    s = fdtd.Session(gpu, sim, 0, sc.pulse, sc.extras)
    assert not s.variant.startswith("TMA"), s.variant
    s.close()
    b = fdtd.run(gpu, sim, 0, sc.pulse, sc.extras, keep_fields=True)
    for name in ("e", "h", "series"):
        assert np.array_equal(getattr(a, name), getattr(b, name)), name
