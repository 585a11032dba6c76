"""The antenna workflow of sims-antenna (src/fdtd/{mod,mesh,engine}.rs, src/solve.rs:416-490) run on
this engine, held to the answers the reference's own tests hold (crates/sims-antenna/tests/fdtd.rs):

  - the half-wave dipole conserves power to 1 %, has the dipole's 2.15 +/- 0.05 dBi directivity and
    resonates between 960 and 1010 MHz (tests/fdtd.rs:45-56);
  - the same dipole on the oracle (the CPU restatement of the reference's CPU FDTD) gives the same
    impedance sweep and radiated power (the CPU-vs-GPU test of tests/fdtd.rs:58-71);
  - Sheen's microstrip patch, built from boxes, matches best within 1.5 % of the measured 7.5 GHz
    with S11 below -10 dB (tests/fdtd.rs:88-167; the meshed-triangle variant needs the reference's
    rasteriser and is not run);
  - the volume result reports a broadside gain within 0.2 dB of its dBi figure and a null toward
    the dipole's axis (tests/fdtd.rs:181-190).
These pin the engine and the oracle to physical answers that the reference itself asserts.
"""
import math

import numpy as np
import pytest

from antenna_models import OracleRaster, dipole, radiated, resonance, sheen
from fieldgrid_b200 import antenna as A
from fieldgrid_b200 import fdtd
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dipole_out(gpu):
    return A.run_gpu(dipole(), A.Options(), g=gpu)


def test_a_dipole_conserves_power_and_has_dipole_directivity(dipole_out):
    out = dipole_out
    total, peak = radiated(out.far.intensities)
    eff = total / out.p_in
    d = 10.0 * math.log10(4.0 * math.pi * peak / total)
    f = resonance(out.sweep.freqs, out.sweep.z)
    print(f"dipole: {out.stats.steps} steps, {out.stats.cells} cells, decay {out.stats.decay_db:.1f} dB, "
          f"power balance {eff:.4f}, directivity {d:.3f} dBi, resonance {f / 1e6:.1f} MHz, Z0 {out.z0:.2f}")
    assert abs(eff - 1.0) < 0.01, eff
    assert abs(d - 2.15) < 0.05, d
    assert 960e6 <= f < 1010e6, f


def test_the_dipole_on_the_gpu_agrees_with_the_oracle(dipole_out):
    model, opts = dipole(), A.Options()
    s = A.setup(model, opts, sim_factory=lambda *a: O.OracleSim(*a, bits=32),
                patch_fn=lambda sim, inset: fdtd.Patches(*O.patches(sim, inset)))
    pos, area = s.patches.pos, s.patches.area
    rec = O.run_cpu(s.sim, 0, fdtd.Pulse(s.f0, s.fc), A.extras(s, opts))
    steps = int(rec.steps)
    assert steps == dipole_out.stats.steps
    v, i = A.port_spectra(rec.series, steps, 1, 0, s.sim.dt, s.freqs)
    z_cpu = v / i
    for a, b in list(zip(z_cpu, dipole_out.sweep.z))[::10]:
        assert abs(a - b) < 0.01 * abs(a) + 0.5, (a, b)
    tc, pc = radiated(lambda d: O.far_eval(pos, area, rec.ntff, 1, 0, s.f0, d)[1])
    tg, pg = radiated(dipole_out.far.intensities)
    print(f"dipole oracle vs gpu: Z rel {np.max(np.abs(z_cpu - dipole_out.sweep.z) / np.abs(z_cpu)):.2e}, "
          f"total {tc / tg - 1:.2e}, peak {pc / pg - 1:.2e}")
    assert abs(tc / tg - 1.0) < 0.01 and abs(pc / pg - 1.0) < 0.01


@pytest.mark.parametrize("meshed", [False, True])
def test_sheens_microstrip_patch_resonates_where_it_was_measured(gpu, meshed):
    """tests/fdtd.rs:158-165 (sims-antenna), box and meshed (rasterised) forms."""
    out = A.run_gpu(sheen(meshed), A.Options(far_field=False), g=gpu)
    s11 = np.abs(out.s11())
    q = int(np.argmin(s11))
    f, db = float(out.sweep.freqs[q]), 20.0 * math.log10(s11[q])
    print(f"sheen (meshed {meshed}): {out.stats.steps} steps, {out.stats.cells} cells: S11 {db:.1f} dB at "
          f"{f / 1e9:.4f} GHz")
    assert abs(f / 7.5e9 - 1.0) < 0.015, f
    assert db < -10.0, db


def test_a_volume_result_reports_consistent_gains(dipole_out):
    r = A.volume_result(dipole_out)
    broadside = r.gain_dbi((1.0, 0.0, 0.0))
    print(f"volume result: dbi {r.dbi:.3f} directivity {r.directivity:.3f} efficiency {r.efficiency:.4f} "
          f"broadside {broadside:.3f}")
    assert abs(broadside - r.dbi) < 0.2, (broadside, r.dbi)
    assert r.gain_dbi((0.0, 0.0, 1.0)) < r.dbi - 20.0


def test_the_cuda_rasteriser_builds_the_oracles_sim_arguments(gpu):
    """The meshed Sheen patch's materials and PEC mask through the CUDA rasteriser equal those
    through the oracle's, bit for bit."""
    from fieldgrid_b200.raster import GpuRaster
    model = sheen(True)
    grid = A.mesh(model, 8)
    a = A.sim_args(grid, model, model.port, GpuRaster(gpu))
    b = A.sim_args(grid, model, model.port, OracleRaster())
    for name in ("eps", "inf", "sigma", "debye"):
        assert np.array_equal(getattr(a[1], name), getattr(b[1], name)), name
    assert np.array_equal(np.asarray(a[2]), np.asarray(b[2]))
    assert np.asarray(a[2]).any()

