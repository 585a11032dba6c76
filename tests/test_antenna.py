"""Host-side parts of the antenna workflow (no GPU): the mesher's own test (sims-antenna
src/fdtd/mesh.rs:136-171), the port spectra of finish (src/fdtd/mod.rs:237-266) against a direct
DFT, the port and metal-edge builders, and the half-wave dipole run on the oracle, held to the
reference's answers for it (tests/fdtd.rs:45-56): this pins the oracle to physics the reference
asserts, with the same mesh, set-up and finish code the GPU path uses."""
import math

import numpy as np
import pytest

from antenna_models import OracleRaster, dipole, radiated, resonance, sheen
from meshes import plate
from fieldgrid_b200 import antenna as A
from fieldgrid_b200 import fdtd
from oracle import oracle as O


def test_a_patch_mesh_keeps_its_lines_and_grows_smoothly():
    """mesh.rs:138-171."""
    m = A.Model(metal=[A.Aabb.new((-0.04, -0.04, 0.0), (0.04, 0.04, 0.0)),
                       A.Aabb.new((-0.02, -0.015, 0.0016), (0.02, 0.015, 0.0016))],
                dielectrics=[A.Dielectric(A.Aabb.new((-0.04, -0.04, 0.0), (0.04, 0.04, 0.0016)), 4.3, 0.02)],
                port=A.Port((0.005, 0.0, 0.0), (0.005, 0.0, 0.0016), 50.0), f0=2.4e9, span=0.2, fine=0.0)
    g = A.mesh(m, 8)
    for a, must in ((0, (0.005, 0.005)), (2, (0.0, 0.0016))):
        for v in must:
            assert np.any(np.abs(g.axis(a) - v) < 1e-7), (a, v)
    fine = A.C0 / (m.f0 * (1.0 + m.span)) / 80.0
    for v, inward in ((-0.02, 1.0), (0.02, -1.0)):
        for off in (inward * fine / 3.0, -inward * 2.0 * fine / 3.0):
            assert np.any(np.abs(g.x - (v + off)) < 1e-7), (v, off)
    for a in range(3):
        d = np.diff(g.axis(a))
        assert np.all(d > 0.0)
        assert np.all(d[1:] / d[:-1] < 1.9) and np.all(d[:-1] / d[1:] < 1.9), a
    inside = int(np.sum((g.z > 1e-9) & (g.z < 0.0016 - 1e-9)))
    assert inside >= 3, inside
    assert g.cells() < 3_000_000


def test_port_spectra_match_a_direct_dft():
    rng = np.random.default_rng(3)
    steps, ports, dt = 700, 2, 1.7e-12
    series = rng.standard_normal(steps * ports * 2).astype(np.float32)
    freqs = np.array([1e9, 7.5e9, 2.2e10])
    for port in range(ports):
        v, i = A.port_spectra(series, steps, ports, port, dt, freqs)
        s = series.reshape(steps, ports, 2)[:, port].astype(np.float64)
        n = np.arange(steps)
        w = 2 * math.pi * freqs[:, None]
        v_ref = np.sum(s[:, 0] * dt * np.exp(-1j * w * (n + 1) * dt), axis=1)
        i_ref = np.sum(s[:, 1] * dt * np.exp(-1j * w * (n + 0.5) * dt), axis=1)
        assert np.allclose(v, v_ref, rtol=1e-9, atol=1e-9 * np.abs(v_ref).max())
        assert np.allclose(i, i_ref, rtol=1e-9, atol=1e-9 * np.abs(i_ref).max())
    with pytest.raises(fdtd.FdtdError):
        A.port_spectra(series, steps, ports, ports, dt, freqs)


def test_port_and_metal_edges_follow_the_grid():
    g = fdtd.Grid.uniform((0.0, 0.0, 0.0), (0.01, 0.01, 0.01), (10, 10, 10), 2)
    p = A.port_def(g, A.Port((0.0051, 0.0049, 0.002), (0.0051, 0.0049, 0.0061), 50.0))
    assert [(e.comp, tuple(e.at)) for e in p.columns[0]] == [(2, (5, 5, 2)), (2, (5, 5, 3)), (2, (5, 5, 4)),
                                                             (2, (5, 5, 5))]
    mask = A.metal_edges(g, [A.Aabb.new((0.002, 0.003, 0.004), (0.005, 0.006, 0.004))])
    # a plate in z = 0.004: x and y edges of its plane, no z edges
    assert mask[2].sum() == 0
    assert mask[0].sum() == 3 * 4 and mask[1].sum() == 4 * 3
    assert mask[0][2:5, 3:7, 4].all() and mask[1][2:6, 3:6, 4].all()


def test_the_oracle_dipole_conserves_power_and_has_dipole_directivity():
    """tests/fdtd.rs:45-56 on the oracle: power balance within 1 %, directivity 2.15 +/- 0.05 dBi,
    resonance in [960, 1010) MHz."""
    opts = A.Options()
    s = A.setup(dipole(), opts, sim_factory=lambda *a: O.OracleSim(*a, bits=32),
                patch_fn=lambda sim, inset: fdtd.Patches(*O.patches(sim, inset)))
    rec = O.run_cpu(s.sim, 0, fdtd.Pulse(s.f0, s.fc), A.extras(s, opts))
    steps = int(rec.steps)
    v, i = A.port_spectra(rec.series, steps, 1, 0, s.sim.dt, np.concatenate([s.freqs, [s.f0]]))
    z = v / i
    p_in = 0.5 * (v[-1] * np.conj(i[-1])).real
    total, peak = radiated(lambda d: O.far_eval(s.patches.pos, s.patches.area, rec.ntff, 1, 0, s.f0, d)[1])
    eff = total / p_in
    d = 10.0 * math.log10(4.0 * math.pi * peak / total)
    res = resonance(s.freqs, z[:-1])
    print(f"oracle dipole: {steps} steps, power balance {eff:.4f}, directivity {d:.3f} dBi, resonance {res / 1e6:.1f} MHz")
    assert abs(eff - 1.0) < 0.01, eff
    assert abs(d - 2.15) < 0.05, d
    assert 960e6 <= res < 1010e6, res


def test_an_open_dielectric_mesh_is_refused():
    """tests/fdtd.rs:167-177 (sims-antenna)."""
    model = sheen(True)
    model.parts.append(A.Part(plate([0.0, 0.0], [1e-3, 1e-3], 2e-3), A.DielectricStuff(3.0, 0.0)))
    with pytest.raises(fdtd.FdtdError, match="^a dielectric part is not a closed mesh$"):
        A.setup(model, A.Options(far_field=False, max_steps=10), raster=OracleRaster())


def test_the_meshed_board_fills_the_cells_of_the_box_board():
    """Sheen's patch meshed (tests/fdtd.rs:119-127): its board, a closed cuboid whose faces the
    mesher pins to grid lines (mod.rs:78-88), gives the box board's materials cell for cell, and
    its metal plates mark edges on the planes z = 0 and z = h only."""
    meshed, boxed = sheen(True), sheen(False)
    grid = A.mesh(meshed, 8)
    r = OracleRaster()
    m1 = A.materials(grid, meshed, r)
    m2 = A.materials(grid, boxed)
    for name in ("eps", "inf", "sigma"):
        assert np.array_equal(getattr(m1, name), getattr(m2, name)), name
    assert np.count_nonzero(m1.eps != 1.0) > 1000
    args = A.sim_args(grid, meshed, meshed.port, r)
    n = grid.dims()
    mask = np.asarray(args[2]).reshape(3, *n)
    h = 0.794e-3
    ks = set(np.nonzero(mask.any(axis=(0, 1, 2)))[0].tolist())
    planes = {int(np.argmin(np.abs(grid.z - 0.0))), int(np.argmin(np.abs(grid.z - h)))}
    assert ks == planes, (ks, planes)
    assert not mask[2].any()     # flat plates mark no z edges

