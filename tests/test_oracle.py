"""Pins the oracle (the CPU restatement of sims-field's FDTD) to the reference's own known-answer
tests, re-expressed: crates/sims-field/src/fdtd/run.rs:775-858 and crates/sims-field/tests/fdtd.rs.
CPU only."""
import math

import numpy as np
import pytest

from fieldgrid_b200 import workloads as W
from fieldgrid_b200.fdtd import C0, Edge, Extras, Materials, Media, PortDef, idx
from fieldgrid_b200.grid import Grid
from oracle import oracle as O


def _line(n):
    return [i * 1e-3 * (1.0 + 0.1 * i) for i in range(n)]


def test_a_port_loop_circles_only_its_own_columns():
    """run.rs:775-823: a ring port's loop is the superposition of its single-column loops."""
    grid = Grid(_line(9), _line(8), _line(7), 0)

    def column(i, j):
        return [Edge(2, (i, j, 3))]

    ring = [column(i, j) for i in range(2, 5) for j in range(2, 5) if (i, j) != (3, 3)]
    ports = [PortDef("p", ring, 50.0, False)] + [PortDef("q", [column(i, j)], 50.0, False)
                                                  for i in range(2, 5) for j in range(2, 5)]
    sim = O.OracleSim(grid, Materials.new(grid), None, [], ports, [], Media(), bits=32)
    n = grid.dims()
    got = sim.port_loop(0, 2, 3)
    singles = {}
    q = 1
    for i in range(2, 5):
        for j in range(2, 5):
            singles[(i, j)] = sim.port_loop(q, 2, 3)
            q += 1
    want = {}
    for c in ring:
        for id_, comp, w in singles[(c[0].at[0], c[0].at[1])]:
            want[(id_, comp)] = want.get((id_, comp), 0.0) + w
    want = {k: v for k, v in want.items() if abs(v) > 1e-12}
    assert len(got) == 16 and len(want) == 16
    for id_, comp, w in got:
        assert abs(want[(id_, comp)] - w) < 1e-15
    for id_, comp, w in singles[(3, 3)]:
        back = [g for g in got if g[0] == id_ and g[1] == comp]
        assert back and back[0][2] == -w
    single_x = singles[(3, 3)]
    sq = lambda i, j: idx(n, i, j, 3)  # noqa: E731
    assert len(single_x) == 4
    assert any(s[0] == sq(3, 3) and s[1] == 1 and s[2] > 0 for s in single_x)
    assert any(s[0] == sq(2, 3) and s[1] == 1 and s[2] < 0 for s in single_x)
    assert any(s[0] == sq(3, 3) and s[1] == 0 and s[2] < 0 for s in single_x)
    assert any(s[0] == sq(3, 2) and s[1] == 0 and s[2] > 0 for s in single_x)


def test_coefficient_sets_give_back_every_edge():
    """run.rs:825-858: CoefSets round-trips every (ca, cb), narrow (u16 pairs) and wide (u32)."""
    grid = Grid(_line(9), _line(8), _line(7), 0)
    mats = Materials.new(grid)
    mats.eps[:] = 1.0 + (np.arange(mats.eps.size) % 5)
    mats.sigma[:] = (np.arange(mats.sigma.size) % 3) * 0.01
    port = PortDef("p", [[Edge(2, (4, 4, 3))]], 50.0, False)

    def pec(c, p):
        return (c == 0) & (p[2] == 2)

    sim = O.OracleSim(grid, mats, pec, [], [port], [], Media(), bits=32)
    nn = int(np.prod(grid.dims()))
    cas = [sim.coefs(c) for c in range(3)]
    for narrow in (1 << 16, 1):
        index, sets, wide = sim.coef_sets(narrow)
        assert wide == (narrow == 1)
        assert sets.shape[0] > 2
        flat = index if wide else np.stack([index & 0xFFFF, index >> 16], 1).reshape(-1)[: 3 * nn]
        for c in range(3):
            ca, cb = cas[c]
            got = sets[flat[c * nn:(c + 1) * nn]]
            assert np.array_equal(got[:, 1], cb.astype(np.float32))
            m = cb != 0
            assert np.array_equal(got[m, 0], ca[m].astype(np.float32))


def _spectrum_peak(v, dt, fa):
    s = np.arange(len(v))
    cands = [fa * (0.97 + 0.06 * q / 400.0) for q in range(401)]
    mags = [abs(np.sum(v * np.exp(-1j * 2 * math.pi * f * dt * s))) for f in cands]
    return cands[int(np.argmax(mags))]


def test_an_empty_cavity_rings_at_its_analytic_modes():
    """tests/fdtd.rs:189-236: TE/TM 110, 210, 111 within 0.4 % of c/2 sqrt(...)."""
    sc = W.cavity()
    sim = O.OracleSim(*sc.args(), bits=32)
    rec = O.run_cpu(sim, 0, sc.pulse, sc.extras)
    v = rec.series[0::2]
    a, b, d = sc.info["a"], sc.info["b"], sc.info["d"]
    for m, n_, p in [(1, 1, 0), (2, 1, 0), (1, 1, 1)]:
        fa = C0 / 2.0 * math.sqrt((m / a) ** 2 + (n_ / b) ** 2 + (p / d) ** 2)
        peak = _spectrum_peak(v, sim.dt, fa)
        assert abs(peak / fa - 1.0) < 0.004, (m, n_, p, peak, fa)


def test_thin_wires_at_either_end_of_their_radius_stay_stable():
    """tests/fdtd.rs:238-269: over 40 000 steps the late peak stays below twice the early one."""
    for radius in (0.09e-3, 1.7e-3):
        sc = W.wire_cavity(radius)
        sim = O.OracleSim(*sc.args(), bits=32)
        rec = O.run_cpu(sim, 0, sc.pulse, sc.extras)
        v = np.abs(rec.series[0::2])
        early, late = v[5000:10000].max(), v[35000:40000].max()
        assert late < 2.0 * early, (radius, early, late)


def test_a_thin_wire_outside_its_radius_range_is_refused():
    """tests/fdtd.rs:271-286."""
    ax = [i * 1e-3 for i in range(11)]
    grid = Grid(ax, ax, ax, 0)
    for radius in (0.6e-3, 0.01e-3):
        with pytest.raises(O.OracleError) as e:
            O.OracleSim(grid, Materials.new(grid), None, [], [], [], Media(wires=[(Edge(2, (5, 5, 4)), radius)]))
        assert "from a 55th to half of its cell" in str(e.value)


def test_a_run_stops_when_progress_says_so():
    """tests/fdtd.rs:176-187."""
    sc = W.everything(steps=5000)
    sim = O.OracleSim(*sc.args(), bits=32)
    calls = []

    def progress(steps, decay):
        calls.append(steps)
        return len(calls) < 2

    with pytest.raises(O.OracleError) as e:
        O.run_cpu(sim, 0, sc.pulse, sc.extras, progress)
    assert str(e.value) == "cancelled"
    assert len(calls) == 2


def test_f32_and_f64_runs_agree_on_the_every_feature_scene():
    """The f32 restatement stays close to its own FP64 run (the error budget the engine's
    parity is stated against)."""
    sc = W.everything(steps=600)
    s32 = O.OracleSim(*sc.args(), bits=32)
    s64 = O.OracleSim(*sc.args(), bits=64)
    r32 = O.run_cpu(s32, 0, sc.pulse, sc.extras)
    r64 = O.run_cpu(s64, 0, sc.pulse, sc.extras)
    for a, b in ((r32.series, r64.series), (r32.plane, r64.plane)):
        err = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert err < 1e-3, err


def test_patches_cover_the_box_faces():
    """ntff.rs:11-59: 2 * (faces) patches, each with 12 in-grid node ids and a normal axis."""
    sc = W.dielectric_box(16, pml=3, steps=1)
    sim = O.OracleSim(*sc.args(), bits=32)
    pos, area, gpu = O.patches(sim, 1)
    n = sc.grid.dims()
    side = n[0] - 1 - 2 * (3 + 1)
    assert pos.shape[0] == 6 * side * side
    g = gpu.reshape(-1, 13)
    assert set(np.unique(g[:, 0] & 3)) == {0, 1, 2}
    assert g[:, 1:].max() < np.prod(n)
    assert np.allclose(area, 1e-6)
