"""The engine's host side, without a GPU: the C ABI loads and exports every declared symbol, the
product's Sim::try_new matches the oracle's bit for bit, and the refusals carry the reference's
texts. CPU only."""
import ctypes as C

import numpy as np
import pytest

from fieldgrid_b200 import _lib
from fieldgrid_b200 import fdtd
from fieldgrid_b200 import workloads as W
from fieldgrid_b200.fdtd import Edge, Materials, Media
from fieldgrid_b200.grid import Grid
from oracle import oracle as O


def test_the_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = _lib.exported_symbols()
    assert len(names) > 40
    for name in names:
        assert hasattr(L, name), name
    assert L.fg_version().decode().startswith("fieldgrid-b200")


SCENES = [
    lambda: W.everything(),
    lambda: W.dielectric_box(24, pml=5),
    lambda: W.spheres(40, pml=5, count=10, rmin=3, rmax=9),
    lambda: W.patch_antenna(40, 40, 36, pml=5, patch=(10, 8)),
    lambda: W.cavity(),
    lambda: W.wire_cavity(0.09e-3),
]


@pytest.mark.parametrize("make", SCENES)
def test_setup_matches_the_oracle_bit_for_bit(make):
    sc = make()
    ps = fdtd.Sim.try_new(*sc.args())
    os_ = O.OracleSim(*sc.args(), bits=32)
    assert ps.dt == os_.dt
    assert ps.dims() == tuple(sc.grid.dims())
    for c in range(3):
        ca, cb = ps.coefs(c)
        oca, ocb = os_.coefs(c)
        assert np.array_equal(cb, ocb.astype(np.float32))
        m = ocb != 0
        assert np.array_equal(ca[m], oca[m].astype(np.float32))
    for what in ("debye_edges", "wires", "inductors", "sheets", "ports", "port_src0"):
        assert ps.count(what) == os_.count(what), what
    if ps.count("wires"):
        pw = ps.wires
        h, e, c = os_.wires()
        assert np.array_equal(pw[:, 0], h.astype(np.uint32))
        assert np.array_equal(pw[:, 1::2], e.astype(np.uint32))
        assert np.array_equal(pw[:, 2::2].copy().view(np.float32), c.astype(np.float32))


def test_node_classes_stay_few():
    sc = W.dielectric_box(32, pml=6)
    assert fdtd.Sim.try_new(*sc.args()).coef_classes() <= 256


def test_a_thin_wire_outside_its_radius_range_is_refused():
    ax = [i * 1e-3 for i in range(11)]
    grid = Grid(ax, ax, ax, 0)
    for radius in (0.6e-3, 0.01e-3):
        with pytest.raises(fdtd.FdtdError) as e:
            fdtd.Sim.try_new(grid, Materials.new(grid), None, [], [], [], Media(wires=[(Edge(2, (5, 5, 4)), radius)]))
        assert "from a 55th to half of its cell" in str(e.value)


def test_a_wire_in_the_absorbing_layer_is_refused():
    ax = [i * 1e-3 for i in range(21)]
    grid = Grid(ax, ax, ax, 4)
    with pytest.raises(fdtd.FdtdError) as e:
        fdtd.Sim.try_new(grid, Materials.new(grid), None, [], [], [], Media(wires=[(Edge(2, (3, 10, 10)), 2e-4)]))
    assert "clear of the grid's absorbing layer" in str(e.value)


def test_run_without_a_gpu_is_refused():
    """The Option<&Gpu> entry with None: this engine has no CPU path."""
    sc = W.dielectric_box(12, pml=2, steps=10)
    sim = fdtd.Sim.try_new(*sc.args())
    with pytest.raises(fdtd.FdtdError) as e:
        fdtd.run(None, sim, 0, sc.pulse, sc.extras)
    assert e.value.code == 3


def test_time_step_matches_the_formula():
    g = Grid.uniform((0, 0, 0), (1e-2, 2e-2, 3e-2), (10, 10, 10), 0)
    want = 0.99 / (fdtd.C0 * np.sqrt(3.0 / (1e-3) ** 2 * 0 + 1 / 1e-6 + 1 / 4e-6 + 1 / 9e-6))
    assert abs(fdtd.time_step(g) - want) / want < 1e-15


def test_patches_match_the_oracle():
    sc = W.patch_antenna(36, 36, 30, pml=4, patch=(8, 6))
    ps = fdtd.Sim.try_new(*sc.args())
    os_ = O.OracleSim(*sc.args(), bits=32)
    a = fdtd.patches(ps, 3)
    pos, area, gpu = O.patches(os_, 3)
    assert np.array_equal(a.gpu, gpu)
    assert np.array_equal(a.pos, pos)
    assert np.array_equal(a.area, area)


def test_far_field_on_the_host_matches_the_oracle():
    rng = np.random.default_rng(5)
    sc = W.patch_antenna(36, 36, 30, pml=4, patch=(8, 6))
    ps = fdtd.Sim.try_new(*sc.args())
    p = fdtd.patches(ps, 3)
    nf = 2
    acc = rng.standard_normal(p.area.size * nf * 12).astype(np.float32)
    dirs = rng.standard_normal((17, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    far = fdtd.Far.load(p, acc, nf, 1, 10e9, (0.5, -0.25))
    got = far.fields(dirs)
    want, inten = O.far_eval(p.pos, p.area, acc, nf, 1, 10e9, dirs, (0.5, -0.25))
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    assert np.allclose(far.intensities(dirs), inten, rtol=1e-12)
    t, pk = far.radiated(6)
    t2, pk2 = O.far_radiated(p.pos, p.area, acc, nf, 1, 10e9, 6, (0.5, -0.25))
    assert abs(t - t2) <= 1e-12 * abs(t2) and abs(pk - pk2) <= 1e-12 * abs(pk2)


def test_setup_is_fast_at_a_million_nodes():
    import time
    sc = W.spheres(100, pml=8, count=20, rmin=4, rmax=12)
    t = time.time()
    fdtd.Sim.try_new(*sc.args())
    assert time.time() - t < 30.0
