"""Batches of uneven grids (fg_batch_*): every grid's series and final fields equal stepping that
grid alone with the fused step, bit for bit, with a fixed shape and after the autotuner."""
import numpy as np
import pytest

from fieldgrid_b200 import fdtd
from fieldgrid_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scenes():
    return W.batch_grids(count=5, lo=16, hi=48, pml=4, steps=64, seed=11)


def alone(gpu, sc, steps):
    sim = fdtd.Sim.try_new(*sc.args())
    s = fdtd.Session(gpu, sim, 0, sc.pulse, sc.extras)
    s.step(steps)
    nn = int(np.prod(sc.grid.dims()))
    out = (s.read("series", steps * 2), s.read("e", 3 * nn), s.read("h", 3 * nn))
    s.close()
    return out


def check(gpu, b, scenes, steps):
    for q, sc in enumerate(scenes):
        nn = int(np.prod(sc.grid.dims()))
        ser, e, h = alone(gpu, sc, steps)
        assert np.array_equal(b.read(q, "series", steps * 2), ser), q
        assert np.array_equal(b.read(q, "e", 3 * nn), e), q
        assert np.array_equal(b.read(q, "h", 3 * nn), h), q
        assert np.abs(e).max() > 0


def test_a_batch_steps_each_grid_as_alone(gpu, scenes):
    sims = [fdtd.Sim.try_new(*sc.args()) for sc in scenes]
    b = fdtd.Batch(gpu, sims, [sc.pulse for sc in scenes], 64, tune=False, tile=1, seg=16, graph_steps=8)
    b.step(7)    # odd counts: the single-step graphs of both parities
    b.step(33)
    assert b.info()["steps"] == 40
    check(gpu, b, scenes, 40)
    b.close()


@pytest.mark.parametrize("tile,seg,name", [(3, 0, "graph branches"), (4, 0, "graph branches, direct march"),
                                          (4, 50, "graph branches, direct march"), (5, 0, "merged TMA launches")])
def test_graph_branches_step_each_grid_as_alone(gpu, scenes, tile, seg, name):
    """Branches of each grid's own step: the TMA march, the direct-load march for all grids, and
    the direct-load march for the grids under 50 thousand nodes only (a mix); and the merged
    launches (one TMA march and one shell launch of each kind over all grids)."""
    sims = [fdtd.Sim.try_new(*sc.args()) for sc in scenes]
    b = fdtd.Batch(gpu, sims, [sc.pulse for sc in scenes], 64, tune=False, tile=tile, seg=seg, graph_steps=4)
    assert b.info()["tile"] == name
    b.step(9)
    check(gpu, b, scenes, 9)
    b.close()


def test_the_tuned_batch_starts_from_step_zero(gpu, scenes):
    sims = [fdtd.Sim.try_new(*sc.args()) for sc in scenes]
    b = fdtd.Batch(gpu, sims, [sc.pulse for sc in scenes], 64, tune=True)
    info = b.info()
    assert info["steps"] == 0 and info["tuned_ms_per_step"] > 0 and info["persistent_blocks"] > 0
    b.step(24)
    check(gpu, b, scenes, 24)
    b.close()


def test_a_batch_refuses_wires_and_sheets(gpu):
    sc = W.everything(steps=10, fused=True)
    with pytest.raises(fdtd.FdtdError, match="no thin wires"):
        fdtd.Batch(gpu, [fdtd.Sim.try_new(*sc.args())], [sc.pulse], 10)


def test_merged_launches_on_larger_uneven_grids(gpu):
    """The merged mode on grids with Debye spheres, k-layer tiles and shells of different sizes,
    an odd step count: each grid bit for bit as stepped alone."""
    scenes = W.batch_grids(count=6, lo=40, hi=96, pml=6, steps=40, seed=5)
    sims = [fdtd.Sim.try_new(*sc.args()) for sc in scenes]
    b = fdtd.Batch(gpu, sims, [sc.pulse for sc in scenes], 40, tune=False, tile=5, graph_steps=8)
    assert b.info()["tile"] == "merged TMA launches"
    b.step(3)
    b.step(18)
    check(gpu, b, scenes, 21)
    b.close()


def test_merged_launches_with_grids_that_march_on_their_own(gpu):
    """A grid with no clean box for the TMA march (8 cells and a 4-cell CPML) first, then grids
    that the merged march covers: the first marches on its own inside the merged step, and every
    grid matches stepping it alone."""
    scenes = W.batch_grids(count=1, lo=8, hi=8, pml=4, steps=24, seed=3) + \
        W.batch_grids(count=4, lo=40, hi=72, pml=5, steps=24, seed=9)
    sims = [fdtd.Sim.try_new(*sc.args()) for sc in scenes]
    b = fdtd.Batch(gpu, sims, [sc.pulse for sc in scenes], 24, tune=False, tile=5, graph_steps=4)
    b.step(11)
    check(gpu, b, scenes, 11)
    b.close()

