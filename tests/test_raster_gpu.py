"""The CUDA rasteriser (csrc/raster.cu through the C ABI) against the oracle's restatement of
raster.rs / bvh.rs: every mask bit for bit, on the reference's test meshes and on larger ones
(a 48-ring sphere, a torus, a slanted plate) over graded and uniform grids."""
import numpy as np
import pytest

from fieldgrid_b200 import raster as R
from fieldgrid_b200.grid import Grading, Grid, centres, graded, uniform
from oracle import oracle as O
from tests.meshes import cuboid, plate, quad, sphere, torus

pytestmark = pytest.mark.gpu


def _graded_line():
    return np.array(graded([-1.0, 1.0], Grading([(0.0, 0.01)], lambda _x: 0.05, 1.1, 0.0)))


MESHES = {
    "box": lambda: cuboid([0.22, 0.31, 0.405], [0.71, 0.66, 0.9]),
    "thin_plate": lambda: cuboid([0.15, 0.15, 0.52], [0.85, 0.85, 0.54]),
    "sphere": lambda: sphere(0.3, 48, (0.5, 0.48, 0.52)),
    "torus": lambda: torus(0.28, 0.09, 40, 20, (0.5, 0.5, 0.5)),
    "empty": lambda: np.zeros((0, 3, 3)),
}


@pytest.mark.parametrize("name", list(MESHES))
@pytest.mark.parametrize("order", ["ijk", "xfast"])
def test_fill_equals_the_oracle(gpu, name, order):
    line = uniform(0.0, 1.0, 40)
    mesh = MESHES[name]()
    got = R.fill(gpu, mesh, [line, line, line], order)
    n = [len(line)] * 3
    inside, thin = O.raster_fill(mesh, [line] * 3, n, 0 if order == "ijk" else 1)
    assert np.array_equal(got.inside, np.nonzero(inside)[0])
    assert np.array_equal(got.thin, np.nonzero(thin)[0])
    if name in ("box", "sphere", "torus"):
        assert len(got.inside) > 0


def test_fill_of_a_sphere_on_a_graded_grid(gpu):
    """raster.rs tests:61-79's sphere on its graded cell centres."""
    cells = centres(_graded_line())
    mesh = sphere(0.6, 48)
    got = R.fill(gpu, mesh, [cells] * 3, "xfast")
    inside, thin = O.raster_fill(mesh, [cells] * 3, None, 1)
    assert np.array_equal(got.inside, np.nonzero(inside)[0])
    assert np.array_equal(got.thin, np.nonzero(thin)[0])


def _grids():
    line = _graded_line()
    return {"uniform": Grid(uniform(0.0, 1.0, 20), uniform(0.0, 1.0, 20), uniform(0.0, 1.0, 20), 0),
            "graded": Grid(line * 0.5 + 0.5, line * 0.5 + 0.5, line * 0.5 + 0.5, 0)}


@pytest.mark.parametrize("grid", ["uniform", "graded"])
@pytest.mark.parametrize("name", ["box", "sphere", "torus"])
def test_solid_edges_and_cells_equal_the_oracle(gpu, grid, name):
    g = _grids()[grid]
    mesh = {"box": cuboid([0.22, 0.31, 0.41], [0.68, 0.59, 0.77]), "sphere": sphere(0.3, 48, (0.5, 0.48, 0.52)),
            "torus": torus(0.28, 0.09, 40, 20, (0.5, 0.5, 0.5))}[name]
    got = R.solid_edges(gpu, mesh, g)
    want = O.raster_solid_edges(mesh, g)
    for c in range(3):
        assert np.array_equal(got[c], want[c]), c
    assert any(m.any() for m in got)
    assert np.array_equal(R.solid_cells(gpu, mesh, g), O.raster_solid_cells(mesh, g))


@pytest.mark.parametrize("grid", ["uniform", "graded"])
@pytest.mark.parametrize("name", ["plate", "between", "slanted", "sphere_shell"])
def test_sheet_edges_equal_the_oracle(gpu, grid, name):
    g = _grids()[grid]
    mesh = {"plate": plate([0.2, 0.3], [0.6, 0.5], 0.5), "between": plate([0.2, 0.2], [0.6, 0.6], 0.538),
            "slanted": quad([0.2, 0.2, 0.3], [0.7, 0.2, 0.3], [0.7, 0.6, 0.7], [0.2, 0.6, 0.7]),
            "sphere_shell": sphere(0.3, 24, (0.5, 0.48, 0.52))}[name]
    got = R.sheet_edges(gpu, mesh, g)
    want = O.raster_sheet_edges(mesh, g)
    for c in range(3):
        assert np.array_equal(got[c], want[c]), c
    assert any(m.any() for m in got)

