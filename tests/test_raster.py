"""The oracle's rasteriser (oracle/raster_oracle.cpp, a restatement of raster.rs and bvh.rs)
against the reference's own rasteriser tests, re-expressed: crates/sims-field/tests/raster.rs
(fill: a box fills exactly its samples, a sphere's volume on a graded grid, a thin plate kept as a
skin, an empty mesh) and crates/sims-field/tests/mesh.rs (closed, sheet_edges on and between grid
planes, solid_edges / solid_cells of a box, a slanted plate's staircase). CPU only."""
import math

import numpy as np

from fieldgrid_b200.grid import Grading, Grid, centres, graded, uniform
from oracle import oracle as O
from tests.meshes import cuboid, plate, quad, sphere, torus


def _unpack_xfast(n, c):
    return c % n[0], c // n[0] % n[1], c // (n[0] * n[1])


def test_a_box_fills_exactly_the_samples_inside_it():
    """raster.rs tests:44-59."""
    line = uniform(0.0, 1.0, 20)
    n = [len(line)] * 3
    inside, thin = O.raster_fill(cuboid([0.22, 0.31, 0.405], [0.71, 0.66, 0.9]), [line] * 3, n, 1)

    def want(a, b):
        return sum(1 for s in line if a < s < b)
    ids = np.nonzero(inside)[0]
    assert len(ids) == want(0.22, 0.71) * want(0.31, 0.66) * want(0.405, 0.9)
    for c in ids:
        i, j, k = _unpack_xfast(n, int(c))
        assert 0.22 < line[i] < 0.71 and 0.31 < line[j] < 0.66 and 0.405 < line[k] < 0.9
    assert not thin.any()


def test_a_sphere_fills_its_volume_on_a_graded_grid():
    """raster.rs tests:61-79."""
    line = np.array(graded([-1.0, 1.0], Grading([(0.0, 0.01)], lambda _x: 0.05, 1.1, 0.0)))
    cells = centres(line)
    widths = np.diff(line)
    n = [len(cells)] * 3
    inside, _ = O.raster_fill(sphere(0.6, 48), [cells] * 3, n, 1)
    volume = 0.0
    for c in np.nonzero(inside)[0]:
        i, j, k = _unpack_xfast(n, int(c))
        volume += widths[i] * widths[j] * widths[k]
    exact = 4.0 / 3.0 * math.pi * 0.6 ** 3
    assert abs(volume / exact - 1.0) < 0.02, (volume, exact)


def test_a_plate_thinner_than_a_cell_is_kept_as_a_skin():
    """raster.rs tests:81-92."""
    line = uniform(0.0, 1.0, 10)
    n = [len(line)] * 3
    inside, thin = O.raster_fill(cuboid([0.15, 0.15, 0.52], [0.85, 0.85, 0.54]), [line] * 3, n, 1)
    assert not inside.any()
    k = int(np.nonzero(np.abs(line - 0.5) < 1e-12)[0][0])
    inner = sum(1 for s in line if 0.15 < s < 0.85)
    ids = np.nonzero(thin)[0]
    assert len(ids) == inner * inner
    assert all(_unpack_xfast(n, int(c))[2] == k for c in ids)


def test_nothing_to_fill_from_an_empty_mesh():
    """raster.rs tests:94-99."""
    line = uniform(0.0, 1.0, 4)
    inside, thin = O.raster_fill(np.zeros((0, 3, 3)), [line] * 3)
    assert not inside.any() and not thin.any()


def _grid():
    return Grid(uniform(0.0, 1.0, 20), uniform(0.0, 1.0, 20), uniform(0.0, 1.0, 20), 0)


def test_a_box_is_closed_and_a_plate_is_not():
    """mesh.rs tests:28-33."""
    assert O.raster_closed(cuboid([0.1] * 3, [0.4] * 3))
    assert not O.raster_closed(plate([0.1, 0.1], [0.4, 0.4], 0.5))
    assert not O.raster_closed(np.zeros((0, 3, 3)))


def test_a_plate_on_a_grid_plane_marks_the_edges_it_covers():
    """mesh.rs tests:35-62."""
    g = _grid()
    n = g.dims()
    mask = O.raster_sheet_edges(plate([0.2, 0.3], [0.6, 0.5], 0.5), g)
    lo, hi = (0.2, 0.3), (0.6, 0.5)
    for c in range(3):
        m = mask[c].reshape(n)
        want = np.zeros(n, bool)
        if c != 2:
            for i in range(n[0]):
                for j in range(n[1]):
                    p = (i, j, 10)
                    if p[c] + 1 >= n[c]:
                        continue
                    ok = True
                    for a in range(2):
                        x = g.axis(a)[p[a]]
                        if a == c:
                            ok &= x >= lo[a] - 1e-9 and g.axis(a)[p[a] + 1] <= hi[a] + 1e-9
                        else:
                            ok &= lo[a] - 1e-9 <= x <= hi[a] + 1e-9
                    want[i, j, 10] = ok
        assert np.array_equal(m, want), c


def test_a_plate_between_planes_lands_on_the_nearest_one():
    """mesh.rs tests:64-74."""
    g = _grid()
    n = g.dims()
    for z, k in [(0.512, 10), (0.538, 11), (0.525, 11), (0.5, 10)]:
        mask = O.raster_sheet_edges(plate([0.2, 0.2], [0.6, 0.6], z), g)
        planes = sorted(set(int(i) % n[2] for i in np.nonzero(mask[0])[0]))
        assert planes == [k], z


def test_a_solid_box_fills_the_edges_inside_it():
    """mesh.rs tests:76-113."""
    g = _grid()
    n = g.dims()
    lo, hi = [0.22, 0.31, 0.41], [0.68, 0.59, 0.77]
    mesh = cuboid(lo, hi)
    mask = O.raster_solid_edges(mesh, g)
    for c in range(3):
        m = mask[c].reshape(n)
        for i in range(n[0]):
            for j in range(n[1]):
                for k in range(n[2]):
                    p = (i, j, k)
                    if p[c] + 1 >= n[c]:
                        continue
                    mid = [0.5 * (g.axis(a)[p[a]] + g.axis(a)[p[a] + 1]) if a == c else g.axis(a)[p[a]]
                           for a in range(3)]
                    assert m[i, j, k] == all(lo[a] < mid[a] < hi[a] for a in range(3)), (c, p)
    cells = O.raster_solid_cells(mesh, g)

    def centre(a, b):
        return sum(1 for i in range(20) if a < (i + 0.5) / 20.0 < b)
    assert cells.sum() == centre(0.22, 0.68) * centre(0.31, 0.59) * centre(0.41, 0.77)


def test_a_slanted_plate_marks_a_staircase_that_stays_on_it():
    """mesh.rs tests:115-135."""
    g = _grid()
    n = g.dims()
    tri = quad([0.2, 0.2, 0.3], [0.7, 0.2, 0.3], [0.7, 0.6, 0.7], [0.2, 0.6, 0.7])
    mask = O.raster_sheet_edges(tri, g)
    count = 0
    for c in range(3):
        for ident in np.nonzero(mask[c])[0]:
            p = (ident // (n[1] * n[2]), ident // n[2] % n[1], ident % n[2])
            mid = [0.5 * (g.axis(a)[p[a]] + g.axis(a)[p[a] + 1]) if a == c else g.axis(a)[p[a]] for a in range(3)]
            d = (mid[2] - 0.3) - (mid[1] - 0.2)
            assert abs(d) / math.sqrt(2.0) <= 0.5 * 0.05 * math.sqrt(2.0) + 1e-9, (c, p, d)
            count += 1
    assert count > 200, count


def test_the_product_closed_check_equals_the_oracle():
    """fg_raster_closed (host code in the library) against the oracle on closed and open meshes."""
    from fieldgrid_b200 import raster as R
    for mesh, want in [(cuboid([0.1] * 3, [0.4] * 3), True), (np.array(plate([0.1, 0.1], [0.4, 0.4], 0.5)), False),
                       (sphere(0.3, 24), True), (torus(0.3, 0.1, 24, 12), True), (np.zeros((0, 3, 3)), False),
                       (sphere(0.3, 24)[:-1], False)]:
        assert R.closed(mesh) == want == O.raster_closed(mesh)
