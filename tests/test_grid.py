"""The node-line helpers against the reference's own cases (crates/sims-field/tests/grid.rs). CPU only."""
from fieldgrid_b200.grid import Grading, Grid, cell_of, centres, graded, nearest, pad, smooth, uniform


def test_nearest_picks_the_closer_line_and_clamps_at_the_ends():
    line = [0.0, 1.0, 3.0, 7.0]
    assert nearest(line, -5.0) == 0
    assert nearest(line, 0.4) == 0
    assert nearest(line, 0.5) == 0
    assert nearest(line, 0.6) == 1
    assert nearest(line, 2.1) == 2
    assert nearest(line, 5.0) == 2
    assert nearest(line, 99.0) == 3


def test_cell_of_stays_inside_the_cells():
    line = [0.0, 1.0, 3.0, 7.0]
    assert cell_of(line, -1.0) == 0
    assert cell_of(line, 0.0) == 0
    assert cell_of(line, 1.0) == 1
    assert cell_of(line, 6.9) == 2
    assert cell_of(line, 7.0) == 2
    assert cell_of(line, 70.0) == 2


def test_a_uniform_grid_counts_its_cells():
    g = Grid.uniform((0.0, 0.0, 0.0), (1.0, 2.0, 3.0), (2, 4, 6), 3)
    assert g.dims() == (3, 5, 7)
    assert g.cells() == 48
    assert list(g.centres(0)) == [0.25, 0.75]
    assert list(uniform(0.0, 1.0, 4)) == [0.0, 0.25, 0.5, 0.75, 1.0]
    assert list(centres([0.0, 2.0, 6.0])) == [1.0, 4.0]


def _grade(fixed, features, coarse, ratio, fill):
    return graded(fixed, Grading(features, lambda _x: coarse, ratio, fill))


def test_graded_lines_keep_the_fixed_lines_and_grow_from_features():
    lines = _grade([1.0, 0.0, 0.3, 0.3], [(0.0, 0.01)], 0.1, 1.3, 0.0)
    for v in (0.0, 0.3, 1.0):
        assert any(abs(x - v) < 1e-12 for x in lines), v
    d = [b - a for a, b in zip(lines[:-1], lines[1:])]
    assert all(x > 0 for x in d)
    assert d[0] < 0.012
    assert all(x <= 0.1 + 1e-9 for x in d)
    for a, b in zip(d[:-1], d[1:]):
        assert b / a < 1.35


def test_the_fill_rule_drops_a_sliver_cell():
    plain = _grade([0.0, 0.11], [], 0.1, 1.3, 0.0)
    filled = _grade([0.0, 0.11], [], 0.1, 1.3, 0.8)
    assert len(plain) == 3
    assert filled == [0.0, 0.11]


def test_smoothing_splits_a_jump():
    line = smooth([0.0, 1.0, 2.0, 10.0], 1.5)
    for w0, w1, w2 in zip(line[:-2], line[1:-1], line[2:]):
        a, b = w1 - w0, w2 - w1
        assert b <= 1.5 * a + 1e-12 and a <= 1.5 * b + 1e-12
    assert line[-1] == 10.0


def test_padding_repeats_the_end_cells():
    assert pad([0.0, 1.0, 3.0], 2) == [-2.0, -1.0, 0.0, 1.0, 3.0, 5.0, 7.0]
