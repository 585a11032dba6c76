"""Rectilinear node lines: the `Grid` of sims-field (crates/sims-field/src/grid.rs).

Host-side helpers that build the node lines a solve runs on. They carry no device work.
"""
from __future__ import annotations

import bisect
import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Grid:
    """Node lines along x, y, z plus the CPML depth in cells (grid.rs:2-7)."""

    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    pml: int = 0

    def __post_init__(self):
        self.x = np.asarray(self.x, dtype=np.float64)
        self.y = np.asarray(self.y, dtype=np.float64)
        self.z = np.asarray(self.z, dtype=np.float64)

    @staticmethod
    def uniform(lo, hi, n, pml: int) -> "Grid":
        """grid.rs:9-13."""
        return Grid(uniform(lo[0], hi[0], n[0]), uniform(lo[1], hi[1], n[1]), uniform(lo[2], hi[2], n[2]), pml)

    def axis(self, a: int) -> np.ndarray:
        return (self.x, self.y, self.z)[a]

    def dims(self):
        """Node counts per axis (cells + 1), grid.rs:24-26."""
        return (len(self.x), len(self.y), len(self.z))

    def cells(self) -> int:
        return (len(self.x) - 1) * (len(self.y) - 1) * (len(self.z) - 1)

    def nearest(self, a: int, v: float) -> int:
        return nearest(self.axis(a), v)

    def cell_of(self, a: int, v: float) -> int:
        return cell_of(self.axis(a), v)

    def centres(self, a: int) -> np.ndarray:
        return centres(self.axis(a))


def uniform(lo: float, hi: float, cells: int) -> np.ndarray:
    """grid.rs:44-46: lo + (hi - lo) * i / cells for i in 0..=cells."""
    return np.array([lo + (hi - lo) * i / cells for i in range(cells + 1)], dtype=np.float64)


def nearest(line, v: float) -> int:
    """Index of the closer node line, clamped at the ends (grid.rs:48-55)."""
    line = list(line)
    i = bisect.bisect_left(line, v)
    if i >= 1 and i < len(line):
        j = i - 1
        if abs(v - line[j]) <= abs(line[i] - v):
            return j
    elif i >= 1 and i >= len(line):
        return i - 1
    return min(i, max(len(line) - 1, 0))


def cell_of(line, v: float) -> int:
    """The cell holding v, kept inside the cells (grid.rs:57-59)."""
    line = list(line)
    p = bisect.bisect_right(line, v)
    return min(max(p - 1, 0), max(len(line) - 2, 0))


def centres(line) -> np.ndarray:
    line = np.asarray(line, dtype=np.float64)
    return 0.5 * (line[:-1] + line[1:])


@dataclass
class Grading:
    """grid.rs:65-70: features (position, cell size), coarse size function, growth ratio, fill."""

    features: list = field(default_factory=list)
    coarse: object = None
    ratio: float = 1.3
    fill: float = 0.0


def graded(fixed, grading: Grading) -> list:
    """Lines through every fixed coordinate, sized to grow from features (grid.rs:72-111)."""
    fixed = sorted(float(v) for v in fixed)
    dedup = []
    for v in fixed:
        if not dedup or abs(v - dedup[-1]) >= 1e-9:
            dedup.append(v)
    fixed = dedup
    ratio = grading.ratio

    def size(x):
        s = grading.coarse(x)
        for at, sz in grading.features:
            s = min(s, sz + (ratio - 1.0) * abs(x - at))
        return s

    if not fixed:
        return []
    out = [fixed[0]]
    steps = 256
    for a, b in zip(fixed[:-1], fixed[1:]):
        acc = [0.0] * (steps + 1)
        for k in range(steps):
            x = a + (b - a) * (k + 0.5) / steps
            acc[k + 1] = acc[k] + (b - a) / steps / size(x)
        fine = max(math.ceil(acc[steps]), 1.0)
        fine = int(fine)
        if acc[steps] / fine >= grading.fill:
            n = fine
        else:
            n = max(int(math.floor(acc[steps] / grading.fill)), 1)
        for c in range(1, n):
            target = acc[steps] * c / n
            k = bisect.bisect_left(acc, target)
            k = min(max(k, 1), steps)
            t = (target - acc[k - 1]) / max(acc[k] - acc[k - 1], 1e-30)
            out.append(a + (b - a) * ((k - 1) + t) / steps)
        out.append(b)
    return out


def smooth(line, limit: float) -> list:
    """Split cells until neighbours differ by at most `limit` (grid.rs:113-132)."""
    line = list(line)
    for _ in range(200):
        d = [line[i + 1] - line[i] for i in range(len(line) - 1)]
        bad = None
        for i in range(len(d)):
            if (i > 0 and d[i] > limit * d[i - 1]) or (i + 1 < len(d) and d[i] > limit * d[i + 1]):
                bad = i
                break
        if bad is None:
            break
        i = bad
        cands = []
        if i >= 1:
            cands.append(d[i - 1])
        if i + 1 < len(d):
            cands.append(d[i + 1])
        small = min(cands) if cands else math.inf
        parts = int(max(math.ceil(d[i] / (limit * small)), 2.0))
        a, b = line[i], line[i + 1]
        extra = [a + (b - a) * k / parts for k in range(1, parts)]
        line[i + 1:i + 1] = extra
    return line


def pad(line, cells: int) -> list:
    """Repeat the end cells `cells` times on both sides (grid.rs:134-145)."""
    line = list(line)
    if len(line) < 2:
        return line
    first = line[1] - line[0]
    last = line[-1] - line[-2]
    pre = [line[0] - first * i for i in range(cells, 0, -1)]
    post = [line[-1] + last * i for i in range(1, cells + 1)]
    return pre + line + post
