"""Triangle meshes for the rasteriser tests: the cuboid and sphere of the reference's raster tests
(crates/sims-field/tests/raster.rs:5-39), the plate and quad of its mesh tests
(crates/sims-field/tests/mesh.rs:5-19), and a torus."""
import math

import numpy as np


def quad(a, b, c, d):
    return [[a, b, c], [a, c, d]]


def plate(lo, hi, z):
    return quad([lo[0], lo[1], z], [hi[0], lo[1], z], [hi[0], hi[1], z], [lo[0], hi[1], z])


def cuboid(lo, hi):
    def p(i):
        return [hi[a] if (i >> a) & 1 else lo[a] for a in range(3)]
    faces = [[0, 2, 3, 1], [4, 5, 7, 6], [0, 1, 5, 4], [2, 6, 7, 3], [0, 4, 6, 2], [1, 3, 7, 5]]
    out = []
    for f in faces:
        out += quad(p(f[0]), p(f[1]), p(f[2]), p(f[3]))
    return np.array(out, np.float64)


def sphere(radius, rings, centre=(0.0, 0.0, 0.0)):
    segments = 2 * rings
    pts = [[0.0, 0.0, radius], [0.0, 0.0, -radius]]
    for r in range(1, rings):
        theta = math.pi * r / rings
        for s in range(segments):
            phi = 2.0 * math.pi * s / segments
            pts.append([radius * math.sin(theta) * math.cos(phi), radius * math.sin(theta) * math.sin(phi),
                        radius * math.cos(theta)])

    def at(r, s):
        return 2 + (r - 1) * segments + s % segments
    tris = []
    for s in range(segments):
        tris.append([0, at(1, s), at(1, s + 1)])
        tris.append([1, at(rings - 1, s + 1), at(rings - 1, s)])
        for r in range(1, rings - 1):
            tris.append([at(r, s), at(r + 1, s), at(r + 1, s + 1)])
            tris.append([at(r, s), at(r + 1, s + 1), at(r, s + 1)])
    p = np.array(pts) + np.array(centre)
    return p[np.array(tris)]


def torus(big, small, n_big, n_small, centre=(0.0, 0.0, 0.0)):
    pts = []
    for i in range(n_big):
        u = 2.0 * math.pi * i / n_big
        for j in range(n_small):
            v = 2.0 * math.pi * j / n_small
            r = big + small * math.cos(v)
            pts.append([r * math.cos(u), r * math.sin(u), small * math.sin(v)])

    def at(i, j):
        return (i % n_big) * n_small + (j % n_small)
    tris = []
    for i in range(n_big):
        for j in range(n_small):
            tris.append([at(i, j), at(i + 1, j), at(i + 1, j + 1)])
            tris.append([at(i, j), at(i + 1, j + 1), at(i, j + 1)])
    p = np.array(pts) + np.array(centre)
    return p[np.array(tris)]
