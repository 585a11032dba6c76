"""The antenna models of sims-antenna's own tests (crates/sims-antenna/tests/fdtd.rs), restated as
fieldgrid_b200.antenna Models for the tests here: the half-wave dipole (:6-22) and Sheen's
microstrip patch in its box and meshed forms (:88-138)."""
import math

import numpy as np

from fieldgrid_b200 import antenna as A
from meshes import cuboid, plate


def dipole() -> A.Model:
    length, gap = 0.141, 0.003
    return A.Model(metal=[A.Aabb.new((0.0, 0.0, -length / 2), (0.0, 0.0, -gap / 2)),
                          A.Aabb.new((0.0, 0.0, gap / 2), (0.0, 0.0, length / 2))],
                   port=A.Port((0.0, 0.0, -gap / 2), (0.0, 0.0, gap / 2), 50.0), f0=1.0e9, span=0.2, fine=gap)


def sheen(meshed: bool = False) -> A.Model:
    mm = 1e-3
    h = 0.794 * mm
    w, l = 12.45 * mm, 16.0 * mm
    lw, loff = 2.46 * mm, 2.09 * mm
    x0, y0 = -w / 2, -l / 2
    line_x = x0 + loff
    edge_y = y0 - 8.0 * mm
    gx = 30.0 * mm
    top = l / 2 + 7.0 * mm
    sheets = [((-gx / 2, edge_y), (gx / 2, top), 0.0), ((x0, y0), (x0 + w, y0 + l), h),
              ((line_x, edge_y), (line_x + lw, y0), h)]
    board = ((-gx / 2, edge_y, 0.0), (gx / 2, top, h))
    model = A.Model(port=A.Port((line_x + lw / 2, edge_y, 0.0), (line_x + lw / 2, edge_y, h), 50.0),
                    f0=7.5e9, span=0.25, fine=0.4 * mm)
    if meshed:
        for lo, hi, z in sheets:
            model.parts.append(A.Part(plate(lo, hi, z), A.Metal()))
        model.parts.append(A.Part(cuboid(board[0], board[1]), A.DielectricStuff(2.2, 0.0)))
    else:
        for lo, hi, z in sheets:
            model.metal.append(A.Aabb.new((lo[0], lo[1], z), (hi[0], hi[1], z)))
        model.dielectrics.append(A.Dielectric(A.Aabb.new(board[0], board[1]), 2.2, 0.0))
    return model


def radiated(u_of_dirs, nt=60, npp=90):
    """tests/fdtd.rs:24-38: total power and peak intensity on a 60 x 90 midpoint grid."""
    th = (np.arange(nt) + 0.5) / nt * math.pi
    ph = (np.arange(npp) + 0.5) / npp * 2.0 * math.pi
    t, p = np.meshgrid(th, ph, indexing="ij")
    d = np.stack([np.sin(t) * np.cos(p), np.sin(t) * np.sin(p), np.cos(t)], -1).reshape(-1, 3)
    w = (np.sin(t) * (math.pi / nt) * (2.0 * math.pi / npp)).reshape(-1)
    u = u_of_dirs(d)
    return float(np.sum(u * w)), float(u.max())


def resonance(freqs, z) -> float:
    """tests/fdtd.rs:40-43: the first frequency where Im Z crosses from negative to non-negative."""
    for q in range(len(z) - 1):
        if z[q].imag < 0.0 and z[q + 1].imag >= 0.0:
            return float(freqs[q])
    return 0.0


class OracleRaster:
    """The oracle's rasteriser (raster_oracle.cpp) in the shape antenna.setup calls."""

    def solid_cells(self, triangles, grid):
        from oracle import oracle as O
        return O.raster_solid_cells(triangles, grid)

    def solid_edges(self, triangles, grid):
        from oracle import oracle as O
        return O.raster_solid_edges(triangles, grid)

    def sheet_edges(self, triangles, grid):
        from oracle import oracle as O
        return O.raster_sheet_edges(triangles, grid)

    def closed(self, triangles) -> bool:
        from oracle import oracle as O
        return O.raster_closed(triangles)

