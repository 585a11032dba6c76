"""Mesh -> grid rasterisation (`sims_field::raster`, crates/sims-field/src/raster.rs, over the
hierarchy of bvh.rs) on the CUDA engine: `fill`, `solid_edges`, `solid_cells`, `sheet_edges` and
`closed`, with the reference's names and argument meaning. Triangles are any array-like of shape
(n, 3, 3) (vertex, coordinate) in f64; the ray casts and the sheet sweep run on the GPU (a `Gpu`
must be given: there is no CPU path), `closed` on the host.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Sequence

import numpy as np

from ._lib import lib
from .fdtd import ERRLEN, FdtdError

_P = C.POINTER


def _tris(triangles) -> np.ndarray:
    t = np.ascontiguousarray(np.asarray(triangles, np.float64).reshape(-1, 3, 3))
    return t


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_P(C.c_double))


def _u8(a: np.ndarray):
    return a.ctypes.data_as(_P(C.c_uint8))


def _check(code: int, err) -> None:
    if code:
        raise FdtdError(err.value.decode(), code)


@dataclass
class Filled:
    """raster.rs:7-11: the samples filled by ray parity (inside) and the thin skins (thin), as
    sorted index arrays."""

    inside: np.ndarray
    thin: np.ndarray


def fill(gpu, triangles, samples: Sequence[Sequence[float]], order: str = "ijk") -> Filled:
    """fill (raster.rs:24-104) on the sample lines `samples` (three sorted lines); indices are
    (i n1 + j) n2 + k for order "ijk" or i + (j + k n1) n0 for "xfast"."""
    t = _tris(triangles)
    s = [np.ascontiguousarray(np.asarray(x, np.float64)) for x in samples]
    total = len(s[0]) * len(s[1]) * len(s[2])
    inside = np.zeros(max(total, 1), np.uint8)
    thin = np.zeros(max(total, 1), np.uint8)
    err = C.create_string_buffer(ERRLEN)
    code = lib().fg_raster_fill(gpu._h, _dp(t), len(t), _dp(s[0]), len(s[0]), _dp(s[1]), len(s[1]), _dp(s[2]),
                                len(s[2]), 0 if order == "ijk" else 1, _u8(inside), _u8(thin), err, ERRLEN)
    _check(code, err)
    return Filled(np.nonzero(inside[:total])[0], np.nonzero(thin[:total])[0])


def _lines(grid):
    return [np.ascontiguousarray(np.asarray(grid.axis(a), np.float64)) for a in range(3)]


def _masks(fn, gpu, triangles, grid) -> List[np.ndarray]:
    t = _tris(triangles)
    x, y, z = _lines(grid)
    nn = len(x) * len(y) * len(z)
    mask = np.zeros(3 * nn, np.uint8)
    err = C.create_string_buffer(ERRLEN)
    code = fn(gpu._h, _dp(t), len(t), _dp(x), len(x), _dp(y), len(y), _dp(z), len(z), _u8(mask), err, ERRLEN)
    _check(code, err)
    return [mask[c * nn:(c + 1) * nn].astype(bool) for c in range(3)]


def solid_edges(gpu, triangles, grid) -> List[np.ndarray]:
    """solid_edges (raster.rs:145-160): per component, the E edges (node index (i ny + j) nz + k)
    whose midpoints the closed mesh holds."""
    return _masks(lib().fg_raster_solid_edges, gpu, triangles, grid)


def sheet_edges(gpu, triangles, grid) -> List[np.ndarray]:
    """sheet_edges (raster.rs:186-264): per component, the E edges the triangles pass through."""
    return _masks(lib().fg_raster_sheet_edges, gpu, triangles, grid)


def solid_cells(gpu, triangles, grid) -> np.ndarray:
    """solid_cells (raster.rs:162-173): the cells ((i (ny-1) + j) (nz-1) + k) whose centres the
    closed mesh holds."""
    t = _tris(triangles)
    x, y, z = _lines(grid)
    n = (len(x) - 1) * (len(y) - 1) * (len(z) - 1)
    mask = np.zeros(max(n, 1), np.uint8)
    err = C.create_string_buffer(ERRLEN)
    code = lib().fg_raster_solid_cells(gpu._h, _dp(t), len(t), _dp(x), len(x), _dp(y), len(y), _dp(z), len(z),
                                       _u8(mask), err, ERRLEN)
    _check(code, err)
    return mask[:n].astype(bool)


def closed(triangles) -> bool:
    """closed (raster.rs:127-143): every edge shared by an even number of triangles."""
    t = _tris(triangles)
    if len(t) == 0:
        return False
    return bool(lib().fg_raster_closed(_dp(t), len(t)))


class GpuRaster:
    """The rasteriser bound to one Gpu, as the antenna workflow calls it."""

    def __init__(self, gpu):
        self.gpu = gpu

    def solid_cells(self, triangles, grid):
        return solid_cells(self.gpu, triangles, grid)

    def solid_edges(self, triangles, grid):
        return solid_edges(self.gpu, triangles, grid)

    def sheet_edges(self, triangles, grid):
        return sheet_edges(self.gpu, triangles, grid)

    def closed(self, triangles) -> bool:
        return closed(triangles)

