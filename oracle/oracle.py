"""TEST INFRASTRUCTURE — Python driver of the oracle (liboracle.so, built from fdtd_oracle.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import this module, as the
checker. It is a CPU restatement of the reference's own CPU FDTD (see fdtd_oracle.hpp); the
product never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass
from typing import Optional

import numpy as np

from fieldgrid_b200 import _abi as A

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None


class OracleError(Exception):
    def __init__(self, message, code=0):
        super().__init__(message)
        self.code = code


def build() -> str:
    """Compiles liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    u64, u32, dbl, vp, cp, sz = C.c_uint64, C.c_uint32, C.c_double, C.c_void_p, C.c_char_p, C.c_size_t
    sig = {
        "fgo_threads": (C.c_int, []),
        "fgo_sim_try_new": (C.c_int, [P(A.fg_sim_spec), C.c_int, P(vp), cp, sz]),
        "fgo_sim_free": (None, [vp]),
        "fgo_sim_dt": (dbl, [vp]),
        "fgo_sim_count": (u64, [vp, cp]),
        "fgo_sim_coefs": (C.c_int, [vp, u32, P(dbl), P(dbl)]),
        "fgo_sim_wires": (C.c_int, [vp, P(u64), P(u64), P(dbl)]),
        "fgo_port_loop": (C.c_int, [vp, u64, u64, u64, P(u64), P(u32), P(dbl), u64, P(u64)]),
        "fgo_coef_sets": (C.c_int, [vp, u64, P(u32), u64, P(C.c_float), u64, P(u64), P(u64), P(C.c_int)]),
        "fgo_run_cpu": (C.c_int, [vp, u64, P(A.fg_pulse), P(A.fg_extras), A.PROGRESS_FN, vp, P(vp), cp, sz]),
        "fgo_record_steps": (u64, [vp]),
        "fgo_record_decay_db": (dbl, [vp]),
        "fgo_record_len": (u64, [vp, cp]),
        "fgo_record_get": (C.c_int, [vp, cp, P(dbl)]),
        "fgo_record_free": (None, [vp]),
        "fgo_patches": (C.c_int, [vp, u64, P(u32), P(dbl), P(dbl), P(u64)]),
        "fgo_far_eval": (C.c_int, [P(dbl), P(dbl), u64, P(C.c_float), u64, u64, dbl, dbl, dbl, P(dbl), u64, P(dbl), P(dbl)]),
        "fgo_far_radiated": (C.c_int, [P(dbl), P(dbl), u64, P(C.c_float), u64, u64, dbl, dbl, dbl, u64, P(dbl), P(dbl)]),
        "fgo_time_steps": (C.c_int, [vp, u64, P(A.fg_pulse), P(A.fg_extras), u64, u64, P(dbl), cp, sz]),
        "fgo_sim_axis": (C.c_int, [vp, u32, P(dbl)]),
        "fgo_sim_list": (C.c_int, [vp, cp, P(u64), P(dbl), P(u64)]),
        "fgo_sim_sheets": (C.c_int, [vp, P(u64), P(dbl), P(u64), P(C.c_float), P(u64)]),
        "fgo_raster_fill": (C.c_int, [P(dbl), u64, P(dbl), u64, P(dbl), u64, P(dbl), u64, P(u64), C.c_int,
                                      P(C.c_uint8), P(C.c_uint8)]),
        "fgo_raster_sheet_edges": (C.c_int, [P(dbl), u64, P(dbl), u64, P(dbl), u64, P(dbl), u64, P(C.c_uint8)]),
        "fgo_raster_closed": (C.c_int, [P(dbl), u64]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def threads() -> int:
    return int(lib().fgo_threads())


class OracleSim:
    """Sim::try_new of the restatement. bits=32 follows the reference's f32 semantics; bits=64
    is the FP64 truth run of the same update."""

    def __init__(self, grid, mats, pec, lumped, ports, resistive, media, bits: int = 32):
        L = lib()
        spec = A.sim_spec(grid, mats, pec, lumped, ports, resistive, media)
        out = C.c_void_p()
        err = C.create_string_buffer(1024)
        code = L.fgo_sim_try_new(C.byref(spec.struct), bits, C.byref(out), err, 1024)
        if code:
            raise OracleError(err.value.decode(), code)
        self._h = out
        self.bits = bits
        self.grid = grid
        self.ports = list(ports or [])

    def __del__(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().fgo_sim_free(self._h)
            self._h = None

    @property
    def dt(self) -> float:
        return lib().fgo_sim_dt(self._h)

    def dims(self):
        return self.grid.dims()

    def count(self, what: str) -> int:
        return int(lib().fgo_sim_count(self._h, what.encode()))

    def coefs(self, comp: int):
        n = self.dims()
        nn = n[0] * n[1] * n[2]
        ca, cb = np.zeros(nn), np.zeros(nn)
        P = C.POINTER(C.c_double)
        lib().fgo_sim_coefs(self._h, comp, ca.ctypes.data_as(P), cb.ctypes.data_as(P))
        return ca, cb

    def wires(self):
        n = self.count("wires")
        h = np.zeros(max(n, 1), np.uint64)
        e = np.zeros(max(4 * n, 1), np.uint64)
        c = np.zeros(max(4 * n, 1), np.float64)
        P = C.POINTER
        lib().fgo_sim_wires(self._h, h.ctypes.data_as(P(C.c_uint64)), e.ctypes.data_as(P(C.c_uint64)),
                            c.ctypes.data_as(P(C.c_double)))
        return h[:n], e[: 4 * n].reshape(n, 4), c[: 4 * n].reshape(n, 4)

    def port_loop(self, port: int, axis: int, k: int):
        P = C.POINTER
        cap = 4096
        ids = np.zeros(cap, np.uint64)
        comps = np.zeros(cap, np.uint32)
        w = np.zeros(cap, np.float64)
        count = C.c_uint64()
        code = lib().fgo_port_loop(self._h, port, axis, k, ids.ctypes.data_as(P(C.c_uint64)),
                                   comps.ctypes.data_as(P(C.c_uint32)), w.ctypes.data_as(P(C.c_double)), cap,
                                   C.byref(count))
        if code:
            raise OracleError("port_loop needs a 32-bit sim")
        n = count.value
        return [(int(ids[q]), int(comps[q]), float(w[q])) for q in range(n)]

    def axis(self, a: int) -> np.ndarray:
        """Sim.ax[a] as an (n, 10) f64 array: inv_d, inv_dd, raw_inv_d, raw_inv_dd, be, ce, bh, ch,
        slot_e, slot_h."""
        n = self.dims()[a]
        out = np.zeros((n, 10))
        lib().fgo_sim_axis(self._h, a, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def items(self, what: str):
        """A sparse list of the Sim: "debye", "sources<p>", "inductors" or "poles", as (idx
        (n, 2) uint64, val (n, 2) f64)."""
        cap = max(self.count("debye_edges"), self.count("inductors"), 64,
                  max((self.count(f"port_src{p}") for p in range(max(len(self.ports), 1))), default=0))
        idx = np.zeros((cap, 2), np.uint64)
        val = np.zeros((cap, 2))
        count = C.c_uint64()
        code = lib().fgo_sim_list(self._h, what.encode(), idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                                  val.ctypes.data_as(C.POINTER(C.c_double)), C.byref(count))
        if code:
            raise OracleError(f"no list {what!r}", code)
        n = count.value
        return idx[:n], val[:n]

    def sheets(self):
        """Sim.sheets as (idx (n, 4) uint64: comp, id, face a, face b; val (n, 4): r, adaptive, len,
        c) and Sim.sheet_table (f32)."""
        L = lib()
        P = C.POINTER
        n, t = C.c_uint64(), C.c_uint64()
        L.fgo_sim_sheets(self._h, C.cast(None, P(C.c_uint64)), C.cast(None, P(C.c_double)), C.byref(n),
                         C.cast(None, P(C.c_float)), C.byref(t))
        idx = np.zeros((max(n.value, 1), 4), np.uint64)
        val = np.zeros((max(n.value, 1), 4))
        table = np.zeros(max(t.value, 1), np.float32)
        L.fgo_sim_sheets(self._h, idx.ctypes.data_as(P(C.c_uint64)), val.ctypes.data_as(P(C.c_double)), C.byref(n),
                         table.ctypes.data_as(P(C.c_float)), C.byref(t))
        return idx[: n.value], val[: n.value], table[: t.value]

    def coef_sets(self, narrow: int):
        L = lib()
        P = C.POINTER
        ni, ns, wide = C.c_uint64(), C.c_uint64(), C.c_int()
        L.fgo_coef_sets(self._h, narrow, C.cast(None, P(C.c_uint32)), 0, C.cast(None, P(C.c_float)), 0,
                        C.byref(ni), C.byref(ns), C.byref(wide))
        index = np.zeros(ni.value, np.uint32)
        sets = np.zeros(2 * ns.value, np.float32)
        L.fgo_coef_sets(self._h, narrow, index.ctypes.data_as(P(C.c_uint32)), ni.value,
                        sets.ctypes.data_as(P(C.c_float)), ns.value, C.byref(ni), C.byref(ns), C.byref(wide))
        return index, sets.reshape(-1, 2), bool(wide.value)


@dataclass
class OracleRecord:
    steps: int
    series: np.ndarray
    decay_db: float
    plane: np.ndarray
    ntff: np.ndarray
    e: Optional[np.ndarray] = None
    h: Optional[np.ndarray] = None


def run_cpu(sim: OracleSim, driven, pulse, extras, progress=None, keep_fields=False) -> OracleRecord:
    """run_cpu (cpu.rs:424-482). Arrays come back as float64 (f32 results widen exactly)."""
    L = lib()
    xs = A.extras_struct(extras, keep_fields)
    pl = A.pulse_struct(pulse)

    def cb(_u, steps, decay):
        return 1 if (progress is None or progress(int(steps), float(decay))) else 0

    cfn = A.PROGRESS_FN(cb)
    out = C.c_void_p()
    err = C.create_string_buffer(1024)
    code = L.fgo_run_cpu(sim._h, driven, C.byref(pl), C.byref(xs.struct), cfn, None, C.byref(out), err, 1024)
    if code:
        raise OracleError(err.value.decode(), code)
    try:
        def get(which):
            n = L.fgo_record_len(out, which.encode())
            a = np.zeros(max(n, 1), np.float64)
            L.fgo_record_get(out, which.encode(), a.ctypes.data_as(C.POINTER(C.c_double)))
            return a[:n]

        rec = OracleRecord(int(L.fgo_record_steps(out)), get("series"), float(L.fgo_record_decay_db(out)),
                           get("plane"), get("ntff"))
        if keep_fields:
            rec.e, rec.h = get("e"), get("h")
        return rec
    finally:
        L.fgo_record_free(out)


def patches(sim: OracleSim, inset: int):
    L = lib()
    P = C.POINTER
    count = C.c_uint64()
    L.fgo_patches(sim._h, inset, C.cast(None, P(C.c_uint32)), C.cast(None, P(C.c_double)),
                  C.cast(None, P(C.c_double)), C.byref(count))
    n = count.value
    gpu = np.zeros(max(13 * n, 1), np.uint32)
    pos = np.zeros(max(3 * n, 1))
    area = np.zeros(max(n, 1))
    L.fgo_patches(sim._h, inset, gpu.ctypes.data_as(P(C.c_uint32)), pos.ctypes.data_as(P(C.c_double)),
                  area.ctypes.data_as(P(C.c_double)), C.byref(count))
    return pos[: 3 * n].reshape(n, 3), area[:n], gpu[: 13 * n]


def far_eval(pos, area, acc, nf, k, freq, dirs, scale=(1.0, 0.0)):
    """Far::load then Far::field and Far::intensity per direction (ntff.rs:77-120)."""
    P = C.POINTER
    pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
    area = np.ascontiguousarray(area, np.float64)
    acc = np.ascontiguousarray(acc, np.float32)
    dirs = np.ascontiguousarray(np.asarray(dirs, np.float64).reshape(-1, 3))
    field = np.zeros((dirs.shape[0], 6))
    inten = np.zeros(dirs.shape[0])
    lib().fgo_far_eval(pos.ctypes.data_as(P(C.c_double)), area.ctypes.data_as(P(C.c_double)), area.size,
                       acc.ctypes.data_as(P(C.c_float)), nf, k, freq, scale[0], scale[1],
                       dirs.ctypes.data_as(P(C.c_double)), dirs.shape[0], field.ctypes.data_as(P(C.c_double)),
                       inten.ctypes.data_as(P(C.c_double)))
    return field[:, 0::2] + 1j * field[:, 1::2], inten


def far_radiated(pos, area, acc, nf, k, freq, steps, scale=(1.0, 0.0)):
    P = C.POINTER
    pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
    area = np.ascontiguousarray(area, np.float64)
    acc = np.ascontiguousarray(acc, np.float32)
    t, p = C.c_double(), C.c_double()
    lib().fgo_far_radiated(pos.ctypes.data_as(P(C.c_double)), area.ctypes.data_as(P(C.c_double)), area.size,
                           acc.ctypes.data_as(P(C.c_float)), nf, k, freq, scale[0], scale[1], steps, C.byref(t),
                           C.byref(p))
    return t.value, p.value


def time_steps(sim: OracleSim, driven, pulse, extras, warmup: int, steps: int) -> float:
    """Seconds for `steps` State::step calls after `warmup` untimed ones (the CPU baseline)."""
    xs = A.extras_struct(extras)
    pl = A.pulse_struct(pulse)
    sec = C.c_double()
    err = C.create_string_buffer(1024)
    code = lib().fgo_time_steps(sim._h, driven, C.byref(pl), C.byref(xs.struct), warmup, steps, C.byref(sec), err, 1024)
    if code:
        raise OracleError(err.value.decode(), code)
    return sec.value


# ---- the rasteriser (raster.rs, bvh.rs) ---------------------------------------------------------

def _tris(triangles):
    return np.ascontiguousarray(np.asarray(triangles, np.float64).reshape(-1, 3, 3))


def raster_fill(triangles, samples, dims=None, order: int = 0):
    """fill (raster.rs:24-104): (inside, thin) byte masks over the index space dims (default: the
    sample counts), order 0 = (i m1 + j) m2 + k, 1 = i + (j + k m1) m0."""
    P = C.POINTER
    t = _tris(triangles)
    s = [np.ascontiguousarray(np.asarray(x, np.float64)) for x in samples]
    m = np.array(dims if dims is not None else [len(x) for x in s], np.uint64)
    total = int(np.prod(m))
    inside = np.zeros(max(total, 1), np.uint8)
    thin = np.zeros(max(total, 1), np.uint8)
    dp = lambda a: a.ctypes.data_as(P(C.c_double))
    lib().fgo_raster_fill(dp(t), len(t), dp(s[0]), len(s[0]), dp(s[1]), len(s[1]), dp(s[2]), len(s[2]),
                          m.ctypes.data_as(P(C.c_uint64)), order, inside.ctypes.data_as(P(C.c_uint8)),
                          thin.ctypes.data_as(P(C.c_uint8)))
    return inside[:total], thin[:total]


def _centres(line):
    line = np.asarray(line, np.float64)
    return 0.5 * (line[:-1] + line[1:])


def raster_solid_edges(triangles, grid):
    """solid_edges (raster.rs:145-160): per component, fill with centres along it."""
    n = grid.dims()
    out = []
    for c in range(3):
        s = [grid.axis(a) if a != c else _centres(grid.axis(a)) for a in range(3)]
        inside, thin = raster_fill(triangles, s, n, 0)
        out.append((inside | thin).astype(bool))
    return out


def raster_solid_cells(triangles, grid):
    """solid_cells (raster.rs:162-173)."""
    s = [_centres(grid.axis(a)) for a in range(3)]
    inside, thin = raster_fill(triangles, s, None, 0)
    return (inside | thin).astype(bool)


def raster_sheet_edges(triangles, grid):
    """sheet_edges (raster.rs:186-264)."""
    P = C.POINTER
    t = _tris(triangles)
    x, y, z = [np.ascontiguousarray(np.asarray(grid.axis(a), np.float64)) for a in range(3)]
    nn = len(x) * len(y) * len(z)
    mask = np.zeros(3 * nn, np.uint8)
    dp = lambda a: a.ctypes.data_as(P(C.c_double))
    lib().fgo_raster_sheet_edges(dp(t), len(t), dp(x), len(x), dp(y), len(y), dp(z), len(z),
                                 mask.ctypes.data_as(P(C.c_uint8)))
    return [mask[c * nn:(c + 1) * nn].astype(bool) for c in range(3)]


def raster_closed(triangles) -> bool:
    """closed (raster.rs:127-143)."""
    t = _tris(triangles)
    return bool(lib().fgo_raster_closed(t.ctypes.data_as(C.POINTER(C.c_double)), len(t)))

