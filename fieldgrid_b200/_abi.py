"""ctypes mirrors of the structs in include/fieldgrid.h and the marshalling of Python setup
objects into them.

This module loads no shared library. The product wrapper (fieldgrid_b200.fdtd) and the test
oracle wrapper both fill these structs, so one scenario description drives both.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

FG_OK = 0
FG_ERR_INVALID = 1
FG_ERR_SETUP = 2
FG_ERR_NO_DEVICE = 3
FG_ERR_TOO_LARGE = 4
FG_ERR_PORT_INDEX = 5
FG_ERR_UNSTABLE = 6
FG_ERR_CANCELLED = 7
FG_ERR_CUDA = 8
FG_ERR_UNSUPPORTED = 9

u64 = C.c_uint64
u32 = C.c_uint32
i32 = C.c_int32
dbl = C.c_double
P = C.POINTER


class fg_edge(C.Structure):
    _fields_ = [("comp", u32), ("reserved", u32), ("at", u64 * 3)]


class fg_lumped(C.Structure):
    _fields_ = [("name", C.c_char_p), ("edges", P(fg_edge)), ("n_edges", u64),
                ("element", i32), ("reserved", i32), ("value", dbl)]


class fg_port(C.Structure):
    _fields_ = [("name", C.c_char_p), ("edges", P(fg_edge)), ("column_len", P(u64)),
                ("n_columns", u64), ("r", dbl), ("reference_above", i32), ("reserved", i32)]


class fg_resistive(C.Structure):
    _fields_ = [("comp", u32), ("adaptive", i32), ("id", u64), ("r", dbl), ("faces", u64 * 2)]


class fg_wire(C.Structure):
    _fields_ = [("edge", fg_edge), ("radius", dbl)]


PEC_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, u32, P(u64))


class fg_sim_spec(C.Structure):
    _fields_ = [
        ("x", P(dbl)), ("nx", u64), ("y", P(dbl)), ("ny", u64), ("z", P(dbl)), ("nz", u64),
        ("pml", u64),
        ("eps", P(C.c_float)), ("sigma", P(C.c_float)), ("inf", P(C.c_float)), ("debye", P(C.c_float)),
        ("pec_mask", P(C.c_uint8)), ("pec_fn", PEC_FN), ("pec_user", C.c_void_p),
        ("lumped", P(fg_lumped)), ("n_lumped", u64),
        ("ports", P(fg_port)), ("n_ports", u64),
        ("resistive", P(fg_resistive)), ("n_resistive", u64),
        ("sheet_table", P(C.c_float)), ("sheet_table_len", u64), ("sheet_states", u64),
        ("debye_poles", P(dbl)), ("n_debye_poles", u64),
        ("wires", P(fg_wire)), ("n_wires", u64),
    ]


class fg_pulse(C.Structure):
    _fields_ = [("f0", dbl), ("fc", dbl)]


class fg_extras(C.Structure):
    _fields_ = [
        ("min_steps", u64), ("max_steps", u64), ("decay_db", dbl),
        ("freqs", P(dbl)), ("n_freqs", u64),
        ("has_plane_k", i32), ("fused_e", i32), ("plane_k", u64),
        ("ntff", P(u32)), ("ntff_len", u64),
        ("check_every", u64),
        ("profile", i32), ("keep_fields", i32),
    ]


PROGRESS_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, u64, dbl)


class fg_flux_spec(C.Structure):
    _fields_ = [("design_lo", C.c_uint64 * 3), ("design_hi", C.c_uint64 * 3), ("plane_k", C.c_uint64),
                ("window_lo", C.c_uint64 * 2), ("window_hi", C.c_uint64 * 2), ("freq", C.c_double),
                ("steps", C.c_uint64), ("checkpoints", C.c_uint64), ("precision", C.c_int32), ("transposes", C.c_int32)]


class fg_flux_result(C.Structure):
    _fields_ = [("objective", C.c_double), ("flux_re", C.c_double), ("flux_im", C.c_double),
                ("forward_ms", C.c_double), ("recompute_ms", C.c_double), ("adjoint_ms", C.c_double),
                ("backward_ms", C.c_double), ("setup_ms", C.c_double),
                ("segments", C.c_uint64), ("segment_len", C.c_uint64), ("design_edges", C.c_uint64)]


class fg_batch_options(C.Structure):
    _fields_ = [("tune", C.c_int), ("tile", C.c_int), ("blocks_per_sm", C.c_int), ("seg", C.c_int),
                ("graph_steps", C.c_int)]


def _ptr(arr: np.ndarray | None, ctype):
    if arr is None:
        return C.cast(None, P(ctype))
    return arr.ctypes.data_as(P(ctype))


def _edge(e) -> fg_edge:
    out = fg_edge()
    out.comp = int(e.comp)
    out.at[0], out.at[1], out.at[2] = (int(v) for v in e.at)
    return out


class Marshalled:
    """Holds a filled struct plus every buffer it points into (kept alive with it)."""

    def __init__(self, struct, keep):
        self.struct = struct
        self._keep = keep


def pec_mask(pec, dims) -> np.ndarray | None:
    """The pec(comp, at) closure of Sim::try_new (sim.rs:355) as a 3*nn byte mask.

    Accepts None, a boolean array of shape (3, n0, n1, n2), or a callable f(c, (i, j, k)).
    A callable is first tried on index arrays (numpy broadcasting); if that does not give a
    full-shape boolean array it is evaluated edge by edge.
    """
    n0, n1, n2 = (int(v) for v in dims)
    if pec is None:
        return None
    if isinstance(pec, np.ndarray):
        m = np.ascontiguousarray(pec, dtype=np.uint8).reshape(3 * n0 * n1 * n2)
        return m
    mask = np.zeros((3, n0, n1, n2), dtype=np.uint8)
    ii, jj, kk = np.meshgrid(np.arange(n0), np.arange(n1), np.arange(n2), indexing="ij")
    try:
        for c in range(3):
            r = pec(c, (ii, jj, kk))
            r = np.broadcast_to(np.asarray(r, dtype=bool), (n0, n1, n2))
            mask[c] = r
        return mask.reshape(-1)
    except (ValueError, TypeError):
        pass
    for c in range(3):
        for i in range(n0):
            for j in range(n1):
                for k in range(n2):
                    if pec(c, (i, j, k)):
                        mask[c, i, j, k] = 1
    return mask.reshape(-1)


def sim_spec(grid, mats, pec, lumped, ports, resistive, media) -> Marshalled:
    """Fills fg_sim_spec from the Python mirror objects of Sim::try_new's arguments."""
    keep = []
    s = fg_sim_spec()
    for name in ("x", "y", "z"):
        line = np.ascontiguousarray(getattr(grid, name), dtype=np.float64)
        keep.append(line)
        setattr(s, name, _ptr(line, dbl))
        setattr(s, "n" + name, line.size)
    s.pml = int(grid.pml)
    for name in ("eps", "sigma", "inf", "debye"):
        arr = None if mats is None else getattr(mats, name, None)
        if arr is not None:
            arr = np.ascontiguousarray(arr, dtype=np.float32).reshape(-1)
            if arr.size != grid.cells():
                raise ValueError(f"materials.{name} has {arr.size} values for {grid.cells()} cells")
            keep.append(arr)
        setattr(s, name, _ptr(arr, C.c_float))
    mask = pec_mask(pec, grid.dims())
    if mask is not None:
        keep.append(mask)
    s.pec_mask = _ptr(mask, C.c_uint8)
    s.pec_fn = PEC_FN()
    s.pec_user = None

    lumped = list(lumped or [])
    la = (fg_lumped * max(len(lumped), 1))()
    for q, l in enumerate(lumped):
        ea = (fg_edge * max(len(l.edges), 1))(*[_edge(e) for e in l.edges])
        keep.append(ea)
        name = l.name.encode()
        keep.append(name)
        la[q].name = name
        la[q].edges = C.cast(ea, P(fg_edge))
        la[q].n_edges = len(l.edges)
        la[q].element = int(l.element.kind)
        la[q].value = float(l.element.value)
    keep.append(la)
    s.lumped, s.n_lumped = C.cast(la, P(fg_lumped)), len(lumped)

    ports = list(ports or [])
    pa = (fg_port * max(len(ports), 1))()
    for q, p in enumerate(ports):
        flat = [e for col in p.columns for e in col]
        ea = (fg_edge * max(len(flat), 1))(*[_edge(e) for e in flat])
        ca = (u64 * max(len(p.columns), 1))(*[len(col) for col in p.columns])
        name = p.name.encode()
        keep.extend([ea, ca, name])
        pa[q].name = name
        pa[q].edges = C.cast(ea, P(fg_edge))
        pa[q].column_len = C.cast(ca, P(u64))
        pa[q].n_columns = len(p.columns)
        pa[q].r = float(p.r)
        pa[q].reference_above = 1 if p.reference_above else 0
    keep.append(pa)
    s.ports, s.n_ports = C.cast(pa, P(fg_port)), len(ports)

    resistive = list(resistive or [])
    ra = (fg_resistive * max(len(resistive), 1))()
    for q, r in enumerate(resistive):
        ra[q].comp = int(r.comp)
        ra[q].adaptive = 1 if r.adaptive else 0
        ra[q].id = int(r.id)
        ra[q].r = float(r.r)
        ra[q].faces[0], ra[q].faces[1] = int(r.faces[0]), int(r.faces[1])
    keep.append(ra)
    s.resistive, s.n_resistive = C.cast(ra, P(fg_resistive)), len(resistive)

    if media is not None and media.sheets is not None:
        table = np.ascontiguousarray(media.sheets.table, dtype=np.float32)
        keep.append(table)
        s.sheet_table, s.sheet_table_len, s.sheet_states = _ptr(table, C.c_float), table.size, int(media.sheets.states)
    else:
        s.sheet_table, s.sheet_table_len, s.sheet_states = _ptr(None, C.c_float), 0, 0
    poles = [] if media is None or media.debye is None else list(media.debye.poles)
    pl = np.ascontiguousarray(np.array(poles, dtype=np.float64).reshape(-1))
    keep.append(pl)
    s.debye_poles, s.n_debye_poles = _ptr(pl, dbl), len(poles)
    wires = [] if media is None else list(media.wires)
    wa = (fg_wire * max(len(wires), 1))()
    for q, (e, radius) in enumerate(wires):
        wa[q].edge = _edge(e)
        wa[q].radius = float(radius)
    keep.append(wa)
    s.wires, s.n_wires = C.cast(wa, P(fg_wire)), len(wires)
    return Marshalled(s, keep)


def extras_struct(extras, keep_fields: bool = False) -> Marshalled:
    keep = []
    x = fg_extras()
    x.min_steps = int(extras.min_steps)
    x.max_steps = int(extras.max_steps)
    x.decay_db = float(extras.decay_db)
    freqs = np.ascontiguousarray(np.array(list(extras.freqs), dtype=np.float64))
    keep.append(freqs)
    x.freqs, x.n_freqs = _ptr(freqs, dbl), freqs.size
    x.has_plane_k = 0 if extras.plane_k is None else 1
    x.plane_k = 0 if extras.plane_k is None else int(extras.plane_k)
    x.fused_e = 1 if extras.fused_e else 0
    if extras.ntff is None:
        x.ntff, x.ntff_len = _ptr(None, u32), 0
    else:
        nt = np.ascontiguousarray(np.asarray(extras.ntff, dtype=np.uint32))
        keep.append(nt)
        if nt.size == 0:
            # Some(vec![]) is still Some: point at a one-element buffer with length 0
            nt = np.zeros(1, dtype=np.uint32)
            keep.append(nt)
            x.ntff, x.ntff_len = _ptr(nt, u32), 0
        else:
            x.ntff, x.ntff_len = _ptr(nt, u32), nt.size
    x.check_every = int(extras.check_every)
    x.profile = 1 if extras.profile else 0
    x.keep_fields = 1 if keep_fields else 0
    return Marshalled(x, keep)


def pulse_struct(pulse) -> fg_pulse:
    p = fg_pulse()
    p.f0, p.fc = float(pulse.f0), float(pulse.fc)
    return p
