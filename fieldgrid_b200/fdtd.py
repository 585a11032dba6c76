"""The Yee-grid FDTD solve with the API of `sims_field::fdtd` (crates/sims-field/src/fdtd/mod.rs).

Names, argument meanings and error texts follow the reference: `Sim.try_new` is Sim::try_new
(sim.rs:352), `run(g, sim, driven, pulse, extras, progress)` is run / run_blocking
(run.rs:379-397), `patches` and `Far` are ntff.rs. Setup (Sim.try_new) runs in the engine's C++
host code, the time stepping runs in its CUDA kernels; both are reached through the C ABI of
include/fieldgrid.h. Errors the reference returns as `Err(String)` raise FdtdError with the
same text. There is no CPU path: `run(None, ...)` raises, as does a missing CUDA device.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

from . import _abi as A
from ._lib import lib
from .grid import Grid

C0 = 299_792_458.0
EPS0 = 8.854_187_812_8e-12
MU0 = 1.256_637_062_12e-6
ETA0 = 376.730_313_668

ERRLEN = 1024


class FdtdError(Exception):
    """An `Err(String)` of the reference; str(e) is its text."""

    def __init__(self, message: str, code: int = 0):
        super().__init__(message)
        self.code = code


def idx(n, i, j, k):
    """sim.rs:8-10."""
    return (i * n[1] + j) * n[2] + k


def unidx(n, id_):
    """sim.rs:642-644."""
    return (id_ // (n[1] * n[2]), (id_ // n[2]) % n[1], id_ % n[2])


def psi_len(n, axis, pml):
    """sim.rs:139-143."""
    if pml == 0:
        return 0
    m = list(n)
    m[axis] = 2 * pml
    return m[0] * m[1] * m[2]


def psi_idx(n, axis, pml, p, slot):
    """sim.rs:659-665."""
    if axis == 0:
        return (slot * n[1] + p[1]) * n[2] + p[2]
    if axis == 1:
        return (p[0] * 2 * pml + slot) * n[2] + p[2]
    return (p[0] * n[1] + p[1]) * 2 * pml + slot


def time_step(grid: Grid) -> float:
    """sim.rs:133-137, evaluated by the engine's host code."""
    L = lib()
    xs = [np.ascontiguousarray(grid.axis(a), dtype=np.float64) for a in range(3)]
    P = C.POINTER(C.c_double)
    return L.fg_time_step(*[v for a in xs for v in (a.ctypes.data_as(P), a.size)])


def pulse_shape(fc: float):
    """(t0, tau) of the Gaussian pulse, sim.rs:646-649."""
    tau = math.sqrt(math.log(10.0)) / (math.pi * fc)
    return 4.0 * tau, tau


def gaussian(f0: float, fc: float) -> Callable[[float], float]:
    """sim.rs:651-657."""
    t0, tau = pulse_shape(fc)

    def g(t: float) -> float:
        x = (t - t0) / tau
        return math.exp(-x * x) * math.cos(2.0 * math.pi * f0 * (t - t0))

    return g


@dataclass
class Edge:
    """sim.rs:145-149."""

    comp: int
    at: tuple


@dataclass
class Element:
    """sim.rs:151-156: use Element.Resistor(r), .Capacitor(c), .Inductor(l)."""

    kind: int
    value: float

    @staticmethod
    def Resistor(r: float) -> "Element":
        return Element(0, r)

    @staticmethod
    def Capacitor(c: float) -> "Element":
        return Element(1, c)

    @staticmethod
    def Inductor(l: float) -> "Element":
        return Element(2, l)


@dataclass
class Lumped:
    """sim.rs:158-163."""

    name: str
    edges: list
    element: Element


@dataclass
class PortDef:
    """sim.rs:165-171."""

    name: str
    columns: list
    r: float
    reference_above: bool = False


@dataclass
class Resistive:
    """sim.rs:208-215."""

    comp: int
    id: int
    r: float
    adaptive: bool
    faces: tuple = (0, 0)


class Materials:
    """Per-cell eps, sigma, eps_inf and Debye weight (sim.rs:217-222, :285-301)."""

    def __init__(self, eps, sigma, inf, debye):
        self.eps = np.asarray(eps, dtype=np.float32).reshape(-1)
        self.sigma = np.asarray(sigma, dtype=np.float32).reshape(-1)
        self.inf = np.asarray(inf, dtype=np.float32).reshape(-1)
        self.debye = np.asarray(debye, dtype=np.float32).reshape(-1)

    @staticmethod
    def new(grid: Grid) -> "Materials":
        c = grid.cells()
        return Materials(np.ones(c, np.float32), np.zeros(c, np.float32), np.ones(c, np.float32),
                         np.zeros(c, np.float32))


@dataclass
class Sheets:
    """sim.rs:224-234: the branch table of resistive sheets and the states per sheet edge."""

    table: list = field(default_factory=lambda: [0.0] * 4)
    states: int = 0


@dataclass
class Debye:
    """One global set of Debye poles (x, a) with per-cell weights (sim.rs:243-283)."""

    poles: list = field(default_factory=list)

    @staticmethod
    def band(f_lo: float, f_hi: float) -> "Debye":
        x0, x1 = 2.0 * math.pi * f_lo / 30.0, 2.0 * math.pi * f_hi * 30.0
        span = math.log(x1 / x0)
        n = int(max(math.ceil(span / 0.7), 1.0))
        h = span / n
        poles = []
        for k in range(n + 1):
            w = 0.5 * h if k == 0 or k == n else h
            poles.append((x0 * math.exp(k * h), w / span))
        return Debye(poles)

    def response(self, w: float):
        re = im = 0.0
        for x, a in self.poles:
            r = w / x
            re += a / (1.0 + r * r)
            im += a * r / (1.0 + r * r)
        return re, im

    def fit(self, er: float, tan: float, f: float):
        if tan <= 0.0 or not self.poles:
            return er, 0.0
        s1, s2 = self.response(2.0 * math.pi * f)
        delta = er * tan / s2
        return er - delta * s1, delta


@dataclass
class Media:
    """sim.rs:236-241."""

    sheets: Sheets = field(default_factory=Sheets)
    debye: Debye = field(default_factory=Debye)
    wires: list = field(default_factory=list)


def _check(code: int, err) -> None:
    if code != A.FG_OK:
        msg = err.value.decode() if hasattr(err, "value") else str(err)
        raise FdtdError(msg, code)


class Sim:
    """sims_field::fdtd::Sim (sim.rs:173-189): the coefficients and element lists of one grid,
    built and owned by the engine's host code. Construct it with Sim.try_new / Sim.new."""

    def __init__(self, handle, grid: Grid, ports):
        self._h = handle
        self.grid = grid
        self.ports = list(ports)
        self.pml = grid.pml

    @staticmethod
    def try_new(grid: Grid, mats: Optional[Materials], pec, lumped, ports, resistive, media: Media) -> "Sim":
        """Sim::try_new (sim.rs:352-554). `pec` is None, a (3, n0, n1, n2) bool array or a callable
        pec(comp, (i, j, k)). Raises FdtdError with the reference's text on refusal."""
        L = lib()
        spec = A.sim_spec(grid, mats, pec, lumped, ports, resistive, media)
        out = C.c_void_p()
        err = C.create_string_buffer(ERRLEN)
        _check(L.fg_sim_try_new(C.byref(spec.struct), C.byref(out), err, ERRLEN), err)
        return Sim(out, grid, ports)

    @staticmethod
    def new(grid, mats, pec, lumped, ports, resistive, media) -> "Sim":
        """Sim::new: try_new that raises (the reference panics) on refusal."""
        return Sim.try_new(grid, mats, pec, lumped, ports, resistive, media)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().fg_sim_free(h)
            except Exception:
                pass
            self._h = None

    @property
    def dt(self) -> float:
        return lib().fg_sim_dt(self._h)

    def dims(self):
        n = (C.c_uint64 * 3)()
        lib().fg_sim_dims(self._h, n)
        return (int(n[0]), int(n[1]), int(n[2]))

    def count(self, what: str) -> int:
        """Lengths of port_src[p] ("port_src{p}"), inductors, sheets, debye_edges, wires, ports."""
        return int(lib().fg_sim_count(self._h, what.encode()))

    @property
    def wires(self) -> np.ndarray:
        """Sim.wires as rows of 9 u32: h, then (e, f32 coefficient bits) x 4."""
        n = self.count("wires")
        out = np.zeros(max(n, 1) * 9, dtype=np.uint32)
        lib().fg_sim_wires(self._h, out.ctypes.data_as(C.POINTER(C.c_uint32)), out.size)
        return out[: n * 9].reshape(n, 9)

    def coefs(self, comp: int):
        """(Sim.ca[comp], Sim.cb[comp]) as float32 arrays of nn."""
        n = self.dims()
        nn = n[0] * n[1] * n[2]
        ca = np.zeros(nn, np.float32)
        cb = np.zeros(nn, np.float32)
        P = C.POINTER(C.c_float)
        _check(lib().fg_sim_coefs(self._h, comp, ca.ctypes.data_as(P), cb.ctypes.data_as(P)), "bad component")
        return ca, cb

    def coef_classes(self) -> int:
        return int(lib().fg_sim_coef_classes(self._h))


@dataclass
class Pulse:
    """run.rs:47-50."""

    f0: float
    fc: float


@dataclass
class Extras:
    """run.rs:34-45."""

    min_steps: int = 0
    max_steps: int = 0
    decay_db: float = 0.0
    freqs: list = field(default_factory=list)
    plane_k: Optional[int] = None
    ntff: Optional[np.ndarray] = None
    fused_e: bool = False
    check_every: int = 0
    profile: bool = False


@dataclass
class Record:
    """run.rs:52-59; `e`/`h` hold the final fields when run(..., keep_fields=True)."""

    steps: int
    ports: int
    series: np.ndarray
    decay_db: float
    plane: np.ndarray
    ntff: np.ndarray
    e: Optional[np.ndarray] = None
    h: Optional[np.ndarray] = None
    h2d: int = 0
    d2h: int = 0


def _copy(ptr, n) -> np.ndarray:
    if not ptr or n == 0:
        return np.zeros(0, np.float32)
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy()


def run(g, sim: Sim, driven: int, pulse: Pulse, extras: Extras,
        progress: Optional[Callable[[int, float], bool]] = None, keep_fields: bool = False) -> Record:
    """run / run_blocking (run.rs:379-397) on the CUDA engine. `g` is a fieldgrid_b200.gpu.Gpu;
    None is the Option<&Gpu> `None` and raises: this engine has no CPU path."""
    L = lib()
    xs = A.extras_struct(extras, keep_fields)
    pl = A.pulse_struct(pulse)
    exc = []

    def cb(_user, steps, decay):
        try:
            return 1 if (progress is None or progress(int(steps), float(decay))) else 0
        except BaseException as e:  # a Python error cancels the run and is re-raised
            exc.append(e)
            return 0

    cfn = A.PROGRESS_FN(cb)
    out = C.c_void_p()
    err = C.create_string_buffer(ERRLEN)
    gh = None if g is None else g._h
    code = L.fg_run(gh, sim._h, driven, C.byref(pl), C.byref(xs.struct), cfn, None, C.byref(out), err, ERRLEN)
    if exc:
        raise exc[0]
    _check(code, err)
    try:
        n = C.c_uint64()
        rec = Record(
            steps=int(L.fg_record_steps(out)),
            ports=int(L.fg_record_ports(out)),
            series=_copy(L.fg_record_series(out, C.byref(n)), n.value),
            decay_db=float(L.fg_record_decay_db(out)),
            plane=_copy(L.fg_record_plane(out, C.byref(n)), n.value),
            ntff=_copy(L.fg_record_ntff(out, C.byref(n)), n.value),
        )
        if keep_fields:
            rec.e = _copy(L.fg_record_e(out, C.byref(n)), n.value)
            rec.h = _copy(L.fg_record_h(out, C.byref(n)), n.value)
        a, b = C.c_uint64(), C.c_uint64()
        L.fg_record_transfer(out, C.byref(a), C.byref(b))
        rec.h2d, rec.d2h = int(a.value), int(b.value)
        return rec
    finally:
        L.fg_record_free(out)


run_blocking = run


class Session:
    """A run's buffers kept in HBM and stepped explicitly (fg_session_*)."""

    def __init__(self, g, sim: Sim, driven: int, pulse: Pulse, extras: Extras):
        L = lib()
        self._xs = A.extras_struct(extras)
        self._pl = A.pulse_struct(pulse)
        out = C.c_void_p()
        err = C.create_string_buffer(ERRLEN)
        _check(L.fg_session_new(None if g is None else g._h, sim._h, driven, C.byref(self._pl),
                                C.byref(self._xs.struct), C.byref(out), err, ERRLEN), err)
        self._h = out
        self.dims = sim.dims()

    def step(self, k: int) -> None:
        code = lib().fg_session_step(self._h, k)
        if code:
            raise FdtdError(lib().fg_last_error().decode(), code)

    def sync(self) -> None:
        code = lib().fg_session_sync(self._h)
        if code:
            raise FdtdError(lib().fg_last_error().decode(), code)

    def energy(self) -> float:
        v = C.c_double()
        code = lib().fg_session_energy(self._h, C.byref(v))
        if code:
            raise FdtdError(lib().fg_last_error().decode(), code)
        return v.value

    @property
    def steps(self) -> int:
        return int(lib().fg_session_steps(self._h))

    def read(self, which: str, n: int) -> np.ndarray:
        out = np.zeros(max(n, 1), np.float32)
        code = lib().fg_session_read(self._h, which.encode(), out.ctypes.data_as(C.POINTER(C.c_float)), n)
        if code:
            raise FdtdError(lib().fg_last_error().decode(), code)
        return out[:n]

    def kernel_times(self, steps: int) -> dict:
        """Mean device ms per launch of each kernel of a step, over `steps` steps launched one
        kernel at a time (the steps count as steps of the run)."""
        cap = 32
        names = C.create_string_buffer(64 * cap)
        ms = (C.c_double * cap)()
        count = C.c_uint64()
        code = lib().fg_session_kernel_times(self._h, steps, names, ms, cap, C.byref(count))
        if code:
            raise FdtdError(lib().fg_last_error().decode(), code)
        out = {}
        for q in range(min(count.value, cap)):
            name = names.raw[64 * q:64 * (q + 1)].split(b"\0", 1)[0].decode()
            out[name] = float(ms[q])
        return out

    @property
    def stream(self) -> int:
        return int(lib().fg_session_stream(self._h) or 0)

    @property
    def launches_per_step(self) -> int:
        return int(lib().fg_session_launches_per_step(self._h))

    @property
    def device_bytes(self) -> int:
        return int(lib().fg_session_device_bytes(self._h))

    @property
    def variant(self) -> str:
        return lib().fg_session_variant(self._h).decode()

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().fg_session_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class Patches:
    """ntff.rs:4-9."""

    pos: np.ndarray
    area: np.ndarray
    gpu: np.ndarray


def patches(sim: Sim, inset: int) -> Patches:
    """ntff.rs:11-59: the near-to-far-field box `inset` cells inside the CPML."""
    L = lib()
    count = C.c_uint64()
    P = C.POINTER
    L.fg_patches(sim._h, inset, C.cast(None, P(C.c_uint32)), C.cast(None, P(C.c_double)),
                 C.cast(None, P(C.c_double)), C.byref(count))
    n = count.value
    gpu = np.zeros(max(13 * n, 1), np.uint32)
    pos = np.zeros(max(3 * n, 1), np.float64)
    area = np.zeros(max(n, 1), np.float64)
    L.fg_patches(sim._h, inset, gpu.ctypes.data_as(P(C.c_uint32)), pos.ctypes.data_as(P(C.c_double)),
                 area.ctypes.data_as(P(C.c_double)), C.byref(count))
    return Patches(pos[: 3 * n].reshape(n, 3), area[:n], gpu[: 13 * n])


class Far:
    """ntff.rs:67-137: far fields from a record's NTFF accumulators. With a Gpu the direction
    sums run on the device."""

    def __init__(self, handle, gpu=None):
        self._h = handle
        self.gpu = gpu

    @staticmethod
    def load(p: Patches, acc, nf: int, k: int, freq: float, scale=(1.0, 0.0), gpu=None) -> "Far":
        L = lib()
        P = C.POINTER
        pos = np.ascontiguousarray(p.pos, dtype=np.float64).reshape(-1)
        area = np.ascontiguousarray(p.area, dtype=np.float64)
        acc = np.ascontiguousarray(acc, dtype=np.float32)
        out = C.c_void_p()
        _check(L.fg_far_load(pos.ctypes.data_as(P(C.c_double)), area.ctypes.data_as(P(C.c_double)), area.size,
                             acc.ctypes.data_as(P(C.c_float)), nf, k, freq, float(scale[0]), float(scale[1]),
                             C.byref(out)), "bad far-field input")
        return Far(out, gpu)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().fg_far_free(h)
            except Exception:
                pass

    def fields(self, dirs) -> np.ndarray:
        """Far::field for many directions: complex array (n, 3)."""
        d = np.ascontiguousarray(np.asarray(dirs, dtype=np.float64).reshape(-1, 3))
        out = np.zeros((d.shape[0], 6), np.float64)
        P = C.POINTER(C.c_double)
        code = lib().fg_far_field(None if self.gpu is None else self.gpu._h, self._h, d.ctypes.data_as(P),
                                  d.shape[0], out.ctypes.data_as(P))
        if code:
            raise FdtdError(lib().fg_last_error().decode(), code)
        return out[:, 0::2] + 1j * out[:, 1::2]

    def field(self, dir_):
        f = self.fields([dir_])[0]
        return [(float(c.real), float(c.imag)) for c in f]

    def intensities(self, dirs) -> np.ndarray:
        d = np.ascontiguousarray(np.asarray(dirs, dtype=np.float64).reshape(-1, 3))
        out = np.zeros(d.shape[0], np.float64)
        P = C.POINTER(C.c_double)
        code = lib().fg_far_intensity(None if self.gpu is None else self.gpu._h, self._h, d.ctypes.data_as(P),
                                      d.shape[0], out.ctypes.data_as(P))
        if code:
            raise FdtdError(lib().fg_last_error().decode(), code)
        return out

    def intensity(self, dir_) -> float:
        return float(self.intensities([dir_])[0])

    def radiated(self, steps: int):
        t, p = C.c_double(), C.c_double()
        code = lib().fg_far_radiated(None if self.gpu is None else self.gpu._h, self._h, steps, C.byref(t), C.byref(p))
        if code:
            raise FdtdError(lib().fg_last_error().decode(), code)
        return t.value, p.value


# ---- adjoint (no counterpart in the reference) ----

@dataclass
class FluxSpec:
    """The flux objective J = |F|^2, F = sum over the (i, j) window of z-plane `plane_k` of
    dA (Ex^ conj(Hy^) - Ey^ conj(Hx^)) at `freq`, and the design box of cells [lo, hi) whose
    relative permittivity and conductivity the gradient is over. `window` None: the nodes inside
    the CPML. `checkpoints` 0 keeps every step's design-edge history; c > 0 keeps about c field
    checkpoints and re-runs each segment in the backward sweep."""
    design_lo: tuple
    design_hi: tuple
    plane_k: int
    freq: float
    steps: int
    window: Optional[tuple] = None   # ((i0, j0), (i1, j1))
    checkpoints: int = 0
    precision: int = 32              # 64: the objective alone, from an FP64 forward on the device
    transposes: int = 0              # 1: the adjoint's E and H transposes as two launches per step

    def struct(self) -> A.fg_flux_spec:
        s = A.fg_flux_spec()
        s.design_lo[:] = [int(v) for v in self.design_lo]
        s.design_hi[:] = [int(v) for v in self.design_hi]
        s.plane_k = int(self.plane_k)
        if self.window is not None:
            s.window_lo[:] = [int(v) for v in self.window[0]]
            s.window_hi[:] = [int(v) for v in self.window[1]]
        s.freq = float(self.freq)
        s.steps = int(self.steps)
        s.checkpoints = int(self.checkpoints)
        s.precision = int(self.precision)
        s.transposes = int(self.transposes)
        return s

    def cells(self) -> int:
        return int(np.prod([h - l for l, h in zip(self.design_lo, self.design_hi)]))

    def shape(self) -> tuple:
        return tuple(int(h - l) for l, h in zip(self.design_lo, self.design_hi))


@dataclass
class FluxResult:
    objective: float
    flux: complex
    grad_eps: Optional[np.ndarray]     # dJ / d eps_r per design cell, shaped like the box
    grad_sigma: Optional[np.ndarray]   # dJ / d sigma (S/m)
    forward_ms: float
    recompute_ms: float
    adjoint_ms: float
    backward_ms: float
    segments: int
    segment_len: int
    design_edges: int
    setup_ms: float = 0.0


def flux_gradient(g, sim: Sim, driven: int, pulse: Pulse, spec: FluxSpec, grad: bool = True) -> FluxResult:
    """The flux objective and, with `grad`, its gradient over the design box (a discrete adjoint of
    the f32 update on the device: one forward run and one backward sweep)."""
    if g is None:
        raise FdtdError("no GPU: this engine has no CPU path", 3)
    L = lib()
    pl = A.pulse_struct(pulse)
    st = spec.struct()
    out = A.fg_flux_result()
    n = spec.cells()
    ge = np.zeros(n, np.float64) if grad else None
    gs = np.zeros(n, np.float64) if grad else None
    P = C.POINTER(C.c_double)
    err = C.create_string_buffer(ERRLEN)
    code = L.fg_flux_gradient(g._h, sim._h, driven, C.byref(pl), C.byref(st), C.byref(out),
                              None if ge is None else ge.ctypes.data_as(P),
                              None if gs is None else gs.ctypes.data_as(P), err, ERRLEN)
    _check(code, err)
    shp = spec.shape()
    return FluxResult(out.objective, complex(out.flux_re, out.flux_im),
                      None if ge is None else ge.reshape(shp), None if gs is None else gs.reshape(shp),
                      out.forward_ms, out.recompute_ms, out.adjoint_ms, out.backward_ms, int(out.segments),
                      int(out.segment_len), int(out.design_edges), out.setup_ms)


def flux_gradient_batch(g, sims, pulses, specs, driven=None, group: int = 16) -> list:
    """Many flux gradients on one GPU (fg_flux_gradient_batch): `group` runs at a time, their
    forwards, objectives and backward sweeps enqueued together on per-run streams. Each result
    equals flux_gradient of that run alone."""
    if g is None:
        raise FdtdError("no GPU: this engine has no CPU path", 3)
    n = len(sims)
    L = lib()
    driven = [0] * n if driven is None else list(driven)
    hs = (C.c_void_p * n)(*[s._h for s in sims])
    dv = (C.c_uint64 * n)(*driven)
    pl = (A.fg_pulse * n)(*[A.pulse_struct(p) for p in pulses])
    st = (A.fg_flux_spec * n)(*[s.struct() for s in specs])
    out = (A.fg_flux_result * n)()
    ge = [np.zeros(s.cells(), np.float64) for s in specs]
    gs = [np.zeros(s.cells(), np.float64) for s in specs]
    P = C.POINTER(C.c_double)
    pe = (P * n)(*[a.ctypes.data_as(P) for a in ge])
    ps = (P * n)(*[a.ctypes.data_as(P) for a in gs])
    err = C.create_string_buffer(ERRLEN)
    code = L.fg_flux_gradient_batch(g._h, hs, dv, pl, st, n, int(group), out, pe, ps, err, ERRLEN)
    _check(code, err)
    res = []
    for q in range(n):
        o = out[q]
        shp = specs[q].shape()
        res.append(FluxResult(o.objective, complex(o.flux_re, o.flux_im), ge[q].reshape(shp), gs[q].reshape(shp),
                              o.forward_ms, o.recompute_ms, o.adjoint_ms, o.backward_ms, int(o.segments),
                              int(o.segment_len), int(o.design_edges), o.setup_ms))
    return res


# ---- batches of independent grids (no counterpart in the reference) ----

class Batch:
    """Many Sims stepped together: one persistent work-list launch marches every grid per step,
    then one launch each for all grids' Debye edges, sources and probes, in a captured graph.
    `tune` times the candidate shapes first (tile, persistent blocks per SM, planes per item) and
    keeps the fastest. Each grid's results equal stepping it alone with the fused step."""

    def __init__(self, g, sims, pulses, max_steps: int, driven=None, tune: bool = True, tile: int = 0,
                 blocks_per_sm: int = 0, seg: int = 32, graph_steps: int = 10):
        if g is None:
            raise FdtdError("no GPU: this engine has no CPU path", 3)
        n = len(sims)
        self._sims = list(sims)   # keep the Sims alive with the batch
        hs = (C.c_void_p * n)(*[s._h for s in sims])
        pl = (A.fg_pulse * n)(*[A.pulse_struct(p) for p in pulses])
        dv = (C.c_uint64 * n)(*([0] * n if driven is None else [int(d) for d in driven]))
        opt = A.fg_batch_options(1 if tune else 0, tile, blocks_per_sm, seg, graph_steps)
        out = C.c_void_p()
        err = C.create_string_buffer(ERRLEN)
        code = lib().fg_batch_new(g._h, hs, dv, pl, n, max_steps, C.byref(opt), C.byref(out), err, ERRLEN)
        _check(code, err)
        self._h = out
        self.size = n

    def step(self, k: int) -> None:
        err = C.create_string_buffer(ERRLEN)
        _check(lib().fg_batch_step(self._h, k, err, ERRLEN), err)

    def sync(self) -> None:
        code = lib().fg_batch_sync(self._h)
        if code:
            raise FdtdError(lib().fg_last_error().decode(), code)

    def read(self, index: int, which: str, n: int) -> np.ndarray:
        out = np.zeros(n, np.float32)
        err = C.create_string_buffer(ERRLEN)
        _check(lib().fg_batch_read(self._h, index, which.encode(), out.ctypes.data_as(C.POINTER(C.c_float)), n,
                                   err, ERRLEN), err)
        return out

    def info(self) -> dict:
        o = A.fg_batch_options()
        pb, tm, st = C.c_int(), C.c_double(), C.c_uint64()
        lib().fg_batch_info(self._h, C.byref(o), C.byref(pb), C.byref(tm), C.byref(st))
        tiles = ["32x8", "64x4", "32x4", "graph branches", "graph branches, direct march", "merged TMA launches"]
        return {"tile": tiles[o.tile], "blocks_per_sm": o.blocks_per_sm, "seg": o.seg,
                "persistent_blocks": pb.value, "tuned_ms_per_step": tm.value, "steps": st.value}

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().fg_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
