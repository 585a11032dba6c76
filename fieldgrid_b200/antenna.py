"""The FDTD antenna workflow of sims-antenna (crates/sims-antenna/src/fdtd/{mod,mesh,engine}.rs,
crates/sims-antenna/src/solve.rs:416-490) on this engine: a box-and-port `Model` is meshed into a
graded `Grid`, turned into a `Sim` (per-cell dielectrics, PEC edges, one lumped port), run on the
GPU until the energy decays, and finished into the input impedance sweep Z(f), S11, the input power
and the far-field box (gain pattern).

Names, argument meanings and error texts follow the reference. `run_gpu` is the reference's
`run_gpu`; there is no CPU path (the reference's `run` calls `run_cpu`, which this package does not
have). Meshed triangle parts (`Part`) go through the CUDA rasteriser (fieldgrid_b200.raster, the
reference's raster.rs): dielectric parts fill the cells whose centres they hold, metal parts mark
the edges they pass through and, when closed, the edges inside them. The V/I spectra of `finish` come from the C ABI's fg_port_spectra (f64, host); the far field from
`fdtd.Far` (f64, device).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np

from . import fdtd
from ._lib import lib
from .grid import Grading, Grid, graded, pad, smooth

C0 = 299_792_458.0          # mod.rs:8-11
EPS0 = 8.854_187_812_8e-12
MU0 = 1.256_637_062_12e-6
ETA0 = 376.730_313_668


@dataclass
class Aabb:
    """mod.rs:13-31."""

    lo: tuple
    hi: tuple

    @staticmethod
    def new(a, b) -> "Aabb":
        return Aabb(tuple(min(a[i], b[i]) for i in range(3)), tuple(max(a[i], b[i]) for i in range(3)))

    def contains_segment(self, a, b, tol: float) -> bool:
        return all(min(a[t], b[t]) >= self.lo[t] - tol and max(a[t], b[t]) <= self.hi[t] + tol for t in range(3))

    def contains(self, p) -> bool:
        return all(self.lo[t] <= p[t] <= self.hi[t] for t in range(3))


@dataclass
class Dielectric:
    """mod.rs:33-38."""

    bounds: Aabb
    eps_r: float
    tan_d: float


@dataclass
class Metal:
    """Stuff::Metal (mod.rs:57-61)."""


@dataclass
class DielectricStuff:
    """Stuff::Dielectric { eps_r, tan_d } (mod.rs:57-61)."""

    eps_r: float
    tan_d: float


@dataclass
class Part:
    """mod.rs:63-115: a triangle mesh ((n, 3, 3) vertices) of one material."""

    triangles: np.ndarray
    stuff: object

    def __post_init__(self):
        self.triangles = np.asarray(self.triangles, np.float64).reshape(-1, 3, 3)

    def bounds(self) -> Optional[Aabb]:
        """mod.rs:69-76."""
        if len(self.triangles) == 0:
            return None
        p = self.triangles.reshape(-1, 3)
        return Aabb(tuple(float(v) for v in p.min(axis=0)), tuple(float(v) for v in p.max(axis=0)))

    def planes(self, axis: int) -> list:
        """mod.rs:78-88: the coordinates of the triangles flat in `axis`, sorted, deduplicated to 1e-9."""
        t = self.triangles
        flat = np.all(np.abs(t[:, :, axis] - t[:, :1, axis]) < 1e-12, axis=1)
        vals = sorted(float(v) for v in t[flat, 0, axis])
        out: list = []
        for v in vals:               # Vec::dedup_by against the last kept value
            if not out or abs(v - out[-1]) >= 1e-9:
                out.append(v)
        return out

    def rims(self, axis: int) -> list:
        """mod.rs:90-114: (coordinate, inward sign) of the boundary edges (used by one triangle)
        that lie flat in `axis` with the triangle's third vertex off that plane."""
        key = [[tuple(np.float64(v).tobytes() for v in p) for p in tri] for tri in self.triangles]
        count: dict = {}
        for tk in key:
            for k in range(3):
                a, b = tk[k], tk[(k + 1) % 3]
                e = (a, b) if a < b else (b, a)
                count[e] = count.get(e, 0) + 1
        out = []
        for tri, tk in zip(self.triangles, key):
            for k in range(3):
                a, b, c = tri[k], tri[(k + 1) % 3], tri[(k + 2) % 3]
                ka, kb = tk[k], tk[(k + 1) % 3]
                once = count.get((ka, kb) if ka < kb else (kb, ka)) == 1
                if not once or abs(a[axis] - b[axis]) > 1e-12 or abs(c[axis] - a[axis]) < 1e-12:
                    continue
                out.append((float(a[axis]), math.copysign(1.0, c[axis] - a[axis])))
        out.sort()
        dedup: list = []
        for v in out:                # dedup_by: equal to 1e-9 with the same sign
            if not dedup or not (abs(v[0] - dedup[-1][0]) < 1e-9 and v[1] == dedup[-1][1]):
                dedup.append(v)
        return dedup


@dataclass
class Wire:
    """mod.rs:40-45."""

    a: tuple
    b: tuple
    radius: float


@dataclass
class Port:
    """mod.rs:47-52."""

    a: tuple
    b: tuple
    r: float


@dataclass
class Model:
    """mod.rs:118-128."""

    parts: list = field(default_factory=list)
    metal: List[Aabb] = field(default_factory=list)
    wires: List[Wire] = field(default_factory=list)
    dielectrics: List[Dielectric] = field(default_factory=list)
    port: Optional[Port] = None
    f0: float = 0.0
    span: float = 0.0
    fine: float = 0.0
    ground_plane_z: Optional[float] = None

    def bounds(self) -> Optional[Aabb]:
        """mod.rs:133-148: the box around metal, wires, dielectrics and the port."""
        boxes = list(self.metal) + [Aabb.new(w.a, w.b) for w in self.wires] + \
            [d.bounds for d in self.dielectrics] + [b for b in (p.bounds() for p in self.parts) if b is not None] + \
            ([Aabb.new(self.port.a, self.port.b)] if self.port else [])
        if not boxes:
            return None
        lo = tuple(min(b.lo[i] for b in boxes) for i in range(3))
        hi = tuple(max(b.hi[i] for b in boxes) for i in range(3))
        return Aabb(lo, hi)


@dataclass
class Sweep:
    freqs: np.ndarray
    z: np.ndarray           # complex input impedance per frequency


@dataclass
class Stats:
    cells: int
    steps: int
    dt: float
    decay_db: float
    gpu: bool


@dataclass
class Outcome:
    """mod.rs:169-176."""

    sweep: Sweep
    z0: complex             # impedance at f0
    p_in: float             # input power at f0, Re(V conj(I)) / 2
    far: Optional[fdtd.Far]
    stats: Stats
    grid: Grid

    def s11(self, z_ref: float = 50.0) -> np.ndarray:
        """The reflection coefficient (Z - z_ref) / (Z + z_ref) over the sweep."""
        return (self.sweep.z - z_ref) / (self.sweep.z + z_ref)


@dataclass
class Options:
    """mod.rs:178-190."""

    points: int = 121
    max_steps: int = 200_000
    decay_db: float = 50.0
    pml: int = 8
    far_field: bool = True


def mesh(model: Model, pml: int) -> Optional[Grid]:
    """mesh.rs:6-133: per axis, lines pinned at metal faces (a third of the fine size inside and
    two thirds outside a wide plate's edge, the edge itself for thin or shared faces), dielectric
    faces and the port's ends, graded from the feature sizes at ratio 1.3 up to lambda/20 in air
    (lambda/20/sqrt(eps_r) inside dielectrics), smoothed to a 1.5 neighbour ratio and padded with
    the CPML cells; the box reaches a quarter wavelength at f0 past the model. Parts pin their flat
    planes and (metal) their rims (mesh.rs:44-70)."""
    bounds = model.bounds()
    if bounds is None:
        return None
    f_max = model.f0 * (1.0 + model.span)
    lam = C0 / f_max
    coarse_air = lam / 20.0
    margin = C0 / model.f0 / 4.0
    fine = model.fine if model.fine > 0.0 else lam / 80.0
    ratio = 1.3
    axes = []
    for a in range(3):
        fixed: list = []
        features: list = []
        pinned = [p for p in ((model.port.a[a], model.port.b[a]) if model.port else ())]
        for mi, m in enumerate(model.metal):
            wide = m.hi[a] - m.lo[a] > 2.0 * fine
            for v, inward in ((m.lo[a], 1.0), (m.hi[a], -1.0)):
                shared = any(abs(p - v) < 1e-9 for p in pinned) or any(
                    oi != mi
                    and all(o.lo[t] <= m.hi[t] and o.hi[t] >= m.lo[t] for t in range(3) if t != a)
                    and (abs(o.lo[a] - v) < 1e-9 or abs(o.hi[a] - v) < 1e-9)
                    for oi, o in enumerate(model.metal))
                if wide and not shared:
                    fixed.append(v + inward * fine / 3.0)
                    fixed.append(v - inward * 2.0 * fine / 3.0)
                else:
                    fixed.append(v)
                features.append((v, fine))
        for part in model.parts:
            b = part.bounds()
            if b is None:
                continue
            if isinstance(part.stuff, DielectricStuff):
                local = lam / 20.0 / math.sqrt(part.stuff.eps_r)
                thick = b.hi[a] - b.lo[a]
                size = max(thick / 4.0, 1e-6) if thick < 4.0 * local else local
            else:
                size = fine
            for v in part.planes(a):
                fixed.append(v)
                features.append((v, size))
            if isinstance(part.stuff, Metal):
                wide = b.hi[a] - b.lo[a] > 2.0 * fine
                for v, inward in part.rims(a):
                    if wide:
                        fixed.append(v + inward * fine / 3.0)
                        fixed.append(v - inward * 2.0 * fine / 3.0)
                    else:
                        fixed.append(v)
                    features.append((v, fine))
            features.append((b.lo[a], size))
            features.append((b.hi[a], size))
        for d in model.dielectrics:
            lo, hi = d.bounds.lo[a], d.bounds.hi[a]
            fixed += [lo, hi]
            local = lam / 20.0 / math.sqrt(d.eps_r)
            thick = hi - lo
            size = max(thick / 4.0, 1e-6) if thick < 4.0 * local else local
            features += [(lo, size), (hi, size), (0.5 * (lo + hi), size)]
        if model.port is not None:
            p = model.port
            for v in (p.a[a], p.b[a]):
                fixed.append(v)
                features.append((v, fine))
            length = abs(p.b[a] - p.a[a])
            if length > 0.0:
                features.append((0.5 * (p.a[a] + p.b[a]), min(length / 2.0, fine * 2.0)))
        fixed += [bounds.lo[a] - margin, bounds.hi[a] + margin]
        fixed.sort()
        dedup: list = []
        for v in fixed:            # Vec::dedup_by against the last kept value
            if not dedup or abs(v - dedup[-1]) >= 1e-7:
                dedup.append(v)
        slow = [(d.bounds.lo[a], d.bounds.hi[a], d.eps_r) for d in model.dielectrics]
        for part in model.parts:
            b = part.bounds()
            if isinstance(part.stuff, DielectricStuff) and b is not None:
                slow.append((b.lo[a], b.hi[a], part.stuff.eps_r))

        def coarse(x, slow=slow):
            s = coarse_air
            for lo, hi, er in slow:
                if lo <= x <= hi:
                    s = min(s, coarse_air / math.sqrt(er))
            return s

        grading = Grading(features=features, coarse=coarse, ratio=ratio, fill=0.0)
        axes.append(np.array(pad(smooth(graded(dedup, grading), 1.5), pml), np.float64))
    return Grid(axes[0], axes[1], axes[2], pml)


def _span(line: np.ndarray, lo: float, hi: float):
    """partition_point(v < lo - 1e-9) and partition_point(v <= hi + 1e-9) (engine.rs:14-18)."""
    return int(np.searchsorted(line, lo - 1e-9, side="left")), int(np.searchsorted(line, hi + 1e-9, side="right"))


def materials(grid: Grid, model: Model, raster=None) -> fdtd.Materials:
    """engine.rs:9-41: each dielectric box sets eps, eps_inf and sigma = w eps0 eps_r tan_d (at f0)
    on the cells between its faces, then each dielectric part on the cells whose centres it holds
    (raster.solid_cells)."""
    nx, ny, nz = grid.dims()
    mats = fdtd.Materials.new(grid)
    w = 2.0 * math.pi * model.f0
    eps = mats.eps.reshape(nx - 1, ny - 1, nz - 1)
    inf = mats.inf.reshape(nx - 1, ny - 1, nz - 1)
    sig = mats.sigma.reshape(nx - 1, ny - 1, nz - 1)
    for d in model.dielectrics:
        r = []
        for a in range(3):
            lo, hi = _span(grid.axis(a), d.bounds.lo[a], d.bounds.hi[a])
            r.append(slice(lo, max(hi - 1, lo)))
        eps[r[0], r[1], r[2]] = np.float32(d.eps_r)
        inf[r[0], r[1], r[2]] = np.float32(d.eps_r)
        sig[r[0], r[1], r[2]] = np.float32(w * EPS0 * d.eps_r * d.tan_d)
    for part in model.parts:
        if not isinstance(part.stuff, DielectricStuff):
            continue
        inside = raster.solid_cells(part.triangles, grid).reshape(nx - 1, ny - 1, nz - 1)
        er, td = part.stuff.eps_r, part.stuff.tan_d
        eps[inside] = np.float32(er)
        inf[inside] = np.float32(er)
        sig[inside] = np.float32(w * EPS0 * er * td)
    return mats


def metal_edges(grid: Grid, metal: List[Aabb]) -> np.ndarray:
    """engine.rs:45-72: per component, the edges inside each metal box (a zero-thickness box
    gives the edges of its plane), as a (3, nx, ny, nz) mask."""
    n = grid.dims()
    mask = np.zeros((3,) + tuple(n), np.uint8)
    for m in metal:
        r = [_span(grid.axis(a), m.lo[a], m.hi[a]) for a in range(3)]
        for c in range(3):
            lim = [list(x) for x in r]
            lim[c][1] = max(lim[c][1] - 1, 0)
            if all(lim[a][0] < lim[a][1] for a in range(3)):
                mask[c, lim[0][0]:lim[0][1], lim[1][0]:lim[1][1], lim[2][0]:lim[2][1]] = 1
    return mask


def port_def(grid: Grid, p: Port) -> fdtd.PortDef:
    """engine.rs:74-92: the port's edges along its longest axis, from the node nearest its low end
    to the node nearest its high end (at least one edge)."""
    spans = [abs(p.b[t] - p.a[t]) for t in range(3)]
    axis = max(range(3), key=lambda t: (spans[t], t))     # Iterator::max_by keeps the last maximum
    at = [grid.nearest(t, min(p.a[t], p.b[t])) for t in range(3)]
    end = grid.nearest(axis, max(p.a[axis], p.b[axis]))
    count = max(end - at[axis], 1) if end > at[axis] else 1
    edges = []
    for s in range(count):
        q = list(at)
        q[axis] += s
        edges.append(fdtd.Edge(axis, tuple(q)))
    return fdtd.PortDef("feed", [edges], p.r, False)


def wire_edges(grid: Grid, wires: List[Wire]):
    """engine.rs:94-111: thin wires as (Edge, radius) along one grid axis."""
    out = []
    for w in wires:
        along = [t for t in range(3) if abs(w.b[t] - w.a[t]) > 1e-9]
        if len(along) != 1:
            raise fdtd.FdtdError("a thin wire must run along one axis of the grid")
        axis = along[0]
        at = [grid.nearest(t, min(w.a[t], w.b[t])) for t in range(3)]
        end = grid.nearest(axis, max(w.a[axis], w.b[axis]))
        for s in range(at[axis], end):
            q = list(at)
            q[axis] = s
            out.append((fdtd.Edge(axis, tuple(q)), w.radius))
    return out


def sim_args(grid: Grid, model: Model, port: Port, raster=None):
    """The arguments of Sim::try_new that engine.rs:105-131 builds: materials, the PEC mask of the
    metal boxes, wires and metal parts (the edges a part passes through and, for a closed part,
    the edges inside it), one port and the thin wires."""
    mats = materials(grid, model, raster)
    wires = wire_edges(grid, model.wires)
    solid = list(model.metal) + [Aabb.new(w.a, w.b) for w in model.wires]
    mask = metal_edges(grid, solid)
    n = tuple(grid.dims())
    for part in model.parts:
        if not isinstance(part.stuff, Metal):
            continue
        more = [raster.sheet_edges(part.triangles, grid)]
        if raster.closed(part.triangles):
            more.append(raster.solid_edges(part.triangles, grid))
        for m in more:
            for c in range(3):
                mask[c] |= np.asarray(m[c], np.uint8).reshape(n)
    return (grid, mats, mask.reshape(-1), [], [port_def(grid, port)], [],
            fdtd.Media(fdtd.Sheets(), fdtd.Debye(), wires))


def build(grid: Grid, model: Model, port: Port, raster=None) -> fdtd.Sim:
    """engine.rs:105-131."""
    return fdtd.Sim.try_new(*sim_args(grid, model, port, raster))


@dataclass
class Setup:
    """mod.rs:192-199."""

    sim: object
    patches: Optional[fdtd.Patches]
    freqs: np.ndarray
    f0: float
    fc: float
    grid: Grid
    args: tuple = ()


def sweep_freqs(model: Model, points: int) -> np.ndarray:
    """mod.rs:215-220: `points` frequencies over f0 (1 -/+ span)."""
    f0 = model.f0
    return np.array([f0 * (1.0 - model.span + 2.0 * model.span * i / max(points - 1, 1)) for i in range(points)])


def setup(model: Model, opts: Options, sim_factory: Callable = None, patch_fn: Callable = None,
          raster=None) -> Setup:
    """mod.rs:195-213. `sim_factory(*args)` builds the Sim, `patch_fn(sim, inset)` its NTFF box and
    `raster` rasterises the parts (defaults: this engine's Sim.try_new, fdtd.patches and the CUDA
    rasteriser on a Gpu opened here when the model has parts)."""
    port = model.port
    if port is None:
        raise fdtd.FdtdError("the model has no port")
    if model.parts and raster is None:
        from .gpu import Gpu
        from .raster import GpuRaster
        raster = GpuRaster(Gpu.open())
    closed = raster.closed if raster is not None else (lambda _t: False)
    if any(isinstance(p.stuff, DielectricStuff) and not closed(p.triangles) for p in model.parts):
        raise fdtd.FdtdError("a dielectric part is not a closed mesh")
    solid = Model(parts=list(model.parts), metal=list(model.metal) + [Aabb.new(w.a, w.b) for w in model.wires],
                  wires=list(model.wires), dielectrics=list(model.dielectrics), port=model.port, f0=model.f0,
                  span=model.span, fine=model.fine, ground_plane_z=model.ground_plane_z)
    grid = mesh(solid, opts.pml)
    if grid is None:
        raise fdtd.FdtdError("nothing to mesh")
    args = sim_args(grid, model, port, raster)
    sim = (sim_factory or fdtd.Sim.try_new)(*args)
    patches = (patch_fn or fdtd.patches)(sim, 3) if opts.far_field else None
    return Setup(sim, patches, sweep_freqs(model, opts.points), model.f0, model.f0 * 0.5, grid, args)


def extras(s: Setup, opts: Options) -> fdtd.Extras:
    """mod.rs:225-235."""
    return fdtd.Extras(max_steps=opts.max_steps, decay_db=opts.decay_db,
                       freqs=[s.f0] if s.patches is not None else [],
                       ntff=s.patches.gpu if s.patches is not None else None, check_every=500, fused_e=True)


def port_spectra(series, steps: int, ports: int, port: int, dt: float, freqs) -> tuple:
    """fg_port_spectra: V(f) and I(f) of one port's series (mod.rs:239-253)."""
    series = np.ascontiguousarray(series, np.float32)
    freqs = np.ascontiguousarray(freqs, np.float64)
    v = np.zeros(2 * len(freqs))
    i = np.zeros(2 * len(freqs))
    P = C.POINTER
    code = lib().fg_port_spectra(series.ctypes.data_as(P(C.c_float)), steps, ports, port, dt,
                                 freqs.ctypes.data_as(P(C.c_double)), len(freqs), v.ctypes.data_as(P(C.c_double)),
                                 i.ctypes.data_as(P(C.c_double)))
    if code:
        raise fdtd.FdtdError(lib().fg_last_error().decode(), code)
    return v[0::2] + 1j * v[1::2], i[0::2] + 1j * i[1::2]


def finish(s: Setup, rec, gpu: bool, far_gpu=None) -> Outcome:
    """mod.rs:237-266: Z(f) = V(f)/I(f) over the sweep and at f0, P_in = Re(V conj(I))/2 at f0, and
    the far-field box from the NTFF accumulators at f0. `rec` is a run's Record."""
    dt = s.sim.dt
    steps = int(rec.steps)
    ports = len(rec.series) // (2 * steps) if steps else 1
    every = np.concatenate([s.freqs, [s.f0]])
    v, i = port_spectra(rec.series, steps, ports, 0, dt, every)
    z = v / i
    far = None
    if s.patches is not None and len(rec.ntff):
        far = fdtd.Far.load(s.patches, rec.ntff, 1, 0, s.f0, (1.0, 0.0), gpu=far_gpu)
    stats = Stats(s.grid.cells(), steps, dt, float(rec.decay_db), gpu)
    return Outcome(Sweep(s.freqs, z[:-1]), complex(z[-1]), float(0.5 * (v[-1] * np.conj(i[-1])).real), far, stats,
                   s.grid)


def run_gpu(model: Model, opts: Options = None, progress=None, g=None) -> Outcome:
    """mod.rs:279-290 on this engine. `g` is an open fieldgrid_b200.gpu.Gpu (opened when None)."""
    from .gpu import Gpu
    opts = opts or Options()
    g = g or Gpu.open()
    from .raster import GpuRaster
    s = setup(model, opts, raster=GpuRaster(g))
    pulse = fdtd.Pulse(s.f0, s.fc)
    rec = fdtd.run(g, s.sim, 0, pulse, extras(s, opts), progress)
    return finish(s, rec, True, far_gpu=g)


def run(model: Model, opts: Options = None, progress=None):
    """The reference's CPU `run` (mod.rs:268-277): this package has no CPU path."""
    raise fdtd.FdtdError("this engine has no CPU path; use run_gpu", 2)


def intensity(f):
    """ntff.rs (sims-antenna) :23-25: sum |E_c|^2 / (2 eta0) over the last axis."""
    f = np.asarray(f)
    return np.sum(np.abs(f) ** 2, axis=-1) / (2.0 * ETA0)


@dataclass
class VolumeResult:
    """The fields of solve.rs's SolveResult that volume_result (solve.rs:416-490) fills."""

    z: complex
    swr: float
    cells: int
    directivity: Optional[float] = None    # dBi
    efficiency: Optional[float] = None
    dbi: Optional[float] = None
    peak: float = 0.0
    _grid: Optional[np.ndarray] = None     # (nt, np, 3) complex far field, normalised to peak 1
    _nt: int = 91
    _np: int = 121

    def pattern(self, d) -> float:
        """The far field's magnitude at direction d, bilinear over the (theta, phi) grid."""
        th = math.acos(max(-1.0, min(1.0, d[2])))
        ph = math.atan2(d[1], d[0])
        if ph < 0.0:
            ph += 2.0 * math.pi
        x = th / math.pi * (self._nt - 1)
        y = ph / (2.0 * math.pi) * (self._np - 1)
        i, j = min(int(math.floor(x)), self._nt - 2), min(int(math.floor(y)), self._np - 2)
        fx, fy = x - i, y - j
        acc = np.zeros(3, complex)
        for di, dj, w in ((0, 0, (1 - fx) * (1 - fy)), (1, 0, fx * (1 - fy)), (0, 1, (1 - fx) * fy), (1, 1, fx * fy)):
            acc += w * self._grid[i + di, j + dj]
        return float(math.sqrt(np.sum(acc.real ** 2) + np.sum(acc.imag ** 2)))

    def gain_dbi(self, d) -> Optional[float]:
        """solve.rs:55-59."""
        if self._grid is None or self.dbi is None:
            return None
        return self.dbi + 20.0 * math.log10(max(self.pattern(d), 1e-12) / max(self.peak, 1e-30))


def swr_of(z: complex, z0: float) -> float:
    """solve.rs:74-77."""
    g = abs(z - z0) / max(abs(z + z0), 1e-12)
    return min((1.0 + g) / max(1.0 - g, 1e-6), 99.0)


def volume_result(out: Outcome) -> VolumeResult:
    """solve.rs:416-490: the far field on a 91 x 121 (theta, phi) grid, its total radiated power
    (band-averaged) and peak intensity, directivity 4 pi U_max / P_rad, efficiency
    min(P_rad / P_in, 1) and the gain in dBi."""
    r = VolumeResult(out.z0, swr_of(out.z0, 50.0), out.stats.cells)
    if out.far is None:
        return r
    nt, npp = 91, 121
    th = np.arange(nt) / (nt - 1) * math.pi
    ph = np.arange(npp) / (npp - 1) * 2.0 * math.pi
    t, p = np.meshgrid(th, ph, indexing="ij")
    dirs = np.stack([np.sin(t) * np.cos(p), np.sin(t) * np.sin(p), np.cos(t)], -1).reshape(-1, 3)
    grid = out.far.fields(dirs).reshape(nt, npp, 3)
    u = np.sum(np.abs(grid) ** 2, -1) / (2.0 * ETA0)
    total = 0.0
    for i in range(nt - 1):
        th0, th1 = i / (nt - 1) * math.pi, (i + 1) / (nt - 1) * math.pi
        band = (math.cos(th0) - math.cos(th1)) * 2.0 * math.pi / (npp - 1)
        avg = (u[i, :-1] + u[i + 1, :-1] + u[i, 1:] + u[i + 1, 1:]) / 4.0
        total += float(np.sum(avg)) * band
    peak = float(u.max())
    norm = 1.0 / max(math.sqrt(peak * 2.0 * ETA0), 1e-300)
    r._grid = grid * norm
    if total > 0.0 and out.p_in > 0.0:
        d = 4.0 * math.pi * peak / total
        eff = min(total / out.p_in, 1.0)
        r.directivity = 10.0 * math.log10(d)
        r.efficiency = eff
        r.dbi = 10.0 * math.log10(d * eff)
        r.peak = 1.0
    return r
