"""Seeded synthetic workloads: the grids, materials, ports and run settings the tests and the
benchmark step. Every random draw comes from SplitMix64 so a workload is the same on any host.

* `everything()`  the all-features scene of sims-field's tests/fdtd.rs:43-125 (graded 26x22x20,
                  Debye slab, PEC, R/L/C, two ports, six adaptive sheets, two thin wires).
* `dielectric_box(...)`  plain FDTD: a cubic grid with a centred eps_r = 4 box, a soft Ez point
                  source (a 1e7-ohm port) at the centre and 4 seeded point probes.
* `spheres(...)`  throughput: seeded random dielectric/Debye spheres and one 50-ohm port.
* `patch_antenna(...)`  antenna far field: a PEC patch on a 2-cell substrate over a PEC ground,
                  fed by a 50-ohm port, with the NTFF box and 3 DFT frequencies.
* `cavity()` / `wire_cavity(radius)`  the closed boxes of tests/fdtd.rs:189-269.

Each builder returns a `Scene` (Sim::try_new arguments plus Pulse and Extras). `scale` arguments
shrink a workload with its proportions kept, for parity runs the CPU oracle finishes quickly.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .fdtd import Debye, Edge, Element, Extras, Lumped, Materials, Media, PortDef, Pulse, Resistive, Sheets, idx
from .grid import Grid, uniform


class SplitMix64:
    """SplitMix64 (Steele, Lea, Flood 2014)."""

    def __init__(self, seed: int):
        self.state = seed & 0xFFFFFFFFFFFFFFFF

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        return z ^ (z >> 31)

    def uniform(self, lo: float, hi: float) -> float:
        """Uniform in [lo, hi) from the top 53 bits."""
        return lo + (hi - lo) * ((self.next_u64() >> 11) * (1.0 / 9007199254740992.0))

    def integer(self, lo: int, hi: int) -> int:
        """Uniform integer in [lo, hi] inclusive."""
        return lo + int(self.next_u64() % (hi - lo + 1))


@dataclass
class Scene:
    name: str
    grid: Grid
    mats: Materials
    pec: object
    lumped: list
    ports: list
    resistive: list
    media: Media
    pulse: Pulse
    extras: Extras
    driven: int = 0
    info: dict = field(default_factory=dict)

    def args(self):
        """The argument tuple of Sim.try_new."""
        return (self.grid, self.mats, self.pec, self.lumped, self.ports, self.resistive, self.media)


def _graded(n: int, start: float, grow: float):
    out = [0.0]
    d = start
    for _ in range(1, n):
        out.append(out[-1] + d)
        d *= grow
    return out


def everything(steps: int = 1500, fused: bool = False) -> Scene:
    """The all-features scene of tests/fdtd.rs:43-125."""
    grid = Grid(_graded(26, 1e-3, 1.01), _graded(22, 1e-3, 1.0), _graded(20, 0.8e-3, 1.02), 4)
    n = grid.dims()
    cells = (n[0] - 1, n[1] - 1, n[2] - 1)
    mats = Materials.new(grid)
    eps = mats.eps.reshape(cells)
    inf = mats.inf.reshape(cells)
    deb = mats.debye.reshape(cells)
    sig = mats.sigma.reshape(cells)
    eps[:, :, 6:9] = 4.0
    inf[:, :, 6:9] = 3.6
    deb[:, :, 6:9] = 0.4
    sig[:, :, 6:9] = 0.002
    debye = Debye.band(1e9, 2e10)

    def pec(c, p):
        return (c != 2) & (p[2] == 6) & (p[0] < 7)

    lumped = [
        Lumped("c", [Edge(2, (14, 11, 6))], Element.Capacitor(1e-12)),
        Lumped("r", [Edge(2, (16, 11, 6))], Element.Resistor(30.0)),
        Lumped("l", [Edge(2, (18, 11, 6))], Element.Inductor(2e-9)),
    ]

    def column(i, j):
        return [Edge(2, (i, j, k)) for k in range(6, 9)]

    ports = [
        PortDef("a", [column(10, 10), column(10, 11)], 50.0, False),
        PortDef("b", [column(20, 12)], 75.0, True),
    ]
    resistive = [Resistive(0, idx(n, i, 8, 9), 0.4, i % 2 == 0, (0, 1)) for i in range(8, 14)]
    wires = [(Edge(2, (8, 16, k)), 0.2e-3) for k in range(10, 14)] + [(Edge(0, (i, 16, 14)), 0.2e-3) for i in range(8, 12)]
    table = [1.0, 1.0, 2.0, 0.0, 0.9, 0.05, 0.8, 0.1, 0.02, 0.01, 1.0, 0.2, 0.1, 0.05, 0.02, 1.2, 0.1, 0.08, 0.03, 0.01]
    media = Media(Sheets(table, 3), debye, wires)
    extras = Extras(max_steps=steps, decay_db=math.inf, freqs=[3e9, 7e9], plane_k=7, ntff=None, fused_e=fused,
                    check_every=250)
    scene = Scene("everything", grid, mats, pec, lumped, ports, resistive, media, Pulse(5e9, 5e9), extras)
    scene.info["ntff_inset"] = 2
    return scene


def _point_port(name, at, r=1e7):
    return PortDef(name, [[Edge(2, tuple(int(v) for v in at))]], r, False)


def dielectric_box(cells: int = 64, dx: float = 1e-3, pml: int = 8, steps: int = 1000, seed: int = 1,
                   fused: bool = True) -> Scene:
    """Plain FDTD: cells^3 uniform grid, centred (cells/4)^3 eps_r = 4 box, soft Ez point source
    (a 1e7-ohm port) at the centre, 4 seeded 1e7-ohm Ez point probes."""
    grid = Grid.uniform((0.0, 0.0, 0.0), (cells * dx,) * 3, (cells,) * 3, pml)
    mats = Materials.new(grid)
    eps = mats.eps.reshape(cells, cells, cells)
    lo, hi = 3 * cells // 8, 5 * cells // 8
    eps[lo:hi, lo:hi, lo:hi] = 4.0
    c = cells // 2
    ports = [_point_port("source", (c, c, c))]
    rng = SplitMix64(seed)
    for q in range(4):
        at = [rng.integer(pml + 2, cells - 2 - pml - 1) for _ in range(3)]
        ports.append(_point_port(f"probe{q}", at))
    extras = Extras(max_steps=steps, decay_db=math.inf, fused_e=fused, check_every=min(steps, 1000) or 1000)
    scene = Scene(f"dielectric box {cells}^3", grid, mats, None, [], ports, [], Media(), Pulse(10e9, 5e9), extras)
    scene.info.update(cells=cells, dx=dx, pml=pml)
    return scene


def sphere_materials(cells, count, rmin, rmax, pml, seed, debye_share=0.2):
    """Seeded random spheres (later ones overwrite earlier ones) on a cell grid of `cells` per axis
    (an int, or a 3-tuple for a box). Returns (Materials arrays eps, sigma, inf, debye) and the
    Debye time constant."""
    dims = (cells,) * 3 if np.isscalar(cells) else tuple(int(v) for v in cells)
    eps = np.ones(dims, np.float32)
    sig = np.zeros(dims, np.float32)
    inf = np.ones(dims, np.float32)
    deb = np.zeros(dims, np.float32)
    rng = SplitMix64(seed)
    tau = rng.uniform(5e-12, 50e-12)
    spheres = []
    for _ in range(count):
        cx, cy, cz = (rng.uniform(pml, dims[a] - pml) for a in range(3))
        r = rng.integer(rmin, rmax)
        er = rng.uniform(1.0, 10.0)
        s = rng.uniform(0.0, 0.05)
        is_debye = rng.uniform(0.0, 1.0) < debye_share
        de = rng.uniform(1.0, 5.0) if is_debye else 0.0
        spheres.append((cx, cy, cz, r, er, s, is_debye, de))
    for cx, cy, cz, r, er, s, is_debye, de in spheres:
        lo = [max(int(math.floor(v - r)), 0) for v in (cx, cy, cz)]
        hi = [min(int(math.ceil(v + r)) + 1, dims[a]) for a, v in enumerate((cx, cy, cz))]
        if any(h <= l for l, h in zip(lo, hi)):
            continue
        x = np.arange(lo[0], hi[0], dtype=np.float64)[:, None, None] + 0.5 - cx
        y = np.arange(lo[1], hi[1], dtype=np.float64)[None, :, None] + 0.5 - cy
        z = np.arange(lo[2], hi[2], dtype=np.float64)[None, None, :] + 0.5 - cz
        m = (x * x + y * y + z * z) <= r * r
        sl = (slice(lo[0], hi[0]), slice(lo[1], hi[1]), slice(lo[2], hi[2]))
        if is_debye:
            eps[sl][m] = er + de
            inf[sl][m] = er
            deb[sl][m] = de
        else:
            eps[sl][m] = er
            inf[sl][m] = 1.0
            deb[sl][m] = 0.0
        sig[sl][m] = s
    return (eps, sig, inf, deb), tau


def spheres(cells: int = 512, dx: float = 1e-3, pml: int = 10, steps: int = 2000, count: int = 200,
            rmin: int = 5, rmax: int = 40, seed: int = 2, fused: bool = True) -> Scene:
    """Throughput: cells^3, seeded random spheres (20 % one-pole Debye sharing one global pole
    1/tau), one 50-ohm z-port at x-node 48 (every f32-stored index stays below 2^24)."""
    grid = Grid.uniform((0.0, 0.0, 0.0), (cells * dx,) * 3, (cells,) * 3, pml)
    (eps, sig, inf, deb), tau = sphere_materials(cells, count, rmin, rmax, pml, seed)
    mats = Materials(eps, sig, inf, deb)
    c = cells // 2
    i_port = min(48, max(pml + 2, cells // 10))
    ports = [PortDef("port", [[Edge(2, (i_port, c, c))]], 50.0, False)]
    media = Media(Sheets(), Debye([(1.0 / tau, 1.0)]), [])
    extras = Extras(max_steps=steps, decay_db=math.inf, fused_e=fused, check_every=1000)
    scene = Scene(f"random spheres {cells}^3", grid, mats, None, [], ports, [], media, Pulse(10e9, 5e9), extras)
    scene.info.update(cells=cells, dx=dx, pml=pml, spheres=count, tau=tau)
    return scene


def patch_antenna(nx: int = 256, ny: int = 256, nz: int = 192, dx: float = 0.25e-3, pml: int = 12,
                  steps: int = 6000, patch=(40, 30), ground=None, fused: bool = True) -> Scene:
    """Antenna far field: PEC ground at z-node kg over the central `ground` cells, a 2-cell
    substrate (eps_r 4.4, sigma 0.002), a PEC patch at kg + 2 and a 50-ohm port from ground to
    patch at an offset feed; DFT at 8, 10, 12 GHz on the NTFF box 3 cells inside the CPML."""
    grid = Grid.uniform((0.0, 0.0, 0.0), (nx * dx, ny * dx, nz * dx), (nx, ny, nz), pml)
    mats = Materials.new(grid)
    kg = pml + max(4, nz // 12)
    if ground is None:
        ground = (int(nx * 0.625), int(ny * 0.625))
    gx0, gy0 = (nx - ground[0]) // 2, (ny - ground[1]) // 2
    gx1, gy1 = gx0 + ground[0], gy0 + ground[1]
    eps = mats.eps.reshape(nx, ny, nz)
    sig = mats.sigma.reshape(nx, ny, nz)
    eps[gx0:gx1, gy0:gy1, kg:kg + 2] = 4.4
    sig[gx0:gx1, gy0:gy1, kg:kg + 2] = 0.002
    px0, py0 = (nx - patch[0]) // 2, (ny - patch[1]) // 2
    px1, py1 = px0 + patch[0], py0 + patch[1]

    def pec(c, p):
        i, j, k = p
        on_ground = (k == kg) & (i >= gx0) & (i < gx1) & (j >= gy0) & (j < gy1)
        on_patch = (k == kg + 2) & (i >= px0) & (i < px1) & (j >= py0) & (j < py1)
        return (c != 2) & (on_ground | on_patch)

    feed = (px0 + patch[0] // 4, (py0 + py1) // 2)
    ports = [PortDef("feed", [[Edge(2, (feed[0], feed[1], kg)), Edge(2, (feed[0], feed[1], kg + 1))]], 50.0, False)]
    extras = Extras(max_steps=steps, decay_db=math.inf, freqs=[8e9, 10e9, 12e9], fused_e=fused, check_every=1000)
    scene = Scene(f"patch antenna {nx}x{ny}x{nz}", grid, mats, pec, [], ports, [], Media(), Pulse(10e9, 5e9), extras)
    scene.info.update(kg=kg, feed=feed, ntff_inset=3, dx=dx, pml=pml)
    return scene


def cavity(steps: int = 40000) -> Scene:
    """The empty PEC cavity on a graded x axis of tests/fdtd.rs:189-215."""
    a, b, d = 0.10, 0.07, 0.05
    xs, t, s = [], 0.0, 0.0035
    while t < a - 1e-9:
        xs.append(t)
        t += s
        s = min(s * 1.06, 0.0055)
    xs.append(a)
    grid = Grid(xs, [b * i / 18 for i in range(19)], [d * i / 13 for i in range(14)], 0)
    n = grid.dims()
    port = PortDef("probe", [[Edge(2, (n[0] // 3, n[1] // 3, n[2] // 3))]], 1e7, False)
    extras = Extras(max_steps=steps, decay_db=math.inf)
    scene = Scene("cavity", grid, Materials.new(grid), None, [], [port], [], Media(), Pulse(3.0e9, 2.5e9), extras)
    scene.info.update(a=a, b=b, d=d)
    return scene


def wire_cavity(radius: float, steps: int = 40000) -> Scene:
    """The thin-wire cavity of tests/fdtd.rs:238-262."""
    a, b, d = 0.10, 0.07, 0.05
    grid = Grid([a * i / 22 for i in range(23)], [b * i / 18 for i in range(19)], [d * i / 13 for i in range(14)], 0)
    n = grid.dims()
    port = PortDef("probe", [[Edge(2, (n[0] // 3, n[1] // 3, n[2] // 3))]], 1e7, False)
    wires = [(Edge(2, (11, 9, k)), radius) for k in range(3, 9)] + [(Edge(0, (i, 9, 9)), radius) for i in range(11, 15)]
    extras = Extras(max_steps=steps, decay_db=math.inf)
    return Scene(f"wire cavity r={radius}", grid, Materials.new(grid), None, [], [port], [], Media(wires=wires),
                 Pulse(3.0e9, 2.5e9), extras)


def flux_design(nx: int = 160, ny: int = 160, nz: int = 96, dx: float = 1e-3, pml: int = 8,
                design: tuple = (32, 32, 8), steps: int = 4000, checkpoints: int = 64, seed: int = 4,
                freq: float = 10e9, debye: bool = False):
    """Adjoint workload: an nx x ny x nz vacuum grid with a 50-ohm z-port source below a design
    block of per-voxel eps_r ~ U[1, 12] and sigma ~ U[0, 0.01] S/m (seed), and the flux objective
    |F|^2 at `freq` on a z-plane above it. With `debye`, a one-pole Debye slab (eps_inf 2, delta
    eps 3, tau 20 ps) stands beside the design block, between its low-x face and the CPML.
    Returns (scene, spec, eps0, sig0): the scene built with the initial design, the FluxSpec, and
    the design arrays (shaped like the block)."""
    from .fdtd import FluxSpec
    grid = Grid.uniform((0.0, 0.0, 0.0), (nx * dx, ny * dx, nz * dx), (nx, ny, nz), pml)
    rng = SplitMix64(seed)
    dw = tuple(int(v) for v in design)
    cnt = dw[0] * dw[1] * dw[2]
    eps0 = np.array([rng.uniform(1.0, 12.0) for _ in range(cnt)], np.float32).reshape(dw)
    sig0 = np.array([rng.uniform(0.0, 0.01) for _ in range(cnt)], np.float32).reshape(dw)
    ks = pml + max(2, nz // 8)                       # source node height
    kd = ks + max(2, nz // 8)                        # design block bottom cell
    kp = min(kd + dw[2] + max(2, nz // 8), nz - pml - 2)   # flux plane
    lo = (nx // 2 - dw[0] // 2, ny // 2 - dw[1] // 2, kd)
    hi = (lo[0] + dw[0], lo[1] + dw[1], lo[2] + dw[2])
    ports = [PortDef("source", [[Edge(2, (nx // 2, ny // 2, ks))]], 50.0, False)]
    extras = Extras(max_steps=steps, decay_db=math.inf, fused_e=True, check_every=min(steps, 1000) or 1000,
                    freqs=[freq], plane_k=kp)
    spec = FluxSpec(design_lo=lo, design_hi=hi, plane_k=kp, freq=freq, steps=steps, checkpoints=checkpoints)

    tau = 20e-12
    media = Media(Sheets(), Debye([(1.0 / tau, 1.0)]), []) if debye else Media()

    def scene(eps=eps0, sig=sig0) -> Scene:
        mats = Materials.new(grid)
        e = mats.eps.reshape(nx, ny, nz)
        s = mats.sigma.reshape(nx, ny, nz)
        e[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = np.asarray(eps, np.float32)
        s[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = np.asarray(sig, np.float32)
        if debye:
            x0 = max(pml + 1, lo[0] - 6)
            box = (slice(x0, lo[0] - 1), slice(lo[1], hi[1]), slice(lo[2] - 1, hi[2] + 1))
            mats.inf.reshape(nx, ny, nz)[box] = 2.0
            mats.debye.reshape(nx, ny, nz)[box] = 3.0
            e[box] = 5.0
        sc = Scene(f"flux design {nx}x{ny}x{nz}, block {dw[0]}x{dw[1]}x{dw[2]}", grid, mats, None, [], ports, [],
                   media, Pulse(freq, freq / 2), extras)
        sc.info.update(dx=dx, pml=pml, design=dw, plane_k=kp)
        return sc

    return scene, spec, eps0, sig0


def batch_grids(count: int = 192, lo: int = 48, hi: int = 160, pml: int = 8, steps: int = 1500, seed: int = 6,
                dx: float = 1e-3):
    """Batched workload: `count` grids, each nx, ny, nz ~ U{lo..hi} in steps of 8 cells (seed), an
    8-cell CPML, seeded random spheres as in the throughput workload (count and radii scaled to the
    grid, 20 % Debye) and one randomly placed 1e7-ohm Ez point source. Returns a list of Scenes."""
    rng = SplitMix64(seed)
    scenes = []
    for b in range(count):
        dims = tuple(8 * rng.integer(lo // 8, hi // 8) for _ in range(3))
        grid = Grid.uniform((0.0, 0.0, 0.0), tuple(d * dx for d in dims), dims, pml)
        nsph = max(4, int(200 * (min(dims) / 512.0) ** 2 * 4))
        (eps, sig, inf, deb), tau = sphere_materials(dims, nsph, max(2, min(dims) // 40), max(4, min(dims) // 6),
                                                     pml, rng.next_u64())
        mats = Materials(eps, sig, inf, deb)
        media = Media(Sheets(), Debye([(1.0 / tau, 1.0)]), [])
        at = tuple(rng.integer(pml + 2, d - pml - 3) for d in dims)
        ports = [_point_port("source", at)]
        extras = Extras(max_steps=steps, decay_db=math.inf, fused_e=True, check_every=min(steps, 1000) or 1000)
        sc = Scene(f"batch grid {b}: {dims[0]}x{dims[1]}x{dims[2]}", grid, mats, None, [], ports, [], media,
                   Pulse(10e9, 5e9), extras)
        sc.info.update(dims=dims, pml=pml, spheres=nsph)
        scenes.append(sc)
    return scenes


def batch_flux(count: int = 192, lo: int = 48, hi: int = 160, pml: int = 8, steps: int = 1500, seed: int = 6,
               dx: float = 1e-3, design: int = 16, checkpoints: int = 39, freq: float = 10e9):
    """Batched adjoint workload: the grids of batch_grids (same seed, so the same dims, spheres and
    Debye pole), each with a centred design^3 block of per-voxel eps_r ~ U[1, 12] and sigma ~ U[0,
    0.01] S/m (cleared of the spheres with a one-cell margin, so no Debye edge reaches it), the
    flux objective at `freq` on a z-plane two nodes above the block, and the point source moved
    below the block when it fell inside the cleared region. Returns [(scene, spec, eps0, sig0)]
    with scene(eps, sig) -> Scene as in flux_design."""
    from .fdtd import FluxSpec
    base = batch_grids(count, lo, hi, pml, steps, seed, dx)
    rng = SplitMix64(seed ^ 0x5EED)
    out = []
    for b, sc0 in enumerate(base):
        dims = sc0.info["dims"]
        d = min(design, min(dims) - 2 * pml - 8)
        blo = tuple(dims[a] // 2 - d // 2 for a in range(3))
        bhi = tuple(v + d for v in blo)
        plane_k = bhi[2] + 2
        eps0 = np.array([rng.uniform(1.0, 12.0) for _ in range(d ** 3)], np.float32).reshape(d, d, d)
        sig0 = np.array([rng.uniform(0.0, 0.01) for _ in range(d ** 3)], np.float32).reshape(d, d, d)
        at = sc0.ports[0].columns[0][0].at
        clear = tuple(slice(blo[a] - 1, bhi[a] + 1) for a in range(3))
        inside = all(blo[a] - 2 <= at[a] <= bhi[a] + 1 for a in range(3))
        src = (blo[0] + d // 2, blo[1] + d // 2, max(pml + 2, blo[2] - 4)) if inside else at
        ports = [_point_port("source", src)]
        extras = Extras(max_steps=steps, decay_db=math.inf, fused_e=True, check_every=min(steps, 1000) or 1000,
                        freqs=[freq], plane_k=plane_k)
        spec = FluxSpec(design_lo=blo, design_hi=bhi, plane_k=plane_k, freq=freq, steps=steps, checkpoints=checkpoints)

        def scene(eps=eps0, sig=sig0, sc0=sc0, dims=dims, blo=blo, bhi=bhi, clear=clear, ports=ports, extras=extras,
                  b=b, plane_k=plane_k) -> Scene:
            m0 = sc0.mats
            shp = tuple(dims)
            e = m0.eps.reshape(shp).copy()
            s = m0.sigma.reshape(shp).copy()
            inf = m0.inf.reshape(shp).copy()
            deb = m0.debye.reshape(shp).copy()
            e[clear], s[clear], inf[clear], deb[clear] = 1.0, 0.0, 1.0, 0.0
            box = tuple(slice(blo[a], bhi[a]) for a in range(3))
            e[box] = np.asarray(eps, np.float32)
            s[box] = np.asarray(sig, np.float32)
            mats = Materials(e, s, inf, deb)
            sc = Scene(f"batch flux {b}: {dims[0]}x{dims[1]}x{dims[2]}", sc0.grid, mats, None, [], ports, [],
                       sc0.media, Pulse(freq, freq / 2), extras)
            sc.info.update(dims=dims, design=(blo, bhi), plane_k=plane_k)
            return sc

        out.append((scene, spec, eps0, sig0))
    return out
