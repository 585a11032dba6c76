"""Test infrastructure: a second, independent CPU restatement of the reference's FDTD step, taken
from its GPU shader (crates/sims-field/src/fdtd/fdtd.wgsl) rather than from its CPU path (cpu.rs,
which the oracle restates). It runs the shader's separate pipeline in the dispatch order of
run.rs:627-648 (wire_h, update_h, sheet_pre, debye_pre, update_e, sheet_post, debye_post, lumped,
then probe and field_dft per step), vectorised over nodes with numpy in f32, on the buffers that
pack() (run.rs:205-345) lays out: fields indexed comp * nn + (i * n1 + j) * n2 + k, the axis
table of 10 values per node, psi slabs indexed as psi_at (fdtd.wgsl:86-92).

The set-up outputs (per-edge ca/cb, axis factors, sparse lists) come from the oracle's Sim: this
file restates the update, not Sim::try_new. Only tests import it, as a checker of the oracle.
"""
from __future__ import annotations

import ctypes
import ctypes.util
import math

import numpy as np

F = np.float32
# The shader's exp / cos / sin are GPU builtins of implementation-defined precision; the f32 libm
# functions stand in for them here, as they do in the reference's CPU path (Rust's f32 methods).
_LIBM = ctypes.CDLL(ctypes.util.find_library("m"))
for _name in ("expf", "cosf", "sinf"):
    getattr(_LIBM, _name).restype = ctypes.c_float
    getattr(_LIBM, _name).argtypes = [ctypes.c_float]


def _expf(x) -> np.float32:
    return F(_LIBM.expf(float(x)))


def _cosf(x) -> np.float32:
    return F(_LIBM.cosf(float(x)))


def _sinf(x) -> np.float32:
    return F(_LIBM.sinf(float(x)))


EPS0 = 8.854_187_812_8e-12     # sim.rs:2
MU0 = 1.256_637_062_12e-6      # sim.rs:3


def pulse_shape(fc: float):
    """sim.rs:646-649."""
    tau = math.sqrt(math.log(10.0)) / (math.pi * fc)
    return 4.0 * tau, tau


class WgslState:
    """The buffers of run.rs:205-345 for one driven port, stepped as fdtd.wgsl's kernels do."""

    def __init__(self, osim, driven: int, f0: float, fc: float, freqs=(), plane_k=None, cap: int = 0):
        n = osim.dims()
        self.n = n
        n0, n1, n2 = n
        self.nn = nn = n0 * n1 * n2
        self.sx, self.sy = n1 * n2, n2
        self.pml = int(osim.grid.pml) if hasattr(osim.grid, "pml") else 0
        self.dt = F(osim.dt)
        # coef_at (fdtd.wgsl:63-69): (ca, cb) of each E edge
        self.ca = np.zeros((3, nn), F)
        self.cb = np.zeros((3, nn), F)
        for c in range(3):
            a, b = osim.coefs(c)
            self.ca[c], self.cb[c] = a.astype(F), b.astype(F)
        # the axis table (run.rs:226-241), fields by the shader's numbering
        self.ax = [osim.axis(a) for a in range(3)]
        self.axf = [x[:, :8].astype(F) for x in self.ax]
        self.slot_e = [x[:, 8].astype(np.int64) for x in self.ax]
        self.slot_h = [x[:, 9].astype(np.int64) for x in self.ax]
        self.e = np.zeros((3, nn), F)
        self.h = np.zeros((3, nn), F)
        w = 2 * self.pml
        # psi slabs (run.rs:214-225) by (field 0 = E / 1 = H, comp, axis), shaped for psi_at
        self.psi = {}
        for fld in range(2):
            for c in range(3):
                for a in range(3):
                    if a == c or self.pml == 0:
                        continue
                    shape = [n0, n1, n2]
                    shape[a] = w
                    self.psi[(fld, c, a)] = np.zeros(shape, F)
        self.k_mu = F(osim.dt / MU0)   # run.rs:441
        t0, tau = pulse_shape(fc)
        self.t0, self.tau, self.w0 = F(t0), F(tau), F(2.0 * math.pi * f0)
        # lumped (run.rs:243-250): sources of the driven port, inductors with their running sum
        idx, val = osim.items(f"sources{driven}")
        self.src_f = (idx[:, 0] * nn + idx[:, 1]).astype(np.int64)
        self.src_v = val[:, 0].astype(F)
        idx, val = osim.items("inductors")
        self.ind_f = (idx[:, 0] * nn + idx[:, 1]).astype(np.int64)
        self.ind_ke, self.ind_ki = val[:, 0].astype(F), val[:, 1].astype(F)
        self.ind_acc = np.zeros(len(self.ind_f), F)
        # wires (run.rs:251-258): h, then (e, c) x 4
        wh, we, wc = osim.wires()
        self.w_h, self.w_e, self.w_c = wh.astype(np.int64), we.astype(np.int64), wc.astype(F)
        # sheets (run.rs:259-289): z-directed ones and k == 0 are skipped
        si, sv, table = osim.sheets()
        keep = [q for q in range(len(si)) if int(si[q, 0]) != 2 and int(si[q, 1]) % n2 != 0]
        si, sv = si[keep], sv[keep]
        comp, ident = si[:, 0].astype(np.int64), si[:, 1].astype(np.int64)
        hc = np.where(comp == 0, 1, 0)
        self.sh_f = comp * nn + ident
        self.sh_ha = hc * nn + ident
        self.sh_hb = hc * nn + ident - 1
        assert len(np.unique(self.sh_f)) == len(self.sh_f)
        self.sh_len, self.sh_c, self.sh_r = sv[:, 2].astype(F), sv[:, 3].astype(F), sv[:, 0].astype(F)
        self.sh_adaptive = sv[:, 1].astype(F)
        ns = len(self.sh_f)
        self.sh_acc = np.zeros((ns, 3), F)                 # aa, bb, ab
        self.sh_m = np.full((ns, 2), F(0.5), F)            # ma, mb
        self.sh_old = np.zeros(ns, F)
        self.sh_iold = np.zeros(ns, F)
        self.sh_face = si[:, 2:4].astype(np.int64)
        self.branch = table.astype(F)
        self.nr = int(table[0]) if len(table) >= 2 else 0
        self.nc = int(table[1]) if len(table) >= 2 else 0
        self.current = np.zeros((ns, self.nr + 2 * self.nc), F)
        # Debye (run.rs:290-301)
        idx, val = osim.items("debye")
        self.deb_f = (idx[:, 0] * nn + idx[:, 1]).astype(np.int64)
        self.deb_dd = val[:, 0].astype(F)
        self.deb_old = np.zeros(len(self.deb_f), F)
        _, poles = osim.items("poles")
        dt = osim.dt
        self.deb_b, self.deb_c = [], []
        for x, a in poles:
            d = 1.0 + 0.5 * x * dt
            self.deb_b.append(F((1.0 - 0.5 * x * dt) / d))
            self.deb_c.append(F(EPS0 * a * x / d))
        self.deb_state = np.zeros((len(self.deb_b), len(self.deb_f)), F)
        # probes (run.rs:302-340)
        self.ports = []
        for p, port in enumerate(osim.ports):
            axis = port.columns[0][0].comp
            mid = port.columns[len(port.columns) // 2]
            polarity = -1.0 if port.reference_above else 1.0
            weight = polarity / len(port.columns)
            d = self._d(axis)
            pe_id, pe_w = [], []
            for col in port.columns:
                for e in col:
                    at = e.at
                    pe_id.append(F((at[0] * n1 + at[1]) * n2 + at[2]))
                    pe_w.append(F(d[at[axis]] * weight))
            height = sum(d[e.at[axis]] for e in mid)
            lp_id, lp_c, lp_w = [], [], []
            for e in mid:
                k = e.at[axis]
                share = polarity * d[k] / height
                for ident, comp, wgt in osim.port_loop(p, axis, k):
                    lp_id.append(F(ident))
                    lp_c.append(F(3 + comp))
                    lp_w.append(F(wgt * share))
            self.ports.append((axis, np.array(pe_id, F), np.array(pe_w, F), np.array(lp_id, F), np.array(lp_c, F),
                               np.array(lp_w, F)))
        self.cap = cap
        self.series = np.zeros((cap, len(self.ports), 2), F)
        # plane DFT (fdtd.wgsl:561-585)
        self.freqs = [float(f) for f in freqs][:4]
        self.omega = [F(2.0 * math.pi * f) for f in self.freqs]
        self.plane_k = plane_k
        self.plane = np.zeros((n0 * n1, len(self.freqs), 10), F) if plane_k is not None and self.freqs else None
        self.state0 = 0          # state[0]: update_h opens step n by incrementing it

    def _d(self, a):
        return self._dline[a]

    # ---- helpers of fdtd.wgsl:71-99
    def _edge_zone(self, a, p):
        """edge_zone (fdtd.wgsl:94-96) over an index array."""
        return (p < self.pml + 1) | (p + self.pml + 2 > self.n[a])

    def _coords(self):
        n0, n1, n2 = self.n
        i, j, k = np.meshgrid(np.arange(n0), np.arange(n1), np.arange(n2), indexing="ij")
        return i.ravel(), j.ravel(), k.ravel()

    def _psi_index(self, a, i, j, k, s):
        """psi_at (fdtd.wgsl:86-92) as an index tuple into the slab of axis a."""
        if a == 0:
            return (s, j, k)
        if a == 1:
            return (i, s, k)
        return (i, j, s)

    # ---- kernels
    def wire_h(self):
        """fdtd.wgsl:452-462: h[wire] += sum over the four terms of c * E."""
        if len(self.w_h) == 0:
            return
        dh = np.zeros(len(self.w_h), F)
        ef = self.e.reshape(-1)
        for t in range(4):
            dh = dh + self.w_c[:, t] * ef[self.w_e[:, t]]
        hf = self.h.reshape(-1)
        for q in range(len(self.w_h)):      # in list order (an H may carry several wires)
            hf[self.w_h[q]] = hf[self.w_h[q]] + dh[q]

    def _curl_h(self, c, u, v, du, dv, pu, pv, sel, I, J, K):
        """curl_h (fdtd.wgsl:98-123) on the node ids `sel`."""
        e = self.e
        ev = e[v][sel + du] - e[v][sel]
        eu = e[u][sel + dv] - e[u][sel]
        t1 = ev * self.axf[u][pu, 0]
        t2 = eu * self.axf[v][pv, 0]
        if self.pml > 0:
            zone = self._edge_zone(u, pu) | self._edge_zone(v, pv)
            for (ax, p, d, tt) in ((u, pu, ev, 0), (v, pv, eu, 1)):
                s = self.slot_h[ax][p]
                m = zone & (s >= 0)
                if not m.any():
                    continue
                slab = self.psi[(1, c, ax)]
                q = self._psi_index(ax, I[m], J[m], K[m], s[m])
                new = self.axf[ax][p[m], 6] * slab[q] + self.axf[ax][p[m], 7] * d[m] * self.axf[ax][p[m], 2]
                slab[q] = new
                if tt == 0:
                    t1[m] = t1[m] + new
                else:
                    t2[m] = t2[m] + new
        self.h[c][sel] = self.h[c][sel] - self.k_mu * (t1 - t2)

    def update_h(self, coords):
        """update_h (fdtd.wgsl:171-186)."""
        self.state0 += 1
        i, j, k = coords
        n0, n1, n2 = self.n
        ids = np.arange(self.nn)
        xi, yj, zk = i + 1 < n0, j + 1 < n1, k + 1 < n2
        m = yj & zk
        self._curl_h(0, 1, 2, self.sy, 1, j[m], k[m], ids[m], i[m], j[m], k[m])
        m = zk & xi
        self._curl_h(1, 2, 0, 1, self.sx, k[m], i[m], ids[m], i[m], j[m], k[m])
        m = xi & yj
        self._curl_h(2, 0, 1, self.sx, self.sy, i[m], j[m], ids[m], i[m], j[m], k[m])

    def _curl_e(self, c, u, v, du, dv, coords):
        """curl_e / curl_of_h (fdtd.wgsl:125-156): edges with cb == 0 are left alone."""
        i, j, k = coords
        pos = {0: i, 1: j, 2: k}
        sel = np.nonzero(self.cb[c] != 0.0)[0]
        I, J, K = i[sel], j[sel], k[sel]
        pu, pv = pos[u][sel], pos[v][sel]
        h = self.h
        assert (sel - du).min(initial=0) >= 0 and (sel - dv).min(initial=0) >= 0
        hv = h[v][sel] - h[v][sel - du]
        hu = h[u][sel] - h[u][sel - dv]
        t1 = hv * self.axf[u][pu, 1]
        t2 = hu * self.axf[v][pv, 1]
        if self.pml > 0:
            zone = self._edge_zone(u, pu) | self._edge_zone(v, pv)
            for (ax, p, d, tt) in ((u, pu, hv, 0), (v, pv, hu, 1)):
                s = self.slot_e[ax][p]
                m = zone & (s >= 0)
                if not m.any():
                    continue
                slab = self.psi[(0, c, ax)]
                q = self._psi_index(ax, I[m], J[m], K[m], s[m])
                new = self.axf[ax][p[m], 4] * slab[q] + self.axf[ax][p[m], 5] * d[m] * self.axf[ax][p[m], 3]
                slab[q] = new
                if tt == 0:
                    t1[m] = t1[m] + new
                else:
                    t2[m] = t2[m] + new
        self.e[c][sel] = self.ca[c][sel] * self.e[c][sel] + self.cb[c][sel] * (t1 - t2)

    def update_e(self, coords):
        """update_e (fdtd.wgsl:188-200)."""
        self._curl_e(0, 1, 2, self.sy, 1, coords)
        self._curl_e(1, 2, 0, 1, self.sx, coords)
        self._curl_e(2, 0, 1, self.sx, self.sy, coords)

    def sheet_pre(self):
        """sheet_pre (fdtd.wgsl:333-340) with sheet_before (fdtd.wgsl:342-363)."""
        if len(self.sh_f) == 0:
            return
        ef, hf = self.e.reshape(-1), self.h.reshape(-1)
        self.sh_old = ef[self.sh_f].copy()
        ha, hb = hf[self.sh_ha], hf[self.sh_hb]
        aa = self.sh_acc[:, 0] + ha * ha
        bb = self.sh_acc[:, 1] + hb * hb
        ab = self.sh_acc[:, 2] + ha * hb
        self.sh_acc = np.stack([aa, bb, ab], axis=1)
        s = aa + bb
        go = ~(s <= F(1e-30))
        scale = np.ones(len(s), F)
        adaptive = self.sh_adaptive != 0.0
        scale = np.where(adaptive, self.sh_m[:, 0] + self.sh_m[:, 1], scale)
        total = aa + bb - F(2.0) * ab
        scale = np.where(adaptive & (total > F(1e-30)),
                         np.clip(s / np.where(total > 0, total, F(1)), F(0.5), F(4.0)), scale).astype(F)
        with np.errstate(divide="ignore", invalid="ignore"):
            ma = scale * aa / s
            mb = scale * bb / s
        self.sh_m = np.where(go[:, None], np.stack([ma, mb], axis=1), self.sh_m).astype(F)

    def sheet_post(self):
        """sheet_after (fdtd.wgsl:382-428)."""
        if len(self.sh_f) == 0:
            return
        br, nr, nc = self.branch, self.nr, self.nc
        stride = 2 + nr + 2 * nc
        faces = 4 + 2 * nr + 4 * nc
        fa = faces + self.sh_face[:, 0] * stride
        fb = faces + self.sh_face[:, 1] * stride
        ma, mb = self.sh_m[:, 0], self.sh_m[:, 1]
        cur = self.current
        hist = (ma * br[fa + 1] + mb * br[fb + 1]) * self.sh_iold
        for k in range(nr):
            hist = hist - (ma * br[fa + 2 + k] + mb * br[fb + 2 + k]) * cur[:, k]
        for k in range(nc):
            o = 2 + nr + 2 * k
            cr = ma * br[fa + o] + mb * br[fb + o]
            ci = ma * br[fa + o + 1] + mb * br[fb + o + 1]
            u = nr + 2 * k
            hist = hist - (cr * cur[:, u] - ci * cur[:, u + 1])
        a = self.sh_r * (ma * br[fa] + mb * br[fb])
        ef = self.e.reshape(-1)
        half = F(0.5) * self.sh_len
        ibar = (half * (ef[self.sh_f] + self.sh_old) + self.sh_r * hist) / (a + half * self.sh_c)
        ef[self.sh_f] = ef[self.sh_f] - self.sh_c * ibar
        self.sh_iold = F(2.0) * ibar - self.sh_iold
        for k in range(nr):
            p = 4 + 2 * k
            cur[:, k] = br[p] * cur[:, k] + br[p + 1] * ibar
        for k in range(nc):
            p = 4 + 2 * nr + 4 * k
            u = nr + 2 * k
            ur, ui = cur[:, u].copy(), cur[:, u + 1].copy()
            cur[:, u] = br[p] * ur - br[p + 1] * ui + br[p + 2] * ibar
            cur[:, u + 1] = br[p] * ui + br[p + 1] * ur + br[p + 3] * ibar

    def debye_pre(self):
        """debye_pre (fdtd.wgsl:469-474): the edge's E before the update."""
        if len(self.deb_f):
            self.deb_old = self.e.reshape(-1)[self.deb_f].copy()

    def debye_post(self):
        """debye_post / debye_after (fdtd.wgsl:476-511)."""
        if len(self.deb_f) == 0:
            return
        ef = self.e.reshape(-1)
        cb = self.cb.reshape(-1)[self.deb_f]
        s0 = np.zeros(len(self.deb_f), F)
        for k, b in enumerate(self.deb_b):
            s0 = s0 + F(0.5) * (F(1.0) + b) * self.deb_state[k]
        nxt = ef[self.deb_f] - cb * s0
        ef[self.deb_f] = nxt
        de = nxt - self.deb_old
        for k, (b, c) in enumerate(zip(self.deb_b, self.deb_c)):
            self.deb_state[k] = b * self.deb_state[k] + self.deb_dd * c * de

    def _pulse(self, t: np.float32) -> np.float32:
        """pulse (fdtd.wgsl:513-516) in f32."""
        x = (t - self.t0) / self.tau
        return F(_expf(-x * x) * _cosf(self.w0 * (t - self.t0)))

    def lumped(self):
        """lumped (fdtd.wgsl:518-545): sources of step n, then inductors."""
        n = self.state0 - 1
        ef = self.e.reshape(-1)
        t = (F(n) + F(0.5)) * self.dt
        if len(self.src_f):
            p = self._pulse(t)
            ef[self.src_f] = ef[self.src_f] - self.src_v * p
        if len(self.ind_f):
            x = ef[self.ind_f] - self.ind_ke * self.ind_acc
            ef[self.ind_f] = x
            self.ind_acc = self.ind_acc + self.ind_ki * x

    @staticmethod
    def _lane_sum(terms: np.ndarray) -> np.float32:
        """probe's sum (fdtd.wgsl:549-575): 256 lanes add strided terms, then a halving tree."""
        lanes = np.zeros(256, F)
        for q, v in enumerate(terms):
            lanes[q % 256] = lanes[q % 256] + v
        s = 128
        while s > 0:
            lanes[:s] = lanes[:s] + lanes[s:2 * s]
            s //= 2
        return lanes[0]

    def probe(self):
        n = self.state0 - 1
        if n >= self.cap:
            return
        ef, hf = self.e.reshape(-1), self.h.reshape(-1)
        nn = self.nn
        for p, (axis, pe_id, pe_w, lp_id, lp_c, lp_w) in enumerate(self.ports):
            v_terms = -(ef[axis * nn + pe_id.astype(np.int64)] * pe_w)
            i_terms = hf[(lp_c.astype(np.int64) - 3) * nn + lp_id.astype(np.int64)] * lp_w
            self.series[n, p, 0] = self._lane_sum(v_terms)
            self.series[n, p, 1] = self._lane_sum(i_terms)

    def field_dft(self):
        """field_dft (fdtd.wgsl:561-585) over the z-plane plane_k."""
        if self.plane is None:
            return
        n0, n1, n2 = self.n
        n = self.state0 - 1
        te = (F(n) + F(1.0)) * self.dt
        th = (F(n) + F(0.5)) * self.dt
        ids = (np.arange(n0 * n1) * n2 + self.plane_k).astype(np.int64)
        f = [self.e[0][ids], self.e[1][ids], self.e[2][ids], self.h[0][ids], self.h[1][ids]]
        for q, w in enumerate(self.omega):
            ce = (_cosf(w * te) * self.dt, -_sinf(w * te) * self.dt)
            ch = (_cosf(w * th) * self.dt, -_sinf(w * th) * self.dt)
            for c in range(5):
                ph = ch if c >= 3 else ce
                self.plane[:, q, 2 * c] = self.plane[:, q, 2 * c] + f[c] * ph[0]
                self.plane[:, q, 2 * c + 1] = self.plane[:, q, 2 * c + 1] + f[c] * ph[1]

    def step(self, coords, wires_after_h: bool = False):
        """One step of the separate pipeline (run.rs:627-648). The shader adds the thin-wire term
        to H before the curl update (wire_h is dispatched first); the reference's CPU path adds it
        after (cpu.rs:269-273), which rounds differently: wires_after_h takes the CPU order."""
        if not wires_after_h:
            self.wire_h()
        self.update_h(coords)
        if wires_after_h:
            self.wire_h()
        self.sheet_pre()
        self.debye_pre()
        self.update_e(coords)
        self.sheet_post()
        self.debye_post()
        self.lumped()
        self.probe()
        self.field_dft()


def run(osim, grid, driven: int, f0: float, fc: float, steps: int, freqs=(), plane_k=None,
        wires_after_h: bool = False) -> WgslState:
    """`steps` steps of the shader's separate pipeline on the oracle Sim's set-up."""
    st = WgslState.__new__(WgslState)
    # cell sizes per axis (sim.rs:29-33), for the probe weights
    st._dline = []
    for a in range(3):
        line = np.asarray(grid.axis(a), np.float64)
        nl = len(line)
        st._dline.append([line[i + 1] - line[i] if i + 1 < nl else line[i] - line[i - 1] for i in range(nl)])
    WgslState.__init__(st, osim, driven, f0, fc, freqs, plane_k, steps)
    coords = st._coords()
    for _ in range(steps):
        st.step(coords, wires_after_h)
    return st
