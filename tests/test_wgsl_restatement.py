"""The oracle (a restatement of the reference's CPU path, cpu.rs) against a second, independent
restatement of the reference's GPU shader (fdtd.wgsl, tests/wgsl_restatement.py) on the same
set-up: the E/H/CPML updates, Debye ADE, lumped sources and inductors, resistive sheets, thin
wires, port probes and plane DFT.

The two reference paths order one operation differently: the shader adds the thin-wire term to H
before the curl update (wire_h is dispatched first, run.rs:615-619 and 627-629), the CPU path
after it (cpu.rs:269-273). Taken in the CPU order, the shader's arithmetic gives the oracle's
fields bit for bit; in its own order the fields near the wires differ by rounding only. The port
series differ by rounding everywhere: the shader sums a probe in f32 over 256 lanes and a halving
tree (fdtd.wgsl:547-576)."""
import numpy as np
import pytest

from fieldgrid_b200 import workloads as W
from oracle import oracle as O
from tests import wgsl_restatement as WR


def _rel(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _both(sc, steps, wires_after_h=True):
    sc.extras.max_steps = steps
    osim = O.OracleSim(*sc.args(), bits=32)
    ref = O.run_cpu(osim, 0, sc.pulse, sc.extras, keep_fields=True)
    st = WR.run(osim, sc.grid, 0, sc.pulse.f0, sc.pulse.fc, steps, sc.extras.freqs, sc.extras.plane_k,
                wires_after_h=wires_after_h)
    st.osim = osim
    return st, ref


def _bits_equal(a, b) -> bool:
    return np.array_equal(np.asarray(a, np.float32).ravel(), np.asarray(b, np.float32).ravel())


def test_every_feature_scene_bit_for_bit_in_the_cpu_wire_order():
    """tests/fdtd.rs:43-125 re-expressed (Debye slab, PEC strip, R/L/C, two ports, adaptive
    sheets, thin wires, plane DFT at 3 and 7 GHz), 300 steps of the separate pipeline."""
    st, ref = _both(W.everything(fused=False), 300)
    assert _bits_equal(st.e, ref.e)
    assert _bits_equal(st.h, ref.h)
    assert _bits_equal(st.plane.ravel(), ref.plane)
    assert np.max(np.abs(ref.e)) > 0 and np.max(np.abs(ref.h)) > 0
    # f32 lane sums against the CPU path's sums: rounding only
    assert _rel(st.series.ravel(), ref.series) < 1e-6


def test_every_feature_scene_in_the_shader_wire_order():
    """The shader's own order: the wire term before the curl update rounds differently; the fields
    stay within f32 rounding of the CPU path's (the bar is the parity bar of this project)."""
    st, ref = _both(W.everything(fused=False), 300, wires_after_h=False)
    assert not _bits_equal(st.h, ref.h)
    assert _rel(st.e, ref.e) < 1e-5
    assert _rel(st.h, ref.h) < 1e-4
    assert _rel(st.series.ravel(), ref.series) < 1e-5
    assert _rel(st.plane.ravel(), ref.plane) < 1e-5


@pytest.mark.parametrize("scene", ["box", "spheres"])
def test_cpml_and_debye_scenes_bit_for_bit(scene):
    """A CPML-heavy dielectric box (6-cell layer on a 24^3 grid, every CPML slab in use) and Debye
    spheres with a CPML: no wires, so the shader's order is the CPU path's."""
    if scene == "box":
        sc = W.dielectric_box(24, pml=6, steps=160, fused=False)
    else:
        sc = W.spheres(24, pml=4, count=5, rmin=2, rmax=5, steps=160, fused=False)
    st, ref = _both(sc, 160, wires_after_h=False)
    if scene == "spheres":
        assert st.osim.count("debye_edges") > 0
    assert _bits_equal(st.e, ref.e)
    assert _bits_equal(st.h, ref.h)
    assert np.max(np.abs(ref.e)) > 0
    assert _rel(st.series.ravel(), ref.series) < 1e-6
