"""The two-step mode: two time steps per x-sweep over the interior tiles (stencil_tb2.cuh), beside
the one-step kernels on the tiles near ports, probes and the CPML's x/y layers, with the z-slab psi
and the Debye state in three time slots. Each node's update is the one-step kernels' arithmetic in
the same order, so a run in this mode must give the one-step run's fields, port series and energy
bit for bit (FIELDGRID_STEP_DEPTH=2 asks for the mode, 1 for the one-step kernels alone), at odd
and even step counts, with and without a CPML, with Debye media, and on a grid whose last tile
owns the extra column of a 64 t + 1 row. One case is also checked against the oracle."""
import numpy as np
import pytest

from conftest import rel_l2
from fieldgrid_b200 import fdtd
from fieldgrid_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _run(gpu, sc, steps, one_step, monkeypatch):
    monkeypatch.setenv("FIELDGRID_STEP_DEPTH", "1" if one_step else "2")
    sim = fdtd.Sim.try_new(*sc.args())
    s = fdtd.Session(gpu, sim, 0, sc.pulse, sc.extras)
    variant = s.variant
    nn = int(np.prod(sc.grid.dims()))
    done = 0
    energies = []
    for chunk in (steps // 3, steps - steps // 3):   # two chunks: graphs of several phases
        s.step(chunk)
        done += chunk
        energies.append(s.energy())
    out = dict(e=s.read("e", 3 * nn), h=s.read("h", 3 * nn), series=s.read("series", done * len(sc.ports) * 2),
               energy=np.array(energies))
    s.close()
    return variant, out


CASES = [
    ("spheres 96^3, CPML 6, Debye", lambda: W.spheres(96, pml=6, count=30, rmin=4, rmax=14, steps=200), 101),
    ("spheres 96^3, no CPML", lambda: W.spheres(96, pml=0, count=30, rmin=4, rmax=14, steps=200), 60),
    ("dielectric box 128^3 (129-node rows), source and probes", lambda: W.dielectric_box(128, steps=200), 77),
]


@pytest.mark.parametrize("name,make,steps", CASES, ids=[c[0] for c in CASES])
def test_two_step_mode_equals_one_step_bit_for_bit(gpu, monkeypatch, name, make, steps):
    v2, two = _run(gpu, make(), steps, False, monkeypatch)
    v1, one = _run(gpu, make(), steps, True, monkeypatch)
    print(f"{name}: {v2}")
    assert v2.startswith("two-step march"), v2
    assert not v1.startswith("two-step march"), v1
    for key in ("e", "h", "series", "energy"):
        a, b = two[key], one[key]
        assert a.shape == b.shape, key
        diff = int(np.count_nonzero(a != b))
        assert diff == 0, (name, key, diff, float(np.max(np.abs(a - b))))


def test_two_step_mode_matches_the_oracle(gpu, monkeypatch):
    sc = W.spheres(96, pml=6, count=30, rmin=4, rmax=14, steps=150)
    monkeypatch.setenv("FIELDGRID_STEP_DEPTH", "2")
    sim = fdtd.Sim.try_new(*sc.args())
    rec = fdtd.run(gpu, sim, 0, sc.pulse, sc.extras, keep_fields=True)
    ref = O.run_cpu(O.OracleSim(*sc.args(), bits=32), 0, sc.pulse, sc.extras, keep_fields=True)
    assert rec.steps == ref.steps == 150
    for name in ("e", "h", "series"):
        err = rel_l2(getattr(rec, name), getattr(ref, name))
        print(f"two-step vs oracle {name}: {err:.2e}")
        assert err <= 1e-4, (name, err)
