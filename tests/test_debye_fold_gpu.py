"""The Debye ADE folded into the TMA march (FIELDGRID_DEBYE_FOLD=1, opt-in): the folded edges'
ADE runs in the march's E half with the list kernel's arithmetic, the edges the march does not
own (shell, a tile's right-edge column) stay on the list, so fields, port series and energy equal
the unfolded run bit for bit; one case also against the oracle."""
import numpy as np
import pytest

from conftest import rel_l2
from fieldgrid_b200 import fdtd
from fieldgrid_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _run(gpu, sc, steps, fold, monkeypatch):
    monkeypatch.setenv("FIELDGRID_DEBYE_FOLD", "1" if fold else "0")
    sim = fdtd.Sim.try_new(*sc.args())
    assert sim.count("debye_edges") > 0
    s = fdtd.Session(gpu, sim, 0, sc.pulse, sc.extras)
    assert ("Debye ADE folded" in s.variant) == fold, s.variant
    nn = int(np.prod(sc.grid.dims()))
    energies = []
    for chunk in (steps // 3, steps - steps // 3):
        s.step(chunk)
        energies.append(s.energy())
    out = dict(e=s.read("e", 3 * nn), h=s.read("h", 3 * nn), series=s.read("series", steps * len(sc.ports) * 2),
               energy=np.array(energies))
    s.close()
    return out


@pytest.mark.parametrize("name,make,steps", [
    ("spheres 96^3, CPML 6", lambda: W.spheres(96, pml=6, count=30, rmin=4, rmax=14, steps=200), 101),
    ("spheres 128^3, no CPML (129-node rows)", lambda: W.spheres(128, pml=0, count=24, rmin=4, rmax=16, steps=200), 60),
])
def test_the_folded_debye_ade_equals_the_list_kernel(gpu, monkeypatch, name, make, steps):
    folded = _run(gpu, make(), steps, True, monkeypatch)
    listed = _run(gpu, make(), steps, False, monkeypatch)
    for key in ("e", "h", "series", "energy"):
        assert np.array_equal(folded[key], listed[key]), (name, key)
    assert np.abs(folded["e"]).max() > 0


def test_the_folded_run_matches_the_oracle(gpu, monkeypatch):
    sc = W.spheres(56, pml=6, count=14, rmin=3, rmax=12, steps=300)
    got = _run(gpu, sc, 300, True, monkeypatch)
    ref = O.run_cpu(O.OracleSim(*sc.args(), bits=32), 0, sc.pulse, sc.extras, keep_fields=True)
    for key in ("e", "h", "series"):
        assert rel_l2(got[key], getattr(ref, key)) <= 1e-4, key
