"""Full-size parity: the CUDA engine against the oracle at the benchmark configurations' full sizes
and step counts, through committed fixtures (tests/golden/make_fullsize.py ran the oracle in f32,
the reference's arithmetic, and in f64, the FP64 truth run of the same update, and kept the port
series, every field component's L2 norm, the fields at 8192 seeded nodes, samples of the plane DFT
or NTFF accumulators and, for the antenna, the far field on the 5-degree grid).

The bar: relative L2 at most 1e-4 against the oracle's f32 run on fields,
series, accumulators and far field, after the full step count. Each case also prints the error of
the GPU run and of the oracle's f32 run against the f64 run (the per-configuration error
statement)."""
import os

import numpy as np
import pytest

from conftest import rel_l2
from fieldgrid_b200 import fdtd
from fieldgrid_b200 import workloads as W

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-4


def _fixture(name):
    return np.load(os.path.join(HERE, "golden", f"{name}.npz"))


def _scene(name):
    if name == "spheres512":
        return W.spheres(512), None
    if name == "patch256":
        return W.patch_antenna(), 3
    scene, _spec, _e, _s = W.flux_design()
    return scene(), None


def _compare(name, gpu):
    fx = _fixture(name)
    sc, inset = _scene(name)
    sc.extras.max_steps = int(fx["steps"])
    sim = fdtd.Sim.try_new(*sc.args())
    patches = None
    if inset is not None:
        patches = fdtd.patches(sim, inset)
        sc.extras.ntff = patches.gpu
    rec = fdtd.run(gpu, sim, 0, sc.pulse, sc.extras, keep_fields=True)
    assert rec.steps == int(fx["steps"])
    nn = int(np.prod(sc.grid.dims()))
    idx = fx["idx"]
    got = {"series": rec.series}
    norms = []
    for which in ("e", "h"):
        a = np.asarray(getattr(rec, which)).reshape(3, nn)
        norms += [float(np.linalg.norm(a[c].astype(np.float64))) for c in range(3)]
        got[which] = a[:, idx]
    got["norms"] = np.array(norms)
    if "plane32" in fx:
        got["plane"] = np.asarray(rec.plane)[fx["plane_idx"]]
    if "ntff32" in fx:
        got["ntff"] = np.asarray(rec.ntff)[fx["ntff_idx"]]
        import tests_far_dirs as D
        far = []
        for k, f in enumerate(fx["freqs"]):
            fl = fdtd.Far.load(patches, rec.ntff, len(fx["freqs"]), k, float(f), gpu=gpu)
            far.append(fl.fields(D.far_dirs()))
        got["far"] = np.stack(far)
    rows = []
    for key in got:
        e32 = rel_l2(got[key], fx[key + "32"])
        e64 = rel_l2(got[key], fx[key + "64"])
        o64 = rel_l2(fx[key + "32"], fx[key + "64"])
        rows.append((key, e32, e64, o64))
        print(f"{name} {key}: gpu vs oracle-f32 {e32:.2e}, gpu vs oracle-f64 {e64:.2e}, oracle-f32 vs f64 {o64:.2e}")
    for key, e32, _e64, _o64 in rows:
        assert e32 <= TOL, (name, key, e32)


@pytest.mark.parametrize("name", [n for n in ("flux160", "spheres512", "patch256")
                                  if os.path.exists(os.path.join(HERE, "golden", f"{n}.npz"))])
def test_full_size_run_matches_the_oracle(gpu, name):
    _compare(name, gpu)
