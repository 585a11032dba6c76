"""The device-side failure path of the TMA march: every mbarrier wait is bounded, and a wait that
runs out sets an error word that the run loop reads at its next energy check and turns into an
error, with the CUDA context left usable.

The failure is made the way a lost copy would look to the kernel, with no fault: a test knob
(FIELDGRID_TEST_STALL_PLANE, read when a session is created) makes the full barrier of one x-plane
expect 16 bytes more than its copies deliver, so the consumers' wait on that plane can never
complete; FIELDGRID_TEST_WAIT_NS shortens the limit from 2 s to 10 ms. The test then checks that
a fresh session on the same device runs clean and matches the oracle.
"""
import os

import pytest

from conftest import rel_l2
from fieldgrid_b200 import fdtd
from fieldgrid_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _scene():
    return W.spheres(40, pml=5, count=8, rmin=3, rmax=9, steps=20, fused=True)


def test_a_wait_that_runs_out_is_reported_and_the_device_stays_usable(gpu, monkeypatch):
    sc = _scene()
    sim = fdtd.Sim.try_new(*sc.args())
    sc.extras.check_every = 10
    monkeypatch.setenv("FIELDGRID_STEP_DEPTH", "1")
    monkeypatch.setenv("FIELDGRID_TEST_STALL_PLANE", "20")   # a plane inside the clean box
    monkeypatch.setenv("FIELDGRID_TEST_WAIT_NS", "10000000")
    s = fdtd.Session(gpu, sim, 0, sc.pulse, sc.extras)
    assert s.variant.startswith("TMA fused march"), s.variant
    s.step(4)
    with pytest.raises(fdtd.FdtdError) as info:
        s.energy()
    assert "bounded wait in the fused step ran out" in str(info.value)
    s.close()
    with pytest.raises(fdtd.FdtdError) as info:
        fdtd.run(gpu, sim, 0, sc.pulse, sc.extras)
    assert "bounded wait in the fused step ran out" in str(info.value)

    # knob off: a new session on the same device runs and matches the oracle
    monkeypatch.delenv("FIELDGRID_TEST_STALL_PLANE")
    monkeypatch.delenv("FIELDGRID_TEST_WAIT_NS")
    sc = _scene()
    sc.extras.max_steps = 60
    rec = fdtd.run(gpu, sim, 0, sc.pulse, sc.extras, keep_fields=True)
    ref = O.run_cpu(O.OracleSim(*sc.args(), bits=32), 0, sc.pulse, sc.extras, keep_fields=True)
    assert rec.steps == ref.steps == 60
    for name in ("e", "h", "series"):
        err = rel_l2(getattr(rec, name), getattr(ref, name))
        assert err <= 1e-4, (name, err)
    assert "FIELDGRID_TEST_STALL_PLANE" not in os.environ
