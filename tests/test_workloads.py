"""Host-side checks of the adjoint workloads and of the batched-gradient call's argument handling
(no GPU needed)."""
import numpy as np
import pytest

from fieldgrid_b200 import fdtd
from fieldgrid_b200 import workloads as W


def test_batch_flux_clears_the_design_block_and_keeps_the_source_out():
    jobs = W.batch_flux(count=8, lo=32, hi=64, pml=4, steps=10, checkpoints=2, design=8)
    for scene, spec, eps0, sig0 in jobs:
        sc = scene()
        dims = sc.info["dims"]
        lo, hi = spec.design_lo, spec.design_hi
        assert eps0.shape == sig0.shape == tuple(h - l for l, h in zip(lo, hi))
        deb = sc.mats.debye.reshape(dims)
        margin = tuple(slice(l - 1, h + 1) for l, h in zip(lo, hi))
        assert not deb[margin].any()                        # no Debye edge reaches the design edges
        box = tuple(slice(l, h) for l, h in zip(lo, hi))
        assert np.array_equal(sc.mats.eps.reshape(dims)[box], eps0)
        at = sc.ports[0].columns[0][0].at
        assert not all(l - 2 <= a <= h + 1 for a, l, h in zip(at, lo, hi))   # source outside the cleared box
        assert hi[2] < spec.plane_k < dims[2] - 4
        fdtd.Sim.try_new(*sc.args())                         # the scene builds


def test_flux_design_debye_slab_sits_beside_the_block():
    scene, spec, _, _ = W.flux_design(24, 24, 24, pml=4, design=(4, 4, 3), steps=10, debye=True)
    sc = scene()
    deb = sc.mats.debye.reshape(24, 24, 24)
    assert deb.sum() > 0
    i = np.nonzero(deb.any(axis=(1, 2)))[0]
    assert i.max() < spec.design_lo[0] - 1                 # a cell of vacuum between slab and block


def test_the_batched_gradient_needs_a_gpu():
    scene, spec, _, _ = W.flux_design(24, 24, 24, pml=4, design=(4, 4, 3), steps=10)
    sc = scene()
    with pytest.raises(fdtd.FdtdError, match="no GPU"):
        fdtd.flux_gradient_batch(None, [fdtd.Sim.try_new(*sc.args())], [sc.pulse], [spec])
