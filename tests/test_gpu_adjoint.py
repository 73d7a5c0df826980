"""The differentiable focal series on the GPU (ms_focal_series /
ms_focal_series_grad) against the FP64 oracle.

The oracle's own gradient is pinned to FP64 central finite differences in
tests/test_oracle_adjoint.py, so agreement here within 1e-4 puts the engine's
FP32 adjoint within 1e-4 of finite differences.  Loss and images: the 1e-5
exit-wave tolerance.  Gradients are compared norm-wise (relative L2 over all
slices, all atoms), which is the error of a gradient step."""
import numpy as np
import pytest

from tests.conftest import FPARAMS

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def engine_cls():
    from cudamultislice_b200 import ManagedMultisliceSimulation, build

    build.build(verbose=False)
    return ManagedMultisliceSimulation


def focal_pair(engine_cls, oracle_mod, nc=2, nzc=2, n=64, ps=0.1, seed=4, kV=200.0):
    """SrTiO3 with small seeded position errors (atoms away from the cut-off
    and clamp kinks), and random targets around 1."""
    from cudamultislice_b200 import structures

    Z, x, y, z = structures.srtio3(nc, nc, nzc)
    rng = np.random.default_rng(seed)
    x = (x + rng.normal(0, 0.05, x.size)).astype(np.float32)
    y = (y + rng.normal(0, 0.05, y.size)).astype(np.float32)
    eng = engine_cls()
    orc = oracle_mod.OracleSimulation()
    for s in (eng, orc):
        s.SetAtoms(Z, x, y, z)
        s.UploadBinnedAtoms()
        s.GetParameterisation(FPARAMS)
        s.ApplyMicroscopeParameters(kV, -500.0, 0.0, 0.0, 1e7, 0.1, 30.0, 20.0)
        s.SetCalculationVariables(ps, -500.0, n, n, s.GetSizeX(), s.GetSizeY(), s.GetSizeZ(), 2.0, 2.0)
        s.PreCalculateFrequencies()
        s.InitialiseWavefunctions(1.9525)
    S = orc.GetSlices(True)
    assert eng.GetSlices(True) == S
    return eng, orc, S


def targets(nd, n, seed=1):
    return (np.random.default_rng(seed).random((nd, n, n)) * 0.5 + 0.75).astype(np.float32)


DEFOCI = np.array([-400.0, 0.0, 300.0], np.float32)


def test_focal_series_forward(engine_cls, oracle_mod):
    eng, orc, S = focal_pair(engine_cls, oracle_mod)
    T = targets(3, 64)
    L, imgs = eng.FocalSeries(DEFOCI, T, S, images=True)
    L0, imgs0 = orc.FocalForward(DEFOCI, T.astype(np.float64), S)
    assert abs(L - L0) / L0 < 1e-5, (L, L0)
    for d in range(3):
        assert rel_l2(imgs[d], imgs0[d]) < 1e-5
    # fewer slices than the structure holds
    L2 = eng.FocalSeries(DEFOCI, T, S - 2)
    L20, _ = orc.FocalForward(DEFOCI, T.astype(np.float64), S - 2)
    assert abs(L2 - L20) / L20 < 1e-5


def test_focal_series_gradient_vs_oracle(engine_cls, oracle_mod):
    eng, orc, S = focal_pair(engine_cls, oracle_mod)
    T = targets(3, 64)
    L, gV, gxy = eng.FocalSeriesGrad(DEFOCI, T, S)
    L0, gV0, gxy0 = orc.FocalGrad(DEFOCI, T.astype(np.float64), S)
    assert abs(L - L0) / L0 < 1e-5
    assert rel_l2(gV, gV0) < GRAD_TOL, rel_l2(gV, gV0)
    for k in range(S):
        assert rel_l2(gV[k], gV0[k]) < 3 * GRAD_TOL, (k, rel_l2(gV[k], gV0[k]))
    assert rel_l2(gxy, gxy0) < GRAD_TOL, rel_l2(gxy, gxy0)


@pytest.mark.parametrize("mode", [1, 2])
def test_focal_gradient_both_potential_sums(engine_cls, oracle_mod, mode):
    """The gradient through the per-sub-plane potential (and its per-sub-plane
    adjoint) and through the separable one (and its adjoint) both match the
    oracle, and each other to well inside the tolerance."""
    eng, orc, S = focal_pair(engine_cls, oracle_mod, nc=3, nzc=3, n=128, ps=0.09, seed=6)
    T = targets(3, 128, seed=5)
    eng.SetPotentialSum(mode)
    L, gV, gxy = eng.FocalSeriesGrad(DEFOCI, T, S)
    assert eng.PotentialSum()[0] == mode
    L0, gV0, gxy0 = orc.FocalGrad(DEFOCI, T.astype(np.float64), S)
    assert abs(L - L0) / L0 < 1e-5
    assert rel_l2(gV, gV0) < GRAD_TOL, rel_l2(gV, gV0)
    assert rel_l2(gxy, gxy0) < GRAD_TOL, rel_l2(gxy, gxy0)
    eng.SetPotentialSum(3 - mode)
    L1, gV1, gxy1 = eng.FocalSeriesGrad(DEFOCI, T, S)
    assert rel_l2(gxy, gxy1) < GRAD_TOL / 2, rel_l2(gxy, gxy1)
    assert rel_l2(gV, gV1) < GRAD_TOL / 2, rel_l2(gV, gV1)


@pytest.mark.parametrize("stride", [1, 2, 4, 0, 1000])
def test_checkpoint_strides_agree(engine_cls, oracle_mod, stride):
    """Every checkpoint stride recomputes the same waves: results agree with
    the single-segment run and with the oracle."""
    eng, orc, S = focal_pair(engine_cls, oracle_mod)
    T = targets(3, 64)
    eng.SetCheckpoint(1000)
    ref = eng.FocalSeriesGrad(DEFOCI, T, S)
    eng.SetCheckpoint(stride)
    L, gV, gxy = eng.FocalSeriesGrad(DEFOCI, T, S)
    # the loss and the atom gradient are FP64 atomic sums: order-dependent in the last bits
    assert L == pytest.approx(ref[0], rel=1e-12)
    assert rel_l2(gV, ref[1]) < 1e-6
    assert rel_l2(gxy, ref[2]) < 1e-6


def test_focal_gradient_larger_grid(engine_cls, oracle_mod):
    """128^2, 4x4 cells in xy, 8 defoci of a -80..+60 nm series, 200 kV."""
    eng, orc, S = focal_pair(engine_cls, oracle_mod, nc=4, nzc=3, n=128, ps=0.13, seed=9)
    df = np.linspace(-800.0, 600.0, 8).astype(np.float32)
    T = targets(8, 128, seed=3)
    L, gV, gxy = eng.FocalSeriesGrad(df, T, S)
    L0, gV0, gxy0 = orc.FocalGrad(df, T.astype(np.float64), S)
    assert abs(L - L0) / L0 < 1e-5
    assert rel_l2(gV, gV0) < GRAD_TOL, rel_l2(gV, gV0)
    assert rel_l2(gxy, gxy0) < GRAD_TOL, rel_l2(gxy, gxy0)


def test_focal_gradient_only_atoms(engine_cls, oracle_mod):
    """dL/dxy without dL/dV (per-slice scratch) equals the full run's."""
    eng, orc, S = focal_pair(engine_cls, oracle_mod)
    T = targets(3, 64)
    full = eng.FocalSeriesGrad(DEFOCI, T, S)
    L, gV, gxy = eng.FocalSeriesGrad(DEFOCI, T, S, want_v=False)
    assert gV is None and L == pytest.approx(full[0], rel=1e-12)
    assert rel_l2(gxy, full[2]) < 1e-9


def test_focal_series_errors(engine_cls, oracle_mod):
    from cudamultislice_b200 import MultisliceError

    eng, orc, S = focal_pair(engine_cls, oracle_mod)
    T = targets(3, 64)
    with pytest.raises(MultisliceError):
        eng.FocalSeries(DEFOCI, T, S + 1)
    with pytest.raises(MultisliceError):
        eng.FocalSeries(DEFOCI, T, 0)
    with pytest.raises(MultisliceError):
        eng.FocalSeries(np.array([np.nan, 0, 0], np.float32), T, S)
    eng.SetSlicePath(1)
    with pytest.raises(MultisliceError):
        eng.FocalSeriesGrad(DEFOCI, T, S)
    eng.SetSlicePath(0)
    eng.SetPotentialMode(True)
    with pytest.raises(MultisliceError):
        eng.FocalSeriesGrad(DEFOCI, T, S)
    # dL/dV alone is available for the projected potential
    L, gV, gxy = eng.FocalSeriesGrad(DEFOCI, T, S, want_xy=False)
    assert np.isfinite(L) and np.all(np.isfinite(gV))
