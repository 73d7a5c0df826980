"""The FP64 oracle's focal-series adjoint against central finite differences.

The loss is L = sum_d sum_px (|B_d psi_S|^2 - T_d)^2, with psi_S the exit wave
after S conventional slices and B_d the coherent imaging transfer at defocus
d.  Gradients are taken with respect to every potential slice (dL/dV) and to
every atom's x/y position through the potential build (dL/dxy).  Finite
differences on positions use the oracle's value-only offset, which leaves the
FP32 cut-off and bin decisions where they were, so that both sides measure
the same piecewise-smooth function."""
import numpy as np
import pytest

from cudamultislice_b200 import structures
from tests.conftest import FPARAMS


def focal_case(oracle_mod):
    Z, x, y, z = structures.srtio3(2, 2, 2)
    rng = np.random.default_rng(4)
    x = x + rng.normal(0, 0.05, x.size).astype(np.float32)
    y = y + rng.normal(0, 0.05, y.size).astype(np.float32)
    o = oracle_mod.OracleSimulation()
    o.SetAtoms(Z, x, y, z)
    o.UploadBinnedAtoms()
    o.GetParameterisation(FPARAMS)
    o.ApplyMicroscopeParameters(200.0, -500.0, 0, 0, 1e7, 0.1, 30, 20)
    o.SetCalculationVariables(0.1, -500.0, 64, 64, o.GetSizeX(), o.GetSizeY(), o.GetSizeZ(), 2.0, 2.0)
    o.PreCalculateFrequencies()
    o.InitialiseWavefunctions(1.9525)
    S = o.GetSlices(True)
    defoci = np.array([-400.0, 0.0, 300.0], np.float32)
    T = np.random.default_rng(1).random((3, 64, 64)) * 0.5 + 0.75
    return o, S, defoci, T


def test_focal_forward_matches_grad_loss(oracle_mod):
    o, S, df, T = focal_case(oracle_mod)
    L, gV, gxy = o.FocalGrad(df, T, S)
    V = np.stack([o.PotentialConventional(n) for n in range(1, S + 1)])
    L0, imgs = o.FocalForward(df, T, S, V)
    assert L0 == pytest.approx(L, rel=1e-14)
    assert np.sum((imgs - T) ** 2) == pytest.approx(L, rel=1e-12)


def test_dLdV_central_differences(oracle_mod):
    o, S, df, T = focal_case(oracle_mod)
    _, gV, _ = o.FocalGrad(df, T, S, want_xy=False)
    V = np.stack([o.PotentialConventional(n) for n in range(1, S + 1)])
    for n, yy, xx in [(0, 7, 3), (2, 10, 20), (4, 33, 33), (S - 1, 5, 50)]:
        h = 1e-3 * max(1.0, abs(V[n, yy, xx]))
        Vp = V.copy()
        Vp[n, yy, xx] += h
        Vm = V.copy()
        Vm[n, yy, xx] -= h
        fd = (o.FocalForward(df, T, S, Vp)[0] - o.FocalForward(df, T, S, Vm)[0]) / (2 * h)
        assert abs(fd - gV[n, yy, xx]) <= 1e-4 * abs(fd) + 1e-12, (n, yy, xx, fd, gV[n, yy, xx])


def test_dLdxy_central_differences(oracle_mod):
    o, S, df, T = focal_case(oracle_mod)
    _, _, gxy = o.FocalGrad(df, T, S)
    h = 1e-6
    for i in (0, 3, 7, 12):
        for ax in (0, 1):
            d = [0.0, 0.0]
            d[ax] = h
            o.SetValueOffset(i, *d)
            Lp = o.FocalForward(df, T, S)[0]
            o.SetValueOffset(i, -d[0], -d[1])
            Lm = o.FocalForward(df, T, S)[0]
            o.SetValueOffset(i, 0.0, 0.0)
            fd = (Lp - Lm) / (2 * h)
            assert abs(fd - gxy[i, ax]) <= 1e-4 * abs(fd) + 1e-9, (i, ax, fd, gxy[i, ax])


def test_dLdxy_translation_sum(oracle_mod):
    """Moving every atom by the same offset equals the sum of the per-atom
    derivatives (linearity of the chain rule)."""
    o, S, df, T = focal_case(oracle_mod)
    _, _, gxy = o.FocalGrad(df, T, S)
    n = gxy.shape[0]
    h = 1e-6
    for i in range(n):
        o.SetValueOffset(i, h, 0.0)
    Lp = o.FocalForward(df, T, S)[0]
    for i in range(n):
        o.SetValueOffset(i, -h, 0.0)
    Lm = o.FocalForward(df, T, S)[0]
    fd = (Lp - Lm) / (2 * h)
    assert abs(fd - gxy[:, 0].sum()) <= 1e-4 * abs(fd) + 1e-8
