"""The FP64 oracle against golden vectors produced by the reference itself.

tests/golden/ref_*.npz were generated by tests/golden/make_golden_ref.py,
which runs the reference engine (GUI Simulation/UnmanagedGUISimulation.cu,
compiled unchanged by oracle/ref_build.sh; string-named constant uploads
routed to their symbols) on a B200.  The reference computes in FP32 with
cuFFT, so its outputs carry FP32 rounding: integer work (the atom index) and
the FP32 set-up scalars must match bit for bit, values within the FP32 error
of a 1e-5-class computation."""
import glob
import os

import numpy as np
import pytest

from tests.conftest import FPARAMS, GOLDEN

CASES = sorted(glob.glob(os.path.join(GOLDEN, "ref_*.npz")))
# measured against the reference's outputs: RS potential 6e-7 (its FP32 vatom
# sums), CTF image 2.3e-7 (FP32 cuFFT and aberration phase), projected
# transmission 1.4e-8; the RS and CTF cases' waves 7e-8 and 2.2e-7
RS_POT_TOL = 1e-6
CTF_TOL = 1e-6
PROJ_TOL = 1e-7


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.complex128) - b) / np.linalg.norm(b))


def oracle_for(oracle_mod, g, tmp_path):
    p = str(tmp_path / "s.xyz")
    with open(p, "w") as f:
        f.write(str(g["xyz"]))
    o = oracle_mod.OracleSimulation()
    o.ImportAtoms(p, False)
    o.UploadBinnedAtoms()
    o.GetParameterisation(FPARAMS)
    o.ApplyMicroscopeParameters(*[float(v) for v in g["micro"]])
    ps, df, xoff, yoff = [float(v) for v in g["calc"]]
    nx, ny, stem = [int(v) for v in g["grid"]]
    if stem:
        o.STEMSetCalculationVariables(ps, df, nx, ny, o.GetSizeX(), o.GetSizeY(), o.GetSizeZ())
    else:
        o.SetCalculationVariables(ps, df, nx, ny, o.GetSizeX(), o.GetSizeY(), o.GetSizeZ(), xoff, yoff)
    o.PreCalculateFrequencies()
    if str(g["mode"]) == "fd":
        o.InitialiseWavefunctions()
    else:
        o.InitialiseWavefunctions(float(g["dz"]))
    if stem:
        o.AllocTDS()
        px, py = [int(v) for v in g["stem_pos"]]
        o.STEMInitialiseWavefunctions(px, py)
    return o


@pytest.mark.skipif(not CASES, reason="golden vectors not generated")
@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(c)[:-4] for c in CASES])
def test_oracle_matches_reference(oracle_mod, path, tmp_path):
    g = np.load(path)
    o = oracle_for(oracle_mod, g, tmp_path)
    # bounding box and atom index: bit-exact
    assert np.array_equal(o.Box(), g["box"])
    off, Z, x, y, z = o.Binned()
    assert np.array_equal(off, g["off"])
    assert np.array_equal(Z, g["bZ"])
    for a, b in ((x, g["bx"]), (y, g["by"]), (z, g["bz"])):
        assert np.array_equal(a, b)
    # FP32 set-up scalars: bit-exact
    sc = o.Scalars()
    ref = g["scalars"]
    assert np.float32(sc["wavel"]) == ref[0]
    assert np.float32(sc["sigma2"]) == ref[1]
    assert np.float32(sc["kmax"]) == ref[4]
    assert np.float32(sc["convdz"]) == ref[5]
    if str(g["mode"]) == "fd":
        assert np.float32(sc["dzFD"]) == ref[2] and int(sc["nFD"]) == int(ref[3])
    # values
    nsteps = int(g["nsteps"])
    for i in range(1, nsteps + 1):
        if str(g["mode"]) == "fd":
            o.MultisliceStepFD(i)
        elif str(g["mode"]) == "rs":
            key = f"rspot_{i}"
            if key in g.files:  # binnedAtomPKernelRS (U.cu:655-727), not exponentiated
                v = o.PotentialRS(i)
                assert rel_l2(g[key], v) < RS_POT_TOL, (i, rel_l2(g[key], v))
            o.MultisliceStepRS(i)
        else:
            key = f"trans_{i}"
            if key in g.files:
                t = np.exp(1j * sc["sigma2"] * o.PotentialConventional(i))
                assert rel_l2(g[key], t) < 1e-7, (i, rel_l2(g[key], t))
            o.MultisliceStepConventional(i)
    e = rel_l2(g["wave"], o.Wave())
    # measured: TEM 2-3e-7, finite differences 5e-8, STEM probe 4e-6 (the probe's
    # unnormalised inverse FFT and L1 sum run in FP32 in the reference)
    tol = 1e-5 if "tds" in g.files else 2e-6
    assert e < tol, e
    if "ctf_image" in g.files:
        # imagingKernel2 (U.cu:1044-1080): the image before the detector chain
        img = o.SimulateImage()
        e_img = rel_l2(np.abs(g["ctf_image"]) ** 2, img)
        assert e_img < CTF_TOL, e_img
    for key in (k for k in g.files if k.startswith("proj_")):
        # binnedAtomPKernel2 (U.cu:513-578) over one-angstrom z-bin b: the
        # oracle's projected slab it = b + 1 of thickness 1
        b = int(key[5:])
        t = np.exp(1j * sc["sigma2"] * o.PotentialProjected(b + 1, 1.0))
        assert rel_l2(g[key], t) < PROJ_TOL, (b, rel_l2(g[key], t))
    if "tds" in g.files:
        o.AddTDSWaves()
        assert rel_l2(g["tds"], o.TDS()) < 1e-5
    if "ew_minmax" in g.files:
        a = np.abs(o.Wave())
        assert abs(a.max() - g["ew_minmax"][1]) / a.max() < 1e-4
        assert abs(a.min() - g["ew_minmax"][0]) / max(a.min(), 1e-3) < 1e-3
