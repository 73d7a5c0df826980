"""Parity of the CUDA engine (through the C ABI) against the FP64 oracle.

Bit-exact for the integer work (atom index); for the floating-point path the
parity tolerance: relative L2 error <= 1e-5 against FP64 for potentials,
exit waves, images and detector signals."""
import numpy as np
import pytest

from tests.conftest import FPARAMS

pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative L2 error against the FP64 oracle


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.complex128) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def engine_cls():
    from cudamultislice_b200 import ManagedMultisliceSimulation, build

    build.build(verbose=False)
    return ManagedMultisliceSimulation


def make_pair(engine_cls, oracle_mod, atoms, n, ps, *, kV=200.0, df=-500.0, Cs=1e7, ap=20.0, beta=0.1,
              delta=30.0, dz=1.9525, xoff=2.0, yoff=2.0, path=0, stem=False, A2=0.0, phi2=0.0):
    Z, x, y, z = atoms
    eng = engine_cls()
    eng.SetSlicePath(path)
    orc = oracle_mod.OracleSimulation()
    for s in (eng, orc):
        s.SetAtoms(Z, x, y, z)
        s.UploadBinnedAtoms()
        s.GetParameterisation(FPARAMS)
        s.ApplyMicroscopeParameters(kV, df, A2, phi2, Cs, beta, delta, ap)
        if stem:
            s.STEMSetCalculationVariables(ps, df, n, n, s.GetSizeX(), s.GetSizeY(), s.GetSizeZ())
        else:
            s.SetCalculationVariables(ps, df, n, n, s.GetSizeX(), s.GetSizeY(), s.GetSizeZ(), xoff, yoff)
        s.PreCalculateFrequencies()
        if not stem:
            s.InitialiseWavefunctions(dz)
    return eng, orc


def sto(nc=2, nz=4):
    from cudamultislice_b200 import structures as S

    return S.srtio3(nc, nc, nz)


# ---------------------------------------------------------------- atom index
@pytest.mark.parametrize("kind", ["random", "srtio3", "tds"])
def test_atom_index_bit_exact(engine_cls, oracle_mod, kind):
    from cudamultislice_b200 import structures as S

    atoms = S.random_atoms(5000, size=(23.0, 17.0, 31.0), seed=11) if kind == "random" else S.srtio3(4, 4, 20)
    eng = engine_cls()
    orc = oracle_mod.OracleSimulation()
    for s in (eng, orc):
        s.SetAtoms(*atoms)
    if kind == "tds":
        eng.UploadBinnedAtomsTDS(0x5EED2026, 3, 0.076)
        orc.UploadBinnedAtomsTDS(0x5EED2026, 3, 0.076)
    else:
        eng.UploadBinnedAtoms()
        orc.UploadBinnedAtoms()
    a, b = eng.Binned(), orc.Binned()
    for u, v in zip(a, b):
        assert u.dtype == v.dtype and np.array_equal(u, v)


def test_atom_index_large(engine_cls, oracle_mod):
    # many atoms per bin and a deep stack: ordering inside bins must be stable
    from cudamultislice_b200 import structures as S

    atoms = S.random_atoms(200000, size=(8.0, 8.0, 40.0), seed=12)
    eng, orc = engine_cls(), oracle_mod.OracleSimulation()
    for s in (eng, orc):
        s.SetAtoms(*atoms)
        s.UploadBinnedAtoms()
    for u, v in zip(eng.Binned(), orc.Binned()):
        assert np.array_equal(u, v)


# ---------------------------------------------------------------- FFT
@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("shape", [(64, 64), (128, 256), (512, 512), (1024, 1024), (256, 64), (1024, 512),
                                   (2048, 2048), (64, 2048), (4096, 4096), (64, 4096), (4096, 256)])
def test_fused_fft_against_numpy(engine_cls, shape, variant):
    rng = np.random.default_rng(7)
    a = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    eng = engine_cls()
    eng.SetFFTPlan(variant)
    for sign, ref in ((-1, np.fft.fft2(a.astype(np.complex128))),
                      (+1, np.fft.ifft2(a.astype(np.complex128)) * a.size)):
        out = eng.FFT2(a, sign)
        assert rel_l2(out, ref) < 1e-6, (shape, sign, variant, rel_l2(out, ref))


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5])
def test_exit_wave_every_fft_plan(engine_cls, oracle_mod, variant):
    eng, orc = make_pair(engine_cls, oracle_mod, sto(2, 4), 256, 0.05)
    eng.SetFFTPlan(variant)
    eng.RunConventional()
    psi = orc.run_conventional()
    assert rel_l2(eng.ExitWave(), psi) < TOL


# ---------------------------------------------------------------- potentials
@pytest.mark.parametrize("tile", [0, 1, 2])
def test_potential_tile_shapes(engine_cls, oracle_mod, tile):
    """Every tile shape of the conventional potential kernel (32x8, 16x16, 64x4)
    gives the oracle's potential; the shapes differ only in summation order."""
    from cudamultislice_b200 import structures as S

    atoms = S.random_atoms(3000, size=(30.0, 27.0, 12.0), seed=21)
    eng, orc = make_pair(engine_cls, oracle_mod, atoms, 256, 0.12)
    eng.SetPotentialTile(tile)
    for it in (3, 5):
        v = eng.PotentialSlice(0, it)
        ref = orc.PotentialConventional(it)
        assert rel_l2(v, ref) < 1e-6, (tile, it, rel_l2(v, ref))
    eng.SetPotentialTile(-1)  # tuned
    assert rel_l2(eng.PotentialSlice(0, 5), orc.PotentialConventional(5)) < 1e-6


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_potential_slices(engine_cls, oracle_mod, kind):
    eng, orc = make_pair(engine_cls, oracle_mod, sto(2, 4), 128, 0.1)
    for it in (2, 4, 6):  # slab 1 lies in the 2 A box padding
        v = eng.PotentialSlice(kind, it)
        ref = {0: orc.PotentialConventional, 1: orc.PotentialFD,
               2: lambda i: orc.PotentialProjected(i, 1.9525)}[kind](it)
        assert np.abs(ref).max() > 0
        e = np.linalg.norm(v - ref) / np.linalg.norm(ref)
        assert e < TOL, (kind, it, e)
        assert np.abs(v - ref).max() / np.abs(ref).max() < 5 * TOL


# ---------------------------------------------------------------- TEM exit wave
@pytest.mark.parametrize("path", [0, 1])
def test_exit_wave_conventional(engine_cls, oracle_mod, path):
    eng, orc = make_pair(engine_cls, oracle_mod, sto(2, 5), 128, 0.1, path=path)
    S = eng.GetSlices(True)
    assert S == orc.GetSlices(True)
    for i in range(1, S + 1):
        eng.MultisliceStepConventional(i)
        orc.MultisliceStepConventional(i)
    e = rel_l2(eng.ExitWave(), orc.Wave())
    assert e < TOL, e


@pytest.mark.parametrize("n", [128, 256])
def test_band_limit_decisions_match_plain_path(engine_cls, oracle_mod, n):
    """The fused column pass keeps k by comparing k^2 with thresholds derived
    from kmax; the plain path keeps sqrtf(k^2) < kmax (CreatePropsKernel).  One
    propagation step on each path must keep the same frequencies: their exit
    waves' spectra agree to rounding everywhere, band edge included."""
    specs = []
    for path in (0, 1):
        eng, _ = make_pair(engine_cls, oracle_mod, sto(2, 2), n, 0.1, path=path)
        eng.MultisliceStepConventional(1)
        specs.append(np.abs(np.fft.fft2(eng.ExitWave().astype(np.complex128))))
    top = specs[1].max()
    kept = specs[1] > 1e-4 * top
    assert kept.sum() > 0 and not kept.all()
    # a frequency kept on one path and dropped on the other would differ by its
    # full amplitude; rounding moves the spectra by about 1e-6 of the maximum
    assert np.abs(specs[0] - specs[1]).max() < 1e-5 * top


def test_run_after_new_atoms_matches_fresh_engine(engine_cls, oracle_mod):
    """RunConventional after SetAtoms + UploadBinnedAtoms (same grid and slice
    count: the slice-loop graph is reused over the rebuilt potential stack)
    equals a fresh engine's run on the new atoms; ExitWave(out=...) fills the
    caller's buffer."""
    Z, x, y, z = sto(2, 5)
    eng, _ = make_pair(engine_cls, oracle_mod, (Z, x, y, z), 128, 0.1)
    eng.SetFFTPlan(3)  # both engines on one plan: bit-identical arithmetic
    eng.RunConventional()
    first = eng.ExitWave()
    inner = (x > x.min() + 0.2) & (x < x.max() - 0.2)  # the box stays as it was
    x2 = np.where(inner, x + np.float32(0.05), x).astype(np.float32)
    eng.SetAtoms(Z, x2, y, z)
    eng.UploadBinnedAtoms()
    eng.InitialiseWavefunctions(1.9525)
    eng.RunConventional()
    buf = np.zeros((128, 128), np.complex64)
    got = eng.ExitWave(out=buf)
    assert got is buf
    fresh, _ = make_pair(engine_cls, oracle_mod, (Z, x2, y, z), 128, 0.1)
    fresh.SetFFTPlan(3)
    fresh.RunConventional()
    assert np.array_equal(buf, fresh.ExitWave())
    assert not np.array_equal(buf, first)
    with pytest.raises(ValueError):
        eng.ExitWave(out=np.zeros((64, 128), np.complex64))


def test_exit_wave_c1_srtio3_256(engine_cls, oracle_mod):
    # SrTiO3 4x4x20 cells, 256^2 over 15.62 A, 1.9525 A slices, 200 kV
    eng, orc = make_pair(engine_cls, oracle_mod, sto(4, 20), 256, 15.62 / 256)
    nslices = eng.RunConventional()
    psi = orc.run_conventional()
    assert nslices == orc.GetSlices(True)
    e = rel_l2(eng.ExitWave(), psi)
    assert e < TOL, e
    # CTF image (Cs = 1 mm, df = -50 nm, 20 mrad)
    eng.SimulateImage(0.0)
    img = orc.SimulateImage()
    assert rel_l2(eng.Image(), img) < TOL


@pytest.mark.parametrize("n", [128, 512, 1024])
def test_run_with_build_overlap(engine_cls, oracle_mod, n):
    """A run whose potential stack must be built overlaps each slice's passes
    with the next slices' potentials (default); it equals the build-first run
    and the oracle, and leaves the stack resident: later runs replay the
    persistent loop (one launch on 512^2 and 1024^2 once the loop variant is
    tuned, in the first of them)."""
    atoms = sto(4, 6)
    ps = 3.905 * 4 / n
    waves = {}
    for overlap in (True, False):
        eng, orc = make_pair(engine_cls, oracle_mod, atoms, n, ps)
        eng.SetBuildOverlap(overlap)
        S = eng.RunConventional()
        waves[overlap] = eng.ExitWave()
        if overlap:
            psi = orc.run_conventional()
            assert S == orc.GetSlices(True)
            assert rel_l2(waves[True], psi) < TOL
            for rep in range(2):
                eng.InitialiseWavefunctions(1.9525)
                l0 = eng.LaunchCount()
                eng.RunConventional()
                if n >= 512 and rep == 1:
                    assert eng.LaunchCount() - l0 == 1
                assert rel_l2(eng.ExitWave(), psi) < TOL
        eng.close()
        orc.close()
    assert rel_l2(waves[True], waves[False]) < 3e-6


def test_stack_builds_bit_identical(engine_cls, oracle_mod):
    """The potential stack's slices are built on three streams (in a run with
    a stack to build, beside the slice passes on another).  With one FFT plan forced (the same per-pass kernels everywhere),
    the step-by-step run (one slice potential at a time on the handle's
    stream), the overlapped run, the build-first run and the overlapped run
    after re-uploading the atoms give bit-identical exit waves."""
    from cudamultislice_b200 import structures as S

    atoms = S.amorphous_carbon((25.0, 25.0, 40.0), density=0.1, min_sep=1.2)
    n = 512
    waves = []
    for mode in ("steps", "overlap", "build_first"):
        eng, orc = make_pair(engine_cls, oracle_mod, atoms, n, 25.0 / n, kV=300.0, dz=2.0)
        orc.close()
        eng.SetFFTPlan(3)
        eng.SetPotentialTile(0)
        eng.SetBuildOverlap(mode == "overlap")
        if mode == "steps":
            for i in range(1, eng.GetSlices(True) + 1):
                eng.MultisliceStepConventional(i)
        else:
            eng.RunConventional()
        waves.append(eng.ExitWave())
        if mode == "overlap":
            for _ in range(2):
                eng.SetAtoms(*atoms)
                eng.UploadBinnedAtoms()
                eng.InitialiseWavefunctions(2.0)
                eng.RunConventional()
                waves.append(eng.ExitWave())
        eng.close()
    for w in waves[1:]:
        assert np.array_equal(w, waves[0])


def test_run_equals_step_loop(engine_cls, oracle_mod):
    eng, _ = make_pair(engine_cls, oracle_mod, sto(2, 5), 256, 0.05)
    S = eng.GetSlices(True)
    for i in range(1, S + 1):
        eng.MultisliceStepConventional(i)
    w1 = eng.ExitWave()
    eng.InitialiseWavefunctions(1.9525)
    eng.RunConventional()
    w2 = eng.ExitWave()
    assert rel_l2(w2, w1.astype(np.complex128)) < 1e-6


def test_fused_and_plain_agree(engine_cls, oracle_mod):
    a, _ = make_pair(engine_cls, oracle_mod, sto(2, 5), 256, 0.05, path=0)
    b, _ = make_pair(engine_cls, oracle_mod, sto(2, 5), 256, 0.05, path=1)
    a.RunConventional()
    b.RunConventional()
    assert rel_l2(a.ExitWave(), b.ExitWave().astype(np.complex128)) < 2 * TOL


@pytest.mark.parametrize("path", [0, 1])
def test_ctf_image(engine_cls, oracle_mod, path):
    eng, orc = make_pair(engine_cls, oracle_mod, sto(2, 3), 128, 0.1, path=path, A2=30.0, phi2=0.4)
    S = eng.GetSlices(True)
    for i in range(1, S + 1):
        eng.MultisliceStepConventional(i)
        orc.MultisliceStepConventional(i)
    eng.AllocHostImage()
    eng.SimulateImage(1000.0)
    ref = orc.SimulateImage()
    assert rel_l2(eng.Image(), ref) < TOL
    assert abs(eng.GetImMax() - ref.max()) / ref.max() < TOL
    assert eng.GetImValue(3, 5) == pytest.approx(ref[5, 3], rel=1e-4)
    c = eng.GetImageContrast(0, 0, 64, 64)
    assert c == pytest.approx(ref[:64, :64].std(), rel=1e-4)


# ---------------------------------------------------------------- STEM
@pytest.mark.parametrize("path", [0, 1])
def test_stem_probe_cbed_and_haadf(engine_cls, oracle_mod, path):
    eng, orc = make_pair(engine_cls, oracle_mod, sto(2, 3), 128, 0.1, kV=300.0, df=0.0, Cs=0.0, ap=25.0,
                         stem=True, path=path)
    eng.AllocTDS()
    orc.AllocTDS()
    for s in (eng, orc):
        s.STEMInitialiseWavefunctions(40, 70)
    S = eng.GetSlices(True)
    for i in range(1, S + 1):
        eng.MultisliceStepConventional(i)
        orc.MultisliceStepConventional(i)
    assert rel_l2(eng.ExitWave(), orc.Wave()) < TOL
    eng.AddTDSWaves()
    orc.AddTDSWaves()
    assert rel_l2(eng.TDS(), orc.TDS()) < TOL
    # a ring inside this grid's band limit (kmax ~ 2.5/A ~ 49 mrad at 300 kV)
    h_e, h_o = eng.AnnularDetector(10.0, 40.0), orc.AnnularDetector(10.0, 40.0)
    assert h_o > 1e-4 and abs(h_e - h_o) / h_o < 1e-4
    # a ring beyond the band limit collects nothing (FP32 rounding only)
    assert eng.AnnularDetector(70.0, 200.0) < 1e-12


# ---------------------------------------------------------------- finite differences
@pytest.mark.parametrize("path", [0, 1])
def test_finite_difference_steps(engine_cls, oracle_mod, path):
    eng, orc = make_pair(engine_cls, oracle_mod, sto(2, 2), 128, 0.1, kV=200.0, path=path)
    for s in (eng, orc):
        s.InitialiseWavefunctions()
        s.SetFDdz(0.05)
    assert eng.GetSlices(False) == orc.GetSlices(False)
    for i in range(1, 41):
        eng.MultisliceStepFD(i)
        orc.MultisliceStepFD(i)
    assert rel_l2(eng.ExitWave(), orc.Wave()) < 5 * TOL


def test_fd_stability_query(engine_cls, oracle_mod):
    eng, orc = make_pair(engine_cls, oracle_mod, sto(2, 2), 128, 0.1)
    sc = orc.Scalars()
    if sc["nFD"] > 0:
        assert eng.GetSlices(False) == int(sc["nFD"])


# ---------------------------------------------------------------- errors
def test_call_order_and_argument_errors(engine_cls, oracle_mod):
    from cudamultislice_b200 import MultisliceError

    eng = engine_cls()
    with pytest.raises(MultisliceError) as e:
        eng.MultisliceStepConventional(1)
    assert e.value.code == 2
    with pytest.raises(MultisliceError) as e:
        eng.GetParameterisation("/nonexistent/fparams.dat")
    assert e.value.code == 4
    with pytest.raises(MultisliceError) as e:
        eng.SetAtoms([0], [1.0], [1.0], [1.0])
    assert e.value.code == 1
    eng.SetAtoms(*sto(1, 1))
    eng.ApplyMicroscopeParameters(200.0, 0, 0, 0, 0, 0, 0, 20)
    with pytest.raises(MultisliceError) as e:
        eng.SetCalculationVariables(0.1, 0, 0, 64, 1, 1, 1)
    assert e.value.code == 1
    with pytest.raises(MultisliceError) as e:
        eng.GetEWValueAbs(0, 0)
    assert e.value.code == 2


def test_import_xyz_reference_table(engine_cls, oracle_mod, tmp_path):
    from cudamultislice_b200 import structures as S

    Z, x, y, z = sto(1, 2)
    p = str(tmp_path / "sto.xyz")
    S.write_xyz(p, Z, x, y, z)
    eng = engine_cls()
    eng.ImportAtoms(p)
    eng.UploadBinnedAtoms()
    orc = oracle_mod.OracleSimulation()
    orc.ImportAtoms(p)
    orc.UploadBinnedAtoms()
    a, b = eng.Binned(), orc.Binned()
    assert np.array_equal(a[1], b[1])  # Ti -> 1 as GetZNum (U.cu:1241)
    assert 22 not in set(a[1].tolist())
    eng.SetElementTable(True)
    eng.ImportAtoms(p)
    eng.UploadBinnedAtoms()
    assert 22 in set(eng.Binned()[1].tolist())


@pytest.mark.parametrize("path", [0, 1])
def test_stem_raster_batched(engine_cls, oracle_mod, path):
    eng, orc = make_pair(engine_cls, oracle_mod, sto(2, 3), 128, 0.1, kV=300.0, df=-50.0, Cs=1e4, ap=25.0,
                         stem=True, path=path)
    px = np.array([10, 64, 100, 3, 77, 120, 50], np.int32)
    py = np.array([20, 64, 7, 99, 33, 110, 50], np.int32)
    sig = eng.StemRaster(px, py, 10.0, 40.0, batch=4)  # two batches, the second partial
    ref = []
    for x, y in zip(px, py):
        orc.STEMInitialiseWavefunctions(int(x), int(y))
        for i in range(1, orc.GetSlices(True) + 1):
            orc.MultisliceStepConventional(i)
        ref.append(orc.AnnularDetector(10.0, 40.0))
    ref = np.array(ref)
    assert np.all(ref > 0)
    assert np.max(np.abs(sig - ref) / ref) < 1e-4, (sig, ref)


def test_fd_readout_then_continue(engine_cls, oracle_mod):
    # reading the wave mid-run must not disturb the fused finite-difference state
    eng, orc = make_pair(engine_cls, oracle_mod, sto(2, 2), 128, 0.1, kV=200.0)
    for s in (eng, orc):
        s.InitialiseWavefunctions()
        s.SetFDdz(0.05)
    for i in range(1, 11):
        eng.MultisliceStepFD(i)
        orc.MultisliceStepFD(i)
    assert rel_l2(eng.ExitWave(), orc.Wave()) < 5 * TOL
    for i in range(11, 21):
        eng.MultisliceStepFD(i)
        orc.MultisliceStepFD(i)
    assert rel_l2(eng.ExitWave(), orc.Wave()) < 5 * TOL
    eng.SimulateImage(0.0)
    assert rel_l2(eng.Image(), orc.SimulateImage()) < 5 * TOL


# ---------------------------------------------------------------- frozen phonons
@pytest.mark.parametrize("path", [0, 1])
def test_frozen_phonon_series(engine_cls, oracle_mod, path):
    """Batched thermal configurations (fused: 2 per launch, 3 in all) against the
    oracle's pass loop: UploadBinnedAtomsTDS, the slices, AddTDSWaves, SimulateImage."""
    eng, orc = make_pair(engine_cls, oracle_mod, sto(2, 2), 128, 0.1, path=path)
    seed, sigma, first, nconf = 0x5EED2026, 0.076, 5, 3
    d, im = eng.FrozenPhonon(seed, first, nconf, sigma, batch=2)
    S = orc.GetSlices(True)
    orc.AllocTDS()
    imgs = []
    for p in range(first, first + nconf):
        orc.UploadBinnedAtomsTDS(seed, p, sigma)
        for i in range(1, S + 1):
            orc.MultisliceStepConventional(i)
        orc.AddTDSWaves()
        imgs.append(orc.SimulateImage())
    assert rel_l2(d, orc.TDS()) < TOL
    assert rel_l2(im, np.mean(imgs, axis=0)) < TOL


# ---------------------------------------------------------------- RS path
def test_rs_potential_and_steps(engine_cls, oracle_mod):
    """MultisliceStepRS as written (ten-term real-space series, 5-point stencil
    with the reference's centre coefficient and edge indices) vs the oracle."""
    eng, orc = make_pair(engine_cls, oracle_mod, sto(2, 2), 128, 0.1)
    for it in (2, 4):
        v = eng.PotentialSlice(3, it)
        assert rel_l2(v, orc.PotentialRS(it)) < TOL
    for it in range(1, 6):
        eng.MultisliceStepRS(it)
        orc.MultisliceStepRS(it)
    assert rel_l2(eng.ExitWave(), orc.Wave()) < TOL


# ---------------------------------------------------------------- mixed grids in one graph
def test_stem_raster_concurrent_mixed_grids(engine_cls, oracle_mod):
    """Two specimens on 128^2 and 256^2 grids, rastered as concurrent branches of
    one CUDA graph, give each handle's own raster (and the oracle's signal)."""
    from cudamultislice_b200 import stem_raster_concurrent

    a, orc_a = make_pair(engine_cls, oracle_mod, sto(2, 3), 128, 0.1, kV=300.0, df=-50.0, Cs=1e4, ap=25.0,
                         stem=True)
    b, _ = make_pair(engine_cls, oracle_mod, sto(3, 2), 256, 0.06, kV=300.0, df=0.0, Cs=0.0, ap=25.0, stem=True)
    pa = (np.array([10, 64, 100, 3, 77], np.int32), np.array([20, 64, 7, 99, 33], np.int32))
    pb = (np.array([0, 128, 200, 17, 90, 250, 31], np.int32), np.array([5, 128, 60, 240, 90, 1, 140], np.int32))
    (sa, sb), ms = stem_raster_concurrent([a, b], [pa, pb], 10.0, 40.0, batch=3)
    ra = a.StemRaster(*pa, 10.0, 40.0, batch=3)
    rb = b.StemRaster(*pb, 10.0, 40.0, batch=3)
    assert ms > 0
    # the 128^2 handle runs per-pass kernels in both arrangements (same
    # arithmetic); the 256^2 handle's own raster runs its slices in the batched
    # persistent loop, the graph branch per pass (FP32 rounding apart)
    np.testing.assert_allclose(sa, ra, rtol=1e-12)
    np.testing.assert_allclose(sb, rb, rtol=1e-6)
    orc_a.STEMInitialiseWavefunctions(int(pa[0][1]), int(pa[1][1]))
    for i in range(1, orc_a.GetSlices(True) + 1):
        orc_a.MultisliceStepConventional(i)
    ref = orc_a.AnnularDetector(10.0, 40.0)
    assert abs(sa[1] - ref) / ref < 1e-4


# ---------------------------------------------------------------- Cs / defocus sweep
@pytest.mark.parametrize("path", [0, 1])
def test_image_series_sweep(engine_cls, oracle_mod, path):
    """Re-imaging one exit wave at several (defocus, Cs) pairs equals
    SimulateImage after ApplyMicroscopeParameters with each pair."""
    eng, orc = make_pair(engine_cls, oracle_mod, sto(2, 4), 128, 0.1, path=path)
    eng.RunConventional()
    psi = orc.run_conventional()
    df = np.array([-800.0, -100.0, 0.0, 450.0], np.float32)
    cs = np.array([1e7, 5e6, 0.0, 1.2e7], np.float32)
    imgs = eng.SimulateImageSeries(df, cs)
    for i in range(df.size):
        orc.ApplyMicroscopeParameters(200.0, float(df[i]), 0.0, 0.0, float(cs[i]), 0.1, 30.0, 20.0)
        assert rel_l2(imgs[i], orc.SimulateImage()) < TOL, i
    # without Cs: the microscope's value
    imgs2 = eng.SimulateImageSeries(df[:1])
    orc.ApplyMicroscopeParameters(200.0, float(df[0]), 0.0, 0.0, 1e7, 0.1, 30.0, 20.0)
    assert rel_l2(imgs2[0], orc.SimulateImage()) < TOL


# ---------------------------------------------------------------- detector noise chain
def test_detector_noise_chain(engine_cls, oracle_mod):
    """SimulateImage's detector chain (DQE, seeded shot noise, NTF, conversion)
    and GetImValue's readout noise vs the oracle fed the same Philox draws.
    Integer rounding of the counts may flip by one count where FP32 and FP64
    land on opposite sides of a half; at 5000 electrons per pixel that stays
    below 1e-4 of the image norm."""
    eng, orc = make_pair(engine_cls, oracle_mod, sto(2, 4), 128, 0.1)
    eng.RunConventional()
    orc.run_conventional()
    r = np.arange(64)
    dqe = (0.7 * np.exp(-r / 30.0) + 0.05).astype(np.float32)
    ntf = (0.9 * np.exp(-r / 40.0) + 0.1).astype(np.float32)
    seed, dose = 0x1234ABCD5678, 5000.0
    eng.SetDetector(dqe, ntf, binning=2, conversion=8.0, seed=seed)
    I = orc.SimulateImage()
    for serial in (0, 1):
        eng.SimulateImage(dose)
        img = eng.Image()
        ref = orc.DetectorChain(I, dose, serial, dqe, ntf, 2, 8.0, seed)
        assert rel_l2(img, ref) < 1e-4, (serial, rel_l2(img, ref))
        if serial == 0:
            first = img
    assert rel_l2(img, first) > 1e-3  # the next image draws new noise
    x, y = 17, 40
    w = oracle_mod.philox([y * 128 + x, 1, 0x4EAD, 0], [seed & 0xFFFFFFFF, seed >> 32])
    z = oracle_mod.clipped_normal(int(w[0]), int(w[1]))
    v = eng.GetImValue(x, y)
    assert abs(v - (4.0 + 1.33 * z + img[y, x])) <= 1e-5 * abs(v)
    # GetDQEImValue (U.cu:2514-2517): the same pixel without the readout noise
    assert eng.GetDQEImValue(x, y) == abs(img[y, x])
    eng.SetDetector(None, None)
    eng.SimulateImage(dose)
    assert rel_l2(eng.Image(), I) < TOL


def test_tiff_readouts(engine_cls, oracle_mod, tmp_path):
    from tests.test_tiff import read_tiff_f32

    eng, _ = make_pair(engine_cls, oracle_mod, sto(2, 2), 128, 0.1)
    eng.RunConventional()
    psi = eng.ExitWave()
    eng.GetExitWave()  # the GUI's order: GetExitWave, then the per-pixel read-outs
    eng.SimulateImage(0.0)
    for what, ref in ((1, psi.real), (2, psi.imag), (4, np.abs(psi)), (0, eng.Image())):
        p = str(tmp_path / f"r{what}.tiff")
        eng.WriteTIFF(what, p)
        _, d = read_tiff_f32(p)
        assert np.allclose(d, ref, rtol=1e-6, atol=1e-7), what


# ---------------------------------------------------------------- non-square grids
@pytest.mark.parametrize("path", [0, 1])
@pytest.mark.parametrize("shape", [(256, 128), (128, 512), (4096, 64), (64, 4096)])
def test_non_square_grid(engine_cls, oracle_mod, shape, path):
    """nx != ny: the row and column passes use different line lengths (and plans)."""
    nx, ny = shape
    Z, x, y, z = sto(3, 2)
    eng = engine_cls()
    eng.SetSlicePath(path)
    orc = oracle_mod.OracleSimulation()
    for s in (eng, orc):
        s.SetAtoms(Z, x, y, z)
        s.UploadBinnedAtoms()
        s.GetParameterisation(FPARAMS)
        s.ApplyMicroscopeParameters(200.0, -300.0, 0.0, 0.0, 1e7, 0.1, 30.0, 20.0)
        s.SetCalculationVariables(0.08, -300.0, nx, ny, s.GetSizeX(), s.GetSizeY(), s.GetSizeZ(), 2.0, 2.0)
        s.PreCalculateFrequencies()
        s.InitialiseWavefunctions(1.9525)
    n = orc.GetSlices(True)
    for i in range(1, n + 1):
        eng.MultisliceStepConventional(i)
        orc.MultisliceStepConventional(i)
    assert rel_l2(eng.ExitWave(), orc.Wave()) < TOL
    eng.SimulateImage(0.0)
    assert rel_l2(eng.Image(), orc.SimulateImage()) < TOL


# ---------------------------------------------------------------- long columns (tensor-copy staging)
@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("shape", [(256, 2048), (512, 4096), (2048, 2048)])
def test_long_column_propagation(engine_cls, oracle_mod, shape, variant):
    """Columns of 2048 and 4096 points: the propagation pass stages its
    columns through shared memory with 2-D tensor copies.  Every FFT plan
    variant, three slices, against the FP64 oracle."""
    nx, ny = shape
    Z, x, y, z = sto(2, 1)
    eng = engine_cls()
    eng.SetFFTPlan(variant)
    orc = oracle_mod.OracleSimulation()
    for s in (eng, orc):
        s.SetAtoms(Z, x, y, z)
        s.UploadBinnedAtoms()
        s.GetParameterisation(FPARAMS)
        s.ApplyMicroscopeParameters(200.0, -300.0, 0.0, 0.0, 1e7, 0.1, 30.0, 20.0)
        s.SetCalculationVariables(0.02, -300.0, nx, ny, s.GetSizeX(), s.GetSizeY(), s.GetSizeZ(), 2.0, 2.0)
        s.PreCalculateFrequencies()
        s.InitialiseWavefunctions(1.9525)
    for i in range(1, 4):
        eng.MultisliceStepConventional(i)
        orc.MultisliceStepConventional(i)
    assert rel_l2(eng.ExitWave(), orc.Wave()) < TOL, (shape, variant)


# ---------------------------------------------------------------- errors of the newer entry points
def test_new_entry_point_errors(engine_cls, oracle_mod, tmp_path):
    from cudamultislice_b200 import MultisliceError, stem_raster_concurrent

    eng, _ = make_pair(engine_cls, oracle_mod, sto(2, 2), 128, 0.1)
    with pytest.raises(MultisliceError) as e:
        eng.FrozenPhonon(1, 0, 0, 0.076)            # no configurations
    assert e.value.code == 1
    with pytest.raises(MultisliceError):
        eng.FrozenPhonon(1, 0, 2, -1.0)             # negative sigma
    with pytest.raises(MultisliceError) as e:
        eng.SimulateImageSeries(np.array([np.inf], np.float32))
    assert e.value.code == 1
    with pytest.raises(MultisliceError):
        eng.SetDetector(np.ones(4, np.float32), np.ones(4, np.float32), binning=0)
    with pytest.raises(MultisliceError):
        eng.SetDetector(-np.ones(4, np.float32), np.ones(4, np.float32))
    with pytest.raises(MultisliceError) as e:
        eng.WriteTIFF(9, str(tmp_path / "x.tiff"))
    assert e.value.code == 1
    with pytest.raises(MultisliceError) as e:
        eng.WriteTIFF(0, str(tmp_path / "x.tiff"))  # no image simulated yet
    assert e.value.code == 2
    with pytest.raises(MultisliceError):
        eng.MultisliceStepRS(0)
    with pytest.raises(MultisliceError):
        eng.SetCheckpoint(-1)
    with pytest.raises(MultisliceError):
        eng.TimePass(0, 32, 0)  # the finite-difference row pass is not a timing target
    s, _ = make_pair(engine_cls, oracle_mod, sto(2, 2), 128, 0.1, stem=True)
    with pytest.raises(MultisliceError):
        stem_raster_concurrent([s], [(np.array([1], np.int32), np.array([1], np.int32))], 40.0, 10.0)
    # the handle stays usable after the failures
    eng.RunConventional()
    eng.SimulateImage(0.0)
    assert np.isfinite(eng.Image()).all()


# ---------------------------------------------------------------- whole FD runs
@pytest.mark.parametrize("path", [0, 1])
def test_run_fd_equals_step_loop_and_oracle(engine_cls, oracle_mod, path):
    """ms_run_fd (band-limited potential planes resident, fused steps replayed
    as one graph) equals ms_multislice_step_fd(1..n) and the oracle's
    MultisliceStep loop (U.cu:2040-2083); odd and even step counts, repeated
    runs (graph replay, and the recapture an odd count's buffer parity needs)."""
    eng, orc = make_pair(engine_cls, oracle_mod, sto(2, 2), 128, 0.1, kV=200.0, path=path)
    for s in (eng, orc):
        s.InitialiseWavefunctions()
        s.SetFDdz(0.05)
    for i in range(1, 42):
        orc.MultisliceStepFD(i)
    ref = orc.Wave()
    for i in range(1, 42):
        eng.MultisliceStepFD(i)
    steps = eng.ExitWave()
    for rep in range(3):
        eng.InitialiseWavefunctions()
        assert eng.RunFD(41) == 41
        w = eng.ExitWave()
        assert rel_l2(w, ref) < 5 * TOL, (rep, rel_l2(w, ref))
        assert rel_l2(w, steps.astype(np.complex128)) < 1e-6, rep
        assert eng.LastDeviceMs() > 0
    eng.InitialiseWavefunctions()
    assert eng.RunFD(40) == 40
    orc.InitialiseWavefunctions()
    orc.SetFDdz(0.05)
    for i in range(1, 41):
        orc.MultisliceStepFD(i)
    assert rel_l2(eng.ExitWave(), orc.Wave()) < 5 * TOL
    # a step after a whole run continues from its state
    eng.MultisliceStepFD(41)
    orc.MultisliceStepFD(41)
    assert rel_l2(eng.ExitWave(), orc.Wave()) < 5 * TOL
