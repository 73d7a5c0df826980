"""The persistent slice loop (one cooperative launch for all slices, grid
barriers between the row and column phases) against the per-pass kernels
and the FP64 oracle, and the bound on its grid-barrier waits.

Reference being replaced: the per-slice launch sequence of
MultisliceStepConv (GUI Simulation/UnmanagedGUISimulation.cu:2085-2124) as
the GUI drives it (CUDA Simulation GUI/MainWindow.xaml.cs:258-283)."""
import numpy as np
import pytest

from tests.conftest import FPARAMS

pytestmark = pytest.mark.gpu

TOL = 1e-5


def rel_l2(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def engine_cls():
    """Engines that build the potential stack before the slices, so that the
    first RunConventional runs the persistent loop too (by default a run with
    a stack to build overlaps the build with per-pass slice steps)."""
    from cudamultislice_b200 import ManagedMultisliceSimulation, build

    build.build(verbose=False)

    def make(*args, **kw):
        e = ManagedMultisliceSimulation(*args, **kw)
        e.SetBuildOverlap(False)
        return e

    return make


def setup(s, atoms, n, ps, kV=200.0, df=-500.0, stem=False):
    s.SetAtoms(*atoms)
    s.UploadBinnedAtoms()
    s.GetParameterisation(FPARAMS)
    s.ApplyMicroscopeParameters(kV, df, 0.0, 0.0, 1e7, 0.1, 30.0, 20.0)
    if stem:
        s.STEMSetCalculationVariables(ps, df, n, n, s.GetSizeX(), s.GetSizeY(), s.GetSizeZ())
    else:
        s.SetCalculationVariables(ps, df, n, n, s.GetSizeX(), s.GetSizeY(), s.GetSizeZ(), 2.0, 2.0)
    s.PreCalculateFrequencies()
    s.InitialiseWavefunctions(1.9525)


@pytest.mark.parametrize("n", [256, 512, 1024])
def test_loop_matches_passes_and_oracle(engine_cls, oracle_mod, n):
    from cudamultislice_b200 import structures as S

    atoms = S.srtio3(4, 4, 6)
    ps = 3.905 * 4 / n
    eng = engine_cls()
    setup(eng, atoms, n, ps)
    nsl = eng.RunConventional()  # persistent loop (default)
    w_loop = eng.ExitWave()
    launches_loop = eng.LaunchCount()
    eng.SetSliceLoop(False)
    eng.InitialiseWavefunctions(1.9525)
    eng.RunConventional()
    w_pass = eng.ExitWave()
    eng.close()
    orc = oracle_mod.OracleSimulation()
    setup(orc, atoms, n, ps)
    psi = orc.run_conventional()
    S_ = orc.GetSlices(True)
    orc.close()
    assert nsl == S_
    assert rel_l2(w_loop, psi) < TOL, rel_l2(w_loop, psi)
    assert rel_l2(w_pass, psi) < TOL
    # same arithmetic per point as the per-pass kernels of the same plan, up to
    # the plan variant the per-pass path was tuned to
    assert rel_l2(w_loop, w_pass) < 3e-6
    assert launches_loop > 0


def test_loop_repeated_runs_and_step_calls_agree(engine_cls, oracle_mod):
    """Replaying the captured loop gives the same wave every time, and equals
    the per-slice MultisliceStepConventional calls."""
    from cudamultislice_b200 import structures as S

    atoms = S.srtio3(4, 4, 5)
    eng = engine_cls()
    setup(eng, atoms, 512, 3.905 * 4 / 512)
    runs = []
    for _ in range(3):
        eng.InitialiseWavefunctions(1.9525)
        eng.RunConventional()
        runs.append(eng.ExitWave())
    assert np.array_equal(runs[0], runs[1]) and np.array_equal(runs[1], runs[2])
    eng.InitialiseWavefunctions(1.9525)
    for i in range(1, eng.GetSlices(True) + 1):
        eng.MultisliceStepConventional(i)
    assert rel_l2(eng.ExitWave(), runs[0]) < 2e-6
    eng.close()


def test_loop_stem_probe(engine_cls, oracle_mod):
    from cudamultislice_b200 import structures as S

    atoms = S.srtio3(4, 4, 4)
    n = 256
    eng, orc = engine_cls(), oracle_mod.OracleSimulation()
    for s in (eng, orc):
        setup(s, atoms, n, 3.905 * 4 / n, kV=300.0, df=0.0, stem=True)
        s.STEMInitialiseWavefunctions(100, 37)
    eng.RunConventional()
    psi = orc.run_conventional()
    assert rel_l2(eng.ExitWave(), psi) < TOL
    eng.close()
    orc.close()


def test_loop_time_slices(engine_cls):
    from cudamultislice_b200 import structures as S

    eng = engine_cls()
    setup(eng, S.srtio3(4, 4, 6), 1024, 3.905 * 4 / 1024)
    nsl = eng.BuildPotentialStack()
    eng.TimeSlices(nsl, 1, breakdown=False)  # builds the propagator tables (one launch)
    l0 = eng.LaunchCount()
    ms, row, col = eng.TimeSlices(nsl, 3, breakdown=True)
    assert ms > 0 and row == 0 and col == 0  # one launch per repetition, no per-pass split
    assert eng.LaunchCount() - l0 == 3
    eng.close()


def test_loop_wait_bound_ends_the_launch_with_an_error(engine_cls, oracle_mod):
    """A grid barrier whose arrivals never come (the test hook asks for one
    more than the grid has) runs out its 20 ms bound: the call fails with a
    status, the context stays usable, and the next run is correct."""
    from cudamultislice_b200 import MultisliceError
    from cudamultislice_b200 import structures as S

    atoms = S.srtio3(2, 2, 3)
    eng = engine_cls()
    setup(eng, atoms, 256, 0.06)
    eng.SetLoopWaitUs(20000)
    eng.SetLoopWaitTest(1)
    with pytest.raises(MultisliceError) as e:
        eng.RunConventional()
    assert e.value.code == 3 and "grid-barrier wait ran out" in str(e.value)
    eng.SetLoopWaitTest(0)
    eng.InitialiseWavefunctions(1.9525)
    eng.RunConventional()
    orc = oracle_mod.OracleSimulation()
    setup(orc, atoms, 256, 0.06)
    assert rel_l2(eng.ExitWave(), orc.run_conventional()) < TOL
    eng.close()
    orc.close()


@pytest.mark.parametrize("variant", list(range(10)))
def test_every_loop_variant(engine_cls, oracle_mod, variant):
    """Each kernel variant of the loop (column unit width, barrier form) gives
    the oracle's exit wave; the tuner's choice is one of them."""
    from cudamultislice_b200 import structures as S

    atoms = S.srtio3(4, 4, 4)
    n = 1024
    eng = engine_cls()
    setup(eng, atoms, n, 3.905 * 4 / n)
    v, cols, grid = eng.SliceLoop()
    assert 0 <= v <= 9 and cols in (2, 4, 8) and grid > 0
    eng.SetLoopVariant(variant)
    assert eng.SliceLoop()[0] == variant
    eng.RunConventional()
    w = eng.ExitWave()
    eng.close()
    orc = oracle_mod.OracleSimulation()
    setup(orc, atoms, n, 3.905 * 4 / n)
    psi = orc.run_conventional()
    orc.close()
    assert rel_l2(w, psi) < TOL


# ---------------------------------------------------------------- batched persistent loop
def stem_pair(engine_cls, oracle_mod, atoms, n, ps):
    eng, orc = engine_cls(), oracle_mod.OracleSimulation()
    for s in (eng, orc):
        setup(s, atoms, n, ps, kV=300.0, df=-50.0, stem=True)
    return eng, orc


def test_batched_loop_raster_matches_passes_and_oracle(engine_cls, oracle_mod):
    """ms_stem_raster with every batch's slices in one persistent launch (256^2,
    batches of 3 over 7 probes) equals the per-pass raster and the oracle's
    per-probe HAADF signal (AnnularDetector after each probe's slice loop)."""
    from cudamultislice_b200 import structures as S

    atoms = S.srtio3(4, 4, 3)
    eng, orc = stem_pair(engine_cls, oracle_mod, atoms, 256, 3.905 * 4 / 256)
    px = np.array([10, 128, 200, 3, 77, 250, 50], np.int32)
    py = np.array([20, 128, 7, 199, 33, 110, 50], np.int32)
    eng.StemRaster(px[:3], py[:3], 10.0, 40.0, batch=3)  # tunes the plans
    l0 = eng.LaunchCount()
    sig = eng.StemRaster(px, py, 10.0, 40.0, batch=3)
    loop_launches = eng.LaunchCount() - l0
    eng.SetSliceLoop(False)
    sig_pass = eng.StemRaster(px, py, 10.0, 40.0, batch=3)
    ref = []
    for x, y in zip(px, py):
        orc.STEMInitialiseWavefunctions(int(x), int(y))
        orc.run_conventional()
        ref.append(orc.AnnularDetector(10.0, 40.0))
    ref = np.array(ref)
    S_ = orc.GetSlices(True)
    eng.close()
    orc.close()
    assert np.max(np.abs(sig - ref) / ref) < 1e-4, (sig, ref)
    assert np.max(np.abs(sig - sig_pass) / sig_pass) < 1e-5
    # three batches: probe preparation (6 launches) plus one loop launch each,
    # where the per-pass raster takes two launches per slice
    assert loop_launches <= 3 * 7 < 3 * (2 * S_)


def test_batched_loop_frozen_phonons(engine_cls, oracle_mod):
    """ms_frozen_phonon with each batch of configurations in one persistent
    launch (per-configuration potential stacks, exp(i sigma V) on the fly)."""
    from cudamultislice_b200 import structures as S

    atoms = S.srtio3(4, 4, 3)
    n = 256
    eng = engine_cls()
    setup(eng, atoms, n, 3.905 * 4 / n)
    seed, sigma, first, nconf = 0x5EED2026, 0.076, 2, 3
    d, im = eng.FrozenPhonon(seed, first, nconf, sigma, batch=2)
    eng.SetSliceLoop(False)
    d2, im2 = eng.FrozenPhonon(seed, first, nconf, sigma, batch=2)
    eng.close()
    orc = oracle_mod.OracleSimulation()
    setup(orc, atoms, n, 3.905 * 4 / n)
    orc.AllocTDS()
    imgs = []
    for p in range(first, first + nconf):
        orc.UploadBinnedAtomsTDS(seed, p, sigma)
        orc.run_conventional()
        orc.AddTDSWaves()
        imgs.append(orc.SimulateImage())
    td = orc.TDS()
    orc.close()
    assert rel_l2(d, td) < TOL
    assert rel_l2(im, np.mean(imgs, axis=0)) < 2 * TOL
    assert rel_l2(d, d2) < 2e-6 and rel_l2(im, im2) < 4e-6


def test_mixed_grids_in_one_persistent_launch(engine_cls, oracle_mod):
    """Two specimens on 512^2 and 256^2: each round takes the next batch of
    both rasters through every slice in one cooperative launch; the signals
    equal each handle's own raster (same per-instance arithmetic; only the
    order of the FP64 detector sums differs) and the oracle's."""
    from cudamultislice_b200 import stem_raster_concurrent
    from cudamultislice_b200 import structures as S

    atoms = S.srtio3(4, 4, 3)
    a, orc_a = stem_pair(engine_cls, oracle_mod, atoms, 512, 3.905 * 4 / 512)
    b, _ = stem_pair(engine_cls, oracle_mod, atoms, 256, 3.905 * 4 / 256)
    pa = (np.array([10, 256, 400, 3, 77], np.int32), np.array([20, 256, 7, 399, 33], np.int32))
    pb = (np.array([0, 128, 200, 17, 90, 250, 31], np.int32), np.array([5, 128, 60, 240, 90, 1, 140], np.int32))
    (sa, sb), ms = stem_raster_concurrent([a, b], [pa, pb], 10.0, 40.0, batch=3)
    ra = a.StemRaster(*pa, 10.0, 40.0, batch=3)
    rb = b.StemRaster(*pb, 10.0, 40.0, batch=3)
    assert ms > 0
    np.testing.assert_allclose(sa, ra, rtol=1e-10)
    np.testing.assert_allclose(sb, rb, rtol=1e-10)
    orc_a.STEMInitialiseWavefunctions(int(pa[0][1]), int(pa[1][1]))
    orc_a.run_conventional()
    ref = orc_a.AnnularDetector(10.0, 40.0)
    assert abs(sa[1] - ref) / ref < 1e-4
    for s in (a, b, orc_a):
        s.close()
