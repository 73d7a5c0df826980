"""The separable conventional potential against the per-sub-plane sum and the
FP64 oracle (binnedAtomPKernel3, GUI Simulation/UnmanagedGUISimulation.cu:582-653).

The separable kernel writes each element's vatom as 12 Gaussians in r^2, so an
atom's 20 sub-planes are summed once per atom; the sub-planes that pass the
reference's FP32 cut-off test are the same as term by term.  Its values must
agree with the FP64 oracle as closely as the per-sub-plane kernel's do
(relative L2 error <= 1e-6 here, well inside the 1e-5 parity tolerance), on
crystals, amorphous and random specimens, thin and thick slices, atoms on
pixel centres and sub-plane heights (the 0.25 A clamp), and deep in a thick
slab."""
import numpy as np
import pytest

from tests.conftest import FPARAMS

pytestmark = pytest.mark.gpu

TOL_SEP = 1e-6  # relative L2 against FP64, separable and per-sub-plane alike


@pytest.fixture(scope="module")
def engine_cls():
    from cudamultislice_b200 import ManagedMultisliceSimulation, build

    build.build(verbose=False)
    return ManagedMultisliceSimulation


def _setup(s, atoms, n, ps, dz, kV=200.0, xoff=2.0, yoff=2.0):
    Z, x, y, z = atoms
    s.SetAtoms(Z, x, y, z)
    s.UploadBinnedAtoms()
    s.GetParameterisation(FPARAMS)
    s.ApplyMicroscopeParameters(kV, -500.0, 0.0, 0.0, 1e7, 0.1, 30.0, 20.0)
    s.SetCalculationVariables(ps, -500.0, n, n, s.GetSizeX(), s.GetSizeY(), s.GetSizeZ(), xoff, yoff)
    s.PreCalculateFrequencies()
    s.InitialiseWavefunctions(dz)


def _cases():
    from cudamultislice_b200 import structures as S

    rng = np.random.default_rng(5)
    # atoms on pixel centres (ps 0.1, offset 2.0 -> x = 2.0 + 0.1 k in the
    # shifted frame) at heights of sub-planes: the clamp path
    k = rng.integers(20, 100, size=(60, 2))
    Zc = rng.choice([6, 8, 14, 38], size=60).astype(np.int32)
    zc = (rng.integers(0, 12, size=60) * 0.2).astype(np.float32)
    onpix = (Zc, (k[:, 0] * 0.1).astype(np.float32), (k[:, 1] * 0.1).astype(np.float32), zc)
    return {
        "srtio3": (S.srtio3(2, 2, 6), 128, 0.1, 1.9525),
        "srtio3_thick_slab": (S.srtio3(2, 2, 40), 128, 0.1, 1.9525),
        "a-c": (S.amorphous_carbon(size=(12.0, 12.0, 14.0), seed=3), 256, 0.05, 2.0),
        "si110": (S.silicon_110(2, 2, 4), 128, 0.09, 1.92),
        "gan": (S.gan_wurtzite_11_20(2, 2, 3), 128, 0.1, 1.5945),
        "random_thin": (S.random_atoms(800, size=(12.0, 12.0, 9.0), seed=7), 128, 0.1, 0.5),
        "on_pixels": (onpix, 128, 0.1, 2.0),
        # coarse pixels over a small box (bins of 0.24 A): a tile's candidate
        # bins exceed 256 segments
        "coarse_small_box": (S.srtio3(2, 2, 4), 64, 0.25, 1.9525),
    }


@pytest.mark.parametrize("tile", [-1, 0, 1, 2, 3])
@pytest.mark.parametrize("case", list(_cases().keys()))
def test_separable_potential(engine_cls, oracle_mod, case, tile):
    """tile -1: the shape the engine tunes; 0..3: each tile shape (two and four
    pixels per thread) forced.  The per-sub-plane kernel is checked alongside."""
    atoms, n, ps, dz = _cases()[case]
    eng = engine_cls()
    orc = oracle_mod.OracleSimulation()
    for s in (eng, orc):
        _setup(s, atoms, n, ps, dz)
    S = eng.GetSlices(True)
    assert eng.PotentialSum()[1] == 2
    its = sorted({2, S // 2, S - 1, S})
    worst = 0.0
    for it in its:
        ref = orc.PotentialConventional(it)
        if np.abs(ref).max() == 0:
            continue
        eng.SetPotentialSum(2)
        eng.SetPotentialTile(tile)
        vs = eng.PotentialSlice(0, it)
        eng.SetPotentialTile(-1)
        assert eng.PotentialSum() == (2, 2)
        eng.SetPotentialSum(1)
        vp = eng.PotentialSlice(0, it)
        assert eng.PotentialSum() == (1, 1)
        es = np.linalg.norm(vs - ref) / np.linalg.norm(ref)
        ep = np.linalg.norm(vp - ref) / np.linalg.norm(ref)
        worst = max(worst, es)
        assert es < TOL_SEP, (case, it, es, ep)
        assert ep < TOL_SEP, (case, it, es, ep)
        assert np.abs(vs - ref).max() < 5 * TOL_SEP * np.abs(ref).max(), (case, it)
        # zero exactly where no atom reaches (the same cut-off decisions)
        assert np.array_equal(vs == 0, vp == 0), (case, it)
    eng.close()
    orc.close()


def test_separable_is_default_and_forced_mode_errors(engine_cls):
    from cudamultislice_b200 import structures as S

    eng = engine_cls()
    _setup(eng, S.srtio3(1, 1, 2), 64, 0.1, 1.9525)
    assert eng.PotentialSum() == (0, 2)
    eng.PotentialSlice(0, 2)
    assert eng.PotentialSum() == (2, 2)
    eng.SetPotentialSum(1)
    assert eng.PotentialSum()[1] == 1
    with pytest.raises(Exception):
        eng.SetPotentialSum(3)
    eng.close()


def test_parameter_file_without_expansion_falls_back(engine_cls, oracle_mod, tmp_path):
    """A parameterisation whose rows the compiled-in expansions do not match
    (carbon's Lorentzian amplitudes scaled by 1.01) takes the per-sub-plane sum
    for specimens holding that element, keeps the separable one for the
    others, and refuses the separable sum when it is forced."""
    from cudamultislice_b200 import structures as S

    P = np.loadtxt(FPARAMS)
    P[5, 0:6:2] *= 1.01
    path = tmp_path / "fparams_modified.dat"
    np.savetxt(path, P)
    carbon = S.amorphous_carbon(size=(10.0, 10.0, 8.0), seed=4)
    eng = engine_cls()
    orc = oracle_mod.OracleSimulation()
    for s in (eng, orc):
        Z, x, y, z = carbon
        s.SetAtoms(Z, x, y, z)
        s.UploadBinnedAtoms()
        s.GetParameterisation(str(path))
        s.ApplyMicroscopeParameters(200.0, -500.0, 0.0, 0.0, 1e7, 0.1, 30.0, 20.0)
        s.SetCalculationVariables(0.1, -500.0, 128, 128, s.GetSizeX(), s.GetSizeY(), s.GetSizeZ(), 2.0, 2.0)
        s.PreCalculateFrequencies()
        s.InitialiseWavefunctions(2.0)
    assert eng.PotentialSum()[1] == 1
    v = eng.PotentialSlice(0, 3)
    assert eng.PotentialSum()[0] == 1
    ref = orc.PotentialConventional(3)
    assert np.linalg.norm(v - ref) / np.linalg.norm(ref) < TOL_SEP
    eng.SetPotentialSum(2)
    with pytest.raises(Exception):
        eng.PotentialSlice(0, 3)
    eng.close()
    orc.close()
    # silicon is unaffected by the carbon row
    eng = engine_cls()
    _setup(eng, S.silicon_110(1, 1, 2), 64, 0.1, 1.92)
    eng.GetParameterisation(str(path))
    assert eng.PotentialSum()[1] == 2
    eng.close()
