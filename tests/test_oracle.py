"""Pins of the FP64 CPU oracle (no GPU).

The reference ships no tests or golden data, so the oracle is pinned by
(1) known answers from mathematics and published tables (Bessel functions,
DFT, Philox test vectors), (2) physical identities of the multislice method,
and (3) golden vectors produced by the reference program itself
(test_golden_reference.py)."""
import numpy as np
import pytest
import scipy.special as sp

from tests.conftest import FPARAMS


def test_bessel_against_scipy(oracle_mod):
    # A&S 9.8.5/9.8.6 are accurate to ~1e-7 relative; the oracle evaluates
    # the same polynomials in FP64 (U.cu:41-111).
    xs = np.concatenate([np.linspace(0.01, 2.0, 80), np.linspace(2.0001, 30, 80)])
    k = np.array([oracle_mod.bessk0(x) for x in xs])
    assert np.max(np.abs(k - sp.k0(xs)) / sp.k0(xs)) < 2e-7
    i = np.array([oracle_mod.bessi0(x) for x in xs[:100]])
    assert np.max(np.abs(i - sp.i0(xs[:100])) / sp.i0(xs[:100])) < 2e-7
    assert oracle_mod.bessk0(0.0) == 1e20  # U.cu:108


@pytest.mark.parametrize("shape", [(8, 8), (64, 32), (30, 48), (7, 5), (256, 128)])
def test_fft_against_numpy(oracle_mod, shape):
    rng = np.random.default_rng(1)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    f = oracle_mod.fft2(a, -1)
    g = np.fft.fft2(a)
    assert np.max(np.abs(f - g)) / np.max(np.abs(g)) < 1e-14
    inv = oracle_mod.fft2(a, +1)
    assert np.max(np.abs(inv - np.fft.ifft2(a) * a.size)) / np.max(np.abs(g)) < 1e-14


def test_philox_known_answers(oracle_mod):
    # Known-answer vectors of Philox4x32-10 (Salmon et al., SC'11, Random123).
    kat = [
        ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
        ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
        ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
         [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
    ]
    for c, k, want in kat:
        assert oracle_mod.philox(c, k).tolist() == want


def test_tds_displacement_statistics(oracle_mod):
    n = 200000
    z = np.zeros(n, np.float32)
    xo, yo, zo = oracle_mod.tds_displace(z, z, z, 1234, 7, 0.076)
    for d in (xo, yo, zo):
        assert abs(d.mean()) < 0.076 * 5 / np.sqrt(n)
        assert abs(d.std() / 0.076 - 1) < 0.01
    # seeded: same inputs, same output; another pass differs
    xo2, _, _ = oracle_mod.tds_displace(z, z, z, 1234, 7, 0.076)
    xo3, _, _ = oracle_mod.tds_displace(z, z, z, 1234, 8, 0.076)
    assert np.array_equal(xo, xo2) and not np.array_equal(xo, xo3)


def test_fparams_table(oracle_mod):
    fp = oracle_mod.parse_fparams(FPARAMS)
    assert fp.shape == (103, 12)
    assert np.all(fp[:, 1::2] >= 0)


def test_projected_equals_integrated_3d_potential(oracle_mod):
    # The projected potential is the z-integral of the 3D potential (Kirkland):
    # int v(sqrt(r^2 + z^2)) dz = vz(r), away from the 0.25 A clamp.
    fp = oracle_mod.parse_fparams(FPARAMS)
    zs = np.linspace(-30, 30, 120001)
    for Z in (6, 14, 38):
        for r in (0.5, 1.0, 1.7):
            v = np.array([oracle_mod.vatom(fp, Z, r * r + t * t) for t in zs[::10]])
            integral = np.trapezoid(v, zs[::10])
            vz = oracle_mod.vzatom2(fp, Z, r * r)
            assert abs(integral - vz) / vz < 2e-3, (Z, r, integral, vz)


def test_element_tables(oracle_mod):
    assert oracle_mod.lib().or_znum(b"Sr", 0) == 38
    assert oracle_mod.lib().or_znum(b"Ti", 0) == 1  # not in U.cu:1188-1243
    assert oracle_mod.lib().or_znum(b"Ti", 1) == 22
    assert oracle_mod.lib().or_znum(b"Ga", 1) == 31
    assert oracle_mod.lib().or_znum(b"Xx", 1) == 1


def _small_sim(oracle_mod, n=64, kV=200.0, dz=1.0):
    from cudamultislice_b200 import structures as S

    Z, x, y, z = S.srtio3(2, 2, 3)
    s = oracle_mod.OracleSimulation()
    s.SetAtoms(Z, x, y, z)
    s.UploadBinnedAtoms()
    s.GetParameterisation(FPARAMS)
    s.ApplyMicroscopeParameters(kV, -500.0, 0.0, 0.0, 1e7, 0.1, 30.0, 20.0)
    ps = (s.GetSizeX() + 0.0) / n
    s.SetCalculationVariables(ps, -500.0, n, n, s.GetSizeX(), s.GetSizeY(), s.GetSizeZ(), 0.0, 0.0)
    s.PreCalculateFrequencies()
    s.InitialiseWavefunctions(dz)
    return s


def test_setup_scalars(oracle_mod):
    s = _small_sim(oracle_mod)
    sc = s.Scalars()
    # relativistic wavelength at 200 kV with the reference's rounded constants
    h, c, e, m = 6.63e-34, 3e8, 1.6e-19, 9.11e-31
    V = 200e3
    lam = h * c / np.sqrt(e * V * (2 * m * c * c + e * V)) * 1e10
    assert abs(sc["wavel"] - lam) / lam < 1e-6
    kx, ky = s.Frequencies()
    assert kx[0] == 0 and ky[0] == 0
    # kmax = half of the largest frequency below Nyquist (U.cu:1929-1953)
    assert abs(sc["kmax"] - kx[31] / 2) < 1e-6


def _gap_sim(oracle_mod, n=64, dz=1.0):
    # two carbon atoms 50 A apart: slices in the middle of the gap hold no
    # potential, so a step there is a pure Fresnel propagation
    s = oracle_mod.OracleSimulation()
    s.SetAtoms([6, 6], [5.0, 5.0], [5.0, 5.0], [0.0, 50.0])
    s.UploadBinnedAtoms()
    s.GetParameterisation(FPARAMS)
    s.ApplyMicroscopeParameters(200.0, 0.0, 0.0, 0.0, 1e7, 0.1, 30.0, 20.0)
    s.SetCalculationVariables(0.2, 0.0, n, n, s.GetSizeX(), s.GetSizeY(), s.GetSizeZ(), 0.0, 0.0)
    s.PreCalculateFrequencies()
    s.InitialiseWavefunctions(dz)
    return s


def test_vacuum_keeps_plane_wave(oracle_mod):
    s = _gap_sim(oracle_mod)
    assert np.all(s.PotentialConventional(25) == 0)
    s.SetWave(np.ones((64, 64), np.complex128))
    s.MultisliceStepConventional(25)
    assert np.max(np.abs(s.Wave() - 1.0)) < 1e-12


def test_propagator_composition_and_unitarity(oracle_mod):
    # one step in vacuum applies exp(-i pi dz lambda k^2) inside the band limit
    # (CreatePropsKernel U.cu:399-428); steps compose and are unitary on
    # band-limited waves (Parseval of the 1/N-normalised pair)
    rng = np.random.default_rng(3)
    n = 64
    s = _gap_sim(oracle_mod, n=n, dz=0.5)
    kx, ky = s.Frequencies()
    sc = s.Scalars()
    K2 = kx[None, :].astype(np.float64) ** 2 + ky[:, None].astype(np.float64) ** 2
    keep = np.sqrt(kx[None, :] ** 2 + ky[:, None] ** 2) < np.float32(sc["kmax"])
    spec = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) * keep
    w = np.fft.ifft2(spec)
    s.SetWave(w)
    s.MultisliceStepConventional(50)
    s.MultisliceStepConventional(51)
    out = s.Wave()
    lam = sc["wavel"]
    expect = np.fft.ifft2(np.fft.fft2(w) * np.exp(-1j * 3.14159265 * 1.0 * lam * K2) * keep)
    assert np.linalg.norm(out - expect) / np.linalg.norm(expect) < 1e-12
    assert abs(np.linalg.norm(out) - np.linalg.norm(w)) / np.linalg.norm(w) < 1e-12


def test_binning_csr_properties(oracle_mod):
    from cudamultislice_b200 import structures as S

    Z, x, y, z = S.random_atoms(3000, size=(20, 20, 15), seed=5)
    s = oracle_mod.OracleSimulation()
    s.SetAtoms(Z, x, y, z)
    s.UploadBinnedAtoms()
    off, bZ, bx, by, bz = s.Binned()
    box = s.Box()
    assert off[0] == 0 and off[-1] == len(Z) and np.all(np.diff(off) >= 0)
    # every atom sits in the bin of its FP32 key, stable order inside a bin
    MaxX, MinX, MaxY, MinY, MaxZ, MinZ = [np.float32(v) for v in box]
    key = (np.floor((np.float32(MaxZ) - z) / np.float32(1)).astype(np.int64) * 2500
           + np.floor(((y - MinY) / (MaxY - MinY)) * np.float32(50)).astype(np.int64) * 50
           + np.floor(((x - MinX) / (MaxX - MinX)) * np.float32(50)).astype(np.int64))
    order = np.argsort(key, kind="stable")
    assert np.array_equal(bx, (x - MinX)[order])
    assert np.array_equal(bZ, Z[order])
    assert np.array_equal(np.bincount(key, minlength=len(off) - 1), np.diff(off))


def test_potential_cache_gives_identical_steps(oracle_mod):
    """CachePotentials (probe rasters over one specimen) changes no result: two
    probe positions, cached and uncached, bit for bit; a set-up change drops
    the cached potentials."""
    from cudamultislice_b200 import structures

    def probe_runs(cache):
        o = oracle_mod.OracleSimulation()
        o.SetAtoms(*structures.srtio3(2, 2, 3))
        o.UploadBinnedAtoms()
        o.GetParameterisation(FPARAMS)
        o.ApplyMicroscopeParameters(300.0, 0.0, 0.0, 0.0, 0.0, 0.1, 30.0, 25.0)
        o.STEMSetCalculationVariables(0.1, 0.0, 64, 64, o.GetSizeX(), o.GetSizeY(), o.GetSizeZ())
        o.PreCalculateFrequencies()
        o.InitialiseWavefunctions(1.0)
        o.CachePotentials(cache)
        out = []
        for px, py in ((10, 20), (40, 33)):
            o.STEMInitialiseWavefunctions(px, py)
            out.append(o.run_conventional())
        # new positions after re-binning: the cache must not serve the old slab
        x = structures.srtio3(2, 2, 3)
        o.SetAtoms(x[0], x[1] + np.float32(0.3), x[2], x[3])
        o.UploadBinnedAtoms()
        o.STEMInitialiseWavefunctions(10, 20)
        out.append(o.run_conventional())
        o.close()
        return out

    for a, b in zip(probe_runs(False), probe_runs(True)):
        assert np.array_equal(a, b)
