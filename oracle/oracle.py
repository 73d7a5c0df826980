"""ctypes binding of the FP64 CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA engine: tests/,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use it;
the product (``cudamultislice_b200``) never imports it.

``OracleSimulation`` mirrors the method list of the reference's managed
wrapper (GUI Simulation/GUI Simulation.h:17-59) so that parity tests read as
the same call sequence run on the engine and on the oracle.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_f = C.c_float
_i = C.c_int
_d = C.c_double
_p = C.c_void_p


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, OpenMP)."""
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < max(
        os.path.getmtime(os.path.join(_HERE, f)) for f in ("ms_oracle.cpp", "ms_oracle.h")
    ):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    sig = {
        "or_bessi0": (_d, [_d]),
        "or_bessk0": (_d, [_d]),
        "or_vzatom2": (_d, [_p, _i, _d]),
        "or_vatom": (_d, [_p, _i, _d]),
        "or_parse_fparams": (_i, [C.c_char_p, _p, C.POINTER(_i)]),
        "or_fft1d": (_i, [_p, _i, _i]),
        "or_fft2d": (_i, [_p, _i, _i, _i]),
        "or_philox4x32_10": (None, [_p, _p, _p]),
        "or_tds_displace": (None, [_p, _p, _p, _i, C.c_uint64, C.c_uint32, _f, _p, _p, _p]),
        "or_znum": (_i, [C.c_char_p, _i]),
        "or_create": (_p, []),
        "or_destroy": (None, [_p]),
        "or_last_error": (C.c_char_p, [_p]),
        "or_set_threads": (_i, [_i]),
        "or_import_atoms": (_i, [_p, C.c_char_p, _i]),
        "or_set_atoms": (_i, [_p, _p, _p, _p, _p, _i]),
        "or_get_box": (_i, [_p, _p]),
        "or_load_fparams": (_i, [_p, C.c_char_p]),
        "or_bin_atoms": (_i, [_p]),
        "or_bin_atoms_tds": (_i, [_p, C.c_uint64, C.c_uint32, _f]),
        "or_get_binned_counts": (_i, [_p, C.POINTER(_i), C.POINTER(_i)]),
        "or_get_binned": (_i, [_p, _p, _p, _p, _p, _p]),
        "or_apply_microscope": (_i, [_p] + [_f] * 8),
        "or_set_calc": (_i, [_p, _f, _f, _i, _i, _f, _f, _f, _f, _f, _i]),
        "or_precalc": (_i, [_p]),
        "or_get_scalars": (_i, [_p, _p]),
        "or_get_frequencies": (_i, [_p, _p, _p]),
        "or_init_waves": (_i, [_p, _f]),
        "or_stem_init_waves": (_i, [_p, _i, _i]),
        "or_set_fd_dz": (_i, [_p, _f]),
        "or_potential_conventional": (_i, [_p, _i, _p]),
        "or_potential_fd": (_i, [_p, _i, _p]),
        "or_potential_projected": (_i, [_p, _i, _f, _p]),
        "or_step_conventional": (_i, [_p, _i]),
        "or_cache_potentials": (_i, [_p, _i]),
        "or_step_given_potential": (_i, [_p, _i, _p]),
        "or_step_projected": (_i, [_p, _i]),
        "or_step_fd": (_i, [_p, _i]),
        "or_potential_rs": (_i, [_p, _i, _p]),
        "or_step_rs": (_i, [_p, _i]),
        "or_get_wave": (_i, [_p, _p]),
        "or_set_wave": (_i, [_p, _p]),
        "or_simulate_image": (_i, [_p, _p]),
        "or_alloc_tds": (_i, [_p]),
        "or_add_tds": (_i, [_p]),
        "or_get_tds": (_i, [_p, _p]),
        "or_annular_detector": (_i, [_p, _f, _f, _p]),
        "or_diffraction": (_i, [_p, _p]),
        "or_focal_forward": (_i, [_p, _p, _i, _p, _p, _i, _p, _p]),
        "or_focal_grad": (_i, [_p, _p, _i, _p, _i, _p, _p, _p]),
        "or_set_value_offset": (_i, [_p, _i, _d, _d]),
        "or_detector_chain": (_i, [_p, _p, _f, C.c_uint32, _p, _p, _i, _i, _f, C.c_uint64, _p]),
        "or_clipped_normal": (_d, [C.c_uint32, C.c_uint32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def set_threads(n: int) -> int:
    return lib().or_set_threads(int(n))


def bessk0(x: float) -> float:
    return lib().or_bessk0(float(x))


def bessi0(x: float) -> float:
    return lib().or_bessi0(float(x))


def parse_fparams(path: str) -> np.ndarray:
    out = np.zeros((103, 12), np.float64)
    n = _i(0)
    rc = lib().or_parse_fparams(path.encode(), _ptr(out), C.byref(n))
    if rc != 0:
        raise OSError(f"cannot parse {path}")
    return out[: n.value]


def vatom(fp: np.ndarray, Z: int, r2: float) -> float:
    fp = np.ascontiguousarray(fp, np.float64)
    return lib().or_vatom(_ptr(fp), int(Z), float(r2))


def vzatom2(fp: np.ndarray, Z: int, r2: float) -> float:
    fp = np.ascontiguousarray(fp, np.float64)
    return lib().or_vzatom2(_ptr(fp), int(Z), float(r2))


def fft2(a: np.ndarray, sign: int = -1) -> np.ndarray:
    b = np.ascontiguousarray(a, np.complex128).copy()
    ny, nx = b.shape
    lib().or_fft2d(_ptr(b), nx, ny, sign)
    return b


def fft1(a: np.ndarray, sign: int = -1) -> np.ndarray:
    b = np.ascontiguousarray(a, np.complex128).copy()
    lib().or_fft1d(_ptr(b), b.size, sign)
    return b


def philox(ctr, key) -> np.ndarray:
    c = np.asarray(ctr, np.uint32)
    k = np.asarray(key, np.uint32)
    o = np.zeros(4, np.uint32)
    lib().or_philox4x32_10(_ptr(c), _ptr(k), _ptr(o))
    return o


def tds_displace(x, y, z, seed: int, pas: int, sigma: float):
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    z = np.ascontiguousarray(z, np.float32)
    xo, yo, zo = np.empty_like(x), np.empty_like(y), np.empty_like(z)
    lib().or_tds_displace(_ptr(x), _ptr(y), _ptr(z), x.size, seed, pas, sigma, _ptr(xo), _ptr(yo), _ptr(zo))
    return xo, yo, zo


class OracleError(RuntimeError):
    pass


class OracleSimulation:
    """FP64 restatement of UnmanagedMultisliceSimulation (U.cu:1293-2791)."""

    def __init__(self):
        self._L = lib()
        self._handle = self._L.or_create()

    @property
    def _h(self):
        # every call passes the handle through here: a closed simulation raises
        # instead of handing a freed pointer to the C library
        if not self._handle:
            raise OracleError("oracle simulation used after close()")
        return self._handle

    def close(self):
        if self._handle:
            self._L.or_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc):
        if rc != 0:
            raise OracleError(self._L.or_last_error(self._h).decode())

    # ---- structure ----
    def ImportAtoms(self, path: str, full_table: bool = False):
        self._chk(self._L.or_import_atoms(self._h, path.encode(), int(full_table)))

    def SetAtoms(self, Z, x, y, z):
        Z = np.ascontiguousarray(Z, np.int32)
        x, y, z = (np.ascontiguousarray(a, np.float32) for a in (x, y, z))
        self._chk(self._L.or_set_atoms(self._h, _ptr(Z), _ptr(x), _ptr(y), _ptr(z), Z.size))

    def Box(self) -> np.ndarray:
        b = np.zeros(6, np.float32)
        self._chk(self._L.or_get_box(self._h, _ptr(b)))
        return b

    def GetSizeX(self):
        b = self.Box()
        return np.float32(b[0] - b[1])

    def GetSizeY(self):
        b = self.Box()
        return np.float32(b[2] - b[3])

    def GetSizeZ(self):
        b = self.Box()
        return np.float32(b[4] - b[5])

    def GetParameterisation(self, path: str):
        self._chk(self._L.or_load_fparams(self._h, path.encode()))

    def UploadBinnedAtoms(self):
        self._chk(self._L.or_bin_atoms(self._h))

    def UploadBinnedAtomsTDS(self, seed: int, pas: int, sigma: float):
        self._chk(self._L.or_bin_atoms_tds(self._h, seed, pas, sigma))

    def Binned(self):
        n, nz = _i(0), _i(0)
        self._chk(self._L.or_get_binned_counts(self._h, C.byref(n), C.byref(nz)))
        off = np.zeros(nz.value * 2500 + 1, np.int32)
        Z = np.zeros(n.value, np.int32)
        x, y, z = (np.zeros(n.value, np.float32) for _ in range(3))
        self._chk(self._L.or_get_binned(self._h, _ptr(off), _ptr(Z), _ptr(x), _ptr(y), _ptr(z)))
        return off, Z, x, y, z

    # ---- set-up ----
    def ApplyMicroscopeParameters(self, kV, df, A2, phi2, Cs, beta, delta, aperture):
        self._chk(self._L.or_apply_microscope(self._h, kV, df, A2, phi2, Cs, beta, delta, aperture))

    def SetCalculationVariables(self, ps, df, nx, ny, sx, sy, sz, xoff=0.0, yoff=0.0):
        self._chk(self._L.or_set_calc(self._h, ps, df, nx, ny, sx, sy, sz, xoff, yoff, 0))
        self.nx, self.ny = nx, ny

    def STEMSetCalculationVariables(self, ps, df, nx, ny, sx, sy, sz):
        self._chk(self._L.or_set_calc(self._h, ps, df, nx, ny, sx, sy, sz, 0.0, 0.0, 1))
        self.nx, self.ny = nx, ny

    def PreCalculateFrequencies(self):
        self._chk(self._L.or_precalc(self._h))

    def Scalars(self) -> dict:
        o = np.zeros(10, np.float64)
        self._chk(self._L.or_get_scalars(self._h, _ptr(o)))
        keys = ["wavel", "sigma2", "dzFD", "nFD", "kmax", "ke2", "convdz", "nconv", "lbx", "lby"]
        return dict(zip(keys, o.tolist()))

    def Frequencies(self):
        kx = np.zeros(self.nx, np.float32)
        ky = np.zeros(self.ny, np.float32)
        self._chk(self._L.or_get_frequencies(self._h, _ptr(kx), _ptr(ky)))
        return kx, ky

    def InitialiseWavefunctions(self, dz: float | None = None):
        self._chk(self._L.or_init_waves(self._h, -1.0 if dz is None else dz))

    def STEMInitialiseWavefunctions(self, px: int, py: int):
        self._chk(self._L.or_stem_init_waves(self._h, px, py))

    def SetFDdz(self, dz: float):
        self._chk(self._L.or_set_fd_dz(self._h, dz))

    def GetSlices(self, conventional: bool) -> int:
        s = self.Scalars()
        return int(s["nconv"] if conventional else s["nFD"])

    # ---- potentials ----
    def PotentialConventional(self, it: int) -> np.ndarray:
        out = np.zeros((self.ny, self.nx), np.float64)
        self._chk(self._L.or_potential_conventional(self._h, it, _ptr(out)))
        return out

    def PotentialFD(self, it: int) -> np.ndarray:
        out = np.zeros((self.ny, self.nx), np.float64)
        self._chk(self._L.or_potential_fd(self._h, it, _ptr(out)))
        return out

    def PotentialProjected(self, it: int, dz: float) -> np.ndarray:
        out = np.zeros((self.ny, self.nx), np.float64)
        self._chk(self._L.or_potential_projected(self._h, it, dz, _ptr(out)))
        return out

    # ---- steps ----
    def MultisliceStepConventional(self, it: int):
        self._chk(self._L.or_step_conventional(self._h, it))

    def StepGivenPotential(self, it: int, V: np.ndarray):
        """Transmission and propagation of one conventional step on V (ny, nx)."""
        v = np.ascontiguousarray(V, np.float64)
        if v.size != self.nx * self.ny:
            raise ValueError("V must hold ny * nx values")
        self._chk(self._L.or_step_given_potential(self._h, int(it), _ptr(v)))

    def CachePotentials(self, on: bool = True):
        """Reuse each iteration's conventional potential across later steps
        (many probe positions over one specimen); dropped on any set-up change."""
        self._chk(self._L.or_cache_potentials(self._h, int(bool(on))))

    def MultisliceStepProjected(self, it: int):
        self._chk(self._L.or_step_projected(self._h, it))

    def MultisliceStepFD(self, it: int):
        self._chk(self._L.or_step_fd(self._h, it))

    def MultisliceStepRS(self, it: int):
        self._chk(self._L.or_step_rs(self._h, it))

    def PotentialRS(self, it: int) -> np.ndarray:
        out = np.zeros((self.ny, self.nx), np.float64)
        self._chk(self._L.or_potential_rs(self._h, it, _ptr(out)))
        return out

    # ---- read-out ----
    def Wave(self) -> np.ndarray:
        out = np.zeros((self.ny, self.nx), np.complex128)
        self._chk(self._L.or_get_wave(self._h, _ptr(out)))
        return out

    def SetWave(self, w: np.ndarray):
        w = np.ascontiguousarray(w, np.complex128)
        self._chk(self._L.or_set_wave(self._h, _ptr(w)))

    def SimulateImage(self) -> np.ndarray:
        out = np.zeros((self.ny, self.nx), np.float64)
        self._chk(self._L.or_simulate_image(self._h, _ptr(out)))
        return out

    def AllocTDS(self):
        self._chk(self._L.or_alloc_tds(self._h))

    def AddTDSWaves(self):
        self._chk(self._L.or_add_tds(self._h))

    def TDS(self) -> np.ndarray:
        out = np.zeros((self.ny, self.nx), np.float64)
        self._chk(self._L.or_get_tds(self._h, _ptr(out)))
        return out

    def Diffraction(self) -> np.ndarray:
        out = np.zeros((self.ny, self.nx), np.float64)
        self._chk(self._L.or_diffraction(self._h, _ptr(out)))
        return out

    def AnnularDetector(self, inner_mrad: float, outer_mrad: float) -> float:
        out = _d(0)
        self._chk(self._L.or_annular_detector(self._h, inner_mrad, outer_mrad, C.byref(out)))
        return out.value

    def run_conventional(self, nslices: int | None = None):
        n = self.GetSlices(True) if nslices is None else nslices
        for i in range(1, n + 1):
            self.MultisliceStepConventional(i)
        return self.Wave()

    # ---- differentiable focal series ----
    def FocalForward(self, defoci, targets, S: int, Vstack=None):
        d = np.ascontiguousarray(defoci, np.float32)
        T = np.ascontiguousarray(targets, np.float64)
        imgs = np.zeros((d.size, self.ny, self.nx), np.float64)
        loss = _d(0)
        Vp = None
        if Vstack is not None:
            Vs = np.ascontiguousarray(Vstack, np.float64)
            Vp = _ptr(Vs)
        self._chk(self._L.or_focal_forward(self._h, _ptr(d), d.size, _ptr(T), Vp, int(S), C.byref(loss),
                                           _ptr(imgs)))
        return loss.value, imgs

    def FocalGrad(self, defoci, targets, S: int, want_xy: bool = True):
        d = np.ascontiguousarray(defoci, np.float32)
        T = np.ascontiguousarray(targets, np.float64)
        gV = np.zeros((S, self.ny, self.nx), np.float64)
        n = self.Binned()[1].size
        gxy = np.zeros((n, 2), np.float64) if want_xy else None
        loss = _d(0)
        self._chk(self._L.or_focal_grad(self._h, _ptr(d), d.size, _ptr(T), int(S), C.byref(loss), _ptr(gV),
                                        _ptr(gxy) if want_xy else None))
        return loss.value, gV, gxy

    def DetectorChain(self, I, dose: float, serial: int, dqe, ntf, binning: int, conversion: float, seed: int):
        I = np.ascontiguousarray(I, np.float64)
        d = np.ascontiguousarray(dqe, np.float32)
        t = np.ascontiguousarray(ntf, np.float32)
        out = np.zeros_like(I)
        self._chk(self._L.or_detector_chain(self._h, _ptr(I), float(dose), int(serial), _ptr(d), _ptr(t), d.size,
                                            int(binning), float(conversion), int(seed), _ptr(out)))
        return out

    def SetValueOffset(self, i: int, dx: float, dy: float):
        self._chk(self._L.or_set_value_offset(self._h, int(i), float(dx), float(dy)))


def clipped_normal(r1: int, r2: int) -> float:
    return lib().or_clipped_normal(int(r1), int(r2))
