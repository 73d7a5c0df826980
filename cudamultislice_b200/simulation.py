"""Python mirror of the reference's simulation API over the C ABI.

``ManagedMultisliceSimulation`` has the method list of the reference's .NET
wrapper (GUI Simulation/GUI Simulation.h:17-59, ManagedMultislice.cpp), so a
script written against the reference's call sequence runs unchanged:

    sim = ManagedMultisliceSimulation()
    sim.ImportAtoms("structure.xyz")
    sim.UploadBinnedAtoms()
    sim.GetParameterisation("fparams.dat")
    sim.ApplyMicroscopeParameters(kV, df, A2, phi2, Cs, beta, delta, aperture)
    sim.SetCalculationVariables(ps, df, nx, ny, sim.GetSizeX(), sim.GetSizeY(), sim.GetSizeZ(), xoff, yoff)
    sim.PreCalculateFrequencies()
    sim.InitialiseWavefunctions(dz)
    for i in range(1, sim.GetSlices(True) + 1):
        sim.MultisliceStepConventional(i)
    sim.GetExitWave()

Every call goes to ``libmslice_b200.so`` (hand-written sm_100a kernels); there
is no CPU implementation behind it.  Errors raise ``MultisliceError`` with the
library's message instead of being ignored.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import MultisliceError, lib

_p = C.c_void_p


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class ManagedMultisliceSimulation:
    """One engine handle (ms_sim) on one GPU."""

    SLICE_PATH_FUSED = 0
    SLICE_PATH_PLAIN = 1

    def __init__(self, device: int = 0):
        self._L = lib()
        h = C.c_void_p()
        rc = self._L.ms_create(int(device), C.byref(h))
        if rc != 0:
            raise MultisliceError(rc, self._L.ms_last_error(None).decode())
        self._h = h
        self.nx = self.ny = 0

    # ---- lifecycle ----
    def close(self):
        if getattr(self, "_h", None):
            self._L.ms_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _chk(self, rc: int):
        if rc != 0:
            raise MultisliceError(rc, self._L.ms_last_error(self._h).decode())

    def _f(self, fn, *args) -> float:
        out = C.c_float()
        self._chk(fn(self._h, *args, C.byref(out)))
        return out.value

    # ---- options ----
    def SetSlicePath(self, path: int):
        self._chk(self._L.ms_set_option(self._h, 0, int(path)))

    def SetElementTable(self, full: bool):
        self._chk(self._L.ms_set_option(self._h, 1, int(bool(full))))

    def SetPotentialMode(self, projected: bool):
        self._chk(self._L.ms_set_option(self._h, 2, int(bool(projected))))

    def SetFFTPlan(self, variant: int):
        """-1: autotuned; 0..5: force a plan variant of the fused passes (3..5: packed butterflies)."""
        self._chk(self._L.ms_set_option(self._h, 3, int(variant)))

    def SetCheckpoint(self, stride: int):
        """Focal-series gradient: slices between stored waves (0: automatic, every
        wave when they fit in an eighth of free device memory, else ceil(sqrt(S)))."""
        self._chk(self._L.ms_set_option(self._h, 4, int(stride)))

    def SetSliceLoop(self, persistent: bool):
        """Conventional slice loop on square 256/512/1024 grids: one persistent
        cooperative launch for all slices (True, the default) or one launch per
        row and column pass (False)."""
        self._chk(self._L.ms_set_option(self._h, 5, 0 if persistent else 1))

    def SetLoopVariant(self, variant: int):
        """Persistent slice loop kernel variant: -1 tuned (default), 0..4 forced."""
        self._chk(self._L.ms_set_option(self._h, 8, int(variant)))

    def SliceLoop(self):
        """(variant, columns per unit, CTAs) of the persistent loop on this grid (variant -1: not used)."""
        v, c, g = C.c_int(), C.c_int(), C.c_int()
        self._chk(self._L.ms_get_slice_loop(self._h, C.byref(v), C.byref(c), C.byref(g)))
        return v.value, c.value, g.value

    def SetPotentialTile(self, tile: int):
        """Conventional potential kernel tile: -1 tuned (default); separable kernel
        0..3 = 16x32, 32x16, 16x64, 32x32 pixels, per sub-plane 0..2 = 32x8, 16x16, 64x4."""
        self._chk(self._L.ms_set_option(self._h, 9, int(tile)))

    def SetBuildOverlap(self, on: bool):
        """RunConventional with a stack to build: overlap each slice's passes
        with the next slices' potentials (True, the default) or build first."""
        self._chk(self._L.ms_set_option(self._h, 11, 1 if on else 0))

    def SetPotentialSum(self, mode: int):
        """Conventional potential's sub-plane sum: 0 separable where it applies
        (default), 1 per (pixel, atom, sub-plane), 2 separable or an error."""
        self._chk(self._L.ms_set_option(self._h, 10, int(mode)))

    def PotentialSum(self):
        """(last, next): how the last conventional potential was summed and how
        the next would be (1 per sub-plane, 2 separable; last 0: none yet)."""
        a, b = C.c_int(), C.c_int()
        self._chk(self._L.ms_get_potential_sum(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def RasterTuning(self):
        """(probes per launch, 1 if the slices ran in the batched persistent loop) of the last raster."""
        b, p = C.c_int(), C.c_int()
        self._chk(self._L.ms_get_raster_tuning(self._h, C.byref(b), C.byref(p)))
        return b.value, p.value

    def SetLoopWaitUs(self, us: int):
        """Bound on each grid-barrier wait of the persistent loop (microseconds)."""
        self._chk(self._L.ms_set_option(self._h, 6, int(us)))

    def SetLoopWaitTest(self, extra: int):
        """Test hook: every grid barrier waits for `extra` arrivals that never come."""
        self._chk(self._L.ms_set_option(self._h, 7, int(extra)))

    # ---- structure ----
    def ImportAtoms(self, filename: str):
        self._chk(self._L.ms_import_atoms(self._h, filename.encode()))

    def SetAtoms(self, Z, x, y, z):
        Z = np.ascontiguousarray(Z, np.int32)
        x, y, z = (np.ascontiguousarray(a, np.float32) for a in (x, y, z))
        if not (Z.size == x.size == y.size == z.size):
            raise ValueError("Z, x, y, z must have the same length")
        self._chk(self._L.ms_set_atoms(self._h, _ptr(Z), _ptr(x), _ptr(y), _ptr(z), Z.size))

    def UploadBinnedAtoms(self):
        self._chk(self._L.ms_upload_binned_atoms(self._h))

    def UploadBinnedAtomsTDS(self, seed: int = 0x5EED2026, pas: int = 0, sigma: float = 0.075):
        self._chk(self._L.ms_upload_binned_atoms_tds(self._h, int(seed), int(pas), float(sigma)))

    def GetParameterisation(self, path: str):
        self._chk(self._L.ms_get_parameterisation(self._h, path.encode()))

    # ---- set-up ----
    def ApplyMicroscopeParameters(self, Voltage, defocus, Mod2f, Arg2f, spherical, B, D, obj):
        self._chk(self._L.ms_apply_microscope_parameters(
            self._h, Voltage, defocus, Mod2f, Arg2f, spherical, B, D, obj))

    def SetCalculationVariables(self, PixelScaleIn, defocus, resX, resY, SizeX, SizeY, SizeZ,
                                blockoffsetx=0.0, blockoffsety=0.0):
        self._chk(self._L.ms_set_calculation_variables(
            self._h, PixelScaleIn, defocus, int(resX), int(resY), SizeX, SizeY, SizeZ, blockoffsetx, blockoffsety))
        self.nx, self.ny = int(resX), int(resY)

    def STEMSetCalculationVariables(self, PixelScaleIn, defocus, resX, resY, SizeX, SizeY, SizeZ):
        self._chk(self._L.ms_stem_set_calculation_variables(
            self._h, PixelScaleIn, defocus, int(resX), int(resY), SizeX, SizeY, SizeZ))
        self.nx, self.ny = int(resX), int(resY)

    def PreCalculateFrequencies(self):
        self._chk(self._L.ms_precalculate_frequencies(self._h))

    def InitialiseWavefunctions(self, dz: float | None = None):
        if dz is None:
            self._chk(self._L.ms_initialise_wavefunctions(self._h))
        else:
            self._chk(self._L.ms_initialise_wavefunctions_dz(self._h, float(dz)))

    def STEMInitialiseWavefunctions(self, posx: int, posy: int):
        self._chk(self._L.ms_stem_initialise_wavefunctions(self._h, int(posx), int(posy)))

    def SetFDdz(self, dz: float):
        self._chk(self._L.ms_set_fd_dz(self._h, float(dz)))

    # ---- steps ----
    def MultisliceStepFD(self, iteration: int):
        self._chk(self._L.ms_multislice_step_fd(self._h, int(iteration)))

    def MultisliceStepConventional(self, iteration: int):
        self._chk(self._L.ms_multislice_step_conventional(self._h, int(iteration)))

    def MultisliceStepRS(self, iteration: int):
        """MultisliceStepRS as written (not exposed by the reference's wrapper)."""
        self._chk(self._L.ms_multislice_step_rs(self._h, int(iteration)))

    # ---- queries ----
    def GetSizeX(self) -> float:
        return self._f(self._L.ms_get_size_x)

    def GetSizeY(self) -> float:
        return self._f(self._L.ms_get_size_y)

    def GetSizeZ(self) -> float:
        return self._f(self._L.ms_get_size_z)

    def GetSlices(self, conventional: bool) -> int:
        out = C.c_int()
        self._chk(self._L.ms_get_slices(self._h, int(bool(conventional)), C.byref(out)))
        return out.value

    def GetKmax(self) -> float:
        return self._f(self._L.ms_get_kmax)

    # ---- read-out ----
    def GetExitWave(self):
        self._chk(self._L.ms_get_exit_wave(self._h))

    def GetSTEMExitWave(self):
        self._chk(self._L.ms_get_stem_exit_wave(self._h))

    def FreeExitWave(self):
        self._chk(self._L.ms_free_exit_wave(self._h))

    def GetEWValueAbs(self, x, y) -> float:
        return self._f(self._L.ms_get_ew_value_abs, int(x), int(y))

    def GetEWValueRe(self, x, y) -> float:
        return self._f(self._L.ms_get_ew_value_re, int(x), int(y))

    def GetEWValueIm(self, x, y) -> float:
        return self._f(self._L.ms_get_ew_value_im, int(x), int(y))

    def GetEWMin(self) -> float:
        return self._f(self._L.ms_get_ew_min)

    def GetEWMax(self) -> float:
        return self._f(self._L.ms_get_ew_max)

    def AllocTDS(self):
        self._chk(self._L.ms_alloc_tds(self._h))

    def AddTDSWaves(self):
        self._chk(self._L.ms_add_tds_waves(self._h))

    def GetTDSMin(self) -> float:
        return self._f(self._L.ms_get_tds_min)

    def GetTDSMax(self) -> float:
        return self._f(self._L.ms_get_tds_max)

    def GetTDSVal(self, x, y) -> float:
        return self._f(self._L.ms_get_tds_val, int(x), int(y))

    def AllocHostImage(self):
        self._chk(self._L.ms_alloc_host_image(self._h))

    def SimulateImage(self, doseperpix: float = 0.0):
        self._chk(self._L.ms_simulate_image(self._h, float(doseperpix)))

    def GetImValue(self, x, y) -> float:
        return self._f(self._L.ms_get_im_value, int(x), int(y))

    def GetDQEImValue(self, x, y) -> float:
        return self._f(self._L.ms_get_dqe_im_value, int(x), int(y))

    def GetImMin(self) -> float:
        return self._f(self._L.ms_get_im_min)

    def GetImMax(self) -> float:
        return self._f(self._L.ms_get_im_max)

    def GetImageContrast(self, t, l, b, r) -> float:
        return self._f(self._L.ms_get_image_contrast, int(t), int(l), int(b), int(r))

    # ---- bulk and batched (new) ----
    def ExitWave(self, out: np.ndarray | None = None) -> np.ndarray:
        """The exit wave (ny, nx) complex64; `out` (C-contiguous, that shape and
        dtype, e.g. a view of pinned host memory) receives it when given."""
        if out is None:
            out = np.empty((self.ny, self.nx), np.complex64)
        elif out.shape != (self.ny, self.nx) or out.dtype != np.complex64 or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous complex64 array of shape {(self.ny, self.nx)}")
        self._chk(self._L.ms_copy_exit_wave(self._h, _ptr(out)))
        return out

    def Image(self) -> np.ndarray:
        out = np.zeros((self.ny, self.nx), np.float32)
        self._chk(self._L.ms_copy_image(self._h, _ptr(out)))
        return out

    def TDS(self) -> np.ndarray:
        out = np.zeros((self.ny, self.nx), np.float32)
        self._chk(self._L.ms_copy_tds(self._h, _ptr(out)))
        return out

    def BuildPotentialStack(self) -> int:
        out = C.c_int()
        self._chk(self._L.ms_build_potential_stack(self._h, C.byref(out)))
        return out.value

    def RunConventional(self) -> int:
        out = C.c_int()
        self._chk(self._L.ms_run_conventional(self._h, C.byref(out)))
        return out.value

    def RunFD(self, nsteps: int = 0) -> int:
        """Finite-difference steps 1..nsteps (0: GetSlices(False)) from the
        initial waves; returns the step count (device time: LastDeviceMs)."""
        out = C.c_int()
        self._chk(self._L.ms_run_fd(self._h, int(nsteps), C.byref(out)))
        return out.value

    def AnnularDetector(self, inner_mrad: float, outer_mrad: float) -> float:
        out = C.c_double()
        self._chk(self._L.ms_annular_detector(self._h, float(inner_mrad), float(outer_mrad), C.byref(out)))
        return out.value

    def StemRaster(self, px, py, inner_mrad: float, outer_mrad: float, batch: int = 16) -> np.ndarray:
        """Annular-detector signal for every probe position (pixels)."""
        px = np.ascontiguousarray(px, np.int32).ravel()
        py = np.ascontiguousarray(py, np.int32).ravel()
        if px.size != py.size:
            raise ValueError("px and py must have the same length")
        out = np.zeros(px.size, np.float64)
        self._chk(self._L.ms_stem_raster(self._h, _ptr(px), _ptr(py), px.size, float(inner_mrad),
                                         float(outer_mrad), int(batch), _ptr(out)))
        return out

    def SetDetector(self, dqe, ntf, binning: int = 4, conversion: float = 8.0, readout_offset: float = 4.0,
                    readout_sigma: float = 1.33, seed: int = 0x5EED2026):
        """Detector model of SimulateImage's noisy chain (radial DQE/NTF tables);
        dqe=None removes it.  The defaults are the reference's constants."""
        if dqe is None:
            self._chk(self._L.ms_set_detector(self._h, None, None, 0, int(binning), float(conversion),
                                              float(readout_offset), float(readout_sigma), int(seed)))
            return
        d = np.ascontiguousarray(dqe, np.float32).ravel()
        t = np.ascontiguousarray(ntf, np.float32).ravel()
        if d.size != t.size:
            raise ValueError("DQE and NTF tables must have the same length")
        self._chk(self._L.ms_set_detector(self._h, _ptr(d), _ptr(t), d.size, int(binning), float(conversion),
                                          float(readout_offset), float(readout_sigma), int(seed)))

    def WriteTIFF(self, what: int, path: str):
        """Float32 TIFF: 0 image, 1 / 2 exit-wave real / imaginary, 3 TDS/CBED, 4 amplitude."""
        self._chk(self._L.ms_write_tiff(self._h, int(what), path.encode()))

    def SimulateImageSeries(self, defoci, cs=None) -> np.ndarray:
        """CTF images of the current exit wave at each defocus (and Cs), (n, ny, nx)."""
        d = np.ascontiguousarray(defoci, np.float32).ravel()
        c = None if cs is None else np.ascontiguousarray(cs, np.float32).ravel()
        if c is not None and c.size != d.size:
            raise ValueError("defoci and cs must have the same length")
        out = np.zeros((d.size, self.ny, self.nx), np.float32)
        self._chk(self._L.ms_simulate_image_series(self._h, _ptr(d), None if c is None else _ptr(c), d.size,
                                                   _ptr(out)))
        return out

    # ---- frozen phonons ----
    def FrozenPhonon(self, seed: int, first_pass: int, nconfigs: int, sigma: float, batch: int = 16,
                     diffraction: bool = True, image: bool = True):
        """Sum of centred |FFT(psi_exit)| and mean CTF image over thermal configurations."""
        d = np.zeros((self.ny, self.nx), np.float32) if diffraction else None
        im = np.zeros((self.ny, self.nx), np.float32) if image else None
        self._chk(self._L.ms_frozen_phonon(self._h, int(seed), int(first_pass), int(nconfigs), float(sigma),
                                           int(batch), _ptr(d) if diffraction else None,
                                           _ptr(im) if image else None))
        return d, im

    # ---- differentiable focal series ----
    def FocalSeries(self, defoci, targets, nslices: int, images: bool = False):
        """Loss sum_d sum_px (I_d - T_d)^2 of the CTF images at `defoci` (A) of
        the wave after conventional slices 1..nslices; with `images`, also the
        simulated images (nd, ny, nx)."""
        d = np.ascontiguousarray(defoci, np.float32).ravel()
        T = np.ascontiguousarray(targets, np.float32)
        if T.size != d.size * self.nx * self.ny:
            raise ValueError("targets must hold nd * ny * nx values")
        loss = C.c_double()
        imgs = np.zeros((d.size, self.ny, self.nx), np.float32) if images else None
        self._chk(self._L.ms_focal_series(self._h, _ptr(d), d.size, _ptr(T), int(nslices), C.byref(loss),
                                          _ptr(imgs) if images else None))
        return (loss.value, imgs) if images else loss.value

    def FocalSeriesGrad(self, defoci, targets, nslices: int, want_v: bool = True, want_xy: bool = True):
        """Loss, dL/dV (nslices, ny, nx) and dL/dxy (n_atoms, 2; input order)."""
        d = np.ascontiguousarray(defoci, np.float32).ravel()
        T = np.ascontiguousarray(targets, np.float32)
        if T.size != d.size * self.nx * self.ny:
            raise ValueError("targets must hold nd * ny * nx values")
        loss = C.c_double()
        gV = np.zeros((int(nslices), self.ny, self.nx), np.float32) if want_v else None
        gxy = None
        if want_xy:
            n, nz = C.c_int(), C.c_int()
            self._chk(self._L.ms_get_binned_counts(self._h, C.byref(n), C.byref(nz)))
            gxy = np.zeros((n.value, 2), np.float64)
        self._chk(self._L.ms_focal_series_grad(self._h, _ptr(d), d.size, _ptr(T), int(nslices), C.byref(loss),
                                               _ptr(gV) if want_v else None, _ptr(gxy) if want_xy else None))
        return loss.value, gV, gxy

    def TimePass(self, pass_: int, op: int, variant: int, batch: int = 1, reps: int = 20) -> float:
        """Microseconds per launch of one fused pass (see ms_time_pass)."""
        out = C.c_float()
        self._chk(self._L.ms_time_pass(self._h, int(pass_), int(op), int(variant), int(batch), int(reps),
                                       C.byref(out)))
        return out.value

    def LastDeviceMs(self) -> float:
        out = C.c_float()
        self._chk(self._L.ms_get_last_device_ms(self._h, C.byref(out)))
        return out.value

    # ---- inspection ----
    def Binned(self):
        n, nz = C.c_int(), C.c_int()
        self._chk(self._L.ms_get_binned_counts(self._h, C.byref(n), C.byref(nz)))
        off = np.zeros(nz.value * 2500 + 1, np.int32)
        Z = np.zeros(n.value, np.int32)
        x, y, z = (np.zeros(n.value, np.float32) for _ in range(3))
        self._chk(self._L.ms_copy_binned(self._h, _ptr(off), _ptr(Z), _ptr(x), _ptr(y), _ptr(z)))
        return off, Z, x, y, z

    def PotentialSlice(self, kind: int, iteration: int) -> np.ndarray:
        out = np.zeros((self.ny, self.nx), np.float32)
        self._chk(self._L.ms_copy_potential_slice(self._h, int(kind), int(iteration), _ptr(out)))
        return out

    def FFT2(self, a: np.ndarray, sign: int = -1) -> np.ndarray:
        a = np.ascontiguousarray(a, np.complex64)
        out = np.zeros_like(a)
        ny, nx = a.shape
        self._chk(self._L.ms_fft2(self._h, _ptr(a), _ptr(out), nx, ny, int(sign)))
        return out

    def TimeSlices(self, steps: int, reps: int = 1, breakdown: bool = True):
        """Device time (ms) of reps x steps conventional steps over the
        resident potential stack; with `breakdown`, also the average duration
        of one row pass and one column pass (fused path)."""
        t, a, b = C.c_float(), C.c_float(), C.c_float()
        if breakdown:
            self._chk(self._L.ms_time_slices(self._h, int(steps), int(reps), C.byref(t), C.byref(a), C.byref(b)))
            return t.value, a.value, b.value
        self._chk(self._L.ms_time_slices(self._h, int(steps), int(reps), C.byref(t), None, None))
        return t.value, None, None

    def FFTPlan(self, batch: int = 1):
        """(row, column) FFT plan variants used for `batch` instances."""
        r, c = C.c_int(), C.c_int()
        self._chk(self._L.ms_get_fft_plan(self._h, int(batch), C.byref(r), C.byref(c)))
        return r.value, c.value

    def LaunchCount(self) -> int:
        out = C.c_longlong()
        self._chk(self._L.ms_get_launch_count(self._h, C.byref(out)))
        return out.value


def stem_raster_concurrent(sims, positions, inner_mrad: float, outer_mrad: float, batch: int = 16):
    """Probe rasters of several handles (different specimens and grid sizes) in
    one CUDA-graph launch; positions[k] = (px, py) for sims[k].  Returns the
    signals per handle and the device milliseconds of the launch."""
    k = len(sims)
    pxs = [np.ascontiguousarray(p[0], np.int32).ravel() for p in positions]
    pys = [np.ascontiguousarray(p[1], np.int32).ravel() for p in positions]
    outs = [np.zeros(a.size, np.float64) for a in pxs]
    hs = (C.c_void_p * k)(*[s._h for s in sims])
    PX = (C.c_void_p * k)(*[a.ctypes.data for a in pxs])
    PY = (C.c_void_p * k)(*[a.ctypes.data for a in pys])
    NN = (C.c_int * k)(*[a.size for a in pxs])
    OUT = (C.c_void_p * k)(*[o.ctypes.data for o in outs])
    sims[0]._chk(sims[0]._L.ms_stem_raster_concurrent(hs, k, PX, PY, NN, float(inner_mrad), float(outer_mrad),
                                                      int(batch), OUT))
    return outs, sims[0].LastDeviceMs()


def write_tiff(path: str, data) -> None:
    """Float32 TIFF of a 2D array (the library's writer, no GPU needed)."""
    a = np.ascontiguousarray(data, np.float32)
    if a.ndim != 2:
        raise ValueError("need a 2D array")
    L = lib()
    rc = L.ms_write_tiff_f32(path.encode(), a.ctypes.data_as(C.c_void_p), a.shape[1], a.shape[0])
    if rc != 0:
        raise MultisliceError(rc, (L.ms_last_error(None) or b"").decode())
