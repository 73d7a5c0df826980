"""The FP32 error floor of a multislice run: the same slice recursion as the
engine, psi <- IFFT(P * FFT(t * psi)), once in complex128 and once with the
transforms in complex64 (scipy.fft's single-precision pocketfft), the
potentials from the FP64 oracle.  It shows how far from FP64 an ideal FP32
implementation lands on a workload, which sets what the engine's parity
tolerances can ask of FP32 arithmetic (tests/test_gpu_full_depth.py).

  python tests/fp32_floor_model.py [512|1024]

Workload: the GaN [11-20] STEM probe of the HAADF configuration (300 kV,
25 mrad, Cs = 0, df = 0, 1.5945 A slices, 80+ slices), 10x6x40 cells on
1024^2 or 5x3x40 on 512^2.  Printed: the relative L2 exit-wave error for
each combination of FP32 transforms, FP32-rounded propagator and
FP32-rounded transmission (True = FP32), and for the separable propagator
px * py rounded to FP32 as the fused column pass forms it.  Measured (1024^2):
FP32 transforms alone 1.0e-5; propagator rounding alone 1.2e-6 (separable
2.0e-6); transmission rounding alone 8e-8.  Test infrastructure: reads the
oracle, never the engine."""
import os
import sys

import numpy as np
import scipy.fft as sf

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from cudamultislice_b200 import FPARAMS  # noqa: E402
from cudamultislice_b200 import structures as S  # noqa: E402
from oracle import oracle  # noqa: E402


def main(n: int) -> None:
    oracle.build()
    atoms = S.gan_wurtzite_11_20(*((10, 6, 40) if n == 1024 else (5, 3, 40)))
    o = oracle.OracleSimulation()
    o.SetAtoms(*atoms)
    o.UploadBinnedAtoms()
    o.GetParameterisation(FPARAMS)
    o.ApplyMicroscopeParameters(300, 0, 0, 0, 0, 0.1, 30, 25)
    ps = o.GetSizeX() / n
    o.STEMSetCalculationVariables(ps, 0, n, n, o.GetSizeX(), o.GetSizeY(), o.GetSizeZ())
    o.PreCalculateFrequencies()
    o.InitialiseWavefunctions(1.5945)
    o.STEMInitialiseWavefunctions(n // 2 + 13, n // 2 + 7)
    psi0 = o.Wave()
    nsl = o.GetSlices(True)
    V = [o.PotentialConventional(i) for i in range(1, nsl + 1)]
    sc = o.Scalars()
    sig, lam, dz = sc["sigma2"], sc["wavel"], 1.5945
    kx, ky = o.Frequencies()
    KX, KY = np.meshgrid(kx.astype(np.float64), ky.astype(np.float64))
    k2 = KX ** 2 + KY ** 2
    mask = np.sqrt(k2.astype(np.float32)) < sc["kmax"]
    P = np.where(mask, np.exp(-1j * np.pi * dz * lam * k2), 0)
    T = [np.exp(1j * sig * v) for v in V]

    def run(fft32, p32, t32, Puse=None):
        psi = psi0.astype(np.complex64 if fft32 else np.complex128)
        Pp = Puse if Puse is not None else (P.astype(np.complex64) if p32 else P)
        for i in range(nsl):
            x = (T[i].astype(np.complex64) if t32 else T[i]) * psi
            F = sf.fft2(x.astype(np.complex64) if fft32 else x) * Pp
            psi = sf.ifft2(F.astype(np.complex64) if fft32 else F)
        return psi.astype(np.complex128)

    ref = run(False, False, False)
    err = lambda w: float(np.linalg.norm(w - ref) / np.linalg.norm(ref))  # noqa: E731
    print(f"{n}^2, {nsl} slices")
    for cfg in [(True, True, True), (True, False, False), (False, True, False), (False, False, True)]:
        print("fft32, P32, t32 =", cfg, err(run(*cfg)))
    pxv = np.exp(-1j * np.pi * dz * lam * kx.astype(np.float64) ** 2)
    pyv = np.exp(-1j * np.pi * dz * lam * ky.astype(np.float64) ** 2)
    Psep = np.where(mask, pxv.astype(np.complex64)[None, :] * pyv.astype(np.complex64)[:, None], 0)
    print("separable propagator rounded to FP32 only:", err(run(False, False, False, Psep.astype(np.complex64))))


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 512)
