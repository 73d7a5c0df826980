"""Generate golden vectors from the reference program itself.

Runs the reference engine (GUI Simulation/UnmanagedGUISimulation.cu, built
unchanged by oracle/ref_build.sh into oracle/_ref/libmsref.so) on a GPU
through the call sequence of its GUI, and stores inputs and outputs as .npz
fixtures.  tests/test_golden_reference.py checks the FP64 oracle against them
on the CPU; the reference is never needed again after generation.

  python tests/golden/make_golden_ref.py OUTDIR      (needs a CUDA GPU)

Cases use only elements of the reference's symbol table, except SrTiO3, whose
Ti the reference maps to Z = 1 (GetZNum U.cu:1241): the fixture pins that too.
"""
from __future__ import annotations

import ctypes as C
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
LIB = os.path.join(ROOT, "oracle", "_ref", "libmsref.so")


def load():
    L = C.CDLL(LIB)
    v, f, i, p = C.c_void_p, C.c_float, C.c_int, C.c_void_p
    sig = {
        "ref_create": (v, []), "ref_import_atoms": (None, [v, C.c_char_p]), "ref_upload_binned": (None, [v]),
        "ref_get_parameterisation": (None, [v]), "ref_apply": (None, [v] + [f] * 8), "ref_box": (None, [v, p]),
        "ref_set_calc": (None, [v, f, f, i, i, f, f, i]), "ref_precalc": (None, [v]), "ref_init": (None, [v, f]),
        "ref_stem_init": (None, [v, i, i]), "ref_slices": (i, [v, i]), "ref_scalars": (None, [v, p]),
        "ref_step_conv": (None, [v, i]), "ref_step_fd": (None, [v, i]), "ref_transmission": (None, [v, p, i]),
        "ref_wave": (None, [v, p, i]), "ref_exit_wave": (None, [v, p, i, p]), "ref_alloc_tds": (None, [v]),
        "ref_add_tds": (None, [v]), "ref_tds": (None, [v, p, i]),
        "ref_binned": (None, [v, i, i, p, p, p, p, p]), "ref_sync": (i, []), "ref_last_cuda_error": (C.c_char_p, []),
        "ref_step_rs": (None, [v, i]), "ref_projected": (None, [v, i, p, i]), "ref_ctf_image": (None, [v, p, i]),
    }
    for n, (r, a) in sig.items():
        fn = getattr(L, n)
        fn.restype = r
        fn.argtypes = a
    return L


def ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def xyz_text(Z, x, y, z):
    sym = {1: "H", 6: "C", 8: "O", 14: "Si", 22: "Ti", 38: "Sr", 7: "N"}
    # the reference's layout: count and comment on one line, then the atoms
    # (LoadAtomFile discards only the rest of the count line, U.cu:1309-1310)
    lines = [f"{len(Z)} golden"]
    lines += [f"{sym[int(a)]} {b:.5f} {c:.5f} {d:.5f}" for a, b, c, d in zip(Z, x, y, z)]
    return "\n".join(lines) + "\n"


def run_case(L, name, text, micro, calc, mode, dz, steps, trans_slices=(), stem_pos=None, ctf=False,
             projected_bins=()):
    ref = L.ref_create()
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "s.xyz")
        with open(path, "w") as fh:
            fh.write(text)
        L.ref_import_atoms(ref, path.encode())
    L.ref_upload_binned(ref)
    cwd = os.getcwd()
    os.chdir(os.path.join(ROOT, "cudamultislice_b200", "data"))  # GetParameterisation reads ./fparams.dat
    try:
        L.ref_get_parameterisation(ref)
    finally:
        os.chdir(cwd)
    L.ref_apply(ref, *micro)
    ps, df, nx, ny, xoff, yoff, stem = calc
    L.ref_set_calc(ref, ps, df, nx, ny, xoff, yoff, stem)
    L.ref_precalc(ref)
    N = nx * ny
    out = {"xyz": np.array(text), "micro": np.array(micro, np.float32), "calc": np.array(calc[:2] + calc[4:6], np.float32),
           "grid": np.array([nx, ny, stem], np.int32), "mode": np.array(mode), "dz": np.float32(dz)}
    box = np.zeros(6, np.float32)
    L.ref_box(ref, ptr(box))
    out["box"] = box
    # atom index
    n = int(text.split()[0])
    nz = int(np.ceil(np.float32(box[4] - box[5])))
    nz += nz == 0
    off = np.zeros(nz * 2500 + 1, np.int32)
    Zb = np.zeros(n, np.int32)
    xb, yb, zb = (np.zeros(n, np.float32) for _ in range(3))
    L.ref_binned(ref, n, nz * 2500, ptr(off), ptr(Zb), ptr(xb), ptr(yb), ptr(zb))
    out.update(off=off, bZ=Zb, bx=xb, by=yb, bz=zb)
    if mode == "fd":
        L.ref_init(ref, -1.0)
    else:
        L.ref_init(ref, dz)
    if stem_pos is not None:
        L.ref_alloc_tds(ref)
        L.ref_stem_init(ref, stem_pos[0], stem_pos[1])
    sc = np.zeros(6, np.float32)
    L.ref_scalars(ref, ptr(sc))
    out["scalars"] = sc
    nsteps = L.ref_slices(ref, 1) if steps is None else steps
    out["nsteps"] = np.int32(nsteps)
    for i in range(1, nsteps + 1):
        if mode == "fd":
            L.ref_step_fd(ref, i)
        elif mode == "rs":
            L.ref_step_rs(ref, i)
            if i in trans_slices:  # devV = {RS potential, 0} of this step
                t = np.zeros(2 * N, np.float32)
                L.ref_transmission(ref, ptr(t), N)
                out[f"rspot_{i}"] = t[0::2].reshape(ny, nx).copy()
        else:
            L.ref_step_conv(ref, i)
            if i in trans_slices:
                t = np.zeros(2 * N, np.float32)
                L.ref_transmission(ref, ptr(t), N)
                out[f"trans_{i}"] = t.view(np.complex64).reshape(ny, nx)
    w = np.zeros(2 * N, np.float32)
    L.ref_wave(ref, ptr(w), N)
    out["wave"] = w.view(np.complex64).reshape(ny, nx)
    if ctf:  # imagingKernel2 on this wave, as SimulateImage applies it
        im = np.zeros(2 * N, np.float32)
        L.ref_ctf_image(ref, ptr(im), N)
        out["ctf_image"] = im.view(np.complex64).reshape(ny, nx)
    for b in projected_bins:  # binnedAtomPKernel2 over one-angstrom z-bin b
        t = np.zeros(2 * N, np.float32)
        L.ref_projected(ref, b, ptr(t), N)
        out[f"proj_{b}"] = t.view(np.complex64).reshape(ny, nx)
    if stem_pos is not None:
        L.ref_add_tds(ref)
        tds = np.zeros(N, np.float32)
        L.ref_tds(ref, ptr(tds), N)
        out["tds"] = tds.reshape(ny, nx)
        out["stem_pos"] = np.array(stem_pos, np.int32)
    else:
        mm = np.zeros(2, np.float32)
        ew = np.zeros(2 * N, np.float32)
        L.ref_exit_wave(ref, ptr(ew), N, ptr(mm))
        out["ew_minmax"] = mm
    rc = L.ref_sync()
    if rc != 0:
        raise RuntimeError(f"{name}: CUDA error {rc}: {L.ref_last_cuda_error().decode()}")
    if not np.all(np.isfinite(out["wave"])):
        raise RuntimeError(f"{name}: non-finite wave")
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden_ref.py OUTDIR")
    outdir = sys.argv[1]
    os.makedirs(outdir, exist_ok=True)
    from cudamultislice_b200 import structures as S

    L = load()
    sto = xyz_text(*S.srtio3(2, 2, 4))
    rnd = xyz_text(*S.random_atoms(150, size=(12.0, 12.0, 10.0), Zs=(6, 8, 14, 38), seed=0x5EED))
    cases = {
        # TEM conventional (MultisliceStepConv), SrTiO3 with Ti -> H as the reference
        "ref_sto_conv_128": dict(text=sto, micro=(200.0, -500.0, 0.0, 0.0, 1e7, 0.1, 30.0, 20.0),
                                 calc=(0.1, -500.0, 128, 128, 2.0, 2.0, 0), mode="conv", dz=1.9525, steps=None,
                                 trans_slices=(1, 3)),
        # random C/O/Si/Sr, 256^2, 300 kV, 1 A slices, offsets
        "ref_rand_conv_256": dict(text=rnd, micro=(300.0, 100.0, 0.0, 0.0, 1.2e7, 0.1, 30.0, 25.0),
                                  calc=(0.0625, 100.0, 256, 256, 1.5, 0.5, 0), mode="conv", dz=1.0, steps=None,
                                  trans_slices=(2, 5)),
        # STEM probe through conventional slices, CBED amplitude (AddTDSWaves)
        "ref_sto_stem_128": dict(text=sto, micro=(300.0, 0.0, 0.0, 0.0, 0.0, 0.1, 30.0, 25.0),
                                 calc=(0.1, 0.0, 128, 128, 0.0, 0.0, 1), mode="conv", dz=1.0, steps=None,
                                 stem_pos=(40, 70)),
        # finite differences with the reference's automatic stable step, 30 steps
        "ref_sto_fd_128": dict(text=sto, micro=(200.0, 0.0, 0.0, 0.0, 1e7, 0.1, 30.0, 20.0),
                               calc=(0.1, 0.0, 128, 128, 0.0, 0.0, 0), mode="fd", dz=-1.0, steps=30),
        # MultisliceStepRS as written, 5 steps, with the RS potential of steps 2 and 4
        "ref_sto_rs_128": dict(text=sto, micro=(200.0, 0.0, 0.0, 0.0, 1e7, 0.1, 30.0, 20.0),
                               calc=(0.1, 0.0, 128, 128, 2.0, 2.0, 0), mode="rs", dz=1.9525, steps=5,
                               trans_slices=(2, 4)),
        # the CTF image (imagingKernel2) of a conventional exit wave, with two-fold
        # astigmatism and both coherence envelopes
        "ref_sto_ctf_128": dict(text=sto, micro=(200.0, -500.0, 30.0, 0.4, 1e7, 0.5, 30.0, 20.0),
                                calc=(0.1, -500.0, 128, 128, 2.0, 2.0, 0), mode="conv", dz=1.9525, steps=None,
                                ctf=True),
        # the projected potential (binnedAtomPKernel2, vzatom2) of three z-bins of
        # the random structure
        "ref_rand_proj_256": dict(text=rnd, micro=(300.0, 100.0, 0.0, 0.0, 1.2e7, 0.1, 30.0, 25.0),
                                  calc=(0.0625, 100.0, 256, 256, 1.5, 0.5, 0), mode="conv", dz=1.0, steps=1,
                                  projected_bins=(3, 6, 9)),
    }
    for name, kw in cases.items():
        out = run_case(L, name, **kw)
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **out)
        print(name, "ok", {k: v.shape for k, v in out.items() if hasattr(v, "shape")}["wave"], flush=True)


if __name__ == "__main__":
    main()
