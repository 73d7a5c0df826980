"""Fit the Gaussian expansions that the separable potential kernel uses.

For every element of ``fparams.dat`` (Kirkland's 12-parameter rows: three
Lorentzian terms a_i, b_i and three Gaussian terms c_i, d_i) this finds J
Gaussians in r^2 with positive weights,

    v(r) ~= sum_j w_j exp(-alpha_j r^2),   0.25 A <= r <= 2.2365 A,

for the atom's 3-D potential as the reference's ``vatom`` defines it
(GUI Simulation/UnmanagedGUISimulation.cu:160-193; 150.4121417 and
266.5157269 are its constants).  The lower end is ``vatom``'s 0.25 A clamp
(closer pixels take the kernel's direct path), the upper end the r^2 < 5 A^2
cut-off with a margin for the exact-position values.  A Gaussian in r^2 is
separable in the pixel's in-plane distance and the sub-plane's height, which
is what lets the kernel sum an atom's sub-planes once per atom instead of once
per pixel.

Method: variable projection (the weights solved by linear least squares for
given exponents, the log-exponents by Levenberg-Marquardt), from several
geometric starting grids, with Lawson-style reweighting toward the minimax
error relative to v(r) at every r.  The engine re-checks every expansion
against the parameter file it actually loads and uses the separable kernel
only for specimens whose elements all pass, so this table is an accelerator,
never an input to the physics.

Usage: python make_gauss_fit.py [--jobs N] [fparams.dat] [out.dat]
Writes one line per element: Z, J, max relative error, then J pairs
(alpha_j, w_j) with alpha in 1/A^2 and w in V; and the same table as C++
source, ``../csrc/ms_gauss_fit.inc``, which the engine compiles in.
``python make_gauss_fit.py --inc-only [out.dat]`` rewrites only the C++ file
from an existing table.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys

import numpy as np

J = 12
R_LO, R_HI = 0.25, 2.2365
HERE = os.path.dirname(os.path.abspath(__file__))
INC = os.path.join(os.path.dirname(HERE), "csrc", "ms_gauss_fit.inc")


def vatom(p, r):
    """vatom (U.cu:160-193) in FP64 without the clamp (r >= 0.25 here)."""
    s = sum(p[2 * i] * np.exp(-2.0 * np.pi * r * np.sqrt(p[2 * i + 1])) for i in range(3))
    g = sum(p[6 + 2 * i] * np.exp(-(np.pi * r) ** 2 / p[7 + 2 * i]) * p[7 + 2 * i] ** -1.5 for i in range(3))
    return 150.4121417 * s / r + 266.5157269 * g


def fit_row(p, nj=J, iters=20):
    import scipy.optimize as so

    r = np.geomspace(R_LO, R_HI, 600)
    rr = r * r
    f = vatom(p, r)
    if not np.all(np.isfinite(f)) or np.any(f <= 0):
        return None
    best = None
    for lo, hi in ((0.3, 100.0), (0.2, 150.0), (0.5, 80.0), (0.1, 300.0)):
        x = np.log(np.geomspace(lo, hi, nj))
        u = np.ones_like(r)
        for _ in range(iters):
            W = u / f

            def proj(x):
                A = np.exp(-np.outer(rr, np.exp(np.clip(x, -12.0, 12.0))))
                w, *_ = np.linalg.lstsq(A * W[:, None], f * W, rcond=None)
                return A, w

            def res(x):
                A, w = proj(x)
                return (A @ w - f) * W

            try:
                sol = so.least_squares(res, x, method="lm", max_nfev=300 * (nj + 1))
            except Exception:
                break
            x = sol.x
            A, w = proj(x)
            e = np.abs(A @ w - f) / f
            ok = np.all(np.isfinite(w)) and np.all(w > 0)
            err = float(e.max()) if ok else 1.0
            if best is None or err < best[0]:
                best = (err, np.exp(np.clip(x, -12.0, 12.0)), w)
            u = u * np.sqrt(e / e.max() + 1e-3)
            u /= u.mean()
    if best is None:
        return None
    # check on a finer grid than the fit's
    rf = np.geomspace(R_LO, R_HI, 20000)
    ff = vatom(p, rf)
    err, al, w = best
    efine = float(np.max(np.abs(np.exp(-np.outer(rf * rf, al)) @ w - ff) / ff))
    order = np.argsort(al)
    return efine, al[order], w[order]


def _job(args):
    z, p = args
    return z, fit_row(np.asarray(p, dtype=np.float64))


def write_inc(dat, inc=INC):
    """C++ table: kGaussFit[Z-1] = {J, alpha_0..alpha_{J-1}, w_0..w_{J-1}}."""
    rows = {}
    for line in open(dat):
        if line.startswith("#") or not line.strip():
            continue
        f = line.split()
        z, nj = int(f[0]), int(f[1])
        vals = [float(v) for v in f[3:3 + 2 * nj]]
        rows[z] = (nj, vals[0::2], vals[1::2])
    out = ["// Generated by cudamultislice_b200/data/make_gauss_fit.py from fparams.dat:",
           "// per element (row Z-1) J, then alpha_j (1/A^2), then w_j (V), of",
           "// vatom(r) ~= sum_j w_j exp(-alpha_j r^2) on 0.25 <= r <= 2.2365 A.",
           f"static const double kGaussFit[103][{1 + 2 * J}] = {{"]
    for z in range(1, 104):
        nj, al, w = rows.get(z, (0, [], []))
        if nj != J:
            out.append("    {0},")
            continue
        out.append("    {%d, %s, %s}," % (nj, ", ".join(repr(a) for a in al), ", ".join(repr(b) for b in w)))
    out.append("};")
    with open(inc, "w") as fh:
        fh.write("\n".join(out) + "\n")


def main(argv):
    if argv and argv[0] == "--inc-only":
        write_inc(argv[1] if len(argv) > 1 else os.path.join(HERE, "fparams_gauss12.dat"))
        return
    jobs = os.cpu_count() or 1
    if "--jobs" in argv:
        k = argv.index("--jobs")
        jobs = int(argv[k + 1])
        argv = argv[:k] + argv[k + 2:]
    src = argv[0] if argv else os.path.join(HERE, "fparams.dat")
    out = argv[1] if len(argv) > 1 else os.path.join(HERE, "fparams_gauss12.dat")
    P = np.loadtxt(src)
    with mp.get_context("spawn").Pool(jobs) as pool:
        results = dict(pool.map(_job, [(z + 1, P[z].tolist()) for z in range(P.shape[0])]))
    with open(out, "w") as fh:
        fh.write(f"# Gaussian expansions of vatom for {os.path.basename(src)}: Z J max_rel_err (alpha_j w_j)*J\n")
        for z in sorted(results):
            res = results[z]
            if res is None:
                fh.write(f"{z} 0 1\n")
                continue
            err, al, w = res
            pairs = " ".join(f"{a:.17g} {b:.17g}" for a, b in zip(al, w))
            fh.write(f"{z} {len(al)} {err:.3e} {pairs}\n")
            print(f"Z {z:3d}: max relative error {err:.2e}", flush=True)
    write_inc(out)


if __name__ == "__main__":
    main(sys.argv[1:])
