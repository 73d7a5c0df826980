"""The Gaussian expansions that the separable potential kernel uses
(cudamultislice_b200/data/fparams_gauss12.dat and its compiled copy
csrc/ms_gauss_fit.inc, made by data/make_gauss_fit.py) against vatom
(GUI Simulation/UnmanagedGUISimulation.cu:160-193) in FP64, for every element
of the stock parameterisation, with the exponents and weights rounded to FP32
as the engine rounds them."""
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DATA = os.path.join(ROOT, "cudamultislice_b200", "data")
INC = os.path.join(ROOT, "cudamultislice_b200", "csrc", "ms_gauss_fit.inc")
TOL = 2e-7  # the engine's acceptance bound, relative to v(r)


def _vatom(p, r):
    pi = 3.141592654
    s = sum(p[2 * i] * np.exp(-2.0 * pi * r * np.sqrt(p[2 * i + 1])) for i in range(3))
    g = sum(p[6 + 2 * i] * np.exp(-(pi * r) ** 2 / p[7 + 2 * i]) * p[7 + 2 * i] ** -1.5 for i in range(3))
    return 150.4121417 * s / r + 266.5157269 * g


def _table():
    rows = {}
    for line in open(os.path.join(DATA, "fparams_gauss12.dat")):
        if line.startswith("#"):
            continue
        f = line.split()
        nj = int(f[1])
        v = [float(t) for t in f[3:3 + 2 * nj]]
        rows[int(f[0])] = (np.array(v[0::2]), np.array(v[1::2]))
    return rows


def test_every_element_within_tolerance():
    P = np.loadtxt(os.path.join(DATA, "fparams.dat"))
    rows = _table()
    r = np.geomspace(0.25, 2.2365, 20000)
    log2e = 1.4426950408889634
    worst = 0.0
    for z in range(1, P.shape[0] + 1):
        al, w = rows[z]
        assert len(al) == 12 and np.all(w > 0) and np.all(al > 0), z
        al32 = (al * log2e).astype(np.float32).astype(np.float64)
        w32 = w.astype(np.float32).astype(np.float64)
        approx = np.exp2(-np.outer(r * r, al32)) @ w32
        v = _vatom(P[z - 1], r)
        e = float(np.max(np.abs(approx - v) / v))
        worst = max(worst, e)
        assert e < TOL, (z, e)
    assert worst < TOL


def test_compiled_copy_matches_table():
    rows = _table()
    txt = open(INC).read()
    body = txt[txt.index("{", txt.index("kGaussFit")) + 1:txt.rindex("}")]
    entries = re.findall(r"\{([^{}]*)\}", body)
    assert len(entries) == 103
    for z, e in enumerate(entries, start=1):
        vals = [float(t) for t in e.split(",") if t.strip()]
        assert int(vals[0]) == 12
        al, w = rows[z]
        assert np.array_equal(np.array(vals[1:13]), al), z
        assert np.array_equal(np.array(vals[13:25]), w), z
