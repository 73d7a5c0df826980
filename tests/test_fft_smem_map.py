"""Shared-memory bank conflicts of the line FFT (CPU check of the map in
cudamultislice_b200/csrc/ms_fft.cuh, padi()).

Every plan of the PlanSel table (parsed from ms_slice_impl.cuh) is walked
through its exchanges: first-pass writes (R1 apart), middle-pass reads
(consecutive) and writes (groups of NS), last-pass reads.  A 64-bit access of a
half-warp (16 lanes) is one wavefront when its points fall in 16 distinct
(point mod 16) classes; lines shorter than 16 threads share a half-warp across
slots SLOT points apart.  The plans that use the XOR map must be
conflict-free.

The column pass (k_pass_b) runs the same plans on the padded map with CW
columns interleaved per warp row (thread t * CW + c of a group owns index t
of column c; slots 16/CW points mod 16 apart): every exchange of every plan
must be conflict-free there too."""
import os
import re
from collections import Counter

import pytest

from tests.conftest import ROOT

IMPL = os.path.join(ROOT, "cudamultislice_b200", "csrc", "ms_slice_impl.cuh")


def plans(packed=False):
    """(length, variant, N, E, radices) of every PlanSel entry; the packed
    variants (3..5, butterflies on FP32x2) with packed=True."""
    text = open(IMPL).read()
    out = []
    pat = (r"PlanSel<(\d+), (\d)>\s*\{ using T = fft::Plan<([\d, ]+), true>; \}" if packed else
           r"PlanSel<(\d+), (\d)>\s*\{ using T = fft::Plan<([\d, ]+)>; \}")
    for m in re.finditer(pat, text):
        args = [int(v) for v in m.group(3).split(",")]
        N, E, radices = args[0], args[1], [r for r in args[2:] if r > 1]
        out.append((int(m.group(1)), int(m.group(2)), N, E, radices))
    return out


def xor_map(R1, P):
    return (R1 in (4, 8)) and P >= 16


def padi(n, R1, P):
    # restatement of padi() in ms_fft.cuh
    if xor_map(R1, P):
        r = n >> 4
        f = ((r ^ ((r & 4) << 1)) & 15) if R1 == 8 else (((r & 3) * 5) & 15)
        return n ^ f
    return n + n // R1


def slot(N, R1, P):
    return N + 8 if xor_map(R1, P) else ((N + N // R1 + 15) // 16) * 16 + 8


def worst_wavefronts(N, E, radices):
    P = N // E
    R1 = radices[0]
    SL = slot(N, R1, P)
    total = P if P >= 32 else 32
    worst = 1

    def lanes(point_of):
        nonlocal worst
        for h in range(0, min(total, 256), 16):
            banks = Counter()
            for lane in range(h, h + 16):
                g, t = divmod(lane, P) if P < 32 else (0, lane)
                banks[(2 * (g * SL + padi(point_of(t), R1, P))) % 32] += 1
            worst = max(worst, max(banks.values()))

    NS = 1
    for p, R in enumerate(radices):
        for b in range(E // R):
            if p == 0:
                for q in range(R):
                    lanes(lambda t: (t + P * b) * R1 + q)
            else:
                for r in range(R):
                    lanes(lambda t: (t + P * b) + r * (N // R))
                if p < len(radices) - 1:
                    for q in range(R):
                        lanes(lambda t: ((t + P * b) // NS) * NS * R + ((t + P * b) & (NS - 1)) + q * NS)
        NS *= R
    return worst


def test_plan_table_parsed():
    ps = plans()
    assert len(ps) == 21 and len(plans(packed=True)) == 21
    for n, v, N, E, radices in ps + plans(packed=True):
        assert n == N and v in (0, 1, 2, 3, 4, 5)
        prod = 1
        for r in radices:
            prod *= r
            assert E % r == 0
        assert prod == N


@pytest.mark.parametrize("plan", plans(), ids=lambda p: f"N{p[0]}v{p[1]}")
def test_exchanges_conflict_free(plan):
    n, v, N, E, radices = plan
    P = N // E
    w = worst_wavefronts(N, E, radices)
    if xor_map(radices[0], P) and not (N == 128 and E == 8):
        assert w == 1, w
    else:
        # padded plans (first radix 16 or 32, or lines of 8 threads) stay
        # conflict-free too, except the 128-point 8-per-thread plan (2-way)
        assert w <= 2
        if radices[0] >= 16:
            assert w == 1, w


def test_map_is_a_permutation():
    for n, v, N, E, radices in plans():
        P = N // E
        pos = {padi(k, radices[0], P) for k in range(N)}
        assert len(pos) == N and max(pos) < slot(N, radices[0], P)


# ---- column pass: interleaved columns on the padded map (ms_slice_impl.cuh)
def cols_per_cta(N, P, narrow=False):
    return (256 // P if P < 64 else 4) // (2 if narrow else 1)


def col_interleave(N, P, narrow=False):
    return min(cols_per_cta(N, P, narrow), 8)


def col_slot(N, R1, P, narrow=False):
    return ((N + N // R1 + 15) // 16) * 16 + 16 // col_interleave(N, P, narrow)


def col_worst_wavefronts(N, E, radices, narrow=False):
    P = N // E
    R1 = radices[0]
    CB, CW = cols_per_cta(N, P, narrow), col_interleave(N, P, narrow)
    GS, LS = CW * P, col_slot(N, R1, P, narrow)
    worst = 1

    def lanes(point_of):
        nonlocal worst
        for h in range(0, CB * P, 16):
            banks = Counter()
            for tid in range(h, h + 16):
                g, gr = divmod(tid, GS)
                c, t = g * CW + gr % CW, gr // CW
                banks[(c * LS + point_of(t) + point_of(t) // R1) % 16] += 1
            worst = max(worst, max(banks.values()))

    NS = 1
    for p, R in enumerate(radices):
        for b in range(E // R):
            if p == 0:
                for q in range(R):
                    lanes(lambda t: (t + P * b) * R1 + q)
            else:
                for r in range(R):
                    lanes(lambda t: (t + P * b) + r * (N // R))
                if p < len(radices) - 1:
                    for q in range(R):
                        lanes(lambda t: ((t + P * b) // NS) * NS * R + ((t + P * b) & (NS - 1)) + q * NS)
        NS *= R
    return worst


@pytest.mark.parametrize("plan", plans() + plans(packed=True), ids=lambda p: f"N{p[0]}v{p[1]}")
def test_column_exchanges_conflict_free(plan):
    # the packed 32-point plans run narrow (half the columns per CTA)
    n, v, N, E, radices = plan
    assert col_worst_wavefronts(N, E, radices, narrow=v >= 3 and E >= 32) == 1
