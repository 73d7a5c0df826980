// ms_fft.cuh -- register/shared-memory Stockham FFT of one line (row or column).
//
// A line of N = E * P complex points is owned by P threads (P <= 32: part of
// one warp; P = 64, 128, 256: whole warps of one CTA).  Thread t holds element
// t + P*j in register j ("strided natural layout"), which makes global loads
// and stores of a line fully coalesced.  The transform is a sequence of
// Stockham radix passes N = R1 * R2 * ... (each radix divides E):
//   pass 1: E/R1 radix-R1 butterflies on registers (no twiddles);
//   middle passes: inputs read from the line's shared slot, twiddles
//     W_{Ns R}^{r k} read from a per-pass [r][k] table (coalesced, L1-resident),
//     outputs written back in Stockham order;
//   last pass: outputs land in the strided natural layout, so the pointwise
//     operation that follows (transmission, propagator) needs no reordering.
// The slot is padded by one point every R1 points so the stride-R1 writes of
// pass 1 hit distinct banks.  In-register butterflies are radix-2 DIF networks
// with compile-time twiddles applied as exact quarter turns plus three-shear
// rotations (twc); trivial twiddles cost no multiply.  Table twiddles are the
// FP32 pairs nearest unit modulus (unit_fp32).
// Forward = exp(-2 pi i jk/N) (cuFFT CUFFT_FORWARD); the inverse is computed as
// conj(FFT(conj(x))) so that a kernel holds one copy of the transform code
// (instruction-cache footprint); both directions unnormalised.
#pragma once
#include "ms_common.cuh"

namespace ms {
namespace fft {

MS_HD constexpr int brev(int v, int bits) {
  int r = 0;
  for (int i = 0; i < bits; ++i) r |= ((v >> i) & 1) << (bits - 1 - i);
  return r;
}
MS_HD constexpr int ilog2(int v) { return v <= 1 ? 0 : 1 + ilog2(v >> 1); }

// tan(k pi / 32) and sin(k pi / 16), k = 1..4: the shear coefficients of a
// rotation by k/32 of a turn.
MS_HD constexpr float shear_t(int k) {
  return k == 1 ? 0.098491403357164248f : k == 2 ? 0.19891236737965801f : k == 3 ? 0.3033466836073424f
                                                                                  : 0.41421356237309503f;
}
MS_HD constexpr float shear_s(int k) {
  return k == 1 ? 0.19509032201612825f : k == 2 ? 0.38268343236508978f : k == 3 ? 0.55557023301960218f
                                                                                 : 0.70710678118654746f;
}

// x * W_M^J, W = exp(-2 pi i / M) forward, exp(+2 pi i / M) inverse; M divides 32.
// The rotation is an exact quarter turn (a swap and negation) followed, for
// the remaining angle r (|r| <= 1/8 turn), by three shears
//   x1 = x - tan(r/2) y,  y1 = y + sin(r) x1,  x2 = x1 - tan(r/2) y1
// (Paeth's decomposition).  Each shear has determinant exactly 1 whatever the
// FP32 rounding of its coefficient, so the rotation does not change the norm
// systematically: a rotation by rounded (cos, sin) scales by |(c, s)| != 1,
// an error that repeats in every transform of every slice and adds up
// coherently over a slice stack.  Three FMAs instead of a complex multiply.
template <int J, int M, bool INV>
MS_D float2 twc(float2 x) {
  constexpr int j = ((J % M) + M) % M * (32 / M);
  if constexpr (j == 0) {
    return x;
  } else {
    // angle in 32nds of a turn, counter-clockwise: -j forward, +j inverse
    constexpr int a = INV ? j : (32 - j) % 32;
    constexpr int q = ((a + 4) / 8) % 4;   // nearest quarter turn
    constexpr int rem = a - 8 * ((a + 4) / 8);  // -4 .. 3
    float2 y = x;
    if constexpr (q == 1) y = make_float2(-x.y, x.x);
    else if constexpr (q == 2) y = make_float2(-x.x, -x.y);
    else if constexpr (q == 3) y = make_float2(x.y, -x.x);
    if constexpr (rem == 0) {
      return y;
    } else {
      constexpr int k = rem > 0 ? rem : -rem;
      constexpr float t = rem > 0 ? shear_t(k) : -shear_t(k);
      constexpr float sn = rem > 0 ? shear_s(k) : -shear_s(k);
      const float x1 = fmaf(-t, y.y, y.x);
      const float y1 = fmaf(sn, x1, y.y);
      const float x2 = fmaf(-t, y1, x1);
      return make_float2(x2, y1);
    }
  }
}

// Complex sum and difference of a butterfly on the packed FP32x2 pipe
// (add/sub.rn.f32x2: both components in one instruction, correctly rounded).
MS_D void addsub_packed(float2 a, float2 b, float2& s, float2& d) {
  unsigned long long pa, pb, ps, pd;
  asm("mov.b64 %0, {%1, %2};" : "=l"(pa) : "f"(a.x), "f"(a.y));
  asm("mov.b64 %0, {%1, %2};" : "=l"(pb) : "f"(b.x), "f"(b.y));
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(ps) : "l"(pa), "l"(pb));
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(pd) : "l"(pa), "l"(pb));
  asm("mov.b64 {%0, %1}, %2;" : "=f"(s.x), "=f"(s.y) : "l"(ps));
  asm("mov.b64 {%0, %1}, %2;" : "=f"(d.x), "=f"(d.y) : "l"(pd));
}

// Radix-2 DIF network on R registers: natural-order input, bit-reversed output.
// PK: butterfly sums and differences on the packed FP32x2 pipe.
template <int R, int SPAN, bool INV, bool PK>
struct Dif {
  template <int START, int J>
  static MS_D void bfly(float2 (&x)[R]) {
    const float2 a = x[START + J], b = x[START + J + SPAN];
    if constexpr (PK) {
      float2 s, d;
      addsub_packed(a, b, s, d);
      x[START + J] = s;
      x[START + J + SPAN] = twc<J, 2 * SPAN, INV>(d);
    } else {
      x[START + J] = cadd(a, b);
      x[START + J + SPAN] = twc<J, 2 * SPAN, INV>(csub(a, b));
    }
    if constexpr (J + 1 < SPAN)
      bfly<START, J + 1>(x);
    else if constexpr (START + 2 * SPAN < R)
      bfly<START + 2 * SPAN, 0>(x);
  }
  static MS_D void run(float2 (&x)[R]) {
    bfly<0, 0>(x);
    if constexpr (SPAN > 1) Dif<R, SPAN / 2, INV, PK>::run(x);
  }
};

template <int R, bool INV, bool PK = false>
MS_D void dft(float2 (&x)[R]) {
  if constexpr (R > 1) Dif<R, R / 2, INV, PK>::run(x);
}

// A factorisation N = R1 * R2 * R3 * R4 (trailing radices 1 = absent) with E
// points per thread; every radix divides E and is at most 32.
template <int N_, int E_, int R1_, int R2_, int R3_ = 1, int R4_ = 1, bool PK_ = false, bool PAD_ = false>
struct Plan {
  static constexpr int N = N_, E = E_, P = N_ / E_;
  static constexpr bool PK = PK_;  // butterflies on the packed FP32x2 pipe
  static constexpr int R1 = R1_, R2 = R2_, R3 = R3_, R4 = R4_;
  static constexpr int NPASS = 1 + (R2_ > 1) + (R3_ > 1) + (R4_ > 1);
  static_assert(R1_ * R2_ * R3_ * R4_ == N_, "radices must multiply to N");
  static_assert(E_ % R1_ == 0 && E_ % R2_ == 0 && E_ % R3_ == 0 && E_ % R4_ == 0, "radix must divide E");
  static_assert(R1_ <= 32 && R2_ <= 32 && R3_ <= 32 && R4_ <= 32, "radix above 32");
  static_assert(P <= 32 || P % 32 == 0, "multi-warp lines need whole warps");
  // Shared-memory map of a line's points (see padi): an XOR swizzle for first
  // radices 4 and 8 on lines of at least 16 threads, else (or with PAD_) one
  // pad point every R1.
  static constexpr bool XOR_MAP = !PAD_ && (R1_ == 4 || R1_ == 8) && P >= 16;
  // Points in one line slot (slots 8 apart mod 16).
  static constexpr int SLOT = XOR_MAP ? N_ + 8 : ((N_ + N_ / R1_ + 15) / 16) * 16 + 8;
  // Twiddle table: pass p >= 2 holds R_p * Ns_p entries [r][k].
  // (absent passes, radix 1, take no entries; the sum never exceeds 2N)
  static constexpr int TW2 = 0, TW3 = TW2 + R2_ * R1_, TW4 = TW3 + (R3_ > 1 ? R3_ * R1_ * R2_ : 0);
  static constexpr int TWSIZE = TW4 + (R4_ > 1 ? R4_ * R1_ * R2_ * R3_ : 0);
  static_assert(TWSIZE <= 2 * N_, "twiddle table larger than 2N");
};

// The same plan on the padded map (the column pass's interleaved threads read
// runs of 16/CW consecutive points per column, which the padded map keeps in
// consecutive banks).
template <class PL>
using PaddedPlan = Plan<PL::N, PL::E, PL::R1, PL::R2, PL::R3, PL::R4, PL::PK, true>;

// Slot position of point n.  A 64-bit access of 16 lanes is one wavefront when
// its points fall in 16 distinct (point mod 16) classes.  Lines read 16
// consecutive, 16-aligned points per half-warp in every pass; the writes of the
// first pass are R1 apart and those of a middle pass with NS < 16 come in
// groups of NS.  Padding one point every R1 serves the strided writes but
// wraps the consecutive reads when R1 < 16; the XOR map n ^ f(n >> 4) permutes
// each aligned block of 16 (reads stay conflict-free) with f chosen so that the
// R1-strided and NS-grouped writes of the plan also land in distinct classes
// (checked exhaustively on the host for every plan).
template <class PL>
MS_D int padi(int n) {
  if constexpr (PL::XOR_MAP) {
    const int r = n >> 4;
    const int f = PL::R1 == 8 ? ((r ^ ((r & 4) << 1)) & 15) : (((r & 3) * 5) & 15);
    return n ^ f;
  } else {
    return n + n / PL::R1;
  }
}

// Barrier of the P threads that own one line: the warp's lanes for P <= 32,
// else named barrier 1 + (line index in the CTA) over P threads, so that the
// lines of a CTA do not wait for one another (lines are contiguous groups of
// P threads; at most 4 lines of P > 32 per CTA).
//
// GS > 0 instead names a group of GS consecutive threads that share their
// lines' exchanges (lines interleaved across the group's warps): the warp for
// GS <= 32, else named barrier 1 + threadIdx.x / GS over GS threads.
template <class PL, int GS = 0>
MS_D void line_sync() {
  constexpr int G = GS > 0 ? GS : PL::P;
  if constexpr (G <= 32)
    __syncwarp();
  else
    asm volatile("bar.sync %0, %1;" ::"r"(1 + (int)threadIdx.x / G), "n"(G) : "memory");
}

// Radix R of pass number IDX (0-based).
template <class PL, int IDX>
struct PassR {
  static constexpr int R = IDX == 0 ? PL::R1 : IDX == 1 ? PL::R2 : IDX == 2 ? PL::R3 : PL::R4;
  static constexpr int NS = IDX == 0 ? 1 : IDX == 1 ? PL::R1 : IDX == 2 ? PL::R1 * PL::R2 : PL::R1 * PL::R2 * PL::R3;
  static constexpr int TW = IDX == 1 ? PL::TW2 : IDX == 2 ? PL::TW3 : PL::TW4;
};

// Twiddles of pass IDX for this thread's butterflies, loaded ahead of the
// barrier that precedes the pass so their latency overlaps the wait.  Plans
// with more than 16 twiddles per thread load them at use instead.
template <class PL, int IDX>
struct TwiddleRegs {
  static constexpr int R = PassR<PL, IDX>::R, NB = PL::E / R;
  static constexpr bool PREFETCH = NB * (R - 1) <= 16;
  float2 w[PREFETCH ? NB * (R - 1) : 1];
  MS_D void load(const float2* __restrict__ tw, int t) {
    if constexpr (PREFETCH) {
      constexpr int NS = PassR<PL, IDX>::NS, TWO = PassR<PL, IDX>::TW;
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const int k = (t + PL::P * b) & (NS - 1);
#pragma unroll
        for (int r = 1; r < R; ++r) w[b * (R - 1) + r - 1] = __ldg(tw + TWO + r * NS + k);
      }
    }
  }
  MS_D float2 get(const float2* __restrict__ tw, int b, int r, int k) const {
    if constexpr (PREFETCH) {
      return w[b * (R - 1) + r - 1];
    } else {
      return __ldg(tw + PassR<PL, IDX>::TW + r * PassR<PL, IDX>::NS + k);
    }
  }
};

// Stockham pass IDX >= 1: the previous pass has written the slot but not yet
// synchronised.  Forward transform only; the inverse is conj(FFT(conj(x))).
template <class PL, int IDX, int GS = 0>
MS_D void forward_pass(float2 (&v)[PL::E], float2* __restrict__ sm, int t, const float2* __restrict__ tw) {
  constexpr int N = PL::N, E = PL::E, P = PL::P;
  constexpr int R = PassR<PL, IDX>::R, NS = PassR<PL, IDX>::NS, LR = ilog2(R);
  constexpr bool LAST = (IDX == PL::NPASS - 1);
  TwiddleRegs<PL, IDX> tr;
  tr.load(tw, t);
  line_sync<PL, GS>();
  if constexpr (LAST) {
#pragma unroll
    for (int b = 0; b < E / R; ++b) {
      const int i = t + P * b;  // i < N/R = NS, so k = i
      float2 x[R];
#pragma unroll
      for (int r = 0; r < R; ++r) x[r] = sm[padi<PL>(i + r * (N / R))];
#pragma unroll
      for (int r = 1; r < R; ++r) x[r] = cmul(x[r], tr.get(tw, b, r, i));
      dft<R, false, PL::PK>(x);
#pragma unroll
      for (int q = 0; q < R; ++q) v[b + q * (E / R)] = x[brev(q, LR)];
    }
    line_sync<PL, GS>();
  } else {
    // read every input of this thread's butterflies, then overwrite the slot
#pragma unroll
    for (int b = 0; b < E / R; ++b) {
      const int i = t + P * b;
#pragma unroll
      for (int r = 0; r < R; ++r) v[b * R + r] = sm[padi<PL>(i + r * (N / R))];
    }
    line_sync<PL, GS>();
#pragma unroll
    for (int b = 0; b < E / R; ++b) {
      const int i = t + P * b;
      const int k = i & (NS - 1);
      float2 x[R];
#pragma unroll
      for (int r = 0; r < R; ++r) x[r] = v[b * R + r];
#pragma unroll
      for (int r = 1; r < R; ++r) x[r] = cmul(x[r], tr.get(tw, b, r, k));
      dft<R, false, PL::PK>(x);
      const int base = (i / NS) * NS * R + k;
#pragma unroll
      for (int q = 0; q < R; ++q) sm[padi<PL>(base + q * NS)] = x[brev(q, LR)];
    }
    forward_pass<PL, IDX + 1, GS>(v, sm, t, tw);
  }
}

// Forward N-point transform of the line held by threads t = 0..P-1 of a
// group.  `sm` is this line's shared slot (PL::SLOT points), `tw` the plan's
// twiddle table.  Every thread of the line's barrier group (line_sync<PL, GS>)
// must call this: it synchronises.  On return the slot may be reused.
template <class PL, int GS = 0>
MS_D void line_fft(float2 (&v)[PL::E], float2* __restrict__ sm, int t, const float2* __restrict__ tw) {
  constexpr int E = PL::E, P = PL::P, R1 = PL::R1, L1 = ilog2(R1);
#pragma unroll
  for (int b = 0; b < E / R1; ++b) {
    float2 x[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) x[r] = v[b + r * (E / R1)];
    dft<R1, false, PL::PK>(x);
    const int i = t + P * b;
#pragma unroll
    for (int q = 0; q < R1; ++q) sm[padi<PL>(i * R1 + q)] = x[brev(q, L1)];
  }
  forward_pass<PL, 1, GS>(v, sm, t, tw);
}

template <int E>
MS_D void conj_all(float2 (&v)[E]) {
#pragma unroll
  for (int j = 0; j < E; ++j) v[j].y = -v[j].y;
}

// Host-side twiddle table of a plan: pass p >= 2 entries W_{Ns R}^{r k},
// r < R_p, k < Ns_p, laid out [r][k] after the previous pass's table.
void make_plan_twiddles(int n, const int* radices, int npass, float2* out);

}  // namespace fft
}  // namespace ms
