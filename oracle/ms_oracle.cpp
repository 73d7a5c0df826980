/*
 * ms_oracle.cpp -- FP64 CPU oracle for the multislice hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine, never part of it.
 * Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.
 *
 * Restates, function by function, the reference engine
 *   GUI Simulation/UnmanagedGUISimulation.cu  (abbreviated U.cu below)
 *   GUI Simulation/unmanagedGUISimulation.cuh (class UnmanagedMultisliceSimulation)
 * with every value in FP64 and every FP32 decision of the reference mirrored
 * bit for bit (see ms_oracle.h).  Build with -ffp-contract=off (oracle/Makefile):
 * the mirrored FP32 expressions must not be fused into FMAs.
 *
 * Parity pinning: tests/test_oracle.py checks the Bessel approximations against
 * scipy, the FFT against numpy, the potential integral identity, Philox
 * known-answer vectors, and the whole path against golden vectors produced by
 * the reference itself (tests/golden/, generator committed beside them).
 */
#include "ms_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <map>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cd;

/* ======================================================================
 * Bessel functions: the polynomial approximations of U.cu:41-111
 * (Abramowitz & Stegun 9.8.1-9.8.2 for I0 and 9.8.5-9.8.6 for K0),
 * evaluated in FP64.  K0(0) returns 1e20 as at U.cu:108.
 * ==================================================================== */
extern "C" double or_bessi0(double x) {
    static const double a[7] = {1.0, 3.5156229, 3.0899424, 1.2067492,
                                0.2659732, 0.0360768, 0.0045813};
    static const double b[9] = {0.39894228, 0.01328592, 0.00225319, -0.00157565,
                                0.00916281, -0.02057706, 0.02635537, -0.01647633,
                                0.00392377};
    double ax = std::fabs(x), s, t;
    if (ax <= 3.75) {
        t = x / 3.75;
        t = t * t;
        s = a[6];
        for (int i = 5; i >= 0; --i) s = s * t + a[i];
    } else {
        t = 3.75 / ax;
        s = b[8];
        for (int i = 7; i >= 0; --i) s = s * t + b[i];
        s = std::exp(ax) * s / std::sqrt(ax);
    }
    return s;
}

extern "C" double or_bessk0(double x) {
    static const double a[7] = {-0.57721566, 0.42278420, 0.23069756, 0.03488590,
                                0.00262698, 0.00010750, 0.00000740};
    static const double b[7] = {1.25331414, -0.07832358, 0.02189568, -0.01062446,
                                0.00587872, -0.00251540, 0.00053208};
    double ax = std::fabs(x), s, x2;
    if (ax > 0.0 && ax <= 2.0) {
        x2 = ax / 2.0;
        x2 = x2 * x2;
        s = a[6];
        for (int i = 5; i >= 0; --i) s = s * x2 + a[i];
        s = -std::log(ax / 2.0) * or_bessi0(x) + s;
    } else if (ax > 2.0) {
        x2 = 2.0 / ax;
        s = b[6];
        for (int i = 5; i >= 0; --i) s = s * x2 + b[i];
        s = std::exp(-ax) * s / std::sqrt(ax);
    } else {
        s = 1.0e20;
    }
    return s;
}

/* Projected potential vz(r), U.cu:119-152.  Input is r^2; r clamped to >= 0.25 A.
 * Row Z-1 of fparams = [a1 b1 a2 b2 a3 b3 | c1 d1 c2 d2 c3 d3]. */
extern "C" double or_vzatom2(const double* fp, int Z, double r2) {
    const double* f = fp + (Z - 1) * 12;
    double r = std::sqrt(std::fabs(r2));
    if (r < 0.25) r = 0.25;
    double suml = 0.0, sumg = 0.0;
    double x = 2.0 * 3.141592654 * r;
    for (int i = 0; i < 6; i += 2) suml += f[i] * or_bessk0(x * std::sqrt(f[i + 1]));
    x = 3.141592654 * r;
    x = x * x;
    for (int i = 6; i < 12; i += 2) sumg += f[i] * std::exp(-x / f[i + 1]) / f[i + 1];
    return 300.8242834 * suml + 150.4121417 * sumg;
}

/* 3D atomic potential v(r), U.cu:160-193.  Input is r^2; r clamped to >= 0.25 A. */
extern "C" double or_vatom(const double* fp, int Z, double r2) {
    const double* f = fp + (Z - 1) * 12;
    double r = std::sqrt(std::fabs(r2));
    if (r < 0.25) r = 0.25;
    double suml = 0.0, sumg = 0.0;
    double x = 2.0 * 3.141592654 * r;
    for (int i = 0; i < 6; i += 2) suml += (1.0 / r) * f[i] * std::exp(-x * std::sqrt(f[i + 1]));
    x = 3.141592654 * r;
    x = x * x;
    for (int i = 6; i < 12; i += 2)
        sumg += f[i] * std::exp(-x / f[i + 1]) * std::pow(f[i + 1], -1.5);
    return 150.4121417 * suml + 266.5157269 * sumg;
}

/* fparams.dat reader, U.cu:1718-1747: whitespace-separated rows of 12 numbers. */
extern "C" int or_parse_fparams(const char* path, double* out, int* nrows) {
    std::ifstream in(path);
    if (!in) return -1;
    int rows = 0;
    double v[12];
    while (rows < 103) {
        int k = 0;
        for (; k < 12; ++k)
            if (!(in >> v[k])) break;
        if (k < 12) break;
        for (int j = 0; j < 12; ++j) out[rows * 12 + j] = v[j];
        ++rows;
    }
    if (nrows) *nrows = rows;
    return rows > 0 ? 0 : -2;
}

/* ======================================================================
 * FP64 FFT: Stockham autosort, any size (each prime factor as a direct DFT
 * butterfly).  sign = -1 is cuFFT's CUFFT_FORWARD, +1 CUFFT_INVERSE; both
 * unnormalised, as cuFFT.
 * ==================================================================== */
namespace {
struct FFTPlan {
    int n;
    int sign;
    std::vector<int> radices;
    std::vector<cd> w; /* w[m] = exp(sign*2*pi*i*m/n) */
    FFTPlan(int n_, int sign_) : n(n_), sign(sign_) {
        int m = n;
        while (m % 4 == 0) { radices.push_back(4); m /= 4; }
        while (m % 2 == 0) { radices.push_back(2); m /= 2; }
        for (int p = 3; m > 1; p += 2) {
            while (m % p == 0) { radices.push_back(p); m /= p; }
            if (p * p > m && m > 1) { radices.push_back(m); m = 1; }
        }
        w.resize(n);
        const long double twopi = 6.283185307179586476925286766559L;
        for (int k = 0; k < n; ++k) {
            long double ang = twopi * (long double)k / (long double)n;
            w[k] = cd((double)std::cos(ang), (double)(sign * std::sin(ang)));
        }
    }
    void exec(cd* data, cd* work) const {
        cd* src = data;
        cd* dst = work;
        int Ns = 1;
        std::vector<cd> x, y;
        for (int R : radices) {
            x.resize(R);
            y.resize(R);
            const int nR = n / R;
            for (int j = 0; j < nR; ++j) {
                const int k = j % Ns;
                const int tstep = n / (Ns * R); /* twiddle exponent unit */
                for (int r = 0; r < R; ++r) {
                    cd v = src[j + r * nR];
                    if (r && k) v *= w[(long long)r * k * tstep % n];
                    x[r] = v;
                }
                for (int q = 0; q < R; ++q) {
                    cd acc = 0;
                    for (int r = 0; r < R; ++r) acc += x[r] * w[(long long)r * q * nR % n];
                    y[q] = acc;
                }
                const int base = (j / Ns) * Ns * R + k;
                for (int q = 0; q < R; ++q) dst[base + q * Ns] = y[q];
            }
            Ns *= R;
            std::swap(src, dst);
        }
        if (src != data) std::copy(src, src + n, data);
    }
};
}  // namespace

extern "C" int or_fft1d(double* data, int n, int sign) {
    if (n <= 0) return -1;
    FFTPlan p(n, sign < 0 ? -1 : 1);
    std::vector<cd> work(n);
    p.exec(reinterpret_cast<cd*>(data), work.data());
    return 0;
}

static void fft2d(cd* a, int nx, int ny, int sign) {
    FFTPlan px(nx, sign), py(ny, sign);
#pragma omp parallel
    {
        std::vector<cd> work(std::max(nx, ny)), col(ny);
#pragma omp for schedule(static)
        for (int y = 0; y < ny; ++y) px.exec(a + (size_t)y * nx, work.data());
#pragma omp for schedule(static)
        for (int x = 0; x < nx; ++x) {
            for (int y = 0; y < ny; ++y) col[y] = a[(size_t)y * nx + x];
            py.exec(col.data(), work.data());
            for (int y = 0; y < ny; ++y) a[(size_t)y * nx + x] = col[y];
        }
    }
}

extern "C" int or_fft2d(double* data, int nx, int ny, int sign) {
    if (nx <= 0 || ny <= 0) return -1;
    fft2d(reinterpret_cast<cd*>(data), nx, ny, sign < 0 ? -1 : 1);
    return 0;
}

/* ======================================================================
 * Philox4x32-10 (J. Salmon, M. Moraes, R. Dror, D. Shaw, "Parallel random
 * numbers: as easy as 1, 2, 3", SC'11) and the thermal displacement built on
 * it.  Replaces the unseeded rand()/Box-Muller of TDSRand (U.cu:29-37).
 * ==================================================================== */
extern "C" void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Displacement of atom a in thermal pass `pass`: counter (a, pass, 0x5EED, 0),
 * key (seed low, seed high); Box-Muller on (u1, u2) and (u3, u4) with
 * u = (r + 0.5) / 2^32; x,y use the first pair, z the cosine of the second. */
extern "C" void or_tds_displace(const float* x, const float* y, const float* z, int n,
                                uint64_t seed, uint32_t pass, float sigma,
                                float* xo, float* yo, float* zo) {
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    const double twopi = 6.283185307179586;
    for (int a = 0; a < n; ++a) {
        uint32_t ctr[4] = {(uint32_t)a, pass, 0x5EEDu, 0u}, r[4];
        or_philox4x32_10(ctr, key, r);
        double u[4];
        for (int j = 0; j < 4; ++j) u[j] = ((double)r[j] + 0.5) * 2.3283064365386963e-10;
        double m0 = std::sqrt(-2.0 * std::log(u[0])), m1 = std::sqrt(-2.0 * std::log(u[2]));
        double n0 = m0 * std::cos(twopi * u[1]);
        double n1 = m0 * std::sin(twopi * u[1]);
        double n2 = m1 * std::cos(twopi * u[3]);
        xo[a] = (float)((double)x[a] + (double)sigma * n0);
        yo[a] = (float)((double)y[a] + (double)sigma * n1);
        zo[a] = (float)((double)z[a] + (double)sigma * n2);
    }
}

/* ======================================================================
 * Element symbols.  Reference table (U.cu:1188-1243): 26 symbols, anything
 * else -> Z = 1.  Full table: Z = 1..103 (the rows of fparams.dat).
 * ==================================================================== */
static const char* kElements[103] = {
    "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S",
    "Cl", "Ar", "K", "Ca", "Sc", "Ti", "V", "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga",
    "Ge", "As", "Se", "Br", "Kr", "Rb", "Sr", "Y", "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd",
    "Ag", "Cd", "In", "Sn", "Sb", "Te", "I", "Xe", "Cs", "Ba", "La", "Ce", "Pr", "Nd", "Pm",
    "Sm", "Eu", "Gd", "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf", "Ta", "W", "Re", "Os",
    "Ir", "Pt", "Au", "Hg", "Tl", "Pb", "Bi", "Po", "At", "Rn", "Fr", "Ra", "Ac", "Th", "Pa",
    "U", "Np", "Pu", "Am", "Cm", "Bk", "Cf", "Es", "Fm", "Md", "No", "Lr"};

extern "C" int or_znum(const char* s, int full_table) {
    static const int ref_z[] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 11, 12, 14, 15, 16, 17, 20, 24,
                                35, 26, 38, 44, 57, 62, 73, 74};
    if (full_table) {
        for (int z = 1; z <= 103; ++z)
            if (std::strcmp(s, kElements[z - 1]) == 0) return z;
        return 1;
    }
    for (int z : ref_z)
        if (std::strcmp(s, kElements[z - 1]) == 0) return z;
    return 1;
}

/* ======================================================================
 * The simulation object.
 * ==================================================================== */
struct or_sim {
    std::string err;
    /* structure (LoadAtomFile) */
    std::vector<int> Z;
    std::vector<float> x, y, z;
    float MaxX = 0, MinX = 0, MaxY = 0, MinY = 0, MaxZ = 0, MinZ = 0;
    bool have_atoms = false;
    /* binned structure */
    int nzb = 0;
    std::vector<int> off, bZ, perm; /* perm: sorted position -> input index */
    std::vector<float> bx, by, bz;
    std::vector<double> valdx, valdy; /* value-only offsets by input index (tests) */
    bool have_bins = false;
    /* Kirkland table */
    std::vector<double> fp;
    bool have_fp = false;
    /* microscope */
    float kV = 0, df = 0, A2 = 0, phi2 = 0, Cs = 0, beta = 0, delta = 0, aperture = 0;
    float A3 = 0, phi3 = 0; /* Mod3fold/Arg3fold are fixed to 0 in the constructor, U.cu:2554 */
    /* calculation variables */
    int nx = 0, ny = 0;
    float ps = 0, xoff = 0, yoff = 0;
    float wavel = 0, sigma2 = 0, ke2 = 0, dzFD = 0, kmax = 0, convdz = 1;
    int nFD = 0, lbx = 0, lby = 0, lbz = 0;
    bool stem = false, have_calc = false, have_freq = false;
    std::vector<float> kx, ky;
    /* waves */
    std::vector<cd> psi0, psi_minus, psi, psi_plus;
    bool have_waves = false;
    std::vector<double> tds;
    /* optional cache of conventional potentials by iteration (tests that run
     * many probes over one specimen); cleared whenever an input of V changes */
    bool vcache_on = false;
    std::map<int, std::vector<double>> vcache;
};

/* Drops cached potentials: called by every set-up step that changes an input
 * of the potential (atoms, table, grid, offsets, slice thickness). */
static void pot_inputs_changed(or_sim* s) { s->vcache.clear(); }

extern "C" or_sim* or_create(void) { return new or_sim(); }
extern "C" void or_destroy(or_sim* s) { delete s; }
extern "C" const char* or_last_error(or_sim* s) { return s ? s->err.c_str() : "null"; }
extern "C" int or_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

static int fail(or_sim* s, const char* msg) {
    s->err = msg;
    return -1;
}

/* Bounding box: U.cu:1326-1355 (index of extreme atom, then +-2 A in FP32). */
static void compute_box(or_sim* s) {
    size_t mx = 0, mnx = 0, my = 0, mny = 0, mz = 0, mnz = 0;
    for (size_t i = 1; i < s->x.size(); ++i) {
        if (s->x[i] > s->x[mx]) mx = i;
        if (s->y[i] > s->y[my]) my = i;
        if (s->z[i] > s->z[mz]) mz = i;
        if (s->x[i] < s->x[mnx]) mnx = i;
        if (s->y[i] < s->y[mny]) mny = i;
        if (s->z[i] < s->z[mnz]) mnz = i;
    }
    s->MaxX = s->x[mx] + 2;
    s->MinX = s->x[mnx] - 2;
    s->MaxY = s->y[my] + 2;
    s->MinY = s->y[mny] - 2;
    s->MaxZ = s->z[mz] + 2;
    s->MinZ = s->z[mnz] - 2;
}

extern "C" int or_set_atoms(or_sim* s, const int* Z, const float* x, const float* y,
                            const float* z, int n) {
    if (n <= 0) return fail(s, "no atoms");
    for (int i = 0; i < n; ++i)
        if (Z[i] < 1 || Z[i] > 103) return fail(s, "atomic number out of range 1..103");
    s->Z.assign(Z, Z + n);
    s->x.assign(x, x + n);
    s->y.assign(y, y + n);
    s->z.assign(z, z + n);
    compute_box(s);
    s->have_atoms = true;
    s->have_bins = false;
    return 0;
}

/* .xyz reader, U.cu:1293-1356: the count, the rest of its line discarded
 * (U.cu:1309-1310), then "symbol x y z" records.  A separate comment line
 * (which the reference would misread as an atom) is skipped. */
extern "C" int or_import_atoms(or_sim* s, const char* path, int full_table) {
    std::ifstream in(path);
    if (!in) return fail(s, "cannot open structure file");
    int n = 0;
    std::string line;
    if (!(in >> n) || n <= 0) return fail(s, "bad atom count");
    std::getline(in, line);
    std::vector<int> Z;
    std::vector<float> x, y, z;
    bool first = true;
    while ((int)Z.size() < n && std::getline(in, line)) {
        std::istringstream ls(line);
        std::string sym;
        float a, b, c;
        const bool blank = line.find_first_not_of(" \t\r") == std::string::npos;
        if (!(ls >> sym >> a >> b >> c)) {
            if (blank) continue;
            if (first) { first = false; continue; }
            return fail(s, "malformed atom record");
        }
        first = false;
        Z.push_back(or_znum(sym.c_str(), full_table));
        x.push_back(a); y.push_back(b); z.push_back(c);
    }
    if ((int)Z.size() < n) return fail(s, "truncated structure file");
    return or_set_atoms(s, Z.data(), x.data(), y.data(), z.data(), n);
}

extern "C" int or_get_box(or_sim* s, float out[6]) {
    if (!s->have_atoms) return fail(s, "no atoms");
    out[0] = s->MaxX; out[1] = s->MinX; out[2] = s->MaxY;
    out[3] = s->MinY; out[4] = s->MaxZ; out[5] = s->MinZ;
    return 0;
}

extern "C" int or_load_fparams(or_sim* s, const char* path) {
    pot_inputs_changed(s);
    s->fp.assign(103 * 12, 0.0);
    int rows = 0;
    if (or_parse_fparams(path, s->fp.data(), &rows) != 0) return fail(s, "cannot read fparams");
    s->have_fp = true;
    return 0;
}

/* ---------------- binning: atombin2 (U.cu:277-303) + host CSR (U.cu:1444-1525) ---------- */
static const int kBins = 50;

static int zbin_count(const or_sim* s) {
    /* nSlices = ceil((MaximumZ-MinimumZ)/dz) with int dz = 1, U.cu:1409-1411 */
    int nz = (int)std::ceil((s->MaxZ - s->MinZ) / (float)1);
    nz += (nz == 0);
    return nz;
}

static void bin_positions(or_sim* s, const float* X, const float* Y, const float* Zp) {
    const size_t n = s->x.size();
    const int nz = zbin_count(s);
    std::vector<int> key(n);
    for (size_t i = 0; i < n; ++i) {
        /* bidx = floor((x-minx)/(maxx-minx)*xBlocks): FP32 sub, div, mul, floor */
        float qx = (X[i] - s->MinX) / (s->MaxX - s->MinX);
        float qy = (Y[i] - s->MinY) / (s->MaxY - s->MinY);
        int bx = (int)std::floor(qx * (float)kBins);
        int by = (int)std::floor(qy * (float)kBins);
        int bz = (int)std::floor((s->MaxZ - Zp[i]) / (float)1);
        /* The reference relies on the +-2 A padding to stay in range
         * (comment at U.cu:293-296); displaced thermal positions are clamped. */
        bx = std::min(std::max(bx, 0), kBins - 1);
        by = std::min(std::max(by, 0), kBins - 1);
        bz = std::min(std::max(bz, 0), nz - 1);
        key[i] = bz * kBins * kBins + by * kBins + bx;
    }
    /* Stable counting sort: slice -> y-bin -> x-bin, input order within a bin. */
    const int nb = nz * kBins * kBins;
    s->off.assign(nb + 1, 0);
    for (size_t i = 0; i < n; ++i) s->off[key[i] + 1]++;
    for (int b = 0; b < nb; ++b) s->off[b + 1] += s->off[b];
    std::vector<int> cur(s->off.begin(), s->off.end() - 1);
    s->bx.resize(n); s->by.resize(n); s->bz.resize(n); s->bZ.resize(n);
    s->perm.resize(n);
    for (size_t i = 0; i < n; ++i) {
        int d = cur[key[i]]++;
        s->perm[d] = (int)i;
        s->bx[d] = X[i] - s->MinX; /* stored shifted by the box minimum, U.cu:1479-1482 */
        s->by[d] = Y[i] - s->MinY;
        s->bz[d] = Zp[i] - s->MinZ;
        s->bZ[d] = s->Z[i];
    }
    s->nzb = nz;
    s->have_bins = true;
}

extern "C" int or_bin_atoms(or_sim* s) {
    if (!s->have_atoms) return fail(s, "no atoms");
    pot_inputs_changed(s);
    bin_positions(s, s->x.data(), s->y.data(), s->z.data());
    return 0;
}

extern "C" int or_bin_atoms_tds(or_sim* s, uint64_t seed, uint32_t pass, float sigma) {
    if (!s->have_atoms) return fail(s, "no atoms");
    pot_inputs_changed(s);
    const int n = (int)s->x.size();
    std::vector<float> X(n), Y(n), Zp(n);
    or_tds_displace(s->x.data(), s->y.data(), s->z.data(), n, seed, pass, sigma,
                    X.data(), Y.data(), Zp.data());
    bin_positions(s, X.data(), Y.data(), Zp.data());
    return 0;
}

extern "C" int or_get_binned_counts(or_sim* s, int* n_atoms, int* n_zbins) {
    if (!s->have_bins) return fail(s, "atoms not binned");
    *n_atoms = (int)s->bx.size();
    *n_zbins = s->nzb;
    return 0;
}

extern "C" int or_get_binned(or_sim* s, int* offsets, int* Z, float* x, float* y, float* z) {
    if (!s->have_bins) return fail(s, "atoms not binned");
    std::copy(s->off.begin(), s->off.end(), offsets);
    std::copy(s->bZ.begin(), s->bZ.end(), Z);
    std::copy(s->bx.begin(), s->bx.end(), x);
    std::copy(s->by.begin(), s->by.end(), y);
    std::copy(s->bz.begin(), s->bz.end(), z);
    return 0;
}

/* ---------------- microscope and set-up (FP32 exactly as the reference host code) ------- */
extern "C" int or_apply_microscope(or_sim* s, float kV, float df, float A2, float phi2,
                                   float Cs, float beta, float delta, float aperture) {
    s->kV = kV; s->df = df; s->A2 = A2; s->phi2 = phi2;
    s->Cs = Cs; s->beta = beta; s->delta = delta; s->aperture = aperture;
    return 0;
}

/* SetCalculationVariables U.cu:1763-1875 (stem = 0) and STEMSetCalculationVariables
 * U.cu:2567-2670 (stem = 1: no block offsets, FD step clamped to 0.06 A). */
extern "C" int or_set_calc(or_sim* s, float ps, float df, int nx, int ny, float sx, float sy,
                           float sizeZ, float xoff, float yoff, int stem) {
    (void)sx; (void)sy;
    pot_inputs_changed(s);
    if (nx <= 0 || ny <= 0 || !(ps > 0)) return fail(s, "bad grid");
    if (!(s->kV > 0)) return fail(s, "accelerating voltage not set");
    if (!s->have_atoms) return fail(s, "no atoms");
    s->nx = nx; s->ny = ny; s->df = df; s->ps = ps;
    s->stem = stem != 0;
    s->xoff = stem ? 0.0f : xoff;
    s->yoff = stem ? 0.0f : yoff;
    const float ksizex = ps * nx, ksizey = ps * ny;
    const float Pi = 3.1415926f;
    const float V = s->kV;
    const float echarge = 1.6e-019f;
    const float wavel = 6.63e-034f * 3e+008f /
                        std::sqrt((echarge * V * 1000 * (2 * 9.11e-031f * 9e+016f + echarge * V * 1000))) *
                        1e+010f;
    const float sigma2 = (2 * Pi / (wavel * V * 1000)) *
                         ((9.11e-031f * 9e+016f + echarge * V * 1000) /
                          (2 * 9.11e-031f * 9e+016f + echarge * V * 1000));
    const float V2 = V * 1000;
    const float fnkx = (float)nx, fnky = (float)ny;
    const float p1 = fnkx / (2 * ksizex), p2 = fnky / (2 * ksizey);
    const float p12 = p1 * p1, p22 = p2 * p2;
    const float ke2 = (.666666f) * (p12 + p22);
    const float qA = (ke2 * ke2 * 16 * Pi * Pi * Pi * Pi) - (32 * Pi * Pi * Pi * ke2 * sigma2 * V2 / wavel) +
                     (16 * Pi * Pi * sigma2 * sigma2 * V2 * V2 / (wavel * wavel));
    const float qB = 16 * Pi * Pi * (ke2 - (sigma2 * V2 / (Pi * wavel)) - (1 / (4 * wavel * wavel)));
    const float qC = 3;
    const float disc = qB * qB - 4 * qA * qC;
    const float b24ac = std::sqrt(disc);
    float msd = (-qB + b24ac) / (2 * qA);
    msd = (float)(0.99 * (double)std::sqrt(msd));
    if (stem && msd > 0.06) msd = (float)0.06;
    int nFD = (int)std::ceil(sizeZ / msd);
    nFD += (nFD == 0);
    s->wavel = wavel;
    s->sigma2 = sigma2;
    s->ke2 = ke2;
    s->dzFD = msd;
    s->nFD = (disc >= 0 && msd > 0) ? nFD : -1;
    s->lbx = (int)std::ceil(std::sqrt(5.0f) / ((s->MaxX - s->MinX) / (kBins)));
    s->lby = (int)std::ceil(std::sqrt(5.0f) / ((s->MaxY - s->MinY) / (kBins)));
    s->lbz = (int)std::ceil(std::sqrt(5.0f) / (float)1);
    s->have_calc = true;
    s->have_freq = false;
    return 0;
}

/* PreCalculateFrequencies U.cu:1877-1964 (the unused 2x grids are not built). */
extern "C" int or_precalc(or_sim* s) {
    if (!s->have_calc) return fail(s, "calculation variables not set");
    pot_inputs_changed(s);
    const int nx = s->nx, ny = s->ny;
    const float ksizex = s->ps * nx, ksizey = s->ps * ny;
    const int imidx = (int)std::floor(nx / 2 + 0.5), imidy = (int)std::floor(ny / 2 + 0.5);
    s->kx.resize(nx);
    s->ky.resize(ny);
    for (int i = 1; i <= nx; ++i)
        s->kx[i - 1] = ((i - 1) > imidx) ? ((i - 1) - nx) / ksizex : (i - 1) / ksizex;
    for (int i = 1; i <= ny; ++i)
        s->ky[i - 1] = ((i - 1) > imidy) ? ((i - 1) - ny) / ksizey : (i - 1) / ksizey;
    if (imidx < 1 || imidy < 1) return fail(s, "grid too small");
    float kmaxx = (float)std::pow((double)(s->kx[imidx - 1] * 1 / 2), 2);
    float kmaxy = (float)std::pow((double)(s->ky[imidy - 1] * 1 / 2), 2);
    float km = (kmaxy <= kmaxx) ? kmaxy : kmaxx;
    s->kmax = std::sqrt(km);
    s->have_freq = true;
    return 0;
}

extern "C" int or_get_scalars(or_sim* s, double out[10]) {
    out[0] = s->wavel; out[1] = s->sigma2; out[2] = s->dzFD; out[3] = s->nFD;
    out[4] = s->kmax; out[5] = s->ke2; out[6] = s->convdz;
    float top = s->MaxZ - s->MinZ;
    out[7] = std::ceil(top / s->convdz);
    out[8] = s->lbx; out[9] = s->lby;
    return 0;
}

extern "C" int or_get_frequencies(or_sim* s, float* kx, float* ky) {
    if (!s->have_freq) return fail(s, "frequencies not computed");
    std::copy(s->kx.begin(), s->kx.end(), kx);
    std::copy(s->ky.begin(), s->ky.end(), ky);
    return 0;
}

/* ---------------- propagator and band limits ---------------- */
/* CreatePropsKernel U.cu:399-428: exp(-i*pi*dz*lambda*k^2) for sqrtf(kx^2+ky^2) < kmax. */
static void make_props(const or_sim* s, float dz, std::vector<cd>& P) {
    const int nx = s->nx, ny = s->ny;
    P.assign((size_t)nx * ny, cd(0, 0));
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            float k0x = s->kx[x] * s->kx[x], k0y = s->ky[y] * s->ky[y];
            if (std::sqrt(k0x + k0y) < s->kmax) {
                double kk = (double)s->kx[x] * s->kx[x] + (double)s->ky[y] * s->ky[y];
                double ph = 3.14159265 * (double)dz * (double)s->wavel * kk;
                P[(size_t)y * nx + x] = cd(std::cos(ph), -std::sin(ph));
            }
        }
}

/* BandLimitKernel U.cu:1025-1042: keep k <= kmax. */
static inline bool band_keep(const or_sim* s, int x, int y) {
    float k = std::sqrt(s->kx[x] * s->kx[x] + s->ky[y] * s->ky[y]);
    return k <= s->kmax;
}

static void ifft_norm(std::vector<cd>& a, int nx, int ny) {
    fft2d(a.data(), nx, ny, +1);
    const double inv = 1.0 / ((double)nx * ny);
    for (auto& v : a) v *= inv;
}

/* ---------------- wave initialisation ---------------- */
/* Second level for finite differences: psi = IFFT(P(dzFD) * FFT(psi_minus)) / N. */
static void propagate_fd_level(or_sim* s) {
    std::vector<cd> P;
    make_props(s, s->dzFD, P);
    s->psi = s->psi_minus;
    fft2d(s->psi.data(), s->nx, s->ny, -1);
    for (size_t i = 0; i < s->psi.size(); ++i) s->psi[i] *= P[i];
    ifft_norm(s->psi, s->nx, s->ny);
}

extern "C" int or_init_waves(or_sim* s, float conv_dz) {
    if (!s->have_freq) return fail(s, "frequencies not computed");
    pot_inputs_changed(s);
    s->convdz = conv_dz > 0 ? conv_dz : 1.0f; /* U.cu:1968 / U.cu:2005 */
    const size_t N = (size_t)s->nx * s->ny;
    s->psi_minus.assign(N, cd(1.0, 0.0));
    s->psi0 = s->psi_minus;
    propagate_fd_level(s);
    s->psi_plus.assign(N, cd(0, 0));
    s->have_waves = true;
    return 0;
}

extern "C" int or_set_fd_dz(or_sim* s, float dz) {
    if (!(dz > 0)) return fail(s, "bad FD dz");
    if (!s->have_atoms) return fail(s, "no atoms");
    s->dzFD = dz;
    int n = (int)std::ceil((s->MaxZ - s->MinZ) / dz);
    s->nFD = n + (n == 0);
    return 0;
}

/* STEMInitialiseWavefunctions U.cu:2672-2724 with STEMinitializingKernel U.cu:354-383. */
extern "C" int or_stem_init_waves(or_sim* s, int px, int py) {
    if (!s->have_freq) return fail(s, "frequencies not computed");
    const int nx = s->nx, ny = s->ny;
    const size_t N = (size_t)nx * ny;
    const float apert = (float)((double)s->aperture * 0.001 / (double)s->wavel);
    std::vector<cd> probe(N, cd(0, 0));
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            float k = std::sqrt(s->kx[x] * s->kx[x] + s->ky[y] * s->ky[y]);
            if (k < apert) {
                double kx = s->kx[x], ky = s->ky[y], k2 = kx * kx + ky * ky;
                double lam = s->wavel;
                double chi = 3.14159265 * lam * k2 * ((double)s->Cs * lam * lam * k2 * 0.5 + (double)s->df);
                double phi = 2 * 3.14159265 * (kx * px * (double)s->ps + ky * py * (double)s->ps);
                probe[(size_t)y * nx + x] = cd(std::cos(phi - chi), std::sin(phi - chi));
            }
        }
    fft2d(probe.data(), nx, ny, +1); /* unnormalised inverse, U.cu:2693 */
    double l1 = 0;
    for (auto& v : probe) l1 += std::abs(v);
    for (auto& v : probe) v /= l1; /* 1 / sum|psi|, U.cu:2698-2705 */
    s->psi_minus = probe;
    s->psi0 = probe;
    propagate_fd_level(s);
    s->psi_plus.assign(N, cd(0, 0));
    s->have_waves = true;
    return 0;
}

/* ---------------- potentials ---------------- */
static int check_pot(or_sim* s) {
    if (!s->have_bins) return fail(s, "atoms not binned");
    if (!s->have_fp) return fail(s, "fparams not loaded");
    if (!s->have_freq) return fail(s, "frequencies not computed");
    return 0;
}

/* Conventional potential, binnedAtomPKernel3 U.cu:582-653.
 * Slice `it` integrates 20 sub-planes z2 = z - m*convdz/20 (m = 1..20) below
 * z = (MaxZ-MinZ) - convdz*it over atoms whose 1-A z-bin lies within +-3 of
 * floor((MaxZ-MinZ) - z), with the r^2 < 5 cutoff per sub-plane. */
/* Sub-plane integrated potential below plane z (FP32 shifted frame): the sum
 * over atoms of the z-bin window K -+ lbz, K = floor((top - z) / 1), and over
 * sub-planes z - m * dz / nsub (m = 1..nsub, FP32 as written) with
 * r^2 < 5 A^2 (FP32), of (dz / nsub) * vatom(r^2).  nsub = 20:
 * binnedAtomPKernel3 (U.cu:582-653); nsub = 10, dz = 1: binnedAtomPKernelRS
 * (U.cu:655-727). */
static int sub_plane_potential(or_sim* s, float z, float dz, int nsub, double* out);

extern "C" int or_potential_conventional(or_sim* s, int it, double* out) {
    if (check_pot(s)) return -1;
    const float z = s->MaxZ - s->MinZ - s->convdz * it; /* U.cu:2097, FP32 */
    return sub_plane_potential(s, z, s->convdz, 20, out);
}

/* binnedAtomPKernelRS at MultisliceStepRS's plane z = top - 1 * it (U.cu:2137). */
extern "C" int or_potential_rs(or_sim* s, int it, double* out) {
    if (check_pot(s)) return -1;
    const float z = s->MaxZ - s->MinZ - (float)(1 * it);
    return sub_plane_potential(s, z, 1.0f, 10, out);
}

static int sub_plane_potential(or_sim* s, float z, float dz, int nsub, double* out) {
    const int nx = s->nx, ny = s->ny, nz = s->nzb;
    const int K = (int)std::floor((s->MaxZ - s->MinZ - z) / (float)1);
    int kt = K - s->lbz, kb = K + s->lbz;
    if (kt < 0) kt = 0;
    if (kb >= nz) kb = nz - 1;
    const float w_x = (s->MaxX - s->MinX) / kBins, w_y = (s->MaxY - s->MinY) / kBins;
    const int rx = (int)std::ceil(2.2361 / w_x) + 1, ry = (int)std::ceil(2.2361 / w_y) + 1;
    float z2f[20];
    double z2d[20];
    for (int m = 1; m <= nsub; ++m) {
        z2f[m - 1] = z - m * dz / (float)nsub;
        z2d[m - 1] = (double)z - m * (double)dz / (double)nsub;
    }
    const double wsub = (double)dz / (double)nsub;
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < ny; ++y) {
        for (int x = 0; x < nx; ++x) {
            const float pxf = s->xoff + x * s->ps, pyf = s->yoff + y * s->ps;
            const double pxd = (double)s->xoff + x * (double)s->ps;
            const double pyd = (double)s->yoff + y * (double)s->ps;
            const int cbx = (int)std::floor(pxf / w_x), cby = (int)std::floor(pyf / w_y);
            double sum = 0;
            for (int k = kt; k <= kb; ++k)
                for (int j = std::max(cby - ry, 0); j <= std::min(cby + ry, kBins - 1); ++j)
                    for (int i = std::max(cbx - rx, 0); i <= std::min(cbx + rx, kBins - 1); ++i) {
                        const int b = k * kBins * kBins + j * kBins + i;
                        for (int l = s->off[b]; l < s->off[b + 1]; ++l) {
                            const float dxf = pxf - s->bx[l], dyf = pyf - s->by[l];
                            const float dxy = dxf * dxf + dyf * dyf;
                            double ox = 0, oy = 0;
                            if (!s->valdx.empty()) { ox = s->valdx[s->perm[l]]; oy = s->valdy[s->perm[l]]; }
                            const double dxd = pxd - (s->bx[l] + ox), dyd = pyd - (s->by[l] + oy);
                            const double dxyd = dxd * dxd + dyd * dyd;
                            for (int m = 0; m < nsub; ++m) {
                                const float dzf = z2f[m] - s->bz[l];
                                const float r2f = dxy + dzf * dzf;
                                if (r2f < 5.0f) {
                                    const double dzd = z2d[m] - s->bz[l];
                                    sum += wsub * or_vatom(s->fp.data(), s->bZ[l], dxyd + dzd * dzd);
                                }
                            }
                        }
                    }
            out[(size_t)y * nx + x] = sum;
        }
    }
    return 0;
}

/* Finite-difference potential, binnedAtomPKernelFD U.cu:883-946: V at the plane
 * z = (MaxZ-MinZ) - dzFD*it, no block offsets, z-bin window +-3, r^2 < 5. */
extern "C" int or_potential_fd(or_sim* s, int it, double* out) {
    if (check_pot(s)) return -1;
    const int nx = s->nx, ny = s->ny, nz = s->nzb;
    const float z = s->MaxZ - s->MinZ - s->dzFD * it; /* U.cu:2051 */
    const int K = (int)std::floor((s->MaxZ - s->MinZ - z) / (float)1);
    int kt = K - s->lbz, kb = K + s->lbz;
    if (kt < 0) kt = 0;
    if (kb >= nz) kb = nz - 1;
    const float w_x = (s->MaxX - s->MinX) / kBins, w_y = (s->MaxY - s->MinY) / kBins;
    const int rx = (int)std::ceil(2.2361 / w_x) + 1, ry = (int)std::ceil(2.2361 / w_y) + 1;
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const float pxf = x * s->ps, pyf = y * s->ps;
            const double pxd = x * (double)s->ps, pyd = y * (double)s->ps;
            const int cbx = (int)std::floor(pxf / w_x), cby = (int)std::floor(pyf / w_y);
            double sum = 0;
            for (int k = kt; k <= kb; ++k)
                for (int j = std::max(cby - ry, 0); j <= std::min(cby + ry, kBins - 1); ++j)
                    for (int i = std::max(cbx - rx, 0); i <= std::min(cbx + rx, kBins - 1); ++i) {
                        const int b = k * kBins * kBins + j * kBins + i;
                        for (int l = s->off[b]; l < s->off[b + 1]; ++l) {
                            const float dxf = pxf - s->bx[l], dyf = pyf - s->by[l], dzf = z - s->bz[l];
                            const float r2f = dxf * dxf + dyf * dyf + dzf * dzf;
                            if (r2f < 5.0f) {
                                const double dxd = pxd - s->bx[l], dyd = pyd - s->by[l];
                                const double dzd = (double)z - s->bz[l];
                                sum += or_vatom(s->fp.data(), s->bZ[l], dxd * dxd + dyd * dyd + dzd * dzd);
                            }
                        }
                    }
            out[(size_t)y * nx + x] = sum;
        }
    return 0;
}

/* Projected-potential mode (vzatom2, U.cu:119-152, with the xy scan of
 * binnedAtomPKernel2 U.cu:513-578): slice `it` (1-based) holds the atoms whose
 * depth d = (MaxZ-MinZ) - z_atom satisfies floorf(d / dz) == it - 1 (FP32);
 * each adds vzatom2 within r^2 < 5 in the plane. */
extern "C" int or_potential_projected(or_sim* s, int it, float dz, double* out) {
    if (check_pot(s)) return -1;
    if (!(dz > 0)) return fail(s, "bad slice thickness");
    const int nx = s->nx, ny = s->ny, nz = s->nzb;
    const float top = s->MaxZ - s->MinZ;
    const float w_x = (s->MaxX - s->MinX) / kBins, w_y = (s->MaxY - s->MinY) / kBins;
    const int rx = (int)std::ceil(2.2361 / w_x) + 1, ry = (int)std::ceil(2.2361 / w_y) + 1;
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const float pxf = s->xoff + x * s->ps, pyf = s->yoff + y * s->ps;
            const double pxd = (double)s->xoff + x * (double)s->ps;
            const double pyd = (double)s->yoff + y * (double)s->ps;
            const int cbx = (int)std::floor(pxf / w_x), cby = (int)std::floor(pyf / w_y);
            double sum = 0;
            for (int k = 0; k < nz; ++k)
                for (int j = std::max(cby - ry, 0); j <= std::min(cby + ry, kBins - 1); ++j)
                    for (int i = std::max(cbx - rx, 0); i <= std::min(cbx + rx, kBins - 1); ++i) {
                        const int b = k * kBins * kBins + j * kBins + i;
                        for (int l = s->off[b]; l < s->off[b + 1]; ++l) {
                            const int slab = (int)std::floor((top - s->bz[l]) / dz);
                            if (slab != it - 1) continue;
                            const float dxf = pxf - s->bx[l], dyf = pyf - s->by[l];
                            const float r2f = dxf * dxf + dyf * dyf;
                            if (r2f < 5.0f) {
                                const double dxd = pxd - s->bx[l], dyd = pyd - s->by[l];
                                sum += or_vzatom2(s->fp.data(), s->bZ[l], dxd * dxd + dyd * dyd);
                            }
                        }
                    }
            out[(size_t)y * nx + x] = sum;
        }
    return 0;
}

/* ---------------- slice steps ---------------- */
/* One transmission + propagation: psi <- IFFT(P * FFT(exp(i*sigma*V) * in)) / N. */
static void tp_step(or_sim* s, const std::vector<double>& V, const std::vector<cd>& in) {
    const int nx = s->nx, ny = s->ny;
    const size_t N = (size_t)nx * ny;
    const double sig = s->sigma2;
    s->psi_plus.resize(N);
    for (size_t i = 0; i < N; ++i) s->psi_plus[i] = std::polar(1.0, sig * V[i]) * in[i];
    std::vector<cd> P;
    make_props(s, s->convdz, P);
    fft2d(s->psi_plus.data(), nx, ny, -1);
    for (size_t i = 0; i < N; ++i) s->psi_plus[i] *= P[i];
    ifft_norm(s->psi_plus, nx, ny);
    s->psi = s->psi_plus;
}

/* MultisliceStepConv U.cu:2085-2124.  Iteration 1 starts from the initial wave
 * (plane wave or probe), later iterations from the current wave. */
/* MultisliceStepRS (U.cu:2126-2178) as written.  Ten terms, m = 1..10, of
 *   w <- w + i pre_m (L w + V w),  pre_m = (1/m) lambda dz / (4 * 3.1415927), dz = 1,
 * where the first term restarts from w = 1 (RSMS U.cu:849-877) and L is the
 * sum of DifferentialXKernel and DifferentialYKernel (U.cu:797-847):
 *   (1/ps^2) (4/3 (w[+1] + w[-1] - w[0]) - 1/12 (w[+2] + w[-2] - w[0]))
 * per direction, with neighbours beyond an edge read at index 0 of that
 * line (the kernels' (i>0)*(i-1) style indices), and V the un-exponentiated
 * RS potential.  Afterwards Psi = w; from the second iteration on
 * PsiMinus = w * Psi_previous (the multiplication is kept, the final copy
 * overwrites Psi with w). */
extern "C" int or_step_rs(or_sim* s, int it) {
    if (!s->have_waves) return fail(s, "waves not initialised");
    const int nx = s->nx, ny = s->ny;
    const size_t N = (size_t)nx * ny;
    std::vector<double> V(N);
    if (or_potential_rs(s, it, V.data())) return -1;
    const double pre0 = (double)s->wavel * 1.0 / (4.0 * 3.1415927);
    const double ips2 = 1.0 / ((double)s->ps * (double)s->ps);
    std::vector<cd> w(N, cd(1.0, 0.0)), nw(N);
    for (int m = 1; m <= 10; ++m) {
        const double pre = pre0 / m;
        if (m == 1) {
            for (size_t i = 0; i < N; ++i) w[i] = cd(1.0, pre * V[i]);
            continue;
        }
#pragma omp parallel for schedule(static)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const size_t i = (size_t)y * nx + x;
                const int p1 = (x > 0) * (x - 1), p2 = (x > 1) * (x - 2);
                const int n1 = (x < nx - 1) * (x + 1), n2 = (x < nx - 2) * (x + 2);
                const int q1 = (y > 0) * (y - 1), q2 = (y > 1) * (y - 2);
                const int o1 = (y < ny - 1) * (y + 1), o2 = (y < ny - 2) * (y + 2);
                const size_t row = (size_t)y * nx;
                const cd c = w[i];
                const cd dx1 = w[row + n1] + w[row + p1] - c, dx2 = w[row + n2] + w[row + p2] - c;
                const cd dy1 = w[(size_t)o1 * nx + x] + w[(size_t)q1 * nx + x] - c;
                const cd dy2 = w[(size_t)o2 * nx + x] + w[(size_t)q2 * nx + x] - c;
                const cd lap = ips2 * (4.0 * dx1 / 3.0 - dx2 / 12.0) + ips2 * (4.0 * dy1 / 3.0 - dy2 / 12.0);
                nw[i] = c + cd(0.0, pre) * (lap + V[i] * c);
            }
        w.swap(nw);
    }
    if (it > 1) {
        s->psi_minus.resize(N);
        for (size_t i = 0; i < N; ++i) s->psi_minus[i] = w[i] * s->psi[i];
    }
    s->psi = w;
    return 0;
}

extern "C" int or_step_conventional(or_sim* s, int it) {
    if (!s->have_waves) return fail(s, "waves not initialised");
    std::vector<cd> in = (it == 1) ? s->psi0 : s->psi;
    if (s->vcache_on) {
        auto f = s->vcache.find(it);
        if (f == s->vcache.end()) {
            std::vector<double> V((size_t)s->nx * s->ny);
            if (or_potential_conventional(s, it, V.data())) return -1;
            f = s->vcache.emplace(it, std::move(V)).first;
        }
        tp_step(s, f->second, in);
        return 0;
    }
    std::vector<double> V((size_t)s->nx * s->ny);
    if (or_potential_conventional(s, it, V.data())) return -1;
    tp_step(s, V, in);
    return 0;
}

/* One conventional step on a caller-given potential V (N doubles, V*A): the
 * transmission and propagation of MultisliceStepConv (U.cu:2101-2122) without
 * the potential build, for timing the slice step alone. */
extern "C" int or_step_given_potential(or_sim* s, int it, const double* V) {
    if (!s->have_waves) return fail(s, "waves not initialised");
    const size_t N = (size_t)s->nx * s->ny;
    std::vector<double> v(V, V + N);
    std::vector<cd> in = (it == 1) ? s->psi0 : s->psi;
    tp_step(s, v, in);
    return 0;
}

/* Keeps (on != 0) or drops the conventional potential of each iteration for
 * reuse by later steps of the same specimen and set-up (many probe positions
 * over one potential stack); off also frees the cache. */
extern "C" int or_cache_potentials(or_sim* s, int on) {
    s->vcache_on = on != 0;
    if (!on) s->vcache.clear();
    return 0;
}

extern "C" int or_step_projected(or_sim* s, int it) {
    if (!s->have_waves) return fail(s, "waves not initialised");
    std::vector<double> V((size_t)s->nx * s->ny);
    if (or_potential_projected(s, it, s->convdz, V.data())) return -1;
    std::vector<cd> in = (it == 1) ? s->psi0 : s->psi;
    tp_step(s, V, in);
    return 0;
}

/* MultisliceStep (finite differences) U.cu:2040-2083 with BandLimitKernel,
 * gradKernel and finiteDifferenceKernel (U.cu:948-1042). */
extern "C" int or_step_fd(or_sim* s, int it) {
    if (!s->have_waves) return fail(s, "waves not initialised");
    if (s->nFD < 0) return fail(s, "no stable finite-difference step for these conditions");
    const int nx = s->nx, ny = s->ny;
    const size_t N = (size_t)nx * ny;
    std::vector<double> Vr(N);
    if (or_potential_fd(s, it, Vr.data())) return -1;
    /* band-limit V */
    std::vector<cd> V(N);
    for (size_t i = 0; i < N; ++i) V[i] = cd(Vr[i], 0.0);
    fft2d(V.data(), nx, ny, -1);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x)
            if (!band_keep(s, x, y)) V[(size_t)y * nx + x] = 0;
    ifft_norm(V, nx, ny);
    /* spectral Laplacian, pi = 3.14159 as at U.cu:959 */
    std::vector<cd> g = s->psi;
    fft2d(g.data(), nx, ny, -1);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            double kk = (double)s->kx[x] * s->kx[x] + (double)s->ky[y] * s->ky[y];
            g[(size_t)y * nx + x] *= -4.0 * 3.14159 * 3.14159 * kk;
        }
    ifft_norm(g, nx, ny);
    /* three-level update, U.cu:995-1023 */
    const double dz = s->dzFD, lam = s->wavel, sig = s->sigma2;
    const cd cminus(1.0, -2 * 3.14159 * dz / lam), cplus(1.0, 2 * 3.14159 * dz / lam);
    const cd rcp = 1.0 / cplus, ratio = cminus / cplus;
    s->psi_plus.resize(N);
    for (size_t i = 0; i < N; ++i) {
        cd A = 2.0 * s->psi[i] - dz * dz * g[i] - dz * dz * 4 * 3.14159 * sig * V[i].real() * s->psi[i] / lam;
        s->psi_plus[i] = rcp * A - ratio * s->psi_minus[i];
    }
    fft2d(s->psi_plus.data(), nx, ny, -1);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x)
            if (!band_keep(s, x, y)) s->psi_plus[(size_t)y * nx + x] = 0;
    ifft_norm(s->psi_plus, nx, ny);
    s->psi_minus = s->psi;
    s->psi = s->psi_plus;
    return 0;
}

extern "C" int or_get_wave(or_sim* s, double* out) {
    if (!s->have_waves) return fail(s, "waves not initialised");
    std::memcpy(out, s->psi.data(), s->psi.size() * sizeof(cd));
    return 0;
}

extern "C" int or_set_wave(or_sim* s, const double* in) {
    if (!s->have_freq) return fail(s, "frequencies not computed");
    const size_t N = (size_t)s->nx * s->ny;
    s->psi.resize(N);
    std::memcpy((void*)s->psi.data(), in, N * sizeof(cd));
    s->have_waves = true;
    return 0;
}

/* ---------------- read-out ---------------- */
/* Deterministic CTF image, SimulateImage U.cu:2311-2343 with imagingKernel2
 * U.cu:1044-1080: I = |IFFT(E_s E_d exp(-i chi) FFT(psi)/sqrt(N))/sqrt(N)|^2
 * inside the objective aperture. */
extern "C" int or_simulate_image(or_sim* s, double* out) {
    if (!s->have_waves) return fail(s, "waves not initialised");
    const int nx = s->nx, ny = s->ny;
    const size_t N = (size_t)nx * ny;
    std::vector<cd> a = s->psi;
    fft2d(a.data(), nx, ny, -1);
    const float wavel = s->wavel;
    const float objap = s->aperture;
    const float objap2 = (((objap * 0.001f) / wavel) * ((objap * 0.001f) / wavel));
    const double lam = wavel, Cs = s->Cs, df = s->df;
    const double beta = (double)(s->beta / 1000), delta = s->delta;
    const double Chi1 = 3.1415926 * lam, Chi2 = 0.5 * Cs * lam * lam;
    const double factor = beta * beta / (4 * lam * lam);
    const double sN = std::sqrt((double)N);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const size_t i = (size_t)y * nx + x;
            const float k2f = s->kx[x] * s->kx[x] + s->ky[y] * s->ky[y];
            if (!(k2f < objap2)) { a[i] = 0; continue; }
            const double kx = s->kx[x], ky = s->ky[y];
            const double k2 = kx * kx + ky * ky, k = std::sqrt(k2);
            const double es = std::exp(-factor * std::pow(3.141593 * k * lam * 2 * df +
                                                          2 * 3.141593 * lam * lam * lam * Cs * k2 * k, 2));
            const double ed = std::exp(-0.25 * delta * delta * 3.141593 * 3.141593 * k2 * k2 * lam * lam);
            const double phi = std::atan2(ky, kx);
            const double chi = Chi1 * k2 *
                               (Chi2 * k2 + df + (double)s->A2 * std::sin(2.0 * (phi - (double)s->phi2)) +
                                2.0 * (double)s->A3 * lam * std::sqrt(k2) * std::sin(3.0 * (phi - (double)s->phi3)) / 3.0);
            a[i] = (a[i] / sN) * std::polar(es * ed, -chi);
        }
    fft2d(a.data(), nx, ny, +1);
    for (size_t i = 0; i < N; ++i) out[i] = std::norm(a[i] / sN);
    return 0;
}

extern "C" int or_alloc_tds(or_sim* s) {
    s->tds.assign((size_t)s->nx * s->ny, 0.0);
    return 0;
}

/* AddTDSWaves U.cu:2734-2766: TDS += |centre(FFT(psi))| (unnormalised FFT,
 * CentreKernel U.cu:964-993 as written). */
extern "C" int or_add_tds(or_sim* s) {
    if (!s->have_waves) return fail(s, "waves not initialised");
    const int nx = s->nx, ny = s->ny;
    if (s->tds.size() != (size_t)nx * ny) or_alloc_tds(s);
    std::vector<cd> a = s->psi;
    fft2d(a.data(), nx, ny, -1);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            int x2 = x + nx / 2, y2 = y + ny / 2;
            if (x >= nx / 2) x2 = x - nx / 2;
            if (y >= ny / 2) y2 = y - ny / 2;
            s->tds[(size_t)y * nx + x] += std::abs(a[(size_t)y2 * nx + x2]);
        }
    return 0;
}

extern "C" int or_get_tds(or_sim* s, double* out) {
    std::copy(s->tds.begin(), s->tds.end(), out);
    return 0;
}

extern "C" int or_diffraction(or_sim* s, double* out) {
    if (!s->have_waves) return fail(s, "waves not initialised");
    const size_t N = (size_t)s->nx * s->ny;
    std::vector<cd> a = s->psi;
    fft2d(a.data(), s->nx, s->ny, -1);
    for (size_t i = 0; i < N; ++i) out[i] = std::norm(a[i]) / (double)N;
    return 0;
}

/* Annular detector (no reference counterpart): sum of |FFT(psi)|^2/N over
 * pixels with kin^2 <= kx^2+ky^2 < kout^2, kin = (inner*0.001f)/wavel (FP32). */
extern "C" int or_annular_detector(or_sim* s, float inner, float outer, double* out) {
    if (!s->have_waves) return fail(s, "waves not initialised");
    const int nx = s->nx, ny = s->ny;
    std::vector<double> I((size_t)nx * ny);
    or_diffraction(s, I.data());
    const float kin = (inner * 0.001f) / s->wavel, kout = (outer * 0.001f) / s->wavel;
    const float kin2 = kin * kin, kout2 = kout * kout;
    double acc = 0;
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const float k2 = s->kx[x] * s->kx[x] + s->ky[y] * s->ky[y];
            if (k2 >= kin2 && k2 < kout2) acc += I[(size_t)y * nx + x];
        }
    *out = acc;
    return 0;
}

/* ======================================================================
 * Differentiable focal series (no reference counterpart): FP64 forward and
 * adjoint used to check the engine's gradient.
 *   psi_n = A(t_n psi_{n-1}),  A = IFFT(P FFT(.))/N,  t_n = exp(i sigma V_n)
 *   phi_d = B_d psi_S,  B_d = IFFT(CTF_d FFT(.)/sqrt N)/sqrt N,  I_d = |phi_d|^2
 *   L = sum_d sum_px (I_d - T_d)^2
 * Adjoint (g = dL/dpsi*):  g_S = sum_d B_d^H [2 (I_d - T_d) phi_d],
 *   h = A^H g_n,  dL/dV_n = -2 sigma Im(conj(h) t_n psi_{n-1}),  g_{n-1} = conj(t_n) h.
 * ==================================================================== */
static void ctf_apply(const or_sim* s, double df, bool conjugate, std::vector<cd>& a) {
    /* a <- IFFT(W FFT(a)/sqrt N)/sqrt N with W the CTF weight of or_simulate_image at defocus df */
    const int nx = s->nx, ny = s->ny;
    const double sN = std::sqrt((double)nx * ny);
    fft2d(a.data(), nx, ny, -1);
    const float wavel = s->wavel, objap = s->aperture;
    const float objap2 = (((objap * 0.001f) / wavel) * ((objap * 0.001f) / wavel));
    const double lam = wavel, Cs = s->Cs;
    const double beta = (double)(s->beta / 1000), delta = s->delta;
    const double Chi1 = 3.1415926 * lam, Chi2 = 0.5 * Cs * lam * lam, factor = beta * beta / (4 * lam * lam);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const size_t i = (size_t)y * nx + x;
            const float k2f = s->kx[x] * s->kx[x] + s->ky[y] * s->ky[y];
            if (!(k2f < objap2)) { a[i] = 0; continue; }
            const double kx = s->kx[x], ky = s->ky[y], k2 = kx * kx + ky * ky, k = std::sqrt(k2);
            const double es = std::exp(-factor * std::pow(3.141593 * k * lam * 2 * df +
                                                          2 * 3.141593 * lam * lam * lam * Cs * k2 * k, 2));
            const double ed = std::exp(-0.25 * delta * delta * 3.141593 * 3.141593 * k2 * k2 * lam * lam);
            const double phi = std::atan2(ky, kx);
            const double chi = Chi1 * k2 * (Chi2 * k2 + df + (double)s->A2 * std::sin(2.0 * (phi - (double)s->phi2)));
            cd w = std::polar(es * ed, -chi);
            if (conjugate) w = std::conj(w);
            a[i] = (a[i] / sN) * w;
        }
    fft2d(a.data(), nx, ny, +1);
    for (auto& v : a) v /= sN;
}

static void propagate(const or_sim* s, const std::vector<cd>& P, bool conjugate, std::vector<cd>& a) {
    fft2d(a.data(), s->nx, s->ny, -1);
    for (size_t i = 0; i < a.size(); ++i) a[i] *= conjugate ? std::conj(P[i]) : P[i];
    ifft_norm(a, s->nx, s->ny);
}

/* Forward of the focal series.  Vstack (S*N, may be NULL: the conventional
 * potentials are computed) and optional images out (nd*N). */
extern "C" int or_focal_forward(or_sim* s, const float* defoci, int nd, const double* targets,
                                const double* Vstack, int S, double* loss, double* images) {
    if (!s->have_waves) return fail(s, "waves not initialised");
    const int nx = s->nx, ny = s->ny;
    const size_t N = (size_t)nx * ny;
    std::vector<cd> P, psi = s->psi0;
    make_props(s, s->convdz, P);
    std::vector<double> V(N);
    for (int n = 1; n <= S; ++n) {
        if (Vstack) std::copy(Vstack + (size_t)(n - 1) * N, Vstack + (size_t)n * N, V.begin());
        else if (or_potential_conventional(s, n, V.data())) return -1;
        for (size_t i = 0; i < N; ++i) psi[i] *= std::polar(1.0, (double)s->sigma2 * V[i]);
        propagate(s, P, false, psi);
    }
    double L = 0;
    for (int d = 0; d < nd; ++d) {
        std::vector<cd> phi = psi;
        ctf_apply(s, defoci[d], false, phi);
        for (size_t i = 0; i < N; ++i) {
            const double I = std::norm(phi[i]);
            const double r = I - targets[(size_t)d * N + i];
            L += r * r;
            if (images) images[(size_t)d * N + i] = I;
        }
    }
    *loss = L;
    return 0;
}

/* dv/d(r^2) of vatom (U.cu:160-193) in FP64; zero inside the 0.25 A clamp. */
static double dvatom_dr2(const double* fp, int Z, double r2) {
    const double* f = fp + (Z - 1) * 12;
    const double r = std::sqrt(r2);
    if (r < 0.25) return 0.0;
    const double pi = 3.141592654;
    double d = 0;
    for (int i = 0; i < 6; i += 2) {
        const double b = 2.0 * pi * std::sqrt(f[i + 1]);
        d += 150.4121417 * f[i] * std::exp(-b * r) * (-1.0 / (r * r) - b / r) / (2.0 * r);
    }
    for (int i = 6; i < 12; i += 2) {
        const double g = pi * pi / f[i + 1];
        d += 266.5157269 * f[i] * std::pow(f[i + 1], -1.5) * std::exp(-g * r2) * (-g);
    }
    return d;
}

/* FP64 loss and gradient: dLdV (S*N) and dLdxy (2*n_atoms, input order;
 * derivative with the box held fixed), either may be NULL. */
extern "C" int or_focal_grad(or_sim* s, const float* defoci, int nd, const double* targets, int S,
                             double* loss, double* dLdV, double* dLdxy) {
    if (!s->have_waves) return fail(s, "waves not initialised");
    if (check_pot(s)) return -1;
    const int nx = s->nx, ny = s->ny;
    const size_t N = (size_t)nx * ny;
    std::vector<cd> P;
    make_props(s, s->convdz, P);
    std::vector<std::vector<cd>> psis(S + 1);
    std::vector<std::vector<double>> Vs(S + 1);
    psis[0] = s->psi0;
    for (int n = 1; n <= S; ++n) {
        Vs[n].resize(N);
        if (or_potential_conventional(s, n, Vs[n].data())) return -1;
        std::vector<cd> a = psis[n - 1];
        for (size_t i = 0; i < N; ++i) a[i] *= std::polar(1.0, (double)s->sigma2 * Vs[n][i]);
        propagate(s, P, false, a);
        psis[n] = a;
    }
    double L = 0;
    std::vector<cd> g(N, cd(0, 0));
    for (int d = 0; d < nd; ++d) {
        std::vector<cd> phi = psis[S];
        ctf_apply(s, defoci[d], false, phi);
        for (size_t i = 0; i < N; ++i) {
            const double I = std::norm(phi[i]);
            const double r = I - targets[(size_t)d * N + i];
            L += r * r;
            phi[i] *= 2.0 * r;
        }
        ctf_apply(s, defoci[d], true, phi);
        for (size_t i = 0; i < N; ++i) g[i] += phi[i];
    }
    *loss = L;
    const double sig = s->sigma2;
    std::vector<double> G(N);
    if (dLdxy) std::fill(dLdxy, dLdxy + 2 * s->x.size(), 0.0);
    const std::vector<int>& perm = s->perm;
    for (int n = S; n >= 1; --n) {
        std::vector<cd> h = g;
        propagate(s, P, true, h);
        for (size_t i = 0; i < N; ++i) {
            const cd t = std::polar(1.0, sig * Vs[n][i]);
            G[i] = -2.0 * sig * std::imag(std::conj(h[i]) * t * psis[n - 1][i]);
            g[i] = std::conj(t) * h[i];
        }
        if (dLdV) std::copy(G.begin(), G.end(), dLdV + (size_t)(n - 1) * N);
        if (dLdxy) {
            /* chain rule through binnedAtomPKernel3's sum, same FP32 decisions */
            const float z = s->MaxZ - s->MinZ - s->convdz * n;
            const int K = (int)std::floor((s->MaxZ - s->MinZ - z) / (float)1);
            const int kt = std::max(K - s->lbz, 0), kb = std::min(K + s->lbz, s->nzb - 1);
            float z2f[20];
            double z2d[20];
            for (int m = 1; m <= 20; ++m) {
                z2f[m - 1] = z - m * s->convdz / 20.0f;
                z2d[m - 1] = (double)z - m * (double)s->convdz / 20.0;
            }
            const double wsub = (double)s->convdz / 20.0;
            const int a0 = s->off[kt * kBins * kBins], a1 = s->off[(kb + 1) * kBins * kBins];
#pragma omp parallel for schedule(dynamic, 8)
            for (int l = a0; l < a1; ++l) {
                double X = s->bx[l], Y = s->by[l];
                if (!s->valdx.empty()) { X += s->valdx[perm[l]]; Y += s->valdy[perm[l]]; }
                const int x0 = std::max(0, (int)std::floor((X - s->xoff - 2.3) / s->ps));
                const int x1 = std::min(nx - 1, (int)std::ceil((X - s->xoff + 2.3) / s->ps));
                const int y0 = std::max(0, (int)std::floor((Y - s->yoff - 2.3) / s->ps));
                const int y1 = std::min(ny - 1, (int)std::ceil((Y - s->yoff + 2.3) / s->ps));
                double gx = 0, gy = 0;
                for (int y = y0; y <= y1; ++y)
                    for (int x = x0; x <= x1; ++x) {
                        const float pxf = s->xoff + x * s->ps, pyf = s->yoff + y * s->ps;
                        const float dxf = pxf - s->bx[l], dyf = pyf - s->by[l];
                        const float dxy = dxf * dxf + dyf * dyf;
                        if (!(dxy < 5.0f)) continue;
                        const double pxd = (double)s->xoff + x * (double)s->ps, pyd = (double)s->yoff + y * (double)s->ps;
                        const double dxd = pxd - X, dyd = pyd - Y;
                        double acc = 0;
                        for (int m = 0; m < 20; ++m) {
                            const float dzf = z2f[m] - s->bz[l];
                            if (!(dxy + dzf * dzf < 5.0f)) continue;
                            const double dzd = z2d[m] - s->bz[l];
                            acc += wsub * dvatom_dr2(s->fp.data(), s->bZ[l], dxd * dxd + dyd * dyd + dzd * dzd);
                        }
                        const double Gp = G[(size_t)y * nx + x];
                        gx += Gp * acc * (-2.0 * dxd);
                        gy += Gp * acc * (-2.0 * dyd);
                    }
                dLdxy[2 * perm[l]] += gx;
                dLdxy[2 * perm[l] + 1] += gy;
            }
        }
    }
    return 0;
}

/* Test hook: offset atom i's position by (dx, dy) in the potential VALUES
 * only; every FP32 decision keeps the stored position.  Finite differences
 * taken this way see no cut-off flips and measure the chain-rule gradient. */
extern "C" int or_set_value_offset(or_sim* s, int i, double dx, double dy) {
    if (!s->have_atoms || i < 0 || i >= (int)s->x.size()) return fail(s, "bad atom index");
    pot_inputs_changed(s);
    if (s->valdx.empty()) {
        s->valdx.assign(s->x.size(), 0.0);
        s->valdy.assign(s->x.size(), 0.0);
    }
    s->valdx[i] = dx;
    s->valdy[i] = dy;
    return 0;
}

/* ======================================================================
 * Detector chain of SimulateImage (U.cu:2345-2437) on an FP64 CTF intensity
 * I (N doubles): F = FFT(I)/sqrt N * sqrt(DQE(r)), a = |IFFT(F)/sqrt N|,
 * counts = round(dose a + sqrt(|dose a|) z), G = FFT(counts)/sqrt N * NTF(r),
 * out = |IFFT(G)/sqrt N| * conversion^2.  r: the table index
 * floor(sqrtf(dx^2 + dy^2) / binning) in FP32 (DQEFunc U.cu:1120-1132),
 * 0.0001 beyond the table; z: the clipped normal of Philox4x32-10 at counter
 * (pixel, serial, 0x5407, 0), key (seed lo, seed hi), Box-Muller as the
 * reference (U.cu:2389-2397) with u = r * 2^-32.
 * ==================================================================== */
extern "C" double or_clipped_normal(uint32_t r1, uint32_t r2) {
    const double u1 = (double)r1 * 2.3283064365386963e-10, u2 = (double)r2 * 2.3283064365386963e-10;
    double z = std::sqrt(-2.0 * std::log(1.17549435e-38 + u1)) * std::sin((double)(2.0f * 3.1415926f) * u2);
    if (z <= -3.0) z = -3.0;
    if (z >= 3.0) z = 3.0;
    return z;
}

static double detector_table(int x, int y, int nx, int ny, const float* tab, int n, int binning) {
    const int xd = x - (x < nx / 2 ? 0 : nx), yd = y - (y < ny / 2 ? 0 : ny);
    const float rad = std::sqrt((float)(xd * xd + yd * yd)) / binning;
    const int r2 = (int)std::floor(rad);
    return r2 <= n - 1 ? (double)tab[r2] : (double)0.0001f;
}

extern "C" int or_detector_chain(or_sim* s, const double* I, float dose, uint32_t serial, const float* dqe,
                                 const float* ntf, int n, int binning, float conversion, uint64_t seed, double* out) {
    const int nx = s->nx, ny = s->ny;
    const size_t N = (size_t)nx * ny;
    const double isN = 1.0 / std::sqrt((double)N);
    std::vector<cd> a(N);
    for (size_t i = 0; i < N; ++i) a[i] = cd(I[i], 0.0);
    fft2d(a.data(), nx, ny, -1);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x)
            a[(size_t)y * nx + x] *= isN * std::sqrt(detector_table(x, y, nx, ny, dqe, n, binning));
    fft2d(a.data(), nx, ny, +1);
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    for (size_t i = 0; i < N; ++i) {
        const double amp = std::abs(a[i] * isN);
        const uint32_t ctr[4] = {(uint32_t)i, serial, 0x5407u, 0u};
        uint32_t r[4];
        or_philox4x32_10(ctr, key, r);
        const double z = or_clipped_normal(r[0], r[1]);
        const double na = (double)dose * amp;
        a[i] = cd(std::round(na + std::sqrt(std::fabs(na)) * z), 0.0);
    }
    fft2d(a.data(), nx, ny, -1);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x)
            a[(size_t)y * nx + x] *= isN * detector_table(x, y, nx, ny, ntf, n, binning);
    fft2d(a.data(), nx, ny, +1);
    const double c2 = (double)conversion * (double)conversion;
    for (size_t i = 0; i < N; ++i) out[i] = std::abs(a[i]) * isN * c2;
    return 0;
}
