// bm3d_oracle.cpp -- CPU oracle for the BM3D / V-BM3D per-frame hot path.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker: only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg may load it. The product (vapoursynth-bm3d_b200/) never links it.
//
// It restates, in plain C++, the arithmetic of the reference plugin
// (HomeOfVapourSynthEvolution/VapourSynth-BM3D v10.1).  Every function cites the reference
// file:line it follows.  Parity status:
//   * block matching (SSD keys, search window, selection incl. libstdc++ tie order), group
//     gather and scatter: PINNED -- checked against the reference's own include/Block.h compiled
//     unmodified (oracle/ref_block_shim.cpp, built into oracle/_ref/) and against committed
//     golden vectors generated from it (tests/golden/).
//   * the 3-D DCT: the reference calls FFTW3f r2r REDFT10/REDFT01 (source/BM3D.cpp:137-151),
//     which is absent here, so the transform is restated from FFTW's published definitions
//     (DCT-II: Y_k = 2 sum_j x_j cos(pi (j+1/2) k / N); DCT-III: Y_k = x_0 + 2 sum_{j>=1}
//     x_j cos(pi j (k+1/2) / N)) as a fixed FP32 factorisation (partial butterfly for power-of-
//     two lengths, direct FMA chains otherwise).  That part is UNPINNED against FFTW's last
//     bits; tests bound it against an FP64 evaluation of the definition.
//   * thresholds, Wiener shrinkage, weights, drivers, V-BM3D matching, VAggregate and the
//     colour conversions are restatements of the cited reference code.
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off; no fast-math, so every float op is IEEE).

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#if defined(__SSE2__)
#include <emmintrin.h>
#include <xmmintrin.h>
#endif

namespace orc {

// ---------------------------------------------------------------------------------------------
// Parameters (source/BM3D.cpp:33-130, source/VBM3D_Base.cpp:32-97)

struct Para {
    int wiener;
    int B, step, G, R, bmstep;
    double thMSE;
    double lambda;
    int radius, psnum, psrange, psstep;
};

// BM3D_Para::BM3D_Para, source/BM3D.cpp:33-107
static void bm3d_profile(int wiener, const std::string &profile, Para &p)
{
    p.wiener = wiener;
    p.B = 8;
    p.R = 16;
    p.bmstep = 1;
    p.lambda = 0.0;
    if (!wiener) { p.step = 4; p.G = 16; p.lambda = 2.7; }
    else { p.step = 3; p.G = 32; }
    if (profile == "fast") {
        p.R = 9; p.G = 8;
        p.step = wiener ? 7 : 8;
    } else if (profile == "lc") {
        p.R = 9;
        if (!wiener) p.step = 6;
        else { p.step = 5; p.G = 16; }
    } else if (profile == "high") {
        p.step = wiener ? 2 : 3;
    } else if (profile == "vn") {
        if (!wiener) { p.step = 4; p.G = 32; p.lambda = 2.8; }
        else { p.B = 11; p.step = 6; }
    }
    p.radius = 0; p.psnum = 0; p.psrange = 0; p.psstep = 0;
}

// VBM3D_Para::VBM3D_Para, source/VBM3D_Base.cpp:32-97 (called after the BM3D base defaults)
static void vbm3d_profile(int wiener, const std::string &profile, Para &p)
{
    bm3d_profile(wiener, profile, p);
    p.radius = 3; p.G = 8; p.R = 12; p.psnum = 2; p.psstep = 1;
    p.psrange = wiener ? 6 : 5;
    if (profile == "fast") { p.radius = 1; p.R = 7; p.psrange = wiener ? 5 : 4; }
    else if (profile == "lc") { p.radius = 2; p.R = 9; p.psrange = wiener ? 5 : 4; }
    else if (profile == "high") { p.radius = 4; p.R = 16; p.psrange = wiener ? 8 : 7; }
    else if (profile == "vn") { p.radius = 4; p.G = 16; }
}

// BM3D_Para::thMSE_Default, source/BM3D.cpp:110-130
static double thmse_default(int wiener, const std::string &profile, double sigma0)
{
    if (!wiener) return profile == "vn" ? 1000 + sigma0 * 150 : 400 + sigma0 * 80;
    return profile == "vn" ? 400 + sigma0 * 40 : 200 + sigma0 * 10;
}

// ---------------------------------------------------------------------------------------------
// Colour matrices (include/Specification.h:53-136 Kr/Kg/Kb, :139-213 RGB->YUV, :297-313 default)

enum { M_GBR = 0, M_BT709 = 1, M_UNSPEC = 2, M_FCC = 4, M_BT470BG = 5, M_SMPTE170M = 6,
       M_SMPTE240M = 7, M_YCGCO = 8, M_BT2020NC = 9, M_BT2020C = 10, M_OPP = 100 };

static void kr_kg_kb(int m, long double &Kr, long double &Kg, long double &Kb)
{
    switch (m) {
    case M_GBR: Kr = 0; Kg = 1; Kb = 0; break;
    case M_BT709: Kr = 0.2126; Kg = 0.7152; Kb = 0.0722; break;
    case M_FCC: Kr = 0.30; Kg = 0.59; Kb = 0.11; break;
    case M_BT470BG: case M_SMPTE170M: Kr = 0.299; Kg = 0.587; Kb = 0.114; break;
    case M_SMPTE240M: Kr = 0.212; Kg = 0.701; Kb = 0.087; break;
    case M_YCGCO: Kr = 0.25; Kg = 0.50; Kb = 0.25; break;
    case M_BT2020NC: case M_BT2020C: Kr = 0.2627; Kg = 0.6780; Kb = 0.0593; break;
    case M_OPP: Kr = 1. / 3.; Kg = 1. / 3.; Kb = 1. / 3.; break;
    default: Kr = 0.2126; Kg = 0.7152; Kb = 0.0722; break;
    }
}

// ColorMatrix_RGB2YUV_Parameter<double>: c = {Yr,Yg,Yb,Ur,Ug,Ub,Vr,Vg,Vb}
static void rgb2yuv_coef(int m, double c[9])
{
    if (m == M_GBR) {
        double v[9] = {0, 1, 0, 0, 0, 1, 1, 0, 0};
        std::memcpy(c, v, sizeof(v));
    } else if (m == M_YCGCO) {
        c[0] = (double)(1.0L / 4.0L); c[1] = (double)(1.0L / 2.0L); c[2] = (double)(1.0L / 4.0L);
        c[3] = (double)(-1.0L / 4.0L); c[4] = (double)(1.0L / 2.0L); c[5] = (double)(-1.0L / 4.0L);
        c[6] = (double)(1.0L / 2.0L); c[7] = 0.0; c[8] = (double)(-1.0L / 2.0L);
    } else if (m == M_OPP) {
        c[0] = (double)(1.0L / 3.0L); c[1] = (double)(1.0L / 3.0L); c[2] = (double)(1.0L / 3.0L);
        c[3] = (double)(1.0L / 2.0L); c[4] = 0.0; c[5] = (double)(-1.0L / 2.0L);
        c[6] = (double)(1.0L / 4.0L); c[7] = (double)(-1.0L / 2.0L); c[8] = (double)(1.0L / 4.0L);
    } else {
        long double Kr, Kg, Kb;
        kr_kg_kb(m, Kr, Kg, Kb);
        double Yr = (double)Kr, Yg = (double)Kg, Yb = (double)Kb;
        c[0] = Yr; c[1] = Yg; c[2] = Yb;
        c[3] = (double)(-Yr * 0.5L / (1.0L - Yb));
        c[4] = (double)(-Yg * 0.5L / (1.0L - Yb));
        c[5] = 0.5;
        c[6] = 0.5;
        c[7] = (double)(-Yg * 0.5L / (1.0L - Yr));
        c[8] = (double)(-Yb * 0.5L / (1.0L - Yr));
    }
}

static int matrix_default(int W, int H)
{
    if (W > 2048 || H > 1536) return M_BT2020NC;
    if (W > 1024 || H > 576) return M_BT709;
    return M_SMPTE170M;
}

// init_filter_data: source/BM3D_Base.cpp:262-283 (identical in source/VBM3D_Base.cpp:382-403)
static void matrix_norms(int m, double norm[3])
{
    double c[9];
    rgb2yuv_coef(m, c);
    norm[0] = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    norm[1] = std::sqrt(c[3] * c[3] + c[4] * c[4] + c[5] * c[5]);
    norm[2] = std::sqrt(c[6] * c[6] + c[7] * c[7] + c[8] * c[8]);
}

// ---------------------------------------------------------------------------------------------
// Per-plane filter data (BM3D_FilterData ctor, source/BM3D.cpp:137-209)

struct PlaneData {
    std::vector<double> finalAMP;             // [n-1]
    std::vector<std::vector<float>> thr;      // [n-1][n*B*B]
    std::vector<float> wsig2;                 // [n-1]
};

static PlaneData make_plane_data(int wiener, double sigma, int G, int B, double lambda)
{
    PlaneData d;
    d.finalAMP.resize(G);
    if (wiener) d.wsig2.resize(G); else d.thr.resize(G);
    for (int i = 1; i <= G; ++i) {
        d.finalAMP[i - 1] = 2 * i * 2 * B * 2 * B;
        double forwardAMP = std::sqrt(d.finalAMP[i - 1]);
        if (wiener) {
            float v = static_cast<float>(sigma * forwardAMP * sigma * forwardAMP);
            float mn = std::numeric_limits<float>::min();
            d.wsig2[i - 1] = v > mn ? v : mn;
        } else {
            double thrBase = sigma * lambda * forwardAMP;
            double t[4] = {thrBase, thrBase * std::sqrt(double(2)), thrBase * double(2),
                           thrBase * std::sqrt(double(8))};
            std::vector<float> &tab = d.thr[i - 1];
            tab.resize((size_t)i * B * B);
            size_t k = 0;
            for (int z = 0; z < i; ++z)
                for (int y = 0; y < B; ++y)
                    for (int x = 0; x < B; ++x) {
                        int flag = (x == 0) + (y == 0) + (z == 0);
                        tab[k++] = static_cast<float>(t[flag]);
                    }
        }
    }
    return d;
}

// ---------------------------------------------------------------------------------------------
// 3-D DCT (replaces FFTW r2r_3d REDFT10 / REDFT01; see header comment)

static bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// 2*cos(pi*a/b) rounded to float; the single formula shared by every table below
static float cos2(long a, long b)
{
    double ang = (double)a * M_PI / (double)b;
    return (float)(2.0 * std::cos(ang));
}

// Tables of length N, built once per N:
//   odd[m][j] = 2cos(pi(2j+1)(2m+1)/(2N))  (m, j < N/2; odd part of the partial butterfly)
//   fwd[k][j] = 2cos(pi(2j+1)k/(2N))       (direct DCT-II)
//   inv[k][j] = 2cos(pi j(2k+1)/(2N))      (direct DCT-III; j = 0 unused, DC enters with weight 1)
struct Tables {
    std::once_flag once;
    std::vector<float> odd, fwd, inv;
};
static Tables g_tables[513];

static const Tables &tables(int N)
{
    Tables &t = g_tables[N];
    std::call_once(t.once, [&t, N]() {
        int h = N / 2;
        t.odd.resize((size_t)h * h);
        for (int m = 0; m < h; ++m)
            for (int j = 0; j < h; ++j)
                t.odd[(size_t)m * h + j] = cos2((long)(2 * j + 1) * (2 * m + 1), 2L * N);
        t.fwd.resize((size_t)N * N);
        t.inv.resize((size_t)N * N);
        for (int k = 0; k < N; ++k)
            for (int j = 0; j < N; ++j) {
                t.fwd[(size_t)k * N + j] = cos2((long)(2 * j + 1) * k, 2L * N);
                t.inv[(size_t)k * N + j] = cos2((long)j * (2 * k + 1), 2L * N);
            }
    });
    return t;
}

static const float *odd_table(int N) { return tables(N).odd.data(); }
static const float *direct_table(int N, bool inverse) { return inverse ? tables(N).inv.data() : tables(N).fwd.data(); }

// Forward DCT-II (REDFT10) of length N (power of two), partial butterfly.
static void fdct_pow2(const float *x, int N, float *X)
{
    if (N == 1) { X[0] = x[0] * 2.0f; return; }
    const int h = N / 2;
    float e[256], o[256], E[256];
    for (int j = 0; j < h; ++j) {
        e[j] = x[j] + x[N - 1 - j];
        o[j] = x[j] - x[N - 1 - j];
    }
    fdct_pow2(e, h, E);
    const float *c = odd_table(N);
    for (int m = 0; m < h; ++m) {
        X[2 * m] = E[m];
        float acc = o[0] * c[(size_t)m * h];
        for (int j = 1; j < h; ++j) acc = std::fmaf(o[j], c[(size_t)m * h + j], acc);
        X[2 * m + 1] = acc;
    }
}

// Inverse DCT-III (REDFT01) of length N (power of two), partial butterfly.
static void idct_pow2(const float *X, int N, float *y)
{
    if (N == 1) { y[0] = X[0]; return; }
    const int h = N / 2;
    float ev[256], E[256];
    for (int m = 0; m < h; ++m) ev[m] = X[2 * m];
    idct_pow2(ev, h, E);
    const float *c = odd_table(N);
    for (int k = 0; k < h; ++k) {
        float acc = X[1] * c[(size_t)k * h];
        for (int m = 1; m < h; ++m) acc = std::fmaf(X[2 * m + 1], c[(size_t)k * h + m], acc);
        y[k] = E[k] + acc;
        y[N - 1 - k] = E[k] - acc;
    }
}

static void fdct_direct(const float *x, int N, float *X)
{
    const float *t = direct_table(N, false);
    for (int k = 0; k < N; ++k) {
        float acc = x[0] * t[(size_t)k * N];
        for (int j = 1; j < N; ++j) acc = std::fmaf(x[j], t[(size_t)k * N + j], acc);
        X[k] = acc;
    }
}

static void idct_direct(const float *X, int N, float *y)
{
    const float *t = direct_table(N, true);
    for (int k = 0; k < N; ++k) {
        float acc = X[0];
        for (int j = 1; j < N; ++j) acc = std::fmaf(X[j], t[(size_t)k * N + j], acc);
        y[k] = acc;
    }
}

static void dct1d(float *data, int N, ptrdiff_t stride, bool inverse)
{
    float in[256], out[256];
    for (int i = 0; i < N; ++i) in[i] = data[i * stride];
    if (is_pow2(N)) { if (inverse) idct_pow2(in, N, out); else fdct_pow2(in, N, out); }
    else { if (inverse) idct_direct(in, N, out); else fdct_direct(in, N, out); }
    for (int i = 0; i < N; ++i) data[i * stride] = out[i];
}

// Group layout: data[(z*B + y)*B + x] (BlockGroup, include/Block.h:1028-1029).
// Forward: x, then y, then z.  Inverse: z, then y, then x.  (Scalar form; dct3d below computes
// the same operation sequence on 8 columns at a time.)
static void dct3d_scalar(float *g, int n, int B, bool inverse)
{
    const ptrdiff_t plane = (ptrdiff_t)B * B;
    if (!inverse) {
        for (int z = 0; z < n; ++z)
            for (int y = 0; y < B; ++y) dct1d(g + z * plane + y * B, B, 1, false);
        for (int z = 0; z < n; ++z)
            for (int x = 0; x < B; ++x) dct1d(g + z * plane + x, B, B, false);
        for (int p = 0; p < plane; ++p) dct1d(g + p, n, plane, false);
    } else {
        for (int p = 0; p < plane; ++p) dct1d(g + p, n, plane, true);
        for (int z = 0; z < n; ++z)
            for (int x = 0; x < B; ++x) dct1d(g + z * plane + x, B, B, true);
        for (int z = 0; z < n; ++z)
            for (int y = 0; y < B; ++y) dct1d(g + z * plane + y * B, B, 1, true);
    }
}

// ---- the same transforms on VL independent columns at once -------------------------------------
// Arrays are [index][lane]; every lane performs exactly the scalar operation sequence above, so
// results are bit-identical (the lane loops only let the compiler use SIMD registers).
constexpr int VL = 8;

static void fdct_pow2_v(const float *x, int N, float *X)
{
    if (N == 1) {
        for (int l = 0; l < VL; ++l) X[l] = x[l] * 2.0f;
        return;
    }
    const int h = N / 2;
    alignas(32) float e[128 * VL], o[128 * VL], E[128 * VL];
    for (int j = 0; j < h; ++j)
        for (int l = 0; l < VL; ++l) {
            e[j * VL + l] = x[j * VL + l] + x[(N - 1 - j) * VL + l];
            o[j * VL + l] = x[j * VL + l] - x[(N - 1 - j) * VL + l];
        }
    fdct_pow2_v(e, h, E);
    const float *c = odd_table(N);
    for (int m = 0; m < h; ++m) {
        alignas(32) float acc[VL];
        const float c0 = c[(size_t)m * h];
        for (int l = 0; l < VL; ++l) {
            X[2 * m * VL + l] = E[m * VL + l];
            acc[l] = o[l] * c0;
        }
        for (int j = 1; j < h; ++j) {
            const float cj = c[(size_t)m * h + j];
            for (int l = 0; l < VL; ++l) acc[l] = std::fmaf(o[j * VL + l], cj, acc[l]);
        }
        for (int l = 0; l < VL; ++l) X[(2 * m + 1) * VL + l] = acc[l];
    }
}

static void idct_pow2_v(const float *X, int N, float *y)
{
    if (N == 1) {
        for (int l = 0; l < VL; ++l) y[l] = X[l];
        return;
    }
    const int h = N / 2;
    alignas(32) float ev[128 * VL], E[128 * VL];
    for (int m = 0; m < h; ++m)
        for (int l = 0; l < VL; ++l) ev[m * VL + l] = X[2 * m * VL + l];
    idct_pow2_v(ev, h, E);
    const float *c = odd_table(N);
    for (int k = 0; k < h; ++k) {
        alignas(32) float acc[VL];
        const float c0 = c[(size_t)k * h];
        for (int l = 0; l < VL; ++l) acc[l] = X[VL + l] * c0;
        for (int m = 1; m < h; ++m) {
            const float cm = c[(size_t)k * h + m];
            for (int l = 0; l < VL; ++l) acc[l] = std::fmaf(X[(2 * m + 1) * VL + l], cm, acc[l]);
        }
        for (int l = 0; l < VL; ++l) {
            y[k * VL + l] = E[k * VL + l] + acc[l];
            y[(N - 1 - k) * VL + l] = E[k * VL + l] - acc[l];
        }
    }
}

static void fdct_direct_v(const float *x, int N, float *X)
{
    const float *t = direct_table(N, false);
    for (int k = 0; k < N; ++k) {
        alignas(32) float acc[VL];
        const float t0 = t[(size_t)k * N];
        for (int l = 0; l < VL; ++l) acc[l] = x[l] * t0;
        for (int j = 1; j < N; ++j) {
            const float tj = t[(size_t)k * N + j];
            for (int l = 0; l < VL; ++l) acc[l] = std::fmaf(x[j * VL + l], tj, acc[l]);
        }
        for (int l = 0; l < VL; ++l) X[k * VL + l] = acc[l];
    }
}

static void idct_direct_v(const float *X, int N, float *y)
{
    const float *t = direct_table(N, true);
    for (int k = 0; k < N; ++k) {
        alignas(32) float acc[VL];
        for (int l = 0; l < VL; ++l) acc[l] = X[l];
        for (int j = 1; j < N; ++j) {
            const float tj = t[(size_t)k * N + j];
            for (int l = 0; l < VL; ++l) acc[l] = std::fmaf(X[j * VL + l], tj, acc[l]);
        }
        for (int l = 0; l < VL; ++l) y[k * VL + l] = acc[l];
    }
}

// Transforms `lanes` (<= VL) strided 1-D sequences of length N: element j of lane l at
// data[l * lstride + j * jstride].
static void dct1d_v(float *data, int N, ptrdiff_t jstride, ptrdiff_t lstride, int lanes, bool inverse)
{
    alignas(32) float in[256 * VL], out[256 * VL];
    for (int j = 0; j < N; ++j)
        for (int l = 0; l < VL; ++l) in[j * VL + l] = l < lanes ? data[l * lstride + j * jstride] : 0.0f;
    if (is_pow2(N)) { if (inverse) idct_pow2_v(in, N, out); else fdct_pow2_v(in, N, out); }
    else { if (inverse) idct_direct_v(in, N, out); else fdct_direct_v(in, N, out); }
    for (int j = 0; j < N; ++j)
        for (int l = 0; l < lanes; ++l) data[l * lstride + j * jstride] = out[j * VL + l];
}

static void dct3d(float *g, int n, int B, bool inverse)
{
    const ptrdiff_t plane = (ptrdiff_t)B * B;
    auto rows = [&](bool inv) {        // along x: lanes are rows y
        for (int z = 0; z < n; ++z)
            for (int y0 = 0; y0 < B; y0 += VL) dct1d_v(g + z * plane + y0 * B, B, 1, B, std::min(VL, B - y0), inv);
    };
    auto cols = [&](bool inv) {        // along y: lanes are columns x
        for (int z = 0; z < n; ++z)
            for (int x0 = 0; x0 < B; x0 += VL) dct1d_v(g + z * plane + x0, B, B, 1, std::min(VL, B - x0), inv);
    };
    auto zs = [&](bool inv) {          // along z: lanes are coefficient positions
        for (int p0 = 0; p0 < plane; p0 += VL) dct1d_v(g + p0, n, plane, 1, (int)std::min<ptrdiff_t>(VL, plane - p0), inv);
    };
    if (!inverse) { rows(false); cols(false); zs(false); }
    else { zs(true); cols(true); rows(true); }
}

// ---------------------------------------------------------------------------------------------
// Statistics for the parity reports (no reference counterpart; they only observe the arithmetic)

struct Stats {
    std::atomic<long long> groups{0};       // groups filtered (per plane)
    std::atomic<long long> coefs{0};        // hard-threshold decisions taken
    std::atomic<long long> flips{0};        // decisions that differ from the FP64 evaluation
    std::atomic<long long> band{0};         // |c| within a relative 2^-10 of its threshold
    std::atomic<long long> blocks{0};       // reference blocks matched
    std::atomic<long long> tie_blocks{0};   // blocks with equal keys inside the kept list or at its cut
};

// FP64 forward 3-D DCT of one group by the REDFT10 definition (Y_k = 2 sum_j x_j cos(pi (j+1/2)
// k / N)) along x, y, then z.  Used only to count threshold decisions that FP32 rounding flips.
static void dct3d_f64(std::vector<double> &g, int n, int B)
{
    const ptrdiff_t plane = (ptrdiff_t)B * B;
    static std::once_flag once[257];
    static std::vector<double> cosk[257];      // [k][j] = 2 cos(pi (j + 1/2) k / N)
    auto table = [](int N) -> const double * {
        std::call_once(once[N], [N]() {
            cosk[N].resize((size_t)N * N);
            for (int k = 0; k < N; ++k)
                for (int j = 0; j < N; ++j) cosk[N][(size_t)k * N + j] = 2.0 * std::cos(M_PI * (j + 0.5) * k / N);
        });
        return cosk[N].data();
    };
    auto line = [&](double *d, int N, ptrdiff_t stride) {
        const double *c = table(N);
        double in[256], out[256];
        for (int j = 0; j < N; ++j) in[j] = d[j * stride];
        for (int k = 0; k < N; ++k) {
            double acc = 0;
            for (int j = 0; j < N; ++j) acc += in[j] * c[(size_t)k * N + j];
            out[k] = acc;
        }
        for (int k = 0; k < N; ++k) d[k * stride] = out[k];
    };
    for (int z = 0; z < n; ++z)
        for (int y = 0; y < B; ++y) line(g.data() + z * plane + y * B, B, 1);
    for (int z = 0; z < n; ++z)
        for (int x = 0; x < B; ++x) line(g.data() + z * plane + x, B, B);
    for (ptrdiff_t q = 0; q < plane; ++q) line(g.data() + q, n, plane);
}

// Tie events of a selected list (include/Block.h:715-728): equal keys among the kept entries
// after the pinned first one, or between the last kept entry and the best one dropped.
static bool has_tie(const std::vector<float> &kept, float best_dropped, bool dropped_any, int first)
{
    for (size_t k = first; k + 1 < kept.size(); ++k)
        if (kept[k] == kept[k + 1]) return true;
    return dropped_any && !kept.empty() && kept.back() == best_dropped;
}

// ---------------------------------------------------------------------------------------------
// Block matching (include/Block.h:554-827)

struct Pos {
    int y, x;
    bool operator<(const Pos &r) const { return y < r.y || (y == r.y && x < r.x); }  // Type.h:216-234
    bool operator==(const Pos &r) const { return y == r.y && x == r.x; }
};

// KeyPair compares the key only (include/Type.h:406-473)
struct Match {
    float key;
    int z, y, x;
    bool operator<(const Match &r) const { return key < r.key; }
};

// SSD in the reference's evaluation order (include/Block.h:575-643): for the first
// B - B%8 columns four partial sums, lane l adding (r-s)^2 of column c+l then c+4+l for every
// 8-column chunk c of every row, combined as ((s0+s1)+s2)+s3; the remaining B%8 columns are
// added afterwards one by one, row by row.
static float ssd(const float *refblk, const float *src, ptrdiff_t stride, int B)
{
    const int residue = B % 8;
    const int simdw = B - residue;
    float dist = 0;
    if (simdw > 0) {
#if defined(__SSE2__)
        __m128 s = _mm_setzero_ps();
        for (int y = 0; y < B; ++y) {
            const float *r = refblk + y * B;
            const float *q = src + y * stride;
            for (int c = 0; c < simdw; c += 8) {
                __m128 d1 = _mm_sub_ps(_mm_loadu_ps(r + c), _mm_loadu_ps(q + c));
                __m128 d2 = _mm_sub_ps(_mm_loadu_ps(r + c + 4), _mm_loadu_ps(q + c + 4));
                s = _mm_add_ps(s, _mm_mul_ps(d1, d1));
                s = _mm_add_ps(s, _mm_mul_ps(d2, d2));
            }
        }
        alignas(16) float l[4];
        _mm_store_ps(l, s);
#else
        float l[4] = {0, 0, 0, 0};
        for (int y = 0; y < B; ++y) {
            const float *r = refblk + y * B;
            const float *q = src + y * stride;
            for (int c = 0; c < simdw; c += 8) {
                for (int k = 0; k < 4; ++k) { float d = r[c + k] - q[c + k]; l[k] = l[k] + d * d; }
                for (int k = 0; k < 4; ++k) { float d = r[c + 4 + k] - q[c + 4 + k]; l[k] = l[k] + d * d; }
            }
        }
#endif
        dist += l[0] + l[1] + l[2] + l[3];
    }
    if (residue > 0) {
        for (int y = 0; y < B; ++y) {
            const float *r = refblk + y * B + simdw;
            const float *q = src + y * stride + simdw;
            for (int c = 0; c < residue; ++c) { float d = r[c] - q[c]; dist += d * d; }
        }
    }
    return dist;
}

// Block::_SearchBoundary, include/Block.h:734-764
static int search_boundary(int pos, int plane_boundary, int range, int step)
{
    range = range / step * step;
    int b;
    if (pos == plane_boundary) b = plane_boundary;
    else if (pos > plane_boundary) { b = pos - range; while (b < plane_boundary) b += step; }
    else { b = pos + range; while (b > plane_boundary) b -= step; }
    return b;
}

struct BMConst {
    double distMul;
    float thSSE;
};

// include/Block.h:557-560 with src_range = 1
static BMConst bm_const(int B, double thMSE)
{
    double MSE2SSE = static_cast<double>(B * B) * 1.0f * 1.0f / double(255 * 255);
    BMConst c;
    c.distMul = double(1) / MSE2SSE;
    c.thSSE = static_cast<float>(thMSE * MSE2SSE);
    return c;
}

// BlockMatchingMulti core (include/Block.h:554-653): append matches over search positions
static void bm_core(std::vector<Match> &code, const float *refblk, int B, const float *src,
                    ptrdiff_t stride, const std::vector<Pos> &sp, const BMConst &k, int z)
{
    for (const Pos &p : sp) {
        float dist = ssd(refblk, src + (ptrdiff_t)p.y * stride + p.x, stride, B);
        if (dist <= k.thSSE && dist != 0)
            code.push_back(Match{static_cast<float>(dist * k.distMul), z, p.y, p.x});
    }
}

static void load_block(const float *plane, ptrdiff_t stride, int j, int i, int B, float *blk)
{
    for (int y = 0; y < B; ++y)
        for (int x = 0; x < B; ++x) blk[y * B + x] = plane[(ptrdiff_t)(j + y) * stride + i + x];
}

// Range form with excludeCurPos = 1 (include/Block.h:683-729): window in raster order minus
// self, self pinned first with key 0, partial_sort of the rest when the list exceeds match_size,
// stable_sort otherwise.
static std::vector<Match> bm_range(const float *plane, int H, int W, ptrdiff_t stride,
                                   int j, int i, int B, int range, int step, double thMSE,
                                   int match_size, int z = 0, bool *ties = nullptr)
{
    range = range / step * step;
    const int l = search_boundary(i, 0, range, step);
    const int r = search_boundary(i, W - B, range, step);
    const int t = search_boundary(j, 0, range, step);
    const int b = search_boundary(j, H - B, range, step);
    std::vector<Pos> sp;
    sp.reserve((size_t)((r - l) / step + 1) * ((b - t) / step + 1));
    for (int y = t; y <= b; y += step)
        for (int x = l; x <= r; x += step)
            if (!(y == j && x == i)) sp.push_back(Pos{y, x});
    // The reference sizes search_pos for the whole lattice (self included) and skips self while
    // filling it, so its last entry keeps the default Pos(0, 0) and is scanned as one more
    // candidate (include/Block.h:692-707).  Self always lies on the lattice.
    sp.push_back(Pos{0, 0});
    float blk[64 * 64];
    load_block(plane, stride, j, i, B, blk);
    std::vector<Match> code;
    code.reserve(sp.size() + 1);
    code.push_back(Match{0.0f, z, j, i});
    bm_core(code, blk, B, plane, stride, sp, bm_const(B, thMSE), z);
    if (match_size > 0 && code.size() > (size_t)match_size) {
        std::partial_sort(code.begin() + 1, code.begin() + match_size, code.end());
        if (ties) {
            float best = std::numeric_limits<float>::infinity();
            for (size_t k = match_size; k < code.size(); ++k) best = std::min(best, code[k].key);
            std::vector<float> kept;
            for (int k = 0; k < match_size; ++k) kept.push_back(code[k].key);
            *ties = has_tie(kept, best, true, 1);
        }
        code.resize(match_size);
    } else {
        std::stable_sort(code.begin(), code.end());
        if (ties) {
            std::vector<float> kept;
            for (const Match &m : code) kept.push_back(m.key);
            *ties = has_tie(kept, 0.0f, false, 1);
        }
    }
    return code;
}

// Search-position form (include/Block.h:655-677)
static std::vector<Match> bm_positions(const float *refblk, int B, const float *src,
                                       ptrdiff_t stride, const std::vector<Pos> &sp,
                                       double thMSE, int match_size, int z)
{
    std::vector<Match> code;
    code.reserve(sp.size());
    bm_core(code, refblk, B, src, stride, sp, bm_const(B, thMSE), z);
    if (match_size > 0 && code.size() > (size_t)match_size) {
        std::partial_sort(code.begin(), code.begin() + match_size, code.end());
        code.resize(match_size);
    } else {
        std::stable_sort(code.begin(), code.end());
    }
    return code;
}

// AddSearchPos / MergeSearchPos / GenSearchPos (include/Block.h:771-827)
static std::vector<Pos> gen_search_pos(const std::vector<Pos> &centers, int H, int W, int B,
                                       int range, int step)
{
    std::vector<Pos> sp;
    for (const Pos &c : centers) {
        int rr = range / step * step;
        const int l = search_boundary(c.x, 0, rr, step);
        const int r = search_boundary(c.x, W - B, rr, step);
        const int t = search_boundary(c.y, 0, rr, step);
        const int b = search_boundary(c.y, H - B, rr, step);
        std::vector<Pos> win;
        for (int y = t; y <= b; y += step)
            for (int x = l; x <= r; x += step) win.push_back(Pos{y, x});
        if (!sp.empty()) {
            std::vector<Pos> merged(sp.size() + win.size());
            std::merge(sp.begin(), sp.end(), win.begin(), win.end(), merged.begin());
            sp.swap(merged);
        } else {
            sp.swap(win);
        }
    }
    sp.erase(std::unique(sp.begin(), sp.end()), sp.end());
    return sp;
}

// ---------------------------------------------------------------------------------------------
// Collaborative filters (source/BM3D_Basic.cpp:72-148, source/BM3D_Final.cpp:50-127 and the
// identical V-BM3D versions) and the scatter (include/Block.h:1239-1387)

struct Accum {
    float *num;   // [frames][H*stride] addressing via z
    float *den;
    ptrdiff_t frame_pitch;   // elements between frame slots (0 for single-frame BM3D)
    ptrdiff_t stride;
};

static void scatter(const float *g, const std::vector<Match> &code, int n, int B,
                    const Accum &acc, float numW, float denW)
{
    for (int k = 0; k < n; ++k) {
        float *num = acc.num + code[k].z * acc.frame_pitch + (ptrdiff_t)code[k].y * acc.stride + code[k].x;
        float *den = acc.den + code[k].z * acc.frame_pitch + (ptrdiff_t)code[k].y * acc.stride + code[k].x;
        const float *s = g + (size_t)k * B * B;
        for (int y = 0; y < B; ++y)
            for (int x = 0; x < B; ++x) {
                num[y * acc.stride + x] += static_cast<float>(s[y * B + x] * numW);
                den[y * acc.stride + x] += denW;
            }
    }
}

static void gather(float *g, const std::vector<Match> &code, int n, int B,
                   const float *const *planes, ptrdiff_t stride)
{
    for (int k = 0; k < n; ++k) {
        const float *p = planes[code[k].z] + (ptrdiff_t)code[k].y * stride + code[k].x;
        for (int y = 0; y < B; ++y)
            for (int x = 0; x < B; ++x) g[(size_t)k * B * B + y * B + x] = p[y * stride + x];
    }
}

// Hard threshold of one group (source/BM3D_Basic.cpp:72-148) up to the scatter: gather, forward
// 3-D DCT, keep c iff |c| > thr, count the retained coefficients, inverse DCT.  The filtered
// group is left in g; numW / denW are the aggregation weights.  With st, the threshold decisions
// are also taken on an FP64 evaluation of the transform and the disagreements counted.
static int cf_basic_filter(const PlaneData &pd, int G, int B, const std::vector<Match> &code,
                           const float *const *src, ptrdiff_t stride, std::vector<float> &g,
                           float &numW, float &denW, Stats *st)
{
    int n = (int)code.size();
    if (G > 0 && n > G) n = G;
    const size_t sz = (size_t)n * B * B;
    g.resize(sz);
    gather(g.data(), code, n, B, src, stride);
    std::vector<double> g64;
    if (st) {
        g64.assign(g.begin(), g.end());
        dct3d_f64(g64, n, B);
    }
    dct3d(g.data(), n, B, false);
    const float *thr = pd.thr[n - 1].data();
    int retained = 0;
    long long flips = 0, band = 0;
    for (size_t q = 0; q < sz; ++q) {
        const bool keep = std::fabs(g[q]) > thr[q];
        if (st) {
            flips += keep != (std::fabs(g64[q]) > (double)thr[q]);
            band += std::fabs(std::fabs(g[q]) - thr[q]) <= thr[q] * (1.0f / 1024.0f);
        }
        if (keep) ++retained;
        else g[q] = 0.0f;
    }
    if (st) {
        st->groups += 1;
        st->coefs += (long long)sz;
        st->flips += flips;
        st->band += band;
    }
    dct3d(g.data(), n, B, true);
    denW = retained < 1 ? 1.0f : 1.0f / static_cast<float>(retained);
    numW = static_cast<float>(denW / pd.finalAMP[n - 1]);
    return n;
}

// wiener_mode 0: exact division with a sequential L2 sum (the reference's non-SSE build,
// source/BM3D_Final.cpp:106-112); 1: the x86 SSE build (source/BM3D_Final.cpp:78-104):
// four-lane L2 partial sums and an approximate reciprocal from _mm_rcp_ps.  rg is scratch.
static int cf_final_filter(const PlaneData &pd, int G, int B, const std::vector<Match> &code,
                           const float *const *src, const float *const *ref, ptrdiff_t stride,
                           std::vector<float> &gv, std::vector<float> &rgv, int wiener_mode,
                           float &numW, float &denW, Stats *st)
{
    int n = (int)code.size();
    if (G > 0 && n > G) n = G;
    const size_t sz = (size_t)n * B * B;
    gv.resize(sz);
    rgv.resize(sz);
    float *g = gv.data();
    float *rg = rgv.data();
    gather(g, code, n, B, src, stride);
    gather(rg, code, n, B, ref, stride);
    dct3d(g, n, B, false);
    dct3d(rg, n, B, false);
    if (st) st->groups += 1;
    const float sig2 = pd.wsig2[n - 1];
    float L2 = 0;
    size_t q = 0;
#if defined(__SSE2__)
    if (wiener_mode == 1) {
        const size_t simdw = sz - sz % 4;
        __m128 sg = _mm_set_ps1(sig2);
        __m128 l2 = _mm_setzero_ps();
        for (; q < simdw; q += 4) {
            __m128 s1 = _mm_loadu_ps(g + q);
            __m128 r1 = _mm_loadu_ps(rg + q);
            __m128 r2 = _mm_mul_ps(r1, r1);
            __m128 w = _mm_mul_ps(r2, _mm_rcp_ps(_mm_add_ps(r2, sg)));
            _mm_storeu_ps(g + q, _mm_mul_ps(s1, w));
            l2 = _mm_add_ps(l2, _mm_mul_ps(w, w));
        }
        alignas(16) float l[4];
        _mm_store_ps(l, l2);
        L2 += l[0] + l[1] + l[2] + l[3];
    }
#endif
    for (; q < sz; ++q) {
        const float r2 = rg[q] * rg[q];
        const float w = r2 / (r2 + sig2);
        g[q] *= w;
        L2 += w * w;
    }
    dct3d(g, n, B, true);
    const float eps = std::numeric_limits<float>::epsilon();
    L2 = L2 > eps ? L2 : eps;
    denW = 1.0f / L2;
    numW = static_cast<float>(denW / pd.finalAMP[n - 1]);
    return n;
}

// Runs f(i, worker) for i in [0, n) on `workers` threads (the caller's thread is worker 0).
template <class F>
static void parallel_for(int n, int workers, F &&f)
{
    if (workers <= 1 || n < 2) {
        for (int i = 0; i < n; ++i) f(i, 0);
        return;
    }
    std::atomic<int> next(0);
    auto run = [&](int w) {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n) break;
            f(i, w);
        }
    };
    std::vector<std::thread> th;
    for (int w = 1; w < workers; ++w) th.emplace_back(run, w);
    run(0);
    for (auto &t : th) t.join();
}

// ---------------------------------------------------------------------------------------------
// Drivers

struct Job {
    Para p;
    int wiener_mode;
    int process[3];
    PlaneData pd[3];
};

static void scan_positions(int extent, int B, int step, std::vector<int> &out)
{
    // BM3D_Process_Base::Kernel ref-block scan with clamping, source/BM3D_Base.cpp:421-443
    out.clear();
    const int last = extent - B;
    for (int j = 0;; j += step) {
        if (j >= last + step) break;
        if (j > last) j = last;
        out.push_back(j);
    }
}

// BlockMatching wrapper (source/BM3D_Base.cpp:473-490)
static std::vector<Match> bm3d_match(const Para &p, const float *refY, int H, int W,
                                     ptrdiff_t stride, int j, int i, Stats *st = nullptr)
{
    if (p.G == 1 || p.thMSE <= 0) return std::vector<Match>(1, Match{0.0f, 0, j, i});
    bool ties = false;
    std::vector<Match> code = bm_range(refY, H, W, stride, j, i, p.B, p.R, p.bmstep, p.thMSE, p.G, 0,
                                       st ? &ties : nullptr);
    if (st) {
        st->blocks += 1;
        st->tie_blocks += ties;
    }
    return code;
}

// One reference block's filtered groups for every processed plane, ready to scatter.
struct BlockOut {
    std::vector<Match> code;
    int n = 0;
    float numW[3], denW[3];
    std::vector<float> g[3];
};

// Block matching and collaborative filtering of the reference blocks at (js[r], is[c]) for rows
// r of a band, computed on `workers` threads, then scattered one block at a time in the scan
// order of BM3D_Process_Base::Kernel (source/BM3D_Base.cpp:290-470), so the sums are the
// reference's sequential ones whatever the number of workers.  match(j, i) gives the list,
// planes(c, src, ref, stride) the planes of component c and acc_of(c) its accumulators.
template <class Match_, class Planes, class AccOf>
static void filter_blocks(const Job &job, const std::vector<int> &js, const std::vector<int> &is,
                          int workers, Match_ &&match, Planes &&planes, AccOf &&acc_of, Stats *st)
{
    const Para &p = job.p;
    std::vector<std::vector<float>> scratch(std::max(1, workers));
    auto compute = [&](BlockOut &o, int j, int i, int w) {
        o.code = match(j, i);
        for (int c = 0; c < 3; ++c) {
            if (!job.process[c]) continue;
            const float *const *s1;
            const float *const *r1;
            ptrdiff_t stride;
            planes(c, s1, r1, stride);
            if (!p.wiener) o.n = cf_basic_filter(job.pd[c], p.G, p.B, o.code, s1, stride, o.g[c], o.numW[c], o.denW[c], st);
            else o.n = cf_final_filter(job.pd[c], p.G, p.B, o.code, s1, r1, stride, o.g[c], scratch[w], job.wiener_mode, o.numW[c], o.denW[c], st);
        }
    };
    auto put = [&](const BlockOut &o) {
        for (int c = 0; c < 3; ++c)
            if (job.process[c]) scatter(o.g[c].data(), o.code, o.n, p.B, acc_of(c), o.numW[c], o.denW[c]);
    };
    if (workers <= 1) {
        BlockOut o;
        for (int j : js)
            for (int i : is) {
                compute(o, j, i, 0);
                put(o);
            }
        return;
    }
    const size_t band_rows = 4;
    std::vector<BlockOut> out;
    for (size_t r0 = 0; r0 < js.size(); r0 += band_rows) {
        const size_t r1 = std::min(js.size(), r0 + band_rows);
        const int nb = (int)((r1 - r0) * is.size());
        out.resize(nb);
        parallel_for(nb, workers, [&](int b, int w) { compute(out[b], js[r0 + b / is.size()], is[b % is.size()], w); });
        for (int b = 0; b < nb; ++b) put(out[b]);
    }
}

// BM3D_Process_Base::Kernel (source/BM3D_Base.cpp:290-470) on float planes.  dst planes are
// used as the numerator accumulators (ResNum aliases dst in the reference).
static void bm3d_frame(const Job &job, int H, int W, ptrdiff_t stride, const float *const src[3],
                       const float *const ref[3], float *const dst[3], int workers = 1, Stats *st = nullptr)
{
    const Para &p = job.p;
    std::vector<float> den[3];
    for (int c = 0; c < 3; ++c)
        if (job.process[c]) {
            den[c].assign((size_t)H * stride, 0.0f);
            std::memset(dst[c], 0, sizeof(float) * (size_t)H * stride);
        }
    std::vector<int> js, is;
    scan_positions(H, p.B, p.step, js);
    scan_positions(W, p.B, p.step, is);
    const float *s1[3][1] = {{src[0]}, {src[1]}, {src[2]}};
    const float *r1[3][1] = {{ref[0]}, {ref[1]}, {ref[2]}};
    filter_blocks(job, js, is, workers,
                  [&](int j, int i) { return bm3d_match(p, ref[0], H, W, stride, j, i, st); },
                  [&](int c, const float *const *&s, const float *const *&r, ptrdiff_t &ld) { s = s1[c]; r = r1[c]; ld = stride; },
                  [&](int c) { return Accum{dst[c], den[c].data(), 0, stride}; }, st);
    for (int c = 0; c < 3; ++c) {
        if (!job.process[c]) continue;
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                size_t q = (size_t)y * stride + x;
                dst[c][q] = dst[c][q] / den[c][q];
            }
    }
}

// VBM3D_Process_Base::BlockMatching (source/VBM3D_Base.cpp:540-659).  refs[f] is frame f of
// the window, cur the index of the current frame in it.
static std::vector<Match> vbm3d_match(const Para &p, const float *const *refs, int frames, int cur,
                                      int H, int W, ptrdiff_t stride, int j, int i, Stats *st = nullptr)
{
    if (p.G == 1 || p.thMSE <= 0) return std::vector<Match>(1, Match{0.0f, cur, j, i});
    std::vector<Match> code = bm_range(refs[cur], H, W, stride, j, i, p.B, p.R, p.bmstep,
                                       p.thMSE, p.G, cur);
    float blk[64 * 64];
    load_block(refs[cur], stride, j, i, p.B, blk);
    int nextnum = std::min(p.psnum, (int)code.size());
    std::vector<Pos> centers;
    for (int k = 0; k < nextnum; ++k) centers.push_back(Pos{code[k].y, code[k].x});
    const std::vector<Pos> cur_sp = gen_search_pos(centers, H, W, p.B, p.psrange, p.psstep);
    std::vector<Match> all = code;
    for (int dir = -1; dir <= 1; dir += 2) {
        std::vector<Match> fm;
        for (int f = cur + dir; f >= 0 && f < frames; f += dir) {
            if (f == cur + dir) {
                fm = bm_positions(blk, p.B, refs[f], stride, cur_sp, p.thMSE, p.G, f);
            } else {
                int nn = std::min(p.psnum, (int)fm.size());
                std::vector<Pos> pc;
                for (int k = 0; k < nn; ++k) pc.push_back(Pos{fm[k].y, fm[k].x});
                std::vector<Pos> sp = gen_search_pos(pc, H, W, p.B, p.psrange, p.psstep);
                fm = bm_positions(blk, p.B, refs[f], stride, sp, p.thMSE, p.G, f);
            }
            all.insert(all.end(), fm.begin(), fm.end());
        }
    }
    bool ties = false;
    if (p.G > 0 && (int)all.size() > p.G) {
        std::partial_sort(all.begin() + 1, all.begin() + p.G, all.end());
        if (st) {
            float best = std::numeric_limits<float>::infinity();
            for (size_t k = p.G; k < all.size(); ++k) best = std::min(best, all[k].key);
            std::vector<float> kept;
            for (int k = 0; k < p.G; ++k) kept.push_back(all[k].key);
            ties = has_tie(kept, best, true, 1);
        }
        all.resize(p.G);
    } else if (st) {
        std::vector<float> kept;
        for (const Match &m : all) kept.push_back(m.key);
        ties = has_tie(kept, 0.0f, false, 1);
    }
    if (st) {
        st->blocks += 1;
        st->tie_blocks += ties;
    }
    return all;
}

// VBM3D_Process_Base::Kernel (source/VBM3D_Base.cpp:410-537).  dst holds, per plane, the
// (2r+1)*2 stacked slots of height H: slot 2(r+b+f) = numerator, +1 = denominator for window
// frame f (source/VBM3D_Base.cpp:697-720).
static void vbm3d_frame(const Job &job, int H, int W, ptrdiff_t stride, int frames, int cur,
                        int b_offset, const float *const *src[3], const float *const *ref[3],
                        float *const dst[3], int workers = 1, Stats *st = nullptr)
{
    const Para &p = job.p;
    const ptrdiff_t pc = (ptrdiff_t)H * stride;
    for (int c = 0; c < 3; ++c)
        if (job.process[c])
            std::memset(dst[c], 0, sizeof(float) * (size_t)pc * (2 * p.radius + 1) * 2);
    std::vector<int> js, is;
    scan_positions(H, p.B, p.step, js);
    scan_positions(W, p.B, p.step, is);
    filter_blocks(job, js, is, workers,
                  [&](int j, int i) { return vbm3d_match(p, ref[0], frames, cur, H, W, stride, j, i, st); },
                  [&](int c, const float *const *&s, const float *const *&r, ptrdiff_t &ld) { s = src[c]; r = ref[c]; ld = stride; },
                  [&](int c) {
                      float *base = dst[c] + pc * 2 * (p.radius + b_offset);
                      return Accum{base, base + pc, 2 * pc, stride};
                  }, st);
}

} // namespace orc

// =============================================================================================
// C interface (ctypes)

using namespace orc;

extern "C" {

struct oracle_params {
    int wiener;            // 0 = Basic/VBasic, 1 = Final/VFinal
    int B, step, G, R, bmstep;
    double th_mse;         // as given by the user (before the matrix normalisation)
    double lambda;         // hard_thr
    double sigma[3];
    int matrix;            // resolved matrix id (never 2)
    int process[3];
    int radius, psnum, psrange, psstep;
    int wiener_mode;       // 0 exact (non-SSE build), 1 rcpps (x86 SSE build)
};

// Profile defaults (A1).  vbm3d selects the V-BM3D variant.
int oracle_default_params(int wiener, int vbm3d, const char *profile, double sigma0,
                          oracle_params *out)
{
    Para p;
    std::string prof = profile ? profile : "fast";
    if (vbm3d) vbm3d_profile(wiener, prof, p); else bm3d_profile(wiener, prof, p);
    out->wiener = wiener;
    out->B = p.B; out->step = p.step; out->G = p.G; out->R = p.R; out->bmstep = p.bmstep;
    out->lambda = p.lambda;
    out->th_mse = thmse_default(wiener, prof, sigma0);
    out->radius = p.radius; out->psnum = p.psnum; out->psrange = p.psrange; out->psstep = p.psstep;
    return 0;
}

int oracle_matrix_default(int W, int H) { return matrix_default(W, H); }

void oracle_matrix_norms(int matrix, double *norm3) { matrix_norms(matrix, norm3); }

static Job make_job(const oracle_params *a)
{
    Job job;
    job.p.wiener = a->wiener;
    job.p.B = a->B; job.p.step = a->step; job.p.G = a->G; job.p.R = a->R; job.p.bmstep = a->bmstep;
    job.p.lambda = a->lambda;
    job.p.radius = a->radius; job.p.psnum = a->psnum; job.p.psrange = a->psrange; job.p.psstep = a->psstep;
    job.wiener_mode = a->wiener_mode;
    double norm[3];
    matrix_norms(a->matrix, norm);
    job.p.thMSE = a->th_mse * norm[0];
    for (int c = 0; c < 3; ++c) {
        job.process[c] = a->process[c];
        if (a->process[c])
            job.pd[c] = make_plane_data(a->wiener, a->sigma[c] / double(255) * norm[c], a->G, a->B, a->lambda);
    }
    return job;
}

// Filter tables for one plane (A4): thr[G][G*B*B] (Basic) or wsig2[G] (Final), finalAMP[G]
void oracle_filter_tables(int wiener, double sigma_norm, int G, int B, double lambda,
                          double *finalAMP, float *thr, float *wsig2)
{
    PlaneData d = make_plane_data(wiener, sigma_norm, G, B, lambda);
    for (int i = 0; i < G; ++i) {
        finalAMP[i] = d.finalAMP[i];
        if (wiener) wsig2[i] = d.wsig2[i];
        else if (thr) std::memcpy(thr + (size_t)i * G * B * B, d.thr[i].data(), sizeof(float) * (i + 1) * B * B);
    }
}

// Statistics out: [0] groups filtered (per plane), [1] hard-threshold decisions, [2] decisions
// that differ from an FP64 evaluation of the transform (Basic), [3] coefficients within a
// relative 2^-10 of their threshold, [4] reference blocks matched, [5] blocks with tie events.
static void put_stats(const Stats &st, long long *out)
{
    if (!out) return;
    out[0] = st.groups; out[1] = st.coefs; out[2] = st.flips; out[3] = st.band;
    out[4] = st.blocks; out[5] = st.tie_blocks;
}

// Splits `threads` into frame workers (one frame each, as VapourSynth's fmParallel runs frames)
// and, when there are fewer frames than threads, workers inside each frame.
static void split_threads(int threads, int nframes, int &frame_workers, int &intra)
{
    if (threads < 1) threads = 1;
    frame_workers = std::max(1, std::min(threads, nframes));
    intra = std::max(1, threads / frame_workers);
}

// BM3D over a batch of frames of float planes.  Layout [frame][plane][H][stride]; planes that
// are not processed are copied through.  Frames run in parallel on `threads` host threads (one
// frame per thread, as VapourSynth's fmParallel does); with fewer frames than threads, each frame
// also splits its reference blocks over the spare threads (the aggregation stays sequential).
// stats: null, or 6 counters (put_stats), which add an FP64 transform per group.
int oracle_bm3d_ex(const oracle_params *a, int nframes, int nplanes, int H, int W, int stride,
                   const float *src, const float *ref, float *dst, int threads, long long *stats)
{
    Job job = make_job(a);
    if (nplanes == 1) { job.process[1] = job.process[2] = 0; }
    const size_t pc = (size_t)H * stride;
    Stats st;
    Stats *stp = stats ? &st : nullptr;
    int fw, intra;
    split_threads(threads, nframes, fw, intra);
    std::atomic<int> next(0);
    auto work = [&]() {
        for (;;) {
            int f = next.fetch_add(1);
            if (f >= nframes) break;
            const float *s[3], *r[3];
            float *d[3];
            for (int c = 0; c < 3; ++c) {
                int cc = c < nplanes ? c : 0;
                s[c] = src + ((size_t)f * nplanes + cc) * pc;
                r[c] = ref + ((size_t)f * nplanes + cc) * pc;
                d[c] = dst + ((size_t)f * nplanes + cc) * pc;
            }
            for (int c = 0; c < nplanes; ++c)
                if (!job.process[c]) std::memcpy(d[c], s[c], sizeof(float) * pc);
            bm3d_frame(job, H, W, stride, s, r, d, intra, stp);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < fw; ++t) th.emplace_back(work);
    work();
    for (auto &t : th) t.join();
    put_stats(st, stats);
    return 0;
}

int oracle_bm3d(const oracle_params *a, int nframes, int nplanes, int H, int W, int stride,
                const float *src, const float *ref, float *dst, int threads)
{
    return oracle_bm3d_ex(a, nframes, nplanes, H, W, stride, src, ref, dst, threads, nullptr);
}

// Match lists of every reference block of one frame (debug/parity).  Row-major over the
// ref-block scan; per block: count, then G entries (key, y, x).  Blocks are matched on `threads`
// host threads; stats (null or 6 counters) receives [4] blocks and [5] blocks with tie events.
int oracle_bm3d_matches_ex(const oracle_params *a, int H, int W, int stride, const float *refY,
                           int *counts, int *ys, int *xs, float *keys, int threads, long long *stats)
{
    Job job = make_job(a);
    std::vector<int> js, is;
    scan_positions(H, job.p.B, job.p.step, js);
    scan_positions(W, job.p.B, job.p.step, is);
    Stats st;
    const int nb = (int)(js.size() * is.size());
    parallel_for(nb, std::max(1, threads), [&](int b, int) {
        const int j = js[b / is.size()], i = is[b % is.size()];
        std::vector<Match> code = bm3d_match(job.p, refY, H, W, stride, j, i, stats ? &st : nullptr);
        counts[b] = (int)code.size();
        for (size_t k = 0; k < code.size(); ++k) {
            ys[(size_t)b * job.p.G + k] = code[k].y;
            xs[(size_t)b * job.p.G + k] = code[k].x;
            keys[(size_t)b * job.p.G + k] = code[k].key;
        }
    });
    put_stats(st, stats);
    return nb;
}

int oracle_bm3d_matches(const oracle_params *a, int H, int W, int stride, const float *refY,
                        int *counts, int *ys, int *xs, float *keys)
{
    return oracle_bm3d_matches_ex(a, H, W, stride, refY, counts, ys, xs, keys, 1, nullptr);
}

// V-BM3D match lists for one output frame n (debug/parity); entries carry the window frame z.
int oracle_vbm3d_matches_ex(const oracle_params *a, int nframes_total, int n, int H, int W, int stride,
                            const float *refY_clip /*[F][H][stride]*/, int *counts, int *zs, int *ys,
                            int *xs, float *keys, int threads, long long *stats)
{
    Job job = make_job(a);
    const int r = job.p.radius;
    const int b_off = -std::min(n, r);
    const int f_off = std::min(nframes_total - 1 - n, r);
    const int frames = f_off - b_off + 1;
    const int cur = -b_off;
    std::vector<const float *> refs(frames);
    for (int f = 0; f < frames; ++f) refs[f] = refY_clip + (size_t)(n + b_off + f) * H * stride;
    std::vector<int> js, is;
    scan_positions(H, job.p.B, job.p.step, js);
    scan_positions(W, job.p.B, job.p.step, is);
    Stats st;
    const int nb = (int)(js.size() * is.size());
    parallel_for(nb, std::max(1, threads), [&](int b, int) {
        const int j = js[b / is.size()], i = is[b % is.size()];
        std::vector<Match> code = vbm3d_match(job.p, refs.data(), frames, cur, H, W, stride, j, i, stats ? &st : nullptr);
        counts[b] = (int)code.size();
        for (size_t k = 0; k < code.size(); ++k) {
            zs[(size_t)b * job.p.G + k] = code[k].z;
            ys[(size_t)b * job.p.G + k] = code[k].y;
            xs[(size_t)b * job.p.G + k] = code[k].x;
            keys[(size_t)b * job.p.G + k] = code[k].key;
        }
    });
    put_stats(st, stats);
    return nb;
}

int oracle_vbm3d_matches(const oracle_params *a, int nframes_total, int n, int H, int W, int stride,
                         const float *refY_clip, int *counts, int *zs, int *ys, int *xs, float *keys)
{
    return oracle_vbm3d_matches_ex(a, nframes_total, n, H, W, stride, refY_clip, counts, zs, ys, xs, keys, 1, nullptr);
}

// V-BM3D for output frames [n0, n0+count) of a clip of nframes_total float frames.
// src/ref clip layout [F][plane][H][stride]; dst layout [count][plane][(2r+1)*2][H][stride].
// threads and stats as in oracle_bm3d_ex.
int oracle_vbm3d_ex(const oracle_params *a, int nframes_total, int n0, int count, int nplanes,
                    int H, int W, int stride, const float *src, const float *ref, float *dst,
                    int threads, long long *stats)
{
    Job job = make_job(a);
    Stats st;
    Stats *stp = stats ? &st : nullptr;
    int fw, intra;
    split_threads(threads, count, fw, intra);
    if (nplanes == 1) { job.process[1] = job.process[2] = 0; }
    const size_t pc = (size_t)H * stride;
    const int r = job.p.radius;
    const size_t slots = (size_t)(2 * r + 1) * 2;
    std::atomic<int> next(0);
    auto work = [&]() {
        for (;;) {
            int k = next.fetch_add(1);
            if (k >= count) break;
            int n = n0 + k;
            const int b_off = -std::min(n, r);
            const int f_off = std::min(nframes_total - 1 - n, r);
            const int frames = f_off - b_off + 1;
            const int cur = -b_off;
            std::vector<const float *> sv[3], rv[3];
            for (int c = 0; c < 3; ++c) {
                int cc = c < nplanes ? c : 0;
                for (int f = 0; f < frames; ++f) {
                    sv[c].push_back(src + ((size_t)(n + b_off + f) * nplanes + cc) * pc);
                    rv[c].push_back(ref + ((size_t)(n + b_off + f) * nplanes + cc) * pc);
                }
            }
            const float *const *s3[3] = {sv[0].data(), sv[1].data(), sv[2].data()};
            const float *const *r3[3] = {rv[0].data(), rv[1].data(), rv[2].data()};
            float *d3[3];
            for (int c = 0; c < 3; ++c) {
                int cc = c < nplanes ? c : 0;
                d3[c] = dst + ((size_t)k * nplanes + cc) * slots * pc;
            }
            vbm3d_frame(job, H, W, stride, frames, cur, b_off, s3, r3, d3, intra, stp);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < fw; ++t) th.emplace_back(work);
    work();
    for (auto &t : th) t.join();
    put_stats(st, stats);
    return 0;
}

int oracle_vbm3d(const oracle_params *a, int nframes_total, int n0, int count, int nplanes,
                 int H, int W, int stride, const float *src, const float *ref, float *dst,
                 int threads)
{
    return oracle_vbm3d_ex(a, nframes_total, n0, count, nplanes, H, W, stride, src, ref, dst, threads, nullptr);
}

// VAggregate_Process::Kernel (source/VAggregate.cpp:93-160) for output frame n.
// stacked layout [F][plane][(2r+1)*2][H][stride]; dst [plane][H][stride] float.
int oracle_vaggregate(int radius, int nframes_total, int n, int nplanes, const int *process,
                      int H, int W, int stride, const float *stacked, float *dst)
{
    const size_t pc = (size_t)H * stride;
    const size_t slots = (size_t)(2 * radius + 1) * 2;
    const int b_off = -std::min(n, radius);
    const int f_off = std::min(nframes_total - 1 - n, radius);
    const int frames = f_off - b_off + 1;
    for (int c = 0; c < nplanes; ++c) {
        if (!process[c]) continue;
        std::vector<const float *> num(frames), den(frames);
        for (int i = 0, o = radius - b_off; i < frames; ++i, --o) {
            const float *base = stacked + ((size_t)(n + b_off + i) * nplanes + c) * slots * pc;
            num[i] = base + pc * (o * 2);
            den[i] = base + pc * (o * 2 + 1);
        }
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                size_t q = (size_t)y * stride + x;
                float nm = 0, dn = 0;
                for (int f = 0; f < frames; ++f) { nm += num[f][q]; dn += den[f][q]; }
                dst[c * pc + q] = nm / dn;
            }
    }
    return 0;
}

// 3-D transform of one group in place (debug/parity of the DCT factorisation).
void oracle_dct3d(float *g, int n, int B, int inverse) { dct3d(g, n, B, inverse != 0); }
void oracle_dct3d_scalar(float *g, int n, int B, int inverse) { dct3d_scalar(g, n, B, inverse != 0); }

// Raw tables (debug/parity): odd-part matrix of length N (h*h) and direct tables (N*N).
void oracle_dct_tables(int N, float *odd, float *fwd, float *inv)
{
    if (odd && is_pow2(N) && N >= 2) std::memcpy(odd, odd_table(N), sizeof(float) * (N / 2) * (N / 2));
    if (fwd) std::memcpy(fwd, direct_table(N, false), sizeof(float) * N * N);
    if (inv) std::memcpy(inv, direct_table(N, true), sizeof(float) * N * N);
}

// ---------------------------------------------------------------------------------------------
// Conversions (include/Conversion.hpp:36-417, include/Helper.h:285-351)

// Quantisation parameters for integer samples (GetQuanPara, include/Helper.h:301-336)
static void quan_int(int bps, int full, int chroma, int &fl, int &ne, int &ce)
{
    if (full) { fl = 0; ne = chroma ? (1 << (bps - 1)) : fl; ce = (1 << bps) - 1; }
    else { fl = 16 << (bps - 8); ne = chroma ? (1 << (bps - 1)) : fl; ce = chroma ? 240 << (bps - 8) : 235 << (bps - 8); }
}

static float clipf(float v, float lo, float hi) { return v <= lo ? lo : v >= hi ? hi : v; }

// Int2Float (Conversion.hpp:424-437 -> RangeConvert :36-78) for a plane of uint8/uint16
void oracle_int2float(const void *src, int bytes, int bps, int full, int chroma, int H, int W,
                      int src_stride, int dst_stride, float *dst)
{
    int sf, sn, sc;
    quan_int(bps, full, chroma, sf, sn, sc);
    const float df = chroma ? -0.5f : 0.0f, dn = 0.0f, dc = chroma ? 0.5f : 1.0f;
    const int srange = sc - sf;
    const float drange = dc - df;
    const bool src_pc_chroma = sf < sn && (sf + sc) % 2 == 1;
    const bool clip = src_pc_chroma;
    const float gain = drange / srange;
    const float offset = -static_cast<float>(sn) * gain + dn;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            float v = bytes == 1 ? (float)((const uint8_t *)src)[(size_t)y * src_stride + x]
                                 : (float)((const uint16_t *)src)[(size_t)y * src_stride + x];
            float t = v * gain + offset;
            dst[(size_t)y * dst_stride + x] = clip ? clipf(t, df, dc) : t;
        }
}

// Float2Int (Conversion.hpp:439-452 -> RangeConvert with clip=true)
void oracle_float2int(const float *src, int bytes, int bps, int full, int chroma, int H, int W,
                      int src_stride, int dst_stride, void *dst)
{
    int df, dn, dc;
    quan_int(bps, full, chroma, df, dn, dc);
    const float sf = chroma ? -0.5f : 0.0f, sn = 0.0f, sc = chroma ? 0.5f : 1.0f;
    const float srange = sc - sf;
    const int drange = dc - df;
    const bool dst_pc_chroma = df < dn && (df + dc) % 2 == 1;
    const float gain = static_cast<float>(drange) / srange;
    float offset = -sn * gain + dn;
    offset += dst_pc_chroma ? 0.499999f : 0.5f;
    const float lo = (float)df, hi = (float)dc;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            float t = clipf(src[(size_t)y * src_stride + x] * gain + offset, lo, hi);
            if (bytes == 1) ((uint8_t *)dst)[(size_t)y * dst_stride + x] = (uint8_t)t;
            else ((uint16_t *)dst)[(size_t)y * dst_stride + x] = (uint16_t)t;
        }
}

// MatrixConvert_RGB2YUV OPP branch (Conversion.hpp:205-236) float->float, full range, no clip
void oracle_rgb2opp_float(const float *R, const float *Gp, const float *Bp, int H, int W, int stride,
                          float *Y, float *U, float *V)
{
    const float sRange = 1.0f - 0.0f;
    const float gainY = (1.0f - 0.0f) / (sRange * 3.0f);
    const float offsetY = -0.0f * 3.0f * gainY + 0.0f;
    const float gainU = (0.5f - -0.5f) / (sRange * 2.0f);
    const float gainV = (0.5f - -0.5f) / (sRange * 4.0f);
    const float offsetC = 0.0f;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            size_t q = (size_t)y * stride + x;
            float r = R[q], g = Gp[q], b = Bp[q];
            Y[q] = (r + g + b) * gainY + offsetY;
            U[q] = (r - b) * gainU + offsetC;
            V[q] = (r - g * 2.0f + b) * gainV + offsetC;
        }
}

// MatrixConvert_YUV2RGB OPP branch (Conversion.hpp:369-392, coefficients
// Specification.h:253-269) float->float, full range, no clip
void oracle_opp2rgb_float(const float *Y, const float *U, const float *V, int H, int W, int stride,
                          float *R, float *Gp, float *Bp)
{
    const float Ry = (float)1.0L, Ru = (float)1.0L, Rv = (float)(2.0L / 3.0L);
    const float Gy = (float)1.0L, Gv = (float)(-4.0L / 3.0L);
    const float By = (float)1.0L, Bu = (float)-1.0L, Bv = (float)(2.0L / 3.0L);
    const float Gu = 0.0f;
    const float offR = -0.0f * Ry - 0.0f * (Ru + Rv) + 0.0f;
    const float offG = -0.0f * Gy - 0.0f * (Gu + Gv) + 0.0f;
    const float offB = -0.0f * By - 0.0f * (Bu + Bv) + 0.0f;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            size_t q = (size_t)y * stride + x;
            float yy = Y[q], u = U[q], v = V[q];
            R[q] = Ry * yy + Ru * u + Rv * v + offR;
            Gp[q] = Gy * yy + Gv * v + offG;
            Bp[q] = By * yy + Bu * u + Bv * v + offB;
        }
}


// Samples of 1 (uint8), 2 (uint16) or 4 (float) bytes.
static float load_sample(const void *p, int bytes, size_t q)
{
    if (bytes == 1) return (float)((const uint8_t *)p)[q];
    if (bytes == 2) return (float)((const uint16_t *)p)[q];
    return ((const float *)p)[q];
}

static void store_sample(void *p, int bytes, size_t q, float v)
{
    if (bytes == 1) ((uint8_t *)p)[q] = (uint8_t)v;          // static_cast truncation
    else if (bytes == 2) ((uint16_t *)p)[q] = (uint16_t)v;
    else ((float *)p)[q] = v;
}

// Full-range quantisation of a format (GetQuanPara, include/Helper.h:286-351): integer formats
// [0, 2^b - 1] with chroma neutral 2^(b-1); float luma [0, 1], chroma [-0.5, 0.5] around 0.
struct Quan {
    float floorY, ceilY, floorC, neutralC, ceilC;
    bool pc_chroma;       // _IsPCChroma (include/Helper.h:363-372)
};

static Quan quan_full(int bytes, int bits)
{
    Quan q;
    if (bytes == 4) {
        q.floorY = 0.0f; q.ceilY = 1.0f; q.floorC = -0.5f; q.neutralC = 0.0f; q.ceilC = 0.5f;
        q.pc_chroma = false;
    } else {
        int fl, ne, ce;
        quan_int(bits, 1, 0, fl, ne, ce);
        q.floorY = (float)fl; q.ceilY = (float)ce;
        quan_int(bits, 1, 1, fl, ne, ce);
        q.floorC = (float)fl; q.neutralC = (float)ne; q.ceilC = (float)ce;
        q.pc_chroma = fl < ne && (fl + ce) % 2 == 1;
    }
    return q;
}

// MatrixConvert_RGB2YUV, OPP branch (include/Conversion.hpp:205-236), for any sample types
// (RGB2OPP_Process::process_core, include/RGB2OPP.h:185-205; RGB2FloatYUV, Conversion.hpp:470-487):
// full range on both sides; integer destinations get the +0.5 (+0.499999 for PC-range chroma)
// rounding offset, and with clip the results are clipped to the destination range.
void oracle_rgb2opp_any(const void *R, const void *G, const void *B, int in_bytes, int in_bits,
                        void *Y, void *U, void *V, int out_bytes, int out_bits, int H, int W,
                        int stride, int clip)
{
    const Quan s = quan_full(in_bytes, in_bits), d = quan_full(out_bytes, out_bits);
    const bool dst_float = out_bytes == 4;
    const float sRange = s.ceilY - s.floorY;
    const float dRangeY = d.ceilY - d.floorY, dRangeC = d.ceilC - d.floorC;
    const float gainY = dRangeY / (sRange * 3.0f);
    float offsetY = -s.floorY * 3.0f * gainY + d.floorY;
    if (!dst_float) offsetY += 0.5f;
    const float gainU = dRangeC / (sRange * 2.0f);
    const float gainV = dRangeC / (sRange * 4.0f);
    float offsetC = d.neutralC;
    if (!dst_float) offsetC += d.pc_chroma ? 0.499999f : 0.5f;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const size_t q = (size_t)y * stride + x;
            const float r = load_sample(R, in_bytes, q), g = load_sample(G, in_bytes, q), b = load_sample(B, in_bytes, q);
            float t = (r + g + b) * gainY + offsetY;
            store_sample(Y, out_bytes, q, clip ? clipf(t, d.floorY, d.ceilY) : t);
            t = (r - b) * gainU + offsetC;
            store_sample(U, out_bytes, q, clip ? clipf(t, d.floorC, d.ceilC) : t);
            t = (r - g * 2.0f + b) * gainV + offsetC;
            store_sample(V, out_bytes, q, clip ? clipf(t, d.floorC, d.ceilC) : t);
        }
}

// ConvertToY, OPP branch (include/Conversion.hpp:103-116) into float, full range, no clip
// (RGB2FloatY, Conversion.hpp:455-468): Basic's ref plane of an RGB clip.
void oracle_rgb2y_any(const void *R, const void *G, const void *B, int in_bytes, int in_bits, int H, int W,
                      int stride, float *Y)
{
    const Quan s = quan_full(in_bytes, in_bits);
    const float sRange = s.ceilY - s.floorY;
    const float gain = (1.0f - 0.0f) / (sRange * 3.0f);
    const float offset = -s.floorY * 3.0f * gain + 0.0f;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const size_t q = (size_t)y * stride + x;
            Y[q] = (load_sample(R, in_bytes, q) + load_sample(G, in_bytes, q) + load_sample(B, in_bytes, q)) * gain + offset;
        }
}

// MatrixConvert_YUV2RGB, OPP branch (include/Conversion.hpp:290-392, coefficients
// include/Specification.h:253-269), for any sample types (OPP2RGB_Process::process_core,
// include/OPP2RGB.h:185-205; FloatYUV2RGB, Conversion.hpp:489-506), full range.
void oracle_opp2rgb_any(const void *Y, const void *U, const void *V, int in_bytes, int in_bits,
                        void *R, void *G, void *B, int out_bytes, int out_bits, int H, int W,
                        int stride, int clip)
{
    const Quan s = quan_full(in_bytes, in_bits), d = quan_full(out_bytes, out_bits);
    const bool dst_float = out_bytes == 4;
    const float dRange = d.ceilY - d.floorY;
    const float gainY = dRange / (s.ceilY - s.floorY);
    const float gainC = dRange / (s.ceilC - s.floorC);
    float Ry = (float)1.0L, Ru = (float)1.0L, Rv = (float)(2.0L / 3.0L);
    float Gy = (float)1.0L, Gu = (float)0.0L, Gv = (float)(-4.0L / 3.0L);
    float By = (float)1.0L, Bu = (float)-1.0L, Bv = (float)(2.0L / 3.0L);
    Ry *= gainY; Ru *= gainC; Rv *= gainC;
    Gy *= gainY; Gu *= gainC; Gv *= gainC;
    By *= gainY; Bu *= gainC; Bv *= gainC;
    float oR = -s.floorY * Ry - s.neutralC * (Ru + Rv) + d.floorY;
    float oG = -s.floorY * Gy - s.neutralC * (Gu + Gv) + d.floorY;
    float oB = -s.floorY * By - s.neutralC * (Bu + Bv) + d.floorY;
    if (!dst_float) { oR += 0.5f; oG += 0.5f; oB += 0.5f; }
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const size_t q = (size_t)y * stride + x;
            const float yy = load_sample(Y, in_bytes, q), u = load_sample(U, in_bytes, q), v = load_sample(V, in_bytes, q);
            float t = Ry * yy + Ru * u + Rv * v + oR;
            store_sample(R, out_bytes, q, clip ? clipf(t, d.floorY, d.ceilY) : t);
            t = Gy * yy + Gv * v + oG;
            store_sample(G, out_bytes, q, clip ? clipf(t, d.floorY, d.ceilY) : t);
            t = By * yy + Bu * u + Bv * v + oB;
            store_sample(B, out_bytes, q, clip ? clipf(t, d.floorY, d.ceilY) : t);
        }
}

} // extern "C"
