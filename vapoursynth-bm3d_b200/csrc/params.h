// params.h -- host-side restatement of the reference's parameter layer: profile presets,
// colour-matrix normalisation and per-plane filter tables.
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <limits>
#include <string>
#include <vector>

namespace bm3d {

// ColorMatrix (include/Specification.h:53-68)
enum Matrix {
    MAT_GBR = 0, MAT_BT709 = 1, MAT_UNSPEC = 2, MAT_FCC = 4, MAT_BT470BG = 5, MAT_SMPTE170M = 6,
    MAT_SMPTE240M = 7, MAT_YCGCO = 8, MAT_BT2020NC = 9, MAT_BT2020C = 10, MAT_OPP = 100
};

struct Params {
    bool wiener = false;
    std::string profile = "fast";
    double sigma[3] = {10.0, 10.0, 10.0};
    int B = 8, step = 4, G = 16, R = 16, bmstep = 1;
    double thMSE = 0.0;
    double lambda = 0.0;
    int radius = 0, psnum = 0, psrange = 0, psstep = 0;
};

// BM3D_Para::BM3D_Para (source/BM3D.cpp:33-107)
inline Params bm3d_profile(bool wiener, const std::string &profile)
{
    Params p;
    p.wiener = wiener;
    p.profile = profile;
    p.B = 8;
    p.R = 16;
    p.bmstep = 1;
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
    return p;
}

// VBM3D_Para::VBM3D_Para (source/VBM3D_Base.cpp:32-97): the BM3D preset, then V overrides
inline Params vbm3d_profile(bool wiener, const std::string &profile)
{
    Params p = bm3d_profile(wiener, profile);
    p.radius = 3; p.G = 8; p.R = 12; p.psnum = 2; p.psstep = 1;
    p.psrange = wiener ? 6 : 5;
    if (profile == "fast") { p.radius = 1; p.R = 7; p.psrange = wiener ? 5 : 4; }
    else if (profile == "lc") { p.radius = 2; p.R = 9; p.psrange = wiener ? 5 : 4; }
    else if (profile == "high") { p.radius = 4; p.R = 16; p.psrange = wiener ? 8 : 7; }
    else if (profile == "vn") { p.radius = 4; p.G = 16; }
    return p;
}

// BM3D_Para::thMSE_Default (source/BM3D.cpp:110-130)
inline double thmse_default(bool wiener, const std::string &profile, double sigma0)
{
    if (!wiener) return profile == "vn" ? 1000 + sigma0 * 150 : 400 + sigma0 * 80;
    return profile == "vn" ? 400 + sigma0 * 40 : 200 + sigma0 * 10;
}

// ColorMatrix_Default (include/Specification.h:297-313)
inline int matrix_default(int W, int H)
{
    if (W > 2048 || H > 1536) return MAT_BT2020NC;
    if (W > 1024 || H > 576) return MAT_BT709;
    return MAT_SMPTE170M;
}

// Row norms of ColorMatrix_RGB2YUV_Parameter<double> (include/Specification.h:139-213) as used by
// init_filter_data (source/BM3D_Base.cpp:262-283).
inline void matrix_norms(int m, double norm[3])
{
    double c[9];
    if (m == MAT_GBR) {
        const double v[9] = {0, 1, 0, 0, 0, 1, 1, 0, 0};
        for (int k = 0; k < 9; ++k) c[k] = v[k];
    } else if (m == MAT_YCGCO) {
        c[0] = (double)(1.0L / 4.0L); c[1] = (double)(1.0L / 2.0L); c[2] = (double)(1.0L / 4.0L);
        c[3] = (double)(-1.0L / 4.0L); c[4] = (double)(1.0L / 2.0L); c[5] = (double)(-1.0L / 4.0L);
        c[6] = (double)(1.0L / 2.0L); c[7] = 0.0; c[8] = (double)(-1.0L / 2.0L);
    } else if (m == MAT_OPP) {
        c[0] = (double)(1.0L / 3.0L); c[1] = (double)(1.0L / 3.0L); c[2] = (double)(1.0L / 3.0L);
        c[3] = (double)(1.0L / 2.0L); c[4] = 0.0; c[5] = (double)(-1.0L / 2.0L);
        c[6] = (double)(1.0L / 4.0L); c[7] = (double)(-1.0L / 2.0L); c[8] = (double)(1.0L / 4.0L);
    } else {
        long double Kr, Kg, Kb;
        switch (m) {
        case MAT_BT709: Kr = 0.2126; Kg = 0.7152; Kb = 0.0722; break;
        case MAT_FCC: Kr = 0.30; Kg = 0.59; Kb = 0.11; break;
        case MAT_BT470BG: case MAT_SMPTE170M: Kr = 0.299; Kg = 0.587; Kb = 0.114; break;
        case MAT_SMPTE240M: Kr = 0.212; Kg = 0.701; Kb = 0.087; break;
        case MAT_BT2020NC: case MAT_BT2020C: Kr = 0.2627; Kg = 0.6780; Kb = 0.0593; break;
        default: Kr = 0.2126; Kg = 0.7152; Kb = 0.0722; break;
        }
        const double Yr = (double)Kr, Yg = (double)Kg, Yb = (double)Kb;
        c[0] = Yr; c[1] = Yg; c[2] = Yb;
        c[3] = (double)(-Yr * 0.5L / (1.0L - Yb));
        c[4] = (double)(-Yg * 0.5L / (1.0L - Yb));
        c[5] = 0.5;
        c[6] = 0.5;
        c[7] = (double)(-Yg * 0.5L / (1.0L - Yr));
        c[8] = (double)(-Yb * 0.5L / (1.0L - Yr));
    }
    norm[0] = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    norm[1] = std::sqrt(c[3] * c[3] + c[4] * c[4] + c[5] * c[5]);
    norm[2] = std::sqrt(c[6] * c[6] + c[7] * c[7] + c[8] * c[8]);
}

// Per-plane tables of BM3D_FilterData (source/BM3D.cpp:137-209):
//   amp[n-1] = finalAMP = 2n * 2B * 2B; thr4[n-1][flag] = float(sigma*lambda*sqrt(finalAMP) *
//   {1, sqrt 2, 2, sqrt 8}[flag]) with flag = #(x==0, y==0, z==0); wsig2[n-1] =
//   max(FLT_MIN, float(sigma*sqrt(finalAMP)*sigma*sqrt(finalAMP))).
struct PlaneTables {
    std::vector<double> amp;
    std::vector<float> thr4;     // [G][4]
    std::vector<float> wsig2;    // [G]
};

inline PlaneTables plane_tables(bool wiener, double sigma, int G, int B, double lambda)
{
    PlaneTables t;
    t.amp.resize(G);
    t.thr4.assign((size_t)G * 4, 0.0f);
    t.wsig2.assign(G, 0.0f);
    for (int i = 1; i <= G; ++i) {
        t.amp[i - 1] = 2 * i * 2 * B * 2 * B;
        const double forwardAMP = std::sqrt(t.amp[i - 1]);
        if (wiener) {
            const float v = static_cast<float>(sigma * forwardAMP * sigma * forwardAMP);
            const float mn = std::numeric_limits<float>::min();
            t.wsig2[i - 1] = v > mn ? v : mn;
        } else {
            const double thrBase = sigma * lambda * forwardAMP;
            t.thr4[(i - 1) * 4 + 0] = static_cast<float>(thrBase);
            t.thr4[(i - 1) * 4 + 1] = static_cast<float>(thrBase * std::sqrt(double(2)));
            t.thr4[(i - 1) * 4 + 2] = static_cast<float>(thrBase * double(2));
            t.thr4[(i - 1) * 4 + 3] = static_cast<float>(thrBase * std::sqrt(double(8)));
        }
    }
    return t;
}

// 2*cos(pi*a/b) rounded to float: the single formula behind every DCT table.
inline float cos2(long a, long b)
{
    const double ang = (double)a * M_PI / (double)b;
    return (float)(2.0 * std::cos(ang));
}

// Reference-block scan with clamping (source/BM3D_Base.cpp:421-443)
inline std::vector<int> scan_positions(int extent, int B, int step)
{
    std::vector<int> out;
    const int last = extent - B;
    for (int j = 0;; j += step) {
        if (j >= last + step) break;
        if (j > last) j = last;
        out.push_back(j);
    }
    return out;
}

}  // namespace bm3d
