// fp64.cuh -- FP64 GPU oracle of the collaborative filter and aggregation.
//
// Recomputes, in double precision, what K3+K4 compute from the same inputs and match lists:
// gather -> forward 3-D DCT (REDFT10 along x, y, z) -> hard threshold (Basic) or Wiener shrinkage
// (Final) -> inverse 3-D DCT (REDFT01) -> weighted aggregation of numerator and denominator ->
// num / den (source/BM3D_Basic.cpp:72-148, source/BM3D_Final.cpp:50-127,
// include/Block.h:1239-1345, source/BM3D_Base.cpp:348-351).  Thresholds and Wiener variances are
// derived in double from sigma, lambda and the group length, transforms use double cosines, and
// the sums are double atomics.  It is an inspection tool for the error of the FP32 and tf32
// forms; no production path calls it.
#pragma once

#include "args.h"
#include "cf.cuh"

namespace bm3d {

// In-place 1-D transform of one N-point line (N <= 64, stride `st`); `tmp` holds N doubles.
// inverse = 0: y_k = 2 sum_j x_j cos(pi (2j + 1) k / 2N); inverse = 1: x_j = y_0 + 2 sum_{k>=1}
// y_k cos(pi k (2j + 1) / 2N).
__device__ inline void dct_line_f64(double *v, double *tmp, int N, int st, bool inverse)
{
    for (int i = 0; i < N; ++i) tmp[i] = v[i * st];
    for (int o = 0; o < N; ++o) {
        double acc = 0.0;
        if (!inverse) {
            for (int i = 0; i < N; ++i) acc += tmp[i] * 2.0 * cos(M_PI * (2 * i + 1) * o / (2.0 * N));
        } else {
            acc = tmp[0];
            for (int i = 1; i < N; ++i) acc += tmp[i] * 2.0 * cos(M_PI * i * (2 * o + 1) / (2.0 * N));
        }
        v[o * st] = acc;
    }
}

// 3-D transform of an n x B x B group ([z][y][x]) by the CTA: forward x, y, z; inverse z, y, x.
__device__ inline void dct3d_f64(double *g, double *tmp, int n, int B, bool inverse)
{
    const int plane = B * B;
    const int nl_xy = n * B;              // lines along x (and along y)
    for (int pass = 0; pass < 3; ++pass) {
        const int axis = inverse ? 2 - pass : pass;   // 0 = x, 1 = y, 2 = z
        const int lines = axis == 2 ? plane : nl_xy;
        for (int l = threadIdx.x; l < lines; l += blockDim.x) {
            double *t = tmp + threadIdx.x * 64;
            if (axis == 0) dct_line_f64(g + l * B, t, B, 1, inverse);
            else if (axis == 1) dct_line_f64(g + (l / B) * plane + (l % B), t, B, B, inverse);
            else dct_line_f64(g + l, t, n, plane, inverse);
        }
        __syncthreads();
    }
}

// One CTA of 64 threads per group (G <= 64, B <= 64); dynamic shared memory: 2 * G * B * B
// doubles (source, reference) and 64 doubles of line buffer per thread.
__global__ void cf_fp64_kernel(CFArgs a, F64Args f)
{
    extern __shared__ double dsm[];
    const long long grp = blockIdx.x;
    const int B = a.B, plane = B * B;
    const int n = min(a.count[grp], a.G);
    double *g = dsm;
    double *rg = g + (long long)a.G * plane;
    double *tmp = rg + (long long)a.G * plane;
    const uint32_t *pl = a.pos + grp * a.G;
    __shared__ double red;
    for (int p = 0; p < 3; ++p) {
        if (!a.process[p]) continue;
        for (int idx = threadIdx.x; idx < n * plane; idx += blockDim.x) {
            const int k = idx / plane, e = idx - k * plane, y = e / B, x = e - y * B;
            const GroupLoc L = locate(a, p, grp, pl[k]);
            g[idx] = (double)L.src[(long long)(L.y + y) * a.ld + L.x + x];
            if (a.wiener) rg[idx] = (double)L.ref[(long long)(L.y + y) * a.ld + L.x + x];
        }
        __syncthreads();
        dct3d_f64(g, tmp, n, B, false);
        if (a.wiener) dct3d_f64(rg, tmp, n, B, false);
        const double amp = 2.0 * n * 2.0 * B * 2.0 * B;
        const double s = f.sigma[p] * sqrt(amp);
        if (threadIdx.x == 0) red = 0.0;
        __syncthreads();
        double part = 0.0;
        for (int idx = threadIdx.x; idx < n * plane; idx += blockDim.x) {
            if (!a.wiener) {
                const int k = idx / plane, e = idx - k * plane, y = e / B, x = e - y * B;
                const int flag = (x == 0) + (y == 0) + (k == 0);
                const double mul = flag == 0 ? 1.0 : flag == 1 ? sqrt(2.0) : flag == 2 ? 2.0 : sqrt(8.0);
                const bool keep = fabs(g[idx]) > s * f.lambda * mul;
                if (!keep) g[idx] = 0.0;
                part += keep ? 1.0 : 0.0;
            } else {
                const double r2 = rg[idx] * rg[idx];
                const double w = r2 / (r2 + s * s);
                g[idx] *= w;
                part += w * w;
            }
        }
        atomicAdd(&red, part);
        __syncthreads();
        dct3d_f64(g, tmp, n, B, true);
        double denW;
        if (!a.wiener) denW = red < 1.0 ? 1.0 : 1.0 / red;
        else denW = 1.0 / (red > 1.1920928955078125e-07 ? red : 1.1920928955078125e-07);
        const double numW = denW / amp;
        const long long fr = grp / a.blocks_per_frame;
        for (int idx = threadIdx.x; idx < n * plane; idx += blockDim.x) {
            const int k = idx / plane, e = idx - k * plane, y = e / B, x = e - y * B;
            const GroupLoc L = locate(a, p, grp, pl[k]);
            const long long o = (fr * a.H + L.y + y) * f.out_stride + L.x + x;
            atomicAdd(f.num[p] + o, g[idx] * numW);
            atomicAdd(f.den[p] + o, denW);
        }
        __syncthreads();
    }
}

__global__ void finalize_fp64_kernel(F64Args f, int W, int H, int nframes, int process0, int process1, int process2)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int p = blockIdx.z % 3, fr = blockIdx.z / 3;
    const int pr = p == 0 ? process0 : p == 1 ? process1 : process2;
    if (x >= W || !pr || fr >= nframes) return;
    const long long o = ((long long)fr * H + y) * f.out_stride + x;
    f.num[p][o] = f.num[p][o] / f.den[p][o];
}

}  // namespace bm3d
