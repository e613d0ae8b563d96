// common.cuh -- device-side building blocks shared by the BM3D / V-BM3D kernels (sm_100a).
//
// Arithmetic contract: every floating-point step that decides a result bit (SSD accumulation,
// the 3-D DCT, the shrinkage weights) is written with the explicit round-to-nearest intrinsics
// (__fadd_rn, __fsub_rn, __fmul_rn, __fmaf_rn, __fdiv_rn) so that nvcc's FMA contraction can
// never change the evaluation order the reference (and the CPU oracle) uses.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "args.h"

namespace bm3d {

// ---------------------------------------------------------------------------------------------
// DCT tables.  The transform replaces FFTW's r2r REDFT10 (forward) and REDFT01 (inverse), the
// 3-D transforms of source/BM3D.cpp:137-151.  Definitions (FFTW's, unnormalised):
//   forward  X_k = 2 sum_{j<N} x_j cos(pi (2j+1) k / 2N)
//   inverse  y_k = X_0 + 2 sum_{1<=j<N} X_j cos(pi j (2k+1) / 2N)
// Factorisation used for every power-of-two N (partial butterfly):
//   forward: e_j = x_j + x_{N-1-j}, o_j = x_j - x_{N-1-j}; X_{2m} = F_{N/2}(e)_m;
//            X_{2m+1} = fma-chain over j of o_j * c_N[m][j]; F_1(x) = 2 x_0
//   inverse: E = I_{N/2}(X_0, X_2, ...); O_k = fma-chain over m of X_{2m+1} * c_N[k][m];
//            y_k = E_k + O_k, y_{N-1-k} = E_k - O_k; I_1(X) = X_0
// with c_N[m][j] = float(2 cos(pi (2j+1)(2m+1) / 2N)).  Other N use direct FMA chains over the
// full matrices (fwd[k][j] = float(2cos(pi(2j+1)k/2N)), inv[k][j] = float(2cos(pi j(2k+1)/2N))).
// Each chain starts with a plain multiply (forward, odd parts) or with X_0 (direct inverse) and
// adds terms in ascending index order.  The CPU oracle implements the same sequence.

// Offsets of c_N inside the packed odd-table array, N = 2 .. 256.
__host__ __device__ constexpr int odd_off(int N)
{
    return N == 2 ? 0 : N == 4 ? 1 : N == 8 ? 5 : N == 16 ? 21 : N == 32 ? 85 : N == 64 ? 341
         : N == 128 ? 1365 : N == 256 ? 5461 : -1;
}
constexpr int kOddConstFloats = 1365;     // N = 2..64 live in constant memory
constexpr int kOddAllFloats = 21845;      // N = 2..256 (global copy for the generic path)

// Defined once: common.cuh is included by the single kernel translation unit (kernels.cu).
__constant__ float c_odd[kOddConstFloats];

__device__ __forceinline__ float odd_coef(int N, int m, int j)
{
    return c_odd[odd_off(N) + m * (N / 2) + j];
}

// Forward DCT-II of a register array (N a power of two, fully unrolled).
template <int N>
__device__ __forceinline__ void fdct_reg(const float (&x)[N], float (&X)[N])
{
    if constexpr (N == 1) {
        X[0] = __fmul_rn(x[0], 2.0f);
    } else {
        constexpr int h = N / 2;
        float e[h], o[h], E[h];
#pragma unroll
        for (int j = 0; j < h; ++j) {
            e[j] = __fadd_rn(x[j], x[N - 1 - j]);
            o[j] = __fsub_rn(x[j], x[N - 1 - j]);
        }
        fdct_reg<h>(e, E);
#pragma unroll
        for (int m = 0; m < h; ++m) {
            X[2 * m] = E[m];
            float acc = __fmul_rn(o[0], c_odd[odd_off(N) + m * h]);
#pragma unroll
            for (int j = 1; j < h; ++j) acc = __fmaf_rn(o[j], c_odd[odd_off(N) + m * h + j], acc);
            X[2 * m + 1] = acc;
        }
    }
}

// Inverse DCT-III of a register array (N a power of two, fully unrolled).
template <int N>
__device__ __forceinline__ void idct_reg(const float (&X)[N], float (&y)[N])
{
    if constexpr (N == 1) {
        y[0] = X[0];
    } else {
        constexpr int h = N / 2;
        float ev[h], E[h];
#pragma unroll
        for (int m = 0; m < h; ++m) ev[m] = X[2 * m];
        idct_reg<h>(ev, E);
#pragma unroll
        for (int k = 0; k < h; ++k) {
            float acc = __fmul_rn(X[1], c_odd[odd_off(N) + k * h]);
#pragma unroll
            for (int m = 1; m < h; ++m) acc = __fmaf_rn(X[2 * m + 1], c_odd[odd_off(N) + k * h + m], acc);
            y[k] = __fadd_rn(E[k], acc);
            y[N - 1 - k] = __fsub_rn(E[k], acc);
        }
    }
}

// Runtime-length versions on a strided array (generic path).  `tmp` must hold 2*N floats.
// odd_all: all odd tables (N = 2..256); fwd/inv: direct tables for this N (non-power-of-two).
__device__ inline void fdct_any(float *v, int N, int stride, float *tmp, const float *odd_all,
                                const float *fwd)
{
    if ((N & (N - 1)) == 0) {
        // level by level: the odd outputs of level L land at index (2m+1) << L
        float *cur = tmp, *nxt = tmp + N;
        for (int j = 0; j < N; ++j) cur[j] = v[j * stride];
        int len = N, shift = 0;
        while (len > 1) {
            const int h = len / 2;
            const float *c = odd_all + odd_off(len);
            for (int j = 0; j < h; ++j) {
                nxt[j] = __fadd_rn(cur[j], cur[len - 1 - j]);
                cur[len - 1 - j] = __fsub_rn(cur[j], cur[len - 1 - j]);   // o_j stored at the top
            }
            for (int m = 0; m < h; ++m) {
                float acc = __fmul_rn(cur[len - 1], c[m * h]);
                for (int j = 1; j < h; ++j) acc = __fmaf_rn(cur[len - 1 - j], c[m * h + j], acc);
                v[((2 * m + 1) << shift) * stride] = acc;
            }
            float *t = cur; cur = nxt; nxt = t;
            len = h;
            ++shift;
        }
        v[0] = __fmul_rn(cur[0], 2.0f);
    } else {
        for (int j = 0; j < N; ++j) tmp[j] = v[j * stride];
        for (int k = 0; k < N; ++k) {
            float acc = __fmul_rn(tmp[0], fwd[k * N]);
            for (int j = 1; j < N; ++j) acc = __fmaf_rn(tmp[j], fwd[k * N + j], acc);
            v[k * stride] = acc;
        }
    }
}

__device__ inline void idct_any(float *v, int N, int stride, float *tmp, const float *odd_all,
                                const float *inv)
{
    if ((N & (N - 1)) == 0) {
        // bottom-up: level of length len reads the odd inputs X[(2m+1) * (N/len)]
        float *cur = tmp, *nxt = tmp + N;
        cur[0] = v[0];
        for (int len = 2; len <= N; len *= 2) {
            const int h = len / 2;
            const int s = N / len;
            const float *c = odd_all + odd_off(len);
            for (int k = 0; k < h; ++k) {
                float acc = __fmul_rn(v[s * stride], c[k * h]);
                for (int m = 1; m < h; ++m) acc = __fmaf_rn(v[(2 * m + 1) * s * stride], c[k * h + m], acc);
                nxt[k] = __fadd_rn(cur[k], acc);
                nxt[len - 1 - k] = __fsub_rn(cur[k], acc);
            }
            float *t = cur; cur = nxt; nxt = t;
        }
        for (int k = 0; k < N; ++k) v[k * stride] = cur[k];
    } else {
        for (int j = 0; j < N; ++j) tmp[j] = v[j * stride];
        for (int k = 0; k < N; ++k) {
            float acc = tmp[0];
            for (int j = 1; j < N; ++j) acc = __fmaf_rn(tmp[j], inv[k * N + j], acc);
            v[k * stride] = acc;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Warp helpers

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace bm3d
