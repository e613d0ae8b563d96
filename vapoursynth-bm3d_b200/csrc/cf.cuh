// cf.cuh -- K3+K4: collaborative filtering of every group and its aggregation.
//
// Replaces BM3D_Basic_Process::CollaborativeFilter (source/BM3D_Basic.cpp:72-148),
// BM3D_Final_Process::CollaborativeFilter (source/BM3D_Final.cpp:50-127), their V-BM3D twins
// (source/VBM3D_Basic.cpp:72-148, source/VBM3D_Final.cpp:50-127) and the scatter
// BlockGroup::AddTo / CountTo (include/Block.h:1239-1387):
//   gather n = min(|matches|, group_size) blocks in match order -> forward 3-D DCT (x, y, z) ->
//   Basic: keep c iff |c| > thr[n][z][y][x], count kept R, denW = R<1 ? 1 : 1/R
//   Final: w = r^2 / (r^2 + sigma^2[n]) from the reference group, s *= w, L2 = sum w^2,
//          denW = 1 / max(FLT_EPSILON, L2)
//   -> inverse 3-D DCT (z, y, x) -> numW = denW / finalAMP[n]
//   -> num[p] += v * numW over each block footprint, den[p] += denW.
// The denominator is accumulated as one weight per block origin (wmap) and expanded by a
// B x B box sum in the finalize kernel; the numerator is added per pixel.  Summation order of
// the aggregation therefore differs from the reference's sequential order (float atomics), which
// is why outputs are compared with a tolerance while match lists and transforms are exact.
// The Final L2 sum uses a tree order (the reference's SSE and scalar builds already disagree
// on it); it only scales a group weight.
#pragma once

#include "common.cuh"
#include "args.h"

namespace bm3d {


// ---- 8x8 2-D transforms in registers (forward: x then y; inverse: y then x) -----------------

__device__ __forceinline__ void fwd2d8(float (&b)[64])
{
#pragma unroll
    for (int y = 0; y < 8; ++y) {
        float in[8], out[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) in[k] = b[y * 8 + k];
        fdct_reg<8>(in, out);
#pragma unroll
        for (int k = 0; k < 8; ++k) b[y * 8 + k] = out[k];
    }
#pragma unroll
    for (int x = 0; x < 8; ++x) {
        float in[8], out[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) in[k] = b[k * 8 + x];
        fdct_reg<8>(in, out);
#pragma unroll
        for (int k = 0; k < 8; ++k) b[k * 8 + x] = out[k];
    }
}

__device__ __forceinline__ void inv2d8(float (&b)[64])
{
#pragma unroll
    for (int x = 0; x < 8; ++x) {
        float in[8], out[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) in[k] = b[k * 8 + x];
        idct_reg<8>(in, out);
#pragma unroll
        for (int k = 0; k < 8; ++k) b[k * 8 + x] = out[k];
    }
#pragma unroll
    for (int y = 0; y < 8; ++y) {
        float in[8], out[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) in[k] = b[y * 8 + k];
        idct_reg<8>(in, out);
#pragma unroll
        for (int k = 0; k < 8; ++k) b[y * 8 + k] = out[k];
    }
}

struct GroupLoc {
    const float *src;      // plane origin for this block (frame resolved)
    const float *ref;
    float *num;
    float *wmap;
    int y, x;
};

__device__ __forceinline__ GroupLoc locate(const CFArgs &a, int p, long long grp, uint32_t pk)
{
    GroupLoc g;
    const long long f = grp / a.blocks_per_frame;
    if (!a.vbm3d) {
        g.y = unpack_y(pk);
        g.x = unpack_x(pk);
        g.src = a.src[p] + f * a.frame_stride;
        g.ref = a.ref[p] + f * a.frame_stride;
        g.num = a.num[p] + f * a.frame_stride;
        g.wmap = a.wmap[p] + f * a.frame_stride;
    } else {
        const int z = unpack3_z(pk);
        g.y = unpack3_y(pk);
        g.x = unpack3_x(pk);
        const long long fr = (long long)a.win_base[f] + z;
        g.src = a.src[p] + fr * a.frame_stride;
        g.ref = a.ref[p] + fr * a.frame_stride;
        const long long slot = f * a.slots + a.slot0[f] + z;
        g.num = a.num[p] + slot * a.acc_stride;
        g.wmap = a.wmap[p] + slot * a.acc_stride;
    }
    return g;
}

// ---- fast path: B = 8, full groups of G in {8, 16, 32}; lane = block for the 2-D stages,
//      lane = coefficient column(s) for the z stage; transposes through padded shared memory ----

template <int G, bool WIENER>
__global__ void __launch_bounds__(128) cf_fast_kernel(CFArgs a)
{
    constexpr int GPW = 32 / G;      // groups per warp
    constexpr int C = 64 / G;        // coefficient columns per lane in the z stage
    constexpr int TP = 65;           // padded row pitch of the transpose buffer
    extern __shared__ float smem[];
    const int lane = (int)lane_id();
    const int warp = threadIdx.x >> 5;
    const int sub = lane / G;
    const int z = lane - sub * G;
    float *T = smem + warp * (WIENER ? 2 : 1) * 32 * TP;
    float *T2 = T + 32 * TP;

    const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long wg = (long long)blockIdx.x * (blockDim.x >> 5) + warp; wg * GPW < a.ngroups; wg += nwarps) {
        const long long grp = wg * GPW + sub;
        const bool inrange = grp < a.ngroups;
        const int n = inrange ? a.count[grp] : 0;
        const bool active = inrange && n == G;
        const uint32_t pk = active ? a.pos[grp * G + z] : a.pos[0];
        const long long g0 = active ? grp : 0;

        for (int p = 0; p < 3; ++p) {
            if (!a.process[p]) continue;
            const GroupLoc L = locate(a, p, g0, pk);
            float blk[64];
            {
                const float *sp = L.src + (long long)L.y * a.ld + L.x;
#pragma unroll
                for (int y = 0; y < 8; ++y)
#pragma unroll
                    for (int x = 0; x < 8; ++x) blk[y * 8 + x] = __ldg(sp + (long long)y * a.ld + x);
            }
            fwd2d8(blk);
#pragma unroll
            for (int e = 0; e < 64; ++e) T[lane * TP + e] = blk[e];
            if constexpr (WIENER) {
                const float *rp = L.ref + (long long)L.y * a.ld + L.x;
#pragma unroll
                for (int y = 0; y < 8; ++y)
#pragma unroll
                    for (int x = 0; x < 8; ++x) blk[y * 8 + x] = __ldg(rp + (long long)y * a.ld + x);
                fwd2d8(blk);
#pragma unroll
                for (int e = 0; e < 64; ++e) T2[lane * TP + e] = blk[e];
            }
            __syncwarp();

            int kept = 0;
            float l2 = 0.0f;
#pragma unroll 1
            for (int q = 0; q < C; ++q) {
                const int c = z + q * G;             // coefficient column (y*8 + x)
                float col[G], X[G];
#pragma unroll
                for (int zz = 0; zz < G; ++zz) col[zz] = T[(sub * G + zz) * TP + c];
                fdct_reg<G>(col, X);
                if constexpr (!WIENER) {
                    const int fxy = ((c & 7) == 0) + ((c >> 3) == 0);
                    const float t0 = a.thr4[p][G - 1][fxy + 1];   // z == 0
                    const float t1 = a.thr4[p][G - 1][fxy];       // z > 0
#pragma unroll
                    for (int zz = 0; zz < G; ++zz) {
                        const float th = zz == 0 ? t0 : t1;
                        const bool keep = fabsf(X[zz]) > th;
                        kept += keep;
                        X[zz] = keep ? X[zz] : 0.0f;
                    }
                } else {
                    float rc[G], R[G];
#pragma unroll
                    for (int zz = 0; zz < G; ++zz) rc[zz] = T2[(sub * G + zz) * TP + c];
                    fdct_reg<G>(rc, R);
                    const float sg = a.wsig2[p][G - 1];
#pragma unroll
                    for (int zz = 0; zz < G; ++zz) {
                        const float r2 = __fmul_rn(R[zz], R[zz]);
                        const float w = __fdiv_rn(r2, __fadd_rn(r2, sg));
                        X[zz] = __fmul_rn(X[zz], w);
                        l2 = __fadd_rn(l2, __fmul_rn(w, w));
                    }
                }
                idct_reg<G>(X, col);
#pragma unroll
                for (int zz = 0; zz < G; ++zz) T[(sub * G + zz) * TP + c] = col[zz];
            }
            // reduce over the G lanes of this group
#pragma unroll
            for (int o = G / 2; o > 0; o >>= 1) {
                if constexpr (!WIENER) kept += __shfl_xor_sync(0xffffffffu, kept, o);
                else l2 = __fadd_rn(l2, __shfl_xor_sync(0xffffffffu, l2, o));
            }
            __syncwarp();
#pragma unroll
            for (int e = 0; e < 64; ++e) blk[e] = T[lane * TP + e];
            __syncwarp();
            inv2d8(blk);

            float denW;
            if constexpr (!WIENER) {
                denW = kept < 1 ? 1.0f : __fdiv_rn(1.0f, (float)kept);
            } else {
                const float eps = 1.1920928955078125e-07f;
                denW = __fdiv_rn(1.0f, l2 > eps ? l2 : eps);
            }
            const float numW = __fdiv_rn(denW, a.amp[G - 1]);
            if (active) {
                float *np = L.num + (long long)L.y * a.ld + L.x;
#pragma unroll
                for (int y = 0; y < 8; ++y)
#pragma unroll
                    for (int x = 0; x < 8; ++x) atomicAdd(np + (long long)y * a.ld + x, __fmul_rn(blk[y * 8 + x], numW));
                atomicAdd(L.wmap + (long long)L.y * a.ld + L.x, denW);
            }
        }
    }
}

// ---- generic path: any B <= 64, any n <= 256; one warp per group, data in global scratch ----

__device__ __forceinline__ const float *dtab_for(const CFArgs &a, int N, bool inverse)
{
    const int off = a.dtab_off[N];
    return off < 0 ? nullptr : a.dtab + off + (inverse ? N * N : 0);
}

__device__ void dct3d_warp(float *g, int n, int B, bool inverse, const CFArgs &a, float *tmp)
{
    const int lane = (int)lane_id();
    const int plane = B * B;
    const float *fB = dtab_for(a, B, inverse);
    const float *fn = dtab_for(a, n, inverse);
    if (!inverse) {
        for (int t = lane; t < n * B; t += 32) fdct_any(g + t * B, B, 1, tmp, a.odd_all, fB);
        __syncwarp();
        for (int t = lane; t < n * B; t += 32) {
            const int k = t / B, x = t - k * B;
            fdct_any(g + k * plane + x, B, B, tmp, a.odd_all, fB);
        }
        __syncwarp();
        for (int t = lane; t < plane; t += 32) fdct_any(g + t, n, plane, tmp, a.odd_all, fn);
        __syncwarp();
    } else {
        for (int t = lane; t < plane; t += 32) idct_any(g + t, n, plane, tmp, a.odd_all, fn);
        __syncwarp();
        for (int t = lane; t < n * B; t += 32) {
            const int k = t / B, x = t - k * B;
            idct_any(g + k * plane + x, B, B, tmp, a.odd_all, fB);
        }
        __syncwarp();
        for (int t = lane; t < n * B; t += 32) idct_any(g + t * B, B, 1, tmp, a.odd_all, fB);
        __syncwarp();
    }
}

__global__ void __launch_bounds__(128) cf_generic_kernel(CFArgs a)
{
    const int lane = (int)lane_id();
    const long long warp_global = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
    float *g = a.scratch + warp_global * a.scratch_per_warp;
    const int B = a.B;
    const int plane = B * B;
    float *rg = g + (long long)a.G * plane;
    float tmp[512];

    for (long long grp = warp_global; grp < a.ngroups; grp += nwarps) {
        int n = a.count[grp];
        if (n > a.G) n = a.G;
        if (a.skip_full && n == a.G) continue;
        const int sz = n * plane;
        const uint32_t *pl = a.pos + grp * a.G;
        for (int p = 0; p < 3; ++p) {
            if (!a.process[p]) continue;
            for (int idx = lane; idx < sz; idx += 32) {
                const int k = idx / plane, e = idx - k * plane;
                const int y = e / B, x = e - y * B;
                const GroupLoc L = locate(a, p, grp, pl[k]);
                g[idx] = L.src[(long long)(L.y + y) * a.ld + L.x + x];
                if (a.wiener) rg[idx] = L.ref[(long long)(L.y + y) * a.ld + L.x + x];
            }
            __syncwarp();
            dct3d_warp(g, n, B, false, a, tmp);
            if (a.wiener) dct3d_warp(rg, n, B, false, a, tmp);
            int kept = 0;
            float l2 = 0.0f;
            for (int idx = lane; idx < sz; idx += 32) {
                const float v = g[idx];
                if (!a.wiener) {
                    const int k = idx / plane, e = idx - k * plane;
                    const int y = e / B, x = e - y * B;
                    const int flag = (x == 0) + (y == 0) + (k == 0);
                    const bool keep = fabsf(v) > a.thr4[p][n - 1][flag];
                    kept += keep;
                    g[idx] = keep ? v : 0.0f;
                } else {
                    const float r = rg[idx];
                    const float r2 = __fmul_rn(r, r);
                    const float w = __fdiv_rn(r2, __fadd_rn(r2, a.wsig2[p][n - 1]));
                    g[idx] = __fmul_rn(v, w);
                    l2 = __fadd_rn(l2, __fmul_rn(w, w));
                }
            }
            kept = warp_sum(kept);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) l2 = __fadd_rn(l2, __shfl_xor_sync(0xffffffffu, l2, o));
            __syncwarp();
            dct3d_warp(g, n, B, true, a, tmp);
            float denW;
            if (!a.wiener) denW = kept < 1 ? 1.0f : __fdiv_rn(1.0f, (float)kept);
            else {
                const float eps = 1.1920928955078125e-07f;
                denW = __fdiv_rn(1.0f, l2 > eps ? l2 : eps);
            }
            const float numW = __fdiv_rn(denW, a.amp[n - 1]);
            for (int idx = lane; idx < sz; idx += 32) {
                const int k = idx / plane, e = idx - k * plane;
                const int y = e / B, x = e - y * B;
                const GroupLoc L = locate(a, p, grp, pl[k]);
                atomicAdd(L.num + (long long)(L.y + y) * a.ld + L.x + x, __fmul_rn(g[idx], numW));
            }
            for (int k = lane; k < n; k += 32) {
                const GroupLoc L = locate(a, p, grp, pl[k]);
                atomicAdd(L.wmap + (long long)L.y * a.ld + L.x, denW);
            }
            __syncwarp();
        }
    }
}

}  // namespace bm3d
