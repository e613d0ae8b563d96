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

// ---- fast path: B = 8, groups of n <= G blocks, G in {8, 16, 32} ---------------------------------
// A warp works on 32/G groups at a time.  Lane = block for the 2-D transforms (registers); the
// transpose buffer T[32][kTP] (row = block, column = 2-D coefficient y*8+x) hands the coefficients
// to the z stage, where each lane takes 64/G columns.

constexpr int kTP = 65;   // padded row pitch: rows and columns are both bank-conflict free

// z stage of one coefficient column (stride kTP): forward DCT along z, hard threshold with t0
// (z == 0) / t1 (z > 0) (Basic) or multiplication by the Wiener weights in Wc (Final), inverse
// DCT along z, in place.  Returns the kept count (Basic) or the column's sum of squared weights
// (Final).
template <int G, bool WIENER>
__device__ __noinline__ float zstage_column(float *Tc, const float *Wc, float t0, float t1)
{
    float col[G], X[G];
#pragma unroll
    for (int zz = 0; zz < G; ++zz) col[zz] = Tc[zz * kTP];
    fdct_reg<G>(col, X);
    float r = 0.0f;
    if constexpr (!WIENER) {
        int k = 0;
#pragma unroll
        for (int zz = 0; zz < G; ++zz) {
            const float th = zz == 0 ? t0 : t1;
            const bool keep = fabsf(X[zz]) > th;
            k += keep;
            X[zz] = keep ? X[zz] : 0.0f;
        }
        r = (float)k;
    } else {
#pragma unroll
        for (int zz = 0; zz < G; ++zz) {
            const float w = Wc[zz * kTP];
            X[zz] = __fmul_rn(X[zz], w);
            r = __fadd_rn(r, __fmul_rn(w, w));
        }
    }
    idct_reg<G>(X, col);
#pragma unroll
    for (int zz = 0; zz < G; ++zz) Tc[zz * kTP] = col[zz];
    return r;
}

// Wiener weights of one reference-group column: forward DCT along z, then
// w = r^2 / (r^2 + sg) written back in place.
template <int G>
__device__ __noinline__ void wiener_column(float *Wc, float sg)
{
    float col[G], R[G];
#pragma unroll
    for (int zz = 0; zz < G; ++zz) col[zz] = Wc[zz * kTP];
    fdct_reg<G>(col, R);
#pragma unroll
    for (int zz = 0; zz < G; ++zz) {
        const float r2 = __fmul_rn(R[zz], R[zz]);
        Wc[zz * kTP] = __fdiv_rn(r2, __fadd_rn(r2, sg));
    }
}

// Non-power-of-two group length n (< G): direct FMA chains over the n x n tables (the oracle's
// fdct_direct / idct_direct), t[k][0] x[0] then fused multiply-adds over j = 1 .. n - 1 for every
// output k.  Eight outputs advance together, so that each step reads x[j] once (from shared
// memory) and runs eight independent chains; the arrays indexed by k (the spectrum, the outputs
// of the inverse) are touched O(n) times only.
constexpr int kDirectChains = 8;

// out_c[k] = sum_j t[k][j] x_c[j] for k < n and the two columns c of a lane, x_c[j] = in_c[j * kTP];
// the first term a product (forward tables) or the bare x_c[0] (inverse tables, t[k][0] = 1).
// Each table entry is loaded once for both columns.
__device__ __forceinline__ void direct_sums2(const float *in0, const float *in1, const float *t, int n, bool first_mul,
                                             float *out0, float *out1)
{
    for (int k0 = 0; k0 < n; k0 += kDirectChains) {
        const float *tk[kDirectChains];
#pragma unroll
        for (int i = 0; i < kDirectChains; ++i) tk[i] = t + min(k0 + i, n - 1) * n;
        float a0[kDirectChains], a1[kDirectChains];
        const float x0 = in0[0], y0 = in1[0];
#pragma unroll
        for (int i = 0; i < kDirectChains; ++i) {
            const float f = first_mul ? __ldg(tk[i]) : 1.0f;
            a0[i] = first_mul ? __fmul_rn(x0, f) : x0;
            a1[i] = first_mul ? __fmul_rn(y0, f) : y0;
        }
#pragma unroll 2
        for (int j = 1; j < n; ++j) {
            const float xj = in0[j * kTP], yj = in1[j * kTP];
#pragma unroll
            for (int i = 0; i < kDirectChains; ++i) {
                const float f = __ldg(tk[i] + j);
                a0[i] = __fmaf_rn(xj, f, a0[i]);
                a1[i] = __fmaf_rn(yj, f, a1[i]);
            }
        }
#pragma unroll
        for (int i = 0; i < kDirectChains; ++i)
            if (k0 + i < n) {
                out0[k0 + i] = a0[i];
                out1[k0 + i] = a1[i];
            }
    }
}

// hard threshold (t0: kz = 0, t1: the rest) or Wiener weights (W) of a spectrum of length n;
// returns the kept count or the sum of the squared weights, accumulated in kz order
template <bool WIENER>
__device__ __forceinline__ float shrink_direct(float *X, const float *W, float t0, float t1, int n)
{
    float r = 0.0f;
    if constexpr (!WIENER) {
        int kk = 0;
        for (int zz = 0; zz < n; ++zz) {
            const float th = zz == 0 ? t0 : t1;
            const bool keep = fabsf(X[zz]) > th;
            kk += keep;
            X[zz] = keep ? X[zz] : 0.0f;
        }
        r = (float)kk;
    } else {
        for (int zz = 0; zz < n; ++zz) {
            const float w = W[zz * kTP];
            X[zz] = __fmul_rn(X[zz], w);
            r = __fadd_rn(r, __fmul_rn(w, w));
        }
    }
    return r;
}

// the z stage of two columns of length n < G (forward, shrinkage, inverse; results in place);
// r[c] as shrink_direct's
template <bool WIENER>
__device__ __noinline__ void zstage_direct2(float *T0, float *T1, const float *W0, const float *W1, float t00, float t10,
                                            float t01, float t11, int n, const float *fwd, const float *inv, float *r)
{
    float X0[32], X1[32];
    direct_sums2(T0, T1, fwd, n, true, X0, X1);
    r[0] = shrink_direct<WIENER>(X0, W0, t00, t10, n);
    r[1] = shrink_direct<WIENER>(X1, W1, t01, t11, n);
    // the spectra go back into the columns, the inverse reads them from there
    for (int zz = 0; zz < n; ++zz) {
        T0[zz * kTP] = X0[zz];
        T1[zz * kTP] = X1[zz];
    }
    direct_sums2(T0, T1, inv, n, false, X0, X1);
    for (int k = 0; k < n; ++k) {
        T0[k * kTP] = X0[k];
        T1[k * kTP] = X1[k];
    }
}

// Wiener weights of two columns of length n < G (direct sums as above), written back in place
__device__ __noinline__ void wiener_direct2(float *W0, float *W1, float sg, int n, const float *fwd)
{
    float X0[32], X1[32];
    direct_sums2(W0, W1, fwd, n, true, X0, X1);
    for (int k = 0; k < n; ++k) {
        const float r0 = __fmul_rn(X0[k], X0[k]), r1 = __fmul_rn(X1[k], X1[k]);
        W0[k * kTP] = __fdiv_rn(r0, __fadd_rn(r0, sg));
        W1[k * kTP] = __fdiv_rn(r1, __fadd_rn(r1, sg));
    }
}

// lengths the unrolled column transforms handle; the rest take the direct sums
template <int G>
__device__ __forceinline__ bool direct_length(int n)
{
    return !(n == G || (G > 16 && n == 16) || (G > 8 && n == 8) || n == 4 || n == 2 || n == 1);
}

template <int G, bool WIENER>
__device__ __forceinline__ float zstage_any(float *Tc, const float *Wc, float t0, float t1, int n, const float *fwd,
                                            const float *inv)
{
    if (n == G) return zstage_column<G, WIENER>(Tc, Wc, t0, t1);
    if (G > 16 && n == 16) return zstage_column<(G > 16 ? 16 : 1), WIENER>(Tc, Wc, t0, t1);
    if (G > 8 && n == 8) return zstage_column<(G > 8 ? 8 : 1), WIENER>(Tc, Wc, t0, t1);
    if (n == 4) return zstage_column<4, WIENER>(Tc, Wc, t0, t1);
    if (n == 2) return zstage_column<2, WIENER>(Tc, Wc, t0, t1);
    return zstage_column<1, WIENER>(Tc, Wc, t0, t1);   // n == 1 (direct lengths go in pairs)
}

template <int G>
__device__ __forceinline__ void wiener_any(float *Wc, float sg, int n, const float *fwd)
{
    if (n == G) wiener_column<G>(Wc, sg);
    else if (G > 16 && n == 16) wiener_column<(G > 16 ? 16 : 1)>(Wc, sg);
    else if (G > 8 && n == 8) wiener_column<(G > 8 ? 8 : 1)>(Wc, sg);
    else if (n == 4) wiener_column<4>(Wc, sg);
    else if (n == 2) wiener_column<2>(Wc, sg);
    else wiener_column<1>(Wc, sg);   // n == 1 (direct lengths go in pairs)
}

__device__ __forceinline__ const float *dtab_for(const CFArgs &a, int N, bool inverse)
{
    const int off = a.dtab_off[N];
    return off < 0 ? nullptr : a.dtab + off + (inverse ? N * N : 0);
}

// Indices of the groups with fewer than G blocks (the ones the tensor-core filter leaves), in any
// order (their aggregation is order-free atomics): one warp-aggregated atomic per warp step.
__global__ void cf_partial_list_kernel(const int *__restrict__ count, long long ngroups, int G, long long *__restrict__ list,
                                       unsigned int *__restrict__ n)
{
    const int lane = (int)lane_id();
    for (long long g0 = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); g0 < ngroups;
         g0 += (long long)gridDim.x * blockDim.x) {
        const long long g = g0 + lane;
        const bool part = g < ngroups && count[g] < G;
        const unsigned m = __ballot_sync(0xffffffffu, part);
        unsigned base = 0;
        if (lane == 0 && m) base = atomicAdd(n, (unsigned)__popc(m));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (part) list[base + __popc(m & ((1u << lane) - 1u))] = g;
    }
}

// The collaborative-filter kernel: per-lane gathers straight into registers, register-resident
// 2-D transforms, the z stage inline for full groups (out-of-line calls only for the rare partial
// groups), and per-lane global float atomics into the numerator and per-origin weight planes.
// Shared memory holds only the transpose buffers (T, and T2 for the Wiener weights).  Measured on
// B200 against two alternatives -- a shared-memory tile accumulator per CTA and fully out-of-line
// stages with coalesced gathers -- this layout was the fastest: occupancy and latency hiding
// matter more here than atomic traffic.
__device__ __forceinline__ void load_block8(float (&blk)[64], const float *sp, int ld)
{
#pragma unroll
    for (int y = 0; y < 8; ++y)
#pragma unroll
        for (int x = 0; x < 8; ++x) blk[y * 8 + x] = __ldg(sp + (long long)y * ld + x);
}

template <int G, bool WIENER>
__global__ void __launch_bounds__(128) cf_fast_kernel(CFArgs a)
{
    constexpr int GPW = 32 / G;
    constexpr int C = 64 / G;
    extern __shared__ float smem[];
    const int lane = (int)lane_id();
    const int warp = threadIdx.x >> 5;
    const int nwarp = blockDim.x >> 5;
    const int sub = lane / G;
    const int z = lane - sub * G;
    float *T = smem + warp * (WIENER ? 2 : 1) * 32 * kTP;
    float *T2 = T + 32 * kTP;

    const long long nwarps = (long long)gridDim.x * nwarp;
    // with a partial-group list the warps walk the list, else every group.  With one group per
    // warp, each plane of a listed group is a slot of its own: the list is short (the groups the
    // tensor-core kernel left) and its groups are slow (direct sums of any length), so three
    // times the warps share it.
    constexpr bool kPlaneSlots = GPW == 1;
    const bool split = a.plist && kPlaneSlots;
    const long long nitems = a.plist ? (long long)*a.plist_n * (split ? 3 : 1) : a.ngroups;
    for (long long wg = (long long)blockIdx.x * nwarp + warp; wg * GPW < nitems; wg += nwarps) {
        const long long item = wg * GPW + sub;
        const bool inrange = item < nitems;
        const int pslot = split ? (int)(item % 3) : -1;
        const long long grp = a.plist ? (inrange ? a.plist[split ? item / 3 : item] : 0) : item;
        const long long g0 = inrange ? grp : 0;
        const int n = min(a.count[g0], G);
        // skip_full: full groups were filtered by the tensor-core kernel; only partial ones here
        const bool taken = a.skip_full && n == G;
        if (__all_sync(0xffffffffu, taken || !inrange)) continue;
        const bool active = inrange && z < n && !taken;
        const bool full = __all_sync(0xffffffffu, n == G);
        const uint32_t pk = a.pos[g0 * G + min(z, n - 1)];
        for (int p = 0; p < 3; ++p) {
            if (!a.process[p] || (pslot >= 0 && p != pslot)) continue;
            const GroupLoc L = locate(a, p, g0, pk);
            float blk[64];
            if constexpr (WIENER) {
                load_block8(blk, L.ref + (long long)L.y * a.ld + L.x, a.ld);
                fwd2d8(blk);
#pragma unroll
                for (int e = 0; e < 64; ++e) T2[lane * kTP + e] = blk[e];
                __syncwarp();
                const float sg = a.wsig2[p][n - 1];
                if (full) {
#pragma unroll 1
                    for (int q = 0; q < C; ++q) {
                        float *Wc = T2 + sub * G * kTP + z + q * G;
                        float col[G], R[G];
#pragma unroll
                        for (int zz = 0; zz < G; ++zz) col[zz] = Wc[zz * kTP];
                        fdct_reg<G>(col, R);
#pragma unroll
                        for (int zz = 0; zz < G; ++zz) {
                            const float r2 = __fmul_rn(R[zz], R[zz]);
                            Wc[zz * kTP] = __fdiv_rn(r2, __fadd_rn(r2, sg));
                        }
                    }
                } else {
                    const float *fwd = n == G ? nullptr : dtab_for(a, n, false);
                    if (direct_length<G>(n)) {
#pragma unroll 1
                        for (int q = 0; q < C; q += 2)
                            wiener_direct2(T2 + sub * G * kTP + z + q * G, T2 + sub * G * kTP + z + (q + 1) * G, sg, n, fwd);
                    } else {
#pragma unroll 1
                        for (int q = 0; q < C; ++q) wiener_any<G>(T2 + sub * G * kTP + z + q * G, sg, n, fwd);
                    }
                }
                __syncwarp();
            }
            load_block8(blk, L.src + (long long)L.y * a.ld + L.x, a.ld);
            fwd2d8(blk);
#pragma unroll
            for (int e = 0; e < 64; ++e) T[lane * kTP + e] = blk[e];
            __syncwarp();
            int kept = 0;
            float l2 = 0.0f;
            if (full) {
#pragma unroll 1
                for (int q = 0; q < C; ++q) {
                    const int c = z + q * G;
                    float *Tc = T + sub * G * kTP + c;
                    float col[G], X[G];
#pragma unroll
                    for (int zz = 0; zz < G; ++zz) col[zz] = Tc[zz * kTP];
                    fdct_reg<G>(col, X);
                    if constexpr (!WIENER) {
                        const int fxy = ((c & 7) == 0) + ((c >> 3) == 0);
                        const float t0 = a.thr4[p][G - 1][fxy + 1];
                        const float t1 = a.thr4[p][G - 1][fxy];
#pragma unroll
                        for (int zz = 0; zz < G; ++zz) {
                            const float th = zz == 0 ? t0 : t1;
                            const bool keep = fabsf(X[zz]) > th;
                            kept += keep;
                            X[zz] = keep ? X[zz] : 0.0f;
                        }
                    } else {
                        const float *Wc = T2 + sub * G * kTP + c;
#pragma unroll
                        for (int zz = 0; zz < G; ++zz) {
                            const float w = Wc[zz * kTP];
                            X[zz] = __fmul_rn(X[zz], w);
                            l2 = __fadd_rn(l2, __fmul_rn(w, w));
                        }
                    }
                    idct_reg<G>(X, col);
#pragma unroll
                    for (int zz = 0; zz < G; ++zz) Tc[zz * kTP] = col[zz];
                }
            } else {
                const float *fwd = dtab_for(a, n, false);
                const float *inv = dtab_for(a, n, true);
                if (direct_length<G>(n)) {
                    // a length without an unrolled transform: the direct sums, two columns at a time
#pragma unroll 1
                    for (int q = 0; q < C; q += 2) {
                        const int ca = z + q * G, cb = ca + G;
                        const int fa = ((ca & 7) == 0) + ((ca >> 3) == 0), fb = ((cb & 7) == 0) + ((cb >> 3) == 0);
                        float r[2];
                        float *c0 = T + sub * G * kTP + ca;
                        const float *w0 = WIENER ? T2 + sub * G * kTP + ca : nullptr;
                        zstage_direct2<WIENER>(c0, c0 + G, w0, WIENER ? w0 + G : nullptr,
                                               WIENER ? 0.0f : a.thr4[p][n - 1][fa + 1], WIENER ? 0.0f : a.thr4[p][n - 1][fa],
                                               WIENER ? 0.0f : a.thr4[p][n - 1][fb + 1], WIENER ? 0.0f : a.thr4[p][n - 1][fb],
                                               n, fwd, inv, r);
                        if constexpr (!WIENER) kept += (int)r[0] + (int)r[1];
                        else l2 = __fadd_rn(__fadd_rn(l2, r[0]), r[1]);
                    }
                } else {
#pragma unroll 1
                    for (int q = 0; q < C; ++q) {
                        const int c = z + q * G;
                        const int fxy = ((c & 7) == 0) + ((c >> 3) == 0);
                        const float t0 = WIENER ? 0.0f : a.thr4[p][n - 1][fxy + 1];
                        const float t1 = WIENER ? 0.0f : a.thr4[p][n - 1][fxy];
                        const float r = zstage_any<G, WIENER>(T + sub * G * kTP + c, WIENER ? T2 + sub * G * kTP + c : nullptr,
                                                              t0, t1, n, nullptr, nullptr);
                        if constexpr (!WIENER) kept += (int)r;
                        else l2 = __fadd_rn(l2, r);
                    }
                }
            }
#pragma unroll
            for (int o = G / 2; o > 0; o >>= 1) {
                if constexpr (!WIENER) kept += __shfl_xor_sync(0xffffffffu, kept, o);
                else l2 = __fadd_rn(l2, __shfl_xor_sync(0xffffffffu, l2, o));
            }
            if constexpr (!WIENER)
                if (a.retained && inrange && !taken && z == 0) a.retained[(long long)p * a.ngroups + g0] = kept;
            __syncwarp();
#pragma unroll
            for (int e = 0; e < 64; ++e) blk[e] = T[lane * kTP + e];
            __syncwarp();
            inv2d8(blk);
            float denW;
            if constexpr (!WIENER) {
                denW = kept < 1 ? 1.0f : __fdiv_rn(1.0f, (float)kept);
            } else {
                const float eps = 1.1920928955078125e-07f;
                denW = __fdiv_rn(1.0f, l2 > eps ? l2 : eps);
            }
            const float numW = __fdiv_rn(denW, a.amp[n - 1]);
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

// The warp's 32 blocks (lane i's block at sp of lane i) into rows i of S (pitch kTP), one block per
// step with lane = (row, column) of the block: each load instruction touches one block's 4 rows
// instead of 32 blocks, which is what the memory system can serve.  Then every lane reads its own
// row back into registers.
__device__ __forceinline__ void gather_blocks8(float (&blk)[64], float *S, const float *sp, int ld, int lane)
{
    const int ry = lane >> 3, cx = lane & 7;
#pragma unroll 4
    for (int i = 0; i < 32; ++i) {
        const float *q = reinterpret_cast<const float *>(__shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(sp), i));
        S[i * kTP + lane] = __ldg(q + (long long)ry * ld + cx);
        S[i * kTP + 32 + lane] = __ldg(q + (long long)(ry + 4) * ld + cx);
    }
    __syncwarp();
#pragma unroll
    for (int e = 0; e < 64; ++e) blk[e] = S[lane * kTP + e];
    __syncwarp();
}

// The run kernel, for the Final estimate over all groups of a BM3D frame: a run of kCfRunGroups
// consecutive groups (consecutive reference blocks of one row) per CTA, one warp per G-group slot.  The blocks a run adds lie in one box of the
// image (the search windows of its reference blocks); in region mode the run adds them into that
// box in shared memory, in 64-bit fixed point (native integer atomics: shared-memory float
// atomics are emulated), and flushes the box to the numerator plane once per plane with one
// vector atomic per 4 pixels.  Flushing per run rather than per few groups matters: global
// atomics on pixels that many neighbouring runs cover serialise at the L2.
// Eight warps per CTA and one CTA per SM: the Final's two transpose buffers per warp and the box
// fill the shared memory.  Measured on B200 for the Basic estimate (fewer, lighter overlaps) and
// for the partial groups of the precision form (few active warps per run), the per-lane kernel
// above is faster, so those keep it.
constexpr int kCfWarps = 8;
constexpr int kCfRunGroups = 32;
constexpr int kCfCells = 7168;                 // int64 cells of the box (57 KB)
constexpr float kCfFix = 4294967296.0f;        // 2^32: fixed-point scale of the box
constexpr float kCfUnfix = 2.3283064365386963e-10f;   // 2^-32
// Terms at or above 2^19 go to the plane directly: a pixel takes at most 32 groups x 64 block
// positions = 2^11 terms per run, so the box sums stay below 2^62 in fixed point.
constexpr float kCfFixMax = 524288.0f;

template <int G, bool WIENER>
__global__ void __launch_bounds__(kCfWarps * 32, 1) cf_run_kernel(CFArgs a)
{
    constexpr int GPW = 32 / G;
    constexpr int C = 64 / G;
    constexpr int TPG = kCfWarps * GPW;                         // groups per pass of the warps
    constexpr int RUN = kCfRunGroups / TPG > 0 ? kCfRunGroups / TPG : 1;   // passes per run
    extern __shared__ float smem[];
    const int lane = (int)lane_id();
    const int warp = threadIdx.x >> 5;
    const int sub = lane / G;
    const int z = lane - sub * G;
    float *T = smem + warp * (WIENER ? 2 : 1) * 32 * kTP;
    float *T2 = T + 32 * kTP;
    unsigned long long *Rq = reinterpret_cast<unsigned long long *>(smem + kCfWarps * (WIENER ? 2 : 1) * 32 * kTP);
    int *rb = reinterpret_cast<int *>(Rq + kCfCells);            // [warp][8] bounds
    for (int e = threadIdx.x; e < kCfCells; e += blockDim.x) Rq[e] = 0ull;
    __syncthreads();
    const int ry = lane >> 3, cx = lane & 7;

    for (long long run = blockIdx.x; run * RUN * TPG < a.ngroups; run += gridDim.x) {
        // bounds of the blocks the run adds
        int y0 = 0, x0 = 0, rh = 0, rw = 0, rp = 0, frame = 0;
        bool region = false;
        if (!a.skip_full && !a.vbm3d) {
            int v[6] = {1 << 30, 1 << 30, -1, -1, 1 << 30, -1};
            for (int t = 0; t < RUN; ++t) {
                const long long grp = ((run * RUN + t) * kCfWarps + warp) * GPW + sub;
                if (grp >= a.ngroups) continue;
                const int n = min(a.count[grp], G);
                if (z >= n) continue;
                const uint32_t pk = a.pos[grp * G + z];
                const int py = unpack_y(pk), px = unpack_x(pk), f = (int)(grp / a.blocks_per_frame);
                v[0] = min(v[0], py); v[1] = min(v[1], px); v[2] = max(v[2], py); v[3] = max(v[3], px);
                v[4] = min(v[4], f); v[5] = max(v[5], f);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                v[0] = min(v[0], __shfl_xor_sync(0xffffffffu, v[0], o));
                v[1] = min(v[1], __shfl_xor_sync(0xffffffffu, v[1], o));
                v[2] = max(v[2], __shfl_xor_sync(0xffffffffu, v[2], o));
                v[3] = max(v[3], __shfl_xor_sync(0xffffffffu, v[3], o));
                v[4] = min(v[4], __shfl_xor_sync(0xffffffffu, v[4], o));
                v[5] = max(v[5], __shfl_xor_sync(0xffffffffu, v[5], o));
            }
            if (lane == 0)
                for (int k = 0; k < 6; ++k) rb[warp * 8 + k] = v[k];
            __syncthreads();
            for (int w = 0; w < kCfWarps; ++w) {
                v[0] = min(v[0], rb[w * 8]); v[1] = min(v[1], rb[w * 8 + 1]);
                v[2] = max(v[2], rb[w * 8 + 2]); v[3] = max(v[3], rb[w * 8 + 3]);
                v[4] = min(v[4], rb[w * 8 + 4]); v[5] = max(v[5], rb[w * 8 + 5]);
            }
            __syncthreads();
            if (v[2] >= 0 && v[4] == v[5]) {
                y0 = v[0];
                x0 = v[1] & ~3;
                rh = v[2] + 8 - v[0];
                rw = min((v[3] + 8 - x0 + 3) & ~3, a.ld - x0);    // whole 16-byte chunks within the row
                rp = rw + ((24 - (rw & 15)) & 15);    // pitch = 8 mod 16 cells: 2 wavefronts per block step
                region = rh * rp <= kCfCells;
                frame = v[4];
            }
        }
        for (int p = 0; p < 3; ++p) {
            if (!a.process[p]) continue;
            for (int t = 0; t < RUN; ++t) {
                const long long grp = ((run * RUN + t) * kCfWarps + warp) * GPW + sub;
                const bool inrange = grp < a.ngroups;
                const long long g0 = inrange ? grp : 0;
                const int n = min(a.count[g0], G);
                // skip_full: full groups were filtered by the tensor-core kernel; only partial ones here
                const bool taken = a.skip_full && n == G;
                const bool skipw = __all_sync(0xffffffffu, taken || !inrange);
                const bool active = inrange && z < n && !taken;
                const bool full = __all_sync(0xffffffffu, n == G);
                const uint32_t pk = a.pos[g0 * G + min(z, n - 1)];
                const GroupLoc L = locate(a, p, g0, pk);
                float blk[64];
                float denW = 0.0f;
                if (!skipw) {
                if constexpr (WIENER) {
                    gather_blocks8(blk, T2, L.ref + (long long)L.y * a.ld + L.x, a.ld, lane);
                    fwd2d8(blk);
    #pragma unroll
                    for (int e = 0; e < 64; ++e) T2[lane * kTP + e] = blk[e];
                    __syncwarp();
                    const float sg = a.wsig2[p][n - 1];
                    if (full) {
    #pragma unroll 1
                        for (int q = 0; q < C; ++q) {
                            float *Wc = T2 + sub * G * kTP + z + q * G;
                            float col[G], R[G];
    #pragma unroll
                            for (int zz = 0; zz < G; ++zz) col[zz] = Wc[zz * kTP];
                            fdct_reg<G>(col, R);
    #pragma unroll
                            for (int zz = 0; zz < G; ++zz) {
                                const float r2 = __fmul_rn(R[zz], R[zz]);
                                Wc[zz * kTP] = __fdiv_rn(r2, __fadd_rn(r2, sg));
                            }
                        }
                    } else {
                        const float *fwd = n == G ? nullptr : dtab_for(a, n, false);
                        if (direct_length<G>(n)) {
#pragma unroll 1
                            for (int q = 0; q < C; q += 2)
                                wiener_direct2(T2 + sub * G * kTP + z + q * G, T2 + sub * G * kTP + z + (q + 1) * G, sg, n, fwd);
                        } else {
#pragma unroll 1
                            for (int q = 0; q < C; ++q) wiener_any<G>(T2 + sub * G * kTP + z + q * G, sg, n, fwd);
                        }
                    }
                    __syncwarp();
                }
                gather_blocks8(blk, T, L.src + (long long)L.y * a.ld + L.x, a.ld, lane);
                fwd2d8(blk);
    #pragma unroll
                for (int e = 0; e < 64; ++e) T[lane * kTP + e] = blk[e];
                __syncwarp();
                int kept = 0;
                float l2 = 0.0f;
                if (full) {
    #pragma unroll 1
                    for (int q = 0; q < C; ++q) {
                        const int c = z + q * G;
                        float *Tc = T + sub * G * kTP + c;
                        float col[G], X[G];
    #pragma unroll
                        for (int zz = 0; zz < G; ++zz) col[zz] = Tc[zz * kTP];
                        fdct_reg<G>(col, X);
                        if constexpr (!WIENER) {
                            const int fxy = ((c & 7) == 0) + ((c >> 3) == 0);
                            const float t0 = a.thr4[p][G - 1][fxy + 1];
                            const float t1 = a.thr4[p][G - 1][fxy];
    #pragma unroll
                            for (int zz = 0; zz < G; ++zz) {
                                const float th = zz == 0 ? t0 : t1;
                                const bool keep = fabsf(X[zz]) > th;
                                kept += keep;
                                X[zz] = keep ? X[zz] : 0.0f;
                            }
                        } else {
                            const float *Wc = T2 + sub * G * kTP + c;
    #pragma unroll
                            for (int zz = 0; zz < G; ++zz) {
                                const float w = Wc[zz * kTP];
                                X[zz] = __fmul_rn(X[zz], w);
                                l2 = __fadd_rn(l2, __fmul_rn(w, w));
                            }
                        }
                        idct_reg<G>(X, col);
    #pragma unroll
                        for (int zz = 0; zz < G; ++zz) Tc[zz * kTP] = col[zz];
                    }
                } else {
                    const float *fwd = dtab_for(a, n, false);
                    const float *inv = dtab_for(a, n, true);
                    if (direct_length<G>(n)) {
                        // a length without an unrolled transform: the direct sums, two columns at a time
#pragma unroll 1
                        for (int q = 0; q < C; q += 2) {
                            const int ca = z + q * G, cb = ca + G;
                            const int fa = ((ca & 7) == 0) + ((ca >> 3) == 0), fb = ((cb & 7) == 0) + ((cb >> 3) == 0);
                            float r[2];
                            float *c0 = T + sub * G * kTP + ca;
                            const float *w0 = WIENER ? T2 + sub * G * kTP + ca : nullptr;
                            zstage_direct2<WIENER>(c0, c0 + G, w0, WIENER ? w0 + G : nullptr,
                                                   WIENER ? 0.0f : a.thr4[p][n - 1][fa + 1], WIENER ? 0.0f : a.thr4[p][n - 1][fa],
                                                   WIENER ? 0.0f : a.thr4[p][n - 1][fb + 1], WIENER ? 0.0f : a.thr4[p][n - 1][fb],
                                                   n, fwd, inv, r);
                            if constexpr (!WIENER) kept += (int)r[0] + (int)r[1];
                            else l2 = __fadd_rn(__fadd_rn(l2, r[0]), r[1]);
                        }
                    } else {
#pragma unroll 1
                        for (int q = 0; q < C; ++q) {
                            const int c = z + q * G;
                            const int fxy = ((c & 7) == 0) + ((c >> 3) == 0);
                            const float t0 = WIENER ? 0.0f : a.thr4[p][n - 1][fxy + 1];
                            const float t1 = WIENER ? 0.0f : a.thr4[p][n - 1][fxy];
                            const float r = zstage_any<G, WIENER>(T + sub * G * kTP + c, WIENER ? T2 + sub * G * kTP + c : nullptr,
                                                                  t0, t1, n, nullptr, nullptr);
                            if constexpr (!WIENER) kept += (int)r;
                            else l2 = __fadd_rn(l2, r);
                        }
                    }
                }
    #pragma unroll
                for (int o = G / 2; o > 0; o >>= 1) {
                    if constexpr (!WIENER) kept += __shfl_xor_sync(0xffffffffu, kept, o);
                    else l2 = __fadd_rn(l2, __shfl_xor_sync(0xffffffffu, l2, o));
                }
                __syncwarp();
    #pragma unroll
                for (int e = 0; e < 64; ++e) blk[e] = T[lane * kTP + e];
                __syncwarp();
                inv2d8(blk);
                if constexpr (!WIENER) {
                    denW = kept < 1 ? 1.0f : __fdiv_rn(1.0f, (float)kept);
                } else {
                    const float eps = 1.1920928955078125e-07f;
                    denW = __fdiv_rn(1.0f, l2 > eps ? l2 : eps);
                }
                const float numW = __fdiv_rn(denW, a.amp[n - 1]);
    #pragma unroll
                for (int e = 0; e < 64; ++e) T[lane * kTP + e] = __fmul_rn(blk[e], numW);
                __syncwarp();
                }   // !skipw
                // aggregation one block per step (lane = pixel row / column), as for the gathers
                if (!skipw) {
                    if (region) {
#pragma unroll 4
                        for (int i = 0; i < 32; ++i) {
                            const bool ai = __shfl_sync(0xffffffffu, active, i);
                            const uint32_t pi = __shfl_sync(0xffffffffu, pk, i);
                            if (ai) {
                                const int by = unpack_y(pi) - y0, bx = unpack_x(pi) - x0;
#pragma unroll
                                for (int h = 0; h < 2; ++h) {
                                    const float val = T[i * kTP + 32 * h + lane];
                                    const int yy = by + ry + 4 * h, xx = bx + cx;
                                    if (fabsf(val) < kCfFixMax)
                                        atomicAdd(Rq + yy * rp + xx, (unsigned long long)__float2ll_rn(val * kCfFix));
                                    else
                                        atomicAdd(a.num[p] + (long long)frame * a.frame_stride + (long long)(y0 + yy) * a.ld + x0 + xx, val);
                                }
                            }
                        }
                    } else {
                        float *np = L.num + (long long)L.y * a.ld + L.x;
#pragma unroll 4
                        for (int i = 0; i < 32; ++i) {
                            const bool ai = __shfl_sync(0xffffffffu, active, i);
                            float *q = reinterpret_cast<float *>(__shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(np), i));
                            if (ai) {
                                atomicAdd(q + (long long)ry * a.ld + cx, T[i * kTP + lane]);
                                atomicAdd(q + (long long)(ry + 4) * a.ld + cx, T[i * kTP + 32 + lane]);
                            }
                        }
                    }
                }
                __syncwarp();
                if (active) atomicAdd(L.wmap + (long long)L.y * a.ld + L.x, denW);
            }
            if (region) {
                // the box to the numerator plane, then cleared for the next plane / run
                __syncthreads();
                float *nbase = a.num[p] + (long long)frame * a.frame_stride + (long long)y0 * a.ld + x0;
                // two cells per thread: one 16-byte shared load per lane, contiguous across the warp
                const int nv = rh * (rw >> 1);
                for (int e = threadIdx.x; e < nv; e += blockDim.x) {
                    const int yy = e / (rw >> 1), c2 = e - yy * (rw >> 1);
                    ulonglong2 *cell = reinterpret_cast<ulonglong2 *>(Rq + yy * rp + 2 * c2);
                    const ulonglong2 q = *cell;
                    if (q.x | q.y) {
                        atomicAdd(reinterpret_cast<float2 *>(nbase + (long long)yy * a.ld + 2 * c2),
                                  make_float2(__ll2float_rn((long long)q.x) * kCfUnfix, __ll2float_rn((long long)q.y) * kCfUnfix));
                        *cell = make_ulonglong2(0ull, 0ull);
                    }
                }
                __syncthreads();
            }
        }
    }
}

// ---- generic path: any B <= 64, any n <= 256; one warp per group, data in global scratch ----

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
