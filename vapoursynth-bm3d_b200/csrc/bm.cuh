// bm.cuh -- K1: full-search block matching of every reference block (BM3D, and the current
// frame of V-BM3D).
//
// Replaces Block::BlockMatchingMulti, range form (include/Block.h:683-729, core :554-653) as
// called by BM3D_Process_Base::BlockMatching (source/BM3D_Base.cpp:473-490).  Semantics kept:
//   * the search lattice is the window of SearchBoundary (include/Block.h:734-769) in raster
//     order (y outer, x inner) without the reference block itself, followed by one extra
//     candidate at (0, 0): the reference sizes its position list for the full lattice and skips
//     self while filling it, so the last slot keeps a default-constructed Pos(0, 0);
//   * SSD summed exactly as the SSE2 build does (four lane sums over the 8-column chunks of
//     every row, lane l taking column c+l then c+4+l, combined ((s0+s1)+s2)+s3, then the
//     B%8 leftover columns added one by one);
//   * a candidate is kept iff dist <= thSSE and dist != 0, with key float(double(dist)*distMul);
//   * the reference block is pinned first (key 0); the rest is partial_sort-ed when more than
//     group_size-1 candidates survive, stable_sort-ed otherwise (see select.cuh).
//
// Layout: one warp per reference block, WARPS warps per CTA along a row of reference blocks.
// The CTA stages the union of its search windows in shared memory once; each warp keeps its
// reference block in registers and writes one distance per lattice position into its own
// shared-memory slice, then selects.
#pragma once

#include "select.cuh"
#include "args.h"
#include "tc.cuh"

namespace bm3d {


// Block::_SearchBoundary (include/Block.h:734-764) in closed form.
__host__ __device__ __forceinline__ int search_boundary(int pos, int plane_boundary, int range, int step)
{
    range = range / step * step;
    if (pos == plane_boundary) return plane_boundary;
    if (pos > plane_boundary) {
        int b = pos - range;
        if (b < plane_boundary) b += (plane_boundary - b + step - 1) / step * step;
        return b;
    }
    int b = pos + range;
    if (b > plane_boundary) b -= (b - plane_boundary + step - 1) / step * step;
    return b;
}

__device__ __forceinline__ float dist_to_key(float d, double distMul)
{
    return __double2float_rn(__dmul_rn((double)d, distMul));
}

__device__ __forceinline__ bool dist_valid(float d, float thSSE) { return d <= thSSE && d != 0.0f; }

// Per-warp selection over sd[0..ctot) (distances in scan order).  Writes the final list for one
// reference block.  `pos_of(c)` maps a scan index to a packed position.
template <typename PosOf>
__device__ void select_and_emit(float *sd, int ctot, uint32_t *list, float *hk, int *hi,
                                const BMArgs &a, uint32_t ref_pos, size_t ob, PosOf pos_of)
{
    const int lane = (int)lane_id();
    const int G = a.G;
    const int K = G - 1;
    uint32_t *opos = a.out_pos + ob * G;
    float *okey = a.out_key ? a.out_key + ob * G : nullptr;

    // count valid candidates and keep each lane's two best (dist, index) composites.  Lane l
    // takes element (l + 7 k) mod 32 of round k: with the plain stride the best candidates of a
    // smooth window (a compact patch around the reference position) fall on few lanes, so that
    // two per lane would often not cover the top group_size
    int cnt = 0;
    uint64_t b1 = ~0ull, b2 = ~0ull;
    for (int c0 = 0; c0 < ctot; c0 += 32) {
        const int c = c0 + ((lane + 7 * (c0 >> 5)) & 31);
        if (c >= ctot) continue;
        const float d = sd[c];
        if (dist_valid(d, a.thSSE)) {
            ++cnt;
            const uint64_t v = compose(d, (uint32_t)c);
            if (v < b1) { b2 = b1; b1 = v; } else if (v < b2) { b2 = v; }
        }
    }
    const int nvalid = warp_sum(cnt);
    const unsigned lt = (1u << lane) - 1u;

    if (lane == 0) {
        opos[0] = ref_pos;
        if (okey) okey[0] = 0.0f;
    }

    bool slow = G > 32;
    if (!slow) {
        if (nvalid <= K) {
            // stable_sort branch: every valid candidate, ordered by (key, scan index)
            int base = 0;
            for (int c0 = 0; c0 < ctot; c0 += 32) {
                const int c = c0 + lane;
                const bool ok = c < ctot && dist_valid(sd[c], a.thSSE);
                const unsigned m = __ballot_sync(0xffffffffu, ok);
                if (ok) list[base + __popc(m & lt)] = (uint32_t)c;
                base += __popc(m);
            }
            __syncwarp();
            uint64_t v[1];
            v[0] = ~0ull;
            if (lane < nvalid) {
                const uint32_t c = list[lane];
                v[0] = compose(dist_to_key(sd[c], a.distMul), c);
            }
            warp_bitonic_u64<1>(v);
            if (lane < nvalid) {
                const uint32_t c = (uint32_t)v[0];
                opos[1 + lane] = pos_of(c);
                if (okey) okey[1 + lane] = __uint_as_float((uint32_t)(v[0] >> 32));
            }
            if (lane == 0) a.out_n[ob] = 1 + nvalid;
            return;
        }
        // partial_sort branch, fast path
        uint64_t v[2] = {b1, b2};
        warp_bitonic_u64<2>(v);
        const uint64_t T = __shfl_sync(0xffffffffu, v[0], K);
        int m = 0;
        for (int c0 = 0; c0 < ctot; c0 += 32) {
            const int c = c0 + lane;
            bool ok = false;
            if (c < ctot) {
                const float d = sd[c];
                ok = dist_valid(d, a.thSSE) && compose(d, (uint32_t)c) <= T;
            }
            const unsigned msk = __ballot_sync(0xffffffffu, ok);
            if (ok && m + __popc(msk & lt) < 64) list[m + __popc(msk & lt)] = (uint32_t)c;
            m += __popc(msk);
        }
        __syncwarp();
        if (m <= 64) {
            v[0] = ~0ull;
            v[1] = ~0ull;
            if (lane < m) v[0] = compose(sd[list[lane]], list[lane]);
            if (lane + 32 < m) v[1] = compose(sd[list[lane + 32]], list[lane + 32]);
            warp_bitonic_u64<2>(v);
            // ranks 0..K sit in v[0] of lanes 0..K
            const uint32_t c = (uint32_t)v[0];
            const float key = lane <= K ? dist_to_key(__uint_as_float((uint32_t)(v[0] >> 32)), a.distMul) : 0.0f;
            const float prev = __shfl_up_sync(0xffffffffu, key, 1);
            const bool bad = lane >= 1 && lane <= K && !(prev < key);
            if (!__any_sync(0xffffffffu, bad)) {
                if (lane < K) {
                    opos[1 + lane] = pos_of(c);
                    if (okey) okey[1 + lane] = key;
                }
                if (lane == 0) a.out_n[ob] = G;
                return;
            }
        }
        slow = true;
    }

    // exact path: keys for every candidate (invalid -> -1), then one lane runs the reference's
    // heap-select + sort-heap (or the stable insertion sort) over the scan-ordered array
    for (int c = lane; c < ctot; c += 32) {
        const float d = sd[c];
        sd[c] = dist_valid(d, a.thSSE) ? dist_to_key(d, a.distMul) : -1.0f;
    }
    __syncwarp();
    if (lane == 0) {
        if (a.stats) atomicAdd(a.stats, 1ull);
        int n;
        if (nvalid <= K) {
            n = 0;
            for (int c = 0; c < ctot; ++c)
                if (sd[c] >= 0.0f) { hk[n] = sd[c]; hi[n] = c; ++n; }
            stable_sort_keys(hk, hi, n);
        } else {
            n = 0;
            int c = 0;
            for (; c < ctot && n < K; ++c)
                if (sd[c] >= 0.0f) { hk[n] = sd[c]; hi[n] = c; ++n; }
            heap_make(hk, hi, K);
            for (; c < ctot; ++c)
                if (sd[c] >= 0.0f) heap_offer(hk, hi, K, sd[c], c);
            heap_sort(hk, hi, K);
        }
        for (int k = 0; k < n; ++k) {
            opos[1 + k] = pos_of((uint32_t)hi[k]);
            if (okey) okey[1 + k] = hk[k];
        }
        a.out_n[ob] = 1 + n;
    }
}

// SSD of the warp's reference block (registers) against candidates.  B == 8 specialisation.
// acc order: per row, lane sums k += (r[k]-w[k])^2 then k += (r[4+k]-w[4+k])^2.
__device__ __forceinline__ float lane_combine(const float (&s)[4])
{
    return __fadd_rn(__fadd_rn(__fadd_rn(s[0], s[1]), s[2]), s[3]);
}

// Packed pairs of fp32 values (sm_100 f32x2 arithmetic: two IEEE round-to-nearest operations per
// instruction, each lane exactly as the scalar instruction would round it).  The B = 8 kernel
// forms the differences and squares of two adjacent columns at once and adds the squares into
// the four SSE lane sums with scalar adds: the compiler fuses a packed multiply followed by a
// packed add into one fused multiply-add (single rounding), which would not match the
// reference's separately rounded square and sum.
typedef unsigned long long f32x2;

__device__ __forceinline__ f32x2 pack2(float lo, float hi)
{
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}

__device__ __forceinline__ void unpack2(f32x2 v, float &lo, float &hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}

__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b)
{
    f32x2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b)
{
    f32x2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

// acc[2p] += d.lo^2, acc[2p + 1] += d.hi^2 for the column pair p of a row
__device__ __forceinline__ void add_sq2(float (&acc)[4], int p, f32x2 d)
{
    float lo, hi;
    unpack2(mul2(d, d), lo, hi);
    acc[2 * p] = __fadd_rn(acc[2 * p], lo);
    acc[2 * p + 1] = __fadd_rn(acc[2 * p + 1], hi);
}

// Exact SSD of the 8 x 8 blocks at r (pitch rs) and w (pitch ws) in the reference's SSE2 order:
// four lane sums, lane k taking column k and then column 4 + k of every row, combined
// ((s0 + s1) + s2) + s3; every square and sum separately rounded (the packed kernel's arithmetic).
__device__ __forceinline__ float exact_ssd8(const float *r, int rs, const float *w, long long ws)
{
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int y = 0; y < 8; ++y) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float d = __fsub_rn(r[y * rs + k], w[y * ws + k]);
            acc[k] = __fadd_rn(acc[k], __fmul_rn(d, d));
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float d = __fsub_rn(r[y * rs + 4 + k], w[y * ws + 4 + k]);
            acc[k] = __fadd_rn(acc[k], __fmul_rn(d, d));
        }
    }
    return lane_combine(acc);
}

// exact_ssd8 with the reference block held as packed pairs rbp[y * 4 + m] = (r[y][2m], r[y][2m + 1])
__device__ __forceinline__ float exact_ssd8_rb(const f32x2 (&rbp)[32], const float *w, int ws)
{
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int y = 0; y < 8; ++y)
#pragma unroll
        for (int h = 0; h < 4; ++h) add_sq2(acc, h & 1, sub2(rbp[y * 4 + h], pack2(w[y * ws + 2 * h], w[y * ws + 2 * h + 1])));
    return lane_combine(acc);
}

// Exact SSD (the reference's order) of the 8 x 8 reference block at rp (window, pitch wp) against
// every lattice candidate (rows t + ry s, columns l + c s; window origin wy0, wx0) into
// sd[ry * ncols + c], and against the trailing (0, 0) candidate of `plane` into sd[nrows * ncols].
// One warp.
__device__ __forceinline__ void ssd8_lattice(float *sd, const float *win, int wp, int wy0, int wx0, const float *rp,
                                             int t, int l, int s, int nrows, int ncols, const float *plane, long long ld)
{
    const int lane = (int)lane_id();
    const int clat = nrows * ncols;
    // reference block as packed pairs: rbp[y * 4 + m] = (rb[y][2m], rb[y][2m + 1])
    f32x2 rbp[32];
#pragma unroll
    for (int y = 0; y < 8; ++y)
#pragma unroll
        for (int m = 0; m < 4; ++m) rbp[y * 4 + m] = pack2(rp[y * wp + 2 * m], rp[y * wp + 2 * m + 1]);

    // item = 4 horizontally adjacent candidates; consecutive lanes take consecutive rows of
    // the same quad column (with the odd window pitch their loads hit distinct banks)
    const int nq = (ncols + 3) >> 2;
    const int items = nrows * nq;
    for (int it = lane; it < items; it += 32) {
        const int q = it / nrows;
        const int ry = it - q * nrows;
        const int cy = t + ry * s;
        const int cx0 = l + 4 * q * s;
        float acc[4][4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[u][k] = 0.0f;
        const float *wr = win + (cy - wy0) * wp + (cx0 - wx0);
        if (s == 1) {
#pragma unroll
            for (int y = 0; y < 8; ++y) {
                float w[11];
#pragma unroll
                for (int k = 0; k < 11; ++k) w[k] = wr[y * wp + k];
                // window pairs starting at even (E) and odd (O) columns
                f32x2 E[5], O[5];
#pragma unroll
                for (int m = 0; m < 5; ++m) {
                    E[m] = pack2(w[2 * m], w[2 * m + 1]);
                    O[m] = pack2(w[2 * m + 1], w[2 * m + 2]);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const f32x2 *Wp = (u & 1) ? O : E;
                    const int m0 = u >> 1;
                    // columns 0..3 (lane k takes column k), then 4..7 (lane k takes 4 + k)
#pragma unroll
                    for (int h = 0; h < 4; ++h) add_sq2(acc[u], h & 1, sub2(rbp[y * 4 + h], Wp[m0 + h]));
                }
            }
        } else {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (4 * q + u >= ncols) break;
                const float *wu = wr + u * s;
#pragma unroll
                for (int y = 0; y < 8; ++y) {
#pragma unroll
                    for (int h = 0; h < 4; ++h)
                        add_sq2(acc[u], h & 1, sub2(rbp[y * 4 + h], pack2(wu[y * wp + 2 * h], wu[y * wp + 2 * h + 1])));
                }
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int c = 4 * q + u;
            if (c < ncols) sd[ry * ncols + c] = lane_combine(acc[u]);
        }
    }
    if (lane == 0) {
        // the trailing (0, 0) candidate, read from global memory
        float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        for (int y = 0; y < 8; ++y) {
            const float *g = plane + (long long)y * ld;
#pragma unroll
            for (int h = 0; h < 4; ++h) add_sq2(acc, h & 1, sub2(rbp[y * 4 + h], pack2(__ldg(g + 2 * h), __ldg(g + 2 * h + 1))));
        }
        sd[clat] = lane_combine(acc);
    }
}

template <int BT>
__global__ void __launch_bounds__(256) bm_full_kernel(BMArgs a)
{
    extern __shared__ float smem[];
    const int lane = (int)lane_id();
    const int warp = threadIdx.x >> 5;
    const int f = blockIdx.z;
    const int by = blockIdx.y;
    const int bx0 = blockIdx.x * a.warps;
    const int bx = bx0 + warp;
    const int B = BT > 0 ? BT : a.B;
    const float *plane = a.ref + (long long)f * a.frame_stride;

    const int j = a.scan_y[by];
    const int xfirst = a.scan_x[bx0];
    const int xlast = a.scan_x[min(bx0 + a.warps, a.nbx) - 1];
    const int wy0 = max(0, j - a.range), wy1 = min(a.H, j + a.range + B);
    const int wx0 = max(0, xfirst - a.range), wx1 = min(a.W, xlast + a.range + B);
    const int ww = wx1 - wx0;
    const int wp = a.win_pitch;

    // window rows, one warp per row, asynchronous 4-byte copies (no register round trip)
    float *win = smem;
    for (int yy = warp; yy < wy1 - wy0; yy += (int)(blockDim.x >> 5)) {
        const float *src = plane + (long long)(wy0 + yy) * a.ld + wx0;
        float *dst = win + yy * wp;
        for (int xx = lane; xx < ww; xx += 32) tc::cp_async4(dst + xx, src + xx);
    }
    tc::cp_async_wait_all();
    __syncthreads();
    if (bx >= a.nbx) return;

    float *wbase = smem + a.win_h * wp + warp * bm_warp_floats(a.cand_cap, a.G, a.B, BT == 0);
    float *sd = wbase;
    uint32_t *list = reinterpret_cast<uint32_t *>(wbase + a.cand_cap);
    float *hk = wbase + a.cand_cap + 64;
    int *hi = reinterpret_cast<int *>(hk + a.G);

    const int i = a.scan_x[bx];
    const size_t ob = ((size_t)f * a.nby + by) * a.nbx + bx;
    const uint32_t ref_pos = pack_yx(j, i);

    if (a.G == 1) {
        if (lane == 0) {
            a.out_pos[ob * a.G] = ref_pos;
            if (a.out_key) a.out_key[ob * a.G] = 0.0f;
            a.out_n[ob] = 1;
        }
        return;
    }

    const int s = a.step;
    const int t = search_boundary(j, 0, a.range, s);
    const int b = search_boundary(j, a.H - B, a.range, s);
    const int l = search_boundary(i, 0, a.range, s);
    const int r = search_boundary(i, a.W - B, a.range, s);
    const int nrows = (b - t) / s + 1;
    const int ncols = (r - l) / s + 1;
    const int clat = nrows * ncols;
    const int ctot = clat + 1;

    if constexpr (BT == 8) {
        ssd8_lattice(sd, win, wp, wy0, wx0, win + (j - wy0) * wp + (i - wx0), t, l, s, nrows, ncols, plane, a.ld);
    } else {
        // generic block size: reference block staged in this warp's shared slice
        float *rblk = hk + 2 * a.G;
        for (int idx = lane; idx < B * B; idx += 32) {
            const int y = idx / B, x = idx - y * B;
            rblk[idx] = win[(j - wy0 + y) * wp + (i - wx0) + x];
        }
        __syncwarp();
        const int res = B % 8, simdw = B - res;
        for (int c = lane; c < ctot; c += 32) {
            const float *src;
            long long sld;
            if (c < clat) {
                const int ry = c / ncols, cc = c - ry * ncols;
                src = win + (t + ry * s - wy0) * wp + (l + cc * s - wx0);
                sld = wp;
            } else {
                src = plane;
                sld = a.ld;
            }
            float dist = 0.0f;
            if (simdw > 0) {
                float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                for (int y = 0; y < B; ++y)
                    for (int c0 = 0; c0 < simdw; c0 += 8) {
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const float d = __fsub_rn(rblk[y * B + c0 + k], src[y * sld + c0 + k]);
                            acc[k] = __fadd_rn(acc[k], __fmul_rn(d, d));
                        }
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const float d = __fsub_rn(rblk[y * B + c0 + 4 + k], src[y * sld + c0 + 4 + k]);
                            acc[k] = __fadd_rn(acc[k], __fmul_rn(d, d));
                        }
                    }
                dist = __fadd_rn(dist, lane_combine(acc));
            }
            for (int y = 0; y < B; ++y)
                for (int x = simdw; x < B; ++x) {
                    const float d = __fsub_rn(rblk[y * B + x], src[y * sld + x]);
                    dist = __fadd_rn(dist, __fmul_rn(d, d));
                }
            sd[c] = dist;
        }
    }
    __syncwarp();

    auto pos_of = [=](uint32_t c) -> uint32_t {
        if ((int)c >= clat) return pack_yx(0, 0);
        const int ry = (int)c / ncols, cc = (int)c - ry * ncols;
        return pack_yx(t + ry * s, l + cc * s);
    };
    select_and_emit(sd, ctot, list, hk, hi, a, ref_pos, ob, pos_of);
}

}  // namespace bm3d
