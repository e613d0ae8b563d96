// bm_tc.cuh -- precision form of the full-search block matching (B = 8, candidate step 1): the
// cross terms of the SSD on the 16-bit tensor cores, an error-bounded short list, and the exact
// FP32 SSD of the short list in the reference's summation order.
//
// Same contract as bm_full_kernel (Block::BlockMatchingMulti, include/Block.h:554-729, window
// include/Block.h:734-769, selection include/Block.h:715-728): the lists it writes are the plain
// kernel's lists.  Distances are only *estimated* on the tensor cores,
//     SSD(a, b) = |a - c|^2 + |b - c|^2 - 2 (a - c).(b - c)       (c: the window mean),
// with the centred values scaled by a power of two s into [-1, 1], (b - c) s rounded to fp16 and
// (a - c) s split into two fp16 terms.  With unit roundoff 2^-11, Cauchy-Schwarz over the 64
// products, the fp16 subnormal spacing and the fp32 sums, |estimate - exact| <= mg =
//     (2^-10 * 1.01 + 2^-16) |a - c| max|b - c| + 2^-20 / s (|a - c| + max|b - c|)
//     + 2^-16 (|a - c|^2 + max|b - c|^2).
// (fp16 rather than bf16: pixel values are bounded, so after the exact power-of-two scaling the
// 11-bit significand is usable and the band of undecided candidates is 8x narrower.)  The
// candidates whose estimate can still reach the top group_size - 1 (estimate - mg <= the
// (group_size - 1)-th smallest estimate + mg) are re-evaluated exactly and selected on exact keys.
// Whenever the bound cannot settle the list -- more than 128 candidates in the band, too few
// exactly valid candidates below the bound, or equal keys among the output (the reference's tie
// order) -- the warp computes every exact distance and runs the plain selection.  The output is
// therefore always the plain kernel's output; the tensor cores only cut the number of exact SSDs.
//
// Layout: one CTA (one warp per reference block) per run of at most kBmtRefs consecutive
// reference blocks of one row whose search windows span at most kBmtCols = 64 candidate columns.
// U[y'][x] holds the 8 pixels (y', x .. x + 7) as 16 bytes, so the 8 x 8 block at (y, x) is rows
// y .. y + 7 of U at column x and a core matrix (8 candidates x 8 pixels of one image row) is 128
// contiguous bytes: the A operand needs no im2col.  With 64 columns per image row of U, one
// M = 128 product covers two candidate rows (lanes 0-63: row y, lanes 64-127: row y + 1, the
// descriptor simply running on into the next row of U), and the B operand holds the high terms of
// the reference blocks in N-rows 0-7 and the low terms in rows 8-15: one M = 128, N = 16, K = 64
// fp16 product per pair of candidate rows gives D[x][n] + D[x][8 + n] = (b(y, x) - c).(a_n - c) s^2.
#pragma once

#include <cuda_fp16.h>

#include "bm.cuh"
#include "tc.cuh"

namespace bm3d {

constexpr int kBmtThreads = 32 * kBmtRefs;
constexpr int kBmtPairsPerPhase = 16;     // candidate-row pairs in tensor memory at once (16 columns each)
constexpr uint32_t kBmtWaitLimit = 1u << 24;

__host__ __device__ constexpr uint32_t idesc_f16(int M, int N)
{
    return (1u << 4)                    // D format f32
         | (0u << 7)                    // A format f16
         | (0u << 10)                   // B format f16
         | ((uint32_t)(N >> 3) << 17)
         | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_ss_f16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc, bool accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                 ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"((uint32_t)accumulate));
}

__global__ void __launch_bounds__(kBmtThreads) bm_tc_kernel(BMArgs a, BmtLayout L)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ __align__(8) uint64_t mdrain;    // drains the products before the time-out path frees
    __shared__ uint32_t tslot;
    __shared__ float red[3][kBmtRefs];          // [1] candidate norm maxima, [2] window sums
    __shared__ float wlo[kBmtRefs], whi[kBmtRefs];
    __shared__ float s_na[kBmtRefs];           // centred reference norms
    __shared__ int s_i[kBmtRefs], s_l[kBmtRefs], s_nc[kBmtRefs];   // column, first candidate column and count
    __shared__ int fail_flag;
    __shared__ float z00[64];                  // the trailing candidate: the block at (0, 0) of the plane

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int f = blockIdx.z;
    const int by = blockIdx.y;
    const int bx0 = blockIdx.x * L.nrc;
    const int nref = min(L.nrc, a.nbx - bx0);
    const float *plane = a.ref + (long long)f * a.frame_stride;
    const int R = a.range;
    const int j = a.scan_y[by];
    // candidate lattice (step 1): rows [t, b] for every reference block of the row, columns
    // [max(0, i - R), min(W - 8, i + R)] for reference block i; the union starts at the first
    // block's left edge
    const int t = max(0, j - R), b = min(a.H - 8, j + R);
    const int nrows = b - t + 1;
    const int xl = max(0, a.scan_x[bx0] - R);
    const int xr = min(a.W - 8, a.scan_x[bx0 + nref - 1] + R);
    const int ncc = xr - xl + 1;                       // <= kBmtCols (host check)
    const int wy0 = t, wx0 = xl;
    const int wrows = nrows + 7, wcols = ncc + 7;

    unsigned char *U = sm + L.offU;
    unsigned char *Rb = sm + L.offR;
    float *win = reinterpret_cast<float *>(sm + L.offWin);
    float *sdall = reinterpret_cast<float *>(sm + L.offSd);
    float *rsq = reinterpret_cast<float *>(sm + L.offRsq);   // row sums of squares (centred)

    if (warp == 0) tc::tmem_alloc(&tslot, 256);
    if (tid < 3) tc::mbar_init(tid < 2 ? &mbar[tid] : &mdrain, 1);
    if (tid == 0) fail_flag = 0;
    if (tid < kBmtRefs) {
        int i = -1, l = 0, nc = 0;
        if (tid < nref) {
            i = a.scan_x[bx0 + tid];
            l = max(0, i - R);
            nc = min(a.W - 8, i + R) - l + 1;
        }
        s_i[tid] = i;
        s_l[tid] = l;
        s_nc[tid] = nc;
    }

    // 1. window rows, asynchronous 4-byte copies
    for (int yy = warp; yy < wrows; yy += kBmtRefs) {
        const float *src = plane + (long long)(wy0 + yy) * a.ld + wx0;
        float *dst = win + yy * L.wp;
        for (int xx = lane; xx < wcols; xx += 32) tc::cp_async4(dst + xx, src + xx);
    }
    if (tid < 64) tc::cp_async4(&z00[tid], plane + (long long)(tid >> 3) * a.ld + (tid & 7));
    tc::cp_async_wait_all();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();

    // 2. centring constant: the mean of the window (any constant gives the same exact result;
    //    a central one keeps the fp16 terms and the error bound small), and the scale
    float cmean, sc, inv_s;
    {
        float s = 0.0f, lo = 3.0e38f, hi = -3.0e38f;
        for (int yy = warp; yy < wrows; yy += kBmtRefs)
            for (int xx = lane; xx < wcols; xx += 32) {
                const float v = win[yy * L.wp + xx];
                s += v;
                lo = fminf(lo, v);
                hi = fmaxf(hi, v);
            }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_xor_sync(0xffffffffu, s, o);
            lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (lane == 0) {
            red[2][warp] = s;
            wlo[warp] = lo;
            whi[warp] = hi;
        }
        __syncthreads();
        float tot = 0.0f;
#pragma unroll
        for (int w = 0; w < kBmtRefs; ++w) {
            tot += red[2][w];
            lo = fminf(lo, wlo[w]);
            hi = fmaxf(hi, whi[w]);
        }
        cmean = tot / (float)(wrows * wcols);
        // power-of-two scale taking the centred values into [-1, 1] (exact in fp32)
        const float amax = fmaxf(hi - cmean, cmean - lo);
        int ex = 0;
        if (amax > 0.0f) frexpf(amax, &ex);      // amax < 2^ex
        sc = ldexpf(1.0f, -ex);
        inv_s = ldexpf(1.0f, ex);
    }

    // 3. U (fp16, 8 pixels per candidate column and image row; one zero row past the window, read
    //    by the upper lanes of the last product) and the row sums of squares
    for (int e = tid; e < (L.wh + 1) * kBmtCols; e += kBmtThreads) {
        const int yy = e / kBmtCols, m = e - yy * kBmtCols;
        uint32_t h[4] = {0u, 0u, 0u, 0u};
        float sq = 0.0f;
        if (yy < wrows && m < ncc) {
            const float *w = win + yy * L.wp + m;
#pragma unroll
            for (int v = 0; v < 8; v += 2) {
                const float d0 = w[v] - cmean, d1 = w[v + 1] - cmean;
                sq = fmaf(d0, d0, sq);
                sq = fmaf(d1, d1, sq);
                const __half2 p = __floats2half2_rn(d0 * sc, d1 * sc);
                h[v >> 1] = *reinterpret_cast<const uint32_t *>(&p);
            }
        }
        *reinterpret_cast<uint4 *>(U + yy * (kBmtCols * 16) + m * 16) = make_uint4(h[0], h[1], h[2], h[3]);
        if (yy < L.wh) rsq[yy * kBmtCols + m] = sq;
    }
    // reference blocks: high terms in N-rows 0-7, low terms in rows 8-15 of the B operand (K-major,
    // no swizzle): byte(n, k) = (k / 8) * 256 + (n / 8) * 128 + (n % 8) * 16 + (k % 8) * 2, k = 8 u + v
    {
        const int n = warp;
        float na_part = 0.0f;
        for (int e = lane; e < 64; e += 32) {
            const int u = e >> 3, v = e & 7;
            float d = 0.0f;
            if (n < nref) d = win[(j - wy0 + u) * L.wp + (a.scan_x[bx0 + n] - wx0) + v] - cmean;
            const __half hi = __float2half_rn(d * sc);
            const __half lo = __float2half_rn(d * sc - __half2float(hi));
            const int off = u * 256 + n * 16 + v * 2;
            *reinterpret_cast<__half *>(Rb + off) = hi;
            *reinterpret_cast<__half *>(Rb + off + 128) = lo;
            na_part = fmaf(d, d, na_part);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) na_part += __shfl_xor_sync(0xffffffffu, na_part, o);
        if (lane == 0) s_na[n] = na_part;
    }
    // U and the reference blocks to the tensor cores' view
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = tslot;

    // 4. products: pair p = candidate rows 2p (lanes 0-63) and 2p + 1 (lanes 64-127) into tensor
    //    columns 16 (p % 16) .. +16; at most 16 pairs per phase
    const int npairs = (nrows + 1) >> 1;
    const int nphases = (npairs + kBmtPairsPerPhase - 1) / kBmtPairsPerPhase;
    constexpr uint32_t IDF = idesc_f16(128, 16);
    const uint32_t sU = tc::smem_u32(U), sR = tc::smem_u32(Rb);
    // descriptors: A = U from image row 2 pp + 2 s4 on (LBO: next image row, SBO: next 8
    // candidates), B = the reference blocks at K step s4 (LBO: next 8 pixels, SBO: low terms)
    const uint64_t descA = tc::make_desc(sU, kBmtCols * 16, 128);
    uint64_t descB[4];
#pragma unroll
    for (int s4 = 0; s4 < 4; ++s4) descB[s4] = tc::make_desc(sR + (uint32_t)(s4 * 512), 256, 128);
    auto issue = [&](int ph) {
        for (int pp = ph * kBmtPairsPerPhase; pp < min(npairs, (ph + 1) * kBmtPairsPerPhase); ++pp) {
            const uint32_t d = tm + (uint32_t)((pp % kBmtPairsPerPhase) * 16);
#pragma unroll
            for (int s4 = 0; s4 < 4; ++s4)   // image rows 2 pp + 2 s4 on; start address in 16-byte units
                mma_ss_f16(d, descA + (uint64_t)((2 * pp + 2 * s4) * kBmtCols), descB[s4], IDF, s4 > 0);
        }
        tc::mma_commit(&mbar[ph & 1]);
    };
    if (tid == 0) issue(0);

    // readout: lane quarter q of the tensor memory; the two warps of a quarter take alternate pairs
    const int q = warp & 3;
    const int half = warp >> 2;
    const int tl = 32 * q + lane;                      // tensor-memory lane of this thread
    const int m = tl & 63;                             // candidate column
    const int par = tl >> 6;                           // row within the pair
    const int X = xl + m;
    const float s2 = inv_s * inv_s;
    // this thread's column within each reference block's lattice (-1: outside its window)
    int cb[kBmtRefs], ncr[kBmtRefs];
    float nar[kBmtRefs];
    bool selfc[kBmtRefs];
#pragma unroll
    for (int n = 0; n < kBmtRefs; ++n) {
        const int c0 = X - s_l[n];
        const bool in = n < nref && m < ncc && c0 >= 0 && c0 < s_nc[n];
        cb[n] = in ? n * L.cs + c0 : -1;
        ncr[n] = s_nc[n];
        nar[n] = s_na[n];
        selfc[n] = X == s_i[n];
    }
    float nbm = 0.0f;                                  // largest candidate norm this thread saw
    auto emit = [&](int r, const float (&dv)[16]) {
        if (r >= nrows || m >= ncc) return;
        // centred norm of candidate (r, m): the row sums of squares of its 8 rows
        float nbv = 0.0f;
#pragma unroll
        for (int u = 0; u < 8; ++u) nbv += rsq[(r + u) * kBmtCols + m];
        nbm = fmaxf(nbm, nbv);
        const bool selfrow = t + r == j;
#pragma unroll
        for (int n = 0; n < kBmtRefs; ++n) {
            if (cb[n] < 0) continue;
            // the block itself (distance 0) is never a valid candidate
            const float est = selfrow && selfc[n] ? 3.0e38f : nar[n] + nbv - 2.0f * ((dv[n] + dv[8 + n]) * s2);
            sdall[cb[n] + r * ncr[n]] = est;
        }
    };
    bool ok = true;
    for (int ph = 0; ph < nphases; ++ph) {
        ok = tc::mbar_wait_bounded(&mbar[ph & 1], (uint32_t)((ph >> 1) & 1), kBmtWaitLimit) && ok;
        tc::fence_after_sync();
        const int pend = min(npairs, (ph + 1) * kBmtPairsPerPhase);
        // two pairs per tensor-memory round trip (pairs pp and pp + 2 of this warp's half)
        for (int pp = ph * kBmtPairsPerPhase + half; pp < pend; pp += 4) {
            float d0[16], d1[16];
            const uint32_t lrow = (uint32_t)(32 * q) << 16;
            tc::tmem_ld16(tm + lrow + (uint32_t)((pp % kBmtPairsPerPhase) * 16), d0);
            const bool two = pp + 2 < pend;
            if (two) tc::tmem_ld16(tm + lrow + (uint32_t)(((pp + 2) % kBmtPairsPerPhase) * 16), d1);
            tc::tmem_wait_ld();
            emit(2 * pp + par, d0);
            if (two) emit(2 * (pp + 2) + par, d1);
        }
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (tid == 0 && ok && ph + 1 < nphases) issue(ph + 1);
    }
    // After a timed-out wait, products may still be writing tensor memory: one more commit, which
    // arrives once every product the issuing thread started has completed, is waited for (bounded)
    // before the columns are released.
    if (__syncthreads_or(!ok)) {
        if (tid == 0) tc::mma_commit(&mdrain);
        const bool drained = tc::mbar_wait_bounded(&mdrain, 0, kBmtWaitLimit);
        tc::fence_after_sync();
        if (tid == 0) atomicExch(&fail_flag, drained ? 1 : 2);
        __syncthreads();
    }
    if (warp == 0) tc::tmem_free(tm, 256);              // every load has completed (barrier above)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nbm = fmaxf(nbm, __shfl_xor_sync(0xffffffffu, nbm, o));
    if (lane == 0) red[1][warp] = nbm;
    __syncthreads();
    const bool tc_failed = fail_flag != 0;
    nbm = 0.0f;
#pragma unroll
    for (int w = 0; w < kBmtRefs; ++w) nbm = fmaxf(nbm, red[1][w]);

    // 5. selection, one warp per reference block
    if (warp < nref) {
        const int n = warp;
        const int i = a.scan_x[bx0 + n];
        const int l = max(0, i - R), rgt = min(a.W - 8, i + R);
        const int ncols = rgt - l + 1;
        const int clat = nrows * ncols;
        const int ctot = clat + 1;
        float *sd = sdall + n * L.cs;
        uint32_t *list = reinterpret_cast<uint32_t *>(sm + L.offScr) + n * 192;
        float *hk = reinterpret_cast<float *>(list + 128);
        int *hi = reinterpret_cast<int *>(hk + 32);
        const size_t ob = ((size_t)f * a.nby + by) * a.nbx + bx0 + n;
        const uint32_t ref_pos = pack_yx(j, i);
        const float *rp = win + (j - wy0) * L.wp + (i - wx0);
        auto pos_of = [=](uint32_t c) -> uint32_t {
            if ((int)c >= clat) return pack_yx(0, 0);
            const int ry = (int)c / ncols, cc = (int)c - ry * ncols;
            return pack_yx(t + ry, l + cc);
        };
        auto exact_of = [&](uint32_t c) -> float {
            if ((int)c >= clat) return exact_ssd8(rp, L.wp, z00, 8);
            const int ry = (int)c / ncols, cc = (int)c - ry * ncols;
            return exact_ssd8(rp, L.wp, win + ry * L.wp + (l + cc - wx0), L.wp);
        };
        const int G = a.G, K = G - 1;
        bool done = false;
        if (G == 1) {
            if (lane == 0) {
                a.out_pos[ob * G] = ref_pos;
                if (a.out_key) a.out_key[ob * G] = 0.0f;
                a.out_n[ob] = 1;
            }
            done = true;
        }
        if (!done && !tc_failed && G <= 32) {
            if (lane == 0) sd[clat] = exact_of((uint32_t)clat);   // the trailing (0, 0) candidate, exact
            __syncwarp();
            const float na = s_na[n];
            const float sa = sqrtf(na), sb = sqrtf(nbm);
            const float mg = (0.0009765625f * 1.01f + 1.52587890625e-05f) * sa * sb +
                             9.5367431640625e-07f * inv_s * (sa + sb) + 1.52587890625e-05f * (na + nbm);
            // pass 1: the K + 1 smallest upper bounds among candidates surely under the threshold
            // (values only: two per lane, then the (K + 1)-th of the 64)
            float f1 = 3.0e38f, f2 = 3.0e38f;
            int nsure = 0;
            for (int c0 = 0; c0 < ctot; c0 += 32) {
                const int c = c0 + ((lane + 7 * (c0 >> 5)) & 31);
                if (c >= ctot) continue;
                const float hv = sd[c] + mg;
                if (hv <= a.thSSE) {
                    ++nsure;
                    const float h = fmaxf(hv, 0.0f);
                    f2 = fminf(f2, fmaxf(f1, h));
                    f1 = fminf(f1, h);
                }
            }
            nsure = warp_sum(nsure);
            float v2[2] = {f1, f2};
            warp_bitonic_f32<2>(v2);
            const float TK = __shfl_sync(0xffffffffu, v2[0], K);
            // bound: the first K + 1 exact distances are <= bnd (K + 1 candidates have upper bounds
            // there), everything whose lower bound lies above it is settled
            const bool complete = nsure <= K;               // then every possibly valid candidate is listed
            const float bnd = complete ? a.thSSE : fminf(a.thSSE, TK);
            // pass 2: the band of candidates whose lower bound is within it
            int ms = 0;
            const unsigned lt = (1u << lane) - 1u;
            for (int c0 = 0; c0 < ctot; c0 += 32) {
                const int c = c0 + lane;
                const bool in = c < ctot && sd[c] - mg <= bnd;
                const unsigned msk = __ballot_sync(0xffffffffu, in);
                if (in && ms + __popc(msk & lt) < 128) list[ms + __popc(msk & lt)] = (uint32_t)c;
                ms += __popc(msk);
            }
            __syncwarp();
            if (ms <= 128) {
                // exact distances of the band (the reference block in registers as packed pairs);
                // invalid ones sort last
                f32x2 rbp[32];
#pragma unroll
                for (int y = 0; y < 8; ++y)
#pragma unroll
                    for (int m = 0; m < 4; ++m) rbp[y * 4 + m] = pack2(rp[y * L.wp + 2 * m], rp[y * L.wp + 2 * m + 1]);
                uint64_t v[4] = {~0ull, ~0ull, ~0ull, ~0ull};
                int nval = 0, nbelow = 0;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int idx = lane + 32 * e;
                    if (idx < ms) {
                        const uint32_t c = list[idx];
                        float d;
                        if ((int)c >= clat) {
                            d = exact_of(c);
                        } else {
                            const int ry = (int)c / ncols, cc = (int)c - ry * ncols;
                            d = exact_ssd8_rb(rbp, win + ry * L.wp + (l + cc - wx0), L.wp);
                        }
                        if (dist_valid(d, a.thSSE)) {
                            v[e] = compose(d, c);
                            ++nval;
                            nbelow += d <= bnd;
                        }
                    }
                }
                nval = warp_sum(nval);
                nbelow = warp_sum(nbelow);
                // complete: every possibly valid candidate is in the band.  Otherwise the band holds
                // at least K + 1 exactly valid candidates at or below bnd and everything outside
                // lies above bnd, so the band's first K + 1 are the first K + 1 overall (the last
                // one decides whether the cut falls between equal keys).
                if (complete || nbelow > K) {
                    if (ms <= 32) warp_bitonic_u64<1>(*reinterpret_cast<uint64_t (*)[1]>(v));
                    else if (ms <= 64) warp_bitonic_u64<2>(*reinterpret_cast<uint64_t (*)[2]>(v));
                    else warp_bitonic_u64<4>(v);
                    const int nout = min(nval, K);
                    // the reference's tie order only matters for equal keys: then fall back
                    const float key = lane <= nout && lane < nval ? dist_to_key(__uint_as_float((uint32_t)(v[0] >> 32)), a.distMul) : 0.0f;
                    const float prev = __shfl_up_sync(0xffffffffu, key, 1);
                    const bool bad = lane >= 1 && lane <= nout && lane < nval && !(prev < key);
                    if (!__any_sync(0xffffffffu, bad)) {
                        if (lane == 0) {
                            a.out_pos[ob * G] = ref_pos;
                            if (a.out_key) a.out_key[ob * G] = 0.0f;
                            a.out_n[ob] = 1 + nout;
                        }
                        if (lane < nout) {
                            a.out_pos[ob * G + 1 + lane] = pos_of((uint32_t)v[0]);
                            if (a.out_key) a.out_key[ob * G + 1 + lane] = key;
                        }
                        done = true;
                    }
                }
            } else {
                // a band too wide for registers: the exact distances of the band overwrite its
                // estimates, the rest is marked invalid (it lies above the cut), and the (K + 1)
                // smallest come out as in the plain selection: each lane's best two, the cut at
                // the (K + 1)-th of their union, everything under it sorted.  Equal keys in the
                // list or at the cut still take the exact path below.
                int nval = 0, nbelow = 0;
                uint64_t c1 = ~0ull, c2 = ~0ull;
                for (int c0 = 0; c0 < ctot; c0 += 32) {
                    const int c = c0 + ((lane + 7 * (c0 >> 5)) & 31);
                    if (c >= ctot) continue;
                    float d = 3.0e38f;
                    if (sd[c] - mg <= bnd) d = exact_of((uint32_t)c);
                    sd[c] = d;
                    if (dist_valid(d, a.thSSE)) {
                        ++nval;
                        nbelow += d <= bnd;
                        const uint64_t v = compose(d, (uint32_t)c);
                        if (v < c1) { c2 = c1; c1 = v; } else if (v < c2) { c2 = v; }
                    }
                }
                nval = warp_sum(nval);
                nbelow = warp_sum(nbelow);
                __syncwarp();
                if (complete || nbelow > K) {
                    uint64_t w2[2] = {c1, c2};
                    warp_bitonic_u64<2>(w2);
                    const int nout = min(nval, K);
                    // every valid one when at most K + 1, else the cut at the (K + 1)-th of the union
                    const uint64_t T = nval <= K + 1 ? ~0ull : __shfl_sync(0xffffffffu, w2[0], K);
                    int m = 0;
                    for (int c0 = 0; c0 < ctot; c0 += 32) {
                        const int c = c0 + lane;
                        const bool in = c < ctot && dist_valid(sd[c], a.thSSE) && compose(sd[c], (uint32_t)c) <= T;
                        const unsigned msk = __ballot_sync(0xffffffffu, in);
                        if (in && m + __popc(msk & lt) < 64) list[m + __popc(msk & lt)] = (uint32_t)c;
                        m += __popc(msk);
                    }
                    __syncwarp();
                    if (m <= 64) {
                        uint64_t v[2] = {~0ull, ~0ull};
                        if (lane < m) v[0] = compose(sd[list[lane]], list[lane]);
                        if (lane + 32 < m) v[1] = compose(sd[list[lane + 32]], list[lane + 32]);
                        warp_bitonic_u64<2>(v);
                        const float key = lane <= nout && lane < nval ? dist_to_key(__uint_as_float((uint32_t)(v[0] >> 32)), a.distMul) : 0.0f;
                        const float prev = __shfl_up_sync(0xffffffffu, key, 1);
                        const bool bad = lane >= 1 && lane <= nout && lane < nval && !(prev < key);
                        if (!__any_sync(0xffffffffu, bad)) {
                            if (lane == 0) {
                                a.out_pos[ob * G] = ref_pos;
                                if (a.out_key) a.out_key[ob * G] = 0.0f;
                                a.out_n[ob] = 1 + nout;
                            }
                            if (lane < nout) {
                                a.out_pos[ob * G + 1 + lane] = pos_of((uint32_t)v[0]);
                                if (a.out_key) a.out_key[ob * G + 1 + lane] = key;
                            }
                            done = true;
                        }
                    }
                }
                __syncwarp();
            }
        }
        if (!done) {
            // every exact distance, then the plain selection
            if (lane == 0 && a.stats) atomicAdd(a.stats + 1, 1ull);
            ssd8_lattice(sd, win, L.wp, wy0, wx0, rp, t, l, 1, nrows, ncols, plane, a.ld);
            __syncwarp();
            select_and_emit(sd, ctot, list, hk, hi, a, ref_pos, ob, pos_of);
        }
    }
    if (tc_failed && tid == 0 && a.stats) atomicAdd(a.stats + 2, 1ull);
}

}  // namespace bm3d
