// select.cuh -- match-list selection with the reference's exact ordering semantics.
//
// The reference keeps the best group_size matches with std::partial_sort on a key-only
// comparator (include/Block.h:714-722, 668-676; source/VBM3D_Base.cpp:652-656; KeyPair
// compares .first only, include/Type.h:454-457) and otherwise std::stable_sort.  Which of two
// equal keys survives, and in which order, is therefore whatever libstdc++'s heap-select and
// sort-heap produce on the scan-ordered candidate array.  The functions below restate those
// published heap algorithms (binary max-heap, hole sifting to a leaf then sifting back up) so
// that ties resolve exactly as in the reference build; the warp-parallel fast path is used
// only when it provably yields the same list (all selected keys distinct and a strict gap at
// the cut).
#pragma once

#include "common.cuh"

namespace bm3d {

// ---- single-thread heap primitives over (key, id) arrays (key-only comparisons) -------------

__device__ __forceinline__ void heap_push(float *hk, int *hi, int hole, int top, float vk, int vi)
{
    int parent = (hole - 1) / 2;
    while (hole > top && hk[parent] < vk) {
        hk[hole] = hk[parent];
        hi[hole] = hi[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    hk[hole] = vk;
    hi[hole] = vi;
}

__device__ __forceinline__ void heap_adjust(float *hk, int *hi, int hole, int len, float vk, int vi)
{
    const int top = hole;
    int child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (hk[child] < hk[child - 1]) child--;
        hk[hole] = hk[child];
        hi[hole] = hi[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        hk[hole] = hk[child - 1];
        hi[hole] = hi[child - 1];
        hole = child - 1;
    }
    heap_push(hk, hi, hole, top, vk, vi);
}

__device__ __forceinline__ void heap_make(float *hk, int *hi, int len)
{
    if (len < 2) return;
    int parent = (len - 2) / 2;
    for (;;) {
        const float vk = hk[parent];
        const int vi = hi[parent];
        heap_adjust(hk, hi, parent, len, vk, vi);
        if (parent == 0) return;
        parent--;
    }
}

// One heap-select step for the element following the heap: replaces the maximum when smaller.
__device__ __forceinline__ void heap_offer(float *hk, int *hi, int len, float vk, int vi)
{
    if (vk < hk[0]) heap_adjust(hk, hi, 0, len, vk, vi);
}

__device__ __forceinline__ void heap_sort(float *hk, int *hi, int len)
{
    while (len > 1) {
        --len;
        const float vk = hk[len];
        const int vi = hi[len];
        hk[len] = hk[0];
        hi[len] = hi[0];
        heap_adjust(hk, hi, 0, len, vk, vi);
    }
}

// Stable insertion sort by key (std::stable_sort semantics for a key-only comparator).
__device__ __forceinline__ void stable_sort_keys(float *k, int *id, int n)
{
    for (int a = 1; a < n; ++a) {
        const float vk = k[a];
        const int vi = id[a];
        int b = a - 1;
        while (b >= 0 && vk < k[b]) {
            k[b + 1] = k[b];
            id[b + 1] = id[b];
            --b;
        }
        k[b + 1] = vk;
        id[b + 1] = vi;
    }
}

// ---- warp bitonic sort of 32*V uint64 values, striped layout (element e*32+lane) -----------

template <int V>
__device__ __forceinline__ void warp_bitonic_u64(uint64_t (&v)[V])
{
    constexpr int M = 32 * V;
    const int lane = (int)lane_id();
#pragma unroll
    for (int k = 2; k <= M; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
            for (int e = 0; e < V; ++e) {
                const int i = e * 32 + lane;
                const bool up = (i & k) == 0;
                if (j >= 32) {
                    const int pe = e ^ (j >> 5);
                    if (pe > e) {
                        const uint64_t a = v[e], b = v[pe];
                        const bool sw = up ? (a > b) : (a < b);
                        v[e] = sw ? b : a;
                        v[pe] = sw ? a : b;
                    }
                } else {
                    const uint64_t a = v[e];
                    const uint64_t o = __shfl_xor_sync(0xffffffffu, a, j);
                    const bool lower = (lane & j) == 0;
                    const uint64_t mn = a < o ? a : o;
                    const uint64_t mx = a < o ? o : a;
                    v[e] = (lower == up) ? mn : mx;
                }
            }
        }
    }
}

// The same network over floats (values only).
template <int V>
__device__ __forceinline__ void warp_bitonic_f32(float (&v)[V])
{
    constexpr int M = 32 * V;
    const int lane = (int)lane_id();
#pragma unroll
    for (int k = 2; k <= M; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
            for (int e = 0; e < V; ++e) {
                const int i = e * 32 + lane;
                const bool up = (i & k) == 0;
                if (j >= 32) {
                    const int pe = e ^ (j >> 5);
                    if (pe > e) {
                        const float a = v[e], b = v[pe];
                        v[e] = up ? fminf(a, b) : fmaxf(a, b);
                        v[pe] = up ? fmaxf(a, b) : fminf(a, b);
                    }
                } else {
                    const float a = v[e];
                    const float o = __shfl_xor_sync(0xffffffffu, a, j);
                    const bool lower = (lane & j) == 0;
                    v[e] = (lower == up) ? fminf(a, o) : fmaxf(a, o);
                }
            }
        }
    }
}

__device__ __forceinline__ uint64_t compose(float positive_value, uint32_t idx)
{
    return ((uint64_t)__float_as_uint(positive_value) << 32) | idx;
}

// Warp-wide radix selection over n non-negative scores sc[0..n) (their bit patterns order like the
// values): the score S of rank `rank` (0-based, rank < n) and how many entries equal to S come
// before it in that order (returned in rank).  With them, the rank + 1 smallest (score, index)
// pairs are every entry below S plus the first rank + 1 entries equal to S in index order.
// Five passes of 7, 7, 7, 7 and 3 bits with a 128-bin histogram in hist (128 ints of shared
// memory owned by the warp).
__device__ __forceinline__ uint32_t warp_radix_cut(const float *sc, int n, int &rank, int *hist)
{
    const int lane = (int)(threadIdx.x & 31);
    uint32_t prefix = 0, pmask = 0;
    for (int pass = 0; pass < 5; ++pass) {
        const int shift = pass < 4 ? 24 - 7 * pass : 0;
        const uint32_t dmask = pass < 4 ? 127u : 7u;
        for (int e = lane; e < 128; e += 32) hist[e] = 0;
        __syncwarp();
        for (int c = lane; c < n; c += 32) {
            const uint32_t u = __float_as_uint(sc[c]);
            if ((u & pmask) == prefix) atomicAdd(&hist[(u >> shift) & dmask], 1);
        }
        __syncwarp();
        int h[4], tot = 0;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            h[e] = hist[4 * lane + e];
            tot += h[e];
        }
        int incl = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int excl = incl - tot;
        const bool own = rank >= excl && rank < incl;
        int dsel = 0, before = 0;
        if (own) {
            int run = excl;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                if (rank >= run && rank < run + h[e]) {
                    dsel = 4 * lane + e;
                    before = run;
                }
                run += h[e];
            }
        }
        const int src = __ffs(__ballot_sync(0xffffffffu, own)) - 1;
        dsel = __shfl_sync(0xffffffffu, dsel, src);
        before = __shfl_sync(0xffffffffu, before, src);
        rank -= before;
        prefix |= (uint32_t)dsel << shift;
        pmask |= dmask << shift;
        __syncwarp();
    }
    return prefix;
}

}  // namespace bm3d
