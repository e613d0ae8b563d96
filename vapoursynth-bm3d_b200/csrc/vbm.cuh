// vbm.cuh -- K2: V-BM3D spatio-temporal grouping (predictive search).
//
// Replaces VBM3D_Process_Base::BlockMatching (source/VBM3D_Base.cpp:540-659):
//   1. full search in the current frame (K1 semantics, reference pinned first);
//   2. the first ps_num entries of that list (reference included) seed the predictive search:
//      GenSearchPos builds the sorted, de-duplicated union of (2*ps_range/ps_step+1)^2 windows
//      around them (include/Block.h:771-827);
//   3. frames cur-1 .. 0 and then cur+1 .. last are searched over such unions, each frame seeded
//      by the previous frame's best ps_num (the first step of each direction uses the current
//      frame's union); per frame the matches with 0 < dist <= thSSE are kept, partial_sort-ed to
//      group_size when more survive, stable_sort-ed otherwise (include/Block.h:655-677);
//   4. the concatenation [current, backward..., forward...] is partial_sort-ed from the second
//      entry when longer than group_size (source/VBM3D_Base.cpp:652-656).
// One warp per reference block.  The current-frame list comes from K1 (run with keys); this
// kernel performs steps 2-4.
#pragma once

#include "select.cuh"
#include "args.h"
#include "bm.cuh"
#include "proposal.cuh"

namespace bm3d {


__device__ __forceinline__ float ssd8_global(const float (&rb)[64], const float *src, int ld)
{
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int y = 0; y < 8; ++y) {
        const float *g = src + (long long)y * ld;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float d = __fsub_rn(rb[y * 8 + k], __ldg(g + k));
            acc[k] = __fadd_rn(acc[k], __fmul_rn(d, d));
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float d = __fsub_rn(rb[y * 8 + 4 + k], __ldg(g + 4 + k));
            acc[k] = __fadd_rn(acc[k], __fmul_rn(d, d));
        }
    }
    return lane_combine(acc);
}

__device__ __forceinline__ float ssd_any_global(const float *rblk, int B, const float *src, int ld)
{
    const int res = B % 8, simdw = B - res;
    float dist = 0.0f;
    if (simdw > 0) {
        float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        for (int y = 0; y < B; ++y)
            for (int c0 = 0; c0 < simdw; c0 += 8) {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float d = __fsub_rn(rblk[y * B + c0 + k], __ldg(src + (long long)y * ld + c0 + k));
                    acc[k] = __fadd_rn(acc[k], __fmul_rn(d, d));
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float d = __fsub_rn(rblk[y * B + c0 + 4 + k], __ldg(src + (long long)y * ld + c0 + 4 + k));
                    acc[k] = __fadd_rn(acc[k], __fmul_rn(d, d));
                }
            }
        dist = __fadd_rn(dist, lane_combine(acc));
    }
    for (int y = 0; y < B; ++y)
        for (int x = simdw; x < B; ++x) {
            const float d = __fsub_rn(rblk[y * B + x], __ldg(src + (long long)y * ld + x));
            dist = __fadd_rn(dist, __fmul_rn(d, d));
        }
    return dist;
}

// Union of lattice windows around `nc` centres, sorted by (y, x) and de-duplicated, written
// to sp (packed y<<16|x).  Returns the count.  Warp-cooperative: the union is built as a
// sorted merge, one centre at a time, mirroring MergeSearchPos + unique.
__device__ int gen_search_pos_warp(const uint32_t *centres, int nc, int H, int W, int B, int range,
                                   int step, uint32_t *sp, uint32_t *tmp, int cap)
{
    const int lane = (int)lane_id();
    int n = 0;
    for (int ci = 0; ci < nc; ++ci) {
        const int cy = unpack_y(centres[ci]), cx = unpack_x(centres[ci]);
        const int l = search_boundary(cx, 0, range, step);
        const int r = search_boundary(cx, W - B, range, step);
        const int t = search_boundary(cy, 0, range, step);
        const int b = search_boundary(cy, H - B, range, step);
        const int ncol = (r - l) / step + 1;
        const int nrow = (b - t) / step + 1;
        const int nw = ncol * nrow;
        // merge sp[0..n) with the window (both sorted) into tmp, keeping duplicates out
        // rank of each element in the other list gives its merged position
        int total = 0;
        for (int k = lane; k < n; k += 32) {
            const uint32_t v = sp[k];
            // count window elements < v
            const int vy = unpack_y(v), vx = unpack_x(v);
            int rows_before = vy <= t ? 0 : vy > b ? nrow : (vy - t + step - 1) / step;
            int cnt = rows_before * ncol;
            if (vy >= t && vy <= b && (vy - t) % step == 0) {
                int cols_before = vx <= l ? 0 : vx > r ? ncol : (vx - l + step - 1) / step;
                cnt += cols_before;
            }
            tmp[k + cnt] = v;
        }
        for (int k = lane; k < nw; k += 32) {
            const int ry = k / ncol, cc = k - ry * ncol;
            const uint32_t v = pack_yx(t + ry * step, l + cc * step);
            // count sp elements <= v (equal elements from the first range come first)
            int lo = 0, hi = n;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (sp[mid] <= v) lo = mid + 1; else hi = mid;
            }
            tmp[k + lo] = v;
        }
        total = n + nw;
        __syncwarp();
        // unique (adjacent duplicates) while copying back
        int out = 0;
        for (int k0 = 0; k0 < total; k0 += 32) {
            const int k = k0 + lane;
            bool keep = false;
            uint32_t v = 0;
            if (k < total) {
                v = tmp[k];
                keep = k == 0 || tmp[k - 1] != v;
            }
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                const int d = out + __popc(m & ((1u << lane) - 1u));
                if (d < cap) sp[d] = v;
            }
            out += __popc(m);
        }
        __syncwarp();
        n = out < cap ? out : cap;
    }
    return n;
}

// Per-frame selection of the search-position form: partial_sort(begin, begin + G) when more
// than G survive, stable_sort otherwise.  Keys computed for all valid (invalid = -1).
// Result (sorted keys + scan indices) in hk/hi; returns the count.
__device__ int select_positions(float *sk, int ns, int G, float *hk, int *hi)
{
    const int lane = (int)lane_id();
    int cnt = 0;
    for (int c = lane; c < ns; c += 32) cnt += sk[c] >= 0.0f;
    const int nvalid = warp_sum(cnt);
    int n = 0;
    if (lane == 0) {
        if (nvalid > G) {
            int c = 0;
            for (; c < ns && n < G; ++c)
                if (sk[c] >= 0.0f) { hk[n] = sk[c]; hi[n] = c; ++n; }
            heap_make(hk, hi, G);
            for (; c < ns; ++c)
                if (sk[c] >= 0.0f) heap_offer(hk, hi, G, sk[c], c);
            heap_sort(hk, hi, G);
        } else {
            for (int c = 0; c < ns; ++c)
                if (sk[c] >= 0.0f) { hk[n] = sk[c]; hi[n] = c; ++n; }
            stable_sort_keys(hk, hi, n);
        }
    }
    n = __shfl_sync(0xffffffffu, n, 0);
    __syncwarp();
    return n;
}

__global__ void __launch_bounds__(128) vbm_predict_kernel(VBMArgs a)
{
    extern __shared__ float smem[];
    const int lane = (int)lane_id();
    const int warp = threadIdx.x >> 5;
    const int f = blockIdx.z;
    const int by = blockIdx.y;
    const int bx = blockIdx.x * a.warps + warp;
    if (bx >= a.nbx) return;

    // per-warp shared layout
    const int per_warp = vbm_warp_floats(a.sp_cap, a.list_cap, a.G, a.ps_num, a.B);
    float *base = smem + (size_t)warp * per_warp;
    uint32_t *sp = reinterpret_cast<uint32_t *>(base);
    uint32_t *tmp = sp + a.sp_cap;
    float *sk = reinterpret_cast<float *>(tmp + vbm_tmp_cap(a.sp_cap));
    float *lk = sk + a.sp_cap;                                  // concatenated keys
    uint32_t *lp = reinterpret_cast<uint32_t *>(lk + a.list_cap); // concatenated positions (zyx)
    float *fk = reinterpret_cast<float *>(lp + a.list_cap);     // per-frame selection keys
    int *fi = reinterpret_cast<int *>(fk + a.list_cap);
    uint32_t *cen = reinterpret_cast<uint32_t *>(fi + a.list_cap);
    float *hk = reinterpret_cast<float *>(cen + a.ps_num);
    int *hi = reinterpret_cast<int *>(hk + a.G);
    float *rblk = reinterpret_cast<float *>(hi + a.G);

    const int frames = a.win_len[f];
    const int cur = a.win_cur[f];
    const int wbase = a.win_base[f];
    const int B = a.B;
    const int G = a.G;
    const int j = a.scan_y[by], i = a.scan_x[bx];
    const size_t ob = ((size_t)f * a.nby + by) * a.nbx + bx;
    const float *curplane = a.ref + (long long)(wbase + cur) * a.frame_stride;

    // current-frame list
    const int n0 = a.cur_n[ob];
    int L = 0;
    for (int k = lane; k < n0; k += 32) {
        const uint32_t p = a.cur_pos[ob * G + k];
        lp[k] = pack_zyx(cur, unpack_y(p), unpack_x(p));
        lk[k] = a.cur_key[ob * G + k];
    }
    L = n0;
    if (G == 1) {
        if (lane == 0) {
            a.out_pos[ob * G] = pack_zyx(cur, j, i);
            if (a.out_key) a.out_key[ob * G] = 0.0f;
            a.out_n[ob] = 1;
        }
        return;
    }
    for (int idx = lane; idx < B * B; idx += 32) {
        const int y = idx / B, x = idx - y * B;
        rblk[idx] = curplane[(long long)(j + y) * a.ld + i + x];
    }
    __syncwarp();
    float rb[64];
    if (B == 8) {
#pragma unroll
        for (int e = 0; e < 64; ++e) rb[e] = rblk[e];
    }

    // learned proposals: descriptor of the reference block (current frame)
    const __nv_bfloat16 *dsc = static_cast<const __nv_bfloat16 *>(a.desc);
    const int Wd = a.W - 7;
    float da[kPropCh];
    if (dsc) load_desc(dsc + (long long)(wbase + cur) * a.desc_frame * kPropCh, (long long)j * Wd + i, da);

    // seeds from the current frame
    const int ncen0 = min(a.ps_num, n0);
    for (int k = lane; k < ncen0; k += 32) {
        const uint32_t p = a.cur_pos[ob * G + k];
        cen[k] = p;
    }
    __syncwarp();

    for (int dir = -1; dir <= 1; dir += 2) {
        int ncen = ncen0;
        if (dir == 1) {
            for (int k = lane; k < ncen0; k += 32) cen[k] = a.cur_pos[ob * G + k];
            __syncwarp();
        }
        for (int fz = cur + dir; fz >= 0 && fz < frames; fz += dir) {
            const int ns = gen_search_pos_warp(cen, ncen, a.H, a.W, B, a.ps_range, a.ps_step, sp, tmp, a.sp_cap);
            const float *plane = a.ref + (long long)(wbase + fz) * a.frame_stride;
            if (dsc && B == 8 && ns > a.nprop) {
                // learned proposals: the nprop positions of smallest descriptor distance (ties by
                // position order) get exact distances, the others are left out of this frame's list
                const __nv_bfloat16 *dz = dsc + (long long)(wbase + fz) * a.desc_frame * kPropCh;
                for (int c = lane; c < ns; c += 32) {
                    float dc[kPropCh];
                    load_desc(dz, (long long)unpack_y(sp[c]) * Wd + unpack_x(sp[c]), dc);
                    float sc = 0.0f;
#pragma unroll
                    for (int k = 0; k < kPropCh; ++k) sc = fmaf(da[k] - dc[k], da[k] - dc[k], sc);
                    sk[c] = sc;
                }
                __syncwarp();
                // the nprop smallest (score, position index) by radix selection (tmp is free here)
                int rank = a.nprop - 1;
                const uint32_t cutv = warp_radix_cut(sk, ns, rank, reinterpret_cast<int *>(tmp));
                const unsigned lt = (1u << lane) - 1u;
                int eq = 0;
                for (int c0 = 0; c0 < ns; c0 += 32) {
                    const int c = c0 + lane;
                    const uint32_t u = c < ns ? __float_as_uint(sk[c]) : 0xffffffffu;
                    const bool isq = c < ns && u == cutv;
                    const unsigned mq = __ballot_sync(0xffffffffu, isq);
                    const bool in = c < ns && (u < cutv || (isq && eq + __popc(mq & lt) <= rank));
                    eq += __popc(mq);
                    if (c < ns) {
                        float key = -1.0f;
                        if (in) {
                            const float d = ssd8_global(rb, plane + (long long)unpack_y(sp[c]) * a.ld + unpack_x(sp[c]), a.ld);
                            key = dist_valid(d, a.thSSE) ? dist_to_key(d, a.distMul) : -1.0f;
                        }
                        sk[c] = key;
                    }
                }
            } else {
                for (int c = lane; c < ns; c += 32) {
                    const int y = unpack_y(sp[c]), x = unpack_x(sp[c]);
                    const float *src = plane + (long long)y * a.ld + x;
                    const float d = B == 8 ? ssd8_global(rb, src, a.ld) : ssd_any_global(rblk, B, src, a.ld);
                    sk[c] = dist_valid(d, a.thSSE) ? dist_to_key(d, a.distMul) : -1.0f;
                }
            }
            __syncwarp();
            const int nf = select_positions(sk, ns, G, fk, fi);
            for (int k = lane; k < nf; k += 32) {
                const uint32_t p = sp[fi[k]];
                if (L + k < a.list_cap) {
                    lp[L + k] = pack_zyx(fz, unpack_y(p), unpack_x(p));
                    lk[L + k] = fk[k];
                }
            }
            // next seeds: first ps_num of this frame's list
            const int nn = min(a.ps_num, nf);
            __syncwarp();
            for (int k = lane; k < nn; k += 32) cen[k] = sp[fi[k]];
            ncen = nn;
            L += nf;
            __syncwarp();
        }
    }
    if (L > a.list_cap) L = a.list_cap;

    // final merge: partial_sort(begin + 1, begin + G) if longer than G
    uint32_t *op = a.out_pos + ob * G;
    float *ok = a.out_key ? a.out_key + ob * G : nullptr;
    if (L > G) {
        if (lane == 0) {
            const int K = G - 1;
            for (int k = 0; k < K; ++k) { hk[k] = lk[1 + k]; hi[k] = 1 + k; }
            heap_make(hk, hi, K);
            for (int c = 1 + K; c < L; ++c) heap_offer(hk, hi, K, lk[c], c);
            heap_sort(hk, hi, K);
            op[0] = lp[0];
            if (ok) ok[0] = lk[0];
            for (int k = 0; k < K; ++k) {
                op[1 + k] = lp[hi[k]];
                if (ok) ok[1 + k] = hk[k];
            }
            a.out_n[ob] = G;
        }
    } else {
        for (int k = lane; k < L; k += 32) {
            op[k] = lp[k];
            if (ok) ok[k] = lk[k];
        }
        if (lane == 0) a.out_n[ob] = L;
    }
}

}  // namespace bm3d
