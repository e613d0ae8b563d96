// proposal.cuh -- learned block-matching proposal (precision form "learned"): a two-layer
// convolutional feature network (3x3, 1 -> 16 channels, ReLU, 3x3, 16 -> 16) pooled into a
// 16-dimensional descriptor per block position (channel c averaged over quadrant c % 4 of the
// 8x8 block, so the descriptor keeps the block's coarse layout), its training kernels (ranking
// loss, backward pass, Adam), and the matching kernel that ranks the search window by descriptor
// distance, keeps the best proposals and re-ranks them with the exact FP32 SSD.
//
// No reference counterpart: the reference searches exhaustively (Block::BlockMatchingMulti,
// include/Block.h:683-729).  The lists written here keep its contract for what is written (the
// reference block first, then candidates with dist <= thSSE and dist != 0 ordered by the exact
// key, at most group_size), but a candidate that the proposals miss is missing from the list.
//
// Numerics: weights and accumulation in fp32; the activations (hidden layer H, features F) and
// the descriptors D are stored as bf16.
//
// Weight vector (kPropWeights floats): w1[16][9], b1[16], w2[16][16][9], b2[16]; taps k = 3 dy + dx
// over offsets dy, dx in {-1, 0, 1}; zero padding at the plane borders.
#pragma once

#include <cuda_bf16.h>

#include "args.h"
#include "bm.cuh"

namespace bm3d {

constexpr int kPropCh = 16;
constexpr int kPropW1 = 0, kPropB1 = 144, kPropW2 = 160, kPropB2 = 2464;
constexpr int kPropWeights = 2480;

// ---- forward -------------------------------------------------------------------------------------

// H[c][y][x] = ReLU(b1[c] + sum_k w1[c][k] x(y + dy, x + dx)), bf16, planar [16][H][W]
__global__ void prop_conv1_kernel(const float *__restrict__ x, int ld, int W, int H, const float *__restrict__ wt,
                                  __nv_bfloat16 *__restrict__ hid)
{
    __shared__ float w[160];
    for (int i = threadIdx.x; i < 160; i += blockDim.x) w[i] = wt[kPropW1 + i];
    __syncthreads();
    const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y;
    if (px >= W) return;
    float v[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const int yy = py + k / 3 - 1, xx = px + k % 3 - 1;
        v[k] = (yy >= 0 && yy < H && xx >= 0 && xx < W) ? x[(long long)yy * ld + xx] : 0.0f;
    }
#pragma unroll
    for (int c = 0; c < kPropCh; ++c) {
        float s = w[kPropB1 + c];
#pragma unroll
        for (int k = 0; k < 9; ++k) s = fmaf(w[c * 9 + k], v[k], s);
        hid[((long long)c * H + py) * W + px] = __float2bfloat16_rn(fmaxf(s, 0.0f));
    }
}

// F[c][y][x] = b2[c] + sum_{i,k} w2[c][i][k] H[i](y + dy, x + dx), bf16 planar [16][H][W].  Each
// thread computes 4 consecutive pixels, so every weight read from shared memory serves 4 products
// (the sum order per output is the same as one pixel per thread: i outer, tap k inner).
constexpr int kPropConv2Px = 4;
__global__ void prop_conv2_kernel(const __nv_bfloat16 *__restrict__ hid, int W, int H, const float *__restrict__ wt,
                                  __nv_bfloat16 *__restrict__ feat)
{
    __shared__ float w[kPropCh * kPropCh * 9 + kPropCh];
    for (int i = threadIdx.x; i < kPropCh * kPropCh * 9 + kPropCh; i += blockDim.x) w[i] = wt[kPropW2 + i];
    __syncthreads();
    const int px0 = (blockIdx.x * blockDim.x + threadIdx.x) * kPropConv2Px, py = blockIdx.y;
    if (px0 >= W) return;
    float acc[kPropConv2Px][kPropCh];
#pragma unroll
    for (int q = 0; q < kPropConv2Px; ++q)
#pragma unroll
        for (int c = 0; c < kPropCh; ++c) acc[q][c] = w[kPropCh * kPropCh * 9 + c];
    for (int i = 0; i < kPropCh; ++i) {
        float v[3][kPropConv2Px + 2];
#pragma unroll
        for (int dy = 0; dy < 3; ++dy) {
            const int yy = py + dy - 1;
#pragma unroll
            for (int u = 0; u < kPropConv2Px + 2; ++u) {
                const int xx = px0 + u - 1;
                v[dy][u] = (yy >= 0 && yy < H && xx >= 0 && xx < W) ? __bfloat162float(hid[((long long)i * H + yy) * W + xx]) : 0.0f;
            }
        }
#pragma unroll
        for (int k = 0; k < 9; ++k)
#pragma unroll
            for (int c = 0; c < kPropCh; ++c) {
                const float wv = w[(c * kPropCh + i) * 9 + k];
#pragma unroll
                for (int q = 0; q < kPropConv2Px; ++q) acc[q][c] = fmaf(wv, v[k / 3][q + k % 3], acc[q][c]);
            }
    }
#pragma unroll
    for (int q = 0; q < kPropConv2Px; ++q)
        if (px0 + q < W)
#pragma unroll
            for (int c = 0; c < kPropCh; ++c) feat[((long long)c * H + py) * W + px0 + q] = __float2bfloat16_rn(acc[q][c]);
}

// Block descriptors: D[y][x][c] = mean of F[c] over the 4x4 quadrant q = c % 4 (rows 4 (q / 2) ..,
// columns 4 (q % 2) ..) of the 8x8 block at (y, x), y <= H - 8, x <= W - 8, bf16 interleaved
// [H - 7][W - 7][16] (32 bytes per position).  Row sums of 4 first (rs, fp32 [16][H][W - 3]).
__global__ void prop_rowsum_kernel(const __nv_bfloat16 *__restrict__ feat, int W, int H, float *__restrict__ rs)
{
    const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y, c = blockIdx.z;
    const int Wr = W - 3;
    if (px >= Wr) return;
    const __nv_bfloat16 *f = feat + ((long long)c * H + py) * W + px;
    float s = 0.0f;
#pragma unroll
    for (int v = 0; v < 4; ++v) s += __bfloat162float(f[v]);
    rs[((long long)c * H + py) * Wr + px] = s;
}

__global__ void prop_desc_kernel(const float *__restrict__ rs, int W, int H, __nv_bfloat16 *__restrict__ desc)
{
    const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y;
    const int Wd = W - 7, Wr = W - 3;
    if (px >= Wd || py >= H - 7) return;
    __nv_bfloat16 out[kPropCh];
#pragma unroll
    for (int c = 0; c < kPropCh; ++c) {
        const int q = c & 3;
        const float *r = rs + ((long long)c * H + py + 4 * (q >> 1)) * Wr + px + 4 * (q & 1);
        float s = 0.0f;
#pragma unroll
        for (int u = 0; u < 4; ++u) s += r[(long long)u * Wr];
        out[c] = __float2bfloat16_rn(s * (1.0f / 16.0f));
    }
    uint4 *d = reinterpret_cast<uint4 *>(desc + ((long long)py * Wd + px) * kPropCh);
    d[0] = *reinterpret_cast<const uint4 *>(out);
    d[1] = *reinterpret_cast<const uint4 *>(out + 8);
}

__device__ __forceinline__ void load_desc(const __nv_bfloat16 *desc, long long idx, float (&v)[kPropCh])
{
    const uint4 *p = reinterpret_cast<const uint4 *>(desc + idx * kPropCh);
    const uint4 q0 = __ldg(p), q1 = __ldg(p + 1);
    const uint32_t u[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        v[2 * i] = __uint_as_float(u[i] << 16);
        v[2 * i + 1] = __uint_as_float(u[i] & 0xffff0000u);
    }
}

// ---- training --------------------------------------------------------------------------------------

// One ranking triplet (reference a, candidates p and n, all block positions of frame f).
struct PropTriplet {
    int f, ay, ax, py, px, ny, nx;
};

// Logistic ranking loss per triplet, L = softplus(s_ap - s_an) with s = |D(a) - D(b)|^2 (the
// triplet is ordered so that p is the closer candidate by exact SSD); accumulates the loss and
// dL/dD into gD (fp32 [frame][H - 7][W - 7][16]).
__global__ void prop_rank_loss_kernel(const PropTriplet *__restrict__ tr, int ntr, const __nv_bfloat16 *__restrict__ desc,
                                      long long dstride, int Wd, float *__restrict__ gD, float scale, float *__restrict__ loss)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (t < ntr) {
        const PropTriplet q = tr[t];
        const long long base = (long long)q.f * dstride;
        const long long ia = base + (long long)q.ay * Wd + q.ax, ip = base + (long long)q.py * Wd + q.px,
                        in = base + (long long)q.ny * Wd + q.nx;
        float a[kPropCh], p[kPropCh], n[kPropCh];
        load_desc(desc, ia, a);
        load_desc(desc, ip, p);
        load_desc(desc, in, n);
        float sp = 0.0f, sn = 0.0f;
#pragma unroll
        for (int c = 0; c < kPropCh; ++c) {
            sp = fmaf(a[c] - p[c], a[c] - p[c], sp);
            sn = fmaf(a[c] - n[c], a[c] - n[c], sn);
        }
        const float z = sp - sn;
        l = z > 20.0f ? z : log1pf(expf(z));
        const float g = scale / (1.0f + expf(-z));          // dL/dz (mean over the batch)
#pragma unroll
        for (int c = 0; c < kPropCh; ++c) {
            const float dap = 2.0f * (a[c] - p[c]), dan = 2.0f * (a[c] - n[c]);
            atomicAdd(gD + ia * kPropCh + c, g * (dap - dan));
            atomicAdd(gD + ip * kPropCh + c, -g * dap);
            atomicAdd(gD + in * kPropCh + c, g * dan);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l * scale);
}

// dF[c](y, x) = (1/16) sum of gD[b][c] over the blocks b whose quadrant c % 4 covers (y, x), fp32
// planar [16][H][W]
__global__ void prop_desc_bwd_kernel(const float *__restrict__ gD, int W, int H, float *__restrict__ dF)
{
    const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y;
    if (px >= W) return;
    const int Wd = W - 7, Hd = H - 7;
    float s[kPropCh];
#pragma unroll
    for (int c = 0; c < kPropCh; ++c) s[c] = 0.0f;
    for (int u = 0; u < 8; ++u) {
        const int by = py - u;
        if (by < 0 || by >= Hd) continue;
        for (int v = 0; v < 8; ++v) {
            const int bx = px - v;
            if (bx < 0 || bx >= Wd) continue;
            const int q = 2 * (u >> 2) + (v >> 2);       // quadrant of the block that holds (y, x)
            const float *g = gD + ((long long)by * Wd + bx) * kPropCh;
#pragma unroll
            for (int c = q; c < kPropCh; c += 4) s[c] += g[c];
        }
    }
#pragma unroll
    for (int c = 0; c < kPropCh; ++c) dF[((long long)c * H + py) * W + px] = s[c] * (1.0f / 16.0f);
}

// conv2 backward: dW2[c][i][k] += dF[c](p) H[i](p + k), db2[c] += dF[c](p) (block partial sums in
// shared memory, then one atomic per weight); dH[i](p) = sum_{c,k} w2[c][i][k] dF[c](p - k),
// masked by the ReLU (H > 0), fp32 planar [16][H][W].
__global__ void prop_conv2_bwd_kernel(const __nv_bfloat16 *__restrict__ hid, const float *__restrict__ dF, int W, int H,
                                      const float *__restrict__ wt, float *__restrict__ gw, float *__restrict__ dH)
{
    __shared__ float w[kPropCh * kPropCh * 9];
    __shared__ float gs[kPropCh * kPropCh * 9 + kPropCh];
    for (int i = threadIdx.x; i < kPropCh * kPropCh * 9; i += blockDim.x) w[i] = wt[kPropW2 + i];
    for (int i = threadIdx.x; i < kPropCh * kPropCh * 9 + kPropCh; i += blockDim.x) gs[i] = 0.0f;
    __syncthreads();
    const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y;
    const bool in = px < W;
    float df[kPropCh];
#pragma unroll
    for (int c = 0; c < kPropCh; ++c) df[c] = in ? dF[((long long)c * H + py) * W + px] : 0.0f;
    // weight gradients (warps whose pixels carry no gradient skip them)
    bool any = false;
#pragma unroll
    for (int c = 0; c < kPropCh; ++c) any = any || df[c] != 0.0f;
    if (__any_sync(0xffffffffu, any))
    for (int i = 0; i < kPropCh; ++i) {
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            const int yy = py + k / 3 - 1, xx = px + k % 3 - 1;
            const float h = (in && yy >= 0 && yy < H && xx >= 0 && xx < W) ? __bfloat162float(hid[((long long)i * H + yy) * W + xx]) : 0.0f;
#pragma unroll
            for (int c = 0; c < kPropCh; ++c) {
                float g = df[c] * h;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
                if ((threadIdx.x & 31) == 0) atomicAdd(&gs[(c * kPropCh + i) * 9 + k], g);
            }
        }
    }
#pragma unroll
    for (int c = 0; c < kPropCh; ++c) {
        float g = df[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&gs[kPropCh * kPropCh * 9 + c], g);
    }
    // input gradient (transposed convolution), masked by the ReLU
    if (in) {
        for (int i = 0; i < kPropCh; ++i) {
            float s = 0.0f;
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                const int yy = py - (k / 3 - 1), xx = px - (k % 3 - 1);
                if (yy < 0 || yy >= H || xx < 0 || xx >= W) continue;
#pragma unroll
                for (int c = 0; c < kPropCh; ++c) s = fmaf(w[(c * kPropCh + i) * 9 + k], dF[((long long)c * H + yy) * W + xx], s);
            }
            const float h = __bfloat162float(hid[((long long)i * H + py) * W + px]);
            dH[((long long)i * H + py) * W + px] = h > 0.0f ? s : 0.0f;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kPropCh * kPropCh * 9 + kPropCh; i += blockDim.x) atomicAdd(gw + kPropW2 + i, gs[i]);
}

// conv1 backward: dW1[c][k] += dH[c](p) x(p + k), db1[c] += dH[c](p)
__global__ void prop_conv1_bwd_kernel(const float *__restrict__ x, int ld, const float *__restrict__ dH, int W, int H,
                                      float *__restrict__ gw)
{
    __shared__ float gs[160];
    for (int i = threadIdx.x; i < 160; i += blockDim.x) gs[i] = 0.0f;
    __syncthreads();
    const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y;
    const bool in = px < W;
    float v[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const int yy = py + k / 3 - 1, xx = px + k % 3 - 1;
        v[k] = (in && yy >= 0 && yy < H && xx >= 0 && xx < W) ? x[(long long)yy * ld + xx] : 0.0f;
    }
#pragma unroll
    for (int c = 0; c < kPropCh; ++c) {
        const float d = in ? dH[((long long)c * H + py) * W + px] : 0.0f;
#pragma unroll
        for (int k = 0; k < 10; ++k) {
            float g = k < 9 ? d * v[k] : d;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
            if ((threadIdx.x & 31) == 0) atomicAdd(&gs[k < 9 ? c * 9 + k : kPropB1 + c], g);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 160; i += blockDim.x) atomicAdd(gw + kPropW1 + i, gs[i]);
}

// Adam step (bias-corrected), one thread per weight
__global__ void prop_adam_kernel(float *__restrict__ wt, const float *__restrict__ g, float *__restrict__ m,
                                 float *__restrict__ v, float lr, float b1t, float b2t)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kPropWeights) return;
    const float gi = g[i];
    m[i] = 0.9f * m[i] + 0.1f * gi;
    v[i] = 0.999f * v[i] + 0.001f * gi * gi;
    const float mh = m[i] / (1.0f - b1t), vh = v[i] / (1.0f - b2t);
    wt[i] -= lr * mh / (sqrtf(vh) + 1e-8f);
}

// ---- matching with proposals -------------------------------------------------------------------

// One warp per reference block, CTA = a row of a.warps blocks (window staged as in bm_full_kernel).
// Every lattice candidate (and the trailing (0, 0) one) is scored by |D(ref) - D(cand)|^2; the
// nprop best scores are proposals; their exact SSDs (the reference's order) decide validity and the
// order of the list.
__global__ void __launch_bounds__(256) bm_learned_kernel(BMArgs a, const __nv_bfloat16 *__restrict__ desc, int nprop)
{
    extern __shared__ float smem[];
    const int lane = (int)lane_id();
    const int warp = threadIdx.x >> 5;
    const int f = blockIdx.z;
    const int by = blockIdx.y;
    const int bx0 = blockIdx.x * a.warps;
    const int bx = bx0 + warp;
    const float *plane = a.ref + (long long)f * a.frame_stride;
    const int Wd = a.W - 7, Hd = a.H - 7;
    const __nv_bfloat16 *dsc = desc + (long long)f * Hd * Wd * kPropCh;

    const int j = a.scan_y[by];
    const int xfirst = a.scan_x[bx0];
    const int xlast = a.scan_x[min(bx0 + a.warps, a.nbx) - 1];
    const int wy0 = max(0, j - a.range), wy1 = min(a.H, j + a.range + 8);
    const int wx0 = max(0, xfirst - a.range), wx1 = min(a.W, xlast + a.range + 8);
    const int ww = wx1 - wx0;
    const int wp = a.win_pitch;
    float *win = smem;
    for (int yy = warp; yy < wy1 - wy0; yy += (int)(blockDim.x >> 5)) {
        const float *src = plane + (long long)(wy0 + yy) * a.ld + wx0;
        float *dst = win + yy * wp;
        for (int xx = lane; xx < ww; xx += 32) tc::cp_async4(dst + xx, src + xx);
    }
    tc::cp_async_wait_all();
    __syncthreads();
    if (bx >= a.nbx) return;

    float *sd = smem + a.win_h * wp + warp * prop_warp_floats(a.cand_cap);
    uint32_t *list = reinterpret_cast<uint32_t *>(sd + a.cand_cap);
    const int i = a.scan_x[bx];
    const size_t ob = ((size_t)f * a.nby + by) * a.nbx + bx;
    const int G = a.G, K = G - 1;
    uint32_t *opos = a.out_pos + ob * G;
    if (lane == 0) {
        opos[0] = pack_yx(j, i);
        if (a.out_key) a.out_key[ob * G] = 0.0f;
    }
    if (G == 1) {
        if (lane == 0) a.out_n[ob] = 1;
        return;
    }
    const int s = a.step;
    const int t = search_boundary(j, 0, a.range, s);
    const int b = search_boundary(j, a.H - 8, a.range, s);
    const int l = search_boundary(i, 0, a.range, s);
    const int r = search_boundary(i, a.W - 8, a.range, s);
    const int ncols = (r - l) / s + 1;
    const int clat = ((b - t) / s + 1) * ncols;
    const int ctot = clat + 1;
    float da[kPropCh];
    load_desc(dsc, (long long)j * Wd + i, da);
    // scores of every candidate (the block itself excluded)
    for (int c = lane; c < ctot; c += 32) {
        int cy = 0, cx = 0;
        if (c < clat) {
            const int ry = c / ncols;
            cy = t + ry * s;
            cx = l + (c - ry * ncols) * s;
        }
        float dc[kPropCh];
        load_desc(dsc, (long long)cy * Wd + cx, dc);
        float sc = 0.0f;
#pragma unroll
        for (int k = 0; k < kPropCh; ++k) sc = fmaf(da[k] - dc[k], da[k] - dc[k], sc);
        sd[c] = (c < clat && cy == j && cx == i) ? 3.0e38f : sc;
    }
    __syncwarp();
    // the nprop (<= 128) best scores: four per lane, a 128-entry sort gives a cut at or above the
    // true nprop-th score; every candidate at or below it (at most 128 kept) sorted, the first nprop
    uint64_t bb[4] = {~0ull, ~0ull, ~0ull, ~0ull};
    for (int c0 = 0; c0 < ctot; c0 += 32) {
        const int c = c0 + ((lane + 7 * (c0 >> 5)) & 31);
        if (c >= ctot) continue;
        uint64_t v = compose(sd[c], (uint32_t)c);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const uint64_t lo = v < bb[e] ? v : bb[e];
            v = v < bb[e] ? bb[e] : v;
            bb[e] = lo;
        }
    }
    warp_bitonic_u64<4>(bb);
    const int pr = min(nprop, 128) - 1;                 // rank of the last proposal
    uint64_t cv[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) cv[e] = __shfl_sync(0xffffffffu, bb[e], pr & 31);
    uint64_t cut = cv[pr >> 5];
    const unsigned lt = (1u << lane) - 1u;
    auto collect = [&]() {
        int cnt = 0;
        for (int c0 = 0; c0 < ctot; c0 += 32) {
            const int c = c0 + lane;
            const bool in = c < ctot && compose(sd[c], (uint32_t)c) <= cut;
            const unsigned msk = __ballot_sync(0xffffffffu, in);
            if (in && cnt + __popc(msk & lt) < 128) list[cnt + __popc(msk & lt)] = (uint32_t)c;
            cnt += __popc(msk);
        }
        __syncwarp();
        return cnt;
    };
    int m = collect();
    if (m > 128) {
        // More than 128 candidates at or below the cut (the union of per-lane lists can put it
        // well above the true nprop-th score): radix selection of the (pr + 1)-th smallest score
        // (scores are non-negative, so their bit patterns order like the values), 7 bits at a
        // time with a 128-bin histogram in the list buffer; then every candidate below that
        // score and, of those equal to it, the first ones in scan order -- exactly the pr + 1
        // smallest (score, index) keys.
        if (lane == 0 && a.stats) atomicAdd(a.stats + 1, 1ull);
        int rank = pr;
        const uint32_t prefix = warp_radix_cut(sd, ctot, rank, reinterpret_cast<int *>(list));
        // prefix = the score of rank pr; rank = its position among the candidates of that score
        int cnt = 0, eq = 0;
        for (int c0 = 0; c0 < ctot; c0 += 32) {
            const int c = c0 + lane;
            const uint32_t u = c < ctot ? __float_as_uint(sd[c]) : 0xffffffffu;
            const bool isq = c < ctot && u == prefix;
            const unsigned mq = __ballot_sync(0xffffffffu, isq);
            const bool in = c < ctot && (u < prefix || (isq && eq + __popc(mq & lt) <= rank));
            const unsigned msk = __ballot_sync(0xffffffffu, in);
            if (in) list[cnt + __popc(msk & lt)] = (uint32_t)c;
            cnt += __popc(msk);
            eq += __popc(mq);
        }
        __syncwarp();
        m = cnt;
    }
    m = min(m, 128);
    if (m > pr + 1) {
        uint64_t sv[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int idx = lane + 32 * e;
            sv[e] = idx < m ? compose(sd[list[idx]], list[idx]) : ~0ull;
        }
        warp_bitonic_u64<4>(sv);
        __syncwarp();
#pragma unroll
        for (int e = 0; e < 4; ++e) list[lane + 32 * e] = (uint32_t)sv[e];
        __syncwarp();
        m = pr + 1;
    }
    if (a.out_prop) {
        uint32_t *op = a.out_prop + ob * nprop;
        for (int e = lane; e < nprop; e += 32) op[e] = e < m ? list[e] : 0xffffffffu;
    }
    // exact distances of the proposals, valid ones ordered by (key, scan index)
    const float *rp = win + (j - wy0) * wp + (i - wx0);
    uint64_t v[4] = {~0ull, ~0ull, ~0ull, ~0ull};
    int nval = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int idx = lane + 32 * e;
        if (idx < m) {
            const uint32_t c = list[idx];
            float d;
            if ((int)c >= clat) {
                d = exact_ssd8(rp, wp, plane, a.ld);
            } else {
                const int ry = (int)c / ncols, cc = (int)c - ry * ncols;
                d = exact_ssd8(rp, wp, win + (t + ry * s - wy0) * wp + (l + cc * s - wx0), wp);
            }
            if (dist_valid(d, a.thSSE)) {
                v[e] = compose(dist_to_key(d, a.distMul), c);
                ++nval;
            }
        }
    }
    nval = warp_sum(nval);
    if (m <= 64) warp_bitonic_u64<2>(*reinterpret_cast<uint64_t (*)[2]>(v));
    else warp_bitonic_u64<4>(v);
    const int nout = min(nval, K);
    if (lane < nout) {
        const uint32_t c = (uint32_t)v[0];
        uint32_t pos = pack_yx(0, 0);
        if ((int)c < clat) {
            const int ry = (int)c / ncols, cc = (int)c - ry * ncols;
            pos = pack_yx(t + ry * s, l + cc * s);
        }
        opos[1 + lane] = pos;
        if (a.out_key) a.out_key[ob * G + 1 + lane] = __uint_as_float((uint32_t)(v[0] >> 32));
    }
    if (lane == 0) a.out_n[ob] = 1 + nout;
}

// Training triplets: reference block b of frame f (uniform over the lattice of block positions),
// p = a random entry among the first 16 of its exhaustive list (ranks 1 .. 15), n = half of the
// time a later entry of the list (ranks 16 .., the hard negatives), else a uniform candidate of
// its search window; p and n ordered by exact SSD so that p is the closer one.
__device__ __forceinline__ uint32_t prop_hash(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__global__ void prop_sample_kernel(const float *__restrict__ frames, long long fstride, int ld, int W, int H, int nframes,
                                   const uint32_t *__restrict__ lists, const int *__restrict__ counts, int G,
                                   const int *__restrict__ sy, const int *__restrict__ sx, int nby, int nbx, int range,
                                   uint32_t seed, PropTriplet *__restrict__ out, int ntr)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntr) return;
    uint32_t h = prop_hash(seed * 0x9e3779b9u + (uint32_t)t);
    const int f = (int)(h % (uint32_t)nframes);
    h = prop_hash(h);
    const int by = (int)(h % (uint32_t)nby);
    h = prop_hash(h);
    const int bx = (int)(h % (uint32_t)nbx);
    const long long ob = ((long long)f * nby + by) * nbx + bx;
    const int ay = sy[by], ax = sx[bx];
    const int n = counts[ob];
    h = prop_hash(h);
    int py = ay, px = ax;
    const int npos = min(n, 16);
    if (npos > 1) {
        const uint32_t pk = lists[ob * G + 1 + (int)(h % (uint32_t)(npos - 1))];
        py = unpack_y(pk);
        px = unpack_x(pk);
    }
    h = prop_hash(h);
    int qy, qx;
    if ((h & 1u) && n > 16) {
        const uint32_t pk = lists[ob * G + 16 + (int)((h >> 1) % (uint32_t)(n - 16))];
        qy = unpack_y(pk);
        qx = unpack_x(pk);
    } else {
        const int y0 = max(0, ay - range), y1 = min(H - 8, ay + range);
        const int x0 = max(0, ax - range), x1 = min(W - 8, ax + range);
        qy = y0 + (int)((h >> 1) % (uint32_t)(y1 - y0 + 1));
        h = prop_hash(h);
        qx = x0 + (int)(h % (uint32_t)(x1 - x0 + 1));
    }
    const float *pl = frames + (long long)f * fstride;
    const float *ra = pl + (long long)ay * ld + ax;
    const float dp = exact_ssd8(ra, ld, pl + (long long)py * ld + px, ld);
    const float dq = exact_ssd8(ra, ld, pl + (long long)qy * ld + qx, ld);
    PropTriplet q;
    q.f = f;
    q.ay = ay;
    q.ax = ax;
    if (dp <= dq) {
        q.py = py; q.px = px; q.ny = qy; q.nx = qx;
    } else {
        q.py = qy; q.px = qx; q.ny = py; q.nx = px;
    }
    out[t] = q;
}

}  // namespace bm3d
