// convert.cuh -- K5: per-pixel kernels around the hot path.
//   * ingest / egress: integer<->float range conversion and RGB<->OPP matrix conversion, with
//     the gains and offsets computed on the host exactly as include/Conversion.hpp:36-417 does
//     (RangeConvert, ConvertToY, MatrixConvert_RGB2YUV / _YUV2RGB, OPP branches);
//   * finalize: den = B x B box sum of the per-origin weights, out = num / den
//     (source/BM3D_Base.cpp:348-351, 455-469);
//   * VAggregate: num = sum_f num_f, den = sum_f den_f, out = num / den over the temporal window
//     (source/VAggregate.cpp:93-160, slot selection :194-202).
#pragma once

#include "common.cuh"
#include "args.h"

namespace bm3d {



__device__ __forceinline__ float load_sample(const PlanePtr &p, int kind, int y, int x)
{
    const char *row = static_cast<const char *>(p.ptr) + (long long)y * p.stride;
    if (kind == SK_U8) return (float)reinterpret_cast<const uint8_t *>(row)[x];
    if (kind == SK_U16) return (float)reinterpret_cast<const uint16_t *>(row)[x];
    return reinterpret_cast<const float *>(row)[x];
}

__device__ __forceinline__ void store_sample(const PlanePtr &p, int kind, int y, int x, float v)
{
    char *row = static_cast<char *>(p.ptr) + (long long)y * p.stride;
    if (kind == SK_U8) reinterpret_cast<uint8_t *>(row)[x] = (uint8_t)v;       // truncation, as static_cast
    else if (kind == SK_U16) reinterpret_cast<uint16_t *>(row)[x] = (uint16_t)v;
    else reinterpret_cast<float *>(row)[x] = v;
}

__device__ __forceinline__ float clip_ref(float v, float lo, float hi)
{
    // Clip() of include/Helper.h:395-399
    return v <= lo ? lo : v >= hi ? hi : v;
}



__global__ void convert_kernel(ConvProgram pr, const PlanePtr *in, const PlanePtr *out)
{
    const int f = blockIdx.z;
    const int y = blockIdx.y;
    const PlanePtr *pi = in + f * pr.nin;
    const PlanePtr *po = out + f * pr.nout;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < pr.W; x += gridDim.x * blockDim.x) {
        if (pr.raw) {
            for (int c = 0; c < pr.nin; ++c) {
                if (!po[c].ptr) continue;
                const char *si = static_cast<const char *>(pi[c].ptr) + (long long)y * pi[c].stride;
                char *so = static_cast<char *>(po[c].ptr) + (long long)y * po[c].stride;
                if (pr.in_kind == SK_U8) reinterpret_cast<uint8_t *>(so)[x] = reinterpret_cast<const uint8_t *>(si)[x];
                else if (pr.in_kind == SK_U16) reinterpret_cast<uint16_t *>(so)[x] = reinterpret_cast<const uint16_t *>(si)[x];
                else reinterpret_cast<float *>(so)[x] = reinterpret_cast<const float *>(si)[x];
            }
        } else if (pr.mode == 0) {
            for (int c = 0; c < pr.nin; ++c) {
                if (!po[c].ptr) continue;
                const LinearOp &o = pr.op[c];
                float t = __fadd_rn(__fmul_rn(load_sample(pi[c], pr.in_kind, y, x), o.gain), o.offset);
                if (o.clip) t = clip_ref(t, o.lo, o.hi);
                store_sample(po[c], pr.out_kind, y, x, t);
            }
        } else if (pr.mode == 1 || pr.mode == 2) {
            const float R = load_sample(pi[0], pr.in_kind, y, x);
            const float Gc = load_sample(pi[1], pr.in_kind, y, x);
            const float Bc = load_sample(pi[2], pr.in_kind, y, x);
            float t = __fadd_rn(__fmul_rn(__fadd_rn(__fadd_rn(R, Gc), Bc), pr.op[0].gain), pr.op[0].offset);
            if (pr.op[0].clip) t = clip_ref(t, pr.op[0].lo, pr.op[0].hi);
            store_sample(po[0], pr.out_kind, y, x, t);
            if (pr.mode == 1) {
                float u = __fadd_rn(__fmul_rn(__fsub_rn(R, Bc), pr.op[1].gain), pr.op[1].offset);
                if (pr.op[1].clip) u = clip_ref(u, pr.op[1].lo, pr.op[1].hi);
                if (po[1].ptr) store_sample(po[1], pr.out_kind, y, x, u);
                float v = __fadd_rn(__fmul_rn(__fadd_rn(__fsub_rn(R, __fmul_rn(Gc, 2.0f)), Bc), pr.op[2].gain), pr.op[2].offset);
                if (pr.op[2].clip) v = clip_ref(v, pr.op[2].lo, pr.op[2].hi);
                if (po[2].ptr) store_sample(po[2], pr.out_kind, y, x, v);
            }
        } else {
            const float Y = load_sample(pi[0], pr.in_kind, y, x);
            const float U = load_sample(pi[1], pr.in_kind, y, x);
            const float V = load_sample(pi[2], pr.in_kind, y, x);
            const float *k = pr.coef;
            float r = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(k[0], Y), __fmul_rn(k[1], U)), __fmul_rn(k[2], V)), pr.off[0]);
            float g = __fadd_rn(__fadd_rn(__fmul_rn(k[3], Y), __fmul_rn(k[5], V)), pr.off[1]);
            float b = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(k[6], Y), __fmul_rn(k[7], U)), __fmul_rn(k[8], V)), pr.off[2]);
            if (pr.op[0].clip) {
                r = clip_ref(r, pr.op[0].lo, pr.op[0].hi);
                g = clip_ref(g, pr.op[0].lo, pr.op[0].hi);
                b = clip_ref(b, pr.op[0].lo, pr.op[0].hi);
            }
            store_sample(po[0], pr.out_kind, y, x, r);
            store_sample(po[1], pr.out_kind, y, x, g);
            store_sample(po[2], pr.out_kind, y, x, b);
        }
    }
}


// Tile of the denominator (the B x B box sum of the per-origin weight map wm) for output rows
// [ty0, ty0 + kFinTH) and columns [tx0, tx0 + kFinTW): the weight region with its (B - 1) halo is
// staged in shared memory, summed along x, then along y (2B additions per pixel instead of B^2).
// On return den[r * kFinTW + c] holds the denominator of pixel (ty0 + r, tx0 + c).
constexpr int kFinTH = 32, kFinTW = 64;

__host__ __device__ inline int finalize_smem_floats(int B)
{
    return (kFinTH + B - 1) * (kFinTW + B - 1) + (kFinTH + B - 1) * kFinTW + kFinTH * kFinTW;
}

__device__ __forceinline__ float *box_den_tile(float *sm, const float *wm, int ld, int H, int W, int B, int ty0, int tx0)
{
    const int RH = kFinTH + B - 1, RW = kFinTW + B - 1;
    float *reg = sm;
    float *hs = sm + RH * RW;
    float *den = hs + RH * kFinTW;
    for (int e = threadIdx.x; e < RH * RW; e += blockDim.x) {
        const int r = e / RW, c = e - r * RW;
        const int yy = ty0 - (B - 1) + r, xx = tx0 - (B - 1) + c;
        reg[e] = (yy >= 0 && xx >= 0 && yy < H && xx < W) ? wm[(long long)yy * ld + xx] : 0.0f;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < RH * kFinTW; e += blockDim.x) {
        const int r = e / kFinTW, c = e - r * kFinTW;
        float v = 0.0f;
        for (int k = 0; k < B; ++k) v = __fadd_rn(v, reg[r * RW + c + k]);
        hs[e] = v;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kFinTH * kFinTW; e += blockDim.x) {
        const int r = e / kFinTW, c = e - r * kFinTW;
        float v = 0.0f;
        for (int k = 0; k < B; ++k) v = __fadd_rn(v, hs[(r + k) * kFinTW + c]);
        den[e] = v;
    }
    __syncthreads();
    return den;
}

// grid (tiles along x, tiles along y, frames * 3 planes)
__global__ void __launch_bounds__(256) finalize_kernel(FinalizeArgs a)
{
    extern __shared__ float fsm[];
    const int f = blockIdx.z / 3, p = blockIdx.z % 3;
    if (!a.process[p]) return;
    const int ty0 = blockIdx.y * kFinTH, tx0 = blockIdx.x * kFinTW;
    const long long fo = (long long)f * a.frame_stride;
    const float *den = box_den_tile(fsm, a.wmap[p] + fo, a.ld, a.H, a.W, a.B, ty0, tx0);
    const float *nm = a.num[p] + fo;
    float *o = a.out[p] + fo;
    for (int e = threadIdx.x; e < kFinTH * kFinTW; e += blockDim.x) {
        const int r = e / kFinTW, c = e - r * kFinTW;
        const int y = ty0 + r, x = tx0 + c;
        if (y < a.H && x < a.W) o[(long long)y * a.ld + x] = __fdiv_rn(nm[(long long)y * a.ld + x], den[e]);
    }
}


__global__ void vaggregate_kernel(VAggArgs a)
{
    const int f = blockIdx.z;
    const int p = blockIdx.y % 3;
    if (!a.process[p]) return;
    const int y = blockIdx.y / 3;
    const int frames = a.nframes[f];
    const int boff = a.b_off[f];
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < a.W; x += gridDim.x * blockDim.x) {
        float num = 0.0f, den = 0.0f;
        for (int i = 0, o = a.radius - boff; i < frames; ++i, --o) {
            const PlanePtr &pp = a.in[(f * a.frames_max + i) * 3 + p];
            const char *base = static_cast<const char *>(pp.ptr);
            const float *nrow = reinterpret_cast<const float *>(base + ((long long)o * 2 * a.H + y) * pp.stride);
            const float *drow = reinterpret_cast<const float *>(base + ((long long)(o * 2 + 1) * a.H + y) * pp.stride);
            num = __fadd_rn(num, nrow[x]);
            den = __fadd_rn(den, drow[x]);
        }
        a.out[p][(long long)f * a.frame_stride + (long long)y * a.ld + x] = __fdiv_rn(num, den);
    }
}

// grid (tiles along x, slots * tiles along y, frames * 3 planes)
__global__ void __launch_bounds__(256) vstack_kernel(VStackArgs a)
{
    extern __shared__ float fsm[];
    const int f = blockIdx.z / 3;
    const int p = blockIdx.z % 3;
    if (!a.process[p]) return;
    const int tiles_y = (a.H + kFinTH - 1) / kFinTH;
    const int s = blockIdx.y / tiles_y;
    const int ty0 = (blockIdx.y - s * tiles_y) * kFinTH, tx0 = blockIdx.x * kFinTW;
    const long long so = ((long long)f * a.slots + s) * a.slot_stride;
    const float *den = box_den_tile(fsm, a.wmap[p] + so, a.ld, a.H, a.W, a.B, ty0, tx0);
    const float *nm = a.num[p] + so;
    const PlanePtr &o = a.out[f * 3 + p];
    for (int e = threadIdx.x; e < kFinTH * kFinTW; e += blockDim.x) {
        const int r = e / kFinTW, c = e - r * kFinTW;
        const int y = ty0 + r, x = tx0 + c;
        if (y >= a.H || x >= a.W) continue;
        float *nrow = reinterpret_cast<float *>(static_cast<char *>(o.ptr) + ((long long)(2 * s) * a.H + y) * o.stride);
        float *drow = reinterpret_cast<float *>(static_cast<char *>(o.ptr) + ((long long)(2 * s + 1) * a.H + y) * o.stride);
        nrow[x] = nm[(long long)y * a.ld + x];
        drow[x] = den[e];
    }
}

}  // namespace bm3d
