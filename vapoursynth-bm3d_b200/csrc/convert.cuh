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


__global__ void finalize_kernel(FinalizeArgs a)
{
    const int f = blockIdx.z;
    const int p = blockIdx.y % 3;
    if (!a.process[p]) return;
    const int y = blockIdx.y / 3;
    const long long fo = (long long)f * a.frame_stride;
    const float *wm = a.wmap[p] + fo;
    const float *nm = a.num[p] + fo;
    float *o = a.out[p] + fo;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < a.W; x += gridDim.x * blockDim.x) {
        float den = 0.0f;
        const int y0 = max(0, y - a.B + 1), x0 = max(0, x - a.B + 1);
        for (int yy = y0; yy <= y; ++yy)
            for (int xx = x0; xx <= x; ++xx) den = __fadd_rn(den, wm[(long long)yy * a.ld + xx]);
        o[(long long)y * a.ld + x] = __fdiv_rn(nm[(long long)y * a.ld + x], den);
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

__global__ void vstack_kernel(VStackArgs a)
{
    const int f = blockIdx.z / 3;
    const int p = blockIdx.z % 3;
    if (!a.process[p]) return;
    const int s = blockIdx.y / a.H;
    const int y = blockIdx.y - s * a.H;
    const long long so = ((long long)f * a.slots + s) * a.slot_stride;
    const float *wm = a.wmap[p] + so;
    const float *nm = a.num[p] + so;
    const PlanePtr &o = a.out[f * 3 + p];
    float *nrow = reinterpret_cast<float *>(static_cast<char *>(o.ptr) + ((long long)(2 * s) * a.H + y) * o.stride);
    float *drow = reinterpret_cast<float *>(static_cast<char *>(o.ptr) + ((long long)(2 * s + 1) * a.H + y) * o.stride);
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < a.W; x += gridDim.x * blockDim.x) {
        float den = 0.0f;
        const int y0 = max(0, y - a.B + 1), x0 = max(0, x - a.B + 1);
        for (int yy = y0; yy <= y; ++yy)
            for (int xx = x0; xx <= x; ++xx) den = __fadd_rn(den, wm[(long long)yy * a.ld + xx]);
        nrow[x] = nm[(long long)y * a.ld + x];
        drow[x] = den;
    }
}

}  // namespace bm3d
