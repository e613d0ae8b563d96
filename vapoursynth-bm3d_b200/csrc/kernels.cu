// kernels.cu -- the single CUDA translation unit holding every sm_100a kernel of the library
// (block matching, predictive search, collaborative filter, conversions) and their launchers.

#include "common.cuh"
#include "select.cuh"
#include "bm.cuh"
#include "bm_tc.cuh"
#include "proposal.cuh"
#include "vbm.cuh"
#include "cf.cuh"
#include "cf_tc.cuh"
#include "fp64.cuh"
#include "convert.cuh"
#include "launch.h"
#include "params.h"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

namespace bm3d {

// Every kernel launch of the library goes through a launcher below and is counted here.
static std::atomic<unsigned long long> g_launches{0};
unsigned long long launch_count() { return g_launches.load(); }
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
#define COUNT_LAUNCH() g_launches.fetch_add(1, std::memory_order_relaxed)

cudaError_t upload_odd_tables(const float *host_odd_all)
{
    return cudaMemcpyToSymbol(c_odd, host_odd_all, sizeof(float) * kOddConstFloats);
}

template <typename K>
static cudaError_t allow_smem(K kernel, size_t bytes)
{
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

cudaError_t launch_bm_tc(const BMArgs &a, const BmtLayout &L, int nframes, cudaStream_t s)
{
    dim3 grid((a.nbx + L.nrc - 1) / L.nrc, a.nby, nframes);
    // at most two CTAs per SM, so that their 256 tensor-memory columns each are never contended
    const size_t smem = std::max<size_t>((size_t)L.bytes, 76 * 1024);
    cudaError_t e;
    if ((e = allow_smem(bm_tc_kernel, smem)) != cudaSuccess) return e;
    COUNT_LAUNCH();
    bm_tc_kernel<<<grid, kBmtThreads, smem, s>>>(a, L);
    return cudaGetLastError();
}

// ---- learned proposal ----------------------------------------------------------------------------

int prop_triplet_bytes() { return (int)sizeof(PropTriplet); }

cudaError_t launch_prop_features(const float *x, int ld, int W, int H, const float *wt, void *hid, void *feat, float *rs,
                                 void *desc, cudaStream_t s)
{
    if (W < 8 || H < 8) return cudaErrorInvalidValue;
    auto *h = static_cast<__nv_bfloat16 *>(hid);
    auto *f = static_cast<__nv_bfloat16 *>(feat);
    const dim3 blk(128);
    COUNT_LAUNCH();
    prop_conv1_kernel<<<dim3((W + 127) / 128, H), blk, 0, s>>>(x, ld, W, H, wt, h);
    COUNT_LAUNCH();
    prop_conv2_kernel<<<dim3((W + 128 * kPropConv2Px - 1) / (128 * kPropConv2Px), H), blk, 0, s>>>(h, W, H, wt, f);
    COUNT_LAUNCH();
    prop_rowsum_kernel<<<dim3((W - 3 + 127) / 128, H, kPropCh), blk, 0, s>>>(f, W, H, rs);
    COUNT_LAUNCH();
    prop_desc_kernel<<<dim3((W - 7 + 127) / 128, H - 7), blk, 0, s>>>(rs, W, H, static_cast<__nv_bfloat16 *>(desc));
    return cudaGetLastError();
}

cudaError_t launch_prop_loss(const void *triplets, int ntr, const void *desc, long long dstride, int Wd, float *gD,
                             float scale, float *loss, cudaStream_t s)
{
    COUNT_LAUNCH();
    prop_rank_loss_kernel<<<(ntr + 127) / 128, 128, 0, s>>>(static_cast<const PropTriplet *>(triplets), ntr,
                                                           static_cast<const __nv_bfloat16 *>(desc), dstride, Wd, gD, scale, loss);
    return cudaGetLastError();
}

cudaError_t launch_prop_backward(const float *x, int ld, int W, int H, const float *wt, const void *hid, const float *gD,
                                 float *dF, float *dH, float *gw, cudaStream_t s)
{
    const dim3 blk(128), grd((W + 127) / 128, H);
    COUNT_LAUNCH();
    prop_desc_bwd_kernel<<<grd, blk, 0, s>>>(gD, W, H, dF);
    COUNT_LAUNCH();
    prop_conv2_bwd_kernel<<<grd, blk, 0, s>>>(static_cast<const __nv_bfloat16 *>(hid), dF, W, H, wt, gw, dH);
    COUNT_LAUNCH();
    prop_conv1_bwd_kernel<<<grd, blk, 0, s>>>(x, ld, dH, W, H, gw);
    return cudaGetLastError();
}

cudaError_t launch_prop_adam(float *wt, const float *g, float *m, float *v, float lr, float b1t, float b2t, cudaStream_t s)
{
    COUNT_LAUNCH();
    prop_adam_kernel<<<(kPropWeights + 255) / 256, 256, 0, s>>>(wt, g, m, v, lr, b1t, b2t);
    return cudaGetLastError();
}

cudaError_t launch_prop_sample(const float *frames, long long fstride, int ld, int W, int H, int nframes, const uint32_t *lists,
                               const int *counts, int G, const int *sy, const int *sx, int nby, int nbx, int range,
                               uint32_t seed, void *out, int ntr, cudaStream_t s)
{
    COUNT_LAUNCH();
    prop_sample_kernel<<<(ntr + 127) / 128, 128, 0, s>>>(frames, fstride, ld, W, H, nframes, lists, counts, G, sy, sx, nby,
                                                        nbx, range, seed, static_cast<PropTriplet *>(out), ntr);
    return cudaGetLastError();
}

cudaError_t launch_bm_learned(const BMArgs &a, const void *desc, int nprop, int nframes, size_t smem, cudaStream_t s)
{
    if (a.B != 8 || a.G > 32) return cudaErrorInvalidValue;
    dim3 grid((a.nbx + a.warps - 1) / a.warps, a.nby, nframes);
    cudaError_t e;
    if ((e = allow_smem(bm_learned_kernel, smem)) != cudaSuccess) return e;
    COUNT_LAUNCH();
    bm_learned_kernel<<<grid, 32 * a.warps, smem, s>>>(a, static_cast<const __nv_bfloat16 *>(desc), nprop);
    return cudaGetLastError();
}

cudaError_t launch_bm_full(const BMArgs &a, int nframes, size_t smem, cudaStream_t s)
{
    dim3 grid((a.nbx + a.warps - 1) / a.warps, a.nby, nframes);
    dim3 block(32 * a.warps);
    cudaError_t e;
    if (a.B == 8) {
        if ((e = allow_smem(bm_full_kernel<8>, smem)) != cudaSuccess) return e;
        COUNT_LAUNCH();
        bm_full_kernel<8><<<grid, block, smem, s>>>(a);
    } else {
        if ((e = allow_smem(bm_full_kernel<0>, smem)) != cudaSuccess) return e;
        COUNT_LAUNCH();
        bm_full_kernel<0><<<grid, block, smem, s>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t launch_vbm_predict(const VBMArgs &a, int nframes, size_t smem, cudaStream_t s)
{
    dim3 grid((a.nbx + a.warps - 1) / a.warps, a.nby, nframes);
    dim3 block(32 * a.warps);
    cudaError_t e;
    if ((e = allow_smem(vbm_predict_kernel, smem)) != cudaSuccess) return e;
    COUNT_LAUNCH();
    vbm_predict_kernel<<<grid, block, smem, s>>>(a);
    return cudaGetLastError();
}

int cf_fast_supported(int B, int G) { return B == 8 && (G == 8 || G == 16 || G == 32); }

template <int G, bool W>
static cudaError_t launch_cf_fast_t(const CFArgs &a, cudaStream_t s)
{
    cudaError_t e;
    if constexpr (W) if (!a.skip_full && !a.vbm3d) {
        // Final over all groups of BM3D frames: runs of consecutive groups, one per CTA
        const size_t smem = (size_t)kCfWarps * 2 * 32 * kTP * sizeof(float) + kCfCells * sizeof(unsigned long long) +
                            kCfWarps * 8 * sizeof(int);
        const long long runs = (a.ngroups + kCfRunGroups - 1) / kCfRunGroups;
        const int grid = (int)std::max<long long>(1, std::min<long long>(runs, 1LL << 20));
        if ((e = allow_smem(cf_run_kernel<G, W>, smem)) != cudaSuccess) return e;
        COUNT_LAUNCH();
        cf_run_kernel<G, W><<<grid, 32 * kCfWarps, smem, s>>>(a);
        return cudaGetLastError();
    }
    // per-lane kernel: 4 warps per CTA, grid-stride over the groups
    const int warps = 4;
    const long long warps_needed = (a.ngroups + (32 / G) - 1) / (32 / G);
    const int grid = (int)std::max<long long>(1, std::min<long long>((warps_needed + warps - 1) / warps, 148LL * 64));
    const size_t smem = (size_t)warps * (W ? 2 : 1) * 32 * kTP * sizeof(float);
    if ((e = allow_smem(cf_fast_kernel<G, W>, smem)) != cudaSuccess) return e;
    COUNT_LAUNCH();
    cf_fast_kernel<G, W><<<grid, 32 * warps, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_cf_partial_list(const int *count, long long ngroups, int G, long long *list, unsigned int *n, cudaStream_t s)
{
    const long long blocks = std::max<long long>(1, std::min<long long>((ngroups + 255) / 256, 148LL * 16));
    COUNT_LAUNCH();
    cf_partial_list_kernel<<<(unsigned)blocks, 256, 0, s>>>(count, ngroups, G, list, n);
    return cudaGetLastError();
}

cudaError_t launch_cf_fast(const CFArgs &a, cudaStream_t s)
{
    if (a.B != 8) return cudaErrorInvalidValue;
    const bool w = a.wiener != 0;
    switch (a.G) {
    case 8: return w ? launch_cf_fast_t<8, true>(a, s) : launch_cf_fast_t<8, false>(a, s);
    case 16: return w ? launch_cf_fast_t<16, true>(a, s) : launch_cf_fast_t<16, false>(a, s);
    case 32: return w ? launch_cf_fast_t<32, true>(a, s) : launch_cf_fast_t<32, false>(a, s);
    default: return cudaErrorInvalidValue;
    }
}

// ---- precision form: tensor-core collaborative filter ------------------------------------------

int cf_tc_supported(int B, int G) { return B == 8 && (G == 8 || G == 16 || G == 32); }

// tf32 value of x, rounded to nearest (ties away), as the tensor cores read it
static float round_tf32(float x)
{
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

template <int G>
static void tc_tables_t(std::vector<unsigned char> &img)
{
    using Lay = TcLayout<G>;
    img.assign(Lay::kTableBytes, 0);
    auto put = [&](uint32_t off, double v) {
        const float f = round_tf32((float)v);
        std::memcpy(img.data() + off, &f, 4);
    };
    // REDFT10 C[k][j] = 2 cos(pi (j + 1/2) k / N); REDFT01 Ci[j][k] = k == 0 ? 1 : 2 cos(pi k (j + 1/2) / N)
    auto fwd = [](int N, int k, int j) { return (double)cos2((long)(2 * j + 1) * k, 2L * N); };
    auto inv = [](int N, int j, int k) { return k == 0 ? 1.0 : (double)cos2((long)k * (2 * j + 1), 2L * N); };
    for (int w = 0; w < 128 / G; ++w)        // one copy of the matrices per group of a tile
        for (int kz = 0; kz < G; ++kz)
            for (int jz = 0; jz < G; ++jz) {
                put(Lay::kZf + tc_kmajor(G * w + kz, jz, G), fwd(G, kz, jz));
                put(Lay::kZi + tc_kmajor(G * w + jz, kz, G), inv(G, jz, kz));
            }
    for (int ky = 0; ky < 8; ++ky)
        for (int kx = 0; kx < 8; ++kx)
            for (int y = 0; y < 8; ++y)
                for (int x = 0; x < 8; ++x) {
                    const int c = ky * 8 + kx, px = y * 8 + x;
                    put(Lay::kKf + tc_kmajor(c, px, 64), fwd(8, ky, y) * fwd(8, kx, x));
                    put(Lay::kKi + tc_kmajor(px, c, 64), inv(8, y, ky) * inv(8, x, kx));
                }
}

// Rows of the n-point z-stage matrices, n = 1 .. G, as the Wiener kernels load them into tensor
// memory for tiles with a short group: [n - 1][forward, inverse][row j][G], forward row j = the
// REDFT10 coefficients of frequency j, inverse row j = the REDFT01 coefficients of block j, zero
// past n (rows and columns).
void cf_tc_partial_tables(int G, std::vector<float> &out)
{
    out.assign((size_t)G * 2 * G * G, 0.0f);
    for (int n = 1; n <= G; ++n)
        for (int r = 0; r < n; ++r)
            for (int k = 0; k < n; ++k) {
                float *f = out.data() + (size_t)(n - 1) * 2 * G * G;
                f[r * G + k] = round_tf32((float)cos2((long)(2 * k + 1) * r, 2L * n));
                f[G * G + r * G + k] = round_tf32(k == 0 ? 1.0f : (float)cos2((long)k * (2 * r + 1), 2L * n));
            }
}

int cf_tc_handles_partial(int B, int G, int wiener)
{
    if (!cf_tc_supported(B, G) || !wiener) return 0;
    return G == 16 ? TcShape<16, true>::kShort : G == 32 ? TcShape<32, true>::kShort : TcShape<8, true>::kShort;
}

void cf_tc_tables(int G, std::vector<unsigned char> &img)
{
    if (G == 8) tc_tables_t<8>(img);
    else if (G == 16) tc_tables_t<16>(img);
    else tc_tables_t<32>(img);
}

template <int G, bool W, bool ZT = false>
static cudaError_t launch_cf_tc_t(const CFArgs &a, const void *tables, int *status, cudaStream_t s)
{
    using Shp = TcShape<G, W, ZT>;
    // 227 KB per CTA, less the kernel's 1 KB of static shared memory (barriers, aligned)
    static_assert(Shp::kSmem <= 232448 - 1024, "tensor-core filter: shared memory over the per-CTA limit");
    const size_t smem = (size_t)Shp::kSmem;
    cudaError_t e;
    if ((e = allow_smem(cf_tc_kernel<G, W, ZT>, smem)) != cudaSuccess) return e;
    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    // one CTA per SM (shared memory and all 512 tensor-memory columns are taken)
    const long long ntiles = (a.ngroups + TcLayout<G>::kGroups - 1) / TcLayout<G>::kGroups;
    const long long grid = std::max<long long>(1, std::min<long long>((ntiles + Shp::kWG - 1) / Shp::kWG, sms));
    COUNT_LAUNCH();
    cf_tc_kernel<G, W, ZT><<<(unsigned)grid, Shp::kTeam * Shp::kWG, smem, s>>>(a, static_cast<const float4 *>(tables), ntiles, status);
    return cudaGetLastError();
}

int cf_tc_zt_supported(int B, int G, int wiener) { return B == 8 && G == 32 && wiener; }

cudaError_t launch_cf_tile_lists(const int *count, long long ngroups, int G, int *full, unsigned int *nfull,
                                 int *shrt, unsigned int *nshort, int *chunk_counts, cudaStream_t s)
{
    const long long ntiles = (ngroups + 128 / G - 1) / (128 / G);
    const long long chunks = std::max<long long>(1, (ntiles + kTileChunk - 1) / kTileChunk);
    COUNT_LAUNCH();
    cf_tile_count_kernel<<<(unsigned)chunks, 256, 0, s>>>(count, ngroups, G, ntiles, chunk_counts);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    COUNT_LAUNCH();
    cf_tile_lists_kernel<<<(unsigned)chunks, 256, 0, s>>>(count, ngroups, G, ntiles, chunk_counts, full, nfull, shrt, nshort);
    return cudaGetLastError();
}

long long cf_tile_chunks(long long ngroups, int G)
{
    const long long ntiles = (ngroups + 128 / G - 1) / (128 / G);
    return std::max<long long>(1, (ntiles + kTileChunk - 1) / kTileChunk);
}

cudaError_t launch_cf_tc_zt(const CFArgs &a, const void *tables, int *status, cudaStream_t s)
{
    if (!cf_tc_zt_supported(a.B, a.G, a.wiener)) return cudaErrorInvalidValue;
    return launch_cf_tc_t<32, true, true>(a, tables, status, s);
}

// Dz as [kz][b] and Ci as [b][kz], K-major without swizzle (the transposed z stage's B operands)
void cf_tc_zt_tables(int G, std::vector<float> &out)
{
    out.assign((size_t)2 * G * G, 0.0f);
    for (int r = 0; r < G; ++r)
        for (int k = 0; k < G; ++k) {
            out[tc_kmajor(r, k, G) / 4] = round_tf32((float)cos2((long)(2 * k + 1) * r, 2L * G));
            out[G * G + tc_kmajor(r, k, G) / 4] = round_tf32(k == 0 ? 1.0f : (float)cos2((long)k * (2 * r + 1), 2L * G));
        }
}

cudaError_t launch_cf_tc(const CFArgs &a, const void *tables, int *status, cudaStream_t s)
{
    if (!cf_tc_supported(a.B, a.G)) return cudaErrorInvalidValue;
    const bool w = a.wiener != 0;
    switch (a.G) {
    case 8: return w ? launch_cf_tc_t<8, true>(a, tables, status, s) : launch_cf_tc_t<8, false>(a, tables, status, s);
    case 16: return w ? launch_cf_tc_t<16, true>(a, tables, status, s) : launch_cf_tc_t<16, false>(a, tables, status, s);
    default: return w ? launch_cf_tc_t<32, true>(a, tables, status, s) : launch_cf_tc_t<32, false>(a, tables, status, s);
    }
}

// ---- FP64 oracle (inspection) --------------------------------------------------------------------

size_t cf_fp64_smem(int B, int G) { return sizeof(double) * ((size_t)2 * G * B * B + 64 * 64); }

cudaError_t launch_cf_fp64(const CFArgs &a, const F64Args &f, cudaStream_t s)
{
    const size_t smem = cf_fp64_smem(a.B, a.G);
    cudaError_t e;
    // always raised: the kernel's static shared memory comes on top of the dynamic part
    if ((e = cudaFuncSetAttribute(cf_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
        return e;
    COUNT_LAUNCH();
    cf_fp64_kernel<<<(unsigned)a.ngroups, 64, smem, s>>>(a, f);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    dim3 grid((a.W + 127) / 128, a.H, 3);
    COUNT_LAUNCH();
    finalize_fp64_kernel<<<grid, 128, 0, s>>>(f, a.W, a.H, 1, a.process[0], a.process[1], a.process[2]);
    return cudaGetLastError();
}

cudaError_t launch_cf_generic(const CFArgs &a, int warps, int grid, cudaStream_t s)
{
    COUNT_LAUNCH();
    cf_generic_kernel<<<grid, 32 * warps, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_convert(const ConvProgram &pr, const PlanePtr *in, const PlanePtr *out, int nframes,
                           cudaStream_t s)
{
    dim3 block(256);
    dim3 grid((pr.W + 255) / 256, pr.H, nframes);
    COUNT_LAUNCH();
    convert_kernel<<<grid, block, 0, s>>>(pr, in, out);
    return cudaGetLastError();
}

cudaError_t launch_finalize(const FinalizeArgs &a, int nframes, cudaStream_t s)
{
    const size_t smem = sizeof(float) * (size_t)finalize_smem_floats(a.B);
    cudaError_t e;
    if ((e = allow_smem(finalize_kernel, smem)) != cudaSuccess) return e;
    dim3 grid((a.W + kFinTW - 1) / kFinTW, (a.H + kFinTH - 1) / kFinTH, nframes * 3);
    COUNT_LAUNCH();
    finalize_kernel<<<grid, 256, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_vaggregate(const VAggArgs &a, int nframes, cudaStream_t s)
{
    dim3 block(256);
    dim3 grid((a.W + 255) / 256, a.H * 3, nframes);
    COUNT_LAUNCH();
    vaggregate_kernel<<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_vstack(const VStackArgs &a, int nframes, cudaStream_t s)
{
    const size_t smem = sizeof(float) * (size_t)finalize_smem_floats(a.B);
    cudaError_t e;
    if ((e = allow_smem(vstack_kernel, smem)) != cudaSuccess) return e;
    dim3 grid((a.W + kFinTW - 1) / kFinTW, a.slots * ((a.H + kFinTH - 1) / kFinTH), nframes * 3);
    COUNT_LAUNCH();
    vstack_kernel<<<grid, 256, smem, s>>>(a);
    return cudaGetLastError();
}

// ---- transform-only test kernels ------------------------------------------------------------

template <int G>
__global__ void dct_fast_test_kernel(float *data, int inverse)
{
    __shared__ float T[32 * 65];
    const int lane = threadIdx.x;
    float *g = data + (long long)blockIdx.x * G * 64;
    constexpr int C = 64 / G;
    if (!inverse) {
        if (lane < G) {
            float blk[64];
#pragma unroll
            for (int e = 0; e < 64; ++e) blk[e] = g[lane * 64 + e];
            fwd2d8(blk);
#pragma unroll
            for (int e = 0; e < 64; ++e) T[lane * 65 + e] = blk[e];
        }
        __syncwarp();
        if (lane < G) {
#pragma unroll
            for (int q = 0; q < C; ++q) {
                const int c = lane + q * G;
                float col[G], X[G];
#pragma unroll
                for (int zz = 0; zz < G; ++zz) col[zz] = T[zz * 65 + c];
                fdct_reg<G>(col, X);
#pragma unroll
                for (int zz = 0; zz < G; ++zz) g[zz * 64 + c] = X[zz];
            }
        }
    } else {
        if (lane < G) {
#pragma unroll
            for (int q = 0; q < C; ++q) {
                const int c = lane + q * G;
                float col[G], X[G];
#pragma unroll
                for (int zz = 0; zz < G; ++zz) X[zz] = g[zz * 64 + c];
                idct_reg<G>(X, col);
#pragma unroll
                for (int zz = 0; zz < G; ++zz) T[zz * 65 + c] = col[zz];
            }
        }
        __syncwarp();
        if (lane < G) {
            float blk[64];
#pragma unroll
            for (int e = 0; e < 64; ++e) blk[e] = T[lane * 65 + e];
            inv2d8(blk);
#pragma unroll
            for (int e = 0; e < 64; ++e) g[lane * 64 + e] = blk[e];
        }
    }
}

__global__ void dct_generic_test_kernel(float *data, int n, int B, int inverse, CFArgs a)
{
    float tmp[512];
    float *g = data + (long long)blockIdx.x * n * B * B;
    dct3d_warp(g, n, B, inverse != 0, a, tmp);
}

cudaError_t launch_dct3d_test(float *data, int ngroups, int n, int B, int inverse, int fast,
                              const float *odd_all, const float *dtab, const int *dtab_off,
                              cudaStream_t s)
{
    if (fast) {
        if (B != 8) return cudaErrorInvalidValue;
        switch (n) {
        case 8: dct_fast_test_kernel<8><<<ngroups, 32, 0, s>>>(data, inverse); break;
        case 16: dct_fast_test_kernel<16><<<ngroups, 32, 0, s>>>(data, inverse); break;
        case 32: dct_fast_test_kernel<32><<<ngroups, 32, 0, s>>>(data, inverse); break;
        default: return cudaErrorInvalidValue;
        }
    } else {
        CFArgs a{};
        a.odd_all = odd_all;
        a.dtab = dtab;
        a.dtab_off = dtab_off;
        dct_generic_test_kernel<<<ngroups, 32, 0, s>>>(data, n, B, inverse, a);
    }
    return cudaGetLastError();
}

}  // namespace bm3d
