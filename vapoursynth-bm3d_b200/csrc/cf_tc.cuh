// cf_tc.cuh -- precision form of the collaborative filter: the 3-D DCTs of full groups as tf32
// matrix products on the sm_100a tensor cores (tcgen05, fp32 accumulation in tensor memory).
//
// Same arithmetic contract as cf_fast_kernel (source/BM3D_Basic.cpp:72-148,
// source/BM3D_Final.cpp:50-127, aggregation include/Block.h:1239-1387) except that the transforms
// are dense matrix products with tf32 operands, so coefficients carry ~2^-11 relative error: the
// output is close to, not bit-identical with, the plain FP32 path.  The hard-threshold kernels
// handle full groups (n == G) only, and the plain kernel filters the partial ones afterwards; the
// Wiener kernels with G = 16 / 32 filter every group, a short one (n < G) with the n-point
// transforms in its rows of the z-stage matrices.
//
// A tile is 128 blocks = 128 / G groups of one plane, handled by one warpgroup (128 threads);
// thread r owns row r = block (r % G) of group r / G.  A CTA runs several warpgroups, each on its
// own stream of tiles with its own shared-memory operands, mbarrier and 128 tensor-memory columns,
// so that one warpgroup's gathers and atomics overlap another's tensor-core work; the DCT tables
// are shared.  Every shared-memory operand is K-major (the tf32 kind takes no MN-major operands):
//   1. gather  X[b][pixel] (A operand, 128-byte swizzle); Final also gathers the reference group
//      R.  A warp copies one block per step (lane = pixel row / column) with asynchronous
//      global -> shared copies, so each instruction touches the block's own 4 rows instead of 32
//      blocks and no register waits for the data; the block origins come from the owning lanes
//      by shuffles
//   2. 2-D DCT Y = X . K2 into tensor memory cols [0, 64) (ref [64, 128))
//   3. transpose: each thread reads its row of Y and writes it as column b of Yt[coef][b], a B
//      operand with 128-byte swizzle (conflict-free column writes); Final stacks the reference
//      coefficients below (rows 64..127), so one N = 128 product transforms both
//   4. z-DCT   Z = Zf . Yt_w per group w into cols [0, 64) (ref [64, 128)); the A operand Zf
//      stacks 128 / G copies of the G x G DCT matrix and every output lane outside group w's rows
//      [G w, G w + G) is disabled in that product
//   5. shrink  thread r owns row (group, z-frequency) of 64 coefficients: hard threshold (Basic)
//      or Wiener weights from the reference spectrum (Final); the group's count / L2 is a
//      reduction over its G lanes; S goes back to shared memory as St[coef][kz] (swizzled B)
//   6. inverse z into cols [0, 64), then inverse 2-D with A read from tensor memory into
//      cols [64, 128)
//   7. aggregate: the inverse rows go through shared memory so that a warp adds one block per
//      step with lane = pixel; in region mode into the staged region (fixed-point integer
//      atomics, then one pass of vector atomics to the numerator plane), otherwise straight to the
//      numerator plane (one 32-byte sector per block row and atomic instruction instead of 32
//      scattered sectors); the block weight goes to the weight map as in the plain kernel.
// The transposed form (ZT, Wiener filter with G = 32, tiles of full groups) replaces steps 3-6:
//   3'. each thread writes its block row's coefficients as column b % 64 of row (b / 64, c) of a
//      source and a reference A operand (K = the 64 blocks of half tile b / 64)
//   4'. z-DCT with the coefficients on the lanes: per half tile and group, D[(h, c)][32 g' + kz] =
//      sum_b Ys[(h, c)][32 g' + b] Dz[kz][b], an M = 128, N = 32 product per K step (B = Dz in
//      shared memory): each product is the group's own transform, nothing is masked
//   5'. Wiener shrinkage per thread on its coefficient's 32 z frequencies of source and reference;
//      the shrunk values go back to tensor memory and the group sums of the squared weights are
//      combined over the two warps of the half tile's coefficients
//   6'. inverse z with A = S from tensor memory and B = Ci, then a transpose back to block rows
//      (an A operand in shared memory) for the inverse 2-D product
// The tiles are taken from a list (a.tlist) when one is given: the transposed form walks the
// tiles of full groups and the masked form the tiles with a short group.
// Every wait on the tensor cores is bounded; on time-out the warpgroup records the failure in
// *status and stops; the CTA releases its tensor memory and returns.
#pragma once

#include "args.h"
#include "cf.cuh"
#include "tc.cuh"

namespace bm3d {

// Byte layout of the constant tables in shared memory (host builds the same image).
template <int G>
struct TcLayout {
    static constexpr int kGroups = 128 / G;            // groups per tile
    static constexpr int kZRows = 128;                 // 128 / G stacked copies of the G x G DCT matrix
    static constexpr int kZBytes = kZRows * G * 4;
    static constexpr int kKBytes = 64 * 64 * 4;
    static constexpr int kZf = 0;                       // forward z matrix stack (K-major)
    static constexpr int kZi = kZf + kZBytes;           // inverse z matrix stack (K-major)
    static constexpr int kKf = kZi + kZBytes;           // forward 2-D matrix, [coef][pixel] (K-major)
    static constexpr int kKi = kKf + kKBytes;           // inverse 2-D matrix, [pixel][coef] (K-major)
    static constexpr int kTableBytes = kKi + kKBytes;
    static constexpr int kXBytes = 128 * 64 * 4;        // one 128 x 64 data operand
    // image offset of the transposed form's z-stage matrices (after the fp64 tables, the fp32 DC
    // tables and the n-point rows): Dz as [kz][b] and Ci as [b][kz], K-major, no swizzle
    static constexpr int kZtOff = kTableBytes + (64 + G * G) * 8 + (2 * G * G + 2 * G * G * G) * 4;
    static constexpr int kZtBytes = 2 * G * G * 4;
};

// Tile teams per CTA: shared memory holds the tables and, per team, one (Basic) or two (Final)
// 32 KB operands; tensor memory gives 128 columns to each of at most 4.  A team is one warp per
// 32-row quarter of the tile (kSplit = 1) or two (kSplit = 2: the two warps of a quarter share its
// columns and gather / aggregation steps), so that the kernels limited to two teams by shared
// memory (Final, and Basic with G = 32) still run 16 warps per SM.
// ZT (Wiener filter, G = 32): the transposed z stage.  The z products put the coefficients of a
// half tile on the tensor-memory lanes and the half's two groups on the columns, so each product
// is the group's own 32-point transform (N = 32) instead of a 128-lane product with three
// quarters of its lanes disabled: a quarter of the tensor work of the z stages.
template <int G, bool WIENER, bool ZT = false>
struct TcShape {
    static_assert(!ZT || (WIENER && G == 32), "transposed z stage: Wiener filter with G = 32 only");
    static constexpr bool kTwo = WIENER || G == 32;     // two teams (shared memory), split quarters
    static constexpr int kWG = kTwo ? 2 : 4;
    static constexpr int kSplit = kTwo ? 2 : 1;
    static constexpr int kTeam = 128 * kSplit;          // threads per team
    static constexpr int kData = TcLayout<G>::kXBytes * (WIENER ? 2 : 1);
    static constexpr int kPart = kSplit == 2 ? kTeam * 4 : 0; // per-row partial sums of the two halves
    // With two teams, tensor memory has room for the z-stage matrix stacks (G columns each): the
    // z products then read A from tensor memory and only B from shared memory, and the stacks
    // need no shared-memory copy.
    static constexpr bool kZInTmem = !ZT && kWG == 2 && G >= 16;
    static constexpr int kTmemCols = kWG == 4 ? 512 : (kZInTmem ? 512 : 256);
    static constexpr int kZCol = 128 * kWG;              // first column of the stacks
    // Wiener filter with the stacks in tensor memory: groups of fewer than G blocks are filtered
    // here too.  A tile holding one gets its own stacks (per team, after the shared ones) whose
    // rows of group w are the n_w-point matrices (zero past n_w), so each group's z products are
    // its own length's transforms.
    static constexpr bool kShort = WIENER && kZInTmem;
    static constexpr int kPCol = kZCol + 2 * G;
    static_assert(!kShort || kPCol + kWG * 2 * G <= kTmemCols, "tensor memory: per-team stacks do not fit");
    static constexpr int kTabOff = kZInTmem || ZT ? TcLayout<G>::kKf : 0;   // first table byte kept in shared memory
    static constexpr int kZtBytes = ZT ? TcLayout<G>::kZtBytes : 0;   // (ZT) z-stage B operands after the tables
    // Image boxes of the region mode: Final with the stacks in tensor memory keeps a source box,
    // a reference box and the aggregation box, so that the next plane's boxes load while this
    // plane is filtered; otherwise one box serves the gathers and the aggregation in turn.
    static constexpr int kBoxes = WIENER && (kZInTmem || ZT) ? 3 : 1;
    // (ZT) the aggregation box lives in the data region (its second half is free by then)
    static constexpr int kBoxesExtra = ZT ? 2 : kBoxes;
    static constexpr int kRegion = kBoxes == 3 ? 2560 : 3072;   // floats per box
    // three-box form: a table of the tile's rows (block position in the box, weight) that the
    // block-step loops read with one broadcast load instead of three or four shuffles
    static constexpr int kRowTab = kBoxes == 3 ? 128 * 8 : 0;
    static constexpr int kExtra = kPart + kRegion * 4 * kBoxesExtra + 256 + kRowTab;   // + 2 x [4 quarters][8] ints of scratch
    static constexpr int kSmem = (kData + kExtra) * kWG + TcLayout<G>::kTableBytes - kTabOff + kZtBytes;
};

// byte offset of element (row, k) of a K-major operand with `kdim` columns
__host__ __device__ constexpr uint32_t tc_kmajor(int row, int k, int kdim)
{
    return (uint32_t)((row / 8) * (kdim / 4) * 128 + (k / 4) * 128 + (row % 8) * 16 + (k % 4) * 4);
}

constexpr uint32_t kTcWaitLimit = 1u << 24;

// floor(v / d) = umulhi(v, div_magic(d)) for 0 <= v < 2^16 and 1 <= d < 2^8: the magic number
// exceeds 2^32 / d by less than 1, which moves v / d by less than 2^-16 < 1 / d
__device__ __forceinline__ uint32_t div_magic(uint32_t d) { return 0xffffffffu / d + 1u; }

// mean of the 64 pixels of a block held two per lane by a warp
__device__ __forceinline__ float block_mean(float v0, float v1)
{
    float s = v0 + v1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s * (1.0f / 64.0f);
}

// means of N blocks (N = 4 or 8) whose pixels a warp holds two per lane, s[k] = the lane's sum for
// block k: log2(N) halving steps (each lane keeps half of its values and receives the other half
// of its partner's) leave one block's partial sum per lane, the remaining steps finish it, and
// one shuffle per block brings every mean to every lane (9 + 8 shuffles for 8 blocks instead of 40)
template <int N>
__device__ __forceinline__ void block_means(float (&s)[N], int lane)
{
    constexpr int L = N == 8 ? 3 : 2;
#pragma unroll
    for (int st = 0; st < L; ++st) {
        const int off = 16 >> st, h = N >> (st + 1);
        const bool up = (lane & off) != 0;
#pragma unroll
        for (int k = 0; k < h; ++k) {
            const float keep = up ? s[k + h] : s[k];
            const float send = up ? s[k] : s[k + h];
            s[k] = keep + __shfl_xor_sync(0xffffffffu, send, off);
        }
    }
    float w = s[0];
#pragma unroll
    for (int off = 16 >> L; off > 0; off >>= 1) w += __shfl_xor_sync(0xffffffffu, w, off);
    // block v's sum is held by the lanes whose bits (4, 3[, 2]) spell v's bits from the top
#pragma unroll
    for (int v = 0; v < N; ++v) {
        int src = 0;
#pragma unroll
        for (int st = 0; st < L; ++st) src |= ((v >> (L - 1 - st)) & 1) << (4 - st);
        s[v] = __shfl_sync(0xffffffffu, w, src) * (1.0f / 64.0f);
    }
}

// Tiles (128 / G consecutive groups) split into those whose groups are all full and those with a
// short group, both lists in ascending tile order (the persistent filter kernels walk them, and
// neighbouring teams on neighbouring tiles keep the image rows and accumulators in L2).  Chunks of
// kTileChunk tiles, one CTA each: the first kernel counts each chunk's full and short tiles, the
// second adds the counts of the chunks before its own and writes its tiles at their ranks.
constexpr int kTileChunk = 2048;             // 256 threads x 8 consecutive tiles

__device__ __forceinline__ bool tile_full(const int *__restrict__ count, long long ngroups, int G, long long tl)
{
    const int gpt = 128 / G;
    bool all = true;
    for (int k = 0; k < gpt; ++k) {
        const long long g = tl * gpt + k;
        if (g < ngroups && count[g] < G) all = false;
    }
    return all;
}

__global__ void __launch_bounds__(256) cf_tile_count_kernel(const int *__restrict__ count, long long ngroups, int G,
                                                            long long ntiles, int *__restrict__ chunk_counts)
{
    __shared__ int sf[8], ss[8];
    const long long base = (long long)blockIdx.x * kTileChunk + threadIdx.x * 8;
    int nf = 0, ns = 0;
    for (int k = 0; k < 8; ++k) {
        const long long tl = base + k;
        if (tl >= ntiles) break;
        if (tile_full(count, ngroups, G, tl)) ++nf; else ++ns;
    }
    for (int o = 16; o > 0; o >>= 1) {
        nf += __shfl_xor_sync(0xffffffffu, nf, o);
        ns += __shfl_xor_sync(0xffffffffu, ns, o);
    }
    if ((threadIdx.x & 31) == 0) { sf[threadIdx.x >> 5] = nf; ss[threadIdx.x >> 5] = ns; }
    __syncthreads();
    if (threadIdx.x == 0) {
        int tf = 0, ts = 0;
        for (int w = 0; w < 8; ++w) { tf += sf[w]; ts += ss[w]; }
        chunk_counts[2 * blockIdx.x] = tf;
        chunk_counts[2 * blockIdx.x + 1] = ts;
    }
}

__global__ void __launch_bounds__(256) cf_tile_lists_kernel(const int *__restrict__ count, long long ngroups, int G,
                                                            long long ntiles, const int *__restrict__ chunk_counts,
                                                            int *__restrict__ full, unsigned int *__restrict__ nfull,
                                                            int *__restrict__ shrt, unsigned int *__restrict__ nshort)
{
    __shared__ int sf[8], ss[8], bf, bs;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    // the chunk's first ranks: the counts of the chunks before it
    int pf = 0, ps = 0;
    for (int c = t; c < (int)blockIdx.x; c += 256) { pf += chunk_counts[2 * c]; ps += chunk_counts[2 * c + 1]; }
    const long long base = (long long)blockIdx.x * kTileChunk + t * 8;
    unsigned fm = 0;                         // bit k: tile base + k is full
    int nf = 0, ns = 0;
    for (int k = 0; k < 8; ++k) {
        const long long tl = base + k;
        if (tl >= ntiles) break;
        if (tile_full(count, ngroups, G, tl)) { fm |= 1u << k; ++nf; } else { ++ns; }
    }
    // exclusive prefix of (nf, ns) over the CTA's threads, in thread order
    int xf = nf, xs = ns;
    for (int o = 1; o < 32; o <<= 1) {
        const int yf = __shfl_up_sync(0xffffffffu, xf, o), ys = __shfl_up_sync(0xffffffffu, xs, o);
        if (lane >= o) { xf += yf; xs += ys; }
    }
    for (int o = 16; o > 0; o >>= 1) { pf += __shfl_xor_sync(0xffffffffu, pf, o); ps += __shfl_xor_sync(0xffffffffu, ps, o); }
    if (lane == 31) { sf[w] = xf; ss[w] = xs; }
    if (t == 0) { bf = 0; bs = 0; }
    __syncthreads();
    if (lane == 0) { atomicAdd(&bf, pf); atomicAdd(&bs, ps); }
    int wf = 0, ws = 0;
    for (int k = 0; k < w; ++k) { wf += sf[k]; ws += ss[k]; }
    __syncthreads();
    int of = bf + wf + xf - nf, os = bs + ws + xs - ns;
    for (int k = 0; k < 8; ++k) {
        const long long tl = base + k;
        if (tl >= ntiles) break;
        if (fm >> k & 1u) full[of++] = (int)tl; else shrt[os++] = (int)tl;
    }
    if (blockIdx.x == gridDim.x - 1 && t == 255) {
        int tf = 0, ts = 0;
        for (int k = 0; k < 8; ++k) { tf += sf[k]; ts += ss[k]; }
        *nfull = (unsigned)(bf + tf);
        *nshort = (unsigned)(bs + ts);
    }
}

template <int G, bool WIENER, bool ZT = false>
__global__ void __launch_bounds__(TcShape<G, WIENER, ZT>::kTeam * TcShape<G, WIENER, ZT>::kWG, 1)
cf_tc_kernel(CFArgs a, const float4 *tables, long long ntiles, int *status)
{
    using Lay = TcLayout<G>;
    using Shp = TcShape<G, WIENER, ZT>;
    constexpr int GPT = Lay::kGroups;
    constexpr int NWG = Shp::kWG;
    constexpr int SPLIT = Shp::kSplit;
    constexpr int TEAM = Shp::kTeam;
    constexpr int NC = 64 / SPLIT;                   // columns per thread in the row phases
    constexpr int NI = 32 / SPLIT;                   // blocks per warp in the block-step phases
    constexpr int NT = WIENER ? 128 : 64;            // rows of the z-stage B operand
    extern __shared__ __align__(1024) unsigned char tsm[];
    __shared__ __align__(8) uint64_t mbar[NWG];
    __shared__ __align__(8) uint64_t mdrain[NWG];   // drains a team's products on the time-out path
    __shared__ uint32_t tslot;

    const int wg = threadIdx.x / TEAM;
    const int t = threadIdx.x % TEAM;
    const int r = t & 127;                           // row of the tile (tensor-memory lane)
    const int half = t >> 7;                         // column half (SPLIT = 2)
    const int cb = half * NC;                        // first column of this thread
    const int warp = threadIdx.x >> 5;
    const uint32_t bar_id = 1 + wg;
    const int wsub = r / G;                          // group within the tile
    const int j = r % G;                             // block index in the group / z-frequency
    unsigned char *D = tsm + Shp::kData * wg;        // X | R, then Yt, then St
    unsigned char *extra = tsm + Shp::kData * NWG + Shp::kExtra * wg;
    float *part = reinterpret_cast<float *>(extra);
    float *boxes = reinterpret_cast<float *>(extra + Shp::kPart);
    // aggregation box (ZT: in the second half of the data region, zeroed before each use)
    float *Rg = ZT ? reinterpret_cast<float *>(D + Lay::kXBytes) : boxes;
    float *Bs = Shp::kBoxes == 3 ? (ZT ? boxes : boxes + Shp::kRegion) : Rg;              // source box
    float *Br = Shp::kBoxes == 3 ? (ZT ? boxes + Shp::kRegion : boxes + 2 * Shp::kRegion) : Rg;   // reference box
    int *bbx = reinterpret_cast<int *>(extra + Shp::kPart + Shp::kRegion * 4 * Shp::kBoxesExtra);   // [4 quarters][8]: maxima
    int *bnd = bbx + 32;                                                  // [4 quarters][8]: tile bounds
    // [128]: (y - y0) << 16 | (x - x0) of the row's block in the box (-1: not this kernel's), numW bits
    int2 *rowtab = reinterpret_cast<int2 *>(extra + Shp::kPart + Shp::kRegion * 4 * Shp::kBoxesExtra + 256);
    // table byte b lives at tab + b (b >= kTabOff)
    unsigned char *tab = tsm + (Shp::kData + Shp::kExtra) * NWG - Shp::kTabOff;

    for (int i = threadIdx.x; i < (Lay::kTableBytes - Shp::kTabOff) / 16; i += blockDim.x)
        reinterpret_cast<float4 *>(tab + Shp::kTabOff)[i] = tables[Shp::kTabOff / 16 + i];
    for (int i = threadIdx.x; i < Shp::kZtBytes / 16; i += blockDim.x)
        reinterpret_cast<float4 *>(tab + Lay::kTableBytes)[i] = tables[Lay::kZtOff / 16 + i];
    if constexpr (Shp::kBoxes == 3 && !ZT)
        for (int i = t; i < Shp::kRegion; i += TEAM) Rg[i] = 0.0f;   // the aggregation box starts (and stays) zero
    if (warp == 0) tc::tmem_alloc(&tslot, Shp::kTmemCols);
    if (t == 0) {
        tc::mbar_init(&mbar[wg], 1);
        tc::mbar_init(&mdrain[wg], 1);
    }
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = tslot;
    if constexpr (Shp::kZInTmem) {
        // row threadIdx.x of both stacks -> tensor-memory lane threadIdx.x (warps 0..3)
        if (threadIdx.x < 128) {
            const uint32_t lr = (uint32_t)(32 * (threadIdx.x >> 5)) << 16;
#pragma unroll
            for (int m = 0; m < 2; ++m)
#pragma unroll
                for (int k0 = 0; k0 < G; k0 += 16) {
                    float v[16];
#pragma unroll
                    for (int e = 0; e < 16; ++e)
                        v[e] = __ldg(reinterpret_cast<const float *>(tables) + ((m ? Lay::kZi : Lay::kZf) + tc_kmajor(threadIdx.x, k0 + e, G)) / 4);
                    tc::tmem_st16(tm + lr + Shp::kZCol + m * G + k0, v);
                }
            tc::tmem_wait_st();
        }
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
    }
    const uint32_t tb = tm + 128 * wg;               // this warpgroup's columns
    const uint32_t lrow = (uint32_t)(32 * (warp & 3)) << 16;
    // (with the stacks in tensor memory, sZf / sZi only tell the two z products apart)
    const uint32_t sZf = Shp::kZInTmem ? 0u : tc::smem_u32(tab + Lay::kZf);
    const uint32_t sZi = Shp::kZInTmem ? 1u : tc::smem_u32(tab + Lay::kZi);
    const uint32_t sKf = tc::smem_u32(tab + Lay::kKf), sKi = tc::smem_u32(tab + Lay::kKi);
    const uint32_t sD = tc::smem_u32(D);
    constexpr uint32_t ID64 = tc::idesc_tf32(128, 64, 0, 0);
    constexpr uint32_t IDZT = tc::idesc_tf32(128, 32, 0, 0);
    // (ZT) Dz as [kz][b] and Ci as [b][kz] after the 2-D tables
    const uint32_t sZt = tc::smem_u32(tab + Lay::kTableBytes), sCi = sZt + (uint32_t)(G * G * 4);
    constexpr uint32_t IDZ = tc::idesc_tf32(128, NT, 0, 0);
    uint64_t *mb = &mbar[wg];
    uint32_t phase = 0;

    // Only the issuing warp polls the mbarrier; the team's other warps sleep in the barrier that
    // passes its result on, instead of taking issue slots from the other team with their polls.
    auto wait_mma = [&]() -> bool {
        bool ok = true;
        if (t < 32) ok = tc::mbar_wait_bounded(mb, phase, kTcWaitLimit);
        phase ^= 1u;
        const bool all = tc::wg_and(bar_id, TEAM, ok);
        tc::fence_after_sync();
        return all;
    };
    auto publish = [&]() {
        tc::fence_proxy_async_smem();
        tc::fence_before_sync();
        tc::wg_sync(bar_id, TEAM);
        tc::fence_after_sync();
    };
    // Descriptor arithmetic: a descriptor's start address is in 16-byte units in its low bits, so
    // the K steps of an operand are its first descriptor plus constants (the issue loops below are
    // unrolled, so each product is one add and the instruction).
    // 2-D stage, A in shared memory: D[d0, +64) = X . K (X swizzled [128][64], K [64 n][64 k])
    auto xy_ss = [&](uint32_t d0, uint32_t sx, uint32_t sk) {
        const uint64_t ad = tc::make_desc_sw128(sx, 1024), bd = tc::make_desc(sk, 128, 2048);
#pragma unroll
        for (int s = 0; s < 8; ++s)
            tc::mma_tf32_ss(tb + d0, ad + (uint64_t)(((s / 4) * 16 * 1024 + (s % 4) * 32) >> 4), bd + (uint64_t)(s * 16), ID64, s > 0);
    };
    // two independent 2-D products (source and reference) issued alternately
    auto xy_ss2 = [&](uint32_t d0, uint32_t sx, uint32_t d1, uint32_t sy, uint32_t sk) {
        const uint64_t ax = tc::make_desc_sw128(sx, 1024), ay = tc::make_desc_sw128(sy, 1024), bd = tc::make_desc(sk, 128, 2048);
#pragma unroll
        for (int s = 0; s < 8; ++s) {
            const uint64_t ao = (uint64_t)(((s / 4) * 16 * 1024 + (s % 4) * 32) >> 4);
            tc::mma_tf32_ss(tb + d0, ax + ao, bd + (uint64_t)(s * 16), ID64, s > 0);
            tc::mma_tf32_ss(tb + d1, ay + ao, bd + (uint64_t)(s * 16), ID64, s > 0);
        }
    };
    // 2-D stage, A in tensor memory: D[d0, +64) = T[a0, +64) . K
    auto xy_ts = [&](uint32_t d0, uint32_t a0, uint32_t sk) {
        const uint64_t bd = tc::make_desc(sk, 128, 2048);
#pragma unroll
        for (int s = 0; s < 8; ++s)
            tc::mma_tf32_ts(tb + d0, tb + a0 + 8 * s, bd + (uint64_t)(s * 16), ID64, s > 0);
    };
    // z stage: rows of group w of D[d0, +nt) = Zstack . Bt_w (K range of group w), every other
    // output lane disabled; Bt swizzled [nt rows][128 k]
    // The per-group chains are independent (disjoint output lanes), so consecutive products go
    // to different groups: K step outer, group inner.
    uint32_t zcol = Shp::kZCol;                      // first column of the stacks the z products read
    auto z_stage = [&](uint32_t d0, uint32_t sz, int nt, uint32_t idesc) {
#pragma unroll 1
        for (int s = 0; s < G / 8; ++s) {
            const uint64_t ad = tc::make_desc(sz + s * 256, 128, (G / 4) * 128);
#pragma unroll 1
            for (int w = 0; w < GPT; ++w) {
                uint32_t m[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int lo = G * w - 32 * q, hi = lo + G;      // enabled lanes of word q: [lo, hi)
                    const uint32_t en = (hi <= 0 || lo >= 32) ? 0u
                                      : (G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (lo < 0 ? 0 : lo)));
                    m[q] = ~en;
                }
                const uint32_t k0 = (uint32_t)(G * w + 8 * s);
                const uint64_t bd = tc::make_desc_sw128(sD + (k0 / 32) * (nt / 8) * 1024 + ((k0 % 32) / 8) * 32, 1024);
                if constexpr (Shp::kZInTmem)
                    tc::mma_ts_tf32_masked(tb + d0, tm + zcol + (sz == sZi ? G : 0) + 8 * s, bd, idesc, s > 0,
                                           m[0], m[1], m[2], m[3]);
                else
                    tc::mma_ss_tf32_masked(tb + d0, ad, bd, idesc, s > 0, m[0], m[1], m[2], m[3]);
            }
        }
    };
    // this thread's columns of its tensor-memory row (c0 + cb ..) -> column r, rows row0 + cb .., of Bt
    auto row_to_column = [&](uint32_t c0, int row0, int nt) {
        float v[NC];
#pragma unroll
        for (int q = 0; q < NC; q += 16) tc::tmem_ld16(tb + lrow + c0 + cb + q, *reinterpret_cast<float (*)[16]>(v + q));
        tc::tmem_wait_ld();
#pragma unroll
        for (int e = 0; e < NC; ++e) *reinterpret_cast<float *>(D + tc::sw128_offset(row0 + cb + e, r, nt)) = v[e];
    };

    // A tile as this thread sees it: its row's group and block, and the team's image box.
    struct Tile {
        long long g0;
        uint32_t pk;
        int cnt;                         // the row's group count (used a tile after its load)
        bool inr;                        // the row's group exists
        bool region;
        int y0, x0, rh, rw, rp, frame;   // box origin, rows, width and shared-memory row pitch
    };
    const int lane = r & 31, ry = lane >> 3, cx = lane & 7;
    const int b0 = r & ~31;
    // Region mode (BM3D): every full group of the tile lies in one frame and the bounding box of
    // its blocks (the same for the three planes) fits a box buffer; the box is then staged with
    // aligned 16-byte copies and the blocks are cut out of shared memory, and the aggregation adds
    // into a box before one pass of vector atomics.  Otherwise blocks are copied and added one by
    // one.  Every thread of the team calls bound_tile at the same point (it holds a team barrier).
    // tiles: all of them, or those of a list (a.tlist, *a.tlist_n entries)
    const long long nlist = a.tlist ? (long long)*a.tlist_n : ntiles;
    // the tile id of list entry i, loaded a tile before the tile's own loads need it
    auto tile_id = [&](long long i) -> long long { return a.tlist ? (i < nlist ? (long long)a.tlist[i] : ntiles) : i; };
    auto fetch_tile = [&](long long tid) {
        Tile T;
        const long long grp = tid * GPT + wsub;
        T.inr = tid < ntiles && grp < a.ngroups;
        T.g0 = T.inr ? grp : 0;
        T.cnt = a.count[T.g0];
        T.pk = a.pos[T.g0 * G + j];
        T.region = false;
        T.y0 = T.x0 = T.rh = T.rw = T.rp = T.frame = 0;
        return T;
    };
    // full groups are filtered here; with kShort every group, block j if j < its count
    auto tile_mine = [&](const Tile &T) { return T.inr && (Shp::kShort ? j < T.cnt : T.cnt >= G); };
    auto bound_tile = [&](Tile &T) {
        if (!a.vbm3d) {
            const bool tmine = tile_mine(T);
            const long long f = T.g0 / a.blocks_per_frame;
            const int py = unpack_y(T.pk), px = unpack_x(T.pk);
            int ymin = tmine ? py : 1 << 30, xmin = tmine ? px : 1 << 30;
            int ymax = tmine ? py : -1, xmax = tmine ? px : -1;
            int fmin = tmine ? (int)f : 1 << 30, fmax = tmine ? (int)f : -1;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                ymin = min(ymin, __shfl_xor_sync(0xffffffffu, ymin, o));
                xmin = min(xmin, __shfl_xor_sync(0xffffffffu, xmin, o));
                ymax = max(ymax, __shfl_xor_sync(0xffffffffu, ymax, o));
                xmax = max(xmax, __shfl_xor_sync(0xffffffffu, xmax, o));
                fmin = min(fmin, __shfl_xor_sync(0xffffffffu, fmin, o));
                fmax = max(fmax, __shfl_xor_sync(0xffffffffu, fmax, o));
            }
            if (half == 0 && lane == 0) {
                int *q = bnd + 8 * (r >> 5);
                q[0] = ymin; q[1] = xmin; q[2] = ymax; q[3] = xmax; q[4] = fmin; q[5] = fmax;
            }
            tc::wg_sync(bar_id, TEAM);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                ymin = min(ymin, bnd[8 * q]); xmin = min(xmin, bnd[8 * q + 1]);
                ymax = max(ymax, bnd[8 * q + 2]); xmax = max(xmax, bnd[8 * q + 3]);
                fmin = min(fmin, bnd[8 * q + 4]); fmax = max(fmax, bnd[8 * q + 5]);
            }
            if (ymax >= 0 && fmin == fmax) {
                T.y0 = ymin;
                T.x0 = xmin & ~3;
                T.rh = ymax + 8 - ymin;
                // whole 16-byte chunks, never past the padded row (ld is a multiple of 32)
                T.rw = min((xmax + 8 - T.x0 + 3) & ~3, a.ld - T.x0);
                // pitch = 8 mod 16 words: the 4 rows x 8 columns a warp touches in a block step
                // fall in 32 distinct banks
                T.rp = T.rw + ((24 - (T.rw & 15)) & 15);
                T.region = T.rh * T.rp <= Shp::kRegion;
                T.frame = fmin;
            }
        }
    };
    // source and reference boxes of plane pp of tile T (three-box form), as asynchronous copies
    auto load_boxes = [&](const Tile &T, int pp) {
        const long long fo = (long long)T.frame * a.frame_stride + (long long)T.y0 * a.ld + T.x0;
        const int w4 = T.rw >> 2, nv = T.rh * w4;
        const uint32_t md = div_magic((uint32_t)w4);
        for (int v = t; v < nv; v += TEAM) {
            const int yy = (int)__umulhi((uint32_t)v, md), c4 = v - yy * w4;
            const long long go = fo + (long long)yy * a.ld + 4 * c4;
            tc::cp_async16(Bs + yy * T.rp + 4 * c4, a.src[pp] + go);
            tc::cp_async16(Br + yy * T.rp + 4 * c4, a.ref[pp] + go);
        }
    };
    auto next_plane = [&](int pp) {
        while (pp < 3 && !a.process[pp]) ++pp;
        return pp;
    };
    const int pfirst = next_plane(0);
    const long long tstride = (long long)gridDim.x * NWG;
    // fp64 tables after the tensor-core image: C8[u][y] = 2 cos(pi (2y + 1) u / 16), then the
    // z matrix Dz[kz][b] = 2 cos(pi (2b + 1) kz / 2G) (hard-threshold recheck and block means)
    const double *xtab = reinterpret_cast<const double *>(reinterpret_cast<const unsigned char *>(tables) + Lay::kTableBytes);
    // then, in fp32, Dz as [b][kz] (dzt) and the inverse z matrix Ci[b][kz] as [kz][b] (dzi;
    // Ci[b][0] = 1, Ci[b][kz] = Dz[kz][b]): a warp's lanes read consecutive words
    const float *dzt = reinterpret_cast<const float *>(xtab + 64 + G * G);
    const float *dzi = dzt + G * G;
    // then (kShort) the rows of the n-point stacks, n = 1 .. G: [n - 1][forward, inverse][row][G]
    const float *ztn = dzi + G * G;
    unsigned long long n_recheck = 0, n_changed = 0;

    bool failed = false;
    Tile cur = fetch_tile(tile_id((long long)blockIdx.x * NWG + wg));
    bound_tile(cur);
    long long nid = tile_id((long long)blockIdx.x * NWG + wg + tstride);
    if constexpr (Shp::kBoxes == 3)
        if (cur.region && pfirst < 3) load_boxes(cur, pfirst);
    for (long long tile = (long long)blockIdx.x * NWG + wg; tile < nlist && !failed; tile += tstride) {
        // the next tile's bounds (and, in the three-box form, its first boxes) are taken during
        // the gather of this tile's last plane
        Tile nxt = fetch_tile(nid);                  // loads in flight during this tile
        nid = tile_id(tile + 2 * tstride);
        const long long g0 = cur.g0;
        const bool mine = tile_mine(cur);
        const uint32_t pk = cur.pk;
        const bool region = cur.region;
        const int y0 = cur.y0, x0 = cur.x0, rh = cur.rh, rw = cur.rw, rp = cur.rp, frame = cur.frame;
        // blocks in this row's group (rows past the last group read group 0's count: unused)
        auto group_n = [&]() { return Shp::kShort ? min(max(a.count[g0], 1), G) : G; };
        if constexpr (Shp::kShort) {
            // a tile with a short group: this team's stacks get each group's own matrices (the
            // previous tile's products have completed: every product is waited for)
            const int gn = group_n();
            const bool tpart = !tc::wg_and(bar_id, TEAM, gn == G);
            zcol = tpart ? (uint32_t)(Shp::kPCol + wg * 2 * G) : (uint32_t)Shp::kZCol;
            if (tpart && t < 128) {
                const float *zr = ztn + (size_t)(gn - 1) * 2 * G * G + (size_t)j * G;
#pragma unroll
                for (int m = 0; m < 2; ++m)
#pragma unroll
                    for (int k0 = 0; k0 < G; k0 += 16) {
                        float v[16];
#pragma unroll
                        for (int e = 0; e < 16; ++e) v[e] = __ldg(zr + m * G * G + k0 + e);
                        tc::tmem_st16(tm + lrow + zcol + m * G + k0, v);
                    }
                tc::tmem_wait_st();
            }
        }
        for (int p = 0; p < 3 && !failed; ++p) {
            if (!a.process[p]) continue;
            const GroupLoc L = locate(a, p, g0, pk);
            const bool last = next_plane(p + 1) >= 3;
            // Every block enters the products with a level removed, so that the tf32 rounding
            // scales with the block's detail, not its level.  Hard threshold: each block's own
            // mean; the means' transform (the (0, 0) coefficients of every z frequency) is added
            // back in fp32 before the shrinkage and the shrunk (0, 0) coefficients leave the
            // inverse products and come back as one fp32 constant per block.  Wiener filter: one
            // level per group (the mean of its first block, source and reference), which only
            // the (0, 0, 0) coefficient carries: 512 G times the level, added back exactly, and
            // the shrunk (0, 0, 0) coefficient alone leaves the inverse products.
            float my_mu = 0.0f, my_mur = 0.0f;
            // (Wiener) groups of this warp's block steps and the first row of the first one
            constexpr int GW = NI / G > 1 ? NI / G : 1;
            const int gfirst = ((b0 + half * NI) / G) * G;
            // 1. gather (rows of foreign or partial groups are zero), one block per warp step
            if (region) {
                if constexpr (Shp::kBoxes == 3) {
                    if (half == 0) rowtab[r].x = mine ? ((L.y - y0) << 16) | (L.x - x0) : -1;
                    tc::cp_async_wait_all();
                    tc::wg_sync(bar_id, TEAM);
                    // (the three-box form is the Wiener filter's) the levels of this warp's groups
                    float lv[4];
#pragma unroll
                    for (int k = 0; k < 2; ++k) {
                        const int pq = k < GW ? rowtab[gfirst + k * G].x : -1;
                        const int o = pq >= 0 ? ((pq >> 16) + ry) * rp + (pq & 0xffff) + cx : 0;
                        lv[2 * k] = pq >= 0 ? Bs[o] + Bs[o + 4 * rp] : 0.f;
                        lv[2 * k + 1] = pq >= 0 ? Br[o] + Br[o + 4 * rp] : 0.f;
                    }
                    block_means<4>(lv, lane);
                    if (lane == 0)
#pragma unroll
                        for (int k = 0; k < GW; ++k) {
                            part[gfirst + k * G] = lv[2 * k];
                            part[128 + gfirst + k * G] = lv[2 * k + 1];
                        }
                    // four block steps per round: their loads are issued before any store (rounds
                    // unrolled: the swizzle of each step's row is a constant)
#pragma unroll
                    for (int ii = 0; ii < NI; ii += 4) {
                        const int i0 = half * NI + ii;
                        int pq[4];
                        float v0[4], v1[4], u0[4], u1[4];
#pragma unroll
                        for (int k = 0; k < 4; ++k) pq[k] = rowtab[b0 + i0 + k].x;
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const bool mi = pq[k] >= 0;
                            const int o = mi ? ((pq[k] >> 16) + ry) * rp + (pq[k] & 0xffff) + cx : 0;
                            v0[k] = mi ? Bs[o] : 0.f;
                            v1[k] = mi ? Bs[o + 4 * rp] : 0.f;
                            u0[k] = mi ? Br[o] : 0.f;
                            u1[k] = mi ? Br[o + 4 * rp] : 0.f;
                        }
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const int i = i0 + k;
                            const bool g1 = GW > 1 && b0 + i - gfirst >= G;
                            // rows past a short group's count stay zero
                            const bool mi = pq[k] >= 0;
                            const float ms = mi ? (g1 ? lv[2] : lv[0]) : 0.f, mr = mi ? (g1 ? lv[3] : lv[1]) : 0.f;
                            *reinterpret_cast<float *>(D + tc::sw128_offset(b0 + i, lane, 128)) = v0[k] - ms;
                            *reinterpret_cast<float *>(D + tc::sw128_offset(b0 + i, lane + 32, 128)) = v1[k] - ms;
                            *reinterpret_cast<float *>(D + Lay::kXBytes + tc::sw128_offset(b0 + i, lane, 128)) = u0[k] - mr;
                            *reinterpret_cast<float *>(D + Lay::kXBytes + tc::sw128_offset(b0 + i, lane + 32, 128)) = u1[k] - mr;
                        }
                    }
                    tc::wg_sync(bar_id, TEAM);
                    // the next plane's boxes load while this plane is filtered
                    if (!last) load_boxes(cur, next_plane(p + 1));
                } else {
                    const long long fo = (long long)frame * a.frame_stride;
                    const int nv = rh * (rw >> 2);
                    for (int pass = WIENER ? 0 : 1; pass < 2; ++pass) {
                        // pass 0: reference plane -> R; pass 1: source plane -> X
                        const float *plane = (pass == 0 ? a.ref[p] : a.src[p]) + fo + (long long)y0 * a.ld + x0;
                        unsigned char *dst = D + (pass == 0 ? Lay::kXBytes : 0);
                        for (int v = t; v < nv; v += TEAM) {
                            const int yy = v / (rw >> 2), c4 = v - yy * (rw >> 2);
                            tc::cp_async16(Rg + yy * rp + 4 * c4, plane + (long long)yy * a.ld + 4 * c4);
                        }
                        tc::cp_async_wait_all();
                        tc::wg_sync(bar_id, TEAM);
                        // (Wiener) the levels of this warp's groups in this plane
                        float lp[4] = {0.f, 0.f, 0.f, 0.f};
                        if constexpr (WIENER) {
#pragma unroll
                            for (int k = 0; k < 2; ++k) {
                                const int sl = (gfirst + k * G - b0) & 31;
                                const bool mi = __shfl_sync(0xffffffffu, mine, sl) && k < GW;
                                const int by = __shfl_sync(0xffffffffu, L.y, sl) - y0;
                                const int bx = __shfl_sync(0xffffffffu, L.x, sl) - x0;
                                const int o = mi ? (by + ry) * rp + bx + cx : 0;
                                lp[k] = mi ? Rg[o] + Rg[o + 4 * rp] : 0.f;
                            }
                            block_means<4>(lp, lane);
                            if (lane == 0)
#pragma unroll
                                for (int k = 0; k < GW; ++k) part[(pass == 0 ? 128 : 0) + gfirst + k * G] = lp[k];
                        }
                        // four block steps per round: their loads are issued before any store
                        for (int i0 = half * NI; i0 < half * NI + NI; i0 += 4) {
                            float v0[4], v1[4];
#pragma unroll
                            for (int k = 0; k < 4; ++k) {
                                const bool mi = __shfl_sync(0xffffffffu, mine, i0 + k);
                                const int by = __shfl_sync(0xffffffffu, L.y, i0 + k) - y0;
                                const int bx = __shfl_sync(0xffffffffu, L.x, i0 + k) - x0;
                                const int o = mi ? (by + ry) * rp + bx + cx : 0;
                                v0[k] = mi ? Rg[o] : 0.f;
                                v1[k] = mi ? Rg[o + 4 * rp] : 0.f;
                            }
                            float m4[4];
                            if constexpr (WIENER) {
#pragma unroll
                                for (int k = 0; k < 4; ++k) m4[k] = GW > 1 && b0 + i0 + k - gfirst >= G ? lp[1] : lp[0];
                            } else {
#pragma unroll
                                for (int k = 0; k < 4; ++k) m4[k] = v0[k] + v1[k];
                                block_means<4>(m4, lane);
                                if constexpr (SPLIT >= 2)
                                    if (lane == 0)
                                        *reinterpret_cast<float4 *>(part + b0 + i0) = make_float4(m4[0], m4[1], m4[2], m4[3]);
                            }
#pragma unroll
                            for (int k = 0; k < 4; ++k) {
                                const int i = i0 + k;
                                const float mu = m4[k];
                                if (lane == i) my_mu = mu;
                                *reinterpret_cast<float *>(dst + tc::sw128_offset(b0 + i, lane, 128)) = v0[k] - mu;
                                *reinterpret_cast<float *>(dst + tc::sw128_offset(b0 + i, lane + 32, 128)) = v1[k] - mu;
                            }
                        }
                        tc::wg_sync(bar_id, TEAM);
                    }
                    if constexpr (SPLIT >= 2) my_mu = part[r];
                }
            } else {
                const float *sp = L.src + (long long)L.y * a.ld + L.x;
                const float *rp = L.ref + (long long)L.y * a.ld + L.x;
#pragma unroll 4
                for (int i = half * NI; i < half * NI + NI; ++i) {
                    const bool mi = __shfl_sync(0xffffffffu, mine, i);
                    const float *si = reinterpret_cast<const float *>(__shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(sp), i));
                    unsigned char *d0 = D + tc::sw128_offset(b0 + i, lane, 128);
                    unsigned char *d1 = D + tc::sw128_offset(b0 + i, lane + 32, 128);
                    if (mi) {
                        tc::cp_async4(d0, si + (long long)ry * a.ld + cx);
                        tc::cp_async4(d1, si + (long long)(ry + 4) * a.ld + cx);
                    } else {
                        *reinterpret_cast<float *>(d0) = 0.0f;
                        *reinterpret_cast<float *>(d1) = 0.0f;
                    }
                    if constexpr (WIENER) {
                        const float *ri = reinterpret_cast<const float *>(__shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(rp), i));
                        if (mi) {
                            tc::cp_async4(d0 + Lay::kXBytes, ri + (long long)ry * a.ld + cx);
                            tc::cp_async4(d1 + Lay::kXBytes, ri + (long long)(ry + 4) * a.ld + cx);
                        } else {
                            *reinterpret_cast<float *>(d0 + Lay::kXBytes) = 0.0f;
                            *reinterpret_cast<float *>(d1 + Lay::kXBytes) = 0.0f;
                        }
                    }
                }
                tc::cp_async_wait_all();
                float lp[4] = {0.f, 0.f, 0.f, 0.f};
                if constexpr (WIENER) {
                    // the levels of this warp's groups (a group's first block may have been copied
                    // by the other warp of the quarter)
                    tc::wg_sync(bar_id, TEAM);
#pragma unroll
                    for (int k = 0; k < 2; ++k)
#pragma unroll
                        for (int op = 0; op < 2; ++op) {
                            const int row = k < GW ? gfirst + k * G : gfirst;
                            const float *d0 = reinterpret_cast<const float *>(D + op * Lay::kXBytes + tc::sw128_offset(row, lane, 128));
                            const float *d1 = reinterpret_cast<const float *>(D + op * Lay::kXBytes + tc::sw128_offset(row, lane + 32, 128));
                            lp[2 * k + op] = k < GW ? *d0 + *d1 : 0.f;
                        }
                    block_means<4>(lp, lane);
                    if (lane == 0)
#pragma unroll
                        for (int k = 0; k < GW; ++k) {
                            part[gfirst + k * G] = lp[2 * k];
                            part[128 + gfirst + k * G] = lp[2 * k + 1];
                        }
                    // every warp has read its levels before any block is changed
                    tc::wg_sync(bar_id, TEAM);
                }
                // each lane re-reads only the elements its own copies wrote
#pragma unroll 4
                for (int i = half * NI; i < half * NI + NI; ++i) {
                    // (kShort) rows past a short group's count stay zero
                    if (Shp::kShort && !__shfl_sync(0xffffffffu, mine, i)) continue;
#pragma unroll
                    for (int op = 0; op < (WIENER ? 2 : 1); ++op) {
                        float *d0 = reinterpret_cast<float *>(D + op * Lay::kXBytes + tc::sw128_offset(b0 + i, lane, 128));
                        float *d1 = reinterpret_cast<float *>(D + op * Lay::kXBytes + tc::sw128_offset(b0 + i, lane + 32, 128));
                        float mu;
                        if constexpr (WIENER) {
                            const bool g1 = GW > 1 && b0 + i - gfirst >= G;
                            mu = g1 ? lp[2 + op] : lp[op];
                        } else {
                            mu = block_mean(*d0, *d1);
                            if constexpr (SPLIT >= 2) if (lane == 0) part[b0 + i] = mu;
                        }
                        *d0 -= mu;
                        *d1 -= mu;
                        if (op == 0 && lane == i) my_mu = mu;
                    }
                }
                if constexpr (SPLIT >= 2) {
                    tc::wg_sync(bar_id, TEAM);
                    my_mu = part[r];
                }
            }
            // (Wiener) the group's levels, read before the shrinkage reuses the scratch row
            if constexpr (WIENER && !ZT) {
                my_mu = part[r];
                my_mur = part[128 + r];
            }
            if (last) {
                bound_tile(nxt);
                if constexpr (Shp::kBoxes == 3)
                    if (nxt.region) load_boxes(nxt, pfirst);
            }
            publish();
            // 2. 2-D DCT
            if (t == 0) {
                if constexpr (WIENER) xy_ss2(0, sD, 64, sD + Lay::kXBytes, sKf);
                else xy_ss(0, sD, sKf);
                tc::mma_commit(mb);
            }
            if (!wait_mma()) { failed = true; break; }
            float denW = 0.0f, numW = 0.0f;
            float s00 = 0.0f;                          // (old z stage) this row's shrunk (0, 0) coefficient
            if constexpr (ZT) {
                // 3'. transpose into the z-stage A operands: row (h, c) of Ys holds coefficient c of
                // the blocks 64 h .. 64 h + 63 (K); Yr the same for the reference
                const int rb = 64 * (r >> 6), kb = r & 63;
#pragma unroll
                for (int op = 0; op < 2; ++op) {
                    float v[NC];
#pragma unroll
                    for (int q = 0; q < NC; q += 16) tc::tmem_ld16(tb + lrow + 64 * op + cb + q, *reinterpret_cast<float (*)[16]>(v + q));
                    tc::tmem_wait_ld();
#pragma unroll
                    for (int e = 0; e < NC; ++e)
                        *reinterpret_cast<float *>(D + op * Lay::kXBytes + tc::sw128_offset(rb + cb + e, kb, 128)) = v[e];
                }
                publish();
                // 4'. z-DCT: lanes (h, c), columns 32 g' + kz of group g' of half h: the K range of
                // the group's 32 blocks times Dz[kz][b] (source into cols 0-63, reference 64-127)
                if (t == 0) {
                    // K step outer: consecutive products go to the four independent chains
                    const uint64_t ad = tc::make_desc_sw128(sD, 1024), bd = tc::make_desc(sZt, 128, 1024);
#pragma unroll
                    for (int s = 0; s < 4; ++s)
#pragma unroll
                        for (int op = 0; op < 2; ++op)
#pragma unroll
                            for (int w2 = 0; w2 < 2; ++w2)
                                tc::mma_tf32_ss(tb + 64 * op + 32 * w2,
                                                ad + (uint64_t)((op * Lay::kXBytes + w2 * 16 * 1024 + s * 32) >> 4),
                                                bd + (uint64_t)(s * 16), IDZT, s > 0);
                    tc::mma_commit(mb);
                }
                if (!wait_mma()) { failed = true; break; }
                // 5'. Wiener shrinkage: thread (h, c) holds coefficient c of the 32 z frequencies of
                // group g = 2 h + half, source and reference
                {
                    const int c = r & 63, g = 2 * (r >> 6) + half;
                    float z[32], rr[32];
                    tc::tmem_ld16(tb + lrow + cb, *reinterpret_cast<float (*)[16]>(z));
                    tc::tmem_ld16(tb + lrow + cb + 16, *reinterpret_cast<float (*)[16]>(z + 16));
                    tc::tmem_ld16(tb + lrow + 64 + cb, *reinterpret_cast<float (*)[16]>(rr));
                    tc::tmem_ld16(tb + lrow + 64 + cb + 16, *reinterpret_cast<float (*)[16]>(rr + 16));
                    tc::tmem_wait_ld();
                    if (c == 0) {
                        // the group's levels: (0, 0, 0) = 2 G sum (256 level) of the 2-D DC
                        z[0] += part[32 * g] * (float)(512 * G);
                        rr[0] += part[128 + 32 * g] * (float)(512 * G);
                    }
                    // Wiener weights two coefficients at a time (packed fp32 pairs)
                    const float sg = a.wsig2[p][G - 1];
                    const tc::f2 sg2 = tc::pk(sg, sg);
                    tc::f2 acc2 = tc::pk(0.0f, 0.0f);
#pragma unroll
                    for (int e = 0; e < 32; e += 2) {
                        const tc::f2 rv = tc::pk(rr[e], rr[e + 1]);
                        const tc::f2 r2 = tc::mul2(rv, rv);
                        const tc::f2 den = tc::fma2(rv, rv, sg2);
                        float d0, d1;
                        tc::upk(den, d0, d1);
                        const tc::f2 w = tc::mul2(r2, tc::pk(__fdividef(1.0f, d0), __fdividef(1.0f, d1)));
                        tc::upk(tc::mul2(tc::pk(z[e], z[e + 1]), w), z[e], z[e + 1]);
                        acc2 = tc::fma2(w, w, acc2);
                    }
                    float acc, acc_hi;
                    tc::upk(acc2, acc, acc_hi);
                    acc += acc_hi;
                    if (c == 0) {
                        // S(0, 0, 0) leaves the inverse products (added back per block, exactly)
                        part[32 * g] = z[0];
                        z[0] = 0.0f;
                    }
                    tc::tmem_st16(tb + lrow + cb, *reinterpret_cast<const float (*)[16]>(z));
                    tc::tmem_st16(tb + lrow + cb + 16, *reinterpret_cast<const float (*)[16]>(z + 16));
                    tc::tmem_wait_st();
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
                    if (lane == 0) part[1 + 2 * g + ((r >> 5) & 1)] = acc;
                }
                publish();
                // 6'. inverse z: T[(h, c)][32 g' + b] = sum_kz S[(h, c)][32 g' + kz] Ci[b][kz] (A from
                // tensor memory) into cols 64-127
                if (t == 0) {
                    const uint64_t bd = tc::make_desc(sCi, 128, 1024);
#pragma unroll
                    for (int s = 0; s < 4; ++s)
#pragma unroll
                        for (int w2 = 0; w2 < 2; ++w2)
                            tc::mma_tf32_ts(tb + 64 + 32 * w2, tb + 32 * w2 + 8 * s, bd + (uint64_t)(s * 16), IDZT, s > 0);
                    tc::mma_commit(mb);
                }
                if (!wait_mma()) { failed = true; break; }
                // T back to rows of blocks: At[b][c] (A operand of the inverse 2-D product)
                {
                    float v[NC];
#pragma unroll
                    for (int q = 0; q < NC; q += 16) tc::tmem_ld16(tb + lrow + 64 + cb + q, *reinterpret_cast<float (*)[16]>(v + q));
                    tc::tmem_wait_ld();
#pragma unroll
                    for (int e = 0; e < NC; ++e)
                        *reinterpret_cast<float *>(D + tc::sw128_offset(rb + cb + e, kb, 128)) = v[e];
                }
                publish();
                if (t == 0) {
                    xy_ss(0, sD, sKi);
                    tc::mma_commit(mb);
                }
                if (!wait_mma()) { failed = true; break; }
                // the block's group weights
                {
                    const int g = r / G;
                    const float acc = part[1 + 2 * g] + part[2 + 2 * g];
                    const float eps = 1.1920928955078125e-07f;
                    denW = 1.0f / (acc > eps ? acc : eps);
                    numW = denW / a.amp[G - 1];
                }
            } else {
            // 3. transpose into the z-stage B operand (reference rows below the source rows)
            row_to_column(0, 0, NT);
            if constexpr (WIENER) row_to_column(64, 64, NT);
            publish();
            // 4. z-DCT of source (and reference) in one pass
            if (t == 0) {
                z_stage(0, sZf, NT, IDZ);
                tc::mma_commit(mb);
            }
            if (!wait_mma()) { failed = true; break; }
            // 5. shrinkage, one row of 64 coefficients per thread
            float acc = 0.0f;
            const int gn = group_n();
            float thr[3];                              // by the number of zero (y, x) frequencies
#pragma unroll
            for (int k = 0; k < 3; ++k) thr[k] = WIENER ? 0.0f : a.thr4[p][G - 1][(j == 0) + k];
            // (hard threshold) the exact z transform of the block means' (0, 0) coefficients 256 mu
            // (only the first column half holds column 0)
            float dcz = 0.0f, dczr = 0.0f;
            uint64_t flags = 0;                        // columns (relative to cb) to recompute
            if constexpr (WIENER) {
                // the group's levels: sum_b Dz[0][b] = 2 G, sum_b Dz[kz][b] = 0 for kz > 0
                if (half == 0 && j == 0) {
                    dcz = my_mu * (float)(2 * gn);
                    dczr = my_mur * (float)(2 * gn);
                }
            } else if constexpr (SPLIT >= 2) {
                if (half == 0) {
                    // the group's means from shared memory, four per broadcast load
                    const float4 *m4 = reinterpret_cast<const float4 *>(part + (r / G) * G);
#pragma unroll 2
                    for (int b4 = 0; b4 < G / 4; ++b4) {
                        const float4 m = m4[b4];
                        const float d0 = __ldg(dzt + (4 * b4) * G + j), d1 = __ldg(dzt + (4 * b4 + 1) * G + j);
                        const float d2 = __ldg(dzt + (4 * b4 + 2) * G + j), d3 = __ldg(dzt + (4 * b4 + 3) * G + j);
                        dcz = fmaf(d0, m.x, fmaf(d1, m.y, fmaf(d2, m.z, fmaf(d3, m.w, dcz))));
                    }
                }
            } else {
                const int gl = (lane / G) * G;         // lane of the group's first block
#pragma unroll 4
                for (int b = 0; b < G; ++b)
                    dcz = fmaf(__ldg(dzt + b * G + j), __shfl_sync(0xffffffffu, my_mu, gl + b), dcz);
            }
            dcz *= 256.0f;
            dczr *= 256.0f;
            // the recheck interval [lo, hi] of |c| around each of the three threshold classes
            float tlo[3], thi[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float band = WIENER ? 0.0f : a.recheck_band;
                tlo[k] = mine ? thr[k] * (1.0f - band) : 3.0e38f;
                thi[k] = thr[k] * (1.0f + band);
            }
#pragma unroll
            for (int c0 = 0; c0 < NC; c0 += 32) {
                float z[32];
                tc::tmem_ld16(tb + lrow + cb + c0, *reinterpret_cast<float (*)[16]>(z));
                tc::tmem_ld16(tb + lrow + cb + c0 + 16, *reinterpret_cast<float (*)[16]>(z + 16));
                if constexpr (WIENER) {
                    float rr[32];
                    tc::tmem_ld16(tb + lrow + 64 + cb + c0, *reinterpret_cast<float (*)[16]>(rr));
                    tc::tmem_ld16(tb + lrow + 64 + cb + c0 + 16, *reinterpret_cast<float (*)[16]>(rr + 16));
                    tc::tmem_wait_ld();
                    if (cb + c0 == 0) {
                        z[0] += dcz;
                        rr[0] += dczr;
                    }
                    const float sg = a.wsig2[p][gn - 1];
#pragma unroll
                    for (int e = 0; e < 32; ++e) {
                        const float r2 = rr[e] * rr[e];
                        const float w = __fdividef(r2, r2 + sg);
                        z[e] *= w;
                        acc = fmaf(w, w, acc);
                    }
                } else {
                    tc::tmem_wait_ld();
                    if (cb + c0 == 0) z[0] += dcz;
#pragma unroll
                    for (int e = 0; e < 32; ++e) {
                        const int c = cb + c0 + e;
                        const int k = ((c & 7) == 0) + ((c >> 3) == 0);
                        const float az = fabsf(z[e]);
                        const bool keep = az > thr[k];
                        if (az >= tlo[k] && az <= thi[k]) flags |= 1ull << (c0 + e);
                        acc += keep ? 1.0f : 0.0f;
                        z[e] = keep ? z[e] : 0.0f;
                    }
                }
#pragma unroll
                for (int e = 0; e < 32; ++e) *reinterpret_cast<float *>(D + tc::sw128_offset(cb + c0 + e, r, 64)) = z[e];
            }
            if constexpr (!WIENER) {
                // coefficients near their threshold: the value from the pixels in double precision
                // decides, sum_b Dz[kz][b] sum_y C8[u][y] sum_x C8[v][x] x_b(y, x); the warp
                // computes one at a time, lane = (pixel row y, every fourth block)
                while (true) {
                    const unsigned anyf = __ballot_sync(0xffffffffu, flags != 0ull);
                    if (!anyf) break;
                    const int ldr = __ffs(anyf) - 1;
                    const uint64_t lf = __shfl_sync(0xffffffffu, flags, ldr);
                    const int c = cb + __ffsll((long long)lf) - 1;
                    const int u = c >> 3, v = c & 7, kz = ldr % G, gl = (ldr / G) * G;
                    const int yy = lane & 7;
                    double sum = 0.0;
#pragma unroll
                    for (int k = 0; k < G / 4; ++k) {
                        const int bb = (lane >> 3) + 4 * k;
                        const float *px;
                        long long pitch;
                        if (region) {
                            const int by = __shfl_sync(0xffffffffu, L.y, gl + bb) - y0, bx = __shfl_sync(0xffffffffu, L.x, gl + bb) - x0;
                            px = Rg + (by + yy) * rp + bx;
                            pitch = rp;
                        } else {
                            const float *sp = L.src + (long long)L.y * a.ld + L.x;
                            px = reinterpret_cast<const float *>(__shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(sp), gl + bb)) +
                                 (long long)yy * a.ld;
                            pitch = a.ld;
                        }
                        (void)pitch;
                        double rs = 0.0;
#pragma unroll
                        for (int x = 0; x < 8; ++x) rs = fma(__ldg(xtab + v * 8 + x), (double)px[x], rs);
                        sum = fma(__ldg(xtab + 64 + kz * G + bb) * __ldg(xtab + u * 8 + yy), rs, sum);
                    }
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
                    if (lane == ldr) {
                        flags &= flags - 1;
                        float *sv = reinterpret_cast<float *>(D + tc::sw128_offset(c, r, 64));
                        const float th = thr[((c & 7) == 0) + ((c >> 3) == 0)];
                        const bool keep_old = *sv != 0.0f, keep_new = fabs(sum) > (double)th;
                        *sv = keep_new ? (float)sum : 0.0f;
                        acc += (keep_new ? 1.0f : 0.0f) - (keep_old ? 1.0f : 0.0f);
                        ++n_recheck;
                        n_changed += keep_new != keep_old;
                    }
                }
            }
            // the shrunk (0, 0) coefficient of this row (Wiener: of the group's kz = 0 row) leaves
            // the inverse products
            if (cb == 0 && (!WIENER || j == 0)) {
                float *s0p = reinterpret_cast<float *>(D + tc::sw128_offset(0, r, 64));
                s00 = *s0p;
                *s0p = 0.0f;
            }
#pragma unroll
            for (int o = G / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if constexpr (SPLIT == 2) {
                // the group's sum is the sum of the two column halves
                part[t] = acc;
                tc::wg_sync(bar_id, TEAM);
                acc = part[r] + part[r + 128];
            }
            if constexpr (!WIENER)
                if (a.retained && mine && j == 0 && half == 0) a.retained[(long long)p * a.ngroups + g0] = (int)acc;
            if constexpr (WIENER) {
                const float eps = 1.1920928955078125e-07f;
                denW = 1.0f / (acc > eps ? acc : eps);
            } else {
                denW = acc < 1.0f ? 1.0f : 1.0f / acc;
            }
            numW = denW / a.amp[gn - 1];
            publish();
            // (the barriers of the two inverse waits below order this before the aggregation)
            if constexpr (SPLIT >= 2) if (half == 0) part[r] = s00;
            // 6. inverse z, then inverse 2-D
            if (t == 0) {
                z_stage(0, sZi, 64, ID64);
                tc::mma_commit(mb);
            }
            if (!wait_mma()) { failed = true; break; }
            if (t == 0) {
                xy_ts(64, 0, sKi);
                tc::mma_commit(mb);
            }
            if (!wait_mma()) { failed = true; break; }
            }
            // 7. aggregation: rows -> shared memory (this quarter's 32 rows), then one block per step
            {
                float v[NC];
#pragma unroll
                for (int c0 = 0; c0 < NC; c0 += 16) tc::tmem_ld16(tb + lrow + (ZT ? 0 : 64) + cb + c0, *reinterpret_cast<float (*)[16]>(v + c0));
                // the inverse of the (0, 0) coefficients: block j of the group gets
                // sum_kz Ci[j][kz] S(kz, 0, 0), Ci[j][0] = 1, Ci[j][kz] = Dz[kz][j]
                float dcb = 0.0f;
                if constexpr (WIENER) {
                    dcb = part[(r / G) * G];           // the inverse of S(0, 0, 0) alone: a constant
                } else if constexpr (SPLIT >= 2) {
                    const float4 *s4 = reinterpret_cast<const float4 *>(part + (r / G) * G);
#pragma unroll 2
                    for (int k4 = 0; k4 < G / 4; ++k4) {
                        const float4 sk = s4[k4];
                        dcb = fmaf(__ldg(dzi + (4 * k4) * G + j), sk.x, dcb);
                        dcb = fmaf(__ldg(dzi + (4 * k4 + 1) * G + j), sk.y, dcb);
                        dcb = fmaf(__ldg(dzi + (4 * k4 + 2) * G + j), sk.z, dcb);
                        dcb = fmaf(__ldg(dzi + (4 * k4 + 3) * G + j), sk.w, dcb);
                    }
                } else {
                    const int gl = (lane / G) * G;
#pragma unroll 4
                    for (int kz = 0; kz < G; ++kz)
                        dcb = fmaf(__ldg(dzi + kz * G + j), __shfl_sync(0xffffffffu, s00, gl + kz), dcb);
                }
                tc::tmem_wait_ld();
#pragma unroll
                for (int c = 0; c < NC; ++c) v[c] += dcb;
#pragma unroll
                for (int c = 0; c < NC; c += 4)
                    *reinterpret_cast<float4 *>(D + tc::sw128_offset(r, cb + c, 128)) = make_float4(v[c], v[c + 1], v[c + 2], v[c + 3]);
                // Region mode accumulates in 32-bit fixed point: integer shared-memory atomics are
                // native, float ones are not.  The scale is a power of two chosen per tile so that
                // 128 contributions of the largest magnitude stay below 2^30.
                float cmax = 0.0f;
                if (region && mine) {
#pragma unroll
                    for (int c = 0; c < NC; ++c) cmax = fmaxf(cmax, fabsf(v[c]));
                    cmax *= numW;
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) cmax = fmaxf(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
                if ((t & 31) == 0) reinterpret_cast<float *>(bbx)[t >> 5] = cmax;
                if constexpr (Shp::kBoxes == 3)
                    if (half == 0) rowtab[r].y = __float_as_int(numW);
                int *Ri = reinterpret_cast<int *>(Rg);
                if ((Shp::kBoxes == 1 || ZT) && region)   // (the three-box form clears it in the flush)
                    for (int e = t; e < rh * rp; e += TEAM) Ri[e] = 0;
                tc::wg_sync(bar_id, TEAM);
                float scale = 1073741824.0f;                 // 2^30
                if (region) {
#pragma unroll
                    for (int q = 0; q < TEAM / 32; ++q) cmax = fmaxf(cmax, reinterpret_cast<const float *>(bbx)[q]);
                    if (cmax > 1e-20f) {
                        int ex;
                        frexpf(1073741824.0f / (128.0f * cmax), &ex);   // 2^(ex-1) <= bound < 2^ex
                        scale = ldexpf(1.0f, ex - 1);
                    } else if (cmax > 0.0f) {
                        scale = 1.0e30f;                         // contributions below 1e-20
                    }
                }
                float *np = L.num + (long long)L.y * a.ld + L.x;
                if (Shp::kBoxes == 3 && region) {
                    // four block steps per round: rows and table entries loaded before the atomics
#pragma unroll
                    for (int ii = 0; ii < NI; ii += 4) {
                        const int i0 = half * NI + ii;
                        int2 q[4];
                        float x0v[4], x1v[4];
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            q[k] = rowtab[b0 + i0 + k];
                            x0v[k] = *reinterpret_cast<const float *>(D + tc::sw128_offset(b0 + i0 + k, lane, 128));
                            x1v[k] = *reinterpret_cast<const float *>(D + tc::sw128_offset(b0 + i0 + k, lane + 32, 128));
                        }
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            if (q[k].x >= 0) {
                                const int o = ((q[k].x >> 16) + ry) * rp + (q[k].x & 0xffff) + cx;
                                const float ws = __int_as_float(q[k].y) * scale;
                                atomicAdd(Ri + o, __float2int_rn(x0v[k] * ws));
                                atomicAdd(Ri + o + 4 * rp, __float2int_rn(x1v[k] * ws));
                            }
                    }
                }
                if (Shp::kBoxes == 1 && region) {
                    for (int i0 = half * NI; i0 < half * NI + NI; i0 += 4) {
                        int o[4];
                        float ws[4], x0v[4], x1v[4];
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const bool mi = __shfl_sync(0xffffffffu, mine, i0 + k);
                            ws[k] = __shfl_sync(0xffffffffu, numW, i0 + k) * scale;
                            const int by = __shfl_sync(0xffffffffu, L.y, i0 + k) - y0;
                            const int bx = __shfl_sync(0xffffffffu, L.x, i0 + k) - x0;
                            o[k] = mi ? (by + ry) * rp + bx + cx : -1;
                            x0v[k] = *reinterpret_cast<const float *>(D + tc::sw128_offset(b0 + i0 + k, lane, 128));
                            x1v[k] = *reinterpret_cast<const float *>(D + tc::sw128_offset(b0 + i0 + k, lane + 32, 128));
                        }
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            if (o[k] >= 0) {
                                atomicAdd(Ri + o[k], __float2int_rn(x0v[k] * ws[k]));
                                atomicAdd(Ri + o[k] + 4 * rp, __float2int_rn(x1v[k] * ws[k]));
                            }
                    }
                }
#pragma unroll 4
                for (int i = half * NI; i < half * NI + NI; ++i) {
                    if (region) break;
                    const bool mi = __shfl_sync(0xffffffffu, mine, i);
                    const float wi = __shfl_sync(0xffffffffu, numW, i);
                    {
                        float *ni = reinterpret_cast<float *>(__shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(np), i));
                        if (mi) {
                            const float x0v = *reinterpret_cast<const float *>(D + tc::sw128_offset(b0 + i, lane, 128));
                            const float x1v = *reinterpret_cast<const float *>(D + tc::sw128_offset(b0 + i, lane + 32, 128));
                            atomicAdd(ni + (long long)ry * a.ld + cx, x0v * wi);
                            atomicAdd(ni + (long long)(ry + 4) * a.ld + cx, x1v * wi);
                        }
                    }
                }
                if (region) {
                    // the region's sums, one vector atomic per 4 pixels (untouched ones skipped)
                    tc::wg_sync(bar_id, TEAM);
                    float *nbase = a.num[p] + (long long)frame * a.frame_stride + (long long)y0 * a.ld + x0;
                    const int w4 = rw >> 2, nv = rh * w4;
                    const uint32_t md = div_magic((uint32_t)w4);
                    for (int e = t; e < nv; e += TEAM) {
                        const int yy = (int)__umulhi((uint32_t)e, md), c4 = e - yy * w4;
                        const int4 qi = *reinterpret_cast<const int4 *>(Ri + yy * rp + 4 * c4);
                        if (qi.x != 0 || qi.y != 0 || qi.z != 0 || qi.w != 0) {
                            const float inv = 1.0f / scale;
                            const float4 q = make_float4((float)qi.x * inv, (float)qi.y * inv, (float)qi.z * inv, (float)qi.w * inv);
                            atomicAdd(reinterpret_cast<float4 *>(nbase + (long long)yy * a.ld + 4 * c4), q);
                            // (the three-box form keeps its box zero; ZT zeroes it before each use)
                            if constexpr (Shp::kBoxes == 3 && !ZT) *reinterpret_cast<int4 *>(Ri + yy * rp + 4 * c4) = make_int4(0, 0, 0, 0);
                        }
                    }
                }
            }
            if (mine && half == 0) atomicAdd(L.wmap + (long long)L.y * a.ld + L.x, denW);
            tc::fence_before_sync();
            tc::wg_sync(bar_id, TEAM);
            tc::fence_after_sync();
        }
        cur = nxt;
    }
    tc::cp_async_wait_all();                          // no box copy outlives the kernel
    if (failed) {
        // a timed-out wait leaves products possibly in flight: one more commit, which arrives once
        // every product the issuing thread started has completed, is waited for (bounded) before
        // the tensor memory is released; status 1 = time-out, 3 = the drain timed out as well
        if (t == 0) tc::mma_commit(&mdrain[wg]);
        const bool drained = tc::mbar_wait_bounded(&mdrain[wg], 0, kTcWaitLimit);
        tc::fence_after_sync();
        if (t == 0) atomicOr(status, drained ? 1 : 3);
    }
    if (!WIENER && a.tc_stats && n_recheck) {
        atomicAdd(a.tc_stats, n_recheck);
        atomicAdd(a.tc_stats + 1, n_changed);
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_free(tm, Shp::kTmemCols);
}

}  // namespace bm3d
