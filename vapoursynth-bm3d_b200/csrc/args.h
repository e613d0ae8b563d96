// args.h -- plain argument structures shared by the host code and the kernels (no device code).
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define BM3D_HD __host__ __device__
#else
#define BM3D_HD
#endif

namespace bm3d {

// ---------------------------------------------------------------------------------------------
// Packed block positions.  BM3D lists: (y << 16) | x.  V-BM3D lists: (z << 26) | (y << 13) | x
// with z the frame index inside the temporal window (< 64) and y, x < 8192.

BM3D_HD inline uint32_t pack_yx(int y, int x) { return ((uint32_t)y << 16) | (uint32_t)x; }
BM3D_HD inline int unpack_y(uint32_t p) { return (int)(p >> 16); }
BM3D_HD inline int unpack_x(uint32_t p) { return (int)(p & 0xffffu); }

BM3D_HD inline uint32_t pack_zyx(int z, int y, int x) { return ((uint32_t)z << 26) | ((uint32_t)y << 13) | (uint32_t)x; }
BM3D_HD inline int unpack3_z(uint32_t p) { return (int)(p >> 26); }
BM3D_HD inline int unpack3_y(uint32_t p) { return (int)((p >> 13) & 0x1fffu); }
BM3D_HD inline int unpack3_x(uint32_t p) { return (int)(p & 0x1fffu); }

// Shared-memory floats per warp (host and device must agree).
BM3D_HD inline int bm_warp_floats(int cand_cap, int G, int B, bool generic)
{
    return cand_cap + 64 + 2 * G + (generic ? B * B : 0);
}
// bm_learned_kernel: scores, then a 128-entry candidate list
BM3D_HD inline int prop_warp_floats(int cand_cap) { return cand_cap + 128; }
// per warp: sp, tmp (at least 128 entries: also the radix-selection histogram), sk, the
// concatenated list (keys, positions), the per-frame selection, centres, heap, reference block
BM3D_HD inline int vbm_tmp_cap(int sp_cap) { return sp_cap > 128 ? sp_cap : 128; }
BM3D_HD inline int vbm_warp_floats(int sp_cap, int list_cap, int G, int ps_num, int B)
{
    return 2 * sp_cap + vbm_tmp_cap(sp_cap) + 4 * list_cap + 2 * G + ps_num + B * B;
}

// Precision-form block matching (bm_tc_kernel): at most kBmtRefs reference blocks per CTA and
// kBmtCols candidate columns (the union of their search windows along the row).
constexpr int kBmtRefs = 8;
constexpr int kBmtCols = 64;

// Shared-memory layout of bm_tc_kernel for a search range (candidate step 1), plane height and
// reference block step.
struct BmtLayout {
    int wh;           // window rows (<= 2 range + 8)
    int wp;           // window pitch in floats (odd)
    int nr;           // candidate rows (<= 2 range + 1)
    int cs;           // per-reference distance slots (>= (2 range + 1)^2 + 1, even)
    int nrc;          // reference blocks per CTA (their windows span <= kBmtCols columns)
    int offU, offR, offWin, offRsq, offSd, offScr, bytes;
};

// nrc = 0: the range is too wide for the form
inline BmtLayout bmt_layout(int range, int H, int block_step)
{
    BmtLayout L{};
    const int span = 2 * range + 1;
    L.nrc = span > kBmtCols ? 0 : (kBmtCols - span) / block_step + 1;
    if (L.nrc > kBmtRefs) L.nrc = kBmtRefs;
    L.nr = span < H - 7 ? span : H - 7;
    L.wh = L.nr + 7;
    L.wp = (kBmtCols + 7) | 1;
    L.cs = (span * span + 1 + 1) & ~1;
    int o = 0;
    L.offU = o;   o += (L.wh + 1) * kBmtCols * 16;           // fp16 candidate rows (+1 zero row)
    L.offR = o;   o += 16 * 64 * 2;                          // reference blocks: high terms, low terms
    L.offWin = o; o += (L.wh * L.wp * 4 + 15) & ~15;         // fp32 window
    L.offRsq = o; o += L.wh * kBmtCols * 4;                  // row sums of squares of the candidates
    L.offSd = o;  o += kBmtRefs * L.cs * 4;                  // distance estimates
    L.offScr = o; o += kBmtRefs * 192 * 4;                   // per-warp selection scratch
    L.bytes = o;
    return L;
}

enum SampleKind : int { SK_U8 = 0, SK_U16 = 1, SK_F32 = 2 };

struct BMArgs {
    const float *ref;          // plane of frame 0; frame f at ref + f * frame_stride
    long long frame_stride;
    int ld, H, W;
    int B, range, step;        // range already rounded down to a multiple of step
    int G;
    float thSSE;
    double distMul;
    const int *scan_y;
    const int *scan_x;
    int nby, nbx;
    uint32_t *out_pos;         // [frame][by][bx][G], packed (y << 16) | x
    int *out_n;                // [frame][by][bx]
    float *out_key;            // optional, [frame][by][bx][G]
    unsigned long long *stats; // optional: [0] blocks that took the exact heap path, [1] precision
                               // forms: blocks that needed an exact fallback, [2] tensor-core time-outs
    uint32_t *out_prop;        // optional (learned proposals): [frame][by][bx][nprop] candidate
                               // indices of each block's proposal set, unused slots 0xffffffff
    int warps;                 // warps per CTA
    int win_h, win_pitch;      // shared window capacity
    int cand_cap;              // per-warp distance slots (>= lattice + 1)
};

struct CFArgs {
    // planes of frame 0 (float workspace), frame f at + f * frame_stride
    const float *src[3];
    const float *ref[3];
    float *num[3];
    float *wmap[3];
    long long frame_stride;
    int ld, H, W;
    int process[3];
    int B, G;
    int wiener;
    // match lists: groups ordered [frame][by][bx]; blocks_per_frame = nby * nbx
    const uint32_t *pos;       // [group][G], packed (y<<16)|x, or (z<<26)|(y<<13)|x for V-BM3D
    const int *count;          // [group]
    long long ngroups;
    long long blocks_per_frame;
    int vbm3d;                 // positions carry a window frame index
    // V-BM3D: planes of window frame z for output frame f are at src[p] + (win_base[f] + z) *
    // frame_stride; accumulator slot for window frame z at num[p] + (f * slots + slot0[f] + z) * acc_stride
    const int *win_base;       // [frame] first clip frame of the window (V-BM3D)
    const int *slot0;          // [frame] first slot index (V-BM3D)
    int slots;                 // slots per output frame (2r+1)
    long long acc_stride;      // elements between accumulator slots
    // filter data per plane
    float thr4[3][256][4];     // [plane][n-1][flag]   (Basic)
    float wsig2[3][256];       // [plane][n-1]         (Final)
    float amp[256];            // finalAMP[n-1] = 2n*2B*2B (exact in float)
    // generic path
    const float *odd_all;      // odd tables N = 2..256
    const float *dtab;         // direct tables (fwd then inv) for non-power-of-two N
    const int *dtab_off;       // [N] offset of the fwd table of length N in dtab (-1 if absent)
    float *scratch;            // per-warp scratch for the generic path
    long long scratch_per_warp;
    int skip_full;             // generic kernel: skip groups the fast kernel handles
    // optional (fast kernel with skip_full): the partial groups' indices and their count on the
    // device; the kernel then walks this list instead of every group
    const long long *plist;
    const unsigned int *plist_n;
    // optional (tensor-core kernels): the tiles to filter, *tlist_n entries, instead of all
    const int *tlist;
    const unsigned int *tlist_n;
    // precision form, hard threshold: a coefficient whose tensor-core value lies within
    // recheck_band * thr of its threshold is recomputed in fp32 from the pixels before the keep /
    // zero decision (0 disables); tc_stats counts [0] coefficients recomputed, [1] decisions the
    // recomputation changed
    float recheck_band;
    unsigned long long *tc_stats;
    // optional (hard threshold): retained-coefficient count of every group, [plane][group]
    int *retained;
};

struct VBMArgs {
    const float *ref;             // reference Y planes of the clip window workspace
    long long frame_stride;
    int ld, H, W;
    int B, G, ps_num, ps_range, ps_step;   // ps_range already rounded to a multiple of ps_step
    float thSSE;
    double distMul;
    const int *scan_y, *scan_x;
    int nby, nbx;
    // per output frame f of the batch: window start (clip frame index in the workspace), length,
    // index of the current frame inside the window
    const int *win_base, *win_len, *win_cur;
    // current-frame lists from K1: [f][by][bx][G] positions (y<<16|x), keys, counts
    const uint32_t *cur_pos;
    const float *cur_key;
    const int *cur_n;
    // output: [f][by][bx][G] packed (z<<26|y<<13|x), optional keys, counts
    uint32_t *out_pos;
    float *out_key;
    int *out_n;
    unsigned long long *stats;
    int warps;
    int sp_cap;                   // capacity of the per-warp search-position list
    int list_cap;                 // capacity of the per-warp concatenated list
    // learned proposals (optional): bf16 descriptors of the window frames, desc_frame elements
    // of kPropCh values per frame; the other frames' search positions are ranked by descriptor
    // distance and only the best nprop get exact distances
    const void *desc;
    long long desc_frame;
    int nprop;
};

struct PlanePtr {
    void *ptr;
    long long stride;   // bytes
};

// One linear channel: out = clip?(in * gain + offset)
struct LinearOp {
    float gain, offset, lo, hi;
    int clip;
};

// Conversion program for one frame set.  mode:
//   0 LINEAR  : out[c] = op[c](in[c])                       (RangeConvert)
//   1 RGB2OPP : Y = ((R+G)+B)*gY+oY, U = (R-B)*gU+oC, V = ((R-2G)+B)*gV+oC   (MatrixConvert_RGB2YUV)
//   2 RGB2Y   : Y = ((R+G)+B)*g+o                               (ConvertToY, OPP)
//   3 OPP2RGB : R = ((Ry*Y+Ru*U)+Rv*V)+oR, G = (Gy*Y+Gv*V)+oG, B = ((By*Y+Bu*U)+Bv*V)+oB
struct ConvProgram {
    int mode;
    int raw;                // 1: plain copy (same sample kind in and out)
    int in_kind, out_kind;
    int nin, nout;
    LinearOp op[3];
    float coef[9];          // OPP2RGB: Ry Ru Rv Gy Gu Gv By Bu Bv (already scaled by the gains)
    float off[3];
    int W, H;
};

// finalize: out = num / box_B(wmap) for processed planes of a batch of frames.
// FP64 oracle outputs and constants (inspection only)
struct F64Args {
    double *num[3];
    double *den[3];          // per-pixel denominator (not the per-origin weight map)
    double sigma[3];         // sigma / 255 * matrix norm, per plane
    double lambda;
    long long out_stride;    // doubles between rows of num / den
};

struct FinalizeArgs {
    const float *num[3];
    const float *wmap[3];
    float *out[3];
    long long frame_stride;
    int ld, H, W, B;
    int process[3];
};

// VAggregate for a batch of output frames.  in[(f * frames_max + i) * 3 + p] points to plane p of
// the stacked frame n + b_off + i; slot o = radius - b_off - i holds the numerator, o + 1 the
// denominator.  The result is written as float into out workspace planes.
struct VAggArgs {
    const PlanePtr *in;
    int frames_max;
    const int *nframes;     // [f] window length
    const int *b_off;       // [f]
    float *out[3];
    long long frame_stride;
    int ld, H, W, radius;
    int process[3];
};

// V-BM3D output: per output frame f and window slot s, writes the numerator plane (slot 2s) and
// the denominator plane (slot 2s+1, the B x B box sum of the per-origin weights) into the
// stacked float frame (height H * slots * 2).
struct VStackArgs {
    const float *num[3];
    const float *wmap[3];
    long long slot_stride;     // elements between accumulator slots
    int ld, H, W, B, slots;
    int process[3];
    const PlanePtr *out;       // [f * 3 + p]
};

}  // namespace bm3d
