// ref_block_shim.cpp -- builds the reference plugin's own include/Block.h (unmodified, read in
// place from the reference checkout) into oracle/_ref/librefblock.so so that the oracle's block
// matching, search-window generation, group gather and scatter can be pinned to the reference's
// code bit for bit.  TEST INFRASTRUCTURE ONLY (see oracle/Makefile).
//
// Block.h includes "Helper.h", which needs the VapourSynth SDK (absent here).  Pre-defining its
// include guard and supplying the four helpers Block.h uses (AlignedMalloc, AlignedFree, Min,
// Max -- include/Helper.h:138-153, :383-393) is the whole shim.  Type.h (Pos, Pos3, KeyPair,
// TypeMax) is included from the reference unchanged.  Compiled for plain x86-64, so Block.h
// takes its __SSE2__ path exactly as the shipped x86 plugin does.

#include <cassert>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <type_traits>
#include <utility>
#include <vector>
#include <algorithm>
#include <emmintrin.h>

#include "Type.h"

#define HELPER_H_

template <typename T>
void AlignedMalloc(T *&mem, size_t count, size_t alignment = 64)
{
    size_t bytes = (sizeof(T) * count + alignment - 1) / alignment * alignment;
    mem = static_cast<T *>(std::aligned_alloc(alignment, bytes ? bytes : alignment));
}

template <typename T>
void AlignedFree(T *&mem)
{
    std::free(mem);
    mem = nullptr;
}

template <typename T> T Min(const T &a, const T &b) { return b < a ? b : a; }
template <typename T> T Max(const T &a, const T &b) { return b > a ? b : a; }

#include "Block.h"

typedef Block<FLType, FLType> block_type;
typedef BlockGroup<FLType, FLType> group_type;

static int emit(const block_type::PosPairCode &code, float *keys, int *ys, int *xs, int cap)
{
    int n = (int)code.size();
    for (int k = 0; k < n && k < cap; ++k) {
        keys[k] = code[k].first;
        ys[k] = code[k].second.y;
        xs[k] = code[k].second.x;
    }
    return n;
}

extern "C" {

// Block::BlockMatchingMulti, range form, excludeCurPos = 1, sorted (include/Block.h:683-729),
// exactly as BM3D_Process_Base::BlockMatching calls it (source/BM3D_Base.cpp:480-489).
int ref_bm_range(const float *plane, int H, int W, int stride, int j, int i, int B, int range,
                 int step, double thMSE, int match_size, float *keys, int *ys, int *xs, int cap)
{
    block_type blk(plane, stride, B, B, Pos(j, i));
    auto code = blk.BlockMatchingMulti(plane, H, W, stride, FLType(1), range, step, thMSE, 1,
                                       (size_t)match_size, true);
    return emit(code, keys, ys, xs, cap);
}

// Search-position form (include/Block.h:655-677); the reference block is taken from refplane at
// (j, i), the candidates from srcplane.
int ref_bm_positions(const float *refplane, int stride, int j, int i, int B, const float *srcplane,
                     const int *py, const int *px, int npos, double thMSE, int match_size,
                     float *keys, int *ys, int *xs, int cap)
{
    block_type blk(refplane, stride, B, B, Pos(j, i));
    block_type::PosCode sp;
    for (int k = 0; k < npos; ++k) sp.push_back(Pos(py[k], px[k]));
    auto code = blk.BlockMatchingMulti(srcplane, stride, FLType(1), sp, thMSE, (size_t)match_size, true);
    return emit(code, keys, ys, xs, cap);
}

// Block::GenSearchPos (include/Block.h:813-827)
int ref_gen_search_pos(const int *cy, const int *cx, int ncenters, int H, int W, int B, int range,
                       int step, int *oy, int *ox, int cap)
{
    block_type blk(B, B, Pos(0, 0), true, 0);
    block_type::PosCode centers;
    for (int k = 0; k < ncenters; ++k) centers.push_back(Pos(cy[k], cx[k]));
    auto sp = blk.GenSearchPos(centers, H, W, range, step);
    int n = (int)sp.size();
    for (int k = 0; k < n && k < cap; ++k) { oy[k] = sp[k].y; ox[k] = sp[k].x; }
    return n;
}

// V-BM3D grouping for one reference block: the reference's VBM3D_Process_Base::BlockMatching
// (source/VBM3D_Base.cpp:540-659) restated line by line on top of the reference's own Block.h
// primitives and Pos3/KeyPair types.  refs[f] = frame f of the window, cur = current frame index.
int ref_vbm3d_match(const float *const *refs, int frames, int cur, int H, int W, int stride,
                    int j, int i, int B, int bm_range, int bm_step, int G, int ps_num,
                    int ps_range, int ps_step, double thMSE, float *keys, int *zs, int *ys,
                    int *xs, int cap)
{
    typedef group_type::Pos3Pair Pos3Pair;
    typedef group_type::Pos3PairCode Pos3PairCode;
    Pos3PairCode matchCode;
    if (G == 1 || thMSE <= 0) {
        matchCode.push_back(Pos3Pair(0.0f, Pos3(cur, j, i)));
    } else {
        block_type refBlock(refs[cur], stride, B, B, Pos(j, i));
        block_type::PosPairCode frameMatch;
        block_type::PosCode prePosCode;
        int f = cur;
        frameMatch = refBlock.BlockMatchingMulti(refs[f], H, W, stride, FLType(1), bm_range, bm_step,
                                                 thMSE, 1, (size_t)G, true);
        for (auto &x : frameMatch) matchCode.push_back(Pos3Pair(x.first, Pos3(x.second, f)));
        int nextPosNum = Min(ps_num, (int)frameMatch.size());
        block_type::PosCode curPosCode;
        for (int k = 0; k < nextPosNum; ++k) curPosCode.push_back(frameMatch[k].second);
        block_type::PosCode curSearchPos = refBlock.GenSearchPos(curPosCode, H, W, ps_range, ps_step);
        for (int dir = -1; dir <= 1; dir += 2) {
            for (f = cur + dir; f >= 0 && f < frames; f += dir) {
                if (f == cur + dir) {
                    frameMatch = refBlock.BlockMatchingMulti(refs[f], stride, FLType(1), curSearchPos,
                                                             thMSE, (size_t)G, true);
                } else {
                    int nn = Min(ps_num, (int)frameMatch.size());
                    prePosCode.resize(nn);
                    for (int k = 0; k < nn; ++k) prePosCode[k] = frameMatch[k].second;
                    block_type::PosCode searchPos = refBlock.GenSearchPos(prePosCode, H, W, ps_range, ps_step);
                    frameMatch = refBlock.BlockMatchingMulti(refs[f], stride, FLType(1), searchPos,
                                                             thMSE, (size_t)G, true);
                }
                for (auto &x : frameMatch) matchCode.push_back(Pos3Pair(x.first, Pos3(x.second, f)));
            }
        }
        if (G > 0 && (int)matchCode.size() > G) {
            std::partial_sort(matchCode.begin() + 1, matchCode.begin() + G, matchCode.end());
            matchCode.resize(G);
        }
    }
    int n = (int)matchCode.size();
    for (int k = 0; k < n && k < cap; ++k) {
        keys[k] = matchCode[k].first;
        zs[k] = matchCode[k].second.z;
        ys[k] = matchCode[k].second.y;
        xs[k] = matchCode[k].second.x;
    }
    return n;
}

// BlockGroup gather (include/Block.h:1126-1146) of n blocks at (ys, xs) into out[n][B][B]
void ref_group_gather(const float *plane, int stride, const int *ys, const int *xs, int n, int B, float *out)
{
    block_type::PosPairCode code;
    for (int k = 0; k < n; ++k) code.push_back(block_type::PosPair(0.0f, Pos(ys[k], xs[k])));
    group_type g(plane, stride, code, n, B, B);
    std::memcpy(out, g.data(), sizeof(float) * n * B * B);
}

// BlockGroup::AddTo(dst, stride, gain) and CountTo(dst, stride, value)
// (include/Block.h:1239-1259, 1326-1345)
void ref_group_scatter(const float *data, const int *ys, const int *xs, int n, int B, float gain,
                       float value, float *num, float *den, int stride)
{
    block_type::PosPairCode code;
    for (int k = 0; k < n; ++k) code.push_back(block_type::PosPair(0.0f, Pos(ys[k], xs[k])));
    group_type g(num, stride, code, n, B, B);    // gathers (overwritten below)
    std::memcpy(g.data(), data, sizeof(float) * n * B * B);
    g.AddTo(num, stride, gain);
    g.CountTo(den, stride, value);
}

}  // extern "C"
