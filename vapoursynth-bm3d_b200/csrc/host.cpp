// host.cpp -- host side of the library: the reference plugin's argument processing and filter
// objects restated in C++ over the sm_100a kernels, and the C ABI of include/bm3d_b200.h.
//
// Per output batch the flow is: stage frames (host -> device when needed), convert them into a
// float workspace (K5), block matching (K1, and K2 for V-BM3D), collaborative filtering with
// aggregation (K3+K4), normalisation / stacking (K5), conversion back to the output format and,
// for host frames, device -> host copies.  Everything between the conversions stays on the GPU.

#include "bm3d_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "launch.h"
#include "proposal_weights.h"
#include "params.h"

namespace bm3d {

// ---------------------------------------------------------------------------------------------
// errors and logging

static thread_local std::string g_error;
static std::mutex g_log_mutex;
static bm3d_log_fn g_log_fn = nullptr;
static void *g_log_user = nullptr;

static int fail(int code, const std::string &msg)
{
    g_error = msg;
    return code;
}

// Error text for the entry points defined in other translation units.
int set_error(int code, const std::string &msg) { return fail(code, msg); }
void clear_error() { g_error.clear(); }

static void log_warning(const std::string &msg)
{
    std::lock_guard<std::mutex> lk(g_log_mutex);
    if (g_log_fn) g_log_fn(2, msg.c_str(), g_log_user);
    else std::fprintf(stderr, "%s\n", msg.c_str());
}

struct CudaError {
    cudaError_t e;
    const char *what;
};

#define CU(expr)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess) throw CudaError{e_, #expr};                                \
    } while (0)

// ---------------------------------------------------------------------------------------------
// argument map (VSMap analogue)

struct MapValue {
    int kind;   // 0 int, 1 float, 2 data, 3 clip
    int64_t i = 0;
    double f = 0.0;
    std::string s;
    bm3d_video_info clip{};
};

}  // namespace bm3d

struct bm3d_map {
    std::map<std::string, std::vector<bm3d::MapValue>> e;
};

namespace bm3d {

// mapNumElements: -1 when the key is absent
static int map_num(const bm3d_map *m, const char *key)
{
    auto it = m->e.find(key);
    return it == m->e.end() ? -1 : (int)it->second.size();
}

// mapGetIntSaturated (saturates to int)
static int map_get_int(const bm3d_map *m, const char *key, int idx, int *err)
{
    auto it = m->e.find(key);
    if (it == m->e.end() || idx >= (int)it->second.size() || it->second[idx].kind != 0) {
        *err = 1;
        return 0;
    }
    *err = 0;
    const int64_t v = it->second[idx].i;
    return v > INT32_MAX ? INT32_MAX : v < INT32_MIN ? INT32_MIN : (int)v;
}

// mapGetInt (int64)
static int64_t map_get_int64(const bm3d_map *m, const char *key, int idx, int *err)
{
    auto it = m->e.find(key);
    if (it == m->e.end() || idx >= (int)it->second.size() || it->second[idx].kind != 0) {
        *err = 1;
        return 0;
    }
    *err = 0;
    return it->second[idx].i;
}

// mapGetFloat (integers convert, as VapourSynth converts int arguments of float parameters)
static double map_get_float(const bm3d_map *m, const char *key, int idx, int *err)
{
    auto it = m->e.find(key);
    if (it == m->e.end() || idx >= (int)it->second.size()) { *err = 1; return 0.0; }
    const MapValue &v = it->second[idx];
    if (v.kind == 1) { *err = 0; return v.f; }
    if (v.kind == 0) { *err = 0; return (double)v.i; }
    *err = 1;
    return 0.0;
}

static const char *map_get_data(const bm3d_map *m, const char *key, int idx, int *err)
{
    auto it = m->e.find(key);
    if (it == m->e.end() || idx >= (int)it->second.size() || it->second[idx].kind != 2) { *err = 1; return nullptr; }
    *err = 0;
    return it->second[idx].s.c_str();
}

static bool map_get_clip(const bm3d_map *m, const char *key, bm3d_video_info *out)
{
    auto it = m->e.find(key);
    if (it == m->e.end() || it->second.empty() || it->second[0].kind != 3) return false;
    *out = it->second[0].clip;
    return true;
}

// Argument specs registered by VapourSynthPluginInit2 (source/VSPlugin.cpp:430-517).  The
// VapourSynth core checks names, types and required arguments before the plugin sees them; the
// same check is done here so that malformed maps are rejected before arguments_process.
struct ArgSpec {
    const char *name;
    int kind;        // 0 int, 1 float, 2 data, 3 clip
    bool array;
    bool optional;
};

static const std::vector<ArgSpec> &argspec(const std::string &fn)
{
    static const std::vector<ArgSpec> conv = {{"input", 3, false, false}, {"sample", 0, false, true}};
    static const std::vector<ArgSpec> basic = {
        {"input", 3, false, false}, {"ref", 3, false, true}, {"profile", 2, false, true},
        {"sigma", 1, true, true}, {"block_size", 0, false, true}, {"block_step", 0, false, true},
        {"group_size", 0, false, true}, {"bm_range", 0, false, true}, {"bm_step", 0, false, true},
        {"th_mse", 1, false, true}, {"hard_thr", 1, false, true}, {"matrix", 0, false, true}, {"precision", 2, false, true}};
    static const std::vector<ArgSpec> fin = {
        {"input", 3, false, false}, {"ref", 3, false, false}, {"profile", 2, false, true},
        {"sigma", 1, true, true}, {"block_size", 0, false, true}, {"block_step", 0, false, true},
        {"group_size", 0, false, true}, {"bm_range", 0, false, true}, {"bm_step", 0, false, true},
        {"th_mse", 1, false, true}, {"matrix", 0, false, true}, {"precision", 2, false, true}};
    static const std::vector<ArgSpec> vbasic = {
        {"input", 3, false, false}, {"ref", 3, false, true}, {"profile", 2, false, true},
        {"sigma", 1, true, true}, {"radius", 0, false, true}, {"block_size", 0, false, true},
        {"block_step", 0, false, true}, {"group_size", 0, false, true}, {"bm_range", 0, false, true},
        {"bm_step", 0, false, true}, {"ps_num", 0, false, true}, {"ps_range", 0, false, true},
        {"ps_step", 0, false, true}, {"th_mse", 1, false, true}, {"hard_thr", 1, false, true},
        {"matrix", 0, false, true}, {"precision", 2, false, true}, {"aggregate", 0, false, true},
        {"sample", 0, false, true}};
    static const std::vector<ArgSpec> vfinal = {
        {"input", 3, false, false}, {"ref", 3, false, false}, {"profile", 2, false, true},
        {"sigma", 1, true, true}, {"radius", 0, false, true}, {"block_size", 0, false, true},
        {"block_step", 0, false, true}, {"group_size", 0, false, true}, {"bm_range", 0, false, true},
        {"bm_step", 0, false, true}, {"ps_num", 0, false, true}, {"ps_range", 0, false, true},
        {"ps_step", 0, false, true}, {"th_mse", 1, false, true}, {"matrix", 0, false, true}, {"precision", 2, false, true},
        {"aggregate", 0, false, true}, {"sample", 0, false, true}};
    static const std::vector<ArgSpec> vagg = {
        {"input", 3, false, false}, {"radius", 0, false, true}, {"sample", 0, false, true}};
    static const std::vector<ArgSpec> none;
    if (fn == "RGB2OPP" || fn == "OPP2RGB") return conv;
    if (fn == "Basic") return basic;
    if (fn == "Final") return fin;
    if (fn == "VBasic") return vbasic;
    if (fn == "VFinal") return vfinal;
    if (fn == "VAggregate") return vagg;
    return none;
}

static int check_argspec(const std::string &fn, const bm3d_map *m)
{
    const auto &spec = argspec(fn);
    for (const auto &kv : m->e) {
        const ArgSpec *s = nullptr;
        for (const auto &a : spec)
            if (kv.first == a.name) s = &a;
        if (!s) return fail(BM3D_ERR_ARG, fn + ": Function does not take argument(s) named " + kv.first);
        for (const auto &v : kv.second) {
            const bool ok = v.kind == s->kind || (s->kind == 1 && v.kind == 0);
            if (!ok) return fail(BM3D_ERR_ARG, fn + ": Argument " + kv.first + " has the wrong type");
        }
        if (!s->array && kv.second.size() > 1)
            return fail(BM3D_ERR_ARG, fn + ": Argument " + kv.first + " is not an array");
    }
    for (const auto &a : spec)
        if (!a.optional && map_num(m, a.name) < 1)
            return fail(BM3D_ERR_ARG, fn + ": Argument " + std::string(a.name) + " is required");
    return BM3D_OK;
}

// ---------------------------------------------------------------------------------------------
// device memory helpers

struct DevBuf {
    void *p = nullptr;
    size_t n = 0;
    ~DevBuf() { if (p) cudaFree(p); }
    void *get(size_t bytes)
    {
        if (bytes > n) {
            if (p) CU(cudaFree(p));
            p = nullptr;
            n = 0;
            CU(cudaMalloc(&p, bytes));
            n = bytes;
        }
        return p;
    }
    template <typename T> T *as() const { return static_cast<T *>(p); }
};

// Per-device constant data (DCT odd tables).
struct DeviceTables {
    bool ready = false;
    float *odd_all = nullptr;
};
static std::mutex g_dev_mutex;
static std::map<int, DeviceTables> g_dev;

static std::vector<float> host_odd_tables()
{
    std::vector<float> t(21845, 0.0f);
    for (int N = 2; N <= 256; N *= 2) {
        const int h = N / 2;
        int off = N == 2 ? 0 : N == 4 ? 1 : N == 8 ? 5 : N == 16 ? 21 : N == 32 ? 85 : N == 64 ? 341 : N == 128 ? 1365 : 5461;
        for (int m = 0; m < h; ++m)
            for (int j = 0; j < h; ++j) t[off + m * h + j] = cos2((long)(2 * j + 1) * (2 * m + 1), 2L * N);
    }
    return t;
}

static const DeviceTables &device_tables()
{
    int dev = 0;
    CU(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_dev_mutex);
    DeviceTables &t = g_dev[dev];
    if (!t.ready) {
        const std::vector<float> odd = host_odd_tables();
        CU(upload_odd_tables(odd.data()));
        CU(cudaMalloc(&t.odd_all, sizeof(float) * odd.size()));
        CU(cudaMemcpy(t.odd_all, odd.data(), sizeof(float) * odd.size(), cudaMemcpyHostToDevice));
        t.ready = true;
    }
    return t;
}

// Direct (non-power-of-two) DCT tables for the lengths a filter can meet: fwd then inv per N.
struct DirectTables {
    DevBuf tab, off;
};

static void build_direct_tables(DirectTables &d, const std::vector<int> &lengths)
{
    std::vector<int> off(257, -1);
    std::vector<float> data;
    for (int N : lengths) {
        if (N < 1 || N > 256 || (N & (N - 1)) == 0 || off[N] >= 0) continue;
        off[N] = (int)data.size();
        for (int k = 0; k < N; ++k)
            for (int j = 0; j < N; ++j) data.push_back(cos2((long)(2 * j + 1) * k, 2L * N));
        for (int k = 0; k < N; ++k)
            for (int j = 0; j < N; ++j) data.push_back(cos2((long)j * (2 * k + 1), 2L * N));
    }
    if (data.empty()) data.push_back(0.0f);
    CU(cudaMemcpy(d.tab.get(sizeof(float) * data.size()), data.data(), sizeof(float) * data.size(), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(d.off.get(sizeof(int) * off.size()), off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice));
}

// ---------------------------------------------------------------------------------------------
// conversion programs (include/Conversion.hpp, include/Helper.h:285-351)

static int sample_kind(const bm3d_video_info &vi)
{
    if (vi.sample_type == BM3D_FLOAT) return SK_F32;
    return vi.bits_per_sample <= 8 ? SK_U8 : SK_U16;
}

static int bytes_per_sample(const bm3d_video_info &vi)
{
    return vi.sample_type == BM3D_FLOAT ? 4 : (vi.bits_per_sample <= 8 ? 1 : 2);
}

// GetQuanPara for integers
static void quan_int(int bps, bool full, bool chroma, int &fl, int &ne, int &ce)
{
    if (full) { fl = 0; ne = chroma ? (1 << (bps - 1)) : fl; ce = (1 << bps) - 1; }
    else { fl = 16 << (bps - 8); ne = chroma ? (1 << (bps - 1)) : fl; ce = chroma ? 240 << (bps - 8) : 235 << (bps - 8); }
}

static ConvProgram raw_program(int kind, int nplanes, int W, int H)
{
    ConvProgram p{};
    p.raw = 1;
    p.in_kind = p.out_kind = kind;
    p.nin = p.nout = nplanes;
    p.W = W;
    p.H = H;
    return p;
}

// Int2Float for one plane (RangeConvert: integer -> float, clip only for PC-range chroma)
static LinearOp int2float_op(int bps, bool full, bool chroma)
{
    int sf, sn, sc;
    quan_int(bps, full, chroma, sf, sn, sc);
    const float df = chroma ? -0.5f : 0.0f, dn = 0.0f, dc = chroma ? 0.5f : 1.0f;
    const float drange = dc - df;
    const int srange = sc - sf;
    LinearOp o{};
    o.gain = drange / srange;
    o.offset = -static_cast<float>(sn) * o.gain + dn;
    o.clip = (sf < sn && (sf + sc) % 2 == 1) ? 1 : 0;
    o.lo = df;
    o.hi = dc;
    return o;
}

// Float2Int for one plane (RangeConvert: float -> integer, clipped, rounding offset)
static LinearOp float2int_op(int bps, bool full, bool chroma)
{
    int df, dn, dc;
    quan_int(bps, full, chroma, df, dn, dc);
    const float sf = chroma ? -0.5f : 0.0f, sn = 0.0f, sc = chroma ? 0.5f : 1.0f;
    const int drange = dc - df;
    const float srange = sc - sf;
    const bool pc = df < dn && (df + dc) % 2 == 1;
    LinearOp o{};
    o.gain = static_cast<float>(drange) / srange;
    o.offset = -sn * o.gain + dn;
    o.offset += static_cast<float>(pc ? 0.499999 : 0.5);
    o.clip = 1;
    o.lo = (float)df;
    o.hi = (float)dc;
    return o;
}

// MatrixConvert_RGB2YUV, OPP branch (Conversion.hpp:205-236), full range both sides.
// in: 8-16 bit integer or float; out: 16-bit integer (out_float = false) or float.
static ConvProgram rgb2opp_program(int in_kind, int in_bits, int out_kind, int out_bits, int W, int H,
                                   bool y_only)
{
    ConvProgram p{};
    p.mode = y_only ? 2 : 1;
    p.in_kind = in_kind;
    p.out_kind = out_kind;
    p.nin = 3;
    p.nout = y_only ? 1 : 3;
    p.W = W;
    p.H = H;
    const bool dst_float = out_kind == SK_F32;
    const bool src_float = in_kind == SK_F32;
    float dFloorY, dCeilY, dFloorC, dNeutralC, dCeilC;
    if (dst_float) { dFloorY = 0; dCeilY = 1; dFloorC = -0.5f; dNeutralC = 0; dCeilC = 0.5f; }
    else {
        int fl, ne, ce;
        quan_int(out_bits, true, false, fl, ne, ce);
        dFloorY = (float)fl; dCeilY = (float)ce;
        quan_int(out_bits, true, true, fl, ne, ce);
        dFloorC = (float)fl; dNeutralC = (float)ne; dCeilC = (float)ce;
    }
    float sRange, sFloor;
    if (src_float) { sFloor = 0.0f; sRange = 1.0f - 0.0f; }
    else { sFloor = 0.0f; sRange = (float)((1 << in_bits) - 1 - 0); }
    // integer destinations: dRange is an int difference converted to float
    const float dRangeY = dCeilY - dFloorY;
    const float dRangeC = dCeilC - dFloorC;
    const bool dst_pc_chroma = !dst_float && dFloorC < dNeutralC && ((int)(dFloorC + dCeilC)) % 2 == 1;
    const float gainY = dRangeY / (sRange * 3.0f);
    float offsetY = -sFloor * 3.0f * gainY + dFloorY;
    if (!dst_float) offsetY += 0.5f;
    const float gainU = dRangeC / (sRange * 2.0f);
    const float gainV = dRangeC / (sRange * 4.0f);
    float offsetC = dNeutralC;
    if (!dst_float) offsetC += static_cast<float>(dst_pc_chroma ? 0.499999 : 0.5);
    const int clip = dst_float ? 0 : 1;
    p.op[0] = LinearOp{gainY, offsetY, dFloorY, dCeilY, clip};
    p.op[1] = LinearOp{gainU, offsetC, dFloorC, dCeilC, clip};
    p.op[2] = LinearOp{gainV, offsetC, dFloorC, dCeilC, clip};
    return p;
}

// ConvertToY, OPP branch (Conversion.hpp:103-116) into float, full range, no clip
static ConvProgram rgb2y_program(int in_kind, int in_bits, int W, int H)
{
    ConvProgram p = rgb2opp_program(in_kind, in_bits, SK_F32, 32, W, H, true);
    return p;
}

// MatrixConvert_YUV2RGB, OPP branch (Conversion.hpp:290-417, Specification.h:253-269)
static ConvProgram opp2rgb_program(int in_kind, int in_bits, int out_kind, int out_bits, int W, int H)
{
    ConvProgram p{};
    p.mode = 3;
    p.in_kind = in_kind;
    p.out_kind = out_kind;
    p.nin = 3;
    p.nout = 3;
    p.W = W;
    p.H = H;
    const bool dst_float = out_kind == SK_F32;
    const bool src_float = in_kind == SK_F32;
    float dFloor, dCeil;
    if (dst_float) { dFloor = 0.0f; dCeil = 1.0f; }
    else { dFloor = 0.0f; dCeil = (float)((1 << out_bits) - 1); }
    float sFloorY, sCeilY, sFloorC, sNeutralC, sCeilC;
    if (src_float) { sFloorY = 0; sCeilY = 1; sFloorC = -0.5f; sNeutralC = 0; sCeilC = 0.5f; }
    else {
        int fl, ne, ce;
        quan_int(in_bits, true, false, fl, ne, ce);
        sFloorY = (float)fl; sCeilY = (float)ce;
        quan_int(in_bits, true, true, fl, ne, ce);
        sFloorC = (float)fl; sNeutralC = (float)ne; sCeilC = (float)ce;
    }
    const float dRange = dCeil - dFloor;
    const float gainY = dRange / (sCeilY - sFloorY);
    const float gainC = dRange / (sCeilC - sFloorC);
    float Ry = (float)1.0L, Ru = (float)1.0L, Rv = (float)(2.0L / 3.0L);
    float Gy = (float)1.0L, Gu = (float)0.0L, Gv = (float)(-4.0L / 3.0L);
    float By = (float)1.0L, Bu = (float)-1.0L, Bv = (float)(2.0L / 3.0L);
    Ry *= gainY; Ru *= gainC; Rv *= gainC;
    Gy *= gainY; Gu *= gainC; Gv *= gainC;
    By *= gainY; Bu *= gainC; Bv *= gainC;
    float oR = -sFloorY * Ry - sNeutralC * (Ru + Rv) + dFloor;
    float oG = -sFloorY * Gy - sNeutralC * (Gu + Gv) + dFloor;
    float oB = -sFloorY * By - sNeutralC * (Bu + Bv) + dFloor;
    if (!dst_float) { oR += 0.5f; oG += 0.5f; oB += 0.5f; }
    const float k[9] = {Ry, Ru, Rv, Gy, Gu, Gv, By, Bu, Bv};
    for (int i = 0; i < 9; ++i) p.coef[i] = k[i];
    p.off[0] = oR; p.off[1] = oG; p.off[2] = oB;
    p.op[0] = LinearOp{1.0f, 0.0f, dFloor, dCeil, dst_float ? 0 : 1};
    return p;
}

// ---------------------------------------------------------------------------------------------
// frames: staging host planes on the device

struct PlaneGeom {
    int width_bytes;
    int height;
};

class Stager {
public:
    // Device views of frame planes; host planes are copied into staging buffers that are kept
    // between calls (no allocation once the pool has grown to the batch's needs).
    PlanePtr view(const bm3d_frame &fr, int p, const PlaneGeom &g, cudaStream_t s)
    {
        if (fr.memory == BM3D_MEM_DEVICE) return PlanePtr{fr.data[p], fr.stride[p]};
        const size_t pitch = ((size_t)g.width_bytes + 255) / 256 * 256;
        void *d = next(pitch * g.height);
        CU(cudaMemcpy2DAsync(d, pitch, fr.data[p], fr.stride[p], g.width_bytes, g.height, cudaMemcpyHostToDevice, s));
        return PlanePtr{d, (long long)pitch};
    }
    // Device target for an output plane; host targets get a staging buffer copied back by flush().
    PlanePtr target(const bm3d_frame &fr, int p, const PlaneGeom &g)
    {
        if (fr.memory == BM3D_MEM_DEVICE) return PlanePtr{fr.data[p], fr.stride[p]};
        const size_t pitch = ((size_t)g.width_bytes + 255) / 256 * 256;
        void *d = next(pitch * g.height);
        pending_.push_back(Pending{fr.data[p], fr.stride[p], d, pitch, g});
        return PlanePtr{d, (long long)pitch};
    }
    void flush(cudaStream_t s)
    {
        for (const Pending &q : pending_)
            CU(cudaMemcpy2DAsync(q.host, q.host_stride, q.dev, q.pitch, q.g.width_bytes, q.g.height, cudaMemcpyDeviceToHost, s));
        pending_.clear();
    }
    // Called once the stream has drained: the buffers may be reused by the next call.
    void release()
    {
        used_ = 0;
        pending_.clear();
    }

private:
    void *next(size_t bytes)
    {
        if (used_ == bufs_.size()) bufs_.emplace_back(new DevBuf());
        return bufs_[used_++]->get(bytes);
    }
    struct Pending {
        void *host;
        int64_t host_stride;
        void *dev;
        size_t pitch;
        PlaneGeom g;
    };
    std::vector<std::unique_ptr<DevBuf>> bufs_;
    size_t used_ = 0;
    std::vector<Pending> pending_;
};

static bool frame_ok(const bm3d_frame *f, int planes)
{
    if (!f) return false;
    for (int p = 0; p < planes; ++p)
        if (!f->data[p]) return false;
    return f->memory == BM3D_MEM_HOST || f->memory == BM3D_MEM_DEVICE;
}

static bool all_device(int n, const bm3d_frame *const *fr)
{
    for (int i = 0; i < n; ++i)
        if (fr[i] && fr[i]->memory != BM3D_MEM_DEVICE) return false;
    return true;
}

// ---------------------------------------------------------------------------------------------
// filter base

class Filter {
public:
    std::string fn;
    bm3d_video_info vi{}, rvi{}, ovi{};
    bool rdef = false;
    cudaStream_t stream = nullptr;
    cudaStream_t own = nullptr;
    unsigned long long *stats = nullptr;      // [0] exact-heap selections, [1] precision-form matching
                                              // fallbacks, [2] precision-form tensor-core time-outs
    unsigned long long last_slow = 0;
    unsigned long long last_stats[3] = {0, 0, 0};
    // stage timing (CUDA events on the filter's stream): 0 ingest, 1 block matching,
    // 2 predictive search, 3 collaborative filter + aggregation, 4 normalise / stack, 5 egress
    static constexpr int kStages = 6;
    bool profiling = false;
    bool prof_valid = false;
    cudaEvent_t ev[kStages + 1] = {};

    virtual ~Filter()
    {
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
        if (stats) cudaFree(stats);
        if (own) cudaStreamDestroy(own);
    }
    void set_profiling(bool on)
    {
        if (on && !ev[0])
            for (auto &e : ev) CU(cudaEventCreate(&e));
        profiling = on;
        prof_valid = false;
    }
    void mark(int i)
    {
        if (profiling) {
            CU(cudaEventRecord(ev[i], stream));
            if (i == kStages) prof_valid = true;
        }
    }
    std::string err(const std::string &m) const { return "bm3d." + fn + ": " + m; }
    virtual void window(int n, int count, int *first, int *num) const
    {
        *first = n;
        *num = count;
    }
    virtual int run(int n, int count, const bm3d_frame *const *src, const bm3d_frame *const *ref,
                    bm3d_frame *const *dst, bool sync) = 0;
    virtual int matches(int, int *, int *, int *, int *, float *, int) { return -1; }
    virtual int reference_fp64(int, double *, long long) { return -1; }
    virtual int retained(int, int *, int) { return -1; }
    // called after the filter's stream was synchronised (device-side error flags)
    virtual void synced() {}
    // the stats counters after the stream was synchronised
    void read_stats()
    {
        CU(cudaMemcpy(last_stats, stats, sizeof(last_stats), cudaMemcpyDeviceToHost));
        last_slow = last_stats[0];
    }
    int nplanes() const { return vi.color_family == BM3D_GRAY ? 1 : 3; }
    void init_stream()
    {
        CU(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
        stream = own;
        CU(cudaMalloc(&stats, 3 * sizeof(unsigned long long)));
    }

protected:
    Stager stager_;
    DevBuf ptr_in_, ptr_out_;
    // uploads a PlanePtr table to the device (small)
    PlanePtr *upload_ptrs(DevBuf &buf, const std::vector<PlanePtr> &v)
    {
        PlanePtr *d = static_cast<PlanePtr *>(buf.get(sizeof(PlanePtr) * std::max<size_t>(v.size(), 1)));
        CU(cudaMemcpyAsync(d, v.data(), sizeof(PlanePtr) * v.size(), cudaMemcpyHostToDevice, stream));
        return d;
    }
};

static bool valid_clip(const bm3d_video_info &vi)
{
    // vsh::isConstantVideoFormat: known format, non-zero dimensions
    return vi.width > 0 && vi.height > 0 && vi.color_family >= BM3D_GRAY && vi.color_family <= BM3D_YUV &&
           (vi.sample_type == BM3D_INTEGER || vi.sample_type == BM3D_FLOAT) && vi.bits_per_sample > 0;
}

static bool same_format(const bm3d_video_info &a, const bm3d_video_info &b)
{
    return a.color_family == b.color_family && a.sample_type == b.sample_type &&
           a.bits_per_sample == b.bits_per_sample && a.subsampling_w == b.subsampling_w &&
           a.subsampling_h == b.subsampling_h;
}

static void copy_props(const bm3d_frame *src, bm3d_frame *dst)
{
    dst->prop_bm3d_opp = src->prop_bm3d_opp;
    dst->prop_range = src->prop_range;
    dst->prop_matrix = src->prop_matrix;
    dst->prop_v_radius = src->prop_v_radius;
    dst->prop_v_process_count = src->prop_v_process_count;
    for (int i = 0; i < 3; ++i) dst->prop_v_process[i] = src->prop_v_process[i];
}

// ---------------------------------------------------------------------------------------------
// RGB2OPP / OPP2RGB (include/RGB2OPP.h, include/OPP2RGB.h)

class ConvFilter : public Filter {
public:
    bool to_opp = true;
    int sample = 0;

    int create(const bm3d_map *in)
    {
        int error;
        if (!map_get_clip(in, "input", &vi) || !valid_clip(vi))
            return fail(BM3D_ERR_ARG, err("Invalid input clip, only constant format input supported"));
        if ((vi.sample_type == BM3D_INTEGER && vi.bits_per_sample > 16) ||
            (vi.sample_type == BM3D_FLOAT && vi.bits_per_sample != 32))
            return fail(BM3D_ERR_ARG, err("Invalid input clip, only 8-16 bit int or 32 bit float formats supported"));
        if (to_opp && vi.color_family != BM3D_RGB)
            return fail(BM3D_ERR_ARG, err("Invalid input clip, must be of RGB color family"));
        if (!to_opp && vi.color_family != BM3D_YUV)
            return fail(BM3D_ERR_ARG, err("Invalid input clip, must be of YUV color family"));
        int64_t s = map_get_int64(in, "sample", 0, &error);
        if (error) s = 0;
        else if (s != 0 && s != 1)
            return fail(BM3D_ERR_ARG, err("Invalid 'sample' assigned, must be 0 (integer sample type) or 1 (float sample type)"));
        sample = (int)s;
        ovi = vi;
        ovi.color_family = to_opp ? BM3D_YUV : BM3D_RGB;
        ovi.sample_type = sample;
        ovi.bits_per_sample = sample == 1 ? 32 : 16;
        ovi.subsampling_w = ovi.subsampling_h = 0;
        init_stream();
        return BM3D_OK;
    }

    int run(int n, int count, const bm3d_frame *const *src, const bm3d_frame *const *, bm3d_frame *const *dst,
            bool sync) override
    {
        const int W = vi.width, H = vi.height;
        const PlaneGeom gi{W * bytes_per_sample(vi), H};
        const PlaneGeom go{W * bytes_per_sample(ovi), H};
        std::vector<PlanePtr> in, out;
        for (int k = 0; k < count; ++k) {
            if (!frame_ok(src[k], 3) || !frame_ok(dst[k], 3)) return fail(BM3D_ERR_STATE, err("missing frame planes"));
            for (int p = 0; p < 3; ++p) in.push_back(stager_.view(*src[k], p, gi, stream));
            for (int p = 0; p < 3; ++p) out.push_back(stager_.target(*dst[k], p, go));
        }
        const ConvProgram pr = to_opp
            ? rgb2opp_program(sample_kind(vi), vi.bits_per_sample, sample_kind(ovi), ovi.bits_per_sample, W, H, false)
            : opp2rgb_program(sample_kind(vi), vi.bits_per_sample, sample_kind(ovi), ovi.bits_per_sample, W, H);
        CU(launch_convert(pr, upload_ptrs(ptr_in_, in), upload_ptrs(ptr_out_, out), count, stream));
        stager_.flush(stream);
        for (int k = 0; k < count; ++k) {
            copy_props(src[k], dst[k]);
            if (to_opp) { dst[k]->prop_matrix = 2; dst[k]->prop_bm3d_opp = 1; }
            else { dst[k]->prop_matrix = 0; dst[k]->prop_bm3d_opp = -1; }
        }
        if (sync) CU(cudaStreamSynchronize(stream));
        if (sync) stager_.release();
        (void)n;
        return BM3D_OK;
    }
};

// ---------------------------------------------------------------------------------------------
// Learned block-matching proposal: device buffers and the descriptor pass

// Precision form, hard threshold: coefficients whose tensor-core value lies within this fraction
// of their threshold are recomputed from the pixels in double precision before the keep / zero
// decision.  The tf32 products of mean-free blocks stay inside it: with this band the decisions
// left differing from the plain path's are the plain FP32 transform's own flips against exact
// arithmetic (the test suite sweeps the band and counts them against the oracle's).
constexpr float kRecheckBand = 1.0f / 64.0f;

// proposals per reference block that the learned form re-ranks exactly (of about 1,089 at range 16)
constexpr int kLearnedProposals = 96;
// V-BM3D: proposals per reference block and other frame of the window, out of the predictive
// search positions (up to ps_num * (2 ps_range + 1)^2, 162 to 242 with the default profiles)
constexpr int kLearnedFrameProposals = 32;

struct PropBuffers {
    DevBuf hid, feat, rs, desc, grad_d, dF, dH;
};

// bf16 descriptors [frame][H - 7][W - 7][16] of nframes planes (frame stride fs, pitch ld)
static void prop_descriptors(const float *planes, long long fs, int ld, int W, int H, int nframes, const float *wt,
                             PropBuffers &pb, cudaStream_t stream)
{
    const size_t px = (size_t)W * H, npos = (size_t)(W - 7) * (H - 7);
    void *hid = pb.hid.get(2 * 16 * px);
    void *feat = pb.feat.get(2 * 16 * px);
    float *rs = static_cast<float *>(pb.rs.get(4 * 16 * (size_t)H * (W - 3)));
    unsigned char *desc = static_cast<unsigned char *>(pb.desc.get(2 * 16 * npos * nframes));
    for (int k = 0; k < nframes; ++k)
        CU(launch_prop_features(planes + (long long)k * fs, ld, W, H, wt, hid, feat, rs, desc + 2 * 16 * npos * k, stream));
}

// ---------------------------------------------------------------------------------------------
// Shared state of Basic / Final / VBasic / VFinal

class BM3DBase : public Filter {
public:
    bool wiener = false;
    bool vbm3d = false;
    bool tc = false;            // precision form: tensor-core matching estimates (argument "precision")
    bool tc_cf = false;         // precision form: tensor-core transforms as well
    bool learned = false;       // precision "learned": block matching by learned proposals
    // extension of VBasic / VFinal: aggregate = 1 returns VAggregate(radius, sample) of the
    // filter's output directly, without the stacked clip
    bool aggregate = false;
    int agg_sample = 0;
    DevBuf prop_wt;             // proposal network weights (device)
    PropBuffers prop_bufs;
    double plane_sigma[3] = {0, 0, 0};
    Params para, para_default;
    int matrix = MAT_UNSPEC;
    int process[3] = {1, 1, 1};
    PlaneTables tables[3];
    double normY = 1.0;
    float thSSE = 0.0f;
    double distMul = 0.0;
    std::vector<int> sy, sx;

    // BM3D_Data_Base::arguments_process (source/BM3D_Base.cpp:32-259) and
    // VBM3D_Data_Base::arguments_process (source/VBM3D_Base.cpp:104-379), same order and text.
    int arguments(const bm3d_map *in)
    {
        int error;
        if (!map_get_clip(in, "input", &vi) || !valid_clip(vi))
            return fail(BM3D_ERR_ARG, err("Invalid input clip, only constant format input supported"));
        if ((vi.sample_type == BM3D_INTEGER && vi.bits_per_sample > 16) ||
            (vi.sample_type == BM3D_FLOAT && vi.bits_per_sample != 32))
            return fail(BM3D_ERR_ARG, err("Invalid input clip, only 8-16 bit integer or 32 bit float formats supported"));
        if (!map_get_clip(in, "ref", &rvi)) {
            rdef = false;
            rvi = vi;
        } else {
            rdef = true;
            if (!valid_clip(rvi))
                return fail(BM3D_ERR_ARG, err("Invalid clip \"ref\", only constant format input supported"));
            if (!same_format(rvi, vi))
                return fail(BM3D_ERR_ARG, err("input clip and clip \"ref\" must be of the same format"));
            if (rvi.width != vi.width || rvi.height != vi.height)
                return fail(BM3D_ERR_ARG, err("input clip and clip \"ref\" must be of the same width and height"));
            if (rvi.num_frames != vi.num_frames)
                return fail(BM3D_ERR_ARG, err("input clip and clip \"ref\" must have the same number of frames"));
        }
        // profile
        const char *prof = map_get_data(in, "profile", 0, &error);
        para.profile = error ? para_default.profile : std::string(prof);
        if (para.profile != "fast" && para.profile != "lc" && para.profile != "np" && para.profile != "high" &&
            para.profile != "vn")
            return fail(BM3D_ERR_ARG, err("Unrecognized \"profile\" specified, should be \"fast\", \"lc\", \"np\", \"high\" or \"vn\""));
        para_default = vbm3d ? vbm3d_profile(wiener, para.profile) : bm3d_profile(wiener, para.profile);
        // sigma
        int m = map_num(in, "sigma");
        if (m > 0) {
            int i;
            if (m > 3) m = 3;
            for (i = 0; i < m; ++i) {
                para.sigma[i] = map_get_float(in, "sigma", i, &error);
                if (para.sigma[i] < 0)
                    return fail(BM3D_ERR_ARG, err("Invalid \"sigma\" assigned, must be a non-negative floating point number"));
            }
            for (; i < 3; ++i) para.sigma[i] = para.sigma[i - 1];
        } else {
            for (int i = 0; i < 3; ++i) para.sigma[i] = para_default.sigma[i];
        }
        if (vbm3d) {
            para.radius = map_get_int(in, "radius", 0, &error);
            if (error) para.radius = para_default.radius;
            else if (para.radius < 1 || para.radius > 16)
                return fail(BM3D_ERR_ARG, err("Invalid \"radius\" assigned, must be an integer in [1, 16]"));
        }
        para.B = map_get_int(in, "block_size", 0, &error);
        if (error) para.B = para_default.B;
        else if (para.B < 1 || para.B > 64)
            return fail(BM3D_ERR_ARG, err("Invalid \"block_size\" assigned, must be an integer in [1, 64]"));
        else if (para.B > vi.width || para.B > vi.height)
            return fail(BM3D_ERR_ARG, err("Invalid \"block_size\" assigned, must not exceed width or height of the frame"));
        para.step = map_get_int(in, "block_step", 0, &error);
        if (error) para.step = para_default.step;
        else if (para.step < 1 || para.step > para.B)
            return fail(BM3D_ERR_ARG, err("Invalid \"block_step\" assigned, must be an integer in [1, block_size]"));
        para.G = map_get_int(in, "group_size", 0, &error);
        if (error) para.G = para_default.G;
        else if (para.G < 1 || para.G > 256)
            return fail(BM3D_ERR_ARG, err("Invalid \"group_size\" assigned, must be an integer in [1, 256]"));
        para.R = map_get_int(in, "bm_range", 0, &error);
        if (error) para.R = para_default.R;
        else if (para.R < 1)
            return fail(BM3D_ERR_ARG, err("Invalid \"bm_range\" assigned, must be a positive integer"));
        para.bmstep = map_get_int(in, "bm_step", 0, &error);
        if (error) para.bmstep = para_default.bmstep;
        else if (para.bmstep < 1 || para.bmstep > para.R)
            return fail(BM3D_ERR_ARG, err("Invalid \"bm_step\" assigned, must be an integer in [1, bm_range]"));
        if (vbm3d) {
            para.psnum = map_get_int(in, "ps_num", 0, &error);
            if (error) para.psnum = para_default.psnum;
            else if (para.psnum < 1 || para.psnum > para.G)
                return fail(BM3D_ERR_ARG, err("Invalid \"ps_num\" assigned, must be an integer in [1, group_size]"));
            para.psrange = map_get_int(in, "ps_range", 0, &error);
            if (error) para.psrange = para_default.psrange;
            else if (para.psrange < 1)
                return fail(BM3D_ERR_ARG, err("Invalid \"ps_range\" assigned, must be a positive integer"));
            para.psstep = map_get_int(in, "ps_step", 0, &error);
            if (error) para.psstep = para_default.psstep;
            else if (para.psstep < 1 || para.psstep > para.psrange)
                return fail(BM3D_ERR_ARG, err("Invalid \"ps_step\" assigned, must be an integer in [1, ps_range]"));
        }
        para.thMSE = map_get_float(in, "th_mse", 0, &error);
        if (error) para.thMSE = thmse_default(wiener, para.profile, para.sigma[0]);
        else if (para.thMSE <= 0)
            return fail(BM3D_ERR_ARG, err("Invalid \"th_mse\" assigned, must be a positive floating point number"));
        const int64_t mtx = map_get_int64(in, "matrix", 0, &error);
        matrix = (int)mtx;
        if (vi.color_family == BM3D_RGB) matrix = MAT_OPP;
        else if (error || matrix == MAT_UNSPEC) matrix = matrix_default(vi.width, vi.height);
        else if (matrix != MAT_GBR && matrix != MAT_BT709 && matrix != MAT_FCC && matrix != MAT_BT470BG &&
                 matrix != MAT_SMPTE170M && matrix != MAT_SMPTE240M && matrix != MAT_YCGCO &&
                 matrix != MAT_BT2020NC && matrix != MAT_BT2020C && matrix != MAT_OPP)
            return fail(BM3D_ERR_ARG, err("Unsupported \"matrix\" specified"));
        for (int i = 0; i < 3; ++i)
            if (vi.color_family != BM3D_RGB && para.sigma[i] == 0) process[i] = 0;
        if (process[1] || process[2]) {
            if (vi.subsampling_h || vi.subsampling_w)
                return fail(BM3D_ERR_ARG, err("input clip: sub-sampled format is not supported when chroma is processed, convert it to YUV444 or RGB first. "
                                              "For the best quality, RGB colorspace is recommended as input."));
            if (rvi.subsampling_h || rvi.subsampling_w)
                return fail(BM3D_ERR_ARG, err("clip \"ref\": sub-sampled format is not supported when chroma is processed, convert it to YUV444 or RGB first. "
                                              "For the best quality, RGB colorspace is recommended as input."));
        }
        if (!wiener) {
            // BM3D_Basic_Data / VBM3D_Basic_Data: hard_thr (source/BM3D_Basic.cpp:44-53)
            para.lambda = map_get_float(in, "hard_thr", 0, &error);
            if (error) para.lambda = para_default.lambda;
            else if (para.lambda <= 0)
                return fail(BM3D_ERR_ARG, err("Invalid \"hard_thr\" assigned, must be a positive floating point number"));
        }
        // extension: "precision" selects the plain FP32 path ("fp32", default), the tensor-core
        // precision form ("tf32"), its matching alone with the plain transforms ("tf32_match":
        // the same lists, so the output of "fp32") or the learned proposals ("learned")
        const char *prec = map_get_data(in, "precision", 0, &error);
        if (!error) {
            const std::string pr(prec);
            if (pr == "tf32") tc = tc_cf = true;
            else if (pr == "tf32_match") tc = true;
            else if (pr == "learned") tc = tc_cf = learned = true;
            else if (pr != "fp32") return fail(BM3D_ERR_ARG, err("Invalid \"precision\" assigned, must be \"fp32\", \"tf32\", \"tf32_match\" or \"learned\""));
        }
        if (vbm3d) {
            const int64_t ag = map_get_int64(in, "aggregate", 0, &error);
            if (!error) {
                if (ag != 0 && ag != 1)
                    return fail(BM3D_ERR_ARG, err("Invalid \"aggregate\" assigned, must be 0 (stacked output) or 1 (aggregated output)"));
                aggregate = ag == 1;
            }
            const int64_t sm = map_get_int64(in, "sample", 0, &error);
            if (!error) {
                if (sm != 0 && sm != 1)
                    return fail(BM3D_ERR_ARG, err("Invalid 'sample' assigned, must be 0 (integer sample type) or 1 (float sample type)"));
                agg_sample = (int)sm;
            }
        }
        return BM3D_OK;
    }

    // init_filter_data (source/BM3D_Base.cpp:262-283) plus the block-matching constants
    // (include/Block.h:557-560)
    int init_filter_data()
    {
        double norm[3];
        matrix_norms(matrix, norm);
        normY = norm[0];
        for (int c = 0; c < 3; ++c) plane_sigma[c] = para.sigma[c] / double(255) * norm[c];
        para.thMSE *= normY;
        for (int c = 0; c < 3; ++c)
            if (process[c]) tables[c] = plane_tables(wiener, para.sigma[c] / double(255) * norm[c], para.G, para.B, para.lambda);
        const double MSE2SSE = static_cast<double>(para.B * para.B) * 1.0f * 1.0f / double(255 * 255);
        distMul = double(1) / MSE2SSE;
        thSSE = static_cast<float>(para.thMSE * MSE2SSE);
        sy = scan_positions(vi.height, para.B, para.step);
        sx = scan_positions(vi.width, para.B, para.step);
        if (vi.width > (vbm3d ? 8191 : 65535) || vi.height > (vbm3d ? 8191 : 65535))
            return fail(BM3D_ERR_UNSUPPORTED, err("frame dimensions beyond the supported maximum"));
        return BM3D_OK;
    }

    // ---- workspace ----
    int W = 0, H = 0, ld = 0;
    long long fs = 0;                      // floats per frame plane
    DevBuf ws_src[3], ws_ref[3], acc_num[3], acc_w[3];
    DevBuf m_pos, m_n, m_key, v_pos, v_n, v_key;
    DevBuf d_sy, d_sx, scratch;
    DevBuf d_winb, d_winl, d_winc, d_slot0;
    DevBuf tc_tab, tc_status, plist, plist_n, tlists, tlist_n;
    // precision form, hard threshold: the recheck band (fraction of the threshold), the counters of
    // the last call ([0] coefficients recomputed in fp32, [1] decisions changed) and the retained-
    // coefficient count of every group of the last call ([plane][group])
    float recheck_band = kRecheckBand;
    DevBuf tc_counts, retained_buf;
    unsigned long long last_tc_counts[2] = {0, 0};
    DirectTables dtabs;
    int last_count = 0;

    int setup_device()
    {
        W = vi.width;
        H = vi.height;
        ld = (W + 31) / 32 * 32;
        fs = (long long)H * ld;
        const DeviceTables &dt = device_tables();
        (void)dt;
        CU(cudaMemcpy(d_sy.get(sizeof(int) * sy.size()), sy.data(), sizeof(int) * sy.size(), cudaMemcpyHostToDevice));
        CU(cudaMemcpy(d_sx.get(sizeof(int) * sx.size()), sx.data(), sizeof(int) * sx.size(), cudaMemcpyHostToDevice));
        std::vector<int> lengths;
        for (int n = 1; n <= para.G; ++n) lengths.push_back(n);
        lengths.push_back(para.B);
        build_direct_tables(dtabs, lengths);
        if (tc_cf && cf_tc_supported(para.B, para.G)) {
            std::vector<unsigned char> img;
            cf_tc_tables(para.G, img);
            // fp64 tables of the hard-threshold recheck after the image: C8[u][y], Dz[kz][b]
            std::vector<double> xt;
            const double pi = 3.14159265358979323846;
            for (int u = 0; u < 8; ++u)
                for (int y = 0; y < 8; ++y) xt.push_back(2.0 * std::cos(pi * (2 * y + 1) * u / 16.0));
            for (int kz = 0; kz < para.G; ++kz)
                for (int b = 0; b < para.G; ++b) xt.push_back(2.0 * std::cos(pi * (2 * b + 1) * kz / (2.0 * para.G)));
            const size_t base = img.size();
            img.resize(base + xt.size() * sizeof(double));
            std::memcpy(img.data() + base, xt.data(), xt.size() * sizeof(double));
            // then, in fp32 for the per-block DC terms, the forward z matrix as [b][kz] and the
            // inverse one (Dz with row 0 replaced by ones) as [kz][b]: the lanes of a warp
            // (consecutive kz, resp. b) read consecutive words
            std::vector<float> ft;
            const double *dz = xt.data() + 64;
            for (int b = 0; b < para.G; ++b)
                for (int kz = 0; kz < para.G; ++kz) ft.push_back((float)dz[kz * para.G + b]);
            for (int kz = 0; kz < para.G; ++kz)
                for (int b = 0; b < para.G; ++b) ft.push_back(kz == 0 ? 1.0f : (float)dz[kz * para.G + b]);
            // then the rows of the n-point z-stage matrices (Wiener kernels, tiles with short groups)
            std::vector<float> pt;
            cf_tc_partial_tables(para.G, pt);
            ft.insert(ft.end(), pt.begin(), pt.end());
            // then the transposed z stage's B operands
            cf_tc_zt_tables(para.G, pt);
            ft.insert(ft.end(), pt.begin(), pt.end());
            const size_t fbase = img.size();
            img.resize(fbase + ft.size() * sizeof(float));
            std::memcpy(img.data() + fbase, ft.data(), ft.size() * sizeof(float));
            CU(cudaMemcpy(tc_tab.get(img.size()), img.data(), img.size(), cudaMemcpyHostToDevice));
            CU(cudaMemset(tc_status.get(sizeof(int)), 0, sizeof(int)));
        }
        return BM3D_OK;
    }

    void synced() override
    {
        read_stats();
        check_tc_status();
    }

    // time-out flag of the tensor-core kernel (read after the stream is synchronised)
    void check_tc_status()
    {
        if (tc_counts.p) CU(cudaMemcpy(last_tc_counts, tc_counts.p, sizeof(last_tc_counts), cudaMemcpyDeviceToHost));
        if (!tc_status.p) return;
        int st = 0;
        CU(cudaMemcpy(&st, tc_status.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (st) throw std::runtime_error(err(st & 2 ? "tensor-core collaborative filter timed out (products still in flight after the drain wait)"
                                                   : "tensor-core collaborative filter timed out"));
    }

    // float workspace conversion of one input frame set into plane slot `slot`
    void ingest(const bm3d_frame &fr, bool is_ref, int slot, bool full)
    {
        const int np = nplanes();
        const PlaneGeom g{W * bytes_per_sample(vi), H};
        DevBuf *ws = is_ref ? ws_ref : ws_src;
        std::vector<PlanePtr> in, out;
        const int kind = sample_kind(vi);
        if (vi.color_family == BM3D_RGB) {
            for (int p = 0; p < 3; ++p) in.push_back(stager_.view(fr, p, g, stream));
            // Basic's ref needs only Y (RGB2FloatY), everything else the three OPP planes
            const bool y_only = is_ref && !wiener;
            for (int p = 0; p < (y_only ? 1 : 3); ++p)
                out.push_back(PlanePtr{ws[p].as<float>() + slot * fs, (long long)ld * 4});
            const ConvProgram pr = y_only ? rgb2y_program(kind, vi.bits_per_sample, W, H)
                                          : rgb2opp_program(kind, vi.bits_per_sample, SK_F32, 32, W, H, false);
            CU(launch_convert(pr, upload_ptrs(conv_in_[conv_i_], in), upload_ptrs(conv_out_[conv_i_], out), 1, stream));
            conv_i_ = (conv_i_ + 1) % kConvSlots;
            return;
        }
        for (int p = 0; p < np; ++p) {
            // which planes are needed: src -> processed planes (+ Y when it is the matching plane);
            // ref -> Y, and the processed chroma planes for the Wiener filter
            bool need;
            if (!is_ref) need = process[p] || (p == 0 && !rdef);
            else need = p == 0 || (wiener && process[p]);
            if (!need) continue;
            std::vector<PlanePtr> i1{stager_.view(fr, p, g, stream)};
            std::vector<PlanePtr> o1{PlanePtr{ws[p].as<float>() + slot * fs, (long long)ld * 4}};
            ConvProgram pr{};
            if (kind == SK_F32) pr = raw_program(SK_F32, 1, W, H);
            else {
                pr.mode = 0;
                pr.in_kind = kind;
                pr.out_kind = SK_F32;
                pr.nin = pr.nout = 1;
                pr.W = W;
                pr.H = H;
                pr.op[0] = int2float_op(vi.bits_per_sample, full, p > 0);
            }
            CU(launch_convert(pr, upload_ptrs(conv_in_[conv_i_], i1), upload_ptrs(conv_out_[conv_i_], o1), 1, stream));
            conv_i_ = (conv_i_ + 1) % kConvSlots;
        }
    }

    // ingest of frames fr[0..count) into workspace slots slot0.. in one conversion launch when
    // their range flags agree (always for float input), else frame by frame
    void ingest_all(const bm3d_frame *const *fr, int count, bool is_ref, int slot0, const std::vector<bool> &full)
    {
        bool same = true;
        for (int k = 1; k < count; ++k) same = same && full[k] == full[0];
        const int kind = sample_kind(vi);
        if (count <= 1 || (!same && kind != SK_F32)) {
            for (int k = 0; k < count; ++k) ingest(*fr[k], is_ref, slot0 + k, full[k]);
            return;
        }
        const int np = nplanes();
        const PlaneGeom g{W * bytes_per_sample(vi), H};
        DevBuf *ws = is_ref ? ws_ref : ws_src;
        std::vector<PlanePtr> in, out;
        ConvProgram pr{};
        if (vi.color_family == BM3D_RGB) {
            const bool y_only = is_ref && !wiener;
            for (int k = 0; k < count; ++k) {
                for (int p = 0; p < 3; ++p) in.push_back(stager_.view(*fr[k], p, g, stream));
                for (int p = 0; p < (y_only ? 1 : 3); ++p)
                    out.push_back(PlanePtr{ws[p].as<float>() + (slot0 + k) * fs, (long long)ld * 4});
            }
            pr = y_only ? rgb2y_program(kind, vi.bits_per_sample, W, H)
                        : rgb2opp_program(kind, vi.bits_per_sample, SK_F32, 32, W, H, false);
        } else {
            // every plane of the format in one program; planes not needed get no output
            if (kind == SK_F32) pr = raw_program(SK_F32, np, W, H);
            else {
                pr.mode = 0;
                pr.in_kind = kind;
                pr.out_kind = SK_F32;
                pr.nin = pr.nout = np;
                pr.W = W;
                pr.H = H;
                for (int p = 0; p < np; ++p) pr.op[p] = int2float_op(vi.bits_per_sample, full[0], p > 0);
            }
            for (int k = 0; k < count; ++k)
                for (int p = 0; p < np; ++p) {
                    const bool need = !is_ref ? (process[p] || (p == 0 && !rdef)) : (p == 0 || (wiener && process[p]));
                    in.push_back(need ? stager_.view(*fr[k], p, g, stream) : PlanePtr{nullptr, 0});
                    out.push_back(need ? PlanePtr{ws[p].as<float>() + (slot0 + k) * fs, (long long)ld * 4} : PlanePtr{nullptr, 0});
                }
        }
        CU(launch_convert(pr, upload_ptrs(conv_in_[conv_i_], in), upload_ptrs(conv_out_[conv_i_], out), count, stream));
        conv_i_ = (conv_i_ + 1) % kConvSlots;
    }

    // BM3D_Process_Base::NewFrame / VBM3D_Process_Base::NewFrame property handling
    bool frame_full(const bm3d_frame &fr)
    {
        int64_t opp = fr.prop_bm3d_opp;
        if (opp < 0) opp = 0;
        else if (opp == 1 && vi.color_family != BM3D_RGB && matrix != MAT_OPP)
            log_warning(vbm3d ? "bm3d.VBasic/bm3d.VFinal - warning: There's a frame property \"BM3D_OPP=1\" indicating opponent color space input. You should specify \"matrix=100\" in the filter's argument."
                              : "bm3d.Basic/bm3d.Final - warning: There's a frame property \"BM3D_OPP=1\" indicating opponent color space input. You should specify \"matrix=100\" in the filter's argument.");
        if (fr.prop_range < 0 || opp == 1) return true;
        return fr.prop_range != 0;
    }

    void ensure_ws(int nslots, int nout)
    {
        for (int p = 0; p < 3; ++p) {
            ws_src[p].get(sizeof(float) * fs * nslots);
            if (rdef) ws_ref[p].get(sizeof(float) * fs * nslots);
        }
        const size_t nb = (size_t)sy.size() * sx.size() * nout;
        m_pos.get(sizeof(uint32_t) * nb * para.G);
        m_n.get(sizeof(int) * nb);
        m_key.get(sizeof(float) * nb * para.G);
    }

    bool learned_matching() const { return learned && para.B == 8 && para.G >= 2 && para.G <= 32; }

    void ensure_prop_weights()
    {
        if (!prop_wt.p)
            CU(cudaMemcpy(prop_wt.get(sizeof(float) * kProposalWeightCount), kProposalWeights,
                          sizeof(float) * kProposalWeightCount, cudaMemcpyHostToDevice));
    }

    // K1 over `nout` consecutive frames whose Y planes start at workspace slot `slot0`;
    // desc_window: descriptors already computed for the workspace slots (learned form, V-BM3D)
    void run_bm(int slot0, int nout, uint32_t *pos, int *cnt, float *key, const void *desc_window = nullptr)
    {
        DevBuf *refws = rdef ? ws_ref : ws_src;
        BMArgs a{};
        a.ref = refws[0].as<float>() + slot0 * fs;
        a.frame_stride = fs;
        a.ld = ld;
        a.H = H;
        a.W = W;
        a.B = para.B;
        a.range = para.R / para.bmstep * para.bmstep;
        a.step = para.bmstep;
        a.G = para.G;
        a.thSSE = thSSE;
        a.distMul = distMul;
        a.scan_y = d_sy.as<int>();
        a.scan_x = d_sx.as<int>();
        a.nby = (int)sy.size();
        a.nbx = (int)sx.size();
        a.out_pos = pos;
        a.out_n = cnt;
        a.out_key = key;
        a.stats = stats;
        const int lat = (2 * a.range / a.step + 1);
        a.cand_cap = lat * lat + 1;
        a.win_h = std::min(H, 2 * a.range + a.B);
        const bool use_learned = learned_matching();
        if (tc && !use_learned && para.B == 8 && a.step == 1 && para.G >= 2 && para.G <= 32) {
            // precision form: distance estimates on the tensor cores, exact lists
            const BmtLayout L = bmt_layout(a.range, H, para.step);
            if (L.nrc >= 1 && L.bytes <= 200 * 1024) {
                CU(launch_bm_tc(a, L, nout, stream));
                return;
            }
        }
        size_t smem = 0;
        int warps = 8;
        for (; warps >= 1; warps /= 2) {
            a.warps = warps;
            // odd pitch: the lanes of a warp read consecutive window rows, which then fall in
            // distinct shared-memory banks
            a.win_pitch = (std::min(W, (warps - 1) * para.step + 2 * a.range + a.B) + 4) | 1;
            smem = sizeof(float) * ((size_t)a.win_h * a.win_pitch + (size_t)warps * bm_warp_floats(a.cand_cap, a.G, a.B, a.B != 8));
            if (smem <= 200 * 1024) break;
        }
        if (warps < 1) throw std::runtime_error(err("bm_range / block_size too large for the shared-memory search window"));
        if (use_learned) {
            // learned proposals: descriptors of every block position, then the best
            // kLearnedProposals candidates by descriptor distance re-ranked with the exact SSD
            const void *desc = nullptr;
            if (desc_window) {
                desc = static_cast<const unsigned char *>(desc_window) + (size_t)slot0 * 2 * 16 * (size_t)(W - 7) * (H - 7);
            } else {
                ensure_prop_weights();
                prop_descriptors(a.ref, fs, ld, W, H, nout, prop_wt.as<float>(), prop_bufs, stream);
                desc = prop_bufs.desc.p;
            }
            const size_t psmem = sizeof(float) * ((size_t)a.win_h * a.win_pitch + (size_t)a.warps * prop_warp_floats(a.cand_cap));
            CU(launch_bm_learned(a, desc, kLearnedProposals, nout, psmem, stream));
            return;
        }
        CU(launch_bm_full(a, nout, smem, stream));
    }

    // K3+K4 over groups already in pos/cnt
    void run_cf(long long ngroups, long long blocks_per_frame, const uint32_t *pos, const int *cnt,
                bool v, const int *winb, const int *slot0, int slots, long long acc_stride)
    {
        CFArgs a{};
        const DeviceTables &dt = device_tables();
        DevBuf *refws = rdef ? ws_ref : ws_src;
        for (int p = 0; p < 3; ++p) {
            a.src[p] = ws_src[p].as<float>();
            a.ref[p] = (wiener ? refws[p].as<float>() : ws_src[p].as<float>());
            a.num[p] = acc_num[p].as<float>();
            a.wmap[p] = acc_w[p].as<float>();
            a.process[p] = process[p] && p < nplanes();
            if (!a.process[p]) continue;
            for (int n = 0; n < para.G; ++n) {
                for (int k = 0; k < 4; ++k) a.thr4[p][n][k] = tables[p].thr4[n * 4 + k];
                a.wsig2[p][n] = tables[p].wsig2[n];
            }
        }
        for (int n = 0; n < para.G; ++n) a.amp[n] = (float)tables[process[0] ? 0 : process[1] ? 1 : 2].amp[n];
        a.frame_stride = fs;
        a.ld = ld;
        a.H = H;
        a.W = W;
        a.B = para.B;
        a.G = para.G;
        a.wiener = wiener;
        a.pos = pos;
        a.count = cnt;
        a.ngroups = ngroups;
        a.blocks_per_frame = blocks_per_frame;
        a.vbm3d = v;
        a.win_base = winb;
        a.slot0 = slot0;
        a.slots = slots;
        a.acc_stride = acc_stride;
        a.odd_all = dt.odd_all;
        a.dtab = dtabs.tab.as<float>();
        a.dtab_off = dtabs.off.as<int>();
        const bool fast = cf_fast_supported(para.B, para.G);
        if (!wiener) {
            // retained counts of every group (inspection), written by the filter kernels
            a.retained = static_cast<int *>(retained_buf.get(sizeof(int) * 3 * (size_t)std::max<long long>(1, ngroups)));
            CU(cudaMemsetAsync(a.retained, 0xff, sizeof(int) * 3 * (size_t)std::max<long long>(1, ngroups), stream));
        }
        if (fast && tc && tc_tab.p) {
            a.recheck_band = recheck_band;
            a.tc_stats = static_cast<unsigned long long *>(tc_counts.get(2 * sizeof(unsigned long long)));
            CU(cudaMemsetAsync(a.tc_stats, 0, 2 * sizeof(unsigned long long), stream));
            // precision form: full groups on the tensor cores, partial ones on the plain kernel
            // unless the tensor-core kernel takes them too (Wiener filter, G = 16 / 32)
            if (cf_tc_zt_supported(para.B, para.G, wiener)) {
                // tiles of full groups on the transposed z stage, tiles with a short group on the
                // kernel with per-tile n-point matrices
                const long long ntiles = (ngroups + 128 / para.G - 1) / (128 / para.G);
                const long long nch = cf_tile_chunks(ngroups, para.G);
                int *tl = static_cast<int *>(tlists.get(sizeof(int) * (2 * (size_t)std::max<long long>(1, ntiles) + 2 * (size_t)nch)));
                unsigned int *tn = static_cast<unsigned int *>(tlist_n.get(2 * sizeof(unsigned int)));
                CU(launch_cf_tile_lists(cnt, ngroups, para.G, tl, tn, tl + ntiles, tn + 1, tl + 2 * ntiles, stream));
                a.tlist = tl;
                a.tlist_n = tn;
                CU(launch_cf_tc_zt(a, tc_tab.p, tc_status.as<int>(), stream));
                a.tlist = tl + ntiles;
                a.tlist_n = tn + 1;
                CU(launch_cf_tc(a, tc_tab.p, tc_status.as<int>(), stream));
                return;
            }
            CU(launch_cf_tc(a, tc_tab.p, tc_status.as<int>(), stream));
            if (cf_tc_handles_partial(para.B, para.G, wiener)) return;
            a.skip_full = 1;
            // the plain kernel walks a list of the partial groups instead of skipping the full ones
            long long *pl = static_cast<long long *>(plist.get(sizeof(long long) * (size_t)std::max<long long>(1, ngroups)));
            unsigned int *pn = static_cast<unsigned int *>(plist_n.get(sizeof(unsigned int)));
            CU(cudaMemsetAsync(pn, 0, sizeof(unsigned int), stream));
            CU(launch_cf_partial_list(cnt, ngroups, para.G, pl, pn, stream));
            a.plist = pl;
            a.plist_n = pn;
        }
        if (fast) CU(launch_cf_fast(a, stream));
        if (!fast) {
            // generic path: block sizes other than 8 and group sizes outside {8, 16, 32}; one warp
            // per group with a global scratch slot per resident warp (at most 1 GiB in total)
            const long long slot_floats = (long long)para.G * para.B * para.B * 2;
            long long gwarps = std::min<long long>(148LL * 16, std::max<long long>(1, (1LL << 28) / (slot_floats * 4)));
            gwarps = std::max<long long>(4, gwarps / 4 * 4);
            a.scratch = static_cast<float *>(scratch.get(sizeof(float) * slot_floats * gwarps));
            a.scratch_per_warp = slot_floats;
            a.skip_full = 0;
            CU(launch_cf_generic(a, 4, (int)(gwarps / 4), stream));
        }
    }

    // FP64 oracle of frame k of the last batch (BM3D filters): planes [p][H][W] to host memory
    int reference_fp64(int k, double *out, long long plane_stride) override
    {
        if (vbm3d || k < 0 || k >= last_count) return -1;
        if (para.G > 64 || para.B > 64 || cf_fp64_smem(para.B, para.G) > 200 * 1024) return -1;
        const long long bpf = (long long)sy.size() * sx.size();
        CFArgs a{};
        DevBuf *refws = rdef ? ws_ref : ws_src;
        F64Args f{};
        DevBuf nd[3], dd[3];
        const size_t pl = (size_t)H * W;
        for (int p = 0; p < 3; ++p) {
            a.process[p] = process[p] && p < nplanes();
            a.src[p] = ws_src[p].as<float>() + k * fs;
            a.ref[p] = (wiener ? refws[p].as<float>() : ws_src[p].as<float>()) + k * fs;
            f.sigma[p] = plane_sigma[p];
            if (!a.process[p]) continue;
            f.num[p] = static_cast<double *>(nd[p].get(sizeof(double) * pl));
            f.den[p] = static_cast<double *>(dd[p].get(sizeof(double) * pl));
            CU(cudaMemsetAsync(f.num[p], 0, sizeof(double) * pl, stream));
            CU(cudaMemsetAsync(f.den[p], 0, sizeof(double) * pl, stream));
        }
        f.lambda = para.lambda;
        f.out_stride = W;
        a.frame_stride = fs;
        a.ld = ld;
        a.H = H;
        a.W = W;
        a.B = para.B;
        a.G = para.G;
        a.wiener = wiener;
        a.pos = m_pos.as<uint32_t>() + (size_t)k * bpf * para.G;
        a.count = m_n.as<int>() + (size_t)k * bpf;
        a.ngroups = bpf;
        a.blocks_per_frame = bpf;
        CU(launch_cf_fp64(a, f, stream));
        CU(cudaStreamSynchronize(stream));
        for (int p = 0; p < 3; ++p)
            if (a.process[p]) CU(cudaMemcpy(out + p * plane_stride, f.num[p], sizeof(double) * pl, cudaMemcpyDeviceToHost));
        return 0;
    }

    // retained counts of frame k of the last call: [3][blocks per frame], -1 where not recorded
    int retained(int k, int *out, int cap) override
    {
        if (vbm3d || wiener || k < 0 || k >= last_count || !retained_buf.p) return -1;
        const size_t nb = sy.size() * sx.size();
        if ((size_t)cap < 3 * nb) return -1;
        CU(cudaStreamSynchronize(stream));
        const size_t ng = nb * last_count;
        for (int p = 0; p < 3; ++p)
            CU(cudaMemcpy(out + p * nb, retained_buf.as<int>() + p * ng + k * nb, sizeof(int) * nb, cudaMemcpyDeviceToHost));
        return (int)nb;
    }

    int matches(int k, int *counts, int *zs, int *ys, int *xs, float *keys, int cap) override
    {
        if (k < 0 || k >= last_count) return -1;
        const size_t nb = sy.size() * sx.size();
        if ((size_t)cap < nb) return -1;
        std::vector<int> n(nb);
        std::vector<uint32_t> p(nb * para.G);
        std::vector<float> kk(nb * para.G);
        const uint32_t *P = vbm3d ? v_pos.as<uint32_t>() : m_pos.as<uint32_t>();
        const int *Nn = vbm3d ? v_n.as<int>() : m_n.as<int>();
        const float *Kk = vbm3d ? v_key.as<float>() : m_key.as<float>();
        CU(cudaStreamSynchronize(stream));
        CU(cudaMemcpy(n.data(), Nn + k * nb, sizeof(int) * nb, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(p.data(), P + k * nb * para.G, sizeof(uint32_t) * nb * para.G, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(kk.data(), Kk + k * nb * para.G, sizeof(float) * nb * para.G, cudaMemcpyDeviceToHost));
        for (size_t b = 0; b < nb; ++b) {
            counts[b] = n[b];
            for (int e = 0; e < para.G; ++e) {
                const size_t q = b * para.G + e;
                if (e < n[b]) {
                    if (vbm3d) { zs[q] = unpack3_z(p[q]); ys[q] = unpack3_y(p[q]); xs[q] = unpack3_x(p[q]); }
                    else { zs[q] = 0; ys[q] = unpack_y(p[q]); xs[q] = unpack_x(p[q]); }
                    keys[q] = kk[q];
                } else {
                    zs[q] = ys[q] = xs[q] = -1;
                    keys[q] = 0.0f;
                }
            }
        }
        return (int)nb;
    }

protected:
    static constexpr int kConvSlots = 64;
    DevBuf conv_in_[kConvSlots], conv_out_[kConvSlots];
    int conv_i_ = 0;
};

// ---------------------------------------------------------------------------------------------
// Basic / Final (BM3D_Process_Base, source/BM3D_Base.cpp:290-754)

class BM3DFilter : public BM3DBase {
public:
    int create(const bm3d_map *in)
    {
        int r = arguments(in);
        if (r) return r;
        r = init_filter_data();
        if (r) return r;
        ovi = vi;
        init_stream();
        return setup_device();
    }

    int run(int n, int count, const bm3d_frame *const *src, const bm3d_frame *const *ref, bm3d_frame *const *dst,
            bool sync) override
    {
        const int np = nplanes();
        for (int k = 0; k < count; ++k) {
            if (!frame_ok(src[k], np) || !frame_ok(dst[k], np)) return fail(BM3D_ERR_STATE, err("missing frame planes"));
            if (rdef && !frame_ok(ref ? ref[k] : nullptr, np)) return fail(BM3D_ERR_STATE, err("missing ref frame planes"));
        }
        bool any = false;
        for (int p = 0; p < np; ++p) any = any || process[p];
        const PlaneGeom g{W * bytes_per_sample(vi), H};
        if (!any) {
            // VSProcess::process returns the source frame unchanged
            for (int k = 0; k < count; ++k) {
                std::vector<PlanePtr> i1, o1;
                for (int p = 0; p < np; ++p) { i1.push_back(stager_.view(*src[k], p, g, stream)); o1.push_back(stager_.target(*dst[k], p, g)); }
                CU(launch_convert(raw_program(sample_kind(vi), np, W, H), upload_ptrs(conv_in_[conv_i_], i1), upload_ptrs(conv_out_[conv_i_], o1), 1, stream));
                conv_i_ = (conv_i_ + 1) % kConvSlots;
                copy_props(src[k], dst[k]);
            }
            stager_.flush(stream);
            if (sync) { CU(cudaStreamSynchronize(stream)); stager_.release(); }
            return BM3D_OK;
        }
        ensure_ws(count, count);
        for (int p = 0; p < 3; ++p)
            if (process[p] && p < np) {
                acc_num[p].get(sizeof(float) * fs * count);
                acc_w[p].get(sizeof(float) * fs * count);
            }
        CU(cudaMemsetAsync(stats, 0, 3 * sizeof(unsigned long long), stream));
        mark(0);
        std::vector<bool> full(count);
        for (int k = 0; k < count; ++k) full[k] = frame_full(*src[k]);
        ingest_all(src, count, false, 0, full);
        if (rdef) ingest_all(ref, count, true, 0, full);
        mark(1);
        run_bm(0, count, m_pos.as<uint32_t>(), m_n.as<int>(), m_key.as<float>());
        mark(2);
        mark(3);
        for (int p = 0; p < np; ++p)
            if (process[p]) {
                CU(cudaMemsetAsync(acc_num[p].p, 0, sizeof(float) * fs * count, stream));
                CU(cudaMemsetAsync(acc_w[p].p, 0, sizeof(float) * fs * count, stream));
            }
        const long long bpf = (long long)sy.size() * sx.size();
        run_cf(bpf * count, bpf, m_pos.as<uint32_t>(), m_n.as<int>(), false, nullptr, nullptr, 1, 0);
        mark(4);
        FinalizeArgs fa{};
        for (int p = 0; p < 3; ++p) {
            fa.process[p] = process[p] && p < np;
            fa.num[p] = acc_num[p].as<float>();
            fa.wmap[p] = acc_w[p].as<float>();
            fa.out[p] = acc_num[p].as<float>();
        }
        fa.frame_stride = fs;
        fa.ld = ld;
        fa.H = H;
        fa.W = W;
        fa.B = para.B;
        CU(launch_finalize(fa, count, stream));
        mark(5);
        // egress: one conversion launch for the batch when every plane is processed and the
        // frames' range flags agree (or the output is float), else frame by frame
        const int kind = sample_kind(vi);
        bool batch = count > 1;
        for (int k = 1; k < count; ++k) batch = batch && (full[k] == full[0] || kind == SK_F32);
        for (int p = 0; p < np; ++p) batch = batch && (process[p] || vi.color_family == BM3D_RGB);
        if (batch) {
            std::vector<PlanePtr> i1, o1;
            ConvProgram pr{};
            for (int k = 0; k < count; ++k)
                for (int p = 0; p < np; ++p) {
                    i1.push_back(PlanePtr{acc_num[p].as<float>() + k * fs, (long long)ld * 4});
                    o1.push_back(stager_.target(*dst[k], p, g));
                }
            if (vi.color_family == BM3D_RGB) pr = opp2rgb_program(SK_F32, 32, kind, vi.bits_per_sample, W, H);
            else if (kind == SK_F32) pr = raw_program(SK_F32, np, W, H);
            else {
                pr.mode = 0; pr.in_kind = SK_F32; pr.out_kind = kind; pr.nin = pr.nout = np; pr.W = W; pr.H = H;
                for (int p = 0; p < np; ++p) pr.op[p] = float2int_op(vi.bits_per_sample, full[0], p > 0);
            }
            CU(launch_convert(pr, upload_ptrs(conv_in_[conv_i_], i1), upload_ptrs(conv_out_[conv_i_], o1), count, stream));
            conv_i_ = (conv_i_ + 1) % kConvSlots;
        }
        for (int k = 0; k < count; ++k) {
            if (batch) {
                copy_props(src[k], dst[k]);
                continue;
            }
            std::vector<PlanePtr> i1, o1;
            if (vi.color_family == BM3D_RGB) {
                for (int p = 0; p < 3; ++p) i1.push_back(PlanePtr{acc_num[p].as<float>() + k * fs, (long long)ld * 4});
                for (int p = 0; p < 3; ++p) o1.push_back(stager_.target(*dst[k], p, g));
                CU(launch_convert(opp2rgb_program(SK_F32, 32, kind, vi.bits_per_sample, W, H),
                                  upload_ptrs(conv_in_[conv_i_], i1), upload_ptrs(conv_out_[conv_i_], o1), 1, stream));
                conv_i_ = (conv_i_ + 1) % kConvSlots;
            } else {
                for (int p = 0; p < np; ++p) {
                    std::vector<PlanePtr> a1, b1;
                    ConvProgram pr{};
                    b1.push_back(stager_.target(*dst[k], p, g));
                    if (process[p]) {
                        a1.push_back(PlanePtr{acc_num[p].as<float>() + k * fs, (long long)ld * 4});
                        if (kind == SK_F32) pr = raw_program(SK_F32, 1, W, H);
                        else {
                            pr.mode = 0; pr.in_kind = SK_F32; pr.out_kind = kind; pr.nin = pr.nout = 1; pr.W = W; pr.H = H;
                            pr.op[0] = float2int_op(vi.bits_per_sample, full[k], p > 0);
                        }
                    } else {
                        // planes not processed are copied from the source (VSProcess::_NewFrame)
                        a1.push_back(stager_.view(*src[k], p, g, stream));
                        pr = raw_program(kind, 1, W, H);
                    }
                    CU(launch_convert(pr, upload_ptrs(conv_in_[conv_i_], a1), upload_ptrs(conv_out_[conv_i_], b1), 1, stream));
                    conv_i_ = (conv_i_ + 1) % kConvSlots;
                }
            }
            copy_props(src[k], dst[k]);
        }
        stager_.flush(stream);
        mark(6);
        last_count = count;
        if (sync) {
            CU(cudaStreamSynchronize(stream));
            read_stats();
            check_tc_status();
            stager_.release();
        }
        (void)n;
        return BM3D_OK;
    }
};

// ---------------------------------------------------------------------------------------------
// VBasic / VFinal (VBM3D_Process_Base, source/VBM3D_Base.cpp:410-1039)

class VBM3DFilter : public BM3DBase {
public:
    int create(const bm3d_map *in)
    {
        int r = arguments(in);
        if (r) return r;
        r = init_filter_data();
        if (r) return r;
        if (2 * para.radius + 1 > 63)
            return fail(BM3D_ERR_UNSUPPORTED, err("radius beyond the supported maximum"));
        ovi = vi;
        ovi.color_family = vi.color_family == BM3D_RGB ? BM3D_YUV : vi.color_family;
        if (aggregate) {
            // the output of VAggregate(radius, sample) applied to the stacked clip
            // (source/VAggregate.cpp, VAggregate_Create): same size, 16-bit or float
            ovi.sample_type = agg_sample;
            ovi.bits_per_sample = agg_sample == 1 ? 32 : 16;
        } else {
            ovi.sample_type = BM3D_FLOAT;
            ovi.bits_per_sample = 32;
            ovi.height = vi.height * (para.radius * 2 + 1) * 2;
        }
        init_stream();
        return setup_device();
    }

    // Reference frames whose groups reach output frames [n, n + count): the frames themselves
    // (stacked output), or every frame within the radius of one of them (aggregated output).
    void ref_range(int n, int count, int *r0, int *cnt) const
    {
        const int r = aggregate ? para.radius : 0;
        *r0 = std::max(0, n - r);
        *cnt = std::min(vi.num_frames - 1, n + count - 1 + r) - *r0 + 1;
    }

    void window(int n, int count, int *first, int *num) const override
    {
        const int r = para.radius;
        int r0, rc;
        ref_range(n, count, &r0, &rc);
        const int f0 = std::max(0, r0 - r);
        const int f1 = std::min(vi.num_frames - 1, r0 + rc - 1 + r);
        *first = f0;
        *num = f1 - f0 + 1;
    }

    int run(int n, int count, const bm3d_frame *const *src, const bm3d_frame *const *ref, bm3d_frame *const *dst,
            bool sync) override
    {
        const int np = nplanes();
        int first, nwin;
        window(n, count, &first, &nwin);
        for (int i = 0; i < nwin; ++i) {
            if (!frame_ok(src[i], np)) return fail(BM3D_ERR_STATE, err("missing frame planes"));
            if (rdef && !frame_ok(ref ? ref[i] : nullptr, np)) return fail(BM3D_ERR_STATE, err("missing ref frame planes"));
        }
        for (int k = 0; k < count; ++k)
            if (!frame_ok(dst[k], np)) return fail(BM3D_ERR_STATE, err("missing output frame planes"));
        const int r = para.radius;
        const int slots = 2 * r + 1;
        // reference frames [r0, r0 + rc) are filtered; their groups land in the accumulators of
        // their window frames: per reference frame and window slot (stacked output), or per window
        // frame of the batch (aggregated output: the sums over reference frames are VAggregate's)
        int r0, rc;
        ref_range(n, count, &r0, &rc);
        const long long acc_planes = aggregate ? nwin : (long long)slots * rc;
        ensure_ws(nwin, rc);
        const size_t nb = (size_t)sy.size() * sx.size() * rc;
        v_pos.get(sizeof(uint32_t) * nb * para.G);
        v_n.get(sizeof(int) * nb);
        v_key.get(sizeof(float) * nb * para.G);
        for (int p = 0; p < 3; ++p)
            if (process[p] && p < np) {
                acc_num[p].get(sizeof(float) * fs * acc_planes);
                acc_w[p].get(sizeof(float) * fs * acc_planes);
            }
        CU(cudaMemsetAsync(stats, 0, 3 * sizeof(unsigned long long), stream));
        // window frames into the workspace; properties of each output frame's own source frame
        std::vector<bool> full(nwin);
        for (int i = 0; i < nwin; ++i) full[i] = true;
        for (int k = 0; k < count; ++k) full[n + k - first] = frame_full(*src[n + k - first]);
        mark(0);
        // Int2Float of window frames uses the current frame's range flag; frames outside the
        // output batch use their own (identical for constant-range clips)
        for (int i = 0; i < nwin; ++i)
            if (!(i >= n - first && i < n - first + count)) full[i] = frame_full_quiet(*src[i]);
        ingest_all(src, nwin, false, 0, full);
        if (rdef) ingest_all(ref, nwin, true, 0, full);
        mark(1);
        // learned form: descriptors of every window frame, for the current-frame proposals and
        // for the other frames' predictive search
        const void *dwin = nullptr;
        if (learned_matching()) {
            ensure_prop_weights();
            prop_descriptors((rdef ? ws_ref : ws_src)[0].as<float>(), fs, ld, W, H, nwin, prop_wt.as<float>(), prop_bufs, stream);
            dwin = prop_bufs.desc.p;
        }
        // K1 on the reference frames
        run_bm(r0 - first, rc, m_pos.as<uint32_t>(), m_n.as<int>(), m_key.as<float>(), dwin);
        mark(2);
        // window tables
        std::vector<int> winb(rc), winl(rc), winc(rc), s0(rc);
        for (int k = 0; k < rc; ++k) {
            const int nn = r0 + k;
            const int boff = -std::min(nn, r);
            const int foff = std::min(vi.num_frames - 1 - nn, r);
            winb[k] = nn + boff - first;
            winl[k] = foff - boff + 1;
            winc[k] = -boff;
            s0[k] = aggregate ? winb[k] : r + boff;
        }
        CU(cudaMemcpyAsync(d_winb.get(sizeof(int) * rc), winb.data(), sizeof(int) * rc, cudaMemcpyHostToDevice, stream));
        CU(cudaMemcpyAsync(d_winl.get(sizeof(int) * rc), winl.data(), sizeof(int) * rc, cudaMemcpyHostToDevice, stream));
        CU(cudaMemcpyAsync(d_winc.get(sizeof(int) * rc), winc.data(), sizeof(int) * rc, cudaMemcpyHostToDevice, stream));
        CU(cudaMemcpyAsync(d_slot0.get(sizeof(int) * rc), s0.data(), sizeof(int) * rc, cudaMemcpyHostToDevice, stream));
        // K2
        VBMArgs va{};
        DevBuf *refws = rdef ? ws_ref : ws_src;
        va.ref = refws[0].as<float>();
        va.frame_stride = fs;
        va.ld = ld;
        va.H = H;
        va.W = W;
        va.B = para.B;
        va.G = para.G;
        va.ps_num = para.psnum;
        va.ps_range = para.psrange / para.psstep * para.psstep;
        va.ps_step = para.psstep;
        va.thSSE = thSSE;
        va.distMul = distMul;
        va.scan_y = d_sy.as<int>();
        va.scan_x = d_sx.as<int>();
        va.nby = (int)sy.size();
        va.nbx = (int)sx.size();
        va.win_base = d_winb.as<int>();
        va.win_len = d_winl.as<int>();
        va.win_cur = d_winc.as<int>();
        va.cur_pos = m_pos.as<uint32_t>();
        va.cur_key = m_key.as<float>();
        va.cur_n = m_n.as<int>();
        va.out_pos = v_pos.as<uint32_t>();
        va.out_key = v_key.as<float>();
        va.out_n = v_n.as<int>();
        va.stats = stats;
        const int wl = 2 * (va.ps_range / va.ps_step) + 1;
        va.sp_cap = para.psnum * wl * wl;
        va.list_cap = para.G * slots;
        va.desc = dwin;
        va.desc_frame = (long long)(W - 7) * (H - 7);
        va.nprop = kLearnedFrameProposals;
        size_t smem = 0;
        int warps = 4;
        for (; warps >= 1; warps /= 2) {
            smem = sizeof(float) * (size_t)warps * vbm_warp_floats(va.sp_cap, va.list_cap, va.G, va.ps_num, va.B);
            if (smem <= 200 * 1024) break;
        }
        if (warps < 1) return fail(BM3D_ERR_UNSUPPORTED, err("ps_num / ps_range too large for the predictive-search buffers"));
        va.warps = warps;
        CU(launch_vbm_predict(va, rc, smem, stream));
        mark(3);
        // K3+K4 into the accumulators
        for (int p = 0; p < np; ++p)
            if (process[p]) {
                CU(cudaMemsetAsync(acc_num[p].p, 0, sizeof(float) * fs * acc_planes, stream));
                CU(cudaMemsetAsync(acc_w[p].p, 0, sizeof(float) * fs * acc_planes, stream));
            }
        const long long bpf = (long long)sy.size() * sx.size();
        run_cf(bpf * rc, bpf, v_pos.as<uint32_t>(), v_n.as<int>(), true, d_winb.as<int>(), d_slot0.as<int>(),
               aggregate ? 0 : slots, fs);
        mark(4);
        if (aggregate) aggregated_output(n, count, first, src, dst);
        else stacked_output(count, dst);
        mark(5);
        stager_.flush(stream);
        mark(6);
        for (int k = 0; k < count; ++k) {
            const bm3d_frame *sf = src[n + k - first];
            copy_props(sf, dst[k]);
            if (vi.color_family == BM3D_RGB) dst[k]->prop_bm3d_opp = 1;
            if (aggregate) {
                // VAggregate deletes the V-BM3D properties (include/VAggregate.h:147-231)
                dst[k]->prop_v_radius = -1;
                dst[k]->prop_v_process_count = -1;
            } else {
                dst[k]->prop_v_radius = r;
                dst[k]->prop_v_process_count = 3;
                for (int p = 0; p < 3; ++p) dst[k]->prop_v_process[p] = process[p];
            }
        }
        last_count = rc;
        if (sync) {
            CU(cudaStreamSynchronize(stream));
            read_stats();
            check_tc_status();
            stager_.release();
        }
        return BM3D_OK;
    }

private:
    // VBasic / VFinal stacked clip (VBM3D_Process_Base, include/VBM3D_Base.h:284-312): slot
    // 2(r+k) numerator, 2(r+k)+1 denominator of window frame k
    void stacked_output(int count, bm3d_frame *const *dst)
    {
        const int np = nplanes();
        const PlaneGeom go{W * 4, ovi.height};
        std::vector<PlanePtr> outs;
        for (int k = 0; k < count; ++k)
            for (int p = 0; p < 3; ++p) {
                if (p < np && process[p]) {
                    PlanePtr t = stager_.target(*dst[k], p, go);
                    CU(cudaMemset2DAsync(t.ptr, t.stride, 0, (size_t)W * 4, ovi.height, stream));
                    outs.push_back(t);
                } else {
                    outs.push_back(PlanePtr{nullptr, 0});
                }
            }
        VStackArgs sa{};
        for (int p = 0; p < 3; ++p) {
            sa.num[p] = acc_num[p].as<float>();
            sa.wmap[p] = acc_w[p].as<float>();
            sa.process[p] = process[p] && p < np;
        }
        sa.slot_stride = fs;
        sa.ld = ld;
        sa.H = H;
        sa.W = W;
        sa.B = para.B;
        sa.slots = 2 * para.radius + 1;
        sa.out = upload_ptrs(ptr_out_, outs);
        CU(launch_vstack(sa, count, stream));
    }

    // Aggregated output: frame m's accumulators already hold the sums over every reference frame
    // within the radius (VAggregate_Process::Kernel, source/VAggregate.cpp:93-160); normalise them
    // in place and convert to the output format (Float2Int to 16 bits, or float).  Planes that
    // are not processed come out zero, as VAggregate writes them.
    void aggregated_output(int n, int count, int first, const bm3d_frame *const *src, bm3d_frame *const *dst)
    {
        const int np = nplanes();
        FinalizeArgs fa{};
        float *agg[3] = {nullptr, nullptr, nullptr};
        for (int p = 0; p < 3; ++p) {
            fa.process[p] = process[p] && p < np;
            if (!fa.process[p]) continue;
            agg[p] = acc_num[p].as<float>() + (long long)(n - first) * fs;
            fa.num[p] = agg[p];
            fa.wmap[p] = acc_w[p].as<float>() + (long long)(n - first) * fs;
            fa.out[p] = agg[p];
        }
        fa.frame_stride = fs;
        fa.ld = ld;
        fa.H = H;
        fa.W = W;
        fa.B = para.B;
        CU(launch_finalize(fa, count, stream));
        const PlaneGeom go{W * bytes_per_sample(ovi), H};
        for (int k = 0; k < count; ++k) {
            const bm3d_frame &sf = *src[n + k - first];
            const int64_t opp = vi.color_family == BM3D_RGB ? 1 : (sf.prop_bm3d_opp < 0 ? 0 : sf.prop_bm3d_opp);
            const bool full = (sf.prop_range < 0 || opp == 1) ? true : sf.prop_range != 0;
            for (int p = 0; p < np; ++p) {
                PlanePtr t = stager_.target(*dst[k], p, go);
                if (!process[p]) {
                    CU(cudaMemset2DAsync(t.ptr, t.stride, 0, (size_t)go.width_bytes, H, stream));
                    continue;
                }
                std::vector<PlanePtr> a1{PlanePtr{agg[p] + (long long)k * fs, (long long)ld * 4}}, b1{t};
                ConvProgram pr{};
                if (agg_sample == 1) pr = raw_program(SK_F32, 1, W, H);
                else {
                    pr.mode = 0; pr.in_kind = SK_F32; pr.out_kind = SK_U16; pr.nin = pr.nout = 1; pr.W = W; pr.H = H;
                    pr.op[0] = float2int_op(16, full, p > 0);
                }
                CU(launch_convert(pr, upload_ptrs(conv_in_[conv_i_], a1), upload_ptrs(conv_out_[conv_i_], b1), 1, stream));
                conv_i_ = (conv_i_ + 1) % kConvSlots;
            }
        }
    }

    bool frame_full_quiet(const bm3d_frame &fr) const
    {
        int64_t opp = fr.prop_bm3d_opp < 0 ? 0 : fr.prop_bm3d_opp;
        if (fr.prop_range < 0 || opp == 1) return true;
        return fr.prop_range != 0;
    }
};

// ---------------------------------------------------------------------------------------------
// VAggregate (source/VAggregate.cpp, include/VAggregate.h)

class VAggFilter : public Filter {
public:
    int radius = 1;
    int sample = 0;
    DevBuf ws[3];

    int create(const bm3d_map *in)
    {
        int error;
        if (!map_get_clip(in, "input", &vi) || !valid_clip(vi))
            return fail(BM3D_ERR_ARG, err("Invalid input clip, only constant format input supported"));
        if (vi.sample_type != BM3D_FLOAT || vi.bits_per_sample != 32)
            return fail(BM3D_ERR_ARG, err("Invalid input clip, only accept 32 bit float format clip from bm3d.VBasic or bm3d.VFinal"));
        if (vi.color_family == BM3D_RGB)
            return fail(BM3D_ERR_ARG, err("Invalid input clip, must be of Gray or YUV color family"));
        radius = map_get_int(in, "radius", 0, &error);
        if (error) radius = 1;
        else if (radius < 1 || radius > 16)
            return fail(BM3D_ERR_ARG, err("Invalid \"radius\" assigned, must be an integer in [1, 16]"));
        int64_t s = map_get_int64(in, "sample", 0, &error);
        if (error) s = 0;
        else if (s != 0 && s != 1)
            return fail(BM3D_ERR_ARG, err("Invalid 'sample' assigned, must be 0 (integer sample type) or 1 (float sample type)"));
        sample = (int)s;
        ovi = vi;
        ovi.sample_type = sample;
        ovi.bits_per_sample = sample == 1 ? 32 : 16;
        ovi.height = vi.height / (radius * 2 + 1) / 2;
        init_stream();
        return BM3D_OK;
    }

    void window(int n, int count, int *first, int *num) const override
    {
        const int f0 = std::max(0, n - radius);
        const int f1 = std::min(vi.num_frames - 1, n + count - 1 + radius);
        *first = f0;
        *num = f1 - f0 + 1;
    }

    int run(int n, int count, const bm3d_frame *const *src, const bm3d_frame *const *, bm3d_frame *const *dst,
            bool sync) override
    {
        const int np = vi.color_family == BM3D_GRAY ? 1 : 3;
        int first, nwin;
        window(n, count, &first, &nwin);
        for (int i = 0; i < nwin; ++i)
            if (!frame_ok(src[i], np)) return fail(BM3D_ERR_STATE, err("missing frame planes"));
        for (int k = 0; k < count; ++k)
            if (!frame_ok(dst[k], np)) return fail(BM3D_ERR_STATE, err("missing output frame planes"));
        const int Ho = ovi.height, W = vi.width;
        const int ld = (W + 31) / 32 * 32;
        const long long fs = (long long)Ho * ld;
        const PlaneGeom gi{W * 4, vi.height};
        const PlaneGeom go{W * bytes_per_sample(ovi), Ho};
        std::vector<PlanePtr> in((size_t)count * (2 * radius + 1) * 3, PlanePtr{nullptr, 0});
        std::vector<PlanePtr> views((size_t)nwin * 3, PlanePtr{nullptr, 0});
        for (int i = 0; i < nwin; ++i)
            for (int p = 0; p < np; ++p) views[i * 3 + p] = stager_.view(*src[i], p, gi, stream);
        std::vector<int> nfr(count), boff(count);
        int proc[3] = {1, 1, 1};
        std::vector<bool> full(count);
        for (int k = 0; k < count; ++k) {
            const int nn = n + k;
            const bm3d_frame &cf = *src[nn - first];
            // VAggregate_Process::NewFrame property checks (include/VAggregate.h:147-231)
            if (cf.prop_v_radius < 0)
                log_warning("bm3d.VAggregate - warning: No frame property \"BM3D_V_radius\" exists in the input frame. Make sure you call bm3d.VAggregate next to bm3d.VBasic or bm3d.VFinal.");
            else if (cf.prop_v_radius != radius)
                log_warning("bm3d.VAggregate - warning: Mismatch between argument \"radius=" + std::to_string(radius) +
                            "\" and the input frame property \"BM3D_V_radius=" + std::to_string(cf.prop_v_radius) +
                            "\" which indicates the radius used in previous filter (bm3d.VBasic or bm3d.VFinal).");
            if (cf.prop_v_process_count != 3) {
                log_warning("bm3d.VAggregate - warning: No frame property \"BM3D_V_process\" exists in the input frame. Make sure you call bm3d.VAggregate next to bm3d.VBasic or bm3d.VFinal.");
                proc[0] = proc[1] = proc[2] = 1;
            } else {
                for (int p = 0; p < 3; ++p) proc[p] = (int)cf.prop_v_process[p];
            }
            const int64_t opp = cf.prop_bm3d_opp < 0 ? 0 : cf.prop_bm3d_opp;
            full[k] = (cf.prop_range < 0 || opp == 1) ? true : cf.prop_range != 0;
            boff[k] = -std::min(nn, radius);
            const int foff = std::min(vi.num_frames - 1 - nn, radius);
            nfr[k] = foff - boff[k] + 1;
            for (int i = 0; i < nfr[k]; ++i)
                for (int p = 0; p < np; ++p) in[((size_t)k * (2 * radius + 1) + i) * 3 + p] = views[(nn + boff[k] + i - first) * 3 + p];
        }
        for (int p = 0; p < np; ++p) ws[p].get(sizeof(float) * fs * count);
        std::vector<int> hdr(2 * count);
        for (int k = 0; k < count; ++k) { hdr[k] = nfr[k]; hdr[count + k] = boff[k]; }
        int *dh = static_cast<int *>(hdrbuf_.get(sizeof(int) * hdr.size()));
        CU(cudaMemcpyAsync(dh, hdr.data(), sizeof(int) * hdr.size(), cudaMemcpyHostToDevice, stream));
        VAggArgs a{};
        a.in = upload_ptrs(ptr_in_, in);
        a.frames_max = 2 * radius + 1;
        a.nframes = dh;
        a.b_off = dh + count;
        for (int p = 0; p < 3; ++p) {
            a.out[p] = p < np ? ws[p].as<float>() : nullptr;
            a.process[p] = p < np && proc[p];
        }
        a.frame_stride = fs;
        a.ld = ld;
        a.H = Ho;
        a.W = W;
        a.radius = radius;
        CU(launch_vaggregate(a, count, stream));
        for (int k = 0; k < count; ++k) {
            for (int p = 0; p < np; ++p) {
                PlanePtr t = stager_.target(*dst[k], p, go);
                if (!proc[p]) {
                    CU(cudaMemset2DAsync(t.ptr, t.stride, 0, (size_t)go.width_bytes, Ho, stream));
                    continue;
                }
                std::vector<PlanePtr> a1{PlanePtr{ws[p].as<float>() + k * fs, (long long)ld * 4}}, b1{t};
                ConvProgram pr{};
                if (sample == 1) pr = raw_program(SK_F32, 1, W, Ho);
                else {
                    pr.mode = 0; pr.in_kind = SK_F32; pr.out_kind = SK_U16; pr.nin = pr.nout = 1; pr.W = W; pr.H = Ho;
                    pr.op[0] = float2int_op(16, full[k], p > 0);
                }
                CU(launch_convert(pr, upload_ptrs(conv_in_[conv_i_], a1), upload_ptrs(conv_out_[conv_i_], b1), 1, stream));
                conv_i_ = (conv_i_ + 1) % kConvSlots;
            }
            copy_props(src[n + k - first], dst[k]);
            dst[k]->prop_v_radius = -1;
            dst[k]->prop_v_process_count = -1;
        }
        stager_.flush(stream);
        if (sync) { CU(cudaStreamSynchronize(stream)); stager_.release(); }
        return BM3D_OK;
    }

private:
    static constexpr int kConvSlots = 64;
    DevBuf conv_in_[kConvSlots], conv_out_[kConvSlots], hdrbuf_;
    int conv_i_ = 0;
};

}  // namespace bm3d

// =============================================================================================
// C ABI

using namespace bm3d;

struct bm3d_filter {
    std::unique_ptr<Filter> f;
    std::mutex mu;
};

template <typename Fn>
static int guarded(Fn &&fn)
{
    try {
        return fn();
    } catch (const CudaError &e) {
        return fail(BM3D_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e.e) + " (" + e.what + ")");
    } catch (const std::bad_alloc &) {
        return fail(BM3D_ERR_CUDA, "out of host memory");
    } catch (const std::exception &e) {
        return fail(BM3D_ERR_UNSUPPORTED, e.what());
    }
}

extern "C" {

BM3D_API bm3d_map *bm3d_map_create(void) { return new (std::nothrow) bm3d_map(); }
BM3D_API void bm3d_map_free(bm3d_map *m) { delete m; }

BM3D_API int bm3d_map_set_int(bm3d_map *m, const char *key, int64_t v)
{
    if (!m || !key) return fail(BM3D_ERR_STATE, "null map or key");
    MapValue x;
    x.kind = 0;
    x.i = v;
    m->e[key].push_back(x);
    return BM3D_OK;
}

BM3D_API int bm3d_map_set_float(bm3d_map *m, const char *key, double v)
{
    if (!m || !key) return fail(BM3D_ERR_STATE, "null map or key");
    MapValue x;
    x.kind = 1;
    x.f = v;
    m->e[key].push_back(x);
    return BM3D_OK;
}

BM3D_API int bm3d_map_set_data(bm3d_map *m, const char *key, const char *v)
{
    if (!m || !key || !v) return fail(BM3D_ERR_STATE, "null map, key or value");
    MapValue x;
    x.kind = 2;
    x.s = v;
    m->e[key].push_back(x);
    return BM3D_OK;
}

BM3D_API int bm3d_map_set_clip(bm3d_map *m, const char *key, const bm3d_video_info *clip)
{
    if (!m || !key || !clip) return fail(BM3D_ERR_STATE, "null map, key or clip");
    MapValue x;
    x.kind = 3;
    x.clip = *clip;
    m->e[key].push_back(x);
    return BM3D_OK;
}

BM3D_API int bm3d_create(const char *name, const bm3d_map *args, bm3d_filter **out)
{
    g_error.clear();
    if (!name || !args || !out) return fail(BM3D_ERR_STATE, "null argument");
    *out = nullptr;
    const std::string fn = name;
    if (argspec(fn).empty()) return fail(BM3D_ERR_ARG, "bm3d: no function named " + fn);
    int r = check_argspec(fn, args);
    if (r) return r;
    return guarded([&]() -> int {
        // Arguments are validated first (no device needed); device resources are created last,
        // and a missing device surfaces as BM3D_ERR_CUDA.
        std::unique_ptr<Filter> f;
        int rc;
        if (fn == "RGB2OPP" || fn == "OPP2RGB") {
            auto c = std::make_unique<ConvFilter>();
            c->fn = fn;
            c->to_opp = fn == "RGB2OPP";
            rc = c->create(args);
            f = std::move(c);
        } else if (fn == "Basic" || fn == "Final") {
            auto c = std::make_unique<BM3DFilter>();
            c->fn = fn;
            c->wiener = fn == "Final";
            c->para = bm3d_profile(c->wiener, "fast");
            c->para_default = c->para;
            rc = c->create(args);
            f = std::move(c);
        } else if (fn == "VBasic" || fn == "VFinal") {
            auto c = std::make_unique<VBM3DFilter>();
            c->fn = fn;
            c->wiener = fn == "VFinal";
            c->vbm3d = true;
            c->para = vbm3d_profile(c->wiener, "fast");
            c->para_default = c->para;
            rc = c->create(args);
            f = std::move(c);
        } else {
            auto c = std::make_unique<VAggFilter>();
            c->fn = fn;
            rc = c->create(args);
            f = std::move(c);
        }
        if (rc) return rc;
        bm3d_filter *h = new bm3d_filter();
        h->f = std::move(f);
        *out = h;
        return BM3D_OK;
    });
}

BM3D_API int bm3d_output_info(const bm3d_filter *h, bm3d_video_info *out)
{
    if (!h || !out) return fail(BM3D_ERR_STATE, "null argument");
    *out = h->f->ovi;
    return BM3D_OK;
}

BM3D_API int bm3d_frame_window(const bm3d_filter *h, int n, int count, int *first, int *num)
{
    if (!h || !first || !num) return fail(BM3D_ERR_STATE, "null argument");
    if (count < 1 || n < 0 || n + count > h->f->vi.num_frames)
        return fail(BM3D_ERR_STATE, "bm3d." + h->f->fn + ": frame range outside the clip");
    h->f->window(n, count, first, num);
    return BM3D_OK;
}

static int get_frames_impl(bm3d_filter *h, int n, int count, const bm3d_frame *const *src,
                           const bm3d_frame *const *ref, bm3d_frame *const *dst, bool sync)
{
    g_error.clear();
    if (!h || !src || !dst) return fail(BM3D_ERR_STATE, "null argument");
    if (count < 1 || n < 0 || n + count > h->f->vi.num_frames)
        return fail(BM3D_ERR_STATE, "bm3d." + h->f->fn + ": frame range outside the clip");
    std::lock_guard<std::mutex> lk(h->mu);
    return guarded([&]() { return h->f->run(n, count, src, ref, dst, sync); });
}

BM3D_API int bm3d_get_frames(bm3d_filter *h, int n, int count, const bm3d_frame *const *src,
                             const bm3d_frame *const *ref, bm3d_frame *const *dst)
{
    return get_frames_impl(h, n, count, src, ref, dst, true);
}

BM3D_API int bm3d_get_frames_async(bm3d_filter *h, int n, int count, const bm3d_frame *const *src,
                                   const bm3d_frame *const *ref, bm3d_frame *const *dst)
{
    int first = 0, num = 0;
    if (h && count >= 1 && n >= 0 && n + count <= h->f->vi.num_frames) h->f->window(n, count, &first, &num);
    const bool dev = src && dst && all_device(num, src) && all_device(count, dst) && (!ref || all_device(num, ref));
    return get_frames_impl(h, n, count, src, ref, dst, !dev);
}

BM3D_API int bm3d_set_stream(bm3d_filter *h, void *s)
{
    if (!h) return fail(BM3D_ERR_STATE, "null filter");
    std::lock_guard<std::mutex> lk(h->mu);
    h->f->stream = s ? static_cast<cudaStream_t>(s) : h->f->own;
    return BM3D_OK;
}

BM3D_API int bm3d_synchronize(bm3d_filter *h)
{
    if (!h) return fail(BM3D_ERR_STATE, "null filter");
    return guarded([&]() {
        CU(cudaStreamSynchronize(h->f->stream));
        h->f->synced();
        return (int)BM3D_OK;
    });
}

BM3D_API void bm3d_free(bm3d_filter *h) { delete h; }

BM3D_API const char *bm3d_get_error(void) { return g_error.c_str(); }

BM3D_API void bm3d_set_log_callback(bm3d_log_fn fn, void *user)
{
    std::lock_guard<std::mutex> lk(g_log_mutex);
    g_log_fn = fn;
    g_log_user = user;
}

BM3D_API int bm3d_debug_matches(bm3d_filter *h, int k, int *counts, int *zs, int *ys, int *xs, float *keys,
                                int capacity_blocks)
{
    if (!h || !counts || !zs || !ys || !xs || !keys) return -1;
    std::lock_guard<std::mutex> lk(h->mu);
    int r = -1;
    guarded([&]() {
        r = h->f->matches(k, counts, zs, ys, xs, keys, capacity_blocks);
        return 0;
    });
    return r;
}

BM3D_API int bm3d_set_profiling(bm3d_filter *h, int enable)
{
    if (!h) return fail(BM3D_ERR_STATE, "null filter");
    std::lock_guard<std::mutex> lk(h->mu);
    return guarded([&]() {
        h->f->set_profiling(enable != 0);
        return (int)BM3D_OK;
    });
}

BM3D_API int bm3d_debug_stage_times(bm3d_filter *h, double *ms, int capacity)
{
    if (!h || !ms) return -1;
    std::lock_guard<std::mutex> lk(h->mu);
    Filter *f = h->f.get();
    if (!f->profiling || !f->prof_valid) return 0;
    int n = 0;
    guarded([&]() {
        CU(cudaEventSynchronize(f->ev[Filter::kStages]));
        for (int i = 0; i < Filter::kStages && i < capacity; ++i) {
            float t = 0.0f;
            CU(cudaEventElapsedTime(&t, f->ev[i], f->ev[i + 1]));
            ms[i] = t;
            n = i + 1;
        }
        return 0;
    });
    return n;
}

BM3D_API int bm3d_debug_reference_fp64(bm3d_filter *h, int k, double *planes, int64_t plane_stride)
{
    if (!h || !planes) return -1;
    std::lock_guard<std::mutex> lk(h->mu);
    int r = -1;
    guarded([&]() {
        r = h->f->reference_fp64(k, planes, (long long)plane_stride);
        return 0;
    });
    return r;
}

BM3D_API int64_t bm3d_debug_launch_count(void) { return (int64_t)launch_count(); }

BM3D_API int64_t bm3d_debug_slow_blocks(bm3d_filter *h)
{
    if (!h) return -1;
    return (int64_t)h->f->last_slow;
}

BM3D_API int bm3d_debug_bm_tc_counts(bm3d_filter *h, int64_t *fallbacks, int64_t *timeouts)
{
    if (!h) return -1;
    if (fallbacks) *fallbacks = (int64_t)h->f->last_stats[1];
    if (timeouts) *timeouts = (int64_t)h->f->last_stats[2];
    return 0;
}

BM3D_API int bm3d_debug_threshold_rechecks(bm3d_filter *h, int64_t *rechecked, int64_t *changed)
{
    if (!h) return -1;
    BM3DBase *b = dynamic_cast<BM3DBase *>(h->f.get());
    if (!b) return -1;
    if (rechecked) *rechecked = (int64_t)b->last_tc_counts[0];
    if (changed) *changed = (int64_t)b->last_tc_counts[1];
    return 0;
}

BM3D_API int bm3d_debug_set_recheck_band(bm3d_filter *h, float band)
{
    if (!h || !(band >= 0.0f)) return -1;
    BM3DBase *b = dynamic_cast<BM3DBase *>(h->f.get());
    if (!b) return -1;
    b->recheck_band = band;
    return 0;
}

BM3D_API int bm3d_debug_retained_counts(bm3d_filter *h, int k, int *counts, int capacity)
{
    if (!h || !counts) return -1;
    return guarded([&]() -> int { return h->f->retained(k, counts, capacity); });
}

// ---- learned proposal: training and inspection -------------------------------------------------

// Exhaustive lists (exact SSD, no threshold) of nframes planes for block step `step`, group G,
// range R, candidate step 1: the training targets and the recall reference.
static void exhaustive_lists(const float *planes, long long fs, int ld, int W, int H, int nframes, int step, int G, int R,
                             float thsse, const int *dsy, const int *dsx, int nby, int nbx, uint32_t *pos, int *cnt,
                             const void *desc, int nprop, cudaStream_t stream, uint32_t *props = nullptr,
                             unsigned long long *stats = nullptr)
{
    BMArgs a{};
    a.ref = planes;
    a.frame_stride = fs;
    a.ld = ld;
    a.H = H;
    a.W = W;
    a.B = 8;
    a.range = R;
    a.step = 1;
    a.G = G;
    a.thSSE = thsse;
    a.distMul = 1.0;
    a.scan_y = dsy;
    a.scan_x = dsx;
    a.nby = nby;
    a.nbx = nbx;
    a.out_pos = pos;
    a.out_n = cnt;
    a.out_key = nullptr;
    a.stats = stats;
    a.out_prop = props;
    a.cand_cap = (2 * R + 1) * (2 * R + 1) + 1;
    a.win_h = std::min(H, 2 * R + 8);
    size_t smem = 0;
    int warps = 8;
    for (; warps >= 1; warps /= 2) {
        a.warps = warps;
        a.win_pitch = (std::min(W, (warps - 1) * step + 2 * R + 8) + 4) | 1;
        smem = sizeof(float) * ((size_t)a.win_h * a.win_pitch + (size_t)warps * bm_warp_floats(a.cand_cap, G, 8, false));
        if (smem <= 200 * 1024) break;
    }
    if (warps < 1) throw std::runtime_error("bm_range too large");
    if (desc) CU(launch_bm_learned(a, desc, nprop, nframes,
                                   sizeof(float) * ((size_t)a.win_h * a.win_pitch + (size_t)a.warps * prop_warp_floats(a.cand_cap)),
                                   stream));
    else CU(launch_bm_full(a, nframes, smem, stream));
}

BM3D_API int bm3d_proposal_default_weights(float *out, int capacity)
{
    if (!out || capacity < kProposalWeightCount) return fail(BM3D_ERR_STATE, "bm3d_proposal_default_weights: buffer too small");
    std::memcpy(out, kProposalWeights, sizeof(float) * kProposalWeightCount);
    return kProposalWeightCount;
}

BM3D_API int bm3d_proposal_descriptors(const float *frame, int width, int height, const float *weights, float *desc_out)
{
    g_error.clear();
    if (!frame || !weights || !desc_out || width < 8 || height < 8) return fail(BM3D_ERR_STATE, "bad arguments");
    return guarded([&]() -> int {
        DevBuf x, wt;
        PropBuffers pb;
        CU(cudaMemcpy(x.get(sizeof(float) * width * height), frame, sizeof(float) * width * height, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(wt.get(sizeof(float) * kProposalWeightCount), weights, sizeof(float) * kProposalWeightCount, cudaMemcpyHostToDevice));
        prop_descriptors(x.as<float>(), 0, width, width, height, 1, wt.as<float>(), pb, 0);
        const size_t n = (size_t)16 * (width - 7) * (height - 7);
        std::vector<uint16_t> h(n);
        CU(cudaMemcpy(h.data(), pb.desc.p, 2 * n, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; ++i) {
            const uint32_t u = (uint32_t)h[i] << 16;
            std::memcpy(desc_out + i, &u, 4);
        }
        return (int)BM3D_OK;
    });
}

// Loss and weight gradients for given triplets (ay, ax, py, px, ny, nx: block positions of one
// plane, p the candidate that should rank closer): L = mean softplus(s_ap - s_an).
BM3D_API int bm3d_proposal_gradients(const float *frame, int width, int height, const float *weights, const int *triplets,
                                     int ntriplets, float *loss, float *grad)
{
    g_error.clear();
    if (!frame || !weights || !triplets || ntriplets < 1 || !loss || !grad || width < 8 || height < 8)
        return fail(BM3D_ERR_STATE, "bad arguments");
    return guarded([&]() -> int {
        const int Wd = width - 7, Hd = height - 7;
        for (int t = 0; t < 6 * ntriplets; ++t)
            if (triplets[t] < 0 || triplets[t] >= ((t % 2) ? Wd : Hd)) throw std::runtime_error("triplet position outside the plane");
        DevBuf x, wt, tr, gD, dF, dH, gw, dl;
        PropBuffers pb;
        CU(cudaMemcpy(x.get(sizeof(float) * width * height), frame, sizeof(float) * width * height, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(wt.get(sizeof(float) * kProposalWeightCount), weights, sizeof(float) * kProposalWeightCount, cudaMemcpyHostToDevice));
        std::vector<int> trh(7 * (size_t)ntriplets);
        for (int t = 0; t < ntriplets; ++t) {
            trh[7 * t] = 0;
            for (int k = 0; k < 6; ++k) trh[7 * t + 1 + k] = triplets[6 * t + k];
        }
        if (prop_triplet_bytes() != 7 * (int)sizeof(int)) throw std::runtime_error("triplet layout");
        CU(cudaMemcpy(tr.get(trh.size() * sizeof(int)), trh.data(), trh.size() * sizeof(int), cudaMemcpyHostToDevice));
        prop_descriptors(x.as<float>(), 0, width, width, height, 1, wt.as<float>(), pb, 0);
        const size_t npos = (size_t)Wd * Hd, px = (size_t)width * height;
        CU(cudaMemset(gD.get(sizeof(float) * 16 * npos), 0, sizeof(float) * 16 * npos));
        CU(cudaMemset(gw.get(sizeof(float) * kProposalWeightCount), 0, sizeof(float) * kProposalWeightCount));
        CU(cudaMemset(dl.get(sizeof(float)), 0, sizeof(float)));
        CU(launch_prop_loss(tr.p, ntriplets, pb.desc.p, (long long)npos, Wd, gD.as<float>(), 1.0f / ntriplets, dl.as<float>(), 0));
        CU(launch_prop_backward(x.as<float>(), width, width, height, wt.as<float>(), pb.hid.p, gD.as<float>(),
                                static_cast<float *>(dF.get(sizeof(float) * 16 * px)), static_cast<float *>(dH.get(sizeof(float) * 16 * px)),
                                gw.as<float>(), 0));
        CU(cudaDeviceSynchronize());
        CU(cudaMemcpy(loss, dl.p, sizeof(float), cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(grad, gw.p, sizeof(float) * kProposalWeightCount, cudaMemcpyDeviceToHost));
        return (int)BM3D_OK;
    });
}

// Trains the proposal network on nframes GRAY planes [n][height][width] (host, float): per
// iteration `batch` triplets (reference block on the block-step-4 lattice, one of the first 16
// entries of its exhaustive 32-list, and either a later entry or a uniform candidate of its +-16
// window), logistic ranking loss, Adam.
// weights: initial values in, trained values out; losses[iters]: the mean loss per iteration.
BM3D_API int bm3d_proposal_train(const float *frames, int nframes, int width, int height, int iters, int batch, float lr,
                                 uint64_t seed, float *weights, float *losses)
{
    g_error.clear();
    if (!frames || nframes < 1 || width < 48 || height < 48 || iters < 1 || batch < 1 || !weights || !losses)
        return fail(BM3D_ERR_STATE, "bad arguments");
    return guarded([&]() -> int {
        const int W = width, H = height, Wd = W - 7, Hd = H - 7, G = 32, R = 16, step = 4;
        const size_t px = (size_t)W * H, npos = (size_t)Wd * Hd;
        const long long fs = (long long)px;
        DevBuf x, wt, mo, vo, gw, tr, gD, dF, dH, dl, hidall, feat, rs, desc, lp, ln, dsy, dsx;
        CU(cudaMemcpy(x.get(sizeof(float) * px * nframes), frames, sizeof(float) * px * nframes, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(wt.get(sizeof(float) * kProposalWeightCount), weights, sizeof(float) * kProposalWeightCount, cudaMemcpyHostToDevice));
        CU(cudaMemset(mo.get(sizeof(float) * kProposalWeightCount), 0, sizeof(float) * kProposalWeightCount));
        CU(cudaMemset(vo.get(sizeof(float) * kProposalWeightCount), 0, sizeof(float) * kProposalWeightCount));
        CU(cudaMemset(dl.get(sizeof(float) * iters), 0, sizeof(float) * iters));
        const std::vector<int> syh = scan_positions(H, 8, step), sxh = scan_positions(W, 8, step);
        CU(cudaMemcpy(dsy.get(sizeof(int) * syh.size()), syh.data(), sizeof(int) * syh.size(), cudaMemcpyHostToDevice));
        CU(cudaMemcpy(dsx.get(sizeof(int) * sxh.size()), sxh.data(), sizeof(int) * sxh.size(), cudaMemcpyHostToDevice));
        const int nby = (int)syh.size(), nbx = (int)sxh.size();
        const size_t nb = (size_t)nby * nbx * nframes;
        exhaustive_lists(x.as<float>(), fs, W, W, H, nframes, step, G, R, 3.0e38f, dsy.as<int>(), dsx.as<int>(), nby, nbx,
                         static_cast<uint32_t *>(lp.get(sizeof(uint32_t) * nb * G)), static_cast<int *>(ln.get(sizeof(int) * nb)),
                         nullptr, 0, 0);
        unsigned char *hid = static_cast<unsigned char *>(hidall.get(2 * 16 * px * nframes));
        unsigned char *dsc = static_cast<unsigned char *>(desc.get(2 * 16 * npos * nframes));
        float *g = static_cast<float *>(gD.get(sizeof(float) * 16 * npos * nframes));
        tr.get((size_t)prop_triplet_bytes() * batch);
        float b1t = 1.0f, b2t = 1.0f;
        for (int it = 0; it < iters; ++it) {
            for (int k = 0; k < nframes; ++k)
                CU(launch_prop_features(x.as<float>() + k * fs, W, W, H, wt.as<float>(), hid + 2 * 16 * px * k,
                                        feat.get(2 * 16 * px), static_cast<float *>(rs.get(sizeof(float) * 16 * (size_t)H * (W - 3))),
                                        dsc + 2 * 16 * npos * k, 0));
            CU(launch_prop_sample(x.as<float>(), fs, W, W, H, nframes, lp.as<uint32_t>(), ln.as<int>(), G, dsy.as<int>(),
                                  dsx.as<int>(), nby, nbx, R, (uint32_t)(seed * 1000003ull + (uint64_t)it), tr.p, batch, 0));
            CU(cudaMemsetAsync(g, 0, sizeof(float) * 16 * npos * nframes, 0));
            CU(cudaMemsetAsync(gw.get(sizeof(float) * kProposalWeightCount), 0, sizeof(float) * kProposalWeightCount, 0));
            CU(launch_prop_loss(tr.p, batch, dsc, (long long)npos, Wd, g, 1.0f / batch, dl.as<float>() + it, 0));
            for (int k = 0; k < nframes; ++k)
                CU(launch_prop_backward(x.as<float>() + k * fs, W, W, H, wt.as<float>(), hid + 2 * 16 * px * k, g + 16 * npos * k,
                                        static_cast<float *>(dF.get(sizeof(float) * 16 * px)),
                                        static_cast<float *>(dH.get(sizeof(float) * 16 * px)), gw.as<float>(), 0));
            b1t *= 0.9f;
            b2t *= 0.999f;
            CU(launch_prop_adam(wt.as<float>(), gw.as<float>(), mo.as<float>(), vo.as<float>(), lr, b1t, b2t, 0));
        }
        CU(cudaDeviceSynchronize());
        CU(cudaMemcpy(weights, wt.p, sizeof(float) * kProposalWeightCount, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(losses, dl.p, sizeof(float) * iters, cudaMemcpyDeviceToHost));
        return (int)BM3D_OK;
    });
}

// Lists of one GRAY plane (block step `step`, group G, range R, candidate step 1, threshold
// th_sse on the exact SSD): exhaustive when weights is null, else the learned proposals (the
// best nprop candidates by descriptor distance, re-ranked exactly).  counts[nblocks], ys/xs
// [nblocks][G]; returns the number of reference blocks.
BM3D_API int bm3d_proposal_match(const float *frame, int width, int height, const float *weights, int step, int G, int R,
                                 float th_sse, int nprop, int *counts, int *ys, int *xs, int capacity)
{
    g_error.clear();
    if (!frame || !counts || !ys || !xs || width < 8 || height < 8 || G < 1 || G > 32 || R < 1 || step < 1 || nprop < 1 ||
        nprop > 128)
        return fail(BM3D_ERR_STATE, "bad arguments");
    return guarded([&]() -> int {
        const std::vector<int> syh = scan_positions(height, 8, step), sxh = scan_positions(width, 8, step);
        const int nby = (int)syh.size(), nbx = (int)sxh.size(), nb = nby * nbx;
        if (nb > capacity) throw std::runtime_error("capacity too small");
        DevBuf x, wt, dsy, dsx, lp, ln;
        PropBuffers pb;
        CU(cudaMemcpy(x.get(sizeof(float) * width * height), frame, sizeof(float) * width * height, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(dsy.get(sizeof(int) * nby), syh.data(), sizeof(int) * nby, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(dsx.get(sizeof(int) * nbx), sxh.data(), sizeof(int) * nbx, cudaMemcpyHostToDevice));
        const void *desc = nullptr;
        if (weights) {
            CU(cudaMemcpy(wt.get(sizeof(float) * kProposalWeightCount), weights, sizeof(float) * kProposalWeightCount, cudaMemcpyHostToDevice));
            prop_descriptors(x.as<float>(), 0, width, width, height, 1, wt.as<float>(), pb, 0);
            desc = pb.desc.p;
        }
        exhaustive_lists(x.as<float>(), 0, width, width, height, 1, step, G, R, th_sse, dsy.as<int>(), dsx.as<int>(), nby, nbx,
                         static_cast<uint32_t *>(lp.get(sizeof(uint32_t) * nb * G)), static_cast<int *>(ln.get(sizeof(int) * nb)),
                         desc, nprop, 0);
        std::vector<uint32_t> P((size_t)nb * G);
        CU(cudaDeviceSynchronize());
        CU(cudaMemcpy(counts, ln.p, sizeof(int) * nb, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(P.data(), lp.p, sizeof(uint32_t) * P.size(), cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < P.size(); ++i) {
            ys[i] = (int)unpack_y(P[i]);
            xs[i] = (int)unpack_x(P[i]);
        }
        return nb;
    });
}

// Proposal sets of the learned matching of one GRAY plane (candidate step 1): for every reference
// block (block step `step`, range R) the indices, in raster order of its search window, of the
// nprop candidates it re-ranks exactly; unused slots 0xffffffff.  *overflow_blocks receives the
// number of blocks whose cut needed the exact selection.
BM3D_API int bm3d_debug_proposal_sets(const float *frame, int width, int height, const float *weights, int step, int R,
                                      int nprop, uint32_t *sets, int64_t *overflow_blocks, int capacity)
{
    g_error.clear();
    if (!frame || !weights || !sets || width < 8 || height < 8 || R < 1 || step < 1 || nprop < 1 || nprop > 128)
        return fail(BM3D_ERR_STATE, "bad arguments");
    return guarded([&]() -> int {
        const std::vector<int> syh = scan_positions(height, 8, step), sxh = scan_positions(width, 8, step);
        const int nby = (int)syh.size(), nbx = (int)sxh.size(), nb = nby * nbx;
        if (nb > capacity) throw std::runtime_error("capacity too small");
        const int G = 2;
        DevBuf x, wt, dsy, dsx, lp, ln, pp, st;
        PropBuffers pb;
        CU(cudaMemcpy(x.get(sizeof(float) * width * height), frame, sizeof(float) * width * height, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(dsy.get(sizeof(int) * nby), syh.data(), sizeof(int) * nby, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(dsx.get(sizeof(int) * nbx), sxh.data(), sizeof(int) * nbx, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(wt.get(sizeof(float) * kProposalWeightCount), weights, sizeof(float) * kProposalWeightCount, cudaMemcpyHostToDevice));
        CU(cudaMemset(st.get(4 * sizeof(unsigned long long)), 0, 4 * sizeof(unsigned long long)));
        prop_descriptors(x.as<float>(), 0, width, width, height, 1, wt.as<float>(), pb, 0);
        exhaustive_lists(x.as<float>(), 0, width, width, height, 1, step, G, R, 1e30f, dsy.as<int>(), dsx.as<int>(), nby, nbx,
                         static_cast<uint32_t *>(lp.get(sizeof(uint32_t) * nb * G)), static_cast<int *>(ln.get(sizeof(int) * nb)),
                         pb.desc.p, nprop, 0, static_cast<uint32_t *>(pp.get(sizeof(uint32_t) * (size_t)nb * nprop)),
                         static_cast<unsigned long long *>(st.p));
        CU(cudaDeviceSynchronize());
        CU(cudaMemcpy(sets, pp.p, sizeof(uint32_t) * (size_t)nb * nprop, cudaMemcpyDeviceToHost));
        unsigned long long h[4];
        CU(cudaMemcpy(h, st.p, sizeof(h), cudaMemcpyDeviceToHost));
        if (overflow_blocks) *overflow_blocks = (int64_t)h[1];
        return nb;
    });
}

BM3D_API int bm3d_debug_dct3d(float *groups, int ngroups, int n, int B, int inverse, int fast)
{
    g_error.clear();
    if (!groups || ngroups < 1 || n < 1 || n > 256 || B < 1 || B > 64) return fail(BM3D_ERR_STATE, "bad arguments");
    return guarded([&]() -> int {
        const DeviceTables &dt = device_tables();
        DirectTables d;
        build_direct_tables(d, std::vector<int>{n, B});
        DevBuf buf;
        const size_t bytes = sizeof(float) * (size_t)ngroups * n * B * B;
        float *dp = static_cast<float *>(buf.get(bytes));
        CU(cudaMemcpy(dp, groups, bytes, cudaMemcpyHostToDevice));
        CU(launch_dct3d_test(dp, ngroups, n, B, inverse, fast, dt.odd_all, d.tab.as<float>(), d.off.as<int>(), 0));
        CU(cudaDeviceSynchronize());
        CU(cudaMemcpy(groups, dp, bytes, cudaMemcpyDeviceToHost));
        return (int)BM3D_OK;
    });
}

}  // extern "C"
