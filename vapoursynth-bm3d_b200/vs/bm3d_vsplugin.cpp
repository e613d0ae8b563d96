// bm3d_vsplugin.cpp -- VapourSynth (API 4) adapter over the C ABI of include/bm3d_b200.h.
//
// Registers the reference plugin's identity and its seven functions with the same argument
// specifications (source/VSPlugin.cpp:424-518): id "com.vapoursynth.bm3d", namespace "bm3d",
// version 10.1; RGB2OPP, OPP2RGB, Basic, Final, VBasic, VFinal, VAggregate.  Scripts that call
// core.bm3d.* (and wrappers such as mvsfunc.BM3D) run unchanged on the GPU library.
//
// Every function goes through one generic path:
//   create   VSMap arguments -> bm3d_map (same names and types) -> bm3d_create; an argument error
//            is reported with mapSetError and the library's reference-identical message
//            ("bm3d.<Func>: ..."); the output VSVideoInfo comes from bm3d_output_info.
//   getFrame arInitial: the frames bm3d_frame_window names (the +-radius window of VBasic /
//            VFinal / VAggregate, source/VSPlugin.cpp:238-263); arAllFramesReady: the planes of
//            those frames are handed to bm3d_get_frames as host memory together with the frame
//            properties the reference reads (BM3D_OPP, _Range, _Matrix, BM3D_V_radius,
//            BM3D_V_process), and the properties it writes or deletes are applied to the new
//            frame (whose other properties come from the source frame, as in the reference).
//   free     bm3d_free, then the nodes.
// Warnings the library logs (the reference's logMessage(mtWarning, ...)) go to the core's log.
//
// The filter objects of the library keep device workspaces and are not meant for concurrent
// calls, so the functions are created with fmParallelRequests and each instance serialises its
// frame computations with a mutex; the GPU work of one frame is itself fully parallel.
//
// Built only where the VapourSynth SDK header (VapourSynth4.h) is installed: build.py compiles
// this file into lib/libbm3d_vs.so, linked against lib/libbm3d_b200.so.

#include <VapourSynth4.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "bm3d_b200.h"

namespace {

// the core whose script is calling into the library on this thread (for the log callback)
struct LogTarget {
    const VSAPI *vsapi = nullptr;
    VSCore *core = nullptr;
};
thread_local LogTarget t_log;

void log_to_core(int, const char *msg, void *)
{
    if (t_log.vsapi && t_log.core) t_log.vsapi->logMessage(mtWarning, msg, t_log.core);
}

struct LogScope {
    LogScope(const VSAPI *api, VSCore *core) { t_log.vsapi = api; t_log.core = core; }
    ~LogScope() { t_log = LogTarget(); }
};

struct Instance {
    std::string name;
    bm3d_filter *filter = nullptr;
    VSNode *input = nullptr;
    VSNode *ref = nullptr;
    VSVideoInfo vi{};          // output
    std::mutex lock;
};

bm3d_video_info to_info(const VSVideoInfo *vi)
{
    bm3d_video_info b{};
    b.color_family = vi->format.colorFamily;
    b.sample_type = vi->format.sampleType;
    b.bits_per_sample = vi->format.bitsPerSample;
    b.subsampling_w = vi->format.subSamplingW;
    b.subsampling_h = vi->format.subSamplingH;
    b.width = vi->width;
    b.height = vi->height;
    b.num_frames = vi->numFrames;
    return b;
}

int64_t prop_int(const VSAPI *vsapi, const VSMap *m, const char *key)
{
    int err = 0;
    const int64_t v = vsapi->mapGetInt(m, key, 0, &err);
    return err ? -1 : v;
}

// The frame's planes (host memory) and the properties the library reads.
bm3d_frame to_frame(const VSAPI *vsapi, const VSFrame *f, int planes)
{
    bm3d_frame b{};
    for (int p = 0; p < planes; ++p) {
        b.data[p] = const_cast<uint8_t *>(vsapi->getReadPtr(f, p));
        b.stride[p] = vsapi->getStride(f, p);
    }
    b.memory = BM3D_MEM_HOST;
    const VSMap *m = vsapi->getFramePropertiesRO(f);
    b.prop_bm3d_opp = prop_int(vsapi, m, "BM3D_OPP");
    b.prop_range = prop_int(vsapi, m, "_Range");
    b.prop_matrix = prop_int(vsapi, m, "_Matrix");
    b.prop_v_radius = prop_int(vsapi, m, "BM3D_V_radius");
    const int nv = vsapi->mapNumElements(m, "BM3D_V_process");
    b.prop_v_process_count = nv < 0 ? -1 : nv;
    for (int i = 0; i < nv && i < 3; ++i) {
        int err = 0;
        b.prop_v_process[i] = vsapi->mapGetInt(m, "BM3D_V_process", i, &err);
    }
    return b;
}

void set_or_delete(const VSAPI *vsapi, VSMap *m, const char *key, int64_t v)
{
    if (v < 0) vsapi->mapDeleteKey(m, key);
    else vsapi->mapSetInt(m, key, v, maReplace);
}

const VSFrame *VS_CC get_frame(int n, int reason, void *data, void **, VSFrameContext *ctx, VSCore *core,
                               const VSAPI *vsapi)
{
    Instance *d = static_cast<Instance *>(data);
    int first = 0, num = 0;
    if (bm3d_frame_window(d->filter, n, 1, &first, &num) != BM3D_OK) {
        vsapi->setFilterError(bm3d_get_error(), ctx);
        return nullptr;
    }
    if (reason == arInitial) {
        for (int i = first; i < first + num; ++i) {
            vsapi->requestFrameFilter(i, d->input, ctx);
            if (d->ref) vsapi->requestFrameFilter(i, d->ref, ctx);
        }
        return nullptr;
    }
    if (reason != arAllFramesReady) return nullptr;

    const VSVideoInfo *ivi = vsapi->getVideoInfo(d->input);
    const int in_planes = ivi->format.numPlanes;
    std::vector<const VSFrame *> sf(num), rf(d->ref ? num : 0);
    std::vector<bm3d_frame> sb(num), rb(d->ref ? num : 0);
    std::vector<const bm3d_frame *> sp(num), rp(d->ref ? num : 0);
    for (int i = 0; i < num; ++i) {
        sf[i] = vsapi->getFrameFilter(first + i, d->input, ctx);
        sb[i] = to_frame(vsapi, sf[i], in_planes);
        sp[i] = &sb[i];
        if (d->ref) {
            rf[i] = vsapi->getFrameFilter(first + i, d->ref, ctx);
            rb[i] = to_frame(vsapi, rf[i], in_planes);
            rp[i] = &rb[i];
        }
    }
    // the output frame takes the source frame's properties, then the library's changes
    VSFrame *dst = vsapi->newVideoFrame(&d->vi.format, d->vi.width, d->vi.height, sf[n - first], core);
    bm3d_frame db{};
    for (int p = 0; p < d->vi.format.numPlanes; ++p) {
        db.data[p] = vsapi->getWritePtr(dst, p);
        db.stride[p] = vsapi->getStride(dst, p);
    }
    db.memory = BM3D_MEM_HOST;
    bm3d_frame *dp = &db;
    int rc;
    {
        std::lock_guard<std::mutex> lk(d->lock);
        LogScope ls(vsapi, core);
        rc = bm3d_get_frames(d->filter, n, 1, sp.data(), d->ref ? rp.data() : nullptr, &dp);
    }
    for (const VSFrame *f : sf) vsapi->freeFrame(f);
    for (const VSFrame *f : rf) vsapi->freeFrame(f);
    if (rc != BM3D_OK) {
        vsapi->freeFrame(dst);
        vsapi->setFilterError(bm3d_get_error(), ctx);
        return nullptr;
    }
    VSMap *m = vsapi->getFramePropertiesRW(dst);
    set_or_delete(vsapi, m, "BM3D_OPP", db.prop_bm3d_opp);
    set_or_delete(vsapi, m, "_Range", db.prop_range);
    set_or_delete(vsapi, m, "_Matrix", db.prop_matrix);
    set_or_delete(vsapi, m, "BM3D_V_radius", db.prop_v_radius);
    if (db.prop_v_process_count < 0) vsapi->mapDeleteKey(m, "BM3D_V_process");
    else vsapi->mapSetIntArray(m, "BM3D_V_process", db.prop_v_process, db.prop_v_process_count);
    return dst;
}

void VS_CC free_instance(void *data, VSCore *, const VSAPI *vsapi)
{
    Instance *d = static_cast<Instance *>(data);
    if (d->filter) bm3d_free(d->filter);
    if (d->input) vsapi->freeNode(d->input);
    if (d->ref) vsapi->freeNode(d->ref);
    delete d;
}

// One create function for the seven: userData is the function name.
void VS_CC create(const VSMap *in, VSMap *out, void *user, VSCore *core, const VSAPI *vsapi)
{
    const char *name = static_cast<const char *>(user);
    Instance *d = new Instance;
    d->name = name;
    bm3d_map *m = bm3d_map_create();
    const int nkeys = vsapi->mapNumKeys(in);
    for (int k = 0; k < nkeys; ++k) {
        const char *key = vsapi->mapGetKey(in, k);
        const int ne = vsapi->mapNumElements(in, key);
        int err = 0;
        switch (vsapi->mapGetType(in, key)) {
        case ptInt:
            for (int i = 0; i < ne; ++i) bm3d_map_set_int(m, key, vsapi->mapGetInt(in, key, i, &err));
            break;
        case ptFloat:
            for (int i = 0; i < ne; ++i) bm3d_map_set_float(m, key, vsapi->mapGetFloat(in, key, i, &err));
            break;
        case ptData:
            for (int i = 0; i < ne; ++i) bm3d_map_set_data(m, key, vsapi->mapGetData(in, key, i, &err));
            break;
        case ptVideoNode: {
            VSNode *node = vsapi->mapGetNode(in, key, 0, &err);
            const bm3d_video_info bi = to_info(vsapi->getVideoInfo(node));
            bm3d_map_set_clip(m, key, &bi);
            if (!std::strcmp(key, "input")) d->input = node;
            else if (!std::strcmp(key, "ref")) d->ref = node;
            else vsapi->freeNode(node);
            break;
        }
        default:
            break;
        }
    }
    int rc;
    {
        LogScope ls(vsapi, core);
        rc = bm3d_create(name, m, &d->filter);
    }
    bm3d_map_free(m);
    if (rc != BM3D_OK) {
        vsapi->mapSetError(out, bm3d_get_error());
        free_instance(d, core, vsapi);
        return;
    }
    bm3d_video_info o{};
    bm3d_output_info(d->filter, &o);
    d->vi = *vsapi->getVideoInfo(d->input);      // frame rate and length of the input
    if (!vsapi->queryVideoFormat(&d->vi.format, o.color_family, o.sample_type, o.bits_per_sample, o.subsampling_w,
                                 o.subsampling_h, core)) {
        vsapi->mapSetError(out, ("bm3d." + d->name + ": output format not available").c_str());
        free_instance(d, core, vsapi);
        return;
    }
    d->vi.width = o.width;
    d->vi.height = o.height;
    d->vi.numFrames = o.num_frames;
    // spatial functions need exactly frame n; the V-BM3D ones a window (source/VSPlugin.cpp:77-416)
    const bool temporal = !std::strcmp(name, "VBasic") || !std::strcmp(name, "VFinal") || !std::strcmp(name, "VAggregate");
    std::vector<VSFilterDependency> deps{{d->input, temporal ? rpGeneral : rpStrictSpatial}};
    if (d->ref) deps.push_back({d->ref, temporal ? rpGeneral : rpStrictSpatial});
    vsapi->createVideoFilter(out, name, &d->vi, get_frame, free_instance, fmParallelRequests, deps.data(),
                             (int)deps.size(), d, core);
}

}  // namespace

VS_EXTERNAL_API(void) VapourSynthPluginInit2(VSPlugin *plugin, const VSPLUGINAPI *vspapi)
{
    vspapi->configPlugin("com.vapoursynth.bm3d", "bm3d", "Implementation of BM3D denoising filter for VapourSynth.",
                         VS_MAKE_VERSION(10, 1), VAPOURSYNTH_API_VERSION, 0, plugin);
    bm3d_set_log_callback(log_to_core, nullptr);
    // argument lists of source/VSPlugin.cpp:430-517; "precision" (and, for VBasic / VFinal,
    // "aggregate" / "sample") are this library's extensions
    static const char *const conv = "input:vnode;sample:int:opt;";
    static const char *const common = "profile:data:opt;sigma:float[]:opt;";
    static const char *const shape = "block_size:int:opt;block_step:int:opt;group_size:int:opt;bm_range:int:opt;bm_step:int:opt;";
    static const char *const pred = "ps_num:int:opt;ps_range:int:opt;ps_step:int:opt;";
    static const std::string basic = std::string("input:vnode;ref:vnode:opt;") + common + shape +
                                     "th_mse:float:opt;hard_thr:float:opt;matrix:int:opt;precision:data:opt;";
    static const std::string fin = std::string("input:vnode;ref:vnode;") + common + shape +
                                   "th_mse:float:opt;matrix:int:opt;precision:data:opt;";
    static const std::string vbasic = std::string("input:vnode;ref:vnode:opt;") + common + "radius:int:opt;" + shape + pred +
                                      "th_mse:float:opt;hard_thr:float:opt;matrix:int:opt;precision:data:opt;"
                                      "aggregate:int:opt;sample:int:opt;";
    static const std::string vfinal = std::string("input:vnode;ref:vnode;") + common + "radius:int:opt;" + shape + pred +
                                      "th_mse:float:opt;matrix:int:opt;precision:data:opt;aggregate:int:opt;sample:int:opt;";
    static const char *const vagg = "input:vnode;radius:int:opt;sample:int:opt;";
    static char n_rgb2opp[] = "RGB2OPP", n_opp2rgb[] = "OPP2RGB", n_basic[] = "Basic", n_final[] = "Final",
                n_vbasic[] = "VBasic", n_vfinal[] = "VFinal", n_vagg[] = "VAggregate";
    vspapi->registerFunction(n_rgb2opp, conv, "clip:vnode;", create, n_rgb2opp, plugin);
    vspapi->registerFunction(n_opp2rgb, conv, "clip:vnode;", create, n_opp2rgb, plugin);
    vspapi->registerFunction(n_basic, basic.c_str(), "clip:vnode;", create, n_basic, plugin);
    vspapi->registerFunction(n_final, fin.c_str(), "clip:vnode;", create, n_final, plugin);
    vspapi->registerFunction(n_vbasic, vbasic.c_str(), "clip:vnode;", create, n_vbasic, plugin);
    vspapi->registerFunction(n_vfinal, vfinal.c_str(), "clip:vnode;", create, n_vfinal, plugin);
    vspapi->registerFunction(n_vagg, vagg, "clip:vnode;", create, n_vagg, plugin);
}
