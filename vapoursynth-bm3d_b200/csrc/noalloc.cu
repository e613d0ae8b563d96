// noalloc.cu -- bm3d_basic_noalloc: the Basic estimate of one float plane with no device
// allocation at all.
//
// Some callers cannot let a library call cudaMalloc.  Media servers and plugin hosts often hand
// all of a GPU's memory to their own pool allocator when they start, so an allocation from
// outside that pool fails or breaks their memory accounting; real-time pipelines forbid
// cudaMalloc / cudaFree because those calls synchronise the whole device and stall every other
// stream.  The filter objects of host.cpp allocate their workspaces on first use, so such callers
// cannot use them.  This entry point runs the same kernels (block matching, collaborative filter,
// normalisation) on work buffers carved out of one file-scope device array that is part of the
// library's device image: a call allocates nothing.
//
// The array has a fixed size, kScratchBytes (48 MiB: a 1920x1080 plane at every profile fits),
// and every GPU that loads the library's device code holds it until the process exits.  All calls
// share it and it keeps the contents of the last call, so each call clears the accumulators that
// must start at zero, and two calls that overlap on the GPU (different streams, or threads that
// do not order their calls) race with each other.  The set-up of a device (the array's address
// and the constant tables) is done once per process: a caller that resets the device
// (cudaDeviceReset) after its first call gets a reloaded, zeroed array and must not call again.

#include "bm3d_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "launch.h"
#include "params.h"

static constexpr size_t kScratchBytes = size_t(48) << 20;
static constexpr long long kScratchFloats = (long long)(kScratchBytes / sizeof(float));

// The work buffers of every call.  In host code this name is only a stand-in for the device
// array; the device address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) float g_noalloc_scratch[kScratchFloats];

namespace bm3d {

// error text for bm3d_get_error (host.cpp)
int set_error(int code, const std::string &msg);
void clear_error();

namespace {

// Layout of the array, in floats; every region starts on a 256-byte boundary.
//   [0, 320)              int offsets of the direct DCT tables, indexed by length N (-1: none)
//   [320, kTableFloats)   direct DCT tables (forward then inverse) of every non-power-of-two
//                         length up to the largest Basic group size, 32
//   then per call: input plane copy, numerator, weight map (each H x ld), match positions,
//   match counts, row and column scan positions.
constexpr int kMaxGroup = 32;
constexpr int kOffFloats = 320;
constexpr long long kTableFloats = 20480;
constexpr int kMaxDevices = 64;

long long round64(long long n) { return (n + 63) / 64 * 64; }

std::mutex g_setup_mutex;
float *g_dev_scratch[kMaxDevices];       // device address of the array, per device (set-up done)

// Host image of the table region and of the constant odd tables (N = 2..64), built once.
float g_table_image[kTableFloats];
float g_odd_image[1365];
bool g_images_ready = false;

void build_images()
{
    int off[kMaxGroup + 1];
    long long pos = kOffFloats;
    for (int N = 0; N <= kMaxGroup; ++N) {
        off[N] = -1;
        if (N < 1 || (N & (N - 1)) == 0) continue;
        off[N] = (int)(pos - kOffFloats);
        for (int k = 0; k < N; ++k)
            for (int j = 0; j < N; ++j) g_table_image[pos++] = cos2((long)(2 * j + 1) * k, 2L * N);
        for (int k = 0; k < N; ++k)
            for (int j = 0; j < N; ++j) g_table_image[pos++] = cos2((long)j * (2 * k + 1), 2L * N);
    }
    for (int N = 0; N < kOffFloats; ++N) {
        const int v = N <= kMaxGroup ? off[N] : -1;
        std::memcpy(&g_table_image[N], &v, sizeof(int));
    }
    int o = 0;
    for (int N = 2; N <= 64; N *= 2) {
        const int h = N / 2;
        for (int m = 0; m < h; ++m)
            for (int j = 0; j < h; ++j) g_odd_image[o + m * h + j] = cos2((long)(2 * j + 1) * (2 * m + 1), 2L * N);
        o += h * h;
    }
    g_images_ready = true;
}

std::string cuda_text(const char *what, cudaError_t e)
{
    return std::string("bm3d_basic_noalloc: ") + what + " failed: " + cudaGetErrorString(e);
}

// Set-up of the current device, once: look up the array's device address and fill the constant
// tables (synchronous copies).
int setup_device(int dev, float **out)
{
    std::lock_guard<std::mutex> lk(g_setup_mutex);
    if (g_dev_scratch[dev]) {
        *out = g_dev_scratch[dev];
        return BM3D_OK;
    }
    if (!g_images_ready) build_images();
    float *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return set_error(BM3D_ERR_CUDA, cuda_text("cudaGetSymbolAddress", e));
    if ((e = upload_odd_tables(g_odd_image)) != cudaSuccess) return set_error(BM3D_ERR_CUDA, cuda_text("table upload", e));
    if ((e = cudaMemcpy(ptr, g_table_image, sizeof(g_table_image), cudaMemcpyHostToDevice)) != cudaSuccess)
        return set_error(BM3D_ERR_CUDA, cuda_text("table upload", e));
    g_dev_scratch[dev] = ptr;
    *out = ptr;
    return BM3D_OK;
}

// Number of reference-block positions along one axis: the clamped scan of
// source/BM3D_Base.cpp:421-443 (0, step, 2*step, ..., then extent - B).
int scan_count(int extent, int B, int step)
{
    const int last = extent - B;
    int n = 0;
    for (int j = 0;; j += step) {
        if (j >= last + step) break;
        if (j > last) j = last;
        ++n;
    }
    return n;
}

__global__ void noalloc_scan_kernel(int *sy, int ny, int lasty, int *sx, int nx, int lastx, int step)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ny) sy[i] = min(i * step, lasty);
    if (i < nx) sx[i] = min(i * step, lastx);
}

}  // namespace
}  // namespace bm3d

using namespace bm3d;

extern "C" BM3D_API int bm3d_basic_noalloc(const float *src, float *dst, int width, int height, int64_t stride,
                                           const char *profile, double sigma, void *stream)
{
    clear_error();
    const char *prof = profile ? profile : "fast";
    if (std::strcmp(prof, "fast") && std::strcmp(prof, "lc") && std::strcmp(prof, "np") && std::strcmp(prof, "high") &&
        std::strcmp(prof, "vn"))
        return set_error(BM3D_ERR_ARG, "bm3d_basic_noalloc: Unrecognized \"profile\" specified, should be \"fast\", \"lc\", \"np\", \"high\" or \"vn\"");
    if (!(sigma >= 0.0))
        return set_error(BM3D_ERR_ARG, "bm3d_basic_noalloc: Invalid \"sigma\" assigned, must be a non-negative floating point number");
    const Params para = bm3d_profile(false, prof);
    const int B = para.B, G = para.G;
    if (width < B || height < B || width > 65535 || height > 65535)
        return set_error(BM3D_ERR_ARG, "bm3d_basic_noalloc: width and height must be in [8, 65535]");
    if (stride < (int64_t)width * 4 || stride % 4 != 0)
        return set_error(BM3D_ERR_ARG, "bm3d_basic_noalloc: stride must be a multiple of 4 bytes and at least width * 4");
    if (!src || !dst) return set_error(BM3D_ERR_STATE, "bm3d_basic_noalloc: src and dst must be device pointers");

    // scratch layout of this call, checked against the fixed size before anything runs
    const int ld = (width + 31) / 32 * 32;
    const long long P = (long long)height * ld;
    const int nby = scan_count(height, B, para.step), nbx = scan_count(width, B, para.step);
    const long long nb = (long long)nby * nbx;
    const long long o_src = kTableFloats;
    const long long o_num = o_src + round64(P);
    const long long o_wm = o_num + round64(P);
    const long long o_pos = o_wm + round64(P);
    const long long o_cnt = o_pos + round64(nb * G);
    const long long o_sy = o_cnt + round64(nb);
    const long long o_sx = o_sy + round64(nby);
    const long long need = o_sx + round64(nbx);
    if (need > kScratchFloats) {
        char msg[256];
        std::snprintf(msg, sizeof msg,
                      "bm3d_basic_noalloc: a %dx%d plane with profile \"%s\" needs %.1f MiB of scratch, more than the "
                      "fixed %zu MiB (a 1920x1080 plane fits at every profile)",
                      width, height, prof, need * 4.0 / 1048576.0, kScratchBytes >> 20);
        return set_error(BM3D_ERR_UNSUPPORTED, msg);
    }

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(BM3D_ERR_CUDA, cuda_text("cudaGetDevice", e));
    if (dev < 0 || dev >= kMaxDevices) return set_error(BM3D_ERR_UNSUPPORTED, "bm3d_basic_noalloc: device ordinal beyond 63");
    float *base = nullptr;
    if (int r = setup_device(dev, &base)) return r;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    if (sigma == 0.0) {
        // nothing to process: the reference returns the source frame
        e = cudaMemcpy2DAsync(dst, (size_t)stride, src, (size_t)stride, (size_t)width * 4, height, cudaMemcpyDeviceToDevice, s);
        return e == cudaSuccess ? (int)BM3D_OK : set_error(BM3D_ERR_CUDA, cuda_text("copy", e));
    }

    // filter constants of a GRAY clip with the default matrix (BM3D_Data_Base::arguments_process
    // and init_filter_data, source/BM3D_Base.cpp:32-283)
    double norm[3];
    matrix_norms(matrix_default(width, height), norm);
    const double thMSE = thmse_default(false, para.profile, sigma) * norm[0];
    const double MSE2SSE = static_cast<double>(B * B) * 1.0f * 1.0f / double(255 * 255);
    const double plane_sigma = sigma / double(255) * norm[0];

    float *S = base + o_src, *num = base + o_num, *wm = base + o_wm;
    uint32_t *pos = reinterpret_cast<uint32_t *>(base + o_pos);
    int *cnt = reinterpret_cast<int *>(base + o_cnt);
    int *sy = reinterpret_cast<int *>(base + o_sy), *sx = reinterpret_cast<int *>(base + o_sx);

    if ((e = cudaMemcpy2DAsync(S, (size_t)ld * 4, src, (size_t)stride, (size_t)width * 4, height, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
        return set_error(BM3D_ERR_CUDA, cuda_text("input copy", e));
    // the accumulators keep the previous call's sums: clear them
    if ((e = cudaMemsetAsync(num, 0, sizeof(float) * P, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(wm, 0, sizeof(float) * P, s)) != cudaSuccess)
        return set_error(BM3D_ERR_CUDA, cuda_text("accumulator clear", e));
    const int nscan = std::max(nby, nbx);
    count_launch();
    noalloc_scan_kernel<<<(nscan + 255) / 256, 256, 0, s>>>(sy, nby, height - B, sx, nbx, width - B, para.step);
    if ((e = cudaGetLastError()) != cudaSuccess) return set_error(BM3D_ERR_CUDA, cuda_text("scan kernel launch", e));

    // block matching (same launch shape as the filter objects)
    BMArgs ba{};
    ba.ref = S;
    ba.frame_stride = P;
    ba.ld = ld;
    ba.H = height;
    ba.W = width;
    ba.B = B;
    ba.range = para.R / para.bmstep * para.bmstep;
    ba.step = para.bmstep;
    ba.G = G;
    ba.thSSE = static_cast<float>(thMSE * MSE2SSE);
    ba.distMul = double(1) / MSE2SSE;
    ba.scan_y = sy;
    ba.scan_x = sx;
    ba.nby = nby;
    ba.nbx = nbx;
    ba.out_pos = pos;
    ba.out_n = cnt;
    const int lat = 2 * ba.range / ba.step + 1;
    ba.cand_cap = lat * lat + 1;
    ba.win_h = std::min(height, 2 * ba.range + B);
    size_t smem = 0;
    int warps = 8;
    for (; warps >= 1; warps /= 2) {
        ba.warps = warps;
        ba.win_pitch = (std::min(width, (warps - 1) * para.step + 2 * ba.range + B) + 4) | 1;
        smem = sizeof(float) * ((size_t)ba.win_h * ba.win_pitch + (size_t)warps * bm_warp_floats(ba.cand_cap, G, B, false));
        if (smem <= 200 * 1024) break;
    }
    if (warps < 1)
        return set_error(BM3D_ERR_UNSUPPORTED, "bm3d_basic_noalloc: bm_range / block_size too large for the shared-memory search window");
    if ((e = launch_bm_full(ba, 1, smem, s)) != cudaSuccess) return set_error(BM3D_ERR_CUDA, cuda_text("block matching", e));

    // collaborative filter with hard thresholding; per-plane tables of BM3D_FilterData
    // (source/BM3D.cpp:137-209) for the one plane
    CFArgs ca{};
    ca.src[0] = S;
    ca.ref[0] = S;
    ca.num[0] = num;
    ca.wmap[0] = wm;
    ca.process[0] = 1;
    for (int n = 1; n <= G; ++n) {
        const double amp = 2 * n * 2 * B * 2 * B;
        const double thrBase = plane_sigma * para.lambda * std::sqrt(amp);
        ca.thr4[0][n - 1][0] = static_cast<float>(thrBase);
        ca.thr4[0][n - 1][1] = static_cast<float>(thrBase * std::sqrt(double(2)));
        ca.thr4[0][n - 1][2] = static_cast<float>(thrBase * double(2));
        ca.thr4[0][n - 1][3] = static_cast<float>(thrBase * std::sqrt(double(8)));
        ca.amp[n - 1] = static_cast<float>(amp);
    }
    ca.frame_stride = P;
    ca.ld = ld;
    ca.H = height;
    ca.W = width;
    ca.B = B;
    ca.G = G;
    ca.wiener = 0;
    ca.pos = pos;
    ca.count = cnt;
    ca.ngroups = nb;
    ca.blocks_per_frame = nb;
    ca.slots = 1;
    ca.dtab_off = reinterpret_cast<const int *>(base);
    ca.dtab = base + kOffFloats;
    if ((e = launch_cf_fast(ca, s)) != cudaSuccess) return set_error(BM3D_ERR_CUDA, cuda_text("collaborative filter", e));

    // normalisation in place, then the plane out to the caller
    FinalizeArgs fa{};
    fa.process[0] = 1;
    fa.num[0] = num;
    fa.wmap[0] = wm;
    fa.out[0] = num;
    fa.frame_stride = P;
    fa.ld = ld;
    fa.H = height;
    fa.W = width;
    fa.B = B;
    if ((e = launch_finalize(fa, 1, s)) != cudaSuccess) return set_error(BM3D_ERR_CUDA, cuda_text("normalisation", e));
    if ((e = cudaMemcpy2DAsync(dst, (size_t)stride, num, (size_t)ld * 4, (size_t)width * 4, height, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
        return set_error(BM3D_ERR_CUDA, cuda_text("output copy", e));
    return BM3D_OK;
}
