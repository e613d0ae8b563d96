// launch.h -- host-side entry points of the kernel translation unit (kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>
#include "args.h"

namespace bm3d {

// Copies the odd-part DCT tables for N = 2..64 into constant memory of the current device.
cudaError_t upload_odd_tables(const float *host_odd_all);

cudaError_t launch_bm_full(const BMArgs &a, int nframes, size_t smem_bytes, cudaStream_t s);
// Learned proposal (no reference counterpart): feature network forward into bf16 hidden /
// feature planes [16][H][W] (hid, feat), fp32 row sums rs [16][H][W - 7] and bf16 block descriptors
// desc [H - 7][W - 7][16]; ranking loss, backward pass (dF, dH fp32 [16][H][W]; weight gradients
// accumulated into gw), Adam, triplet sampling, and the matching kernel over descriptors.
int prop_triplet_bytes();
cudaError_t launch_prop_features(const float *x, int ld, int W, int H, const float *wt, void *hid, void *feat, float *rs,
                                 void *desc, cudaStream_t s);
cudaError_t launch_prop_loss(const void *triplets, int ntr, const void *desc, long long dstride, int Wd, float *gD,
                             float scale, float *loss, cudaStream_t s);
cudaError_t launch_prop_backward(const float *x, int ld, int W, int H, const float *wt, const void *hid, const float *gD,
                                 float *dF, float *dH, float *gw, cudaStream_t s);
cudaError_t launch_prop_adam(float *wt, const float *g, float *m, float *v, float lr, float b1t, float b2t, cudaStream_t s);
cudaError_t launch_prop_sample(const float *frames, long long fstride, int ld, int W, int H, int nframes, const uint32_t *lists,
                               const int *counts, int G, const int *sy, const int *sx, int nby, int nbx, int range,
                               uint32_t seed, void *out, int ntr, cudaStream_t s);
cudaError_t launch_bm_learned(const BMArgs &a, const void *desc, int nprop, int nframes, size_t smem, cudaStream_t s);

// Precision-form full search (B = 8, candidate step 1, group size <= 32, search windows of
// L.nrc consecutive reference blocks within 64 candidate columns): same lists as launch_bm_full.
cudaError_t launch_bm_tc(const BMArgs &a, const BmtLayout &L, int nframes, cudaStream_t s);
cudaError_t launch_vbm_predict(const VBMArgs &a, int nframes, size_t smem_bytes, cudaStream_t s);
// Fast collaborative filter (B = 8, G in {8, 16, 32}, any group length n <= G); sizes its own
// grid (one CTA per run of consecutive groups); returns cudaErrorInvalidValue for other shapes.
cudaError_t launch_cf_fast(const CFArgs &a, cudaStream_t s);
// Indices of the groups with count < G into list (device counter n, zeroed by the caller).
cudaError_t launch_cf_partial_list(const int *count, long long ngroups, int G, long long *list, unsigned int *n, cudaStream_t s);
cudaError_t launch_cf_generic(const CFArgs &a, int warps, int grid, cudaStream_t s);
cudaError_t launch_convert(const ConvProgram &pr, const PlanePtr *in_dev, const PlanePtr *out_dev,
                           int nframes, cudaStream_t s);
cudaError_t launch_finalize(const FinalizeArgs &a, int nframes, cudaStream_t s);
cudaError_t launch_vaggregate(const VAggArgs &a, int nframes, cudaStream_t s);
cudaError_t launch_vstack(const VStackArgs &a, int nframes, cudaStream_t s);

// Transform-only entry points used by the bit-exactness tests: ngroups groups of n blocks of
// B x B floats (layout [group][z][y][x]) transformed in place.  fast selects the register path
// (B = 8, n in {8, 16, 32}).
cudaError_t launch_dct3d_test(float *data, int ngroups, int n, int B, int inverse, int fast,
                              const float *odd_all, const float *dtab, const int *dtab_off,
                              cudaStream_t s);

int cf_fast_supported(int B, int G);

// Precision form: collaborative filter of the full groups (n == G) on the tensor cores (tf32
// transforms); partial groups are left to launch_cf_fast with skip_full = 1.  `tables` is the
// device copy of the image cf_tc_tables builds for G; *status becomes 1 if a tensor-core wait
// timed out.
int cf_tc_supported(int B, int G);
void cf_tc_tables(int G, std::vector<unsigned char> &img);
void cf_tc_partial_tables(int G, std::vector<float> &out);
// 1 if the tensor-core kernel for (B, G, wiener) also filters the groups of fewer than G blocks
int cf_tc_handles_partial(int B, int G, int wiener);
// Transposed z stage (Wiener filter, B = 8, G = 32): the kernel for the tiles whose groups are all
// full; launch_cf_tile_lists splits the tiles into those and the ones with a short group (device
// lists in ascending order and their counts), for a.tlist / a.tlist_n.
int cf_tc_zt_supported(int B, int G, int wiener);
void cf_tc_zt_tables(int G, std::vector<float> &out);
cudaError_t launch_cf_tile_lists(const int *count, long long ngroups, int G, int *full, unsigned int *nfull,
                                 int *shrt, unsigned int *nshort, int *chunk_counts, cudaStream_t s);
long long cf_tile_chunks(long long ngroups, int G);   // ints of chunk_counts = 2 x this
cudaError_t launch_cf_tc_zt(const CFArgs &a, const void *tables, int *status, cudaStream_t s);
cudaError_t launch_cf_tc(const CFArgs &a, const void *tables, int *status, cudaStream_t s);

// FP64 oracle of the collaborative filter, aggregation and normalisation for the groups of one
// frame (a.ngroups = a.blocks_per_frame); writes num / den into f.num.  Inspection only.
struct F64Args;
size_t cf_fp64_smem(int B, int G);
cudaError_t launch_cf_fp64(const CFArgs &a, const F64Args &f, cudaStream_t s);

// Number of kernels launched by this library since load; count_launch() adds one for a kernel
// launched outside this translation unit.
unsigned long long launch_count();
void count_launch();

}  // namespace bm3d
