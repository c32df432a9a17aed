// Launchers shared between the kernel translation units and the C ABI layer.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "pd_common.cuh"

namespace pd {

constexpr int SEL_THREADS = 256;
constexpr int SEL_PER_THREAD = 4;
constexpr int SEL_BLOCK = SEL_THREADS * SEL_PER_THREAD;

// pd_select.cu
__global__ void k_window_counts(Geo g, const uint8_t* mask4, int32_t* cnt);
__global__ void k_patch_flags(Geo g, int mode, const uint8_t* mask3, const int32_t* cnt, double thr,
                              uint8_t* flags);
__global__ void k_block_counts(const uint8_t* flags, int64_t n, int32_t* bc);
__global__ void k_scan_counts(int32_t* bc, int64_t nb, int32_t* total_out);
__global__ void k_compact(const uint8_t* flags, int64_t n, const int32_t* boff, int32_t* list);

// Per-patch work buffers for one chunk of listed patches.
// Device error word codes (0 = ok): 4-6 a bounded TMA / MMA wait of the tensor-core
// Gram timed out; PD_DEVERR_NONFINITE a processed patch holds a NaN or inf sample.
constexpr int PD_DEVERR_NONFINITE = 7;

// One volume of a batched call (pd_denoise_batch): its geometry, buffers and
// per-volume decision parameters, read by the patch kernels through vol_of.
struct VolDesc {
  Geo g;
  const void* in;
  const double* noise_std;
  void* out;
  float* wacc;
  float* nacc;
  float* nctr;
  int32_t* rank_map;
  int32_t* prank;   // per listed patch of this volume
  float* pnoise;
  double threshold;  // raw
  double mp_median;  // optimal
  int64_t first;     // work-list position of the volume's first patch
};

// Host-built table of a batched call, passed by value to k_batch_setup (the
// volumes are in work-list order: volume v's patches start at d.first).
struct BatchVolume {
  VolDesc d;
  const int32_t* list;  // the volume's selected patches
  int64_t count;
};
struct BatchTable {
  BatchVolume v[PD_BATCH_MAX_VOLUMES];
};
void launch_batch_setup(const BatchTable& t, int nv, int64_t total, VolDesc* vols, int32_t* list, int32_t* vol_of,
                        cudaStream_t s);

struct PatchWork {
  const int32_t* list;  // linear patch indices of the chunk (within their volume)
  int32_t count;        // patches in the chunk
  float* mean;          // [count][n] (complex: 2n floats)
  float* gram;          // [count][gram_stride] packed lower Gram
  int64_t gram_stride;  // floats per patch
  float* vec;           // [count][vec_stride] active eigenvectors, column a at a*2n floats
  int64_t vec_stride;   // floats per patch (2 n n)
  float* coef;          // [count][n] synthesis coefficients
  int32_t* n_active;    // [count]
  int32_t* rank;        // [count] maxidx
  float* noise;         // [count] noise_var (NaN if none)
  double* prior;        // [count] hybrid varest / optimal sigma prior
  int* err;             // device error word (0 = ok)
  int* ctr;             // tile counter of a persistent kernel (zeroed before each launch)
  void* packed;         // mixed precision: bf16 hi/lo operands of the chunk
  int32_t n_stride;     // frames per patch slot of mean / coef (the largest n of a batch)
  const VolDesc* vols;  // batched call: the volumes (NULL: one volume, the launch's Geo)
  const int32_t* vol_of;  // batched call: volume of each chunk patch
};

// pd_gram.cu
void launch_patch_mean(const Geo& g, bool cplx, const void* in, const PatchWork& w, cudaStream_t s);
void launch_prior(const Geo& g, int method, const double* noise_std, const PatchWork& w, cudaStream_t s);
void launch_gram_fp32(const Geo& g, bool cplx, const void* in, const PatchWork& w, cudaStream_t s);

// pd_eig.cu
struct EigParams {
  int method;  // PD_METHOD_*, EIG_MODE_TOP1 (MC threshold) or EIG_MODE_FULL
  int loss;
  int has_prior;
  int rows;  // M
  int cols;  // frames
  double threshold_scale;
  double threshold;
  double mp_median;
  const double* d_threshold;  // raw / NORDIC: read the threshold here when not NULL
  int only_unfinished;        // 1: solve only the patches with n_active < 0 (left by k_sub)
  size_t smem_bytes;          // batched calls: dynamic shared memory for the launch (0: by n)
};
constexpr int EIG_MODE_TOP1 = 100;
// every eigenpair, descending: vectors into w.vec, eigenvalues (true units) into
// w.coef, n_active = n (the backward pass's factorisation)
constexpr int EIG_MODE_FULL = 101;
cudaError_t launch_eig(bool cplx, int n, const EigParams& ep, const PatchWork& w, cudaStream_t s,
                       const pd_adaptive* ad = nullptr);
size_t eig_smem_bytes(bool cplx, int n, bool* in_smem);
// whether k_eig runs patches of n frames in small (128-thread) CTAs, and the
// dynamic shared memory its launch for them takes
bool eig_small(bool cplx, int n);
size_t eig_launch_smem(bool cplx, int n);

// pd_sub.cu: subspace solver of the hard-threshold rule (mixed precision path)
bool sub_supported(bool cplx, int n, int rows);
cudaError_t launch_sub(bool cplx, int n, const EigParams& ep, const PatchWork& w, cudaStream_t s);

// pd_synth.cu
struct SynthArgs {
  int recombination;
  void* out;            // accumulation volume (float or complex)
  float* weight_acc;    // [nvox * gt]
  float* noise_acc;     // [nvox * gt]
  float* noise_ctr;     // 4D
  int32_t* rank_map;    // 4D
  int32_t* patch_rank;  // per listed patch (global list position)
  float* patch_noise;
  int64_t list_offset;  // position of the chunk inside the full list
  int wide;             // high ranks expected (adaptive shrinkage): the grouped-reduction kernel
  int row_blocks;       // CTAs per patch (0: by the patch's rows, at most 8)
};
void launch_synth(const Geo& g, bool cplx, const void* in, const PatchWork& w, const SynthArgs& a,
                  cudaStream_t s);
void launch_finalize(const Geo& g, bool cplx, int recombination, void* out, const float* weight_acc,
                     const float* noise_acc, const float* noise_ctr, float* weights, float* noise_map,
                     const uint8_t* mask, int mask_is_4d, cudaStream_t s);

// pd_backward.cu: adjoint of the low-rank patch denoiser (real volumes)
struct BwdWork {
  int recombination;    // PD_RECOMB_WEIGHTED or PD_RECOMB_AVERAGE
  int shrink;           // 0 soft threshold at stdest * level, 1 hard at the patch rank
  double level;         // soft: tau_p = stdest_p * level
  const int32_t* rank;  // [count] the forward's maxidx per patch
  float* cross;         // [count][mat_stride] Xc^T Gb
  float* k1;            // [count][mat_stride] V E V^T
  float* k2;            // [count][mat_stride] V diag(h/s) V^T
  int64_t mat_stride;   // floats per patch (n * n)
  float* gmean;         // [count][n] mean row of Gb
  float* u;             // [count][n] gmean (I - K2)
  double* dlevel;       // [count] dL/dlevel per patch (soft), 0 (hard)
};
bool bwd_supported(int n);
cudaError_t launch_backward(const Geo& g, const float* in, const float* gout, const float* wts, float* gin,
                            const PatchWork& w, const BwdWork& b, cudaStream_t s);

// pd_gram_tma.cu (pack + TMA-fed tcgen05)
// The mixed path's packed operands of a chunk, in bf16 elements from
// PatchWork::packed: the Gram's column-major hi / lo [count][N][kp] and, for the
// tensor-core synthesis, the row-major copy [count][kp][kn] and the synthesis
// matrix [count][N][kn] (hi / lo each). N real columns, kp = rows rounded up to
// 64, kn = N rounded up to 64.
struct PackedLayout {
  int N;
  int64_t kp, kn;
  bool synth_tc;
  int64_t hi, lo, rows_hi, rows_lo, coef_hi, coef_lo, total;
};
PackedLayout packed_layout(int n, bool cplx, int M, bool synth_tc, int count);
size_t packed_bytes_per_patch(int n, bool cplx, int M, bool synth_tc);
cudaError_t make_bf16_map(CUtensorMap* m, const void* base, int64_t inner, int64_t rows, int64_t depth,
                          int box_rows = 128);
cudaError_t launch_gram_packed(const Geo& g, bool cplx, const void* in, const PatchWork& w, void* packed,
                               cudaStream_t s, bool synth_tc = false);
// pd_synth_tc.cu: the tensor-core synthesis (mixed path, weighted / average
// recombination) from the packed row-major operands launch_gram_packed wrote
cudaError_t launch_synth_tc(const Geo& g, bool cplx, const PatchWork& w, const SynthArgs& a, cudaStream_t s);

// pd_mc.cu
// Bartlett-sampled Wishart Grams: n_iter packed d x d Grams distributed as G^T G
// for m x d standard Gaussian G (m >= d); Lbuf holds n_iter d x d floats.
void launch_wishart(int64_t m, int d, int n_iter, uint64_t seed, float* Lbuf, float* gram, int64_t gram_stride,
                    cudaStream_t s);
int64_t mc_chunks(int64_t rows);
// pd_noise.cu
void launch_estimate_noise(const float* in, bool cplx, const int64_t dims[3], const int blk[3], int T, double* mean,
                           double* m2, double* out, cudaStream_t s);
void launch_mc_level(const double* lam, int n_iter, double noise_std, double* out, cudaStream_t s);
void launch_mc_gram(int64_t rows, int cols, int n_iter, uint64_t seed, float* part, float* gram,
                    int64_t gram_stride, cudaStream_t s);

}  // namespace pd
