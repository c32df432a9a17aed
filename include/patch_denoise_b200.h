/*
 * patch_denoise_b200.h -- C ABI of the B200 (sm_100a) space-time low-rank
 * denoising library (libpd_b200.so).
 *
 * The reference (paquiteau/patch-denoising) is pure Python; its hot path is the
 * per-patch loop of BaseSpaceTimeDenoiser.denoise (src/patch_denoise/space_time/
 * base.py:177-270) calling the per-method _patch_processing plug-ins
 * (space_time/lowrank.py). These entry points replace that loop. Each one names
 * the reference interface it stands in for. All buffers are caller-owned device
 * memory (plain pointers + sizes); every call is asynchronous on the given stream
 * unless its comment says it synchronises. No call throws: the status code says
 * what went wrong and pd_last_error() gives a message.
 *
 * Data layout: a 4D volume (X, Y, Z, T) in C order (T fastest). Inputs of fewer
 * spatial dimensions are padded with leading unit axes by pd_geometry_init.
 * Complex volumes are interleaved float pairs (complex64).
 */
#ifndef PATCH_DENOISE_B200_H
#define PATCH_DENOISE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t pd_status;
#define PD_OK 0
#define PD_ERR_INVALID 1     /* bad argument: the reference raises ValueError   */
#define PD_ERR_UNSUPPORTED 2 /* valid but not handled by this build            */
#define PD_ERR_CUDA 3        /* a CUDA runtime call failed                      */
#define PD_ERR_WORKSPACE 4   /* workspace smaller than the queried size         */

#define PD_METHOD_MPPCA 0   /* MPPCADenoiser      (space_time/lowrank.py:28-63)   */
#define PD_METHOD_HYBRID 1  /* HybridPCADenoiser  (space_time/lowrank.py:67-119)  */
#define PD_METHOD_RAW 2     /* RawSVDDenoiser / NordicDenoiser hard threshold
                               (space_time/lowrank.py:123-246)                    */
#define PD_METHOD_OPTIMAL 3 /* OptimalSVDDenoiser (space_time/lowrank.py:284-407) */
#define PD_METHOD_ADAPTIVE 4 /* AdaptiveDenoiser  (space_time/lowrank.py:410-636):
                                pd_adaptive_denoise_patches only                  */

/* Adaptive trace-norm shrinkage d = s max(1 - (tau/s)^gamma, 0) (Josse & Sardy). */
#define PD_ADAPTIVE_SURE 0  /* tau by SURE per candidate gamma, lowest cost wins */
#define PD_ADAPTIVE_GSURE 1 /* the same with the generalised SURE cost           */
#define PD_ADAPTIVE_QUT 2   /* tau = stdest * qut_level; gamma fixed or by SURE  */
#define PD_ADAPTIVE_MAX_GAMMA 32

#define PD_RECOMB_WEIGHTED 0 /* theta = 1 / (2 + maxidx)  (base.py:246-249) */
#define PD_RECOMB_AVERAGE 1  /* theta = 1                 (base.py:250-252) */
#define PD_RECOMB_CENTER 2   /* centre element only       (base.py:244-245) */

#define PD_LOSS_FRO 0 /* _opt_fro_shrink (space_time/lowrank.py:272-280) */
#define PD_LOSS_NUC 1 /* _opt_nuc_shrink (space_time/lowrank.py:263-269) */
#define PD_LOSS_OPE 2 /* _opt_ope_shrink (space_time/lowrank.py:258-260) */

#define PD_PRECISION_FP32 0  /* FP32 SIMT Gram                                  */
#define PD_PRECISION_MIXED 1 /* BF16 tcgen05 Gram + FP32 subspace refinement    */

/* Patch geometry of the strided sliding view.
 * Mirrors PatchedArray.__init__ (space_time/base.py:24-82). */
typedef struct pd_geometry {
  int64_t shape[4]; /* (X, Y, Z, T), leading axes padded with 1            */
  int64_t patch[4]; /* patch extent per axis (clamped to the axis)         */
  int64_t step[4];  /* patch - overlap, taken before clamping              */
  int64_t grid[4];  /* number of patch positions per axis                  */
  int64_t n_patches;
  int64_t rows; /* M = voxels per patch (Casorati rows)                    */
  int64_t cols; /* frames per patch (Casorati columns)                     */
} pd_geometry;

/* Per-call method parameters. */
typedef struct pd_params {
  int32_t method;        /* PD_METHOD_*                                     */
  int32_t recombination; /* PD_RECOMB_*                                     */
  int32_t loss;          /* PD_LOSS_* (optimal only)                        */
  int32_t precision;     /* PD_PRECISION_*                                  */
  int32_t is_complex;    /* input/output are complex64                      */
  int32_t has_prior;     /* noise_std map given (hybrid / optimal)          */
  double threshold_scale; /* MP-PCA threshold_scale                         */
  double threshold;       /* raw / NORDIC singular-value threshold          */
  double mp_median;       /* optimal: Marchenko-Pastur median for beta      */
} pd_params;

/* Parameters of PD_METHOD_ADAPTIVE (AdaptiveDenoiser.denoise's tau0 / gamma0 and
 * method, space_time/lowrank.py:546-605). */
typedef struct pd_adaptive {
  int32_t mode;     /* PD_ADAPTIVE_*                                                  */
  int32_t n_gamma;  /* SURE / GSURE: candidates in gamma[] (1..PD_ADAPTIVE_MAX_GAMMA);
                       QUT: 1 = gamma[0] is fixed, 0 = gamma estimated by SURE       */
  int32_t has_tau0; /* SURE / GSURE: 1 = the log-tau search starts at tau0,
                       0 = at log(median singular value)                             */
  int32_t reserved;
  double tau0;      /* log tau                                                        */
  double qut_level; /* QUT: pd_adaptive_qut_level's quantile                          */
  double gamma[PD_ADAPTIVE_MAX_GAMMA];
} pd_adaptive;

/* Library version (major*10000 + minor*100 + patch). */
int32_t pd_version(void);

/* Message of the last failing call on this host thread (empty if none). */
const char* pd_last_error(void);

/* Fill *g from the full (time-appended) patch shape and overlap.
 * Replaces PatchedArray.__init__ (space_time/base.py:24-82) applied to the
 * output of BaseSpaceTimeDenoiser._get_patch_param (base.py:359-384).
 * ndim in [2, 4]; returns PD_ERR_INVALID where the reference raises. */
pd_status pd_geometry_init(int32_t ndim, const int64_t* shape, const int64_t* patch_shape,
                           const int64_t* patch_overlap, pd_geometry* g);

/* Median of the Marchenko-Pastur law of aspect ratio beta, by the reference's
 * 5-point dichotomy on the closed-form CDF (host, FP64).
 * Replaces marchenko_pastur_median (space_time/utils.py:149-204). */
pd_status pd_mp_median(double beta, double eps, double* out);

/* Scratch bytes pd_select_patches needs. */
pd_status pd_select_workspace_size(const pd_geometry* g, size_t* bytes);

/* Mask scoring and compaction: d_patch_list[0 .. *d_count) receives, in
 * ascending order, every linear patch index whose mask fill satisfies
 * 100 * sum(mask in patch) / patch size > mask_threshold. d_mask is uint8 of
 * shape (X,Y,Z) (mask_is_4d = 0) or (X,Y,Z,T) (mask_is_4d = 1), or NULL for an
 * all-true mask. d_patch_list holds n_patches int32.
 * Replaces the selection loop of BaseSpaceTimeDenoiser.denoise (base.py:202-227). */
pd_status pd_select_patches(const pd_geometry* g, const uint8_t* d_mask, int32_t mask_is_4d,
                            double mask_threshold, int32_t* d_patch_list, int32_t* d_count,
                            void* d_workspace, size_t workspace_bytes, void* stream);

/* Scratch bytes pd_denoise_patches needs for n_selected patches. */
pd_status pd_denoise_workspace_size(const pd_geometry* g, const pd_params* p, int64_t n_selected,
                                    size_t* bytes);

/* Denoise the listed patches and accumulate them.
 *   d_in          input volume (float32 or complex64), read only
 *   d_noise_std   spatial noise_std map (float64, X*Y*Z) when p->has_prior, else NULL
 *   d_out_acc     output volume, same type as d_in, zeroed by the caller; receives
 *                 sum theta * patch (weighted/average) or the centre elements
 *   d_weight_acc  float32 [X*Y*Z*grid[3]]: sum of theta per voxel and time window
 *   d_noise_acc   float32 [X*Y*Z*grid[3]]: sum of theta * noise_var (finite only)
 *   d_noise_ctr   float32 4D map: centre-element noise_var (center recombination)
 *   d_rank_map    int32 4D map: max maxidx of the patches centred on each voxel
 *   d_patch_rank  int32 [n_selected]: maxidx per listed patch
 *   d_patch_noise float32 [n_selected]: noise_var per listed patch (NaN if none)
 * All accumulators are zeroed by the caller.
 * Replaces the hot loop of BaseSpaceTimeDenoiser.denoise (base.py:235-258) and the
 * _patch_processing plug-ins of MPPCADenoiser, HybridPCADenoiser, RawSVDDenoiser,
 * NordicDenoiser and OptimalSVDDenoiser (space_time/lowrank.py:42-407). */
pd_status pd_denoise_patches(const pd_geometry* g, const pd_params* p, const void* d_in,
                             const double* d_noise_std, const int32_t* d_patch_list,
                             int64_t n_selected, void* d_out_acc, float* d_weight_acc,
                             float* d_noise_acc, float* d_noise_ctr, int32_t* d_rank_map,
                             int32_t* d_patch_rank, float* d_patch_noise, void* d_workspace,
                             size_t workspace_bytes, void* stream);

/* Normalisation and masking: d_out /= weights (weighted/average), expand the
 * window accumulators into the 4D float32 d_weights and d_noise_map, then zero
 * every element outside the mask (NULL mask = all true).
 * Replaces base.py:262-270. */
pd_status pd_finalize(const pd_geometry* g, const pd_params* p, void* d_out,
                      const float* d_weight_acc, const float* d_noise_acc,
                      const float* d_noise_ctr, float* d_weights, float* d_noise_map,
                      const uint8_t* d_mask, int32_t mask_is_4d, void* stream);

/* Scratch bytes pd_nordic_mc_threshold needs. */
pd_status pd_nordic_workspace_size(int64_t rows, int64_t cols, int32_t n_iter, size_t* bytes);

/* NORDIC Monte-Carlo level: mean over n_iter draws of the largest singular value
 * of a rows x cols standard Gaussian matrix (counter-based Philox normals, seeded),
 * written to *out on the host. Synchronises the stream.
 * Replaces the Monte-Carlo loop of NordicDenoiser.denoise (space_time/lowrank.py:221-232). */
pd_status pd_nordic_mc_threshold(int64_t rows, int64_t cols, int32_t n_iter, uint64_t seed,
                                 int32_t precision, double* out, void* d_workspace,
                                 size_t workspace_bytes, void* stream);

/* NORDIC in one call, without a host round trip for the Monte-Carlo level.
 * The reference computes the level on the host (space_time/lowrank.py:221-242)
 * and then runs the patch loop with threshold = noise_std * level; this call
 * does both on the device, in stream order: the draws (pd_nordic_mc_threshold's
 * computation, with mc_rows x g->cols draws), the level, then the patch loop,
 * whose eigensolver reads the threshold from device memory.
 * p->method must be PD_METHOD_RAW; p->threshold is ignored.
 *   d_level   2 doubles on the device: [0] the level, [1] noise_std * level
 *   d_mc_ws   pd_nordic_workspace_size(mc_rows, g->cols, n_iter) bytes
 *   mc_rows   0: no draws; d_level already holds the level of an earlier call
 *             on the same stream (a volume processed in several patch ranges)
 * The other arguments are those of pd_denoise_patches (no noise map). Check
 * both workspaces with pd_workspace_check. Replaces NordicDenoiser.denoise's level
 * and patch loop (space_time/lowrank.py:221-246 and base.py:235-258). */
pd_status pd_nordic_denoise_patches(const pd_geometry* g, const pd_params* p, double noise_std, int64_t mc_rows,
                                    int32_t n_iter, uint64_t seed, double* d_level, void* d_mc_ws,
                                    size_t mc_ws_bytes, const void* d_in, const int32_t* d_patch_list,
                                    int64_t n_selected, void* d_out_acc, float* d_weight_acc, float* d_noise_acc,
                                    float* d_noise_ctr, int32_t* d_rank_map, int32_t* d_patch_rank,
                                    float* d_patch_noise, void* d_workspace, size_t workspace_bytes, void* stream);

/* Quantile of the largest singular value of n_sim standard Gaussian rows x cols
 * draws at probability 1 - 1/sqrt(log(max(rows, cols))) (numpy.quantile's
 * linear interpolation), to *out. The reference draws n_sim matrices of the
 * patch's shape scaled by its noise estimate for every patch and takes this
 * quantile (space_time/lowrank.py:464-475); the quantile scales with the noise
 * estimate, so one set of draws per call gives every patch's tau. The draws are
 * pd_nordic_mc_threshold's (same seed convention and precision); workspace
 * pd_nordic_workspace_size(rows, cols, n_sim). Synchronises the stream. */
pd_status pd_adaptive_qut_level(int64_t rows, int64_t cols, int32_t n_sim, uint64_t seed, int32_t precision,
                                double* out, void* d_workspace, size_t workspace_bytes, void* stream);

/* pd_denoise_patches for AdaptiveDenoiser (space_time/lowrank.py:607-636):
 * p->method must be PD_METHOD_ADAPTIVE and p->has_prior 1, with d_noise_std
 * the spatial noise_std map (the patch's noise estimate is
 * sqrt(mean noise_std^2 over the patch)). Per patch the full singular
 * spectrum comes from the Gram route; the SURE / GSURE cost
 * (_sure_atn_cost, lowrank.py:410-447) is minimised over log tau (SURE /
 * GSURE, every candidate gamma) or over log(gamma - 1) (QUT without a fixed
 * gamma) by a bracketing line search and Brent's method on the device,
 * in place of scipy.optimize.minimize (BFGS). Then d = s max(1 - (tau/s)^gamma, 0),
 * maxidx = number of nonzero d. Workspace: pd_denoise_workspace_size. */
pd_status pd_adaptive_denoise_patches(const pd_geometry* g, const pd_params* p, const pd_adaptive* a,
                                      const void* d_in, const double* d_noise_std, const int32_t* d_patch_list,
                                      int64_t n_selected, void* d_out_acc, float* d_weight_acc, float* d_noise_acc,
                                      float* d_noise_ctr, int32_t* d_rank_map, int32_t* d_patch_rank,
                                      float* d_patch_noise, void* d_workspace, size_t workspace_bytes,
                                      void* stream);

/* pd_denoise_patches without a workspace argument. No counterpart in the
 * reference. It is for callers that cannot allocate device memory while they
 * denoise, e.g. a host application that manages a fixed device-memory budget
 * itself, or a loop where cudaMalloc's implicit synchronisation is not
 * acceptable. The scratch is a static 32 MiB device array inside the library
 * that every GPU loading the library keeps until exit. Patches are processed
 * in chunks that fit it. A geometry whose single-patch scratch exceeds 32 MiB
 * returns PD_ERR_WORKSPACE. Every call looks up the array's device address on
 * the current device; the first call on a device also loads the library's
 * device code there, so make it before any stream capture. Read the device
 * error word (NaN / inf samples, timed-out waits) with pd_noalloc_check. All
 * calls share the array, so calls that overlap on the GPU (other streams or
 * host threads) race.
 * Arguments are those of pd_denoise_patches minus the workspace. */
pd_status pd_denoise_patches_noalloc(const pd_geometry* g, const pd_params* p, const void* d_in,
                                     const double* d_noise_std, const int32_t* d_patch_list, int64_t n_selected,
                                     void* d_out_acc, float* d_weight_acc, float* d_noise_acc, float* d_noise_ctr,
                                     int32_t* d_rank_map, int32_t* d_patch_rank, float* d_patch_noise, void* stream);

/* Companion of pd_denoise_patches_noalloc, with no counterpart in the reference:
 * the caller of the no-allocation entry point has no workspace pointer to hand
 * to pd_workspace_check, because its scratch (and the device error word at its
 * start) is the library's static array. This synchronises the stream and reads
 * that word: PD_ERR_INVALID if a processed patch held a NaN or infinite sample,
 * PD_ERR_CUDA if a bounded device-side wait timed out, PD_OK otherwise. */
pd_status pd_noalloc_check(void* stream);

/* One volume of a batched call: its geometry, device buffers (as for
 * pd_denoise_patches) and per-volume rule parameters. */
typedef struct pd_volume {
  pd_geometry geometry;
  const void* d_in;           /* float32 or complex64 volume                       */
  const double* d_noise_std;  /* spatial noise_std map when the method needs one   */
  const int32_t* d_patch_list; /* the volume's selected patches (pd_select_patches) */
  int64_t n_selected;
  void* d_out_acc;
  float* d_weight_acc;
  float* d_noise_acc;
  float* d_noise_ctr;
  int32_t* d_rank_map;
  int32_t* d_patch_rank;      /* [n_selected]                                      */
  float* d_patch_noise;       /* [n_selected]                                      */
  double threshold;           /* raw: the singular-value threshold                 */
  double mp_median;           /* optimal: Marchenko-Pastur median of T / M         */
} pd_volume;

#define PD_BATCH_MAX_VOLUMES 64

/* Launch-shape choices of a batched call (an autotuner picks them by timing). */
typedef struct pd_batch_tuning {
  int32_t synth_row_blocks; /* CTAs per patch in the synthesis scatter; 0 = by the patch's rows */
  int32_t order_by_cost;    /* 1: volumes in descending per-patch cost order (frames^3), 0: as given */
  int64_t chunk_patches;    /* patches per launch; 0 = as many as the workspace holds */
} pd_batch_tuning;

/* Scratch bytes pd_denoise_batch needs (chunk_patches as in pd_batch_tuning). */
pd_status pd_denoise_batch_workspace_size(const pd_volume* vols, int32_t n_vols, const pd_params* p,
                                          int64_t chunk_patches, size_t* bytes);

/* pd_denoise_patches over up to PD_BATCH_MAX_VOLUMES volumes of uneven shape in
 * one set of launches: the volumes' selected patches form one work list (its
 * order by tuning->order_by_cost), and every patch kernel reads its patch's
 * volume (geometry, buffers, threshold / MP median) from a device table, so a
 * launch spans every volume. Plain FP32 kernels; methods MP-PCA, hybrid, raw and
 * optimal (p->threshold and p->mp_median are taken per volume). No reference
 * counterpart: the reference denoises one volume per call (base.py:177-270) and
 * its GPU module batches the patches of one volume (gpu/main.py:186-244).
 * Normalise each volume with pd_finalize afterwards. tuning may be NULL. */
pd_status pd_denoise_batch(const pd_volume* vols, int32_t n_vols, const pd_params* p,
                           const pd_batch_tuning* tuning, void* d_workspace, size_t workspace_bytes,
                           void* stream);

/* Scratch bytes pd_lowrank_backward needs for n_selected patches. */
pd_status pd_lowrank_backward_workspace_size(const pd_geometry* g, int64_t n_selected, size_t* bytes);

/* Gradient of the low-rank patch denoiser with respect to its input and its
 * threshold (real float32 volumes, weighted or average recombination). The
 * reference has no gradient; this is the adjoint of its forward path
 * (BaseSpaceTimeDenoiser.denoise, space_time/base.py:177-270) with the shrinkage
 *   shrink 0: soft threshold s~ = max(s - tau_p, 0), tau_p = stdest_p * level,
 *             stdest_p = sqrt(mean over the patch of noise_std^2) (the adaptive
 *             trace-norm shrinkage of space_time/lowrank.py:459-461 at gamma 1);
 *   shrink 1: hard threshold at the forward's rank (MP-PCA / hybrid / raw rules
 *             at a fixed decision; the threshold gradient is then zero).
 * Every patch's factorisation is recomputed (mean, Gram, all eigenpairs).
 *   d_in, d_patch_list, d_patch_rank  the forward's input, patch list and maxidx
 *   d_weights   the forward's 4D float32 weights (recombination normaliser)
 *   d_gout      upstream gradient, the input's shape
 *   d_gin       gradient with respect to the input, zeroed by the caller (accumulated)
 *   d_dlevel    float64 [n_selected]: each patch's dL/dlevel (0 for shrink 1)
 * Needs more voxels than frames per patch and at most 128 frames. */
pd_status pd_lowrank_backward(const pd_geometry* g, int32_t recombination, int32_t shrink, const float* d_in,
                              const double* d_noise_std, double level, const int32_t* d_patch_list,
                              int64_t n_selected, const int32_t* d_patch_rank, const float* d_weights,
                              const float* d_gout, float* d_gin, double* d_dlevel, void* d_workspace,
                              size_t workspace_bytes, void* stream);

/* Scratch bytes pd_estimate_noise needs (shape as for pd_estimate_noise). */
pd_status pd_estimate_noise_workspace_size(int32_t ndim, const int64_t* shape, int32_t is_complex, size_t* bytes);

/* Noise map of a noise-only sequence: for every block of block_size voxels per
 * spatial axis (every position), the population standard deviation of the
 * block's samples over all frames, written at the voxel block_size / 2 past the
 * block's corner; other voxels get 0. shape = (spatial..., frames), 1 to 3
 * spatial axes, each longer than block_size. d_in float32 or complex64 (is_complex),
 * C order; d_noise_map float64 of the spatial shape.
 * Replaces estimate_noise (space_time/utils.py:207-242). */
pd_status pd_estimate_noise(int32_t ndim, const int64_t* shape, int32_t is_complex, const void* d_in,
                            int32_t block_size, double* d_noise_map, void* d_workspace, size_t workspace_bytes,
                            void* stream);

/* Synchronise the stream and read the workspace's device error word from the
 * last call on it: PD_ERR_INVALID if a processed patch holds a NaN or infinite
 * sample (the reference's LAPACK calls raise ValueError on those), PD_ERR_CUDA
 * if a bounded device-side wait timed out. */
pd_status pd_workspace_check(const void* d_workspace, void* stream);

/* Kernel timing (no reference counterpart; used by bench.py for the roofline).
 * When enabled, every kernel launch of the library on this host thread's calls
 * is bracketed by CUDA events on its stream. pd_profile_collect synchronises
 * those events and writes one line per kernel, "name launches total_ms\n", into
 * buf (truncated to len), then clears the record. */
pd_status pd_profile_enable(int32_t on);
pd_status pd_profile_collect(char* buf, size_t len);

#ifdef __cplusplus
}
#endif
#endif /* PATCH_DENOISE_B200_H */
