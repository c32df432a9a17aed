// C ABI of libpd_b200.so: argument checking, workspace carving and the launch
// sequence. See include/patch_denoise_b200.h for the contract of each call.
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>

#include <algorithm>
#include <string>
#include <vector>

#include "pd_common.cuh"
#include "pd_kernels.cuh"
#include "pd_profile.cuh"

using namespace pd;

namespace {

thread_local std::string g_err;

pd_status fail(pd_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return st;
}

pd_status cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) return fail(PD_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return PD_OK;
}

#define PD_TRY(x)                      \
  do {                                 \
    const pd_status _st = (x);         \
    if (_st != PD_OK) return _st;      \
  } while (0)

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct Carver {
  char* base;
  size_t off = 0;
  explicit Carver(void* b) : base((char*)b) {}
  template <class T>
  T* take(size_t count) {
    T* p = (T*)(base ? base + off : nullptr);
    off += align256(count * sizeof(T));
    return p;
  }
};

constexpr int MAX_FRAMES = 448;
constexpr int MAX_ROWS = 16384;
constexpr size_t DEFAULT_CHUNK_BUDGET = size_t(4) << 30;
constexpr size_t BATCH_CHUNK_BUDGET = size_t(16) << 30;  // a batch spans many volumes: fewer, larger chunks

int64_t gram_stride_floats(int n, bool cplx) {
  int64_t f = pk_size(n) * (cplx ? 2 : 1);
  return (f + 63) & ~int64_t(63);
}
int64_t vec_stride_floats(int n) { return ((int64_t)2 * n * n + 63) & ~int64_t(63); }

size_t per_patch_bytes(int n, bool cplx, size_t packed = 0) {
  Carver c(nullptr);
  // carve one patch worth of every buffer (upper bound incl. alignment)
  size_t b = packed;
  b += (size_t)n * (cplx ? 8 : 4);                  // mean
  b += (size_t)gram_stride_floats(n, cplx) * 4;     // gram
  b += (size_t)vec_stride_floats(n) * 4;            // vec
  b += (size_t)n * 4;                               // coef
  b += 4 + 4 + 4 + 8;                               // n_active, rank, noise, prior
  (void)c;
  return b;
}

PatchWork carve_work(void* ws, int count, int n, bool cplx, size_t* used, size_t packed_per_patch = 0) {
  Carver c(ws);
  PatchWork w{};
  w.err = c.take<int>(1);  // always at offset 0 of the workspace
  w.ctr = c.take<int>(1);  // tile counter of the persistent tensor-core kernels
  w.count = count;
  w.n_stride = n;
  w.packed = packed_per_patch ? (void*)c.take<uint8_t>(packed_per_patch * count) : nullptr;
  w.mean = c.take<float>((size_t)count * n * (cplx ? 2 : 1));
  w.gram_stride = gram_stride_floats(n, cplx);
  w.gram = c.take<float>((size_t)count * w.gram_stride);
  w.vec_stride = vec_stride_floats(n);
  w.vec = c.take<float>((size_t)count * w.vec_stride);
  w.coef = c.take<float>((size_t)count * n);
  w.n_active = c.take<int32_t>(count);
  w.rank = c.take<int32_t>(count);
  w.noise = c.take<float>(count);
  w.prior = c.take<double>(count);
  *used = c.off;
  return w;
}

size_t work_bytes(int count, int n, bool cplx, size_t packed_per_patch = 0) {
  size_t used;
  carve_work(nullptr, count, n, cplx, &used, packed_per_patch);
  return used;
}

// The mixed path synthesises high-rank patches (the adaptive rules keep whole
// spectra) on the tensor cores; center recombination writes one row per patch
// and keeps the SIMT kernel.
bool synth_tc_used(const pd_params* p) {
  return p->precision == PD_PRECISION_MIXED && p->method == PD_METHOD_ADAPTIVE &&
         p->recombination != PD_RECOMB_CENTER;
}

size_t packed_of(const pd_geometry* g, const pd_params* p) {
  return p->precision == PD_PRECISION_MIXED
             ? packed_bytes_per_patch((int)g->cols, p->is_complex != 0, (int)g->rows, synth_tc_used(p))
             : 0;
}

pd_status check_geometry(const pd_geometry* g) {
  if (!g) return fail(PD_ERR_INVALID, "geometry is NULL");
  for (int i = 0; i < 4; ++i)
    if (g->shape[i] < 1 || g->patch[i] < 1 || g->grid[i] < 1)
      return fail(PD_ERR_INVALID, "geometry is not initialised");
  return PD_OK;
}

pd_status check_params(const pd_geometry* g, const pd_params* p) {
  if (!p) return fail(PD_ERR_INVALID, "params is NULL");
  if (p->method < PD_METHOD_MPPCA || p->method > PD_METHOD_ADAPTIVE)
    return fail(PD_ERR_INVALID, "unknown method %d", p->method);
  if (p->recombination < PD_RECOMB_WEIGHTED || p->recombination > PD_RECOMB_CENTER)
    return fail(PD_ERR_INVALID, "recombination must be one of 'weighted', 'average', 'center'");
  if (p->loss < PD_LOSS_FRO || p->loss > PD_LOSS_OPE) return fail(PD_ERR_INVALID, "unknown loss %d", p->loss);
  const int64_t n = g->cols, M = g->rows;
  if (n > MAX_FRAMES)
    return fail(PD_ERR_UNSUPPORTED, "patch spans %lld frames; this build handles at most %d", (long long)n,
                MAX_FRAMES);
  if (M > MAX_ROWS)
    return fail(PD_ERR_UNSUPPORTED, "patch has %lld voxels; this build handles at most %d", (long long)M,
                MAX_ROWS);
  if (M < 2) return fail(PD_ERR_INVALID, "a patch needs at least 2 voxels");
  if ((p->method == PD_METHOD_MPPCA || p->method == PD_METHOD_HYBRID) && n < 10)
    return fail(PD_ERR_INVALID, "MP-PCA / hybrid-PCA need at least 10 frames per patch (top-10 eigenvalues)");
  if (p->precision != PD_PRECISION_FP32 && p->precision != PD_PRECISION_MIXED)
    return fail(PD_ERR_INVALID, "unknown precision %d", p->precision);
  return PD_OK;
}

// Marchenko-Pastur CDF, closed form of the integral of
// sqrt((b-t)(t-a)) / (2 pi beta t) from a to x, a = (1-sqrt(beta))^2, b = (1+sqrt(beta))^2.
// Antiderivative: R + (a+b)/2 asin((2t-a-b)/(b-a)) - sqrt(ab) asin(((a+b)t-2ab)/((b-a)t)).
double mp_cdf(double x, double beta) {
  const double a = (1 - sqrt(beta)) * (1 - sqrt(beta));
  const double b = (1 + sqrt(beta)) * (1 + sqrt(beta));
  if (x <= a) return 0.0;
  if (x >= b) return 1.0;
  auto clamp1 = [](double u) { return u > 1.0 ? 1.0 : (u < -1.0 ? -1.0 : u); };
  auto G = [&](double t) {
    const double R = sqrt(fmax((b - t) * (t - a), 0.0));
    double v = R + 0.5 * (a + b) * asin(clamp1((2 * t - a - b) / (b - a)));
    const double sab = sqrt(a * b);
    if (sab > 0.0) v -= sab * asin(clamp1(((a + b) * t - 2 * a * b) / ((b - a) * t)));
    return v;
  };
  return (G(x) - G(a)) / (2.0 * M_PI * beta);
}

// A non-blocking side stream with its fork and join events, per device and
// host thread (created on first use, kept for the thread's lifetime).
struct SideStream {
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};

pd_status side_stream(SideStream** out) {
  static thread_local SideStream per_dev[64];
  int dev = 0;
  PD_TRY(cuda_check(cudaGetDevice(&dev), "current device"));
  if (dev < 0 || dev >= 64) return fail(PD_ERR_UNSUPPORTED, "device index %d", dev);
  SideStream& ss = per_dev[dev];
  if (!ss.stream) {
    PD_TRY(cuda_check(cudaStreamCreateWithFlags(&ss.stream, cudaStreamNonBlocking), "side stream"));
    PD_TRY(cuda_check(cudaEventCreateWithFlags(&ss.fork, cudaEventDisableTiming), "fork event"));
    PD_TRY(cuda_check(cudaEventCreateWithFlags(&ss.join, cudaEventDisableTiming), "join event"));
  }
  *out = &ss;
  return PD_OK;
}

}  // namespace

extern "C" {

int32_t pd_version(void) { return 100; }

const char* pd_last_error(void) { return g_err.c_str(); }

pd_status pd_geometry_init(int32_t ndim, const int64_t* shape, const int64_t* patch_shape,
                           const int64_t* patch_overlap, pd_geometry* g) {
  g_err.clear();
  if (!shape || !patch_shape || !patch_overlap || !g) return fail(PD_ERR_INVALID, "NULL argument");
  if (ndim < 2 || ndim > 4)
    return fail(PD_ERR_UNSUPPORTED, "inputs with %d dimensions are not supported (2 to 4)", ndim);
  int64_t ps[4], st[4], sh[4], gr[4];
  const int pad = 4 - ndim;
  for (int i = 0; i < 4; ++i) {
    if (i < pad) {
      sh[i] = 1;
      ps[i] = 1;
      st[i] = 1;
      gr[i] = 1;
      continue;
    }
    const int k = i - pad;
    sh[i] = shape[k];
    if (sh[i] < 1) return fail(PD_ERR_INVALID, "empty input axis %d", k);
    const int64_t step = patch_shape[k] - patch_overlap[k];
    if (step < 0) return fail(PD_ERR_INVALID, "overlap should be smaller than patch on every dimension.");
    if (patch_shape[k] < 1) return fail(PD_ERR_INVALID, "patch extent must be positive");
    if (patch_shape[k] > sh[i])
      return fail(PD_ERR_INVALID,
                  "patch extent %lld exceeds the input extent %lld along axis %d (the Casorati reshape of the "
                  "reference fails)",
                  (long long)patch_shape[k], (long long)sh[i], k);
    ps[i] = patch_shape[k];
    st[i] = step;
    if (ps[i] < sh[i])
      gr[i] = step > 0 ? (sh[i] - ps[i]) / step + 1 : 1;
    else
      gr[i] = 1;
  }
  int64_t np = 1;
  for (int i = 0; i < 4; ++i) {
    g->shape[i] = sh[i];
    g->patch[i] = ps[i];
    g->step[i] = st[i];
    g->grid[i] = gr[i];
    np *= gr[i];
  }
  if (np > INT32_MAX) return fail(PD_ERR_UNSUPPORTED, "more than 2^31 patches");
  g->n_patches = np;
  g->rows = ps[0] * ps[1] * ps[2];
  g->cols = ps[3];
  return PD_OK;
}

pd_status pd_mp_median(double beta, double eps, double* out) {
  g_err.clear();
  if (!out) return fail(PD_ERR_INVALID, "NULL output");
  if (!(0 <= beta && beta <= 1)) return fail(PD_ERR_INVALID, "Aspect Ratio should be between 0 and 1");
  const double a = (1 - sqrt(beta)) * (1 - sqrt(beta));
  const double b = (1 + sqrt(beta)) * (1 + sqrt(beta));
  double lo = a, hi = b;
  bool moved = true;
  int rounds = 0;
  while (moved && (hi - lo) > eps && rounds < 20) {
    moved = false;
    double pts[5];
    const double step = (hi - lo) / 4.0;
    for (int i = 0; i < 4; ++i) pts[i] = (double)i * step + lo;
    pts[4] = hi;
    double cdf[5];
    for (int i = 0; i < 5; ++i) cdf[i] = mp_cdf(pts[i], beta);
    bool any_lo = false, any_hi = false;
    double nlo = -INFINITY, nhi = INFINITY;
    for (int i = 0; i < 5; ++i) {
      if (cdf[i] < 0.5) {
        any_lo = true;
        nlo = fmax(nlo, pts[i]);
      }
      if (cdf[i] > 0.5) {
        any_hi = true;
        nhi = fmin(nhi, pts[i]);
      }
    }
    if (any_lo) {
      lo = nlo;
      moved = true;
    }
    if (any_hi) {
      hi = nhi;
      moved = true;
    }
    ++rounds;
  }
  *out = (lo + hi) / 2;
  return PD_OK;
}

pd_status pd_select_workspace_size(const pd_geometry* g, size_t* bytes) {
  g_err.clear();
  PD_TRY(check_geometry(g));
  if (!bytes) return fail(PD_ERR_INVALID, "NULL output");
  const int64_t np = g->n_patches;
  const int64_t nb = (np + SEL_BLOCK - 1) / SEL_BLOCK;
  const int64_t nvox = g->shape[0] * g->shape[1] * g->shape[2];
  *bytes = align256(np) + align256(sizeof(int32_t) * nb) + align256(sizeof(int32_t) * nvox * g->grid[3]);
  return PD_OK;
}

pd_status pd_select_patches(const pd_geometry* g, const uint8_t* d_mask, int32_t mask_is_4d, double mask_threshold,
                            int32_t* d_patch_list, int32_t* d_count, void* d_ws, size_t ws_bytes, void* stream) {
  g_err.clear();
  PD_TRY(check_geometry(g));
  if (!d_patch_list || !d_count) return fail(PD_ERR_INVALID, "NULL output buffer");
  size_t need;
  PD_TRY(pd_select_workspace_size(g, &need));
  if (ws_bytes < need || !d_ws) return fail(PD_ERR_WORKSPACE, "select workspace too small (%zu < %zu)", ws_bytes, need);
  cudaStream_t s = (cudaStream_t)stream;
  const Geo G = to_geo(*g);
  const int64_t np = g->n_patches;
  const int64_t nb = (np + SEL_BLOCK - 1) / SEL_BLOCK;
  Carver c(d_ws);
  uint8_t* flags = c.take<uint8_t>(np);
  int32_t* bc = c.take<int32_t>(nb);
  int32_t* cnt = c.take<int32_t>(g->shape[0] * g->shape[1] * g->shape[2] * g->grid[3]);
  int mode = 0;
  if (d_mask) {
    if (mask_is_4d) {
      mode = 2;
      const int64_t tot = g->shape[0] * g->shape[1] * g->shape[2] * g->grid[3];
      const int blocks = (int)std::min<int64_t>((tot + 255) / 256, 148 * 16);
      PD_TIMED("select", s, k_window_counts<<<blocks, 256, 0, s>>>(G, d_mask, cnt));
    } else {
      mode = 1;
    }
  }
  {
    const int64_t warps = np;
    const int blocks = (int)std::min<int64_t>((warps * 32 + 255) / 256, 148 * 64);
    PD_TIMED("select", s,
             k_patch_flags<<<blocks, 256, 0, s>>>(G, mode, mode == 1 ? d_mask : nullptr, cnt, mask_threshold, flags));
  }
  PD_TIMED("select", s, k_block_counts<<<(unsigned)nb, SEL_THREADS, 0, s>>>(flags, np, bc));
  PD_TIMED("select", s, k_scan_counts<<<1, 1024, 0, s>>>(bc, nb, d_count));
  PD_TIMED("select", s, k_compact<<<(unsigned)nb, SEL_THREADS, 0, s>>>(flags, np, bc, d_patch_list));
  return cuda_check(cudaGetLastError(), "pd_select_patches launch");
}

pd_status pd_denoise_workspace_size(const pd_geometry* g, const pd_params* p, int64_t n_selected, size_t* bytes) {
  g_err.clear();
  PD_TRY(check_geometry(g));
  PD_TRY(check_params(g, p));
  if (!bytes) return fail(PD_ERR_INVALID, "NULL output");
  if (n_selected < 0) return fail(PD_ERR_INVALID, "negative patch count");
  const int n = (int)g->cols;
  const bool cplx = p->is_complex != 0;
  const size_t pk_b = packed_of(g, p);
  const size_t pp = per_patch_bytes(n, cplx, pk_b);
  int64_t chunk = (int64_t)std::max<size_t>(1, DEFAULT_CHUNK_BUDGET / pp);
  chunk = std::min<int64_t>(chunk, std::max<int64_t>(n_selected, 1));
  *bytes = work_bytes((int)chunk, n, cplx, pk_b);
  return PD_OK;
}

// pd_denoise_patches with the raw threshold optionally read on the device
// (d_thr; NULL = p->threshold), for the one-call NORDIC path.
static pd_status denoise_patches_impl(const pd_geometry* g, const pd_params* p, const void* d_in,
                                      const double* d_noise_std, const int32_t* d_patch_list, int64_t n_selected,
                                      void* d_out_acc, float* d_weight_acc, float* d_noise_acc, float* d_noise_ctr,
                                      int32_t* d_rank_map, int32_t* d_patch_rank, float* d_patch_noise, void* d_ws,
                                      size_t ws_bytes, void* stream, const double* d_thr,
                                      const pd_adaptive* ad = nullptr, cudaEvent_t eig_after = nullptr) {
  PD_TRY(check_geometry(g));
  PD_TRY(check_params(g, p));
  if ((p->method == PD_METHOD_ADAPTIVE) != (ad != nullptr))
    return fail(PD_ERR_INVALID, "PD_METHOD_ADAPTIVE runs through pd_adaptive_denoise_patches only");
  if (n_selected == 0) return PD_OK;
  if (!d_in || !d_patch_list || !d_out_acc || !d_weight_acc || !d_noise_acc || !d_noise_ctr || !d_rank_map ||
      !d_patch_rank || !d_patch_noise)
    return fail(PD_ERR_INVALID, "NULL buffer");
  if ((p->method == PD_METHOD_HYBRID || p->method == PD_METHOD_ADAPTIVE ||
       (p->method == PD_METHOD_OPTIMAL && p->has_prior)) &&
      !d_noise_std)
    return fail(PD_ERR_INVALID, "this method needs the noise_std map");
  const int n = (int)g->cols;
  const bool cplx = p->is_complex != 0;
  const size_t pk_b = packed_of(g, p);
  const size_t one = work_bytes(1, n, cplx, pk_b);
  if (!d_ws || ws_bytes < one) return fail(PD_ERR_WORKSPACE, "workspace too small (%zu < %zu)", ws_bytes, one);
  // largest chunk that fits
  int64_t chunk = std::max<int64_t>(1, (int64_t)(ws_bytes / per_patch_bytes(n, cplx, pk_b)));
  chunk = std::min<int64_t>(chunk, n_selected);
  while (chunk > 1 && work_bytes((int)chunk, n, cplx, pk_b) > ws_bytes) --chunk;
  cudaStream_t s = (cudaStream_t)stream;
  const Geo G = to_geo(*g);
  EigParams ep{};
  ep.method = p->method;
  ep.loss = p->loss;
  ep.has_prior = p->has_prior;
  ep.rows = (int)g->rows;
  ep.cols = n;
  ep.threshold_scale = p->threshold_scale;
  ep.threshold = p->threshold;
  ep.mp_median = p->mp_median;
  ep.d_threshold = d_thr;
  ep.only_unfinished = 0;
  PD_TRY(cuda_check(cudaMemsetAsync(d_ws, 0, sizeof(int), s), "clear error word"));
  for (int64_t off = 0; off < n_selected; off += chunk) {
    const int cnt = (int)std::min<int64_t>(chunk, n_selected - off);
    size_t used;
    PatchWork w = carve_work(d_ws, cnt, n, cplx, &used, pk_b);
    w.list = d_patch_list + off;
    launch_patch_mean(G, cplx, d_in, w, s);
    if (p->method == PD_METHOD_HYBRID || p->method == PD_METHOD_ADAPTIVE ||
        (p->method == PD_METHOD_OPTIMAL && p->has_prior))
      launch_prior(G, p->method, d_noise_std, w, s);
    const bool tc_synth = synth_tc_used(p);
    if (p->precision == PD_PRECISION_MIXED)
      PD_TRY(cuda_check(launch_gram_packed(G, cplx, d_in, w, w.packed, s, tc_synth), "tensor-core Gram launch"));
    else
      launch_gram_fp32(G, cplx, d_in, w, s);
    if (eig_after && off == 0)  // the threshold comes from work on another stream
      PD_TRY(cuda_check(cudaStreamWaitEvent(s, eig_after, 0), "join the Monte-Carlo stream"));
    if (p->precision == PD_PRECISION_MIXED && p->method == PD_METHOD_RAW && sub_supported(cplx, n, (int)g->rows)) {
      // the subspace solver for the patches it certifies, the full solver for the rest
      PD_TRY(cuda_check(launch_sub(cplx, n, ep, w, s), "subspace eigensolver launch"));
      EigParams rest = ep;
      rest.only_unfinished = 1;
      PD_TRY(cuda_check(launch_eig(cplx, n, rest, w, s, ad), "eigensolver launch"));
    } else {
      PD_TRY(cuda_check(launch_eig(cplx, n, ep, w, s, ad), "eigensolver launch"));
    }
    SynthArgs sa;
    sa.recombination = p->recombination;
    sa.out = d_out_acc;
    sa.weight_acc = d_weight_acc;
    sa.noise_acc = d_noise_acc;
    sa.noise_ctr = d_noise_ctr;
    sa.rank_map = d_rank_map;
    sa.patch_rank = d_patch_rank;
    sa.patch_noise = d_patch_noise;
    sa.list_offset = off;
    sa.wide = p->method == PD_METHOD_ADAPTIVE ? 1 : 0;
    sa.row_blocks = 0;
    if (tc_synth)
      PD_TRY(cuda_check(launch_synth_tc(G, cplx, w, sa, s), "tensor-core synthesis launch"));
    else
      launch_synth(G, cplx, d_in, w, sa, s);
    PD_TRY(cuda_check(cudaGetLastError(), "pd_denoise_patches launch"));
  }
  return PD_OK;
}

pd_status pd_denoise_patches(const pd_geometry* g, const pd_params* p, const void* d_in, const double* d_noise_std,
                             const int32_t* d_patch_list, int64_t n_selected, void* d_out_acc, float* d_weight_acc,
                             float* d_noise_acc, float* d_noise_ctr, int32_t* d_rank_map, int32_t* d_patch_rank,
                             float* d_patch_noise, void* d_ws, size_t ws_bytes, void* stream) {
  g_err.clear();
  return denoise_patches_impl(g, p, d_in, d_noise_std, d_patch_list, n_selected, d_out_acc, d_weight_acc, d_noise_acc,
                              d_noise_ctr, d_rank_map, d_patch_rank, d_patch_noise, d_ws, ws_bytes, stream, nullptr);
}

pd_status pd_finalize(const pd_geometry* g, const pd_params* p, void* d_out, const float* d_weight_acc,
                      const float* d_noise_acc, const float* d_noise_ctr, float* d_weights, float* d_noise_map,
                      const uint8_t* d_mask, int32_t mask_is_4d, void* stream) {
  g_err.clear();
  PD_TRY(check_geometry(g));
  if (!p) return fail(PD_ERR_INVALID, "params is NULL");
  if (!d_out || !d_weight_acc || !d_noise_acc || !d_noise_ctr || !d_weights || !d_noise_map)
    return fail(PD_ERR_INVALID, "NULL buffer");
  launch_finalize(to_geo(*g), p->is_complex != 0, p->recombination, d_out, d_weight_acc, d_noise_acc, d_noise_ctr,
                  d_weights, d_noise_map, d_mask, mask_is_4d, (cudaStream_t)stream);
  return cuda_check(cudaGetLastError(), "pd_finalize launch");
}

pd_status pd_nordic_workspace_size(int64_t rows, int64_t cols, int32_t n_iter, size_t* bytes) {
  g_err.clear();
  if (!bytes) return fail(PD_ERR_INVALID, "NULL output");
  if (rows < 1 || cols < 1 || n_iter < 1) return fail(PD_ERR_INVALID, "empty Monte-Carlo problem");
  if (cols > MAX_FRAMES) return fail(PD_ERR_UNSUPPORTED, "at most %d frames", MAX_FRAMES);
  const size_t simt = align256(sizeof(float) * (size_t)n_iter * mc_chunks(rows) * pk_size((int)cols));
  const int64_t d = std::min(rows, cols);
  const size_t wish = align256(sizeof(float) * (size_t)n_iter * d * d);
  *bytes = work_bytes(n_iter, (int)cols, false) + std::max(simt, wish);
  return PD_OK;
}

// Launches the Monte-Carlo draws, their Grams and the top-1 eigenvalues on s
// (eigenvalues to w.prior[0..n_iter)); no host synchronisation.
static pd_status mc_launch(int64_t rows, int64_t cols, int32_t n_iter, uint64_t seed, int32_t precision, void* d_ws,
                           size_t ws_bytes, cudaStream_t s, PatchWork* out) {
  size_t need;
  PD_TRY(pd_nordic_workspace_size(rows, cols, n_iter, &need));
  if (!d_ws || ws_bytes < need) return fail(PD_ERR_WORKSPACE, "workspace too small (%zu < %zu)", ws_bytes, need);
  if (n_iter > 4096) return fail(PD_ERR_UNSUPPORTED, "at most 4096 Monte-Carlo draws");
  const int n = (int)cols;
  size_t used;
  PatchWork w = carve_work(d_ws, n_iter, n, false, &used);
  PD_TRY(cuda_check(cudaMemsetAsync(w.err, 0, sizeof(int), s), "clear error word"));
  int ne = n;  // order of the Grams whose top eigenvalue is taken
  if (precision == PD_PRECISION_MIXED) {
    // the chosen path: each draw's Gram sampled directly from its Wishart law
    // (Bartlett), of order min(rows, cols) (G G^T and G^T G share their top eigenvalue)
    ne = (int)std::min<int64_t>(rows, n);
    launch_wishart(std::max<int64_t>(rows, n), ne, n_iter, seed, (float*)((char*)d_ws + used), w.gram,
                   w.gram_stride, s);
  } else {
    // plain FP32: the explicit rows x cols Gaussian draws and their Grams, as the reference
    float* part = (float*)((char*)d_ws + used);
    launch_mc_gram(rows, n, n_iter, seed, part, w.gram, w.gram_stride, s);
  }
  EigParams ep{};
  ep.method = EIG_MODE_TOP1;
  ep.rows = (int)std::min<int64_t>(rows, INT32_MAX);
  ep.cols = ne;
  PD_TRY(cuda_check(launch_eig(false, ne, ep, w, s), "Monte-Carlo eigensolver launch"));
  *out = w;
  return PD_OK;
}

pd_status pd_nordic_mc_threshold(int64_t rows, int64_t cols, int32_t n_iter, uint64_t seed, int32_t precision,
                                 double* out, void* d_ws, size_t ws_bytes, void* stream) {
  g_err.clear();
  if (!out) return fail(PD_ERR_INVALID, "NULL output");
  cudaStream_t s = (cudaStream_t)stream;
  PatchWork w;
  PD_TRY(mc_launch(rows, cols, n_iter, seed, precision, d_ws, ws_bytes, s, &w));
  double lam[4096];
  PD_TRY(cuda_check(cudaMemcpyAsync(lam, w.prior, sizeof(double) * n_iter, cudaMemcpyDeviceToHost, s), "copy"));
  PD_TRY(cuda_check(cudaStreamSynchronize(s), "Monte-Carlo sync"));
  int err = 0;
  PD_TRY(cuda_check(cudaMemcpy(&err, w.err, sizeof(int), cudaMemcpyDeviceToHost), "copy error word"));
  if (err) return fail(PD_ERR_CUDA, "a device-side wait timed out (code %d)", err);
  double acc = 0.0;
  for (int i = 0; i < n_iter; ++i) acc += sqrt(fmax(lam[i], 0.0));
  *out = acc / n_iter;
  return PD_OK;
}

pd_status pd_nordic_denoise_patches(const pd_geometry* g, const pd_params* p, double noise_std, int64_t mc_rows,
                                    int32_t n_iter, uint64_t seed, double* d_level, void* d_mc_ws, size_t mc_ws_bytes,
                                    const void* d_in, const int32_t* d_patch_list, int64_t n_selected,
                                    void* d_out_acc, float* d_weight_acc, float* d_noise_acc, float* d_noise_ctr,
                                    int32_t* d_rank_map, int32_t* d_patch_rank, float* d_patch_noise, void* d_ws,
                                    size_t ws_bytes, void* stream) {
  g_err.clear();
  PD_TRY(check_geometry(g));
  PD_TRY(check_params(g, p));
  if (p->method != PD_METHOD_RAW) return fail(PD_ERR_INVALID, "pd_nordic_denoise_patches needs method RAW");
  if (!d_level) return fail(PD_ERR_INVALID, "NULL level output");
  cudaStream_t s = (cudaStream_t)stream;
  if (mc_rows < 0) return fail(PD_ERR_INVALID, "negative Monte-Carlo row count");
  cudaEvent_t joined = nullptr;
  if (mc_rows > 0) {
    // the draws, their Grams and top-1 eigenvalues, then the level and the
    // threshold on the device. On the chosen path this chain is a few small
    // launches on about ten SMs, so it runs on a side stream beside the patch
    // means, packing and Grams, and the eigensolver waits for it.
    cudaStream_t ms = s;
    if (p->precision == PD_PRECISION_MIXED) {
      SideStream* side = nullptr;
      PD_TRY(side_stream(&side));
      PD_TRY(cuda_check(cudaEventRecord(side->fork, s), "fork the Monte-Carlo stream"));
      PD_TRY(cuda_check(cudaStreamWaitEvent(side->stream, side->fork, 0), "fork the Monte-Carlo stream"));
      ms = side->stream;
      joined = side->join;
    }
    PatchWork mw;
    PD_TRY(mc_launch(mc_rows, g->cols, n_iter, seed, p->precision, d_mc_ws, mc_ws_bytes, ms, &mw));
    launch_mc_level(mw.prior, n_iter, noise_std, d_level, ms);
    PD_TRY(cuda_check(cudaGetLastError(), "Monte-Carlo level launch"));
    if (joined) PD_TRY(cuda_check(cudaEventRecord(joined, ms), "join the Monte-Carlo stream"));
  }
  // the patch loop reads the threshold from d_level[1]
  const pd_status st = denoise_patches_impl(g, p, d_in, nullptr, d_patch_list, n_selected, d_out_acc, d_weight_acc,
                                            d_noise_acc, d_noise_ctr, d_rank_map, d_patch_rank, d_patch_noise, d_ws,
                                            ws_bytes, stream, d_level + 1, nullptr, joined);
  if (joined && n_selected == 0)  // nothing waited for the side stream: join it here
    PD_TRY(cuda_check(cudaStreamWaitEvent(s, joined, 0), "join the Monte-Carlo stream"));
  return st;
}

pd_status pd_adaptive_qut_level(int64_t rows, int64_t cols, int32_t n_sim, uint64_t seed, int32_t precision,
                                double* out, void* d_ws, size_t ws_bytes, void* stream) {
  g_err.clear();
  if (!out) return fail(PD_ERR_INVALID, "NULL output");
  if (n_sim < 1) return fail(PD_ERR_INVALID, "nbsim must be at least 1");
  if (rows < 1 || cols < 1) return fail(PD_ERR_INVALID, "empty Monte-Carlo problem");
  // the quantile's probability; numpy.quantile rejects it outside [0, 1]
  // (max(rows, cols) < 3), as the reference then fails
  const double q = 1.0 - 1.0 / sqrt(log((double)std::max(rows, cols)));
  if (!(q >= 0.0 && q <= 1.0)) return fail(PD_ERR_INVALID, "Quantiles must be in the range [0, 1]");
  cudaStream_t s = (cudaStream_t)stream;
  PatchWork w;
  PD_TRY(mc_launch(rows, cols, n_sim, seed, precision, d_ws, ws_bytes, s, &w));
  std::vector<double> lam((size_t)n_sim);
  PD_TRY(cuda_check(cudaMemcpyAsync(lam.data(), w.prior, sizeof(double) * n_sim, cudaMemcpyDeviceToHost, s),
                    "copy"));
  PD_TRY(cuda_check(cudaStreamSynchronize(s), "Monte-Carlo sync"));
  int err = 0;
  PD_TRY(cuda_check(cudaMemcpy(&err, w.err, sizeof(int), cudaMemcpyDeviceToHost), "copy error word"));
  if (err) return fail(PD_ERR_CUDA, "a device-side wait timed out (code %d)", err);
  // numpy.quantile(maxd, q), default linear method: sorted v, h = (N - 1) q,
  // v[floor h] + (h - floor h) (v[floor h + 1] - v[floor h])
  for (auto& v : lam) v = sqrt(fmax(v, 0.0));
  std::sort(lam.begin(), lam.end());
  const double h = (double)(n_sim - 1) * q;
  const int64_t lo = std::min<int64_t>(std::max<int64_t>((int64_t)floor(h), 0), n_sim - 1);
  const int64_t hi = std::min<int64_t>(lo + 1, n_sim - 1);
  *out = lam[lo] + (h - (double)lo) * (lam[hi] - lam[lo]);
  return PD_OK;
}

pd_status pd_adaptive_denoise_patches(const pd_geometry* g, const pd_params* p, const pd_adaptive* a,
                                      const void* d_in, const double* d_noise_std, const int32_t* d_patch_list,
                                      int64_t n_selected, void* d_out_acc, float* d_weight_acc, float* d_noise_acc,
                                      float* d_noise_ctr, int32_t* d_rank_map, int32_t* d_patch_rank,
                                      float* d_patch_noise, void* d_ws, size_t ws_bytes, void* stream) {
  g_err.clear();
  if (!p || p->method != PD_METHOD_ADAPTIVE)
    return fail(PD_ERR_INVALID, "pd_adaptive_denoise_patches needs method PD_METHOD_ADAPTIVE");
  if (!a) return fail(PD_ERR_INVALID, "NULL adaptive parameters");
  if (a->mode < PD_ADAPTIVE_SURE || a->mode > PD_ADAPTIVE_QUT)
    return fail(PD_ERR_INVALID, "unknown adaptive mode %d", a->mode);
  if (a->mode == PD_ADAPTIVE_QUT) {
    if (a->n_gamma < 0 || a->n_gamma > 1) return fail(PD_ERR_INVALID, "QUT takes one fixed gamma or none");
    if (!(a->qut_level > 0.0)) return fail(PD_ERR_INVALID, "QUT needs a positive Monte-Carlo level");
  } else if (a->n_gamma < 1 || a->n_gamma > PD_ADAPTIVE_MAX_GAMMA) {
    return fail(PD_ERR_INVALID, "SURE / GSURE need 1 to %d candidate gammas", PD_ADAPTIVE_MAX_GAMMA);
  }
  if (!p->has_prior) return fail(PD_ERR_INVALID, "the adaptive denoiser needs the noise_std map");
  return denoise_patches_impl(g, p, d_in, d_noise_std, d_patch_list, n_selected, d_out_acc, d_weight_acc,
                              d_noise_acc, d_noise_ctr, d_rank_map, d_patch_rank, d_patch_noise, d_ws, ws_bytes,
                              stream, nullptr, a);
}

// ---------------------------------------------------------------------------
// Batched calls over many volumes
// ---------------------------------------------------------------------------
static pd_status batch_check(const pd_volume* vols, int32_t n_vols, const pd_params* p, int* n_max, int* m_max,
                             int64_t* total) {
  if (!vols || n_vols < 1) return fail(PD_ERR_INVALID, "no volumes");
  if (n_vols > PD_BATCH_MAX_VOLUMES)
    return fail(PD_ERR_UNSUPPORTED, "at most %d volumes per batch", PD_BATCH_MAX_VOLUMES);
  if (!p) return fail(PD_ERR_INVALID, "params is NULL");
  if (p->precision != PD_PRECISION_FP32) return fail(PD_ERR_UNSUPPORTED, "batched calls run the FP32 kernels");
  if (p->method == PD_METHOD_ADAPTIVE) return fail(PD_ERR_UNSUPPORTED, "batched calls take MP-PCA, hybrid, raw, optimal");
  *n_max = 0;
  *m_max = 0;
  *total = 0;
  for (int v = 0; v < n_vols; ++v) {
    PD_TRY(check_geometry(&vols[v].geometry));
    PD_TRY(check_params(&vols[v].geometry, p));
    if (vols[v].n_selected < 0) return fail(PD_ERR_INVALID, "negative patch count");
    *n_max = std::max(*n_max, (int)vols[v].geometry.cols);
    *m_max = std::max(*m_max, (int)vols[v].geometry.rows);
    *total += vols[v].n_selected;
  }
  return PD_OK;
}

static size_t batch_table_bytes(int32_t n_vols, int64_t total) {
  return align256(sizeof(VolDesc) * n_vols) + 2 * align256(sizeof(int32_t) * std::max<int64_t>(total, 1));
}

pd_status pd_denoise_batch_workspace_size(const pd_volume* vols, int32_t n_vols, const pd_params* p,
                                          int64_t chunk_patches, size_t* bytes) {
  g_err.clear();
  int n_max, m_max;
  int64_t total;
  PD_TRY(batch_check(vols, n_vols, p, &n_max, &m_max, &total));
  if (!bytes) return fail(PD_ERR_INVALID, "NULL output");
  const bool cplx = p->is_complex != 0;
  int64_t chunk = (int64_t)std::max<size_t>(1, BATCH_CHUNK_BUDGET / per_patch_bytes(n_max, cplx));
  if (chunk_patches > 0) chunk = std::min(chunk, chunk_patches);
  chunk = std::min<int64_t>(chunk, std::max<int64_t>(total, 1));
  *bytes = work_bytes((int)chunk, n_max, cplx) + batch_table_bytes(n_vols, total);
  return PD_OK;
}

pd_status pd_denoise_batch(const pd_volume* vols, int32_t n_vols, const pd_params* p, const pd_batch_tuning* tuning,
                           void* d_ws, size_t ws_bytes, void* stream) {
  g_err.clear();
  int n_max, m_max;
  int64_t total;
  PD_TRY(batch_check(vols, n_vols, p, &n_max, &m_max, &total));
  const bool cplx = p->is_complex != 0;
  for (int v = 0; v < n_vols; ++v) {
    const pd_volume& vv = vols[v];
    if (vv.n_selected > 0 && (!vv.d_in || !vv.d_patch_list || !vv.d_out_acc || !vv.d_weight_acc ||
                              !vv.d_noise_acc || !vv.d_noise_ctr || !vv.d_rank_map || !vv.d_patch_rank ||
                              !vv.d_patch_noise))
      return fail(PD_ERR_INVALID, "NULL buffer in volume %d", v);
    if ((p->method == PD_METHOD_HYBRID || (p->method == PD_METHOD_OPTIMAL && p->has_prior)) && !vv.d_noise_std)
      return fail(PD_ERR_INVALID, "volume %d needs its noise_std map", v);
  }
  if (total == 0) return PD_OK;
  pd_batch_tuning tn{};
  tn.order_by_cost = 1;
  if (tuning) tn = *tuning;
  // work-list order: the costliest patches (eigensolver ~ frames^3) first, so
  // the last wave holds the cheapest ones
  std::vector<int> order(n_vols);
  for (int v = 0; v < n_vols; ++v) order[v] = v;
  if (tn.order_by_cost)
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return vols[a].geometry.cols > vols[b].geometry.cols; });
  // the table: error word and patch work first (offset 0 of the workspace), then volumes and lists
  const size_t tbl = batch_table_bytes(n_vols, total);
  if (!d_ws || ws_bytes < tbl + work_bytes(1, n_max, cplx))
    return fail(PD_ERR_WORKSPACE, "workspace too small (%zu < %zu)", ws_bytes, tbl + work_bytes(1, n_max, cplx));
  const size_t room = ws_bytes - tbl;
  int64_t chunk = std::max<int64_t>(1, (int64_t)(room / per_patch_bytes(n_max, cplx)));
  if (tn.chunk_patches > 0) chunk = std::min(chunk, tn.chunk_patches);
  chunk = std::min(chunk, total);
  while (chunk > 1 && work_bytes((int)chunk, n_max, cplx) > room) --chunk;
  size_t used;
  carve_work(d_ws, (int)chunk, n_max, cplx, &used);
  char* tb = (char*)d_ws + used;
  VolDesc* d_vols = (VolDesc*)tb;
  int32_t* d_list = (int32_t*)(tb + align256(sizeof(VolDesc) * n_vols));
  int32_t* d_volof = d_list + align256(sizeof(int32_t) * total) / sizeof(int32_t);
  static thread_local BatchTable t;  // 16 KB: a kernel parameter, built on the host
  int64_t first = 0;
  for (int k = 0; k < n_vols; ++k) {
    const pd_volume& vv = vols[order[k]];
    VolDesc& d = t.v[k].d;
    d.g = to_geo(vv.geometry);
    d.in = vv.d_in;
    d.noise_std = vv.d_noise_std;
    d.out = vv.d_out_acc;
    d.wacc = vv.d_weight_acc;
    d.nacc = vv.d_noise_acc;
    d.nctr = vv.d_noise_ctr;
    d.rank_map = vv.d_rank_map;
    d.prank = vv.d_patch_rank;
    d.pnoise = vv.d_patch_noise;
    d.threshold = vv.threshold;
    d.mp_median = vv.mp_median;
    d.first = first;
    t.v[k].list = vv.d_patch_list;
    t.v[k].count = vv.n_selected;
    first += vv.n_selected;
  }
  cudaStream_t s = (cudaStream_t)stream;
  PD_TRY(cuda_check(cudaMemsetAsync(d_ws, 0, sizeof(int), s), "clear error word"));
  launch_batch_setup(t, n_vols, total, d_vols, d_list, d_volof, s);
  // the launch shapes follow the largest patch of the batch; each CTA reads its own
  Geo G{};
  G.rows = m_max;
  G.cols = n_max;
  EigParams ep{};
  ep.method = p->method;
  ep.loss = p->loss;
  ep.has_prior = p->has_prior;
  ep.rows = m_max;
  ep.cols = n_max;
  ep.threshold_scale = p->threshold_scale;
  // chunks of at most `chunk` patches that do not mix the kernels' frame-count
  // classes (their register slots per lane are sized by the largest frame count
  // of a launch), in work-list order
  // (the classes also separate the patches the eigensolver runs in small CTAs,
  // so a batched patch takes the same kernel variant as a one-volume call)
  auto frame_class = [cplx](int64_t n) {
    const int c = n <= 64 ? 0 : n <= 128 ? 1 : n <= 224 ? 2 : n <= 320 ? 3 : 4;
    return 2 * c + (eig_small(cplx, (int)n) ? 0 : 1);
  };
  std::vector<std::pair<int64_t, int64_t>> pieces;  // (offset, count)
  {
    int64_t start = 0, len = 0;
    int cls = -1;
    for (int k = 0; k < n_vols; ++k) {
      int64_t f = t.v[k].d.first, c = t.v[k].count;
      if (c == 0) continue;
      const int kc = frame_class(t.v[k].d.g.cols);
      if (len > 0 && kc != cls) {
        pieces.emplace_back(start, len);
        len = 0;
      }
      cls = kc;
      while (c > 0) {
        if (len == 0) start = f;
        const int64_t take = std::min<int64_t>(c, chunk - len);
        len += take;
        f += take;
        c -= take;
        if (len == chunk) {
          pieces.emplace_back(start, len);
          len = 0;
        }
      }
    }
    if (len > 0) pieces.emplace_back(start, len);
  }
  for (const auto& pc : pieces) {
    const int64_t off = pc.first;
    const int cnt = (int)pc.second;
    PatchWork w = carve_work(d_ws, cnt, n_max, cplx, &used);
    w.list = d_list + off;
    w.vols = d_vols;
    w.vol_of = d_volof + off;
    // this chunk's volumes set its launch shapes (the work list is in volume order)
    int nc = 0, mc = 0;
    size_t esm = 0;
    for (int k = 0; k < n_vols; ++k) {
      const int64_t f = t.v[k].d.first, c = t.v[k].count;
      if (c == 0 || f + c <= off || f >= off + cnt) continue;
      nc = std::max(nc, (int)t.v[k].d.g.cols);
      mc = std::max(mc, (int)t.v[k].d.g.rows);
      esm = std::max(esm, eig_launch_smem(cplx, (int)t.v[k].d.g.cols));
    }
    G.rows = mc;
    G.cols = nc;
    ep.rows = mc;
    ep.cols = nc;
    ep.smem_bytes = esm;
    launch_patch_mean(G, cplx, nullptr, w, s);
    if (p->method == PD_METHOD_HYBRID || (p->method == PD_METHOD_OPTIMAL && p->has_prior))
      launch_prior(G, p->method, nullptr, w, s);
    launch_gram_fp32(G, cplx, nullptr, w, s);
    PD_TRY(cuda_check(launch_eig(cplx, nc, ep, w, s), "eigensolver launch"));
    SynthArgs sa{};
    sa.recombination = p->recombination;
    sa.list_offset = off;
    sa.row_blocks = tn.synth_row_blocks;
    launch_synth(G, cplx, nullptr, w, sa, s);
    PD_TRY(cuda_check(cudaGetLastError(), "pd_denoise_batch launch"));
  }
  return PD_OK;
}

// ---------------------------------------------------------------------------
// Backward pass of the low-rank denoiser (real volumes)
// ---------------------------------------------------------------------------
static size_t bwd_extra_bytes(int count, int n) {
  Carver c(nullptr);
  c.take<float>((size_t)count * n * n);  // cross
  c.take<float>((size_t)count * n * n);  // k1
  c.take<float>((size_t)count * n * n);  // k2
  c.take<float>((size_t)count * n);      // gmean
  c.take<float>((size_t)count * n);      // u
  return c.off;
}

static pd_status check_backward(const pd_geometry* g, int32_t recombination, int32_t shrink) {
  PD_TRY(check_geometry(g));
  if (recombination != PD_RECOMB_WEIGHTED && recombination != PD_RECOMB_AVERAGE)
    return fail(PD_ERR_INVALID, "the backward pass needs 'weighted' or 'average' recombination");
  if (shrink != 0 && shrink != 1) return fail(PD_ERR_INVALID, "shrink must be 0 (soft) or 1 (hard)");
  if (!bwd_supported((int)g->cols))
    return fail(PD_ERR_UNSUPPORTED, "the backward pass handles at most 128 frames per patch (got %lld)",
                (long long)g->cols);
  if (g->rows <= g->cols)
    return fail(PD_ERR_UNSUPPORTED, "the backward pass needs more voxels than frames per patch (M > T)");
  return PD_OK;
}

pd_status pd_lowrank_backward_workspace_size(const pd_geometry* g, int64_t n_selected, size_t* bytes) {
  g_err.clear();
  PD_TRY(check_backward(g, PD_RECOMB_AVERAGE, 0));
  if (!bytes) return fail(PD_ERR_INVALID, "NULL output");
  const int n = (int)g->cols;
  const size_t pp = per_patch_bytes(n, false) + (size_t)3 * n * n * 4 + (size_t)2 * n * 4 + 5 * 256;
  int64_t chunk = (int64_t)std::max<size_t>(1, DEFAULT_CHUNK_BUDGET / pp);
  chunk = std::min<int64_t>(chunk, std::max<int64_t>(n_selected, 1));
  *bytes = work_bytes((int)chunk, n, false) + bwd_extra_bytes((int)chunk, n);
  return PD_OK;
}

pd_status pd_lowrank_backward(const pd_geometry* g, int32_t recombination, int32_t shrink, const float* d_in,
                              const double* d_noise_std, double level, const int32_t* d_patch_list,
                              int64_t n_selected, const int32_t* d_patch_rank, const float* d_weights,
                              const float* d_gout, float* d_gin, double* d_dlevel, void* d_ws, size_t ws_bytes,
                              void* stream) {
  g_err.clear();
  PD_TRY(check_backward(g, recombination, shrink));
  if (n_selected == 0) return PD_OK;
  if (!d_in || !d_patch_list || !d_patch_rank || !d_weights || !d_gout || !d_gin || !d_dlevel)
    return fail(PD_ERR_INVALID, "NULL buffer");
  if (shrink == 0 && !d_noise_std) return fail(PD_ERR_INVALID, "the soft threshold needs the noise_std map");
  const int n = (int)g->cols;
  const size_t one = work_bytes(1, n, false) + bwd_extra_bytes(1, n);
  if (!d_ws || ws_bytes < one) return fail(PD_ERR_WORKSPACE, "workspace too small (%zu < %zu)", ws_bytes, one);
  // per-patch bytes without the alignment slack: an upper bound on the chunk
  const size_t pp = per_patch_bytes(n, false) + (size_t)3 * n * n * 4 + (size_t)2 * n * 4;
  int64_t chunk = std::min<int64_t>(n_selected, std::max<int64_t>(1, (int64_t)(ws_bytes / pp)));
  while (chunk > 1 && work_bytes((int)chunk, n, false) + bwd_extra_bytes((int)chunk, n) > ws_bytes) --chunk;
  cudaStream_t s = (cudaStream_t)stream;
  const Geo G = to_geo(*g);
  EigParams ep{};
  ep.method = EIG_MODE_FULL;
  ep.rows = (int)g->rows;
  ep.cols = n;
  PD_TRY(cuda_check(cudaMemsetAsync(d_ws, 0, sizeof(int), s), "clear error word"));
  for (int64_t off = 0; off < n_selected; off += chunk) {
    const int cnt = (int)std::min<int64_t>(chunk, n_selected - off);
    size_t used;
    PatchWork w = carve_work(d_ws, cnt, n, false, &used);
    w.list = d_patch_list + off;
    Carver c((char*)d_ws + used);
    BwdWork b{};
    b.recombination = recombination;
    b.shrink = shrink;
    b.level = level;
    b.rank = d_patch_rank + off;
    b.cross = c.take<float>((size_t)cnt * n * n);
    b.k1 = c.take<float>((size_t)cnt * n * n);
    b.k2 = c.take<float>((size_t)cnt * n * n);
    b.mat_stride = (int64_t)n * n;
    b.gmean = c.take<float>((size_t)cnt * n);
    b.u = c.take<float>((size_t)cnt * n);
    b.dlevel = d_dlevel + off;
    // the forward's factorisation, recomputed in FP32: mean, Gram, every eigenpair
    launch_patch_mean(G, false, d_in, w, s);
    if (shrink == 0) launch_prior(G, PD_METHOD_ADAPTIVE, d_noise_std, w, s);
    launch_gram_fp32(G, false, d_in, w, s);
    PD_TRY(cuda_check(launch_eig(false, n, ep, w, s), "eigensolver launch"));
    PD_TRY(cuda_check(launch_backward(G, d_in, d_gout, d_weights, d_gin, w, b, s), "backward launch"));
  }
  return PD_OK;
}

// Spatial extents padded to 3 axes (block 1 on padded axes) and frame count.
static pd_status noise_geometry(int32_t ndim, const int64_t* shape, int32_t block, int64_t dims[3], int blk[3],
                                int* frames) {
  if (!shape || ndim < 2 || ndim > 4) return fail(PD_ERR_INVALID, "need 1 to 3 spatial axes and a time axis");
  if (block < 1) return fail(PD_ERR_INVALID, "block_size must be at least 1");
  const int nsp = ndim - 1;
  for (int i = 0; i < 3; ++i) {
    dims[i] = i < nsp ? shape[i] : 1;
    blk[i] = i < nsp ? block : 1;
    if (i < nsp && shape[i] <= block)
      return fail(PD_ERR_INVALID, "axis %d has %lld voxels, not more than block_size %d", i, (long long)shape[i],
                  block);
  }
  if (shape[ndim - 1] < 1 || shape[ndim - 1] > INT32_MAX) return fail(PD_ERR_INVALID, "bad frame count");
  *frames = (int)shape[ndim - 1];
  return PD_OK;
}

pd_status pd_estimate_noise_workspace_size(int32_t ndim, const int64_t* shape, int32_t is_complex, size_t* bytes) {
  g_err.clear();
  if (!bytes) return fail(PD_ERR_INVALID, "NULL output");
  int64_t dims[3];
  int blk[3], T;
  PD_TRY(noise_geometry(ndim, shape, 1, dims, blk, &T));
  const size_t nvox = (size_t)(dims[0] * dims[1] * dims[2]);
  *bytes = align256(sizeof(double) * nvox * (is_complex ? 2 : 1)) + align256(sizeof(double) * nvox);
  return PD_OK;
}

pd_status pd_estimate_noise(int32_t ndim, const int64_t* shape, int32_t is_complex, const void* d_in,
                            int32_t block_size, double* d_noise_map, void* d_ws, size_t ws_bytes, void* stream) {
  g_err.clear();
  int64_t dims[3];
  int blk[3], T;
  PD_TRY(noise_geometry(ndim, shape, block_size, dims, blk, &T));
  if (!d_in || !d_noise_map) return fail(PD_ERR_INVALID, "NULL buffer");
  size_t need;
  PD_TRY(pd_estimate_noise_workspace_size(ndim, shape, is_complex, &need));
  if (!d_ws || ws_bytes < need) return fail(PD_ERR_WORKSPACE, "workspace too small (%zu < %zu)", ws_bytes, need);
  const size_t nvox = (size_t)(dims[0] * dims[1] * dims[2]);
  Carver c(d_ws);
  double* mean = c.take<double>(nvox * (is_complex ? 2 : 1));
  double* m2 = c.take<double>(nvox);
  launch_estimate_noise((const float*)d_in, is_complex != 0, dims, blk, T, mean, m2, d_noise_map,
                        (cudaStream_t)stream);
  return cuda_check(cudaGetLastError(), "pd_estimate_noise launch");
}

pd_status pd_workspace_check(const void* d_workspace, void* stream) {
  g_err.clear();
  if (!d_workspace) return fail(PD_ERR_INVALID, "NULL workspace");
  int err = 0;
  cudaStream_t s = (cudaStream_t)stream;
  PD_TRY(cuda_check(cudaMemcpyAsync(&err, d_workspace, sizeof(int), cudaMemcpyDeviceToHost, s), "copy error word"));
  PD_TRY(cuda_check(cudaStreamSynchronize(s), "workspace check sync"));
  if (err == PD_DEVERR_NONFINITE) return fail(PD_ERR_INVALID, "array must not contain infs or NaNs");
  if (err) return fail(PD_ERR_CUDA, "a device-side wait timed out (code %d)", err);
  return PD_OK;
}

}  // extern "C"

namespace pd {
// Sets the message pd_last_error() returns on this host thread.
void set_last_error(const char* msg) { g_err = msg; }
}  // namespace pd
