// Patch mean, noise-prior reduction and the plain FP32 (SIMT) centred Gram.
//
// Casorati matrix of a patch: row r = voxel r of the patch (C order over the
// spatial patch), column t = frame t0 + t; rows are contiguous runs of frames in
// the (X,Y,Z,T) volume. The mean is over voxels (axis 0), as in eig_analysis /
// svd_analysis (space_time/utils.py:73,128). The Gram is C = Xc^H Xc (frames x
// frames, unscaled), stored packed lower column-major per patch.
#include "pd_common.cuh"
#include "pd_kernels.cuh"
#include "pd_profile.cuh"

namespace pd {

constexpr int MEAN_THREADS = 256;
constexpr int GT = 64;   // Gram tile edge
constexpr int GK = 16;   // rows per k step
constexpr int GRAM_THREADS = 256;

// grid: patches x 64-column chunks, flattened patch-major; 256 threads = 64
// columns x 4 row groups. A thread sums the rows r = group (mod 4) of its column
// with two FP64 partial sums (more loads in flight); the groups' sums combine
// in a fixed order, so the mean is deterministic.
constexpr int MEAN_COLS = 64;
constexpr int MEAN_GROUPS = MEAN_THREADS / MEAN_COLS;

template <bool CPLX>
__global__ void __launch_bounds__(MEAN_THREADS) k_patch_mean(Geo g, const typename Elem<CPLX>::T* __restrict__ in,
                                                             PatchWork w, int chunks) {
  using T = typename Elem<CPLX>::T;
  extern __shared__ int64_t rowbase[];
  __shared__ double part[MEAN_GROUPS][MEAN_COLS][2];
  const int p = (int)(blockIdx.x / (unsigned)chunks);
  const int c0 = (int)(blockIdx.x - (unsigned)p * (unsigned)chunks) * MEAN_COLS;
  if (w.vols) {  // batched call: this patch's volume
    const VolDesc& v = w.vols[w.vol_of[p]];
    g = v.g;
    in = reinterpret_cast<const T*>(v.in);
  }
  const int64_t idx = w.list[p];
  int64_t o[4];
  patch_origin(g, idx, o);
  const int M = g.rows, n = g.cols;
  if (c0 >= n) return;  // a batched chunk sized for a longer volume
  for (int r = threadIdx.x; r < M; r += blockDim.x) rowbase[r] = row_voxel(g, o, r) * g.shape[3] + o[3];
  __syncthreads();
  const int c = threadIdx.x % MEAN_COLS, grp = threadIdx.x / MEAN_COLS;
  const int t = c0 + c;
  double sx[2] = {0.0, 0.0}, sy[2] = {0.0, 0.0};
  if (t < n) {
    int r = grp;
    for (; r + MEAN_GROUPS < M; r += 2 * MEAN_GROUPS) {
      const T a = in[rowbase[r] + t];
      const T b = in[rowbase[r + MEAN_GROUPS] + t];
      if constexpr (CPLX) {
        sx[0] += a.x;
        sy[0] += a.y;
        sx[1] += b.x;
        sy[1] += b.y;
      } else {
        sx[0] += a;
        sx[1] += b;
      }
    }
    if (r < M) {
      const T a = in[rowbase[r] + t];
      if constexpr (CPLX) {
        sx[0] += a.x;
        sy[0] += a.y;
      } else {
        sx[0] += a;
      }
    }
  }
  part[grp][c][0] = sx[0] + sx[1];
  part[grp][c][1] = sy[0] + sy[1];
  __syncthreads();
  if (grp == 0 && t < n) {
    double ax = part[0][c][0], ay = part[0][c][1];
#pragma unroll
    for (int q = 1; q < MEAN_GROUPS; ++q) {
      ax += part[q][c][0];
      ay += part[q][c][1];
    }
    T* mean = reinterpret_cast<T*>(w.mean) + (int64_t)p * w.n_stride;
    if constexpr (CPLX) {
      mean[t] = cf{(float)(ax / M), (float)(ay / M)};
    } else {
      mean[t] = (float)(ax / M);
    }
    // A NaN or infinite sample makes the sum non-finite (float samples cannot
    // overflow an FP64 sum): the reference's LAPACK calls reject such a patch
    // ("array must not contain infs or NaNs"), so flag it.
    if (!isfinite(ax) || !isfinite(ay)) atomicExch(w.err, PD_DEVERR_NONFINITE);
  }
}

// Hybrid: varest = mean(noise_std^2) over the patch; optimal: sigma = mean(|noise_std|);
// adaptive: mean(noise_std^2), whose root is the patch's stdest.
// (space_time/lowrank.py:106, :389 and :617; the maps are constant along time so
// the 4D patch mean equals the spatial one.)
__global__ void k_prior(Geo g, int method, const double* ns, PatchWork w) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int p = warp; p < w.count; p += nwarps) {
    if (w.vols) {  // batched call: this patch's volume
      const VolDesc& v = w.vols[w.vol_of[p]];
      g = v.g;
      ns = v.noise_std;
    }
    int64_t o[4];
    patch_origin(g, w.list[p], o);
    double s = 0.0;
    for (int r = lane; r < g.rows; r += 32) {
      const double v = ns[row_voxel(g, o, r)];
      s += (method == PD_METHOD_HYBRID || method == PD_METHOD_ADAPTIVE) ? v * v : sqrt(v * v);
    }
    s = warp_sum(s);
    if (lane == 0) w.prior[p] = s / g.rows;
  }
}

// Tile pair index -> (bi, bj), bi >= bj, row-major over the lower block triangle.
__device__ __forceinline__ void tile_pair(int t, int& bi, int& bj) {
  int i = (int)((sqrtf(8.f * t + 1.f) - 1.f) * 0.5f);
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  while (i * (i + 1) / 2 > t) --i;
  bi = i;
  bj = t - i * (i + 1) / 2;
}

// Register-tiled 64x64 block of C = Xc^H Xc for one patch (grid.x = patch,
// grid.y = lower tile pair).
template <bool CPLX>
__global__ void __launch_bounds__(GRAM_THREADS) k_gram_fp32(Geo g, const typename Elem<CPLX>::T* __restrict__ in,
                                                            PatchWork w) {
  using T = typename Elem<CPLX>::T;
  __shared__ T As[GK][GT];
  __shared__ T Bs[GK][GT];
  __shared__ T mA[GT], mB[GT];
  __shared__ int64_t rb[GK];
  const int p = blockIdx.x;
  if (w.vols) {  // batched call: this patch's volume
    const VolDesc& v = w.vols[w.vol_of[p]];
    g = v.g;
    in = reinterpret_cast<const T*>(v.in);
  }
  int bi, bj;
  tile_pair(blockIdx.y, bi, bj);
  const int n = g.cols, M = g.rows;
  if (bi * GT >= n) return;  // a tile of a larger patch of the batch
  int64_t o[4];
  patch_origin(g, w.list[p], o);
  const T* mean = reinterpret_cast<const T*>(w.mean) + (int64_t)p * w.n_stride;
  const int tid = threadIdx.x;
  if (tid < GT) {
    const int ca = bi * GT + tid, cb = bj * GT + tid;
    mA[tid] = ca < n ? mean[ca] : zero<T>();
    mB[tid] = cb < n ? mean[cb] : zero<T>();
  }
  const int ty = tid / 16, tx = tid % 16;
  const int lc = tid % GT, lr = tid / GT;  // load column, first load row
  T acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = zero<T>();
  const bool diag = (bi == bj);
  const int ca = bi * GT + lc, cb = bj * GT + lc;
  for (int r0 = 0; r0 < M; r0 += GK) {
    __syncthreads();
    if (tid < GK) rb[tid] = (r0 + tid < M) ? row_voxel(g, o, r0 + tid) * g.shape[3] + o[3] : -1;
    __syncthreads();
#pragma unroll
    for (int q = 0; q < GK / 4; ++q) {
      const int kk = lr + 4 * q;
      const int64_t base = rb[kk];
      T va = zero<T>(), vb = zero<T>();
      if (base >= 0) {
        if (ca < n) va = in[base + ca] - mA[lc];
        if (!diag && cb < n) vb = in[base + cb] - mB[lc];
      }
      As[kk][lc] = va;
      if (!diag) Bs[kk][lc] = vb;
    }
    __syncthreads();
    const T(*Bp)[GT] = diag ? As : Bs;
    // two-level sum: the 16 rows of this step, then the running total
    T part[4][4];
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y) part[x][y] = zero<T>();
#pragma unroll
    for (int kk = 0; kk < GK; ++kk) {
      T a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a[q] = As[kk][ty * 4 + q];
        b[q] = Bp[kk][tx * 4 + q];
      }
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) part[x][y] = part[x][y] + cmulc(a[x], b[y]);
    }
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y) acc[x][y] = acc[x][y] + part[x][y];
  }
  T* C = reinterpret_cast<T*>(w.gram) + (int64_t)p * (w.gram_stride / (CPLX ? 2 : 1));
#pragma unroll
  for (int x = 0; x < 4; ++x) {
    const int i = bi * GT + ty * 4 + x;
#pragma unroll
    for (int y = 0; y < 4; ++y) {
      const int j = bj * GT + tx * 4 + y;
      if (i < n && j <= i) C[pk(i, j, n)] = acc[x][y];
    }
  }
}

void launch_patch_mean(const Geo& g, bool cplx, const void* in, const PatchWork& w, cudaStream_t s) {
  const size_t smem = sizeof(int64_t) * (size_t)g.rows;
  if (smem > 48 * 1024) {
    cudaFuncSetAttribute(k_patch_mean<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_patch_mean<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  const int chunks = (g.cols + MEAN_COLS - 1) / MEAN_COLS;
  const unsigned grid = (unsigned)((int64_t)w.count * chunks);
  if (cplx)
    PD_TIMED("patch_mean", s, k_patch_mean<true><<<grid, MEAN_THREADS, smem, s>>>(g, (const cf*)in, w, chunks));
  else
    PD_TIMED("patch_mean", s, k_patch_mean<false><<<grid, MEAN_THREADS, smem, s>>>(g, (const float*)in, w, chunks));
}

void launch_prior(const Geo& g, int method, const double* ns, const PatchWork& w, cudaStream_t s) {
  const int blocks = (w.count * 32 + 255) / 256;
  PD_TIMED("prior", s, k_prior<<<blocks, 256, 0, s>>>(g, method, ns, w));
}

void launch_gram_fp32(const Geo& g, bool cplx, const void* in, const PatchWork& w, cudaStream_t s) {
  const int nt = (g.cols + GT - 1) / GT;
  dim3 grid(w.count, nt * (nt + 1) / 2);
  if (cplx)
    PD_TIMED("gram_fp32", s, k_gram_fp32<true><<<grid, GRAM_THREADS, 0, s>>>(g, (const cf*)in, w));
  else
    PD_TIMED("gram_fp32", s, k_gram_fp32<false><<<grid, GRAM_THREADS, 0, s>>>(g, (const float*)in, w));
}

}  // namespace pd
