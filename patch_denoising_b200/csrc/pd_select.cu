// Patch selection: mask fill per patch and ascending compaction of the kept
// patch indices. Mirrors the selection loop of BaseSpaceTimeDenoiser.denoise
// (space_time/base.py:202-227): keep patch i iff 100 * sum(mask patch) / size > thr.
#include "pd_common.cuh"
#include "pd_kernels.cuh"

namespace pd {

// Per voxel and time window: number of true mask frames inside the window.
__global__ void k_window_counts(Geo g, const uint8_t* __restrict__ mask4, int32_t* __restrict__ cnt) {
  const int64_t nvox = g.shape[0] * g.shape[1] * g.shape[2];
  const int64_t gt_n = g.grid[3];
  const int64_t total = nvox * gt_n;
  const int64_t T = g.shape[3];
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = e / gt_n, w = e % gt_n;
    const uint8_t* m = mask4 + v * T + w * g.step[3];
    int32_t c = 0;
    for (int64_t t = 0; t < g.patch[3]; ++t) c += m[t] != 0;
    cnt[e] = c;
  }
}

// One warp per patch: count true mask elements in the 4D patch and decide.
// mode 0: no mask (all true); 1: 3D mask broadcast over time; 2: 4D mask via
// the per-window counts.
__global__ void k_patch_flags(Geo g, int mode, const uint8_t* __restrict__ mask3,
                              const int32_t* __restrict__ cnt, double thr,
                              uint8_t* __restrict__ flags) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t size = (int64_t)g.rows * g.patch[3];
  for (int64_t p = warp; p < g.n_patches; p += nwarps) {
    long long c = 0;
    if (mode == 0) {
      c = size;
    } else {
      int64_t o[4];
      patch_origin(g, p, o);
      const int64_t w = patch_window(g, p);
      for (int r = lane; r < g.rows; r += 32) {
        const int64_t v = row_voxel(g, o, r);
        c += (mode == 1) ? (long long)(mask3[v] != 0) * g.patch[3]
                         : (long long)cnt[v * g.grid[3] + w];
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
    }
    if (lane == 0) {
      // (100 * count) / size > thr, in IEEE double exactly as NumPy evaluates it.
      const double frac = (double)(100 * c) / (double)size;
      flags[p] = frac > thr ? 1 : 0;
    }
  }
}

// Inclusive block scan of one int per thread (blockDim.x <= 1024). Returns the
// inclusive prefix; *total receives the block total.
__device__ __forceinline__ int block_incl_scan(int v, int* warp_tot, int* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  if (lane == 31) warp_tot[w] = v;
  __syncthreads();
  if (w == 0) {
    int t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += u;
    }
    if (lane < nw) warp_tot[lane] = t;
  }
  __syncthreads();
  if (w > 0) v += warp_tot[w - 1];
  *total = warp_tot[nw - 1];
  __syncthreads();
  return v;
}

// Count kept flags per SEL_BLOCK-sized chunk.
__global__ void k_block_counts(const uint8_t* __restrict__ flags, int64_t n, int32_t* __restrict__ bc) {
  __shared__ int wt[32];
  const int64_t base = (int64_t)blockIdx.x * SEL_BLOCK + (int64_t)threadIdx.x * SEL_PER_THREAD;
  int c = 0;
#pragma unroll
  for (int i = 0; i < SEL_PER_THREAD; ++i)
    if (base + i < n) c += flags[base + i];
  int tot;
  block_incl_scan(c, wt, &tot);
  if (threadIdx.x == 0) bc[blockIdx.x] = tot;
}

// Exclusive scan of the block counts (single block); writes the total kept.
__global__ void k_scan_counts(int32_t* __restrict__ bc, int64_t nb, int32_t* __restrict__ total_out) {
  __shared__ int wt[32];
  int carry = 0;
  for (int64_t s = 0; s < nb; s += blockDim.x) {
    const int64_t i = s + threadIdx.x;
    const int v = i < nb ? bc[i] : 0;
    int tot;
    const int incl = block_incl_scan(v, wt, &tot);
    if (i < nb) bc[i] = carry + incl - v;
    carry += tot;
  }
  if (threadIdx.x == 0) *total_out = carry;
}

// Write the kept indices, ascending.
__global__ void k_compact(const uint8_t* __restrict__ flags, int64_t n, const int32_t* __restrict__ boff,
                          int32_t* __restrict__ list) {
  __shared__ int wt[32];
  const int64_t base = (int64_t)blockIdx.x * SEL_BLOCK + (int64_t)threadIdx.x * SEL_PER_THREAD;
  int c = 0;
#pragma unroll
  for (int i = 0; i < SEL_PER_THREAD; ++i)
    if (base + i < n) c += flags[base + i];
  int tot;
  const int incl = block_incl_scan(c, wt, &tot);
  int pos = boff[blockIdx.x] + incl - c;
#pragma unroll
  for (int i = 0; i < SEL_PER_THREAD; ++i)
    if (base + i < n && flags[base + i]) list[pos++] = (int32_t)(base + i);
}

}  // namespace pd
