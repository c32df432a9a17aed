// Noise map of a noise-only sequence: estimate_noise (space_time/utils.py:207-242).
//
// The reference visits every block of b voxels per spatial axis (overlap b - 1,
// so every position: utils.py:226-228 with get_patch_locs, utils.py:8-55) and
// writes, at the voxel b // 2 past the block's corner, the population standard
// deviation of the block's samples over all frames. Here that is two passes:
//   k_voxel_moments  a warp per voxel: mean and sum of squared deviations over
//                    the frames from shifted FP64 sums (one read, HBM-bound);
//   k_block_std      a thread per voxel: if it is a block centre, combine the
//                    block's b^d voxel moments exactly (equal counts T:
//                    M2 = sum_v [M2_v + T |mean_v - mean|^2]) and take
//                    sqrt(M2 / (b^d T)); otherwise 0.
#include <cuda_runtime.h>

#include <algorithm>

#include "pd_common.cuh"
#include "pd_kernels.cuh"
#include "pd_profile.cuh"

namespace pd {

// One read of each voxel's frames: sums of (x - x0) and |x - x0|^2 with x0 the
// voxel's first frame (the shift keeps the FP64 moments exact to rounding for
// any mean), then mean = x0 + S / T and M2 = Q - |S|^2 / T.
template <bool CPLX>
__global__ void __launch_bounds__(256) k_voxel_moments(const float* __restrict__ in, int64_t nvox, int T,
                                                       double* __restrict__ mean, double* __restrict__ m2) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t v = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; v < nvox; v += warps) {
    double sr = 0.0, si = 0.0, q = 0.0, x0r, x0i = 0.0;
    // four loads in flight per lane before the FP64 arithmetic
    if constexpr (CPLX) {
      const float2* row = reinterpret_cast<const float2*>(in) + v * T;
      const float2 f = row[0];
      x0r = f.x;
      x0i = f.y;
      for (int t0 = lane; t0 < T; t0 += 128) {
        float2 x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) x[u] = (t0 + 32 * u < T) ? row[t0 + 32 * u] : f;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const double dr = (double)x[u].x - x0r, di = (double)x[u].y - x0i;  // padding adds 0
          sr += dr;
          si += di;
          q += dr * dr + di * di;
        }
      }
    } else {
      const float* row = in + v * T;
      const float f = row[0];
      x0r = f;
      for (int t0 = lane; t0 < T; t0 += 128) {
        float x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) x[u] = (t0 + 32 * u < T) ? row[t0 + 32 * u] : f;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const double dr = (double)x[u] - x0r;  // padding adds 0
          sr += dr;
          q += dr * dr;
        }
      }
    }
    sr = warp_sum(sr);
    if (CPLX) si = warp_sum(si);
    q = warp_sum(q);
    if (lane == 0) {
      mean[(CPLX ? 2 : 1) * v] = x0r + sr / T;
      if (CPLX) mean[2 * v + 1] = x0i + si / T;
      m2[v] = fmax(q - (sr * sr + si * si) / T, 0.0);
    }
  }
}

// dims: spatial extents padded to 3 (padded axes have extent 1 and block 1).
template <bool CPLX>
__global__ void __launch_bounds__(256) k_block_std(const double* __restrict__ mean, const double* __restrict__ m2,
                                                   int64_t d0, int64_t d1, int64_t d2, int b0, int b1, int b2, int T,
                                                   double* __restrict__ out) {
  const int64_t nvox = d0 * d1 * d2;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nvox; v += (int64_t)gridDim.x * blockDim.x) {
    const int64_t z = v % d2, y = (v / d2) % d1, x = v / (d1 * d2);
    const int64_t t0 = x - b0 / 2, t1 = y - b1 / 2, t2 = z - b2 / 2;  // block corner
    if (t0 < 0 || t1 < 0 || t2 < 0 || t0 > d0 - b0 || t1 > d1 - b1 || t2 > d2 - b2) {
      out[v] = 0.0;
      continue;
    }
    const int K = b0 * b1 * b2;
    double ur = 0.0, ui = 0.0;
    for (int i = 0; i < b0; ++i)
      for (int j = 0; j < b1; ++j)
        for (int k = 0; k < b2; ++k) {
          const int64_t w = ((t0 + i) * d1 + (t1 + j)) * d2 + (t2 + k);
          ur += mean[(CPLX ? 2 : 1) * w];
          if (CPLX) ui += mean[2 * w + 1];
        }
    ur /= K;
    ui /= K;
    double q = 0.0;
    for (int i = 0; i < b0; ++i)
      for (int j = 0; j < b1; ++j)
        for (int k = 0; k < b2; ++k) {
          const int64_t w = ((t0 + i) * d1 + (t1 + j)) * d2 + (t2 + k);
          const double dr = mean[(CPLX ? 2 : 1) * w] - ur;
          const double di = CPLX ? mean[2 * w + 1] - ui : 0.0;
          q += m2[w] + (double)T * (dr * dr + di * di);
        }
    out[v] = sqrt(q / ((double)K * T));
  }
}

void launch_estimate_noise(const float* in, bool cplx, const int64_t dims[3], const int blk[3], int T, double* mean,
                           double* m2, double* out, cudaStream_t s) {
  const int64_t nvox = dims[0] * dims[1] * dims[2];
  const int64_t b1 = std::min<int64_t>((nvox * 32 + 255) / 256, 148 * 64);
  const int64_t b2 = std::min<int64_t>((nvox + 255) / 256, 148 * 64);
  if (cplx) {
    PD_TIMED("noise_moments", s, k_voxel_moments<true><<<(unsigned)b1, 256, 0, s>>>(in, nvox, T, mean, m2));
    PD_TIMED("noise_block_std", s,
             k_block_std<true><<<(unsigned)b2, 256, 0, s>>>(mean, m2, dims[0], dims[1], dims[2], blk[0], blk[1],
                                                            blk[2], T, out));
  } else {
    PD_TIMED("noise_moments", s, k_voxel_moments<false><<<(unsigned)b1, 256, 0, s>>>(in, nvox, T, mean, m2));
    PD_TIMED("noise_block_std", s,
             k_block_std<false><<<(unsigned)b2, 256, 0, s>>>(mean, m2, dims[0], dims[1], dims[2], blk[0], blk[1],
                                                             blk[2], T, out));
  }
}

}  // namespace pd
