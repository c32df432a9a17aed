// NORDIC Monte-Carlo level (space_time/lowrank.py:221-232): for each draw, the
// Gram G^T G of a rows x cols standard Gaussian matrix, accumulated over row
// chunks. The largest eigenvalue of each Gram (k_eig in top-1 mode) is the
// squared largest singular value of the draw.
//
// Gaussian entries are generated on the fly (pd_rng.cuh): element (r, c) of
// draw d is a pure function of (seed, d, r, c).
#include "pd_common.cuh"
#include "pd_kernels.cuh"
#include "pd_profile.cuh"
#include "pd_rng.cuh"

namespace pd {

constexpr int MC_T = 64;
constexpr int MC_K = 16;
constexpr int MC_THREADS = 256;
constexpr int64_t MC_ROWS_PER_CTA = 4096;

__device__ __forceinline__ void mc_tile_pair(int t, int& bi, int& bj) {
  int i = (int)((sqrtf(8.f * t + 1.f) - 1.f) * 0.5f);
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  while (i * (i + 1) / 2 > t) --i;
  bi = i;
  bj = t - i * (i + 1) / 2;
}

// grid: (row chunks, tile pairs, draws). Each CTA writes its chunk's partial
// packed Gram; k_mc_reduce sums the chunks in a fixed order (deterministic).
__global__ void __launch_bounds__(MC_THREADS) k_mc_gram(int64_t rows, int cols, uint64_t seed, float* part,
                                                        int64_t part_stride) {
  __shared__ float As[MC_K][MC_T];
  __shared__ float Bs[MC_K][MC_T];
  const int draw = blockIdx.z;
  int bi, bj;
  mc_tile_pair(blockIdx.y, bi, bj);
  const int64_t rbeg = (int64_t)blockIdx.x * MC_ROWS_PER_CTA;
  int64_t rend = rbeg + MC_ROWS_PER_CTA;
  if (rend > rows) rend = rows;
  const int tid = threadIdx.x, ty = tid / 16, tx = tid % 16;
  const int lr = tid / 16, lg = tid % 16;  // load row (0..15), 4-column group (0..15)
  float acc[4][4] = {};
  const bool diag = bi == bj;
  for (int64_t r0 = rbeg; r0 < rend; r0 += MC_K) {
    const int64_t r = r0 + lr;
    float za[4] = {0.f, 0.f, 0.f, 0.f}, zb[4] = {0.f, 0.f, 0.f, 0.f};
    if (r < rend) {
      const int ca = bi * MC_T + lg * 4;
      if (ca < cols) normals4(seed, (uint32_t)draw, (uint64_t)r, (uint32_t)(ca >> 2), za);
      if (!diag) {
        const int cb = bj * MC_T + lg * 4;
        if (cb < cols) normals4(seed, (uint32_t)draw, (uint64_t)r, (uint32_t)(cb >> 2), zb);
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int ca = bi * MC_T + lg * 4 + q, cb = bj * MC_T + lg * 4 + q;
      As[lr][lg * 4 + q] = ca < cols ? za[q] : 0.f;
      if (!diag) Bs[lr][lg * 4 + q] = cb < cols ? zb[q] : 0.f;
    }
    __syncthreads();
    const float(*Bp)[MC_T] = diag ? As : Bs;
#pragma unroll
    for (int kk = 0; kk < MC_K; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a[q] = As[kk][ty * 4 + q];
        b[q] = Bp[kk][tx * 4 + q];
      }
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) acc[x][y] = fmaf(a[x], b[y], acc[x][y]);
    }
    __syncthreads();
  }
  float* C = part + ((int64_t)draw * gridDim.x + blockIdx.x) * part_stride;
#pragma unroll
  for (int x = 0; x < 4; ++x) {
    const int i = bi * MC_T + ty * 4 + x;
#pragma unroll
    for (int y = 0; y < 4; ++y) {
      const int j = bj * MC_T + tx * 4 + y;
      if (i < cols && j <= i) C[pk(i, j, cols)] = acc[x][y];
    }
  }
}

// gram[d][e] = sum over chunks c (in order) of part[d][c][e], accumulated in FP64.
__global__ void k_mc_reduce(const float* __restrict__ part, int64_t part_stride, int chunks, int64_t np,
                            float* __restrict__ gram, int64_t gram_stride) {
  const int d = blockIdx.y;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < np; e += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int c = 0; c < chunks; ++c) s += part[((int64_t)d * chunks + c) * part_stride + e];
    gram[(int64_t)d * gram_stride + e] = (float)s;
  }
}

int64_t mc_chunks(int64_t rows) { return (rows + MC_ROWS_PER_CTA - 1) / MC_ROWS_PER_CTA; }

void launch_chunk_reduce(const float* part, int64_t part_stride, int chunks, int64_t np, int draws, float* gram,
                         int64_t gram_stride, cudaStream_t s) {
  dim3 rgrid((unsigned)((np + 255) / 256), draws);
  PD_TIMED("mc_reduce", s, k_mc_reduce<<<rgrid, 256, 0, s>>>(part, part_stride, chunks, np, gram, gram_stride));
}

// level = mean_i sqrt(max(lam_i, 0)) in draw order (the host formula of
// pd_nordic_mc_threshold, so both give the same double); out = {level, noise_std * level}.
__global__ void k_mc_level(const double* __restrict__ lam, int n_iter, double noise_std, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double acc = 0.0;
    for (int i = 0; i < n_iter; ++i) acc += sqrt(fmax(lam[i], 0.0));
    const double level = acc / n_iter;
    out[0] = level;
    out[1] = noise_std * level;
  }
}

void launch_mc_level(const double* lam, int n_iter, double noise_std, double* out, cudaStream_t s) {
  PD_TIMED("mc_level", s, k_mc_level<<<1, 32, 0, s>>>(lam, n_iter, noise_std, out));
}

void launch_mc_gram(int64_t rows, int cols, int n_iter, uint64_t seed, float* part, float* gram,
                    int64_t gram_stride, cudaStream_t s) {
  const int nt = (cols + MC_T - 1) / MC_T;
  const int64_t chunks = mc_chunks(rows);
  const int64_t np = pk_size(cols);
  dim3 grid((unsigned)chunks, nt * (nt + 1) / 2, n_iter);
  PD_TIMED("mc_gram", s, k_mc_gram<<<grid, MC_THREADS, 0, s>>>(rows, cols, seed, part, np));
  dim3 rgrid((unsigned)((np + 255) / 256), n_iter);
  PD_TIMED("mc_reduce", s, k_mc_reduce<<<rgrid, 256, 0, s>>>(part, np, (int)chunks, np, gram, gram_stride));
}

}  // namespace pd
