// NORDIC Monte-Carlo level (space_time/lowrank.py:221-232): for each draw, the
// Gram G^T G of a rows x cols standard Gaussian matrix, accumulated over row
// chunks. The largest eigenvalue of each Gram (k_eig in top-1 mode) is the
// squared largest singular value of the draw.
//
// Gaussian entries are generated on the fly (pd_rng.cuh): element (r, c) of
// draw d is a pure function of (seed, d, r, c).
#include <algorithm>

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

namespace pd {

// ---------------------------------------------------------------------------
// Wishart Grams by Bartlett's decomposition (M. S. Bartlett, 1933): for G an
// m x d standard Gaussian matrix (m >= d), G^T G has the law of L L^T with L
// lower triangular, L_ij ~ N(0, 1) for i > j and L_ii^2 ~ chi-square with
// m - i degrees of freedom (i = 0 .. d - 1), all independent. Its largest
// eigenvalue is then distributed as the squared largest singular value of G,
// from d (d + 1) / 2 random numbers instead of m d.
// ---------------------------------------------------------------------------

// Gamma(a, 1) variate (Marsaglia & Tsang, ACM TOMS 2000; a < 1 through
// Gamma(a + 1) U^(1/a)), FP64, from counter-based uniforms and normals of
// (seed, draw, i); bounded to 64 rejection rounds (the acceptance rate exceeds
// 95 % for every a).
__device__ double gamma_mt(double a, uint64_t seed, uint32_t draw, uint32_t i) {
  double boost = 1.0;
  uint32_t ctr = 0;
  auto words = [&](uint32_t c[4]) {
    c[0] = ctr++;
    c[1] = i;
    c[2] = 0x80000000u;  // a counter space of its own (off-diagonal rows use row hi = 0)
    c[3] = draw;
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  };
  if (a < 1.0) {
    uint32_t c[4];
    words(c);
    const double u = ((double)c[0] + 1.0) * 2.3283064365386963e-10;
    boost = pow(u, 1.0 / a);
    a += 1.0;
  }
  const double dd = a - 1.0 / 3.0, cc = 1.0 / sqrt(9.0 * dd);
  for (int it = 0; it < 64; ++it) {
    uint32_t c[4];
    words(c);
    const double u1 = ((double)c[0] + 1.0) * 2.3283064365386963e-10;
    const double u2 = (double)c[1] * 2.3283064365386963e-10;
    const double x = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
    double v = 1.0 + cc * x;
    if (v <= 0.0) continue;
    v = v * v * v;
    const double u = ((double)c[2] + 1.0) * 2.3283064365386963e-10;
    if (u < 1.0 - 0.0331 * x * x * x * x || log(u) < 0.5 * x * x + dd * (1.0 - v + log(v))) return dd * v * boost;
  }
  return dd * boost;  // not reached in practice: the mean
}

// L of every draw (d x d, row-major, lower part): grid-stride over (draw, row,
// group of four columns); the diagonal by gamma_mt.
__global__ void __launch_bounds__(256) k_wishart_l(int64_t m, int d, int draws, uint64_t seed,
                                                   float* __restrict__ Lbuf) {
  const int ng = (d + 3) / 4;
  const int64_t items = (int64_t)draws * d * ng;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < items; t += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t draw = (uint32_t)(t / ((int64_t)d * ng));
    const int rem = (int)(t - (int64_t)draw * d * ng);
    const int i = rem / ng, cg = rem % ng;
    float* L = Lbuf + (int64_t)draw * d * d;
    if (4 * cg < i) {
      float z[4];
      normals4(seed, draw, (uint64_t)i, (uint32_t)cg, z);
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (4 * cg + q < i) L[(int64_t)i * d + 4 * cg + q] = z[q];
    }
    if (cg == i / 4)  // the thread of the diagonal's column group
      L[(int64_t)i * d + i] = (float)sqrt(2.0 * gamma_mt(0.5 * (double)(m - i), seed, draw, (uint32_t)i));
  }
}

// W = L L^T, packed lower: grid (lower 32 x 32 tile pairs, draws); W_ij =
// sum_{k <= j} L_ik L_jk through 32-wide K slabs in shared memory.
constexpr int WT = 32;
__global__ void __launch_bounds__(256) k_wishart_w(int d, const float* __restrict__ Lbuf, float* __restrict__ gram,
                                                   int64_t gram_stride) {
  __shared__ float As[WT][WT + 1], Bs[WT][WT + 1];
  int bi, bj;
  mc_tile_pair(blockIdx.x, bi, bj);
  const int draw = blockIdx.y;
  const float* L = Lbuf + (int64_t)draw * d * d;
  const int tid = threadIdx.x, ty = tid / 16, tx = tid % 16;  // 2 x 2 outputs per thread
  float acc[2][2] = {};
  const int kend = min((bj + 1) * WT, d);  // L_jk = 0 for k > j
  for (int k0 = 0; k0 < kend; k0 += WT) {
    for (int e = tid; e < WT * WT; e += 256) {
      const int r = e / WT, c = e % WT;
      const int ia = bi * WT + r, ib = bj * WT + r, k = k0 + c;
      As[r][c] = (ia < d && k <= ia) ? L[(int64_t)ia * d + k] : 0.f;
      Bs[r][c] = (ib < d && k <= ib) ? L[(int64_t)ib * d + k] : 0.f;
    }
    __syncthreads();
#pragma unroll 8
    for (int c = 0; c < WT; ++c) {
#pragma unroll
      for (int x = 0; x < 2; ++x)
#pragma unroll
        for (int y = 0; y < 2; ++y) acc[x][y] = fmaf(As[ty * 2 + x][c], Bs[tx * 2 + y][c], acc[x][y]);
    }
    __syncthreads();
  }
  float* W = gram + (int64_t)draw * gram_stride;
#pragma unroll
  for (int x = 0; x < 2; ++x)
#pragma unroll
    for (int y = 0; y < 2; ++y) {
      const int i = bi * WT + ty * 2 + x, j = bj * WT + tx * 2 + y;
      if (i < d && j <= i) W[pk(i, j, d)] = acc[x][y];
    }
}

void launch_wishart(int64_t m, int d, int n_iter, uint64_t seed, float* Lbuf, float* gram, int64_t gram_stride,
                    cudaStream_t s) {
  const int64_t items = (int64_t)n_iter * d * ((d + 3) / 4);
  const int blocks = (int)std::min<int64_t>((items + 255) / 256, 148 * 8);
  PD_TIMED("mc_wishart", s, k_wishart_l<<<blocks, 256, 0, s>>>(m, d, n_iter, seed, Lbuf));
  const int nt = (d + WT - 1) / WT;
  dim3 grid(nt * (nt + 1) / 2, n_iter);
  PD_TIMED("mc_wishart", s, k_wishart_w<<<grid, 256, 0, s>>>(d, Lbuf, gram, gram_stride));
}

}  // namespace pd
