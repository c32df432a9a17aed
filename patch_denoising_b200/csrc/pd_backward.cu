// Backward pass of the low-rank patch denoiser (real volumes): the adjoint of
// extract -> centre -> spectral shrinkage -> recombine -> normalise, for
//   soft:  s~_i = max(s_i - tau_p, 0), tau_p = stdest_p * level (singular-value
//          soft thresholding: the adaptive trace-norm shrinkage with gamma = 1,
//          space_time/lowrank.py:459-461);
//   hard:  s~_i = s_i for the top rank_p components, 0 after (the MP-PCA /
//          hybrid / raw rules at a fixed decision).
// The forward keeps only the input, the patch list and the per-patch ranks;
// every factorisation is recomputed here (mean, Gram, full eigendecomposition).
//
// Per patch, with Xc = X - 1 mu^T (M x T, M > T), Xc = U S V^T, the output
// block Y = U h(S) V^T + 1 mu^T and its upstream gradient Gb (M x T), the
// spectral-function adjoint (Lewis; Candes, Sing-Long & Trzasko 2013) in the
// Gram basis reads, with A = U^T Gb V = S^-1 V^T (Xc^T Gb) V:
//   D_ii = h'(s_i) A_ii,
//   D_ij = [A_ij (h_i s_i - h_j s_j) + A_ji (h_i s_j - h_j s_i)] / (s_i^2 - s_j^2),
//   E    = S^-1 (D - A diag(h/s)),
//   dL/dXc = Xc K1 + Gb K2,  K1 = V E V^T,  K2 = V diag(h/s) V^T,
//   dL/dX  = dL/dXc + 1 u^T,  u = mean_r(Gb) (I - K2),
//   dL/dtau_p = -sum_{s_i > tau_p} A_ii (soft; 0 for hard).
// Where s_i^2 - s_j^2 falls below DEGEN_REL of s_i^2 + s_j^2 the pair takes
// the limit: h'((s_i + s_j) / 2) sym(A)_ij + (h_i + h_j) / (s_i + s_j) skew(A)_ij.
//
// Recombination: out = (sum_p theta_p scatter(Y_p)) / W, W = sum theta (theta
// constant in the input almost everywhere), so Gb_p = theta_p gather(G / W):
// the adjoint of recombination is a gather, and that of extraction a scatter-add.
#include <float.h>

#include "pd_common.cuh"
#include "pd_kernels.cuh"
#include "pd_profile.cuh"

namespace pd {

constexpr int BW_THREADS = 256;
constexpr int BT = 64;  // cross-Gram tile edge
constexpr int BK = 16;  // rows per k step
constexpr double DEGEN_REL = 1e-6;

__host__ __device__ inline int bw_ld(int n) { return n | 1; }  // odd: conflict-free strided reads

// Gb[r][t] = theta * gout / weights at row r, frame t of the patch (0 where the
// weight is zero or not finite).
__device__ __forceinline__ float gbar(const float* gout, const float* wts, int64_t at, float theta) {
  const float wv = wts[at];
  return (wv > 0.f && isfinite(wv)) ? theta * gout[at] / wv : 0.f;
}

__device__ __forceinline__ float patch_theta(int recomb, int rank) {
  return recomb == PD_RECOMB_WEIGHTED ? (float)(1.0 / (2.0 + (double)rank)) : 1.f;
}

// cross[p] = Xc^T Gb (n x n, row-major, ld n): grid (patch, tile row, tile col).
__global__ void __launch_bounds__(BW_THREADS) k_bwd_cross(Geo g, const float* __restrict__ in,
                                                          const float* __restrict__ gout, const float* __restrict__ wts,
                                                          PatchWork w, BwdWork b) {
  __shared__ float As[BK][BT];
  __shared__ float Bs[BK][BT];
  __shared__ float mA[BT];
  __shared__ int64_t rb[BK];
  const int p = blockIdx.x, bi = blockIdx.y, bj = blockIdx.z;
  const int n = g.cols, M = g.rows, tid = threadIdx.x;
  int64_t o[4];
  patch_origin(g, w.list[p], o);
  const float theta = patch_theta(b.recombination, b.rank[p]);
  const float* mean = w.mean + (int64_t)p * n;
  if (tid < BT) mA[tid] = bi * BT + tid < n ? mean[bi * BT + tid] : 0.f;
  const int ty = tid / 16, tx = tid % 16, lc = tid % BT, lr = tid / BT;
  const int ca = bi * BT + lc, cb = bj * BT + lc;
  float acc[4][4] = {};
  for (int r0 = 0; r0 < M; r0 += BK) {
    __syncthreads();
    if (tid < BK) rb[tid] = (r0 + tid < M) ? row_voxel(g, o, r0 + tid) * g.shape[3] + o[3] : -1;
    __syncthreads();
#pragma unroll
    for (int q = 0; q < BK / 4; ++q) {
      const int kk = lr + 4 * q;
      const int64_t base = rb[kk];
      float va = 0.f, vb = 0.f;
      if (base >= 0) {
        if (ca < n) va = in[base + ca] - mA[lc];
        if (cb < n) vb = gbar(gout, wts, base + cb, theta);
      }
      As[kk][lc] = va;
      Bs[kk][lc] = vb;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      float a[4], c[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a[q] = As[kk][ty * 4 + q];
        c[q] = Bs[kk][tx * 4 + q];
      }
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) acc[x][y] += a[x] * c[y];
    }
  }
  float* C = b.cross + (int64_t)p * b.mat_stride;
#pragma unroll
  for (int x = 0; x < 4; ++x) {
    const int i = bi * BT + ty * 4 + x;
#pragma unroll
    for (int y = 0; y < 4; ++y) {
      const int j = bj * BT + tx * 4 + y;
      if (i < n && j < n) C[i * n + j] = acc[x][y];
    }
  }
}

// gmean[p][t] = mean over the patch's rows of Gb[r][t] (FP64 sums).
__global__ void __launch_bounds__(BW_THREADS) k_bwd_gmean(Geo g, const float* __restrict__ gout,
                                                          const float* __restrict__ wts, PatchWork w, BwdWork b) {
  extern __shared__ int64_t rowbase[];
  const int p = blockIdx.x;
  int64_t o[4];
  patch_origin(g, w.list[p], o);
  const int M = g.rows, n = g.cols;
  const float theta = patch_theta(b.recombination, b.rank[p]);
  for (int r = threadIdx.x; r < M; r += blockDim.x) rowbase[r] = row_voxel(g, o, r) * g.shape[3] + o[3];
  __syncthreads();
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    double s = 0.0;
    for (int r = 0; r < M; ++r) s += gbar(gout, wts, rowbase[r] + t, theta);
    b.gmean[(int64_t)p * n + t] = (float)(s / M);
  }
}

// C = op(A) op(B), n x n in shared memory with leading dimension ld (odd);
// op(X)[i][k] = TA/TB ? X[k][i] : X[i][k]. 256 threads, n <= 128: thread
// (ty, tx) computes rows ty + 16 a, columns tx + 16 c (a, c < 8).
template <bool TA, bool TB>
__device__ void bw_mm(const float* A, const float* B, float* C, int n, int ld) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float acc[8][8];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[a][c] = 0.f;
  for (int k = 0; k < n; ++k) {
    float av[8], bv[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int i = min(ty + 16 * q, n - 1), j = min(tx + 16 * q, n - 1);
      av[q] = TA ? A[k * ld + i] : A[i * ld + k];
      bv[q] = TB ? B[j * ld + k] : B[k * ld + j];
    }
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[a][c] += av[a] * bv[c];
  }
  __syncthreads();  // C may alias an operand read above by other threads
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int i = ty + 16 * a;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int j = tx + 16 * c;
      if (i < n && j < n) C[i * ld + j] = acc[a][c];
    }
  }
  __syncthreads();
}

// Per patch: A, D, E, K1, K2, u and dL/dlevel (one CTA per patch, n <= 128).
__global__ void __launch_bounds__(BW_THREADS, 1) k_bwd_small(int n, int M, PatchWork w, BwdWork b) {
  extern __shared__ __align__(16) float smf[];
  const int ld = bw_ld(n);
  float* V = smf;              // V[t][a], column a = eigenvector a (descending)
  float* X = V + n * ld;       // work matrix
  float* Y = X + n * ld;       // work matrix
  float* sg = Y + n * ld;      // singular values
  float* h = sg + n;           // h(s)
  float* hp = h + n;           // h'(s)
  float* c = hp + n;           // h(s) / s
  float* gm = c + n;           // mean row of Gb
  __shared__ double s_red[BW_THREADS / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int p = blockIdx.x;
  const float* vb = w.vec + (int64_t)p * w.vec_stride;
  for (int t = tid; t < n * n; t += BW_THREADS) {
    const int a = t / n, r = t % n;
    V[r * ld + a] = vb[(int64_t)a * 2 * n + r];
  }
  const double tau = b.shrink == 0 ? sqrt(fmax(w.prior[p], 0.0)) * b.level : 0.0;
  const int rank = b.rank[p];
  for (int a = tid; a < n; a += BW_THREADS) {
    const float s = sqrtf(fmaxf(w.coef[(int64_t)p * n + a], 0.f));
    sg[a] = s;
    float hv, hd;
    if (b.shrink == 0) {
      hv = fmaxf(s - (float)tau, 0.f);
      hd = s > (float)tau ? 1.f : 0.f;
    } else {
      hv = a < rank ? s : 0.f;
      hd = a < rank ? 1.f : 0.f;
    }
    h[a] = hv;
    hp[a] = hd;
    c[a] = s > 0.f ? hv / s : 0.f;
    gm[a] = b.gmean[(int64_t)p * n + a];
  }
  const float* cr = b.cross + (int64_t)p * b.mat_stride;
  for (int t = tid; t < n * n; t += BW_THREADS) X[(t / n) * ld + (t % n)] = cr[t];
  __syncthreads();
  bw_mm<false, false>(X, V, Y, n, ld);  // Y = (Xc^T Gb) V
  bw_mm<true, false>(V, Y, X, n, ld);   // X = V^T Y, then A = S^-1 X
  for (int t = tid; t < n * n; t += BW_THREADS) {
    const int i = t / n;
    X[i * ld + (t % n)] = sg[i] > 0.f ? X[i * ld + (t % n)] / sg[i] : 0.f;
  }
  __syncthreads();
  // E (into Y) and the threshold gradient
  double dt = 0.0;
  for (int t = tid; t < n * n; t += BW_THREADS) {
    const int i = t / n, j = t % n;
    const float aij = X[i * ld + j];
    float d;
    if (i == j) {
      d = hp[i] * aij;
      if (hp[i] > 0.f) dt -= aij;
    } else {
      const float aji = X[j * ld + i];
      const double si = sg[i], sj = sg[j];
      const double den = si * si - sj * sj;
      if (fabs(den) > DEGEN_REL * (si * si + sj * sj)) {
        d = (float)(((double)aij * (h[i] * si - h[j] * sj) + (double)aji * (h[i] * sj - h[j] * si)) / den);
      } else {
        const double hmid = b.shrink == 0 ? ((0.5 * (si + sj) > tau) ? 1.0 : 0.0) : 0.5 * (hp[i] + hp[j]);
        const double sum = si + sj;
        d = (float)(hmid * 0.5 * (aij + aji) + (sum > 0.0 ? (h[i] + h[j]) / sum : 0.0) * 0.5 * (aij - aji));
      }
    }
    Y[i * ld + j] = sg[i] > 0.f ? (d - aij * c[j]) / sg[i] : 0.f;
  }
  dt = warp_sum(dt);
  if (lane == 0) s_red[warp] = dt;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int k = 0; k < BW_THREADS / 32; ++k) s += s_red[k];
    // dL/dlevel of this patch: tau_p = stdest_p * level
    b.dlevel[p] = b.shrink == 0 ? s * sqrt(fmax(w.prior[p], 0.0)) : 0.0;
  }
  bw_mm<false, false>(V, Y, X, n, ld);  // X = V E
  bw_mm<false, true>(X, V, Y, n, ld);   // Y = V E V^T = K1
  float* k1 = b.k1 + (int64_t)p * b.mat_stride;
  float* k2 = b.k2 + (int64_t)p * b.mat_stride;
  for (int t = tid; t < n * n; t += BW_THREADS) k1[t] = Y[(t / n) * ld + (t % n)];
  // K2 = V diag(c) V^T: X = V diag(c), then X V^T
  for (int t = tid; t < n * n; t += BW_THREADS) {
    const int r = t / n, a = t % n;
    X[r * ld + a] = V[r * ld + a] * c[a];
  }
  __syncthreads();
  bw_mm<false, true>(X, V, Y, n, ld);
  for (int t = tid; t < n * n; t += BW_THREADS) k2[t] = Y[(t / n) * ld + (t % n)];
  // u = gm (I - K2)
  for (int j = tid; j < n; j += BW_THREADS) {
    float s = gm[j];
    for (int k = 0; k < n; ++k) s -= gm[k] * Y[k * ld + j];
    b.u[(int64_t)p * n + j] = s;
  }
}

// dL/dx += scatter(Xc K1 + Gb K2 + 1 u^T): grid (patch, row block), K1 and K2
// in shared memory. A warp takes AP_ROWS rows at a time, staged k-major (row
// index fastest, so one 16-byte load gives four rows of a frame k); a lane
// holds AP_ROWS x JT outputs (frames lane, lane + 32, ...).
constexpr int AP_ROWS = 8;
constexpr int AP_JT = 4;  // frames per lane: n <= 128
__global__ void __launch_bounds__(BW_THREADS) k_bwd_apply(Geo g, const float* __restrict__ in,
                                                          const float* __restrict__ gout, const float* __restrict__ wts,
                                                          float* __restrict__ gin, PatchWork w, BwdWork b, int ysplit) {
  extern __shared__ __align__(16) float smf[];
  const int n = g.cols, M = g.rows;
  float* K1 = smf;                        // n x n
  float* K2 = K1 + n * n;                 // n x n
  float* xs = K1 + ((2 * n * n + 3) & ~3);  // [warps][n][AP_ROWS] centred rows, k-major (16-byte aligned)
  float* gs = xs + (BW_THREADS / 32) * AP_ROWS * n;  // [warps][n][AP_ROWS] Gb rows, k-major
  float* mu = gs + (BW_THREADS / 32) * AP_ROWS * n;  // [n]
  float* uu = mu + n;                                // [n]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int p = (int)(blockIdx.x / (unsigned)ysplit);
  const int yb = (int)(blockIdx.x - (unsigned)p * (unsigned)ysplit);
  int64_t o[4];
  patch_origin(g, w.list[p], o);
  const float theta = patch_theta(b.recombination, b.rank[p]);
  const float* k1 = b.k1 + (int64_t)p * b.mat_stride;
  const float* k2 = b.k2 + (int64_t)p * b.mat_stride;
  for (int t = tid; t < n * n; t += BW_THREADS) {
    K1[t] = k1[t];
    K2[t] = k2[t];
  }
  for (int t = tid; t < n; t += BW_THREADS) {
    mu[t] = w.mean[(int64_t)p * n + t];
    uu[t] = b.u[(int64_t)p * n + t];
  }
  __syncthreads();
  float* xw = xs + warp * AP_ROWS * n;
  float* gw = gs + warp * AP_ROWS * n;
  const int rstep = ysplit * (BW_THREADS / 32) * AP_ROWS;
  for (int r0 = (yb * (BW_THREADS / 32) + warp) * AP_ROWS; r0 < M; r0 += rstep) {
    int64_t base[AP_ROWS];
#pragma unroll
    for (int q = 0; q < AP_ROWS; ++q) {
      const int r = r0 + q;
      base[q] = r < M ? row_voxel(g, o, r) * g.shape[3] + o[3] : -1;
      for (int t = lane; t < n; t += 32) {
        xw[t * AP_ROWS + q] = base[q] >= 0 ? in[base[q] + t] - mu[t] : 0.f;
        gw[t * AP_ROWS + q] = base[q] >= 0 ? gbar(gout, wts, base[q] + t, theta) : 0.f;
      }
    }
    __syncwarp();
    float acc[AP_ROWS][AP_JT];
#pragma unroll
    for (int q = 0; q < AP_ROWS; ++q)
#pragma unroll
      for (int c = 0; c < AP_JT; ++c) acc[q][c] = 0.f;
    for (int k = 0; k < n; ++k) {
      float a1[AP_JT], a2[AP_JT];
#pragma unroll
      for (int c = 0; c < AP_JT; ++c) {
        const int j = lane + 32 * c;
        a1[c] = j < n ? K1[k * n + j] : 0.f;
        a2[c] = j < n ? K2[k * n + j] : 0.f;
      }
      const float4* xk = reinterpret_cast<const float4*>(xw + k * AP_ROWS);
      const float4* gk = reinterpret_cast<const float4*>(gw + k * AP_ROWS);
#pragma unroll
      for (int h = 0; h < AP_ROWS / 4; ++h) {
        const float4 xv = xk[h], gv = gk[h];
        const float xr[4] = {xv.x, xv.y, xv.z, xv.w}, gr[4] = {gv.x, gv.y, gv.z, gv.w};
#pragma unroll
        for (int e = 0; e < 4; ++e)
#pragma unroll
          for (int c = 0; c < AP_JT; ++c) acc[4 * h + e][c] += xr[e] * a1[c] + gr[e] * a2[c];
      }
    }
#pragma unroll
    for (int q = 0; q < AP_ROWS; ++q) {
      if (base[q] < 0) continue;
#pragma unroll
      for (int c = 0; c < AP_JT; ++c) {
        const int j = lane + 32 * c;
        if (j < n) atomicAdd(gin + base[q] + j, acc[q][c] + uu[j]);
      }
    }
    __syncwarp();
  }
}

size_t bwd_small_smem(int n) { return sizeof(float) * ((size_t)3 * n * bw_ld(n) + 5 * (size_t)n); }
size_t bwd_apply_smem(int n) {
  return sizeof(float) * ((((size_t)2 * n * n + 3) & ~(size_t)3) + 2 * (size_t)(BW_THREADS / 32) * AP_ROWS * n +
                          2 * (size_t)n);
}
bool bwd_supported(int n) { return n <= 128 && bwd_apply_smem(n) <= 227 * 1024 && bwd_small_smem(n) <= 227 * 1024; }

cudaError_t launch_backward(const Geo& g, const float* in, const float* gout, const float* wts, float* gin,
                            const PatchWork& w, const BwdWork& b, cudaStream_t s) {
  const int n = g.cols;
  const int nt = (n + BT - 1) / BT;
  dim3 grid(w.count, nt, nt);
  PD_TIMED("bwd_cross", s, k_bwd_cross<<<grid, BW_THREADS, 0, s>>>(g, in, gout, wts, w, b));
  const size_t gsm = sizeof(int64_t) * (size_t)g.rows;
  if (gsm > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_bwd_gmean, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gsm);
    if (e != cudaSuccess) return e;
  }
  PD_TIMED("bwd_gmean", s, k_bwd_gmean<<<w.count, BW_THREADS, gsm, s>>>(g, gout, wts, w, b));
  const size_t ssm = bwd_small_smem(n);
  cudaError_t e = cudaFuncSetAttribute(k_bwd_small, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssm);
  if (e != cudaSuccess) return e;
  PD_TIMED("bwd_small", s, k_bwd_small<<<w.count, BW_THREADS, ssm, s>>>(n, g.rows, w, b));
  const size_t asm_ = bwd_apply_smem(n);
  e = cudaFuncSetAttribute(k_bwd_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)asm_);
  if (e != cudaSuccess) return e;
  const int per = (BW_THREADS / 32) * AP_ROWS;
  const int ysplit = (g.rows + 4 * per - 1) / (4 * per);  // about four row groups per warp
  PD_TIMED("bwd_apply", s,
           k_bwd_apply<<<(unsigned)(w.count * ysplit), BW_THREADS, asm_, s>>>(g, in, gout, wts, gin, w, b, ysplit));
  return cudaGetLastError();
}

}  // namespace pd
