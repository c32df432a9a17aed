// Subspace eigensolver for the hard-threshold rule on the mixed-precision path
// (RawSVDDenoiser / NordicDenoiser, space_time/lowrank.py:170-184): one CTA per
// patch finds the eigenpairs of the scaled Gram C that lie above the known
// threshold, without reducing the whole matrix to tridiagonal form.
//
//  1. Block power iteration on P columns: Y = C Q, then Q = orth(Y) by
//     Cholesky QR (the P x P Gram Y^H Y, its Cholesky factor R and R^-1 in
//     FP64, Q = Y R^-1 in FP32), a second pass
//     before each Rayleigh-Ritz check (CholQR2). Columns converge to the
//     eigenvectors above the bulk at the rate lambda_{P+1} / lambda_i per step.
//  2. Rayleigh-Ritz: Z = C Q, H = Q^H Z (P x P Hermitian), cyclic Jacobi
//     eigensolver of H in FP32 (round-robin ordering, one warp), Ritz vectors
//     V = Q W, C V = Z W and their residuals ||C v_i - theta_i v_i||.
//  3. The reference rule rank = #{ sqrt(theta_i) > threshold } on the Ritz
//     values (FP64), accepted only when it is certified: fewer than P Ritz
//     values above the threshold, the smallest Ritz value below a quarter of
//     it (the block reaches into the bulk, so no eigenvalue above the threshold
//     is missing), the kept pairs' residuals below SUB_TOLR of their values, and
//     the first excluded Ritz value plus its residual below the threshold. A
//     certified patch gets its Ritz vectors as the active components; any
//     other patch is left to k_eig (n_active = -1), which then runs the full
//     Householder solver on it.
//
// C stays in shared memory (packed lower, FP32) for every product; the solver
// applies where that and the P-column blocks fit (sub_supported). A first pass
// runs with P = 8 columns, which certifies patches that keep up to 7
// components; the patches it leaves get a pass with P = 16 (up to 15), and any
// still left get k_eig.
#include <float.h>

#include "pd_common.cuh"
#include "pd_kernels.cuh"
#include "pd_profile.cuh"

namespace pd {

constexpr int SUB_THREADS = 512;
constexpr int SUB_NW = SUB_THREADS / 32;
constexpr int SUB_FIRST = 3;     // power steps before the first Rayleigh-Ritz check
constexpr int SUB_MORE = 2;      // power steps between later checks
constexpr int SUB_CHECKS = 4;    // checks before the patch goes to k_eig
constexpr int SUB_SWEEPS = 8;    // Jacobi sweeps at most
constexpr float SUB_TOLR = 2e-5f;
constexpr size_t SUB_SMEM_LIMIT = 227 * 1024 - 1024;

struct SubLayout {
  size_t a, q, y, g, part, r, h, w, th, perm, res, total;
  int slices;  // row slices of the P x P Gram products (partials in `part`)
};

__host__ __device__ inline size_t sub_al(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline SubLayout sub_layout_s(bool cplx, int n, int P, int slices) {
  const size_t es = cplx ? 8 : 4;
  const size_t PP = (size_t)P * P;
  SubLayout L;
  size_t o = 0;
  L.slices = slices;
  L.a = o;
  o += sub_al((size_t)pk_size(n) * es);
  L.q = o;
  o += sub_al((size_t)n * P * es);
  L.y = o;
  o += sub_al((size_t)n * P * es);
  L.g = o;
  o += sub_al(PP * 16);  // FP64 complex Gram (real: imaginary parts stay 0)
  L.part = o;
  o += slices > 1 ? sub_al(PP * 16 * slices) : 0;
  L.r = o;
  o += sub_al(PP * es);  // R^-1 of the Cholesky factor, FP32
  L.h = o;
  o += sub_al(PP * es);
  L.w = o;
  o += sub_al(PP * es);
  L.th = o;
  o += sub_al((size_t)P * 4);
  L.perm = o;
  o += sub_al((size_t)P * 4);
  L.res = o;
  o += sub_al((size_t)P * 4);
  L.total = o;
  return L;
}

__host__ __device__ inline SubLayout sub_layout(bool cplx, int n, int P) {
  const SubLayout two = sub_layout_s(cplx, n, P, 2);
  return two.total <= SUB_SMEM_LIMIT ? two : sub_layout_s(cplx, n, P, 1);
}

static bool sub_fits(bool cplx, int n, int rows, int P) {
  return n >= 3 * P && rows > 2 * P && sub_layout(cplx, n, P).total <= SUB_SMEM_LIMIT;
}

bool sub_supported(bool cplx, int n, int rows) { return sub_fits(cplx, n, rows, 8); }

// ---------------------------------------------------------------------------
// Small helpers (T = float or cf)
// ---------------------------------------------------------------------------
// conj(a) * b in FP64
__device__ __forceinline__ double2 d2conjmul(float a, float b) { return make_double2((double)a * b, 0.0); }
__device__ __forceinline__ double2 d2conjmul(cf a, cf b) {
  const double ax = a.x, ay = a.y, bx = b.x, by = b.y;
  return make_double2(ax * bx + ay * by, ax * by - ay * bx);
}
template <class T>
__device__ __forceinline__ T from_d2(double2 v);
template <>
__device__ __forceinline__ float from_d2<float>(double2 v) { return (float)v.x; }
template <>
__device__ __forceinline__ cf from_d2<cf>(double2 v) { return cf{(float)v.x, (float)v.y}; }

// acc[0..NH) += c * Q[k][NH h .. NH h + NH)
template <bool CPLX, int NH>
__device__ __forceinline__ void sub_fma(typename Elem<CPLX>::T* acc, typename Elem<CPLX>::T c, const float4* q4) {
  if constexpr (CPLX) {
#pragma unroll
    for (int j = 0; j < NH / 2; ++j) {
      const float4 v = q4[j];
      acc[2 * j] = acc[2 * j] + c * cf{v.x, v.y};
      acc[2 * j + 1] = acc[2 * j + 1] + c * cf{v.z, v.w};
    }
  } else {
#pragma unroll
    for (int j = 0; j < NH / 4; ++j) {
      const float4 v = q4[j];
      acc[4 * j] += c * v.x;
      acc[4 * j + 1] += c * v.y;
      acc[4 * j + 2] += c * v.z;
      acc[4 * j + 3] += c * v.w;
    }
  }
}

// Y = C Q over the packed lower C (n x n Hermitian), Q and Y row-major n x P.
// A warp owns 16 rows r0..r0+15; lane (r, h) accumulates row r0 + r against
// columns (P/2) h .. (P/2) h + P/2 - 1. C(row, k) is the stored column-k entry for row >= k (every
// k < r0), else the conjugate of the entry stored in column row at row k
// (every k >= r0 + 16); only the 16 k of the diagonal block take both forms.
template <bool CPLX, int P>
__device__ void sub_product(const typename Elem<CPLX>::T* __restrict__ A, int n,
                            const typename Elem<CPLX>::T* __restrict__ Q, typename Elem<CPLX>::T* __restrict__ Y) {
  using T = typename Elem<CPLX>::T;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r = lane & 15, h = lane >> 4;
  for (int rb = warp; rb * 16 < n; rb += SUB_NW) {
    const int r0 = rb * 16, row = r0 + r;
    const bool live = row < n;
    const int rowc = live ? row : n - 1;  // clamped: loads stay in bounds, results are dropped
    const int cbr = (int)pk(rowc, rowc, n) - rowc;
    constexpr int NH = P / 2;
    T acc[NH];
#pragma unroll
    for (int j = 0; j < NH; ++j) acc[j] = zero<T>();
    const float4* qb = reinterpret_cast<const float4*>(Q) + h * (NH * sizeof(T) / 16);
    constexpr int QS = P * sizeof(T) / 16;  // float4 per row of Q
    int cbk = 0;                                // pk(k, k, n) - k
    int k = 0;
    for (; k + 4 <= r0; k += 4) {
      T c[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        c[u] = A[cbk + rowc];
        cbk += n - (k + u) - 1;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) sub_fma<CPLX, NH>(acc, c[u], qb + (k + u) * QS);
    }
    for (; k < r0; ++k) {
      sub_fma<CPLX, NH>(acc, A[cbk + rowc], qb + k * QS);
      cbk += n - k - 1;
    }
    const int ke = min(r0 + 16, n);
    for (; k < ke; ++k) {
      const T c = rowc >= k ? A[cbk + rowc] : cj(A[cbr + k]);
      sub_fma<CPLX, NH>(acc, c, qb + k * QS);
      cbk += n - k - 1;
    }
    for (; k + 4 <= n; k += 4) {
      T c[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) c[u] = cj(A[cbr + k + u]);
#pragma unroll
      for (int u = 0; u < 4; ++u) sub_fma<CPLX, NH>(acc, c[u], qb + (k + u) * QS);
    }
    for (; k < n; ++k) sub_fma<CPLX, NH>(acc, cj(A[cbr + k]), qb + k * QS);
    if (live) {
#pragma unroll
      for (int j = 0; j < NH; ++j) Y[row * P + h * NH + j] = acc[j];
    }
  }
}

// G_ab = sum_r conj(X_ra) Y_rb (FP64) for a <= b, over L.slices row slices
// (partials in `part`, then summed). Ends with a block barrier.
template <bool CPLX, int P>
__device__ void sub_gram(int n, const typename Elem<CPLX>::T* __restrict__ X,
                         const typename Elem<CPLX>::T* __restrict__ Yv, double2* G, double2* part, int slices) {
  constexpr int PP = P * P;
  const int tid = threadIdx.x;
  for (int t = tid; t < PP * slices; t += SUB_THREADS) {
    const int u = t % PP, sl = t / PP;
    const int a = u / P, b = u % P;
    if (a > b) continue;
    const int rlo = sl * n / slices, rhi = (sl + 1) * n / slices;
    double sr0 = 0.0, si0 = 0.0, sr1 = 0.0, si1 = 0.0;
    int r = rlo;
    for (; r + 2 <= rhi; r += 2) {
      const double2 v0 = d2conjmul(X[r * P + a], Yv[r * P + b]);
      const double2 v1 = d2conjmul(X[(r + 1) * P + a], Yv[(r + 1) * P + b]);
      sr0 += v0.x;
      si0 += v0.y;
      sr1 += v1.x;
      si1 += v1.y;
    }
    if (r < rhi) {
      const double2 v0 = d2conjmul(X[r * P + a], Yv[r * P + b]);
      sr0 += v0.x;
      si0 += v0.y;
    }
    const double2 v = make_double2(sr0 + sr1, si0 + si1);
    if (slices == 1) G[u] = v;
    else part[t] = v;
  }
  __syncthreads();
  if (slices > 1) {
    for (int u = tid; u < PP; u += SUB_THREADS) {
      if (u / P > u % P) continue;
      double2 v = part[u];
      for (int sl = 1; sl < slices; ++sl) {
        v.x += part[sl * PP + u].x;
        v.y += part[sl * PP + u].y;
      }
      G[u] = v;
    }
    __syncthreads();
  }
}

// Q = orth(Y) by one Cholesky-QR pass: G = Y^H Y (FP64), G = R^H R and R^-1
// (warp 0, FP64; R^-1 stored in FP32 in R), Q = Y R^-1. Returns false (on
// every thread) if G is not numerically positive definite. Ends with a block
// barrier.
template <bool CPLX, int P>
__device__ bool sub_cholqr(int n, const typename Elem<CPLX>::T* __restrict__ Y, typename Elem<CPLX>::T* __restrict__ Q,
                           double2* G, double2* part, int slices, typename Elem<CPLX>::T* R, int* s_ok) {
  using T = typename Elem<CPLX>::T;
  const int tid = threadIdx.x, lane = tid & 31;
  sub_gram<CPLX, P>(n, Y, Y, G, part, slices);
  if (tid < 32) {
    // right-looking Cholesky on the upper triangle: lane j owns column j
    const double g00 = G[0].x;
    bool ok = g00 > 0.0;
    for (int k = 0; k < P; ++k) {
      const double d = G[k * P + k].x;
      if (!(d > 1e-13 * g00)) ok = false;
      const double rkk = sqrt(fmax(d, 1e-300));
      __syncwarp();
      if (lane > k && lane < P) {
        const double2 gk = G[k * P + lane];
        G[k * P + lane] = make_double2(gk.x / rkk, gk.y / rkk);
      }
      if (lane == k) G[k * P + k] = make_double2(rkk, 0.0);
      __syncwarp();
      if (lane > k && lane < P) {
        const double2 rkj = G[k * P + lane];
        for (int i = k + 1; i <= lane; ++i) {
          const double2 rki = G[k * P + i];
          // G_ij -= conj(R_ki) R_kj
          const double2 gij = G[i * P + lane];
          G[i * P + lane] =
              make_double2(gij.x - (rki.x * rkj.x + rki.y * rkj.y), gij.y - (rki.x * rkj.y - rki.y * rkj.x));
        }
      }
      __syncwarp();
    }
    // R^-1 (upper): lane j back-substitutes column j in FP64; x_i (i < j) is
    // kept in the unused lower triangle of G at (j, i), x_j = 1 / R_jj
    if (lane < P) {
      const int j = lane;
      const double xj = 1.0 / G[j * P + j].x;
      for (int i = j - 1; i >= 0; --i) {
        double ar = 0.0, ai = 0.0;
        for (int k = i + 1; k <= j; ++k) {
          const double2 rik = G[i * P + k];
          const double2 xk = k == j ? make_double2(xj, 0.0) : G[j * P + k];
          ar += rik.x * xk.x - rik.y * xk.y;
          ai += rik.x * xk.y + rik.y * xk.x;
        }
        const double rii = G[i * P + i].x;
        G[j * P + i] = make_double2(-ar / rii, -ai / rii);
      }
    }
    __syncwarp();
    for (int u = lane; u < P * P; u += 32) {
      const int a = u / P, c = u % P;
      R[u] = a < c ? from_d2<T>(G[c * P + a]) : (a == c ? from_d2<T>(make_double2(1.0 / G[c * P + c].x, 0.0))
                                                          : zero<T>());
    }
    if (lane == 0) *s_ok = ok ? 1 : 0;
  }
  __syncthreads();
  const bool ok = *s_ok != 0;
  // Q = Y R^-1, a thread per entry
  for (int t = tid; t < n * P; t += SUB_THREADS) {
    const int r = t / P, c = t % P;
    T acc = zero<T>();
    for (int a = 0; a <= c; ++a) acc = acc + mul(Y[r * P + a], R[a * P + c]);
    Q[t] = acc;
  }
  __syncthreads();
  return ok;
}

// Eigenpairs of the P x P Hermitian H (full storage, overwritten) by warp 0:
// cyclic Jacobi with the round-robin ordering, P/2 disjoint rotations per round.
// W receives the eigenvectors (columns), diag(H) the eigenvalues. For the pair
// (p, q) with H_pq = |b| e^{i phi}, J = diag(1, e^{-i phi}) R, R the real
// rotation that diagonalises [[H_pp, |b|], [|b|, H_qq]] (t the smaller root of
// t^2 + 2 tau t - 1 = 0, tau = (H_qq - H_pp) / (2 |b|); Golub & Van Loan 8.5.2).
// The other warps return at once.
template <bool CPLX, int P>
__device__ void sub_jacobi(typename Elem<CPLX>::T* H, typename Elem<CPLX>::T* W) {
  using T = typename Elem<CPLX>::T;
  constexpr int NP = P / 2;
  const int lane = threadIdx.x;
  __shared__ float s_c[NP], s_s[NP], s_er[NP], s_ei[NP];
  __shared__ int s_p[NP], s_q[NP];
  if (threadIdx.x >= 32) return;
  for (int t = lane; t < P * P; t += 32) {
    if constexpr (CPLX) W[t] = cf{(t / P) == (t % P) ? 1.f : 0.f, 0.f};
    else W[t] = (t / P) == (t % P) ? 1.f : 0.f;
  }
  __syncwarp();
  for (int sweep = 0; sweep < SUB_SWEEPS; ++sweep) {
    // stop once every off-diagonal entry is negligible against the diagonal
    float off = 0.f, dg = 0.f;
    for (int t = lane; t < P * P; t += 32) {
      const int i = t / P, j = t % P;
      if (i == j) dg = fmaxf(dg, fabsf(re(H[t])));
      else if (i < j) off = fmaxf(off, abs2(H[t]));
    }
    off = warp_max(off);
    dg = warp_max(dg);
    if (off <= 1e-12f * dg * dg) break;
    for (int round = 0; round < P - 1; ++round) {
      if (lane < NP) {
        int p, q;
        if (lane == 0) {
          p = round;
          q = P - 1;
        } else {
          p = (round + lane) % (P - 1);
          q = (round - lane + (P - 1)) % (P - 1);
        }
        if (p > q) {
          const int t = p;
          p = q;
          q = t;
        }
        const float app = re(H[p * P + p]), aqq = re(H[q * P + q]);
        const T b = H[p * P + q];
        const float ab = sqrtf(abs2(b));
        float c = 1.f, s = 0.f, er = 1.f, ei = 0.f;
        if (ab > 0.f) {
          const float tau = (aqq - app) / (2.f * ab);
          const float t = (tau >= 0.f ? 1.f : -1.f) / (fabsf(tau) + sqrtf(1.f + tau * tau));
          c = rsqrtf(1.f + t * t);
          s = t * c;
          if constexpr (CPLX) {
            er = b.x / ab;  // e^{i phi}
            ei = b.y / ab;
          } else {
            er = b / ab;  // sign of b
          }
        }
        s_c[lane] = c;
        s_s[lane] = s;
        s_er[lane] = er;
        s_ei[lane] = ei;
        s_p[lane] = p;
        s_q[lane] = q;
      }
      __syncwarp();
      // rows: [H_p.; H_q.] <- J^H [H_p.; H_q.], J = [[c, s], [-s e^{-i phi}, c e^{-i phi}]]
#pragma unroll
      for (int t = lane; t < NP * P; t += 32) {
        const int k = t / P, j = t % P;
        const int p = s_p[k], q = s_q[k];
        const float c = s_c[k], s = s_s[k];
        const T hp = H[p * P + j], hq = H[q * P + j];
        if constexpr (CPLX) {
          const cf eq = cf{s_er[k], s_ei[k]} * hq;
          H[p * P + j] = hp * c - eq * s;
          H[q * P + j] = hp * s + eq * c;
        } else {
          const float eq = s_er[k] * hq;
          H[p * P + j] = c * hp - s * eq;
          H[q * P + j] = s * hp + c * eq;
        }
      }
      __syncwarp();
      // columns: [H_.p, H_.q] <- [H_.p, H_.q] J; the same for W
#pragma unroll
      for (int t = lane; t < 2 * NP * P; t += 32) {
        const int which = t / (NP * P), u = t % (NP * P);
        const int k = u / P, i = u % P;
        T* X = which ? W : H;
        const int p = s_p[k], q = s_q[k];
        const float c = s_c[k], s = s_s[k];
        const T xp = X[i * P + p], xq = X[i * P + q];
        if constexpr (CPLX) {
          const cf xe = xq * cf{s_er[k], -s_ei[k]};
          X[i * P + p] = xp * c - xe * s;
          X[i * P + q] = xp * s + xe * c;
        } else {
          const float xe = s_er[k] * xq;
          X[i * P + p] = c * xp - s * xe;
          X[i * P + q] = s * xp + c * xe;
        }
      }
      __syncwarp();
    }
  }
}

// ---------------------------------------------------------------------------
// The kernel: one CTA per patch; n_active = -1 hands the patch to k_eig.
// ---------------------------------------------------------------------------
template <bool CPLX, int P>
__global__ void __launch_bounds__(SUB_THREADS, 1) k_sub(int n, EigParams ep, PatchWork w) {
  using T = typename Elem<CPLX>::T;
  extern __shared__ __align__(16) unsigned char sm[];
  const SubLayout L = sub_layout(CPLX, n, P);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int p = blockIdx.x;
  if (ep.only_unfinished && w.n_active[p] >= 0) return;  // certified by an earlier pass
  T* A = reinterpret_cast<T*>(sm + L.a);
  T* q = reinterpret_cast<T*>(sm + L.q);
  T* y = reinterpret_cast<T*>(sm + L.y);
  double2* G = reinterpret_cast<double2*>(sm + L.g);
  double2* part = reinterpret_cast<double2*>(sm + L.part);
  T* R = reinterpret_cast<T*>(sm + L.r);
  T* H = reinterpret_cast<T*>(sm + L.h);
  T* W = reinterpret_cast<T*>(sm + L.w);
  float* th = reinterpret_cast<float*>(sm + L.th);
  int* perm = reinterpret_cast<int*>(sm + L.perm);
  float* res2 = reinterpret_cast<float*>(sm + L.res);
  const int S = L.slices;
  __shared__ int s_ok, s_done;
  __shared__ double s_md;
  __shared__ float s_red[SUB_NW];
  auto swap_qy = [&] {
    T* t_ = q;
    q = y;
    y = t_;
  };

  // stage and scale the Gram (by 1 / max diagonal, as k_eig)
  const T* Gg = reinterpret_cast<const T*>(w.gram + (int64_t)p * w.gram_stride);
  const int np = (int)pk_size(n);
  for (int i = tid; i < np; i += SUB_THREADS) A[i] = Gg[i];
  __syncthreads();
  float md = 0.f;
  for (int i = tid; i < n; i += SUB_THREADS) md = fmaxf(md, re(A[pk(i, i, n)]));
  md = warp_max(md);
  if (lane == 0) s_red[warp] = md;
  __syncthreads();
  md = warp_max(lane < SUB_NW ? s_red[lane] : 0.f);
  const float sc = md > 0.f ? 1.f / md : 1.f;
  if (tid == 0) s_md = md > 0.f ? (double)md : 1.0;
  for (int i = tid; i < np; i += SUB_THREADS) A[i] = A[i] * sc;
  // pseudo-random start block (a fixed hash of the row and column)
  for (int t = tid; t < n * P; t += SUB_THREADS) {
    uint32_t hsh = (uint32_t)(t + 17) * 2654435761u;
    hsh ^= hsh >> 13;
    hsh *= 0x5bd1e995u;
    hsh ^= hsh >> 15;
    const float u = (float)(hsh & 0xffff) * (1.f / 65536.f) - 0.5f;
    const float v = (float)(hsh >> 16) * (1.f / 65536.f) - 0.5f;
    if constexpr (CPLX) q[t] = cf{u, v};
    else q[t] = u;
  }
  __syncthreads();
  bool ok = true;
  const double md64 = s_md;
  const double thr = ep.d_threshold ? *ep.d_threshold : ep.threshold;
  const double thr2s = thr * thr / md64;  // the threshold on scaled eigenvalues
  int steps = SUB_FIRST;
  for (int check = 0; ok && check < SUB_CHECKS; ++check) {
    // power steps: one Cholesky-QR each, a second one before Rayleigh-Ritz
    for (int it = 0; ok && it < steps; ++it) {
      sub_product<CPLX, P>(A, n, q, y);
      __syncthreads();
      ok = sub_cholqr<CPLX, P>(n, y, q, G, part, S, R, &s_ok);
    }
    ok = ok && sub_cholqr<CPLX, P>(n, q, y, G, part, S, R, &s_ok);
    if (!ok) break;
    swap_qy();
    // Rayleigh-Ritz: Z = C Q (into y), H = Q^H Z
    sub_product<CPLX, P>(A, n, q, y);
    __syncthreads();
    sub_gram<CPLX, P>(n, q, y, G, part, S);
    for (int u = tid; u < P * P; u += SUB_THREADS) {
      const int a = u / P, b = u % P;
      if (a > b) continue;
      double2 v = G[u];
      if (a == b) v.y = 0.0;
      H[a * P + b] = from_d2<T>(v);
      H[b * P + a] = from_d2<T>(make_double2(v.x, -v.y));
    }
    if (tid < P) res2[tid] = 0.f;
    __syncthreads();
    sub_jacobi<CPLX, P>(H, W);
    __syncthreads();
    // descending order of the Ritz values
    if (tid < P) {
      const float v = re(H[tid * P + tid]);
      int rk = 0;
      for (int j = 0; j < P; ++j) {
        const float u = re(H[j * P + j]);
        rk += (u > v || (u == v && j < tid)) ? 1 : 0;
      }
      perm[rk] = tid;
      th[rk] = v;
    }
    __syncthreads();
    // V = Q W and C V = Z W in sorted order, in place: a warp owns 32 / P rows
    // (a lane per entry), reads them, then overwrites them; the squared residuals
    // |(C V)_ri - theta_i V_ri|^2 are summed per column
    for (int base = warp * 32; base < n * P; base += SUB_THREADS) {
      const int t = base + lane;
      const bool act = t < n * P;
      const int r = act ? t / P : 0, i = t % P;
      T v = zero<T>(), z = zero<T>();
      if (act) {
        const int c = perm[i];
#pragma unroll
        for (int a = 0; a < P; ++a) {
          const T wac = W[a * P + c];
          v = v + mul(q[r * P + a], wac);
          z = z + mul(y[r * P + a], wac);
        }
      }
      __syncwarp();
      float e2 = 0.f;
      if (act) {
        q[r * P + i] = v;
        y[r * P + i] = z;
        e2 = abs2(z - v * th[i]);
      }
#pragma unroll
      for (int o = 16; o >= P; o >>= 1) e2 += __shfl_xor_sync(0xffffffffu, e2, o);
      if (lane < P) atomicAdd(&res2[lane], e2);
    }
    __syncthreads();
    if (tid == 0) {
      // the reference rule on the Ritz values: s_i = sqrt(theta_i) > threshold
      int cnt = 0;
      while (cnt < P && sqrt(fmax((double)th[cnt], 0.0) * md64) > thr) ++cnt;
      bool cert = cnt < P && (double)th[P - 1] < 0.25 * thr2s;
      for (int i = 0; cert && i < cnt; ++i) cert = sqrtf(res2[i]) <= SUB_TOLR * th[i];
      if (cert) cert = (double)th[cnt] + sqrt((double)res2[cnt]) < thr2s;
      s_done = cert ? 1 + cnt : 0;
      if (cert) {
        w.rank[p] = cnt;
        w.noise[p] = nanf("");
        w.n_active[p] = cnt;
      }
    }
    __syncthreads();
    if (s_done) {
      const int act = s_done - 1;
      // Ritz vectors of the kept components, column a at a * 2n floats
      float* vbase = w.vec + (int64_t)p * w.vec_stride;
      for (int t = tid; t < act * n; t += SUB_THREADS) {
        const int a = t / n, r = t % n;
        const T v = q[r * P + a];
        if constexpr (CPLX) reinterpret_cast<cf*>(vbase + (int64_t)a * 2 * n)[r] = v;
        else vbase[(int64_t)a * 2 * n + r] = v;
      }
      for (int a = tid; a < act; a += SUB_THREADS) w.coef[(int64_t)p * n + a] = 1.f;
      return;
    }
    // the next power step starts from C V (in y)
    ok = sub_cholqr<CPLX, P>(n, y, q, G, part, S, R, &s_ok);
    steps = SUB_MORE - 1;
  }
  if (tid == 0) w.n_active[p] = -1;  // not certified: the full solver takes it
}

template <bool CPLX, int P>
static cudaError_t sub_pass(int n, const EigParams& ep, const PatchWork& w, cudaStream_t s) {
  const size_t smem = sub_layout(CPLX, n, P).total;
  cudaError_t err = cudaFuncSetAttribute(k_sub<CPLX, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  PD_TIMED(P == 8 ? "eig_sub8" : "eig_sub16", s, k_sub<CPLX, P><<<w.count, SUB_THREADS, smem, s>>>(n, ep, w));
  return cudaGetLastError();
}

// P = 8 on every patch, then P = 16 on the patches it did not certify (when
// that block fits); the caller's k_eig pass takes what is left.
cudaError_t launch_sub(bool cplx, int n, const EigParams& ep, const PatchWork& w, cudaStream_t s) {
  const int rows = ep.rows;
  EigParams e8 = ep;
  e8.only_unfinished = 0;
  cudaError_t err = cplx ? sub_pass<true, 8>(n, e8, w, s) : sub_pass<false, 8>(n, e8, w, s);
  if (err != cudaSuccess || !sub_fits(cplx, n, rows, 16)) return err;
  EigParams e16 = ep;
  e16.only_unfinished = 1;
  return cplx ? sub_pass<true, 16>(n, e16, w, s) : sub_pass<false, 16>(n, e16, w, s);
}

}  // namespace pd
