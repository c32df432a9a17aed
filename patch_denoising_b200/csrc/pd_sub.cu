// Subspace eigensolver for the hard-threshold rule on the mixed-precision path
// (RawSVDDenoiser / NordicDenoiser, space_time/lowrank.py:170-184): one CTA per
// patch finds the eigenpairs of the scaled Gram C that lie above the known
// threshold, without reducing the whole matrix to tridiagonal form.
//
//  1. Block power iteration on P = 16 columns: Y = C Q, then Q = orth(Y) by
//     Cholesky QR applied twice (CholQR2: the P x P Gram Y^H Y and its Cholesky
//     factor in FP64, Q = Y R^-1 in FP32). Columns converge to the eigenvectors
//     above the bulk at the rate lambda_{P+1} / lambda_i per step.
//  2. Rayleigh-Ritz: Z = C Q, H = Q^H Z (P x P Hermitian), cyclic Jacobi
//     eigensolver of H in FP32 (parallel round-robin ordering), Ritz vectors
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
// applies where that and the P-column blocks fit (sub_supported).
#include <float.h>

#include "pd_common.cuh"
#include "pd_kernels.cuh"
#include "pd_profile.cuh"

namespace pd {

constexpr int SUB_THREADS = 512;
constexpr int SUB_NW = SUB_THREADS / 32;
constexpr int SUB_P = 16;        // block columns
constexpr int SUB_FIRST = 3;     // power steps before the first Rayleigh-Ritz check
constexpr int SUB_MORE = 2;      // power steps between later checks
constexpr int SUB_CHECKS = 4;    // checks before the patch goes to k_eig
constexpr int SUB_SWEEPS = 10;   // Jacobi sweeps at most
constexpr float SUB_TOLR = 2e-5f;
constexpr size_t SUB_SMEM_LIMIT = 227 * 1024 - 1024;

struct SubLayout {
  size_t a, q, y, g, rinv, h, w, th, perm, res, total;
};

__host__ __device__ inline size_t sub_al(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline SubLayout sub_layout(bool cplx, int n) {
  const size_t es = cplx ? 8 : 4;
  SubLayout L;
  size_t o = 0;
  L.a = o;
  o += sub_al((size_t)pk_size(n) * es);
  L.q = o;
  o += sub_al((size_t)n * SUB_P * es);
  L.y = o;
  o += sub_al((size_t)n * SUB_P * es);
  L.g = o;
  o += sub_al((size_t)SUB_P * SUB_P * 16);  // FP64 complex Gram (real: imaginary parts stay 0)
  L.rinv = o;
  o += sub_al((size_t)SUB_P * SUB_P * es);
  L.h = o;
  o += sub_al((size_t)SUB_P * SUB_P * es);
  L.w = o;
  o += sub_al((size_t)SUB_P * SUB_P * es);
  L.th = o;
  o += sub_al(SUB_P * 4);
  L.perm = o;
  o += sub_al(SUB_P * 4);
  L.res = o;
  o += sub_al((size_t)SUB_NW * SUB_P * 4);
  L.total = o;
  return L;
}

bool sub_supported(bool cplx, int n, int rows) {
  return n >= 3 * SUB_P && rows > 2 * SUB_P && sub_layout(cplx, n).total <= SUB_SMEM_LIMIT;
}

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

// Y = C Q over the packed lower C (n x n Hermitian), Q and Y row-major n x P.
// A warp owns 16 rows; lane (r, h) accumulates row r against columns 8h..8h+7.
// C(row, k) is the stored column-k entry for row >= k, else the conjugate of
// the entry stored in column row at row k.
template <bool CPLX>
__device__ void sub_product(const typename Elem<CPLX>::T* __restrict__ A, int n,
                            const typename Elem<CPLX>::T* __restrict__ Q, typename Elem<CPLX>::T* __restrict__ Y) {
  using T = typename Elem<CPLX>::T;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r = lane & 15, h = lane >> 4;
  for (int rb = warp; rb * 16 < n; rb += SUB_NW) {
    const int row = rb * 16 + r;
    const bool live = row < n;
    const int64_t cbr = live ? pk(row, row, n) - row : 0;
    T acc[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j] = zero<T>();
    int64_t cbk = 0;  // pk(k, k, n) - k
    for (int k = 0; k < n; ++k) {
      T c = zero<T>();
      if (live) c = row >= k ? A[cbk + row] : cj(A[cbr + k]);
      const float4* q4 = reinterpret_cast<const float4*>(Q + (int64_t)k * SUB_P + h * 8);
      if constexpr (CPLX) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const float4 v = q4[j];
          acc[2 * j] = acc[2 * j] + c * cf{v.x, v.y};
          acc[2 * j + 1] = acc[2 * j + 1] + c * cf{v.z, v.w};
        }
      } else {
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const float4 v = q4[j];
          acc[4 * j] += c * v.x;
          acc[4 * j + 1] += c * v.y;
          acc[4 * j + 2] += c * v.z;
          acc[4 * j + 3] += c * v.w;
        }
      }
      cbk += n - k - 1;
    }
    if (live) {
#pragma unroll
      for (int j = 0; j < 8; ++j) Y[(int64_t)row * SUB_P + h * 8 + j] = acc[j];
    }
  }
}

// Q = orth(Y) by one Cholesky-QR pass: G = Y^H Y (FP64), G = R^H R (warp 0,
// FP64), Q = Y R^-1. Returns false (on every thread) if G is not numerically
// positive definite. Ends with a block barrier.
template <bool CPLX>
__device__ bool sub_cholqr(int n, const typename Elem<CPLX>::T* __restrict__ Y, typename Elem<CPLX>::T* __restrict__ Q,
                           double2* G, typename Elem<CPLX>::T* Rinv, int* s_ok) {
  using T = typename Elem<CPLX>::T;
  const int tid = threadIdx.x, lane = tid & 31;
  constexpr int P = SUB_P;
  // Gram: a thread per upper entry (a <= b)
  for (int t = tid; t < P * P; t += SUB_THREADS) {
    const int a = t / P, b = t % P;
    if (a > b) continue;
    double sr = 0.0, si = 0.0;
    for (int r = 0; r < n; ++r) {
      const double2 v = d2conjmul(Y[(int64_t)r * P + a], Y[(int64_t)r * P + b]);
      sr += v.x;
      si += v.y;
    }
    G[a * P + b] = make_double2(sr, si);
  }
  __syncthreads();
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
      __syncwarp();
      if (lane == k) G[k * P + k] = make_double2(rkk, 0.0);
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
    // R^-1 (upper): lane j solves R x = e_j by back substitution
    if (lane < P) {
      const int j = lane;
      double2 x[P];
#pragma unroll
      for (int i = 0; i < P; ++i) x[i] = make_double2(0.0, 0.0);
      for (int i = j; i >= 0; --i) {
        double2 acc = make_double2(i == j ? 1.0 : 0.0, 0.0);
        for (int k = i + 1; k <= j; ++k) {
          const double2 rik = G[i * P + k];
          acc.x -= rik.x * x[k].x - rik.y * x[k].y;
          acc.y -= rik.x * x[k].y + rik.y * x[k].x;
        }
        const double rii = G[i * P + i].x;
        x[i] = make_double2(acc.x / rii, acc.y / rii);
      }
#pragma unroll
      for (int i = 0; i < P; ++i) Rinv[i * P + j] = from_d2<T>(x[i]);
    }
    if (lane == 0) *s_ok = ok ? 1 : 0;
  }
  __syncthreads();
  const bool ok = *s_ok != 0;
  // Q = Y R^-1, a thread per (row, column)
  for (int t = tid; t < n * P; t += SUB_THREADS) {
    const int r = t / P, c = t % P;
    T acc = zero<T>();
    for (int a = 0; a <= c; ++a) acc = acc + mul(Y[(int64_t)r * P + a], Rinv[a * P + c]);
    Q[(int64_t)r * P + c] = acc;
  }
  __syncthreads();
  return ok;
}

// Eigenpairs of the P x P Hermitian H (full storage, overwritten): cyclic
// Jacobi with the round-robin ordering, P/2 disjoint rotations per round, run
// by warps 0-1 with a named barrier (the other warps return at once). W
// receives the eigenvectors (columns), diag(H) the eigenvalues. For the pair
// (p, q) with H_pq = |b| e^{i phi}, J = diag(1, e^{-i phi}) R, R the real
// rotation that diagonalises [[H_pp, |b|], [|b|, H_qq]] (t the smaller root of
// t^2 + 2 tau t - 1 = 0, tau = (H_qq - H_pp) / (2 |b|); Golub & Van Loan 8.5.2).
template <bool CPLX>
__device__ void sub_jacobi(typename Elem<CPLX>::T* H, typename Elem<CPLX>::T* W) {
  using T = typename Elem<CPLX>::T;
  constexpr int P = SUB_P, NP = SUB_P / 2;
  const int tid = threadIdx.x;
  __shared__ float s_c[NP], s_s[NP], s_er[NP], s_ei[NP];
  __shared__ int s_p[NP], s_q[NP];
  __shared__ int s_stop;
  if (tid >= 64) return;
  auto bar = [] { asm volatile("bar.sync 1, 64;" ::: "memory"); };
  for (int t = tid; t < P * P; t += 64) {
    if constexpr (CPLX) W[t] = cf{(t / P) == (t % P) ? 1.f : 0.f, 0.f};
    else W[t] = (t / P) == (t % P) ? 1.f : 0.f;
  }
  bar();
  for (int sweep = 0; sweep < SUB_SWEEPS; ++sweep) {
    // stop once every off-diagonal entry is negligible against the diagonal
    if (tid == 0) {
      float off = 0.f, dg = 0.f;
      for (int i = 0; i < P; ++i) {
        dg = fmaxf(dg, fabsf(re(H[i * P + i])));
        for (int j = i + 1; j < P; ++j) off = fmaxf(off, sqrtf(abs2(H[i * P + j])));
      }
      s_stop = (off <= 1e-7f * dg) ? 1 : 0;
    }
    bar();
    if (s_stop) break;
    for (int round = 0; round < P - 1; ++round) {
      if (tid < NP) {
        int p, q;
        if (tid == 0) {
          p = round;
          q = P - 1;
        } else {
          p = (round + tid) % (P - 1);
          q = (round - tid + (P - 1)) % (P - 1);
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
        s_c[tid] = c;
        s_s[tid] = s;
        s_er[tid] = er;
        s_ei[tid] = ei;
        s_p[tid] = p;
        s_q[tid] = q;
      }
      bar();
      // rows: [H_p.; H_q.] <- J^H [H_p.; H_q.], J = [[c, s], [-s e^{-i phi}, c e^{-i phi}]]
      for (int t = tid; t < NP * P; t += 64) {
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
      bar();
      // columns: [H_.p, H_.q] <- [H_.p, H_.q] J; the same for W
      for (int t = tid; t < 2 * NP * P; t += 64) {
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
      bar();
    }
  }
}

// ---------------------------------------------------------------------------
// The kernel: one CTA per patch; n_active = -1 hands the patch to k_eig.
// ---------------------------------------------------------------------------
template <bool CPLX>
__global__ void __launch_bounds__(SUB_THREADS, 1) k_sub(int n, EigParams ep, PatchWork w) {
  using T = typename Elem<CPLX>::T;
  constexpr int P = SUB_P;
  extern __shared__ __align__(16) unsigned char sm[];
  const SubLayout L = sub_layout(CPLX, n);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int p = blockIdx.x;
  T* A = reinterpret_cast<T*>(sm + L.a);
  T* q = reinterpret_cast<T*>(sm + L.q);
  T* y = reinterpret_cast<T*>(sm + L.y);
  double2* G = reinterpret_cast<double2*>(sm + L.g);
  T* Rinv = reinterpret_cast<T*>(sm + L.rinv);
  T* H = reinterpret_cast<T*>(sm + L.h);
  T* W = reinterpret_cast<T*>(sm + L.w);
  float* th = reinterpret_cast<float*>(sm + L.th);
  int* perm = reinterpret_cast<int*>(sm + L.perm);
  float* rpart = reinterpret_cast<float*>(sm + L.res);
  __shared__ int s_ok, s_done;
  __shared__ double s_md;
  __shared__ float s_red[SUB_NW];

  // stage and scale the Gram (by 1 / max diagonal, as k_eig)
  const T* Gg = reinterpret_cast<const T*>(w.gram + (int64_t)p * w.gram_stride);
  const int64_t np = pk_size(n);
  for (int64_t i = tid; i < np; i += SUB_THREADS) A[i] = Gg[i];
  __syncthreads();
  float md = 0.f;
  for (int i = tid; i < n; i += SUB_THREADS) md = fmaxf(md, re(A[pk(i, i, n)]));
  md = warp_max(md);
  if (lane == 0) s_red[warp] = md;
  __syncthreads();
  md = warp_max(lane < SUB_NW ? s_red[lane] : 0.f);
  const float sc = md > 0.f ? 1.f / md : 1.f;
  if (tid == 0) s_md = md > 0.f ? (double)md : 1.0;
  for (int64_t i = tid; i < np; i += SUB_THREADS) A[i] = A[i] * sc;
  // pseudo-random start block (a fixed hash of the row and column)
  for (int t = tid; t < n * P; t += SUB_THREADS) {
    uint32_t hsh = (uint32_t)(t + 17) * 2654435761u;
    hsh ^= hsh >> 13;
    hsh *= 0x5bd1e995u;
    hsh ^= hsh >> 15;
    const float u = (float)(hsh & 0xffff) * (1.f / 65536.f) - 0.5f;
    const float v = (float)(hsh >> 16) * (1.f / 65536.f) - 0.5f;
    if constexpr (CPLX) y[t] = cf{u, v};
    else y[t] = u;
  }
  __syncthreads();
  bool ok = sub_cholqr<CPLX>(n, y, q, G, Rinv, &s_ok);
  ok = ok && sub_cholqr<CPLX>(n, q, y, G, Rinv, &s_ok);
  {
    T* t_ = q;
    q = y;
    y = t_;
  }
  const double md64 = s_md;
  const double thr = ep.d_threshold ? *ep.d_threshold : ep.threshold;
  const double thr2s = thr * thr / md64;  // the threshold on scaled eigenvalues
  int steps = SUB_FIRST;
  for (int check = 0; ok && check < SUB_CHECKS; ++check) {
    for (int it = 0; ok && it < steps; ++it) {
      sub_product<CPLX>(A, n, q, y);
      __syncthreads();
      ok = sub_cholqr<CPLX>(n, y, q, G, Rinv, &s_ok);
      ok = ok && sub_cholqr<CPLX>(n, q, y, G, Rinv, &s_ok);
      T* t_ = q;
      q = y;
      y = t_;
    }
    if (!ok) break;
    // Rayleigh-Ritz: Z = C Q (into y), H = Q^H Z
    sub_product<CPLX>(A, n, q, y);
    __syncthreads();
    for (int t = tid; t < P * P; t += SUB_THREADS) {
      const int a = t / P, b = t % P;
      if (a > b) continue;
      double sr = 0.0, si = 0.0;
      for (int r = 0; r < n; ++r) {
        const double2 v = d2conjmul(q[(int64_t)r * P + a], y[(int64_t)r * P + b]);
        sr += v.x;
        si += v.y;
      }
      if (a == b) si = 0.0;
      H[a * P + b] = from_d2<T>(make_double2(sr, si));
      H[b * P + a] = from_d2<T>(make_double2(sr, -si));
    }
    __syncthreads();
    sub_jacobi<CPLX>(H, W);
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
    // V = Q W and C V = Z W in sorted order, in place (a thread per row), with
    // per-warp partial sums of the squared residuals
    float r2[P];
#pragma unroll
    for (int i = 0; i < P; ++i) r2[i] = 0.f;
    for (int r = tid; r < n; r += SUB_THREADS) {
      T qr[P], vr[P];
#pragma unroll
      for (int a = 0; a < P; ++a) qr[a] = q[(int64_t)r * P + a];
#pragma unroll
      for (int i = 0; i < P; ++i) {
        const int c = perm[i];
        T acc = zero<T>();
#pragma unroll
        for (int a = 0; a < P; ++a) acc = acc + mul(qr[a], W[a * P + c]);
        vr[i] = acc;
      }
#pragma unroll
      for (int a = 0; a < P; ++a) {
        q[(int64_t)r * P + a] = vr[a];
        qr[a] = y[(int64_t)r * P + a];
      }
#pragma unroll
      for (int i = 0; i < P; ++i) {
        const int c = perm[i];
        T acc = zero<T>();
#pragma unroll
        for (int a = 0; a < P; ++a) acc = acc + mul(qr[a], W[a * P + c]);
        y[(int64_t)r * P + i] = acc;
        r2[i] += abs2(acc - vr[i] * th[i]);
      }
    }
#pragma unroll
    for (int i = 0; i < P; ++i) {
      const float s = warp_sum(r2[i]);
      if (lane == 0) rpart[warp * P + i] = s;
    }
    __syncthreads();
    if (tid == 0) {
      float res[P];
      for (int i = 0; i < P; ++i) {
        float s = 0.f;
        for (int k = 0; k < SUB_NW; ++k) s += rpart[k * P + i];
        res[i] = sqrtf(s);
      }
      // the reference rule on the Ritz values: s_i = sqrt(theta_i) > threshold
      int cnt = 0;
      while (cnt < P && sqrt(fmax((double)th[cnt], 0.0) * md64) > thr) ++cnt;
      bool cert = cnt < P && (double)th[P - 1] < 0.25 * thr2s;
      for (int i = 0; cert && i < cnt; ++i) cert = res[i] <= SUB_TOLR * th[i];
      if (cert) cert = (double)th[cnt] + (double)res[cnt] < thr2s;
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
        const T v = q[(int64_t)r * P + a];
        if constexpr (CPLX) reinterpret_cast<cf*>(vbase + (int64_t)a * 2 * n)[r] = v;
        else vbase[(int64_t)a * 2 * n + r] = v;
      }
      for (int a = tid; a < act; a += SUB_THREADS) w.coef[(int64_t)p * n + a] = 1.f;
      return;
    }
    // the next power step starts from C V (in y)
    ok = sub_cholqr<CPLX>(n, y, q, G, Rinv, &s_ok);
    ok = ok && sub_cholqr<CPLX>(n, q, y, G, Rinv, &s_ok);
    T* t_ = q;
    q = y;
    y = t_;
    steps = SUB_MORE - 1;
  }
  if (tid == 0) w.n_active[p] = -1;  // not certified: the full solver takes it
}

cudaError_t launch_sub(bool cplx, int n, const EigParams& ep, const PatchWork& w, cudaStream_t s) {
  const size_t smem = sub_layout(cplx, n).total;
  auto kern = cplx ? k_sub<true> : k_sub<false>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  PD_TIMED("eig_sub", s, kern<<<w.count, SUB_THREADS, smem, s>>>(n, ep, w));
  return cudaGetLastError();
}

}  // namespace pd
