// Per-patch Hermitian eigensolver and threshold rules (one CTA per patch: 512
// threads, or 128 threads and four CTAs per SM for patches of at most 128
// frames whose layout fits a quarter of shared memory).
//
//  1. The packed lower Gram C = Xc^H Xc (n = frames) is staged in shared memory
//     when it fits (else worked on in place in global memory) and scaled by
//     1 / max(diag).
//  2. Householder reduction to real symmetric tridiagonal form T = Q^H C Q
//     (H_j = I - tau_j v_j v_j^H, v_j stored below the subdiagonal), the
//     classical unblocked algorithm (Golub & Van Loan, sec. 8.3.1).
//  3. Eigenvalues of T at requested indices by Sturm counts: a few by
//     multisection (one warp evaluates 32 points per round, shrinking the
//     bracket 33x), a whole spectrum by bisection with a thread per eigenvalue.
//  4. The reference threshold rule of the method, evaluated in FP64 on the
//     eigenvalues (space_time/lowrank.py: MP-PCA :42-63, Hybrid :104-119,
//     Raw/NORDIC :170-184, Optimal :379-407), gives maxidx, noise_var and the
//     active components with their synthesis coefficients.
//  5. Eigenvectors of T for the active components by the twisted factorisation
//     (Parlett & Dhillon, 1997), re-orthogonalised inside eigenvalue clusters
//     (block classical Gram-Schmidt for whole bulks), then back-transformed by
//     the reflectors, a warp applying each reflector to a group of vectors:
//     eigenvectors of C.
#include <float.h>

#include "pd_common.cuh"
#include "pd_kernels.cuh"
#include "pd_profile.cuh"
#include "pd_rules.cuh"

namespace pd {

constexpr int EIG_THREADS = 512;
constexpr int EIG_NW = EIG_THREADS / 32;
constexpr float CAND_MARGIN = 1e-3f;

struct EigLayout {
  size_t a, d, e, e2, tau, vb, wb, pw, pd, idx, lam, aidx, alam, acoef, total;
};

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) & ~size_t(15); }

// th: the CTA's threads. pw holds a row of partial products per warp in the
// tridiagonalisation, and later the adaptive rule's 3 n doubles and the block
// re-orthogonalisation's 16 n floats: at least 64 n bytes.
__host__ __device__ inline EigLayout eig_layout(bool cplx, int n, bool in_smem, int th = EIG_THREADS) {
  const size_t es = cplx ? 8 : 4;
  EigLayout L;
  size_t o = 0;
  L.a = o;
  o += in_smem ? al16((size_t)pk_size(n) * es) : 0;
  L.d = o;
  o += al16(4 * (size_t)n);
  L.e = o;
  o += al16(4 * (size_t)n);
  L.e2 = o;
  o += al16(4 * (size_t)n);
  L.tau = o;
  o += al16(es * n);
  L.vb = o;
  o += al16(es * 2 * n);
  L.wb = o;
  o += al16(es * 2 * n);
  L.pw = o;
  {
    const size_t per_warp = es * n * (size_t)(th / 32), scratch = 64 * (size_t)n;
    o += al16(per_warp > scratch ? per_warp : scratch);
  }
  L.pd = o;
  o += al16(es * n);
  L.idx = o;
  o += al16(4 * (size_t)n);
  L.lam = o;
  o += al16(4 * (size_t)n);
  L.aidx = o;
  o += al16(4 * (size_t)n);
  L.alam = o;
  o += al16(4 * (size_t)n);
  L.acoef = o;
  o += al16(4 * (size_t)n);
  L.total = o;
  return L;
}

constexpr size_t EIG_SMEM_LIMIT = 227 * 1024 - 2048;  // leave room for static shared

size_t eig_smem_bytes(bool cplx, int n, bool* in_smem) {
  EigLayout L = eig_layout(cplx, n, true);
  if (L.total <= EIG_SMEM_LIMIT) {
    *in_smem = true;
    return L.total;
  }
  *in_smem = false;
  return eig_layout(cplx, n, false).total;
}

// ---------------------------------------------------------------------------
// Reductions with static shared scratch
// ---------------------------------------------------------------------------
__device__ __forceinline__ float bsum_f(float v) {
  __shared__ float red[32];
  return block_sum<float>(v, red);
}
__device__ __forceinline__ cf bsum_c(cf v) {
  __shared__ cf redc[32];
  return block_sum<cf>(v, redc);
}
template <class T>
__device__ __forceinline__ T bsum(T v);
template <>
__device__ __forceinline__ float bsum<float>(float v) { return bsum_f(v); }
template <>
__device__ __forceinline__ cf bsum<cf>(cf v) { return bsum_c(v); }

__device__ __forceinline__ float bmax_f(float v) {
  __shared__ float red[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  float r = lane < (int)((blockDim.x + 31) >> 5) ? red[lane] : -FLT_MAX;
  return warp_max(r);
}
__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// ---------------------------------------------------------------------------
// Householder tridiagonalisation (lower storage, packed), after LAPACK
// zhetd2 / ssytd2 with uplo = 'L' (the reduction behind scipy's eigh): step j
// reflects column j below the subdiagonal with H_j = I - tau_j v_j v_j^H,
// v_j(j+1) = 1, and updates the trailing block A22 <- A22 - v w^H - w v^H with
// p = A22 v, w = tau p + alpha v, alpha = -tau/2 (tau p)^H v.
//
// Four block barriers per step. The rank-2 update of step j-1 and the product
// p_j = A22 v_j of step j share one pass over A22, so each stored element is
// loaded, updated, stored and multiplied once per step; only column j, which
// reflector j is built from, takes its update ahead of the pass.
//   phase 1 (all):    alpha_{j-1} (each warp, from the per-warp partials);
//                     column j -= update_{j-1}, a thread per row; its norm
//                     (barrier); reflector j, its scalars formed by every
//                     thread                                    (barrier)
//   phase 2 (all):    A22 -= update_{j-1}; partial sums of A22 v_j: warps own
//                     columns k, lanes own rows i = lane + 32 s (registers); the
//                     row part A22(i,k) v_k accumulates in registers, the
//                     transposed part sum_i conj(A22(i,k)) v_i is reduced over
//                     lanes eight columns at a time (reduce-scatter butterfly)
//                                                               (barrier)
//   phase 3 (all):    p_j from the partials; tau_j p_j; partials of (tau p)^H v
//                                                               (barrier)
// v and tau p live in two buffers of n entries indexed by row (step parity).
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ T shfl_idx(T v, int src);
template <>
__device__ __forceinline__ float shfl_idx<float>(float v, int src) { return __shfl_sync(0xffffffffu, v, src); }
template <>
__device__ __forceinline__ cf shfl_idx<cf>(cf v, int src) {
  return cf{__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src)};
}
template <bool CPLX, int NS, int TH>
__device__ void tridiagonalize(typename Elem<CPLX>::T* A, int n, float* d, float* e, typename Elem<CPLX>::T* tau,
                               typename Elem<CPLX>::T* vb, typename Elem<CPLX>::T* wb,
                               typename Elem<CPLX>::T* pw, typename Elem<CPLX>::T* pd) {
  using T = typename Elem<CPLX>::T;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  __shared__ T s_red[(TH / 32)];     // per-warp partials of (tau p)^H v
  __shared__ float s_x2[(TH / 32)];  // per-warp partials of the column norm
  __shared__ T s_sub;             // A(j+1, j) after its last update
  T one;
  if constexpr (CPLX) one = cf{1.f, 0.f};
  else one = 1.f;
  // buffer 1 holds "step -1": v = w = 0, so the first pending update is exactly zero
  for (int i = tid; i < 2 * n; i += TH) {
    vb[i] = zero<T>();
    wb[i] = zero<T>();
  }
  if (tid < (TH / 32)) s_red[tid] = zero<T>();
  T tau_prev = zero<T>();  // tau of the previous step (every thread)
  __syncthreads();
  for (int j = 0; j < n - 1; ++j) {
    const int m = n - j - 1;
    const int cur = j & 1;
    T* vc = vb + cur * n;
    T* wc = wb + cur * n;
    const T* vp = vb + (cur ^ 1) * n;
    const T* wp = wb + (cur ^ 1) * n;
    // ---- phase 1 (all): finish column j (thread t owns row j + t), build reflector j
    T al, tj = zero<T>();
    {
      T dot = lane < (TH / 32) ? s_red[lane] : zero<T>();
      dot = warp_sum(dot);
      al = mul(tau_prev, dot) * -0.5f;  // w_{j-1} = tau p + al v
      const int r = j + tid;            // n - j <= n <= TH rows
      T a = zero<T>();
      float x2 = 0.f;
      if (r < n) {
        const T vj = vp[j];
        const T cuj = cj(wp[j] + mul(al, vj)), cvj = cj(vj);
        const T v = vp[r];
        const T u = wp[r] + mul(al, v);
        a = A[pk(r, j, n)] - (mul(v, cuj) + mul(u, cvj));
        if (r >= j + 2) x2 = abs2(a);
      }
      x2 = warp_sum(x2);
      if (lane == 0) s_x2[warp] = x2;
      if (tid == 1) s_sub = a;  // A(j+1, j)
      if (tid == 0) d[j] = re(a);
      __syncthreads();
      float xn2 = lane < (TH / 32) ? s_x2[lane] : 0.f;
      xn2 = warp_sum(xn2);
      const T alpha = s_sub;
      const float ar = re(alpha);
      float ai = 0.f;
      if constexpr (CPLX) ai = alpha.y;
      const bool refl = !(xn2 == 0.f && ai == 0.f);
      T inv = zero<T>();
      float ej = ar;
      if (refl) {  // every thread forms the same scalars
        const float nrm = sqrtf(ar * ar + ai * ai + xn2);
        const float beta = ar >= 0.f ? -nrm : nrm;
        if constexpr (CPLX) {
          tj = cf{(beta - ar) / beta, -ai / beta};
          const float dr = ar - beta, di = ai;
          const float den = dr * dr + di * di;
          inv = cf{dr / den, -di / den};
        } else {
          tj = (beta - ar) / beta;
          inv = 1.f / (ar - beta);
        }
        ej = beta;
      }
      if (r > j && r < n) {
        T v = zero<T>();
        if (refl) {
          v = (r == j + 1) ? one : mul(a, inv);
          if (r > j + 1) A[pk(r, j, n)] = v;
        }
        vc[r] = v;
      }
      if (tid == 0) {
        e[j] = ej;
        tau[j] = tj;
      }
      tau_prev = tj;
    }
    __syncthreads();
    // ---- phase 2 (all): A22 -= update_{j-1}; partial sums of p = A22 v_j
    {
      T vo[NS], uo[NS], vn[NS], acc[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const int i = lane + 32 * s, r = j + 1 + i;
        vo[s] = zero<T>();
        uo[s] = zero<T>();
        vn[s] = zero<T>();
        acc[s] = zero<T>();
        if (i < m) {
          vo[s] = vp[r];
          uo[s] = wp[r] + mul(al, vo[s]);
          vn[s] = vc[r];
        }
      }
      for (int k0 = warp; k0 < m; k0 += 8 * (TH / 32)) {
        T dp[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          dp[q] = zero<T>();
          const int k = k0 + q * (TH / 32);
          if (k < m) {
            const int c = j + 1 + k;
            const T vok = vp[c];
            const T cvo = cj(vok), cuo = cj(wp[c] + mul(al, vok)), vk = vc[c];
            const int cb = (int)pk(c, c, n) - k;  // + i gives A22(i, k)
#pragma unroll
            for (int s = 0; s < NS; ++s) {
              const int i = lane + 32 * s;
              if (i >= k && i < m) {
                T a = A[cb + i] - (mul(vo[s], cuo) + mul(uo[s], cvo));
                if constexpr (CPLX) {
                  if (i == k) a.y = 0.f;  // Hermitian diagonal stays real
                }
                A[cb + i] = a;
                acc[s] = acc[s] + mul(a, vk);
                if (i > k) dp[q] = dp[q] + cmulc(a, vn[s]);
              }
            }
          }
        }
        int slot;
        const T tot = reduce_scatter8<T>(dp, lane, &slot);
        const int k = k0 + slot * (TH / 32);
        if ((lane & 3) == 0 && k < m) pd[j + 1 + k] = tot;
      }
      T* mine = pw + warp * n;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const int i = lane + 32 * s;
        if (i < m) mine[j + 1 + i] = acc[s];
      }
    }
    __syncthreads();
    // ---- phase 3 (all): w = tau p, partials of w^H v
    {
      T dpart = zero<T>();
      if (tid < m) {
        const int r = j + 1 + tid;
        T pv = pd[r];
#pragma unroll 4
        for (int w = 0; w < (TH / 32); ++w) pv = pv + pw[w * n + r];
        const T wv = mul(tj, pv);
        wc[r] = wv;
        dpart = cmulc(wv, vc[r]);
      }
      dpart = warp_sum(dpart);
      if (lane == 0) s_red[warp] = dpart;
    }
    __syncthreads();
  }
  if (tid == 0) {
    if (n == 1) {
      d[0] = re(A[0]);
      e[0] = 0.f;
    } else {
      // the last diagonal entry takes the update of step n-2
      T dot = zero<T>();
      for (int w = 0; w < (TH / 32); ++w) dot = dot + s_red[w];
      const T al = mul(tau[n - 2], dot) * -0.5f;
      const int c = (n - 2) & 1;
      const T v = vb[c * n + n - 1];
      const T u = wb[c * n + n - 1] + mul(al, v);
      const T a = A[pk(n - 1, n - 1, n)] - (mul(v, cj(u)) + mul(u, cj(v)));
      d[n - 1] = re(a);
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Sturm counts and multisection
// ---------------------------------------------------------------------------
__device__ __forceinline__ int sturm_count(const float* d, const float* e2, int n, float x, float pivmin) {
  float q = d[0] - x;
  if (fabsf(q) < pivmin) q = -pivmin;
  int c = q < 0.f;
  for (int i = 1; i < n; ++i) {
    q = (d[i] - x) - e2[i - 1] / q;
    if (fabsf(q) < pivmin) q = -pivmin;
    c += q < 0.f;
  }
  return c;
}

// k-th smallest eigenvalue (0-based) of the tridiagonal; called by a whole warp.
__device__ float warp_kth(const float* d, const float* e2, int n, int k, float lo, float hi, float pivmin,
                          float abstol) {
  const int lane = threadIdx.x & 31;
  for (int it = 0; it < 10; ++it) {
    const float width = hi - lo;
    const float tol = fmaxf(2.f * FLT_EPSILON * fmaxf(fabsf(lo), fabsf(hi)), abstol);
    if (!(width > tol)) break;
    const float x = lo + width * ((float)(lane + 1) * (1.f / 33.f));
    const int c = sturm_count(d, e2, n, x, pivmin);
    const float clo = (c <= k) ? x : lo;
    const float chi = (c > k) ? x : hi;
    lo = warp_max(clo);
    hi = warp_min(chi);
    if (hi < lo) hi = lo;
  }
  return 0.5f * (lo + hi);
}

struct TriInfo {
  float gl, gu, pivmin, abstol, tnorm;
};

// Eigenvalues at indices idx[0..cnt) into out[]. A few: a warp each, by
// 33-way multisection. Many (whole spectra): a thread each, by bisection with
// the same stopping rule (the Sturm counts of all eigenvalues then run side by
// side instead of 32 points of one eigenvalue per round).
template <int TH>
__device__ void cta_eigs(const float* d, const float* e2, int n, const TriInfo& ti, const int* idx,
                         float* out, int cnt) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (cnt > 2 * (TH / 32)) {
    for (int q = threadIdx.x; q < cnt; q += TH) {
      const int k = idx[q];
      float lo = ti.gl, hi = ti.gu;
      for (int it = 0; it < 64; ++it) {
        const float tol = fmaxf(2.f * FLT_EPSILON * fmaxf(fabsf(lo), fabsf(hi)), ti.abstol);
        if (!(hi - lo > tol)) break;
        const float x = 0.5f * (lo + hi);
        if (sturm_count(d, e2, n, x, ti.pivmin) <= k) lo = x;
        else hi = x;
      }
      out[q] = 0.5f * (lo + hi);
    }
  } else {
    for (int q = warp; q < cnt; q += (TH / 32)) {
      const float v = warp_kth(d, e2, n, idx[q], ti.gl, ti.gu, ti.pivmin, ti.abstol);
      if (lane == 0) out[q] = v;
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Largest eigenvalue of a real symmetric packed matrix: the noise level of a
// NORDIC Monte-Carlo draw (space_time/lowrank.py:222-232 averages the top
// singular value of each Gaussian draw). Lanczos with full re-orthogonalisation
// (two classical Gram-Schmidt passes per step) from a fixed start vector, then
// multisection on the Lanczos tridiagonal. On the Gram of a tall Gaussian
// matrix with 200 columns, 48 steps bring the top Ritz value to 1e-13
// (relative) of the top eigenvalue in exact arithmetic, so the FP32 result
// is limited by rounding alone. The matrix is scaled so that
// its largest diagonal entry is 1, hence its top eigenvalue is >= 1.
// ---------------------------------------------------------------------------
constexpr int LANCZOS_STEPS = 48;

// Q: (min(n, LANCZOS_STEPS) + 1) * n floats of scratch; al, be, be2: n floats each.
// FULL = false: A is packed lower (ld unused); true: a full row-major square
// with leading dimension ld (odd, so a thread per row reads conflict-free).
template <bool FULL, int TH>
__device__ float lanczos_top1(const float* A, int n, int ld, float* Q, float* al, float* be, float* be2) {
  __shared__ float s_coef[LANCZOS_STEPS];
  __shared__ float s_val;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int kmax = n < LANCZOS_STEPS ? n : LANCZOS_STEPS;
  float* wv = Q + (int64_t)kmax * n;
  float part = 0.f;
  for (int i = tid; i < n; i += TH) {
    uint32_t h = (uint32_t)(i + 7) * 2654435761u;
    h ^= h >> 13;
    h *= 0x5bd1e995u;
    h ^= h >> 15;
    const float x = 1.0f + (float)(h & 0xffff) * (1.f / 65536.f);
    Q[i] = x;
    part += x * x;
  }
  const float nr = rsqrtf(bsum_f(part));
  for (int i = tid; i < n; i += TH) Q[i] *= nr;
  __syncthreads();
  int kk = kmax;
  for (int j = 0; j < kmax; ++j) {
    const float* qj = Q + (int64_t)j * n;
    if constexpr (FULL) {
      // w = A q_j: a thread per row
      for (int r = tid; r < n; r += TH) {
        const float* row = A + (int64_t)r * ld;
        float s0 = 0.f, s1 = 0.f;
        int k = 0;
        for (; k + 1 < n; k += 2) {
          s0 += row[k] * qj[k];
          s1 += row[k + 1] * qj[k + 1];
        }
        if (k < n) s0 += row[k] * qj[k];
        wv[r] = s0 + s1;
      }
    } else {
      // w = A q_j: a warp per row, lanes over the columns
      for (int r = warp; r < n; r += (TH / 32)) {
        float s = 0.f;
        for (int k = lane; k < n; k += 32) s += A[k <= r ? pk(r, k, n) : pk(k, r, n)] * qj[k];
        s = warp_sum(s);
        if (lane == 0) wv[r] = s;
      }
    }
    __syncthreads();
    float b2p = 0.f;
    for (int pass = 0; pass < 2; ++pass) {
      for (int c = warp; c <= j; c += (TH / 32)) {
        const float* qc = Q + (int64_t)c * n;
        float s = 0.f;
        for (int i = lane; i < n; i += 32) s += qc[i] * wv[i];
        s = warp_sum(s);
        if (lane == 0) s_coef[c] = s;
      }
      __syncthreads();
      if (pass == 0 && tid == 0) al[j] = s_coef[j];
      b2p = 0.f;
      for (int i = tid; i < n; i += TH) {
        float s = wv[i];
#pragma unroll 8
        for (int c = 0; c <= j; ++c) s -= s_coef[c] * Q[(int64_t)c * n + i];
        wv[i] = s;
        b2p += s * s;
      }
      __syncthreads();
    }
    const float b2 = bsum_f(b2p);
    if (tid == 0) {
      be2[j] = b2;
      be[j] = sqrtf(b2);
    }
    if (j + 1 >= kmax || !(b2 > 1e-12f)) {
      kk = j + 1;
      break;
    }
    const float inv = rsqrtf(b2);
    float* qn = Q + (int64_t)(j + 1) * n;
    for (int i = tid; i < n; i += TH) qn[i] = wv[i] * inv;
    __syncthreads();
  }
  __syncthreads();
  // top eigenvalue of the kk x kk Lanczos tridiagonal (al, be)
  if (warp == 0) {
    float lo = FLT_MAX, hi = -FLT_MAX, emax = 0.f, tn = 0.f;
    for (int i = lane; i < kk; i += 32) {
      const float el = i > 0 ? be[i - 1] : 0.f, er = i < kk - 1 ? be[i] : 0.f;
      lo = fminf(lo, al[i] - el - er);
      hi = fmaxf(hi, al[i] + el + er);
      emax = fmaxf(emax, er * er);
      tn = fmaxf(tn, fabsf(al[i]) + el + er);
    }
    lo = -warp_max(-lo);
    hi = warp_max(hi);
    emax = warp_max(emax);
    tn = warp_max(tn);
    const float pv = FLT_MIN * fmaxf(1.f, emax);
    const float v = warp_kth(al, be2, kk, kk - 1, lo - 2.f * FLT_EPSILON * tn - pv, hi + 2.f * FLT_EPSILON * tn + pv,
                             pv, 0.5f * FLT_EPSILON * tn);
    if (lane == 0) s_val = v;
  }
  __syncthreads();
  return s_val;
}

// ---------------------------------------------------------------------------
// Reference shrinkers (space_time/lowrank.py:250-280), FP64, NaN -> 0 applied
// by the caller as at :398.
// ---------------------------------------------------------------------------
__device__ double opt_loss_x(double y, double beta) {
  const double t = y * y - beta - 1.0;
  const double v = sqrt(0.5 * (t + sqrt(t * t - 4.0 * beta)));
  return v * ((y >= 1.0 + sqrt(beta)) ? 1.0 : 0.0);
}
__device__ double shrink(int loss, double y, double beta) {
  if (loss == PD_LOSS_OPE) {
    const double x = opt_loss_x(y, beta);
    return isnan(x) ? x : fmax(x, 0.0);
  }
  if (loss == PD_LOSS_NUC) {
    const double x = opt_loss_x(y, beta);
    const double num = x * x * x * x - sqrt(beta) * x * y - beta;
    const double top = isnan(num) ? num : fmax(0.0, num);
    return top / (x * x * y);
  }
  const double t = (y * y - beta - 1.0);
  const double q = t * t - 4.0 * beta;
  return sqrt(fmax(q, 0.0) / y);
}

// ---------------------------------------------------------------------------
// Adaptive trace-norm shrinkage (AdaptiveDenoiser, space_time/lowrank.py:410-636)
// ---------------------------------------------------------------------------
// Singular values s (descending), their logs, and si_i = sum_{j != i} 1 / (s_i^2 - s_j^2).
struct AdSpec {
  const double* s;
  const double* ls;
  const double* si;
  int nv;
  double M, T, sigma;
  bool gsure;
};

// numpy.maximum(x, 0): NaN propagates
__device__ __forceinline__ double np_max0(double x) { return x != x ? x : (x > 0.0 ? x : 0.0); }

// _sure_atn_cost (lowrank.py:410-447) at log tau = lt and gamma, in FP64; one
// warp, every lane returns the same value. d_i = s_i max(1 - (tau/s_i)^gamma, 0);
// div = sum_i [1 + (gamma-1)(tau/s_i)^gamma](s_i >= tau) + |M - T| d_i / s_i
// + 2 sum_ij D_ij with D_ij = s_i d_i / (s_i^2 - s_j^2) off the diagonal, so
// sum_ij D_ij = sum_i s_i d_i si_i; rss = sum_i (d_i - s_i)^2.
// SURE: sigma^2 (2 div - M T) + rss; GSURE: rss / (1 - div / (M T))^2.
__device__ double ad_cost(const AdSpec& c, double lt, double gamma) {
  const int lane = threadIdx.x & 31;
  const double tau = exp(lt);
  double dv = 0.0, sd = 0.0, rss = 0.0;
  for (int k = lane; k < c.nv; k += 32) {
    const double s = c.s[k];
    // a zero singular value (a rank-deficient patch, M <= T) adds nothing: in
    // the limit s -> 0 its d, indicator and d / s terms all vanish, as they do
    // for the tiny value the reference's SVD returns there
    if (!(s > 0.0)) continue;
    const double r = exp(gamma * (lt - c.ls[k]));  // (tau / s)^gamma
    const double dh = s * np_max0(1.0 - r);
    dv += (1.0 + (gamma - 1.0) * r) * (s >= tau ? 1.0 : 0.0) + fabs(c.M - c.T) * dh / s;
    sd += s * dh * c.si[k];
    rss += (dh - s) * (dh - s);
  }
  dv = warp_sum(dv);
  sd = warp_sum(sd);
  rss = warp_sum(rss);
  const double div = dv + 2.0 * sd;
  if (c.gsure) {
    const double q = 1.0 - div / c.M / c.T;
    return rss / (q * q);
  }
  return c.sigma * c.sigma * (2.0 * div - c.M * c.T) + rss;
}

// Brent's minimisation on [a, b] (golden section with parabolic steps;
// R. P. Brent, Algorithms for Minimization without Derivatives, 1973, ch. 5),
// relative tolerance tol. f must return the same value on every lane.
template <class F>
__device__ double brent_min(const F& f, double a, double b, double tol) {
  const double cg = 0.3819660112501051;  // (3 - sqrt 5) / 2
  double x = a + cg * (b - a), w = x, v = x;
  double fx = f(x), fw = fx, fv = fx;
  double d = 0.0, e = 0.0;
  for (int it = 0; it < 200; ++it) {
    const double m = 0.5 * (a + b);
    const double tol1 = tol * fabs(x) + 1e-12, tol2 = 2.0 * tol1;
    if (fabs(x - m) <= tol2 - 0.5 * (b - a)) break;
    bool golden = true;
    if (fabs(e) > tol1) {
      const double r = (x - w) * (fx - fv);
      double q = (x - v) * (fx - fw);
      double pp = (x - v) * q - (x - w) * r;
      q = 2.0 * (q - r);
      if (q > 0.0) pp = -pp;
      else q = -q;
      const double e_old = e;
      e = d;
      if (fabs(pp) < fabs(0.5 * q * e_old) && pp > q * (a - x) && pp < q * (b - x)) {
        d = pp / q;
        const double u = x + d;
        if (u - a < tol2 || b - u < tol2) d = x < m ? tol1 : -tol1;
        golden = false;
      }
    }
    if (golden) {
      e = x < m ? b - x : a - x;
      d = cg * e;
    }
    const double u = fabs(d) >= tol1 ? x + d : x + (d > 0.0 ? tol1 : -tol1);
    const double fu = f(u);
    if (fu <= fx) {
      if (u < x) b = x;
      else a = x;
      v = w;
      fv = fw;
      w = x;
      fw = fx;
      x = u;
      fx = fu;
    } else {
      if (u < x) a = u;
      else b = u;
      if (fu <= fw || w == x) {
        v = w;
        fv = fw;
        w = u;
        fw = fu;
      } else if (fu <= fv || v == x || v == w) {
        v = u;
        fv = fu;
      }
    }
  }
  return x;
}

// The local minimum of f on [xlo, xhi] that scipy.optimize.minimize (BFGS,
// forward-difference gradient with step 1.49e-8) heads for from x0: the first
// line-search trial point of BFGS is x0 - g min(1, 1.01 / |g|) with g the slope
// at x0; from there the step grows by the golden ratio while the cost keeps
// falling, and Brent's method refines the minimum inside the bracket. The
// bounds keep the search where the cost is numerically meaningful.
template <class F>
__device__ double ad_minimize(const F& f, double x0, double xlo, double xhi) {
  x0 = fmin(fmax(x0, xlo), xhi);
  const double fa0 = f(x0);
  const double g = (f(x0 + 1.4901161193847656e-08) - fa0) / 1.4901161193847656e-08;
  if (!(fabs(g) > 0.0)) return x0;  // flat or NaN
  double a = x0, fa = fa0;
  double b = fmin(fmax(x0 - g * fmin(1.0, 1.01 / fabs(g)), xlo), xhi);
  if (b == a) return x0;
  double fb = f(b);
  double lo, hi;
  if (fb < fa) {
    double c = fmin(fmax(b + 1.618033988749895 * (b - a), xlo), xhi), fc = f(c);
    for (int it = 0; it < 60 && fc < fb && c != b && xlo < c && c < xhi; ++it) {
      a = b;
      fa = fb;
      b = c;
      fb = fc;
      c = fmin(fmax(b + 1.618033988749895 * (b - a), xlo), xhi);
      fc = f(c);
    }
    lo = fmin(a, c);
    hi = fmax(a, c);
  } else {
    lo = fmin(a, b);
    hi = fmax(a, b);
  }
  return brent_min(f, lo, hi, 1e-10);
}

// The adaptive rule for one patch (the caller's whole CTA): the full spectrum,
// the (G)SURE minimisation and the shrinkage coefficients. Compiled only into
// k_eig's ADAPT instantiation, so that its FP64 search leaves the other
// methods' kernels as they are. scratch: 3 n doubles of shared memory.
template <int TH>
__device__ __forceinline__ void adaptive_rule(const EigParams& ep, const pd_adaptive& ad, const PatchWork& w, int p,
                                              int n, const float* d,
                                           const float* e2, const TriInfo& ti, int* idx, float* lam, int* aidx,
                                           float* alam, float* acoef, double* scratch, double tscale, double M,
                                           double pt, int* s_act) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (ad.mode == PD_ADAPTIVE_QUT && ad.n_gamma >= 1) {
    // QUT with a fixed gamma: tau = stdest * level is known (lowrank.py:464-475)
    // and d = s max(1 - (tau / s)^gamma, 0) (lowrank.py:459-461) is nonzero
    // exactly for s > tau, a prefix of the descending spectrum: only those
    // eigenvalues are needed (candidates by a Sturm count, as the raw rule)
    __shared__ int s_c0q;
    const double tau = sqrt(w.prior[p]) * ad.qut_level;
    if (tid == 0) s_c0q = sturm_count(d, e2, n, (float)(tau * tau / tscale * (1.0 - CAND_MARGIN)), ti.pivmin);
    __syncthreads();
    const int nc = n - s_c0q;
    for (int i = tid; i < nc; i += TH) idx[i] = s_c0q + i;
    __syncthreads();
    cta_eigs<TH>(d, e2, n, ti, idx, lam, nc);
    if (tid == 0) {
      const double gq = ad.gamma[0], lt = log(tau);
      int r = 0;
      for (int i = nc - 1; i >= 0; --i) {
        const double sv = sqrt(fmax((double)lam[i] * tscale, 0.0));
        if (!(sv > 0.0)) break;
        const double dh = sv * np_max0(1.0 - exp(gq * (lt - log(sv))));
        if (dh == 0.0) break;
        aidx[r] = idx[i];
        alam[r] = lam[i];
        acoef[r] = (float)(dh / sv);
        ++r;
      }
      w.rank[p] = r;
      w.noise[p] = nanf("");
      *s_act = r;
    }
    __syncthreads();
    return;
  }
  // the whole spectrum: singular values s = sqrt(eigenvalue) in numpy.svd's
  // (descending) order, min(M, n) of them
  for (int i = tid; i < n; i += TH) idx[i] = i;
  __syncthreads();
  cta_eigs<TH>(d, e2, n, ti, idx, lam, n);
  const int nv = ep.rows < n ? ep.rows : n;
  double* sv = scratch;
  double* lsv = sv + n;
  double* si = lsv + n;
  // a centred M x T patch with M <= T has rank M - 1 at most: its singular
  // values from index M - 1 on are zero (the Gram's rounding leaves them small)
  const int nz = ep.rows <= n ? ep.rows - 1 : nv;
  for (int k = tid; k < nv; k += TH) {
    sv[k] = k < nz ? sqrt(fmax((double)lam[n - 1 - k] * tscale, 0.0)) : 0.0;
    lsv[k] = log(sv[k]);
  }
  __syncthreads();
  for (int k = tid; k < nv; k += TH) {
    const double a2 = sv[k] * sv[k];
    double acc = 0.0;
    if (a2 > 0.0)  // zero singular values are skipped by the cost (their si is unused)
      for (int q = 0; q < nv; ++q)
        if (q != k) acc += 1.0 / (a2 - sv[q] * sv[q]);
    si[k] = acc;
  }
  __shared__ int s_npos;  // positive singular values (descending, so a prefix)
  if (tid == 0) {
    int np_ = 0;
    while (np_ < nv && sv[np_] > 0.0) ++np_;
    s_npos = np_;
  }
  __syncthreads();
  __shared__ double s_cost[PD_ADAPTIVE_MAX_GAMMA], s_x[PD_ADAPTIVE_MAX_GAMMA];
  __shared__ double s_gamma, s_lt;
  const AdSpec c{sv, lsv, si, nv, M, pt, sqrt(w.prior[p]), ad.mode == PD_ADAPTIVE_GSURE};
  if (ad.mode == PD_ADAPTIVE_QUT) {
    // tau = stdest * level (lowrank.py:464-475); gamma fixed, or exp(x) + 1 with
    // x minimising the cost from 0 (lowrank.py:477-492)
    const double lt = log(c.sigma * ad.qut_level);
    if (warp == 0) {
      double gq = ad.n_gamma >= 1 ? ad.gamma[0] : 0.0;
      if (ad.n_gamma < 1)
        gq = exp(ad_minimize([&](double x) { return ad_cost(c, lt, exp(x) + 1.0); }, 0.0, -700.0, 700.0)) + 1.0;
      if (lane == 0) {
        s_gamma = gq;
        s_lt = lt;
      }
    }
  } else {
    // every candidate gamma: log tau from log(median s) (or tau0) by the search,
    // the lowest cost wins, the first on ties (lowrank.py:497-533); a warp per
    // candidate. log tau stays within 10 of the log spectrum: far below the
    // smallest singular value every d equals s to rounding and the GSURE cost
    // is 0/0 (rss and 1 - div/(M T) both vanish with gamma = 1).
    const int npos = s_npos > 0 ? s_npos : 1;
    const double xlo = lsv[npos - 1] - 10.0, xhi = lsv[0] + 10.0;
    double x0 = ad.tau0;
    if (!ad.has_tau0) {
      const double med = (nv & 1) ? sv[nv / 2] : 0.5 * (sv[nv / 2 - 1] + sv[nv / 2]);
      x0 = med > 0.0 ? log(med) : xlo;  // a median of zeros: start at the smallest positive value
    }
    for (int q = warp; q < ad.n_gamma; q += (TH / 32)) {
      const double gq = ad.gamma[q];
      const double x = ad_minimize([&](double xx) { return ad_cost(c, xx, gq); }, x0, xlo, xhi);
      const double cost = ad_cost(c, x, gq);
      if (lane == 0) {
        s_cost[q] = cost;
        s_x[q] = x;
      }
    }
    __syncthreads();
    if (tid == 0) {
      int bq = 0;  // no finite cost at all (the reference fails there): the first candidate
      double best = INFINITY;
      for (int q = 0; q < ad.n_gamma; ++q)
        if (s_cost[q] < best) {
          best = s_cost[q];
          bq = q;
        }
      s_gamma = ad.gamma[bq];
      s_lt = s_x[bq];
    }
  }
  __syncthreads();
  if (tid == 0) {
    // _atn_shrink (lowrank.py:459-461); maxidx = last nonzero + 1 (lowrank.py:628-635)
    const double gq = s_gamma, lt = s_lt;
    int maxidx = 0;
    for (int k = 0; k < nv; ++k) {
      const double dh = sv[k] * np_max0(1.0 - exp(gq * (lt - lsv[k])));
      if (dh != 0.0) maxidx = k + 1;  // NaN counts as nonzero, as in numpy
      acoef[k] = sv[k] > 0.0 ? (float)(dh / sv[k]) : 0.f;
    }
    for (int k = 0; k < maxidx; ++k) {
      aidx[k] = n - 1 - k;
      alam[k] = lam[n - 1 - k];
    }
    w.rank[p] = maxidx;
    w.noise[p] = nanf("");
    *s_act = maxidx;
  }
  __syncthreads();}

// ---------------------------------------------------------------------------
// The kernel
// ---------------------------------------------------------------------------
template <bool CPLX, int NS, bool ADAPT, int TH>
// ADAPT: with the adaptive rule (PD_METHOD_ADAPTIVE launches only).
// in_smem: bit 0 = the packed matrix lives in shared memory, bit 1 = the
// Lanczos basis of the top-1 mode does too (after the layout's end).
__global__ void __launch_bounds__(TH, TH >= 512 ? 1 : 4) k_eig(int n, EigParams ep, PatchWork w, int in_smem,
                                                       pd_adaptive ad) {
  using T = typename Elem<CPLX>::T;
  extern __shared__ __align__(16) unsigned char sm[];
  const int p = blockIdx.x;
  if (w.vols) {
    // batched call: this patch's volume sets the frames and the rule's
    // parameters; the packed matrix goes to shared memory when it fits the
    // launch's allocation (sized for the batch's largest patch)
    const VolDesc& v = w.vols[w.vol_of[p]];
    n = v.g.cols;
    ep.rows = v.g.rows;
    ep.cols = n;
    ep.threshold = v.threshold;
    ep.mp_median = v.mp_median;
    uint32_t dyn;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
    in_smem = eig_layout(CPLX, n, true, TH).total <= dyn ? 1 : 0;
  }
  const EigLayout L = eig_layout(CPLX, n, (in_smem & 1) != 0, TH);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (ep.only_unfinished && w.n_active[p] >= 0) return;  // solved by k_sub
  T* G = reinterpret_cast<T*>(w.gram + (int64_t)p * w.gram_stride);
  T* A = (in_smem & 1) ? reinterpret_cast<T*>(sm + L.a) : G;
  float* d = reinterpret_cast<float*>(sm + L.d);
  float* e = reinterpret_cast<float*>(sm + L.e);
  float* e2 = reinterpret_cast<float*>(sm + L.e2);
  T* tau = reinterpret_cast<T*>(sm + L.tau);
  T* vb = reinterpret_cast<T*>(sm + L.vb);
  T* wb = reinterpret_cast<T*>(sm + L.wb);
  T* pw = reinterpret_cast<T*>(sm + L.pw);
  T* pd = reinterpret_cast<T*>(sm + L.pd);
  int* idx = reinterpret_cast<int*>(sm + L.idx);
  float* lam = reinterpret_cast<float*>(sm + L.lam);
  int* aidx = reinterpret_cast<int*>(sm + L.aidx);
  float* alam = reinterpret_cast<float*>(sm + L.alam);
  float* acoef = reinterpret_cast<float*>(sm + L.acoef);
  __shared__ int s_cnt, s_act, s_c0, s_c1;
  __shared__ double s_scale_true;  // 1/sc: true eigenvalue = scaled * this
  __shared__ double s_x0;
  __shared__ double s_thr;  // raw / NORDIC threshold on singular values

  const int64_t np = pk_size(n);
  if (in_smem & 1) {
    for (int64_t i = tid; i < np; i += TH) A[i] = G[i];
    __syncthreads();
  }
  // scale by 1 / max diagonal
  float md = 0.f;
  for (int i = tid; i < n; i += TH) md = fmaxf(md, re(A[pk(i, i, n)]));
  md = bmax_f(md);
  const float sc = md > 0.f ? 1.f / md : 1.f;
  if (tid == 0) s_scale_true = md > 0.f ? (double)md : 1.0;
  __syncthreads();
  for (int64_t i = tid; i < np; i += TH) A[i] = A[i] * sc;
  __syncthreads();

  if constexpr (!CPLX) {
    if (ep.method == EIG_MODE_TOP1) {  // Monte-Carlo level: top eigenvalue only
      float* Q = (in_smem & 2) ? reinterpret_cast<float*>(sm + L.total) : w.vec + (int64_t)p * w.vec_stride;
      const float lam1 = lanczos_top1<false, TH>(A, n, 0, Q, d, e, e2);
      if (tid == 0) {
        w.prior[p] = (double)lam1 * s_scale_true;
        w.n_active[p] = 0;
      }
      return;
    }
  }
  tridiagonalize<CPLX, NS, TH>(A, n, d, e, tau, vb, wb, pw, pd);

  // e2, Gershgorin bounds, tolerances
  float glo = FLT_MAX, ghi = -FLT_MAX, emax = 0.f, tn = 0.f;
  for (int i = tid; i < n; i += TH) {
    const float el = i > 0 ? fabsf(e[i - 1]) : 0.f;
    const float er = i < n - 1 ? fabsf(e[i]) : 0.f;
    if (i < n - 1) e2[i] = e[i] * e[i];
    glo = fminf(glo, d[i] - el - er);
    ghi = fmaxf(ghi, d[i] + el + er);
    emax = fmaxf(emax, er * er);
    tn = fmaxf(tn, fabsf(d[i]) + el + er);
  }
  glo = -bmax_f(-glo);
  ghi = bmax_f(ghi);
  emax = bmax_f(emax);
  tn = bmax_f(tn);
  TriInfo ti;
  ti.tnorm = tn;
  ti.pivmin = FLT_MIN * fmaxf(1.f, emax);
  ti.abstol = 0.5f * FLT_EPSILON * tn;
  ti.gl = glo - 2.f * FLT_EPSILON * tn - ti.pivmin;
  ti.gu = ghi + 2.f * FLT_EPSILON * tn + ti.pivmin;
  __syncthreads();

  const double tscale = s_scale_true;  // true = scaled * tscale
  const double M = (double)ep.rows, pt = (double)ep.cols;

  // ---------------------------------------------------------------- decisions
  if (ADAPT && ep.method == EIG_MODE_FULL) {  // the whole decomposition (ADAPT instantiation)
    for (int i = tid; i < n; i += TH) idx[i] = i;
    __syncthreads();
    cta_eigs<TH>(d, e2, n, ti, idx, lam, n);
    for (int a = tid; a < n; a += TH) {
      aidx[a] = n - 1 - a;
      alam[a] = lam[n - 1 - a];
      acoef[a] = (float)((double)lam[n - 1 - a] * tscale);
    }
    if (tid == 0) s_act = n;
    __syncthreads();
  } else if (ADAPT && ep.method == PD_METHOD_ADAPTIVE) {  // compiled into the ADAPT instantiation only
    adaptive_rule<TH>(ep, ad, w, p, n, d, e2, ti, idx, lam, aidx, alam, acoef, reinterpret_cast<double*>(pw), tscale, M,
                  pt, &s_act);
  } else if (ep.method == PD_METHOD_MPPCA || ep.method == PD_METHOD_HYBRID) {
    const int ne = n < 10 ? n : 10;
    if (tid < ne) idx[tid] = n - ne + tid;
    __syncthreads();
    cta_eigs<TH>(d, e2, n, ti, idx, lam, ne);
    if (tid == 0) {
      int k;
      double var;
      mp_hybrid_rule(ep.method == PD_METHOD_MPPCA, ep.threshold_scale, ep.method == PD_METHOD_HYBRID ? w.prior[p] : 0.0,
                     lam, ne, tscale, M, pt, &k, &var);
      w.rank[p] = k;
      w.noise[p] = (float)var;
      const int act = k < ne ? k : ne;
      for (int a = 0; a < act; ++a) {
        aidx[a] = n - 1 - a;  // descending eigenvalue order
        alam[a] = lam[ne - 1 - a];
        acoef[a] = 1.f;
      }
      s_act = act;
    }
    __syncthreads();
  } else if (ep.method == PD_METHOD_RAW) {
    if (tid == 0) {
      s_thr = ep.d_threshold ? *ep.d_threshold : ep.threshold;
      const double x = s_thr * s_thr / tscale;  // scaled threshold on eigenvalues
      s_c0 = sturm_count(d, e2, n, (float)(x * (1.0 - CAND_MARGIN)), ti.pivmin);
    }
    __syncthreads();
    const int nc = n - s_c0;
    for (int i = tid; i < nc; i += TH) idx[i] = s_c0 + i;
    __syncthreads();
    cta_eigs<TH>(d, e2, n, ti, idx, lam, nc);
    if (tid == 0) {
      int r = 0;
      for (int i = nc - 1; i >= 0; --i) {
        const double s = sqrt(fmax((double)lam[i] * tscale, 0.0));
        if (s > s_thr) {
          aidx[r] = idx[i];
          alam[r] = lam[i];
          acoef[r] = 1.f;
          ++r;
        }
      }
      w.rank[p] = r;
      w.noise[p] = nanf("");
      s_act = r;
    }
    __syncthreads();
  } else {  // PD_METHOD_OPTIMAL
    if (tid == 0) {
      if (n & 1) {
        idx[0] = (n - 1) / 2;
        s_cnt = 1;
      } else {
        idx[0] = n / 2 - 1;
        idx[1] = n / 2;
        s_cnt = 2;
      }
    }
    __syncthreads();
    cta_eigs<TH>(d, e2, n, ti, idx, lam, s_cnt);
    if (tid == 0) {
      double smed;
      if (n & 1)
        smed = sqrt(fmax((double)lam[0] * tscale, 0.0));
      else
        smed = 0.5 * (sqrt(fmax((double)lam[0] * tscale, 0.0)) + sqrt(fmax((double)lam[1] * tscale, 0.0)));
      const double sigma = ep.has_prior ? w.prior[p] : smed / sqrt(pt * ep.mp_median);
      const double scale = sqrt(pt) * sigma;
      const double beta = pt / M;
      s_x0 = scale;
      const double hi = scale * (1.0 + sqrt(beta));
      const double lo = scale * (1.0 - sqrt(beta));
      s_c0 = n - sturm_count(d, e2, n, (float)(hi * hi / tscale * (1.0 - CAND_MARGIN)), ti.pivmin);
      int nb = 0;
      if (ep.loss == PD_LOSS_FRO && lo > 0.0)
        nb = sturm_count(d, e2, n, (float)(lo * lo / tscale * (1.0 + CAND_MARGIN)), ti.pivmin);
      if (nb > n - s_c0) nb = n - s_c0;
      s_c1 = nb;
    }
    __syncthreads();
    const int ntop = s_c0, nbot = s_c1;
    for (int i = tid; i < nbot; i += TH) idx[i] = i;
    for (int i = tid; i < ntop; i += TH) idx[nbot + i] = n - ntop + i;
    __syncthreads();
    cta_eigs<TH>(d, e2, n, ti, idx, lam, nbot + ntop);
    if (tid == 0) {
      const double scale = s_x0;
      const double beta = pt / M;
      int act = 0, maxidx = 0;
      for (int q = nbot + ntop - 1; q >= 0; --q) {  // descending eigenvalue order
        const double s = sqrt(fmax((double)lam[q] * tscale, 0.0));
        double sh = scale * shrink(ep.loss, s / scale, beta);
        if (isnan(sh)) sh = 0.0;
        if (sh != 0.0) {
          aidx[act] = idx[q];
          alam[act] = lam[q];
          acoef[act] = (float)(sh / s);
          ++act;
          const int desc = n - 1 - idx[q];
          if (desc + 1 > maxidx) maxidx = desc + 1;
        }
      }
      w.rank[p] = maxidx;
      w.noise[p] = nanf("");
      s_act = act;
    }
    __syncthreads();
  }

  // ------------------------------------------------------------ eigenvectors
  const int act = s_act;
  const int n2 = 2 * n;
  float* vbase = w.vec + (int64_t)p * w.vec_stride;
  for (int a = tid; a < act; a += TH) {
    float* z = vbase + (int64_t)a * n2;  // z[0..n): vector (first D-)
    float* Dp = z + n;                   // D+ scratch
    const float lm = alam[a];
    const float pv = ti.pivmin;
    float q = d[0] - lm;
    if (fabsf(q) < pv) q = -pv;
    Dp[0] = q;
    for (int i = 1; i < n; ++i) {
      q = (d[i] - lm) - e2[i - 1] / q;
      if (fabsf(q) < pv) q = -pv;
      Dp[i] = q;
    }
    q = d[n - 1] - lm;
    if (fabsf(q) < pv) q = -pv;
    z[n - 1] = q;
    for (int i = n - 2; i >= 0; --i) {
      q = (d[i] - lm) - e2[i] / q;
      if (fabsf(q) < pv) q = -pv;
      z[i] = q;
    }
    int r = 0;
    float best = FLT_MAX;
    for (int i = 0; i < n; ++i) {
      const float gm = fabsf(Dp[i] + z[i] - (d[i] - lm));
      if (gm < best) {
        best = gm;
        r = i;
      }
    }
    // the running element stays in a register (no reload of what this thread
    // stored one step earlier); z[i] holds D-(i) until it is overwritten
    z[r] = 1.f;
    float s2 = 1.f, zv = 1.f;
    for (int i = r + 1; i < n; ++i) {
      zv = -(e[i - 1] / z[i]) * zv;
      z[i] = zv;
      s2 += zv * zv;
    }
    zv = 1.f;
    for (int i = r - 1; i >= 0; --i) {
      zv = -(e[i] / Dp[i]) * zv;
      z[i] = zv;
      s2 += zv * zv;
    }
    const float inv = rsqrtf(s2);
    for (int i = 0; i < n; ++i) z[i] *= inv;
  }
  __syncthreads();

  // re-orthogonalise inside clusters (descending order; rare for the low-rank
  // rules, a whole noise bulk for the adaptive ones)
  {
    const float ortol = 1e-3f * ti.tnorm;
    // norm of za, orthogonalised against [cstart, a); a collapsed vector is
    // replaced by inverse iteration from a pseudo-random start; normalised
    auto finish = [&](float* za, int a, int cstart) {
      float part = 0.f;
      for (int i = tid; i < n; i += TH) part += za[i] * za[i];
      float nr = sqrtf(bsum_f(part));
      if (nr < 0.05f) {
        // collapsed: inverse iteration from a pseudo-random start, orthogonalised
        const float* Dp = za + n;
        for (int it = 0; it < 3; ++it) {
          if (it == 0)
            for (int i = tid; i < n; i += TH) {
              uint32_t h = (uint32_t)(i + 1) * 2654435761u ^ (uint32_t)(a + 7) * 40503u;
              h ^= h >> 13;
              h *= 0x5bd1e995u;
              h ^= h >> 15;
              za[i] = (float)(h & 0xffff) / 65536.f - 0.5f;
            }
          __syncthreads();
          for (int b = cstart; b < a; ++b) {
            const float* zb = vbase + (int64_t)b * n2;
            float pp = 0.f;
            for (int i = tid; i < n; i += TH) pp += za[i] * zb[i];
            const float dt = bsum_f(pp);
            for (int i = tid; i < n; i += TH) za[i] -= dt * zb[i];
            __syncthreads();
          }
          if (tid == 0) {  // solve (T - lam I) x = za with T - lam I = L D L^T
            for (int i = 1; i < n; ++i) za[i] -= (e[i - 1] / Dp[i - 1]) * za[i - 1];
            for (int i = 0; i < n; ++i) za[i] /= Dp[i];
            for (int i = n - 2; i >= 0; --i) za[i] -= (e[i] / Dp[i]) * za[i + 1];
          }
          __syncthreads();
          float pp = 0.f;
          for (int i = tid; i < n; i += TH) pp += za[i] * za[i];
          const float iv = rsqrtf(bsum_f(pp));
          for (int i = tid; i < n; i += TH) za[i] *= iv;
          __syncthreads();
        }
        for (int b = cstart; b < a; ++b) {
          const float* zb = vbase + (int64_t)b * n2;
          float pp = 0.f;
          for (int i = tid; i < n; i += TH) pp += za[i] * zb[i];
          const float dt = bsum_f(pp);
          for (int i = tid; i < n; i += TH) za[i] -= dt * zb[i];
          __syncthreads();
        }
        part = 0.f;
        for (int i = tid; i < n; i += TH) part += za[i] * za[i];
        nr = sqrtf(bsum_f(part));
      }
      const float iv = nr > 0.f ? 1.f / nr : 0.f;
      for (int i = tid; i < n; i += TH) za[i] *= iv;
      __syncthreads();
    };
    if constexpr (ADAPT) {
      // A noise bulk is one cluster of up to n vectors: block classical
      // Gram-Schmidt, twice. RB vectors at a time are staged in shared memory
      // and projected against the earlier vectors of their cluster (each
      // earlier vector is read once per block, a warp per earlier vector for
      // the dot products), then against each other.
      constexpr int RB = 8;
      int* cst = reinterpret_cast<int*>(lam);  // cluster start of each vector (lam is free here)
      float* blk = reinterpret_cast<float*>(pw);  // [RB][n]; pw (>= 16 n floats) is free after the rule
      float* dots = blk + RB * n;                 // [RB][act]
      if (tid == 0) {
        int c0 = 0;
        cst[0] = 0;
        for (int q = 1; q < act; ++q) {
          if (alam[q - 1] - alam[q] > ortol) c0 = q;
          cst[q] = c0;
        }
      }
      __syncthreads();
      for (int a0 = 1; a0 < act; a0 += RB) {
        const int nb = min(RB, act - a0);
        const int lo = cst[a0];
        for (int q = tid; q < nb * n; q += TH) {
          const int k = q / n, i = q - k * n;
          blk[k * n + i] = vbase[(int64_t)(a0 + k) * n2 + i];
        }
        __syncthreads();
        for (int pass = 0; pass < 2 && lo < a0; ++pass) {
          for (int b = lo + warp; b < a0; b += (TH / 32)) {
            const float* zb = vbase + (int64_t)b * n2;
            float dp[RB];
#pragma unroll
            for (int k = 0; k < RB; ++k) dp[k] = 0.f;
            for (int i = lane; i < n; i += 32) {
              const float zv = zb[i];
#pragma unroll
              for (int k = 0; k < RB; ++k)
                if (k < nb) dp[k] += zv * blk[k * n + i];
            }
#pragma unroll
            for (int k = 0; k < RB; ++k) {
              if (k >= nb) break;
              const float t = warp_sum(dp[k]);
              if (lane == 0) dots[k * act + b] = b >= cst[a0 + k] ? t : 0.f;
            }
          }
          __syncthreads();
          for (int i = tid; i < n; i += TH) {
            float acc[RB];
#pragma unroll
            for (int k = 0; k < RB; ++k) acc[k] = 0.f;
            for (int b = lo; b < a0; ++b) {
              const float zv = vbase[(int64_t)b * n2 + i];
#pragma unroll
              for (int k = 0; k < RB; ++k) acc[k] += dots[k * act + b] * zv;
            }
#pragma unroll
            for (int k = 0; k < RB; ++k)
              if (k < nb) blk[k * n + i] -= acc[k];
          }
          __syncthreads();
        }
        // within the block, in order; each vector is final (and back in
        // global memory) before the next one is projected against it
        for (int k = 0; k < nb; ++k) {
          const int a = a0 + k;
          float* za = vbase + (int64_t)a * n2;
          if (cst[a] == a) {  // starts a cluster: nothing to project out
            __syncthreads();
            continue;
          }
          const int j0 = max(cst[a], a0) - a0;
          for (int pass = 0; pass < 2 && j0 < k; ++pass) {
            for (int j = j0 + warp; j < k; j += (TH / 32)) {
              float dp = 0.f;
              for (int i = lane; i < n; i += 32) dp += blk[j * n + i] * blk[k * n + i];
              dp = warp_sum(dp);
              if (lane == 0) dots[j] = dp;
            }
            __syncthreads();
            for (int i = tid; i < n; i += TH) {
              float v = blk[k * n + i];
              for (int j = j0; j < k; ++j) v -= dots[j] * blk[j * n + i];
              blk[k * n + i] = v;
            }
            __syncthreads();
          }
          for (int i = tid; i < n; i += TH) za[i] = blk[k * n + i];
          __syncthreads();
          finish(za, a, cst[a]);
          for (int i = tid; i < n; i += TH) blk[k * n + i] = za[i];
          __syncthreads();
        }
      }
    } else {
      int cstart = 0;
      for (int a = 1; a < act; ++a) {
        if (alam[a - 1] - alam[a] > ortol) {
          cstart = a;
          continue;
        }
        float* za = vbase + (int64_t)a * n2;
        for (int b = cstart; b < a; ++b) {
          const float* zb = vbase + (int64_t)b * n2;
          float part = 0.f;
          for (int i = tid; i < n; i += TH) part += za[i] * zb[i];
          const float dt = bsum_f(part);
          for (int i = tid; i < n; i += TH) za[i] -= dt * zb[i];
          __syncthreads();
        }
        finish(za, a, cstart);
      }
    }
  }

  // back-transform: y = H_0 H_1 ... H_{n-2} z. A warp applies each reflector
  // to VG vectors at once: the reflector column is read once for all of them
  // and their VG dot products reduce in parallel (whole spectra: act = n).
  constexpr int VGR = 48 / (NS * (CPLX ? 2 : 1));
  constexpr int VG = VGR < 1 ? 1 : (VGR > 8 ? 8 : VGR);
  for (int g0 = warp * VG; g0 < act; g0 += (TH / 32) * VG) {
    T y[VG][NS];
#pragma unroll
    for (int v = 0; v < VG; ++v) {
      const float* col = vbase + (int64_t)(g0 + v) * n2;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const int i = lane + 32 * s;
        const float zv = (g0 + v < act && i < n) ? col[i] : 0.f;
        if constexpr (CPLX) y[v][s] = cf{zv, 0.f};
        else y[v][s] = zv;
      }
    }
    for (int j = n - 2; j >= 0; --j) {
      const T tj = tau[j];
      if (abs2(tj) == 0.f) continue;
      T hv[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const int i = lane + 32 * s;
        if (i == j + 1) {
          if constexpr (CPLX) hv[s] = cf{1.f, 0.f};
          else hv[s] = 1.f;
        } else {
          hv[s] = (i > j + 1 && i < n) ? A[pk(i, j, n)] : zero<T>();
        }
      }
      T dt[VG];
#pragma unroll
      for (int v = 0; v < VG; ++v) {
        T part = zero<T>();
#pragma unroll
        for (int s = 0; s < NS; ++s) part = part + cmulc(hv[s], y[v][s]);
        dt[v] = part;
      }
#pragma unroll
      for (int v = 0; v < VG; ++v) dt[v] = mul(tj, warp_sum(dt[v]));
#pragma unroll
      for (int v = 0; v < VG; ++v)
#pragma unroll
        for (int s = 0; s < NS; ++s) y[v][s] = y[v][s] - mul(hv[s], dt[v]);
    }
    __syncwarp();
#pragma unroll
    for (int v = 0; v < VG; ++v) {
      if (g0 + v >= act) break;
      float* col = vbase + (int64_t)(g0 + v) * n2;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const int i = lane + 32 * s;
        if (i < n) {
          if constexpr (CPLX) reinterpret_cast<cf*>(col)[i] = y[v][s];
          else col[i] = y[v][s];
        }
      }
    }
  }
  for (int a = tid; a < act; a += TH) w.coef[(int64_t)p * w.n_stride + a] = acoef[a];
  if (tid == 0) w.n_active[p] = act;
}

// Top-1 eigenvalue of each real packed Gram (the NORDIC Monte-Carlo draws),
// the matrix scaled by its largest diagonal entry and expanded to a full square
// with odd leading dimension in shared memory, so the Lanczos product is a
// plain row-times-vector per thread. One CTA per draw.
__host__ __device__ inline int top1_ld(int n) { return n | 1; }
size_t top1_smem_bytes(int n) {
  const int kmax = n < LANCZOS_STEPS ? n : LANCZOS_STEPS;
  return sizeof(float) * ((size_t)n * top1_ld(n) + (size_t)(kmax + 1) * n + 3 * (size_t)n);
}

__global__ void __launch_bounds__(EIG_THREADS, 1) k_top1(int n, PatchWork w) {
  extern __shared__ __align__(16) unsigned char sm[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int p = blockIdx.x;
  const int ld = top1_ld(n);
  const int kmax = n < LANCZOS_STEPS ? n : LANCZOS_STEPS;
  float* F = reinterpret_cast<float*>(sm);
  float* Q = F + (size_t)n * ld;
  float* al = Q + (size_t)(kmax + 1) * n;
  float* be = al + n;
  float* be2 = be + n;
  __shared__ double s_md;
  const float* G = w.gram + (int64_t)p * w.gram_stride;
  float md = 0.f;
  for (int i = tid; i < n; i += EIG_THREADS) md = fmaxf(md, G[pk(i, i, n)]);
  md = bmax_f(md);
  const float sc = md > 0.f ? 1.f / md : 1.f;
  if (tid == 0) s_md = md > 0.f ? (double)md : 1.0;
  for (int j = warp; j < n; j += EIG_NW) {
    const int64_t cb = pk(j, j, n) - j;
    for (int i = j + lane; i < n; i += 32) {
      const float v = G[cb + i] * sc;
      F[(size_t)i * ld + j] = v;
      F[(size_t)j * ld + i] = v;
    }
  }
  __syncthreads();
  const float lam = lanczos_top1<true, EIG_THREADS>(F, n, ld, Q, al, be, be2);
  if (tid == 0) {
    w.prior[p] = (double)lam * s_md;
    w.n_active[p] = 0;
  }
}

// Small patches (n <= 128, so a thread per row of the tridiagonalisation) run
// 128-thread CTAs, four per SM when their layout fits EIG_SMALL_SMEM each: the
// latency-bound steps of four patches overlap instead of one patch's steps
// leaving the SM idle.
constexpr int EIG_SMALL_THREADS = 128;
constexpr size_t EIG_SMALL_SMEM = 227 * 1024 / 4 - 2048;

bool eig_small(bool cplx, int n) {
  return n <= EIG_SMALL_THREADS && eig_layout(cplx, n, true, EIG_SMALL_THREADS).total <= EIG_SMALL_SMEM;
}

size_t eig_launch_smem(bool cplx, int n) {
  if (eig_small(cplx, n)) return eig_layout(cplx, n, true, EIG_SMALL_THREADS).total;
  bool in_smem;
  return eig_smem_bytes(cplx, n, &in_smem);
}

template <bool CPLX, int NS, int TH>
static cudaError_t eig_launch(int n, const EigParams& ep, const PatchWork& w, cudaStream_t s, const pd_adaptive* ad,
                              size_t smem, int flags) {
  auto kern = (ep.method == PD_METHOD_ADAPTIVE || ep.method == EIG_MODE_FULL) ? k_eig<CPLX, NS, true, TH>
                                                                               : k_eig<CPLX, NS, false, TH>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  pd_adaptive a{};
  if (ad) a = *ad;
  PD_TIMED(ep.method == EIG_MODE_TOP1 ? "eig_mc" : "eig", s, kern<<<w.count, TH, smem, s>>>(n, ep, w, flags, a));
  return cudaGetLastError();
}

template <bool CPLX, int NS>
static cudaError_t eig_ns(int n, const EigParams& ep, const PatchWork& w, cudaStream_t s, const pd_adaptive* ad) {
  if constexpr (NS * 32 <= EIG_SMALL_THREADS) {
    const size_t small = eig_layout(CPLX, n, true, EIG_SMALL_THREADS).total;
    if (ep.method != EIG_MODE_TOP1 && eig_small(CPLX, n) && ep.smem_bytes <= EIG_SMALL_SMEM)
      return eig_launch<CPLX, NS, EIG_SMALL_THREADS>(n, ep, w, s, ad, small > ep.smem_bytes ? small : ep.smem_bytes,
                                                     1);
  }
  bool in_smem;
  size_t smem = eig_smem_bytes(CPLX, n, &in_smem);
  if (ep.smem_bytes > smem) smem = ep.smem_bytes;  // a batch whose smaller patches fit shared memory
  int flags = in_smem ? 1 : 0;
  if (!CPLX && ep.method == EIG_MODE_TOP1 && in_smem) {
    const size_t q = al16(sizeof(float) * (size_t)((n < LANCZOS_STEPS ? n : LANCZOS_STEPS) + 1) * n);
    if (smem + q <= EIG_SMEM_LIMIT) {
      smem += q;
      flags |= 2;
    }
  }
  return eig_launch<CPLX, NS, EIG_THREADS>(n, ep, w, s, ad, smem, flags);
}

template <bool CPLX>
static cudaError_t eig_dispatch(int n, const EigParams& ep, const PatchWork& w, cudaStream_t s,
                                const pd_adaptive* ad) {
  if (n <= 64) return eig_ns<CPLX, 2>(n, ep, w, s, ad);
  if (n <= 128) return eig_ns<CPLX, 4>(n, ep, w, s, ad);
  if (n <= 224) return eig_ns<CPLX, 7>(n, ep, w, s, ad);
  if (n <= 320) return eig_ns<CPLX, 10>(n, ep, w, s, ad);
  return eig_ns<CPLX, 14>(n, ep, w, s, ad);
}

cudaError_t launch_eig(bool cplx, int n, const EigParams& ep, const PatchWork& w, cudaStream_t s,
                       const pd_adaptive* ad) {
  if (!cplx && ep.method == EIG_MODE_TOP1) {
    const size_t smem = top1_smem_bytes(n);
    if (smem <= EIG_SMEM_LIMIT) {
      cudaError_t err = cudaFuncSetAttribute(k_top1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (err != cudaSuccess) return err;
      PD_TIMED("eig_mc", s, k_top1<<<w.count, EIG_THREADS, smem, s>>>(n, w));
      return cudaGetLastError();
    }
  }
  return cplx ? eig_dispatch<true>(n, ep, w, s, ad) : eig_dispatch<false>(n, ep, w, s, ad);
}

}  // namespace pd
