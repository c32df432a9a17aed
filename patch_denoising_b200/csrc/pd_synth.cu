// Low-rank synthesis fused with the recombination scatter, and the final
// normalisation / masking pass.
//
// For a patch with active eigenvectors V (frames x a) and coefficients c:
//   out_r = (x_r - mean) V diag(c) V^H + mean      (row r of the Casorati matrix)
// which equals eig_synthesis (space_time/utils.py:140-146) for c = 1 and
// svd_synthesis with shrunk values (utils.py:81-99) for c = s~/s. The result is
// scattered into the volume with theta = 1/(2+maxidx) (weighted), 1 (average),
// or written at the patch centre only (center), as in base.py:243-252.
#include <float.h>

#include "pd_common.cuh"
#include "pd_kernels.cuh"
#include "pd_profile.cuh"

namespace pd {

constexpr int SYN_THREADS = 256;
constexpr int SYN_NW = SYN_THREADS / 32;

__device__ __forceinline__ void acc_add(float* p, float v) { atomicAdd(p, v); }
__device__ __forceinline__ void acc_add(cf* p, cf v) {
  atomicAdd(reinterpret_cast<float2*>(p), make_float2(v.x, v.y));
}

// WIDE: with the grouped reduction for ranks above 8 (adaptive launches only;
// its registers would cost the low-rank methods occupancy). BATCH: the patch's
// volume comes from the batched call's table (kept out of the one-volume
// instantiations, whose registers it would raise from 80 to 97).
template <bool CPLX, int NS, int R, bool WIDE, bool BATCH>
__global__ void __launch_bounds__(SYN_THREADS) k_synth(Geo g, const typename Elem<CPLX>::T* __restrict__ in,
                                                       PatchWork w, SynthArgs sa, int ysplit) {
  using T = typename Elem<CPLX>::T;
  extern __shared__ __align__(16) unsigned char sm[];
  // grid: patches x ysplit row blocks, flattened patch-major (the blocks of a
  // patch, and of its overlapping neighbours, read and scatter to the same
  // voxels close together in time)
  const int p = (int)(blockIdx.x / (unsigned)ysplit);
  const int yb = (int)(blockIdx.x - (unsigned)p * (unsigned)ysplit);
  if constexpr (BATCH) {  // batched call: this patch's volume and its output buffers
    const VolDesc& v = w.vols[w.vol_of[p]];
    g = v.g;
    in = reinterpret_cast<const T*>(v.in);
    sa.out = v.out;
    sa.weight_acc = v.wacc;
    sa.noise_acc = v.nacc;
    sa.noise_ctr = v.nctr;
    sa.rank_map = v.rank_map;
    sa.patch_rank = v.prank - v.first;  // records at the volume's own list positions
    sa.patch_noise = v.pnoise - v.first;
  }
  const int n = g.cols, M = g.rows;
  T* ys = reinterpret_cast<T*>(sm);  // [SYN_NW][R][n]
  T* smean = ys + SYN_NW * R * n;    // [n]
  float* scoef = reinterpret_cast<float*>(smean + n);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t pidx = w.list[p];
  int64_t o[4];
  patch_origin(g, pidx, o);
  const int64_t gt = patch_window(g, pidx);
  const int act = w.n_active[p];
  const int rank = w.rank[p];
  const float nv = w.noise[p];
  const T* mean = reinterpret_cast<const T*>(w.mean) + (int64_t)p * w.n_stride;
  for (int t = tid; t < n; t += SYN_THREADS) smean[t] = mean[t];
  for (int a = tid; a < act; a += SYN_THREADS) scoef[a] = w.coef[(int64_t)p * w.n_stride + a];
  const float* vb = w.vec + (int64_t)p * w.vec_stride;
  const int n2 = 2 * n;
  const int64_t T4 = g.shape[3];
  const bool center = (sa.recombination == PD_RECOMB_CENTER);
  const float theta = (sa.recombination == PD_RECOMB_WEIGHTED) ? (float)(1.0 / (2.0 + (double)rank)) : 1.f;
  const int rc = (int)(((g.patch[0] / 2) * g.patch[1] + g.patch[1] / 2) * g.patch[2] + g.patch[2] / 2);
  const int tc = (int)(g.patch[3] / 2);
  if (yb == 0 && tid == 0) {
    sa.patch_rank[sa.list_offset + p] = rank;
    sa.patch_noise[sa.list_offset + p] = nv;
  }
  __syncthreads();

  auto vat = [&](int a, int t) -> T {
    if constexpr (CPLX) return reinterpret_cast<const cf*>(vb + (int64_t)a * n2)[t];
    else return vb[(int64_t)a * n2 + t];
  };

  const int rstep = ysplit * SYN_NW * R;
  int r0 = (yb * SYN_NW + warp) * R;
  if (center) r0 = (yb == 0 && warp == 0) ? rc : M;  // one row only
  for (; r0 < M; r0 += center ? M : rstep) {
    int64_t base[R];
    bool ok[R];
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int r = r0 + q;
      ok[q] = (r < M) && (!center || q == 0);
      base[q] = ok[q] ? row_voxel(g, o, r) * T4 + o[3] : 0;
    }
    T* yw = ys + (int64_t)warp * R * n;
    {
      T x[R][NS];
#pragma unroll
      for (int q = 0; q < R; ++q)
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          const int t = lane + 32 * s;
          x[q][s] = (ok[q] && t < n) ? in[base[q] + t] - smean[t] : zero<T>();
        }
      int a = 0;
      if (WIDE && act > 8) {
        // a high rank (the adaptive shrinkage keeps whole spectra): the row
        // sums of eight components leave in one reduce-scatter butterfly
        // instead of eight warp sums
        for (; a + 8 <= act; a += 8) {
          T pg[R][8];
#pragma unroll
          for (int q = 0; q < R; ++q)
#pragma unroll
            for (int g = 0; g < 8; ++g) pg[q][g] = zero<T>();
#pragma unroll
          for (int g = 0; g < 8; ++g)
#pragma unroll
            for (int s = 0; s < NS; ++s) {
              const int t = lane + 32 * s;
              if (t < n) {
                const T v = vat(a + g, t);
#pragma unroll
                for (int q = 0; q < R; ++q) pg[q][g] = pg[q][g] + mul(x[q][s], v);
              }
            }
#pragma unroll
          for (int q = 0; q < R; ++q) {
            int slot;
            const T tot = reduce_scatter8<T>(pg[q], lane, &slot);
            if ((lane & 3) == 0) yw[q * n + a + slot] = tot * scoef[a + slot];
          }
        }
      }
      for (; a < act; ++a) {
        T pa[R];
#pragma unroll
        for (int q = 0; q < R; ++q) pa[q] = zero<T>();
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          const int t = lane + 32 * s;
          if (t < n) {
            const T v = vat(a, t);
#pragma unroll
            for (int q = 0; q < R; ++q) pa[q] = pa[q] + mul(x[q][s], v);
          }
        }
        const float ca = scoef[a];
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const T y = warp_sum(pa[q]);
          if (lane == 0) yw[q * n + a] = y * ca;
        }
      }
    }
    __syncwarp();
    T ov[R][NS];
#pragma unroll
    for (int q = 0; q < R; ++q)
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const int t = lane + 32 * s;
        ov[q][s] = t < n ? smean[t] : zero<T>();
      }
    for (int a = 0; a < act; ++a) {
      T yq[R];
#pragma unroll
      for (int q = 0; q < R; ++q) yq[q] = yw[q * n + a];
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const int t = lane + 32 * s;
        if (t < n) {
          const T v = cj(vat(a, t));
#pragma unroll
          for (int q = 0; q < R; ++q) ov[q][s] = ov[q][s] + mul(yq[q], v);
        }
      }
    }
    __syncwarp();
    T* out = reinterpret_cast<T*>(sa.out);
#pragma unroll
    for (int q = 0; q < R; ++q) {
      if (!ok[q]) continue;
      if (center) {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          const int t = lane + 32 * s;
          if (t == tc) out[base[q] + t] = ov[q][s];
          if (t < n) atomicMax(&sa.rank_map[base[q] + t], rank);
          if (t == tc && !isnan(nv)) sa.noise_ctr[base[q] + t] = nv;
        }
      } else {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          const int t = lane + 32 * s;
          if (t < n) acc_add(out + base[q] + t, ov[q][s] * theta);
        }
        if (lane == 0) {
          const int64_t vox = (base[q] - o[3]) / T4;
          atomicAdd(&sa.weight_acc[vox * g.grid[3] + gt], theta);
          if (!isnan(nv)) atomicAdd(&sa.noise_acc[vox * g.grid[3] + gt], theta * nv);
        }
        if (r0 + q == rc) {
#pragma unroll
          for (int s = 0; s < NS; ++s) {
            const int t = lane + 32 * s;
            if (t < n) atomicMax(&sa.rank_map[base[q] + t], rank);
          }
        }
      }
    }
    __syncwarp();
  }
}

template <bool CPLX, int NS>
static void synth_ns(const Geo& g, const void* in, const PatchWork& w, const SynthArgs& a, cudaStream_t s) {
  using T = typename Elem<CPLX>::T;
  constexpr int R = CPLX ? 2 : 4;
  const int n = g.cols;
  const size_t smem = sizeof(T) * ((size_t)SYN_NW * R * n + n) + sizeof(float) * n + 16;
  auto kern = a.wide ? k_synth<CPLX, NS, R, true, false>
                     : (w.vols ? k_synth<CPLX, NS, R, false, true> : k_synth<CPLX, NS, R, false, false>);
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int rows_per_block = SYN_NW * R;
  int ysplit = (g.rows + rows_per_block - 1) / rows_per_block;
  if (ysplit > 8) ysplit = 8;
  if (a.row_blocks > 0) ysplit = a.row_blocks;  // a tuned split
  if (a.recombination == PD_RECOMB_CENTER) ysplit = 1;
  const unsigned grid = (unsigned)((int64_t)w.count * ysplit);
  PD_TIMED("synth_scatter", s, kern<<<grid, SYN_THREADS, smem, s>>>(g, (const T*)in, w, a, ysplit));
}

template <bool CPLX>
static void synth_dispatch(const Geo& g, const void* in, const PatchWork& w, const SynthArgs& a, cudaStream_t s) {
  const int n = g.cols;
  if (n <= 64) synth_ns<CPLX, 2>(g, in, w, a, s);
  else if (n <= 128) synth_ns<CPLX, 4>(g, in, w, a, s);
  else if (n <= 224) synth_ns<CPLX, 7>(g, in, w, a, s);
  else if (n <= 320) synth_ns<CPLX, 10>(g, in, w, a, s);
  else synth_ns<CPLX, 14>(g, in, w, a, s);
}

void launch_synth(const Geo& g, bool cplx, const void* in, const PatchWork& w, const SynthArgs& a,
                  cudaStream_t s) {
  if (cplx) synth_dispatch<true>(g, in, w, a, s);
  else synth_dispatch<false>(g, in, w, a, s);
}

// out /= weights (weighted / average), expand window sums to 4D, mask.
// A work item is FQ consecutive frames of one voxel: one index division per
// item, and with T % FQ == 0 (VEC) every access is a 16-byte vector.
constexpr int FQ = 4;

template <bool CPLX, bool VEC, class I>
__device__ __forceinline__ void finalize_items(const Geo& g, int recomb, typename Elem<CPLX>::T* __restrict__ out,
                                               const float* __restrict__ wacc, const float* __restrict__ nacc,
                                               const float* __restrict__ nctr, float* __restrict__ weights,
                                               float* __restrict__ noise_map, const uint8_t* __restrict__ mask,
                                               int mask_is_4d, I items, I groups) {
  using T = typename Elem<CPLX>::T;
  const I T4 = (I)g.shape[3];
  const int ngt = (int)g.grid[3];
  for (I it = (I)blockIdx.x * blockDim.x + threadIdx.x; it < items; it += (I)gridDim.x * blockDim.x) {
    const I v = it / groups;
    const int t0 = (int)(it - v * groups) * FQ;
    const int64_t e0 = (int64_t)v * T4 + t0;
    float ws[FQ], ns[FQ];
#pragma unroll
    for (int q = 0; q < FQ; ++q) ws[q] = ns[q] = 0.f;
    for (int k = 0; k < ngt; ++k) {
      const int lo = k * (int)g.step[3], hi = lo + (int)g.patch[3];
      if (t0 + FQ <= lo || t0 >= hi) continue;
      const float wk = wacc[(int64_t)v * ngt + k], nk = nacc[(int64_t)v * ngt + k];
#pragma unroll
      for (int q = 0; q < FQ; ++q) {
        if (t0 + q >= lo && t0 + q < hi) {
          ws[q] += wk;
          ns[q] += nk;
        }
      }
    }
    T val[FQ];
    float nm[FQ];
    bool keep[FQ];
    if constexpr (VEC) {
      if constexpr (CPLX) {
        const float4 a = *reinterpret_cast<const float4*>(out + e0);
        const float4 b = *reinterpret_cast<const float4*>(out + e0 + 2);
        val[0] = cf{a.x, a.y};
        val[1] = cf{a.z, a.w};
        val[2] = cf{b.x, b.y};
        val[3] = cf{b.z, b.w};
      } else {
        const float4 a = *reinterpret_cast<const float4*>(out + e0);
        val[0] = a.x;
        val[1] = a.y;
        val[2] = a.z;
        val[3] = a.w;
      }
      if (recomb == PD_RECOMB_CENTER) {
        const float4 c = *reinterpret_cast<const float4*>(nctr + e0);
        nm[0] = c.x;
        nm[1] = c.y;
        nm[2] = c.z;
        nm[3] = c.w;
      }
    } else {
#pragma unroll
      for (int q = 0; q < FQ; ++q) {
        val[q] = zero<T>();
        nm[q] = 0.f;
        if (t0 + q < T4) {
          val[q] = out[e0 + q];
          if (recomb == PD_RECOMB_CENTER) nm[q] = nctr[e0 + q];
        }
      }
    }
#pragma unroll
    for (int q = 0; q < FQ; ++q) {
      keep[q] = mask == nullptr ? true : (mask_is_4d ? mask[e0 + q] != 0 : mask[v] != 0);
      if (!VEC && t0 + q >= T4) keep[q] = false;
      if (recomb != PD_RECOMB_CENTER) {
        if constexpr (CPLX) val[q] = cf{val[q].x / ws[q], val[q].y / ws[q]};
        else val[q] = val[q] / ws[q];
        nm[q] = ns[q] / ws[q];
      }
      if (!keep[q]) {
        val[q] = zero<T>();
        nm[q] = 0.f;
      }
    }
    if constexpr (VEC) {
      if constexpr (CPLX) {
        *reinterpret_cast<float4*>(out + e0) = make_float4(val[0].x, val[0].y, val[1].x, val[1].y);
        *reinterpret_cast<float4*>(out + e0 + 2) = make_float4(val[2].x, val[2].y, val[3].x, val[3].y);
      } else {
        *reinterpret_cast<float4*>(out + e0) = make_float4(val[0], val[1], val[2], val[3]);
      }
      *reinterpret_cast<float4*>(weights + e0) = make_float4(ws[0], ws[1], ws[2], ws[3]);
      *reinterpret_cast<float4*>(noise_map + e0) = make_float4(nm[0], nm[1], nm[2], nm[3]);
    } else {
#pragma unroll
      for (int q = 0; q < FQ; ++q) {
        if (t0 + q < T4) {
          out[e0 + q] = val[q];
          weights[e0 + q] = ws[q];
          noise_map[e0 + q] = nm[q];
        }
      }
    }
  }
}

template <bool CPLX, bool VEC>
__global__ void __launch_bounds__(256) k_finalize(Geo g, int recomb, typename Elem<CPLX>::T* __restrict__ out,
                                                  const float* __restrict__ wacc, const float* __restrict__ nacc,
                                                  const float* __restrict__ nctr, float* __restrict__ weights,
                                                  float* __restrict__ noise_map, const uint8_t* __restrict__ mask,
                                                  int mask_is_4d) {
  const int64_t groups = (g.shape[3] + FQ - 1) / FQ;
  const int64_t items = g.shape[0] * g.shape[1] * g.shape[2] * groups;
  if (items + (int64_t)gridDim.x * blockDim.x < (int64_t)0x7fffffff)
    finalize_items<CPLX, VEC, int>(g, recomb, out, wacc, nacc, nctr, weights, noise_map, mask, mask_is_4d,
                                   (int)items, (int)groups);
  else
    finalize_items<CPLX, VEC, int64_t>(g, recomb, out, wacc, nacc, nctr, weights, noise_map, mask, mask_is_4d,
                                       items, groups);
}

void launch_finalize(const Geo& g, bool cplx, int recomb, void* out, const float* wacc, const float* nacc,
                     const float* nctr, float* weights, float* noise_map, const uint8_t* mask, int mask_is_4d,
                     cudaStream_t s) {
  const int64_t items = g.shape[0] * g.shape[1] * g.shape[2] * ((g.shape[3] + FQ - 1) / FQ);
  int64_t blocks = (items + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  // 16-byte vectors need every item to start on a multiple of FQ frames and
  // 16-byte aligned buffers
  const auto al = [](const void* q) { return q == nullptr || (reinterpret_cast<uintptr_t>(q) & 15) == 0; };
  const bool vec = g.shape[3] % FQ == 0 && al(out) && al(weights) && al(noise_map) && al(nctr);
#define PD_FIN(C, V, TT)                                                                                      \
  PD_TIMED("finalize", s, (k_finalize<C, V><<<(int)blocks, 256, 0, s>>>(g, recomb, (TT*)out, wacc, nacc, nctr, \
                                                                         weights, noise_map, mask, mask_is_4d)))
  if (cplx) {
    if (vec) PD_FIN(true, true, cf);
    else PD_FIN(true, false, cf);
  } else {
    if (vec) PD_FIN(false, true, float);
    else PD_FIN(false, false, float);
  }
#undef PD_FIN
}

}  // namespace pd
