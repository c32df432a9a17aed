// Tensor-core synthesis for high ranks (the mixed path's adaptive shrinkage).
//
// The adaptive rules keep most or all of a patch's spectrum, so its synthesis
// out = Xc V diag(c) V^H + mean (space_time/utils.py:81-99) is a dense product
// Xc K with K = V diag(c) V^H (n x n). In the real embedding of complex data,
// x -> [re, im] interleaved and k = a + ib -> [[a, b], [-b, a]], it is one real
// GEMM of the patch's M x N rows (N = 2n) with an N x N matrix.
//
// k_synth_coef: K per patch, split into bf16 hi / lo and written K-major as
//   the A operand A[j][i] = K_emb[i][j] ([N][kn], zero columns past N).
// k_synth_tc: persistent, warp-specialised tcgen05 GEMM
//   D[j][v] = sum_i A[j][i] Xc_emb[v][i]   (hi*hi + hi*lo + lo*hi, fp32 in TMEM)
//   over tiles of 128 output columns j x 256 voxels v; Xc_emb is the row-major
//   split copy k_pack_patches writes. Warp 4 issues the TMA loads into a
//   2-stage ring, warp 5 the MMAs into one of two TMEM accumulators, warps 0-3
//   drain the other accumulator: + mean, x theta, and a float atomic add into
//   the volume (a warp adds 32 consecutive floats of a voxel's frames), plus
//   the per-window weight / noise sums and the rank map, as k_synth.
#include <cuda.h>
#include <cuda_runtime.h>

#include "pd_common.cuh"
#include "pd_kernels.cuh"
#include "pd_profile.cuh"
#include "pd_tc.cuh"

namespace pd {

namespace {
constexpr int ST_BM = 128;  // output columns per tile (MMA M)
constexpr int ST_BN = 256;  // voxels per tile (MMA N)
constexpr int ST_STAGES = 2;
constexpr int ST_THREADS = 192;  // warps 0-3 epilogue, 4 TMA, 5 MMA
constexpr uint32_t ST_TILE_A = ST_BM * 128;  // 64 bf16 of K per row
constexpr uint32_t ST_TILE_B = ST_BN * 128;
constexpr uint32_t ST_STAGE = 2 * (ST_TILE_A + ST_TILE_B);  // hi and lo
constexpr int CF_T = 64;                                     // K tile of k_synth_coef (entries of the n x n matrix)
constexpr int CF_A = 16;                                     // components per shared-memory step

size_t st_smem() { return 1024 + (size_t)ST_STAGES * ST_STAGE + 2 * ST_BN * 8 + 2 * ST_BN * 8 + 256; }
}  // namespace

// ---------------------------------------------------------------------------
// K = V diag(c) V^H as the bf16 hi / lo A operand
// ---------------------------------------------------------------------------
__device__ __forceinline__ void st_pack2(__nv_bfloat16* hi, __nv_bfloat16* lo, int64_t off, float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  const float2 f = __bfloat1622float2(h);
  *reinterpret_cast<__nv_bfloat162*>(hi + off) = h;
  *reinterpret_cast<__nv_bfloat162*>(lo + off) = __floats2bfloat162_rn(a - f.x, b - f.y);
}

// grid: patches x the tiles (ti >= tj) of K's lower triangle (64 x 64
// entries each), 256 threads; a thread holds 4 consecutive i x 4 j (strided by
// 16). K is Hermitian: an off-diagonal tile also writes its mirror (j, i).
template <bool CPLX>
__global__ void __launch_bounds__(256) k_synth_coef(int n, PatchWork w, int64_t kn, __nv_bfloat16* __restrict__ ahi,
                                                    __nv_bfloat16* __restrict__ alo) {
  using T = typename Elem<CPLX>::T;
  __shared__ __align__(16) T vi[CF_A][CF_T];
  __shared__ __align__(16) T vj[CF_A][CF_T];
  __shared__ float cs[CF_A];
  const int tiles = (n + CF_T - 1) / CF_T;
  const int per = tiles * (tiles + 1) / 2;
  const int p = (int)(blockIdx.x / (unsigned)per);
  int t = (int)(blockIdx.x - (unsigned)p * (unsigned)per);
  int ti = 0;
  while (t > ti) {  // lower-triangle tile t -> (ti, tj), tj <= ti
    t -= ti + 1;
    ++ti;
  }
  const int tj = t;
  const int i0 = ti * CF_T, j0 = tj * CF_T;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int act = w.n_active[p];
  const float* vb = w.vec + (int64_t)p * w.vec_stride;
  const float* cb = w.coef + (int64_t)p * w.n_stride;
  const int n2 = 2 * n;
  T acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = zero<T>();
  for (int a0 = 0; a0 < act; a0 += CF_A) {
    __syncthreads();
    for (int e = tid; e < CF_A * CF_T; e += 256) {
      const int aa = e / CF_T, ii = e - aa * CF_T, a = a0 + aa;
      T x = zero<T>(), y = zero<T>();
      if (a < act) {
        if constexpr (CPLX) {
          const cf* col = reinterpret_cast<const cf*>(vb + (int64_t)a * n2);
          if (i0 + ii < n) x = col[i0 + ii];
          if (j0 + ii < n) y = col[j0 + ii];
        } else {
          if (i0 + ii < n) x = vb[(int64_t)a * n2 + i0 + ii];
          if (j0 + ii < n) y = vb[(int64_t)a * n2 + j0 + ii];
        }
      }
      vi[aa][ii] = x;
      vj[aa][ii] = y;
    }
    if (tid < CF_A) cs[tid] = a0 + tid < act ? cb[a0 + tid] : 0.f;
    __syncthreads();
#pragma unroll 4
    for (int aa = 0; aa < CF_A; ++aa) {
      const float c = cs[aa];
      T x[4], y[4];
      // the thread's four consecutive i in 16-byte loads (a half-warp shares them)
      if constexpr (CPLX) {
        const float4 u0 = *reinterpret_cast<const float4*>(&vi[aa][4 * tx]);
        const float4 u1 = *reinterpret_cast<const float4*>(&vi[aa][4 * tx + 2]);
        x[0] = cf{u0.x, u0.y};
        x[1] = cf{u0.z, u0.w};
        x[2] = cf{u1.x, u1.y};
        x[3] = cf{u1.z, u1.w};
      } else {
        const float4 u0 = *reinterpret_cast<const float4*>(&vi[aa][4 * tx]);
        x[0] = u0.x;
        x[1] = u0.y;
        x[2] = u0.z;
        x[3] = u0.w;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        x[q] = x[q] * c;
        y[q] = vj[aa][ty + 16 * q];
      }
#pragma unroll
      for (int qi = 0; qi < 4; ++qi)
#pragma unroll
        for (int qj = 0; qj < 4; ++qj) {
          if constexpr (CPLX) acc[qi][qj] = acc[qi][qj] + cmulc(y[qj], x[qi]);  // c V_ia conj(V_ja)
          else acc[qi][qj] += x[qi] * y[qj];
        }
    }
  }
  // A[j][i] = K_emb[i][j]: complex entry (i, j) = a + ib fills rows 2j, 2j+1,
  // columns 2i, 2i+1 with [a, -b] and [b, a]; its mirror (j, i) = a - ib fills
  // rows 2i, 2i+1, columns 2j, 2j+1 with [a, b] and [-b, a]
  __nv_bfloat16* hp = ahi + (int64_t)p * (CPLX ? 2 * n : n) * kn;
  __nv_bfloat16* lp = alo + (int64_t)p * (CPLX ? 2 * n : n) * kn;
  const int ib = i0 + 4 * tx;
  const bool mirror = ti != tj;
#pragma unroll
  for (int qj = 0; qj < 4; ++qj) {
    const int j = j0 + ty + 16 * qj;
    if (j >= n) continue;
    if constexpr (CPLX) {
      const int64_t r0 = (int64_t)(2 * j) * kn, r1 = r0 + kn;
#pragma unroll
      for (int qi = 0; qi < 4; ++qi) {
        const int64_t c = 2 * (int64_t)(ib + qi);
        if (c >= kn) break;
        const cf k = ib + qi < n ? acc[qi][qj] : cf{0.f, 0.f};
        st_pack2(hp, lp, r0 + c, k.x, -k.y);
        st_pack2(hp, lp, r1 + c, k.y, k.x);
        if (mirror && ib + qi < n) {
          const int64_t m0 = (int64_t)(2 * (ib + qi)) * kn + 2 * j;
          st_pack2(hp, lp, m0, k.x, k.y);
          st_pack2(hp, lp, m0 + kn, -k.y, k.x);
        }
      }
    } else {
      const int64_t r0 = (int64_t)j * kn;
#pragma unroll
      for (int qi = 0; qi < 4; qi += 2) {
        const int64_t c = ib + qi;
        if (c >= kn) break;
        st_pack2(hp, lp, r0 + c, ib + qi < n ? acc[qi][qj] : 0.f, ib + qi + 1 < n ? acc[qi + 1][qj] : 0.f);
      }
      if (mirror) {
#pragma unroll
        for (int qi = 0; qi < 4; ++qi) {
          if (ib + qi >= n) break;
          const int64_t m0 = (int64_t)(ib + qi) * kn + j;
          const __nv_bfloat16 h = __float2bfloat16_rn(acc[qi][qj]);
          hp[m0] = h;
          lp[m0] = __float2bfloat16_rn(acc[qi][qj] - __bfloat162float(h));
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// The GEMM with the recombination epilogue
// ---------------------------------------------------------------------------
struct StArgs {
  int N;          // real columns
  int64_t kn;     // K extent (N rounded up to 64)
  int nj, nv;     // tiles per patch along output columns / voxels
  int tiles;      // count * nj * nv
  int cplx;
};

__device__ __forceinline__ void st_tile(const StArgs& a, int t, int& p, int& jt, int& vt) {
  const int per = a.nj * a.nv;
  p = t / per;
  const int r = t - p * per;
  vt = r / a.nj;
  jt = r - vt * a.nj;
}

__global__ void __launch_bounds__(ST_THREADS, 1) k_synth_tc(const __grid_constant__ CUtensorMap map_ahi,
                                                            const __grid_constant__ CUtensorMap map_alo,
                                                            const __grid_constant__ CUtensorMap map_bhi,
                                                            const __grid_constant__ CUtensorMap map_blo, Geo g,
                                                            PatchWork w, SynthArgs sa, StArgs a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int M = (int)g.rows, N = a.N;
  int64_t* vbase = reinterpret_cast<int64_t*>(sm + ST_STAGES * ST_STAGE);  // [2][ST_BN] float offsets
  int64_t* vvox = vbase + 2 * ST_BN;                                       // [2][ST_BN] voxel indices
  uint64_t* bars = reinterpret_cast<uint64_t*>(vvox + 2 * ST_BN);
  uint64_t* full = bars;                   // [ST_STAGES]
  uint64_t* empty = bars + ST_STAGES;      // [ST_STAGES]
  uint64_t* tfull = bars + 2 * ST_STAGES;  // [2]
  uint64_t* tempty = tfull + 2;            // [2]
  uint64_t* done = tempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);  // any role gave up
  volatile int* epi_abort = abort_flag + 1;  // written and read by the epilogue warps only

  if (tid == 0) {
    for (int s = 0; s < ST_STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);  // one arrival per epilogue warp
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    *epi_abort = 0;
    mbar_fence_init();
  }
  if (warp == 0) {
    tmem_alloc(tmem_slot, 512);  // two 256-column accumulators
    tc_fence_before();
  }
  __syncthreads();
  tc_fence_after();
  const uint32_t taddr = *tmem_slot;
  const uint32_t sbase = smem_u32(sm);
  const int nch = (int)(a.kn / 64);
  const int fs = a.cplx ? 2 : 1;

  if (warp == 4) {
    // ------------------------------------------------------------ TMA producer
    if (lane == 0) {
      int c = 0;
      for (int t = blockIdx.x; t < a.tiles && !*abort_flag; t += gridDim.x) {
        int p, jt, vt;
        st_tile(a, t, p, jt, vt);
        for (int k = 0; k < nch; ++k, ++c) {
          const int s = c % ST_STAGES;
          if (c >= ST_STAGES && !mbar_wait(&empty[s], ((c / ST_STAGES) - 1) & 1)) {
            atomicExch(w.err, 4);
            *abort_flag = 1;
            break;
          }
          const uint32_t st = sbase + s * ST_STAGE;
          const uint32_t fb = smem_u32(&full[s]);
          mbar_expect_tx(&full[s], ST_STAGE);
          const int kc = k * 64;
          tma_load_3d(st, &map_ahi, kc, jt * ST_BM, p, fb);
          tma_load_3d(st + ST_TILE_A, &map_bhi, kc, vt * ST_BN, p, fb);
          tma_load_3d(st + ST_TILE_A + ST_TILE_B / 2, &map_bhi, kc, vt * ST_BN + ST_BN / 2, p, fb);
          const uint32_t lo = st + ST_TILE_A + ST_TILE_B;
          tma_load_3d(lo, &map_alo, kc, jt * ST_BM, p, fb);
          tma_load_3d(lo + ST_TILE_A, &map_blo, kc, vt * ST_BN, p, fb);
          tma_load_3d(lo + ST_TILE_A + ST_TILE_B / 2, &map_blo, kc, vt * ST_BN + ST_BN / 2, p, fb);
        }
      }
      // the last loads have landed before the CTA may exit (at once unless a
      // wait above gave up with copies in flight)
      for (int q = c > ST_STAGES ? c - ST_STAGES : 0; q < c; ++q) mbar_wait(&full[q % ST_STAGES], (q / ST_STAGES) & 1);
    }
  } else if (warp == 5) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      int c = 0, i = 0;
      for (int t = blockIdx.x; t < a.tiles && !*abort_flag; t += gridDim.x, ++i) {
        int p, jt, vt;
        st_tile(a, t, p, jt, vt);
        const int nvox = min(ST_BN, M - vt * ST_BN);
        const int npad = (nvox + 15) & ~15;
        const uint32_t idesc = umma_idesc_bf16(npad);
        const int b = i & 1;
        if (i >= 2 && !mbar_wait(&tempty[b], ((i >> 1) - 1) & 1)) {
          atomicExch(w.err, 5);
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        const uint32_t acc = taddr + (uint32_t)(b * ST_BN);
        bool ok = true;
        for (int k = 0; k < nch; ++k, ++c) {
          const int s = c % ST_STAGES;
          if (!mbar_wait(&full[s], (c / ST_STAGES) & 1)) {
            atomicExch(w.err, 5);
            *abort_flag = 1;
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t st = sbase + s * ST_STAGE;
          const uint32_t ahi = st, bhi = st + ST_TILE_A, alo = st + ST_TILE_A + ST_TILE_B, blo = alo + ST_TILE_A;
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            const uint32_t kb = kk * 32;
            const uint64_t da = umma_desc_sw128(ahi + kb), db = umma_desc_sw128(bhi + kb);
            umma_bf16(acc, da, db, idesc, (k | kk) != 0 ? 1u : 0u);
            umma_bf16(acc, da, umma_desc_sw128(blo + kb), idesc, 1u);
            umma_bf16(acc, umma_desc_sw128(alo + kb), db, idesc, 1u);
          }
          umma_commit(&empty[s]);
        }
        if (!ok) break;
        umma_commit(&tfull[b]);
      }
      umma_commit(done);
    }
  } else {
    // ------------------------------------------------------------ epilogue (warps 0-3)
    const int64_t T4 = g.shape[3];
    const int rc = (int)(((g.patch[0] / 2) * g.patch[1] + g.patch[1] / 2) * g.patch[2] + g.patch[2] / 2);
    int i = 0;
    for (int t = blockIdx.x; t < a.tiles; t += gridDim.x, ++i) {
      int p, jt, vt;
      st_tile(a, t, p, jt, vt);
      const int b = i & 1;
      const int64_t pidx = w.list[p];
      int64_t o[4];
      patch_origin(g, pidx, o);
      const int nvox = min(ST_BN, M - vt * ST_BN);
      // voxel offsets of this tile (the four epilogue warps only)
      for (int q = tid; q < nvox; q += 128) {
        const int64_t vox = row_voxel(g, o, vt * ST_BN + q);
        vvox[b * ST_BN + q] = vox;
        vbase[b * ST_BN + q] = (vox * T4 + o[3]) * fs;
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");
      const int rank = w.rank[p];
      const float nv = w.noise[p];
      const float theta = (sa.recombination == PD_RECOMB_WEIGHTED) ? (float)(1.0 / (2.0 + (double)rank)) : 1.f;
      if (jt == 0) {
        // the per-window weight / noise sums and the records (once per voxel / patch)
        const int64_t gt = patch_window(g, pidx);
        for (int q = tid; q < nvox; q += 128) {
          const int64_t vox = vvox[b * ST_BN + q];
          atomicAdd(&sa.weight_acc[vox * g.grid[3] + gt], theta);
          if (!isnan(nv)) atomicAdd(&sa.noise_acc[vox * g.grid[3] + gt], theta * nv);
        }
        if (rc >= vt * ST_BN && rc < vt * ST_BN + nvox) {
          const int64_t rb = vbase[b * ST_BN + rc - vt * ST_BN] / fs;
          for (int q = tid; q < (int)g.cols; q += 128) atomicMax(&sa.rank_map[rb + q], rank);
        }
        if (vt == 0 && tid == 0) {
          sa.patch_rank[sa.list_offset + p] = rank;
          sa.patch_noise[sa.list_offset + p] = nv;
        }
      }
      const int j = jt * ST_BM + warp * 32 + lane;
      const float mu = j < N ? w.mean[(int64_t)p * w.n_stride * fs + j] : 0.f;
      const bool ok = !*abort_flag && mbar_wait(&tfull[b], (i >> 1) & 1);
      if (!ok && lane == 0) {
        atomicExch(w.err, 6);
        *epi_abort = 1;
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");
      if (*epi_abort) break;  // the same decision in all four warps
      tc_fence_after();
      const uint32_t lane_addr = taddr + (uint32_t)(b * ST_BN) + ((uint32_t)(warp * 32) << 16);
      float* out = reinterpret_cast<float*>(sa.out);
      for (int cc = 0; cc < nvox; cc += 16) {
        float v[16];
        tmem_ld16(lane_addr + cc, v);
        if (j < N) {
#pragma unroll
          for (int q = 0; q < 16; ++q)
            if (cc + q < nvox) atomicAdd(out + vbase[b * ST_BN + cc + q] + j, (v[q] + mu) * theta);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[b]);
      asm volatile("bar.sync 1, 128;" ::: "memory");  // the voxel table of buffer b is free again
    }
  }
  __syncwarp();
  // every MMA has completed before TMEM is released
  if (warp == 0) {
    const bool ok = mbar_wait(done, 0);
    if (!ok && lane == 0) atomicExch(w.err, 6);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(taddr, 512);
  }
}

cudaError_t launch_synth_tc(const Geo& g, bool cplx, const PatchWork& w, const SynthArgs& sa, cudaStream_t s) {
  const PackedLayout L = packed_layout(g.cols, cplx, g.rows, true, w.count);
  __nv_bfloat16* base = reinterpret_cast<__nv_bfloat16*>(w.packed);
  const int n = g.cols;
  const int tiles = (n + CF_T - 1) / CF_T;
  const unsigned cgrid = (unsigned)((int64_t)w.count * tiles * (tiles + 1) / 2);
  if (cplx)
    PD_TIMED("synth_coef", s,
             k_synth_coef<true><<<cgrid, 256, 0, s>>>(n, w, L.kn, base + L.coef_hi, base + L.coef_lo));
  else
    PD_TIMED("synth_coef", s,
             k_synth_coef<false><<<cgrid, 256, 0, s>>>(n, w, L.kn, base + L.coef_hi, base + L.coef_lo));
  CUtensorMap ahi, alo, bhi, blo;
  cudaError_t e = make_bf16_map(&ahi, base + L.coef_hi, L.kn, L.N, w.count);
  if (e == cudaSuccess) e = make_bf16_map(&alo, base + L.coef_lo, L.kn, L.N, w.count);
  if (e == cudaSuccess) e = make_bf16_map(&bhi, base + L.rows_hi, L.kn, L.kp, w.count);
  if (e == cudaSuccess) e = make_bf16_map(&blo, base + L.rows_lo, L.kn, L.kp, w.count);
  if (e != cudaSuccess) return e;
  StArgs a{};
  a.N = L.N;
  a.kn = L.kn;
  a.nj = (L.N + ST_BM - 1) / ST_BM;
  a.nv = (g.rows + ST_BN - 1) / ST_BN;
  a.cplx = cplx ? 1 : 0;
  const int64_t tiles_all = (int64_t)w.count * a.nj * a.nv;
  if (tiles_all > INT32_MAX) return cudaErrorInvalidConfiguration;
  a.tiles = (int)tiles_all;
  const size_t smem = st_smem();
  e = cudaFuncSetAttribute(k_synth_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const unsigned grid = (unsigned)std::min<int64_t>(tiles_all, sms);
  PD_TIMED("synth_tc", s, k_synth_tc<<<grid, ST_THREADS, smem, s>>>(ahi, alo, bhi, blo, g, w, sa, a));
  return cudaGetLastError();
}

}  // namespace pd
