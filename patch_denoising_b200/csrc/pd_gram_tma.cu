// Mixed-precision Gram, operands packed once and fed to tcgen05 by TMA.
//
// k_pack_patches: for every listed patch, the centred Casorati matrix X (M rows
//   x N real columns; a complex patch is its interleaved real view, N = 2 n) is
//   written transposed as two bf16 matrices Xhi^T, Xlo^T (N rows x Kp, Kp = M
//   rounded up to 64, zero padded), x = hi + lo to about 16 bits. Reads are
//   coalesced along frames, writes along voxels through a shared-memory
//   transpose; the kernel is memory bound and runs at full occupancy.
// k_gram_tma: tiles = (patch, 128 x <=256 block of the lower Gram). When N is
//   not a multiple of 128 (N = 400 for 200 complex frames), the last, partial
//   128-row block would compute mostly padding: its rows are produced instead
//   as a strip of columns, G[0:N, Nmain:N] (Nmain = N rounded down to 128), by
//   symmetry, from a narrow B box (the remainder rows only).
//   Persistent (one CTA per SM over the tiles) and warp-specialised: one
//   thread issues cp.async.bulk.tensor loads (128-byte swizzle, the canonical
//   K-major layout of tcgen05) into a 2-stage ring guarded by mbarriers with
//   transaction counts; one thread issues tcgen05.mma (hi*hi + hi*lo + lo*hi)
//   into one of two TMEM accumulators; four warps read the other accumulator
//   and write the packed Gram (complex via 2x2 blocks).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "pd_common.cuh"
#include "pd_kernels.cuh"
#include "pd_profile.cuh"
#include "pd_rng.cuh"
#include "pd_tc.cuh"

namespace pd {

constexpr int PK_R = 64;  // K rows per pack tile
constexpr int PK_C = 64;  // columns per pack tile
constexpr int TM_BM = 128;
constexpr int TM_BN = 256;
constexpr int TM_BOX = 128;  // rows per TMA box
constexpr int TM_STAGES = 2;  // operand stages (hi and lo of A and B each)
constexpr int TM_TQ = 4;      // claimed tile indices in flight between the roles
constexpr int TM_THREADS = 192;  // warps 0-3 epilogue, 4 TMA, 5 MMA
constexpr uint32_t TM_TILE_A = TM_BM * 128;
constexpr uint32_t TM_TILE_B = TM_BN * 128;

__host__ __device__ inline int64_t pack_k(int64_t rows) { return (rows + 63) & ~int64_t(63); }

// ---------------------------------------------------------------------------
// Packing
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pack_store(__nv_bfloat16* hi, __nv_bfloat16* lo, int64_t off, float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  *reinterpret_cast<__nv_bfloat162*>(hi + off) = h;
  if (lo) {
    const float2 f = __bfloat1622float2(h);
    *reinterpret_cast<__nv_bfloat162*>(lo + off) = __floats2bfloat162_rn(a - f.x, b - f.y);
  }
}

// grid: patches x ceil(N / 64) column tiles x ks K segments, flattened
// patch-major (a patch's CTAs, and its neighbours', which share voxels, run
// close together, so the volume is read from DRAM about once); 256 threads.
// A CTA walks the 64-voxel K tiles of its segment: the patch origin is
// unravelled once, each tile's voxel offsets are formed one tile ahead, and the
// next tile's loads are in flight while the current one is transposed
// through shared memory and stored.
__global__ void __launch_bounds__(256) k_pack_patches(Geo g, const float* __restrict__ in, int N, int cplx,
                                                      const float* __restrict__ mean, const int32_t* __restrict__ list,
                                                      __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo,
                                                      int64_t kp, int ks, __nv_bfloat16* __restrict__ rhi,
                                                      __nv_bfloat16* __restrict__ rlo, int64_t kn) {
  __shared__ float tile[PK_R][PK_C + 1];
  __shared__ int64_t rbs[2][PK_R];
  const int kt_all = (int)(kp / PK_R), ct = (N + PK_C - 1) / PK_C;
  const unsigned per = (unsigned)(ct * ks);
  const int p = (int)(blockIdx.x / per);
  const unsigned t = blockIdx.x - (unsigned)p * per;
  const int seg = (int)(t % (unsigned)ks), c0 = (int)(t / (unsigned)ks) * PK_C;
  const int kt_per = (kt_all + ks - 1) / ks;
  const int kt0 = seg * kt_per, kt1 = min(kt0 + kt_per, kt_all);
  if (kt0 >= kt1) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int64_t o[4];
  patch_origin(g, list[p], o);
  const int64_t fs = cplx ? 2 : 1;
  const int c = tid % PK_C;
  const int col = c0 + c;
  const float mu = col < N ? mean[(int64_t)p * N + col] : 0.f;
  __nv_bfloat16* hp = hi + (int64_t)p * N * kp;
  __nv_bfloat16* lp = lo ? lo + (int64_t)p * N * kp : nullptr;
  constexpr int RPT = PK_R / (256 / PK_C);  // rows loaded per thread and tile (16)
  if (tid < PK_R) {
    const int r = kt0 * PK_R + tid;
    rbs[kt0 & 1][tid] = r < g.rows ? (row_voxel(g, o, r) * g.shape[3] + o[3]) * fs : -1;
  }
  __syncthreads();
  float v[RPT];
#pragma unroll
  for (int i = 0; i < RPT; ++i) {
    const int64_t base = rbs[kt0 & 1][tid / PK_C + i * (256 / PK_C)];
    v[i] = (base >= 0 && col < N) ? __ldg(in + base + col) : 0.f;
  }
  for (int kt = kt0; kt < kt1; ++kt) {
    if (tid < PK_R && kt + 1 < kt1) {
      const int r = (kt + 1) * PK_R + tid;
      rbs[(kt + 1) & 1][tid] = r < g.rows ? (row_voxel(g, o, r) * g.shape[3] + o[3]) * fs : -1;
    }
    __syncthreads();  // the previous tile has been read out of shared memory
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
      const int rr = tid / PK_C + i * (256 / PK_C);
      tile[rr][c] = rbs[kt & 1][rr] >= 0 && col < N ? v[i] - mu : 0.f;
    }
    __syncthreads();  // tile kt and the offsets of tile kt + 1 are visible
    if (kt + 1 < kt1) {
#pragma unroll
      for (int i = 0; i < RPT; ++i) {
        const int64_t base = rbs[(kt + 1) & 1][tid / PK_C + i * (256 / PK_C)];
        v[i] = (base >= 0 && col < N) ? __ldg(in + base + col) : 0.f;
      }
    }
    // each warp writes 64 K-values (128 B) of a column per step
    const int r0 = kt * PK_R;
    for (int cc = warp; cc < PK_C; cc += 8) {
      const int colw = c0 + cc;
      if (colw >= N) break;
      const int64_t off = (int64_t)colw * kp + r0 + 2 * lane;
      pack_store(hp, lp, off, tile[2 * lane][cc], tile[2 * lane + 1][cc]);
    }
    if (rhi) {
      // the row-major copy for the tensor-core synthesis: 64 columns (128 B) of
      // a row per warp step, zeros past N (the tile holds zeros there)
      for (int rr = warp; rr < PK_R; rr += 8) {
        const int64_t off = ((int64_t)p * kp + r0 + rr) * kn + c0 + 2 * lane;
        pack_store(rhi, rlo, off, tile[rr][2 * lane], tile[rr][2 * lane + 1]);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// TMA + tcgen05 Gram
// ---------------------------------------------------------------------------
struct TmaArgs {
  int N;       // real columns of X (= rows of the packed operand)
  int nmain;   // rows covered by whole 128-row blocks when strips are used (else N)
  int sbox;    // rows of the strip's B box (the remainder rounded up to 16), 0 without strips
  int n_out;   // output order (N or N/2 for complex)
  int cplx;
  int64_t kp;  // packed K extent
  int nblk;    // Gram blocks per patch
  int count;   // patches
  int* ctr;    // next unclaimed tile (zero at launch)
  float* out;
  int64_t out_stride;
  int* err;
};

// Block idx of a patch: A rows from arow, B rows from brow, ncols valid
// columns; strip blocks take B from the narrow map.
struct TmBlock {
  int arow, brow, ncols, strip;
};
__host__ __device__ inline TmBlock tm_block_of(int idx, int N, int nmain) {
  for (int rb = 0; rb * TM_BM < nmain; ++rb) {
    const int lim = min((rb + 1) * TM_BM, nmain == N ? N : nmain);
    const int nbs = (lim + TM_BN - 1) / TM_BN;
    if (idx < nbs) return TmBlock{rb * TM_BM, idx * TM_BN, min(lim - idx * TM_BN, TM_BN), 0};
    idx -= nbs;
  }
  return TmBlock{idx * TM_BM, nmain, N - nmain, 1};  // strip: rows idx*128.., columns nmain..N
}

__host__ __device__ inline int tm_blocks(int N, int nmain) {
  int t = 0;
  for (int rb = 0; rb * TM_BM < nmain; ++rb) {
    const int lim = min((rb + 1) * TM_BM, nmain == N ? N : nmain);
    t += (lim + TM_BN - 1) / TM_BN;
  }
  if (nmain < N) t += (N + TM_BM - 1) / TM_BM;
  return t;
}

// Persistent and warp-specialised: one CTA per SM walks the (patch, block)
// tiles. Warp 4 issues the TMA loads into a 2-stage ring (running ahead into
// the next tile), warp 5 the MMAs into one of two 256-column TMEM accumulators,
// warps 0-3 write the other accumulator's block into the packed Gram, so a
// tile's epilogue overlaps the next tile's loads and MMAs.
__device__ __forceinline__ void tm_store(const TmaArgs& a, const TmBlock& blk, float* out, int i, int cc,
                                         const float v[16]) {
  const int N = a.N;
  if (!a.cplx) {
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int j = blk.brow + cc + q;
      if (i >= N || (cc + q) >= blk.ncols) continue;
      if (!blk.strip && j <= i) out[pk(i, j, N)] = v[q];
      if (blk.strip && j >= i) out[pk(j, i, N)] = v[q];  // G[i][j] = G[j][i], stored as the lower (j, i)
    }
  } else {
    float vp[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) vp[q] = __shfl_xor_sync(0xffffffffu, v[q], 1);
    if ((i & 1) == 0) {
      const int ic = i >> 1, n = a.n_out;
      cf* oc = reinterpret_cast<cf*>(out);
#pragma unroll
      for (int q = 0; q < 16; q += 2) {
        const int jc = (blk.brow + cc + q) >> 1;
        if (ic >= n || (cc + q) >= blk.ncols) continue;
        if (!blk.strip && jc <= ic) oc[pk(ic, jc, n)] = cf{v[q] + vp[q + 1], v[q + 1] - vp[q]};
        // strip: the lower entry (jc, ic) is the conjugate of (ic, jc)
        if (blk.strip && jc >= ic) oc[pk(jc, ic, n)] = cf{v[q] + vp[q + 1], vp[q] - v[q + 1]};
      }
    }
  }
}

__global__ void __launch_bounds__(TM_THREADS, 1) k_gram_tma(const __grid_constant__ CUtensorMap map_hi,
                                                             const __grid_constant__ CUtensorMap map_lo,
                                                             const __grid_constant__ CUtensorMap smap_hi,
                                                             const __grid_constant__ CUtensorMap smap_lo, TmaArgs a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int N = a.N;
  constexpr uint32_t STAGE = 2 * (TM_TILE_A + TM_TILE_B);  // hi, then lo
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + TM_STAGES * STAGE);
  uint64_t* full = bars;                   // [TM_STAGES]
  uint64_t* empty = bars + TM_STAGES;      // [TM_STAGES]
  uint64_t* tfull = bars + 2 * TM_STAGES;  // [2]
  uint64_t* tempty = tfull + 2;            // [2]
  uint64_t* done = tempty + 2;
  uint64_t* qfull = done + 1;      // [TM_TQ] a claimed tile index is in the queue
  uint64_t* qempty = qfull + TM_TQ;  // [TM_TQ] its slot is free again
  volatile int* tileq = reinterpret_cast<volatile int*>(qempty + TM_TQ);  // [TM_TQ]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(const_cast<int*>(tileq) + TM_TQ);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);  // any role gave up
  volatile int* epi_abort = abort_flag + 1;  // written and read by the epilogue warps only
  volatile int* tileq_epi = abort_flag + 2;  // the epilogue's current tile (its warp 0 writes it)

  if (tid == 0) {
    for (int s = 0; s < TM_STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);  // one arrival per epilogue warp
    }
    mbar_init(done, 1);
    for (int q = 0; q < TM_TQ; ++q) {
      mbar_init(&qfull[q], 1);
      mbar_init(&qempty[q], 1);
    }
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
  const int nch = (int)((a.kp + 63) / 64);
  const int tiles = a.count * a.nblk;
  // Tiles are claimed in (patch, block) order from a global counter (a CTA
  // that starts late, its SM held by another stream's kernel, takes fewer):
  // a patch's blocks, and its overlapping neighbours', read the same operand
  // rows close together in time (L2). The producer passes each claimed index
  // to the MMA and epilogue warps through a small shared-memory queue; -1 ends.
  // Returns the i-th claimed tile for a consumer role (-1: none left or a wait gave up).
  auto next_tile = [&](int i) -> int {
    const int q = i % TM_TQ;
    if (!mbar_wait(&qfull[q], (i / TM_TQ) & 1)) return -1;
    return tileq[q];
  };

  if (warp == 4) {
    // ------------------------------------------------------------ TMA producer
    if (lane == 0) {
      int c = 0;
      for (int i = 0;; ++i) {
        const int q = i % TM_TQ;
        if (i >= TM_TQ && !mbar_wait(&qempty[q], ((i / TM_TQ) - 1) & 1)) {
          atomicExch(a.err, 4);
          *abort_flag = 1;
        }
        int t = *abort_flag ? -1 : atomicAdd(a.ctr, 1);
        if (t >= tiles) t = -1;
        tileq[q] = t;
        mbar_arrive(&qfull[q]);
        if (t < 0) break;
        const int p = t / a.nblk;
        const TmBlock blk = tm_block_of(t - p * a.nblk, N, a.nmain);
        const int npad = (blk.ncols + 15) & ~15;
        const int nbox = blk.strip ? 1 : (npad + TM_BOX - 1) / TM_BOX;
        const uint32_t bbox = blk.strip ? (uint32_t)a.sbox * 128u : (uint32_t)TM_BOX * 128u;
        const uint32_t tx = 2u * (TM_TILE_A + (uint32_t)nbox * bbox);
        const void* bh = blk.strip ? (const void*)&smap_hi : (const void*)&map_hi;
        const void* bl = blk.strip ? (const void*)&smap_lo : (const void*)&map_lo;
        bool ok = true;
        for (int k = 0; k < nch; ++k, ++c) {
          const int s = c % TM_STAGES;
          if (c >= TM_STAGES && !mbar_wait(&empty[s], ((c / TM_STAGES) - 1) & 1)) {
            atomicExch(a.err, 4);
            *abort_flag = 1;
            ok = false;
            break;
          }
          const uint32_t st = sbase + s * STAGE;
          const uint32_t fb = smem_u32(&full[s]);
          mbar_expect_tx(&full[s], tx);
          const int kc = k * 64;
          tma_load_3d(st, &map_hi, kc, blk.arow, p, fb);
          for (int q = 0; q < nbox; ++q) tma_load_3d(st + TM_TILE_A + q * TM_BOX * 128, bh, kc, blk.brow + q * TM_BOX, p, fb);
          const uint32_t lo = st + TM_TILE_A + TM_TILE_B;
          tma_load_3d(lo, &map_lo, kc, blk.arow, p, fb);
          for (int q = 0; q < nbox; ++q) tma_load_3d(lo + TM_TILE_A + q * TM_BOX * 128, bl, kc, blk.brow + q * TM_BOX, p, fb);
        }
        if (!ok) break;
      }
      // the last loads have landed before the CTA may exit (at once unless a
      // wait above gave up with copies in flight)
      for (int q = c > TM_STAGES ? c - TM_STAGES : 0; q < c; ++q) mbar_wait(&full[q % TM_STAGES], (q / TM_STAGES) & 1);
    }
  } else if (warp == 5) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      int c = 0;
      for (int i = 0;; ++i) {
        const int t = *abort_flag ? -1 : next_tile(i);
        if (t < 0) break;
        const int p = t / a.nblk;
        const TmBlock blk = tm_block_of(t - p * a.nblk, N, a.nmain);
        const int npad = (blk.ncols + 15) & ~15;
        const uint32_t idesc = umma_idesc_bf16(npad);
        const int b = i & 1;
        if (i >= 2 && !mbar_wait(&tempty[b], ((i >> 1) - 1) & 1)) {
          atomicExch(a.err, 5);
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        const uint32_t acc = taddr + (uint32_t)(b * TM_BN);
        bool ok = true;
        for (int k = 0; k < nch; ++k, ++c) {
          const int s = c % TM_STAGES;
          if (!mbar_wait(&full[s], (c / TM_STAGES) & 1)) {
            atomicExch(a.err, 5);
            *abort_flag = 1;
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t st = sbase + s * STAGE;
          const uint32_t ahi = st, bhi = st + TM_TILE_A, alo = st + TM_TILE_A + TM_TILE_B, blo = alo + TM_TILE_A;
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
    for (int i = 0;; ++i) {
      // warp 0 takes the tile index and the tile's accumulator; the others follow at the barrier
      int t = -1;
      if (warp == 0) {
        t = *abort_flag ? -1 : next_tile(i);
        if (lane == 0) {
          tileq_epi[0] = t;
          if (t >= 0 && !mbar_wait(&tfull[i & 1], (i >> 1) & 1)) {
            atomicExch(a.err, 6);
            *epi_abort = 1;
          }
          if (t >= 0) mbar_arrive(&qempty[i % TM_TQ]);  // the index has been read by every role
        }
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");
      t = tileq_epi[0];
      if (t < 0 || *epi_abort) break;  // the same decision in all four warps
      const int p = t / a.nblk;
      const TmBlock blk = tm_block_of(t - p * a.nblk, N, a.nmain);
      const int npad = (blk.ncols + 15) & ~15;
      const int b = i & 1;
      tc_fence_after();
      float* out = a.out + (int64_t)p * a.out_stride;
      const int row = blk.arow + warp * 32 + lane;
      const uint32_t lane_addr = taddr + (uint32_t)(b * TM_BN) + ((uint32_t)(warp * 32) << 16);
      for (int cc = 0; cc < npad; cc += 16) {
        float v[16];
        tmem_ld16(lane_addr + cc, v);
        tm_store(a, blk, out, row, cc, v);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[b]);
      asm volatile("bar.sync 1, 128;" ::: "memory");  // tileq_epi is free for the next tile
    }
  }
  __syncwarp();
  // every MMA has completed before TMEM is released
  if (warp == 0) {
    const bool ok = mbar_wait(done, 0);
    if (!ok && lane == 0) atomicExch(a.err, 6);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(taddr, 512);
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace {
using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
std::mutex g_enc_mu;
EncodeFn g_encode = nullptr;

cudaError_t get_encode(EncodeFn* fn) {
  std::lock_guard<std::mutex> lk(g_enc_mu);
  if (!g_encode) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
    if (e != cudaSuccess) return e;
    if (q != cudaDriverEntryPointSuccess || !p) return cudaErrorNotSupported;
    g_encode = reinterpret_cast<EncodeFn>(p);
  }
  *fn = g_encode;
  return cudaSuccess;
}

}  // namespace

// 3D bf16 map over [depth][rows][inner] (inner contiguous, a multiple of 64):
// box 64 x 128 x 1, 128-byte swizzle (the K-major operand layout of tcgen05).
// Rows past `rows` read as zeros.
cudaError_t make_bf16_map(CUtensorMap* m, const void* base, int64_t inner, int64_t rows, int64_t depth,
                          int box_rows) {
  EncodeFn enc;
  cudaError_t e = get_encode(&enc);
  if (e != cudaSuccess) return e;
  cuuint64_t dims[3] = {(cuuint64_t)inner, (cuuint64_t)rows, (cuuint64_t)depth};
  cuuint64_t strides[2] = {(cuuint64_t)inner * 2, (cuuint64_t)inner * 2 * rows};
  cuuint32_t box[3] = {64, (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

namespace {
size_t tm_smem() {
  return 1024 + TM_STAGES * (size_t)2 * (TM_TILE_A + TM_TILE_B) + (2 * TM_STAGES + 5 + 2 * TM_TQ) * 8 +
         TM_TQ * 4 + 32;
}
}  // namespace

PackedLayout packed_layout(int n, bool cplx, int M, bool synth_tc, int count) {
  PackedLayout L{};
  L.N = cplx ? 2 * n : n;
  L.kp = pack_k(M);
  L.kn = pack_k(L.N);
  L.synth_tc = synth_tc;
  const int64_t gram_el = (int64_t)L.N * L.kp, rows_el = L.kp * L.kn, coef_el = (int64_t)L.N * L.kn;
  L.hi = 0;
  L.lo = L.hi + count * gram_el;
  L.rows_hi = L.lo + count * gram_el;
  L.rows_lo = L.rows_hi + (synth_tc ? count * rows_el : 0);
  L.coef_hi = L.rows_lo + (synth_tc ? count * rows_el : 0);
  L.coef_lo = L.coef_hi + (synth_tc ? count * coef_el : 0);
  L.total = L.coef_lo + (synth_tc ? count * coef_el : 0);
  return L;
}

size_t packed_bytes_per_patch(int n, bool cplx, int M, bool synth_tc) {
  return (size_t)packed_layout(n, cplx, M, synth_tc, 1).total * sizeof(__nv_bfloat16);
}

cudaError_t launch_gram_packed(const Geo& g, bool cplx, const void* in, const PatchWork& w, void* packed,
                               cudaStream_t s, bool synth_tc) {
  const PackedLayout L = packed_layout(g.cols, cplx, g.rows, synth_tc, w.count);
  const int N = L.N;
  const int64_t kp = L.kp;
  __nv_bfloat16* base = reinterpret_cast<__nv_bfloat16*>(packed);
  __nv_bfloat16* hi = base + L.hi;
  __nv_bfloat16* lo = base + L.lo;
  __nv_bfloat16* rhi = synth_tc ? base + L.rows_hi : nullptr;
  __nv_bfloat16* rlo = synth_tc ? base + L.rows_lo : nullptr;
  // K segments per column tile: enough CTAs for about eight waves of 8 per SM
  const int64_t ktiles = kp / PK_R, ctiles = (N + PK_C - 1) / PK_C;
  const int ks = (int)std::min<int64_t>(ktiles, std::max<int64_t>(1, (148 * 8 * 8) / ((int64_t)w.count * ctiles)));
  // strips when N has whole 128-row blocks and a remainder
  const int nmain = (N >= TM_BM && N % TM_BM != 0) ? N / TM_BM * TM_BM : N;
  const int sbox = nmain < N ? ((N - nmain + 15) & ~15) : 0;
  if ((int64_t)w.count * ctiles * ks > INT32_MAX || (int64_t)w.count * tm_blocks(N, nmain) > INT32_MAX)
    return cudaErrorInvalidConfiguration;
  const unsigned pg = (unsigned)(w.count * ctiles * ks);
  PD_TIMED("pack", s,
           k_pack_patches<<<pg, 256, 0, s>>>(g, (const float*)in, N, cplx ? 1 : 0, w.mean, w.list, hi, lo, kp, ks,
                                             rhi, rlo, L.kn));
  CUtensorMap mh, ml;
  cudaError_t e = make_bf16_map(&mh, hi, kp, N, w.count);
  if (e != cudaSuccess) return e;
  e = make_bf16_map(&ml, lo, kp, N, w.count);
  if (e != cudaSuccess) return e;
  CUtensorMap sh = mh, sl = ml;  // the strip's narrow B boxes
  if (sbox) {
    e = make_bf16_map(&sh, hi, kp, N, w.count, sbox);
    if (e != cudaSuccess) return e;
    e = make_bf16_map(&sl, lo, kp, N, w.count, sbox);
    if (e != cudaSuccess) return e;
  }
  TmaArgs a{};
  a.N = N;
  a.n_out = g.cols;
  a.cplx = cplx ? 1 : 0;
  a.kp = kp;
  a.nmain = nmain;
  a.sbox = sbox;
  a.nblk = tm_blocks(N, nmain);
  a.out = w.gram;
  a.out_stride = w.gram_stride;
  a.err = w.err;
  const size_t smem = tm_smem();
  e = cudaFuncSetAttribute(k_gram_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  a.count = w.count;
  a.ctr = w.ctr;
  if (cudaError_t ez = cudaMemsetAsync(w.ctr, 0, sizeof(int), s); ez != cudaSuccess) return ez;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const unsigned grid = (unsigned)std::min<int64_t>((int64_t)w.count * a.nblk, sms);
  PD_TIMED("gram_tc", s, k_gram_tma<<<grid, TM_THREADS, smem, s>>>(mh, ml, sh, sl, a));
  return cudaGetLastError();
}

}  // namespace pd
