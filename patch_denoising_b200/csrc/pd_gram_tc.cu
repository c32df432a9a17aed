// Tensor-core (tcgen05) centred Gram for the mixed-precision path.
//
// C = X^T X for X = the centred Casorati matrix of a patch (M rows x N columns;
// a complex patch is its interleaved real view with N = 2 n, and the complex
// Gram is recombined from 2x2 blocks in the epilogue:
//   C_ij = (G[2i][2j] + G[2i+1][2j+1]) + i (G[2i][2j+1] - G[2i+1][2j])).
// Each CTA owns a 128-row x (<= 256)-column block of the lower block triangle:
//   producer warps 0-7 gather 64 patch rows per stage from the volume (coalesced
//   along frames), subtract the mean, split each value into bf16 hi (+ bf16 lo
//   when split = 3) and store K-major 128-byte-swizzled operand tiles;
//   warp 8 (one thread) issues tcgen05.mma (M = 128, N <= 256, K = 16) with the
//   accumulator in TMEM and signals stage reuse through tcgen05.commit;
//   warps 0-3 read the accumulator with tcgen05.ld and write the packed Gram.
// split = 3 computes hi*hi + hi*lo + lo*hi (about 16 significant bits per
// product), split = 1 the plain bf16 product.
//
// The same kernel computes the Gram of a dense row-major matrix (the NORDIC
// Monte-Carlo draws) over row chunks, writing one partial Gram per chunk.
#include "pd_common.cuh"
#include "pd_kernels.cuh"
#include "pd_profile.cuh"
#include "pd_tc.cuh"

namespace pd {

constexpr int TC_KC = 64;  // K rows per stage (one 128-byte swizzle atom of bf16)
constexpr int TC_PROD = 256;
constexpr int TC_THREADS = TC_PROD + 32;
constexpr int TC_BM = 128;
constexpr int TC_BN = 256;
constexpr int TC_STAGES = 2;
constexpr uint32_t TILE_A = TC_BM * 128;  // bytes of a 128-row tile
constexpr uint32_t TILE_B = TC_BN * 128;

struct TcArgs {
  Geo g;
  const float* in;  // volume (patch mode) or dense matrix, as floats
  int N;            // real columns
  int n_out;        // output matrix order (N, or N/2 for complex)
  int cplx;
  int split;
  int dense;
  const float* mean;  // patch mode: N floats per patch
  const int32_t* list;
  float* out;  // packed lower output(s)
  int64_t out_stride;
  int64_t rows;          // dense: total rows
  int64_t rows_per_cta;  // dense: rows per chunk
  int* err;
};


__device__ __forceinline__ void block_of(int idx, int N, int& rb, int& nb, int& ncols) {
  for (rb = 0;; ++rb) {
    const int lim = min((rb + 1) * TC_BM, N);
    const int nbs = (lim + TC_BN - 1) / TC_BN;
    if (idx < nbs) {
      nb = idx;
      ncols = min(lim - nb * TC_BN, TC_BN);
      return;
    }
    idx -= nbs;
  }
}

__host__ inline int blocks_per_gram(int N) {
  int t = 0;
  for (int rb = 0; rb * TC_BM < N; ++rb) {
    const int lim = (rb + 1) * TC_BM < N ? (rb + 1) * TC_BM : N;
    t += (lim + TC_BN - 1) / TC_BN;
  }
  return t;
}

__global__ void __launch_bounds__(TC_THREADS, 1) k_gram_tc(TcArgs a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int N = a.N;
  const uint32_t stage_bytes = (a.split == 3 ? 2u : 1u) * (TILE_A + TILE_B);
  float* mean_s = reinterpret_cast<float*>(sm + TC_STAGES * stage_bytes);
  int64_t* rowbase = reinterpret_cast<int64_t*>(mean_s + ((N + 3) & ~3));  // [TC_STAGES][TC_KC]
  uint64_t* bars = reinterpret_cast<uint64_t*>(rowbase + TC_STAGES * TC_KC);
  uint64_t* full = bars;
  uint64_t* empty = bars + TC_STAGES;
  uint64_t* done = bars + 2 * TC_STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  int* ok_flag = reinterpret_cast<int*>(tmem_slot + 1);  // [TC_STAGES]

  int rb, nb, ncols;
  block_of(blockIdx.y, N, rb, nb, ncols);
  const int npad = (ncols + 15) & ~15;
  uint32_t tcols = 32;
  while (tcols < (uint32_t)npad) tcols <<= 1;

  // patch / chunk
  int64_t r_begin = 0, r_end = 0, o[4] = {0, 0, 0, 0};
  const float* mean = nullptr;
  float* out = nullptr;
  if (a.dense) {
    r_begin = (int64_t)blockIdx.x * a.rows_per_cta;
    r_end = min(r_begin + a.rows_per_cta, a.rows);
    out = a.out + ((int64_t)blockIdx.z * gridDim.x + blockIdx.x) * a.out_stride;
  } else {
    const int p = blockIdx.x;
    patch_origin(a.g, a.list[p], o);
    r_end = a.g.rows;
    mean = a.mean + (int64_t)p * N;
    out = a.out + (int64_t)p * a.out_stride;
  }
  const int64_t nrows = r_end - r_begin;
  const int nch = (int)((nrows + TC_KC - 1) / TC_KC);

  if (tid == 0) {
    for (int s = 0; s < TC_STAGES; ++s) {
      mbar_init(&full[s], TC_PROD);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    mbar_fence_init();
  }
  if (warp == 8) {
    tmem_alloc(tmem_slot, tcols);
    tc_fence_before();
  }
  for (int c = tid; c < N; c += TC_THREADS) mean_s[c] = mean ? mean[c] : 0.f;
  __syncthreads();
  tc_fence_after();
  const uint32_t taddr = *tmem_slot;
  const uint32_t sbase = smem_u32(sm);

  if (warp < 8) {
    // ------------------------------------------------------------ producers
    const int ptid = tid;
    const int rowsB = npad;
    const int trows = TC_BM + rowsB;
    for (int c = 0; c < nch; ++c) {
      const int s = c % TC_STAGES;
      if (c >= TC_STAGES) {
        if (ptid == 0) ok_flag[s] = mbar_wait(&empty[s], ((c / TC_STAGES) - 1) & 1) ? 1 : 0;
      } else if (ptid == 0) {
        ok_flag[s] = 1;
      }
      if (ptid < TC_KC) {
        const int64_t r = r_begin + (int64_t)c * TC_KC + ptid;
        int64_t base = -1;
        if (r < r_end) {
          if (a.dense)
            base = r * N;
          else
            base = (row_voxel(a.g, o, (int)r) * a.g.shape[3] + o[3]) * (a.cplx ? 2 : 1);
        }
        rowbase[s * TC_KC + ptid] = base;
      }
      asm volatile("bar.sync 1, 256;" ::: "memory");
      if (!ok_flag[s]) {
        if (ptid == 0) atomicExch(a.err, 1);
        break;
      }
      uint8_t* st = sm + s * stage_bytes;
      const int64_t* rbs = rowbase + s * TC_KC;
      auto store8 = [&](int row, int g8, bool isA, const float x[8]) {
        uint4 hi;
        hi.x = pack_bf16(x[0], x[1]);
        hi.y = pack_bf16(x[2], x[3]);
        hi.z = pack_bf16(x[4], x[5]);
        hi.w = pack_bf16(x[6], x[7]);
        const uint32_t off = sw128_off(row, g8) + (isA ? 0u : TILE_A);
        *reinterpret_cast<uint4*>(st + off) = hi;
        if (a.split == 3) {
          const __nv_bfloat162* hp = reinterpret_cast<const __nv_bfloat162*>(&hi);
          float l[8];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const float2 f = __bfloat1622float2(hp[q]);
            l[2 * q] = x[2 * q] - f.x;
            l[2 * q + 1] = x[2 * q + 1] - f.y;
          }
          uint4 lo;
          lo.x = pack_bf16(l[0], l[1]);
          lo.y = pack_bf16(l[2], l[3]);
          lo.z = pack_bf16(l[4], l[5]);
          lo.w = pack_bf16(l[6], l[7]);
          *reinterpret_cast<uint4*>(st + TILE_A + TILE_B + off) = lo;
        }
      };
      // tasks: one tile row (an X column) x 8 K rows
      for (int task = ptid; task < trows * 8; task += TC_PROD) {
        const int trow = task % trows, g8 = task / trows;
        const bool isA = trow < TC_BM;
        const int row = isA ? trow : trow - TC_BM;
        const int col = isA ? rb * TC_BM + row : nb * TC_BN + row;
        const bool colok = col < N && (isA || row < ncols);
        float x[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int64_t base = rbs[g8 * 8 + q];
          x[q] = (colok && base >= 0) ? __ldg(a.in + base + col) - mean_s[col] : 0.f;
        }
        store8(row, g8, isA, x);
      }
      fence_async_smem();
      mbar_arrive(&full[s]);
    }
  } else if (lane == 0) {
    // ------------------------------------------------------------ MMA issuer
    const uint32_t idesc = umma_idesc_bf16(npad);
    bool ok = true;
    for (int c = 0; c < nch && ok; ++c) {
      const int s = c % TC_STAGES;
      if (!mbar_wait(&full[s], (c / TC_STAGES) & 1)) {
        ok = false;
        atomicExch(a.err, 2);
        break;
      }
      tc_fence_after();
      const uint32_t st = sbase + s * stage_bytes;
      const uint32_t ahi = st, bhi = st + TILE_A, alo = st + TILE_A + TILE_B, blo = alo + TILE_A;
#pragma unroll
      for (int k = 0; k < TC_KC / 16; ++k) {
        const uint32_t kb = k * 32;
        const uint64_t da = umma_desc_sw128(ahi + kb), db = umma_desc_sw128(bhi + kb);
        umma_bf16(taddr, da, db, idesc, (c | k) != 0 ? 1u : 0u);
        if (a.split == 3) {
          umma_bf16(taddr, da, umma_desc_sw128(blo + kb), idesc, 1u);
          umma_bf16(taddr, umma_desc_sw128(alo + kb), db, idesc, 1u);
        }
      }
      umma_commit(&empty[s]);
    }
    umma_commit(done);
  }

  // ------------------------------------------------------------ epilogue
  if (warp < 4) {
    const bool ok = mbar_wait(done, 0);
    __syncwarp();
    tc_fence_after();
    if (!ok && lane == 0) atomicExch(a.err, 3);
    const int i = rb * TC_BM + warp * 32 + lane;  // row of the real Gram
    const uint32_t lane_addr = taddr + ((uint32_t)(warp * 32) << 16);
    for (int cc = 0; cc < npad; cc += 16) {
      float v[16];
      tmem_ld16(lane_addr + cc, v);
      if (!a.cplx) {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const int j = nb * TC_BN + cc + q;
          if (ok && i < N && j <= i && (cc + q) < ncols) out[pk(i, j, N)] = v[q];
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
            const int jc = (nb * TC_BN + cc + q) >> 1;
            if (ok && ic < n && jc <= ic && (cc + q) < ncols)
              oc[pk(ic, jc, n)] = cf{v[q] + vp[q + 1], v[q + 1] - vp[q]};
          }
        }
      }
    }
    tc_fence_before();
  }
  __syncthreads();
  if (warp == 8) {
    tc_fence_after();
    tmem_dealloc(taddr, tcols);
  }
}

static size_t tc_smem(int N, int split) {
  const size_t stage = (split == 3 ? 2 : 1) * (size_t)(TILE_A + TILE_B);
  return 1024 + TC_STAGES * stage + sizeof(float) * ((N + 3) & ~3) + sizeof(int64_t) * TC_STAGES * TC_KC +
         sizeof(uint64_t) * (2 * TC_STAGES + 1) + 16 + 4 * TC_STAGES;
}

cudaError_t launch_gram_tc(const Geo& g, bool cplx, const void* in, const PatchWork& w, int split, int* err,
                           cudaStream_t s) {
  TcArgs a{};
  a.g = g;
  a.in = (const float*)in;
  a.N = cplx ? 2 * g.cols : g.cols;
  a.n_out = g.cols;
  a.cplx = cplx ? 1 : 0;
  a.split = split;
  a.dense = 0;
  a.mean = w.mean;
  a.list = w.list;
  a.out = w.gram;
  a.out_stride = w.gram_stride;
  a.err = err;
  const size_t smem = tc_smem(a.N, split);
  cudaError_t e = cudaFuncSetAttribute(k_gram_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid(w.count, blocks_per_gram(a.N));
  PD_TIMED("gram_tc", s, k_gram_tc<<<grid, TC_THREADS, smem, s>>>(a));
  return cudaGetLastError();
}

// Gram of a dense row-major rows x cols matrix, one packed partial per row chunk.
cudaError_t launch_dense_gram_tc(const float* mat, int64_t rows, int cols, int64_t rows_per_cta, float* part,
                                 int64_t part_stride, int split, int* err, cudaStream_t s) {
  TcArgs a{};
  a.in = mat;
  a.N = cols;
  a.n_out = cols;
  a.split = split;
  a.dense = 1;
  a.out = part;
  a.out_stride = part_stride;
  a.rows = rows;
  a.rows_per_cta = rows_per_cta;
  a.err = err;
  const size_t smem = tc_smem(cols, split);
  cudaError_t e = cudaFuncSetAttribute(k_gram_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int64_t chunks = (rows + rows_per_cta - 1) / rows_per_cta;
  dim3 grid((unsigned)chunks, blocks_per_gram(cols), 1);
  PD_TIMED("mc_gram_tc", s, k_gram_tc<<<grid, TC_THREADS, smem, s>>>(a));
  return cudaGetLastError();
}

}  // namespace pd
