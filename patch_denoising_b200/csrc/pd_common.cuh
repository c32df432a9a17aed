// Common device-side definitions for the sm_100a denoising kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/patch_denoise_b200.h"

namespace pd {

// ---------------------------------------------------------------------------
// Scalars: real float or interleaved complex float (complex64).
// ---------------------------------------------------------------------------
struct cf {
  float x, y;
};

__host__ __device__ __forceinline__ cf mk(float a, float b) { return cf{a, b}; }
__device__ __forceinline__ cf operator+(cf a, cf b) { return cf{a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ cf operator-(cf a, cf b) { return cf{a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ cf operator*(cf a, float s) { return cf{a.x * s, a.y * s}; }
__device__ __forceinline__ cf operator*(cf a, cf b) {
  return cf{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}

// conj helpers (identity for real)
__device__ __forceinline__ float cj(float a) { return a; }
__device__ __forceinline__ cf cj(cf a) { return cf{a.x, -a.y}; }
__device__ __forceinline__ float re(float a) { return a; }
__device__ __forceinline__ float re(cf a) { return a.x; }
__device__ __forceinline__ float abs2(float a) { return a * a; }
__device__ __forceinline__ float abs2(cf a) { return a.x * a.x + a.y * a.y; }
template <class T>
__device__ __forceinline__ T zero();
template <>
__device__ __forceinline__ float zero<float>() { return 0.f; }
template <>
__device__ __forceinline__ cf zero<cf>() { return cf{0.f, 0.f}; }
// conj(a) * b
__device__ __forceinline__ float cmulc(float a, float b) { return a * b; }
__device__ __forceinline__ cf cmulc(cf a, cf b) {
  return cf{a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x};
}
// a * b (no conj), real scale
__device__ __forceinline__ float mul(float a, float b) { return a * b; }
__device__ __forceinline__ cf mul(cf a, cf b) { return a * b; }
__device__ __forceinline__ float scal(float a, float s) { return a * s; }
__device__ __forceinline__ cf scal(cf a, float s) { return cf{a.x * s, a.y * s}; }

template <bool CPLX>
struct Elem {
  using T = float;
};
template <>
struct Elem<true> {
  using T = cf;
};

// ---------------------------------------------------------------------------
// Geometry passed by value to kernels.
// ---------------------------------------------------------------------------
struct Geo {
  int64_t shape[4];
  int64_t patch[4];
  int64_t step[4];
  int64_t grid[4];
  int64_t n_patches;
  int32_t rows;  // M
  int32_t cols;  // frames per patch (n of the T-Gram)
};

__host__ __device__ __forceinline__ Geo to_geo(const pd_geometry& g) {
  Geo o;
  for (int i = 0; i < 4; ++i) {
    o.shape[i] = g.shape[i];
    o.patch[i] = g.patch[i];
    o.step[i] = g.step[i];
    o.grid[i] = g.grid[i];
  }
  o.n_patches = g.n_patches;
  o.rows = (int32_t)g.rows;
  o.cols = (int32_t)g.cols;
  return o;
}

// Origin (x0, y0, z0, t0) of linear patch index idx (C-order unravel over grid).
__device__ __forceinline__ void patch_origin(const Geo& g, int64_t idx, int64_t o[4]) {
  int64_t r = idx;
  int64_t gi[4];
  for (int d = 3; d >= 0; --d) {
    gi[d] = r % g.grid[d];
    r /= g.grid[d];
  }
  for (int d = 0; d < 4; ++d) o[d] = gi[d] * g.step[d];
}

// Time-window index of linear patch idx (its grid coordinate along t).
__device__ __forceinline__ int64_t patch_window(const Geo& g, int64_t idx) {
  return idx % g.grid[3];
}

// Linear voxel (x,y,z) index of Casorati row r of a patch with origin o.
__device__ __forceinline__ int64_t row_voxel(const Geo& g, const int64_t o[4], int r) {
  const int pz = (int)g.patch[2], py = (int)g.patch[1];
  const int k = r % pz;
  const int t = r / pz;
  const int j = t % py;
  const int i = t / py;
  return ((o[0] + i) * g.shape[1] + (o[1] + j)) * g.shape[2] + (o[2] + k);
}

// Packed column-major lower-triangular storage of an n x n Hermitian matrix.
__host__ __device__ __forceinline__ int64_t pk(int i, int j, int n) {
  // requires i >= j
  return (int64_t)j * n - ((int64_t)j * (j - 1)) / 2 + (i - j);
}
__host__ __device__ __forceinline__ int64_t pk_size(int n) { return (int64_t)n * (n + 1) / 2; }

// ---------------------------------------------------------------------------
// Reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ cf warp_sum(cf v) {
  return cf{warp_sum(v.x), warp_sum(v.y)};
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <class T>
__device__ __forceinline__ T shfl_x(T v, int m);
template <>
__device__ __forceinline__ float shfl_x<float>(float v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
template <>
__device__ __forceinline__ cf shfl_x<cf>(cf v, int m) {
  return cf{__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m)};
}

// dp[q] (q < 8) summed over the warp; lane returns (column slot, total) with
// slot = 4*b16 + 2*b8 + b4 valid on lanes with (lane & 3) == 0.
template <class T>
__device__ __forceinline__ T reduce_scatter8(const T dp[8], int lane, int* slot) {
  const bool b16 = lane & 16, b8 = lane & 8, b4 = lane & 4;
  T k4[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const T snd = b16 ? dp[q] : dp[q + 4];
    const T rcv = shfl_x(snd, 16);
    k4[q] = (b16 ? dp[q + 4] : dp[q]) + rcv;
  }
  T k2[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const T snd = b8 ? k4[q] : k4[q + 2];
    const T rcv = shfl_x(snd, 8);
    k2[q] = (b8 ? k4[q + 2] : k4[q]) + rcv;
  }
  const T snd = b4 ? k2[0] : k2[1];
  const T rcv = shfl_x(snd, 4);
  T k1 = (b4 ? k2[1] : k2[0]) + rcv;
  k1 = k1 + shfl_x(k1, 2);
  k1 = k1 + shfl_x(k1, 1);
  *slot = (b16 ? 4 : 0) + (b8 ? 2 : 0) + (b4 ? 1 : 0);
  return k1;
}

// Block-wide sum; red must hold >= 32 entries of T. All threads get the result.
template <class T>
__device__ __forceinline__ T block_sum(T v, T* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  T r = (lane < nw) ? red[lane] : zero<T>();
  r = warp_sum(r);
  return r;
}
template <>
__device__ __forceinline__ double zero<double>() { return 0.0; }

}  // namespace pd
