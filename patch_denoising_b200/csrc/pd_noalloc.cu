// pd_denoise_patches_noalloc: pd_denoise_patches with its scratch memory in a
// file-scope device array instead of a caller-provided workspace.
//
// Some callers cannot allocate device memory while they denoise: a host
// application that hands the library a fixed device-memory budget it manages
// itself (an inference server's pool, a plugin inside an imaging pipeline), or
// a latency-sensitive loop where cudaMalloc's implicit device synchronisation is
// not acceptable. They still own and pass every input and output buffer; only
// the per-patch scratch (means, Grams, eigenvectors, coefficients, the device
// error word) comes from the static array below.
//
// The array is PD_NOALLOC_SCRATCH_BYTES (32 MiB). Every GPU that loads this
// library keeps it allocated until the process exits. Patches are processed in
// chunks that fit it; a patch geometry whose single-patch scratch exceeds it is
// rejected with PD_ERR_WORKSPACE.
#include <cuda_runtime.h>

#include <mutex>

#include "pd_common.cuh"

#define PD_NOALLOC_SCRATCH_BYTES (32u << 20)

// Device-side scratch shared by every call on a device. Host code must not use
// this symbol as an address: its host-side name is only a stand-in for the
// device array, so the device address is obtained with cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[PD_NOALLOC_SCRATCH_BYTES];

namespace pd {
void set_last_error(const char* msg);
}

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};
}  // namespace

extern "C" pd_status pd_denoise_patches_noalloc(const pd_geometry* g, const pd_params* p, const void* d_in,
                                                const double* d_noise_std, const int32_t* d_patch_list,
                                                int64_t n_selected, void* d_out_acc, float* d_weight_acc,
                                                float* d_noise_acc, float* d_noise_ctr, int32_t* d_rank_map,
                                                int32_t* d_patch_rank, float* d_patch_noise, void* stream) {
  // Per-patch scratch bytes must fit the static array at least once.
  size_t one = 0;
  pd_status st = pd_denoise_workspace_size(g, p, 1, &one);
  if (st != PD_OK) return st;
  if (one > PD_NOALLOC_SCRATCH_BYTES) {
    pd::set_last_error(
        "pd_denoise_patches_noalloc: one patch of this geometry needs more scratch than the 32 MiB static array; "
        "use pd_denoise_patches with a caller-allocated workspace");
    return PD_ERR_WORKSPACE;
  }
  // Device address of the scratch array for the current device, set up once per
  // device (the first call on a device does this; make that call before any
  // stream capture).
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    pd::set_last_error("pd_denoise_patches_noalloc: no usable current CUDA device");
    return PD_ERR_CUDA;
  }
  void* ptr = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
      void* addr = nullptr;
      if (cudaGetSymbolAddress(&addr, g_noalloc_scratch) != cudaSuccess || addr == nullptr) {
        pd::set_last_error("pd_denoise_patches_noalloc: cudaGetSymbolAddress of the static scratch array failed");
        return PD_ERR_CUDA;
      }
      g_scratch_ptr[dev] = addr;
    }
    ptr = g_scratch_ptr[dev];
  }
  // pd_denoise_patches clears the device error word at the start of every call
  // and fully writes every scratch buffer it reads; calls whose work overlaps on
  // the GPU (other streams, other host threads) share this array and race.
  return pd_denoise_patches(g, p, d_in, d_noise_std, d_patch_list, n_selected, d_out_acc, d_weight_acc, d_noise_acc,
                            d_noise_ctr, d_rank_map, d_patch_rank, d_patch_noise, ptr, PD_NOALLOC_SCRATCH_BYTES,
                            stream);
}
