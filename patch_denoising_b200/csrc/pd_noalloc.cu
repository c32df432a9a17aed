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
// Device address of the scratch array on the current device. Looked up on every
// call (a cheap runtime query once the module is loaded), so the address stays
// right after a device reset or a re-created primary context. The first call
// on a device loads the library's device code there: make it before any stream
// capture.
pd_status scratch_address(void** ptr) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    pd::set_last_error("no usable current CUDA device");
    return PD_ERR_CUDA;
  }
  void* addr = nullptr;
  if (cudaGetSymbolAddress(&addr, g_noalloc_scratch) != cudaSuccess || addr == nullptr) {
    pd::set_last_error("cudaGetSymbolAddress of the static scratch array failed");
    return PD_ERR_CUDA;
  }
  *ptr = addr;
  return PD_OK;
}
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
  void* ptr = nullptr;
  st = scratch_address(&ptr);
  if (st != PD_OK) return st;
  // pd_denoise_patches clears the device error word at the start of every call
  // and fully writes every scratch buffer it reads; calls whose work overlaps on
  // the GPU (other streams, other host threads) share this array and race.
  return pd_denoise_patches(g, p, d_in, d_noise_std, d_patch_list, n_selected, d_out_acc, d_weight_acc, d_noise_acc,
                            d_noise_ctr, d_rank_map, d_patch_rank, d_patch_noise, ptr, PD_NOALLOC_SCRATCH_BYTES,
                            stream);
}

// The device error word of the last pd_denoise_patches_noalloc call on this
// stream (it sits at the start of the static array): pd_workspace_check on it.
extern "C" pd_status pd_noalloc_check(void* stream) {
  void* ptr = nullptr;
  const pd_status st = scratch_address(&ptr);
  if (st != PD_OK) return st;
  return pd_workspace_check(ptr, stream);
}
