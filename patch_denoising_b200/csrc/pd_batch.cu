// Batched calls: the work list of many volumes and the table the patch kernels
// read their volume from (PatchWork::vols / vol_of).
#include "pd_common.cuh"
#include "pd_kernels.cuh"
#include "pd_profile.cuh"

namespace pd {

// Copies the volume table into device memory and concatenates the volumes'
// patch lists: list[first_v + i] = list_v[i], vol_of[first_v + i] = v.
__global__ void k_batch_setup(BatchTable t, int nv, int64_t total, VolDesc* vols, int32_t* list, int32_t* vol_of) {
  if (blockIdx.x == 0)
    for (int v = threadIdx.x; v < nv; v += blockDim.x) vols[v] = t.v[v].d;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    int v = 0;
    while (v + 1 < nv && t.v[v + 1].d.first <= i) ++v;
    list[i] = t.v[v].list[i - t.v[v].d.first];
    vol_of[i] = v;
  }
}

void launch_batch_setup(const BatchTable& t, int nv, int64_t total, VolDesc* vols, int32_t* list, int32_t* vol_of,
                        cudaStream_t s) {
  int64_t blocks = (total + 255) / 256;
  if (blocks < 1) blocks = 1;
  if (blocks > 148 * 8) blocks = 148 * 8;
  PD_TIMED("batch_setup", s, k_batch_setup<<<(int)blocks, 256, 0, s>>>(t, nv, total, vols, list, vol_of));
}

}  // namespace pd
