// Opt-in launch timing: PD_TIMED(name, stream, launch) brackets a kernel launch
// with CUDA events when profiling is enabled.
#pragma once
#include <cuda_runtime.h>

namespace pd {
bool profile_on();
void profile_begin(const char* name, cudaStream_t s);
void profile_end(cudaStream_t s);
}  // namespace pd

#define PD_TIMED(name, stream, ...)                        \
  do {                                                     \
    const bool _pd_on = ::pd::profile_on();                \
    if (_pd_on) ::pd::profile_begin((name), (stream));     \
    __VA_ARGS__;                                           \
    if (_pd_on) ::pd::profile_end((stream));               \
  } while (0)
