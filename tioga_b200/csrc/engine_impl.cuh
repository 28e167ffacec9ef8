// Helpers shared by the files that implement Engine's host side.
#pragma once

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "kernels.cuh"

namespace tb {

int fail(cudaError_t e);
int sync_check();  // TIOGA_B200_CHECK=1: synchronise after every launch

static const int kT = 256;

// After every launch: a launch error is reported at once; with
// TIOGA_B200_CHECK=1 in the environment the stream is also synchronised so a
// fault is attributed to the kernel that caused it.
#define TB_LAUNCHED(name) TB_LAUNCHED_ON(name, stream_)
#define TB_LAUNCHED_ON(name, st)                                                       \
  do {                                                                                 \
    nlaunch_++;                                                                        \
    cudaError_t le_ = cudaGetLastError();                                              \
    if (le_ == cudaSuccess && sync_check()) le_ = cudaStreamSynchronize(st);           \
    if (le_ != cudaSuccess) {                                                          \
      fprintf(stderr, "#tioga_b200: kernel %s failed: %s\n", name, cudaGetErrorString(le_)); \
      return tb::fail(le_);                                                            \
    }                                                                                  \
  } while (0)

#define TB_TRY(call)      \
  do {                    \
    int rc_ = (call);     \
    if (rc_) return rc_;  \
  } while (0)

}  // namespace tb
