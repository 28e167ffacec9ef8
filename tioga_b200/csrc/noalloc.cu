// Donor-stencil interpolation of device-resident fields that allocates no
// device memory.
//
// Who needs it: a solver that advances its time step inside a captured CUDA
// graph cannot call cudaMalloc (allocation is not allowed while a stream is
// being captured and would invalidate the capture), and a solver that hands
// all device memory to its own pool allocator cannot afford one either,
// because cudaMalloc synchronises the whole device and stalls its other
// streams in the middle of the time step.  Such a caller owns the stencils
// and the fields; this entry point only needs a staging area between the
// gather and the scatter, and it keeps that in a fixed device array.
//
// The staging array is file-scope device memory of kNoAllocMaxValues doubles
// (8 MiB).  Every GPU that loads the library holds it until the process
// exits.  All calls share it: two calls that run at the same time on the GPU
// (different streams, or different host threads) race on it and must be
// serialised by the caller, e.g. by issuing them on one stream.  A call fully
// writes every staging slot it later reads, so nothing is carried over from
// the previous call and nothing needs clearing.
//
// Stencils hold 1 to 8 weights (d_nweights[r]); a record outside that range is
// ignored (its receptor keeps its value) rather than summed in part.  Receptor
// entries must be distinct, as tioga_getdonorinfo_'s are: two records that name
// the same receptor node would race in the scatter.
#include <stdio.h>

#include <mutex>

#include "common.cuh"

namespace {

constexpr long long kNoAllocMaxValues = 1ll << 20;  // nrec * nvar at most
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_vals[kNoAllocMaxValues];

// Device address of g_noalloc_vals per device ordinal.  In host code the
// symbol's name is only a host-side stand-in, so the address is looked up once
// per device with cudaGetSymbolAddress while that device is current; the
// mutex makes the first calls of several host threads on one device safe.
double* g_noalloc_ptr[kMaxDevices] = {nullptr};
std::mutex g_noalloc_mu;

// qq[k] = sum over the stencil of q[donor, k] * w, accumulated from 0 in
// stencil order (the same order as the reference's getInterpolatedSolution,
// src/dataUpdate.C:50-57), so the result is bit-identical to
// tioga_dataupdate_mb_.
__global__ void k_noalloc_gather(const int* __restrict__ inode, const double* __restrict__ w,
                                 const int* __restrict__ nw, int nrec, const double* __restrict__ q,
                                 long long nnodes, int nvar, int interptype, double* __restrict__ vals) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrec; r += gridDim.x * blockDim.x) {
    const int n = nw[r];
    if (n < 1 || n > 8) continue;  // ignored record (k_noalloc_scatter skips it too)
    for (int k = 0; k < nvar; k++) {
      double acc = 0;
      for (int m = 0; m < n; m++) {
        const long long node = inode[9 * (long long)r + m];
        const double qv = (interptype == 0) ? q[node * nvar + k] : q[(long long)k * nnodes + node];
        acc += qv * w[9 * (long long)r + m];
      }
      vals[(long long)r * nvar + k] = acc;
    }
  }
}

__global__ void k_noalloc_scatter(const int* __restrict__ recv, const int* __restrict__ nw, int nrec,
                                  const double* __restrict__ vals, long long nnodes, int nvar, int interptype,
                                  double* __restrict__ q) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrec; r += gridDim.x * blockDim.x) {
    if (nw[r] < 1 || nw[r] > 8) continue;
    const long long node = recv[r];
    for (int k = 0; k < nvar; k++) {
      const double v = vals[(long long)r * nvar + k];
      if (interptype == 0) q[node * nvar + k] = v;
      else q[(long long)k * nnodes + node] = v;
    }
  }
}

}  // namespace

#pragma GCC visibility push(default)
extern "C" int tioga_b200_interpolate_noalloc_(const int* d_inode, const double* d_weights,
                                               const int* d_nweights, const int* d_receptor, int nrec,
                                               double* d_q, long long nnodes, int nvar, int interptype,
                                               void* stream) {
  if (nrec < 0 || nvar < 1 || nnodes < 1 || (interptype != 0 && interptype != 1)) {
    fprintf(stderr, "#tioga_b200: interpolate_noalloc: bad arguments (nrec %d, nvar %d, nnodes %lld, "
                    "interptype %d)\n", nrec, nvar, nnodes, interptype);
    return -1;
  }
  if ((long long)nrec * nvar > kNoAllocMaxValues) {
    fprintf(stderr, "#tioga_b200: interpolate_noalloc: nrec*nvar = %lld exceeds the fixed staging "
                    "capacity of %lld values\n", (long long)nrec * nvar, kNoAllocMaxValues);
    return -1;
  }
  if (nrec == 0) return 0;
  if (!d_inode || !d_weights || !d_nweights || !d_receptor || !d_q) {
    fprintf(stderr, "#tioga_b200: interpolate_noalloc: null array\n");
    return -1;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    fprintf(stderr, "#tioga_b200: interpolate_noalloc: no usable current device (%s)\n",
            cudaGetErrorString(e));
    return -2;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* vals = nullptr;
  {
    // set-up on the first call on this device: make that call before any
    // stream capture begins
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_vals);
      if (e != cudaSuccess || !p) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(st, &cs);
        fprintf(stderr, "#tioga_b200: interpolate_noalloc: cudaGetSymbolAddress failed: %s%s\n",
                cudaGetErrorString(e),
                cs != cudaStreamCaptureStatusNone
                    ? " (this was the first call on the device and a stream capture is active: make one call "
                      "before capturing)"
                    : "");
        return -2;
      }
      g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    vals = g_noalloc_ptr[dev];
  }
  const int threads = 128;
  const int blocks = tb::grid_for(nrec, threads);
  k_noalloc_gather<<<blocks, threads, 0, st>>>(d_inode, d_weights, d_nweights, nrec, d_q, nnodes, nvar,
                                               interptype, vals);
  k_noalloc_scatter<<<blocks, threads, 0, st>>>(d_receptor, d_nweights, nrec, vals, nnodes, nvar, interptype,
                                                d_q);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "#tioga_b200: interpolate_noalloc: launch failed: %s\n", cudaGetErrorString(e));
    return -2;
  }
  return 0;
}
#pragma GCC visibility pop
