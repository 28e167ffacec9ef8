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
#include <stdio.h>

#include "common.cuh"

namespace {

constexpr long long kNoAllocMaxValues = 1ll << 20;  // nrec * nvar at most
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_vals[kNoAllocMaxValues];

// Device address of g_noalloc_vals per device ordinal.  In host code the
// symbol's name is only a host-side stand-in, so the address is looked up once
// per device with cudaGetSymbolAddress while that device is current.
double* g_noalloc_ptr[kMaxDevices] = {nullptr};

// qq[k] = sum over the stencil of q[donor, k] * w, accumulated from 0 in
// stencil order (the same order as the reference's getInterpolatedSolution,
// src/dataUpdate.C:50-57), so the result is bit-identical to
// tioga_dataupdate_mb_.
__global__ void k_noalloc_gather(const int* __restrict__ inode, const double* __restrict__ w,
                                 const int* __restrict__ nw, int nrec, const double* __restrict__ q,
                                 long long nnodes, int nvar, int interptype, double* __restrict__ vals) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrec; r += gridDim.x * blockDim.x) {
    const int n = nw[r];
    for (int k = 0; k < nvar; k++) {
      double acc = 0;
      for (int m = 0; m < n && m < 8; m++) {
        const long long node = inode[9 * (long long)r + m];
        const double qv = (interptype == 0) ? q[node * nvar + k] : q[(long long)k * nnodes + node];
        acc += qv * w[9 * (long long)r + m];
      }
      vals[(long long)r * nvar + k] = acc;
    }
  }
}

__global__ void k_noalloc_scatter(const int* __restrict__ recv, int nrec, const double* __restrict__ vals,
                                  long long nnodes, int nvar, int interptype, double* __restrict__ q) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrec; r += gridDim.x * blockDim.x) {
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
  if (!g_noalloc_ptr[dev]) {
    // set-up on the first call on this device (make it before any capture)
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_vals);
    if (e != cudaSuccess || !p) {
      fprintf(stderr, "#tioga_b200: interpolate_noalloc: cudaGetSymbolAddress failed: %s\n",
              cudaGetErrorString(e));
      return -2;
    }
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int threads = 128;
  const int blocks = tb::grid_for(nrec, threads);
  k_noalloc_gather<<<blocks, threads, 0, st>>>(d_inode, d_weights, d_nweights, nrec, d_q, nnodes, nvar,
                                               interptype, g_noalloc_ptr[dev]);
  k_noalloc_scatter<<<blocks, threads, 0, st>>>(d_receptor, nrec, g_noalloc_ptr[dev], nnodes, nvar,
                                                interptype, d_q);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "#tioga_b200: interpolate_noalloc: launch failed: %s\n", cudaGetErrorString(e));
    return -2;
  }
  return 0;
}
#pragma GCC visibility pop
