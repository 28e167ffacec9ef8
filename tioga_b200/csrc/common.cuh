// Shared device code for the TIOGA connectivity path on B200 (sm_100a).
//
// Every translation unit that includes this header is compiled with
// -fmad=false: the FP64 routines below evaluate the reference's expressions
// operation by operation in source order, so cell volumes, Newton iterates
// and interpolation weights are bit-identical to the reference's x86-64 build
// (which has no FMA contraction).  FP32 code that wants fused multiply-adds
// calls __fmaf_rn explicitly.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

namespace tb {

constexpr double kBig = 1.0e+15;      // BIGVALUE, src/codetypes.h:52
constexpr double kTol = 1.0e-10;      // TOL, src/codetypes.h:54
constexpr int kHoleMapSize = 192;     // HOLEMAPSIZE, src/codetypes.h:55
constexpr int kBigInt = 2147483647;   // BIGINT, src/codetypes.h:53
constexpr int kMaxNv = 8;
typedef unsigned short blk_t;        // block index of a node or cell

// error word bits (device-side failures are reported, never trapped)
enum : unsigned {
  kErrNone = 0,
  kErrTraversalOverflow = 1u << 0,
  kErrCapacity = 1u << 1,
  kErrWeightRange = 1u << 2,    // a weight outside [-0.2,1.2]: the reference aborts
  kErrFloodFillBound = 1u << 3,
  kErrBadCell = 1u << 4,
  kErrBadIndex = 1u << 5,     // an index outside its array (skipped)
  kErrBadInput = 1u << 6,     // a caller's node index out of range or a non-finite coordinate
};
// error bits after which a connectivity result is not the reference's
constexpr unsigned kErrFatal = kErrTraversalOverflow | kErrCapacity | kErrWeightRange | kErrFloodFillBound |
                               kErrBadIndex | kErrBadInput;

#define TB_CUDA(call)                                                              \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      fprintf(stderr, "#tioga_b200: CUDA error %s at %s:%d: %s\n", #call, __FILE__, \
              __LINE__, cudaGetErrorString(e_));                                   \
      return tb::fail(e_);                                                         \
    }                                                                              \
  } while (0)

int fail(cudaError_t e);

struct Obb {
  double xc[3], dxc[3], vec[3][3];
};

__host__ __device__ inline double dmin(double a, double b) { return (a < b) ? a : b; }
__host__ __device__ inline double dmax(double a, double b) { return (a > b) ? a : b; }

// ---------------------------------------------------------------------------
// src/math.c:25-81 (solvec) -- Gaussian elimination on a 3x3 system, rows
// swapped only when |a_ii| < 1e-8.  Returns 0 for a singular system.
// ---------------------------------------------------------------------------
__host__ __device__ inline int solve3(double a[3][3], double b[3]) {
  const double eps = 1e-8;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    if (fabs(a[i][i]) < eps) {
      int flag = 1;
      for (int k = i + 1; k < 3 && flag; k++) {
        if (a[k][i] != 0) {
          flag = 0;
          for (int l = 0; l < 3; l++) {
            double t = a[k][l];
            a[k][l] = a[i][l];
            a[i][l] = t;
          }
          double t = b[k];
          b[k] = b[i];
          b[i] = t;
        }
      }
      if (flag) return 0;
    }
#pragma unroll
    for (int k = i + 1; k < 3; k++) {
      double fact = -a[k][i] / a[i][i];
#pragma unroll
      for (int j = 0; j < 3; j++) a[k][j] += fact * a[i][j];
      b[k] += fact * b[i];
    }
  }
#pragma unroll
  for (int i = 2; i >= 0; i--) {
    double sum = 0;
    for (int j = i + 1; j < 3; j++) sum += a[i][j] * b[j];
    b[i] = (b[i] - sum) / a[i][i];
  }
  return 1;
}

// src/math.c:83-146 (newtonSolve): start (0.5,0.5,0.5), at most 500
// iterations, stop when ||rhs||_2 <= 1e-14; singular or not converged gives
// u=2 (a reject).  Returns the iteration count (for the statistics).
__host__ __device__ inline int newton64(const double f[8][3], double& uo, double& vo, double& wo) {
  double u = 0.5, v = 0.5, w = 0.5;
  int iter, ok = 1;
  const int itmax = 500;
  for (iter = 0; iter < itmax; iter++) {
    double uv = u * v, vw = v * w, wu = w * u, uvw = u * v * w;
    double rhs[3], lhs[3][3];
#pragma unroll
    for (int j = 0; j < 3; j++)
      rhs[j] = f[0][j] + f[1][j] * u + f[2][j] * v + f[3][j] * w + f[4][j] * uv + f[5][j] * vw +
               f[6][j] * wu + f[7][j] * uvw;
    double norm = rhs[0] * rhs[0] + rhs[1] * rhs[1] + rhs[2] * rhs[2];
    if (sqrt(norm) <= 1e-14) break;
#pragma unroll
    for (int j = 0; j < 3; j++) {
      lhs[j][0] = f[1][j] + f[4][j] * v + f[6][j] * w + f[7][j] * vw;
      lhs[j][1] = f[2][j] + f[5][j] * w + f[4][j] * u + f[7][j] * wu;
      lhs[j][2] = f[3][j] + f[6][j] * u + f[5][j] * v + f[7][j] * uv;
    }
    ok = solve3(lhs, rhs);
    if (!ok) break;
    u -= (rhs[0] * 1.0);
    v -= (rhs[1] * 1.0);
    w -= (rhs[2] * 1.0);
  }
  if (iter == itmax || !ok) {
    u = 2.0;
    v = w = 0.;
  }
  uo = u;
  vo = v;
  wo = w;
  return iter;
}

// src/math.c:149-294 (computeNodalWeights).  xv holds the nvert vertices.
__host__ __device__ inline int nodal_weights64(const double xv[8][3], const double xp[3],
                                               double frac[8], int nvert) {
  double f[8][3], u, v, w;
  int it = 0;
  switch (nvert) {
    case 4: {
      double a[3][3], b[3];
#pragma unroll
      for (int k = 0; k < 3; k++) {
#pragma unroll
        for (int j = 0; j < 3; j++) a[j][k] = xv[k][j] - xv[3][j];
        b[k] = xp[k] - xv[3][k];
      }
      if (solve3(a, b)) {
        frac[0] = b[0];
        frac[1] = b[1];
        frac[2] = b[2];
        frac[3] = 1. - frac[0] - frac[1] - frac[2];
      } else {
        frac[0] = 1.0;
        frac[1] = frac[2] = frac[3] = 0;
      }
      return 1;
    }
    case 5:
#pragma unroll
      for (int j = 0; j < 3; j++) {
        f[0][j] = xv[0][j] - xp[j];
        f[1][j] = xv[1][j] - xv[0][j];
        f[2][j] = xv[3][j] - xv[0][j];
        f[3][j] = xv[4][j] - xv[0][j];
        f[4][j] = xv[0][j] - xv[1][j] + xv[2][j] - xv[3][j];
        f[5][j] = xv[0][j] - xv[3][j];
        f[6][j] = xv[0][j] - xv[1][j];
        f[7][j] = -xv[0][j] + xv[1][j] - xv[2][j] + xv[3][j];
      }
      it = newton64(f, u, v, w);
      frac[0] = (1.0 - u) * (1.0 - v) * (1.0 - w);
      frac[1] = u * (1.0 - v) * (1.0 - w);
      frac[2] = u * v * (1.0 - w);
      frac[3] = (1.0 - u) * v * (1.0 - w);
      frac[4] = w;
      return it;
    case 6:
#pragma unroll
      for (int j = 0; j < 3; j++) {
        f[0][j] = xv[0][j] - xp[j];
        f[1][j] = xv[1][j] - xv[0][j];
        f[2][j] = xv[2][j] - xv[0][j];
        f[3][j] = xv[3][j] - xv[0][j];
        f[4][j] = 0;
        f[5][j] = xv[0][j] - xv[2][j] - xv[3][j] + xv[5][j];
        f[6][j] = xv[0][j] - xv[1][j] - xv[3][j] + xv[4][j];
        f[7][j] = 0.;
      }
      it = newton64(f, u, v, w);
      {
        double omuv = 1.0 - u - v, omw = 1.0 - w;
        frac[0] = omuv * omw;
        frac[1] = u * omw;
        frac[2] = v * omw;
        frac[3] = omuv * w;
        frac[4] = u * w;
        frac[5] = v * w;
      }
      return it;
    case 8:
#pragma unroll
      for (int j = 0; j < 3; j++) {
        f[0][j] = xv[0][j] - xp[j];
        f[1][j] = xv[1][j] - xv[0][j];
        f[2][j] = xv[3][j] - xv[0][j];
        f[3][j] = xv[4][j] - xv[0][j];
        f[4][j] = xv[0][j] - xv[1][j] + xv[2][j] - xv[3][j];
        f[5][j] = xv[0][j] - xv[3][j] + xv[7][j] - xv[4][j];
        f[6][j] = xv[0][j] - xv[1][j] + xv[5][j] - xv[4][j];
        f[7][j] = -xv[0][j] + xv[1][j] - xv[2][j] + xv[3][j] + xv[4][j] - xv[5][j] + xv[6][j] - xv[7][j];
      }
      it = newton64(f, u, v, w);
      {
        double omu = 1.0 - u, omv = 1.0 - v, omw = 1.0 - w;
        frac[0] = omu * omv * omw;
        frac[1] = u * omv * omw;
        frac[2] = u * v * omw;
        frac[3] = omu * v * omw;
        frac[4] = omu * omv * w;
        frac[5] = u * omv * w;
        frac[6] = u * v * w;
        frac[7] = omu * v * w;
      }
      return it;
    default:
      return -1;
  }
}

// src/checkContainment.C:74-83: 0 = reject, 1 = accept, 2 = accept on a face
// (|frac| < TOL) of a cell that may not donate (cellRes == BIG).
__host__ __device__ inline int classify64(const double frac[8], int nvert, bool big_cell) {
  int prov = 0;
  for (int m = 0; m < nvert; m++) {
    if ((frac[m] + kTol) * (frac[m] - 1.0 - kTol) > 0) return 0;
    if (fabs(frac[m]) < kTol && big_cell) prov = 1;
  }
  return prov ? 2 : 1;
}

// src/searchADTrecursion.C:63-66: the element box test with +-TOL
__host__ __device__ inline bool in_box64(const double p[3], const double lo[3], const double hi[3]) {
  return p[0] >= lo[0] - kTol && p[1] >= lo[1] - kTol && p[2] >= lo[2] - kTol &&
         p[0] <= hi[0] + kTol && p[1] <= hi[1] + kTol && p[2] <= hi[2] + kTol;
}

// The Fortran box product, left to right (src/cellVolume.f90:101-103).
__host__ __device__ inline double box_product(const double* a, const double* b, const double* c) {
  return a[0] * b[1] * c[2] - a[0] * b[2] * c[1] + a[1] * b[2] * c[0] - a[1] * b[0] * c[2] +
         a[2] * b[0] * c[1] - a[2] * b[1] * c[0];
}

// src/math.c:298-330 + src/cellVolume.f90:20-94: signed volume by the
// divergence theorem, quad faces split into four triangles.
__host__ __device__ inline double cell_volume64(const double xv[8][3], int nvert) {
  // face tables (1-based vertex ids) for tet, pyramid, prism, hex
  const signed char nverts[4][6] = {{3, 3, 3, 3, 0, 0}, {4, 3, 3, 3, 3, 0}, {3, 4, 4, 4, 3, 0}, {4, 4, 4, 4, 4, 4}};
  const signed char faces[4][24] = {
      {1, 2, 3, 0, 1, 4, 2, 0, 2, 4, 3, 0, 1, 3, 4, 0, 0, 0, 0, 0, 0, 0, 0, 0},
      {1, 2, 3, 4, 1, 5, 2, 0, 2, 5, 3, 0, 4, 3, 5, 0, 1, 4, 5, 0, 0, 0, 0, 0},
      {1, 2, 3, 0, 1, 4, 5, 2, 2, 5, 6, 3, 1, 3, 6, 4, 4, 6, 5, 0, 0, 0, 0, 0},
      {1, 2, 3, 4, 1, 5, 6, 2, 2, 6, 7, 3, 3, 7, 8, 4, 1, 4, 8, 5, 5, 8, 7, 6}};
  int t, nf;
  switch (nvert) {
    case 4: t = 0; nf = 4; break;
    case 5: t = 1; nf = 5; break;
    case 6: t = 2; nf = 5; break;
    default: t = 3; nf = 6; break;
  }
  double vol = 0.;
  for (int f = 0; f < nf; f++) {
    const double* p1 = xv[faces[t][4 * f + 0] - 1];
    const double* p2 = xv[faces[t][4 * f + 1] - 1];
    const double* p3 = xv[faces[t][4 * f + 2] - 1];
    if (nverts[t][f] == 3) {
      vol = vol - 0.5 * box_product(p1, p2, p3);
    } else {
      const double* p4 = xv[faces[t][4 * f + 3] - 1];
      vol = vol - 0.25 * box_product(p1, p2, p3);
      vol = vol - 0.25 * box_product(p1, p3, p4);
      vol = vol - 0.25 * box_product(p1, p2, p4);
      vol = vol - 0.25 * box_product(p2, p3, p4);
    }
  }
  return vol / 3.0;
}

// src/utils.c:170-185 (checkHoleMap): C truncation toward zero, outside -> 0
struct HoleMapDev {
  int tagidx;  // mesh tag - 1
  int nx[3];
  double ext[6];
  const unsigned char* hole;  // 1 = inside a hole
};

__device__ inline int check_holemap(const double* x, const HoleMapDev& h) {
  double dx[3];
  int ix[3];
#pragma unroll
  for (int i = 0; i < 3; i++) dx[i] = (h.ext[i + 3] - h.ext[i]) / h.nx[i];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    ix[i] = (int)((x[i] - h.ext[i]) / dx[i]);
    if (ix[i] < 0 || ix[i] > h.nx[i] - 1) return 0;
  }
  return h.hole[(size_t)ix[2] * h.nx[1] * h.nx[0] + (size_t)ix[1] * h.nx[0] + ix[0]];
}

inline int grid_for(long long n, int threads, int max_blocks = 148 * 16) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return (int)b;
}

}  // namespace tb
