// Lagrange hexahedra of degree p with equispaced nodes: the element
// arithmetic of the high-order path on the device.
//
// An element's (p+1)^3 degrees of freedom are stored element-major in
// tensor order (node (i, j, k) at ((k (p+1) + j) (p+1) + i), i fastest),
// with reference coordinates (r, s, t) in [0, 1]^3 and node (i, j, k) at
// (i/p, j/p, k/p).  The inclusion test is Newton's method on the
// isoparametric map from the element centre; the weights are the basis
// functions at the inverted point.  Every operation is written out in a
// fixed order (compiled without contraction), so the FP64 results are the
// same bits as a host implementation of the same expressions.
#pragma once

namespace tb {

constexpr int kHoMaxN = 11;          // (p+1) per axis at most: NFRAC = 1331 = 11^3 weights
constexpr double kHoTol = 1e-10;     // inclusion tolerance in reference coordinates

// 1-D Lagrange basis on the nodes i/p and its derivative
__device__ inline void ho_basis1(int p, double r, double* l, double* dl) {
  for (int i = 0; i <= p; i++) {
    const double xi = (double)i / p;
    double v = 1.0, d = 0.0;
    for (int m = 0; m <= p; m++) {
      if (m == i) continue;
      const double xm = (double)m / p;
      const double den = xi - xm;
      d = d * ((r - xm) / den) + v / den;
      v = v * ((r - xm) / den);
    }
    l[i] = v;
    dl[i] = d;
  }
}

// map and Jacobian of the element with DOF coordinates X at u
__device__ inline void ho_map(int p, const double* __restrict__ X, const double u[3], double x[3],
                              double J[3][3]) {
  const int n1 = p + 1;
  double lr[kHoMaxN], ls[kHoMaxN], lt[kHoMaxN], dr[kHoMaxN], ds[kHoMaxN], dt[kHoMaxN];
  ho_basis1(p, u[0], lr, dr);
  ho_basis1(p, u[1], ls, ds);
  ho_basis1(p, u[2], lt, dt);
  for (int a = 0; a < 3; a++) {
    x[a] = 0.0;
    J[a][0] = J[a][1] = J[a][2] = 0.0;
  }
  for (int k = 0; k < n1; k++)
    for (int j = 0; j < n1; j++)
      for (int i = 0; i < n1; i++) {
        const double* P = X + 3 * ((k * n1 + j) * n1 + i);
        const double w = (lr[i] * ls[j]) * lt[k];
        const double wr = (dr[i] * ls[j]) * lt[k];
        const double ws = (lr[i] * ds[j]) * lt[k];
        const double wt = (lr[i] * ls[j]) * dt[k];
        for (int a = 0; a < 3; a++) {
          x[a] = x[a] + w * P[a];
          J[a][0] = J[a][0] + wr * P[a];
          J[a][1] = J[a][1] + ws * P[a];
          J[a][2] = J[a][2] + wt * P[a];
        }
      }
}

// Newton inversion from the element centre; true when the update fell below
// 1e-14 (sum of magnitudes) within 50 steps
__device__ inline bool ho_invert(int p, const double* __restrict__ X, const double* xp, double u[3]) {
  u[0] = u[1] = u[2] = 0.5;
  for (int it = 0; it < 50; it++) {
    double x[3], J[3][3];
    ho_map(p, X, u, x, J);
    const double f0 = xp[0] - x[0], f1 = xp[1] - x[1], f2 = xp[2] - x[2];
    const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
    if (!(fabs(det) > 1e-300)) return false;
    // Cramer's rule: du = J^-1 f
    const double d0 = (f0 * c00 + f1 * (J[0][2] * J[2][1] - J[0][1] * J[2][2]) +
                       f2 * (J[0][1] * J[1][2] - J[0][2] * J[1][1])) / det;
    const double d1 = (f0 * c01 + f1 * (J[0][0] * J[2][2] - J[0][2] * J[2][0]) +
                       f2 * (J[0][2] * J[1][0] - J[0][0] * J[1][2])) / det;
    const double d2 = (f0 * c02 + f1 * (J[0][1] * J[2][0] - J[0][0] * J[2][1]) +
                       f2 * (J[0][0] * J[1][1] - J[0][1] * J[1][0])) / det;
    u[0] = u[0] + d0;
    u[1] = u[1] + d1;
    u[2] = u[2] + d2;
    if (fabs(d0) + fabs(d1) + fabs(d2) < 1e-14) return true;
  }
  return false;
}

__device__ inline bool ho_inside(const double u[3]) {
  return u[0] >= -kHoTol && u[0] <= 1.0 + kHoTol && u[1] >= -kHoTol && u[1] <= 1.0 + kHoTol &&
         u[2] >= -kHoTol && u[2] <= 1.0 + kHoTol;
}

// the (p+1)^3 weights at u, tensor order
__device__ inline void ho_weights(int p, const double u[3], double* w) {
  const int n1 = p + 1;
  double lr[kHoMaxN], ls[kHoMaxN], lt[kHoMaxN], d[kHoMaxN];
  ho_basis1(p, u[0], lr, d);
  ho_basis1(p, u[1], ls, d);
  ho_basis1(p, u[2], lt, d);
  int m = 0;
  for (int k = 0; k < n1; k++)
    for (int j = 0; j < n1; j++)
      for (int i = 0; i < n1; i++, m++) w[m] = (lr[i] * ls[j]) * lt[k];
}

// The same three functions for a degree known at compile time: the loops
// unroll and the basis values stay in registers.  Every operation is the one
// of the generic form above, in the same order (a constant divisor is still
// an IEEE division), so the results are the same bits.
template <int P>
__device__ __forceinline__ void ho_basis1_t(double r, double* l, double* dl) {
#pragma unroll
  for (int i = 0; i <= P; i++) {
    const double xi = (double)i / P;
    double v = 1.0, d = 0.0;
#pragma unroll
    for (int m = 0; m <= P; m++) {
      if (m == i) continue;
      const double xm = (double)m / P;
      const double den = xi - xm;
      d = d * ((r - xm) / den) + v / den;
      v = v * ((r - xm) / den);
    }
    l[i] = v;
    dl[i] = d;
  }
}

template <int P>
__device__ __forceinline__ void ho_map_t(const double* __restrict__ X, const double u[3], double x[3],
                                         double J[3][3]) {
  constexpr int n1 = P + 1;
  double lr[n1], ls[n1], lt[n1], dr[n1], ds[n1], dt[n1];
  ho_basis1_t<P>(u[0], lr, dr);
  ho_basis1_t<P>(u[1], ls, ds);
  ho_basis1_t<P>(u[2], lt, dt);
#pragma unroll
  for (int a = 0; a < 3; a++) {
    x[a] = 0.0;
    J[a][0] = J[a][1] = J[a][2] = 0.0;
  }
#pragma unroll 1
  for (int k = 0; k < n1; k++)
#pragma unroll 1
    for (int j = 0; j < n1; j++) {
      const double lsj = ls[j], dsj = ds[j], ltk = lt[k], dtk = dt[k];
      const double* Pj = X + 3 * ((k * n1 + j) * n1);
#pragma unroll
      for (int i = 0; i < n1; i++) {
        const double* Pp = Pj + 3 * i;
        const double w = (lr[i] * lsj) * ltk;
        const double wr = (dr[i] * lsj) * ltk;
        const double ws = (lr[i] * dsj) * ltk;
        const double wt = (lr[i] * lsj) * dtk;
#pragma unroll
        for (int a = 0; a < 3; a++) {
          x[a] = x[a] + w * Pp[a];
          J[a][0] = J[a][0] + wr * Pp[a];
          J[a][1] = J[a][1] + ws * Pp[a];
          J[a][2] = J[a][2] + wt * Pp[a];
        }
      }
    }
}

template <int P>
__device__ inline bool ho_invert_t(const double* __restrict__ X, const double* xp, double u[3]) {
  u[0] = u[1] = u[2] = 0.5;
  for (int it = 0; it < 50; it++) {
    double x[3], J[3][3];
    ho_map_t<P>(X, u, x, J);
    const double f0 = xp[0] - x[0], f1 = xp[1] - x[1], f2 = xp[2] - x[2];
    const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
    if (!(fabs(det) > 1e-300)) return false;
    const double d0 = (f0 * c00 + f1 * (J[0][2] * J[2][1] - J[0][1] * J[2][2]) +
                       f2 * (J[0][1] * J[1][2] - J[0][2] * J[1][1])) / det;
    const double d1 = (f0 * c01 + f1 * (J[0][0] * J[2][2] - J[0][2] * J[2][0]) +
                       f2 * (J[0][2] * J[1][0] - J[0][0] * J[1][2])) / det;
    const double d2 = (f0 * c02 + f1 * (J[0][1] * J[2][0] - J[0][0] * J[2][1]) +
                       f2 * (J[0][0] * J[1][1] - J[0][1] * J[1][0])) / det;
    u[0] = u[0] + d0;
    u[1] = u[1] + d1;
    u[2] = u[2] + d2;
    if (fabs(d0) + fabs(d1) + fabs(d2) < 1e-14) return true;
  }
  return false;
}

template <int P>
__device__ __forceinline__ void ho_weights_t(const double u[3], double* w) {
  constexpr int n1 = P + 1;
  double lr[n1], ls[n1], lt[n1], d[n1];
  ho_basis1_t<P>(u[0], lr, d);
  ho_basis1_t<P>(u[1], ls, d);
  ho_basis1_t<P>(u[2], lt, d);
#pragma unroll
  for (int k = 0; k < n1; k++)
#pragma unroll
    for (int j = 0; j < n1; j++)
#pragma unroll
      for (int i = 0; i < n1; i++) w[(k * n1 + j) * n1 + i] = (lr[i] * ls[j]) * lt[k];
}

// degree dispatch: the common degrees take the unrolled forms
__device__ inline bool ho_invert_any(int p, const double* __restrict__ X, const double* xp, double u[3]) {
  switch (p) {
    case 1: return ho_invert_t<1>(X, xp, u);
    case 2: return ho_invert_t<2>(X, xp, u);
    case 3: return ho_invert_t<3>(X, xp, u);
    default: return ho_invert(p, X, xp, u);
  }
}
__device__ inline void ho_weights_any(int p, const double u[3], double* w) {
  switch (p) {
    case 1: ho_weights_t<1>(u, w); break;
    case 2: ho_weights_t<2>(u, w); break;
    case 3: ho_weights_t<3>(u, w); break;
    default: ho_weights(p, u, w);
  }
}

// FP32 screen of the inclusion test for the split-precision form: Newton on
// the element map in FP32, on offsets from the element's first DOF (so the
// coordinates' common part does not cost precision).  Returns 1 when it
// converged clearly inside (every reference coordinate within [1e-3,
// 1 - 1e-3]), 0 clearly outside (one below -1e-3 or above 1 + 1e-3), -1
// otherwise (near a face, no convergence in 20 steps, a near-singular map).
// Both iterate from the same centre and converge to the same point to about
// 1e-6, so a clear outside is the FP64 test's reject; a clear inside is not
// enough for an accept, which also needs the FP64 update to fall below 1e-14.
__device__ inline void ho_basis1f(int p, float r, float* l, float* dl) {
  for (int i = 0; i <= p; i++) {
    const float xi = (float)i / p;
    float v = 1.f, d = 0.f;
    for (int m = 0; m <= p; m++) {
      if (m == i) continue;
      const float xm = (float)m / p;
      const float den = xi - xm;
      d = d * ((r - xm) / den) + v / den;
      v = v * ((r - xm) / den);
    }
    l[i] = v;
    dl[i] = d;
  }
}

__device__ inline int ho_screen32(int p, const double* __restrict__ X, const double* xp) {
  const int n1 = p + 1;
  const double x0[3] = {X[0], X[1], X[2]};
  const float fp[3] = {(float)(xp[0] - x0[0]), (float)(xp[1] - x0[1]), (float)(xp[2] - x0[2])};
  float u[3] = {0.5f, 0.5f, 0.5f};
  for (int it = 0; it < 20; it++) {
    float lr[kHoMaxN], ls[kHoMaxN], lt[kHoMaxN], dr[kHoMaxN], ds[kHoMaxN], dt[kHoMaxN];
    ho_basis1f(p, u[0], lr, dr);
    ho_basis1f(p, u[1], ls, ds);
    ho_basis1f(p, u[2], lt, dt);
    float x[3] = {0.f, 0.f, 0.f}, J[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    for (int k = 0; k < n1; k++)
      for (int j = 0; j < n1; j++)
        for (int i = 0; i < n1; i++) {
          const double* P = X + 3 * ((k * n1 + j) * n1 + i);
          const float w = (lr[i] * ls[j]) * lt[k];
          const float wr = (dr[i] * ls[j]) * lt[k];
          const float ws = (lr[i] * ds[j]) * lt[k];
          const float wt = (lr[i] * ls[j]) * dt[k];
          for (int a = 0; a < 3; a++) {
            const float pa = (float)(P[a] - x0[a]);
            x[a] = __fmaf_rn(w, pa, x[a]);
            J[a][0] = __fmaf_rn(wr, pa, J[a][0]);
            J[a][1] = __fmaf_rn(ws, pa, J[a][1]);
            J[a][2] = __fmaf_rn(wt, pa, J[a][2]);
          }
        }
    const float f0 = fp[0] - x[0], f1 = fp[1] - x[1], f2 = fp[2] - x[2];
    const float c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    const float c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    const float c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    const float det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
    const float n0 = sqrtf(J[0][0] * J[0][0] + J[1][0] * J[1][0] + J[2][0] * J[2][0]);
    const float nn1 = sqrtf(J[0][1] * J[0][1] + J[1][1] * J[1][1] + J[2][1] * J[2][1]);
    const float n2 = sqrtf(J[0][2] * J[0][2] + J[1][2] * J[1][2] + J[2][2] * J[2][2]);
    const float scale = n0 * nn1 * n2;
    if (!(scale > 0.f) || !(fabsf(det) > 1e-3f * scale)) return -1;
    const float id = 1.f / det;
    const float d0 = (f0 * c00 + f1 * (J[0][2] * J[2][1] - J[0][1] * J[2][2]) +
                      f2 * (J[0][1] * J[1][2] - J[0][2] * J[1][1])) * id;
    const float d1 = (f0 * c01 + f1 * (J[0][0] * J[2][2] - J[0][2] * J[2][0]) +
                      f2 * (J[0][2] * J[1][0] - J[0][0] * J[1][2])) * id;
    const float d2 = (f0 * c02 + f1 * (J[0][1] * J[2][0] - J[0][0] * J[2][1]) +
                      f2 * (J[0][0] * J[1][1] - J[0][1] * J[1][0])) * id;
    u[0] += d0;
    u[1] += d1;
    u[2] += d2;
    if (!(fabsf(u[0]) < 1e3f && fabsf(u[1]) < 1e3f && fabsf(u[2]) < 1e3f)) return -1;
    if (fabsf(d0) + fabsf(d1) + fabsf(d2) < 1e-5f) {
      constexpr float e = 1e-3f;
      bool in = true;
      for (int k = 0; k < 3; k++) {
        if (u[k] < -e || u[k] > 1.f + e) return 0;
        in = in && u[k] >= e && u[k] <= 1.f - e;
      }
      return in ? 1 : -1;
    }
  }
  return -1;
}

}  // namespace tb
