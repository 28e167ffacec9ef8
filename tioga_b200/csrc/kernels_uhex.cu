// The uniform-hex fast path (tioga::set_uniform_hex_flag, tioga.h:195-201):
// a block of identical rectangular hexahedra is searched by an index lookup
// in a cell map instead of its tree.
//   set-up, at preprocess (MeshBlock::check_for_uniform_hex and
//   create_hex_cell_map, MeshBlock.C:1249-1409): every hex is tested on the
//   device (k_uhex_check), the node extents along the block's axes are
//   reduced exactly (k_uhex_extent), and the map gets each cell id at the
//   index of its centroid, the last cell winning (k_uhex_map);
//   search, every call (MeshBlock::search_uniform_hex, search.C:271-341):
//   one thread per query point of such a donor block (k_uhex_search).
// The FP64 expressions follow the reference's order (the library is built
// with -fmad=false), so indices and cell choices are the same.
#include "kernels.cuh"

namespace tb {

__device__ __forceinline__ double tdot3(const double a[3], const double b[3], const double c[3]) {
  double dp = 0.0;  // math.c:331-337
  for (int k = 0; k < 3; k++) dp += ((a[k] - c[k]) * (b[k] - c[k]));
  return dp;
}

// Any hex of block b that is degenerate (two consecutive vertex ids equal),
// not rectangular at vertices 0, 2, 5, 6, 7 within TOL, or whose squared edge
// lengths differ from the first hex's (dx0) by more than TOL sets *bad.
__global__ void k_uhex_check(const double* __restrict__ x, const int* __restrict__ conn8,
                             const BlockInfo* __restrict__ bi, int b, double d0, double d1, double d2,
                             unsigned* __restrict__ bad) {
  const BlockInfo& B = bi[b];
  bool fail = false;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < B.ncells;
       i += (long long)gridDim.x * blockDim.x) {
    const long long c = B.cell_off + i;
    double xv[8][3];
    int vold = -1;
    for (int m = 0; m < 8; m++) {
      const int v = conn8[8 * c + m];
      fail = fail || (v == vold);
      vold = v;
      for (int k = 0; k < 3; k++) xv[m][k] = x[3 * (long long)v + k];
    }
    fail = fail || fabs(tdot3(xv[1], xv[3], xv[0])) > kTol || fabs(tdot3(xv[1], xv[3], xv[2])) > kTol ||
           fabs(tdot3(xv[3], xv[4], xv[0])) > kTol || fabs(tdot3(xv[3], xv[4], xv[7])) > kTol ||
           fabs(tdot3(xv[4], xv[1], xv[0])) > kTol || fabs(tdot3(xv[4], xv[1], xv[5])) > kTol ||
           fabs(tdot3(xv[5], xv[7], xv[6])) > kTol;
    fail = fail || fabs(d0 - tdot3(xv[1], xv[1], xv[0])) > kTol || fabs(d1 - tdot3(xv[3], xv[3], xv[0])) > kTol ||
           fabs(d2 - tdot3(xv[4], xv[4], xv[0])) > kTol;
  }
  if (__any_sync(0xffffffffu, fail) && (threadIdx.x & 31) == 0) atomicOr(bad, 1u);
}

// min/max over the block's nodes of x . vec[j] (MeshBlock.C:1327-1342), as
// ordered keys: red[j] = min, red[j + 3] = max
__global__ void k_uhex_extent(const double* __restrict__ x, long long node_off, long long nnodes, UhexAxes A,
                              unsigned long long* __restrict__ red) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nnodes;
       i += (long long)gridDim.x * blockDim.x) {
    const double* p = x + 3 * (node_off + i);
    for (int j = 0; j < 3; j++) {
      double xd = 0;
      for (int k = 0; k < 3; k++) xd += p[k] * A.vec[j][k];
      lo[j] = dmin(lo[j], xd);
      hi[j] = dmax(hi[j], xd);
    }
  }
  for (int j = 0; j < 3; j++)
    for (int o = 16; o > 0; o >>= 1) {
      lo[j] = dmin(lo[j], __shfl_xor_sync(0xffffffffu, lo[j], o));
      hi[j] = dmax(hi[j], __shfl_xor_sync(0xffffffffu, hi[j], o));
    }
  if ((threadIdx.x & 31) == 0)
    for (int j = 0; j < 3; j++) {
      atomicMin(&red[j], dkey(lo[j]));
      atomicMax(&red[j + 3], dkey(hi[j]));
    }
}

// map[index of the centroid of (vertex 0, vertex 6)] = the caller's cell id,
// the largest id winning as the reference's sequential loop does
// (MeshBlock.C:1389-1408); a centroid outside the map, which a uniform box
// cannot have, is skipped (the reference writes it unchecked).
__global__ void k_uhex_map(const double* __restrict__ x, const int* __restrict__ conn8,
                           const int* __restrict__ sorted_cell, const BlockInfo* __restrict__ bi, int b,
                           int* __restrict__ map) {
  const BlockInfo& B = bi[b];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < B.ncells;
       i += (long long)gridDim.x * blockDim.x) {
    const long long s = B.cell_off + i;  // storage position
    const int orig = sorted_cell[s] - B.cell_off;
    const int ln = conn8[8 * s], tn = conn8[8 * s + 6];
    double xc[3], xd[3];
    int idx[3];
    bool ok = true;
    for (int j = 0; j < 3; j++) xc[j] = 0.5 * (x[3 * (long long)ln + j] + x[3 * (long long)tn + j]);
    for (int j = 0; j < 3; j++) {
      xd[j] = 0;
      for (int k = 0; k < 3; k++) xd[j] += (xc[k] - B.uxlow[k]) * B.uvec[j][k];
      idx[j] = (int)(xd[j] / B.udx[j]);
      ok = ok && idx[j] >= 0 && idx[j] < B.uidims[j];
    }
    if (ok)
      atomicMax(&map[B.umap_off + ((long long)idx[2] * B.uidims[1] + idx[1]) * B.uidims[0] + idx[0]], orig);
  }
}

// Donor cell of every query point whose donor block is a uniform box
// (search.C:293-334): the map cell at the point's index, or, while that is
// missing (-1) or a cell of BIG resolution, the cells at the corners of a cube
// of side 4 TOL around the point.  The reference's corner loop also tests a
// never-written malloc'd word against -1 (search.C:311, dId[0]); it is taken as
// not -1.  No containment test: the lookup is the search, as in the reference.
__global__ void k_uhex_search(const double* __restrict__ x, const int* __restrict__ qnode,
                              const int* __restrict__ qdon, long long nq, const BlockInfo* __restrict__ bi,
                              const int* __restrict__ map, const double* __restrict__ cell_res,
                              const int* __restrict__ inv_sorted, int* __restrict__ qcell,
                              unsigned char* __restrict__ qtie) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    const BlockInfo& B = bi[qdon[q]];
    if (!B.uhex) continue;
    const double* p = x + 3 * (long long)qnode[q];
    const int* d = B.uidims;
    const int* M = map + B.umap_off;
    double xd[3];
    int idx[3];
    for (int j = 0; j < 3; j++) {
      xd[j] = 0;
      for (int k = 0; k < 3; k++) xd[j] += (p[k] - B.uxlow[k]) * B.uvec[j][k];
      idx[j] = (int)(xd[j] / B.udx[j]);
    }
    int id0 = -1;
    if (xd[0] > -kTol && xd[0] < d[0] * B.udx[0] + kTol && xd[1] > -kTol && xd[1] < d[1] * B.udx[1] + kTol &&
        xd[2] > -kTol && xd[2] < d[2] * B.udx[2] + kTol) {
      for (int k = 0; k < 3; k++) {
        if (idx[k] == d[k]) idx[k]--;
        idx[k] = min(max(idx[k], 0), d[k] - 1);
      }
      id0 = M[((long long)idx[2] * d[1] + idx[1]) * d[0] + idx[0]];
      bool big = (id0 > -1) ? (cell_res[inv_sorted[B.cell_off + id0]] == kBig) : true;
      for (int jj = 0; jj < 8 && big; jj++) {
        for (int k = 0; k < 3; k++) {
          const double corner = (2 * ((jj & (1 << k)) >> k) - 1) * 2 * kTol;
          idx[k] = (int)((xd[k] + corner) / B.udx[k]);
          if (idx[k] == d[k]) idx[k]--;
          idx[k] = min(max(idx[k], 0), d[k] - 1);  // (in range for any map cell wider than 3 TOL)
        }
        const int dt = M[((long long)idx[2] * d[1] + idx[1]) * d[0] + idx[0]];
        big = (dt > -1) ? (cell_res[inv_sorted[B.cell_off + dt]] == kBig) : true;
        id0 = (id0 == -1) ? dt : (!big ? dt : id0);
      }
    }
    qcell[q] = id0 >= 0 ? inv_sorted[B.cell_off + id0] : -1;
    qtie[q] = 0;
  }
}

}  // namespace tb
