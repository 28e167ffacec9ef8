// Connectivity kernels: hole maps (src/holeMap.C:40-188, MeshBlock.C:637-772,
// utils.c:192-295), box pairs (exchangeBoxes.C:34-272, utils.c:297-384,
// MeshBlock.C:774-838), query gathering (exchangeSearchData.C:27-263,
// MeshBlock.C:953-1117), the bounding-volume tree refit and the fused
// tree-search + Newton containment kernel (search.C:78-269,
// searchADTrecursion.C:26-101, checkContainment.C:27-96, math.c:25-294).
#include <cub/block/block_scan.cuh>

#include "kernels.cuh"

namespace tb {

// ===========================================================================
// hole maps
// ===========================================================================
__global__ void k_wall_bounds(const double* __restrict__ x, const int* __restrict__ wall_list, int off,
                              int n, unsigned long long* __restrict__ bb) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double* p = x + 3 * (long long)wall_list[off + i];
    for (int j = 0; j < 3; j++) {
      lo[j] = dmin(lo[j], p[j]);
      hi[j] = dmax(hi[j], p[j]);
    }
  }
  for (int j = 0; j < 3; j++) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[j] = dmin(lo[j], __shfl_xor_sync(0xffffffffu, lo[j], o));
      hi[j] = dmax(hi[j], __shfl_xor_sync(0xffffffffu, hi[j], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
    for (int j = 0; j < 3; j++) {
      atomicMin(&bb[j], dkey(lo[j]));
      atomicMax(&bb[j + 3], dkey(hi[j]));
    }
  }
}

// extents and sizes exactly as holeMap.C:118-140
__global__ void k_holemap_setup(const unsigned long long* __restrict__ bb, HoleMapInfo* __restrict__ hm,
                                int t) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  HoleMapInfo& h = hm[t];
  double ds[3];
  for (int j = 0; j < 3; j++) {
    h.ext[j] = dkey_inv(bb[6 * t + j]);
    h.ext[j + 3] = dkey_inv(bb[6 * t + j + 3]);
    ds[j] = h.ext[j + 3] - h.ext[j];
  }
  double dsmax = dmax(ds[0], ds[1]);
  dsmax = dmax(dsmax, ds[2]);
  double dsbox = dsmax / kHoleMapSize;
  for (int j = 0; j < 3; j++) {
    h.ext[j] -= (2 * dsbox);
    h.ext[j + 3] += (2 * dsbox);
    h.nx[j] = (int)floor(dmax((h.ext[j + 3] - h.ext[j]) / dsbox, 1));
  }
  h.exist = 1;
}

__global__ void k_holemap_mark(const double* __restrict__ x, const int* __restrict__ conn8,
                               const unsigned char* __restrict__ cell_nv, int cell_off, int ncells,
                               const unsigned char* __restrict__ wallf, const HoleMapInfo* __restrict__ hmp,
                               unsigned char* __restrict__ sam) {
  const HoleMapInfo h = *hmp;
  double ds[3];
  for (int k = 0; k < 3; k++) ds[k] = (h.ext[k + 3] - h.ext[k]) / h.nx[k];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncells; i += gridDim.x * blockDim.x) {
    long long c = (long long)cell_off + i;
    int nv = cell_nv[c];
    const int* cv = conn8 + 8 * c;
    int wall = 0;
    for (int m = 0; m < nv; m++) wall |= wallf[cv[m]];
    if (!wall) continue;
    int imin[3] = {kBigInt, kBigInt, kBigInt}, imax[3] = {-kBigInt, -kBigInt, -kBigInt};
    for (int m = 0; m < nv; m++) {
      const double* p = x + 3 * (long long)cv[m];
      for (int k = 0; k < 3; k++) {
        int iv = (int)floor((p[k] - h.ext[k]) / ds[k]);
        imin[k] = min(imin[k], iv);
        imax[k] = max(imax[k], iv);
      }
    }
    for (int j = 0; j < 3; j++) {
      imin[j] = max(imin[j], 0);
      imax[j] = min(imax[j], h.nx[j] - 1);
    }
    for (int kk = imin[2]; kk < imax[2] + 1; kk++)
      for (int jj = imin[1]; jj < imax[1] + 1; jj++)
        for (int ii = imin[0]; ii < imax[0] + 1; ii++)
          sam[(size_t)kk * h.nx[1] * h.nx[0] + (size_t)jj * h.nx[0] + ii] = 2;
  }
}

// Plane-wise flood fill for isym = 1, 2, 3 (4-neighbour fills inside planes
// normal to x, y, z).  One CTA owns one plane in shared memory, seeds the
// six box faces with 1 (utils.c:206-226) and alternates forward/backward line
// sweeps along both in-plane axes until nothing changes.  The painted set is
// the closure of the seeds through unmarked cells, the same fixed point as
// the reference's Gauss-Seidel sweeps (utils.c:227-290), which is
// independent of the visiting order.  With seed == 2 (6-neighbour mode) the
// kernel only seeds the faces.
__global__ void k_holemap_fill_planes(unsigned char* __restrict__ sam, const HoleMapInfo* __restrict__ hmp,
                                      int isym, int seed_only, unsigned* __restrict__ changed,
                                      unsigned* __restrict__ err) {
  extern __shared__ unsigned char s[];
  const HoleMapInfo h = *hmp;
  const int n[3] = {h.nx[0], h.nx[1], h.nx[2]};
  const long long st[3] = {1, n[0], (long long)n[0] * n[1]};
  int pa, a0, a1;  // plane-normal axis and the two in-plane axes
  if (isym == 1) { pa = 0; a0 = 1; a1 = 2; }
  else if (isym == 2) { pa = 1; a0 = 0; a1 = 2; }
  else { pa = 2; a0 = 0; a1 = 1; }
  const int n0 = n[a0], n1 = n[a1];
  for (int plane = blockIdx.x; plane < n[pa]; plane += gridDim.x) {
    const bool face_plane = (plane == 0 || plane == n[pa] - 1);
    const long long base = plane * st[pa];
    for (int t = threadIdx.x; t < n0 * n1; t += blockDim.x) {
      int i0 = t % n0, i1 = t / n0;
      unsigned char v = sam[base + i0 * st[a0] + i1 * st[a1]];
      if (face_plane || i0 == 0 || i0 == n0 - 1 || i1 == 0 || i1 == n1 - 1) v = 1;
      s[t] = v;
    }
    __syncthreads();
    if (!seed_only && !face_plane) {
      int rounds = 0;
      const int max_rounds = n0 * n1 + 2;
      for (;;) {
        int ch = 0;
        // lines along a0 (fixed i1)
        for (int i1 = 1 + threadIdx.x; i1 < n1 - 1; i1 += blockDim.x) {
          unsigned char* L = s + i1 * n0;
          for (int i0 = 1; i0 < n0 - 1; i0++)
            if (L[i0] == 0 && L[i0 - 1] == 1) { L[i0] = 1; ch = 1; }
          for (int i0 = n0 - 2; i0 >= 1; i0--)
            if (L[i0] == 0 && L[i0 + 1] == 1) { L[i0] = 1; ch = 1; }
        }
        __syncthreads();
        // lines along a1 (fixed i0)
        for (int i0 = 1 + threadIdx.x; i0 < n0 - 1; i0 += blockDim.x) {
          for (int i1 = 1; i1 < n1 - 1; i1++)
            if (s[i1 * n0 + i0] == 0 && s[(i1 - 1) * n0 + i0] == 1) { s[i1 * n0 + i0] = 1; ch = 1; }
          for (int i1 = n1 - 2; i1 >= 1; i1--)
            if (s[i1 * n0 + i0] == 0 && s[(i1 + 1) * n0 + i0] == 1) { s[i1 * n0 + i0] = 1; ch = 1; }
        }
        int any = __syncthreads_or(ch);
        if (!any) break;
        if (++rounds > max_rounds) {
          if (threadIdx.x == 0) atomicOr(err, kErrFloodFillBound);
          break;
        }
      }
    }
    for (int t = threadIdx.x; t < n0 * n1; t += blockDim.x) {
      int i0 = t % n0, i1 = t / n0;
      sam[base + i0 * st[a0] + i1 * st[a1]] = s[t];
    }
    __syncthreads();
  }
  (void)changed;
}

// 6-neighbour mode: one forward and one backward sweep along `axis` for every
// line of interior cells; repeated over the three axes until no change.
__global__ void k_holemap_lines(unsigned char* __restrict__ sam, const HoleMapInfo* __restrict__ hmp,
                                int axis, unsigned* __restrict__ changed) {
  const HoleMapInfo h = *hmp;
  const int n[3] = {h.nx[0], h.nx[1], h.nx[2]};
  const long long st[3] = {1, n[0], (long long)n[0] * n[1]};
  int b0 = (axis == 0) ? 1 : 0, b1 = (axis == 2) ? 1 : 2;
  long long nlines = (long long)n[b0] * n[b1];
  int ch = 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nlines;
       t += (long long)gridDim.x * blockDim.x) {
    int i0 = (int)(t % n[b0]), i1 = (int)(t / n[b0]);
    if (i0 == 0 || i0 == n[b0] - 1 || i1 == 0 || i1 == n[b1] - 1) continue;
    unsigned char* L = sam + i0 * st[b0] + i1 * st[b1];
    long long s = st[axis];
    for (int k = 1; k < n[axis] - 1; k++)
      if (L[k * s] == 0 && L[(k - 1) * s] == 1) { L[k * s] = 1; ch = 1; }
    for (int k = n[axis] - 2; k >= 1; k--)
      if (L[k * s] == 0 && L[(k + 1) * s] == 1) { L[k * s] = 1; ch = 1; }
  }
  if (ch) atomicOr(changed, 1u);
}

// hole = unreached or wall-marked (utils.c:291-294)
__global__ void k_holemap_final(unsigned char* __restrict__ sam, const HoleMapInfo* __restrict__ hmp) {
  const HoleMapInfo h = *hmp;
  long long n = (long long)h.nx[0] * h.nx[1] * h.nx[2];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    unsigned char v = sam[i];
    sam[i] = (v == 0 || v == 2) ? 1 : 0;
  }
}

// ===========================================================================
// box pairs
// ===========================================================================
// src/utils.c:297-384: separating-axis test of two oriented boxes
__device__ int obb_intersect(const double vA[3][3], const double xA[3], const double dxA[3],
                             const double vB[3][3], const double xB[3], const double dxB[3]) {
  const double eps = 1e-12;
  double D[3], c[3][3], r, r0, r1, d1, d2;
  for (int i = 0; i < 3; i++) D[i] = xB[i] - xA[i];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      c[i][j] = 0;
      for (int k = 0; k < 3; k++) c[i][j] = c[i][j] + vA[i][k] * vB[j][k];
    }
  for (int i = 0; i < 3; i++) {
    r0 = dxA[i];
    r1 = 0;
    r = 0;
    for (int j = 0; j < 3; j++) {
      r1 += dxB[j] * fabs(c[i][j]);
      r += fabs(vA[i][j]) * D[j];
    }
    if (r > (r0 + r1 + eps)) return 0;
  }
  for (int i = 0; i < 3; i++) {
    r1 = dxB[i];
    r0 = 0;
    r = 0;
    for (int j = 0; j < 3; j++) {
      r0 += dxA[j] * fabs(c[j][i]);
      r += fabs(vB[i][j]) * D[j];
    }
    if (r > (r0 + r1 + eps)) return 0;
  }
  for (int i = 0; i < 3; i++) {
    int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
    for (int j = 0; j < 3; j++) {
      int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
      r0 = dxA[i1] * fabs(c[i2][j]) + dxA[i2] * fabs(c[i1][j]);
      r1 = dxB[j1] * fabs(c[i][j2]) + dxB[j2] * fabs(c[i][j1]);
      d2 = 0;
      d1 = 0;
      for (int k = 0; k < 3; k++) {
        d2 += vA[i2][k] * D[k];
        d1 += vA[i1][k] * D[k];
      }
      r = fabs(c[i1][j] * d2 - c[i2][j] * d1);
      if (r > (r0 + r1 + eps)) return 0;
    }
  }
  return 1;
}

// pairs listed donor-outer, receptor-inner as in exchangeBoxes.C:133-160
__global__ void k_pairs(BlockInfo* __restrict__ bi, int nb, PairInfo* __restrict__ pairs,
                        int* __restrict__ npairs) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int np = 0;
  for (int ob = 0; ob < nb; ob++)
    for (int ib = 0; ib < nb; ib++) {
      const Obb& a = bi[ib].obb;
      const Obb& o = bi[ob].obb;
      if (abs(bi[ob].tag) == bi[ib].tag) continue;
      if (obb_intersect(a.vec, a.xc, a.dxc, o.vec, o.xc, o.dxc) ||
          obb_intersect(o.vec, o.xc, o.dxc, a.vec, a.xc, a.dxc)) {
        pairs[np].rec = ib;
        pairs[np].don = ob;
        np++;
      }
    }
  *npairs = np;
}

// Region of the donor's cells whose boxes overlap the receptor's OBB, in the
// donor's OBB frame (getReducedOBB).  One pass over the donor's cells serves
// every pair that has this donor.  acc holds 6 ordered keys per pair.
__global__ void k_reduced_obb(const double* __restrict__ x, const int* __restrict__ conn8,
                              const unsigned char* __restrict__ cell_nv, const BlockInfo* __restrict__ bi,
                              int don, PairInfo* __restrict__ pairs, int npairs,
                              unsigned long long* __restrict__ acc) {
  const BlockInfo& D = bi[don];
  const int lane = threadIdx.x & 31;
  const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long base = warp0 * 32; base < D.ncells; base += nwarps * 32) {
    long long i = base + lane;
    bool valid = i < D.ncells;
    double xv[8][3];
    int nv = 0;
    if (valid) {
      long long c = (long long)D.cell_off + i;
      nv = cell_nv[c];
      gather_vertices(x, conn8 + 8 * c, nv, xv);
    }
    for (int p = 0; p < npairs; p++) {
      if (pairs[p].don != don) continue;
      const Obb& R = bi[pairs[p].rec].obb;
      bool ov = false;
      double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
      if (valid) {
        double bb[6] = {kBig, kBig, kBig, -kBig, -kBig, -kBig};
        for (int m = 0; m < nv; m++) {
          double xd[3];
          for (int j = 0; j < 3; j++) {
            xd[j] = 0;
            for (int k = 0; k < 3; k++) xd[j] += (xv[m][k] - R.xc[k]) * R.vec[j][k];
          }
          for (int j = 0; j < 3; j++) {
            bb[j] = dmin(bb[j], xd[j]);
            bb[j + 3] = dmax(bb[j + 3], xd[j]);
          }
        }
        ov = true;
        for (int j = 0; j < 3; j++) ov = ov && !(bb[j] > R.dxc[j]);
        for (int j = 0; j < 3; j++) ov = ov && !(bb[j + 3] < -R.dxc[j]);
        if (ov) {
          for (int m = 0; m < nv; m++) {
            for (int j = 0; j < 3; j++) {
              double xd = 0;
              for (int k = 0; k < 3; k++) xd += (xv[m][k] - D.obb.xc[k]) * D.obb.vec[j][k];
              lo[j] = dmin(lo[j], xd);
              hi[j] = dmax(hi[j], xd);
            }
          }
        }
      }
      if (__any_sync(0xffffffffu, ov)) {
        for (int j = 0; j < 3; j++)
          for (int o = 16; o > 0; o >>= 1) {
            lo[j] = dmin(lo[j], __shfl_xor_sync(0xffffffffu, lo[j], o));
            hi[j] = dmax(hi[j], __shfl_xor_sync(0xffffffffu, hi[j], o));
          }
        if (lane == 0)
          for (int j = 0; j < 3; j++) {
            atomicMin(&acc[6 * p + j], dkey(lo[j]));
            atomicMax(&acc[6 * p + j + 3], dkey(hi[j]));
          }
      }
    }
  }
}

__global__ void k_pair_finish(const BlockInfo* __restrict__ bi, PairInfo* __restrict__ pairs, int npairs,
                              const unsigned long long* __restrict__ acc) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  const Obb& o = bi[pairs[p].don].obb;
  double rd[6];
  for (int k = 0; k < 6; k++) rd[k] = dkey_inv(acc[6 * p + k]);
  Obb r;
  for (int j = 0; j < 3; j++) {
    r.xc[j] = o.xc[j];
    for (int k = 0; k < 3; k++) r.xc[j] += ((rd[k] + rd[k + 3]) * 0.5) * o.vec[k][j];
    r.dxc[j] = (rd[j + 3] - rd[j]) * 0.51;
    for (int k = 0; k < 3; k++) r.vec[j][k] = o.vec[j][k];
  }
  for (int k = 0; k < 6; k++) pairs[p].rd[k] = rd[k];
  pairs[p].region = r;
}

// ===========================================================================
// bounding-volume tree: cell boxes in Morton order, leaves of kLeafCells
// cells, implicit complete binary tree (heap order) per block
// ===========================================================================
__device__ __forceinline__ float f_rd(double v) { return __double2float_rd(v); }
__device__ __forceinline__ float f_ru(double v) { return __double2float_ru(v); }

__global__ void k_cell_boxes(const double* __restrict__ x, const int* __restrict__ conn8,
                             const unsigned char* __restrict__ cell_nv, const int* __restrict__ sorted_cell,
                             long long ctot, float4* __restrict__ cbox, double* __restrict__ cbox64) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < ctot;
       j += (long long)gridDim.x * blockDim.x) {
    int c = sorted_cell[j];
    int nv = cell_nv[c];
    const int* cv = conn8 + 8 * (long long)c;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int m = 0; m < nv; m++) {
      const double* p = x + 3 * (long long)cv[m];
      for (int k = 0; k < 3; k++) {
        lo[k] = dmin(lo[k], p[k]);
        hi[k] = dmax(hi[k], p[k]);
      }
    }
    cbox[2 * j] = make_float4(f_rd(lo[0]), f_rd(lo[1]), f_rd(lo[2]), f_ru(hi[0]));
    cbox[2 * j + 1] = make_float4(f_ru(hi[1]), f_ru(hi[2]), 0.f, 0.f);
    if (cbox64) {
      double* o = cbox64 + 6 * j;
      o[0] = lo[0]; o[1] = lo[1]; o[2] = lo[2];
      o[3] = hi[0]; o[4] = hi[1]; o[5] = hi[2];
    }
  }
}

// Leaves, then parents bottom-up: the second child to finish builds the
// parent (the usual refit with per-node arrival counters).
__global__ void k_tree_leaves(const BlockInfo* __restrict__ bi, int nb, const float4* __restrict__ cbox,
                              const double* __restrict__ cbox64, float4* __restrict__ tnode,
                              double* __restrict__ tnode64, int* __restrict__ visit, long long total_leaves,
                              const long long* __restrict__ leaf_base) {
  for (long long L = blockIdx.x * (long long)blockDim.x + threadIdx.x; L < total_leaves;
       L += (long long)gridDim.x * blockDim.x) {
    int b = 0;
    while (b + 1 < nb && leaf_base[b + 1] <= L) b++;
    const BlockInfo& B = bi[b];
    int leaf = (int)(L - leaf_base[b]);
    int j0 = leaf * kLeafCells, j1 = min(j0 + kLeafCells, B.ncells);
    float lo0 = INFINITY, lo1 = INFINITY, lo2 = INFINITY, hi0 = -INFINITY, hi1 = -INFINITY, hi2 = -INFINITY;
    double d[6] = {1e300, 1e300, 1e300, -1e300, -1e300, -1e300};
    for (int j = j0; j < j1; j++) {
      long long s = (long long)B.cell_off + j;
      float4 a = cbox[2 * s], c = cbox[2 * s + 1];
      lo0 = fminf(lo0, a.x); lo1 = fminf(lo1, a.y); lo2 = fminf(lo2, a.z);
      hi0 = fmaxf(hi0, a.w); hi1 = fmaxf(hi1, c.x); hi2 = fmaxf(hi2, c.y);
      if (tnode64)
        for (int k = 0; k < 3; k++) {
          d[k] = dmin(d[k], cbox64[6 * s + k]);
          d[k + 3] = dmax(d[k + 3], cbox64[6 * s + k + 3]);
        }
    }
    int node = B.P - 1 + leaf;
    long long gn = (long long)B.tree_off + node;
    tnode[2 * gn] = make_float4(lo0, lo1, lo2, hi0);
    tnode[2 * gn + 1] = make_float4(hi1, hi2, 0.f, 0.f);
    if (tnode64)
      for (int k = 0; k < 6; k++) tnode64[6 * gn + k] = d[k];
    while (node > 0) {
      int parent = (node - 1) >> 1;
      __threadfence();
      long long gp = (long long)B.tree_off + parent;
      if (atomicAdd(&visit[gp], 1) == 0) break;  // the sibling builds it
      long long gl = (long long)B.tree_off + 2 * parent + 1, gr = gl + 1;
      float4 la = __ldcg(&tnode[2 * gl]), lb = __ldcg(&tnode[2 * gl + 1]);
      float4 ra = __ldcg(&tnode[2 * gr]), rb = __ldcg(&tnode[2 * gr + 1]);
      tnode[2 * gp] = make_float4(fminf(la.x, ra.x), fminf(la.y, ra.y), fminf(la.z, ra.z), fmaxf(la.w, ra.w));
      tnode[2 * gp + 1] = make_float4(fmaxf(lb.x, rb.x), fmaxf(lb.y, rb.y), 0.f, 0.f);
      if (tnode64)
        for (int k = 0; k < 6; k++) {
          double u = __ldcg(&tnode64[6 * gl + k]), v = __ldcg(&tnode64[6 * gr + k]);
          tnode64[6 * gp + k] = (k < 3) ? dmin(u, v) : dmax(u, v);
        }
      node = parent;
    }
  }
}

// ===========================================================================
// query points: receptor nodes inside each pair's donor region
// (getQueryPoints2's exact test, |xd| <= dxc on all three axes), written in
// pair order then node order by an ordered two-pass compaction
// ===========================================================================
constexpr int kQThreads = 256;
constexpr int kQItems = 8;

__device__ __forceinline__ bool in_region(const double* p, const Obb& r) {
  double xd[3];
  for (int j = 0; j < 3; j++) {
    xd[j] = 0;
    for (int k = 0; k < 3; k++) xd[j] += (p[k] - r.xc[k]) * r.vec[j][k];
  }
  return fabs(xd[0]) <= r.dxc[0] && fabs(xd[1]) <= r.dxc[1] && fabs(xd[2]) <= r.dxc[2];
}

__global__ void __launch_bounds__(kQThreads) k_query_count(const double* __restrict__ x,
                                                           const BlockInfo* __restrict__ bi,
                                                           const PairInfo* __restrict__ pairs, int tiles_x,
                                                           int tile, int* __restrict__ tile_cnt) {
  const int p = blockIdx.y;
  const PairInfo& P = pairs[p];
  const BlockInfo& R = bi[P.rec];
  const Obb reg = P.region;
  int cnt = 0;
  for (int t = blockIdx.x; t < tiles_x; t += gridDim.x) {
    int n0 = t * tile;
    cnt = 0;
    for (int k = 0; k < kQItems; k++) {
      int i = n0 + threadIdx.x * kQItems + k;
      if (i < R.nnodes && in_region(x + 3 * ((long long)R.node_off + i), reg)) cnt++;
    }
    __shared__ int sh[kQThreads / 32];
    int w = cnt;
    for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = w;
    __syncthreads();
    if (threadIdx.x == 0) {
      int s = 0;
      for (int k = 0; k < kQThreads / 32; k++) s += sh[k];
      tile_cnt[(long long)p * tiles_x + t] = s;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kQThreads) k_query_write(const double* __restrict__ x,
                                                           const BlockInfo* __restrict__ bi,
                                                           const PairInfo* __restrict__ pairs, int tiles_x,
                                                           int tile, const int* __restrict__ tile_off,
                                                           const double* __restrict__ node_res,
                                                           int* __restrict__ qnode, int* __restrict__ qdon,
                                                           double* __restrict__ qres) {
  typedef cub::BlockScan<int, kQThreads> Scan;
  __shared__ typename Scan::TempStorage tmp;
  const int p = blockIdx.y;
  const PairInfo& P = pairs[p];
  const BlockInfo& R = bi[P.rec];
  const Obb reg = P.region;
  for (int t = blockIdx.x; t < tiles_x; t += gridDim.x) {
    int n0 = t * tile;
    unsigned mask = 0;
    int cnt = 0;
    for (int k = 0; k < kQItems; k++) {
      int i = n0 + threadIdx.x * kQItems + k;
      if (i < R.nnodes && in_region(x + 3 * ((long long)R.node_off + i), reg)) {
        mask |= 1u << k;
        cnt++;
      }
    }
    int pos;
    Scan(tmp).ExclusiveSum(cnt, pos);
    long long o = (long long)tile_off[(long long)p * tiles_x + t] + pos;
    for (int k = 0; k < kQItems; k++) {
      if (mask & (1u << k)) {
        int g = R.node_off + n0 + threadIdx.x * kQItems + k;
        qnode[o] = g;
        qdon[o] = P.don;
        qres[o] = node_res[g];
        o++;
      }
    }
    __syncthreads();
  }
}

// ===========================================================================
// fused tree search + containment
// ===========================================================================
// FP32 screen of the Newton inversion (hex 8, prism 6, pyramid 5) on
// coordinates relative to vertex 0.  Returns 0 reject, 1 clean interior
// accept, -1 undecided (the FP64 path decides).
__device__ __forceinline__ int screen32(const double xv[8][3], const double p[3], int nv) {
  constexpr float kEps = 2e-3f;
  float y[8][3], yp[3];
#pragma unroll
  for (int m = 0; m < 8; m++)
    if (m < nv)
#pragma unroll
      for (int j = 0; j < 3; j++) y[m][j] = (float)(xv[m][j] - xv[0][j]);
#pragma unroll
  for (int j = 0; j < 3; j++) yp[j] = (float)(p[j] - xv[0][j]);
  float f[8][3];
#pragma unroll
  for (int j = 0; j < 3; j++) {
    f[0][j] = -yp[j];
    if (nv == 8) {
      f[1][j] = y[1][j];
      f[2][j] = y[3][j];
      f[3][j] = y[4][j];
      f[4][j] = -y[1][j] + y[2][j] - y[3][j];
      f[5][j] = -y[3][j] + y[7][j] - y[4][j];
      f[6][j] = -y[1][j] + y[5][j] - y[4][j];
      f[7][j] = y[1][j] - y[2][j] + y[3][j] + y[4][j] - y[5][j] + y[6][j] - y[7][j];
    } else if (nv == 6) {
      f[1][j] = y[1][j];
      f[2][j] = y[2][j];
      f[3][j] = y[3][j];
      f[4][j] = 0.f;
      f[5][j] = -y[2][j] - y[3][j] + y[5][j];
      f[6][j] = -y[1][j] - y[3][j] + y[4][j];
      f[7][j] = 0.f;
    } else {
      f[1][j] = y[1][j];
      f[2][j] = y[3][j];
      f[3][j] = y[4][j];
      f[4][j] = -y[1][j] + y[2][j] - y[3][j];
      f[5][j] = -y[3][j];
      f[6][j] = -y[1][j];
      f[7][j] = y[1][j] - y[2][j] + y[3][j];
    }
  }
  float u = 0.5f, v = 0.5f, w = 0.5f;
  bool conv = false;
  float cond = 0.f;
  for (int it = 0; it < 16; it++) {
    float uv = u * v, vw = v * w, wu = w * u, uvw = uv * w;
    float r[3], J[3][3];
#pragma unroll
    for (int j = 0; j < 3; j++) {
      r[j] = __fmaf_rn(f[7][j], uvw, __fmaf_rn(f[6][j], wu, __fmaf_rn(f[5][j], vw, __fmaf_rn(f[4][j], uv,
             __fmaf_rn(f[3][j], w, __fmaf_rn(f[2][j], v, __fmaf_rn(f[1][j], u, f[0][j])))))));
      J[j][0] = __fmaf_rn(f[7][j], vw, __fmaf_rn(f[6][j], w, __fmaf_rn(f[4][j], v, f[1][j])));
      J[j][1] = __fmaf_rn(f[7][j], wu, __fmaf_rn(f[4][j], u, __fmaf_rn(f[5][j], w, f[2][j])));
      J[j][2] = __fmaf_rn(f[7][j], uv, __fmaf_rn(f[5][j], v, __fmaf_rn(f[6][j], u, f[3][j])));
    }
    float c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    float c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    float c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    float det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
    float n0 = sqrtf(J[0][0] * J[0][0] + J[1][0] * J[1][0] + J[2][0] * J[2][0]);
    float n1 = sqrtf(J[0][1] * J[0][1] + J[1][1] * J[1][1] + J[2][1] * J[2][1]);
    float n2 = sqrtf(J[0][2] * J[0][2] + J[1][2] * J[1][2] + J[2][2] * J[2][2]);
    float scale = n0 * n1 * n2;
    if (!(scale > 0.f)) return -1;
    cond = fabsf(det) / scale;
    if (cond < 1e-3f) return -1;  // near-singular map: let FP64 decide
    float id = 1.f / det;
    float du = (r[0] * c00 + r[1] * (J[0][2] * J[2][1] - J[0][1] * J[2][2]) +
                r[2] * (J[0][1] * J[1][2] - J[0][2] * J[1][1])) * id;
    float dv = (r[0] * c01 + r[1] * (J[0][0] * J[2][2] - J[0][2] * J[2][0]) +
                r[2] * (J[0][2] * J[1][0] - J[0][0] * J[1][2])) * id;
    float dw = (r[0] * c02 + r[1] * (J[0][1] * J[2][0] - J[0][0] * J[2][1]) +
                r[2] * (J[0][0] * J[1][1] - J[0][1] * J[1][0])) * id;
    u -= du;
    v -= dv;
    w -= dw;
    if (!(fabsf(u) < 1e3f && fabsf(v) < 1e3f && fabsf(w) < 1e3f)) return -1;
    if (fabsf(du) + fabsf(dv) + fabsf(dw) < 1e-6f) {
      conv = true;
      break;
    }
  }
  if (!conv) return -1;
  float fr[8];
  int n;
  if (nv == 8) {
    float a = 1.f - u, b = 1.f - v, c = 1.f - w;
    fr[0] = a * b * c; fr[1] = u * b * c; fr[2] = u * v * c; fr[3] = a * v * c;
    fr[4] = a * b * w; fr[5] = u * b * w; fr[6] = u * v * w; fr[7] = a * v * w;
    n = 8;
  } else if (nv == 6) {
    float a = 1.f - u - v, c = 1.f - w;
    fr[0] = a * c; fr[1] = u * c; fr[2] = v * c; fr[3] = a * w; fr[4] = u * w; fr[5] = v * w;
    n = 6;
  } else {
    float a = 1.f - u, b = 1.f - v, c = 1.f - w;
    fr[0] = a * b * c; fr[1] = u * b * c; fr[2] = u * v * c; fr[3] = a * v * c; fr[4] = w;
    n = 5;
  }
  bool interior = true;
  for (int m = 0; m < n; m++) {
    if (fr[m] < -kEps || fr[m] > 1.f + kEps) return 0;
    if (fr[m] < kEps || fr[m] > 1.f - kEps) interior = false;
  }
  return interior ? 1 : -1;
}

template <int FORM>
__global__ void __launch_bounds__(128) k_search(
    const double* __restrict__ x, const int* __restrict__ conn8, const unsigned char* __restrict__ cell_nv,
    const double* __restrict__ cell_res, const BlockInfo* __restrict__ bi, const int* __restrict__ sorted_cell,
    const float4* __restrict__ cbox, const double* __restrict__ cbox64, const float4* __restrict__ tnode,
    const double* __restrict__ tnode64, const int* __restrict__ qnode, const int* __restrict__ qdon,
    long long nq, int early_exit, int* __restrict__ qcell, unsigned char* __restrict__ qtie,
    unsigned long long* __restrict__ counters) {
  unsigned long long my_cand = 0, my_refine = 0, my_tie = 0, my_found = 0, my_verts = 0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    const int g = qnode[q];
    const int a = qdon[q];
    const int P = bi[a].P, toff = bi[a].tree_off, coff = bi[a].cell_off, nc = bi[a].ncells;
    const double p[3] = {x[3 * (long long)g], x[3 * (long long)g + 1], x[3 * (long long)g + 2]};
    const float p0 = (float)p[0], p1 = (float)p[1], p2 = (float)p[2];
    const float e0 = fabsf(p0) * 4.8e-7f + 1e-9f, e1 = fabsf(p1) * 4.8e-7f + 1e-9f,
                e2 = fabsf(p2) * 4.8e-7f + 1e-9f;
    int best_clean = 0x7fffffff, best_prov = 0x7fffffff, nacc = 0, nprov = 0;
    bool stop = false;
    int node = 0;
    for (;;) {
      bool hit;
      const long long gn = (long long)toff + node;
      if (FORM == 0) {
        const double* b = tnode64 + 6 * gn;
        hit = p[0] >= b[0] - kTol && p[1] >= b[1] - kTol && p[2] >= b[2] - kTol && p[0] <= b[3] + kTol &&
              p[1] <= b[4] + kTol && p[2] <= b[5] + kTol;
      } else {
        const float4 A = tnode[2 * gn], B = tnode[2 * gn + 1];
        hit = p0 >= A.x - e0 && p1 >= A.y - e1 && p2 >= A.z - e2 && p0 <= A.w + e0 && p1 <= B.x + e1 &&
              p2 <= B.y + e2;
      }
      if (hit) {
        if (node < P - 1) {
          node = 2 * node + 1;
          continue;
        }
        const int leaf = node - (P - 1);
        const int j0 = leaf * kLeafCells, j1 = min(j0 + kLeafCells, nc);
        for (int j = j0; j < j1 && !stop; j++) {
          const long long s = (long long)coff + j;
          bool pass;
          if (FORM == 0) {
            const double* b = cbox64 + 6 * s;
            const double lo[3] = {b[0], b[1], b[2]}, hi[3] = {b[3], b[4], b[5]};
            pass = in_box64(p, lo, hi);
          } else {
            const float4 A = cbox[2 * s], B = cbox[2 * s + 1];
            pass = p0 >= A.x - e0 && p1 >= A.y - e1 && p2 >= A.z - e2 && p0 <= A.w + e0 && p1 <= B.x + e1 &&
                   p2 <= B.y + e2;
          }
          if (!pass) continue;
          const int c = sorted_cell[s];
          const int nv = cell_nv[c];
          const int4 c0 = *reinterpret_cast<const int4*>(conn8 + 8 * (long long)c);
          const int4 c1 = *reinterpret_cast<const int4*>(conn8 + 8 * (long long)c + 4);
          const int cv[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
          double xv[8][3];
          gather_vertices(x, cv, nv, xv);
          if (FORM == 1) {  // exact FP64 element box (searchADTrecursion.C:63-66)
            double lo[3] = {xv[0][0], xv[0][1], xv[0][2]}, hi[3] = {xv[0][0], xv[0][1], xv[0][2]};
            for (int m = 1; m < nv; m++)
              for (int k = 0; k < 3; k++) {
                lo[k] = dmin(lo[k], xv[m][k]);
                hi[k] = dmax(hi[k], xv[m][k]);
              }
            if (!in_box64(p, lo, hi)) continue;
          }
          my_cand++;
          my_verts += nv;
          const bool big = cell_res[c] == kBig;
          int cls = -1;
          if (FORM == 1 && nv != 4) cls = screen32(xv, p, nv);
          if (cls < 0) {
            double frac[8];
            nodal_weights64(xv, p, frac, nv);
            cls = classify64(frac, nv, big);
            if (FORM == 1) my_refine++;
          } else if (cls == 1 && early_exit) {
            stop = true;
          }
          if (cls == 1) {
            nacc++;
            best_clean = min(best_clean, c);
          } else if (cls == 2) {
            nacc++;
            nprov++;
            best_prov = min(best_prov, c);
          }
        }
        if (stop) break;
      }
      while (node > 0 && !(node & 1)) node = (node - 1) >> 1;
      if (node == 0) break;
      node++;
    }
    int donor = (best_clean != 0x7fffffff) ? best_clean : ((best_prov != 0x7fffffff) ? best_prov : -1);
    qcell[q] = donor;
    unsigned char tie = (unsigned char)((nacc >= 2 ? 1 : 0) | (nprov >= 1 ? 2 : 0));
    qtie[q] = tie;
    my_tie += (tie != 0);
    my_found += (donor >= 0);
  }
  // counters: 0 candidates, 1 FP64 refinements, 2 ties, 3 found
  for (int o = 16; o > 0; o >>= 1) {
    my_cand += __shfl_xor_sync(0xffffffffu, my_cand, o);
    my_refine += __shfl_xor_sync(0xffffffffu, my_refine, o);
    my_tie += __shfl_xor_sync(0xffffffffu, my_tie, o);
    my_found += __shfl_xor_sync(0xffffffffu, my_found, o);
    my_verts += __shfl_xor_sync(0xffffffffu, my_verts, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&counters[0], my_cand);
    atomicAdd(&counters[1], my_refine);
    atomicAdd(&counters[2], my_tie);
    atomicAdd(&counters[3], my_found);
    atomicAdd(&counters[6], my_verts);
  }
}

void launch_search(int form, int blocks, int threads, cudaStream_t st, const double* x, const int* conn8,
                   const unsigned char* cell_nv, const double* cell_res, const BlockInfo* bi,
                   const int* sorted_cell, const float4* cbox, const double* cbox64, const float4* tnode,
                   const double* tnode64, const int* qnode, const int* qdon, long long nq, int early_exit,
                   int* qcell, unsigned char* qtie, unsigned long long* counters) {
  if (form == 0)
    k_search<0><<<blocks, threads, 0, st>>>(x, conn8, cell_nv, cell_res, bi, sorted_cell, cbox, cbox64, tnode,
                                            tnode64, qnode, qdon, nq, 0, qcell, qtie, counters);
  else
    k_search<1><<<blocks, threads, 0, st>>>(x, conn8, cell_nv, cell_res, bi, sorted_cell, cbox, cbox64, tnode,
                                            tnode64, qnode, qdon, nq, early_exit, qcell, qtie, counters);
}

}  // namespace tb
