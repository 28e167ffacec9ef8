// Preprocess kernels: connectivity upload, node->cell incidence lists, cell
// volumes, node resolutions, oriented bounding boxes, mandatory receptors and
// the mexclude sweeps (src/MeshBlock.C:74-339, src/utils.c:25-165).
#include "kernels.cuh"

namespace tb {

// ---------------------------------------------------------------------------
// connectivity: 1-based per-type arrays -> padded 8-wide global node ids
// ---------------------------------------------------------------------------
// 1-based caller connectivity -> padded global ids.  An index outside
// 1..nnodes is replaced by the block's first node and reported (kErrBadInput):
// the registration then fails before any kernel reads the cell.
__global__ void k_conn_convert(const int* __restrict__ raw, int nc, int nv, int node_off, int nnodes,
                               int cell_base, int blk, int* __restrict__ conn8,
                               unsigned char* __restrict__ cell_nv, blk_t* __restrict__ cell_blk,
                               unsigned* __restrict__ err) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nc;
       i += (long long)gridDim.x * blockDim.x) {
    long long c = cell_base + i;
    int v[8];
#pragma unroll
    for (int m = 0; m < 8; m++) {
      int r = (m < nv) ? raw[i * nv + m] : 1;
      if (r < 1 || r > nnodes) {
        atomicOr(err, kErrBadInput);
        r = 1;
      }
      v[m] = (m < nv) ? node_off + r - 1 : -1;
    }
    int4* dst = reinterpret_cast<int4*>(conn8 + 8 * c);
    dst[0] = make_int4(v[0], v[1], v[2], v[3]);
    dst[1] = make_int4(v[4], v[5], v[6], v[7]);
    cell_nv[c] = (unsigned char)nv;
    cell_blk[c] = (blk_t)blk;
  }
}

// every coordinate finite, else kErrBadInput (the call then stops before any
// kernel derives an index from a coordinate)
__global__ void k_check_finite(const double* __restrict__ x, long long n, unsigned* __restrict__ err) {
  bool bad = false;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    bad = bad || !isfinite(x[i]);
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(err, kErrBadInput);
}

__global__ void k_node_blk(int node_off, int nnodes, int blk, blk_t* node_blk) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nnodes;
       i += (long long)gridDim.x * blockDim.x)
    node_blk[node_off + i] = (blk_t)blk;
}

// wall or overset-boundary node list (1-based); an index outside 1..nnodes is
// replaced by the first node and reported (kErrBadInput)
__global__ void k_mark_list(const int* __restrict__ list, int n, int node_off, int nnodes, int* __restrict__ glist,
                            int goff, unsigned char* __restrict__ flag, unsigned* __restrict__ err) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    int r = list[i];
    if (r < 1 || r > nnodes) {
      atomicOr(err, kErrBadInput);
      r = 1;
    }
    int g = node_off + r - 1;
    glist[goff + i] = g;
    flag[g] = 1;
  }
}

// ---------------------------------------------------------------------------
// node -> cell incidence lists (CSR), each list sorted by cell id so that the
// node resolution sums in the reference's cell order (MeshBlock.C:129-156)
// ---------------------------------------------------------------------------
__global__ void k_csr_count(const int* __restrict__ conn8, const unsigned char* __restrict__ cell_nv,
                            long long ctot, int* __restrict__ deg) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ctot;
       c += (long long)gridDim.x * blockDim.x) {
    int nv = cell_nv[c];
    for (int m = 0; m < nv; m++) atomicAdd(&deg[conn8[8 * c + m]], 1);
  }
}

__global__ void k_csr_fill(const int* __restrict__ conn8, const unsigned char* __restrict__ cell_nv,
                           long long ctot, const int* __restrict__ off, int* __restrict__ cursor,
                           int* __restrict__ cells) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ctot;
       c += (long long)gridDim.x * blockDim.x) {
    int nv = cell_nv[c];
    for (int m = 0; m < nv; m++) {
      int g = conn8[8 * c + m];
      int pos = atomicAdd(&cursor[g], 1);
      cells[off[g] + pos] = (int)c;
    }
  }
}

__global__ void k_csr_sort(const int* __restrict__ off, long long ntot, int* __restrict__ cells) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
       g += (long long)gridDim.x * blockDim.x) {
    int a = off[g], b = off[g + 1];
    for (int i = a + 1; i < b; i++) {
      int key = cells[i];
      int j = i - 1;
      while (j >= a && cells[j] > key) {
        cells[j + 1] = cells[j];
        j--;
      }
      cells[j + 1] = key;
    }
  }
}

// ---------------------------------------------------------------------------
// cell volumes and node resolutions (MeshBlock.C:129-196)
// ---------------------------------------------------------------------------
__global__ void k_cell_volume(const double* __restrict__ x, const int* __restrict__ conn8,
                              const unsigned char* __restrict__ cell_nv,
                              const blk_t* __restrict__ cell_blk,
                              const BlockInfo* __restrict__ bi, long long ctot,
                              double* __restrict__ cell_res) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ctot;
       c += (long long)gridDim.x * blockDim.x) {
    if (bi[cell_blk[c]].has_user_res) continue;
    int nv = cell_nv[c];
    double xv[8][3];
    gather_vertices(x, conn8 + 8 * c, nv, xv);
    cell_res[c] = cell_volume64(xv, nv) * 1.0;  // resolutionScale == 1
  }
}

__global__ void k_node_res(const int* __restrict__ off, const int* __restrict__ cells,
                           const double* __restrict__ cell_res, const blk_t* __restrict__ node_blk,
                           const BlockInfo* __restrict__ bi, long long ntot, double* __restrict__ node_res) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
       g += (long long)gridDim.x * blockDim.x) {
    if (bi[node_blk[g]].has_user_res) continue;
    int a = off[g], b = off[g + 1];
    double s = 0.0;
    for (int i = a; i < b; i++) s += cell_res[cells[i]];
    if (b - a != 0) s /= (b - a);
    node_res[g] = s;
  }
}

// nodes of cells touching an overset-boundary node: nodeRes = BIG and the
// first mexclude frontier (MeshBlock.C:230-284)
__global__ void k_mandatory(const int* __restrict__ conn8, const unsigned char* __restrict__ cell_nv,
                            long long ctot, const unsigned char* __restrict__ obcf,
                            double* __restrict__ node_res, unsigned char* __restrict__ ex0,
                            unsigned char* __restrict__ ex1) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ctot;
       c += (long long)gridDim.x * blockDim.x) {
    int nv = cell_nv[c];
    const int* cv = conn8 + 8 * c;
    int tagged = 0;
    for (int m = 0; m < nv; m++) tagged |= obcf[cv[m]];
    if (!tagged) continue;
    for (int m = 0; m < nv; m++) {
      node_res[cv[m]] = kBig;
      ex0[cv[m]] = 1;
      ex1[cv[m]] = 1;
    }
  }
}

// one mexclude round (MeshBlock.C:307-335): cells touching the frontier may
// not donate and their nodes join the next frontier
__global__ void k_mexclude(const int* __restrict__ conn8, const unsigned char* __restrict__ cell_nv,
                           long long ctot, const unsigned char* __restrict__ ex0,
                           unsigned char* __restrict__ ex1, double* __restrict__ cell_res) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ctot;
       c += (long long)gridDim.x * blockDim.x) {
    int nv = cell_nv[c];
    const int* cv = conn8 + 8 * c;
    int hit = 0;
    for (int m = 0; m < nv; m++) hit |= (ex0[cv[m]] == 1);
    if (hit) cell_res[c] = kBig;
    if (cell_res[c] == kBig)
      for (int m = 0; m < nv; m++)
        if (ex0[cv[m]] != 1) ex1[cv[m]] = 1;
  }
}

__global__ void k_copy_u8(const unsigned char* __restrict__ a, unsigned char* __restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = a[i];
}

__global__ void k_fill_int(int* __restrict__ a, int v, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    a[i] = v;
}

// ---------------------------------------------------------------------------
// oriented bounding box of a node range (utils.c:25-165).  The sums are
// reduced per CTA and then in CTA order, so the result is reproducible (the
// reference sums sequentially; the box only culls, so the rounding of its
// last bits cannot change a result).
// ---------------------------------------------------------------------------
// Every block at once: blockIdx.y is the block, gridDim.x CTAs share its
// nodes (the same split for any number of blocks, so a block's box does not
// depend on the others).
__global__ void k_obb_partial(const double* __restrict__ x, const BlockInfo* __restrict__ bi, int pass,
                              double* __restrict__ part_all) {
  // pass 0: sums of x; pass 1: covariance; pass 2: min/max of the projections
  // and of the raw coordinates
  const BlockInfo& B = bi[blockIdx.y];
  const int off = B.node_off, n = B.nnodes;
  if (n == 0 || (pass == 1 && n < 4)) return;
  const Obb* __restrict__ obb = &B.obb;
  double* __restrict__ part = part_all + 12 * (size_t)gridDim.x * blockIdx.y;
  double acc[12];
  for (int k = 0; k < 12; k++) acc[k] = (pass == 2) ? ((k % 2 == 0) ? 1e300 : -1e300) : 0.0;
  double xc0 = 0, xc1 = 0, xc2 = 0;
  if (pass >= 1) {
    xc0 = obb->xc[0];
    xc1 = obb->xc[1];
    xc2 = obb->xc[2];
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double* p = x + 3 * ((long long)off + i);
    if (pass == 0) {
      acc[0] += p[0];
      acc[1] += p[1];
      acc[2] += p[2];
    } else if (pass == 1) {
      double a = p[0] - xc0, b = p[1] - xc1, c = p[2] - xc2;
      acc[0] += a * a;
      acc[1] += b * b;
      acc[2] += c * c;
      acc[3] += a * b;
      acc[4] += a * c;
      acc[5] += b * c;
    } else {
      for (int j = 0; j < 3; j++) {
        double xd = 0;
        for (int k = 0; k < 3; k++) xd += (p[k] - obb->xc[k]) * obb->vec[j][k];
        acc[2 * j] = dmin(acc[2 * j], xd);
        acc[2 * j + 1] = dmax(acc[2 * j + 1], xd);
        acc[6 + 2 * j] = dmin(acc[6 + 2 * j], p[j]);
        acc[6 + 2 * j + 1] = dmax(acc[6 + 2 * j + 1], p[j]);
      }
    }
  }
  __shared__ double sh[256 * 12];
  for (int k = 0; k < 12; k++) sh[threadIdx.x * 12 + k] = acc[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    double r[12];
    for (int k = 0; k < 12; k++) r[k] = sh[k];
    for (int t = 1; t < blockDim.x; t++)
      for (int k = 0; k < 12; k++) {
        double v = sh[t * 12 + k];
        if (pass == 2) r[k] = (k % 2 == 0) ? dmin(r[k], v) : dmax(r[k], v);
        else r[k] += v;
      }
    for (int k = 0; k < 12; k++) part[blockIdx.x * 12 + k] = r[k];
  }
}

// src/kaiser.f:29-180 (Kaiser's JK eigen method), one thread
__device__ void kaiser3(double* a, double* eigenv) {
  const int n = 3, nrows = 3;
#define A_(i, j) a[((j)-1) * nrows + ((i)-1)]
  double ss = 0.0, trace = 0.0;
  for (int j = 1; j <= n; j++) {
    trace = trace + A_(j, j);
    for (int i = 1; i <= n; i++) ss = ss + A_(i, j) * A_(i, j);
  }
  double eps = 1.0e-12 * ss / n;
  int nn = n * (n - 1) / 2, ncount = nn;
  bool done = false;
  for (int iter = 0; iter < 10 && !done; iter++) {
    for (int j = 1; j <= n - 1 && !done; j++)
      for (int k = j + 1; k <= n; k++) {
        double halfp = 0.0, q = 0.0;
        for (int i = 1; i <= n; i++) {
          double xj = A_(i, j), xk = A_(i, k);
          halfp = halfp + xj * xk;
          q = q + (xj + xk) * (xj - xk);
        }
        double p = halfp + halfp, absp = fabs(p);
        if (absp < eps && q >= 0.0) {
          ncount = ncount - 1;
          if (ncount <= 0) {
            done = true;
            break;
          }
          continue;
        }
        double absq = fabs(q), cs, sn;
        if (absp <= absq) {
          double tn = absp / absq;
          cs = 1.0 / sqrt(1.0 + tn * tn);
          sn = tn * cs;
        } else {
          double ctn = absq / absp;
          sn = 1.0 / sqrt(1.0 + ctn * ctn);
          cs = ctn * sn;
        }
        cs = sqrt((1.0 + cs) * 0.5);
        sn = sn / (cs + cs);
        if (q < 0.0) {
          double t = cs;
          cs = sn;
          sn = t;
        }
        if (p < 0.0) sn = -sn;
        for (int i = 1; i <= n; i++) {
          double t = A_(i, j);
          A_(i, j) = t * cs + A_(i, k) * sn;
          A_(i, k) = -t * sn + A_(i, k) * cs;
        }
      }
    if (!done) ncount = nn;
  }
  for (int j = 1; j <= n; j++) {
    double t = 0.0;
    for (int i = 1; i <= n; i++) t = t + A_(i, j) * A_(i, j);
    eigenv[j - 1] = sqrt(t);
  }
  for (int j = 1; j <= n; j++) {
    double t = (eigenv[j - 1] > 0.0) ? 1.0 / eigenv[j - 1] : 0.0;
    for (int i = 1; i <= n; i++) A_(i, j) = A_(i, j) * t;
  }
#undef A_
}

__global__ void k_obb_finish(const double* __restrict__ part_all, int nparts, int pass, const double* __restrict__ x,
                             BlockInfo* __restrict__ bi_all, int nb) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  BlockInfo* __restrict__ bi = bi_all + b;
  const int off = bi->node_off, n = bi->nnodes;
  if (n == 0 || (pass == 1 && n < 4)) return;
  const double* __restrict__ part = part_all + 12 * (size_t)nparts * b;
  Obb* __restrict__ obb = &bi->obb;
  double r[12];
  for (int k = 0; k < 12; k++) r[k] = part[k];
  for (int t = 1; t < nparts; t++)
    for (int k = 0; k < 12; k++) {
      double v = part[t * 12 + k];
      if (pass == 2) r[k] = (k % 2 == 0) ? dmin(r[k], v) : dmax(r[k], v);
      else r[k] += v;
    }
  Obb& o = *obb;
  if (pass == 0) {
    o.xc[0] = r[0] / n;
    o.xc[1] = r[1] / n;
    o.xc[2] = r[2] / n;
    if (n < 4) {  // utils.c:52-83
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) o.vec[i][j] = (i == j) ? 1.0 : 0.0;
      const double* p = x + 3 * (long long)off;
      if (n == 1) {
        o.dxc[0] = o.dxc[1] = o.dxc[2] = 1e-3;
      } else if (n == 2) {
        for (int j = 0; j < 3; j++) o.dxc[j] = dmax(1e-3, fabs(p[3 + j] - p[j])) * 0.5;
      } else {
        for (int i = 0; i < n; i++)
          for (int j = 0; j < 3; j++) o.dxc[j] = dmax(1e-3, fabs(p[3 * i + j] - p[0]));
      }
    }
  } else if (pass == 1) {
    double aa[9], eig[3];
    aa[0] = r[0];
    aa[4] = r[1];
    aa[8] = r[2];
    aa[3] = r[3];
    aa[6] = r[4];
    aa[7] = r[5];
    aa[1] = aa[3];
    aa[2] = aa[6];
    aa[5] = aa[7];
    kaiser3(aa, eig);
    for (int i = 0, m = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) o.vec[i][j] = aa[m++];
  } else if (n < 4) {  // the box stays as set from the points; the raw box feeds the Morton keys
    for (int j = 0; j < 3; j++) {
      bi->bb_lo[j] = (float)r[6 + 2 * j];
      bi->bb_hi[j] = (float)r[6 + 2 * j + 1];
    }
    return;
  } else {
    double xd[3];
    for (int j = 0; j < 3; j++) {
      o.dxc[j] = (r[2 * j + 1] - r[2 * j]) * 0.5 * 1.01;
      xd[j] = (r[2 * j + 1] + r[2 * j]) * 0.5;
    }
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++) o.xc[j] += (xd[k] * o.vec[k][j]);
    for (int j = 0; j < 3; j++) {
      bi->bb_lo[j] = (float)r[6 + 2 * j];
      bi->bb_hi[j] = (float)r[6 + 2 * j + 1];
    }
  }
  bi->obb = o;
}

// ---------------------------------------------------------------------------
// Morton keys of cell centroids, block id in the high word
// ---------------------------------------------------------------------------
__device__ inline unsigned spread10(unsigned v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

__global__ void k_morton(const double* __restrict__ x, const int* __restrict__ conn8,
                         const unsigned char* __restrict__ cell_nv,
                         const blk_t* __restrict__ cell_blk, const BlockInfo* __restrict__ bi,
                         long long ctot, unsigned long long* __restrict__ key, int* __restrict__ val) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ctot;
       c += (long long)gridDim.x * blockDim.x) {
    int nv = cell_nv[c], b = cell_blk[c];
    const int* cv = conn8 + 8 * c;
    double s[3] = {0, 0, 0};
    for (int m = 0; m < nv; m++)
      for (int j = 0; j < 3; j++) s[j] += x[3 * (long long)cv[m] + j];
    unsigned code = 0;
    for (int j = 0; j < 3; j++) {
      float lo = bi[b].bb_lo[j], hi = bi[b].bb_hi[j];
      float t = (hi > lo) ? (float)(s[j] / nv - lo) / (hi - lo) : 0.f;
      t = fminf(fmaxf(t, 0.f), 1.f);
      unsigned q = (unsigned)(t * 1023.f);
      code |= spread10(q) << j;
    }
    key[c] = ((unsigned long long)b << 32) | code;
    val[c] = (int)c;
  }
}

// Morton keys of node positions, block id in the high word (the order in
// which query points are gathered, so a warp's queries are neighbours)
__global__ void k_morton_nodes(const double* __restrict__ x, const blk_t* __restrict__ node_blk,
                               const BlockInfo* __restrict__ bi, long long ntot, unsigned long long* __restrict__ key,
                               int* __restrict__ val) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
       g += (long long)gridDim.x * blockDim.x) {
    const int b = node_blk[g];
    unsigned code = 0;
    for (int j = 0; j < 3; j++) {
      float lo = bi[b].bb_lo[j], hi = bi[b].bb_hi[j];
      float t = (hi > lo) ? (float)(x[3 * g + j] - lo) / (hi - lo) : 0.f;
      t = fminf(fmaxf(t, 0.f), 1.f);
      code |= spread10((unsigned)(t * 1023.f)) << j;
    }
    key[g] = ((unsigned long long)b << 32) | code;
    val[g] = (int)g;
  }
}

// Cell arrays from registration order to storage (Morton) order:
// dst[s] = src[perm[s]].
__global__ void k_permute_cells(const int* __restrict__ perm, long long n, const int* __restrict__ conn8,
                                const unsigned char* __restrict__ nv, const blk_t* __restrict__ blk,
                                int* __restrict__ conn8_out, unsigned char* __restrict__ nv_out,
                                blk_t* __restrict__ blk_out) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n;
       s += (long long)gridDim.x * blockDim.x) {
    const long long c = perm[s];
    const int4* src = reinterpret_cast<const int4*>(conn8 + 8 * c);
    int4* dst = reinterpret_cast<int4*>(conn8_out + 8 * s);
    dst[0] = src[0];
    dst[1] = src[1];
    nv_out[s] = nv[c];
    blk_out[s] = blk[c];
  }
}

// idx[i] = map[idx[i]] (node->cell lists from registration to storage ids;
// each list keeps its registration order, the order of the reference's sums)
__global__ void k_remap(int* __restrict__ idx, long long n, const int* __restrict__ map) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    idx[i] = map[idx[i]];
}

// dst[inv[c]] = src[c] for doubles (user cell resolutions into storage order)
__global__ void k_scatter_f64(const double* __restrict__ src, long long n, const int* __restrict__ inv,
                              long long base, double* __restrict__ dst) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x)
    dst[inv[base + c]] = src[c];
}

__global__ void k_invert(const int* __restrict__ perm, long long n, int* __restrict__ inv) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n;
       s += (long long)gridDim.x * blockDim.x)
    inv[perm[s]] = (int)s;
}

// x <- a x + b for n nodes, each product and sum in a fixed order (the same
// bits as the same expression evaluated on the host without contraction)
__global__ void k_rigid(double* __restrict__ x, int n, Rigid m) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double* p = x + 3 * (long long)i;
    const double x0 = p[0], x1 = p[1], x2 = p[2];
    for (int k = 0; k < 3; k++) p[k] = ((m.a[3 * k] * x0 + m.a[3 * k + 1] * x1) + m.a[3 * k + 2] * x2) + m.b[k];
  }
}

}  // namespace tb
