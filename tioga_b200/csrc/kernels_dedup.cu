// Coincident query points: uniquenodes_octree / uniqNodesTree
// (src/utils.c:622-737), called by MeshBlock::search (src/search.C:242-263).
//
// The reference merges query points of one donor block that lie within TOL
// of each other (L1) and share the receptor mesh tag: the lower query index
// takes the larger receptor resolution, the higher one points to the lower
// one's representative (xtag), only representatives are searched and the
// others copy their donor, the donor side sends res_search[xtag[i]]
// (src/bookKeeping.C:108), and resetCoincident (src/bookKeeping.C:572-597)
// keeps a copy cancelled only if every copy is.
//
// Which points are compared, and in which order, follows the reference's
// octree exactly:
//  * a subset of more than 20 points is split at the middle of its bounding
//    box (widened by TOL) into octants, unless all of them fall into one
//    octant; the subsets depend only on the points, not on their order;
//  * each split reverses the order within an octant, so the points of a leaf
//    are in the donor list's order after an even number of splits and in the
//    reverse order after an odd number;
//  * the donor list's order is pair order, then the receptor block's
//    10x10x10 OBB bin (MeshBlock.C:171-224), then descending node id within a
//    bin, as getQueryPoints2 visits them (MeshBlock.C:953-1117).
// Here the subsets are emulated level by level on the device (exact FP64 box
// reductions with ordered keys, the reference's midpoint and octant
// arithmetic), and one thread per leaf runs the reference's pairwise loop in
// that order.
#include "kernels.cuh"

namespace tb {

// the 10x10x10 bin of every node in its block's OBB frame (MeshBlock.C:171-224)
__global__ void k_node_bins(const double* __restrict__ x, const blk_t* __restrict__ node_blk,
                            const BlockInfo* __restrict__ bi, long long ntot, short* __restrict__ node_bin) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
       g += (long long)gridDim.x * blockDim.x) {
    const Obb& o = bi[node_blk[g]].obb;
    int idx[3];
    for (int j = 0; j < 3; j++) {
      double xd = o.dxc[j];
      for (int k = 0; k < 3; k++) xd += (x[3 * g + k] - o.xc[k]) * o.vec[j][k];
      const double mdx = 2 * o.dxc[j] / 10;
      int i = (mdx > 0) ? (int)(xd / mdx) : 0;
      idx[j] = min(max(i, 0), 9);
    }
    node_bin[g] = (short)(idx[2] * 100 + idx[1] * 10 + idx[0]);
  }
}

// ---------------------------------------------------------------------------
// Preprocess gate: does any block hold two nodes closer than delta (L1)?
// Each node files itself under every cell of a per-block grid that its
// delta-box touches (one cell, rarely two per axis), so two such nodes always
// share a key; runs of equal keys are then compared pairwise.
// ---------------------------------------------------------------------------
constexpr int kCoinBits = 17;  // grid cells per axis: 2^17 (block id in the key's top 13 bits)

__device__ __forceinline__ void coin_frame(const BlockInfo& B, double& s, double& delta) {
  double ext = 0;
  for (int k = 0; k < 3; k++) ext = fmax(ext, (double)B.bb_hi[k] - (double)B.bb_lo[k]);
  s = fmax(ext / (double)(1 << kCoinBits), 40.0 * kTol);
  delta = 0.25 * s;
}

// the cell indices of axis k that p's delta-box touches: c0 .. c0 + n - 1
__device__ __forceinline__ void coin_axis(double p, double lo, double s, double delta, int& c0, int& n) {
  const int cmax = (1 << kCoinBits) - 1;
  const int c = min(max((int)floor((p - lo) / s), 0), cmax);
  const int a = min(max((int)floor((p - delta - lo) / s), 0), cmax);
  const int b = min(max((int)floor((p + delta - lo) / s), 0), cmax);
  c0 = min(a, c);
  n = max(b, c) - c0 + 1;
}

__global__ void k_coin_count(const double* __restrict__ x, const blk_t* __restrict__ node_blk,
                             const BlockInfo* __restrict__ bi, long long ntot, int* __restrict__ cnt) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
       g += (long long)gridDim.x * blockDim.x) {
    const BlockInfo& B = bi[node_blk[g]];
    double s, delta;
    coin_frame(B, s, delta);
    int m = 1;
    for (int k = 0; k < 3; k++) {
      int c0, n;
      coin_axis(x[3 * g + k], B.bb_lo[k], s, delta, c0, n);
      m *= n;
    }
    cnt[g] = m;
  }
}

__global__ void k_coin_fill(const double* __restrict__ x, const blk_t* __restrict__ node_blk,
                            const BlockInfo* __restrict__ bi, long long ntot, const int* __restrict__ off,
                            unsigned long long* __restrict__ key, int* __restrict__ val) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
       g += (long long)gridDim.x * blockDim.x) {
    const int b = node_blk[g];
    const BlockInfo& B = bi[b];
    double s, delta;
    coin_frame(B, s, delta);
    int c0[3], n[3];
    for (int k = 0; k < 3; k++) coin_axis(x[3 * g + k], B.bb_lo[k], s, delta, c0[k], n[k]);
    int o = off[g];
    for (int i = 0; i < n[0]; i++)
      for (int j = 0; j < n[1]; j++)
        for (int k = 0; k < n[2]; k++) {
          key[o] = ((unsigned long long)b << 51) | ((unsigned long long)(c0[0] + i) << 34) |
                   ((unsigned long long)(c0[1] + j) << 17) | (unsigned long long)(c0[2] + k);
          val[o] = (int)g;
          o++;
        }
  }
}

__global__ void k_coin_check(const unsigned long long* __restrict__ key, const int* __restrict__ val, long long n,
                             const double* __restrict__ x, const blk_t* __restrict__ node_blk,
                             const BlockInfo* __restrict__ bi, unsigned* __restrict__ flag) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x + 1; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (key[i] != key[i - 1]) continue;
    const int g = val[i];
    double s, delta;
    coin_frame(bi[node_blk[g]], s, delta);
    for (long long j = i - 1, steps = 0; j >= 0 && key[j] == key[i] && steps < 4096; j--, steps++) {
      const int h = val[j];
      const double d = fabs(x[3ll * g] - x[3ll * h]) + fabs(x[3ll * g + 1] - x[3ll * h + 1]) +
                       fabs(x[3ll * g + 2] - x[3ll * h + 2]);
      if (d < delta) {
        atomicOr(flag, 1u);
        return;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Per call: donor-list order of every query, then the octree emulation.
// ---------------------------------------------------------------------------
// key = pair | receptor bin | descending node id (the pairs are sorted by
// donor block, so a donor's pairs are consecutive and in list order); sorting
// the queries by it gives every donor's list in the reference's order (gpos =
// position in that sorted order)
__global__ void k_dedup_keys(const int* __restrict__ qnode, const int* __restrict__ qdon, long long nq,
                             const int* __restrict__ pair_qoff, int npairs, const int* __restrict__ pair_rank,
                             const short* __restrict__ node_bin, unsigned long long* __restrict__ key,
                             int* __restrict__ val) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = npairs - 1;  // the last pair whose first query is <= q
    while (lo < hi) {
      const int m = (lo + hi + 1) >> 1;
      if (pair_qoff[m] <= q) lo = m;
      else hi = m - 1;
    }
    const int g = qnode[q];
    key[q] = ((unsigned long long)lo << 41) | ((unsigned long long)node_bin[g] << 31) |
             (unsigned long long)(0x7fffffff - g);
    val[q] = (int)q;
  }
}

// the same for the high-order path's receptor points: within a pair the
// donor list holds them in point order (getExtraQueryPoints, highOrder.C:272-319)
__global__ void k_dedup_keys_pts(const int* __restrict__ qpt_local, const int* __restrict__ qdon, long long nq,
                                 const int* __restrict__ pair_qoff, int npairs, const int* __restrict__ pair_rank,
                                 unsigned long long* __restrict__ key, int* __restrict__ val) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = npairs - 1;
    while (lo < hi) {
      const int m = (lo + hi + 1) >> 1;
      if (pair_qoff[m] <= q) lo = m;
      else hi = m - 1;
    }
    key[q] = ((unsigned long long)lo << 40) | (unsigned long long)qpt_local[q];
    val[q] = (int)q;
  }
}

// gpos-indexed copies: point, receptor mesh tag, resolution, xtag = self
// (query q is point qnode[q] of x; its receptor block is node_blk[qnode[q]],
// or qrec[q] when node_blk is null)
__global__ void k_dedup_gather(const int* __restrict__ refq, long long n, const int* __restrict__ qnode,
                               const double* __restrict__ qres, const double* __restrict__ x,
                               const blk_t* __restrict__ node_blk, const int* __restrict__ qrec,
                               const BlockInfo* __restrict__ bi, double* __restrict__ xg, int* __restrict__ mtag,
                               double* __restrict__ rtag, int* __restrict__ itag, int* __restrict__ perm,
                               int* __restrict__ gpos_of) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int q = refq[i];
    const int g = qnode[q];
    for (int k = 0; k < 3; k++) xg[3 * i + k] = x[3ll * g + k];
    mtag[i] = bi[node_blk ? node_blk[g] : qrec[q]].tag;
    rtag[i] = qres[q];
    itag[i] = (int)i;
    perm[i] = (int)i;
    gpos_of[q] = (int)i;
  }
}

// a chunk of an active subset: positions [c.y, c.y + c.z) of subset c.x
__global__ void k_dedup_box(const int4* __restrict__ chunks, const int* __restrict__ perm,
                            const double* __restrict__ xg, unsigned long long* __restrict__ box) {
  const int4 c = chunks[blockIdx.x];
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = c.y + threadIdx.x; i < c.y + c.z; i += blockDim.x) {
    const double* p = xg + 3ll * perm[i];
    for (int k = 0; k < 3; k++) {
      lo[k] = dmin(lo[k], p[k]);
      hi[k] = dmax(hi[k], p[k]);
    }
  }
  for (int k = 0; k < 3; k++)
    for (int o = 16; o > 0; o >>= 1) {
      lo[k] = dmin(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
      hi[k] = dmax(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
    }
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 3; k++) {
      atomicMin(&box[6 * c.x + k], dkey(lo[k]));
      atomicMax(&box[6 * c.x + k + 3], dkey(hi[k]));
    }
}

// octant of every point of an active subset, counted per subset
// (uniqNodesTree: xmid = (xmax + xmin) * 0.5, dx = (xmax - xmin) * 0.5 + TOL,
// iv = floor((x - xmid) / dx) + 1, box = 4 iv0 + 2 iv1 + iv2)
__global__ void k_dedup_octant(const int4* __restrict__ chunks, const int* __restrict__ perm,
                               const double* __restrict__ xg, const unsigned long long* __restrict__ box,
                               unsigned char* __restrict__ oct, int* __restrict__ cnt) {
  __shared__ int s_cnt[8];
  __shared__ double s_mid[3], s_dx[3];
  const int4 c = chunks[blockIdx.x];
  if (threadIdx.x < 8) s_cnt[threadIdx.x] = 0;
  if (threadIdx.x < 3) {
    const double xmin = dkey_inv(box[6 * c.x + threadIdx.x]), xmax = dkey_inv(box[6 * c.x + threadIdx.x + 3]);
    s_mid[threadIdx.x] = (xmax + xmin) * 0.5;
    s_dx[threadIdx.x] = (xmax - xmin) * 0.5 + kTol;
  }
  __syncthreads();
  for (int i = c.y + threadIdx.x; i < c.y + c.z; i += blockDim.x) {
    const double* p = xg + 3ll * perm[i];
    int iv[3];
    for (int k = 0; k < 3; k++) {
      const double xp = p[k] - s_mid[k];
      iv[k] = min(max((int)floor(xp / s_dx[k]) + 1, 0), 1);
    }
    const int b = 4 * iv[0] + 2 * iv[1] + iv[2];
    oct[i] = (unsigned char)b;
    atomicAdd(&s_cnt[b], 1);
  }
  __syncthreads();
  if (threadIdx.x < 8 && s_cnt[threadIdx.x]) atomicAdd(&cnt[8 * c.x + threadIdx.x], s_cnt[threadIdx.x]);
}

// partition keys: subset start, then octant (0 outside splitting subsets)
__global__ void k_dedup_pkeys(const int* __restrict__ segstart, const unsigned char* __restrict__ oct, long long n,
                              unsigned long long* __restrict__ key) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    key[i] = ((unsigned long long)segstart[i] << 3) | oct[i];
}

// subset start of every position of the subsets in `chunks`
__global__ void k_dedup_segfill(const int4* __restrict__ chunks, const int* __restrict__ starts,
                                int* __restrict__ segstart) {
  const int4 c = chunks[blockIdx.x];
  for (int i = c.y + threadIdx.x; i < c.y + c.z; i += blockDim.x) segstart[i] = starts[c.x];
}

// the reference's pairwise loop over one leaf (uniqNodesTree, utils.c:693-713);
// leaf = (start, count, depth): members perm[start ..] in ascending donor-list
// order, visited in that order after an even number of splits, else reversed
__global__ void k_dedup_leaves(const int4* __restrict__ leaves, int nleaves, const int* __restrict__ perm,
                               const double* __restrict__ xg, const int* __restrict__ mtag,
                               double* __restrict__ rtag, int* __restrict__ itag) {
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < nleaves; l += gridDim.x * blockDim.x) {
    const int4 L = leaves[l];
    const int n = L.y;
    const bool rev = L.z & 1;
    for (int i = 0; i < n; i++) {
      const int p1 = perm[L.x + (rev ? n - 1 - i : i)];
      for (int j = i + 1; j < n; j++) {
        const int p2 = perm[L.x + (rev ? n - 1 - j : j)];
        if (fabs(xg[3ll * p1] - xg[3ll * p2]) + fabs(xg[3ll * p1 + 1] - xg[3ll * p2 + 1]) +
                    fabs(xg[3ll * p1 + 2] - xg[3ll * p2 + 2]) < kTol &&
            mtag[p1] == mtag[p2]) {
          if (p1 > p2) {
            rtag[p2] = dmax(rtag[p1], rtag[p2]);
            itag[p1] = itag[p2];
          } else {
            rtag[p1] = dmax(rtag[p1], rtag[p2]);
            itag[p2] = itag[p1];
          }
        }
      }
    }
  }
}

// per query: xtag (gpos), representative (query id; the one really searched,
// every xtag chain points to lower positions and ends there) and the
// receptor resolution the donor side reports, res_search[xtag[i]]
__global__ void k_dedup_apply(const int* __restrict__ refq, long long n, const int* __restrict__ itag,
                              const double* __restrict__ rtag, double* __restrict__ qres,
                              int* __restrict__ q_xt, int* __restrict__ q_rep, unsigned* __restrict__ err,
                              unsigned long long* __restrict__ counters) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int q = refq[i];
    const int xt = itag[i];
    qres[q] = rtag[xt];
    q_xt[q] = xt;
    int r = (int)i;
    for (int guard = 0; itag[r] != r; guard++) {
      if (guard > (1 << 20) || itag[r] > r) {
        atomicOr(err, kErrBadIndex);
        break;
      }
      r = itag[r];
    }
    q_rep[q] = refq[r];
    if (xt != (int)i) atomicAdd(&counters[7], 1ull);  // merged into another query
  }
}

// ---------------------------------------------------------------------------
// The node-global-id merge (uniquenode_map, search.C:48-74, in the build with
// TIOGA_HAS_NODEGID): in every donor's list (positions in the reference's
// order), the first query with a node id represents all later ones with that
// id and takes their largest resolution.  Positions are sorted stably by id,
// then by donor block, so each (donor, id) run is in position order.
// ---------------------------------------------------------------------------
__global__ void k_gid_keys(const int* __restrict__ refq, long long n, const int* __restrict__ qnode,
                           const int* __restrict__ qdon, const unsigned long long* __restrict__ node_gid,
                           unsigned long long* __restrict__ gkey, int* __restrict__ dkey16, int* __restrict__ pos) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int q = refq[i];
    gkey[i] = node_gid[qnode[q]];
    dkey16[i] = qdon[q];
    pos[i] = (int)i;
  }
}

// sorted index j: head of its (donor, id) run -> j, else 0 (a max-scan then
// gives every entry its run's first index)
__global__ void k_gid_heads(const int* __restrict__ pos, long long n, const unsigned long long* __restrict__ gkey_of_pos,
                            const int* __restrict__ don_of_pos, int* __restrict__ head) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    bool h = j == 0;
    if (!h) {
      const int a = pos[j], b = pos[j - 1];
      h = gkey_of_pos[a] != gkey_of_pos[b] || don_of_pos[a] != don_of_pos[b];
    }
    head[j] = h ? (int)j : 0;
  }
}

// itag[position] = its run's first position; the run's largest resolution at
// that first position (ordered keys, exact)
__global__ void k_gid_apply(const int* __restrict__ pos, const int* __restrict__ first, long long n,
                            int* __restrict__ itag, const double* __restrict__ rtag,
                            unsigned long long* __restrict__ rmax) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    const int rep = pos[first[j]];
    itag[pos[j]] = rep;
    atomicMax(&rmax[rep], dkey(rtag[pos[j]]));
  }
}

__global__ void k_gather_i32(const int* __restrict__ src, const int* __restrict__ idx, long long n,
                             int* __restrict__ out) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x)
    out[j] = src[idx[j]];
}

__global__ void k_gid_res(const int* __restrict__ itag, long long n, const unsigned long long* __restrict__ rmax,
                          double* __restrict__ rtag) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    if (itag[i] == (int)i) rtag[i] = dkey_inv(rmax[i]);
}

// after the search: a merged query takes its representative's donor
__global__ void k_dedup_copy(const int* __restrict__ q_rep, long long nq, int* __restrict__ qcell,
                             unsigned char* __restrict__ qtie) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    const int r = q_rep[q];
    if (r != q) {
      qcell[q] = qcell[r];
      qtie[q] = qtie[r];
    }
  }
}

// resetCoincident (bookKeeping.C:572-597): over the records of the donor's
// queries, a cancelled record stays cancelled only if every record sharing
// its xtag is
__global__ void k_reset_coincident_min(const int* __restrict__ interp2rec, const int* __restrict__ q_xt,
                                       long long nq, const unsigned char* __restrict__ it_cancel,
                                       int* __restrict__ ireset) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    const int r = interp2rec[q];
    if (r >= 0) atomicMin(&ireset[q_xt[q]], (int)it_cancel[r]);
  }
}

__global__ void k_reset_coincident_set(const int* __restrict__ interp2rec, const int* __restrict__ q_xt,
                                       long long nq, const int* __restrict__ ireset,
                                       unsigned char* __restrict__ it_cancel) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    const int r = interp2rec[q];
    if (r >= 0 && it_cancel[r] == 1) it_cancel[r] = (unsigned char)ireset[q_xt[q]];
  }
}

}  // namespace tb
