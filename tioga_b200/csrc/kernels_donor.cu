// Donor bookkeeping kernels (src/exchangeDonors.C:25-301,
// src/bookKeeping.C:74-648, src/linklist.c:62-104), cell iblanks
// (src/highOrder.C:88-150) and the data-update gather/scatter
// (src/dataUpdate.C:27-119, src/tioga.C:336-524).
#include "kernels.cuh"

namespace tb {

constexpr int kMaxK = 16;  // donor blocks a receptor node can hear from

struct Cand {
  double dres;
  int a, q;
};

// The receptor node's donor list: one candidate per donor block, delivered in
// donor-block order and inserted before the first entry whose |donorRes|
// exceeds the new one (linklist.c:62-104).  Returns the list length.
__device__ __forceinline__ int donor_list(long long g, const int* __restrict__ slot, int K,
                                          const int* __restrict__ qcell, const double* __restrict__ cell_res,
                                          Cand* L) {
  int n = 0;
  for (int a = 0; a < K; a++) {
    int q = slot[g * K + a];
    if (q < 0) continue;
    const int cell = qcell[q];
    if (cell < 0) continue;  // slots are only set for queries with a donor
    Cand c{cell_res[cell], a, q};
    int pos = n;
    for (int k = 0; k < n; k++)
      if (fabs(L[k].dres) > c.dres) {
        pos = k;
        break;
      }
    for (int k = n; k > pos; k--) L[k] = L[k - 1];
    L[pos] = c;
    n++;
  }
  return n;
}

__global__ void k_fill_slots(const int* __restrict__ qnode, const int* __restrict__ qdon,
                             const int* __restrict__ qcell, long long nq, int K, long long ntot,
                             long long ctot, const BlockInfo* __restrict__ bi, int nb, int* __restrict__ slot,
                             unsigned* __restrict__ err) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    const int c = qcell[q];
    if (c < 0) continue;
    const int g = qnode[q], d = qdon[q];
    const int a = (d >= 0 && d < nb) ? d - bi[d].sblk0 : -1;  // the donor's index within its system
    if (c >= ctot || g < 0 || g >= ntot || a < 0 || a >= K) {
      atomicOr(err, kErrBadIndex);
      continue;
    }
    slot[(long long)g * K + a] = (int)q;
  }
}

// ---------------------------------------------------------------------------
// Sparse donor phase.  Only a small part of the nodes is ever touched: the
// queried nodes with a donor, the nodes inside a foreign wall mesh's hole
// map, the nfringe layers around the holes and the donor cells' vertices.
// Every per-node state array (iblank, m0/m1, slot, cmark, reset_t) is kept in
// its rest state between calls, and each call undoes exactly what the
// previous one marked, from its lists.  mlist holds the holes first
// (dcnt[kHoles] of them) and then the nfringe layers (dcnt[kMarked] in all).
// ---------------------------------------------------------------------------

// first donor block with a candidate for node g is the node's owner query
__device__ __forceinline__ bool owner_query(const int* __restrict__ slot, int K, long long g, int q) {
  for (int a = 0; a < K; a++) {
    const int s = slot[g * K + a];
    if (s >= 0) return s == q;
  }
  return false;
}

__device__ __forceinline__ void mark_hole(int g, int* __restrict__ iblank, unsigned char* __restrict__ m0,
                                          int* __restrict__ m1, int* __restrict__ mlist, int* __restrict__ dcnt,
                                          unsigned long long* __restrict__ counters) {
  iblank[g] = 0;
  m0[g] = 1;
  m1[g] = 1;
  mlist[atomicAdd(&dcnt[kMarked], 1)] = g;
  atomicAdd(&counters[4], 1ull);
}

// Start of a call: back to the rest state from the previous call's lists
// (holes and kept receptors -> iblank 1 and their cells' iblank 1; marked
// nodes -> m0 = m1 = 0).  prev_R records of the previous call.
__global__ void k_donor_reset(const int* __restrict__ mlist, const int* __restrict__ dcnt,
                              const int* __restrict__ it_rec, const unsigned char* __restrict__ it_cancel,
                              int prev_R, const int* __restrict__ csr_off, const int* __restrict__ csr_cell,
                              int* __restrict__ iblank, unsigned char* __restrict__ m0, int* __restrict__ m1,
                              int* __restrict__ iblank_cell) {
  const int nh = dcnt[kHoles], nm = dcnt[kMarked];
  const int n = max(nm, nh + prev_R);
  const int lane = threadIdx.x & 31;  // a warp per entry, its lanes over the node's cells
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    if (i < nm && lane == 0) {
      m0[mlist[i]] = 0;
      m1[mlist[i]] = 0;
    }
    int v = -1;  // a node that ended the previous call with iblank 0 or -1
    if (i < nh) v = mlist[i];
    else if (i < nh + prev_R) v = it_rec[i - nh];  // cancelled ones too (reduce_fringes may have holed them)
    if (v < 0) continue;
    if (lane == 0) iblank[v] = 1;
    for (int k = csr_off[v] + lane; k < csr_off[v + 1]; k += 32) iblank_cell[csr_cell[k]] = 1;
  }
}

// processDonors first pass (bookKeeping.C:158-237) for the queried nodes that
// have donors: holes from the hole maps of wall-bearing meshes that supplied
// none of them, node resolution raised to the candidates' receptor
// resolutions.  One thread per node (its owner query).
__global__ void k_classify_queried(const double* __restrict__ x, const blk_t* __restrict__ node_blk,
                                   const BlockInfo* __restrict__ bi, const int* __restrict__ slot, int K,
                                   const int* __restrict__ qnode, const int* __restrict__ qcell, long long nq,
                                   const double* __restrict__ qres, const HoleMapDev* __restrict__ hm,
                                   int* __restrict__ iblank, double* __restrict__ node_res,
                                   unsigned char* __restrict__ m0, int* __restrict__ m1, int* __restrict__ mlist,
                                   int* __restrict__ dcnt, unsigned long long* __restrict__ counters) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    if (qcell[q] < 0) continue;
    const int g = qnode[q];
    if (!owner_query(slot, K, g, (int)q)) continue;
    const BlockInfo& B = bi[node_blk[g]];
    const int tag = B.tag;
    unsigned long long seen[2] = {0ull, 0ull};
    double nres = node_res[g];
    for (int a = 0; a < K; a++) {
      const int s = slot[(long long)g * K + a];
      if (s < 0) continue;
      const int t = bi[B.sblk0 + a].tag - 1;
      seen[t >> 6] |= 1ull << (t & 63);
      nres = dmax(nres, qres[s]);
    }
    const double p[3] = {x[3 * (long long)g], x[3 * (long long)g + 1], x[3 * (long long)g + 2]};
    bool hole = false;
    for (int h = B.hm_lo; h < B.hm_hi && !hole; h++) {
      const int ht = hm[h].tagidx;
      if (ht == tag - 1 || ((seen[ht >> 6] >> (ht & 63)) & 1ull)) continue;
      hole = check_holemap(p, hm[h]) != 0;
    }
    node_res[g] = nres;
    if (hole) mark_hole(g, iblank, m0, m1, mlist, dcnt, counters);
  }
}

// The same pass for nodes without a donor: every foreign wall mesh's hole
// map applies.  One CTA per tile of kNodeTile Morton-ordered nodes; only
// tiles whose box meets a foreign hole map's reach are walked.  A point is
// in a map only if it lies within one map cell beyond the map's extent (the
// index truncates toward zero), so the reach is the extent widened by one
// cell and rounded outward.
__global__ void __launch_bounds__(256) k_classify_tiles(
    const double* __restrict__ x, const BlockInfo* __restrict__ bi, int nb, const long long* __restrict__ tile_base,
    const float4* __restrict__ tbox, const int* __restrict__ node_order, const int* __restrict__ slot, int K,
    const HoleMapDev* __restrict__ hm, int* __restrict__ iblank, unsigned char* __restrict__ m0,
    int* __restrict__ m1, int* __restrict__ mlist, int* __restrict__ dcnt, unsigned long long* __restrict__ counters) {
  __shared__ unsigned s_maps;  // foreign maps that reach the tile (bit h; all bits set past 32 maps)
  const long long T = blockIdx.x;
  const int b = block_of_tile(tile_base, nb, T);
  const BlockInfo& B = bi[b];
  if (threadIdx.x == 0) {
    const float4 A = tbox[2 * T], C = tbox[2 * T + 1];
    const float lo[3] = {A.x, A.y, A.z}, hi[3] = {A.w, C.x, C.y};
    unsigned m = 0;
    for (int h = B.hm_lo; h < B.hm_hi; h++) {
      if (hm[h].tagidx == B.tag - 1) continue;
      bool meet = true;
      for (int k = 0; k < 3; k++) {
        const double dx = (hm[h].ext[k + 3] - hm[h].ext[k]) / hm[h].nx[k];
        const double sl = 1e-6 * (fabs(hm[h].ext[k]) + fabs(hm[h].ext[k + 3]) + dx);
        const float rlo = __double2float_rd(hm[h].ext[k] - dx - sl);
        const float rhi = __double2float_ru(hm[h].ext[k + 3] + dx + sl);
        meet = meet && !(hi[k] < rlo) && !(lo[k] > rhi);
      }
      if (meet) m |= (h - B.hm_lo < 32) ? (1u << (h - B.hm_lo)) : 0xffffffffu;
    }
    s_maps = m;
  }
  __syncthreads();
  const unsigned maps = s_maps;
  if (!maps) return;
  const int t0 = (int)(T - tile_base[b]) * kNodeTile;
  for (int i = t0 + threadIdx.x; i < min(t0 + kNodeTile, B.nnodes); i += blockDim.x) {
    const int g = node_order[B.node_off + i];
    bool has = false;
    for (int a = 0; a < K && !has; a++) has = slot[(long long)g * K + a] >= 0;
    if (has) continue;  // classified with its owner query
    const double p[3] = {x[3 * (long long)g], x[3 * (long long)g + 1], x[3 * (long long)g + 2]};
    bool hole = false;
    for (int h = B.hm_lo; h < B.hm_hi && !hole; h++) {
      if (h - B.hm_lo < 32 && !((maps >> (h - B.hm_lo)) & 1u)) continue;
      if (hm[h].tagidx == B.tag - 1) continue;
      hole = check_holemap(p, hm[h]) != 0;
    }
    if (hole) mark_hole(g, iblank, m0, m1, mlist, dcnt, counters);
  }
}

// frontier bounds of the nfringe layers: seg[0..1] and seg[2..3] alternate
__global__ void k_front_init(int* __restrict__ dcnt) {
  dcnt[kHoles] = dcnt[kMarked];
  dcnt[kSeg] = 0;
  dcnt[kSeg + 1] = dcnt[kMarked];
}

// one nfringe layer (bookKeeping.C:250-271): every node of a cell that
// touches the previous layer joins the next one.  Only cells around the
// previous layer's new nodes can add nodes.
__global__ void k_dilate_front(int iter, const int* __restrict__ csr_off, const int* __restrict__ csr_cell,
                               const int* __restrict__ conn8, const unsigned char* __restrict__ cell_nv,
                               const blk_t* __restrict__ cell_blk, const BlockInfo* __restrict__ bi,
                               const unsigned char* __restrict__ m0, int* __restrict__ m1, int* __restrict__ mlist,
                               int* __restrict__ dcnt) {
  const int* seg = dcnt + kSeg + 2 * (iter & 1);
  const int s0 = seg[0], s1 = seg[1];
  const int lane = threadIdx.x & 31;  // a warp per frontier node, its lanes over the node's cells
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = s0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < s1; i += nw) {
    const int u = mlist[i];
    for (int k = csr_off[u] + lane; k < csr_off[u + 1]; k += 32) {
      const int c = csr_cell[k];
      if (iter >= bi[cell_blk[c]].nfringe) continue;
      const int nv = cell_nv[c];
      const int* cv = conn8 + 8 * (long long)c;
      for (int m = 0; m < nv; m++) {
        const int v = cv[m];
        if (m0[v] != 1 && atomicExch(&m1[v], 1) == 0) mlist[atomicAdd(&dcnt[kMarked], 1)] = v;
      }
    }
  }
}

// the new layer joins m0, and it is the next frontier
__global__ void k_front_next(int iter, unsigned char* __restrict__ m0, const int* __restrict__ mlist,
                             int* __restrict__ dcnt) {
  const int* seg = dcnt + kSeg + 2 * (iter & 1);
  const int s1 = seg[1], e = dcnt[kMarked];
  for (int i = s1 + blockIdx.x * blockDim.x + threadIdx.x; i < e; i += gridDim.x * blockDim.x) m0[mlist[i]] = 1;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    int* nseg = dcnt + kSeg + 2 * ((iter + 1) & 1);
    nseg[0] = s1;
    nseg[1] = e;
  }
}

// fringe nodes that are not holes become mandatory receptors (nodeRes = BIG)
__global__ void k_fringe_big_list(const int* __restrict__ mlist, const int* __restrict__ dcnt,
                                  const int* __restrict__ iblank, double* __restrict__ node_res) {
  const int nh = dcnt[kHoles], nm = dcnt[kMarked];
  for (int i = nh + blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += gridDim.x * blockDim.x) {
    const int v = mlist[i];
    if (iblank[v]) node_res[v] = kBig;
  }
}

// fringe choice (bookKeeping.C:278-352): the first candidate in list order
// that is finer than the node donates; the record is keyed by (donor block,
// receptor node), which is the order the donor side processes them in.  One
// thread per node with donors (its owner query).
__global__ void k_select(const blk_t* __restrict__ node_blk, const BlockInfo* __restrict__ bi,
                         const int* __restrict__ slot, int K, const int* __restrict__ qnode,
                         const int* __restrict__ qcell, long long nq, const double* __restrict__ cell_res,
                         int* __restrict__ iblank, const double* __restrict__ node_res,
                         unsigned long long* __restrict__ rkey, int* __restrict__ rval, int* __restrict__ rcount,
                         int rcap, unsigned* __restrict__ err) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    if (qcell[q] < 0) continue;
    const int g = qnode[q];
    if (!owner_query(slot, K, g, (int)q)) continue;
    if (iblank[g] == 0) continue;
    Cand L[kMaxK];
    const int n = donor_list(g, slot, K, qcell, cell_res, L);
    const double nres = node_res[g];
    const int b0 = bi[node_blk[g]].sblk0;  // donor indices are system-local
    for (int k = 0; k < n; k++) {
      if (L[k].dres < nres) {
        iblank[g] = -bi[b0 + L[k].a].tag;
        const int r = atomicAdd(rcount, 1);
        if (r >= rcap) {
          atomicOr(err, kErrCapacity);
          break;
        }
        rkey[r] = ((unsigned long long)(b0 + L[k].a) << 32) | (unsigned long long)g;
        rval[r] = L[k].q;
        break;
      }
    }
  }
}

// findInterpData, first part (bookKeeping.C:431-470): records of mandatory
// receptors (receptorRes == BIG) mark the donor cell's non-mandatory hole and
// fringe nodes for cancellation, and the earliest such record resets a fringe
// node's iblank to 1 for every later record of that donor block.
__global__ void k_interp_marks(const unsigned long long* __restrict__ rkey, const int* __restrict__ rval,
                               const int* __restrict__ rcount, const int* __restrict__ qcell,
                               const int* __restrict__ conn8, const unsigned char* __restrict__ cell_nv,
                               const int* __restrict__ iblank, const double* __restrict__ node_res,
                               int* __restrict__ cmark, int* __restrict__ reset_t, int* __restrict__ cmlist,
                               int* __restrict__ dcnt) {
  const int R = *rcount;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    const int g = (int)(rkey[r] & 0xffffffffull);
    const double rres = fabs(node_res[g]);
    if (rres != kBig) continue;
    const int c = qcell[rval[r]];
    if (c < 0) continue;
    const int nv = cell_nv[c];
    const int* cv = conn8 + 8 * (long long)c;
    for (int m = 0; m < nv; m++) {
      const int v = cv[m];
      if (iblank[v] <= 0 && node_res[v] != kBig) {
        if (atomicExch(&cmark[v], 1) == 0) cmlist[atomicAdd(&dcnt[kCancelMarks], 1)] = v;
        if (iblank[v] < 0) atomicMin(&reset_t[v], r);
      }
    }
  }
}

// findInterpData, second part (bookKeeping.C:410-532): acceptance against the
// donor cell's node states as the sequential loop would see them at this
// record, FP64 weights, and the interpolation record.
__global__ void k_interp(const double* __restrict__ x, const unsigned long long* __restrict__ rkey,
                         const int* __restrict__ rval, const int* __restrict__ rcount,
                         const int* __restrict__ qcell, const int* __restrict__ conn8,
                         const unsigned char* __restrict__ cell_nv, const blk_t* __restrict__ node_blk,
                         const BlockInfo* __restrict__ bi, const int* __restrict__ iblank,
                         const double* __restrict__ node_res, const int* __restrict__ reset_t,
                         const int* __restrict__ orig_cell, int* __restrict__ it_node,
                         double* __restrict__ it_w, int* __restrict__ it_rec,
                         int* __restrict__ it_don, unsigned char* __restrict__ it_nv,
                         unsigned char* __restrict__ it_cancel, double* __restrict__ rres_out,
                         int* __restrict__ interp2rec, unsigned* __restrict__ err) {
  const int R = *rcount;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    const unsigned long long key = rkey[r];
    const int g = (int)(key & 0xffffffffull);
    const int a = (int)(key >> 32);
    const int q = rval[r];
    const double rres2 = node_res[g];  // resolutionScale == 1: sent unsigned
    const double rres = fabs(rres2);
    const int mtagrecv = bi[node_blk[g]].tag;
    const int c = qcell[q];
    if (c < 0) {
      atomicOr(err, kErrBadIndex);
      it_cancel[r] = 1;
      it_nv[r] = 0;
      continue;
    }
    const int nv = cell_nv[c];
    const int* cv = conn8 + 8 * (long long)c;
    int accept = 1;
    double xv[8][3];
    for (int m = 0; m < nv; m++) {
      const int v = cv[m];
      const int ibv = (reset_t[v] < r) ? 1 : iblank[v];
      if (ibv <= 0 && rres2 > 0.0) {
        if (node_res[v] == kBig) accept = 0;
        if (abs(ibv) == mtagrecv) accept = 0;
      }
      const double* pv = x + 3 * (long long)v;
      xv[m][0] = pv[0];
      xv[m][1] = pv[1];
      xv[m][2] = pv[2];
    }
    const double xp[3] = {x[3 * (long long)g], x[3 * (long long)g + 1], x[3 * (long long)g + 2]};
    double frac[8];
    nodal_weights64(xv, xp, frac, nv);
    const int noff = bi[a].node_off;
    for (int m = 0; m < nv; m++) {
      it_node[9 * (long long)r + m] = cv[m] - noff;
      it_w[9 * (long long)r + m] = frac[m];
      if (frac[m] < -0.2 || frac[m] > 1.2) atomicOr(err, kErrWeightRange);
    }
    it_node[9 * (long long)r + nv] = orig_cell[c] - bi[a].cell_off;  // the caller's cell id
    it_w[9 * (long long)r + nv] = 0.0;
    it_nv[r] = (unsigned char)nv;
    it_rec[r] = g;
    it_don[r] = a;
    it_cancel[r] = (accept == 0 && rres != kBig) ? 1 : 0;
    rres_out[r] = rres2;
    interp2rec[q] = r;
  }
}

// getCancellationData + cancelDonor (bookKeeping.C:542-570): each marked
// node cancels the interpolation of the head of its own donor list
__global__ void k_cancel(const int* __restrict__ cmlist, const int* __restrict__ dcnt, const int* __restrict__ slot,
                         int K, const int* __restrict__ qcell, const double* __restrict__ cell_res,
                         const int* __restrict__ interp2rec, unsigned char* __restrict__ it_cancel) {
  const int n = dcnt[kCancelMarks];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int v = cmlist[i];
    Cand L[kMaxK];
    const int nl = donor_list(v, slot, K, qcell, cell_res, L);
    if (nl == 0) continue;
    const int r = interp2rec[L[0].q];
    if (r >= 0) it_cancel[r] = 1;
  }
}

// clearIblanks + setIblanks (bookKeeping.C:615-648): the only negative
// iblanks are the records' receptors (-meshtag); they end as -1, or 1 when
// cancelled
__global__ void k_iblank_final(const int* __restrict__ it_rec, const unsigned char* __restrict__ it_cancel,
                               const int* __restrict__ rcount, int* __restrict__ iblank,
                               unsigned long long* __restrict__ counters) {
  const int R = *rcount;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    const bool keep = !it_cancel[r];
    iblank[it_rec[r]] = keep ? -1 : 1;
    if (keep) atomicAdd(&counters[5], 1ull);
  }
}

// End of a call: back to the rest state for the next one (slots of the
// queries with a donor, cancel marks and their reset times).
__global__ void k_donor_clear(const int* __restrict__ qnode, const int* __restrict__ qdon,
                              const int* __restrict__ qcell, long long nq, int K, const BlockInfo* __restrict__ bi,
                              int* __restrict__ slot, const int* __restrict__ cmlist, const int* __restrict__ dcnt,
                              int* __restrict__ cmark, int* __restrict__ reset_t) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq; q += stride)
    if (qcell[q] >= 0) slot[(long long)qnode[q] * K + qdon[q] - bi[qdon[q]].sblk0] = -1;
  const int n = dcnt[kCancelMarks];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
    cmark[cmlist[i]] = 0;
    reset_t[cmlist[i]] = 0x7fffffff;
  }
}

// getCellIblanks (highOrder.C:88-150)
__device__ __forceinline__ int cell_iblank_of(const int* __restrict__ conn8, const unsigned char* __restrict__ cell_nv,
                                              const int* __restrict__ iblank, long long c) {
  const int nv = cell_nv[c];
  const int* cv = conn8 + 8 * c;
  int v = 1, flag = 1, ncount = 0;
  for (int m = 0; m < nv && flag; m++) {
    const int ib = iblank[cv[m]];
    if (ib == 0) {
      v = 0;
      flag = 0;
    }
    ncount += (ib == -1);
  }
  if (flag && ncount == nv) v = -1;
  return v;
}

// Only cells with a node whose iblank is not 1 can differ from 1: the cells
// around the holes and the final receptors (every other cell is 1 already).
__global__ void k_cell_iblank_sparse(const int* __restrict__ mlist, const int* __restrict__ dcnt,
                                     const int* __restrict__ it_rec, const unsigned char* __restrict__ it_cancel,
                                     const int* __restrict__ rcount, const int* __restrict__ csr_off,
                                     const int* __restrict__ csr_cell, const int* __restrict__ conn8,
                                     const unsigned char* __restrict__ cell_nv, const int* __restrict__ iblank,
                                     int* __restrict__ iblank_cell) {
  const int nh = dcnt[kHoles], R = *rcount;
  const int sub = threadIdx.x & 7;  // eight lanes per node (a hexahedral node has eight cells) over its cells
  const int ng = (gridDim.x * blockDim.x) >> 3;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 3; i < nh + R; i += ng) {
    int v;
    if (i < nh) v = mlist[i];
    else if (!it_cancel[i - nh]) v = it_rec[i - nh];
    else continue;
    for (int k = csr_off[v] + sub; k < csr_off[v + 1]; k += 8) {
      const int c = csr_cell[k];
      iblank_cell[c] = cell_iblank_of(conn8, cell_nv, iblank, c);
    }
  }
}

// cells of one block back in the caller's order: out[i] = src[inv[base + i]]
__global__ void k_gather_cells_i32(const int* __restrict__ src, const int* __restrict__ inv, long long base,
                                   int n, int* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = src[inv[base + i]];
}

// ---------------------------------------------------------------------------
// data update: weighted gather in the donor block, then scatter into the
// receptor block (two kernels, so every gather reads the values from before
// the update, as the reference's packet exchange does)
// ---------------------------------------------------------------------------
__global__ void k_interp_gather(const int* __restrict__ it_node, const double* __restrict__ it_w,
                                const int* __restrict__ it_don, const unsigned char* __restrict__ it_nv,
                                const unsigned char* __restrict__ it_cancel, const int* __restrict__ rcount,
                                const BlockInfo* __restrict__ bi, const double* const* __restrict__ qptr, int nvar,
                                int interptype, double* __restrict__ vals) {
  const int R = *rcount;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    if (it_cancel[r]) continue;
    const BlockInfo& D = bi[it_don[r]];
    const double* qb = qptr[it_don[r]];
    const int nv = it_nv[r];
    for (int k0 = 0; k0 < nvar; k0 += 8) {
      const int kn = min(8, nvar - k0);
      double acc[8];
#pragma unroll
      for (int k = 0; k < 8; k++) acc[k] = 0;
      for (int m = 0; m < nv; m++) {
        const int node = it_node[9 * (long long)r + m];
        const double w = it_w[9 * (long long)r + m];
#pragma unroll
        for (int k = 0; k < 8; k++) {
          if (k < kn) {
            const double qv = (interptype == 0) ? qb[(long long)node * nvar + k0 + k]
                                                : qb[(long long)(k0 + k) * D.nnodes + node];
            acc[k] += qv * w;
          }
        }
      }
      for (int k = 0; k < kn; k++) vals[(long long)r * nvar + k0 + k] = acc[k];
    }
  }
}

__global__ void k_interp_scatter(const int* __restrict__ it_rec, const unsigned char* __restrict__ it_cancel,
                                 const int* __restrict__ rcount, const blk_t* __restrict__ node_blk,
                                 const BlockInfo* __restrict__ bi, const double* __restrict__ vals, int nvar,
                                 int interptype, double* const* __restrict__ qptr) {
  const int R = *rcount;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    if (it_cancel[r]) continue;
    const int g = it_rec[r];
    const int rb = node_blk[g];
    const BlockInfo& B = bi[rb];
    const int local = g - B.node_off;
    double* qb = qptr[rb];
    for (int k = 0; k < nvar; k++) {
      if (interptype == 0) qb[(long long)local * nvar + k] = vals[(long long)r * nvar + k];
      else qb[(long long)k * B.nnodes + local] = vals[(long long)r * nvar + k];
    }
  }
}

// ---------------------------------------------------------------------------
// tioga::reduce_fringes (tioga.C:737-885, bookKeeping.C:650-760), on the
// records of the last connectivity call.  Only cells around a receptor node
// can change anything (a cell only restores receptor nodes), so the layers
// are grown over the receptors' cells.
// ---------------------------------------------------------------------------
__global__ void k_rf_init(const int* __restrict__ iblank, long long n, int* __restrict__ red, int* __restrict__ tmp) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int v = iblank[i] > 0 ? iblank[i] : 0;
    red[i] = v;
    tmp[i] = v;
  }
}

// one layer: a cell with some but not all nodes in the reduced set (1 or
// restored -1) restores its receptor nodes; a warp per receptor, its lanes
// over the receptor's cells
__global__ void k_rf_layer(int iter, const int* __restrict__ it_rec, const unsigned char* __restrict__ it_cancel,
                           const int* __restrict__ rcount, const int* __restrict__ csr_off,
                           const int* __restrict__ csr_cell, const int* __restrict__ conn8,
                           const unsigned char* __restrict__ cell_nv, const blk_t* __restrict__ cell_blk,
                           const BlockInfo* __restrict__ bi, const int* __restrict__ iblank,
                           const int* __restrict__ red, int* __restrict__ tmp) {
  const int R = *rcount;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < R; r += nw) {
    if (it_cancel[r]) continue;
    const int g = it_rec[r];
    for (int k = csr_off[g] + lane; k < csr_off[g + 1]; k += 32) {
      const int c = csr_cell[k];
      if (iter >= bi[cell_blk[c]].nfringe + 1) continue;
      const int nv = cell_nv[c];
      const int* cv = conn8 + 8 * (long long)c;
      int ncount = 0;
      for (int m = 0; m < nv; m++) {
        const int v = red[cv[m]];
        ncount += (v == 1 || v < 0);
      }
      if (ncount > 0 && ncount < nv)
        for (int m = 0; m < nv; m++) {
          const int v = cv[m];
          if (tmp[v] == 0 && iblank[v] < 0) tmp[v] = iblank[v];  // every writer writes the same value
        }
    }
  }
}

__global__ void k_rf_copy(const int* __restrict__ it_rec, const unsigned char* __restrict__ it_cancel,
                          const int* __restrict__ rcount, const int* __restrict__ tmp, int* __restrict__ red) {
  const int R = *rcount;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x)
    if (!it_cancel[r]) red[it_rec[r]] = tmp[it_rec[r]];
}

// receptors outside the reduced set cancel the interpolation of the head of
// their donor list, which is their own record (getCancellationData,
// cancelDonor); `was` keeps which records were live before
__global__ void k_rf_cancel(const int* __restrict__ it_rec, const int* __restrict__ rcount, const int* __restrict__ red,
                            unsigned char* __restrict__ it_cancel, unsigned char* __restrict__ was) {
  const int R = *rcount;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    was[r] = !it_cancel[r];
    if (!it_cancel[r] && red[it_rec[r]] == 0) it_cancel[r] = 1;
  }
}

// clearIblanks + setIblanks (bookKeeping.C:615-648): the receptors of the
// live records become -1 if their record survived, else 0 when outside the
// reduced set (1 otherwise); holes stay 0
__global__ void k_rf_iblank(const int* __restrict__ it_rec, const unsigned char* __restrict__ it_cancel,
                            const unsigned char* __restrict__ was, const int* __restrict__ rcount,
                            const int* __restrict__ red, int* __restrict__ iblank,
                            unsigned long long* __restrict__ counters) {
  const int R = *rcount;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    if (!was[r]) continue;
    const int g = it_rec[r];
    if (!it_cancel[r]) {
      iblank[g] = -1;
      atomicAdd(&counters[5], 1ull);
    } else {
      iblank[g] = red[g] == 0 ? 0 : 1;
      if (red[g] == 0) atomicAdd(&counters[4], 1ull);
    }
  }
}

}  // namespace tb
