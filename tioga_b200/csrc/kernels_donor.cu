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
                             long long ctot, int* __restrict__ slot, unsigned* __restrict__ err) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    const int c = qcell[q];
    if (c < 0) continue;
    const int g = qnode[q], a = qdon[q];
    if (c >= ctot || g < 0 || g >= ntot || a < 0 || a >= K) {
      atomicOr(err, kErrBadIndex);
      continue;
    }
    slot[(long long)g * K + a] = (int)q;
  }
}

// processDonors first pass (bookKeeping.C:158-237): holes from the hole maps
// of wall-bearing meshes that supplied no donor, node resolution raised to
// the candidates' receptor resolutions.
__global__ void k_process_donors(const double* __restrict__ x, const unsigned char* __restrict__ node_blk,
                                 const BlockInfo* __restrict__ bi, const int* __restrict__ slot, int K,
                                 const double* __restrict__ qres, const HoleMapDev* __restrict__ hm, int nhm,
                                 long long ntot, int* __restrict__ iblank, double* __restrict__ node_res,
                                 unsigned char* __restrict__ m0, unsigned char* __restrict__ m1) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
       g += (long long)gridDim.x * blockDim.x) {
    const int b = node_blk[g];
    const int tag = bi[b].tag;
    unsigned long long seen[2] = {0ull, 0ull};
    int ncand = 0;
    double nres = node_res[g];
    for (int a = 0; a < K; a++) {
      int q = slot[g * K + a];
      if (q < 0) continue;
      ncand++;
      int t = bi[a].tag - 1;
      seen[t >> 6] |= 1ull << (t & 63);
      nres = dmax(nres, qres[q]);
    }
    int ib = 1;
    const double p[3] = {x[3 * g], x[3 * g + 1], x[3 * g + 2]};
    for (int h = 0; h < nhm; h++) {
      const HoleMapDev& H = hm[h];
      int ht = H.tagidx;
      if (ht == tag - 1) continue;
      if (ncand > 0 && ((seen[ht >> 6] >> (ht & 63)) & 1ull)) continue;
      if (check_holemap(p, H)) {
        ib = 0;
        break;
      }
    }
    iblank[g] = ib;
    if (ncand > 0) node_res[g] = nres;
    m0[g] = m1[g] = (ib == 0);
  }
}

// one nfringe layer (bookKeeping.C:250-271): every node of a cell that
// touches the current layer joins the next one
__global__ void k_dilate(const int* __restrict__ conn8, const unsigned char* __restrict__ cell_nv,
                         const unsigned char* __restrict__ cell_blk, const BlockInfo* __restrict__ bi,
                         long long ctot, int iter, const unsigned char* __restrict__ m0,
                         unsigned char* __restrict__ m1) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ctot;
       c += (long long)gridDim.x * blockDim.x) {
    if (iter >= bi[cell_blk[c]].nfringe) continue;
    const int nv = cell_nv[c];
    const int* cv = conn8 + 8 * c;
    int hit = 0;
    for (int m = 0; m < nv; m++) hit |= (m0[cv[m]] == 1);
    if (!hit) continue;
    for (int m = 0; m < nv; m++)
      if (m0[cv[m]] != 1) m1[cv[m]] = 1;
  }
}

__global__ void k_fringe_big(const unsigned char* __restrict__ m1, const int* __restrict__ iblank,
                             long long ntot, double* __restrict__ node_res) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
       g += (long long)gridDim.x * blockDim.x)
    if (m1[g] && iblank[g]) node_res[g] = kBig;
}

// fringe choice (bookKeeping.C:278-352): the first candidate in list order
// that is finer than the node donates; the record is keyed by (donor block,
// receptor node), which is the order the donor side processes them in.
__global__ void k_select(const unsigned char* __restrict__ node_blk, const BlockInfo* __restrict__ bi,
                         const int* __restrict__ slot, int K, const int* __restrict__ qcell,
                         const double* __restrict__ cell_res, long long ntot, int* __restrict__ iblank,
                         const double* __restrict__ node_res, unsigned long long* __restrict__ rkey,
                         int* __restrict__ rval, int* __restrict__ rcount, int rcap,
                         unsigned* __restrict__ err) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
       g += (long long)gridDim.x * blockDim.x) {
    if (iblank[g] == 0) continue;
    Cand L[kMaxK];
    int n = donor_list(g, slot, K, qcell, cell_res, L);
    if (n == 0) continue;
    const double nres = node_res[g];
    for (int k = 0; k < n; k++) {
      if (L[k].dres < nres) {
        iblank[g] = -bi[L[k].a].tag;
        int r = atomicAdd(rcount, 1);
        if (r >= rcap) {
          atomicOr(err, kErrCapacity);
          break;
        }
        rkey[r] = ((unsigned long long)L[k].a << 32) | (unsigned long long)g;
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
                               unsigned char* __restrict__ cmark, int* __restrict__ reset_t) {
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
        cmark[v] = 1;
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
                         const unsigned char* __restrict__ cell_nv, const unsigned char* __restrict__ node_blk,
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
__global__ void k_cancel(const unsigned char* __restrict__ cmark, long long ntot, const int* __restrict__ slot,
                         int K, const int* __restrict__ qcell, const double* __restrict__ cell_res,
                         const int* __restrict__ interp2rec, unsigned char* __restrict__ it_cancel) {
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < ntot;
       v += (long long)gridDim.x * blockDim.x) {
    if (!cmark[v]) continue;
    Cand L[kMaxK];
    int n = donor_list(v, slot, K, qcell, cell_res, L);
    if (n == 0) continue;
    int r = interp2rec[L[0].q];
    if (r >= 0) it_cancel[r] = 1;
  }
}

// clearIblanks + setIblanks (bookKeeping.C:615-648)
__global__ void k_iblank_clear(int* __restrict__ iblank, long long ntot) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
       g += (long long)gridDim.x * blockDim.x)
    if (iblank[g] < 0) iblank[g] = 1;
}

__global__ void k_iblank_set(const int* __restrict__ it_rec, const unsigned char* __restrict__ it_cancel,
                             const int* __restrict__ rcount, int* __restrict__ iblank) {
  const int R = *rcount;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x)
    if (!it_cancel[r]) iblank[it_rec[r]] = -1;
}

// getCellIblanks (highOrder.C:88-150)
__global__ void k_cell_iblank(const int* __restrict__ conn8, const unsigned char* __restrict__ cell_nv,
                              long long ctot, const int* __restrict__ iblank, const int* __restrict__ orig_cell,
                              int* __restrict__ iblank_cell) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ctot;
       c += (long long)gridDim.x * blockDim.x) {
    const int nv = cell_nv[c];
    const int* cv = conn8 + 8 * c;
    int v = 1, flag = 1, ncount = 0;
    for (int m = 0; m < nv && flag; m++) {
      int ib = iblank[cv[m]];
      if (ib == 0) {
        v = 0;
        flag = 0;
      }
      ncount += (ib == -1);
    }
    if (flag && ncount == nv) v = -1;
    iblank_cell[c] = v;
  }
}

// cells of one block back in the caller's order: out[i] = src[inv[base + i]]
__global__ void k_gather_cells_i32(const int* __restrict__ src, const int* __restrict__ inv, long long base,
                                   int n, int* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = src[inv[base + i]];
}

__global__ void k_count_iblank(const int* __restrict__ iblank, long long ntot,
                               unsigned long long* __restrict__ counters) {
  unsigned long long h = 0, r = 0;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ntot;
       g += (long long)gridDim.x * blockDim.x) {
    h += (iblank[g] == 0);
    r += (iblank[g] < 0);
  }
  for (int o = 16; o > 0; o >>= 1) {
    h += __shfl_xor_sync(0xffffffffu, h, o);
    r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&counters[4], h);
    atomicAdd(&counters[5], r);
  }
}

// ---------------------------------------------------------------------------
// data update: weighted gather in the donor block, then scatter into the
// receptor block (two kernels, so every gather reads the values from before
// the update, as the reference's packet exchange does)
// ---------------------------------------------------------------------------
__global__ void k_interp_gather(const int* __restrict__ it_node, const double* __restrict__ it_w,
                                const int* __restrict__ it_don, const unsigned char* __restrict__ it_nv,
                                const unsigned char* __restrict__ it_cancel, const int* __restrict__ rcount,
                                const BlockInfo* __restrict__ bi, const double* __restrict__ q, int nvar,
                                int interptype, double* __restrict__ vals) {
  const int R = *rcount;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    if (it_cancel[r]) continue;
    const BlockInfo& D = bi[it_don[r]];
    const double* qb = q + (long long)D.node_off * nvar;
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
                                 const int* __restrict__ rcount, const unsigned char* __restrict__ node_blk,
                                 const BlockInfo* __restrict__ bi, const double* __restrict__ vals, int nvar,
                                 int interptype, double* __restrict__ q) {
  const int R = *rcount;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
    if (it_cancel[r]) continue;
    const int g = it_rec[r];
    const BlockInfo& B = bi[node_blk[g]];
    const int local = g - B.node_off;
    double* qb = q + (long long)B.node_off * nvar;
    for (int k = 0; k < nvar; k++) {
      if (interptype == 0) qb[(long long)local * nvar + k] = vals[(long long)r * nvar + k];
      else qb[(long long)k * B.nnodes + local] = vals[(long long)r * nvar + k];
    }
  }
}

}  // namespace tb
