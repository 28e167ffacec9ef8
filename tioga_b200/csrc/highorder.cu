// The high-order path: tioga_performconnectivity_highorder_ and the point
// data update that follows it (src/tioga.C:162-178 and 336-524 with
// at_points = 1; src/highOrder.C:152-566; src/exchangeSearchData.C:69-80).
//
// The reference asks the solver's callbacks (src/MeshBlock.h:79-83) for each
// receptor cell's points, for the donor inclusion test and for the donor
// weights.  Host callbacks cannot run inside a device search, so this
// library takes the element description itself: Lagrange hexahedra of degree
// p with equispaced nodes, their degrees of freedom stored element-major
// (tioga_b200_set_highorder_lagrange_), and evaluates what such callbacks
// compute on the device (ho_lagrange.cuh):
//   get_nodes_per_cell / get_receptor_nodes  the (p+1)^3 DOFs of the cell
//   donor_inclusion_test                     Newton on the element map, pass
//                                            when r, s, t lie in [-1e-10, 1+1e-10]
//   donor_frac                               the basis at the inverted point
//   convert_to_modal                         nodal values stay as they are
// The flow is the reference's: receptor cells are the cells whose iblank is
// -1 after the last connectivity call; their points inside a pair's box are
// searched in the donor block (coincident points merged as uniqNodesTree
// does, candidates from the registered corners' boxes); points whose donor
// is a field cell get weights; the data update interpolates the donors'
// values, keeps for every point the last donor block that reached it, turns
// receptor cells with an unreached point into field cells (or holes inside a
// foreign hole map) and writes the rest into the receptor cells' DOFs.
#include <algorithm>

#include "engine_impl.cuh"
#include "ho_lagrange.cuh"

namespace tb {

// receptor cells in caller order (iblank_cell == -1), all blocks concatenated
__global__ void k_ho_rcflag(const int* __restrict__ iblank_cell, const int* __restrict__ inv_sorted, long long ctot,
                            int* __restrict__ flag) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ctot;
       c += (long long)gridDim.x * blockDim.x)
    flag[c] = iblank_cell[inv_sorted[c]] == -1;
}

__global__ void k_ho_rclist(const int* __restrict__ flag, const int* __restrict__ off, long long ctot,
                            const BlockInfo* __restrict__ bi, int nb, int* __restrict__ ctag) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ctot;
       c += (long long)gridDim.x * blockDim.x) {
    if (!flag[c]) continue;
    int b = 0;
    while (b + 1 < nb && bi[b + 1].cell_off <= c) b++;
    ctag[off[c]] = (int)(c - bi[b].cell_off);  // block-local caller id
  }
}

// the points of one block's receptor cells, cell after cell, DOF order
__global__ void k_ho_points(const int* __restrict__ ctag, int nrc, int npts, const double* __restrict__ xdof,
                            double* __restrict__ pts) {
  const long long n = (long long)nrc * npts;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long src = (long long)ctag[i / npts] * npts + i % npts;
    for (int k = 0; k < 3; k++) pts[3 * i + k] = xdof[3 * src + k];
  }
}

// getExtraQueryPoints (highOrder.C:285-297): points inside the pair's box
__global__ void k_ho_qflag(const double* __restrict__ pts, long long n, const PairInfo* __restrict__ pair,
                           int* __restrict__ flag) {
  const Obb o = pair->region;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double xd[3];
    for (int j = 0; j < 3; j++) xd[j] = 0;
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++) xd[j] += (pts[3 * i + k] - o.xc[k]) * o.vec[j][k];
    flag[i] = fabs(xd[0]) <= o.dxc[0] && fabs(xd[1]) <= o.dxc[1] && fabs(xd[2]) <= o.dxc[2];
  }
}

__global__ void k_ho_qwrite(const int* __restrict__ flag, const int* __restrict__ off, long long n, long long pt0,
                            long long q0, int don, int rec, int* __restrict__ qpt, int* __restrict__ qloc,
                            int* __restrict__ qdon, int* __restrict__ qrec, double* __restrict__ qres) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (!flag[i]) continue;
    const long long q = q0 + off[i];
    qpt[q] = (int)(pt0 + i);
    qloc[q] = (int)i;
    qdon[q] = don;
    qrec[q] = rec;
    qres[q] = kBig;  // res_search of extra points (highOrder.C:313)
  }
}

// candidate (query, storage cell): the registered corners' box +-TOL (the
// ADT's element boxes, search.C:196-214), then the inclusion test
__global__ void k_ho_candidates(const double* __restrict__ pts, const double* __restrict__ x,
                                const int* __restrict__ conn8, const unsigned char* __restrict__ cell_nv,
                                const int* __restrict__ sorted_cell, const BlockInfo* __restrict__ bi,
                                const HoDev* __restrict__ hd, const double* __restrict__ xdof,
                                const int* __restrict__ qpt, const int* __restrict__ qdon, const int2* __restrict__ cand,
                                long long ncand, int form, int* __restrict__ qbest, int* __restrict__ npass,
                                unsigned long long* __restrict__ counters) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ncand;
       i += (long long)gridDim.x * blockDim.x) {
    const int2 cq = cand[i];
    const int q = cq.x;
    const long long s = cq.y;
    const double* xp = pts + 3ll * qpt[q];
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    const int nv = cell_nv[s];
    for (int m = 0; m < nv; m++) {
      const double* v = x + 3ll * conn8[8 * s + m];
      for (int k = 0; k < 3; k++) {
        lo[k] = dmin(lo[k], v[k]);
        hi[k] = dmax(hi[k], v[k]);
      }
    }
    if (!in_box64(xp, lo, hi)) continue;
    const int a = qdon[q];
    const int lc = sorted_cell[s] - bi[a].cell_off;
    const HoDev h = hd[a];
    const double* X = xdof + 3 * (h.dof_off + (long long)lc * h.npts);
    // split form: an FP32 Newton rejects the clear outsiders; every other
    // candidate takes the FP64 test, accepts included, since its fixed 1e-14
    // stopping rule can fail to converge inside an element (the update cannot
    // always get below 1e-14 in FP64), and that failure rejects the point
    const int screen = form ? ho_screen32(h.p, X, xp) : -1;
    bool pass = false;
    if (screen != 0) {
      double u[3];
      pass = ho_invert_any(h.p, X, xp, u) && ho_inside(u);
      atomicAdd(&counters[9], 1ull);
    }
    atomicAdd(&counters[10], 1ull);
    if (pass) {
      atomicMin(&qbest[q], lc);
      atomicAdd(&npass[q], 1);
    }
  }
}

// a query's donor: the lowest cell id among the cells that pass (the
// reference takes the first in its ADT's pre-order; several passing cells
// are counted as ties)
__global__ void k_ho_finish(const int* __restrict__ qbest, const int* __restrict__ npass, long long nq,
                            int* __restrict__ qcell, unsigned long long* __restrict__ counters) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    const int b = qbest[q];
    qcell[q] = (b == 0x7fffffff) ? -1 : b;
    if (npass[q] >= 2) atomicAdd(&counters[2], 1ull);
    if (b != 0x7fffffff) atomicAdd(&counters[3], 1ull);
  }
}

__global__ void k_ho_copyrep(const int* __restrict__ q_rep, long long nq, int* __restrict__ qcell) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    const int r = q_rep[q];
    if (r != q) qcell[q] = qcell[r];
  }
}

// processPointDonors (highOrder.C:321-419): a point with a donor that is a
// field cell gets a record
__global__ void k_ho_rflag(const int* __restrict__ qcell, const int* __restrict__ qdon, long long nq,
                           const BlockInfo* __restrict__ bi, const int* __restrict__ inv_sorted,
                           const int* __restrict__ iblank_cell, int* __restrict__ flag) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    const int c = qcell[q];
    flag[q] = c >= 0 && iblank_cell[inv_sorted[bi[qdon[q]].cell_off + c]] == 1;
  }
}

// records (receptor block, point in that block, donor block, donor cell) and
// their weights (stride wstride), inverted again from the point
__global__ void k_ho_records(const int* __restrict__ flag, const int* __restrict__ off, long long nq,
                             const int* __restrict__ qcell, const int* __restrict__ qdon,
                             const int* __restrict__ qrec, const int* __restrict__ qloc,
                             const int* __restrict__ qpt, const double* __restrict__ pts,
                             const HoDev* __restrict__ hd, const double* __restrict__ xdof, int wstride,
                             int4* __restrict__ rec, double* __restrict__ w) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nq;
       q += (long long)gridDim.x * blockDim.x) {
    if (!flag[q]) continue;
    const long long r = off[q];
    const int a = qdon[q], c = qcell[q];
    rec[r] = make_int4(qrec[q], qloc[q], a, c);
    const HoDev h = hd[a];
    double u[3];
    ho_invert_any(h.p, xdof + 3 * (h.dof_off + (long long)c * h.npts), pts + 3ll * qpt[q], u);
    ho_weights_any(h.p, u, w + r * wstride);
  }
}

// data update at points: the last donor block to reach a point wins
__global__ void k_ho_winner(const int4* __restrict__ rec, long long nrec, const long long* __restrict__ pt_off,
                            int* __restrict__ win) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nrec;
       r += (long long)gridDim.x * blockDim.x) {
    const int4 R = rec[r];
    atomicMax(&win[pt_off[R.x] + R.y], R.z);
  }
}

// getInterpolatedSolutionAtPoints (highOrder.C:437-458): the winning
// record's values, summed over the weights in order
__global__ void k_ho_values(const int4* __restrict__ rec, long long nrec, const long long* __restrict__ pt_off,
                            const int* __restrict__ win, const HoDev* __restrict__ hd,
                            const long long* __restrict__ qoff, const double* __restrict__ q, int nvar,
                            const double* __restrict__ w, int wstride, double* __restrict__ qtmp) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nrec;
       r += (long long)gridDim.x * blockDim.x) {
    const int4 R = rec[r];
    const long long pt = pt_off[R.x] + R.y;
    if (win[pt] != R.z) continue;
    const HoDev h = hd[R.z];
    const double* qd = q + qoff[R.z] + (long long)R.w * h.npts * nvar;
    for (int k = 0; k < nvar; k++) {
      double acc = 0;
      for (int m = 0; m < h.npts; m++) acc += qd[m * nvar + k] * w[r * wstride + m];
      qtmp[pt * nvar + k] = acc;
    }
  }
}

// clearOrphans (highOrder.C:152-186): the last unreached point of a
// receptor cell decides: a hole if it lies in a foreign wall mesh's hole
// map, else a field cell
__global__ void k_ho_orphans(const int* __restrict__ ctag, const int* __restrict__ rc_blk, long long nrc,
                             const long long* __restrict__ rc_off, const long long* __restrict__ pt_off,
                             const HoDev* __restrict__ hd, const int* __restrict__ win,
                             const double* __restrict__ pts, const BlockInfo* __restrict__ bi,
                             const int* __restrict__ inv_sorted, const HoleMapDev* __restrict__ hm, int nhm,
                             int* __restrict__ iblank_cell, unsigned long long* __restrict__ counters) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nrc;
       i += (long long)gridDim.x * blockDim.x) {
    const int b = rc_blk[i];
    const int npts = hd[b].npts;
    const long long p0 = pt_off[b] + (i - rc_off[b]) * npts;
    int reject = 0;
    for (int j = 0; j < npts; j++) {
      if (win[p0 + j] >= 0) continue;
      reject = 2;
      for (int k = bi[b].hm_lo; k < bi[b].hm_hi; k++)
        if (hm[k].tagidx != bi[b].tag - 1 && check_holemap(pts + 3 * (p0 + j), hm[k])) {
          reject = 1;
          break;
        }
    }
    if (reject) {
      iblank_cell[inv_sorted[bi[b].cell_off + ctag[i]]] = (reject == 1) ? 0 : 1;
      atomicAdd(&counters[8], 1ull);
    }
  }
}

// updatePointData (highOrder.C:487-505) into a device solution
__global__ void k_ho_scatter(const int* __restrict__ ctag, const int* __restrict__ rc_blk, long long nrc,
                             const long long* __restrict__ rc_off, const long long* __restrict__ pt_off,
                             const HoDev* __restrict__ hd, const BlockInfo* __restrict__ bi,
                             const int* __restrict__ inv_sorted, const int* __restrict__ iblank_cell,
                             const long long* __restrict__ qoff, const double* __restrict__ qtmp, int nvar,
                             double* __restrict__ q) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nrc;
       i += (long long)gridDim.x * blockDim.x) {
    const int b = rc_blk[i];
    if (iblank_cell[inv_sorted[bi[b].cell_off + ctag[i]]] != -1) continue;
    const int npts = hd[b].npts;
    const long long p0 = pt_off[b] + (i - rc_off[b]) * npts;
    double* qd = q + qoff[b] + (long long)ctag[i] * npts * nvar;
    for (long long k = 0; k < (long long)npts * nvar; k++) qd[k] = qtmp[p0 * nvar + k];
  }
}

// ---------------------------------------------------------------------------
int Engine::set_highorder(int tag, int p, const double* xdof) {
  int ib = find_tag(tag);
  if (ib < 0 || p < 1 || p + 1 > kHoMaxN || !xdof) {
    fprintf(stderr, "#tioga_b200: set_highorder_lagrange: unknown tag %d, degree %d outside 1..%d or no DOFs\n",
            tag, p, kHoMaxN - 1);
    return -1;
  }
  if ((int)ho_.size() < (int)hb_.size()) ho_.resize(hb_.size());
  ho_[ib].p = p;
  ho_[ib].npts = (p + 1) * (p + 1) * (p + 1);
  ho_[ib].hxdof = xdof;
  ho_dof_on_device_ = false;
  ihigh_ = true;
  return 0;
}

int Engine::connectivity_highorder() {
  if (!connected_) {
    fprintf(stderr, "#tioga_b200: performconnectivity_highorder needs performconnectivity first\n");
    return -1;
  }
  if (nsystems() > 1) {
    fprintf(stderr, "#tioga_b200: the high-order path takes one overset system per instance\n");
    return -1;
  }
  const int nb = (int)hb_.size();
  if ((int)ho_.size() < nb) ho_.resize(nb);
  for (int b = 0; b < nb; b++)
    if (!ho_[b].hxdof) {
      fprintf(stderr, "#tioga_b200: performconnectivity_highorder: block %d has no element description "
                      "(tioga_b200_set_highorder_lagrange_); solver callbacks cannot run in the device search\n",
              hb_[b].tag);
      return -1;
    }
  ho_done_ = false;
  // element DOF coordinates, re-read like the corner coordinates
  std::vector<HoDev> hd(nb);
  long long ndof = 0;
  for (int b = 0; b < nb; b++) {
    hd[b] = HoDev{ho_[b].p, ho_[b].npts, ndof};
    ndof += (long long)hb_[b].ncells * ho_[b].npts;
  }
  TB_CUDA(ho_dev_.ensure(nb));
  TB_CUDA(cudaMemcpyAsync(ho_dev_.p, hd.data(), nb * sizeof(HoDev), cudaMemcpyHostToDevice, stream_));
  // (kept on the device when the caller declares its coordinates unmoved)
  if (!(coords_resident_ && ho_dof_on_device_ && ho_xdof_.n >= 3 * (size_t)std::max(1ll, ndof))) {
    TB_CUDA(ho_xdof_.ensure(3 * std::max(1ll, ndof)));
    for (int b = 0; b < nb; b++)
      TB_CUDA(cudaMemcpyAsync(ho_xdof_.p + 3 * hd[b].dof_off, ho_[b].hxdof,
                              3 * (size_t)hb_[b].ncells * ho_[b].npts * sizeof(double), cudaMemcpyHostToDevice,
                              stream_));
    ho_dof_on_device_ = true;
  }
  // receptor cells (getInternalNodes, highOrder.C:208-247)
  DBuf<int> flag, off;
  TB_CUDA(flag.ensure(ctot_ + 1));
  TB_CUDA(off.ensure(ctot_ + 1));
  k_ho_rcflag<<<grid_for(ctot_, kT), kT, 0, stream_>>>(iblank_cell_.p, inv_sorted_.p, ctot_, flag.p);
  TB_LAUNCHED("k_ho_rcflag");
  TB_CUDA(cudaMemsetAsync(flag.p + ctot_, 0, sizeof(int), stream_));
  size_t tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp, flag.p, off.p, (int)(ctot_ + 1), stream_);
  TB_CUDA(cub_tmp_.ensure(tmp));
  cub::DeviceScan::ExclusiveSum(cub_tmp_.p, tmp, flag.p, off.p, (int)(ctot_ + 1), stream_);
  std::vector<int> boff(nb + 1);
  for (int b = 0; b <= nb; b++) {
    const long long c = (b < nb) ? bi_[b].cell_off : ctot_;
    TB_CUDA(cudaMemcpyAsync(&boff[b], off.p + c, sizeof(int), cudaMemcpyDeviceToHost, stream_));
  }
  TB_CUDA(cudaStreamSynchronize(stream_));
  const long long nrc = boff[nb];
  TB_CUDA(ho_ctag_.ensure(std::max(1ll, nrc)));
  k_ho_rclist<<<grid_for(ctot_, kT), kT, 0, stream_>>>(flag.p, off.p, ctot_, d_bi_.p, nb, ho_ctag_.p);
  TB_LAUNCHED("k_ho_rclist");
  ho_rc_off_.assign(nb + 1, 0);
  ho_pt_off_.assign(nb + 1, 0);
  std::vector<int> rc_blk(std::max(1ll, nrc));
  for (int b = 0; b < nb; b++) {
    ho_rc_off_[b + 1] = boff[b + 1];
    ho_pt_off_[b + 1] = ho_pt_off_[b] + (long long)(boff[b + 1] - boff[b]) * ho_[b].npts;
    for (int i = boff[b]; i < boff[b + 1]; i++) rc_blk[i] = b;
  }
  ho_nrc_ = nrc;
  const long long ntp = ho_pt_off_[nb];
  TB_CUDA(ho_rcblk_.ensure(std::max(1ll, nrc)));
  TB_CUDA(cudaMemcpyAsync(ho_rcblk_.p, rc_blk.data(), std::max(1ll, nrc) * sizeof(int), cudaMemcpyHostToDevice,
                          stream_));
  TB_CUDA(ho_rcoff_d_.ensure(nb + 1));
  TB_CUDA(ho_ptoff_d_.ensure(nb + 1));
  TB_CUDA(cudaMemcpyAsync(ho_rcoff_d_.p, ho_rc_off_.data(), (nb + 1) * sizeof(long long), cudaMemcpyHostToDevice,
                          stream_));
  TB_CUDA(cudaMemcpyAsync(ho_ptoff_d_.p, ho_pt_off_.data(), (nb + 1) * sizeof(long long), cudaMemcpyHostToDevice,
                          stream_));
  TB_CUDA(ho_pts_.ensure(3 * std::max(1ll, ntp)));
  for (int b = 0; b < nb; b++) {
    const int n = boff[b + 1] - boff[b];
    if (n == 0) continue;
    k_ho_points<<<grid_for((long long)n * ho_[b].npts, kT), kT, 0, stream_>>>(
        ho_ctag_.p + boff[b], n, ho_[b].npts, ho_xdof_.p + 3 * hd[b].dof_off, ho_pts_.p + 3 * ho_pt_off_[b]);
    TB_LAUNCHED("k_ho_points");
  }
  // query points per pair, pair-major, point order (exchangeSearchData(1))
  std::vector<int> qoff(npairs_ + 1, 0);
  long long nq = 0;
  TB_CUDA(flag.ensure(std::max(1ll, ntp) + 1));
  TB_CUDA(off.ensure(std::max(1ll, ntp) + 1));
  for (int p = 0; p < npairs_; p++) {
    qoff[p] = (int)nq;
    const int r = h_pairs_[p].rec;
    const long long n = ho_pt_off_[r + 1] - ho_pt_off_[r];
    if (n == 0) continue;
    k_ho_qflag<<<grid_for(n, kT), kT, 0, stream_>>>(ho_pts_.p + 3 * ho_pt_off_[r], n, d_pairs_.p + p, flag.p);
    TB_LAUNCHED("k_ho_qflag");
    TB_CUDA(cudaMemsetAsync(flag.p + n, 0, sizeof(int), stream_));
    tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, flag.p, off.p, (int)(n + 1), stream_);
    TB_CUDA(cub_tmp_.ensure(tmp));
    cub::DeviceScan::ExclusiveSum(cub_tmp_.p, tmp, flag.p, off.p, (int)(n + 1), stream_);
    int cnt = 0;
    TB_CUDA(cudaMemcpyAsync(&cnt, off.p + n, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaStreamSynchronize(stream_));
    if (cnt == 0) continue;
    const long long need = nq + cnt;
    if (need > ho_qcap_) {  // grow, keeping the queries written so far
      const long long cap = std::max(need, 2 * ho_qcap_);
      DBuf<int> a, b2, c, d;
      DBuf<double> e;
      TB_CUDA(a.ensure(cap));
      TB_CUDA(b2.ensure(cap));
      TB_CUDA(c.ensure(cap));
      TB_CUDA(d.ensure(cap));
      TB_CUDA(e.ensure(cap));
      if (nq > 0) {
        TB_CUDA(cudaMemcpyAsync(a.p, ho_qpt_.p, nq * sizeof(int), cudaMemcpyDeviceToDevice, stream_));
        TB_CUDA(cudaMemcpyAsync(b2.p, ho_qloc_.p, nq * sizeof(int), cudaMemcpyDeviceToDevice, stream_));
        TB_CUDA(cudaMemcpyAsync(c.p, ho_qdon_.p, nq * sizeof(int), cudaMemcpyDeviceToDevice, stream_));
        TB_CUDA(cudaMemcpyAsync(d.p, ho_qrec_.p, nq * sizeof(int), cudaMemcpyDeviceToDevice, stream_));
        TB_CUDA(cudaMemcpyAsync(e.p, ho_qres_.p, nq * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
      }
      TB_CUDA(cudaStreamSynchronize(stream_));
      std::swap(ho_qpt_, a);
      std::swap(ho_qloc_, b2);
      std::swap(ho_qdon_, c);
      std::swap(ho_qrec_, d);
      std::swap(ho_qres_, e);
      ho_qcap_ = cap;
    }
    k_ho_qwrite<<<grid_for(n, kT), kT, 0, stream_>>>(flag.p, off.p, n, ho_pt_off_[r], nq, h_pairs_[p].don, r,
                                                     ho_qpt_.p, ho_qloc_.p, ho_qdon_.p, ho_qrec_.p, ho_qres_.p);
    TB_LAUNCHED("k_ho_qwrite");
    nq += cnt;
  }
  qoff[npairs_] = (int)nq;
  ho_nq_ = nq;
  ho_nrecs_ = 0;
  if (nq == 0) {
    ho_done_ = true;
    return 0;
  }
  // coincident points (uniqNodesTree over each donor's list)
  TB_CUDA(cudaMemsetAsync(counters_.p, 0, 16 * sizeof(unsigned long long), stream_));
  DedupQueries Q{nq, ho_qpt_.p, ho_qdon_.p, ho_qloc_.p, ho_qrec_.p, ho_qres_.p, ho_pts_.p, nullptr};
  TB_TRY(dedup_merge(Q, qoff));
  // candidates from the corner boxes, then the inclusion test
  unsigned count = 0;
  TB_TRY(traverse_and_gather(ho_pts_.p, ho_qpt_.p, ho_qdon_.p, nq, count));
  TB_CUDA(ho_qbest_.ensure(nq));
  TB_CUDA(ho_npass_.ensure(nq));
  TB_CUDA(ho_qcell_.ensure(nq));
  k_fill_int<<<grid_for(nq, kT), kT, 0, stream_>>>(ho_qbest_.p, 0x7fffffff, nq);
  TB_LAUNCHED("k_fill_int");
  TB_CUDA(cudaMemsetAsync(ho_npass_.p, 0, nq * sizeof(int), stream_));
  if (count > 0) {
    k_ho_candidates<<<grid_for(count, 128), 128, 0, stream_>>>(
        ho_pts_.p, x_.p, conn8_.p, cell_nv_.p, sorted_cell_.p, d_bi_.p, ho_dev_.p, ho_xdof_.p, ho_qpt_.p,
        ho_qdon_.p, cand_.p, count, precision_ == 2 ? 1 : 0, ho_qbest_.p, ho_npass_.p, counters_.p);
    TB_LAUNCHED("k_ho_candidates");
  }
  k_ho_finish<<<grid_for(nq, kT), kT, 0, stream_>>>(ho_qbest_.p, ho_npass_.p, nq, ho_qcell_.p, counters_.p);
  TB_LAUNCHED("k_ho_finish");
  k_ho_copyrep<<<grid_for(nq, kT), kT, 0, stream_>>>(q_rep_.p, nq, ho_qcell_.p);
  TB_LAUNCHED("k_ho_copyrep");
  // point donors that are field cells, with their weights
  TB_CUDA(flag.ensure(nq + 1));
  TB_CUDA(off.ensure(nq + 1));
  k_ho_rflag<<<grid_for(nq, kT), kT, 0, stream_>>>(ho_qcell_.p, ho_qdon_.p, nq, d_bi_.p, inv_sorted_.p,
                                                   iblank_cell_.p, flag.p);
  TB_LAUNCHED("k_ho_rflag");
  TB_CUDA(cudaMemsetAsync(flag.p + nq, 0, sizeof(int), stream_));
  tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp, flag.p, off.p, (int)(nq + 1), stream_);
  TB_CUDA(cub_tmp_.ensure(tmp));
  cub::DeviceScan::ExclusiveSum(cub_tmp_.p, tmp, flag.p, off.p, (int)(nq + 1), stream_);
  int nr = 0;
  TB_CUDA(cudaMemcpyAsync(&nr, off.p + nq, sizeof(int), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  ho_wstride_ = 1;
  for (int b = 0; b < nb; b++) ho_wstride_ = std::max(ho_wstride_, ho_[b].npts);
  TB_CUDA(ho_rec_.ensure(std::max(1, nr)));
  TB_CUDA(ho_w_.ensure((size_t)std::max(1, nr) * ho_wstride_));
  if (nr > 0) {
    k_ho_records<<<grid_for(nq, 128), 128, 0, stream_>>>(flag.p, off.p, nq, ho_qcell_.p, ho_qdon_.p, ho_qrec_.p,
                                                         ho_qloc_.p, ho_qpt_.p, ho_pts_.p, ho_dev_.p, ho_xdof_.p,
                                                         ho_wstride_, ho_rec_.p, ho_w_.p);
    TB_LAUNCHED("k_ho_records");
  }
  ho_nrecs_ = nr;
  unsigned long long cnt[16];
  TB_CUDA(cudaMemcpyAsync(cnt, counters_.p, sizeof(cnt), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  ho_stats_ = {nq, (long long)cnt[3], (long long)cnt[2], (long long)nr, (long long)cnt[7], 0, (long long)cnt[10],
               (long long)cnt[9]};
  ho_done_ = true;
  return 0;
}

// tioga_dataupdate_mb_ after the high-order connectivity: ROW solutions,
// every block's DOF array element-major with nvar values per DOF
int Engine::dataupdate_highorder(int nvar, int interptype) {
  if (!ho_done_) {
    fprintf(stderr, "#tioga_b200: high-order data update needs performconnectivity_highorder first\n");
    return -1;
  }
  const int nb = (int)hb_.size();
  bool device = true, host = true;
  for (auto& H : hb_) {
    if (!H.hq && !H.dq) {
      printf("Solution data not set, cannot update \n");
      return 0;
    }
    device = device && H.dq;
    host = host && H.hq;
  }
  if (npairs_ == 0) return 0;
  if (interptype != 0) {  // the reference fills no values for COLUMN here (highOrder.C:474-476)
    fprintf(stderr, "#tioga_b200: the high-order data update handles ROW layouts only\n");
    return -1;
  }
  if (!device && !host) {
    fprintf(stderr, "#tioga_b200: register every block's solution on the same side (host or device)\n");
    return -1;
  }
  std::vector<long long> qo(nb + 1, 0);
  for (int b = 0; b < nb; b++) qo[b + 1] = qo[b] + (long long)hb_[b].ncells * ho_[b].npts * nvar;
  TB_CUDA(ho_q_.ensure(std::max(1ll, qo[nb])));
  for (int b = 0; b < nb; b++)
    TB_CUDA(cudaMemcpyAsync(ho_q_.p + qo[b], host ? hb_[b].hq : hb_[b].dq, (qo[b + 1] - qo[b]) * sizeof(double),
                            host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, stream_));
  TB_CUDA(ho_qoff_d_.ensure(nb + 1));
  TB_CUDA(cudaMemcpyAsync(ho_qoff_d_.p, qo.data(), (nb + 1) * sizeof(long long), cudaMemcpyHostToDevice, stream_));
  const long long ntp = ho_pt_off_[nb];
  TB_CUDA(ho_win_.ensure(std::max(1ll, ntp)));
  TB_CUDA(ho_qtmp_.ensure(std::max(1ll, ntp) * nvar));
  k_fill_int<<<grid_for(std::max(1ll, ntp), kT), kT, 0, stream_>>>(ho_win_.p, -1, std::max(1ll, ntp));
  TB_LAUNCHED("k_fill_int");
  TB_CUDA(cudaMemsetAsync(ho_qtmp_.p, 0, std::max(1ll, ntp) * nvar * sizeof(double), stream_));
  TB_CUDA(cudaMemsetAsync(counters_.p + 8, 0, sizeof(unsigned long long), stream_));
  if (ho_nrecs_ > 0) {
    k_ho_winner<<<grid_for(ho_nrecs_, kT), kT, 0, stream_>>>(ho_rec_.p, ho_nrecs_, ho_ptoff_d_.p, ho_win_.p);
    TB_LAUNCHED("k_ho_winner");
    k_ho_values<<<grid_for(ho_nrecs_, 128), 128, 0, stream_>>>(ho_rec_.p, ho_nrecs_, ho_ptoff_d_.p, ho_win_.p,
                                                               ho_dev_.p, ho_qoff_d_.p, ho_q_.p, nvar, ho_w_.p,
                                                               ho_wstride_, ho_qtmp_.p);
    TB_LAUNCHED("k_ho_values");
  }
  if (ho_nrc_ > 0) {
    k_ho_orphans<<<grid_for(ho_nrc_, 128), 128, 0, stream_>>>(ho_ctag_.p, ho_rcblk_.p, ho_nrc_, ho_rcoff_d_.p,
                                                              ho_ptoff_d_.p, ho_dev_.p, ho_win_.p, ho_pts_.p,
                                                              d_bi_.p, inv_sorted_.p, d_hmdev_.p, nhm_,
                                                              iblank_cell_.p, counters_.p);
    TB_LAUNCHED("k_ho_orphans");
    k_ho_scatter<<<grid_for(ho_nrc_, 128), 128, 0, stream_>>>(ho_ctag_.p, ho_rcblk_.p, ho_nrc_, ho_rcoff_d_.p,
                                                              ho_ptoff_d_.p, ho_dev_.p, d_bi_.p, inv_sorted_.p,
                                                              iblank_cell_.p, ho_qoff_d_.p, ho_qtmp_.p, nvar,
                                                              ho_q_.p);
    TB_LAUNCHED("k_ho_scatter");
  }
  // the updated DOF arrays back to the caller, and the cell iblanks the
  // orphan rule changed
  for (int b = 0; b < nb; b++)
    TB_CUDA(cudaMemcpyAsync(host ? hb_[b].hq : hb_[b].dq, ho_q_.p + qo[b], (qo[b + 1] - qo[b]) * sizeof(double),
                            host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, stream_));
  unsigned long long orphans = 0;
  TB_CUDA(cudaMemcpyAsync(&orphans, counters_.p + 8, sizeof(orphans), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  ho_stats_.norphan_cells = (long long)orphans;
  for (int b = 0; b < nb; b++)
    if (hb_[b].h_iblank_cell) TB_TRY(cell_iblank(hb_[b].tag, hb_[b].h_iblank_cell));
  return 0;
}

// records of donor block `tag`, in its list order: (receptor block index,
// point in that block, donor cell (block-local caller id), weights count)
// and the weights (stride 1331)
int Engine::point_donors(int tag, int* out, double* w) {
  int ib = find_tag(tag);
  if (ib < 0 || !ho_done_ || ho_nrecs_ == 0) return 0;
  std::vector<int4> rec(ho_nrecs_);
  std::vector<double> ww((size_t)ho_nrecs_ * ho_wstride_);
  TB_CUDA(cudaMemcpyAsync(rec.data(), ho_rec_.p, rec.size() * sizeof(int4), cudaMemcpyDeviceToHost, stream_));
  if (w)
    TB_CUDA(cudaMemcpyAsync(ww.data(), ho_w_.p, ww.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  int n = 0;
  for (long long r = 0; r < ho_nrecs_; r++) {
    if (rec[r].z != ib) continue;
    if (out) {
      out[4 * n] = rec[r].x;
      out[4 * n + 1] = rec[r].y;
      out[4 * n + 2] = rec[r].w;
      out[4 * n + 3] = ho_[ib].npts;
    }
    if (w) std::copy(ww.begin() + r * ho_wstride_, ww.begin() + r * ho_wstride_ + ho_[ib].npts, w + (size_t)1331 * n);
    n++;
  }
  return n;
}

}  // namespace tb
