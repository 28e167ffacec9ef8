// Host orchestration of the B200 connectivity path: preprocess, connectivity,
// data update and the donor queries, all on one CUDA stream.
#include <algorithm>
#include <cstring>

#include "engine_impl.cuh"

namespace tb {

static int g_last_cuda_error = 0;
thread_local long long* g_dbuf_account = nullptr;
thread_local cudaStream_t g_dbuf_stream = nullptr;
thread_local cudaMemPool_t g_dbuf_pool = nullptr;
int fail(cudaError_t e) {
  g_last_cuda_error = (int)e;
  return -(int)e - 1000;
}

int sync_check() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("TIOGA_B200_CHECK");
    v = (e && e[0] == '1') ? 1 : 0;
  }
  return v;
}

Engine::Engine() {
  cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking);
  stream_ = own_stream_;
  for (auto& e : ev_) cudaEventCreate(&e);
  for (auto& e : sev_) cudaEventCreate(&e);
  for (auto& e : cev_) cudaEventCreate(&e);
  cudaEventCreateWithFlags(&pev_, cudaEventDisableTiming);
  cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking);
  for (auto& e : hev_) cudaEventCreate(&e);
  for (auto& e : cib_ev_) cudaEventCreate(&e);
  cudaEventCreateWithFlags(&dr_ev_, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&rf_ev_, cudaEventDisableTiming);
  cudaStreamCreateWithFlags(&up_, cudaStreamNonBlocking);
  cudaEventCreateWithFlags(&up_start_, cudaEventDisableTiming);
}

Engine::~Engine() {
  unpin_caller_arrays();
  if (stream_) cudaStreamSynchronize(stream_);
  if (pre_exec_) cudaGraphExecDestroy(pre_exec_);
  for (auto& e : ev_) cudaEventDestroy(e);
  for (auto& e : sev_) cudaEventDestroy(e);
  for (auto& e : cev_) cudaEventDestroy(e);
  cudaEventDestroy(pev_);
  if (side_) cudaStreamSynchronize(side_);
  for (auto& e : hev_) cudaEventDestroy(e);
  for (auto& e : cib_ev_) cudaEventDestroy(e);
  cudaEventDestroy(dr_ev_);
  cudaEventDestroy(rf_ev_);
  if (up_) cudaStreamSynchronize(up_);
  for (auto& e : up_ev_) cudaEventDestroy(e);
  cudaEventDestroy(up_start_);
  if (up_) cudaStreamDestroy(up_);
  if (side_) cudaStreamDestroy(side_);
  if (h_hm_init_) cudaFreeHost(h_hm_init_);
  if (h_hm_info_) cudaFreeHost(h_hm_info_);
  if (h_hm_dev_) cudaFreeHost(h_hm_dev_);
  x_.release(); node_res_.release(); cell_res_.release(); iblank_.release(); iblank_cell_.release();
  conn8_.release(); node_blk_.release(); cell_blk_.release(); cell_nv_.release(); wallf_.release();
  obcf_.release(); ex0_.release(); ex1_.release(); m0_.release(); m1_.release(); cmark_.release();
  wall_list_.release(); obc_list_.release(); csr_off_.release(); csr_cell_.release(); deg_.release();
  d_bi_.release(); d_pairs_.release(); d_npairs_.release(); d_hm_.release(); d_hmdev_.release();
  hm_state_.release();
  wall_bb_.release(); sorted_cell_.release(); cbox_.release(); xf_.release(); tnode_.release(); tnode64_.release();
  leaves_.release(); lbox_.release(); pair_ext_.release(); gparent_.release(); gnk_.release(); up_leaf_ids_.release();
  up_tile_ids_.release();
  gnint_.release(); refit_start_.release(); refit_cnt_.release();
  mlist_.release(); cmlist_.release(); dcnt_.release(); node_bin_.release();
  cbox64_.release(); qnode_.release(); qdon_.release(); qcell_.release(); qres_.release();
  qtie_.release(); qcount_.release(); tile_cnt_.release(); tile_off_.release(); tile_mask_.release(); slot_.release();
  rkey_.release(); rkey_alt_.release(); rval_.release(); rval_alt_.release(); rcount_.release();
  reset_t_.release(); interp2rec_.release(); it_node_.release(); it_w_.release(); it_rec_.release();
  it_don_.release(); it_nv_.release(); it_cancel_.release(); rres_.release(); q_.release();
  qvals_.release(); d_qptr_.release(); cub_tmp_.release(); red_.release(); err_.release(); coord_err_.release();
  counters_.release();
  mkey_.release(); mkey_alt_.release(); mval_alt_.release();
  d_pcand_.release(); d_pfirst_.release(); d_chunks_.release(); d_chunk_cta_.release(); d_pair_t0_.release();
  rf_red_.release(); rf_tmp_.release(); rf_was_.release(); uhex_map_.release(); uhex_red_.release();
  node_gid_d_.release(); gm_k0_.release(); gm_k1_.release(); gm_max_.release(); gm_a_.release(); gm_b_.release();
  gm_c_.release(); gm_d_.release();
  d_wall_.release(); wall_cells_.release(); wall_box_.release(); wall_box_first_.release();
  cg_cnt_.release(); cg_off_.release(); cg_v0_.release(); cg_v1_.release(); cg_k0_.release(); cg_k1_.release();
  cg_flag_.release();
  if (own_stream_) cudaStreamDestroy(own_stream_);
}

// Work on the caller's stream (nullptr: back to the library's own stream).
void Engine::set_stream(cudaStream_t s) {
  cudaStreamSynchronize(stream_);
  stream_ = s ? s : own_stream_;
}

int Engine::find_tag(int tag) const { return find_block(cur_sys_, tag); }

int Engine::nsystems() const {
  int n = 0;
  for (size_t b = 0; b < hb_.size(); b++) n += (b == 0 || hb_[b].sys != hb_[b - 1].sys);
  return n;
}

int Engine::find_block(int sys, int tag) const {
  auto it = tag2idx_.find(((long long)sys << 32) | (unsigned)tag);
  return it == tag2idx_.end() ? -1 : it->second;
}

// src/tioga.C:64-86 + MeshBlock.C:37-72: one block per mesh tag; a second
// registration of a tag replaces that block's data.  Pointers stay the
// caller's.  Blocks of several independent overset systems may share one
// engine (system ids >= 0, each with its own tags); the blocks are kept
// grouped by system, in registration order within a system.
int Engine::register_block(int tag, int nnodes, double* x, int* ibl, int nwbc, int nobc, int* wbc,
                           int* obc, int ntypes, const int* nv, const int* nc, int** conn) {
  return register_block_sys(0, tag, nnodes, x, ibl, nwbc, nobc, wbc, obc, ntypes, nv, nc, conn);
}

int Engine::register_block_sys(int sys, int tag, int nnodes, double* x, int* ibl, int nwbc, int nobc, int* wbc,
                               int* obc, int ntypes, const int* nv, const int* nc, int** conn) {
  if (ntypes < 1 || ntypes > 4) {
    fprintf(stderr, "#tioga_b200: %d cell types given, 1..4 supported\n", ntypes);
    return -1;
  }
  for (int t = 0; t < ntypes; t++)
    if (nv[t] != 4 && nv[t] != 5 && nv[t] != 6 && nv[t] != 8) {
      fprintf(stderr, "#tioga_b200: cells with %d vertices are not supported\n", nv[t]);
      return -1;
    }
  if (tag < 1 || tag > 128) {
    fprintf(stderr, "#tioga_b200: mesh tags must lie in 1..128 (got %d)\n", tag);
    return -1;
  }
  if (sys < 0) {
    fprintf(stderr, "#tioga_b200: system ids must be >= 0 (got %d)\n", sys);
    return -1;
  }
  int ib = find_block(sys, tag);
  if (ib < 0) {
    int in_sys = 0;
    for (const HostBlock& H : hb_) in_sys += (H.sys == sys);
    if (in_sys >= kMaxSysBlocks) {
      fprintf(stderr, "#tioga_b200: at most %d blocks per system\n", kMaxSysBlocks);
      return -1;
    }
    if ((int)hb_.size() >= kMaxEngineBlocks) {
      fprintf(stderr, "#tioga_b200: at most %d blocks per instance\n", kMaxEngineBlocks);
      return -1;
    }
    // after the last block of a system with an id <= sys
    int pos = (int)hb_.size();
    while (pos > 0 && hb_[pos - 1].sys > sys) pos--;
    hb_.insert(hb_.begin() + pos, HostBlock{});
    if (pos < (int)ho_.size()) ho_.insert(ho_.begin() + pos, HoBlockDesc{});
    tag2idx_.clear();
    for (int b = 0; b < (int)hb_.size(); b++)
      if (b != pos) tag2idx_[((long long)hb_[b].sys << 32) | (unsigned)hb_[b].tag] = b;
    tag2idx_[((long long)sys << 32) | (unsigned)tag] = pos;
    ib = pos;
  }
  HostBlock& b = hb_[ib];
  b.sys = sys;
  b.tag = tag;
  b.nnodes = nnodes;
  b.hx = x;
  b.hibl = ibl;
  b.nwbc = nwbc;
  b.nobc = nobc;
  b.hwbc = wbc;
  b.hobc = obc;
  b.ntypes = ntypes;
  b.ncells = 0;
  for (int t = 0; t < 4; t++) {
    b.nv[t] = t < ntypes ? nv[t] : 0;
    b.nc[t] = t < ntypes ? nc[t] : 0;
    b.hconn[t] = t < ntypes ? conn[t] : nullptr;
    b.ncells += b.nc[t];
  }
  b.cell_gid = nullptr;  // registerGridData without cell ids (src/MeshBlock.C:60)
  topo_dirty_ = true;
  coords_on_device_ = false;
  gate_valid_ = false;
  ho_dof_on_device_ = false;
  preprocessed_ = false;
  connected_ = false;
  return 0;
}

int Engine::set_resolutions(int tag, double* nres, double* cres) {
  int ib = find_tag(tag);
  if (ib < 0) return -1;
  hb_[ib].user_nres = nres;
  hb_[ib].user_cres = cres;
  return 0;
}

int Engine::set_cell_iblank(int tag, int* ibc) {
  int ib = find_tag(tag);
  if (ib < 0) return -1;
  hb_[ib].h_iblank_cell = ibc;
  return 0;
}

int Engine::register_iblank_device(int tag, int* d_ibl) {
  int ib = find_tag(tag);
  if (ib < 0) return -1;
  hb_[ib].dibl = d_ibl;
  return 0;
}

int Engine::register_solution(int tag, double* q, bool device) {
  int ib = find_tag(tag);
  if (ib < 0 || !connected_) {
    fprintf(stderr, "#tioga_b200: registersolution needs a known tag after performconnectivity\n");
    return -1;
  }
  if (device) {
    hb_[ib].dq = q;
    hb_[ib].hq = nullptr;
  } else {
    hb_[ib].hq = q;
    hb_[ib].dq = nullptr;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// topology upload (once per registration)
// ---------------------------------------------------------------------------
int Engine::upload_topology() {
  const int nb = (int)hb_.size();
  bi_.assign(nb, BlockInfo{});
  ntot_ = 0;
  ctot_ = 0;
  long long nwall = 0, nobcn = 0;
  maxtag_ = 0;
  for (int b = 0; b < nb; b++) {
    BlockInfo& B = bi_[b];
    const HostBlock& H = hb_[b];
    B.tag = H.tag;
    B.nnodes = H.nnodes;
    B.ncells = H.ncells;
    B.node_off = (int)ntot_;
    B.cell_off = (int)ctot_;
    B.ntypes = H.ntypes;
    B.type_off[0] = 0;
    for (int t = 0; t < 4; t++) {
      B.nv[t] = H.nv[t];
      B.type_off[t + 1] = B.type_off[t] + H.nc[t];
    }
    B.nwbc = H.nwbc;
    B.wall_off = (int)nwall;
    B.nobc = H.nobc;
    B.obc_off = (int)nobcn;
    ntot_ += H.nnodes;
    ctot_ += H.ncells;
    nwall += H.nwbc;
    nobcn += H.nobc;
    maxtag_ = std::max(maxtag_, H.tag);
  }
  // systems: consecutive block ranges; one hole map per wall-bearing block,
  // numbered in block order so that a system's maps are consecutive too
  nhm_all_ = 0;
  K_ = 1;
  for (int b = 0; b < nb;) {
    int e = b;
    while (e < nb && hb_[e].sys == hb_[b].sys) e++;
    const int lo = nhm_all_;
    for (int k = b; k < e; k++) bi_[k].hm = hb_[k].nwbc > 0 ? nhm_all_++ : -1;
    for (int k = b; k < e; k++) {
      bi_[k].sys = hb_[k].sys;
      bi_[k].sblk0 = b;
      bi_[k].snb = e - b;
      bi_[k].hm_lo = lo;
      bi_[k].hm_hi = nhm_all_;
    }
    K_ = std::max(K_, e - b);
    b = e;
  }
  if (ntot_ >= (1ll << 31) || ctot_ >= (1ll << 31)) {
    fprintf(stderr, "#tioga_b200: more than 2^31 nodes or cells\n");
    return -1;
  }
  TB_CUDA(x_.ensure(3 * ntot_));
  TB_CUDA(node_res_.ensure(ntot_));
  TB_CUDA(iblank_.ensure(ntot_));
  TB_CUDA(node_blk_.ensure(ntot_));
  TB_CUDA(wallf_.ensure(ntot_));
  TB_CUDA(obcf_.ensure(ntot_));
  TB_CUDA(ex0_.ensure(ntot_));
  TB_CUDA(ex1_.ensure(ntot_));
  TB_CUDA(m0_.ensure(ntot_));
  TB_CUDA(m1_.ensure(ntot_));
  TB_CUDA(cmark_.ensure(ntot_));
  TB_CUDA(reset_t_.ensure(ntot_));
  TB_CUDA(cell_res_.ensure(ctot_));
  TB_CUDA(iblank_cell_.ensure(ctot_));
  TB_CUDA(conn8_.ensure(8 * ctot_));
  TB_CUDA(cell_blk_.ensure(ctot_));
  TB_CUDA(cell_nv_.ensure(ctot_));
  TB_CUDA(wall_list_.ensure(nwall));
  TB_CUDA(obc_list_.ensure(nobcn));
  TB_CUDA(slot_.ensure(ntot_ * K_));
  TB_CUDA(d_bi_.ensure(nb));
  TB_CUDA(err_.ensure(4));
  TB_CUDA(counters_.ensure(16));
  TB_CUDA(cudaMemsetAsync(wallf_.p, 0, ntot_, stream_));
  TB_CUDA(cudaMemsetAsync(obcf_.p, 0, ntot_, stream_));
  TB_CUDA(cudaMemsetAsync(err_.p, 0, 4 * sizeof(unsigned), stream_));
  // staging buffer for the 1-based caller arrays
  size_t stage = 0;
  for (auto& H : hb_) {
    for (int t = 0; t < H.ntypes; t++) stage = std::max(stage, (size_t)H.nc[t] * H.nv[t]);
    stage = std::max(stage, (size_t)H.nwbc);
    stage = std::max(stage, (size_t)H.nobc);
  }
  DBuf<int> stg;
  TB_CUDA(stg.ensure(stage));
  for (int b = 0; b < nb; b++) {
    const HostBlock& H = hb_[b];
    const BlockInfo& B = bi_[b];
    k_node_blk<<<grid_for(H.nnodes, kT), kT, 0, stream_>>>(B.node_off, H.nnodes, b, node_blk_.p);
    TB_LAUNCHED("k_node_blk");
    for (int t = 0; t < H.ntypes; t++) {
      size_t n = (size_t)H.nc[t] * H.nv[t];
      if (n == 0) continue;
      TB_CUDA(cudaMemcpyAsync(stg.p, H.hconn[t], n * sizeof(int), cudaMemcpyHostToDevice, stream_));
      k_conn_convert<<<grid_for(H.nc[t], kT), kT, 0, stream_>>>(stg.p, H.nc[t], H.nv[t], B.node_off, H.nnodes,
                                                                B.cell_off + B.type_off[t], b, conn8_.p,
                                                                cell_nv_.p, cell_blk_.p, err_.p);
      TB_LAUNCHED("k_conn_convert");
      TB_CUDA(cudaStreamSynchronize(stream_));  // the staging buffer is reused
    }
    if (H.nwbc > 0) {
      TB_CUDA(cudaMemcpyAsync(stg.p, H.hwbc, H.nwbc * sizeof(int), cudaMemcpyHostToDevice, stream_));
      k_mark_list<<<grid_for(H.nwbc, kT), kT, 0, stream_>>>(stg.p, H.nwbc, B.node_off, H.nnodes, wall_list_.p,
                                                            B.wall_off, wallf_.p, err_.p);
      TB_LAUNCHED("k_mark_list");
      TB_CUDA(cudaStreamSynchronize(stream_));
    }
    if (H.nobc > 0) {
      TB_CUDA(cudaMemcpyAsync(stg.p, H.hobc, H.nobc * sizeof(int), cudaMemcpyHostToDevice, stream_));
      k_mark_list<<<grid_for(H.nobc, kT), kT, 0, stream_>>>(stg.p, H.nobc, B.node_off, H.nnodes, obc_list_.p,
                                                            B.obc_off, obcf_.p, err_.p);
      TB_LAUNCHED("k_mark_list");
      TB_CUDA(cudaStreamSynchronize(stream_));
    }
  }
  stg.release();
  if (pin_host_) pin_caller_arrays();
  {
    unsigned e = 0;
    TB_CUDA(cudaMemcpyAsync(&e, err_.p, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaStreamSynchronize(stream_));
    if (e & kErrBadInput) {
      fprintf(stderr, "#tioga_b200: a connectivity, wall or overset-boundary node index lies outside 1..nnodes\n");
      TB_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(unsigned), stream_));
      return -1;
    }
  }
  TB_TRY(build_csr());
  // block pairs that may intersect: different mesh tags of one system, donor
  // outer, receptor inner (exchangeBoxes.C:133-160)
  std::vector<int2> cand;
  for (int ob = 0; ob < nb; ob++)
    for (int ib = bi_[ob].sblk0; ib < bi_[ob].sblk0 + bi_[ob].snb; ib++)
      if (hb_[ib].tag != hb_[ob].tag) cand.push_back(make_int2(ob, ib));
  npcand_ = (int)cand.size();
  TB_CUDA(d_pcand_.ensure(std::max(npcand_, 1)));
  if (npcand_ > 0)
    TB_CUDA(cudaMemcpyAsync(d_pcand_.p, cand.data(), cand.size() * sizeof(int2), cudaMemcpyHostToDevice, stream_));
  // wall-bearing blocks
  h_wall_.clear();
  for (int b = 0; b < nb; b++)
    if (bi_[b].hm >= 0)
      h_wall_.push_back(WallBlock{bi_[b].wall_off, bi_[b].nwbc, bi_[b].cell_off, bi_[b].ncells, bi_[b].hm});
  TB_CUDA(d_wall_.ensure(std::max<size_t>(h_wall_.size(), 1)));
  if (!h_wall_.empty())
    TB_CUDA(cudaMemcpyAsync(d_wall_.p, h_wall_.data(), h_wall_.size() * sizeof(WallBlock), cudaMemcpyHostToDevice,
                            stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));  // host tables above go out of scope
  // hole map state: one fixed-size slab per wall-bearing block
  if (nhm_all_ > 0) {  // no stale wall marks (2) in a fresh map: the plane fill treats the rest as unmarked
    TB_CUDA(hm_state_.ensure((size_t)nhm_all_ * kHoleMapCap));
    TB_CUDA(cudaMemsetAsync(hm_state_.p, 0, (size_t)nhm_all_ * kHoleMapCap, stream_));
  }
  TB_CUDA(d_hm_.ensure(std::max(nhm_all_, 1)));
  TB_CUDA(wall_bb_.ensure(6 * std::max(nhm_all_, 1)));
  TB_CUDA(d_hmdev_.ensure(std::max(nhm_all_, 1)));
  topo_dirty_ = false;
  interps_fetched_ = false;
  topo_gen_++;
  return 0;
}

int Engine::build_csr() {
  TB_CUDA(deg_.ensure(ntot_ + 1));
  TB_CUDA(csr_off_.ensure(ntot_ + 1));
  TB_CUDA(cudaMemsetAsync(deg_.p, 0, (ntot_ + 1) * sizeof(int), stream_));
  k_csr_count<<<grid_for(ctot_, kT), kT, 0, stream_>>>(conn8_.p, cell_nv_.p, ctot_, deg_.p);
  TB_LAUNCHED("k_csr_count");
  size_t tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp, deg_.p, csr_off_.p, (int)(ntot_ + 1), stream_);
  TB_CUDA(cub_tmp_.ensure(tmp));
  cub::DeviceScan::ExclusiveSum(cub_tmp_.p, tmp, deg_.p, csr_off_.p, (int)(ntot_ + 1), stream_);
  int total = 0;
  TB_CUDA(cudaMemcpyAsync(&total, csr_off_.p + ntot_, sizeof(int), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  inc_tot_ = total;
  TB_CUDA(csr_cell_.ensure(total));
  TB_CUDA(cudaMemsetAsync(deg_.p, 0, (ntot_ + 1) * sizeof(int), stream_));
  k_csr_fill<<<grid_for(ctot_, kT), kT, 0, stream_>>>(conn8_.p, cell_nv_.p, ctot_, csr_off_.p, deg_.p,
                                                      csr_cell_.p);
  TB_LAUNCHED("k_csr_fill");
  k_csr_sort<<<grid_for(ntot_, kT), kT, 0, stream_>>>(csr_off_.p, ntot_, csr_cell_.p);
  TB_LAUNCHED("k_csr_sort");
  return 0;
}

// The caller's coordinate and iblank arrays stay valid while they are
// registered (MeshBlock.C:37-72), and every connectivity call copies them to
// and from the device, so pageable ones are page-locked once per topology:
// their copies then run at the full PCIe rate instead of through staging
// buffers.  Arrays that are pinned already, or that cannot be registered,
// are left as they are.  The registrations end with the topology (a new
// registration, tioga_delete_).
void Engine::pin_caller_arrays() {
  unpin_caller_arrays();
  auto pin = [&](void* p, size_t bytes) {
    if (!p || bytes == 0) return;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    if (a.type != cudaMemoryTypeUnregistered) return;
    if (cudaHostRegister(p, bytes, cudaHostRegisterDefault) == cudaSuccess) pinned_.push_back(p);
    else cudaGetLastError();
  };
  for (const HostBlock& H : hb_) {
    pin(H.hx, 3 * (size_t)H.nnodes * sizeof(double));
    pin(H.hibl, (size_t)H.nnodes * sizeof(int));
  }
}

void Engine::unpin_caller_arrays() {
  for (void* p : pinned_) cudaHostUnregister(p);
  pinned_.clear();
  cudaGetLastError();
}

int Engine::upload_coords() {
  for (size_t b = 0; b < hb_.size(); b++)
    TB_CUDA(cudaMemcpyAsync(x_.p + 3 * (long long)bi_[b].node_off, hb_[b].hx,
                            3 * (size_t)hb_[b].nnodes * sizeof(double), cudaMemcpyHostToDevice, stream_));
  coords_on_device_ = true;
  gate_valid_ = false;  // the caller may have moved the nodes any way
  return check_coords();
}

// The leaves of each upload chunk: a leaf belongs to the chunk that holds its
// largest vertex id, so its cell boxes can be made once that chunk has landed
// (chunks land in order).  Leaf ids sorted by chunk, offsets on the host.
int Engine::build_upload_chunks() {
  const long long nl = nleaf_total_;
  const int nch = (int)((ntot_ + up_chunk_ - 1) / up_chunk_);
  h_up_leaf_off_.assign(nch + 1, 0);
  if (nl == 0 || nch == 0) return 0;
  DBuf<int> key, id, key2;
  TB_CUDA(key.ensure(nl));
  TB_CUDA(id.ensure(nl));
  TB_CUDA(key2.ensure(nl));
  TB_CUDA(up_leaf_ids_.ensure(nl));
  k_leaf_chunk<<<grid_for(nl, kT), kT, 0, stream_>>>(leaves_.p, nl, conn8_.p, cell_nv_.p, up_chunk_, key.p, id.p);
  TB_LAUNCHED("k_leaf_chunk");
  int hi_bit = 1;
  while ((1 << hi_bit) < nch) hi_bit++;
  size_t tmp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp, key.p, key2.p, id.p, up_leaf_ids_.p, (int)nl, 0, hi_bit, stream_);
  TB_CUDA(cub_tmp_.ensure(tmp));
  cub::DeviceRadixSort::SortPairs(cub_tmp_.p, tmp, key.p, key2.p, id.p, up_leaf_ids_.p, (int)nl, 0, hi_bit,
                                  stream_);
  std::vector<int> hk(nl);
  TB_CUDA(cudaMemcpyAsync(hk.data(), key2.p, nl * sizeof(int), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  for (long long l = 0; l < nl; l++) h_up_leaf_off_[hk[l] + 1]++;
  for (int k = 0; k < nch; k++) h_up_leaf_off_[k + 1] += h_up_leaf_off_[k];
  return 0;
}

// The node tiles of each upload chunk, as for the leaves: a tile's box can be
// made once the chunk holding its largest node id has landed.
int Engine::build_tile_chunks() {
  const long long nt = h_tile_base_.empty() ? 0 : h_tile_base_.back();
  const int nch = (int)((ntot_ + up_chunk_ - 1) / up_chunk_);
  h_up_tile_off_.assign(nch + 1, 0);
  if (nt == 0 || nch == 0) return 0;
  DBuf<int> key, id, key2;
  TB_CUDA(key.ensure(nt));
  TB_CUDA(id.ensure(nt));
  TB_CUDA(key2.ensure(nt));
  TB_CUDA(up_tile_ids_.ensure(nt));
  k_tile_chunk<<<grid_for(nt, kT), kT, 0, stream_>>>(d_bi_.p, (int)bi_.size(), tile_base_.p, node_order_.p,
                                                     up_chunk_, key.p, id.p);
  TB_LAUNCHED("k_tile_chunk");
  int hi_bit = 1;
  while ((1 << hi_bit) < nch) hi_bit++;
  size_t tmp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp, key.p, key2.p, id.p, up_tile_ids_.p, (int)nt, 0, hi_bit, stream_);
  TB_CUDA(cub_tmp_.ensure(tmp));
  cub::DeviceRadixSort::SortPairs(cub_tmp_.p, tmp, key.p, key2.p, id.p, up_tile_ids_.p, (int)nt, 0, hi_bit,
                                  stream_);
  std::vector<int> hk(nt);
  TB_CUDA(cudaMemcpyAsync(hk.data(), key2.p, nt * sizeof(int), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  for (long long i = 0; i < nt; i++) h_up_tile_off_[hk[i] + 1]++;
  for (int k = 0; k < nch; k++) h_up_tile_off_[k + 1] += h_up_tile_off_[k];
  return 0;
}

// Coordinates up in chunks on up_; as chunk k lands the main stream checks
// it is finite, makes its FP32 copy and the cell boxes of chunk k's leaves
// (k_cell_boxes over an id list), while the next chunks are in flight.  The
// host reads the finite check once the last chunk is done, before any
// kernel derives an index from a coordinate.
int Engine::upload_chunked() {
  const int nch = (int)h_up_leaf_off_.size() - 1;
  while ((int)up_ev_.size() < nch) {
    cudaEvent_t e;
    TB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    up_ev_.push_back(e);
  }
  TB_CUDA(xf_.ensure(ntot_));
  TB_CUDA(lbox_.ensure(2 * nleaf_total_));
  TB_CUDA(coord_err_.ensure(1));
  TB_CUDA(cudaMemsetAsync(coord_err_.p, 0, sizeof(unsigned), stream_));
  TB_CUDA(cudaEventRecord(up_start_, stream_));
  TB_CUDA(cudaStreamWaitEvent(up_, up_start_, 0));
  for (int k = 0; k < nch; k++) {
    const long long g0 = (long long)k * up_chunk_, g1 = std::min<long long>(ntot_, g0 + up_chunk_);
    for (size_t b = 0; b < hb_.size(); b++) {
      const long long o = bi_[b].node_off, e = o + hb_[b].nnodes;
      const long long a = std::max(g0, o), z = std::min(g1, e);
      if (a < z)
        TB_CUDA(cudaMemcpyAsync(x_.p + 3 * a, hb_[b].hx + 3 * (a - o), 3 * (size_t)(z - a) * sizeof(double),
                                cudaMemcpyHostToDevice, up_));
    }
    TB_CUDA(cudaEventRecord(up_ev_[k], up_));
  }
  const int mb = tune_.cell_box_per_sm;
  for (int k = 0; k < nch; k++) {
    const long long g0 = (long long)k * up_chunk_, g1 = std::min<long long>(ntot_, g0 + up_chunk_);
    TB_CUDA(cudaStreamWaitEvent(stream_, up_ev_[k], 0));
    k_check_finite<<<grid_for(3 * (g1 - g0), kT), kT, 0, stream_>>>(x_.p + 3 * g0, 3 * (g1 - g0), coord_err_.p);
    TB_LAUNCHED("k_check_finite");
    k_round_nodes<<<grid_for(g1 - g0, kT), kT, 0, stream_>>>(x_.p, g0, g1, xf_.p);
    TB_LAUNCHED("k_round_nodes");
    if (h_up_tile_off_.size() == h_up_leaf_off_.size()) {  // the tiles whose last node is in this chunk
      const long long t0 = h_up_tile_off_[k], ntl = h_up_tile_off_[k + 1] - t0;
      if (ntl > 0) {
        k_node_tiles<<<(unsigned)ntl, 256, 0, stream_>>>(x_.p, d_bi_.p, (int)bi_.size(), tile_base_.p, tbox_.p,
                                                         node_order_.p, nullptr, up_tile_ids_.p + t0);
        TB_LAUNCHED("k_node_tiles");
      }
    }
    const long long l0 = h_up_leaf_off_[k], nl = h_up_leaf_off_[k + 1] - l0;
    if (nl > 0) {
      launch_cell_boxes(mb, (int)grid_for(nl * kMaxLeafCells, 256, 148 * mb), stream_, xf_.p, conn8_.p, cell_nv_.p,
                        leaves_.p, up_leaf_ids_.p + l0, nl, cbox_.p, tnode_.p, lbox_.p);
      TB_LAUNCHED("k_cell_boxes");
    }
  }
  unsigned e = 0;
  TB_CUDA(cudaMemcpyAsync(&e, coord_err_.p, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  if (e) {
    fprintf(stderr, "#tioga_b200: a node coordinate is not finite (NaN or infinite)\n");
    coords_on_device_ = false;
    return -1;
  }
  coords_on_device_ = true;
  gate_valid_ = false;  // the caller may have moved the nodes any way
  boxes_ready_ = true;
  tiles_ready_ = h_up_tile_off_.size() == h_up_leaf_off_.size();
  return 0;
}

// Refuse non-finite coordinates before any kernel derives an index (hole-map
// cells, Morton keys) from them.
int Engine::check_coords() {
  TB_CUDA(coord_err_.ensure(1));
  TB_CUDA(cudaMemsetAsync(coord_err_.p, 0, sizeof(unsigned), stream_));
  if (ntot_ > 0) {
    k_check_finite<<<grid_for(3 * ntot_, kT), kT, 0, stream_>>>(x_.p, 3 * ntot_, coord_err_.p);
    TB_LAUNCHED("k_check_finite");
  }
  unsigned e = 0;
  TB_CUDA(cudaMemcpyAsync(&e, coord_err_.p, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  if (e) {
    fprintf(stderr, "#tioga_b200: a node coordinate is not finite (NaN or infinite)\n");
    coords_on_device_ = false;
    return -1;
  }
  return 0;
}

// device coordinates -> the caller's arrays (after rigid motions on the device)
int Engine::download_coords() {
  if (!coords_on_device_) return 0;
  for (size_t b = 0; b < hb_.size(); b++)
    TB_CUDA(cudaMemcpyAsync(hb_[b].hx, x_.p + 3 * (long long)bi_[b].node_off,
                            3 * (size_t)hb_[b].nnodes * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  return 0;
}

int Engine::apply_rigid(int block, const double* A, const double* b) {
  if (block < 0 || block >= (int)hb_.size() || topo_dirty_ || !coords_on_device_) {
    fprintf(stderr, "#tioga_b200: rigid motion needs a preprocessed block with device coordinates\n");
    return -1;
  }
  Rigid m;
  for (int k = 0; k < 9; k++) m.a[k] = A[k];
  for (int k = 0; k < 3; k++) m.b[k] = b[k];
  const int n = hb_[block].nnodes;
  if (n > 0) {
    k_rigid<<<grid_for(n, kT), kT, 0, stream_>>>(x_.p + 3 * (long long)bi_[block].node_off, n, m);
    TB_LAUNCHED("k_rigid");
  }
  return 0;
}

int Engine::compute_obbs() {
  // every block at once: 148 CTAs per block, three passes (sums, covariance,
  // projections), each finished by one thread per block
  const int nparts = 148;
  const int nb = (int)hb_.size();
  if (nb == 0) return 0;
  TB_CUDA(red_.ensure(12 * (size_t)nparts * nb));
  for (int pass = 0; pass < 3; pass++) {
    k_obb_partial<<<dim3(nparts, nb), 256, 0, stream_>>>(x_.p, d_bi_.p, pass, red_.p);
    TB_LAUNCHED("k_obb_partial");
    k_obb_finish<<<(nb + 127) / 128, 128, 0, stream_>>>(red_.p, nparts, pass, x_.p, d_bi_.p, nb);
    TB_LAUNCHED("k_obb_finish");
  }
  return 0;
}

int Engine::build_tree_topology() {
  // Morton order of the cell centroids per block (block id in the key's
  // high word), leaves of consecutive cells, one implicit 4-ary tree per
  // block.  Rebuilt only when the registration changes; every connectivity
  // call refits the boxes to the current coordinates.
  TB_CUDA(mkey_.ensure(ctot_));
  TB_CUDA(mkey_alt_.ensure(ctot_));
  TB_CUDA(sorted_cell_.ensure(ctot_));
  TB_CUDA(mval_alt_.ensure(ctot_));
  k_morton<<<grid_for(ctot_, kT), kT, 0, stream_>>>(x_.p, conn8_.p, cell_nv_.p, cell_blk_.p, d_bi_.p,
                                                    ctot_, mkey_.p, mval_alt_.p);
  TB_LAUNCHED("k_morton");
  size_t tmp = 0;
  int key_bits = 32;  // 30-bit Morton code, block id from bit 32
  while ((1ll << (key_bits - 32)) < (long long)bi_.size()) key_bits++;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp, mkey_.p, mkey_alt_.p, mval_alt_.p, sorted_cell_.p,
                                  (int)ctot_, 0, key_bits, stream_);
  TB_CUDA(cub_tmp_.ensure(tmp));
  cub::DeviceRadixSort::SortPairs(cub_tmp_.p, tmp, mkey_.p, mkey_alt_.p, mval_alt_.p, sorted_cell_.p,
                                  (int)ctot_, 0, key_bits, stream_);
  // From here on every cell array is in storage (Morton) order; sorted_cell_
  // maps a storage position to the caller's cell id and inv_sorted_ back.
  TB_CUDA(inv_sorted_.ensure(ctot_));
  k_invert<<<grid_for(ctot_, kT), kT, 0, stream_>>>(sorted_cell_.p, ctot_, inv_sorted_.p);
  TB_LAUNCHED("k_invert");
  {
    DBuf<int> conn2;
    DBuf<unsigned char> nv2;
    DBuf<blk_t> blk2;
    TB_CUDA(conn2.ensure(8 * ctot_));
    TB_CUDA(nv2.ensure(ctot_));
    TB_CUDA(blk2.ensure(ctot_));
    k_permute_cells<<<grid_for(ctot_, kT), kT, 0, stream_>>>(sorted_cell_.p, ctot_, conn8_.p, cell_nv_.p,
                                                              cell_blk_.p, conn2.p, nv2.p, blk2.p);
    TB_LAUNCHED("k_permute_cells");
    std::swap(conn8_, conn2);
    std::swap(cell_nv_, nv2);
    std::swap(cell_blk_, blk2);
    k_remap<<<grid_for(inc_tot_, kT), kT, 0, stream_>>>(csr_cell_.p, inc_tot_, inv_sorted_.p);
    TB_LAUNCHED("k_remap");
    TB_CUDA(cudaStreamSynchronize(stream_));
    conn2.release();
    nv2.release();
    blk2.release();
  }
  // Morton order of each block's nodes: the order query points are gathered in
  TB_CUDA(node_order_.ensure(ntot_));
  {
    DBuf<unsigned long long> k0, k1;
    DBuf<int> v0;
    TB_CUDA(k0.ensure(ntot_));
    TB_CUDA(k1.ensure(ntot_));
    TB_CUDA(v0.ensure(ntot_));
    k_morton_nodes<<<grid_for(ntot_, kT), kT, 0, stream_>>>(x_.p, node_blk_.p, d_bi_.p, ntot_, k0.p, v0.p);
    TB_LAUNCHED("k_morton_nodes");
    size_t tmpn = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmpn, k0.p, k1.p, v0.p, node_order_.p, (int)ntot_, 0, key_bits,
                                    stream_);
    TB_CUDA(cub_tmp_.ensure(tmpn));
    cub::DeviceRadixSort::SortPairs(cub_tmp_.p, tmpn, k0.p, k1.p, v0.p, node_order_.p, (int)ntot_, 0, key_bits,
                                    stream_);
    TB_CUDA(cudaStreamSynchronize(stream_));
    k0.release();
    k1.release();
    v0.release();
  }
  // 4-ary radix tree per block over the sorted Morton keys (still in
  // mkey_alt_), built level by level; group b holds block b's root
  {
    const int nb = (int)bi_.size();
    long long gcap = std::max<long long>(2 * nb, ctot_ / 8 + 16);  // grows if needed
    DBuf<int2> tlink, kids;
    DBuf<int> ca, cb, cs, na, nbuf, ns, nk, isint, ioff, koff, leaf_at;
    TB_CUDA(tlink.ensure(4 * gcap));
    TB_CUDA(cudaMemsetAsync(tlink.p, 0, 4 * gcap * sizeof(int2), stream_));
    TB_CUDA(gparent_.ensure(gcap));
    TB_CUDA(gnk_.ensure(gcap));
    TB_CUDA(leaf_at.ensure(ctot_));
    TB_CUDA(cudaMemsetAsync(leaf_at.p, 0xff, ctot_ * sizeof(int), stream_));
    std::vector<int> h_a, h_b, h_s, h_par(nb, -1), h_nk(nb, 1);
    for (int b = 0; b < nb; b++) {
      bi_[b].root = bi_[b].ncells > 0 ? 4 * b : -1;
      if (bi_[b].ncells > 0) {
        h_a.push_back(bi_[b].cell_off);
        h_b.push_back(bi_[b].cell_off + bi_[b].ncells);
        h_s.push_back(4 * b);
      }
    }
    TB_CUDA(cudaMemcpyAsync(gparent_.p, h_par.data(), nb * sizeof(int), cudaMemcpyHostToDevice, stream_));
    TB_CUDA(cudaMemcpyAsync(gnk_.p, h_nk.data(), nb * sizeof(int), cudaMemcpyHostToDevice, stream_));
    int n = (int)h_a.size();
    TB_CUDA(ca.ensure(std::max(n, 1)));
    TB_CUDA(cb.ensure(std::max(n, 1)));
    TB_CUDA(cs.ensure(std::max(n, 1)));
    TB_CUDA(cudaMemcpyAsync(ca.p, h_a.data(), n * sizeof(int), cudaMemcpyHostToDevice, stream_));
    TB_CUDA(cudaMemcpyAsync(cb.p, h_b.data(), n * sizeof(int), cudaMemcpyHostToDevice, stream_));
    TB_CUDA(cudaMemcpyAsync(cs.p, h_s.data(), n * sizeof(int), cudaMemcpyHostToDevice, stream_));
    TB_CUDA(cudaStreamSynchronize(stream_));  // host staging vectors go out of scope level by level
    long long g0 = nb;
    int depth = 0;
    while (n > 0) {
      TB_CUDA(kids.ensure(4 * (size_t)n));
      TB_CUDA(nk.ensure(n + 1));
      TB_CUDA(isint.ensure(n + 1));
      TB_CUDA(ioff.ensure(n + 1));
      TB_CUDA(koff.ensure(n + 1));
      k_tree_split<<<grid_for(n, kT), kT, 0, stream_>>>(mkey_alt_.p, n, ca.p, cb.p, cs.p, kids.p, nk.p, isint.p,
                                                        tlink.p, leaf_at.p);
      TB_LAUNCHED("k_tree_split");
      TB_CUDA(cudaMemsetAsync(nk.p + n, 0, sizeof(int), stream_));
      TB_CUDA(cudaMemsetAsync(isint.p + n, 0, sizeof(int), stream_));
      size_t tmp = 0;
      cub::DeviceScan::ExclusiveSum(nullptr, tmp, isint.p, ioff.p, n + 1, stream_);
      TB_CUDA(cub_tmp_.ensure(tmp));
      cub::DeviceScan::ExclusiveSum(cub_tmp_.p, tmp, isint.p, ioff.p, n + 1, stream_);
      cub::DeviceScan::ExclusiveSum(nullptr, tmp, nk.p, koff.p, n + 1, stream_);
      TB_CUDA(cub_tmp_.ensure(tmp));
      cub::DeviceScan::ExclusiveSum(cub_tmp_.p, tmp, nk.p, koff.p, n + 1, stream_);
      int nint = 0, nnext = 0;
      TB_CUDA(cudaMemcpyAsync(&nint, ioff.p + n, sizeof(int), cudaMemcpyDeviceToHost, stream_));
      TB_CUDA(cudaMemcpyAsync(&nnext, koff.p + n, sizeof(int), cudaMemcpyDeviceToHost, stream_));
      TB_CUDA(cudaStreamSynchronize(stream_));
      if (nint > 0 && depth >= kMaxTreeDepth) {  // the traversal keeps one entry per internal level
        fprintf(stderr, "#tioga_b200: cell tree deeper than %d levels\n", kMaxTreeDepth);
        return -1;
      }
      if (g0 + nint > gcap) {  // grow the per-slot and per-group tables, keeping their contents
        const long long ncap = std::max(2 * gcap, g0 + nint);
        DBuf<int2> t2;
        DBuf<int> p2, k2;
        TB_CUDA(t2.ensure(4 * ncap));
        TB_CUDA(p2.ensure(ncap));
        TB_CUDA(k2.ensure(ncap));
        TB_CUDA(cudaMemsetAsync(t2.p, 0, 4 * ncap * sizeof(int2), stream_));
        TB_CUDA(cudaMemcpyAsync(t2.p, tlink.p, 4 * gcap * sizeof(int2), cudaMemcpyDeviceToDevice, stream_));
        TB_CUDA(cudaMemcpyAsync(p2.p, gparent_.p, gcap * sizeof(int), cudaMemcpyDeviceToDevice, stream_));
        TB_CUDA(cudaMemcpyAsync(k2.p, gnk_.p, gcap * sizeof(int), cudaMemcpyDeviceToDevice, stream_));
        TB_CUDA(cudaStreamSynchronize(stream_));
        std::swap(tlink, t2);
        std::swap(gparent_, p2);
        std::swap(gnk_, k2);
        gcap = ncap;
      }
      TB_CUDA(na.ensure(std::max(nnext, 1)));
      TB_CUDA(nbuf.ensure(std::max(nnext, 1)));
      TB_CUDA(ns.ensure(std::max(nnext, 1)));
      k_tree_link<<<grid_for(n, kT), kT, 0, stream_>>>(n, cs.p, kids.p, nk.p, isint.p, ioff.p, koff.p, (int)g0,
                                                       tlink.p, gparent_.p, gnk_.p, na.p, nbuf.p, ns.p);
      TB_LAUNCHED("k_tree_link");
      g0 += nint;
      std::swap(ca, na);
      std::swap(cb, nbuf);
      std::swap(cs, ns);
      n = nnext;
      if (n > 0) depth++;
    }
    tree_depth_ = depth;
    tree_nodes_ = 4 * g0;
    TB_CUDA(tnode_.ensure(2 * tree_nodes_));
    k_tree_init<<<grid_for(tree_nodes_, kT), kT, 0, stream_>>>(tlink.p, tree_nodes_, tnode_.p);
    TB_LAUNCHED("k_tree_init");
    // the one-launch refit's counts and starting groups
    {
      const int ng = (int)(tree_nodes_ / 4);
      TB_CUDA(gnint_.ensure(std::max(ng, 1)));
      TB_CUDA(refit_start_.ensure(std::max(ng, 1)));
      TB_CUDA(refit_cnt_.ensure(std::max(ng, 1)));
      DBuf<int> ns;
      TB_CUDA(ns.ensure(1));
      TB_CUDA(cudaMemsetAsync(ns.p, 0, sizeof(int), stream_));
      if (ng > nb) {
        k_group_nint<<<grid_for(ng - nb, kT), kT, 0, stream_>>>(tnode_.p, nb, ng, gnint_.p, refit_start_.p, ns.p);
        TB_LAUNCHED("k_group_nint");
      }
      TB_CUDA(cudaMemcpyAsync(&nrefit_start_, ns.p, sizeof(int), cudaMemcpyDeviceToHost, stream_));
      TB_CUDA(cudaStreamSynchronize(stream_));
    }
    tnode64_empty_ = false;
    // leaves in storage order
    DBuf<int> flag, loff;
    TB_CUDA(flag.ensure(ctot_ + 1));
    TB_CUDA(loff.ensure(ctot_ + 1));
    k_leaf_flags<<<grid_for(ctot_, kT), kT, 0, stream_>>>(leaf_at.p, ctot_, flag.p);
    TB_LAUNCHED("k_leaf_flags");
    TB_CUDA(cudaMemsetAsync(flag.p + ctot_, 0, sizeof(int), stream_));
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, flag.p, loff.p, (int)(ctot_ + 1), stream_);
    TB_CUDA(cub_tmp_.ensure(tmp));
    cub::DeviceScan::ExclusiveSum(cub_tmp_.p, tmp, flag.p, loff.p, (int)(ctot_ + 1), stream_);
    int nl = 0;
    TB_CUDA(cudaMemcpyAsync(&nl, loff.p + ctot_, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaStreamSynchronize(stream_));
    nleaf_total_ = nl;
    TB_CUDA(leaves_.ensure(std::max(nl, 1)));
    k_leaf_list<<<grid_for(ctot_, kT), kT, 0, stream_>>>(leaf_at.p, loff.p, ctot_, tlink.p, cell_blk_.p,
                                                         leaves_.p);
    TB_LAUNCHED("k_leaf_list");
    // leaves of block b: [blk_leaf_[b], blk_leaf_[b + 1])
    DBuf<int> first;
    TB_CUDA(first.ensure(nb));
    TB_CUDA(cudaMemsetAsync(first.p, 0xff, nb * sizeof(int), stream_));
    if (nl > 0) {
      k_block_leaves<<<grid_for(nl, kT), kT, 0, stream_>>>(leaves_.p, nl, first.p);
      TB_LAUNCHED("k_block_leaves");
    }
    h_blk_leaf_.assign(nb + 1, nl);
    TB_CUDA(cudaMemcpyAsync(h_blk_leaf_.data(), first.p, nb * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaStreamSynchronize(stream_));
    for (int b = nb - 1; b >= 0; b--)
      if (h_blk_leaf_[b] < 0) h_blk_leaf_[b] = h_blk_leaf_[b + 1];
    TB_TRY(build_upload_chunks());
  }
  // cells (storage order) that mark their wall-bearing block's hole map
  {
    DBuf<int> flag, off;
    TB_CUDA(flag.ensure(ctot_ + 1));
    TB_CUDA(off.ensure(ctot_ + 1));
    k_wall_cell_flags<<<grid_for(ctot_, kT), kT, 0, stream_>>>(conn8_.p, cell_nv_.p, cell_blk_.p, d_bi_.p, wallf_.p,
                                                               ctot_, flag.p);
    TB_LAUNCHED("k_wall_cell_flags");
    TB_CUDA(cudaMemsetAsync(flag.p + ctot_, 0, sizeof(int), stream_));
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, flag.p, off.p, (int)(ctot_ + 1), stream_);
    TB_CUDA(cub_tmp_.ensure(tmp));
    cub::DeviceScan::ExclusiveSum(cub_tmp_.p, tmp, flag.p, off.p, (int)(ctot_ + 1), stream_);
    int nwc = 0;
    TB_CUDA(cudaMemcpyAsync(&nwc, off.p + ctot_, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaStreamSynchronize(stream_));
    nwall_cells_ = nwc;
    TB_CUDA(wall_cells_.ensure(std::max(nwc, 1)));
    const int nh = std::max(nhm_all_, 1);
    TB_CUDA(wall_box_first_.ensure(nh + 1));
    TB_CUDA(wall_box_.ensure(std::max(nwc, 1)));
    TB_CUDA(cudaMemsetAsync(wall_box_first_.p, 0xff, (nh + 1) * sizeof(int), stream_));
    if (nwc > 0) {
      k_wall_cell_list<<<grid_for(ctot_, kT), kT, 0, stream_>>>(flag.p, off.p, ctot_, wall_cells_.p);
      TB_LAUNCHED("k_wall_cell_list");
      k_wall_map_first<<<grid_for(nwc, kT), kT, 0, stream_>>>(wall_cells_.p, nwc, cell_blk_.p, d_bi_.p,
                                                              wall_box_first_.p);
      TB_LAUNCHED("k_wall_map_first");
    }
    // wall cells of map t: [first[t], first[t + 1]) (maps without any: empty)
    std::vector<int> first(nh + 1);
    TB_CUDA(cudaMemcpyAsync(first.data(), wall_box_first_.p, nh * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaStreamSynchronize(stream_));
    first[nh] = nwc;
    for (int t = nh - 1; t >= 0; t--)
      if (first[t] < 0) first[t] = first[t + 1];
    TB_CUDA(cudaMemcpyAsync(wall_box_first_.p, first.data(), (nh + 1) * sizeof(int), cudaMemcpyHostToDevice,
                            stream_));
    TB_CUDA(cudaStreamSynchronize(stream_));
  }
  // query-gathering tiles of kNodeTile nodes per block
  h_tile_base_.assign(bi_.size() + 1, 0);
  for (size_t b = 0; b < bi_.size(); b++)
    h_tile_base_[b + 1] = h_tile_base_[b] + (bi_[b].nnodes + kNodeTile - 1) / kNodeTile;
  TB_CUDA(tile_base_.ensure(bi_.size() + 1));
  TB_CUDA(cudaMemcpyAsync(tile_base_.p, h_tile_base_.data(), h_tile_base_.size() * sizeof(long long),
                          cudaMemcpyHostToDevice, stream_));
  TB_CUDA(tbox_.ensure(2 * std::max(1ll, h_tile_base_.back())));
  TB_CUDA(cbox_.ensure(3 * ctot_));
  TB_TRY(build_tile_chunks());
  TB_CUDA(cudaStreamSynchronize(stream_));  // host tables above stay valid
  topo_gen_++;  // the cell arrays were replaced by their storage-order copies
  return 0;
}

// ---------------------------------------------------------------------------
// preprocess (src/tioga.C:95-110, MeshBlock.C:74-339)
// ---------------------------------------------------------------------------
int Engine::preprocess() {
  if (hb_.empty()) return 0;
  bool fresh = topo_dirty_;
  if (topo_dirty_) {
    int rc = upload_topology();
    if (rc) return rc;
  }
  for (auto& B : bi_) B.nfringe = nfringe_;
  for (size_t b = 0; b < hb_.size(); b++) bi_[b].has_user_res = (hb_[b].user_nres || hb_[b].user_cres);
  TB_CUDA(cudaMemcpyAsync(d_bi_.p, bi_.data(), bi_.size() * sizeof(BlockInfo), cudaMemcpyHostToDevice,
                          stream_));
  if (!coords_resident_ || !coords_on_device_ || fresh) TB_TRY(upload_coords());
  TB_TRY(compute_obbs());
  // keep the OBBs and block boxes on the host too
  TB_CUDA(cudaMemcpyAsync(bi_.data(), d_bi_.p, bi_.size() * sizeof(BlockInfo), cudaMemcpyDeviceToHost,
                          stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  if (fresh || tree_nodes_ == 0) {
    TB_TRY(build_tree_topology());  // also puts the cell arrays in storage order
    TB_CUDA(cudaMemcpyAsync(d_bi_.p, bi_.data(), bi_.size() * sizeof(BlockInfo), cudaMemcpyHostToDevice,
                            stream_));
  }
  // rigid motions keep every distance (to rounding far below the gate's
  // distance), so the gate of the last preprocess still holds after them
  if (!gate_valid_) TB_TRY(dedup_gate());
  gate_valid_ = true;
  TB_TRY(setup_uniform_hex());
  for (size_t b = 0; b < hb_.size(); b++) {
    const HostBlock& H = hb_[b];
    if (!bi_[b].has_user_res) continue;
    TB_CUDA(cudaMemcpyAsync(node_res_.p + bi_[b].node_off, H.user_nres, H.nnodes * sizeof(double),
                            cudaMemcpyHostToDevice, stream_));
    DBuf<double> stage;
    TB_CUDA(stage.ensure(H.ncells));
    TB_CUDA(cudaMemcpyAsync(stage.p, H.user_cres, H.ncells * sizeof(double), cudaMemcpyHostToDevice, stream_));
    k_scatter_f64<<<grid_for(H.ncells, kT), kT, 0, stream_>>>(stage.p, H.ncells, inv_sorted_.p, bi_[b].cell_off,
                                                               cell_res_.p);
    TB_LAUNCHED("k_scatter_f64");
    TB_CUDA(cudaStreamSynchronize(stream_));
    stage.release();
  }
  bool user_res = false;
  for (const BlockInfo& B : bi_) user_res = user_res || B.has_user_res;
  bool ran = false;
  if (use_graphs_ && stream_ == own_stream_ && !sync_check() && !user_res) {
    // the resolution and iblank stage is the same launches for a topology:
    // captured once into a CUDA graph and replayed by every later preprocess
    // (the serving form's time steps).  Any capture failure falls back to
    // plain launches for good.
    const long long key = topo_gen_ * 64 + mexclude_;
    if (!pre_exec_ || pre_key_ != key) {
      if (pre_exec_) cudaGraphExecDestroy(pre_exec_);
      pre_exec_ = nullptr;
      const long long n0 = nlaunch_;
      cudaGraph_t g = nullptr;
      if (cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const int rc = preprocess_resolutions();
        const cudaError_t e = cudaStreamEndCapture(stream_, &g);
        if (rc == 0 && e == cudaSuccess && g && cudaGraphInstantiate(&pre_exec_, g, 0) == cudaSuccess) {
          pre_key_ = key;
          pre_nlaunch_ = nlaunch_ - n0;
        } else {
          pre_exec_ = nullptr;
          use_graphs_ = false;
        }
        if (g) cudaGraphDestroy(g);
      } else {
        use_graphs_ = false;
      }
      cudaGetLastError();  // a failed capture leaves no sticky error
      nlaunch_ = n0;
    }
    if (pre_exec_) {
      TB_CUDA(cudaGraphLaunch(pre_exec_, stream_));
      nlaunch_ += pre_nlaunch_;
      ran = true;
    }
  }
  if (!ran) TB_TRY(preprocess_resolutions());
  for (size_t b = 0; b < hb_.size(); b++) {  // preprocess sets iblank = 1 (MeshBlock.C:80)
    HostBlock& H = hb_[b];
    if (H.dibl)
      TB_CUDA(cudaMemcpyAsync(H.dibl, iblank_.p + bi_[b].node_off, H.nnodes * sizeof(int),
                              cudaMemcpyDeviceToDevice, stream_));
    else if (!serving_)
      for (int i = 0; i < H.nnodes; i++) H.hibl[i] = 1;
  }
  TB_CUDA(cudaStreamSynchronize(stream_));
  preprocessed_ = true;
  donor_rest_ = false;
  connected_ = false;
  interps_fetched_ = false;
  return 0;
}

// Cell volumes and node resolutions (tagBoundary, MeshBlock.C:94-339), the
// mandatory receptors and mexclude rounds, and iblank = 1: launches only, on
// buffers fixed by the topology (a CUDA graph can hold them).
int Engine::preprocess_resolutions() {
  k_cell_volume<<<grid_for(ctot_, kT), kT, 0, stream_>>>(x_.p, conn8_.p, cell_nv_.p, cell_blk_.p, d_bi_.p,
                                                          ctot_, cell_res_.p);
  TB_LAUNCHED("k_cell_volume");
  k_node_res<<<grid_for(ntot_, kT), kT, 0, stream_>>>(csr_off_.p, csr_cell_.p, cell_res_.p, node_blk_.p,
                                                       d_bi_.p, ntot_, node_res_.p);
  TB_LAUNCHED("k_node_res");
  TB_CUDA(cudaMemsetAsync(ex0_.p, 0, ntot_, stream_));
  TB_CUDA(cudaMemsetAsync(ex1_.p, 0, ntot_, stream_));
  k_mandatory<<<grid_for(ctot_, kT), kT, 0, stream_>>>(conn8_.p, cell_nv_.p, ctot_, obcf_.p, node_res_.p,
                                                        ex0_.p, ex1_.p);
  TB_LAUNCHED("k_mandatory");
  for (int it = 0; it < mexclude_; it++) {
    k_mexclude<<<grid_for(ctot_, kT), kT, 0, stream_>>>(conn8_.p, cell_nv_.p, ctot_, ex0_.p, ex1_.p,
                                                         cell_res_.p);
    TB_LAUNCHED("k_mexclude");
    k_copy_u8<<<grid_for(ntot_, kT), kT, 0, stream_>>>(ex1_.p, ex0_.p, ntot_);
    TB_LAUNCHED("k_copy_u8");
  }
  k_fill_int<<<grid_for(ntot_, kT), kT, 0, stream_>>>(iblank_.p, 1, ntot_);
  TB_LAUNCHED("k_fill_int");
  return 0;
}

// ---------------------------------------------------------------------------
// connectivity (src/tioga.C:112-160)
// ---------------------------------------------------------------------------
// Every wall-bearing block's map at once: wall bounds -> extents and sizes
// -> mark -> fill -> final, on the side stream after hev_[0].  The first
// half ends with the maps' extents copied to pinned host memory (hev_[1]);
// holemaps_end reads them once the main stream's work is queued.
int Engine::holemaps_begin() {
  const int nh = nhm_all_;
  nhm_ = 0;
  hm_pending_ = false;
  if (nh == 0) return 0;
  if (h_hm_cap_ < nh) {
    if (h_hm_init_) cudaFreeHost(h_hm_init_);
    if (h_hm_info_) cudaFreeHost(h_hm_info_);
    if (h_hm_dev_) cudaFreeHost(h_hm_dev_);
    h_hm_init_ = nullptr;
    h_hm_info_ = nullptr;
    h_hm_dev_ = nullptr;
    h_hm_cap_ = 0;
    TB_CUDA(cudaMallocHost(&h_hm_init_, 6 * (size_t)nh * sizeof(unsigned long long)));
    TB_CUDA(cudaMallocHost(&h_hm_info_, (size_t)nh * sizeof(HoleMapInfo)));
    TB_CUDA(cudaMallocHost(&h_hm_dev_, (size_t)nh * sizeof(HoleMapDev)));
    h_hm_cap_ = nh;
  }
  cudaStream_t hs = side_;
  TB_CUDA(cudaStreamWaitEvent(hs, hev_[0], 0));
  for (int t = 0; t < nh; t++)
    for (int j = 0; j < 3; j++) {  // identity elements of min (all ones) and max (zero) over ordered keys
      h_hm_init_[6 * t + j] = ~0ull;
      h_hm_init_[6 * t + j + 3] = 0ull;
    }
  TB_CUDA(cudaMemcpyAsync(wall_bb_.p, h_hm_init_, 6 * (size_t)nh * sizeof(unsigned long long),
                          cudaMemcpyHostToDevice, hs));
  const unsigned nw = (unsigned)h_wall_.size();
  int maxw = 1;
  for (const WallBlock& W : h_wall_) maxw = std::max(maxw, W.nwall);
  k_wall_bounds<<<dim3(grid_for(maxw, kT, 148), nw), kT, 0, hs>>>(x_.p, wall_list_.p, d_wall_.p, wall_bb_.p);
  TB_LAUNCHED_ON("k_wall_bounds", hs);
  k_holemap_setup<<<(nh + 127) / 128, 128, 0, hs>>>(wall_bb_.p, d_hm_.p, nh);
  TB_LAUNCHED_ON("k_holemap_setup", hs);
  const bool planar = (isym_ == 1 || isym_ == 2 || isym_ == 3);
  // the plane fill rewrites every cell of its map, so only this call's marks
  // (2) count there; the 6-neighbour fill reads the map as it is
  if (!planar) TB_CUDA(cudaMemsetAsync(hm_state_.p, 0, (size_t)nh * kHoleMapCap, hs));
  if (nwall_cells_ > 0 && planar) {  // the boxes the plane fill marks in shared memory
    k_holemap_boxes<<<grid_for(nwall_cells_, kT), kT, 0, hs>>>(x_.p, conn8_.p, cell_nv_.p, wall_cells_.p,
                                                               nwall_cells_, cell_blk_.p, d_bi_.p, d_hm_.p,
                                                               wall_box_.p);
    TB_LAUNCHED_ON("k_holemap_boxes", hs);
  } else if (nwall_cells_ > 0) {
    k_holemap_mark<<<grid_for(nwall_cells_, kT), kT, 0, hs>>>(x_.p, conn8_.p, cell_nv_.p, wall_cells_.p,
                                                              nwall_cells_, cell_blk_.p, d_bi_.p, d_hm_.p,
                                                              hm_state_.p, kHoleMapCap);
    TB_LAUNCHED_ON("k_holemap_mark", hs);
  }
  TB_CUDA(cudaMemcpyAsync(h_hm_info_, d_hm_.p, nh * sizeof(HoleMapInfo), cudaMemcpyDeviceToHost, hs));
  TB_CUDA(cudaEventRecord(hev_[1], hs));
  hm_pending_ = true;
  return 0;
}

int Engine::holemaps_end() {
  const int nh = nhm_all_;
  if (!hm_pending_) {  // no maps: the donor phase's wait on hev_[2] passes at once
    TB_CUDA(cudaEventRecord(hev_[2], side_));
    return 0;
  }
  hm_pending_ = false;
  cudaStream_t hs = side_;
  TB_CUDA(cudaEventSynchronize(hev_[1]));
  const HoleMapInfo* hinfo = h_hm_info_;
  const bool planar = (isym_ == 1 || isym_ == 2 || isym_ == 3);
  const int isym = isym_;
  const int pa = (isym == 1) ? 0 : (isym == 2) ? 1 : 2;
  const int a0 = (pa == 0) ? 1 : 0, a1 = (pa == 2) ? 1 : 2;
  int maxpl = 1;
  size_t smem = 1;
  long long maxcells = 1;
  for (int t = 0; t < nh; t++) {
    const HoleMapInfo& h = hinfo[t];
    if (h.nx[0] > 197 || h.nx[1] > 197 || h.nx[2] > 197 || h.nx[0] < 1 || h.nx[1] < 1 || h.nx[2] < 1) {
      fprintf(stderr, "#tioga_b200: hole map %d has an unexpected size\n", t);
      TB_CUDA(cudaEventRecord(hev_[2], hs));
      return -1;
    }
    maxpl = std::max(maxpl, h.nx[pa]);
    smem = std::max(smem, (size_t)h.nx[a0] * h.nx[a1]);
    maxcells = std::max(maxcells, (long long)h.nx[0] * h.nx[1] * h.nx[2]);
    stats_.holemap_cells += (long long)h.nx[0] * h.nx[1] * h.nx[2];
  }
  if (planar) {  // fill and final map in one pass
    k_holemap_fill_bits<<<dim3(std::min(maxpl, 148 * 4), nh), 256, 0, hs>>>(
        hm_state_.p, d_hm_.p, kHoleMapCap, wall_box_.p, wall_box_first_.p, isym, test_fill_rounds_, err_.p);
    TB_LAUNCHED_ON("k_holemap_fill_bits", hs);
  } else {
    k_holemap_fill_planes<<<dim3(std::min(maxpl, 148 * 4), nh), 256, smem, hs>>>(hm_state_.p, d_hm_.p,
                                                                                kHoleMapCap, 3, 1, err_.p);
    TB_LAUNCHED_ON("k_holemap_fill_planes", hs);  // 6-neighbour fill: line sweeps over the three axes until no map changes
    unsigned* d_changed = err_.p + 1;
    int maxsum = 0;
    for (int t = 0; t < nh; t++) maxsum = std::max(maxsum, hinfo[t].nx[0] + hinfo[t].nx[1] + hinfo[t].nx[2]);
    for (int round = 0; round < 4 * maxsum; round++) {
      TB_CUDA(cudaMemsetAsync(d_changed, 0, sizeof(unsigned), hs));
      for (int axis = 0; axis < 3; axis++) {
        k_holemap_lines<<<dim3(grid_for(maxcells / 64 + 1, kT), nh), kT, 0, hs>>>(hm_state_.p, d_hm_.p,
                                                                                 kHoleMapCap, axis, d_changed);
        TB_LAUNCHED_ON("k_holemap_lines", hs);
      }
      unsigned ch = 0;
      TB_CUDA(cudaMemcpyAsync(&ch, d_changed, sizeof(unsigned), cudaMemcpyDeviceToHost, hs));
      TB_CUDA(cudaStreamSynchronize(hs));
      if (!ch) break;
    }
    k_holemap_final<<<dim3(grid_for(maxcells, kT), nh), kT, 0, hs>>>(hm_state_.p, d_hm_.p, kHoleMapCap);
    TB_LAUNCHED_ON("k_holemap_final", hs);
  }
  for (int b = 0; b < (int)bi_.size(); b++) {
    const int t = bi_[b].hm;
    if (t < 0) continue;
    HoleMapDev& d = h_hm_dev_[t];
    d.tagidx = bi_[b].tag - 1;
    for (int j = 0; j < 3; j++) d.nx[j] = hinfo[t].nx[j];
    for (int j = 0; j < 6; j++) d.ext[j] = hinfo[t].ext[j];
    d.hole = hm_state_.p + (size_t)t * kHoleMapCap;
  }
  nhm_ = nh;
  // pinned source: the copy does not hold the host; the buffer is next
  // written by the next call, after this call's final synchronisation
  TB_CUDA(cudaMemcpyAsync(d_hmdev_.p, h_hm_dev_, nh * sizeof(HoleMapDev), cudaMemcpyHostToDevice, hs));
  TB_CUDA(cudaEventRecord(hev_[2], hs));
  return 0;
}

int Engine::run_pairs_and_refit() {
  const int nb = (int)hb_.size();
  TB_CUDA(d_pairs_.ensure(npcand_ + 1));
  TB_CUDA(d_npairs_.ensure(1));
  TB_CUDA(d_pfirst_.ensure(nb + 1));
  k_pairs<<<1, 1024, 0, stream_>>>(d_bi_.p, nb, d_pcand_.p, npcand_, d_pairs_.p, d_npairs_.p, d_pfirst_.p);
  TB_LAUNCHED("k_pairs");
  TB_CUDA(cudaMemcpyAsync(&npairs_, d_npairs_.p, sizeof(int), cudaMemcpyDeviceToHost, stream_));
  h_pairs_.resize(npcand_ + 1);
  h_pfirst_.resize(nb + 1);
  TB_CUDA(cudaMemcpyAsync(h_pairs_.data(), d_pairs_.p, (npcand_ + 1) * sizeof(PairInfo), cudaMemcpyDeviceToHost,
                          stream_));
  TB_CUDA(cudaMemcpyAsync(h_pfirst_.data(), d_pfirst_.p, (nb + 1) * sizeof(int), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaEventRecord(pev_, stream_));
  // the node tiles' boxes (query gathering, hole search) and, for the split
  // form's cell boxes, the FP32 copy of the coordinates, while the host
  // waits for the pairs
  if (precision_ != 0) TB_CUDA(xf_.ensure(ntot_));
  if (h_tile_base_.back() > 0 && !tiles_ready_) {  // (else made during the chunked upload)
    k_node_tiles<<<(unsigned)h_tile_base_.back(), 256, 0, stream_>>>(x_.p, d_bi_.p, nb, tile_base_.p, tbox_.p,
                                                                      node_order_.p,
                                                                      precision_ != 0 && !boxes_ready_ ? xf_.p
                                                                                                       : nullptr,
                                                                      nullptr);
    TB_LAUNCHED("k_node_tiles");
  }
  TB_CUDA(cudaEventSynchronize(pev_));
  if (npairs_ == 0) return 0;
  // refit to the current coordinates: one pass over the cells (tree-order
  // cell boxes + reduced boxes of every pair), then the tree levels, then the
  // node tiles of the query gathering
  const bool fp64 = (precision_ == 0);
  if (fp64) {
    TB_CUDA(cbox64_.ensure(6 * ctot_));
    TB_CUDA(tnode64_.ensure(6 * tree_nodes_));
    if (!tnode64_empty_) {
      k_tree_init64<<<grid_for(tree_nodes_, kT), kT, 0, stream_>>>(tree_nodes_, tnode64_.p);
      TB_LAUNCHED("k_tree_init64");
      tnode64_empty_ = true;
    }
  }
  std::vector<unsigned long long> acc(6 * npairs_);
  for (int p = 0; p < npairs_; p++)
    for (int j = 0; j < 3; j++) {  // BIG / -BIG as getReducedOBB starts (MeshBlock.C:790-794)
      double lo = kBig, hi = -kBig;
      unsigned long long bl, bh;
      memcpy(&bl, &lo, 8);
      memcpy(&bh, &hi, 8);
      acc[6 * p + j] = (bl & 0x8000000000000000ull) ? ~bl : (bl | 0x8000000000000000ull);
      acc[6 * p + j + 3] = (bh & 0x8000000000000000ull) ? ~bh : (bh | 0x8000000000000000ull);
    }
  TB_CUDA(pair_acc_.ensure(6 * npairs_));
  TB_CUDA(cudaMemcpyAsync(pair_acc_.p, acc.data(), acc.size() * sizeof(unsigned long long),
                          cudaMemcpyHostToDevice, stream_));
  if (!fp64) {  // the seeds of the extents' bounds start open
    std::vector<int> ext(6 * npairs_);
    for (int i = 0; i < 6 * npairs_; i++) ext[i] = (i % 6 < 3) ? 0x7fffffff : (int)0x80000000;
    TB_CUDA(pair_ext_.ensure(6 * npairs_));
    TB_CUDA(cudaMemcpyAsync(pair_ext_.p, ext.data(), ext.size() * sizeof(int), cudaMemcpyHostToDevice, stream_));
  }
  // chunks of consecutive blocks whose pairs fit one CTA's shared memory;
  // the CTAs of one launch are split among the chunks by leaf count.  The
  // FP64 kernel writes every cell's box, so its chunks cover every block;
  // the split form's pair kernel only visits blocks that donate to a pair.
  const int kChunkPairs = std::max(16, std::min(128, tune_.chunk_pairs));
  const std::vector<int>& item_of_blk = h_blk_leaf_;
  // leaves a CTA of 256 threads takes at once: a lane per cell in the FP64
  // kernel, a lane per leaf in the split form's scan
  const long long per_cta = fp64 ? 256 / kMaxLeafCells : 256;
  auto donates = [&](int b) { return fp64 || h_pfirst_[b + 1] > h_pfirst_[b]; };
  std::vector<int4> chunks;
  long long nitems = 0;
  for (int b = 0; b < nb;) {
    if (!donates(b)) {
      b++;
      continue;
    }
    int e = b + 1;
    while (e < nb && donates(e) && h_pfirst_[e + 1] - h_pfirst_[b] <= kChunkPairs) e++;
    chunks.push_back(make_int4(item_of_blk[b], item_of_blk[e], h_pfirst_[b], h_pfirst_[e] - h_pfirst_[b]));
    nitems += item_of_blk[e] - item_of_blk[b];
    b = e;
  }
  const long long want = grid_for(nitems * (256 / per_cta), 256, 148 * tune_.cell_pass_per_sm);
  std::vector<int> ccta(chunks.size() + 1, 0);
  int maxnp = 1;
  for (size_t k = 0; k < chunks.size(); k++) {
    const long long nl = chunks[k].y - chunks[k].x;
    long long n = nitems > 0 ? (want * nl + nitems - 1) / nitems : 1;
    n = std::max(1ll, std::min(n, (nl + per_cta - 1) / per_cta));
    ccta[k + 1] = ccta[k] + (int)n;
    maxnp = std::max(maxnp, chunks[k].w);
  }
  TB_CUDA(d_chunks_.ensure(chunks.size()));
  TB_CUDA(d_chunk_cta_.ensure(ccta.size()));
  TB_CUDA(cudaMemcpyAsync(d_chunks_.p, chunks.data(), chunks.size() * sizeof(int4), cudaMemcpyHostToDevice, stream_));
  TB_CUDA(cudaMemcpyAsync(d_chunk_cta_.p, ccta.data(), ccta.size() * sizeof(int), cudaMemcpyHostToDevice, stream_));
  TB_CUDA(cudaEventRecord(cev_[0], stream_));
  const size_t smem = (size_t)maxnp * (6 * sizeof(unsigned long long) + sizeof(PairCull) + 6 * sizeof(int));
  if (fp64) {
    launch_cell_pass64(tune_.cell_pass_per_sm, ccta.back(), smem, stream_, x_.p, conn8_.p, cell_nv_.p, d_bi_.p,
                       leaves_.p, d_chunks_.p, d_chunk_cta_.p, (int)chunks.size(), d_pfirst_.p, d_pairs_.p,
                       cbox64_.p, tnode_.p, tnode64_.p, pair_acc_.p);
    TB_CUDA(cudaEventRecord(cev_[2], stream_));
    TB_CUDA(cudaEventRecord(hev_[0], stream_));  // the hole maps may start
  } else {
    const int mb = tune_.cell_box_per_sm;
    TB_CUDA(lbox_.ensure(2 * nleaf_total_));
    if (!boxes_ready_) {  // else made during the chunked upload
      launch_cell_boxes(mb, (int)grid_for(nleaf_total_ * kMaxLeafCells, 256, 148 * mb), stream_, xf_.p, conn8_.p,
                        cell_nv_.p, leaves_.p, nullptr, nleaf_total_, cbox_.p, tnode_.p, lbox_.p);
      TB_LAUNCHED("k_cell_boxes");
    }
    TB_CUDA(cudaEventRecord(hev_[0], stream_));  // the hole maps may start
    TB_CUDA(cudaEventRecord(cev_[2], stream_));
    launch_cell_pairs(tune_.cell_pass_per_sm, ccta.back(), smem, stream_, x_.p, conn8_.p, cell_nv_.p, d_bi_.p,
                      leaves_.p, d_chunks_.p, d_chunk_cta_.p, (int)chunks.size(), d_pfirst_.p, d_pairs_.p, cbox_.p,
                      lbox_.p, pair_ext_.p, pair_acc_.p);
    TB_LAUNCHED("k_leaf_seeds");
  }
  TB_LAUNCHED("k_cell_pass");
  TB_CUDA(cudaEventRecord(cev_[1], stream_));
  cell_timed_ = true;
  // internal nodes from the leaves the cell pass wrote, in one launch on the
  // side stream: only the traversal reads them (it waits for rf_ev_)
  TB_CUDA(cudaStreamWaitEvent(side_, hev_[0], 0));
  if (nrefit_start_ > 0) {
    TB_CUDA(cudaMemsetAsync(refit_cnt_.p, 0, (tree_nodes_ / 4) * sizeof(int), side_));
    k_refit_fused<<<grid_for(nrefit_start_, kT), kT, 0, side_>>>(refit_start_.p, nrefit_start_, gparent_.p,
                                                                 gnint_.p, (int)hb_.size(), refit_cnt_.p, tnode_.p,
                                                                 fp64 ? tnode64_.p : nullptr);
    TB_LAUNCHED_ON("k_refit_fused", side_);
  }
  TB_CUDA(cudaEventRecord(rf_ev_, side_));
  k_pair_finish<<<(npairs_ + 63) / 64, 64, 0, stream_>>>(d_bi_.p, d_pairs_.p, npairs_, pair_acc_.p);
  TB_LAUNCHED("k_pair_finish");
  return 0;
}

int Engine::run_queries() {
  // ordered compaction of each pair's receptor nodes inside the donor region,
  // over one list of every pair's node tiles
  const int tile = kNodeTile;  // 256 threads x 8 nodes, one node tile
  h_pair_t0_.assign(npairs_ + 1, 0);
  for (int p = 0; p < npairs_; p++)
    h_pair_t0_[p + 1] = h_pair_t0_[p] + (bi_[h_pairs_[p].rec].nnodes + tile - 1) / tile;
  const long long ntiles = h_pair_t0_[npairs_];
  TB_CUDA(d_pair_t0_.ensure(npairs_ + 1));
  TB_CUDA(cudaMemcpyAsync(d_pair_t0_.p, h_pair_t0_.data(), (npairs_ + 1) * sizeof(long long), cudaMemcpyHostToDevice,
                          stream_));
  TB_CUDA(tile_cnt_.ensure(ntiles + 1));
  TB_CUDA(tile_off_.ensure(ntiles + 1));
  TB_CUDA(cudaMemsetAsync(tile_cnt_.p, 0, (ntiles + 1) * sizeof(int), stream_));
  const unsigned grid = (unsigned)std::max(1ll, std::min(ntiles, 148ll * tune_.query_per_sm));
  TB_CUDA(tile_mask_.ensure(ntiles * 256));  // per tile and thread: which of its 8 nodes are inside
  k_query_count<<<grid, 256, 0, stream_>>>(x_.p, d_bi_.p, d_pairs_.p, npairs_, d_pair_t0_.p, tile, tile_cnt_.p,
                                           tbox_.p, tile_base_.p, node_order_.p, tile_mask_.p);
  TB_LAUNCHED("k_query_count");
  size_t tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp, tile_cnt_.p, tile_off_.p, (int)(ntiles + 1), stream_);
  TB_CUDA(cub_tmp_.ensure(tmp));
  cub::DeviceScan::ExclusiveSum(cub_tmp_.p, tmp, tile_cnt_.p, tile_off_.p, (int)(ntiles + 1), stream_);
  int nq = 0;
  TB_CUDA(cudaMemcpyAsync(&nq, tile_off_.p + ntiles, sizeof(int), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  nq_ = nq;
  TB_CUDA(qnode_.ensure(nq));
  TB_CUDA(qdon_.ensure(nq));
  TB_CUDA(qres_.ensure(nq));
  TB_CUDA(qcell_.ensure(nq));
  TB_CUDA(qtie_.ensure(nq));
  TB_CUDA(interp2rec_.ensure(nq));
  if (nq > 0) {
    k_query_write<<<grid, 256, 0, stream_>>>(d_bi_.p, d_pairs_.p, npairs_, d_pair_t0_.p, tile, tile_off_.p,
                                             node_res_.p, qnode_.p, qdon_.p, qres_.p, node_order_.p, tile_mask_.p);
    TB_LAUNCHED("k_query_write");
  }
  dedup_ran_ = false;
  if (nodegid_merge_ && nq > 0) TB_TRY(run_gid_merge());
  else if (dedup_active_ && nq > 0) TB_TRY(run_dedup());
  return 0;
}

// search in four stages: traversal -> candidate list -> one thread per
// candidate (exact box test, FP32 screen) -> FP64 refinement -> outcome
int Engine::run_search() {
  TB_CUDA(scount_.ensure(2));
  TB_CUDA(cudaMemsetAsync(scount_.p, 0, 2 * sizeof(unsigned), stream_));
  ncand_ = 0;
  if (nq_ == 0) return 0;
  const int form = (precision_ == 0) ? 0 : 1;
  TB_CUDA(qkey_.ensure(nq_));
  TB_CUDA(qacc_.ensure(nq_));
  TB_CUDA(cudaMemsetAsync(qkey_.p, 0xff, nq_ * sizeof(unsigned long long), stream_));
  TB_CUDA(cudaMemsetAsync(qacc_.p, 0, nq_ * sizeof(unsigned), stream_));
  unsigned count = 0;
  TB_CUDA(cudaEventRecord(sev_[0], stream_));
  TB_TRY(traverse_and_gather(x_.p, qnode_.p, qdon_.p, nq_, count, any_uhex_ ? 1 : 0));
  ncand_ = count;
  TB_CUDA(cudaEventRecord(sev_[1], stream_));
  if (count > 0) {
    TB_CUDA(refine_.ensure(count));
    launch_candidates(form, grid_for(count, 256, 148 * tune_.candidates_per_sm), stream_, x_.p, conn8_.p, cell_nv_.p, cell_res_.p, sorted_cell_.p,
                      qnode_.p, cand_.p, (int)count, qkey_.p, qacc_.p, refine_.p, scount_.p + 1, counters_.p);
    TB_LAUNCHED("k_candidates");
    TB_CUDA(cudaEventRecord(sev_[2], stream_));
    if (form == 1) {
      k_refine<<<grid_for(count / 4 + 1, 128), 128, 0, stream_>>>(x_.p, conn8_.p, cell_nv_.p, cell_res_.p,
                                                                  sorted_cell_.p, qnode_.p, cand_.p, refine_.p,
                                                                  scount_.p + 1, qkey_.p, qacc_.p);
      TB_LAUNCHED("k_refine");
    }
  }
  if (count == 0) TB_CUDA(cudaEventRecord(sev_[2], stream_));
  TB_CUDA(cudaEventRecord(sev_[3], stream_));
  k_search_finish<<<grid_for(nq_, kT), kT, 0, stream_>>>(qkey_.p, qacc_.p, nq_, inv_sorted_.p, qcell_.p, qtie_.p,
                                                         counters_.p);
  TB_LAUNCHED("k_search_finish");
  if (any_uhex_) {  // donors that are uniform boxes: the index lookup (search.C:271-341)
    k_uhex_search<<<grid_for(nq_, kT), kT, 0, stream_>>>(x_.p, qnode_.p, qdon_.p, nq_, d_bi_.p, uhex_map_.p,
                                                         cell_res_.p, inv_sorted_.p, qcell_.p, qtie_.p);
    TB_LAUNCHED("k_uhex_search");
  }
  if (dedup_ran_) {  // merged coincident points take their representative's donor
    k_dedup_copy<<<grid_for(nq_, kT), kT, 0, stream_>>>(q_rep_.p, nq_, qcell_.p, qtie_.p);
    TB_LAUNCHED("k_dedup_copy");
  }
  search_timed_ = true;
  return 0;
}

// Candidate cells of every query point (point qn[i] of xq, donor block
// qd[i]): stack-free traversal of the donor's tree into per-query slots and
// an overflow list, then one dense query-ordered list in cand_.  The FP32
// form of the tree is used unless the FP64 form is selected.
int Engine::traverse_and_gather(const double* xq, const int* qn, const int* qd, long long nq, unsigned& count,
                                int skip_uhex) {
  const int form = (precision_ == 0) ? 0 : 1;
  TB_CUDA(slots_.ensure((size_t)nq * kSlots));
  TB_CUDA(ncand_q_.ensure(nq + 1));
  TB_CUDA(cand_off_.ensure(nq + 1));
  TB_CUDA(scount_.ensure(2));
  TB_CUDA(cudaMemsetAsync(ncand_q_.p + nq, 0, sizeof(int), stream_));
  long long ovf_cap = std::max<long long>(cand_cap_, std::max<long long>(nq / 8, 1 << 16));
  unsigned novf = 0;
  count = 0;
  // traversal and the scan of the per-query counts, then one read-back of
  // the overflow count and the total; an overflow grows the list and repeats
  for (int attempt = 0; attempt < 2; attempt++) {
    TB_CUDA(ovf_.ensure(ovf_cap));
    TB_CUDA(cudaMemsetAsync(scount_.p, 0, sizeof(unsigned), stream_));
    launch_traverse(form, tune_.traverse_variant, grid_for(nq, 256, 148 * tune_.traverse_per_sm), stream_, xq,
                    d_bi_.p, cbox_.p,
                    form == 0 ? cbox64_.p : nullptr, tnode_.p, form == 0 ? tnode64_.p : nullptr, qn, qd, nq,
                    slots_.p, ncand_q_.p, ovf_.p, (int)ovf_cap, scount_.p, err_.p, skip_uhex);
    TB_LAUNCHED("k_traverse");
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, ncand_q_.p, cand_off_.p, (int)(nq + 1), stream_);
    TB_CUDA(cub_tmp_.ensure(tmp));
    cub::DeviceScan::ExclusiveSum(cub_tmp_.p, tmp, ncand_q_.p, cand_off_.p, (int)(nq + 1), stream_);
    TB_CUDA(cudaMemcpyAsync(&novf, scount_.p, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaMemcpyAsync(&count, cand_off_.p + nq, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaStreamSynchronize(stream_));
    cand_cap_ = ovf_cap;
    if ((long long)novf <= ovf_cap) break;
    ovf_cap = (long long)novf + novf / 4 + 1024;  // grow the overflow list and traverse again
  }
  TB_CUDA(cand_.ensure(std::max(1u, count)));
  if (count > 0) {
    k_gather_candidates<<<grid_for(nq, kT), kT, 0, stream_>>>(slots_.p, ncand_q_.p, cand_off_.p, nq, ovf_.p,
                                                              scount_.p, (int)ovf_cap, cand_.p);
    TB_LAUNCHED("k_gather_candidates");
  }
  // the overflow counter's word is reused by the refinement count
  TB_CUDA(cudaMemsetAsync(scount_.p + 1, 0, sizeof(unsigned), stream_));
  return 0;
}

// Coincident query points.  At preprocess: every node's OBB bin (the order in
// which the reference lists a receptor block's query points) and whether any
// block holds two nodes closer than the gate distance (a per-block grid of
// 2^18 cells per axis, distance a quarter cell, never below 10 TOL).  Blocks
// without such nodes cannot produce query points within TOL of each other,
// and the per-call merge is skipped.  Nodes farther apart than the gate
// distance at preprocess that later move within TOL of each other are not
// merged until the next preprocess.
int Engine::dedup_gate() {
  dedup_active_ = false;
  TB_CUDA(node_bin_.ensure(ntot_));
  k_node_bins<<<grid_for(ntot_, kT), kT, 0, stream_>>>(x_.p, node_blk_.p, d_bi_.p, ntot_, node_bin_.p);
  TB_LAUNCHED("k_node_bins");
  DBuf<int>& cnt = cg_cnt_;
  DBuf<int>& off = cg_off_;
  DBuf<int>& v0 = cg_v0_;
  DBuf<int>& v1 = cg_v1_;
  DBuf<unsigned long long>& k0 = cg_k0_;
  DBuf<unsigned long long>& k1 = cg_k1_;
  DBuf<unsigned>& flag = cg_flag_;
  TB_CUDA(cnt.ensure(ntot_ + 1));
  TB_CUDA(off.ensure(ntot_ + 1));
  k_coin_count<<<grid_for(ntot_, kT), kT, 0, stream_>>>(x_.p, node_blk_.p, d_bi_.p, ntot_, cnt.p);
  TB_LAUNCHED("k_coin_count");
  TB_CUDA(cudaMemsetAsync(cnt.p + ntot_, 0, sizeof(int), stream_));
  size_t tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt.p, off.p, (int)(ntot_ + 1), stream_);
  TB_CUDA(cub_tmp_.ensure(tmp));
  cub::DeviceScan::ExclusiveSum(cub_tmp_.p, tmp, cnt.p, off.p, (int)(ntot_ + 1), stream_);
  int total = 0;
  TB_CUDA(cudaMemcpyAsync(&total, off.p + ntot_, sizeof(int), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  if (total < 2) return 0;
  TB_CUDA(k0.ensure(total));
  TB_CUDA(k1.ensure(total));
  TB_CUDA(v0.ensure(total));
  TB_CUDA(v1.ensure(total));
  TB_CUDA(flag.ensure(1));
  TB_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(unsigned), stream_));
  k_coin_fill<<<grid_for(ntot_, kT), kT, 0, stream_>>>(x_.p, node_blk_.p, d_bi_.p, ntot_, off.p, k0.p, v0.p);
  TB_LAUNCHED("k_coin_fill");
  tmp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp, k0.p, k1.p, v0.p, v1.p, total, 0, 64, stream_);
  TB_CUDA(cub_tmp_.ensure(tmp));
  cub::DeviceRadixSort::SortPairs(cub_tmp_.p, tmp, k0.p, k1.p, v0.p, v1.p, total, 0, 64, stream_);
  k_coin_check<<<grid_for(total, kT), kT, 0, stream_>>>(k1.p, v1.p, total, x_.p, node_blk_.p, d_bi_.p, flag.p);
  TB_LAUNCHED("k_coin_check");
  unsigned f = 0;
  TB_CUDA(cudaMemcpyAsync(&f, flag.p, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  dedup_active_ = f != 0;
  return 0;
}

// The per-call merge (uniqNodesTree): donor-list order, octree subsets level
// by level, the pairwise loop per leaf, then xtag / representative / merged
// resolution per query.
int Engine::run_dedup() {
  // queries of pair p are [qoff[p], qoff[p+1])
  std::vector<int> h_toff(h_pair_t0_.back() + 1);
  TB_CUDA(cudaMemcpyAsync(h_toff.data(), tile_off_.p, h_toff.size() * sizeof(int), cudaMemcpyDeviceToHost,
                          stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  std::vector<int> qoff(npairs_ + 1);
  for (int p = 0; p < npairs_; p++) qoff[p] = h_toff[h_pair_t0_[p]];
  qoff[npairs_] = (int)nq_;
  DedupQueries Q{nq_, qnode_.p, qdon_.p, nullptr, nullptr, qres_.p, x_.p, node_blk_.p};
  TB_TRY(dedup_merge(Q, qoff));
  dedup_ran_ = true;
  return 0;
}

// The node-global-id merge (the TIOGA_HAS_NODEGID build's uniquenode_map,
// search.C:48-74) over the node queries: every donor's list in the
// reference's order (the same keys as the octree merge), then each (donor,
// node id) run's first entry represents the others and takes their largest
// resolution.  Every block needs its node ids.
int Engine::run_gid_merge() {
  const long long n = nq_;
  for (const HostBlock& H : hb_)
    if (!H.node_gid) {
      fprintf(stderr, "#tioga_b200: the node-id merge needs every block's node ids (tioga_b200_registernodegid_)\n");
      return -1;
    }
  TB_CUDA(node_gid_d_.ensure(ntot_));
  for (size_t b = 0; b < hb_.size(); b++)
    TB_CUDA(cudaMemcpyAsync(node_gid_d_.p + bi_[b].node_off, hb_[b].node_gid, hb_[b].nnodes * sizeof(uint64_t),
                            cudaMemcpyHostToDevice, stream_));
  std::vector<int> h_toff(h_pair_t0_.back() + 1);
  TB_CUDA(cudaMemcpyAsync(h_toff.data(), tile_off_.p, h_toff.size() * sizeof(int), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  std::vector<int> qoff(npairs_ + 1);
  for (int p = 0; p < npairs_; p++) qoff[p] = h_toff[h_pair_t0_[p]];
  qoff[npairs_] = (int)n;
  // the donors' lists in the reference's order: position i holds query refq[i]
  const int np = npairs_;
  std::vector<int> prank(np), seen(hb_.size(), 0);
  for (int p = 0; p < np; p++) prank[p] = seen[h_pairs_[p].don]++;
  TB_CUDA(dd_pqoff_.ensure(np + 1));
  TB_CUDA(dd_prank_.ensure(np));
  TB_CUDA(cudaMemcpyAsync(dd_pqoff_.p, qoff.data(), (np + 1) * sizeof(int), cudaMemcpyHostToDevice, stream_));
  TB_CUDA(cudaMemcpyAsync(dd_prank_.p, prank.data(), np * sizeof(int), cudaMemcpyHostToDevice, stream_));
  TB_CUDA(dd_key_.ensure(n));
  TB_CUDA(dd_key2_.ensure(n));
  TB_CUDA(dd_perm_.ensure(n));
  TB_CUDA(dd_refq_.ensure(n));
  TB_CUDA(dd_x_.ensure(3 * n));
  TB_CUDA(dd_mtag_.ensure(n));
  TB_CUDA(dd_rtag_.ensure(n));
  TB_CUDA(dd_itag_.ensure(n));
  TB_CUDA(q_gpos_.ensure(n));
  TB_CUDA(q_xt_.ensure(n));
  TB_CUDA(q_rep_.ensure(n));
  k_dedup_keys<<<grid_for(n, kT), kT, 0, stream_>>>(qnode_.p, qdon_.p, n, dd_pqoff_.p, np, dd_prank_.p, node_bin_.p,
                                                    dd_key_.p, dd_perm_.p);
  TB_LAUNCHED("k_dedup_keys");
  size_t tmp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp, dd_key_.p, dd_key2_.p, dd_perm_.p, dd_refq_.p, (int)n, 0, 64, stream_);
  TB_CUDA(cub_tmp_.ensure(tmp));
  cub::DeviceRadixSort::SortPairs(cub_tmp_.p, tmp, dd_key_.p, dd_key2_.p, dd_perm_.p, dd_refq_.p, (int)n, 0, 64,
                                  stream_);
  k_dedup_gather<<<grid_for(n, kT), kT, 0, stream_>>>(dd_refq_.p, n, qnode_.p, qres_.p, x_.p, node_blk_.p, nullptr,
                                                      d_bi_.p, dd_x_.p, dd_mtag_.p, dd_rtag_.p, dd_itag_.p,
                                                      dd_perm_.p, q_gpos_.p);
  TB_LAUNCHED("k_dedup_gather");
  // (donor, node id) runs in position order: stable sorts by id, then by donor
  TB_CUDA(gm_k0_.ensure(n));
  TB_CUDA(gm_k1_.ensure(n));
  TB_CUDA(gm_max_.ensure(n));
  TB_CUDA(gm_a_.ensure(n));
  TB_CUDA(gm_b_.ensure(n));
  TB_CUDA(gm_c_.ensure(n));
  TB_CUDA(gm_d_.ensure(n));
  k_gid_keys<<<grid_for(n, kT), kT, 0, stream_>>>(dd_refq_.p, n, qnode_.p, qdon_.p, node_gid_d_.p, gm_k0_.p,
                                                  gm_a_.p, gm_b_.p);  // id, donor, position (by position)
  TB_LAUNCHED("k_gid_keys");
  tmp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp, gm_k0_.p, gm_k1_.p, gm_b_.p, gm_c_.p, (int)n, 0, 64, stream_);
  TB_CUDA(cub_tmp_.ensure(tmp));
  cub::DeviceRadixSort::SortPairs(cub_tmp_.p, tmp, gm_k0_.p, gm_k1_.p, gm_b_.p, gm_c_.p, (int)n, 0, 64, stream_);
  k_gather_i32<<<grid_for(n, kT), kT, 0, stream_>>>(gm_a_.p, gm_c_.p, n, gm_d_.p);  // donors in id order
  TB_LAUNCHED("k_gather_i32");
  tmp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp, gm_d_.p, gm_b_.p, gm_c_.p, dd_perm_.p, (int)n, 0, 16, stream_);
  TB_CUDA(cub_tmp_.ensure(tmp));
  cub::DeviceRadixSort::SortPairs(cub_tmp_.p, tmp, gm_d_.p, gm_b_.p, gm_c_.p, dd_perm_.p, (int)n, 0, 16, stream_);
  // dd_perm_: positions sorted by (donor, id, position); ids and donors by position: gm_k0_ was sorted in
  // place into gm_k1_, so take the ids again
  k_gid_keys<<<grid_for(n, kT), kT, 0, stream_>>>(dd_refq_.p, n, qnode_.p, qdon_.p, node_gid_d_.p, gm_k0_.p,
                                                  gm_a_.p, gm_b_.p);
  TB_LAUNCHED("k_gid_keys");
  k_gid_heads<<<grid_for(n, kT), kT, 0, stream_>>>(dd_perm_.p, n, gm_k0_.p, gm_a_.p, gm_c_.p);
  TB_LAUNCHED("k_gid_heads");
  tmp = 0;
  cub::DeviceScan::InclusiveScan(nullptr, tmp, gm_c_.p, gm_d_.p, cub::Max(), (int)n, stream_);
  TB_CUDA(cub_tmp_.ensure(tmp));
  cub::DeviceScan::InclusiveScan(cub_tmp_.p, tmp, gm_c_.p, gm_d_.p, cub::Max(), (int)n, stream_);
  TB_CUDA(cudaMemsetAsync(gm_max_.p, 0, n * sizeof(unsigned long long), stream_));
  k_gid_apply<<<grid_for(n, kT), kT, 0, stream_>>>(dd_perm_.p, gm_d_.p, n, dd_itag_.p, dd_rtag_.p, gm_max_.p);
  TB_LAUNCHED("k_gid_apply");
  k_gid_res<<<grid_for(n, kT), kT, 0, stream_>>>(dd_itag_.p, n, gm_max_.p, dd_rtag_.p);
  TB_LAUNCHED("k_gid_res");
  k_dedup_apply<<<grid_for(n, kT), kT, 0, stream_>>>(dd_refq_.p, n, dd_itag_.p, dd_rtag_.p, qres_.p, q_xt_.p,
                                                     q_rep_.p, err_.p, counters_.p);
  TB_LAUNCHED("k_dedup_apply");
  TB_CUDA(cudaStreamSynchronize(stream_));  // host staging vectors go out of scope
  dedup_ran_ = true;
  return 0;
}

// The merge over any query list that is pair-major: node queries (keys from
// the OBB bins) or the high-order path's points (keys from the point order).
int Engine::dedup_merge(const DedupQueries& Qd, const std::vector<int>& qoff) {
  const long long n = Qd.n;
  const int np = npairs_;
  std::vector<int> prank(np);
  const int nb = (int)hb_.size();
  std::vector<long long> dcount(nb, 0);
  std::vector<int> seen(nb, 0);
  for (int p = 0; p < np; p++) {
    prank[p] = seen[h_pairs_[p].don]++;
    dcount[h_pairs_[p].don] += qoff[p + 1] - qoff[p];
  }
  TB_CUDA(dd_pqoff_.ensure(np + 1));
  TB_CUDA(dd_prank_.ensure(np));
  TB_CUDA(cudaMemcpyAsync(dd_pqoff_.p, qoff.data(), (np + 1) * sizeof(int), cudaMemcpyHostToDevice, stream_));
  TB_CUDA(cudaMemcpyAsync(dd_prank_.p, prank.data(), np * sizeof(int), cudaMemcpyHostToDevice, stream_));
  TB_CUDA(dd_key_.ensure(n));
  TB_CUDA(dd_key2_.ensure(n));
  TB_CUDA(dd_perm_.ensure(n));
  TB_CUDA(dd_perm2_.ensure(n));
  TB_CUDA(dd_refq_.ensure(n));
  TB_CUDA(dd_x_.ensure(3 * n));
  TB_CUDA(dd_mtag_.ensure(n));
  TB_CUDA(dd_rtag_.ensure(n));
  TB_CUDA(dd_itag_.ensure(n));
  TB_CUDA(dd_seg_.ensure(n));
  TB_CUDA(dd_oct_.ensure(n));
  TB_CUDA(q_gpos_.ensure(n));
  TB_CUDA(q_xt_.ensure(n));
  TB_CUDA(q_rep_.ensure(n));
  if (Qd.qpt_local) {
    k_dedup_keys_pts<<<grid_for(n, kT), kT, 0, stream_>>>(Qd.qpt_local, Qd.qdon, n, dd_pqoff_.p, np, dd_prank_.p,
                                                          dd_key_.p, dd_perm_.p);
    TB_LAUNCHED("k_dedup_keys_pts");
  } else {
    k_dedup_keys<<<grid_for(n, kT), kT, 0, stream_>>>(Qd.qid, Qd.qdon, n, dd_pqoff_.p, np, dd_prank_.p,
                                                      node_bin_.p, dd_key_.p, dd_perm_.p);
    TB_LAUNCHED("k_dedup_keys");
  }
  size_t tmp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp, dd_key_.p, dd_key2_.p, dd_perm_.p, dd_refq_.p, (int)n, 0, 64,
                                  stream_);
  TB_CUDA(cub_tmp_.ensure(tmp));
  cub::DeviceRadixSort::SortPairs(cub_tmp_.p, tmp, dd_key_.p, dd_key2_.p, dd_perm_.p, dd_refq_.p, (int)n, 0, 64,
                                  stream_);
  k_dedup_gather<<<grid_for(n, kT), kT, 0, stream_>>>(dd_refq_.p, n, Qd.qid, Qd.qres, Qd.coords, Qd.node_blk,
                                                      Qd.qrec, d_bi_.p, dd_x_.p, dd_mtag_.p, dd_rtag_.p, dd_itag_.p,
                                                      dd_perm_.p, q_gpos_.p);
  TB_LAUNCHED("k_dedup_gather");
  // subsets: (start, count, splits so far); the donors' lists to begin with
  struct Seg {
    int start, len, depth;
  };
  std::vector<Seg> segs, next;
  std::vector<int4> leaves;
  long long pos = 0;
  for (int d = 0; d < nb; d++) {
    if (dcount[d] > 0) segs.push_back(Seg{(int)pos, (int)dcount[d], 0});
    pos += dcount[d];
  }
  constexpr int kChunk = 4096;
  auto chunks_of = [&](const std::vector<Seg>& v, std::vector<int4>& ch, std::vector<int>& starts) {
    ch.clear();
    starts.clear();
    for (size_t a = 0; a < v.size(); a++) {
      starts.push_back(v[a].start);
      for (int c = 0; c < v[a].len; c += kChunk)
        ch.push_back(make_int4((int)a, v[a].start + c, std::min(kChunk, v[a].len - c), 0));
    }
  };
  std::vector<int4> ch;
  std::vector<int> starts;
  chunks_of(segs, ch, starts);
  if (!ch.empty()) {
    TB_CUDA(dd_chunks_.ensure(ch.size()));
    TB_CUDA(dd_starts_.ensure(starts.size()));
    TB_CUDA(cudaMemcpyAsync(dd_chunks_.p, ch.data(), ch.size() * sizeof(int4), cudaMemcpyHostToDevice, stream_));
    TB_CUDA(cudaMemcpyAsync(dd_starts_.p, starts.data(), starts.size() * sizeof(int), cudaMemcpyHostToDevice,
                            stream_));
    k_dedup_segfill<<<(unsigned)ch.size(), 256, 0, stream_>>>(dd_chunks_.p, dd_starts_.p, dd_seg_.p);
    TB_LAUNCHED("k_dedup_segfill");
  }
  for (int level = 0; level < 128 && !segs.empty(); level++) {
    std::vector<Seg> act;
    for (const Seg& g : segs) {
      if (g.len > kDedupLeaf) act.push_back(g);
      else leaves.push_back(make_int4(g.start, g.len, g.depth, 0));
    }
    if (act.empty()) break;
    chunks_of(act, ch, starts);
    const int na = (int)act.size();
    TB_CUDA(dd_chunks_.ensure(ch.size()));
    TB_CUDA(cudaMemcpyAsync(dd_chunks_.p, ch.data(), ch.size() * sizeof(int4), cudaMemcpyHostToDevice, stream_));
    std::vector<unsigned long long> box(6 * (size_t)na);
    for (int a = 0; a < na; a++)
      for (int k = 0; k < 3; k++) {
        box[6 * a + k] = ~0ull;
        box[6 * a + k + 3] = 0ull;
      }
    TB_CUDA(dd_box_.ensure(box.size()));
    TB_CUDA(cudaMemcpyAsync(dd_box_.p, box.data(), box.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice,
                            stream_));
    TB_CUDA(dd_cnt_.ensure(8 * (size_t)na));
    TB_CUDA(cudaMemsetAsync(dd_cnt_.p, 0, 8 * (size_t)na * sizeof(int), stream_));
    TB_CUDA(cudaMemsetAsync(dd_oct_.p, 0, n, stream_));
    k_dedup_box<<<(unsigned)ch.size(), 256, 0, stream_>>>(dd_chunks_.p, dd_perm_.p, dd_x_.p, dd_box_.p);
    TB_LAUNCHED("k_dedup_box");
    k_dedup_octant<<<(unsigned)ch.size(), 256, 0, stream_>>>(dd_chunks_.p, dd_perm_.p, dd_x_.p, dd_box_.p,
                                                             dd_oct_.p, dd_cnt_.p);
    TB_LAUNCHED("k_dedup_octant");
    std::vector<int> cnt(8 * (size_t)na);
    TB_CUDA(cudaMemcpyAsync(cnt.data(), dd_cnt_.p, cnt.size() * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaStreamSynchronize(stream_));
    next.clear();
    for (int a = 0; a < na; a++) {
      bool one = false;  // every point in one octant: compared as it is (icheck)
      for (int j = 0; j < 8; j++) one = one || cnt[8 * a + j] == act[a].len;
      if (one) {
        leaves.push_back(make_int4(act[a].start, act[a].len, act[a].depth, 0));
        continue;
      }
      int c = act[a].start;
      for (int j = 0; j < 8; j++) {
        const int m = cnt[8 * a + j];
        if (m > 0) next.push_back(Seg{c, m, act[a].depth + 1});
        c += m;
      }
    }
    // stable partition of every splitting subset by octant (the others have
    // one octant, or none, and keep their order)
    int bits = 3;
    while ((1ll << (bits - 3)) <= n) bits++;
    k_dedup_pkeys<<<grid_for(n, kT), kT, 0, stream_>>>(dd_seg_.p, dd_oct_.p, n, dd_key_.p);
    TB_LAUNCHED("k_dedup_pkeys");
    tmp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, dd_key_.p, dd_key2_.p, dd_perm_.p, dd_perm2_.p, (int)n, 0, bits,
                                    stream_);
    TB_CUDA(cub_tmp_.ensure(tmp));
    cub::DeviceRadixSort::SortPairs(cub_tmp_.p, tmp, dd_key_.p, dd_key2_.p, dd_perm_.p, dd_perm2_.p, (int)n, 0,
                                    bits, stream_);
    std::swap(dd_perm_, dd_perm2_);
    chunks_of(next, ch, starts);
    if (!ch.empty()) {
      TB_CUDA(dd_chunks_.ensure(ch.size()));
      TB_CUDA(dd_starts_.ensure(starts.size()));
      TB_CUDA(cudaMemcpyAsync(dd_chunks_.p, ch.data(), ch.size() * sizeof(int4), cudaMemcpyHostToDevice, stream_));
      TB_CUDA(cudaMemcpyAsync(dd_starts_.p, starts.data(), starts.size() * sizeof(int), cudaMemcpyHostToDevice,
                              stream_));
      k_dedup_segfill<<<(unsigned)ch.size(), 256, 0, stream_>>>(dd_chunks_.p, dd_starts_.p, dd_seg_.p);
      TB_LAUNCHED("k_dedup_segfill");
    }
    segs.swap(next);
    TB_CUDA(cudaStreamSynchronize(stream_));  // host tables are reused next level
  }
  for (const Seg& g : segs) leaves.push_back(make_int4(g.start, g.len, g.depth, 0));
  if (!leaves.empty()) {
    TB_CUDA(dd_leaves_.ensure(leaves.size()));
    TB_CUDA(cudaMemcpyAsync(dd_leaves_.p, leaves.data(), leaves.size() * sizeof(int4), cudaMemcpyHostToDevice,
                            stream_));
    k_dedup_leaves<<<grid_for((long long)leaves.size(), 128), 128, 0, stream_>>>(
        dd_leaves_.p, (int)leaves.size(), dd_perm_.p, dd_x_.p, dd_mtag_.p, dd_rtag_.p, dd_itag_.p);
    TB_LAUNCHED("k_dedup_leaves");
  }
  k_dedup_apply<<<grid_for(n, kT), kT, 0, stream_>>>(dd_refq_.p, n, dd_itag_.p, dd_rtag_.p, (double*)Qd.qres,
                                                     q_xt_.p, q_rep_.p, err_.p, counters_.p);
  TB_LAUNCHED("k_dedup_apply");
  TB_CUDA(cudaStreamSynchronize(stream_));  // host staging vectors go out of scope
  return 0;
}

// Per-node donor state at rest: iblank 1 (set by preprocess), no marks, no
// slots, every cell iblank 1.  Each call leaves it so (k_donor_reset at the
// start undoes the previous call's holes, receptors and layers).
int Engine::donor_rest_init() {
  TB_CUDA(mlist_.ensure(ntot_));
  TB_CUDA(cmlist_.ensure(ntot_));
  TB_CUDA(dcnt_.ensure(8));
  TB_CUDA(cudaMemsetAsync(dcnt_.p, 0, 8 * sizeof(int), stream_));
  TB_CUDA(cudaMemsetAsync(m0_.p, 0, ntot_, stream_));
  TB_CUDA(cudaMemsetAsync(m1_.p, 0, ntot_ * sizeof(int), stream_));
  TB_CUDA(cudaMemsetAsync(cmark_.p, 0, ntot_ * sizeof(int), stream_));
  TB_CUDA(cudaMemsetAsync(slot_.p, 0xff, (size_t)ntot_ * K_ * sizeof(int), stream_));
  k_fill_int<<<grid_for(ntot_, kT), kT, 0, stream_>>>(reset_t_.p, 0x7fffffff, ntot_);
  TB_LAUNCHED("k_fill_int");
  k_fill_int<<<grid_for(ctot_, kT), kT, 0, stream_>>>(iblank_cell_.p, 1, ctot_);
  TB_LAUNCHED("k_fill_int");
  prev_nrec_ = 0;
  donor_rest_ = true;
  return 0;
}

// Undo the previous call's holes, receptors and layers on the side stream
// (after the call's start on the main stream); nothing before the donor
// phase reads that state, and the donor phase waits for the side stream.
int Engine::donor_reset_begin() {
  if (!donor_rest_) TB_TRY(donor_rest_init());
  TB_CUDA(it_rec_.ensure(1));
  TB_CUDA(it_cancel_.ensure(1));
  TB_CUDA(cudaEventRecord(dr_ev_, stream_));
  TB_CUDA(cudaStreamWaitEvent(side_, dr_ev_, 0));
  k_donor_reset<<<148 * 16, kT, 0, side_>>>(mlist_.p, dcnt_.p, it_rec_.p, it_cancel_.p, prev_nrec_, csr_off_.p,
                                            csr_cell_.p, iblank_.p, m0_.p, m1_.p, iblank_cell_.p);
  TB_LAUNCHED_ON("k_donor_reset", side_);
  prev_nrec_ = 0;
  TB_CUDA(cudaMemsetAsync(dcnt_.p, 0, 8 * sizeof(int), side_));
  return 0;
}

int Engine::run_donors() {
  // candidate slots: one per (receptor node, donor block)
  if (nq_ > 0) {
    k_fill_slots<<<grid_for(nq_, kT), kT, 0, stream_>>>(qnode_.p, qdon_.p, qcell_.p, nq_, K_, ntot_, ctot_,
                                                        d_bi_.p, (int)hb_.size(), slot_.p, err_.p);
    TB_LAUNCHED("k_fill_slots");
    k_classify_queried<<<grid_for(nq_, kT), kT, 0, stream_>>>(x_.p, node_blk_.p, d_bi_.p, slot_.p, K_, qnode_.p,
                                                              qcell_.p, nq_, qres_.p, d_hmdev_.p, iblank_.p,
                                                              node_res_.p, m0_.p, m1_.p, mlist_.p, dcnt_.p,
                                                              counters_.p);
    TB_LAUNCHED("k_classify_queried");
  }
  if (nhm_ > 0 && h_tile_base_.back() > 0) {
    k_classify_tiles<<<(unsigned)h_tile_base_.back(), 256, 0, stream_>>>(
        x_.p, d_bi_.p, (int)hb_.size(), tile_base_.p, tbox_.p, node_order_.p, slot_.p, K_, d_hmdev_.p,
        iblank_.p, m0_.p, m1_.p, mlist_.p, dcnt_.p, counters_.p);
    TB_LAUNCHED("k_classify_tiles");
  }
  // nfringe layers around the holes, then the layers' nodes become mandatory
  k_front_init<<<1, 1, 0, stream_>>>(dcnt_.p);
  TB_LAUNCHED("k_front_init");
  int maxfr = 0;
  for (auto& B : bi_) maxfr = std::max(maxfr, B.nfringe);
  for (int it = 0; it < maxfr; it++) {
    k_dilate_front<<<148 * 16, kT, 0, stream_>>>(it, csr_off_.p, csr_cell_.p, conn8_.p, cell_nv_.p, cell_blk_.p,
                                                d_bi_.p, m0_.p, m1_.p, mlist_.p, dcnt_.p);
    TB_LAUNCHED("k_dilate_front");
    k_front_next<<<148 * 4, kT, 0, stream_>>>(it, m0_.p, mlist_.p, dcnt_.p);
    TB_LAUNCHED("k_front_next");
  }
  k_fringe_big_list<<<148 * 4, kT, 0, stream_>>>(mlist_.p, dcnt_.p, iblank_.p, node_res_.p);
  TB_LAUNCHED("k_fringe_big_list");
  // fringe choice -> records keyed (donor block, receptor node)
  TB_CUDA(rcount_.ensure(2));
  TB_CUDA(cudaMemsetAsync(rcount_.p, 0, 2 * sizeof(int), stream_));
  long long rcap = std::max<long long>(1, std::min<long long>(ntot_, nq_));
  if (test_rcap_ > 0) rcap = std::min<long long>(rcap, test_rcap_);  // tioga_b200_set_test_bound_
  TB_CUDA(rkey_.ensure(rcap));
  TB_CUDA(rkey_alt_.ensure(rcap));
  TB_CUDA(rval_.ensure(rcap));
  TB_CUDA(rval_alt_.ensure(rcap));
  int R = 0;
  if (nq_ > 0) {
    k_select<<<grid_for(nq_, kT), kT, 0, stream_>>>(node_blk_.p, d_bi_.p, slot_.p, K_, qnode_.p, qcell_.p, nq_,
                                                    cell_res_.p, iblank_.p, node_res_.p, rkey_alt_.p, rval_alt_.p,
                                                    rcount_.p, (int)rcap, err_.p);
    TB_LAUNCHED("k_select");
    TB_CUDA(cudaMemcpyAsync(&R, rcount_.p, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaStreamSynchronize(stream_));
  }
  if (R > rcap) {  // cannot happen: one record per receptor node at most
    fprintf(stderr, "#tioga_b200: donor records overflowed their capacity\n");
    R = (int)rcap;
    TB_CUDA(cudaMemcpyAsync(rcount_.p, &R, sizeof(int), cudaMemcpyHostToDevice, stream_));
  }
  nrec_ = R;
  if (R > 0) {
    size_t tmp = 0;
    int hi_bit = 32;  // receptor node below, donor block from bit 32
    while ((1ll << (hi_bit - 32)) < (long long)hb_.size()) hi_bit++;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, rkey_alt_.p, rkey_.p, rval_alt_.p, rval_.p, R, 0, hi_bit,
                                    stream_);
    TB_CUDA(cub_tmp_.ensure(tmp));
    cub::DeviceRadixSort::SortPairs(cub_tmp_.p, tmp, rkey_alt_.p, rkey_.p, rval_alt_.p, rval_.p, R, 0,
                                    hi_bit, stream_);
  }
  TB_CUDA(it_node_.ensure(9 * (size_t)std::max(R, 1)));
  TB_CUDA(it_w_.ensure(9 * (size_t)std::max(R, 1)));
  TB_CUDA(it_rec_.ensure(std::max(R, 1)));
  TB_CUDA(it_don_.ensure(std::max(R, 1)));
  TB_CUDA(it_nv_.ensure(std::max(R, 1)));
  TB_CUDA(it_cancel_.ensure(std::max(R, 1)));
  TB_CUDA(rres_.ensure(std::max(R, 1)));
  if (nq_ > 0) {
    k_fill_int<<<grid_for(nq_, kT), kT, 0, stream_>>>(interp2rec_.p, -1, nq_);
    TB_LAUNCHED("k_fill_int");
  }
  if (R > 0) {
    k_interp_marks<<<grid_for(R, kT), kT, 0, stream_>>>(rkey_.p, rval_.p, rcount_.p, qcell_.p, conn8_.p,
                                                         cell_nv_.p, iblank_.p, node_res_.p, cmark_.p,
                                                         reset_t_.p, cmlist_.p, dcnt_.p);
    TB_LAUNCHED("k_interp_marks");
    k_interp<<<grid_for(R, 128), 128, 0, stream_>>>(x_.p, rkey_.p, rval_.p, rcount_.p, qcell_.p, conn8_.p,
                                                     cell_nv_.p, node_blk_.p, d_bi_.p, iblank_.p, node_res_.p,
                                                     reset_t_.p, sorted_cell_.p, it_node_.p, it_w_.p, it_rec_.p,
                                                     it_don_.p,
                                                     it_nv_.p, it_cancel_.p, rres_.p, interp2rec_.p, err_.p);
    TB_LAUNCHED("k_interp");
    k_cancel<<<148 * 4, kT, 0, stream_>>>(cmlist_.p, dcnt_.p, slot_.p, K_, qcell_.p, cell_res_.p, interp2rec_.p,
                                           it_cancel_.p);
    TB_LAUNCHED("k_cancel");
    if (dedup_ran_) {  // resetCoincident
      TB_CUDA(dd_ireset_.ensure(nq_));
      k_fill_int<<<grid_for(nq_, kT), kT, 0, stream_>>>(dd_ireset_.p, 1, nq_);
      TB_LAUNCHED("k_fill_int");
      k_reset_coincident_min<<<grid_for(nq_, kT), kT, 0, stream_>>>(interp2rec_.p, q_xt_.p, nq_, it_cancel_.p,
                                                                    dd_ireset_.p);
      TB_LAUNCHED("k_reset_coincident_min");
      k_reset_coincident_set<<<grid_for(nq_, kT), kT, 0, stream_>>>(interp2rec_.p, q_xt_.p, nq_, dd_ireset_.p,
                                                                    it_cancel_.p);
      TB_LAUNCHED("k_reset_coincident_set");
    }
    k_iblank_final<<<grid_for(R, kT), kT, 0, stream_>>>(it_rec_.p, it_cancel_.p, rcount_.p, iblank_.p,
                                                        counters_.p);
    TB_LAUNCHED("k_iblank_final");
  }
  prev_nrec_ = R;
  return 0;
}

// tioga_writeoutputfiles_ -> tioga::writeData (tioga.C:526-531) ->
// MeshBlock::writeFlowFile (MeshBlock.C:510-635): one Tecplot FEPOINT file
// per block, flow%05d.dat by block index, with the same fields and formats
// (coordinates, iblank, mesh tag, the registered solution, bricks, wall and
// overset-boundary node lists), written from the caller's arrays.
int Engine::write_output(int nvar, int interptype) {
  if (!connected_) {
    fprintf(stderr, "#tioga_b200: writeoutputfiles needs performconnectivity first\n");
    return -1;
  }
  for (size_t ib = 0; ib < hb_.size(); ib++) {
    const HostBlock& H = hb_[ib];
    if (!H.hq && !H.dq) {
      fprintf(stderr, "#tioga_b200: writeoutputfiles: block %d has no registered solution\n", H.tag);
      return -1;
    }
    std::vector<int> ibl_h;
    const int* ibl = H.hibl;
    if (H.dibl) {
      ibl_h.resize(H.nnodes);
      TB_CUDA(cudaMemcpyAsync(ibl_h.data(), H.dibl, H.nnodes * sizeof(int), cudaMemcpyDeviceToHost, stream_));
      ibl = ibl_h.data();
    }
    std::vector<double> q_h;
    const double* q = H.hq;
    if (!q) {
      q_h.resize((size_t)H.nnodes * nvar);
      TB_CUDA(cudaMemcpyAsync(q_h.data(), H.dq, q_h.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_));
      q = q_h.data();
    }
    TB_CUDA(cudaStreamSynchronize(stream_));
    char intstring[16], fname[32];
    snprintf(intstring, sizeof(intstring), "%d", 100000 + (int)ib);
    snprintf(fname, sizeof(fname), "flow%s.dat", intstring + 1);
    FILE* fp = fopen(fname, "w");
    if (!fp) {
      fprintf(stderr, "#tioga_b200: writeoutputfiles: cannot open %s\n", fname);
      return -1;
    }
    fprintf(fp, "TITLE =\"Tioga output\"\n");
    fprintf(fp, "VARIABLES=\"X\",\"Y\",\"Z\",\"IBLANK\",\"BTAG\" ");
    for (int i = 0; i < nvar; i++) fprintf(fp, "\"Q%d\",", i);
    fprintf(fp, "\n");
    fprintf(fp, "ZONE T=\"VOL_MIXED\",N=%d E=%d ET=BRICK, F=FEPOINT\n", H.nnodes, H.ncells);
    for (int i = 0; i < H.nnodes; i++) {
      fprintf(fp, "%lf %lf %lf %d %d ", H.hx[3 * i], H.hx[3 * i + 1], H.hx[3 * i + 2], ibl[i], H.tag);
      for (int j = 0; j < nvar; j++)
        fprintf(fp, "%lf ", interptype == 0 ? q[(size_t)i * nvar + j] : q[(size_t)j * H.nnodes + i]);
      fprintf(fp, "\n");
    }
    // bricks: tets, pyramids and prisms with repeated corners (1-based as given)
    static const int kBrick[4][8] = {{0, 1, 2, 2, 3, 3, 3, 3},   // 4 vertices
                                     {0, 1, 2, 3, 4, 4, 4, 4},   // 5
                                     {0, 1, 2, 2, 3, 4, 5, 5},   // 6
                                     {0, 1, 2, 3, 4, 5, 6, 7}};  // 8
    for (int n = 0; n < H.ntypes; n++) {
      const int nvert = H.nv[n];
      const int* pat = kBrick[nvert == 4 ? 0 : nvert == 5 ? 1 : nvert == 6 ? 2 : 3];
      const int* cv = H.hconn[n];
      for (int i = 0; i < H.nc[n]; i++) {
        const int* c = cv + (size_t)nvert * i;
        fprintf(fp, "%d %d %d %d %d %d %d %d\n", c[pat[0]], c[pat[1]], c[pat[2]], c[pat[3]], c[pat[4]], c[pat[5]],
                c[pat[6]], c[pat[7]]);
      }
    }
    fprintf(fp, "%d\n", H.nwbc);
    for (int i = 0; i < H.nwbc; i++) fprintf(fp, "%d\n", H.hwbc[i]);
    fprintf(fp, "%d\n", H.nobc);
    for (int i = 0; i < H.nobc; i++) fprintf(fp, "%d\n", H.hobc[i]);
    fclose(fp);
  }
  return 0;
}

// tioga_reduce_fringes_ (tioga.C:737-885): on the last connectivity call's
// results; the cell iblanks are left as that call computed them, as the
// reference does
int Engine::reduce_fringes() {
  if (!connected_) {
    fprintf(stderr, "#tioga_b200: reduce_fringes needs performconnectivity first\n");
    return -1;
  }
  TB_CUDA(rf_red_.ensure(std::max(1ll, ntot_)));
  TB_CUDA(rf_tmp_.ensure(std::max(1ll, ntot_)));
  TB_CUDA(rf_was_.ensure(std::max(1ll, nrec_)));
  k_rf_init<<<grid_for(std::max(1ll, ntot_), kT), kT, 0, stream_>>>(iblank_.p, ntot_, rf_red_.p, rf_tmp_.p);
  TB_LAUNCHED("k_rf_init");
  TB_CUDA(cudaMemsetAsync(counters_.p, 0, 16 * sizeof(unsigned long long), stream_));
  if (nrec_ > 0) {
    int layers = 0;
    for (const BlockInfo& B : bi_) layers = std::max(layers, B.nfringe + 1);
    for (int it = 0; it < layers; it++) {
      k_rf_layer<<<148 * 16, kT, 0, stream_>>>(it, it_rec_.p, it_cancel_.p, rcount_.p, csr_off_.p, csr_cell_.p,
                                               conn8_.p, cell_nv_.p, cell_blk_.p, d_bi_.p, iblank_.p, rf_red_.p,
                                               rf_tmp_.p);
      TB_LAUNCHED("k_rf_layer");
      k_rf_copy<<<grid_for(nrec_, kT), kT, 0, stream_>>>(it_rec_.p, it_cancel_.p, rcount_.p, rf_tmp_.p, rf_red_.p);
      TB_LAUNCHED("k_rf_copy");
    }
    k_rf_cancel<<<grid_for(nrec_, kT), kT, 0, stream_>>>(it_rec_.p, rcount_.p, rf_red_.p, it_cancel_.p, rf_was_.p);
    TB_LAUNCHED("k_rf_cancel");
    if (dedup_ran_) {  // resetCoincident (bookKeeping.C:572-597) again
      k_fill_int<<<grid_for(nq_, kT), kT, 0, stream_>>>(dd_ireset_.p, 1, nq_);
      TB_LAUNCHED("k_fill_int");
      k_reset_coincident_min<<<grid_for(nq_, kT), kT, 0, stream_>>>(interp2rec_.p, q_xt_.p, nq_, it_cancel_.p,
                                                                    dd_ireset_.p);
      TB_LAUNCHED("k_reset_coincident_min");
      k_reset_coincident_set<<<grid_for(nq_, kT), kT, 0, stream_>>>(interp2rec_.p, q_xt_.p, nq_, dd_ireset_.p,
                                                                    it_cancel_.p);
      TB_LAUNCHED("k_reset_coincident_set");
    }
    k_rf_iblank<<<grid_for(nrec_, kT), kT, 0, stream_>>>(it_rec_.p, it_cancel_.p, rf_was_.p, rcount_.p, rf_red_.p,
                                                         iblank_.p, counters_.p);
    TB_LAUNCHED("k_rf_iblank");
  }
  TB_TRY(download_iblank());
  unsigned long long cnt[16];
  TB_CUDA(cudaMemcpyAsync(cnt, counters_.p, sizeof(cnt), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  stats_.nreceptor = (long long)cnt[5];
  stats_.nhole += (long long)cnt[4];
  interps_fetched_ = false;
  return 0;
}

int Engine::run_celliblank() {
  // cells around the holes and the final receptors (all others are 1), then
  // the donor slots and cancel marks back to rest, on the side stream while
  // the main stream copies the node iblanks out; download_iblank waits for
  // them before it copies the cell iblanks
  TB_CUDA(cudaEventRecord(cib_ev_[0], stream_));
  TB_CUDA(cudaStreamWaitEvent(side_, cib_ev_[0], 0));
  k_cell_iblank_sparse<<<148 * 16, kT, 0, side_>>>(mlist_.p, dcnt_.p, it_rec_.p, it_cancel_.p, rcount_.p,
                                                  csr_off_.p, csr_cell_.p, conn8_.p, cell_nv_.p, iblank_.p,
                                                  iblank_cell_.p);
  TB_LAUNCHED_ON("k_cell_iblank_sparse", side_);
  // back to rest for the next call: slots, cancel marks
  k_donor_clear<<<grid_for(std::max<long long>(nq_, 1), kT), kT, 0, side_>>>(
      qnode_.p, qdon_.p, qcell_.p, nq_, K_, d_bi_.p, slot_.p, cmlist_.p, dcnt_.p, cmark_.p, reset_t_.p);
  TB_LAUNCHED_ON("k_donor_clear", side_);
  TB_CUDA(cudaEventRecord(cib_ev_[1], side_));
  return 0;
}

int Engine::download_iblank() {
  for (size_t b = 0; b < hb_.size(); b++) {
    if (hb_[b].dibl)
      TB_CUDA(cudaMemcpyAsync(hb_[b].dibl, iblank_.p + bi_[b].node_off, hb_[b].nnodes * sizeof(int),
                              cudaMemcpyDeviceToDevice, stream_));
    else
      TB_CUDA(cudaMemcpyAsync(hb_[b].hibl, iblank_.p + bi_[b].node_off, hb_[b].nnodes * sizeof(int),
                              cudaMemcpyDeviceToHost, stream_));
  }
  TB_CUDA(cudaStreamWaitEvent(stream_, cib_ev_[1], 0));  // the cell iblanks (run_celliblank, side stream)
  for (size_t b = 0; b < hb_.size(); b++) {
    if (hb_[b].h_iblank_cell) {
      TB_CUDA(cell_stage_.ensure(hb_[b].ncells));
      k_gather_cells_i32<<<grid_for(hb_[b].ncells, kT), kT, 0, stream_>>>(iblank_cell_.p, inv_sorted_.p,
                                                                          bi_[b].cell_off, hb_[b].ncells,
                                                                          cell_stage_.p);
      TB_LAUNCHED("k_gather_cells_i32");
      TB_CUDA(cudaMemcpyAsync(hb_[b].h_iblank_cell, cell_stage_.p, hb_[b].ncells * sizeof(int),
                              cudaMemcpyDeviceToHost, stream_));
      TB_CUDA(cudaStreamSynchronize(stream_));  // the staging buffer is reused
    }
  }
  return 0;
}

int Engine::autotune(int reps) {
  if (!preprocessed_) {
    fprintf(stderr, "#tioga_b200: autotune needs preprocess_grids first\n");
    return -1;
  }
  struct Knob {
    int* v;
    std::vector<int> cand;
    float Timing::*phase;
  };
  const Knob knobs[] = {
      {&tune_.cell_pass_per_sm, {2, 3, 4}, &Timing::cell_pass},
      {&tune_.chunk_pairs, {32, 64, 128}, &Timing::cell_pass},
      {&tune_.query_per_sm, {4, 8, 16, 32, 64}, &Timing::query},
      {&tune_.cell_box_per_sm, {4, 6, 8}, &Timing::cell_boxes},
      {&tune_.traverse_variant, {0, 1}, &Timing::traverse},
      {&tune_.traverse_per_sm, {16, 32, 64, 128}, &Timing::traverse},
      {&tune_.candidates_per_sm, {8, 16, 32, 64}, &Timing::candidates},
  };
  reps = std::max(1, reps);
  // Shapes are timed on device-resident coordinates (a first call uploads
  // them): with an upload every call, the split form makes its cell boxes
  // inside the chunked upload, where the box kernel's shape is not timed.
  struct Restore {
    int& flag;
    int value;
    ~Restore() { flag = value; }
  } restore{coords_resident_, coords_resident_};
  coords_resident_ = 1;
  TB_TRY(connectivity());
  for (const Knob& k : knobs) {
    int best = *k.v;
    float tbest = 1e30f;
    for (int c : k.cand) {
      *k.v = c;
      float t = 1e30f;
      for (int r = 0; r < reps; r++) {
        TB_TRY(connectivity());
        t = std::min(t, timing_.*k.phase);
      }
      if (t < tbest) {
        tbest = t;
        best = c;
      }
    }
    *k.v = best;
  }
  return connectivity();  // leave the instance with results of the chosen shapes
}

int Engine::connectivity() {
  if (!preprocessed_) {
    fprintf(stderr, "#tioga_b200: performconnectivity called before preprocess_grids\n");
    return -1;
  }
  stats_ = Stats{};
  nlaunch_ = 0;
  search_timed_ = false;
  cell_timed_ = false;
  interps_fetched_ = false;
  TB_CUDA(cudaEventRecord(ev_[0], stream_));
  TB_CUDA(cudaMemsetAsync(counters_.p, 0, 16 * sizeof(unsigned long long), stream_));
  TB_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(unsigned), stream_));  // this call's device errors only
  // the side stream is idle unless the last call stopped early (its pinned
  // staging is reused below); then the previous call's donor marks go back
  // to rest on it, beside everything up to the donor phase
  TB_CUDA(cudaStreamSynchronize(side_));
  TB_TRY(donor_reset_begin());
  boxes_ready_ = false;
  tiles_ready_ = false;
  if (!coords_resident_ || !coords_on_device_) {
    if (precision_ != 0 && nleaf_total_ > 0 && h_up_leaf_off_.size() > 1) TB_TRY(upload_chunked());
    else TB_TRY(upload_coords());
  }
  TB_CUDA(cudaEventRecord(ev_[1], stream_));
  // The hole maps run on the side stream after the cell boxes (hev_[0],
  // recorded again after the box kernel), beside the latency-bound pair,
  // query and search kernels; the donor phase waits for them.
  TB_CUDA(cudaEventRecord(hev_[0], stream_));
  TB_CUDA(cudaEventRecord(ev_[2], stream_));
  int rc = run_pairs_and_refit();
  if (rc) return rc;
  rc = holemaps_begin();
  if (rc) return rc;
  rc = holemaps_end();
  if (rc) return rc;
  TB_CUDA(cudaEventRecord(ev_[3], stream_));
  nq_ = 0;
  nrec_ = 0;
  if (npairs_ > 0) {
    rc = run_queries();
    if (rc) return rc;
    TB_CUDA(cudaEventRecord(ev_[4], stream_));
    TB_CUDA(cudaStreamWaitEvent(stream_, rf_ev_, 0));  // the refitted tree
    rc = run_search();
    if (rc) return rc;
  } else {
    TB_CUDA(cudaEventRecord(ev_[4], stream_));
  }
  TB_CUDA(cudaEventRecord(ev_[5], stream_));
  TB_CUDA(cudaStreamWaitEvent(stream_, hev_[2], 0));
  rc = run_donors();
  if (rc) return rc;
  TB_CUDA(cudaEventRecord(ev_[6], stream_));
  rc = run_celliblank();
  if (rc) return rc;
  TB_CUDA(cudaEventRecord(ev_[7], stream_));
  TB_TRY(download_iblank());
  TB_CUDA(cudaEventRecord(ev_[8], stream_));
  unsigned long long cnt[16];
  unsigned err = 0;
  TB_CUDA(cudaMemcpyAsync(cnt, counters_.p, sizeof(cnt), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaMemcpyAsync(&err, err_.p, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
  unsigned sc[2] = {0, 0};
  if (npairs_ > 0) TB_CUDA(cudaMemcpyAsync(sc, scount_.p, sizeof(sc), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  stats_.nquery = nq_;
  stats_.ncand = (long long)cnt[0];
  stats_.nrefine = (long long)sc[1];
  stats_.nties = (long long)cnt[2];
  stats_.ndonor = (long long)cnt[3];
  stats_.nhole = (long long)cnt[4];
  stats_.nreceptor = (long long)cnt[5];
  stats_.nrecords = nrec_;
  stats_.nleaf = nleaf_total_;
  stats_.nmerged = (long long)cnt[7];
  stats_.npairs = npairs_;
  stats_.launches = nlaunch_;
  stats_.cand_verts = (long long)cnt[6];
  stats_.error = err;
  float ms[9];
  for (int i = 1; i < 9; i++) cudaEventElapsedTime(&ms[i], ev_[i - 1], ev_[i]);
  timing_.upload = ms[1];
  timing_.holemap = 0;  // on the side stream, beside the cell pass and the search
  cudaEventElapsedTime(&timing_.holemap, hev_[0], hev_[2]);
  timing_.boxes = ms[3];
  timing_.query = ms[4];
  timing_.search = ms[5];
  timing_.donors = ms[6];
  timing_.celliblank = 0;  // on the side stream, beside the node iblanks' copies
  cudaEventElapsedTime(&timing_.celliblank, cib_ev_[0], cib_ev_[1]);
  timing_.download = ms[8];
  cudaEventElapsedTime(&timing_.total, ev_[0], ev_[8]);
  timing_.traverse = timing_.candidates = timing_.refine = 0;
  timing_.cell_pass = 0;
  timing_.cell_boxes = 0;
  if (cell_timed_) {
    cudaEventElapsedTime(&timing_.cell_pass, cev_[0], cev_[1]);
    cudaEventElapsedTime(&timing_.cell_boxes, cev_[0], cev_[2]);
  }
  if (search_timed_) {
    cudaEventElapsedTime(&timing_.traverse, sev_[0], sev_[1]);
    cudaEventElapsedTime(&timing_.candidates, sev_[1], sev_[2]);
    cudaEventElapsedTime(&timing_.refine, sev_[2], sev_[3]);
  }
  if (err & kErrWeightRange)
    fprintf(stderr, "#tioga_b200: an interpolation weight fell outside [-0.2,1.2] (the reference aborts)\n");
  if (err & kErrFloodFillBound) fprintf(stderr, "#tioga_b200: hole-map fill hit its round limit\n");
  if (err & kErrCapacity) fprintf(stderr, "#tioga_b200: donor records overflowed their capacity\n");
  if (err & kErrTraversalOverflow) fprintf(stderr, "#tioga_b200: a tree walk went deeper than its stack\n");
  if (err & kErrBadIndex) fprintf(stderr, "#tioga_b200: an index fell outside its array and was skipped\n");
  connected_ = true;
  ihigh_global_ = ihigh_;  // tioga.C:138
  ho_done_ = false;
  // a device bound that ran out or a weight the reference would abort on:
  // the call completes, its error bits go to tioga_b200_last_error()
  return (int)(err & kErrFatal);
}

// ---------------------------------------------------------------------------
// queries on the interpolation lists (dataUpdate.C:121-159)
// ---------------------------------------------------------------------------
int Engine::fetch_interps() {
  if (interps_fetched_) return 0;
  const long long R = nrec_;
  h_it_node_.resize(9 * R);
  h_it_w_.resize(9 * R);
  h_it_rec_.resize(R);
  h_it_don_.resize(R);
  h_it_nv_.resize(R);
  h_it_cancel_.resize(R);
  if (R > 0) {
    TB_CUDA(cudaMemcpyAsync(h_it_node_.data(), it_node_.p, 9 * R * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaMemcpyAsync(h_it_w_.data(), it_w_.p, 9 * R * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaMemcpyAsync(h_it_rec_.data(), it_rec_.p, R * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaMemcpyAsync(h_it_don_.data(), it_don_.p, R * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaMemcpyAsync(h_it_nv_.data(), it_nv_.p, R, cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaMemcpyAsync(h_it_cancel_.data(), it_cancel_.p, R, cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaStreamSynchronize(stream_));
  }
  interps_fetched_ = true;
  return 0;
}

int Engine::donor_count(int tag, int* dcount, int* fcount) {
  *dcount = *fcount = 0;
  if (!connected_ || npairs_ == 0) return 0;
  int ib = find_tag(tag);
  if (ib < 0) return -1;
  int rc = fetch_interps();
  if (rc) return rc;
  for (long long r = 0; r < nrec_; r++)
    if (h_it_don_[r] == ib && !h_it_cancel_[r]) {
      (*dcount)++;
      (*fcount) += h_it_nv_[r] + 1;
    }
  return 0;
}

int Engine::donor_info(int tag, int* receptors, int* indices, double* frac) {
  if (!connected_ || npairs_ == 0) return 0;
  int ib = find_tag(tag);
  if (ib < 0) return -1;
  int rc = fetch_interps();
  if (rc) return rc;
  std::vector<int> first(bi_.size());
  for (size_t b = 0; b < bi_.size(); b++) first[b] = bi_[b].node_off;
  long long j = 0, k = 0;
  for (long long r = 0; r < nrec_; r++) {
    if (h_it_don_[r] != ib || h_it_cancel_[r]) continue;
    const int nv = h_it_nv_[r];
    for (int m = 0; m < nv + 1; m++) {
      indices[j] = h_it_node_[9 * r + m];
      frac[j] = h_it_w_[9 * r + m];
      j++;
    }
    const int g = h_it_rec_[r];
    const int rb = (int)(std::upper_bound(first.begin(), first.end(), g) - first.begin()) - 1;
    receptors[k++] = 0;  // rank of the receptor: the only one
    receptors[k++] = g - bi_[rb].node_off;
    receptors[k++] = rb - bi_[rb].sblk0;  // the receptor block's index within its system
    receptors[k++] = nv;
  }
  return 0;
}

int Engine::set_node_gid(int tag, const uint64_t* gid) {
  int ib = find_tag(tag);
  if (ib < 0) return -1;
  hb_[ib].node_gid = gid;
  return 0;
}

int Engine::set_uniform_hex_flag(int tag, int flag) {
  int ib = find_tag(tag);
  if (ib < 0) return -1;
  hb_[ib].uniform_flag = flag;
  return 0;
}

// The uniform-hex set-up of every flagged block (MeshBlock::preprocess,
// MeshBlock.C:84-87): check_for_uniform_hex (MeshBlock.C:1249-1372) and
// create_hex_cell_map (:1374-1409).  The first hex's squared edge lengths
// and the last hex's edges (the reference's loop leaves them in dx and xv)
// are read from the caller's arrays; every hex is checked on the device.
// Deviation: a flagged block that is no longer uniform at a later preprocess
// goes back to its tree (the reference keeps its stale map).
int Engine::setup_uniform_hex() {
  bool any_flag = false;
  for (const HostBlock& H : hb_) any_flag = any_flag || H.uniform_flag;
  if (!any_flag && !any_uhex_) return 0;
  any_uhex_ = false;
  long long map_total = 0;
  TB_CUDA(uhex_red_.ensure(8));
  unsigned* bad = reinterpret_cast<unsigned*>(uhex_red_.p + 6);
  for (size_t b = 0; b < hb_.size(); b++) {
    HostBlock& H = hb_[b];
    BlockInfo& B = bi_[b];
    B.uhex = 0;
    H.uniform = 0;
    if (!H.uniform_flag || H.ntypes != 1 || H.nv[0] != 8 || H.nc[0] < 1) continue;
    double first[8][3], last[8][3];
    const int* c0 = H.hconn[0];
    const int* cl = H.hconn[0] + 8 * (long long)(H.nc[0] - 1);
    for (int m = 0; m < 8; m++)
      for (int k = 0; k < 3; k++) {
        first[m][k] = H.hx[3 * (long long)(c0[m] - 1) + k];
        last[m][k] = H.hx[3 * (long long)(cl[m] - 1) + k];
      }
    auto tdot = [](const double* a, const double* p, const double* c) {
      double dp = 0.0;
      for (int k = 0; k < 3; k++) dp += ((a[k] - c[k]) * (p[k] - c[k]));
      return dp;
    };
    double d[3] = {tdot(first[1], first[1], first[0]), tdot(first[3], first[3], first[0]),
                   tdot(first[4], first[4], first[0])};
    TB_CUDA(cudaMemsetAsync(bad, 0, sizeof(unsigned), stream_));
    k_uhex_check<<<grid_for(H.ncells, kT), kT, 0, stream_>>>(x_.p, conn8_.p, d_bi_.p, (int)b, d[0], d[1], d[2],
                                                             bad);
    TB_LAUNCHED("k_uhex_check");
    unsigned h_bad = 0;
    TB_CUDA(cudaMemcpyAsync(&h_bad, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaStreamSynchronize(stream_));
    if (h_bad) continue;
    double dx[3], vec[3][3];
    for (int j = 0; j < 3; j++) dx[j] = sqrt(d[j]);
    for (int k = 0; k < 3; k++) vec[0][k] = (last[1][k] - last[0][k]) / dx[0];
    for (int k = 0; k < 3; k++) vec[1][k] = (last[3][k] - last[0][k]) / dx[1];
    for (int k = 0; k < 3; k++) vec[2][k] = (last[4][k] - last[0][k]) / dx[2];
    unsigned long long init[6] = {~0ull, ~0ull, ~0ull, 0ull, 0ull, 0ull};
    TB_CUDA(cudaMemcpyAsync(uhex_red_.p, init, sizeof(init), cudaMemcpyHostToDevice, stream_));
    UhexAxes A;
    memcpy(A.vec, vec, sizeof(vec));
    k_uhex_extent<<<grid_for(H.nnodes, kT), kT, 0, stream_>>>(x_.p, B.node_off, H.nnodes, A, uhex_red_.p);
    TB_LAUNCHED("k_uhex_extent");
    unsigned long long red[6];
    TB_CUDA(cudaMemcpyAsync(red, uhex_red_.p, sizeof(red), cudaMemcpyDeviceToHost, stream_));
    TB_CUDA(cudaStreamSynchronize(stream_));
    double xmin[3], xmax[3], dxc[3], xd[3], xc[3];
    for (int j = 0; j < 3; j++) {
      xmin[j] = dkey_inv(red[j]) - kTol;
      xmax[j] = dkey_inv(red[j + 3]) + kTol;
      dxc[j] = (xmax[j] - xmin[j]) * 0.5;
      xd[j] = (xmax[j] + xmin[j]) * 0.5;
    }
    for (int j = 0; j < 3; j++) {
      xc[j] = 0.0;
      for (int k = 0; k < 3; k++) xc[j] += (xd[k] * vec[k][j]);
    }
    long long nmap = 1;
    bool ok = true;
    for (int j = 0; j < 3; j++) {
      B.uxlow[j] = xc[j];
      for (int k = 0; k < 3; k++) B.uxlow[j] -= (dxc[k] * vec[k][j]);
      const double r = round(2 * dxc[j] / dx[j]);
      ok = ok && r >= 1 && r < 2147483647.0;
      B.uidims[j] = ok ? (int)r : 1;
      B.udx[j] = (2 * dxc[j]) / B.uidims[j];
      nmap *= B.uidims[j];
      for (int k = 0; k < 3; k++) B.uvec[j][k] = vec[j][k];
    }
    if (!ok || nmap > 4ll * H.ncells + 1024) {  // not the box of its own cells: keep the tree
      fprintf(stderr, "#tioga_b200: block %d passed the uniform-hex test but its cell map does not fit\n",
              H.tag);
      continue;
    }
    B.uhex = 1;
    H.uniform = 1;
    B.umap_off = map_total;
    map_total += nmap;
    any_uhex_ = true;
  }
  TB_CUDA(cudaMemcpyAsync(d_bi_.p, bi_.data(), bi_.size() * sizeof(BlockInfo), cudaMemcpyHostToDevice, stream_));
  if (any_uhex_) {
    TB_CUDA(uhex_map_.ensure(map_total));
    TB_CUDA(cudaMemsetAsync(uhex_map_.p, 0xff, map_total * sizeof(int), stream_));
    for (size_t b = 0; b < hb_.size(); b++)
      if (bi_[b].uhex) {
        k_uhex_map<<<grid_for(hb_[b].ncells, kT), kT, 0, stream_>>>(x_.p, conn8_.p, sorted_cell_.p, d_bi_.p,
                                                                    (int)b, uhex_map_.p);
        TB_LAUNCHED("k_uhex_map");
      }
  }
  TB_CUDA(cudaStreamSynchronize(stream_));  // the host block table goes on changing
  return 0;
}

int Engine::set_cell_gid(int tag, const uint64_t* gid) {
  int ib = find_tag(tag);
  if (ib < 0) return -1;
  hb_[ib].cell_gid = gid;
  return 0;
}

// tioga::getReceptorInfo (src/tioga.C:572-671) on one rank: the donor blocks
// in registration order, each block's live records in list order
// (MeshBlock::getReceptorInfo, src/dataUpdate.C:161-178), every record as
// (receptor node, mesh tag of the receptor block, the donor cell's global id
// as two ints: its eight bytes copied, low word first on a little-endian host).
long long Engine::receptor_info(int* out, long long cap) {
  if (!connected_ || npairs_ == 0) return 0;
  if (fetch_interps()) return -1;
  std::vector<int> first(bi_.size());
  for (size_t b = 0; b < bi_.size(); b++) first[b] = bi_[b].node_off;
  long long k = 0;
  for (int ib = 0; ib < (int)hb_.size(); ib++) {
    if (hb_[ib].sys != cur_sys_) continue;
    for (long long r = 0; r < nrec_; r++) {
      if (h_it_don_[r] != ib || h_it_cancel_[r]) continue;
      if (!hb_[ib].cell_gid) {  // the reference reads through a null pointer here
        fprintf(stderr, "#tioga_b200: block %d donates but has no cell global ids\n", hb_[ib].tag);
        return -1;
      }
      const int g = h_it_rec_[r];
      const int rb = (int)(std::upper_bound(first.begin(), first.end(), g) - first.begin()) - 1;
      const uint64_t gid = hb_[ib].cell_gid[h_it_node_[9 * r + h_it_nv_[r]]];
      int v[4] = {g - bi_[rb].node_off, hb_[rb].tag, 0, 0};
      std::memcpy(&v[2], &gid, sizeof(gid));
      for (int m = 0; m < 4; m++, k++)
        if (out && k < cap) out[k] = v[m];
    }
  }
  return k;
}

int Engine::cell_iblank(int tag, int* out) {
  int ib = find_tag(tag);
  if (ib < 0 || !connected_) return -1;
  TB_CUDA(cell_stage_.ensure(bi_[ib].ncells));
  k_gather_cells_i32<<<grid_for(bi_[ib].ncells, kT), kT, 0, stream_>>>(iblank_cell_.p, inv_sorted_.p,
                                                                       bi_[ib].cell_off, bi_[ib].ncells,
                                                                       cell_stage_.p);
  TB_LAUNCHED("k_gather_cells_i32");
  TB_CUDA(cudaMemcpyAsync(out, cell_stage_.p, bi_[ib].ncells * sizeof(int), cudaMemcpyDeviceToHost, stream_));
  TB_CUDA(cudaStreamSynchronize(stream_));
  return 0;
}

// ---------------------------------------------------------------------------
// data update (src/tioga.C:336-524)
// ---------------------------------------------------------------------------
int Engine::dataupdate(int nvar, int interptype) {
  if (!connected_) return -1;
  bool device = true, host = true;
  for (auto& H : hb_) {
    if (!H.hq && !H.dq) {
      printf("Solution data not set, cannot update \n");
      return 0;
    }
    device = device && H.dq;
    host = host && H.hq;
  }
  if (npairs_ == 0 || nrec_ == 0) return 0;
  if (!device && !host) {
    fprintf(stderr, "#tioga_b200: register every block's solution on the same side (host or device)\n");
    return -1;
  }
  TB_CUDA(qvals_.ensure((size_t)nrec_ * nvar));
  // every block's solution on the device: the caller's own arrays (device
  // solutions, read and written in place), or one upload of the host arrays
  std::vector<double*> qptr(hb_.size());
  if (host) {
    TB_CUDA(q_.ensure((size_t)ntot_ * nvar));
    for (size_t b = 0; b < hb_.size(); b++) {
      qptr[b] = q_.p + (size_t)bi_[b].node_off * nvar;
      TB_CUDA(cudaMemcpyAsync(qptr[b], hb_[b].hq, (size_t)hb_[b].nnodes * nvar * sizeof(double),
                              cudaMemcpyHostToDevice, stream_));
    }
  } else {
    for (size_t b = 0; b < hb_.size(); b++) qptr[b] = hb_[b].dq;
  }
  TB_CUDA(d_qptr_.ensure(hb_.size()));
  TB_CUDA(cudaMemcpyAsync(d_qptr_.p, qptr.data(), qptr.size() * sizeof(double*), cudaMemcpyHostToDevice, stream_));
  k_interp_gather<<<grid_for(nrec_, 128), 128, 0, stream_>>>(it_node_.p, it_w_.p, it_don_.p, it_nv_.p,
                                                              it_cancel_.p, rcount_.p, d_bi_.p, d_qptr_.p, nvar,
                                                              interptype, qvals_.p);
  TB_LAUNCHED("k_interp_gather");
  if (host) {
    int rc = fetch_interps();
    if (rc) return rc;
    std::vector<double> vals((size_t)nrec_ * nvar);
    TB_CUDA(cudaMemcpyAsync(vals.data(), qvals_.p, vals.size() * sizeof(double), cudaMemcpyDeviceToHost,
                            stream_));
    TB_CUDA(cudaStreamSynchronize(stream_));
    // scatter into the caller's arrays (updateSolnData, dataUpdate.C:105-119)
    std::vector<int> first(bi_.size());
    for (size_t b = 0; b < bi_.size(); b++) first[b] = bi_[b].node_off;
    for (long long r = 0; r < nrec_; r++) {
      if (h_it_cancel_[r]) continue;
      const int g = h_it_rec_[r];
      // the last block whose first node is <= g (empty blocks share an offset with the next one)
      const int rb = (int)(std::upper_bound(first.begin(), first.end(), g) - first.begin()) - 1;
      const int local = g - bi_[rb].node_off;
      double* q = hb_[rb].hq;
      for (int k = 0; k < nvar; k++) {
        if (interptype == 0) q[(size_t)local * nvar + k] = vals[(size_t)r * nvar + k];
        else q[(size_t)k * hb_[rb].nnodes + local] = vals[(size_t)r * nvar + k];
      }
    }
  } else {
    // the receptors' values straight into the caller's device arrays; the
    // gather finished before (same stream), so every value read was the
    // pre-update one, as with the reference's packet exchange
    k_interp_scatter<<<grid_for(nrec_, kT), kT, 0, stream_>>>(it_rec_.p, it_cancel_.p, rcount_.p, node_blk_.p,
                                                               d_bi_.p, qvals_.p, nvar, interptype, d_qptr_.p);
    TB_LAUNCHED("k_interp_scatter");
    TB_CUDA(cudaStreamSynchronize(stream_));
  }
  return 0;
}

}  // namespace tb
