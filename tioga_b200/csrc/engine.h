// Host-side engine of the B200 TIOGA connectivity path.
//
// Layout in HBM: the nodes and cells of every registered block are
// concatenated into flat arrays (block b owns nodes [node_off, node_off+nnodes)
// and cells [cell_off, cell_off+ncells)), so each stage of the path is one
// launch over all blocks.  Connectivity is stored padded to 8 vertices per
// cell with global (0-based) node ids.  The reference's MPI packet exchanges
// (src/exchangeBoxes.C, exchangeSearchData.C, exchangeDonors.C) become device
// buffers written by one kernel and read by the next.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <vector>

#include "common.cuh"

namespace tb {

constexpr int kMaxLeafCells = 8; // cells per tree leaf at most
// device counters of the sparse donor phase (dcnt_)
constexpr int kHoles = 0;        // holes, the first entries of the marked-node list
constexpr int kMarked = 1;       // holes plus nfringe layers
constexpr int kCancelMarks = 2;  // nodes marked for cancellation
constexpr int kSeg = 4;          // two alternating frontier ranges of the marked list (4 ints)
constexpr int kDedupLeaf = 20;   // uniqNodesTree compares subsets of at most 20 points pairwise
constexpr int kMaxTreeDepth = 32; // tree levels below the root at most (30-bit keys: 29 reachable)
constexpr int kNodeTile = 2048; // nodes per query-gathering tile
constexpr int kSlots = 8;       // inline search candidates per query
constexpr int kMaxBlocks = 100; // MAXBLOCKS, src/globals.h:29
constexpr int kMaxSysBlocks = 16;      // blocks of one overset system (donor lists per node)
constexpr int kMaxEngineBlocks = 8192;
constexpr size_t kHoleMapCap = 197ull * 197ull * 197ull;  // bytes of one hole map at most // blocks of all systems of one engine (16-bit block ids)

// Device bytes of the engine whose calls this thread is running (the
// serving form's admission accounting); null: not counted.
extern thread_local long long* g_dbuf_account;
// When set, buffers are allocated and freed stream-ordered on this stream
// (cudaMallocAsync / cudaFreeAsync), so engines that run side by side on their
// own streams never wait for each other's frees; null: cudaMalloc / cudaFree.
extern thread_local cudaStream_t g_dbuf_stream;
// With g_dbuf_stream: the pool the stream-ordered allocations come from
// (null: the device's current pool).
extern thread_local cudaMemPool_t g_dbuf_pool;

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  long long* acct = nullptr;  // where this allocation is counted
  cudaStream_t st = nullptr;  // stream-ordered allocation: its stream
  bool async = false;
  cudaError_t ensure(size_t count) {
    if (count <= n && p) return cudaSuccess;
    // a buffer that has to grow again gets a quarter more, so slowly growing
    // sizes (moving meshes) do not reallocate every call
    const size_t grow = (p && count) ? count / 4 : 0;
    release();
    size_t c = count ? count + grow : 1;
    async = g_dbuf_stream != nullptr;
    st = g_dbuf_stream;
    cudaError_t e = !async ? cudaMalloc(&p, c * sizeof(T))
                    : g_dbuf_pool ? cudaMallocFromPoolAsync((void**)&p, c * sizeof(T), g_dbuf_pool, st)
                                  : cudaMallocAsync((void**)&p, c * sizeof(T), st);
    if (e == cudaSuccess) {
      n = c;
      acct = g_dbuf_account;
      if (acct) *acct += (long long)(c * sizeof(T));
    } else {
      p = nullptr;
    }
    return e;
  }
  void release() {
    if (p) {
      if (async) cudaFreeAsync(p, st);
      else cudaFree(p);
      if (acct) *acct -= (long long)(n * sizeof(T));
    }
    p = nullptr;
    n = 0;
    acct = nullptr;
    async = false;
    st = nullptr;
  }
};

// POD block descriptor mirrored to the device
struct BlockInfo {
  int tag;
  int nnodes, ncells;
  int node_off, cell_off;
  int ntypes;
  int type_off[5];  // cell offsets of the types inside the block
  int nv[4];
  int nwbc, wall_off;  // wall nodes in the global wall list
  int nobc, obc_off;
  int nfringe;         // snapshot taken at preprocess (tioga.C:95-110)
  int root;            // slot of the block's tree root (4 * block), -1 without cells
  int has_user_res;
  // overset system of the block: every system is connected on its own (pairs,
  // hole maps and donor lists never cross systems); its blocks are
  // consecutive, sblk0 .. sblk0 + snb - 1, in registration order
  int sys, sblk0, snb;
  int hm_lo, hm_hi;    // the system's hole maps: d_hmdev_[hm_lo .. hm_hi)
  int hm;              // the block's own hole map (wall-bearing blocks), else -1
  // uniform-hex fast path (tioga::set_uniform_hex_flag): a box of identical
  // rectangular hexahedra searched by index lookup in its cell map
  int uhex;            // 1: the lookup replaces the tree search for this donor
  int uidims[3];
  double uvec[3][3], uxlow[3], udx[3];
  long long umap_off;  // its map in uhex_map_
  Obb obb;
  float bb_lo[3], bb_hi[3];  // block box for the Morton keys
};

struct PairInfo {  // one (receptor block, donor block) pair, src/exchangeBoxes.C:133-160
  int rec, don;
  double rd[6];    // reduced box accumulator in the donor's OBB frame (ordered bits)
  Obb region;      // donor cells overlapping the receptor OBB, donor axes
  double wbox[6];  // world-axis box holding the region (tile culling)
};

// Per-pair data of the cell pass's FP32 bounds, kept in shared memory: both
// boxes' centres in FP64 (so the centre differences are exact to FP32
// rounding), their axes and the receptor box's half sizes in FP32.
struct PairCull {
  double rxc[3];  // receptor box centre
  double dxc[3];  // donor box centre
  float rvec[9];  // receptor axes, row j = axis j
  float rdxc[3];  // receptor half sizes
  float dvec[9];  // donor axes
  int don;        // donor block
  int pair;       // index in the pair list
};


// the axes of a uniform-hex block (rows), passed by value to a kernel
struct UhexAxes {
  double vec[3][3];
};

// rigid motion x <- a x + b (a row-major)
struct Rigid {
  double a[9], b[3];
};

// one wall-bearing block: its wall nodes in the global wall list, its cells,
// its hole map
struct WallBlock {
  int wall_off, nwall, cell_off, ncells, hm;
};

struct HoleMapInfo {
  int exist;
  int nx[3];
  double ext[6];
};

// High-order elements of one block: Lagrange hexahedra of degree p, DOF
// coordinates element-major (caller-owned, re-read at every high-order call)
struct HoBlockDesc {
  int p = 0, npts = 0;
  const double* hxdof = nullptr;
};
struct HoDev {  // per block, on the device
  int p, npts;
  long long dof_off;  // first DOF of the block in the concatenated DOF array
};
struct HoStats {
  long long npoints = 0, ndonor = 0, nties = 0, nrecords = 0, nmerged = 0, norphan_cells = 0;
  long long ncand = 0, nrefine = 0;  // inclusion tests of in-box candidates, and those decided in FP64
};

// A pair-major query list for the coincident-point merge: query q is point
// qid[q] of `coords` with donor block qdon[q]; node queries give node_blk
// (receptor block per node), point queries give qpt_local (the point's index
// in its receptor block, the list order) and qrec (receptor block per query).
struct DedupQueries {
  long long n;
  const int* qid;
  const int* qdon;
  const int* qpt_local;
  const int* qrec;
  const double* qres;
  const double* coords;
  const blk_t* node_blk;
};

struct HostBlock {
  int sys = 0;
  int tag = 0, nnodes = 0, ncells = 0, ntypes = 0;
  int nv[4] = {0, 0, 0, 0}, nc[4] = {0, 0, 0, 0};
  double* hx = nullptr;
  int* hibl = nullptr;
  int nwbc = 0, nobc = 0;
  int* hwbc = nullptr;
  int* hobc = nullptr;
  int* hconn[4] = {nullptr, nullptr, nullptr, nullptr};
  double* user_nres = nullptr;
  double* user_cres = nullptr;
  int* h_iblank_cell = nullptr;  // caller array (tioga_setcelliblank_)
  const uint64_t* node_gid = nullptr;  // caller's node global ids (registerGridData's node_gid)
  int uniform_flag = 0;          // tioga::set_uniform_hex_flag: check for a uniform box at preprocess
  int uniform = 0;               // found uniform at the last preprocess
  double* hq = nullptr;          // registered host solution
  double* dq = nullptr;          // registered device solution
  int* dibl = nullptr;           // caller's device iblank array (optional)
  const uint64_t* cell_gid = nullptr;  // caller's cell global ids (registerGridData's cell_gid)
};

struct Stats {
  long long nquery = 0;       // Q: query points handed to donor searches
  long long ndonor = 0;       // queries with a donor cell
  long long nties = 0;        // queries whose donor depends on the search order
  long long ncand = 0;        // candidate cells tested with Newton
  long long nrefine = 0;      // FP64 refinements in the split-precision form
  long long nreceptor = 0;    // final iblank == -1
  long long nhole = 0;        // final iblank == 0
  long long nrecords = 0;     // chosen donors (before cancellation)
  long long nleaf = 0;        // tree leaves (the cell pass's units of work, with the cells)
  long long nmerged = 0;      // query points merged into a coincident one (not searched themselves)
  long long npairs = 0;       // intersecting (receptor, donor) block pairs
  long long launches = 0;     // kernels this library launched in the call
  long long cand_verts = 0;   // sum of the vertex counts of the Newton candidates
  long long holemap_cells = 0; // cells of this call's hole maps
  unsigned error = 0;
};

// Launch shapes the autotuner chooses among (results never depend on them):
// CTAs per SM of the cell pass, the query gathering, the traversal and the
// candidate screen, and the pairs one cell-pass CTA holds in shared memory.
struct Tuning {
  int cell_pass_per_sm = 3, query_per_sm = 16, traverse_per_sm = 64, candidates_per_sm = 16, chunk_pairs = 128;
  int cell_box_per_sm = 6;  // split form: CTAs per SM of the box kernel (4, 6 or 8)
  int traverse_variant = 0; // split form: k_traverse (0) or k_traverse_ww, leaves postponed (1)
};

struct Timing {
  float holemap = 0, boxes = 0, refit = 0, query = 0, search = 0, donors = 0, celliblank = 0,
        total = 0, upload = 0, download = 0;
  float traverse = 0, candidates = 0, refine = 0;  // stages of the search
  float cell_pass = 0;                              // the cell pass kernel(s) alone
  float cell_boxes = 0;                             // split form: its box kernel alone
};

class Engine {
 public:
  // high-order path
  int set_highorder(int tag, int p, const double* xdof);
  void set_highorder_callbacks() { ihigh_ = true; }
  // Lowered device bounds for tests of the error paths (0 = the normal
  // bound): which 0 = hole-map fill rounds, 1 = donor-record capacity.
  // launch shapes set by hand (the tuning array's order; values <= 0 keep
  // the current shape; [6] takes the traversal variant plus one)
  int set_tuning(const int in[7]) {
    int* v[5] = {&tune_.cell_pass_per_sm, &tune_.chunk_pairs, &tune_.query_per_sm, &tune_.traverse_per_sm,
                 &tune_.candidates_per_sm};
    for (int i = 0; i < 5; i++)
      if (in[i] > 0) *v[i] = in[i];
    if (in[5] > 0) tune_.cell_box_per_sm = in[5];
    if (in[6] == 1 || in[6] == 2) tune_.traverse_variant = in[6] - 1;
    return 0;
  }
  int set_test_bound(int which, int value) {
    if (which == 0) test_fill_rounds_ = value;
    else if (which == 1) test_rcap_ = value;
    else if (which == 2) up_chunk_ = value > 0 ? value : kUpChunk;  // takes effect at the next preprocess
    else return -1;
    return 0;
  }
  int connectivity_highorder();
  int dataupdate_highorder(int nvar, int interptype);
  int point_donors(int tag, int* out, double* w);
  bool ihigh_global() const { return ihigh_global_; }
  const HoStats& ho_stats() const { return ho_stats_; }
  Engine();
  ~Engine();

  // registration / settings (src/tioga.C:64-93, tioga.h:181-205)
  int register_block(int tag, int nnodes, double* x, int* ibl, int nwbc, int nobc, int* wbc,
                     int* obc, int ntypes, const int* nv, const int* nc, int** conn);
  int register_block_sys(int sys, int tag, int nnodes, double* x, int* ibl, int nwbc, int nobc, int* wbc,
                         int* obc, int ntypes, const int* nv, const int* nc, int** conn);
  int find_block(int sys, int tag) const;
  int nsystems() const;
  void select_system(int sys) { cur_sys_ = sys; }
  int selected_system() const { return cur_sys_; }
  void set_symmetry(int s) { isym_ = s; }
  void set_nfringe(int n) { nfringe_ = n; }
  void set_mexclude(int m) { mexclude_ = m; }
  int set_resolutions(int tag, double* nres, double* cres);
  int set_cell_iblank(int tag, int* ibc);
  int register_solution(int tag, double* q, bool device);
  int register_iblank_device(int tag, int* d_ibl);
  void set_precision(int p) { precision_ = p; }
  void set_coords_resident(int r) { coords_resident_ = r; }
  // serving form: rigid motion of a block's device coordinates (x <- A x + b,
  // A row-major), the caller's iblank array of a block, the device
  // coordinates written back to the caller's arrays, device bytes held
  int apply_rigid(int block, const double* A, const double* b);
  void set_host_iblank(int block, int* ibl) { hb_[block].hibl = ibl; }
  int download_coords();
  long long* byte_counter() { return &dev_bytes_; }
  // serving: preprocess leaves the caller's iblank alone (connectivity
  // rewrites all of it)
  void set_serving(bool v) { serving_ = v; }
  long long device_bytes() const { return dev_bytes_; }
  void set_stream(cudaStream_t s);

  // the path
  int preprocess();
  int connectivity();
  // times each launch shape of every tuned kernel over `reps` connectivity
  // calls (coordinate descent, one knob after the other) and keeps the
  // fastest; needs a preprocessed instance
  int autotune(int reps);
  // tioga_reduce_fringes_: keep the receptors within nfringe+1 layers of the
  // field, hole the others (after connectivity)
  int reduce_fringes();
  // tioga_writeoutputfiles_: the Tecplot flow files of every block
  int write_output(int nvar, int interptype);
  const Tuning& tuning() const { return tune_; }
  int dataupdate(int nvar, int interptype);

  // queries (src/dataUpdate.C:121-159, tioga.C:533-570)
  int donor_count(int tag, int* dcount, int* fcount);
  int donor_info(int tag, int* receptors, int* indices, double* frac);
  int set_cell_gid(int tag, const uint64_t* gid);
  int set_uniform_hex_flag(int tag, int flag);
  int set_node_gid(int tag, const uint64_t* gid);
  void set_nodegid_merge(int on) { nodegid_merge_ = on != 0; }
  void set_pin_host(int on) {
    pin_host_ = on != 0;
    if (!pin_host_) unpin_caller_arrays();
  }
  // tioga::getReceptorInfo: 4 ints per live record of the selected system;
  // writes min(count, cap) ints to out (may be null) and returns the count,
  // or < 0 on error
  long long receptor_info(int* out, long long cap);
  int cell_iblank(int tag, int* out);
  const Stats& stats() const { return stats_; }
  const Timing& timing() const { return timing_; }
  cudaStream_t stream() const { return stream_; }
  int nblocks() const { return (int)hb_.size(); }
  int first_tag() const { return hb_.empty() ? -1 : hb_[0].tag; }
  int last_error() const { return last_error_; }

 private:
  int upload_topology();
  int build_csr();
  int compute_obbs();
  int build_tree_topology();
  int upload_coords();
  int check_coords();
  int build_upload_chunks();  // preprocess: the leaves of each upload chunk
  int build_tile_chunks();    // preprocess: the node tiles of each upload chunk
  int upload_chunked();       // coordinates up in chunks, the cell boxes made as they land
  int donor_reset_begin(); // side stream: the previous call's donor marks back to rest
  int holemaps_begin();    // side stream: wall bounds, map extents, wall-cell boxes, extents to the host
  int holemaps_end();      // host: map sizes; side stream: fill and final maps (joined before the donors)
  int preprocess_resolutions();
  int run_pairs_and_refit();
  int setup_uniform_hex();
  int run_gid_merge();
  void pin_caller_arrays();
  void unpin_caller_arrays();
  int run_queries();
  int run_search();
  int run_donors();
  int donor_rest_init();
  int dedup_gate();
  int run_dedup();
  int dedup_merge(const DedupQueries& Q, const std::vector<int>& qoff);
  int traverse_and_gather(const double* xq, const int* qn, const int* qd, long long nq, unsigned& count,
                          int skip_uhex = 0);
  int run_celliblank();
  int download_iblank();
  int fetch_interps();
  int find_tag(int tag) const;

  std::vector<HostBlock> hb_;
  std::vector<BlockInfo> bi_;
  std::map<long long, int> tag2idx_;  // (system << 32 | tag) -> block
  int isym_ = 3, nfringe_ = 1, mexclude_ = 3;
  int precision_ = 1;        // 0 = FP64 throughout, 1 = FP32 screen + FP64 refine
  int coords_resident_ = 0;  // 1: the caller promises x has not moved
  bool coords_on_device_ = false;  // x_ holds the registered blocks' coordinates
  long long dev_bytes_ = 0;        // device bytes of this engine's buffers (when counted)
  bool serving_ = false;
  long long topo_gen_ = 0;             // bumped whenever the topology buffers are replaced
  cudaGraphExec_t pre_exec_ = nullptr;  // preprocess_resolutions as a graph, for topology pre_key_
  long long pre_key_ = -1, pre_nlaunch_ = 0;
  bool use_graphs_ = true;
  bool topo_dirty_ = true;
  bool preprocessed_ = false;
  bool connected_ = false;
  int npairs_ = 0;
  int maxtag_ = 0;
  int cur_sys_ = 0;               // system whose tags the tag-based calls address
  int nhm_ = 0;
  long long nq_ = 0;
  std::vector<PairInfo> h_pairs_;
  DBuf<int> visit_;
  DBuf<long long> leafbase_;
  DBuf<unsigned long long> pair_acc_;
  // search stages
  DBuf<unsigned long long> qkey_;
  DBuf<unsigned> qacc_, scount_;
  DBuf<int2> cand_;
  DBuf<int> refine_;
  long long cand_cap_ = 0, ncand_ = 0;
  bool search_timed_ = false;
  // tree refit and query tiles
  DBuf<int> inv_sorted_;
  DBuf<long long> tile_base_;
  std::vector<long long> h_tile_base_;
  DBuf<float4> tbox_;
  DBuf<int> node_order_;    // Morton order of each block's nodes
  DBuf<int> slots_, ncand_q_, cand_off_;
  DBuf<int3> ovf_;
  DBuf<int> cell_stage_;     // one block's cells in the caller's order
  long long ntot_ = 0, ctot_ = 0, inc_tot_ = 0;
  int last_error_ = 0;
  cudaStream_t stream_ = nullptr;
  cudaStream_t own_stream_ = nullptr;
  long long nlaunch_ = 0;
  cudaEvent_t ev_[12];
  // The hole maps run on a stream of their own beside the cell pass, the
  // query gathering and the search, and join before the donor phase:
  // hev_[0] = the coordinates are on the device (main stream), [1] = the
  // maps' extents are on the host, [2] = the maps are done (side stream).
  cudaStream_t side_ = nullptr;
  cudaEvent_t hev_[3];
  cudaEvent_t cib_ev_[2];  // the cell iblanks on the side stream: start (main), done (side)
  cudaEvent_t dr_ev_;      // call start (main): the previous call's donor marks go back to rest on the side stream
  cudaEvent_t rf_ev_;      // the tree refit (side stream) is done: the traversal may start
  // Chunked upload (split form, coordinates not resident): the coordinates go
  // up in chunks of kUpChunk global node ids on up_, and as each lands the
  // main stream checks it, makes its FP32 copy and the cell boxes of the
  // leaves whose last vertex it holds, beside the rest of the upload.
  static constexpr int kUpChunk = 1 << 21;
  int up_chunk_ = kUpChunk;  // the chunk size in use (smaller only in tests)
  cudaStream_t up_ = nullptr;
  cudaEvent_t up_start_ = nullptr;
  std::vector<cudaEvent_t> up_ev_;
  DBuf<int> up_leaf_ids_;                 // leaf ids sorted by upload chunk
  std::vector<long long> h_up_leaf_off_;  // chunk k's leaves: up_leaf_ids_[off[k] .. off[k + 1])
  DBuf<int> up_tile_ids_;                 // node-tile ids sorted by upload chunk
  std::vector<long long> h_up_tile_off_;  // chunk k's tiles: up_tile_ids_[off[k] .. off[k + 1])
  bool boxes_ready_ = false;              // this call's cell boxes were made during the upload
  bool tiles_ready_ = false;              // and its node tiles' boxes
  bool hm_pending_ = false;  // holemaps_begin ran and holemaps_end has not
  // pinned host staging of the hole maps (so the side stream's copies never
  // block the host): ordered-key initial bounds, extents read back, map views
  unsigned long long* h_hm_init_ = nullptr;
  HoleMapInfo* h_hm_info_ = nullptr;
  HoleMapDev* h_hm_dev_ = nullptr;
  int h_hm_cap_ = 0;
  cudaEvent_t sev_[4];
  cudaEvent_t cev_[3];  // around the cell pass (split form: and between its two kernels)
  cudaEvent_t pev_;     // the pairs' copy to the host has landed
  bool cell_timed_ = false;

  // flat device arrays
  DBuf<double> x_, node_res_, cell_res_;
  DBuf<int> iblank_, iblank_cell_, conn8_;
  DBuf<blk_t> node_blk_, cell_blk_;
  DBuf<unsigned char> cell_nv_, wallf_, obcf_, ex0_, ex1_, m0_;
  DBuf<int> m1_, cmark_;            // nfringe marks and cancel marks (first marker wins an atomicExch)
  DBuf<int> mlist_, cmlist_, dcnt_;  // marked nodes (holes first), cancel-marked nodes, their counters
  // coincident query points (uniqNodesTree)
  DBuf<short> node_bin_;            // 10x10x10 OBB bin of every node (donor-list order)
  bool dedup_active_ = false;       // some block has nodes within the gate's distance
  bool gate_valid_ = false;         // the gate holds for the device coordinates (moved rigidly since)
  bool dedup_ran_ = false;          // this call merged coincident query points
  DBuf<int> q_xt_, q_rep_, q_gpos_, dd_refq_, dd_perm_, dd_perm2_, dd_mtag_, dd_itag_, dd_seg_, dd_cnt_, dd_ireset_;
  DBuf<double> dd_x_, dd_rtag_;
  DBuf<unsigned long long> dd_key_, dd_key2_, dd_box_;
  DBuf<unsigned char> dd_oct_;
  DBuf<int> cg_cnt_, cg_off_, cg_v0_, cg_v1_;   // preprocess gate scratch
  DBuf<unsigned long long> cg_k0_, cg_k1_;
  DBuf<unsigned> cg_flag_;
  DBuf<int4> dd_chunks_, dd_leaves_;
  DBuf<int> dd_starts_, dd_pqoff_, dd_prank_;
  // high-order path
  std::vector<HoBlockDesc> ho_;
  bool ihigh_ = false, ihigh_global_ = false, ho_done_ = false;
  bool ho_dof_on_device_ = false;  // ho_xdof_ holds the registered DOF coordinates
  DBuf<HoDev> ho_dev_;
  DBuf<double> ho_xdof_, ho_pts_, ho_qres_, ho_w_, ho_q_, ho_qtmp_;
  DBuf<int> ho_ctag_, ho_rcblk_, ho_qpt_, ho_qloc_, ho_qdon_, ho_qrec_, ho_qbest_, ho_npass_, ho_qcell_, ho_win_;
  DBuf<long long> ho_rcoff_d_, ho_ptoff_d_, ho_qoff_d_;
  DBuf<int4> ho_rec_;
  std::vector<long long> ho_rc_off_, ho_pt_off_;
  long long ho_nrc_ = 0, ho_nq_ = 0, ho_nrecs_ = 0, ho_qcap_ = 0;
  int ho_wstride_ = 1;
  HoStats ho_stats_;
  int prev_nrec_ = 0;               // records of the previous call (their receptors are reset next call)
  bool donor_rest_ = false;         // per-node donor state is in its rest state
  DBuf<int> wall_list_, obc_list_;
  DBuf<int> csr_off_, csr_cell_, deg_;
  DBuf<BlockInfo> d_bi_;
  DBuf<PairInfo> d_pairs_;
  DBuf<int2> d_pcand_;              // (donor, receptor) blocks that may pair, donor-major
  int npcand_ = 0;
  DBuf<int> d_pfirst_;              // first pair of every donor block (nb + 1)
  std::vector<int> h_pfirst_;
  DBuf<int4> d_chunks_;             // cell pass: (first leaf, end leaf, first pair, pairs) per chunk
  DBuf<int> d_chunk_cta_;
  std::vector<int> h_blk_leaf_;     // leaves of block b: [h_blk_leaf_[b], h_blk_leaf_[b + 1])
  DBuf<long long> d_pair_t0_;       // query tiles of pair p: [pair_t0[p], pair_t0[p + 1])
  std::vector<long long> h_pair_t0_;
  std::vector<WallBlock> h_wall_;
  DBuf<int> wall_cells_;            // cells touching a wall node, storage order (hole-map marking)
  int nwall_cells_ = 0;
  DBuf<unsigned long long> wall_box_;  // each wall cell's marked index box this call (packed)
  DBuf<int> wall_box_first_;        // wall cells of hole map t: [first[t], first[t + 1])
  DBuf<WallBlock> d_wall_;
  DBuf<int> d_npairs_;
  DBuf<HoleMapInfo> d_hm_;
  DBuf<HoleMapDev> d_hmdev_;
  DBuf<unsigned char> hm_state_;  // kHoleMapCap bytes per hole map
  int nhm_all_ = 0;               // wall-bearing blocks (hole maps) of all systems
  DBuf<unsigned long long> wall_bb_;
  // tree
  DBuf<int> sorted_cell_;
  DBuf<float2> cbox_;      // split form: 3 per sorted cell (FP32 box rounded outward, 24 bytes)
  DBuf<float4> lbox_;      // split form: 2 per leaf, in leaf order (its box, and its block in the 7th word)
  DBuf<int> pair_ext_;     // split form: 6 per pair, the seeds of the extents' bounds (fkey order)
  DBuf<float4> xf_;        // coordinates rounded to FP32, one per node (split-form cell boxes)
  DBuf<float4> tnode_;     // 2 per tree node
  DBuf<double> tnode64_;   // 6 per tree node (FP64 form)
  DBuf<double> cbox64_;    // 6 per sorted cell (FP64 form)
  long long tree_nodes_ = 0;      // slots, four per group
  long long nleaf_total_ = 0;     // leaves, all blocks
  int tree_depth_ = 0;            // deepest level below a root
  bool tnode64_empty_ = false;    // tnode64_ initialised to empty boxes for this topology
  DBuf<int4> leaves_;             // (first cell, cells, slot, block), storage order
  DBuf<int> gparent_, gnk_;      // per slot group: parent slot, children
  DBuf<int> gnint_, refit_start_, refit_cnt_;  // one-launch refit: internal children, starting groups, counts
  int nrefit_start_ = 0;
  // queries
  DBuf<int> qnode_, qdon_, qcell_;
  DBuf<double> qres_;
  DBuf<unsigned char> qtie_;
  DBuf<int> qcount_;
  DBuf<int> tile_cnt_, tile_off_;
  DBuf<unsigned char> tile_mask_;  // query gathering: per node tile and thread, its 8 nodes' region test
  long long qcap_ = 0;
  // donors
  DBuf<int> slot_;          // K per node
  int K_ = 1;
  DBuf<unsigned long long> rkey_, rkey_alt_;
  DBuf<int> rval_, rval_alt_;
  DBuf<int> rcount_;
  DBuf<int> reset_t_;
  DBuf<int> interp2rec_;    // per query
  DBuf<int> it_node_;       // 9 per record (nv donor nodes + donor cell, block-local)
  DBuf<double> it_w_;       // 9 per record
  DBuf<int> it_rec_;        // receptor global node per record
  DBuf<int> it_don_;        // donor block per record
  DBuf<unsigned char> it_nv_, it_cancel_;
  DBuf<double> rres_;       // receptor resolution per record
  DBuf<int> rf_red_, rf_tmp_;        // reduce_fringes: reduced iblank and its next layer, per node
  DBuf<unsigned char> rf_was_;      // reduce_fringes: records live before it
  long long nrec_ = 0;
  // data update
  DBuf<double> q_, qvals_;
  DBuf<double*> d_qptr_;   // every block's solution on the device (data update)
  // scratch for CUB and reductions
  DBuf<unsigned char> cub_tmp_;
  DBuf<double> red_;
  DBuf<unsigned> err_;
  DBuf<unsigned> coord_err_;  // non-finite coordinate flag (check_coords)
  int test_fill_rounds_ = 0, test_rcap_ = 0;  // set_test_bound
  DBuf<int> uhex_map_;                  // cell maps of the uniform-hex blocks
  DBuf<unsigned long long> uhex_red_;   // set-up scratch: extents, check flag
  bool any_uhex_ = false;
  bool nodegid_merge_ = false;         // coincident query points merged by node id (TIOGA_HAS_NODEGID)
  std::vector<void*> pinned_;          // caller arrays this engine page-locked (cudaHostRegister)
  bool pin_host_ = true;               // page-lock pageable caller arrays (tioga_b200_set_pin_host_)
  DBuf<unsigned long long> node_gid_d_, gm_k0_, gm_k1_, gm_max_;
  DBuf<int> gm_a_, gm_b_, gm_c_, gm_d_;
  DBuf<unsigned long long> counters_;
  DBuf<unsigned long long> mkey_, mkey_alt_;
  DBuf<int> mval_alt_;

  // host copies of the interpolation lists (filled lazily for queries)
  bool interps_fetched_ = false;
  std::vector<int> h_it_node_, h_it_rec_, h_it_don_;
  std::vector<double> h_it_w_;
  std::vector<unsigned char> h_it_nv_, h_it_cancel_;

  Stats stats_;
  Timing timing_;
  Tuning tune_;
};

}  // namespace tb
