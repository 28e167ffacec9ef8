// Kernel declarations and small device helpers shared by the kernel files.
#pragma once

#include <string.h>

#include "common.cuh"
#include "engine.h"

namespace tb {


__device__ __forceinline__ void gather_vertices(const double* __restrict__ x, const int* __restrict__ cv,
                                                int nv, double xv[8][3]) {
#pragma unroll
  for (int m = 0; m < 8; m++) {
    if (m < nv) {
      const double* p = x + 3 * (long long)cv[m];
      xv[m][0] = p[0];
      xv[m][1] = p[1];
      xv[m][2] = p[2];
    }
  }
}

// order-preserving map of a double onto an unsigned 64-bit key, so that
// atomicMin/atomicMax on the key are exact min/max on the double
__device__ __forceinline__ unsigned long long dkey(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__host__ __device__ inline double dkey_inv(unsigned long long k) {
  unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
  double d;
  memcpy(&d, &b, sizeof(d));
  return d;
}

// the last block whose first node tile is <= T (tile_base[b] = first tile of block b)
__device__ __forceinline__ int block_of_tile(const long long* __restrict__ tile_base, int nb, long long T) {
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    const int m = (lo + hi + 1) >> 1;
    if (tile_base[m] <= T) lo = m;
    else hi = m - 1;
  }
  return lo;
}

// ---- preprocess (kernels_pre.cu) ----
__global__ void k_conn_convert(const int* raw, int nc, int nv, int node_off, int nnodes, int cell_base, int blk,
                               int* conn8, unsigned char* cell_nv, blk_t* cell_blk, unsigned* err);
__global__ void k_check_finite(const double* x, long long n, unsigned* err);
__global__ void k_node_blk(int node_off, int nnodes, int blk, blk_t* node_blk);
__global__ void k_mark_list(const int* list, int n, int node_off, int nnodes, int* glist, int goff,
                            unsigned char* flag, unsigned* err);
__global__ void k_csr_count(const int* conn8, const unsigned char* cell_nv, long long ctot, int* deg);
__global__ void k_csr_fill(const int* conn8, const unsigned char* cell_nv, long long ctot,
                           const int* off, int* cursor, int* cells);
__global__ void k_csr_sort(const int* off, long long ntot, int* cells);
__global__ void k_cell_volume(const double* x, const int* conn8, const unsigned char* cell_nv,
                              const blk_t* cell_blk, const BlockInfo* bi, long long ctot,
                              double* cell_res);
__global__ void k_node_res(const int* off, const int* cells, const double* cell_res,
                           const blk_t* node_blk, const BlockInfo* bi, long long ntot,
                           double* node_res);
__global__ void k_mandatory(const int* conn8, const unsigned char* cell_nv, long long ctot,
                            const unsigned char* obcf, double* node_res, unsigned char* ex0,
                            unsigned char* ex1);
__global__ void k_mexclude(const int* conn8, const unsigned char* cell_nv, long long ctot,
                           const unsigned char* ex0, unsigned char* ex1, double* cell_res);
__global__ void k_copy_u8(const unsigned char* a, unsigned char* b, long long n);
__global__ void k_fill_int(int* a, int v, long long n);
__global__ void k_rigid(double* x, int n, Rigid m);
__global__ void k_obb_partial(const double* x, const BlockInfo* bi, int pass, double* part);
__global__ void k_obb_finish(const double* part, int nparts, int pass, const double* x, BlockInfo* bi, int nb);
__global__ void k_morton(const double* x, const int* conn8, const unsigned char* cell_nv,
                         const blk_t* cell_blk, const BlockInfo* bi, long long ctot,
                         unsigned long long* key, int* val);

// ---- connectivity (kernels_conn.cu) ----
__global__ void k_wall_bounds(const double* x, const int* wall_list, const WallBlock* wt, unsigned long long* bb);
__global__ void k_holemap_setup(const unsigned long long* bb, HoleMapInfo* hm, int nhm);
__global__ void k_holemap_mark(const double* x, const int* conn8, const unsigned char* cell_nv, const int* wall_cells,
                               int nwc, const blk_t* cell_blk, const BlockInfo* bi, const HoleMapInfo* hm,
                               unsigned char* sam, size_t cap);
__global__ void k_wall_cell_flags(const int* conn8, const unsigned char* cell_nv, const blk_t* cell_blk,
                                  const BlockInfo* bi, const unsigned char* wallf, long long ctot, int* flag);
__global__ void k_wall_cell_list(const int* flag, const int* off, long long ctot, int* list);
__global__ void k_holemap_fill_bits(unsigned char* sam, const HoleMapInfo* hm, size_t cap, const unsigned long long* box,
                                    const int* box_first, int isym, int round_cap, unsigned* err);
__global__ void k_wall_map_first(const int* wall_cells, int nwc, const blk_t* cell_blk, const BlockInfo* bi,
                                 int* first);
__global__ void k_holemap_boxes(const double* x, const int* conn8, const unsigned char* cell_nv, const int* wall_cells,
                                int nwc, const blk_t* cell_blk, const BlockInfo* bi, const HoleMapInfo* hm,
                                unsigned long long* box);
__global__ void k_holemap_fill_planes(unsigned char* sam, const HoleMapInfo* hm, size_t cap, int isym, int seed,
                                      unsigned* err);
__global__ void k_holemap_lines(unsigned char* sam, const HoleMapInfo* hm, size_t cap, int axis, unsigned* changed);
__global__ void k_holemap_final(unsigned char* sam, const HoleMapInfo* hm, size_t cap);
__global__ void k_pairs(const BlockInfo* bi, int nb, const int2* cand, int ncand, PairInfo* pairs, int* npairs,
                        int* pfirst);
__global__ void k_pair_finish(const BlockInfo* bi, PairInfo* pairs, int npairs,
                              const unsigned long long* acc);
void launch_cell_boxes(int minb, int grid, cudaStream_t st, const float4* xf, const int* conn8,
                       const unsigned char* cell_nv, const int4* leaves, const int* ids, long long nleaf, float2* cbox,
                       float4* tnode, float4* lbox);
__global__ void k_leaf_chunk(const int4* leaves, long long nleaf, const int* conn8, const unsigned char* cell_nv,
                             int chunk, int* key, int* id);
__global__ void k_round_nodes(const double* x, long long lo, long long hi, float4* xf);
void launch_cell_pairs(int minb, int grid, size_t smem, cudaStream_t st, const double* x, const int* conn8,
                       const unsigned char* cell_nv, const BlockInfo* bi, const int4* leaves, const int4* chunks,
                       const int* chunk_cta, int nchunks, const int* pfirst, const PairInfo* pairs,
                       const float2* cbox, const float4* lbox, int* ext, unsigned long long* acc);
void launch_cell_pass64(int minb, int grid, size_t smem, cudaStream_t st, const double* x, const int* conn8,
                        const unsigned char* cell_nv, const BlockInfo* bi, const int4* leaves, const int4* chunks,
                        const int* chunk_cta, int nchunks, const int* pfirst, const PairInfo* pairs, double* cbox64,
                        float4* tnode, double* tnode64, unsigned long long* acc);

__global__ void k_tree_split(const unsigned long long* key, int n, const int* ca, const int* cb, const int* cslot,
                             int2* kids, int* nk, int* isint, int2* tlink, int* leaf_at);
__global__ void k_tree_link(int n, const int* cslot, const int2* kids, const int* nk, const int* isint,
                            const int* ioff, const int* koff, int g0, int2* tlink, int* gparent, int* gnk, int* na,
                            int* nb, int* nslot);
__global__ void k_tree_init(const int2* tlink, long long nslots, float4* tnode);
__global__ void k_tree_init64(long long nslots, double* t64);
__global__ void k_leaf_flags(const int* leaf_at, long long ctot, int* flag);
__global__ void k_leaf_list(const int* leaf_at, const int* loff, long long ctot, const int2* tlink,
                            const blk_t* cell_blk, int4* leaves);
__global__ void k_block_leaves(const int4* leaves, long long nleaf, int* first);
__global__ void k_group_nint(const float4* tnode, int g_root, int ngroups, int* nint, int* start, int* nstart);
__global__ void k_refit_fused(const int* start, int nstart, const int* gparent, const int* nint, int g_root,
                              int* cnt, float4* tnode, double* tnode64);
__global__ void k_node_tiles(const double* x, const BlockInfo* bi, int nb, const long long* tile_base,
                             float4* tbox, const int* node_order, float4* xf, const int* ids);
__global__ void k_tile_chunk(const BlockInfo* bi, int nb, const long long* tile_base, const int* node_order, int chunk,
                             int* key, int* id);
__global__ void k_morton_nodes(const double* x, const blk_t* node_blk, const BlockInfo* bi,
                               long long ntot, unsigned long long* key, int* val);
__global__ void k_invert(const int* perm, long long n, int* inv);
__global__ void k_permute_cells(const int* perm, long long n, const int* conn8, const unsigned char* nv,
                                const blk_t* blk, int* conn8_out, unsigned char* nv_out,
                                blk_t* blk_out);
__global__ void k_remap(int* idx, long long n, const int* map);
__global__ void k_scatter_f64(const double* src, long long n, const int* inv, long long base, double* dst);
__global__ void k_query_count(const double* x, const BlockInfo* bi, const PairInfo* pairs, int npairs,
                              const long long* pair_t0, int tile, int* tile_cnt, const float4* tbox,
                              const long long* tile_base, const int* node_order, unsigned char* tile_mask);
__global__ void k_query_write(const BlockInfo* bi, const PairInfo* pairs, int npairs, const long long* pair_t0,
                              int tile, const int* tile_off, const double* node_res, int* qnode, int* qdon,
                              double* qres, const int* node_order, const unsigned char* tile_mask);
// host launchers of the templated search stages (same translation unit as
// their instantiations)
void launch_traverse(int form, int variant, int blocks, cudaStream_t st, const double* x, const BlockInfo* bi,
                     const float2* cbox, const double* cbox64, const float4* tnode, const double* tnode64,
                     const int* qnode, const int* qdon, long long nq, int* slots, int* ncand_q, int3* ovf,
                     int ovf_cap, unsigned* novf, unsigned* err, int skip_uhex);
__global__ void k_gather_candidates(const int* slots, const int* ncand_q, const int* off, long long nq,
                                    const int3* ovf, const unsigned* novf, int ovf_cap, int2* cand);
void launch_candidates(int form, int blocks, cudaStream_t st, const double* x, const int* conn8,
                       const unsigned char* cell_nv, const double* cell_res, const int* sorted_cell,
                       const int* qnode, const int2* cand, int ncand, unsigned long long* qkey, unsigned* qacc,
                       int* refine, unsigned* nrefine, unsigned long long* counters);
__global__ void k_refine(const double* x, const int* conn8, const unsigned char* cell_nv, const double* cell_res,
                         const int* sorted_cell, const int* qnode, const int2* cand, const int* refine,
                         const unsigned* nrefine, unsigned long long* qkey, unsigned* qacc);
__global__ void k_search_finish(const unsigned long long* qkey, const unsigned* qacc, long long nq,
                                const int* inv_sorted, int* qcell, unsigned char* qtie,
                                unsigned long long* counters);

// ---- uniform-hex fast path (kernels_uhex.cu) ----
__global__ void k_uhex_check(const double* x, const int* conn8, const BlockInfo* bi, int b, double d0, double d1,
                             double d2, unsigned* bad);
__global__ void k_uhex_extent(const double* x, long long node_off, long long nnodes, UhexAxes A,
                              unsigned long long* red);
__global__ void k_uhex_map(const double* x, const int* conn8, const int* sorted_cell, const BlockInfo* bi, int b,
                           int* map);
__global__ void k_uhex_search(const double* x, const int* qnode, const int* qdon, long long nq, const BlockInfo* bi,
                              const int* map, const double* cell_res, const int* inv_sorted, int* qcell,
                              unsigned char* qtie);

// ---- donors (kernels_donor.cu) ----
__global__ void k_fill_slots(const int* qnode, const int* qdon, const int* qcell, long long nq, int K,
                             long long ntot, long long ctot, const BlockInfo* bi, int nb, int* slot, unsigned* err);
__global__ void k_donor_reset(const int* mlist, const int* dcnt, const int* it_rec, const unsigned char* it_cancel,
                              int prev_R, const int* csr_off, const int* csr_cell, int* iblank, unsigned char* m0,
                              int* m1, int* iblank_cell);
__global__ void k_classify_queried(const double* x, const blk_t* node_blk, const BlockInfo* bi,
                                   const int* slot, int K, const int* qnode, const int* qcell, long long nq,
                                   const double* qres, const HoleMapDev* hm, int* iblank, double* node_res,
                                   unsigned char* m0, int* m1, int* mlist, int* dcnt, unsigned long long* counters);
__global__ void k_classify_tiles(const double* x, const BlockInfo* bi, int nb, const long long* tile_base,
                                 const float4* tbox, const int* node_order, const int* slot, int K,
                                 const HoleMapDev* hm, int* iblank, unsigned char* m0, int* m1, int* mlist,
                                 int* dcnt, unsigned long long* counters);
__global__ void k_front_init(int* dcnt);
__global__ void k_dilate_front(int iter, const int* csr_off, const int* csr_cell, const int* conn8,
                               const unsigned char* cell_nv, const blk_t* cell_blk, const BlockInfo* bi,
                               const unsigned char* m0, int* m1, int* mlist, int* dcnt);
__global__ void k_front_next(int iter, unsigned char* m0, const int* mlist, int* dcnt);
__global__ void k_fringe_big_list(const int* mlist, const int* dcnt, const int* iblank, double* node_res);
__global__ void k_select(const blk_t* node_blk, const BlockInfo* bi, const int* slot, int K,
                         const int* qnode, const int* qcell, long long nq, const double* cell_res, int* iblank,
                         const double* node_res, unsigned long long* rkey, int* rval, int* rcount, int rcap,
                         unsigned* err);
__global__ void k_interp_marks(const unsigned long long* rkey, const int* rval, const int* rcount,
                               const int* qcell, const int* conn8, const unsigned char* cell_nv,
                               const int* iblank, const double* node_res, int* cmark, int* reset_t, int* cmlist,
                               int* dcnt);
__global__ void k_interp(const double* x, const unsigned long long* rkey, const int* rval,
                         const int* rcount, const int* qcell, const int* conn8,
                         const unsigned char* cell_nv, const blk_t* node_blk,
                         const BlockInfo* bi, const int* iblank, const double* node_res,
                         const int* reset_t, const int* orig_cell, int* it_node, double* it_w, int* it_rec,
                         int* it_don, unsigned char* it_nv, unsigned char* it_cancel, double* rres,
                         int* interp2rec, unsigned* err);
__global__ void k_node_bins(const double* x, const blk_t* node_blk, const BlockInfo* bi, long long ntot,
                            short* node_bin);
__global__ void k_coin_count(const double* x, const blk_t* node_blk, const BlockInfo* bi, long long ntot,
                             int* cnt);
__global__ void k_coin_fill(const double* x, const blk_t* node_blk, const BlockInfo* bi, long long ntot,
                            const int* off, unsigned long long* key, int* val);
__global__ void k_coin_check(const unsigned long long* key, const int* val, long long n, const double* x,
                             const blk_t* node_blk, const BlockInfo* bi, unsigned* flag);
__global__ void k_dedup_keys(const int* qnode, const int* qdon, long long nq, const int* pair_qoff, int npairs,
                             const int* pair_rank, const short* node_bin, unsigned long long* key, int* val);
__global__ void k_dedup_keys_pts(const int* qpt_local, const int* qdon, long long nq, const int* pair_qoff,
                                 int npairs, const int* pair_rank, unsigned long long* key, int* val);
__global__ void k_dedup_gather(const int* refq, long long n, const int* qnode, const double* qres, const double* x,
                               const blk_t* node_blk, const int* qrec, const BlockInfo* bi, double* xg,
                               int* mtag, double* rtag, int* itag, int* perm, int* gpos_of);
__global__ void k_dedup_box(const int4* chunks, const int* perm, const double* xg, unsigned long long* box);
__global__ void k_dedup_octant(const int4* chunks, const int* perm, const double* xg, const unsigned long long* box,
                               unsigned char* oct, int* cnt);
__global__ void k_dedup_pkeys(const int* segstart, const unsigned char* oct, long long n, unsigned long long* key);
__global__ void k_dedup_segfill(const int4* chunks, const int* starts, int* segstart);
__global__ void k_dedup_leaves(const int4* leaves, int nleaves, const int* perm, const double* xg, const int* mtag,
                               double* rtag, int* itag);
__global__ void k_dedup_apply(const int* refq, long long n, const int* itag, const double* rtag, double* qres,
                              int* q_xt, int* q_rep, unsigned* err, unsigned long long* counters);
__global__ void k_dedup_copy(const int* q_rep, long long nq, int* qcell, unsigned char* qtie);
__global__ void k_gid_keys(const int* refq, long long n, const int* qnode, const int* qdon,
                           const unsigned long long* node_gid, unsigned long long* gkey, int* dkey16, int* pos);
__global__ void k_gid_heads(const int* pos, long long n, const unsigned long long* gkey_of_pos, const int* don_of_pos,
                            int* head);
__global__ void k_gid_apply(const int* pos, const int* first, long long n, int* itag, const double* rtag,
                            unsigned long long* rmax);
__global__ void k_gid_res(const int* itag, long long n, const unsigned long long* rmax, double* rtag);
__global__ void k_gather_i32(const int* src, const int* idx, long long n, int* out);
__global__ void k_reset_coincident_min(const int* interp2rec, const int* q_xt, long long nq,
                                       const unsigned char* it_cancel, int* ireset);
__global__ void k_reset_coincident_set(const int* interp2rec, const int* q_xt, long long nq, const int* ireset,
                                       unsigned char* it_cancel);
__global__ void k_cancel(const int* cmlist, const int* dcnt, const int* slot, int K, const int* qcell,
                         const double* cell_res, const int* interp2rec, unsigned char* it_cancel);
__global__ void k_iblank_final(const int* it_rec, const unsigned char* it_cancel, const int* rcount, int* iblank,
                               unsigned long long* counters);
__global__ void k_donor_clear(const int* qnode, const int* qdon, const int* qcell, long long nq, int K,
                              const BlockInfo* bi, int* slot, const int* cmlist, const int* dcnt, int* cmark,
                              int* reset_t);
__global__ void k_rf_init(const int* iblank, long long n, int* red, int* tmp);
__global__ void k_rf_layer(int iter, const int* it_rec, const unsigned char* it_cancel, const int* rcount,
                           const int* csr_off, const int* csr_cell, const int* conn8, const unsigned char* cell_nv,
                           const blk_t* cell_blk, const BlockInfo* bi, const int* iblank, const int* red, int* tmp);
__global__ void k_rf_copy(const int* it_rec, const unsigned char* it_cancel, const int* rcount, const int* tmp,
                          int* red);
__global__ void k_rf_cancel(const int* it_rec, const int* rcount, const int* red, unsigned char* it_cancel,
                            unsigned char* was);
__global__ void k_rf_iblank(const int* it_rec, const unsigned char* it_cancel, const unsigned char* was,
                            const int* rcount, const int* red, int* iblank, unsigned long long* counters);
__global__ void k_cell_iblank_sparse(const int* mlist, const int* dcnt, const int* it_rec,
                                     const unsigned char* it_cancel, const int* rcount, const int* csr_off,
                                     const int* csr_cell, const int* conn8, const unsigned char* cell_nv,
                                     const int* iblank, int* iblank_cell);
__global__ void k_gather_cells_i32(const int* src, const int* inv, long long base, int n, int* out);
__global__ void k_interp_gather(const int* it_node, const double* it_w, const int* it_don,
                                const unsigned char* it_nv, const unsigned char* it_cancel,
                                const int* rcount, const BlockInfo* bi, const double* const* qptr, int nvar,
                                int interptype, double* vals);
__global__ void k_interp_scatter(const int* it_rec, const unsigned char* it_cancel, const int* rcount,
                                 const blk_t* node_blk, const BlockInfo* bi, const double* vals,
                                 int nvar, int interptype, double* const* qptr);

}  // namespace tb
