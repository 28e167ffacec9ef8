/*
 * tioga_b200 -- the TIOGA overset-connectivity C API on a B200 GPU.
 *
 * libtioga_b200.so exports the symbols of TIOGA's C/Fortran interface
 * (src/tiogaInterface.C in the TIOGA sources), so a solver that links
 * against TIOGA links against this library unchanged.  Every scalar is passed
 * by pointer (Fortran binding), connectivity and boundary-node lists are
 * 1-based, and every array stays the caller's: the library keeps the
 * pointers and reads coordinates again at each preprocess/connectivity call.
 * All mesh blocks live on one GPU; TIOGA's MPI exchanges are device-buffer
 * hand-offs inside the library.
 *
 * Errors: the TIOGA functions return void, as in TIOGA.  A failure prints a
 * "#tioga_b200:" line on stderr and is kept for tioga_b200_last_error().
 * The library never aborts the process and never traps on the device.
 */
#ifndef TIOGA_B200_H
#define TIOGA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- TIOGA's interface (src/tiogaInterface.C) -------------------------- */

/* tiogaInterface.C:38 -- Fortran communicator handle; one rank, ignored. */
void tioga_init_f90_(int *scomm);
/* tiogaInterface.C:61 -- MPI_Comm is an int (MPICH) or a pointer (Open MPI):
 * taken as an opaque word and ignored (one rank). */
void tioga_init_(intptr_t comm);

/* tiogaInterface.C:84-105 -- register a block; the varargs are *ntypes
 * triples (int *nv, int *nc, int *vconn) with nv in {4,5,6,8}. */
void tioga_registergrid_data_(int *btag, int *nnodes, double *xyz, int *ibl, int *nwbc, int *nobc,
                              int *wbcnode, int *obcnode, int *ntypes, ...);
/* tiogaInterface.C:108-130 -- the same with an explicit 1-based block id. */
void tioga_registergrid_data_mb_(int *bid, int *btag, int *nnodes, double *xyz, int *ibl, int *nwbc,
                                 int *nobc, int *wbcnode, int *obcnode, int *ntypes, ...);

/* tiogaInterface.C:150-153 -- cell volumes, node resolutions, mandatory
 * receptors, oriented boxes; sets every iblank to 1. */
void tioga_preprocess_grids_(void);
/* tiogaInterface.C:155-158 -- hole maps, box pairs, donor search, donor
 * selection and cancellation; writes ibl[] in {1, 0, -1}. */
void tioga_performconnectivity_(void);

/* tiogaInterface.C:170-173 -- bind block btag's solution (host array,
 * updated in place by the next data update). */
void tioga_registersolution_(int *btag, double *q);
/* tiogaInterface.C:175-216 -- interpolate nvar fields into every receptor;
 * itype contains "row" (q[node*nvar+k]) or "column" (q[k*nnodes+node]). */
void tioga_dataupdate_mb_(int *nvar, char *itype);
/* tiogaInterface.C:218-224 -- TIOGA looks up mesh tag 0 here, which never
 * exists; this library binds q to the first registered block. */
void tioga_dataupdate_(double *q, int *nvar, char *itype);

/* tiogaInterface.C:244-251 -- donor stencils held by block btag: dcount
 * receptors and fcount = sum(nweights + 1) indices/weights. */
void tioga_getdonorcount_(int *btag, int *dcount, int *fcount);
/* receptors[4*i..] = {rank, receptor node, receptor block, nweights};
 * indices: donor nodes then the donor cell id; frac: weights then 0. */
void tioga_getdonorinfo_(int *btag, int *receptors, int *indices, double *frac, int *dcount);

/* tiogaInterface.C:253-316 -- settings */
void tioga_setsymmetry_(int *isym);
void tioga_setresolutions_(double *nres, double *cres);
void tioga_setresolutions_multi_(int *btag, double *nres, double *cres);
void tioga_setcelliblank_(int *iblank_cell);
void tioga_setnfringe_(int *nfringe);
void tioga_setmexclude_(int *mexclude);
/* tiogaInterface.C:317-326 */
void tioga_delete_(void);

/* tiogaInterface.C:160-163: the high-order connectivity (tioga.C:162-178):
 * the points of every receptor cell (cell iblank -1 after the last
 * performconnectivity) are searched in the donor blocks, and points whose
 * donor is a field cell get interpolation weights.  The following
 * tioga_dataupdate_mb_ then interpolates at those points (ROW solutions,
 * element-major DOFs) and updates the receptor cells (highOrder.C:152-566).
 * Every block's elements must be described with
 * tioga_b200_set_highorder_lagrange_. */
void tioga_performconnectivity_highorder_(void);
/* tiogaInterface.C:273-285.  Recorded (it switches the data update to the
 * point form), but the solver's host callbacks cannot run in the device
 * search; describe the elements with tioga_b200_set_highorder_lagrange_. */
void tioga_set_highorder_callback_(void (*f1)(int *, int *), void (*f2)(int *, int *, double *),
                                   void (*f3)(int *, double *, int *, double *),
                                   void (*f4)(int *, double *, int *, int *, double *, double *, int *),
                                   void (*f5)(int *, int *, double *, int *, int *, double *));

/* tiogaInterface.C:302-305 -- after performconnectivity: keep only the
 * receptors within nfringe+1 layers of the field nodes (tioga.C:737-885,
 * bookKeeping.C:650-760); the others' interpolations are cancelled and
 * they become holes.  ibl[] is rewritten; the cell iblanks stay as the
 * connectivity call left them, as in TIOGA. */
void tioga_reduce_fringes_(void);

/* tiogaInterface.C:226-243 -- one Tecplot file per block, flowNNNNN.dat by
 * block index (tioga.C:526-531, MeshBlock.C:510-635): coordinates, iblank,
 * mesh tag and the registered solution per node, then the cells as bricks
 * and the wall and overset-boundary node lists; same formats as TIOGA.
 * Every block's solution must be registered. */
void tioga_writeoutputfiles_(int *nvar, char *itype);

/* Entry points of TIOGA outside the accelerated path (AMR/Cartesian,
 * p4est; tiogaInterface.C:132-148, 287-299, and the AMR connectivity).
 * They are exported so that existing solvers link; each reports "not
 * supported" and sets the last error. */
void tioga_performconnectivity_amr_(void);
void tioga_register_amr_global_data_(int *nf, int *qstride, double *qnodein, int *idata, double *rdata,
                                     int *ngridsin, int *qnodesize);
void tioga_register_amr_patch_count_(int *npatches);
void tioga_register_amr_local_data_(int *ipatch, int *global_id, int *iblank, double *q);
void tioga_set_p4est_(void);
void tioga_set_amr_callback_(void (*f1)(int *, double *, int *, double *));
void tioga_set_p4est_search_callback_(void (*f1)(double *xsearch, int *process_id, int *cell_id, int *npts),
                                      void (*f2)(int *pid, int *iflag));

/* ---- additions of this library (no counterpart in TIOGA) -------------- */

/* The elements of block btag for the high-order path, in place of the
 * solver callbacks: Lagrange hexahedra of degree `order` (1..10) with
 * equispaced nodes.  xdof holds every cell's (order+1)^3 DOF coordinates,
 * cell after cell in the block's cell order, tensor order within a cell
 * (node (i, j, k) at ((k (order+1) + j) (order+1) + i), reference point
 * (i, j, k) / order, i along the cell's first corner edge v0->v1, j along
 * v0->v3, k along v0->v4).  Caller-owned like the coordinates, read again by
 * every tioga_performconnectivity_highorder_.  The solution arrays of the
 * high-order data update are laid out the same way, nvar values per DOF.
 * What the device computes is what such callbacks would: the cell's DOFs
 * as its receptor points, Newton inversion of the element map from the
 * centre (|update| < 1e-14 within 50 steps) as the inclusion test with
 * r, s, t in [-1e-10, 1 + 1e-10], the basis at the inverted point as the
 * weights, and nodal values written back unchanged. */
void tioga_b200_set_highorder_lagrange_(int *btag, int *order, double *xdof);
/* Point donors of donor block btag after the high-order connectivity, in
 * its list order: out[4 i ..] = (receptor block index, point index in that
 * block, donor cell, weight count), w[1331 i ..] = weights.  Returns the
 * count; out or w may be NULL. */
int tioga_b200_pointdonors_(int *btag, int *out, double *w);
/* High-order counters: [0] query points, [1] with a donor, [2] ties,
 * [3] interpolation records, [4] coincident points merged, [5] receptor
 * cells changed by the orphan rule in the last data update, [6] inclusion
 * tests (candidates whose box holds the point), [7] of those decided by the
 * FP64 Newton (all of them in the FP64 form; in the split form the rest are
 * clear cases of an FP32 Newton). */
void tioga_b200_highorder_stats_(long long out[8]);

/* Batched form: the blocks of many independent overset systems in one
 * instance, in place of the reference's one system per init ... delete
 * sequence (driver/poisson_mms.f90:111-253 re-initialises per system).
 * Registers a block of system *sys (>= 0) with the arguments of
 * tioga_registergrid_data_ (src/tiogaInterface.C:84-105, cell types as the
 * trailing varargs triples).  Each system has its own mesh tags and is
 * connected exactly as if it were alone (pairs, hole maps, donor lists and
 * iblank -meshtag values never cross systems), while every stage of
 * preprocess, connectivity and data update is one launch over all systems.
 * At most 16 blocks per system and 8192 in all; the high-order path takes
 * one system per instance. */
void tioga_b200_registergrid_sys_(int *sys, int *btag, int *nnodes, double *xyz, int *ibl, int *nwbc,
                                  int *nobc, int *wbcnode, int *obcnode, int *ntypes, ...);
/* The system whose mesh tags the tag-based calls (registergrid_data_,
 * registersolution_, setresolutions_multi_, getdonorcount_/getdonorinfo_,
 * the tioga_b200_ block calls) address from now on; 0 by default. */
void tioga_b200_select_system_(int *sys);
/* Systems registered in the instance. */
int tioga_b200_nsystems_(void);

/* Cell global ids of block btag: one uint64_t per cell in registration
 * order, the cell_gid argument of the C++ tioga::registerGridData
 * (src/tioga.h:121-123, kept by MeshBlock::setData, src/MeshBlock.C:60),
 * which the C API does not pass.  The array stays the caller's; registering
 * the block again clears it, as registerGridData without ids does. */
void tioga_b200_registercellgid_(int *btag, uint64_t *cell_gid);
/* tioga::getReceptorInfo (src/tioga.C:572-671) of the selected system, for
 * C callers: the count of receptors it returns, then their records, four
 * ints each.  Donor blocks come in registration order and each block's live
 * interpolation records in list order (MeshBlock::getReceptorInfo,
 * src/dataUpdate.C:161-178): receptor node (0-based), mesh tag of the
 * receptor block, and the donor cell's global id as two ints (its eight
 * bytes copied, low word first on a little-endian host).  A donating block
 * without cell ids is an error (tioga_b200_last_error() != 0); the reference
 * reads through a null pointer there. */
void tioga_b200_getreceptorcount_(int *nreceptors);
void tioga_b200_getreceptorinfo_(int *receptors);

/* Serving form: a request loop over many resident systems, each request
 * one time step of one system (the per-step sequence preprocess ->
 * performconnectivity -> dataupdate of src/tiogaInterface.C:150-216 for that
 * system alone).  Independent of the global instance above; thread-safe.
 * `nslots` requests run at once (each on its own CUDA stream), taken in
 * arrival order as slots free up; a system is made resident (its topology,
 * cell trees, hole maps and coordinates kept on the device between its
 * requests) when it fits `hbm_budget_bytes` and at most `max_resident`
 * systems are resident; idle systems are evicted least recently used first
 * (their device coordinates written back to the caller's xyz arrays).
 * Requests of one system run in submission order, one at a time.  Device
 * buffers come from the server's own stream-ordered memory pool, which
 * reserves min(hbm_budget_bytes, free device memory - 2 GiB) at creation
 * and keeps what is freed, so requests do not wait on pool growth.  Returns
 * NULL without a CUDA device. */
void *tioga_b200_server_create(long long hbm_budget_bytes, int nslots, int max_resident);
void tioga_b200_server_destroy(void *srv);
/* A block of system `sys`, with tioga_registergrid_data_'s arguments by
 * value (vconn[t]: the t-th cell type's 1-based connectivity).  The arrays
 * stay the caller's and must outlive the server; blocks are added before
 * the system's first request. */
int tioga_b200_server_add_block(void *srv, int sys, int btag, int nnodes, double *xyz, int *ibl, int nwbc, int nobc,
                                int *wbcnode, int *obcnode, int ntypes, const int *nv, const int *nc,
                                int *const *vconn);
/* One time step of system `sys`: the rigid motions x <- A x + b of the
 * blocks move_tags[0..nmoves) (moves[12 m ..]: A row-major, then b; applied
 * on the device to the resident coordinates, each component evaluated as
 * ((A[k][0] x + A[k][1] y) + A[k][2] z) + b[k]), then preprocess,
 * connectivity, and, when q is given, the data update of nvar fields in
 * the ROW layout into q[block] (blocks in the order they were added).
 * iblank goes to ibl_out[block] when given, else to the arrays given at
 * add_block.  The arrays must stay untouched until the request is waited
 * for.  Returns a ticket (> 0) or -1. */
long long tioga_b200_server_submit(void *srv, int sys, int nmoves, const int *move_tags, const double *moves,
                                   int nvar, double *const *q, int *const *ibl_out);
/* The same with the fields on the device when q_on_device is 1 (a GPU
 * solver's arrays, same layout): the data update then reads and writes them
 * in place, with no host copies. */
long long tioga_b200_server_submit_fields(void *srv, int sys, int nmoves, const int *move_tags, const double *moves,
                                          int nvar, double *const *q, int q_on_device, int *const *ibl_out);
/* Blocks until the request is done: times_ms = (submit -> done, submit ->
 * start, start -> done, then the host time of its preprocess, connectivity
 * and data update), counts = (query points, receptors, holes, status).
 * Returns the request's status: 0 = success, a negative engine error code,
 * -3 = the system alone needs more device memory than the budget (refused,
 * nothing ran), -4 = cancelled before it started; -1 for an unknown ticket. */
int tioga_b200_server_wait(void *srv, long long ticket, double times_ms[6], long long counts[4]);
/* tioga_b200_server_wait for at most timeout_ms: -5 when the request is not
 * done by then (it goes on, and the ticket stays valid for another wait). */
int tioga_b200_server_wait_timeout(void *srv, long long ticket, double timeout_ms, double times_ms[6],
                                   long long counts[4]);
/* Cancel a request that has not started: it completes with status -4.
 * Returns 0, or -1 when the request is running, done or unknown. */
int tioga_b200_server_cancel(void *srv, long long ticket);
/* [0] resident systems, [1] device bytes they hold, [2] admissions,
 * [3] evictions, [4] completed requests, [5] queued requests, [6] budget,
 * [7] peak device bytes held, [8] bytes reserved in the server's memory
 * pool at creation, [9] bytes the pool holds now. */
void tioga_b200_server_stats(void *srv, long long out[16]);

/* Autotuner: after tioga_preprocess_grids_, times every launch shape of the
 * tuned kernels (CTAs per SM of the cell pass, with its register budget cut
 * to match; of the query gathering, the traversal and the candidate
 * screen; pairs per cell-pass CTA) over *reps
 * connectivity calls each, one knob after the other, and keeps the fastest
 * for the instance's later calls.  The results of a call do not depend on
 * the shapes; the instance ends with a connectivity call's results. */
void tioga_b200_autotune_(int *reps);
/* The shapes in use: [0] cell-pass CTAs per SM, [1] pairs per cell-pass CTA,
 * [2] query CTAs per SM, [3] traversal CTAs per SM, [4] candidate CTAs per SM,
 * [5] CTAs per SM of the split form's cell-box kernel, [6] the split form's
 * traversal: 0 walks and tests leaves as it meets them, 1 postpones leaves
 * until every lane of a warp holds one. */
void tioga_b200_tuning_(int out[8]);
/* Set the shapes by hand, in tioga_b200_tuning_'s order [0..6]; values <= 0
 * keep a shape, except [6], which takes the traversal variant plus one (1 or
 * 2; 0 keeps it). */
void tioga_b200_set_tuning_(const int in[7]);

/* 0 when the last call succeeded, else a negative code. */
int tioga_b200_last_error(void);
/* 1 when a CUDA device is present and the library initialised it. */
int tioga_b200_device_ok(void);
/* Search arithmetic: 0 = FP64 throughout; 1 (default) = FP32 tree boxes and
 * an FP32 screen of the Newton inversion with FP64 refinement of every
 * undecided candidate; 2 = as 1, and the high-order inclusion test also
 * screened in FP32 (clear outsiders rejected; every other candidate still
 * takes the FP64 test, whose fixed 1e-14 stopping rule must be replayed, so
 * on meshes whose candidates mostly pass this costs more than it saves).
 * Results are identical in every mode. */
void tioga_b200_set_precision_(int *mode);
/* 1: the coordinates have not moved since the last call, so connectivity
 * skips their upload.  Default 0 (TIOGA re-reads x at every call). */
void tioga_b200_set_coords_resident_(int *flag);
/* Bind block btag's solution as a DEVICE array (same layout as the host
 * one); tioga_dataupdate_mb_ then updates it without host copies. */
void tioga_b200_registersolution_device_(int *btag, double *dq);
/* Write block btag's node iblank into a DEVICE array of nnodes ints instead
 * of the host array given at registration (solvers that keep iblank on the
 * GPU); NULL returns to the host array. */
void tioga_b200_registeriblank_device_(int *btag, int *d_ibl);
/* Cell iblank of block btag (ncells ints), for any block. */
void tioga_b200_getcelliblank_(int *btag, int *iblank_cell);
/* Counters of the last connectivity call: [0] query points, [1] queries with
 * a donor, [2] order-dependent ties, [3] Newton candidates, [4] FP64
 * refinements, [5] receptors, [6] holes, [7] donor records, [8] device
 * error bits, [9] pairs of blocks, [10] kernels launched by the library,
 * [11] sum of the candidates' vertex counts, [12] leaves of the cell trees,
 * [13] query points merged into a coincident one (uniqNodesTree). */
void tioga_b200_stats_(long long out[16]);
/* More counters of the last connectivity call: [0] cells of its hole maps. */
void tioga_b200_stats2_(long long out[8]);
/* Run on the caller's CUDA stream (a cudaStream_t; NULL restores the
 * library's own stream), e.g. to time the calls with the caller's events. */
void tioga_b200_set_stream_(void *stream);
/* Interpolate nvar fields of a device array d_q in place from donor
 * stencils the caller keeps on the device, allocating no device memory
 * (no counterpart in TIOGA).  For callers that cannot allocate: a solver
 * whose time step runs inside a captured CUDA graph (cudaMalloc is not
 * allowed while a stream is captured), or one whose memory pool must not be
 * disturbed by cudaMalloc's device-wide synchronisation.  Stencil r has
 * d_nweights[r] entries, 1 to 8 (a record outside that range is ignored and
 * its receptor keeps its value), at d_inode[9r+m] (node index into d_q) with
 * weights d_weights[9r+m], and writes node d_receptor[r]; receptors must be
 * distinct (as getdonorinfo's are), or their writes race; interptype 0 is
 * row layout (q[node*nvar+k]), 1 column (q[k*nnodes+node]).  The
 * gather-to-scatter staging lives in a fixed device array of 2^20 doubles:
 * nrec*nvar above that is rejected (-1).  The first call on a device looks up
 * that array's address (make it before any stream capture); calls that
 * overlap on the GPU share the array and race.  Asynchronous on `stream`;
 * returns 0, -1 for bad arguments, -2 for a CUDA error. */
int tioga_b200_interpolate_noalloc_(const int *d_inode, const double *d_weights, const int *d_nweights,
                                    const int *d_receptor, int nrec, double *d_q, long long nnodes,
                                    int nvar, int interptype, void *stream);
/* Page-locking of the caller's arrays (on by default): at the next
 * preprocess that uploads the topology, pageable coordinate and iblank
 * arrays are registered with cudaHostRegister (they must stay valid anyway,
 * src/MeshBlock.C:37-72), so the copies of every connectivity call run at the
 * full PCIe rate; *on = 0 releases them and leaves arrays as they are. */
void tioga_b200_set_pin_host_(int *on);
/* Node global ids of block btag (nnodes uint64_t; caller-owned, kept like the
 * other registered arrays): the node_gid of tioga::registerGridData
 * (src/tioga.C:64-85), which the C API does not pass. */
void tioga_b200_registernodegid_(int *btag, uint64_t *node_gid);
/* *on = 1: coincident query points of a donor are merged by node global id
 * (uniquenode_map, src/search.C:48-74), as the reference built with
 * TIOGA_HAS_NODEGID does, instead of by the octree over their coordinates;
 * every block then needs its node ids (tioga_b200_registernodegid_).  The
 * high-order point search keeps the octree merge. */
void tioga_b200_set_nodegid_merge_(int *on);
/* tioga::set_uniform_hex_flag (src/tioga.h:195-201), which the reference
 * offers through its C++ class only: at the next preprocess, block btag is
 * tested for a box of identical rectangular hexahedra
 * (MeshBlock::check_for_uniform_hex, src/MeshBlock.C:1249-1372) and, when it
 * is one, searched by index lookup in a cell map instead of its tree
 * (MeshBlock::search_uniform_hex, src/search.C:271-341).  The high-order
 * point search keeps the tree for such blocks. */
void tioga_b200_set_uniform_hex_flag_(int *btag, int *flag);
/* For tests: lower one bound to *value (0 restores it).  *which 0 = line
 * passes of a hole-map fill (at the bound the fill stops and error bit 8 is
 * reported), 1 = donor-record capacity (error bit 2); the connectivity call
 * then returns its error bits through tioga_b200_last_error().  2 = nodes
 * per chunk of the split form's chunked coordinate upload (from the next
 * preprocess), to run it over many chunks on small meshes.  No counterpart
 * in TIOGA. */
void tioga_b200_set_test_bound_(int *which, int *value);
/* Device time (ms) of the last connectivity call per phase: [0] coordinate
 * upload, [1] hole maps, [2] box pairs + tree refit, [3] query gather,
 * [4] search, [5] donor bookkeeping, [6] cell iblank, [7] iblank download,
 * [8] total; inside the search: [9] traversal, [10] candidate screen,
 * [11] FP64 refinement; [12] the cell pass alone (cell and leaf boxes,
 * reduced boxes), inside [2]; [13] the split form's cell-box kernel alone,
 * inside [12]. */
void tioga_b200_timing_(float out[16]);

#ifdef __cplusplus
}
#endif

#endif /* TIOGA_B200_H */
