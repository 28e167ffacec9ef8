// The TIOGA C ABI (src/tiogaInterface.C:36-328) over the B200 engine.  One
// global instance, like TIOGA's `tg` (src/globals.h:31): the interface is not
// reentrant.
#include <stdarg.h>
#include <string.h>

#include "engine.h"

#pragma GCC visibility push(default)
#include "../../include/tioga_b200.h"

namespace {
tb::Engine* g_tg = nullptr;
int g_err = 0;
int g_dev_ok = -1;

bool device_ok() {
  if (g_dev_ok < 0) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    g_dev_ok = (e == cudaSuccess && n > 0) ? 1 : 0;
    if (!g_dev_ok)
      fprintf(stderr, "#tioga_b200: no CUDA device (%s); the GPU library cannot run\n",
              cudaGetErrorString(e));
  }
  return g_dev_ok == 1;
}

bool ready(const char* fn) {
  if (!g_tg) {
    fprintf(stderr, "#tioga_b200: %s called before tioga_init_\n", fn);
    g_err = -2;
    return false;
  }
  return true;
}

void set_rc(int rc) { g_err = rc; }

void register_va(int btag, int nnodes, double* xyz, int* ibl, int nwbc, int nobc, int* wbc, int* obc,
                 int ntypes, va_list ap) {
  if (!ready("tioga_registergrid_data")) return;
  int nv[4] = {0, 0, 0, 0}, nc[4] = {0, 0, 0, 0};
  int* conn[4] = {nullptr, nullptr, nullptr, nullptr};
  if (ntypes < 1 || ntypes > 4) {
    fprintf(stderr, "#tioga_b200: %d cell types (1..4 supported)\n", ntypes);
    g_err = -3;
    return;
  }
  for (int i = 0; i < ntypes; i++) {
    nv[i] = *va_arg(ap, int*);
    nc[i] = *va_arg(ap, int*);
    conn[i] = va_arg(ap, int*);
  }
  set_rc(g_tg->register_block_sys(g_tg->selected_system(), btag, nnodes, xyz, ibl, nwbc, nobc, wbc, obc, ntypes,
                                  nv, nc, conn));
}

void unsupported(const char* fn) {
  fprintf(stderr, "#tioga_b200: %s is outside the accelerated path and not supported\n", fn);
  g_err = -4;
}
}  // namespace

extern "C" {

void tioga_init_(intptr_t comm) {
  (void)comm;
  g_err = 0;
  if (!device_ok()) {
    g_err = -1;
    return;
  }
  delete g_tg;
  g_tg = new tb::Engine();
}

void tioga_init_f90_(int* scomm) {
  (void)scomm;
  tioga_init_(0);
}

void tioga_registergrid_data_(int* btag, int* nnodes, double* xyz, int* ibl, int* nwbc, int* nobc,
                              int* wbcnode, int* obcnode, int* ntypes, ...) {
  va_list ap;
  va_start(ap, ntypes);
  register_va(*btag, *nnodes, xyz, ibl, *nwbc, *nobc, wbcnode, obcnode, *ntypes, ap);
  va_end(ap);
}

void tioga_registergrid_data_mb_(int* bid, int* btag, int* nnodes, double* xyz, int* ibl, int* nwbc,
                                 int* nobc, int* wbcnode, int* obcnode, int* ntypes, ...) {
  (void)bid;  // blocks are identified by their mesh tag (tioga.C:68-80)
  va_list ap;
  va_start(ap, ntypes);
  register_va(*btag, *nnodes, xyz, ibl, *nwbc, *nobc, wbcnode, obcnode, *ntypes, ap);
  va_end(ap);
}

void tioga_b200_registergrid_sys_(int* sys, int* btag, int* nnodes, double* xyz, int* ibl, int* nwbc, int* nobc,
                                  int* wbcnode, int* obcnode, int* ntypes, ...) {
  if (!ready("tioga_b200_registergrid_sys_")) return;
  g_tg->select_system(*sys);
  va_list ap;
  va_start(ap, ntypes);
  register_va(*btag, *nnodes, xyz, ibl, *nwbc, *nobc, wbcnode, obcnode, *ntypes, ap);
  va_end(ap);
}

void tioga_b200_select_system_(int* sys) {
  if (ready("tioga_b200_select_system_")) g_tg->select_system(*sys);
}

int tioga_b200_nsystems_(void) { return g_tg ? g_tg->nsystems() : 0; }

void tioga_preprocess_grids_(void) {
  if (ready("tioga_preprocess_grids_")) set_rc(g_tg->preprocess());
}

void tioga_performconnectivity_(void) {
  if (ready("tioga_performconnectivity_")) set_rc(g_tg->connectivity());
}

void tioga_registersolution_(int* btag, double* q) {
  if (ready("tioga_registersolution_")) set_rc(g_tg->register_solution(*btag, q, false));
}

void tioga_dataupdate_mb_(int* nvar, char* itype) {
  if (!ready("tioga_dataupdate_mb_")) return;
  int t;
  if (strstr(itype, "row")) t = 0;
  else if (strstr(itype, "column")) t = 1;
  else {
    printf("#tiogaInterface.C:dataupdate_:unknown data orientation\n");
    return;
  }
  // after high-order registration the update goes to the points (tiogaInterface.C:194-214)
  if (g_tg->ihigh_global()) set_rc(g_tg->dataupdate_highorder(*nvar, t));
  else set_rc(g_tg->dataupdate(*nvar, t));
}

void tioga_dataupdate_(double* q, int* nvar, char* itype) {
  if (!ready("tioga_dataupdate_")) return;
  // TIOGA registers q under mesh tag 0, which no block has; bind it to the
  // first block instead.
  if (g_tg->nblocks() < 1) return;
  int tag = g_tg->first_tag();
  int rc = g_tg->register_solution(tag, q, false);
  if (rc) {
    set_rc(rc);
    return;
  }
  tioga_dataupdate_mb_(nvar, itype);
}

void tioga_getdonorcount_(int* btag, int* dcount, int* fcount) {
  *dcount = *fcount = 0;
  if (ready("tioga_getdonorcount_")) set_rc(g_tg->donor_count(*btag, dcount, fcount));
}

void tioga_getdonorinfo_(int* btag, int* receptors, int* indices, double* frac, int* dcount) {
  (void)dcount;
  if (ready("tioga_getdonorinfo_")) set_rc(g_tg->donor_info(*btag, receptors, indices, frac));
}

void tioga_b200_registercellgid_(int* btag, uint64_t* cell_gid) {
  if (ready("tioga_b200_registercellgid_")) set_rc(g_tg->set_cell_gid(*btag, cell_gid));
}

void tioga_b200_getreceptorcount_(int* nreceptors) {
  *nreceptors = 0;
  if (!ready("tioga_b200_getreceptorcount_")) return;
  const long long n = g_tg->receptor_info(nullptr, 0);
  set_rc(n < 0 ? -1 : 0);
  if (n > 0) *nreceptors = (int)(n / 4);
}

void tioga_b200_getreceptorinfo_(int* receptors) {
  if (!ready("tioga_b200_getreceptorinfo_")) return;
  const long long n = g_tg->receptor_info(receptors, 1ll << 62);
  set_rc(n < 0 ? -1 : 0);
}

void tioga_setsymmetry_(int* isym) {
  if (ready("tioga_setsymmetry_")) g_tg->set_symmetry(*isym);
}
void tioga_setnfringe_(int* nfringe) {
  if (ready("tioga_setnfringe_")) g_tg->set_nfringe(*nfringe);
}
void tioga_setmexclude_(int* mexclude) {
  if (ready("tioga_setmexclude_")) g_tg->set_mexclude(*mexclude);
}
void tioga_setresolutions_(double* nres, double* cres) {
  if (ready("tioga_setresolutions_") && g_tg->nblocks() > 0)
    set_rc(g_tg->set_resolutions(g_tg->first_tag(), nres, cres));
}
void tioga_setresolutions_multi_(int* btag, double* nres, double* cres) {
  if (ready("tioga_setresolutions_multi_")) set_rc(g_tg->set_resolutions(*btag, nres, cres));
}
void tioga_setcelliblank_(int* iblank_cell) {
  if (ready("tioga_setcelliblank_") && g_tg->nblocks() > 0)
    set_rc(g_tg->set_cell_iblank(g_tg->first_tag(), iblank_cell));
}

void tioga_delete_(void) {
  delete g_tg;
  g_tg = nullptr;
}

void tioga_performconnectivity_highorder_(void) {
  if (ready("tioga_performconnectivity_highorder_")) set_rc(g_tg->connectivity_highorder());
}
void tioga_performconnectivity_amr_(void) { unsupported("tioga_performconnectivity_amr_"); }
void tioga_register_amr_global_data_(int*, int*, double*, int*, double*, int*, int*) {
  unsupported("tioga_register_amr_global_data_");
}
void tioga_register_amr_patch_count_(int*) { unsupported("tioga_register_amr_patch_count_"); }
void tioga_register_amr_local_data_(int*, int*, int*, double*) { unsupported("tioga_register_amr_local_data_"); }
void tioga_set_p4est_(void) { unsupported("tioga_set_p4est_"); }
void tioga_set_amr_callback_(void (*)(int*, double*, int*, double*)) { unsupported("tioga_set_amr_callback_"); }
void tioga_set_p4est_search_callback_(void (*)(double*, int*, int*, int*), void (*)(int*, int*)) {
  unsupported("tioga_set_p4est_search_callback_");
}
// The callbacks are recorded (they switch the data update to the point
// form, as in tioga.h:211-223), but a device search cannot call host code:
// the elements must also be described with tioga_b200_set_highorder_lagrange_.
void tioga_set_highorder_callback_(void (*)(int*, int*), void (*)(int*, int*, double*),
                                   void (*)(int*, double*, int*, double*),
                                   void (*)(int*, double*, int*, int*, double*, double*, int*),
                                   void (*)(int*, int*, double*, int*, int*, double*)) {
  if (ready("tioga_set_highorder_callback_")) g_tg->set_highorder_callbacks();
}
void tioga_b200_set_highorder_lagrange_(int* btag, int* order, double* xdof) {
  if (ready("tioga_b200_set_highorder_lagrange_")) set_rc(g_tg->set_highorder(*btag, *order, xdof));
}
int tioga_b200_pointdonors_(int* btag, int* out, double* w) {
  if (!ready("tioga_b200_pointdonors_")) return 0;
  return g_tg->point_donors(*btag, out, w);
}
void tioga_b200_highorder_stats_(long long out[8]) {
  for (int i = 0; i < 8; i++) out[i] = 0;
  if (!g_tg) return;
  const tb::HoStats& s = g_tg->ho_stats();
  out[0] = s.npoints;
  out[1] = s.ndonor;
  out[2] = s.nties;
  out[3] = s.nrecords;
  out[4] = s.nmerged;
  out[5] = s.norphan_cells;
  out[6] = s.ncand;
  out[7] = s.nrefine;
}
void tioga_reduce_fringes_(void) {
  if (ready("tioga_reduce_fringes_")) set_rc(g_tg->reduce_fringes());
}
void tioga_writeoutputfiles_(int* nvar, char* itype) {
  if (!ready("tioga_writeoutputfiles_")) return;
  int t;
  if (strstr(itype, "row")) t = 0;
  else if (strstr(itype, "column")) t = 1;
  else {
    printf("#tiogaInterface.C:dataupdate_:unknown data orientation\n");
    return;
  }
  set_rc(g_tg->write_output(*nvar, t));
}

int tioga_b200_last_error(void) { return g_err; }
int tioga_b200_device_ok(void) { return device_ok() ? 1 : 0; }

void tioga_b200_set_precision_(int* mode) {
  if (ready("tioga_b200_set_precision_")) g_tg->set_precision(*mode);
}
void tioga_b200_set_coords_resident_(int* flag) {
  if (ready("tioga_b200_set_coords_resident_")) g_tg->set_coords_resident(*flag);
}
void tioga_b200_registersolution_device_(int* btag, double* dq) {
  if (ready("tioga_b200_registersolution_device_")) set_rc(g_tg->register_solution(*btag, dq, true));
}
void tioga_b200_registeriblank_device_(int* btag, int* d_ibl) {
  if (ready("tioga_b200_registeriblank_device_")) set_rc(g_tg->register_iblank_device(*btag, d_ibl));
}
void tioga_b200_getcelliblank_(int* btag, int* out) {
  if (ready("tioga_b200_getcelliblank_")) set_rc(g_tg->cell_iblank(*btag, out));
}

void tioga_b200_stats_(long long out[16]) {
  for (int i = 0; i < 16; i++) out[i] = 0;
  if (!g_tg) return;
  const tb::Stats& s = g_tg->stats();
  out[0] = s.nquery;
  out[1] = s.ndonor;
  out[2] = s.nties;
  out[3] = s.ncand;
  out[4] = s.nrefine;
  out[5] = s.nreceptor;
  out[6] = s.nhole;
  out[7] = s.nrecords;
  out[8] = s.error;
  out[9] = s.npairs;
  out[10] = s.launches;
  out[11] = s.cand_verts;
  out[12] = s.nleaf;
  out[13] = s.nmerged;
}

void tioga_b200_registernodegid_(int* btag, uint64_t* node_gid) {
  if (ready("tioga_b200_registernodegid_")) set_rc(g_tg->set_node_gid(*btag, node_gid));
}

void tioga_b200_set_pin_host_(int* on) {
  if (ready("tioga_b200_set_pin_host_")) {
    g_tg->set_pin_host(*on);
    set_rc(0);
  }
}

void tioga_b200_set_nodegid_merge_(int* on) {
  if (ready("tioga_b200_set_nodegid_merge_")) {
    g_tg->set_nodegid_merge(*on);
    set_rc(0);
  }
}

void tioga_b200_set_uniform_hex_flag_(int* btag, int* flag) {
  if (ready("tioga_b200_set_uniform_hex_flag_")) set_rc(g_tg->set_uniform_hex_flag(*btag, *flag));
}

void tioga_b200_set_test_bound_(int* which, int* value) {
  if (ready("tioga_b200_set_test_bound_")) set_rc(g_tg->set_test_bound(*which, *value));
}

void tioga_b200_stats2_(long long out[8]) {
  for (int i = 0; i < 8; i++) out[i] = 0;
  if (!g_tg) return;
  out[0] = g_tg->stats().holemap_cells;
}

void tioga_b200_autotune_(int* reps) {
  if (ready("tioga_b200_autotune_")) set_rc(g_tg->autotune(*reps));
}

void tioga_b200_tuning_(int out[8]) {
  for (int i = 0; i < 8; i++) out[i] = 0;
  if (!g_tg) return;
  const tb::Tuning& t = g_tg->tuning();
  out[0] = t.cell_pass_per_sm;
  out[1] = t.chunk_pairs;
  out[2] = t.query_per_sm;
  out[3] = t.traverse_per_sm;
  out[4] = t.candidates_per_sm;
  out[5] = t.cell_box_per_sm;
  out[6] = t.traverse_variant;
}

void tioga_b200_set_tuning_(const int in[7]) {
  if (!ready("tioga_b200_set_tuning_")) return;
  set_rc(g_tg->set_tuning(in));
}

void tioga_b200_set_stream_(void* stream) {
  if (ready("tioga_b200_set_stream_")) g_tg->set_stream((cudaStream_t)stream);
}

void tioga_b200_timing_(float out[16]) {
  for (int i = 0; i < 16; i++) out[i] = 0;
  if (!g_tg) return;
  const tb::Timing& t = g_tg->timing();
  out[0] = t.upload;
  out[1] = t.holemap;
  out[2] = t.boxes;
  out[3] = t.query;
  out[4] = t.search;
  out[5] = t.donors;
  out[6] = t.celliblank;
  out[7] = t.download;
  out[8] = t.total;
  out[9] = t.traverse;
  out[10] = t.candidates;
  out[11] = t.refine;
  out[12] = t.cell_pass;
  out[13] = t.cell_boxes;
}

}  // extern "C"

#pragma GCC visibility pop
