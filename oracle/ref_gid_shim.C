// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// Two entry points linked into _ref/libtioga_ref.so, so that the tests can
// drive the reference's cell-global-id path, which only its C++ class offers,
// through ctypes:
//   refshim_registergrid_gid_  the arguments of tioga_registergrid_data_mb_
//                              (src/tiogaInterface.C:107-129) with the cell
//                              global ids in front, handed to
//                              tioga::registerGridData (src/tioga.C:64-85)
//   refshim_registergrid_gids_ the same with the nodes' global ids too, for the
//                              reference built with TIOGA_HAS_NODEGID
//                              (_ref/libtioga_ref_nodegid.so)
//   refshim_getreceptorinfo_   tioga::getReceptorInfo (src/tioga.C:572-671)
//   refshim_set_uniform_hex_flag_  tioga::set_uniform_hex_flag (src/tioga.h:195-201),
//                              the uniform-hex search's switch
// The instance is the C API's own (the global `tg` of src/globals.h), so the
// rest of a test drives the reference through its C API as usual.
#include <algorithm>
#include <cstdarg>
#include <cstdint>
#include <cstring>
#include <vector>

#include "tioga.h"

extern TIOGA::tioga* tg;

namespace {
struct Registration {  // what the block's MeshBlock keeps pointers to
  std::vector<int> nv, nc;
  std::vector<int*> conn;
};
Registration g_reg[128];
std::vector<int> g_receptors;
}  // namespace

namespace {
void register_gids(uint64_t* cell_gid, uint64_t* node_gid, int* bid, int* btag, int* nnodes, double* xyz, int* ibl,
                   int* nwbc, int* nobc, int* wbcnode, int* obcnode, int* ntypes, va_list args) {
  Registration& R = g_reg[*bid - 1];
  std::vector<int> nv(*ntypes), nc(*ntypes);
  std::vector<int*> conn(*ntypes);
  for (int t = 0; t < *ntypes; t++) {
    nv[t] = *va_arg(args, int*);
    nc[t] = *va_arg(args, int*);
    conn[t] = va_arg(args, int*);
  }
  R.nv.swap(nv);
  R.nc.swap(nc);
  R.conn.swap(conn);
  tg->registerGridData(*btag, *nnodes, xyz, ibl, *nwbc, *nobc, wbcnode, obcnode, *ntypes, R.nv.data(), R.nc.data(),
                       R.conn.data(), cell_gid, node_gid);
}
}  // namespace

extern "C" {

void refshim_registergrid_gid_(uint64_t* cell_gid, int* bid, int* btag, int* nnodes, double* xyz, int* ibl,
                               int* nwbc, int* nobc, int* wbcnode, int* obcnode, int* ntypes, ...) {
  va_list args;
  va_start(args, ntypes);
  register_gids(cell_gid, nullptr, bid, btag, nnodes, xyz, ibl, nwbc, nobc, wbcnode, obcnode, ntypes, args);
  va_end(args);
}

// the same with the nodes' global ids as well (registerGridData's node_gid,
// which a build with TIOGA_HAS_NODEGID requires, MeshBlock.C:68-71)
void refshim_registergrid_gids_(uint64_t* cell_gid, uint64_t* node_gid, int* bid, int* btag, int* nnodes,
                                double* xyz, int* ibl, int* nwbc, int* nobc, int* wbcnode, int* obcnode, int* ntypes,
                                ...) {
  va_list args;
  va_start(args, ntypes);
  register_gids(cell_gid, node_gid, bid, btag, nnodes, xyz, ibl, nwbc, nobc, wbcnode, obcnode, ntypes, args);
  va_end(args);
}

// The number of ints getReceptorInfo returns (four per receptor); the first
// min(count, cap) of them are copied to out when out is not null.
int refshim_getreceptorinfo_(int* out, int cap) {
  g_receptors.clear();
  tg->getReceptorInfo(g_receptors);
  const int n = (int)g_receptors.size();
  if (out && n > 0) std::memcpy(out, g_receptors.data(), sizeof(int) * std::min(n, cap));
  return n;
}

void refshim_set_uniform_hex_flag_(int* btag, int* flag) { tg->set_uniform_hex_flag(*btag, *flag); }

}  // extern "C"
