// data_cgx.cc -- data<CCTK_REAL8>::transfer_from_innerloop through libcgx:
// the body CarpetLib's data.cc (CarpetLib/src/data.cc:465-483) gets when its
// grid functions are device-resident.  A maintainer puts this specialisation
// into CarpetLib/src/data.cc (before the explicit instantiations at its end)
// and links libcgx.so; it compiles against CarpetLib's own headers (the
// oracle's shim stands in for the Cactus flesh when building it standalone:
// tests/test_carpet_shim.py).
//
// Residency: storage() must be a device pointer here, i.e. the grid
// function's memory lives in HBM (Carpet's Accelerator_* aliased functions
// track where the valid copy is; Carpet/src/Comm.cc:215-250).
#include <cctk.h>

#include <vector>

#include "data.hh"
#include "operators.hh"

#include "cgx_carpet.hh"

namespace CarpetLib {

// CarpetLib's numbering is the C-ABI's
static_assert(int(op_error) == CGX_OP_ERROR && int(op_none) == CGX_OP_NONE && int(op_sync) == CGX_OP_SYNC &&
                  int(op_restrict) == CGX_OP_RESTRICT && int(op_copy) == CGX_OP_COPY &&
                  int(op_Lagrange) == CGX_OP_LAGRANGE && int(op_ENO) == CGX_OP_ENO &&
                  int(op_WENO) == CGX_OP_WENO && int(op_TVD) == CGX_OP_TVD &&
                  int(op_Lagrange_monotone) == CGX_OP_LAGRANGE_MONOTONE,
              "operator_type values");
static_assert(int(vertex_centered) == CGX_VERTEX && int(cell_centered) == CGX_CELL, "centering values");

template <>
void data<CCTK_REAL8>::transfer_from_innerloop(vector<gdata const *> const &gsrcs,
                                               vector<CCTK_REAL> const &times, ibbox const &dstbox,
                                               ibbox const &srcbox, islab const *restrict const slabinfo,
                                               CCTK_REAL const time, int const order_space,
                                               int const order_time) {
  assert(has_storage());
  assert(dist::rank() == proc());
  // the default stream of the calling thread; a Carpet build with streams
  // would pass its own
  int const rc = cgx_carpet::transfer<gdata, ibbox, islab>(
      int(transport_operator), int(cent), this, gsrcs, times, dstbox, srcbox, slabinfo, time, order_space,
      order_time, nullptr);
  if (rc != CGX_OK) CCTK_VERROR("cgx_transfer: %s", cgx_last_error());
}

} // namespace CarpetLib
