// cgx_carpet.hh -- the CarpetLib side of the drop-in: marshalling from
// CarpetLib's types (gdata / data<T>, ibbox, islab) to the C-ABI of
// include/cgx.h.  Compiled inside CarpetLib (see carpet_b200/carpet/data_cgx.cc
// and INTEGRATION.md); nothing here depends on the rest of this package.
//
// The layout follows what CarpetLib itself hands its operators:
//   * an array is (storage(), padded_shape(), extent()) of a gdata
//     (CarpetLib/src/gdata.hh:111-155; the operators take exactly these,
//     data.cc:600-613);
//   * a box is int[9] {lower[3], upper[3], stride[3]}, the memory layout of
//     bbox<int,3> that data.cc:212-214 reinterpret_casts to int[3][3] for
//     the Fortran operators;
//   * the slab offset is islab::offset (gdata.hh:25-31), or null;
//   * operator_type and centering keep CarpetLib's enum values
//     (operators.hh:8-25, defs.hh:134), which cgx.h's CGX_OP_* / CGX_VERTEX
//     / CGX_CELL equal (checked at compile time in data_cgx.cc).
#ifndef CGX_CARPET_HH
#define CGX_CARPET_HH

#include <vector>

#include "cgx.h"

namespace cgx_carpet {

// bbox<int,3> -> {lower[3], upper[3], stride[3]}
template <class Box> inline void box9(Box const &b, int out[9]) {
  for (int d = 0; d < 3; ++d) {
    out[d] = b.lower()[d];
    out[3 + d] = b.upper()[d];
    out[6 + d] = b.stride()[d];
  }
}

// one component at one timelevel (a gdata with CCTK_REAL8 storage on this
// process's device)
template <class G> inline cgx_array as_cgx(G const *g) {
  cgx_array a;
  a.data = static_cast<double *>(const_cast<void *>(g->storage()));
  for (int d = 0; d < 3; ++d) a.padext[d] = g->padded_shape()[d];
  box9(g->extent(), a.bbox);
  return a;
}

// gdata::transfer_data's local work for one box-pair: the arguments of
// data<T>::transfer_from_innerloop (CarpetLib/src/data.cc:465-483)
// marshalled into cgx_transfer.  Returns cgx_transfer's status.
template <class G, class Box, class Slab>
inline int transfer(int op, int cent, G *dst, std::vector<G const *> const &srcs,
                    std::vector<double> const &times, Box const &dstbox, Box const &srcbox,
                    Slab const *slabinfo, double time, int order_space, int order_time, void *stream) {
  cgx_array d = as_cgx(dst);
  std::vector<cgx_array> s;
  s.reserve(srcs.size());
  for (G const *g : srcs) s.push_back(as_cgx(g));
  int db[9], sb[9];
  box9(dstbox, db);
  box9(srcbox, sb);
  return cgx_transfer(op, cent, &d, s.data(), times.data(), (int)srcs.size(), db, sb,
                      slabinfo ? &slabinfo->offset[0] : nullptr, time, order_space, order_time, stream);
}

} // namespace cgx_carpet

#endif // CGX_CARPET_HH
