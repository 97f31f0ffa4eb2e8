// C entry points onto CarpetLib's own grid-transfer operators, compiled
// unchanged from the reference sources by oracle/Makefile against the
// stand-in headers in oracle/shim/.  TEST INFRASTRUCTURE: only the tests,
// the smoke check and the CPU baseline of bench.py load the resulting
// oracle/_ref/libcarpetref*.so; the product never does.
//
// Boxes are passed as int[9] = {lower[3], upper[3], stride[3]}, the layout
// CarpetLib itself hands to its Fortran operators (CarpetLib/src/data.cc:
// 212-214 reinterpret_casts an ibbox3 to int[3][3]).  Every entry point
// returns 0 on success and 1 when the operator raised a Cactus error; the
// message is then available from cgxref_last_error().
#include <cstring>
#include <exception>
#include <string>

#include "cctk.h"
#include "gdata.hh"
#include "operator_prototypes_3d.hh"

using namespace CarpetLib;

extern "C" int cgx_shim_use_openmp;

namespace {
thread_local std::string last_error;

ivect3 iv(const int *p) { return ivect3(p[0], p[1], p[2]); }
ibbox3 ib(const int *p) {
  return ibbox3(ivect3(p[0], p[1], p[2]), ivect3(p[3], p[4], p[5]),
                ivect3(p[6], p[7], p[8]));
}

typedef void (*op_t)(double const *, ivect3 const &, ivect3 const &, double *,
                     ivect3 const &, ivect3 const &, ibbox3 const &,
                     ibbox3 const &, ibbox3 const &, ibbox3 const &, void *);

// The OpenMP split of CarpetLib/src/data.cc:56-93 (call_operator): each
// thread takes a slab of the destination region along its longest axis.
// The operators are pointwise, so the split never changes a result.
void call_operator(op_t op, double const *src, ivect3 const &srcpadext,
                   ivect3 const &srcext, double *dst, ivect3 const &dstpadext,
                   ivect3 const &dstext, ibbox3 const &srcbbox,
                   ibbox3 const &dstbbox, ibbox3 const &srcregbbox,
                   ibbox3 const &dstregbbox) {
  if (!cgx_shim_use_openmp) {
    op(src, srcpadext, srcext, dst, dstpadext, dstext, srcbbox, dstbbox,
       srcregbbox, dstregbbox, nullptr);
    return;
  }
  std::string err;
#pragma omp parallel
  {
    int const nthreads = omp_get_num_threads();
    int const me = omp_get_thread_num();
    int const dir = maxloc(dstregbbox.shape());
    int const stride = dstregbbox.stride()[dir];
    int const first = dstregbbox.lower()[dir];
    int const last = dstregbbox.upper()[dir] + stride;
    int const npoints = last - first;
    int const mine = (npoints / stride + nthreads - 1) / nthreads * stride;
    int const myfirst = std::min(last, first + me * mine);
    int const mylast = std::min(last, myfirst + mine);
    ibbox3 const myreg(dstregbbox.lower().replace(dir, myfirst),
                       dstregbbox.upper().replace(dir, mylast - stride),
                       dstregbbox.stride());
    if (!myreg.empty()) {
      try {
        op(src, srcpadext, srcext, dst, dstpadext, dstext, srcbbox, dstbbox,
           srcregbbox, myreg, nullptr);
      } catch (std::exception const &e) {
#pragma omp critical
        err = e.what();
      }
    }
  }
  if (!err.empty())
    throw std::runtime_error(err);
}

template <class F> int guarded(F f) {
  try {
    f();
    return 0;
  } catch (std::exception const &e) {
    last_error = e.what();
    return 1;
  }
}
} // namespace

#define OPARGS                                                                 \
  const double *src, const int *srcpadext, const int *srcext, double *dst,     \
      const int *dstpadext, const int *dstext, const int *srcbbox,             \
      const int *dstbbox, const int *srcregbbox, const int *dstregbbox
#define OPCALL                                                                 \
  src, iv(srcpadext), iv(srcext), dst, iv(dstpadext), iv(dstext), ib(srcbbox), \
      ib(dstbbox), ib(srcregbbox), ib(dstregbbox)

extern "C" {

const char *cgxref_last_error(void) { return last_error.c_str(); }
void cgxref_set_openmp(int on) { cgx_shim_use_openmp = on; }

// copy_3d (CarpetLib/src/copy_3d.cc:25-122); slab_offset may be NULL.
int cgxref_copy_3d(OPARGS, const int *slab_offset) {
  return guarded([&] {
    islab slab;
    if (slab_offset)
      slab.offset = iv(slab_offset);
    copy_3d<double>(OPCALL, slab_offset ? (void *)&slab : nullptr);
  });
}

// prolongate_3d_rf2<double,ORDER> (CarpetLib/src/prolongate_3d_rf2.cc:356)
int cgxref_prolongate_3d_rf2(int order, OPARGS) {
  return guarded([&] {
    op_t op = nullptr;
    switch (order) {
    case 1: op = &prolongate_3d_rf2<double, 1>; break;
    case 3: op = &prolongate_3d_rf2<double, 3>; break;
    case 5: op = &prolongate_3d_rf2<double, 5>; break;
    case 7: op = &prolongate_3d_rf2<double, 7>; break;
    case 9: op = &prolongate_3d_rf2<double, 9>; break;
    case 11: op = &prolongate_3d_rf2<double, 11>; break;
    default: throw std::runtime_error("no vertex-centred stencil of this order");
    }
    call_operator(op, OPCALL);
  });
}

// prolongate_3d_cc_rf2<double,ORDER> (CarpetLib/src/prolongate_3d_cc_rf2.cc:238)
int cgxref_prolongate_3d_cc_rf2(int order, OPARGS) {
  return guarded([&] {
    op_t op = nullptr;
    switch (order) {
    case 0: op = &prolongate_3d_cc_rf2<double, 0>; break;
    case 1: op = &prolongate_3d_cc_rf2<double, 1>; break;
    case 2: op = &prolongate_3d_cc_rf2<double, 2>; break;
    case 3: op = &prolongate_3d_cc_rf2<double, 3>; break;
    case 4: op = &prolongate_3d_cc_rf2<double, 4>; break;
    case 5: op = &prolongate_3d_cc_rf2<double, 5>; break;
    default: throw std::runtime_error("no cell-centred stencil of this order");
    }
    call_operator(op, OPCALL);
  });
}

// prolongate_3d_cc_eno_rf2<double,ORDER>
// (CarpetLib/src/prolongate_3d_cc_eno_rf2.cc:944), ORDER 2 or 3
int cgxref_prolongate_3d_cc_eno_rf2(int order, OPARGS) {
  return guarded([&] {
    op_t op = nullptr;
    switch (order) {
    case 2: op = &prolongate_3d_cc_eno_rf2<double, 2>; break;
    case 3: op = &prolongate_3d_cc_eno_rf2<double, 3>; break;
    default: throw std::runtime_error("no cell-centred ENO stencil of this order");
    }
    call_operator(op, OPCALL);
  });
}

// prolongate_3d_o5_monotone_rf2 (CarpetLib/src/prolongate_3d_o5_monotone_rf2.cc:45)
int cgxref_prolongate_3d_o5_monotone_rf2(OPARGS) {
  return guarded([&] { call_operator(&prolongate_3d_o5_monotone_rf2<double>, OPCALL); });
}

// restrict_3d_rf2 (CarpetLib/src/restrict_3d_rf2.cc:25); called directly,
// as CarpetLib/src/data.cc:1041 does through call_operator.
int cgxref_restrict_3d_rf2(OPARGS) {
  return guarded([&] { call_operator(&restrict_3d_rf2<double>, OPCALL); });
}

// restrict_3d_cc_rf2 (CarpetLib/src/restrict_3d_cc_rf2.cc:23); CarpetLib
// calls it without call_operator (data.cc:1100-1105).
int cgxref_restrict_3d_cc_rf2(OPARGS) {
  return guarded([&] { restrict_3d_cc_rf2<double>(OPCALL, nullptr); });
}

// restrict_3d_cc_o3_rf2 / restrict_3d_cc_o5_rf2
// (CarpetLib/src/restrict_3d_cc_o3_rf2.cc:33, restrict_3d_cc_o5_rf2.cc:79);
// CarpetLib calls them without call_operator (data.cc:1065-1085).
int cgxref_restrict_3d_cc_o3_rf2(OPARGS) {
  return guarded([&] { restrict_3d_cc_o3_rf2<double>(OPCALL, nullptr); });
}
int cgxref_restrict_3d_cc_o5_rf2(OPARGS) {
  return guarded([&] { restrict_3d_cc_o5_rf2<double>(OPCALL, nullptr); });
}

#define TIARGS                                                                 \
  const int *srcpadext, const int *srcext, double *dst, double t,              \
      const int *dstpadext, const int *dstext, const int *srcbbox,             \
      const int *dstbbox, const int *srcregbbox, const int *dstregbbox
#define TICALL                                                                 \
  iv(srcpadext), iv(srcext), dst, t, iv(dstpadext), iv(dstext), ib(srcbbox),   \
      ib(dstbbox), ib(srcregbbox), ib(dstregbbox), nullptr

// The time interpolators open their own OpenMP region
// (CarpetLib/src/interpolate_3d_2tl.cc:245, interpolate_3d_3tl.cc:385,
// interpolate_eno_3d_3tl.cc:141).
// interpolate_3d_2tl (CarpetLib/src/interpolate_3d_2tl.cc:24)
int cgxref_interpolate_3d_2tl(const double *src1, double t1,
                              const double *src2, double t2, TIARGS) {
  return guarded(
      [&] { interpolate_3d_2tl<double>(src1, t1, src2, t2, TICALL); });
}

// interpolate_3d_3tl (CarpetLib/src/interpolate_3d_3tl.cc:24)
int cgxref_interpolate_3d_3tl(const double *src1, double t1,
                              const double *src2, double t2,
                              const double *src3, double t3, TIARGS) {
  return guarded([&] {
    interpolate_3d_3tl<double>(src1, t1, src2, t2, src3, t3, TICALL);
  });
}

// interpolate_3d_4tl (CarpetLib/src/interpolate_3d_4tl.cc:24)
int cgxref_interpolate_3d_4tl(const double *src1, double t1, const double *src2, double t2,
                              const double *src3, double t3, const double *src4, double t4,
                              TIARGS) {
  return guarded([&] {
    interpolate_3d_4tl<double>(src1, t1, src2, t2, src3, t3, src4, t4, TICALL);
  });
}

// interpolate_3d_5tl (CarpetLib/src/interpolate_3d_5tl.cc:24)
int cgxref_interpolate_3d_5tl(const double *src1, double t1, const double *src2, double t2,
                              const double *src3, double t3, const double *src4, double t4,
                              const double *src5, double t5, TIARGS) {
  return guarded([&] {
    interpolate_3d_5tl<double>(src1, t1, src2, t2, src3, t3, src4, t4, src5, t5, TICALL);
  });
}

// interpolate_eno_3d_3tl (CarpetLib/src/interpolate_eno_3d_3tl.cc:32)
int cgxref_interpolate_eno_3d_3tl(const double *src1, double t1,
                                  const double *src2, double t2,
                                  const double *src3, double t3, TIARGS) {
  return guarded([&] {
    interpolate_eno_3d_3tl<double>(src1, t1, src2, t2, src3, t3, TICALL);
  });
}

} // extern "C"

// ---------------------------------------------------------------------------
// A list of box-pairs of one grid function through CarpetLib's own local
// transfer path, data<T>::transfer_time (CarpetLib/src/data.cc:486-534),
// with the loop over the pairs in C++ so that the CPU baseline times the
// operators rather than the caller: for each pair, with ntl > 1 one
// temporary per timelevel over the destination box (allocated and freed per
// call, as data.cc:506-520 does), the spatial operator into each, then
// time_interpolate into the destination (data.cc:1183-1259); with ntl == 1
// the spatial operator straight into the destination.  The spatial operator
// follows transfer_p_r (data.cc:537-556): copy_3d without call_operator
// (copy_from_innerloop, data.cc:433-462), prolongate_3d_rf2<order_space>
// and restrict_3d_rf2 through call_operator (data.cc:600-613, 1039-1046).
//
// kind 0 = copy, 1 = vertex-centred Lagrange prolongation, 2 = injection.
// Arrays are {data, padext[3], bbox[9]}; src holds npairs * ntl arrays,
// pair-major.
struct cgxref_arr {
  double *data;
  int padext[3];
  int bbox[9];
};

namespace {
ivect3 shape_of(const int *b) {
  return ivect3((b[3] - b[0]) / b[6] + 1, (b[4] - b[1]) / b[7] + 1, (b[5] - b[2]) / b[8] + 1);
}
op_t vc_operator(int order) {
  switch (order) {
  case 1: return &prolongate_3d_rf2<double, 1>;
  case 3: return &prolongate_3d_rf2<double, 3>;
  case 5: return &prolongate_3d_rf2<double, 5>;
  case 7: return &prolongate_3d_rf2<double, 7>;
  case 9: return &prolongate_3d_rf2<double, 9>;
  case 11: return &prolongate_3d_rf2<double, 11>;
  }
  throw std::runtime_error("no vertex-centred stencil of this order");
}
// transfer_p_r of one timelevel into (out, outpad, outbox)
void spatial(int kind, int order, const cgxref_arr &src, double *out, ivect3 const &outpad,
             ibbox3 const &outbox, ibbox3 const &dstbox, ibbox3 const &srcbox) {
  ivect3 const spad = iv(src.padext), sext = shape_of(src.bbox);
  ibbox3 const sbb = ib(src.bbox);
  ivect3 const oext = outbox.sizes();
  switch (kind) {
  case 0:
    copy_3d<double>(src.data, spad, sext, out, outpad, oext, sbb, outbox, srcbox, dstbox, nullptr);
    return;
  case 1:
    call_operator(vc_operator(order), src.data, spad, sext, out, outpad, oext, sbb, outbox, srcbox,
                  dstbox);
    return;
  case 2:
    call_operator(&restrict_3d_rf2<double>, src.data, spad, sext, out, outpad, oext, sbb, outbox,
                  srcbox, dstbox);
    return;
  }
  throw std::runtime_error("unknown transfer kind");
}
} // namespace

extern "C" int cgxref_transfer_pairs(int kind, int order_space, int npairs, const cgxref_arr *dst,
                                     const cgxref_arr *src, int ntl, const int *dstboxes,
                                     const int *srcboxes, const double *times, double time) {
  return guarded([&] {
    if (ntl < 1 || ntl > 3) throw std::runtime_error("1 to 3 timelevels");
    for (int p = 0; p < npairs; ++p) {
      const cgxref_arr &d = dst[p];
      ibbox3 const dstbox = ib(dstboxes + 9 * p), srcbox = ib(srcboxes + 9 * p);
      ibbox3 const dbb = ib(d.bbox);
      ivect3 const dpad = iv(d.padext), dext = shape_of(d.bbox);
      if (ntl == 1) {
        spatial(kind, order_space, src[(size_t)p * ntl], d.data, dpad, dbb, dstbox, srcbox);
        continue;
      }
      ivect3 const tsz = dstbox.sizes();
      size_t const n = (size_t)tsz[0] * tsz[1] * tsz[2];
      double *tmp[3] = {nullptr, nullptr, nullptr};
      for (int t = 0; t < ntl; ++t) tmp[t] = new double[n];
      for (int t = 0; t < ntl; ++t)
        spatial(kind, order_space, src[(size_t)p * ntl + t], tmp[t], tsz, dstbox, dstbox, srcbox);
      if (ntl == 2)
        interpolate_3d_2tl<double>(tmp[0], times[0], tmp[1], times[1], tsz, tsz, d.data, time, dpad,
                                   dext, dstbox, dbb, dstbox, dstbox, nullptr);
      else
        interpolate_3d_3tl<double>(tmp[0], times[0], tmp[1], times[1], tmp[2], times[2], tsz, tsz,
                                   d.data, time, dpad, dext, dstbox, dbb, dstbox, dstbox, nullptr);
      for (int t = 0; t < ntl; ++t) delete[] tmp[t];
    }
  });
}
