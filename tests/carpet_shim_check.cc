// The CarpetLib-side marshalling of carpet_b200/carpet/cgx_carpet.hh against
// CarpetLib's own types (bbox, vect, islab), run on the CPU with a stand-in
// for cgx_transfer that records its arguments.  Built and run by
// tests/test_carpet_shim.py.
#include <cctk.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "bbox.hh"
#include "gdata.hh"
#include "vect.hh"

#include "cgx_carpet.hh"

using namespace CarpetLib;

namespace {
struct Seen {
  int op, cent, nsrc, order_space, order_time, slab[3], has_slab;
  cgx_array dst, srcs[3];
  double times[3], time;
  int dstbox[9], srcbox[9];
  void *stream;
} seen;

// one component's accessors, as gdata has them (gdata.hh:111-155)
struct Array {
  void *mem;
  ivect pad;
  ibbox ext;
  void const *storage() const { return mem; }
  ivect const &padded_shape() const { return pad; }
  ibbox const &extent() const { return ext; }
};

int fails = 0;
void expect(bool ok, const char *what) {
  if (!ok) {
    std::printf("FAIL %s\n", what);
    ++fails;
  }
}
} // namespace

extern "C" int cgx_transfer(int op, int cent, const cgx_array *dst, const cgx_array *srcs, const double *times,
                            int nsrc, const int dstbox[9], const int srcbox[9], const int *slab_offset,
                            double time, int order_space, int order_time, void *stream) {
  seen.op = op;
  seen.cent = cent;
  seen.dst = *dst;
  seen.nsrc = nsrc;
  for (int i = 0; i < nsrc && i < 3; ++i) {
    seen.srcs[i] = srcs[i];
    seen.times[i] = times[i];
  }
  std::memcpy(seen.dstbox, dstbox, sizeof seen.dstbox);
  std::memcpy(seen.srcbox, srcbox, sizeof seen.srcbox);
  seen.has_slab = slab_offset != nullptr;
  if (slab_offset) std::memcpy(seen.slab, slab_offset, sizeof seen.slab);
  seen.time = time;
  seen.order_space = order_space;
  seen.order_time = order_time;
  seen.stream = stream;
  return CGX_OK;
}
extern "C" const char *cgx_last_error(void) { return ""; }

int main() {
  // the box layout CarpetLib hands its Fortran operators (data.cc:212-214)
  ibbox const b(ivect(-3, 4, 10), ivect(9, 16, 30), ivect(1, 2, 2));
  int b9[9];
  cgx_carpet::box9(b, b9);
  expect(std::memcmp(b9, reinterpret_cast<int const *>(&b), sizeof b9) == 0,
         "box9 is the memory layout of bbox<int,3>");
  const int want9[9] = {-3, 4, 10, 9, 16, 30, 1, 2, 2};
  expect(std::memcmp(b9, want9, sizeof b9) == 0, "box9 = lower, upper, stride");

  static double m[4][64];
  ibbox const fine(ivect(0, 0, 0), ivect(14, 6, 4), ivect(1, 1, 1));
  ibbox const coarse(ivect(-4, -2, -2), ivect(16, 8, 6), ivect(2, 2, 2));
  Array dst{m[0], ivect(16, 7, 5), fine};
  std::vector<Array const *> srcs;
  Array s0{m[1], ivect(12, 6, 5), coarse}, s1{m[2], ivect(12, 6, 5), coarse}, s2{m[3], ivect(12, 6, 5), coarse};
  srcs.push_back(&s0);
  srcs.push_back(&s1);
  srcs.push_back(&s2);
  std::vector<double> times{0.5, 0.375, 0.25};
  ibbox const dstbox(ivect(2, 1, 0), ivect(12, 5, 4), ivect(1, 1, 1));
  ibbox const srcbox(ivect(-2, 0, -2), ivect(14, 6, 6), ivect(2, 2, 2));
  islab slab;
  slab.offset = ivect(1, -2, 3);

  int rc = cgx_carpet::transfer<Array, ibbox, islab>(int(op_Lagrange), int(vertex_centered), &dst, srcs, times,
                                                     dstbox, srcbox, &slab, 0.4375, 5, 2, nullptr);
  expect(rc == CGX_OK, "status");
  expect(seen.op == CGX_OP_LAGRANGE && seen.cent == CGX_VERTEX, "operator and centring");
  expect(seen.dst.data == m[0], "destination storage");
  expect(seen.dst.padext[0] == 16 && seen.dst.padext[1] == 7 && seen.dst.padext[2] == 5, "padded shape");
  int f9[9];
  cgx_carpet::box9(fine, f9);
  expect(std::memcmp(seen.dst.bbox, f9, sizeof f9) == 0, "destination extent");
  expect(seen.nsrc == 3, "timelevels");
  for (int i = 0; i < 3; ++i) {
    expect(seen.srcs[i].data == m[1 + i], "source storage");
    expect(seen.times[i] == times[i], "times");
  }
  int d9[9], s9[9];
  cgx_carpet::box9(dstbox, d9);
  cgx_carpet::box9(srcbox, s9);
  expect(std::memcmp(seen.dstbox, d9, sizeof d9) == 0, "recv box");
  expect(std::memcmp(seen.srcbox, s9, sizeof s9) == 0, "send box");
  expect(seen.has_slab && seen.slab[0] == 1 && seen.slab[1] == -2 && seen.slab[2] == 3, "slab offset");
  expect(seen.time == 0.4375 && seen.order_space == 5 && seen.order_time == 2, "time and orders");

  rc = cgx_carpet::transfer<Array, ibbox, islab>(int(op_copy), int(cell_centered), &dst, srcs, times, dstbox,
                                                 srcbox, nullptr, 0.0, 1, 0, nullptr);
  expect(!seen.has_slab && seen.op == CGX_OP_COPY && seen.cent == CGX_CELL, "no slab; copy, cell centring");

  if (fails) return 1;
  std::printf("carpet shim marshalling ok\n");
  return 0;
}
