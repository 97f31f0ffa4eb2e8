// Runtime support for the shim-built CarpetLib operators (test
// infrastructure for the oracle only): Cactus error reporting becomes a
// C++ exception that the C wrappers in ref_api.cc turn into a status code,
// the OpenMP switch the operators read through DECLARE_CCTK_PARAMETERS,
// and the two CarpetLib helpers the operator objects link against.
#include <cstdarg>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "cctk.h"
#include "nompi.h"

extern "C" {
int cgx_shim_use_openmp = 1;
}

struct cgx_shim_exception : std::runtime_error {
  using std::runtime_error::runtime_error;
};

extern "C" void cgx_shim_error(int level, int line, const char *file,
                               const char *msg) {
  if (level > 0)
    return; // warnings of level >= 1 do not abort in Cactus either
  char buf[512];
  snprintf(buf, sizeof buf, "%s:%d: %s", file, line, msg);
  throw cgx_shim_exception(buf);
}

extern "C" void cgx_shim_verror(int level, int line, const char *file,
                                const char *fmt, ...) {
  char msg[400];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, sizeof msg, fmt, ap);
  va_end(ap);
  cgx_shim_error(level, line, file, msg);
}

namespace CarpetLib {
// Integer power by repeated squaring; only the coefficient self-tests
// (coeffs1d<>::test) call it, with a 1000-ulp tolerance.
template <class T> T ipow(T x, int y) {
  T res = T(1);
  bool neg = y < 0;
  unsigned n = neg ? unsigned(-y) : unsigned(y);
  while (n) {
    if (n & 1u)
      res *= x;
    x *= x;
    n >>= 1;
  }
  return neg ? T(1) / res : res;
}
template double ipow<double>(double, int);

namespace dist {
struct mpi_struct_descr_t;
// Only reached when MPI datatypes for bboxes are built, which the oracle
// never does.
MPI_Datatype create_mpi_datatype(size_t, mpi_struct_descr_t const *,
                                 char const *, size_t) {
  throw cgx_shim_exception("MPI datatypes are not available in the oracle");
}
} // namespace dist
} // namespace CarpetLib

#include <istream>
namespace CarpetLib {
// Stream parsing helpers of CarpetLib/src/defs.cc, pulled in by the bbox
// and vect input operators that the oracle never calls.
void skipws(std::istream &is) { is >> std::ws; }
void expect(std::istream &, char) {
  throw cgx_shim_exception("bbox parsing is not available in the oracle");
}
void consume(std::istream &, char) {
  throw cgx_shim_exception("bbox parsing is not available in the oracle");
}
void consume(std::istream &, char const *) {
  throw cgx_shim_exception("bbox parsing is not available in the oracle");
}
} // namespace CarpetLib

// Container helpers of CarpetLib/src/defs.cc and the slab printer of
// gdata.cc that the bbox/vect objects and copy_3d's error message refer to.
#include "bbox.hh"
#include "gdata.hh"
namespace CarpetLib {
template <class T> size_t memoryof(std::vector<T> const &c) {
  return sizeof c + c.capacity() * sizeof(T);
}
template size_t memoryof(std::vector<ibbox> const &);
template <class T> std::ostream &output(std::ostream &os, const std::vector<T> &v) {
  os << "[";
  for (size_t i = 0; i < v.size(); ++i)
    os << (i ? "," : "") << v[i];
  return os << "]";
}
template std::ostream &output(std::ostream &, const std::vector<ibbox> &);
template std::ostream &output(std::ostream &, const std::vector<int> &);
template <class T> std::istream &input(std::istream &is, std::vector<T> &) {
  throw cgx_shim_exception("vector parsing is not available in the oracle");
  return is;
}
template std::istream &input(std::istream &, std::vector<ibbox> &);
template <typename T, int D>
std::ostream &operator<<(std::ostream &os, slab<T, D> const &s) {
  return os << "slab{offset=" << s.offset << ",is_centered=" << s.is_centered
            << "}";
}
template std::ostream &operator<<(std::ostream &, slab<int, 3> const &);
} // namespace CarpetLib
