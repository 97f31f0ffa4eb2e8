/* Stand-in for the EinsteinToolkit Vectors thorn's vectors.h with a
 * scalar vector type (vector size 1).  madd(a,b,c) = a*b + c; whether
 * that becomes one fused multiply-add is decided by the compiler flag
 * (-ffp-contract=off for the canonical two-rounding order). */
#ifndef CGX_SHIM_VECTORS_H
#define CGX_SHIM_VECTORS_H
#define CCTK_REAL_VEC_SIZE 1
namespace CarpetLib {
template <typename T> struct vecprops {
  typedef T vector_t;
  static inline int size() { return 1; }
  static inline vector_t load(T const &a) { return a; }
  static inline vector_t loadu(T const &a) { return a; }
  static inline T elt(vector_t const &x, int) { return x; }
  static inline vector_t mul(vector_t const &x, vector_t const &y) { return x * y; }
  static inline vector_t madd(vector_t const &x, vector_t const &y,
                              vector_t const &z) { return x * y + z; }
};
}
#endif
