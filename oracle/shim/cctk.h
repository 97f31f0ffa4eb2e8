/* Stand-in for the Cactus flesh header, just enough for CarpetLib's
 * grid-transfer operator sources to compile outside Cactus.
 * Test infrastructure for the oracle build only. */
#ifndef CGX_SHIM_CCTK_H
#define CGX_SHIM_CCTK_H
#include <stddef.h>
#ifdef __cplusplus
#include <complex>
#include <stdexcept>
#include <string>
#endif

#define CCTK_REAL_PRECISION_8 1
#define CCTK_REAL_PRECISION 8
#define CCTK_INTEGER_PRECISION_4 1
#define HAVE_CCTK_REAL8 1
#define HAVE_CCTK_INT4 1
#define HAVE_CCTK_CXX_AUTO_SPECIFIER 1
#define HAVE_CCTK_CXX_LAMBDA 1
#define HAVE_CCTK_CXX_RANGE_BASED_FOR 1
#define CARPET_DISABLE_BBOXSET2 1

typedef double CCTK_REAL;
typedef double CCTK_REAL8;
typedef int CCTK_INT;
typedef int CCTK_INT4;
typedef unsigned char CCTK_BYTE;
#ifdef __cplusplus
typedef std::complex<double> CCTK_COMPLEX16;
typedef CCTK_COMPLEX16 CCTK_COMPLEX;
#define HAVE_CCTK_COMPLEX16 1
static inline CCTK_COMPLEX16 CCTK_Cmplx16(double re, double im) { return CCTK_COMPLEX16(re, im); }
#endif

#define CCTK_VARIABLE_INT 1
#define CCTK_VARIABLE_REAL 2
#define CCTK_VARIABLE_COMPLEX 3
#define CCTK_VARIABLE_INT4 4
#define CCTK_VARIABLE_REAL8 5
#define CCTK_VARIABLE_BYTE 6
#define CCTK_VARIABLE_COMPLEX16 7

#define CCTK_ATTRIBUTE_ALIGNED(x) __attribute__((__aligned__(x)))
#define CCTK_ATTRIBUTE_PURE __attribute__((__pure__))
#define CCTK_ATTRIBUTE_CONST __attribute__((__const__))
#define CCTK_MEMBER_ATTRIBUTE_CONST __attribute__((__const__))
#define CCTK_ATTRIBUTE_NORETURN __attribute__((__noreturn__))
#define CCTK_MEMBER_ATTRIBUTE_PURE __attribute__((__pure__))
#define CCTK_ATTRIBUTE_UNUSED __attribute__((__unused__))
#define CCTK_BUILTIN_UNREACHABLE() __builtin_unreachable()
#define CCTK_BUILTIN_EXPECT(x, y) __builtin_expect(x, y)
#ifdef __cplusplus
#define restrict __restrict__
#endif
#define CCTK_FCALL
#define CCTK_FNAME(x) x##_
#define CCTK_THORNSTRING "CarpetLib"

#define CCTK_WARN_ABORT 0
#define CCTK_WARN_ALERT 1
#define CCTK_WARN_COMPLAIN 2
#define CCTK_WARN_PICKY 3
#define CCTK_WARN_DEBUG 4

#ifdef __cplusplus
extern "C" {
#endif
/* Errors become C++ exceptions so the oracle's C entry points can turn
 * them into status codes instead of aborting the process. */
void cgx_shim_error(int level, int line, const char *file, const char *msg);
void cgx_shim_verror(int level, int line, const char *file, const char *fmt, ...);
#ifdef __cplusplus
}
#endif

#define CCTK_WARN(level, msg) cgx_shim_error(level, __LINE__, __FILE__, msg)
#define CCTK_ERROR(msg) cgx_shim_error(0, __LINE__, __FILE__, msg)
#define CCTK_VWARN(level, ...) cgx_shim_verror(level, __LINE__, __FILE__, __VA_ARGS__)
#define CCTK_VERROR(...) cgx_shim_verror(0, __LINE__, __FILE__, __VA_ARGS__)
#define CCTK_VError(line, file, thorn, ...) cgx_shim_verror(0, line, file, __VA_ARGS__)
#define CCTK_VInfo(thorn, ...) ((void)0)
#define CCTK_INFO(msg) ((void)0)
#define CCTK_FullName(i) ((char *)0)

#define CCTK_ARGUMENTS void *cctkGH_
#define DECLARE_CCTK_ARGUMENTS
#define DECLARE_CCTK_ARGUMENTS_CarpetLib_test_prolongate_3d_rf2
#define DECLARE_CCTK_ARGUMENTS_CarpetLib_test_prolongate_3d_cc_rf2
#endif
