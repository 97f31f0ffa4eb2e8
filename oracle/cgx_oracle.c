/*
 * cgx_oracle.c -- CPU restatement of CarpetLib's grid-transfer hot path.
 *
 * TEST INFRASTRUCTURE.  This file is the oracle: the parity tests, the
 * smoke check and the CPU-baseline leg of bench.py call it as the checker.
 * Nothing in the product (carpet_b200/, include/) links, loads or calls it,
 * and the product has no CPU fallback through it.
 *
 * Built with -ffp-contract=off (oracle/Makefile), so every a*b + c written
 * below rounds twice unless it is an explicit fma().
 *
 * Every function below restates one reference routine, cited by
 * file:line inside the EinsteinToolkit/Carpet sources.  The arithmetic
 * follows the reference's operation order exactly:
 *   fma == 0  two roundings per multiply-add, the order of a build with
 *             -ffp-contract=off (the canonical order);
 *   fma == 1  every multiply-add contracted the way GCC contracts the same
 *             expressions under -mfma -ffp-contract=fast.
 * Both are pinned bit-for-bit against the reference's own operators,
 * compiled unchanged (oracle/Makefile -> oracle/_ref/), by tests/ -- except
 * the vertex-centred ENO of prolongate_3d_real8_eno.F90, which is Fortran:
 * with no Fortran compiler here its parity is unpinned by a compiled
 * reference, and tests/test_eno_restatement.py checks it instead against a
 * second, independent restatement of the Fortran source and against the
 * properties the routine guarantees.
 *
 * Boxes are int[9] = {lower[3], upper[3], stride[3]} (inclusive bounds), the
 * layout CarpetLib passes to its Fortran operators (data.cc:212-214).
 * Arrays are x-fastest: index = i + padext[0]*(j + padext[1]*k)
 * (operator_prototypes_3d.hh:17-28).  Every entry point returns 0 on success
 * or a CGXO_E* code where the reference would abort; the message is
 * available from cgxo_last_error().
 */
#include <math.h>
#include <stddef.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define CGXO_OK 0
#define CGXO_EINVAL 1       /* inconsistent strides / boxes / times */
#define CGXO_EUNSUPPORTED 2 /* operator outside the restated set */
#define CGXO_ENOMEM 3

/* operator_type, CarpetLib/src/operators.hh:8-25 */
enum { op_error, op_none, op_sync, op_restrict, op_copy, op_Lagrange, op_ENO,
       op_WENO, op_TVD, op_Lagrange_monotone };
/* centering, CarpetLib/src/defs.hh:134 */
enum { error_centered, vertex_centered, cell_centered };

static _Thread_local char last_error[512];

const char *cgxo_last_error(void) { return last_error; }

static int fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(last_error, sizeof last_error, fmt, ap);
  va_end(ap);
  return code;
}

/* ------------------------------------------------------------------ */
/* bbox helpers, CarpetLib/src/bbox.cc                                 */

typedef struct { int lo[3], up[3], str[3]; } box_t;

static box_t mkbox(const int *b) {
  box_t r;
  for (int d = 0; d < 3; ++d) {
    r.lo[d] = b[d];
    r.up[d] = b[3 + d];
    r.str[d] = b[6 + d];
  }
  return r;
}
/* bbox::empty, bbox.hh:101 */
static int box_empty(const box_t *b) {
  for (int d = 0; d < 3; ++d)
    if (b->lo[d] > b->up[d]) return 1;
  return 0;
}
/* bbox::shape / sizes, bbox.cc:64-70 */
static int box_size(const box_t *b, int d) {
  return box_empty(b) ? 0 : (b->up[d] - b->lo[d] + b->str[d]) / b->str[d];
}
/* bbox::is_contained_in, bbox.cc:103-109 (no alignment check) */
static int box_in(const box_t *a, const box_t *b) {
  if (box_empty(a)) return 1;
  for (int d = 0; d < 3; ++d)
    if (a->lo[d] < b->lo[d] || a->up[d] > b->up[d]) return 0;
  return 1;
}
/* bbox::expand(lo, hi), bbox.cc:180-191 */
static box_t box_expand(const box_t *b, const int *lo, const int *hi) {
  box_t r = *b;
  for (int d = 0; d < 3; ++d) {
    r.lo[d] = b->lo[d] - lo[d] * b->str[d];
    r.up[d] = b->up[d] + hi[d] * b->str[d];
  }
  return r;
}
static int imod(int x, int y) { int r = x % y; return r < 0 ? r + y : r; }
/* bbox::expanded_for, bbox.cc:208-219 */
static box_t box_expanded_for(const box_t *a, const box_t *b) {
  box_t r;
  for (int d = 0; d < 3; ++d) {
    int str = b->str[d];
    int loff = imod(a->lo[d] - b->lo[d], str);
    int uoff = imod(a->up[d] - b->lo[d], str);
    r.lo[d] = a->lo[d] - loff;
    r.up[d] = a->up[d] + (str - uoff) % str;
    r.str[d] = str;
  }
  return r;
}
static int same_stride(const box_t *a, const box_t *b) {
  for (int d = 0; d < 3; ++d)
    if (a->str[d] != b->str[d]) return 0;
  return 1;
}

#define IDX(i, j, k, pad) \
  ((size_t)(i) + (size_t)(pad)[0] * ((size_t)(j) + (size_t)(pad)[1] * (size_t)(k)))

/* ------------------------------------------------------------------ */
/* copy_3d, CarpetLib/src/copy_3d.cc:25-122                             */

int cgxo_copy_3d(const double *src, const int *srcpadext, const int *srcext,
                 double *dst, const int *dstpadext, const int *dstext,
                 const int *srcbbox_, const int *dstbbox_,
                 const int *srcregbbox_, const int *dstregbbox_,
                 const int *slab_offset) {
  box_t srcbbox = mkbox(srcbbox_), dstbbox = mkbox(dstbbox_);
  box_t srcreg1 = mkbox(srcregbbox_), dstreg = mkbox(dstregbbox_);
  (void)srcext; (void)dstext;
  /* copy_3d.cc:36-49 */
  if (!same_stride(&srcbbox, &dstreg) || !same_stride(&dstbbox, &dstreg) ||
      !same_stride(&srcreg1, &dstreg))
    return fail(CGXO_EINVAL, "copy_3d: strides disagree");
  /* copy_3d.cc:53-55 */
  if (box_empty(&dstreg))
    return fail(CGXO_EINVAL, "copy_3d: region extent is empty");
  /* copy_3d.cc:57-58: srcregbbox = dstregbbox.shift(slab.offset) */
  box_t srcreg = dstreg;
  if (slab_offset)
    for (int d = 0; d < 3; ++d) {
      srcreg.lo[d] += slab_offset[d] * dstreg.str[d];
      srcreg.up[d] += slab_offset[d] * dstreg.str[d];
    }
  /* copy_3d.cc:59 */
  if (!box_in(&srcreg, &srcreg1))
    return fail(CGXO_EINVAL, "copy_3d: shifted source region outside srcregbbox");
  /* copy_3d.cc:63-74 */
  if (!box_in(&srcreg, &srcbbox) || !box_in(&dstreg, &dstbbox))
    return fail(CGXO_EINVAL, "copy_3d: region extent is not contained in array extent");
  int regext[3], srcoff[3], dstoff[3];
  for (int d = 0; d < 3; ++d) {
    regext[d] = box_size(&dstreg, d);
    if ((srcreg.lo[d] - srcbbox.lo[d]) % srcbbox.str[d] ||
        (dstreg.lo[d] - dstbbox.lo[d]) % dstbbox.str[d])
      return fail(CGXO_EINVAL, "copy_3d: region not aligned with array");
    srcoff[d] = (srcreg.lo[d] - srcbbox.lo[d]) / srcbbox.str[d];
    dstoff[d] = (dstreg.lo[d] - dstbbox.lo[d]) / dstbbox.str[d];
  }
  /* copy_3d.cc:113-121 */
  for (int k = 0; k < regext[2]; ++k)
    for (int j = 0; j < regext[1]; ++j)
      for (int i = 0; i < regext[0]; ++i)
        dst[IDX(dstoff[0] + i, dstoff[1] + j, dstoff[2] + k, dstpadext)] =
            src[IDX(srcoff[0] + i, srcoff[1] + j, srcoff[2] + k, srcpadext)];
  return CGXO_OK;
}

/* ------------------------------------------------------------------ */
/* Multiply-add in the two orders.                                     */

/* a*b + c; fma==0 rounds the product first */
static inline double madd(int fma_, double a, double b, double c) {
  return fma_ ? fma(a, b, c) : a * b + c; /* built with -ffp-contract=off */
}

/* ------------------------------------------------------------------ */
/* prolongate_3d_rf2, CarpetLib/src/prolongate_3d_rf2.cc:356-675       */

/* coeffs1d<RT,ORDER>::coeffs, prolongate_3d_rf2.cc:92-124, numerators over
 * 2, 16, 256, 2048, 65536, 524288 */
static const double vc_num1[] = {1, 1};
static const double vc_num3[] = {-1, 9, 9, -1};
static const double vc_num5[] = {3, -25, 150, 150, -25, 3};
static const double vc_num7[] = {-5, 49, -245, 1225, 1225, -245, 49, -5};
static const double vc_num9[] = {35,    -405, 2268, -8820, 39690,
                                 39690, -8820, 2268, -405,  35};
static const double vc_num11[] = {-63,    847,    -5445,  22869, -76230, 320166,
                                  320166, -76230, 22869,  -5445, 847,    -63};

static int vc_coeffs(int order, double *c) {
  const double *num;
  double den;
  switch (order) {
  case 1: num = vc_num1; den = 2.0; break;
  case 3: num = vc_num3; den = 16.0; break;
  case 5: num = vc_num5; den = 256.0; break;
  case 7: num = vc_num7; den = 2048.0; break;
  case 9: num = vc_num9; den = 65536.0; break;
  case 11: num = vc_num11; den = 524288.0; break;
  default: return 0;
  }
  /* "+n / RT(den)" : one correctly rounded division (exact dyadics) */
  for (int i = 0; i <= order; ++i) c[i] = num[i] / den;
  return order + 1;
}

/* interp1 with the scalar Vectors order (vector size 1),
 * prolongate_3d_rf2.cc:174-249:
 *   vres = c0*p0; vres = madd(c_m, p_m, vres) ...; res = 0 + vres */
static inline double vc_line(int fma_, const double *c, int n, const double *p,
                             ptrdiff_t stride) {
  double v = c[0] * p[0];
  for (int m = 1; m < n; ++m) v = madd(fma_, c[m], p[m * stride], v);
  return 0.0 + v;
}
/* interp2 / interp3 outer sums, prolongate_3d_rf2.cc:262-295:
 *   res = 0; res += c_m * inner_m */
static inline double acc_sum(int fma_, const double *c, int n, const double *v) {
  double res = 0.0;
  for (int m = 0; m < n; ++m) res = madd(fma_, c[m], v[m], res);
  return res;
}

int cgxo_prolongate_3d_rf2(int order, int fma_, const double *src,
                           const int *srcpadext, const int *srcext, double *dst,
                           const int *dstpadext, const int *dstext,
                           const int *srcbbox_, const int *dstbbox_,
                           const int *srcregbbox_, const int *regbbox_) {
  (void)srcregbbox_; (void)dstext;
  double c[12];
  int n = vc_coeffs(order, c);
  if (!n) return fail(CGXO_EUNSUPPORTED, "prolongate_3d_rf2: no stencil of order %d", order);
  box_t srcbbox = mkbox(srcbbox_), dstbbox = mkbox(dstbbox_), reg = mkbox(regbbox_);
  /* prolongate_3d_rf2.cc:373-391 */
  for (int d = 0; d < 3; ++d) {
    if (srcbbox.str[d] <= reg.str[d] || dstbbox.str[d] != reg.str[d])
      return fail(CGXO_EINVAL, "prolongate_3d_rf2: strides disagree");
    if (srcbbox.str[d] != 2 * dstbbox.str[d])
      return fail(CGXO_EINVAL, "prolongate_3d_rf2: source strides are not twice the destination strides");
    if (srcbbox.lo[d] % srcbbox.str[d] || dstbbox.lo[d] % dstbbox.str[d] ||
        reg.lo[d] % reg.str[d])
      return fail(CGXO_EINVAL, "prolongate_3d_rf2: bbox is not aligned with vertices");
  }
  if (box_empty(&reg))
    return fail(CGXO_EINVAL, "prolongate_3d_rf2: region extent is empty");
  /* prolongate_3d_rf2.cc:393-417 */
  int regext[3], srcoff[3], dstoff[3], offlo[3], offhi[3];
  for (int d = 0; d < 3; ++d) {
    regext[d] = box_size(&reg, d);
    srcoff[d] = (reg.lo[d] - srcbbox.lo[d]) / reg.str[d];
    dstoff[d] = (reg.lo[d] - dstbbox.lo[d]) / reg.str[d];
    int needlo = srcoff[d] % 2 != 0;
    int needhi = (srcoff[d] + regext[d] - 1) % 2 != 0;
    offlo[d] = needlo ? order / 2 + 1 : (regext[d] > 1 ? order / 2 : 0);
    offhi[d] = needhi ? order / 2 + 1 : (regext[d] > 1 ? order / 2 : 0);
  }
  box_t ex = box_expand(&reg, offlo, offhi);
  if (!box_in(&ex, &srcbbox) || !box_in(&reg, &dstbbox))
    return fail(CGXO_EINVAL, "prolongate_3d_rf2: region extent is not contained in array extent");
  const int imin = -(order + 1) / 2 + 1; /* coeffs1d::imin, :32 */
  (void)srcext;
  double ybuf[12], zbuf[12];
  /* The goto-nest of :468-674 visits fine point (i,j,k) with parity
   * (srcoff+i)%2 and coarse base (srcoff+i)/2 in every direction. */
  for (int k = 0; k < regext[2]; ++k) {
    int sk = srcoff[2] + k, dk = sk & 1, ks = sk >> 1;
    for (int j = 0; j < regext[1]; ++j) {
      int sj = srcoff[1] + j, dj = sj & 1, js = sj >> 1;
      for (int i = 0; i < regext[0]; ++i) {
        int si = srcoff[0] + i, di = si & 1, is = si >> 1;
        double res;
        /* interp3<di,dj,dk>: z outer, y middle, x inner */
        int nk = dk ? n : 1, nj = dj ? n : 1;
        int k0 = dk ? ks + imin : ks, j0 = dj ? js + imin : js;
        for (int kk = 0; kk < nk; ++kk) {
          for (int jj = 0; jj < nj; ++jj) {
            const double *p = &src[IDX(is, j0 + jj, k0 + kk, srcpadext)];
            /* interp1<di>: di==0 returns *p (:163-164) */
            ybuf[jj] = di ? vc_line(fma_, c, n, p + imin, 1) : *p;
          }
          zbuf[kk] = dj ? acc_sum(fma_, c, n, ybuf) : ybuf[0];
        }
        res = dk ? acc_sum(fma_, c, n, zbuf) : zbuf[0];
        dst[IDX(dstoff[0] + i, dstoff[1] + j, dstoff[2] + k, dstpadext)] = res;
      }
    }
  }
  return CGXO_OK;
}

/* ------------------------------------------------------------------ */
/* prolongate_3d_cc_rf2, CarpetLib/src/prolongate_3d_cc_rf2.cc:238-579 */

/* coeffs1dc<RT,ORDER>::coeffs, prolongate_3d_cc_rf2.cc:116-139 */
static int cc_coeffs(int order, double *c) {
  static const double n0[] = {1}, n1[] = {1, 3}, n2[] = {5, 30, -3},
                      n3[] = {-5, 35, 105, -7},
                      n4[] = {-45, 420, 1890, -252, 35},
                      n5[] = {63, -495, 2310, 6930, -693, 77};
  static const double dens[] = {1.0, 4.0, 32.0, 128.0, 2048.0, 8192.0};
  static const double *nums[] = {n0, n1, n2, n3, n4, n5};
  if (order < 0 || order > 5) return 0;
  for (int i = 0; i <= order; ++i) c[i] = nums[order][i] / dens[order];
  return order + 1;
}
/* coeffs1d<RT,ORDER,di>::imin, :57 */
static int cc_imin(int order, int di) {
  int n = order + 1;
  return -n / 2 + (order % 2 != 0 ? di : 0);
}
/* coeffs1d::get, :60-72: reversed for di == 1 */
static void cc_stencil(int order, int di, const double *c, double *out) {
  int n = order + 1;
  for (int m = 0; m < n; ++m) out[m] = di == 0 ? c[m] : c[n - 1 - m];
}

int cgxo_prolongate_3d_cc_rf2(int order, int fma_, const double *src,
                              const int *srcpadext, const int *srcext,
                              double *dst, const int *dstpadext,
                              const int *dstext, const int *srcbbox_,
                              const int *dstbbox_, const int *srcregbbox_,
                              const int *regbbox_) {
  (void)srcregbbox_; (void)dstext; (void)srcext;
  double c[6], st[2][6];
  int n = cc_coeffs(order, c);
  if (!n) return fail(CGXO_EUNSUPPORTED, "prolongate_3d_cc_rf2: no stencil of order %d", order);
  cc_stencil(order, 0, c, st[0]);
  cc_stencil(order, 1, c, st[1]);
  box_t srcbbox = mkbox(srcbbox_), dstbbox = mkbox(dstbbox_), reg = mkbox(regbbox_);
  /* :253-272 */
  for (int d = 0; d < 3; ++d) {
    if (srcbbox.str[d] <= reg.str[d] || dstbbox.str[d] != reg.str[d])
      return fail(CGXO_EINVAL, "prolongate_3d_cc_rf2: strides disagree");
    if (srcbbox.str[d] != 2 * dstbbox.str[d])
      return fail(CGXO_EINVAL, "prolongate_3d_cc_rf2: source strides are not twice the destination strides");
    if (dstbbox.str[d] % 2 != 0)
      return fail(CGXO_EINVAL, "prolongate_3d_cc_rf2: destination strides are not even");
  }
  if (box_empty(&reg))
    return fail(CGXO_EINVAL, "prolongate_3d_cc_rf2: region extent is empty");
  /* :274-321 */
  int regext[3], srcoff[3], dstoff[3], offlo[3], offhi[3];
  for (int d = 0; d < 3; ++d) {
    regext[d] = box_size(&reg, d);
    int h = reg.str[d] / 2;
    if ((reg.lo[d] - srcbbox.lo[d] + h) % reg.str[d] ||
        (reg.lo[d] - dstbbox.lo[d]) % reg.str[d] ||
        (reg.up[d] - srcbbox.lo[d] + h) % reg.str[d])
      return fail(CGXO_EINVAL, "prolongate_3d_cc_rf2: region not aligned");
    srcoff[d] = (reg.lo[d] - srcbbox.lo[d] + h) / reg.str[d];
    dstoff[d] = (reg.lo[d] - dstbbox.lo[d]) / reg.str[d];
    int srcend = (reg.up[d] - srcbbox.lo[d] + h) / reg.str[d];
    int nlo = srcoff[d] % 2, nhi = srcend % 2;
    offlo[d] = -cc_imin(order, nlo);
    offhi[d] = cc_imin(order, nhi) + n - 1;
  }
  box_t ex = box_expand(&reg, offlo, offhi);
  if (!box_in(&ex, &srcbbox) || !box_in(&reg, &dstbbox))
    return fail(CGXO_EINVAL, "prolongate_3d_cc_rf2: region extent is not contained in array extent");
  double ybuf[6], zbuf[6];
  /* same goto-nest as the vertex-centred operator (:372-579) */
  for (int k = 0; k < regext[2]; ++k) {
    int sk = srcoff[2] + k, dk = sk & 1, ks = sk >> 1;
    int k0 = ks + cc_imin(order, dk);
    for (int j = 0; j < regext[1]; ++j) {
      int sj = srcoff[1] + j, dj = sj & 1, js = sj >> 1;
      int j0 = js + cc_imin(order, dj);
      for (int i = 0; i < regext[0]; ++i) {
        int si = srcoff[0] + i, di = si & 1, is = si >> 1;
        int i0 = is + cc_imin(order, di);
        /* interp3 (:184-195), interp2 (:170-181), interp1 (:157-167):
         * every level is res = 0; res += c*inner */
        for (int kk = 0; kk < n; ++kk) {
          for (int jj = 0; jj < n; ++jj)
            ybuf[jj] = acc_sum(fma_, st[di], n,
                               &src[IDX(i0, j0 + jj, k0 + kk, srcpadext)]);
          zbuf[kk] = acc_sum(fma_, st[dj], n, ybuf);
        }
        dst[IDX(dstoff[0] + i, dstoff[1] + j, dstoff[2] + k, dstpadext)] =
            acc_sum(fma_, st[dk], n, zbuf);
      }
    }
  }
  return CGXO_OK;
}

/* ------------------------------------------------------------------ */
/* prolongate_3d_real8_eno, CarpetLib/src/prolongate_3d_real8_eno.F90   */

/* eno1d, prolongate_3d_real8_eno.F90:23-76 (Fortran left-to-right
 * evaluation; q[0..3] are q(1..4)) */
static double eno1d(int fma_, const double *q) {
  const double eighth = 1.0 / 8.0, half = 0.5;
  double diffleft = (q[0] + q[2]) - 2.0 * q[1];
  double diffright = (q[1] + q[3]) - 2.0 * q[2];
  double r;
  if (fabs(diffleft) < fabs(diffright)) {
    /* eighth * (-q(1) + six * q(2) + three * q(3)) */
    double t = madd(fma_, 6.0, q[1], -q[0]);
    t = madd(fma_, 3.0, q[2], t);
    r = eighth * t;
  } else {
    /* eighth * (three * q(2) + six * q(3) - q(4)) */
    double t = madd(fma_, 3.0, q[1], 6.0 * q[2]);
    t = t - q[3];
    r = eighth * t;
  }
  if ((r - q[1]) * (q[2] - r) < 0.0 || diffleft * diffright <= 0.0)
    r = half * (q[1] + q[2]);
  return r;
}

int cgxo_prolongate_3d_eno(int fma_, const double *src, const int *srcpadext,
                           const int *srcext, double *dst, const int *dstpadext,
                           const int *dstext, const int *srcbbox_,
                           const int *dstbbox_, const int *srcregbbox_,
                           const int *regbbox_) {
  (void)srcregbbox_;
  box_t srcbbox = mkbox(srcbbox_), dstbbox = mkbox(dstbbox_), reg = mkbox(regbbox_);
  int fac[3], srcoff[3], dstoff[3], regext[3];
  /* F90:122-166 */
  for (int d = 0; d < 3; ++d) {
    if (srcbbox.str[d] == 0 || dstbbox.str[d] == 0 || reg.str[d] == 0)
      return fail(CGXO_EINVAL, "prolongate_3d_eno: stride is zero");
    if (srcbbox.str[d] <= reg.str[d] || dstbbox.str[d] != reg.str[d])
      return fail(CGXO_EINVAL, "prolongate_3d_eno: strides disagree");
    if (srcbbox.str[d] % dstbbox.str[d] != 0)
      return fail(CGXO_EINVAL, "prolongate_3d_eno: strides are not integer multiples");
    if (srcbbox.lo[d] % srcbbox.str[d] || dstbbox.lo[d] % dstbbox.str[d] ||
        reg.lo[d] % reg.str[d])
      return fail(CGXO_EINVAL, "prolongate_3d_eno: array origins are not multiples of the strides");
    if (reg.lo[d] > reg.up[d])
      return fail(CGXO_EINVAL, "prolongate_3d_eno: region extent is empty");
    int ext = (reg.up[d] - reg.lo[d]) / reg.str[d] + 1;
    int f = srcbbox.str[d] / dstbbox.str[d];
    int off = (reg.lo[d] - srcbbox.lo[d]) / dstbbox.str[d];
    int olo = reg.str[d];
    if ((off + 0) % f == 0) { olo = 0; if (ext > 1) olo = reg.str[d]; }
    int ohi = reg.str[d];
    if ((off + ext - 1) % f == 0) { ohi = 0; if (ext > 1) ohi = reg.str[d]; }
    if (reg.lo[d] - olo < srcbbox.lo[d] || reg.up[d] + ohi > srcbbox.up[d] ||
        reg.lo[d] < dstbbox.lo[d] || reg.up[d] > dstbbox.up[d])
      return fail(CGXO_EINVAL, "prolongate_3d_eno: region extent is not contained in array extent");
  }
  /* F90:168-175 */
  for (int d = 0; d < 3; ++d)
    if (srcext[d] != (srcbbox.up[d] - srcbbox.lo[d]) / srcbbox.str[d] + 1 ||
        dstext[d] != (dstbbox.up[d] - dstbbox.lo[d]) / dstbbox.str[d] + 1)
      return fail(CGXO_EINVAL, "prolongate_3d_eno: array sizes don't agree with bounding boxes");
  for (int d = 0; d < 3; ++d) {
    regext[d] = (reg.up[d] - reg.lo[d]) / reg.str[d] + 1;
    fac[d] = srcbbox.str[d] / dstbbox.str[d];
    srcoff[d] = (reg.lo[d] - srcbbox.lo[d]) / dstbbox.str[d];
    dstoff[d] = (reg.lo[d] - dstbbox.lo[d]) / dstbbox.str[d];
  }
  /* F90:195-285; Fortran index i0+1 is C index i0, i0:i0+3 is i0-1..i0+2 */
  for (int k = 0; k < regext[2]; ++k)
    for (int j = 0; j < regext[1]; ++j)
      for (int i = 0; i < regext[0]; ++i) {
        int i0 = (srcoff[0] + i) / fac[0], fi = (srcoff[0] + i) % fac[0];
        int j0 = (srcoff[1] + j) / fac[1], fj = (srcoff[1] + j) % fac[1];
        int k0 = (srcoff[2] + k) / fac[2], fk = (srcoff[2] + k) % fac[2];
        if (fi > 1 || fj > 1 || fk > 1)
          return fail(CGXO_EINVAL, "prolongate_3d_eno: refinement factor must be 2");
        double q[4], t2[4], t1[4][4], r;
#define S(a, b, c) src[IDX(a, b, c, srcpadext)]
        switch (fi + 10 * fj + 100 * fk) {
        case 0: r = S(i0, j0, k0); break;
        case 1:
          for (int m = 0; m < 4; ++m) q[m] = S(i0 - 1 + m, j0, k0);
          r = eno1d(fma_, q); break;
        case 10:
          for (int m = 0; m < 4; ++m) q[m] = S(i0, j0 - 1 + m, k0);
          r = eno1d(fma_, q); break;
        case 11:
          for (int jj = 0; jj < 4; ++jj) {
            for (int m = 0; m < 4; ++m) q[m] = S(i0 - 1 + m, j0 - 1 + jj, k0);
            t2[jj] = eno1d(fma_, q);
          }
          r = eno1d(fma_, t2); break;
        case 100:
          for (int m = 0; m < 4; ++m) q[m] = S(i0, j0, k0 - 1 + m);
          r = eno1d(fma_, q); break;
        case 101:
          for (int kk = 0; kk < 4; ++kk) {
            for (int m = 0; m < 4; ++m) q[m] = S(i0 - 1 + m, j0, k0 - 1 + kk);
            t2[kk] = eno1d(fma_, q);
          }
          r = eno1d(fma_, t2); break;
        case 110:
          for (int kk = 0; kk < 4; ++kk) {
            for (int m = 0; m < 4; ++m) q[m] = S(i0, j0 - 1 + m, k0 - 1 + kk);
            t2[kk] = eno1d(fma_, q);
          }
          r = eno1d(fma_, t2); break;
        default: /* 111, F90:266-279: x rows, then y, then z */
          for (int jj = 0; jj < 4; ++jj)
            for (int kk = 0; kk < 4; ++kk) {
              for (int m = 0; m < 4; ++m) q[m] = S(i0 - 1 + m, j0 - 1 + jj, k0 - 1 + kk);
              t1[jj][kk] = eno1d(fma_, q);
            }
          for (int ii = 0; ii < 4; ++ii) {
            for (int m = 0; m < 4; ++m) q[m] = t1[m][ii];
            t2[ii] = eno1d(fma_, q);
          }
          r = eno1d(fma_, t2); break;
        }
#undef S
        dst[IDX(dstoff[0] + i, dstoff[1] + j, dstoff[2] + k, dstpadext)] = r;
      }
  return CGXO_OK;
}

/* ------------------------------------------------------------------ */
/* prolongate_3d_cc_eno_rf2, CarpetLib/src/prolongate_3d_cc_eno_rf2.cc  */
/* (ORDER 2 and 3; data.cc:689-720 maps order_space 2-4 to 2, 5 to 3)  */

/* coeffs1dc<RT,ORDER,OFFSET> (:144-176), exact dyadic rationals */
static const double ceno_first[2] = {1 / 4.0, 3 / 4.0};                 /* <1,0> */
static const double ceno2_0[3] = {5 / 32.0, 30 / 32.0, -3 / 32.0};      /* <2,0> */
static const double ceno2_m[3] = {-3 / 32.0, 14 / 32.0, 21 / 32.0};     /* <2,-1> */
static const double ceno3_0[4] = {-5 / 128.0, 35 / 128.0, 105 / 128.0, -7 / 128.0};
static const double ceno3_p[4] = {15 / 128.0, 135 / 128.0, -27 / 128.0, 5 / 128.0};
static const double ceno3_m[4] = {7 / 128.0, -33 / 128.0, 77 / 128.0, 77 / 128.0};

/* coeffs1d<>::get (:73-85): res = 0; res += get(i) * f(i) for i from imin,
 * the table reversed for the odd parity; p points at the coarse base */
static double ceno_sum(int fma_, const double *tab, int n, int imin, int di, const double *p) {
  double r = 0.0;
  for (int i = imin; i < imin + n; ++i) {
    int j = di == 0 ? i - imin : n - 1 - (i - imin);
    r = madd(fma_, tab[j], p[i], r);
  }
  return r;
}
/* the undivided differences, diffC1dc (:171-174) applied with coeffs1d::diff
 * (:87-96, never reversed) */
static double ceno_diff(int fma_, int order, int imin, const double *p) {
  static const double d2[3] = {1, -2, 1}, d3[4] = {1, -3, 3, -1};
  const double *d = order == 2 ? d2 : d3;
  double r = 0.0;
  for (int i = imin; i < imin + order + 1; ++i) r = madd(fma_, d[i - imin], p[i], r);
  return r;
}
/* one axis of interp1/interp2/interp3 (:198-371, the three are the same
 * rule): the smoothest of the shifted stencils, first order where the
 * differences change sign or the result leaves [f(di-1), f(di)].  The
 * window is f(-2+di) .. f(1+di) for ORDER 2 and f(-3+di) .. f(2+di) for 3. */
static double ceno1d(int fma_, int order, int di, const double *p) {
  double res;
  if (order == 2) {
    const int shift = di == 0 ? -1 : 1; /* :225-231 */
    double lV = ceno_diff(fma_, 2, -1 + shift, p);
    double rV = ceno_diff(fma_, 2, -1, p);
    if (lV * rV <= 0)
      res = ceno_sum(fma_, ceno_first, 2, -1 + di, di, p);
    else if (fabs(lV) < fabs(rV))
      res = ceno_sum(fma_, ceno2_m, 3, -1 + shift, di, p);
    else
      res = ceno_sum(fma_, ceno2_0, 3, -1, di, p);
  } else {
    /* shifts -1, 0, +1 (:289-306); coeffs1dc<3, di == 0 ? OFFSET : -OFFSET> */
    const double *tl = di == 0 ? ceno3_m : ceno3_p, *tr = di == 0 ? ceno3_p : ceno3_m;
    double V[3];
    V[0] = ceno_diff(fma_, 3, -3 + di, p);
    V[1] = ceno_diff(fma_, 3, -2 + di, p);
    V[2] = ceno_diff(fma_, 3, -1 + di, p);
    if (V[0] * V[2] <= 0 || V[0] * V[1] <= 0 || V[1] * V[2] <= 0)
      return ceno_sum(fma_, ceno_first, 2, -1 + di, di, p); /* :311-329 */
    int min = 1;
    for (int i = 0; i < 3; ++i)
      if (fabs(V[i]) < fabs(V[min])) min = i;
    if (min == 0) res = ceno_sum(fma_, tl, 4, -3 + di, di, p);
    else if (min == 1) res = ceno_sum(fma_, ceno3_0, 4, -2 + di, di, p);
    else res = ceno_sum(fma_, tr, 4, -1 + di, di, p);
  }
  /* :366-395 */
  if ((res - p[di - 1]) * (p[di] - res) < 0)
    res = ceno_sum(fma_, ceno_first, 2, -1 + di, di, p);
  return res;
}

int cgxo_prolongate_3d_cc_eno_rf2(int order, int fma_, const double *src,
                                  const int *srcpadext, const int *srcext,
                                  double *dst, const int *dstpadext,
                                  const int *dstext, const int *srcbbox_,
                                  const int *dstbbox_, const int *srcregbbox_,
                                  const int *regbbox_) {
  (void)srcregbbox_; (void)dstext;
  if (order != 2 && order != 3)
    return fail(CGXO_EUNSUPPORTED, "prolongate_3d_cc_eno_rf2: no stencil of order %d", order);
  box_t srcbbox = mkbox(srcbbox_), dstbbox = mkbox(dstbbox_), reg = mkbox(regbbox_);
  /* :962-981 */
  for (int d = 0; d < 3; ++d) {
    if (srcbbox.str[d] <= reg.str[d] || dstbbox.str[d] != reg.str[d])
      return fail(CGXO_EINVAL, "prolongate_3d_cc_eno_rf2: strides disagree");
    if (srcbbox.str[d] != 2 * dstbbox.str[d])
      return fail(CGXO_EINVAL, "prolongate_3d_cc_eno_rf2: source strides are not twice the destination strides");
    if (dstbbox.str[d] % 2 != 0)
      return fail(CGXO_EINVAL, "prolongate_3d_cc_eno_rf2: destination strides are not even");
  }
  if (box_empty(&reg))
    return fail(CGXO_EINVAL, "prolongate_3d_cc_eno_rf2: region extent is empty");
  /* :983-1031: window of the parity at each end, in fine strides */
  const int mm = order == 2 ? -2 : -3; /* coeffs1d<ORDER,di>::minimin - di */
  int regext[3], srcoff[3], dstoff[3], offlo[3], offhi[3];
  for (int d = 0; d < 3; ++d) {
    regext[d] = box_size(&reg, d);
    int h = reg.str[d] / 2;
    if ((reg.lo[d] - srcbbox.lo[d] + h) % reg.str[d] ||
        (reg.lo[d] - dstbbox.lo[d]) % reg.str[d] ||
        (reg.up[d] - srcbbox.lo[d] + h) % reg.str[d])
      return fail(CGXO_EINVAL, "prolongate_3d_cc_eno_rf2: region not aligned");
    srcoff[d] = (reg.lo[d] - srcbbox.lo[d] + h) / reg.str[d];
    dstoff[d] = (reg.lo[d] - dstbbox.lo[d]) / reg.str[d];
    int srcend = (reg.up[d] - srcbbox.lo[d] + h) / reg.str[d];
    offlo[d] = -(mm + srcoff[d] % 2);
    offhi[d] = -mm + srcend % 2 - 1;
  }
  box_t ex = box_expand(&reg, offlo, offhi);
  if (!box_in(&ex, &srcbbox) || !box_in(&reg, &dstbbox))
    return fail(CGXO_EINVAL, "prolongate_3d_cc_eno_rf2: region extent is not contained in array extent");
  /* that test counts fine strides; the coarse points actually read must be
   * inside the source too (the reference only asserts it, :905-941) */
  for (int d = 0; d < 3; ++d) {
    /* fine point s reads coarse ceil(s/2) + mm .. ceil(s/2) - mm - 1 */
    int s0 = srcoff[d], s1 = srcoff[d] + regext[d] - 1;
    int lo = (s0 + 1) / 2 + mm, hi = (s1 + 1) / 2 - mm - 1;
    if (lo < 0 || hi >= srcext[d])
      return fail(CGXO_EINVAL, "prolongate_3d_cc_eno_rf2: stencil reaches outside the source array");
  }
  const int W = order == 2 ? 2 : 3; /* window f(-W+di) .. f(W-1+di) */
  double xb[8], yb[8];
  for (int k = 0; k < regext[2]; ++k) {
    int sk = srcoff[2] + k, dk = sk & 1, ks = sk >> 1;
    for (int j = 0; j < regext[1]; ++j) {
      int sj = srcoff[1] + j, dj = sj & 1, js = sj >> 1;
      for (int i = 0; i < regext[0]; ++i) {
        int si = srcoff[0] + i, di = si & 1, is = si >> 1;
        /* interp3 over interp2 over interp1 (:722-760) */
        for (int kk = -W + dk; kk < W + dk; ++kk) {
          for (int jj = -W + dj; jj < W + dj; ++jj)
            xb[4 + jj] = ceno1d(fma_, order, di, &src[IDX(is, js + jj, ks + kk, srcpadext)]);
          yb[4 + kk] = ceno1d(fma_, order, dj, &xb[4]);
        }
        dst[IDX(dstoff[0] + i, dstoff[1] + j, dstoff[2] + k, dstpadext)] =
            ceno1d(fma_, order, dk, &yb[4]);
      }
    }
  }
  return CGXO_OK;
}

/* ------------------------------------------------------------------ */
/* prolongate_3d_o5_monotone_rf2, CarpetLib/src/                        */
/* prolongate_3d_o5_monotone_rf2.cc:45-793 (op Lagrange_monotone)       */

/* std::min / std::max, argument order kept (NaN and signed-zero ties) */
static double smin(double a, double b) { return b < a ? b : a; }
static double smax(double a, double b) { return a < b ? b : a; }

/* The fine point with coarse base b[3] whose odd axes are ax[0..n-1]
 * (increasing): n = 0 copies; otherwise the tensor-product order-5 stencil
 * over coarse b-2 .. b+3 on the odd axes, summed left to right with the
 * lowest odd axis fastest and weight f_a * f_b (* f_c) formed left to
 * right; with three odd axes each z plane is its own partial sum and the
 * six are added in order (:499-716).  A result outside the nearest 2/4/8
 * coarse values (min/max nested as min4/max4/min8/max8, :19-43) falls back
 * to linear, bilinear or trilinear interpolation. */
static double mono_point(int fma_, const double *src, const int *pad, const int *b,
                         const int *ax, int n) {
  static const double f[6] = {3.0 / 256, -25.0 / 256, 150.0 / 256, 150.0 / 256, -25.0 / 256,
                              3.0 / 256};
  const double h = 0.5;
#define MS(o0, o1, o2) src[IDX(b[0] + (o0), b[1] + (o1), b[2] + (o2), pad)]
  int e[3][3] = {{0}}; /* unit offset along odd axis m */
  for (int m = 0; m < n; ++m) e[m][ax[m]] = 1;
  if (n == 0) return MS(0, 0, 0);
  double res;
  if (n == 1) {
    res = f[0] * MS(-2 * e[0][0], -2 * e[0][1], -2 * e[0][2]);
    for (int m = 1; m < 6; ++m)
      res = madd(fma_, f[m], MS((m - 2) * e[0][0], (m - 2) * e[0][1], (m - 2) * e[0][2]), res);
    double v0 = MS(0, 0, 0), v1 = MS(e[0][0], e[0][1], e[0][2]);
    if (res > smax(v0, v1) || res < smin(v0, v1)) res = madd(fma_, h, v1, h * v0);
    return res;
  }
  if (n == 2) {
    res = 0;
    for (int q = 0; q < 36; ++q) {
      int m0 = q % 6 - 2, m1 = q / 6 - 2;
      double w = f[q % 6] * f[q / 6];
      double v = MS(m0 * e[0][0] + m1 * e[1][0], m0 * e[0][1] + m1 * e[1][1],
                    m0 * e[0][2] + m1 * e[1][2]);
      res = q == 0 ? w * v : madd(fma_, w, v, res);
    }
    double x1 = MS(0, 0, 0), x2 = MS(e[0][0], e[0][1], e[0][2]), x3 = MS(e[1][0], e[1][1], e[1][2]),
           x4 = MS(e[0][0] + e[1][0], e[0][1] + e[1][1], e[0][2] + e[1][2]);
    if (res > smax(smax(x1, x2), smax(x3, x4)) || res < smin(smin(x1, x2), smin(x3, x4))) {
      const double w = h * h;
      res = w * x1;
      res = madd(fma_, w, x2, res);
      res = madd(fma_, w, x3, res);
      res = madd(fma_, w, x4, res);
    }
    return res;
  }
  double part[6];
  for (int c = 0; c < 6; ++c) {
    double r = 0;
    for (int q = 0; q < 36; ++q) {
      double w = f[q % 6] * f[q / 6] * f[c];
      double v = MS(q % 6 - 2, q / 6 - 2, c - 2);
      r = q == 0 ? w * v : madd(fma_, w, v, r);
    }
    part[c] = r;
  }
  res = part[0];
  for (int c = 1; c < 6; ++c) res = res + part[c];
  /* max8 (:39-43) of x1 (0,0,0), x2 (1,0,0), x3 (0,1,0), x4 (0,0,1),
   * x5 (1,1,0), x6 (1,0,1), x7 (0,1,1), x8 (1,1,1) */
  double x[8] = {MS(0, 0, 0), MS(1, 0, 0), MS(0, 1, 0), MS(0, 0, 1),
                 MS(1, 1, 0), MS(1, 0, 1), MS(0, 1, 1), MS(1, 1, 1)};
  double mx = smax(smax(smax(x[0], x[1]), smax(x[2], x[3])), smax(smax(x[4], x[5]), smax(x[6], x[7])));
  double mn = smin(smin(smin(x[0], x[1]), smin(x[2], x[3])), smin(smin(x[4], x[5]), smin(x[6], x[7])));
  if (res > mx || res < mn) {
    const double w = h * h * h;
    /* :730-738: the z = 0 plane, then the z = 1 plane, each x fastest */
    double r1 = w * x[0];
    r1 = madd(fma_, w, x[1], r1);
    r1 = madd(fma_, w, x[2], r1);
    r1 = madd(fma_, w, x[4], r1);
    double r2 = w * x[3];
    r2 = madd(fma_, w, x[5], r2);
    r2 = madd(fma_, w, x[6], r2);
    r2 = madd(fma_, w, x[7], r2);
    res = r1 + r2;
  }
  return res;
#undef MS
}

int cgxo_prolongate_3d_o5_monotone_rf2(int fma_, const double *src, const int *srcpadext,
                                       const int *srcext, double *dst, const int *dstpadext,
                                       const int *dstext, const int *srcbbox_,
                                       const int *dstbbox_, const int *srcregbbox_,
                                       const int *regbbox_) {
  (void)srcregbbox_; (void)dstext;
  box_t srcbbox = mkbox(srcbbox_), dstbbox = mkbox(dstbbox_), reg = mkbox(regbbox_);
  /* :72-86 */
  for (int d = 0; d < 3; ++d) {
    if (srcbbox.str[d] <= reg.str[d] || dstbbox.str[d] != reg.str[d])
      return fail(CGXO_EINVAL, "prolongate_3d_o5_monotone_rf2: strides disagree");
    if (srcbbox.str[d] != 2 * dstbbox.str[d])
      return fail(CGXO_EINVAL, "prolongate_3d_o5_monotone_rf2: source strides are not twice the destination strides");
  }
  if (box_empty(&reg))
    return fail(CGXO_EINVAL, "prolongate_3d_o5_monotone_rf2: region extent is empty");
  /* :88-104 */
  int regext[3], srcoff[3], dstoff[3], offlo[3], offhi[3];
  for (int d = 0; d < 3; ++d) {
    regext[d] = box_size(&reg, d);
    if ((reg.lo[d] - srcbbox.lo[d]) % reg.str[d] || (reg.lo[d] - dstbbox.lo[d]) % reg.str[d])
      return fail(CGXO_EINVAL, "prolongate_3d_o5_monotone_rf2: region not aligned");
    srcoff[d] = (reg.lo[d] - srcbbox.lo[d]) / reg.str[d];
    dstoff[d] = (reg.lo[d] - dstbbox.lo[d]) / reg.str[d];
    offlo[d] = (srcoff[d] % 2 != 0 || regext[d] > 1) ? 3 : 0;
    offhi[d] = ((srcoff[d] + regext[d] - 1) % 2 != 0 || regext[d] > 1) ? 3 : 0;
  }
  box_t ex = box_expand(&reg, offlo, offhi);
  if (!box_in(&ex, &srcbbox) || !box_in(&reg, &dstbbox))
    return fail(CGXO_EINVAL, "prolongate_3d_o5_monotone_rf2: region extent is not contained in array extent");
  /* the coarse points actually read must be inside the source too: an odd
   * fine point s reads s/2 - 2 .. s/2 + 3, an even one s/2 */
  for (int d = 0; d < 3; ++d) {
    int lo = 1 << 30, hi = -(1 << 30);
    for (int s = srcoff[d]; s < srcoff[d] + regext[d] && s < srcoff[d] + 2; ++s) {
      int a = s % 2 ? s / 2 - 2 : s / 2;
      if (a < lo) lo = a;
    }
    for (int s = srcoff[d] + regext[d] - 1; s >= srcoff[d] && s > srcoff[d] + regext[d] - 3; --s) {
      int a = s % 2 ? s / 2 + 3 : s / 2;
      if (a > hi) hi = a;
    }
    if (lo < 0 || hi >= srcext[d])
      return fail(CGXO_EINVAL, "prolongate_3d_o5_monotone_rf2: stencil reaches outside the source array");
  }
  for (int k = 0; k < regext[2]; ++k)
    for (int j = 0; j < regext[1]; ++j)
      for (int i = 0; i < regext[0]; ++i) {
        const int s[3] = {srcoff[0] + i, srcoff[1] + j, srcoff[2] + k};
        int b[3], ax[3], n = 0;
        for (int d = 0; d < 3; ++d) {
          b[d] = s[d] / 2;
          if (s[d] % 2) ax[n++] = d;
        }
        dst[IDX(dstoff[0] + i, dstoff[1] + j, dstoff[2] + k, dstpadext)] =
            mono_point(fma_, src, srcpadext, b, ax, n);
      }
  return CGXO_OK;
}

/* ------------------------------------------------------------------ */
/* restrict_3d_rf2, CarpetLib/src/restrict_3d_rf2.cc:25-121             */

int cgxo_restrict_3d_rf2(const double *src, const int *srcpadext,
                         const int *srcext, double *dst, const int *dstpadext,
                         const int *dstext, const int *srcbbox_,
                         const int *dstbbox_, const int *srcregbbox_,
                         const int *regbbox_) {
  (void)srcregbbox_; (void)srcext; (void)dstext;
  box_t srcbbox = mkbox(srcbbox_), dstbbox = mkbox(dstbbox_), reg = mkbox(regbbox_);
  for (int d = 0; d < 3; ++d) {
    if (srcbbox.str[d] >= reg.str[d] || dstbbox.str[d] != reg.str[d])
      return fail(CGXO_EINVAL, "restrict_3d_rf2: strides disagree");
    if (2 * srcbbox.str[d] != dstbbox.str[d])
      return fail(CGXO_EINVAL, "restrict_3d_rf2: destination strides are not twice the source strides");
  }
  if (box_empty(&reg))
    return fail(CGXO_EINVAL, "restrict_3d_rf2: region extent is empty");
  if (!box_in(&reg, &srcbbox) || !box_in(&reg, &dstbbox))
    return fail(CGXO_EINVAL, "restrict_3d_rf2: region extent is not contained in array extent");
  int regext[3], srcoff[3], dstoff[3];
  for (int d = 0; d < 3; ++d) {
    regext[d] = box_size(&reg, d);
    if ((reg.lo[d] - srcbbox.lo[d]) % srcbbox.str[d] ||
        (reg.lo[d] - dstbbox.lo[d]) % dstbbox.str[d])
      return fail(CGXO_EINVAL, "restrict_3d_rf2: region not aligned");
    srcoff[d] = (reg.lo[d] - srcbbox.lo[d]) / srcbbox.str[d];
    dstoff[d] = (reg.lo[d] - dstbbox.lo[d]) / dstbbox.str[d];
  }
  for (int k = 0; k < regext[2]; ++k)
    for (int j = 0; j < regext[1]; ++j)
      for (int i = 0; i < regext[0]; ++i)
        dst[IDX(dstoff[0] + i, dstoff[1] + j, dstoff[2] + k, dstpadext)] =
            src[IDX(srcoff[0] + 2 * i, srcoff[1] + 2 * j, srcoff[2] + 2 * k, srcpadext)];
  return CGXO_OK;
}

/* ------------------------------------------------------------------ */
/* restrict_3d_cc_rf2, CarpetLib/src/restrict_3d_cc_rf2.cc:23-152       */

int cgxo_restrict_3d_cc_rf2(int fma_, const double *src, const int *srcpadext,
                            const int *srcext, double *dst,
                            const int *dstpadext, const int *dstext,
                            const int *srcbbox_, const int *dstbbox_,
                            const int *srcregbbox_, const int *regbbox_) {
  (void)srcregbbox_; (void)srcext; (void)dstext;
  box_t srcbbox = mkbox(srcbbox_), dstbbox = mkbox(dstbbox_), reg = mkbox(regbbox_);
  for (int d = 0; d < 3; ++d) {
    if (srcbbox.str[d] >= reg.str[d] || dstbbox.str[d] != reg.str[d])
      return fail(CGXO_EINVAL, "restrict_3d_cc_rf2: strides disagree");
    if (2 * srcbbox.str[d] != dstbbox.str[d])
      return fail(CGXO_EINVAL, "restrict_3d_cc_rf2: destination strides are not twice the source strides");
  }
  if (box_empty(&reg))
    return fail(CGXO_EINVAL, "restrict_3d_cc_rf2: region extent is empty");
  box_t ef = box_expanded_for(&reg, &srcbbox);
  if (!box_in(&ef, &srcbbox) || !box_in(&reg, &dstbbox))
    return fail(CGXO_EINVAL, "restrict_3d_cc_rf2: region extent is not contained in array extent");
  int regext[3], srcoff[3], dstoff[3];
  for (int d = 0; d < 3; ++d) {
    regext[d] = box_size(&reg, d);
    int h = srcbbox.str[d] / 2;
    if (srcbbox.str[d] % 2 || (reg.lo[d] - srcbbox.lo[d] - h) % srcbbox.str[d] ||
        (reg.lo[d] - dstbbox.lo[d]) % dstbbox.str[d])
      return fail(CGXO_EINVAL, "restrict_3d_cc_rf2: region not aligned");
    srcoff[d] = (reg.lo[d] - srcbbox.lo[d] - h) / srcbbox.str[d];
    dstoff[d] = (reg.lo[d] - dstbbox.lo[d]) / dstbbox.str[d];
  }
  /* f1 = f2 = 1/2; every weight f*f*f is 1/8 (:237-240); the sum runs
   * left to right in the order of :252-260 */
  const double w = (0.5 * 0.5) * 0.5;
  static const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0},
                                {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
  for (int k = 0; k < regext[2]; ++k)
    for (int j = 0; j < regext[1]; ++j)
      for (int i = 0; i < regext[0]; ++i) {
        int a = srcoff[0] + 2 * i, b = srcoff[1] + 2 * j, cc = srcoff[2] + 2 * k;
        double res = w * src[IDX(a, b, cc, srcpadext)];
        for (int m = 1; m < 8; ++m)
          res = madd(fma_, w, src[IDX(a + off[m][0], b + off[m][1], cc + off[m][2], srcpadext)], res);
        dst[IDX(dstoff[0] + i, dstoff[1] + j, dstoff[2] + k, dstpadext)] = res;
      }
  return CGXO_OK;
}

/* ------------------------------------------------------------------ */
/* Higher-order cell-centred restriction, selected by CarpetLib's      */
/* use_higher_order_restriction / restriction_order_space parameters   */
/* (data.cc:1061-1097); cgxo_set_restriction mirrors them.             */

static int g_ho_restrict = 0, g_restrict_order = 1;

int cgxo_set_restriction(int use_higher_order, int order) {
  g_ho_restrict = use_higher_order != 0;
  g_restrict_order = order;
  return CGXO_OK;
}

/* region set-up shared by the cc restrictions: offsets of the region's
 * first fine cell (srcoff) and coarse point (dstoff); the source must hold
 * fine cells lo..hi around every coarse point (taps relative to 2i) */
static int cc_restrict_region(const char *who, const int *srcbbox_, const int *dstbbox_,
                              const int *regbbox_, const int *srcext, int lo, int hi,
                              int *regext, int *srcoff, int *dstoff) {
  box_t srcbbox = mkbox(srcbbox_), dstbbox = mkbox(dstbbox_), reg = mkbox(regbbox_);
  for (int d = 0; d < 3; ++d) {
    if (srcbbox.str[d] >= reg.str[d] || dstbbox.str[d] != reg.str[d])
      return fail(CGXO_EINVAL, "%s: strides disagree", who);
    if (2 * srcbbox.str[d] != dstbbox.str[d])
      return fail(CGXO_EINVAL, "%s: destination strides are not twice the source strides", who);
  }
  if (box_empty(&reg)) return fail(CGXO_EINVAL, "%s: region extent is empty", who);
  if (!box_in(&reg, &dstbbox))
    return fail(CGXO_EINVAL, "%s: region extent is not contained in array extent", who);
  for (int d = 0; d < 3; ++d) {
    regext[d] = box_size(&reg, d);
    int h = srcbbox.str[d] / 2;
    if (srcbbox.str[d] % 2 || (reg.lo[d] - srcbbox.lo[d] - h) % srcbbox.str[d] ||
        (reg.lo[d] - dstbbox.lo[d]) % dstbbox.str[d])
      return fail(CGXO_EINVAL, "%s: region not aligned", who);
    srcoff[d] = (reg.lo[d] - srcbbox.lo[d] - h) / srcbbox.str[d];
    dstoff[d] = (reg.lo[d] - dstbbox.lo[d]) / dstbbox.str[d];
    /* every tap inside the source (the stencil's own reach, :128-144) */
    if (srcoff[d] + lo < 0 || srcoff[d] + 2 * (regext[d] - 1) + hi >= srcext[d])
      return fail(CGXO_EINVAL, "%s: stencil reaches outside the source array", who);
  }
  return CGXO_OK;
}

/* restrict_3d_cc_o3_rf2, CarpetLib/src/restrict_3d_cc_o3_rf2.cc:33-229:
 * the 4x4x4 fine cells at 2i-1..2i+2 (per axis), weight c_a c_b c_c / 4096
 * with c = (-1, 9, 9, -1) (f1..f4 = 1, 9, 81, 729 over 4096, :114-119),
 * summed left to right with x fastest, then y, then z (:147-211) */
int cgxo_restrict_3d_cc_o3_rf2(int fma_, const double *src, const int *srcpadext,
                               const int *srcext, double *dst, const int *dstpadext,
                               const int *dstext, const int *srcbbox, const int *dstbbox,
                               const int *srcregbbox, const int *regbbox) {
  (void)srcregbbox; (void)dstext;
  int regext[3], srcoff[3], dstoff[3], rc;
  if ((rc = cc_restrict_region("restrict_3d_cc_o3_rf2", srcbbox, dstbbox, regbbox, srcext, -1, 2,
                               regext, srcoff, dstoff)))
    return rc;
  static const double c1[4] = {-1, 9, 9, -1};
  double w[64];
  for (int c = 0; c < 4; ++c)
    for (int b = 0; b < 4; ++b)
      for (int a = 0; a < 4; ++a) w[(c * 4 + b) * 4 + a] = (c1[a] * c1[b] * c1[c]) / 4096.0;
  for (int k = 0; k < regext[2]; ++k)
    for (int j = 0; j < regext[1]; ++j)
      for (int i = 0; i < regext[0]; ++i) {
        const int x0 = srcoff[0] + 2 * i - 1, y0 = srcoff[1] + 2 * j - 1, z0 = srcoff[2] + 2 * k - 1;
        double res = w[0] * src[IDX(x0, y0, z0, srcpadext)];
        for (int m = 1; m < 64; ++m)
          res = madd(fma_, w[m], src[IDX(x0 + (m & 3), y0 + ((m >> 2) & 3), z0 + (m >> 4), srcpadext)], res);
        dst[IDX(dstoff[0] + i, dstoff[1] + j, dstoff[2] + k, dstpadext)] = res;
      }
  return CGXO_OK;
}

/* restrict_3d_cc_o5_rf2, CarpetLib/src/restrict_3d_cc_o5_rf2.cc:36-78,
 * 159-193: separable, restrict3 over planes 2k-2..2k+3 of restrict2 over
 * rows of restrict1 over cells 2i-2..2i+3, each a left-to-right sum with
 * weights (3, -25, 150, 150, -25, 3) / 256 */
static const double o5w[6] = {3.0 / 256, -25.0 / 256, 150.0 / 256, 150.0 / 256, -25.0 / 256, 3.0 / 256};

static double o5_line(int fma_, const double *p, long long stride) {
  double r = o5w[0] * p[-2 * stride];
  for (int m = 1; m < 6; ++m) r = madd(fma_, o5w[m], p[(m - 2) * stride], r);
  return r;
}

int cgxo_restrict_3d_cc_o5_rf2(int fma_, const double *src, const int *srcpadext,
                               const int *srcext, double *dst, const int *dstpadext,
                               const int *dstext, const int *srcbbox, const int *dstbbox,
                               const int *srcregbbox, const int *regbbox) {
  (void)srcregbbox; (void)dstext;
  int regext[3], srcoff[3], dstoff[3], rc;
  if ((rc = cc_restrict_region("restrict_3d_cc_o5_rf2", srcbbox, dstbbox, regbbox, srcext, -2, 3,
                               regext, srcoff, dstoff)))
    return rc;
  const long long sy = srcpadext[0], sz = (long long)srcpadext[0] * srcpadext[1];
  for (int k = 0; k < regext[2]; ++k)
    for (int j = 0; j < regext[1]; ++j)
      for (int i = 0; i < regext[0]; ++i) {
        const double *p = src + IDX(srcoff[0] + 2 * i, srcoff[1] + 2 * j, srcoff[2] + 2 * k, srcpadext);
        double r3 = 0;
        for (int c = 0; c < 6; ++c) {
          double r2 = 0;
          for (int b = 0; b < 6; ++b) {
            const double r1 = o5_line(fma_, p + (c - 2) * sz + (b - 2) * sy, 1);
            r2 = b ? madd(fma_, o5w[b], r1, r2) : o5w[0] * r1;
          }
          r3 = c ? madd(fma_, o5w[c], r2, r3) : o5w[0] * r2;
        }
        dst[IDX(dstoff[0] + i, dstoff[1] + j, dstoff[2] + k, dstpadext)] = r3;
      }
  return CGXO_OK;
}

/* ------------------------------------------------------------------ */
/* Time interpolation                                                 */

static int ti_region(const box_t *srcbbox, const box_t *dstbbox, const box_t *reg,
                     int *regext, int *srcoff, int *dstoff, const char *who) {
  for (int d = 0; d < 3; ++d)
    if (srcbbox->str[d] != reg->str[d] || dstbbox->str[d] != reg->str[d])
      return fail(CGXO_EINVAL, "%s: strides disagree", who);
  if (box_empty(reg)) return fail(CGXO_EINVAL, "%s: region extent is empty", who);
  if (!box_in(reg, srcbbox) || !box_in(reg, dstbbox))
    return fail(CGXO_EINVAL, "%s: region extent is not contained in array extent", who);
  for (int d = 0; d < 3; ++d) {
    regext[d] = box_size(reg, d);
    srcoff[d] = (reg->lo[d] - srcbbox->lo[d]) / srcbbox->str[d];
    dstoff[d] = (reg->lo[d] - dstbbox->lo[d]) / dstbbox->str[d];
  }
  return CGXO_OK;
}

/* Time-interpolation weights, computed once per call exactly as the
 * reference does.  Returns CGXO_EINVAL for coincident times or
 * extrapolation.  kind: 1 = interpolate_3d_2tl.cc:232-242,
 * 2 = interpolate_3d_3tl.cc:365-382, 3 = interpolate_eno_3d_3tl.cc:105-135
 * (w[0..2] the 3-point weights, w[3..4] the (1,2) pair, w[5..6] the (2,3)
 * pair, w[7] = use_12). */
int cgxo_time_weights(int kind, const double *ts, double t, double *w) {
  if (kind == 4 || kind == 5) {
    /* interpolate_3d_4tl.cc:95-117, interpolate_3d_5tl.cc:100-123: Lagrange
     * in time, numerator and denominator products left to right */
    const int n = kind;
    const double eps = 1.0e-12;
    const char *who = n == 4 ? "interpolate_3d_4tl" : "interpolate_3d_5tl";
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j)
        if (fabs(ts[i] - ts[j]) < eps) return fail(CGXO_EINVAL, "%s: arrays have same time", who);
    double mn = ts[0], mx = ts[0];
    for (int i = 1; i < n; ++i) { mn = fmin(mn, ts[i]); mx = fmax(mx, ts[i]); }
    if (t < mn - eps || t > mx + eps) return fail(CGXO_EINVAL, "%s: extrapolation in time", who);
    for (int i = 0; i < n; ++i) {
      double num = 0, den = 0;
      int first = 1;
      for (int j = 0; j < n; ++j) {
        if (j == i) continue;
        if (first) { num = t - ts[j]; den = ts[i] - ts[j]; first = 0; }
        else { num = num * (t - ts[j]); den = den * (ts[i] - ts[j]); }
      }
      w[i] = num / den;
    }
    return CGXO_OK;
  }
  if (kind == 1) {
    double t1 = ts[0], t2 = ts[1], eps = 1.0e-12;
    if (fabs(t1 - t2) < eps) return fail(CGXO_EINVAL, "interpolate_3d_2tl: arrays have same time");
    if (t < fmin(t1, t2) - eps || t > fmax(t1, t2) + eps)
      return fail(CGXO_EINVAL, "interpolate_3d_2tl: extrapolation in time");
    w[0] = (t - t2) / (t1 - t2);
    w[1] = (t - t1) / (t2 - t1);
    return CGXO_OK;
  }
  double t1 = ts[0], t2 = ts[1], t3 = ts[2];
  if (kind == 2) {
    double eps = 1.0e-12;
    if (fabs(t1 - t2) < eps || fabs(t1 - t3) < eps || fabs(t2 - t3) < eps)
      return fail(CGXO_EINVAL, "interpolate_3d_3tl: arrays have same time");
    if (t < fmin(fmin(t1, t2), t3) - eps || t > fmax(fmax(t1, t2), t3) + eps)
      return fail(CGXO_EINVAL, "interpolate_3d_3tl: extrapolation in time");
  } else {
    double tmin = fmin(t1, fmin(t2, t3)), tmax = fmax(t1, fmax(t2, t3));
    double eps = 1.0e-12 * (tmax - tmin);
    if (fabs(t1 - t2) < eps || fabs(t1 - t3) < eps || fabs(t2 - t3) < eps)
      return fail(CGXO_EINVAL, "interpolate_eno_3d_3tl: arrays have same time");
    if (t < tmin - eps || t > tmax + eps)
      return fail(CGXO_EINVAL, "interpolate_eno_3d_3tl: extrapolation in time");
    w[3] = (t - t2) / (t1 - t2);
    w[4] = (t - t1) / (t2 - t1);
    w[5] = (t - t3) / (t2 - t3);
    w[6] = (t - t2) / (t3 - t2);
    int use12 = t >= fmin(t1, t2) - eps && t <= fmax(t1, t2) + eps;
    int use23 = t >= fmin(t2, t3) - eps && t <= fmax(t2, t3) + eps;
    if (!use12 && !use23) return fail(CGXO_EINVAL, "interpolate_eno_3d_3tl: no bracketing pair");
    w[7] = use12;
  }
  w[0] = (t - t2) * (t - t3) / ((t1 - t2) * (t1 - t3));
  w[1] = (t - t1) * (t - t3) / ((t2 - t1) * (t2 - t3));
  w[2] = (t - t1) * (t - t2) / ((t3 - t1) * (t3 - t2));
  return CGXO_OK;
}

/* GCC contracts s1*a + s2*b as fma(s1, a, s2*b), and then + s3*c as
 * fma(s3, c, previous) */
static inline double tcomb2(int fma_, double s1, double a, double s2, double b) {
  return fma_ ? fma(s1, a, s2 * b) : s1 * a + s2 * b;
}
static inline double tcomb3(int fma_, double s1, double a, double s2, double b,
                            double s3, double c) {
  return madd(fma_, s3, c, tcomb2(fma_, s1, a, s2, b));
}
/* interpolate_eno_3d_3tl.cc:145-162 */
static inline double teno(int fma_, const double *w, double a, double b, double c) {
  double d = tcomb3(fma_, w[0], a, w[1], b, w[2], c);
  double mx = fmax(a, fmax(b, c)), mn = fmin(a, fmin(b, c));
  if (d > mx || d < mn)
    d = w[7] != 0.0 ? tcomb2(fma_, w[3], a, w[4], b) : tcomb2(fma_, w[5], b, w[6], c);
  return d;
}

static int time_interp(int kind, int fma_, const double *const *srcs,
                       const double *ts, const int *srcpadext, double *dst,
                       double t, const int *dstpadext, const int *srcbbox_,
                       const int *dstbbox_, const int *regbbox_) {
  box_t srcbbox = mkbox(srcbbox_), dstbbox = mkbox(dstbbox_), reg = mkbox(regbbox_);
  int regext[3], srcoff[3], dstoff[3], rc;
  const char *who = kind == 1 ? "interpolate_3d_2tl" : kind == 2 ? "interpolate_3d_3tl"
                                                                 : "interpolate_eno_3d_3tl";
  if (kind == 4) who = "interpolate_3d_4tl";
  if (kind == 5) who = "interpolate_3d_5tl";
  if ((rc = ti_region(&srcbbox, &dstbbox, &reg, regext, srcoff, dstoff, who))) return rc;
  double w[8];
  if ((rc = cgxo_time_weights(kind, ts, t, w))) return rc;
  for (int k = 0; k < regext[2]; ++k)
    for (int j = 0; j < regext[1]; ++j)
      for (int i = 0; i < regext[0]; ++i) {
        size_t si = IDX(srcoff[0] + i, srcoff[1] + j, srcoff[2] + k, srcpadext);
        double r;
        if (kind == 1) r = tcomb2(fma_, w[0], srcs[0][si], w[1], srcs[1][si]);
        else if (kind == 2) r = tcomb3(fma_, w[0], srcs[0][si], w[1], srcs[1][si], w[2], srcs[2][si]);
        else if (kind == 3) r = teno(fma_, w, srcs[0][si], srcs[1][si], srcs[2][si]);
        else {
          /* s1*a + s2*b + s3*c + s4*d (+ s5*e), left to right */
          r = tcomb3(fma_, w[0], srcs[0][si], w[1], srcs[1][si], w[2], srcs[2][si]);
          for (int m = 3; m < kind; ++m) r = madd(fma_, w[m], srcs[m][si], r);
        }
        dst[IDX(dstoff[0] + i, dstoff[1] + j, dstoff[2] + k, dstpadext)] = r;
      }
  return CGXO_OK;
}

/* interpolate_3d_2tl, CarpetLib/src/interpolate_3d_2tl.cc:24-117 */
int cgxo_interpolate_3d_2tl(int fma_, const double *src1, double t1,
                            const double *src2, double t2, const int *srcpadext,
                            const int *srcext, double *dst, double t,
                            const int *dstpadext, const int *dstext,
                            const int *srcbbox, const int *dstbbox,
                            const int *srcregbbox, const int *regbbox) {
  (void)srcext; (void)dstext; (void)srcregbbox;
  const double *s[2] = {src1, src2};
  double ts[2] = {t1, t2};
  return time_interp(1, fma_, s, ts, srcpadext, dst, t, dstpadext, srcbbox, dstbbox, regbbox);
}
/* interpolate_3d_3tl, CarpetLib/src/interpolate_3d_3tl.cc:24-126 */
int cgxo_interpolate_3d_3tl(int fma_, const double *src1, double t1,
                            const double *src2, double t2, const double *src3,
                            double t3, const int *srcpadext, const int *srcext,
                            double *dst, double t, const int *dstpadext,
                            const int *dstext, const int *srcbbox,
                            const int *dstbbox, const int *srcregbbox,
                            const int *regbbox) {
  (void)srcext; (void)dstext; (void)srcregbbox;
  const double *s[3] = {src1, src2, src3};
  double ts[3] = {t1, t2, t3};
  return time_interp(2, fma_, s, ts, srcpadext, dst, t, dstpadext, srcbbox, dstbbox, regbbox);
}
/* interpolate_3d_4tl, CarpetLib/src/interpolate_3d_4tl.cc:24-134 */
int cgxo_interpolate_3d_4tl(int fma_, const double *src1, double t1,
                            const double *src2, double t2, const double *src3,
                            double t3, const double *src4, double t4,
                            const int *srcpadext, const int *srcext, double *dst,
                            double t, const int *dstpadext, const int *dstext,
                            const int *srcbbox, const int *dstbbox,
                            const int *srcregbbox, const int *regbbox) {
  (void)srcext; (void)dstext; (void)srcregbbox;
  const double *s[4] = {src1, src2, src3, src4};
  double ts[4] = {t1, t2, t3, t4};
  return time_interp(4, fma_, s, ts, srcpadext, dst, t, dstpadext, srcbbox, dstbbox, regbbox);
}
/* interpolate_3d_5tl, CarpetLib/src/interpolate_3d_5tl.cc:24-139 */
int cgxo_interpolate_3d_5tl(int fma_, const double *src1, double t1,
                            const double *src2, double t2, const double *src3,
                            double t3, const double *src4, double t4,
                            const double *src5, double t5, const int *srcpadext,
                            const int *srcext, double *dst, double t,
                            const int *dstpadext, const int *dstext,
                            const int *srcbbox, const int *dstbbox,
                            const int *srcregbbox, const int *regbbox) {
  (void)srcext; (void)dstext; (void)srcregbbox;
  const double *s[5] = {src1, src2, src3, src4, src5};
  double ts[5] = {t1, t2, t3, t4, t5};
  return time_interp(5, fma_, s, ts, srcpadext, dst, t, dstpadext, srcbbox, dstbbox, regbbox);
}
/* interpolate_eno_3d_3tl, CarpetLib/src/interpolate_eno_3d_3tl.cc:32-165 */
int cgxo_interpolate_eno_3d_3tl(int fma_, const double *src1, double t1,
                                const double *src2, double t2,
                                const double *src3, double t3,
                                const int *srcpadext, const int *srcext,
                                double *dst, double t, const int *dstpadext,
                                const int *dstext, const int *srcbbox,
                                const int *dstbbox, const int *srcregbbox,
                                const int *regbbox) {
  (void)srcext; (void)dstext; (void)srcregbbox;
  const double *s[3] = {src1, src2, src3};
  double ts[3] = {t1, t2, t3};
  return time_interp(3, fma_, s, ts, srcpadext, dst, t, dstpadext, srcbbox, dstbbox, regbbox);
}

/* ------------------------------------------------------------------ */
/* gdata::find_source_timelevel, CarpetLib/src/gdata.cc:288-349         */

int cgxo_find_source_timelevel(const double *times, int ntimes, double time,
                               int order_time, int op, int *timelevel0,
                               int *ntimelevels) {
  if (ntimes <= 0 || order_time < 0)
    return fail(CGXO_EINVAL, "find_source_timelevel: no timelevels");
  const double eps = 1.0e-12;
  double mn = times[0], mx = times[0];
  for (int i = 1; i < ntimes; ++i) {
    if (times[i] < mn) mn = times[i];
    if (times[i] > mx) mx = times[i];
  }
  double some_time = fabs(mn) + fabs(mx) + 1.0;
  if (op != op_copy)
    if (time < mn - eps * some_time || time > mx + eps * some_time)
      return fail(CGXO_EINVAL, "find_source_timelevel: extrapolation in time");
  int tl = -1;
  if (ntimes == 1) tl = 0;
  if (tl == -1 && op == op_copy) tl = 0;
  if (tl == -1)
    for (int i = 0; i < ntimes; ++i)
      if (fabs(times[i] - time) < eps * some_time) { tl = i; break; }
  if (tl >= 0) {
    *timelevel0 = tl;
    *ntimelevels = 1;
  } else {
    *timelevel0 = 0;
    *ntimelevels = order_time + 1;
  }
  if (*timelevel0 + *ntimelevels > ntimes)
    return fail(CGXO_EINVAL, "find_source_timelevel: not enough timelevels");
  return CGXO_OK;
}

/* ------------------------------------------------------------------ */
/* data<T>::transfer_time / transfer_p_r / transfer_prolongate /        */
/* transfer_restrict / time_interpolate, CarpetLib/src/data.cc          */

static int sizes_of(const int *b, int *ext) {
  box_t bb = mkbox(b);
  for (int d = 0; d < 3; ++d) ext[d] = box_size(&bb, d);
  return 0;
}

/* transfer_p_r, data.cc:537-556, with the dispatch tables of
 * transfer_prolongate (data.cc:582-725) and transfer_restrict
 * (data.cc:1030-1135) for the restated operators */
static int transfer_p_r(int fma_, int op, int cent, double *dst,
                        const int *dstpadext, const int *dstbbox,
                        const double *src, const int *srcpadext,
                        const int *srcbbox, const int *dstbox,
                        const int *srcbox, const int *slab_offset,
                        int order_space) {
  int srcext[3], dstext[3];
  sizes_of(srcbbox, srcext);
  sizes_of(dstbbox, dstext);
  int eq = 1, gt = 1, lt = 1;
  for (int d = 0; d < 3; ++d) {
    eq &= srcbbox[6 + d] == dstbbox[6 + d];
    gt &= srcbbox[6 + d] > dstbbox[6 + d];
    lt &= srcbbox[6 + d] < dstbbox[6 + d];
  }
  if (eq) /* copy_from_innerloop, data.cc:433-462 */
    return cgxo_copy_3d(src, srcpadext, srcext, dst, dstpadext, dstext,
                        srcbbox, dstbbox, srcbox, dstbox, slab_offset);
  if (gt) {
    if (op == op_sync || op == op_restrict)
      return fail(CGXO_EINVAL, "transfer_p_r: prolongation with a sync/restrict operator");
    if (slab_offset) return fail(CGXO_EINVAL, "transfer_p_r: slab with prolongation");
    if (op == op_copy || op == op_Lagrange) {
      if (cent == vertex_centered)
        return cgxo_prolongate_3d_rf2(order_space, fma_, src, srcpadext, srcext, dst,
                                      dstpadext, dstext, srcbbox, dstbbox, srcbox, dstbox);
      if (cent == cell_centered)
        return cgxo_prolongate_3d_cc_rf2(order_space, fma_, src, srcpadext, srcext, dst,
                                         dstpadext, dstext, srcbbox, dstbbox, srcbox, dstbox);
      return fail(CGXO_EINVAL, "transfer_prolongate: bad centering");
    }
    if (op == op_ENO && cent == vertex_centered) {
      if (order_space == 3 || order_space == 5) /* data.cc:660-686 */
        return cgxo_prolongate_3d_eno(fma_, src, srcpadext, srcext, dst, dstpadext,
                                      dstext, srcbbox, dstbbox, srcbox, dstbox);
      return fail(CGXO_EINVAL, "transfer_prolongate: no ENO stencil for this order");
    }
    if (op == op_Lagrange_monotone) {
      /* data.cc:807-833: order 5 only, for every centring */
      if (order_space == 1 || order_space == 3)
        return fail(CGXO_EINVAL, "There is no stencil for op=\"Lagrange_monotone\" with order_space=%d",
                    order_space);
      if (order_space != 5)
        return fail(CGXO_EINVAL, "There is no stencil for op=\"Lagrange_monotone\" with order_space!=5");
      return cgxo_prolongate_3d_o5_monotone_rf2(fma_, src, srcpadext, srcext, dst, dstpadext,
                                                dstext, srcbbox, dstbbox, srcbox, dstbox);
    }
    if (op == op_WENO) {
      /* data.cc:722-752: vertex-centred order 5 runs the ENO operator */
      if (cent == cell_centered)
        return fail(CGXO_EINVAL, "There are currently no cell-centred stencils for op=\"WENO\"");
      if (cent != vertex_centered) return fail(CGXO_EINVAL, "transfer_prolongate: bad centering");
      if (order_space == 1 || order_space == 3)
        return fail(CGXO_EINVAL, "There is no stencil for op=\"WENO\" with order_space=%d", order_space);
      if (order_space != 5)
        return fail(CGXO_EINVAL, "There is no stencil for op=\"WENO\" with order_space!=5");
      return cgxo_prolongate_3d_eno(fma_, src, srcpadext, srcext, dst, dstpadext, dstext,
                                    srcbbox, dstbbox, srcbox, dstbox);
    }
    if (op == op_ENO && cent == cell_centered) {
      /* data.cc:689-720: orders 2-4 run the second-order stencil, 5 the third */
      if (order_space < 2 || order_space > 5)
        return fail(CGXO_EINVAL, "There is no cell-centred stencil for op=\"ENO\" with "
                                 "order_space not in {2,3,4,5}");
      return cgxo_prolongate_3d_cc_eno_rf2(order_space == 5 ? 3 : 2, fma_, src, srcpadext,
                                           srcext, dst, dstpadext, dstext, srcbbox, dstbbox,
                                           srcbox, dstbox);
    }
    return fail(CGXO_EUNSUPPORTED, "transfer_prolongate: operator outside the restated set");
  }
  if (lt) {
    if (op == op_sync) return fail(CGXO_EINVAL, "transfer_p_r: restriction with a sync operator");
    if (op == op_copy || op == op_Lagrange || op == op_ENO || op == op_WENO ||
        op == op_TVD || op == op_Lagrange_monotone || op == op_restrict) {
      if (cent == vertex_centered) {
        if (slab_offset) return fail(CGXO_EINVAL, "transfer_restrict: slab with restriction");
        return cgxo_restrict_3d_rf2(src, srcpadext, srcext, dst, dstpadext, dstext,
                                    srcbbox, dstbbox, srcbox, dstbox);
      }
      if (cent == cell_centered) {
        /* data.cc:1061-1097: the parameters pick the stencil, except for
         * the ENO and WENO transport operators */
        if (g_ho_restrict && op != op_ENO && op != op_WENO) {
          if (g_restrict_order == 3)
            return cgxo_restrict_3d_cc_o3_rf2(fma_, src, srcpadext, srcext, dst, dstpadext,
                                              dstext, srcbbox, dstbbox, srcbox, dstbox);
          if (g_restrict_order == 5)
            return cgxo_restrict_3d_cc_o5_rf2(fma_, src, srcpadext, srcext, dst, dstpadext,
                                              dstext, srcbbox, dstbbox, srcbox, dstbox);
          if (g_restrict_order != 1)
            return fail(CGXO_EINVAL, "There is no restriction stencil with restriction_order_space==%d",
                        g_restrict_order);
        }
        return cgxo_restrict_3d_cc_rf2(fma_, src, srcpadext, srcext, dst, dstpadext,
                                       dstext, srcbbox, dstbbox, srcbox, dstbox);
      }
      return fail(CGXO_EINVAL, "transfer_restrict: bad centering");
    }
    return fail(CGXO_EUNSUPPORTED, "transfer_restrict: operator outside the restated set");
  }
  return fail(CGXO_EINVAL, "transfer_p_r: mixed strides");
}

/* One box-pair of gdata::transfer_data (gdata.cc:124-286) on one process:
 * find_source_timelevel, then data<T>::transfer_time (data.cc:485-534).
 * srcs[ntimes] share srcpadext/srcbbox. */
int cgxo_transfer(int fma_, int op, int cent, double *dst, const int *dstpadext,
                  const int *dstbbox, const double *const *srcs,
                  const int *srcpadext, const int *srcbbox, const double *times,
                  int ntimes, const int *dstbox, const int *srcbox,
                  const int *slab_offset, double time, int order_space,
                  int order_time) {
  int tl0, ntl, rc;
  if (op == op_error || op == op_none)
    return fail(CGXO_EINVAL, "transfer_data: operator is none/error");
  if ((rc = cgxo_find_source_timelevel(times, ntimes, time, order_time, op, &tl0, &ntl)))
    return rc;
  if (ntl == 1)
    return transfer_p_r(fma_, op, cent, dst, dstpadext, dstbbox, srcs[tl0], srcpadext,
                        srcbbox, dstbox, srcbox, slab_offset, order_space);
  /* data.cc:504-520: temporaries with the extent of dstbox, unpadded */
  int ext[3];
  sizes_of(dstbox, ext);
  size_t npts = (size_t)ext[0] * ext[1] * ext[2];
  double *tmp[5] = {0};
  if (ntl > 5) return fail(CGXO_EINVAL, "time_interpolate: order_time > 4");
  if (ntl > 3 && !(op == op_copy || op == op_Lagrange)) /* data.cc:1295-1297 */
    return fail(CGXO_EINVAL, "time_interpolate: no ENO-family interpolation of order_time %d",
                order_time);
  for (int tl = 0; tl < ntl; ++tl) {
    tmp[tl] = (double *)malloc(npts * sizeof(double) + 8);
    if (!tmp[tl]) { rc = fail(CGXO_ENOMEM, "out of memory"); goto done; }
    if ((rc = transfer_p_r(fma_, op, cent, tmp[tl], ext, dstbox, srcs[tl], srcpadext,
                           srcbbox, dstbox, srcbox, slab_offset, order_space)))
      goto done;
  }
  {
    /* time_interpolate, data.cc:1183-1299 */
    const double *ts = times;
    int dext[3];
    sizes_of(dstbbox, dext);
    int lagr = op == op_copy || op == op_Lagrange;
    int eno = op == op_ENO || op == op_WENO || op == op_TVD || op == op_Lagrange_monotone;
    if (!lagr && !eno) { rc = fail(CGXO_EINVAL, "time_interpolate: bad operator"); goto done; }
    if (order_time == 1)
      rc = cgxo_interpolate_3d_2tl(fma_, tmp[0], ts[0], tmp[1], ts[1], ext, ext, dst, time,
                                   dstpadext, dext, dstbox, dstbbox, dstbox, dstbox);
    else if (lagr && order_time == 2)
      rc = cgxo_interpolate_3d_3tl(fma_, tmp[0], ts[0], tmp[1], ts[1], tmp[2], ts[2], ext,
                                   ext, dst, time, dstpadext, dext, dstbox, dstbbox, dstbox,
                                   dstbox);
    else if (lagr && order_time == 3)
      rc = cgxo_interpolate_3d_4tl(fma_, tmp[0], ts[0], tmp[1], ts[1], tmp[2], ts[2], tmp[3],
                                   ts[3], ext, ext, dst, time, dstpadext, dext, dstbox,
                                   dstbbox, dstbox, dstbox);
    else if (lagr)
      rc = cgxo_interpolate_3d_5tl(fma_, tmp[0], ts[0], tmp[1], ts[1], tmp[2], ts[2], tmp[3],
                                   ts[3], tmp[4], ts[4], ext, ext, dst, time, dstpadext, dext,
                                   dstbox, dstbbox, dstbox, dstbox);
    else
      rc = cgxo_interpolate_eno_3d_3tl(fma_, tmp[0], ts[0], tmp[1], ts[1], tmp[2], ts[2],
                                       ext, ext, dst, time, dstpadext, dext, dstbox,
                                       dstbbox, dstbox, dstbox);
  }
done:
  for (int tl = 0; tl < 5; ++tl) free(tmp[tl]);
  return rc;
}
