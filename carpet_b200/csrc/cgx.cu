// cgx.cu -- kernels and host side of the C-ABI in include/cgx.h.
//
// Host side: restates the argument handling of CarpetLib's transfer path --
// gdata::transfer_data / find_source_timelevel (CarpetLib/src/gdata.cc:124-349)
// and data<T>::transfer_time / transfer_p_r / transfer_prolongate /
// transfer_restrict / time_interpolate (CarpetLib/src/data.cc:485-1299) --
// and turns one box-pair into one device descriptor (cgx::Desc).  The
// reference aborts on bad arguments; here every check returns a status.
//
// Device side: cgx_device.cuh (tile routines) and cgx_kernels.cuh
// (kernels), launched through cgx_kern_*.cu.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/cgx.h"
#include "cgx_device.cuh"
#include "cgx_internal.h"

using namespace cgx;

// ============================================================== host side
namespace {

thread_local std::string g_err;
int g_fp_mode = CGX_FP_EXACT;
// use_higher_order_restriction / restriction_order_space (CarpetLib/param.ccl)
int g_ho_restrict = 0, g_restrict_order = 1;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}
int cuda_fail(cudaError_t e, const char *what) {
  return fail(CGX_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

struct Box {
  int lo[3], up[3], str[3];
  explicit Box(const int *b) {
    for (int d = 0; d < 3; ++d) { lo[d] = b[d]; up[d] = b[3 + d]; str[d] = b[6 + d]; }
  }
  Box() = default;
  bool empty() const {
    for (int d = 0; d < 3; ++d) if (lo[d] > up[d]) return true;
    return false;
  }
  int size(int d) const { return empty() ? 0 : (up[d] - lo[d] + str[d]) / str[d]; }
  long long npoints() const { return (long long)size(0) * size(1) * size(2); }
  // bbox::is_contained_in (bbox.cc:103-109): no alignment check
  bool in(const Box &b) const {
    if (empty()) return true;
    for (int d = 0; d < 3; ++d) if (lo[d] < b.lo[d] || up[d] > b.up[d]) return false;
    return true;
  }
  bool stride_eq(const Box &b) const {
    for (int d = 0; d < 3; ++d) if (str[d] != b.str[d]) return false;
    return true;
  }
};

// The magic number and shift of div_magic (cgx_device.cuh) for divisor n:
// l = ceil(log2 n), m = ceil(2^(31+l) / n), s = l - 1; m = 0 encodes n = 1.
void division_magic(int n, unsigned *m, int *s) {
  if (n <= 1) {
    *m = 0;
    *s = 0;
    return;
  }
  int l = 0;
  while ((1LL << l) < n) ++l;
  const unsigned long long num = 1ULL << (31 + l); // l <= 31
  *m = (unsigned)((num + (unsigned)n - 1) / (unsigned)n);
  *s = l - 1;
}

struct Win { int lo0, hi0, lo1, hi1; };
Win family_window(int kind, int order) {
  if (kind == K_PROLONG_VC) { int lo = -((order + 1) / 2) + 1; return {0, 0, lo, lo + order}; }
  if (kind == K_PROLONG_CC) {
    int n = order + 1, lo0 = -n / 2, lo1 = -n / 2 + (order % 2 ? 1 : 0);
    return {lo0, lo0 + n - 1, lo1, lo1 + n - 1};
  }
  if (kind == K_PROLONG_CC_ENO) return {-order, order - 1, -order + 1, order};
  return {0, 0, -1, 2}; // ENO
}

// Prolongation tiles: ptx fine x (<= PTXMAX) by 2*ptyc-1 fine y (ptyc <=
// pycmax coarse rows) by pz fine z, the widths balanced over the region.
long long prolong_tiles(Desc &d, int pycmax, int pz) {
  const int kind = d.kind;
  long long tot = 1;
  {
    const int ntx = (d.n[0] + PTXMAX - 1) / PTXMAX;
    const int ptx = (d.n[0] + ntx - 1) / ntx;
    int ptyc = std::min(pycmax, NTHREADS / ptx);
    const int nty = (d.n[1] + 2 * ptyc - 2) / (2 * ptyc - 1);
    const int pty = (d.n[1] + nty - 1) / nty;
    ptyc = std::min(ptyc, (pty + 2) / 2);
    d.ptx = (unsigned char)ptx;
    d.ptyc = (unsigned char)ptyc;
    // the tensor-copy box of a tile's coarse plane: all coarse bases of ptx
    // fine points, the stencil window, and one point of even-alignment shift
    const Win w = family_window(kind, d.order);
    const int W = std::max(w.hi0, w.hi1) - std::min(w.lo0, w.lo1);
    d.bx = (unsigned char)(((ptx + 2) / 2 + W + 2) & ~1);
    d.by = (unsigned char)(ptyc + W);
    d.tiles[0] = (d.n[0] + ptx - 1) / ptx;
    d.tiles[1] = (d.n[1] + 2 * ptyc - 2) / (2 * ptyc - 1);
    d.tiles[2] = (d.n[2] + pz - 1) / pz;
    for (int k = 0; k < 3; ++k) tot *= d.tiles[k];
  }
  return tot;
}

// Prolongation tiles of the TMA kernels in tile configuration `config`: as
// prolong_tiles, with as many coarse rows per tile as the configuration's
// threads (one owner per fine x and coarse row), staged box, x-pass rows and
// x items allow for the tile's width (the limits of cgx_tma.cuh): in a
// 128-thread configuration a tile of 16 fine x takes 8 rows, one of 12 takes
// 10 and one of 6 takes 11 (the x-pass rows' limit).
long long prolong_tiles_tma(Desc &d, int config) {
  const TmaCfg &c = TMA_CFGS[config];
  const Win w = family_window(d.kind, d.order);
  const int W = std::max(w.hi0, w.hi1) - std::min(w.lo0, w.lo1);
  const int ntx = (d.n[0] + PTXMAX - 1) / PTXMAX;
  const int ptx = (d.n[0] + ntx - 1) / ntx;
  const int bx = ((ptx + 2) / 2 + W + 2) & ~1;
  const int xr = TMA_XR, nbx = ptx / 2 + 1, ntl = std::max(1, (int)d.ntl);
  int rmax = c.nt / ptx;
  rmax = std::min(rmax, tma_tls(W, c.pyc) / bx - W);
  rmax = std::min(rmax, (tma_xbuf(W, c.pyc, ntl) / xr - 1) / ntl - W);
  rmax = std::min(rmax, tma_items(W, c.pyc) / nbx - W);
  if (rmax < 1) return -1;
  const int nty = (d.n[1] + 2 * rmax - 2) / (2 * rmax - 1);
  const int pty = (d.n[1] + nty - 1) / nty;
  const int ptyc = std::min(rmax, (pty + 2) / 2);
  d.ptx = (unsigned char)ptx;
  d.ptyc = (unsigned char)ptyc;
  d.bx = (unsigned char)bx;
  d.by = (unsigned char)(ptyc + W);
  d.tiles[0] = (d.n[0] + ptx - 1) / ptx;
  d.tiles[1] = (d.n[1] + 2 * ptyc - 2) / (2 * ptyc - 1);
  d.tiles[2] = (d.n[2] + c.pz - 1) / c.pz;
  long long tot = 1;
  for (int k = 0; k < 3; ++k) tot *= d.tiles[k];
  return tot;
}

// Tiles of a descriptor.  Prolongation: the default configuration of
// prolong_tiles (PTYCMAX rows, PTZ fine z).  Copy and restriction: STILE
// consecutive points of the flattened region.
int kind_tiles(Desc &d) {
  const int kind = d.kind;
  const bool prol = is_stencil(kind);
  long long tot = 1;
  if (prol) {
    tot = prolong_tiles(d, PTYCMAX, PTZ);
  } else {
    const long long npts = (long long)d.n[0] * d.n[1] * d.n[2];
    if (npts >= (1LL << 31)) return -1;
    d.tiles[0] = (int)((npts + STILE - 1) / STILE);
    d.tiles[1] = d.tiles[2] = 1;
    tot = d.tiles[0];
    division_magic(d.n[0], &d.mg[0], &d.sh[0]);
    division_magic(d.n[1], &d.mg[1], &d.sh[1]);
  }
  return tot > 0x7fffffff ? -1 : (int)tot;
}

// gdata::find_source_timelevel, CarpetLib/src/gdata.cc:288-349
int find_tl(const double *times, int ntimes, double time, int order_time, int op, int *tl0,
            int *ntl) {
  if (ntimes <= 0 || order_time < 0 || !times)
    return fail(CGX_EINVAL, "find_source_timelevel: no timelevels");
  const double eps = 1.0e-12;
  double mn = times[0], mx = times[0];
  for (int i = 1; i < ntimes; ++i) { mn = std::min(mn, times[i]); mx = std::max(mx, times[i]); }
  const double some_time = std::fabs(mn) + std::fabs(mx) + 1.0;
  if (op != CGX_OP_COPY && (time < mn - eps * some_time || time > mx + eps * some_time))
    return fail(CGX_EINVAL, "find_source_timelevel: extrapolation in time (time=%.17g)", time);
  int tl = -1;
  if (ntimes == 1) tl = 0;
  if (tl == -1 && op == CGX_OP_COPY) tl = 0;
  if (tl == -1)
    for (int i = 0; i < ntimes; ++i)
      if (std::fabs(times[i] - time) < eps * some_time) { tl = i; break; }
  if (tl >= 0) { *tl0 = tl; *ntl = 1; }
  else { *tl0 = 0; *ntl = order_time + 1; }
  if (*tl0 + *ntl > ntimes)
    return fail(CGX_EINVAL, "find_source_timelevel: %d timelevels needed, %d given", *tl0 + *ntl,
                ntimes);
  return CGX_OK;
}

// interpolate_3d_4tl.cc:95-117, interpolate_3d_5tl.cc:100-123: Lagrange
// weights of n = 4 or 5 timelevels, numerator and denominator products
// formed left to right.
int lag_weights(int n, const double *ts, double t, double *w) {
  const double eps = 1.0e-12;
  const char *who = n == 4 ? "interpolate_3d_4tl" : "interpolate_3d_5tl";
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j)
      if (std::fabs(ts[i] - ts[j]) < eps) return fail(CGX_EINVAL, "%s: arrays have same time", who);
  double mn = ts[0], mx = ts[0];
  for (int i = 1; i < n; ++i) { mn = std::fmin(mn, ts[i]); mx = std::fmax(mx, ts[i]); }
  if (t < mn - eps || t > mx + eps) return fail(CGX_EINVAL, "%s: extrapolation in time", who);
  for (int i = 0; i < n; ++i) {
    double num = 0.0, den = 0.0;
    bool first = true;
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      if (first) { num = t - ts[j]; den = ts[i] - ts[j]; first = false; }
      else { num = num * (t - ts[j]); den = den * (ts[i] - ts[j]); }
    }
    w[i] = num / den;
  }
  return CGX_OK;
}

// Time weights exactly as the reference computes them (once per call):
// interpolate_3d_2tl.cc:232-242, interpolate_3d_3tl.cc:365-382,
// interpolate_eno_3d_3tl.cc:105-135.
int time_weights(int tk, const double *ts, double t, double *w) {
  if (tk == T_LIN) {
    const double t1 = ts[0], t2 = ts[1], eps = 1.0e-12;
    if (std::fabs(t1 - t2) < eps) return fail(CGX_EINVAL, "interpolate_3d_2tl: arrays have same time");
    if (t < std::min(t1, t2) - eps || t > std::max(t1, t2) + eps)
      return fail(CGX_EINVAL, "interpolate_3d_2tl: extrapolation in time");
    w[0] = (t - t2) / (t1 - t2);
    w[1] = (t - t1) / (t2 - t1);
    return CGX_OK;
  }
  const double t1 = ts[0], t2 = ts[1], t3 = ts[2];
  if (tk == T_QUAD) {
    const double eps = 1.0e-12;
    if (std::fabs(t1 - t2) < eps || std::fabs(t1 - t3) < eps || std::fabs(t2 - t3) < eps)
      return fail(CGX_EINVAL, "interpolate_3d_3tl: arrays have same time");
    if (t < std::fmin(std::fmin(t1, t2), t3) - eps || t > std::fmax(std::fmax(t1, t2), t3) + eps)
      return fail(CGX_EINVAL, "interpolate_3d_3tl: extrapolation in time");
  } else {
    const double tmin = std::min(t1, std::min(t2, t3)), tmax = std::max(t1, std::max(t2, t3));
    const double eps = 1.0e-12 * (tmax - tmin);
    if (std::fabs(t1 - t2) < eps || std::fabs(t1 - t3) < eps || std::fabs(t2 - t3) < eps)
      return fail(CGX_EINVAL, "interpolate_eno_3d_3tl: arrays have same time");
    if (t < tmin - eps || t > tmax + eps)
      return fail(CGX_EINVAL, "interpolate_eno_3d_3tl: extrapolation in time");
    w[3] = (t - t2) / (t1 - t2);
    w[4] = (t - t1) / (t2 - t1);
    w[5] = (t - t3) / (t2 - t3);
    w[6] = (t - t2) / (t3 - t2);
    const bool use12 = t >= std::min(t1, t2) - eps && t <= std::max(t1, t2) + eps;
    const bool use23 = t >= std::min(t2, t3) - eps && t <= std::max(t2, t3) + eps;
    if (!use12 && !use23) return fail(CGX_EINVAL, "interpolate_eno_3d_3tl: no bracketing pair");
    w[7] = use12 ? 1.0 : 0.0;
  }
  w[0] = (t - t2) * (t - t3) / ((t1 - t2) * (t1 - t3));
  w[1] = (t - t1) * (t - t3) / ((t2 - t1) * (t2 - t3));
  w[2] = (t - t1) * (t - t2) / ((t3 - t1) * (t3 - t2));
  return CGX_OK;
}

// Coarse window [lo, hi] of one parity relative to the coarse base c.
// Every coarse point any fine point of the region reads: the first two and
// last two fine points of each axis bound it.  Used for the exact in-bounds
// check (stricter than the reference's expand() test, which works in fine
// strides) and for the algorithmic byte count.
void stencil_range(const Win &w, int soff, int n, int *cmin, int *cmax) {
  int mn = 1 << 30, mx = -(1 << 30);
  for (int i = 0; i < n; i = (i == 1 && n > 3) ? n - 2 : i + 1) {
    int s = soff + i, c = s >> 1, p = s & 1;
    mn = std::min(mn, c + (p ? w.lo1 : w.lo0));
    mx = std::max(mx, c + (p ? w.hi1 : w.hi0));
  }
  *cmin = mn;
  *cmax = mx;
}

// One box-pair.  With nst > 0 the pair runs transfer_time in its two
// stages (data.cc:506-517): st[t] writes timelevel t's spatial result into
// a temporary of the region's shape, and d (K_TIME) combines the nst
// temporaries into the destination.  The temporaries are bound by bind_tmp.
struct Built {
  Desc d;
  long long bytes;  // algorithmic bytes (reads + writes)
  long long points; // destination points written
  int ntiles;
  int nst;            // timelevels staged through temporaries, or 0
  Desc st[5];
  int st_ntiles;
  long long tmp_elems; // doubles of temporaries
};

void bind_tmp(Built &b, double *tmp) {
  const long long npts = b.tmp_elems / b.nst;
  for (int t = 0; t < b.nst; ++t) b.st[t].dst = tmp + t * npts;
  for (int t = 0; t < 3; ++t) b.d.src[t] = tmp;
}

bool pad_ok(const cgx_array *a) {
  Box b(a->bbox);
  for (int d = 0; d < 3; ++d) {
    if (b.str[d] <= 0) return false;
    if (a->padext[d] < b.size(d)) return false;
  }
  return a->data != nullptr;
}

// The spatial operator of one timelevel: transfer_p_r (data.cc:537-556).
// regdst: the destination bbox the operator sees (dst extent, or dstbox
// itself for the temporaries of data.cc:506-509).
int build_spatial(int op, int cent, const cgx_array *dst, const cgx_array *src,
                  const Box &regdst, const Box &dstbox, const Box &srcbox, const int *slab,
                  int order_space, Built *out) {
  Desc &d = out->d;
  Box sb(src->bbox), db(dst->bbox);
  bool eq = true, gt = true, lt = true;
  for (int k = 0; k < 3; ++k) {
    eq &= sb.str[k] == regdst.str[k];
    gt &= sb.str[k] > regdst.str[k];
    lt &= sb.str[k] < regdst.str[k];
  }
  for (int k = 0; k < 3; ++k) d.sext[k] = sb.size(k);
  d.ssy = src->padext[0];
  d.ssz = (long long)src->padext[0] * src->padext[1];
  if (eq) {
    // copy_from_innerloop -> copy_3d (copy_3d.cc:36-82)
    const Box &reg = dstbox;
    if (!sb.stride_eq(reg) || !regdst.stride_eq(reg) || !srcbox.stride_eq(reg))
      return fail(CGX_EINVAL, "copy_3d: strides disagree");
    if (reg.empty()) return fail(CGX_EINVAL, "copy_3d: region extent is empty");
    Box sreg = reg;
    if (slab)
      for (int k = 0; k < 3; ++k) { sreg.lo[k] += slab[k] * reg.str[k]; sreg.up[k] += slab[k] * reg.str[k]; }
    if (!sreg.in(srcbox)) return fail(CGX_EINVAL, "copy_3d: shifted source region outside srcbox");
    if (!sreg.in(sb) || !reg.in(regdst))
      return fail(CGX_EINVAL, "copy_3d: region extent is not contained in array extent");
    for (int k = 0; k < 3; ++k) {
      if ((sreg.lo[k] - sb.lo[k]) % sb.str[k] || (reg.lo[k] - regdst.lo[k]) % regdst.str[k])
        return fail(CGX_EINVAL, "copy_3d: region not aligned with the arrays");
      d.n[k] = reg.size(k);
      d.soff[k] = (sreg.lo[k] - sb.lo[k]) / sb.str[k];
    }
    d.kind = K_COPY;
    d.order = 0;
    out->points = reg.npoints();
    out->bytes = 16 * out->points;
    return CGX_OK;
  }
  if (gt) {
    if (op == CGX_OP_SYNC || op == CGX_OP_RESTRICT)
      return fail(CGX_EINVAL, "transfer_p_r: prolongation with a sync/restrict operator");
    if (slab) return fail(CGX_EINVAL, "transfer_p_r: slab with prolongation");
    const Box &reg = dstbox;
    int kind;
    if (op == CGX_OP_LAGRANGE_MONOTONE) {
      // data.cc:807-833, prolongate_3d_o5_monotone_rf2.cc:72-104 (any centring)
      if (order_space == 1 || order_space == 3)
        return fail(CGX_EINVAL, "There is no stencil for op=\"Lagrange_monotone\" with order_space=%d",
                    order_space);
      if (order_space != 5)
        return fail(CGX_EINVAL, "There is no stencil for op=\"Lagrange_monotone\" with order_space!=5");
      for (int k = 0; k < 3; ++k) {
        if (sb.str[k] <= reg.str[k] || regdst.str[k] != reg.str[k])
          return fail(CGX_EINVAL, "prolongate_3d_o5_monotone_rf2: strides disagree");
        if (sb.str[k] != 2 * regdst.str[k])
          return fail(CGX_EINVAL, "prolongate_3d_o5_monotone_rf2: source strides are not twice the "
                                  "destination strides");
      }
      if (reg.empty()) return fail(CGX_EINVAL, "prolongate_3d_o5_monotone_rf2: region extent is empty");
      Box ex = reg;
      long long ncoarse = 1;
      for (int k = 0; k < 3; ++k) {
        if ((reg.lo[k] - sb.lo[k]) % reg.str[k] || (reg.lo[k] - regdst.lo[k]) % reg.str[k])
          return fail(CGX_EINVAL, "prolongate_3d_o5_monotone_rf2: region not aligned");
        d.n[k] = reg.size(k);
        d.soff[k] = (reg.lo[k] - sb.lo[k]) / reg.str[k];
        const int s0 = d.soff[k], s1 = s0 + d.n[k] - 1;
        ex.lo[k] -= (s0 % 2 != 0 || d.n[k] > 1 ? 3 : 0) * reg.str[k];
        ex.up[k] += (s1 % 2 != 0 || d.n[k] > 1 ? 3 : 0) * reg.str[k];
        // coarse points read: s/2 for an even fine point s, s/2-2 .. s/2+3 for an odd one
        const int cmin = d.n[k] > 1 || s0 % 2 ? s0 / 2 - 2 : s0 / 2;
        const int cmax = d.n[k] > 1 || s1 % 2 ? (s1 - 1) / 2 + 3 : s1 / 2;
        if (s0 < 0 || cmin < 0 || cmax >= sb.size(k))
          return fail(CGX_EINVAL, "prolongate_3d_o5_monotone_rf2: stencil reaches outside the source array");
        ncoarse *= cmax - cmin + 1;
      }
      if (!ex.in(sb) || !reg.in(regdst))
        return fail(CGX_EINVAL, "prolongate_3d_o5_monotone_rf2: region extent is not contained in array extent");
      d.kind = K_PROLONG_MONO;
      d.order = 5;
      out->points = reg.npoints();
      out->bytes = 8 * out->points + 8 * ncoarse;
      return CGX_OK;
    }
    if (op == CGX_OP_COPY || op == CGX_OP_LAGRANGE) {
      if (cent == CGX_VERTEX) {
        if (order_space != 1 && order_space != 3 && order_space != 5 && order_space != 7 &&
            order_space != 9 && order_space != 11)
          return fail(CGX_EINVAL, "transfer_prolongate: no vertex-centred stencil of order %d",
                      order_space);
        kind = K_PROLONG_VC;
      } else if (cent == CGX_CELL) {
        if (order_space < 0 || order_space > 5)
          return fail(CGX_EINVAL, "transfer_prolongate: no cell-centred stencil of order %d",
                      order_space);
        kind = K_PROLONG_CC;
      } else return fail(CGX_EINVAL, "transfer_prolongate: bad centering");
    } else if (op == CGX_OP_ENO && cent == CGX_CELL) {
      // data.cc:689-720: orders 2-4 run the second-order stencil, 5 the third
      if (order_space < 2 || order_space > 5)
        return fail(CGX_EINVAL, "There is no cell-centred stencil for op=\"ENO\" with "
                                "order_space not in {2,3,4,5}");
      kind = K_PROLONG_CC_ENO;
      order_space = order_space == 5 ? 3 : 2;
    } else if (op == CGX_OP_WENO) {
      // data.cc:722-752: vertex-centred order 5 runs the ENO operator
      if (cent == CGX_CELL)
        return fail(CGX_EINVAL, "There are currently no cell-centred stencils for op=\"WENO\"");
      if (cent != CGX_VERTEX) return fail(CGX_EINVAL, "transfer_prolongate: bad centering");
      if (order_space == 1 || order_space == 3)
        return fail(CGX_EINVAL, "There is no stencil for op=\"WENO\" with order_space=%d", order_space);
      if (order_space != 5)
        return fail(CGX_EINVAL, "There is no stencil for op=\"WENO\" with order_space!=5");
      kind = K_PROLONG_ENO;
    } else if (op == CGX_OP_ENO) {
      if (cent != CGX_VERTEX) return fail(CGX_EINVAL, "transfer_prolongate: bad centering");
      if (order_space != 3 && order_space != 5) // data.cc:660-686
        return fail(CGX_EINVAL, "transfer_prolongate: no ENO stencil of order %d", order_space);
      kind = K_PROLONG_ENO;
    } else return fail(CGX_EUNSUPPORTED, "transfer_prolongate: operator %d is not provided", op);

    // argument checks of prolongate_3d_rf2.cc:373-417,
    // prolongate_3d_cc_rf2.cc:253-321, prolongate_3d_real8_eno.F90:122-175,
    // prolongate_3d_cc_eno_rf2.cc:962-1031
    const bool cellk = kind == K_PROLONG_CC || kind == K_PROLONG_CC_ENO;
    for (int k = 0; k < 3; ++k) {
      if (sb.str[k] <= reg.str[k] || regdst.str[k] != reg.str[k])
        return fail(CGX_EINVAL, "prolongate: strides disagree");
      if (sb.str[k] != 2 * regdst.str[k])
        return fail(CGX_EINVAL, "prolongate: source strides are not twice the destination strides");
      if (!cellk &&
          (sb.lo[k] % sb.str[k] || regdst.lo[k] % regdst.str[k] || reg.lo[k] % reg.str[k]))
        return fail(CGX_EINVAL, "prolongate: bbox is not aligned with vertices");
      if (cellk && regdst.str[k] % 2)
        return fail(CGX_EINVAL, "prolongate_3d_cc_rf2: destination strides are not even");
    }
    if (reg.empty()) return fail(CGX_EINVAL, "prolongate: region extent is empty");
    if (!reg.in(regdst)) return fail(CGX_EINVAL, "prolongate: region extent is not contained in array extent");
    const Win w = family_window(kind, order_space);
    long long ncoarse = 1;
    for (int k = 0; k < 3; ++k) {
      const int h = cellk ? reg.str[k] / 2 : 0;
      if ((reg.lo[k] - sb.lo[k] + h) % reg.str[k] || (reg.lo[k] - regdst.lo[k]) % reg.str[k])
        return fail(CGX_EINVAL, "prolongate: region not aligned with the arrays");
      d.n[k] = reg.size(k);
      d.soff[k] = (reg.lo[k] - sb.lo[k] + h) / reg.str[k];
      if (d.soff[k] < 0) return fail(CGX_EINVAL, "prolongate: region extent is not contained in array extent");
      int cmin, cmax;
      stencil_range(w, d.soff[k], d.n[k], &cmin, &cmax);
      if (cmin < 0 || cmax >= sb.size(k))
        return fail(CGX_EINVAL, "prolongate: stencil reaches outside the source array "
                                "(axis %d, coarse %d..%d of %d)", k, cmin, cmax, sb.size(k));
      ncoarse *= cmax - cmin + 1;
    }
    // the reference's own containment test (expand in fine strides)
    if (kind == K_PROLONG_VC) {
      Box ex = reg;
      for (int k = 0; k < 3; ++k) {
        int n = reg.size(k);
        bool nlo = d.soff[k] % 2 != 0, nhi = (d.soff[k] + n - 1) % 2 != 0;
        int olo = nlo ? order_space / 2 + 1 : (n > 1 ? order_space / 2 : 0);
        int ohi = nhi ? order_space / 2 + 1 : (n > 1 ? order_space / 2 : 0);
        ex.lo[k] -= olo * reg.str[k];
        ex.up[k] += ohi * reg.str[k];
      }
      if (!ex.in(sb)) return fail(CGX_EINVAL, "prolongate_3d_rf2: region extent is not contained in array extent");
    } else if (kind == K_PROLONG_CC_ENO) {
      // prolongate_3d_cc_eno_rf2.cc:994-1031: the window of the parity at
      // each end, counted in fine strides
      Box ex = reg;
      for (int k = 0; k < 3; ++k) {
        const int send = d.soff[k] + reg.size(k) - 1;
        ex.lo[k] -= (order_space - d.soff[k] % 2) * reg.str[k];
        ex.up[k] += (order_space + send % 2 - 1) * reg.str[k];
      }
      if (!ex.in(sb))
        return fail(CGX_EINVAL, "prolongate_3d_cc_eno_rf2: region extent is not contained in array extent");
    }
    d.kind = kind;
    d.order = order_space;
    out->points = reg.npoints();
    out->bytes = 8 * out->points + 8 * ncoarse; // per timelevel source added by caller
    return CGX_OK;
  }
  if (lt) {
    if (op == CGX_OP_SYNC) return fail(CGX_EINVAL, "transfer_p_r: restriction with a sync operator");
    if (!(op == CGX_OP_COPY || op == CGX_OP_LAGRANGE || op == CGX_OP_ENO || op == CGX_OP_WENO ||
          op == CGX_OP_TVD || op == CGX_OP_LAGRANGE_MONOTONE || op == CGX_OP_RESTRICT))
      return fail(CGX_EUNSUPPORTED, "transfer_restrict: operator %d is not provided", op);
    const Box &reg = dstbox;
    // restrict_3d_rf2.cc:38-68, restrict_3d_cc_rf2.cc:172-207
    for (int k = 0; k < 3; ++k) {
      if (sb.str[k] >= reg.str[k] || regdst.str[k] != reg.str[k])
        return fail(CGX_EINVAL, "restrict: strides disagree");
      if (2 * sb.str[k] != regdst.str[k])
        return fail(CGX_EINVAL, "restrict: destination strides are not twice the source strides");
    }
    if (reg.empty()) return fail(CGX_EINVAL, "restrict: region extent is empty");
    if (cent == CGX_VERTEX) {
      if (slab) return fail(CGX_EINVAL, "transfer_restrict: slab with restriction");
      if (!reg.in(sb) || !reg.in(regdst))
        return fail(CGX_EINVAL, "restrict_3d_rf2: region extent is not contained in array extent");
      for (int k = 0; k < 3; ++k) {
        if ((reg.lo[k] - sb.lo[k]) % sb.str[k] || (reg.lo[k] - regdst.lo[k]) % regdst.str[k])
          return fail(CGX_EINVAL, "restrict_3d_rf2: region not aligned");
        d.n[k] = reg.size(k);
        d.soff[k] = (reg.lo[k] - sb.lo[k]) / sb.str[k];
        if (d.soff[k] + 2 * (d.n[k] - 1) >= sb.size(k))
          return fail(CGX_EINVAL, "restrict_3d_rf2: region extent is not contained in array extent");
      }
      d.kind = K_RESTRICT_VC;
      out->points = reg.npoints();
      out->bytes = 16 * out->points;
    } else if (cent == CGX_CELL) {
      // data.cc:1061-1097: the parameters pick the stencil, except for the
      // ENO and WENO transport operators
      int ho = 0;
      if (g_ho_restrict && op != CGX_OP_ENO && op != CGX_OP_WENO) {
        if (g_restrict_order == 3 || g_restrict_order == 5) ho = g_restrict_order;
        else if (g_restrict_order != 1)
          return fail(CGX_EINVAL, "There is no restriction stencil with restriction_order_space==%d",
                      g_restrict_order);
      }
      if (ho) {
        // restrict_3d_cc_o3_rf2.cc:33-144 / restrict_3d_cc_o5_rf2.cc:79-157:
        // the fine cells 2i+lo .. 2i+hi (per axis) around every coarse point
        // must lie inside the source
        const char *who = ho == 3 ? "restrict_3d_cc_o3_rf2" : "restrict_3d_cc_o5_rf2";
        const int lo = ho == 3 ? -1 : -2, hi = ho == 3 ? 2 : 3;
        if (!reg.in(regdst)) return fail(CGX_EINVAL, "%s: region extent is not contained in array extent", who);
        for (int k = 0; k < 3; ++k) {
          int h = sb.str[k] / 2;
          if (sb.str[k] % 2 || (reg.lo[k] - sb.lo[k] - h) % sb.str[k] ||
              (reg.lo[k] - regdst.lo[k]) % regdst.str[k])
            return fail(CGX_EINVAL, "%s: region not aligned", who);
          d.n[k] = reg.size(k);
          d.soff[k] = (reg.lo[k] - sb.lo[k] - h) / sb.str[k];
          if (d.soff[k] + lo < 0 || d.soff[k] + 2 * (d.n[k] - 1) + hi >= sb.size(k))
            return fail(CGX_EINVAL, "%s: stencil reaches outside the source array", who);
        }
        d.kind = ho == 3 ? K_RESTRICT_CC3 : K_RESTRICT_CC5;
        out->points = reg.npoints();
        // compulsory traffic: the 8 fine cells under each coarse point once
        // (the wider stencils re-read neighbours from cache) and the write
        out->bytes = 72 * out->points;
        d.order = 0;
        return CGX_OK;
      }
      // bbox::expanded_for (bbox.cc:208-219) of the region onto the source
      Box ef = reg;
      for (int k = 0; k < 3; ++k) {
        int s = sb.str[k];
        auto imod = [](int x, int y) { int r = x % y; return r < 0 ? r + y : r; };
        int loff = imod(reg.lo[k] - sb.lo[k], s), uoff = imod(reg.up[k] - sb.lo[k], s);
        ef.lo[k] = reg.lo[k] - loff;
        ef.up[k] = reg.up[k] + (s - uoff) % s;
        ef.str[k] = s;
      }
      if (!ef.in(sb) || !reg.in(regdst))
        return fail(CGX_EINVAL, "restrict_3d_cc_rf2: region extent is not contained in array extent");
      for (int k = 0; k < 3; ++k) {
        int h = sb.str[k] / 2;
        if (sb.str[k] % 2 || (reg.lo[k] - sb.lo[k] - h) % sb.str[k] ||
            (reg.lo[k] - regdst.lo[k]) % regdst.str[k])
          return fail(CGX_EINVAL, "restrict_3d_cc_rf2: region not aligned");
        d.n[k] = reg.size(k);
        d.soff[k] = (reg.lo[k] - sb.lo[k] - h) / sb.str[k];
        if (d.soff[k] < 0 || d.soff[k] + 2 * d.n[k] - 1 >= sb.size(k))
          return fail(CGX_EINVAL, "restrict_3d_cc_rf2: region extent is not contained in array extent");
      }
      d.kind = K_RESTRICT_CC;
      out->points = reg.npoints();
      out->bytes = 72 * out->points;
    } else return fail(CGX_EINVAL, "transfer_restrict: bad centering");
    d.order = 0;
    return CGX_OK;
  }
  return fail(CGX_EINVAL, "transfer_p_r: mixed strides");
}

// One box-pair: gdata::transfer_data on one process + transfer_time.
int build(int op, int cent, const cgx_array *dst, const cgx_array *srcs, const double *times,
          int nsrc, const int *dstbox_, const int *srcbox_, const int *slab, double time,
          int order_space, int order_time, Built *out) {
  if (!dst || !srcs || !dstbox_ || !srcbox_) return fail(CGX_EINVAL, "transfer: null argument");
  if (op == CGX_OP_ERROR || op == CGX_OP_NONE)
    return fail(CGX_EINVAL, "transfer_data: operator is none/error");
  if (nsrc < 1 || nsrc > 16) return fail(CGX_EINVAL, "transfer_data: bad number of sources");
  if (!pad_ok(dst)) return fail(CGX_EINVAL, "transfer: bad destination array");
  for (int t = 0; t < nsrc; ++t) {
    if (!pad_ok(&srcs[t])) return fail(CGX_EINVAL, "transfer: bad source array %d", t);
    for (int k = 0; k < 3; ++k)
      if (srcs[t].padext[k] != srcs[0].padext[k])
        return fail(CGX_EINVAL, "transfer: source timelevels differ in shape");
    for (int k = 0; k < 9; ++k)
      if (srcs[t].bbox[k] != srcs[0].bbox[k])
        return fail(CGX_EINVAL, "transfer: source timelevels differ in extent");
  }
  const Box dstbox(dstbox_), srcbox(srcbox_), db(dst->bbox);
  // gdata.cc:139-147
  if (dstbox.empty()) return fail(CGX_EINVAL, "transfer_data: empty dstbox");
  if (srcbox.empty()) return fail(CGX_EINVAL, "transfer_data: empty srcbox");
  for (int k = 0; k < 3; ++k)
    if (dstbox.lo[k] < db.lo[k] || dstbox.up[k] > db.up[k] || dstbox.str[k] != db.str[k] ||
        (dstbox.lo[k] - db.lo[k]) % dstbox.str[k])
      return fail(CGX_EINVAL, "transfer_data: dstbox is not inside the destination");
  int tl0, ntl, rc;
  if ((rc = find_tl(times, nsrc, time, order_time, op, &tl0, &ntl))) return rc;
  Built b;
  memset(&b, 0, sizeof b);
  Desc &d = b.d;
  // with time interpolation the operator writes a temporary of extent
  // dstbox (data.cc:506-509) and time_interpolate reads it with region
  // dstbox (data.cc:517): the fused kernel writes dst directly
  const Box &regdst = ntl > 1 ? dstbox : db;
  if ((rc = build_spatial(op, cent, dst, &srcs[tl0], regdst, dstbox, srcbox, slab, order_space, &b)))
    return rc;
  int tk = T_NONE;
  if (ntl > 1) {
    const bool lagr = op == CGX_OP_COPY || op == CGX_OP_LAGRANGE;
    const bool eno = op == CGX_OP_ENO || op == CGX_OP_WENO || op == CGX_OP_TVD ||
                     op == CGX_OP_LAGRANGE_MONOTONE;
    if (!lagr && !eno) return fail(CGX_EINVAL, "time_interpolate: bad operator");
    if (order_time == 1) tk = T_LIN;
    else if (order_time == 2) tk = lagr ? T_QUAD : T_ENO;
    else if (order_time <= 4) {
      if (!lagr) // data.cc:1295-1297
        return fail(CGX_EINVAL, "time_interpolate: no ENO-family interpolation of order_time %d",
                    order_time);
      tk = T_LAG;
    } else return fail(CGX_EINVAL, "time_interpolate: order_time %d", order_time);
    rc = tk == T_LAG ? lag_weights(ntl, times + tl0, time, d.w) : time_weights(tk, times + tl0, time, d.w);
    if (rc) return rc;
  }
  d.ntl = ntl;
  d.tkind = tk;
  for (int t = 0; t < 3; ++t) d.src[t] = srcs[tl0 + std::min(t, ntl - 1)].data;
  d.dst = dst->data;
  d.dsy = dst->padext[0];
  d.dsz = (long long)dst->padext[0] * dst->padext[1];
  for (int k = 0; k < 3; ++k) d.doff[k] = (dstbox.lo[k] - db.lo[k]) / db.str[k];
  // algorithmic bytes: destination written once, every timelevel's source
  // read once (copy and restrictions counted per point above)
  const long long src_bytes = b.bytes - 8 * b.points; // one timelevel's reads
  b.bytes = 8 * b.points + (long long)ntl * src_bytes;
  // the fused kernels interpolate up to 3 timelevels after copies and
  // prolongations; restrictions between timelevels and 4 or 5 timelevels
  // run the reference's two stages
  if (ntl > 3 || (ntl > 1 && !(d.kind == K_COPY || is_stencil(d.kind)))) {
    const long long npts = (long long)d.n[0] * d.n[1] * d.n[2];
    for (int t = 0; t < ntl; ++t) {
      Desc &s = b.st[t];
      s = d;
      s.ntl = 1;
      s.tkind = T_NONE;
      for (int q = 0; q < 3; ++q) s.src[q] = srcs[tl0 + t].data;
      s.dst = nullptr;
      s.dsy = d.n[0];
      s.dsz = (long long)d.n[0] * d.n[1];
      for (int k = 0; k < 3; ++k) s.doff[k] = 0;
      b.st_ntiles = kind_tiles(s);
      if (b.st_ntiles <= 0) return fail(CGX_EINVAL, "transfer: region too large");
    }
    d.kind = K_TIME;
    d.order = 0;
    for (int k = 0; k < 3; ++k) d.soff[k] = 0;
    for (int q = 0; q < 3; ++q) d.src[q] = nullptr;
    b.nst = ntl;
    b.tmp_elems = ntl * npts;
  }
  b.ntiles = kind_tiles(d);
  if (b.ntiles <= 0) return fail(CGX_EINVAL, "transfer: region too large");
  *out = b;
  return CGX_OK;
}

int launch_pair(const Desc &d, int ntiles, int fp, int *status, cudaStream_t s);

// The two stages of a staged pair on one stream, with stream-ordered
// temporaries.
int launch_staged(Built &b, int fp, int *status, cudaStream_t s) {
  double *tmp = nullptr;
  cudaError_t e = cudaMallocAsync(&tmp, (size_t)b.tmp_elems * sizeof(double), s);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
  bind_tmp(b, tmp);
  int rc = CGX_OK;
  for (int t = 0; t < b.nst && rc == CGX_OK; ++t) rc = launch_pair(b.st[t], b.st_ntiles, fp, status, s);
  if (rc == CGX_OK) rc = launch_pair(b.d, b.ntiles, fp, status, s);
  e = cudaFreeAsync(tmp, s);
  if (rc == CGX_OK && e != cudaSuccess) rc = cuda_fail(e, "cudaFreeAsync");
  return rc;
}

int launch_pair(const Desc &d, int ntiles, int fp, int *status, cudaStream_t s) {
  const bool high = d.kind == K_PROLONG_VC && d.order >= 7;
  if (high) return klaunch_pair_hi(fp, d, ntiles, status, s);
  if (!is_stencil(d.kind))
    return fp == CGX_FP_FMA ? klaunch_spair_f1(d, ntiles, status, s) : klaunch_spair_f0(d, ntiles, status, s);
  return fp == CGX_FP_FMA ? klaunch_pair_f1(d, ntiles, status, s) : klaunch_pair_f0(d, ntiles, status, s);
}

// One persistent kernel per non-empty segment of a tile map, each with its
// own work counter (counter[i], zero on entry).
// the TMA kernels' launchers, [fused][family part][configuration]
using TmaLaunch = int (*)(int, const Desc *, const CUtensorMap *, const int2 *, long long,
                          unsigned long long *, int *, cudaStream_t);
#define CGX_TMA_ROW(F, P)                                                                      \
  {klaunch_tma_f##F##_p##P##_c0, klaunch_tma_f##F##_p##P##_c1, klaunch_tma_f##F##_p##P##_c2, \
   klaunch_tma_f##F##_p##P##_c3, klaunch_tma_f##F##_p##P##_c4}
const TmaLaunch kTmaLaunch[2][2][TMA_NCFG] = {{CGX_TMA_ROW(0, 0), CGX_TMA_ROW(0, 1)},
                                              {CGX_TMA_ROW(1, 0), CGX_TMA_ROW(1, 1)}};
#undef CGX_TMA_ROW

int launch_map_capped(int fp, const Desc *d, const CUtensorMap *maps, const int2 *tmap,
                      const long long seg[NSEG + 1], const int *cfg, unsigned long long *counter, int *status,
                      cudaStream_t s);
// failure injection for the tests of the bounded device waits
// (cgx_debug_skip_tma_plane)
bool g_debug_skip_tma = false;

// with the batch's CTA caps in force for these launches only
int launch_map(int fp, const Desc *d, const CUtensorMap *maps, const int2 *tmap,
               const long long seg[NSEG + 1], const int *cfg, unsigned long long *counter, int *status,
               cudaStream_t s, const int *caps = nullptr) {
  g_cta_cap[0] = caps ? caps[0] : 0;
  g_cta_cap[1] = caps ? caps[1] : 0;
  const int rc = launch_map_capped(fp, d, maps, tmap, seg, cfg, counter, status, s);
  g_cta_cap[0] = g_cta_cap[1] = 0;
  return rc;
}
int launch_map_capped(int fp, const Desc *d, const CUtensorMap *maps, const int2 *tmap,
                      const long long seg[NSEG + 1], const int *cfg, unsigned long long *counter, int *status,
                      cudaStream_t s) {
  const bool f = fp == CGX_FP_FMA;
  for (int i = 0; i < NSEG; ++i) {
    const long long n = seg[i + 1] - seg[i];
    if (n <= 0) continue;
    const int2 *tm = tmap + seg[i];
    unsigned long long *c = counter + i;
    int rc;
    if (i < TV_COUNT) {
      const int k = cfg ? cfg[i] : 0;
      if (k < 0 || k >= TMA_NCFG) return fail(CGX_EINVAL, "bad tile configuration %d", k);
      rc = kTmaLaunch[f][i / 4 >= 5][k](i | (g_debug_skip_tma ? 1 << 30 : 0), d, maps, tm, n, c, status, s);
    } else if (i == SEG_STENCIL) {
      rc = f ? klaunch_map_f1(d, tm, n, c, status, s) : klaunch_map_f0(d, tm, n, c, status, s);
    } else {
      rc = f ? klaunch_stream_f1(i - SEG_STREAM, d, tm, n, c, status, s)
             : klaunch_stream_f0(i - SEG_STREAM, d, tm, n, c, status, s);
    }
    if (rc) return rc;
  }
  return CGX_OK;
}

// cuTensorMapEncodeTiled from the driver, found once; null without a driver
PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      cudaGetLastError();
  }
  return fn;
}

} // namespace

// ============================================================== batches
struct cgx_batch {
  std::vector<Desc> descs;
  std::vector<long long> bytes, points;
  std::vector<int> ntiles;
  std::vector<unsigned char> high; // vertex-centred orders 7..11: per-box kernels
  Desc *d_descs = nullptr;
  long long *d_prefix = nullptr;
  size_t d_cap = 0;
  int2 *d_tmap = nullptr; // (descriptor, local tile) of every queued tile
  size_t tmap_cap = 0;
  CUtensorMap *d_maps = nullptr; // 3 per queued descriptor (d_cap of them)
  int n_uploaded = 0;     // descriptors in the persistent kernel's queue
  long long tiles_uploaded = 0;
  long long seg[NSEG + 1] = {0}; // the tile map's segments
  int tma_cfg[TV_COUNT] = {0};    // tile configuration of each TMA variant
  std::vector<int> high_idx; // descriptors launched per box
  unsigned long long *d_counter = nullptr; // one per tile-map segment
  int *d_status = nullptr;
  int fp_mode = CGX_FP_EXACT;
  // staged pairs: offsets (doubles) into the batch's temporaries of a
  // descriptor's destination (stage 1) or sources (stage 2), else -1
  std::vector<long long> tdst, tsrc;
  long long tmp_elems = 0;
  int nstage1 = 0;       // stage-1 descriptors (not pairs of their own)
  double *d_tmp = nullptr;
  size_t tmp_cap = 0;    // doubles
  std::vector<Desc> pdescs; // descs with the temporaries bound
  // streams and events of the concurrent segment launch (created at upload,
  // on the device current then)
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> ev; // ev[0] forks, ev[1 + k] joins side[k]
  // CTAs per SM of the TMA and the streaming kernels (0: as many as fit)
  int max_ctas[2] = {0, 0};
  // dependency group of every descriptor (cgx_batch_set_group; the chain)
  int cur_group = 0;
  std::vector<int> group;
};

namespace {
void batch_push(cgx_batch *b, const Desc &d, long long bytes, long long points, int ntiles,
                long long tdst, long long tsrc) {
  b->descs.push_back(d);
  b->bytes.push_back(bytes);
  b->points.push_back(points);
  b->ntiles.push_back(ntiles);
  b->high.push_back(d.kind == K_PROLONG_VC && d.order >= 7);
  b->tdst.push_back(tdst);
  b->tsrc.push_back(tsrc);
  b->group.push_back(b->cur_group);
}
void batch_add_built(cgx_batch *b, const Built &x) {
  if (!x.nst) {
    batch_push(b, x.d, x.bytes, x.points, x.ntiles, -1, -1);
    return;
  }
  const long long base = b->tmp_elems, npts = x.tmp_elems / x.nst;
  for (int t = 0; t < x.nst; ++t) batch_push(b, x.st[t], 0, 0, x.st_ntiles, base + t * npts, -1);
  batch_push(b, x.d, x.bytes, x.points, x.ntiles, -1, base);
  b->nstage1 += x.nst;
  b->tmp_elems += x.tmp_elems;
}
// the batch's temporaries, and pdescs: the descriptors with them bound
int batch_bind(cgx_batch *b) {
  if ((size_t)b->tmp_elems > b->tmp_cap) {
    cudaFree(b->d_tmp);
    b->d_tmp = nullptr;
    b->tmp_cap = 0;
    cudaError_t e = cudaMalloc(&b->d_tmp, (size_t)b->tmp_elems * sizeof(double));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc (temporaries)");
    b->tmp_cap = (size_t)b->tmp_elems;
  }
  b->pdescs = b->descs;
  for (size_t i = 0; i < b->pdescs.size(); ++i) {
    if (b->tdst[i] >= 0) b->pdescs[i].dst = b->d_tmp + b->tdst[i];
    if (b->tsrc[i] >= 0)
      for (int t = 0; t < 3; ++t) b->pdescs[i].src[t] = b->d_tmp + b->tsrc[i];
  }
  return CGX_OK;
}
} // namespace

struct cgx_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

extern "C" {

const char *cgx_last_error(void) { return g_err.c_str(); }
const char *cgx_version(void) { return "cgx 0.1 sm_100a fp64"; }

int cgx_init(int device, int fp_mode) {
  if (fp_mode != CGX_FP_EXACT && fp_mode != CGX_FP_FMA) return fail(CGX_EINVAL, "bad fp mode");
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  g_fp_mode = fp_mode;
  return CGX_OK;
}

int cgx_set_fp_mode(int fp_mode) {
  if (fp_mode != CGX_FP_EXACT && fp_mode != CGX_FP_FMA) return fail(CGX_EINVAL, "bad fp mode");
  g_fp_mode = fp_mode;
  return CGX_OK;
}

int cgx_set_restriction(int use_higher_order, int order) {
  g_ho_restrict = use_higher_order != 0;
  g_restrict_order = order;
  return CGX_OK;
}

int cgx_find_source_timelevel(const double *times, int ntimes, double time, int order_time,
                              int op, int *timelevel0, int *ntimelevels) {
  return find_tl(times, ntimes, time, order_time, op, timelevel0, ntimelevels);
}

int cgx_transfer(int op, int cent, const cgx_array *dst, const cgx_array *srcs, const double *times,
                 int nsrc, const int dstbox[9], const int srcbox[9], const int *slab_offset,
                 double time, int order_space, int order_time, void *stream) {
  Built b;
  int rc = build(op, cent, dst, srcs, times, nsrc, dstbox, srcbox, slab_offset, time, order_space,
                 order_time, &b);
  if (rc) return rc;
  if (b.nst) return launch_staged(b, g_fp_mode, nullptr, (cudaStream_t)stream);
  return launch_pair(b.d, b.ntiles, g_fp_mode, nullptr, (cudaStream_t)stream);
}

int cgx_copy(int op, int cent, const cgx_array *dst, const cgx_array *src, const int dstbox[9],
             const int srcbox[9], const int *slab_offset, void *stream) {
  // gdata::copy_data, gdata.cc:110-122
  const double t0 = 0.0;
  return cgx_transfer(op, cent, dst, src, &t0, 1, dstbox, srcbox, slab_offset, 0.0,
                      cent == CGX_VERTEX ? 1 : 0, 0, stream);
}

int cgx_batch_create(cgx_batch **out) {
  if (!out) return fail(CGX_EINVAL, "null batch");
  cgx_batch *b = new cgx_batch();
  // per segment a claim counter and, NSEG further, an exit count (the
  // kernels reset both when they finish)
  cudaError_t e = cudaMalloc(&b->d_counter, 2 * NSEG * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(b->d_counter, 0, 2 * NSEG * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_status, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(b->d_status, 0, sizeof(int));
  if (e != cudaSuccess) {
    cudaFree(b->d_counter);
    delete b;
    return cuda_fail(e, "cudaMalloc");
  }
  *out = b;
  return CGX_OK;
}

int cgx_batch_destroy(cgx_batch *b) {
  if (!b) return CGX_OK;
  cudaFree(b->d_descs);
  cudaFree(b->d_prefix);
  cudaFree(b->d_tmap);
  cudaFree(b->d_maps);
  cudaFree(b->d_counter);
  cudaFree(b->d_status);
  cudaFree(b->d_tmp);
  for (cudaStream_t x : b->side) cudaStreamDestroy(x);
  for (cudaEvent_t x : b->ev) cudaEventDestroy(x);
  delete b;
  return CGX_OK;
}

int cgx_batch_clear(cgx_batch *b) {
  if (!b) return fail(CGX_EINVAL, "null batch");
  b->descs.clear();
  b->bytes.clear();
  b->points.clear();
  b->ntiles.clear();
  b->high.clear();
  b->tdst.clear();
  b->tsrc.clear();
  b->group.clear();
  b->cur_group = 0;
  b->tmp_elems = 0;
  b->nstage1 = 0;
  return CGX_OK;
}

int cgx_debug_skip_tma_plane(int enable) {
  g_debug_skip_tma = enable != 0;
  return CGX_OK;
}

int cgx_batch_set_max_ctas(cgx_batch *b, int tma_per_sm, int stream_per_sm) {
  if (!b) return fail(CGX_EINVAL, "null batch");
  if (tma_per_sm < 0 || stream_per_sm < 0) return fail(CGX_EINVAL, "CTA caps must not be negative");
  b->max_ctas[0] = tma_per_sm;
  b->max_ctas[1] = stream_per_sm;
  return CGX_OK;
}

int cgx_batch_set_group(cgx_batch *b, int group) {
  if (!b) return fail(CGX_EINVAL, "null batch");
  if (group < 0) return fail(CGX_EINVAL, "group must not be negative");
  b->cur_group = group;
  return CGX_OK;
}

int cgx_batch_add(cgx_batch *b, int op, int cent, const cgx_array *dst, const cgx_array *srcs,
                  const double *times, int nsrc, const int dstbox[9], const int srcbox[9],
                  const int *slab_offset, double time, int order_space, int order_time) {
  if (!b) return fail(CGX_EINVAL, "null batch");
  Built x;
  int rc = build(op, cent, dst, srcs, times, nsrc, dstbox, srcbox, slab_offset, time, order_space,
                 order_time, &x);
  if (rc) return rc;
  batch_add_built(b, x);
  return CGX_OK;
}

int cgx_batch_add_many(cgx_batch *b, int op, int cent, const cgx_array *arrays, int npairs,
                       const int *dst_idx, const int *src_idx, int nsrc, const double *times,
                       const int *dstboxes, const int *srcboxes, double time, int order_space,
                       int order_time) {
  if (!b || npairs < 0 || nsrc < 1 || nsrc > 5 ||
      (npairs > 0 && (!arrays || !dst_idx || !src_idx || !dstboxes || !srcboxes)))
    return fail(CGX_EINVAL, "add_many: bad arguments");
  b->descs.reserve(b->descs.size() + npairs);
  cgx_array srcs[5];
  for (int i = 0; i < npairs; ++i) {
    for (int t = 0; t < nsrc; ++t) srcs[t] = arrays[src_idx[nsrc * i + t]];
    Built x;
    int rc = build(op, cent, &arrays[dst_idx[i]], srcs, times, nsrc, dstboxes + 9 * (size_t)i,
                   srcboxes + 9 * (size_t)i, nullptr, time, order_space, order_time, &x);
    if (rc) return rc;
    batch_add_built(b, x);
  }
  return CGX_OK;
}

int cgx_batch_stats(const cgx_batch *b, int64_t *npairs, int64_t *ntiles, int64_t *dst_points,
                    int64_t *bytes) {
  if (!b) return fail(CGX_EINVAL, "null batch");
  int64_t t = 0, p = 0, by = 0;
  for (size_t i = 0; i < b->descs.size(); ++i) { t += b->ntiles[i]; p += b->points[i]; by += b->bytes[i]; }
  if (npairs) *npairs = (int64_t)b->descs.size() - b->nstage1;
  if (ntiles) *ntiles = t;
  if (dst_points) *dst_points = p;
  if (bytes) *bytes = by;
  return CGX_OK;
}

static int ensure_side_streams(cgx_batch *b);
int cgx_batch_upload(cgx_batch *b, void *stream) {
  if (!b) return fail(CGX_EINVAL, "null batch");
  cudaStream_t s = (cudaStream_t)stream;
  int brc = batch_bind(b);
  if (brc) return brc;
  // queue order: by tile-map segment (prolongation, then each streaming
  // variant); within a segment, largest work per tile first, so that a
  // persistent kernel's last claims are small ones
  std::vector<int> order;
  b->high_idx.clear();
  for (size_t i = 0; i < b->descs.size(); ++i) {
    if (b->high[i]) b->high_idx.push_back((int)i);
    else order.push_back((int)i);
  }
  // prolongation descriptors whose arrays TMA can stage are tiled in their
  // variant's configuration and get tensor maps
  std::vector<CUtensorMap> em(3 * b->descs.size());
  std::vector<Desc> dq(b->pdescs);
  std::vector<long long> ntq(b->ntiles.begin(), b->ntiles.end());
  for (int i : order) {
    if (!is_stencil(dq[i].kind)) continue;
    const int v = tma_variant(dq[i]);
    Desc t = dq[i];
    long long nt = 0;
    if (v >= 0) nt = prolong_tiles_tma(t, b->tma_cfg[v]);
    if (v >= 0 && nt > 0 && nt < (1LL << 31) && encode_tma_maps(t, &em[3 * (size_t)i])) {
      dq[i] = t;
      ntq[i] = nt;
    } else {
      dq[i].bx = 0;
    }
  }
  auto weight = [&](int i) { return (double)b->points[i] / (double)std::max(1LL, ntq[i]); };
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
    const int sa = segment_of(dq[a]), sc = segment_of(dq[c]);
    if (sa != sc) return sa < sc;
    return weight(a) > weight(c);
  });
  const size_t n = order.size();
  if (n > b->d_cap) {
    cudaFree(b->d_descs);
    cudaFree(b->d_prefix);
    cudaFree(b->d_maps);
    b->d_descs = nullptr;
    b->d_prefix = nullptr;
    b->d_maps = nullptr;
    size_t cap = std::max<size_t>(n, 64);
    cudaError_t e = cudaMalloc(&b->d_descs, cap * sizeof(Desc));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_prefix, cap * sizeof(long long));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_maps, 3 * cap * sizeof(CUtensorMap));
    if (e != cudaSuccess) { b->d_cap = 0; return cuda_fail(e, "cudaMalloc"); }
    b->d_cap = cap;
  }
  std::vector<Desc> hd(n);
  std::vector<CUtensorMap> hm3(3 * n);
  std::vector<long long> hp(n);
  long long acc = 0;
  long long cnt[NSEG] = {0};
  for (size_t i = 0; i < n; ++i) {
    hd[i] = dq[order[i]];
    for (int t = 0; t < 3; ++t) hm3[3 * i + t] = em[3 * (size_t)order[i] + t];
    hp[i] = acc;
    acc += ntq[order[i]];
    cnt[segment_of(hd[i])] += ntq[order[i]];
  }
  b->seg[0] = 0;
  for (int i = 0; i < NSEG; ++i) b->seg[i + 1] = b->seg[i] + cnt[i];
  b->n_uploaded = (int)n;
  b->tiles_uploaded = acc;
  b->fp_mode = g_fp_mode;
  if ((size_t)acc > b->tmap_cap) {
    cudaFree(b->d_tmap);
    b->d_tmap = nullptr;
    size_t cap = std::max<size_t>((size_t)acc, 1024);
    cudaError_t e = cudaMalloc(&b->d_tmap, cap * sizeof(int2));
    if (e != cudaSuccess) { b->tmap_cap = 0; return cuda_fail(e, "cudaMalloc"); }
    b->tmap_cap = cap;
  }
  std::vector<int2> hm((size_t)acc);
  for (size_t i = 0; i < n; ++i)
    for (long long k = 0; k < ntq[order[i]]; ++k) hm[(size_t)hp[i] + k] = make_int2((int)i, (int)k);
  if (n) {
    cudaError_t e = cudaMemcpyAsync(b->d_descs, hd.data(), n * sizeof(Desc), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(b->d_prefix, hp.data(), n * sizeof(long long), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(b->d_tmap, hm.data(), hm.size() * sizeof(int2), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(b->d_maps, hm3.data(), hm3.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s); // host vectors are temporaries
    if (e != cudaSuccess) return cuda_fail(e, "descriptor upload");
  }
  return ensure_side_streams(b);
}

// The tile map's segments, one kernel each.  Pairs of a batch write
// disjoint points and read none that another pair writes, so the segments
// are independent, except the time-combination segment (the last), which
// reads the temporaries that its staged pairs' first stages write in the
// other segments.  Every other non-empty segment therefore runs on a
// stream of its own, forked from s and joined back into it (which also
// works while s is being captured), and the time segment runs on s after
// the join.  A batch with one such segment launches as one chain on s.
// indices of the non-empty segments before the time segment
static int concurrent_segments(const cgx_batch *b, int *idx) {
  constexpr int TSEG = SEG_STREAM + SV_TIME;
  int n = 0;
  for (int i = 0; i < TSEG; ++i)
    if (b->seg[i + 1] > b->seg[i]) idx[n++] = i;
  return n;
}

// The side streams and events of the concurrent launch, created when the
// batch is uploaded (on the device current then), so that no launch -- a
// captured one included -- creates any.
static int ensure_side_streams(cgx_batch *b) {
  int idx[NSEG];
  const int n = concurrent_segments(b, idx);
  const size_t nside = n > 1 ? (size_t)n - 1 : 0;
  while (b->side.size() < nside) {
    cudaStream_t x = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreateWithFlags");
    b->side.push_back(x);
  }
  while (b->ev.size() < nside + 1) {
    cudaEvent_t x = nullptr;
    cudaError_t e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_fail(e, "cudaEventCreateWithFlags");
    b->ev.push_back(x);
  }
  return CGX_OK;
}

static int launch_segments(cgx_batch *b, cudaStream_t s) {
  int need = 0;
  const int rc = launch_map_concurrent(b->fp_mode, b->d_descs, b->d_maps, b->d_tmap, b->seg, b->tma_cfg,
                                       b->d_counter, b->d_status, s, b->side.data(), b->ev.data(),
                                       (int)std::min(b->side.size(), b->ev.size() ? b->ev.size() - 1 : 0),
                                       &need, b->max_ctas);
  if (rc == CGX_EINVAL && need > 0)
    return fail(CGX_EINVAL, "batch launch: the batch was not uploaded on this device");
  return rc;
}

int cgx_batch_launch(cgx_batch *b, void *stream) {
  if (!b) return fail(CGX_EINVAL, "null batch");
  cudaStream_t s = (cudaStream_t)stream;
  // the per-box descriptors first: a staged pair's first stage may be one,
  // and its second stage runs in the last segment of the tile map
  for (int i : b->high_idx) {
    int rc = launch_pair(b->pdescs[i], b->ntiles[i], b->fp_mode, b->d_status, s);
    if (rc) return rc;
  }
  if (b->n_uploaded > 0) {
    // the segment kernels leave their counters at zero: no memset between
    // the launches, which run chained on each stream
    int rc = launch_segments(b, s);
    if (rc) return rc;
  }
  return CGX_OK;
}

// The autotuner: for every TMA prolongation variant present, run its
// segment of the batch in each tile configuration (one untimed launch, then
// `reps` launches timed one by one with events; the median scores) and keep
// the fastest; then upload with the choices.  Repeated launches of a batch write the same values
// (pairs write disjoint points and read none of them), so tuning on the
// caller's own data is safe.
static_assert(CGX_TMA_VARIANTS == TV_COUNT && CGX_TMA_CONFIGS == TMA_NCFG, "tuning constants of the C-ABI");
int cgx_batch_autotune(cgx_batch *b, int reps, void *stream, int *chosen) {
  if (!b || reps < 1) return fail(CGX_EINVAL, "autotune: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  int rc = cgx_batch_upload(b, stream);
  if (rc) return rc;
  bool present[TV_COUNT];
  for (int v = 0; v < TV_COUNT; ++v) present[v] = b->seg[v + 1] > b->seg[v];
  // each launch timed on its own; a configuration scores the median
  std::vector<cudaEvent_t> ev(2 * (size_t)reps, nullptr);
  cudaError_t e = cudaSuccess;
  for (auto &x : ev)
    if (e == cudaSuccess) e = cudaEventCreate(&x);
  if (e != cudaSuccess) {
    for (auto x : ev)
      if (x) cudaEventDestroy(x);
    return cuda_fail(e, "cudaEventCreate");
  }
  auto run_segment = [&](int v) {
    long long sg[NSEG + 1];
    for (int i = 0; i <= NSEG; ++i) sg[i] = i <= v ? b->seg[v] : b->seg[v + 1];
    cudaError_t m = cudaMemsetAsync(b->d_counter, 0, NSEG * sizeof(unsigned long long), s);
    if (m != cudaSuccess) return cuda_fail(m, "cudaMemsetAsync");
    return launch_map(b->fp_mode, b->d_descs, b->d_maps, b->d_tmap, sg, b->tma_cfg, b->d_counter,
                      b->d_status, s);
  };
  for (int v = 0; v < TV_COUNT && rc == CGX_OK; ++v) {
    if (!present[v]) continue;
    int best = 0;
    float best_ms = 0.f;
    for (int c = 0; c < TMA_NCFG && rc == CGX_OK; ++c) {
      b->tma_cfg[v] = c;
      if ((rc = cgx_batch_upload(b, stream))) break;
      if ((rc = run_segment(v))) break;
      for (int r = 0; r < reps && rc == CGX_OK && e == cudaSuccess; ++r) {
        e = cudaEventRecord(ev[2 * r], s);
        if (e == cudaSuccess) rc = run_segment(v);
        if (e == cudaSuccess) e = cudaEventRecord(ev[2 * r + 1], s);
      }
      if (e == cudaSuccess) e = cudaEventSynchronize(ev[2 * reps - 1]);
      std::vector<float> t((size_t)reps, 0.f);
      for (int r = 0; r < reps && e == cudaSuccess; ++r) e = cudaEventElapsedTime(&t[r], ev[2 * r], ev[2 * r + 1]);
      if (e != cudaSuccess) rc = cuda_fail(e, "autotune timing");
      if (rc) break;
      std::sort(t.begin(), t.end());
      const float ms = t[(size_t)reps / 2];
      if (c == 0 || ms < best_ms) {
        best = c;
        best_ms = ms;
      }
    }
    b->tma_cfg[v] = best;
  }
  for (auto x : ev) cudaEventDestroy(x);
  if (rc) return rc;
  if (chosen)
    for (int v = 0; v < TV_COUNT; ++v) chosen[v] = present[v] ? b->tma_cfg[v] : -1;
  return cgx_batch_upload(b, stream);
}

int cgx_batch_set_config(cgx_batch *b, int variant, int config) {
  if (!b || variant < -1 || variant >= TV_COUNT || config < 0 || config >= TMA_NCFG)
    return fail(CGX_EINVAL, "set_config: variant %d / configuration %d out of range", variant, config);
  for (int v = 0; v < TV_COUNT; ++v)
    if (variant < 0 || v == variant) b->tma_cfg[v] = config;
  return CGX_OK;
}

int cgx_batch_kernels(const cgx_batch *b, int *nkernels) {
  if (!b || !nkernels) return fail(CGX_EINVAL, "null batch");
  int n = (int)b->high_idx.size();
  if (b->n_uploaded > 0)
    for (int i = 0; i < NSEG; ++i) n += b->seg[i + 1] > b->seg[i];
  *nkernels = n;
  return CGX_OK;
}

int cgx_batch_launch_per_box(cgx_batch *b, void *stream) {
  if (!b) return fail(CGX_EINVAL, "null batch");
  int brc = batch_bind(b);
  if (brc) return brc;
  // in queue order: a staged pair's stages follow one another
  for (size_t i = 0; i < b->pdescs.size(); ++i) {
    int rc = launch_pair(b->pdescs[i], b->ntiles[i], g_fp_mode, b->d_status, (cudaStream_t)stream);
    if (rc) return rc;
  }
  return CGX_OK;
}

int cgx_batch_check(cgx_batch *b, void *stream) {
  if (!b) return fail(CGX_EINVAL, "null batch");
  int st = 0;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(&st, b->d_status, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "status read");
  if (st) {
    // a kernel that gave up may have left its counters behind
    cudaMemsetAsync(b->d_status, 0, sizeof(int), s);
    cudaMemsetAsync(b->d_counter, 0, 2 * NSEG * sizeof(unsigned long long), s);
    return fail(st, "a kernel reported status %d", st);
  }
  return CGX_OK;
}

int cgx_graph_begin(void *stream) {
  cudaError_t e = cudaStreamBeginCapture((cudaStream_t)stream, cudaStreamCaptureModeThreadLocal);
  return e == cudaSuccess ? CGX_OK : cuda_fail(e, "cudaStreamBeginCapture");
}

int cgx_graph_end(void *stream, cgx_graph **out) {
  if (!out) return fail(CGX_EINVAL, "null graph");
  cgx_graph *g = new cgx_graph();
  cudaError_t e = cudaStreamEndCapture((cudaStream_t)stream, &g->graph);
  if (e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (e != cudaSuccess) {
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return cuda_fail(e, "graph capture");
  }
  *out = g;
  return CGX_OK;
}

int cgx_graph_launch(cgx_graph *g, void *stream) {
  if (!g) return fail(CGX_EINVAL, "null graph");
  cudaError_t e = cudaGraphLaunch(g->exec, (cudaStream_t)stream);
  return e == cudaSuccess ? CGX_OK : cuda_fail(e, "cudaGraphLaunch");
}

int cgx_graph_destroy(cgx_graph *g) {
  if (!g) return CGX_OK;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return CGX_OK;
}

int cgx_malloc(void **ptr, size_t bytes) {
  cudaError_t e = cudaMalloc(ptr, bytes);
  return e == cudaSuccess ? CGX_OK : cuda_fail(e, "cudaMalloc");
}
int cgx_free(void *ptr) {
  cudaError_t e = cudaFree(ptr);
  return e == cudaSuccess ? CGX_OK : cuda_fail(e, "cudaFree");
}
int cgx_memcpy_htod(void *dst, const void *src, size_t bytes, void *stream) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, (cudaStream_t)stream);
  return e == cudaSuccess ? CGX_OK : cuda_fail(e, "cudaMemcpyAsync");
}
int cgx_memcpy_dtoh(void *dst, const void *src, size_t bytes, void *stream) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, (cudaStream_t)stream);
  return e == cudaSuccess ? CGX_OK : cuda_fail(e, "cudaMemcpyAsync");
}
int cgx_stream_sync(void *stream) {
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  return e == cudaSuccess ? CGX_OK : cuda_fail(e, "cudaStreamSynchronize");
}

} // extern "C"


// ============================================================== chain
// A sequence of batches run as ONE persistent launch (cgx_chain.cuh): the
// tiles of batch j wait, group by group, for the previous batch of their
// group.  The descriptors, tensor maps and tile list are built here from the
// batches' host-side pairs.
struct cgx_chain {
  std::vector<cgx_batch *> batches;
  bool debug_hold = false; // cgx_chain_debug_hold
  int order = -1; // vertex-centred prolongation order of every prolongation pair
  int fp_mode = CGX_FP_EXACT;
  Desc *d_descs = nullptr;
  CUtensorMap *d_maps = nullptr;
  ChainTile *d_tiles = nullptr;
  unsigned *d_need = nullptr, *d_done = nullptr;
  unsigned long long *d_ctl = nullptr;
  int *d_status = nullptr;
  long long ntiles = 0;
  int ncounters = 0;
  long long pairs = 0, points = 0, bytes = 0;
};

namespace {
void chain_free(cgx_chain *c) {
  cudaFree(c->d_descs);
  cudaFree(c->d_maps);
  cudaFree(c->d_tiles);
  cudaFree(c->d_need);
  cudaFree(c->d_done);
  cudaFree(c->d_ctl);
  cudaFree(c->d_status);
  c->d_descs = nullptr;
  c->d_maps = nullptr;
  c->d_tiles = nullptr;
  c->d_need = c->d_done = nullptr;
  c->d_ctl = nullptr;
  c->d_status = nullptr;
  c->ntiles = 0;
  c->ncounters = 0;
}
} // namespace

extern "C" {

int cgx_chain_create(cgx_chain **out) {
  if (!out) return fail(CGX_EINVAL, "null chain");
  *out = new cgx_chain();
  return CGX_OK;
}

int cgx_chain_destroy(cgx_chain *c) {
  if (!c) return CGX_OK;
  chain_free(c);
  delete c;
  return CGX_OK;
}

int cgx_chain_debug_hold(cgx_chain *c, int hold) {
  if (!c) return fail(CGX_EINVAL, "null chain");
  c->debug_hold = hold != 0;
  return CGX_OK;
}

int cgx_chain_add(cgx_chain *c, cgx_batch *b) {
  if (!c || !b) return fail(CGX_EINVAL, "null chain or batch");
  c->batches.push_back(b);
  return CGX_OK;
}

int cgx_chain_upload(cgx_chain *c, void *stream) {
  if (!c) return fail(CGX_EINVAL, "null chain");
  cudaStream_t s = (cudaStream_t)stream;
  constexpr int CFG = 1; // the chain kernel's prolongation tile configuration
  std::vector<Desc> hd;
  std::vector<CUtensorMap> hm;
  std::vector<ChainTile> ht;
  std::vector<unsigned> need;
  int order = -1;
  long long pairs = 0, points = 0, bytes = 0;
  std::map<int, int> last_of_group; // group -> its latest counter
  for (size_t j = 0; j < c->batches.size(); ++j) {
    const cgx_batch *b = c->batches[j];
    if (b->nstage1)
      return fail(CGX_EUNSUPPORTED, "chain: batch %zu has transfers through temporaries", j);
    // this batch's descriptors group by group
    std::map<int, std::vector<int>> by_group;
    for (size_t i = 0; i < b->descs.size(); ++i) by_group[b->group[i]].push_back((int)i);
    for (auto &kv : by_group) {
      const int counter = (int)need.size();
      auto it = last_of_group.find(kv.first);
      const int dep = it == last_of_group.end() ? -1 : it->second;
      last_of_group[kv.first] = counter;
      unsigned count = 0;
      for (int i : kv.second) {
        Desc d = b->descs[i];
        long long nt = 0;
        CUtensorMap maps[3] = {};
        if (d.kind == K_PROLONG_VC) {
          const bool time_ok = d.ntl == 1 || (d.ntl == 3 && d.tkind == T_QUAD);
          if (!time_ok || (d.order != 1 && d.order != 3 && d.order != 5))
            return fail(CGX_EUNSUPPORTED,
                        "chain: batch %zu pair %d: only vertex-centred orders 1/3/5 with one "
                        "timelevel or quadratic time interpolation",
                        j, i);
          if (order >= 0 && d.order != order)
            return fail(CGX_EUNSUPPORTED, "chain: prolongation orders %d and %d mixed", order, d.order);
          order = d.order;
          nt = prolong_tiles_tma(d, CFG);
          if (nt <= 0 || nt >= (1LL << 31) || !encode_tma_maps(d, maps))
            return fail(CGX_EUNSUPPORTED,
                        "chain: batch %zu pair %d: the source arrays cannot be staged by TMA "
                        "(16-byte aligned base, even row and plane pitch)",
                        j, i);
        } else if ((d.kind == K_COPY && d.ntl == 1) || d.kind == K_RESTRICT_VC) {
          nt = b->ntiles[i];
        } else {
          return fail(CGX_EUNSUPPORTED,
                      "chain: batch %zu pair %d: only vertex-centred prolongation, one-timelevel "
                      "copies and injection run in the chain kernel",
                      j, i);
        }
        const int di = (int)hd.size();
        hd.push_back(d);
        for (int t = 0; t < 3; ++t) hm.push_back(maps[t]);
        for (long long k = 0; k < nt; ++k) ht.push_back(ChainTile{di, (int)k, counter, dep});
        count += (unsigned)nt;
        ++pairs;
        points += b->points[i];
        bytes += b->bytes[i];
      }
      need.push_back(count);
    }
  }
  if (hd.size() >= (size_t)INT_MAX || ht.size() >= (size_t)INT_MAX)
    return fail(CGX_EINVAL, "chain: too many pairs or tiles");
  if (c->debug_hold) // failure injection: no dependency is ever satisfied
    for (unsigned &n : need) n += 1;
  chain_free(c);
  const size_t nd = std::max<size_t>(hd.size(), 1), nt = std::max<size_t>(ht.size(), 1),
               nc = std::max<size_t>(need.size(), 1);
  cudaError_t e = cudaMalloc(&c->d_descs, nd * sizeof(Desc));
  if (e == cudaSuccess) e = cudaMalloc(&c->d_maps, 3 * nd * sizeof(CUtensorMap));
  if (e == cudaSuccess) e = cudaMalloc(&c->d_tiles, nt * sizeof(ChainTile));
  if (e == cudaSuccess) e = cudaMalloc(&c->d_need, nc * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMalloc(&c->d_done, nc * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMalloc(&c->d_ctl, CHAIN_CTL_WORDS * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&c->d_status, sizeof(int));
  if (e != cudaSuccess) {
    chain_free(c);
    return cuda_fail(e, "cudaMalloc (chain)");
  }
  if (!hd.empty()) e = cudaMemcpyAsync(c->d_descs, hd.data(), hd.size() * sizeof(Desc), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && !hm.empty())
    e = cudaMemcpyAsync(c->d_maps, hm.data(), hm.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && !ht.empty())
    e = cudaMemcpyAsync(c->d_tiles, ht.data(), ht.size() * sizeof(ChainTile), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && !need.empty())
    e = cudaMemcpyAsync(c->d_need, need.data(), need.size() * sizeof(unsigned), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_done, 0, nc * sizeof(unsigned), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_ctl, 0, CHAIN_CTL_WORDS * sizeof(unsigned long long), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_status, 0, sizeof(int), s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s); // the host vectors are temporaries
  if (e != cudaSuccess) {
    chain_free(c);
    return cuda_fail(e, "chain upload");
  }
  c->ntiles = (long long)ht.size();
  c->ncounters = (int)need.size();
  c->order = order < 0 ? 5 : order;
  c->fp_mode = g_fp_mode;
  c->pairs = pairs;
  c->points = points;
  c->bytes = bytes;
  return CGX_OK;
}

int cgx_chain_launch(cgx_chain *c, void *stream) {
  if (!c) return fail(CGX_EINVAL, "null chain");
  if (c->ntiles == 0) return CGX_OK;
  return klaunch_chain(c->fp_mode == CGX_FP_FMA ? 1 : 0, c->order, c->d_descs, c->d_maps, c->d_tiles, c->ntiles,
                       c->d_need, c->d_done, c->ncounters, c->d_ctl, c->d_status, (cudaStream_t)stream);
}

int cgx_chain_check(cgx_chain *c, void *stream) {
  if (!c) return fail(CGX_EINVAL, "null chain");
  if (!c->d_status) return CGX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  int st = 0;
  cudaError_t e = cudaMemcpyAsync(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "chain status read-back");
  if (st) {
    // the kernel resets its counters on exit; clear the status for reuse
    e = cudaMemsetAsync(c->d_status, 0, sizeof(int), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return fail(CGX_EDEVICE, "chain: a bounded device wait gave up (status %d)", st);
  }
  return CGX_OK;
}

int cgx_chain_stats(const cgx_chain *c, int64_t *npairs, int64_t *ntiles, int64_t *dst_points,
                    int64_t *bytes) {
  if (!c) return fail(CGX_EINVAL, "null chain");
  if (npairs) *npairs = c->pairs;
  if (ntiles) *ntiles = c->ntiles;
  if (dst_points) *dst_points = c->points;
  if (bytes) *bytes = c->bytes;
  return CGX_OK;
}

} // extern "C"

// ============================================================== no-allocation form
// cgx_transfer_pairs_noalloc runs a list of box-pairs through the persistent
// kernel without allocating device memory.  The kernel's scratch -- the
// descriptor queue, the tile prefix sums, the work counter and the status
// word -- lives in one fixed-size array in the library's own device image,
// created when a GPU loads the library and held until the process exits.
namespace {

constexpr int kNoAllocMaxPairs = CGX_NOALLOC_MAX_PAIRS;
constexpr size_t kNoAllocDescBytes = sizeof(Desc) * kNoAllocMaxPairs;
constexpr size_t kNoAllocPrefixOff = (kNoAllocDescBytes + 255) / 256 * 256;
constexpr size_t kNoAllocCounterOff =
    (kNoAllocPrefixOff + sizeof(long long) * kNoAllocMaxPairs + 255) / 256 * 256;
constexpr size_t kNoAllocBytes = kNoAllocCounterOff + 256; // counter + status

// The scratch itself.  In host code this name only stands in for the symbol:
// its device address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
unsigned char *g_noalloc_dev[kMaxDevices] = {nullptr};

// Device address of the scratch on the current device; the first call on a
// device looks it up (that call must not be inside a stream capture).
int noalloc_scratch(unsigned char **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(CGX_EINVAL, "device index %d out of range", dev);
  if (!g_noalloc_dev[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress");
    g_noalloc_dev[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_noalloc_dev[dev];
  return CGX_OK;
}

} // namespace

extern "C" int cgx_transfer_pairs_noalloc(const cgx_pair *pairs, int npairs, void *stream) {
  if (npairs < 0 || (npairs > 0 && !pairs)) return fail(CGX_EINVAL, "bad pair list");
  if (npairs > kNoAllocMaxPairs)
    return fail(CGX_EINVAL,
                "cgx_transfer_pairs_noalloc: %d box-pairs exceed the fixed maximum of %d; "
                "split the list or use cgx_batch_*",
                npairs, kNoAllocMaxPairs);
  if (npairs == 0) return CGX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  // The descriptors are copied from host memory that lives only for this
  // call; a capture would record copies that read it after the call.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t ce = cudaStreamIsCapturing(s, &cap);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamIsCapturing");
  if (cap != cudaStreamCaptureStatusNone)
    return fail(CGX_EUNSUPPORTED, "cgx_transfer_pairs_noalloc cannot run inside a stream capture: "
                                  "it copies its descriptors from host memory that the call does "
                                  "not keep");
  unsigned char *base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc) return rc;
  Desc *d_descs = reinterpret_cast<Desc *>(base);
  long long *d_prefix = reinterpret_cast<long long *>(base + kNoAllocPrefixOff);
  unsigned long long *d_counter = reinterpret_cast<unsigned long long *>(base + kNoAllocCounterOff);
  int *d_status = reinterpret_cast<int *>(base + kNoAllocCounterOff + sizeof(unsigned long long));

  // Validate on the host into small stack chunks and copy each chunk into
  // the scratch; cudaMemcpyAsync has staged pageable sources when it returns.
  constexpr int kChunk = 16;
  Desc hd[kChunk];
  long long hp[kChunk];
  long long tiles = 0;
  for (int i0 = 0; i0 < npairs; i0 += kChunk) {
    const int n = std::min(kChunk, npairs - i0);
    for (int i = 0; i < n; ++i) {
      const cgx_pair &p = pairs[i0 + i];
      if (p.nsrc < 1 || p.nsrc > 3)
        return fail(CGX_EINVAL, "pair %d: nsrc must be 1..3", i0 + i);
      Built b;
      rc = build(p.op, p.cent, &p.dst, p.srcs, p.times, p.nsrc, p.dstbox, p.srcbox,
                 p.has_slab ? p.slab_offset : nullptr, p.time, p.order_space, p.order_time, &b);
      if (rc) return rc;
      if (b.nst)
        return fail(CGX_EUNSUPPORTED,
                    "pair %d: a transfer through per-timelevel temporaries (restriction between "
                    "timelevels, order_time 3 or 4) is not available without allocation", i0 + i);
      if (b.d.kind == K_PROLONG_VC && b.d.order >= 7)
        return fail(CGX_EUNSUPPORTED,
                    "pair %d: vertex-centred order %d is not available without allocation",
                    i0 + i, b.d.order);
      hd[i] = b.d;
      hp[i] = tiles;
      tiles += b.ntiles;
    }
    cudaError_t e = cudaMemcpyAsync(d_descs + i0, hd, n * sizeof(Desc), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_prefix + i0, hp, n * sizeof(long long), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "scratch upload");
  }
  // the work counter and the status word start at zero on every call
  cudaError_t e = cudaMemsetAsync(base + kNoAllocCounterOff, 0, 256, s);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
  return g_fp_mode == CGX_FP_FMA
             ? klaunch_search_f1(d_descs, d_prefix, npairs, tiles, d_counter, d_status, s)
             : klaunch_search_f0(d_descs, d_prefix, npairs, tiles, d_counter, d_status, s);
}

// The status word the kernel of the last cgx_transfer_pairs_noalloc call on
// the current device left in the fixed scratch (the next call clears it).
// Waits for the stream, then reads the word into host memory; allocates
// nothing.
extern "C" int cgx_noalloc_check(void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  unsigned char *base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc) return rc;
  int status = 0;
  cudaError_t e = cudaMemcpyAsync(&status, base + kNoAllocCounterOff + sizeof(unsigned long long),
                                  sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "status read-back");
  if (status)
    return fail(status, "cgx_transfer_pairs_noalloc: the kernel reported status %d (a bounded "
                        "device wait gave up, or a descriptor had no tile routine)", status);
  return CGX_OK;
}

// ============================================================== internal API
namespace cgx {

int launch_map_concurrent(int fp, const Desc *d, const CUtensorMap *maps, const int2 *tmap,
                          const long long seg[NSEG + 1], const int *cfg, unsigned long long *counter,
                          int *status, cudaStream_t s, const cudaStream_t *side, const cudaEvent_t *ev,
                          int nside_have, int *need, const int *caps) {
  constexpr int TSEG = SEG_STREAM + SV_TIME;
  static_assert(TSEG == NSEG - 1, "the time combination is the last segment");
  int idx[NSEG], n = 0;
  for (int i = 0; i < TSEG; ++i)
    if (seg[i + 1] > seg[i]) idx[n++] = i;
  *need = 0;
  if (n <= 1) return launch_map(fp, d, maps, tmap, seg, cfg, counter, status, s, caps);
  const int nside = n - 1;
  if (nside_have < nside) {
    *need = nside;
    return fail(CGX_EINVAL, "concurrent launch: %d side streams needed, %d given", nside, nside_have);
  }
  // a segment array in which only segment i is non-empty
  auto only = [&](int i, long long *sg) {
    for (int k = 0; k <= NSEG; ++k) sg[k] = k <= i ? seg[i] : seg[i + 1];
  };
  // fork: every side stream that has waited on ev[0] is joined below, also
  // when a later fork step or a launch fails (a capture stays joined)
  int forked = 0;
  cudaError_t e = cudaEventRecord(ev[0], s);
  while (e == cudaSuccess && forked < nside) {
    e = cudaStreamWaitEvent(side[forked], ev[0], 0);
    if (e == cudaSuccess) ++forked;
  }
  int rc = e != cudaSuccess ? cuda_fail(e, "fork of the segment streams") : CGX_OK;
  for (int j = 0; j < n && rc == CGX_OK; ++j) {
    long long sg[NSEG + 1];
    only(idx[j], sg);
    rc = launch_map(fp, d, maps, tmap, sg, cfg, counter, status, j == 0 ? s : side[j - 1], caps);
  }
  // join every forked side stream, also after a failure
  cudaError_t je = cudaSuccess;
  for (int k = 0; k < forked; ++k) {
    cudaError_t r = cudaEventRecord(ev[1 + k], side[k]);
    if (r == cudaSuccess) r = cudaStreamWaitEvent(s, ev[1 + k], 0);
    if (r != cudaSuccess && je == cudaSuccess) je = r;
  }
  if (rc) return rc;
  if (je != cudaSuccess) return cuda_fail(je, "join of the segment streams");
  if (seg[TSEG + 1] > seg[TSEG]) {
    long long sg[NSEG + 1];
    only(TSEG, sg);
    rc = launch_map(fp, d, maps, tmap, sg, cfg, counter, status, s, caps);
  }
  return rc;
}

thread_local int g_cta_cap[2] = {0, 0};

int host_build(int op, int cent, const cgx_array *dst, const cgx_array *srcs, const double *times,
               int nsrc, const int *dstbox, const int *srcbox, const int *slab, double time,
               int order_space, int order_time, BuiltPair *out) {
  Built b;
  int rc = build(op, cent, dst, srcs, times, nsrc, dstbox, srcbox, slab, time, order_space,
                 order_time, &b);
  if (rc) return rc;
  if (b.nst) return fail(CGX_EUNSUPPORTED, "a transfer through per-timelevel temporaries");
  out->d = b.d;
  out->bytes = b.bytes;
  out->points = b.points;
  out->ntiles = b.ntiles;
  return CGX_OK;
}

int batch_pairs(const cgx_batch *b, const Desc **descs, const int **ntiles, const long long **points,
                const long long **bytes, int *n) {
  if (!b) return fail(CGX_EINVAL, "null batch");
  for (size_t i = 0; i < b->high.size(); ++i)
    if (b->high[i]) return fail(CGX_EUNSUPPORTED, "vertex-centred orders 7-11 cannot be served");
  if (b->nstage1)
    return fail(CGX_EUNSUPPORTED, "transfers through per-timelevel temporaries cannot be served");
  *descs = b->descs.data();
  *ntiles = b->ntiles.data();
  *points = b->points.data();
  *bytes = b->bytes.data();
  *n = (int)b->descs.size();
  return CGX_OK;
}

int launch_tile_map(const Desc *d_descs, const CUtensorMap *d_maps, const int2 *d_tmap,
                    const long long seg[NSEG + 1], unsigned long long *d_counter, int *d_status, int fp,
                    cudaStream_t s) {
  if (seg[NSEG] <= 0) return CGX_OK;
  cudaError_t e = cudaMemsetAsync(d_counter, 0, NSEG * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
  return launch_map(fp, d_descs, d_maps, d_tmap, seg, nullptr, d_counter, d_status, s);
}

// A prolongation descriptor's tiles in TMA tile configuration `config`
// (the tiling of a batch upload); returns the tile count, <= 0 if none.
long long tile_prolongation(Desc &d, int config) {
  return prolong_tiles_tma(d, config);
}

bool encode_tma_maps(const Desc &d, CUtensorMap maps[3]) {
  if (!is_stencil(d.kind) || d.bx == 0 || tma_variant(d) < 0) return false;
  // row and plane pitches must be multiples of 16 bytes
  if (d.ssy % 2 || d.ssz % 2 || d.ssz >= (1LL << 37)) return false;
  PFN_cuTensorMapEncodeTiled_v12000 enc = tma_encoder();
  if (!enc) return false;
  for (int t = 0; t < d.ntl; ++t) {
    if (reinterpret_cast<uintptr_t>(d.src[t]) % 16) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)d.sext[0], (cuuint64_t)d.sext[1], (cuuint64_t)d.sext[2]};
    const cuuint64_t strides[2] = {(cuuint64_t)d.ssy * 8, (cuuint64_t)d.ssz * 8};
    const cuuint32_t box[3] = {d.bx, d.by, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(&maps[t], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double *>(d.src[t]), dims,
                     strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
  }
  return true;
}

int launch_one_pair(const Desc &d, int ntiles, int fp, int *status, cudaStream_t s) {
  return launch_pair(d, ntiles, fp, status, s);
}

int current_fp_mode() { return g_fp_mode; }

int set_error(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

int cuda_error(cudaError_t e, const char *what) { return cuda_fail(e, what); }

} // namespace cgx
