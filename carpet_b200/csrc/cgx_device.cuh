// cgx_device.cuh -- device side of the grid-transfer kernels (sm_100a, FP64).
//
// One descriptor describes one box-pair: a destination region and where its
// sources lie.  A descriptor is cut into tiles; one CTA of 256 threads runs
// one tile at a time.  The same tile routines serve the plain per-box kernel
// (a grid of the pair's tiles) and the persistent batched kernel (tiles taken
// from a device work queue across many pairs).
//
// Arithmetic follows CarpetLib's operation order exactly (see the operator
// families below); FMA selects whether each multiply-add is fused
// (__fma_rn) or rounded twice (__dmul_rn then __dadd_rn).  The intrinsics
// are never contracted by the compiler, so the exact mode is bit-identical
// to the reference built without contraction.
#pragma once
#include <cstdint>

namespace cgx {

enum Kind : int {
  K_COPY = 0,        // copy_3d (+ time interpolation when ntl > 1)
  K_RESTRICT_VC = 1, // restrict_3d_rf2 (injection)
  K_RESTRICT_CC = 2, // restrict_3d_cc_rf2 (8-point average)
  K_PROLONG_VC = 3,  // prolongate_3d_rf2<ORDER>
  K_PROLONG_CC = 4,  // prolongate_3d_cc_rf2<ORDER>
  K_PROLONG_ENO = 5, // prolongate_3d_real8_eno
  K_NKINDS = 6
};

enum TKind : int { T_NONE = 0, T_LIN = 1, T_QUAD = 2, T_ENO = 3 };

// Tile geometry.
constexpr int NTHREADS = 256;
// prolongation: 32 fine x (one per lane) by 14 fine y (8 coarse rows, one
// per warp) by a z chunk marched plane by plane
constexpr int PTX = 32, PTY = 14, PTZ = 32;
// copy / restriction: 32 x by 8 y by 8 z destination points
constexpr int CTX = 32, CTY = 8, CTZ = 8;

struct Desc {
  int kind, order, ntl, tkind;
  int n[3];     // destination region extent (points)
  int soff[3];  // source offset of the region start (meaning per kind)
  int doff[3];  // destination index of the region start
  int sext[3];  // logical extent of the source arrays (load clamp)
  int tiles[3]; // tile grid over the region
  int pad_;
  long long ssy, ssz; // source strides (elements) in y and z
  long long dsy, dsz; // destination strides
  const double *src[3];
  double *dst;
  double w[8]; // time weights (layout of the oracle's cgxo_time_weights)
};

// ---------------------------------------------------------------- arithmetic
template <int FMA> __device__ __forceinline__ double madd(double a, double b, double c) {
  if (FMA)
    return __fma_rn(a, b, c);
  return __dadd_rn(__dmul_rn(a, b), c);
}
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }

// Coefficients as exact dyadic rationals (numerator / 2^k).
// prolongate_3d_rf2.cc:92-124
__device__ __forceinline__ double vc_coeff(int order, int m) {
  switch (order) {
  case 1: return 0.5;
  case 3: { const double c[4] = {-1, 9, 9, -1}; return c[m] * 0.0625; }
  case 5: { const double c[6] = {3, -25, 150, 150, -25, 3}; return c[m] * (1.0 / 256); }
  case 7: { const double c[8] = {-5, 49, -245, 1225, 1225, -245, 49, -5}; return c[m] * (1.0 / 2048); }
  case 9: { const double c[10] = {35, -405, 2268, -8820, 39690, 39690, -8820, 2268, -405, 35};
            return c[m] * (1.0 / 65536); }
  default: { const double c[12] = {-63, 847, -5445, 22869, -76230, 320166,
                                    320166, -76230, 22869, -5445, 847, -63};
             return c[m] * (1.0 / 524288); }
  }
}
// prolongate_3d_cc_rf2.cc:116-139; di == 1 reverses the stencil (:67)
__device__ __forceinline__ double cc_coeff(int order, int di, int m) {
  int n = order + 1;
  int j = di ? n - 1 - m : m;
  switch (order) {
  case 0: return 1.0;
  case 1: { const double c[2] = {1, 3}; return c[j] * 0.25; }
  case 2: { const double c[3] = {5, 30, -3}; return c[j] * (1.0 / 32); }
  case 3: { const double c[4] = {-5, 35, 105, -7}; return c[j] * (1.0 / 128); }
  case 4: { const double c[5] = {-45, 420, 1890, -252, 35}; return c[j] * (1.0 / 2048); }
  default: { const double c[6] = {63, -495, 2310, 6930, -693, 77}; return c[j] * (1.0 / 8192); }
  }
}

// ---------------------------------------------------------------- families
// A family is a separable 1-D rule: the fine point with source position s
// (fine units) has coarse base c = s >> 1 and parity p = s & 1; its value on
// one axis is a function of the coarse values around c.  [LO, HI] is the
// union of the windows of both parities relative to c.  CarpetLib nests the
// axes as interp3(z) of interp2(y) of interp1(x), so the separable passes
// x -> y -> z reproduce its arithmetic exactly.

// vertex-centred Lagrange, prolongate_3d_rf2.cc:151-295
template <int ORDER> struct VC {
  static constexpr int N = ORDER + 1;
  static constexpr int LO = -(N / 2) + 1; // coeffs1d::imin
  static constexpr int HI = LO + N - 1;
  // x pass (interp1, :157-259, scalar Vectors order): vres = c0*p0;
  // vres = madd(c_m, p_m, vres); res = 0 + vres.  p points at coarse c.
  template <int FMA, class G> __device__ __forceinline__ static double first(int par, G get) {
    if (!par) return get(0); // interp0: no arithmetic
    double v = mul(vc_coeff(ORDER, 0), get(LO));
#pragma unroll
    for (int m = 1; m < N; ++m) v = madd<FMA>(vc_coeff(ORDER, m), get(LO + m), v);
    return add(0.0, v);
  }
  // y and z passes (interp2/interp3, :262-295): res = 0; res += c_m*v_m
  template <int FMA, class G> __device__ __forceinline__ static double next(int par, G get) {
    if (!par) return get(0);
    double r = 0.0;
#pragma unroll
    for (int m = 0; m < N; ++m) r = madd<FMA>(vc_coeff(ORDER, m), get(LO + m), r);
    return r;
  }
};

// cell-centred Lagrange, prolongate_3d_cc_rf2.cc:150-195: every axis is
// interpolated, res = 0; res += c_m*v_m, with a parity-dependent window
template <int ORDER> struct CC {
  static constexpr int N = ORDER + 1;
  static constexpr int LO0 = -N / 2;
  static constexpr int LO1 = -N / 2 + (ORDER % 2 != 0 ? 1 : 0);
  static constexpr int LO = LO0;
  static constexpr int HI = LO1 + N - 1;
  template <int FMA, class G> __device__ __forceinline__ static double next(int par, G get) {
    double r = 0.0;
    if (!par) {
#pragma unroll
      for (int m = 0; m < N; ++m) r = madd<FMA>(cc_coeff(ORDER, 0, m), get(LO0 + m), r);
    } else {
#pragma unroll
      for (int m = 0; m < N; ++m) r = madd<FMA>(cc_coeff(ORDER, 1, m), get(LO1 + m), r);
    }
    return r;
  }
  template <int FMA, class G> __device__ __forceinline__ static double first(int par, G get) {
    return next<FMA>(par, get);
  }
};

// vertex-centred ENO, prolongate_3d_real8_eno.F90:23-76 (eno1d) and the
// x -> y -> z nesting of :195-285
struct ENO {
  static constexpr int LO = -1, HI = 2;
  template <int FMA>
  __device__ __forceinline__ static double eno1d(double q1, double q2, double q3, double q4) {
    double dl = __dsub_rn(__dadd_rn(q1, q3), __dmul_rn(2.0, q2));
    double dr = __dsub_rn(__dadd_rn(q2, q4), __dmul_rn(2.0, q3));
    double r;
    if (fabs(dl) < fabs(dr)) {
      // eighth * (-q(1) + six * q(2) + three * q(3))
      double t = FMA ? __fma_rn(6.0, q2, -q1) : __dadd_rn(-q1, __dmul_rn(6.0, q2));
      t = madd<FMA>(3.0, q3, t);
      r = __dmul_rn(0.125, t);
    } else {
      // eighth * (three * q(2) + six * q(3) - q(4))
      double t = madd<FMA>(3.0, q2, __dmul_rn(6.0, q3));
      t = __dsub_rn(t, q4);
      r = __dmul_rn(0.125, t);
    }
    if (__dmul_rn(__dsub_rn(r, q2), __dsub_rn(q3, r)) < 0.0 || __dmul_rn(dl, dr) <= 0.0)
      r = __dmul_rn(0.5, __dadd_rn(q2, q3));
    return r;
  }
  template <int FMA, class G> __device__ __forceinline__ static double next(int par, G get) {
    if (!par) return get(0);
    return eno1d<FMA>(get(-1), get(0), get(1), get(2));
  }
  template <int FMA, class G> __device__ __forceinline__ static double first(int par, G get) {
    return next<FMA>(par, get);
  }
};

// ---------------------------------------------------------------- time
// interpolate_3d_2tl.cc:248-249, interpolate_3d_3tl.cc:388-390,
// interpolate_eno_3d_3tl.cc:145-162.  The fused order contracts
// s1*a + s2*b as fma(s1, a, s2*b), then + s3*c as fma(s3, c, .).
template <int FMA> __device__ __forceinline__ double tcomb2(double s1, double a, double s2, double b) {
  if (FMA) return __fma_rn(s1, a, __dmul_rn(s2, b));
  return __dadd_rn(__dmul_rn(s1, a), __dmul_rn(s2, b));
}
template <int FMA, int TK, int NTL>
__device__ __forceinline__ double tcombine(const double *w, const double *v) {
  if (NTL == 1) return v[0];
  if (TK == T_LIN) return tcomb2<FMA>(w[0], v[0], w[1], v[1]);
  double d = madd<FMA>(w[2], v[2], tcomb2<FMA>(w[0], v[0], w[1], v[1]));
  if (TK == T_ENO) {
    double a = v[0], b = v[1], c = v[2];
    double mx = b < c ? c : b; mx = a < mx ? mx : a; // std::max nesting
    double mn = c < b ? c : b; mn = mn < a ? mn : a; // std::min nesting
    if (d > mx || d < mn)
      d = w[7] != 0.0 ? tcomb2<FMA>(w[3], a, w[4], b) : tcomb2<FMA>(w[5], b, w[6], c);
  }
  return d;
}

// ---------------------------------------------------------------- cp.async
__device__ __forceinline__ void cp_async8(double *smem, const double *gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ---------------------------------------------------------------- copy-like
// copy_3d (copy_3d.cc:113-121) with optional time interpolation of the
// copied timelevels (transfer_time with equal strides, data.cc:506-517),
// restrict_3d_rf2 (restrict_3d_rf2.cc:102-108) and restrict_3d_cc_rf2
// (restrict_3d_cc_rf2.cc:246-262).  soff is the source index of the region
// start; the restrictions step by 2 in the source.
template <int FMA, int NTL, int TK>
__device__ void copy_tile(const Desc &d, int tile) {
  int tx = tile % d.tiles[0], r = tile / d.tiles[0];
  int ty = r % d.tiles[1], tz = r / d.tiles[1];
  int i = tx * CTX + (threadIdx.x & 31);
  int j = ty * CTY + (threadIdx.x >> 5);
  if (i >= d.n[0] || j >= d.n[1]) return;
  int k0 = tz * CTZ, k1 = min(k0 + CTZ, d.n[2]);
  for (int k = k0; k < k1; ++k) {
    long long si = (d.soff[0] + i) + (d.soff[1] + j) * d.ssy + (d.soff[2] + k) * d.ssz;
    double v[NTL];
#pragma unroll
    for (int t = 0; t < NTL; ++t) v[t] = __ldg(d.src[t] + si);
    d.dst[(d.doff[0] + i) + (d.doff[1] + j) * d.dsy + (d.doff[2] + k) * d.dsz] =
        tcombine<FMA, TK, NTL>(d.w, v);
  }
}

__device__ void restrict_vc_tile(const Desc &d, int tile) {
  int tx = tile % d.tiles[0], r = tile / d.tiles[0];
  int ty = r % d.tiles[1], tz = r / d.tiles[1];
  int i = tx * CTX + (threadIdx.x & 31);
  int j = ty * CTY + (threadIdx.x >> 5);
  if (i >= d.n[0] || j >= d.n[1]) return;
  int k0 = tz * CTZ, k1 = min(k0 + CTZ, d.n[2]);
  const double *s = d.src[0];
  for (int k = k0; k < k1; ++k)
    d.dst[(d.doff[0] + i) + (d.doff[1] + j) * d.dsy + (d.doff[2] + k) * d.dsz] =
        __ldg(s + (d.soff[0] + 2 * i) + (d.soff[1] + 2 * j) * d.ssy + (d.soff[2] + 2 * k) * d.ssz);
}

template <int FMA>
__device__ void restrict_cc_tile(const Desc &d, int tile) {
  int tx = tile % d.tiles[0], r = tile / d.tiles[0];
  int ty = r % d.tiles[1], tz = r / d.tiles[1];
  int i = tx * CTX + (threadIdx.x & 31);
  int j = ty * CTY + (threadIdx.x >> 5);
  if (i >= d.n[0] || j >= d.n[1]) return;
  int k0 = tz * CTZ, k1 = min(k0 + CTZ, d.n[2]);
  const double *s = d.src[0];
  const double w = 0.125; // f1*f1*f1 with f1 = f2 = 1/2
  for (int k = k0; k < k1; ++k) {
    const double *p = s + (d.soff[0] + 2 * i) + (d.soff[1] + 2 * j) * d.ssy + (d.soff[2] + 2 * k) * d.ssz;
    // order of restrict_3d_cc_rf2.cc:253-260
    double res = mul(w, __ldg(p));
    res = madd<FMA>(w, __ldg(p + 1), res);
    res = madd<FMA>(w, __ldg(p + d.ssy), res);
    res = madd<FMA>(w, __ldg(p + 1 + d.ssy), res);
    res = madd<FMA>(w, __ldg(p + d.ssz), res);
    res = madd<FMA>(w, __ldg(p + 1 + d.ssz), res);
    res = madd<FMA>(w, __ldg(p + d.ssy + d.ssz), res);
    res = madd<FMA>(w, __ldg(p + 1 + d.ssy + d.ssz), res);
    d.dst[(d.doff[0] + i) + (d.doff[1] + j) * d.dsy + (d.doff[2] + k) * d.dsz] = res;
  }
}

// ---------------------------------------------------------------- prolongation
// Shared-memory plan per CTA (doubles):
//   coarse planes  NB x NTL x CY x CXP   (ring buffer filled by cp.async)
//   x-pass rows    NTL x CY x PTX
template <class F> struct PGeom {
  static constexpr int W = F::HI - F::LO;         // window width - 1
  static constexpr int CX = PTX / 2 + 1 + W;      // coarse x per plane
  static constexpr int CXP = CX + (CX % 2 == 0);  // odd row pitch: fewer bank conflicts
  static constexpr int CY = PTY / 2 + 1 + W;      // coarse y per plane
  static constexpr int Q = W + 1;                 // z window (register queue)
  static constexpr int PD = 2;                    // prefetch distance (planes)
  static constexpr int NB = PD + 1;               // ring buffer depth
  static constexpr int XR = PTX + 1;              // x-pass row pitch
};
template <class F, int NTL> struct PSmem {
  using G = PGeom<F>;
  static constexpr int plane = G::CY * G::CXP;
  static constexpr int coarse = G::NB * NTL * plane;
  static constexpr int xrows = NTL * G::CY * G::XR;
  static constexpr int total = coarse + xrows; // doubles
};

template <class F, int FMA, int NTL, int TK>
__device__ void prolong_tile(const Desc &d, int tile, double *sm) {
  using G = PGeom<F>;
  using S = PSmem<F, NTL>;
  constexpr int LO = F::LO, HI = F::HI, Q = G::Q;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  int tx = tile % d.tiles[0], rr = tile / d.tiles[0];
  int ty = rr % d.tiles[1], tz = rr / d.tiles[1];
  const int fx0 = tx * PTX, fy0 = ty * PTY, fz0 = tz * PTZ;
  const int nfx = min(PTX, d.n[0] - fx0), nfy = min(PTY, d.n[1] - fy0), nfz = min(PTZ, d.n[2] - fz0);
  // source positions (fine units) of the tile's first points
  const int sx0 = d.soff[0] + fx0, sy0 = d.soff[1] + fy0, sz0 = d.soff[2] + fz0;
  // coarse index ranges held in shared memory
  const int cx0 = (sx0 >> 1) + LO, cx1 = ((sx0 + nfx - 1) >> 1) + HI;
  const int cy0 = (sy0 >> 1) + LO, cy1 = ((sy0 + nfy - 1) >> 1) + HI;
  const int cz0 = (sz0 >> 1) + LO, cz1 = ((sz0 + nfz - 1) >> 1) + HI;
  const int ncx = cx1 - cx0 + 1, ncy = cy1 - cy0 + 1;

  double *coarse = sm;
  double *xrow = sm + S::coarse;

  // --- stage one coarse plane of every timelevel (clamped to the array)
  auto stage = [&](int cz, int buf) {
    const int per = ncx * ncy;
    const bool zin = cz >= 0 && cz < d.sext[2];
    for (int e = threadIdx.x; e < per * NTL; e += NTHREADS) {
      int t = e / per, q = e - t * per;
      int yy = q / ncx, xx = q - yy * ncx;
      int gx = cx0 + xx, gy = cy0 + yy;
      double *sp = coarse + ((buf * NTL + t) * G::CY + yy) * G::CXP + xx;
      if (zin && gx >= 0 && gx < d.sext[0] && gy >= 0 && gy < d.sext[1])
        cp_async8(sp, d.src[t] + gx + gy * d.ssy + (long long)cz * d.ssz);
      else
        *sp = 0.0; // never read by a valid output (host checks the stencils)
    }
  };

  // --- y pass owner: lane <-> fine x, warp <-> coarse y row
  const int my_fx = lane;                 // tile-relative fine x
  const int my_cy = (sy0 >> 1) + warp;    // coarse y of this thread
  // the thread's fine y points: source positions 2*my_cy and 2*my_cy+1
  const int ys0 = 2 * my_cy, ys1 = 2 * my_cy + 1;
  const bool v0 = ys0 >= sy0 && ys0 < sy0 + nfy && my_fx < nfx;
  const bool v1 = ys1 >= sy0 && ys1 < sy0 + nfy && my_fx < nfx;

  double yq[NTL][2][Q]; // z window of y-pass results
#pragma unroll
  for (int t = 0; t < NTL; ++t)
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int q = 0; q < Q; ++q) yq[t][h][q] = 0.0;

  // prologue: planes cz0 .. cz0+PD-1
#pragma unroll
  for (int p = 0; p < G::PD; ++p) {
    if (cz0 + p <= cz1) stage(cz0 + p, p % G::NB);
    cp_async_commit();
  }

  const int nplanes = cz1 - cz0 + 1;
  for (int pi = 0; pi < nplanes; ++pi) {
    const int cz = cz0 + pi;
    if (cz + G::PD <= cz1) stage(cz + G::PD, (pi + G::PD) % G::NB);
    cp_async_commit();
    cp_async_wait<G::PD>();
    __syncthreads(); // plane cz visible; previous y pass done with xrow
    const int buf = pi % G::NB;

    // --- x pass: rows (t, yy) of the plane, one fine x per lane-slot
    {
      const int items = NTL * ncy * PTX;
      for (int e = threadIdx.x; e < items; e += NTHREADS) {
        int fx = e & (PTX - 1), ty_ = e / PTX;
        int t = ty_ / ncy, yy = ty_ - t * ncy;
        if (fx < nfx) {
          int s = sx0 + fx;
          const double *row = coarse + ((buf * NTL + t) * G::CY + yy) * G::CXP + ((s >> 1) - cx0);
          xrow[(t * G::CY + yy) * G::XR + fx] =
              F::template first<FMA>(s & 1, [&](int m) { return row[m]; });
        }
      }
    }
    __syncthreads();

    // --- y pass into the z window
    {
      const int yrow = my_cy - cy0; // index of coarse row my_cy in the plane
#pragma unroll
      for (int t = 0; t < NTL; ++t) {
#pragma unroll
        for (int q = 0; q < Q - 1; ++q) {
          yq[t][0][q] = yq[t][0][q + 1];
          yq[t][1][q] = yq[t][1][q + 1];
        }
        if (v0 || v1) {
          const double *col = xrow + (t * G::CY + yrow) * G::XR + my_fx;
          auto get = [&](int m) { return col[m * G::XR]; };
          yq[t][0][Q - 1] = v0 ? F::template next<FMA>(0, get) : 0.0;
          yq[t][1][Q - 1] = v1 ? F::template next<FMA>(1, get) : 0.0;
        }
      }
    }

    // --- z pass: the window now holds coarse planes cz-Q+1 .. cz, i.e.
    // cb+LO .. cb+HI for the coarse base cb = cz - HI
    const int cb = cz - HI;
#pragma unroll
    for (int zp = 0; zp < 2; ++zp) {
      const int zs = 2 * cb + zp;
      if (zs < sz0 || zs >= sz0 + nfz) continue;
      const long long zoff = (long long)(d.doff[2] + fz0 + (zs - sz0)) * d.dsz;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (!(h ? v1 : v0)) continue;
        double v[NTL];
#pragma unroll
        for (int t = 0; t < NTL; ++t)
          v[t] = F::template next<FMA>(zp, [&](int m) { return yq[t][h][m - LO]; });
        const int fy = (h ? ys1 : ys0) - sy0;
        d.dst[(d.doff[0] + fx0 + my_fx) + (long long)(d.doff[1] + fy0 + fy) * d.dsy + zoff] =
            tcombine<FMA, TK, NTL>(d.w, v);
      }
    }
  }
  cp_async_wait<0>();
  __syncthreads(); // shared memory free for the next tile
}

} // namespace cgx
