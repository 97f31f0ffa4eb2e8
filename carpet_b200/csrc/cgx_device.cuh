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
#include <type_traits>
#include <utility>

namespace cgx {

enum Kind : int {
  K_COPY = 0,        // copy_3d (+ time interpolation when ntl > 1)
  K_RESTRICT_VC = 1, // restrict_3d_rf2 (injection)
  K_RESTRICT_CC = 2, // restrict_3d_cc_rf2 (8-point average)
  K_PROLONG_VC = 3,  // prolongate_3d_rf2<ORDER>
  K_PROLONG_CC = 4,  // prolongate_3d_cc_rf2<ORDER>
  K_PROLONG_ENO = 5, // prolongate_3d_real8_eno
  K_RESTRICT_CC3 = 6, // restrict_3d_cc_o3_rf2 (4x4x4 cells)
  K_RESTRICT_CC5 = 7, // restrict_3d_cc_o5_rf2 (6x6x6 cells, separable)
  K_PROLONG_CC_ENO = 8, // prolongate_3d_cc_eno_rf2<ORDER>, ORDER (d.order) 2 or 3
  K_TIME = 9,           // time_interpolate of per-timelevel temporaries
  K_PROLONG_MONO = 10,  // prolongate_3d_o5_monotone_rf2
  K_NKINDS = 11
};

// T_LAG: interpolate_3d_4tl / interpolate_3d_5tl (ntl 4 or 5)
enum TKind : int { T_NONE = 0, T_LIN = 1, T_QUAD = 2, T_ENO = 3, T_LAG = 4 };

// Tile geometry.
constexpr int NTHREADS = 256;
constexpr int NWARPS = NTHREADS / 32;
// prolongation: a tile is ptx fine x (at most PTXMAX, so at most 9 coarse
// bases) by 2*ptyc-1 fine y (at most ptyc coarse rows) by a PTZ chunk of fine
// z that the CTA marches plane by plane.  ptx and ptyc are chosen per
// descriptor, balanced over the region; ptx*ptyc <= NTHREADS, one thread per
// (fine x, coarse y row) column.
constexpr int PTXMAX = 16, PTYCMAX = 16, PTZ = 64;

struct Desc {
  int kind, order, ntl, tkind;
  int n[3];     // destination region extent (points)
  int soff[3];  // source offset of the region start (meaning per kind)
  int doff[3];  // destination index of the region start
  int sext[3];  // logical extent of the source arrays (load clamp)
  int tiles[3]; // tile grid over the region
  unsigned char ptx, ptyc; // prolongation tile shape (fine x, coarse y rows)
  unsigned char bx, by;    // tensor-copy box of a tile's coarse plane; bx = 0: not staged by TMA
  long long ssy, ssz; // source strides (elements) in y and z
  long long dsy, dsz; // destination strides
  unsigned mg[2]; // streaming kinds: division magic for n[0], n[1] (div_magic)
  int sh[2];
  const double *src[3];
  double *dst;
  double w[8]; // time weights (layout of the oracle's cgxo_time_weights)
};

// compile-time loop: f(std::integral_constant<int, 0>()) ... f(<N-1>)
template <class Fn, int... I>
__device__ __forceinline__ void static_for_impl(Fn &&f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>()), ...);
}
template <int N, class Fn> __device__ __forceinline__ void static_for(Fn &&f) {
  static_for_impl(f, std::make_integer_sequence<int, N>());
}

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

// cell-centred ENO, prolongate_3d_cc_eno_rf2.cc:198-400 (interp1, interp2
// and interp3 apply the same rule on their axis).  Relative to the coarse
// base c, the fine point of parity DI reads f(-W+DI) .. f(W-1+DI), W = ORDER.
// coeffs1dc<RT,ORDER,OFFSET> (:144-176) as exact dyadic rationals; table t:
// 0 <1,0>, 1 <2,0>, 2 <2,-1>, 3 <3,0>, 4 <3,+1>, 5 <3,-1>.
__device__ __forceinline__ constexpr double ceno_coeff(int t, int j) {
  return t == 0 ? (j == 0 ? 1.0 : 3.0) / 4
       : t == 1 ? (j == 0 ? 5.0 : j == 1 ? 30.0 : -3.0) / 32
       : t == 2 ? (j == 0 ? -3.0 : j == 1 ? 14.0 : 21.0) / 32
       : t == 3 ? (j == 0 ? -5.0 : j == 1 ? 35.0 : j == 2 ? 105.0 : -7.0) / 128
       : t == 4 ? (j == 0 ? 15.0 : j == 1 ? 135.0 : j == 2 ? -27.0 : 5.0) / 128
                : (j == 0 ? 7.0 : j == 1 ? -33.0 : 77.0) / 128;
}
template <int ORDER> struct CCENO {
  static_assert(ORDER == 2 || ORDER == 3, "cell-centred ENO orders 2 and 3");
  static constexpr int LO = -ORDER, HI = ORDER;
  // coeffs1d::get summed from imin: res = 0; res += c*f (reversed for DI=1)
  template <int FMA, int DI, int T, int N, int IMIN, class G>
  __device__ __forceinline__ static double sum(G get) {
    double r = 0.0;
    static_for<N>([&](auto M) {
      constexpr int m = decltype(M)::value;
      r = madd<FMA>(ceno_coeff(T, DI == 0 ? m : N - 1 - m), get(IMIN + m), r);
    });
    return r;
  }
  // undivided differences (diffC1dc, :171-174; never reversed)
  template <int FMA, int IMIN, class G> __device__ __forceinline__ static double diff(G get) {
    double r = 0.0;
    static_for<ORDER + 1>([&](auto M) {
      constexpr int m = decltype(M)::value;
      constexpr double c = ORDER == 2 ? (m == 1 ? -2.0 : 1.0)
                                      : (m == 0 ? 1.0 : m == 1 ? -3.0 : m == 2 ? 3.0 : -1.0);
      r = madd<FMA>(c, get(IMIN + m), r);
    });
    return r;
  }
  template <int FMA, int DI, class G> __device__ __forceinline__ static double rule(G get) {
    const double first = sum<FMA, DI, 0, 2, -1 + DI>(get); // coeffs1d<RT,1,di,0>
    double res;
    if (ORDER == 2) {
      constexpr int SH = DI == 0 ? -1 : 1; // :225-231
      const double lV = diff<FMA, -1 + SH>(get), rV = diff<FMA, -1>(get);
      if (__dmul_rn(lV, rV) <= 0.0) res = first;
      else if (fabs(lV) < fabs(rV)) res = sum<FMA, DI, 2, 3, -1 + SH>(get);
      else res = sum<FMA, DI, 1, 3, -1>(get);
    } else {
      const double V0 = diff<FMA, -3 + DI>(get), V1 = diff<FMA, -2 + DI>(get),
                   V2 = diff<FMA, -1 + DI>(get);
      if (__dmul_rn(V0, V2) <= 0.0 || __dmul_rn(V0, V1) <= 0.0 || __dmul_rn(V1, V2) <= 0.0)
        return first; // :311-329, without the final test
      int mn = 1;
      if (fabs(V0) < fabs(V1)) mn = 0;
      if (fabs(V2) < fabs(mn == 0 ? V0 : V1)) mn = 2;
      // coeffs1dc<3, di == 0 ? OFFSET : -OFFSET> for OFFSET -1, 0, +1
      if (mn == 0) res = sum<FMA, DI, DI == 0 ? 5 : 4, 4, -3 + DI>(get);
      else if (mn == 1) res = sum<FMA, DI, 3, 4, -2 + DI>(get);
      else res = sum<FMA, DI, DI == 0 ? 4 : 5, 4, -1 + DI>(get);
    }
    // :366-395: a result outside the two nearest values falls back
    if (__dmul_rn(__dsub_rn(res, get(DI - 1)), __dsub_rn(get(DI), res)) < 0.0) res = first;
    return res;
  }
  template <int FMA, class G> __device__ __forceinline__ static double next(int par, G get) {
    return par ? rule<FMA, 1>(get) : rule<FMA, 0>(get);
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
//
// These are pure streaming operations on regions of any shape -- ghost
// zones are 3 points thin in one direction.  A tile is STILE consecutive
// points of the region flattened x-fastest, run by the LANES threads of a
// CTA: every lane is busy whatever the shape, consecutive lanes touch
// consecutive x, and each thread issues a group of loads before its stores.  A flat index is split into (i, j, k) by
// 32-bit multiply-high with precomputed magic numbers.
constexpr int STILE = 1024;

// The streaming kinds, one persistent kernel each.
enum StreamVariant : int {
  SV_COPY1 = 0,       // copy, one timelevel
  SV_COPY2 = 1,       // copy, linear time interpolation
  SV_COPY3Q = 2,      // copy, quadratic time interpolation
  SV_COPY3E = 3,      // copy, ENO time interpolation
  SV_RESTRICT_VC = 4, // injection
  SV_RESTRICT_CC = 5, // 8-point average
  SV_RESTRICT_CC3 = 6, // third-order cell-centred restriction
  SV_RESTRICT_CC5 = 7, // fifth-order cell-centred restriction
  SV_MONO = 8,         // monotone order-5 prolongation
  SV_TIME = 9,         // time combination of temporaries (K_TIME)
  SV_COUNT = 10
};
// A batch launches its segments in order: the time combination of staged
// transfers must come after every kind that writes their temporaries.
static_assert(SV_TIME == SV_COUNT - 1, "the time combination is the last streaming variant");

template <class D> __host__ __device__ __forceinline__ int stream_variant(const D &d) {
  if (d.kind == K_RESTRICT_VC) return SV_RESTRICT_VC;
  if (d.kind == K_RESTRICT_CC) return SV_RESTRICT_CC;
  if (d.kind == K_RESTRICT_CC3) return SV_RESTRICT_CC3;
  if (d.kind == K_RESTRICT_CC5) return SV_RESTRICT_CC5;
  if (d.kind == K_TIME) return SV_TIME;
  if (d.kind == K_PROLONG_MONO) return SV_MONO;
  if (d.kind != K_COPY) return -1;
  if (d.ntl == 1) return SV_COPY1;
  if (d.ntl == 2) return SV_COPY2;
  return d.tkind == T_ENO ? SV_COPY3E : SV_COPY3Q;
}

// Source loads of the streaming tiles: through the read-only path (__ldg)
// in kernels whose sources no CTA of the same launch writes; cached in L2
// only (__ldcg, coherent across SMs) in the chain kernel, whose later tiles
// read what earlier tiles of the same launch wrote.
template <bool CG> __device__ __forceinline__ double ld_src(const double *p) {
  if (CG) return __ldcg(p);
  return __ldg(p);
}

// floor(p / n) for 0 <= p < 2^31 (Granlund & Montgomery, "Division by
// invariant integers using multiplication", 1994, theorem 4.2 with N = 31):
// with l = ceil(log2 n), m = ceil(2^(31+l) / n) < 2^32 and s = l - 1,
// floor(p / n) = umulhi(p, m) >> s; m = 0 encodes n = 1.
__device__ __forceinline__ unsigned div_magic(unsigned p, unsigned m, int s) {
  return m ? (__umulhi(p, m) >> s) : p;
}

template <class D>
__device__ __forceinline__ void unflatten(const D &d, unsigned p, int &i, int &j, int &k) {
  const unsigned q = div_magic(p, d.mg[0], d.sh[0]);
  i = (int)(p - q * (unsigned)d.n[0]);
  const unsigned r = div_magic(q, d.mg[1], d.sh[1]);
  j = (int)(q - r * (unsigned)d.n[1]);
  k = (int)r;
}

// group sizes: points whose loads a thread issues before it stores them
template <int LANES, int NTL> __host__ __device__ constexpr int stream_group() {
  return (STILE / LANES) < (NTL == 1 ? 8 : 4) ? (STILE / LANES) : (NTL == 1 ? 8 : 4);
}

template <int FMA, int NTL, int TK, int LANES, class D, bool CG = false, int PTS = STILE, int GMAX = 8>
__device__ __forceinline__ void copy_tile(const D &d, int tile, int lid) {
  // ENO time interpolation holds more per point: smaller groups
  constexpr int PER = PTS / LANES;
  constexpr int G0 = PER < (NTL == 1 ? GMAX : 4) ? PER : (NTL == 1 ? GMAX : 4);
  constexpr int G = G0 / (TK == T_ENO ? 2 : 1);
  const unsigned npts = (unsigned)d.n[0] * d.n[1] * d.n[2];
  const unsigned p0 = (unsigned)tile * PTS + lid;
  const double *src[NTL];
#pragma unroll
  for (int t = 0; t < NTL; ++t) src[t] = d.src[t] + (d.soff[0] + d.soff[1] * d.ssy + d.soff[2] * d.ssz);
  double *dst = d.dst + (d.doff[0] + d.doff[1] * d.dsy + d.doff[2] * d.dsz);
  double w[NTL == 1 ? 1 : 8];
#pragma unroll
  for (int k = 0; k < (NTL == 1 ? 1 : 8); ++k) w[k] = NTL == 1 ? 0.0 : d.w[k];
#pragma unroll
  for (int r0 = 0; r0 < PER; r0 += G) {
    double v[G][NTL];
#pragma unroll
    for (int r = 0; r < G; ++r) {
      const unsigned p = p0 + (r0 + r) * LANES;
      if (p < npts) {
        int i, j, k;
        unflatten(d, p, i, j, k);
        const long long si = i + j * d.ssy + k * d.ssz;
#pragma unroll
        for (int t = 0; t < NTL; ++t) v[r][t] = ld_src<CG>(src[t] + si);
      }
    }
    // the destination index is recomputed rather than held across the loads
#pragma unroll
    for (int r = 0; r < G; ++r) {
      const unsigned p = p0 + (r0 + r) * LANES;
      if (p < npts) {
        int i, j, k;
        unflatten(d, p, i, j, k);
        dst[i + j * d.dsy + k * d.dsz] = tcombine<FMA, TK, NTL>(w, v[r]);
      }
    }
  }
}

template <int LANES, class D, bool CG = false, int PTS = STILE, int GMAX = 8>
__device__ __forceinline__ void restrict_vc_tile(const D &d, int tile, int lid) {
  constexpr int PER = PTS / LANES, G = PER < GMAX ? PER : GMAX;
  const unsigned npts = (unsigned)d.n[0] * d.n[1] * d.n[2];
  const unsigned p0 = (unsigned)tile * PTS + lid;
  const double *s = d.src[0] + (d.soff[0] + d.soff[1] * d.ssy + d.soff[2] * d.ssz);
  double *dst = d.dst + (d.doff[0] + d.doff[1] * d.dsy + d.doff[2] * d.dsz);
#pragma unroll
  for (int r0 = 0; r0 < PER; r0 += G) {
    double v[G];
#pragma unroll
    for (int r = 0; r < G; ++r) {
      const unsigned p = p0 + (r0 + r) * LANES;
      if (p < npts) {
        int i, j, k;
        unflatten(d, p, i, j, k);
        v[r] = ld_src<CG>(s + 2 * (i + j * d.ssy + k * d.ssz));
      }
    }
#pragma unroll
    for (int r = 0; r < G; ++r) {
      const unsigned p = p0 + (r0 + r) * LANES;
      if (p < npts) {
        int i, j, k;
        unflatten(d, p, i, j, k);
        dst[i + j * d.dsy + k * d.dsz] = v[r];
      }
    }
  }
}

template <int FMA, int LANES, class D>
__device__ __forceinline__ void restrict_cc_tile(const D &d, int tile, int lid) {
  constexpr int PER = STILE / LANES;
  const unsigned npts = (unsigned)d.n[0] * d.n[1] * d.n[2];
  const unsigned p0 = (unsigned)tile * STILE + lid;
  const double *s0 = d.src[0] + (d.soff[0] + d.soff[1] * d.ssy + d.soff[2] * d.ssz);
  double *dst = d.dst + (d.doff[0] + d.doff[1] * d.dsy + d.doff[2] * d.dsz);
  const long long ssy = d.ssy, ssz = d.ssz;
  const double w = 0.125; // f1*f1*f1 with f1 = f2 = 1/2
#pragma unroll 2
  for (int r = 0; r < PER; ++r) {
    const unsigned p = p0 + r * LANES;
    if (p >= npts) break;
    int i, j, k;
    unflatten(d, p, i, j, k);
    const double *q = s0 + 2 * (i + j * ssy + k * ssz);
    const double a0 = __ldg(q), a1 = __ldg(q + 1), a2 = __ldg(q + ssy), a3 = __ldg(q + 1 + ssy);
    const double a4 = __ldg(q + ssz), a5 = __ldg(q + 1 + ssz);
    const double a6 = __ldg(q + ssy + ssz), a7 = __ldg(q + 1 + ssy + ssz);
    // order of restrict_3d_cc_rf2.cc:253-260
    double res = mul(w, a0);
    res = madd<FMA>(w, a1, res);
    res = madd<FMA>(w, a2, res);
    res = madd<FMA>(w, a3, res);
    res = madd<FMA>(w, a4, res);
    res = madd<FMA>(w, a5, res);
    res = madd<FMA>(w, a6, res);
    res = madd<FMA>(w, a7, res);
    dst[i + j * d.dsy + k * d.dsz] = res;
  }
}

// The second stage of transfer_time (data.cc:506-517) where the fused
// kernels do not apply: d.src[0] holds d.ntl temporaries of the region's
// shape, one after another, x fastest and unpadded; time_interpolate
// (data.cc:1183-1299) combines them into the destination.  4 and 5
// timelevels sum s1*a + s2*b + s3*c + s4*d (+ s5*e) left to right
// (interpolate_3d_4tl.cc:126-131, interpolate_3d_5tl.cc:128-132).
template <int FMA, int LANES, class D>
__device__ __forceinline__ void time_tile(const D &d, int tile, int lid) {
  constexpr int PER = STILE / LANES;
  const unsigned npts = (unsigned)d.n[0] * d.n[1] * d.n[2];
  const unsigned p0 = (unsigned)tile * STILE + lid;
  const double *tmp = d.src[0];
  double *dst = d.dst + (d.doff[0] + d.doff[1] * d.dsy + d.doff[2] * d.dsz);
  const int ntl = d.ntl, tk = d.tkind;
  double w[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) w[k] = d.w[k];
#pragma unroll 2
  for (int r = 0; r < PER; ++r) {
    const unsigned p = p0 + r * LANES;
    if (p >= npts) break;
    double v[5];
#pragma unroll
    for (int t = 0; t < 5; ++t) v[t] = t < ntl ? __ldg(tmp + (size_t)t * npts + p) : 0.0;
    double res;
    if (ntl == 2) res = tcombine<FMA, T_LIN, 2>(w, v);
    else if (ntl == 3 && tk == T_ENO) res = tcombine<FMA, T_ENO, 3>(w, v);
    else {
      res = tcombine<FMA, T_QUAD, 3>(w, v);
      if (ntl >= 4) res = madd<FMA>(w[3], v[3], res);
      if (ntl == 5) res = madd<FMA>(w[4], v[4], res);
    }
    int i, j, k;
    unflatten(d, p, i, j, k);
    dst[i + j * d.dsy + k * d.dsz] = res;
  }
}

// prolongate_3d_o5_monotone_rf2 (prolongate_3d_o5_monotone_rf2.cc:45-793),
// one fine point per lane.  q points at the coarse base; odd axes take the
// tensor-product order-5 stencil over coarse -2 .. +3, summed left to right
// with the lowest odd axis fastest (weights f_a * f_b * f_c formed left to
// right); with three odd axes every z plane is a partial sum of its own and
// the six are added in order (:499-716).  A result outside the nearest 2/4/8
// coarse values (std::min/std::max nested as min4/max4/min8/max8, :19-43)
// falls back to linear, bilinear or trilinear interpolation.
__device__ __forceinline__ double smin(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double smax(double a, double b) { return a < b ? b : a; }
__device__ __forceinline__ constexpr double mono_f(int m) {
  return (m == 0 || m == 5 ? 3.0 : m == 1 || m == 4 ? -25.0 : 150.0) / 256;
}
template <int FMA>
__device__ __forceinline__ double mono_point(const double *q, int ox, int oy, int oz, long long sy,
                                             long long sz) {
  const int n = ox + oy + oz;
  if (n == 0) return __ldg(q);
  if (n == 1) {
    const long long s = ox ? 1 : oy ? sy : sz;
    double res = mul(mono_f(0), __ldg(q - 2 * s));
#pragma unroll
    for (int m = 1; m < 6; ++m) res = madd<FMA>(mono_f(m), __ldg(q + (m - 2) * s), res);
    const double v0 = __ldg(q), v1 = __ldg(q + s);
    if (res > smax(v0, v1) || res < smin(v0, v1)) res = madd<FMA>(0.5, v1, mul(0.5, v0));
    return res;
  }
  if (n == 2) {
    const long long s0 = ox ? 1 : sy, s1 = oz ? sz : sy;
    double res = 0.0;
#pragma unroll
    for (int b = 0; b < 6; ++b) {
      const double *row = q + (b - 2) * s1 - 2 * s0;
#pragma unroll
      for (int a = 0; a < 6; ++a) {
        const double w = mono_f(a) * mono_f(b);
        const double v = __ldg(row + a * s0);
        res = (a == 0 && b == 0) ? mul(w, v) : madd<FMA>(w, v, res);
      }
    }
    const double x1 = __ldg(q), x2 = __ldg(q + s0), x3 = __ldg(q + s1), x4 = __ldg(q + s0 + s1);
    if (res > smax(smax(x1, x2), smax(x3, x4)) || res < smin(smin(x1, x2), smin(x3, x4))) {
      res = mul(0.25, x1);
      res = madd<FMA>(0.25, x2, res);
      res = madd<FMA>(0.25, x3, res);
      res = madd<FMA>(0.25, x4, res);
    }
    return res;
  }
  double res = 0.0;
#pragma unroll 1
  for (int c = 0; c < 6; ++c) {
    const double fc = (c == 0 || c == 5) ? mono_f(0) : (c == 1 || c == 4) ? mono_f(1) : mono_f(2);
    const double *pl = q + (c - 2) * sz;
    double r = 0.0;
#pragma unroll
    for (int b = 0; b < 6; ++b) {
      const double *row = pl + (b - 2) * sy - 2;
#pragma unroll
      for (int a = 0; a < 6; ++a) {
        const double w = __dmul_rn(mono_f(a) * mono_f(b), fc);
        const double v = __ldg(row + a);
        r = (a == 0 && b == 0) ? mul(w, v) : madd<FMA>(w, v, r);
      }
    }
    res = c == 0 ? r : add(res, r);
  }
  // max8 / min8 of (0,0,0), (1,0,0), (0,1,0), (0,0,1), (1,1,0), (1,0,1), (0,1,1), (1,1,1)
  const double x0 = __ldg(q), x1 = __ldg(q + 1), x2 = __ldg(q + sy), x3 = __ldg(q + sz);
  const double x4 = __ldg(q + 1 + sy), x5 = __ldg(q + 1 + sz), x6 = __ldg(q + sy + sz);
  const double x7 = __ldg(q + 1 + sy + sz);
  const double mx = smax(smax(smax(x0, x1), smax(x2, x3)), smax(smax(x4, x5), smax(x6, x7)));
  const double mn = smin(smin(smin(x0, x1), smin(x2, x3)), smin(smin(x4, x5), smin(x6, x7)));
  if (res > mx || res < mn) {
    // :730-738: the z = 0 plane, then the z = 1 plane, x fastest
    double r1 = mul(0.125, x0);
    r1 = madd<FMA>(0.125, x1, r1);
    r1 = madd<FMA>(0.125, x2, r1);
    r1 = madd<FMA>(0.125, x4, r1);
    double r2 = mul(0.125, x3);
    r2 = madd<FMA>(0.125, x5, r2);
    r2 = madd<FMA>(0.125, x6, r2);
    r2 = madd<FMA>(0.125, x7, r2);
    res = add(r1, r2);
  }
  return res;
}

template <int FMA, int LANES, class D>
__device__ __forceinline__ void mono_tile(const D &d, int tile, int lid) {
  constexpr int PER = STILE / LANES;
  const unsigned npts = (unsigned)d.n[0] * d.n[1] * d.n[2];
  const unsigned p0 = (unsigned)tile * STILE + lid;
  const long long sy = d.ssy, sz = d.ssz;
  double *dst = d.dst + (d.doff[0] + d.doff[1] * d.dsy + d.doff[2] * d.dsz);
#pragma unroll 1
  for (int r = 0; r < PER; ++r) {
    const unsigned p = p0 + r * LANES;
    if (p >= npts) break;
    int i, j, k;
    unflatten(d, p, i, j, k);
    const int fx = d.soff[0] + i, fy = d.soff[1] + j, fz = d.soff[2] + k;
    const double *q = d.src[0] + ((fx >> 1) + (fy >> 1) * sy + (long long)(fz >> 1) * sz);
    dst[i + j * d.dsy + k * d.dsz] = mono_point<FMA>(q, fx & 1, fy & 1, fz & 1, sy, sz);
  }
}

// restrict_3d_cc_o3_rf2 (restrict_3d_cc_o3_rf2.cc:147-211): the 4x4x4 fine
// cells 2i-1 .. 2i+2 per axis (from the region's first cell soff), weights
// c_a c_b c_c / 4096 with c = (-1, 9, 9, -1), summed left to right, x
// fastest; the first term is a plain product.
template <int FMA, int LANES, class D>
__device__ __forceinline__ void restrict_cc3_tile(const D &d, int tile, int lid) {
  constexpr int PER = STILE / LANES;
  const unsigned npts = (unsigned)d.n[0] * d.n[1] * d.n[2];
  const unsigned p0 = (unsigned)tile * STILE + lid;
  const long long ssy = d.ssy, ssz = d.ssz;
  const double *s0 = d.src[0] + (d.soff[0] - 1 + (d.soff[1] - 1) * ssy + (d.soff[2] - 1) * ssz);
  double *dst = d.dst + (d.doff[0] + d.doff[1] * d.dsy + d.doff[2] * d.dsz);
#pragma unroll 1
  for (int r = 0; r < PER; ++r) {
    const unsigned p = p0 + r * LANES;
    if (p >= npts) break;
    int i, j, k;
    unflatten(d, p, i, j, k);
    const double *q = s0 + 2 * (i + j * ssy + k * ssz);
    double res = 0.0;
    // one plane of 16 cells per pass; every weight is an exact binary
    // fraction, so forming it from the plane's factor loses nothing
#pragma unroll 1
    for (int c = 0; c < 4; ++c) {
      const double cz = (c == 0 || c == 3) ? -1.0 : 9.0;
      const double *qz = q + c * ssz;
      static_for<16>([&](auto M) {
        constexpr int m = decltype(M)::value;
        constexpr double cx = (m & 3) == 0 || (m & 3) == 3 ? -1.0 : 9.0;
        constexpr double cy = (m >> 2) == 0 || (m >> 2) == 3 ? -1.0 : 9.0;
        const double w = cx * cy * cz / 4096.0;
        const double v = __ldg(qz + (m & 3) + (m >> 2) * ssy);
        res = (m == 0 && c == 0) ? mul(w, v) : madd<FMA>(w, v, res);
      });
    }
    dst[i + j * d.dsy + k * d.dsz] = res;
  }
}

// restrict_3d_cc_o5_rf2 (restrict_3d_cc_o5_rf2.cc:36-78): restrict3 over the
// planes 2k-2 .. 2k+3 of restrict2 over rows of restrict1 over the cells
// 2i-2 .. 2i+3, each a left-to-right sum with weights (3, -25, 150, 150,
// -25, 3) / 256, the first term a plain product.
template <int FMA, int LANES, class D>
__device__ __forceinline__ void restrict_cc5_tile(const D &d, int tile, int lid) {
  constexpr int PER = STILE / LANES;
  const unsigned npts = (unsigned)d.n[0] * d.n[1] * d.n[2];
  const unsigned p0 = (unsigned)tile * STILE + lid;
  const long long ssy = d.ssy, ssz = d.ssz;
  const double *s0 = d.src[0] + (d.soff[0] - 2 + (d.soff[1] - 2) * ssy + (d.soff[2] - 2) * ssz);
  double *dst = d.dst + (d.doff[0] + d.doff[1] * d.dsy + d.doff[2] * d.dsz);
  constexpr double w[6] = {3.0 / 256, -25.0 / 256, 150.0 / 256, 150.0 / 256, -25.0 / 256, 3.0 / 256};
#pragma unroll 1
  for (int r = 0; r < PER; ++r) {
    const unsigned p = p0 + r * LANES;
    if (p >= npts) break;
    int i, j, k;
    unflatten(d, p, i, j, k);
    const double *q = s0 + 2 * (i + j * ssy + k * ssz);
    double r3 = 0.0;
#pragma unroll 1
    for (int c = 0; c < 6; ++c) {
      double r2 = 0.0;
#pragma unroll
      for (int b = 0; b < 6; ++b) {
        const double *row = q + c * ssz + b * ssy;
        double r1 = mul(w[0], __ldg(row));
#pragma unroll
        for (int a = 1; a < 6; ++a) r1 = madd<FMA>(w[a], __ldg(row + a), r1);
        r2 = b == 0 ? mul(w[0], r1) : madd<FMA>(w[b], r1, r2);
      }
      const double wc = (c == 0 || c == 5) ? w[0] : (c == 1 || c == 4) ? w[1] : w[2];
      r3 = c == 0 ? mul(wc, r2) : madd<FMA>(wc, r2, r3);
    }
    dst[i + j * d.dsy + k * d.dsz] = r3;
  }
}

// ---------------------------------------------------------------- prolongation
// Shared-memory plan per CTA (doubles):
//   coarse planes  NB x NTL x CY x CXP   (ring buffer filled by cp.async)
//   x-pass rows    NTL x CY x PTX
template <class F> struct PGeom {
  static constexpr int W = F::HI - F::LO;         // window width - 1
  static constexpr int CX = 16 + W;               // coarse x per plane (16 bases)
  static constexpr int CXP = CX + (CX % 2 == 0);  // odd row pitch: fewer bank conflicts
  static constexpr int CY = PTYCMAX + W;          // coarse y per plane
  static constexpr int Q = W + 1;                 // z window (register queue)
  static constexpr int PD = 2;                    // prefetch distance (planes)
  static constexpr int NB = PD + 2;               // staging ring slots
  static constexpr int XR = 34;                   // x-pass row pitch (2 x 16 + 2)
};
template <class F, int NTL> struct PSmem {
  using G = PGeom<F>;
  static constexpr int plane = G::CY * G::CXP;
  static constexpr int coarse = (G::NB * NTL * plane + 1) / 2 * 2; // x-pass rows 16-B aligned
  static constexpr int xbuf = NTL * G::CY * G::XR; // one plane of x-pass rows
  static constexpr int total = coarse + 2 * xbuf;   // doubles
};

template <class F, int FMA, int NTL, int TK, class D>
__device__ void prolong_tile(D &d, int tile, double *sm) {
  using G = PGeom<F>;
  using S = PSmem<F, NTL>;
  constexpr int LO = F::LO, HI = F::HI, Q = G::Q, W = G::W;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ptx = d.ptx, ptyc = d.ptyc, pty = 2 * ptyc - 1;

  const int tx = tile % d.tiles[0], rr = tile / d.tiles[0];
  const int ty = rr % d.tiles[1], tz = rr / d.tiles[1];
  const int fx0 = tx * ptx, fy0 = ty * pty, fz0 = tz * PTZ;
  const int nfx = min(ptx, d.n[0] - fx0), nfy = min(pty, d.n[1] - fy0), nfz = min(PTZ, d.n[2] - fz0);
  // source positions (fine units) of the tile's first points
  const int sx0 = d.soff[0] + fx0, sy0 = d.soff[1] + fy0, sz0 = d.soff[2] + fz0;
  // coarse index ranges held in shared memory
  const int cx0 = (sx0 >> 1) + LO, cx1 = ((sx0 + nfx - 1) >> 1) + HI;
  const int cy0 = (sy0 >> 1) + LO, cy1 = ((sy0 + nfy - 1) >> 1) + HI;
  const int cz0 = (sz0 >> 1) + LO, cz1 = ((sz0 + nfz - 1) >> 1) + HI;
  const int ncx = cx1 - cx0 + 1, ncy = cy1 - cy0 + 1;
  const int nrows = NTL * ncy; // staged rows per plane: (timelevel, coarse y)
  const int c_first = sx0 >> 1, c_last = (sx0 + nfx - 1) >> 1;
  const int xoff = sx0 - 2 * c_first; // fine x of the tile's first point in x-pass rows

  double *coarse = sm;
  double *xrows = sm + S::coarse;

  // --- staging: warp w copies rows w, w+8, ...; lane = coarse x (< 32)
  const int gx = cx0 + lane;
  const bool xin = lane < ncx && gx >= 0 && gx < d.sext[0];
  auto stage = [&](int cz, int slot) {
    const bool zin = cz >= 0 && cz < d.sext[2];
    int t = 0, yy = warp;
    for (int r = warp; r < nrows; r += NWARPS, yy += NWARPS) {
      while (yy >= ncy) { yy -= ncy; ++t; }
      if (lane < ncx) {
        const int gy = cy0 + yy;
        double *sp = coarse + ((slot * NTL + t) * G::CY + yy) * G::CXP + lane;
        if (zin && xin && gy >= 0 && gy < d.sext[1])
          cp_async8(sp, d.src[t] + gx + gy * d.ssy + (long long)cz * d.ssz);
        else
          *sp = 0.0; // never read by a valid output (host checks the stencils)
      }
    }
  };

  // --- x pass: one coarse base per lane (both its fine points, the copy at
  // 2c and the interpolant at 2c+1), two rows per warp; x-pass rows are
  // indexed by fine position minus 2*c_first
  const int ci = lane & 15, half = lane >> 4;
  const bool cv = ci <= c_last - c_first;
  auto xpass = [&](int slot, double *__restrict__ xr) {
    constexpr int RP = (NTL * G::CY + 1) / 2;      // row pairs, upper bound
    constexpr int RQ = (RP + NWARPS - 1) / NWARPS; // row pairs per warp
    const double *__restrict__ cs = coarse;
#pragma unroll
    for (int q = 0; q < RQ; ++q) {
      const int r = 2 * (warp + NWARPS * q) + half;
      if (r < nrows && cv) {
        const int t = (r >= ncy) + (NTL > 2 && r >= 2 * ncy);
        const int yy = r - t * ncy;
        const double *row = cs + ((slot * NTL + t) * G::CY + yy) * G::CXP + (ci - LO);
        auto get = [&](int m) { return row[m]; };
        const double xe = F::template first<FMA>(0, get);
        const double xo = F::template first<FMA>(1, get);
        *reinterpret_cast<double2 *>(xr + (t * G::CY + yy) * G::XR + 2 * ci) = make_double2(xe, xo);
      }
    }
  };

  // --- y/z owner: thread = (fine x, coarse y row), both fine y parities
  const int my_fx = tid % ptx, my_cyr = tid / ptx;
  const int my_cy = (sy0 >> 1) + my_cyr;
  const int ys0 = 2 * my_cy, ys1 = ys0 + 1;
  const bool act = my_cyr < ptyc && my_fx < nfx;
  const bool v0 = act && ys0 >= sy0 && ys0 < sy0 + nfy;
  const bool v1 = act && ys1 >= sy0 && ys1 < sy0 + nfy;
  const int yrow = my_cy - cy0; // index of coarse row my_cy in the plane
  double *out = d.dst + (d.doff[0] + fx0 + my_fx) + (long long)(d.doff[1] + fy0) * d.dsy +
                (long long)(d.doff[2] + fz0) * d.dsz;

  // z window: yq[t][h][s] holds the y-pass result of plane p in slot p % Q
  double yq[NTL][2][Q];
#pragma unroll
  for (int t = 0; t < NTL; ++t)
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int q = 0; q < Q; ++q) yq[t][h][q] = 0.0;

  // y pass of plane p (slot U = p % Q, static) from its x-pass rows, then
  // the z outputs whose window plane p completes: coarse base cb = cz - HI,
  // window planes p-W .. p in slots (U+1+k) % Q
  auto yzpass = [&](auto Ut, int p, const double *__restrict__ xr) {
    constexpr int U = decltype(Ut)::value;
    if (v0 || v1) {
#pragma unroll
      for (int t = 0; t < NTL; ++t) {
        const double *col = xr + (t * G::CY + yrow) * G::XR + my_fx + xoff;
        auto get = [&](int m) { return col[m * G::XR]; };
        yq[t][0][U] = F::template next<FMA>(0, get);
        yq[t][1][U] = F::template next<FMA>(1, get);
      }
    }
    const int cb = cz0 + p - HI;
#pragma unroll
    for (int zp = 0; zp < 2; ++zp) {
      const int zs = 2 * cb + zp;
      if (zs < sz0 || zs >= sz0 + nfz) continue;
      double *o = out + (long long)(zs - sz0) * d.dsz;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (!(h ? v1 : v0)) continue;
        double v[NTL];
#pragma unroll
        for (int t = 0; t < NTL; ++t)
          v[t] = F::template next<FMA>(zp, [&](int m) { return yq[t][h][(U + 1 + (m - LO)) % Q]; });
        o[(long long)((h ? ys1 : ys0) - sy0) * d.dsy] = tcombine<FMA, TK, NTL>(d.w, v);
      }
    }
  };

  // Pipeline, one barrier per plane: iteration i stages plane i+PD, runs
  // the x pass of plane i into x-pass buffer i%2 and the y/z passes of plane
  // i-1 from buffer (i-1)%2.  The staging ring has PD+2 slots, so the slot
  // being refilled was last read two iterations ago.  The loop is unrolled
  // by Q so that every z-window slot index is a compile-time constant.
  const int nplanes = cz1 - cz0 + 1;
#pragma unroll
  for (int p = 0; p < G::PD; ++p) {
    if (p < nplanes) stage(cz0 + p, p);
    cp_async_commit();
  }
  auto iteration = [&](auto Ut, int i) {
    // Ut: the static value of (i - 1) % Q
    if (i + G::PD < nplanes) stage(cz0 + i + G::PD, (i + G::PD) % G::NB);
    cp_async_commit();
    cp_async_wait<G::PD>();
    __syncthreads();
    if (i < nplanes) xpass(i % G::NB, xrows + (i & 1) * S::xbuf);
    if (i >= 1) yzpass(Ut, i - 1, xrows + ((i - 1) & 1) * S::xbuf);
  };
  iteration(std::integral_constant<int, Q - 1>(), 0); // i = 0: x pass only
  for (int i0 = 1; i0 <= nplanes; i0 += Q) {
    static_for<Q>([&](auto Ut) {
      constexpr int u = decltype(Ut)::value;
      const int i = i0 + u;
      if (i <= nplanes) iteration(std::integral_constant<int, u>(), i);
    });
  }
  cp_async_wait<0>();
  __syncthreads(); // shared memory free for the next tile
  (void)W;
}

} // namespace cgx
