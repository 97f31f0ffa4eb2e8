// cgx_tma.cuh -- prolongation with TMA staging (device code).
//
// The same separable x -> y -> z arithmetic as prolong_tile (cgx_device.cuh),
// organised so that every thread's work is fixed per tile and the plane loop
// is straight-line code:
//
//   * one elected thread stages each coarse plane with one bulk tensor copy
//     per timelevel (cp.async.bulk.tensor, a box of bx x by coarse points),
//     completing on an mbarrier per ring slot; boxes may start outside the
//     array (zero fill), which only masked outputs read;
//   * the x pass is a flat list of (timelevel, coarse row, coarse base)
//     items spread over all threads, whatever the tile's shape; each item's
//     shared-memory offsets are computed once per tile;
//   * the y/z pass keeps its thread = (fine x, coarse y row) mapping and
//     register z window; threads without a point compute on clamped
//     indices and their stores are masked, so no branch diverges.
//
// A descriptor is eligible when its source arrays can be described to the
// tensor-copy unit (16-byte aligned base, even row and plane pitches); the
// host builds one CUtensorMap per timelevel at upload time.
#pragma once
#include <cuda.h>

#include "cgx_device.cuh"

namespace cgx {

// Tile configurations the autotuner chooses between: threads per CTA, coarse
// y rows per tile (threads / 16: one thread per fine x and coarse row), fine
// z points per tile, CTAs per SM the register allocation must allow, and
// planes staged ahead of the x pass.  Configuration 0 is the default.
struct TmaCfg {
  int nt, pyc, pz, mb, pd;
};
constexpr TmaCfg TMA_CFGS[] = {
    {256, 16, 64, 2, 3}, {128, 8, 64, 4, 3}, {128, 8, 32, 4, 3}, {128, 8, 64, 5, 2}, {128, 8, 32, 6, 2}};
constexpr int TMA_NCFG = 5;
constexpr int TMA_NB_MAX = 5; // ring slots, at most (pd + 2)

// Shared-memory geometry of a tile configuration with PYC coarse rows for a
// stencil window of width W (host and device).  A tile of ptx fine x uses
// ptx * ptyc owner threads; ptyc may exceed PYC when ptx < 16, as far as the
// staged box, the x-pass rows and the x items fit (tma_rows_max, host).
//   coarse box      bx = (ptx + 2) / 2 bases + the window + one point of
//                   even-alignment shift, rounded up to even; by = ptyc + W
//                   rows; bx * by <= tma_tls doubles per (slot, timelevel)
//   x-pass rows     ntl * by rows of pitch TMA_XR (two fine points per coarse
//                   base: at most ptx + 2 <= 18), + one spare row for masked
//                   x items; a half-warp of the y pass reads one row when
//                   ptx = 16, at most three short rows otherwise
//   x items         (timelevel, coarse row, coarse base), at most
//                   ntl * tma_items per tile
constexpr int TMA_EXTRA_ROWS = 3; // rows staged beyond PYC + W (for ptx < 16)
__host__ __device__ constexpr int tma_bxmax(int W) { return ((PTXMAX + 2) / 2 + W + 2) & ~1; }
__host__ __device__ constexpr int tma_bymax(int W, int pyc) { return pyc + W + TMA_EXTRA_ROWS; }
__host__ __device__ constexpr int tma_tls(int W, int pyc) { return (tma_bxmax(W) * tma_bymax(W, pyc) + 15) / 16 * 16; }
constexpr int TMA_XR = PTXMAX + 2; // even: 16-byte rows
__host__ __device__ constexpr int tma_xbuf(int W, int pyc, int ntl) { return (ntl * tma_bymax(W, pyc) + 1) * TMA_XR; }
__host__ __device__ constexpr int tma_items(int W, int pyc) { return (pyc + W) * ((PTXMAX + 2) / 2); }

template <class F, int PYC = PTYCMAX> struct TGeom {
  static constexpr int W = F::HI - F::LO;
  static constexpr int TLS = tma_tls(W, PYC); // doubles per (slot, timelevel)
  static constexpr int ITEMS = tma_items(W, PYC);
  static constexpr int Q = W + 1;
};
template <class F, int NTL, int PYC = PTYCMAX, int NB = 5> struct TSmem {
  using G = TGeom<F, PYC>;
  static constexpr int coarse = NB * NTL * G::TLS;
  static constexpr int xbuf = tma_xbuf(G::W, PYC, NTL);
  static constexpr int total = coarse + 2 * xbuf; // doubles
};

// The TMA kernels' variants: family (VC 1/3/5, CC 0-5, ENO) x time
// interpolation (one timelevel, linear, quadratic, ENO).
constexpr int TV_FAMILIES = 10;
constexpr int TV_COUNT = 4 * TV_FAMILIES;
template <class D> __host__ __device__ __forceinline__ int tma_variant(const D &d) {
  int f = -1;
  if (d.kind == K_PROLONG_VC) f = d.order == 1 ? 0 : d.order == 3 ? 1 : d.order == 5 ? 2 : -1;
  else if (d.kind == K_PROLONG_CC) f = d.order >= 0 && d.order <= 5 ? 3 + d.order : -1;
  else if (d.kind == K_PROLONG_ENO) f = 9;
  if (f < 0) return -1;
  const int tv = d.ntl == 1 ? 0 : d.ntl == 2 ? 1 : d.tkind == T_ENO ? 3 : 2;
  return 4 * f + tv;
}

// ---------------------------------------------------------------- PTX
__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile("{\n"
               " .reg .pred p;\n"
               " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
               " selp.u32 %0, 1, 0, p;\n"
               "}\n"
               : "=r"(ok)
               : "r"(smem_u32(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}
// Waits for the phase of the given parity; gives up after about 2^31 clock
// cycles (a second) and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > (1LL << 31)) return false;
  return true;
}
// One box of a 3-d tensor map into shared memory, completing on *bar.
__device__ __forceinline__ void tma_load_3d(double *dst, const CUtensorMap *map, uint64_t *bar, int x, int y,
                                            int z) {
  asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
               " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_u32(dst)),
               "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
               : "memory");
}

// Ring state of one CTA: planes staged so far (plane g uses slot g % NB,
// whose phase g / NB completes when it lands), and a flag that a wait ran
// out.  Everything here is uniform over the CTA.
struct TmaRing {
  uint64_t *bars; // pd + 2 mbarriers, arrival count 1
  int *abort;     // shared flag, set when a wait gave up
  unsigned g;     // planes staged by this CTA before the current tile
  // failure injection for the tests of the bounded waits
  // (cgx_debug_skip_tma_plane): the plane of this CTA's first tile that is
  // never staged, so that the wait for it runs out; -1 in normal use
  int skip = -1;
};

// One prolongation tile.  Returns false when a wait gave up (the CTA then
// stops; the status word holds CGX_EDEVICE).
template <class F, int FMA, int NTL, int TK, int CFG>
__device__ bool prolong_tile_tma(const Desc &d, const CUtensorMap *__restrict__ maps, int tile, double *sm,
                                 TmaRing &ring, int *status) {
  constexpr int NT = TMA_CFGS[CFG].nt, PYC = TMA_CFGS[CFG].pyc, PZ = TMA_CFGS[CFG].pz;
  constexpr int PD = TMA_CFGS[CFG].pd, NB = PD + 2;
  using G = TGeom<F, PYC>;
  using S = TSmem<F, NTL, PYC, NB>;
  constexpr int LO = F::LO, HI = F::HI, Q = G::Q;
  constexpr bool SPLIT = NTL == 1;
  const int tid = threadIdx.x;
  const int ptx = d.ptx, ptyc = d.ptyc, pty = 2 * ptyc - 1;
  const int BX = d.bx, BY = d.by;
  // x-pass rows: BY per timelevel, pitch XR
  constexpr int XR = TMA_XR;
  const int CY = BY;

  const int tx = tile % d.tiles[0], rr = tile / d.tiles[0];
  const int ty = rr % d.tiles[1], tz = rr / d.tiles[1];
  const int fx0 = tx * ptx, fy0 = ty * pty, fz0 = tz * PZ;
  const int nfx = min(ptx, d.n[0] - fx0), nfy = min(pty, d.n[1] - fy0), nfz = min(PZ, d.n[2] - fz0);
  const int sx0 = d.soff[0] + fx0, sy0 = d.soff[1] + fy0, sz0 = d.soff[2] + fz0;
  const int c_first = sx0 >> 1, c_last = (sx0 + nfx - 1) >> 1;
  const int cx0 = c_first + LO;
  const int bx0 = cx0 & ~1; // box start: an even x coordinate
  const int xs = cx0 - bx0;
  const int cy0 = (sy0 >> 1) + LO, cy1 = ((sy0 + nfy - 1) >> 1) + HI;
  const int cz0 = (sz0 >> 1) + LO, cz1 = ((sz0 + nfz - 1) >> 1) + HI;
  const int nbx = c_last - c_first + 1, ncy = cy1 - cy0 + 1;
  const int nplanes = cz1 - cz0 + 1;
  const int xoff = sx0 - 2 * c_first;
  const unsigned g0 = ring.g;

  double *coarse = sm;
  double *xrows = sm + S::coarse;

  int issued = 0; // planes staged so far (elected thread)
  const int skip = g0 == 0 ? ring.skip : -1;
  int islot = (int)(g0 % NB); // multi-timelevel: ring slot of the next plane staged
  auto issue = [&](int p) {   // elected thread: stage plane p (p = 0, 1, ...)
    issued = p + 1;
    int slot;
    if constexpr (SPLIT) {
      slot = (int)((g0 + (unsigned)p) % NB);
    } else {
      slot = islot;
      if (++islot == NB) islot = 0;
    }
    if (p == skip) return; // failure injection: this plane never lands
    mbar_expect_tx(&ring.bars[slot], (unsigned)(NTL * BX * BY * 8));
#pragma unroll
    for (int t = 0; t < NTL; ++t)
      tma_load_3d(coarse + (slot * NTL + t) * G::TLS, maps + t, &ring.bars[slot], bx0, cy0, cz0 + p);
  };

  // --- x items: (timelevel, row, base) spread over the CTA
  constexpr int IT = (NTL * G::ITEMS + NT - 1) / NT; // ncy * nbx <= ITEMS
  const int per_t = ncy * nbx, count = NTL * per_t;
  int xsrc[IT], xdst[IT];
#pragma unroll
  for (int k = 0; k < IT; ++k) {
    const int it = tid + k * NT;
    if (it < count) {
      const int t = it / per_t, rem = it - t * per_t;
      const int r = rem / nbx, b = rem - r * nbx;
      xsrc[k] = t * G::TLS + r * BX + xs + b; // window element j of base b at xsrc + j - LO
      xdst[k] = (t * CY + r) * XR + 2 * b;
    } else {
      xsrc[k] = 0;
      xdst[k] = NTL * CY * XR; // the spare row
    }
  }
  auto xpass = [&](int slot, double *__restrict__ xr) {
    const double *__restrict__ cs = coarse + slot * NTL * G::TLS - LO;
    // every thread runs its items of all rounds but, without SPLIT, the last
    // one when the tile has no item there (items past the plane's count read
    // the slot's first points and write the spare row)
#pragma unroll
    for (int k = 0; k < IT; ++k) {
      if (SPLIT || k < IT - 1 || k * NT < count) { // uniform
        const double *row = cs + xsrc[k];
        auto get = [&](int m) { return row[m]; };
        const double xe = F::template first<FMA>(0, get);
        const double xo = F::template first<FMA>(1, get);
        *reinterpret_cast<double2 *>(xr + xdst[k]) = make_double2(xe, xo);
      }
    }
  };

  // --- y/z owner: thread = (fine x, coarse y row) = (tid % ptx, tid / ptx);
  // threads past the ptx * ptyc owners address row ptyc - 1 and store nothing
  static_assert(PTXMAX == 16 && NT == 16 * PYC, "y/z thread layout of a full-width tile");
  const int my_fx = tid % ptx, my_cyr_all = tid / ptx;
  const bool tact = my_cyr_all < ptyc;
  const int my_cyr = tact ? my_cyr_all : ptyc - 1;
  const bool wact = (tid & ~31) / ptx < ptyc; // warp holds an owner
  const int my_cy = (sy0 >> 1) + my_cyr;
  const int ys0 = 2 * my_cy;
  const bool xin = tact && my_fx < nfx;
  const bool v0 = xin && ys0 >= sy0 && ys0 < sy0 + nfy;
  const bool v1 = xin && ys0 + 1 >= sy0 && ys0 + 1 < sy0 + nfy;
  const int ycol = (my_cyr - LO) * XR + my_fx + xoff;
  const long long dsy = d.dsy, dsz = d.dsz;
  double *const obase = d.dst + (d.doff[0] + fx0 + my_fx) + (long long)(d.doff[1] + fy0 + ys0 - sy0) * dsy +
                        (long long)(d.doff[2] + fz0 - sz0) * dsz;
  double w[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) w[k] = (NTL == 1 || (TK != T_ENO && k >= NTL)) ? 0.0 : d.w[k];

  double yq[NTL][2][Q];
#pragma unroll
  for (int t = 0; t < NTL; ++t)
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int q = 0; q < Q; ++q) yq[t][h][q] = 0.0;

  // o0: this thread's store address in fine plane 2 * (cz0 + p - HI), carried
  // by the multi-timelevel loop (the one-timelevel loop computes it here)
  auto yzpass = [&](auto Ut, int p, const double *__restrict__ xr, double *o0) {
    constexpr int U = decltype(Ut)::value;
    if (!wact) return; // warp-uniform
#pragma unroll
    for (int t = 0; t < NTL; ++t) {
      const double *col = xr + t * CY * XR + ycol;
      auto get = [&](int m) { return col[m * XR]; };
      yq[t][0][U] = F::template next<FMA>(0, get);
      yq[t][1][U] = F::template next<FMA>(1, get);
    }
    const int cb = cz0 + p - HI;
#pragma unroll
    for (int zp = 0; zp < 2; ++zp) {
      const int zs = 2 * cb + zp;
      const bool zok = zs >= sz0 && zs < sz0 + nfz; // uniform
      double *o;
      if constexpr (SPLIT) o = obase + (long long)zs * dsz;
      else o = zp ? o0 + dsz : o0;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        double v[NTL];
#pragma unroll
        for (int t = 0; t < NTL; ++t)
          v[t] = F::template next<FMA>(zp, [&](int m) { return yq[t][h][(U + 1 + (m - LO)) % Q]; });
        const double r = tcombine<FMA, TK, NTL>(w, v);
        if (zok && (h ? v1 : v0)) o[h ? dsy : 0] = r;
      }
    }
  };

  // Pipeline as in prolong_tile, one barrier per plane; the elected thread
  // stages plane i + PD at the start of iteration i, into the slot last read
  // by the x pass of plane i + PD - NB = i - 2.
  if (tid == 0) {
#pragma unroll
    for (int p = 0; p < PD; ++p)
      if (p < nplanes) issue(p);
  }
  // One-timelevel iteration i: stage plane i + PD; wait for plane i (the
  // barrier also reduces the waits' failures, __syncthreads_or), run its x
  // pass (DX: i < nplanes) and the y/z pass of plane i - 1 (DY: i >= 1).
  // Multi-timelevel iteration i (iteration_rt): stage plane i + PD, run the
  // y/z pass of plane i - 1 first -- on x-pass rows finished before the
  // previous iteration's barrier -- which gives the copies of plane i a
  // long pass's time to land, then wait for plane i, run its x pass, and
  // end with the barrier.  With
  // SPLIT (one timelevel: a short loop body) the whole groups of Q
  // iterations run without per-iteration checks and a second unrolled copy
  // handles the last ones.
  bool ok = true;
  auto iteration = [&](auto Ut, int i, auto DX, auto DY) {
    constexpr bool X = decltype(DX)::value, Y = decltype(DY)::value;
    if (!ok) return; // uniform: a wait gave up
    if (tid == 0 && i + PD < nplanes) issue(i + PD);
    const unsigned g = g0 + (unsigned)i;
    const int fail = X ? !mbar_wait_bounded(&ring.bars[g % NB], (g / NB) & 1) : 0;
    if (__syncthreads_or(fail)) {
      if (tid == 0) *ring.abort = 1;
      ok = false;
      return;
    }
    if (X) xpass((int)(g % NB), xrows + (i & 1) * S::xbuf);
    if (Y) yzpass(Ut, i - 1, xrows + ((i - 1) & 1) * S::xbuf, nullptr);
  };
  // the same iteration with run-time checks, one unrolled copy: the loop of
  // the multi-timelevel variants, whose long bodies make a second unrolled
  // copy (and its register allocation) cost more than the checks.  Its
  // plane-dependent addresses are carried from one iteration to the next
  // rather than recomputed: the ring slot and phase of plane i (slot
  // (g0 + i) % NB, phase (g0 + i) / NB), the x-pass rows of planes i and
  // i - 1, and the store address of the y/z pass's plane i - 1.
  int rslot = (int)(g0 % NB);
  unsigned rpar = (g0 / NB) & 1;
  double *oz = obase + (long long)(2 * (cz0 - HI)) * dsz;
  const long long dz2 = 2 * dsz;
  double *xcur = xrows, *xprev = xrows + S::xbuf; // x-pass rows of planes i, i - 1
  auto iteration_rt = [&](auto Ut, int i) {
    if (tid == 0 && i + PD < nplanes) issue(i + PD);
    if (i >= 1) {
      yzpass(Ut, i - 1, xprev, oz);
      oz += dz2;
    }
    const bool landed = i < nplanes && mbar_wait_bounded(&ring.bars[rslot], rpar);
    if (landed) xpass(rslot, xcur);
    double *const xt = xcur;
    xcur = xprev;
    xprev = xt;
    if (++rslot == NB) {
      rslot = 0;
      rpar ^= 1u;
    }
    if (__syncthreads_or(i < nplanes && !landed)) { // a wait gave up
      if (tid == 0) *ring.abort = 1;
      ok = false;
    }
  };
  using T_ = std::true_type;
  using F_ = std::false_type;
  int i0 = 1;
  if (SPLIT) {
    iteration(std::integral_constant<int, Q - 1>(), 0, T_(), F_());
    // whole groups of Q iterations with both passes, then the last ones
    for (; ok && i0 + Q <= nplanes; i0 += Q)
      static_for<Q>([&](auto Ut) { iteration(Ut, i0 + decltype(Ut)::value, T_(), T_()); });
    static_for<Q>([&](auto Ut) {
      const int i = i0 + decltype(Ut)::value;
      if (ok && i < nplanes) iteration(Ut, i, T_(), T_());
      else if (ok && i == nplanes) iteration(Ut, i, F_(), T_());
    });
  } else {
    iteration_rt(std::integral_constant<int, Q - 1>(), 0);
    for (; ok && i0 <= nplanes; i0 += Q)
      static_for<Q>([&](auto Ut) {
        const int i = i0 + decltype(Ut)::value;
        if (ok && i <= nplanes) iteration_rt(Ut, i);
      });
  }
  if (!ok) {
    // a wait gave up: wait (bounded) for every plane staged, so that no
    // copy lands after the CTA has left
    if (tid == 0) {
      if (status) atomicCAS(status, 0, CGX_EDEVICE);
      for (int i = 0; i < issued; ++i) {
        if (i == skip) continue;
        const unsigned g = g0 + (unsigned)i;
        mbar_wait_bounded(&ring.bars[g % NB], (g / NB) & 1);
      }
    }
    __syncthreads();
    return false;
  }
  ring.g = g0 + (unsigned)nplanes;
  __syncthreads(); // shared memory free for the next tile
  return true;
}

} // namespace cgx
