// cgx_kernels.cuh -- the kernels: tile dispatch and the three launch forms.
// Included only by the kernel translation units (cgx_kern_*.cu), each of
// which instantiates and launches one floating-point mode / order range.
//
//   k_pair       grid = the tiles of one descriptor (the plain per-box form);
//   k_batch_map  persistent, one CTA per SM slot, tiles of many descriptors
//                taken from a device work counter through a tile map;
//   k_batch      the same, finding each tile's descriptor by binary search
//                over tile offsets (the bounded-scratch form of the
//                no-allocation entry point).
#pragma once
#include <cuda_runtime.h>

#include "../../include/cgx.h"
#include "cgx_device.cuh"
#include "cgx_internal.h"
#include "cgx_tma.cuh"

namespace cgx {
namespace kern {

__device__ __forceinline__ void report(int *status, int code) {
  if (status) atomicCAS(status, 0, code);
}

// dynamic shared memory of the largest variant a kernel dispatches
template <int MAXORDER> constexpr int smem_doubles() {
  return PSmem<VC<MAXORDER>, 3>::total > PSmem<CC<5>, 3>::total
             ? PSmem<VC<MAXORDER>, 3>::total
             : PSmem<CC<5>, 3>::total;
}

// Every tile routine is its own non-inlined function, so that each variant
// gets its own register allocation instead of sharing one across the whole
// dispatch switch.  The descriptor is always in shared memory.
template <class F, int FMA, int NTL, int TK>
__device__ __noinline__ void prolong_entry(const Desc &d, int tile, double *sm) {
  prolong_tile<F, FMA, NTL, TK>(d, tile, sm);
}
template <int FMA, int NTL, int TK>
__device__ __noinline__ void copy_entry(const Desc &d, int tile) {
  copy_tile<FMA, NTL, TK, NTHREADS>(d, tile, threadIdx.x);
}
static __device__ __noinline__ void restrict_vc_entry(const Desc &d, int tile) {
  restrict_vc_tile<NTHREADS>(d, tile, threadIdx.x);
}
template <int FMA> __device__ __noinline__ void restrict_cc_entry(const Desc &d, int tile) {
  restrict_cc_tile<FMA, NTHREADS>(d, tile, threadIdx.x);
}
template <int FMA> __device__ __noinline__ void restrict_cc3_entry(const Desc &d, int tile) {
  restrict_cc3_tile<FMA, NTHREADS>(d, tile, threadIdx.x);
}
template <int FMA> __device__ __noinline__ void restrict_cc5_entry(const Desc &d, int tile) {
  restrict_cc5_tile<FMA, NTHREADS>(d, tile, threadIdx.x);
}
template <int FMA> __device__ __noinline__ void mono_entry(const Desc &d, int tile) {
  mono_tile<FMA, NTHREADS>(d, tile, threadIdx.x);
}

template <class F, int FMA>
__device__ __forceinline__ void prolong_ntl(const Desc &d, int tile, double *sm) {
  switch (d.ntl) {
  case 1: prolong_entry<F, FMA, 1, T_NONE>(d, tile, sm); break;
  case 2: prolong_entry<F, FMA, 2, T_LIN>(d, tile, sm); break;
  default:
    if (d.tkind == T_ENO) prolong_entry<F, FMA, 3, T_ENO>(d, tile, sm);
    else prolong_entry<F, FMA, 3, T_QUAD>(d, tile, sm);
  }
}

// HIGH selects the vertex-centred orders 7/9/11, which live in their own
// kernel so that their larger register windows do not lower the occupancy
// of the common orders.
template <int FMA, bool HIGH>
__device__ __forceinline__ void run_tile(const Desc &d, int tile, double *sm, int *status) {
  switch (d.kind) {
  case K_COPY:
    if (d.ntl == 1) copy_entry<FMA, 1, T_NONE>(d, tile);
    else if (d.ntl == 2) copy_entry<FMA, 2, T_LIN>(d, tile);
    else if (d.tkind == T_ENO) copy_entry<FMA, 3, T_ENO>(d, tile);
    else copy_entry<FMA, 3, T_QUAD>(d, tile);
    return;
  case K_RESTRICT_VC: restrict_vc_entry(d, tile); return;
  case K_RESTRICT_CC: restrict_cc_entry<FMA>(d, tile); return;
  case K_RESTRICT_CC3: restrict_cc3_entry<FMA>(d, tile); return;
  case K_RESTRICT_CC5: restrict_cc5_entry<FMA>(d, tile); return;
  case K_PROLONG_MONO: mono_entry<FMA>(d, tile); return;
  case K_PROLONG_VC:
    if (HIGH) {
      switch (d.order) {
      case 7: prolong_ntl<VC<7>, FMA>(d, tile, sm); return;
      case 9: prolong_ntl<VC<9>, FMA>(d, tile, sm); return;
      case 11: prolong_ntl<VC<11>, FMA>(d, tile, sm); return;
      }
    } else {
      switch (d.order) {
      case 1: prolong_ntl<VC<1>, FMA>(d, tile, sm); return;
      case 3: prolong_ntl<VC<3>, FMA>(d, tile, sm); return;
      case 5: prolong_ntl<VC<5>, FMA>(d, tile, sm); return;
      }
    }
    break;
  case K_PROLONG_CC_ENO:
    if (!HIGH) {
      if (d.order == 2) { prolong_ntl<CCENO<2>, FMA>(d, tile, sm); return; }
      if (d.order == 3) { prolong_ntl<CCENO<3>, FMA>(d, tile, sm); return; }
    }
    break;
  case K_PROLONG_CC:
    if (!HIGH) {
      switch (d.order) {
      case 0: prolong_ntl<CC<0>, FMA>(d, tile, sm); return;
      case 1: prolong_ntl<CC<1>, FMA>(d, tile, sm); return;
      case 2: prolong_ntl<CC<2>, FMA>(d, tile, sm); return;
      case 3: prolong_ntl<CC<3>, FMA>(d, tile, sm); return;
      case 4: prolong_ntl<CC<4>, FMA>(d, tile, sm); return;
      case 5: prolong_ntl<CC<5>, FMA>(d, tile, sm); return;
      }
    }
    break;
  case K_PROLONG_ENO:
    if (!HIGH) { prolong_ntl<ENO, FMA>(d, tile, sm); return; }
    break;
  }
  if (threadIdx.x == 0) report(status, CGX_EDEVICE);
}

template <int FMA, bool HIGH>
__global__ void __launch_bounds__(NTHREADS, 2)
    k_pair(const __grid_constant__ Desc d, int *status) {
  extern __shared__ __align__(16) double sm[];
  __shared__ __align__(16) Desc s_d;
  if (threadIdx.x == 0) s_d = d; // field-wise copy out of the parameter space
  __syncthreads();
  run_tile<FMA, HIGH>(s_d, blockIdx.x, sm, status);
}

// Persistent form: each CTA repeatedly claims the next tile index from
// *counter; prefix[i] is the first global tile of descriptor i.
template <int FMA>
__global__ void __launch_bounds__(NTHREADS, 2)
    k_batch(const Desc *__restrict__ descs, const long long *__restrict__ prefix, int ndesc,
            long long ntiles, unsigned long long *counter, int *status) {
  extern __shared__ __align__(16) double sm[];
  __shared__ long long s_tile;
  __shared__ int s_desc;
  // the claimed descriptor, staged in shared memory: tile code reads it like
  // the kernel-parameter descriptor of k_pair
  __shared__ __align__(16) Desc s_d;
  static_assert(sizeof(Desc) % 8 == 0 && sizeof(Desc) / 8 <= NTHREADS, "descriptor staging");
  for (;;) {
    if (threadIdx.x == 0) {
      long long t = (long long)atomicAdd(counter, 1ULL);
      int lo = 0, hi = ndesc - 1;
      if (t < ntiles) {
        while (lo < hi) { // last descriptor with prefix <= t
          int mid = (lo + hi + 1) >> 1;
          if (prefix[mid] <= t) lo = mid;
          else hi = mid - 1;
        }
      }
      s_tile = t;
      s_desc = lo;
    }
    __syncthreads();
    const long long t = s_tile;
    const int di = s_desc;
    if (t >= ntiles) break;
    if (threadIdx.x < sizeof(Desc) / 8)
      reinterpret_cast<unsigned long long *>(&s_d)[threadIdx.x] =
          __ldg(reinterpret_cast<const unsigned long long *>(descs + di) + threadIdx.x);
    __syncthreads();
    run_tile<FMA, false>(s_d, (int)(t - prefix[di]), sm, status);
    __syncthreads(); // s_tile, s_desc and s_d are free for the next claim
  }
}

// ---------------------------------------------------------------- chaining
// The persistent kernels of a batch run back to back with programmatic
// dependent launch: a kernel waits for its predecessor's completion (and
// memory) before it touches anything, and a CTA that has claimed its last
// tile lets the successor's CTAs be scheduled.  Both are no-ops for a launch
// without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Claim counters reset themselves, so that no memset precedes a launch:
// counter[NSEG] counts the CTAs that have finished claiming, and the last
// one zeroes both for the segment's next launch.  Called by thread 0 after
// its last claim; the fence orders every CTA's claims before its count.
__device__ __forceinline__ void claims_done(unsigned long long *counter) {
  __threadfence();
  unsigned long long *left = counter + NSEG;
  if (atomicAdd(left, 1ULL) == (unsigned long long)gridDim.x - 1) {
    atomicExch(counter, 0ULL);
    atomicExch(left, 0ULL);
  }
}

// Persistent form fed by a tile map: tmap[t] = (descriptor, tile within it).
// Thread 0 claims the next tile when the current one starts, so the
// claim's round trip overlaps the tile's work; only the map read is exposed.
template <int FMA>
__global__ void __launch_bounds__(NTHREADS, 2)
    k_batch_map(const Desc *__restrict__ descs, const int2 *__restrict__ tmap, long long ntiles,
                unsigned long long *counter, int *status) {
  extern __shared__ __align__(16) double sm[];
  __shared__ long long s_t;
  __shared__ int2 s_m;
  __shared__ __align__(16) Desc s_d;
  pdl_wait();
  if (threadIdx.x == 0) {
    const long long t = (long long)atomicAdd(counter, 1ULL);
    s_t = t;
    s_m = t < ntiles ? tmap[t] : make_int2(0, 0);
  }
  __syncthreads();
  for (;;) {
    const long long t = s_t;
    const int2 m = s_m;
    if (t >= ntiles) {
      if (threadIdx.x == 0) claims_done(counter);
      break;
    }
    if (threadIdx.x < sizeof(Desc) / 8)
      reinterpret_cast<unsigned long long *>(&s_d)[threadIdx.x] =
          __ldg(reinterpret_cast<const unsigned long long *>(descs + m.x) + threadIdx.x);
    unsigned long long tn = 0;
    if (threadIdx.x == 0) tn = atomicAdd(counter, 1ULL);
    __syncthreads();
    run_tile<FMA, false>(s_d, m.y, sm, status);
    __syncthreads(); // everyone is done with s_d, s_t and s_m
    if (threadIdx.x == 0) {
      s_t = (long long)tn;
      s_m = (long long)tn < ntiles ? tmap[tn] : make_int2(0, 0);
    }
    __syncthreads();
  }
}


// Streaming kernels (copy and restrictions): no shared-memory stage, so
// they run at high occupancy -- many warps keep their loads in flight.
constexpr int STREAM_BLOCKS_PER_SM = 4;
// the persistent streaming kernels: smaller CTAs, more of them per SM
constexpr int STREAM_THREADS = 128, STREAM_MAP_BLOCKS_PER_SM = 8;

// one streaming variant's tile, run by LANES threads (lid: 0 .. LANES-1);
// V is a StreamVariant
template <int FMA, int V, int LANES>
__device__ __forceinline__ void stream_tile(const Desc &d, int tile, int lid) {
  if (V == SV_COPY1) copy_tile<FMA, 1, T_NONE, LANES>(d, tile, lid);
  else if (V == SV_COPY2) copy_tile<FMA, 2, T_LIN, LANES>(d, tile, lid);
  else if (V == SV_COPY3Q) copy_tile<FMA, 3, T_QUAD, LANES>(d, tile, lid);
  else if (V == SV_COPY3E) copy_tile<FMA, 3, T_ENO, LANES>(d, tile, lid);
  else if (V == SV_RESTRICT_VC) restrict_vc_tile<LANES>(d, tile, lid);
  else if (V == SV_RESTRICT_CC) restrict_cc_tile<FMA, LANES>(d, tile, lid);
  else if (V == SV_RESTRICT_CC3) restrict_cc3_tile<FMA, LANES>(d, tile, lid);
  else if (V == SV_RESTRICT_CC5) restrict_cc5_tile<FMA, LANES>(d, tile, lid);
  else if (V == SV_TIME) time_tile<FMA, LANES>(d, tile, lid);
  else mono_tile<FMA, LANES>(d, tile, lid);
}

// Per-box form: a CTA per tile, every variant in one dispatch.  The
// descriptor parameter is uniform, so its fields are read from the
// parameter space.
template <int FMA>
__global__ void __launch_bounds__(NTHREADS, STREAM_BLOCKS_PER_SM)
    k_spair(const __grid_constant__ Desc d, int *status) {
  __shared__ __align__(16) Desc s_d;
  if (threadIdx.x == 0) s_d = d;
  __syncthreads();
  const int t = blockIdx.x, l = threadIdx.x;
  switch (stream_variant(s_d)) {
  case SV_COPY1: stream_tile<FMA, SV_COPY1, NTHREADS>(s_d, t, l); return;
  case SV_COPY2: stream_tile<FMA, SV_COPY2, NTHREADS>(s_d, t, l); return;
  case SV_COPY3Q: stream_tile<FMA, SV_COPY3Q, NTHREADS>(s_d, t, l); return;
  case SV_COPY3E: stream_tile<FMA, SV_COPY3E, NTHREADS>(s_d, t, l); return;
  case SV_RESTRICT_VC: stream_tile<FMA, SV_RESTRICT_VC, NTHREADS>(s_d, t, l); return;
  case SV_RESTRICT_CC: stream_tile<FMA, SV_RESTRICT_CC, NTHREADS>(s_d, t, l); return;
  case SV_RESTRICT_CC3: stream_tile<FMA, SV_RESTRICT_CC3, NTHREADS>(s_d, t, l); return;
  case SV_RESTRICT_CC5: stream_tile<FMA, SV_RESTRICT_CC5, NTHREADS>(s_d, t, l); return;
  case SV_TIME: stream_tile<FMA, SV_TIME, NTHREADS>(s_d, t, l); return;
  case SV_MONO: stream_tile<FMA, SV_MONO, NTHREADS>(s_d, t, l); return;
  }
  if (threadIdx.x == 0) report(status, CGX_EDEVICE);
}

// Persistent form: one kernel per variant over that variant's segment of
// the tile map, a CTA per tile.  One barrier per tile: thread 0 claims the
// tile after next (a three-slot ring of claims) and the CTA stages the next
// tile's descriptor into the second of two shared buffers while the current
// tile runs.
template <int FMA, int V>
__global__ void __launch_bounds__(STREAM_THREADS, STREAM_MAP_BLOCKS_PER_SM)
    k_stream_map(const Desc *__restrict__ descs, const int2 *__restrict__ tmap, long long ntiles,
                 unsigned long long *counter, int *status) {
  __shared__ __align__(16) Desc s_d[2];
  __shared__ long long s_t[3];
  __shared__ int2 s_m[3];
  const int tid = threadIdx.x;
  constexpr int DW = sizeof(Desc) / 8;
  auto claim = [&](int slot) {
    const long long t = (long long)atomicAdd(counter, 1ULL);
    s_t[slot] = t;
    s_m[slot] = t < ntiles ? tmap[t] : make_int2(0, 0);
  };
  auto stage = [&](int buf, int slot) {
    if (tid < DW && s_t[slot] < ntiles)
      reinterpret_cast<unsigned long long *>(&s_d[buf])[tid] =
          __ldg(reinterpret_cast<const unsigned long long *>(descs + s_m[slot].x) + tid);
  };
  pdl_wait();
  if (tid == 0) {
    claim(0);
    claim(1);
  }
  __syncthreads();
  stage(0, 0);
  __syncthreads();
  for (int i = 0;; ++i) {
    const int slot = i % 3, buf = i & 1;
    if (s_t[slot] >= ntiles) {
      if (tid == 0) claims_done(counter);
      break;
    }
    if (s_t[(i + 1) % 3] >= ntiles) pdl_trigger(); // this CTA's last tile
    const int tile = s_m[slot].y;
    if (tid == 0) claim((i + 2) % 3);
    stage(buf ^ 1, (i + 1) % 3);
    if (stream_variant(s_d[buf]) == V) stream_tile<FMA, V, STREAM_THREADS>(s_d[buf], tile, tid);
    else if (tid == 0) report(status, CGX_EDEVICE);
    __syncthreads();
  }
}

// ---------------------------------------------------------------- TMA form
// One persistent kernel per prolongation variant (family, order, time
// interpolation), so that each gets its own register allocation; maps[3 * i
// + t] is the tensor map of descriptor i's timelevel t.  The claim loop is
// that of k_stream_map.
template <int FMA, class F, int NTL, int TK, int CFG>
__global__ void __launch_bounds__(TMA_CFGS[CFG].nt, TMA_CFGS[CFG].mb)
    k_tma_map(const Desc *__restrict__ descs, const CUtensorMap *__restrict__ maps,
              const int2 *__restrict__ tmap, long long ntiles, unsigned long long *counter, int *status,
              int variant) {
  extern __shared__ __align__(128) double smraw[];
  // 128-byte aligned start, derived from smraw so that the compiler keeps
  // every access in the shared address space
  const unsigned sbase = smem_u32(smraw);
  double *sm = smraw + ((((sbase + 127u) & ~127u) - sbase) >> 3);
  __shared__ long long s_t, s_next;
  __shared__ int2 s_m;
  __shared__ __align__(16) Desc s_d;
  __shared__ __align__(8) uint64_t s_bars[TMA_NB_MAX];
  __shared__ int s_abort;
  // bit 30 of variant: failure injection (cgx_debug_skip_tma_plane)
  const int skip = (variant >> 30) & 1 ? 0 : -1;
  variant &= ~(1 << 30);
  pdl_wait();
  if (threadIdx.x == 0) {
    for (int i = 0; i < TMA_NB_MAX; ++i) mbar_init(&s_bars[i], 1);
    mbar_fence_init();
    s_abort = 0;
    const long long t = (long long)atomicAdd(counter, 1ULL);
    s_t = t;
    s_m = t < ntiles ? tmap[t] : make_int2(0, 0);
  }
  __syncthreads();
  TmaRing ring{s_bars, &s_abort, 0u, skip};
  for (;;) {
    if (s_t >= ntiles) {
      if (threadIdx.x == 0) claims_done(counter);
      break;
    }
    const int2 m = s_m;
    if (threadIdx.x < sizeof(Desc) / 8)
      reinterpret_cast<unsigned long long *>(&s_d)[threadIdx.x] =
          __ldg(reinterpret_cast<const unsigned long long *>(descs + m.x) + threadIdx.x);
    if (threadIdx.x == 0) s_next = (long long)atomicAdd(counter, 1ULL);
    __syncthreads();
    if (s_next >= ntiles) pdl_trigger(); // this CTA's last tile
    if (tma_variant(s_d) == variant) {
      if (!prolong_tile_tma<F, FMA, NTL, TK, CFG>(s_d, maps + 3 * (size_t)m.x, m.y, sm, ring, status)) {
        if (threadIdx.x == 0) claims_done(counter);
        return;
      }
    } else if (threadIdx.x == 0) {
      report(status, CGX_EDEVICE);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const long long tn = s_next;
      s_t = tn;
      s_m = tn < ntiles ? tmap[tn] : make_int2(0, 0);
    }
    __syncthreads();
  }
}

// dynamic shared memory of the widest variant a kernel dispatches
inline size_t smem_bytes(bool high) {
  return sizeof(double) * (high ? smem_doubles<11>() : smem_doubles<5>());
}

} // namespace kern
} // namespace cgx
