// cgx_chain.cuh -- the chain kernel: a whole sequence of dependent batches
// (one coarse Berger-Oliger step: every boundary prolongation, ghost sync
// and restriction of every level) in ONE persistent launch.
//
// The host lays every tile of every batch into one list, batch by batch and,
// within a batch, group by group (a group is an independent data stream --
// one grid function, whose arrays no other group reads or writes).  A tile
// of batch j and group g may start once every tile of the previous batch of
// group g has completed: the order of the reference's calls is kept per
// grid function, while the tiles of the next phase of other grid functions
// fill the SMs that a phase's last tiles leave idle, and compute-bound
// prolongation tiles share the SMs with memory-bound copy tiles.
//
// Progress: CTAs claim tiles in list order from one counter, and a tile only
// ever waits for tiles earlier in the list, which were claimed before it by
// CTAs that are resident and run them to completion.  The earliest tile not
// yet complete therefore never waits, so the launch cannot deadlock.  Every
// wait is bounded (about a second); a wait that gives up, or a TMA copy that
// never lands, sets the launch's abort word and the status word
// (CGX_EDEVICE), after which every CTA skips the work of the tiles it claims
// and the launch drains.
//
// Memory ordering: a tile's completion is published by its CTA barrier
// followed by thread 0's fence and counter increment (release); the waiting
// CTA's thread 0 reads the counter with acquire semantics, then a proxy
// fence orders its TMA reads after it, then the CTA barrier releases the
// other threads, whose source loads bypass L1 (ld.global.cg).
#pragma once
#include "cgx_kern_launch.cuh"

namespace cgx {
namespace kern {

// the control words of a chain launch (CHAIN_CTL_WORDS of them)
constexpr int CHAIN_CLAIM = 0, CHAIN_EXIT = 1, CHAIN_ABORT = 2;
static_assert(CHAIN_ABORT < CHAIN_CTL_WORDS, "chain control words");
// about a second at B200 clocks
constexpr long long CHAIN_WAIT_CYCLES = 1LL << 31;
// points per copy or injection tile in the chain (16 per thread of 128):
// larger than the streaming kernels' tiles, since the chain's CTAs are
// fewer per SM and every thread must keep more loads in flight
constexpr int CHAIN_STILE = 2048;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

// Thread 0: waits until *cnt reaches need; false when the launch was
// aborted meanwhile or the wait ran past its limit.
__device__ __forceinline__ bool chain_wait(const unsigned *cnt, unsigned need, const unsigned long long *abort) {
  if (ld_acquire_u32(cnt) >= need) return true;
  const long long t0 = clock64();
  for (;;) {
    __nanosleep(64);
    if (ld_acquire_u32(cnt) >= need) return true;
    if (ld_relaxed_u64(abort)) return false;
    if (clock64() - t0 > CHAIN_WAIT_CYCLES) return false;
  }
}

// The streaming tiles are calls of their own: inlined beside the
// prolongation tiles they would make the register allocator spill the
// latter's stencil windows; as calls they cost a call per 2048 points.
template <int FMA, int NT>
__device__ __noinline__ void chain_copy(const Desc &d, int tile, int tid) {
  copy_tile<FMA, 1, T_NONE, NT, Desc, true, CHAIN_STILE, 16>(d, tile, tid);
}
template <int NT> __device__ __noinline__ void chain_inject(const Desc &d, int tile, int tid) {
  restrict_vc_tile<NT, Desc, true, CHAIN_STILE, 16>(d, tile, tid);
}

template <int FMA, int ORDER, int CFG>
__global__ void __launch_bounds__(TMA_CFGS[CFG].nt, TMA_CFGS[CFG].mb)
    k_chain(const Desc *__restrict__ descs, const CUtensorMap *__restrict__ maps,
            const ChainTile *__restrict__ tiles, long long ntiles, const unsigned *__restrict__ need,
            unsigned *done, int ncounters, unsigned long long *ctl, int *status) {
  constexpr int NT = TMA_CFGS[CFG].nt;
  extern __shared__ __align__(128) double smraw[];
  const unsigned sbase = smem_u32(smraw);
  double *sm = smraw + ((((sbase + 127u) & ~127u) - sbase) >> 3);
  // a ring of four claims (tile index and list entry) and two descriptor
  // buffers: while tile i runs, tile i+1's descriptor and tile i+2's entry
  // are copied into shared memory (cp.async) and the claim of tile i+3 is in
  // flight, so that no claim, entry or descriptor latency lies between tiles
  __shared__ long long s_idx[4];
  __shared__ __align__(16) ChainTile s_ct[4];
  __shared__ __align__(16) Desc s_d[2];
  __shared__ int s_go, s_last;
  __shared__ __align__(8) uint64_t s_bars[TMA_NB_MAX];
  __shared__ int s_abort;
  const int tid = threadIdx.x;
  constexpr int DW = sizeof(Desc) / 16;
  static_assert(sizeof(Desc) % 16 == 0 && DW <= NT, "descriptor staging");
  auto cp16 = [](void *smem, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
  };
  auto stage_desc = [&](int slot, int buf) { // threads < DW
    if (tid < DW && s_idx[slot] < ntiles)
      cp16(reinterpret_cast<char *>(&s_d[buf]) + 16 * tid,
           reinterpret_cast<const char *>(descs + s_ct[slot].desc) + 16 * tid);
  };
  auto fail_launch = [&]() { // thread 0
    atomicExch(&ctl[CHAIN_ABORT], 1ULL);
    report(status, CGX_EDEVICE);
  };
  pdl_wait();
  unsigned long long tn = 0; // thread 0: the claim in flight
  if (tid == 0) {
    for (int i = 0; i < TMA_NB_MAX; ++i) mbar_init(&s_bars[i], 1);
    mbar_fence_init();
    s_abort = 0;
    for (int k = 0; k < 2; ++k) {
      const long long t = (long long)atomicAdd(&ctl[CHAIN_CLAIM], 1ULL);
      s_idx[k] = t;
      if (t < ntiles) s_ct[k] = tiles[t];
    }
    tn = atomicAdd(&ctl[CHAIN_CLAIM], 1ULL);
  }
  __syncthreads();
  stage_desc(0, 0);
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  if (tid == 0) { // the first tile's dependency
    bool ok = !ld_relaxed_u64(&ctl[CHAIN_ABORT]);
    const int dep = s_ct[0].dep;
    if (ok && s_idx[0] < ntiles && dep >= 0) ok = chain_wait(done + dep, __ldg(need + dep), &ctl[CHAIN_ABORT]);
    if (!ok) fail_launch();
    fence_proxy_async_global();
    s_go = ok;
  }
  __syncthreads();
  TmaRing ring{s_bars, &s_abort, 0u};
  bool ring_ok = true; // false once a TMA wait of this CTA gave up
  for (int i = 0;; ++i) {
    const int slot = i & 3, buf = i & 1;
    if (s_idx[slot] >= ntiles) break;
    const int nslot = (i + 1) & 3;
    // claims, entries and the next descriptor, all asynchronous
    unsigned next_seen = 0;
    if (tid == 0) {
      const int cs = (i + 2) & 3;
      s_idx[cs] = (long long)tn;
      if ((long long)tn < ntiles) cp16(&s_ct[cs], tiles + tn);
      tn = atomicAdd(&ctl[CHAIN_CLAIM], 1ULL);
      const int dep = s_ct[nslot].dep;
      if (s_idx[nslot] < ntiles && dep >= 0) {
        asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(next_seen) : "l"(done + dep) : "memory");
      }
    }
    stage_desc(nslot, buf ^ 1);
    if (s_go) {
      const Desc &d = s_d[buf];
      if (d.kind == K_PROLONG_VC) {
        const CUtensorMap *m = maps + 3 * (size_t)s_ct[slot].desc;
        const int tile = s_ct[slot].tile;
        const bool r = d.ntl == 1 ? prolong_tile_tma<VC<ORDER>, FMA, 1, T_NONE, CFG>(d, m, tile, sm, ring, status)
                                  : prolong_tile_tma<VC<ORDER>, FMA, 3, T_QUAD, CFG>(d, m, tile, sm, ring, status);
        if (!r) { // the CTA's ring is no longer in a known state
          ring_ok = false;
          if (tid == 0) atomicExch(&ctl[CHAIN_ABORT], 1ULL);
        }
      } else if (d.kind == K_COPY) {
        chain_copy<FMA, NT>(d, s_ct[slot].tile, tid);
      } else if (d.kind == K_RESTRICT_VC) {
        chain_inject<NT>(d, s_ct[slot].tile, tid);
      } else if (tid == 0) {
        fail_launch();
      }
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads(); // every store of tile i is issued; the staged entries are visible
    if (tid == 0) {
      // one fence: releases tile i's stores before its counter, and (after
      // the relaxed read of the next tile's counter above) acquires what
      // that read observed
      __threadfence();
      atomicAdd(done + s_ct[slot].own, 1u);
      bool ok = ring_ok && !ld_relaxed_u64(&ctl[CHAIN_ABORT]);
      const int dep = s_ct[nslot].dep;
      if (ok && s_idx[nslot] < ntiles && dep >= 0) {
        const unsigned nd = __ldg(need + dep);
        if (next_seen < nd) ok = chain_wait(done + dep, nd, &ctl[CHAIN_ABORT]);
      }
      if (!ok) fail_launch();
      fence_proxy_async_global(); // the next tile's TMA reads come after the acquire
      s_go = ok;
    }
    __syncthreads();
  }
  pdl_trigger(); // this CTA is done: the next launch's CTAs may take its place
  // the last CTA to leave resets the counters for the next launch: every
  // other CTA has completed all its tiles by then
  if (tid == 0) {
    __threadfence();
    s_last = atomicAdd(&ctl[CHAIN_EXIT], 1ULL) == (unsigned long long)gridDim.x - 1;
  }
  __syncthreads();
  if (s_last) {
    for (int i = tid; i < ncounters; i += NT) done[i] = 0u;
    if (tid == 0) {
      ctl[CHAIN_CLAIM] = 0ULL;
      ctl[CHAIN_EXIT] = 0ULL;
      ctl[CHAIN_ABORT] = 0ULL;
    }
    __threadfence();
  }
}

template <int ORDER, int CFG> constexpr size_t chain_smem_bytes() {
  return sizeof(double) * TSmem<VC<ORDER>, 3, TMA_CFGS[CFG].pyc, TMA_CFGS[CFG].pd + 2>::total + 128;
}

template <int FMA, int ORDER, int CFG>
int launch_chain_t(const Desc *d_descs, const CUtensorMap *d_maps, const ChainTile *d_tiles, long long ntiles,
                   const unsigned *d_need, unsigned *d_done, int ncounters, unsigned long long *d_ctl,
                   int *d_status, cudaStream_t s) {
  constexpr int NT = TMA_CFGS[CFG].nt;
  constexpr size_t smem = chain_smem_bytes<ORDER, CFG>();
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_chain<FMA, ORDER, CFG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return cuda_error(e, "cudaFuncSetAttribute");
    attr = true;
  }
  int grid = 0;
  persistent_grid(k_chain<FMA, ORDER, CFG>, smem, ntiles, &grid, NT);
  cudaError_t e = launch_chained(k_chain<FMA, ORDER, CFG>, grid, NT, smem, s, d_descs, d_maps, d_tiles, ntiles,
                                 d_need, d_done, ncounters, d_ctl, d_status);
  return e == cudaSuccess ? CGX_OK : cuda_error(e, "k_chain launch");
}

} // namespace kern
} // namespace cgx
