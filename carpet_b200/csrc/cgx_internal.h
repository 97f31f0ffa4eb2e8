// cgx_internal.h -- pieces of the library shared between its translation
// units (not part of the C-ABI).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/cgx.h"
#include "cgx_device.cuh"
#include "cgx_tma.cuh"

namespace cgx {

// One validated box-pair: the device descriptor, its tile count and its
// algorithmic traffic.
struct BuiltPair {
  Desc d;
  long long bytes;  // algorithmic bytes (reads + writes)
  long long points; // destination points written
  int ntiles;
};

// Validation and descriptor building of cgx_transfer (cgx.cu).
int host_build(int op, int cent, const cgx_array *dst, const cgx_array *srcs, const double *times,
               int nsrc, const int *dstbox, const int *srcbox, const int *slab, double time,
               int order_space, int order_time, BuiltPair *out);

// The host-side descriptors of a batch (cgx.cu).
int batch_pairs(const cgx_batch *b, const Desc **descs, const int **ntiles, const long long **points,
                const long long **bytes, int *n);

// A tile map is laid out in segments, one persistent kernel each: segment v
// < TV_COUNT holds the prolongation tiles of TMA variant v, segment
// SEG_STENCIL the other prolongation tiles (cp.async staging), segment
// SEG_STREAM + v the tiles of streaming variant v.  seg[i] .. seg[i+1] is
// segment i's range.
constexpr int SEG_STENCIL = TV_COUNT;
constexpr int SEG_STREAM = TV_COUNT + 1;
constexpr int NSEG = SEG_STREAM + SV_COUNT;

// Persistent-kernel launches over the non-empty segments of a device tile
// map (cgx.cu); d_maps[3 * i + t] is the tensor map of descriptor i's
// timelevel t (read for segment 0 only); d_counter points to NSEG work
// counters, which this zeroes; grids sized to the device.
int launch_tile_map(const Desc *d_descs, const CUtensorMap *d_maps, const int2 *d_tmap,
                    const long long seg[NSEG + 1], unsigned long long *d_counter, int *d_status, int fp,
                    cudaStream_t s);

// The segments of a tile map launched concurrently (cgx.cu): every
// non-empty segment but the time combination on a stream of its own
// (side[0 .. nside-1], forked from s with ev[0] and joined back with
// ev[1 + k]), then the time segment on s; nside + 1 events.  Returns the
// number of side streams needed in *need when they do not suffice.
int launch_map_concurrent(int fp, const Desc *d, const CUtensorMap *maps, const int2 *tmap,
                          const long long seg[NSEG + 1], const int *cfg, unsigned long long *counter,
                          int *status, cudaStream_t s, const cudaStream_t *side, const cudaEvent_t *ev,
                          int nside, int *need, const int *caps = nullptr);
constexpr int CONCURRENT_SIDE_MAX = NSEG;

// The tensor maps of a prolongation descriptor's source timelevels (cgx.cu):
// true when the arrays can be staged by TMA (then maps[0 .. ntl-1] are
// set), false otherwise.
bool encode_tma_maps(const Desc &d, CUtensorMap maps[3]);
// tiles of a prolongation descriptor in TMA tile configuration `config`
long long tile_prolongation(Desc &d, int config);

// One plain per-box launch (cgx.cu).
int launch_one_pair(const Desc &d, int ntiles, int fp, int *status, cudaStream_t s);

// kernel launchers (cgx_kern_f0.cu, cgx_kern_f1.cu, cgx_kern_hi.cu)
int klaunch_pair_f0(const Desc &d, int ntiles, int *status, cudaStream_t s);
int klaunch_pair_f1(const Desc &d, int ntiles, int *status, cudaStream_t s);
int klaunch_pair_hi(int fp, const Desc &d, int ntiles, int *status, cudaStream_t s);
int klaunch_map_f0(const Desc *d, const int2 *tmap, long long ntiles, unsigned long long *counter,
                   int *status, cudaStream_t s);
int klaunch_map_f1(const Desc *d, const int2 *tmap, long long ntiles, unsigned long long *counter,
                   int *status, cudaStream_t s);
int klaunch_search_f0(const Desc *d, const long long *prefix, int ndesc, long long ntiles,
                      unsigned long long *counter, int *status, cudaStream_t s);
int klaunch_search_f1(const Desc *d, const long long *prefix, int ndesc, long long ntiles,
                      unsigned long long *counter, int *status, cudaStream_t s);

int klaunch_spair_f0(const Desc &d, int ntiles, int *status, cudaStream_t s);
int klaunch_spair_f1(const Desc &d, int ntiles, int *status, cudaStream_t s);
// TMA prolongation kernels: f<mode>_p0 families 0-4 (VC 1/3/5, CC 0/1),
// _p1 families 5-9 (CC 2-5, ENO), _c<k> tile configuration TMA_CFGS[k];
// variant = 4 * family + time variant
#define CGX_TMA_DECL(F, P, C)                                                                          \
  int klaunch_tma_f##F##_p##P##_c##C(int variant, const Desc *d, const CUtensorMap *maps,             \
                                     const int2 *tmap, long long ntiles, unsigned long long *counter, \
                                     int *status, cudaStream_t s);
#define CGX_TMA_DECL5(F, P) \
  CGX_TMA_DECL(F, P, 0) CGX_TMA_DECL(F, P, 1) CGX_TMA_DECL(F, P, 2) CGX_TMA_DECL(F, P, 3) CGX_TMA_DECL(F, P, 4)
CGX_TMA_DECL5(0, 0) CGX_TMA_DECL5(0, 1) CGX_TMA_DECL5(1, 0) CGX_TMA_DECL5(1, 1)
#undef CGX_TMA_DECL5
#undef CGX_TMA_DECL
int klaunch_stream_f0(int variant, const Desc *d, const int2 *tmap, long long ntiles,
                      unsigned long long *counter, int *status, cudaStream_t s);
int klaunch_stream_f1(int variant, const Desc *d, const int2 *tmap, long long ntiles,
                      unsigned long long *counter, int *status, cudaStream_t s);

// stencil (prolongation) kinds run in the shared-memory kernels, the others
// in the streaming kernels
inline bool is_stencil(int kind) {
  return kind == K_PROLONG_VC || kind == K_PROLONG_CC || kind == K_PROLONG_ENO ||
         kind == K_PROLONG_CC_ENO;
}
inline int segment_of(const Desc &d) {
  if (!is_stencil(d.kind)) return SEG_STREAM + stream_variant(d);
  const int v = d.bx ? tma_variant(d) : -1;
  return v >= 0 ? v : SEG_STENCIL;
}

// One entry of a chain's tile list (cgx_chain.cuh): descriptor, tile
// within it, the completion counter it increments, the counter it waits on
// (-1: none).
struct ChainTile {
  int desc, tile, own, dep;
};
// control words of a chain launch: claim counter, exit counter, abort word
constexpr int CHAIN_CTL_WORDS = 4;
// the chain kernel of a floating-point mode and vertex-centred order
// (cgx_kern_chain.cu)
int klaunch_chain(int fp, int order, const Desc *d, const CUtensorMap *maps, const ChainTile *tiles,
                  long long ntiles, const unsigned *need, unsigned *done, int ncounters,
                  unsigned long long *ctl, int *status, cudaStream_t s);

// CTAs per SM the persistent kernels of the launch in progress on this host
// thread may use (0: as many as fit), [0] the TMA prolongation kernels, [1]
// the streaming kernels; set by launch_map from the batch
// (cgx_batch_set_max_ctas), read by the launchers.  A cap below the
// occupancy limit leaves room on every SM for another stream's kernel.
extern thread_local int g_cta_cap[2];

int current_fp_mode();
int set_error(int code, const char *fmt, ...);
int cuda_error(cudaError_t e, const char *what);

} // namespace cgx
