/*
 * cgx.h -- C-ABI of the B200 grid-transfer library (libcgx.so).
 *
 * Drop-in for the per-box-pair entry point of CarpetLib's transfer path:
 * every grid function lives in device memory (HBM) of one GPU; the host
 * passes device pointers, boxes and operator parameters, and the library
 * launches hand-written sm_100a FP64 kernels.  No entry point aborts: each
 * returns CGX_OK or a CGX_E* status; cgx_last_error() gives the message.
 *
 * Conventions shared with CarpetLib:
 *   boxes   int[9] = {lower[3], upper[3], stride[3]}, inclusive bounds in the
 *           global integer index space (bbox<int,3>, CarpetLib/src/bbox.hh:34-70;
 *           the int[3][3] layout CarpetLib passes to Fortran, data.cc:212-214);
 *   arrays  x-fastest, element (i,j,k) at i + padext[0]*(j + padext[1]*k)
 *           (index3, CarpetLib/src/operator_prototypes_3d.hh:17-28); the logical
 *           extent of an array is its bbox, padext[d] >= bbox size;
 *   op      operator_type values of CarpetLib/src/operators.hh:8-25;
 *   cent    centering values of CarpetLib/src/defs.hh:134.
 */
#ifndef CGX_H
#define CGX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define CGX_OK 0
#define CGX_EINVAL 1       /* inconsistent boxes/strides/times (CarpetLib aborts) */
#define CGX_EUNSUPPORTED 2 /* operator/order not provided on the GPU */
#define CGX_ENOMEM 3
#define CGX_ECUDA 4        /* a CUDA runtime call failed */
#define CGX_EDEVICE 5      /* a kernel reported a bad descriptor */

/* operator_type, CarpetLib/src/operators.hh:8-25 */
#define CGX_OP_ERROR 0
#define CGX_OP_NONE 1
#define CGX_OP_SYNC 2
#define CGX_OP_RESTRICT 3
#define CGX_OP_COPY 4
#define CGX_OP_LAGRANGE 5
#define CGX_OP_ENO 6
#define CGX_OP_WENO 7
#define CGX_OP_TVD 8
#define CGX_OP_LAGRANGE_MONOTONE 9

/* centering, CarpetLib/src/defs.hh:134 */
#define CGX_VERTEX 1
#define CGX_CELL 2

/* floating-point modes of the stencil arithmetic */
#define CGX_FP_EXACT 0 /* reference operation order, two roundings per
                          multiply-add: bit-exact with CarpetLib built
                          without contraction */
#define CGX_FP_FMA 1   /* same order, every multiply-add fused */

/* One device array of a grid function: one component at one timelevel.
 * Mirrors what data<T> hands its operators: storage(), padded_shape(),
 * extent() (CarpetLib/src/data.cc:610-614). */
typedef struct cgx_array {
  double *data;  /* device pointer */
  int padext[3]; /* padded extent (x, y, z) in elements */
  int bbox[9];   /* logical extent {lower[3], upper[3], stride[3]} */
} cgx_array;

/* Library state: floating-point mode and the default device. */
int cgx_init(int device, int fp_mode);
int cgx_set_fp_mode(int fp_mode);
/* CarpetLib's use_higher_order_restriction and restriction_order_space
 * parameters (CarpetLib/param.ccl; data.cc:1061-1097): with the first set,
 * cell-centred restriction of a non-ENO/WENO operator uses
 * restrict_3d_cc_o3_rf2 (order 3) or restrict_3d_cc_o5_rf2 (order 5);
 * order 1 keeps restrict_3d_cc_rf2, any other order makes such transfers
 * fail with CGX_EINVAL.  Process-wide; default off. */
int cgx_set_restriction(int use_higher_order, int order);
const char *cgx_last_error(void);
const char *cgx_version(void);

/*
 * cgx_transfer -- the plain per-box form: one box-pair of
 *   gdata::transfer_data(dst, state, srcs, times, dstbox, srcbox, slabinfo,
 *                        dstproc, srcproc, time, order_space, order_time)
 * (CarpetLib/src/gdata.hh:186-191, gdata.cc:124-286) on one process, i.e.
 *   data<T>::transfer_from_innerloop (CarpetLib/src/data.cc:464-483).
 * Same timelevel selection (gdata::find_source_timelevel, gdata.cc:288-349),
 * same stride dispatch (transfer_p_r, data.cc:537-556), same operator tables
 * (transfer_prolongate data.cc:573-725, transfer_restrict data.cc:1030-1135,
 * time_interpolate data.cc:1183-1299), same argument checks as status codes.
 * The spatial operator and the time interpolation run fused in one kernel,
 * in the reference's order (space per timelevel, then time), for copies and
 * prolongations with up to 3 timelevels.  Restriction between timelevels and
 * 4 or 5 timelevels (interpolate_3d_4tl / 5tl) run the reference's two
 * stages: per-timelevel temporaries (stream-ordered allocation), then the
 * time combination.
 * Operators: vertex-centred Lagrange 1-11, cell-centred Lagrange 0-5,
 * vertex-centred ENO 3/5 and WENO 5 (the ENO operator), cell-centred ENO 2-5,
 * Lagrange_monotone 5, injection, cell-centred restriction (orders 1/3/5 by
 * cgx_set_restriction), copy with slab offset; other operators return
 * CGX_EUNSUPPORTED.
 *   srcs[nsrc], times[nsrc]: source timelevels (same padext/bbox each);
 *   slab_offset: NULL or int[3], the islab offset of copy_3d (copy_3d.cc:57);
 *   stream: a cudaStream_t (NULL = default stream).
 * Asynchronous: returns after the launch.
 */
int cgx_transfer(int op, int cent, const cgx_array *dst, const cgx_array *srcs,
                 const double *times, int nsrc, const int dstbox[9],
                 const int srcbox[9], const int *slab_offset, double time,
                 int order_space, int order_time, void *stream);

/* gdata::copy_data (CarpetLib/src/gdata.cc:110-122): transfer_data with
 * order_space = (cent == vertex ? 1 : 0), order_time = 0, time 0. */
int cgx_copy(int op, int cent, const cgx_array *dst, const cgx_array *src,
             const int dstbox[9], const int srcbox[9], const int *slab_offset,
             void *stream);

/* The timelevel selection alone (gdata::find_source_timelevel). */
int cgx_find_source_timelevel(const double *times, int ntimes, double time,
                              int order_time, int op, int *timelevel0,
                              int *ntimelevels);

/*
 * Batched form: many box-pairs -- of one refinement level or of several
 * hierarchies, uneven sizes, mixed operators -- validated once on the host
 * into flat descriptors, then run by one persistent kernel that takes tiles
 * from a device work queue.  Replaces the loop of ggf::transfer_from_all
 * (CarpetLib/src/ggf.cc:500-591) over a sendrecv_pseudoregion list.
 */
typedef struct cgx_batch cgx_batch;
int cgx_batch_create(cgx_batch **out);
int cgx_batch_destroy(cgx_batch *b);
int cgx_batch_clear(cgx_batch *b);
/* same arguments and checks as cgx_transfer; appends one box-pair */
int cgx_batch_add(cgx_batch *b, int op, int cent, const cgx_array *dst,
                  const cgx_array *srcs, const double *times, int nsrc,
                  const int dstbox[9], const int srcbox[9],
                  const int *slab_offset, double time, int order_space,
                  int order_time);
/* many box-pairs at once (no counterpart in the reference: the loop of
 * ggf::transfer_from_all, CarpetLib/src/ggf.cc:500-591, over a pair list,
 * in one call): pair i writes arrays[dst_idx[i]] in dstboxes[9i..] from the
 * nsrc arrays arrays[src_idx[nsrc*i + t]] in srcboxes[9i..]; every pair
 * shares op, cent, times, time and the orders.  Stops at the first invalid
 * pair (the ones before it stay added). */
int cgx_batch_add_many(cgx_batch *b, int op, int cent, const cgx_array *arrays, int npairs,
                       const int *dst_idx, const int *src_idx, int nsrc, const double *times,
                       const int *dstboxes, const int *srcboxes, double time, int order_space,
                       int order_time);
/* number of box-pairs, tiles and algorithmic bytes (reads + writes) */
int cgx_batch_stats(const cgx_batch *b, int64_t *npairs, int64_t *ntiles,
                    int64_t *dst_points, int64_t *bytes);
/* copy descriptors to the device (once per schedule; graph-safe after) */
int cgx_batch_upload(cgx_batch *b, void *stream);
/* the uploaded box-pairs, one persistent kernel per kind of tile (a
 * homogeneous batch -- one operator, order and timelevel count -- is one
 * kernel).  Several kernels run concurrently on streams the batch owns,
 * forked from and joined back into `stream` (also inside a capture); the
 * time combination of staged transfers runs last, on `stream`.  Work issued
 * on `stream` after the call waits for all of it. */
int cgx_batch_launch(cgx_batch *b, void *stream);
/* kernels one cgx_batch_launch issues for the current upload (no
 * counterpart in the reference: a measurement aid) */
int cgx_batch_kernels(const cgx_batch *b, int *nkernels);
/* Tile-shape autotuner (no counterpart in the reference): uploads the
 * batch, times every prolongation variant it holds in each of the library's
 * tile configurations (reps launches each, on the caller's arrays -- the
 * results written are those of a normal launch) and keeps the fastest.
 * chosen (nullable) receives CGX_TMA_VARIANTS entries: the configuration
 * index per variant, -1 where the batch has none.  Synchronises stream. */
#define CGX_TMA_VARIANTS 40
#define CGX_TMA_CONFIGS 5
int cgx_batch_autotune(cgx_batch *b, int reps, void *stream, int *chosen);
/* pin the tile configuration (0 .. CGX_TMA_CONFIGS-1) of one prolongation
 * variant, or of all with variant = -1 (e.g. a saved autotune result);
 * takes effect at the next cgx_batch_upload */
int cgx_batch_set_config(cgx_batch *b, int variant, int config);
/* CTAs per SM that the batch's persistent kernels may use: tma_per_sm for
 * the TMA prolongation kernels, stream_per_sm for the streaming (copy,
 * restriction) kernels; 0 = as many as fit (the default).  Below the
 * occupancy limit, a batch leaves room on every SM for a kernel on another
 * stream (the grid functions of another group), so that a compute-bound
 * prolongation and a memory-bound sync can run on the same SMs at once.
 * Takes effect at the next launch.  No counterpart in the reference. */
int cgx_batch_set_max_ctas(cgx_batch *b, int tma_per_sm, int stream_per_sm);
/* plain per-box launches of the same descriptors (one kernel per pair) */
int cgx_batch_launch_per_box(cgx_batch *b, void *stream);
/* ---- host schedules: the send/recv region lists of dh (CarpetLib/src/
 * dh.cc) for box hierarchies.  Components are given by their interior (the
 * component's share of its level) and exterior (grown by the ghost zones)
 * boxes, int[9] each; refined levels by their boxes.  Each call writes up to
 * max pairs and sets *npairs to the number the schedule has (CGX_ENOMEM when
 * that is more than max: call again with room for *npairs). */
typedef struct cgx_pair_box {
  int dst_comp, src_comp;
  int dstbox[9], srcbox[9];
} cgx_pair_box;
/* ghost sync within a level, dh.cc:837-894 */
int cgx_sched_sync(int ncomp, const int *interior, const int *exterior, cgx_pair_box *out, int max,
                   int *npairs);
/* boundary prolongation of the fine boxes' outer ghost+buffer layers from
 * the coarse components, send boxes grown by order/2, dh.cc:896-977 */
int cgx_sched_prolong(int nbox, const int *fboxes, int nfcomp, const int *finterior, int nccomp,
                      const int *cinterior, const int *cexterior, int ghost, int buffer, int order,
                      cgx_pair_box *out, int max, int *npairs);
/* restriction of the coarse points under the fine boxes' active regions,
 * dh.cc:981-1088 (dst: coarse component, src: fine component) */
int cgx_sched_restrict(int nbox, const int *fboxes, int nfcomp, const int *finterior, int nccomp,
                       const int *cinterior, int ghost, int buffer, cgx_pair_box *out, int max,
                       int *npairs);
/* regrid fill of one refined level, dh.cc:1717-1830: copies from the old
 * components' interiors, prolongation from the coarse components for the
 * rest of every new component's exterior */
int cgx_sched_old2new(int nnew, const int *new_exterior, int nold, const int *old_interior, int nccomp,
                      const int *cinterior, const int *cexterior, int order, cgx_pair_box *copies,
                      int max_copies, int *ncopies, cgx_pair_box *prols, int max_prols, int *nprols);

/*
 * The dh schedule producer for arbitrary component sets: the region algebra
 * of dh::regrid (CarpetLib/src/dh.cc:300-1088) for vertex-centred
 * hierarchies with refinement factor 2.  Input per level l: its domain
 * (h.baseextent: the whole domain at the level's stride, domains[9 l ..])
 * and its ncomps[l] component interiors (disjoint boxes, consecutive in
 * interiors[]).  Each component's exterior is its interior grown by `ghost`
 * on faces off the domain boundary; boundary_width points of the domain
 * boundary are outer boundary; buffer zones are the owned points within
 * `buffer` of the level's not-owned region.  Schedules (cgx_dh_pairs):
 *   CGX_DH_SYNC     level l's ghost zones from its other components'
 *                   interiors (dh.cc:837-894);
 *   CGX_DH_BNDPROL  what sync leaves, and the buffer zones, of level l from
 *                   level l-1, send boxes grown by order/2 (dh.cc:896-977);
 *   CGX_DH_RESTRICT the points of level l under level l+1's active region
 *                   from level l+1, into every component's exterior
 *                   (restrict_into_ghosts, CarpetLib's default) or interior
 *                   (dh.cc:981-1088).
 * Every point is received once, from the component the reference's order
 * picks; the reference's consistency checks return CGX_EINVAL.
 */
#define CGX_DH_SYNC 0
#define CGX_DH_BNDPROL 1
#define CGX_DH_RESTRICT 2
typedef struct cgx_dh cgx_dh;
int cgx_dh_create(cgx_dh **out, int nlevels, const int *domains, const int *ncomps, const int *interiors,
                  int ghost, int buffer, int boundary_width, int order, int restrict_into_ghosts);
int cgx_dh_destroy(cgx_dh *h);
/* the ncomps[level] component exteriors, 9 ints each */
int cgx_dh_exteriors(const cgx_dh *h, int level, int *out);
/* a schedule of `level`; *n is its length (CGX_EINVAL when above max) */
int cgx_dh_pairs(const cgx_dh *h, int level, int kind, cgx_pair_box *out, int max, int *n);

/* device status word of the last launches: 0 or a CGX_E* code */
int cgx_batch_check(cgx_batch *b, void *stream);

/*
 * CUDA graphs: capture a sequence of batch launches (a Berger-Oliger
 * substep) once and replay it.  Begin/end bracket ordinary calls on
 * `stream`.
 */
typedef struct cgx_graph cgx_graph;
int cgx_graph_begin(void *stream);
int cgx_graph_end(void *stream, cgx_graph **out);
int cgx_graph_launch(cgx_graph *g, void *stream);
int cgx_graph_destroy(cgx_graph *g);

/*
 * Served form: transfer requests from many independent AMR hierarchies.
 * NO COUNTERPART IN THE REFERENCE (Carpet runs one hierarchy per job); the
 * operations served are the reference's (sync, boundary prolongation,
 * restriction of one level), each defined once from a cgx_batch holding its
 * box-pairs; its descriptors and tensor maps are uploaded once into a
 * device pool.  A worker thread continuously batches pending requests -- the
 * oldest of every hierarchy, one per hierarchy per launch -- into the
 * persistent kernels on four launch slots; a hierarchy's requests run one
 * after another in arrival order (a launch that takes a hierarchy still in
 * flight on another slot waits for that slot on the device, so the host
 * prepares the next launches while the GPU runs the earlier ones).
 * CGX_SERVE_PLAIN serves one request at a time through per-box launches
 * (the baseline).  max_pairs is the descriptor pool's initial capacity (it
 * grows as operations are defined), max_tiles a launch's tile capacity.
 * Hierarchies are admitted
 * against an HBM budget with cgx_server_admit/release; admission, release
 * and cgx_server_define_op are allowed while the worker runs, so that a
 * hierarchy admitted mid-stream is served from its first request on.  A
 * launch's segments (prolongation, copy, restriction kernels) run
 * concurrently on side streams of the slot.  The report's bytes are the
 * algorithmic bytes of the completed requests.
 */
#define CGX_SERVE_BATCHED 0
#define CGX_SERVE_PLAIN 1
typedef struct cgx_server cgx_server;
typedef struct cgx_server_report {
  int64_t requests, launches, fine_points, hbm_used;
  double p50_ms, p99_ms, mean_ms, makespan_s, points_per_s, mean_batch;
  int64_t bytes;      /* algorithmic bytes of the completed requests */
  double bytes_per_s; /* bytes / makespan */
} cgx_server_report;
int cgx_server_create(cgx_server **out, int mode, int64_t hbm_budget_bytes,
                      int max_pairs, int64_t max_tiles, int64_t max_requests);
int cgx_server_destroy(cgx_server *s);
int cgx_server_admit(cgx_server *s, int64_t bytes);   /* CGX_ENOMEM if over budget */
int cgx_server_release(cgx_server *s, int64_t bytes);
int cgx_server_define_op(cgx_server *s, int hier, const cgx_batch *pairs, int *op_id);
/* tile configuration of a TMA prolongation variant (-1: all), as
 * cgx_batch_set_config; applies to operations defined after the call */
int cgx_server_set_config(cgx_server *s, int variant, int config);
int cgx_server_start(cgx_server *s);
int cgx_server_submit(cgx_server *s, int op_id, int64_t *request_id);
/* submit op_ids[i] at arrival_s[i] seconds after the call (a load replay) */
int cgx_server_replay(cgx_server *s, const int *op_ids, const double *arrival_s, int n);
/* wait until every submitted request is done; returns the worker's first
 * error, with its message: CGX_EDEVICE when a served launch's kernels gave up
 * a bounded device wait (each launch's status is read back when its slot
 * retires), a launch error otherwise */
int cgx_server_drain(cgx_server *s);
int cgx_server_stats(cgx_server *s, cgx_server_report *rep);
int cgx_server_latencies(cgx_server *s, double *out_ms, int64_t n);

/*
 * Chain form: a sequence of batches as ONE persistent launch.  NO
 * COUNTERPART IN THE REFERENCE, which makes the same transfers one call at a
 * time (the phases of a Berger-Oliger step: Carpet/src/Evolve.cc:44-121).
 *
 * cgx_batch_set_group(b, g) tags the pairs added to b afterwards with the
 * dependency group g (default 0): pairs of different groups must touch
 * disjoint arrays throughout the chain -- one grid function per group, say.
 * cgx_chain_add appends batches in call order; cgx_chain_upload builds one
 * tile list over all of them.  In the launch, a tile of batch j and group g
 * starts once every tile of the latest earlier batch with pairs of group g
 * has completed, so each group sees the batches in order while the groups'
 * tiles of different batches share the GPU.  The result equals running the
 * batches one after another (bit for bit).  Accepted pairs: vertex-centred
 * Lagrange prolongation of one order (1, 3 or 5) with one timelevel or
 * quadratic time interpolation over three, on arrays TMA can stage (16-byte
 * aligned base, even row and plane pitch); one-timelevel copies; injection.
 * Anything else returns CGX_EUNSUPPORTED at upload.  The floating-point mode
 * is the one current at upload.  The batches must stay alive and unchanged
 * while the chain is used; cgx_chain_upload reads them, the launch does not.
 * Every device wait is bounded; cgx_chain_check reports CGX_EDEVICE if one
 * gave up.  Capturable in a CUDA graph.
 */
typedef struct cgx_chain cgx_chain;
int cgx_batch_set_group(cgx_batch *b, int group);
int cgx_chain_create(cgx_chain **out);
int cgx_chain_destroy(cgx_chain *c);
int cgx_chain_add(cgx_chain *c, cgx_batch *b);
int cgx_chain_upload(cgx_chain *c, void *stream);
int cgx_chain_launch(cgx_chain *c, void *stream);
int cgx_chain_check(cgx_chain *c, void *stream);
int cgx_chain_stats(const cgx_chain *c, int64_t *npairs, int64_t *ntiles, int64_t *dst_points,
                    int64_t *bytes);

/*
 * Failure injection, for the tests of the bounded device waits.  NO
 * COUNTERPART IN THE REFERENCE.  Every wait of the kernels on a device event
 * (a TMA copy landing on its mbarrier, a chain tile's dependency counter)
 * gives up after about 2^31 clock cycles (a second), records CGX_EDEVICE in
 * the launch's status word and lets the launch drain, so that the context
 * stays usable; the batch / chain check then reports CGX_EDEVICE.
 *   cgx_debug_skip_tma_plane(1): the TMA prolongation kernels launched from
 *     now on never stage the first plane of each CTA's first tile, so that
 *     the wait for it runs out (0 restores normal operation);
 *   cgx_chain_debug_hold(c, 1): the next cgx_chain_upload of c requires one
 *     more completed tile of every counter than exists, so that every
 *     dependency wait runs out (0 and a new upload restore it).
 * Off by default; process-wide (the first) or per chain (the second).
 */
int cgx_debug_skip_tma_plane(int enable);
int cgx_chain_debug_hold(cgx_chain *c, int hold);

/*
 * No-allocation form.  NO COUNTERPART IN THE REFERENCE: CarpetLib has no
 * device path at all; this entry point exists for callers of this library
 * that must not allocate device memory -- code that runs while a CUDA graph
 * is being captured elsewhere in the process, hosts that reserve all device
 * memory for their own pool, or time-critical loops that cannot afford the
 * device-wide synchronisation cudaMalloc/cudaFree imply.
 *
 * Runs up to CGX_NOALLOC_MAX_PAIRS box-pairs (same meaning and checks as
 * cgx_transfer; at most 3 source timelevels each; vertex-centred orders
 * 7/9/11 are not available here) through the persistent kernel.  Its
 * scratch -- descriptors, tile offsets, work counter -- is one fixed array
 * of under 0.5 MiB (room for CGX_NOALLOC_MAX_PAIRS descriptors) inside the
 * library's device image, which every GPU that loads the library holds until
 * the process exits; nothing is allocated.
 * The first call on a device looks up that array's device address.  The
 * descriptors are copied from host memory that the call does not keep, so a
 * call made while its stream is being captured returns CGX_EUNSUPPORTED.
 * All calls share the one array: calls whose kernels overlap on the GPU
 * (other streams, or other host threads) race and must be serialised by the
 * caller.  Returns CGX_EINVAL for more than CGX_NOALLOC_MAX_PAIRS pairs.
 * Asynchronous; cgx_noalloc_check reads the kernel's status afterwards.
 */
#define CGX_NOALLOC_MAX_PAIRS 2048
typedef struct cgx_pair {
  int op, cent;
  cgx_array dst;
  cgx_array srcs[3];
  double times[3];
  int nsrc;
  int dstbox[9], srcbox[9];
  int has_slab;
  int slab_offset[3];
  double time;
  int order_space, order_time;
} cgx_pair;
int cgx_transfer_pairs_noalloc(const cgx_pair *pairs, int npairs, void *stream);
/* Waits for the stream and returns the status the last
 * cgx_transfer_pairs_noalloc kernel on the current device left in the fixed
 * scratch: CGX_OK, or CGX_EDEVICE when a bounded device wait gave up.
 * Allocates nothing.  No counterpart in the reference (part of the
 * no-allocation form above). */
int cgx_noalloc_check(void *stream);

/* device memory helpers for callers without their own allocator */
int cgx_malloc(void **ptr, size_t bytes);
int cgx_free(void *ptr);
int cgx_memcpy_htod(void *dst, const void *src, size_t bytes, void *stream);
int cgx_memcpy_dtoh(void *dst, const void *src, size_t bytes, void *stream);
int cgx_stream_sync(void *stream);

#ifdef __cplusplus
}
#endif
#endif /* CGX_H */
