// cgx_server.cu -- the served form: transfer requests from many independent
// AMR hierarchies, continuously batched into the persistent kernel.
//
// A request names an operation template -- the box-pairs of one transfer
// (a sync, a boundary prolongation or a restriction of one level of one
// hierarchy, over all of its grid functions) -- defined once from a
// cgx_batch.  An operation's descriptors and tensor maps are uploaded once,
// into a device pool that every launch reads, and its tiles are kept as
// (pool descriptor, tile) entries by segment; a launch only concatenates
// those entries into one tile map.  The worker thread keeps several launch
// slots.  Whenever a slot is free it takes, in arrival order, the oldest
// pending request of every hierarchy (one request per hierarchy per launch)
// and launches the persistent kernels on that slot's stream.  A hierarchy
// whose previous request is still in flight on another slot may be taken:
// the slot's stream then waits for that slot's completion event before its
// kernels, so each hierarchy sees its requests applied one after another in
// arrival order -- the results are those of running them alone
// (tests/test_gpu_serving.py) -- while the host prepares the next launches
// as the device runs the earlier ones.
//
// The plain mode serves the same stream through the per-box drop-in: one
// request at a time, one kernel launch per box-pair.
//
// Hierarchies are admitted against an HBM budget (cgx_server_admit /
// cgx_server_release account the device memory their grid functions use),
// also while the worker runs: operations of a newly admitted hierarchy can be
// defined at any time, and its requests join the stream from then on.
//
// A slot launches the concatenated requests' segments (prolongation kinds,
// copies, restrictions) concurrently: each non-empty segment but the last on
// a side stream of the slot, forked from and joined back into the slot's
// stream, so that a mixed launch's kernels share the GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cgx.h"
#include "cgx_internal.h"

using namespace cgx;

namespace {

using clk = std::chrono::steady_clock;

// launch slots of the batched mode: with several, the host prepares the next
// launches while the device runs earlier ones (a launch that takes a
// hierarchy in flight on another slot waits for that slot on the device)
constexpr int SERVER_SLOTS = 4;

struct OpTemplate {
  int hier;
  std::vector<Desc> descs; // host copies: the plain mode's per-box launches
  std::vector<int> ntiles;
  long long tiles = 0, points = 0, bytes = 0;
  // the operation's tiles by tile-map segment, (descriptor in the server's
  // device pool, tile): a launch concatenates these
  std::vector<int2> seg_tiles[NSEG];
};

struct Request {
  int op;
  double t_arrive = 0, t_launch = 0, t_done = 0; // seconds since the server epoch
};

struct Slot {
  cudaStream_t stream = nullptr;
  // done: the launch's kernels have finished (later launches of the same
  // hierarchies wait for it on the device); fin: its status has also been
  // read back (the worker retires the slot on it, sleeping if it must)
  cudaEvent_t done = nullptr, fin = nullptr;
  // the concurrent segment launch: side streams, fork and join events
  cudaStream_t side[CONCURRENT_SIDE_MAX] = {};
  cudaEvent_t ev[CONCURRENT_SIDE_MAX + 1] = {};
  int2 *d_tmap = nullptr, *h_tmap = nullptr;
  unsigned long long *d_counter = nullptr;
  // the launch's device status (a bounded wait that gave up: CGX_EDEVICE),
  // zeroed before the kernels and copied to pinned memory after them; the
  // worker reads it when it retires the slot
  int *d_status = nullptr, *h_status = nullptr;
  size_t tile_cap = 0;
  bool busy = false;
  std::vector<int> reqs;
  long long seq = 0; // launch order of the slot's current work
};

// Every operation's descriptors and tensor maps (3 per descriptor), in
// device memory for the server's lifetime.  Growing the pool copies it into
// a larger allocation; the old one stays allocated (launches in flight read
// it) until the server is destroyed.
struct Pool {
  Desc *descs = nullptr;
  CUtensorMap *maps = nullptr;
  size_t used = 0, cap = 0;
  std::vector<void *> old; // superseded allocations
};

} // namespace

struct cgx_server {
  int mode = CGX_SERVE_BATCHED;
  int fp = CGX_FP_EXACT;
  long long budget = 0, used = 0;
  // operations: appended under mu (also while the worker runs); a deque
  // keeps the address of every element, which the worker uses after
  // releasing the lock
  std::deque<OpTemplate> ops;
  std::vector<Request> reqs; // reserved at creation: never reallocated
  size_t max_requests = 0;
  // per hierarchy: the slot of its latest launched request while that is
  // in flight, else -1
  std::vector<signed char> hier_last;
  std::deque<int> pending;
  Pool pool;             // grows under define_mu, read by the worker under mu
  std::mutex define_mu;  // serialises cgx_server_define_op
  // the pool's uploads and copies, each waited for before the pool or the
  // operation is published
  cudaStream_t upload = nullptr;
  // tile configuration per TMA prolongation variant (cgx_server_set_config),
  // applied to operations defined afterwards
  int tma_cfg[TV_COUNT] = {};
  std::mutex mu;
  std::condition_variable cv;
  std::thread worker;
  std::atomic<bool> stop{false};
  std::atomic<long long> completed{0};
  long long submitted = 0;
  Slot slots[SERVER_SLOTS];
  clk::time_point epoch = clk::now();
  long long launches = 0, batched_requests = 0;
  // the worker's first error and its message, which drain() reports in the
  // caller's thread (under err_mu; taken after mu where both are held)
  int error = CGX_OK;
  std::string error_msg;
  std::mutex err_mu;

  double now() const { return std::chrono::duration<double>(clk::now() - epoch).count(); }
};

namespace {

// Records the worker's first error: a status code whose message the calling
// thread has just set (cgx_last_error is per thread).
void note_error(cgx_server *sv, int rc) {
  if (rc == CGX_OK) return;
  std::lock_guard<std::mutex> g(sv->err_mu);
  if (sv->error != CGX_OK) return;
  sv->error = rc;
  sv->error_msg = cgx_last_error();
}

int slot_init(Slot &s, size_t tile_cap) {
  cudaError_t e = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
  // blocking sync: a worker that waits on it sleeps instead of spinning
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.fin, cudaEventDisableTiming | cudaEventBlockingSync);
  if (e == cudaSuccess) e = cudaMalloc(&s.d_tmap, tile_cap * sizeof(int2));
  if (e == cudaSuccess) e = cudaMallocHost(&s.h_tmap, tile_cap * sizeof(int2));
  // claim counters and exit counts (cgx_kernels.cuh, claims_done)
  if (e == cudaSuccess) e = cudaMalloc(&s.d_counter, 2 * NSEG * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(s.d_counter, 0, 2 * NSEG * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&s.d_status, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(s.d_status, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMallocHost(&s.h_status, sizeof(int));
  if (e == cudaSuccess) *s.h_status = 0;
  for (int k = 0; k < CONCURRENT_SIDE_MAX && e == cudaSuccess; ++k)
    e = cudaStreamCreateWithFlags(&s.side[k], cudaStreamNonBlocking);
  for (int k = 0; k <= CONCURRENT_SIDE_MAX && e == cudaSuccess; ++k)
    e = cudaEventCreateWithFlags(&s.ev[k], cudaEventDisableTiming);
  if (e != cudaSuccess) return cuda_error(e, "server slot allocation");
  s.tile_cap = tile_cap;
  return CGX_OK;
}

// The descriptor pool with room for at least `need` descriptors (called
// under define_mu; publishes a new pool under mu).
int pool_reserve(cgx_server *sv, size_t need) {
  Pool &p = sv->pool;
  if (need <= p.cap) return CGX_OK;
  const size_t cap = p.cap ? std::max<size_t>(2 * p.cap, need) : need;
  Desc *d = nullptr;
  CUtensorMap *m = nullptr;
  cudaError_t e = cudaMalloc(&d, cap * sizeof(Desc));
  if (e == cudaSuccess) e = cudaMalloc(&m, 3 * cap * sizeof(CUtensorMap));
  if (e == cudaSuccess && p.used)
    e = cudaMemcpyAsync(d, p.descs, p.used * sizeof(Desc), cudaMemcpyDeviceToDevice, sv->upload);
  if (e == cudaSuccess && p.used)
    e = cudaMemcpyAsync(m, p.maps, 3 * p.used * sizeof(CUtensorMap), cudaMemcpyDeviceToDevice, sv->upload);
  // a device-to-device copy returns before it completes: wait for it
  if (e == cudaSuccess) e = cudaStreamSynchronize(sv->upload);
  if (e != cudaSuccess) {
    cudaFree(d);
    cudaFree(m);
    return cuda_error(e, "server descriptor pool");
  }
  std::lock_guard<std::mutex> g(sv->mu);
  if (p.descs) {
    p.old.push_back(p.descs);
    p.old.push_back(p.maps);
  }
  p.descs = d;
  p.maps = m;
  p.cap = cap;
  return CGX_OK;
}

void pool_free(Pool &p) {
  cudaFree(p.descs);
  cudaFree(p.maps);
  for (void *x : p.old) cudaFree(x);
  p = Pool();
}

void slot_free(Slot &s) {
  if (s.stream) cudaStreamSynchronize(s.stream);
  cudaFree(s.d_tmap);
  cudaFreeHost(s.h_tmap);
  cudaFree(s.d_counter);
  cudaFree(s.d_status);
  cudaFreeHost(s.h_status);
  if (s.done) cudaEventDestroy(s.done);
  if (s.fin) cudaEventDestroy(s.fin);
  for (cudaStream_t x : s.side)
    if (x) cudaStreamDestroy(x);
  for (cudaEvent_t x : s.ev)
    if (x) cudaEventDestroy(x);
  if (s.stream) cudaStreamDestroy(s.stream);
  s = Slot();
}

// Retire a slot whose kernel has finished.
void retire(cgx_server *sv, int slot) {
  Slot &s = sv->slots[slot];
  const double t = sv->now();
  std::lock_guard<std::mutex> g(sv->mu);
  if (*s.h_status != CGX_OK) {
    // a kernel of this launch gave up a bounded wait: its requests' results
    // are not valid; drain() reports it
    note_error(sv, set_error(CGX_EDEVICE, "served launch %lld: a device wait ran out (status %d)", s.seq,
                             *s.h_status));
    *s.h_status = CGX_OK;
  }
  for (int r : s.reqs) {
    sv->reqs[r].t_done = t;
    signed char &last = sv->hier_last[sv->ops[sv->reqs[r].op].hier];
    if (last == slot) last = -1; // no later launch took this hierarchy
  }
  sv->completed += (long long)s.reqs.size();
  s.reqs.clear();
  s.busy = false;
  sv->cv.notify_all();
}

// Batched mode: take, in arrival order, the oldest pending request of every
// hierarchy (one per hierarchy per launch) that fits the slot, and launch
// them together.  A hierarchy whose previous request is in flight on another
// slot makes this slot's stream wait for that slot's completion.
bool launch_batch(cgx_server *sv, int slot) {
  Slot &s = sv->slots[slot];
  std::vector<int> take;
  std::vector<const OpTemplate *> tops; // the taken requests' operations
  size_t ntiles = 0;
  bool wait_for[SERVER_SLOTS] = {};
  const Desc *pdescs;
  const CUtensorMap *pmaps;
  {
    std::lock_guard<std::mutex> g(sv->mu);
    pdescs = sv->pool.descs;
    pmaps = sv->pool.maps;
    std::vector<char> seen(sv->hier_last.size(), 0);
    for (auto it = sv->pending.begin(); it != sv->pending.end();) {
      const OpTemplate &op = sv->ops[sv->reqs[*it].op];
      if (seen[op.hier]) { // keep this hierarchy's later requests behind it
        ++it;
        continue;
      }
      seen[op.hier] = 1;
      if (ntiles + (size_t)op.tiles > s.tile_cap) {
        if (take.empty()) { // larger than a slot (define_op rejects these): drop it
          note_error(sv, set_error(CGX_EINVAL, "request larger than a server slot"));
          sv->reqs[*it].t_done = -1.0;
          sv->completed += 1;
          it = sv->pending.erase(it);
          continue;
        }
        ++it;
        continue;
      }
      take.push_back(*it);
      tops.push_back(&op);
      ntiles += (size_t)op.tiles;
      signed char &last = sv->hier_last[op.hier];
      if (last >= 0) wait_for[last] = true;
      last = (signed char)slot;
      it = sv->pending.erase(it);
    }
  }
  if (take.empty()) return false;
  // the tile map, segment by segment (prolongation tiles of all requests,
  // then each streaming variant's), one persistent kernel per segment; the
  // entries already name pool descriptors
  size_t ti = 0;
  long long seg[NSEG + 1];
  for (int g = 0; g < NSEG; ++g) {
    seg[g] = (long long)ti;
    for (const OpTemplate *op : tops) {
      const std::vector<int2> &v = op->seg_tiles[g];
      if (!v.empty()) memcpy(s.h_tmap + ti, v.data(), v.size() * sizeof(int2));
      ti += v.size();
    }
  }
  seg[NSEG] = (long long)ti;
  const double t = sv->now();
  for (int r : take) sv->reqs[r].t_launch = t;
  // the slot's own uploads and resets first, then the waits for the slots
  // that hold these hierarchies' previous requests: only the kernels sit
  // behind those on the device
  cudaError_t e = cudaMemcpyAsync(s.d_tmap, s.h_tmap, ti * sizeof(int2), cudaMemcpyHostToDevice, s.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(s.d_status, 0, sizeof(int), s.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(s.d_counter, 0, NSEG * sizeof(unsigned long long), s.stream);
  for (int k = 0; k < SERVER_SLOTS && e == cudaSuccess; ++k)
    if (wait_for[k]) e = cudaStreamWaitEvent(s.stream, sv->slots[k].done, 0);
  int rc = e == cudaSuccess ? CGX_OK : cuda_error(e, "server slot upload");
  if (rc == CGX_OK && seg[NSEG] > 0) {
    int need = 0;
    rc = launch_map_concurrent(sv->fp, pdescs, pmaps, s.d_tmap, seg, sv->tma_cfg, s.d_counter, s.d_status,
                               s.stream, s.side, s.ev, CONCURRENT_SIDE_MAX, &need);
  }
  note_error(sv, rc);
  e = cudaEventRecord(s.done, s.stream);
  if (e != cudaSuccess) note_error(sv, cuda_error(e, "cudaEventRecord"));
  e = cudaMemcpyAsync(s.h_status, s.d_status, sizeof(int), cudaMemcpyDeviceToHost, s.stream);
  if (e != cudaSuccess) note_error(sv, cuda_error(e, "server status read-back"));
  e = cudaEventRecord(s.fin, s.stream);
  if (e != cudaSuccess) note_error(sv, cuda_error(e, "cudaEventRecord"));
  s.reqs = take;
  s.busy = true;
  s.seq = sv->launches;
  sv->launches++;
  sv->batched_requests += (long long)take.size();
  return true;
}

// Plain mode: one request, one launch per box-pair, in arrival order.
bool launch_plain(cgx_server *sv, Slot &s) {
  int r;
  const OpTemplate *opp;
  {
    std::lock_guard<std::mutex> g(sv->mu);
    if (sv->pending.empty()) return false;
    r = sv->pending.front();
    sv->pending.pop_front();
    opp = &sv->ops[sv->reqs[r].op];
  }
  const OpTemplate &op = *opp;
  sv->reqs[r].t_launch = sv->now();
  cudaError_t e = cudaMemsetAsync(s.d_status, 0, sizeof(int), s.stream);
  if (e != cudaSuccess) note_error(sv, cuda_error(e, "cudaMemsetAsync"));
  for (size_t k = 0; k < op.descs.size(); ++k) {
    int rc = launch_one_pair(op.descs[k], op.ntiles[k], sv->fp, s.d_status, s.stream);
    note_error(sv, rc);
  }
  e = cudaMemcpyAsync(s.h_status, s.d_status, sizeof(int), cudaMemcpyDeviceToHost, s.stream);
  if (e != cudaSuccess) note_error(sv, cuda_error(e, "server status read-back"));
  e = cudaEventRecord(s.fin, s.stream);
  if (e != cudaSuccess) note_error(sv, cuda_error(e, "cudaEventRecord"));
  s.reqs.assign(1, r);
  s.busy = true;
  s.seq = sv->launches;
  sv->launches += (long long)op.descs.size();
  sv->batched_requests += 1;
  return true;
}

void worker_loop(cgx_server *sv) {
  const int nslots = sv->mode == CGX_SERVE_BATCHED ? SERVER_SLOTS : 1;
  for (;;) {
    bool progress = false;
    for (int i = 0; i < nslots; ++i) {
      Slot &s = sv->slots[i];
      if (s.busy && cudaEventQuery(s.fin) == cudaSuccess) {
        retire(sv, i);
        progress = true;
      }
    }
    for (int i = 0; i < nslots; ++i) {
      Slot &s = sv->slots[i];
      if (!s.busy) {
        bool l = sv->mode == CGX_SERVE_BATCHED ? launch_batch(sv, i) : launch_plain(sv, s);
        progress |= l;
      }
    }
    if (progress) continue;
    bool any_busy = false;
    for (int i = 0; i < nslots; ++i) any_busy |= sv->slots[i].busy;
    if (sv->stop.load() && !any_busy) {
      std::lock_guard<std::mutex> g(sv->mu);
      if (sv->pending.empty()) return;
    }
    if (any_busy) {
      bool all_busy = true;
      int oldest = -1;
      for (int i = 0; i < nslots; ++i) {
        all_busy &= sv->slots[i].busy;
        if (sv->slots[i].busy && (oldest < 0 || sv->slots[i].seq < sv->slots[oldest].seq)) oldest = i;
      }
      if (all_busy) {
        // nothing can launch before a slot frees: sleep on the oldest
        // slot's blocking-sync event (no core spins meanwhile)
        cudaEventSynchronize(sv->slots[oldest].fin);
      } else {
        // a free slot and nothing pending: wake for a new request or,
        // after a short while, to poll the busy slot again
        std::unique_lock<std::mutex> g(sv->mu);
        sv->cv.wait_for(g, std::chrono::microseconds(20),
                        [&] { return !sv->pending.empty() || sv->stop.load(); });
      }
    } else {
      std::unique_lock<std::mutex> g(sv->mu);
      sv->cv.wait_for(g, std::chrono::microseconds(200),
                      [&] { return !sv->pending.empty() || sv->stop.load(); });
    }
  }
}

double percentile(std::vector<double> v, double p) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  double idx = p * (double)(v.size() - 1);
  size_t lo = (size_t)idx;
  size_t hi = std::min(lo + 1, v.size() - 1);
  double f = idx - (double)lo;
  return v[lo] * (1 - f) + v[hi] * f;
}

} // namespace

extern "C" {

int cgx_server_create(cgx_server **out, int mode, int64_t hbm_budget_bytes, int max_pairs,
                      int64_t max_tiles, int64_t max_requests) {
  if (!out || max_requests <= 0) return set_error(CGX_EINVAL, "bad server arguments");
  if (mode != CGX_SERVE_BATCHED && mode != CGX_SERVE_PLAIN)
    return set_error(CGX_EINVAL, "bad serving mode");
  if (max_pairs <= 0 || max_tiles <= 0) return set_error(CGX_EINVAL, "bad slot capacity");
  cgx_server *sv = new cgx_server();
  sv->mode = mode;
  sv->budget = hbm_budget_bytes;
  sv->fp = current_fp_mode();
  sv->max_requests = (size_t)max_requests;
  sv->reqs.reserve(sv->max_requests);
  const int nslots = mode == CGX_SERVE_BATCHED ? SERVER_SLOTS : 1;
  for (int i = 0; i < nslots; ++i) {
    int rc = slot_init(sv->slots[i], (size_t)max_tiles);
    if (rc) {
      for (int j = 0; j <= i; ++j) slot_free(sv->slots[j]);
      delete sv;
      return rc;
    }
  }
  if (mode == CGX_SERVE_BATCHED) {
    cudaError_t e = cudaStreamCreateWithFlags(&sv->upload, cudaStreamNonBlocking);
    int rc = e == cudaSuccess ? pool_reserve(sv, (size_t)max_pairs) : cuda_error(e, "server upload stream");
    if (rc) {
      for (int j = 0; j < nslots; ++j) slot_free(sv->slots[j]);
      pool_free(sv->pool);
      if (sv->upload) cudaStreamDestroy(sv->upload);
      delete sv;
      return rc;
    }
  }
  *out = sv;
  return CGX_OK;
}

int cgx_server_destroy(cgx_server *sv) {
  if (!sv) return CGX_OK;
  if (sv->worker.joinable()) {
    sv->stop = true;
    sv->cv.notify_all();
    sv->worker.join();
  }
  for (int i = 0; i < SERVER_SLOTS; ++i) slot_free(sv->slots[i]);
  pool_free(sv->pool);
  if (sv->upload) cudaStreamDestroy(sv->upload);
  delete sv;
  return CGX_OK;
}

int cgx_server_admit(cgx_server *sv, int64_t bytes) {
  if (!sv || bytes < 0) return set_error(CGX_EINVAL, "bad admission");
  std::lock_guard<std::mutex> g(sv->mu);
  if (sv->used + bytes > sv->budget)
    return set_error(CGX_ENOMEM, "HBM budget: %lld of %lld bytes in use, %lld more requested",
                     (long long)sv->used, (long long)sv->budget, (long long)bytes);
  sv->used += bytes;
  return CGX_OK;
}

int cgx_server_release(cgx_server *sv, int64_t bytes) {
  if (!sv || bytes < 0) return set_error(CGX_EINVAL, "bad release");
  std::lock_guard<std::mutex> g(sv->mu);
  sv->used = std::max<long long>(0, sv->used - bytes);
  return CGX_OK;
}

int cgx_server_define_op(cgx_server *sv, int hier, const cgx_batch *pairs, int *op_id) {
  if (!sv || !op_id || hier < 0) return set_error(CGX_EINVAL, "bad operation");
  const Desc *d;
  const int *nt;
  const long long *pts, *byt;
  int n;
  int rc = batch_pairs(pairs, &d, &nt, &pts, &byt, &n);
  if (rc) return rc;
  OpTemplate op;
  op.hier = hier;
  op.descs.assign(d, d + n);
  op.ntiles.assign(nt, nt + n);
  // the pool's copies: prolongations that TMA can stage are tiled in their
  // variant's configuration and get tensor maps; the others run in the
  // cp.async form on their default tiles
  std::vector<Desc> pd(op.descs);
  std::vector<long long> pnt(nt, nt + n);
  std::vector<CUtensorMap> maps(3 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    if (!is_stencil(pd[i].kind)) continue;
    const int v = tma_variant(pd[i]);
    Desc t = pd[i];
    long long tn = 0;
    if (v >= 0) tn = tile_prolongation(t, sv->tma_cfg[v]);
    if (v >= 0 && tn > 0 && tn < (1LL << 31) && encode_tma_maps(t, &maps[3 * (size_t)i])) {
      pd[i] = t;
      pnt[i] = tn;
    } else {
      pd[i].bx = 0;
    }
  }
  for (int i = 0; i < n; ++i) {
    op.tiles += sv->mode == CGX_SERVE_BATCHED ? pnt[i] : nt[i];
    op.points += pts[i];
    op.bytes += byt[i];
  }
  if ((size_t)op.tiles > sv->slots[0].tile_cap) return set_error(CGX_EINVAL, "operation larger than a server slot");
  // batched mode: the descriptors and tensor maps go into the device pool
  // once (synchronous copies: the operation is usable when this returns),
  // and the tiles are kept with pool indices
  std::lock_guard<std::mutex> dg(sv->define_mu);
  if (sv->mode == CGX_SERVE_BATCHED && n > 0) {
    rc = pool_reserve(sv, sv->pool.used + (size_t)n);
    if (rc) return rc;
    const size_t base = sv->pool.used;
    cudaError_t e = cudaMemcpyAsync(sv->pool.descs + base, pd.data(), (size_t)n * sizeof(Desc),
                                    cudaMemcpyHostToDevice, sv->upload);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(sv->pool.maps + 3 * base, maps.data(), 3 * (size_t)n * sizeof(CUtensorMap),
                          cudaMemcpyHostToDevice, sv->upload);
    // from pageable memory a copy may return before its DMA lands: the
    // operation is published only once the upload has completed
    if (e == cudaSuccess) e = cudaStreamSynchronize(sv->upload);
    if (e != cudaSuccess) return cuda_error(e, "server operation upload");
    for (int i = 0; i < n; ++i) {
      std::vector<int2> &st = op.seg_tiles[segment_of(pd[i])];
      for (long long j = 0; j < pnt[i]; ++j) st.push_back(make_int2((int)(base + (size_t)i), (int)j));
    }
    sv->pool.used = base + (size_t)n;
  }
  std::lock_guard<std::mutex> g(sv->mu); // the worker may be running
  sv->ops.push_back(std::move(op));
  if ((int)sv->hier_last.size() <= hier) sv->hier_last.resize(hier + 1, -1);
  *op_id = (int)sv->ops.size() - 1;
  return CGX_OK;
}

int cgx_server_set_config(cgx_server *sv, int variant, int config) {
  if (!sv || variant < -1 || variant >= TV_COUNT || config < 0 || config >= TMA_NCFG)
    return set_error(CGX_EINVAL, "server set_config: variant %d / configuration %d out of range", variant,
                     config);
  std::lock_guard<std::mutex> dg(sv->define_mu);
  for (int v = 0; v < TV_COUNT; ++v)
    if (variant < 0 || v == variant) sv->tma_cfg[v] = config;
  return CGX_OK;
}

int cgx_server_start(cgx_server *sv) {
  if (!sv) return set_error(CGX_EINVAL, "null server");
  if (sv->worker.joinable()) return CGX_OK;
  sv->stop = false;
  sv->fp = current_fp_mode();
  sv->epoch = clk::now();
  sv->worker = std::thread(worker_loop, sv);
  return CGX_OK;
}

int cgx_server_submit(cgx_server *sv, int op_id, int64_t *request_id) {
  if (!sv || op_id < 0) return set_error(CGX_EINVAL, "bad request");
  {
    std::lock_guard<std::mutex> g(sv->mu);
    if (op_id >= (int)sv->ops.size()) return set_error(CGX_EINVAL, "bad request: no operation %d", op_id);
    if (sv->reqs.size() >= sv->max_requests)
      return set_error(CGX_ENOMEM, "request log full (%zu requests)", sv->max_requests);
    Request r;
    r.op = op_id;
    r.t_arrive = sv->now();
    sv->reqs.push_back(r);
    sv->pending.push_back((int)sv->reqs.size() - 1);
    sv->submitted++;
    if (request_id) *request_id = (int64_t)sv->reqs.size() - 1;
  }
  sv->cv.notify_all();
  return CGX_OK;
}

int cgx_server_replay(cgx_server *sv, const int *op_ids, const double *arrival_s, int n) {
  if (!sv || (n > 0 && (!op_ids || !arrival_s))) return set_error(CGX_EINVAL, "bad trace");
  int rc = cgx_server_start(sv);
  if (rc) return rc;
  const double t0 = sv->now();
  for (int i = 0; i < n; ++i) {
    const double due = t0 + arrival_s[i];
    while (sv->now() < due) { /* spin: sub-microsecond arrival accuracy */ }
    if ((rc = cgx_server_submit(sv, op_ids[i], nullptr))) return rc;
  }
  return CGX_OK;
}

int cgx_server_drain(cgx_server *sv) {
  if (!sv) return set_error(CGX_EINVAL, "null server");
  std::unique_lock<std::mutex> g(sv->mu);
  // bounded: a stream of work that does not finish in 10 minutes is an error
  if (!sv->cv.wait_for(g, std::chrono::seconds(600),
                       [&] { return sv->completed.load() >= sv->submitted; }))
    return set_error(CGX_ECUDA, "server drain timed out");
  std::lock_guard<std::mutex> e(sv->err_mu);
  if (sv->error) return set_error(sv->error, "%s", sv->error_msg.c_str());
  return CGX_OK;
}

int cgx_server_stats(cgx_server *sv, cgx_server_report *rep) {
  if (!sv || !rep) return set_error(CGX_EINVAL, "null argument");
  std::lock_guard<std::mutex> g(sv->mu);
  std::vector<double> lat;
  double first = 1e300, last = 0;
  long long points = 0, bytes = 0, done = 0;
  for (const Request &r : sv->reqs) {
    if (r.t_done <= 0) continue;
    lat.push_back(1e3 * (r.t_done - r.t_arrive));
    first = std::min(first, r.t_arrive);
    last = std::max(last, r.t_done);
    points += sv->ops[r.op].points;
    bytes += sv->ops[r.op].bytes;
    ++done;
  }
  memset(rep, 0, sizeof *rep);
  rep->requests = done;
  rep->launches = sv->launches;
  rep->p50_ms = percentile(lat, 0.50);
  rep->p99_ms = percentile(lat, 0.99);
  rep->mean_ms = lat.empty() ? 0 : [&] { double s = 0; for (double x : lat) s += x; return s / lat.size(); }();
  rep->makespan_s = done ? last - first : 0;
  rep->fine_points = points;
  rep->points_per_s = rep->makespan_s > 0 ? (double)points / rep->makespan_s : 0;
  rep->mean_batch = sv->launches ? (double)sv->batched_requests /
                                       (double)(sv->mode == CGX_SERVE_BATCHED ? sv->launches : done)
                                 : 0;
  rep->hbm_used = sv->used;
  rep->bytes = bytes;
  rep->bytes_per_s = rep->makespan_s > 0 ? (double)bytes / rep->makespan_s : 0;
  return CGX_OK;
}

int cgx_server_latencies(cgx_server *sv, double *out_ms, int64_t n) {
  if (!sv || !out_ms) return set_error(CGX_EINVAL, "null argument");
  std::lock_guard<std::mutex> g(sv->mu);
  int64_t k = 0;
  for (const Request &r : sv->reqs) {
    if (k >= n) break;
    out_ms[k++] = r.t_done > 0 ? 1e3 * (r.t_done - r.t_arrive) : -1.0;
  }
  return CGX_OK;
}

} // extern "C"
