// Request server: compress / decompress requests of mixed sizes, served with
// continuous batching on device-resident buffers.
//
// The server owns `slots` workers; each worker has its own CUDA stream, a
// workspace (szp_b200_ctx) and a batch compressor, all kept for the server's
// lifetime.  Requests wait in one FIFO queue.  A free worker takes the head of
// the queue when the HBM budget admits it (the estimated device working set of
// the requests in flight stays within the budget; a request larger than the
// whole budget runs alone); if the head is a compression it also takes the
// compressions queued behind it, up to max_batch requests and a working set of
// budget / slots, and runs them as one batched launch.  Workers run
// concurrently on their own streams, so requests that arrive while others are
// on the GPU start as soon as a slot and memory free up and their work
// overlaps on the device.  Each request records its arrival, start and
// completion times on the server clock.
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "tsz_ops.h"
#include "tsz_runtime.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Item {
  szp_b200_request *r;
  size_t cost;
};

struct Slot {
  szp_b200_ctx *ctx = nullptr;
  szp_b200_batch *batch = nullptr;
  cudaStream_t stream = nullptr;
};

// element count of a request's geometry (0 when invalid or overflowing)
size_t elems_of(const szp_b200_geom &g) {
  unsigned long long n = 0;
  tsz::Geom kg;
  return tsz::geom_elements(g, &n, &kg) ? (size_t)n : 0;
}

}  // namespace

struct szp_b200_server {
  szp_b200_server_config cfg{};
  int device = 0;
  Clock::time_point t0;
  std::vector<Slot> slots;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Item> q;
  size_t inflight_bytes = 0;
  int inflight = 0;
  bool stop = false;
  // statistics
  unsigned long long submitted = 0, completed = 0, failed = 0, batches = 0, batched_requests = 0;
  size_t max_inflight_bytes = 0;
  int max_concurrent = 0;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace tsz {

// Estimated device working set of a request beyond its caller-owned buffers
// (bytes per element: compression keeps CP pairs, bins, ranks and encoder
// scratch; decompression keeps the raw copy, tags, ranks and the
// post-processing lists).
static size_t request_cost(const szp_b200_request *r) {
  const size_t n = elems_of(r->geom);
  return r->op == SZP_B200_OP_COMPRESS ? 40 * n + (1u << 20) : 32 * n + (1u << 20);
}

static void fail_request(szp_b200_request *r, const char *msg) {
  r->status = -1;
  snprintf(r->message, sizeof(r->message), "%s", msg);
}

static int compress_group(Slot &sl, szp_b200_request **rs, int count) {
  std::vector<szp_b200_batch_field> fs(count);
  for (int k = 0; k < count; k++) {
    const szp_b200_request *r = rs[k];
    szp_b200_batch_field &f = fs[k];
    memset(&f, 0, sizeof(f));
    f.d_data = r->d_data;
    f.geom = r->geom;
    f.errBound = r->errBound;
    f.rel = r->rel;
    f.d_topo = r->d_topo;
    f.topo_cap = r->topo_bytes;
    f.d_sort = r->d_sort;
    f.sort_cap = r->sort_bytes;
  }
  const int rc = szp_b200_batch_compress(sl.batch, fs.data(), count);
  if (rc == 0) {
    for (int k = 0; k < count; k++) {
      rs[k]->status = 0;
      rs[k]->sizes = fs[k].sizes;
      rs[k]->abs_eb = fs[k].abs_eb;
      rs[k]->message[0] = 0;
    }
  }
  return rc;
}

// A compression of at least this many elements fills the GPU by itself: it
// runs alone through the fused single-field path (the blockSize-64 encoder
// and the single-field rank), and smaller ones are merged into batched
// launches behind a small head.
constexpr size_t kAloneElems = (size_t)1 << 21;
// Elements of one merged launch at most: the workers' batch compressors are
// sized for it up front (szp_b200_server_reserve), so serving allocates
// nothing -- a buffer that grew would free memory, which waits for every
// stream of the device.
constexpr size_t kBatchElems = (size_t)1 << 24;

static int compress_alone(Slot &sl, szp_b200_request *r) {
  float eb = r->errBound;
  if (r->rel) {
    // the batch compressor resolves relative bounds on the device; one field
    // alone goes through it as a batch of one
    return 1;
  }
  szp_b200_sizes sz{};
  const int rc = szp_b200_topo_compress_dev(sl.ctx, r->d_data, r->geom, eb, r->blockSize, r->d_topo, r->d_sort,
                                            nullptr, &sz);
  if (rc == 0) {
    r->status = 0;
    r->sizes = sz;
    r->abs_eb = eb;
    r->message[0] = 0;
  }
  return rc ? -1 : 0;
}

static void run_group(szp_b200_server *S, Slot &sl, std::vector<Item> &grp) {
  const double ts = S->now();
  for (auto &it : grp) it.r->t_start = ts;
  szp_b200_request *head = grp[0].r;
  if (head->op == SZP_B200_OP_COMPRESS && grp.size() == 1 && elems_of(head->geom) >= kAloneElems &&
      head->blockSize == 64) {
    const int rc = compress_alone(sl, head);
    if (rc <= 0) {
      if (rc < 0) fail_request(head, szp_b200_last_error());
      head->t_done = S->now();
      return;
    }
  }
  if (head->op == SZP_B200_OP_COMPRESS) {
    std::vector<szp_b200_request *> rs;
    for (auto &it : grp) rs.push_back(it.r);
    if (compress_group(sl, rs.data(), (int)rs.size())) {
      // a merged launch that failed (e.g. its scratch did not fit) is retried
      // request by request, so one request's failure stays its own
      const std::string first = szp_b200_last_error();
      for (auto *r : rs) {
        if (rs.size() == 1 || compress_group(sl, &r, 1)) fail_request(r, rs.size() == 1 ? first.c_str()
                                                                                        : szp_b200_last_error());
        r->t_done = S->now();
      }
      return;
    }
    const double td = S->now();
    for (auto *r : rs) r->t_done = td;
  } else {
    const int rc = szp_b200_topo_decompress_dev(sl.ctx, head->d_topo, head->topo_bytes, head->d_sort,
                                                head->sort_bytes, nullptr, head->geom, head->errBound,
                                                head->blockSize, head->d_out, nullptr, head->postprocess);
    if (rc) fail_request(head, szp_b200_last_error());
    else { head->status = 0; head->message[0] = 0; }
    head->t_done = S->now();
  }
}

static void worker_main(szp_b200_server *S, int w) {
  cudaSetDevice(S->device);
  Slot &sl = S->slots[w];
  const size_t batch_cap = S->cfg.hbm_budget / (size_t)S->cfg.slots;
  std::vector<Item> grp;
  while (true) {
    grp.clear();
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_work.wait(lk, [&] {
        if (S->stop) return true;
        if (S->q.empty()) return false;
        const Item &h = S->q.front();
        return S->inflight == 0 || S->inflight_bytes + h.cost <= S->cfg.hbm_budget;
      });
      if (S->q.empty()) {
        if (S->stop) break;
        continue;
      }
      grp.push_back(S->q.front());
      S->q.pop_front();
      size_t bytes = grp[0].cost;
      if (grp[0].r->op == SZP_B200_OP_COMPRESS && elems_of(grp[0].r->geom) < kAloneElems) {
        // continuous batching: small compressions queued behind a small head
        // join its launch (large ones run alone on the fused path)
        size_t elems = elems_of(grp[0].r->geom);
        for (auto it = S->q.begin(); it != S->q.end() && (int)grp.size() < S->cfg.max_batch;) {
          const size_t ne = elems_of(it->r->geom);
          if (it->r->op == SZP_B200_OP_COMPRESS && it->r->blockSize == grp[0].r->blockSize && ne < kAloneElems &&
              elems + ne <= kBatchElems && bytes + it->cost <= batch_cap &&
              S->inflight_bytes + bytes + it->cost <= S->cfg.hbm_budget) {
            bytes += it->cost;
            elems += ne;
            grp.push_back(*it);
            it = S->q.erase(it);
          } else {
            ++it;
          }
        }
      }
      S->inflight_bytes += bytes;
      S->inflight += (int)grp.size();
      if (S->inflight_bytes > S->max_inflight_bytes) S->max_inflight_bytes = S->inflight_bytes;
      if (S->inflight > S->max_concurrent) S->max_concurrent = S->inflight;
      if (grp[0].r->op == SZP_B200_OP_COMPRESS && elems_of(grp[0].r->geom) < kAloneElems) {
        S->batches++;
        S->batched_requests += grp.size();
      }
    }
    run_group(S, sl, grp);
    {
      std::lock_guard<std::mutex> lk(S->mu);
      for (auto &it : grp) {
        S->inflight_bytes -= it.cost;
        S->inflight--;
        S->completed++;
        if (it.r->status) S->failed++;
        it.r->done = 1;
      }
    }
    S->cv_work.notify_all();
    S->cv_done.notify_all();
  }
}

}  // namespace tsz

using namespace tsz;

extern "C" {

szp_b200_server *szp_b200_server_create(const szp_b200_server_config *cfg) {
  clear_error();
  if (!cfg || cfg->slots <= 0 || cfg->slots > 64 || cfg->max_batch <= 0 || cfg->blockSize <= 0 ||
      cfg->blockSize > 256) {
    set_error("szp_b200_server_create: invalid configuration");
    return nullptr;
  }
  auto *S = new szp_b200_server();
  S->cfg = *cfg;
  if (S->cfg.hbm_budget == 0) S->cfg.hbm_budget = (size_t)120 << 30;
  S->t0 = Clock::now();
  if (cuda_fail(cudaGetDevice(&S->device), "cudaGetDevice")) { delete S; return nullptr; }
  S->slots.resize(cfg->slots);
  bool ok = true;
  for (auto &sl : S->slots) {
    if (cuda_fail(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking), "cudaStreamCreate")) {
      ok = false;
      break;
    }
    sl.ctx = szp_b200_ctx_create(sl.stream);
    // the workers' streams share the GPU: no cooperative launches on them
    if (sl.ctx) sl.ctx->coop_off = true;
    sl.batch = sl.ctx ? szp_b200_batch_create(sl.stream, cfg->blockSize) : nullptr;
    if (!sl.ctx || !sl.batch) { ok = false; break; }
  }
  if (!ok) {
    const std::string msg = last_error();
    szp_b200_server_destroy(S);
    set_error("szp_b200_server_create: %s", msg.c_str());
    return nullptr;
  }
  for (int w = 0; w < cfg->slots; w++) S->workers.emplace_back(worker_main, S, w);
  return S;
}

void szp_b200_server_destroy(szp_b200_server *S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  for (auto &t : S->workers) t.join();
  for (auto &sl : S->slots) {
    if (sl.batch) szp_b200_batch_destroy(sl.batch);
    if (sl.ctx) szp_b200_ctx_destroy(sl.ctx);
    if (sl.stream) cudaStreamDestroy(sl.stream);
  }
  delete S;
}

double szp_b200_server_now(szp_b200_server *S) { return S ? S->now() : 0.0; }

int szp_b200_server_reserve(szp_b200_server *S, size_t max_elements) {
  clear_error();
  if (!S) { set_error("null argument"); return -1; }
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->inflight || !S->q.empty()) { set_error("szp_b200_server_reserve: requests are in flight"); return -1; }
  }
  for (auto &sl : S->slots)
    if (ctx_reserve_for(sl.ctx, max_elements, S->cfg.blockSize) ||
        szp_b200_batch_reserve(sl.batch, S->cfg.max_batch, kBatchElems))
      return -1;
  return 0;
}

int szp_b200_server_submit(szp_b200_server *S, szp_b200_request *r) {
  clear_error();
  if (!S || !r) { set_error("null argument"); return -1; }
  if (r->op != SZP_B200_OP_COMPRESS && r->op != SZP_B200_OP_DECOMPRESS) { set_error("unknown op"); return -1; }
  if (elems_of(r->geom) == 0) { set_error("invalid geometry"); return -1; }
  if (r->op == SZP_B200_OP_COMPRESS && r->blockSize != S->cfg.blockSize) {
    set_error("compress request blockSize %d differs from the server's %d", r->blockSize, S->cfg.blockSize);
    return -1;
  }
  r->done = 0;
  r->status = 1;
  r->message[0] = 0;
  r->t_start = r->t_done = 0.0;
  if (r->t_arrival <= 0.0) r->t_arrival = S->now();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->q.push_back({r, request_cost(r)});
    S->submitted++;
  }
  S->cv_work.notify_one();
  return 0;
}

int szp_b200_server_wait(szp_b200_server *S, szp_b200_request *r, double timeout_s) {
  if (!S || !r) return -1;
  std::unique_lock<std::mutex> lk(S->mu);
  const bool ok = S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return r->done != 0; });
  return ok ? 0 : 1;
}

int szp_b200_server_drain(szp_b200_server *S, double timeout_s) {
  if (!S) return -1;
  std::unique_lock<std::mutex> lk(S->mu);
  const bool ok = S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                      [&] { return S->completed == S->submitted; });
  return ok ? 0 : 1;
}

int szp_b200_server_run_trace(szp_b200_server *S, szp_b200_request *reqs, int n, const double *arrival_s,
                              double timeout_s) {
  clear_error();
  if (!S || (!reqs && n)) { set_error("null argument"); return -1; }
  const double base = S->now();
  for (int i = 0; i < n; i++) {
    const double at = base + (arrival_s ? arrival_s[i] : 0.0);
    while (true) {
      const double dt = at - S->now();
      if (dt <= 0) break;
      if (dt > 2e-4) std::this_thread::sleep_for(std::chrono::duration<double>(dt - 1e-4));
    }
    reqs[i].t_arrival = at > 0.0 ? at : 1e-9;
    if (szp_b200_server_submit(S, &reqs[i])) return -1;
  }
  return szp_b200_server_drain(S, timeout_s);
}

int szp_b200_server_stats(szp_b200_server *S, szp_b200_server_stats_t *st) {
  if (!S || !st) return -1;
  std::lock_guard<std::mutex> lk(S->mu);
  st->submitted = S->submitted;
  st->completed = S->completed;
  st->failed = S->failed;
  st->batches = S->batches;
  st->batched_requests = S->batched_requests;
  st->max_inflight_bytes = S->max_inflight_bytes;
  st->max_concurrent = S->max_concurrent;
  return 0;
}

}  // extern "C"
