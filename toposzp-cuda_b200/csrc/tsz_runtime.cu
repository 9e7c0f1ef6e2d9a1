// Host runtime: error state, workspaces, scratch arenas.
#include "tsz_runtime.h"

#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <vector>

namespace tsz {

static thread_local std::string g_err;

void set_error(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
}

void clear_error() { g_err.clear(); }
const char *last_error() { return g_err.c_str(); }

bool cuda_fail(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return false;
  set_error("%s: %s", what, cudaGetErrorString(e));
  return true;
}

bool Arena::reserve(size_t bytes) {
  used = 0;
  if (bytes <= cap) return true;
  release();
  size_t want = bytes + bytes / 8 + (1u << 20);
  if (cudaMalloc(&base, want) != cudaSuccess) {
    cudaGetLastError();
    base = nullptr;
    cap = 0;
    set_error("device allocation of %zu bytes failed", want);
    return false;
  }
  cap = want;
  return true;
}

void Arena::release() {
  if (base) cudaFree(base);
  base = nullptr;
  cap = 0;
  used = 0;
}

static bool ctx_init(szp_b200_ctx *c, cudaStream_t s) {
  if (cuda_fail(cudaGetDevice(&c->device), "cudaGetDevice")) return false;
  cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device);
  if (s) {
    c->stream = s;
    c->own_stream = false;
  } else {
    if (cuda_fail(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate"))
      return false;
    c->own_stream = true;
  }
  if (cuda_fail(cudaMallocHost(&c->h_words, 64 * sizeof(unsigned long long)), "cudaMallocHost"))
    return false;
  if (cuda_fail(cudaMalloc(&c->d_words, 64 * sizeof(unsigned long long)), "cudaMalloc"))
    return false;
  return true;
}

void tl_begin(szp_b200_ctx *ctx) {
  ctx->nstage = 0;
  if (!ctx->ev[0]) {
    for (int i = 0; i <= szp_b200_ctx::kMaxStages; i++) cudaEventCreate(&ctx->ev[i]);
  }
  ctx->timeline_started = cudaEventRecord(ctx->ev[0], ctx->stream) == cudaSuccess;
}

void tl_mark(szp_b200_ctx *ctx, const char *name) {
  if (!ctx->timeline_started || ctx->nstage >= szp_b200_ctx::kMaxStages) return;
  ctx->stage_name[ctx->nstage] = name;
  cudaEventRecord(ctx->ev[ctx->nstage + 1], ctx->stream);
  ctx->nstage++;
}

cudaStream_t copy_stream(szp_b200_ctx *ctx) {
  if (!ctx->copy_stream) {
    if (cuda_fail(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking), "cudaStreamCreate"))
      return nullptr;
    if (cuda_fail(cudaEventCreateWithFlags(&ctx->copy_ev, cudaEventDisableTiming), "cudaEventCreate")) {
      cudaStreamDestroy(ctx->copy_stream);
      ctx->copy_stream = nullptr;
      return nullptr;
    }
  }
  return ctx->copy_stream;
}

cudaStream_t d2h_stream(szp_b200_ctx *ctx) {
  if (!ctx->d2h_stream &&
      cuda_fail(cudaStreamCreateWithFlags(&ctx->d2h_stream, cudaStreamNonBlocking), "cudaStreamCreate"))
    return nullptr;
  return ctx->d2h_stream;
}

static void ctx_free(szp_b200_ctx *c) {
  if (!c) return;
  if (c->d2h_stream) { cudaStreamSynchronize(c->d2h_stream); cudaStreamDestroy(c->d2h_stream); }
  c->d2h_stream = nullptr;
  if (c->copy_stream) { cudaStreamSynchronize(c->copy_stream); cudaStreamDestroy(c->copy_stream); }
  if (c->copy_ev) cudaEventDestroy(c->copy_ev);
  c->copy_stream = nullptr;
  c->copy_ev = nullptr;
  for (int i = 0; i < szp_b200_ctx::kChunkEvents; i++)
    if (c->chunk_ev[i]) { cudaEventDestroy(c->chunk_ev[i]); c->chunk_ev[i] = nullptr; }
  for (int i = 0; i < szp_b200_ctx::kChunkEvents; i++)
    if (c->part_ev[i]) { cudaEventDestroy(c->part_ev[i]); c->part_ev[i] = nullptr; }
  for (int i = 0; i <= szp_b200_ctx::kMaxStages; i++)
    if (c->ev[i]) { cudaEventDestroy(c->ev[i]); c->ev[i] = nullptr; }
  c->scratch.release();
  if (c->post_S) cudaFree(c->post_S);
  c->post_S = nullptr;
  c->io.release();
  if (c->h_words) cudaFreeHost(c->h_words);
  if (c->d_words) cudaFree(c->d_words);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  c->h_words = nullptr;
  c->d_words = nullptr;
  c->stream = nullptr;
}

// One default workspace per (thread, device); released at thread exit.
struct DefaultCtxs {
  std::vector<szp_b200_ctx *> v;
  ~DefaultCtxs() {
    for (auto *c : v) {
      if (c) { ctx_free(c); delete c; }
    }
  }
};
static thread_local DefaultCtxs g_defaults;

szp_b200_ctx *default_ctx() {
  int dev = 0;
  if (cuda_fail(cudaGetDevice(&dev), "cudaGetDevice")) return nullptr;
  if ((int)g_defaults.v.size() <= dev) g_defaults.v.resize(dev + 1, nullptr);
  if (!g_defaults.v[dev]) {
    auto *c = new szp_b200_ctx();
    if (!ctx_init(c, nullptr)) { ctx_free(c); delete c; return nullptr; }
    g_defaults.v[dev] = c;
  }
  return g_defaults.v[dev];
}

}  // namespace tsz

extern "C" {

const char *szp_b200_last_error(void) { return tsz::last_error(); }

const char *szp_b200_version(void) { return "toposzp-b200 1.0 (sm_100a)"; }

szp_b200_ctx *szp_b200_ctx_create(void *cuda_stream) {
  tsz::clear_error();
  auto *c = new szp_b200_ctx();
  if (!tsz::ctx_init(c, (cudaStream_t)cuda_stream)) {
    tsz::ctx_free(c);
    delete c;
    return nullptr;
  }
  return c;
}

void szp_b200_ctx_destroy(szp_b200_ctx *ctx) {
  tsz::DeviceGuard dg(ctx);
  if (!ctx) return;
  tsz::ctx_free(ctx);
  delete ctx;
}

int szp_b200_ctx_stage_times(szp_b200_ctx *ctx, const char **names, float *ms, int max) {
  if (!ctx || !ctx->timeline_started) return 0;
  if (cudaEventSynchronize(ctx->ev[ctx->nstage]) != cudaSuccess) return 0;
  int k = ctx->nstage < max ? ctx->nstage : max;
  for (int i = 0; i < k; i++) {
    names[i] = ctx->stage_name[i];
    ms[i] = 0.f;
    cudaEventElapsedTime(&ms[i], ctx->ev[i], ctx->ev[i + 1]);
  }
  return k;
}

unsigned long long szp_b200_ctx_launches(szp_b200_ctx *ctx) { return ctx ? ctx->launches : 0ull; }

}  // extern "C"
