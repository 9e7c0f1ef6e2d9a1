// Host runtime: per-thread error state, device workspaces and scratch arenas.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "../../include/szp_b200.h"

namespace tsz {

void set_error(const char *fmt, ...);
void clear_error();
const char *last_error();

// Grow-only device scratch arena, carved per call with 256-byte alignment.
struct Arena {
  unsigned char *base = nullptr;
  size_t cap = 0;
  size_t used = 0;
  bool reserve(size_t bytes);   // ensures capacity (may reallocate; contents lost)
  void reset() { used = 0; }
  template <class T> T *take(size_t count) {
    size_t bytes = (count * sizeof(T) + 255) & ~(size_t)255;
    if (used + bytes > cap) return nullptr;
    T *p = reinterpret_cast<T *>(base + used);
    used += bytes;
    return p;
  }
  void release();
};

}  // namespace tsz

struct szp_b200_ctx {
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  tsz::Arena scratch;       // per-call temporaries
  tsz::Arena io;            // device copies of host inputs / outputs (API path)
  unsigned long long *h_words = nullptr;   // pinned host words for small D2H reads
  unsigned long long *d_words = nullptr;   // device status words
  unsigned long long *post_S = nullptr;    // post-processing result words (generation-tagged)
  unsigned long long post_S_cap = 0;
  unsigned post_gen = 0;
  // stage timeline of the last call (CUDA events on the workspace stream)
  static constexpr int kMaxStages = 24;
  cudaEvent_t ev[kMaxStages + 1] = {};
  const char *stage_name[kMaxStages] = {};
  int nstage = 0;
  bool timeline_started = false;
  unsigned long long launches = 0;         // kernels launched through this workspace
  // second stream for host copies that overlap work on `stream` (created on first use)
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t copy_ev = nullptr;
  cudaStream_t d2h_stream = nullptr;         // device-to-host copies that overlap copy_stream
  static constexpr int kChunkEvents = 16;
  cudaEvent_t chunk_ev[kChunkEvents] = {};   // parts of a chunked host-to-device copy
  cudaEvent_t part_ev[kChunkEvents] = {};    // encoder launches of a chunked encode
  // no cooperative launches on this workspace's stream (set for server
  // workers, whose streams share the GPU)
  bool coop_off = false;
};

namespace tsz {
// Makes the workspace's device current for the duration of a call (a thread
// other than the one that created the workspace may start on another
// device) and restores the caller's device afterwards.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(const szp_b200_ctx *ctx) {
    int cur = 0;
    if (ctx && cudaGetDevice(&cur) == cudaSuccess && cur != ctx->device && cudaSetDevice(ctx->device) == cudaSuccess)
      prev = cur;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard &) = delete;
  DeviceGuard &operator=(const DeviceGuard &) = delete;
};
}  // namespace tsz

namespace tsz {

// Per-thread default workspace used by the reference-compatible entry points.
szp_b200_ctx *default_ctx();

// Stage timeline: tl_begin() at the start of a call, tl_mark(name) after
// each stage's work has been enqueued on ctx->stream.
void tl_begin(szp_b200_ctx *ctx);
void tl_mark(szp_b200_ctx *ctx, const char *name);

// The workspace's copy stream and its event (created on first use); null on failure.
cudaStream_t copy_stream(szp_b200_ctx *ctx);
// A second copy stream for device-to-host copies that run beside copy_stream.
cudaStream_t d2h_stream(szp_b200_ctx *ctx);

// Rounds a byte count up to 256.
inline size_t a256(size_t b) { return (b + 255) & ~(size_t)255; }

// CUDA error -> message; returns true on failure.
bool cuda_fail(cudaError_t e, const char *what);

}  // namespace tsz
