// Topology-stream encoder that allocates nothing.
//
// Who needs it: callers that may not let a library allocate device memory.
//  - code inside a framework or server that owns every device allocation
//    (a caching allocator or a fixed arena sized at start-up), where a
//    library-side cudaMalloc fragments or exceeds the budget the owner planned;
//  - latency-critical paths, where cudaMalloc / cudaFree can synchronise the
//    device and stall every stream on it.
// The caller passes the field and the output buffer.  The only scratch the
// encoder needs -- one look-back descriptor per tile plus a few status words
// -- lives in a file-scope __device__ array of fixed size, so the call makes
// no allocation of any kind (no cudaMalloc, no cudaFree, no library routine
// that allocates).
//
// Limits and rules:
//  - Scratch: 131072 tile descriptors (4 MiB, held on every device that loads
//    the library).  One tile is 2048 elements at blockSize 64 (256 at
//    blockSize 1), so fields up to 268,435,456 elements fit at blockSize 64;
//    larger fields are rejected with an error, nothing is launched.
//  - The descriptors and status words must start at zero; the call clears
//    them on the caller's stream before its kernel runs.
//  - The first call on each device resolves the scratch address with that
//    device current (cudaGetSymbolAddress); make it before any stream capture
//    begins on that device.
//  - All calls on one device share the scratch: calls that overlap in time
//    (other threads, other streams) race and corrupt each other's output.
//    Serialise them.
//  - Synchronous: returns after the stream has finished the call's work.
#include <mutex>

#include "tsz_codec.h"
#include "tsz_ops.h"
#include "tsz_runtime.h"

namespace tsz {

constexpr size_t kNoAllocTiles = 131072;
constexpr size_t kNoAllocWords = 16;
constexpr size_t kNoAllocBytes = kNoAllocTiles * sizeof(TileDesc) + kNoAllocWords * 8;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// device address of g_noalloc_scratch, resolved once per device
constexpr int kNoAllocMaxDevices = 64;
static void *g_noalloc_ptr[kNoAllocMaxDevices];
static std::mutex g_noalloc_mu;

static void *noalloc_scratch_address(int dev) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    set_error("szp_b200_topo_encode_noalloc: device %d out of range", dev);
    return nullptr;
  }
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      set_error("cudaGetSymbolAddress(no-allocation scratch) failed: %s", cudaGetErrorString(e));
      return nullptr;
    }
    g_noalloc_ptr[dev] = p;
  }
  return g_noalloc_ptr[dev];
}

}  // namespace tsz

using namespace tsz;

extern "C" SZP_B200_API int szp_b200_topo_encode_noalloc(const float *d_data, szp_b200_geom geom,
                                                         float absErrBound, int blockSize,
                                                         unsigned char *d_topo, size_t topo_cap,
                                                         size_t *topo_bytes, void *cuda_stream) {
  clear_error();
  if (!d_data || !d_topo || !topo_bytes) {
    set_error("szp_b200_topo_encode_noalloc: null argument");
    return -1;
  }
  *topo_bytes = 0;
  if (!(absErrBound > 0.0f)) {
    set_error("szp_b200_topo_encode_noalloc: error bound must be positive");
    return -1;
  }
  if (blockSize <= 0 || blockSize > kMaxBlockSize) {
    set_error("szp_b200_topo_encode_noalloc: blockSize %d out of range [1, %d]", blockSize, kMaxBlockSize);
    return -1;
  }
  Geom g;
  unsigned long long n = 0;
  if (!geom_elements(geom, &n, &g)) {
    set_error("szp_b200_topo_encode_noalloc: invalid geometry");
    return -1;
  }
  const unsigned long long nb = (n + blockSize - 1) / blockSize;
  const unsigned long long tb = (unsigned long long)enc_tile_blocks(blockSize);
  const unsigned long long ntiles = (nb + tb - 1) / tb;
  if (ntiles > kNoAllocTiles) {
    set_error("szp_b200_topo_encode_noalloc: %llu elements need %llu tile descriptors, the fixed "
              "scratch holds %zu (at most %llu elements at blockSize %d)",
              n, ntiles, kNoAllocTiles, (unsigned long long)kNoAllocTiles * tb * blockSize, blockSize);
    return -1;
  }
  if (topo_cap < 8) {
    set_error("szp_b200_topo_encode_noalloc: output buffer smaller than the 8-byte header");
    return -1;
  }
  int dev = 0, sms = 0;
  if (cuda_fail(cudaGetDevice(&dev), "cudaGetDevice") ||
      cuda_fail(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count"))
    return -1;
  unsigned char *base = static_cast<unsigned char *>(noalloc_scratch_address(dev));
  if (!base) return -1;
  TileDesc *desc = reinterpret_cast<TileDesc *>(base);
  unsigned long long *w = reinterpret_cast<unsigned long long *>(base + kNoAllocTiles * sizeof(TileDesc));
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
  // scratch keeps the previous call's contents: clear what the kernel expects at zero
  if (cuda_fail(cudaMemsetAsync(desc, 0, ntiles * sizeof(TileDesc), s), "memset") ||
      cuda_fail(cudaMemsetAsync(w, 0, kNoAllocWords * 8, s), "memset") ||
      cuda_fail(cudaMemsetAsync(d_topo, 0, 8, s), "memset"))
    return -1;
  EncArgs a{};
  a.data = d_data;
  a.n = n;
  a.B = blockSize;
  a.eb = absErrBound;
  a.inv = 1.0 / (double)absErrBound;
  a.g = g;
  a.out = d_topo + 8;
  a.out_cap = topo_cap - 8;
  a.desc = desc;
  a.tile_ctr = reinterpret_cast<unsigned *>(w + 3);
  a.err = reinterpret_cast<int *>(w + 4);
  a.total = w;
  a.cp_mode = kCpNone;
  unsigned long long grid = (unsigned long long)sms * 8ull;
  if (ntiles < grid) grid = ntiles;
  if (grid < 1) grid = 1;
  if (cuda_fail(launch_encode(kEncClassify, a, s, (int)grid), "no-allocation encode launch")) return -1;
  unsigned long long hw[5] = {0, 0, 0, 0, 0};
  if (cuda_fail(cudaMemcpyAsync(hw, w, sizeof(hw), cudaMemcpyDeviceToHost, s), "D2H totals") ||
      cuda_fail(cudaStreamSynchronize(s), "no-allocation encode"))
    return -1;
  const int err = (int)(hw[4] & 0xffffffffu);
  if (err) {
    set_error("szp_b200_topo_encode_noalloc: encoder reported status %d%s", err,
              err == kErrOutputOverflow ? " (output buffer too small)" : "");
    return -1;
  }
  *topo_bytes = 8 + hw[0];
  return 0;
}
