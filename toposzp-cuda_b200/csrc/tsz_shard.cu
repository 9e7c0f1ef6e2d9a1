// Pieces of a compression of one field split across devices (one process per
// device, block-aligned flat-index slabs; the exchange steps -- stream
// offsets, the global bin rank of the critical points, the sort-position
// blocks that straddle two slabs -- run in the host layer over
// torch.distributed):
//   * a slab's topology blocks and its critical-point pairs, from the slab's
//     values plus a halo of one plane (one row in 2D) + 1 element either side
//     (the blockSize-64 fused encoder with a global index base);
//   * the quantization bin of each pair (the owner of a bin in the exchange);
//   * the dense rank of a set of pairs inside their bins (the rank stage);
//   * the integer stream of a run of sort positions.
// Streams concatenated in slab order are the single-device streams byte for
// byte: blocks never straddle slabs, and the bins of the exchanged pairs are
// the ones the single-device rank computes.
#include <cstring>

#include "tsz_enc64.h"
#include "tsz_ops.h"

namespace tsz {

__global__ void pair_bins_kernel(const uint2 *__restrict__ pairs, unsigned long long K, float eb, double inv,
                                 int *__restrict__ bins) {
  for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < K;
       k += (unsigned long long)gridDim.x * blockDim.x)
    bins[k] = quant_bin(code_float(pairs[k].x), eb, inv);
}

}  // namespace tsz

using namespace tsz;

extern "C" {

SZP_B200_API int szp_b200_topo_encode_slab_dev(szp_b200_ctx *ctx, const float *d_slab, size_t halo_lo,
                                               szp_b200_geom geom, float absErrBound, int blockSize, size_t begin,
                                               size_t end, unsigned char *d_payload, size_t payload_cap,
                                               void *d_pairs, size_t pairs_cap, szp_b200_slab_sizes *sizes) {
  clear_error();
  DeviceGuard dg(ctx);
  if (!ctx || !d_slab || !d_payload || !sizes || (!d_pairs && pairs_cap)) {
    set_error("szp_b200_topo_encode_slab_dev: null argument");
    return -1;
  }
  memset(sizes, 0, sizeof(*sizes));
  unsigned long long n;
  Geom g;
  if (!geom_elements(geom, &n, &g)) { set_error("szp_b200_topo_encode_slab_dev: invalid geometry"); return -1; }
  if (blockSize != 64) { set_error("szp_b200_topo_encode_slab_dev: slabs are encoded at blockSize 64"); return -1; }
  if (begin >= end || end > n || begin % 64 || (end % 64 && end != n)) {
    set_error("szp_b200_topo_encode_slab_dev: slab [%zu, %zu) must be block-aligned inside [0, %llu)", begin, end, n);
    return -1;
  }
  const unsigned long long reach = (g.nd == 3 ? (unsigned long long)g.plane : (unsigned long long)g.d3) + 1;
  if (halo_lo > begin || halo_lo < (begin < reach ? begin : reach) || halo_lo % 4) {
    set_error("szp_b200_topo_encode_slab_dev: halo_lo %zu must be a multiple of 4 covering min(begin, %llu)", halo_lo,
              reach);
    return -1;
  }
  if (reinterpret_cast<uintptr_t>(d_slab) & 15) {
    set_error("szp_b200_topo_encode_slab_dev: slab buffer must be 16-byte aligned");
    return -1;
  }
  if (!(absErrBound > 0.0f)) { set_error("szp_b200_topo_encode_slab_dev: error bound must be > 0"); return -1; }
  const unsigned long long m = end - begin;
  const unsigned long long ntiles = enc64_tiles(m);
  if (!ctx->scratch.reserve(a256((ntiles + 1) * sizeof(TileDesc)) + 4096)) return -1;
  TileDesc *desc = ctx->scratch.take<TileDesc>(ntiles + 1);
  unsigned long long *w = ctx->d_words;  // [0..2] totals, [3] tile counter, [4] err
  cudaStream_t s = ctx->stream;
  if (cuda_fail(cudaMemsetAsync(desc, 0, (ntiles + 1) * sizeof(TileDesc), s), "memset") ||
      cuda_fail(cudaMemsetAsync(w, 0, 8 * sizeof(unsigned long long), s), "memset"))
    return -1;
  Enc64Args a{};
  // indexed by global element: element `begin - halo_lo` is the slab buffer's first
  a.data = reinterpret_cast<const float *>(reinterpret_cast<uintptr_t>(d_slab) - (begin - halo_lo) * sizeof(float));
  a.base = begin;
  a.n = m;
  a.inv = 1.0 / (double)absErrBound;
  a.g = g;
  a.out = d_payload;
  a.out_cap = payload_cap;
  a.desc = desc;
  a.tile_ctr = reinterpret_cast<unsigned *>(w + 3);
  a.err = reinterpret_cast<int *>(w + 4);
  a.total = w;
  a.cp_out = static_cast<uint2 *>(d_pairs);
  a.cp_cap = pairs_cap;
  if (cuda_fail(launch_enc64_args(a, s, ctx->sm_count), "slab encode launch")) return -1;
  ctx->launches += 1;
  if (cuda_fail(cudaMemcpyAsync(ctx->h_words, w, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s),
                "D2H totals") ||
      cuda_fail(cudaStreamSynchronize(s), "slab encode"))
    return -1;
  const int err = (int)(ctx->h_words[4] & 0xffffffffu);
  if (err) { set_error("slab encoder reported status %d", err); return -1; }
  sizes->payload_bytes = ctx->h_words[0];
  sizes->cp_count = ctx->h_words[1];
  sizes->extrema_count = ctx->h_words[2];
  return 0;
}

SZP_B200_API int szp_b200_pair_bins_dev(szp_b200_ctx *ctx, const void *d_pairs, size_t K, float absErrBound,
                                        int *d_bins) {
  clear_error();
  DeviceGuard dg(ctx);
  if (!ctx || (K && (!d_pairs || !d_bins))) { set_error("szp_b200_pair_bins_dev: null argument"); return -1; }
  if (K == 0) return 0;
  const unsigned long long gmax = (unsigned long long)ctx->sm_count * 8;
  const unsigned grid = (unsigned)((K + 255) / 256 < gmax ? (K + 255) / 256 : gmax);
  pair_bins_kernel<<<grid, 256, 0, ctx->stream>>>(static_cast<const uint2 *>(d_pairs), K, absErrBound,
                                                  1.0 / (double)absErrBound, d_bins);
  ctx->launches += 1;
  if (cuda_fail(cudaGetLastError(), "bins launch")) return -1;
  return cuda_fail(cudaStreamSynchronize(ctx->stream), "bins") ? -1 : 0;
}

SZP_B200_API int szp_b200_rank_pairs_dev(szp_b200_ctx *ctx, const void *d_pairs, size_t K, size_t E,
                                         float absErrBound, int *d_sp) {
  clear_error();
  DeviceGuard dg(ctx);
  if (!ctx || (K && !d_pairs) || (E && !d_sp)) { set_error("szp_b200_rank_pairs_dev: null argument"); return -1; }
  if (K == 0 || E == 0) return 0;
  if (!ctx->scratch.reserve(rank_scratch_bytes(K, ctx->sm_count) + 4096)) return -1;
  if (rank_positions(ctx, static_cast<const uint2 *>(d_pairs), nullptr, K, E, absErrBound, d_sp)) return -1;
  return cuda_fail(cudaStreamSynchronize(ctx->stream), "rank") ? -1 : 0;
}

SZP_B200_API int szp_b200_encode_ints_dev(szp_b200_ctx *ctx, const int *d_vals, size_t n, int blockSize,
                                          unsigned char *d_out, size_t out_cap, size_t *out_bytes) {
  clear_error();
  DeviceGuard dg(ctx);
  if (!ctx || !d_vals || !d_out || !out_bytes) { set_error("szp_b200_encode_ints_dev: null argument"); return -1; }
  *out_bytes = 0;
  if (n == 0) { set_error("szp_b200_encode_ints_dev: no values"); return -1; }
  if (!valid_block_size(blockSize, "szp_b200_encode_ints_dev")) return -1;
  const unsigned long long nb = (n + blockSize - 1) / blockSize;
  if (!ctx->scratch.reserve(a256((nb / enc_tile_blocks(blockSize) + 2) * sizeof(TileDesc)) + 4096)) return -1;
  unsigned long long tot[3];
  const Geom g = make_geom(2, 1, (long long)n, 1);
  if (encode_pass(ctx, kEncInts, nullptr, d_vals, nullptr, n, blockSize, 1.0f, g, d_out, out_cap, nullptr, kCpNone,
                  nullptr, 0, tot))
    return -1;
  *out_bytes = 8 + tot[0];
  return 0;
}

}  // extern "C"
