// Build-time shim (oracle/_ref only): one of the reference's CUDA source
// files (REF_CUDA_SRC: the 2D and 3D topology libraries, the decompressors,
// the plain compressors) compiled where it lies.
//
// The library's common header does not compile under nvcc 12.9 (its
// dimension check jumps with goto over an initialised declaration, which is
// ill-formed C++), and these files use six names from it.  The shim defines
// the header's include guard and supplies those six with the header's
// contracts: on a CUDA error, a block size outside [1, max + 1], a dimension
// <= 0 or a product of dimensions that overflows size_t, print a message and
// exit the process.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>

#define SZP_CUDA_COMMON_CUH 1
#define SZP_CUDA_TOPO_MAX_BLOCK 256
#define SZP_CUDA_MAX_BLOCK 1024

#define CUDA_CHECK(call)                                                        \
  do {                                                                          \
    const cudaError_t ref_shim_status = (call);                                 \
    if (ref_shim_status != cudaSuccess) {                                       \
      std::fprintf(stderr, "reference CUDA call failed (%s:%d): %s\n", __FILE__, \
                   __LINE__, cudaGetErrorString(ref_shim_status));              \
      std::exit(EXIT_FAILURE);                                                  \
    }                                                                           \
  } while (0)
#define CUDA_CHECK_KERNEL() CUDA_CHECK(cudaGetLastError())

static inline void szp_cuda_validate_blocksize(int blockSize, int maxBlock, const char *fn) {
  if (blockSize >= 1 && blockSize <= maxBlock + 1) return;
  std::fprintf(stderr, "%s: block size %d not in [1, %d]\n", fn, blockSize, maxBlock + 1);
  std::exit(EXIT_FAILURE);
}

static inline size_t szp_cuda_validate_dims(int d1, int d2, int d3, const char *fn) {
  const bool positive = d1 > 0 && d2 > 0 && d3 > 0;
  const size_t a = positive ? (size_t)d1 : 0, b = positive ? (size_t)d2 : 0, c = positive ? (size_t)d3 : 0;
  if (!positive || a > SIZE_MAX / b || a * b > SIZE_MAX / c) {
    std::fprintf(stderr, "%s: invalid dimensions %d x %d x %d\n", fn, d1, d2, d3);
    std::exit(EXIT_FAILURE);
  }
  return a * b * c;
}

static inline size_t szp_cuda_validate_dims_2d(int rows, int cols, const char *fn) {
  return szp_cuda_validate_dims(rows, cols, 1, fn);
}

#include REF_CUDA_SRC
