// Build-time shim (oracle/_ref only): exposes the reference 2D driver's
// host-side post-processing functions, compiled from the reference source
// file where it lies.  The driver's main() is renamed to an unused static
// function so that only the post-processing code is emitted.
#define main toposzp_ref_unused_main_2d
static int toposzp_ref_unused_main_2d(int, char **);
#include REF_DRIVER_2D
#undef main

extern "C" {
void ref2d_stencils(float *data, const float *orig, const int *types, const int *sp,
                    int rows, int cols, float eb, size_t n_sp)
{ apply_stencils_clamped(data, orig, types, sp, rows, cols, eb, n_sp); }
void ref2d_enforce(const int *types, float *data, const float *orig, int rows, int cols,
                   float eps, float eb)
{ restore_extrema_clamped(types, data, orig, rows, cols, eps, eb); }
int ref2d_rbf(float *data, const int *types, const float *orig, int rows, int cols,
              float eps, float eb)
{ return rbf_restore_saddles(data, types, orig, rows, cols, eps, eb); }
}
