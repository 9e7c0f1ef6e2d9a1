// Build-time shim (oracle/_ref only): exposes the reference 3D driver's
// host-side post-processing functions, compiled from the reference source
// file where it lies.  The driver's main() is renamed to an unused static
// function so that only the post-processing code is emitted.
#define main toposzp_ref_unused_main_3d
static int toposzp_ref_unused_main_3d(int, char **);
#include REF_DRIVER_3D
#undef main

extern "C" {
void ref3d_stencils(float *data, const float *orig, const int *types, const int *sp,
                    int d1, int d2, int d3, float eb, size_t n_sp)
{ apply_stencils_3d(data, orig, types, sp, d1, d2, d3, eb, n_sp); }
void ref3d_enforce(const int *types, float *data, const float *orig, int d1, int d2, int d3,
                   float eps, float eb)
{ restore_extrema_3d(types, data, orig, d1, d2, d3, eps, eb); }
int ref3d_rbf(float *data, const int *types, const float *orig, int d1, int d2, int d3,
              float eps, float eb)
{ return rbf_restore_saddles_3d(data, types, orig, d1, d2, d3, eps, eb); }
int ref3d_axis_saddles(float *data, const int *types, const float *orig, int d1, int d2,
                       int d3, float eb)
{ return stencil_restore_saddles_3d(data, types, orig, d1, d2, d3, eb); }
}
