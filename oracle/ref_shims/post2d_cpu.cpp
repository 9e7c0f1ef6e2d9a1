// Build-time shim (oracle/_ref only): the reference CPU decompress driver's
// 2D post-processing (example/testfloat_decompress_fastmode1_topology.cc:
// 43-660), compiled from the source file where it lies.  The driver's main()
// is renamed to an unused static function so only the post-processing code is
// emitted; ref2dcpu_post runs the driver's post-processing sequence (its main
// from the decoded field, types and sort positions on, :826-966) on caller
// buffers: extremum locks, false-negative saddles by eps-classification,
// parameter estimation and targeted RBF when there are any, stencils, then
// the restoration of the extrema from their types.
#define main toposzp_ref_unused_main_cpu2d
static int toposzp_ref_unused_main_cpu2d(int, char **);
#include REF_DRIVER_CPU2D
#undef main

extern "C" int ref2dcpu_post(float *data, const int *types, const int *sp, size_t extrema, int rows, int cols,
                             float errBound, double *sigma_out, int *ksize_out, float *eps_out) {
  const size_t n = (size_t)rows * (size_t)cols;
  int *types_orig = (int *)malloc(n * sizeof(int));
  int *sort_positions = (int *)calloc(n ? n : 1, sizeof(int));
  float *orig_decomp = (float *)malloc(n * sizeof(float));
  int *decomp_types = (int *)calloc(n, sizeof(int));
  unsigned char *fn_mask = (unsigned char *)calloc(n, 1);
  memcpy(types_orig, types, n * sizeof(int));
  size_t e = extrema < n ? extrema : n;
  if (sp && e) memcpy(sort_positions, sp, e * sizeof(int));
  unsigned char *locks = build_extrema_locks_from_types(types_orig, rows, cols);
  memcpy(orig_decomp, data, n * sizeof(float));
  int *mapping = extrema > 0 ? build_sort_position_mapping(types_orig, sort_positions, extrema, rows, cols) : NULL;
  const float eps = fmaxf(1e-6f, 0.1f * errBound);
  for (int i = 1; i < rows - 1; i++)
    for (int j = 1; j < cols - 1; j++) decomp_types[i * cols + j] = cls_idx(data, rows, cols, i, j, eps);
  int fn_saddles = 0;
  for (int i = 1; i < rows - 1; i++)
    for (int j = 1; j < cols - 1; j++) {
      const int idx = i * cols + j;
      if (types_orig[idx] == 3 && decomp_types[idx] != 3) { fn_mask[idx] = 1; fn_saddles++; }
    }
  *sigma_out = 0.0;
  *ksize_out = 0;
  *eps_out = 0.0f;
  if (fn_saddles > 0) {
    estimate_rbf_parameters(data, rows, cols, errBound, fn_saddles, sigma_out, ksize_out, eps_out);
    rbf_smooth_saddle_points_safe_extrema_aware_targeted(data, types_orig, locks, fn_mask, rows, cols, *sigma_out,
                                                         *ksize_out, *eps_out, errBound);
  }
  apply_stencils_on_critical_points(data, types_orig, sort_positions, mapping, rows, cols, errBound, extrema);
  restore_extrema_from_types(types_orig, data, orig_decomp, rows, cols, eps, errBound);
  free(types_orig); free(sort_positions); free(orig_decomp); free(decomp_types); free(fn_mask); free(locks);
  if (mapping) free(mapping);
  return fn_saddles;
}
