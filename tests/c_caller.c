/*
 * A plain C caller of include/huv_b200.h, as a reference-side binding (a
 * Rust `extern "C"` block or a ctypes table) would use it.
 *
 * Test infrastructure: tests/test_c_abi.py compiles this file with
 * -DHUV_EXPECT_<struct>_SIZE=<n> and -DHUV_EXPECT_<struct>_<field>=<offset>
 * taken from the Python ctypes mirror, so a layout mismatch between the
 * header and any binding built from the same field list fails the build.
 *
 *   c_caller layout          print every struct's size and field offsets
 *   c_caller create          build an engine on the host, print diagnostics
 *   c_caller image OUT.bin   also image two seeded clips through
 *                            huv_image_batch_host and write them (needs a GPU)
 */
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "huv_b200.h"

#define CHECK_SIZE(T) _Static_assert(sizeof(T) == HUV_EXPECT_##T##_SIZE, "sizeof " #T " differs from the binding")
#define CHECK_OFF(T, F) \
  _Static_assert(offsetof(T, F) == HUV_EXPECT_##T##_##F, "offsetof " #T "." #F " differs from the binding")

#ifdef HUV_EXPECT_huv_source_SIZE
CHECK_SIZE(huv_source);
CHECK_OFF(huv_source, wavelength_nm);
CHECK_OFF(huv_source, fill);
CHECK_OFF(huv_source, p);
CHECK_SIZE(huv_optics);
CHECK_OFF(huv_optics, kind);
CHECK_OFF(huv_optics, na);
CHECK_OFF(huv_optics, flare_fraction);
CHECK_OFF(huv_optics, immersion_index);
CHECK_OFF(huv_optics, central_obscuration);
CHECK_OFF(huv_optics, transmission);
CHECK_OFF(huv_optics, paraxial_defocus);
CHECK_SIZE(huv_grid);
CHECK_OFF(huv_grid, size);
CHECK_OFF(huv_grid, pixel_nm);
CHECK_SIZE(huv_settings);
CHECK_OFF(huv_settings, max_kernels);
CHECK_OFF(huv_settings, kernel_energy_fraction);
CHECK_OFF(huv_settings, source_points_per_axis);
CHECK_OFF(huv_settings, normalization);
CHECK_OFF(huv_settings, kernel_cache_capacity);
CHECK_OFF(huv_settings, kernel_build);
CHECK_SIZE(huv_diagnostics);
CHECK_OFF(huv_diagnostics, num_kernels);
CHECK_OFF(huv_diagnostics, captured_energy_fraction);
CHECK_OFF(huv_diagnostics, num_frequencies);
CHECK_OFF(huv_diagnostics, num_columns);
CHECK_OFF(huv_diagnostics, method);
CHECK_OFF(huv_diagnostics, support_exceeds_nyquist);
CHECK_OFF(huv_diagnostics, clear_field_intensity);
CHECK_OFF(huv_diagnostics, normalized);
CHECK_OFF(huv_diagnostics, band_half_width);
CHECK_OFF(huv_diagnostics, num_source_points);
CHECK_SIZE(huv_rect);
CHECK_SIZE(huv_rect_clips);
CHECK_OFF(huv_rect_clips, rects);
CHECK_OFF(huv_rect_clips, offsets);
CHECK_OFF(huv_rect_clips, feature_re);
CHECK_OFF(huv_rect_clips, background_im);
CHECK_SIZE(huv_batch);
CHECK_OFF(huv_batch, n_clips);
CHECK_OFF(huv_batch, input_kind);
CHECK_OFF(huv_batch, input);
CHECK_OFF(huv_batch, pixel_transfer);
CHECK_OFF(huv_batch, defocus_nm);
CHECK_OFF(huv_batch, form);
CHECK_OFF(huv_batch, eval_grid);
CHECK_SIZE(huv_kernel_set);
CHECK_OFF(huv_kernel_set, grid_size);
CHECK_OFF(huv_kernel_set, pixel_nm);
CHECK_OFF(huv_kernel_set, n_kernels);
CHECK_OFF(huv_kernel_set, eigenvalues);
CHECK_OFF(huv_kernel_set, kernels);
CHECK_OFF(huv_kernel_set, defocus_nm);
CHECK_OFF(huv_kernel_set, wavelength_nm);
CHECK_OFF(huv_kernel_set, captured_energy_fraction);
CHECK_OFF(huv_kernel_set, flare_fraction);
CHECK_SIZE(huv_clip);
CHECK_OFF(huv_clip, engine);
CHECK_OFF(huv_clip, max_kernels);
CHECK_OFF(huv_clip, input_kind);
CHECK_OFF(huv_clip, input);
CHECK_OFF(huv_clip, out);
CHECK_SIZE(huv_ilt_params);
CHECK_OFF(huv_ilt_params, cost_kind);
CHECK_OFF(huv_ilt_params, threshold);
CHECK_OFF(huv_ilt_params, absorber);
CHECK_OFF(huv_ilt_params, defocus_nm);
CHECK_SIZE(huv_ilt_opt);
CHECK_OFF(huv_ilt_opt, max_iterations);
CHECK_OFF(huv_ilt_opt, learning_rate);
CHECK_OFF(huv_ilt_opt, convergence_tol);
CHECK_SIZE(huv_surrogate_ilt);
CHECK_OFF(huv_surrogate_ilt, judge_every);
CHECK_OFF(huv_surrogate_ilt, error_bound);
CHECK_OFF(huv_surrogate_ilt, n_judges);
CHECK_OFF(huv_surrogate_ilt, judge_errors);
#endif

#define P(T) printf("%s\"%s\": %zu", first ? "" : ", ", #T, sizeof(T)), first = 0

static int fail(huv_status s, const char* what) {
  fprintf(stderr, "%s: status %d: %s\n", what, (int)s, huv_last_error());
  return 1;
}

/* The clips of the image mode: a centred clear square and a vertical line
 * pair on a dark field, 128 x 128 u8. */
static void clips(uint8_t* r) {
  memset(r, 0, 2 * 128 * 128);
  for (int y = 48; y < 80; ++y)
    for (int x = 48; x < 80; ++x) r[y * 128 + x] = 1;
  for (int y = 0; y < 128; ++y)
    for (int x = 0; x < 128; ++x)
      if ((x >= 40 && x < 56) || (x >= 72 && x < 88)) r[128 * 128 + y * 128 + x] = 1;
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  if (!strcmp(argv[1], "layout")) {
    int first = 1;
    printf("{");
    P(huv_source);
    P(huv_optics);
    P(huv_grid);
    P(huv_settings);
    P(huv_diagnostics);
    P(huv_rect);
    P(huv_rect_clips);
    P(huv_batch);
    P(huv_kernel_set);
    P(huv_clip);
    P(huv_ilt_params);
    P(huv_ilt_opt);
    P(huv_surrogate_ilt);
    printf("}\n");
    return 0;
  }
  /* EUV 13.5 nm, NA 0.33, conventional sigma 0.5, 128 x 128 at 1 nm, K <= 16 */
  huv_source src = {13.5, HUV_FILL_CONVENTIONAL, {0.5, 0, 0, 0}};
  huv_optics opt = {HUV_OPTICS_EUV, 0.33, 0.0, 1.0, 0.0, 1.0, 0};
  huv_grid grid = {128, 1.0};
  huv_settings st = {16, 1.0, 0, 0, 32, HUV_BUILD_HOST};
  void* eng = NULL;
  huv_status s = huv_engine_create(&src, &opt, &grid, &st, 0, &eng);
  if (s != HUV_OK) return fail(s, "huv_engine_create");
  huv_diagnostics d;
  s = huv_engine_diagnostics(eng, 0.0, &d);
  if (s != HUV_OK) return fail(s, "huv_engine_diagnostics");
  printf("{\"num_kernels\": %d, \"band_half_width\": %d, \"num_frequencies\": %d, \"clear_field\": %.17g}\n",
         d.num_kernels, d.band_half_width, d.num_frequencies, d.clear_field_intensity);
  /* a bad argument comes back as a status, never as an exception */
  huv_settings bad = st;
  bad.max_kernels = 0;
  void* none = NULL;
  if (huv_engine_create(&src, &opt, &grid, &bad, 0, &none) != HUV_ERR_INVALID_PARAMETER || none) return 3;
  if (!strcmp(argv[1], "image") && argc > 2) {
    uint8_t* r = (uint8_t*)malloc(2 * 128 * 128);
    float* out = (float*)malloc(sizeof(float) * 2 * 128 * 128);
    clips(r);
    huv_batch b = {2, HUV_INPUT_RASTER_U8, r, 1, 0.0, HUV_FORM_AUTO, 0};
    s = huv_image_batch_host(eng, &b, out, NULL);
    if (s != HUV_OK) return fail(s, "huv_image_batch_host");
    FILE* f = fopen(argv[2], "wb");
    if (!f || fwrite(out, sizeof(float), 2 * 128 * 128, f) != 2 * 128 * 128) return 4;
    fclose(f);
    free(r);
    free(out);
  }
  huv_engine_destroy(eng);
  return 0;
}
