// Host-side FP64 model: pupil fills, pupils, source sampling, SOCS kernel
// build.  This is the set-up half of the engine; everything per-image runs on
// the device.
#pragma once

#include <complex>
#include <cstdint>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/huv_b200.h"

namespace huv {

using cd = std::complex<double>;

// Error carrying a huv_status; caught at the C ABI and turned into a code.
struct Error : std::runtime_error {
  huv_status status;
  Error(huv_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

// ---------------------------------------------------------------- fills --
// Pupil-fill intensity at a normalised pupil coordinate (sigma units).
struct Fill {
  int kind = HUV_FILL_CONVENTIONAL;
  double p[4] = {0, 0, 0, 0};
  // Precomputed pole centres for the dipole fill.
  double pole[2][2] = {{0, 0}, {0, 0}};
  void prepare();
  double operator()(double x, double y) const;
};

// ---------------------------------------------------------------- optics --
struct Optics {
  int kind = HUV_OPTICS_PROJECTION;
  double na = 0.75;
  double flare = 0.02;
  double medium = 1.0;
  double obscuration = 0.0;
  double transmission = 1.0;
  bool paraxial = false;
  double cutoff(double lambda) const { return na / lambda; }
  cd pupil(double fx, double fy, double z, double lambda) const;
};

double defocus_phase(double z, double na_rho, double medium, double lambda, bool paraxial);

// ---------------------------------------------------------------- source --
struct SourcePoint {
  double sx, sy, w;
};

std::vector<SourcePoint> sample_source(const Fill& fill, int points_per_axis, double df_sigma);

// ---------------------------------------------------------------- kernels --
struct KernelSet {
  int n = 0;                       // grid size
  std::vector<int64_t> support;    // flat indices i*n + j (row i = y order)
  std::vector<double> eigenvalues; // raw (absolute), decreasing, retained
  std::vector<double> all_values;  // every eigenvalue of the decomposition (re-truncation)
  std::vector<cd> values;          // K * S, kernel-major
  double trace = 0, clear_field = 0, pupil_peak = 0;
  int method = 0;                  // 0 dense_tcc, 1 dense_gram
  int num_columns = 0;
  bool exceeds_nyquist = false;
  double defocus_nm = 0, wavelength_nm = 0;
  int num_kernels() const { return static_cast<int>(eigenvalues.size()); }
  int band_half_width() const;     // max |order| over the support
  double divisor(int normalization) const;  // 0 if images stay absolute
};

int select_kernel_count(const std::vector<double>& values, double trace, int max_kernels,
                        double fraction);

KernelSet build_kernels(const std::vector<SourcePoint>& points, const Optics& optics, int n,
                        double pixel_nm, double lambda, int max_kernels, double fraction,
                        double defocus_nm, int force_method = -1);

// The same kernel set built with the A matrix and its products on GPU
// `device` in FP64 (csrc/cuda/kbuild.cu); reference_rule selects the
// reference's solver rule (randomized subspace iteration for large problems).
KernelSet build_kernels_device(const std::vector<SourcePoint>& points, const Optics& optics, int n,
                               double pixel_nm, double lambda, int max_kernels, double fraction,
                               double defocus_nm, int device, bool reference_rule);

// Hermitian eigensolver (column-major n x n input, both triangles read).
// Returns eigenvalues in decreasing order and the first `count` eigenvectors
// (column-major n x count).
void hermitian_eigen(int n, const std::vector<cd>& h, std::vector<double>& values,
                     std::vector<cd>& vectors, int count_hint_max);

// Worker count for host-parallel loops.
int host_threads();
void parallel_for(int64_t n, const std::function<void(int64_t, int64_t)>& body);
// While alive, parallel_for on this thread runs serially (for callers that
// parallelise at a coarser grain themselves).
struct SerialHostScope {
  SerialHostScope();
  ~SerialHostScope();
  bool prev;
};

}  // namespace huv
