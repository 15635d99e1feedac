/*
 * huv_b200.h - C ABI of the B200 SOCS aerial-image engine.
 *
 * The boundary replaces the reference's imaging call
 *   AerialImageEngine::{with_settings, compute, compute_from_transmittance,
 *   compute_from_spectrum, kernels, kernel_diagnostics, clear_field_intensity}
 *   (crates/highuvlith-core/src/aerial.rs:1521-1967)
 * and its Python face SimulationEngine (crates/highuvlith-py/src/py_simulation.rs:89-566).
 *
 * Rules: no exceptions cross the ABI; every call returns a huv_status and the
 * message of the last failure on the calling thread is in huv_last_error().
 * Output buffers are caller-owned.  Device pointers are CUDA device addresses
 * on the engine's device; host pointers are ordinary host memory.  One engine
 * may be used from several host threads; calls on one engine are serialised
 * internally.  Streams are passed as `void*` (a cudaStream_t; NULL = the
 * legacy default stream).  FP64 is used only on the host while building
 * kernels (TCC assembly, Hermitian eigensolve, truncation); images are FP32.
 */
#ifndef HUV_B200_H
#define HUV_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes; mirror LithographyError (crates/highuvlith-core/src/error.rs:1-72)
 * plus device-side failures. */
typedef enum {
  HUV_OK = 0,
  HUV_ERR_INVALID_PARAMETER = 1,       /* InvalidParameter */
  HUV_ERR_GRID_NOT_POWER_OF_TWO = 2,   /* GridSizeNotPowerOfTwo */
  HUV_ERR_NO_DIFFRACTION_ORDERS = 3,   /* NoDiffractionOrders */
  HUV_ERR_PUPIL_SAMPLING_TOO_DENSE = 4,/* PupilSamplingTooDense */
  HUV_ERR_TCC_DECOMPOSITION = 5,       /* TccDecomposition (eigensolver failed) */
  HUV_ERR_DIMENSION_MISMATCH = 6,      /* DimensionMismatch */
  HUV_ERR_NUMERICAL = 7,               /* NumericalError */
  HUV_ERR_CUDA = 8,                    /* a CUDA runtime call failed */
  HUV_ERR_OUT_OF_MEMORY = 9,           /* device or host allocation failed */
  HUV_ERR_DEVICE_TIMEOUT = 10,         /* a bounded device-side wait gave up */
  HUV_ERR_UNSUPPORTED = 11             /* valid request the library does not serve */
} huv_status;

/* Pupil fills (crates/highuvlith-core/src/source.rs:163-186, 1178-1248) plus the
 * quasar fill (four annular sectors centred on the diagonals), which the
 * reference expresses as a custom LithographySource::intensity_at. */
typedef enum {
  HUV_FILL_CONVENTIONAL = 0, /* p0 = sigma */
  HUV_FILL_ANNULAR = 1,      /* p0 = sigma_inner, p1 = sigma_outer */
  HUV_FILL_QUADRUPOLE = 2,   /* p0 = sigma_center, p1 = sigma_radius, p2 = opening_angle_deg */
  HUV_FILL_DIPOLE = 3,       /* p0 = sigma_center, p1 = sigma_radius, p2 = orientation_deg */
  HUV_FILL_GAUSSIAN = 4,     /* p0 = sigma (CoherentGaussian) */
  HUV_FILL_QUASAR = 5        /* p0 = sigma_inner, p1 = sigma_outer, p2 = opening_angle_deg */
} huv_fill_kind;

typedef struct {
  double wavelength_nm; /* LithographySource::wavelength_nm (source.rs:59) */
  int32_t fill;         /* huv_fill_kind */
  double p[4];
} huv_source;

/* Optics (optics/mod.rs:193-357, optics/euv.rs:51-160): scalar pupils. */
typedef enum { HUV_OPTICS_PROJECTION = 0, HUV_OPTICS_EUV = 1 } huv_optics_kind;

typedef struct {
  int32_t kind;               /* huv_optics_kind */
  double na;
  double flare_fraction;      /* ProjectionOptics::flare_fraction / EuvProjectionOptics::flare */
  double immersion_index;     /* ProjectionOptics only (1 = dry) */
  double central_obscuration; /* EUV only, fraction of NA */
  double transmission;        /* EUV only (1 in the presets) */
  int32_t paraxial_defocus;   /* 0 = exact defocus phase */
} huv_optics;

typedef struct {
  int32_t size;    /* GridConfig::size, power of two */
  double pixel_nm; /* GridConfig::pixel_nm */
} huv_grid;

/* ImagingSettings (aerial.rs:166-206), scalar imaging, exact defocus. */
typedef struct {
  int32_t max_kernels;            /* >= 1 */
  double kernel_energy_fraction;  /* (0, 1] */
  int32_t source_points_per_axis; /* 0 = adaptive sampling, n >= 1 = n x n grid */
  int32_t normalization;          /* 0 = clear field (relative), 1 = absolute */
  int32_t kernel_cache_capacity;  /* kernel sets kept per engine (focus planes) */
  int32_t kernel_build;           /* huv_kernel_build: where the FP64 kernel set is built */
} huv_settings;

/* Where the FP64 SOCS kernel set is built (KernelBuilder::build, aerial.rs:1041-1317). */
typedef enum {
  HUV_BUILD_HOST = 0,          /* host C++, dense Hermitian eigensolve */
  HUV_BUILD_DEVICE = 1,        /* A matrix and its products on the GPU (FP64), dense eigensolve */
  HUV_BUILD_DEVICE_RULE = 2    /* as 1, with the reference's solver rule (aerial.rs:1116-1128):
                                  randomized subspace iteration when the problem is large */
} huv_kernel_build;

/* KernelDiagnostics (aerial.rs:254-276). method: 0 dense_tcc, 1 dense_gram. */
typedef struct {
  int32_t num_kernels;
  double captured_energy_fraction;
  int32_t num_frequencies;
  int32_t num_columns;
  int32_t method;
  int32_t support_exceeds_nyquist;
  double clear_field_intensity;
  int32_t normalized;
  int32_t band_half_width; /* h: the support lies in orders [-h, h]^2 */
  int32_t num_source_points;
} huv_diagnostics;

/* Mask input kinds for the batched image call. */
typedef enum {
  HUV_INPUT_RASTER_U8 = 0,       /* N*N uint8 transmittance 0/1 (binary mask raster) */
  HUV_INPUT_RASTER_F32 = 1,      /* N*N float real transmittance */
  HUV_INPUT_TRANSMITTANCE_C64 = 2,/* N*N interleaved (re, im) float complex transmittance */
  HUV_INPUT_RECTS = 3            /* a huv_rect_clips in host memory: exact analytic spectrum */
} huv_input_kind;

/* A rectangle feature (mask.rs Feature::Rect): centre (x, y) and size (w, h)
 * in nm, field coordinates centred on the grid (pixel centres at
 * -L/2 + (j + 1/2) p).  Sub-pixel positions and overlaps are allowed. */
typedef struct {
  double x, y, w, h;
} huv_rect;

/* Rectangle clips for HUV_INPUT_RECTS: clip c is the union of
 * rects[offsets[c] .. offsets[c + 1]) with amplitude `feature` on a field of
 * amplitude `background` (binary dark field: feature 1, background 0; clear
 * field with opaque features: feature 0, background 1; an attenuated PSM puts
 * its complex absorber amplitude on either).  The spectrum is Mask::spectrum's
 * closed form (mask.rs:616-657, 1439-1503) over the disjoint cells of the
 * union (mask.rs:1365-1437), evaluated on the band on the GPU; pixel_transfer
 * is ignored (the spectrum is exact). */
typedef struct {
  const huv_rect* rects;
  const int32_t* offsets;   /* n_clips + 1 non-decreasing indexes into rects */
  double feature_re, feature_im;
  double background_re, background_im;
} huv_rect_clips;

/* Which device form evaluates the SOCS sum. */
typedef enum {
  HUV_FORM_AUTO = 0, /* hybrid where its kernels apply, else FFT (huv_plan_* times the forms per group) */
  HUV_FORM_FFT = 1,  /* plain FP32 FFT form */
  HUV_FORM_TC = 2,   /* split-BF16x3 tcgen05 DFT-GEMM form (row transforms as FP32 FFTs) */
  HUV_FORM_TC_ROWS = 3, /* the same with the row transforms as tcgen05 DFT-GEMMs too */
  HUV_FORM_HYBRID = 4   /* FP32 FFT field pass on the evaluation grid + tcgen05 band interpolation
                           (separable, split-FP16x3, on evaluation grids of at most 192 points) */
} huv_form;

typedef struct {
  int32_t n_clips;
  int32_t input_kind;     /* huv_input_kind */
  const void* input;      /* device pointer: n_clips rasters of N*N, [y, x] row-major */
  int32_t pixel_transfer; /* 1: spectrum of a pixel-aligned raster (Mask::spectrum, mask.rs:630-635);
                             0: plain FFT of the samples (compute_from_transmittance, aerial.rs:1789) */
  double defocus_nm;      /* focus plane; kernel sets are built and cached per plane */
  int32_t form;           /* huv_form */
  int32_t eval_grid;      /* 0 = automatic (the smallest supported M > 4h: 160, 192 or 384 for the FFT
                             and hybrid forms where they beat the next power of two, a power of two of
                             at least 128 for the tensor-core y-contraction); N = evaluate on the full
                             grid; M < N (power of two, or 160 / 192 / 384 for the FFT and hybrid
                             forms, M > 4h) = exact evaluation on an M grid + exact band interpolation */
} huv_batch;

/* Last error message on this thread (never NULL). */
const char* huv_last_error(void);
/* Library version string. */
const char* huv_version(void);

/* Engine construction: source sampling + in-focus FP64 kernel build
 * (AerialImageEngine::with_settings, aerial.rs:1521-1637).  `device` is the
 * CUDA ordinal used for device kernel sets and images; the host build needs
 * no device. */
huv_status huv_engine_create(const huv_source* source, const huv_optics* optics,
                             const huv_grid* grid, const huv_settings* settings,
                             int32_t device, void** engine_out);
void huv_engine_destroy(void* engine);

/* A caller-built SOCS kernel set for one focus plane, in the layout of the
 * reference's KernelSet (aerial.rs:216-228) as AerialImageEngine::kernels
 * returns it (aerial.rs:1912-1942): for the set's grid the image before
 * flare is sum_k eigenvalues[k] |IFFT(kernels[k] . spectrum)|^2, with the
 * normalisation already folded into the eigenvalues. */
typedef struct {
  int32_t grid_size;               /* n: each kernel is n x n (power of two, 8 .. 8192) */
  double pixel_nm;                 /* grid pixel (reported only) */
  int32_t n_kernels;               /* K >= 1 */
  const double* eigenvalues;       /* K, non-increasing, >= 0 (KernelSet::eigenvalues) */
  const double* kernels;           /* K * n * n complex, (re, im) interleaved, k-major, FFT layout
                                      [ky][kx]; zero outside the frequency support (KernelSet::kernels) */
  double defocus_nm;               /* focus plane the set was built for (KernelSet::defocus_nm) */
  double wavelength_nm;            /* KernelSet::wavelength_nm (reported only) */
  double captured_energy_fraction; /* KernelSet::captured_energy_fraction, in (0, 1] */
  double flare_fraction;           /* uniform flare after the SOCS sum, in [0, 1)
                                      (the optics' flare, aerial.rs:1741-1748) */
} huv_kernel_set;

/* An engine over a caller-supplied kernel set (replaces the kernel upload
 * a Rust caller of AerialImageEngine::kernels would need; the reference's
 * engines always build their own kernels, aerial.rs:1521-1637).  The set is
 * copied (its support and values, as the engine's own sets are held), so
 * the caller's arrays may be freed on return.  The handle serves every
 * imaging entry point (huv_image_batch, _host, _noalloc, plans, ILT) at the
 * set's own focus plane: a batch names defocus_nm = 0 or the set's
 * defocus_nm; any other plane is HUV_ERR_UNSUPPORTED (the engine has no
 * source or optics to build it).  Destroy with huv_engine_destroy.  Needs no
 * device until the first imaging call. */
huv_status huv_kernelset_create(const huv_kernel_set* set, int32_t device, void** engine_out);

/* Source points (AerialImageEngine::source_points): xyw is count*3 doubles. */
huv_status huv_engine_source_points(void* engine, double* xyw, int32_t capacity, int32_t* count);

/* kernel_diagnostics (aerial.rs:1946-1958) at the centre wavelength. */
huv_status huv_engine_diagnostics(void* engine, double defocus_nm, huv_diagnostics* out);

/* clear_field_intensity (aerial.rs:1965-1967). */
huv_status huv_engine_clear_field(void* engine, double defocus_nm, double* out);

/* kernels(z) (aerial.rs:1912-1942): eigenvalues (already divided by the
 * normalisation) and dense N*N kernels in FFT layout, interleaved (re, im)
 * doubles, k-major.  Pass kernels = NULL to query the count only. */
huv_status huv_engine_kernels(void* engine, double defocus_nm, double* eigenvalues,
                              double* kernels, int32_t capacity, int32_t* count);

/* Batched aerial images on the device: out is n_clips*N*N floats (device),
 * [clip][y][x], pixel centres x_j = -L/2 + (j + 1/2) p.  Equivalent per clip to
 * compute(mask, z) (pixel_transfer = 1) or compute_from_transmittance(t, z)
 * (pixel_transfer = 0), normalisation and flare included (aerial.rs:1775-1816).
 * Device rasters and out must be 16-byte aligned (HUV_ERR_INVALID_PARAMETER). */
huv_status huv_image_batch(void* engine, const huv_batch* batch, float* out, void* stream);

/* Same call with HOST input and output buffers: copies in, images, copies out
 * on `stream` and synchronises it (the reference-facing end-to-end call). */
huv_status huv_image_batch_host(void* engine, const huv_batch* batch, float* out_host, void* stream);

/* Through-focus imaging: compute_through_focus (aerial.rs:1820-1825) and
 * process::batch_defocus (process.rs:1303-1313) for a batch of clips.
 * out (device) is n_planes*n_clips*N*N floats, [plane][clip][y][x]; the
 * batch's own defocus_nm is ignored.  Kernel sets of planes not yet cached
 * are built concurrently on the host (one plane per thread, FP64), then every
 * plane is imaged on `stream`. */
huv_status huv_image_focus_sweep(void* engine, const huv_batch* batch, const double* focus_nm, int32_t n_planes,
                                 float* out, void* stream);

/* Uneven batches (no counterpart in the reference, which images one clip per
 * call): clips of different grids, sources and kernel budgets in one CUDA
 * graph.  Each clip names the engine built for its source and grid and its
 * own kernel budget; the kernel count is re-truncated from that engine's
 * eigenvalues with the reference's rule (select_kernel_count,
 * aerial.rs:992-1029).  Inputs/outputs are device buffers fixed at creation:
 * write new rasters into the same buffers and launch again.  Engines must
 * outlive the plan and must not be used concurrently with its launches. */
typedef struct {
  void* engine;        /* engine for this clip's source and grid (in-focus kernel set) */
  int32_t max_kernels; /* this clip's kernel budget */
  int32_t input_kind;  /* huv_input_kind */
  const void* input;   /* device raster N*N */
  float* out;          /* device image N*N */
} huv_clip;

/* Group, autotune (autotune != 0: time each candidate form and evaluation
 * grid on the group's own clips; results cached per (N, h, K, kind)),
 * pre-allocate, run once and capture the whole batch into one CUDA graph. */
huv_status huv_plan_create(const huv_clip* clips, int32_t n_clips, int32_t pixel_transfer, int32_t autotune,
                           void** plan_out);
/* One cudaGraphLaunch of the whole uneven batch on `stream`. */
huv_status huv_plan_launch(void* plan, void* stream);
/* JSON description of the groups and the tuned choices. */
huv_status huv_plan_describe(void* plan, char* buf, int32_t capacity);
void huv_plan_destroy(void* plan);

/* Pixel ILT (crates/highuvlith-core/src/ilt.rs).  One process condition
 * (focus, dose, weight); m = sigmoid(beta theta), t = a + (1 - a) m with a
 * real absorber amplitude a (0 = binary). */
typedef struct {
  int32_t cost_kind;          /* 0 ImageFidelity, 1 ResistContour (ilt.rs:126-144) */
  double threshold;           /* ResistContour print threshold */
  double steepness;           /* ResistContour sigmoid steepness alpha */
  double beta;                /* mask sigmoid steepness (ILTConfig::sigmoid_steepness, default 4) */
  double tv_weight;           /* total-variation weight mu_TV (default 0.01) */
  double tv_epsilon;          /* TV smoothing (default 0.01) */
  double binarization_weight; /* mu_B (default 0) */
  double dose;                /* ProcessCondition::dose */
  double weight;              /* ProcessCondition::weight */
  double absorber;            /* real absorber amplitude a in [0, 1) */
  double defocus_nm;          /* ProcessCondition::defocus_nm */
} huv_ilt_params;

typedef struct {
  int32_t max_iterations;  /* ILTConfig::max_iterations */
  double learning_rate;    /* initial max |d theta| of a step (default 0.5) */
  double convergence_tol;  /* relative decrease tolerance (default 1e-4) */
} huv_ilt_opt;

/* Cost and exact adjoint gradient dC/dtheta for n_masks masks at once
 * (IltProblem::cost_and_gradient_with, ilt.rs:667-738).  theta, target, grad:
 * device arrays of n_masks*N*N floats; cost_host: n_masks doubles (the call
 * synchronises `stream`).  grad = NULL computes the cost only (IltProblem::cost,
 * ilt.rs:648-659). */
huv_status huv_ilt_cost_grad(void* engine, const huv_ilt_params* params, int32_t n_masks, const float* theta,
                             const float* target, double* cost_host, float* grad, void* stream);

/* optimize_ilt's stage loop (run_stage, ilt.rs:755-866) for n_masks masks
 * concurrently: CG Polak-Ribiere+ with Armijo backtracking, per mask.  theta
 * (device) is updated in place.  final_cost, iterations: n_masks each (host);
 * history: n_masks*(max_iterations+1) doubles (host, NaN after termination)
 * or NULL. */
huv_status huv_ilt_optimize(void* engine, const huv_ilt_params* params, const huv_ilt_opt* opt, int32_t n_masks,
                            float* theta, const float* target, double* final_cost, int32_t* iterations,
                            double* history, void* stream);

/* Surrogate-assisted ILT: no reference counterpart (the reference's
 * optimizer, run_stage in ilt.rs:755-866, images every iterate with SOCS).
 * Costs and gradients come from an FNO image model (huv_fno_create, grid equal
 * to the engine's); every judge_every iterations exact SOCS re-images all
 * masks and, when the largest relative image error max|I_fno - I_socs| /
 * max|I_socs| exceeds error_bound, SOCS takes over for the rest of the run.
 * final_cost is always the exact SOCS cost. */
typedef struct {
  int32_t judge_every;         /* in: iterations between exact judges (5) */
  double error_bound;          /* in: relative image error that triggers takeover */
  int32_t surrogate_iterations;/* out: iterations costed by the surrogate */
  int32_t exact_iterations;    /* out: iterations costed by SOCS */
  int32_t takeover_iteration;  /* out: iteration SOCS took over at, -1 if never */
  int32_t n_judges;            /* out: judges run (first 64 errors kept) */
  double judge_errors[64];     /* out: worst relative error at each judge */
} huv_surrogate_ilt;

huv_status huv_ilt_optimize_surrogate(void* engine, void* fno, const huv_ilt_params* params, const huv_ilt_opt* opt,
                                      int32_t n_masks, float* theta, const float* target, huv_surrogate_ilt* sur,
                                      double* final_cost, int32_t* iterations, double* history, void* stream);

/* Fourier-neural-operator surrogate of the image (no counterpart in the
 * reference).  Maps a transmittance map (grid x grid floats, [y, x]) to the
 * normalised aerial image.  Width 64, `modes` x `modes` retained Fourier modes
 * (2 * modes along y), `layers` Fourier layers with GELU, projection 64 -> 128
 * -> 1.  Activations are stored in BF16, arithmetic is FP32, parameters FP32
 * (flat vector, seeded initialisation).  All array arguments are device
 * pointers unless named *_host. */
huv_status huv_fno_create(int32_t grid, int32_t width, int32_t modes, int32_t layers, int32_t proj, uint64_t seed,
                          int32_t device, void** fno_out);
void huv_fno_destroy(void* fno);
/* Copy the parameters to the host (host = NULL: count only). */
huv_status huv_fno_params(void* fno, float* host, int64_t capacity, int64_t* count);
huv_status huv_fno_set_params(void* fno, const float* host, int64_t count);
/* images = FNO(masks) for `batch` maps. */
huv_status huv_fno_forward(void* fno, int32_t batch, const float* masks, float* images, void* stream);
/* Gradient of the MSE to `targets` (or, targets = NULL, of sum(dout . FNO))
 * with respect to the parameters (param_grad) and the input (dmask). */
huv_status huv_fno_backward(void* fno, int32_t batch, const float* masks, const float* targets, const float* dout,
                            float* param_grad, float* dmask, float* loss_host, void* stream);
/* One Adam step on the MSE to `targets`. */
huv_status huv_fno_train_step(void* fno, int32_t batch, const float* masks, const float* targets, float lr,
                              float weight_decay, float* loss_host, void* stream);
/* Synchronise `stream` and report HUV_ERR_DEVICE_TIMEOUT if a bounded wait of
 * an FNO tensor-core kernel gave up since the last check (the results of those
 * calls are then not valid); the flag is cleared.  huv_fno_backward and
 * huv_fno_train_step check it themselves before returning; huv_fno_forward
 * leaves the stream asynchronous, so its callers check here. */
huv_status huv_fno_device_status(void* fno, void* stream);

/* Allocation-free variant of huv_image_batch (no counterpart in the
 * reference, which has no device path).  For callers that cannot call
 * cudaMalloc: applications whose memory pool already owns the device, and
 * latency-critical loops that cannot take cudaMalloc's device-wide
 * synchronisation.  Runs the plain FP32 FFT form with all intermediates in
 * one fixed 32 MiB device array compiled into the library (every GPU that
 * loads the library holds it until exit); batches are processed in chunks
 * that fit it, and a grid whose single clip does not fit is rejected with
 * HUV_ERR_INVALID_PARAMETER.  The first call on a device performs the
 * set-up (takes the array's device address).  All calls share the array:
 * calls that overlap on the GPU race.
 * form must be HUV_FORM_AUTO or HUV_FORM_FFT.  The engine's focus-plane
 * cache is only read: a plane it does not hold is built on the host for
 * this call and not cached, and on an engine whose kernels are built on the
 * GPU (kernel_build DEVICE or DEVICE_RULE) an uncached plane is rejected
 * with HUV_ERR_UNSUPPORTED (image it once with huv_image_batch first). */
huv_status huv_image_batch_noalloc(void* engine, const huv_batch* batch, float* out, void* stream);

/* Synchronise `stream` and report device-side failures of earlier calls on
 * this engine: HUV_ERR_DEVICE_TIMEOUT when a bounded device wait gave up
 * (the flag is cleared by the report).  The device calls above are
 * asynchronous and cannot report such failures themselves. */
huv_status huv_device_status(void* engine, void* stream);

/* Test hook for the give-up path of the bounded waits (no counterpart in
 * the reference).  ns > 0: every tensor-core GEMM launched afterwards (the
 * TC and hybrid forms) first waits ns nanoseconds on a barrier nothing
 * arrives at; the wait runs out, the kernel records the failure, unwinds
 * (in-flight copies drained, tensor memory freed) and the next
 * huv_device_status reports HUV_ERR_DEVICE_TIMEOUT.  ns <= 0 turns it off
 * (the default).  Process-wide; not for production use. */
huv_status huv_debug_probe_wait(int64_t ns);

/* Axis-aligned rectangles -> pixel-aligned binary rasters on the device
 * (mask.rs:1717-1741 for pixel-aligned Rect features on a dark- or bright-field
 * binary mask).  rects: n_rects*4 int32 (x0, y0, w, h) in pixels, row-major from
 * the field corner; clip_offsets: n_clips+1 prefix offsets into rects. */
huv_status huv_rasterize_rects(int32_t n, int32_t n_clips, const int32_t* rects_dev,
                               const int32_t* clip_offsets_dev, int32_t dark_field,
                               uint8_t* raster_out_dev, void* stream);

/* Measurement hooks (no counterpart in the reference, which has no device
 * path).  While profiling is on, each launch of the dominant SOCS kernel is
 * bracketed by CUDA events recorded on its own stream.  huv_profile_read
 * synchronises those events, returns the summed kernel time, the number of
 * bracketed launches, the number of all kernel launches made by this engine
 * since the last read, and the dominant kernel's name, then resets. */
huv_status huv_profile_enable(void* engine, int32_t on);
huv_status huv_profile_read(void* engine, double* dominant_ms, int32_t* dominant_launches,
                            int64_t* total_launches, char* dominant_name, int32_t name_capacity);
/* Every timed region since the last huv_profile_read as JSON
 * {"name": [launches, total_ms], ...} (does not reset; measurement hook). */
huv_status huv_profile_regions(void* engine, char* json, int32_t capacity);

#ifdef __cplusplus
}
#endif
#endif /* HUV_B200_H */
