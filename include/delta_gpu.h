/* delta_gpu.h -- C ABI of the B200 (sm_100a) difference-imaging hot path.
 *
 * Drop-in boundary for tkillestein/delta 1.1.1: every entry point below
 * replaces one function of the reference's nanobind module `delta._core`
 * (src/bindings.cpp) and the C++ core function it wraps; the citation on each
 * declaration names both. Plain pointers and sizes only; no exceptions cross
 * this boundary. All functions return an int status (DGPU_OK == 0); the text of
 * the last failure on a context is available from dgpu_last_error().
 *
 * Memory: image arguments are either host or device pointers, chosen per call
 * by `mem` (DGPU_MEM_HOST: the library stages copies on its stream and
 * synchronises before returning; DGPU_MEM_DEVICE: pointers are used in place,
 * work is stream-ordered on the context's stream and the call returns without
 * a final synchronisation unless the algorithm itself needs a host decision).
 * Images are row-major float32 (index y*width + x), masks uint8 bit flags
 * (include/delta/image.hpp:14-22), optional layers are NULL.
 *
 * Threading: one context per host thread; calls on a context are serialised on
 * its stream.
 */
#ifndef DELTA_GPU_H_
#define DELTA_GPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define DGPU_OK 0
#define DGPU_ERR_INVALID 1   /* bad argument / shape: the reference's invalid_argument, shape runtime_error */
#define DGPU_ERR_RUNTIME 2   /* algorithmic failure the reference reports as runtime_error */
#define DGPU_ERR_CUDA 3      /* CUDA runtime error */
#define DGPU_ERR_LIMIT 4     /* a device loop hit its iteration cap (no spin, no trap) */
#define DGPU_ERR_CAPACITY 5  /* caller buffer too small; the needed size was written back */
#define DGPU_ERR_NO_DEVICE 6 /* no CUDA device / library built without one */

#define DGPU_MEM_HOST 0
#define DGPU_MEM_DEVICE 1

/* Arithmetic of the normal-equation build in dgpu_fit_kernel / dgpu_solve_*. */
#define DGPU_PREC_FP64 0  /* FP64 SIMT (accuracy reference) */
#define DGPU_PREC_FP32 1  /* "plain": FP32 SIMT products and accumulation */
#define DGPU_PREC_MIXED 2 /* "mixed": BF16x3 split tcgen05 products, FP32 accumulate,
                             FP64 cross-CTA reduce, Cholesky and one refinement step */
#define DGPU_PREC_TF32 3  /* "tf32": one TF32 tcgen05 product (kind::tf32), FP32 accumulate,
                             then as "mixed" (FP64 reduce, Cholesky, one refinement step) */

typedef struct dgpu_context dgpu_context;

/* ---- context ------------------------------------------------------------ */
int dgpu_device_count(int* count);
int dgpu_create(int device, dgpu_context** out);
void dgpu_destroy(dgpu_context* ctx);
/* Run subsequent work on a caller stream (a cudaStream_t); NULL restores the
 * context's own stream, which is non-blocking: it does NOT order after work on
 * the legacy default stream. A caller whose buffers are produced on the legacy
 * default stream passes cudaStreamLegacy ((void*)0x1) here. Switching streams
 * waits for the work already queued on the previous one; setting the current
 * stream again is free. */
int dgpu_set_stream(dgpu_context* ctx, void* stream);
int dgpu_synchronize(dgpu_context* ctx);
const char* dgpu_last_error(const dgpu_context* ctx);
/* Per-label device time of the last instrumented call (the reference's
 * DELTA_TIMING labels, src/timing.cpp:19-46); fills up to `cap` entries and
 * returns the count through *n. Enabled by DELTA_TIMING=1. */
int dgpu_drain_timing(dgpu_context* ctx, char (*labels)[64], double* seconds, int cap, int* n);
/* Switch the per-stage device timers on or off for this context (overrides
 * DELTA_TIMING); stage events are recorded without synchronising. */
int dgpu_set_timing(dgpu_context* ctx, int on);
/* Number of kernels this library has launched in the process so far. */
int dgpu_launch_count(unsigned long long* count);
/* The autotuner's choices so far, as text lines "key -> choice (candidate:
 * time, ...)". No reference counterpart: the library times the candidate
 * launch parameters of a kernel (e.g. the model convolve's tile height) on the
 * first call with a new shape class, keeps the fastest for the process, and
 * every candidate gives the same results. DELTA_AUTOTUNE=0 disables the
 * timing (the heuristic choice is used). Writes at most cap bytes (NUL
 * terminated) and the full size through *needed. */
int dgpu_autotune_table(char* out, size_t cap, size_t* needed);
/* Iteration cap of every union-find search and link loop of the catalog's
 * labelling on this context (no reference counterpart: the reference's CPU
 * union-find has no cap). A loop that reaches it stops, the pixels it left
 * unresolved get label 0, and the call returns DGPU_ERR_LIMIT; the context
 * stays usable. cap <= 0 restores the default (2^24, far above any real
 * chain). Lowering it is how the failure path is tested. */
int dgpu_set_label_loop_cap(dgpu_context* ctx, int cap);
/* Reduced-precision fallback of the kernel fit on this context (no reference
 * counterpart: the reference builds its normal equations in FP64 only). With
 * enabled != 0 (the default) a DGPU_PREC_MIXED / DGPU_PREC_TF32 fit whose
 * FP64 refinement correction exceeds 1e-2 of theta, whose solve is
 * non-finite, or whose chosen system needed the LDLT fallback is redone with
 * FP64 normal equations (precision_used reports which ran). With enabled == 0
 * the tensor-core result is returned as it is, with its refine_correction:
 * this is how the precision study measures each build's own error. */
int dgpu_set_precision_fallback(dgpu_context* ctx, int enabled);

/* ---- basis (host math) ---------------------------------------------------- */
/* GaussHermiteBasis::default_radius, src/basis.cpp:9-12. */
int dgpu_default_radius(double beta, int n_max);
/* gauss_hermite_basis1d, src/bindings.cpp:171-184 -> src/basis.cpp:14-59.
 * out: (n_max+1) x (2r+1) float64; radius 0 resolves the default. */
int dgpu_gauss_hermite_basis1d(double beta, int n_max, int radius, double* out, int* ksize);
/* gauss_hermite_kernels, src/bindings.cpp:187-206 -> src/basis.cpp:66-79.
 * orders: nc x 2 int32 (nx, ny); kernels: nc x ks x ks float32. */
int dgpu_gauss_hermite_kernels(double beta, int n_max, int radius, int32_t* orders,
                               float* kernels, int* ksize);
/* component_sums, src/basis.cpp:81-93; out: nc float64. */
int dgpu_component_sums(double beta, int n_max, int radius, double* out);

/* ---- thin-plate spline (host math) ---------------------------------------- */
/* grid_knots, src/spatial.cpp:113-129; out: (nx*ny) x 2 float64. */
int dgpu_grid_knots(double x0, double y0, double x1, double y1, int nx, int ny, double* out);
/* tps_design, src/bindings.cpp:487-490 -> src/spatial.cpp:67-97. out: m x k. */
int dgpu_tps_design(const double* knots, int k, const double* points, int64_t m, double* out);
/* tps_penalty, src/bindings.cpp:492-494 -> src/spatial.cpp:20-65. out: k x k. */
int dgpu_tps_penalty(const double* knots, int k, double* out);
/* tps_fit, src/bindings.cpp:496-500 -> src/spatial.cpp:131-140. out: k. */
int dgpu_tps_fit(const double* knots, int k, const double* points, int64_t m,
                 const double* values, double lam, double* out);
/* tps_evaluate, src/bindings.cpp:502-506. out: m. */
int dgpu_tps_evaluate(const double* knots, int k, const double* points, int64_t m,
                      const double* coeffs, double* out);

/* ---- kernel model ---------------------------------------------------------- */
/* A fitted solution: knots (k x 2), theta ((nc+1)*k, ordered
 * [c_0 | ... | c_{nc-1} | b], include/delta/solve.hpp:12-15), basis. */
typedef struct {
  const double* knots; /* host, k x 2 */
  int n_knots;
  const double* theta; /* host, n_theta */
  int64_t n_theta;
  double beta;
  int n_max;
  int radius; /* 0 -> default_radius */
} dgpu_model;

/* ---- convolution ------------------------------------------------------------ */
/* basis_convolve, src/bindings.cpp:209-227 -> src/convolve.cpp:90-113.
 * out: nc x h x w float32. */
int dgpu_basis_convolve(dgpu_context* ctx, int mem, const float* image, int64_t width,
                        int64_t height, double beta, int n_max, int radius, float* out);

/* ---- full-frame subtraction -------------------------------------------------- */
/* subtract, src/bindings.cpp:603-638 -> delta::subtract, src/subtract.cpp:429-966
 * (include/delta/subtract.hpp:75-78).
 * out_variance is written when either variance layer is given, out_mask when
 * either mask is given or saturation > 0 (pass NULL to skip otherwise). The
 * flags *has_variance / *has_mask report which outputs were produced. */
int dgpu_subtract(dgpu_context* ctx, int mem, int64_t width, int64_t height,
                  const float* science, const float* reference, const float* science_var,
                  const float* reference_var, const uint8_t* science_mask,
                  const uint8_t* reference_mask, const dgpu_model* model, double saturation,
                  float* out_difference, float* out_variance, uint8_t* out_mask,
                  int* has_variance, int* has_mask);

/* photometric_scale, src/bindings.cpp:696-708 -> src/fit.cpp:513-530. out: h x w. */
int dgpu_photometric_scale(dgpu_context* ctx, int mem, const double* knots, int n_knots,
                           const double* theta, int64_t n_theta, const double* component_sums,
                           int nc, int64_t height, int64_t width, float* out);
/* In-place sign flip of an n-element float image: the transients-positive
 * convention applied to the difference when the science frame is the one
 * convolved (python/delta/pipeline.py:687-689, np.negative on the host there). */
int dgpu_negate(dgpu_context* ctx, int mem, float* data, int64_t n);
/* In-place v *= scale (the scale rounded to float32 first, one float32
 * product per element) and v = value over n float32 elements: the variance
 * rescale of Subtractor(rescale_variance=True) (python/delta/pipeline.py:
 * 692-698, `variance * variance_scale` on float32 there) and the constant
 * score variance of a frame without variance layers (pipeline.py:774-779). */
int dgpu_scale(dgpu_context* ctx, int mem, float* data, int64_t n, double scale);
/* Median of z^2 = D^2 / Var (FP64) over the pixels with Var > 0, D and Var
 * finite and mask 0 (mask may be NULL): the statistic of the variance
 * rescale (python/delta/pipeline.py _variance_rescale_factor, numpy's median
 * of the FP64 values, the two middle values averaged for an even count),
 * selected on the device. *count receives the number of good pixels (0 leaves
 * *median = 0). */
int dgpu_z2_median(dgpu_context* ctx, int mem, int64_t n, const float* difference, const float* variance,
                   const uint8_t* mask, double* median, int64_t* count);
int dgpu_fill(dgpu_context* ctx, int mem, float* data, int64_t n, double value);
/* Copy of `bytes` from device memory to pinned host memory, ordered on the
 * context's stream through the copy engine (asynchronous: synchronize that
 * stream before reading host_dst). No counterpart in the reference, which has
 * no device: it serves the batch layer. Every stream's device-to-host
 * copy-engine transfers share one queue in submission order, so the library
 * keeps its own small read-backs (status words, counts, stamp lists, theta,
 * catalog rows) out of that queue: they go by SM stores into a mapped pinned
 * area of the context, and a frame's 200 MB download queued here does not
 * hold the frames still computing. Errors: DGPU_ERR_INVALID when host_dst is
 * not pinned host memory or device_src is not device memory. */
int dgpu_copy_to_host(dgpu_context* ctx, void* host_dst, const void* device_src, int64_t bytes);
/* ---- FITS image layers ------------------------------------------------------------ */
/* read_fits, src/bindings.cpp:128-145 -> delta::io::read_image, src/io.cpp:79-130.
 * Host only (no device, no context). dgpu_fits_probe gives the data layer's
 * size and whether VARIANCE / MASK extensions exist; dgpu_fits_read fills
 * caller buffers of width * height values (variance / mask may be NULL to
 * skip a layer), and fails with DGPU_ERR_INVALID without writing when the
 * file's data layer is not width x height. The data layer is the primary image, or the DIFFERENCE
 * extension when the primary holds no 2-D image. Any BITPIX is converted with
 * BSCALE / BZERO; tile-compressed HDUs are refused (DGPU_ERR_RUNTIME). Errors
 * read back with dgpu_last_error(NULL). */
int dgpu_fits_probe(const char* path, int64_t* width, int64_t* height, int* has_variance, int* has_mask);
int dgpu_fits_read(const char* path, int64_t width, int64_t height, float* data, float* variance,
                   uint8_t* mask);
/* write_fits, src/bindings.cpp:147-166 -> delta::io::write_image, src/io.cpp:132-178:
 * a float32 primary image, then VARIANCE (float32) and MASK (byte) image
 * extensions when given. Fails if the file exists unless overwrite != 0. */
int dgpu_fits_write(const char* path, int64_t width, int64_t height, const float* data, const float* variance,
                    const uint8_t* mask, int overwrite);
/* photometric_scale_at, src/bindings.cpp:711-719 -> src/fit.cpp:532-544. out: m. */
int dgpu_photometric_scale_at(const double* knots, int n_knots, const double* theta,
                              int64_t n_theta, const double* component_sums, int nc,
                              const double* points, int64_t m, double* out);

/* ---- penalised GLS + stamp fit ------------------------------------------------ */
/* Result of a GLS solve (include/delta/solve.hpp:16-26) plus the
 * fit_kernel diagnostics (include/delta/fit.hpp:16-37). Array members are
 * caller buffers: theta[(nc+1)*k], lambda_grid / gcv_curve[n_lambda],
 * component_sums[nc], stamp_*[n_stamps supplied]; the stamp arrays receive
 * the n_stamps_total contributing stamps in supplied order. */
typedef struct {
  double* theta;
  double* lambda_grid;
  double* gcv_curve;
  double* component_sums;
  int32_t* stamp_x;
  int32_t* stamp_y;
  double* stamp_chi2;
  uint8_t* stamp_accepted;
  int n_components;
  int n_spatial;
  double lambda;
  double gcv;
  double effective_dof;
  double rss;
  double reduced_chi2;
  int64_t n_pixels;
  int n_stamps_used;
  int n_stamps_total;
  int n_stamps_rejected;
  int64_t cv_exact_design_bytes;
  int n_lambda_out; /* entries written to lambda_grid / gcv_curve (0 for a fixed-lambda solve) */
  /* Beyond the reference's fields: the normal-equation arithmetic that produced
   * theta (DGPU_PREC_*; mixed falls back to fp64 when its FP64 refinement step
   * shows the BF16x3 solve too inaccurate for the system's conditioning), and
   * ||correction|| / ||theta|| of the last mixed refinement step (0 otherwise). */
  double refine_correction;
  int precision_used;
  /* 1 when the selected system's Cholesky met a non-positive pivot and theta /
   * edf come from the pivoted LDL^T fallback (the reference's LLT -> LDLT
   * fallback, src/solve.cpp:177-181); 0 otherwise. */
  int used_ldlt;
} dgpu_gls_result;

/* fit_kernel, src/bindings.cpp:643-693 -> delta::fit_kernel, src/fit.cpp:63-511
 * (include/delta/fit.hpp:65-72). Images follow `mem`; knots, stamp lists and
 * lambda_grid are host arrays. `precision` is a DGPU_PREC_* value selecting the
 * normal-equation arithmetic (the solve is FP64 in every mode). */
int dgpu_fit_kernel(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* science,
                    const float* reference, const float* science_var, const float* reference_var,
                    const uint8_t* science_mask, const uint8_t* reference_mask, const double* knots,
                    int n_knots, const int32_t* stamp_x, const int32_t* stamp_y, int n_stamps,
                    int stamp_radius, double beta, int n_max, int radius, const double* lambda_grid,
                    int n_lambda, double clip_sigma, int clip_iterations, int min_stamps, int cv_folds,
                    int precision, dgpu_gls_result* out);

/* solve_gls / solve_gls_gcv / solve_gls_cv, src/bindings.cpp:530-566 ->
 * src/solve.cpp:208-225, 421-431. Host arrays: points m x 2, target / weights
 * m, bn m x nc (row-major), group m (CV). lam is used by solve_gls only. */
int dgpu_solve_gls(dgpu_context* ctx, const double* knots, int n_knots, const double* points, int64_t m,
                   const double* target, const double* weights, const double* bn, int nc, double lam,
                   int precision, dgpu_gls_result* out);
int dgpu_solve_gls_gcv(dgpu_context* ctx, const double* knots, int n_knots, const double* points, int64_t m,
                       const double* target, const double* weights, const double* bn, int nc,
                       const double* lambda_grid, int n_lambda, int precision, dgpu_gls_result* out);
int dgpu_solve_gls_cv(dgpu_context* ctx, const double* knots, int n_knots, const double* points, int64_t m,
                      const double* target, const double* weights, const double* bn, int nc,
                      const double* lambda_grid, int n_lambda, const int32_t* group, int n_groups,
                      int precision, dgpu_gls_result* out);

/* ---- differentiation: weighted chi^2 of the kernel model -------------------------- */
/* No reference counterpart (the reference has no gradient code). The model is
 * the subtraction's (src/subtract.cpp:466-639, the same sanitised reference,
 * lattice-blended fields and basis) with the kernel shifted by (dx, dy) pixels
 * and its convolved part scaled by `scale`:
 *   M = scale * sum_c a_c(x) [g_nx(u - dx) g_ny(v - dy) (*) R~](x) + b(x),
 *   chi2 = sum_x W(x) (S(x) - M(x))^2 over pixels with W > 0 and a finite S.
 * Images follow `mem`; weights (W) is float32 h x w, 0 excluding a pixel;
 * reference_mask may be NULL. Outputs (host): chi2; the gradients are
 * optional (NULL skips them): grad_theta (n_theta, same layout as theta),
 * grad_shift (2: d/ddx, d/ddy), grad_scale (1), and grad_reference (h x w
 * float32, follows `mem`; the correlation of the field-weighted residual with
 * the flipped kernel field, 0 where the reference was replaced by the fill
 * value, which is held constant). The convolved basis images are recomputed
 * per tile, never stored. n_max <= 8. */
int dgpu_kernel_chi2(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* science,
                     const float* reference, const uint8_t* reference_mask, const float* weights,
                     const dgpu_model* model, double dx, double dy, double scale, double* chi2, double* grad_theta,
                     double* grad_shift, double* grad_scale, float* grad_reference);

/* GCV score of the stamp fit as a function of log lambda, the kernel shift and
 * the scale, with its gradient through the adjoint of the normal-equation map
 * (no reference counterpart). The stamp rows are fit_kernel's
 * (src/fit.cpp:63-229, first-pass weights 1 / (Var_t + Var_c), no clipping)
 * with every B_n convolved with the basis shifted by (dx, dy) and scaled by
 * `scale`; the solve at lambda = exp(log_lambda) is the reference's solve_at
 * (src/solve.cpp:147-193): GCV = n RSS / (n - edf)^2. Images follow `mem`;
 * knots and stamp lists are host arrays. Outputs (host): values[4] = {gcv,
 * rss, edf, n}; theta ((nc+1)*k, optional); grad_gcv[4] and grad_rss[4]
 * (optional) = d/d{log lambda, dx, dy, scale} of GCV and of the weighted RSS.
 * At most 32 knots. */
int dgpu_stamp_gcv(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* science,
                   const float* reference, const float* science_var, const float* reference_var,
                   const uint8_t* science_mask, const uint8_t* reference_mask, const double* knots, int n_knots,
                   const int32_t* stamp_x, const int32_t* stamp_y, int n_stamps, int stamp_radius, double beta,
                   int n_max, int radius, double log_lambda, double dx, double dy, double scale, double* values,
                   double* theta, double* grad_gcv, double* grad_rss);

/* ---- noise decorrelation (ZOGY) ------------------------------------------------ */
/* decorrelate, src/bindings.cpp:766-792 -> delta::decorrelate, src/noise.cpp:228-483
 * (include/delta/noise.hpp:64-68). Outputs: whitened difference and its
 * post-whitening variance, h x w float32. */
int dgpu_decorrelate(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* difference,
                     const dgpu_model* model, const float* var_science, const float* var_reference, int block,
                     int kernel_cell_blocks, float* out_difference, float* out_variance);
/* whiten_score_psf, src/bindings.cpp:796-874 -> delta::whiten_psf,
 * src/noise.cpp:485-533. psf / out: host, psf_size^2. */
int dgpu_whiten_score_psf(dgpu_context* ctx, int mem, const float* psf, int psf_size, const dgpu_model* model,
                          int64_t width, int64_t height, const float* var_science, const float* var_reference,
                          int block, float* out);
/* decorrelate_block, src/bindings.cpp:725-745 -> src/noise.cpp:98-137. Host arrays. */
int dgpu_decorrelate_block(dgpu_context* ctx, const float* image, int n, const float* kernel, int ksize,
                           double var_science, double var_reference, float* out);
/* decorrelation_kernel, src/bindings.cpp:748-760 -> src/noise.cpp:139-161. Host arrays. */
int dgpu_decorrelation_kernel(dgpu_context* ctx, const float* kernel, int ksize, double var_science,
                              double var_reference, int n, float* out);

/* ---- stamp selection ------------------------------------------------------------ */
typedef struct {
  int stamp_radius;       /* 15 */
  double threshold_sigma; /* 5.0 */
  int max_stamps;         /* 200 */
  double saturation;      /* 0.0 */
  int isolation_radius;   /* 0 -> 2 * stamp_radius */
  int border;             /* 0 -> stamp_radius */
  int fwhm_radius;        /* 0 -> max(5, stamp_radius / 2) */
  int match_radius;       /* 2 */
} dgpu_detect_params;

/* Allocation-free dgpu_estimate_background (no reference counterpart).
 * For callers that must not allocate device memory during processing: for
 * example a loop under a fixed memory budget, or code that cannot accept the
 * device-wide synchronisation that cudaMalloc/cudaFree imply. It needs no
 * context: it runs on the calling thread's current device, on `stream`
 * (NULL = legacy default stream), with `data` (float32, width x height) and the
 * optional `mask` (uint8) in device memory, and returns after synchronising
 * `stream`. Its scratch is one fixed array of 2 MiB + 1 KiB per device inside
 * the library (it holds the at most 2^19 sample keys of any frame below 2^31
 * pixels); the select state in it is cleared at the start of every call.
 * Limits: frames up to 2^31 - 1 pixels (larger -> DGPU_ERR_INVALID). Every
 * call looks up that array's address on the current device
 * (cudaGetSymbolAddress, which allocates nothing); the first call on a device
 * may also load the library's device code, so make it before any stream
 * capture. Calls that overlap in time on the
 * same device (other streams or threads) share the array and race: serialise
 * them. Results equal dgpu_estimate_background's (median, 1.4826 * MAD).
 * Errors: status code, text from dgpu_last_error(NULL). */
int dgpu_estimate_background_noalloc(const float* data, const uint8_t* mask, int64_t width, int64_t height,
                                     void* stream, double* median, double* sigma);
/* estimate_background, src/bindings.cpp:232-237 -> src/detect.cpp:84-113. */
int dgpu_estimate_background(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* data,
                             const uint8_t* mask, double* median, double* sigma);
/* detect_stamps, src/bindings.cpp:240-274 -> src/detect.cpp:159-241. Host output
 * columns hold up to `capacity` stamps; *count receives the number found. */
int dgpu_detect_stamps(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* data,
                       const uint8_t* mask, const dgpu_detect_params* params, int capacity, int32_t* x, int32_t* y,
                       double* flux, double* snr, double* fwhm, int* count);
/* select_stamps, src/bindings.cpp:278-315 -> src/detect.cpp:260-314 (catalog
 * positions when cat_x / cat_y are given, host arrays). */
int dgpu_select_stamps(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* science,
                       const float* reference, const uint8_t* science_mask, const uint8_t* reference_mask,
                       const int32_t* cat_x, const int32_t* cat_y, int n_cat, const dgpu_detect_params* params,
                       int capacity, int32_t* x, int32_t* y, double* fwhm_science, double* fwhm_reference,
                       double* median_fwhm_science, double* median_fwhm_reference, int* direction_is_reference,
                       int* count);
/* Median unit-sum PSF stamp of the listed sources (the score path's
 * _estimate_psf, python/delta/pipeline.py:285-302). out: host (2r+1)^2. */
int dgpu_estimate_psf(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* image,
                      const int32_t* xs, const int32_t* ys, int n, int radius, float* out);
/* weighted_mean, src/bindings.cpp:107-124. */
int dgpu_weighted_mean(dgpu_context* ctx, int mem, int64_t n, const float* data, const float* variance,
                       const uint8_t* mask, double* out);

/* ---- matched filter ---------------------------------------------------------- */
/* matched_filter, src/bindings.cpp:878-898 -> src/noise.cpp:535-632
 * (include/delta/noise.hpp:88-93). out: h x w float32. */
int dgpu_matched_filter(dgpu_context* ctx, int mem, int64_t width, int64_t height,
                        const float* image, const float* psf, int psf_size,
                        const float* variance, float* out);

/* ---- catalog ----------------------------------------------------------------- */
typedef struct {
  double threshold_sigma;        /* 5.0 */
  double threshold_sigma_dipole; /* 3.0 */
  double expected_fwhm;          /* 3.5 */
  double fwhm_tolerance_lo;      /* 0.3 */
  double fwhm_tolerance_hi;      /* 3.0 */
  int aperture_radius;           /* 0 */
  int exclude_bad_pixels;        /* 1 */
  int return_negative;           /* 0 */
  int fit_psf_shape;             /* 0 */
  double shape_chi2_tolerance;   /* 3.0 */
  double bright_star_radius;     /* 0.0 */
  int max_shape_fit;             /* 5000 */
} dgpu_catalog_params;

/* Column pointers for dgpu_catalog_fetch (host memory, `count` entries each). */
typedef struct {
  double* x;
  double* y;
  int32_t* peak_x;
  int32_t* peak_y;
  double* peak_snr;
  int32_t* n_pix;
  double* flux;
  double* expected_n_pix;
  double* fwhm_ratio;
  uint8_t* fwhm_consistent;
  uint8_t* mask_flags;
  uint8_t* is_dipole;
  uint8_t* quality;
  double* psf_chi2;
  int32_t* psf_chi2_dof;
  double* psf_amplitude;
  double* psf_amplitude_err;
  uint8_t* shape_consistent;
  double* bright_star_dist;
  uint8_t* near_bright_star;
} dgpu_catalog_columns;

/* build_catalog, src/bindings.cpp:348-483 -> delta::build_catalog,
 * src/catalog.cpp:600-697 (include/delta/catalog.hpp:117-121).
 * Labels, reduces and (optionally) enriches on the device; the entries stay in
 * the context until dgpu_catalog_fetch copies them out. *count receives the
 * number of entries. variance / psf / bright_* are optional (NULL). */
int dgpu_build_catalog(dgpu_context* ctx, int mem, int64_t width, int64_t height,
                       const float* score, const float* difference, const uint8_t* mask,
                       const dgpu_catalog_params* params, const float* variance,
                       const float* psf, int psf_size, const double* bright_x,
                       const double* bright_y, int n_bright, int* count);
int dgpu_catalog_fetch(dgpu_context* ctx, const dgpu_catalog_columns* cols, int count);
/* Label image of the last dgpu_build_catalog (polarity it returned), int32 h x w,
 * 0 = background, 1..n numbered by each component's first pixel in raster order
 * (the numbering of src/catalog.cpp:105-261). */
int dgpu_catalog_labels(dgpu_context* ctx, int mem, int32_t* labels, int64_t n);

/* ---- batch of frames ---------------------------------------------------------- */
/* One frame pair: row-major layers of width x height (host or device per the
 * call's `mem`); optional layers NULL. */
typedef struct {
  int64_t width, height;
  const float* science;
  const float* reference;
  const float* science_var;
  const float* reference_var;
  const uint8_t* science_mask;
  const uint8_t* reference_mask;
} dgpu_frame;

/* Subtractor settings of the batch (python/delta/pipeline.py:308-384; the
 * reference's defaults in brackets). */
typedef struct {
  int n_max;                      /* 6 */
  int n_knots;                    /* 5 (knots per axis) */
  int radius;                     /* 0: default radius */
  int stamp_radius;               /* 15 */
  double threshold_sigma;         /* 5.0 (stamp detection) */
  int max_stamps;                 /* 200 */
  double saturation;              /* 0.0 */
  int fwhm_radius;                /* 0 */
  int match_radius;               /* 2 */
  const double* lambda_grid;      /* NULL: logspace(-6, 6, 25) */
  int n_lambda;
  double clip_sigma;              /* 4.0 */
  int clip_iterations;            /* 5 */
  int min_stamps;                 /* 5 */
  int cv_folds;                   /* 5 (0 or 1: GCV) */
  int precision;                  /* DGPU_PREC_* */
  int decorrelate;                /* 1 */
  int block;                      /* 256 */
  int score;                      /* 1 (needs variance layers) */
  int catalog;                    /* 1 (with score) */
  double catalog_threshold_sigma; /* 5.0 */
  int frames_in_flight;           /* 4 */
  int device;                     /* CUDA device index */
  int graphs;                     /* 1: record the post-fit segment as a CUDA graph (see below) */
} dgpu_batch_config;

/* Products of one frame. Image buffers are caller memory of width x height
 * (host or device per `mem`; NULL skips a product): difference (whitened
 * when decorrelated) and its variance, mask, score. theta: (nc+1)*k host
 * values or NULL. Catalog: columns of `catalog_capacity` entries (host); the
 * rows are copied only when catalog_count <= catalog_capacity
 * (catalog_fetched = 1). status / error: this frame's outcome. */
typedef struct {
  float* difference;
  float* variance;
  uint8_t* mask;
  float* score;
  double* theta;
  dgpu_catalog_columns catalog;
  int catalog_capacity;
  /* outputs */
  int64_t n_theta;
  double lambda;
  double beta;
  int direction_is_reference;
  int n_stamps_used;
  int has_variance;
  int has_mask;
  int catalog_count;
  int catalog_fetched;
  int status;
  char error[256];
  double seconds;     /* wall time of the frame on its worker */
  int graph_replayed; /* 1: the post-fit segment ran as a recorded graph */
} dgpu_frame_result;

/* subtract() over many frames of any sizes (the reference's per-frame
 * Subtractor.subtract, python/delta/pipeline.py:430-806, applied to a list of
 * pairs as pipeline.py:872-908 does for apply). Frames are processed longest
 * first by frames_in_flight worker threads, each with its own context and
 * stream from a process-wide pool (workspace kept between calls). Returns
 * DGPU_OK when every frame succeeded, else the first failed frame's status
 * (each frame's status / error are in its result); text via
 * dgpu_last_error(NULL).
 *
 * With cfg->graphs != 0 the device work after the kernel fit (subtraction,
 * sign, decorrelation: some forty launches) runs as one CUDA graph launch.
 * No reference counterpart. A worker context runs the first frame of each
 * layer configuration and shape directly (that sizes its workspace and
 * settles the autotuner); later frames of that key are recorded into a graph
 * -- the frame's small tables go through a pinned arena of the context --
 * and the key's executable graph is updated in place (instantiated when the
 * update is refused) and launched. A recording that meets anything that
 * cannot be recorded is dropped and the segment run directly. Results are the
 * same bits either way. */
int dgpu_subtract_batch(const dgpu_batch_config* cfg, int mem, int n_frames, const dgpu_frame* frames,
                        dgpu_frame_result* results);

#ifdef __cplusplus
}
#endif

#endif /* DELTA_GPU_H_ */
