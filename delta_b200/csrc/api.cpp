// C-ABI entry points of libdelta_gpu.so (declared in include/delta_gpu.h).
// Each entry point validates its arguments like the reference binding
// (src/bindings.cpp), stages host buffers when mem == DGPU_MEM_HOST, runs the
// sm_100a kernels on the context stream and converts any failure into a status
// code plus dgpu_last_error() text. No exception crosses this boundary.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <stdexcept>

#include <utility>

#include "internal.h"

using namespace dgpu;

namespace dgpu {
std::string& free_error() {
  thread_local std::string e;  // errors of context-free entry points
  return e;
}
}  // namespace dgpu

namespace {

template <class F>
int guarded(dgpu_context* ctx, F&& f) {
  return run_entry(ctx, false, false, std::forward<F>(f));
}

template <class F>
int guarded_free(F&& f) {
  try {
    f();
    return DGPU_OK;
  } catch (const Failure& e) {
    dgpu::free_error() = e.what();
    return e.code;
  } catch (const std::exception& e) {
    dgpu::free_error() = e.what();
    return DGPU_ERR_RUNTIME;
  }
}

void check_dims(int64_t w, int64_t h) {
  if (w <= 0 || h <= 0) fail(DGPU_ERR_INVALID, "image must be non-empty");
  if (w > (1 << 30) || h > (1 << 30) || w * h >= (int64_t(1) << 31))
    fail(DGPU_ERR_INVALID, "image too large (axis < 2^30 and < 2^31 pixels supported)");
}

struct ModelHost {
  ThinPlate tp;
  Basis basis;
  int nf;
  ModelHost(const dgpu_model* m)
      : tp(m->knots, m->n_knots), basis(m->beta, m->n_max, m->radius), nf(basis.nc + 1) {
    if (m->n_theta != static_cast<int64_t>(tp.k) * nf)
      fail(DGPU_ERR_RUNTIME, "subtract: theta size does not match k*(nc+1)");
  }
};

std::vector<int2> orders_of(const Basis& b) {
  std::vector<int2> o(b.nc);
  for (int i = 0; i < b.nc; ++i) o[i] = make_int2(b.orders[i].first, b.orders[i].second);
  return o;
}

}  // namespace

extern "C" {

int dgpu_device_count(int* count) {
  int n = 0;
  const cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    *count = 0;
    dgpu::free_error() = cudaGetErrorString(e);
    return DGPU_ERR_NO_DEVICE;
  }
  *count = n;
  return DGPU_OK;
}

int dgpu_create(int device, dgpu_context** out) {
  return guarded_free([&] {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) fail(DGPU_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= n) fail(DGPU_ERR_INVALID, "device index out of range");
    DGPU_CUDA(cudaSetDevice(device));
    keep_pool_memory(device);
    auto* c = new Context();
    c->device = device;
    DGPU_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
    c->stream = c->own_stream;
    DGPU_CUDA(cudaMalloc(&c->d_status, sizeof(unsigned)));
    DGPU_CUDA(cudaMemset(c->d_status, 0, sizeof(unsigned)));
    const char* tv = std::getenv("DELTA_TIMING");
    c->timing_enabled = tv != nullptr && tv[0] != '\0' && std::string(tv) != "0";
    *out = reinterpret_cast<dgpu_context*>(c);
  });
}

void dgpu_destroy(dgpu_context* ctx) {
  if (!ctx) return;
  auto* c = reinterpret_cast<Context*>(ctx);
  cudaSetDevice(c->device);
  for (int i = 0; i < kSlotCount; ++i)
    if (c->slot_ptr[i]) cudaFreeAsync(c->slot_ptr[i], c->stream);
  cudaStreamSynchronize(c->stream);
  for (auto& kv : c->graphs)
    if (kv.second) cudaGraphExecDestroy(kv.second);
  if (c->arena.base) cudaFreeHost(c->arena.base);
  if (c->d_status) cudaFree(c->d_status);
  if (c->rb_host) cudaFreeHost(c->rb_host);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
}

int dgpu_set_stream(dgpu_context* ctx, void* stream) {
  return guarded(ctx, [&](Context& c) {
    const cudaStream_t next = stream ? static_cast<cudaStream_t>(stream) : c.own_stream;
    if (next == c.stream) return;
    // Work already queued on the old stream must finish before the new one runs.
    DGPU_CUDA(cudaStreamSynchronize(c.stream));
    c.stream = next;
  });
}

int dgpu_synchronize(dgpu_context* ctx) {
  return guarded(ctx, [&](Context& c) { DGPU_CUDA(cudaStreamSynchronize(c.stream)); });
}

const char* dgpu_last_error(const dgpu_context* ctx) {
  if (ctx) return reinterpret_cast<const Context*>(ctx)->last_error.c_str();
  return dgpu::free_error().c_str();
}

int dgpu_set_timing(dgpu_context* ctx, int on) {
  return guarded(ctx, [&](Context& c) {
    resolve_timing(c);
    c.timing_enabled = on != 0;
  });
}

int dgpu_autotune_table(char* out, size_t cap, size_t* needed) {
  return guarded_free([&] {
    const std::string t = autotuner().report();
    if (needed) *needed = t.size() + 1;
    if (out && cap > 0) {
      const size_t n = std::min(cap - 1, t.size());
      std::memcpy(out, t.data(), n);
      out[n] = '\0';
    }
  });
}

int dgpu_set_label_loop_cap(dgpu_context* ctx, int cap) {
  return guarded(ctx, [&](Context& c) { c.label_loop_cap = cap > 0 ? cap : Context::kDefaultLabelLoopCap; });
}

int dgpu_set_precision_fallback(dgpu_context* ctx, int enabled) {
  return guarded(ctx, [&](Context& c) { c.precision_fallback = enabled != 0; });
}

int dgpu_launch_count(unsigned long long* count) {
  *count = launch_count();
  return DGPU_OK;
}

int dgpu_drain_timing(dgpu_context* ctx, char (*labels)[64], double* seconds, int cap, int* n) {
  return guarded(ctx, [&](Context& c) {
    resolve_timing(c);
    const int cnt = static_cast<int>(c.timing.size());
    for (int i = 0; i < cnt && i < cap; ++i) {
      std::strncpy(labels[i], c.timing[i].first.c_str(), 63);
      labels[i][63] = '\0';
      seconds[i] = c.timing[i].second;
    }
    *n = cnt;
    c.timing.clear();
  });
}

// ---- basis ----------------------------------------------------------------

int dgpu_default_radius(double beta, int n_max) { return default_radius(beta, n_max); }

int dgpu_gauss_hermite_basis1d(double beta, int n_max, int radius, double* out, int* ksize) {
  return guarded_free([&] {
    const Basis b(beta, n_max, radius);
    if (ksize) *ksize = b.ks;
    if (out) std::memcpy(out, b.b1d.data(), sizeof(double) * b.b1d.size());
  });
}

int dgpu_gauss_hermite_kernels(double beta, int n_max, int radius, int32_t* orders, float* kernels,
                               int* ksize) {
  return guarded_free([&] {
    const Basis b(beta, n_max, radius);
    if (ksize) *ksize = b.ks;
    for (int c = 0; c < b.nc; ++c) {
      if (orders) {
        orders[2 * c] = b.orders[c].first;
        orders[2 * c + 1] = b.orders[c].second;
      }
      if (kernels) {
        const auto k = b.kernel2d(c);
        std::memcpy(kernels + static_cast<size_t>(c) * b.ks * b.ks, k.data(), sizeof(float) * k.size());
      }
    }
  });
}

int dgpu_component_sums(double beta, int n_max, int radius, double* out) {
  return guarded_free([&] {
    const Basis b(beta, n_max, radius);
    const auto s = b.component_sums();
    std::memcpy(out, s.data(), sizeof(double) * s.size());
  });
}

// ---- thin-plate spline ------------------------------------------------------

int dgpu_grid_knots(double x0, double y0, double x1, double y1, int nx, int ny, double* out) {
  return guarded_free([&] {
    if (nx < 1 || ny < 1) fail(DGPU_ERR_INVALID, "nx, ny must be >= 1");
    int idx = 0;
    for (int iy = 0; iy < ny; ++iy) {
      const double fy = ny == 1 ? 0.5 : static_cast<double>(iy) / (ny - 1);
      const double y = y0 + fy * (y1 - y0);
      for (int ix = 0; ix < nx; ++ix) {
        const double fx = nx == 1 ? 0.5 : static_cast<double>(ix) / (nx - 1);
        out[2 * idx] = x0 + fx * (x1 - x0);
        out[2 * idx + 1] = y;
        ++idx;
      }
    }
  });
}

int dgpu_tps_design(const double* knots, int k, const double* points, int64_t m, double* out) {
  return guarded_free([&] {
    const ThinPlate tp(knots, k);
    for (int64_t i = 0; i < m; ++i) tp.design_row(points[2 * i], points[2 * i + 1], out + i * k);
  });
}

int dgpu_tps_penalty(const double* knots, int k, double* out) {
  return guarded_free([&] {
    const ThinPlate tp(knots, k);
    std::memcpy(out, tp.penalty.data(), sizeof(double) * k * k);
  });
}

// Symmetric positive-(semi)definite solve with Cholesky, falling back to
// partial-pivoting Gaussian elimination (the reference uses Eigen's LDLT).
static void small_solve(int n, std::vector<double> a, std::vector<double> b, double* x) {
  std::vector<double> l(a);
  bool ok = true;
  for (int j = 0; j < n && ok; ++j) {
    double d = l[j * n + j];
    for (int k = 0; k < j; ++k) d -= l[j * n + k] * l[j * n + k];
    if (!(d > 0.0)) {
      ok = false;
      break;
    }
    d = std::sqrt(d);
    l[j * n + j] = d;
    for (int i = j + 1; i < n; ++i) {
      double s = l[i * n + j];
      for (int k = 0; k < j; ++k) s -= l[i * n + k] * l[j * n + k];
      l[i * n + j] = s / d;
    }
  }
  if (ok) {
    std::vector<double> y(n);
    for (int i = 0; i < n; ++i) {
      double s = b[i];
      for (int k = 0; k < i; ++k) s -= l[i * n + k] * y[k];
      y[i] = s / l[i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
      double s = y[i];
      for (int k = i + 1; k < n; ++k) s -= l[k * n + i] * x[k];
      x[i] = s / l[i * n + i];
    }
    return;
  }
  std::vector<int> piv(n);
  for (int i = 0; i < n; ++i) piv[i] = i;
  for (int j = 0; j < n; ++j) {
    int p = j;
    for (int i = j + 1; i < n; ++i)
      if (std::fabs(a[i * n + j]) > std::fabs(a[p * n + j])) p = i;
    if (p != j) {
      for (int k = 0; k < n; ++k) std::swap(a[j * n + k], a[p * n + k]);
      std::swap(b[j], b[p]);
    }
    const double d = a[j * n + j];
    if (d == 0.0) continue;
    for (int i = j + 1; i < n; ++i) {
      const double f = a[i * n + j] / d;
      for (int k = j; k < n; ++k) a[i * n + k] -= f * a[j * n + k];
      b[i] -= f * b[j];
    }
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = b[i];
    for (int k = i + 1; k < n; ++k) s -= a[i * n + k] * x[k];
    x[i] = a[i * n + i] != 0.0 ? s / a[i * n + i] : 0.0;
  }
}

int dgpu_tps_fit(const double* knots, int k, const double* points, int64_t m, const double* values,
                 double lam, double* out) {
  return guarded_free([&] {
    const ThinPlate tp(knots, k);
    std::vector<double> a(static_cast<size_t>(k) * k, 0.0), b(k, 0.0), row(k);
    for (int64_t i = 0; i < m; ++i) {
      tp.design_row(points[2 * i], points[2 * i + 1], row.data());
      for (int p = 0; p < k; ++p) {
        b[p] += row[p] * values[i];
        for (int q = 0; q < k; ++q) a[p * k + q] += row[p] * row[q];
      }
    }
    for (int p = 0; p < k * k; ++p) a[p] += lam * tp.penalty[p];
    small_solve(k, a, b, out);
  });
}

int dgpu_tps_evaluate(const double* knots, int k, const double* points, int64_t m, const double* coeffs,
                      double* out) {
  return guarded_free([&] {
    const ThinPlate tp(knots, k);
    std::vector<double> row(k);
    for (int64_t i = 0; i < m; ++i) {
      tp.design_row(points[2 * i], points[2 * i + 1], row.data());
      double s = 0.0;
      for (int p = 0; p < k; ++p) s += row[p] * coeffs[p];
      out[i] = s;
    }
  });
}

// ---- convolution ------------------------------------------------------------

int dgpu_basis_convolve(dgpu_context* ctx, int mem, const float* image, int64_t width, int64_t height,
                        double beta, int n_max, int radius, float* out) {
  return guarded(ctx, [&](Context& c) {
    check_dims(width, height);
    const int w = static_cast<int>(width), h = static_cast<int>(height);
    const Basis b(beta, n_max, radius);
    const size_t n = static_cast<size_t>(w) * h;
    reset_status(c);
    const float* img = static_cast<const float*>(stage_in(c, mem, image, sizeof(float) * n, kSlotInRef));
    float* o = static_cast<float*>(out_buf(c, mem, out, sizeof(float) * n * b.nc, kSlotOutDiff));
    const auto taps = b.taps();
    float* dt = static_cast<float*>(c.slot(kSlotTaps, sizeof(float) * taps.size()));
    DGPU_CUDA(h2d_async(dt, taps.data(), sizeof(float) * taps.size(), c.stream));
    const auto ord = orders_of(b);
    int2* dord = static_cast<int2*>(c.slot(kSlotScratch2, sizeof(int2) * ord.size()));
    DGPU_CUDA(h2d_async(dord, ord.data(), sizeof(int2) * ord.size(), c.stream));
    SubtractArgs a{};
    a.w = w;
    a.h = h;
    a.ref = img;
    a.n_max = b.n_max;
    a.ks = b.ks;
    a.nc = b.nc;
    a.taps = dt;
    a.diff = o;
    launch_model_convolve_orders(c.stream, a, dord, true);
    stage_out(c, mem, out, o, sizeof(float) * n * b.nc);
    check_status(c);
  });
}

// ---- subtraction --------------------------------------------------------------

int dgpu_subtract(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* science,
                  const float* reference, const float* science_var, const float* reference_var,
                  const uint8_t* science_mask, const uint8_t* reference_mask, const dgpu_model* model,
                  double saturation, float* out_difference, float* out_variance, uint8_t* out_mask,
                  int* has_variance, int* has_mask) {
  return guarded(ctx, [&](Context& c) {
    check_dims(width, height);
    if (!science || !reference || !model) fail(DGPU_ERR_INVALID, "subtract: missing input");
    const int w = static_cast<int>(width), h = static_cast<int>(height);
    const size_t n = static_cast<size_t>(w) * h;
    const ModelHost mh(model);
    const Basis& b = mh.basis;
    cudaStream_t s = c.stream;
    reset_status(c);
    const auto* sci = static_cast<const float*>(stage_in(c, mem, science, 4 * n, kSlotInSci));
    const auto* ref = static_cast<const float*>(stage_in(c, mem, reference, 4 * n, kSlotInRef));
    const auto* vs = static_cast<const float*>(stage_in(c, mem, science_var, 4 * n, kSlotInVarS));
    const auto* vr = static_cast<const float*>(stage_in(c, mem, reference_var, 4 * n, kSlotInVarR));
    const auto* sm = static_cast<const uint8_t*>(stage_in(c, mem, science_mask, n, kSlotInMaskS));
    const auto* rm = static_cast<const uint8_t*>(stage_in(c, mem, reference_mask, n, kSlotInMaskR));
    const bool want_var = vs != nullptr || vr != nullptr;
    const bool want_mask = sm != nullptr || rm != nullptr || saturation > 0.0;
    if (has_variance) *has_variance = want_var ? 1 : 0;
    if (has_mask) *has_mask = want_mask ? 1 : 0;
    float* diff = static_cast<float*>(out_buf(c, mem, out_difference, 4 * n, kSlotOutDiff));
    float* var = want_var ? static_cast<float*>(out_buf(c, mem, out_variance, 4 * n, kSlotOutVar)) : nullptr;
    uint8_t* mask = want_mask ? static_cast<uint8_t*>(out_buf(c, mem, out_mask, n, kSlotOutMask)) : nullptr;

    DevFields F;
    {
      StageTimer t(c, "subtract: spatial fields");
      F = build_fields(c, mh.tp, model->theta, mh.nf, w, h);
    }
    float* scal = static_cast<float*>(c.slot(kSlotScratch1, 64));  // [0] ref fill, [1] diff fill
    {
      StageTimer t(c, "subtract: sanitise reference");
      launch_strided_median(c, kSampleReference, static_cast<int64_t>(n), ref, rm, scal);
    }
    {
      const auto taps = b.taps();
      float* dt = static_cast<float*>(c.slot(kSlotTaps, sizeof(float) * taps.size()));
      DGPU_CUDA(h2d_async(dt, taps.data(), sizeof(float) * taps.size(), s));
      const auto ord = orders_of(b);
      int2* dord = static_cast<int2*>(c.slot(kSlotScratch2, sizeof(int2) * ord.size()));
      DGPU_CUDA(h2d_async(dord, ord.data(), sizeof(int2) * ord.size(), s));
      StageTimer t(c, "subtract: model convolve");
      SubtractArgs a{};
      a.w = w;
      a.h = h;
      a.sci = sci;
      a.ref = ref;
      a.ref_mask = rm;
      a.F = F;
      a.n_max = b.n_max;
      a.ks = b.ks;
      a.nc = b.nc;
      a.taps = dt;
      a.fill = scal;
      a.diff = diff;
      launch_model_convolve_orders(s, a, dord, false);
    }
    if (want_var) {
      StageTimer t(c, "subtract: variance propagation");
      float* phi = nullptr;
      if (vr) {
        std::vector<float> ph(static_cast<size_t>(b.nc) * b.ks * b.ks);
        for (int q = 0; q < b.nc; ++q) {
          const auto k2 = b.kernel2d(q);
          std::copy(k2.begin(), k2.end(), ph.begin() + static_cast<size_t>(q) * b.ks * b.ks);
        }
        phi = static_cast<float*>(c.slot(kSlotPhi, sizeof(float) * ph.size()));
        DGPU_CUDA(h2d_async(phi, ph.data(), sizeof(float) * ph.size(), s));
      }
      launch_variance(s, w, h, F, phi, b.radius, b.nc, vs, vr, var);
    }
    if (want_mask) {
      StageTimer t(c, "subtract: mask growth");
      uint8_t* eb = static_cast<uint8_t*>(c.slot(kSlotExactBad, n));
      launch_mask(s, w, h, sci, ref, sm, rm, saturation, b.radius, diff, mask, eb);
      launch_strided_median(c, kSampleDifference, static_cast<int64_t>(n), diff, mask, scal + 1);
      launch_mask_fill(s, static_cast<int64_t>(n), mask, eb, scal + 1, diff, var);
    }
    stage_out(c, mem, out_difference, diff, 4 * n);
    if (want_var) stage_out(c, mem, out_variance, var, 4 * n);
    if (want_mask) stage_out(c, mem, out_mask, mask, n);
    if (mem == DGPU_MEM_HOST) check_status(c);
  });
}

int dgpu_photometric_scale(dgpu_context* ctx, int mem, const double* knots, int n_knots, const double* theta,
                           int64_t n_theta, const double* component_sums, int nc, int64_t height,
                           int64_t width, float* out) {
  return guarded(ctx, [&](Context& c) {
    check_dims(width, height);
    const ThinPlate tp(knots, n_knots);
    if (n_theta != static_cast<int64_t>(tp.k) * (nc + 1))
      fail(DGPU_ERR_RUNTIME, "photometric_scale: theta size mismatch");
    const int w = static_cast<int>(width), h = static_cast<int>(height);
    const size_t n = static_cast<size_t>(w) * h;
    reset_status(c);
    const DevFields F = build_fields(c, tp, theta, nc + 1, w, h);
    std::vector<float> sums(nc);
    for (int q = 0; q < nc; ++q) sums[q] = static_cast<float>(component_sums[q]);
    float* ds = static_cast<float*>(c.slot(kSlotScratch2, sizeof(float) * std::max(nc, 1)));
    DGPU_CUDA(h2d_async(ds, sums.data(), sizeof(float) * nc, c.stream));
    float* o = static_cast<float*>(out_buf(c, mem, out, 4 * n, kSlotOutDiff));
    launch_photometric_scale(c.stream, F, ds, nc, o);
    stage_out(c, mem, out, o, 4 * n);
    if (mem == DGPU_MEM_HOST) check_status(c);
  });
}

int dgpu_estimate_background_noalloc(const float* data, const uint8_t* mask, int64_t width, int64_t height,
                                     void* stream, double* median, double* sigma) {
  return guarded_free([&] {
    check_dims(width, height);
    if (!data || !median || !sigma) fail(DGPU_ERR_INVALID, "estimate_background_noalloc: missing argument");
    float r[2] = {0.0f, 0.0f};
    background_noalloc(width * height, data, mask, static_cast<cudaStream_t>(stream), r);
    *median = static_cast<double>(r[0]);
    *sigma = 1.4826 * static_cast<double>(r[1]);
  });
}

int dgpu_scale(dgpu_context* ctx, int mem, float* data, int64_t n, double scale) {
  return guarded(ctx, [&](Context& c) {
    if (n < 0) fail(DGPU_ERR_INVALID, "scale: n must be >= 0");
    if (n == 0) return;
    if (!data) fail(DGPU_ERR_INVALID, "scale: missing buffer");
    const size_t bytes = 4 * static_cast<size_t>(n);
    float* d = mem == DGPU_MEM_DEVICE ? data : static_cast<float*>(c.slot(kSlotOutVar, bytes));
    if (mem != DGPU_MEM_DEVICE) DGPU_CUDA(h2d_async(d, data, bytes, c.stream));
    launch_scale_fill(c.stream, n, d, static_cast<float>(scale), false, 0.0f);
    stage_out(c, mem, data, d, bytes);
    if (mem == DGPU_MEM_HOST) DGPU_CUDA(cudaStreamSynchronize(c.stream));
  });
}

int dgpu_z2_median(dgpu_context* ctx, int mem, int64_t n, const float* difference, const float* variance,
                   const uint8_t* mask, double* median, int64_t* count) {
  return guarded(ctx, [&](Context& c) {
    if (n < 0 || !difference || !variance || !median || !count) fail(DGPU_ERR_INVALID, "z2_median: missing argument");
    *median = 0.0;
    *count = 0;
    if (n == 0) return;
    const size_t nn = static_cast<size_t>(n);
    const auto* d = static_cast<const float*>(stage_in(c, mem, difference, 4 * nn, kSlotOutDiff));
    const auto* v = static_cast<const float*>(stage_in(c, mem, variance, 4 * nn, kSlotOutVar));
    const auto* m = static_cast<const uint8_t*>(stage_in(c, mem, mask, nn, kSlotOutMask));
    auto* keys = static_cast<unsigned long long*>(c.slot(kSlotScratch0, 8 * nn));
    auto* st = static_cast<unsigned long long*>(c.slot(kSlotScratch2, 8 * 8 + 512 * 4));
    launch_z2_median(c.stream, n, d, v, m, keys, st, reinterpret_cast<unsigned int*>(st + 8));
    unsigned long long h[5];
    read_back(c, h, st, sizeof(h));
    sync_reads(c);
    *count = static_cast<int64_t>(h[0]);
    if (h[0] == 0) return;
    double a, b;
    std::memcpy(&a, &h[3], 8);
    std::memcpy(&b, &h[4], 8);
    *median = (a + b) / 2.0;
  });
}

int dgpu_fill(dgpu_context* ctx, int mem, float* data, int64_t n, double value) {
  return guarded(ctx, [&](Context& c) {
    if (n < 0) fail(DGPU_ERR_INVALID, "fill: n must be >= 0");
    if (n == 0) return;
    if (!data) fail(DGPU_ERR_INVALID, "fill: missing buffer");
    const size_t bytes = 4 * static_cast<size_t>(n);
    float* d = mem == DGPU_MEM_DEVICE ? data : static_cast<float*>(c.slot(kSlotOutVar, bytes));
    launch_scale_fill(c.stream, n, d, 1.0f, true, static_cast<float>(value));
    stage_out(c, mem, data, d, bytes);
    if (mem == DGPU_MEM_HOST) DGPU_CUDA(cudaStreamSynchronize(c.stream));
  });
}

int dgpu_negate(dgpu_context* ctx, int mem, float* data, int64_t n) {
  return guarded(ctx, [&](Context& c) {
    if (n < 0) fail(DGPU_ERR_INVALID, "negate: n must be >= 0");
    if (n == 0) return;
    if (!data) fail(DGPU_ERR_INVALID, "negate: missing buffer");
    const size_t bytes = 4 * static_cast<size_t>(n);
    float* d = mem == DGPU_MEM_DEVICE ? data : static_cast<float*>(c.slot(kSlotOutDiff, bytes));
    if (mem != DGPU_MEM_DEVICE)
      DGPU_CUDA(h2d_async(d, data, bytes, c.stream));
    launch_negate(c.stream, n, d);
    stage_out(c, mem, data, d, bytes);
    if (mem == DGPU_MEM_HOST) DGPU_CUDA(cudaStreamSynchronize(c.stream));
  });
}

int dgpu_copy_to_host(dgpu_context* ctx, void* host_dst, const void* device_src, int64_t bytes) {
  return guarded(ctx, [&](Context& c) {
    if (bytes < 0) fail(DGPU_ERR_INVALID, "copy_to_host: bytes must be >= 0");
    if (bytes == 0) return;
    if (!host_dst || !device_src) fail(DGPU_ERR_INVALID, "copy_to_host: missing buffer");
    cudaPointerAttributes pa{};
    DGPU_CUDA(cudaPointerGetAttributes(&pa, host_dst));
    if (pa.type != cudaMemoryTypeHost) fail(DGPU_ERR_INVALID, "copy_to_host: destination is not pinned host memory");
    cudaPointerAttributes ps{};
    DGPU_CUDA(cudaPointerGetAttributes(&ps, device_src));
    if (ps.type != cudaMemoryTypeDevice) fail(DGPU_ERR_INVALID, "copy_to_host: source is not device memory");
    DGPU_CUDA(cudaMemcpyAsync(host_dst, device_src, static_cast<size_t>(bytes), cudaMemcpyDeviceToHost, c.stream));
  });
}

int dgpu_photometric_scale_at(const double* knots, int n_knots, const double* theta, int64_t n_theta,
                              const double* component_sums, int nc, const double* points, int64_t m,
                              double* out) {
  return guarded_free([&] {
    const ThinPlate tp(knots, n_knots);
    if (n_theta != static_cast<int64_t>(tp.k) * (nc + 1))
      fail(DGPU_ERR_RUNTIME, "photometric_scale: theta size mismatch");
    std::vector<double> row(tp.k);
    for (int64_t i = 0; i < m; ++i) {
      tp.design_row(points[2 * i], points[2 * i + 1], row.data());
      double s = 0.0;
      for (int q = 0; q < nc; ++q) {
        double f = 0.0;
        for (int p = 0; p < tp.k; ++p) f += row[p] * theta[static_cast<size_t>(q) * tp.k + p];
        s += f * component_sums[q];
      }
      out[i] = s;
    }
  });
}

// ---- matched filter -------------------------------------------------------------

int dgpu_matched_filter(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* image,
                        const float* psf, int psf_size, const float* variance, float* out) {
  return guarded(ctx, [&](Context& c) {
    check_dims(width, height);
    if (psf_size < 1 || !psf) fail(DGPU_ERR_INVALID, "matched_filter: psf must be non-empty");
    if (!image || !variance) fail(DGPU_ERR_INVALID, "matched_filter: missing input");
    const int w = static_cast<int>(width), h = static_cast<int>(height);
    const size_t n = static_cast<size_t>(w) * h;
    reset_status(c);
    // sum psf^2 in float, sequential, fused (src/noise.cpp:547-548).
    float sumpsf2 = 0.0f;
    for (int i = 0; i < psf_size * psf_size; ++i) sumpsf2 = std::fmaf(psf[i], psf[i], sumpsf2);
    const auto* img = static_cast<const float*>(stage_in(c, mem, image, 4 * n, kSlotInSci));
    const auto* var = static_cast<const float*>(stage_in(c, mem, variance, 4 * n, kSlotInVarS));
    float* o = static_cast<float*>(out_buf(c, mem, out, 4 * n, kSlotOutScore));
    float* dpsf = static_cast<float*>(c.slot(kSlotPsf, sizeof(float) * psf_size * psf_size));
    DGPU_CUDA(h2d_async(dpsf, psf, sizeof(float) * psf_size * psf_size, c.stream));
    {
      StageTimer t(c, "score: blocked correlation");
      const size_t ntiles = static_cast<size_t>((w + 63) / 64) * ((h + 31) / 32);
      int* nf_buf = static_cast<int*>(c.slot(kSlotScratch0, sizeof(int) * (ntiles + 1)));
      launch_matched_filter(c.stream, w, h, img, var, dpsf, psf_size, sumpsf2, o, nf_buf);
    }
    stage_out(c, mem, out, o, 4 * n);
    if (mem == DGPU_MEM_HOST) check_status(c);
  });
}

// ---- catalog ----------------------------------------------------------------------

int dgpu_build_catalog(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* score,
                       const float* difference, const uint8_t* mask, const dgpu_catalog_params* params,
                       const float* variance, const float* psf, int psf_size, const double* bright_x,
                       const double* bright_y, int n_bright, int* count) {
  return guarded(ctx, [&](Context& c) {
    check_dims(width, height);
    if (!score || !difference || !params) fail(DGPU_ERR_INVALID, "build_catalog: missing input");
    if ((bright_x == nullptr) != (bright_y == nullptr))
      fail(DGPU_ERR_RUNTIME, "build_catalog: supply both bright_x and bright_y, or neither");
    const int w = static_cast<int>(width), h = static_cast<int>(height);
    const size_t n = static_cast<size_t>(w) * h;
    reset_status(c);
    const auto* sc = static_cast<const float*>(stage_in(c, mem, score, 4 * n, kSlotInSci));
    const auto* df = static_cast<const float*>(stage_in(c, mem, difference, 4 * n, kSlotInRef));
    const auto* mk = static_cast<const uint8_t*>(stage_in(c, mem, mask, n, kSlotInMaskS));
    const auto* vr = static_cast<const float*>(stage_in(c, mem, variance, 4 * n, kSlotInVarS));
    float* dpsf = nullptr;
    if (psf && psf_size > 0) {
      dpsf = static_cast<float*>(c.slot(kSlotPsf, sizeof(float) * psf_size * psf_size));
      DGPU_CUDA(h2d_async(dpsf, psf, sizeof(float) * psf_size * psf_size, c.stream));
    }
    double* dbx = nullptr;
    if (bright_x && n_bright > 0) {
      dbx = static_cast<double*>(c.slot(kSlotBright, sizeof(double) * 2 * n_bright));
      DGPU_CUDA(h2d_async(dbx, bright_x, sizeof(double) * n_bright, c.stream));
      DGPU_CUDA(h2d_async(dbx + n_bright, bright_y, sizeof(double) * n_bright, c.stream));
    }
    const int cnt = run_catalog(c, w, h, sc, df, mk, *params, vr, dpsf, psf_size, dbx,
                                dbx ? dbx + n_bright : nullptr, n_bright);
    check_status(c);
    *count = cnt;
  });
}

int dgpu_catalog_fetch(dgpu_context* ctx, const dgpu_catalog_columns* o, int count) {
  return guarded(ctx, [&](Context& c) {
    if (count != c.cat_count) fail(DGPU_ERR_CAPACITY, "catalog_fetch: count does not match the last catalog");
    const size_t n = static_cast<size_t>(count);
    auto cp = [&](auto* dst, const auto* src) {
      if (dst) std::memcpy(dst, src, sizeof(*src) * n);
    };
    const double* d = c.cat_d.data();
    const int32_t* i = c.cat_i.data();
    const uint8_t* u = c.cat_u8.data();
    cp(o->x, d + 0 * n);
    cp(o->y, d + 1 * n);
    cp(o->peak_snr, d + 2 * n);
    cp(o->flux, d + 3 * n);
    cp(o->expected_n_pix, d + 4 * n);
    cp(o->fwhm_ratio, d + 5 * n);
    cp(o->psf_chi2, d + 6 * n);
    cp(o->psf_amplitude, d + 7 * n);
    cp(o->psf_amplitude_err, d + 8 * n);
    cp(o->bright_star_dist, d + 9 * n);
    cp(o->peak_x, i + 0 * n);
    cp(o->peak_y, i + 1 * n);
    cp(o->n_pix, i + 2 * n);
    cp(o->psf_chi2_dof, i + 3 * n);
    cp(o->fwhm_consistent, u + 0 * n);
    cp(o->mask_flags, u + 1 * n);
    cp(o->is_dipole, u + 2 * n);
    cp(o->quality, u + 3 * n);
    cp(o->shape_consistent, u + 4 * n);
    cp(o->near_bright_star, u + 5 * n);
  });
}

int dgpu_catalog_labels(dgpu_context* ctx, int mem, int32_t* labels, int64_t n) {
  return guarded(ctx, [&](Context& c) {
    if (n != c.cat_npix) fail(DGPU_ERR_CAPACITY, "catalog_labels: size does not match the last catalog");
    const void* src = c.slot_ptr[kSlotLabels];
    if (!src) fail(DGPU_ERR_RUNTIME, "catalog_labels: no catalog has been built");
    if (mem == DGPU_MEM_DEVICE)
      DGPU_CUDA(cudaMemcpyAsync(labels, src, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, c.stream));
    else
      DGPU_CUDA(cudaMemcpyAsync(labels, src, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, c.stream));
    DGPU_CUDA(cudaStreamSynchronize(c.stream));
  });
}

}  // extern "C"
