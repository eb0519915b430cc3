// C-ABI entry points of stamp selection, PSF estimation and weighted_mean.
// The per-pixel scans, order statistics, footprint / moment evaluations and the
// greedy isolation run on the device (k_detect.cu); the cross-match of the two
// detection lists (<= max_stamps each) and the FWHM medians are host glue.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

#include "detect_internal.h"

using namespace dgpu;

namespace {

template <class F>
int guarded(dgpu_context* ctx, F&& f) {
  return run_entry(ctx, true, false, std::forward<F>(f));
}

DetectParamsDev resolve(const dgpu_detect_params* p) {
  DetectParamsDev d;
  d.stamp_radius = p->stamp_radius;
  d.threshold_sigma = p->threshold_sigma;
  d.max_stamps = p->max_stamps;
  d.saturation = p->saturation;
  d.isolation_radius = p->isolation_radius > 0 ? p->isolation_radius : 2 * p->stamp_radius;
  d.border = p->border > 0 ? p->border : p->stamp_radius;
  d.fwhm_radius = p->fwhm_radius > 0 ? p->fwhm_radius : std::max(5, p->stamp_radius / 2);
  d.match_radius = p->match_radius;
  return d;
}

// median_of (src/detect.cpp:28-40): non-finite removed, upper median, NaN if empty.
double median_finite(std::vector<double> v) {
  v.erase(std::remove_if(v.begin(), v.end(), [](double x) { return !std::isfinite(x); }), v.end());
  if (v.empty()) return std::numeric_limits<double>::quiet_NaN();
  const size_t mid = v.size() / 2;
  std::nth_element(v.begin(), v.begin() + mid, v.end());
  return v[mid];
}

void dims(int64_t w, int64_t h) {
  if (w <= 0 || h <= 0) fail(DGPU_ERR_INVALID, "image must be non-empty");
  if (w * h >= (int64_t(1) << 31)) fail(DGPU_ERR_INVALID, "image too large");
}

}  // namespace

extern "C" {

int dgpu_estimate_background(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* data,
                             const uint8_t* mask, double* median, double* sigma) {
  return guarded(ctx, [&](Context& c) {
    dims(width, height);
    const size_t n = static_cast<size_t>(width) * height;
    const auto* d = static_cast<const float*>(stage_in(c, mem, data, 4 * n, kSlotInSci));
    const auto* m = static_cast<const uint8_t*>(stage_in(c, mem, mask, n, kSlotInMaskS));
    run_background(c, static_cast<int64_t>(n), d, m, median, sigma);
  });
}

int dgpu_detect_stamps(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* data,
                       const uint8_t* mask, const dgpu_detect_params* params, int capacity, int32_t* x, int32_t* y,
                       double* flux, double* snr, double* fwhm, int* count) {
  return guarded(ctx, [&](Context& c) {
    dims(width, height);
    const int w = static_cast<int>(width), h = static_cast<int>(height);
    const size_t n = static_cast<size_t>(w) * h;
    const auto* d = static_cast<const float*>(stage_in(c, mem, data, 4 * n, kSlotInSci));
    const auto* m = static_cast<const uint8_t*>(stage_in(c, mem, mask, n, kSlotInMaskS));
    DetectHost r;
    const int k = run_detect(c, w, h, d, m, resolve(params), 0, r);
    *count = k;
    for (int i = 0; i < k && i < capacity; ++i) {
      x[i] = r.x[i];
      y[i] = r.y[i];
      flux[i] = r.flux[i];
      snr[i] = r.snr[i];
      fwhm[i] = r.fwhm[i];
    }
    check_status(c);
  });
}

int dgpu_select_stamps(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* science,
                       const float* reference, const uint8_t* science_mask, const uint8_t* reference_mask,
                       const int32_t* cat_x, const int32_t* cat_y, int n_cat, const dgpu_detect_params* params,
                       int capacity, int32_t* x, int32_t* y, double* fwhm_science, double* fwhm_reference,
                       double* median_fwhm_science, double* median_fwhm_reference, int* direction_is_reference,
                       int* count) {
  return guarded(ctx, [&](Context& c) {
    dims(width, height);
    const int w = static_cast<int>(width), h = static_cast<int>(height);
    const size_t n = static_cast<size_t>(w) * h;
    const auto* s = static_cast<const float*>(stage_in(c, mem, science, 4 * n, kSlotInSci));
    const auto* r = static_cast<const float*>(stage_in(c, mem, reference, 4 * n, kSlotInRef));
    const auto* sm = static_cast<const uint8_t*>(stage_in(c, mem, science_mask, n, kSlotInMaskS));
    const auto* rm = static_cast<const uint8_t*>(stage_in(c, mem, reference_mask, n, kSlotInMaskR));
    const DetectParamsDev p = resolve(params);
    std::vector<int> ox, oy;
    std::vector<double> fs, fr;
    if (cat_x && cat_y) {
      std::vector<int> ok;
      std::vector<double> a, b;
      double ms = 0, mr = 0;
      run_catalog_stamps(c, w, h, s, sm, r, rm, cat_x, cat_y, n_cat, p, ok, a, b, &ms, &mr);
      for (int i = 0; i < n_cat; ++i)
        if (ok[i]) {
          ox.push_back(cat_x[i]);
          oy.push_back(cat_y[i]);
          fs.push_back(a[i]);
          fr.push_back(b[i]);
        }
    } else {
      DetectHost ds, dr;
      run_detect_pair(c, w, h, s, sm, r, rm, p, ds, dr);
      const long tol2 = static_cast<long>(p.match_radius) * p.match_radius;
      for (size_t i = 0; i < dr.x.size(); ++i) {
        int best = -1;
        long best_d2 = tol2 + 1;
        for (size_t j = 0; j < ds.x.size(); ++j) {
          const long dx = dr.x[i] - ds.x[j], dy = dr.y[i] - ds.y[j];
          const long d2 = dx * dx + dy * dy;
          if (d2 <= tol2 && d2 < best_d2) {
            best_d2 = d2;
            best = static_cast<int>(j);
          }
        }
        if (best < 0) continue;
        ox.push_back(dr.x[i]);
        oy.push_back(dr.y[i]);
        fs.push_back(ds.fwhm[best]);
        fr.push_back(dr.fwhm[i]);
      }
    }
    const int k = static_cast<int>(ox.size());
    *count = k;
    for (int i = 0; i < k && i < capacity; ++i) {
      x[i] = ox[i];
      y[i] = oy[i];
      fwhm_science[i] = fs[i];
      fwhm_reference[i] = fr[i];
    }
    const double mfs = median_finite(fs), mfr = median_finite(fr);
    *median_fwhm_science = mfs;
    *median_fwhm_reference = mfr;
    *direction_is_reference = (mfr <= mfs) ? 1 : 0;
    check_status(c);
  });
}

int dgpu_estimate_psf(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* image, const int32_t* xs,
                      const int32_t* ys, int n, int radius, float* out) {
  return guarded(ctx, [&](Context& c) {
    dims(width, height);
    if (radius < 0) fail(DGPU_ERR_INVALID, "psf radius must be >= 0");
    const int w = static_cast<int>(width), h = static_cast<int>(height);
    const size_t npx = static_cast<size_t>(w) * h;
    const auto* img = static_cast<const float*>(stage_in(c, mem, image, 4 * npx, kSlotInSci));
    int* dxy = static_cast<int*>(c.slot(kSlotBright, sizeof(int) * 2 * std::max(n, 1)));
    if (n) {
      DGPU_CUDA(h2d_async(dxy, xs, sizeof(int) * n, c.stream));
      DGPU_CUDA(h2d_async(dxy + n, ys, sizeof(int) * n, c.stream));
    }
    const int side = 2 * radius + 1, np = side * side;
    double* dout = static_cast<double*>(c.slot(kSlotPsf, sizeof(double) * np));
    int used = 0;
    if (n > 0) launch_psf_estimate(c, w, h, img, dxy, dxy + n, n, radius, dout, &used);
    if (used == 0) fail(DGPU_ERR_INVALID, "no usable sources for PSF estimation");
    std::vector<double> psf(np);
    read_back(c, psf.data(), dout, sizeof(double) * np);
    sync_reads(c);
    double s = 0.0;
    for (double v : psf) s += v;
    for (int i = 0; i < np; ++i) out[i] = static_cast<float>(psf[i] / s);
    c.last_error.clear();
    reset_status(c);
  });
}

int dgpu_weighted_mean(dgpu_context* ctx, int mem, int64_t n, const float* data, const float* variance,
                       const uint8_t* mask, double* out) {
  return guarded(ctx, [&](Context& c) {
    if (n <= 0) {
      *out = 0.0;
      return;
    }
    const auto* d = static_cast<const float*>(stage_in(c, mem, data, 4 * n, kSlotInSci));
    const auto* v = static_cast<const float*>(stage_in(c, mem, variance, 4 * n, kSlotInVarS));
    const auto* m = static_cast<const uint8_t*>(stage_in(c, mem, mask, n, kSlotInMaskS));
    double sums[2];
    launch_weighted_mean(c, n, d, v, m, sums);
    *out = sums[0] > 0.0 ? sums[1] / sums[0] : 0.0;
  });
}

}  // extern "C"
