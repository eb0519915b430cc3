// C-ABI wrapper around the reference's own Eigen-free sources -- TEST
// INFRASTRUCTURE ONLY (the checker, never the product).
//
// oracle/Makefile compiles this file together with the reference sources where
// they lie (src/basis.cpp, src/convolve.cpp, src/detect.cpp, src/timing.cpp)
// into oracle/_ref/libdelta_ref.so. src/catalog.cpp is #included into this
// translation unit (via -I<reference>/src) so the anonymous-namespace
// label_components() can be called directly to pin CCL labels, not only the
// public build_catalog(). No reference source is copied into this repository.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "catalog.cpp"  // reference src/catalog.cpp (whole TU)
#include "delta/basis.hpp"
#include "delta/convolve.hpp"
#include "delta/detect.hpp"

extern "C" {

// GaussHermiteBasis::basis1d for every order (src/basis.cpp:14-59).
int ref_basis1d(double beta, int n_max, int radius, double* out) {
  try {
    delta::GaussHermiteBasis b(beta, n_max, radius);
    const int ks = b.ksize();
    for (int n = 0; n <= n_max; ++n)
      std::memcpy(out + static_cast<size_t>(n) * ks, b.basis1d(n).data(), sizeof(double) * ks);
    return 0;
  } catch (...) {
    return 1;
  }
}

// delta::basis_convolve (src/convolve.cpp:90-113): out is (nc, h, w) float32.
int ref_basis_convolve(const float* img, int w, int h, double beta, int n_max, int radius,
                       float* out) {
  try {
    delta::ImageF im(w, h, img);
    delta::GaussHermiteBasis b(beta, n_max, radius);
    const auto stack = delta::basis_convolve(im, b);
    const size_t n = static_cast<size_t>(w) * h;
    for (size_t c = 0; c < stack.size(); ++c)
      std::memcpy(out + c * n, stack[c].data(), sizeof(float) * n);
    return 0;
  } catch (...) {
    return 1;
  }
}

// label_components (src/catalog.cpp:105-261) over a 0/1 seed image.
int ref_label_components(const uint8_t* seed, int w, int h, int32_t* labels) {
  std::vector<std::uint8_t> s(seed, seed + static_cast<size_t>(w) * h);
  const auto lr = delta::label_components(s, w, h);
  std::memcpy(labels, lr.labels.data(), sizeof(int32_t) * lr.labels.size());
  return lr.n_components;
}

// build_catalog (src/catalog.cpp:600-697). Columns are written for up to
// `capacity` entries; the return value is the entry count (or -1 on error).
int ref_build_catalog(const float* score, const float* difference, const uint8_t* mask, int w,
                      int h, double threshold_sigma, double threshold_sigma_dipole,
                      double expected_fwhm, double fwhm_tolerance_lo, double fwhm_tolerance_hi,
                      int aperture_radius, int exclude_bad_pixels, int return_negative,
                      int fit_psf_shape, double shape_chi2_tolerance, const float* variance,
                      const float* psf, int psf_size, double bright_star_radius,
                      int max_shape_fit, const double* bright_x, const double* bright_y,
                      int n_bright, int capacity, double* x, double* y, int32_t* peak_x,
                      int32_t* peak_y, double* peak_snr, int32_t* n_pix, double* flux,
                      double* expected_n_pix, double* fwhm_ratio, uint8_t* fwhm_consistent,
                      uint8_t* mask_flags, uint8_t* is_dipole, uint8_t* quality,
                      double* psf_chi2, int32_t* psf_chi2_dof, double* psf_amplitude,
                      double* psf_amplitude_err, uint8_t* shape_consistent,
                      double* bright_star_dist, uint8_t* near_bright_star) {
  try {
    delta::ImageF sc(w, h, score);
    if (mask) sc.mask().assign(mask, mask + static_cast<size_t>(w) * h);
    delta::ImageF df(w, h, difference);
    delta::ImageF var;
    if (variance) var = delta::ImageF(w, h, variance);
    std::vector<float> psfv;
    if (psf) psfv.assign(psf, psf + static_cast<size_t>(psf_size) * psf_size);
    std::vector<double> bx, by;
    if (bright_x) {
      bx.assign(bright_x, bright_x + n_bright);
      by.assign(bright_y, bright_y + n_bright);
    }
    delta::CatalogParams p;
    p.threshold_sigma = threshold_sigma;
    p.threshold_sigma_dipole = threshold_sigma_dipole;
    p.expected_fwhm = expected_fwhm;
    p.fwhm_tolerance_lo = fwhm_tolerance_lo;
    p.fwhm_tolerance_hi = fwhm_tolerance_hi;
    p.aperture_radius = aperture_radius;
    p.exclude_bad_pixels = exclude_bad_pixels != 0;
    p.fit_psf_shape = fit_psf_shape != 0;
    p.shape_chi2_tolerance = shape_chi2_tolerance;
    p.bright_star_radius = bright_star_radius;
    p.max_shape_fit = max_shape_fit;
    delta::CatalogAux aux;
    if (variance) aux.variance = &var;
    if (psf) {
      aux.psf = &psfv;
      aux.psf_size = psf_size;
    }
    if (bright_x) {
      aux.bright_x = &bx;
      aux.bright_y = &by;
    }
    const auto entries = delta::build_catalog(sc, df, p, return_negative != 0, aux);
    const int n = static_cast<int>(entries.size());
    for (int i = 0; i < n && i < capacity; ++i) {
      const auto& e = entries[i];
      x[i] = e.x;
      y[i] = e.y;
      peak_x[i] = e.peak_x;
      peak_y[i] = e.peak_y;
      peak_snr[i] = e.peak_snr;
      n_pix[i] = e.n_pix;
      flux[i] = e.flux;
      expected_n_pix[i] = e.expected_n_pix;
      fwhm_ratio[i] = e.fwhm_ratio;
      fwhm_consistent[i] = e.fwhm_consistent ? 1 : 0;
      mask_flags[i] = e.mask_flags;
      is_dipole[i] = e.is_dipole ? 1 : 0;
      quality[i] = e.quality;
      psf_chi2[i] = e.psf_chi2;
      psf_chi2_dof[i] = e.psf_chi2_dof;
      psf_amplitude[i] = e.psf_amplitude;
      psf_amplitude_err[i] = e.psf_amplitude_err;
      shape_consistent[i] = e.shape_consistent ? 1 : 0;
      bright_star_dist[i] = e.bright_star_dist;
      near_bright_star[i] = e.near_bright_star ? 1 : 0;
    }
    return n;
  } catch (...) {
    return -1;
  }
}

// estimate_background (src/detect.cpp:84-113).
int ref_estimate_background(const float* data, const uint8_t* mask, int w, int h, double* median,
                            double* sigma) {
  delta::ImageF im(w, h, data);
  if (mask) im.mask().assign(mask, mask + static_cast<size_t>(w) * h);
  const auto bg = delta::estimate_background(im);
  *median = bg.median;
  *sigma = bg.sigma;
  return 0;
}

static delta::DetectParams make_params(int stamp_radius, double threshold_sigma, int max_stamps,
                                       double saturation, int isolation_radius, int border,
                                       int fwhm_radius, int match_radius) {
  delta::DetectParams p;
  p.stamp_radius = stamp_radius;
  p.threshold_sigma = threshold_sigma;
  p.max_stamps = max_stamps;
  p.saturation = saturation;
  p.isolation_radius = isolation_radius;
  p.border = border;
  p.fwhm_radius = fwhm_radius;
  p.match_radius = match_radius;
  return p;
}

// select_stamps / select_stamps_from_catalog (src/detect.cpp:260-314).
// Returns the stamp count (columns written up to `capacity`), -1 on error.
int ref_select_stamps(const float* sci, const float* ref, const uint8_t* sci_mask,
                      const uint8_t* ref_mask, int w, int h, const int32_t* cat_x,
                      const int32_t* cat_y, int n_cat, int stamp_radius, double threshold_sigma,
                      int max_stamps, double saturation, int isolation_radius, int border,
                      int fwhm_radius, int match_radius, int capacity, int32_t* out_x,
                      int32_t* out_y, double* fwhm_sci, double* fwhm_ref, double* med_sci,
                      double* med_ref, int* direction_is_reference) {
  try {
    delta::ImageF s(w, h, sci), r(w, h, ref);
    if (sci_mask) s.mask().assign(sci_mask, sci_mask + static_cast<size_t>(w) * h);
    if (ref_mask) r.mask().assign(ref_mask, ref_mask + static_cast<size_t>(w) * h);
    const auto p = make_params(stamp_radius, threshold_sigma, max_stamps, saturation,
                               isolation_radius, border, fwhm_radius, match_radius);
    delta::StampSelection sel;
    if (cat_x) {
      std::vector<int> xs(cat_x, cat_x + n_cat), ys(cat_y, cat_y + n_cat);
      sel = delta::select_stamps_from_catalog(s, r, xs, ys, p);
    } else {
      sel = delta::select_stamps(s, r, p);
    }
    const int n = static_cast<int>(sel.x.size());
    for (int i = 0; i < n && i < capacity; ++i) {
      out_x[i] = sel.x[i];
      out_y[i] = sel.y[i];
      fwhm_sci[i] = sel.fwhm_science[i];
      fwhm_ref[i] = sel.fwhm_reference[i];
    }
    *med_sci = sel.median_fwhm_science;
    *med_ref = sel.median_fwhm_reference;
    *direction_is_reference =
        sel.direction == delta::ConvolveDirection::kConvolveReference ? 1 : 0;
    return n;
  } catch (...) {
    return -1;
  }
}

}  // extern "C"
