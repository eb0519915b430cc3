// Stamp-selection types and launchers (k_detect.cu).
#pragma once

#include "internal.h"

namespace dgpu {

struct DetectParamsDev {
  int stamp_radius = 15;
  double threshold_sigma = 5.0;
  int max_stamps = 200;
  double saturation = 0.0;
  int isolation_radius = 30;  // resolved
  int border = 15;            // resolved
  int fwhm_radius = 7;        // resolved
  int match_radius = 2;
};

struct DetectHost {
  double median = 0.0, sigma = 0.0;
  std::vector<int> x, y;
  std::vector<double> flux, snr, fwhm;
};

int run_detect(Context& c, int w, int h, const float* img, const uint8_t* mask, const DetectParamsDev& p, int which,
               DetectHost& res);
// run_detect of two images (workspace slots 0 and 1) sharing each synchronisation.
void run_detect_pair(Context& c, int w, int h, const float* img0, const uint8_t* mask0, const float* img1,
                     const uint8_t* mask1, const DetectParamsDev& p, DetectHost& res0, DetectHost& res1);
void run_background(Context& c, int64_t n, const float* img, const uint8_t* mask, double* median, double* sigma);
void run_catalog_stamps(Context& c, int w, int h, const float* sci, const uint8_t* sm, const float* ref,
                        const uint8_t* rm, const int* xs_host, const int* ys_host, int n, const DetectParamsDev& p,
                        std::vector<int>& ok, std::vector<double>& fs, std::vector<double>& fr, double* med_sci,
                        double* med_ref);
void launch_psf_estimate(Context& c, int w, int h, const float* img, const int* xs, const int* ys, int n, int radius,
                         double* out, int* n_used);
void launch_weighted_mean(Context& c, int64_t n, const float* d, const float* v, const uint8_t* m, double* out2);

}  // namespace dgpu
