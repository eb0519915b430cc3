// Gradient of the stamp fit's GCV score (k_gcv_grad.cu, dgpu_stamp_gcv in api_fit.cpp).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "internal.h"

namespace dgpu {

struct GcvScalars {
  double rss, edf, n, gcv, alpha, beta, lam, drss_dloglam, dgcv_dloglam;
};

struct GcvRowsArgs {
  int64_t N = 0;                    // row slots
  int nc = 0, k = 0, nq = 0;        // components, knots, columns of F
  const uint8_t* valid = nullptr;
  const double* w = nullptr;
  const double* t = nullptr;
  const double* d = nullptr;        // N x k design rows
  const double* bn = nullptr;       // N x nc, s * B_n (shifted basis)
  const double* bnx = nullptr;      // N x nc, s * B_n of the x-derivative taps
  const double* bny = nullptr;      // N x nc, s * B_n of the y-derivative taps
  const double* theta = nullptr;    // P
  const double* z = nullptr;        // P
  const double* X = nullptr;        // P x (1 + nq): [theta | H], row-major
  const GcvScalars* scal = nullptr;
  double scale = 1.0;
  double* partial = nullptr;        // gcv_rows_blocks x 6
};

int gcv_rhs_cols(int P, int k, int r);
void launch_build_rhs_f(cudaStream_t st, int P, int k, int r, const double* rhs, const double* fk, double* B);
size_t gcv_stats_doubles(int P, int k, int r);
// work layout: theta (P), ftheta (nq), z (P), stats (3 nq), sums (3).
// launch_gcv_theta fills theta and ftheta from X = [theta | H]; launch_gcv_stats
// (after the RSS `raw` of theta is known) the rest and the scalars.
void launch_gcv_theta(cudaStream_t st, int P, int k, int r, const double* X, const double* fk, double* work);
void launch_gcv_stats(cudaStream_t st, int P, int k, int r, const double* X, const double* fk, double lam,
                      const double* raw, const long long* n, double* work, GcvScalars* scal);
int gcv_rows_blocks(int64_t N);
void launch_gcv_rows(cudaStream_t st, const GcvRowsArgs& a, double* out6);

}  // namespace dgpu
