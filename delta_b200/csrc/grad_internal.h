// Weighted chi^2 of the kernel model and its adjoints (k_grad.cu, api_grad.cpp).
#pragma once

#include <cuda_runtime.h>

#include "internal.h"

namespace dgpu {

constexpr int kGradMaxNx = 9;   // n_max <= 8
constexpr int kGradMaxNc = 45;  // (n_max+1)(n_max+2)/2 at n_max 8

struct Chi2Args {
  int w = 0, h = 0;
  const float* sci = nullptr;
  const float* ref = nullptr;
  const uint8_t* rmask = nullptr;
  const float* weight = nullptr;  // W(x); 0 excludes a pixel
  const float* fill = nullptr;    // device: sanitised-reference fill value
  DevFields F;
  int n_max = 0, ks = 0, nc = 0;
  const int2* orders = nullptr;
  const float* gx = nullptr;   // g_n(u - dx), (n_max+1) x ks
  const float* dgx = nullptr;  // g_n'(u - dx)
  const float* gy = nullptr;   // g_n(v - dy)
  const float* dgy = nullptr;  // g_n'(v - dy)
  float scale = 1.0f;
  float* q = nullptr;          // optional: nf x (w*h), dchi2 / da_c(x)
  float* p = nullptr;          // optional: w*h, rbar * s (for the reference adjoint)
  double* partial = nullptr;   // chi2_tile_blocks x 4: chi2, d/ds, d/ddx, d/ddy
};

struct AdjRefArgs {
  int w = 0, h = 0;
  const float* p = nullptr;    // rbar * s
  const float* ref = nullptr;
  const uint8_t* rmask = nullptr;
  DevFields F;
  int ks = 0, nc = 0;
  const int2* orders = nullptr;
  const float* gx = nullptr;   // device taps (global), as in Chi2Args
  const float* gy = nullptr;
  float* out = nullptr;        // dchi2 / dR, w*h
};

size_t chi2_tile_smem(int n_max, int ks);
int chi2_tile_blocks(int w, int h);
void launch_chi2_tile(cudaStream_t st, const Chi2Args& a);
void launch_sum_rows(cudaStream_t st, const double* part, int nrows, int ncols, double* out);
int theta_grad_blocks();
void launch_theta_grad(cudaStream_t st, int w, int h, int nf, int k, const float* q, const DevFields& D,
                       double* part);
void launch_adjoint_reference(cudaStream_t st, const AdjRefArgs& a);

}  // namespace dgpu
