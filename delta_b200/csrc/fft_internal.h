// ZOGY decorrelation FFT launchers (k_fft.cu).
#pragma once

#include "internal.h"

namespace dgpu {

struct FftGeom {
  int n = 256;           // block side (power of two)
  int logn = 8;
  int rows_per_cta = 32; // row-pass lines per CTA
  int cols_per_cta = 8;  // column-pass lines per CTA
  int extra_bx = 0, extra_by = 0;  // window of the extra block-variance item
};

FftGeom make_fft_geom(int n);
void launch_rows_fwd(cudaStream_t s, const FftGeom& g, int mode, int nitems, const float* src, int w, int h,
                     const int* oxs, const int* oys, int nox, float2* spec);
void launch_cols(cudaStream_t s, const FftGeom& g, int mode, int nitems, float2* spec, const double* cell_power,
                 const double* cell_sumk2, const int* block_cell, const double* vsr, double* power_out);
void launch_rows_inv(cudaStream_t s, const FftGeom& g, int mode, int nitems, const float2* spec, const int* items,
                     int w, int h, const int* oxs, const int* oys, int nox, const double* hwin, const double* vsr,
                     const double* cell_sumk2, const int* block_cell, float* acc, float* var_acc, float* dense_out);
void launch_block_var(cudaStream_t s, const FftGeom& g, int nitems, int nextra, const float* vs, const float* vr,
                      int w, int h, const int* oxs, const int* oys, int nox, double* vsr);
void launch_local_kernels(cudaStream_t s, const FftGeom& g, int ncell, const TpsDev& t, const double* theta, int nc,
                          const float* phi, int ks, const double* centres, double* sumk2, float* dense,
                          float* kern_out);
void launch_ola_normalise(cudaStream_t s, int w, int h, const double* wx_total, const double* wy_total, float* acc,
                          float* var_acc);

}  // namespace dgpu
