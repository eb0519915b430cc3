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
  // Optional twiddle table (launch_twiddle_table): n/2 forward and inverse
  // length-n twiddles, n/4 forward and inverse length-n/2 twiddles, then n/2+1
  // forward and inverse r2c split factors. Null: kernels compute them.
  const float2* tw_tab = nullptr;
};

FftGeom make_fft_geom(int n);
size_t twiddle_table_len(int n);
void launch_twiddle_table(cudaStream_t s, int n, float2* tab);
void launch_rows_fwd(cudaStream_t s, const FftGeom& g, int mode, int nitems, const float* src, int w, int h,
                     const int* oxs, const int* oys, int nox, float2* spec);
void launch_cols(cudaStream_t s, const FftGeom& g, int mode, int nitems, float2* spec, const double* cell_power,
                 const double* cell_sumk2, const int* block_cell, const double* vsr, double* power_out);
void launch_rows_inv(cudaStream_t s, const FftGeom& g, int mode, int nitems, const float2* spec, const int* items,
                     int w, int h, const int* oxs, const int* oys, int nox, const double* hwin, const double* vsr,
                     const double* cell_sumk2, const int* block_cell, float* acc, float* var_acc, float* dense_out);
// The three passes of mode 0 (r2c rows, filtered columns, raw c2r rows into
// dense_out) fused per block in one cluster launch; needs n = 256 and tw_tab.
bool block_filter_fused(const FftGeom& g);
void launch_block_filter(cudaStream_t s, const FftGeom& g, int nitems, const float* src, int w, int h,
                         const int* oxs, const int* oys, int nox, const double* cell_power, const double* cell_sumk2,
                         const int* block_cell, const double* vsr, double* bnum, float* dense_out);
void launch_block_var(cudaStream_t s, const FftGeom& g, int nitems, int nextra, const float* vs, const float* vr,
                      int w, int h, const int* oxs, const int* oys, int nox, double* vsr);
void launch_local_kernels(cudaStream_t s, const FftGeom& g, int ncell, const TpsDev& t, const double* theta, int nc,
                          const float* phi, int ks, const double* centres, double* sumk2, float* dense,
                          float* kern_out);
void launch_ola_normalise(cudaStream_t s, int w, int h, const double* wx_total, const double* wy_total, float* acc,
                          float* var_acc);
// Overlap-add of the raw block outputs `bout` (item x n x n) into acc / var_acc,
// in the reference's colour order, normalised by the weight sums.
void launch_ola_gather(cudaStream_t s, int w, int h, int n, const int* oxs, int nox, const int* oys, int noy,
                       const double* hwin, const float* bout, const double* bnum, const double* wx_total,
                       const double* wy_total, float* acc, float* var_acc);

}  // namespace dgpu
