// GCV / CV helper launchers (k_gls.cu).
#pragma once

#include "fit_internal.h"

namespace dgpu {

// out[s] = y - 2 (theta_s - anchor) . r + (theta_s - anchor)^T M (theta_s - anchor),
// with y, r and the anchor chosen by r_index; anchor null: theta_s itself.
void launch_quad_err(Context& c, int nsys, int P, const double* theta, const double* M, const int* m_index,
                     const double* r, const int* r_index, const double* y, double* out,
                     const double* anchor = nullptr);
// theta0 = the row of theta (P per row) at argmin(curve), chosen on the device.
void launch_argmin_copy(cudaStream_t st, int nsys, const double* curve, const double* theta, int P,
                        double* theta0);
void launch_gcv_finish(cudaStream_t st, int nsys, const double* raw, const double* edf, const int* ok,
                       const long long* n, double* rss, double* gcv);
void launch_fold_train(cudaStream_t st, int groups, size_t len, const double* part, double* all, double* train);
void launch_stamp_moments(cudaStream_t st, int n_stamps, int nc, int SS, const FitRows& R, const uint8_t* accepted,
                          double* As, double* rs, double* ds2, double* cen);
void launch_stamped_assemble(cudaStream_t st, int groups, int nstamp, int nf, int k, const int* fold,
                             const double* As, const double* rs, const double* ds2, const double* dsd, double* Mg,
                             double* rg, double* yg);
void launch_refine_update(cudaStream_t st, int P, int k, const double* pen, double lam, const double* theta,
                          double* r);
void launch_axpy(cudaStream_t st, int n, const double* d, double* x);

}  // namespace dgpu
