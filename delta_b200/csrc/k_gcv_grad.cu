// Gradient of the stamp fit's GCV score (reference src/solve.cpp:147-193,
// GCV = n RSS / (n - edf)^2) and of its weighted residual sum of squares RSS,
// with respect to log lambda, the kernel shift (dx, dy) and the scale s, by the
// adjoint of the normal-equation map. No reference counterpart.
//
// The stamp rows are X_row = u(row) (x) d(row) (u_c = s B_n,c for c < nc, the
// B_n convolved with the shifted basis; u_nc = 1 for the background; d the
// thin-plate design row), M = X^T W X, b = X^T W t, A = M + lambda P0 with
// P0 = F F^T, theta = A^-1 b, H = A^-1 F. With g = dRSS/dtheta = -2 lambda P0 theta
// and z = A^-1 g = -2 lambda H (F^T theta):
//   dRSS/dM = theta theta^T - sym(z theta^T),  dRSS/db = -2 theta + z,
//   dedf/dM = lambda H H^T,                   dedf/db = 0,
//   dGCV = alpha dRSS + beta dedf,  alpha = n/(n-edf)^2, beta = 2 n RSS/(n-edf)^3,
//   dRSS/dlambda = 2 lambda (F^T theta)^T (F^T H) (F^T theta),
//   dedf/dlambda = -tr(F^T H) + lambda ||F^T H||_F^2.
// Back through X: Xbar = 2 W X Mbar + W t bbar^T, and per row
// Ubar_c = sum_j d_j Xbar_(c,j); then dx += sum_c Ubar_c dU_c/ddx with
// dU_c/ddx = -s B^x_n,c (the B_n of the x-derivative taps), dy alike, and
// ds += sum_c Ubar_c u_c / s. The H H^T part is applied column by column of H
// (Y_q = X_row h_q, then Y_q (d-contracted h_q)), so no P x P matrix is formed.
#include <cuda_runtime.h>

#include <algorithm>

#include "dev_common.cuh"
#include "fit_internal.h"
#include "gcv_grad_internal.h"

namespace dgpu {

// B = [rhs | F] (P x (1 + nf r)), F = blockdiag(fk) over the nf fields.
__global__ void k_build_rhs_f(int P, int k, int r, const double* __restrict__ rhs, const double* __restrict__ fk,
                              double* __restrict__ B) {
  const int m = 1 + (P / k) * r;
  const int64_t n = static_cast<int64_t>(P) * m;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int p = static_cast<int>(e / m), col = static_cast<int>(e - static_cast<int64_t>(p) * m);
    double v;
    if (col == 0) {
      v = rhs[p];
    } else {
      const int q = col - 1, fb = q / r, i = q - fb * r;
      v = (p / k == fb) ? fk[(p % k) * r + i] : 0.0;
    }
    B[e] = v;
  }
}

// theta (column 0 of X) contiguous; ftheta_q = f_q . theta.
__global__ void k_theta_ftheta(int P, int k, int r, const double* __restrict__ X, const double* __restrict__ fk,
                               double* __restrict__ theta, double* __restrict__ ftheta) {
  const int m = 1 + (P / k) * r;
  for (int p = threadIdx.x; p < P; p += blockDim.x) theta[p] = X[static_cast<size_t>(p) * m];
  for (int q = threadIdx.x; q < m - 1; q += blockDim.x) {
    const int fb = q / r, i = q - fb * r;
    double s = 0.0;
    for (int j = 0; j < k; ++j) s = fma(fk[j * r + i], X[static_cast<size_t>(fb * k + j) * m], s);
    ftheta[q] = s;
  }
}

// Row q of G = F^T H: stats[q] = {G_qq, sum_q' G_qq'^2, ftheta_q * (G ftheta)_q}.
__global__ void k_fth_rows(int P, int k, int r, const double* __restrict__ X, const double* __restrict__ fk,
                           const double* __restrict__ ftheta, double* __restrict__ stats) {
  const int m = 1 + (P / k) * r, nq = m - 1;
  const int q = blockIdx.x, fb = q / r, i = q - fb * r;
  __shared__ double red[3][32];
  double sq = 0.0, gf = 0.0, diag = 0.0;
  for (int q2 = threadIdx.x; q2 < nq; q2 += blockDim.x) {
    double g = 0.0;
    for (int j = 0; j < k; ++j) g = fma(fk[j * r + i], X[static_cast<size_t>(fb * k + j) * m + 1 + q2], g);
    sq = fma(g, g, sq);
    gf = fma(g, ftheta[q2], gf);
    if (q2 == q) diag = g;
  }
  for (int o = 16; o > 0; o >>= 1) {
    sq += __shfl_xor_sync(0xffffffffu, sq, o);
    gf += __shfl_xor_sync(0xffffffffu, gf, o);
    diag += __shfl_xor_sync(0xffffffffu, diag, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][warp] = diag;
    red[1][warp] = sq;
    red[2][warp] = gf;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += red[threadIdx.x][w];
    stats[static_cast<size_t>(q) * 3 + threadIdx.x] = threadIdx.x == 2 ? t * ftheta[q] : t;
  }
}

// z = -2 lambda H ftheta.
__global__ void k_zvec(int P, int k, int r, const double* __restrict__ X, const double* __restrict__ ftheta, double lam,
                       double* __restrict__ z) {
  const int m = 1 + (P / k) * r;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  double s = 0.0;
  for (int q = 0; q < m - 1; ++q) s = fma(X[static_cast<size_t>(p) * m + 1 + q], ftheta[q], s);
  z[p] = -2.0 * lam * s;
}

// GCV scalars from the fixed-order sums. sums = {trace G, ||G||^2, ftheta^T G ftheta};
// raw = ywy - 2 theta.b + theta^T M theta; n rows.
__global__ void k_gcv_scalars(int P, double lam, const double* __restrict__ sums, const double* __restrict__ raw,
                              const long long* __restrict__ n, GcvScalars* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double nn = static_cast<double>(*n);
  double rss = *raw;
  if (rss < 0.0) rss = 0.0;
  const double edf = static_cast<double>(P) - lam * sums[0];
  const double den = nn - edf;
  GcvScalars s;
  s.rss = rss;
  s.edf = edf;
  s.n = nn;
  s.gcv = den > 0.0 ? nn * rss / (den * den) : __longlong_as_double(0x7ff0000000000000ll);
  s.alpha = den > 0.0 ? nn / (den * den) : 0.0;
  s.beta = den > 0.0 ? 2.0 * nn * rss / (den * den * den) : 0.0;
  const double drss = 2.0 * lam * sums[2];
  const double dedf = -sums[0] + lam * sums[1];
  s.drss_dloglam = lam * drss;
  s.dgcv_dloglam = lam * (s.alpha * drss + s.beta * dedf);
  s.lam = lam;
  *out = s;
}

constexpr int kGrRows = 128;  // rows (threads) per block
constexpr int kGrQc = 8;      // columns of H staged per step
constexpr int kGrMaxK = 32;

// Per block: {dGCV/ddx, dGCV/ddy, dGCV/ds, dRSS/ddx, dRSS/ddy, dRSS/ds} over its rows.
__global__ void __launch_bounds__(kGrRows) k_gcv_rows(GcvRowsArgs a) {
  extern __shared__ __align__(16) double gsm[];
  const int nc = a.nc, nf = nc + 1, k = a.k, P = nf * k, nq = a.nq, m = nq + 1;
  double* sh = gsm;                             // P x kGrQc
  double* su = sh + static_cast<size_t>(P) * kGrQc;  // nc x rows: u
  double* sx = su + static_cast<size_t>(nc) * kGrRows;
  double* sy = sx + static_cast<size_t>(nc) * kGrRows;
  const int tid = threadIdx.x;
  const int64_t row = static_cast<int64_t>(blockIdx.x) * kGrRows + tid;
  const bool live = row < a.N && a.valid[row] && a.w[row] > 0.0;
  const GcvScalars S = *a.scal;
  const double wr = live ? a.w[row] : 0.0, tr = live ? a.t[row] : 0.0;
  double d[kGrMaxK];
#pragma unroll
  for (int j = 0; j < kGrMaxK; ++j) d[j] = (live && j < k) ? a.d[row * k + j] : 0.0;
  for (int c = 0; c < nc; ++c) {
    su[c * kGrRows + tid] = live ? a.bn[row * nc + c] : 0.0;
    sx[c * kGrRows + tid] = live ? a.bnx[row * nc + c] : 0.0;
    sy[c * kGrRows + tid] = live ? a.bny[row * nc + c] : 0.0;
  }
  double g[6] = {0, 0, 0, 0, 0, 0};
  const double inv_s = 1.0 / a.scale;
  if (live) {
    // X theta and X z.
    double xt = 0.0, xz = 0.0;
    for (int c = 0; c < nf; ++c) {
      double dt = 0.0, dz = 0.0;
#pragma unroll
      for (int j = 0; j < kGrMaxK; ++j)
        if (j < k) {
          dt = fma(d[j], a.theta[c * k + j], dt);
          dz = fma(d[j], a.z[c * k + j], dz);
        }
      const double u = c < nc ? su[c * kGrRows + tid] : 1.0;
      xt = fma(u, dt, xt);
      xz = fma(u, dz, xz);
    }
    for (int c = 0; c < nc; ++c) {
      double dt = 0.0, dz = 0.0;
#pragma unroll
      for (int j = 0; j < kGrMaxK; ++j)
        if (j < k) {
          dt = fma(d[j], a.theta[c * k + j], dt);
          dz = fma(d[j], a.z[c * k + j], dz);
        }
      // RSS part (alpha = 1): 2 w (X Mbar)_c + w t bbar_c, d-contracted.
      const double ur = 2.0 * wr * (xt * dt - 0.5 * (xz * dt + xt * dz)) + wr * tr * (-2.0 * dt + dz);
      const double u = su[c * kGrRows + tid];
      const double bx = sx[c * kGrRows + tid], by = sy[c * kGrRows + tid];
      g[3] -= ur * bx;
      g[4] -= ur * by;
      g[5] += ur * u * inv_s;
      const double ug = S.alpha * ur;
      g[0] -= ug * bx;
      g[1] -= ug * by;
      g[2] += ug * u * inv_s;
    }
  }
  // dedf part of GCV: 2 w beta lambda sum_q Y_q (d-contracted h_q), Y_q = X_row h_q.
  const double coef = 2.0 * wr * S.beta * S.lam;
  for (int q0 = 0; q0 < nq; q0 += kGrQc) {
    const int qn = min(kGrQc, nq - q0);
    __syncthreads();
    for (int e = tid; e < P * kGrQc; e += blockDim.x) {
      const int p = e / kGrQc, qq = e - p * kGrQc;
      sh[e] = qq < qn ? a.X[static_cast<size_t>(p) * m + 1 + q0 + qq] : 0.0;
    }
    __syncthreads();
    if (!live) continue;
    for (int qq = 0; qq < qn; ++qq) {
      double yq = 0.0, sxq = 0.0, syq = 0.0, suq = 0.0;
      for (int c = 0; c < nf; ++c) {
        const double* hc = sh + static_cast<size_t>(c) * k * kGrQc + qq;
        double dh = 0.0;
#pragma unroll
        for (int j = 0; j < kGrMaxK; ++j)
          if (j < k) dh = fma(d[j], hc[j * kGrQc], dh);
        if (c < nc) {
          const double u = su[c * kGrRows + tid];
          yq = fma(u, dh, yq);
          suq = fma(u, dh, suq);
          sxq = fma(sx[c * kGrRows + tid], dh, sxq);
          syq = fma(sy[c * kGrRows + tid], dh, syq);
        } else {
          yq += dh;
        }
      }
      const double cy = coef * yq;
      g[0] -= cy * sxq;
      g[1] -= cy * syq;
      g[2] += cy * suq * inv_s;
    }
  }
  // Fixed-order block reduction.
  __shared__ double red[6][kGrRows / 32];
  for (int i = 0; i < 6; ++i) {
    double v = g[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((tid & 31) == 0) red[i][tid >> 5] = v;
  }
  __syncthreads();
  if (tid < 6) {
    double t = 0.0;
    for (int w = 0; w < kGrRows / 32; ++w) t += red[tid][w];
    a.partial[static_cast<size_t>(blockIdx.x) * 6 + tid] = t;
  }
}

// Fixed-order column sums (one thread per column, rows in order).
__global__ void k_colsum(const double* __restrict__ part, int nrows, int ncols, double* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncols) return;
  double t = 0.0;
  for (int r = 0; r < nrows; ++r) t += part[static_cast<size_t>(r) * ncols + c];
  out[c] = t;
}

int gcv_rhs_cols(int P, int k, int r) { return 1 + (P / k) * r; }

void launch_build_rhs_f(cudaStream_t st, int P, int k, int r, const double* rhs, const double* fk, double* B) {
  const int64_t n = static_cast<int64_t>(P) * gcv_rhs_cols(P, k, r);
  k_build_rhs_f<<<static_cast<int>(std::min<int64_t>((n + 255) / 256, 1184)), 256, 0, st>>>(P, k, r, rhs, fk, B);
  DGPU_LAUNCH("k_build_rhs_f");
}

void launch_gcv_theta(cudaStream_t st, int P, int k, int r, const double* X, const double* fk, double* work) {
  const int nq = gcv_rhs_cols(P, k, r) - 1;
  k_theta_ftheta<<<1, 512, 0, st>>>(P, k, r, X, fk, work, work + P);
  DGPU_LAUNCH("k_theta_ftheta");
  (void)nq;
}

void launch_gcv_stats(cudaStream_t st, int P, int k, int r, const double* X, const double* fk, double lam,
                      const double* raw, const long long* n, double* work, GcvScalars* scal) {
  const int nq = gcv_rhs_cols(P, k, r) - 1;
  double* theta = work;
  double* ftheta = theta + P;
  double* z = ftheta + nq;
  double* stats = z + P;
  double* sums = stats + 3 * static_cast<size_t>(nq);
  (void)theta;
  k_fth_rows<<<nq, 256, 0, st>>>(P, k, r, X, fk, ftheta, stats);
  DGPU_LAUNCH("k_fth_rows");
  k_colsum<<<1, 32, 0, st>>>(stats, nq, 3, sums);
  DGPU_LAUNCH("k_colsum");
  k_zvec<<<(P + 127) / 128, 128, 0, st>>>(P, k, r, X, ftheta, lam, z);
  DGPU_LAUNCH("k_zvec");
  k_gcv_scalars<<<1, 32, 0, st>>>(P, lam, sums, raw, n, scal);
  DGPU_LAUNCH("k_gcv_scalars");
}

size_t gcv_stats_doubles(int P, int k, int r) {
  const int nq = gcv_rhs_cols(P, k, r) - 1;
  return 2 * static_cast<size_t>(P) + 4 * static_cast<size_t>(nq) + 8;
}

int gcv_rows_blocks(int64_t N) { return static_cast<int>((N + kGrRows - 1) / kGrRows); }

void launch_gcv_rows(cudaStream_t st, const GcvRowsArgs& a, double* out6) {
  if (a.k > kGrMaxK) fail(DGPU_ERR_INVALID, "stamp_gcv: at most 32 knots are supported");
  const int P = (a.nc + 1) * a.k;
  const size_t smem = sizeof(double) * (static_cast<size_t>(P) * kGrQc + 3 * static_cast<size_t>(a.nc) * kGrRows);
  if (smem > 200 * 1024) fail(DGPU_ERR_INVALID, "stamp_gcv: basis too large for the row contraction");
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_gcv_rows), smem);
  const int nb = gcv_rows_blocks(a.N);
  k_gcv_rows<<<nb, kGrRows, smem, st>>>(a);
  DGPU_LAUNCH("k_gcv_rows");
  k_colsum<<<1, 32, 0, st>>>(a.partial, nb, 6, out6);
  DGPU_LAUNCH("k_colsum");
}

}  // namespace dgpu
