// GCV / CV evaluation kernels on top of the batched solver:
//   * rss and GCV per system (src/solve.cpp:183-191):
//       rss = max(ywy - 2 theta.rhs + theta^T M theta, 0),
//       gcv = n rss / (n - edf)^2 (inf when n <= edf or the factorisation failed);
//   * CV held-out error per (lambda, fold) (src/solve.cpp:334-335);
//   * fold training systems M - M_g, rhs - rhs_g (src/solve.cpp:300-305);
//   * per-stamp moments and the Kronecker fold assembly of the stamped CV
//     solve (src/solve.cpp:584-629).
#include <cuda_runtime.h>

#include <algorithm>

#include "dev_common.cuh"
#include "fit_internal.h"
#include "gls_internal.h"

namespace dgpu {

__device__ double block_sum(double v, double* red) {
  red[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < static_cast<unsigned>(o)) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  const double r = red[0];
  __syncthreads();
  return r;
}

// theta^T Mq theta - 2 theta . rq + yq for system s (M/r/y chosen by index).
// With an anchor theta0 (one per r index) the vector is theta - theta0: given
// rq = X^T W e0 and yq = e0^T W e0 for the residual e0 = t - X theta0, that is
// the rss of theta expanded around theta0, whose quadratic term is small near
// the anchor.
// Grid (row blocks of kQRows, systems): each CTA forms the partial sums of its
// rows (one warp per row of M, coalesced); k_quad_finish adds the row blocks
// of each system in a fixed order.
constexpr int kQRows = 32;

__global__ void __launch_bounds__(256)
k_quad_err(int P, const double* __restrict__ theta, const double* __restrict__ M, const int* __restrict__ m_index,
           const double* __restrict__ r, const int* __restrict__ r_index, const double* __restrict__ anchor,
           double* __restrict__ part) {
  __shared__ double red[256];
  __shared__ double th[1024];
  const int b = blockIdx.x, s = blockIdx.y, nb = gridDim.x;
  const double* Mq = M + (m_index ? static_cast<size_t>(m_index[s]) * P * P : 0);
  const double* rq = r + (r_index ? static_cast<size_t>(r_index[s]) * P : 0);
  const double* aq = anchor ? anchor + (r_index ? static_cast<size_t>(r_index[s]) * P : 0) : nullptr;
  for (int p = threadIdx.x; p < P; p += blockDim.x)
    th[p] = theta[static_cast<size_t>(s) * P + p] - (aq ? aq[p] : 0.0);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int p0 = b * kQRows, p1 = min(P, p0 + kQRows);
  double quad = 0.0, lin = 0.0;
  for (int p = p0 + warp; p < p1; p += nw) {
    const double* row = Mq + static_cast<size_t>(p) * P;
    double a = 0.0;
    for (int q = lane; q < P; q += 32) a = fma(row[q], th[q], a);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if (lane == 0) quad = fma(th[p], a, quad);
  }
  for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) lin = fma(th[p], rq[p], lin);
  const double Q = block_sum(quad, red);
  const double L = block_sum(lin, red);
  if (threadIdx.x == 0) {
    part[(static_cast<size_t>(s) * nb + b) * 2] = Q;
    part[(static_cast<size_t>(s) * nb + b) * 2 + 1] = L;
  }
}

__global__ void k_quad_finish(int nsys, int nb, const double* __restrict__ part, const double* __restrict__ y,
                              const int* __restrict__ r_index, double* __restrict__ out) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nsys; s += gridDim.x * blockDim.x) {
    double Q = 0.0, L = 0.0;
    for (int b = 0; b < nb; ++b) {
      Q += part[(static_cast<size_t>(s) * nb + b) * 2];
      L += part[(static_cast<size_t>(s) * nb + b) * 2 + 1];
    }
    out[s] = y[r_index ? r_index[s] : 0] - 2.0 * L + Q;
  }
}

// theta0 = theta of the first system with the smallest curve value (NaN never
// wins; all-NaN picks system 0), the host's argmin rule.
__global__ void k_argmin_copy(int nsys, const double* __restrict__ curve, const double* __restrict__ theta, int P,
                              double* __restrict__ theta0) {
  __shared__ int s_best;
  if (threadIdx.x == 0) {
    int b = 0;
    double bg = __longlong_as_double(0x7ff0000000000000ll);
    for (int i = 0; i < nsys; ++i)
      if (curve[i] < bg) {
        bg = curve[i];
        b = i;
      }
    s_best = b;
  }
  __syncthreads();
  const double* src = theta + static_cast<size_t>(s_best) * P;
  for (int p = threadIdx.x; p < P; p += blockDim.x) theta0[p] = src[p];
}

void launch_argmin_copy(cudaStream_t st, int nsys, const double* curve, const double* theta, int P,
                        double* theta0) {
  k_argmin_copy<<<1, 256, 0, st>>>(nsys, curve, theta, P, theta0);
  DGPU_LAUNCH("k_argmin_copy");
}

void launch_quad_err(Context& c, int nsys, int P, const double* theta, const double* M, const int* m_index,
                     const double* r, const int* r_index, const double* y, double* out, const double* anchor) {
  if (nsys == 0) return;
  const int nb = (P + kQRows - 1) / kQRows;
  double* part = static_cast<double*>(c.slot(kSlotGlsPart, sizeof(double) * 2 * static_cast<size_t>(nb) * nsys));
  k_quad_err<<<dim3(nb, nsys), 256, 0, c.stream>>>(P, theta, M, m_index, r, r_index, anchor, part);
  DGPU_LAUNCH("k_quad_err");
  k_quad_finish<<<(nsys + 127) / 128, 128, 0, c.stream>>>(nsys, nb, part, y, r_index, out);
  DGPU_LAUNCH("k_quad_finish");
}

__global__ void k_gcv_finish(int nsys, const double* __restrict__ raw, const double* __restrict__ edf,
                             const int* __restrict__ ok, const long long* __restrict__ n, double* __restrict__ rss,
                             double* __restrict__ gcv) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  double r = raw[s];
  if (r < 0.0) r = 0.0;
  rss[s] = r;
  const double nn = static_cast<double>(*n);
  const double denom = nn - edf[s];
  gcv[s] = (ok[s] && denom > 0.0) ? nn * r / (denom * denom) : __longlong_as_double(0x7ff0000000000000ll);
}

void launch_gcv_finish(cudaStream_t st, int nsys, const double* raw, const double* edf, const int* ok,
                       const long long* n, double* rss, double* gcv) {
  k_gcv_finish<<<(nsys + 127) / 128, 128, 0, st>>>(nsys, raw, edf, ok, n, rss, gcv);
  DGPU_LAUNCH("k_gcv_finish");
}

// out[g] = all - part[g] for g < groups (matrices or vectors of length len).
__global__ void k_sub_parts(int groups, size_t len, const double* __restrict__ all, const double* __restrict__ part,
                            double* __restrict__ out) {
  const size_t total = static_cast<size_t>(groups) * len;
  for (size_t e = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<size_t>(gridDim.x) * blockDim.x)
    out[e] = all[e % len] - part[e];
}

__global__ void k_sum_parts(int groups, size_t len, const double* __restrict__ part, double* __restrict__ all) {
  for (size_t e = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < len;
       e += static_cast<size_t>(gridDim.x) * blockDim.x) {
    double s = 0.0;
    for (int g = 0; g < groups; ++g) s += part[static_cast<size_t>(g) * len + e];
    all[e] = s;
  }
}

void launch_fold_train(cudaStream_t st, int groups, size_t len, const double* part, double* all, double* train) {
  const int blocks = static_cast<int>(std::min<size_t>((len + 255) / 256, 148 * 8));
  k_sum_parts<<<std::max(blocks, 1), 256, 0, st>>>(groups, len, part, all);
  DGPU_LAUNCH("k_sum_parts");
  const int b2 = static_cast<int>(std::min<size_t>((groups * len + 255) / 256, 148 * 8));
  k_sub_parts<<<std::max(b2, 1), 256, 0, st>>>(groups, len, all, part, train);
  DGPU_LAUNCH("k_sub_parts");
}

// Per-stamp moments over the stamp's active rows: A_s = sum w b b^T (nf x nf,
// full), r_s = sum w t b, ds2_s = sum w t^2, pixel-centroid sums.
__global__ void __launch_bounds__(256)
k_stamp_moments(int nc, int SS, FitRows R, const uint8_t* __restrict__ accepted, double* __restrict__ As,
                double* __restrict__ rs, double* __restrict__ ds2, double* __restrict__ cen) {
  const int s = blockIdx.x, nf = nc + 1;
  const bool act_stamp = accepted[s] != 0;
  // entries: nf*nf (A) + nf (r) + 1 (ds2) + 3 (sx, sy, count); one thread per
  // entry, rows summed in order.
  const int ne = nf * nf + nf + 4;
  for (int e = threadIdx.x; e < ne; e += blockDim.x) {
    double acc = 0.0;
    if (act_stamp) {
      for (int i = 0; i < SS; ++i) {
        const size_t row = static_cast<size_t>(s) * SS + i;
        if (!R.valid[row]) continue;
        const double w = R.w[row], t = R.t[row];
        double v;
        if (e < nf * nf) {
          const int a = e / nf, b = e % nf;
          const double ba = a < nc ? R.bn[row * nc + a] : 1.0;
          const double bb = b < nc ? R.bn[row * nc + b] : 1.0;
          v = w * ba * bb;
        } else if (e < nf * nf + nf) {
          const int a = e - nf * nf;
          const double ba = a < nc ? R.bn[row * nc + a] : 1.0;
          v = w * t * ba;
        } else if (e == nf * nf + nf) {
          v = w * t * t;
        } else if (e == nf * nf + nf + 1) {
          v = static_cast<double>(R.px[row]);
        } else if (e == nf * nf + nf + 2) {
          v = static_cast<double>(R.py[row]);
        } else {
          v = 1.0;
        }
        acc += v;
      }
    }
    const double tot = acc;
    if (e < nf * nf)
      As[static_cast<size_t>(s) * nf * nf + e] = tot;
    else if (e < nf * nf + nf)
      rs[static_cast<size_t>(s) * nf + (e - nf * nf)] = tot;
    else if (e == nf * nf + nf)
      ds2[s] = tot;
    else
      cen[static_cast<size_t>(s) * 3 + (e - nf * nf - nf - 1)] = tot;
  }
}

void launch_stamp_moments(cudaStream_t st, int n_stamps, int nc, int SS, const FitRows& R, const uint8_t* accepted,
                          double* As, double* rs, double* ds2, double* cen) {
  if (n_stamps == 0) return;
  k_stamp_moments<<<n_stamps, 256, 0, st>>>(nc, SS, R, accepted, As, rs, ds2, cen);
  DGPU_LAUNCH("k_stamp_moments");
}

// Fold assembly M_g = sum_{s in g} A_s (x) d_s d_s^T, rf_g(c-block) = sum r_s(c) d_s,
// ysq_g = sum ds2_s (src/solve.cpp:605-629).
__global__ void k_stamped_assemble(int groups, int nstamp, int nf, int k, const int* __restrict__ fold,
                                   const double* __restrict__ As, const double* __restrict__ rs,
                                   const double* __restrict__ ds2, const double* __restrict__ dsd,
                                   double* __restrict__ Mg, double* __restrict__ rg, double* __restrict__ yg) {
  const int P = nf * k;
  const size_t per = static_cast<size_t>(P) * P + P + 1;
  const size_t total = static_cast<size_t>(groups) * per;
  for (size_t e = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int g = static_cast<int>(e / per);
    const size_t o = e - static_cast<size_t>(g) * per;
    double acc = 0.0;
    if (o < static_cast<size_t>(P) * P) {
      const int p = static_cast<int>(o / P), q = static_cast<int>(o % P);
      const int c = p / k, m = p % k, c2 = q / k, m2 = q % k;
      for (int s = 0; s < nstamp; ++s) {
        if (fold[s] != g) continue;
        acc += As[static_cast<size_t>(s) * nf * nf + c * nf + c2] * (dsd[static_cast<size_t>(s) * k + m] *
                                                                       dsd[static_cast<size_t>(s) * k + m2]);
      }
      Mg[static_cast<size_t>(g) * P * P + o] = acc;
    } else if (o < static_cast<size_t>(P) * P + P) {
      const int p = static_cast<int>(o - static_cast<size_t>(P) * P);
      const int c = p / k, m = p % k;
      for (int s = 0; s < nstamp; ++s)
        if (fold[s] == g) acc += rs[static_cast<size_t>(s) * nf + c] * dsd[static_cast<size_t>(s) * k + m];
      rg[static_cast<size_t>(g) * P + p] = acc;
    } else {
      for (int s = 0; s < nstamp; ++s)
        if (fold[s] == g) acc += ds2[s];
      yg[g] = acc;
    }
  }
}

void launch_stamped_assemble(cudaStream_t st, int groups, int nstamp, int nf, int k, const int* fold,
                             const double* As, const double* rs, const double* ds2, const double* dsd, double* Mg,
                             double* rg, double* yg) {
  const size_t P = static_cast<size_t>(nf) * k;
  const size_t total = static_cast<size_t>(groups) * (P * P + P + 1);
  const int blocks = static_cast<int>(std::min<size_t>((total + 255) / 256, 148 * 16));
  k_stamped_assemble<<<std::max(blocks, 1), 256, 0, st>>>(groups, nstamp, nf, k, fold, As, rs, ds2, dsd, Mg, rg, yg);
  DGPU_LAUNCH("k_stamped_assemble");
}

// theta += delta (refinement).
__global__ void k_axpy(int n, const double* __restrict__ d, double* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += d[i];
}

// r = r - lam * P0 theta  (P0 = blockdiag pen), for the refinement residual.
__global__ void k_sub_penalty(int P, int k, const double* __restrict__ pen, double lam, const double* __restrict__ th,
                              double* __restrict__ r) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const int b = p / k, m = p % k;
  double a = 0.0;
  for (int q = 0; q < k; ++q) a = fma(pen[m * k + q], th[b * k + q], a);
  r[p] -= lam * a;
}

void launch_refine_update(cudaStream_t st, int P, int k, const double* pen, double lam, const double* theta,
                          double* r) {
  k_sub_penalty<<<(P + 255) / 256, 256, 0, st>>>(P, k, pen, lam, theta, r);
  DGPU_LAUNCH("k_sub_penalty");
}

void launch_axpy(cudaStream_t st, int n, const double* d, double* x) {
  k_axpy<<<(n + 255) / 256, 256, 0, st>>>(n, d, x);
  DGPU_LAUNCH("k_axpy");
}

}  // namespace dgpu
