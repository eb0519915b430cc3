// Pivoted LDL^T fallback of the batched GLS solver (reference
// src/solve.cpp:177-181 for GCV / fixed lambda, :328-333 for CV folds).
//
// The batched Cholesky (k_solve_cluster) marks a system whose factorisation
// met a non-positive pivot with ok = 0. This kernel then redoes exactly those
// systems the way the reference does when Eigen's LLT fails: Eigen 3.4's
// pivoted LDLT of A = M + lambda P0, theta = A^+ rhs and the effective degrees
// of freedom edf = tr(A^+ M), where A^+ is the LDLT solve with the
// pseudo-inverse of D (1/d where |d| > the smallest normal double, else 0).
// The pivot order is Eigen's: at step k the remaining diagonal entry of
// largest magnitude, read before that step's update (the left-looking variant
// never updates the trailing diagonal early), first on ties.
//
// It runs after every batched solve: a block whose systems all succeeded exits
// after reading their ok flags. Failed systems are rare (an under-constrained
// field at lambda ~ 0), so one 1024-thread CTA takes a system at a time, with
// the matrix in a global workspace (L2-resident):
//   factor   P left-looking steps: pivot search (block argmax), symmetric
//            swap of full rows and columns, d_k by a block reduction, column k
//            of L by one warp per row (contiguous row reads);
//   theta    forward substitution by one warp (row-oriented), D^+, backward
//            substitution column-oriented by the block, inverse permutation;
//   edf      Z = L^-T D^+ L^-1 (Pi M Pi^T) with one thread per column (no
//            synchronisation between columns), summed down the diagonal in a
//            fixed order.
// A solved system is marked ok = 2, so callers can tell which arithmetic
// produced it. The trace costs O(P^3) and the whole fallback a few
// milliseconds at P ~ 500; it replaces a failed fit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>

#include "dev_common.cuh"
#include "fit_internal.h"

namespace dgpu {

constexpr int kLdltThreads = 1024;
constexpr int kLdltBlocks = 4;

size_t ldlt_work_doubles(int P) { return static_cast<size_t>(kLdltBlocks) * (2 * static_cast<size_t>(P) * P + P); }

namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum in a fixed order (warp sums, then warp 0 over the warps).
__device__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double t = lane < static_cast<int>(blockDim.x >> 5) ? red[lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) red[32] = t;
  }
  __syncthreads();
  return red[32];
}

}  // namespace

__global__ void __launch_bounds__(kLdltThreads) k_ldlt_fallback(SolveBatch b, double* __restrict__ work) {
  __shared__ double s_temp[1024];  // d_j L_kj of the current step; later the solve vector
  __shared__ double s_red[33];
  __shared__ double s_best[32];
  __shared__ int s_bidx[32];
  __shared__ int s_piv;
  __shared__ double s_dk;
  __shared__ int s_perm[1024];  // position -> original index
  const int P = b.P, kk = b.k, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarp = blockDim.x >> 5;
  const size_t PP = static_cast<size_t>(P) * P;
  double* A = work + static_cast<size_t>(blockIdx.x) * (2 * PP + P);
  double* Y = A + PP;
  double* dinv = Y + PP;
  for (int s = blockIdx.x; s < b.nsys; s += gridDim.x) {
    if (b.ok[s]) continue;  // same value for every thread of the block
    const double lam = b.lam[s];
    const double* M = b.M + static_cast<size_t>(b.m_index ? b.m_index[s] : 0) * PP;
    const double* rhs = b.rhs + static_cast<size_t>(b.r_index ? b.r_index[s] : 0) * P;
    // A = M + lambda P0 (P0 = one k x k penalty block per field).
    for (size_t e = tid; e < PP; e += blockDim.x) {
      const int i = static_cast<int>(e / P), j = static_cast<int>(e - static_cast<size_t>(i) * P);
      double v = M[e];
      if (i / kk == j / kk) v = fma(lam, b.pen[(i % kk) * kk + (j % kk)], v);
      A[e] = v;
    }
    for (int i = tid; i < P; i += blockDim.x) s_perm[i] = i;
    __syncthreads();

    int n_steps = P;
    for (int k = 0; k < P; ++k) {
      // Pivot: largest |A_ii| over i >= k, first on ties.
      double best = -1.0;
      int bi = P;
      for (int i = k + tid; i < P; i += blockDim.x) {
        const double v = fabs(A[static_cast<size_t>(i) * P + i]);
        if (v > best) {
          best = v;
          bi = i;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov > best || (ov == best && oi < bi)) {
          best = ov;
          bi = oi;
        }
      }
      if (lane == 0) {
        s_best[warp] = best;
        s_bidx[warp] = bi;
      }
      __syncthreads();
      if (tid == 0) {
        double bb = s_best[0];
        int ii = s_bidx[0];
        for (int w = 1; w < nwarp; ++w)
          if (s_best[w] > bb || (s_best[w] == bb && s_bidx[w] < ii)) {
            bb = s_best[w];
            ii = s_bidx[w];
          }
        // An all-zero diagonal at the first step: nothing to factor (D = 0).
        s_piv = (k == 0 && !(bb > 0.0)) ? -1 : (ii < P ? ii : k);
      }
      __syncthreads();
      const int piv = s_piv;
      if (piv < 0) {
        n_steps = 0;
        break;
      }
      if (piv != k) {
        for (int j = tid; j < P; j += blockDim.x) {
          const double t = A[static_cast<size_t>(k) * P + j];
          A[static_cast<size_t>(k) * P + j] = A[static_cast<size_t>(piv) * P + j];
          A[static_cast<size_t>(piv) * P + j] = t;
        }
        __syncthreads();
        for (int i = tid; i < P; i += blockDim.x) {
          const double t = A[static_cast<size_t>(i) * P + k];
          A[static_cast<size_t>(i) * P + k] = A[static_cast<size_t>(i) * P + piv];
          A[static_cast<size_t>(i) * P + piv] = t;
        }
        if (tid == 0) {
          const int t = s_perm[k];
          s_perm[k] = s_perm[piv];
          s_perm[piv] = t;
        }
        __syncthreads();
      }
      const double* Ak = A + static_cast<size_t>(k) * P;
      double part = 0.0;
      for (int j = tid; j < k; j += blockDim.x) {
        const double t = A[static_cast<size_t>(j) * P + j] * Ak[j];
        s_temp[j] = t;
        part = fma(Ak[j], t, part);
      }
      const double red = block_sum(part, s_red);  // synchronises: s_temp complete
      if (tid == 0) {
        const double dk = Ak[k] - red;
        A[static_cast<size_t>(k) * P + k] = dk;
        s_dk = dk;
      }
      __syncthreads();
      const double dk = s_dk;
      for (int i = k + 1 + warp; i < P; i += nwarp) {
        const double* Ai = A + static_cast<size_t>(i) * P;
        double acc = 0.0;
        for (int j = lane; j < k; j += 32) acc = fma(Ai[j], s_temp[j], acc);
        acc = warp_sum(acc);
        if (lane == 0) {
          const double v = Ai[k] - acc;
          A[static_cast<size_t>(i) * P + k] = dk != 0.0 ? v / dk : v;
        }
      }
      __syncthreads();
    }
    // Pseudo-inverse of D.
    for (int i = tid; i < P; i += blockDim.x) {
      const double d = n_steps ? A[static_cast<size_t>(i) * P + i] : 0.0;
      dinv[i] = fabs(d) > DBL_MIN ? 1.0 / d : 0.0;
    }
    __syncthreads();

    // theta: x = Pi rhs; forward L (unit, row-oriented, one warp); D^+;
    // backward L^T (column t of L^T = row t of L, the block over i < t).
    if (warp == 0) {
      for (int i = 0; i < P; ++i) {
        const double* Ai = A + static_cast<size_t>(i) * P;
        double acc = 0.0;
        for (int j = lane; j < i; j += 32) acc = fma(Ai[j], s_temp[j], acc);
        acc = warp_sum(acc);
        if (lane == 0) s_temp[i] = rhs[s_perm[i]] - acc;
        __syncwarp();
      }
    }
    __syncthreads();
    for (int i = tid; i < P; i += blockDim.x) s_temp[i] *= dinv[i];
    __syncthreads();
    for (int t = P - 1; t > 0; --t) {
      const double zt = s_temp[t];
      const double* At = A + static_cast<size_t>(t) * P;
      for (int i = tid; i < t; i += blockDim.x) s_temp[i] = fma(-At[i], zt, s_temp[i]);
      __syncthreads();
    }
    for (int i = tid; i < P; i += blockDim.x) b.theta[static_cast<size_t>(s) * P + s_perm[i]] = s_temp[i];

    // edf = tr(A^+ M) = sum_c Z_cc, Z = L^-T D^+ L^-1 B, B = Pi M Pi^T; thread c owns column c.
    double zc = 0.0;
    if (tid < P) {
      const int c = tid, oc = s_perm[c];
      for (int i = 0; i < P; ++i) {
        const double* Ai = A + static_cast<size_t>(i) * P;
        double v = M[static_cast<size_t>(s_perm[i]) * P + oc];  // B = Pi M Pi^T: the trace is of A^+ M
        for (int j = 0; j < i; ++j) v = fma(-Ai[j], Y[static_cast<size_t>(j) * P + c], v);
        Y[static_cast<size_t>(i) * P + c] = v;
      }
      for (int i = 0; i < P; ++i) Y[static_cast<size_t>(i) * P + c] *= dinv[i];
      for (int i = P - 1; i >= c; --i) {
        double v = Y[static_cast<size_t>(i) * P + c];
        for (int t = i + 1; t < P; ++t) v = fma(-A[static_cast<size_t>(t) * P + i], Y[static_cast<size_t>(t) * P + c], v);
        Y[static_cast<size_t>(i) * P + c] = v;
      }
      zc = Y[static_cast<size_t>(c) * P + c];
    }
    // Fixed-order sum over the columns.
    __syncthreads();
    s_temp[tid] = tid < P ? zc : 0.0;
    __syncthreads();
    if (tid == 0) {
      double e = 0.0;
      for (int c = 0; c < P; ++c) e += s_temp[c];
      b.edf[s] = e;
      b.ok[s] = 2;
    }
    __syncthreads();
  }
}

void launch_ldlt_fallback(Context& c, const SolveBatch& b) {
  if (b.nsys <= 0) return;
  if (b.P > kLdltThreads) fail(DGPU_ERR_INVALID, "solve: the LDLT fallback supports at most 1024 unknowns");
  double* work = static_cast<double*>(c.slot(kSlotLdlt, sizeof(double) * ldlt_work_doubles(b.P)));
  const int blocks = std::min(b.nsys, kLdltBlocks);
  k_ldlt_fallback<<<blocks, kLdltThreads, 0, c.stream>>>(b, work);
  DGPU_LAUNCH("k_ldlt_fallback");
}

}  // namespace dgpu
