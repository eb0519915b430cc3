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
// never updates the trailing diagonal early), first on ties. Because that
// order depends on the diagonal alone, it is replayed first and the permuted
// matrix factored without pivoting by a blocked algorithm (the same factors;
// the sums are taken in another order, so they agree to rounding).
//
// It runs after every batched solve, as three launches over chunks of up to
// kLdltChunk systems (a system whose Cholesky succeeded leaves each of them at
// once); a failed system gets a 1024-thread CTA for the factorisation and
// theta, then P / 128 CTAs for the trace, with its matrices in a per-system
// global workspace (L2-resident):
//   factor   the pivot order by one warp over the diagonal, then panels of 32
//            columns: the diagonal block by one warp, the rows below by one
//            thread each, the trailing lower triangle minus W L^T in 4 x 4
//            register blocks (build_pivoted, ldlt_blocked);
//   theta    forward substitution by one warp (row-oriented), D^+, backward
//            substitution column-oriented by the block, inverse permutation;
//   edf      Z = L^-T D^+ L^-1 (Pi M Pi^T) with one thread per column (no
//            synchronisation between columns), the diagonal summed in a fixed
//            order by the finishing launch.
// A solved system is marked ok = 2, so callers can tell which arithmetic
// produced it. Failed systems are rare for a well-posed fit, but a basis far
// narrower than the pixel scale makes every small-lambda system singular, so
// all of a batch's failures are factored at once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>

#include "dev_common.cuh"
#include "fit_internal.h"

namespace dgpu {

constexpr int kLdltThreads = 1024;
constexpr int kLdltChunk = 32;      // systems per round of the three launches
constexpr int kLdltTraceThreads = 128;

constexpr int kLb = 32;  // panel width of the blocked factorisation

// Per-system workspace: A (P x P, then L and D), Y (P x P), D^+ (P), the trace
// column terms (P), the transposed panels W^T and L^T of the factorisation
// (2 x kLb x P) as doubles; then per system the permutation (P) and a
// factored flag as ints.
__host__ __device__ inline size_t ldlt_sys_doubles(int P) {
  return 2 * static_cast<size_t>(P) * P + 2 * static_cast<size_t>(P) + 2 * static_cast<size_t>(kLb) * P;
}
size_t ldlt_work_bytes(int P, int nsys) {
  return sizeof(double) * ldlt_sys_doubles(P) * nsys + sizeof(int) * (static_cast<size_t>(P) + 1) * nsys;
}

namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace

// Block-shared scratch of the factorisation and solves.
struct LdltShared {
  double temp[1024];  // the pivot replay's diagonal; later a solve vector
  int piv;            // -1: the whole diagonal is zero
  int perm[1024];     // position -> original index
};

// Eigen's pivot order, from the diagonal alone: its LDLT is left-looking, so
// the trailing diagonal is never updated before its own step and step k's
// pivot (the largest |A_ii| over the positions not yet factored, first on
// ties) depends only on the diagonal of A = M + lambda P0 and the swaps made
// so far. One warp replays the P steps on the diagonal; the permuted matrix
// B = Pi A Pi^T is then factored without pivoting. Returns false when the
// whole diagonal is zero (Eigen then factors nothing).
__device__ bool build_pivoted(double* B, const double* M, int P, int kk, double lam, const double* pen,
                              LdltShared& S) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double* dg = S.temp;
  for (int i = tid; i < P; i += blockDim.x) {
    dg[i] = fma(lam, pen[(i % kk) * kk + (i % kk)], M[static_cast<size_t>(i) * P + i]);
    S.perm[i] = i;
  }
  if (tid == 0) S.piv = 0;
  __syncthreads();
  if (warp == 0) {
    for (int k = 0; k < P; ++k) {
      double best = -1.0;
      int bi = P;
      for (int i = k + lane; i < P; i += 32) {
        const double v = fabs(dg[i]);
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
      if (k == 0 && !(best > 0.0)) {
        if (lane == 0) S.piv = -1;
        break;
      }
      if (lane == 0 && bi < P && bi != k) {
        const double t = dg[k];
        dg[k] = dg[bi];
        dg[bi] = t;
        const int q = S.perm[k];
        S.perm[k] = S.perm[bi];
        S.perm[bi] = q;
      }
      __syncwarp();
    }
  }
  __syncthreads();
  if (S.piv < 0) return false;
  const size_t PP = static_cast<size_t>(P) * P;
  for (size_t e = threadIdx.x; e < PP; e += blockDim.x) {
    const int i = static_cast<int>(e / P), j = static_cast<int>(e - static_cast<size_t>(i) * P);
    const int pi = S.perm[i], pj = S.perm[j];
    double v = M[static_cast<size_t>(pi) * P + pj];
    if (pi / kk == pj / kk) v = fma(lam, pen[(pi % kk) * kk + (pj % kk)], v);
    B[e] = v;
  }
  __syncthreads();
  return true;
}

// LDL^T of B without pivoting (the lower triangle; L below the diagonal, D on
// it), right-looking over panels of kLb columns:
//   (a) the panel's diagonal block by one warp, left-looking inside it;
//   (b) the panel's rows below by one thread each, against the block;
//   (c) the trailing lower triangle minus W L^T (W = L D, both panels kept
//       transposed so a column read is contiguous), 4 x 4 entries per thread.
// A zero d_k leaves its column undivided, as Eigen does. Wt, Lt: kLb x P each.
__device__ void ldlt_blocked(double* B, int P, double* Wt, double* Lt) {
  __shared__ double blk[kLb][kLb + 1];
  __shared__ double dblk[kLb];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int p0 = 0; p0 < P; p0 += kLb) {
    const int nb = min(kLb, P - p0);
    if (warp == 0) {
      if (lane < nb)
        for (int c = 0; c <= lane; ++c) blk[lane][c] = B[static_cast<size_t>(p0 + lane) * P + p0 + c];
      __syncwarp();
      for (int k = 0; k < nb; ++k) {
        if (lane == k) {
          double d = blk[k][k];
          for (int j = 0; j < k; ++j) d = fma(-blk[k][j], dblk[j] * blk[k][j], d);
          dblk[k] = d;
        }
        __syncwarp();
        const double dk = dblk[k];
        if (lane > k && lane < nb) {
          double v = blk[lane][k];
          for (int j = 0; j < k; ++j) v = fma(-blk[lane][j], dblk[j] * blk[k][j], v);
          blk[lane][k] = dk != 0.0 ? v / dk : v;
        }
        __syncwarp();
      }
      if (lane < nb) {
        double* Br = B + static_cast<size_t>(p0 + lane) * P + p0;
        for (int c = 0; c < lane; ++c) Br[c] = blk[lane][c];
        Br[lane] = dblk[lane];
      }
    }
    __syncthreads();
    const int r0 = p0 + nb;
    for (int i = r0 + tid; i < P; i += blockDim.x) {
      double* Bi = B + static_cast<size_t>(i) * P + p0;
      for (int k = 0; k < nb; ++k) {
        double v = Bi[k];
        for (int j = 0; j < k; ++j) v = fma(-Bi[j], dblk[j] * blk[k][j], v);
        const double dk = dblk[k];
        const double l = dk != 0.0 ? v / dk : v;
        Bi[k] = l;
        Lt[static_cast<size_t>(k) * P + i] = l;
        Wt[static_cast<size_t>(k) * P + i] = l * dk;
      }
    }
    __syncthreads();
    const int T = P - r0;
    if (T > 0) {
      const int nt = (T + 3) / 4;
      const int nblocks = nt * (nt + 1) / 2;
      for (int b = tid; b < nblocks; b += blockDim.x) {
        int bi = static_cast<int>((sqrt(8.0 * b + 1.0) - 1.0) * 0.5);
        while ((bi + 1) * (bi + 2) / 2 <= b) ++bi;
        while (bi * (bi + 1) / 2 > b) --bi;
        const int bj = b - bi * (bi + 1) / 2;
        const int i0 = r0 + 4 * bi, j0 = r0 + 4 * bj;
        double acc[4][4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
        for (int k = 0; k < nb; ++k) {
          const double* wr = Wt + static_cast<size_t>(k) * P;
          const double* lr = Lt + static_cast<size_t>(k) * P;
          double wv[4], lv[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            wv[u] = i0 + u < P ? wr[i0 + u] : 0.0;
            lv[u] = j0 + u < P ? lr[j0 + u] : 0.0;
          }
#pragma unroll
          for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] = fma(wv[u], lv[v], acc[u][v]);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            const int ii = i0 + u, jj = j0 + v;
            if (ii < P && jj <= ii) B[static_cast<size_t>(ii) * P + jj] -= acc[u][v];
          }
      }
    }
    __syncthreads();
  }
}

// Pseudo-inverse of D.
__device__ void ldlt_dinv(const double* A, int P, int n_steps, double* dinv) {
  for (int i = threadIdx.x; i < P; i += blockDim.x) {
    const double d = n_steps ? A[static_cast<size_t>(i) * P + i] : 0.0;
    dinv[i] = fabs(d) > DBL_MIN ? 1.0 / d : 0.0;
  }
  __syncthreads();
}

struct LdltWork {
  double* d;  // chunk x ldlt_sys_doubles(P)
  int* i;     // chunk x (P + 1): permutation, factored flag
};

// One CTA per system of the chunk [s0, s0 + gridDim.x): factor and theta of a
// failed system; the factored flag tells the next two launches which systems
// to finish.
__global__ void __launch_bounds__(kLdltThreads) k_ldlt_factor(SolveBatch b, int s0, LdltWork wk) {
  __shared__ LdltShared S;
  const int P = b.P, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const size_t PP = static_cast<size_t>(P) * P;
  const int s = s0 + static_cast<int>(blockIdx.x);
  double* A = wk.d + blockIdx.x * ldlt_sys_doubles(P);
  double* dinv = A + 2 * PP;
  int* perm = wk.i + blockIdx.x * (static_cast<size_t>(P) + 1);
  int* factored = perm + P;
  if (b.ok[s]) {  // same value for every thread of the block
    if (tid == 0) *factored = 0;
    return;
  }
  const double lam = b.lam[s];
  const double* M = b.M + static_cast<size_t>(b.m_index ? b.m_index[s] : 0) * PP;
  const double* rhs = b.rhs + static_cast<size_t>(b.r_index ? b.r_index[s] : 0) * P;
  double* Wt = A + 2 * PP + 2 * static_cast<size_t>(P);
  const bool any = build_pivoted(A, M, P, b.k, lam, b.pen, S);
  if (any) ldlt_blocked(A, P, Wt, Wt + static_cast<size_t>(kLb) * P);
  ldlt_dinv(A, P, any ? P : 0, dinv);

  // theta: x = Pi rhs; forward L (unit, row-oriented, one warp); D^+;
  // backward L^T (column t of L^T = row t of L, the block over i < t).
  if (warp == 0) {
    for (int i = 0; i < P; ++i) {
      const double* Ai = A + static_cast<size_t>(i) * P;
      double acc = 0.0;
      for (int j = lane; j < i; j += 32) acc = fma(Ai[j], S.temp[j], acc);
      acc = warp_sum(acc);
      if (lane == 0) S.temp[i] = rhs[S.perm[i]] - acc;
      __syncwarp();
    }
  }
  __syncthreads();
  for (int i = tid; i < P; i += blockDim.x) S.temp[i] *= dinv[i];
  __syncthreads();
  for (int t = P - 1; t > 0; --t) {
    const double zt = S.temp[t];
    const double* At = A + static_cast<size_t>(t) * P;
    for (int i = tid; i < t; i += blockDim.x) S.temp[i] = fma(-At[i], zt, S.temp[i]);
    __syncthreads();
  }
  for (int i = tid; i < P; i += blockDim.x) {
    b.theta[static_cast<size_t>(s) * P + S.perm[i]] = S.temp[i];
    perm[i] = S.perm[i];
  }
  if (tid == 0) *factored = 1;
}

// Y[:, c] <- L^-T D^+ L^-1 Y[:, c] for the thread's column c (Y is P rows of
// stride ldy), the CTA's columns together, by panels of kLb rows. Per panel the
// threads solve its triangular block with their panel values in registers,
// then update the rows still to come with the panel's L read once into shared
// memory (chunks of kTrRows rows): every L value is a broadcast shared load,
// every y value one coalesced load and store. The backward pass stops at the
// panel holding row `stop` (rows above it are left unfinished).
constexpr int kTrRows = 64;

__device__ void panel_solve(const double* A, int P, const double* dinv, double* Y, size_t ldy, int c, bool act,
                            int stop) {
  __shared__ double lp[kLb][kLb + 1];      // the panel's diagonal block
  __shared__ double ls[kTrRows][kLb + 1];  // a chunk of the panel's other rows (forward) / columns (backward)
  const int tid = threadIdx.x, nt = blockDim.x;
  double yp[kLb];
  // Forward: y = L^-1 b (L unit lower).
  for (int p0 = 0; p0 < P; p0 += kLb) {
    const int nb = min(kLb, P - p0);
    __syncthreads();
    for (int e = tid; e < nb * nb; e += nt) {
      const int r = e / nb, q = e - r * nb;
      lp[r][q] = q < r ? A[static_cast<size_t>(p0 + r) * P + p0 + q] : 0.0;
    }
    __syncthreads();
    if (act) {
#pragma unroll
      for (int k = 0; k < kLb; ++k) {
        if (k < nb) {
          double v = Y[static_cast<size_t>(p0 + k) * ldy + c];
#pragma unroll
          for (int j = 0; j < k; ++j) v = fma(-lp[k][j], yp[j], v);
          yp[k] = v;
          Y[static_cast<size_t>(p0 + k) * ldy + c] = v;
        }
      }
    }
    for (int r0 = p0 + nb; r0 < P; r0 += kTrRows) {
      const int nr = min(kTrRows, P - r0);
      __syncthreads();
      for (int e = tid; e < nr * nb; e += nt) {
        const int r = e / nb, q = e - r * nb;
        ls[r][q] = A[static_cast<size_t>(r0 + r) * P + p0 + q];
      }
      __syncthreads();
      if (act) {
        for (int r = 0; r < nr; ++r) {
          double* yr = Y + static_cast<size_t>(r0 + r) * ldy + c;
          double v = *yr;
#pragma unroll
          for (int k = 0; k < kLb; ++k)
            if (k < nb) v = fma(-ls[r][k], yp[k], v);
          *yr = v;
        }
      }
    }
  }
  // D^+.
  if (act)
    for (int i = 0; i < P; ++i) Y[static_cast<size_t>(i) * ldy + c] *= dinv[i];
  // Backward: x = L^-T y, panels from the last down to the one holding `stop`.
  const int last = ((P - 1) / kLb) * kLb;
  for (int p0 = last; p0 + kLb > stop; p0 -= kLb) {
    const int nb = min(kLb, P - p0);
    __syncthreads();
    for (int e = tid; e < nb * nb; e += nt) {
      const int r = e / nb, q = e - r * nb;
      lp[r][q] = q < r ? A[static_cast<size_t>(p0 + r) * P + p0 + q] : 0.0;
    }
    __syncthreads();
    if (act) {
#pragma unroll
      for (int kk = kLb - 1; kk >= 0; --kk) {
        if (kk < nb) {
          double v = Y[static_cast<size_t>(p0 + kk) * ldy + c];
#pragma unroll
          for (int t = kk + 1; t < kLb; ++t)
            if (t < nb) v = fma(-lp[t][kk], yp[t], v);
          yp[kk] = v;
          Y[static_cast<size_t>(p0 + kk) * ldy + c] = v;
        }
      }
    }
    // rows r in [stop, p0) above the panel: y_r -= sum_t L[p0 + t][r] x_t
    const int rlo = min(stop, p0);
    for (int r0 = rlo; r0 < p0; r0 += kTrRows) {
      const int nr = min(kTrRows, p0 - r0);
      __syncthreads();
      for (int e = tid; e < nr * nb; e += nt) {
        const int q = e / nr, r = e - q * nr;  // consecutive threads read consecutive columns of row p0 + q
        ls[r][q] = A[static_cast<size_t>(p0 + q) * P + r0 + r];
      }
      __syncthreads();
      if (act) {
        for (int r = 0; r < nr; ++r) {
          double* yr = Y + static_cast<size_t>(r0 + r) * ldy + c;
          double v = *yr;
#pragma unroll
          for (int t = 0; t < kLb; ++t)
            if (t < nb) v = fma(-ls[r][t], yp[t], v);
          *yr = v;
        }
      }
    }
    if (p0 == 0) break;
  }
}

// edf terms Z_cc, Z = L^-T D^+ L^-1 B, B = Pi M Pi^T: thread c solves column c
// (x_c needs x_t, t > c only, so the backward pass stops at the CTA's first
// column). Grid: (chunk systems, ceil(P / kLdltTraceThreads)).
__global__ void __launch_bounds__(kLdltTraceThreads) k_ldlt_trace(SolveBatch b, int s0, LdltWork wk) {
  const int P = b.P;
  const size_t PP = static_cast<size_t>(P) * P;
  const int s = s0 + static_cast<int>(blockIdx.x);
  double* A = wk.d + blockIdx.x * ldlt_sys_doubles(P);
  double* Y = A + PP;
  const double* dinv = A + 2 * PP;
  double* zc = A + 2 * PP + P;
  const int* perm = wk.i + blockIdx.x * (static_cast<size_t>(P) + 1);
  if (!perm[P]) return;  // the same for the whole CTA
  const int c0 = static_cast<int>(blockIdx.y) * kLdltTraceThreads;
  const int c = c0 + static_cast<int>(threadIdx.x);
  const bool act = c < P;
  const double* M = b.M + static_cast<size_t>(b.m_index ? b.m_index[s] : 0) * PP;
  if (act) {
    const int oc = perm[c];
    for (int i = 0; i < P; ++i) Y[static_cast<size_t>(i) * P + c] = M[static_cast<size_t>(perm[i]) * P + oc];
  }
  panel_solve(A, P, dinv, Y, P, c, act, c0);
  if (act) zc[c] = Y[static_cast<size_t>(c) * P + c];
}

// edf = sum_c Z_cc in column order; ok = 2.
__global__ void k_ldlt_finish(SolveBatch b, int s0, LdltWork wk) {
  const int P = b.P;
  const size_t PP = static_cast<size_t>(P) * P;
  const int s = s0 + static_cast<int>(blockIdx.x);
  const int* perm = wk.i + blockIdx.x * (static_cast<size_t>(P) + 1);
  if (threadIdx.x != 0 || !perm[P]) return;
  const double* zc = wk.d + blockIdx.x * ldlt_sys_doubles(P) + 2 * PP + P;
  double e = 0.0;
  for (int c = 0; c < P; ++c) e += zc[c];
  b.edf[s] = e;
  b.ok[s] = 2;
}

// X = A^+ B for A = M + lambda P0: B and X are P x m, row-major, in the
// original order. The same factorisation as the fallback (one CTA), then the
// columns of B by the panel solve (m / kLdltTraceThreads CTAs); used where
// many right-hand sides share one system. Workspace: A (P x P), Y (P x m),
// D^+ (P), the factorisation's panels (2 kLb P), the permutation (P ints).
__global__ void __launch_bounds__(kLdltThreads) k_sym_factor(int P, int kk, const double* __restrict__ M, double lam,
                                                             const double* __restrict__ pen, double* __restrict__ A,
                                                             double* __restrict__ dinv, int* __restrict__ perm) {
  __shared__ LdltShared S;
  double* Wt = dinv + P;  // 2 x kLb x P panel workspace
  const bool any = build_pivoted(A, M, P, kk, lam, pen, S);
  if (any) ldlt_blocked(A, P, Wt, Wt + static_cast<size_t>(kLb) * P);
  ldlt_dinv(A, P, any ? P : 0, dinv);
  for (int i = threadIdx.x; i < P; i += blockDim.x) perm[i] = S.perm[i];
}

__global__ void __launch_bounds__(kLdltTraceThreads) k_sym_solve_cols(int P, const double* __restrict__ A,
                                                                      const double* __restrict__ dinv,
                                                                      const int* __restrict__ perm,
                                                                      const double* __restrict__ B, int m,
                                                                      double* __restrict__ Y, double* __restrict__ X) {
  const int c = static_cast<int>(blockIdx.x) * kLdltTraceThreads + static_cast<int>(threadIdx.x);
  const bool act = c < m;
  if (act)
    for (int i = 0; i < P; ++i) Y[static_cast<size_t>(i) * m + c] = B[static_cast<size_t>(perm[i]) * m + c];
  panel_solve(A, P, dinv, Y, m, c, act, 0);
  if (act)
    for (int i = 0; i < P; ++i) X[static_cast<size_t>(perm[i]) * m + c] = Y[static_cast<size_t>(i) * m + c];
}

void launch_sym_solve_many(Context& c, int P, int k, const double* M, double lam, const double* pen, const double* B,
                           int m, double* X) {
  if (P > kLdltThreads) fail(DGPU_ERR_INVALID, "solve: at most 1024 unknowns are supported");
  const size_t PP = static_cast<size_t>(P) * P, Pm = static_cast<size_t>(P) * m;
  char* work = static_cast<char*>(c.slot(
      kSlotGrad6, sizeof(double) * (PP + Pm + P + 2 * static_cast<size_t>(kLb) * P) + sizeof(int) * P + 16));
  double* A = reinterpret_cast<double*>(work);
  double* Y = A + PP;
  double* dinv = Y + Pm;
  int* perm = reinterpret_cast<int*>(dinv + P + 2 * static_cast<size_t>(kLb) * P);
  k_sym_factor<<<1, kLdltThreads, 0, c.stream>>>(P, k, M, lam, pen, A, dinv, perm);
  DGPU_LAUNCH("k_sym_factor");
  if (m <= 0) return;
  k_sym_solve_cols<<<(m + kLdltTraceThreads - 1) / kLdltTraceThreads, kLdltTraceThreads, 0, c.stream>>>(
      P, A, dinv, perm, B, m, Y, X);
  DGPU_LAUNCH("k_sym_solve_cols");
}

void launch_ldlt_fallback(Context& c, const SolveBatch& b) {
  if (b.nsys <= 0) return;
  if (b.P > kLdltThreads) fail(DGPU_ERR_INVALID, "solve: the LDLT fallback supports at most 1024 unknowns");
  const int chunk = std::min(b.nsys, kLdltChunk);
  char* work = static_cast<char*>(c.slot(kSlotLdlt, ldlt_work_bytes(b.P, chunk)));
  LdltWork wk;
  wk.d = reinterpret_cast<double*>(work);
  wk.i = reinterpret_cast<int*>(work + sizeof(double) * ldlt_sys_doubles(b.P) * chunk);
  for (int s0 = 0; s0 < b.nsys; s0 += chunk) {
    const int m = std::min(chunk, b.nsys - s0);
    k_ldlt_factor<<<m, kLdltThreads, 0, c.stream>>>(b, s0, wk);
    DGPU_LAUNCH("k_ldlt_factor");
    k_ldlt_trace<<<dim3(m, (b.P + kLdltTraceThreads - 1) / kLdltTraceThreads), kLdltTraceThreads, 0, c.stream>>>(
        b, s0, wk);
    DGPU_LAUNCH("k_ldlt_trace");
    k_ldlt_finish<<<m, 32, 0, c.stream>>>(b, s0, wk);
    DGPU_LAUNCH("k_ldlt_finish");
  }
}

}  // namespace dgpu
