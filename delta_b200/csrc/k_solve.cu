// Batched penalised-GLS solver on the device (reference src/solve.cpp:147-193,
// 227-262): for every system s of a batch (the lambda grid, or the lambda x
// fold grid of a CV search)
//   A_s = M_s + lambda_s P0,  A_s = L L^T (FP64 Cholesky),
//   theta_s = L^-T L^-1 rhs_s,  edf_s = P - lambda_s ||L^-1 F||_F^2
// (the reference's exact trace identity, F F^T = P0).
//
// One cooperative launch sweeps all systems at once: 32 x 32 FP64 tiles,
// right-looking Cholesky (diagonal factor + inverse, panel solve by the
// diagonal inverse, trailing update), then the off-diagonal tiles of L^-1
// column by column, then per-system solves and traces. Work items of each
// phase are spread over every CTA of the grid; phases are separated by a grid
// barrier whose spin is bounded (a stalled barrier sets the status word and
// returns instead of hanging). A non-positive pivot marks the system failed
// (ok = 0): the reference then falls back to LDLT.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "dev_common.cuh"
#include "fit_internal.h"

namespace dgpu {

constexpr int kT = 32;  // tile side
constexpr long long kBarrierSpinCap = 1ll << 24;

int solve_pp(int P) { return (P + kT - 1) / kT * kT; }

__device__ void grid_barrier(unsigned* bar, unsigned* status) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = bar + 1;
    const unsigned g = *gen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u);
    if (arrived == gridDim.x - 1) {
      bar[0] = 0u;
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long long it = 0;
      while (*gen == g) {
        if (++it > kBarrierSpinCap) {
          atomicOr(status, kStatusLoopLimit);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

struct Tiles {
  double a[kT][kT + 1];
  double b[kT][kT + 1];
  double c[kT][kT + 1];
  double v[1024];
  double red[256];
};

__device__ __forceinline__ double* tile_ptr(double* base, int Pp, int ti, int tj) {
  return base + static_cast<size_t>(ti) * kT * Pp + static_cast<size_t>(tj) * kT;
}

__device__ void load_tile(double (*t)[kT + 1], const double* g, int Pp) {
  for (int e = threadIdx.x; e < kT * kT; e += blockDim.x) t[e / kT][e % kT] = g[static_cast<size_t>(e / kT) * Pp + e % kT];
}
__device__ void store_tile(double* g, double (*t)[kT + 1], int Pp) {
  for (int e = threadIdx.x; e < kT * kT; e += blockDim.x) g[static_cast<size_t>(e / kT) * Pp + e % kT] = t[e / kT][e % kT];
}

// acc(2x2 per thread) += A B^T over the 32-wide inner dimension.
__device__ __forceinline__ void mma_nt(double (*A)[kT + 1], double (*B)[kT + 1], double acc[2][2]) {
  const int ra = (threadIdx.x / 16) * 2, rb = (threadIdx.x % 16) * 2;
#pragma unroll 8
  for (int q = 0; q < kT; ++q) {
    const double a0 = A[ra][q], a1 = A[ra + 1][q];
    const double b0 = B[rb][q], b1 = B[rb + 1][q];
    acc[0][0] = fma(a0, b0, acc[0][0]);
    acc[0][1] = fma(a0, b1, acc[0][1]);
    acc[1][0] = fma(a1, b0, acc[1][0]);
    acc[1][1] = fma(a1, b1, acc[1][1]);
  }
}

__device__ __forceinline__ void acc_to_tile(double (*C)[kT + 1], double acc[2][2], double scale, bool add) {
  const int ra = (threadIdx.x / 16) * 2, rb = (threadIdx.x % 16) * 2;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) C[ra + i][rb + j] = (add ? C[ra + i][rb + j] : 0.0) + scale * acc[i][j];
}

__global__ void __launch_bounds__(256) k_solve_batch(SolveBatch b, int Pp) {
  extern __shared__ __align__(16) unsigned char raw[];
  Tiles& T = *reinterpret_cast<Tiles*>(raw);
  const int P = b.P, k = b.k, nb = Pp / kT;
  const size_t mat = static_cast<size_t>(Pp) * Pp;

  // Phase 0: A_s = M + lambda P0 (lower tiles, identity padding); clear Linv.
  {
    const size_t total = static_cast<size_t>(b.nsys) * mat;
    for (size_t e = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
         e += static_cast<size_t>(gridDim.x) * blockDim.x) {
      const int s = static_cast<int>(e / mat);
      const size_t o = e - static_cast<size_t>(s) * mat;
      const int i = static_cast<int>(o / Pp), j = static_cast<int>(o % Pp);
      double v;
      if (i < P && j < P) {
        const double* M = b.M + (b.m_index ? static_cast<size_t>(b.m_index[s]) * P * P : 0);
        v = M[static_cast<size_t>(i) * P + j];
        if (i / k == j / k) v += b.lam[s] * b.pen[(i % k) * k + (j % k)];
      } else {
        v = (i == j) ? 1.0 : 0.0;
      }
      b.A[e] = v;
      b.Linv[e] = 0.0;
    }
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < b.nsys; s += gridDim.x * blockDim.x) b.ok[s] = 1;
  }
  grid_barrier(b.barrier, b.status);

  for (int j = 0; j < nb; ++j) {
    // (a) factor the diagonal tile and invert it.
    for (int s = blockIdx.x; s < b.nsys; s += gridDim.x) {
      double* A = b.A + static_cast<size_t>(s) * mat;
      double* Li = b.Linv + static_cast<size_t>(s) * mat;
      load_tile(T.a, tile_ptr(A, Pp, j, j), Pp);
      __syncthreads();
      for (int q = 0; q < kT; ++q) {
        if (threadIdx.x == 0) {
          double d = T.a[q][q];
          if (!(d > 0.0)) {
            b.ok[s] = 0;
            d = 1.0;
          }
          T.a[q][q] = sqrt(d);
        }
        __syncthreads();
        if (threadIdx.x > q && threadIdx.x < kT) T.a[threadIdx.x][q] /= T.a[q][q];
        __syncthreads();
        for (int e = threadIdx.x; e < kT * kT; e += blockDim.x) {
          const int r = e / kT, m = e % kT;
          if (r > q && m > q && m <= r) T.a[r][m] -= T.a[r][q] * T.a[m][q];
        }
        __syncthreads();
      }
      if (threadIdx.x < kT) {
        const int col = threadIdx.x;
        for (int r = 0; r < kT; ++r) {
          if (r < col) {
            T.b[r][col] = 0.0;
            continue;
          }
          double sum = (r == col) ? 1.0 : 0.0;
          for (int m = col; m < r; ++m) sum -= T.a[r][m] * T.b[m][col];
          T.b[r][col] = sum / T.a[r][r];
        }
      }
      __syncthreads();
      // zero the strict upper triangle of the stored diagonal factor
      for (int e = threadIdx.x; e < kT * kT; e += blockDim.x)
        if (e % kT > e / kT) T.a[e / kT][e % kT] = 0.0;
      __syncthreads();
      store_tile(tile_ptr(A, Pp, j, j), T.a, Pp);
      store_tile(tile_ptr(Li, Pp, j, j), T.b, Pp);
      __syncthreads();
    }
    grid_barrier(b.barrier, b.status);
    const int below = nb - j - 1;
    if (below > 0) {
      // (b) panel: L_ij = A_ij Linv_jj^T.
      for (int task = blockIdx.x; task < b.nsys * below; task += gridDim.x) {
        const int s = task / below, i = j + 1 + task % below;
        double* A = b.A + static_cast<size_t>(s) * mat;
        const double* Li = b.Linv + static_cast<size_t>(s) * mat;
        load_tile(T.a, tile_ptr(A, Pp, i, j), Pp);
        load_tile(T.b, const_cast<double*>(tile_ptr(const_cast<double*>(Li), Pp, j, j)), Pp);
        __syncthreads();
        double acc[2][2] = {{0, 0}, {0, 0}};
        mma_nt(T.a, T.b, acc);
        __syncthreads();
        acc_to_tile(T.c, acc, 1.0, false);
        __syncthreads();
        store_tile(tile_ptr(A, Pp, i, j), T.c, Pp);
        __syncthreads();
      }
      grid_barrier(b.barrier, b.status);
      // (c) trailing update: A_im -= L_ij L_mj^T for j < m <= i.
      const int ntile = below * (below + 1) / 2;
      for (int task = blockIdx.x; task < b.nsys * ntile; task += gridDim.x) {
        const int s = task / ntile;
        int t = task % ntile;
        int ii = 0;
        while (t > ii) {
          t -= ii + 1;
          ++ii;
        }
        const int i = j + 1 + ii, m = j + 1 + t;
        double* A = b.A + static_cast<size_t>(s) * mat;
        load_tile(T.a, tile_ptr(A, Pp, i, j), Pp);
        load_tile(T.b, tile_ptr(A, Pp, m, j), Pp);
        load_tile(T.c, tile_ptr(A, Pp, i, m), Pp);
        __syncthreads();
        double acc[2][2] = {{0, 0}, {0, 0}};
        mma_nt(T.a, T.b, acc);
        acc_to_tile(T.c, acc, -1.0, true);
        __syncthreads();
        store_tile(tile_ptr(A, Pp, i, m), T.c, Pp);
        __syncthreads();
      }
      grid_barrier(b.barrier, b.status);
    }
  }

  // Off-diagonal tiles of L^-1: Linv_ij = -Linv_ii sum_{q=j}^{i-1} L_iq Linv_qj.
  for (int st = 1; st < nb; ++st) {
    const int ncol = nb - st;
    for (int task = blockIdx.x; task < b.nsys * ncol; task += gridDim.x) {
      const int s = task / ncol, j = task % ncol, i = j + st;
      const double* A = b.A + static_cast<size_t>(s) * mat;
      double* Li = b.Linv + static_cast<size_t>(s) * mat;
      double acc[2][2] = {{0, 0}, {0, 0}};
      for (int q = j; q < i; ++q) {
        load_tile(T.a, const_cast<double*>(tile_ptr(const_cast<double*>(A), Pp, i, q)), Pp);
        // B^T layout: need (Linv_qj)^T rows -> load transposed.
        const double* lq = tile_ptr(Li, Pp, q, j);
        for (int e = threadIdx.x; e < kT * kT; e += blockDim.x)
          T.b[e % kT][e / kT] = lq[static_cast<size_t>(e / kT) * Pp + e % kT];
        __syncthreads();
        mma_nt(T.a, T.b, acc);
        __syncthreads();
      }
      acc_to_tile(T.c, acc, 1.0, false);  // S = sum L_iq Linv_qj
      load_tile(T.a, tile_ptr(Li, Pp, i, i), Pp);
      __syncthreads();
      // Linv_ij = -Linv_ii S  (A = Linv_ii, B^T = S -> transpose S into T.b)
      for (int e = threadIdx.x; e < kT * kT; e += blockDim.x) T.b[e % kT][e / kT] = T.c[e / kT][e % kT];
      __syncthreads();
      double acc2[2][2] = {{0, 0}, {0, 0}};
      mma_nt(T.a, T.b, acc2);
      __syncthreads();
      acc_to_tile(T.c, acc2, -1.0, false);
      __syncthreads();
      store_tile(tile_ptr(Li, Pp, i, j), T.c, Pp);
      __syncthreads();
    }
    grid_barrier(b.barrier, b.status);
  }

  // Per-system theta and trace.
  for (int s = blockIdx.x; s < b.nsys; s += gridDim.x) {
    const double* Li = b.Linv + static_cast<size_t>(s) * mat;
    const double* rhs = b.rhs + (b.r_index ? static_cast<size_t>(b.r_index[s]) * P : 0);
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
      double y = 0.0;
      for (int q = 0; q <= p; ++q) y = fma(Li[static_cast<size_t>(p) * Pp + q], rhs[q], y);
      T.v[p] = y;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < P; q += blockDim.x) {
      double th = 0.0;
      for (int p = q; p < P; ++p) th = fma(Li[static_cast<size_t>(p) * Pp + q], T.v[p], th);
      b.theta[static_cast<size_t>(s) * P + q] = th;
    }
    // ||L^-1 F||^2 with F = blockdiag(fk): block bb touches columns bb*k..bb*k+k-1.
    double part = 0.0;
    const int nrow_tot = b.nf * P;
    for (int e = threadIdx.x; e < nrow_tot; e += blockDim.x) {
      const int bb = e / P, p = e - bb * P;
      if (p < bb * k) continue;
      const double* lrow = Li + static_cast<size_t>(p) * Pp + bb * k;
      for (int jj = 0; jj < b.r; ++jj) {
        double z = 0.0;
        for (int m = 0; m < k; ++m) z = fma(lrow[m], b.fk[m * b.r + jj], z);
        part = fma(z, z, part);
      }
    }
    T.red[threadIdx.x] = part;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if (threadIdx.x < static_cast<unsigned>(o)) T.red[threadIdx.x] += T.red[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) b.edf[s] = static_cast<double>(P) - b.lam[s] * T.red[0];
    __syncthreads();
  }
}

void launch_solve_batch(Context& c, const SolveBatch& b) {
  const int Pp = solve_pp(b.P);
  if (b.P > 1024) fail(DGPU_ERR_INVALID, "solve: more than 1024 unknowns is not supported");
  const size_t smem = sizeof(Tiles);
  DGPU_CUDA(cudaFuncSetAttribute(k_solve_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  int per_sm = 0;
  DGPU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve_batch, 256, smem));
  int sms = 0;
  DGPU_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device));
  const int nb = Pp / kT;
  const int max_tasks = std::max(b.nsys * nb * (nb + 1) / 2, b.nsys);
  const int grid = std::max(1, std::min(per_sm * sms, max_tasks));
  DGPU_CUDA(cudaMemsetAsync(b.barrier, 0, 2 * sizeof(unsigned), c.stream));
  SolveBatch bb = b;
  int ppv = Pp;
  void* args[] = {&bb, &ppv};
  DGPU_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_solve_batch), dim3(grid), dim3(256), args, smem,
                                        c.stream));
  count_launch();
}

// out = A_s^{-1} v = Linv_s^T (Linv_s v), single CTA.
__global__ void k_apply_inverse(const double* __restrict__ Li, int P, int Pp, const double* __restrict__ v,
                                double* __restrict__ out) {
  __shared__ double y[1024];
  for (int p = threadIdx.x; p < P; p += blockDim.x) {
    double a = 0.0;
    for (int q = 0; q <= p; ++q) a = fma(Li[static_cast<size_t>(p) * Pp + q], v[q], a);
    y[p] = a;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < P; q += blockDim.x) {
    double a = 0.0;
    for (int p = q; p < P; ++p) a = fma(Li[static_cast<size_t>(p) * Pp + q], y[p], a);
    out[q] = a;
  }
}

void launch_apply_inverse(cudaStream_t st, const SolveBatch& b, int s, const double* v, double* out) {
  const int Pp = solve_pp(b.P);
  k_apply_inverse<<<1, 512, 0, st>>>(b.Linv + static_cast<size_t>(s) * Pp * Pp, b.P, Pp, v, out);
  DGPU_LAUNCH("k_apply_inverse");
}

}  // namespace dgpu
