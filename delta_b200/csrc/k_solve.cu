// Batched penalised-GLS solver on the device (reference src/solve.cpp:147-193,
// 227-262): for every system s of a batch (the lambda grid, or the lambda x
// fold grid of a CV search)
//   A_s = M_s + lambda_s P0,  A_s = L L^T (FP64 Cholesky),
//   theta_s = L^-T L^-1 rhs_s,  edf_s = P - lambda_s ||L^-1 F||_F^2
// (the reference's exact trace identity, F F^T = P0).
//
// One thread-block cluster per system (systems never wait on each other):
// 32 x 32 FP64 tiles in global memory (L2-resident: a 464-unknown system is
// 1.8 MB), right-looking blocked Cholesky whose phases are separated by
// hardware cluster barriers. Rank 0 of the cluster updates and factors the
// next diagonal tile while the other ranks apply the rest of the trailing
// update (one-tile look-ahead), so each tile column costs two cluster
// barriers. The tile columns of L^-1 are independent and are spread over the
// ranks without further barriers. The trace is reduced per rank and summed in
// rank order (deterministic). A non-positive pivot marks the system failed
// (ok = 0): the reference then falls back to LDLT.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "dev_common.cuh"
#include "fit_internal.h"

namespace cg = cooperative_groups;

namespace dgpu {

constexpr int kT = 32;  // tile side
constexpr int kSolveThreads = 256;

int solve_pp(int P) { return (P + kT - 1) / kT * kT; }

struct Tiles {
  double a[kT][kT + 1];
  double b[kT][kT + 1];
  double c[kT][kT + 1];
  double v[1024];
  double red[kSolveThreads];
};

__device__ __forceinline__ double* tile_ptr(double* base, int Pp, int ti, int tj) {
  return base + static_cast<size_t>(ti) * kT * Pp + static_cast<size_t>(tj) * kT;
}

__device__ __forceinline__ void load_tile(double (*t)[kT + 1], const double* g, int Pp) {
  for (int e = threadIdx.x; e < kT * kT; e += blockDim.x) t[e / kT][e % kT] = g[static_cast<size_t>(e / kT) * Pp + e % kT];
}
__device__ __forceinline__ void load_tile_t(double (*t)[kT + 1], const double* g, int Pp) {
  for (int e = threadIdx.x; e < kT * kT; e += blockDim.x) t[e % kT][e / kT] = g[static_cast<size_t>(e / kT) * Pp + e % kT];
}
__device__ __forceinline__ void store_tile(double* g, double (*t)[kT + 1], int Pp) {
  for (int e = threadIdx.x; e < kT * kT; e += blockDim.x) g[static_cast<size_t>(e / kT) * Pp + e % kT] = t[e / kT][e % kT];
}

// acc += A B^T over the 32-wide inner dimension with FP64 tensor-core MMAs
// (mma.sync m8n8k4, f64): the 32 x 32 output is 4 x 4 blocks of 8 x 8; warp w
// owns row block w / 2 and column blocks 2 (w % 2) and 2 (w % 2) + 1, two
// accumulators of two doubles per thread (D fragment: row lane / 4, columns
// 2 (lane % 4) + {0, 1}). A fragment: A[row lane / 4][k + lane % 4];
// B fragment (B^T column-major): B[col lane / 4][k + lane % 4].
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void mma_nt(double (*A)[kT + 1], double (*B)[kT + 1], double acc[2][2]) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ra = (warp >> 1) * 8 + (lane >> 2);
  const int cb0 = (warp & 1) * 16 + (lane >> 2);
  const int kq = lane & 3;
#pragma unroll
  for (int k0 = 0; k0 < kT; k0 += 4) {
    const double a = A[ra][k0 + kq];
    const double b0 = B[cb0][k0 + kq];
    const double b1 = B[cb0 + 8][k0 + kq];
    dmma_8x8x4(acc[0], a, b0);
    dmma_8x8x4(acc[1], a, b1);
  }
}

__device__ __forceinline__ void acc_to_tile(double (*C)[kT + 1], const double acc[2][2], double scale, bool add) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = (warp >> 1) * 8 + (lane >> 2);
#pragma unroll
  for (int blk = 0; blk < 2; ++blk) {
    const int c0 = (warp & 1) * 16 + blk * 8 + (lane & 3) * 2;
#pragma unroll
    for (int i = 0; i < 2; ++i) C[r][c0 + i] = (add ? C[r][c0 + i] : 0.0) + scale * acc[blk][i];
  }
}

// Global writes of this CTA become visible to the cluster, then all ranks meet.
__device__ __forceinline__ void cluster_step(const cg::cluster_group& cl) {
  __threadfence();
  cl.sync();
}

// Factor the diagonal tile held in T.a (lower part used; upper zeroed on
// store) and put its inverse in T.b; stores both tiles. A non-positive pivot
// clears *ok and continues with pivot 1.
__device__ void factor_diag(Tiles& T, double* A, double* Li, int Pp, int j, int* ok) {
  for (int q = 0; q < kT; ++q) {
    if (threadIdx.x == 0) {
      double d = T.a[q][q];
      if (!(d > 0.0)) {
        *ok = 0;
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
  for (int e = threadIdx.x; e < kT * kT; e += blockDim.x)
    if (e % kT > e / kT) T.a[e / kT][e % kT] = 0.0;
  __syncthreads();
  store_tile(tile_ptr(A, Pp, j, j), T.a, Pp);
  store_tile(tile_ptr(Li, Pp, j, j), T.b, Pp);
  __syncthreads();
}

// A_im -= L_ij L_mj^T; the updated tile stays in T.c and is stored.
__device__ void trailing_tile(Tiles& T, double* A, int Pp, int i, int m, int j) {
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

__global__ void __launch_bounds__(kSolveThreads) k_solve_cluster(SolveBatch b, int Pp) {
  extern __shared__ __align__(16) unsigned char raw[];
  Tiles& T = *reinterpret_cast<Tiles*>(raw);
  const cg::cluster_group cl = cg::this_cluster();
  const int cn = static_cast<int>(cl.num_blocks());
  const int rank = static_cast<int>(cl.block_rank());
  const int s = blockIdx.x / cn;
  const int P = b.P, k = b.k, nb = Pp / kT;
  const size_t mat = static_cast<size_t>(Pp) * Pp;
  double* A = b.A + static_cast<size_t>(s) * mat;
  double* Li = b.Linv + static_cast<size_t>(s) * mat;
  const double* M = b.M + (b.m_index ? static_cast<size_t>(b.m_index[s]) * P * P : 0);
  const double lam = b.lam[s];
  __shared__ int s_ok;
  if (threadIdx.x == 0) s_ok = 1;

  // A = M + lambda P0 on the lower tiles through the diagonal tile (identity
  // padding), rows spread over the ranks.
  for (int i = rank; i < Pp; i += cn) {
    const int jmax = (i / kT) * kT + kT;
    for (int j = threadIdx.x; j < jmax; j += blockDim.x) {
      double v;
      if (i < P && j < P) {
        v = M[static_cast<size_t>(i) * P + j];
        if (i / k == j / k) v += lam * b.pen[(i % k) * k + (j % k)];
      } else {
        v = (i == j) ? 1.0 : 0.0;
      }
      A[static_cast<size_t>(i) * Pp + j] = v;
    }
  }
  cluster_step(cl);
  if (rank == 0) {
    load_tile(T.a, tile_ptr(A, Pp, 0, 0), Pp);
    __syncthreads();
    factor_diag(T, A, Li, Pp, 0, &s_ok);
  }
  cluster_step(cl);

  for (int j = 0; j + 1 < nb; ++j) {
    const int below = nb - j - 1;
    // Panel: L_ij = A_ij Linv_jj^T for i > j, over all ranks.
    for (int t = rank; t < below; t += cn) {
      const int i = j + 1 + t;
      load_tile(T.a, tile_ptr(A, Pp, i, j), Pp);
      load_tile(T.b, tile_ptr(Li, Pp, j, j), Pp);
      __syncthreads();
      double acc[2][2] = {{0, 0}, {0, 0}};
      mma_nt(T.a, T.b, acc);
      __syncthreads();
      acc_to_tile(T.c, acc, 1.0, false);
      __syncthreads();
      store_tile(tile_ptr(A, Pp, i, j), T.c, Pp);
      __syncthreads();
    }
    cluster_step(cl);
    // Trailing update A_im -= L_ij L_mj^T, j < m <= i. Tile index 0 is the next
    // diagonal tile: rank 0 updates and factors it while the other ranks share
    // the remaining tiles.
    if (rank == 0) {
      trailing_tile(T, A, Pp, j + 1, j + 1, j);
      for (int e = threadIdx.x; e < kT * kT; e += blockDim.x) T.a[e / kT][e % kT] = T.c[e / kT][e % kT];
      __syncthreads();
      factor_diag(T, A, Li, Pp, j + 1, &s_ok);
    }
    const int ntile = below * (below + 1) / 2;
    const int workers = cn > 1 ? cn - 1 : 1;
    const int wrank = cn > 1 ? rank - 1 : 0;
    if (cn == 1 || rank > 0) {
      for (int t = 1 + wrank; t < ntile; t += workers) {
        int tt = t, ii = 0;
        while (tt > ii) {
          tt -= ii + 1;
          ++ii;
        }
        trailing_tile(T, A, Pp, j + 1 + ii, j + 1 + tt, j);
      }
    }
    cluster_step(cl);
  }

  // Off-diagonal tiles of L^-1, column by column (columns are independent):
  // Linv_ij = -Linv_ii sum_{q=j}^{i-1} L_iq Linv_qj. Columns are dealt in a
  // snake order so the long early columns spread over the ranks.
  for (int j = 0; j + 1 < nb; ++j) {
    const int lane = j % (2 * cn);
    const int owner = lane < cn ? lane : 2 * cn - 1 - lane;
    if (owner != rank) continue;
    for (int i = j + 1; i < nb; ++i) {
      double acc[2][2] = {{0, 0}, {0, 0}};
      for (int q = j; q < i; ++q) {
        load_tile(T.a, tile_ptr(A, Pp, i, q), Pp);
        load_tile_t(T.b, tile_ptr(Li, Pp, q, j), Pp);
        __syncthreads();
        mma_nt(T.a, T.b, acc);
        __syncthreads();
      }
      acc_to_tile(T.c, acc, 1.0, false);  // S = sum L_iq Linv_qj
      load_tile(T.a, tile_ptr(Li, Pp, i, i), Pp);
      __syncthreads();
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
  }
  cluster_step(cl);

  // ||L^-1 F||^2 with F = blockdiag(fk): rows p spread over the ranks; block
  // bb touches columns bb*k .. bb*k + k - 1, of which only those <= p are non-zero.
  double part = 0.0;
  for (int e = rank * blockDim.x + threadIdx.x; e < b.nf * P; e += cn * blockDim.x) {
    const int bb = e / P, p = e - bb * P;
    if (p < bb * k) continue;
    const double* lrow = Li + static_cast<size_t>(p) * Pp + bb * k;
    const int mmax = min(k, p - bb * k + 1);
    for (int jj = 0; jj < b.r; ++jj) {
      double z = 0.0;
      for (int m = 0; m < mmax; ++m) z = fma(lrow[m], b.fk[m * b.r + jj], z);
      part = fma(z, z, part);
    }
  }
  T.red[threadIdx.x] = part;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < static_cast<unsigned>(o)) T.red[threadIdx.x] += T.red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) b.partial[static_cast<size_t>(s) * cn + rank] = T.red[0];
  cluster_step(cl);
  if (rank != 0) return;
  if (threadIdx.x == 0) {
    double tr = 0.0;
    for (int q = 0; q < cn; ++q) tr += b.partial[static_cast<size_t>(s) * cn + q];
    b.edf[s] = static_cast<double>(P) - lam * tr;
    b.ok[s] = s_ok;
  }
  // theta = Linv^T (Linv rhs): y by warp-per-row dot products, then by columns.
  const double* rhs = b.rhs + (b.r_index ? static_cast<size_t>(b.r_index[s]) * P : 0);
  const int warp = threadIdx.x / 32, ln = threadIdx.x % 32, nw = blockDim.x / 32;
  for (int p = warp; p < P; p += nw) {
    const double* row = Li + static_cast<size_t>(p) * Pp;
    double y = 0.0;
    for (int q = ln; q <= p; q += 32) y = fma(row[q], rhs[q], y);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) y += __shfl_down_sync(0xffffffffu, y, o);
    if (ln == 0) T.v[p] = y;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < P; q += blockDim.x) {
    double th = 0.0;
    for (int p = q; p < P; ++p) th = fma(Li[static_cast<size_t>(p) * Pp + q], T.v[p], th);
    b.theta[static_cast<size_t>(s) * P + q] = th;
  }
}

int solve_cluster_size(int nsys) {
  // About two CTAs per SM over the batch, at most the portable cluster size 8.
  const int want = std::min(8, std::max(1, (148 * 2) / std::max(nsys, 1)));
  int cn = 1;
  while (cn * 2 <= want) cn *= 2;
  return cn;
}

void launch_solve_batch(Context& c, const SolveBatch& b) {
  const int Pp = solve_pp(b.P);
  if (b.P > 1024) fail(DGPU_ERR_INVALID, "solve: more than 1024 unknowns is not supported");
  if (b.nsys <= 0) return;
  const int cn = solve_cluster_size(b.nsys);
  const size_t smem = sizeof(Tiles);
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_solve_cluster), smem);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(static_cast<unsigned>(b.nsys * cn));
  cfg.blockDim = dim3(kSolveThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = static_cast<unsigned>(cn);
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  SolveBatch bb = b;
  DGPU_CUDA(cudaLaunchKernelEx(&cfg, k_solve_cluster, bb, Pp));
  DGPU_LAUNCH("k_solve_cluster");
}

// out = A_s^{-1} v = Linv_s^T (Linv_s v), single CTA: y by warp-per-row dot
// products; then every warp adds y_p Linv[p][:] over its rows p into its own
// shared-memory accumulator (lanes over columns, coalesced), and the warps'
// accumulators are summed in warp order.
constexpr int kAiThreads = 512;

__global__ void __launch_bounds__(kAiThreads) k_apply_inverse(const double* __restrict__ Li, int P, int Pp,
                                                               const double* __restrict__ v,
                                                               double* __restrict__ out) {
  extern __shared__ double aism[];
  double* y = aism;              // P
  double* accw = aism + P;       // nw x P
  const int warp = threadIdx.x / 32, ln = threadIdx.x % 32, nw = blockDim.x / 32;
  for (int p = warp; p < P; p += nw) {
    const double* row = Li + static_cast<size_t>(p) * Pp;
    double a = 0.0;
    for (int q = ln; q <= p; q += 32) a = fma(row[q], v[q], a);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if (ln == 0) y[p] = a;
  }
  for (int i = threadIdx.x; i < nw * P; i += blockDim.x) accw[i] = 0.0;
  __syncthreads();
  double* mine = accw + static_cast<size_t>(warp) * P;
  for (int p = warp; p < P; p += nw) {
    const double* row = Li + static_cast<size_t>(p) * Pp;
    const double yp = y[p];
    for (int q = ln; q <= p; q += 32) mine[q] = fma(row[q], yp, mine[q]);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < P; q += blockDim.x) {
    double a = 0.0;
    for (int w2 = 0; w2 < nw; ++w2) a += accw[static_cast<size_t>(w2) * P + q];
    out[q] = a;
  }
}

void launch_apply_inverse(cudaStream_t st, const SolveBatch& b, int s, const double* v, double* out) {
  const int Pp = solve_pp(b.P);
  const size_t smem = sizeof(double) * static_cast<size_t>(b.P) * (1 + kAiThreads / 32);
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_apply_inverse), smem);
  k_apply_inverse<<<1, kAiThreads, smem, st>>>(b.Linv + static_cast<size_t>(s) * Pp * Pp, b.P, Pp, v, out);
  DGPU_LAUNCH("k_apply_inverse");
}

}  // namespace dgpu
