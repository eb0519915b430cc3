// Batched penalised-GLS solver on the device (reference src/solve.cpp:147-193,
// 227-262): for every system s of a batch (the lambda grid, or the lambda x
// fold grid of a CV search)
//   A_s = M_s + lambda_s P0,  A_s = L L^T (FP64 Cholesky),
//   theta_s = L^-T L^-1 rhs_s,  edf_s = P - lambda_s ||L^-1 F||_F^2
// (the reference's exact trace identity, F F^T = P0).
//
// One thread-block cluster per system (systems never wait on each other).
// The matrix lives in global memory (L2-resident) as 32 x 32 FP64 tiles and
// is factored by a right-looking blocked Cholesky whose phases are separated
// by hardware cluster barriers. Below A the rows E = [rhs^T; F^T] are
// appended: the same panel steps that turn A's column tiles into L turn E
// into E L^-T = [(L^-1 rhs)^T; (L^-1 F)^T], so y = L^-1 rhs and the trace
// come out of the factorisation with no inverse of L. E's F rows are zero
// left of their field block, and tiles left of that never enter the
// computation. Per tile column j:
//   panel     L_ij = A_ij Dinv_j^T for the tiles below the diagonal and the
//             active E tiles (Dinv_j = L_jj^-1), all ranks;
//   trailing  A_im -= L_ij L_mj^T, E_cm -= X_cj L_mj^T; rank 0 first updates
//             and factors the next diagonal tile (one-tile look-ahead, one
//             warp, LDL^T with the tile's rows in registers) and then takes a
//             reduced share of the remaining tiles.
// Tile operands are staged with double-buffered cp.async copies, products on
// the FP64 tensor cores (mma.sync m8n8k4). A is never assembled: M + lambda
// P0 is read at a tile's first touch, and E is generated at its first touch. theta = L^-T y by back
// substitution on rank 0. The trace is reduced per rank in a fixed order and
// summed in rank order (deterministic). A non-positive pivot marks the system
// failed (ok = 0): the reference then falls back to LDLT.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "dev_common.cuh"
#include "fit_internal.h"

namespace cg = cooperative_groups;

namespace dgpu {

constexpr int kT = 32;    // tile side
constexpr int kLd = 36;   // shared tile row stride (doubles): 16-byte rows, conflict-free fragments
constexpr int kTS = kT * kLd;
constexpr int kSolveThreads = 256;
constexpr int kRank0Debt = 3;  // trailing tiles rank 0 skips for its diagonal factorisation

int solve_pp(int P) { return (P + kT - 1) / kT * kT; }
int solve_ep(int nf, int r) { return (nf * r + 1 + kT - 1) / kT * kT; }
size_t solve_sys_doubles(int P, int nf, int r) {
  const size_t Pp = solve_pp(P);
  return Pp * Pp + static_cast<size_t>(solve_ep(nf, r)) * Pp + Pp * kT;
}

struct SolveSmem {
  double op[2][3][kTS];  // double-buffered job operands: C (updated), left, right
  double d[kTS];         // Dinv_j in the panel phase; the diagonal tile in the trailing phase
  double v[1024];        // y / theta in the back substitution
  double red[kSolveThreads];
};

__device__ __forceinline__ void cp16(void* sdst, const void* gsrc) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// 32 x 32 tile (row stride ld doubles, 16-byte aligned rows) into a kLd-strided
// shared tile: 512 16-byte chunks.
__device__ __forceinline__ void tile_async(double* s, const double* g, int ld) {
  for (int q = threadIdx.x; q < kT * kT / 2; q += blockDim.x) {
    const int r = q >> 4, c = (q & 15) * 2;
    cp16(s + r * kLd + c, g + static_cast<size_t>(r) * ld + c);
  }
}

__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// acc += A B^T over the 32-wide inner dimension (shared tiles, stride kLd).
// The 32 x 32 output is 4 x 4 blocks of 8 x 8; warp w owns row block w / 2
// and column blocks 2 (w % 2), 2 (w % 2) + 1. A fragment: A[row lane / 4][k +
// lane % 4]; B fragment: B[col lane / 4][k + lane % 4]; D fragment: row lane /
// 4, columns 2 (lane % 4) + {0, 1}.
__device__ __forceinline__ void mma_nt(const double* A, const double* B, double (&acc)[2][2]) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ra = (warp >> 1) * 8 + (lane >> 2);
  const int cb0 = (warp & 1) * 16 + (lane >> 2);
  const int kq = lane & 3;
#pragma unroll
  for (int k0 = 0; k0 < kT; k0 += 4) {
    const double a = A[ra * kLd + k0 + kq];
    const double b0 = B[cb0 * kLd + k0 + kq];
    const double b1 = B[(cb0 + 8) * kLd + k0 + kq];
    dmma_8x8x4(acc[0], a, b0);
    dmma_8x8x4(acc[1], a, b1);
  }
}
__device__ __forceinline__ int frag_row() { return ((threadIdx.x >> 5) >> 1) * 8 + ((threadIdx.x & 31) >> 2); }
__device__ __forceinline__ int frag_col(int blk) {
  return ((threadIdx.x >> 5) & 1) * 16 + blk * 8 + (threadIdx.x & 3) * 2;
}

// Global writes of this CTA become visible to the cluster, then all ranks meet.
__device__ __forceinline__ void cluster_step(const cg::cluster_group& cl) {
  __threadfence();
  cl.sync();
}

// Run this rank's jobs first, next(first), ... (< nt) with the operands of the
// next job in flight while the current one computes. load(buf, t) issues the
// copies of job t into the three tiles of buf; compute(buf, t) uses them.
template <class Next, class Load, class Compute>
__device__ __forceinline__ void run_jobs(SolveSmem& S, int first, int nt, Next next, Load load, Compute compute) {
  if (first >= nt) return;
  int cur = 0;
  load(S.op[0], first);
  cp_commit();
  for (int t = first; t < nt;) {
    const int tn = next(t);
    if (tn < nt) load(S.op[cur ^ 1], tn);
    cp_commit();
    cp_wait1();
    __syncthreads();
    compute(S.op[cur], t);
    __syncthreads();
    cur ^= 1;
    t = tn;
  }
}

// Right-looking LDL^T of N columns held in registers, lane = row: the pivot
// of column q is on lane base + q. Afterwards a[q] holds the unit factor
// l_rq below the pivot, the pivot d_q on it and zero above. One reciprocal
// per column is the only long-latency step of the chain.
template <int N>
__device__ __forceinline__ void ldl_cols(double (&a)[N], int lane, int base, int& bad) {
#pragma unroll
  for (int q = 0; q < N; ++q) {
    double d = __shfl_sync(0xffffffffu, a[q], base + q);
    if (!(d > 0.0)) {
      bad = 1;
      d = 1.0;
    }
    const double u = a[q];
    const double l = u * __drcp_rn(d);
#pragma unroll
    for (int m = q + 1; m < N; ++m) {
      const double um = __shfl_sync(0xffffffffu, u, base + m);
      if (lane >= base + m) a[m] = fma(-l, um, a[m]);
    }
    a[q] = lane > base + q ? l : (lane == base + q ? d : 0.0);
  }
}

// Factor the symmetric tile in S.d (lower part used): L_jj into the A tile
// gL (upper zeroed) and Dinv_j = L_jj^-1 into gD (row stride kT). One warp,
// lane = row: LDL^T in two 16-column halves (columns 0-15 of all rows, the
// Schur complement of the lower-right block, its factorisation), then
// L = Lu D^1/2 and L^-1 = D^-1/2 Lu^-1, lane c forming column c of Lu^-1 by
// blocks: x = Lu11^-1 e_c, z = Lu22^-1 (e_c - Lu21 x). A non-positive pivot
// clears *ok and continues with pivot 1.
constexpr int kFs = kT + 1;
constexpr int kH = kT / 2;
__device__ __noinline__ void factor_tile(SolveSmem& S, double* gL, int ldL, double* gD, int* ok) {
  double* f = S.op[0][2];         // 32 x kFs: Lu below the diagonal, D on it
  double* xs = S.op[1][0];        // 32 x kFs: Lu^-1
  double* sd = S.op[1][1];        // sqrt(D)
  double* isd = S.op[1][1] + kT;  // 1 / sqrt(D)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) {
    const double* t = S.d + lane * kLd;
    int bad = 0;
    double a[kH];
#pragma unroll
    for (int m = 0; m < kH; ++m) a[m] = t[m];
    ldl_cols<kH>(a, lane, 0, bad);
#pragma unroll
    for (int m = 0; m < kH; ++m) f[lane * kFs + m] = a[m];
    __syncwarp();
    double bq[kH];
#pragma unroll
    for (int m = 0; m < kH; ++m) bq[m] = t[kH + m];
#pragma unroll
    for (int p = 0; p < kH; ++p) {
      const double w = f[lane * kFs + p] * f[p * kFs + p];
#pragma unroll
      for (int m = 0; m < kH; ++m) bq[m] = fma(-w, f[(kH + m) * kFs + p], bq[m]);
    }
    ldl_cols<kH>(bq, lane, kH, bad);
#pragma unroll
    for (int m = 0; m < kH; ++m) f[lane * kFs + kH + m] = lane >= kH ? bq[m] : 0.0;
    if (bad && lane == 0) *ok = 0;
    __syncwarp();
    const double sq = sqrt(f[lane * kFs + lane]);
    sd[lane] = sq;
    isd[lane] = 1.0 / sq;
    double x[kH];
#pragma unroll
    for (int r = 0; r < kH; ++r) {
      double s0 = (r == lane) ? 1.0 : 0.0, s1 = 0.0;
#pragma unroll
      for (int m = 0; m + 1 < r; m += 2) {
        s0 = fma(-f[r * kFs + m], x[m], s0);
        s1 = fma(-f[r * kFs + m + 1], x[m + 1], s1);
      }
      if (r & 1) s0 = fma(-f[r * kFs + r - 1], x[r - 1], s0);
      x[r] = s0 + s1;
    }
#pragma unroll
    for (int r = 0; r < kH; ++r) xs[r * kFs + lane] = x[r];
    double z[kH];
#pragma unroll
    for (int r = 0; r < kH; ++r) z[r] = (kH + r == lane) ? 1.0 : 0.0;
#pragma unroll
    for (int p = 0; p < kH; ++p) {
      const double xp = xs[p * kFs + lane];
#pragma unroll
      for (int r = 0; r < kH; ++r) z[r] = fma(-f[(kH + r) * kFs + p], xp, z[r]);
    }
#pragma unroll
    for (int r = 0; r < kH; ++r) {
      double s0 = z[r];
#pragma unroll
      for (int m = 0; m < r; ++m) s0 = fma(-f[(kH + r) * kFs + kH + m], z[m], s0);
      z[r] = s0;
    }
#pragma unroll
    for (int r = 0; r < kH; ++r) xs[(kH + r) * kFs + lane] = z[r];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < kT * kT; e += blockDim.x) {
    const int r = e >> 5, c = e & 31;
    gL[static_cast<size_t>(r) * ldL + c] = c < r ? f[r * kFs + c] * sd[c] : (c == r ? sd[r] : 0.0);
    gD[e] = xs[r * kFs + c] * isd[r];
  }
  __syncthreads();
}

// First column tile of E tile row c that can be non-zero: row 0 is rhs
// (dense); row e >= 1 is F^T row e - 1, non-zero only over its field block.
__device__ __forceinline__ int e_start(int c, int r, int k) {
  if (c == 0 || r == 0) return 0;
  return (((kT * c - 1) / r) * k) / kT;
}

// One system's operands and workspace.
struct Sys {
  double* A;           // Pp x Pp: L in the lower tiles
  double* E;           // Ep x Pp: appended rows
  double* Dv;          // nb x 32 x 32: inverses of the diagonal tiles
  const double* M;     // P x P
  const double* rhs;   // P
  const double* pen;   // k x k
  const double* fk;    // k x r
  double lam;
  int P, Pp, k, r, nfr;
  bool mvec;           // rows of M 16-byte aligned (P even)
};

__device__ __forceinline__ double* a_tile(const Sys& y, int ti, int tj) {
  return y.A + static_cast<size_t>(ti) * kT * y.Pp + tj * kT;
}
__device__ __forceinline__ double* e_tile(const Sys& y, int c, int tj) {
  return y.E + static_cast<size_t>(c) * kT * y.Pp + tj * kT;
}

// Initial value of E (row, col): rhs in row 0, F^T below, zero padding.
__device__ __forceinline__ double e_init(const Sys& y, int row, int col) {
  if (row == 0) return col < y.P ? y.rhs[col] : 0.0;
  if (row > y.nfr) return 0.0;
  const int fb = (row - 1) / y.r, jj = (row - 1) - fb * y.r, m = col - fb * y.k;
  return (m >= 0 && m < y.k) ? y.fk[m * y.r + jj] : 0.0;
}

// Does A tile (ti, tj) hold an element of a diagonal field block (penalised)?
__device__ __forceinline__ bool a_pen_tile(const Sys& y, int ti, int tj) {
  const int r0 = ti * kT, c0 = tj * kT;
  if (r0 >= y.P || c0 >= y.P) return false;
  const int r1 = min(r0 + kT - 1, y.P - 1), c1 = min(c0 + kT - 1, y.P - 1);
  return max(r0 / y.k, c0 / y.k) <= min(r1 / y.k, c1 / y.k);
}

// Stage A tile (ti, tj) into the shared tile s: from the workspace, or at its
// first touch from M (identity padding outside P x P); the penalty of a first
// touch is added by a_pen_fix once the copies have landed.
__device__ __forceinline__ void a_stage(double* s, const Sys& y, int ti, int tj, bool first) {
  if (!first) {
    tile_async(s, a_tile(y, ti, tj), y.Pp);
    return;
  }
  for (int q = threadIdx.x; q < kT * kT / 2; q += blockDim.x) {
    const int r = q >> 4, c = (q & 15) * 2;
    const int row = ti * kT + r, col = tj * kT + c;
    if (y.mvec && row < y.P && col + 1 < y.P) {
      cp16(s + r * kLd + c, y.M + static_cast<size_t>(row) * y.P + col);
    } else {
#pragma unroll
      for (int u = 0; u < 2; ++u)
        s[r * kLd + c + u] = (row < y.P && col + u < y.P) ? y.M[static_cast<size_t>(row) * y.P + col + u]
                                                          : (row == col + u ? 1.0 : 0.0);
    }
  }
}
// A = M + lambda P0 on the diagonal field blocks of a staged first-touch tile.
__device__ __forceinline__ void a_pen_fix(double* s, const Sys& y, int ti, int tj) {
  for (int e = threadIdx.x; e < kT * kT; e += blockDim.x) {
    const int r = e >> 5, c = e & 31, row = ti * kT + r, col = tj * kT + c;
    if (row < y.P && col < y.P && row / y.k == col / y.k)
      s[r * kLd + c] = fma(y.lam, y.pen[(row % y.k) * y.k + col % y.k], s[r * kLd + c]);
  }
}
// Stage E tile (c, tj): from the workspace, or generated at its first touch.
__device__ __forceinline__ void e_stage(double* s, const Sys& y, int c, int tj, bool first) {
  if (!first) {
    tile_async(s, e_tile(y, c, tj), y.Pp);
    return;
  }
  for (int e = threadIdx.x; e < kT * kT; e += blockDim.x)
    s[(e >> 5) * kLd + (e & 31)] = e_init(y, c * kT + (e >> 5), tj * kT + (e & 31));
}

__global__ void __launch_bounds__(kSolveThreads, 2) k_solve_cluster(SolveBatch b, int Pp, int Ep, size_t sys_stride) {
  extern __shared__ __align__(16) unsigned char raw[];
  SolveSmem& S = *reinterpret_cast<SolveSmem*>(raw);
  const cg::cluster_group cl = cg::this_cluster();
  const int cn = static_cast<int>(cl.num_blocks());
  const int rank = static_cast<int>(cl.block_rank());
  const int s = blockIdx.x / cn;
  const int tid = threadIdx.x;
  Sys y;
  y.A = b.A + static_cast<size_t>(s) * sys_stride;
  y.E = y.A + static_cast<size_t>(Pp) * Pp;
  y.Dv = y.E + static_cast<size_t>(Ep) * Pp;
  y.P = b.P;
  y.Pp = Pp;
  y.k = b.k;
  y.r = b.r;
  y.nfr = b.nf * b.r;
  y.M = b.M + (b.m_index ? static_cast<size_t>(b.m_index[s]) * y.P * y.P : 0);
  y.rhs = b.rhs + (b.r_index ? static_cast<size_t>(b.r_index[s]) * y.P : 0);
  y.pen = b.pen;
  y.fk = b.fk;
  y.lam = b.lam[s];
  y.mvec = (y.P & 1) == 0;
  const int nb = Pp / kT, ne = Ep / kT;
  __shared__ int s_ok;
  if (tid == 0) s_ok = 1;

  // Diagonal tile 0 (first touch).
  if (rank == 0) {
    a_stage(S.d, y, 0, 0, true);
    cp_commit();
    cp_wait0();
    __syncthreads();
    a_pen_fix(S.d, y, 0, 0);
    __syncthreads();
    factor_tile(S, y.A, Pp, y.Dv, &s_ok);
  }
  cluster_step(cl);

  double tr = 0.0;  // this thread's share of ||L^-1 F||^2
  for (int j = 0; j < nb; ++j) {
    const int below = nb - j - 1;
    int nact = 0;
    while (nact < ne && e_start(nact, y.r, y.k) <= j) ++nact;
    // Panel: tiles below the diagonal of column j, then the active E tiles.
    {
      const int nt = below + nact;
      if (rank < nt) {
        tile_async(S.d, y.Dv + static_cast<size_t>(j) * kT * kT, kT);
        run_jobs(
            S, rank, nt, [&](int t) { return t + cn; },
            [&](double (*buf)[kTS], int t) {
              if (t < below)
                a_stage(buf[0], y, j + 1 + t, j, j == 0);
              else
                e_stage(buf[0], y, t - below, j, e_start(t - below, y.r, y.k) == j);
            },
            [&](double (*buf)[kTS], int t) {
              if (t < below && j == 0 && a_pen_tile(y, j + 1 + t, j)) {
                a_pen_fix(buf[0], y, j + 1 + t, j);
                __syncthreads();
              }
              double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
              mma_nt(buf[0], S.d, acc);
              double* g = t < below ? a_tile(y, j + 1 + t, j) : e_tile(y, t - below, j);
              const int r0 = frag_row();
              const bool erow = t >= below && !(t == below && r0 == 0);
#pragma unroll
              for (int blk = 0; blk < 2; ++blk) {
                const int c0 = frag_col(blk);
                *reinterpret_cast<double2*>(g + static_cast<size_t>(r0) * Pp + c0) = make_double2(acc[blk][0], acc[blk][1]);
                if (erow) tr = fma(acc[blk][0], acc[blk][0], fma(acc[blk][1], acc[blk][1], tr));
              }
            });
      }
    }
    cluster_step(cl);
    if (below == 0) break;
    // Trailing update. Job list: A tiles (i, m), j < m <= i, in row order
    // without (j+1, j+1); then E tiles (c, m), c < nact, m > j.
    {
      if (rank == 0) {
        // Next diagonal tile: A_{j+1,j+1} -= L_{j+1,j} L_{j+1,j}^T, factor.
        a_stage(S.op[0][0], y, j + 1, j + 1, j == 0);
        tile_async(S.op[0][1], a_tile(y, j + 1, j), Pp);
        cp_commit();
        cp_wait0();
        __syncthreads();
        if (j == 0) {
          a_pen_fix(S.op[0][0], y, j + 1, j + 1);
          __syncthreads();
        }
        double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
        mma_nt(S.op[0][1], S.op[0][1], acc);
        const int r0 = frag_row();
#pragma unroll
        for (int blk = 0; blk < 2; ++blk) {
          const int c0 = frag_col(blk);
          S.d[r0 * kLd + c0] = S.op[0][0][r0 * kLd + c0] - acc[blk][0];
          S.d[r0 * kLd + c0 + 1] = S.op[0][0][r0 * kLd + c0 + 1] - acc[blk][1];
        }
        __syncthreads();
        factor_tile(S, a_tile(y, j + 1, j + 1), Pp, y.Dv + static_cast<size_t>(j + 1) * kT * kT, &s_ok);
      }
      const int nta = below * (below + 1) / 2 - 1;
      const int nt = nta + nact * below;
      // Rank 0 skips the first kRank0Debt rounds of the deal.
      const int debt = cn > 1 ? kRank0Debt * (cn - 1) : 0;
      auto owner_next = [&](int t) {
        if (t < debt) {
          const int tn = t + (cn - 1);
          return tn < debt ? tn : debt + rank;
        }
        return t + cn;
      };
      const int first = (cn == 1 || rank == 0) ? debt : rank - 1;
      // Job t -> (is E, tile row, tile column m).
      auto decode = [&](int t, int& ti, int& m) {
        if (t < nta) {
          int tt = t + 1, ii = 0;
          while (tt > ii) {
            tt -= ii + 1;
            ++ii;
          }
          ti = j + 1 + ii;
          m = j + 1 + tt;
          return false;
        }
        const int u = t - nta;
        ti = u / below;
        m = j + 1 + (u - ti * below);
        return true;
      };
      run_jobs(
          S, first, nt, owner_next,
          [&](double (*buf)[kTS], int t) {
            int ti, m;
            if (decode(t, ti, m)) {
              e_stage(buf[0], y, ti, m, e_start(ti, y.r, y.k) == j);
              tile_async(buf[1], e_tile(y, ti, j), Pp);
            } else {
              a_stage(buf[0], y, ti, m, j == 0);
              tile_async(buf[1], a_tile(y, ti, j), Pp);
            }
            tile_async(buf[2], a_tile(y, m, j), Pp);
          },
          [&](double (*buf)[kTS], int t) {
            int ti, m;
            const bool is_e = decode(t, ti, m);
            if (!is_e && j == 0 && a_pen_tile(y, ti, m)) {
              a_pen_fix(buf[0], y, ti, m);
              __syncthreads();
            }
            double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
            mma_nt(buf[1], buf[2], acc);
            double* c = is_e ? e_tile(y, ti, m) : a_tile(y, ti, m);
            const int r0 = frag_row();
#pragma unroll
            for (int blk = 0; blk < 2; ++blk) {
              const int c0 = frag_col(blk);
              const double2 old = *reinterpret_cast<const double2*>(buf[0] + r0 * kLd + c0);
              *reinterpret_cast<double2*>(c + static_cast<size_t>(r0) * Pp + c0) =
                  make_double2(old.x - acc[blk][0], old.y - acc[blk][1]);
            }
          });
    }
    cluster_step(cl);
  }

  // Trace partial of this rank (fixed-order tree), then rank 0 finishes.
  S.red[tid] = tr;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (tid < o) S.red[tid] += S.red[tid + o];
    __syncthreads();
  }
  if (tid == 0) b.partial[static_cast<size_t>(s) * cn + rank] = S.red[0];
  cluster_step(cl);
  if (rank != 0) return;
  if (tid == 0) {
    double t2 = 0.0;
    for (int q = 0; q < cn; ++q) t2 += b.partial[static_cast<size_t>(s) * cn + q];
    b.edf[s] = static_cast<double>(y.P) - y.lam * t2;
    b.ok[s] = s_ok;
  }
  // theta = L^-T y, y = E row 0: column tiles from the last, each
  // theta_i = Dinv_i^T y_i, then y_q -= L_iq^T theta_i for q < i.
  double* v = S.v;
  const int warp = tid >> 5, ln = tid & 31;
  for (int q = tid; q < Pp; q += blockDim.x) v[q] = __ldcg(y.E + q);
  __syncthreads();
  for (int i = nb - 1; i >= 0; --i) {
    if (warp == 0) {
      const double* D = y.Dv + static_cast<size_t>(i) * kT * kT;
      double t0 = 0.0, t1 = 0.0;
#pragma unroll
      for (int r = 0; r < kT; r += 2) {
        t0 = fma(__ldcg(D + r * kT + ln), v[i * kT + r], t0);
        t1 = fma(__ldcg(D + (r + 1) * kT + ln), v[i * kT + r + 1], t1);
      }
      __syncwarp();
      v[i * kT + ln] = t0 + t1;
    }
    __syncthreads();
    for (int q = tid; q < i * kT; q += blockDim.x) {
      const double* Lc = y.A + static_cast<size_t>(i) * kT * Pp + q;
      double a0 = v[q], a1 = 0.0;
#pragma unroll
      for (int r = 0; r < kT; r += 2) {
        a0 = fma(-__ldcg(Lc + static_cast<size_t>(r) * Pp), v[i * kT + r], a0);
        a1 = fma(-__ldcg(Lc + static_cast<size_t>(r + 1) * Pp), v[i * kT + r + 1], a1);
      }
      v[q] = a0 + a1;
    }
    __syncthreads();
  }
  for (int q = tid; q < y.P; q += blockDim.x) b.theta[static_cast<size_t>(s) * y.P + q] = v[q];
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
  const int Ep = solve_ep(b.nf, b.r);
  if (b.P > 1024) fail(DGPU_ERR_INVALID, "solve: more than 1024 unknowns is not supported");
  if (b.k > 1024 || b.r > b.k) fail(DGPU_ERR_INVALID, "solve: penalty factor shape is not supported");
  if (b.nsys <= 0) return;
  const int cn = solve_cluster_size(b.nsys);
  const size_t smem = sizeof(SolveSmem);
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
  DGPU_CUDA(cudaLaunchKernelEx(&cfg, k_solve_cluster, bb, Pp, Ep, solve_sys_doubles(b.P, b.nf, b.r)));
  DGPU_LAUNCH("k_solve_cluster");
}

// out = A_s^{-1} v = L^-T (L^-1 v) from system s's factor tiles, one CTA:
// forward over the column tiles (y_i = Dinv_i y_i, then y_p -= L_pi y_i for
// the rows below, a thread per row), then the back substitution of the solver.
constexpr int kAiThreads = 512;

__global__ void __launch_bounds__(kAiThreads) k_apply_inverse(const double* __restrict__ L, const double* __restrict__ Dv,
                                                               int P, int Pp, const double* __restrict__ vin,
                                                               double* __restrict__ out) {
  __shared__ double y[1024];
  __shared__ double dt[kT * (kT + 1)];
  const int tid = threadIdx.x, warp = tid >> 5, ln = tid & 31;
  const int nb = Pp / kT;
  for (int q = tid; q < Pp; q += blockDim.x) y[q] = q < P ? vin[q] : 0.0;
  for (int i = 0; i < nb; ++i) {
    for (int e = tid; e < kT * kT; e += blockDim.x) dt[(e >> 5) * (kT + 1) + (e & 31)] = Dv[static_cast<size_t>(i) * kT * kT + e];
    __syncthreads();
    if (warp == 0) {
      double t0 = 0.0, t1 = 0.0;
#pragma unroll
      for (int c = 0; c < kT; c += 2) {
        t0 = fma(dt[ln * (kT + 1) + c], y[i * kT + c], t0);
        t1 = fma(dt[ln * (kT + 1) + c + 1], y[i * kT + c + 1], t1);
      }
      __syncwarp();
      y[i * kT + ln] = t0 + t1;
    }
    __syncthreads();
    for (int p = (i + 1) * kT + tid; p < Pp; p += blockDim.x) {
      const double2* Lr = reinterpret_cast<const double2*>(L + static_cast<size_t>(p) * Pp + i * kT);
      double a0 = y[p], a1 = 0.0;
#pragma unroll
      for (int c = 0; c < kT / 2; ++c) {
        const double2 l2 = __ldg(Lr + c);
        a0 = fma(-l2.x, y[i * kT + 2 * c], a0);
        a1 = fma(-l2.y, y[i * kT + 2 * c + 1], a1);
      }
      y[p] = a0 + a1;
    }
    __syncthreads();
  }
  for (int i = nb - 1; i >= 0; --i) {
    if (warp == 0) {
      const double* D = Dv + static_cast<size_t>(i) * kT * kT;
      double t0 = 0.0, t1 = 0.0;
#pragma unroll
      for (int r = 0; r < kT; r += 2) {
        t0 = fma(D[r * kT + ln], y[i * kT + r], t0);
        t1 = fma(D[(r + 1) * kT + ln], y[i * kT + r + 1], t1);
      }
      __syncwarp();
      y[i * kT + ln] = t0 + t1;
    }
    __syncthreads();
    for (int q = tid; q < i * kT; q += blockDim.x) {
      const double* Lc = L + static_cast<size_t>(i) * kT * Pp + q;
      double a0 = y[q], a1 = 0.0;
#pragma unroll
      for (int r = 0; r < kT; r += 2) {
        a0 = fma(-Lc[static_cast<size_t>(r) * Pp], y[i * kT + r], a0);
        a1 = fma(-Lc[static_cast<size_t>(r + 1) * Pp], y[i * kT + r + 1], a1);
      }
      y[q] = a0 + a1;
    }
    __syncthreads();
  }
  for (int q = tid; q < P; q += blockDim.x) out[q] = y[q];
}

void launch_apply_inverse(cudaStream_t st, const SolveBatch& b, int s, const double* v, double* out) {
  const int Pp = solve_pp(b.P);
  const double* A = b.A + static_cast<size_t>(s) * solve_sys_doubles(b.P, b.nf, b.r);
  const double* Dv = A + static_cast<size_t>(Pp) * Pp + static_cast<size_t>(solve_ep(b.nf, b.r)) * Pp;
  k_apply_inverse<<<1, kAiThreads, 0, st>>>(A, Dv, b.P, Pp, v, out);
  DGPU_LAUNCH("k_apply_inverse");
}

}  // namespace dgpu
