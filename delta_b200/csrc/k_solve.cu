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
//   trailing  A_im -= L_ij L_mj^T, E_cm -= X_cj L_mj^T over ranks 1..; rank 0
//             meanwhile updates and factors the next diagonal tile (one-tile
//             look-ahead, LDL^T with the tile's rows in registers).
// The workspace is tile-major (each tile one contiguous block with the
// shared-memory row stride), so tile operands are staged by double-buffered
// single bulk async copies completing on an mbarrier; products run on the
// FP64 tensor cores (mma.sync m8n8k4). A is never assembled: M, converted to
// tiles once per distinct matrix, is read at a tile's first touch and the
// penalty added there; E is generated at its first touch. theta = L^-T y by back
// substitution on rank 0. The trace is reduced per rank in a fixed order and
// summed in rank order (deterministic). A non-positive pivot marks the system
// failed (ok = 0); k_ldlt.cu then redoes it by pivoted LDL^T, as the reference
// falls back from LLT to LDLT.
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
constexpr int kMaxTiles = 40;  // tile rows of E (and columns of A) per system

// Workspace, tile-major: every 32 x 32 tile is one contiguous kTS block with
// the shared-memory row stride kLd, so a tile moves with one bulk copy. Per
// system: the lower tiles of A (row-major triangle), the ne x nb tiles of E,
// the nb tiles of Dinv; then the lower tiles of each distinct M (identity
// padding outside P x P).
int solve_pp(int P) { return (P + kT - 1) / kT * kT; }
int solve_ep(int nf, int r) { return (nf * r + 1 + kT - 1) / kT * kT; }
size_t solve_sys_doubles(int P, int nf, int r) {
  const size_t nb = solve_pp(P) / kT, ne = solve_ep(nf, r) / kT;
  return (nb * (nb + 1) / 2 + ne * nb + nb) * kTS;
}
size_t solve_m_doubles(int P) {
  const size_t nb = solve_pp(P) / kT;
  return nb * (nb + 1) / 2 * kTS;
}
size_t solve_work_doubles(int P, int nf, int r, int nsys, int nm) {
  return static_cast<size_t>(nsys) * solve_sys_doubles(P, nf, r) + static_cast<size_t>(std::max(nm, 1)) * solve_m_doubles(P);
}
__host__ __device__ __forceinline__ int tri_index(int ti, int tj) { return ti * (ti + 1) / 2 + tj; }

struct SolveSmem {
  double op[2][3][kTS];  // double-buffered job operands: C (updated), left, right
  double d[kTS];         // Dinv_j in the panel phase; the diagonal tile in the trailing phase
  double v[1024];        // y / theta in the back substitution
  double red[kSolveThreads];
  uint64_t bar[3];       // mbarriers: job buffers 0 and 1, the diagonal tile
};

constexpr long long kSolveSpin = 1ll << 22;  // bounded mbarrier wait (iterations)

__device__ __forceinline__ uint32_t saddr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// 1-D bulk async copy global -> this CTA's shared memory completing on `bar`
// (no multicast); dst, src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(saddr(dst)), "l"(src), "r"(bytes), "r"(saddr(bar))
               : "memory");
}
// Generic-proxy accesses of this CTA (ordered by a preceding barrier) before
// the async-proxy writes the issuing thread starts next.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}
// Bounded wait for the phase of `bar` with the given parity; false on expiry.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  const uint32_t a = saddr(bar);
  for (long long it = 0; it < kSolveSpin; ++it) {
    uint32_t done = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Staging of one job: lane `slot` of warp 0 moves a whole tile with one bulk
// copy and counts its bytes in tx; every lane of warp 0 then arrives on the
// buffer's mbarrier (32 arrivals) with its byte count.
__device__ __forceinline__ void tile_bulk(double* s, const double* g, int slot, uint64_t* bar, uint32_t& tx) {
  if (threadIdx.x == slot) {
    bulk_g2s(s, g, kTS * 8, bar);
    tx += kTS * 8;
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
// next job in flight while the current one computes. load(buf, t, bar, tx)
// stages job t into the three tiles of buf (bulk copies counted in tx,
// generated values stored directly); compute(buf, t) uses them. par holds
// the expected phase parity of each mbarrier.
template <class Next, class Load, class Compute>
__device__ __forceinline__ void run_jobs(SolveSmem& S, unsigned& par, unsigned* status, int first, int nt, Next next,
                                         Load load, Compute compute) {
  if (first >= nt) return;
  const bool w0 = threadIdx.x < 32;
  auto issue = [&](int b, int t) {
    if (w0) fence_proxy_async();
    uint32_t tx = 0;
    load(S.op[b], t, &S.bar[b], tx);
    if (w0) mbar_arrive_tx(&S.bar[b], tx);
  };
  int cur = 0;
  issue(0, first);
  for (int t = first; t < nt;) {
    const int tn = next(t);
    if (tn < nt) issue(cur ^ 1, tn);
    if (!mbar_wait(&S.bar[cur], (par >> cur) & 1u)) set_status(status, kStatusLoopLimit);
    par ^= 1u << cur;
    __syncthreads();
    compute(S.op[cur], t);
    __syncthreads();
    cur ^= 1;
    t = tn;
  }
}

// 1 / d to within an ulp: the hardware approximation (rcp.approx.ftz.f64)
// refined by two Newton-Raphson steps x <- x + x (1 - d x), each of which
// squares the relative error. d is a positive normal pivot.
__device__ __forceinline__ double rcp_newton(double d) {
  double x;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(x) : "d"(d));
  double e = fma(-d, x, 1.0);
  x = fma(x, e, x);
  e = fma(-d, x, 1.0);
  return fma(x, e, x);
}

// Right-looking LDL^T of N columns held in registers, lane = row: the pivot
// of column q is on lane base + q; column q is broadcast through col (32
// doubles of shared memory). Afterwards a[q] holds the unit factor l_rq
// below the pivot, the pivot d_q on it and zero above.
template <int N>
__device__ __forceinline__ void ldl_cols(double (&a)[N], int lane, int base, int& bad, double* col) {
#pragma unroll
  for (int q = 0; q < N; ++q) {
    double d = __shfl_sync(0xffffffffu, a[q], base + q);
    if (!(d > 0.0)) {
      bad = 1;
      d = 1.0;
    }
    const double u = a[q];
    col[lane] = u;
    const double l = u * rcp_newton(d);
    __syncwarp();
#pragma unroll
    for (int m = q + 1; m < N; ++m) {
      const double um = col[base + m];
      if (lane >= base + m) a[m] = fma(-l, um, a[m]);
    }
    __syncwarp();
    a[q] = lane > base + q ? l : (lane == base + q ? d : 0.0);
  }
}

// Factor the symmetric tile in S.d (lower part used): L_jj into the A tile
// gL (upper zeroed) and Dinv_j = L_jj^-1 into the tile gD. LDL^T in
// two 16-column halves, lane = row (warp 0): columns 0-15 of all rows; the
// Schur complement of the lower-right block (all warps); its factorisation.
// Then L = Lu D^1/2 and L^-1 = D^-1/2 Lu^-1 with Lu^-1 by blocks: x = Lu11^-1
// (warp 0, lane = column), z0 = e - Lu21 x (all warps), z = Lu22^-1 z0 (warp
// 0). A non-positive pivot clears *ok and continues with pivot 1.
constexpr int kFs = kT + 1;
constexpr int kH = kT / 2;
__device__ __noinline__ void factor_tile(SolveSmem& S, double* gL, double* gD, int* ok) {
  double* f = S.op[0][2];         // 32 x kFs: Lu below the diagonal, D on it
  double* xs = S.op[1][0];        // 32 x kFs: Lu^-1
  double* sd = S.op[1][1];        // sqrt(D)
  double* isd = S.op[1][1] + kT;  // 1 / sqrt(D)
  double* col = S.op[1][1] + 2 * kT;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int bad = 0;
  if (warp == 0) {
    const double* t = S.d + lane * kLd;
    double a[kH];
#pragma unroll
    for (int m = 0; m < kH; ++m) a[m] = t[m];
    ldl_cols<kH>(a, lane, 0, bad, col);
#pragma unroll
    for (int m = 0; m < kH; ++m) f[lane * kFs + m] = a[m];
  }
  __syncthreads();
  // Schur complement of the lower-right block: thread (r, m), m <= r.
  {
    const int r = tid >> 4, m = tid & 15;
    if (m <= r) {
      double v = S.d[(kH + r) * kLd + kH + m];
#pragma unroll
      for (int p = 0; p < kH; ++p) v = fma(-f[(kH + r) * kFs + p] * f[p * kFs + p], f[(kH + m) * kFs + p], v);
      f[(kH + r) * kFs + kH + m] = v;
    }
  }
  __syncthreads();
  if (warp == 0) {
    double bq[kH];
#pragma unroll
    for (int m = 0; m < kH; ++m) bq[m] = lane >= kH ? f[lane * kFs + kH + m] : 0.0;
    ldl_cols<kH>(bq, lane, kH, bad, col);
#pragma unroll
    for (int m = 0; m < kH; ++m) f[lane * kFs + kH + m] = lane >= kH ? bq[m] : 0.0;
    if (bad && lane == 0) *ok = 0;
    __syncwarp();
    const double sq = sqrt(f[lane * kFs + lane]);
    sd[lane] = sq;
    isd[lane] = 1.0 / sq;
    // x = Lu11^-1 e_lane (zero for lanes >= 16).
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
  }
  __syncthreads();
  // z0 = e_c - Lu21 x: thread (r, c) for c < 16; columns c >= 16 are e_c.
  {
    const int r = tid >> 4, c = tid & 15;
    double v = 0.0;
#pragma unroll
    for (int p = 0; p < kH; ++p) v = fma(-f[(kH + r) * kFs + p], xs[p * kFs + c], v);
    xs[(kH + r) * kFs + c] = v;
    xs[(kH + r) * kFs + kH + c] = (r == c) ? 1.0 : 0.0;
  }
  __syncthreads();
  if (warp == 0) {
    double z[kH];
#pragma unroll
    for (int r = 0; r < kH; ++r) {
      double s0 = xs[(kH + r) * kFs + lane];
#pragma unroll
      for (int m = 0; m < r; ++m) s0 = fma(-f[(kH + r) * kFs + kH + m], z[m], s0);
      z[r] = s0;
    }
#pragma unroll
    for (int r = 0; r < kH; ++r) xs[(kH + r) * kFs + lane] = z[r];
  }
  __syncthreads();
  for (int e = tid; e < kT * kT; e += blockDim.x) {
    const int r = e >> 5, c = e & 31;
    gL[r * kLd + c] = c < r ? f[r * kFs + c] * sd[c] : (c == r ? sd[r] : 0.0);
    gD[r * kLd + c] = xs[r * kFs + c] * isd[r];
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
  double* A;           // lower tiles: L
  double* E;           // ne x nb tiles: appended rows
  double* Dv;          // nb tiles: inverses of the diagonal tiles
  const double* Mt;    // lower tiles of M
  const double* rhs;   // P
  const double* pen;   // k x k
  const double* fk;    // k x r
  double lam;
  int P, Pp, k, r, nfr, nb;
};

__device__ __forceinline__ double* a_tile(const Sys& y, int ti, int tj) {
  return y.A + static_cast<size_t>(tri_index(ti, tj)) * kTS;
}
__device__ __forceinline__ double* e_tile(const Sys& y, int c, int tj) {
  return y.E + static_cast<size_t>(c * y.nb + tj) * kTS;
}
__device__ __forceinline__ double* d_tile(const Sys& y, int j) { return y.Dv + static_cast<size_t>(j) * kTS; }

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
// first touch from the converted M (the penalty of a first touch is added by
// a_pen_fix once the copy has landed).
__device__ __forceinline__ void a_stage(double* s, const Sys& y, int ti, int tj, bool first, int slot,
                                        uint64_t* bar, uint32_t& tx) {
  tile_bulk(s, first ? y.Mt + static_cast<size_t>(tri_index(ti, tj)) * kTS : a_tile(y, ti, tj), slot, bar, tx);
}
// A = M + lambda P0 on the diagonal field blocks of a staged first-touch tile
// (a warp per row, lane = column).
__device__ __forceinline__ void a_pen_fix(double* s, const Sys& y, int ti, int tj) {
  const int lane = threadIdx.x & 31, col = tj * kT + lane;
  if (col >= y.P) return;
  const int cb = col / y.k, cm = col - cb * y.k;
  for (int r = threadIdx.x >> 5; r < kT; r += blockDim.x >> 5) {
    const int row = ti * kT + r;
    if (row >= y.P) break;
    const int rb = row / y.k;
    if (rb == cb) s[r * kLd + lane] = fma(y.lam, y.pen[(row - rb * y.k) * y.k + cm], s[r * kLd + lane]);
  }
}
// Stage E tile (c, tj): from the workspace, or generated at its first touch
// (a warp per row, lane = column).
__device__ __forceinline__ void e_stage(double* s, const Sys& y, int c, int tj, bool first, int slot,
                                        uint64_t* bar, uint32_t& tx) {
  if (!first) {
    tile_bulk(s, e_tile(y, c, tj), slot, bar, tx);
    return;
  }
  const int lane = threadIdx.x & 31, col = tj * kT + lane;
  for (int r = threadIdx.x >> 5; r < kT; r += blockDim.x >> 5) {
    const int row = c * kT + r;
    double v = 0.0;
    if (row == 0) {
      v = col < y.P ? y.rhs[col] : 0.0;
    } else if (row <= y.nfr) {
      const int fb = (row - 1) / y.r, jj = (row - 1) - fb * y.r, m = col - fb * y.k;
      if (m >= 0 && m < y.k) v = y.fk[m * y.r + jj];
    }
    s[r * kLd + lane] = v;
  }
}

__global__ void __launch_bounds__(kSolveThreads, 2) k_solve_cluster(SolveBatch b, int Pp, int Ep, size_t sys_stride, const double* __restrict__ Mt) {
  extern __shared__ __align__(16) unsigned char raw[];
  SolveSmem& S = *reinterpret_cast<SolveSmem*>(raw);
  const cg::cluster_group cl = cg::this_cluster();
  const int cn = static_cast<int>(cl.num_blocks());
  const int rank = static_cast<int>(cl.block_rank());
  const int s = blockIdx.x / cn;
  const int tid = threadIdx.x;
  Sys y;
  y.A = b.A + static_cast<size_t>(s) * sys_stride;
  const int nb = Pp / kT, ne = Ep / kT;
  y.nb = nb;
  y.E = y.A + static_cast<size_t>(nb * (nb + 1) / 2) * kTS;
  y.Dv = y.E + static_cast<size_t>(ne * nb) * kTS;
  y.P = b.P;
  y.Pp = Pp;
  y.k = b.k;
  y.r = b.r;
  y.nfr = b.nf * b.r;
  y.Mt = Mt + (b.m_index ? static_cast<size_t>(b.m_index[s]) * (nb * (nb + 1) / 2) * kTS : 0);
  y.rhs = b.rhs + (b.r_index ? static_cast<size_t>(b.r_index[s]) * y.P : 0);
  y.pen = b.pen;
  y.fk = b.fk;
  y.lam = b.lam[s];
  __shared__ int s_ok;
  __shared__ int s_estart[kMaxTiles];
  if (tid == 0) {
    s_ok = 1;
    for (int q = 0; q < 3; ++q)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 32;" ::"r"(saddr(&S.bar[q])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int c = tid; c < ne; c += blockDim.x) s_estart[c] = e_start(c, y.r, y.k);
  __syncthreads();
  unsigned par = 0;  // expected phase parity of S.bar[0..2]
  const bool w0 = tid < 32;
  // Stage the diagonal tile job on S.bar[2]: stage(bar, tx) issues it.
  auto stage_diag = [&](auto stage) {
    if (w0) fence_proxy_async();
    uint32_t tx = 0;
    stage(&S.bar[2], tx);
    if (w0) mbar_arrive_tx(&S.bar[2], tx);
    if (!mbar_wait(&S.bar[2], (par >> 2) & 1u)) set_status(b.status, kStatusLoopLimit);
    par ^= 4u;
    __syncthreads();
  };

  // Diagonal tile 0 (first touch).
  if (rank == 0) {
    stage_diag([&](uint64_t* bar, uint32_t& tx) { a_stage(S.d, y, 0, 0, true, 0, bar, tx); });
    a_pen_fix(S.d, y, 0, 0);
    __syncthreads();
    factor_tile(S, a_tile(y, 0, 0), d_tile(y, 0), &s_ok);
  }
  cluster_step(cl);

  double tr = 0.0;  // this thread's share of ||L^-1 F||^2
  for (int j = 0; j < nb; ++j) {
    const int below = nb - j - 1;
    int nact = 0;
    while (nact < ne && s_estart[nact] <= j) ++nact;
    // Panel: tiles below the diagonal of column j, then the active E tiles.
    {
      const int nt = below + nact;
      if (rank < nt) {
        run_jobs(
            S, par, b.status, rank, nt, [&](int t) { return t + cn; },
            [&](double (*buf)[kTS], int t, uint64_t* bar, uint32_t& tx) {
              // Dinv_j rides with this rank's first panel job.
              if (t == rank) tile_bulk(S.d, d_tile(y, j), 1, bar, tx);
              if (t < below)
                a_stage(buf[0], y, j + 1 + t, j, j == 0, 0, bar, tx);
              else
                e_stage(buf[0], y, t - below, j, s_estart[t - below] == j, 0, bar, tx);
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
                *reinterpret_cast<double2*>(g + r0 * kLd + c0) = make_double2(acc[blk][0], acc[blk][1]);
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
        stage_diag([&](uint64_t* bar, uint32_t& tx) {
          a_stage(S.op[0][0], y, j + 1, j + 1, j == 0, 0, bar, tx);
          tile_bulk(S.op[0][1], a_tile(y, j + 1, j), 1, bar, tx);
        });
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
        factor_tile(S, a_tile(y, j + 1, j + 1), d_tile(y, j + 1), &s_ok);
      }
      const int nta = below * (below + 1) / 2 - 1;
      const int nt = nta + nact * below;
      // Rank 0 factors the next diagonal tile meanwhile and takes no jobs;
      // a cluster of one does everything.
      const int workers = cn > 1 ? cn - 1 : 1;
      const int first = cn > 1 ? (rank == 0 ? nt : rank - 1) : 0;
      auto owner_next = [&](int t) { return t + workers; };
      // Job t -> (is E, tile row, tile column m).
      auto decode = [&](int t, int& ti, int& m) {
        if (t < nta) {
          // Lower triangle of the trailing block, row-major, diagonal
          // included: index t + 1 -> (ii, tt), ii (ii + 1) / 2 <= t + 1.
          const int idx = t + 1;
          int ii = static_cast<int>((sqrtf(8.0f * static_cast<float>(idx) + 1.0f) - 1.0f) * 0.5f);
          if ((ii + 1) * (ii + 2) / 2 <= idx) ++ii;
          if (ii * (ii + 1) / 2 > idx) --ii;
          ti = j + 1 + ii;
          m = j + 1 + (idx - ii * (ii + 1) / 2);
          return false;
        }
        const int u = t - nta;
        ti = u / below;
        m = j + 1 + (u - ti * below);
        return true;
      };
      run_jobs(
          S, par, b.status, first, nt, owner_next,
          [&](double (*buf)[kTS], int t, uint64_t* bar, uint32_t& tx) {
            int ti, m;
            if (decode(t, ti, m)) {
              e_stage(buf[0], y, ti, m, s_estart[ti] == j, 0, bar, tx);
              tile_bulk(buf[1], e_tile(y, ti, j), 1, bar, tx);
            } else {
              a_stage(buf[0], y, ti, m, j == 0, 0, bar, tx);
              tile_bulk(buf[1], a_tile(y, ti, j), 1, bar, tx);
            }
            tile_bulk(buf[2], a_tile(y, m, j), 2, bar, tx);
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
              *reinterpret_cast<double2*>(c + r0 * kLd + c0) = make_double2(old.x - acc[blk][0], old.y - acc[blk][1]);
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
  for (int q = tid; q < Pp; q += blockDim.x) v[q] = __ldcg(e_tile(y, 0, q >> 5) + (q & 31));
  __syncthreads();
  for (int i = nb - 1; i >= 0; --i) {
    if (warp == 0) {
      const double* D = d_tile(y, i);
      double t0 = 0.0, t1 = 0.0;
#pragma unroll
      for (int r = 0; r < kT; r += 2) {
        t0 = fma(__ldcg(D + r * kLd + ln), v[i * kT + r], t0);
        t1 = fma(__ldcg(D + (r + 1) * kLd + ln), v[i * kT + r + 1], t1);
      }
      __syncwarp();
      v[i * kT + ln] = t0 + t1;
    }
    __syncthreads();
    for (int q = tid; q < i * kT; q += blockDim.x) {
      const double* Lc = a_tile(y, i, q >> 5) + (q & 31);
      double a0 = v[q], a1 = 0.0;
#pragma unroll
      for (int r = 0; r < kT; r += 2) {
        a0 = fma(-__ldcg(Lc + r * kLd), v[i * kT + r], a0);
        a1 = fma(-__ldcg(Lc + (r + 1) * kLd), v[i * kT + r + 1], a1);
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

// The lower tiles of each distinct M in the tile-major layout, identity
// padding outside P x P (grid: tiles x matrices).
__global__ void __launch_bounds__(256) k_solve_prep(const double* __restrict__ M, int P, double* __restrict__ Mt) {
  const int u = blockIdx.x, m = blockIdx.y;
  int ti = static_cast<int>((sqrtf(8.0f * static_cast<float>(u) + 1.0f) - 1.0f) * 0.5f);
  if (tri_index(ti + 1, 0) <= u) ++ti;
  if (tri_index(ti, 0) > u) --ti;
  const int tj = u - tri_index(ti, 0);
  const double* Mm = M + static_cast<size_t>(m) * P * P;
  double* dst = Mt + (static_cast<size_t>(m) * gridDim.x + u) * kTS;
  for (int e = threadIdx.x; e < kT * kT; e += blockDim.x) {
    const int r = e >> 5, c = e & 31, row = ti * kT + r, col = tj * kT + c;
    dst[r * kLd + c] = (row < P && col < P) ? Mm[static_cast<size_t>(row) * P + col] : (row == col ? 1.0 : 0.0);
  }
}

void launch_solve_batch(Context& c, const SolveBatch& b) {
  const int Pp = solve_pp(b.P);
  const int Ep = solve_ep(b.nf, b.r);
  if (b.P > 1024) fail(DGPU_ERR_INVALID, "solve: more than 1024 unknowns is not supported");
  if (Ep / kT > kMaxTiles) fail(DGPU_ERR_INVALID, "solve: penalty factor too wide");
  if (b.k > 1024 || b.r > b.k) fail(DGPU_ERR_INVALID, "solve: penalty factor shape is not supported");
  if (b.nsys <= 0) return;
  const int nb = Pp / kT, nm = std::max(b.nm, 1);
  const size_t sys_stride = solve_sys_doubles(b.P, b.nf, b.r);
  double* Mt = b.A + static_cast<size_t>(b.nsys) * sys_stride;
  k_solve_prep<<<dim3(static_cast<unsigned>(nb * (nb + 1) / 2), static_cast<unsigned>(nm)), 256, 0, c.stream>>>(b.M, b.P, Mt);
  DGPU_LAUNCH("k_solve_prep");
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
  DGPU_CUDA(cudaLaunchKernelEx(&cfg, k_solve_cluster, bb, Pp, Ep, sys_stride, static_cast<const double*>(Mt)));
  DGPU_LAUNCH("k_solve_cluster");
  // Systems whose Cholesky met a non-positive pivot are redone by pivoted
  // LDL^T, as the reference falls back from LLT to LDLT (src/solve.cpp:177-181).
  if (b.skip_ldlt) return;
  StageTimer t(c, "fit: LDLT fallback");
  launch_ldlt_fallback(c, b);
}

// out = A_s^{-1} v = L^-T (L^-1 v) from system s's factor tiles, one CTA.
// The tiles are first pulled into L2 (one bulk prefetch per tile; streaming
// kernels that ran since the solve may have evicted them) and, up to 24 tile
// columns, every Dinv tile into shared memory. Forward over the column tiles:
// y_i = Dinv_i y_i (warp 0), then y_p -= L_pi y_i for the rows below (a thread
// per row); backward: theta_i = Dinv_i^T y_i, then y_q -= L_iq^T theta_i (a
// thread per column). Each thread's first row (column) of the next step is
// loaded into registers while the current step finishes, so the L2 latency
// overlaps the step's barriers and the diagonal solve.
constexpr int kAiThreads = 512;
constexpr int kDs = kT * (kT + 1);  // one Dinv tile in shared memory, padded rows
constexpr int kAiPreloadTiles = 24;

int apply_inverse_smem(int nb) { return static_cast<int>(sizeof(double)) * kDs * (nb <= kAiPreloadTiles ? nb : 1); }

__device__ __forceinline__ void ai_row(const double* __restrict__ A, int tile, int rr, double (&v)[kT]) {
  const double2* src = reinterpret_cast<const double2*>(A + static_cast<size_t>(tile) * kTS + rr * kLd);
#pragma unroll
  for (int c = 0; c < kT / 2; ++c) {
    const double2 t = __ldg(src + c);
    v[2 * c] = t.x;
    v[2 * c + 1] = t.y;
  }
}

__device__ __forceinline__ void ai_col(const double* __restrict__ A, int tile, int cc, double (&v)[kT]) {
  const double* src = A + static_cast<size_t>(tile) * kTS + cc;
#pragma unroll
  for (int r = 0; r < kT; ++r) v[r] = __ldg(src + r * kLd);
}

__global__ void __launch_bounds__(kAiThreads) k_apply_inverse(const double* __restrict__ A, const double* __restrict__ Dv,
                                                               int P, int Pp, const double* __restrict__ vin,
                                                               double* __restrict__ out) {
  extern __shared__ double dsm[];  // Dinv tiles (all, or the current one)
  __shared__ double y[1024];
  const int tid = threadIdx.x, warp = tid >> 5, ln = tid & 31;
  const int nb = Pp / kT, na = nb * (nb + 1) / 2;
  const bool all = nb <= kAiPreloadTiles;
  for (int u = tid; u < na + nb; u += blockDim.x) {
    const double* tile = u < na ? A + static_cast<size_t>(u) * kTS : Dv + static_cast<size_t>(u - na) * kTS;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(tile), "r"(static_cast<unsigned>(kTS * 8)) : "memory");
  }
  for (int q = tid; q < Pp; q += blockDim.x) y[q] = q < P ? vin[q] : 0.0;
  if (all)
    for (int e = tid; e < nb * kT * kT; e += blockDim.x) {
      const int t = e / (kT * kT), rc = e - t * (kT * kT);
      dsm[t * kDs + (rc >> 5) * (kT + 1) + (rc & 31)] = Dv[static_cast<size_t>(t) * kTS + (rc >> 5) * kLd + (rc & 31)];
    }
  double lv[kT];
  {
    const int p = kT + tid;
    if (p < Pp) ai_row(A, tri_index(p >> 5, 0), p & 31, lv);
  }
  __syncthreads();
  for (int i = 0; i < nb; ++i) {
    const double* D = dsm + (all ? i * kDs : 0);
    if (!all) {
      const double* Dg = Dv + static_cast<size_t>(i) * kTS;
      for (int e = tid; e < kT * kT; e += blockDim.x) dsm[(e >> 5) * (kT + 1) + (e & 31)] = Dg[(e >> 5) * kLd + (e & 31)];
      __syncthreads();
    }
    if (warp == 0) {
      double t0 = 0.0, t1 = 0.0;
#pragma unroll
      for (int c = 0; c < kT; c += 2) {
        t0 = fma(D[ln * (kT + 1) + c], y[i * kT + c], t0);
        t1 = fma(D[ln * (kT + 1) + c + 1], y[i * kT + c + 1], t1);
      }
      __syncwarp();
      y[i * kT + ln] = t0 + t1;
    }
    __syncthreads();
    const int p = (i + 1) * kT + tid;
    if (p < Pp) {
      double a0 = y[p], a1 = 0.0;
#pragma unroll
      for (int c = 0; c < kT / 2; ++c) {
        a0 = fma(-lv[2 * c], y[i * kT + 2 * c], a0);
        a1 = fma(-lv[2 * c + 1], y[i * kT + 2 * c + 1], a1);
      }
      y[p] = a0 + a1;
    }
    for (int p2 = p + kAiThreads; p2 < Pp; p2 += kAiThreads) {
      double l2[kT];
      ai_row(A, tri_index(p2 >> 5, i), p2 & 31, l2);
      double a0 = y[p2], a1 = 0.0;
#pragma unroll
      for (int c = 0; c < kT / 2; ++c) {
        a0 = fma(-l2[2 * c], y[i * kT + 2 * c], a0);
        a1 = fma(-l2[2 * c + 1], y[i * kT + 2 * c + 1], a1);
      }
      y[p2] = a0 + a1;
    }
    const int pn = (i + 2) * kT + tid;  // this thread's first row of the next step
    if (i + 1 < nb && pn < Pp) ai_row(A, tri_index(pn >> 5, i + 1), pn & 31, lv);
    __syncthreads();
  }
  {
    const int q = tid;
    if (nb > 1 && q < (nb - 1) * kT) ai_col(A, tri_index(nb - 1, q >> 5), q & 31, lv);
  }
  for (int i = nb - 1; i >= 0; --i) {
    if (warp == 0) {
      double t0 = 0.0, t1 = 0.0;
      if (all) {
        const double* D = dsm + i * kDs;
#pragma unroll
        for (int r = 0; r < kT; r += 2) {
          t0 = fma(D[r * (kT + 1) + ln], y[i * kT + r], t0);
          t1 = fma(D[(r + 1) * (kT + 1) + ln], y[i * kT + r + 1], t1);
        }
      } else {
        const double* D = Dv + static_cast<size_t>(i) * kTS;
#pragma unroll
        for (int r = 0; r < kT; r += 2) {
          t0 = fma(D[r * kLd + ln], y[i * kT + r], t0);
          t1 = fma(D[(r + 1) * kLd + ln], y[i * kT + r + 1], t1);
        }
      }
      __syncwarp();
      y[i * kT + ln] = t0 + t1;
    }
    __syncthreads();
    const int q = tid;
    if (q < i * kT) {
      double a0 = y[q], a1 = 0.0;
#pragma unroll
      for (int r = 0; r < kT; r += 2) {
        a0 = fma(-lv[r], y[i * kT + r], a0);
        a1 = fma(-lv[r + 1], y[i * kT + r + 1], a1);
      }
      y[q] = a0 + a1;
    }
    for (int q2 = q + kAiThreads; q2 < i * kT; q2 += kAiThreads) {
      double c2[kT];
      ai_col(A, tri_index(i, q2 >> 5), q2 & 31, c2);
      double a0 = y[q2], a1 = 0.0;
#pragma unroll
      for (int r = 0; r < kT; r += 2) {
        a0 = fma(-c2[r], y[i * kT + r], a0);
        a1 = fma(-c2[r + 1], y[i * kT + r + 1], a1);
      }
      y[q2] = a0 + a1;
    }
    if (i >= 1 && q < (i - 1) * kT) ai_col(A, tri_index(i - 1, q >> 5), q & 31, lv);
    __syncthreads();
  }
  for (int q = tid; q < P; q += blockDim.x) out[q] = y[q];
}

void launch_apply_inverse(cudaStream_t st, const SolveBatch& b, int s, const double* v, double* out) {
  const int Pp = solve_pp(b.P), nb = Pp / kT, ne = solve_ep(b.nf, b.r) / kT;
  const double* A = b.A + static_cast<size_t>(s) * solve_sys_doubles(b.P, b.nf, b.r);
  const double* Dv = A + static_cast<size_t>(nb * (nb + 1) / 2 + ne * nb) * kTS;
  const int smem = apply_inverse_smem(nb);
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_apply_inverse), smem);
  k_apply_inverse<<<1, kAiThreads, smem, st>>>(A, Dv, b.P, Pp, v, out);
  DGPU_LAUNCH("k_apply_inverse");
}

}  // namespace dgpu
