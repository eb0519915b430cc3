// Stamp fit kernels (reference src/fit.cpp:63-511, src/solve.cpp:70-145):
//   * per-stamp gather: sanitised reference patch (stamp + kernel halo, clipped
//     to the frame), per-stamp separable B_n in shared memory, pixel validity,
//     row emission into fixed per-stamp slots (stamp-major, then y, then x --
//     the reference's merged row order);
//   * thin-plate design rows (FP64);
//   * normal equations in the Kronecker-packed form
//       M[(c,m),(c',m')] = G[{c,c'}][{m,m'}],
//       G = sum_i w_i vec(b_i b_i^T)_sym vec(d_i d_i^T)_sym^T,  b_i = [bn_i, 1],
//     a (nf(nf+1)/2) x N x (k(k+1)/2) contraction -- 1.8x fewer products than
//     the P x P rank update -- in FP64 or FP32 SIMT with FP64 split-K reduction;
//   * rhs / ywy / active-row count, and the FP64 residual right-hand side
//     X^T W (t - X theta) used by the refinement step;
//   * per-stamp chi^2 and the K^2 (x) Var_c reweight with K frozen at each stamp
//     centre (src/fit.cpp:38-59, 389-454).
#include <cuda_runtime.h>

#include <algorithm>

#include "dev_common.cuh"
#include "fit_internal.h"

namespace dgpu {

__device__ __forceinline__ double tps_green_dev(double r2) { return r2 <= 0.0 ? 0.0 : 0.5 * r2 * log(r2); }

// design(p) = [sigma Z | 1 | u | v] (src/spatial.cpp:67-97).
__device__ void design_row_dev(const TpsDev& t, double x, double y, double* out) {
  const int k = t.k, nr = k - 3;
  const double ux = (x - t.cx) / t.scale, uy = (y - t.cy) / t.scale;
  for (int m = 0; m < nr; ++m) out[m] = 0.0;
  for (int j = 0; j < k; ++j) {
    const double dx = ux - t.kn[2 * j], dy = uy - t.kn[2 * j + 1];
    const double s = tps_green_dev(dx * dx + dy * dy);
    for (int m = 0; m < nr; ++m) out[m] = fma(s, t.z[j * nr + m], out[m]);
  }
  out[nr] = 1.0;
  out[nr + 1] = ux;
  out[nr + 2] = uy;
}

// ---------------------------------------------------------------------------
// Stamp gather (src/fit.cpp:117-194).
// ---------------------------------------------------------------------------
template <int NX>
__global__ void __launch_bounds__(256)
k_stamp_gather(StampGeom g, const int* __restrict__ stamp_x, const int* __restrict__ stamp_y,
               const float* __restrict__ sci, const float* __restrict__ ref,
               const float* __restrict__ vs, const float* __restrict__ vr,
               const uint8_t* __restrict__ sm, const uint8_t* __restrict__ rm,
               const float* __restrict__ taps, const float* __restrict__ taps_y, const int2* __restrict__ orders,
               const float* __restrict__ fillp, FitRows R) {
  // taps_y: the y-pass table (the same as taps for the plain basis; a
  // different one for the shifted / derivative basis of the gradients).
  extern __shared__ __align__(16) float fsm[];
  const int s = blockIdx.x;
  const int tid = threadIdx.x;
  const size_t base = static_cast<size_t>(s) * g.SS;
  const int nc = g.nc, ks = g.ks, kh = g.r;
  for (int i = tid; i < g.SS; i += blockDim.x) {
    R.valid[base + i] = 0;
    R.t[base + i] = 0.0;
    R.vt[base + i] = 0.0;
    R.vc[base + i] = 0.0;
    R.px[base + i] = 0;
    R.py[base + i] = 0;
  }
  for (int i = tid; i < g.SS * nc; i += blockDim.x) R.bn[base * nc + i] = 0.0;
  const int cx = stamp_x[s], cy = stamp_y[s];
  const int x0 = max(0, cx - g.sr), x1 = min(g.w - 1, cx + g.sr);
  const int y0 = max(0, cy - g.sr), y1 = min(g.h - 1, cy + g.sr);
  __shared__ int s_used;
  if (tid == 0) s_used = 0;
  if (x1 < x0 || y1 < y0) {
    if (tid == 0) R.stamp_used[s] = 0;
    return;
  }
  const int ex0 = max(0, x0 - g.r), ex1 = min(g.w - 1, x1 + g.r);
  const int ey0 = max(0, y0 - g.r), ey1 = min(g.h - 1, y1 + g.r);
  const int pw = ex1 - ex0 + 1, ph = ey1 - ey0 + 1;
  const int sw = x1 - x0 + 1, shh = y1 - y0 + 1;
  float* patch = fsm;                           // ph x pw
  float* tx = patch + g.pmax * g.pmax;          // NX x ph x sw
  float* kt = tx + NX * g.pmax * g.S;           // NX x ks (x pass)
  float* kty = kt + NX * ks;                    // NX x ks (y pass)
  const float fill = *fillp;
  for (int i = tid; i < NX * ks; i += blockDim.x) {
    kt[i] = taps[i];
    kty[i] = taps_y[i];
  }
  for (int i = tid; i < ph * pw; i += blockDim.x) {
    const int yy = i / pw, xx = i - yy * pw;
    const size_t idx = static_cast<size_t>(ey0 + yy) * g.w + ex0 + xx;
    const float v = ref[idx];
    const bool bad = (rm && rm[idx] != 0) || !isfinite(v);
    patch[i] = bad ? fill : v;
  }
  __syncthreads();
  // x-pass over every patch row, stamp columns only (out-of-patch taps skipped).
  for (int i = tid; i < ph * sw; i += blockDim.x) {
    const int yy = i / sw, lx = i - yy * sw;
    const int pc = x0 - ex0 + lx;
    float acc[NX];
#pragma unroll
    for (int q = 0; q < NX; ++q) acc[q] = 0.0f;
    for (int j = 0; j < ks; ++j) {
      const int sc = pc + kh - j;
      if (sc < 0 || sc >= pw) continue;
      const float v = patch[yy * pw + sc];
#pragma unroll
      for (int q = 0; q < NX; ++q) acc[q] = __fmaf_rn(kt[q * ks + j], v, acc[q]);
    }
#pragma unroll
    for (int q = 0; q < NX; ++q) tx[(q * ph + yy) * sw + lx] = acc[q];
  }
  __syncthreads();
  int used = 0;
  for (int i = tid; i < shh * sw; i += blockDim.x) {
    const int ly = i / sw, lx = i - ly * sw;
    const int y = y0 + ly, x = x0 + lx;
    const size_t idx = static_cast<size_t>(y) * g.w + x;
    if (sm && sm[idx] != 0) continue;
    if (rm && rm[idx] != 0) continue;
    const float sv = sci[idx];
    if (!isfinite(sv)) continue;
    const double vtv = vs ? static_cast<double>(vs[idx]) : 0.0;
    const double vcv = (g.have_cvar && vr) ? static_cast<double>(vr[idx]) : 0.0;
    if (g.have_var && !(vtv + vcv > 0.0)) continue;
    const int prow = y - ey0;
    const size_t ri = base + static_cast<size_t>(y - (cy - g.sr)) * g.S + (x - (cx - g.sr));
    bool fin = true;
    for (int n = 0; n < nc; ++n) {
      const int2 o = orders[n];
      const float* ky = kty + o.y * ks;
      const float* col = tx + static_cast<size_t>(o.x) * ph * sw + lx;
      float acc = 0.0f;
      for (int j = 0; j < ks; ++j) {
        const int sr2 = prow + kh - j;
        if (sr2 < 0 || sr2 >= ph) continue;
        acc = __fmaf_rn(ky[j], col[sr2 * sw], acc);
      }
      if (!isfinite(acc)) fin = false;
      R.bn[ri * nc + n] = static_cast<double>(acc);
    }
    if (!fin) {
      for (int n = 0; n < nc; ++n) R.bn[ri * nc + n] = 0.0;
      continue;
    }
    R.valid[ri] = 1;
    R.t[ri] = static_cast<double>(sv);
    R.vt[ri] = vtv;
    R.vc[ri] = vcv;
    R.px[ri] = x;
    R.py[ri] = y;
    used = 1;
  }
  if (used) atomicOr(&s_used, 1);
  __syncthreads();
  if (tid == 0) R.stamp_used[s] = s_used;
}

template <int NX>
static void launch_gather_t(cudaStream_t st, const StampGeom& g, size_t smem, int n_stamps,
                            const int* sx, const int* sy, const float* sci, const float* ref,
                            const float* vs, const float* vr, const uint8_t* sm, const uint8_t* rm,
                            const float* taps, const float* taps_y, const int2* orders, const float* fill,
                            const FitRows& R) {
  auto kern = k_stamp_gather<NX>;
  ensure_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
  kern<<<n_stamps, 256, smem, st>>>(g, sx, sy, sci, ref, vs, vr, sm, rm, taps, taps_y, orders, fill, R);
  DGPU_LAUNCH("k_stamp_gather");
}

void launch_stamp_gather(cudaStream_t st, const StampGeom& g, int n_stamps, const int* sx, const int* sy,
                         const float* sci, const float* ref, const float* vs, const float* vr,
                         const uint8_t* sm, const uint8_t* rm, const float* taps, const int2* orders,
                         const float* fill, const FitRows& R, const float* taps_y) {
  if (n_stamps == 0) return;
  if (taps_y == nullptr) taps_y = taps;
  const int nx = g.n_max + 1;
  const size_t smem = sizeof(float) * (static_cast<size_t>(g.pmax) * g.pmax +
                                       static_cast<size_t>(nx) * g.pmax * g.S + 2 * static_cast<size_t>(nx) * g.ks);
  if (smem > 200 * 1024) fail(DGPU_ERR_INVALID, "fit_kernel: stamp + kernel footprint too large");
  switch (nx) {
#define DGPU_G(N) case N: launch_gather_t<N>(st, g, smem, n_stamps, sx, sy, sci, ref, vs, vr, sm, rm, taps, taps_y, orders, fill, R); break;
    DGPU_G(1) DGPU_G(2) DGPU_G(3) DGPU_G(4) DGPU_G(5) DGPU_G(6) DGPU_G(7) DGPU_G(8) DGPU_G(9) DGPU_G(10) DGPU_G(11)
#undef DGPU_G
    default: fail(DGPU_ERR_INVALID, "fit_kernel: n_max above 10 is not supported");
  }
}

// Design rows + first-pass weights 1/(Var_t + Var_c) (src/fit.cpp:248-250, 282-287).
__global__ void k_design_weights(int64_t N, TpsDev t, FitRows R, int have_var) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < N;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double* d = R.d + i * t.k;
    if (!R.valid[i]) {
      for (int m = 0; m < t.k; ++m) d[m] = 0.0;
      R.w[i] = 0.0;
      continue;
    }
    design_row_dev(t, static_cast<double>(R.px[i]), static_cast<double>(R.py[i]), d);
    R.w[i] = have_var ? 1.0 / (R.vt[i] + R.vc[i]) : 1.0;
  }
}

// The same rows with the thin-plate constants in shared memory and the
// k - 3 null-space sums in registers (same FMA order per value), for k - 3 <= NR.
template <int NR>
__global__ void __launch_bounds__(256) k_design_weights_r(int64_t N, TpsDev t, FitRows R, int have_var) {
  extern __shared__ double tsm[];
  const int k = t.k, nr = k - 3;
  double* kn = tsm;       // k x 2
  double* z = tsm + 2 * k;  // k x nr
  for (int e = threadIdx.x; e < 2 * k; e += blockDim.x) kn[e] = t.kn[e];
  for (int e = threadIdx.x; e < k * nr; e += blockDim.x) z[e] = t.z[e];
  __syncthreads();
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < N;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double* d = R.d + i * k;
    if (!R.valid[i]) {
      for (int m = 0; m < k; ++m) d[m] = 0.0;
      R.w[i] = 0.0;
      continue;
    }
    const double ux = (static_cast<double>(R.px[i]) - t.cx) / t.scale, uy = (static_cast<double>(R.py[i]) - t.cy) / t.scale;
    double acc[NR];
#pragma unroll
    for (int m = 0; m < NR; ++m) acc[m] = 0.0;
    for (int j = 0; j < k; ++j) {
      const double dx = ux - kn[2 * j], dy = uy - kn[2 * j + 1];
      const double sg = tps_green_dev(dx * dx + dy * dy);
#pragma unroll
      for (int m = 0; m < NR; ++m)
        if (m < nr) acc[m] = fma(sg, z[j * nr + m], acc[m]);
    }
#pragma unroll
    for (int m = 0; m < NR; ++m)
      if (m < nr) d[m] = acc[m];
    d[nr] = 1.0;
    d[nr + 1] = ux;
    d[nr + 2] = uy;
    R.w[i] = have_var ? 1.0 / (R.vt[i] + R.vc[i]) : 1.0;
  }
}

void launch_design_weights(cudaStream_t st, int64_t N, const TpsDev& t, const FitRows& R, int have_var) {
  const int blocks = std::max(1, static_cast<int>(std::min<int64_t>((N + 255) / 256, 148 * 8)));
  const int nr = t.k - 3;
  const size_t smem = sizeof(double) * static_cast<size_t>(t.k) * (2 + std::max(nr, 0));
  if (nr >= 0 && nr <= 16) {
    ensure_dynamic_smem(reinterpret_cast<const void*>(k_design_weights_r<16>), smem);
    k_design_weights_r<16><<<blocks, 256, smem, st>>>(N, t, R, have_var);
  } else if (nr > 16 && nr <= 32) {
    ensure_dynamic_smem(reinterpret_cast<const void*>(k_design_weights_r<32>), smem);
    k_design_weights_r<32><<<blocks, 256, smem, st>>>(N, t, R, have_var);
  } else {
    k_design_weights<<<blocks, 256, 0, st>>>(N, t, R, have_var);
  }
  DGPU_LAUNCH("k_design_weights");
}

// ---------------------------------------------------------------------------
// Kronecker-packed normal equations, SIMT (FP64 or FP32 products/accumulation).
// ---------------------------------------------------------------------------
constexpr int kNeT = 64;  // u and v tile
constexpr int kNeR = 32;  // rows per shared-memory chunk

template <typename T>
__global__ void __launch_bounds__(256)
k_normal_kron(int64_t N, int nc, int k, int SS, FitRows R, const uint8_t* __restrict__ accepted,
              const int2* __restrict__ upairs, int Mu, const int2* __restrict__ vpairs, int Nv,
              int64_t rows_per_split, double* __restrict__ gpart) {
  __shared__ T Us[kNeR][kNeT + 1];
  __shared__ T Vs[kNeR][kNeT + 1];
  const int u0 = blockIdx.x * kNeT, v0 = blockIdx.y * kNeT;
  const int64_t rbeg = static_cast<int64_t>(blockIdx.z) * rows_per_split;
  const int64_t rend = min(N, rbeg + rows_per_split);
  const int tid = threadIdx.x;
  const int tu = tid % 16, tv = tid / 16;
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
  for (int64_t r0 = rbeg; r0 < rend; r0 += kNeR) {
    for (int e = tid; e < kNeR * kNeT; e += blockDim.x) {
      const int rr = e / kNeT, cc = e - rr * kNeT;
      const int64_t row = r0 + rr;
      const bool act = row < rend && R.valid[row] && accepted[row / SS];
      T uval = T(0), vval = T(0);
      if (act) {
        const int u = u0 + cc;
        if (u < Mu) {
          const int2 p = upairs[u];
          const T b1 = p.x < nc ? static_cast<T>(R.bn[row * nc + p.x]) : T(1);
          const T b2 = p.y < nc ? static_cast<T>(R.bn[row * nc + p.y]) : T(1);
          uval = b1 * b2;
        }
        const int v = v0 + cc;
        if (v < Nv) {
          const int2 q = vpairs[v];
          const T wv = static_cast<T>(R.w[row]);
          vval = (wv * static_cast<T>(R.d[row * k + q.x])) * static_cast<T>(R.d[row * k + q.y]);
        }
      }
      Us[rr][cc] = uval;
      Vs[rr][cc] = vval;
    }
    __syncthreads();
#pragma unroll 4
    for (int rr = 0; rr < kNeR; ++rr) {
      T a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = Us[rr][tu * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Vs[rr][tv * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  double* out = gpart + static_cast<size_t>(blockIdx.z) * Mu * Nv;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int u = u0 + tu * 4 + i;
    if (u >= Mu) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int v = v0 + tv * 4 + j;
      if (v < Nv) out[static_cast<size_t>(u) * Nv + v] = static_cast<double>(acc[i][j]);
    }
  }
}

// G = sum_z gpart[z] (fixed order), then M[p][q] = G[{c,c'}][{m,m'}].
__global__ void k_reduce_g(int nsplit, int MuNv, const double* __restrict__ gpart, double* __restrict__ g) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < MuNv; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int z = 0; z < nsplit; ++z) s += gpart[static_cast<size_t>(z) * MuNv + i];
    g[i] = s;
  }
}

__device__ __forceinline__ int sym_pair(int a, int b, int n) {
  if (a > b) {
    const int t = a;
    a = b;
    b = t;
  }
  return a * n - a * (a - 1) / 2 + (b - a);
}

__global__ void k_expand_m(int nf, int k, int Nv, const double* __restrict__ g, double* __restrict__ M) {
  const int P = nf * k;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P * P; i += gridDim.x * blockDim.x) {
    const int p = i / P, q = i - p * P;
    const int c = p / k, m = p - c * k, c2 = q / k, m2 = q - c2 * k;
    M[i] = g[static_cast<size_t>(sym_pair(c, c2, nf)) * Nv + sym_pair(m, m2, k)];
  }
}

void launch_normal_equations(Context& c, int prec, int64_t N, int nc, int k, int SS, const FitRows& R,
                             const uint8_t* accepted, double* M) {
  cudaStream_t st = c.stream;
  const int nf = nc + 1;
  const int Mu = nf * (nf + 1) / 2, Nv = k * (k + 1) / 2;
  std::vector<int2> up, vp;
  for (int a = 0; a < nf; ++a)
    for (int b = a; b < nf; ++b) up.push_back(make_int2(a, b));
  for (int a = 0; a < k; ++a)
    for (int b = a; b < k; ++b) vp.push_back(make_int2(a, b));
  int2* dpairs = static_cast<int2*>(c.slot(kSlotFit10, sizeof(int2) * (Mu + Nv)));
  DGPU_CUDA(h2d_async(dpairs, up.data(), sizeof(int2) * Mu, st));
  DGPU_CUDA(h2d_async(dpairs + Mu, vp.data(), sizeof(int2) * Nv, st));
  double* g = static_cast<double*>(c.slot(kSlotFit12, sizeof(double) * static_cast<size_t>(Mu) * Nv));
  if (prec == DGPU_PREC_MIXED || prec == DGPU_PREC_TF32) {
    launch_normal_tc(c, N, nc, k, SS, R, accepted, dpairs, Mu, dpairs + Mu, Nv, kSlotFit11, g,
                     prec == DGPU_PREC_TF32);
  } else {
    const int gx = (Mu + kNeT - 1) / kNeT, gy = (Nv + kNeT - 1) / kNeT;
    // Split K (rows) so the grid covers the GPU a few times over.
    const int64_t target_splits = std::max<int64_t>(1, (148 * 6) / (gx * gy));
    int64_t rps = std::max<int64_t>(kNeR * 8, (N + target_splits - 1) / target_splits);
    rps = (rps + kNeR - 1) / kNeR * kNeR;
    const int nsplit = static_cast<int>((N + rps - 1) / rps);
    double* gpart = static_cast<double*>(c.slot(kSlotFit11, sizeof(double) * static_cast<size_t>(nsplit) * Mu * Nv));
    dim3 grid(gx, gy, nsplit);
    if (prec == DGPU_PREC_FP32)
      k_normal_kron<float><<<grid, 256, 0, st>>>(N, nc, k, SS, R, accepted, dpairs, Mu, dpairs + Mu, Nv, rps, gpart);
    else
      k_normal_kron<double><<<grid, 256, 0, st>>>(N, nc, k, SS, R, accepted, dpairs, Mu, dpairs + Mu, Nv, rps, gpart);
    DGPU_LAUNCH("k_normal_kron");
    k_reduce_g<<<std::min(148 * 4, (Mu * Nv + 255) / 256), 256, 0, st>>>(nsplit, Mu * Nv, gpart, g);
    DGPU_LAUNCH("k_reduce_g");
  }
  const int P = nf * k;
  k_expand_m<<<std::min(148 * 8, (P * P + 255) / 256), 256, 0, st>>>(nf, k, Nv, g, M);
  DGPU_LAUNCH("k_expand_m");
}

// ---------------------------------------------------------------------------
// rhs = sum_i w_i e_i (b_i (x) d_i) with e_i = t_i (plain rhs) or
// e_i = t_i - x_i . theta (FP64 refinement residual), plus ywy = sum w e^2
// and the active-row count. One CTA per row chunk, rows staged in shared memory.
// ---------------------------------------------------------------------------
constexpr int kRhsRows = 128;

// model_i = sum_c b_c (d_i . theta_c) in field order (background b = 1 last),
// with theta in shared memory and the design row in registers.
template <int KMAX>
__device__ __forceinline__ double row_model(const double* __restrict__ d_row, const double* __restrict__ b_row,
                                            int nc, int k, const double* __restrict__ th) {
  double dr[KMAX];
#pragma unroll
  for (int m = 0; m < KMAX; ++m) dr[m] = m < k ? d_row[m] : 0.0;
  double model = 0.0;
  for (int c2 = 0; c2 <= nc; ++c2) {
    const double* tc = th + c2 * k;
    double f = 0.0;
#pragma unroll
    for (int m = 0; m < KMAX; ++m)
      if (m < k) f = fma(dr[m], tc[m], f);
    const double b = c2 < nc ? b_row[c2] : 1.0;
    model = fma(f, b, model);
  }
  return model;
}

__device__ __forceinline__ double row_model_any(const double* d_row, const double* b_row, int nc, int k,
                                                const double* th) {
  if (k <= 16) return row_model<16>(d_row, b_row, nc, k, th);
  if (k <= 32) return row_model<32>(d_row, b_row, nc, k, th);
  double model = 0.0;
  for (int c2 = 0; c2 <= nc; ++c2) {
    double f = 0.0;
    for (int m = 0; m < k; ++m) f = fma(d_row[m], th[c2 * k + m], f);
    model = fma(f, c2 < nc ? b_row[c2] : 1.0, model);
  }
  return model;
}

__global__ void __launch_bounds__(256)
k_rhs(int64_t N, int nc, int k, int SS, FitRows R, const uint8_t* __restrict__ accepted,
      const double* __restrict__ theta, int64_t rows_per_split, double* __restrict__ rpart,
      double* __restrict__ ypart, long long* __restrict__ npart) {
  extern __shared__ double rsm[];
  const int nf = nc + 1, P = nf * k;
  double* sb = rsm;                       // kRhsRows x nf
  double* sd = sb + kRhsRows * nf;        // kRhsRows x k
  double* se = sd + kRhsRows * k;         // kRhsRows : w * e
  double* sy = se + kRhsRows;             // kRhsRows : w * t * t
  double* sth = sy + kRhsRows;            // P (theta, when given)
  int* sa = reinterpret_cast<int*>(sth + P);  // active flags
  const int64_t rbeg = static_cast<int64_t>(blockIdx.x) * rows_per_split;
  const int64_t rend = min(N, rbeg + rows_per_split);
  const int tid = threadIdx.x;
  if (theta)
    for (int p = tid; p < P; p += blockDim.x) sth[p] = theta[p];
  double acc[4] = {0.0, 0.0, 0.0, 0.0};  // p = tid + 256*j
  double yacc = 0.0;
  long long nacc = 0;
  for (int64_t r0 = rbeg; r0 < rend; r0 += kRhsRows) {
    for (int e = tid; e < kRhsRows * nf; e += blockDim.x) {
      const int rr = e / nf, c2 = e - rr * nf;
      const int64_t row = r0 + rr;
      double b = 0.0;
      if (row < rend) b = c2 < nc ? R.bn[row * nc + c2] : 1.0;
      sb[e] = b;
    }
    for (int e = tid; e < kRhsRows * k; e += blockDim.x) {
      const int rr = e / k, m = e - rr * k;
      const int64_t row = r0 + rr;
      sd[e] = row < rend ? R.d[row * k + m] : 0.0;
    }
    __syncthreads();
    for (int e = tid; e < kRhsRows; e += blockDim.x) {
      const int64_t row = r0 + e;
      const bool act = row < rend && R.valid[row] && accepted[row / SS];
      sa[e] = act ? 1 : 0;
      double we = 0.0, wtt = 0.0;
      if (act) {
        double t = R.t[row];
        const double wv = R.w[row];
        if (theta) t = t - row_model_any(sd + e * k, sb + e * nf, nc, k, sth);
        wtt = wv * t * t;
        we = wv * t;
      }
      se[e] = we;
      sy[e] = wtt;
    }
    __syncthreads();
    for (int j = 0; j < 4; ++j) {
      const int p = tid + 256 * j;
      if (p >= P) break;
      const int c2 = p / k, m = p - c2 * k;
      double a = acc[j];
      for (int rr = 0; rr < kRhsRows; ++rr) a = fma(se[rr] * sb[rr * nf + c2], sd[rr * k + m], a);
      acc[j] = a;
    }
    if (tid == 0)
      for (int rr = 0; rr < kRhsRows; ++rr) {
        yacc += sy[rr];
        nacc += sa[rr];
      }
    __syncthreads();
  }
  for (int j = 0; j < 4; ++j) {
    const int p = tid + 256 * j;
    if (p < P) rpart[static_cast<size_t>(blockIdx.x) * P + p] = acc[j];
  }
  if (tid == 0) {
    ypart[blockIdx.x] = yacc;
    npart[blockIdx.x] = nacc;
  }
}

// The same sums on the FP64 tensor cores (mma.sync m8n8k4) for nc + 1 <= 32
// fields and k <= 8 KT: a warp streams 32-row blocks. Refinement: the model
// terms x_i . theta of 8 rows at a time are one product of the rows' design
// values with theta (held in registers as B fragments), contracted with the
// rows' b values and reduced over the 4 lanes that share a row. The sums
// out[c][m] += sum_i (w_i e_i b_ic) d_im are a product with the rows as the
// inner dimension, 4 rows per step. Rows that are not active contribute
// exact zeros (their values are never multiplied). Each CTA adds its warps'
// sums in warp order.
__device__ __forceinline__ void dmma_884(double (&d)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

template <int KT>
__global__ void __launch_bounds__(256, KT == 2 ? 2 : 1)
k_rhs_mma(int64_t N, int nc, int k, int SS, FitRows R, const uint8_t* __restrict__ accepted,
          const double* __restrict__ theta, int64_t blocks_per_cta, double* __restrict__ rpart,
          double* __restrict__ ypart, long long* __restrict__ npart) {
  constexpr int KS = 2 * KT;  // 4-wide steps over the design values
  __shared__ double s_we[8][32];
  __shared__ double s_model[8][32];
  __shared__ double s_y[8];
  __shared__ long long s_n[8];
  extern __shared__ double red[];  // 8 x P
  const int nf = nc + 1, P = nf * k;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, q = lane >> 2, kq = lane & 3;
  double bt[4][KS];
#pragma unroll
  for (int n = 0; n < 4; ++n)
#pragma unroll
    for (int ks = 0; ks < KS; ++ks) {
      const int c = 8 * n + q, m = 4 * ks + kq;
      bt[n][ks] = (theta != nullptr && c < nf && m < k) ? theta[c * k + m] : 0.0;
    }
  double acc[4][KT][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < KT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  double yacc = 0.0;
  long long nacc = 0;
  const int64_t nblk = (N + 31) / 32;
  const int64_t b0 = static_cast<int64_t>(blockIdx.x) * blocks_per_cta;
  const int64_t b1 = min(nblk, b0 + blocks_per_cta);
  for (int64_t blk = b0 + warp; blk < b1; blk += 8) {
    const int64_t r0 = blk * 32;
    const int64_t row = r0 + lane;
    const bool act = row < N && R.valid[row] && accepted[row / SS];
    double t = 0.0, wv = 0.0;
    if (act) {
      t = R.t[row];
      wv = R.w[row];
      if (theta == nullptr) yacc = fma(wv * t, t, yacc);
      ++nacc;
    }
    if (theta != nullptr) {
#pragma unroll
      for (int rt = 0; rt < 4; ++rt) {
        const int64_t mr = r0 + rt * 8 + q;
        const bool in = mr < N;
        // This row's design values and b values first (all loads in flight).
        double dv[KS], bv[8];
#pragma unroll
        for (int ks = 0; ks < KS; ++ks) {
          const int m = 4 * ks + kq;
          dv[ks] = (in && m < k) ? R.d[mr * k + m] : 0.0;
        }
#pragma unroll
        for (int n = 0; n < 4; ++n)
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const int c = 8 * n + 2 * kq + i;
            bv[2 * n + i] = !in ? 0.0 : (c < nc ? R.bn[mr * nc + c] : (c == nc ? 1.0 : 0.0));
          }
        double qa[4][2];
#pragma unroll
        for (int n = 0; n < 4; ++n) qa[n][0] = qa[n][1] = 0.0;
#pragma unroll
        for (int ks = 0; ks < KS; ++ks)
#pragma unroll
          for (int n = 0; n < 4; ++n) dmma_884(qa[n], dv[ks], bt[n][ks]);
        double part = 0.0;
#pragma unroll
        for (int n = 0; n < 4; ++n)
#pragma unroll
          for (int i = 0; i < 2; ++i) part = fma(bv[2 * n + i], qa[n][i], part);
        part += __shfl_xor_sync(0xffffffffu, part, 1);
        part += __shfl_xor_sync(0xffffffffu, part, 2);
        if (kq == 0) s_model[warp][rt * 8 + q] = part;
      }
      __syncwarp();
      if (act) {
        t = t - s_model[warp][lane];
        yacc = fma(wv * t, t, yacc);
      }
    }
    s_we[warp][lane] = act ? wv * t : 0.0;
    __syncwarp();
    // Two 4-row steps per round: all eight operand loads of a round are in
    // flight before its products.
#pragma unroll 1
    for (int ks0 = 0; ks0 < 8; ks0 += 2) {
      double a[2][4], bb[2][KT];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int rl = 4 * (ks0 + u) + kq;
        const int64_t ar = r0 + rl;
        const double we = s_we[warp][rl];
        const bool live = we != 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int c = 8 * i + q;
          a[u][i] = !live ? 0.0 : we * (c < nc ? R.bn[ar * nc + c] : (c == nc ? 1.0 : 0.0));
        }
#pragma unroll
        for (int j = 0; j < KT; ++j) {
          const int m = 8 * j + q;
          bb[u][j] = (live && m < k) ? R.d[ar * k + m] : 0.0;
        }
      }
#pragma unroll
      for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < KT; ++j) dmma_884(acc[i][j], a[u][i], bb[u][j]);
    }
    __syncwarp();
  }
  // Warp sums into shared memory, then added over the warps in order.
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < KT; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int c = 8 * i + q, m = 8 * j + 2 * kq + e;
        if (c < nf && m < k) red[warp * P + c * k + m] = acc[i][j][e];
      }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    yacc += __shfl_xor_sync(0xffffffffu, yacc, o);
    nacc += __shfl_xor_sync(0xffffffffu, nacc, o);
  }
  if (lane == 0) {
    s_y[warp] = yacc;
    s_n[warp] = nacc;
  }
  __syncthreads();
  for (int p = threadIdx.x; p < P; p += blockDim.x) {
    double v = 0.0;
    for (int w2 = 0; w2 < 8; ++w2) v += red[w2 * P + p];
    rpart[static_cast<size_t>(blockIdx.x) * P + p] = v;
  }
  if (threadIdx.x == 0) {
    double y = 0.0;
    long long n = 0;
    for (int w2 = 0; w2 < 8; ++w2) {
      y += s_y[w2];
      n += s_n[w2];
    }
    ypart[blockIdx.x] = y;
    npart[blockIdx.x] = n;
  }
}

// Sum of the per-split partials: warp w of a CTA owns unknown 8 blockIdx + w,
// its lanes stride the splits (four loads in flight), then a fixed shuffle
// tree. Block 0's last warp also sums ywy and the row count.
__global__ void __launch_bounds__(256)
k_reduce_rhs(int nsplit, int P, const double* __restrict__ rpart, const double* __restrict__ ypart,
             const long long* __restrict__ npart, double* __restrict__ rhs, double* ywy, long long* n) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int p = blockIdx.x * 8 + warp;
  if (p < P) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int z = lane;
    for (; z + 96 < nsplit; z += 128) {
      s0 += rpart[static_cast<size_t>(z) * P + p];
      s1 += rpart[static_cast<size_t>(z + 32) * P + p];
      s2 += rpart[static_cast<size_t>(z + 64) * P + p];
      s3 += rpart[static_cast<size_t>(z + 96) * P + p];
    }
    for (; z < nsplit; z += 32) s0 += rpart[static_cast<size_t>(z) * P + p];
    double s = (s0 + s1) + (s2 + s3);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) rhs[p] = s;
  }
  if (blockIdx.x == 0 && warp == 7) {
    double y = 0.0;
    long long c = 0;
    for (int z = lane; z < nsplit; z += 32) {
      y += ypart[z];
      c += npart[z];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      y += __shfl_xor_sync(0xffffffffu, y, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (lane == 0) {
      if (ywy) *ywy = y;
      if (n) *n = c;
    }
  }
}

void launch_rhs(Context& c, int64_t N, int nc, int k, int SS, const FitRows& R, const uint8_t* accepted,
                const double* theta, double* rhs, double* ywy, long long* n) {
  cudaStream_t st = c.stream;
  const int P = (nc + 1) * k;
  if (P > 1024) fail(DGPU_ERR_INVALID, "fit: more than 1024 unknowns is not supported");
  const bool mma = nc + 1 <= 32 && k <= 32;
  int nsplit;
  int64_t rps = 0, bpc = 0;
  if (mma) {
    // Row blocks of 32 spread over one wave of CTAs (two per SM with the
    // 16-wide design, one with the 32-wide), at least one block per warp.
    const int64_t nblk = (N + 31) / 32;
    const int64_t wave = 148 * (k <= 16 ? 2 : 1);
    bpc = std::max<int64_t>(8, (nblk + wave - 1) / wave);
    nsplit = static_cast<int>(std::max<int64_t>(1, (nblk + bpc - 1) / bpc));
  } else {
    rps = std::max<int64_t>(kRhsRows * 2, (N + 148 * 2 - 1) / (148 * 2));
    rps = (rps + kRhsRows - 1) / kRhsRows * kRhsRows;
    nsplit = static_cast<int>(std::max<int64_t>(1, (N + rps - 1) / rps));
  }
  char* buf = static_cast<char*>(c.slot(kSlotFit13, (sizeof(double) * (P + 1) + sizeof(long long)) * nsplit + 64));
  double* rpart = reinterpret_cast<double*>(buf);
  double* ypart = rpart + static_cast<size_t>(nsplit) * P;
  long long* npart = reinterpret_cast<long long*>(ypart + nsplit);
  if (mma) {
    const size_t smem = sizeof(double) * 8 * static_cast<size_t>(P);
    if (k <= 16) {
      ensure_dynamic_smem(reinterpret_cast<const void*>(k_rhs_mma<2>), smem);
      k_rhs_mma<2><<<nsplit, 256, smem, st>>>(N, nc, k, SS, R, accepted, theta, bpc, rpart, ypart, npart);
    } else {
      ensure_dynamic_smem(reinterpret_cast<const void*>(k_rhs_mma<4>), smem);
      k_rhs_mma<4><<<nsplit, 256, smem, st>>>(N, nc, k, SS, R, accepted, theta, bpc, rpart, ypart, npart);
    }
    DGPU_LAUNCH("k_rhs_mma");
  } else {
    const size_t smem =
        sizeof(double) * (kRhsRows * (nc + 1) + kRhsRows * k + 2 * kRhsRows + P) + sizeof(int) * kRhsRows;
    ensure_dynamic_smem(reinterpret_cast<const void*>(k_rhs), smem);
    k_rhs<<<nsplit, 256, smem, st>>>(N, nc, k, SS, R, accepted, theta, rps, rpart, ypart, npart);
    DGPU_LAUNCH("k_rhs");
  }
  k_reduce_rhs<<<(P + 7) / 8, 256, 0, st>>>(nsplit, P, rpart, ypart, npart, rhs, ywy, n);
  DGPU_LAUNCH("k_reduce_rhs");
}

// ---------------------------------------------------------------------------
// Per-stamp chi^2 (src/fit.cpp:389-406): sum of w r^2 over the stamp's active
// rows / count; NaN for stamps without active rows. Each stamp's rows are split
// into kChi2Parts contiguous parts, one CTA each (partial sums in a fixed
// order), and k_stamp_chi2_finish adds the parts in part order.
// ---------------------------------------------------------------------------
constexpr int kChi2Parts = 4;

__global__ void __launch_bounds__(256)
k_stamp_chi2(int nc, int k, int SS, FitRows R, const uint8_t* __restrict__ accepted,
             const double* __restrict__ theta, double* __restrict__ psum, int* __restrict__ pcnt) {
  extern __shared__ double cth[];  // theta, (nc + 1) * k
  __shared__ double ssum[256];
  __shared__ int scnt[256];
  const int s = blockIdx.x, part = blockIdx.y;
  const int P = (nc + 1) * k;
  const int per = (SS + kChi2Parts - 1) / kChi2Parts;
  const int i0 = part * per, i1 = min(SS, i0 + per);
  double acc = 0.0;
  int n = 0;
  if (accepted[s]) {
    for (int p = threadIdx.x; p < P; p += blockDim.x) cth[p] = theta[p];
    __syncthreads();
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
      const size_t row = static_cast<size_t>(s) * SS + i;
      if (!R.valid[row]) continue;
      const double model = row_model_any(R.d + row * k, R.bn + row * nc, nc, k, cth);
      const double res = R.t[row] - model;
      acc += R.w[row] * res * res;
      ++n;
    }
  }
  ssum[threadIdx.x] = acc;
  scnt[threadIdx.x] = n;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < static_cast<unsigned>(o)) {
      ssum[threadIdx.x] += ssum[threadIdx.x + o];
      scnt[threadIdx.x] += scnt[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    psum[s * kChi2Parts + part] = ssum[0];
    pcnt[s * kChi2Parts + part] = scnt[0];
  }
}

__global__ void k_stamp_chi2_finish(int n_stamps, const double* __restrict__ psum, const int* __restrict__ pcnt,
                                    double* __restrict__ chi2, int* __restrict__ cnt) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_stamps) return;
  double a = 0.0;
  int n = 0;
#pragma unroll
  for (int g = 0; g < kChi2Parts; ++g) {
    a += psum[s * kChi2Parts + g];
    n += pcnt[s * kChi2Parts + g];
  }
  cnt[s] = n;
  chi2[s] = n > 0 ? a / n : __longlong_as_double(0x7ff8000000000000ll);
}

size_t stamp_chi2_scratch_bytes(int n_stamps) {
  return (sizeof(double) + sizeof(int)) * kChi2Parts * static_cast<size_t>(std::max(n_stamps, 1)) + 16;
}

void launch_stamp_chi2(cudaStream_t st, int n_stamps, int nc, int k, int SS, const FitRows& R,
                       const uint8_t* accepted, const double* theta, double* chi2, int* cnt, void* scratch) {
  if (n_stamps == 0) return;
  double* psum = static_cast<double*>(scratch);
  int* pcnt = reinterpret_cast<int*>(psum + static_cast<size_t>(kChi2Parts) * n_stamps);
  k_stamp_chi2<<<dim3(n_stamps, kChi2Parts), 256, sizeof(double) * (nc + 1) * k, st>>>(nc, k, SS, R, accepted, theta,
                                                                                       psum, pcnt);
  DGPU_LAUNCH("k_stamp_chi2");
  k_stamp_chi2_finish<<<(n_stamps + 127) / 128, 128, 0, st>>>(n_stamps, psum, pcnt, chi2, cnt);
  DGPU_LAUNCH("k_stamp_chi2_finish");
}

// ---------------------------------------------------------------------------
// IRLS reweight (src/fit.cpp:411-454): K = sum_n float(a_n(stamp centre)) phi_n
// squared elementwise; w = 1 / (Var_t + (K^2 (x) Var_c)) over each active row,
// masked / non-positive / non-finite reference variance skipped, FP64 sum in
// (dv, du) order. Science-variance only: w = 1 / Var_t.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_reweight(StampGeom g, TpsDev t, const int* __restrict__ stamp_x, const int* __restrict__ stamp_y,
           FitRows R, const uint8_t* __restrict__ accepted, const int* __restrict__ cnt,
           const double* __restrict__ theta, const float* __restrict__ phi, const float* __restrict__ vr,
           const uint8_t* __restrict__ rm) {
  extern __shared__ __align__(16) double wsmd[];
  const int s = blockIdx.x;
  if (!accepted[s] || cnt[s] == 0) return;
  const int ks = g.ks, kk = ks * ks, r = g.r;
  const int nc = g.nc;
  // K^2 and the reference-variance window as doubles (exact conversions of
  // the float values the reference multiplies).
  double* k2 = wsmd;             // kk
  double* win = wsmd + kk;       // (S + 2r)^2, invalid samples = 0
  const int side = g.S + 2 * r;
  const int wx0 = stamp_x[s] - g.sr - r, wy0 = stamp_y[s] - g.sr - r;
  __shared__ float an[64];
  __shared__ double dsh[64];
  if (g.have_cvar) {
    if (threadIdx.x == 0) {
      design_row_dev(t, static_cast<double>(stamp_x[s]), static_cast<double>(stamp_y[s]), dsh);
      for (int n = 0; n < nc; ++n) {
        double f = 0.0;
        for (int m = 0; m < t.k; ++m) f = fma(dsh[m], theta[n * t.k + m], f);
        an[n] = static_cast<float>(f);
      }
    }
    // Off-frame, masked, non-positive and non-finite samples contribute nothing
    // (src/fit.cpp:38-59 skips them): store 0, which leaves the FP64 sum unchanged.
    for (int i = threadIdx.x; i < side * side + 4; i += blockDim.x) {
      const int yy = wy0 + i / side, xx = wx0 + i % side;
      float v = 0.0f;
      if (i < side * side && yy >= 0 && yy < g.h && xx >= 0 && xx < g.w) {
        const size_t idx = static_cast<size_t>(yy) * g.w + xx;
        const float x = vr[idx];
        if (!(rm && rm[idx] != 0) && x > 0.0f && isfinite(x)) v = x;
      }
      win[i] = static_cast<double>(v);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kk; i += blockDim.x) {
      float v = 0.0f;
      for (int n = 0; n < nc; ++n) v = __fmaf_rn(an[n], phi[static_cast<size_t>(n) * kk + i], v);
      k2[i] = static_cast<double>(v * v);
    }
    __syncthreads();
  }
  if (!g.have_cvar) {
    for (int i = threadIdx.x; i < g.SS; i += blockDim.x) {
      const size_t row = static_cast<size_t>(s) * g.SS + i;
      if (R.valid[row] && R.vt[row] > 0.0) R.w[row] = 1.0 / R.vt[row];
    }
    return;
  }
  // Four horizontally adjacent rows of the stamp per thread, each an FMA
  // chain in (dv, du) order. For a fixed dv the four share one sliding run of
  // window values: one shared load per du step feeds four FMAs. Row (ly, lx)
  // of the stamp sits at window offset (ly + r) * side + lx + r.
  const int S = g.S, strips = (S + 3) / 4;
  for (int t = threadIdx.x; t < strips * S; t += blockDim.x) {
    const int ly = t / strips, lx0 = 4 * (t - ly * strips);
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int dv = -r; dv <= r; ++dv) {
      const double* krow = k2 + (dv + r) * ks;
      // window row of (y - dv); column of output q at du: lx0 + q + r - du
      const double* wrow = win + (ly + r - dv) * side + lx0;
      double w0 = wrow[2 * r], w1 = wrow[2 * r + 1], w2 = wrow[2 * r + 2], w3 = wrow[2 * r + 3];
      for (int du = -r; du <= r; ++du) {
        const double c = krow[du + r];
        acc[0] = fma(c, w0, acc[0]);
        acc[1] = fma(c, w1, acc[1]);
        acc[2] = fma(c, w2, acc[2]);
        acc[3] = fma(c, w3, acc[3]);
        if (du < r) {
          w3 = w2;
          w2 = w1;
          w1 = w0;
          w0 = wrow[r - du - 1];
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int lx = lx0 + q;
      if (lx >= S) break;
      const size_t row = static_cast<size_t>(s) * g.SS + static_cast<size_t>(ly) * S + lx;
      if (!R.valid[row]) continue;
      const double rv = R.vt[row] + acc[q];
      if (rv > 0.0) R.w[row] = 1.0 / rv;
    }
  }
}

void launch_reweight(cudaStream_t st, const StampGeom& g, int n_stamps, const TpsDev& t, const int* sx,
                     const int* sy, const FitRows& R, const uint8_t* accepted, const int* cnt,
                     const double* theta, const float* phi, const float* vr, const uint8_t* rm) {
  if (n_stamps == 0) return;
  const size_t side = static_cast<size_t>(g.S) + 2 * g.r;
  // (+4: the last window row's sliding runs of the four-row strips read up to
  // three values past it, for outputs beyond the stamp that are never stored)
  const size_t smem = sizeof(double) * (static_cast<size_t>(g.ks) * g.ks + side * side + 4);
  if (smem > 200 * 1024) fail(DGPU_ERR_INVALID, "fit_kernel: stamp plus kernel footprint too large for the reweight");
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_reweight), smem);
  k_reweight<<<n_stamps, 256, smem, st>>>(g, t, sx, sy, R, accepted, cnt, theta, phi, vr, rm);
  DGPU_LAUNCH("k_reweight");
}

}  // namespace dgpu
