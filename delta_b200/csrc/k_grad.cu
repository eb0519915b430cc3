// Weighted chi^2 of the spatially varying kernel model and its adjoints.
//
// The model is the subtraction's (src/subtract.cpp:466-639) with two more
// parameters, a sub-pixel shift d = (dx, dy) of the kernel and a photometric
// scale s:
//   M(x) = s * sum_c a_c(x) C_c(x) + b(x),   C_c = K_c^d (*) R~,
//   K_c^d(u, v) = g_nx(u - dx) g_ny(v - dy),
// with the reference sanitised as the subtraction does (masked / non-finite
// pixels -> the fill value, off-frame -> 0) and a_c, b blended from the coarse
// lattice of theta. The objective is chi^2 = sum_x W(x) (S(x) - M(x))^2 over
// pixels with W > 0 and a finite S.
//
// k_chi2_tile (one CTA per 32 x 16 output tile) recomputes, from the staged
// reference window, the x passes with g and g' and the y passes of every
// component for C_c, C^x_c = g'_nx g_ny (*) R~ and C^y_c = g_nx g'_ny (*) R~
// (so dC_c/ddx = -C^x_c, dC_c/ddy = -C^y_c): the N_basis convolved images are
// never stored. Per pixel, with rbar = -2 W (S - M):
//   dchi2/ds   += rbar sum_c a_c C_c
//   dchi2/ddx  -= rbar s sum_c a_c C^x_c     (dy alike)
//   q_c(x)      = rbar s C_c (c < nc),  q_nc = rbar   (dchi2/da_c(x))
// chi^2 and the scalar gradients are reduced per CTA in FP64 and summed in a
// fixed order. q is written out (nf values per pixel) for the field adjoint.
//
// k_theta_grad: dchi2/dtheta_{c,j} = sum_x q_c(x) D_j(x), where D_j(x) is the
// same lattice blend applied to the j-th design function (the fields of the
// identity theta): the adjoint of the lattice evaluation and blend.
//
// k_adjoint_reference: dchi2/dR(y) = sum_c sum_u K_c^d(u) p(y + u) a_c(y + u)
// with p = rbar s: the correlation of the field-weighted residual with the
// flipped kernel field, zero where the reference was replaced by the fill
// value (which is held constant).
#include <cuda_runtime.h>

#include <algorithm>

#include "dev_common.cuh"
#include "grad_internal.h"

namespace dgpu {

constexpr int kGTW = 32;  // tile width
constexpr int kGTH = 16;  // tile height
constexpr int kGThreads = 256;

namespace {

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace

size_t chi2_tile_smem(int n_max, int ks) {
  const int kh = (ks - 1) / 2, nx = n_max + 1;
  const int nrows = kGTH + 2 * kh, wcols = kGTW + 2 * kh;
  return sizeof(float) * (static_cast<size_t>(nrows) * wcols + 2 * static_cast<size_t>(nx) * nrows * kGTW +
                          4 * static_cast<size_t>(nx) * ks);
}

__global__ void __launch_bounds__(kGThreads) k_chi2_tile(Chi2Args a) {
  extern __shared__ __align__(16) float smem[];
  const int ks = a.ks, kh = (ks - 1) / 2, nx = a.n_max + 1;
  const int nrows = kGTH + 2 * kh, wcols = kGTW + 2 * kh;
  float* win = smem;                                        // nrows x wcols
  float* tx = win + nrows * wcols;                          // nx x nrows x 32: g_nx (*)_x R~
  float* tdx = tx + nx * nrows * kGTW;                      // nx x nrows x 32: g'_nx (*)_x R~
  float* gx = tdx + nx * nrows * kGTW;                      // nx x ks
  float* dgx = gx + nx * ks;
  float* gy = dgx + nx * ks;
  float* dgy = gy + nx * ks;
  const int bx = blockIdx.x * kGTW, by = blockIdx.y * kGTH, tid = threadIdx.x;
  const int w = a.w, h = a.h;
  const float fill = *a.fill;
  for (int i = tid; i < nx * ks; i += blockDim.x) {
    gx[i] = a.gx[i];
    dgx[i] = a.dgx[i];
    gy[i] = a.gy[i];
    dgy[i] = a.dgy[i];
  }
  for (int i = tid; i < nrows * wcols; i += blockDim.x) {
    const int r = i / wcols, c = i - r * wcols;
    const int yy = by - kh + r, xx = bx - kh + c;
    float v = 0.0f;
    if (yy >= 0 && yy < h && xx >= 0 && xx < w) {
      const size_t idx = static_cast<size_t>(yy) * w + xx;
      v = __ldg(a.ref + idx);
      if ((a.rmask && __ldg(a.rmask + idx) != 0) || !isfinite(v)) v = fill;
    }
    win[i] = v;
  }
  __syncthreads();
  // x passes: tx[q][r][lx] = sum_j g_q[j] R~[r][lx + 2kh - j] (and tdx with g').
  for (int it = tid; it < nrows * kGTW; it += blockDim.x) {
    const int r = it / kGTW, lx = it - r * kGTW;
    const float* row = win + r * wcols + lx + 2 * kh;
    float acc[kGradMaxNx], accd[kGradMaxNx];
#pragma unroll
    for (int q = 0; q < kGradMaxNx; ++q) acc[q] = accd[q] = 0.0f;
    for (int j = 0; j < ks; ++j) {
      const float v = row[-j];
#pragma unroll
      for (int q = 0; q < kGradMaxNx; ++q) {
        if (q < nx) {
          acc[q] = fmaf(gx[q * ks + j], v, acc[q]);
          accd[q] = fmaf(dgx[q * ks + j], v, accd[q]);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kGradMaxNx; ++q) {
      if (q < nx) {
        tx[(q * nrows + r) * kGTW + lx] = acc[q];
        tdx[(q * nrows + r) * kGTW + lx] = accd[q];
      }
    }
  }
  __syncthreads();
  double chi = 0.0, g_s = 0.0, g_dx = 0.0, g_dy = 0.0;
  const int lx = tid % kGTW;
  const float s = a.scale;
  const size_t N = static_cast<size_t>(w) * h;
  for (int ly = tid / kGTW; ly < kGTH; ly += kGThreads / kGTW) {
    const int x = bx + lx, y = by + ly;
    if (x >= w || y >= h) continue;
    const size_t idx = static_cast<size_t>(y) * w + x;
    float m0 = 0.0f, mx = 0.0f, my = 0.0f;
    float cv[kGradMaxNc];  // C_c of this pixel, kept for q
    // per component: C, C^x, C^y at (lx, ly): buffer row ly + 2kh - j.
    for (int c = 0; c < a.nc; ++c) {
      const int2 o = a.orders[c];
      const float* col = tx + (o.x * nrows + ly + 2 * kh) * kGTW + lx;
      const float* cold = tdx + (o.x * nrows + ly + 2 * kh) * kGTW + lx;
      const float* g = gy + o.y * ks;
      const float* dg = dgy + o.y * ks;
      float cc = 0.0f, cx = 0.0f, cy = 0.0f;
      for (int j = 0; j < ks; ++j) {
        const float t = col[-j * kGTW];
        cc = fmaf(g[j], t, cc);
        cy = fmaf(dg[j], t, cy);
        cx = fmaf(g[j], cold[-j * kGTW], cx);
      }
      const float ac = field_point(a.F, c, x, y);
      m0 = fmaf(ac, cc, m0);
      mx = fmaf(ac, cx, mx);
      my = fmaf(ac, cy, my);
      cv[c] = cc;
    }
    const float bg = field_point(a.F, a.nc, x, y);
    const float model = fmaf(s, m0, bg);
    const float sv = __ldg(a.sci + idx);
    const float wt = __ldg(a.weight + idx);
    const bool ok = wt > 0.0f && isfinite(sv) && isfinite(model);
    const float r = ok ? sv - model : 0.0f;
    const float rb = ok ? -2.0f * wt * r : 0.0f;
    if (ok) {
      chi += static_cast<double>(wt) * static_cast<double>(r) * static_cast<double>(r);
      g_s += static_cast<double>(rb) * static_cast<double>(m0);
      g_dx -= static_cast<double>(rb) * static_cast<double>(s) * static_cast<double>(mx);
      g_dy -= static_cast<double>(rb) * static_cast<double>(s) * static_cast<double>(my);
    }
    if (a.q) {
      const float f = rb * s;
      for (int c = 0; c < a.nc; ++c) a.q[static_cast<size_t>(c) * N + idx] = f * cv[c];
      a.q[static_cast<size_t>(a.nc) * N + idx] = rb;
    }
    if (a.p) a.p[idx] = rb * s;
  }
  // Fixed-order block reduction of the four sums.
  __shared__ double red[4][kGThreads / 32];
  chi = warp_sum_d(chi);
  g_s = warp_sum_d(g_s);
  g_dx = warp_sum_d(g_dx);
  g_dy = warp_sum_d(g_dy);
  const int warp = tid >> 5;
  if ((tid & 31) == 0) {
    red[0][warp] = chi;
    red[1][warp] = g_s;
    red[2][warp] = g_dx;
    red[3][warp] = g_dy;
  }
  __syncthreads();
  if (tid < 4) {
    double t = 0.0;
    for (int i = 0; i < kGThreads / 32; ++i) t += red[tid][i];
    a.partial[static_cast<size_t>(blockIdx.y * gridDim.x + blockIdx.x) * 4 + tid] = t;
  }
}

// out[c] = sum over rows r of part[r * ncols + c], rows in order (one thread per column).
__global__ void k_sum_rows(const double* __restrict__ part, int nrows, int ncols, double* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncols) return;
  double t = 0.0;
  for (int r = 0; r < nrows; ++r) t += part[static_cast<size_t>(r) * ncols + c];
  out[c] = t;
}

constexpr int kTgChunk = 256;
constexpr int kTgStride = kTgChunk + 1;  // padded rows: a warp reads 16+ rows at one column
constexpr int kTgThreads = 512;

// Per block: sum over its pixel chunks of q_c(x) D_j(x) -> part[block][c * k + j].
__global__ void __launch_bounds__(kTgThreads) k_theta_grad(int w, int h, int nf, int k, const float* __restrict__ q,
                                                           DevFields D, double* __restrict__ part) {
  extern __shared__ __align__(16) float sm[];
  float* sq = sm;                    // nf x chunk (row stride kTgStride)
  float* sd = sq + nf * kTgStride;   // k x chunk
  const size_t N = static_cast<size_t>(w) * h;
  const int pairs = nf * k;
  double acc[(64 * 64 + kTgThreads - 1) / kTgThreads];
  const int per = (pairs + kTgThreads - 1) / kTgThreads;
  for (int i = 0; i < per; ++i) acc[i] = 0.0;
  for (size_t base = static_cast<size_t>(blockIdx.x) * kTgChunk; base < N;
       base += static_cast<size_t>(gridDim.x) * kTgChunk) {
    const int n = static_cast<int>(min(static_cast<size_t>(kTgChunk), N - base));
    __syncthreads();
    for (int i = threadIdx.x; i < nf * kTgChunk; i += blockDim.x) {
      const int c = i / kTgChunk, pp = i - c * kTgChunk;
      sq[c * kTgStride + pp] = pp < n ? q[static_cast<size_t>(c) * N + base + pp] : 0.0f;
    }
    for (int i = threadIdx.x; i < k * kTgChunk; i += blockDim.x) {
      const int j = i / kTgChunk, pp = i - j * kTgChunk;
      float v = 0.0f;
      if (pp < n) {
        const size_t idx = base + pp;
        v = field_point(D, j, static_cast<int>(idx % w), static_cast<int>(idx / w));
      }
      sd[j * kTgStride + pp] = v;
    }
    __syncthreads();
    for (int i = 0; i < per; ++i) {
      const int t = threadIdx.x + i * kTgThreads;
      if (t >= pairs) break;
      const int c = t / k, j = t - c * k;
      const float* a0 = sq + c * kTgStride;
      const float* b0 = sd + j * kTgStride;
      double s = 0.0;
      for (int pp = 0; pp < n; ++pp) s = fma(static_cast<double>(a0[pp]), static_cast<double>(b0[pp]), s);
      acc[i] += s;
    }
  }
  for (int i = 0; i < per; ++i) {
    const int t = threadIdx.x + i * kTgThreads;
    if (t < pairs) part[static_cast<size_t>(blockIdx.x) * pairs + t] = acc[i];
  }
}

size_t adjoint_ref_smem(int ks) {
  const int kh = (ks - 1) / 2;
  const int nrows = kGTH + 2 * kh, wcols = kGTW + 2 * kh;
  return sizeof(float) * (2 * static_cast<size_t>(nrows) * wcols + static_cast<size_t>(nrows) * kGTW);
}

// rbar_R(y) = sum_c sum_{u,v} g_nx(u - dx) g_ny(v - dy) (p a_c)(y + (u, v)), p = rbar s.
__global__ void __launch_bounds__(kGThreads) k_adjoint_reference(AdjRefArgs a) {
  extern __shared__ __align__(16) float smem[];
  const int ks = a.ks, kh = (ks - 1) / 2;
  const int nrows = kGTH + 2 * kh, wcols = kGTW + 2 * kh;
  float* pw = smem;                  // p over the window
  float* pc = pw + nrows * wcols;    // p * a_c over the window
  float* xb = pc + nrows * wcols;    // x correlation, nrows x 32
  const int bx = blockIdx.x * kGTW, by = blockIdx.y * kGTH, tid = threadIdx.x;
  const int w = a.w, h = a.h;
  for (int i = tid; i < nrows * wcols; i += blockDim.x) {
    const int r = i / wcols, c = i - r * wcols;
    const int yy = by - kh + r, xx = bx - kh + c;
    pw[i] = (yy >= 0 && yy < h && xx >= 0 && xx < w) ? a.p[static_cast<size_t>(yy) * w + xx] : 0.0f;
  }
  float out[kGTH / (kGThreads / kGTW)];
  constexpr int kRows = kGTH / (kGThreads / kGTW);
  for (int i = 0; i < kRows; ++i) out[i] = 0.0f;
  const int lx = tid % kGTW, ly0 = tid / kGTW;
  for (int c = 0; c < a.nc; ++c) {
    const int2 o = a.orders[c];
    __syncthreads();
    for (int i = tid; i < nrows * wcols; i += blockDim.x) {
      const int r = i / wcols, cc = i - r * wcols;
      const int yy = by - kh + r, xx = bx - kh + cc;
      const float v = pw[i];
      pc[i] = (v != 0.0f) ? v * field_point(a.F, c, xx, yy) : 0.0f;
    }
    __syncthreads();
    // x correlation: xb[r][lx] = sum_j g_nx[j] pc[r][lx + j] (offset u = j - kh).
    const float* g = a.gx + o.x * ks;
    for (int it = tid; it < nrows * kGTW; it += blockDim.x) {
      const int r = it / kGTW, l = it - r * kGTW;
      const float* row = pc + r * wcols + l;
      float acc = 0.0f;
      for (int j = 0; j < ks; ++j) acc = fmaf(__ldg(g + j), row[j], acc);
      xb[r * kGTW + l] = acc;
    }
    __syncthreads();
    const float* gyy = a.gy + o.y * ks;
    for (int i = 0; i < kRows; ++i) {
      const int ly = ly0 + i * (kGThreads / kGTW);
      float acc = out[i];
      for (int j = 0; j < ks; ++j) acc = fmaf(__ldg(gyy + j), xb[(ly + j) * kGTW + lx], acc);
      out[i] = acc;
    }
  }
  for (int i = 0; i < kRows; ++i) {
    const int x = bx + lx, y = by + ly0 + i * (kGThreads / kGTW);
    if (x >= w || y >= h) continue;
    const size_t idx = static_cast<size_t>(y) * w + x;
    const float rv = __ldg(a.ref + idx);
    const bool replaced = (a.rmask && __ldg(a.rmask + idx) != 0) || !isfinite(rv);
    a.out[idx] = replaced ? 0.0f : out[i];
  }
}

void launch_chi2_tile(cudaStream_t st, const Chi2Args& a) {
  const dim3 grid(ceil_div(a.w, kGTW), ceil_div(a.h, kGTH));
  const size_t smem = chi2_tile_smem(a.n_max, a.ks);
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_chi2_tile), smem);
  k_chi2_tile<<<grid, kGThreads, smem, st>>>(a);
  DGPU_LAUNCH("k_chi2_tile");
}

int chi2_tile_blocks(int w, int h) { return ceil_div(w, kGTW) * ceil_div(h, kGTH); }

void launch_sum_rows(cudaStream_t st, const double* part, int nrows, int ncols, double* out) {
  k_sum_rows<<<ceil_div(ncols, 128), 128, 0, st>>>(part, nrows, ncols, out);
  DGPU_LAUNCH("k_sum_rows");
}

int theta_grad_blocks() { return 148 * 2; }

void launch_theta_grad(cudaStream_t st, int w, int h, int nf, int k, const float* q, const DevFields& D,
                       double* part) {
  if (nf * k > 64 * 64) fail(DGPU_ERR_INVALID, "gradient: too many field coefficients");
  const size_t smem = sizeof(float) * static_cast<size_t>(nf + k) * kTgStride;
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_theta_grad), smem);
  k_theta_grad<<<theta_grad_blocks(), kTgThreads, smem, st>>>(w, h, nf, k, q, D, part);
  DGPU_LAUNCH("k_theta_grad");
}

void launch_adjoint_reference(cudaStream_t st, const AdjRefArgs& a) {
  const dim3 grid(ceil_div(a.w, kGTW), ceil_div(a.h, kGTH));
  const size_t smem = adjoint_ref_smem(a.ks);
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_adjoint_reference), smem);
  k_adjoint_reference<<<grid, kGThreads, smem, st>>>(a);
  DGPU_LAUNCH("k_adjoint_reference");
}

}  // namespace dgpu
