// Full-frame subtraction kernels (sm_100a, FP32 SIMT):
//   * thin-plate field lattice / exact fields (FP64),
//   * fused tile model convolve D = S - b - sum_n a_n (g_ny *_y (g_nx *_x R~)),
//   * block-effective variance K^2 (x) Var(R) + Var(S),
//   * mask growth (separable OR dilation in shared memory) and exact-bad fill,
//   * radix-select upper median of a stride-7 sample (fill values).
// Reference: src/subtract.cpp:20-966.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cmath>

#include "dev_common.cuh"
#include "select_internal.h"

namespace dgpu {

// ---------------------------------------------------------------------------
// Thin-plate fields
// ---------------------------------------------------------------------------

__device__ __forceinline__ double tps_green_d(double r2) { return r2 <= 0.0 ? 0.0 : 0.5 * r2 * log(r2); }

// fields(p, f) = design(p) . theta[f*k:(f+1)*k], design = [sigma Z | 1 | u | v]
// (src/spatial.cpp:67-97, src/subtract.cpp:58-63).
__device__ void eval_fields_at(const TpsDev t, const double* __restrict__ theta, int nf, double x,
                               double y, double* out /* nf */) {
  constexpr int kMaxK = 64;
  double d[kMaxK];
  const int k = t.k, nr = k - 3;
  const double ux = (x - t.cx) / t.scale, uy = (y - t.cy) / t.scale;
  for (int m = 0; m < nr; ++m) d[m] = 0.0;
  for (int j = 0; j < k; ++j) {
    const double dx = ux - t.kn[2 * j], dy = uy - t.kn[2 * j + 1];
    const double s = tps_green_d(dx * dx + dy * dy);
    for (int m = 0; m < nr; ++m) d[m] = fma(s, t.z[j * nr + m], d[m]);
  }
  d[nr] = 1.0;
  d[nr + 1] = ux;
  d[nr + 2] = uy;
  for (int f = 0; f < nf; ++f) {
    double acc = 0.0;
    const double* th = theta + static_cast<size_t>(f) * k;
    for (int m = 0; m < k; ++m) acc = fma(d[m], th[m], acc);
    out[f] = acc;
  }
}

__global__ void k_lattice(TpsDev t, const double* __restrict__ theta, int nf,
                          const int* __restrict__ gx, const int* __restrict__ gy, int ncx, int ncy,
                          double* __restrict__ lat, float* __restrict__ latf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncx * ncy) return;
  const int ix = i % ncx, iy = i / ncx;
  double f[64];
  eval_fields_at(t, theta, nf, static_cast<double>(gx[ix]), static_cast<double>(gy[iy]), f);
  for (int q = 0; q < nf; ++q) {
    const size_t o = (static_cast<size_t>(q) * ncy + iy) * ncx + ix;
    lat[o] = f[q];
    latf[o] = static_cast<float>(f[q]);
  }
}

__global__ void k_exact_fields(TpsDev t, const double* __restrict__ theta, int nf, int w, int h,
                               float* __restrict__ full) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<int64_t>(w) * h) return;
  const int x = static_cast<int>(i % w), y = static_cast<int>(i / w);
  double f[64];
  eval_fields_at(t, theta, nf, static_cast<double>(x), static_cast<double>(y), f);
  for (int q = 0; q < nf; ++q) full[static_cast<size_t>(q) * w * h + i] = static_cast<float>(f[q]);
}

void launch_lattice(cudaStream_t s, const TpsDev& t, const double* theta, int nf, const int* gx,
                    const int* gy, int ncx, int ncy, double* lat, float* latf) {
  const int n = ncx * ncy;
  k_lattice<<<ceil_div(n, 128), 128, 0, s>>>(t, theta, nf, gx, gy, ncx, ncy, lat, latf);
  DGPU_LAUNCH("k_lattice");
}

void launch_exact_fields(cudaStream_t s, const TpsDev& t, const double* theta, int nf, int w, int h,
                         float* full) {
  const int64_t n = static_cast<int64_t>(w) * h;
  k_exact_fields<<<ceil_div(n, 128), 128, 0, s>>>(t, theta, nf, w, h, full);
  DGPU_LAUNCH("k_exact_fields");
}

// ---------------------------------------------------------------------------
// Fused model convolve (src/subtract.cpp:466-639).
//
// One CTA per 32 x TH output tile. The sanitised reference window (tile + kh
// halo, masked / non-finite -> fill, off-frame -> 0) is staged in shared
// memory; the NX = n_max+1 shared x-passes are computed into shared memory for
// the tile rows plus the y halo (each thread: 4 columns x all nx, sliding a
// 4-wide register window so every staged value is loaded once per tap); the
// y-pass of every component then runs out of shared memory with each thread
// holding 4 output rows of 2 adjacent columns in registers as float2 (taps in
// blocks of 8, the 11 row pairs a block touches in registers, one packed FMA
// per tap and row), and a_n / b are blended from the coarse lattice in
// registers, the corners re-read only when the coarse cell row changes. Per output
// pixel the accumulation order is the reference's: x taps j = 0..ks-1, then
// components in basis order, each y tap j ascending, d -= a_n * bn (FMA).
// Off-frame rows of the x-pass buffer are exact zeros, which leaves every
// clipped y sum bit-identical to the reference's jmin/jmax loop.
// ---------------------------------------------------------------------------

constexpr int kMcTW = 32;   // tile width (columns)
constexpr int kMcPad = 8;   // zero rows in front of each x-pass buffer (y-pass reads reach row -7)
constexpr int kMcYR = 4;    // output rows per thread in the y pass (2 columns each)
constexpr int kMcXPT = 4;   // output columns per thread in the x pass

// Tap rows in shared memory are padded to a multiple of 8 floats (zeros), so
// both passes read them as 16-byte vectors (the y pass reads 8 taps at j0 + 0..7).
__host__ __device__ constexpr int mc_tap_stride(int ks) { return (ks + 7) & ~7; }

struct McSmem {
  int nrows, gbw_pad, lat_nx, lat_ny, cx0, cy0;
};

template <int NX, bool STACK>
__global__ void __launch_bounds__(256)
k_model_convolve(int w, int h, const float* __restrict__ sci, const float* __restrict__ ref,
                 const uint8_t* __restrict__ rmask, DevFields F, const float* __restrict__ taps,
                 const int2* __restrict__ orders, int ks, int nc, const float* __restrict__ fillp,
                 float* __restrict__ diff, int TH) {
  // STACK == true is delta::basis_convolve (src/convolve.cpp:90-113): the raw
  // image (no sanitising), every component's B_n written to diff[n*h*w + ...].
  extern __shared__ __align__(16) float smem[];
  const int kh = (ks - 1) / 2;
  const int nrows = TH + 2 * kh;
  const int gbw = kMcTW + 2 * kh;
  const int gbw_pad = (gbw + 3) & ~3;
  const int kts = mc_tap_stride(ks);
  const int trows = nrows + kMcPad;
  float* rtile = smem;                                       // nrows x gbw_pad
  float* txs = rtile + nrows * gbw_pad;                      // NX x (kMcPad zero rows + nrows) x kMcTW
  float* ktaps = txs + NX * trows * kMcTW;                   // NX x kts (zero padded, 16-byte aligned rows)
  const int bx = blockIdx.x * kMcTW, by = blockIdx.y * TH;
  const float fill = STACK ? 0.0f : *fillp;
  const int tid = threadIdx.x;

  for (int i = tid; i < NX * kts; i += blockDim.x) {
    const int q = i / kts, j = i - q * kts;
    ktaps[i] = j < ks ? taps[q * ks + j] : 0.0f;
  }
  for (int i = tid; i < NX * kMcPad * kMcTW; i += blockDim.x) {
    const int q = i / (kMcPad * kMcTW);
    txs[q * trows * kMcTW + (i - q * kMcPad * kMcTW)] = 0.0f;
  }
  for (int i = tid; i < nrows * gbw; i += blockDim.x) {
    const int r = i / gbw, c = i - r * gbw;
    const int gy = by - kh + r, gx = bx - kh + c;
    float v = 0.0f;
    if (gy >= 0 && gy < h && gx >= 0 && gx < w) {
      const size_t idx = static_cast<size_t>(gy) * w + gx;
      v = __ldg(ref + idx);
      if (!STACK) {
        const bool bad = (rmask && __ldg(rmask + idx) != 0) || !isfinite(v);
        if (bad) v = fill;
      }
    }
    rtile[r * gbw_pad + c] = v;
  }
  __syncthreads();

  // ---- x pass: txs[nx][r][lx] = sum_j k[nx][j] * R~[y][x + kh - j] ----
  const int ngrp = kMcTW / kMcXPT;
  for (int it = tid; it < nrows * ngrp; it += blockDim.x) {
    const int r = it / ngrp, cg = it - r * ngrp;
    const int gy = by - kh + r;
    const int c0 = cg * kMcXPT;
    float acc[NX][kMcXPT];
#pragma unroll
    for (int q = 0; q < NX; ++q)
#pragma unroll
      for (int i = 0; i < kMcXPT; ++i) acc[q][i] = 0.0f;
    if (gy >= 0 && gy < h) {
      const float* row = rtile + r * gbw_pad + c0 + 2 * kh;  // column of tap j=0, output 0
      float win[kMcXPT];
#pragma unroll
      for (int i = 0; i < kMcXPT; ++i) win[i] = row[i];
      // Taps in groups of 4, one 16-byte load per component per group.
      for (int j0 = 0; j0 < ks; j0 += 4) {
        float4 kq[NX];
#pragma unroll
        for (int q = 0; q < NX; ++q) kq[q] = *reinterpret_cast<const float4*>(ktaps + q * kts + j0);
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const int j = j0 + jj;
          if (j >= ks) break;
          if (j > 0) {
#pragma unroll
            for (int i = kMcXPT - 1; i > 0; --i) win[i] = win[i - 1];
            win[0] = row[-j];
          }
#pragma unroll
          for (int q = 0; q < NX; ++q) {
            const float kc = jj == 0 ? kq[q].x : jj == 1 ? kq[q].y : jj == 2 ? kq[q].z : kq[q].w;
#pragma unroll
            for (int i = 0; i < kMcXPT; ++i) acc[q][i] = __fmaf_rn(kc, win[i], acc[q][i]);
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < NX; ++q) {
      float4 v = make_float4(acc[q][0], acc[q][1], acc[q][2], acc[q][3]);
      *reinterpret_cast<float4*>(txs + (q * trows + kMcPad + r) * kMcTW + c0) = v;
    }
  }
  __syncthreads();

  // ---- y pass + field blend: 2 adjacent columns x 4 rows per thread ----
  // Column pairs move as float2 (one 8-byte shared load per buffer row) and
  // every tap is one packed FMA (__ffma2_rn: an IEEE fma per lane, so each
  // output is the same FMA chain as a scalar loop).
  const int lx0 = 2 * (tid % (kMcTW / 2));
  const int ly0 = (tid / (kMcTW / 2)) * kMcYR;
  if (ly0 >= TH) return;
  const int x0 = bx + lx0;
  bool xin[2];
  int xcl[2];
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    xin[u] = x0 + u < w;
    xcl[u] = xin[u] ? x0 + u : w - 1;
  }
  float2 d2[kMcYR];
  int jx[2] = {0, 0};
  float wxv[2] = {0.0f, 0.0f};
  int jy[kMcYR];
  float fy[kMcYR];
  if (!STACK && !F.exact) {
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      jx[u] = F.cellx[xcl[u]];
      wxv[u] = F.wx[xcl[u]];
    }
  }
#pragma unroll
  for (int i = 0; i < kMcYR; ++i) {
    const int y = min(by + ly0 + i, h - 1);
    if (!STACK && !F.exact) {
      jy[i] = F.celly[y];
      fy[i] = F.wy[y];
    } else {
      jy[i] = 0;
      fy[i] = 0.0f;
    }
  }
  // Field values a_f(x, y_i) of both columns; the lattice corners are re-read
  // only when the coarse cell row changes.
  auto fields_of = [&](int f, float2 (&a)[kMcYR]) {
    if (F.exact) {
#pragma unroll
      for (int i = 0; i < kMcYR; ++i) {
        const int y = min(by + ly0 + i, h - 1);
        const float* fr = F.full + (static_cast<size_t>(f) * h + y) * w;
        a[i] = make_float2(__ldg(fr + xcl[0]), __ldg(fr + xcl[1]));
      }
      return;
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      int cj = -1;
      float a00 = 0.0f, a01 = 0.0f, a10 = 0.0f, a11 = 0.0f;
#pragma unroll
      for (int i = 0; i < kMcYR; ++i) {
        if (jy[i] != cj) {
          cj = jy[i];
          const float* c0 = F.latf + (static_cast<size_t>(f) * F.ncy + cj) * F.ncx + jx[u];
          const float* c1 = c0 + F.ncx;
          a00 = __ldg(c0);
          a01 = __ldg(c0 + 1);
          a10 = __ldg(c1);
          a11 = __ldg(c1 + 1);
        }
        const float v = cell_blend(a00, a01, a10, a11, fy[i], wxv[u]);
        if (u == 0) a[i].x = v; else a[i].y = v;
      }
    }
  };
  if (!STACK) {
    float2 bg[kMcYR];
    fields_of(nc, bg);
#pragma unroll
    for (int i = 0; i < kMcYR; ++i) {
      const int y = min(by + ly0 + i, h - 1);
      const float* sr = sci + static_cast<size_t>(y) * w;
      d2[i] = make_float2(__ldg(sr + xcl[0]) - bg[i].x, __ldg(sr + xcl[1]) - bg[i].y);
    }
  }
  for (int n = 0; n < nc; ++n) {
    const int2 o = orders[n];
    // Row kMcPad of the component's buffer is row 0; the pad rows above are
    // zeros, so the reads of rows -7..-1 (taps past the top of the frame) need
    // no test.
    const float2* col =
        reinterpret_cast<const float2*>(txs + (static_cast<size_t>(o.x) * trows + kMcPad) * kMcTW + lx0);
    const float* ky = ktaps + o.y * kts;
    // Output row ly0+i needs buffer row ly0 + i + 2kh - j. Taps go in blocks of
    // 8 with the rows of a block held in registers (static indices), each
    // output still summing its taps j = 0..ks-1 in order.
    const int base = ly0 + 2 * kh;
    float2 bn[kMcYR];
#pragma unroll
    for (int i = 0; i < kMcYR; ++i) bn[i] = make_float2(0.0f, 0.0f);
    for (int j0 = 0; j0 < ks; j0 += 8) {
      float2 v[kMcYR + 7];  // v[t] = buffer row base - j0 - 7 + t
      const float2* vb = col + (base - j0 - 7) * (kMcTW / 2);
#pragma unroll
      for (int t = 0; t < kMcYR + 7; ++t) v[t] = vb[t * (kMcTW / 2)];
      const float4 ka = *reinterpret_cast<const float4*>(ky + j0);
      const float4 kb = *reinterpret_cast<const float4*>(ky + j0 + 4);
      const float kv[8] = {ka.x, ka.y, ka.z, ka.w, kb.x, kb.y, kb.z, kb.w};
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) {
        if (j0 + jj < ks) {
          const float c = kv[jj];
          const float2 cc = make_float2(c, c);
#pragma unroll
          for (int i = 0; i < kMcYR; ++i) bn[i] = __ffma2_rn(cc, v[i - jj + 7], bn[i]);
        }
      }
    }
    if (STACK) {
#pragma unroll
      for (int i = 0; i < kMcYR; ++i) {
        const int y = by + ly0 + i;
        if (y >= h) continue;
        float* dr = diff + (static_cast<size_t>(n) * h + y) * w;
        if (xin[0]) dr[x0] = bn[i].x;
        if (xin[1]) dr[x0 + 1] = bn[i].y;
      }
      continue;
    }
    float2 a[kMcYR];
    fields_of(n, a);
#pragma unroll
    for (int i = 0; i < kMcYR; ++i) d2[i] = __ffma2_rn(make_float2(-a[i].x, -a[i].y), bn[i], d2[i]);
  }
  if constexpr (!STACK) {
#pragma unroll
    for (int i = 0; i < kMcYR; ++i) {
      const int y = by + ly0 + i;
      if (y >= h) continue;
      const size_t o = static_cast<size_t>(y) * w + x0;
      if (xin[0] && xin[1] && (o & 1) == 0) {
        *reinterpret_cast<float2*>(diff + o) = d2[i];
      } else {
        if (xin[0]) diff[o] = d2[i].x;
        if (xin[1]) diff[o + 1] = d2[i].y;
      }
    }
  }
}

template <int NX, bool STACK>
static void launch_mc(cudaStream_t s, const SubtractArgs& a, const int2* orders, int TH, size_t smem) {
  auto kern = k_model_convolve<NX, STACK>;
  ensure_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
  dim3 grid(ceil_div(a.w, kMcTW), ceil_div(a.h, TH));
  const int threads = (kMcTW / 2) * (TH / kMcYR);
  kern<<<grid, threads, smem, s>>>(a.w, a.h, a.sci, a.ref, a.ref_mask, a.F, a.taps, orders, a.ks,
                                   a.nc, a.fill, a.diff, TH);
  DGPU_LAUNCH("k_model_convolve");
}

size_t model_convolve_smem(int nx, int ks, int TH) {
  const int kh = (ks - 1) / 2;
  const int nrows = TH + 2 * kh;
  const int gbw_pad = ((kMcTW + 2 * kh) + 3) & ~3;
  return sizeof(float) * (static_cast<size_t>(nrows) * gbw_pad +
                          static_cast<size_t>(nx) * (nrows + kMcPad) * kMcTW + static_cast<size_t>(nx) * mc_tap_stride(ks));
}

size_t model_convolve_fast_smem(int nx, int ks, int TH, const DevFields& F);
bool model_convolve_fast_available(int nx, int ks);
bool launch_model_convolve_fast(cudaStream_t s, const SubtractArgs& a, const int2* orders, int TH);

static void launch_mc_th(cudaStream_t s, const SubtractArgs& a, const int2* orders, bool stack, int TH) {
  const int nx = a.n_max + 1;
  // The common basis shapes run the compile-time-shaped kernel (same bits;
  // DELTA_MODEL_CONVOLVE_GENERIC=1 forces this generic one, a diagnostic the
  // tests use to compare the two).
  const char* generic = std::getenv("DELTA_MODEL_CONVOLVE_GENERIC");
  if (!stack && !(generic && generic[0] == '1') && launch_model_convolve_fast(s, a, orders, TH)) return;
  const size_t smem = model_convolve_smem(nx, a.ks, TH);
  switch (nx) {
    case 1: stack ? launch_mc<1, true>(s, a, orders, TH, smem) : launch_mc<1, false>(s, a, orders, TH, smem); break;
    case 2: stack ? launch_mc<2, true>(s, a, orders, TH, smem) : launch_mc<2, false>(s, a, orders, TH, smem); break;
    case 3: stack ? launch_mc<3, true>(s, a, orders, TH, smem) : launch_mc<3, false>(s, a, orders, TH, smem); break;
    case 4: stack ? launch_mc<4, true>(s, a, orders, TH, smem) : launch_mc<4, false>(s, a, orders, TH, smem); break;
    case 5: stack ? launch_mc<5, true>(s, a, orders, TH, smem) : launch_mc<5, false>(s, a, orders, TH, smem); break;
    case 6: stack ? launch_mc<6, true>(s, a, orders, TH, smem) : launch_mc<6, false>(s, a, orders, TH, smem); break;
    case 7: stack ? launch_mc<7, true>(s, a, orders, TH, smem) : launch_mc<7, false>(s, a, orders, TH, smem); break;
    case 8: stack ? launch_mc<8, true>(s, a, orders, TH, smem) : launch_mc<8, false>(s, a, orders, TH, smem); break;
    case 9: stack ? launch_mc<9, true>(s, a, orders, TH, smem) : launch_mc<9, false>(s, a, orders, TH, smem); break;
    case 10: stack ? launch_mc<10, true>(s, a, orders, TH, smem) : launch_mc<10, false>(s, a, orders, TH, smem); break;
    case 11: stack ? launch_mc<11, true>(s, a, orders, TH, smem) : launch_mc<11, false>(s, a, orders, TH, smem); break;
    default: fail(DGPU_ERR_INVALID, "subtract: n_max above 10 is not supported by the tile engine");
  }
}

// The tile height is autotuned per (components, kernel size, frame size class):
// each height gives the same bits (the per-pixel order of every sum is fixed),
// only the redundant x-pass halo and the CTAs per SM differ. The first
// candidate is the heuristic: the tallest tile that still lets two CTAs share
// an SM, otherwise the tallest that fits.
void launch_model_convolve_orders(cudaStream_t s, const SubtractArgs& a, const int2* orders, bool stack) {
  const int nx = a.n_max + 1;
  const bool fast = !stack && model_convolve_fast_available(nx, a.ks);
  auto smem_of = [&](int th) { return fast ? model_convolve_fast_smem(nx, a.ks, th, a.F) : model_convolve_smem(nx, a.ks, th); };
  const size_t kTwoPerSm = 112 * 1024, kMaxSmem = 200 * 1024;
  int TH = 64;
  while (TH > 8 && smem_of(TH) > kTwoPerSm) TH /= 2;
  if (smem_of(TH) > kTwoPerSm) {
    TH = 64;
    while (TH > 8 && smem_of(TH) > kMaxSmem) TH /= 2;
  }
  if (smem_of(TH) > kMaxSmem) fail(DGPU_ERR_INVALID, "subtract: kernel footprint too large for the tile engine");
  std::vector<int> cands{TH};
  for (int t : {64, 32, 16})
    if (t != TH && smem_of(t) <= kMaxSmem) cands.push_back(t);
  int size_class = 0;
  for (int64_t px = static_cast<int64_t>(a.w) * a.h; px > 1; px >>= 2) ++size_class;
  // DELTA_MODEL_CONVOLVE_TH forces one candidate (a diagnostic: the tests
  // check that every tile height gives the same bits).
  if (const char* f = std::getenv("DELTA_MODEL_CONVOLVE_TH")) {
    const int th = std::atoi(f);
    if (std::find(cands.begin(), cands.end(), th) != cands.end()) {
      launch_mc_th(s, a, orders, stack, th);
      return;
    }
  }
  const std::string key = std::string("model_convolve") + (stack ? "/stack" : fast ? "/fast" : "") + "/nx" +
                          std::to_string(nx) +
                          "/ks" + std::to_string(a.ks) + "/px4^" + std::to_string(size_class);
  autotune(s, key, cands, [&](int th) { launch_mc_th(s, a, orders, stack, th); });
}

// ---------------------------------------------------------------------------
// Variance propagation (src/subtract.cpp:641-824): per 64x64 block, K frozen at
// the block centre, squared and mirrored, footprint shrunk to the centred box
// holding (1 - 1e-4f) of sum K^2, flat-window shortcut Q * Var(R) when the
// window's (max - min) <= 1e-3f * max, otherwise the dense correlation in
// (ly, lx) tap order; then + Var(S).
// ---------------------------------------------------------------------------

constexpr int kVarB = 64;
constexpr int kVarMaxRk = 64;

__global__ void __launch_bounds__(256)
k_variance(int w, int h, DevFields F, const float* __restrict__ phi, int rk, int nc,
           const float* __restrict__ var_s, const float* __restrict__ var_r,
           float* __restrict__ var_out) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int ks = 2 * rk + 1;
  const int kk = ks * ks;
  const int iw = kVarB + 2 * rk;
  float* kf = reinterpret_cast<float*>(smraw);        // kk, mirrored K^2
  float* k1 = kf + kk;                                // kk, K (unsquared)
  float* win = k1 + kk;                               // iw * iw
  float* an = win + iw * iw;                          // nc
  __shared__ double s_qsum;
  __shared__ double s_box[kVarMaxRk];
  __shared__ float s_min[8], s_max[8];
  const int tid = threadIdx.x;
  const int bx = blockIdx.x * kVarB, by = blockIdx.y * kVarB;
  const int bw = min(kVarB, w - bx), bh = min(kVarB, h - by);

  if (var_r != nullptr) {
    const int cpx = min(bx + bw / 2, w - 1), cpy = min(by + bh / 2, h - 1);
    for (int n = tid; n < nc; n += blockDim.x) an[n] = field_point(F, n, cpx, cpy);
    __syncthreads();
    // K at the block centre, squared, mirrored: kf[kk-1-i] = K[i]^2.
    for (int i = tid; i < kk; i += blockDim.x) {
      float k2 = 0.0f;
      for (int n = 0; n < nc; ++n) k2 = __fmaf_rn(an[n], __ldg(phi + static_cast<size_t>(n) * kk + i), k2);
      k1[i] = k2;
      kf[kk - 1 - i] = k2 * k2;
    }
    __syncthreads();
    // Warp 1, lane 0: qsum = sum_i double(K_i)^2 in index order (the squares
    // are exact in double). Warp 0: lane L sums the centred box of half-width
    // L (and L + 32) in row-major order. The other warps gather the window
    // meanwhile; every thread picks the first box reaching the target after
    // the barrier below.
    if (tid == 32) {
      double q = 0.0;
      for (int i = 0; i < kk; ++i) q = fma(static_cast<double>(k1[i]), static_cast<double>(k1[i]), q);
      s_qsum = q;
    } else if (tid < 32) {
      for (int hw = tid; hw < rk; hw += 32) {
        double box = 0.0;
        const int lo = rk - hw, hi = rk + hw;
        for (int yy = lo; yy <= hi; ++yy)
          for (int xx = lo; xx <= hi; ++xx) box += static_cast<double>(kf[yy * ks + xx]);
        s_box[hw] = box;
      }
    }
    // Gather the zero-padded window, its min / max and whether it is all finite.
    float lmin = INFINITY, lmax = -INFINITY;
    int finite = 1;
    const int iwh = bh + 2 * rk, iww = bw + 2 * rk;
    for (int i = tid; i < iwh * iww; i += blockDim.x) {
      const int r = i / iww, c = i - r * iww;
      const int gy = by - rk + r, gx = bx - rk + c;
      const float v = (gy < 0 || gy >= h || gx < 0 || gx >= w) ? 0.0f : __ldg(var_r + static_cast<size_t>(gy) * w + gx);
      win[r * iw + c] = v;
      lmin = fminf(lmin, v);
      lmax = fmaxf(lmax, v);
      finite &= isfinite(v) ? 1 : 0;
    }
    for (int o = 16; o > 0; o >>= 1) {
      lmin = fminf(lmin, __shfl_xor_sync(0xffffffffu, lmin, o));
      lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    }
    if ((tid & 31) == 0) {
      s_min[tid >> 5] = lmin;
      s_max[tid >> 5] = lmax;
    }
    // A zero tap adds an exact +-0 to a sum that is never -0 when the window is
    // finite, so the reference's zero-tap skip only matters otherwise.
    const bool all_finite = __syncthreads_and(finite) != 0;
    float wmin = s_min[0], wmax = s_max[0];
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) {
      wmin = fminf(wmin, s_min[i]);
      wmax = fmaxf(wmax, s_max[i]);
    }
    int hw = rk;
    {
      const double target = (1.0 - static_cast<double>(1e-4f)) * s_qsum;
      for (int b = 0; b < rk; ++b)
        if (s_box[b] >= target) {
          hw = b;
          break;
        }
    }
    const bool flat = wmax > 0.0f && (wmax - wmin) <= 1e-3f * wmax;
    const float q = static_cast<float>(s_qsum);
    const int lo = rk - hw, hi = rk + hw;
    // 4 x 4 outputs per thread: rows oy0 .. oy0+3, columns tx + 16 j (strided,
    // so a warp's window loads hit distinct banks). Per output the taps are
    // still accumulated in (ly, lx) order.
    const int tx = tid & 15, oy0 = (tid >> 4) * 4;
    // acc[i][p] holds columns 2p and 2p + 1 of row i as a pair: one packed FMA
    // (__ffma2_rn, an IEEE fma per lane) per tap for two columns.
    float2 acc[4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int p = 0; p < 2; ++p) acc[i][p] = make_float2(0.0f, 0.0f);
    if (flat) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int p = 0; p < 2; ++p) {
          const float* wp = win + (oy0 + i + rk) * iw + tx + 32 * p + rk;
          acc[i][p] = make_float2(q * wp[0], q * wp[16]);
        }
    } else {
      for (int r = 0; r <= 3 + 2 * hw; ++r) {
        const float* wrp = win + (oy0 + lo + r) * iw + tx;
        for (int lx = lo; lx <= hi; ++lx) {
          float2 v[2];
#pragma unroll
          for (int p = 0; p < 2; ++p) v[p] = make_float2(wrp[32 * p + lx], wrp[32 * p + 16 + lx]);
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int ly = lo + r - i;
            if (ly < lo || ly > hi) continue;
            const float c = kf[ly * ks + lx];
            if (!all_finite && c == 0.0f) continue;
            const float2 cc = make_float2(c, c);
#pragma unroll
            for (int p = 0; p < 2; ++p) acc[i][p] = __ffma2_rn(cc, v[p], acc[i][p]);
          }
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int p = 0; p < 2; ++p) acc[i][p] = make_float2(0.0f + acc[i][p].x, 0.0f + acc[i][p].y);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int oy = oy0 + i;
      if (oy >= bh) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int ox = tx + 16 * j;
        if (ox >= bw) continue;
        const size_t o = static_cast<size_t>(by + oy) * w + bx + ox;
        float v = (j & 1) ? acc[i][j >> 1].y : acc[i][j >> 1].x;
        if (var_s) v = v + __ldg(var_s + o);
        var_out[o] = v;
      }
    }
  } else {
    for (int p = tid; p < bw * bh; p += blockDim.x) {
      const int oy = p / bw, ox = p - oy * bw;
      const size_t o = static_cast<size_t>(by + oy) * w + bx + ox;
      var_out[o] = 0.0f + __ldg(var_s + o);
    }
  }
}

void launch_variance(cudaStream_t s, int w, int h, const DevFields& F, const float* phi, int rk,
                     int nc, const float* var_s, const float* var_r, float* var_out) {
  const int ks = 2 * rk + 1;
  const int iw = kVarB + 2 * rk;
  const size_t smem = sizeof(float) * (2 * static_cast<size_t>(ks) * ks + static_cast<size_t>(iw) * iw + nc + 4);
  if (smem > 200 * 1024 || rk > kVarMaxRk)
    fail(DGPU_ERR_INVALID, "subtract: kernel radius too large for the variance engine");
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_variance), smem);
  dim3 grid(ceil_div(w, kVarB), ceil_div(h, kVarB));
  k_variance<<<grid, 256, smem, s>>>(w, h, F, phi, rk, nc, var_s, var_r, var_out);
  DGPU_LAUNCH("k_variance");
}

// ---------------------------------------------------------------------------
// Mask growth (src/subtract.cpp:826-914): science-side flags 1:1, reference
// flags and saturated reference pixels OR-dilated by r (box), edge border r,
// non-finite difference. One CTA per 32x32 tile with the (32+2r)^2 grow window
// built on the fly in shared memory (x-dilate, then y-dilate).
// exact_bad records the undilated garbage pixels for the fill pass.
// ---------------------------------------------------------------------------

constexpr int kMkT = 32;

__global__ void __launch_bounds__(256)
k_mask(int w, int h, const float* __restrict__ sci, const float* __restrict__ ref,
       const uint8_t* __restrict__ sm, const uint8_t* __restrict__ rm, int has_sat, float sat, int r,
       const float* __restrict__ diff, uint8_t* __restrict__ mask_out, uint8_t* __restrict__ exact_bad) {
  extern __shared__ uint8_t msm[];
  const int gw = kMkT + 2 * r;
  uint8_t* g = msm;              // gw x gw grow sources
  uint8_t* gxr = g + gw * gw;    // gw rows x 32 cols after the x dilation
  const int bx = blockIdx.x * kMkT, by = blockIdx.y * kMkT;
  const int tid = threadIdx.x;
  const bool need_grow = (rm != nullptr) || has_sat;
  if (need_grow) {
    for (int i = tid; i < gw * gw; i += blockDim.x) {
      const int yy = i / gw, xx = i - yy * gw;
      const int gy = by - r + yy, gx = bx - r + xx;
      uint8_t v = 0;
      if (gy >= 0 && gy < h && gx >= 0 && gx < w) {
        const size_t idx = static_cast<size_t>(gy) * w + gx;
        if (rm) v |= rm[idx];
        if (has_sat && ref[idx] >= sat) v |= 2;
      }
      g[i] = v;
    }
    __syncthreads();
    for (int i = tid; i < gw * kMkT; i += blockDim.x) {
      const int yy = i / kMkT, xx = i - yy * kMkT;
      uint8_t acc = 0;
      for (int d = 0; d <= 2 * r; ++d) acc |= g[yy * gw + xx + d];
      gxr[i] = acc;
    }
    __syncthreads();
  }
  for (int i = tid; i < kMkT * kMkT; i += blockDim.x) {
    const int ly = i / kMkT, lx = i - ly * kMkT;
    const int x = bx + lx, y = by + ly;
    if (x >= w || y >= h) continue;
    const size_t idx = static_cast<size_t>(y) * w + x;
    uint8_t m = 0;
    uint8_t eb = 0;
    if (sm && sm[idx]) {
      m |= sm[idx];
      eb = 1;
    }
    if (rm && rm[idx]) eb = 1;
    if (has_sat) {
      if (ref[idx] >= sat) eb = 1;
      if (sci[idx] >= sat) {
        m |= 2;
        eb = 1;
      }
    }
    if (need_grow) {
      uint8_t acc = 0;
      for (int d = 0; d <= 2 * r; ++d) acc |= gxr[(ly + d) * kMkT + lx];
      m |= acc;
    }
    if (x < r || x >= w - r || y < r || y >= h - r) m |= 16;
    if (!isfinite(diff[idx])) {
      m |= 8;
      eb = 1;
    }
    mask_out[idx] = m;
    exact_bad[idx] = eb;
  }
}

void launch_mask(cudaStream_t s, int w, int h, const float* sci, const float* ref,
                 const uint8_t* sm, const uint8_t* rm, double saturation, int r, const float* diff,
                 uint8_t* mask_out, uint8_t* exact_bad) {
  const int gw = kMkT + 2 * r;
  const size_t smem = static_cast<size_t>(gw) * gw + static_cast<size_t>(gw) * kMkT;
  if (smem > 200 * 1024) fail(DGPU_ERR_INVALID, "subtract: kernel radius too large for mask growth");
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_mask), smem);
  dim3 grid(ceil_div(w, kMkT), ceil_div(h, kMkT));
  const int has_sat = saturation > 0.0 ? 1 : 0;
  k_mask<<<grid, 256, smem, s>>>(w, h, sci, ref, sm, rm, has_sat, static_cast<float>(saturation), r,
                                 diff, mask_out, exact_bad);
  DGPU_LAUNCH("k_mask");
}

__global__ void k_mask_fill(int64_t n, const uint8_t* __restrict__ mask,
                            const uint8_t* __restrict__ exact_bad, const float* __restrict__ fillp,
                            float* __restrict__ diff, float* __restrict__ var) {
  const float fill = *fillp;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (mask[i] != 0 && exact_bad[i]) {
      diff[i] = fill;
      if (var) var[i] = 0.0f;
    }
  }
}

void launch_mask_fill(cudaStream_t s, int64_t n, const uint8_t* mask, const uint8_t* exact_bad,
                      const float* fill, float* diff, float* var) {
  const int blocks = static_cast<int>(std::min<int64_t>(ceil_div(n, 256), 148 * 16));
  k_mask_fill<<<blocks, 256, 0, s>>>(n, mask, exact_bad, fill, diff, var);
  DGPU_LAUNCH("k_mask_fill");
}

// ---------------------------------------------------------------------------
// Upper median of a stride-7 sample by exact radix select (8 bits per pass over
// the monotone uint32 key). Matches std::nth_element(size/2) on the sample
// (src/subtract.cpp:20-51 for the reference fill, 915-945 for the difference
// fill). An empty sample yields 0.
// ---------------------------------------------------------------------------

void launch_strided_median(Context& c, int kind, int64_t n, const float* values, const uint8_t* mask,
                           float* d_result) {
  // kind 0 (reference): good finite reference pixels; kind 1 (difference):
  // unmasked finite difference pixels (mask is the grown output mask).
  (void)kind;
  cudaStream_t s = c.stream;
  const int64_t nsamp = (n + 6) / 7;
  auto* st = static_cast<RadixSelect*>(c.slot(kSlotSelect, sizeof(RadixSelect)));
  auto* keys = static_cast<uint32_t*>(c.slot(kSlotSamples, sizeof(uint32_t) * std::max<int64_t>(nsamp, 1)));
  DGPU_CUDA(cudaMemsetAsync(st, 0, sizeof(RadixSelect), s));
  launch_sample_keys(s, n, 7, values, mask, keys, st);
  launch_select_upper_median(s, st, keys, nsamp, d_result);
}

// photometric_scale (src/fit.cpp:513-530): out = sum_c float(S_c) * a_c in
// component order, fused.
__global__ void k_photometric_scale(DevFields F, const float* __restrict__ sums, int nc,
                                    float* __restrict__ out) {
  const int64_t n = static_cast<int64_t>(F.w) * F.h;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int x = static_cast<int>(i % F.w), y = static_cast<int>(i / F.w);
    float acc = 0.0f;
    for (int q = 0; q < nc; ++q) acc = __fmaf_rn(sums[q], field_point(F, q, x, y), acc);
    out[i] = acc;
  }
}

void launch_photometric_scale(cudaStream_t s, const DevFields& F, const float* sums, int nc, float* out) {
  const int64_t n = static_cast<int64_t>(F.w) * F.h;
  const int blocks = static_cast<int>(std::min<int64_t>(ceil_div(n, 256), 148 * 16));
  k_photometric_scale<<<blocks, 256, 0, s>>>(F, sums, nc, out);
  DGPU_LAUNCH("k_photometric_scale");
}

// Transients-positive sign flip of the difference (python/delta/pipeline.py:687-689),
// in place: float4 body, scalar tail.
// v = v * scale (float32 product, the scalar rounded to float first), or
// v = value everywhere when fill is set.
__global__ void k_scale_fill(int64_t n, float* __restrict__ v, float scale, int fill, float value) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    v[i] = fill ? value : v[i] * scale;
}

void launch_scale_fill(cudaStream_t s, int64_t n, float* v, float scale, bool fill, float value) {
  const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, 148 * 16));
  k_scale_fill<<<std::max(blocks, 1), 256, 0, s>>>(n, v, scale, fill ? 1 : 0, value);
  DGPU_LAUNCH("k_scale_fill");
}

__global__ void k_negate(int64_t n, float* __restrict__ v) {
  const int64_t n4 = (reinterpret_cast<uintptr_t>(v) & 15) ? 0 : n / 4;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  float4* v4 = reinterpret_cast<float4*>(v);
  for (int64_t i = t; i < n4; i += stride) {
    float4 a = v4[i];
    a.x = -a.x;
    a.y = -a.y;
    a.z = -a.z;
    a.w = -a.w;
    v4[i] = a;
  }
  for (int64_t i = 4 * n4 + t; i < n; i += stride) v[i] = -v[i];
}

void launch_negate(cudaStream_t s, int64_t n, float* v) {
  if (n <= 0) return;
  const int blocks = static_cast<int>(std::min<int64_t>(ceil_div(ceil_div(n, 4), 256), 148 * 8));
  k_negate<<<blocks, 256, 0, s>>>(n, v);
  DGPU_LAUNCH("k_negate");
}

// Device memory -> the context's mapped pinned read-back area by SM stores:
// range blockIdx.y of the list (16 bytes at a time when both ends are 16-byte
// aligned).
__global__ void k_read_back(ReadBackList l) {
  const int it = blockIdx.y;
  if (it >= l.n) return;
  const unsigned char* __restrict__ src = l.src[it];
  unsigned char* dst = l.dst[it];
  const size_t n = l.bytes[it];
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  size_t head = 0;
  if (((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15u) == 0) {
    const size_t n16 = n / 16;
    for (size_t i = t; i < n16; i += stride)
      reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(src)[i];
    head = n16 * 16;
  }
  for (size_t i = head + t; i < n; i += stride) dst[i] = src[i];
}

void launch_read_back(cudaStream_t s, const ReadBackList& l) {
  if (l.n <= 0) return;
  unsigned long long most = 0;
  for (int i = 0; i < l.n; ++i) most = std::max(most, l.bytes[i]);
  const unsigned bx = static_cast<unsigned>(std::min<unsigned long long>((most + 4095) / 4096, 32));
  k_read_back<<<dim3(std::max(bx, 1u), static_cast<unsigned>(l.n)), 256, 0, s>>>(l);
  DGPU_LAUNCH("k_read_back");
}

}  // namespace dgpu

// ---------------------------------------------------------------------------
// Median of z^2 = D^2 / Var over the good pixels, exactly as numpy's median of
// the FP64 values (python/delta/pipeline.py's _variance_rescale_factor): the
// two middle ranks (lo = (m-1)/2, hi = m/2) of the FP64 keys found by one
// 64-bit radix select (8 passes of 8-bit digits, both ranks per pass), then
// (a + b) / 2 on the host. z^2 >= 0 and finite, so the keys order as their bit
// patterns. Good pixels: Var > 0, D and Var finite, mask 0.
// ---------------------------------------------------------------------------
namespace dgpu {

__global__ void k_z2_keys(int64_t n, const float* __restrict__ d, const float* __restrict__ v,
                          const uint8_t* __restrict__ m, unsigned long long* __restrict__ keys,
                          unsigned long long* __restrict__ count) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float dv = d[i], vv = v[i];
    if (!(vv > 0.0f) || !isfinite(dv) || !isfinite(vv) || (m && m[i] != 0)) continue;
    const double x = static_cast<double>(dv);
    const double z2 = x * x / static_cast<double>(vv);
    keys[atomicAdd(count, 1ull)] = static_cast<unsigned long long>(__double_as_longlong(z2));
  }
}

// state: [0] count, [1] rank lo, [2] rank hi, [3] prefix lo, [4] prefix hi; hist: 2 x 256.
__global__ void k_z2_hist(const unsigned long long* __restrict__ keys, unsigned long long* __restrict__ state,
                          int shift, unsigned int* __restrict__ hist) {
  __shared__ unsigned int h[2][256];
  for (int i = threadIdx.x; i < 512; i += blockDim.x) h[i >> 8][i & 255] = 0;
  __syncthreads();
  const unsigned long long n = state[0];
  const unsigned long long himask = shift >= 56 ? 0ull : (~0ull << (shift + 8));
  const unsigned long long p0 = state[3] & himask, p1 = state[4] & himask;
  for (unsigned long long i = static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    const unsigned long long k = keys[i];
    const unsigned dgt = static_cast<unsigned>((k >> shift) & 0xffull);
    if ((k & himask) == p0) atomicAdd(&h[0][dgt], 1u);
    if ((k & himask) == p1) atomicAdd(&h[1][dgt], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 512; i += blockDim.x) {
    const unsigned c = h[i >> 8][i & 255];
    if (c) atomicAdd(&hist[i], c);
  }
}

__global__ void k_z2_pick(unsigned long long* __restrict__ state, int shift, unsigned int* __restrict__ hist) {
  if (threadIdx.x >= 2) return;
  const int t = threadIdx.x;
  unsigned long long rank = state[1 + t];
  unsigned long long cum = 0;
  int d = 0;
  for (; d < 256; ++d) {
    const unsigned long long c = hist[t * 256 + d];
    if (rank < cum + c) break;
    cum += c;
  }
  if (d > 255) d = 255;  // unreachable while the rank is below the count
  state[1 + t] = rank - cum;
  state[3 + t] |= static_cast<unsigned long long>(d) << shift;
}

__global__ void k_z2_init(unsigned long long* __restrict__ state) {
  if (threadIdx.x == 0) {
    const unsigned long long n = state[0];
    state[1] = n ? (n - 1) / 2 : 0;
    state[2] = n / 2;
    state[3] = 0;
    state[4] = 0;
  }
}

void launch_z2_median(cudaStream_t s, int64_t n, const float* d, const float* v, const uint8_t* m,
                      unsigned long long* keys, unsigned long long* state, unsigned int* hist) {
  DGPU_CUDA(cudaMemsetAsync(state, 0, 5 * sizeof(unsigned long long), s));
  const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, 148 * 8));
  k_z2_keys<<<std::max(blocks, 1), 256, 0, s>>>(n, d, v, m, keys, state);
  DGPU_LAUNCH("k_z2_keys");
  k_z2_init<<<1, 32, 0, s>>>(state);
  DGPU_LAUNCH("k_z2_init");
  for (int shift = 56; shift >= 0; shift -= 8) {
    DGPU_CUDA(cudaMemsetAsync(hist, 0, 512 * sizeof(unsigned int), s));
    k_z2_hist<<<std::max(blocks, 1), 256, 0, s>>>(keys, state, shift, hist);
    DGPU_LAUNCH("k_z2_hist");
    k_z2_pick<<<1, 32, 0, s>>>(state, shift, hist);
    DGPU_LAUNCH("k_z2_pick");
  }
}

}  // namespace dgpu
