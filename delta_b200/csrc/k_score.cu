// Match-filtered score (src/noise.cpp:535-632), sm_100a FP32 SIMT.
//
// score(x) = (sum_u psf(u) D(x+u)) / sqrt(var(x) * sum psf^2), zero-padded,
// 0 where var <= 0. One CTA per 64 x 32 tile; the haloed D window is staged in
// shared memory and each thread holds 8 output rows of one column in
// registers. For each staged window row the thread loads the ks values it
// needs once and applies them to every output row whose tap row matches, so
// per output the taps are accumulated in the reference's (ly, lx) order with
// fused multiply-adds, zero taps skipped exactly as the reference does.
// For the common sizes the PSF side is a template parameter and the taps live
// in constant memory, so each FMA takes its tap as an immediate constant-bank
// operand (no load); other sizes use a generic variant with taps in shared
// memory.
#include <cuda_runtime.h>

#include "dev_common.cuh"

namespace dgpu {

constexpr int kMfTW = 64;
constexpr int kMfTH = 32;
constexpr int kMfRPT = 8;
// The taps travel by value in the kernel parameter block (constant bank), so
// concurrent launches with different PSFs cannot interfere.
template <int PS>
struct PsfTaps {
  float v[PS * PS];
};

template <int PS>
__global__ void __launch_bounds__(256, 6)
k_matched_filter_t(int w, int h, const float* __restrict__ img, const float* __restrict__ var,
                   const __grid_constant__ PsfTaps<PS> c_psf, float sumpsf2,
                   float* __restrict__ out, int* __restrict__ nf_count, int* __restrict__ nf_tiles) {
  constexpr int R = PS / 2;
  constexpr int WH = kMfTH + 2 * R;
  constexpr int WW = kMfTW + 2 * R;
  __shared__ float win[WH][WW];
  const int bx = blockIdx.x * kMfTW, by = blockIdx.y * kMfTH;
  const int tid = threadIdx.x;
  int finite = 1;
  for (int i = tid; i < WH * WW; i += blockDim.x) {
    const int r = i / WW, c = i - r * WW;
    const int gy = by - R + r, gx = bx - R + c;
    const float v = (gy < 0 || gy >= h || gx < 0 || gx >= w) ? 0.0f : __ldg(img + static_cast<size_t>(gy) * w + gx);
    finite &= isfinite(v) ? 1 : 0;
    win[r][c] = v;
  }
  // With every staged value finite, a zero tap adds an exact +-0 to a sum that
  // is never -0, so skipping it (as the reference does) and not skipping it
  // give the same bits: such tiles drop the per-tap test. Tiles with a
  // non-finite value are listed for k_matched_filter_g, which keeps the test.
  if (!__syncthreads_and(finite)) {
    if (tid == 0) nf_tiles[atomicAdd(nf_count, 1)] = blockIdx.y * gridDim.x + blockIdx.x;
    return;
  }
  const int lx = tid % kMfTW;
  const int ly0 = (tid / kMfTW) * kMfRPT;
  float acc[kMfRPT];
#pragma unroll
  for (int i = 0; i < kMfRPT; ++i) acc[i] = 0.0f;
#pragma unroll
  for (int wr = 0; wr < kMfRPT + PS - 1; ++wr) {
    const float* row = &win[ly0 + wr][lx];
#pragma unroll
    for (int lx2 = 0; lx2 < PS; ++lx2) {
      const float v = row[lx2];
#pragma unroll
      for (int i = 0; i < kMfRPT; ++i) {
        const int ly = wr - i;
        if (ly >= 0 && ly < PS) acc[i] = __fmaf_rn(c_psf.v[ly * PS + lx2], v, acc[i]);
      }
    }
  }
  const int x = bx + lx;
  if (x >= w) return;
#pragma unroll
  for (int i = 0; i < kMfRPT; ++i) {
    const int y = by + ly0 + i;
    if (y >= h) break;
    const size_t o = static_cast<size_t>(y) * w + x;
    const float v = __ldg(var + o);
    out[o] = v > 0.0f ? __fdiv_rn(acc[i], __fsqrt_rn(v * sumpsf2)) : 0.0f;
  }
}

// Generic PSF sizes (taps in shared memory), and the non-finite tiles listed
// by k_matched_filter_t: with `tiles` set, CTAs stride over the *ntile listed
// tile indices instead of the grid.
__global__ void __launch_bounds__(256)
k_matched_filter_g(int w, int h, const float* __restrict__ img, const float* __restrict__ var,
                   const float* __restrict__ psf, int ps, float sumpsf2, float* __restrict__ out,
                   const int* __restrict__ ntile, const int* __restrict__ tiles) {
  extern __shared__ float sm[];
  const int r = ps / 2;
  const int wh = kMfTH + 2 * r, ww = kMfTW + 2 * r;
  float* sp = sm;              // ps*ps taps
  float* win = sp + ps * ps;   // wh x ww
  const int tid = threadIdx.x;
  const int tiles_x = (w + kMfTW - 1) / kMfTW;
  const int count = tiles ? *ntile : gridDim.x * gridDim.y;
  for (int i = tid; i < ps * ps; i += blockDim.x) sp[i] = psf[i];
  for (int t = tiles ? blockIdx.x : blockIdx.y * gridDim.x + blockIdx.x; t < count;
       t += tiles ? gridDim.x : count) {
    const int tile = tiles ? tiles[t] : t;
    const int bx = (tile % tiles_x) * kMfTW, by = (tile / tiles_x) * kMfTH;
    __syncthreads();
    for (int i = tid; i < wh * ww; i += blockDim.x) {
      const int rr = i / ww, c = i - rr * ww;
      const int gy = by - r + rr, gx = bx - r + c;
      win[i] = (gy < 0 || gy >= h || gx < 0 || gx >= w) ? 0.0f : __ldg(img + static_cast<size_t>(gy) * w + gx);
    }
    __syncthreads();
    const int lx = tid % kMfTW;
    const int ly0 = (tid / kMfTW) * kMfRPT;
    float acc[kMfRPT];
#pragma unroll
    for (int i = 0; i < kMfRPT; ++i) acc[i] = 0.0f;
    for (int wr = 0; wr < kMfRPT + ps - 1; ++wr) {
      const float* row = win + (ly0 + wr) * ww + lx;
      for (int lx2 = 0; lx2 < ps; ++lx2) {
        const float v = row[lx2];
#pragma unroll
        for (int i = 0; i < kMfRPT; ++i) {
          const int ly = wr - i;
          if (ly >= 0 && ly < ps) {
            const float p = sp[ly * ps + lx2];
            if (p != 0.0f) acc[i] = __fmaf_rn(p, v, acc[i]);
          }
        }
      }
    }
    const int x = bx + lx;
    if (x < w) {
#pragma unroll
      for (int i = 0; i < kMfRPT; ++i) {
        const int y = by + ly0 + i;
        if (y >= h) break;
        const size_t o = static_cast<size_t>(y) * w + x;
        const float v = __ldg(var + o);
        out[o] = v > 0.0f ? __fdiv_rn(acc[i], __fsqrt_rn(v * sumpsf2)) : 0.0f;
      }
    }
  }
}

template <int PS>
static void launch_mf_t(cudaStream_t s, int w, int h, const float* img, const float* var,
                        const float* psf_host, float sumpsf2, float* out, int* nf_buf) {
  PsfTaps<PS> taps;
  for (int i = 0; i < PS * PS; ++i) taps.v[i] = psf_host[i];
  dim3 grid(ceil_div(w, kMfTW), ceil_div(h, kMfTH));
  k_matched_filter_t<PS><<<grid, 256, 0, s>>>(w, h, img, var, taps, sumpsf2, out, nf_buf, nf_buf + 1);
  DGPU_LAUNCH("k_matched_filter");
}

// psf_host: the taps in host memory (template path); psf_dev: the same taps on
// the device (generic path); nf_buf: 1 + tile-count ints of device scratch for
// the list of tiles holding a non-finite value.
void launch_matched_filter(cudaStream_t s, int w, int h, const float* img, const float* var,
                           const float* psf_host, const float* psf_dev, int ps, float sumpsf2,
                           float* out, int* nf_buf) {
  const int r = ps / 2;
  const size_t smem = sizeof(float) * (static_cast<size_t>(ps) * ps +
                                       static_cast<size_t>(kMfTH + 2 * r) * (kMfTW + 2 * r));
  if (smem > 200 * 1024) fail(DGPU_ERR_INVALID, "matched_filter: psf too large");
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_matched_filter_g), smem);
  const dim3 grid(ceil_div(w, kMfTW), ceil_div(h, kMfTH));
  bool templated = true;
  DGPU_CUDA(cudaMemsetAsync(nf_buf, 0, sizeof(int), s));
  switch (ps) {
    case 3: launch_mf_t<3>(s, w, h, img, var, psf_host, sumpsf2, out, nf_buf); break;
    case 5: launch_mf_t<5>(s, w, h, img, var, psf_host, sumpsf2, out, nf_buf); break;
    case 7: launch_mf_t<7>(s, w, h, img, var, psf_host, sumpsf2, out, nf_buf); break;
    case 9: launch_mf_t<9>(s, w, h, img, var, psf_host, sumpsf2, out, nf_buf); break;
    case 11: launch_mf_t<11>(s, w, h, img, var, psf_host, sumpsf2, out, nf_buf); break;
    case 13: launch_mf_t<13>(s, w, h, img, var, psf_host, sumpsf2, out, nf_buf); break;
    case 15: launch_mf_t<15>(s, w, h, img, var, psf_host, sumpsf2, out, nf_buf); break;
    case 17: launch_mf_t<17>(s, w, h, img, var, psf_host, sumpsf2, out, nf_buf); break;
    case 19: launch_mf_t<19>(s, w, h, img, var, psf_host, sumpsf2, out, nf_buf); break;
    case 21: launch_mf_t<21>(s, w, h, img, var, psf_host, sumpsf2, out, nf_buf); break;
    default: templated = false; break;
  }
  if (templated) {
    // Listed tiles (usually none): a small persistent grid strides the list.
    k_matched_filter_g<<<148, 256, smem, s>>>(w, h, img, var, psf_dev, ps, sumpsf2, out, nf_buf, nf_buf + 1);
    DGPU_LAUNCH("k_matched_filter_g");
    return;
  }
  k_matched_filter_g<<<grid, 256, smem, s>>>(w, h, img, var, psf_dev, ps, sumpsf2, out, nullptr, nullptr);
  DGPU_LAUNCH("k_matched_filter_g");
}

}  // namespace dgpu
