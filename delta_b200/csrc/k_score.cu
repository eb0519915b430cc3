// Match-filtered score (src/noise.cpp:535-632), sm_100a FP32 SIMT.
//
// score(x) = (sum_u psf(u) D(x+u)) / sqrt(var(x) * sum psf^2), zero-padded,
// 0 where var <= 0.
//
// Common PSF sides (template PS): one CTA of 16 x 16 threads per 128 x 128
// output tile, each thread an 8 x 8 block of outputs (8 rows of 8 adjacent
// columns) in registers. The haloed D window and the taps (rows padded to a
// multiple of 4) are staged in shared memory. The thread walks the window rows
// of its block: it reads the row's 8 + PS - 1 values once (16-byte vector
// loads) and, for every output row i whose tap row ly = wr - i is in range,
// the 17-tap row ly (broadcast vector loads) and applies it to the 8 outputs
// of that row. Each output therefore accumulates its taps in the reference's
// (ly, lx) order with fused multiply-adds; the ratio of FMAs to shared loads
// is about 24 to 1, so the kernel is FP32-FMA-bound.
//
// With every staged value finite, a zero tap adds an exact +-0 to a sum that
// is never -0, so skipping it (as the reference does) and not skipping it give
// the same bits: such tiles drop the per-tap test. A tile holding a non-finite
// value is listed for k_matched_filter_g, which keeps the test. Other PSF sides
// use k_matched_filter_g for every tile.
#include <cuda_runtime.h>

#include "dev_common.cuh"

namespace dgpu {

constexpr int kMfR = 8;                 // output rows per thread
constexpr int kMfC = 8;                 // output columns per thread
constexpr int kMfTX = 16, kMfTY = 16;   // threads per CTA along x, y
constexpr int kMfBW = kMfTX * kMfC;     // tile width (128)
constexpr int kMfBH = kMfTY * kMfR;     // tile height (128)
// Tile of the generic kernel (64 x 32, one column of 8 rows per thread).
constexpr int kMfTW = 64;
constexpr int kMfTH = 32;
constexpr int kMfRPT = 8;

template <int PS>
struct MfGeom {
  static constexpr int R = PS / 2;
  static constexpr int SEG4 = (kMfC + PS - 1 + 3) / 4;      // 16-byte loads per window row per thread
  static constexpr int WW = kMfBW - kMfC + 4 * SEG4;        // staged window width (floats, multiple of 4)
  static constexpr int WH = kMfBH + PS - 1;                 // staged window height
  static constexpr int TS = (PS + 3) & ~3;                  // tap row stride
  static constexpr size_t smem = sizeof(float) * (static_cast<size_t>(WH) * WW + static_cast<size_t>(PS) * TS);
};

template <int PS>
__global__ void __launch_bounds__(kMfTX * kMfTY, 2)
k_matched_filter_t(int w, int h, const float* __restrict__ img, const float* __restrict__ var,
                   const float* __restrict__ psf, float sumpsf2, float* __restrict__ out, int* __restrict__ nf_count,
                   int* __restrict__ nf_tiles) {
  using G = MfGeom<PS>;
  extern __shared__ __align__(16) float msm[];
  float* win = msm;                  // WH x WW
  float* tap = win + G::WH * G::WW;  // PS x TS, zero padded
  const int bx = blockIdx.x * kMfBW, by = blockIdx.y * kMfBH;
  const int tid = threadIdx.x;
  for (int i = tid; i < PS * G::TS; i += blockDim.x) {
    const int r = i / G::TS, c = i - r * G::TS;
    tap[i] = c < PS ? __ldg(psf + r * PS + c) : 0.0f;
  }
  int finite = 1;
  for (int i = tid; i < G::WH * G::WW; i += blockDim.x) {
    const int r = i / G::WW, c = i - r * G::WW;
    const int gy = by - G::R + r, gx = bx - G::R + c;
    const float v = (gy < 0 || gy >= h || gx < 0 || gx >= w) ? 0.0f : __ldg(img + static_cast<size_t>(gy) * w + gx);
    finite &= isfinite(v) ? 1 : 0;
    win[i] = v;
  }
  if (!__syncthreads_and(finite)) {
    if (tid == 0) nf_tiles[atomicAdd(nf_count, 1)] = blockIdx.y * gridDim.x + blockIdx.x;
    return;
  }
  const int c0 = (tid % kMfTX) * kMfC, r0 = (tid / kMfTX) * kMfR;
  float acc[kMfR][kMfC];
#pragma unroll
  for (int i = 0; i < kMfR; ++i)
#pragma unroll
    for (int c = 0; c < kMfC; ++c) acc[i][c] = 0.0f;
#pragma unroll 1
  for (int wr = 0; wr < kMfR + PS - 1; ++wr) {
    float seg[4 * G::SEG4];
    const float4* src = reinterpret_cast<const float4*>(win + (r0 + wr) * G::WW + c0);
#pragma unroll
    for (int k = 0; k < G::SEG4; ++k) {
      const float4 q = src[k];
      seg[4 * k] = q.x;
      seg[4 * k + 1] = q.y;
      seg[4 * k + 2] = q.z;
      seg[4 * k + 3] = q.w;
    }
#pragma unroll
    for (int i = 0; i < kMfR; ++i) {
      const int ly = wr - i;
      if (ly < 0 || ly >= PS) continue;  // the same for every thread
      float t[G::TS];
      const float4* tp = reinterpret_cast<const float4*>(tap + ly * G::TS);
#pragma unroll
      for (int k = 0; k < G::TS / 4; ++k) {
        const float4 q = tp[k];
        t[4 * k] = q.x;
        t[4 * k + 1] = q.y;
        t[4 * k + 2] = q.z;
        t[4 * k + 3] = q.w;
      }
#pragma unroll
      for (int lx = 0; lx < PS; ++lx)
#pragma unroll
        for (int c = 0; c < kMfC; ++c) acc[i][c] = __fmaf_rn(t[lx], seg[c + lx], acc[i][c]);
    }
  }
#pragma unroll
  for (int i = 0; i < kMfR; ++i) {
    const int y = by + r0 + i;
    if (y >= h) break;
#pragma unroll
    for (int c = 0; c < kMfC; ++c) {
      const int x = bx + c0 + c;
      if (x < w) {
        const size_t o = static_cast<size_t>(y) * w + x;
        const float v = __ldg(var + o);
        out[o] = v > 0.0f ? __fdiv_rn(acc[i][c], __fsqrt_rn(v * sumpsf2)) : 0.0f;
      }
    }
  }
}

// Generic PSF sizes (taps in shared memory), and the non-finite tiles listed
// by k_matched_filter_t: with `tiles` set, CTAs stride over the 64 x 32
// sub-tiles of the *ntile listed 128 x 128 tiles instead of the grid.
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
  constexpr int kSubX = kMfBW / kMfTW, kSub = kSubX * (kMfBH / kMfTH);
  const int tiles_x = (w + kMfTW - 1) / kMfTW;
  const int big_x = (w + kMfBW - 1) / kMfBW;
  const int count = tiles ? *ntile * kSub : gridDim.x * gridDim.y;
  for (int i = tid; i < ps * ps; i += blockDim.x) sp[i] = psf[i];
  for (int t = tiles ? blockIdx.x : blockIdx.y * gridDim.x + blockIdx.x; t < count;
       t += tiles ? gridDim.x : count) {
    int bx, by;
    if (tiles) {
      const int big = tiles[t / kSub], sub = t % kSub;
      bx = (big % big_x) * kMfBW + (sub % kSubX) * kMfTW;
      by = (big / big_x) * kMfBH + (sub / kSubX) * kMfTH;
      if (bx >= w || by >= h) continue;  // the same for the whole CTA
    } else {
      bx = (t % tiles_x) * kMfTW;
      by = (t / tiles_x) * kMfTH;
    }
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
static void launch_mf_t(cudaStream_t s, int w, int h, const float* img, const float* var, const float* psf_dev,
                        float sumpsf2, float* out, int* nf_buf) {
  auto kern = k_matched_filter_t<PS>;
  ensure_dynamic_smem(reinterpret_cast<const void*>(kern), MfGeom<PS>::smem);
  dim3 grid(ceil_div(w, kMfBW), ceil_div(h, kMfBH));
  kern<<<grid, kMfTX * kMfTY, MfGeom<PS>::smem, s>>>(w, h, img, var, psf_dev, sumpsf2, out, nf_buf, nf_buf + 1);
  DGPU_LAUNCH("k_matched_filter");
}

// psf_dev: the taps on the device; nf_buf: 1 + tile-count ints of device
// scratch for the list of tiles holding a non-finite value (at least one per
// 64 x 32 tile of the frame).
void launch_matched_filter(cudaStream_t s, int w, int h, const float* img, const float* var,
                           const float* psf_dev, int ps, float sumpsf2, float* out, int* nf_buf) {
  const int r = ps / 2;
  const size_t smem = sizeof(float) * (static_cast<size_t>(ps) * ps +
                                       static_cast<size_t>(kMfTH + 2 * r) * (kMfTW + 2 * r));
  if (smem > 200 * 1024) fail(DGPU_ERR_INVALID, "matched_filter: psf too large");
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_matched_filter_g), smem);
  const dim3 grid(ceil_div(w, kMfTW), ceil_div(h, kMfTH));
  bool templated = true;
  DGPU_CUDA(cudaMemsetAsync(nf_buf, 0, sizeof(int), s));
  switch (ps) {
    case 3: launch_mf_t<3>(s, w, h, img, var, psf_dev, sumpsf2, out, nf_buf); break;
    case 5: launch_mf_t<5>(s, w, h, img, var, psf_dev, sumpsf2, out, nf_buf); break;
    case 7: launch_mf_t<7>(s, w, h, img, var, psf_dev, sumpsf2, out, nf_buf); break;
    case 9: launch_mf_t<9>(s, w, h, img, var, psf_dev, sumpsf2, out, nf_buf); break;
    case 11: launch_mf_t<11>(s, w, h, img, var, psf_dev, sumpsf2, out, nf_buf); break;
    case 13: launch_mf_t<13>(s, w, h, img, var, psf_dev, sumpsf2, out, nf_buf); break;
    case 15: launch_mf_t<15>(s, w, h, img, var, psf_dev, sumpsf2, out, nf_buf); break;
    case 17: launch_mf_t<17>(s, w, h, img, var, psf_dev, sumpsf2, out, nf_buf); break;
    case 19: launch_mf_t<19>(s, w, h, img, var, psf_dev, sumpsf2, out, nf_buf); break;
    case 21: launch_mf_t<21>(s, w, h, img, var, psf_dev, sumpsf2, out, nf_buf); break;
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
