// Model convolve of the subtraction (src/subtract.cpp:466-639) for the common
// basis shapes: the tile engine of k_model_convolve (k_subtract.cu) with the
// component count NX = n_max + 1 and the tap count padded to KSP = 8 KB known
// at compile time.
//
// What changes against the generic kernel, and why the bits do not:
//   * Both passes run their taps in fully unrolled blocks with no per-tap
//     bound test. Taps j >= ks are zeros (tap rows are zero padded to KSP) and
//     the reference window carries 8 zero columns on its left and the x-pass
//     buffer 8 zero rows on top, so the extra taps read finite zeros. With
//     every staged value finite (the sanitised reference; its x-pass sums
//     stay finite for any image below ~1e37) a zero tap adds an exact +-0 to a
//     sum that starts at +0 and is never -0, so each output keeps the
//     reference's sum over j = 0..ks-1 bit for bit.
//   * The x pass works on row pairs: the reference window is staged with
//     rows 2p and 2p + 1 interleaved, so one 8-byte load gives both rows'
//     sample and one packed FMA (an IEEE fma per lane) applies a tap to both;
//     each thread holds 2 columns x 2 rows x NX components, its 2-wide
//     sliding window in registers across the unrolled taps, and reads the taps
//     duplicated (k, k) two at a time with 16-byte loads. Off-frame rows are
//     staged as zeros, so their x sums are exact +0 without a row test.
//   * The lattice corners of the cells the tile touches (every field) are
//     staged in shared memory once, so the blend of each component reads no
//     global memory.
//   * The field blend works on the two columns of a thread as one packed pair:
//     per coarse cell row the corner differences e = a10 - a00, t = a01 - a00,
//     g = (a11 - a10) - t, then per row base = fma(e, fy, a00),
//     slope = fma(g, fy, t), a = fma(slope, wx, base) -- the operations and
//     rounding of cell_blend, lane by lane.
// Everything else (tile staging, the zero rows above the x-pass buffer, the
// per-pixel order x taps -> components in basis order -> y taps -> d -= a bn)
// is the generic kernel's.
#include <cuda_runtime.h>

#include <algorithm>

#include "dev_common.cuh"

namespace dgpu {

namespace {

constexpr int kFTW = 32;   // tile width (columns)
constexpr int kFPad = 8;   // zero rows in front of each x-pass buffer
constexpr int kFLPad = 8;  // zero columns left of the reference window
constexpr int kFYR = 4;    // output rows per thread in the y pass (2 columns each)

__host__ __device__ constexpr int fast_rw(int ks) { return (kFLPad + kFTW + (ks - 1) + 3) & ~3; }

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fsub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }

template <int NX, int KB>
__global__ void __launch_bounds__(256)
k_model_convolve_f(int w, int h, const float* __restrict__ sci, const float* __restrict__ ref,
                   const uint8_t* __restrict__ rmask, DevFields F, const float* __restrict__ taps,
                   const int2* __restrict__ orders, int ks, int nc, const float* __restrict__ fillp,
                   float* __restrict__ diff, int TH, int lat_cap) {
  constexpr int KSP = 8 * KB;
  extern __shared__ __align__(16) float smem[];
  const int kh = (ks - 1) / 2;
  const int nrows = TH + 2 * kh;
  const int gbw = kFTW + 2 * kh;
  const int rw = fast_rw(ks);
  const int trows = nrows + kFPad;
  const int npair = (nrows + 1) / 2;
  float* rtile = smem;                          // npair x rw row pairs; column kFLPad + c <-> frame column bx - kh + c
  float* txs = rtile + 2 * npair * rw;          // NX x (kFPad zero rows + nrows) x kFTW
  float* ktaps = txs + NX * trows * kFTW;       // NX x KSP, zero padded
  float2* ktaps2 = reinterpret_cast<float2*>(ktaps + NX * KSP);  // the same taps duplicated (k, k)
  float* slat = ktaps + 3 * NX * KSP;           // nf x lly x llx lattice corners (lat_cap floats)
  const int bx = blockIdx.x * kFTW, by = blockIdx.y * TH;
  const float fill = *fillp;
  const int tid = threadIdx.x;

  // Corners of the lattice cells this tile touches (same cells for the whole CTA).
  int lcx0 = 0, lcy0 = 0, llx = 0, lly = 0;
  bool staged = false;
  if (!F.exact) {
    lcx0 = F.cellx[bx];
    lcy0 = F.celly[by];
    llx = F.cellx[min(bx + kFTW - 1, w - 1)] + 2 - lcx0;
    lly = F.celly[min(by + TH - 1, h - 1)] + 2 - lcy0;
    staged = F.nf * llx * lly <= lat_cap;
    if (staged)
      for (int i = tid; i < F.nf * lly * llx; i += blockDim.x) {
        const int f = i / (lly * llx), r = (i / llx) % lly, c = i % llx;
        slat[i] = __ldg(F.latf + (static_cast<size_t>(f) * F.ncy + lcy0 + r) * F.ncx + lcx0 + c);
      }
  }

  for (int i = tid; i < NX * KSP; i += blockDim.x) {
    const int q = i / KSP, j = i - q * KSP;
    const float k = j < ks ? taps[q * ks + j] : 0.0f;
    ktaps[i] = k;
    ktaps2[i] = make_float2(k, k);
  }
  for (int i = tid; i < NX * kFPad * kFTW; i += blockDim.x) {
    const int q = i / (kFPad * kFTW);
    txs[q * trows * kFTW + (i - q * kFPad * kFTW)] = 0.0f;
  }
  for (int i = tid; i < 2 * npair * rw; i += blockDim.x) {
    const int r = i / rw, cc = i - r * rw, c = cc - kFLPad;
    const int gy = by - kh + r, gx = bx - kh + c;
    float v = 0.0f;
    if (r < nrows && c >= 0 && c < gbw && gy >= 0 && gy < h && gx >= 0 && gx < w) {
      const size_t idx = static_cast<size_t>(gy) * w + gx;
      v = __ldg(ref + idx);
      const bool bad = (rmask && __ldg(rmask + idx) != 0) || !isfinite(v);
      if (bad) v = fill;
    }
    rtile[((r >> 1) * rw + cc) * 2 + (r & 1)] = v;
  }
  __syncthreads();

  // ---- x pass: txs[nx][r][lx] = sum_j k[nx][j] * R~[y][x + kh - j], rows in pairs ----
  constexpr int ngrp = kFTW / 2;
  const float2* rt2 = reinterpret_cast<const float2*>(rtile);
  for (int it = tid; it < npair * ngrp; it += blockDim.x) {
    const int rp = it / ngrp, cg = it - rp * ngrp;
    const int c0 = cg * 2;
    const float2* row = rt2 + rp * rw + kFLPad + c0 + 2 * kh;  // column of tap j=0, output 0
    float2 acc[NX][2];
#pragma unroll
    for (int q = 0; q < NX; ++q) acc[q][0] = acc[q][1] = make_float2(0.0f, 0.0f);
    float2 win[2] = {row[0], row[1]};
#pragma unroll
    for (int j0 = 0; j0 < KSP; j0 += 2) {
      float4 kq[NX];
#pragma unroll
      for (int q = 0; q < NX; ++q) kq[q] = *reinterpret_cast<const float4*>(ktaps2 + q * KSP + j0);
#pragma unroll
      for (int jj = 0; jj < 2; ++jj) {
        const int j = j0 + jj;
        if (j > 0) {
          win[1] = win[0];
          win[0] = row[-j];
        }
#pragma unroll
        for (int q = 0; q < NX; ++q) {
          const float2 kc = jj == 0 ? make_float2(kq[q].x, kq[q].y) : make_float2(kq[q].z, kq[q].w);
          acc[q][0] = __ffma2_rn(kc, win[0], acc[q][0]);
          acc[q][1] = __ffma2_rn(kc, win[1], acc[q][1]);
        }
      }
    }
    const int r = 2 * rp;
#pragma unroll
    for (int q = 0; q < NX; ++q) {
      *reinterpret_cast<float2*>(txs + (q * trows + kFPad + r) * kFTW + c0) = make_float2(acc[q][0].x, acc[q][1].x);
      if (r + 1 < nrows)
        *reinterpret_cast<float2*>(txs + (q * trows + kFPad + r + 1) * kFTW + c0) =
            make_float2(acc[q][0].y, acc[q][1].y);
    }
  }
  __syncthreads();

  // ---- y pass + field blend: 2 adjacent columns x 4 rows per thread ----
  const int lx0 = 2 * (tid % (kFTW / 2));
  const int ly0 = (tid / (kFTW / 2)) * kFYR;
  if (ly0 >= TH) return;
  const int x0 = bx + lx0;
  bool xin[2];
  int xcl[2];
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    xin[u] = x0 + u < w;
    xcl[u] = xin[u] ? x0 + u : w - 1;
  }
  int jx[2] = {0, 0};
  float2 wx2 = make_float2(0.0f, 0.0f);
  int jy[kFYR];
  float2 fy2[kFYR];
  if (!F.exact) {
    jx[0] = F.cellx[xcl[0]];
    jx[1] = F.cellx[xcl[1]];
    wx2 = make_float2(F.wx[xcl[0]], F.wx[xcl[1]]);
  }
#pragma unroll
  for (int i = 0; i < kFYR; ++i) {
    const int y = min(by + ly0 + i, h - 1);
    jy[i] = F.exact ? 0 : F.celly[y];
    fy2[i] = f2(F.exact ? 0.0f : F.wy[y]);
  }
  // Field values a_f(x, y_i) of both columns (packed), the corners re-read
  // only when the coarse cell row changes.
  auto fields_of = [&](int f, float2 (&a)[kFYR]) {
    if (F.exact) {
#pragma unroll
      for (int i = 0; i < kFYR; ++i) {
        const int y = min(by + ly0 + i, h - 1);
        const float* fr = F.full + (static_cast<size_t>(f) * h + y) * w;
        a[i] = make_float2(__ldg(fr + xcl[0]), __ldg(fr + xcl[1]));
      }
      return;
    }
    int cj = -1;
    float2 a00, e, t, g;
#pragma unroll
    for (int i = 0; i < kFYR; ++i) {
      if (jy[i] != cj) {
        cj = jy[i];
        float2 a01, a10, a11;
        if (staged) {
          const float* r0 = slat + (f * lly + (cj - lcy0)) * llx - lcx0;
          const float* r1 = r0 + llx;
          a00 = make_float2(r0[jx[0]], r0[jx[1]]);
          a01 = make_float2(r0[jx[0] + 1], r0[jx[1] + 1]);
          a10 = make_float2(r1[jx[0]], r1[jx[1]]);
          a11 = make_float2(r1[jx[0] + 1], r1[jx[1] + 1]);
        } else {
          const float* r0 = F.latf + (static_cast<size_t>(f) * F.ncy + cj) * F.ncx;
          const float* r1 = r0 + F.ncx;
          a00 = make_float2(__ldg(r0 + jx[0]), __ldg(r0 + jx[1]));
          a01 = make_float2(__ldg(r0 + jx[0] + 1), __ldg(r0 + jx[1] + 1));
          a10 = make_float2(__ldg(r1 + jx[0]), __ldg(r1 + jx[1]));
          a11 = make_float2(__ldg(r1 + jx[0] + 1), __ldg(r1 + jx[1] + 1));
        }
        e = fsub2(a10, a00);
        t = fsub2(a01, a00);
        g = fsub2(fsub2(a11, a10), t);
      }
      const float2 base = __ffma2_rn(e, fy2[i], a00);
      const float2 slope = __ffma2_rn(g, fy2[i], t);
      a[i] = __ffma2_rn(slope, wx2, base);
    }
  };
  float2 d2[kFYR];
  {
    float2 bg[kFYR];
    fields_of(nc, bg);
#pragma unroll
    for (int i = 0; i < kFYR; ++i) {
      const int y = min(by + ly0 + i, h - 1);
      const float* sr = sci + static_cast<size_t>(y) * w;
      d2[i] = fsub2(make_float2(__ldg(sr + xcl[0]), __ldg(sr + xcl[1])), bg[i]);
    }
  }
  const int base = ly0 + 2 * kh;
  for (int n = 0; n < nc; ++n) {
    const int2 o = orders[n];
    const float2* col = reinterpret_cast<const float2*>(txs + (static_cast<size_t>(o.x) * trows + kFPad) * kFTW + lx0);
    const float* ky = ktaps + o.y * KSP;
    float2 bn[kFYR];
#pragma unroll
    for (int i = 0; i < kFYR; ++i) bn[i] = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int j0 = 0; j0 < KSP; j0 += 8) {
      float2 v[kFYR + 7];  // v[t] = buffer row base - j0 - 7 + t
      const float2* vb = col + (base - j0 - 7) * (kFTW / 2);
#pragma unroll
      for (int t = 0; t < kFYR + 7; ++t) v[t] = vb[t * (kFTW / 2)];
      const float4 ka = *reinterpret_cast<const float4*>(ky + j0);
      const float4 kb = *reinterpret_cast<const float4*>(ky + j0 + 4);
      const float kv[8] = {ka.x, ka.y, ka.z, ka.w, kb.x, kb.y, kb.z, kb.w};
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) {
        const float2 cc = f2(kv[jj]);
#pragma unroll
        for (int i = 0; i < kFYR; ++i) bn[i] = __ffma2_rn(cc, v[i - jj + 7], bn[i]);
      }
    }
    float2 a[kFYR];
    fields_of(n, a);
#pragma unroll
    for (int i = 0; i < kFYR; ++i) d2[i] = __ffma2_rn(make_float2(-a[i].x, -a[i].y), bn[i], d2[i]);
  }
#pragma unroll
  for (int i = 0; i < kFYR; ++i) {
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

// Floats of shared memory for the lattice corners a tile of TH rows touches.
int lattice_cap(const DevFields& F, int TH) {
  if (F.exact || F.stride <= 0) return 0;
  const int lx = std::min(F.ncx, (kFTW - 1) / F.stride + 3), ly = std::min(F.ncy, (TH - 1) / F.stride + 3);
  return F.nf * lx * ly;
}

template <int NX, int KB>
void launch_f(cudaStream_t s, const SubtractArgs& a, const int2* orders, int TH, size_t smem) {
  auto kern = k_model_convolve_f<NX, KB>;
  ensure_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
  dim3 grid(ceil_div(a.w, kFTW), ceil_div(a.h, TH));
  const int threads = (kFTW / 2) * (TH / kFYR);
  kern<<<grid, threads, smem, s>>>(a.w, a.h, a.sci, a.ref, a.ref_mask, a.F, a.taps, orders, a.ks, a.nc, a.fill,
                                   a.diff, TH, lattice_cap(a.F, TH));
  DGPU_LAUNCH("k_model_convolve_f");
}

template <int NX>
bool launch_nx(cudaStream_t s, const SubtractArgs& a, const int2* orders, int TH, size_t smem, int kb) {
  switch (kb) {
    case 2: launch_f<NX, 2>(s, a, orders, TH, smem); return true;
    case 3: launch_f<NX, 3>(s, a, orders, TH, smem); return true;
    case 4: launch_f<NX, 4>(s, a, orders, TH, smem); return true;
    case 5: launch_f<NX, 5>(s, a, orders, TH, smem); return true;
    default: return false;
  }
}

}  // namespace

size_t model_convolve_fast_smem(int nx, int ks, int TH, const DevFields& F) {
  const int kh = (ks - 1) / 2;
  const int nrows = TH + 2 * kh;
  const int kb = (ks + 7) / 8;
  return sizeof(float) * (2 * static_cast<size_t>((nrows + 1) / 2) * fast_rw(ks) +
                          static_cast<size_t>(nx) * (nrows + kFPad) * kFTW + static_cast<size_t>(nx) * 3 * 8 * kb +
                          static_cast<size_t>(lattice_cap(F, TH)));
}

bool model_convolve_fast_available(int nx, int ks) {
  const int kb = (ks + 7) / 8;
  return (nx == 3 || nx == 4 || nx == 5 || nx == 6 || nx == 7) && kb >= 2 && kb <= 5;
}

bool launch_model_convolve_fast(cudaStream_t s, const SubtractArgs& a, const int2* orders, int TH) {
  const int nx = a.n_max + 1;
  if (!model_convolve_fast_available(nx, a.ks)) return false;
  const size_t smem = model_convolve_fast_smem(nx, a.ks, TH, a.F);
  const int kb = (a.ks + 7) / 8;
  switch (nx) {
    case 3: return launch_nx<3>(s, a, orders, TH, smem, kb);
    case 4: return launch_nx<4>(s, a, orders, TH, smem, kb);
    case 5: return launch_nx<5>(s, a, orders, TH, smem, kb);
    case 6: return launch_nx<6>(s, a, orders, TH, smem, kb);
    case 7: return launch_nx<7>(s, a, orders, TH, smem, kb);
    default: return false;
  }
}

}  // namespace dgpu
