// ZOGY noise decorrelation (reference src/noise.cpp:65-533), sm_100a.
//
// Per overlap-add block (n x n, n a power of two, stride n/2, reflect padded):
//   row pass    : n real rows -> n/2-point complex FFT of the even/odd packing
//                 -> Hermitian split -> n/2+1 bins per row (r2c);
//   column pass : n-point complex FFT down each of the n/2+1 columns, the
//                 decorrelation filter Phi = sqrt(vs + vr sum K^2) /
//                 sqrt(vs + vr |Khat|^2) applied in place (|Khat|^2 from the
//                 per-cell cache, vs / vr the block's subsampled medians), then
//                 the inverse column FFT;
//   row inverse : Hermitian merge -> n/2-point inverse FFT -> n real samples.
// For n = 256 the three passes run fused in k_block_filter (one 4-CTA cluster
// per block, the spectrum in distributed shared memory); otherwise as three
// kernels through a scratch spectrum. The raw block outputs are then
// overlap-added by k_ola_gather: every pixel sums its Hann-weighted blocks in
// the reference's 9-colour order (ix % 3, iy % 3), with the float rounding of
// the reference's colour passes, and divides by the weight sums.
// Lines of 128 / 256 points use a four-step FFT (16-point DFTs in registers);
// other lengths a radix-2 shared-memory FFT. Twiddles are FP64-derived.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "dev_common.cuh"
#include "fft_internal.h"

namespace dgpu {

namespace cg = cooperative_groups;

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// tw[k] = exp(sign 2 pi i k / m), k < m/2.
__device__ void make_twiddles(float2* tw, int m, int sign) {
  for (int k = threadIdx.x; k < m / 2; k += blockDim.x) {
    double s, c;
    sincospi(2.0 * k / m, &s, &c);
    tw[k] = make_float2(static_cast<float>(c), static_cast<float>(sign * s));
  }
}

// Twiddle table offsets (see FftGeom::tw_tab).
__device__ __forceinline__ int tw_off_inv_n(int n) { return n / 2; }
__device__ __forceinline__ int tw_off_fwd_hn(int n) { return n; }
__device__ __forceinline__ int tw_off_inv_hn(int n) { return n + n / 4; }
__device__ __forceinline__ int tw_off_split_fwd(int n) { return n + n / 2; }
__device__ __forceinline__ int tw_off_split_inv(int n) { return n + n / 2 + n / 2 + 1; }

__device__ __forceinline__ void copy_tw(float2* dst, const float2* src, int count) {
  for (int k = threadIdx.x; k < count; k += blockDim.x) dst[k] = src[k];
}

// Same values as make_twiddles / the split factors below, once per call.
__global__ void k_twiddle_table(int n, float2* tab) {
  const int hn = n / 2;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n / 2; k += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(2.0 * k / n, &s, &c);
    tab[k] = make_float2(static_cast<float>(c), static_cast<float>(-s));
    tab[tw_off_inv_n(n) + k] = make_float2(static_cast<float>(c), static_cast<float>(s));
  }
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < hn / 2; k += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(2.0 * k / hn, &s, &c);
    tab[tw_off_fwd_hn(n) + k] = make_float2(static_cast<float>(c), static_cast<float>(-s));
    tab[tw_off_inv_hn(n) + k] = make_float2(static_cast<float>(c), static_cast<float>(s));
  }
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= hn; k += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(2.0 * k / n, &s, &c);
    tab[tw_off_split_fwd(n) + k] = make_float2(static_cast<float>(c), static_cast<float>(-s));
    tab[tw_off_split_inv(n) + k] = make_float2(static_cast<float>(c), static_cast<float>(s));
  }
}

// In-place radix-2 DIT FFT of L lines of length m in shared memory, line l at
// x + l * ls (ls = m for packed rows; m + 1 for transposed column lines, which
// keeps the strided accesses of a warp on distinct banks).
__device__ void smem_fft(float2* x, int L, int m, int logm, const float2* tw, int ls) {
  for (int e = threadIdx.x; e < L * m; e += blockDim.x) {
    const int line = e / m, j = e - line * m;
    const int rj = static_cast<int>(__brev(static_cast<unsigned>(j)) >> (32 - logm));
    if (j < rj) {
      const float2 t = x[line * ls + j];
      x[line * ls + j] = x[line * ls + rj];
      x[line * ls + rj] = t;
    }
  }
  __syncthreads();
  for (int half = 1; half < m; half <<= 1) {
    const int tstep = m / (2 * half);
    for (int b = threadIdx.x; b < L * (m / 2); b += blockDim.x) {
      const int line = b / (m / 2), j = b - line * (m / 2);
      const int pos = j & (half - 1);
      const int i0 = ((j - pos) << 1) + pos, i1 = i0 + half;
      float2* xl = x + line * ls;
      const float2 a = xl[i0];
      const float2 c = cmul(xl[i1], tw[pos * tstep]);
      xl[i0] = cadd(a, c);
      xl[i1] = csub(a, c);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Four-step FFT of lines of length N = 16 * N2 (N = 128 or 256): pass A does a
// 16-point DFT in registers over the stride-N2 samples of each residue n2,
// multiplies by W_N^(n2 k1) and writes a padded k1-major layout; pass B does the
// N2-point DFT in registers and writes natural order. Two shared-memory round
// trips per line instead of log2(N) + 1. tw[k] = W_N^k for k < N/2 (the sign
// of W selects forward or inverse); lines need ls >= N + 17; 256 threads.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int bitrev_c(int i, int bits) {
  int r = 0;
  for (int b = 0; b < bits; ++b) r |= ((i >> b) & 1) << (bits - 1 - b);
  return r;
}

// v * W_16^j for the unrolled (compile-time) j of a register FFT, SIGN = -1
// forward (W = exp(-2 pi i / 16)), +1 inverse: j = 0 is the identity, j = 4
// the exact swap by -+i, the others one complex multiply by constants equal to
// the twiddle table's float values (cos / sin of j pi / 8 rounded from FP64).
template <int SIGN>
__device__ __forceinline__ float2 mul_w16(float2 v, int j) {
  if (j == 0) return v;
  if (j == 4) return SIGN < 0 ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
  float c, sn;
  switch (j) {
    case 1: c = 0.923879532511286738f; sn = 0.382683432365089772f; break;
    case 2: c = 0.707106781186547524f; sn = 0.707106781186547524f; break;
    case 3: c = 0.382683432365089772f; sn = 0.923879532511286738f; break;
    case 5: c = -0.382683432365089772f; sn = 0.923879532511286738f; break;
    case 6: c = -0.707106781186547524f; sn = 0.707106781186547524f; break;
    default: c = -0.923879532511286738f; sn = 0.382683432365089772f; break;  // j == 7
  }
  return cmul(v, make_float2(c, SIGN < 0 ? -sn : sn));
}

// In-register radix-2 FFT of M = 8 or 16 points (a sub-FFT of a four-step
// line of N = 128 or 256): every butterfly twiddle is a 16th root of unity,
// W_16^(pos * 8 / half), so none is loaded.
template <int M, int LOGM, int SIGN>
__device__ __forceinline__ void reg_fft(float2 (&v)[M]) {
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const int r = bitrev_c(i, LOGM);
    if (i < r) {
      const float2 t = v[i];
      v[i] = v[r];
      v[r] = t;
    }
  }
#pragma unroll
  for (int half = 1; half < M; half <<= 1) {
#pragma unroll
    for (int j = 0; j < M / 2; ++j) {
      const int pos = j & (half - 1);
      const int i0 = ((j - pos) << 1) + pos, i1 = i0 + half;
      const float2 a = v[i0];
      const float2 c = mul_w16<SIGN>(v[i1], pos * 8 / half);
      v[i0] = cadd(a, c);
      v[i1] = csub(a, c);
    }
  }
}

template <int N, int SIGN>
__device__ void fft_lines_4step_d(float2* x, int L, int ls, const float2* tw) {
  constexpr int N1 = 16, N2 = N / 16;
  constexpr int LOGN2 = N == 256 ? 4 : 3;
  constexpr int kLinesA = 256 / N2, kLinesB = 256 / N1;
  for (int l0 = 0; l0 < L; l0 += kLinesA) {
    const int line = l0 + threadIdx.x / N2, n2 = threadIdx.x % N2;
    const bool act = line < L;
    float2 v[N1];
    if (act) {
      float2* xl = x + line * ls;
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) v[n1] = xl[N2 * n1 + n2];
      reg_fft<N1, 4, SIGN>(v);
#pragma unroll
      for (int k1 = 1; k1 < N1; ++k1) {
        const int m = n2 * k1;
        float2 w = tw[m < N / 2 ? m : m - N / 2];
        if (m >= N / 2) w = make_float2(-w.x, -w.y);
        v[k1] = cmul(v[k1], w);
      }
    }
    __syncthreads();
    if (act) {
      float2* xl = x + line * ls;
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) xl[k1 * (N2 + 1) + n2] = v[k1];
    }
    __syncthreads();
  }
  for (int l0 = 0; l0 < L; l0 += kLinesB) {
    const int line = l0 + threadIdx.x / N1, k1 = threadIdx.x % N1;
    const bool act = line < L;
    float2 u[N2];
    if (act) {
      const float2* xl = x + line * ls;
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) u[n2] = xl[k1 * (N2 + 1) + n2];
      reg_fft<N2, LOGN2, SIGN>(u);
    }
    __syncthreads();
    if (act) {
      float2* xl = x + line * ls;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) xl[k1 + N1 * k2] = u[k2];
    }
    __syncthreads();
  }
}

// Line stride for an FFT of length m: room for the four-step layout where it
// applies (odd in float2 units past a multiple of 16, so transposed column
// accesses stay on distinct banks).
__host__ __device__ __forceinline__ int fft_ls(int m, bool transposed) {
  if (m == 128 || m == 256) return m + 17;
  return transposed ? m + 1 : m;
}

// Dispatch: four-step for 128 / 256, radix-2 otherwise. SIGN is the
// direction of `tw` (-1 forward, +1 inverse), known at every call site.
template <int SIGN>
__device__ __forceinline__ void fft_lines(float2* x, int L, int m, int logm, const float2* tw, int ls) {
  if (m == 256)
    fft_lines_4step_d<256, SIGN>(x, L, ls, tw);
  else if (m == 128)
    fft_lines_4step_d<128, SIGN>(x, L, ls, tw);
  else
    smem_fft(x, L, m, logm, tw, ls);
}

__device__ __forceinline__ int reflect_clamp(int s, int len) {
  if (s < 0) s = -s - 1;
  if (s >= len) s = 2 * len - s - 1;
  return min(max(s, 0), len - 1);
}

// ---------------------------------------------------------------------------
// Row pass (r2c). mode 0: block rows of the frame, reflect padded
// (src/noise.cpp:392-406); mode 1: rows of a dense n x n real image per item.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_rows_fwd(FftGeom G, int mode, const float* __restrict__ src, int w, int h, const int* __restrict__ oxs,
           const int* __restrict__ oys, int nox, float2* __restrict__ spec) {
  extern __shared__ __align__(16) float2 fsm2[];
  const int n = G.n, hn = n / 2, nb = hn + 1;
  const int rows = G.rows_per_cta;
  const int zl = fft_ls(hn, false);
  float2* z = fsm2;                 // rows x zl
  float2* tw = z + rows * zl;       // hn/2 (length-hn FFT)
  float2* twn = tw + hn / 2 + 1;    // hn (W^k, k < hn + 1) for the split
  const int item = blockIdx.x, r0 = blockIdx.y * rows;
  if (G.tw_tab) {
    copy_tw(tw, G.tw_tab + tw_off_fwd_hn(n), hn / 2);
    copy_tw(twn, G.tw_tab + tw_off_split_fwd(n), hn + 1);
  } else {
    make_twiddles(tw, hn, -1);
    for (int k = threadIdx.x; k <= hn; k += blockDim.x) {
      double s, c;
      sincospi(2.0 * k / n, &s, &c);
      twn[k] = make_float2(static_cast<float>(c), static_cast<float>(-s));
    }
  }
  int bx = 0, by = 0;
  if (mode == 0) {
    bx = oxs[item % nox];
    by = oys[item / nox];
  }
  for (int e = threadIdx.x; e < rows * hn; e += blockDim.x) {
    const int rr = e / hn, j = e - rr * hn;
    const int row = r0 + rr;
    float a, b;
    if (mode == 0) {
      const int sy = reflect_clamp(by + row, h);
      const float* srow = src + static_cast<size_t>(sy) * w;
      a = srow[reflect_clamp(bx + 2 * j, w)];
      b = srow[reflect_clamp(bx + 2 * j + 1, w)];
    } else {
      const float* srow = src + (static_cast<size_t>(item) * n + row) * n;
      a = srow[2 * j];
      b = srow[2 * j + 1];
    }
    z[rr * zl + j] = make_float2(a, b);
  }
  __syncthreads();
  fft_lines<-1>(z, rows, hn, G.logn - 1, tw, zl);
  for (int e = threadIdx.x; e < rows * nb; e += blockDim.x) {
    const int rr = e / nb, k = e - rr * nb;
    const float2 zk = z[rr * zl + (k % hn)];
    const float2 zc = cconj(z[rr * zl + ((hn - k) % hn)]);
    const float2 ev = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
    const float2 d = csub(zk, zc);                         // 2i O
    const float2 od = make_float2(0.5f * d.y, -0.5f * d.x);  // O = d / (2i)
    spec[(static_cast<size_t>(item) * n + r0 + rr) * nb + k] = cadd(ev, cmul(twn[k], od));
  }
}

// ---------------------------------------------------------------------------
// Column pass. mode 0: forward, multiply by the block filter, inverse (in
// place); mode 1: forward and write |X|^2 in FP64 (kernel-power cache).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_cols(FftGeom G, int mode, float2* __restrict__ spec, const double* __restrict__ cell_power,
       const double* __restrict__ cell_sumk2, const int* __restrict__ block_cell, const double* __restrict__ vsr,
       double* __restrict__ power_out) {
  extern __shared__ __align__(16) float2 fsm2[];
  const int n = G.n, nb = n / 2 + 1;
  const int C = G.cols_per_cta;
  const int ls = fft_ls(n, true);  // padded column-line stride (bank-conflict free transposes)
  float2* x = fsm2;            // C x ls
  float2* tw = x + C * ls;     // n/2
  const int item = blockIdx.x, c0 = blockIdx.y * C;
  const int ncol = min(C, nb - c0);
  if (G.tw_tab)
    copy_tw(tw, G.tw_tab, n / 2);
  else
    make_twiddles(tw, n, -1);
  float2* sp = spec + static_cast<size_t>(item) * n * nb;
  if (mode == 2) {
    // Spectrum = the real filter itself (decorrelation_kernel_image, src/noise.cpp:139-146).
    for (int e = threadIdx.x; e < C * ls; e += blockDim.x) x[e] = make_float2(0.f, 0.f);
  } else {
    for (int e = threadIdx.x; e < C * n; e += blockDim.x) {
      const int row = e / C, cc = e - row * C;
      x[cc * ls + row] = cc < ncol ? sp[static_cast<size_t>(row) * nb + c0 + cc] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    fft_lines<-1>(x, C, n, G.logn, tw, ls);
  }
  if (mode == 1) {
    for (int e = threadIdx.x; e < C * n; e += blockDim.x) {
      const int row = e / C, cc = e - row * C;
      if (cc >= ncol) continue;
      const float2 v = x[cc * ls + row];
      const double re = v.x, im = v.y;
      power_out[(static_cast<size_t>(item) * n + row) * nb + c0 + cc] = re * re + im * im;
    }
    return;
  }
  // Filter (src/noise.cpp:414-422), then the inverse column FFT.
  const int cell = block_cell[item];
  const double vs = vsr[2 * item], vr = vsr[2 * item + 1];
  const double cnum = sqrt(fmax(vs + vr * cell_sumk2[cell], 0.0));
  if (mode == 0 && blockIdx.y == 0 && threadIdx.x == 0 && power_out) power_out[item] = cnum * cnum;  // block num
  const double* pw = cell_power + static_cast<size_t>(cell) * n * nb;
  for (int e = threadIdx.x; e < C * n; e += blockDim.x) {
    const int row = e / C, cc = e - row * C;
    if (cc >= ncol) continue;
    const double denom = vs + vr * pw[static_cast<size_t>(row) * nb + c0 + cc];
    const float f = denom > 0.0 ? static_cast<float>(cnum / sqrt(denom)) : 0.0f;
    float2& xv = x[cc * ls + row];
    xv = mode == 2 ? make_float2(f, 0.0f) : make_float2(xv.x * f, xv.y * f);
  }
  __syncthreads();
  if (G.tw_tab)
    copy_tw(tw, G.tw_tab + tw_off_inv_n(n), n / 2);
  else
    make_twiddles(tw, n, +1);
  __syncthreads();
  fft_lines<1>(x, C, n, G.logn, tw, ls);
  for (int e = threadIdx.x; e < C * n; e += blockDim.x) {
    const int row = e / C, cc = e - row * C;
    if (cc < ncol) sp[static_cast<size_t>(row) * nb + c0 + cc] = x[cc * ls + row];
  }
}

// ---------------------------------------------------------------------------
// Row inverse (c2r). mode 0: Hann overlap-add of the blocks of one colour into
// acc / var_acc (src/noise.cpp:430-452); mode 1: plain store x 1/n^2 into a
// dense n x n real output per item.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_rows_inv(FftGeom G, int mode, const float2* __restrict__ spec, const int* __restrict__ items, int w, int h,
           const int* __restrict__ oxs, const int* __restrict__ oys, int nox, const double* __restrict__ hwin,
           const double* __restrict__ vsr, const double* __restrict__ cell_sumk2, const int* __restrict__ block_cell,
           float* __restrict__ acc, float* __restrict__ var_acc, float* __restrict__ dense_out) {
  extern __shared__ __align__(16) float2 fsm2[];
  const int n = G.n, hn = n / 2, nb = hn + 1;
  const int rows = G.rows_per_cta;
  const int zl = fft_ls(hn, false);
  float2* z = fsm2;
  float2* tw = z + rows * zl;
  float2* twn = tw + hn / 2 + 1;
  const int item = mode == 0 ? items[blockIdx.x] : blockIdx.x;
  const int r0 = blockIdx.y * rows;
  if (G.tw_tab) {
    copy_tw(tw, G.tw_tab + tw_off_inv_hn(n), hn / 2);
    copy_tw(twn, G.tw_tab + tw_off_split_inv(n), hn + 1);  // W^-k
  } else {
    make_twiddles(tw, hn, +1);
    for (int k = threadIdx.x; k <= hn; k += blockDim.x) {
      double s, c;
      sincospi(2.0 * k / n, &s, &c);
      twn[k] = make_float2(static_cast<float>(c), static_cast<float>(s));  // W^-k
    }
  }
  __syncthreads();
  const float2* sp = spec + static_cast<size_t>(item) * n * nb;
  for (int e = threadIdx.x; e < rows * hn; e += blockDim.x) {
    const int rr = e / hn, k = e - rr * hn;
    const float2* xr = sp + static_cast<size_t>(r0 + rr) * nb;
    float2 xk = xr[k];
    float2 xc = cconj(xr[hn - k]);
    if (k == 0) {  // c2r ignores the imaginary parts of the DC and Nyquist bins
      xk.y = 0.0f;
      xc.y = 0.0f;
    }
    const float2 e2 = cadd(xk, xc);
    const float2 o2 = cmul(csub(xk, xc), twn[k]);
    z[rr * zl + k] = make_float2(e2.x - o2.y, e2.y + o2.x);  // 2E + i 2O
  }
  __syncthreads();
  fft_lines<1>(z, rows, hn, G.logn - 1, tw, zl);
  const float inv_n2 = 1.0f / static_cast<float>(static_cast<size_t>(n) * n);
  if (mode == 2) {  // raw real block output for the overlap-add gather (dense_out: item x n x n)
    for (int e = threadIdx.x; e < rows * n; e += blockDim.x) {
      const int rr = e / n, m = e - rr * n;
      const float2 v = z[rr * zl + (m >> 1)];
      dense_out[(static_cast<size_t>(item) * n + r0 + rr) * n + m] = (m & 1) ? v.y : v.x;
    }
    return;
  }
  if (mode == 1) {
    for (int e = threadIdx.x; e < rows * n; e += blockDim.x) {
      const int rr = e / n, m = e - rr * n;
      const float2 v = z[rr * zl + (m >> 1)];
      dense_out[(static_cast<size_t>(item) * n + r0 + rr) * n + m] = ((m & 1) ? v.y : v.x) * inv_n2;
    }
    return;
  }
  const int bx = oxs[item % nox], by = oys[item / nox];
  const int cell = block_cell[item];
  const double vs = vsr[2 * item], vr = vsr[2 * item + 1];
  const double cnum = sqrt(fmax(vs + vr * cell_sumk2[cell], 0.0));
  const double num = cnum * cnum;
  for (int e = threadIdx.x; e < rows * n; e += blockDim.x) {
    const int rr = e / n, m = e - rr * n;
    const int iy = r0 + rr;
    const int y = by + iy, x = bx + m;
    if (y < 0 || y >= h || x < 0 || x >= w) continue;
    const float2 v = z[rr * zl + (m >> 1)];
    const float f = (m & 1) ? v.y : v.x;
    const double wy_sig = hwin[iy] * static_cast<double>(inv_n2);
    const double wy_var = hwin[iy];
    const double wx = hwin[m];
    const size_t o = static_cast<size_t>(y) * w + x;
    acc[o] = static_cast<float>(static_cast<double>(acc[o]) + wy_sig * wx * static_cast<double>(f));
    var_acc[o] = static_cast<float>(static_cast<double>(var_acc[o]) + wy_var * wx * num);
  }
}

// ---------------------------------------------------------------------------
// Fused block filter for the default 256 x 256 block (mode 0 of the three
// passes above, in one launch): one cluster of 4 CTAs per block. Rank r keeps
// spectrum columns [32 r, 32 r + 32) as transposed column lines in its shared
// memory (with the Nyquist column packed into rank 0's DC line, see bf_owner)
// and runs the row passes of rows 64 r .. 64 r + 63. Row pass: the r2c rows
// are scattered into the owners' column lines (distributed shared memory);
// column pass: forward FFT, filter, inverse FFT on local lines; row inverse:
// every row gathers its bins from the owners, c2r, raw block output
// (item x n x n) for the overlap-add gather. The row and column arithmetic is
// that of k_rows_fwd / k_cols / k_rows_inv except for the packed DC / Nyquist
// pair (the same transforms to FP32 rounding); the spectrum never leaves the
// chip.
// ---------------------------------------------------------------------------
constexpr int kBfRanks = 4;
constexpr int kBfN = 256;
constexpr int kBfBatch = 16;  // rows per row-pass batch
constexpr int kBfCols = 32;   // column lines per rank

// Bins 1..127 of every row live in line k % 32 of rank k / 32. The DC (k = 0)
// and Nyquist (k = 128) bins of a real row are real, so their two columns share
// rank 0's line 0 as one complex sequence (DC in the real part, Nyquist in the
// imaginary part): one column FFT carries both, and every rank holds 32 lines.
__device__ __forceinline__ int bf_owner(int k) { return k >> 5; }
__device__ __forceinline__ int bf_cb(int r) { return 32 * r; }

__global__ void __cluster_dims__(kBfRanks, 1, 1) __launch_bounds__(256, 2)
k_block_filter(FftGeom G, const float* __restrict__ src, int w, int h, const int* __restrict__ oxs,
               const int* __restrict__ oys, int nox, const double* __restrict__ cell_power,
               const double* __restrict__ cell_sumk2, const int* __restrict__ block_cell,
               const double* __restrict__ vsr, double* __restrict__ bnum, float* __restrict__ dense_out) {
  extern __shared__ __align__(16) float2 fsm2[];
  constexpr int n = kBfN, hn = n / 2, nb = hn + 1;
  const int ls = fft_ls(n, true), zl = fft_ls(hn, false);
  cg::cluster_group cl = cg::this_cluster();
  const int rank = static_cast<int>(cl.block_rank());
  const int item = blockIdx.x / kBfRanks;
  float2* x = fsm2;                      // kBfCols x ls column lines
  float2* z = x + kBfCols * ls;          // kBfBatch x zl row lines
  float2* tw = z + kBfBatch * zl;        // the whole twiddle table
  copy_tw(tw, G.tw_tab, n + n / 2 + 2 * nb);
  const float2* tw_fwd_n = tw;
  const float2* tw_inv_n = tw + n / 2;
  const float2* tw_fwd_hn = tw + n;
  const float2* tw_inv_hn = tw + n + n / 4;
  const float2* split_fwd = tw + n + n / 2;
  const float2* split_inv = split_fwd + nb;
  // Element (column k, row) of the block spectrum in its owner's lines.
  auto bin = [&](int k, int row) {
    const int q = bf_owner(k);
    return cl.map_shared_rank(x + (k - bf_cb(q)) * ls + row, q);
  };
  const int bx = oxs[item % nox], by = oys[item / nox];
  const int ncol = kBfCols;
  const int rbeg = rank * (n / kBfRanks), rend = rbeg + n / kBfRanks;
  cl.sync();  // every rank has started before its shared memory is written

  // Row pass (r2c), scattered to the column owners. 256 threads: each loop
  // below has a fixed trip count, so its loads are all in flight together.
  const int tid = threadIdx.x;
  // The next batch's samples are loaded while this batch transforms.
  constexpr int kPer = kBfBatch * hn / 256;
  float2 v[kPer];
  auto load_batch = [&](int b) {
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int e = tid + 256 * i, rr = e / hn, j = e - rr * hn;
      const int sy = reflect_clamp(by + b + rr, h);
      const float* srow = src + static_cast<size_t>(sy) * w;
      v[i] = make_float2(__ldg(srow + reflect_clamp(bx + 2 * j, w)), __ldg(srow + reflect_clamp(bx + 2 * j + 1, w)));
    }
  };
  load_batch(rbeg);
  for (int b0 = rbeg; b0 < rend; b0 += kBfBatch) {
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int e = tid + 256 * i, rr = e / hn, j = e - rr * hn;
      z[rr * zl + j] = v[i];
    }
    if (b0 + kBfBatch < rend) load_batch(b0 + kBfBatch);
    __syncthreads();
    fft_lines<-1>(z, kBfBatch, hn, G.logn - 1, tw_fwd_hn, zl);
#pragma unroll
    for (int i = 0; i < (kBfBatch * nb + 255) / 256; ++i) {
      const int e = tid + 256 * i;
      if (e >= kBfBatch * nb) break;
      const int rr = e / nb, k = e - rr * nb;
      const float2 zk = z[rr * zl + (k % hn)];
      const float2 zc = cconj(z[rr * zl + ((hn - k) % hn)]);
      const float2 ev = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
      const float2 d = csub(zk, zc);
      const float2 od = make_float2(0.5f * d.y, -0.5f * d.x);
      const float2 X = cadd(ev, cmul(split_fwd[k], od));
      if (k == 0 || k == hn)  // real: into the packed line (separate 4-byte words)
        reinterpret_cast<float*>(cl.map_shared_rank(x + b0 + rr, 0))[k == 0 ? 0 : 1] = X.x;
      else
        *bin(k, b0 + rr) = X;
    }
    __syncthreads();
  }
  cl.sync();

  // Column pass: forward, filter (src/noise.cpp:414-422), inverse. Filter:
  // lane = column (coalesced kernel-power loads), warps over rows; rank 0's
  // packed line by a thread per bin pair (k, n - k): the transform Z of
  // DC + i Nyquist splits into A = (Z_k + conj Z_-k) / 2 (the DC column's) and
  // B = (Z_k - conj Z_-k) / 2i (the Nyquist column's), each is filtered with
  // its own column's factor, and A + iB is put back.
  fft_lines<-1>(x, ncol, n, G.logn, tw_fwd_n, ls);
  {
    const int cell = block_cell[item];
    const double vs = vsr[2 * item], vr = vsr[2 * item + 1];
    const double cnum = sqrt(fmax(vs + vr * cell_sumk2[cell], 0.0));
    if (rank == 0 && tid == 0 && bnum) bnum[item] = cnum * cnum;
    const double* pw = cell_power + static_cast<size_t>(cell) * n * nb + bf_cb(rank);
    auto scale = [&](int cc, int row, double p) {
      const double denom = vs + vr * p;
      const float f = denom > 0.0 ? static_cast<float>(cnum / sqrt(denom)) : 0.0f;
      float2& xv = x[cc * ls + row];
      xv = make_float2(xv.x * f, xv.y * f);
    };
    const int cc = tid & 31, r0 = tid >> 5;
    if (rank != 0 || cc != 0) {
      for (int rb = 0; rb < n; rb += 64) {
        double p[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) p[i] = __ldg(pw + static_cast<size_t>(rb + r0 + 8 * i) * nb + cc);
#pragma unroll
        for (int i = 0; i < 8; ++i) scale(cc, rb + r0 + 8 * i, p[i]);
      }
    }
    if (rank == 0 && tid <= hn) {
      auto factor = [&](int row, int col) {
        const double denom = vs + vr * __ldg(pw + static_cast<size_t>(row) * nb + col);
        return denom > 0.0 ? static_cast<float>(cnum / sqrt(denom)) : 0.0f;
      };
      const int k = tid, m = (n - k) & (n - 1);
      const float2 zk = x[k], zmc = cconj(x[m]);
      const float2 a = make_float2(0.5f * (zk.x + zmc.x), 0.5f * (zk.y + zmc.y));
      const float2 dd = csub(zk, zmc);
      const float2 b = make_float2(0.5f * dd.y, -0.5f * dd.x);
      const float fa = factor(k, 0), fb = factor(k, hn);
      x[k] = make_float2(a.x * fa - b.y * fb, a.y * fa + b.x * fb);
      if (m != k) {
        const float ga = factor(m, 0), gb = factor(m, hn);  // A_-k = conj A_k, B_-k = conj B_k
        x[m] = make_float2(a.x * ga + b.y * gb, -a.y * ga + b.x * gb);
      }
    }
  }
  __syncthreads();
  fft_lines<1>(x, ncol, n, G.logn, tw_inv_n, ls);
  cl.sync();

  // Row inverse (c2r): gather each row's bins from the owners; the next
  // batch's bins are requested while this batch transforms.
  float2 xk[kPer], xc[kPer];
  auto gather_batch = [&](int b) {
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int e = tid + 256 * i, rr = e / hn, k = e - rr * hn;
      if (k == 0) {  // the packed line: DC in the real part, Nyquist in the imaginary part
        const float2 p = *cl.map_shared_rank(x + b + rr, 0);
        xk[i] = make_float2(p.x, 0.0f);
        xc[i] = make_float2(p.y, 0.0f);
      } else {
        xk[i] = *bin(k, b + rr);
        xc[i] = cconj(*bin(hn - k, b + rr));
      }
    }
  };
  gather_batch(rbeg);
  for (int b0 = rbeg; b0 < rend; b0 += kBfBatch) {
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int e = tid + 256 * i, rr = e / hn, k = e - rr * hn;
      float2 a = xk[i], c = xc[i];
      if (k == 0) {  // c2r ignores the imaginary parts of the DC and Nyquist bins
        a.y = 0.0f;
        c.y = 0.0f;
      }
      const float2 e2 = cadd(a, c);
      const float2 o2 = cmul(csub(a, c), split_inv[k]);
      z[rr * zl + k] = make_float2(e2.x - o2.y, e2.y + o2.x);  // 2E + i 2O
    }
    if (b0 + kBfBatch < rend) gather_batch(b0 + kBfBatch);
    __syncthreads();
    fft_lines<1>(z, kBfBatch, hn, G.logn - 1, tw_inv_hn, zl);
#pragma unroll 4
    for (int i = 0; i < kBfBatch * n / 256; ++i) {
      const int e = tid + 256 * i, rr = e / n, m = e - rr * n;
      const float2 v = z[rr * zl + (m >> 1)];
      dense_out[(static_cast<size_t>(item) * n + b0 + rr) * n + m] = (m & 1) ? v.y : v.x;
    }
    __syncthreads();
  }
  cl.sync();  // this CTA's lines stay alive until every rank has gathered
}

// Overlap-add as a gather (src/noise.cpp:430-479): every frame pixel sums the
// Hann-weighted outputs of the (at most 3 x 3) blocks covering it in colour
// order q = (ix % 3) * 3 + (iy % 3) -- the order of the reference's 9-colour
// passes -- with the same float rounding after each block, then divides by the
// separable weight sum. bout holds each block's raw c2r output (item x n x n).
// One CTA per tile of kOlaTW columns x kOlaTH rows, one thread per column: a
// thread finds its column's covering blocks (in colour order) and their Hann
// weights once, the CTA finds each row's once (shared memory), and every pixel
// then reads only its block outputs.
constexpr int kOlaTW = 128;
constexpr int kOlaTH = 16;

// Covering origins of coordinate c, in colour order (index % 3 = 0, 1, 2):
// idx[k] (or -1) and the offset inside the block. Origins are ascending and
// the covering ones form a run of at most 3.
__device__ __forceinline__ void ola_cover(int c, const int* __restrict__ o, int no, int n, int (&idx)[3],
                                          int (&off)[3]) {
  const int s = max(n / 2, 1);
  int hi = min(c / s, no - 1);
  while (hi + 1 < no && o[hi + 1] <= c) ++hi;
  while (hi > 0 && o[hi] > c) --hi;
  int lo = hi;
  while (lo > 0 && lo > hi - 2 && o[lo - 1] + n > c) --lo;
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const int ix = hi - (((hi - r) % 3) + 3) % 3;
    idx[r] = ix >= lo ? ix : -1;
    off[r] = ix >= lo ? c - o[ix] : 0;
  }
}

__global__ void __launch_bounds__(kOlaTW)
k_ola_gather(int w, int h, int n, const int* __restrict__ oxs, int nox, const int* __restrict__ oys, int noy,
             const double* __restrict__ hwin, const float* __restrict__ bout, const double* __restrict__ bnum,
             const double* __restrict__ wx_total, const double* __restrict__ wy_total, float* __restrict__ acc,
             float* __restrict__ var_acc) {
  __shared__ int r_iy[kOlaTH][3], r_ly[kOlaTH][3];
  __shared__ double r_wyt[kOlaTH];
  const int x = blockIdx.x * kOlaTW + threadIdx.x;
  const int y0 = blockIdx.y * kOlaTH;
  if (threadIdx.x < kOlaTH && y0 + static_cast<int>(threadIdx.x) < h) {
    const int y = y0 + threadIdx.x;
    int iy[3], ly[3];
    ola_cover(y, oys, noy, n, iy, ly);
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      r_iy[threadIdx.x][r] = iy[r];
      r_ly[threadIdx.x][r] = ly[r];
    }
    r_wyt[threadIdx.x] = wy_total[y];
  }
  __syncthreads();
  if (x >= w) return;
  int ix[3], lx[3];
  ola_cover(x, oxs, nox, n, ix, lx);
  double wxv[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) wxv[r] = ix[r] >= 0 ? hwin[lx[r]] : 0.0;
  const double wxt = wx_total[x];
  const double inv_n2 = static_cast<double>(1.0f / static_cast<float>(static_cast<size_t>(n) * n));
  const int rows = min(kOlaTH, h - y0);
  for (int t = 0; t < rows; ++t) {
    const int y = y0 + t;
    float a = 0.0f, v = 0.0f;
#pragma unroll
    for (int ca = 0; ca < 3; ++ca) {  // colour q = (ix % 3) * 3 + (iy % 3), ascending
      if (ix[ca] < 0) continue;
#pragma unroll
      for (int cb = 0; cb < 3; ++cb) {
        const int iy = r_iy[t][cb];
        if (iy < 0) continue;
        const int item = iy * nox + ix[ca];
        const int ly = r_ly[t][cb];
        const float f = bout[(static_cast<size_t>(item) * n + ly) * n + lx[ca]];
        const double num = bnum[item];
        const double wy_sig = hwin[ly] * inv_n2;
        const double wy_var = hwin[ly];
        a = static_cast<float>(static_cast<double>(a) + wy_sig * wxv[ca] * static_cast<double>(f));
        v = static_cast<float>(static_cast<double>(v) + wy_var * wxv[ca] * num);
      }
    }
    const double ws = r_wyt[t] * wxt;
    const size_t o = static_cast<size_t>(y) * w + x;
    if (ws > 0.0) {
      acc[o] = static_cast<float>(static_cast<double>(a) / ws);
      var_acc[o] = static_cast<float>(static_cast<double>(v) / ws);
    } else {
      acc[o] = 0.0f;
      var_acc[o] = 0.0f;
    }
  }
}

// Subsampled block noise: upper median of finite positive var[y][x] over the
// block's step-(n/64) grid (src/noise.cpp:200-224). One CTA per (block, layer):
// samples go to fixed slots (invalid ones as +inf, which rank last), the valid
// count comes from a block reduction, and an 8-bit radix select in shared
// memory returns the element of rank count / 2 -- the same value a sort gives.
__global__ void __launch_bounds__(512)
k_block_var(FftGeom G, const float* __restrict__ vs, const float* __restrict__ vr, int w, int h,
            const int* __restrict__ oxs, const int* __restrict__ oys, int nox, int nitem, double* __restrict__ vsr) {
  extern __shared__ uint32_t keys[];
  __shared__ unsigned hist[256];
  __shared__ unsigned s_rank, s_prefix, s_cnt;
  const int item = blockIdx.x, layer = blockIdx.y;
  const float* var = layer == 0 ? vs : vr;
  const int n = G.n;
  const int step = max(1, n / 64);
  const int ns = (n + step - 1) / step;
  const int m = ns * ns;
  int bx, by;
  if (item < nitem) {
    bx = oxs[item % nox];
    by = oys[item / nox];
  } else {  // the whiten_score_psf window
    bx = G.extra_bx;
    by = G.extra_by;
  }
  unsigned mine = 0;
  for (int e = threadIdx.x; e < m; e += blockDim.x) {
    const int yy = by + (e / ns) * step, xx = bx + (e % ns) * step;
    float v = INFINITY;
    if (yy >= 0 && yy < h && xx >= 0 && xx < w) {
      const float x = var[static_cast<size_t>(yy) * w + xx];
      if (isfinite(x) && x > 0.0f) {
        v = x;
        ++mine;
      }
    }
    keys[e] = __float_as_uint(v);  // positive floats (and +inf) order as their bit patterns
  }
  if (threadIdx.x == 0) s_cnt = 0;
  __syncthreads();
  const unsigned wsum = __reduce_add_sync(0xffffffffu, mine);
  if ((threadIdx.x & 31) == 0) atomicAdd(&s_cnt, wsum);
  __syncthreads();
  const unsigned cnt = s_cnt;
  if (cnt == 0) {
    if (threadIdx.x == 0) vsr[2 * item + layer] = 0.0;
    return;
  }
  if (threadIdx.x == 0) {
    s_rank = cnt / 2;
    s_prefix = 0;
  }
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const unsigned prefix = s_prefix;
    const unsigned himask = shift >= 24 ? 0u : (0xffffffffu << (shift + 8));
    for (int e = threadIdx.x; e < m; e += blockDim.x) {
      const uint32_t k = keys[e];
      if ((k & himask) == (prefix & himask)) atomicAdd(&hist[(k >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // one warp: 8 bins per lane, warp prefix sums, pick the digit holding the rank
      const int lane = threadIdx.x;
      unsigned local = 0;
      for (int j = 0; j < 8; ++j) local += hist[lane * 8 + j];
      unsigned incl = local;
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      const unsigned excl = incl - local;
      const unsigned rank = s_rank;
      const bool here = rank >= excl && rank < incl;
      const unsigned who = __ballot_sync(0xffffffffu, here);
      if (here) {
        unsigned cum = excl;
        int d = lane * 8;
        for (int j = 0; j < 8; ++j, ++d) {
          const unsigned c = hist[d];
          if (rank < cum + c) break;
          cum += c;
        }
        s_rank = rank - cum;
        s_prefix = prefix | (static_cast<unsigned>(d) << shift);
      }
      (void)who;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) vsr[2 * item + layer] = static_cast<double>(__uint_as_float(s_prefix));
}

// Local kernel per cell: K = sum_n float(a_n(cx,cy)) phi_n (exact thin-plate
// fields at the cell's representative block centre), sum K^2 in FP64, and its
// zero-phase embedding into an n x n real image (src/noise.cpp:65-84, 167-189,
// 329-343). `dense` must be zeroed beforehand.
__global__ void __launch_bounds__(256)
k_local_kernels(FftGeom G, TpsDev t, const double* __restrict__ theta, int nc, const float* __restrict__ phi,
                int ks, const double* __restrict__ centres, double* __restrict__ sumk2, float* __restrict__ dense,
                float* __restrict__ kern_out) {
  extern __shared__ float kk[];
  __shared__ float an[64];
  __shared__ double red[256];
  const int cell = blockIdx.x, n = G.n;
  if (threadIdx.x == 0) {
    double d[64];
    const double cx = centres[2 * cell], cy = centres[2 * cell + 1];
    const int k = t.k, nr = k - 3;
    const double ux = (cx - t.cx) / t.scale, uy = (cy - t.cy) / t.scale;
    for (int m = 0; m < nr; ++m) d[m] = 0.0;
    for (int j = 0; j < k; ++j) {
      const double dx = ux - t.kn[2 * j], dy = uy - t.kn[2 * j + 1];
      const double r2 = dx * dx + dy * dy;
      const double s = r2 <= 0.0 ? 0.0 : 0.5 * r2 * log(r2);
      for (int m = 0; m < nr; ++m) d[m] = fma(s, t.z[j * nr + m], d[m]);
    }
    d[nr] = 1.0;
    d[nr + 1] = ux;
    d[nr + 2] = uy;
    for (int q = 0; q < nc; ++q) {
      double f = 0.0;
      for (int m = 0; m < k; ++m) f = fma(d[m], theta[q * k + m], f);
      an[q] = static_cast<float>(f);
    }
  }
  __syncthreads();
  const int r = ks / 2;
  double part = 0.0;
  for (int i = threadIdx.x; i < ks * ks; i += blockDim.x) {
    float v = 0.0f;
    for (int q = 0; q < nc; ++q) v = __fmaf_rn(an[q], phi[static_cast<size_t>(q) * ks * ks + i], v);
    kk[i] = v;
    part = fma(static_cast<double>(v), static_cast<double>(v), part);
    const int ky = i / ks, kx = i - ky * ks;
    const int gy = ((ky - r) % n + n) % n, gx = ((kx - r) % n + n) % n;
    if (dense) dense[(static_cast<size_t>(cell) * n + gy) * n + gx] = v;
    if (kern_out) kern_out[static_cast<size_t>(cell) * ks * ks + i] = v;
  }
  red[threadIdx.x] = part;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < static_cast<unsigned>(o)) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0 && sumk2) sumk2[cell] = red[0];
}

// Normalise by the separable Hann weight sum (src/noise.cpp:458-479).
__global__ void k_ola_normalise(int w, int h, const double* __restrict__ wx_total, const double* __restrict__ wy_total,
                                float* __restrict__ acc, float* __restrict__ var_acc) {
  const int64_t n = static_cast<int64_t>(w) * h;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int x = static_cast<int>(i % w), y = static_cast<int>(i / w);
    const double ws = wy_total[y] * wx_total[x];
    if (ws > 0.0) {
      acc[i] = static_cast<float>(static_cast<double>(acc[i]) / ws);
      var_acc[i] = static_cast<float>(static_cast<double>(var_acc[i]) / ws);
    } else {
      acc[i] = 0.0f;
      var_acc[i] = 0.0f;
    }
  }
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
static size_t rows_smem(const FftGeom& g) {
  const int hn = g.n / 2;
  return sizeof(float2) * (static_cast<size_t>(g.rows_per_cta) * fft_ls(hn, false) + hn / 2 + 1 + hn + 1);
}
static size_t cols_smem(const FftGeom& g) {
  return sizeof(float2) * (static_cast<size_t>(g.cols_per_cta) * fft_ls(g.n, true) + g.n / 2 + 1);
}

size_t twiddle_table_len(int n) { return static_cast<size_t>(n) + n / 2 + 2 * (n / 2 + 1); }

void launch_twiddle_table(cudaStream_t s, int n, float2* tab) {
  k_twiddle_table<<<1, 256, 0, s>>>(n, tab);
  DGPU_LAUNCH("k_twiddle_table");
}

FftGeom make_fft_geom(int n) {
  FftGeom g;
  g.n = n;
  g.logn = 0;
  while ((1 << g.logn) < n) ++g.logn;
  g.rows_per_cta = std::max(1, std::min(n, 16384 / std::max(n / 2, 1)));  // <= 128 KB of spectrum
  g.rows_per_cta = std::min(g.rows_per_cta, 64);
  g.cols_per_cta = std::max(1, std::min(n / 2 + 1, 8192 / n));
  return g;
}

void launch_rows_fwd(cudaStream_t s, const FftGeom& g, int mode, int nitems, const float* src, int w, int h,
                     const int* oxs, const int* oys, int nox, float2* spec) {
  const size_t smem = rows_smem(g);
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_rows_fwd), smem);
  dim3 grid(nitems, (g.n + g.rows_per_cta - 1) / g.rows_per_cta);
  k_rows_fwd<<<grid, 256, smem, s>>>(g, mode, src, w, h, oxs, oys, nox, spec);
  DGPU_LAUNCH("k_rows_fwd");
}

void launch_cols(cudaStream_t s, const FftGeom& g, int mode, int nitems, float2* spec, const double* cell_power,
                 const double* cell_sumk2, const int* block_cell, const double* vsr, double* power_out) {
  const size_t smem = cols_smem(g);
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_cols), smem);
  dim3 grid(nitems, (g.n / 2 + 1 + g.cols_per_cta - 1) / g.cols_per_cta);
  k_cols<<<grid, 256, smem, s>>>(g, mode, spec, cell_power, cell_sumk2, block_cell, vsr, power_out);
  DGPU_LAUNCH("k_cols");
}

void launch_rows_inv(cudaStream_t s, const FftGeom& g, int mode, int nitems, const float2* spec, const int* items,
                     int w, int h, const int* oxs, const int* oys, int nox, const double* hwin, const double* vsr,
                     const double* cell_sumk2, const int* block_cell, float* acc, float* var_acc, float* dense_out) {
  if (nitems == 0) return;
  const size_t smem = rows_smem(g);
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_rows_inv), smem);
  dim3 grid(nitems, (g.n + g.rows_per_cta - 1) / g.rows_per_cta);
  k_rows_inv<<<grid, 256, smem, s>>>(g, mode, spec, items, w, h, oxs, oys, nox, hwin, vsr, cell_sumk2, block_cell,
                                     acc, var_acc, dense_out);
  DGPU_LAUNCH("k_rows_inv");
}

void launch_block_var(cudaStream_t s, const FftGeom& g, int nitems, int nextra, const float* vs, const float* vr,
                      int w, int h, const int* oxs, const int* oys, int nox, double* vsr) {
  const int step = std::max(1, g.n / 64);
  const int ns = (g.n + step - 1) / step;
  const size_t smem = sizeof(uint32_t) * static_cast<size_t>(ns) * ns;
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_block_var), smem);
  dim3 grid(nitems + nextra, 2);
  k_block_var<<<grid, 512, smem, s>>>(g, vs, vr, w, h, oxs, oys, nox, nitems, vsr);
  DGPU_LAUNCH("k_block_var");
}

void launch_local_kernels(cudaStream_t s, const FftGeom& g, int ncell, const TpsDev& t, const double* theta, int nc,
                          const float* phi, int ks, const double* centres, double* sumk2, float* dense,
                          float* kern_out) {
  const size_t smem = sizeof(float) * static_cast<size_t>(ks) * ks;
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_local_kernels), smem);
  k_local_kernels<<<ncell, 256, smem, s>>>(g, t, theta, nc, phi, ks, centres, sumk2, dense, kern_out);
  DGPU_LAUNCH("k_local_kernels");
}

bool block_filter_fused(const FftGeom& g) { return g.n == kBfN && g.tw_tab != nullptr; }

void launch_block_filter(cudaStream_t s, const FftGeom& g, int nitems, const float* src, int w, int h,
                         const int* oxs, const int* oys, int nox, const double* cell_power, const double* cell_sumk2,
                         const int* block_cell, const double* vsr, double* bnum, float* dense_out) {
  if (!block_filter_fused(g)) fail(DGPU_ERR_INVALID, "decorrelate: fused block filter needs n = 256 and a twiddle table");
  if (nitems == 0) return;
  const size_t smem = sizeof(float2) * (static_cast<size_t>(kBfCols) * fft_ls(kBfN, true) +
                                        static_cast<size_t>(kBfBatch) * fft_ls(kBfN / 2, false) + twiddle_table_len(kBfN));
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_block_filter), smem);
  k_block_filter<<<nitems * kBfRanks, 256, smem, s>>>(g, src, w, h, oxs, oys, nox, cell_power, cell_sumk2, block_cell,
                                                       vsr, bnum, dense_out);
  DGPU_LAUNCH("k_block_filter");
}

void launch_ola_gather(cudaStream_t s, int w, int h, int n, const int* oxs, int nox, const int* oys, int noy,
                       const double* hwin, const float* bout, const double* bnum, const double* wx_total,
                       const double* wy_total, float* acc, float* var_acc) {
  if (w <= 0 || h <= 0) return;
  const dim3 grid(static_cast<unsigned>(ceil_div(w, kOlaTW)), static_cast<unsigned>(ceil_div(h, kOlaTH)));
  k_ola_gather<<<grid, kOlaTW, 0, s>>>(w, h, n, oxs, nox, oys, noy, hwin, bout, bnum, wx_total, wy_total, acc,
                                       var_acc);
  DGPU_LAUNCH("k_ola_gather");
}

void launch_ola_normalise(cudaStream_t s, int w, int h, const double* wx_total, const double* wy_total, float* acc,
                          float* var_acc) {
  const int64_t n = static_cast<int64_t>(w) * h;
  const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, 148 * 16));
  k_ola_normalise<<<blocks, 256, 0, s>>>(w, h, wx_total, wy_total, acc, var_acc);
  DGPU_LAUNCH("k_ola_normalise");
}

}  // namespace dgpu
