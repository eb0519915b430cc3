// Stamp selection on the device (reference src/detect.cpp:84-314) and the
// median PSF stamp of the score path (python/delta/pipeline.py:285-302).
//
//  * background: median and 1.4826 * MAD of a flat-index-strided sample of the
//    finite, unmasked pixels (step n / 2^18), by exact radix select;
//  * peaks: 3x3 strict local maxima above median + k sigma inside the border,
//    with a fully on-frame, finite, unmasked, unsaturated stamp footprint;
//  * per-candidate flux-weighted second-moment FWHM (FP64);
//  * candidates sorted by flux descending (raster index ascending on ties),
//    then brightest-first greedy isolation in one CTA, chunk by chunk.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <string>

#include "dev_common.cuh"
#include "select_internal.h"
#include "detect_internal.h"

namespace dgpu {

// ---------------------------------------------------------------------------
// Sample medians: the radix select of k_select.cu on a flat-index-strided
// sample, and the absolute-deviation transform for the MAD.
// ---------------------------------------------------------------------------
// keys <- key(|value - med|) in place (src/detect.cpp:110).
__global__ void k_abs_dev(const RadixSelect* st, const float* __restrict__ med, uint32_t* __restrict__ keys) {
  const unsigned count = st->count;
  const float m = *med;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    keys[i] = float_key(fabsf(key_float(keys[i]) - m));
}

static void select_median(cudaStream_t s, RadixSelect* st, const uint32_t* keys, int64_t cap, float* out) {
  launch_select_upper_median(s, st, keys, cap, out);
}

// bgout[0] = median (float), bgout[1] = MAD (float)
void launch_background(Context& c, int64_t n, const float* img, const uint8_t* mask, float* bgout, Slot sel_slot,
                       Slot key_slot) {
  cudaStream_t s = c.stream;
  constexpr int64_t kTarget = 1 << 18;
  const int64_t step = n > kTarget ? n / kTarget : 1;
  const int64_t ns = (n + step - 1) / step;
  RadixSelect* st = static_cast<RadixSelect*>(c.slot(sel_slot, sizeof(RadixSelect)));
  uint32_t* keys = static_cast<uint32_t*>(c.slot(key_slot, sizeof(uint32_t) * std::max<int64_t>(ns, 1)));
  DGPU_CUDA(cudaMemsetAsync(st, 0, sizeof(RadixSelect), s));
  const int blocks = static_cast<int>(std::min<int64_t>((ns + 255) / 256, 148 * 8));
  launch_sample_keys(s, n, step, img, mask, keys, st);
  select_median(s, st, keys, ns, bgout);
  k_abs_dev<<<std::max(blocks, 1), 256, 0, s>>>(st, bgout, keys);
  DGPU_LAUNCH("k_abs_dev");
  select_median(s, st, keys, ns, bgout + 1);
}

// ---------------------------------------------------------------------------
// Candidates
// ---------------------------------------------------------------------------
__device__ bool footprint_ok_dev(const float* img, const uint8_t* mask, int w, int h, int x, int y, int r,
                                 double sat) {
  if (x - r < 0 || x + r >= w || y - r < 0 || y + r >= h) return false;
  for (int dy = -r; dy <= r; ++dy)
    for (int dx = -r; dx <= r; ++dx) {
      const size_t i = static_cast<size_t>(y + dy) * w + (x + dx);
      const float v = img[i];
      if (!isfinite(v)) return false;
      if (mask && mask[i] != 0) return false;
      if (sat > 0.0 && static_cast<double>(v) >= sat) return false;
    }
  return true;
}

// estimate_fwhm (src/detect.cpp:115-157), FP64.
__device__ double fwhm_dev(const float* img, int w, int h, int x, int y, int r, double bg) {
  double sum = 0.0, sx = 0.0, sy = 0.0;
  for (int dy = -r; dy <= r; ++dy) {
    const int yy = y + dy;
    if (yy < 0 || yy >= h) continue;
    for (int dx = -r; dx <= r; ++dx) {
      const int xx = x + dx;
      if (xx < 0 || xx >= w) continue;
      const double f = static_cast<double>(img[static_cast<size_t>(yy) * w + xx]) - bg;
      const double wt = f > 0.0 ? f : 0.0;
      sum += wt;
      sx += wt * dx;
      sy += wt * dy;
    }
  }
  if (sum <= 0.0) return __longlong_as_double(0x7ff8000000000000ll);
  const double mx = sx / sum, my = sy / sum;
  double sxx = 0.0, syy = 0.0;
  for (int dy = -r; dy <= r; ++dy) {
    const int yy = y + dy;
    if (yy < 0 || yy >= h) continue;
    for (int dx = -r; dx <= r; ++dx) {
      const int xx = x + dx;
      if (xx < 0 || xx >= w) continue;
      const double f = static_cast<double>(img[static_cast<size_t>(yy) * w + xx]) - bg;
      const double wt = f > 0.0 ? f : 0.0;
      sxx += wt * (dx - mx) * (dx - mx);
      syy += wt * (dy - my) * (dy - my);
    }
  }
  const double var = 0.5 * (sxx / sum + syy / sum);
  if (var <= 0.0) return __longlong_as_double(0x7ff8000000000000ll);
  return 2.354820045030949 * sqrt(var);
}

__global__ void k_peaks(int w, int h, const float* __restrict__ img, const float* __restrict__ bg,
                        DetectParamsDev p, unsigned* count, int cap, int* __restrict__ cand) {
  const double med = static_cast<double>(bg[0]);
  const double sigma = 1.4826 * static_cast<double>(bg[1]);
  const double thr = med + p.threshold_sigma * (sigma > 0.0 ? sigma : 1.0);
  const int b = p.border;
  const int64_t n = static_cast<int64_t>(w) * h;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int x = static_cast<int>(i % w), y = static_cast<int>(i / w);
    if (y < b || y >= h - b || x < b || x >= w - b) continue;
    if (x < 1 || y < 1 || x >= w - 1 || y >= h - 1) continue;  // 3x3 window on frame
    const double v = static_cast<double>(img[i]);
    if (!(v > thr)) continue;
    bool peak = true;
    for (int dy = -1; dy <= 1 && peak; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        if (dx == 0 && dy == 0) continue;
        if (static_cast<double>(img[i + static_cast<int64_t>(dy) * w + dx]) > v) {
          peak = false;
          break;
        }
      }
    if (!peak) continue;
    const unsigned slot = atomicAdd(count, 1u);
    if (static_cast<int>(slot) < cap) cand[slot] = static_cast<int>(i);
  }
}

// Stamp footprint of every 3x3 peak, one warp per peak: fully on the frame,
// finite, unmasked and below saturation (src/detect.cpp:190-214).
__global__ void k_footprint(int w, int h, const float* __restrict__ img, const uint8_t* __restrict__ mask,
                            DetectParamsDev p, const unsigned* __restrict__ n_peaks, int cap,
                            const int* __restrict__ peaks, unsigned* count, int* __restrict__ cand) {
  const int lane = threadIdx.x & 31;
  const int nwarp = static_cast<int>((gridDim.x * blockDim.x) >> 5);
  const int np = min(static_cast<int>(*n_peaks), cap);
  const int r = p.stamp_radius;
  for (int c = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5); c < np; c += nwarp) {
    const int i = peaks[c];
    const int x = i % w, y = i / w;
    if (x - r < 0 || x + r >= w || y - r < 0 || y + r >= h) continue;
    bool ok = true;
    for (int dy = -r; dy <= r && ok; ++dy) {
      for (int dx = lane - r; dx <= r; dx += 32) {
        const size_t j = static_cast<size_t>(y + dy) * w + (x + dx);
        const float v = img[j];
        if (!isfinite(v) || (mask && mask[j] != 0) || (p.saturation > 0.0 && static_cast<double>(v) >= p.saturation))
          ok = false;
      }
      ok = __all_sync(0xffffffffu, ok);
    }
    if (ok && lane == 0) {
      const unsigned slot = atomicAdd(count, 1u);
      if (static_cast<int>(slot) < cap) cand[slot] = i;
    }
  }
}

// Sort keys: (flux descending, index ascending) -> ascending uint64.
__global__ void k_cand_keys(const unsigned* count, int cap, const int* __restrict__ cand, const float* __restrict__ img,
                            unsigned long long* __restrict__ keys, int* __restrict__ vals) {
  const int nc = min(static_cast<int>(*count), cap);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
    const int idx = cand[i];
    const uint32_t fk = ~float_key(img[idx]);  // descending value
    keys[i] = (static_cast<unsigned long long>(fk) << 32) | static_cast<unsigned>(idx);
    vals[i] = idx;
  }
}

// Brightest-first greedy isolation (src/detect.cpp:223-240) in one CTA.
// Output: kept raster indices in order; *n_kept.
__global__ void __launch_bounds__(1024)
k_isolate(int w, const unsigned* count, int cap, const int* __restrict__ sorted_idx, long long iso2, int max_stamps,
          int* __restrict__ kept, int* n_kept, unsigned* status) {
  extern __shared__ int ks[];  // kept x, y interleaved (2 * max_stamps)
  __shared__ int s_nk;
  __shared__ unsigned char pass[1024];
  __shared__ int cx[1024], cy[1024];
  const int nc = min(static_cast<int>(*count), cap);
  if (threadIdx.x == 0) s_nk = 0;
  __syncthreads();
  for (int base = 0; base < nc; base += blockDim.x) {
    if (s_nk >= max_stamps) break;
    const int i = base + threadIdx.x;
    bool ok = false;
    if (i < nc) {
      const int idx = sorted_idx[i];
      const int x = idx % w, y = idx / w;
      cx[threadIdx.x] = x;
      cy[threadIdx.x] = y;
      ok = true;
      const int nk = s_nk;
      for (int k = 0; k < nk; ++k) {
        const long long dx = x - ks[2 * k], dy = y - ks[2 * k + 1];
        if (dx * dx + dy * dy < iso2) {
          ok = false;
          break;
        }
      }
    }
    pass[threadIdx.x] = ok ? 1 : 0;
    __syncthreads();
    // Sequential resolution within the chunk by warp 0.
    if (threadIdx.x < 32) {
      const int lim = min(static_cast<int>(blockDim.x), nc - base);
      int nk = s_nk;
      const int chunk_start = nk;
      // The candidates that passed, in order, 32 flags per ballot.
      for (int t0 = 0; t0 < lim && nk < max_stamps; t0 += 32) {
        unsigned todo = __ballot_sync(0xffffffffu, t0 + static_cast<int>(threadIdx.x) < lim && pass[t0 + threadIdx.x]);
        while (todo && nk < max_stamps) {
          const int t = t0 + __ffs(todo) - 1;
          todo &= todo - 1;
          bool iso = true;
          for (int k = chunk_start + threadIdx.x; k < nk; k += 32) {
            const long long dx = cx[t] - ks[2 * k], dy = cy[t] - ks[2 * k + 1];
            if (dx * dx + dy * dy < iso2) iso = false;
          }
          iso = __all_sync(0xffffffffu, iso);
          if (iso) {
            if (threadIdx.x == 0) {
              ks[2 * nk] = cx[t];
              ks[2 * nk + 1] = cy[t];
              kept[nk] = cy[t] * w + cx[t];
            }
            __syncwarp();
            ++nk;
          }
        }
      }
      if (threadIdx.x == 0) s_nk = nk;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *n_kept = s_nk;
  (void)status;
}

// One CTA per kept stamp: the threads stage the clipped weights
// max(f - bg, 0) of the FWHM window in shared memory (0 off the frame, which
// adds an exact zero where the reference skips the pixel), then thread 0 runs
// the two FP64 moment passes of fwhm_dev in the same (dy, dx) order.
__global__ void __launch_bounds__(256) k_stamp_props(int w, int h, const float* __restrict__ img,
                                                      const float* __restrict__ bg, const int* __restrict__ kept,
                                                      const int* __restrict__ n_kept, int fwhm_radius,
                                                      double* __restrict__ flux, double* __restrict__ snr,
                                                      double* __restrict__ fwhm) {
  extern __shared__ double wt[];  // (2r+1)^2
  const int i = blockIdx.x;
  if (i >= *n_kept) return;
  const double med = static_cast<double>(bg[0]);
  const double sigma = 1.4826 * static_cast<double>(bg[1]);
  const int idx = kept[i];
  const int x = idx % w, y = idx / w;
  const int r = fwhm_radius, side = 2 * r + 1;
  for (int e = threadIdx.x; e < side * side; e += blockDim.x) {
    const int yy = y - r + e / side, xx = x - r + e % side;
    double v = 0.0;
    if (yy >= 0 && yy < h && xx >= 0 && xx < w) {
      const double f = static_cast<double>(img[static_cast<size_t>(yy) * w + xx]) - med;
      v = f > 0.0 ? f : 0.0;
    }
    wt[e] = v;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const double f0 = static_cast<double>(img[idx]) - med;
  flux[i] = f0;
  snr[i] = sigma > 0.0 ? f0 / sigma : f0;
  double sum = 0.0, sx = 0.0, sy = 0.0;
  for (int dy = -r; dy <= r; ++dy)
    for (int dx = -r; dx <= r; ++dx) {
      const double wv = wt[(dy + r) * side + dx + r];
      sum += wv;
      sx += wv * dx;
      sy += wv * dy;
    }
  double out = __longlong_as_double(0x7ff8000000000000ll);
  if (sum > 0.0) {
    const double mx = sx / sum, my = sy / sum;
    double sxx = 0.0, syy = 0.0;
    for (int dy = -r; dy <= r; ++dy)
      for (int dx = -r; dx <= r; ++dx) {
        const double wv = wt[(dy + r) * side + dx + r];
        sxx += wv * (dx - mx) * (dx - mx);
        syy += wv * (dy - my) * (dy - my);
      }
    const double var = 0.5 * (sxx / sum + syy / sum);
    if (var > 0.0) out = 2.354820045030949 * sqrt(var);
  }
  fwhm[i] = out;
}

// Catalog positions: footprint check on both images + FWHM on both
// (select_stamps_from_catalog, src/detect.cpp:289-314).
__global__ void k_catalog_stamps(int w, int h, const float* __restrict__ sci, const uint8_t* __restrict__ sm,
                                 const float* __restrict__ ref, const uint8_t* __restrict__ rm,
                                 const float* __restrict__ bg_sci, const float* __restrict__ bg_ref,
                                 const int* __restrict__ xs, const int* __restrict__ ys, int n, DetectParamsDev p,
                                 int* __restrict__ ok, double* __restrict__ fs, double* __restrict__ fr) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int x = xs[i], y = ys[i];
    const bool good = footprint_ok_dev(sci, sm, w, h, x, y, p.stamp_radius, p.saturation) &&
                      footprint_ok_dev(ref, rm, w, h, x, y, p.stamp_radius, p.saturation);
    ok[i] = good ? 1 : 0;
    if (good) {
      fs[i] = fwhm_dev(sci, w, h, x, y, p.fwhm_radius, static_cast<double>(bg_sci[0]));
      fr[i] = fwhm_dev(ref, w, h, x, y, p.fwhm_radius, static_cast<double>(bg_ref[0]));
    }
  }
}

// Median unit-sum PSF of the listed stamps (python/delta/pipeline.py:285-302):
// per stamp cut - median(cut) normalised by its positive total; per pixel the
// median across stamps (mean of the two middle values for an even count),
// clipped at 0 and renormalised. FP64. One CTA per stamp, then one per pixel.
__global__ void k_psf_stamps(int w, int h, const float* __restrict__ img, const int* __restrict__ xs,
                             const int* __restrict__ ys, int n, int radius, double* __restrict__ cuts,
                             int* __restrict__ use) {
  extern __shared__ double sv[];  // side^2 padded to a power of two
  const int s = blockIdx.x;
  const int side = 2 * radius + 1, np = side * side;
  int cap = 1;
  while (cap < np) cap <<= 1;
  const int x = xs[s], y = ys[s];
  const bool inside = !(x - radius < 0 || x + radius >= w || y - radius < 0 || y + radius >= h);
  if (!inside) {
    if (threadIdx.x == 0) use[s] = 0;
    return;
  }
  double* srt = sv + cap;
  for (int i = threadIdx.x; i < cap; i += blockDim.x) {
    double v = INFINITY;
    if (i < np) v = static_cast<double>(img[static_cast<size_t>(y - radius + i / side) * w + (x - radius + i % side)]);
    sv[i] = v;
    srt[i] = v;
  }
  __syncthreads();
  for (int size = 2; size <= cap; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < cap; i += blockDim.x) {
        const int j = i ^ stride;
        if (j > i) {
          const bool up = (i & size) == 0;
          const double a = srt[i], b = srt[j];
          if ((a > b) == up) {
            srt[i] = b;
            srt[j] = a;
          }
        }
      }
      __syncthreads();
    }
  const double med = (np & 1) ? srt[np / 2] : 0.5 * (srt[np / 2 - 1] + srt[np / 2]);
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int i = 0; i < np; ++i) tot += sv[i] - med;
    use[s] = tot > 0.0 ? 1 : 0;
    srt[0] = tot;
  }
  __syncthreads();
  const double tot = srt[0];
  for (int i = threadIdx.x; i < np; i += blockDim.x) cuts[static_cast<size_t>(s) * np + i] = (sv[i] - med) / tot;
}

// Median over the used stamps of pixel p (a CTA per pixel): each used value's
// rank among the used values (ties broken by stamp index) is counted in
// parallel; the values of rank cnt/2 (and cnt/2 - 1) give the median.
__global__ void __launch_bounds__(256) k_psf_median(int n, int np, const double* __restrict__ cuts,
                                                     const int* __restrict__ use, double* __restrict__ out,
                                                     unsigned* status) {
  extern __shared__ double col[];
  int* used = reinterpret_cast<int*>(col + n);
  const int p = blockIdx.x;
  __shared__ int cnt;
  __shared__ double lo, hi;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int mine = 0;
  for (int s = threadIdx.x; s < n; s += blockDim.x) {
    const int u = use[s] != 0;
    used[s] = u;
    col[s] = u ? cuts[static_cast<size_t>(s) * np + p] : 0.0;
    mine += u;
  }
  atomicAdd(&cnt, mine);
  __syncthreads();
  const int c = cnt;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    if (!used[i]) continue;
    const double v = col[i];
    int rank = 0;
    for (int j = 0; j < n; ++j)
      if (used[j] && (col[j] < v || (col[j] == v && j < i))) ++rank;
    if (rank == c / 2) hi = v;
    if (rank == c / 2 - 1) lo = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    if (c > 0) m = (c & 1) ? hi : 0.5 * (lo + hi);
    out[p] = m > 0.0 ? m : 0.0;
    if (c == 0) atomicOr(status, kStatusBounds);
  }
}

void launch_psf_estimate(Context& c, int w, int h, const float* img, const int* xs, const int* ys, int n, int radius,
                         double* out, int* n_used) {
  cudaStream_t s = c.stream;
  const int side = 2 * radius + 1, np = side * side;
  int cap = 1;
  while (cap < np) cap <<= 1;
  double* cuts = static_cast<double*>(c.slot(kSlotScratch0, sizeof(double) * static_cast<size_t>(std::max(n, 1)) * np));
  int* use = static_cast<int*>(c.slot(kSlotBlockCounts, sizeof(int) * std::max(n, 1)));
  const size_t smem = sizeof(double) * 2 * cap;
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_psf_stamps), smem);
  k_psf_stamps<<<n, 256, smem, s>>>(w, h, img, xs, ys, n, radius, cuts, use);
  DGPU_LAUNCH("k_psf_stamps");
  const size_t smem2 = (sizeof(double) + sizeof(int)) * std::max(n, 1);
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_psf_median), smem2);
  k_psf_median<<<np, 256, smem2, s>>>(n, np, cuts, use, out, c.d_status);
  DGPU_LAUNCH("k_psf_median");
  std::vector<int> hu(n);
  if (n) read_back(c, hu.data(), use, sizeof(int) * n);
  sync_reads(c);
  int u = 0;
  for (int v : hu) u += v;
  *n_used = u;
}

// weighted_mean (src/bindings.cpp:107-124): FP64 partial sums per CTA.
__global__ void k_weighted_mean(int64_t n, const float* __restrict__ d, const float* __restrict__ v,
                                const uint8_t* __restrict__ m, double* __restrict__ part) {
  __shared__ double s1[256], s2[256];
  double a = 0.0, b = 0.0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (m[i] != 0) continue;
    if (!(v[i] > 0.0f)) continue;
    const double wv = 1.0 / static_cast<double>(v[i]);
    a += wv;
    b += wv * static_cast<double>(d[i]);
  }
  s1[threadIdx.x] = a;
  s2[threadIdx.x] = b;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < static_cast<unsigned>(o)) {
      s1[threadIdx.x] += s1[threadIdx.x + o];
      s2[threadIdx.x] += s2[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s1[0];
    part[2 * blockIdx.x + 1] = s2[0];
  }
}

void launch_weighted_mean(Context& c, int64_t n, const float* d, const float* v, const uint8_t* m, double* out2) {
  const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, 296));
  double* part = static_cast<double*>(c.slot(kSlotScratch1, sizeof(double) * 2 * blocks));
  k_weighted_mean<<<blocks, 256, 0, c.stream>>>(n, d, v, m, part);
  DGPU_LAUNCH("k_weighted_mean");
  std::vector<double> hp(2 * blocks);
  read_back(c, hp.data(), part, sizeof(double) * 2 * blocks);
  sync_reads(c);
  double a = 0.0, b = 0.0;
  for (int i = 0; i < blocks; ++i) {
    a += hp[2 * i];
    b += hp[2 * i + 1];
  }
  out2[0] = a;
  out2[1] = b;
}

// The detect pipeline of one image in three phases, each ending in read-backs
// that the caller's sync_reads completes: (1) background, 3x3 peaks and the
// footprint test -> candidate counts; (2) brightest-first sort and greedy
// isolation -> kept count; (3) the kept stamps' flux, S/N and FWHM. Two
// images (their own workspace slots, `which` 0 and 1) can run phase by phase
// so that they share each synchronisation.
struct DetectJob {
  const float* img;
  const uint8_t* mask;
  int which;
  DetectHost* res;
  float* bg;
  unsigned* count;
  int *cand, *sorted, *kept, *vals, *nk;
  unsigned long long *keys, *keys2;
  unsigned hc[2] = {0, 0};
  float hbg[2] = {0.0f, 0.0f};
  int nkept = 0;
  std::vector<int> hk;
};
constexpr int kDetectCap = 1 << 20;

static void detect_phase1(Context& c, int w, int h, const DetectParamsDev& p, DetectJob& j) {
  cudaStream_t s = c.stream;
  const int64_t n = static_cast<int64_t>(w) * h;
  const Slot ss = j.which ? kSlotFit12 : kSlotFit10, ks = j.which ? kSlotFit13 : kSlotFit11;
  j.bg = static_cast<float*>(c.slot(j.which ? kSlotFit15 : kSlotFit14, 64));
  launch_background(c, n, j.img, j.mask, j.bg, ss, ks);
  const int cap = kDetectCap;
  char* buf = static_cast<char*>(
      c.slot(j.which ? kSlotFft1 : kSlotFft0, (sizeof(int) * 3 + 2 * sizeof(unsigned long long)) * cap + 256));
  j.count = reinterpret_cast<unsigned*>(buf);
  j.cand = reinterpret_cast<int*>(buf + 64);
  j.sorted = j.cand + cap;
  j.kept = j.sorted + cap;
  j.keys = reinterpret_cast<unsigned long long*>(j.kept + cap);
  j.keys2 = j.keys + cap;
  j.vals = static_cast<int*>(c.slot(j.which ? kSlotFft3 : kSlotFft2, sizeof(int) * cap + 64));
  j.nk = j.vals + cap;
  unsigned* n_peaks = j.count + 1;  // 3x3 peaks before the footprint test; `sorted` holds them until the sort
  DGPU_CUDA(cudaMemsetAsync(j.count, 0, 2 * sizeof(unsigned), s));
  const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, 148 * 16));
  k_peaks<<<blocks, 256, 0, s>>>(w, h, j.img, j.bg, p, n_peaks, cap, j.sorted);
  DGPU_LAUNCH("k_peaks");
  k_footprint<<<148 * 8, 256, 0, s>>>(w, h, j.img, j.mask, p, n_peaks, cap, j.sorted, j.count, j.cand);
  DGPU_LAUNCH("k_footprint");
  read_back(c, j.hc, j.count, 2 * sizeof(unsigned));
  read_back(c, j.hbg, j.bg, sizeof(j.hbg));
}

// After phase 1's sync. Returns whether a read-back was queued.
static bool detect_phase2(Context& c, int w, const DetectParamsDev& p, DetectJob& j) {
  cudaStream_t s = c.stream;
  const int cap = kDetectCap;
  if (j.hc[1] > static_cast<unsigned>(cap)) fail(DGPU_ERR_RUNTIME, "detect_stamps: more than 2^20 peak candidates");
  const int nc = static_cast<int>(j.hc[0]);
  j.nkept = 0;
  if (nc <= 0) return false;
  k_cand_keys<<<(nc + 255) / 256, 256, 0, s>>>(j.count, cap, j.cand, j.img, j.keys, j.vals);
  DGPU_LAUNCH("k_cand_keys");
  size_t tmp_bytes = 0;
  DGPU_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, j.keys, j.keys2, j.vals, j.sorted, nc, 0, 64, s));
  void* tmp = c.slot(j.which ? kSlotFft5 : kSlotFft4, tmp_bytes + 16);
  DGPU_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, j.keys, j.keys2, j.vals, j.sorted, nc, 0, 64, s));
  const long long iso = p.isolation_radius;
  const size_t smem = sizeof(int) * 2 * std::max(p.max_stamps, 1);
  if (smem > 160 * 1024) fail(DGPU_ERR_INVALID, "detect_stamps: max_stamps above 20480 is not supported");
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_isolate), smem);
  k_isolate<<<1, 1024, smem, s>>>(w, j.count, cap, j.sorted, iso * iso, p.max_stamps, j.kept, j.nk, c.d_status);
  DGPU_LAUNCH("k_isolate");
  read_back(c, &j.nkept, j.nk, sizeof(int));
  return true;
}

// After phase 2's sync. Returns whether a read-back was queued.
static bool detect_phase3(Context& c, int w, int h, const DetectParamsDev& p, DetectJob& j) {
  cudaStream_t s = c.stream;
  DetectHost& res = *j.res;
  res.median = static_cast<double>(j.hbg[0]);
  res.sigma = 1.4826 * static_cast<double>(j.hbg[1]);
  const int nkept = j.nkept;
  res.x.assign(nkept, 0);
  res.y.assign(nkept, 0);
  res.flux.assign(nkept, 0);
  res.snr.assign(nkept, 0);
  res.fwhm.assign(nkept, 0);
  if (nkept <= 0) return false;
  double* props =
      static_cast<double*>(c.slot(j.which ? kSlotCompOut : kSlotCompStats, sizeof(double) * 3 * nkept));
  const size_t psmem = sizeof(double) * static_cast<size_t>(2 * p.fwhm_radius + 1) * (2 * p.fwhm_radius + 1);
  if (psmem > 200 * 1024) fail(DGPU_ERR_INVALID, "detect_stamps: fwhm_radius too large");
  ensure_dynamic_smem(reinterpret_cast<const void*>(k_stamp_props), psmem);
  k_stamp_props<<<nkept, 256, psmem, s>>>(w, h, j.img, j.bg, j.kept, j.nk, p.fwhm_radius, props, props + nkept,
                                          props + 2 * nkept);
  DGPU_LAUNCH("k_stamp_props");
  j.hk.assign(nkept, 0);
  read_back(c, j.hk.data(), j.kept, sizeof(int) * nkept);
  read_back(c, res.flux.data(), props, sizeof(double) * nkept);
  read_back(c, res.snr.data(), props + nkept, sizeof(double) * nkept);
  read_back(c, res.fwhm.data(), props + 2 * nkept, sizeof(double) * nkept);
  return true;
}

static void detect_finish(int w, DetectJob& j) {
  for (int i = 0; i < j.nkept; ++i) {
    j.res->x[i] = j.hk[i] % w;
    j.res->y[i] = j.hk[i] / w;
  }
}

// Full detect pipeline for one image. Returns the kept count; host copies of
// x, y, flux, snr, fwhm in `res`.
int run_detect(Context& c, int w, int h, const float* img, const uint8_t* mask, const DetectParamsDev& p, int which,
               DetectHost& res) {
  DetectJob j;
  j.img = img;
  j.mask = mask;
  j.which = which;
  j.res = &res;
  detect_phase1(c, w, h, p, j);
  sync_reads(c);
  if (detect_phase2(c, w, p, j)) sync_reads(c);
  if (detect_phase3(c, w, h, p, j)) sync_reads(c);
  detect_finish(w, j);
  return j.nkept;
}

// Both images of a pair, phase by phase: three synchronisations, not six.
void run_detect_pair(Context& c, int w, int h, const float* img0, const uint8_t* mask0, const float* img1,
                     const uint8_t* mask1, const DetectParamsDev& p, DetectHost& res0, DetectHost& res1) {
  DetectJob j[2];
  j[0].img = img0;
  j[0].mask = mask0;
  j[0].which = 0;
  j[0].res = &res0;
  j[1].img = img1;
  j[1].mask = mask1;
  j[1].which = 1;
  j[1].res = &res1;
  detect_phase1(c, w, h, p, j[0]);
  detect_phase1(c, w, h, p, j[1]);
  sync_reads(c);
  bool q = detect_phase2(c, w, p, j[0]);
  q = detect_phase2(c, w, p, j[1]) || q;
  if (q) sync_reads(c);
  q = detect_phase3(c, w, h, p, j[0]);
  q = detect_phase3(c, w, h, p, j[1]) || q;
  if (q) sync_reads(c);
  detect_finish(w, j[0]);
  detect_finish(w, j[1]);
}

void run_background(Context& c, int64_t n, const float* img, const uint8_t* mask, double* median, double* sigma) {
  float* bg = static_cast<float*>(c.slot(kSlotFit14, 64));
  launch_background(c, n, img, mask, bg, kSlotFit10, kSlotFit11);
  float hbg[2];
  read_back(c, hbg, bg, sizeof(hbg));
  sync_reads(c);
  *median = static_cast<double>(hbg[0]);
  *sigma = 1.4826 * static_cast<double>(hbg[1]);
}

void run_catalog_stamps(Context& c, int w, int h, const float* sci, const uint8_t* sm, const float* ref,
                        const uint8_t* rm, const int* xs_host, const int* ys_host, int n, const DetectParamsDev& p,
                        std::vector<int>& ok, std::vector<double>& fs, std::vector<double>& fr, double* med_sci,
                        double* med_ref) {
  cudaStream_t s = c.stream;
  const int64_t npx = static_cast<int64_t>(w) * h;
  float* bgs = static_cast<float*>(c.slot(kSlotFit14, 64));
  float* bgr = static_cast<float*>(c.slot(kSlotFit15, 64));
  launch_background(c, npx, sci, sm, bgs, kSlotFit10, kSlotFit11);
  launch_background(c, npx, ref, rm, bgr, kSlotFit12, kSlotFit13);
  int* dxy = static_cast<int*>(c.slot(kSlotBright, sizeof(int) * 2 * std::max(n, 1)));
  DGPU_CUDA(h2d_async(dxy, xs_host, sizeof(int) * n, s));
  DGPU_CUDA(h2d_async(dxy + n, ys_host, sizeof(int) * n, s));
  char* ob = static_cast<char*>(c.slot(kSlotCompStats, (sizeof(int) + 2 * sizeof(double)) * std::max(n, 1) + 64));
  double* dfs = reinterpret_cast<double*>(ob);
  double* dfr = dfs + std::max(n, 1);
  int* dok = reinterpret_cast<int*>(dfr + std::max(n, 1));
  if (n > 0) {
    k_catalog_stamps<<<(n + 127) / 128, 128, 0, s>>>(w, h, sci, sm, ref, rm, bgs, bgr, dxy, dxy + n, n, p, dok, dfs,
                                                     dfr);
    DGPU_LAUNCH("k_catalog_stamps");
  }
  ok.assign(n, 0);
  fs.assign(n, 0.0);
  fr.assign(n, 0.0);
  float hb[2];
  if (n) {
    read_back(c, ok.data(), dok, sizeof(int) * n);
    read_back(c, fs.data(), dfs, sizeof(double) * n);
    read_back(c, fr.data(), dfr, sizeof(double) * n);
  }
  read_back(c, hb, bgs, sizeof(float) * 2);
  sync_reads(c);
  *med_sci = hb[0];
  read_back(c, hb, bgr, sizeof(float) * 2);
  sync_reads(c);
  *med_ref = hb[0];
}

// ---------------------------------------------------------------------------
// Allocation-free background estimate (dgpu_estimate_background_noalloc).
//
// Same algorithm and kernels as launch_background, with the sample keys and
// the radix-select state in one fixed, file-scope device array instead of the
// context's workspace. The sample has at most 2^19 entries for any frame below
// 2^31 pixels (step = n / 2^18 gives ceil(n / step) < 2^19), so the array is
// 2 MiB + 1 KiB per device. Each call clears the select state (its counter
// must start at zero) on the caller's stream before use. The array is shared
// by every call on a device: calls that overlap in time (other streams or
// threads) race on it and must be serialised by the caller.
// ---------------------------------------------------------------------------
namespace {

constexpr int64_t kNoAllocMaxSamples = int64_t(1) << 19;

struct NoAllocBackground {
  RadixSelect sel;          // count / rank / prefix / histogram: cleared by every call
  float result[4];  // [0] median, [1] MAD
  uint32_t keys[kNoAllocMaxSamples];
};

static __device__ __align__(256) NoAllocBackground g_noalloc_background;

// Device address of the array on the current device. Resolved on every call
// (a cheap lookup, no allocation) rather than cached: after a device reset the
// runtime reloads the module and the array may sit at a new address.
NoAllocBackground* noalloc_background_scratch() {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_background);
  if (e != cudaSuccess)
    fail(DGPU_ERR_CUDA, std::string("estimate_background_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  return static_cast<NoAllocBackground*>(p);
}

}  // namespace

void background_noalloc(int64_t n, const float* img, const uint8_t* mask, cudaStream_t s, float* out2) {
  constexpr int64_t kTarget = 1 << 18;
  const int64_t step = n > kTarget ? n / kTarget : 1;
  const int64_t ns = (n + step - 1) / step;
  if (ns > kNoAllocMaxSamples)
    fail(DGPU_ERR_INVALID, "estimate_background_noalloc: sample exceeds the fixed 2^19-entry scratch");
  NoAllocBackground* sc = noalloc_background_scratch();
  RadixSelect* st = &sc->sel;
  uint32_t* keys = sc->keys;
  float* res = sc->result;
  DGPU_CUDA(cudaMemsetAsync(st, 0, sizeof(RadixSelect), s));
  const int blocks = static_cast<int>(std::min<int64_t>((ns + 255) / 256, 148 * 8));
  launch_sample_keys(s, n, step, img, mask, keys, st);
  select_median(s, st, keys, ns, res);
  k_abs_dev<<<std::max(blocks, 1), 256, 0, s>>>(st, res, keys);
  DGPU_LAUNCH("k_abs_dev");
  select_median(s, st, keys, ns, res + 1);
  DGPU_CUDA(cudaMemcpyAsync(out2, res, 2 * sizeof(float), cudaMemcpyDeviceToHost, s));
  DGPU_CUDA(cudaStreamSynchronize(s));
}

}  // namespace dgpu
