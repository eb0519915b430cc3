// Connected-component source catalog (src/catalog.cpp:61-697) on sm_100a.
//
// Seeds -> 8-connected union-find labelling with atomicMin linking (every
// parent index is below its child, so each component's root is its minimum
// linear index) -> roots ranked in raster order by a block count + scan, which
// reproduces the reference's final numbering exactly (label = rank of the
// component's first pixel in raster order, src/catalog.cpp:124-260) ->
// per-label reductions with atomics (count, |score|-weighted sums in FP64,
// peak with the lowest-index tie-break of src/catalog.cpp:362-371, mask OR over
// footprint + 8-ring) -> per-component finishing (centroid, FWHM consistency,
// aperture flux, quality bits, dipole flag, optional PSF-shape fit and
// bright-star distance). Every data-dependent loop is capped; hitting a cap
// sets the context status word and the call reports DGPU_ERR_LIMIT.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "dev_common.cuh"

namespace dgpu {


__global__ void k_seed(int64_t n, const float* __restrict__ score, const uint8_t* __restrict__ mask,
                       int exclude, float thr_pos, float thr_neg, uint8_t* __restrict__ seeds) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float v = score[i];
    const bool fin = isfinite(v);
    const bool good = !(exclude && mask != nullptr && mask[i] != 0);
    uint8_t s = 0;
    if (fin && v >= thr_pos && good) s |= 1;
    if (fin && v <= -thr_neg && good) s |= 2;
    seeds[i] = s;
  }
}

__device__ __forceinline__ int find_root(const int* L, int i, unsigned* st, int cap) {
  for (int it = 0; it < cap; ++it) {
    const int p = L[i];
    if (p == i) return i;
    i = p;
  }
  set_status(st, kStatusLoopLimit);
  return i;
}

__device__ void unite(int* L, int a, int b, unsigned* st, int cap) {
  for (int it = 0; it < cap; ++it) {
    a = find_root(L, a, st, cap);
    b = find_root(L, b, st, cap);
    if (a == b) return;
    if (a < b) {
      const int t = a;
      a = b;
      b = t;
    }
    const int old = atomicMin(&L[a], b);
    if (old == a) return;
    a = old;
  }
  set_status(st, kStatusLoopLimit);
}

__global__ void k_label_init(int64_t n, const uint8_t* __restrict__ seeds, uint8_t bit, int* __restrict__ L) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    L[i] = (seeds[i] & bit) ? static_cast<int>(i) : -1;
}

__global__ void k_label_merge(int w, int h, const uint8_t* __restrict__ seeds, uint8_t bit, int* L,
                              unsigned* st, int cap) {
  const int64_t n = static_cast<int64_t>(w) * h;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (!(seeds[i] & bit)) continue;
    const int x = static_cast<int>(i % w), y = static_cast<int>(i / w);
    const int me = static_cast<int>(i);
    if (x > 0 && (seeds[i - 1] & bit)) unite(L, me, me - 1, st, cap);
    if (y > 0) {
      const int64_t a = i - w;
      if (x > 0 && (seeds[a - 1] & bit)) unite(L, me, static_cast<int>(a - 1), st, cap);
      if (seeds[a] & bit) unite(L, me, static_cast<int>(a), st, cap);
      if (x + 1 < w && (seeds[a + 1] & bit)) unite(L, me, static_cast<int>(a + 1), st, cap);
    }
  }
}

__global__ void k_label_flatten(int64_t n, int* L, unsigned* st, int cap) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (L[i] >= 0) L[i] = find_root(L, static_cast<int>(i), st, cap);
  }
}

constexpr int kRankBlock = 1024;

__global__ void k_root_count(int64_t n, const int* __restrict__ L, int* __restrict__ counts) {
  __shared__ int s;
  if (threadIdx.x == 0) s = 0;
  __syncthreads();
  const int64_t i = static_cast<int64_t>(blockIdx.x) * kRankBlock + threadIdx.x;
  const bool root = i < n && L[i] == static_cast<int>(i);
  const unsigned bal = __ballot_sync(0xffffffffu, root);
  if ((threadIdx.x & 31) == 0 && bal) atomicAdd(&s, __popc(bal));
  __syncthreads();
  if (threadIdx.x == 0) counts[blockIdx.x] = s;
}

// Exclusive scan of per-block root counts in one CTA; writes the total.
__global__ void k_scan_counts(int nb, int* counts, int* total) {
  __shared__ int part[1024];
  const int per = (nb + blockDim.x - 1) / blockDim.x;
  const int lo = threadIdx.x * per, hi = min(nb, lo + per);
  int s = 0;
  for (int i = lo; i < hi; ++i) s += counts[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int off = 1; off < static_cast<int>(blockDim.x); off <<= 1) {
    const int v = threadIdx.x >= static_cast<unsigned>(off) ? part[threadIdx.x - off] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = part[threadIdx.x] - s;
  for (int i = lo; i < hi; ++i) {
    const int c = counts[i];
    counts[i] = run;
    run += c;
  }
  if (threadIdx.x == blockDim.x - 1) *total = part[threadIdx.x];
}

// rank_at[root] = raster rank of the root (0-based).
__global__ void k_root_rank(int64_t n, const int* __restrict__ L, const int* __restrict__ offsets,
                            int* __restrict__ rank_at) {
  __shared__ int warp_tot[kRankBlock / 32];
  const int64_t i = static_cast<int64_t>(blockIdx.x) * kRankBlock + threadIdx.x;
  const bool root = i < n && L[i] == static_cast<int>(i);
  const unsigned bal = __ballot_sync(0xffffffffu, root);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) warp_tot[wid] = __popc(bal);
  __syncthreads();
  if (wid == 0) {
    int v = warp_tot[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += u;
    }
    warp_tot[lane] = v - warp_tot[lane];  // exclusive
  }
  __syncthreads();
  if (root) rank_at[i] = offsets[blockIdx.x] + warp_tot[wid] + __popc(bal & ((1u << lane) - 1));
}

// Only a root carries a rank, so a pixel maps to a label only through a root:
// one left pointing at a non-root (a capped search gave up) gets label 0 and
// the bounds status, which keeps every label within [1, number of roots].
__global__ void k_label_final(int64_t n, const int* __restrict__ L, const int* __restrict__ rank_at,
                              int* __restrict__ labels, unsigned* st) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int r = L[i];
    int lbl = 0;
    if (r >= 0) {
      if (L[r] == r)
        lbl = rank_at[r] + 1;
      else
        set_status(st, kStatusBounds);
    }
    labels[i] = lbl;
  }
}

// Per-component accumulators (index label-1).
struct CompStats {
  int* count;
  double* sum;
  double* sx;
  double* sy;
  unsigned long long* peak;  // (bits(|score|) << 32) | ~idx -> max gives lowest idx on ties
  unsigned* mask_or;
  unsigned* touched;
  int* first;  // minimum linear index (the root)
};

__global__ void k_comp_reduce(int w, int h, const int* __restrict__ labels, const float* __restrict__ score,
                              const uint8_t* __restrict__ mask, CompStats cs) {
  const int64_t n = static_cast<int64_t>(w) * h;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int lbl = labels[i];
    if (lbl <= 0) continue;
    const int c = lbl - 1;
    const int x = static_cast<int>(i % w), y = static_cast<int>(i / w);
    const double v = static_cast<double>(score[i]);
    const double wt = fabs(v);
    atomicAdd(&cs.count[c], 1);
    atomicAdd(&cs.sum[c], wt);
    atomicAdd(&cs.sx[c], wt * x);
    atomicAdd(&cs.sy[c], wt * y);
    const unsigned long long key =
        (static_cast<unsigned long long>(__float_as_uint(fabsf(score[i]))) << 32) |
        static_cast<unsigned long long>(0xffffffffu - static_cast<unsigned>(i));
    atomicMax(&cs.peak[c], key);
    atomicMin(&cs.first[c], static_cast<int>(i));
    if (mask) {
      unsigned m = mask[i];
      for (int dy = -1; dy <= 1; ++dy) {
        const int yy = y + dy;
        if (yy < 0 || yy >= h) continue;
        for (int dx = -1; dx <= 1; ++dx) {
          if (dx == 0 && dy == 0) continue;
          const int xx = x + dx;
          if (xx < 0 || xx >= w) continue;
          const int64_t j = static_cast<int64_t>(yy) * w + xx;
          if (labels[j] != lbl) m |= mask[j];
        }
      }
      if (m) atomicOr(&cs.mask_or[c], m);
    }
  }
}

// Opposite-polarity seeds touching a label's 3x3 neighbourhood
// (flag_dipole_positives, src/catalog.cpp:431-458).
__global__ void k_dipole_touch(int w, int h, const uint8_t* __restrict__ seeds, uint8_t other_bit,
                               const int* __restrict__ labels, unsigned* touched) {
  const int64_t n = static_cast<int64_t>(w) * h;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (!(seeds[i] & other_bit)) continue;
    const int x = static_cast<int>(i % w), y = static_cast<int>(i / w);
    for (int dy = -1; dy <= 1; ++dy) {
      const int yy = y + dy;
      if (yy < 0 || yy >= h) continue;
      for (int dx = -1; dx <= 1; ++dx) {
        const int xx = x + dx;
        if (xx < 0 || xx >= w) continue;
        const int l = labels[static_cast<int64_t>(yy) * w + xx];
        if (l > 0) touched[l - 1] = 1u;
      }
    }
  }
}

struct CompOut {
  double* x;
  double* y;
  int* peak_x;
  int* peak_y;
  double* peak_snr;
  int* n_pix;
  double* flux;
  double* expected_n_pix;
  double* fwhm_ratio;
  uint8_t* fwhm_consistent;
  uint8_t* mask_flags;
  uint8_t* is_dipole;
  uint8_t* quality;
  double* psf_chi2;
  int* psf_chi2_dof;
  double* psf_amplitude;
  double* psf_amplitude_err;
  uint8_t* shape_consistent;
  double* bright_star_dist;
  uint8_t* near_bright_star;
};

struct FinishParams {
  double threshold;  // the seeding threshold of this polarity
  double expected_fwhm, tol_lo, tol_hi;
  int aperture_radius;
  int do_shape, do_bright;
  double shape_tol, bright_radius;
  int psf_size;
};

__device__ long lround_away(double v) { return static_cast<long>(v >= 0 ? floor(v + 0.5) : -floor(-v + 0.5)); }

// summarize_component (src/catalog.cpp:337-418) finishing + dipole flag +
// enrich_entries (src/catalog.cpp:476-596).
__global__ void k_comp_finish(int ncomp, int w, int h, const float* __restrict__ score,
                              const float* __restrict__ diff, const uint8_t* __restrict__ mask,
                              const float* __restrict__ variance, const float* __restrict__ psf,
                              const double* __restrict__ bx, const double* __restrict__ by, int nb,
                              CompStats cs, FinishParams fp, CompOut o) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncomp) return;
  const double kFwhmPerSigma = 2.354820045030949;
  const double kPi = 3.14159265358979323846;
  const int cnt = cs.count[c];
  const double sum = cs.sum[c];
  const int first = cs.first[c];
  double x = sum > 0.0 ? cs.sx[c] / sum : static_cast<double>(first % w);
  double y = sum > 0.0 ? cs.sy[c] / sum : static_cast<double>(first / w);
  const unsigned long long pk = cs.peak[c];
  const int pidx = static_cast<int>(0xffffffffu - static_cast<unsigned>(pk & 0xffffffffull));
  const double peak_snr = static_cast<double>(score[pidx]);
  o.x[c] = x;
  o.y[c] = y;
  o.peak_x[c] = pidx % w;
  o.peak_y[c] = pidx / w;
  o.peak_snr[c] = peak_snr;
  o.n_pix[c] = cnt;
  const unsigned mflags = cs.mask_or[c] & 0xffu;
  o.mask_flags[c] = static_cast<uint8_t>(mflags);
  const double sigma = fp.expected_fwhm / kFwhmPerSigma;
  const double ratio = fp.threshold > 0.0 ? fabs(peak_snr) / fp.threshold : 0.0;
  const double log_term = ratio > 0.0 ? log(ratio * ratio) : 0.0;
  const double expn = kPi * sigma * sigma * fmax(0.0, log_term);
  const double fr = expn > 0.0 ? cnt / expn : INFINITY;
  const bool consistent = fr >= fp.tol_lo && fr <= fp.tol_hi;
  o.expected_n_pix[c] = expn;
  o.fwhm_ratio[c] = fr;
  o.fwhm_consistent[c] = consistent ? 1 : 0;
  const int radius = fp.aperture_radius > 0 ? fp.aperture_radius
                                            : max(1, static_cast<int>(lround_away(3.0 * sigma)));
  {
    const int x0 = static_cast<int>(lround_away(x)), y0 = static_cast<int>(lround_away(y));
    const double r2 = static_cast<double>(radius) * radius;
    double fsum = 0.0;
    for (int dy = -radius; dy <= radius; ++dy) {
      const int yy = y0 + dy;
      if (yy < 0 || yy >= h) continue;
      for (int dx = -radius; dx <= radius; ++dx) {
        if (dx * dx + dy * dy > r2) continue;
        const int xx = x0 + dx;
        if (xx < 0 || xx >= w) continue;
        const float v = diff[static_cast<int64_t>(yy) * w + xx];
        if (isfinite(v)) fsum += static_cast<double>(v);
      }
    }
    o.flux[c] = fsum;
  }
  uint8_t q = 0;
  if (!consistent) q |= 1u;
  if (mflags != 0) q |= 4u;
  const bool dip = cs.touched[c] != 0;
  o.is_dipole[c] = dip ? 1 : 0;
  if (dip) q |= 2u;
  o.psf_chi2[c] = 0.0;
  o.psf_chi2_dof[c] = 0;
  o.psf_amplitude[c] = 0.0;
  o.psf_amplitude_err[c] = 0.0;
  o.shape_consistent[c] = 1;
  o.bright_star_dist[c] = INFINITY;
  o.near_bright_star[c] = 0;
  if (fp.do_shape) {
    const int ps = fp.psf_size, r = ps / 2;
    const int x0 = static_cast<int>(lround_away(x)), y0 = static_cast<int>(lround_away(y));
    double swdp = 0.0, swpp = 0.0;
    int used = 0;
    for (int pass = 0; pass < 2; ++pass) {
      double amp = pass ? swdp / swpp : 0.0;
      double chi2 = 0.0;
      for (int dy = -r; dy <= r; ++dy) {
        const int yy = y0 + dy;
        if (yy < 0 || yy >= h) continue;
        for (int dx = -r; dx <= r; ++dx) {
          const int xx = x0 + dx;
          if (xx < 0 || xx >= w) continue;
          const int64_t idx = static_cast<int64_t>(yy) * w + xx;
          if (mask && mask[idx] != 0) continue;
          const float v = variance[idx];
          const float d = diff[idx];
          if (!(v > 0.0f) || !isfinite(v) || !isfinite(d)) continue;
          const float p = psf[(dy + r) * ps + (dx + r)];
          if (pass == 0) {
            const double wgt = 1.0 / static_cast<double>(v);
            swdp += wgt * static_cast<double>(d) * p;
            swpp += wgt * static_cast<double>(p) * p;
            ++used;
          } else {
            const double res = static_cast<double>(d) - amp * static_cast<double>(p);
            chi2 += res * res / static_cast<double>(v);
          }
        }
      }
      if (pass == 0 && (used < 3 || !(swpp > 0.0))) break;
      if (pass == 1) {
        o.psf_amplitude[c] = amp;
        o.psf_amplitude_err[c] = sqrt(1.0 / swpp);
        o.psf_chi2[c] = chi2;
        o.psf_chi2_dof[c] = used - 1;
        const bool sc = (used - 1) > 0 ? (chi2 / (used - 1) <= fp.shape_tol) : true;
        o.shape_consistent[c] = sc ? 1 : 0;
        if (!sc) q |= 8u;
      }
    }
  }
  if (fp.do_bright) {
    double best2 = INFINITY;
    for (int i = 0; i < nb; ++i) {
      const double dx = x - bx[i], dy = y - by[i];
      const double d2 = dx * dx + dy * dy;
      if (d2 < best2) best2 = d2;
    }
    const double dist = sqrt(best2);
    o.bright_star_dist[c] = dist;
    const bool near = dist <= fp.bright_radius;
    o.near_bright_star[c] = near ? 1 : 0;
    if (near) q |= 16u;
  }
  o.quality[c] = q;
}

// ---------------------------------------------------------------------------
// Host driver
// ---------------------------------------------------------------------------

static int grid_for(int64_t n, int threads = 256) {
  return static_cast<int>(std::min<int64_t>((n + threads - 1) / threads, 148 * 16));
}

// Label the seeds carrying `bit`; labels written to `labels`, returns count.
static int label_polarity(Context& c, int w, int h, const uint8_t* seeds, uint8_t bit, int* labels) {
  cudaStream_t s = c.stream;
  const int64_t n = static_cast<int64_t>(w) * h;
  int* L = static_cast<int*>(c.slot(kSlotScratch0, sizeof(int) * n));
  int* rank_at = static_cast<int*>(c.slot(kSlotRootRank, sizeof(int) * n));
  const int nb = static_cast<int>((n + kRankBlock - 1) / kRankBlock);
  int* counts = static_cast<int*>(c.slot(kSlotBlockCounts, sizeof(int) * (nb + 2)));
  k_label_init<<<grid_for(n), 256, 0, s>>>(n, seeds, bit, L);
  DGPU_LAUNCH("k_label_init");
  k_label_merge<<<grid_for(n), 256, 0, s>>>(w, h, seeds, bit, L, c.d_status, c.label_loop_cap);
  DGPU_LAUNCH("k_label_merge");
  k_label_flatten<<<grid_for(n), 256, 0, s>>>(n, L, c.d_status, c.label_loop_cap);
  DGPU_LAUNCH("k_label_flatten");
  k_root_count<<<nb, kRankBlock, 0, s>>>(n, L, counts);
  DGPU_LAUNCH("k_root_count");
  k_scan_counts<<<1, 1024, 0, s>>>(nb, counts, counts + nb);
  DGPU_LAUNCH("k_scan_counts");
  k_root_rank<<<nb, kRankBlock, 0, s>>>(n, L, counts, rank_at);
  DGPU_LAUNCH("k_root_rank");
  k_label_final<<<grid_for(n), 256, 0, s>>>(n, L, rank_at, labels, c.d_status);
  DGPU_LAUNCH("k_label_final");
  int total = 0;
  read_back(c, &total, counts + nb, sizeof(int));
  sync_reads(c);
  return total;
}

int run_catalog(Context& c, int w, int h, const float* score, const float* diff, const uint8_t* mask,
                const dgpu_catalog_params& p, const float* variance, const float* psf, int psf_size,
                const double* bright_x, const double* bright_y, int n_bright) {
  cudaStream_t s = c.stream;
  const int64_t n = static_cast<int64_t>(w) * h;
  uint8_t* seeds = static_cast<uint8_t*>(c.slot(kSlotSeedPos, n));
  int* labels = static_cast<int*>(c.slot(kSlotLabels, sizeof(int) * n));
  {
    StageTimer t(c, "catalog: seed");
    k_seed<<<grid_for(n), 256, 0, s>>>(n, score, mask, p.exclude_bad_pixels ? 1 : 0,
                                       static_cast<float>(p.threshold_sigma),
                                       static_cast<float>(p.threshold_sigma_dipole), seeds);
    DGPU_LAUNCH("k_seed");
  }
  const bool neg = p.return_negative != 0;
  const uint8_t bit = neg ? 2 : 1, other = neg ? 1 : 2;
  int ncomp;
  {
    StageTimer t(c, neg ? "catalog: label negative" : "catalog: label positive");
    ncomp = label_polarity(c, w, h, seeds, bit, labels);
  }
  c.cat_npix = n;
  c.cat_count = ncomp;
  c.cat_d.assign(static_cast<size_t>(ncomp) * 12, 0.0);
  c.cat_i.assign(static_cast<size_t>(ncomp) * 4, 0);
  c.cat_u8.assign(static_cast<size_t>(ncomp) * 8, 0);
  if (ncomp == 0) return 0;

  StageTimer t(c, neg ? "catalog: summarize negative" : "catalog: summarize positive");
  // Stats arrays in one slot.
  const size_t nc = static_cast<size_t>(ncomp);
  const size_t stats_bytes = nc * (4 + 8 * 3 + 8 + 4 + 4 + 4) + 256;
  char* sb = static_cast<char*>(c.slot(kSlotCompStats, stats_bytes));
  CompStats cs;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* p2 = sb + off;
    off += (bytes + 15) & ~size_t(15);
    return p2;
  };
  cs.peak = reinterpret_cast<unsigned long long*>(take(8 * nc));
  cs.sum = reinterpret_cast<double*>(take(8 * nc));
  cs.sx = reinterpret_cast<double*>(take(8 * nc));
  cs.sy = reinterpret_cast<double*>(take(8 * nc));
  cs.count = reinterpret_cast<int*>(take(4 * nc));
  cs.mask_or = reinterpret_cast<unsigned*>(take(4 * nc));
  cs.touched = reinterpret_cast<unsigned*>(take(4 * nc));
  size_t zero_bytes = off;
  cs.first = reinterpret_cast<int*>(take(4 * nc));
  (void)stats_bytes;
  DGPU_CUDA(cudaMemsetAsync(sb, 0, zero_bytes, s));
  DGPU_CUDA(cudaMemsetAsync(cs.first, 0x7f, 4 * nc, s));
  k_comp_reduce<<<grid_for(n), 256, 0, s>>>(w, h, labels, score, mask, cs);
  DGPU_LAUNCH("k_comp_reduce");
  k_dipole_touch<<<grid_for(n), 256, 0, s>>>(w, h, seeds, other, labels, cs.touched);
  DGPU_LAUNCH("k_dipole_touch");

  // Output columns: 12 doubles, 4 int32 (peak_x, peak_y, n_pix, psf_chi2_dof), 8 u8.
  const size_t out_bytes = nc * (12 * 8 + 4 * 4 + 8) + 512;
  char* ob = static_cast<char*>(c.slot(kSlotCompOut, out_bytes));
  double* dcol = reinterpret_cast<double*>(ob);
  int* icol = reinterpret_cast<int*>(ob + nc * 12 * 8);
  uint8_t* ucol = reinterpret_cast<uint8_t*>(ob + nc * (12 * 8 + 4 * 4));
  CompOut o;
  o.x = dcol + 0 * nc;
  o.y = dcol + 1 * nc;
  o.peak_snr = dcol + 2 * nc;
  o.flux = dcol + 3 * nc;
  o.expected_n_pix = dcol + 4 * nc;
  o.fwhm_ratio = dcol + 5 * nc;
  o.psf_chi2 = dcol + 6 * nc;
  o.psf_amplitude = dcol + 7 * nc;
  o.psf_amplitude_err = dcol + 8 * nc;
  o.bright_star_dist = dcol + 9 * nc;
  o.peak_x = icol + 0 * nc;
  o.peak_y = icol + 1 * nc;
  o.n_pix = icol + 2 * nc;
  o.psf_chi2_dof = icol + 3 * nc;
  o.fwhm_consistent = ucol + 0 * nc;
  o.mask_flags = ucol + 1 * nc;
  o.is_dipole = ucol + 2 * nc;
  o.quality = ucol + 3 * nc;
  o.shape_consistent = ucol + 4 * nc;
  o.near_bright_star = ucol + 5 * nc;

  FinishParams fp;
  fp.threshold = neg ? p.threshold_sigma_dipole : p.threshold_sigma;
  fp.expected_fwhm = p.expected_fwhm;
  fp.tol_lo = p.fwhm_tolerance_lo;
  fp.tol_hi = p.fwhm_tolerance_hi;
  fp.aperture_radius = p.aperture_radius;
  const bool enrich = ncomp <= std::max(0, p.max_shape_fit);
  fp.do_shape = (enrich && p.fit_psf_shape && psf != nullptr && variance != nullptr && psf_size > 0) ? 1 : 0;
  fp.do_bright = (enrich && bright_x != nullptr && bright_y != nullptr && n_bright > 0) ? 1 : 0;
  fp.shape_tol = p.shape_chi2_tolerance;
  fp.bright_radius = p.bright_star_radius > 0.0 ? p.bright_star_radius : 3.0 * p.expected_fwhm;
  fp.psf_size = psf_size;
  k_comp_finish<<<(ncomp + 127) / 128, 128, 0, s>>>(ncomp, w, h, score, diff, mask, variance, psf,
                                                     bright_x, bright_y, n_bright, cs, fp, o);
  DGPU_LAUNCH("k_comp_finish");
  // Bring the columns back into the context (host).
  std::vector<char> host(out_bytes);
  read_back(c, host.data(), ob, nc * (12 * 8 + 4 * 4 + 8));
  sync_reads(c);
  std::memcpy(c.cat_d.data(), host.data(), nc * 12 * 8);
  std::memcpy(c.cat_i.data(), host.data() + nc * 12 * 8, nc * 4 * 4);
  std::memcpy(c.cat_u8.data(), host.data() + nc * (12 * 8 + 4 * 4), nc * 8);
  return ncomp;
}

}  // namespace dgpu
