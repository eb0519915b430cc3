/* C restatement of the reference's float32 hot loops -- TEST INFRASTRUCTURE.
 *
 * Used as (a) a fast checker for the CUDA path and (b) the timed CPU baseline
 * ("port") in bench.py. Each loop follows the reference's per-pixel
 * accumulation order; the products that the reference build (-O3
 * -march=x86-64-v3, GCC's default -ffp-contract=fast) fuses into FMAs are
 * written as explicit fmaf() so the arithmetic is pinned regardless of how this
 * file itself is vectorised.
 *
 * Fields (a_n, b) are passed either as full-resolution float arrays (the
 * reference's exact small-frame path) or as the FP64 coarse lattice plus the
 * per-axis cell index / weight tables (src/subtract.cpp:167-316).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int exact, nf, w, h;
  const float* full; /* exact: nf * h * w */
  const double* lat; /* coarse: nf * ncy * ncx */
  int ncx, ncy;
  const int* cellx;
  const float* wx;
  const int* celly;
  const float* wy;
} oc_fields;

/* CoarseFields::point, src/subtract.cpp:187-205. */
static inline float field_point(const oc_fields* F, int f, int x, int y) {
  if (F->exact) return F->full[((size_t)f * F->h + y) * F->w + x];
  const int jx = F->cellx[x], jy = F->celly[y];
  const double* c0 = F->lat + ((size_t)f * F->ncy + jy) * F->ncx;
  const double* c1 = c0 + F->ncx;
  const float a00 = (float)c0[jx], a01 = (float)c0[jx + 1];
  const float a10 = (float)c1[jx], a11 = (float)c1[jx + 1];
  const float fy = F->wy[y];
  const float base = fmaf(a10 - a00, fy, a00);
  const float top = a01 - a00;
  const float slope = fmaf((a11 - a10) - top, fy, top);
  return fmaf(slope, F->wx[x], base);
}

static oc_fields make_fields(int exact, int nf, int w, int h, const float* full, const double* lat,
                             int ncx, int ncy, const int* cellx, const float* wx, const int* celly,
                             const float* wy) {
  oc_fields F;
  F.exact = exact; F.nf = nf; F.w = w; F.h = h; F.full = full; F.lat = lat;
  F.ncx = ncx; F.ncy = ncy; F.cellx = cellx; F.wx = wx; F.celly = celly; F.wy = wy;
  return F;
}

/* Full-resolution field f (evaluate_fields / fill_tile), src/subtract.cpp:211-247. */
void oc_field_full(int exact, int nf, int w, int h, const float* full, const double* lat, int ncx,
                   int ncy, const int* cellx, const float* wx, const int* celly, const float* wy,
                   int f, float* out) {
  oc_fields F = make_fields(exact, nf, w, h, full, lat, ncx, ncy, cellx, wx, celly, wy);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) out[(size_t)y * w + x] = field_point(&F, f, x, y);
}

/* Model convolve, src/subtract.cpp:466-639: D = S - b - sum_n a_n B_n with the
 * sanitised reference (fill for masked / non-finite, 0 off-frame), x taps in
 * order j = 0..ks-1 from 0, then per component the clipped y taps, then
 * d -= a_n * bn. taps: (n_max+1) x ks float32; ord_nx/ord_ny: nc orders. */
void oc_subtract_model(const float* sci, const float* ref, const uint8_t* ref_mask, int w, int h,
                       int exact, int nf, const float* full, const double* lat, int ncx, int ncy,
                       const int* cellx, const float* wx, const int* celly, const float* wy,
                       int n_max, int ks, const float* taps, const int* ord_nx, const int* ord_ny,
                       float fill, float* diff) {
  oc_fields F = make_fields(exact, nf, w, h, full, lat, ncx, ncy, cellx, wx, celly, wy);
  const int kh = (ks - 1) / 2;
  const int nc = nf - 1;
  const size_t n = (size_t)w * h;
  float* clean = (float*)malloc(sizeof(float) * n);
  float* tx = (float*)malloc(sizeof(float) * n * (size_t)(n_max + 1));
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; ++i) {
    const float v = ref[i];
    const int bad = (ref_mask && ref_mask[i] != 0) || !isfinite(v);
    clean[i] = bad ? fill : v;
  }
  for (int nx = 0; nx <= n_max; ++nx) {
    const float* k = taps + (size_t)nx * ks;
    float* t = tx + (size_t)nx * n;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < h; ++y) {
      const float* row = clean + (size_t)y * w;
      for (int x = 0; x < w; ++x) {
        float acc = 0.0f;
        for (int j = 0; j < ks; ++j) {
          const int sx = x + kh - j;
          const float v = (sx >= 0 && sx < w) ? row[sx] : 0.0f;
          acc = fmaf(k[j], v, acc);
        }
        t[(size_t)y * w + x] = acc;
      }
    }
  }
#pragma omp parallel for schedule(static)
  for (int y = 0; y < h; ++y) {
    const int jmin = (y + kh - h + 1) > 0 ? (y + kh - h + 1) : 0;
    const int jmax = (ks - 1) < (y + kh) ? (ks - 1) : (y + kh);
    for (int x = 0; x < w; ++x) {
      const size_t i = (size_t)y * w + x;
      float d = sci[i] - field_point(&F, nc, x, y);
      for (int c = 0; c < nc; ++c) {
        const float* ky = taps + (size_t)ord_ny[c] * ks;
        const float* t = tx + (size_t)ord_nx[c] * n;
        float bn = 0.0f;
        for (int j = jmin; j <= jmax; ++j) bn = fmaf(ky[j], t[(size_t)(y + kh - j) * w + x], bn);
        d = fmaf(-field_point(&F, c, x, y), bn, d);
      }
      diff[i] = d;
    }
  }
  free(tx);
  free(clean);
}

/* Variance, src/subtract.cpp:641-824. phi: nc x ks x ks float32 footprints;
 * var_r / var_s may be NULL (var_out is then the science term / zero). */
void oc_variance(const float* var_s, const float* var_r, int w, int h, int exact, int nf,
                 const float* full, const double* lat, int ncx, int ncy, const int* cellx,
                 const float* wx, const int* celly, const float* wy, int rk, const float* phi,
                 float* var_out) {
  oc_fields F = make_fields(exact, nf, w, h, full, lat, ncx, ncy, cellx, wx, celly, wy);
  const int nc = nf - 1;
  const int ks = 2 * rk + 1;
  const size_t kk = (size_t)ks * ks;
  memset(var_out, 0, sizeof(float) * (size_t)w * h);
  if (var_r) {
    const int bsz = 64;
    const int nbx = (w + bsz - 1) / bsz, nby = (h + bsz - 1) / bsz;
#pragma omp parallel for schedule(dynamic)
    for (int bi = 0; bi < nbx * nby; ++bi) {
      const int bx = (bi % nbx) * bsz, by = (bi / nbx) * bsz;
      const int bw = (w - bx) < bsz ? (w - bx) : bsz;
      const int bh = (h - by) < bsz ? (h - by) : bsz;
      const int cpx = (bx + bw / 2) < (w - 1) ? (bx + bw / 2) : (w - 1);
      const int cpy = (by + bh / 2) < (h - 1) ? (by + bh / 2) : (h - 1);
      float* k2 = (float*)calloc(kk, sizeof(float));
      float* kf = (float*)malloc(sizeof(float) * kk);
      for (int c = 0; c < nc; ++c) {
        const float an = field_point(&F, c, cpx, cpy);
        const float* p = phi + (size_t)c * kk;
        for (size_t i = 0; i < kk; ++i) k2[i] = fmaf(an, p[i], k2[i]);
      }
      double qsum = 0.0;
      for (size_t i = 0; i < kk; ++i) {
        const float v = k2[i];
        kf[kk - 1 - i] = v * v;
        qsum = fma((double)v, (double)v, qsum);
      }
      int hw = 0;
      {
        const double target = (1.0 - (double)1e-4f) * qsum;
        for (; hw < rk; ++hw) {
          double box = 0.0;
          const int lo = rk - hw, hi = rk + hw;
          for (int yy = lo; yy <= hi; ++yy)
            for (int xx = lo; xx <= hi; ++xx) box += (double)kf[(size_t)yy * ks + xx];
          if (box >= target) break;
        }
      }
      const int lo = rk - hw, hi = rk + hw;
      const int iwh = bh + 2 * rk, iww = bw + 2 * rk;
      float* win = (float*)malloc(sizeof(float) * (size_t)iwh * iww);
      float wmin = INFINITY, wmax = -INFINITY;
      for (int iy = 0; iy < iwh; ++iy) {
        const int gy = by - rk + iy;
        for (int ix = 0; ix < iww; ++ix) {
          const int gx = bx - rk + ix;
          const float v = (gy < 0 || gy >= h || gx < 0 || gx >= w) ? 0.0f : var_r[(size_t)gy * w + gx];
          win[(size_t)iy * iww + ix] = v;
          if (v < wmin) wmin = v;
          if (v > wmax) wmax = v;
        }
      }
      if (wmax > 0.0f && (wmax - wmin) <= 1e-3f * wmax) {
        const float q = (float)qsum;
        for (int oy = 0; oy < bh; ++oy)
          for (int ox = 0; ox < bw; ++ox)
            var_out[(size_t)(by + oy) * w + bx + ox] =
                fmaf(q, win[(size_t)(oy + rk) * iww + ox + rk], 0.0f);
      } else {
        for (int oy = 0; oy < bh; ++oy)
          for (int ox = 0; ox < bw; ++ox) {
            float acc = 0.0f;
            for (int ly = lo; ly <= hi; ++ly)
              for (int lx = lo; lx <= hi; ++lx) {
                const float c = kf[(size_t)ly * ks + lx];
                if (c == 0.0f) continue;
                acc = fmaf(c, win[(size_t)(oy + ly) * iww + ox + lx], acc);
              }
            var_out[(size_t)(by + oy) * w + bx + ox] = 0.0f + acc;
          }
      }
      free(win);
      free(kf);
      free(k2);
    }
  }
  if (var_s) {
    const size_t n = (size_t)w * h;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i) var_out[i] += var_s[i];
  }
}

/* Mask growth + exact-bad fill, src/subtract.cpp:826-963. Writes mask_out and
 * patches diff / var (var may be NULL). Returns the fill value through *fill. */
static int cmp_float(const void* a, const void* b) {
  const float x = *(const float*)a, y = *(const float*)b;
  return (x > y) - (x < y);
}

void oc_mask(const float* sci, const float* ref, const uint8_t* sm, const uint8_t* rm, int w, int h,
             double saturation, int r, float* diff, float* var, uint8_t* mask_out, float* fill_out) {
  const size_t n = (size_t)w * h;
  const int has_sat = saturation > 0.0;
  const float sat = (float)saturation;
  const int need_grow = rm != NULL || has_sat;
  uint8_t* grow = (uint8_t*)calloc(n, 1);
  uint8_t* tmp = (uint8_t*)calloc(n, 1);
  char* eb = (char*)calloc(n, 1);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; ++i) {
    uint8_t direct = 0, g = 0;
    char e = 0;
    if (sm && sm[i]) { direct |= sm[i]; e = 1; }
    if (rm && rm[i]) { g |= rm[i]; e = 1; }
    if (has_sat) {
      if (ref[i] >= sat) { g |= 2; e = 1; }
      if (sci[i] >= sat) { direct |= 2; e = 1; }
    }
    mask_out[i] = direct;
    grow[i] = g;
    eb[i] = e;
  }
  if (need_grow && r > 0) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) {
        const int x0 = x - r < 0 ? 0 : x - r, x1 = x + r > w - 1 ? w - 1 : x + r;
        uint8_t acc = 0;
        for (int xx = x0; xx <= x1; ++xx) acc |= grow[(size_t)y * w + xx];
        tmp[(size_t)y * w + x] = acc;
      }
#pragma omp parallel for schedule(static)
    for (int y = 0; y < h; ++y) {
      const int y0 = y - r < 0 ? 0 : y - r, y1 = y + r > h - 1 ? h - 1 : y + r;
      for (int x = 0; x < w; ++x) {
        uint8_t acc = 0;
        for (int yy = y0; yy <= y1; ++yy) acc |= tmp[(size_t)yy * w + x];
        grow[(size_t)y * w + x] = acc;
      }
    }
  }
#pragma omp parallel for schedule(static)
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const size_t i = (size_t)y * w + x;
      if (need_grow) mask_out[i] |= grow[i];
      if (x < r || x >= w - r || y < r || y >= h - r) mask_out[i] |= 16;
      if (!isfinite(diff[i])) { mask_out[i] |= 8; eb[i] = 1; }
    }
  const size_t nsamp = (n + 6) / 7;
  float* good = (float*)malloc(sizeof(float) * (nsamp + 1));
  size_t ng = 0;
  for (size_t j = 0; j < nsamp; ++j) {
    const size_t i = 7 * j;
    if (mask_out[i] == 0 && isfinite(diff[i])) good[ng++] = diff[i];
  }
  float fill = 0.0f;
  if (ng) {
    qsort(good, ng, sizeof(float), cmp_float);
    fill = good[ng / 2];
  }
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; ++i) {
    if (mask_out[i] == 0) continue;
    if (eb[i]) {
      diff[i] = fill;
      if (var) var[i] = 0.0f;
    }
  }
  *fill_out = fill;
  free(good);
  free(eb);
  free(tmp);
  free(grow);
}

/* Matched filter, src/noise.cpp:535-632: per pixel, taps in (ly, lx) order
 * skipping zero taps, then acc / sqrt(var * sum psf^2). */
void oc_matched_filter(const float* img, const float* var, int w, int h, const float* psf, int ps,
                       float* out) {
  const int r = ps / 2;
  float sumpsf2 = 0.0f;
  for (int i = 0; i < ps * ps; ++i) sumpsf2 = fmaf(psf[i], psf[i], sumpsf2);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      float acc = 0.0f;
      for (int ly = 0; ly < ps; ++ly) {
        const int gy = y - r + ly;
        for (int lx = 0; lx < ps; ++lx) {
          const float p = psf[ly * ps + lx];
          if (p == 0.0f) continue;
          const int gx = x - r + lx;
          const float v = (gy < 0 || gy >= h || gx < 0 || gx >= w) ? 0.0f : img[(size_t)gy * w + gx];
          acc = fmaf(p, v, acc);
        }
      }
      const float v = var[(size_t)y * w + x];
      out[(size_t)y * w + x] = v > 0.0f ? acc / sqrtf(v * sumpsf2) : 0.0f;
    }
}
