// Host driver of the ZOGY decorrelation (reference src/noise.cpp:228-533,
// src/bindings.cpp:725-874). Block geometry and the Hann tables are tiny host
// tables; all FFT, filter and overlap-add work is on the device (k_fft.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "fft_internal.h"

using namespace dgpu;

namespace {

template <class T>
T* up(Context& c, Slot s, const T* host, size_t n) {
  T* d = static_cast<T*>(c.slot(s, sizeof(T) * std::max<size_t>(n, 1)));
  if (n) DGPU_CUDA(h2d_async(d, host, sizeof(T) * n, c.stream));
  return d;
}

template <class F>
int guarded(dgpu_context* ctx, F&& f) {
  return run_entry(ctx, true, false, std::forward<F>(f));
}

bool pow2(int n) { return n >= 8 && (n & (n - 1)) == 0; }

std::vector<int> origins(int extent, int blk, int strd) {
  std::vector<int> o;
  if (extent <= blk) return {0};
  for (int p = 0; p + blk <= extent; p += strd) o.push_back(p);
  if (o.back() + blk < extent) o.push_back(extent - blk);
  return o;
}

std::vector<double> hann(int n) {
  const double pi = 3.14159265358979323846;
  std::vector<double> h(n);
  for (int i = 0; i < n; ++i) h[i] = 0.5 * (1.0 - std::cos(2.0 * pi * (i + 0.5) / n));
  return h;
}

std::vector<float> phi_of(const Basis& b) {
  std::vector<float> ph(static_cast<size_t>(b.nc) * b.ks * b.ks);
  for (int q = 0; q < b.nc; ++q) {
    const auto k2 = b.kernel2d(q);
    std::copy(k2.begin(), k2.end(), ph.begin() + static_cast<size_t>(q) * b.ks * b.ks);
  }
  return ph;
}

// |Khat|^2 of a host kernel (zero-phase embedded) and sum K^2 into device
// buffers (decorrelation_filter, src/noise.cpp:98-117).
void kernel_power_host(Context& c, const FftGeom& g, const float* kernel, int ks, double* d_power, double* d_sumk2) {
  const int n = g.n, nb = n / 2 + 1;
  std::vector<float> dense(static_cast<size_t>(n) * n, 0.0f);
  double s2 = 0.0;
  const int r = ks / 2;
  for (int ky = 0; ky < ks; ++ky)
    for (int kx = 0; kx < ks; ++kx) {
      const int gy = ((ky - r) % n + n) % n, gx = ((kx - r) % n + n) % n;
      const float v = kernel[ky * ks + kx];
      dense[static_cast<size_t>(gy) * n + gx] = v;
      s2 += static_cast<double>(v) * v;
    }
  float* dd = up(c, kSlotFft3, dense.data(), dense.size());
  float2* spec = static_cast<float2*>(c.slot(kSlotFft4, sizeof(float2) * static_cast<size_t>(n) * nb));
  launch_rows_fwd(c.stream, g, 1, 1, dd, 0, 0, nullptr, nullptr, 1, spec);
  launch_cols(c.stream, g, 1, 1, spec, nullptr, nullptr, nullptr, nullptr, d_power);
  DGPU_CUDA(h2d_async(d_sumk2, &s2, sizeof(double), c.stream));
  DGPU_CUDA(cudaStreamSynchronize(c.stream));
}

}  // namespace

extern "C" {

int dgpu_decorrelate(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* difference,
                     const dgpu_model* model, const float* var_science, const float* var_reference, int block,
                     int kernel_cell_blocks, float* out_difference, float* out_variance) {
  return guarded(ctx, [&](Context& c) {
    if (width <= 0 || height <= 0) fail(DGPU_ERR_INVALID, "image must be non-empty");
    if (!pow2(block)) fail(DGPU_ERR_RUNTIME, "decorrelate: block must be a power of two >= 8");
    if (block > 1024) fail(DGPU_ERR_INVALID, "decorrelate: block above 1024 is not supported");
    if (!difference || !var_science || !var_reference || !model) fail(DGPU_ERR_INVALID, "decorrelate: missing input");
    const int w = static_cast<int>(width), h = static_cast<int>(height);
    const size_t npx = static_cast<size_t>(w) * h;
    const Basis b(model->beta, model->n_max, model->radius);
    const ThinPlate tp(model->knots, model->n_knots);
    const int nc = b.nc;
    if (model->n_theta != static_cast<int64_t>(tp.k) * (nc + 1))
      fail(DGPU_ERR_RUNTIME, "decorrelate: theta size does not match k*(nc+1)");
    cudaStream_t s = c.stream;
    const auto* D = static_cast<const float*>(stage_in(c, mem, difference, 4 * npx, kSlotInSci));
    const auto* vs = static_cast<const float*>(stage_in(c, mem, var_science, 4 * npx, kSlotInVarS));
    const auto* vr = static_cast<const float*>(stage_in(c, mem, var_reference, 4 * npx, kSlotInVarR));
    float* acc = static_cast<float*>(out_buf(c, mem, out_difference, 4 * npx, kSlotOutDiff));
    float* vacc = static_cast<float*>(out_buf(c, mem, out_variance, 4 * npx, kSlotOutVar));
    FftGeom g = make_fft_geom(block);
    float2* twtab = static_cast<float2*>(c.slot(kSlotGlsPart, sizeof(float2) * twiddle_table_len(block)));
    launch_twiddle_table(c.stream, block, twtab);
    g.tw_tab = twtab;
    const int n = block, nb = n / 2 + 1, stride = block / 2;
    const std::vector<int> oxs = origins(w, block, stride), oys = origins(h, block, stride);
    const int nox = static_cast<int>(oxs.size()), noy = static_cast<int>(oys.size());
    const int nblk = nox * noy;
    int kgroup = kernel_cell_blocks;
    if (kgroup <= 0) {
      const double spacing = tp.min_knot_spacing();
      kgroup = 1;
      if (spacing > 0.0 && stride > 0) kgroup = std::max(1, static_cast<int>(std::lround((spacing / 4) / stride)));
    }
    const int ncellx = (nox + kgroup - 1) / kgroup, ncelly = (noy + kgroup - 1) / kgroup;
    const int ncell = ncellx * ncelly;
    std::vector<double> centres(2 * static_cast<size_t>(ncell));
    for (int ci = 0; ci < ncell; ++ci) {
      const int cix = ci % ncellx, ciy = ci / ncellx;
      const int repx = std::min(cix * kgroup + kgroup / 2, nox - 1);
      const int repy = std::min(ciy * kgroup + kgroup / 2, noy - 1);
      centres[2 * ci] = std::clamp(oxs[repx] + block / 2.0, 0.0, w - 1.0);
      centres[2 * ci + 1] = std::clamp(oys[repy] + block / 2.0, 0.0, h - 1.0);
    }
    std::vector<int> block_cell(nblk);
    for (int iy = 0; iy < noy; ++iy)
      for (int ix = 0; ix < nox; ++ix) block_cell[iy * nox + ix] = (iy / kgroup) * ncellx + (ix / kgroup);
    const std::vector<double> hw = hann(n);
    std::vector<double> wxt(w, 0.0), wyt(h, 0.0);
    for (int bx : oxs)
      for (int i = 0; i < n; ++i)
        if (bx + i >= 0 && bx + i < w) wxt[bx + i] += hw[i];
    for (int by : oys)
      for (int i = 0; i < n; ++i)
        if (by + i >= 0 && by + i < h) wyt[by + i] += hw[i];
    // Device tables (one slot, packed).
    std::vector<int> itab;
    itab.insert(itab.end(), oxs.begin(), oxs.end());
    itab.insert(itab.end(), oys.begin(), oys.end());
    itab.insert(itab.end(), block_cell.begin(), block_cell.end());
    int* dit = up(c, kSlotCellX, itab.data(), itab.size());
    const int* d_oxs = dit;
    const int* d_oys = dit + nox;
    const int* d_bcell = d_oys + noy;
    std::vector<double> dtab;
    dtab.insert(dtab.end(), hw.begin(), hw.end());
    dtab.insert(dtab.end(), wxt.begin(), wxt.end());
    dtab.insert(dtab.end(), wyt.begin(), wyt.end());
    dtab.insert(dtab.end(), centres.begin(), centres.end());
    double* ddt = up(c, kSlotLattice, dtab.data(), dtab.size());
    const double* d_hw = ddt;
    const double* d_wxt = d_hw + n;
    const double* d_wyt = d_wxt + w;
    const double* d_cen = d_wyt + h;
    const auto ph = phi_of(b);
    float* d_phi = up(c, kSlotPhi, ph.data(), ph.size());
    double* d_theta = up(c, kSlotTheta, model->theta, static_cast<size_t>(model->n_theta));
    const TpsDev t = upload_tps(c, tp);
    // Per-cell |Khat|^2 and sum K^2.
    double* cell_power = static_cast<double*>(c.slot(kSlotFft5, sizeof(double) * static_cast<size_t>(ncell) * n * nb));
    double* vbuf = static_cast<double*>(c.slot(kSlotFft1, sizeof(double) * (ncell + 2 * static_cast<size_t>(nblk) + 4)));
    double* cell_sumk2 = vbuf;
    double* vsr = vbuf + ncell;
    float2* spec = static_cast<float2*>(
        c.slot(kSlotFft0, sizeof(float2) * static_cast<size_t>(std::max(nblk, ncell)) * n * nb));
    {
      StageTimer tm(c, "decorrelate: kernel-power cache");
      float* dense = static_cast<float*>(c.slot(kSlotFft3, sizeof(float) * static_cast<size_t>(ncell) * n * n));
      DGPU_CUDA(cudaMemsetAsync(dense, 0, sizeof(float) * static_cast<size_t>(ncell) * n * n, s));
      launch_local_kernels(s, g, ncell, t, d_theta, nc, d_phi, b.ks, d_cen, cell_sumk2, dense, nullptr);
      launch_rows_fwd(s, g, 1, ncell, dense, 0, 0, nullptr, nullptr, 1, spec);
      launch_cols(s, g, 1, ncell, spec, nullptr, nullptr, nullptr, nullptr, cell_power);
    }
    {
      StageTimer tm(c, "decorrelate: block filter+blend");
      launch_block_var(s, g, nblk, 0, vs, vr, w, h, d_oxs, d_oys, nox, vsr);
      double* bnum = static_cast<double*>(c.slot(kSlotFft2, sizeof(double) * static_cast<size_t>(nblk)));
      // Raw c2r outputs of every block, then the overlap-add as a per-pixel gather
      // in the reference's colour order (same sums as 9 colour passes).
      float* bout = static_cast<float*>(c.slot(kSlotFft4, sizeof(float) * static_cast<size_t>(nblk) * n * n));
      if (block_filter_fused(g)) {
        launch_block_filter(s, g, nblk, D, w, h, d_oxs, d_oys, nox, cell_power, cell_sumk2, d_bcell, vsr, bnum, bout);
      } else {
        launch_rows_fwd(s, g, 0, nblk, D, w, h, d_oxs, d_oys, nox, spec);
        launch_cols(s, g, 0, nblk, spec, cell_power, cell_sumk2, d_bcell, vsr, bnum);
        launch_rows_inv(s, g, 2, nblk, spec, nullptr, w, h, d_oxs, d_oys, nox, d_hw, vsr, cell_sumk2, d_bcell,
                        nullptr, nullptr, bout);
      }
    }
    {
      StageTimer tm(c, "decorrelate: normalise");
      launch_ola_gather(s, w, h, n, d_oxs, nox, d_oys, noy, d_hw,
                        static_cast<const float*>(c.slot(kSlotFft4, sizeof(float) * static_cast<size_t>(nblk) * n * n)),
                        static_cast<const double*>(c.slot(kSlotFft2, sizeof(double) * static_cast<size_t>(nblk))),
                        d_wxt, d_wyt, acc, vacc);
    }
    stage_out(c, mem, out_difference, acc, 4 * npx);
    stage_out(c, mem, out_variance, vacc, 4 * npx);
    if (mem == DGPU_MEM_HOST) check_status(c);
    (void)nb;
  });
}

int dgpu_whiten_score_psf(dgpu_context* ctx, int mem, const float* psf, int psf_size, const dgpu_model* model,
                          int64_t width, int64_t height, const float* var_science, const float* var_reference,
                          int block, float* out) {
  return guarded(ctx, [&](Context& c) {
    if (psf_size < 1 || !psf) fail(DGPU_ERR_INVALID, "whiten_score_psf: psf must be non-empty");
    if (block < psf_size) fail(DGPU_ERR_RUNTIME, "whiten_score_psf: block must be >= psf side");
    if (!pow2(block) || block > 1024) fail(DGPU_ERR_RUNTIME, "whiten_score_psf: block must be a power of two in [8, 1024]");
    const int w = static_cast<int>(width), h = static_cast<int>(height);
    const size_t npx = static_cast<size_t>(w) * h;
    const Basis b(model->beta, model->n_max, model->radius);
    const ThinPlate tp(model->knots, model->n_knots);
    const int nc = b.nc, n = block, nb = n / 2 + 1;
    if (model->n_theta != static_cast<int64_t>(tp.k) * (nc + 1))
      fail(DGPU_ERR_RUNTIME, "whiten_score_psf: theta size does not match k*(nc+1)");
    cudaStream_t s = c.stream;
    const auto* vs = static_cast<const float*>(stage_in(c, mem, var_science, 4 * npx, kSlotInVarS));
    const auto* vr = static_cast<const float*>(stage_in(c, mem, var_reference, 4 * npx, kSlotInVarR));
    FftGeom g = make_fft_geom(n);
    g.extra_bx = std::max(0, w / 2 - block / 2);
    g.extra_by = std::max(0, h / 2 - block / 2);
    const double cen[2] = {0.5 * static_cast<double>(w - 1), 0.5 * static_cast<double>(h - 1)};
    double* dcen = up(c, kSlotLattice, cen, 2);
    const auto ph = phi_of(b);
    float* d_phi = up(c, kSlotPhi, ph.data(), ph.size());
    double* d_theta = up(c, kSlotTheta, model->theta, static_cast<size_t>(model->n_theta));
    const TpsDev t = upload_tps(c, tp);
    // dense: [0] kernel embedding, [1] psf embedding
    float* dense = static_cast<float*>(c.slot(kSlotFft3, sizeof(float) * 2 * static_cast<size_t>(n) * n));
    DGPU_CUDA(cudaMemsetAsync(dense, 0, sizeof(float) * 2 * static_cast<size_t>(n) * n, s));
    double* small = static_cast<double*>(c.slot(kSlotFft1, sizeof(double) * 8));
    double* sumk2 = small;
    double* vsr = small + 2;  // (vs, vr) of the centre window
    launch_local_kernels(s, g, 1, t, d_theta, nc, d_phi, b.ks, dcen, sumk2, dense, nullptr);
    {
      std::vector<float> pe(static_cast<size_t>(n) * n, 0.0f);
      const int r = psf_size / 2;
      for (int py = 0; py < psf_size; ++py)
        for (int px = 0; px < psf_size; ++px) {
          const int gy = ((py - r) % n + n) % n, gx = ((px - r) % n + n) % n;
          pe[static_cast<size_t>(gy) * n + gx] = psf[py * psf_size + px];
        }
      DGPU_CUDA(h2d_async(dense + static_cast<size_t>(n) * n, pe.data(), sizeof(float) * pe.size(), s));
      DGPU_CUDA(cudaStreamSynchronize(s));
    }
    launch_block_var(s, g, 0, 1, vs, vr, w, h, nullptr, nullptr, 1, vsr - 0);
    float2* spec = static_cast<float2*>(c.slot(kSlotFft0, sizeof(float2) * 2 * static_cast<size_t>(n) * nb));
    double* power = static_cast<double*>(c.slot(kSlotFft5, sizeof(double) * static_cast<size_t>(n) * nb));
    launch_rows_fwd(s, g, 1, 2, dense, 0, 0, nullptr, nullptr, 1, spec);
    launch_cols(s, g, 1, 1, spec, nullptr, nullptr, nullptr, nullptr, power);
    int zero = 0;
    int* dz = up(c, kSlotCellY, &zero, 1);
    float2* spec_psf = spec + static_cast<size_t>(n) * nb;
    launch_cols(s, g, 0, 1, spec_psf, power, sumk2, dz, vsr, nullptr);
    float* outd = static_cast<float*>(c.slot(kSlotFft4, sizeof(float) * static_cast<size_t>(n) * n));
    launch_rows_inv(s, g, 1, 1, spec_psf, nullptr, 0, 0, nullptr, nullptr, 1, nullptr, nullptr, nullptr, nullptr,
                    nullptr, nullptr, outd);
    std::vector<float> full(static_cast<size_t>(n) * n);
    read_back(c, full.data(), outd, sizeof(float) * full.size());
    sync_reads(c);
    // Centre crop and unit-sum renormalisation (src/noise.cpp:515-531).
    const int r = psf_size / 2;
    double sum = 0.0;
    for (int py = 0; py < psf_size; ++py)
      for (int px = 0; px < psf_size; ++px) {
        const int gy = ((py - r) % n + n) % n, gx = ((px - r) % n + n) % n;
        const float v = full[static_cast<size_t>(gy) * n + gx];
        out[py * psf_size + px] = v;
        sum += static_cast<double>(v);
      }
    if (sum > 0.0) {
      const float inv = static_cast<float>(1.0 / sum);
      for (int i = 0; i < psf_size * psf_size; ++i) out[i] *= inv;
    }
    check_status(c);
  });
}

int dgpu_decorrelate_block(dgpu_context* ctx, const float* image, int n, const float* kernel, int ksize,
                           double var_science, double var_reference, float* out) {
  return guarded(ctx, [&](Context& c) {
    if (!pow2(n) || n > 1024) fail(DGPU_ERR_INVALID, "decorrelate_block: n must be a power of two in [8, 1024]");
    const FftGeom g = make_fft_geom(n);
    const int nb = n / 2 + 1;
    double* power = static_cast<double*>(c.slot(kSlotFft5, sizeof(double) * static_cast<size_t>(n) * nb));
    double* small = static_cast<double*>(c.slot(kSlotFft1, sizeof(double) * 8));
    kernel_power_host(c, g, kernel, ksize, power, small);
    const double vsr[2] = {var_science, var_reference};
    DGPU_CUDA(h2d_async(small + 2, vsr, sizeof(vsr), c.stream));
    int zero = 0;
    int* dz = up(c, kSlotCellY, &zero, 1);
    float* img = up(c, kSlotFft3, image, static_cast<size_t>(n) * n);
    float2* spec = static_cast<float2*>(c.slot(kSlotFft0, sizeof(float2) * static_cast<size_t>(n) * nb));
    launch_rows_fwd(c.stream, g, 1, 1, img, 0, 0, nullptr, nullptr, 1, spec);
    launch_cols(c.stream, g, 0, 1, spec, power, small, dz, small + 2, nullptr);
    float* outd = static_cast<float*>(c.slot(kSlotFft4, sizeof(float) * static_cast<size_t>(n) * n));
    launch_rows_inv(c.stream, g, 1, 1, spec, nullptr, 0, 0, nullptr, nullptr, 1, nullptr, nullptr, nullptr, nullptr,
                    nullptr, nullptr, outd);
    read_back(c, out, outd, sizeof(float) * static_cast<size_t>(n) * n);
    check_status(c);
  });
}

int dgpu_decorrelation_kernel(dgpu_context* ctx, const float* kernel, int ksize, double var_science,
                              double var_reference, int n, float* out) {
  return guarded(ctx, [&](Context& c) {
    if (!pow2(n) || n > 1024) fail(DGPU_ERR_INVALID, "decorrelation_kernel: n must be a power of two in [8, 1024]");
    const FftGeom g = make_fft_geom(n);
    const int nb = n / 2 + 1;
    double* power = static_cast<double*>(c.slot(kSlotFft5, sizeof(double) * static_cast<size_t>(n) * nb));
    double* small = static_cast<double*>(c.slot(kSlotFft1, sizeof(double) * 8));
    kernel_power_host(c, g, kernel, ksize, power, small);
    const double vsr[2] = {var_science, var_reference};
    DGPU_CUDA(h2d_async(small + 2, vsr, sizeof(vsr), c.stream));
    int zero = 0;
    int* dz = up(c, kSlotCellY, &zero, 1);
    float2* spec = static_cast<float2*>(c.slot(kSlotFft0, sizeof(float2) * static_cast<size_t>(n) * nb));
    launch_cols(c.stream, g, 2, 1, spec, power, small, dz, small + 2, nullptr);
    float* outd = static_cast<float*>(c.slot(kSlotFft4, sizeof(float) * static_cast<size_t>(n) * n));
    launch_rows_inv(c.stream, g, 1, 1, spec, nullptr, 0, 0, nullptr, nullptr, 1, nullptr, nullptr, nullptr, nullptr,
                    nullptr, nullptr, outd);
    std::vector<float> full(static_cast<size_t>(n) * n);
    read_back(c, full.data(), outd, sizeof(float) * full.size());
    sync_reads(c);
    const int half = n / 2;
    for (int y = 0; y < n; ++y)
      for (int x = 0; x < n; ++x)
        out[static_cast<size_t>(y) * n + x] = full[static_cast<size_t>((y + half) % n) * n + (x + half) % n];
    check_status(c);
  });
}

}  // extern "C"
