// C-ABI entry point of the kernel-model chi^2 and its gradients
// (dgpu_kernel_chi2, include/delta_gpu.h; kernels in k_grad.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "grad_internal.h"

using namespace dgpu;

namespace {

template <class F>
int guarded(dgpu_context* ctx, F&& f) {
  return run_entry(ctx, false, false, std::forward<F>(f));
}

// Fields of the identity theta on F's lattice geometry (or at every pixel on
// the exact path): field j is the j-th thin-plate design function, blended the
// same way as the model's fields, so it is the adjoint's interpolation weight.
DevFields design_fields(Context& c, const ThinPlate& tp, const DevFields& F, int w, int h) {
  const int k = tp.k;
  std::vector<double> eye(static_cast<size_t>(k) * k, 0.0);
  for (int j = 0; j < k; ++j) eye[static_cast<size_t>(j) * k + j] = 1.0;
  double* d_eye = static_cast<double*>(c.slot(kSlotGrad0, sizeof(double) * eye.size()));
  DGPU_CUDA(h2d_async(d_eye, eye.data(), sizeof(double) * eye.size(), c.stream));
  const TpsDev t = upload_tps(c, tp);
  DevFields D = F;
  D.nf = k;
  if (F.exact) {
    float* full = static_cast<float*>(c.slot(kSlotGrad1, sizeof(float) * static_cast<size_t>(k) * w * h));
    launch_exact_fields(c.stream, t, d_eye, k, w, h, full);
    D.full = full;
    return D;
  }
  const size_t nl = static_cast<size_t>(k) * F.ncx * F.ncy;
  double* lat = static_cast<double*>(c.slot(kSlotGrad1, sizeof(double) * nl));
  float* latf = static_cast<float*>(c.slot(kSlotGrad2, sizeof(float) * nl));
  launch_lattice(c.stream, t, d_eye, k, F.gx, F.gy, F.ncx, F.ncy, lat, latf);
  D.lat = lat;
  D.latf = latf;
  return D;
}

}  // namespace

extern "C" {

int dgpu_kernel_chi2(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* science,
                     const float* reference, const uint8_t* reference_mask, const float* weights,
                     const dgpu_model* model, double dx, double dy, double scale, double* chi2, double* grad_theta,
                     double* grad_shift, double* grad_scale, float* grad_reference) {
  return guarded(ctx, [&](Context& c) {
    if (width <= 0 || height <= 0) fail(DGPU_ERR_INVALID, "kernel_chi2: image must be non-empty");
    if (width > (1 << 30) || height > (1 << 30) || width * height >= (int64_t(1) << 31))
      fail(DGPU_ERR_INVALID, "kernel_chi2: image too large");
    if (!science || !reference || !weights || !model || !chi2) fail(DGPU_ERR_INVALID, "kernel_chi2: missing argument");
    if (!std::isfinite(dx) || !std::isfinite(dy) || !std::isfinite(scale))
      fail(DGPU_ERR_INVALID, "kernel_chi2: shift and scale must be finite");
    const int w = static_cast<int>(width), h = static_cast<int>(height);
    const size_t n = static_cast<size_t>(w) * h;
    ThinPlate tp(model->knots, model->n_knots);
    Basis b(model->beta, model->n_max, model->radius);
    const int nf = b.nc + 1;
    if (model->n_theta != static_cast<int64_t>(tp.k) * nf)
      fail(DGPU_ERR_INVALID, "kernel_chi2: theta size does not match k*(nc+1)");
    if (b.n_max + 1 > kGradMaxNx) fail(DGPU_ERR_INVALID, "kernel_chi2: n_max above 8 is not supported");
    if (chi2_tile_smem(b.n_max, b.ks) > 200 * 1024) fail(DGPU_ERR_INVALID, "kernel_chi2: kernel radius too large");
    cudaStream_t s = c.stream;
    reset_status(c);
    const auto* sci = static_cast<const float*>(stage_in(c, mem, science, 4 * n, kSlotInSci));
    const auto* ref = static_cast<const float*>(stage_in(c, mem, reference, 4 * n, kSlotInRef));
    const auto* wt = static_cast<const float*>(stage_in(c, mem, weights, 4 * n, kSlotInVarS));
    const auto* rm = static_cast<const uint8_t*>(stage_in(c, mem, reference_mask, n, kSlotInMaskR));
    const DevFields F = build_fields(c, tp, model->theta, nf, w, h);
    float* scal = static_cast<float*>(c.slot(kSlotScratch1, 64));
    launch_strided_median(c, kSampleReference, static_cast<int64_t>(n), ref, rm, scal);

    // Shifted taps and their derivatives (float32 copies of the FP64 values).
    std::vector<double> gxd, dgxd, gyd, dgyd;
    b.shifted_taps(dx, gxd, dgxd);
    b.shifted_taps(dy, gyd, dgyd);
    const size_t nt = gxd.size();
    std::vector<float> taps(4 * nt);
    for (size_t i = 0; i < nt; ++i) {
      taps[i] = static_cast<float>(gxd[i]);
      taps[nt + i] = static_cast<float>(dgxd[i]);
      taps[2 * nt + i] = static_cast<float>(gyd[i]);
      taps[3 * nt + i] = static_cast<float>(dgyd[i]);
    }
    std::vector<int2> ord;
    for (const auto& o : b.orders) ord.push_back(make_int2(o.first, o.second));
    float* d_taps = static_cast<float*>(c.slot(kSlotTaps, sizeof(float) * taps.size() + sizeof(int2) * ord.size()));
    int2* d_ord = reinterpret_cast<int2*>(d_taps + taps.size());
    DGPU_CUDA(h2d_async(d_taps, taps.data(), sizeof(float) * taps.size(), s));
    DGPU_CUDA(h2d_async(d_ord, ord.data(), sizeof(int2) * ord.size(), s));

    const bool want_theta = grad_theta != nullptr;
    const bool want_ref = grad_reference != nullptr;
    const int nb = chi2_tile_blocks(w, h);
    double* part = static_cast<double*>(c.slot(kSlotGrad3, sizeof(double) * (4 * static_cast<size_t>(nb) + 4)));
    double* sums = part + 4 * static_cast<size_t>(nb);
    Chi2Args a;
    a.w = w;
    a.h = h;
    a.sci = sci;
    a.ref = ref;
    a.rmask = rm;
    a.weight = wt;
    a.fill = scal;
    a.F = F;
    a.n_max = b.n_max;
    a.ks = b.ks;
    a.nc = b.nc;
    a.orders = d_ord;
    a.gx = d_taps;
    a.dgx = d_taps + nt;
    a.gy = d_taps + 2 * nt;
    a.dgy = d_taps + 3 * nt;
    a.scale = static_cast<float>(scale);
    a.q = want_theta ? static_cast<float*>(c.slot(kSlotGrad4, sizeof(float) * n * nf)) : nullptr;
    a.p = want_ref ? static_cast<float*>(c.slot(kSlotGrad5, sizeof(float) * n)) : nullptr;
    a.partial = part;
    {
      StageTimer t(c, "gradient: chi2 tiles");
      launch_chi2_tile(s, a);
      launch_sum_rows(s, part, nb, 4, sums);
    }
    std::vector<double> gth;
    double* d_gth = nullptr;
    if (want_theta) {
      StageTimer t(c, "gradient: field adjoint");
      const DevFields D = design_fields(c, tp, F, w, h);
      const int tb = theta_grad_blocks();
      const size_t pairs = static_cast<size_t>(nf) * tp.k;
      double* tpart = static_cast<double*>(c.slot(kSlotGrad6, sizeof(double) * (pairs * tb + pairs)));
      d_gth = tpart + pairs * tb;
      launch_theta_grad(s, w, h, nf, tp.k, a.q, D, tpart);
      launch_sum_rows(s, tpart, tb, static_cast<int>(pairs), d_gth);
      gth.resize(pairs);
    }
    if (want_ref) {
      StageTimer t(c, "gradient: reference adjoint");
      AdjRefArgs r;
      r.w = w;
      r.h = h;
      r.p = a.p;
      r.ref = ref;
      r.rmask = rm;
      r.F = F;
      r.ks = b.ks;
      r.nc = b.nc;
      r.orders = d_ord;
      r.gx = a.gx;
      r.gy = a.gy;
      r.out = static_cast<float*>(out_buf(c, mem, grad_reference, 4 * n, kSlotGrad7));
      launch_adjoint_reference(s, r);
      stage_out(c, mem, grad_reference, r.out, 4 * n);
    }
    double hs[4];
    read_back(c, hs, sums, sizeof(hs));
    if (want_theta) read_back(c, gth.data(), d_gth, sizeof(double) * gth.size());
    check_status(c);  // synchronises
    *chi2 = hs[0];
    if (grad_scale) *grad_scale = hs[1];
    if (grad_shift) {
      grad_shift[0] = hs[2];
      grad_shift[1] = hs[3];
    }
    if (want_theta) std::copy(gth.begin(), gth.end(), grad_theta);
  });
}

}  // extern "C"
