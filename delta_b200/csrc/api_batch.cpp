// dgpu_subtract_batch: many frames of any sizes through the whole subtraction
// pipeline, several in flight (include/delta_gpu.h). The per-frame sequence is
// the reference's Subtractor.subtract stage order (python/delta/pipeline.py:
// 430-806): stamp selection -> convolution direction -> default beta -> knots
// -> kernel fit -> subtract (-> sign flip) -> [decorrelate] -> [PSF estimate,
// whitened PSF, matched-filter score] -> [catalog], each stage the library's
// own entry point in device mode on one worker context.
//
// Scheduling: frames are taken in descending pixel count (longest first) by
// `frames_in_flight` host threads, each driving one context with its own
// stream, so one frame's latency-bound phases (selection, the per-lambda
// solves) overlap another's bandwidth-bound ones. Worker contexts come from a
// process-wide pool and keep their workspace across calls. Host frames are
// uploaded once into the worker's workspace and the products copied back.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <thread>
#include <string>
#include <vector>

#include "internal.h"

using namespace dgpu;

namespace {

constexpr double kFwhmToSigma = 1.0 / 2.354820045030949;

// Subtractor._default_beta (python/delta/pipeline.py:267-282).
double default_beta(double fa, double fb) {
  std::vector<double> f;
  for (double v : {fa, fb})
    if (std::isfinite(v) && v > 0.0) f.push_back(v);
  if (f.empty()) return 2.0;
  const double broad = *std::max_element(f.begin(), f.end()), narrow = *std::min_element(f.begin(), f.end());
  const double d = (broad * kFwhmToSigma) * (broad * kFwhmToSigma) - (narrow * kFwhmToSigma) * (narrow * kFwhmToSigma);
  const double ks = d > 0.0 ? std::sqrt(d) : 0.0;
  return std::max(0.8 * ks, 0.5);
}

// numpy's pairwise summation of a contiguous float64 vector (blocks of at
// most 128 summed with eight interleaved partials), so the sums below round
// exactly like the Python pipeline's `.sum()`.
double np_sum(const double* a, size_t n) {
  if (n < 8) {
    double r = 0.0;
    for (size_t i = 0; i < n; ++i) r += a[i];
    return r;
  }
  if (n <= 128) {
    double r[8];
    for (int j = 0; j < 8; ++j) r[j] = a[j];
    size_t i = 8;
    for (; i < n - n % 8; i += 8)
      for (int j = 0; j < 8; ++j) r[j] += a[i + j];
    double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
    for (; i < n; ++i) res += a[i];
    return res;
  }
  size_t n2 = n / 2;
  n2 -= n2 % 8;
  return np_sum(a, n2) + np_sum(a + n2, n - n2);
}

// Second-moment FWHM of a PSF stamp's positive part (python/delta/catalog.py:
// 60-74), with the Python pipeline's element-wise products and sums. This file
// is compiled without floating-point contraction, so no product here is fused
// into an FMA that numpy would round separately.
double psf_fwhm(const std::vector<float>& psf, int side) {
  const size_t n = static_cast<size_t>(side) * side;
  std::vector<double> wgt(n), t(n);
  for (size_t i = 0; i < n; ++i) wgt[i] = std::max(static_cast<double>(psf[i]), 0.0);
  const double tot = np_sum(wgt.data(), n);
  if (!(tot > 0.0)) fail(DGPU_ERR_RUNTIME, "PSF stamp has no positive flux");
  auto moment = [&](bool along_x, double centre, bool second) {
    for (int y = 0; y < side; ++y)
      for (int x = 0; x < side; ++x) {
        const size_t i = static_cast<size_t>(y) * side + x;
        const double c = along_x ? x : y;
        if (second) {
          const double d = c - centre;
          t[i] = wgt[i] * (d * d);
        } else {
          t[i] = wgt[i] * c;
        }
      }
    return np_sum(t.data(), n) / tot;
  };
  const double mx = moment(true, 0.0, false), my = moment(false, 0.0, false);
  const double vx = moment(true, mx, true), vy = moment(false, my, true);
  return std::sqrt(0.5 * (vx + vy)) / kFwhmToSigma;
}

void check_rc(int rc, dgpu_context* ctx) {
  if (rc != DGPU_OK) fail(rc, dgpu_last_error(ctx));
}

// Process-wide pool of worker contexts per device (kept with their workspace).
std::mutex g_pool_mu;
std::vector<std::pair<int, dgpu_context*>> g_pool;

dgpu_context* acquire_context(int device) {
  {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    for (size_t i = 0; i < g_pool.size(); ++i)
      if (g_pool[i].first == device) {
        dgpu_context* c = g_pool[i].second;
        g_pool.erase(g_pool.begin() + static_cast<long>(i));
        return c;
      }
  }
  dgpu_context* c = nullptr;
  const int rc = dgpu_create(device, &c);
  if (rc != DGPU_OK) fail(rc, dgpu_last_error(nullptr));
  return c;
}

void release_context(int device, dgpu_context* c) {
  std::lock_guard<std::mutex> lock(g_pool_mu);
  g_pool.emplace_back(device, c);
}

// Runs `body` (device work on c.stream, no host synchronisation) as a
// recorded CUDA graph when the context has run this key before; see
// dgpu_subtract_batch in include/delta_gpu.h. Returns true when the graph ran.
template <class F>
bool run_segment(Context& c, bool graphs, const std::string& key, F&& body) {
  if (!graphs) {
    body();
    return false;
  }
  const auto it = c.graphs.find(key);
  if (it == c.graphs.end()) {
    body();  // first sight: sizes the workspace, settles the autotuner
    c.graphs.emplace(key, nullptr);
    return false;
  }
  CaptureArena& a = c.arena;
  if (a.overflow || !a.base) {  // (re)size the arena; the previous frame's copies have finished
    const size_t want = std::max<size_t>(size_t(1) << 20, 2 * a.used);
    if (a.base) DGPU_CUDA(cudaFreeHost(a.base));
    a.base = nullptr;
    a.size = 0;
    void* p = nullptr;
    DGPU_CUDA(cudaHostAlloc(&p, want, cudaHostAllocDefault));
    a.base = static_cast<unsigned char*>(p);
    a.size = want;
    a.overflow = false;
  }
  a.used = 0;
  cudaGraph_t g = nullptr;
  DGPU_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
  capture_arena() = &a;
  bool recorded = true;
  try {
    body();
  } catch (const Failure&) {
    recorded = false;
  }
  capture_arena() = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c.stream, &g);
  if (!recorded || e != cudaSuccess || g == nullptr) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    body();
    return false;
  }
  cudaGraphExec_t& ex = it->second;
  if (ex) {
    cudaGraphExecUpdateResultInfo info{};
    if (cudaGraphExecUpdate(ex, g, &info) != cudaSuccess) {
      cudaGetLastError();
      cudaGraphExecDestroy(ex);
      ex = nullptr;
    }
  }
  if (!ex) {
    const cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
    if (ie != cudaSuccess) {
      cudaGetLastError();
      ex = nullptr;
      cudaGraphDestroy(g);
      body();
      return false;
    }
  }
  cudaGraphDestroy(g);
  DGPU_CUDA(cudaGraphLaunch(ex, c.stream));
  return true;
}

const void* upload(Context& c, const void* host, size_t bytes, Slot s) {
  if (!host) return nullptr;
  void* d = c.slot(s, bytes);
  DGPU_CUDA(cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, c.stream));
  return d;
}

void run_frame(dgpu_context* handle, const dgpu_batch_config& cfg, int mem, const dgpu_frame& f, dgpu_frame_result& r) {
  Context& c = *reinterpret_cast<Context*>(handle);
  const int64_t w = f.width, h = f.height;
  if (w <= 0 || h <= 0 || !f.science || !f.reference) fail(DGPU_ERR_INVALID, "subtract_batch: empty frame");
  if (w * h >= (int64_t(1) << 31)) fail(DGPU_ERR_INVALID, "subtract_batch: frame too large");
  const size_t n = static_cast<size_t>(w) * h;
  // Device layers (host frames uploaded once into this worker's workspace).
  const float *sci, *ref, *svar, *rvar;
  const uint8_t *smask, *rmask;
  if (mem == DGPU_MEM_DEVICE) {
    sci = f.science, ref = f.reference, svar = f.science_var, rvar = f.reference_var;
    smask = f.science_mask, rmask = f.reference_mask;
  } else {
    sci = static_cast<const float*>(upload(c, f.science, 4 * n, kSlotBatch0));
    ref = static_cast<const float*>(upload(c, f.reference, 4 * n, kSlotBatch1));
    svar = static_cast<const float*>(upload(c, f.science_var, 4 * n, kSlotBatch2));
    rvar = static_cast<const float*>(upload(c, f.reference_var, 4 * n, kSlotBatch3));
    smask = static_cast<const uint8_t*>(upload(c, f.science_mask, n, kSlotBatch4));
    rmask = static_cast<const uint8_t*>(upload(c, f.reference_mask, n, kSlotBatch5));
  }
  const int D = DGPU_MEM_DEVICE;
  // 1. stamp selection
  dgpu_detect_params dp{cfg.stamp_radius, cfg.threshold_sigma, cfg.max_stamps, cfg.saturation, 0, 0, cfg.fwhm_radius,
                        cfg.match_radius};
  const int cap = std::max(cfg.max_stamps, 1);
  std::vector<int32_t> sx(cap), sy(cap);
  std::vector<double> fs(cap), fr(cap);
  double med_s = 0.0, med_r = 0.0;
  int dir_ref = 0, count = 0;
  check_rc(dgpu_select_stamps(handle, D, w, h, sci, ref, smask, rmask, nullptr, nullptr, 0, &dp, cap, sx.data(),
                              sy.data(), fs.data(), fr.data(), &med_s, &med_r, &dir_ref, &count),
           handle);
  if (count == 0)
    fail(DGPU_ERR_INVALID,
         "no stamps selected; lower threshold_sigma, supply a catalog, or widen match_radius if science/reference "
         "are astrometrically misregistered");
  // 2. direction, beta, knots
  const bool sci_conv = dir_ref == 0;  // "science": the science frame is convolved
  const float* target = sci_conv ? ref : sci;
  const float* conv = sci_conv ? sci : ref;
  const float* tvar = sci_conv ? rvar : svar;
  const float* cvar = sci_conv ? svar : rvar;
  const uint8_t* tmask = sci_conv ? rmask : smask;
  const uint8_t* cmask = sci_conv ? smask : rmask;
  const double beta = default_beta(med_s, med_r);
  const int nk = cfg.n_knots;
  std::vector<double> knots(static_cast<size_t>(nk) * nk * 2);
  check_rc(dgpu_grid_knots(0.0, 0.0, static_cast<double>(w - 1), static_cast<double>(h - 1), nk, nk, knots.data()),
           nullptr);
  // 3. kernel fit
  std::vector<double> grid(cfg.lambda_grid, cfg.lambda_grid + cfg.n_lambda);
  if (grid.empty())
    for (int i = 0; i < 25; ++i) grid.push_back(std::pow(10.0, -6.0 + 0.5 * i));
  const int nc = (cfg.n_max + 1) * (cfg.n_max + 2) / 2, K = nk * nk, P = (nc + 1) * K;
  std::vector<double> theta(P), lam_out(grid.size()), curve(grid.size()), csums(nc), schi(count);
  std::vector<int32_t> stx(count), sty(count);
  std::vector<uint8_t> sacc(count);
  dgpu_gls_result g{};
  g.theta = theta.data();
  g.lambda_grid = lam_out.data();
  g.gcv_curve = curve.data();
  g.component_sums = csums.data();
  g.stamp_x = stx.data();
  g.stamp_y = sty.data();
  g.stamp_chi2 = schi.data();
  g.stamp_accepted = sacc.data();
  check_rc(dgpu_fit_kernel(handle, D, w, h, target, conv, tvar, cvar, tmask, cmask, knots.data(), K, sx.data(),
                           sy.data(), count, cfg.stamp_radius, beta, cfg.n_max, cfg.radius, grid.data(),
                           static_cast<int>(grid.size()), cfg.clip_sigma, cfg.clip_iterations, cfg.min_stamps,
                           cfg.cv_folds, cfg.precision, &g),
           handle);
  // 4. subtract, sign
  const dgpu_model model{knots.data(), K, theta.data(), P, beta, cfg.n_max, cfg.radius};
  const bool out_dev = mem == DGPU_MEM_DEVICE;
  float* diff = static_cast<float*>(c.slot(kSlotBatch6, 4 * n));
  float* var = static_cast<float*>(c.slot(kSlotBatch7, 4 * n));
  uint8_t* mask = static_cast<uint8_t*>(c.slot(kSlotBatch8, n));
  const bool decor = cfg.decorrelate && tvar && cvar;
  float* dw = decor ? static_cast<float*>(c.slot(kSlotBatch9, 4 * n)) : nullptr;
  float* vw = decor ? static_cast<float*>(c.slot(kSlotBatch10, 4 * n)) : nullptr;
  int hv = 0, hm = 0;
  // 4-5. subtract, sign, decorrelate: device work only, recorded as one graph
  // per shape and layer configuration once this context has run it. (The
  // basis radius follows each frame's beta; a frame whose radius needs more
  // workspace than the key's earlier frames is refused while recording and
  // runs directly.)
  char key[256];
  std::snprintf(key, sizeof(key), "%lldx%lld/l%d%d%d%d/s%d/c%d/d%d/b%d/n%d/k%d", static_cast<long long>(w),
                static_cast<long long>(h), tvar != nullptr, cvar != nullptr, tmask != nullptr, cmask != nullptr,
                cfg.saturation > 0.0, sci_conv, decor, cfg.block, cfg.n_max, K);
  r.graph_replayed = run_segment(c, cfg.graphs != 0, key, [&]() {
    check_rc(dgpu_subtract(handle, D, w, h, target, conv, tvar, cvar, tmask, cmask, &model, cfg.saturation, diff,
                           var, mask, &hv, &hm),
             handle);
    if (sci_conv) check_rc(dgpu_negate(handle, D, diff, static_cast<int64_t>(n)), handle);
    if (decor) check_rc(dgpu_decorrelate(handle, D, w, h, diff, &model, tvar, cvar, cfg.block, 0, dw, vw), handle);
  }) ? 1 : 0;
  const float* whitened = decor ? dw : diff;
  const float* white_var = decor ? vw : (hv ? var : nullptr);
  // 6. score and catalog
  const float* score = nullptr;
  int n_cat = 0;
  if (cfg.score) {
    if (!white_var) fail(DGPU_ERR_INVALID, "subtract_batch: the score needs variance layers");
    const int pr = std::min(cfg.stamp_radius, 8), side = 2 * pr + 1;
    std::vector<float> psf(static_cast<size_t>(side) * side), wpsf(psf.size());
    check_rc(dgpu_estimate_psf(handle, D, w, h, target, sx.data(), sy.data(), count, pr, psf.data()), handle);
    if (whitened != diff) {
      check_rc(dgpu_whiten_score_psf(handle, D, psf.data(), side, &model, w, h, tvar, cvar, cfg.block, wpsf.data()),
               handle);
      psf.swap(wpsf);
    }
    float* sc = static_cast<float*>(c.slot(kSlotBatch11, 4 * n));
    check_rc(dgpu_matched_filter(handle, D, w, h, whitened, psf.data(), side, white_var, sc), handle);
    score = sc;
    if (cfg.catalog) {
      dgpu_catalog_params cp{cfg.catalog_threshold_sigma, 3.0, psf_fwhm(psf, side), 0.3, 3.0, 0, 1, 0, 0, 3.0, 0.0,
                             5000};
      check_rc(dgpu_build_catalog(handle, D, w, h, score, whitened, hm ? mask : nullptr, &cp, nullptr, nullptr, 0,
                                  nullptr, nullptr, 0, &n_cat),
               handle);
      r.catalog_count = n_cat;
      r.catalog_fetched = 0;
      if (n_cat <= r.catalog_capacity) {
        if (n_cat > 0) check_rc(dgpu_catalog_fetch(handle, &r.catalog, n_cat), handle);
        r.catalog_fetched = 1;
      }
    }
  }
  // 7. products
  auto put = [&](void* dst, const void* src, size_t bytes) {
    if (!dst || !src) return;
    DGPU_CUDA(cudaMemcpyAsync(dst, src, bytes, out_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c.stream));
  };
  put(r.difference, whitened, 4 * n);
  put(r.variance, white_var, 4 * n);
  put(r.mask, hm ? mask : nullptr, n);
  put(r.score, score, 4 * n);
  DGPU_CUDA(cudaStreamSynchronize(c.stream));
  if (r.theta) std::copy(theta.begin(), theta.end(), r.theta);
  r.n_theta = P;
  r.lambda = g.lambda;
  r.beta = beta;
  r.direction_is_reference = dir_ref;
  r.n_stamps_used = g.n_stamps_used;
  r.has_variance = white_var ? 1 : 0;
  r.has_mask = hm;
}

}  // namespace

extern "C" {

int dgpu_subtract_batch(const dgpu_batch_config* cfg, int mem, int n_frames, const dgpu_frame* frames,
                        dgpu_frame_result* results) {
  if (!cfg || (n_frames > 0 && (!frames || !results))) {
    dgpu::free_error() = "subtract_batch: missing argument";
    return DGPU_ERR_INVALID;
  }
  if (n_frames <= 0) return DGPU_OK;
  if (mem != DGPU_MEM_HOST && mem != DGPU_MEM_DEVICE) {
    dgpu::free_error() = "subtract_batch: mem must be DGPU_MEM_HOST or DGPU_MEM_DEVICE";
    return DGPU_ERR_INVALID;
  }
  // Longest first (descending pixel count, ties by index).
  std::vector<int> order(n_frames);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return frames[a].width * frames[a].height > frames[b].width * frames[b].height;
  });
  const int workers = std::max(1, std::min(cfg->frames_in_flight, n_frames));
  std::atomic<int> next{0};
  auto worker = [&]() {
    dgpu_context* ctx = nullptr;
    try {
      ctx = acquire_context(cfg->device);
    } catch (const Failure& e) {
      for (int i = next.fetch_add(n_frames); i < n_frames; ++i) {
        results[order[i]].status = e.code;
        std::snprintf(results[order[i]].error, sizeof(results[order[i]].error), "%s", e.what());
      }
      return;
    }
    for (int i = next++; i < n_frames; i = next++) {
      dgpu_frame_result& r = results[order[i]];
      const auto t0 = std::chrono::steady_clock::now();
      r.status = DGPU_OK;
      r.error[0] = '\0';
      r.graph_replayed = 0;
      try {
        run_frame(ctx, *cfg, mem, frames[order[i]], r);
      } catch (const Failure& e) {
        r.status = e.code;
        std::snprintf(r.error, sizeof(r.error), "%s", e.what());
        cudaStreamSynchronize(reinterpret_cast<Context*>(ctx)->stream);
      } catch (const std::exception& e) {
        r.status = DGPU_ERR_RUNTIME;
        std::snprintf(r.error, sizeof(r.error), "%s", e.what());
      }
      r.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    release_context(cfg->device, ctx);
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < workers; ++t) pool.emplace_back(worker);
  for (auto& t : pool) t.join();
  for (int i = 0; i < n_frames; ++i)
    if (results[i].status != DGPU_OK) {
      dgpu::free_error() = std::string("subtract_batch: frame ") + std::to_string(i) + ": " + results[i].error;
      return results[i].status;
    }
  return DGPU_OK;
}

}  // extern "C"
