// Host driver of the stamp fit and the penalised-GLS entry points.
//
// The per-pixel / per-row / per-system arithmetic runs on the device
// (k_fit.cu, k_solve.cu, k_gls.cu); this file sequences it and takes the
// reference's small scalar decisions on the host: the lambda argmin, the CV
// coarse-to-fine / warm-start search order (src/solve.cpp:344-402) and the
// per-stamp median/MAD clip (src/fit.cpp:456-491), which read a few hundred
// numbers per IRLS pass.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <limits>
#include <numeric>

#include "fit_internal.h"
#include "gcv_grad_internal.h"
#include "gls_internal.h"

using namespace dgpu;

namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();
constexpr double kNaN = std::numeric_limits<double>::quiet_NaN();

template <class T>
T* up(Context& c, Slot s, const T* host, size_t n) {
  T* d = static_cast<T*>(c.slot(s, sizeof(T) * std::max<size_t>(n, 1)));
  if (n) DGPU_CUDA(h2d_async(d, host, sizeof(T) * n, c.stream));
  return d;
}

template <class T>
std::vector<T> down(Context& c, const T* dev, size_t n) {
  std::vector<T> h(n);
  if (n) read_back(c, h.data(), dev, sizeof(T) * n);
  sync_reads(c);
  return h;
}

// Batched device -> host reads: every add() queues a read-back; run()
// synchronises the stream once and scatters the bytes to their host
// destinations.
class Fetch {
 public:
  Fetch(Context& c, size_t /*max_bytes*/) : c_(c) {}
  template <class T>
  void add(T* host, const T* dev, size_t n) {
    if (n) read_back(c_, host, dev, sizeof(T) * n);
  }
  void run() { sync_reads(c_); }

 private:
  Context& c_;
};

double median_copy(std::vector<double> v) {
  if (v.empty()) return kNaN;
  const size_t mid = v.size() / 2;
  std::nth_element(v.begin(), v.begin() + mid, v.end());
  return v[mid];
}

// The tensor-core builds of the normal equations (BF16x3 "mixed", TF32): both
// are refined by one FP64 step and fall back to FP64 when that step shows them
// too inaccurate for the system.
inline bool tensor_prec(int prec) { return prec == DGPU_PREC_MIXED || prec == DGPU_PREC_TF32; }

struct GlsOut {
  std::vector<double> theta;
  double lambda = 0, gcv = 0, edf = 0, rss = 0;
  long long npix = 0;  // active rows of the fit
  std::vector<double> grid, curve;
  const double* d_theta = nullptr;  // device copy of theta
  double refine_correction = 0.0;   // ||delta|| / ||theta|| of the mixed refinement step
  int prec_used = DGPU_PREC_FP64;
  int ldlt = 0;                     // 1: the chosen system's Cholesky failed, solved by the LDLT fallback
};

// Rows + normal-equation machinery shared by fit_kernel and solve_gls*.
struct Engine {
  Context& c;
  int prec;
  const ThinPlate& tp;
  int nc, nf, k, P;
  int64_t N;
  int SS;
  int n_units;  // stamps (fit) or rows (direct solve)
  FitRows R;
  std::vector<double> pen_host, fk_host;
  int rk = 0;
  double* d_pen = nullptr;
  double* d_fk = nullptr;
  // Optional extra reads joined to a solution's read-back: called with the
  // device theta just before the fetch runs (fit_kernel's per-stamp chi^2).
  std::function<void(const double*, Fetch&)> on_fetch;
  size_t on_fetch_bytes = 0;

  Engine(Context& ctx, int precision, const ThinPlate& t, int nc_, int64_t N_, int SS_, int units)
      : c(ctx), prec(precision), tp(t), nc(nc_), nf(nc_ + 1), k(t.k), P((nc_ + 1) * t.k), N(N_), SS(SS_),
        n_units(units) {
    if (P > 1024) fail(DGPU_ERR_INVALID, "fit: (nc+1)*k above 1024 unknowns is not supported");
    pen_host = tp.penalty;
    fk_host = tp.pen_half(0, &rk);  // one k x r block (nc = 0)
    std::vector<double> pf(pen_host);
    pf.insert(pf.end(), fk_host.begin(), fk_host.end());
    d_pen = up(c, kSlotFit14, pf.data(), pf.size());
    d_fk = d_pen + static_cast<size_t>(k) * k;
  }

  void alloc_rows() {
    const size_t n = static_cast<size_t>(N);
    R.valid = static_cast<uint8_t*>(c.slot(kSlotFit0, n));
    R.t = static_cast<double*>(c.slot(kSlotFit1, 8 * n));
    R.vt = static_cast<double*>(c.slot(kSlotFit2, 8 * n));
    R.vc = static_cast<double*>(c.slot(kSlotFit3, 8 * n));
    R.bn = static_cast<double*>(c.slot(kSlotFit4, 8 * n * nc));
    R.px = static_cast<int*>(c.slot(kSlotFit5, 4 * n));
    R.py = static_cast<int*>(c.slot(kSlotFit6, 4 * n));
    R.d = static_cast<double*>(c.slot(kSlotFit7, 8 * n * k));
    R.w = static_cast<double*>(c.slot(kSlotFit8, 8 * n));
    R.stamp_used = static_cast<int*>(c.slot(kSlotFit9, 4 * std::max(n_units, 1)));
  }

  // Workspace for up to `nsys` systems sharing the solver batch.
  struct Work {
    double *A, *theta, *edf, *raw, *rss, *gcv, *lam;
    int *ok, *midx, *ridx;
    double* partial;
  };
  Work work(int nsys, int nm = 1) {
    Work w{};
    w.A = static_cast<double*>(c.slot(kSlotFft0, sizeof(double) * solve_work_doubles(P, nf, rk, nsys, nm)));
    const size_t small = sizeof(double) * (static_cast<size_t>(nsys) * P + 6 * nsys) + sizeof(int) * 3 * nsys + 64;
    char* sm = static_cast<char*>(c.slot(kSlotFft1, small));
    w.theta = reinterpret_cast<double*>(sm);
    w.edf = w.theta + static_cast<size_t>(nsys) * P;
    w.raw = w.edf + nsys;
    w.rss = w.raw + nsys;
    w.gcv = w.rss + nsys;
    w.lam = w.gcv + nsys;
    w.ok = reinterpret_cast<int*>(w.lam + nsys);
    w.midx = w.ok + nsys;
    w.ridx = w.midx + nsys;
    w.partial = static_cast<double*>(c.slot(kSlotFft2, sizeof(double) * 8 * std::max(nsys, 1)));
    return w;
  }

  void solve(const Work& w, int nsys, const double* M, const int* midx, const double* rhs, const int* ridx,
             int nm = 1) {
    SolveBatch b;
    b.P = P;
    b.k = k;
    b.nf = nf;
    b.r = rk;
    b.nsys = nsys;
    b.M = M;
    b.m_index = midx;
    b.nm = nm;
    b.rhs = rhs;
    b.r_index = ridx;
    b.lam = w.lam;
    b.pen = d_pen;
    b.fk = d_fk;
    b.A = w.A;
    b.theta = w.theta;
    b.edf = w.edf;
    b.ok = w.ok;
    b.status = c.d_status;
    b.partial = w.partial;
    b.skip_ldlt = quick_fallback() ? 1 : 0;
    StageTimer t(c, "fit: lambda-grid solve");
    launch_solve_batch(c, b);
  }

  SolveBatch batch_of(const Work& w) const {
    SolveBatch b;
    b.P = P;
    b.k = k;
    b.nf = nf;
    b.r = rk;
    b.A = w.A;
    return b;
  }

  // M, rhs, ywy, n over the rows whose unit mask is set.
  void assemble(const uint8_t* mask, double* M, double* rhs, double* ywy, long long* n) {
    StageTimer t(c, "fit: normal equations");
    launch_rhs(c, N, nc, k, SS, R, mask, nullptr, rhs, ywy, n);
    launch_normal_equations(c, prec, N, nc, k, SS, R, mask, M);
  }

  // Mixed precision: the residual of an anchor theta0 in FP64 (e0 = t - X theta0),
  // r0 = X^T W e0 and s0 = e0^T W e0, from which the rss of any theta follows
  // as s0 - 2 (theta - theta0) . r0 + (theta - theta0)^T M (theta - theta0).
  // Near the anchor the BF16x3 error of M enters only through the small
  // quadratic term, where ywy - 2 theta . rhs + theta^T M theta would carry it
  // at the scale of ywy (the rss is often 1e-4 of ywy or less).
  struct Anchor {
    double *r0, *rp, *delta, *s0, *theta0, *approx;
  };
  // The anchor's vectors, theta0 and room for `curve` copied curve values.
  Anchor anchor_buffers(int curve = 0) {
    double* a = static_cast<double*>(
        c.slot(kSlotFit15, sizeof(double) * (4 * static_cast<size_t>(P) + 2 + static_cast<size_t>(curve))));
    return Anchor{a, a + P, a + 2 * P, a + 3 * P, a + 3 * P + 2, a + 4 * P + 2};
  }
  void anchor_at(const Anchor& a, const double* theta, const uint8_t* mask) {
    launch_rhs(c, N, nc, k, SS, R, mask, theta, a.r0, a.s0, nullptr);
  }

  // Mixed precision: rss / GCV of every system of the batch around the anchor.
  std::vector<double> anchored_curve(const Work& w, int nsys, const double* M, const Anchor& a,
                                     const double* theta0, const long long* n) {
    launch_quad_err(c, nsys, P, w.theta, M, nullptr, a.r0, nullptr, a.s0, w.raw, theta0);
    launch_gcv_finish(c.stream, nsys, w.raw, w.edf, w.ok, n, w.rss, w.gcv);
    return down(c, w.gcv, nsys);
  }

  GlsOut gcv_once(const std::vector<double>& grid, const uint8_t* mask) {
    if (grid.empty()) fail(DGPU_ERR_RUNTIME, "solve_gls_gcv: lambda_grid is empty");
    const int nl = static_cast<int>(grid.size());
    double* M = static_cast<double*>(c.slot(kSlotScratch1,
                                            sizeof(double) * (static_cast<size_t>(P) * P + P + 2)));
    double* rhs = M + static_cast<size_t>(P) * P;
    double* ywy = rhs + P;
    long long* n = reinterpret_cast<long long*>(ywy + 1);
    assemble(mask, M, rhs, ywy, n);
    Work w = work(nl);
    DGPU_CUDA(h2d_async(w.lam, grid.data(), sizeof(double) * nl, c.stream));
    solve(w, nl, M, nullptr, rhs, nullptr);
    launch_quad_err(c, nl, P, w.theta, M, nullptr, rhs, nullptr, ywy, w.raw);
    launch_gcv_finish(c.stream, nl, w.raw, w.edf, w.ok, n, w.rss, w.gcv);
    GlsOut o;
    o.grid = grid;
    auto argmin = [&](const std::vector<double>& v) {  // first minimum; NaN never wins (launch_argmin_copy)
      int b = 0;
      double bg = kInf;
      for (int i = 0; i < nl; ++i)
        if (v[i] < bg) {
          bg = v[i];
          b = i;
        }
      return b;
    };
    int best = 0, anchored = -1;
    if (tensor_prec(prec)) {
      // Re-evaluate the curve around the provisional minimum until the minimum
      // stays put (it moves at most a grid step or two). The first anchor is
      // picked on the device, so both curves come back in one read.
      const Anchor a = anchor_buffers(nl);
      DGPU_CUDA(cudaMemcpyAsync(a.approx, w.gcv, sizeof(double) * nl, cudaMemcpyDeviceToDevice, c.stream));
      launch_argmin_copy(c.stream, nl, w.gcv, w.theta, P, a.theta0);
      anchor_at(a, a.theta0, mask);
      launch_quad_err(c, nl, P, w.theta, M, nullptr, a.r0, nullptr, a.s0, w.raw, a.theta0);
      launch_gcv_finish(c.stream, nl, w.raw, w.edf, w.ok, n, w.rss, w.gcv);
      std::vector<double> approx(nl);
      std::vector<int> okv(nl);
      o.curve.resize(nl);
      {
        Fetch f(c, sizeof(double) * 2 * nl + sizeof(int) * nl);
        f.add(approx.data(), a.approx, nl);
        f.add(o.curve.data(), w.gcv, nl);
        f.add(okv.data(), w.ok, nl);
        f.run();
      }
      if (quick_fallback() && std::find(okv.begin(), okv.end(), 0) != okv.end()) {
        o.prec_used = prec;  // a Cholesky failed in the reduced-precision system: redo in FP64
        o.ldlt = 1;
        return o;
      }
      anchored = argmin(approx);
      best = argmin(o.curve);
      for (int pass = 1; pass < 3 && anchored != best; ++pass) {
        const double* th0 = w.theta + static_cast<size_t>(best) * P;
        anchor_at(a, th0, mask);
        anchored = best;
        o.curve = anchored_curve(w, nl, M, a, th0, n);
        best = argmin(o.curve);
      }
    } else {
      o.curve = down(c, w.gcv, nl);
      best = argmin(o.curve);
    }
    finish_single(w, best, grid[best], M, n, mask, o, anchored == best);
    return o;
  }

  // A reduced-precision attempt that the FP64 fallback would redo: a system
  // whose Cholesky fails is not LDLT-solved (the whole attempt is redone in
  // FP64 instead, see mixed_failed).
  bool quick_fallback() const { return tensor_prec(prec) && c.precision_fallback; }

  // Mixed precision falls back to FP64 normal equations, for the rest of this
  // fit, when its solve is non-finite or its FP64 refinement correction is
  // above kMixedFallback of theta: one step leaves about the square of that
  // relative error, and past it the BF16x3 system is too far from the FP64 one
  // for the system's conditioning.
  static constexpr double kMixedFallback = 1e-2;
  bool mixed_failed(const GlsOut& o) const {
    if (!tensor_prec(o.prec_used)) return false;
    if (o.ldlt) return true;  // the refinement step applies a Cholesky factor the system does not have
    if (!(o.refine_correction <= kMixedFallback)) return true;
    for (double v : o.theta)
      if (!std::isfinite(v)) return true;
    return false;
  }
  template <class F>
  GlsOut with_fallback(F&& run) {
    GlsOut o = run();
    if (c.precision_fallback && mixed_failed(o)) {
      prec = DGPU_PREC_FP64;
      o = run();
    }
    return o;
  }
  GlsOut gcv(const std::vector<double>& grid, const uint8_t* mask) {
    return with_fallback([&] { return gcv_once(grid, mask); });
  }
  GlsOut fixed(double lam, const uint8_t* mask) {
    return with_fallback([&] { return fixed_once(lam, mask); });
  }
  GlsOut cv(const std::vector<double>& grid, const uint8_t* mask, const std::vector<int>& fold, int G, int warm_start,
            bool stamped) {
    return with_fallback([&] { return cv_once(grid, mask, fold, G, warm_start, stamped); });
  }

  // Fill theta / scalars of system `s` into o. Mixed precision: one FP64
  // refinement step from the anchor residual at theta_s (computed here unless
  // `anchored`), and the rss / GCV of the refined theta around that anchor.
  void finish_single(const Work& w, int s, double lam, const double* M, const long long* n, const uint8_t* mask,
                     GlsOut& o, bool anchored = false) {
    double* th = w.theta + static_cast<size_t>(s) * P;
    // A mixed system that went through the LDLT fallback has no Cholesky
    // factor for the refinement step below; its result is discarded once the
    // ok flag (fetched with theta) shows it, and the fit is redone in FP64
    // (mixed_failed).
    int ok_s = 1;
    if (tensor_prec(prec)) {
      const Anchor a = anchor_buffers();
      if (!anchored) anchor_at(a, th, mask);
      DGPU_CUDA(cudaMemcpyAsync(a.rp, a.r0, sizeof(double) * P, cudaMemcpyDeviceToDevice, c.stream));
      launch_refine_update(c.stream, P, k, d_pen, lam, th, a.rp);
      launch_apply_inverse(c.stream, batch_of(w), s, a.rp, a.delta);
      launch_axpy(c.stream, P, a.delta, th);
      launch_quad_err(c, 1, P, a.delta, M, nullptr, a.r0, nullptr, a.s0, w.raw + s);
      launch_gcv_finish(c.stream, 1, w.raw + s, w.edf + s, w.ok + s, n, w.rss + s, w.gcv + s);
    }
    o.theta.resize(P);
    std::vector<double> delta(tensor_prec(prec) ? P : 0);
    Fetch f(c, sizeof(double) * (2 * P + 4) + on_fetch_bytes);
    f.add(o.theta.data(), th, P);
    f.add(&o.edf, w.edf + s, 1);
    f.add(&o.rss, w.rss + s, 1);
    f.add(&o.gcv, w.gcv + s, 1);
    f.add(&o.npix, n, 1);
    f.add(&ok_s, w.ok + s, 1);
    if (!delta.empty()) f.add(delta.data(), anchor_buffers().delta, P);
    if (on_fetch) on_fetch(th, f);
    f.run();
    o.d_theta = th;
    o.lambda = lam;
    o.prec_used = prec;
    o.ldlt = ok_s == 1 ? 0 : 1;  // 2: LDLT fallback; 0: failed Cholesky left for the FP64 redo
    if (!delta.empty()) {
      double dd = 0.0, tt = 0.0;
      for (int p = 0; p < P; ++p) {
        dd += delta[p] * delta[p];
        tt += o.theta[p] * o.theta[p];
      }
      o.refine_correction = tt > 0.0 ? std::sqrt(dd / tt) : (dd > 0.0 ? kInf : 0.0);
      if (!std::isfinite(dd) || !std::isfinite(tt)) o.refine_correction = kInf;
    }
  }

  // Fixed-lambda solve (src/solve.cpp:208-215).
  GlsOut fixed_once(double lam, const uint8_t* mask) {
    double* M = static_cast<double*>(c.slot(kSlotScratch1, sizeof(double) * (static_cast<size_t>(P) * P + P + 2)));
    double* rhs = M + static_cast<size_t>(P) * P;
    double* ywy = rhs + P;
    long long* n = reinterpret_cast<long long*>(ywy + 1);
    assemble(mask, M, rhs, ywy, n);
    Work w = work(1);
    DGPU_CUDA(h2d_async(w.lam, &lam, sizeof(double), c.stream));
    solve(w, 1, M, nullptr, rhs, nullptr);
    launch_quad_err(c, 1, P, w.theta, M, nullptr, rhs, nullptr, ywy, w.raw);
    launch_gcv_finish(c.stream, 1, w.raw, w.edf, w.ok, n, w.rss, w.gcv);
    GlsOut o;
    finish_single(w, 0, lam, M, n, mask, o);
    return o;
  }

  // Group CV over per-unit folds (fold[u] in [0, G), -1 = excluded).
  // stamped: per-stamp Kronecker build with stamp designs at pixel centroids.
  GlsOut cv_once(const std::vector<double>& grid, const uint8_t* mask, const std::vector<int>& fold, int G,
                 int warm_start, bool stamped) {
    if (grid.empty()) fail(DGPU_ERR_RUNTIME, "solve_gls_cv: lambda_grid is empty");
    const int nl = static_cast<int>(grid.size());
    const size_t PP = static_cast<size_t>(P) * P;
    // fold parts: Mg[G], rg[G], yg[G]; all: Mall, rall, yall; train: Mt[G], rt[G]
    double* base = static_cast<double*>(c.slot(kSlotScratch1,
                                               sizeof(double) * ((2 * G + 1) * (PP + P) + G + 8)));
    double* Mg = base;
    double* Mt = Mg + G * PP;
    double* Mall = Mt + G * PP;
    double* rg = Mall + PP;
    double* rt = rg + static_cast<size_t>(G) * P;
    double* rall = rt + static_cast<size_t>(G) * P;
    double* yg = rall + P;
    double* yall = yg + G;
    long long* nall = reinterpret_cast<long long*>(yall + 1);
    // Active-row count (and per-row ywy) over all folds.
    {
      double* scratch = static_cast<double*>(c.slot(kSlotFit15, sizeof(double) * 2 * P));
      launch_rhs(c, N, nc, k, SS, R, mask, nullptr, scratch, yall, nall);
    }
    if (stamped) {
      // Per-stamp moments + centroids, stamp design on the host (S x k small).
      double* As = static_cast<double*>(c.slot(kSlotFit10, sizeof(double) * static_cast<size_t>(n_units) * (nf * nf + nf + 4)));
      double* rs = As + static_cast<size_t>(n_units) * nf * nf;
      double* ds2 = rs + static_cast<size_t>(n_units) * nf;
      double* cen = ds2 + n_units;
      launch_stamp_moments(c.stream, n_units, nc, SS, R, mask, As, rs, ds2, cen);
      const auto hc = down(c, cen, static_cast<size_t>(n_units) * 3);
      std::vector<double> dsd(static_cast<size_t>(n_units) * k, 0.0);
      std::vector<int> f2(n_units, -1);
      for (int u = 0; u < n_units; ++u) {
        const double cnt = hc[3 * u + 2];
        if (cnt <= 0.0 || fold[u] < 0) continue;
        tp.design_row(hc[3 * u] / cnt, hc[3 * u + 1] / cnt, dsd.data() + static_cast<size_t>(u) * k);
        f2[u] = fold[u];
      }
      double* d_dsd = up(c, kSlotFit13, dsd.data(), dsd.size());
      int* d_fold = static_cast<int*>(c.slot(kSlotBlockCounts, sizeof(int) * std::max(n_units, 1)));
      DGPU_CUDA(h2d_async(d_fold, f2.data(), sizeof(int) * n_units, c.stream));
      launch_stamped_assemble(c.stream, G, n_units, nf, k, d_fold, As, rs, ds2, d_dsd, Mg, rg, yg);
      DGPU_CUDA(cudaStreamSynchronize(c.stream));
    } else {
      uint8_t* fm = static_cast<uint8_t*>(c.slot(kSlotSeedNeg, std::max(n_units, 1)));
      const auto hm = down(c, mask, n_units);
      for (int g = 0; g < G; ++g) {
        std::vector<uint8_t> m(n_units);
        for (int u = 0; u < n_units; ++u) m[u] = (hm[u] && fold[u] == g) ? 1 : 0;
        DGPU_CUDA(h2d_async(fm, m.data(), n_units, c.stream));
        long long* dummy = nall + 1;
        launch_rhs(c, N, nc, k, SS, R, fm, nullptr, rg + static_cast<size_t>(g) * P, yg + g, dummy);
        launch_normal_equations(c, prec, N, nc, k, SS, R, fm,
                                Mg + g * PP);
        DGPU_CUDA(cudaStreamSynchronize(c.stream));
      }
    }
    launch_fold_train(c.stream, G, PP, Mg, Mall, Mt);
    launch_fold_train(c.stream, G, P, rg, rall, rt);
    {
      // yall from the folds (matches cv_finish's sum of ysq[g]).
      std::vector<double> y = down(c, yg, G);
      double ys = 0.0;
      for (double v : y) ys += v;
      DGPU_CUDA(h2d_async(yall, &ys, sizeof(double), c.stream));
      DGPU_CUDA(cudaStreamSynchronize(c.stream));
    }
    std::vector<double> curve(nl, kInf);
    std::vector<char> done(nl, 0);
    Work w = work(std::max(nl * G, 1), G);
    // Mixed precision, row folds: held-out errors around per-fold anchors
    // (th0[g], with the FP64 residual sums r0[g], s0[g] over fold g's rows).
    double* th0 = nullptr;
    double* r0 = nullptr;
    double* s0 = nullptr;
    bool chol_failed = false;  // a reduced-precision fold system failed its Cholesky (quick_fallback)
    auto solve_at = [&](const std::vector<int>& idx) {
      const int m = static_cast<int>(idx.size());
      const int ns = m * G;
      std::vector<double> lam(ns);
      std::vector<int> mi(ns);
      for (int ii = 0; ii < m; ++ii)
        for (int g = 0; g < G; ++g) {
          lam[ii * G + g] = grid[idx[ii]];
          mi[ii * G + g] = g;
        }
      DGPU_CUDA(h2d_async(w.lam, lam.data(), sizeof(double) * ns, c.stream));
      DGPU_CUDA(h2d_async(w.midx, mi.data(), sizeof(int) * ns, c.stream));
      solve(w, ns, Mt, w.midx, rt, w.midx, G);
      return ns;
    };
    auto evaluate = [&](const std::vector<int>& idx) {
      const int m = static_cast<int>(idx.size());
      const int ns = solve_at(idx);
      if (th0)
        launch_quad_err(c, ns, P, w.theta, Mg, w.midx, r0, w.midx, s0, w.raw, th0);
      else
        launch_quad_err(c, ns, P, w.theta, Mg, w.midx, rg, w.midx, yg, w.raw);
      const auto err = down(c, w.raw, ns);
      const auto ok = down(c, w.ok, ns);
      if (quick_fallback())
        for (int v : ok) chol_failed = chol_failed || v == 0;
      for (int ii = 0; ii < m; ++ii) {
        double tot = 0.0;
        for (int g = 0; g < G; ++g) {
          const double e = err[ii * G + g];
          tot += ok[ii * G + g] ? (e > 0.0 ? e : 0.0) : kInf;
        }
        curve[idx[ii]] = tot;
        done[idx[ii]] = 1;
      }
    };
    auto argmin_done = [&]() {
      int b = -1;
      double bc = kInf;
      for (int li = 0; li < nl; ++li)
        if (done[li] && curve[li] < bc) {
          bc = curve[li];
          b = li;
        }
      return b;
    };
    if (warm_start >= 0 && warm_start < nl) {
      std::vector<int> seed;
      for (int li = std::max(0, warm_start - 1); li <= std::min(nl - 1, warm_start + 1); ++li) seed.push_back(li);
      evaluate(seed);
      for (int guard = 0; guard < nl + 2; ++guard) {
        const int b = argmin_done();
        std::vector<int> step;
        if (b > 0 && !done[b - 1]) step.push_back(b - 1);
        if (b >= 0 && b < nl - 1 && !done[b + 1]) step.push_back(b + 1);
        if (step.empty()) break;
        evaluate(step);
      }
    } else {
      std::vector<int> coarse;
      for (int li = 0; li < nl; li += 2) coarse.push_back(li);
      if (coarse.empty() || coarse.back() != nl - 1) coarse.push_back(nl - 1);
      evaluate(coarse);
      int cb = coarse.front();
      for (int li : coarse)
        if (curve[li] < curve[cb]) cb = li;
      std::vector<int> refine_idx;
      for (int li = std::max(0, cb - 2); li <= std::min(nl - 1, cb + 2); ++li)
        if (!done[li]) refine_idx.push_back(li);
      if (!refine_idx.empty()) evaluate(refine_idx);
    }
    int best = 0;
    double bc = kInf;
    for (int li = 0; li < nl; ++li)
      if (done[li] && curve[li] < bc) {
        bc = curve[li];
        best = li;
      }
    if (tensor_prec(prec) && !stamped) {
      // Re-evaluate every searched lambda around the folds' solutions at the
      // provisional minimum until the minimum stays put.
      const size_t gp = static_cast<size_t>(G) * P;
      char* ab = static_cast<char*>(c.slot(kSlotFit12, sizeof(double) * (2 * gp + G) + static_cast<size_t>(G) * n_units));
      double* a_th = reinterpret_cast<double*>(ab);
      double* a_r = a_th + gp;
      double* a_s = a_r + gp;
      uint8_t* fmasks = reinterpret_cast<uint8_t*>(a_s + G);
      {
        const auto hm = down(c, mask, n_units);
        std::vector<uint8_t> m(static_cast<size_t>(G) * n_units, 0);
        for (int g = 0; g < G; ++g)
          for (int u = 0; u < n_units; ++u) m[static_cast<size_t>(g) * n_units + u] = (hm[u] && fold[u] == g) ? 1 : 0;
        DGPU_CUDA(h2d_async(fmasks, m.data(), m.size(), c.stream));
      }
      std::vector<int> searched;
      for (int li = 0; li < nl; ++li)
        if (done[li]) searched.push_back(li);
      for (int pass = 0, anchored = -1; pass < 3 && anchored != best; ++pass) {
        solve_at({best});
        DGPU_CUDA(cudaMemcpyAsync(a_th, w.theta, sizeof(double) * gp, cudaMemcpyDeviceToDevice, c.stream));
        for (int g = 0; g < G; ++g)
          launch_rhs(c, N, nc, k, SS, R, fmasks + static_cast<size_t>(g) * n_units, a_th + static_cast<size_t>(g) * P,
                     a_r + static_cast<size_t>(g) * P, a_s + g, nullptr);
        th0 = a_th;
        r0 = a_r;
        s0 = a_s;
        anchored = best;
        evaluate(searched);
        bc = kInf;
        for (int li : searched)
          if (curve[li] < bc) {
            bc = curve[li];
            best = li;
          }
      }
    }
    // Final all-data fit at the selected lambda.
    Work w1 = work(1);
    DGPU_CUDA(h2d_async(w1.lam, &grid[best], sizeof(double), c.stream));
    solve(w1, 1, Mall, nullptr, rall, nullptr);
    launch_quad_err(c, 1, P, w1.theta, Mall, nullptr, rall, nullptr, yall, w1.raw);
    launch_gcv_finish(c.stream, 1, w1.raw, w1.edf, w1.ok, nall, w1.rss, w1.gcv);
    GlsOut o;
    finish_single(w1, 0, grid[best], Mall, nall, mask, o);
    if (chol_failed) o.ldlt = 1;  // redone in FP64 (mixed_failed)
    o.grid = grid;
    o.curve = curve;
    return o;
  }
};

void write_gls(const GlsOut& o, int nc, int k, dgpu_gls_result* out) {
  std::memcpy(out->theta, o.theta.data(), sizeof(double) * o.theta.size());
  out->n_components = nc;
  out->n_spatial = k;
  out->lambda = o.lambda;
  out->gcv = o.gcv;
  out->effective_dof = o.edf;
  out->rss = o.rss;
  out->n_lambda_out = static_cast<int>(o.grid.size());
  out->refine_correction = o.refine_correction;
  out->precision_used = o.prec_used;
  out->used_ldlt = o.ldlt;
  if (out->lambda_grid && !o.grid.empty()) std::memcpy(out->lambda_grid, o.grid.data(), sizeof(double) * o.grid.size());
  if (out->gcv_curve && !o.curve.empty()) std::memcpy(out->gcv_curve, o.curve.data(), sizeof(double) * o.curve.size());
}

template <class F>
int guarded(dgpu_context* ctx, F&& f) {
  return run_entry(ctx, true, true, std::forward<F>(f));
}

// Rows for the direct solver entry points: one unit per row.
void direct_rows(Engine& E, const double* points, const double* target, const double* weights, const double* bn) {
  const int64_t m = E.N;
  std::vector<uint8_t> valid(m, 1);
  std::vector<double> d(static_cast<size_t>(m) * E.k);
  for (int64_t i = 0; i < m; ++i) E.tp.design_row(points[2 * i], points[2 * i + 1], d.data() + i * E.k);
  E.alloc_rows();
  Context& c = E.c;
  DGPU_CUDA(h2d_async(E.R.valid, valid.data(), m, c.stream));
  DGPU_CUDA(h2d_async(E.R.t, target, 8 * m, c.stream));
  DGPU_CUDA(h2d_async(E.R.w, weights, 8 * m, c.stream));
  if (E.nc) DGPU_CUDA(h2d_async(E.R.bn, bn, 8 * m * E.nc, c.stream));
  DGPU_CUDA(h2d_async(E.R.d, d.data(), 8 * d.size(), c.stream));
  DGPU_CUDA(cudaStreamSynchronize(c.stream));
}

}  // namespace

extern "C" {

int dgpu_solve_gls(dgpu_context* ctx, const double* knots, int n_knots, const double* points, int64_t m,
                   const double* target, const double* weights, const double* bn, int nc, double lam,
                   int precision, dgpu_gls_result* out) {
  return guarded(ctx, [&](Context& c) {
    const ThinPlate tp(knots, n_knots);
    if (m <= 0) fail(DGPU_ERR_RUNTIME, "solve_gls: no rows");
    Engine E(c, precision, tp, nc, m, 1, static_cast<int>(m));
    direct_rows(E, points, target, weights, bn);
    std::vector<uint8_t> ones(m, 1);
    uint8_t* mask = up(c, kSlotSeedPos, ones.data(), ones.size());
    GlsOut o = E.fixed(lam, mask);
    o.grid.clear();
    o.curve.clear();
    write_gls(o, nc, tp.k, out);
  });
}

int dgpu_solve_gls_gcv(dgpu_context* ctx, const double* knots, int n_knots, const double* points, int64_t m,
                       const double* target, const double* weights, const double* bn, int nc,
                       const double* lambda_grid, int n_lambda, int precision, dgpu_gls_result* out) {
  return guarded(ctx, [&](Context& c) {
    const ThinPlate tp(knots, n_knots);
    if (n_lambda <= 0) fail(DGPU_ERR_RUNTIME, "solve_gls_gcv: lambda_grid is empty");
    if (m <= 0) fail(DGPU_ERR_RUNTIME, "solve_gls: no rows");
    Engine E(c, precision, tp, nc, m, 1, static_cast<int>(m));
    direct_rows(E, points, target, weights, bn);
    std::vector<uint8_t> ones(m, 1);
    uint8_t* mask = up(c, kSlotSeedPos, ones.data(), ones.size());
    const GlsOut o = E.gcv(std::vector<double>(lambda_grid, lambda_grid + n_lambda), mask);
    write_gls(o, nc, tp.k, out);
  });
}

int dgpu_solve_gls_cv(dgpu_context* ctx, const double* knots, int n_knots, const double* points, int64_t m,
                      const double* target, const double* weights, const double* bn, int nc,
                      const double* lambda_grid, int n_lambda, const int32_t* group, int n_groups, int precision,
                      dgpu_gls_result* out) {
  return guarded(ctx, [&](Context& c) {
    const ThinPlate tp(knots, n_knots);
    if (n_lambda <= 0) fail(DGPU_ERR_RUNTIME, "solve_gls_cv: lambda_grid is empty");
    if (m <= 0) fail(DGPU_ERR_RUNTIME, "solve_gls: no rows");
    Engine E(c, precision, tp, nc, m, 1, static_cast<int>(m));
    direct_rows(E, points, target, weights, bn);
    std::vector<uint8_t> ones(m, 1);
    uint8_t* mask = up(c, kSlotSeedPos, ones.data(), ones.size());
    const std::vector<double> grid(lambda_grid, lambda_grid + n_lambda);
    GlsOut o;
    if (n_groups < 2) {
      o = E.gcv(grid, mask);
    } else {
      std::vector<int> fold(m);
      for (int64_t i = 0; i < m; ++i) {
        if (group[i] < 0 || group[i] >= n_groups) fail(DGPU_ERR_RUNTIME, "solve_gls_cv: group id out of range");
        fold[i] = group[i];
      }
      o = E.cv(grid, mask, fold, n_groups, -1, false);
    }
    write_gls(o, nc, tp.k, out);
  });
}

int dgpu_fit_kernel(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* science,
                    const float* reference, const float* science_var, const float* reference_var,
                    const uint8_t* science_mask, const uint8_t* reference_mask, const double* knots, int n_knots,
                    const int32_t* stamp_x, const int32_t* stamp_y, int n_stamps, int stamp_radius, double beta,
                    int n_max, int radius, const double* lambda_grid, int n_lambda, double clip_sigma,
                    int clip_iterations, int min_stamps, int cv_folds, int precision, dgpu_gls_result* out) {
  return guarded(ctx, [&](Context& c) {
    if (width <= 0 || height <= 0) fail(DGPU_ERR_INVALID, "image must be non-empty");
    if (width * height >= (int64_t(1) << 31)) fail(DGPU_ERR_INVALID, "image too large");
    if (n_lambda <= 0) fail(DGPU_ERR_RUNTIME, "solve_gls_gcv: lambda_grid is empty");
    if (stamp_radius < 0) fail(DGPU_ERR_INVALID, "stamp_radius must be >= 0");
    const int w = static_cast<int>(width), h = static_cast<int>(height);
    const size_t npx = static_cast<size_t>(w) * h;
    const Basis b(beta, n_max, radius);
    const ThinPlate tp(knots, n_knots);
    const int nc = b.nc, k = tp.k;
    cudaStream_t st = c.stream;
    const auto* sci = static_cast<const float*>(stage_in(c, mem, science, 4 * npx, kSlotInSci));
    const auto* ref = static_cast<const float*>(stage_in(c, mem, reference, 4 * npx, kSlotInRef));
    const auto* vs = static_cast<const float*>(stage_in(c, mem, science_var, 4 * npx, kSlotInVarS));
    const auto* vr = static_cast<const float*>(stage_in(c, mem, reference_var, 4 * npx, kSlotInVarR));
    const auto* sm = static_cast<const uint8_t*>(stage_in(c, mem, science_mask, npx, kSlotInMaskS));
    const auto* rm = static_cast<const uint8_t*>(stage_in(c, mem, reference_mask, npx, kSlotInMaskR));
    const bool have_var = vs != nullptr || vr != nullptr;
    const bool have_cvar = vr != nullptr;

    StampGeom g;
    g.w = w;
    g.h = h;
    g.sr = stamp_radius;
    g.S = 2 * stamp_radius + 1;
    g.SS = g.S * g.S;
    g.r = b.radius;
    g.ks = b.ks;
    g.n_max = n_max;
    g.nc = nc;
    g.pmax = g.S + 2 * b.radius;
    g.have_var = have_var ? 1 : 0;
    g.have_cvar = have_cvar ? 1 : 0;
    const int64_t N = static_cast<int64_t>(n_stamps) * g.SS;
    if (N == 0) fail(DGPU_ERR_RUNTIME, "fit_kernel: no usable stamp pixels");

    Engine E(c, precision, tp, nc, N, g.SS, n_stamps);
    E.alloc_rows();
    float* fill = static_cast<float*>(c.slot(kSlotScratch2, 64));
    {
      StageTimer t(c, "fit: stamp B_n convolve");
      launch_strided_median(c, kSampleReference, static_cast<int64_t>(npx), ref, rm, fill);
      int* dsx = up(c, kSlotBright, reinterpret_cast<const int*>(stamp_x), static_cast<size_t>(n_stamps));
      int* dsy = static_cast<int*>(c.slot(kSlotCompOut, sizeof(int) * std::max(n_stamps, 1)));
      DGPU_CUDA(h2d_async(dsy, stamp_y, sizeof(int) * n_stamps, st));
      const auto taps = b.taps();
      float* dt = up(c, kSlotTaps, taps.data(), taps.size());
      std::vector<int2> ord(nc);
      for (int i = 0; i < nc; ++i) ord[i] = make_int2(b.orders[i].first, b.orders[i].second);
      int2* dord = up(c, kSlotRootRank, ord.data(), ord.size());
      launch_stamp_gather(st, g, n_stamps, dsx, dsy, sci, ref, vs, vr, sm, rm, dt, dord, fill, E.R);
      const TpsDev t2 = upload_tps(c, tp);
      launch_design_weights(st, N, t2, E.R, have_var ? 1 : 0);
    }
    StageTimer solve_timer(c, "fit: GLS solve");
    const auto used = down(c, E.R.stamp_used, n_stamps);
    // Contributing stamps in supplied order (src/fit.cpp:196-229).
    std::vector<int> comp_of(n_stamps, -1), contrib;
    for (int s = 0; s < n_stamps; ++s)
      if (used[s]) {
        comp_of[s] = static_cast<int>(contrib.size());
        contrib.push_back(s);
      }
    const int nct = static_cast<int>(contrib.size());
    if (nct == 0) fail(DGPU_ERR_RUNTIME, "fit_kernel: no usable stamp pixels");
    std::vector<uint8_t> accepted(n_stamps, 0);
    for (int s : contrib) accepted[s] = 1;
    uint8_t* d_acc = static_cast<uint8_t*>(c.slot(kSlotSeedPos, std::max(n_stamps, 1)));
    // Reweight inputs.
    float* phi = nullptr;
    if (have_cvar) {
      std::vector<float> ph(static_cast<size_t>(nc) * b.ks * b.ks);
      for (int q = 0; q < nc; ++q) {
        const auto k2 = b.kernel2d(q);
        std::copy(k2.begin(), k2.end(), ph.begin() + static_cast<size_t>(q) * b.ks * b.ks);
      }
      phi = up(c, kSlotPhi, ph.data(), ph.size());
    }
    const TpsDev tdev = upload_tps(c, tp);
    int* dsx = static_cast<int*>(c.slot(kSlotBright, sizeof(int) * std::max(n_stamps, 1)));
    int* dsy = static_cast<int*>(c.slot(kSlotCompOut, sizeof(int) * std::max(n_stamps, 1)));
    const size_t ns1 = static_cast<size_t>(std::max(n_stamps, 1));
    double* chi2_d = static_cast<double*>(
        c.slot(kSlotCompStats, sizeof(double) * ns1 + sizeof(int) * ns1 + 16 + stamp_chi2_scratch_bytes(n_stamps)));
    int* cnt_d = reinterpret_cast<int*>(chi2_d + ns1);
    void* chi2_scratch = reinterpret_cast<void*>(
        (reinterpret_cast<uintptr_t>(cnt_d + ns1) + 15) & ~static_cast<uintptr_t>(15));  // 16-aligned past cnt_d

    const int clip_passes = (clip_sigma > 0.0 && clip_iterations > 0) ? clip_iterations : 0;
    const int do_iterate = clip_iterations > 0 ? 1 : 0;
    const int min_pass = (do_iterate && have_var) ? 1 : 0;
    const int hard_max = std::max(clip_passes, min_pass);
    const int floor_stamps = std::max(1, std::min(min_stamps, nct));
    const std::vector<double> grid(lambda_grid, lambda_grid + n_lambda);
    int warm_start = -1;
    size_t cv_exact_bytes = 0;
    GlsOut gls;
    std::vector<double> stamp_chi2(n_stamps, kNaN);
    std::vector<int> cnt(n_stamps, 0);
    long long npix = 0;
    double reduced = kNaN;
    const double knot_spacing = tp.min_knot_spacing();
    bool use_stamped = knot_spacing > 0.0 && knot_spacing >= 16.0 * (2.0 * stamp_radius + 1.0);
    if (const char* e = std::getenv("DELTA_STAMP_APPROX")) use_stamped = std::atoi(e) != 0;

    // Per-stamp chi^2 of each solution rides on the solution's own read-back.
    E.on_fetch_bytes = (sizeof(double) + sizeof(int)) * static_cast<size_t>(n_stamps) + 64;
    E.on_fetch = [&](const double* d_theta, Fetch& f) {
      launch_stamp_chi2(st, n_stamps, nc, k, g.SS, E.R, d_acc, d_theta, chi2_d, cnt_d, chi2_scratch);
      f.add(stamp_chi2.data(), chi2_d, n_stamps);
      f.add(cnt.data(), cnt_d, n_stamps);
    };
    for (int iter = 0;; ++iter) {
      DGPU_CUDA(h2d_async(d_acc, accepted.data(), n_stamps, st));
      // The active-row count comes back with the solve (the rows are the same).
      if (cv_folds > 1) {
        std::vector<int> fold(n_stamps, -1);
        for (int s = 0; s < n_stamps; ++s)
          if (comp_of[s] >= 0) fold[s] = comp_of[s] % cv_folds;
        gls = E.cv(grid, d_acc, fold, cv_folds, warm_start, use_stamped);
        warm_start = static_cast<int>(std::min_element(gls.curve.begin(), gls.curve.end()) - gls.curve.begin());
      } else {
        gls = E.gcv(grid, d_acc);
      }
      npix = gls.npix;
      if (npix == 0) fail(DGPU_ERR_RUNTIME, "fit_kernel: all stamp pixels clipped");
      if (cv_folds > 1 && !use_stamped) cv_exact_bytes = static_cast<size_t>(npix) * E.P * sizeof(double);
      const double denom = static_cast<double>(npix) - gls.edf;
      reduced = denom > 0.0 ? gls.rss / denom : kNaN;
      if (have_var) {
        DGPU_CUDA(h2d_async(dsx, stamp_x, sizeof(int) * n_stamps, st));
        DGPU_CUDA(h2d_async(dsy, stamp_y, sizeof(int) * n_stamps, st));
        launch_reweight(st, g, n_stamps, tdev, dsx, dsy, E.R, d_acc, cnt_d, gls.d_theta, phi, vr, rm);
      }
      std::vector<int> to_reject;
      if (clip_passes > 0 && iter < clip_passes) {
        std::vector<double> act;
        for (int s : contrib)
          if (accepted[s] && cnt[s] > 0) act.push_back(stamp_chi2[s]);
        const int n_active = static_cast<int>(act.size());
        if (n_active > floor_stamps) {
          const double med = median_copy(act);
          std::vector<double> dev;
          for (double v : act) dev.push_back(std::fabs(v - med));
          const double thr = med + clip_sigma * 1.4826 * median_copy(dev);
          std::vector<int> cand;
          for (int s : contrib)
            if (accepted[s] && cnt[s] > 0 && stamp_chi2[s] > thr) cand.push_back(s);
          std::stable_sort(cand.begin(), cand.end(), [&](int a2, int b2) { return stamp_chi2[a2] > stamp_chi2[b2]; });
          for (int s : cand) {
            if (n_active - static_cast<int>(to_reject.size()) <= floor_stamps) break;
            to_reject.push_back(s);
          }
        }
      }
      if (to_reject.empty() && iter >= min_pass) break;
      if (iter >= hard_max) break;
      for (int s : to_reject) accepted[s] = 0;
    }
    int n_used = 0;
    for (int s : contrib)
      if (accepted[s] && std::isfinite(stamp_chi2[s])) ++n_used;
    write_gls(gls, nc, k, out);
    const auto sums = b.component_sums();
    if (out->component_sums) std::memcpy(out->component_sums, sums.data(), sizeof(double) * nc);
    out->n_pixels = npix;
    out->n_stamps_total = nct;
    out->n_stamps_used = n_used;
    out->n_stamps_rejected = nct - n_used;
    out->reduced_chi2 = reduced;
    out->cv_exact_design_bytes = static_cast<int64_t>(cv_exact_bytes);
    for (int i = 0; i < nct; ++i) {
      const int s = contrib[i];
      if (out->stamp_x) out->stamp_x[i] = stamp_x[s];
      if (out->stamp_y) out->stamp_y[i] = stamp_y[s];
      if (out->stamp_chi2) out->stamp_chi2[i] = stamp_chi2[s];
      if (out->stamp_accepted) out->stamp_accepted[i] = accepted[s];
    }
  });
}

// GCV score and weighted RSS of the stamp fit at one lambda with the kernel
// basis shifted by (dx, dy) and scaled by s, and their gradients with respect
// to (log lambda, dx, dy, s) through the adjoint of the normal-equation map
// (k_gcv_grad.cu). First-pass weights 1 / (Var_t + Var_c), no clipping.
int dgpu_stamp_gcv(dgpu_context* ctx, int mem, int64_t width, int64_t height, const float* science,
                   const float* reference, const float* science_var, const float* reference_var,
                   const uint8_t* science_mask, const uint8_t* reference_mask, const double* knots, int n_knots,
                   const int32_t* stamp_x, const int32_t* stamp_y, int n_stamps, int stamp_radius, double beta,
                   int n_max, int radius, double log_lambda, double dx, double dy, double scale, double* values,
                   double* theta, double* grad_gcv, double* grad_rss) {
  return guarded(ctx, [&](Context& c) {
    if (width <= 0 || height <= 0) fail(DGPU_ERR_INVALID, "image must be non-empty");
    if (width * height >= (int64_t(1) << 31)) fail(DGPU_ERR_INVALID, "image too large");
    if (!science || !reference || !knots || !values) fail(DGPU_ERR_INVALID, "stamp_gcv: missing argument");
    if (stamp_radius < 0) fail(DGPU_ERR_INVALID, "stamp_radius must be >= 0");
    if (!std::isfinite(log_lambda) || !std::isfinite(dx) || !std::isfinite(dy) || !std::isfinite(scale) ||
        scale == 0.0)
      fail(DGPU_ERR_INVALID, "stamp_gcv: log_lambda, shift and a non-zero scale must be finite");
    if (n_stamps <= 0 || !stamp_x || !stamp_y) fail(DGPU_ERR_RUNTIME, "fit_kernel: no usable stamp pixels");
    const int w = static_cast<int>(width), h = static_cast<int>(height);
    const size_t npx = static_cast<size_t>(w) * h;
    const Basis b(beta, n_max, radius);
    const ThinPlate tp(knots, n_knots);
    const int nc = b.nc, k = tp.k, P = (nc + 1) * k;
    cudaStream_t st = c.stream;
    reset_status(c);
    const auto* sci = static_cast<const float*>(stage_in(c, mem, science, 4 * npx, kSlotInSci));
    const auto* ref = static_cast<const float*>(stage_in(c, mem, reference, 4 * npx, kSlotInRef));
    const auto* vs = static_cast<const float*>(stage_in(c, mem, science_var, 4 * npx, kSlotInVarS));
    const auto* vr = static_cast<const float*>(stage_in(c, mem, reference_var, 4 * npx, kSlotInVarR));
    const auto* sm = static_cast<const uint8_t*>(stage_in(c, mem, science_mask, npx, kSlotInMaskS));
    const auto* rm = static_cast<const uint8_t*>(stage_in(c, mem, reference_mask, npx, kSlotInMaskR));
    const bool have_var = vs != nullptr || vr != nullptr;
    StampGeom g;
    g.w = w;
    g.h = h;
    g.sr = stamp_radius;
    g.S = 2 * stamp_radius + 1;
    g.SS = g.S * g.S;
    g.r = b.radius;
    g.ks = b.ks;
    g.n_max = n_max;
    g.nc = nc;
    g.pmax = g.S + 2 * b.radius;
    g.have_var = have_var ? 1 : 0;
    g.have_cvar = vr != nullptr ? 1 : 0;
    const int64_t N = static_cast<int64_t>(n_stamps) * g.SS;
    Engine E(c, DGPU_PREC_FP64, tp, nc, N, g.SS, n_stamps);
    E.alloc_rows();
    const int rk = E.rk;
    float* fill = static_cast<float*>(c.slot(kSlotScratch2, 64));
    launch_strided_median(c, kSampleReference, static_cast<int64_t>(npx), ref, rm, fill);
    int* dsx = up(c, kSlotBright, reinterpret_cast<const int*>(stamp_x), static_cast<size_t>(n_stamps));
    int* dsy = up(c, kSlotCompOut, reinterpret_cast<const int*>(stamp_y), static_cast<size_t>(n_stamps));
    // Taps: x tables carry the scale (u_c = s B_n), y tables do not.
    std::vector<double> gx, dgx, gy, dgy;
    b.shifted_taps(dx, gx, dgx);
    b.shifted_taps(dy, gy, dgy);
    const size_t nt = gx.size();
    std::vector<float> taps(4 * nt);
    for (size_t i = 0; i < nt; ++i) {
      taps[i] = static_cast<float>(scale * gx[i]);
      taps[nt + i] = static_cast<float>(scale * dgx[i]);
      taps[2 * nt + i] = static_cast<float>(gy[i]);
      taps[3 * nt + i] = static_cast<float>(dgy[i]);
    }
    float* dt = up(c, kSlotTaps, taps.data(), taps.size());
    std::vector<int2> ord(nc);
    for (int i = 0; i < nc; ++i) ord[i] = make_int2(b.orders[i].first, b.orders[i].second);
    int2* dord = up(c, kSlotRootRank, ord.data(), ord.size());
    FitRows Rx = E.R, Ry = E.R;
    Rx.bn = static_cast<double*>(c.slot(kSlotGrad4, sizeof(double) * static_cast<size_t>(N) * nc));
    Ry.bn = static_cast<double*>(c.slot(kSlotGrad5, sizeof(double) * static_cast<size_t>(N) * nc));
    {
      StageTimer t(c, "gradient: stamp B_n convolve");
      // Derivative rows first: the main gather's row flags and values come last.
      launch_stamp_gather(st, g, n_stamps, dsx, dsy, sci, ref, vs, vr, sm, rm, dt + nt, dord, fill, Rx, dt + 2 * nt);
      launch_stamp_gather(st, g, n_stamps, dsx, dsy, sci, ref, vs, vr, sm, rm, dt, dord, fill, Ry, dt + 3 * nt);
      launch_stamp_gather(st, g, n_stamps, dsx, dsy, sci, ref, vs, vr, sm, rm, dt, dord, fill, E.R, dt + 2 * nt);
      launch_design_weights(st, N, upload_tps(c, tp), E.R, have_var ? 1 : 0);
    }
    StageTimer solve_timer(c, "gradient: GCV adjoint");
    std::vector<uint8_t> ones(n_stamps, 1);
    uint8_t* d_acc = up(c, kSlotSeedPos, ones.data(), ones.size());
    double* M = static_cast<double*>(c.slot(kSlotScratch1, sizeof(double) * (static_cast<size_t>(P) * P + P + 4)));
    double* rhs = M + static_cast<size_t>(P) * P;
    double* ywy = rhs + P;
    double* raw = ywy + 1;
    long long* n = reinterpret_cast<long long*>(raw + 1);
    E.assemble(d_acc, M, rhs, ywy, n);
    const double lam = std::exp(log_lambda);
    const int m = gcv_rhs_cols(P, k, rk);
    double* B = static_cast<double*>(c.slot(kSlotGrad3, sizeof(double) * 2 * static_cast<size_t>(P) * m));
    double* X = B + static_cast<size_t>(P) * m;
    launch_build_rhs_f(st, P, k, rk, rhs, E.d_fk, B);
    launch_sym_solve_many(c, P, k, M, lam, E.d_pen, B, m, X);
    double* work = static_cast<double*>(c.slot(kSlotGrad2, sizeof(double) * gcv_stats_doubles(P, k, rk) +
                                                   sizeof(GcvScalars) + 64));
    GcvScalars* scal = reinterpret_cast<GcvScalars*>(work + gcv_stats_doubles(P, k, rk));
    launch_gcv_theta(st, P, k, rk, X, E.d_fk, work);
    launch_quad_err(c, 1, P, work, M, nullptr, rhs, nullptr, ywy, raw);
    launch_gcv_stats(st, P, k, rk, X, E.d_fk, lam, raw, n, work, scal);
    const int nq = m - 1;
    double* out6 = static_cast<double*>(c.slot(kSlotGrad7, sizeof(double) * (6 * static_cast<size_t>(gcv_rows_blocks(N)) + 8)));
    if (grad_gcv || grad_rss) {
      GcvRowsArgs a;
      a.N = N;
      a.nc = nc;
      a.k = k;
      a.nq = nq;
      a.valid = E.R.valid;
      a.w = E.R.w;
      a.t = E.R.t;
      a.d = E.R.d;
      a.bn = E.R.bn;
      a.bnx = Rx.bn;
      a.bny = Ry.bn;
      a.theta = work;
      a.z = work + P + nq;
      a.X = X;
      a.scal = scal;
      a.scale = scale;
      a.partial = out6 + 8;
      launch_gcv_rows(st, a, out6);
    }
    GcvScalars hs{};
    double g6[6] = {0, 0, 0, 0, 0, 0};
    std::vector<double> th(P);
    read_back(c, &hs, scal, sizeof(GcvScalars));
    read_back(c, th.data(), work, sizeof(double) * P);
    if (grad_gcv || grad_rss) read_back(c, g6, out6, sizeof(g6));
    check_status(c);  // synchronises
    if (hs.n <= 0.0) fail(DGPU_ERR_RUNTIME, "fit_kernel: no usable stamp pixels");
    values[0] = hs.gcv;
    values[1] = hs.rss;
    values[2] = hs.edf;
    values[3] = hs.n;
    if (theta) std::copy(th.begin(), th.end(), theta);
    if (grad_gcv) {
      grad_gcv[0] = hs.dgcv_dloglam;
      grad_gcv[1] = g6[0];
      grad_gcv[2] = g6[1];
      grad_gcv[3] = g6[2];
    }
    if (grad_rss) {
      grad_rss[0] = hs.drss_dloglam;
      grad_rss[1] = g6[3];
      grad_rss[2] = g6[4];
      grad_rss[3] = g6[5];
    }
  });
}

}  // extern "C"
