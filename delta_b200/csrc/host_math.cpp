// Host-side FP64 set-up math: Gauss-Hermite taps, thin-plate spline constants,
// coarse-lattice geometry. Small (O(n_max * ks), O(k^3)) and computed once per
// call; the per-pixel work runs on the device.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <limits>

#include "internal.h"

namespace dgpu {

// ---------------------------------------------------------------------------
// Gauss-Hermite basis: g_n(x) = [2^n n! sqrt(pi) beta]^-1/2 H_n(x/beta)
// exp(-x^2/2beta^2), sampled on integer offsets -r..r through the physicists'
// Hermite recurrence, log-normalised (reference src/basis.cpp:9-59). The
// component order (total order, then ny) is the reference's
// (src/basis.cpp:53-58) because theta is laid out in it.
// ---------------------------------------------------------------------------

int default_radius(double beta, int n_max) {
  const double scale = beta * std::sqrt(static_cast<double>(n_max + 1));
  return std::max(static_cast<int>(std::ceil(3.0 * scale)), 3);
}

Basis::Basis(double beta_, int n_max_, int radius_) : beta(beta_), n_max(n_max_) {
  if (!(beta > 0.0)) fail(DGPU_ERR_INVALID, "beta must be > 0");
  if (n_max < 0) fail(DGPU_ERR_INVALID, "n_max must be >= 0");
  radius = radius_ > 0 ? radius_ : default_radius(beta, n_max);
  if (radius < 1) fail(DGPU_ERR_INVALID, "radius must be >= 1");
  ks = 2 * radius + 1;
  const double ln2 = std::log(2.0);
  const double half_ln_pi = 0.5 * std::log(std::acos(-1.0));
  const double ln_beta = std::log(beta);
  std::vector<double> norm(n_max + 1);
  for (int n = 0; n <= n_max; ++n)
    norm[n] = std::exp(-0.5 * (n * ln2 + std::lgamma(n + 1.0) + half_ln_pi + ln_beta));
  b1d.assign(static_cast<size_t>(n_max + 1) * ks, 0.0);
  for (int i = 0; i < ks; ++i) {
    const double t = static_cast<double>(i - radius) / beta;
    const double g = std::exp(-0.5 * t * t);
    double hm1 = 1.0;
    b1d[i] = norm[0] * hm1 * g;
    if (n_max >= 1) {
      double hc = 2.0 * t;
      b1d[static_cast<size_t>(ks) + i] = norm[1] * hc * g;
      for (int n = 2; n <= n_max; ++n) {
        const double hn = 2.0 * t * hc - 2.0 * (n - 1) * hm1;
        b1d[static_cast<size_t>(n) * ks + i] = norm[n] * hn * g;
        hm1 = hc;
        hc = hn;
      }
    }
  }
  for (int total = 0; total <= n_max; ++total)
    for (int ny = 0; ny <= total; ++ny) orders.emplace_back(total - ny, ny);
  nc = static_cast<int>(orders.size());
}

void Basis::shifted_taps(double d, std::vector<double>& g, std::vector<double>& dg) const {
  // g_n(u - d) and g_n'(u - d) at the offsets u = -r..r, with
  // g_n'(x) = norm_n / beta * (2 n H_{n-1}(t) - t H_n(t)) exp(-t^2 / 2), t = x / beta.
  // At d = 0, g is bit-identical to b1d (same arithmetic).
  const double ln2 = std::log(2.0);
  const double half_ln_pi = 0.5 * std::log(std::acos(-1.0));
  const double ln_beta = std::log(beta);
  g.assign(static_cast<size_t>(n_max + 1) * ks, 0.0);
  dg.assign(g.size(), 0.0);
  for (int i = 0; i < ks; ++i) {
    const double t = (static_cast<double>(i - radius) - d) / beta;
    const double e = std::exp(-0.5 * t * t);
    double hm1 = 0.0, hc = 1.0;  // H_{n-1}, H_n
    for (int n = 0; n <= n_max; ++n) {
      const double norm = std::exp(-0.5 * (n * ln2 + std::lgamma(n + 1.0) + half_ln_pi + ln_beta));
      g[static_cast<size_t>(n) * ks + i] = norm * hc * e;
      dg[static_cast<size_t>(n) * ks + i] = norm / beta * (2.0 * n * hm1 - t * hc) * e;
      const double hn = 2.0 * t * hc - 2.0 * n * hm1;
      hm1 = hc;
      hc = hn;
    }
  }
}

std::vector<float> Basis::taps() const {
  std::vector<float> t(b1d.size());
  for (size_t i = 0; i < b1d.size(); ++i) t[i] = static_cast<float>(b1d[i]);
  return t;
}

std::vector<float> Basis::kernel2d(int c) const {
  const int nx = orders.at(c).first, ny = orders.at(c).second;
  std::vector<float> k(static_cast<size_t>(ks) * ks);
  for (int iy = 0; iy < ks; ++iy)
    for (int ix = 0; ix < ks; ++ix)
      k[static_cast<size_t>(iy) * ks + ix] =
          static_cast<float>(b1d[static_cast<size_t>(ny) * ks + iy] * b1d[static_cast<size_t>(nx) * ks + ix]);
  return k;
}

std::vector<double> Basis::component_sums() const {
  std::vector<double> s1(n_max + 1, 0.0);
  for (int n = 0; n <= n_max; ++n)
    for (int i = 0; i < ks; ++i) s1[n] += b1d[static_cast<size_t>(n) * ks + i];
  std::vector<double> out;
  for (auto [nx, ny] : orders) out.push_back(s1[nx] * s1[ny]);
  return out;
}

// ---------------------------------------------------------------------------
// Thin-plate regression spline constants (reference src/spatial.cpp:13-111).
// The null space Z of the affine trend T = [1, u, v] is taken from a
// Householder QR with the LAPACK / Eigen reflector convention
// (beta = -sign(alpha) ||x||, v_0 = 1, tau = (beta - alpha) / beta): theta is
// expressed in that basis, so a fitted solution from the reference drops in.
// ---------------------------------------------------------------------------

static double tps_green(double r2) { return r2 <= 0.0 ? 0.0 : 0.5 * r2 * std::log(r2); }

ThinPlate::ThinPlate(const double* knots, int k_) : k(k_) {
  if (k < 3) fail(DGPU_ERR_INVALID, "need at least 3 knots");
  double sx = 0, sy = 0;
  for (int i = 0; i < k; ++i) {
    sx += knots[2 * i];
    sy += knots[2 * i + 1];
  }
  cx = sx / k;
  cy = sy / k;
  double mx = 0, my = 0;
  for (int i = 0; i < k; ++i) {
    mx = std::max(mx, std::fabs(knots[2 * i] - cx));
    my = std::max(my, std::fabs(knots[2 * i + 1] - cy));
  }
  scale = std::max({mx, my, 1e-12});
  kn.resize(2 * k);
  for (int i = 0; i < k; ++i) {
    kn[2 * i] = (knots[2 * i] - cx) / scale;
    kn[2 * i + 1] = (knots[2 * i + 1] - cy) / scale;
  }
  // Householder QR of T (k x 3), then Q = H0 H1 H2 (k x k).
  std::vector<double> a(static_cast<size_t>(k) * 3);
  for (int i = 0; i < k; ++i) {
    a[3 * i] = 1.0;
    a[3 * i + 1] = kn[2 * i];
    a[3 * i + 2] = kn[2 * i + 1];
  }
  double tau[3];
  for (int j = 0; j < 3; ++j) {
    const double c0 = a[3 * j + j];
    double tail = 0.0;
    for (int i = j + 1; i < k; ++i) tail += a[3 * i + j] * a[3 * i + j];
    double beta;
    if (tail <= DBL_MIN) {
      tau[j] = 0.0;
      beta = c0;
      for (int i = j + 1; i < k; ++i) a[3 * i + j] = 0.0;
    } else {
      beta = std::sqrt(c0 * c0 + tail);
      if (c0 >= 0.0) beta = -beta;
      for (int i = j + 1; i < k; ++i) a[3 * i + j] /= (c0 - beta);
      tau[j] = (beta - c0) / beta;
    }
    a[3 * j + j] = beta;
    for (int col = j + 1; col < 3; ++col) {
      double s = a[3 * j + col];
      for (int i = j + 1; i < k; ++i) s += a[3 * i + j] * a[3 * i + col];
      a[3 * j + col] -= tau[j] * s;
      for (int i = j + 1; i < k; ++i) a[3 * i + col] -= tau[j] * a[3 * i + j] * s;
    }
  }
  std::vector<double> q(static_cast<size_t>(k) * k, 0.0);
  for (int i = 0; i < k; ++i) q[static_cast<size_t>(i) * k + i] = 1.0;
  for (int j = 2; j >= 0; --j) {
    if (tau[j] == 0.0) continue;
    for (int col = 0; col < k; ++col) {
      double s = q[static_cast<size_t>(j) * k + col];
      for (int i = j + 1; i < k; ++i) s += a[3 * i + j] * q[static_cast<size_t>(i) * k + col];
      q[static_cast<size_t>(j) * k + col] -= tau[j] * s;
      for (int i = j + 1; i < k; ++i) q[static_cast<size_t>(i) * k + col] -= tau[j] * a[3 * i + j] * s;
    }
  }
  const int nr = k - 3;
  z.assign(static_cast<size_t>(k) * std::max(nr, 0), 0.0);
  for (int i = 0; i < k; ++i)
    for (int m = 0; m < nr; ++m) z[static_cast<size_t>(i) * nr + m] = q[static_cast<size_t>(i) * k + 3 + m];
  // Bending-energy penalty blkdiag(Z^T E Z, 0_3), symmetrised.
  std::vector<double> e(static_cast<size_t>(k) * k);
  for (int i = 0; i < k; ++i)
    for (int j = 0; j < k; ++j) {
      const double dx = kn[2 * i] - kn[2 * j], dy = kn[2 * i + 1] - kn[2 * j + 1];
      e[static_cast<size_t>(i) * k + j] = tps_green(dx * dx + dy * dy);
    }
  std::vector<double> ez(static_cast<size_t>(k) * std::max(nr, 0), 0.0);
  for (int i = 0; i < k; ++i)
    for (int m = 0; m < nr; ++m) {
      double s = 0.0;
      for (int j = 0; j < k; ++j) s += e[static_cast<size_t>(i) * k + j] * z[static_cast<size_t>(j) * nr + m];
      ez[static_cast<size_t>(i) * nr + m] = s;
    }
  penalty.assign(static_cast<size_t>(k) * k, 0.0);
  for (int m = 0; m < nr; ++m)
    for (int l = 0; l < nr; ++l) {
      double s = 0.0;
      for (int i = 0; i < k; ++i) s += z[static_cast<size_t>(i) * nr + m] * ez[static_cast<size_t>(i) * nr + l];
      penalty[static_cast<size_t>(m) * k + l] = s;
    }
  for (int m = 0; m < k; ++m)
    for (int l = m + 1; l < k; ++l) {
      const double avg = 0.5 * (penalty[static_cast<size_t>(m) * k + l] + penalty[static_cast<size_t>(l) * k + m]);
      penalty[static_cast<size_t>(m) * k + l] = avg;
      penalty[static_cast<size_t>(l) * k + m] = avg;
    }
}

void ThinPlate::design_row(double x, double y, double* out) const {
  const double ux = (x - cx) / scale, uy = (y - cy) / scale;
  const int nr = k - 3;
  for (int m = 0; m < nr; ++m) out[m] = 0.0;
  for (int j = 0; j < k; ++j) {
    const double dx = ux - kn[2 * j], dy = uy - kn[2 * j + 1];
    const double s = tps_green(dx * dx + dy * dy);
    for (int m = 0; m < nr; ++m) out[m] += s * z[static_cast<size_t>(j) * nr + m];
  }
  out[nr] = 1.0;
  out[nr + 1] = ux;
  out[nr + 2] = uy;
}

double ThinPlate::min_knot_spacing() const {
  double best = std::numeric_limits<double>::infinity();
  for (int i = 0; i < k; ++i)
    for (int j = i + 1; j < k; ++j) {
      const double dx = kn[2 * i] - kn[2 * j], dy = kn[2 * i + 1] - kn[2 * j + 1];
      best = std::min(best, dx * dx + dy * dy);
    }
  return std::isfinite(best) ? std::sqrt(best) * scale : 0.0;
}

// Cyclic Jacobi eigensolver for a small symmetric matrix (row-major a, n x n).
// Eigenvalues ascending in w, eigenvectors as columns of v (row-major).
void sym_eig(int n, const double* a_in, double* w, double* v) {
  std::vector<double> a(a_in, a_in + static_cast<size_t>(n) * n);
  for (int i = 0; i < n * n; ++i) v[i] = 0.0;
  for (int i = 0; i < n; ++i) v[i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) (i == j ? diag : off) += a[i * n + j] * a[i * n + j];
    if (off <= 1e-30 * std::max(diag, 1e-300)) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a[p * n + q];
        if (std::fabs(apq) < 1e-300) continue;
        const double app = a[p * n + p], aqq = a[q * n + q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int r = 0; r < n; ++r) {
          const double arp = a[r * n + p], arq = a[r * n + q];
          a[r * n + p] = c * arp - s * arq;
          a[r * n + q] = s * arp + c * arq;
        }
        for (int r = 0; r < n; ++r) {
          const double apr = a[p * n + r], aqr = a[q * n + r];
          a[p * n + r] = c * apr - s * aqr;
          a[q * n + r] = s * apr + c * aqr;
        }
        for (int r = 0; r < n; ++r) {
          const double vrp = v[r * n + p], vrq = v[r * n + q];
          v[r * n + p] = c * vrp - s * vrq;
          v[r * n + q] = s * vrp + c * vrq;
        }
      }
  }
  std::vector<int> idx(n);
  for (int i = 0; i < n; ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int x, int y) { return a[x * n + x] < a[y * n + y]; });
  std::vector<double> vs(v, v + static_cast<size_t>(n) * n);
  for (int j = 0; j < n; ++j) {
    w[j] = a[idx[j] * n + idx[j]];
    for (int r = 0; r < n; ++r) v[r * n + j] = vs[r * n + idx[j]];
  }
}

// Half-factor F (F F^T = P0 = blockdiag(penalty x (nc+1))), keeping the
// eigenpairs above wmax * k * eps (reference src/solve.cpp:47-65).
std::vector<double> ThinPlate::pen_half(int nc, int* r_out) const {
  std::vector<double> w(k), v(static_cast<size_t>(k) * k);
  sym_eig(k, penalty.data(), w.data(), v.data());
  double wmax = 0.0;
  for (double x : w) wmax = std::max(wmax, std::fabs(x));
  const double tol = wmax * k * std::numeric_limits<double>::epsilon();
  std::vector<int> keep;
  for (int i = 0; i < k; ++i)
    if (w[i] > tol) keep.push_back(i);
  const int r = static_cast<int>(keep.size());
  const int nf = nc + 1;
  const int p = nf * k;
  std::vector<double> f(static_cast<size_t>(p) * nf * r, 0.0);
  for (int b = 0; b < nf; ++b)
    for (int i = 0; i < k; ++i)
      for (int j = 0; j < r; ++j)
        f[static_cast<size_t>(b * k + i) * (nf * r) + b * r + j] =
            v[static_cast<size_t>(i) * k + keep[j]] * std::sqrt(w[keep[j]]);
  *r_out = r;
  return f;
}

// ---------------------------------------------------------------------------
// Coarse lattice geometry (reference src/subtract.cpp:107-124, 149-156,
// 265-316): stride = clamp(min_knot_spacing / 16, 1, 64); the exact per-pixel
// path below stride 4 or for frames within two strides.
// ---------------------------------------------------------------------------
FieldGeom make_field_geom(const ThinPlate& tp, int w, int h) {
  FieldGeom g;
  const double spacing = tp.min_knot_spacing();
  int stride = 1;
  if (spacing > 0.0) stride = std::clamp(static_cast<int>(spacing / 16), 1, 64);
  g.stride = stride;
  g.exact = stride < 4 || w <= 2 * stride || h <= 2 * stride;
  if (g.exact) return g;
  for (int p = 0; p < w - 1; p += stride) g.gx.push_back(p);
  g.gx.push_back(w - 1);
  for (int p = 0; p < h - 1; p += stride) g.gy.push_back(p);
  g.gy.push_back(h - 1);
  g.ncx = static_cast<int>(g.gx.size());
  g.ncy = static_cast<int>(g.gy.size());
  g.cellx.resize(w);
  g.wx.resize(w);
  for (int x = 0; x < w; ++x) {
    const int c0 = std::min(x / stride, g.ncx - 2);
    const int x0 = g.gx[c0], x1 = g.gx[c0 + 1];
    g.cellx[x] = c0;
    g.wx[x] = x1 > x0 ? static_cast<float>(x - x0) / static_cast<float>(x1 - x0) : 0.0f;
  }
  g.celly.resize(h);
  g.wy.resize(h);
  for (int y = 0; y < h; ++y) {
    const int c0 = std::min(y / stride, g.ncy - 2);
    const int y0 = g.gy[c0], y1 = g.gy[c0 + 1];
    g.celly[y] = c0;
    g.wy[y] = y1 > y0 ? static_cast<float>(y - y0) / static_cast<float>(y1 - y0) : 0.0f;
  }
  return g;
}

}  // namespace dgpu
