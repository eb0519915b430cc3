/* C restatement of the reference's penalised GLS solve -- TEST INFRASTRUCTURE.
 *
 * The FP64 pieces of delta's kernel fit that dominate its CPU time, written
 * out in C with OpenMP so the timed CPU baseline runs the fit at the speed of
 * compiled code, as the reference's C++ does:
 *
 *   of_assemble   System assembly (src/solve.cpp:70-145): the pre-whitened
 *                 design rows Xs = sqrt(w) [d*bn_0 | ... | d*bn_{nc-1} | d],
 *                 M = Xs^T Xs as a symmetric rank update over row chunks (one
 *                 private P x P partial per thread, reduced at the end),
 *                 rhs = Xs^T (sqrt(w) t), ywy = sum w t^2.
 *   of_solve_grid solve_at for every lambda of a grid (src/solve.cpp:147-193,
 *                 227-262), lambdas in parallel: A = M + lambda P0; Cholesky
 *                 (LLT); theta; edf = P - lambda ||L^-1 F||_F^2 with
 *                 F F^T = P0; on a non-positive pivot the pivoted LDL^T
 *                 fallback with edf = tr(A^-1 M); rss and GCV.
 *   of_ldlt_solve the fallback factorisation alone (for the tests).
 *
 * Third-party arithmetic restated here: Eigen 3.4's LLT and LDLT
 * (un-vendored in the reference, pkg-config "eigen3 >= 3.4"). LLT fails when
 * an updated diagonal entry is <= 0 (a NaN does not fail, as in Eigen).
 * LDLT is Eigen's published algorithm: at step k the remaining diagonal entry
 * of largest magnitude (first on ties, taken before that step's update, i.e.
 * from the not yet updated diagonal) is swapped to position k, the left-
 * looking update gives d_k and column k of L, and the column is divided by
 * d_k only when d_k != 0. Its solve applies the transpositions, the unit lower
 * L, the pseudo-inverse of D (1/d where |d| > DBL_MIN, else 0), L^T and the
 * transpositions in reverse.
 *
 * Matrices are row-major, full symmetric storage.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

enum { kChunkRows = 128, kBI = 4, kBJ = 8 };

/* M (P x P, full), rhs (P), ywy from n design rows. Returns 0, or -1 on an
 * allocation failure. */
int of_assemble(int64_t n, int k, int nc, const double* design, const double* bn, const double* target,
                const double* weights, double* m, double* rhs, double* ywy) {
  const int p = (nc + 1) * k;
  const int pp = (p + kBJ - 1) / kBJ * kBJ; /* padded row length of a chunk */
  const int pb = (p + kBI - 1) / kBI * kBI;
  memset(m, 0, sizeof(double) * (size_t)p * p);
  memset(rhs, 0, sizeof(double) * (size_t)p);
  double y2 = 0.0;
  int fail = 0;
#pragma omp parallel reduction(+ : y2)
  {
    double* x = (double*)calloc((size_t)kChunkRows * pp, sizeof(double));
    double* ml = (double*)calloc((size_t)pb * pp, sizeof(double));
    double* rl = (double*)calloc((size_t)pp, sizeof(double));
    double ds[kChunkRows];
    const int ok = x && ml && rl;
    if (!ok) {
#pragma omp atomic write
      fail = 1;
    }
    /* every thread reaches the worksharing loop; one without buffers skips its chunks */
#pragma omp for schedule(dynamic)
      for (int64_t r0 = 0; r0 < n; r0 += kChunkRows) {
        if (!ok) continue;
        const int nr = (int)(n - r0 < kChunkRows ? n - r0 : kChunkRows);
        for (int r = 0; r < nr; ++r) {
          const int64_t row = r0 + r;
          const double sw = sqrt(weights[row]);
          const double* d = design + row * k;
          double* xr = x + (size_t)r * pp;
          for (int c = 0; c < nc; ++c) {
            const double s = bn[row * nc + c] * sw;
            for (int j = 0; j < k; ++j) xr[c * k + j] = d[j] * s;
          }
          for (int j = 0; j < k; ++j) xr[nc * k + j] = d[j] * sw;
          ds[r] = sw * target[row];
          y2 += weights[row] * target[row] * target[row];
        }
        for (int r = nr; r < kChunkRows; ++r) memset(x + (size_t)r * pp, 0, sizeof(double) * pp);
        /* lower-triangle blocks: rows i0..i0+3, columns j0..j0+7 with j0 <= i0+3 */
        for (int i0 = 0; i0 < p; i0 += kBI) {
          for (int j0 = 0; j0 < i0 + kBI && j0 < p; j0 += kBJ) {
            double acc[kBI][kBJ];
            memset(acc, 0, sizeof(acc));
            for (int r = 0; r < nr; ++r) {
              const double* xr = x + (size_t)r * pp;
              for (int a = 0; a < kBI; ++a) {
                const double xa = (i0 + a < pp) ? xr[i0 + a] : 0.0;
                for (int b = 0; b < kBJ; ++b) acc[a][b] += xa * xr[j0 + b];
              }
            }
            for (int a = 0; a < kBI; ++a)
              for (int b = 0; b < kBJ; ++b) ml[(size_t)(i0 + a) * pp + j0 + b] += acc[a][b];
          }
          for (int a = i0; a < i0 + kBI && a < p; ++a) {
            double s = 0.0;
            for (int r = 0; r < nr; ++r) s += x[(size_t)r * pp + a] * ds[r];
            rl[a] += s;
          }
        }
      }
    if (ok) {
#pragma omp critical
      {
        for (int i = 0; i < p; ++i) {
          for (int j = 0; j <= i; ++j) m[(size_t)i * p + j] += ml[(size_t)i * pp + j];
          rhs[i] += rl[i];
        }
      }
    }
    free(x);
    free(ml);
    free(rl);
  }
  if (fail) return -1;
  for (int i = 0; i < p; ++i)
    for (int j = i + 1; j < p; ++j) m[(size_t)i * p + j] = m[(size_t)j * p + i];
  *ywy = y2;
  return 0;
}

/* In-place Cholesky A = L L^T (lower triangle); 0 on success, -1 when an
 * updated diagonal entry is <= 0. */
static int llt(int p, double* a) {
  for (int j = 0; j < p; ++j) {
    double* aj = a + (size_t)j * p;
    double x = aj[j];
    for (int t = 0; t < j; ++t) x -= aj[t] * aj[t];
    if (x <= 0.0) return -1;
    x = sqrt(x);
    aj[j] = x;
    for (int i = j + 1; i < p; ++i) {
      double* ai = a + (size_t)i * p;
      double s = ai[j];
      for (int t = 0; t < j; ++t) s -= ai[t] * aj[t];
      ai[j] = s / x;
    }
  }
  return 0;
}

/* Solve L L^T x = b in place. */
static void llt_solve(int p, const double* l, double* x) {
  for (int i = 0; i < p; ++i) {
    double s = x[i];
    const double* li = l + (size_t)i * p;
    for (int t = 0; t < i; ++t) s -= li[t] * x[t];
    x[i] = s / li[i];
  }
  for (int i = p - 1; i >= 0; --i) {
    double s = x[i];
    for (int t = i + 1; t < p; ++t) s -= l[(size_t)t * p + i] * x[t];
    x[i] = s / l[(size_t)i * p + i];
  }
}

/* Pivoted LDL^T in place (Eigen's LDLT, see the header). a: full symmetric,
 * overwritten with L below the diagonal and D on it; perm: transpositions. */
static void ldlt(int p, double* a, int* perm, double* temp) {
  for (int k = 0; k < p; ++k) {
    int piv = k;
    double best = fabs(a[(size_t)k * p + k]);
    for (int i = k + 1; i < p; ++i) {
      const double v = fabs(a[(size_t)i * p + i]);
      if (v > best) {
        best = v;
        piv = i;
      }
    }
    if (k == 0 && best == 0.0) {
      /* the whole diagonal is zero: nothing to factor, identity transpositions */
      for (int j = 0; j < p; ++j) perm[j] = j;
      return;
    }
    perm[k] = piv;
    if (piv != k) {
      for (int j = 0; j < p; ++j) {
        const double t = a[(size_t)k * p + j];
        a[(size_t)k * p + j] = a[(size_t)piv * p + j];
        a[(size_t)piv * p + j] = t;
      }
      for (int i = 0; i < p; ++i) {
        const double t = a[(size_t)i * p + k];
        a[(size_t)i * p + k] = a[(size_t)i * p + piv];
        a[(size_t)i * p + piv] = t;
      }
    }
    double* ak = a + (size_t)k * p;
    for (int j = 0; j < k; ++j) temp[j] = a[(size_t)j * p + j] * ak[j];
    double dk = ak[k];
    for (int j = 0; j < k; ++j) dk -= ak[j] * temp[j];
    ak[k] = dk;
    for (int i = k + 1; i < p; ++i) {
      double* ai = a + (size_t)i * p;
      double s = ai[k];
      for (int j = 0; j < k; ++j) s -= ai[j] * temp[j];
      ai[k] = dk != 0.0 ? s / dk : s;
    }
  }
}

static void ldlt_solve(int p, const double* a, const int* perm, double* x) {
  for (int k = 0; k < p; ++k) {
    const double t = x[k];
    x[k] = x[perm[k]];
    x[perm[k]] = t;
  }
  for (int i = 0; i < p; ++i) {
    double s = x[i];
    const double* ai = a + (size_t)i * p;
    for (int t = 0; t < i; ++t) s -= ai[t] * x[t];
    x[i] = s;
  }
  for (int i = 0; i < p; ++i) {
    const double d = a[(size_t)i * p + i];
    x[i] = fabs(d) > DBL_MIN ? x[i] / d : 0.0;
  }
  for (int i = p - 1; i >= 0; --i) {
    double s = x[i];
    for (int t = i + 1; t < p; ++t) s -= a[(size_t)t * p + i] * x[t];
    x[i] = s;
  }
  for (int k = p - 1; k >= 0; --k) {
    const double t = x[k];
    x[k] = x[perm[k]];
    x[perm[k]] = t;
  }
}

/* x = LDLT(A)^-1 b for the tests: a is overwritten by the factor. */
int of_ldlt_solve(int p, double* a, const double* b, double* x) {
  int* perm = (int*)malloc(sizeof(int) * (size_t)p);
  double* temp = (double*)malloc(sizeof(double) * (size_t)(p > 0 ? p : 1));
  if (!perm || !temp) {
    free(perm);
    free(temp);
    return -1;
  }
  ldlt(p, a, perm, temp);
  memcpy(x, b, sizeof(double) * (size_t)p);
  ldlt_solve(p, a, perm, x);
  free(perm);
  free(temp);
  return 0;
}

/* solve_at over a lambda grid. m: P x P; p0: P x P penalty; f: P x nf
 * (F F^T = P0, nf may be 0). Per lambda i: theta[i*P..], edf, rss, gcv,
 * used_ldlt. Returns 0, or -1 on an allocation failure. */
int of_solve_grid(int p, const double* m, const double* p0, const double* rhs, double ywy, int64_t n,
                  const double* f, int nf, const double* lambdas, int n_lambda, double* theta, double* edf,
                  double* rss, double* gcv, int* used_ldlt) {
  int fail = 0;
#pragma omp parallel for schedule(dynamic)
  for (int li = 0; li < n_lambda; ++li) {
    const double lam = lambdas[li];
    double* a = (double*)malloc(sizeof(double) * (size_t)p * p);
    double* col = (double*)malloc(sizeof(double) * (size_t)p);
    int* perm = (int*)malloc(sizeof(int) * (size_t)p);
    if (!a || !col || !perm) {
#pragma omp atomic write
      fail = 1;
      free(a);
      free(col);
      free(perm);
      continue;
    }
    for (size_t i = 0; i < (size_t)p * p; ++i) a[i] = m[i] + lam * p0[i];
    double* th = theta + (size_t)li * p;
    memcpy(th, rhs, sizeof(double) * (size_t)p);
    double e = 0.0;
    if (llt(p, a) == 0) {
      used_ldlt[li] = 0;
      llt_solve(p, a, th);
      if (nf > 0) {
        double sq = 0.0;
        for (int c = 0; c < nf; ++c) {
          for (int i = 0; i < p; ++i) col[i] = f[(size_t)i * nf + c];
          for (int i = 0; i < p; ++i) {
            const double* ai = a + (size_t)i * p;
            double s = col[i];
            for (int t = 0; t < i; ++t) s -= ai[t] * col[t];
            col[i] = s / ai[i];
            sq += col[i] * col[i];
          }
        }
        e = (double)p - lam * sq;
      } else {
        for (int c = 0; c < p; ++c) {
          for (int i = 0; i < p; ++i) col[i] = m[(size_t)i * p + c];
          llt_solve(p, a, col);
          e += col[c];
        }
      }
    } else {
      used_ldlt[li] = 1;
      for (size_t i = 0; i < (size_t)p * p; ++i) a[i] = m[i] + lam * p0[i];
      ldlt(p, a, perm, col);
      ldlt_solve(p, a, perm, th);
      for (int c = 0; c < p; ++c) {
        for (int i = 0; i < p; ++i) col[i] = m[(size_t)i * p + c];
        ldlt_solve(p, a, perm, col);
        e += col[c];
      }
    }
    double tb = 0.0, tmt = 0.0;
    for (int i = 0; i < p; ++i) {
      tb += th[i] * rhs[i];
      double s = 0.0;
      const double* mi = m + (size_t)i * p;
      for (int j = 0; j < p; ++j) s += mi[j] * th[j];
      tmt += th[i] * s;
    }
    double r = ywy - 2.0 * tb + tmt;
    if (r < 0.0) r = 0.0;
    edf[li] = e;
    rss[li] = r;
    const double denom = (double)n - e;
    gcv[li] = denom > 0.0 ? (double)n * r / (denom * denom) : INFINITY;
    free(a);
    free(col);
    free(perm);
  }
  return fail ? -1 : 0;
}
