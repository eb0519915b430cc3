// Internal types of the stamp fit and the batched penalised-GLS solver.
#pragma once

#include "internal.h"

namespace dgpu {

struct StampGeom {
  int w = 0, h = 0;
  int sr = 0, S = 0, SS = 0;  // stamp radius, side 2sr+1, S*S
  int r = 0, ks = 0;          // kernel radius, side 2r+1
  int n_max = 0, nc = 0;
  int pmax = 0;               // max patch side S + 2r
  int have_var = 0, have_cvar = 0;
};

// Per-row buffers; N = n_stamps * SS rows in fixed per-stamp slots.
struct FitRows {
  uint8_t* valid = nullptr;
  double* t = nullptr;
  double* vt = nullptr;
  double* vc = nullptr;
  double* bn = nullptr;  // N x nc (float32 values from the stamp gather)
  int* px = nullptr;
  int* py = nullptr;
  double* d = nullptr;   // N x k design rows
  double* w = nullptr;   // IRLS weights
  int* stamp_used = nullptr;
};

void launch_stamp_gather(cudaStream_t st, const StampGeom& g, int n_stamps, const int* sx, const int* sy,
                         const float* sci, const float* ref, const float* vs, const float* vr,
                         const uint8_t* sm, const uint8_t* rm, const float* taps, const int2* orders,
                         const float* fill, const FitRows& R, const float* taps_y = nullptr);
void launch_design_weights(cudaStream_t st, int64_t N, const TpsDev& t, const FitRows& R, int have_var);
void launch_normal_equations(Context& c, int prec, int64_t N, int nc, int k, int SS, const FitRows& R,
                             const uint8_t* accepted, double* M);
// Mixed precision (BF16x3 tcgen05) Kronecker-packed normal equations:
// G[u][v] (row-major Mu x Nv, FP64) from per-split partials in gpart_slot.
void launch_normal_tc(Context& c, int64_t N, int nc, int k, int SS, const FitRows& R, const uint8_t* accepted,
                      const int2* upairs, int Mu, const int2* vpairs, int Nv, Slot gpart_slot, double* g, bool tf32 = false);
// rhs = X^T W t and ywy = t^T W t over the active rows; with theta, the same
// sums of the residual e = t - X theta (rhs = X^T W e, ywy = e^T W e).
void launch_rhs(Context& c, int64_t N, int nc, int k, int SS, const FitRows& R, const uint8_t* accepted,
                const double* theta, double* rhs, double* ywy, long long* n);
// scratch: stamp_chi2_scratch_bytes(n_stamps) of device memory (8-aligned).
size_t stamp_chi2_scratch_bytes(int n_stamps);
void launch_stamp_chi2(cudaStream_t st, int n_stamps, int nc, int k, int SS, const FitRows& R,
                       const uint8_t* accepted, const double* theta, double* chi2, int* cnt, void* scratch);
void launch_reweight(cudaStream_t st, const StampGeom& g, int n_stamps, const TpsDev& t, const int* sx,
                     const int* sy, const FitRows& R, const uint8_t* accepted, const int* cnt,
                     const double* theta, const float* phi, const float* vr, const uint8_t* rm);

// ---------------------------------------------------------------------------
// Batched penalised GLS: for each system s of a batch, A_s = M_s + lam_s P0
// (P0 = blockdiag of the k x k penalty), Cholesky A_s = L L^T,
// theta_s = A_s^{-1} rhs_s and edf_s = P - lam_s ||L^{-1} F||_F^2. One cluster
// launch, one thread-block cluster per system.
// ---------------------------------------------------------------------------
struct SolveBatch {
  int P = 0, k = 0, nf = 0, r = 0;  // unknowns, knots, fields, rank of the penalty
  int nsys = 0;
  const double* M = nullptr;        // nsys_m x P x P (system s uses M + m_index[s]*P*P)
  const int* m_index = nullptr;     // per system (nullptr -> 0)
  int nm = 1;                       // number of distinct M (m_index values 0 .. nm-1)
  const double* rhs = nullptr;      // per system rhs (rhs + r_index[s]*P)
  const int* r_index = nullptr;
  const double* lam = nullptr;      // nsys
  const double* pen = nullptr;      // k x k
  const double* fk = nullptr;       // k x r half factor of the penalty
  // solve_work_doubles workspace (tile-major): per system L's lower tiles,
  // the appended rows [rhs^T; F^T], the inverses of L's diagonal tiles; then
  // each distinct M converted to tiles.
  double* A = nullptr;
  double* theta = nullptr;          // nsys x P
  double* edf = nullptr;            // nsys
  int* ok = nullptr;                // nsys: 1 Cholesky, 2 LDLT fallback, 0 failed
  unsigned* status = nullptr;
  double* partial = nullptr;        // nsys x 8 per-rank trace partials
  // 1: leave systems whose Cholesky failed at ok = 0 (no LDLT fallback): a
  // reduced-precision attempt that will be redone in FP64 anyway.
  int skip_ldlt = 0;
};
int solve_pp(int P);                               // padded size
int solve_ep(int nf, int r);                       // appended rows, padded
size_t solve_sys_doubles(int P, int nf, int r);    // workspace per system
size_t solve_work_doubles(int P, int nf, int r, int nsys, int nm);
void launch_solve_batch(Context& c, const SolveBatch& b);
// Pivoted LDL^T redo of every system of the batch whose Cholesky failed
// (ok == 0): theta, edf = tr(A^+ M), ok = 2. Launched by launch_solve_batch.
void launch_ldlt_fallback(Context& c, const SolveBatch& b);
// X = (M + lam P0)^+ B by the same pivoted LDL^T, one CTA; B, X: P x m row-major.
void launch_sym_solve_many(Context& c, int P, int k, const double* M, double lam, const double* pen, const double* B,
                           int m, double* X);
// Apply a system's inverse: out = A_s^{-1} v (from the factor tiles of system s).
void launch_apply_inverse(cudaStream_t st, const SolveBatch& b, int s, const double* v, double* out);

}  // namespace dgpu
