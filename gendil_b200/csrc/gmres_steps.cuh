// Scalar steps of restarted GMRES(m) (Solvers/gmres.hpp:74-289) on one system's device state,
// shared by the single-system solvers (krylov.cu) and the batched multi-system solver
// (batch_solve.cu): the caller reduces the inner product the step needs (R) and calls the step
// from one thread.
#pragma once

#include <cfloat>
#include <cmath>

namespace dgop {

struct GMState {
  int done, success, iters, total, k, brk, inactive, max_iters;
  double denom, beta, rel, inv_h, tol;
};

// |b| -> the denominator of every relative residual (gmres.hpp:113-115); state reset
__device__ __forceinline__ void gm_denom(GMState* st, double R, double tol, int max_iters) {
  st->tol = tol;
  st->max_iters = max_iters;
  const double norm_rhs = sqrt(R);
  st->denom = norm_rhs > 0.0 ? norm_rhs : 1.0;
  st->done = 0;
  st->success = 0;
  st->iters = 0;
  st->total = 0;
  st->k = 0;
  st->brk = 0;
  st->inactive = 0;
}

// true residual |b - A x| / denom and the decisions taken after it (gmres.hpp:117-123, 230-236, 269-280)
// phase 0: initial; 1: end of a cycle; 2: residual-only solve (no iterations allowed)
__device__ __forceinline__ void gm_resid(GMState* st, double R, int phase) {
  const double tol = st->tol;
  const int max_iters = st->max_iters;
  const double beta = sqrt(R);
  const double rel = beta / st->denom;
  st->beta = beta;
  st->rel = rel;
  if (phase == 2 || (phase == 1 && st->k == 0)) {
    st->success = rel <= tol;
    st->iters = st->total;
    st->done = 1;
    return;
  }
  if (rel <= tol) {
    st->success = 1;
    st->iters = st->total;
    st->done = 1;
    return;
  }
  if (phase == 1 && st->total >= max_iters) {
    st->success = 0;
    st->iters = st->total;
    st->done = 1;
  }
}

// start of a cycle: reset the rotations and the reduced right-hand side (gmres.hpp:132-146)
__device__ __forceinline__ void gm_cycle_start(GMState* st, double* cs, double* sn, double* e1, double* y, int m) {
  if (st->done) {
    st->inactive = 1;
    return;
  }
  for (int i = 0; i < m; ++i) {
    cs[i] = 1.0;
    sn[i] = 0.0;
    y[i] = 0.0;
  }
  for (int i = 0; i <= m; ++i) e1[i] = 0.0;
  e1[0] = st->beta;
  st->k = 0;
  st->brk = 0;
  st->inactive = st->total >= st->max_iters;
  st->inv_h = 1.0 / st->beta;
}

// Hessenberg column j from R = |w|^2 after the projections: norm, previous rotations, new
// rotation, stopping tests (gmres.hpp:167-222)
__device__ __forceinline__ void gm_column(GMState* st, int j, int m, double* H, double* cs, double* sn, double* e1,
                                          double R) {
  const double tol = st->tol;
  const int max_iters = st->max_iters;
  const double eps = DBL_EPSILON;
  const double beta = st->beta;
  st->total += 1;
#define HH(a, b) H[(b) * (m + 1) + (a)]
  const double h_next = sqrt(R);
  HH(j + 1, j) = h_next;
  for (int i = 0; i < j; ++i) {
    const double h_im = HH(i, j), h_ip = HH(i + 1, j);
    HH(i, j) = cs[i] * h_im + sn[i] * h_ip;
    HH(i + 1, j) = -sn[i] * h_im + cs[i] * h_ip;
  }
  const double h_mm = HH(j, j), h_m1m = HH(j + 1, j);
  const double rho = sqrt(h_mm * h_mm + h_m1m * h_m1m);
  if (rho <= eps * beta) {
    HH(j, j) = 0.0;
    HH(j + 1, j) = 0.0;
    st->k = j;
    st->brk = 1;
    st->inactive = 1;
    return;
  }
  cs[j] = h_mm / rho;
  sn[j] = h_m1m / rho;
  HH(j, j) = rho;
  HH(j + 1, j) = 0.0;
  const double g_m = e1[j], g_m1 = e1[j + 1];
  e1[j] = cs[j] * g_m + sn[j] * g_m1;
  e1[j + 1] = -sn[j] * g_m + cs[j] * g_m1;
  st->k = j + 1;
  const double rel_est = fabs(e1[j + 1]) / st->denom;
  const bool happy = h_next <= eps * beta;
  if (happy || rel_est <= tol) {
    st->brk = 1;
    st->inactive = 1;
    return;
  }
  st->inv_h = 1.0 / h_next;
  if (st->total >= max_iters || j + 1 >= m) st->inactive = 1;
#undef HH
}

// back-substitution in the k x k triangle (gmres.hpp:238-261)
__device__ __forceinline__ void gm_backsub(const GMState* st, const double* H, const double* e1, double* y, int m) {
  if (st->done || st->k == 0) return;
  const double eps = DBL_EPSILON, beta = st->beta;
  const int k = st->k;
  for (int i = k; i-- > 0;) {
    double sum = e1[i];
    for (int j = i + 1; j < k; ++j) sum -= H[j * (m + 1) + i] * y[j];
    const double diag = H[i * (m + 1) + i];
    y[i] = fabs(diag) <= eps * beta ? 0.0 : sum / diag;
  }
}

}  // namespace dgop
