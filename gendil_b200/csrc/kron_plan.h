// Host planner interface for the Kronecker-form operator kernels.
#pragma once

#include "kron.h"

namespace dgop {

struct KronInputs {
  int D = 0, N = 0, Q = 0;
  bool gll = false;
  int flags = 0;
  const int64_t* sizes = nullptr;
  const double* h = nullptr;
  const double* B = nullptr;   // Q x N
  const double* Dq = nullptr;  // Q x Q
  const double* wq = nullptr;  // Q
  SepCoef sigma;
  SepCoef beta[kMaxDim];
  bool inverse_mass = false;  // plan the inverse of the (mass-only) operator
};

// Any dimension (dimension- and size-specific limits are the callers').
KronPlanHost plan_kron(const KronInputs& in);
// The 3D register kernel's plan: D = 3, N <= 4, fewer than 2^32 elements.
KronPlanHost plan_kron3d(const KronInputs& in);

}  // namespace dgop
