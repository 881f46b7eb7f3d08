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
};

KronPlanHost plan_kron3d(const KronInputs& in);

}  // namespace dgop
