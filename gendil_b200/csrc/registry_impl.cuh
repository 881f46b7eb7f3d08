// Helpers for the per-dimension instantiation units (gen_generic_d*.cu).
#pragma once

#include "generic_kernel.cuh"
#include "registry.h"

namespace dgop {

// Which (D, N, Q) are compiled.  Full build: every Q for D <= 3, Q in [N-1, N+2] above (the
// reference's tests and benchmarks use q = p+1 .. p+3).  DGOP_FAST_BUILD compiles only the
// shapes the test-suite and the benchmark workloads use.
constexpr bool generic_enabled(int D, int N, int Q) {
#ifdef DGOP_FAST_BUILD
  constexpr int list[][3] = {
      {1, 1, 1}, {1, 4, 5}, {1, 8, 8}, {1, 3, 4}, {2, 1, 1}, {2, 3, 4}, {2, 5, 3}, {2, 3, 3}, {2, 2, 2},
      {3, 2, 4}, {3, 4, 4}, {3, 4, 6}, {3, 3, 2}, {3, 8, 8}, {3, 1, 2}, {3, 2, 3}, {3, 6, 6}, {3, 3, 3},
      {3, 2, 2}, {3, 5, 5}, {3, 4, 3},
      {4, 3, 3}, {4, 2, 2}, {5, 2, 2}, {6, 2, 2}, {6, 3, 3}};
  for (const auto& c : list)
    if (c[0] == D && c[1] == N && c[2] == Q) return true;
  return false;
#else
  if (D <= 3) return true;
  return Q >= N - 1 && Q <= N + 2;
#endif
}

GenericEntry<double>& generic_slot_f64(int D, int N, int Q);
GenericEntry<float>& generic_slot_f32(int D, int N, int Q);

template <int D, int N, int Q, typename Real>
void launch_generic(const OpParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  generic_kernel<D, N, Q, Real><<<grid, block, smem, s>>>(p);
}

template <int D, int N, int Q, typename Real>
void register_generic_one(GenericEntry<Real>& e) {
  e.launch = &launch_generic<D, N, Q, Real>;
  e.func = reinterpret_cast<const void*>(&generic_kernel<D, N, Q, Real>);
  e.per_elem = GenericShape<D, N, Q>::PER_ELEM;
  e.mats = GenericShape<D, N, Q>::MATS;
}

template <int D, int N, int Q>
void register_generic() {
  register_generic_one<D, N, Q, double>(generic_slot_f64(D, N, Q));
#ifndef DGOP_NO_F32
  register_generic_one<D, N, Q, float>(generic_slot_f32(D, N, Q));
#endif
}

}  // namespace dgop

// Every (N, Q) pair with N = p + 1 in 1..8 and Q in 1..8.
#define DGOP_NQ_ROW(R, N) R(N, 1) R(N, 2) R(N, 3) R(N, 4) R(N, 5) R(N, 6) R(N, 7) R(N, 8)
#define DGOP_NQ_ALL(R) \
  DGOP_NQ_ROW(R, 1) DGOP_NQ_ROW(R, 2) DGOP_NQ_ROW(R, 3) DGOP_NQ_ROW(R, 4) \
  DGOP_NQ_ROW(R, 5) DGOP_NQ_ROW(R, 6) DGOP_NQ_ROW(R, 7) DGOP_NQ_ROW(R, 8)
