// Instantiation unit of the generic element kernel.  Compiled once per (dimension, N) pair with
// -DDGOP_GEN_D=<dim> -DDGOP_GEN_N=<p+1>; registers every enabled quadrature size Q.
#include "registry_impl.cuh"

#ifndef DGOP_GEN_D
#error "DGOP_GEN_D must be defined"
#endif
#ifndef DGOP_GEN_N
#error "DGOP_GEN_N must be defined"
#endif

#define DGOP_CAT_(a, b, c, d) a##b##c##d
#define DGOP_CAT(a, b, c, d) DGOP_CAT_(a, b, c, d)

namespace dgop {

void DGOP_CAT(register_generic_d, DGOP_GEN_D, _n, DGOP_GEN_N)() {
  constexpr int D = DGOP_GEN_D, N = DGOP_GEN_N;
  static_for<1, kMaxQ + 1>([&](auto qc) {
    constexpr int Q = decltype(qc)::value;
    if constexpr (generic_enabled(D, N, Q)) register_generic<D, N, Q>();
  });
}

}  // namespace dgop
