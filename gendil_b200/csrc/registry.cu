// Kernel registry storage and the one-time registration of all instantiation units.
#include <mutex>

#include "kron_registry.h"
#include "registry.h"

namespace dgop {

namespace {
GenericEntry<double> g_f64[kMaxDim][kMaxN][kMaxQ];
GenericEntry<float> g_f32[kMaxDim][kMaxN][kMaxQ];
std::once_flag g_once;
KronEntry<double> g_k64[kKronMaxN + 1];
KronEntry<float> g_k32[kKronMaxN + 1];
KronNDEntry<double> g_n64[kMaxDim][kMaxN];
KronNDEntry<float> g_n32[kMaxDim][kMaxN];
}  // namespace

KronEntry<double>& kron3d_slot_f64(int N) { return g_k64[N]; }
KronEntry<float>& kron3d_slot_f32(int N) { return g_k32[N]; }
KronNDEntry<double>& kronnd_slot_f64(int D, int N) { return g_n64[D - 1][N - 1]; }
KronNDEntry<float>& kronnd_slot_f32(int D, int N) { return g_n32[D - 1][N - 1]; }

GenericEntry<double>& generic_slot_f64(int D, int N, int Q) { return g_f64[D - 1][N - 1][Q - 1]; }
GenericEntry<float>& generic_slot_f32(int D, int N, int Q) { return g_f32[D - 1][N - 1][Q - 1]; }

#define DGOP_DECL_N(D, N) void register_generic_d##D##_n##N();
#define DGOP_DECL_D(D) \
  DGOP_DECL_N(D, 1) DGOP_DECL_N(D, 2) DGOP_DECL_N(D, 3) DGOP_DECL_N(D, 4) \
  DGOP_DECL_N(D, 5) DGOP_DECL_N(D, 6) DGOP_DECL_N(D, 7) DGOP_DECL_N(D, 8)
DGOP_DECL_D(1) DGOP_DECL_D(2) DGOP_DECL_D(3) DGOP_DECL_D(4) DGOP_DECL_D(5) DGOP_DECL_D(6)
#undef DGOP_DECL_D
#undef DGOP_DECL_N

void ensure_registry() {
  std::call_once(g_once, [] {
#define DGOP_CALL_N(D, N) register_generic_d##D##_n##N();
#define DGOP_CALL_D(D) \
  DGOP_CALL_N(D, 1) DGOP_CALL_N(D, 2) DGOP_CALL_N(D, 3) DGOP_CALL_N(D, 4) \
  DGOP_CALL_N(D, 5) DGOP_CALL_N(D, 6) DGOP_CALL_N(D, 7) DGOP_CALL_N(D, 8)
    DGOP_CALL_D(1) DGOP_CALL_D(2) DGOP_CALL_D(3) DGOP_CALL_D(4) DGOP_CALL_D(5) DGOP_CALL_D(6)
    register_kron3d();
    register_kronnd_d1();
    register_kronnd_d2();
    register_kronnd_d3();
    register_kronnd_d4();
    register_kronnd_d5();
    register_kronnd_d6();
#undef DGOP_CALL_D
#undef DGOP_CALL_N
  });
}

const GenericEntry<double>* find_generic_f64(int D, int N, int Q) {
  if (D < 1 || D > kMaxDim || N < 1 || N > kMaxN || Q < 1 || Q > kMaxQ) return nullptr;
  const auto& e = g_f64[D - 1][N - 1][Q - 1];
  return e.launch ? &e : nullptr;
}

const GenericEntry<float>* find_generic_f32(int D, int N, int Q) {
  if (D < 1 || D > kMaxDim || N < 1 || N > kMaxN || Q < 1 || Q > kMaxQ) return nullptr;
  const auto& e = g_f32[D - 1][N - 1][Q - 1];
  return e.launch ? &e : nullptr;
}

}  // namespace dgop
