// Instantiations of the 3D Kronecker-form kernel, N = 1..5, FP64 and FP32, every variant.
#include "kron3d_kernel.cuh"
#include "kron_registry.h"

namespace dgop {

const char* const kKronVariantNames[kKronVariants] = {"stage2-tile", "stage1-tile", "stage2-shfl"};
// (the any-dimension kernel's variants, kronnd_kernel.cuh, named here with the 3D kernel's)
const char* const kKronNDVariantNames[kKronNDVariants] = {"nd-passes", "nd-grouped2", "nd-grouped3"};

namespace {
template <int N, typename Real, int STAGES, bool SHFL>
void launch_kron3d(const KronParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  if (p.has_adv && p.has_mass && !p.mass_merged) kron3d_kernel<N, Real, true, STAGES, SHFL><<<grid, block, smem, s>>>(p);
  else kron3d_kernel<N, Real, false, STAGES, SHFL><<<grid, block, smem, s>>>(p);
}

template <int N, typename Real, int STAGES, bool SHFL>
void fill_variant(KronVariant<Real>& v) {
  v.launch = &launch_kron3d<N, Real, STAGES, SHFL>;
  v.func = reinterpret_cast<const void*>(&kron3d_kernel<N, Real, false, STAGES, SHFL>);
  v.func_sep = reinterpret_cast<const void*>(&kron3d_kernel<N, Real, true, STAGES, SHFL>);
  v.warp_smem = Kron3DShape<N, Real>::warp_smem(STAGES, SHFL);
}

template <int N, typename Real>
void fill(KronEntry<Real>& d) {
  d.epw = Kron3DShape<N, Real>::EPW;
  fill_variant<N, Real, 2, false>(d.v[0]);
  fill_variant<N, Real, 1, false>(d.v[1]);
  if constexpr (Kron3DShape<N, Real>::BUTTERFLY) fill_variant<N, Real, 2, true>(d.v[2]);
}

template <int N>
void reg_one() {
  fill<N, double>(kron3d_slot_f64(N));
  fill<N, float>(kron3d_slot_f32(N));
}
}  // namespace

void register_kron3d() {
  reg_one<1>();
  reg_one<2>();
  reg_one<3>();
  reg_one<4>();
  reg_one<5>();
}

}  // namespace dgop
