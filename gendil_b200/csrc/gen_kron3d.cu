// Instantiations of the 3D Kronecker-form kernel, N = 1..5, FP64 and FP32.
#include "kron3d_kernel.cuh"
#include "kron_registry.h"

namespace dgop {

namespace {
template <int N, typename Real>
void launch_kron3d(const KronParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  if (p.has_adv && p.has_mass && !p.mass_merged) kron3d_kernel<N, Real, true><<<grid, block, smem, s>>>(p);
  else kron3d_kernel<N, Real, false><<<grid, block, smem, s>>>(p);
}

template <int N, typename Real>
void fill(KronEntry<Real>& d) {
  d.launch = &launch_kron3d<N, Real>;
  d.func = reinterpret_cast<const void*>(&kron3d_kernel<N, Real, false>);
  d.func_sep = reinterpret_cast<const void*>(&kron3d_kernel<N, Real, true>);
  d.epw = Kron3DShape<N, Real>::EPW;
  d.warp_smem = Kron3DShape<N, Real>::WARP_SMEM;
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
