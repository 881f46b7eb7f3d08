// Instantiation unit of the any-dimension Kronecker kernel, compiled once per dimension with
// -DDGOP_GEN_D=<dim>: every N = 1..8 whose element (U, W, Y, matrices) fits in shared memory.
#include "kron_registry.h"
#include "kronnd_diff_grad_kernel.cuh"
#include "kronnd_diff_kernel.cuh"
#include "kronnd_kernel.cuh"
#include "kronnd_tc_kernel.cuh"

#ifndef DGOP_GEN_D
#error "DGOP_GEN_D must be defined"
#endif

#define DGOP_CAT2_(a, b) a##b
#define DGOP_CAT2(a, b) DGOP_CAT2_(a, b)

namespace dgop {

namespace {
template <int D, int N, typename Real>
void launch_kronnd(const KronNDParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  kronnd_kernel<D, N, Real><<<grid, block, smem, s>>>(p);
}

template <int D, int N, int G, typename Real>
void launch_kronnd_grouped(const KronNDParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  kronnd_grouped_kernel<D, N, G, Real><<<grid, block, smem, s>>>(p);
}

template <int D, int N>
void launch_kronnd_tc(const KronNDParams<float>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  kronnd_tc_kernel<D, N><<<grid, block, smem, s>>>(p);
}

template <int D, int N, int V, typename Real>
void launch_kronnd_batch(const KronNDParams<Real>* table, const int64_t* first, int count, int eb, dim3 grid,
                         dim3 block, size_t smem, cudaStream_t s) {
  kronnd_batch_kernel<D, N, V, Real><<<grid, block, smem, s>>>(table, first, count, eb);
}

// blocks of 3 axes for the mass-only kernel while they stay 27 values, else 2
template <int N>
constexpr int mass_groups() {
  return N * N * N <= 27 ? 3 : 2;
}

template <int D, int N, typename Real>
void launch_kronnd_mass(const KronNDParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  kronnd_mass_kernel<D, N, mass_groups<N>(), Real><<<grid, block, smem, s>>>(p);
}

template <int D, int N, typename Real>
void launch_kronnd_paired(const KronNDParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  kronnd_paired_kernel<D, N, Real><<<grid, block, smem, s>>>(p);
}

template <int D, int N, typename Real>
void launch_kronnd_diff(const KronDiffParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  kronnd_diff_kernel<D, N, Real><<<grid, block, smem, s>>>(p);
}

template <int D, int N, typename Real>
void launch_kronnd_grad(const KronDiffParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  kronnd_diff_grad_kernel<D, N, Real><<<grid, block, smem, s>>>(p);
}

// one element must fit in 200 KB of shared memory
template <int D, int N, typename Real>
constexpr bool fits() {
  return (int64_t)KronNDShape<D, N>::PER_ELEM * (int64_t)sizeof(Real) <= 200 * 1024;
}

template <int D, int N, typename Real>
void fill(KronNDEntry<Real>& d) {
  if constexpr (fits<D, N, Real>()) {
    d.launch = &launch_kronnd<D, N, Real>;
    d.func = reinterpret_cast<const void*>(&kronnd_kernel<D, N, Real>);
    d.launch_batch[0] = &launch_kronnd_batch<D, N, 0, Real>;
    d.func_batch[0] = reinterpret_cast<const void*>(&kronnd_batch_kernel<D, N, 0, Real>);
    d.per_elem = KronNDShape<D, N>::PER_ELEM;
    // grouped variants while a block (N^G values) stays a register array (blocks of 2 axes up to
    // N = 6: the 2D p = 5 systems, among the slowest to solve, need them most)
    if constexpr (D >= 2 && N >= 2 && N * N <= 36) {
      d.launch_g[0] = &launch_kronnd_grouped<D, N, 2, Real>;
      d.func_g[0] = reinterpret_cast<const void*>(&kronnd_grouped_kernel<D, N, 2, Real>);
      d.launch_m = &launch_kronnd_mass<D, N, Real>;
      d.func_m = reinterpret_cast<const void*>(&kronnd_mass_kernel<D, N, mass_groups<N>(), Real>);
      d.per_elem_m = KronNDMassShape<D, N>::PER_ELEM;
      d.mass_g = mass_groups<N>();
      if constexpr (sizeof(Real) == 8 && N * N <= 27) {
        // (36-value blocks stay single-operator launches: the persistent batch kernel needs about
        // 170 FP64 registers for them, past the 128-register cap that keeps two CTAs per SM)
        d.launch_batch[1] = &launch_kronnd_batch<D, N, 1, Real>;
        d.func_batch[1] = reinterpret_cast<const void*>(&kronnd_batch_kernel<D, N, 1, Real>);
      }
    }
    if constexpr (D % 2 == 0 && N >= 2 && N * N <= 27) {
      d.launch_g[2] = &launch_kronnd_paired<D, N, Real>;
      d.func_g[2] = reinterpret_cast<const void*>(&kronnd_paired_kernel<D, N, Real>);
      if constexpr (sizeof(Real) == 8) {
        d.launch_batch[3] = &launch_kronnd_batch<D, N, 3, Real>;
        d.func_batch[3] = reinterpret_cast<const void*>(&kronnd_batch_kernel<D, N, 3, Real>);
      }
    }
    if constexpr (sizeof(Real) == 4 && KronTCShape<D, N>::OK && KronTCShape<D, N>::WARP_BYTES * 4 <= 200 * 1024) {
      d.launch_tc = &launch_kronnd_tc<D, N>;
      d.func_tc = reinterpret_cast<const void*>(&kronnd_tc_kernel<D, N>);
      d.tc_warp_bytes = KronTCShape<D, N>::WARP_BYTES;
    }
    if constexpr (D >= 3 && N >= 2 && N * N * N <= 27) {
      d.launch_g[1] = &launch_kronnd_grouped<D, N, 3, Real>;
      d.func_g[1] = reinterpret_cast<const void*>(&kronnd_grouped_kernel<D, N, 3, Real>);
      if constexpr (sizeof(Real) == 8) {
        d.launch_batch[2] = &launch_kronnd_batch<D, N, 2, Real>;
        d.func_batch[2] = reinterpret_cast<const void*>(&kronnd_batch_kernel<D, N, 2, Real>);
      }
    }
  }
  if constexpr ((int64_t)(KronDiffShape<D, N>::PER_ELEM + KronDiffShape<D, N>::HDR) * (int64_t)sizeof(Real) <=
                200 * 1024) {
    d.launch_diff = &launch_kronnd_diff<D, N, Real>;
    d.func_diff = reinterpret_cast<const void*>(&kronnd_diff_kernel<D, N, Real>);
    d.per_elem_diff = KronDiffShape<D, N>::PER_ELEM;
    d.header_diff = KronDiffShape<D, N>::HDR;
  }
  if constexpr (sizeof(Real) == 8 &&
                (int64_t)(KronDiffGradShape<D, N>::PER_ELEM + KronDiffGradShape<D, N>::HDR) * (int64_t)sizeof(Real) <=
                    200 * 1024) {
    d.launch_grad = &launch_kronnd_grad<D, N, Real>;
    d.func_grad = reinterpret_cast<const void*>(&kronnd_diff_grad_kernel<D, N, Real>);
    d.per_elem_grad = KronDiffGradShape<D, N>::PER_ELEM;
    d.header_grad = KronDiffGradShape<D, N>::HDR;
  }
}
}  // namespace

void DGOP_CAT2(register_kronnd_d, DGOP_GEN_D)() {
  constexpr int D = DGOP_GEN_D;
  static_for<1, kMaxN + 1>([&](auto nc) {
    constexpr int N = decltype(nc)::value;
    fill<D, N, double>(kronnd_slot_f64(D, N));
    fill<D, N, float>(kronnd_slot_f32(D, N));
  });
}

}  // namespace dgop
