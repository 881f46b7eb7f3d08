// Instantiations of the 3D Kronecker-form kernel, N = 1..5, FP64 and FP32, every variant.
#include "kron3d_kernel.cuh"
#include "kron3d_tma_kernel.cuh"
#include "kron_registry.h"

#include <type_traits>

namespace dgop {

const char* const kKronVariantNames[kKronVariants] = {"stage2-tile", "stage1-tile", "stage2-shfl",
                                                      "tma1-tile",   "tma2-shfl",   "tma2-tile"};
// (the any-dimension kernel's variants, kronnd_kernel.cuh, named here with the 3D kernel's)
const char* const kKronNDVariantNames[kKronNDVariants] = {"nd-passes", "nd-grouped2", "nd-grouped3", "nd-paired",
                                                          "nd-mass"};

namespace {
// The one-stage tile variant at N = 4 (p = 3) is also compiled for the masks kVaryNone and
// kVarySheared; an operator whose mask is exactly one of them runs that kernel, every other
// operator the run-time-mask kernel (same arithmetic, same results).
template <int N, typename Real, bool SEP, int STAGES, bool SHFL, bool DOT>
void launch_kron3d_masked(const KronParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  if constexpr (N == 4 && STAGES == 1 && !SHFL) {
    const int mi = kron_mask_index(p);
    if constexpr (std::is_same<Real, double>::value && !SEP) {
      if (mi == 0) {
        kron3d_kernel_capped<N, STAGES, SHFL, DOT, kVaryNone><<<grid, block, smem, s>>>(p);
        return;
      }
      if (mi == 1) {
        kron3d_kernel_capped<N, STAGES, SHFL, DOT, kVarySheared><<<grid, block, smem, s>>>(p);
        return;
      }
    } else {
      if (mi == 0) {
        kron3d_kernel<N, Real, SEP, STAGES, SHFL, DOT, kVaryNone><<<grid, block, smem, s>>>(p);
        return;
      }
      if (mi == 1) {
        kron3d_kernel<N, Real, SEP, STAGES, SHFL, DOT, kVarySheared><<<grid, block, smem, s>>>(p);
        return;
      }
    }
  }
  kron3d_kernel<N, Real, SEP, STAGES, SHFL, DOT><<<grid, block, smem, s>>>(p);
}

template <int N, typename Real, int STAGES, bool SHFL>
void launch_kron3d(const KronParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  const bool sep = p.has_adv && p.has_mass && !p.mass_merged;
  if constexpr (std::is_same<Real, double>::value) {
    if (p.dot_partials) {
      if (sep) launch_kron3d_masked<N, Real, true, STAGES, SHFL, true>(p, grid, block, smem, s);
      else launch_kron3d_masked<N, Real, false, STAGES, SHFL, true>(p, grid, block, smem, s);
      return;
    }
  }
  if (sep) launch_kron3d_masked<N, Real, true, STAGES, SHFL, false>(p, grid, block, smem, s);
  else launch_kron3d_masked<N, Real, false, STAGES, SHFL, false>(p, grid, block, smem, s);
}

template <int N, typename Real, int STAGES, bool SHFL>
void fill_variant(KronVariant<Real>& v) {
  v.launch = &launch_kron3d<N, Real, STAGES, SHFL>;
  v.func = reinterpret_cast<const void*>(&kron3d_kernel<N, Real, false, STAGES, SHFL>);
  v.func_sep = reinterpret_cast<const void*>(&kron3d_kernel<N, Real, true, STAGES, SHFL>);
  if constexpr (std::is_same<Real, double>::value) {
    v.func_dot[0] = reinterpret_cast<const void*>(&kron3d_kernel<N, Real, false, STAGES, SHFL, true>);
    v.func_dot[1] = reinterpret_cast<const void*>(&kron3d_kernel<N, Real, true, STAGES, SHFL, true>);
  }
  if constexpr (N == 4 && STAGES == 1 && !SHFL) {
    v.func_masked[0][0][1] = reinterpret_cast<const void*>(&kron3d_kernel<N, Real, true, 1, false, false, kVaryNone>);
    v.func_masked[1][0][1] = reinterpret_cast<const void*>(&kron3d_kernel<N, Real, true, 1, false, false, kVarySheared>);
    if constexpr (std::is_same<Real, double>::value) {
      v.func_masked[0][0][0] = reinterpret_cast<const void*>(&kron3d_kernel_capped<N, 1, false, false, kVaryNone>);
      v.func_masked[1][0][0] = reinterpret_cast<const void*>(&kron3d_kernel_capped<N, 1, false, false, kVarySheared>);
      v.func_masked[0][1][0] = reinterpret_cast<const void*>(&kron3d_kernel_capped<N, 1, false, true, kVaryNone>);
      v.func_masked[1][1][0] = reinterpret_cast<const void*>(&kron3d_kernel_capped<N, 1, false, true, kVarySheared>);
      v.func_masked[0][1][1] = reinterpret_cast<const void*>(&kron3d_kernel<N, Real, true, 1, false, true, kVaryNone>);
      v.func_masked[1][1][1] =
          reinterpret_cast<const void*>(&kron3d_kernel<N, Real, true, 1, false, true, kVarySheared>);
    } else {
      v.func_masked[0][0][0] = reinterpret_cast<const void*>(&kron3d_kernel<N, Real, false, 1, false, false, kVaryNone>);
      v.func_masked[1][0][0] =
          reinterpret_cast<const void*>(&kron3d_kernel<N, Real, false, 1, false, false, kVarySheared>);
    }
  }
  v.warp_smem = Kron3DShape<N, Real>::warp_smem(STAGES, SHFL);
  v.threads = kKronThreads;
}

// The one-stage tile variant (the fastest on the 3D p=3 workloads) is also compiled for the
// masks kVaryNone and kVarySheared (kron.h); an operator whose mask is exactly one of them runs
// that kernel, every other operator the run-time-mask kernel (same arithmetic, same results).
template <bool SEP, int STAGES, bool SHFL, bool DOT>
void launch_tma_masked(const KronTmaParams<double>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  if constexpr (STAGES == 1 && !SHFL) {
    const int mi = kron_mask_index(p.k);
    if (mi == 0) {
      kron3d_tma_kernel<SEP, STAGES, SHFL, DOT, kVaryNone><<<grid, block, smem, s>>>(p);
      return;
    }
    if (mi == 1) {
      kron3d_tma_kernel<SEP, STAGES, SHFL, DOT, kVarySheared><<<grid, block, smem, s>>>(p);
      return;
    }
  }
  kron3d_tma_kernel<SEP, STAGES, SHFL, DOT><<<grid, block, smem, s>>>(p);
}

template <int STAGES, bool SHFL>
void launch_tma(const KronTmaParams<double>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  const bool sep = p.k.has_adv && p.k.has_mass && !p.k.mass_merged;
  if (p.k.dot_partials) {
    if (sep) launch_tma_masked<true, STAGES, SHFL, true>(p, grid, block, smem, s);
    else launch_tma_masked<false, STAGES, SHFL, true>(p, grid, block, smem, s);
  } else {
    if (sep) launch_tma_masked<true, STAGES, SHFL, false>(p, grid, block, smem, s);
    else launch_tma_masked<false, STAGES, SHFL, false>(p, grid, block, smem, s);
  }
}

template <int STAGES, bool SHFL>
void fill_tma(KronVariant<double>& v) {
  v.launch_tma = &launch_tma<STAGES, SHFL>;
  v.func = reinterpret_cast<const void*>(&kron3d_tma_kernel<false, STAGES, SHFL>);
  v.func_sep = reinterpret_cast<const void*>(&kron3d_tma_kernel<true, STAGES, SHFL>);
  v.func_dot[0] = reinterpret_cast<const void*>(&kron3d_tma_kernel<false, STAGES, SHFL, true>);
  v.func_dot[1] = reinterpret_cast<const void*>(&kron3d_tma_kernel<true, STAGES, SHFL, true>);
  if constexpr (STAGES == 1 && !SHFL) {
    v.func_masked[0][0][0] = reinterpret_cast<const void*>(&kron3d_tma_kernel<false, 1, false, false, kVaryNone>);
    v.func_masked[0][0][1] = reinterpret_cast<const void*>(&kron3d_tma_kernel<true, 1, false, false, kVaryNone>);
    v.func_masked[0][1][0] = reinterpret_cast<const void*>(&kron3d_tma_kernel<false, 1, false, true, kVaryNone>);
    v.func_masked[0][1][1] = reinterpret_cast<const void*>(&kron3d_tma_kernel<true, 1, false, true, kVaryNone>);
    v.func_masked[1][0][0] = reinterpret_cast<const void*>(&kron3d_tma_kernel<false, 1, false, false, kVarySheared>);
    v.func_masked[1][0][1] = reinterpret_cast<const void*>(&kron3d_tma_kernel<true, 1, false, false, kVarySheared>);
    v.func_masked[1][1][0] = reinterpret_cast<const void*>(&kron3d_tma_kernel<false, 1, false, true, kVarySheared>);
    v.func_masked[1][1][1] = reinterpret_cast<const void*>(&kron3d_tma_kernel<true, 1, false, true, kVarySheared>);
  }
  v.warp_smem = kTmaWarps * tma_warp_bytes(STAGES, SHFL) + 1024;  // bytes per CTA, with the alignment slack
  v.threads = kTmaWarps * 32;
}

template <typename Real>
void face_words(const KronParams<Real>& p, uint32_t* eflags, uint32_t* gwords, cudaStream_t s) {
  const int64_t groups = (p.nelem + 7) / 8;
  const int64_t blocks = (groups * 32 + 255) / 256;
  kron_face_words<Real><<<(unsigned)blocks, 256, 0, s>>>(p, eflags, gwords);
}

template <int N, typename Real>
void fill(KronEntry<Real>& d) {
  d.epw = Kron3DShape<N, Real>::EPW;
  fill_variant<N, Real, 2, false>(d.v[0]);
  fill_variant<N, Real, 1, false>(d.v[1]);
  if constexpr (Kron3DShape<N, Real>::BUTTERFLY) fill_variant<N, Real, 2, true>(d.v[2]);
  if constexpr (N == 4 && std::is_same<Real, double>::value) {
    fill_tma<1, false>(d.v[3]);
    fill_tma<2, true>(d.v[4]);
    fill_tma<2, false>(d.v[5]);
    d.face_words = &face_words<Real>;
  }
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
