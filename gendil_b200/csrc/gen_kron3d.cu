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
template <int N, typename Real, int STAGES, bool SHFL>
void launch_kron3d(const KronParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  const bool sep = p.has_adv && p.has_mass && !p.mass_merged;
  if constexpr (std::is_same<Real, double>::value) {
    if (p.dot_partials) {
      if (sep) kron3d_kernel<N, Real, true, STAGES, SHFL, true><<<grid, block, smem, s>>>(p);
      else kron3d_kernel<N, Real, false, STAGES, SHFL, true><<<grid, block, smem, s>>>(p);
      return;
    }
  }
  if (sep) kron3d_kernel<N, Real, true, STAGES, SHFL><<<grid, block, smem, s>>>(p);
  else kron3d_kernel<N, Real, false, STAGES, SHFL><<<grid, block, smem, s>>>(p);
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
  v.warp_smem = Kron3DShape<N, Real>::warp_smem(STAGES, SHFL);
  v.threads = kKronThreads;
}

// The operator's element-dependent slots as a mask (bit k: slot k varies).
uint32_t vary_mask(const KronParams<double>& k) {
  uint32_t m = 0;
  for (int i = 0; i < kNumSlots; ++i)
    if (k.vary[i]) m |= 1u << i;
  return m;
}

// The one-stage tile variant (the fastest on the 3D p=3 workloads) is also compiled for the
// masks kVaryNone and kVarySheared; an operator whose mask is exactly one of them runs that
// kernel, every other operator the run-time-mask kernel (same arithmetic, same results).
template <bool SEP, int STAGES, bool SHFL, bool DOT>
void launch_tma_masked(const KronTmaParams<double>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) {
  if constexpr (STAGES == 1 && !SHFL) {
    const uint32_t m = vary_mask(p.k);
    if (m == kVaryNone) {
      kron3d_tma_kernel<SEP, STAGES, SHFL, DOT, kVaryNone><<<grid, block, smem, s>>>(p);
      return;
    }
    if (m == kVarySheared) {
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
    int k = 0;
    for (const void* f : {reinterpret_cast<const void*>(&kron3d_tma_kernel<false, 1, false, false, kVaryNone>),
                          reinterpret_cast<const void*>(&kron3d_tma_kernel<true, 1, false, false, kVaryNone>),
                          reinterpret_cast<const void*>(&kron3d_tma_kernel<false, 1, false, true, kVaryNone>),
                          reinterpret_cast<const void*>(&kron3d_tma_kernel<true, 1, false, true, kVaryNone>),
                          reinterpret_cast<const void*>(&kron3d_tma_kernel<false, 1, false, false, kVarySheared>),
                          reinterpret_cast<const void*>(&kron3d_tma_kernel<true, 1, false, false, kVarySheared>),
                          reinterpret_cast<const void*>(&kron3d_tma_kernel<false, 1, false, true, kVarySheared>),
                          reinterpret_cast<const void*>(&kron3d_tma_kernel<true, 1, false, true, kVarySheared>)})
      v.func_masked[k++] = f;
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
