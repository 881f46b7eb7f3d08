// Registry of the Kronecker-form kernels.
#pragma once

#include <cuda_runtime.h>

#include "kron.h"

namespace dgop {

constexpr int kKronThreads = 128;
constexpr int kKronNDThreads = 256;  // threads per CTA of the any-dimension kernel
constexpr int kKronTCThreads = 128;  // tensor-core variant: four warps (elements) per CTA

// Kernel variants of one (N, precision); the autotuner picks one per operator.
//   0: two staging stages, exchanges through the shared tile
//   1: one staging stage (more warps per SM), exchanges through the shared tile
//   2: two staging stages, exchanges by shuffle butterflies (even N only)
//   3-5: element groups moved by the Tensor Memory Accelerator (kron3d_tma_kernel.cuh; N = 4,
//        FP64, x extent a multiple of 8): one stage + tile, two stages + shuffles, two stages + tile
constexpr int kKronVariants = 6;
extern const char* const kKronVariantNames[kKronVariants];

template <typename Real>
struct KronTmaParams;

template <typename Real>
struct KronVariant {
  void (*launch)(const KronParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) = nullptr;
  // bulk-tensor variants take the tensor maps and face words as well
  void (*launch_tma)(const KronTmaParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) = nullptr;
  const void* func = nullptr;      // kernel symbol (mass merged or absent)
  const void* func_sep = nullptr;  // kernel symbol with a separate mass term
  const void* func_dot[2] = {};    // with the inner-product epilogue (mass merged / separate; FP64)
  // compile-time slot-mask forms of the above (one-stage tile variants): [mask index, kron.h]
  // [with the inner-product epilogue][separate mass term]
  const void* func_masked[2][2][2] = {};
  int warp_smem = 0;               // Real values of shared memory per warp (bytes per CTA for bulk-tensor variants)
  int threads = 0;                 // threads per CTA
};

template <typename Real>
struct KronEntry {
  int epw = 0;  // elements per warp group
  KronVariant<Real> v[kKronVariants];
  // per-element face words / per-group slot words of the bulk-tensor variants
  void (*face_words)(const KronParams<Real>& p, uint32_t* eflags, uint32_t* gwords, cudaStream_t s) = nullptr;
};

KronEntry<double>& kron3d_slot_f64(int N);
KronEntry<float>& kron3d_slot_f32(int N);
void register_kron3d();

// Kronecker form, any dimension, shared-memory kernel (kronnd_kernel.cuh).  Variants (the
// autotuner picks one per operator): 0 one shared-memory pass per axis; 1, 2 groups of 2 or 3
// axes per pass in registers; 3 axes a and a + D/2 paired, the two terms of a pair run together
// (even D, operators whose term pairs share their other factors); 4 operators without advection
// terms (mass, mass inverse): groups of 2 axes passed in place, a third of the shared memory.
constexpr int kKronNDVariants = 5;
extern const char* const kKronNDVariantNames[kKronNDVariants];

template <typename Real>
struct KronNDEntry {
  void (*launch)(const KronNDParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) = nullptr;
  const void* func = nullptr;
  // many operators of this (D, N) in one launch (dgop_batch_apply), per variant
  void (*launch_batch[kKronNDVariants])(const KronNDParams<Real>* table, const int64_t* first, int count, int eb,
                                        dim3 grid, dim3 block, size_t smem, cudaStream_t s) = {};
  const void* func_batch[kKronNDVariants] = {};
  int per_elem = 0;  // Real values of shared memory per element
  // grouped variants (kronnd_grouped_kernel), groups of 2 and 3 axes, and the paired variant
  // (kronnd_paired_kernel): same parameters and layout
  void (*launch_g[3])(const KronNDParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) = {};
  const void* func_g[3] = {};
  // mass-only variant (kronnd_mass_kernel, its own layout of per_elem_m values per element)
  void (*launch_m)(const KronNDParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) = nullptr;
  const void* func_m = nullptr;
  int per_elem_m = 0;
  int mass_g = 2;  // axes per block of the mass-only kernel (3 when N^3 <= 27)
  // BF16 tensor-core variant (kronnd_tc_kernel.cuh; FP32 parameters, even D, N^(D/2) <= 32)
  void (*launch_tc)(const KronNDParams<float>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) = nullptr;
  const void* func_tc = nullptr;
  int tc_warp_bytes = 0;
  // interior-penalty diffusion (kronnd_diff_kernel.cuh)
  void (*launch_diff)(const KronDiffParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) = nullptr;
  const void* func_diff = nullptr;
  int per_elem_diff = 0, header_diff = 0;
  // its coefficient gradient (kronnd_diff_grad_kernel.cuh)
  void (*launch_grad)(const KronDiffParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) = nullptr;
  const void* func_grad = nullptr;
  int per_elem_grad = 0, header_grad = 0;
};
KronNDEntry<double>& kronnd_slot_f64(int D, int N);
KronNDEntry<float>& kronnd_slot_f32(int D, int N);
void register_kronnd_d1();
void register_kronnd_d2();
void register_kronnd_d3();
void register_kronnd_d4();
void register_kronnd_d5();
void register_kronnd_d6();

}  // namespace dgop
