// Registry of the Kronecker-form kernels.
#pragma once

#include <cuda_runtime.h>

#include "kron.h"

namespace dgop {

constexpr int kKronThreads = 128;

template <typename Real>
struct KronEntry {
  void (*launch)(const KronParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) = nullptr;
  const void* func = nullptr;      // kernel symbol (mass merged or absent)
  const void* func_sep = nullptr;  // kernel symbol with a separate mass term
  int epw = 0;        // elements per warp group
  int warp_smem = 0;  // Real values of shared memory per warp
};

KronEntry<double>& kron3d_slot_f64(int N);
KronEntry<float>& kron3d_slot_f32(int N);
void register_kron3d();

}  // namespace dgop
