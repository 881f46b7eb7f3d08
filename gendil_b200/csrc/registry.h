// Kernel registry: one entry per compiled (dimension, N, Q) instantiation and precision.
#pragma once

#include <cuda_runtime.h>

#include "dgop_params.h"

namespace dgop {

template <typename Real>
struct GenericEntry {
  void (*launch)(const OpParams<Real>& p, dim3 grid, dim3 block, size_t smem, cudaStream_t s) = nullptr;
  const void* func = nullptr;  // kernel symbol, for attributes and occupancy queries
  int per_elem = 0;            // Real values of work memory per element
  int mats = 0;                // Real values of staged 1D tables
};

// Lookup; nullptr when (D, N, Q) was not compiled.
const GenericEntry<double>* find_generic_f64(int D, int N, int Q);
const GenericEntry<float>* find_generic_f32(int D, int N, int Q);

// Filled once, on first use, by the per-dimension instantiation units.
void ensure_registry();

// Bytes of shared memory for the fixed part of a generic launch with `eb` elements.
inline int generic_fixed_bytes_rt(int D, int mats, int eb, int real_size) {
  return mats * real_size + ((eb * D + 1) & ~1) * 4 + eb * 2 * D * 8;
}

}  // namespace dgop
