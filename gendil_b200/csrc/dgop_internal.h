// Internal definitions shared by the C-ABI implementation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "dgop.h"
#include "dgop_params.h"
#include "kron.h"
#include "kron_registry.h"
#include "registry.h"

struct dgop_space {
  int D = 0, P = 0, n = 0, basis = 0;
  int64_t sizes[DGOP_MAX_DIM] = {};
  double h[DGOP_MAX_DIM] = {}, origin[DGOP_MAX_DIM] = {};
  int periodic[DGOP_MAX_DIM] = {};
  int64_t nelem = 0, ndofs = 0;
};

namespace dgop {

template <typename Real>
struct LaunchCfg {
  const GenericEntry<Real>* entry = nullptr;
  OpParams<Real> params{};  // x, y, alpha, beta_y and flags are set per call
  int eb = 1;
  dim3 grid, block;
  size_t smem = 0;
  Real* d_tab = nullptr;
  Real* d_scratch = nullptr;
  Real* d_elem[kMaxDim + 1] = {};  // converted per-element factors (FP32 only)
  bool ready = false;
};

template <typename Real>
struct KronCfg {
  bool ready = false;
  const KronEntry<Real>* entry = nullptr;
  KronParams<Real> params{};    // forward operator
  KronParams<Real> params_t{};  // transposed operator
  struct Launch {
    bool ok = false;
    dim3 grid, block;
    dim3 grid_dot;  // launches with the inner-product epilogue (that kernel's residency)
    size_t smem = 0;
    float ms = 0.0f;  // autotuner timing (0: not timed)
  } launch[kKronVariants];
  int variant = 0;  // the kernel variant in use
  int fallback = 1;  // fastest variant without bulk-tensor staging (element ranges not in whole groups)
  Real* d_mats = nullptr;
  Real* d_phi = nullptr;
  signed char* d_sgn = nullptr;
  Real* d_elem[4] = {};  // converted per-element factors (FP32 only)
  // bulk-tensor variants: face words per element and slot words per group of 8 elements, for
  // the forward [0] and transposed [1] operator; a device word set when a bounded wait gives up
  uint32_t* d_eflags[2] = {};
  uint32_t* d_gwords[2] = {};
  int* d_err = nullptr;
  // tensor maps of recent (x, y) pairs (opaque CUtensorMap bytes: group, z slices, y slices,
  // one element, out)
  struct MapEntry {
    const void* x = nullptr;
    const void* y = nullptr;
    alignas(64) unsigned char maps[5][128];
  };
  MapEntry map_cache[8];
  int map_next = 0;
};

template <typename Real>
struct KronNDCfg {
  bool ready = false;
  const KronNDEntry<Real>* entry = nullptr;
  KronNDParams<Real> params{};    // forward operator
  KronNDParams<Real> params_t{};  // transposed operator
  dim3 grid, block;
  size_t smem = 0;
  Real* d_mats = nullptr;
  Real* d_phi = nullptr;
  signed char* d_sgn = nullptr;
  Real* d_elem[kMaxDim + 1] = {};  // converted per-element factors (FP32 only)
  // launch shapes of the variants (kKronNDVariants; 0 = grid / smem / params.eb above)
  struct Variant {
    bool ok = false;
    int eb = 0;
    dim3 grid;
    size_t smem = 0;
    float ms = 0.0f;  // autotuner's time per launch (0: not timed)
    int threads = kKronNDThreads;
  } var[kKronNDVariants];
  int variant = 0;
  // BF16 tensor-core launch (FP32 configuration only) and its Kronecker tile tables
  bool tc_ok = false;
  dim3 tc_grid;
  size_t tc_smem = 0;
  void* d_tc_tiles = nullptr;
  float* d_tc_scale = nullptr;
};

template <typename Real>
struct KronDiffCfg {
  bool ready = false;
  const KronNDEntry<Real>* entry = nullptr;
  KronDiffParams<Real> params{};
  dim3 grid, block;
  size_t smem = 0;
  Real* d_mats = nullptr;
  Real* d_mu = nullptr;  // FP32 copy of the per-element diffusivity
  // coefficient-gradient kernel launch (FP64)
  bool grad_ready = false;
  int grad_eb = 0;
  dim3 grad_grid;
  size_t grad_smem = 0;
};

void set_error(const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

}  // namespace dgop

struct dgop_operator {
  dgop_space sp;
  int q = 0;
  int flags = 0;
  double g = 0.0;
  int device = 0;
  int kernel = 0;             // DGOP_KERNEL_GENERIC or DGOP_KERNEL_KRON
  const char* kron_why = "";  // why the Kronecker form is unavailable
  int version = 0;            // bumped whenever the launch configuration changes
  dgop::LaunchCfg<double> f64;
  dgop::LaunchCfg<float> f32;
  dgop::KronCfg<double> k64;
  dgop::KronCfg<float> k32;
  dgop::KronNDCfg<double> n64;
  dgop::KronNDCfg<float> n32;
  dgop::KronDiffCfg<double> s64;  // interior-penalty diffusion (dgop_sipdg_create)
  dgop::KronDiffCfg<float> s32;
  double ip_sigma = 0.0;
};

namespace dgop {
// Optional epilogue of an FP64 apply: partials[b] = sum over CTA b's outputs of z . y in a fixed
// order, entries past the grid zeroed up to `count`.  Kernels that provide it set `*fused`; for
// the others the caller computes the product itself.
struct DotEpilogue {
  const double* z = nullptr;
  double* partials = nullptr;
  int count = 0;
  bool* fused = nullptr;
};
// Launch the operator kernel: y = alpha * Op(x) + beta_y * y, with `extra_flags` or-ed in.
// When `skip` (a device word) is non-zero at run time the launch does nothing.
int launch_f64(dgop_operator* op, double alpha, const double* x, double beta_y, double* y, int extra_flags,
               cudaStream_t s, const int* skip = nullptr, const DotEpilogue* dot = nullptr);
int launch_bf16(dgop_operator* op, float alpha, const float* x, float beta_y, float* y, int extra_flags,
                cudaStream_t s, const int* skip);
int launch_f32(dgop_operator* op, float alpha, const float* x, float beta_y, float* y, int extra_flags,
               cudaStream_t s, const int* skip = nullptr);
// y = Op(x) on the elements [e_begin, e_end) only (y elsewhere untouched; x read around them)
int launch_range_f64(dgop_operator* op, const double* x, double* y, int64_t e_begin, int64_t e_end, cudaStream_t s);
int device_sms(int dev);
template <typename Real>
void free_diff(KronDiffCfg<Real>& K);
}  // namespace dgop
