// Interior-penalty DG diffusion operators (SIPDG / NIPG / IIPG): the host planner of the per-axis
// base matrices and the operator's creation (kernel: kronnd_diff_kernel.cuh).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "basis.h"
#include "dgop_internal.h"

namespace dgop {

template <typename Real>
void free_diff(KronDiffCfg<Real>& K) {
  if (K.d_mats) cudaFree(K.d_mats);
  if (K.d_mu) cudaFree(K.d_mu);
  K = KronDiffCfg<Real>{};
}
template void free_diff<double>(KronDiffCfg<double>&);
template void free_diff<float>(KronDiffCfg<float>&);

namespace {

#define DGOP_CUDA_D(call)                               \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

template <typename Real>
__global__ void to_real(const double* in, Real* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (Real)in[i];
}

// Base matrices of every axis (see kronnd_diff_kernel.cuh), row-major N x N, axis-major, then
// the trace rows l(0), l(1), l'(0), l'(1) of the coefficient-gradient kernel.
bool diff_tables(const dgop_space& s, int q, double kappa, std::vector<double>& mats) {
  const int N = s.n, D = s.D;
  double xq[kMaxQ], wq[kMaxQ], xn[kMaxN], wn[kMaxN];
  if (!gauss_points(1, q, xq, wq)) return false;
  if (!gauss_points(s.basis == DGOP_BASIS_GLL ? 0 : 1, N, xn, wn)) return false;
  double B[kMaxQ][kMaxN], G[kMaxQ][kMaxN], b[2][kMaxN], d[2][kMaxN];
  for (int i = 0; i < q; ++i)
    for (int j = 0; j < N; ++j) {
      B[i][j] = lagrange_value(xn, N, j, xq[i]);
      G[i][j] = lagrange_grad(xn, N, j, xq[i]);
    }
  for (int j = 0; j < N; ++j)
    for (int side = 0; side < 2; ++side) {
      b[side][j] = lagrange_value(xn, N, j, (double)side);
      d[side][j] = lagrange_grad(xn, N, j, (double)side);
    }
  double detJ = 1.0;
  for (int k = 0; k < D; ++k) detJ *= s.h[k];
  mats.assign((size_t)D * kDiffMats * N * N + 4 * N, 0.0);
  double* tv = mats.data() + (size_t)D * kDiffMats * N * N;
  for (int j = 0; j < N; ++j)
    for (int side = 0; side < 2; ++side) {
      tv[side * N + j] = b[side][j];
      tv[(2 + side) * N + j] = d[side][j];
    }
  for (int a = 0; a < D; ++a) {
    const double h = s.h[a], fm = detJ / h;  // face measure
    auto M = [&](int k) { return mats.data() + ((size_t)a * kDiffMats + k) * N * N; };
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) {
        double kk = 0.0, mm = 0.0;
        for (int p = 0; p < q; ++p) {
          kk += G[p][i] * wq[p] * G[p][j];
          mm += B[p][i] * wq[p] * B[p][j];
        }
        M(kDK)[i * N + j] = detJ / (h * h) * kk;
        M(kDM)[i * N + j] = mm;
        for (int side = 0; side < 2; ++side) {
          const double nu = side ? 1.0 : -1.0;
          const int o = 1 - side;
          M(kDP1 + side)[i * N + j] = fm * nu / h * b[side][i] * d[side][j];
          M(kDP2 + side)[i * N + j] = fm * nu / h * d[side][i] * b[side][j];
          M(kDP3 + side)[i * N + j] = fm * kappa / h * b[side][i] * b[side][j];
          M(kDQ1 + side)[i * N + j] = fm * nu / h * b[side][i] * d[o][j];
          M(kDQ2 + side)[i * N + j] = fm * nu / h * d[side][i] * b[o][j];
          M(kDQ3 + side)[i * N + j] = fm * kappa / h * b[side][i] * b[o][j];
        }
      }
  }
  return true;
}

// Launch shape of the coefficient-gradient kernel (FP64); leaves grad_ready false when the element
// does not fit.
int setup_grad(dgop_operator* op, KronDiffCfg<double>& K) {
  const dgop_space& s = op->sp;
  const KronNDEntry<double>* entry = K.entry;
  if (!entry->launch_grad) return DGOP_OK;
  const size_t per = (size_t)entry->per_elem_grad * sizeof(double);
  const size_t hdr = (size_t)entry->header_grad * sizeof(double);
  int eb = 1;
  while (eb < 64 && hdr + per * (eb * 2) <= 96 * 1024) eb *= 2;
  const int64_t lines = (int64_t)(s.ndofs / s.nelem) / s.n;
  while (eb > 1 && (int64_t)(eb / 2) * lines >= kKronNDThreads) eb /= 2;
  int max_smem = 0;
  DGOP_CUDA_D(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, op->device));
  cudaFuncAttributes fa{};
  DGOP_CUDA_D(cudaFuncGetAttributes(&fa, entry->func_grad));
  max_smem -= (int)fa.sharedSizeBytes;
  while (eb > 1 && hdr + per * eb > (size_t)max_smem) eb /= 2;
  if (hdr + per * eb > (size_t)max_smem) return DGOP_OK;
  K.grad_eb = eb;
  K.grad_smem = hdr + per * eb;
  DGOP_CUDA_D(cudaFuncSetAttribute(entry->func_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem));
  int per_sm = 0;
  DGOP_CUDA_D(
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, entry->func_grad, kKronNDThreads, K.grad_smem));
  if (per_sm < 1) return DGOP_OK;
  const int64_t ctas = std::min<int64_t>((s.nelem + eb - 1) / eb, (int64_t)device_sms(op->device) * per_sm);
  K.grad_grid = dim3((unsigned)std::max<int64_t>(ctas, 1));
  K.grad_ready = true;
  return DGOP_OK;
}

template <typename Real>
int setup_diff(dgop_operator* op, KronDiffCfg<Real>& K, const std::vector<double>& mats, const double* mu,
               double sigma, double kappa, int boundary) {
  const dgop_space& s = op->sp;
  const KronNDEntry<Real>* entry = nullptr;
  if constexpr (sizeof(Real) == 8) entry = &kronnd_slot_f64(s.D, s.n);
  else entry = &kronnd_slot_f32(s.D, s.n);
  if (!entry->launch_diff) {
    set_error("no interior-penalty kernel for this (dimension, order): the element exceeds shared memory");
    return DGOP_ERR_UNSUPPORTED;
  }
  K.entry = entry;
  KronDiffParams<Real>& p = K.params;
  std::memset(&p, 0, sizeof(p));
  p.nelem = s.nelem;
  int64_t stride = 1;
  for (int k = 0; k < s.D; ++k) {
    p.sizes[k] = s.sizes[k];
    p.estride[k] = stride;
    stride *= s.sizes[k];
    p.periodic[k] = s.periodic[k];
  }
  p.boundary = boundary;
  p.sigma = (Real)sigma;
  p.kappa = (Real)kappa;
  double detJ = 1.0;
  for (int k = 0; k < s.D; ++k) detJ *= s.h[k];
  for (int k = 0; k < s.D; ++k) p.face_h[k] = (Real)(detJ / (s.h[k] * s.h[k]));
  std::vector<Real> mr(mats.begin(), mats.end());
  Real* dm = nullptr;
  DGOP_CUDA_D(cudaMalloc(&dm, sizeof(Real) * mr.size()));
  K.d_mats = dm;
  DGOP_CUDA_D(cudaMemcpy(dm, mr.data(), sizeof(Real) * mr.size(), cudaMemcpyHostToDevice));
  p.mats = dm;
  if constexpr (sizeof(Real) == 8) {
    p.mu = mu;
  } else {
    DGOP_CUDA_D(cudaMalloc(&K.d_mu, sizeof(Real) * s.nelem));
    to_real<Real><<<256, 256>>>(mu, K.d_mu, s.nelem);
    DGOP_CUDA_D(cudaGetLastError());
    p.mu = K.d_mu;
  }
  // elements per CTA: as many as fit in ~72 KB (three CTAs per SM), then, among the counts down
  // to half of that, the one whose lines fill the CTA's passes best (every pass runs over the
  // lines of all the CTA's elements, kKronNDThreads at a time)
  const size_t per = (size_t)entry->per_elem_diff * sizeof(Real);
  const size_t hdr = (size_t)entry->header_diff * sizeof(Real);
  int max_smem = 0;
  DGOP_CUDA_D(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, op->device));
  cudaFuncAttributes fa{};
  DGOP_CUDA_D(cudaFuncGetAttributes(&fa, entry->func_diff));
  max_smem -= (int)fa.sharedSizeBytes;
  const size_t budget = std::min<size_t>((size_t)max_smem, 72 * 1024);
  int ebmax = (int)std::min<int64_t>(kDiffMaxEB, budget > hdr ? (int64_t)((budget - hdr) / per) : 0);
  if (ebmax < 1 && hdr + per <= (size_t)max_smem) ebmax = 1;
  if (ebmax < 1) {
    set_error("element does not fit in shared memory");
    return DGOP_ERR_UNSUPPORTED;
  }
  const int64_t lines = (int64_t)(s.ndofs / s.nelem) / s.n;
  int eb = ebmax;
  double best = -1.0;
  for (int c = ebmax; c >= std::max(1, ebmax / 2); --c) {
    const int64_t l = c * lines;
    const double use = (double)l / (double)(((l + kKronNDThreads - 1) / kKronNDThreads) * kKronNDThreads);
    if (use > best + 1e-9) {
      best = use;
      eb = c;
    }
  }
  p.eb = eb;
  K.block = dim3(kKronNDThreads);
  K.smem = hdr + per * eb;
  DGOP_CUDA_D(cudaFuncSetAttribute(entry->func_diff, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem));
  int per_sm = 0;
  DGOP_CUDA_D(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, entry->func_diff, kKronNDThreads, K.smem));
  if (per_sm < 1) {
    set_error("interior-penalty kernel cannot be resident");
    return DGOP_ERR_UNSUPPORTED;
  }
  const int64_t ctas = std::min<int64_t>((s.nelem + eb - 1) / eb, (int64_t)device_sms(op->device) * per_sm);
  K.grid = dim3((unsigned)std::max<int64_t>(ctas, 1));
  K.ready = true;
  if constexpr (sizeof(Real) == 8) return setup_grad(op, K);
  return DGOP_OK;
}

}  // namespace
}  // namespace dgop

using namespace dgop;

extern "C" int dgop_sipdg_create(const dgop_space* space, int q, const double* mu, double sigma, double kappa,
                                 int boundary, dgop_operator** out) {
  if (!space || !out || !mu) {
    set_error("dgop_sipdg_create: null argument");
    return DGOP_ERR_ARG;
  }
  *out = nullptr;
  if (q < 1 || q > kMaxQ) {
    set_error("q must be in [1, 8]");
    return DGOP_ERR_ARG;
  }
  ensure_registry();
  auto* op = new (std::nothrow) dgop_operator();
  if (!op) {
    set_error("host allocation failed");
    return DGOP_ERR_ALLOC;
  }
  op->sp = *space;
  op->q = q;
  op->flags = kDiffusion | kFaceInt | (boundary ? kFaceBnd : 0);
  op->ip_sigma = sigma;
  op->kernel = DGOP_KERNEL_DIFF;
  op->kron_why = "interior-penalty diffusion operator";
  cudaGetDevice(&op->device);
  std::vector<double> mats;
  if (!diff_tables(op->sp, q, kappa, mats)) {
    delete op;
    set_error("basis tables");
    return DGOP_ERR_ARG;
  }
  int rc = setup_diff<double>(op, op->s64, mats, mu, sigma, kappa, boundary);
  if (rc == DGOP_OK && setup_diff<float>(op, op->s32, mats, mu, sigma, kappa, boundary) != DGOP_OK) {
    free_diff(op->s32);
    set_error("");
  }
  if (rc != DGOP_OK) {
    free_diff(op->s64);
    delete op;
    return rc;
  }
  *out = op;
  return DGOP_OK;
}

extern "C" int dgop_sipdg_gradient(const dgop_operator* op, const double* u, const double* lambda,
                                   const double* scale, double* out, void* stream) {
  if (!op || !u || !lambda || !out) {
    set_error("dgop_sipdg_gradient: null argument");
    return DGOP_ERR_ARG;
  }
  if (op->kernel != DGOP_KERNEL_DIFF) {
    set_error("dgop_sipdg_gradient: not an interior-penalty diffusion operator");
    return DGOP_ERR_ARG;
  }
  const KronDiffCfg<double>& K = op->s64;
  if (!K.grad_ready) {
    set_error("no coefficient-gradient kernel for this (dimension, order): the element exceeds shared memory");
    return DGOP_ERR_UNSUPPORTED;
  }
  KronDiffParams<double> p = K.params;
  p.x = u;
  p.lam = lambda;
  p.gout = out;
  p.gscale = scale;
  p.eb = K.grad_eb;
  p.e_begin = 0;
  p.skip = nullptr;
  K.entry->launch_grad(p, K.grad_grid, K.block, K.grad_smem, (cudaStream_t)stream);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "coefficient-gradient kernel launch");
  return DGOP_OK;
}
