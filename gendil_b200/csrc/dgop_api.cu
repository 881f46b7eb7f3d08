// C-ABI implementation: spaces, operators, coefficient tables, launch configuration.
#include <cuda.h>  // tensor-map types; cuTensorMapEncodeTiled comes through cudaGetDriverEntryPointByVersion
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <new>
#include <random>
#include <string>
#include <type_traits>
#include <vector>

#include "basis.h"
#include "kron_plan.h"
#include "kron_tma.h"
#include "dgop_internal.h"

namespace dgop {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

int cuda_fail(cudaError_t e, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return DGOP_ERR_CUDA;
}

#define DGOP_CUDA(call)                               \
  do {                                                \
    cudaError_t _e = (call);                          \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

namespace {

// Per-space 1D tables for quadrature size q.
struct Tables1D {
  double xq[kMaxQ], wq[kMaxQ], xn[kMaxN], wn[kMaxN];
  double B[kMaxQ * kMaxN], Dq[kMaxQ * kMaxQ], Bf[2][kMaxN];
};

bool make_tables(const dgop_space& s, int q, Tables1D& t) {
  if (!gauss_points(1, q, t.xq, t.wq)) return false;
  if (!gauss_points(s.basis == DGOP_BASIS_GLL ? 0 : 1, s.n, t.xn, t.wn)) return false;
  for (int i = 0; i < q; ++i)
    for (int j = 0; j < s.n; ++j) t.B[i * s.n + j] = lagrange_value(t.xn, s.n, j, t.xq[i]);
  // collocated derivative on the Gauss points (doftoquad.hpp:142-150): Dq[i][j] = l_j'(x_i)
  for (int i = 0; i < q; ++i)
    for (int j = 0; j < q; ++j) t.Dq[i * q + j] = lagrange_grad(t.xq, q, j, t.xq[i]);
  for (int j = 0; j < s.n; ++j) {
    t.Bf[0][j] = lagrange_value(t.xn, s.n, j, 0.0);
    t.Bf[1][j] = lagrange_value(t.xn, s.n, j, 1.0);
  }
  return true;
}

struct PackedCoef {
  double constant = 0.0;
  int nterms = 0;
  int64_t off[kMaxTerms][kMaxDim];
  const double* elem = nullptr;
};

// Appends the host tables of `c` to `pack` and records their offsets.
int pack_coef(const dgop_space& s, int q, const dgop_coef* c, std::vector<double>& pack, PackedCoef& out) {
  for (auto& row : out.off)
    for (auto& v : row) v = -1;
  if (!c) {
    out.constant = 0.0;
    out.nterms = 0;
    return DGOP_OK;
  }
  if (c->nterms < 0 || c->nterms > DGOP_MAX_TERMS) {
    set_error("coefficient: nterms must be in [0, 4]");
    return DGOP_ERR_ARG;
  }
  out.constant = c->constant;
  out.nterms = c->nterms;
  out.elem = c->element_factor;
  for (int t = 0; t < c->nterms; ++t) {
    for (int k = 0; k < s.D; ++k) {
      const double* tab = c->tables[t][k];
      if (!tab) continue;
      const int64_t len = s.sizes[k] * (q + 2);
      out.off[t][k] = (int64_t)pack.size();
      pack.insert(pack.end(), tab, tab + len);
    }
  }
  return DGOP_OK;
}

int device_sm_count(int dev);
}  // namespace
int device_sms(int dev) { return device_sm_count(dev); }
namespace {
int device_sm_count(int dev) {
  static int cache[64] = {};
  if (dev < 0 || dev >= 64) return 148;
  if (!cache[dev]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    cache[dev] = v;
  }
  return cache[dev];
}

template <typename Real>
__global__ void convert_kernel(const double* in, Real* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (Real)in[i];
}

template <typename Real>
int setup_launch(dgop_operator* op, LaunchCfg<Real>& L, const Tables1D& t, const std::vector<double>& pack,
                 const PackedCoef& sig, const PackedCoef* beta) {
  const dgop_space& s = op->sp;
  const int D = s.D, N = s.n, Q = op->q;
  const GenericEntry<Real>* e = nullptr;
  if constexpr (sizeof(Real) == 8) e = find_generic_f64(D, N, Q);
  else e = find_generic_f32(D, N, Q);
  if (!e || !e->launch) {
    set_error("no kernel compiled for dim=" + std::to_string(D) + " order=" + std::to_string(N - 1) +
              " q=" + std::to_string(Q) + (sizeof(Real) == 8 ? " (fp64)" : " (fp32)"));
    return DGOP_ERR_UNSUPPORTED;
  }
  L.entry = e;
  OpParams<Real>& p = L.params;
  std::memset(&p, 0, sizeof(p));
  p.nelem = s.nelem;
  int64_t stride = 1;
  double detJ = 1.0;
  for (int k = 0; k < D; ++k) {
    p.sizes[k] = s.sizes[k];
    p.estride[k] = stride;
    stride *= s.sizes[k];
    p.periodic[k] = s.periodic[k];
    p.invh[k] = (Real)(1.0 / s.h[k]);
    detJ *= s.h[k];
  }
  p.detJ = (Real)detJ;
  for (int i = 0; i < Q * N; ++i) p.B[i] = (Real)t.B[i];
  for (int i = 0; i < Q * Q; ++i) p.Dq[i] = (Real)t.Dq[i];
  for (int j = 0; j < N; ++j) {
    p.Bf[0][j] = (Real)t.Bf[0][j];
    p.Bf[1][j] = (Real)t.Bf[1][j];
  }
  for (int i = 0; i < Q; ++i) p.wq[i] = (Real)t.wq[i];
  p.tab_ld = Q + 2;
  p.gll = s.basis == DGOP_BASIS_GLL ? 1 : 0;
  p.g = (Real)op->g;
  p.flags = op->flags;
  // tables
  if (!pack.empty()) {
    std::vector<Real> packed(pack.begin(), pack.end());
    DGOP_CUDA(cudaMalloc(&L.d_tab, sizeof(Real) * packed.size()));
    DGOP_CUDA(cudaMemcpy(L.d_tab, packed.data(), sizeof(Real) * packed.size(), cudaMemcpyHostToDevice));
  }
  p.tab = L.d_tab;
  auto fill = [&](CoefDev<Real>& d, const PackedCoef& c, int slot) -> int {
    d.constant = (Real)c.constant;
    d.nterms = c.nterms;
    std::memcpy(d.off, c.off, sizeof(d.off));
    d.elem = nullptr;
    if (c.elem) {
      if constexpr (sizeof(Real) == 8) {
        d.elem = reinterpret_cast<const Real*>(c.elem);
      } else {
        DGOP_CUDA(cudaMalloc(&L.d_elem[slot], sizeof(Real) * s.nelem));
        convert_kernel<Real><<<256, 256>>>(c.elem, L.d_elem[slot], s.nelem);
        DGOP_CUDA(cudaGetLastError());
        d.elem = L.d_elem[slot];
      }
    }
    return DGOP_OK;
  };
  int rc = fill(p.sigma, sig, 0);
  if (rc) return rc;
  for (int k = 0; k < D; ++k) {
    rc = fill(p.beta[k], beta[k], k + 1);
    if (rc) return rc;
  }
  // launch shape
  int max_smem = 0;
  DGOP_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, op->device));
  const int sms = device_sm_count(op->device);
  const int64_t per_elem_bytes = (int64_t)e->per_elem * sizeof(Real);
  const int threads = 256;
  int eb;
  bool use_scratch = false;
  const int64_t budget = 100 * 1024;
  if (per_elem_bytes + generic_fixed_bytes_rt(D, e->mats, 1, sizeof(Real)) > max_smem - 1024) {
    use_scratch = true;
    eb = 1;
  } else {
    eb = (int)std::max<int64_t>(1, std::min<int64_t>(64, budget / per_elem_bytes));
    const int64_t want_ctas = 2LL * sms;
    while (eb > 1 && (s.nelem + eb - 1) / eb < want_ctas) eb /= 2;
  }
  L.eb = eb;
  p.eb = eb;
  size_t smem = generic_fixed_bytes_rt(D, e->mats, eb, sizeof(Real));
  if (!use_scratch) smem += (size_t)eb * per_elem_bytes;
  smem = (smem + 15) & ~size_t(15);
  // the attribute is per kernel: allow the device maximum so operators sharing a kernel never
  // lower each other's limit; occupancy below uses this launch's actual size.
  DGOP_CUDA(cudaFuncSetAttribute(e->func, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem));
  if ((int)smem > max_smem) {
    set_error("shared memory request exceeds the device limit");
    return DGOP_ERR_UNSUPPORTED;
  }
  int per_sm = 0;
  DGOP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, e->func, threads, smem));
  if (per_sm < 1) per_sm = 1;
  const int64_t need = (s.nelem + eb - 1) / eb;
  int64_t grid = std::min<int64_t>(need, (int64_t)sms * per_sm);
  if (use_scratch) {
    grid = std::min<int64_t>(grid, (int64_t)sms * 2);
    p.scratch_per_cta = e->per_elem;
    DGOP_CUDA(cudaMalloc(&L.d_scratch, sizeof(Real) * (size_t)grid * e->per_elem));
    p.scratch = L.d_scratch;
  }
  L.grid = dim3((unsigned)std::max<int64_t>(grid, 1));
  L.block = dim3(threads);
  L.smem = smem;
  L.ready = true;
  return DGOP_OK;
}

// A coefficient in the Kronecker planner's form: a constant, or one product term (no constant).
SepCoef sep_of(const dgop_coef* c) {
  SepCoef s;
  if (!c) {
    s.separable = true;
    s.c = 1.0;
    return s;
  }
  s.has_elem = c->element_factor != nullptr;
  if (c->nterms == 0) {
    s.separable = true;
    s.c = c->constant;
  } else if (c->nterms == 1 && c->constant == 0.0) {
    s.separable = true;
    s.c = 1.0;
    for (int k = 0; k < DGOP_MAX_DIM; ++k) s.tab[k] = c->tables[0][k];
  }
  return s;
}

// cuTensorMapEncodeTiled, fetched from the driver once (no link against libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn tensor_map_encoder() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
    cudaGetLastError();
  });
  return fn;
}

// One FP64 tensor map (dims, byte strides of dims 1.., box) over a 16-byte aligned vector.
int encode_map(CUtensorMap* m, const void* base, int rank, const cuuint64_t* dims, const cuuint64_t* strides,
               const cuuint32_t* box, CUtensorMapSwizzle swizzle) {
  const EncodeTiledFn enc = tensor_map_encoder();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled is unavailable");
    return DGOP_ERR_CUDA;
  }
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (cuuint32_t)rank, const_cast<void*>(base), dims, strides,
                         box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return DGOP_ERR_CUDA;
  }
  return DGOP_OK;
}

// The five maps of the bulk-tensor variants (kron3d_tma_kernel.cuh) for vectors x and y of
// `nelem` elements of 4 x 4 x 4 values.
int encode_tma_maps(KronTmaParams<double>& T, const double* x, double* y, int64_t nelem) {
  const cuuint64_t rows = (cuuint64_t)nelem * 4;
  const cuuint64_t d2[2] = {16, rows}, s2[1] = {128};
  const cuuint32_t b2[2] = {16, 32}, b2e[2] = {16, 4};
  const cuuint64_t d3[3] = {16, 4, (cuuint64_t)nelem}, s3[2] = {128, 512};
  const cuuint32_t b3[3] = {16, 1, 8};
  const cuuint64_t d4[4] = {4, 4, 4, (cuuint64_t)nelem}, s4[3] = {32, 128, 512};
  const cuuint32_t b4[4] = {4, 1, 4, 8};
  int rc = encode_map(&T.win, x, 2, d2, s2, b2, CU_TENSOR_MAP_SWIZZLE_128B);
  if (rc == DGOP_OK) rc = encode_map(&T.zsl, x, 3, d3, s3, b3, CU_TENSOR_MAP_SWIZZLE_128B);
  if (rc == DGOP_OK) rc = encode_map(&T.ysl, x, 4, d4, s4, b4, CU_TENSOR_MAP_SWIZZLE_NONE);
  if (rc == DGOP_OK) rc = encode_map(&T.xel, x, 2, d2, s2, b2e, CU_TENSOR_MAP_SWIZZLE_NONE);
  if (rc == DGOP_OK) rc = encode_map(&T.out, y, 2, d2, s2, b2, CU_TENSOR_MAP_SWIZZLE_128B);
  return rc;
}

// Launch kernel variant v of the 3D Kronecker form with parameters p (x, y, flags, range set).
// Bulk-tensor variants need element ranges in whole groups of 8; other ranges take the fastest
// variant without them.
std::mutex g_map_cache_mutex;

// The five maps for (x, y), from the operator's cache of recent pairs or freshly encoded.
int tma_maps_cached(KronCfg<double>& K, KronTmaParams<double>& T, const double* x, double* y, int64_t nelem) {
  static_assert(sizeof(CUtensorMap) == 128, "tensor map size");
  std::lock_guard<std::mutex> lock(g_map_cache_mutex);
  for (const auto& m : K.map_cache) {
    if (m.x == x && m.y == y) {
      std::memcpy(&T.win, m.maps[0], 128);
      std::memcpy(&T.zsl, m.maps[1], 128);
      std::memcpy(&T.ysl, m.maps[2], 128);
      std::memcpy(&T.xel, m.maps[3], 128);
      std::memcpy(&T.out, m.maps[4], 128);
      return DGOP_OK;
    }
  }
  const int rc = encode_tma_maps(T, x, y, nelem);
  if (rc != DGOP_OK) return rc;
  auto& m = K.map_cache[K.map_next];
  K.map_next = (K.map_next + 1) % 8;
  std::memcpy(m.maps[0], &T.win, 128);
  std::memcpy(m.maps[1], &T.zsl, 128);
  std::memcpy(m.maps[2], &T.ysl, 128);
  std::memcpy(m.maps[3], &T.xel, 128);
  std::memcpy(m.maps[4], &T.out, 128);
  m.x = x;
  m.y = y;
  return DGOP_OK;
}

template <typename Real>
int launch_kron(const dgop_operator* op, KronCfg<Real>& K, int v, const KronParams<Real>& p, cudaStream_t s) {
  const bool whole = p.e_begin % 8 == 0 && p.nelem % 8 == 0;
  if (K.entry->v[v].launch_tma && !whole) v = K.fallback;
  const KronVariant<Real>& kv = K.entry->v[v];
  const auto& L = K.launch[v];
  if (kv.launch_tma) {
    if constexpr (sizeof(Real) == 8) {
      KronTmaParams<double> T;
      std::memset(&T, 0, sizeof(T));
      T.k = p;
      const int rc = tma_maps_cached(K, T, p.x, p.y, op->sp.nelem);
      if (rc != DGOP_OK) return rc;
      const int tr = (p.flags & kTranspose) ? 1 : 0;
      T.eflags = K.d_eflags[tr];
      T.gwords = K.d_gwords[tr];
      T.err = K.d_err;
      for (int& m : T.mat_index) m = -1;
      T.nmat = 0;
      for (int k = 0; k < 8; ++k)
        if (p.vary[tma_yz_slot(k)]) T.mat_index[tma_yz_slot(k)] = T.nmat++;
      kv.launch_tma(T, p.dot_partials ? L.grid_dot : L.grid, L.block, L.smem, s);
    }
  } else {
    kv.launch(p, p.dot_partials ? L.grid_dot : L.grid, L.block, L.smem, s);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "operator kernel launch");
  return DGOP_OK;
}

// Let kernel f use dynamic shared memory up to the device's per-block opt-in limit, net of its
// static shared memory (the attribute is rejected when static + dynamic exceed the limit).
int allow_dynamic_smem(const void* f, int max_smem) {
  cudaFuncAttributes attr;
  DGOP_CUDA(cudaFuncGetAttributes(&attr, f));
  DGOP_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem - (int)attr.sharedSizeBytes));
  return DGOP_OK;
}

template <typename Real>
int upload(Real** dst, const double* src, size_t n) {
  std::vector<Real> tmp(src, src + n);
  DGOP_CUDA(cudaMalloc(dst, sizeof(Real) * (n ? n : 1)));
  if (n) DGOP_CUDA(cudaMemcpy(*dst, tmp.data(), sizeof(Real) * n, cudaMemcpyHostToDevice));
  return DGOP_OK;
}

template <typename Real>
int setup_kron(dgop_operator* op, KronCfg<Real>& K, const KronPlanHost& plan, const double* elem_sigma,
               const double* const* elem_beta) {
  const dgop_space& s = op->sp;
  KronEntry<Real>* entry = nullptr;
  if constexpr (sizeof(Real) == 8) entry = &kron3d_slot_f64(s.n);
  else entry = &kron3d_slot_f32(s.n);
  if (!entry->v[0].launch) {
    set_error("no Kronecker kernel for this order");
    return DGOP_ERR_UNSUPPORTED;
  }
  K.entry = entry;
  KronParams<Real>& p = K.params;
  std::memset(&p, 0, sizeof(p));
  p.nelem = s.nelem;
  p.fdx = FastDiv((uint32_t)s.sizes[0]);
  p.fdy = FastDiv((uint32_t)s.sizes[1]);
  for (int k = 0; k < 3; ++k) {
    p.sizes[k] = s.sizes[k];
    p.periodic[k] = s.periodic[k];
  }
  p.flags = op->flags;
  p.has_adv = plan.has_adv;
  p.has_mass = plan.has_mass;
  p.mass_merged = plan.mass_merged;
  p.g = (Real)op->g;
  int rc = upload<Real>(&K.d_mats, plan.mats.data(), plan.mats.size());
  if (rc) return rc;
  p.mats = K.d_mats;
  // slot -> matrix table; constant tables go to kernel-parameter space
  const int N = s.n;
  // the kernel reads element-dependent matrices with 16-byte loads when N allows them
  const int vec = (N % (16 / (int)sizeof(Real)) == 0) ? 16 / (int)sizeof(Real) : 1;
  bool aligned = true;
  auto put = [&](KronParams<Real>& q, int slot, const KronMat& m) {
    q.vary[slot] = 0;
    q.vm[slot] = m;
    if (m.off < 0) return;  // slot unused by this operator
    if (m.stride == 0) {
      for (int i = 0; i < N * N; ++i) q.cm[slot][i] = (Real)plan.mats[m.off + i];
    } else {
      q.vary[slot] = 1;
      aligned = aligned && m.off % vec == 0 && m.stride % vec == 0;
    }
  };
  if (plan.has_adv) {
    put(p, kSlotDX, plan.D[0]);
    put(p, kSlotDY, plan.D[1]);
    put(p, kSlotDZ, plan.D[2]);
    put(p, kSlotTXY, plan.T[0][1]);
    put(p, kSlotTXZ, plan.T[0][2]);
    put(p, kSlotTYZ, plan.T[1][2]);
    put(p, kSlotTYX, plan.T[1][0]);
    put(p, kSlotTZX, plan.T[2][0]);
    put(p, kSlotTZY, plan.T[2][1]);
    if (plan.has_mass && !plan.mass_merged) {
      put(p, kSlotMD, plan.MD);
      put(p, kSlotMX, plan.MT[0]);
      put(p, kSlotMY, plan.MT[1]);
    }
    std::vector<double> phi;
    std::vector<signed char> sg;
    size_t phi_off[3], sg_off[3][3];
    for (int a = 0; a < 3; ++a) {
      phi_off[a] = phi.size();
      phi.insert(phi.end(), plan.phi[a].begin(), plan.phi[a].end());
      for (int k = 0; k < 3; ++k) {
        sg_off[a][k] = sg.size();
        sg.insert(sg.end(), plan.sgn[a][k].begin(), plan.sgn[a][k].end());
      }
    }
    rc = upload<Real>(&K.d_phi, phi.data(), phi.size());
    if (rc) return rc;
    DGOP_CUDA(cudaMalloc(&K.d_sgn, sg.size() ? sg.size() : 1));
    if (!sg.empty()) DGOP_CUDA(cudaMemcpy(K.d_sgn, sg.data(), sg.size(), cudaMemcpyHostToDevice));
    for (int a = 0; a < 3; ++a) {
      p.phi[a] = K.d_phi + phi_off[a];
      for (int k = 0; k < 3; ++k) p.sgn[a][k] = (k == a) ? nullptr : K.d_sgn + sg_off[a][k];
    }
  } else {
    put(p, kSlotDZ, plan.MD);
    put(p, kSlotTZX, plan.MT[0]);
    put(p, kSlotTZY, plan.MT[1]);
  }
  auto elem_ptr = [&](const double* src, int slot, const Real** dst) -> int {
    *dst = nullptr;
    if (!src) return DGOP_OK;
    if constexpr (sizeof(Real) == 8) {
      *dst = src;
    } else {
      DGOP_CUDA(cudaMalloc(&K.d_elem[slot], sizeof(Real) * s.nelem));
      convert_kernel<Real><<<256, 256>>>(src, K.d_elem[slot], s.nelem);
      DGOP_CUDA(cudaGetLastError());
      *dst = K.d_elem[slot];
    }
    return DGOP_OK;
  };
  for (int a = 0; a < 3; ++a)
    if ((rc = elem_ptr(plan.has_adv ? elem_beta[a] : nullptr, a, &p.elem[a]))) return rc;
  if ((rc = elem_ptr(plan.has_mass ? elem_sigma : nullptr, 3, &p.elem_mass))) return rc;
  // transposed operator: the same blocks with the transposed D matrices
  K.params_t = p;
  if (plan.has_adv) {
    put(K.params_t, kSlotDX, plan.Dt[0]);
    put(K.params_t, kSlotDY, plan.Dt[1]);
    put(K.params_t, kSlotDZ, plan.Dt[2]);
  }
  if (!aligned) {
    set_error("Kronecker matrix table misaligned for vector loads");
    return DGOP_ERR_UNSUPPORTED;
  }
  // persistent grid: every warp walks groups of entry->epw consecutive elements; one launch
  // shape per kernel variant (their shared memory per warp differs)
  int max_smem = 0;
  DGOP_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, op->device));
  const bool sep = plan.has_adv && plan.has_mass && !plan.mass_merged;
  const int64_t groups = (s.nelem + entry->epw - 1) / entry->epw;
  // bulk-tensor variants: groups of 8 elements inside one x-row, plane rows addressable by int
  const bool tma_shape = entry->face_words && s.sizes[0] % 8 == 0 && s.nelem % 8 == 0 &&
                         s.nelem < (int64_t(1) << 29) && tensor_map_encoder() != nullptr;
  if (tma_shape) {
    for (int tr = 0; tr < 2; ++tr) {
      DGOP_CUDA(cudaMalloc(&K.d_eflags[tr], sizeof(uint32_t) * s.nelem));
      DGOP_CUDA(cudaMalloc(&K.d_gwords[tr], sizeof(uint32_t) * (s.nelem / 8)));
      KronParams<Real> q = tr ? K.params_t : p;
      q.flags = op->flags | (tr ? kTranspose : 0);
      entry->face_words(q, K.d_eflags[tr], K.d_gwords[tr], 0);
      DGOP_CUDA(cudaGetLastError());
    }
    DGOP_CUDA(cudaMalloc(&K.d_err, sizeof(int)));
    DGOP_CUDA(cudaMemset(K.d_err, 0, sizeof(int)));
    DGOP_CUDA(cudaDeviceSynchronize());
  }
  int usable = 0;
  for (int v = 0; v < kKronVariants; ++v) {
    const KronVariant<Real>& kv = entry->v[v];
    auto& L = K.launch[v];
    L.ok = false;
    if (!kv.launch && !(kv.launch_tma && tma_shape)) continue;
    const int threads = kv.threads, warps = threads / 32;
    L.block = dim3(threads);
    L.smem = kv.launch_tma ? (size_t)kv.warp_smem : (size_t)warps * kv.warp_smem * sizeof(Real);
    if ((int)L.smem > max_smem - 1024) continue;  // 1 KB covers every variant's static shared memory
    int arc = allow_dynamic_smem(kv.func, max_smem);
    if (arc == DGOP_OK) arc = allow_dynamic_smem(kv.func_sep, max_smem);
    for (const void* f : kv.func_dot)
      if (arc == DGOP_OK && f) arc = allow_dynamic_smem(f, max_smem);
    for (const auto& by_dot : kv.func_masked)
      for (const auto& by_sep : by_dot)
        for (const void* f : by_sep)
          if (arc == DGOP_OK && f) arc = allow_dynamic_smem(f, max_smem);
    if (arc != DGOP_OK) return arc;
    // resident CTAs per SM of the kernels this operator launches (the slot-mask form when its
    // mask has one), plain and with the inner-product epilogue: each gets a grid of that many
    const int mi = kron_mask_index(p);
    const void* kern[2] = {sep ? kv.func_sep : kv.func, kv.func_dot[sep ? 1 : 0]};
    for (int dot = 0; dot < 2; ++dot)
      if (mi >= 0 && kv.func_masked[mi][dot][sep ? 1 : 0]) kern[dot] = kv.func_masked[mi][dot][sep ? 1 : 0];
    int per_sm = 0, per_sm_dot = 0;
    DGOP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern[0], threads, L.smem));
    if (per_sm < 1) continue;
    if (kern[1]) DGOP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_dot, kern[1], threads, L.smem));
    if (per_sm_dot < 1) per_sm_dot = per_sm;
    const int64_t need = (groups + warps - 1) / warps, sms = device_sm_count(op->device);
    L.grid = dim3((unsigned)std::max<int64_t>(std::min<int64_t>(need, sms * per_sm), 1));
    L.grid_dot = dim3((unsigned)std::max<int64_t>(std::min<int64_t>(need, sms * per_sm_dot), 1));
    L.ok = true;
    ++usable;
  }
  K.fallback = K.launch[1].ok ? 1 : 0;
  if (!usable) {
    set_error("Kronecker kernel shared memory exceeds the device limit");
    return DGOP_ERR_UNSUPPORTED;
  }
  K.variant = 0;
  while (!K.launch[K.variant].ok) ++K.variant;
  K.ready = true;
  return DGOP_OK;
}

// Autotuner decisions, shared by the operators of one kernel shape: (kernel family, dimension, N,
// quadrature, precision, term structure, usable variants, element count within a factor 8).  The first operator of a shape is
// timed; later ones take its variant (dgop_operator_set_variant(-1) times again and replaces it).
struct TuneKey {
  int family, D, N, Q, precision, structure, usable, size_class;
  bool operator<(const TuneKey& o) const {
    return std::tie(family, D, N, Q, precision, structure, usable, size_class) <
           std::tie(o.family, o.D, o.N, o.Q, o.precision, o.structure, o.usable, o.size_class);
  }
};
struct TuneRecord {
  int variant = 0, fallback = 1;
  float ms[8] = {};
};
std::mutex g_tune_mutex;
std::map<TuneKey, TuneRecord> g_tune_cache;
thread_local bool g_tune_force = false;  // set by dgop_operator_set_variant(-1)

template <typename Real>
TuneKey tune_key(const dgop_operator* op, int family, int usable, int has_adv, int has_mass, int merged) {
  // element counts in classes of a factor 8 (launch shapes and tails change with the size)
  int size_class = 0;
  for (int64_t e = op->sp.nelem; e >= 8; e /= 8) ++size_class;
  return TuneKey{family, op->sp.D, op->sp.n, op->q, (int)sizeof(Real),
                 (op->flags & (kAdvCell | kFaceInt | kFaceBnd | kInvMass | kMass)) | (has_adv << 8) |
                     (has_mass << 9) | (merged << 10),
                 usable, size_class};
}

// Autotuner: times every usable kernel variant of the operator on scratch vectors (three
// launches after one warm-up, CUDA events) and keeps the fastest.  Operators above
// kTuneMaxDofs keep the default variant (the scratch vectors would cost more than they save).
constexpr int64_t kTuneMaxDofs = int64_t(1) << 26;

template <typename Real>
int autotune_kron(dgop_operator* op, KronCfg<Real>& K) {
  int usable = 0, mask = 0;
  for (int v = 0; v < kKronVariants; ++v) {
    usable += K.launch[v].ok ? 1 : 0;
    mask |= K.launch[v].ok ? 1 << v : 0;
  }
  if (!K.ready || usable < 2 || op->sp.ndofs > kTuneMaxDofs) return DGOP_OK;
  const TuneKey key = tune_key<Real>(op, 0, mask, K.params.has_adv, K.params.has_mass, K.params.mass_merged);
  if (!g_tune_force) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      K.variant = it->second.variant;
      K.fallback = it->second.fallback;
      for (int v = 0; v < kKronVariants; ++v) K.launch[v].ms = it->second.ms[v];
      return DGOP_OK;
    }
  }
  const int64_t n = op->sp.ndofs;
  Real* x = nullptr;
  Real* y = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int best = K.variant;
  float best_ms = 0.0f;
  bool ok = cudaMalloc(&x, sizeof(Real) * n) == cudaSuccess && cudaMalloc(&y, sizeof(Real) * n) == cudaSuccess &&
            cudaMemset(x, 0, sizeof(Real) * n) == cudaSuccess && cudaEventCreate(&e0) == cudaSuccess &&
            cudaEventCreate(&e1) == cudaSuccess;
  for (int v = 0; ok && v < kKronVariants; ++v) {
    auto& L = K.launch[v];
    if (!L.ok) continue;
    KronParams<Real> p = K.params;
    p.x = x;
    p.y = y;
    p.alpha = Real(1);
    p.beta_y = Real(0);
    p.flags = op->flags;
    p.skip = nullptr;
    ok = launch_kron(op, K, v, p, 0) == DGOP_OK;
    cudaEventRecord(e0, 0);
    for (int r = 0; ok && r < 3; ++r) ok = launch_kron(op, K, v, p, 0) == DGOP_OK;
    cudaEventRecord(e1, 0);
    ok = ok && cudaEventSynchronize(e1) == cudaSuccess && cudaGetLastError() == cudaSuccess;
    float ms = 0.0f;
    if (ok) cudaEventElapsedTime(&ms, e0, e1);
    L.ms = ms / 3.0f;
    if (ok && (best_ms == 0.0f || L.ms < best_ms)) {
      best_ms = L.ms;
      best = v;
    }
    if (ok && !K.entry->v[v].launch_tma && (K.launch[K.fallback].ms == 0.0f || L.ms < K.launch[K.fallback].ms))
      K.fallback = v;
  }
  if (x) cudaFree(x);
  if (y) cudaFree(y);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (!ok) {
    cudaGetLastError();
    return DGOP_OK;  // keep the default variant
  }
  K.variant = best;
  TuneRecord rec;
  rec.variant = best;
  rec.fallback = K.fallback;
  for (int v = 0; v < kKronVariants; ++v) rec.ms[v] = K.launch[v].ms;
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  g_tune_cache[key] = rec;
  return DGOP_OK;
}

// BF16 bits of a finite float, rounded to nearest even.
uint16_t to_bf16_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, sizeof(u));
  return (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
}

// Kronecker tiles of the tensor-core variant (kronnd_tc_kernel.cuh): for every term and half of
// the axes, the product of the term's tangential matrices over the half's axes (the identity on
// the term's own axis), one tile per combination of coordinates along the half's axes whose
// matrices vary, scaled by its largest magnitude, as BF16 in a P x (P + 8) padded tile.  Returns
// false (no tensor-core launch) when the tables would exceed 256 MB.
bool build_tc_tiles(const dgop_space& s, const KronPlanHost& plan, KronNDCfg<float>& K) {
  const int D = s.D, N = s.n, H = D / 2;
  int F = 1;
  for (int k = 0; k < H; ++k) F *= N;
  const int P = F <= 16 ? 16 : 32, LD = P + 8;
  auto& p = K.params;
  std::vector<int> terms;
  if (plan.has_adv)
    for (int t = 0; t < D; ++t) terms.push_back(t);
  if (plan.has_mass && !(plan.has_adv && plan.mass_merged)) terms.push_back(D);
  int64_t count = 0;
  for (int t : terms)
    for (int h = 0; h < 2; ++h) {
      const int ax = t < D ? t : D - 1;
      p.tc_base[t][h] = (int)count;
      int64_t mult = 1;
      for (int k = h * H; k < h * H + H; ++k) {
        const KronMat m = t < D ? (k == t ? plan.D[t] : plan.T[t][k]) : (k == D - 1 ? plan.MD : plan.MT[k]);
        p.tc_mult[t][k] = 0;
        if (k != ax && m.off >= 0 && m.stride != 0) {
          p.tc_mult[t][k] = (int)mult;
          mult *= s.sizes[k];
        }
      }
      count += mult;
    }
  const size_t tile = (size_t)P * LD;
  if (count * tile * 2 > (size_t)256 << 20) return false;
  std::vector<uint16_t> tiles((size_t)count * tile, 0);
  std::vector<float> scales((size_t)count, 0.0f);
  std::vector<double> val((size_t)F * F);
  for (int t : terms)
    for (int h = 0; h < 2; ++h) {
      const int ax = t < D ? t : D - 1;
      const int lo = h * H;
      int64_t combos = 1;
      for (int k = lo; k < lo + H; ++k)
        if (p.tc_mult[t][k]) combos *= s.sizes[k];
      for (int64_t cb = 0; cb < combos; ++cb) {
        int64_t c[kMaxDim] = {};
        int64_t rem = cb;
        for (int k = lo; k < lo + H; ++k)
          if (p.tc_mult[t][k]) {
            c[k] = rem % s.sizes[k];
            rem /= s.sizes[k];
          }
        double mx = 0.0;
        for (int r = 0; r < F; ++r)
          for (int q = 0; q < F; ++q) {
            double v = 1.0;
            int rr = r, qq = q;
            for (int k = lo; k < lo + H; ++k) {
              const int i = rr % N, j = qq % N;
              rr /= N;
              qq /= N;
              const KronMat m = t < D ? (k == t ? plan.D[t] : plan.T[t][k]) : (k == D - 1 ? plan.MD : plan.MT[k]);
              if (k == ax) v *= (i == j) ? 1.0 : 0.0;
              else v *= m.off >= 0 ? plan.mats[(size_t)(m.off + c[k] * m.stride + i * N + j)] : 0.0;
            }
            val[(size_t)r * F + q] = v;
            mx = std::max(mx, std::fabs(v));
          }
        const int64_t id = p.tc_base[t][h] + cb;
        scales[(size_t)id] = (float)mx;
        uint16_t* dst = tiles.data() + (size_t)id * tile;
        for (int r = 0; r < F; ++r)
          for (int q = 0; q < F; ++q) dst[(size_t)r * LD + q] = to_bf16_bits(mx > 0 ? (float)(val[(size_t)r * F + q] / mx) : 0.0f);
      }
    }
  if (cudaMalloc(&K.d_tc_tiles, tiles.size() * sizeof(uint16_t)) != cudaSuccess ||
      cudaMalloc(&K.d_tc_scale, scales.size() * sizeof(float)) != cudaSuccess ||
      cudaMemcpy(K.d_tc_tiles, tiles.data(), tiles.size() * sizeof(uint16_t), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(K.d_tc_scale, scales.data(), scales.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  p.tc_tiles = K.d_tc_tiles;
  p.tc_scale = K.d_tc_scale;
  return true;
}

// Any-dimension Kronecker kernel: matrix tables, face tables and launch shape.
// The paired variant's condition (kronnd_paired_kernel): even D, every term pair (a, a + D/2)
// with the same factor tables on the other D - 2 axes, and a separate mass term with the last
// pair's factors outside that pair.  Compared value by value over every element coordinate.
bool pairs_share_factors(const KronPlanHost& plan, const dgop_space& s) {
  const int D = s.D, N = s.n;
  if (D % 2 || D < 2) return false;
  const int H = D / 2;
  auto same = [&](const KronMat& x, const KronMat& y, int k) {
    if (x.off < 0 || y.off < 0) return false;
    const int64_t count = (x.stride || y.stride) ? s.sizes[k] : 1;
    for (int64_t e = 0; e < count; ++e)
      for (int q = 0; q < N * N; ++q)
        if (plan.mats[x.off + e * x.stride + q] != plan.mats[y.off + e * y.stride + q]) return false;
    return true;
  };
  if (plan.has_adv)
    for (int a = 0; a < H; ++a)
      for (int k = 0; k < D; ++k)
        if (k != a && k != a + H && !same(plan.T[a][k], plan.T[a + H][k], k)) return false;
  if (plan.has_adv && plan.has_mass && !plan.mass_merged)
    for (int k = 0; k < D; ++k)
      if (k != H - 1 && k != D - 1 && !same(plan.MT[k], plan.T[H - 1][k], k)) return false;
  return true;
}

template <typename Real>
int setup_kronnd(dgop_operator* op, KronNDCfg<Real>& K, const KronPlanHost& plan, const double* elem_sigma,
                 const double* const* elem_beta) {
  const dgop_space& s = op->sp;
  const int D = s.D, N = s.n;
  const KronNDEntry<Real>* entry = nullptr;
  if constexpr (sizeof(Real) == 8) entry = &kronnd_slot_f64(D, N);
  else entry = &kronnd_slot_f32(D, N);
  if (!entry->launch) {
    set_error("no any-dimension Kronecker kernel for this shape");
    return DGOP_ERR_UNSUPPORTED;
  }
  K.entry = entry;
  KronNDParams<Real>& p = K.params;
  std::memset(&p, 0, sizeof(p));
  p.nelem = s.nelem;
  int64_t stride = 1;
  for (int k = 0; k < D; ++k) {
    p.sizes[k] = s.sizes[k];
    p.estride[k] = stride;
    stride *= s.sizes[k];
    p.periodic[k] = s.periodic[k];
  }
  p.flags = op->flags;
  p.has_adv = plan.has_adv;
  p.has_mass = plan.has_mass;
  p.mass_merged = plan.mass_merged;
  p.g = (Real)op->g;
  int rc = upload<Real>(&K.d_mats, plan.mats.data(), plan.mats.size());
  if (rc) return rc;
  p.mats = K.d_mats;
  for (int a = 0; a < kMaxDim; ++a) {
    for (int k = 0; k < kMaxDim; ++k) p.slot[a][k] = KronMat{};
    p.mslot[a] = KronMat{};
  }
  if (plan.has_adv) {
    for (int a = 0; a < D; ++a)
      for (int k = 0; k < D; ++k) p.slot[a][k] = (k == a) ? plan.D[a] : plan.T[a][k];
    std::vector<double> phi;
    std::vector<signed char> sg;
    size_t phi_off[kMaxDim], sg_off[kMaxDim][kMaxDim];
    for (int a = 0; a < D; ++a) {
      phi_off[a] = phi.size();
      phi.insert(phi.end(), plan.phi[a].begin(), plan.phi[a].end());
      for (int k = 0; k < D; ++k) {
        sg_off[a][k] = sg.size();
        sg.insert(sg.end(), plan.sgn[a][k].begin(), plan.sgn[a][k].end());
      }
    }
    rc = upload<Real>(&K.d_phi, phi.data(), phi.size());
    if (rc) return rc;
    DGOP_CUDA(cudaMalloc(&K.d_sgn, sg.size() ? sg.size() : 1));
    if (!sg.empty()) DGOP_CUDA(cudaMemcpy(K.d_sgn, sg.data(), sg.size(), cudaMemcpyHostToDevice));
    for (int a = 0; a < D; ++a) {
      p.phi[a] = K.d_phi + phi_off[a];
      for (int k = 0; k < D; ++k) p.sgn[a][k] = (k == a) ? nullptr : K.d_sgn + sg_off[a][k];
    }
  }
  if (plan.has_mass && !(plan.has_adv && plan.mass_merged)) {
    p.mslot[D - 1] = plan.MD;
    for (int k = 0; k < D - 1; ++k) p.mslot[k] = plan.MT[k];
  }
  auto elem_ptr = [&](const double* src, int slot, const Real** dst) -> int {
    *dst = nullptr;
    if (!src) return DGOP_OK;
    if constexpr (sizeof(Real) == 8) {
      *dst = src;
    } else {
      DGOP_CUDA(cudaMalloc(&K.d_elem[slot], sizeof(Real) * s.nelem));
      convert_kernel<Real><<<256, 256>>>(src, K.d_elem[slot], s.nelem);
      DGOP_CUDA(cudaGetLastError());
      *dst = K.d_elem[slot];
    }
    return DGOP_OK;
  };
  for (int a = 0; a < D; ++a)
    if ((rc = elem_ptr(plan.has_adv ? elem_beta[a] : nullptr, a, &p.elem[a]))) return rc;
  if ((rc = elem_ptr(plan.has_mass ? elem_sigma : nullptr, kMaxDim, &p.elem_mass))) return rc;
  // elements per CTA: a power of two (the CTA's threads split into equal groups, one per element)
  // as large as fits in ~96 KB, at most 64, and no larger than needed to give every thread a line
  const size_t per = (size_t)entry->per_elem * sizeof(Real);
  int eb = 1;
  while (eb < 64 && per * (eb * 2) <= 96 * 1024) eb *= 2;
  const int64_t lines = (int64_t)(s.ndofs / s.nelem) / N;
  while (eb > 1 && (int64_t)(eb / 2) * lines >= kKronNDThreads) eb /= 2;
  int max_smem = 0;
  DGOP_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, op->device));
  cudaFuncAttributes fa{};
  DGOP_CUDA(cudaFuncGetAttributes(&fa, entry->func));
  max_smem -= (int)fa.sharedSizeBytes;  // the kernel's static shared memory counts against the limit
  while (eb > 1 && per * eb > (size_t)max_smem) eb /= 2;
  if (per * eb > (size_t)max_smem) {
    set_error("element does not fit in shared memory");
    return DGOP_ERR_UNSUPPORTED;
  }
  p.eb = eb;
  K.params_t = p;
  if (plan.has_adv)
    for (int a = 0; a < D; ++a) K.params_t.slot[a][a] = plan.Dt[a];
  K.block = dim3(kKronNDThreads);
  K.smem = per * eb;
  DGOP_CUDA(cudaFuncSetAttribute(entry->func, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem));
  int per_sm = 0;
  DGOP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, entry->func, kKronNDThreads, K.smem));
  if (per_sm < 1) {
    set_error("any-dimension Kronecker kernel cannot be resident");
    return DGOP_ERR_UNSUPPORTED;
  }
  const int64_t ctas = std::min<int64_t>((s.nelem + eb - 1) / eb, (int64_t)device_sm_count(op->device) * per_sm);
  K.grid = dim3((unsigned)std::max<int64_t>(ctas, 1));
  K.var[0] = {true, eb, K.grid, K.smem, 0.0f, kKronNDThreads};
  // grouped variants: elements per CTA so that the blocks of the largest group give every
  // thread about one block, within ~110 KB of shared memory (two CTAs per SM)
  const bool paired = pairs_share_factors(plan, s);
  // the mass-only variant (4): operators without advection terms, its own smaller layout
  for (int v = 1; v < kKronNDVariants; ++v) {
    const bool mass_only = v == 4;
    const int G = mass_only ? entry->mass_g : (v == 3 ? 2 : v + 1);  // paired blocks span two axes
    const void* fn = mass_only ? entry->func_m : entry->func_g[v - 1];
    if (!fn || (v == 3 && !paired) || (mass_only && (plan.has_adv || !plan.has_mass))) continue;
    // the mass-only kernel holds two batches (the next one's input arrives during this one's passes)
    // and one copy of the D mass matrices when they are the same for every element
    const size_t pv = mass_only ? 2 * (size_t)entry->per_elem_m * sizeof(Real) : per;
    const size_t extra = mass_only ? (size_t)D * ((N * N + 3) / 4 * 4) * sizeof(Real) : 0;
    int64_t gsz = 1;
    for (int k = 0; k < std::min(G, D); ++k) gsz *= N;
    const int64_t ipe = (s.ndofs / s.nelem) / gsz;  // blocks per element
    // the mass-only kernel: 128 threads, whole blocks of 3 axes for every thread
    const int threads = mass_only ? 128 : kKronNDThreads;
    int ebv = mass_only ? (int)std::max<int64_t>(1, std::min<int64_t>(64, threads / ipe))
                        : (int)std::max<int64_t>(1, std::min<int64_t>(64, (kKronNDThreads + ipe / 2) / ipe));
    while (ebv > 1 && pv * ebv + extra > std::min<size_t>((size_t)max_smem, 110 * 1024)) --ebv;
    if (pv * ebv + extra > (size_t)max_smem) continue;
    cudaFuncAttributes fv{};
    if (cudaFuncGetAttributes(&fv, fn) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    int max_v = 0;
    DGOP_CUDA(cudaDeviceGetAttribute(&max_v, cudaDevAttrMaxSharedMemoryPerBlockOptin, op->device));
    max_v -= (int)fv.sharedSizeBytes;
    if (pv * ebv + extra > (size_t)max_v) continue;
    DGOP_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, max_v));
    int per_sm_v = 0;
    DGOP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_v, fn, threads, pv * ebv + extra));
    if (per_sm_v < 1) continue;
    const int64_t cv = std::min<int64_t>((s.nelem + ebv - 1) / ebv, (int64_t)device_sm_count(op->device) * per_sm_v);
    K.var[v] = {true, ebv, dim3((unsigned)std::max<int64_t>(cv, 1)), pv * ebv + extra, 0.0f, threads};
  }
  K.variant = 0;
  if constexpr (sizeof(Real) == 4) {
    if (entry->launch_tc && build_tc_tiles(s, plan, K)) {
      // the transposed parameters share the tangential matrices, hence the tiles
      K.params_t.tc_tiles = K.params.tc_tiles;
      K.params_t.tc_scale = K.params.tc_scale;
      std::memcpy(K.params_t.tc_base, K.params.tc_base, sizeof(K.params.tc_base));
      std::memcpy(K.params_t.tc_mult, K.params.tc_mult, sizeof(K.params.tc_mult));
      const size_t tsm = (size_t)entry->tc_warp_bytes * (kKronTCThreads / 32);
      cudaFuncAttributes ft{};
      int max_t = 0;
      if (cudaFuncGetAttributes(&ft, entry->func_tc) == cudaSuccess &&
          cudaDeviceGetAttribute(&max_t, cudaDevAttrMaxSharedMemoryPerBlockOptin, op->device) == cudaSuccess &&
          tsm + ft.sharedSizeBytes <= (size_t)max_t &&
          cudaFuncSetAttribute(entry->func_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               max_t - (int)ft.sharedSizeBytes) == cudaSuccess) {
        int per_sm_t = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_t, entry->func_tc, kKronTCThreads, tsm) ==
                cudaSuccess &&
            per_sm_t >= 1) {
          const int64_t ct = std::min<int64_t>((s.nelem + kKronTCThreads / 32 - 1) / (kKronTCThreads / 32),
                                               (int64_t)device_sm_count(op->device) * per_sm_t);
          K.tc_grid = dim3((unsigned)std::max<int64_t>(ct, 1));
          K.tc_smem = tsm;
          K.tc_ok = true;
        }
      }
      cudaGetLastError();
    }
  }
  K.ready = true;
  return DGOP_OK;
}

// Launch of the any-dimension kernel's variant v with parameters p (p.eb set here).
template <typename Real>
void launch_kronnd_variant(const KronNDCfg<Real>& K, int v, KronNDParams<Real> p, cudaStream_t st) {
  const auto& L = K.var[v];
  p.eb = L.eb;
  if (v == 0) K.entry->launch(p, L.grid, K.block, L.smem, st);
  else if (v == 4) K.entry->launch_m(p, L.grid, dim3(L.threads), L.smem, st);
  else K.entry->launch_g[v - 1](p, L.grid, K.block, L.smem, st);
}

// Time every usable variant on scratch vectors over the first elements (at most kTuneElems, so
// that the cost stays bounded on large meshes) and keep the fastest.
constexpr int64_t kTuneElems = 65536;
template <typename Real>
int autotune_kronnd(dgop_operator* op, KronNDCfg<Real>& K) {
  int usable = 0, mask = 0;
  for (int v = 0; v < kKronNDVariants; ++v) {
    usable += K.var[v].ok ? 1 : 0;
    mask |= K.var[v].ok ? 1 << v : 0;
  }
  if (!K.ready || usable < 2) return DGOP_OK;
  const TuneKey key = tune_key<Real>(op, 1, mask, K.params.has_adv, K.params.has_mass, K.params.mass_merged);
  if (!g_tune_force) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      K.variant = it->second.variant;
      for (int v = 0; v < kKronNDVariants; ++v) K.var[v].ms = it->second.ms[v];
      return DGOP_OK;
    }
  }
  const int64_t n = op->sp.ndofs;
  Real* x = nullptr;
  Real* y = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int best = K.variant;
  float best_ms = 0.0f;
  bool ok = cudaMalloc(&x, sizeof(Real) * n) == cudaSuccess && cudaMalloc(&y, sizeof(Real) * n) == cudaSuccess &&
            cudaMemset(x, 0, sizeof(Real) * n) == cudaSuccess && cudaEventCreate(&e0) == cudaSuccess &&
            cudaEventCreate(&e1) == cudaSuccess;
  for (int v = 0; ok && v < kKronNDVariants; ++v) {
    auto& L = K.var[v];
    if (!L.ok) continue;
    KronNDParams<Real> p = K.params;
    p.x = x;
    p.y = y;
    p.alpha = Real(1);
    p.beta_y = Real(0);
    p.skip = nullptr;
    p.e_begin = 0;
    p.nelem = std::min<int64_t>(op->sp.nelem, kTuneElems);
    launch_kronnd_variant(K, v, p, 0);
    cudaEventRecord(e0, 0);
    for (int r = 0; r < 3; ++r) launch_kronnd_variant(K, v, p, 0);
    cudaEventRecord(e1, 0);
    ok = cudaEventSynchronize(e1) == cudaSuccess && cudaGetLastError() == cudaSuccess;
    float ms = 0.0f;
    if (ok) cudaEventElapsedTime(&ms, e0, e1);
    L.ms = ms / 3.0f;
    if (ok && (best_ms == 0.0f || L.ms < best_ms)) {
      best_ms = L.ms;
      best = v;
    }
  }
  if (x) cudaFree(x);
  if (y) cudaFree(y);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (!ok) {
    cudaGetLastError();
    return DGOP_OK;  // keep the default variant
  }
  K.variant = best;
  TuneRecord rec;
  rec.variant = best;
  for (int v = 0; v < kKronNDVariants; ++v) rec.ms[v] = K.var[v].ms;
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  g_tune_cache[key] = rec;
  return DGOP_OK;
}

template <typename Real>
void free_kronnd(KronNDCfg<Real>& K) {
  if (K.d_tc_tiles) cudaFree(K.d_tc_tiles);
  if (K.d_tc_scale) cudaFree(K.d_tc_scale);
  if (K.d_mats) cudaFree(K.d_mats);
  if (K.d_phi) cudaFree(K.d_phi);
  if (K.d_sgn) cudaFree(K.d_sgn);
  for (auto* p : K.d_elem)
    if (p) cudaFree(p);
  K = KronNDCfg<Real>{};
}

template <typename Real>
void free_kron(KronCfg<Real>& K) {
  for (int tr = 0; tr < 2; ++tr) {
    if (K.d_eflags[tr]) cudaFree(K.d_eflags[tr]);
    if (K.d_gwords[tr]) cudaFree(K.d_gwords[tr]);
  }
  if (K.d_err) cudaFree(K.d_err);
  if (K.d_mats) cudaFree(K.d_mats);
  if (K.d_phi) cudaFree(K.d_phi);
  if (K.d_sgn) cudaFree(K.d_sgn);
  for (auto* p : K.d_elem)
    if (p) cudaFree(p);
  K = KronCfg<Real>{};
}

template <typename Real>
void free_launch(LaunchCfg<Real>& L) {
  if (L.d_tab) cudaFree(L.d_tab);
  if (L.d_scratch) cudaFree(L.d_scratch);
  for (auto* p : L.d_elem)
    if (p) cudaFree(p);
  L = LaunchCfg<Real>{};
}

int create_operator(const dgop_space* space, int q, const dgop_coef* sigma, const dgop_coef* beta, int flags,
                    double g, dgop_operator** out) {
  if (!space || !out) {
    set_error("null space or output handle");
    return DGOP_ERR_ARG;
  }
  *out = nullptr;
  if (q < 1 || q > kMaxQ) {
    set_error("q must be in [1, 8]");
    return DGOP_ERR_ARG;
  }
  if ((flags & (kAdvCell | kFaceInt | kFaceBnd)) && !beta) {
    set_error("advection needs a velocity coefficient (dim entries)");
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
  op->flags = flags;
  op->g = g;
  cudaGetDevice(&op->device);
  Tables1D t;
  if (!make_tables(op->sp, q, t)) {
    delete op;
    set_error("basis tables");
    return DGOP_ERR_ARG;
  }
  std::vector<double> pack;
  PackedCoef sig, bet[kMaxDim];
  dgop_coef one{};
  one.constant = 1.0;
  int rc = pack_coef(op->sp, q, (flags & kMass) ? (sigma ? sigma : &one) : nullptr, pack, sig);
  for (int k = 0; rc == DGOP_OK && k < op->sp.D; ++k)
    rc = pack_coef(op->sp, q, (flags & (kAdvCell | kFaceInt | kFaceBnd)) ? &beta[k] : nullptr, pack, bet[k]);
  std::string generic_err;
  if (rc == DGOP_OK && (flags & kInvMass)) {
    generic_err = "the mass inverse needs the Kronecker form (GLL basis, separable density, no per-element factor)";
  } else if (rc == DGOP_OK) {
    rc = setup_launch<double>(op, op->f64, t, pack, sig, bet);
    if (rc == DGOP_ERR_UNSUPPORTED) {
      // no generic instantiation for this shape: acceptable when the Kronecker kernel covers it
      generic_err = g_last_error;
      free_launch(op->f64);
      rc = DGOP_OK;
    } else if (rc == DGOP_OK) {
      // FP32 path is optional: absent instantiations only disable dgop_apply_f32.
      const int rc32 = setup_launch<float>(op, op->f32, t, pack, sig, bet);
      if (rc32 != DGOP_OK) {
        free_launch(op->f32);
        set_error("");
      }
    }
  }
  if (rc != DGOP_OK) {
    free_launch(op->f64);
    free_launch(op->f32);
    delete op;
    return rc;
  }
  // Kronecker form, when the coefficients and basis allow it (see kron.h)
  {
    KronInputs in;
    in.D = op->sp.D;
    in.N = op->sp.n;
    in.Q = q;
    in.gll = op->sp.basis == DGOP_BASIS_GLL;
    in.flags = flags;
    in.sizes = op->sp.sizes;
    in.h = op->sp.h;
    in.B = t.B;
    in.Dq = t.Dq;
    in.wq = t.wq;
    const dgop_coef* sg = (flags & kMass) ? (sigma ? sigma : &one) : nullptr;
    in.sigma = sep_of(sg);
    in.inverse_mass = (flags & kInvMass) != 0;
    const bool adv = (flags & (kAdvCell | kFaceInt | kFaceBnd)) != 0;
    const double* elem_beta[kMaxDim] = {};
    for (int k = 0; k < op->sp.D; ++k) {
      in.beta[k] = sep_of(adv ? &beta[k] : nullptr);
      elem_beta[k] = adv ? beta[k].element_factor : nullptr;
    }
    // any-dimension kernel: every shape the Kronecker form covers (also the 3D register kernel's,
    // where it is an alternative the caller may select)
    KronPlanHost plan_nd = plan_kron(in);
    if (plan_nd.ok && (int64_t)op->sp.nelem < (int64_t(1) << 40)) {
      const double* es = sg ? sg->element_factor : nullptr;
      if (setup_kronnd<double>(op, op->n64, plan_nd, es, elem_beta) == DGOP_OK) {
        if (setup_kronnd<float>(op, op->n32, plan_nd, es, elem_beta) != DGOP_OK) free_kronnd(op->n32);
        op->kernel = DGOP_KERNEL_KRONND;
      } else {
        free_kronnd(op->n64);
      }
      set_error("");
    }
    KronPlanHost plan = plan_kron3d(in);
    if (plan.ok) {
      const double* es = sg ? sg->element_factor : nullptr;
      const int krc = setup_kron<double>(op, op->k64, plan, es, elem_beta);
      if (krc == DGOP_OK) {
        if (setup_kron<float>(op, op->k32, plan, es, elem_beta) != DGOP_OK) free_kron(op->k32);
        op->kernel = DGOP_KERNEL_KRON;
        autotune_kron(op, op->k64);
        autotune_kron(op, op->k32);
      } else {
        free_kron(op->k64);
        op->kron_why = "Kronecker setup failed";
      }
      set_error("");
    } else {
      op->kron_why = plan.why;
    }
  }
  if (op->kernel == DGOP_KERNEL_KRONND) {
    autotune_kronnd(op, op->n64);
    autotune_kronnd(op, op->n32);
  }
  if (!op->f64.ready && !op->k64.ready && !op->n64.ready) {
    free_launch(op->f32);
    free_kron(op->k32);
    free_kronnd(op->n32);
    delete op;
    set_error(generic_err.empty() ? std::string("no kernel for this operator") : generic_err);
    return DGOP_ERR_UNSUPPORTED;
  }
  *out = op;
  return DGOP_OK;
}

}  // namespace

// y[i] = alpha x[i] (+ beta_y y[i]) for i in [i0, i1): the speed-of-light operator.  The body
// moves 16-byte vectors (x and y equally aligned: the copy starts with the scalar head that
// reaches a 16-byte boundary of y); the scalar path covers the rest.
template <typename Real>
__global__ void __launch_bounds__(256) copy_kernel(const Real* __restrict__ x, Real* __restrict__ y, int64_t i0,
                                                   int64_t i1, Real alpha, Real beta_y, const int* skip) {
  if (skip && *skip) return;
  constexpr int V = 16 / sizeof(Real);
  using Vec = typename std::conditional<sizeof(Real) == 8, double2, float4>::type;
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t nth = (int64_t)gridDim.x * blockDim.x;
  const bool same = ((reinterpret_cast<uintptr_t>(x) ^ reinterpret_cast<uintptr_t>(y)) & 15) == 0;
  int64_t head = i0;
  if (same) {
    while (head < i1 && (reinterpret_cast<uintptr_t>(y + head) & 15)) ++head;
  } else {
    head = i1;  // all scalar
  }
  for (int64_t i = i0 + tid; i < head; i += nth) y[i] = beta_y == Real(0) ? alpha * x[i] : alpha * x[i] + beta_y * y[i];
  const int64_t nvec = (i1 - head) / V;
  const Vec* xv = reinterpret_cast<const Vec*>(x + head);
  Vec* yv = reinterpret_cast<Vec*>(y + head);
  for (int64_t k = tid; k < nvec; k += nth) {
    Vec a = xv[k];
    Real* pa = reinterpret_cast<Real*>(&a);
    if (beta_y == Real(0)) {
      if (alpha != Real(1))
#pragma unroll
        for (int j = 0; j < V; ++j) pa[j] *= alpha;
    } else {
      Vec b = yv[k];
      const Real* pb = reinterpret_cast<const Real*>(&b);
#pragma unroll
      for (int j = 0; j < V; ++j) pa[j] = alpha * pa[j] + beta_y * pb[j];
    }
    yv[k] = a;
  }
  for (int64_t i = head + nvec * V + tid; i < i1; i += nth)
    y[i] = beta_y == Real(0) ? alpha * x[i] : alpha * x[i] + beta_y * y[i];
}

template <typename Real>
static int launch_impl(dgop_operator* op, LaunchCfg<Real>& L, KronCfg<Real>& K, KronNDCfg<Real>& KN,
                       KronDiffCfg<Real>& SD, Real alpha, const Real* x, Real beta_y, Real* y, int extra_flags,
                       cudaStream_t s, const int* skip, int64_t e_begin = 0, int64_t e_end = -1,
                       const DotEpilogue* dot = nullptr) {
  if (e_end < 0) e_end = op->sp.nelem;
  if (dot && dot->fused) *dot->fused = false;
  if (!x || !y) {
    set_error("null vector");
    return DGOP_ERR_ARG;
  }
  if (x == y) {
    set_error("in-place apply is not supported (x and y alias)");
    return DGOP_ERR_ARG;
  }
  const uintptr_t ax = reinterpret_cast<uintptr_t>(x), ay = reinterpret_cast<uintptr_t>(y);
  if (ax % sizeof(Real) || ay % sizeof(Real)) {
    set_error("vectors must be aligned to their element size");
    return DGOP_ERR_ARG;
  }
  // the Kronecker kernel stages element blocks with 16-byte copies; other pointers take the
  // generic kernel, or are rejected when the operator has none
  const bool aligned16 = (ax % 16 == 0) && (ay % 16 == 0);
  if (op->kernel == DGOP_KERNEL_KRON && K.ready && !aligned16 && !L.ready) {
    set_error("the Kronecker kernel needs 16-byte aligned vectors and the operator has no generic kernel");
    return DGOP_ERR_ARG;
  }
  const bool linear = (extra_flags & kLinear) != 0;
  extra_flags &= ~kLinear;
  if (op->kernel == DGOP_KERNEL_COPY) {
    const int64_t nd = op->sp.ndofs / op->sp.nelem;
    const int64_t i0 = e_begin * nd, i1 = e_end * nd;
    if (i1 > i0) {
      const int64_t blocks =
          std::max<int64_t>(1, std::min<int64_t>((int64_t)device_sms(op->device) * 8, (i1 - i0 + 2047) / 2048));
      copy_kernel<Real><<<(unsigned)blocks, 256, 0, s>>>(x, y, i0, i1, alpha, beta_y, skip);
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(e, "speed-of-light kernel launch");
    }
    return DGOP_OK;
  }
  if (op->kernel == DGOP_KERNEL_DIFF) {
    if (!SD.ready) {
      set_error("the diffusion operator has no kernel for this precision");
      return DGOP_ERR_UNSUPPORTED;
    }
    if ((extra_flags & kTranspose) && op->ip_sigma != -1.0) {
      set_error("the transposed interior-penalty operator is provided for the symmetric form (sigma = -1) only");
      return DGOP_ERR_UNSUPPORTED;
    }
    KronDiffParams<Real> p = SD.params;  // symmetric for sigma = -1: the transpose is the operator
    p.x = x;
    p.y = y;
    p.alpha = alpha;
    p.beta_y = beta_y;
    p.skip = skip;
    p.e_begin = e_begin;
    p.nelem = e_end;
    SD.entry->launch_diff(p, SD.grid, SD.block, SD.smem, s);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "operator kernel launch");
    return DGOP_OK;
  }
  if (op->kernel == DGOP_KERNEL_KRONND && KN.ready) {
    KronNDParams<Real> p = (extra_flags & kTranspose) ? KN.params_t : KN.params;
    p.x = x;
    p.y = y;
    p.alpha = alpha;
    p.beta_y = beta_y;
    p.flags = op->flags | extra_flags;
    p.skip = skip;
    p.e_begin = e_begin;
    p.nelem = e_end;
    if (linear) p.g = Real(0);
    launch_kronnd_variant(KN, KN.variant, p, s);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "operator kernel launch");
    return DGOP_OK;
  }
  if (op->kernel == DGOP_KERNEL_KRON && K.ready && aligned16) {
    KronParams<Real> p = (extra_flags & kTranspose) ? K.params_t : K.params;
    p.x = x;
    p.y = y;
    p.alpha = alpha;
    p.beta_y = beta_y;
    p.flags = op->flags | extra_flags;
    p.skip = skip;
    p.e_begin = e_begin;
    p.nelem = e_end;
    if (linear) p.g = Real(0);
    p.dot_z = nullptr;
    p.dot_partials = nullptr;
    p.dot_count = 0;
    if constexpr (sizeof(Real) == 8) {
      // the fused inner product needs a 16-byte aligned z and a grid no larger than the reader's
      // partial count (the fallback variant's grid when the element range forces it)
      const bool whole = e_begin % 8 == 0 && e_end % 8 == 0;
      const int v = (K.entry->v[K.variant].launch_tma && !whole) ? K.fallback : K.variant;
      if (dot && dot->z && dot->partials && reinterpret_cast<uintptr_t>(dot->z) % 16 == 0 &&
          (int64_t)K.launch[v].grid_dot.x <= dot->count) {
        p.dot_z = dot->z;
        p.dot_partials = dot->partials;
        p.dot_count = dot->count;
        if (dot->fused) *dot->fused = true;
      }
    }
    return launch_kron(op, K, K.variant, p, s);
  }
  if (!L.ready) {
    set_error("operator has no kernel for this precision");
    return DGOP_ERR_UNSUPPORTED;
  }
  OpParams<Real> p = L.params;
  p.x = x;
  p.y = y;
  p.alpha = alpha;
  p.beta_y = beta_y;
  p.flags = op->flags | extra_flags;
  p.skip = skip;
  p.e_begin = e_begin;
  p.nelem = e_end;
  if (linear) p.g = Real(0);
  L.entry->launch(p, L.grid, L.block, L.smem, s);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "operator kernel launch");
  return DGOP_OK;
}

int launch_f64(dgop_operator* op, double alpha, const double* x, double beta_y, double* y, int extra_flags,
               cudaStream_t s, const int* skip, const DotEpilogue* dot) {
  return launch_impl<double>(op, op->f64, op->k64, op->n64, op->s64, alpha, x, beta_y, y, extra_flags, s, skip, 0,
                             -1, dot);
}

int launch_f32(dgop_operator* op, float alpha, const float* x, float beta_y, float* y, int extra_flags,
               cudaStream_t s, const int* skip) {
  return launch_impl<float>(op, op->f32, op->k32, op->n32, op->s32, alpha, x, beta_y, y, extra_flags, s, skip);
}

int launch_bf16(dgop_operator* op, float alpha, const float* x, float beta_y, float* y, int extra_flags,
                cudaStream_t s, const int* skip) {
  KronNDCfg<float>& K = op->n32;
  if (!K.ready || !K.tc_ok) {
    set_error("no BF16 tensor-core kernel for this operator (it needs the any-dimension Kronecker form, an even "
              "dimension and (p+1)^(D/2) <= 32)");
    return DGOP_ERR_UNSUPPORTED;
  }
  if (!x || !y || x == y) {
    set_error("null or aliasing vectors");
    return DGOP_ERR_ARG;
  }
  if (reinterpret_cast<uintptr_t>(x) % 4 || reinterpret_cast<uintptr_t>(y) % 4) {
    set_error("vectors must be aligned to their element size");
    return DGOP_ERR_ARG;
  }
  const bool linear = (extra_flags & kLinear) != 0;
  extra_flags &= ~kLinear;
  KronNDParams<float> p = (extra_flags & kTranspose) ? K.params_t : K.params;
  p.x = x;
  p.y = y;
  p.alpha = alpha;
  p.beta_y = beta_y;
  p.flags = op->flags | extra_flags;
  p.skip = skip;
  p.e_begin = 0;
  p.nelem = op->sp.nelem;
  if (linear) p.g = 0.0f;
  K.entry->launch_tc(p, K.tc_grid, dim3(kKronTCThreads), K.tc_smem, s);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "tensor-core kernel launch");
  return DGOP_OK;
}

int launch_range_f64(dgop_operator* op, const double* x, double* y, int64_t e_begin, int64_t e_end, cudaStream_t s) {
  return launch_impl<double>(op, op->f64, op->k64, op->n64, op->s64, 1.0, x, 0.0, y, 0, s, nullptr, e_begin, e_end);
}

}  // namespace dgop

using namespace dgop;

extern "C" {

const char* dgop_last_error(void) { return dgop::g_last_error.c_str(); }

const char* dgop_version(void) { return "dgop-b200 0.1 (sm_100a)"; }

int dgop_fill_random(double* out, int64_t n, unsigned seed, double lo, double hi) {
  if (!out || n < 0) {
    set_error("dgop_fill_random: bad arguments");
    return DGOP_ERR_ARG;
  }
  std::mt19937 rng(seed);
  std::uniform_real_distribution<double> dist(lo, hi);
  for (int64_t i = 0; i < n; ++i) out[i] = dist(rng);
  return DGOP_OK;
}

int dgop_space_create(int dim, const int64_t* n_elem, const double* h, const double* origin, const int* periodic,
                      int order, int basis, dgop_space** out) {
  if (!out) {
    set_error("null output handle");
    return DGOP_ERR_ARG;
  }
  *out = nullptr;
  if (dim < 1 || dim > DGOP_MAX_DIM || !n_elem || !h) {
    set_error("dim must be in [1, 6] and n_elem, h non-null");
    return DGOP_ERR_ARG;
  }
  if (order < 0 || order + 1 > kMaxN) {
    set_error("order must be in [0, 7]");
    return DGOP_ERR_ARG;
  }
  if (basis != DGOP_BASIS_GLL && basis != DGOP_BASIS_GL) {
    set_error("basis must be DGOP_BASIS_GLL or DGOP_BASIS_GL");
    return DGOP_ERR_ARG;
  }
  auto* s = new (std::nothrow) dgop_space();
  if (!s) {
    set_error("host allocation failed");
    return DGOP_ERR_ALLOC;
  }
  s->D = dim;
  s->P = order;
  s->n = order + 1;
  s->basis = basis;
  s->nelem = 1;
  int64_t nd = 1;
  for (int k = 0; k < dim; ++k) {
    if (n_elem[k] < 1 || !(h[k] > 0.0) || !std::isfinite(h[k])) {
      delete s;
      set_error("n_elem must be >= 1 and h > 0 on every axis");
      return DGOP_ERR_ARG;
    }
    s->sizes[k] = n_elem[k];
    s->h[k] = h[k];
    s->origin[k] = origin ? origin[k] : 0.0;
    s->periodic[k] = periodic ? (periodic[k] != 0) : 0;
    s->nelem *= n_elem[k];
    nd *= s->n;
  }
  s->ndofs = s->nelem * nd;
  *out = s;
  return DGOP_OK;
}

int dgop_space_destroy(dgop_space* space) {
  delete space;
  return DGOP_OK;
}

int64_t dgop_space_num_dofs(const dgop_space* space) { return space ? space->ndofs : -1; }

int64_t dgop_space_num_elements(const dgop_space* space) { return space ? space->nelem : -1; }

int dgop_space_coordinates(const dgop_space* space, int q, int axis, double* coords) {
  if (!space || !coords || axis < 0 || axis >= space->D || q < 1 || q > kMaxQ) {
    set_error("dgop_space_coordinates: bad arguments");
    return DGOP_ERR_ARG;
  }
  double xq[kMaxQ], wq[kMaxQ];
  gauss_points(1, q, xq, wq);
  const double h = space->h[axis], o = space->origin[axis];
  for (int64_t e = 0; e < space->sizes[axis]; ++e) {
    // X = cell origin + h * xhat (hypercubecell.hpp:41-52, cartesianndmesh.hpp:95-105)
    const double cell = o + h * (double)e;
    for (int j = 0; j < q; ++j) coords[e * (q + 2) + j] = cell + h * xq[j];
    coords[e * (q + 2) + q] = cell + h * 0.0;
    coords[e * (q + 2) + q + 1] = cell + h * 1.0;
  }
  return DGOP_OK;
}

int dgop_mass_create(const dgop_space* space, int q, const dgop_coef* sigma, dgop_operator** out) {
  return create_operator(space, q, sigma, nullptr, kMass, 0.0, out);
}

int dgop_speed_of_light_create(const dgop_space* space, int q, dgop_operator** out) {
  if (!space || !out) {
    set_error("dgop_speed_of_light_create: null argument");
    return DGOP_ERR_ARG;
  }
  *out = nullptr;
  auto* op = new (std::nothrow) dgop_operator();
  if (!op) {
    set_error("host allocation failed");
    return DGOP_ERR_ALLOC;
  }
  op->sp = *space;
  op->q = q;
  op->flags = 0;
  op->kernel = DGOP_KERNEL_COPY;
  op->kron_why = "speed-of-light copy";
  cudaGetDevice(&op->device);
  *out = op;
  return DGOP_OK;
}

int dgop_mass_inverse_create(const dgop_space* space, int q, const dgop_coef* sigma, dgop_operator** out) {
  return create_operator(space, q, sigma, nullptr, kMass | kInvMass, 0.0, out);
}

int dgop_advection_create(const dgop_space* space, int q, const dgop_coef* beta, int bc, double bc_value,
                          dgop_operator** out) {
  if (bc != DGOP_BC_NONE && bc != DGOP_BC_INFLOW) {
    set_error("bc must be DGOP_BC_NONE or DGOP_BC_INFLOW");
    return DGOP_ERR_ARG;
  }
  const int flags = kAdvCell | kFaceInt | (bc == DGOP_BC_INFLOW ? kFaceBnd : 0);
  return create_operator(space, q, nullptr, beta, flags, bc_value, out);
}

int dgop_mass_advection_create(const dgop_space* space, int q, const dgop_coef* sigma, const dgop_coef* beta,
                               dgop_operator** out) {
  return create_operator(space, q, sigma, beta, kMass | kAdvCell | kFaceInt, 0.0, out);
}

int dgop_system_create(const dgop_space* space, int q, const dgop_coef* sigma, const dgop_coef* beta, int bc,
                       double bc_value, dgop_operator** out) {
  if (bc != DGOP_BC_NONE && bc != DGOP_BC_INFLOW) {
    set_error("bc must be DGOP_BC_NONE or DGOP_BC_INFLOW");
    return DGOP_ERR_ARG;
  }
  const int flags = kMass | kAdvCell | kFaceInt | (bc == DGOP_BC_INFLOW ? kFaceBnd : 0);
  return create_operator(space, q, sigma, beta, flags, bc_value, out);
}

int dgop_operator_destroy(dgop_operator* op) {
  if (!op) return DGOP_OK;
  free_launch(op->f64);
  free_launch(op->f32);
  free_kron(op->k64);
  free_kron(op->k32);
  free_kronnd(op->n64);
  free_kronnd(op->n32);
  free_diff(op->s64);
  free_diff(op->s32);
  delete op;
  return DGOP_OK;
}

int64_t dgop_operator_num_dofs(const dgop_operator* op) { return op ? op->sp.ndofs : -1; }

int dgop_operator_kernel(const dgop_operator* op) { return op ? op->kernel : -1; }

const char* dgop_operator_kernel_note(const dgop_operator* op) { return op ? op->kron_why : ""; }

int dgop_operator_select_kernel(dgop_operator* op, int kernel) {
  if (!op || (kernel != DGOP_KERNEL_GENERIC && kernel != DGOP_KERNEL_KRON && kernel != DGOP_KERNEL_KRONND)) {
    set_error("dgop_operator_select_kernel: bad arguments");
    return DGOP_ERR_ARG;
  }
  if (kernel == DGOP_KERNEL_KRON && !op->k64.ready) {
    set_error(std::string("Kronecker kernel unavailable: ") + op->kron_why);
    return DGOP_ERR_UNSUPPORTED;
  }
  if (kernel == DGOP_KERNEL_KRONND && !op->n64.ready) {
    set_error("any-dimension Kronecker kernel unavailable for this operator");
    return DGOP_ERR_UNSUPPORTED;
  }
  if (kernel == DGOP_KERNEL_GENERIC && !op->f64.ready) {
    set_error("generic kernel not built for this shape");
    return DGOP_ERR_UNSUPPORTED;
  }
  op->kernel = kernel;
  ++op->version;
  return DGOP_OK;
}

static bool uses_kronnd(const dgop_operator* op) { return op->kernel == DGOP_KERNEL_KRONND && op->n64.ready; }

int dgop_operator_variant(const dgop_operator* op) {
  if (!op) return -1;
  if (uses_kronnd(op)) return op->n64.variant;
  if (!op->k64.ready) return -1;
  return op->k64.variant;
}

const char* dgop_operator_variant_name(const dgop_operator* op) {
  const int v = dgop_operator_variant(op);
  if (v < 0) return "";
  return uses_kronnd(op) ? kKronNDVariantNames[v] : kKronVariantNames[v];
}

int dgop_operator_set_variant(dgop_operator* op, int variant) {
  if (op && uses_kronnd(op)) {
    if (variant < -1 || variant >= kKronNDVariants) {
      set_error("dgop_operator_set_variant: bad arguments");
      return DGOP_ERR_ARG;
    }
    if (variant == -1) {
      g_tune_force = true;
      autotune_kronnd(op, op->n64);
      autotune_kronnd(op, op->n32);
      g_tune_force = false;
    } else {
      if (!op->n64.var[variant].ok) {
        set_error(std::string("kernel variant ") + kKronNDVariantNames[variant] +
                  " is not available for this operator");
        return DGOP_ERR_UNSUPPORTED;
      }
      op->n64.variant = variant;
      if (op->n32.ready && op->n32.var[variant].ok) op->n32.variant = variant;
    }
    ++op->version;
    return DGOP_OK;
  }
  if (!op || variant < -1 || variant >= kKronVariants) {
    set_error("dgop_operator_set_variant: bad arguments");
    return DGOP_ERR_ARG;
  }
  if (!op->k64.ready) {
    set_error("dgop_operator_set_variant: the operator has no Kronecker kernel");
    return DGOP_ERR_UNSUPPORTED;
  }
  if (variant == -1) {
    g_tune_force = true;
    autotune_kron(op, op->k64);
    autotune_kron(op, op->k32);
    g_tune_force = false;
  } else {
    if (!op->k64.launch[variant].ok) {
      set_error(std::string("kernel variant ") + kKronVariantNames[variant] + " is not available for this operator");
      return DGOP_ERR_UNSUPPORTED;
    }
    op->k64.variant = variant;
    if (op->k32.ready && op->k32.launch[variant].ok) op->k32.variant = variant;
  }
  ++op->version;
  return DGOP_OK;
}

int dgop_operator_variant_f32(const dgop_operator* op, int* variant, float* ms) {
  if (!op || !variant || !ms) {
    set_error("dgop_operator_variant_f32: null argument");
    return DGOP_ERR_ARG;
  }
  if (op->kernel == DGOP_KERNEL_KRONND && op->n32.ready) {
    *variant = op->n32.variant;
    for (int v = 0; v < kKronNDVariants; ++v) ms[v] = op->n32.var[v].ok ? op->n32.var[v].ms : -1.0f;
  } else if (op->kernel == DGOP_KERNEL_KRON && op->k32.ready) {
    *variant = op->k32.variant;
    for (int v = 0; v < kKronVariants; ++v) ms[v] = op->k32.launch[v].ok ? op->k32.launch[v].ms : -1.0f;
  } else {
    for (int v = 0; v < DGOP_MAX_VARIANTS; ++v) ms[v] = -1.0f;
    *variant = -1;
  }
  return DGOP_OK;
}

int dgop_operator_variant_time(const dgop_operator* op, int variant, float* ms) {
  if (op && ms && uses_kronnd(op) && variant >= 0 && variant < kKronNDVariants) {
    *ms = op->n64.var[variant].ms;
    return DGOP_OK;
  }
  if (!op || !ms || variant < 0 || variant >= kKronVariants || !op->k64.ready) {
    set_error("dgop_operator_variant_time: bad arguments");
    return DGOP_ERR_ARG;
  }
  *ms = op->k64.launch[variant].ms;
  return DGOP_OK;
}

static_assert(kKronVariants <= DGOP_MAX_VARIANTS && kKronNDVariants <= DGOP_MAX_VARIANTS, "variant table size");

int dgop_operator_device_error(const dgop_operator* op, int* error) {
  if (!op || !error) {
    set_error("dgop_operator_device_error: null argument");
    return DGOP_ERR_ARG;
  }
  *error = 0;
  for (int* w : {op->k64.d_err, op->k32.d_err}) {
    if (!w) continue;
    int v = 0;
    DGOP_CUDA(cudaMemcpy(&v, w, sizeof(int), cudaMemcpyDeviceToHost));
    if (v) {
      *error |= v;
      DGOP_CUDA(cudaMemset(w, 0, sizeof(int)));
    }
  }
  return DGOP_OK;
}

int dgop_apply(dgop_operator* op, const double* x, double* y, void* stream) {
  if (!op) {
    set_error("null operator");
    return DGOP_ERR_ARG;
  }
  return launch_f64(op, 1.0, x, 0.0, y, 0, (cudaStream_t)stream);
}

int dgop_apply_ex(dgop_operator* op, double alpha, const double* x, double beta, double* y, void* stream) {
  if (!op) {
    set_error("null operator");
    return DGOP_ERR_ARG;
  }
  return launch_f64(op, alpha, x, beta, y, 0, (cudaStream_t)stream);
}

int dgop_apply_bf16(dgop_operator* op, const float* x, float* y, int transpose, void* stream) {
  if (!op) {
    set_error("null operator");
    return DGOP_ERR_ARG;
  }
  return launch_bf16(op, 1.0f, x, 0.0f, y, transpose ? kTranspose : 0, (cudaStream_t)stream, nullptr);
}

int dgop_apply_transpose(dgop_operator* op, const double* x, double* y, void* stream) {
  if (!op) {
    set_error("null operator");
    return DGOP_ERR_ARG;
  }
  return launch_f64(op, 1.0, x, 0.0, y, kTranspose, (cudaStream_t)stream);
}

int dgop_apply_f32(dgop_operator* op, const float* x, float* y, void* stream) {
  if (!op) {
    set_error("null operator");
    return DGOP_ERR_ARG;
  }
  return launch_f32(op, 1.0f, x, 0.0f, y, 0, (cudaStream_t)stream);
}

}  // extern "C"
