// Device-resident Krylov solvers: unpreconditioned CG and restarted GMRES(m) with modified
// Gram-Schmidt, following the reference's algorithms step by step
// (Solvers/conjugategradient.hpp:125-209, Solvers/gmres.hpp:74-289).
//
// Every step is a kernel whose work is predicated on device-side state words (done / inactive),
// so the host enqueues iterations without waiting and reads the state only occasionally (CG:
// every kCheckEvery iterations; GMRES: once per restart cycle).  Iterations enqueued after
// convergence do nothing; the operator kernels take the same word through their `skip` pointer.
// Scalars (alpha, beta, the Hessenberg column, Givens rotations, stopping tests) never leave the
// device.  Inner products are deterministic: a fixed grid writes per-block partial sums with a
// fixed reduction tree, and every consumer sums the partials in the same fixed order.
#include <cuda.h>  // driver API types only; the functions come through cudaGetDriverEntryPointByVersion
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <new>
#include <string>
#include <mutex>
#include <vector>

#include "dgop_internal.h"
#include "gmres_steps.cuh"

namespace dgop {

namespace {

constexpr int kRB = 592;  // reduction blocks (4 per SM on 148 SMs)
constexpr int kRT = 256;  // threads per reduction block
constexpr int kCheckEvery = 8;  // CG iterations per chunk (even)

// Stride of the solvers' workspace vectors: n rounded up to 64 entries, so every vector starts
// 256-byte aligned (the operator kernels stage elements with 16-byte copies).  Padding entries
// are zero from creation on and stay zero.
inline int64_t vec_stride(int64_t n) { return (n + 63) / 64 * 64; }

// Sum over the block in a fixed order; the result is valid in thread 0.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double ws[kRT / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < kRT / 32 ? ws[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  }
  __syncthreads();
  return s;
}

// Sum of the kRB partials in a fixed order, broadcast to every thread of the block.
__device__ __forceinline__ double reduce_partials(const double* __restrict__ partials) {
  __shared__ double res;
  double v = 0.0;
  for (int i = threadIdx.x; i < kRB; i += kRT) v += partials[i];
  const double s = block_sum(v);
  if (threadIdx.x == 0) res = s;
  __syncthreads();
  return res;
}

__device__ __forceinline__ void write_partial(double* partials, double v) {
  const double s = block_sum(v);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

#define DGOP_GRID_LOOP(i, n) for (int64_t i = blockIdx.x * (int64_t)kRT + threadIdx.x; i < (n); i += (int64_t)kRB * kRT)

// partials <- sum a .* b
// (vectors of any precision; products and sums in FP64)
template <typename T>
__global__ void __launch_bounds__(kRT) k_dot(const T* __restrict__ a, const T* __restrict__ b, int64_t n,
                                             double* partials, const int* skip) {
  if (skip && *skip) return;
  double v = 0.0;
  DGOP_GRID_LOOP(i, n) v += (double)a[i] * (double)b[i];
  write_partial(partials, v);
}

// out <- b - w ; partials <- |out|^2   (V[0] = rhs; V[0] -= w, residual = rhs; residual -= tmp)
__global__ void __launch_bounds__(kRT) k_sub_norm(const double* __restrict__ b, const double* __restrict__ w,
                                                  double* __restrict__ out, int64_t n, double* partials,
                                                  const int* skip) {
  if (skip && *skip) return;
  double v = 0.0;
  DGOP_GRID_LOOP(i, n) {
    const double r = b[i] - w[i];
    out[i] = r;
    v += r * r;
  }
  write_partial(partials, v);
}

// ------------------------------------------------------------------------------- CG

struct CGState {
  int done, success, iters, zero_x;
  int base, max_iters, pad_[2];  // base: iteration index of the current chunk's first iteration
  double tol, rhs_n, r_n, rel;
  double abs_[2];  // (r, r) by iteration parity
};

// conjugategradient.hpp:143-165: norms of the initial residual, early exits.
__global__ void __launch_bounds__(kRT) k_cg_init(CGState* st, const double* partials, double tol, int max_iters) {
  const double R = reduce_partials(partials);
  if (threadIdx.x != 0) return;
  st->tol = tol;
  st->max_iters = max_iters;
  st->done = 0;
  st->success = 0;
  st->iters = 0;
  st->zero_x = 0;
  st->base = 0;
  const double rhs_n = sqrt(R);  // the "rhs norm" is the norm of the initial residual
  st->rhs_n = rhs_n;
  if (rhs_n == 0.0 || rhs_n < 1e-30) {
    st->zero_x = 1;
    st->done = 1;
    st->success = 1;
    st->rel = 0.0;
    return;
  }
  const double r_n = sqrt(R);
  st->r_n = r_n;
  if (r_n < tol * rhs_n) {
    st->done = 1;
    st->success = 1;
    st->rel = sqrt(r_n / rhs_n);
    return;
  }
  st->abs_[0] = R;  // dot(residual, p) with p = residual
}

// p <- r ; x <- 0 for a zero right-hand side
__global__ void __launch_bounds__(kRT) k_cg_init_p(const CGState* st, const double* __restrict__ r,
                                                   double* __restrict__ p, double* __restrict__ x, int64_t n) {
  const int zero_x = st->zero_x;
  DGOP_GRID_LOOP(i, n) {
    p[i] = r[i];
    if (zero_x) x[i] = 0.0;
  }
}

// Iterations run in chunks of kCheckEvery; iteration kk of a chunk is iteration st->base + kk
// of the solve (kCheckEvery is even, so the parity of the two agrees).

// alpha = (r, r) / (p, A p); x += alpha p; r -= alpha A p; partials2 <- |r|^2   (:176-181)
__global__ void __launch_bounds__(kRT) k_cg_update(int kk, const CGState* st, double* __restrict__ x,
                                                   double* __restrict__ r, const double* __restrict__ p,
                                                   const double* __restrict__ ap, int64_t n, const double* partials1,
                                                   double* partials2) {
  if (st->done) return;
  const int k = st->base + kk;
  const double alpha = st->abs_[k & 1] / reduce_partials(partials1);
  double v = 0.0;
  DGOP_GRID_LOOP(i, n) {
    x[i] = x[i] + alpha * p[i];
    const double ri = r[i] + (-alpha) * ap[i];
    r[i] = ri;
    v += ri * ri;
  }
  write_partial(partials2, v);
}

// stopping test, beta = (r_new, r_new) / (r_old, r_old), p = beta p + r   (:183-205)
__global__ void __launch_bounds__(kRT) k_cg_finish(int kk, CGState* st, const double* __restrict__ r,
                                                   double* __restrict__ p, int64_t n, const double* partials2) {
  if (st->done) return;
  const int k = st->base + kk;
  const double tol = st->tol;
  const int max_iters = st->max_iters;
  const double R = reduce_partials(partials2);
  const double r_n = sqrt(R);
  const double rhs_n = st->rhs_n;
  if (r_n < tol * rhs_n) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->r_n = r_n;
      st->iters = k + 1;
      st->rel = sqrt(r_n / rhs_n);
      st->success = 1;
      st->done = 1;
    }
    return;
  }
  const double beta = R / st->abs_[k & 1];
  DGOP_GRID_LOOP(i, n) p[i] = p[i] * beta + r[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->abs_[(k + 1) & 1] = R;
    st->r_n = r_n;
    if (k + 1 >= max_iters) {
      st->iters = max_iters;
      st->rel = sqrt(r_n / rhs_n);
      st->success = 0;
      st->done = 1;
    }
  }
}

// end of a chunk: the next chunk starts kCheckEvery iterations later
__global__ void k_cg_next_chunk(CGState* st) {
  if (!st->done) st->base += kCheckEvery;
}

// max_iters == 0 without early exit: the loop does not run (:207-208)
__global__ void k_cg_no_iters(CGState* st) {
  if (st->done) return;
  st->iters = 0;
  st->rel = sqrt(st->r_n / st->rhs_n);
  st->success = 0;
  st->done = 1;
}

// ------------------------------------------------------------------------------- GMRES

__global__ void __launch_bounds__(kRT) k_gm_denom(GMState* st, const double* partials, double tol, int max_iters) {
  const double R = reduce_partials(partials);
  if (threadIdx.x == 0) gm_denom(st, R, tol, max_iters);
}

// true residual and the decisions after it (gm_resid)
__global__ void __launch_bounds__(kRT) k_gm_resid(GMState* st, const double* partials, int phase) {
  if (st->done) return;
  const double R = reduce_partials(partials);
  if (threadIdx.x == 0) gm_resid(st, R, phase);
}

__global__ void k_gm_cycle_start(GMState* st, double* cs, double* sn, double* e1, double* y, int m) {
  gm_cycle_start(st, cs, sn, e1, y, m);
}

// v <- v * s (s = st->inv_h): V[0] *= 1/beta at a cycle start (j < 0) and V[j+1] = w * (1/h_next)
// after iteration j, when that iteration ran and did not end the cycle
template <typename TS, typename TD>
__global__ void __launch_bounds__(kRT) k_gm_scale(const GMState* st, const TS* __restrict__ src,
                                                  TD* __restrict__ dst, int64_t n, int j) {
  if (st->done || (j >= 0 && (st->brk || st->k != j + 1))) return;
  const double s = st->inv_h;
  DGOP_GRID_LOOP(i, n) dst[i] = (TD)((double)src[i] * s);
}

// one modified Gram-Schmidt step (gmres.hpp:160-165), fused with the next inner product:
// h = (V_i, w) from partials_in; H(i, j) = h; w -= h V_i; partials_out <- (next, w)
// (basis vectors of any precision; the update and the product are formed in FP64)
template <typename T>
__global__ void __launch_bounds__(kRT) k_gm_mgs(const GMState* st, int i, int j, int m, const T* __restrict__ vi,
                                                const T* __restrict__ next, T* __restrict__ w, int64_t n,
                                                double* H, const double* partials_in, double* partials_out) {
  if (st->inactive) return;
  const double h = reduce_partials(partials_in);
  if (blockIdx.x == 0 && threadIdx.x == 0) H[j * (m + 1) + i] = h;
  double v = 0.0;
  const bool self = next == w;
  DGOP_GRID_LOOP(l, n) {
    const T wl = (T)((double)w[l] + (-h) * (double)vi[l]);
    w[l] = wl;
    v += (self ? (double)wl : (double)next[l]) * (double)wl;
  }
  write_partial(partials_out, v);
}

// Hessenberg column j (gm_column) from |w|^2 in the partials
__global__ void __launch_bounds__(kRT) k_gm_column(GMState* st, int j, int m, double* H, double* cs, double* sn,
                                                   double* e1, const double* partials) {
  if (st->inactive) return;
  const double R = reduce_partials(partials);
  if (threadIdx.x == 0) gm_column(st, j, m, H, cs, sn, e1, R);
}

__global__ void k_gm_backsub(const GMState* st, const double* H, const double* e1, double* y, int m) {
  gm_backsub(st, H, e1, y, m);
}

// x += y_i V_i for i < k, in order (the reference's sequence of Axpy calls, gmres.hpp:263-267)
template <typename T>
__global__ void __launch_bounds__(kRT) k_gm_update(const GMState* st, double* __restrict__ x,
                                                   const T* __restrict__ V, int64_t ld, const double* y, int64_t n) {
  if (st->done || st->k == 0) return;
  const int k = st->k;
  DGOP_GRID_LOOP(l, n) {
    double xl = x[l];
    for (int i = 0; i < k; ++i) xl = xl + y[i] * (double)V[(int64_t)i * ld + l];
    x[l] = xl;
  }
}

// ---------------------------------------------- GMRES with iterative refinement (inner basis)

constexpr int kGsChunk = 8;     // basis vectors per block row of the projection pass
constexpr int kGsMaxRestart = 1000;

template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  using type = float4;
  static constexpr int L = 4;
};
template <>
struct Vec16<double> {
  using type = double2;
  static constexpr int L = 2;
};

// wide[i * kRB + block] <- partial (V_i, w) for i <= j (blockIdx.y selects kGsChunk vectors);
// 128-bit accesses over the padded stride, products and sums in FP64
template <typename T>
__global__ void __launch_bounds__(kRT) k_gs_dots(const GMState* st, const T* __restrict__ V, int64_t ld, int j,
                                                 const T* __restrict__ w, double* wide) {
  if (st->inactive) return;
  using V16 = typename Vec16<T>::type;
  constexpr int L = Vec16<T>::L;
  const int i0 = blockIdx.y * kGsChunk;
  const int cnt = min(kGsChunk, j + 1 - i0);
  double acc[kGsChunk];
#pragma unroll
  for (int c = 0; c < kGsChunk; ++c) acc[c] = 0.0;
  const int64_t nv = ld / L;
  const V16* w16 = reinterpret_cast<const V16*>(w);
  const V16* v16 = reinterpret_cast<const V16*>(V + (int64_t)i0 * ld);
  const int64_t ldv = ld / L;
  DGOP_GRID_LOOP(u, nv) {
    T wv[L];
    *reinterpret_cast<V16*>(wv) = w16[u];
#pragma unroll
    for (int c = 0; c < kGsChunk; ++c) {
      if (c < cnt) {
        T vv[L];
        *reinterpret_cast<V16*>(vv) = v16[c * ldv + u];
#pragma unroll
        for (int k = 0; k < L; ++k) acc[c] += (double)vv[k] * (double)wv[k];
      }
    }
  }
#pragma unroll
  for (int c = 0; c < kGsChunk; ++c)
    if (c < cnt) write_partial(wide + (int64_t)(i0 + c) * kRB, acc[c]);
}

// H(i, j) <- (V_i, w), one block per i, partials summed in the fixed order
__global__ void __launch_bounds__(kRT) k_gs_h(const GMState* st, int j, int m, double* H, const double* wide) {
  if (st->inactive) return;
  const int i = blockIdx.x;
  const double h = reduce_partials(wide + (int64_t)i * kRB);
  if (threadIdx.x == 0) H[j * (m + 1) + i] = h;
}

// out <- w - sum_{i <= j} H(i, j) V_i (formed in FP64, stored as T); partials <- |out|^2
template <typename T>
__global__ void __launch_bounds__(kRT) k_gs_update(const GMState* st, const T* __restrict__ V, int64_t ld, int j,
                                                   int m, const double* H, const T* __restrict__ w,
                                                   T* __restrict__ out, double* partials) {
  if (st->inactive) return;
  using V16 = typename Vec16<T>::type;
  constexpr int L = Vec16<T>::L;
  __shared__ double hs[kGsMaxRestart];
  for (int i = threadIdx.x; i <= j; i += kRT) hs[i] = H[j * (m + 1) + i];
  __syncthreads();
  const int64_t nv = ld / L, ldv = ld / L;
  const V16* w16 = reinterpret_cast<const V16*>(w);
  const V16* v16 = reinterpret_cast<const V16*>(V);
  V16* o16 = reinterpret_cast<V16*>(out);
  double sq = 0.0;
  DGOP_GRID_LOOP(u, nv) {
    T wv[L];
    *reinterpret_cast<V16*>(wv) = w16[u];
    double a[L];
#pragma unroll
    for (int k = 0; k < L; ++k) a[k] = (double)wv[k];
#pragma unroll 4
    for (int i = 0; i <= j; ++i) {
      T vv[L];
      *reinterpret_cast<V16*>(vv) = v16[(int64_t)i * ldv + u];
      const double h = hs[i];
#pragma unroll
      for (int k = 0; k < L; ++k) a[k] -= h * (double)vv[k];
    }
    T ov[L];
#pragma unroll
    for (int k = 0; k < L; ++k) {
      ov[k] = (T)a[k];
      sq += (double)ov[k] * (double)ov[k];
    }
    o16[u] = *reinterpret_cast<V16*>(ov);
  }
  write_partial(partials, sq);
}

// v <- v * (1 / H(j + 1, j)) in place, when iteration j ran and did not end the cycle
template <typename T>
__global__ void __launch_bounds__(kRT) k_gs_rescale(const GMState* st, T* v, int64_t ld, int j) {
  if (st->done || st->brk || st->k != j + 1) return;
  using V16 = typename Vec16<T>::type;
  constexpr int L = Vec16<T>::L;
  const double sc = st->inv_h;
  V16* v16 = reinterpret_cast<V16*>(v);
  DGOP_GRID_LOOP(u, ld / L) {
    T a[L];
    *reinterpret_cast<V16*>(a) = v16[u];
#pragma unroll
    for (int k = 0; k < L; ++k) a[k] = (T)((double)a[k] * sc);
    v16[u] = *reinterpret_cast<V16*>(a);
  }
}

// ------------------------------------------------------------- per-element inner products

// out[e] = scale[e] * sum_{i in element e} a_i b_i  (one warp per element, fixed summation order)
__global__ void __launch_bounds__(kRT) k_element_dot(const double* __restrict__ a, const double* __restrict__ b,
                                                     const double* __restrict__ scale, double* __restrict__ out,
                                                     int64_t nelem, int64_t nd) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (kRT / 32);
  for (int64_t e = (int64_t)blockIdx.x * (kRT / 32) + (threadIdx.x >> 5); e < nelem; e += warps) {
    const double* pa = a + e * nd;
    const double* pb = b + e * nd;
    double v = 0.0;
    for (int64_t i = lane; i < nd; i += 32) v += pa[i] * pb[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) out[e] = scale ? scale[e] * v : v;
  }
}

}  // namespace

// Whole-solve loop control: loop[0] counts the segments run in this launch, loop[1] is the
// limit.  k_loop_next runs after every segment and keeps the WHILE node going while the solve
// is not done and fewer than loop[1] segments have run, so the loop ends after at most loop[1]
// segments whatever the solver state holds.
__global__ void k_loop_reset(int* loop, int limit) {
  loop[0] = 0;
  loop[1] = limit;
}
__global__ void k_loop_next(cudaGraphConditionalHandle h, const int* done, int* loop) {
  const int c = ++loop[0];
  cudaGraphSetConditional(h, (*done == 0 && c < loop[1]) ? 1u : 0u);
}

// What a captured solver graph depends on besides device state: b, x, the operator's kernel
// selection and flags, and the preconditioner's.
struct GraphKey {
  const void* b = nullptr;
  const void* x = nullptr;
  int version = -1, flags = -1;
  const dgop_operator* prec = nullptr;
  int prec_version = -1;
};

struct SolverImpl {
  int kind = 0;  // 0: CG, 1: GMRES, 2: GMRES with FP32 inner cycles and FP64 refinement
  int restart = 0;
  dgop_operator* op = nullptr;
  int64_t n = 0;
  double* work = nullptr;      // vectors
  double* partials = nullptr;  // 2 x kRB
  void* state = nullptr;       // CGState / GMState (device)
  double* small = nullptr;     // GMRES: H, cs, sn, e1, y
  int* h_flag = nullptr;       // host copies of `done`, one per segment parity (pinned)
  int inner = 0;               // refinement solver: DGOP_FP64, DGOP_FP32 or DGOP_BF16 inner cycles
  double* wide = nullptr;      // refinement solver: (restart + 1) x kRB projection partials
  // Segments (a CG chunk, a GMRES cycle) are replayed from one CUDA graph, captured for the
  // current (b, x, operator version) and re-captured when any of them changes (tolerance and
  // iteration limit are device state).  With `whole`, the solve is ONE graph launch: a
  // conditional WHILE node replays the segment until the solve is done or the segment limit is
  // reached, with no host round trip between segments.
  bool use_graphs = true;
  bool whole = false;
  cudaStream_t cap = nullptr;
  cudaGraphExec_t exec = nullptr;   // one segment
  cudaGraphExec_t wexec = nullptr;  // the whole solve
  GraphKey key, wkey;
  int* loop = nullptr;  // device: segments run, segment limit (whole-solve graphs)
  int op_flags = 0;     // extra operator flags of every apply (kTranspose: solve with A^T)
  // right preconditioner (GMRES): A P z = b, x = P z; scratch vectors z (inner precision, stride
  // ir_stride(n) for the refinement solver) and t (FP64)
  dgop_operator* prec = nullptr;
  void* pz = nullptr;
  double* pt = nullptr;
  // done-flag reads run one segment behind the enqueued work (no events: read synchronously)
  cudaEvent_t ev[2] = {nullptr, nullptr};
  // the operator kernel forms the first inner product of an iteration (CG: p . Ap; GMRES:
  // V_0 . w) in its epilogue when it can; off: a separate pass, as in the reference
  bool fuse_dot = true;
};

}  // namespace dgop

struct dgop_solver {
  dgop::SolverImpl s;
};

using namespace dgop;

namespace {

#define DGOP_CUDA_S(call)                               \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

#define DGOP_TRY(call)             \
  do {                             \
    const int _rc = (call);        \
    if (_rc != DGOP_OK) return _rc; \
  } while (0)

// `words`: FP64 words of vector workspace
int solver_alloc(dgop_solver* sv, size_t words, size_t state_bytes, size_t small_count) {
  SolverImpl& s = sv->s;
  DGOP_CUDA_S(cudaMalloc(&s.work, sizeof(double) * words));
  DGOP_CUDA_S(cudaMalloc(&s.partials, sizeof(double) * 2 * kRB));
  DGOP_CUDA_S(cudaMalloc(&s.state, state_bytes));
  DGOP_CUDA_S(cudaMemset(s.state, 0, state_bytes));
  if (small_count) DGOP_CUDA_S(cudaMalloc(&s.small, sizeof(double) * small_count));
  DGOP_CUDA_S(cudaMallocHost(&s.h_flag, 2 * sizeof(int)));
  for (auto& e : s.ev) DGOP_CUDA_S(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return DGOP_OK;
}

void solver_free(dgop_solver* sv) {
  SolverImpl& s = sv->s;
  if (s.work) cudaFree(s.work);
  if (s.partials) cudaFree(s.partials);
  if (s.state) cudaFree(s.state);
  if (s.small) cudaFree(s.small);
  if (s.h_flag) cudaFreeHost(s.h_flag);
  if (s.wide) cudaFree(s.wide);
  if (s.pz) cudaFree(s.pz);
  if (s.pt) cudaFree(s.pt);
  if (s.exec) cudaGraphExecDestroy(s.exec);
  if (s.wexec) cudaGraphExecDestroy(s.wexec);
  if (s.loop) cudaFree(s.loop);
  if (s.cap) cudaStreamDestroy(s.cap);
  for (auto e : s.ev)
    if (e) cudaEventDestroy(e);
  s = SolverImpl{};
}

bool key_matches(const GraphKey& k, const SolverImpl& s, const void* b, const void* x) {
  return k.b == b && k.x == x && k.version == s.op->version && k.flags == s.op_flags && k.prec == s.prec &&
         (!s.prec || k.prec_version == s.prec->version);
}
GraphKey key_of(const SolverImpl& s, const void* b, const void* x) {
  return GraphKey{b, x, s.op->version, s.op_flags, s.prec, s.prec ? s.prec->version : -1};
}

// Enqueues one segment on `st`: replays the cached graph, capturing it first when the key
// changed, or launches directly when graphs are off.
template <typename F>
int run_segment(SolverImpl& s, cudaStream_t st, const void* b, const void* x, F&& enqueue) {
  if (!s.use_graphs) return enqueue(st);
  if (!(s.exec && key_matches(s.key, s, b, x))) {
    if (!s.cap) DGOP_CUDA_S(cudaStreamCreateWithFlags(&s.cap, cudaStreamNonBlocking));
    DGOP_CUDA_S(cudaStreamBeginCapture(s.cap, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue(s.cap);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s.cap, &graph);
    if (rc != DGOP_OK || e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return rc != DGOP_OK ? rc : cuda_fail(e, "solver graph capture");
    }
    if (s.exec) cudaGraphExecDestroy(s.exec);
    s.exec = nullptr;
    s.key = GraphKey{};
    const cudaError_t e2 = cudaGraphInstantiateWithFlags(&s.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) {
      s.exec = nullptr;
      return cuda_fail(e2, "solver graph instantiation");
    }
    s.key = key_of(s, b, x);
  }
  DGOP_CUDA_S(cudaGraphLaunch(s.exec, st));
  return DGOP_OK;
}

// Enqueues the rest of the solve on `st` as ONE graph launch: a conditional WHILE node whose
// body is one segment followed by k_loop_next (captured into the node's body graph), run at
// most `limit` times.  The graph is built for the current key and rebuilt when it changes; the
// limit is set by a kernel before each launch, so it needs no rebuild.  Same kernels in the same
// order as the segment-by-segment loop, hence the same results bit for bit.
template <typename F>
int run_whole(SolverImpl& s, cudaStream_t st, const void* b, const void* x, const int* done, int limit,
              F&& enqueue) {
  if (!s.loop) DGOP_CUDA_S(cudaMalloc(&s.loop, 2 * sizeof(int)));
  if (!(s.wexec && key_matches(s.wkey, s, b, x))) {
    if (!s.cap) DGOP_CUDA_S(cudaStreamCreateWithFlags(&s.cap, cudaStreamNonBlocking));
    if (s.wexec) cudaGraphExecDestroy(s.wexec);
    s.wexec = nullptr;
    s.wkey = GraphKey{};
    cudaGraph_t graph = nullptr;
    DGOP_CUDA_S(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle h{};
    cudaGraphNodeParams cp{};
    cudaGraphNode_t node = nullptr;
    cudaError_t e = cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      e = cudaGraphAddNode(&node, graph, nullptr, 0, &cp);
    }
    int rc = DGOP_OK;
    if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(s.cap, cp.conditional.phGraph_out[0], nullptr, nullptr,
                                                            0, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      rc = enqueue(s.cap);
      k_loop_next<<<1, 1, 0, s.cap>>>(h, done, s.loop);
      cudaGraph_t body = nullptr;
      e = cudaStreamEndCapture(s.cap, &body);
    }
    if (rc == DGOP_OK && e == cudaSuccess) e = cudaGraphInstantiateWithFlags(&s.wexec, graph, 0);
    cudaGraphDestroy(graph);
    if (rc != DGOP_OK || e != cudaSuccess) {
      s.wexec = nullptr;
      return rc != DGOP_OK ? rc : cuda_fail(e, "whole-solve graph");
    }
    s.wkey = key_of(s, b, x);
  }
  k_loop_reset<<<1, 1, 0, st>>>(s.loop, limit);
  DGOP_CUDA_S(cudaGetLastError());
  DGOP_CUDA_S(cudaGraphLaunch(s.wexec, st));
  return DGOP_OK;
}

// After segment `seg` was enqueued: starts the read of its `done` word and reports whether the
// solve had finished by the end of segment seg - 1 (one segment of look-ahead, whose kernels are
// no-ops once `done` is set).  Without events the read is synchronous and reports segment seg.
int segment_done(SolverImpl& s, cudaStream_t st, int seg, bool* stop) {
  int* flag = s.h_flag + (seg & 1);
  DGOP_CUDA_S(cudaMemcpyAsync(flag, s.state, sizeof(int), cudaMemcpyDeviceToHost, st));
  if (!s.ev[0]) {
    DGOP_CUDA_S(cudaStreamSynchronize(st));
    *stop = *flag != 0;
    return DGOP_OK;
  }
  DGOP_CUDA_S(cudaEventRecord(s.ev[seg & 1], st));
  *stop = false;
  if (seg > 0) {
    DGOP_CUDA_S(cudaEventSynchronize(s.ev[(seg - 1) & 1]));
    *stop = s.h_flag[(seg - 1) & 1] != 0;
  }
  return DGOP_OK;
}

template <typename State>
int finish(SolverImpl& s, cudaStream_t st, dgop_solve_result* res) {
  State h;
  DGOP_CUDA_S(cudaMemcpyAsync(&h, s.state, sizeof(h), cudaMemcpyDeviceToHost, st));
  DGOP_CUDA_S(cudaStreamSynchronize(st));
  res->success = h.success;
  res->iterations = h.iters;
  res->relative_error = h.rel;
  return DGOP_OK;
}

int cg_solve(SolverImpl& s, const double* b, double* x, int max_iters, double tol, dgop_solve_result* res,
             cudaStream_t st) {
  const int64_t n = s.n;
  double* tmp = s.work;
  double* r = s.work + vec_stride(n);
  double* p = s.work + 2 * vec_stride(n);
  double* pa = s.partials;
  double* pb = s.partials + kRB;
  CGState* cs = static_cast<CGState*>(s.state);
  // 1) r = rhs - A x
  DGOP_TRY(launch_f64(s.op, 1.0, x, 0.0, tmp, s.op_flags, st));
  k_sub_norm<<<kRB, kRT, 0, st>>>(b, tmp, r, n, pa, nullptr);
  k_cg_init<<<1, kRT, 0, st>>>(cs, pa, tol, max_iters);
  k_cg_init_p<<<kRB, kRT, 0, st>>>(cs, r, p, x, n);
  if (max_iters <= 0) k_cg_no_iters<<<1, 1, 0, st>>>(cs);
  DGOP_CUDA_S(cudaGetLastError());
  const int* done = &cs->done;
  auto chunk = [&](cudaStream_t q) -> int {
    for (int kk = 0; kk < kCheckEvery; ++kk) {
      // Ap = A p with p . Ap formed in the operator's epilogue (conjugategradient.hpp:176-179)
      bool fused = false;
      const DotEpilogue de{p, pa, kRB, &fused};
      DGOP_TRY(launch_f64(s.op, 1.0, p, 0.0, tmp, s.op_flags, q, done, s.fuse_dot ? &de : nullptr));
      if (!fused)
        k_dot<<<kRB, kRT, 0, q>>>(static_cast<const double*>(p), static_cast<const double*>(tmp), n, pa, done);
      k_cg_update<<<kRB, kRT, 0, q>>>(kk, cs, x, r, p, tmp, n, pa, pb);
      k_cg_finish<<<kRB, kRT, 0, q>>>(kk, cs, r, p, n, pb);
    }
    k_cg_next_chunk<<<1, 1, 0, q>>>(cs);
    DGOP_CUDA_S(cudaGetLastError());
    return DGOP_OK;
  };
  const int64_t chunks = ((int64_t)std::max(max_iters, 0) + kCheckEvery - 1) / kCheckEvery;
  if (s.whole && s.use_graphs) {
    if (chunks > 0) DGOP_TRY(run_whole(s, st, b, x, done, (int)std::min<int64_t>(chunks, INT32_MAX), chunk));
  } else {
    for (int c = 0; c < chunks; ++c) {
      DGOP_TRY(run_segment(s, st, b, x, chunk));
      bool stop = false;
      DGOP_TRY(segment_done(s, st, c, &stop));
      if (stop) break;
    }
  }
  return finish<CGState>(s, st, res);
}

int gmres_solve(SolverImpl& s, const double* b, double* x, int max_iters, double tol, dgop_solve_result* res,
                cudaStream_t st) {
  const int64_t n = s.n;
  const int m = s.restart;
  double* w = s.work;
  const int64_t ld = vec_stride(n);
  double* V = s.work + ld;  // m + 1 basis vectors, stride ld
  double* pa = s.partials;
  double* pb = s.partials + kRB;
  double* H = s.small;
  double* csv = H + (m + 1) * m;
  double* snv = csv + m;
  double* e1 = snv + m;
  double* y = e1 + m + 1;
  GMState* gs = static_cast<GMState*>(s.state);
  const int* done = &gs->done;
  const int* inactive = &gs->inactive;
  auto residual = [&](int phase, cudaStream_t q) -> int {
    DGOP_TRY(launch_f64(s.op, 1.0, x, 0.0, w, s.op_flags, q, done));
    k_sub_norm<<<kRB, kRT, 0, q>>>(b, w, V, n, pa, done);
    k_gm_resid<<<1, kRT, 0, q>>>(gs, pa, phase);
    DGOP_CUDA_S(cudaGetLastError());
    return DGOP_OK;
  };
  auto cycle = [&](cudaStream_t q) -> int {
    k_gm_cycle_start<<<1, 1, 0, q>>>(gs, csv, snv, e1, y, m);
    k_gm_scale<<<kRB, kRT, 0, q>>>(gs, static_cast<const double*>(V), V, n, -1);
    for (int j = 0; j < m; ++j) {
      double* vj = V + (int64_t)j * ld;
      // w = A v_j (A P v_j) with the first modified Gram-Schmidt product V_0 . w formed in the
      // operator's epilogue (gmres.hpp:157-165)
      bool fused = false;
      const DotEpilogue de{V, pa, kRB, &fused};
      if (s.prec) {
        double* z = static_cast<double*>(s.pz);
        DGOP_TRY(launch_f64(s.prec, 1.0, vj, 0.0, z, 0, q, inactive));
        DGOP_TRY(launch_f64(s.op, 1.0, z, 0.0, w, s.op_flags, q, inactive, s.fuse_dot ? &de : nullptr));
      } else {
        DGOP_TRY(launch_f64(s.op, 1.0, vj, 0.0, w, s.op_flags, q, inactive, s.fuse_dot ? &de : nullptr));
      }
      if (!fused)
        k_dot<<<kRB, kRT, 0, q>>>(static_cast<const double*>(V), static_cast<const double*>(w), n, pa, inactive);
      double* pin = pa;
      double* pout = pb;
      for (int i = 0; i <= j; ++i) {
        const double* next = (i < j) ? V + (int64_t)(i + 1) * ld : w;
        k_gm_mgs<<<kRB, kRT, 0, q>>>(gs, i, j, m, static_cast<const double*>(V + (int64_t)i * ld), next, w, n, H,
                                     pin, pout);
        std::swap(pin, pout);
      }
      k_gm_column<<<1, kRT, 0, q>>>(gs, j, m, H, csv, snv, e1, pin);
      k_gm_scale<<<kRB, kRT, 0, q>>>(gs, static_cast<const double*>(w), V + (int64_t)(j + 1) * ld, n, j);
      DGOP_CUDA_S(cudaGetLastError());
    }
    k_gm_backsub<<<1, 1, 0, q>>>(gs, H, e1, y, m);
    if (s.prec) {
      // x += P (sum_i y_i V_i)
      DGOP_CUDA_S(cudaMemsetAsync(s.pt, 0, sizeof(double) * n, q));
      k_gm_update<<<kRB, kRT, 0, q>>>(gs, s.pt, static_cast<const double*>(V), ld, y, n);
      DGOP_TRY(launch_f64(s.prec, 1.0, s.pt, 1.0, x, 0, q, done));
    } else {
      k_gm_update<<<kRB, kRT, 0, q>>>(gs, x, static_cast<const double*>(V), ld, y, n);
    }
    return residual(1, q);
  };
  k_dot<<<kRB, kRT, 0, st>>>(b, b, n, pa, nullptr);
  k_gm_denom<<<1, kRT, 0, st>>>(gs, pa, tol, max_iters);
  DGOP_CUDA_S(cudaGetLastError());
  if (max_iters <= 0 || m <= 0) {
    DGOP_TRY(residual(2, st));
  } else {
    DGOP_TRY(residual(0, st));
    // every cycle performs at least one iteration or finishes the solve
    if (s.whole && s.use_graphs) {
      DGOP_TRY(run_whole(s, st, b, x, done, max_iters < INT32_MAX ? max_iters + 1 : INT32_MAX, cycle));
    } else {
      for (int c = 0; c <= max_iters; ++c) {
        DGOP_TRY(run_segment(s, st, b, x, cycle));
        bool stop = false;
        DGOP_TRY(segment_done(s, st, c, &stop));
        if (stop) break;
      }
    }
  }
  return finish<GMState>(s, st, res);
}

// Vector stride of the refinement solver's inner workspace (the same rounding as vec_stride).
int64_t ir_stride(int64_t n) { return vec_stride(n); }

int apply_inner(dgop_operator* op, const float* x, float* y, int flags, cudaStream_t st, const int* skip) {
  return launch_f32(op, 1.0f, x, 0.0f, y, kLinear | flags, st, skip);
}
int apply_inner(dgop_operator* op, const double* x, double* y, int flags, cudaStream_t st, const int* skip) {
  return launch_f64(op, 1.0, x, 0.0, y, kLinear | flags, st, skip);
}

// GMRES with iterative refinement: every restart cycle solves the correction equation A d = r
// for the FP64 residual r with inner operator applies and an inner Krylov basis of type T
// (inner products, Hessenberg matrix and rotations in FP64), then x += d in FP64 and the true
// residual is recomputed with the FP64 operator.  The Arnoldi step is classical Gram-Schmidt
// fused into two passes (all projections of w in one pass, the update of w and its norm in the
// next) instead of the reference's j + 1 modified Gram-Schmidt sweeps; the FP64 residual of the
// refinement loop bounds the effect of the weaker orthogonality.  Stopping rules and reported
// quantities are those of gmres_solve.
template <typename T>
int gmres_ir_solve(SolverImpl& s, const double* b, double* x, int max_iters, double tol, dgop_solve_result* res,
                   cudaStream_t st) {
  const int64_t n = s.n;
  const int m = s.restart;
  const int64_t ld = ir_stride(n);
  double* w64 = s.work;
  double* r64 = s.work + vec_stride(n);
  T* w = reinterpret_cast<T*>(s.work + 2 * vec_stride(n));
  T* V = w + ld;  // m + 1 inner basis vectors, stride ld
  double* pa = s.partials;
  double* H = s.small;
  double* csv = H + (m + 1) * m;
  double* snv = csv + m;
  double* e1 = snv + m;
  double* y = e1 + m + 1;
  GMState* gs = static_cast<GMState*>(s.state);
  const int* done = &gs->done;
  const int* inactive = &gs->inactive;
  auto residual = [&](int phase, cudaStream_t q) -> int {
    DGOP_TRY(launch_f64(s.op, 1.0, x, 0.0, w64, s.op_flags, q, done));
    k_sub_norm<<<kRB, kRT, 0, q>>>(b, w64, r64, n, pa, done);
    k_gm_resid<<<1, kRT, 0, q>>>(gs, pa, phase);
    DGOP_CUDA_S(cudaGetLastError());
    return DGOP_OK;
  };
  // the inner operator: the BF16 tensor-core kernel for DGOP_BF16 (FP32 vectors), else the
  // kernel of the inner type
  auto apply_op = [&](const T* in, T* out, cudaStream_t q) -> int {
    if constexpr (sizeof(T) == 4) {
      if (s.inner == DGOP_BF16) return launch_bf16(s.op, 1.0f, in, 0.0f, out, kLinear | s.op_flags, q, inactive);
    }
    return apply_inner(s.op, in, out, s.op_flags, q, inactive);
  };
  auto cycle = [&](cudaStream_t q) -> int {
    k_gm_cycle_start<<<1, 1, 0, q>>>(gs, csv, snv, e1, y, m);
    k_gm_scale<<<kRB, kRT, 0, q>>>(gs, static_cast<const double*>(r64), V, n, -1);  // V0 = r / |r|
    for (int j = 0; j < m; ++j) {
      T* vj = V + (int64_t)j * ld;
      T* vn = vj + ld;
      if (s.prec) {
        T* z = static_cast<T*>(s.pz);
        DGOP_TRY(apply_inner(s.prec, vj, z, 0, q, inactive));
        DGOP_TRY(apply_op(z, w, q));
      } else {
        DGOP_TRY(apply_op(vj, w, q));
      }
      const dim3 dgrid(kRB, (j + 1 + kGsChunk - 1) / kGsChunk);
      k_gs_dots<T><<<dgrid, kRT, 0, q>>>(gs, V, ld, j, w, s.wide);
      k_gs_h<<<j + 1, kRT, 0, q>>>(gs, j, m, H, s.wide);
      k_gs_update<T><<<kRB, kRT, 0, q>>>(gs, V, ld, j, m, H, w, vn, pa);
      k_gm_column<<<1, kRT, 0, q>>>(gs, j, m, H, csv, snv, e1, pa);
      k_gs_rescale<T><<<kRB, kRT, 0, q>>>(gs, vn, ld, j);
      DGOP_CUDA_S(cudaGetLastError());
    }
    k_gm_backsub<<<1, 1, 0, q>>>(gs, H, e1, y, m);
    if (s.prec) {
      DGOP_CUDA_S(cudaMemsetAsync(s.pt, 0, sizeof(double) * n, q));
      k_gm_update<<<kRB, kRT, 0, q>>>(gs, s.pt, static_cast<const T*>(V), ld, y, n);
      DGOP_TRY(launch_f64(s.prec, 1.0, s.pt, 1.0, x, 0, q, done));
    } else {
      k_gm_update<<<kRB, kRT, 0, q>>>(gs, x, static_cast<const T*>(V), ld, y, n);
    }
    return residual(1, q);
  };
  k_dot<<<kRB, kRT, 0, st>>>(b, b, n, pa, nullptr);
  k_gm_denom<<<1, kRT, 0, st>>>(gs, pa, tol, max_iters);
  DGOP_CUDA_S(cudaGetLastError());
  if (max_iters <= 0 || m <= 0) {
    DGOP_TRY(residual(2, st));
  } else {
    DGOP_TRY(residual(0, st));
    if (s.whole && s.use_graphs) {
      DGOP_TRY(run_whole(s, st, b, x, done, max_iters < INT32_MAX ? max_iters + 1 : INT32_MAX, cycle));
    } else {
      for (int c = 0; c <= max_iters; ++c) {
        DGOP_TRY(run_segment(s, st, b, x, cycle));
        bool stop = false;
        DGOP_TRY(segment_done(s, st, c, &stop));
        if (stop) break;
      }
    }
  }
  return finish<GMState>(s, st, res);
}

}  // namespace

extern "C" {

int dgop_gmres_ir_create(dgop_operator* op, int restart, int inner_precision, dgop_solver** out) {
  if (!op || !out || restart < 1 || restart > kGsMaxRestart) {
    set_error("dgop_gmres_ir_create: null argument or restart outside [1, 1000]");
    return DGOP_ERR_ARG;
  }
  *out = nullptr;
  if (inner_precision != DGOP_FP32 && inner_precision != DGOP_FP64 && inner_precision != DGOP_BF16) {
    set_error("dgop_gmres_ir_create: inner_precision must be DGOP_FP32, DGOP_FP64 or DGOP_BF16");
    return DGOP_ERR_ARG;
  }
  if (inner_precision == DGOP_FP32 && !op->f32.ready && !op->k32.ready && !op->n32.ready) {
    set_error("dgop_gmres_ir_create: the operator has no FP32 kernel");
    return DGOP_ERR_UNSUPPORTED;
  }
  if (inner_precision == DGOP_BF16 && !(op->n32.ready && op->n32.tc_ok)) {
    set_error("dgop_gmres_ir_create: the operator has no BF16 tensor-core kernel (any-dimension Kronecker form, "
              "even dimension, (p+1)^(D/2) <= 32)");
    return DGOP_ERR_UNSUPPORTED;
  }
  auto* sv = new (std::nothrow) dgop_solver();
  if (!sv) {
    set_error("host allocation failed");
    return DGOP_ERR_ALLOC;
  }
  SolverImpl& s = sv->s;
  s.kind = 2;
  s.inner = inner_precision;
  s.op = op;
  s.n = op->sp.ndofs;
  s.restart = restart;
  const size_t small = (size_t)(restart + 1) * restart + 2 * restart + (restart + 1) + restart;
  // two FP64 vectors (A x, residual), then restart + 2 inner vectors (w and the basis) at stride
  // ir_stride(n); the padding entries must read as zero, so the workspace starts zeroed
  const size_t inner_words = (size_t)ir_stride(s.n) * (inner_precision != DGOP_FP64 ? 4 : 8) / 8;
  const size_t words = 2 * (size_t)vec_stride(s.n) + (size_t)(restart + 2) * inner_words;
  int rc = solver_alloc(sv, words, sizeof(GMState), small);
  if (rc == DGOP_OK) {
    cudaError_t e = cudaMemset(s.work, 0, sizeof(double) * words);
    if (e == cudaSuccess) e = cudaMalloc(&s.wide, sizeof(double) * (size_t)(restart + 1) * kRB);
    if (e != cudaSuccess) rc = cuda_fail(e, "dgop_gmres_ir_create workspace");
  }
  if (rc != DGOP_OK) {
    solver_free(sv);
    delete sv;
    return rc;
  }
  *out = sv;
  return DGOP_OK;
}

int dgop_cg_create(dgop_operator* op, dgop_solver** out) {
  if (!op || !out) {
    set_error("dgop_cg_create: null argument");
    return DGOP_ERR_ARG;
  }
  *out = nullptr;
  auto* sv = new (std::nothrow) dgop_solver();
  if (!sv) {
    set_error("host allocation failed");
    return DGOP_ERR_ALLOC;
  }
  sv->s.kind = 0;
  sv->s.op = op;
  sv->s.n = op->sp.ndofs;
  const int rc = solver_alloc(sv, 3 * (size_t)vec_stride(sv->s.n), sizeof(CGState), 0);
  if (rc != DGOP_OK) {
    solver_free(sv);
    delete sv;
    return rc;
  }
  *out = sv;
  return DGOP_OK;
}

int dgop_gmres_create(dgop_operator* op, int restart, dgop_solver** out) {
  if (!op || !out || restart < 1 || restart > 1000) {
    set_error("dgop_gmres_create: null argument or restart outside [1, 1000]");
    return DGOP_ERR_ARG;
  }
  *out = nullptr;
  auto* sv = new (std::nothrow) dgop_solver();
  if (!sv) {
    set_error("host allocation failed");
    return DGOP_ERR_ALLOC;
  }
  sv->s.kind = 1;
  sv->s.op = op;
  sv->s.n = op->sp.ndofs;
  sv->s.restart = restart;
  const size_t small = (size_t)(restart + 1) * restart + 2 * restart + (restart + 1) + restart;
  const int rc = solver_alloc(sv, (size_t)(restart + 2) * vec_stride(sv->s.n), sizeof(GMState), small);
  if (rc != DGOP_OK) {
    solver_free(sv);
    delete sv;
    return rc;
  }
  *out = sv;
  return DGOP_OK;
}

int dgop_solver_solve(dgop_solver* sv, const double* b, double* x, int max_iters, double tol,
                      dgop_solve_result* result, void* stream) {
  if (!sv || !b || !x || !result) {
    set_error("dgop_solver_solve: null argument");
    return DGOP_ERR_ARG;
  }
  if (!(tol >= 0.0)) {
    set_error("dgop_solver_solve: tol must be >= 0");
    return DGOP_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (sv->s.kind == 0) return cg_solve(sv->s, b, x, max_iters, tol, result, st);
  if (sv->s.kind == 2)
    return sv->s.inner != DGOP_FP64 ? gmres_ir_solve<float>(sv->s, b, x, max_iters, tol, result, st)
                                    : gmres_ir_solve<double>(sv->s, b, x, max_iters, tol, result, st);
  return gmres_solve(sv->s, b, x, max_iters, tol, result, st);
}

int dgop_solver_set_graphs(dgop_solver* sv, int enable) {
  if (!sv) {
    set_error("dgop_solver_set_graphs: null solver");
    return DGOP_ERR_ARG;
  }
  if (enable < 0 || enable > DGOP_GRAPHS_WHOLE) {
    set_error("dgop_solver_set_graphs: enable must be DGOP_GRAPHS_OFF, DGOP_GRAPHS_SEGMENTS or DGOP_GRAPHS_WHOLE");
    return DGOP_ERR_ARG;
  }
  sv->s.use_graphs = enable != DGOP_GRAPHS_OFF;
  sv->s.whole = enable == DGOP_GRAPHS_WHOLE;
  return DGOP_OK;
}

int dgop_solver_set_preconditioner(dgop_solver* sv, dgop_operator* prec) {
  if (!sv) {
    set_error("dgop_solver_set_preconditioner: null solver");
    return DGOP_ERR_ARG;
  }
  SolverImpl& s = sv->s;
  if (prec && s.kind == 0) {
    set_error("dgop_solver_set_preconditioner: GMRES solvers only");
    return DGOP_ERR_UNSUPPORTED;
  }
  if (prec && prec->sp.ndofs != s.n) {
    set_error("dgop_solver_set_preconditioner: the preconditioner acts on another space");
    return DGOP_ERR_ARG;
  }
  if (prec && s.kind == 2 && s.inner != DGOP_FP64 && !prec->f32.ready && !prec->k32.ready && !prec->n32.ready) {
    set_error("dgop_solver_set_preconditioner: the preconditioner has no FP32 kernel");
    return DGOP_ERR_UNSUPPORTED;
  }
  if (prec && !s.pz) {
    const size_t zbytes = s.kind == 2 ? (size_t)ir_stride(s.n) * (s.inner != DGOP_FP64 ? 4 : 8) : sizeof(double) * s.n;
    cudaError_t e = cudaMalloc(&s.pz, zbytes);
    if (e == cudaSuccess) e = cudaMemset(s.pz, 0, zbytes);
    if (e == cudaSuccess) e = cudaMalloc(&s.pt, sizeof(double) * s.n);
    if (e != cudaSuccess) return cuda_fail(e, "preconditioner workspace");
  }
  s.prec = prec;
  return DGOP_OK;
}

int dgop_solver_set_transpose(dgop_solver* sv, int transpose) {
  if (!sv) {
    set_error("dgop_solver_set_transpose: null solver");
    return DGOP_ERR_ARG;
  }
  sv->s.op_flags = transpose ? kTranspose : 0;
  return DGOP_OK;
}

int dgop_element_dot(const dgop_operator* op, const double* a, const double* b, const double* scale, double* out,
                     void* stream) {
  if (!op || !a || !b || !out) {
    set_error("dgop_element_dot: null argument");
    return DGOP_ERR_ARG;
  }
  const int64_t nelem = op->sp.nelem, nd = op->sp.ndofs / op->sp.nelem;
  const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((nelem + kRT / 32 - 1) / (kRT / 32), 4 * kRB));
  k_element_dot<<<(unsigned)blocks, kRT, 0, (cudaStream_t)stream>>>(a, b, scale, out, nelem, nd);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "dgop_element_dot launch");
  return DGOP_OK;
}

int dgop_solver_set_fused_dot(dgop_solver* sv, int enable) {
  if (!sv) {
    set_error("dgop_solver_set_fused_dot: null solver");
    return DGOP_ERR_ARG;
  }
  sv->s.fuse_dot = enable != 0;
  sv->s.key = GraphKey{};  // re-capture the solver graphs
  sv->s.wkey = GraphKey{};
  return DGOP_OK;
}

int dgop_solver_destroy(dgop_solver* sv) {
  if (!sv) return DGOP_OK;
  solver_free(sv);
  delete sv;
  return DGOP_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// CG with a workspace that is never allocated at run time.
//
// Some callers cannot let a library call cudaMalloc: programs whose host framework owns every
// byte of device memory through its own pool (a caching allocator with a fixed budget), and
// latency-critical loops where cudaMalloc/cudaFree would add a device-wide synchronization.
// For them dgop_cg_solve_static runs the same CG kernels as dgop_cg_create/dgop_solver_solve
// with its three work vectors, partial sums and solver state in one file-scope device array of
// fixed size (every GPU that loads this library holds it, about 6.3 MB, until the process exits).
// ------------------------------------------------------------------------------------------
namespace {

constexpr int64_t kStaticCgWords = 3 * (int64_t)DGOP_STATIC_CG_MAX_DOFS + 2 * kRB + (sizeof(CGState) + 7) / 8;
static __device__ __align__(256) double g_static_cg_scratch[kStaticCgWords];

std::mutex g_static_cg_mutex;
// Device address of the array per device, with the id of the CUDA context it was looked up in:
// a device reset or a new primary context reloads the module at another address, so a cached
// address is only used while the context it came from is still the current one.
struct StaticCgAddr {
  unsigned long long ctx_id = 0;
  double* addr = nullptr;
};
StaticCgAddr g_static_cg_addr[64];
thread_local int g_static_cg_flag[2];  // host copies of the `done` word (pageable; no allocation)

// Id of the calling thread's current CUDA context (0 when none is current).  The two driver
// functions are fetched through the runtime, so the library needs no link against libcuda.
int current_context_id(unsigned long long* id) {
  using GetCurrentFn = CUresult (*)(CUcontext*);
  using GetIdFn = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrentFn get_current = nullptr;
  static GetIdFn get_id = nullptr;
  if (!get_current || !get_id) {
    void* f0 = nullptr;
    void* f1 = nullptr;
    cudaDriverEntryPointQueryResult q0, q1;
    cudaError_t e = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f0, 12000, cudaEnableDefault, &q0);
    if (e == cudaSuccess) e = cudaGetDriverEntryPointByVersion("cuCtxGetId", &f1, 12000, cudaEnableDefault, &q1);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDriverEntryPointByVersion(cuCtxGetCurrent / cuCtxGetId)");
    if (q0 != cudaDriverEntryPointSuccess || q1 != cudaDriverEntryPointSuccess || !f0 || !f1) {
      set_error("dgop_cg_solve_static: the driver does not provide cuCtxGetCurrent / cuCtxGetId");
      return DGOP_ERR_CUDA;
    }
    get_current = reinterpret_cast<GetCurrentFn>(f0);
    get_id = reinterpret_cast<GetIdFn>(f1);
  }
  CUcontext ctx = nullptr;
  *id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return DGOP_OK;
  unsigned long long v = 0;
  if (get_id(ctx, &v) != CUDA_SUCCESS) return DGOP_OK;
  *id = v;
  return DGOP_OK;
}

// Device address of the array for the operator's device, which must be the current device.  In
// host code the array's name is only a stand-in; the kernels must be given this address.  It is
// looked up (cudaGetSymbolAddress) on the first call in a context and again whenever the current
// context is not the one of the cached address.
int static_cg_scratch(const dgop_operator* op, double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev != op->device) {
    set_error("dgop_cg_solve_static: the current device (" + std::to_string(dev) +
              ") differs from the operator's device (" + std::to_string(op->device) + "); make it current first");
    return DGOP_ERR_ARG;
  }
  if (dev < 0 || dev >= 64) {
    set_error("dgop_cg_solve_static: device index out of range");
    return DGOP_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_static_cg_mutex);
  unsigned long long ctx = 0;
  int rc = current_context_id(&ctx);
  if (rc != DGOP_OK) return rc;
  StaticCgAddr& c = g_static_cg_addr[dev];
  if (!c.addr || ctx == 0 || ctx != c.ctx_id) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_cg_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(static CG workspace)");
    rc = current_context_id(&ctx);  // the lookup binds the device's primary context if none was
    if (rc != DGOP_OK) return rc;
    c.addr = static_cast<double*>(p);
    c.ctx_id = ctx;
  }
  *out = c.addr;
  return DGOP_OK;
}

}  // namespace

extern "C" int dgop_cg_solve_static(dgop_operator* op, const double* b, double* x, int max_iters, double tol,
                                    dgop_solve_result* result, void* stream) {
  if (!op || !b || !x || !result) {
    set_error("dgop_cg_solve_static: null argument");
    return DGOP_ERR_ARG;
  }
  if (!(tol >= 0.0)) {
    set_error("dgop_cg_solve_static: tol must be >= 0");
    return DGOP_ERR_ARG;
  }
  const int64_t n = op->sp.ndofs;
  if (n > DGOP_STATIC_CG_MAX_DOFS) {
    set_error("dgop_cg_solve_static: " + std::to_string(n) + " DoFs exceed the static workspace limit of " +
              std::to_string((long long)DGOP_STATIC_CG_MAX_DOFS) + " DoFs; use dgop_cg_create instead");
    return DGOP_ERR_ARG;
  }
  double* base = nullptr;
  const int rc = static_cg_scratch(op, &base);
  if (rc != DGOP_OK) return rc;
  SolverImpl s;
  s.kind = 0;
  s.op = op;
  s.n = n;
  s.work = base;
  s.partials = base + 3 * (int64_t)DGOP_STATIC_CG_MAX_DOFS;
  s.state = base + 3 * (int64_t)DGOP_STATIC_CG_MAX_DOFS + 2 * kRB;
  s.h_flag = g_static_cg_flag;
  s.use_graphs = false;  // direct launches and synchronous done reads: nothing is created
  cudaStream_t st = (cudaStream_t)stream;
  // the array keeps the previous call's contents: start from a cleared solver state
  const cudaError_t e = cudaMemsetAsync(s.state, 0, sizeof(CGState), st);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(static CG state)");
  return cg_solve(s, b, x, max_iters, tol, result, st);
}
