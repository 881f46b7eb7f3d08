// Many independent systems A_i x_i = b_i solved together: restarted GMRES(m) with iterative
// refinement (inner Krylov cycles in FP32 or FP64, residual and solution in FP64; right
// preconditioning by P_i), every system's iterations advanced in lockstep.
//
// Each Krylov step is a fixed sequence of launches for ALL the systems of a wave: one operator
// (and preconditioner) apply per system, each predicated on that system's device state, and one
// launch per vector operation over the wave's concatenated vectors, cut into chunks of kChunk
// values that carry their system's index.  Inner products are reduced per chunk and then per
// system in a fixed order (deterministic).  The scalar steps (Hessenberg column, Givens
// rotations, stopping tests, back-substitution) are those of the single-system solver
// (gmres_steps.cuh), one block per system.  The per-system applies of a step are independent
// branches (16 streams forked and joined), so small systems share the GPU.  A restart cycle of
// the whole wave is captured once as
// a CUDA graph and replayed until every system of the wave has finished; the host reads the wave's
// done flags once per cycle.  Systems that finish early stay idle (their launches return at once).
//
// Workspace (FP64 residual, correction and apply vectors, the inner basis) does not fit for
// thousands of systems at once, so the systems are cut into waves whose workspace fits a budget;
// one arena sized for the largest wave is allocated at creation.  No reference counterpart: the
// reference solves one system per GMRES_no_alloc call (Solvers/gmres.hpp:74).
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <numeric>
#include <vector>

#include "dgop_internal.h"
#include "gmres_steps.cuh"

using namespace dgop;

namespace {

constexpr int kBT = 256;            // threads per block
constexpr int64_t kChunk = 32768;   // values per chunk of a vector operation
constexpr int kDotsPerBlock = 8;    // basis vectors per block row of the projection pass

#define DGOP_CUDA_BS(call)                              \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)
#define DGOP_TRY_BS(call)           \
  do {                              \
    const int _rc = (call);         \
    if (_rc != DGOP_OK) return _rc; \
  } while (0)

inline int64_t stride64(int64_t n) { return (n + 63) / 64 * 64; }

// Per-system record of a wave (device).
template <typename T>
struct Sys {
  const double* b;
  double* x;
  double* w64;  // A x
  double* r64;  // b - A x
  double* pt;   // sum y_i V_i before the preconditioner (FP64)
  T* w;         // inner A P v
  T* z;         // inner P v
  T* V;         // m + 1 basis vectors, stride ld
  int64_t n, ld;
  int64_t c0, c1;  // the system's chunks
  GMState* st;
  double *H, *cs, *sn, *e1, *y;
};

struct Chunk {
  int sys;
  int64_t begin, end;
};

// Block sum in a fixed order; valid in thread 0.
__device__ __forceinline__ double bsum(double v) {
  __shared__ double ws[kBT / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < kBT / 32 ? ws[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  }
  __syncthreads();
  return s;
}

// Sum over system s's chunks of part[c * pw + slot] (fixed order), in thread 0.
template <typename T>
__device__ __forceinline__ double sys_sum(const Sys<T>& S, const double* part, int pw, int slot) {
  double v = 0.0;
  for (int64_t c = S.c0 + threadIdx.x; c < S.c1; c += kBT) v += part[c * pw + slot];
  return bsum(v);
}

#define CHUNK_LOOP(l, C) for (int64_t l = (C).begin + threadIdx.x; l < (C).end; l += kBT)

template <typename T>
__global__ void __launch_bounds__(kBT) kb_norm_b(const Sys<T>* sys, const Chunk* ch, double* part, int pw) {
  const Chunk C = ch[blockIdx.x];
  const Sys<T>& S = sys[C.sys];
  double v = 0.0;
  CHUNK_LOOP(l, C) v += S.b[l] * S.b[l];
  v = bsum(v);
  if (threadIdx.x == 0) part[blockIdx.x * (int64_t)pw] = v;
}

// r = b - A x, part <- |r|^2
template <typename T>
__global__ void __launch_bounds__(kBT) kb_sub_norm(const Sys<T>* sys, const Chunk* ch, double* part, int pw) {
  const Chunk C = ch[blockIdx.x];
  const Sys<T>& S = sys[C.sys];
  if (S.st->done) return;
  double v = 0.0;
  CHUNK_LOOP(l, C) {
    const double r = S.b[l] - S.w64[l];
    S.r64[l] = r;
    v += r * r;
  }
  v = bsum(v);
  if (threadIdx.x == 0) part[blockIdx.x * (int64_t)pw] = v;
}

template <typename T>
__global__ void __launch_bounds__(kBT) kb_denom(const Sys<T>* sys, const double* part, int pw, double tol,
                                                int max_iters) {
  const Sys<T>& S = sys[blockIdx.x];
  const double R = sys_sum(S, part, pw, 0);
  if (threadIdx.x == 0) gm_denom(S.st, R, tol, max_iters);
}

template <typename T>
__global__ void __launch_bounds__(kBT) kb_resid(const Sys<T>* sys, const double* part, int pw, int phase) {
  const Sys<T>& S = sys[blockIdx.x];
  if (S.st->done) return;
  const double R = sys_sum(S, part, pw, 0);
  if (threadIdx.x == 0) gm_resid(S.st, R, phase);
}

template <typename T>
__global__ void kb_cycle_start(const Sys<T>* sys, int count, int m) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const Sys<T>& S = sys[i];
  gm_cycle_start(S.st, S.cs, S.sn, S.e1, S.y, m);
}

// V_0 = r / |r|
template <typename T>
__global__ void __launch_bounds__(kBT) kb_scale_v0(const Sys<T>* sys, const Chunk* ch) {
  const Chunk C = ch[blockIdx.x];
  const Sys<T>& S = sys[C.sys];
  if (S.st->done) return;
  const double s = S.st->inv_h;
  CHUNK_LOOP(l, C) S.V[l] = (T)(S.r64[l] * s);
}

// part[c * pw + i] <- (V_i, w) over chunk c, i <= j (blockIdx.y selects kDotsPerBlock vectors)
template <typename T>
__global__ void __launch_bounds__(kBT) kb_gs_dots(const Sys<T>* sys, const Chunk* ch, int j, double* part, int pw) {
  const Chunk C = ch[blockIdx.x];
  const Sys<T>& S = sys[C.sys];
  if (S.st->inactive) return;
  const int i0 = blockIdx.y * kDotsPerBlock;
  const int cnt = min(kDotsPerBlock, j + 1 - i0);
  double acc[kDotsPerBlock];
#pragma unroll
  for (int c = 0; c < kDotsPerBlock; ++c) acc[c] = 0.0;
  CHUNK_LOOP(l, C) {
    const double wl = (double)S.w[l];
#pragma unroll
    for (int c = 0; c < kDotsPerBlock; ++c)
      if (c < cnt) acc[c] += (double)S.V[(int64_t)(i0 + c) * S.ld + l] * wl;
  }
#pragma unroll
  for (int c = 0; c < kDotsPerBlock; ++c) {
    const double v = bsum(acc[c]);
    if (threadIdx.x == 0 && c < cnt) part[blockIdx.x * (int64_t)pw + i0 + c] = v;
  }
}

// H(i, j) <- sum over the system's chunks (one block per (system, i))
template <typename T>
__global__ void __launch_bounds__(kBT) kb_gs_h(const Sys<T>* sys, int j, int m, const double* part, int pw) {
  const Sys<T>& S = sys[blockIdx.x];
  if (S.st->inactive) return;
  const int i = blockIdx.y;
  const double h = sys_sum(S, part, pw, i);
  if (threadIdx.x == 0) S.H[j * (m + 1) + i] = h;
}

// V_{j+1} <- w - sum_{i <= j} H(i, j) V_i (FP64 arithmetic), part <- |V_{j+1}|^2
template <typename T>
__global__ void __launch_bounds__(kBT) kb_gs_update(const Sys<T>* sys, const Chunk* ch, int j, int m, double* part,
                                                    int pw) {
  const Chunk C = ch[blockIdx.x];
  const Sys<T>& S = sys[C.sys];
  if (S.st->inactive) return;
  T* out = S.V + (int64_t)(j + 1) * S.ld;
  const double* hj = S.H + j * (m + 1);
  double sq = 0.0;
  CHUNK_LOOP(l, C) {
    double a = (double)S.w[l];
    for (int i = 0; i <= j; ++i) a -= hj[i] * (double)S.V[(int64_t)i * S.ld + l];
    const T o = (T)a;
    out[l] = o;
    sq += (double)o * (double)o;
  }
  sq = bsum(sq);
  if (threadIdx.x == 0) part[blockIdx.x * (int64_t)pw] = sq;
}

template <typename T>
__global__ void __launch_bounds__(kBT) kb_column(const Sys<T>* sys, int j, int m, const double* part, int pw) {
  const Sys<T>& S = sys[blockIdx.x];
  if (S.st->inactive) return;
  const double R = sys_sum(S, part, pw, 0);
  if (threadIdx.x == 0) gm_column(S.st, j, m, S.H, S.cs, S.sn, S.e1, R);
}

// V_{j+1} *= 1 / H(j + 1, j) when iteration j ran and did not end the cycle
template <typename T>
__global__ void __launch_bounds__(kBT) kb_rescale(const Sys<T>* sys, const Chunk* ch, int j) {
  const Chunk C = ch[blockIdx.x];
  const Sys<T>& S = sys[C.sys];
  const GMState* st = S.st;
  if (st->done || st->brk || st->k != j + 1) return;
  const double sc = st->inv_h;
  T* v = S.V + (int64_t)(j + 1) * S.ld;
  CHUNK_LOOP(l, C) v[l] = (T)((double)v[l] * sc);
}

template <typename T>
__global__ void kb_backsub(const Sys<T>* sys, int count, int m) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const Sys<T>& S = sys[i];
  gm_backsub(S.st, S.H, S.e1, S.y, m);
}

// dst = sum_{i < k} y_i V_i (to_x: x += instead), FP64, in order
template <typename T>
__global__ void __launch_bounds__(kBT) kb_update(const Sys<T>* sys, const Chunk* ch, int to_x) {
  const Chunk C = ch[blockIdx.x];
  const Sys<T>& S = sys[C.sys];
  const GMState* st = S.st;
  if (st->done || st->k == 0) return;
  const int k = st->k;
  double* dst = to_x ? S.x : S.pt;
  CHUNK_LOOP(l, C) {
    double a = to_x ? dst[l] : 0.0;
    for (int i = 0; i < k; ++i) a = a + S.y[i] * (double)S.V[(int64_t)i * S.ld + l];
    dst[l] = a;
  }
}

// done[i] <- the system's done flag (one value per system, read by the host once per cycle)
template <typename T>
__global__ void kb_done(const Sys<T>* sys, int count, int* done) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) done[i] = sys[i].st->done;
}

}  // namespace

struct dgop_batch_solver {
  std::vector<dgop_operator*> ops, precs;
  int restart = 0;
  int inner = DGOP_FP32;
  std::vector<std::vector<int>> waves;  // system indices per wave
  void* arena = nullptr;                // FP64 and inner vectors of the largest wave
  size_t arena_bytes = 0;
  GMState* states = nullptr;            // one per system
  double* small = nullptr;              // H, cs, sn, e1, y per system
  double* part = nullptr;               // chunk partials of the largest wave
  int64_t max_chunks = 0;
  void* d_sys = nullptr;                // Sys<T> records of the current wave
  Chunk* d_chunks = nullptr;
  int* d_done = nullptr;
  int* h_done = nullptr;                // pinned
  cudaStream_t cap = nullptr;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  // the per-system applies of one step run as parallel branches of the graph: forked from the
  // capture stream onto kBranches streams and joined back (most systems fill only a few CTAs)
  cudaStream_t branch[16] = {};
  cudaEvent_t fork = nullptr, join[16] = {};
};

namespace {

size_t small_per_sys(int m) { return (size_t)(m + 1) * m + m + m + (m + 1) + m; }

template <typename T>
size_t sys_bytes(int64_t n, int m) {
  return sizeof(double) * 3 * stride64(n) + sizeof(T) * (size_t)(m + 3) * stride64(n);
}

void release(dgop_batch_solver* s) {
  if (s->arena) cudaFree(s->arena);
  if (s->states) cudaFree(s->states);
  if (s->small) cudaFree(s->small);
  if (s->part) cudaFree(s->part);
  if (s->d_sys) cudaFree(s->d_sys);
  if (s->d_chunks) cudaFree(s->d_chunks);
  if (s->d_done) cudaFree(s->d_done);
  if (s->h_done) cudaFreeHost(s->h_done);
  if (s->cap) cudaStreamDestroy(s->cap);
  if (s->t0) cudaEventDestroy(s->t0);
  if (s->t1) cudaEventDestroy(s->t1);
  for (int k = 0; k < 16; ++k) {
    if (s->branch[k]) cudaStreamDestroy(s->branch[k]);
    if (s->join[k]) cudaEventDestroy(s->join[k]);
  }
  if (s->fork) cudaEventDestroy(s->fork);
}

template <typename T>
int setup(dgop_batch_solver* s, double budget_bytes) {
  const int m = s->restart;
  const int count = (int)s->ops.size();
  // waves: systems in the given order, each wave's workspace within the budget
  std::vector<int> order(count);
  std::iota(order.begin(), order.end(), 0);
  size_t cur = 0, largest = 0;
  int64_t chunks = 0, max_chunks = 0;
  int max_wave = 0;
  s->waves.clear();
  s->waves.emplace_back();
  for (int i : order) {
    const int64_t n = s->ops[i]->sp.ndofs;
    const size_t bytes = sys_bytes<T>(n, m);
    const int64_t nch = (n + kChunk - 1) / kChunk;
    if (!s->waves.back().empty() && (double)(cur + bytes) > budget_bytes) {
      s->waves.emplace_back();
      cur = 0;
      chunks = 0;
    }
    s->waves.back().push_back(i);
    cur += bytes;
    chunks += nch;
    largest = std::max(largest, cur);
    max_chunks = std::max(max_chunks, chunks);
    max_wave = std::max(max_wave, (int)s->waves.back().size());
  }
  s->arena_bytes = largest;
  s->max_chunks = max_chunks;
  DGOP_CUDA_BS(cudaMalloc(&s->arena, largest));
  DGOP_CUDA_BS(cudaMalloc(&s->states, sizeof(GMState) * count));
  DGOP_CUDA_BS(cudaMemset(s->states, 0, sizeof(GMState) * count));
  DGOP_CUDA_BS(cudaMalloc(&s->small, sizeof(double) * small_per_sys(m) * count));
  DGOP_CUDA_BS(cudaMalloc(&s->part, sizeof(double) * (size_t)max_chunks * (m + 1)));
  DGOP_CUDA_BS(cudaMalloc(&s->d_sys, sizeof(Sys<T>) * max_wave));
  DGOP_CUDA_BS(cudaMalloc(&s->d_chunks, sizeof(Chunk) * max_chunks));
  DGOP_CUDA_BS(cudaMalloc(&s->d_done, sizeof(int) * max_wave));
  DGOP_CUDA_BS(cudaMallocHost(&s->h_done, sizeof(int) * max_wave));
  DGOP_CUDA_BS(cudaStreamCreateWithFlags(&s->cap, cudaStreamNonBlocking));
  DGOP_CUDA_BS(cudaEventCreate(&s->t0));
  DGOP_CUDA_BS(cudaEventCreate(&s->t1));
  DGOP_CUDA_BS(cudaEventCreateWithFlags(&s->fork, cudaEventDisableTiming));
  for (int k = 0; k < 16; ++k) {
    DGOP_CUDA_BS(cudaStreamCreateWithFlags(&s->branch[k], cudaStreamNonBlocking));
    DGOP_CUDA_BS(cudaEventCreateWithFlags(&s->join[k], cudaEventDisableTiming));
  }
  return DGOP_OK;
}

// Run body(k, stream) for every system k of a wave, spread over the branch streams after a fork
// from q and joined back into q (inside a capture these become parallel graph branches).
template <typename F>
int per_system(dgop_batch_solver* s, int count, cudaStream_t q, F&& body) {
  const int nb = std::min(count, 16);
  DGOP_CUDA_BS(cudaEventRecord(s->fork, q));
  for (int k = 0; k < nb; ++k) DGOP_CUDA_BS(cudaStreamWaitEvent(s->branch[k], s->fork, 0));
  for (int k = 0; k < count; ++k) DGOP_TRY_BS(body(k, s->branch[k % nb]));
  for (int k = 0; k < nb; ++k) {
    DGOP_CUDA_BS(cudaEventRecord(s->join[k], s->branch[k]));
    DGOP_CUDA_BS(cudaStreamWaitEvent(q, s->join[k], 0));
  }
  return DGOP_OK;
}

int inner_apply(dgop_operator* op, const float* x, float* y, cudaStream_t q, const int* skip) {
  return launch_f32(op, 1.0f, x, 0.0f, y, kLinear, q, skip);
}
int inner_apply(dgop_operator* op, const double* x, double* y, cudaStream_t q, const int* skip) {
  return launch_f64(op, 1.0, x, 0.0, y, kLinear, q, skip);
}

// Solve the systems of one wave.  `elapsed` (per system, may be null) receives the time from the
// start of the solve to the end of the cycle after which the system was found finished.
template <typename T>
int solve_wave(dgop_batch_solver* s, const std::vector<int>& wave, const double* const* b, double* const* x,
               int max_iters, double tol, cudaStream_t st, double* elapsed) {
  const int m = s->restart;
  const int count = (int)wave.size();
  const int pw = m + 1;
  std::vector<Sys<T>> sys(count);
  std::vector<Chunk> chunks;
  unsigned char* a = static_cast<unsigned char*>(s->arena);
  for (int k = 0; k < count; ++k) {
    const int i = wave[k];
    Sys<T>& S = sys[k];
    const int64_t n = s->ops[i]->sp.ndofs, ld = stride64(n);
    S.b = b[i];
    S.x = x[i];
    S.w64 = reinterpret_cast<double*>(a);
    S.r64 = S.w64 + ld;
    S.pt = S.r64 + ld;
    T* t = reinterpret_cast<T*>(S.pt + ld);
    S.w = t;
    S.z = t + ld;
    S.V = t + 2 * ld;
    a += sys_bytes<T>(n, m);
    S.n = n;
    S.ld = ld;
    S.c0 = (int64_t)chunks.size();
    for (int64_t c = 0; c < n; c += kChunk) chunks.push_back({k, c, std::min(n, c + kChunk)});
    S.c1 = (int64_t)chunks.size();
    S.st = s->states + i;
    double* sm = s->small + small_per_sys(m) * i;
    S.H = sm;
    S.cs = S.H + (m + 1) * m;
    S.sn = S.cs + m;
    S.e1 = S.sn + m;
    S.y = S.e1 + m + 1;
  }
  Sys<T>* dsys = static_cast<Sys<T>*>(s->d_sys);
  DGOP_CUDA_BS(cudaMemcpyAsync(dsys, sys.data(), sizeof(Sys<T>) * count, cudaMemcpyHostToDevice, st));
  DGOP_CUDA_BS(cudaMemcpyAsync(s->d_chunks, chunks.data(), sizeof(Chunk) * chunks.size(), cudaMemcpyHostToDevice, st));
  const unsigned nch = (unsigned)chunks.size();
  const unsigned sysb = (unsigned)((count + kBT - 1) / kBT);

  auto residual = [&](int phase, cudaStream_t q) -> int {
    DGOP_TRY_BS(per_system(s, count, q, [&](int k, cudaStream_t b) {
      return launch_f64(s->ops[wave[k]], 1.0, sys[k].x, 0.0, sys[k].w64, 0, b, &sys[k].st->done);
    }));
    kb_sub_norm<T><<<nch, kBT, 0, q>>>(dsys, s->d_chunks, s->part, pw);
    kb_resid<T><<<count, kBT, 0, q>>>(dsys, s->part, pw, phase);
    DGOP_CUDA_BS(cudaGetLastError());
    return DGOP_OK;
  };
  auto cycle = [&](cudaStream_t q) -> int {
    kb_cycle_start<T><<<sysb, kBT, 0, q>>>(dsys, count, m);
    kb_scale_v0<T><<<nch, kBT, 0, q>>>(dsys, s->d_chunks);
    for (int j = 0; j < m; ++j) {
      DGOP_TRY_BS(per_system(s, count, q, [&](int k, cudaStream_t b) {
        const int i = wave[k];
        const int* skip = &sys[k].st->inactive;
        T* vj = sys[k].V + (int64_t)j * sys[k].ld;
        if (s->precs[i]) {
          DGOP_TRY_BS(inner_apply(s->precs[i], vj, sys[k].z, b, skip));
          return inner_apply(s->ops[i], sys[k].z, sys[k].w, b, skip);
        }
        return inner_apply(s->ops[i], vj, sys[k].w, b, skip);
      }));
      kb_gs_dots<T><<<dim3(nch, (j + kDotsPerBlock) / kDotsPerBlock), kBT, 0, q>>>(dsys, s->d_chunks, j, s->part, pw);
      kb_gs_h<T><<<dim3(count, j + 1), kBT, 0, q>>>(dsys, j, m, s->part, pw);
      kb_gs_update<T><<<nch, kBT, 0, q>>>(dsys, s->d_chunks, j, m, s->part, pw);
      kb_column<T><<<count, kBT, 0, q>>>(dsys, j, m, s->part, pw);
      kb_rescale<T><<<nch, kBT, 0, q>>>(dsys, s->d_chunks, j);
      DGOP_CUDA_BS(cudaGetLastError());
    }
    kb_backsub<T><<<sysb, kBT, 0, q>>>(dsys, count, m);
    if (s->precs[wave[0]]) {
      // x += P (sum y_i V_i) (every system has a preconditioner: dgop_batch_solver_create)
      kb_update<T><<<nch, kBT, 0, q>>>(dsys, s->d_chunks, 0);
      DGOP_TRY_BS(per_system(s, count, q, [&](int k, cudaStream_t b) {
        return launch_f64(s->precs[wave[k]], 1.0, sys[k].pt, 1.0, sys[k].x, 0, b, &sys[k].st->done);
      }));
    } else {
      kb_update<T><<<nch, kBT, 0, q>>>(dsys, s->d_chunks, 1);
    }
    DGOP_CUDA_BS(cudaGetLastError());
    return residual(1, q);
  };

  kb_norm_b<T><<<nch, kBT, 0, st>>>(dsys, s->d_chunks, s->part, pw);
  kb_denom<T><<<count, kBT, 0, st>>>(dsys, s->part, pw, tol, max_iters);
  DGOP_CUDA_BS(cudaGetLastError());
  if (max_iters <= 0 || m <= 0) {
    DGOP_TRY_BS(residual(2, st));
  } else {
    DGOP_TRY_BS(residual(0, st));
    // one restart cycle of the whole wave as a graph, replayed until every system has finished
    DGOP_CUDA_BS(cudaStreamBeginCapture(s->cap, cudaStreamCaptureModeThreadLocal));
    const int crc = cycle(s->cap);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(s->cap, &graph);
    if (crc != DGOP_OK || ce != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return crc != DGOP_OK ? crc : cuda_fail(ce, "batched solver graph capture");
    }
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiateWithFlags(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) return cuda_fail(ie, "batched solver graph instantiation");
    std::vector<char> seen(count, 0);
    int rc = DGOP_OK;
    for (int c = 0; c <= max_iters; ++c) {
      cudaError_t e = cudaGraphLaunch(exec, st);
      if (e == cudaSuccess) {
        kb_done<T><<<sysb, kBT, 0, st>>>(dsys, count, s->d_done);
        e = cudaMemcpyAsync(s->h_done, s->d_done, sizeof(int) * count, cudaMemcpyDeviceToHost, st);
      }
      if (e == cudaSuccess) e = cudaEventRecord(s->t1, st);
      if (e == cudaSuccess) e = cudaEventSynchronize(s->t1);
      if (e != cudaSuccess) {
        rc = cuda_fail(e, "batched solver cycle");
        break;
      }
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, s->t0, s->t1);
      int ndone = 0;
      for (int k = 0; k < count; ++k) {
        if (s->h_done[k]) {
          ++ndone;
          if (!seen[k] && elapsed) elapsed[wave[k]] = ms * 1e-3;
          seen[k] = 1;
        }
      }
      if (ndone == count) break;
    }
    cudaGraphExecDestroy(exec);
    if (rc != DGOP_OK) return rc;
  }
  return DGOP_OK;
}

template <typename T>
int solve_all(dgop_batch_solver* s, const double* const* b, double* const* x, int max_iters, double tol,
              dgop_solve_result* results, double* seconds, cudaStream_t st) {
  const int count = (int)s->ops.size();
  DGOP_CUDA_BS(cudaEventRecord(s->t0, st));
  for (const auto& wave : s->waves) DGOP_TRY_BS(solve_wave<T>(s, wave, b, x, max_iters, tol, st, seconds));
  std::vector<GMState> h(count);
  DGOP_CUDA_BS(cudaMemcpyAsync(h.data(), s->states, sizeof(GMState) * count, cudaMemcpyDeviceToHost, st));
  DGOP_CUDA_BS(cudaStreamSynchronize(st));
  for (int i = 0; i < count; ++i) {
    results[i].success = h[i].success;
    results[i].iterations = h[i].iters;
    results[i].relative_error = h[i].rel;
  }
  if (seconds) {
    // systems that finished during the residual before the first cycle
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, s->t0, s->t1);
    for (int i = 0; i < count; ++i)
      if (seconds[i] < 0.0) seconds[i] = ms * 1e-3;
  }
  return DGOP_OK;
}

}  // namespace

extern "C" {

int dgop_batch_solver_create(dgop_operator* const* ops, dgop_operator* const* precs, int count, int restart,
                             int inner_precision, double workspace_bytes, dgop_batch_solver** out) {
  if (!ops || !out || count < 1 || restart < 1 || restart > 1000) {
    set_error("dgop_batch_solver_create: bad arguments");
    return DGOP_ERR_ARG;
  }
  if (inner_precision != DGOP_FP32 && inner_precision != DGOP_FP64) {
    set_error("dgop_batch_solver_create: inner precision must be DGOP_FP32 or DGOP_FP64");
    return DGOP_ERR_ARG;
  }
  *out = nullptr;
  auto* s = new (std::nothrow) dgop_batch_solver();
  if (!s) {
    set_error("host allocation failed");
    return DGOP_ERR_ALLOC;
  }
  s->restart = restart;
  s->inner = inner_precision;
  bool with = false, without = false;
  for (int i = 0; i < count; ++i) {
    dgop_operator* P = precs ? precs[i] : nullptr;
    if (!ops[i] || (P && P->sp.ndofs != ops[i]->sp.ndofs)) {
      delete s;
      set_error("dgop_batch_solver_create: null operator or preconditioner of another size");
      return DGOP_ERR_ARG;
    }
    if (inner_precision == DGOP_FP32 && !ops[i]->f32.ready && !ops[i]->k32.ready && !ops[i]->n32.ready) {
      delete s;
      set_error("dgop_batch_solver_create: an operator has no FP32 kernel");
      return DGOP_ERR_UNSUPPORTED;
    }
    (P ? with : without) = true;
    s->ops.push_back(ops[i]);
    s->precs.push_back(P);
  }
  if (with && without) {
    delete s;
    set_error("dgop_batch_solver_create: give every system a preconditioner or none");
    return DGOP_ERR_ARG;
  }
  double budget = workspace_bytes;
  if (budget <= 0.0) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      delete s;
      set_error("cudaMemGetInfo failed");
      return DGOP_ERR_CUDA;
    }
    budget = 0.5 * (double)free_b;
  }
  const int rc = inner_precision == DGOP_FP32 ? setup<float>(s, budget) : setup<double>(s, budget);
  if (rc != DGOP_OK) {
    release(s);
    delete s;
    return rc;
  }
  *out = s;
  return DGOP_OK;
}

int dgop_batch_solver_waves(const dgop_batch_solver* s) { return s ? (int)s->waves.size() : -1; }

int dgop_batch_solver_solve(dgop_batch_solver* s, const double* const* b, double* const* x, int max_iters,
                            double tol, dgop_solve_result* results, double* seconds, void* stream) {
  if (!s || !b || !x || !results || !(tol >= 0.0)) {
    set_error("dgop_batch_solver_solve: bad arguments");
    return DGOP_ERR_ARG;
  }
  const int count = (int)s->ops.size();
  for (int i = 0; i < count; ++i) {
    if (!b[i] || !x[i] || b[i] == x[i] || reinterpret_cast<uintptr_t>(x[i]) % 16 ||
        reinterpret_cast<uintptr_t>(b[i]) % 8) {
      set_error("dgop_batch_solver_solve: null, aliasing or misaligned vectors");
      return DGOP_ERR_ARG;
    }
    if (seconds) seconds[i] = -1.0;
  }
  cudaStream_t st = (cudaStream_t)stream;
  return s->inner == DGOP_FP32 ? solve_all<float>(s, b, x, max_iters, tol, results, seconds, st)
                               : solve_all<double>(s, b, x, max_iters, tol, results, seconds, st);
}

int dgop_batch_solver_destroy(dgop_batch_solver* s) {
  if (!s) return DGOP_OK;
  release(s);
  delete s;
  return DGOP_OK;
}

}  // extern "C"
