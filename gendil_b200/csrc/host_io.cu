// Operator applies on host vectors: y_host = A x_host with the host-to-device copy, the apply
// and the device-to-host copy pipelined over slabs of element planes.
//
// The element index runs x fastest, so the planes of the last axis are contiguous ranges of
// elements and DoFs.  Slab k of the input is uploaded on one stream; the apply of slab k starts
// on a second stream once the slabs it reads are on the device (itself and, for operators with
// faces, the next slab; with a periodic last axis the first slab also reads the last one); the
// result of slab k goes back on a third stream as soon as its apply is done.  Upload and download
// use the two copy directions at once, so a host apply costs about one transfer of the vector
// instead of two.
//
// The device copies are double-buffered: consecutive asynchronous applies alternate between two
// (x, y) pairs, so the uploads of one apply run while the downloads of the previous one finish.
// An apply waits only for what reuses its buffers: its uploads for the applies that read the
// pair two calls earlier, its applies for the downloads of that call; and its uploads for the
// downloads of an earlier call whose result vector overlaps its input (chained applies).
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <vector>

#include "dgop_internal.h"

using namespace dgop;

struct dgop_host_io {
  dgop_operator* op = nullptr;
  double* x[2] = {nullptr, nullptr};  // device copies of the input and the result, two pairs
  double* y[2] = {nullptr, nullptr};
  cudaEvent_t read_done[2] = {nullptr, nullptr};  // the last applies that read x[b]
  cudaEvent_t sent[2] = {nullptr, nullptr};       // the last downloads of y[b]
  unsigned calls = 0;
  const double* y_host[2] = {nullptr, nullptr};  // result vector of the last call on pair b
  cudaStream_t up = nullptr, run = nullptr, down = nullptr;
  cudaEvent_t start = nullptr, finished = nullptr;
  std::vector<cudaEvent_t> uploaded, applied;
  std::vector<int64_t> first;  // first element of slab k; first[slabs] = number of elements
};

namespace {

#define DGOP_CUDA_H(call)                               \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

#define DGOP_TRY_H(call)            \
  do {                              \
    const int _rc = (call);         \
    if (_rc != DGOP_OK) return _rc; \
  } while (0)

void release(dgop_host_io* io) {
  for (int b = 0; b < 2; ++b) {
    if (io->x[b]) cudaFree(io->x[b]);
    if (io->y[b]) cudaFree(io->y[b]);
    if (io->read_done[b]) cudaEventDestroy(io->read_done[b]);
    if (io->sent[b]) cudaEventDestroy(io->sent[b]);
  }
  for (cudaStream_t s : {io->up, io->run, io->down})
    if (s) cudaStreamDestroy(s);
  for (cudaEvent_t e : {io->start, io->finished})
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : io->uploaded)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : io->applied)
    if (e) cudaEventDestroy(e);
}

int setup(dgop_host_io* io, int slabs) {
  const dgop_space& sp = io->op->sp;
  const int last = sp.D - 1;
  const int64_t planes = sp.sizes[last];
  const int64_t per_plane = sp.nelem / planes;
  const int k = (int)std::max<int64_t>(1, std::min<int64_t>(slabs, planes));
  for (int i = 0; i <= k; ++i) io->first.push_back(per_plane * ((planes * i) / k));
  for (int b = 0; b < 2; ++b) {
    DGOP_CUDA_H(cudaMalloc(&io->x[b], sizeof(double) * sp.ndofs));
    DGOP_CUDA_H(cudaMalloc(&io->y[b], sizeof(double) * sp.ndofs));
    DGOP_CUDA_H(cudaEventCreateWithFlags(&io->read_done[b], cudaEventDisableTiming));
    DGOP_CUDA_H(cudaEventCreateWithFlags(&io->sent[b], cudaEventDisableTiming));
  }
  DGOP_CUDA_H(cudaStreamCreateWithFlags(&io->up, cudaStreamNonBlocking));
  DGOP_CUDA_H(cudaStreamCreateWithFlags(&io->run, cudaStreamNonBlocking));
  DGOP_CUDA_H(cudaStreamCreateWithFlags(&io->down, cudaStreamNonBlocking));
  DGOP_CUDA_H(cudaEventCreateWithFlags(&io->start, cudaEventDisableTiming));
  DGOP_CUDA_H(cudaEventCreateWithFlags(&io->finished, cudaEventDisableTiming));
  io->uploaded.assign(k, nullptr);
  io->applied.assign(k, nullptr);
  for (int i = 0; i < k; ++i) {
    DGOP_CUDA_H(cudaEventCreateWithFlags(&io->uploaded[i], cudaEventDisableTiming));
    DGOP_CUDA_H(cudaEventCreateWithFlags(&io->applied[i], cudaEventDisableTiming));
  }
  return DGOP_OK;
}

}  // namespace

extern "C" {

int dgop_host_io_create(dgop_operator* op, int slabs, dgop_host_io** out) {
  if (!op || !out) {
    set_error("dgop_host_io_create: null argument");
    return DGOP_ERR_ARG;
  }
  *out = nullptr;
  auto* io = new (std::nothrow) dgop_host_io();
  if (!io) {
    set_error("host allocation failed");
    return DGOP_ERR_ALLOC;
  }
  io->op = op;
  const int rc = setup(io, slabs > 0 ? slabs : 8);
  if (rc != DGOP_OK) {
    release(io);
    delete io;
    return rc;
  }
  *out = io;
  return DGOP_OK;
}

int dgop_host_io_apply_async(dgop_host_io* io, const double* x_host, double* y_host, void* stream) {
  if (!io || !x_host || !y_host) {
    set_error("dgop_host_io_apply: null argument");
    return DGOP_ERR_ARG;
  }
  const dgop_space& sp = io->op->sp;
  const int k = (int)io->uploaded.size();
  const int64_t nd = sp.ndofs / sp.nelem;  // DoFs per element
  const bool faces = (io->op->flags & (kFaceInt | kFaceBnd)) != 0;
  const bool wrap = faces && sp.periodic[sp.D - 1] && k > 1;
  cudaStream_t user = (cudaStream_t)stream;
  const int b = (int)(io->calls & 1u);
  double* x = io->x[b];
  double* y = io->y[b];
  // the copies start after the work already queued on the caller's stream, and once the applies
  // of the call two back (same device pair) no longer read x
  DGOP_CUDA_H(cudaEventRecord(io->start, user));
  DGOP_CUDA_H(cudaStreamWaitEvent(io->up, io->start, 0));
  if (io->calls >= 2) DGOP_CUDA_H(cudaStreamWaitEvent(io->up, io->read_done[b], 0));
  for (int c = 0; c < 2; ++c) {
    const double* yp = io->y_host[c];
    if (yp && x_host < yp + sp.ndofs && yp < x_host + sp.ndofs)
      DGOP_CUDA_H(cudaStreamWaitEvent(io->up, io->sent[c], 0));
  }
  for (int i = 0; i < k; ++i) {
    const int64_t d0 = io->first[i] * nd, dn = (io->first[i + 1] - io->first[i]) * nd;
    DGOP_CUDA_H(cudaMemcpyAsync(x + d0, x_host + d0, sizeof(double) * dn, cudaMemcpyHostToDevice, io->up));
    DGOP_CUDA_H(cudaEventRecord(io->uploaded[i], io->up));
  }
  // y is rewritten once the downloads of the call two back are done
  if (io->calls >= 2) DGOP_CUDA_H(cudaStreamWaitEvent(io->run, io->sent[b], 0));
  for (int i = 0; i < k; ++i) {
    // slabs i - 1 .. i + 1 are read; uploads complete in order, so waiting for the highest is enough
    const int need = (wrap && i == 0) ? k - 1 : (faces ? std::min(i + 1, k - 1) : i);
    DGOP_CUDA_H(cudaStreamWaitEvent(io->run, io->uploaded[need], 0));
    DGOP_TRY_H(launch_range_f64(io->op, x, y, io->first[i], io->first[i + 1], io->run));
    DGOP_CUDA_H(cudaEventRecord(io->applied[i], io->run));
    DGOP_CUDA_H(cudaStreamWaitEvent(io->down, io->applied[i], 0));
    const int64_t d0 = io->first[i] * nd, dn = (io->first[i + 1] - io->first[i]) * nd;
    DGOP_CUDA_H(cudaMemcpyAsync(y_host + d0, y + d0, sizeof(double) * dn, cudaMemcpyDeviceToHost, io->down));
  }
  DGOP_CUDA_H(cudaEventRecord(io->read_done[b], io->run));
  DGOP_CUDA_H(cudaEventRecord(io->sent[b], io->down));
  DGOP_CUDA_H(cudaEventRecord(io->finished, io->down));
  io->y_host[b] = y_host;
  ++io->calls;
  return DGOP_OK;
}

int dgop_host_io_wait(dgop_host_io* io, void* stream) {
  if (!io) {
    set_error("dgop_host_io_wait: null argument");
    return DGOP_ERR_ARG;
  }
  DGOP_CUDA_H(cudaStreamWaitEvent((cudaStream_t)stream, io->finished, 0));
  return DGOP_OK;
}

int dgop_host_io_apply(dgop_host_io* io, const double* x_host, double* y_host, void* stream) {
  DGOP_TRY_H(dgop_host_io_apply_async(io, x_host, y_host, stream));
  DGOP_TRY_H(dgop_host_io_wait(io, stream));
  DGOP_CUDA_H(cudaEventSynchronize(io->finished));
  return DGOP_OK;
}

int dgop_host_io_destroy(dgop_host_io* io) {
  if (!io) return DGOP_OK;
  cudaStreamSynchronize(io->down);
  release(io);
  delete io;
  return DGOP_OK;
}

}  // extern "C"
