// Batches of independent operators: one persistent launch per (dimension, order) class.
//
// Operators on the any-dimension Kronecker kernel are grouped by (D, N, kernel variant); each
// group's parameter
// table (the operators' forward parameters, x and y patched per apply) and the prefix sums of
// their element batches live on the device, and one launch of kronnd_batch_kernel walks every
// element batch of every operator of the group.  Operators on another kernel are applied one
// launch each.  Results equal those of the operators' own applies bit for bit (same arithmetic).
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <tuple>
#include <new>
#include <vector>

#include "dgop_internal.h"

using namespace dgop;

namespace {
struct BatchGroup {
  const KronNDEntry<double>* entry = nullptr;
  int variant = 0;
  std::vector<int> members;                 // indices into the batch
  std::vector<KronNDParams<double>> table;  // host copy (x, y patched per apply)
  std::vector<int64_t> first;
  KronNDParams<double>* d_table = nullptr;
  int64_t* d_first = nullptr;
  KronNDParams<double>* h_pinned = nullptr;  // staging of the table upload
  int eb = 1;
  size_t smem = 0;
  dim3 grid, block;
};
}  // namespace

struct dgop_batch {
  std::vector<dgop_operator*> ops;
  std::vector<BatchGroup> groups;
  std::vector<int> singles;  // operators applied one launch each
  cudaEvent_t uploaded = nullptr;
};

namespace {

#define DGOP_CUDA_B(call)                               \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

void release(dgop_batch* b) {
  for (auto& g : b->groups) {
    if (g.d_table) cudaFree(g.d_table);
    if (g.d_first) cudaFree(g.d_first);
    if (g.h_pinned) cudaFreeHost(g.h_pinned);
  }
  if (b->uploaded) cudaEventDestroy(b->uploaded);
}

int setup(dgop_batch* b) {
  int sms = 0, dev = 0;
  DGOP_CUDA_B(cudaGetDevice(&dev));
  DGOP_CUDA_B(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int max_smem = 0;
  DGOP_CUDA_B(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  std::map<const void*, int> per_sm_of;  // resident CTAs per SM of each batch kernel used
  std::map<std::tuple<int, int, int>, int> index;
  for (int i = 0; i < (int)b->ops.size(); ++i) {
    dgop_operator* op = b->ops[i];
    const int v = op->n64.variant;
    if (op->kernel != DGOP_KERNEL_KRONND || !op->n64.ready || !op->n64.entry->launch_batch[v]) {
      b->singles.push_back(i);
      continue;
    }
    const void* fn = op->n64.entry->func_batch[v];
    auto pit = per_sm_of.find(fn);
    if (pit == per_sm_of.end()) {
      cudaFuncAttributes fa{};
      DGOP_CUDA_B(cudaFuncGetAttributes(&fa, fn));
      DGOP_CUDA_B(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       max_smem - (int)fa.sharedSizeBytes));
      int per_sm = 0;
      DGOP_CUDA_B(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, (int)op->n64.block.x,
                                                                op->n64.var[v].smem));
      pit = per_sm_of.emplace(fn, per_sm < 1 ? 1 : per_sm).first;
    }
    // an instance whose element batches fill every CTA slot twice over keeps its own launch (its
    // parameters in constant memory, no per-batch instance lookup): the persistent kernel gains
    // nothing there and measured a few per cent slower
    const int64_t eb = op->n64.var[v].eb;
    if ((op->sp.nelem + eb - 1) / eb >= 2 * (int64_t)sms * pit->second) {
      b->singles.push_back(i);
      continue;
    }
    const auto key = std::make_tuple(op->sp.D, op->sp.n, v);
    auto it = index.find(key);
    if (it == index.end()) {
      it = index.emplace(key, (int)b->groups.size()).first;
      b->groups.emplace_back();
      b->groups.back().entry = op->n64.entry;
      b->groups.back().variant = v;
      b->groups.back().eb = op->n64.var[v].eb;
      b->groups.back().smem = op->n64.var[v].smem;
      b->groups.back().block = op->n64.block;
    }
    b->groups[it->second].members.push_back(i);
  }
  for (auto& g : b->groups) {
    g.first.push_back(0);
    for (int i : g.members) {
      dgop_operator* op = b->ops[i];
      KronNDParams<double> p = op->n64.params;
      p.eb = g.eb;
      p.e_begin = 0;
      p.nelem = op->sp.nelem;
      p.alpha = 1.0;
      p.beta_y = 0.0;
      p.flags = op->flags;
      p.skip = nullptr;
      g.table.push_back(p);
      g.first.push_back(g.first.back() + (op->sp.nelem + g.eb - 1) / g.eb);
    }
    const size_t tb = sizeof(KronNDParams<double>) * g.table.size();
    DGOP_CUDA_B(cudaMalloc(&g.d_table, tb));
    DGOP_CUDA_B(cudaMallocHost(&g.h_pinned, tb));
    DGOP_CUDA_B(cudaMalloc(&g.d_first, sizeof(int64_t) * g.first.size()));
    DGOP_CUDA_B(cudaMemcpy(g.d_first, g.first.data(), sizeof(int64_t) * g.first.size(), cudaMemcpyHostToDevice));
    const int per_sm = per_sm_of[g.entry->func_batch[g.variant]];
    g.grid = dim3((unsigned)std::max<int64_t>(1, std::min<int64_t>(g.first.back(), (int64_t)sms * per_sm)));
  }
  DGOP_CUDA_B(cudaEventCreateWithFlags(&b->uploaded, cudaEventDisableTiming));
  return DGOP_OK;
}

}  // namespace

extern "C" {

int dgop_batch_create(dgop_operator* const* ops, int count, dgop_batch** out) {
  if (!ops || !out || count < 1) {
    set_error("dgop_batch_create: bad arguments");
    return DGOP_ERR_ARG;
  }
  *out = nullptr;
  auto* b = new (std::nothrow) dgop_batch();
  if (!b) {
    set_error("host allocation failed");
    return DGOP_ERR_ALLOC;
  }
  for (int i = 0; i < count; ++i) {
    if (!ops[i]) {
      delete b;
      set_error("dgop_batch_create: null operator");
      return DGOP_ERR_ARG;
    }
    b->ops.push_back(ops[i]);
  }
  const int rc = setup(b);
  if (rc != DGOP_OK) {
    release(b);
    delete b;
    return rc;
  }
  *out = b;
  return DGOP_OK;
}

int dgop_batch_groups(const dgop_batch* b) { return b ? (int)b->groups.size() : -1; }

int dgop_batch_apply(dgop_batch* b, const double* const* x, double* const* y, void* stream) {
  if (!b || !x || !y) {
    set_error("dgop_batch_apply: null argument");
    return DGOP_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  // the staging buffers of the previous apply may still be in flight
  DGOP_CUDA_B(cudaEventSynchronize(b->uploaded));
  for (auto& g : b->groups) {
    for (size_t k = 0; k < g.members.size(); ++k) {
      const int i = g.members[k];
      if (!x[i] || !y[i] || x[i] == y[i]) {
        set_error("dgop_batch_apply: null or aliasing vectors");
        return DGOP_ERR_ARG;
      }
      g.h_pinned[k] = g.table[k];
      g.h_pinned[k].x = x[i];
      g.h_pinned[k].y = y[i];
    }
    DGOP_CUDA_B(cudaMemcpyAsync(g.d_table, g.h_pinned, sizeof(KronNDParams<double>) * g.members.size(),
                                cudaMemcpyHostToDevice, st));
    g.entry->launch_batch[g.variant](g.d_table, g.d_first, (int)g.members.size(), g.eb, g.grid, g.block, g.smem,
                                     st);
    DGOP_CUDA_B(cudaGetLastError());
  }
  DGOP_CUDA_B(cudaEventRecord(b->uploaded, st));
  for (int i : b->singles) {
    const int rc = dgop_apply(b->ops[i], x[i], y[i], stream);
    if (rc != DGOP_OK) return rc;
  }
  return DGOP_OK;
}

int dgop_batch_destroy(dgop_batch* b) {
  if (!b) return DGOP_OK;
  if (b->uploaded) cudaEventSynchronize(b->uploaded);
  release(b);
  delete b;
  return DGOP_OK;
}

}  // extern "C"
