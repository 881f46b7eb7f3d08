// Parameters of the bulk-tensor (TMA) variants of the 3D Kronecker-form kernel
// (kron3d_tma_kernel.cuh), shared by the kernel and the host dispatcher.
#pragma once

#include <cuda.h>

#include <cstdint>

#include "kron.h"

namespace dgop {

// Face word of an element (kron_face_words): per face f = 2 a + s, 5 bits: kRecCorner, kRecNb,
// kRecG and the trace source in bits 3-4: 0 the group's own planes (x faces), 1 the group's
// staged slice slot of that axis (for x: the neighbour element staged beside the group, in the
// variants that stage it; the others read it from global memory), 2 global memory.
enum : uint32_t { kTmaSrcGroup = 0u, kTmaSrcSlot = 1u, kTmaSrcGlobal = 2u };
// Group word: bits 0-1 y slot, bits 2-3 z slot: 0 none, 1 the - side neighbours, 2 the + side;
// bits 4-5 x slot: 0 none, 1 the - side neighbour of element 0, 2 the + side neighbour of element 7.

template <typename Real>
struct KronTmaParams {
  CUtensorMap win;   // x as rows of 16 values: box 16 x 32 (one group), 128 B swizzle
  CUtensorMap zsl;   // x as (16, 4 z slices, elements): box 16 x 1 x 8, 128 B swizzle
  CUtensorMap ysl;   // x as (4 x, 4 y, 4 z, elements): box 4 x 1 x 4 x 8
  CUtensorMap xel;   // x as rows of 16 values: box 16 x 4 (one element), no swizzle
  CUtensorMap out;   // y as rows of 16 values: box 16 x 32, 128 B swizzle
  KronParams<Real> k;
  const uint32_t* eflags;  // face word per element
  const uint32_t* gwords;  // slot word per group of 8 elements (group = element / 8)
  int* err;                // set when a bounded wait gives up
  // element-dependent matrices of the slots acting along y or z (one coordinate for the whole
  // group): mat_index[slot] is the matrix's place in the stage's matrix area, -1 when the slot
  // is constant or acts along x; nmat of them per group
  int mat_index[kNumSlots];
  int nmat;
};

// Slot k of the slots acting along y (k < 4, coordinate c[1]) and along z (k >= 4, c[2]).
#ifdef __CUDACC__
__host__ __device__
#endif
constexpr int tma_yz_slot(int k) {
  return k == 0 ? kSlotDY : k == 1 ? kSlotTXY : k == 2 ? kSlotTZY : k == 3 ? kSlotMY
       : k == 4 ? kSlotDZ : k == 5 ? kSlotTXZ : k == 6 ? kSlotTYZ : kSlotMD;
}
constexpr int kTmaMatBytes = 16 * 8;  // one 4 x 4 FP64 matrix

constexpr int kTmaGroupBytes = 4096, kTmaSlotBytes = 1024;
// planes, z slot, y slot, up to 8 matrices (1 KB; the stage stays a multiple of 1024 bytes)
constexpr int kTmaStageBytes = kTmaGroupBytes + 3 * kTmaSlotBytes;
constexpr int kTmaTileBytes = 5120;  // exchange tile (8 elements x 78 doubles, rounded up)
constexpr int kTmaElemBytes = 512;   // one element (the x slot, staged in the idle exchange tile)
constexpr int kTmaWarps = 2;         // warps per CTA
constexpr int tma_warp_bytes(int stages, bool shfl) { return stages * kTmaStageBytes + (shfl ? 0 : kTmaTileBytes); }
constexpr int kTmaMaxWaitIters = 1 << 24;                  // polls of one wait, at most
constexpr unsigned long long kTmaWaitNs = 1000000000ull;   // and one second of wall time

}  // namespace dgop
