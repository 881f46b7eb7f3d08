// Kronecker-form DG operator kernel for 3D hexahedra, N = p + 1 = 4, FP64, with element blocks
// moved by the Tensor Memory Accelerator.
//
// Same arithmetic and per-element schedule as kron3d_kernel (9 register-resident n x n passes,
// lane t of an element's 4 lanes holding plane t), different data movement:
//
//  * A warp owns groups of 8 consecutive elements of one x-row (the mesh's x extent is a multiple
//    of 8).  The group's 32 planes (128 B each, 4 KB contiguous in x) arrive in shared memory
//    by ONE cp.async.bulk.tensor load under 128-byte swizzle: plane row r lands with its 16-byte
//    chunk c at chunk c ^ (r & 7), so the 8 lanes of a 128-bit access phase (two elements x four
//    planes) hit 8 different bank groups.  The load completes on an mbarrier (expect_tx), issued
//    by lane 0, waited on by every lane with an iteration limit.
//  * The neighbour slices the group's inflow faces need come in the same transaction: the y
//    neighbours' slices of all 8 elements as one 4D box (x, 1 slice, z, 8 elements; 1 KB) and the
//    z neighbours' slices as one 3D box (16, 1 slice, 8 elements; 1 KB, swizzled).  Which side
//    (if any) a group needs per axis is precomputed per group; x neighbours inside the group are
//    read from the group's own planes, the rest (group ends, periodic wraps, a second side on one
//    axis) straight from global memory (L2-resident: the neighbouring groups were just staged).
//  * The upwind decisions of every face are precomputed per element at operator creation
//    (kron_face_words below); the kernel reads one 32-bit word per element and the face
//    coefficients from the per-axis tables.
//  * Results are written back into the group's planes (same swizzle) and leave with ONE
//    bulk-tensor store; with DOT an epilogue accumulates <z, y> (z = the input, or any vector)
//    into per-CTA partial sums in a fixed order (Krylov inner products without another pass).
//
// Shared memory per warp: STAGES x (4 KB planes + 1 KB z slices + 1 KB y slices), plus the
// exchange tile unless the layout exchanges are shuffle butterflies.  Every swizzled buffer is
// 1024-byte aligned (the swizzle pattern repeats every 8 rows of 128 B).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "kron3d_kernel.cuh"
#include "kron_tma.h"

namespace dgop {

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// Wait for the phase with the given parity by non-blocking polls, backing off after the first
// ones; false when neither the phase completed within kTmaWaitNs of wall time nor within
// kTmaMaxWaitIters polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  const uint64_t t0 = global_ns();
  for (int i = 0; i < kTmaMaxWaitIters; ++i) {
    if (mbar_test_wait(bar, parity)) return true;
    if (i >= 64) {
      __nanosleep(64);
      if ((i & 63) == 0 && global_ns() - t0 > kTmaWaitNs) return false;
    }
  }
  return false;
}
__device__ __forceinline__ void fence_barrier_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
          "r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];\n" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int c0, int c1, const void* src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(c0), "r"(c1), "r"(smem_addr(src))
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

// Double index of value c (0..15) of plane row r in a 128 B-swizzled, 1024-byte aligned buffer.
__device__ __forceinline__ int swz(int r, int c) { return r * 16 + ((((c >> 1) ^ (r & 7))) << 1) + (c & 1); }

// 16-byte shared-memory accesses by byte address.  In a 1024-byte aligned buffer, chunk k of
// row r sits at base + r * 128 + ((k ^ (r & 7)) << 4), and since base + r * 128 has bits 4-6
// clear that is ((base + r * 128) | ((r & 7) << 4)) ^ (k << 4): one XOR per access with a
// per-lane row address computed once.
__device__ __forceinline__ double2 lds_v2(uint32_t a) {
  double2 v;
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];\n" : "=d"(v.x), "=d"(v.y) : "r"(a));
  return v;
}
__device__ __forceinline__ void sts_v2(uint32_t a, double x, double y) {
  asm volatile("st.shared.v2.f64 [%0], {%1, %2};\n" ::"r"(a), "d"(x), "d"(y) : "memory");
}
// Row address of plane row r with its swizzle pattern folded in (see above).
__device__ __forceinline__ uint32_t swz_row(uint32_t base, int r) {
  return (base + (uint32_t)r * 128u) | ((uint32_t)(r & 7) << 4);
}

// Plane t of group element le in layout Z (values [x][y]) / layout Y (plane y = t, values [x][z]).
__device__ __forceinline__ void tma_plane_z(uint32_t grp_sa, int le, int t, double (&u)[4][4]) {
  const uint32_t row = swz_row(grp_sa, 4 * le + t);
#pragma unroll
  for (int y = 0; y < 4; ++y)
#pragma unroll
    for (int x = 0; x < 4; x += 2) {
      const double2 v = lds_v2(row ^ ((uint32_t)(2 * y + x / 2) << 4));  // chunk (4 y + x) / 2
      u[x][y] = v.x;
      u[x + 1][y] = v.y;
    }
}
// Rows 4 le + z, chunk 2 t + x / 2: with l = le & 1 the swizzled chunk is (2 t ^ 4 l) ^ (x / 2 ^ z),
// a per-lane part and a compile-time part; row z adds z * 128 (bits 7-8, clear in the base).
__device__ __forceinline__ void tma_plane_y(uint32_t grp_sa, int le, int t, double (&u)[4][4]) {
  const uint32_t row = (grp_sa + (uint32_t)le * 512u) | ((uint32_t)((2 * t) ^ (4 * (le & 1))) << 4);
#pragma unroll
  for (int z = 0; z < 4; ++z)
#pragma unroll
    for (int x = 0; x < 4; x += 2) {
      const double2 v = lds_v2((row ^ ((uint32_t)((x / 2) ^ z) << 4)) + (uint32_t)z * 128u);
      u[x][z] = v.x;
      u[x + 1][z] = v.y;
    }
}

// Y += A X along the first (FIRST) or second plane index: the products accumulate onto Y in the
// same order as a fresh pass would build them (one fused multiply-add chain per value).
template <bool FIRST, typename Mat>
__device__ __forceinline__ void pass_acc(const Mat& A, const double (&X)[4][4], double (&Y)[4][4]) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      double s = Y[i][j];
#pragma unroll
      for (int r = 0; r < 4; ++r) s += FIRST ? A(i, r) * X[r][j] : A(j, r) * X[i][r];
      Y[i][j] = s;
    }
}

// Slot SLOT's matrix applied along the first (FIRST) or second plane index, Y = A X or, with
// ACC, Y += A X.  Constant matrices come from kernel-parameter space; element-dependent ones from
// the stage's matrix area when the group staged them (slots along y or z), otherwise from global
// memory (slots along x, whose coordinate differs between the group's elements).
template <uint32_t VM, int SLOT, bool FIRST, bool ACC>
__device__ __forceinline__ void tma_apply(const KronTmaParams<double>& T, uint32_t coord, const double* mats,
                                          const double (&X)[4][4], double (&Y)[4][4]) {
  const KronParams<double>& P = T.k;
  bool vary;
  if constexpr (VM == kVaryRuntime) vary = P.vary[SLOT] != 0;
  else vary = ((VM >> SLOT) & 1u) != 0;
  if (vary) {
    RegMat<4, double> A;
    const int mi = T.mat_index[SLOT];
    if (mi >= 0) {
      const double* q = mats + mi * 16;
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; j += 2) {
          const double2 v = *reinterpret_cast<const double2*>(q + i * 4 + j);
          A.a[i][j] = v.x;
          A.a[i][j + 1] = v.y;
        }
    } else {
      const double* q = P.mats + P.vm[SLOT].off + (int64_t)coord * P.vm[SLOT].stride;
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; j += 2) {
          const double2 v = __ldg(reinterpret_cast<const double2*>(q + i * 4 + j));
          A.a[i][j] = v.x;
          A.a[i][j + 1] = v.y;
        }
    }
    if constexpr (ACC) pass_acc<FIRST>(A, X, Y);
    else if constexpr (FIRST) apply_first<4>(A, X, Y);
    else apply_second<4>(A, X, Y);
  } else {
    ParamMat<4, double, SLOT> A{P};
    if constexpr (ACC) pass_acc<FIRST>(A, X, Y);
    else if constexpr (FIRST) apply_first<4>(A, X, Y);
    else apply_second<4>(A, X, Y);
  }
}

// Face terms of axis a added to the D-pass output Pm (slice along the first plane index when
// FIRST), with the coefficients read from the per-axis tables: the corner (own outflow) term
// phi_s(e_a) el_a(e) and the inflow term (forward: the same coefficient; transposed: the
// neighbour's phi at its opposite face times its factor).  nbrow(s, src, d, v) fetches this lane's
// row of the neighbour trace.
// ph holds phi_0(e_a), phi_1(e_a): the caller loads it (one 16-byte load) before the D pass of
// axis a, so the pass covers the load's latency.
__device__ __forceinline__ double2 tma_phi(const KronParams<double>& P, int a, const uint32_t (&c)[3]) {
  return __ldg(reinterpret_cast<const double2*>(P.phi[a] + c[a] * 2));
}

template <bool FIRST, typename NbRow>
__device__ __forceinline__ void tma_faces(const KronParams<double>& P, int a, const uint32_t (&c)[3], int64_t e,
                                          uint32_t ef, double el, double2 ph, const double (&U)[4][4],
                                          double (&Pm)[4][4], NbRow nbrow) {
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const int sl = s ? 3 : 0;
    const uint32_t f = (ef >> (5 * (a * 2 + s))) & 31u;
    if (!(f & (kRecCorner | kRecNb | kRecG))) continue;
    const double k_own = (s ? ph.y : ph.x) * el;
    if (f & kRecCorner) {
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        if (FIRST) Pm[sl][r] += k_own * U[sl][r];
        else Pm[r][sl] += k_own * U[r][sl];
      }
    }
    if (f & (kRecNb | kRecG)) {
      const int64_t d = neighbour_offset(P, a, s, c[a]);
      double k = k_own;
      if (P.flags & kTranspose) {
        const int64_t n = P.sizes[a];
        const uint32_t cn = s ? ((int64_t)c[a] + 1 == n ? 0u : c[a] + 1) : (c[a] == 0 ? (uint32_t)(n - 1) : c[a] - 1);
        k = P.phi[a][cn * 2 + (1 - s)] * (P.elem[a] ? P.elem[a][e + d] : 1.0);
      }
      double v[4];
      if (f & kRecNb) {
        nbrow(s, (int)(f >> 3), d, v);
      } else {
#pragma unroll
        for (int r = 0; r < 4; ++r) v[r] = P.g;
      }
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        if (FIRST) Pm[sl][r] += k * v[r];
        else Pm[r][sl] += k * v[r];
      }
    }
  }
}

template <bool SEP, int STAGES, bool SHFL, bool DOT = false, uint32_t VM = kVaryRuntime>
__global__ void __launch_bounds__(kTmaWarps * 32, 16 / kTmaWarps)
    kron3d_tma_kernel(const __grid_constant__ KronTmaParams<double> T) {
  constexpr int N = 4, EPW = 8;
  using S = Kron3DShape<N, double>;
  static_assert(S::EPW == EPW, "eight elements per warp");
  const KronParams<double>& P = T.k;
  // one stage with the exchange tile: the tile is idle from the end of a group until the x faces
  // of the next have been read, so the x-slot element is staged there
  constexpr bool XSLOT = STAGES == 1 && !SHFL;
  extern __shared__ unsigned char tma_smem_raw[];
  __shared__ uint64_t bars[kTmaWarps][2];
  [[maybe_unused]] __shared__ double wsum[kTmaWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int le = lane >> 2, t = lane & 3;
  if (P.skip && *P.skip) return;  // a finished solve: nothing to do

  const uint32_t raw = smem_addr(tma_smem_raw);
  unsigned char* area = tma_smem_raw + (((raw + 1023u) & ~1023u) - raw) + warp * tma_warp_bytes(STAGES, SHFL);
  [[maybe_unused]] double* tile = reinterpret_cast<double*>(area + STAGES * kTmaStageBytes);
  if (lane == 0) {
    mbar_init(&bars[warp][0], 1);
    mbar_init(&bars[warp][1], 1);
    fence_barrier_init();
  }
  __syncwarp();

  const int64_t ngroups = (P.nelem - P.e_begin) / EPW;
  const int64_t nwarps = (int64_t)gridDim.x * kTmaWarps;
  const bool adv = P.has_adv != 0;
  [[maybe_unused]] const bool dot_in = P.dot_z == P.x;
  [[maybe_unused]] double dot_acc = 0.0;
  uint32_t phase = 0;  // parity of the next completion, one bit per stage
  bool failed = false;

  // lane 0: start the transaction of group g into stage st
  auto issue = [&](int64_t g, int st) {
    const int64_t e0 = P.e_begin + g * EPW;
    unsigned char* sb = area + st * kTmaStageBytes;
    const uint32_t gw = T.gwords[e0 / EPW];
    const uint32_t ys = gw & 3u, zs = (gw >> 2) & 3u, xs = XSLOT ? (gw >> 4) & 3u : 0u;
    uint32_t c[3];
    kron_coords(P, (uint32_t)e0, c);
    const uint32_t bytes = kTmaGroupBytes + (ys ? kTmaSlotBytes : 0) + (zs ? kTmaSlotBytes : 0) +
                           T.nmat * kTmaMatBytes + (xs ? kTmaElemBytes : 0);
    mbar_arrive_expect_tx(&bars[warp][st], bytes);
    tma_load_2d(sb, &T.win, 0, (int)(4 * e0), &bars[warp][st]);
    if (xs) {
      const int s = (int)xs - 1;  // element 0's - side or element 7's + side neighbour
      const int64_t ee = e0 + (s ? 7 : 0);
      const int64_t en = ee + neighbour_offset(P, 0, s, c[0] + (s ? 7u : 0u));
      tma_load_2d(tile, &T.xel, 0, (int)(4 * en), &bars[warp][st]);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int slot = tma_yz_slot(k);
      const int mi = T.mat_index[slot];
      if (mi < 0) continue;
      const double* src = P.mats + P.vm[slot].off + (int64_t)c[k < 4 ? 1 : 2] * P.vm[slot].stride;
      bulk_load(sb + kTmaGroupBytes + 2 * kTmaSlotBytes + mi * kTmaMatBytes, src, kTmaMatBytes, &bars[warp][st]);
    }
    if (zs) {
      const int s = (int)zs - 1;
      const int64_t en = e0 + neighbour_offset(P, 2, s, c[2]);
      tma_load_3d(sb + kTmaGroupBytes, &T.zsl, 0, s ? 0 : 3, (int)en, &bars[warp][st]);
    }
    if (ys) {
      const int s = (int)ys - 1;
      const int64_t en = e0 + neighbour_offset(P, 1, s, c[1]);
      tma_load_4d(sb + kTmaGroupBytes + kTmaSlotBytes, &T.ysl, 0, s ? 0 : 3, 0, (int)en, &bars[warp][st]);
    }
  };

  int64_t g = (int64_t)blockIdx.x * kTmaWarps + warp;
  if (STAGES == 2 && lane == 0 && g < ngroups) issue(g, 0);
  for (int it = 0; g < ngroups; g += nwarps, ++it) {
    const int st = STAGES == 2 ? (it & 1) : 0;
    if (lane == 0) {
      if (STAGES == 2) {
        const int64_t gn = g + nwarps;
        if (gn < ngroups) {
          bulk_wait_read_all();  // the other stage's last store has read its planes
          issue(gn, st ^ 1);
        }
      } else {
        bulk_wait_read_all();
        issue(g, 0);
      }
    }
    const int64_t e0 = P.e_begin + g * EPW;
    const int64_t e = e0 + le;
    uint32_t c[3];
    kron_coords(P, (uint32_t)e, c);
    const uint32_t ef = adv ? __ldg(T.eflags + e) : 0u;
    const double* grp = reinterpret_cast<const double*>(area + st * kTmaStageBytes);
    const uint32_t grp_sa = smem_addr(grp);
    const double* zslot = grp + kTmaGroupBytes / 8;
    const double* yslot = zslot + kTmaSlotBytes / 8;
    const double* mats = yslot + kTmaSlotBytes / 8;

    const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(&bars[warp][st], (phase >> st) & 1u));
    phase ^= 1u << st;
    if (!ok) {
      if (lane == 0) atomicOr(T.err, 1);
      failed = true;
      break;
    }

    double qx[N][N], py[N][N];
    // ------------------------------------------------------------ layout Z (plane z = t)
    if (adv) {
      double u[N][N];
      tma_plane_z(grp_sa, le, t, u);
      {
        double px[N][N];
        const double2 phx = tma_phi(P, 0, c);
        tma_apply<VM, kSlotDX, true, false>(T, c[0], mats, u, px);
        const double elx = P.elem[0] ? P.elem[0][e] : 1.0;
        if (P.elem[0]) {
#pragma unroll
          for (int i = 0; i < N; ++i)
#pragma unroll
            for (int j = 0; j < N; ++j) px[i][j] *= elx;
        }
        tma_faces<true>(P, 0, c, e, ef, elx, phx, u, px, [&](int s, int src, int64_t d, double(&v)[N]) {
          const int sl = s ? 0 : N - 1;  // the neighbour's opposite slice
          if (src == (int)kTmaSrcGroup) {
            const int r = 4 * (le + (s ? 1 : -1)) + t;
#pragma unroll
            for (int q = 0; q < N; ++q) v[q] = grp[swz(r, 4 * q + sl)];
          } else if (XSLOT && src == (int)kTmaSrcSlot) {
            // the staged neighbour element, rows of 16 values (plane z = t), unswizzled
#pragma unroll
            for (int q = 0; q < N; ++q) v[q] = tile[16 * t + 4 * q + sl];
          } else {
            const double* un = P.x + (e + d) * 64 + 16 * t + sl;
#pragma unroll
            for (int q = 0; q < N; ++q) v[q] = un[4 * q];
          }
        });
        tma_apply<VM, kSlotTXY, false, false>(T, c[1], mats, px, qx);
      }
      const double2 phy = tma_phi(P, 1, c);
      tma_apply<VM, kSlotDY, false, false>(T, c[1], mats, u, py);
      const double ely = P.elem[1] ? P.elem[1][e] : 1.0;
      if (P.elem[1]) {
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
          for (int j = 0; j < N; ++j) py[i][j] *= ely;
      }
      tma_faces<false>(P, 1, c, e, ef, ely, phy, u, py, [&](int s, int src, int64_t d, double(&v)[N]) {
        const int sl = s ? 0 : N - 1;
        if (src == (int)kTmaSrcSlot) {
          const double2 a = *reinterpret_cast<const double2*>(yslot + le * 16 + t * 4);
          const double2 b = *reinterpret_cast<const double2*>(yslot + le * 16 + t * 4 + 2);
          v[0] = a.x;
          v[1] = a.y;
          v[2] = b.x;
          v[3] = b.y;
        } else {
          const double* un = P.x + (e + d) * 64 + 16 * t + 4 * sl;
#pragma unroll
          for (int q = 0; q < N; ++q) v[q] = un[q];
        }
      });
      if constexpr (SHFL) {
        exchange_butterfly<N>(t, qx);
        exchange_butterfly<N>(t, py);
      } else {
        exchange_tile<N>(tile, le, t, true, true, qx);
        exchange_tile<N>(tile, le, t, true, true, py);
      }
    }

    // ------------------------------------------------------------ layout Y (plane y = t)
    double out[N][N], qz[N][N];
    [[maybe_unused]] double qm[N][N];
    {
      if (adv) {
        tma_apply<VM, kSlotTXZ, false, false>(T, c[2], mats, qx, out);
        tma_apply<VM, kSlotTYZ, false, false>(T, c[2], mats, py, qx);  // qx reused as scratch
        tma_apply<VM, kSlotTYX, true, true>(T, c[0], mats, qx, out);   // out += Tyx (Tyz py)
      }
      double u[N][N], pz[N][N];
      tma_plane_y(grp_sa, le, t, u);
      [[maybe_unused]] const double2 phz = adv ? tma_phi(P, 2, c) : make_double2(0.0, 0.0);
      tma_apply<VM, kSlotDZ, false, false>(T, c[2], mats, u, pz);
      if (adv) {
        const double elz = P.elem[2] ? P.elem[2][e] : 1.0;
        if (P.elem[2]) {
#pragma unroll
          for (int i = 0; i < N; ++i)
#pragma unroll
            for (int k = 0; k < N; ++k) pz[i][k] *= elz;
        }
        tma_faces<false>(P, 2, c, e, ef, elz, phz, u, pz, [&](int s, int src, int64_t d, double(&v)[N]) {
          const int sl = s ? 0 : N - 1;
          if (src == (int)kTmaSrcSlot) {
            const double2 a = *reinterpret_cast<const double2*>(zslot + swz(le, 4 * t));
            const double2 b = *reinterpret_cast<const double2*>(zslot + swz(le, 4 * t + 2));
            v[0] = a.x;
            v[1] = a.y;
            v[2] = b.x;
            v[3] = b.y;
          } else {
            const double* un = P.x + (e + d) * 64 + 16 * sl + 4 * t;
#pragma unroll
            for (int q = 0; q < N; ++q) v[q] = un[q];
          }
        });
      } else if (P.elem_mass) {
        const double em = P.elem_mass[e];
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
          for (int k = 0; k < N; ++k) pz[i][k] *= em;
      }
      tma_apply<VM, kSlotTZX, true, false>(T, c[0], mats, pz, qz);
      if constexpr (SEP) {
        tma_apply<VM, kSlotMD, false, false>(T, c[2], mats, u, pz);
        if (P.elem_mass) {
          const double em = P.elem_mass[e];
#pragma unroll
          for (int i = 0; i < N; ++i)
#pragma unroll
            for (int k = 0; k < N; ++k) pz[i][k] *= em;
        }
        tma_apply<VM, kSlotMX, true, false>(T, c[0], mats, pz, qm);
      }
    }
    // layout Y -> Z for the terms still missing their y pass, and for `out`
    if constexpr (SHFL) {
      exchange_butterfly<N>(t, qz);
      if (adv) exchange_butterfly<N>(t, out);
      if constexpr (SEP) exchange_butterfly<N>(t, qm);
    } else {
      exchange_tile<N>(tile, le, t, true, false, qz);
      if (adv) exchange_tile<N>(tile, le, t, true, false, out);
      if constexpr (SEP) exchange_tile<N>(tile, le, t, true, false, qm);
    }
    // ------------------------------------------------------------ layout Z, output
    // res = out + Tzy qz (+ My qm): the last passes accumulate onto the x and y terms
    double (&res)[N][N] = out;
    if (adv) tma_apply<VM, kSlotTZY, false, true>(T, c[1], mats, qz, res);
    else tma_apply<VM, kSlotTZY, false, false>(T, c[1], mats, qz, res);
    if constexpr (SEP) tma_apply<VM, kSlotMY, false, true>(T, c[1], mats, qm, res);
    const double alpha = P.alpha, by = P.beta_y;
    if (alpha != 1.0) {
#pragma unroll
      for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) res[i][j] *= alpha;
    }
    if (by != 0.0) {
      const double* yo = P.y + e * 64 + 16 * t;
#pragma unroll
      for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = 0; i < N; i += 2) {
          const double2 v = *reinterpret_cast<const double2*>(yo + 4 * j + i);
          res[i][j] += by * v.x;
          res[i + 1][j] += by * v.y;
        }
    }
    __syncwarp();  // every lane is done reading this stage's planes and slices
    double* gout = const_cast<double*>(grp);
    const uint32_t orow = swz_row(grp_sa, 4 * le + t);  // this lane's plane row (layout Z)
    if constexpr (DOT) {
      double acc = 0.0;
      const double* zp = P.dot_z + e * 64 + 16 * t;
#pragma unroll
      for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = 0; i < N; i += 2) {
          const double2 z = dot_in ? lds_v2(orow ^ ((uint32_t)(2 * j + i / 2) << 4))
                                   : *reinterpret_cast<const double2*>(zp + 4 * j + i);
          acc += res[i][j] * z.x;
          acc += res[i + 1][j] * z.y;
        }
      dot_acc += acc;
    }
#pragma unroll
    for (int j = 0; j < N; ++j)
#pragma unroll
      for (int i = 0; i < N; i += 2) sts_v2(orow ^ ((uint32_t)(2 * j + i / 2) << 4), res[i][j], res[i + 1][j]);
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) {
      tma_store_2d(&T.out, 0, (int)(4 * e0), gout);
      bulk_commit();
    }
  }
  if (lane == 0) bulk_wait_all();
  if constexpr (DOT) {
    // fixed-order sums: lanes (tree), warps (in order), then one partial per CTA; entries past the
    // grid are zeroed so a reader sums a fixed count
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dot_acc += __shfl_down_sync(0xffffffffu, dot_acc, o);
    if (lane == 0) wsum[warp] = dot_acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < kTmaWarps; ++w) s += wsum[w];
      P.dot_partials[blockIdx.x] = failed ? 0.0 : s;
      for (int i = blockIdx.x + gridDim.x; i < P.dot_count; i += gridDim.x) P.dot_partials[i] = 0.0;
    }
  }
}

// Per-element face words and per-group slot words of a Kronecker operator (forward or
// transposed parameters), for kron3d_tma_kernel.  One warp per group of 8 elements; lanes 0-7
// take one element each and decide its faces exactly as kron3d_kernel does per group
// (face_decide); the group stages, per axis y and z, the side its elements need most often.
template <typename Real>
__global__ void kron_face_words(const KronParams<Real> P, uint32_t* eflags, uint32_t* gwords) {
  const int lane = threadIdx.x & 31;
  const int64_t grp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t e = grp * 8 + lane;
  const bool act = lane < 8 && e < P.nelem;
  if (grp * 8 >= P.nelem) return;  // whole warp
  uint32_t bits[6] = {0, 0, 0, 0, 0, 0};
  uint32_t c[3] = {0, 0, 0};
  // operators without advection terms have no faces (and no phi / sign tables): all words zero
  if (act && P.has_adv) {
    kron_coords(P, (uint32_t)e, c);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const Real tsign = tan_sign(P, a, c);
      const Real el = P.elem[a] ? P.elem[a][e] : Real(1);
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        Real phi, coef;
        const FaceDecision f = face_decide(P, a, s, c, e, tsign, el, phi, coef);
        bits[a * 2 + s] = (f.corner ? kRecCorner : 0u) | (f.use_nb ? kRecNb : 0u) | (f.use_g ? kRecG : 0u);
      }
    }
  }
  uint32_t side[3] = {0, 0, 0};
#pragma unroll
  for (int a = 1; a < 3; ++a) {
    const int n0 = __popc(__ballot_sync(0xffffffffu, act && (bits[a * 2] & kRecNb)));
    const int n1 = __popc(__ballot_sync(0xffffffffu, act && (bits[a * 2 + 1] & kRecNb)));
    side[a] = (n0 == 0 && n1 == 0) ? 0u : (n0 >= n1 ? 1u : 2u);
  }
  {
    // x: only element 0's - side and element 7's + side neighbours lie outside the group (its 8
    // elements are consecutive along x within one row); the x slot takes one of them
    const bool x0 = __ballot_sync(0xffffffffu, act && lane == 0 && (bits[0] & kRecNb)) != 0u;
    const bool x1 = __ballot_sync(0xffffffffu, act && lane == 7 && (bits[1] & kRecNb)) != 0u;
    side[0] = x0 ? 1u : (x1 ? 2u : 0u);
  }
  if (act) {
    uint32_t w = 0;
    const int le = lane;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        uint32_t b = bits[a * 2 + s];
        if (b & kRecNb) {
          uint32_t src;
          if (a == 0) {
            const bool inside = s ? (le < 7 && (int64_t)c[0] + 1 < P.sizes[0]) : (le > 0 && c[0] > 0);
            src = inside ? kTmaSrcGroup : (side[0] == (uint32_t)(s + 1) ? kTmaSrcSlot : kTmaSrcGlobal);
          } else {
            src = (side[a] == (uint32_t)(s + 1)) ? kTmaSrcSlot : kTmaSrcGlobal;
          }
          b |= src << 3;
        }
        w |= b << (5 * (a * 2 + s));
      }
    eflags[e] = w;
  }
  if (lane == 0) gwords[grp] = side[1] | (side[2] << 2) | (side[0] << 4);
}

}  // namespace dgop
