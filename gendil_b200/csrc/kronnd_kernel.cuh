// Kronecker-form DG operator kernel for any dimension D and order (N = p + 1), shared memory.
//
// The operator is the sum of D terms (plus a separate mass term when it does not merge), each a
// tensor product of per-axis N x N matrices (kron.h):
//
//   y_e = sum_a  (x)_{k != a} T_ak  [ D_a u_e + faces_a ]
//
// A CTA holds EB elements in shared memory: the input U, one work array W and the accumulator Y.
// Every factor is one pass over the element's N^(D-1) lines along its axis, one line per thread,
// read into registers and written back in place (lines are disjoint, so W needs no second
// buffer); the last tangential pass of a term accumulates into Y.  The face terms of axis a are
// added to the faces' slices of D_a U before the tangential passes (GLL: the trace is the slice),
// with the upwind neighbour's trace read from global memory.  Matrices (constant or depending on
// the element's coordinate along their axis) are copied per element into shared memory.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "dgop_params.h"
#include "generic_kernel.cuh"
#include "kron.h"

namespace dgop {


__host__ __device__ constexpr int kpow(int b, int e) { return e == 0 ? 1 : b * kpow(b, e - 1); }

template <int D, int N>
struct KronNDShape {
  static constexpr int ND = kpow(N, D);  // DoFs per element
  static constexpr int NL = ND / N;      // lines per pass
  static constexpr int NS = D * D + D;   // matrix slots: D terms x D axes, plus the mass term
  static constexpr int MAT = N * N;
  // per element: U, W, Y, the slot matrices, and 2D face records (corner, neighbour / inflow
  // coefficient) + one flag byte per face (16 bytes, whatever the Real).  The matrix area and
  // every matrix start on a multiple of 4 values (16 bytes in FP32, 32 in FP64), so a pass reads
  // its matrix with 16-byte loads.
  static constexpr int MATP = (MAT + 3) / 4 * 4;    // stride of the slot matrices
  static constexpr int MOFF = (3 * ND + 3) / 4 * 4;  // offset of the matrix area
  static constexpr int ROFF = MOFF + NS * MATP;       // offset of the face records
  static constexpr int REC = 4 * D + 16 / (int)sizeof(float);
  static constexpr int PER_ELEM = (ROFF + REC + 3) / 4 * 4;
};

// Matrix of a pass: in registers for N <= 4 (loaded once per pass), read from shared memory
// otherwise.
template <int N, typename Real, bool REG = (N <= 4)>
struct PassMat;
template <int N, typename Real>
struct PassMat<N, Real, true> {
  Real a[N * N];
  __device__ __forceinline__ explicit PassMat(const Real* m) {
#pragma unroll
    for (int i = 0; i < N * N; ++i) a[i] = m[i];
  }
  __device__ __forceinline__ Real operator()(int j, int i) const { return a[j * N + i]; }
};
template <int N, typename Real>
struct PassMat<N, Real, false> {
  const Real* m;
  __device__ __forceinline__ explicit PassMat(const Real* p) : m(p) {}
  __device__ __forceinline__ Real operator()(int j, int i) const { return m[j * N + i]; }
};

// A slot matrix of the per-element matrix area (KronNDShape::MATP: 16-byte aligned, padded to a
// multiple of 4 values): in registers for N <= 4, read with 16-byte loads; as PassMat otherwise.
template <int N, typename Real, bool REG = (N <= 4)>
struct SlotMat : PassMat<N, Real, false> {
  __device__ __forceinline__ explicit SlotMat(const Real* p) : PassMat<N, Real, false>(p) {}
};
template <int N, typename Real>
struct SlotMat<N, Real, true> {
  static constexpr int V = 16 / (int)sizeof(Real);  // values per 16-byte load
  static constexpr int NV = (N * N + V - 1) / V;    // loads (within the padded slot)
  Real a[NV * V];
  __device__ __forceinline__ explicit SlotMat(const Real* m) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      if constexpr (V == 4) {
        const float4 w = reinterpret_cast<const float4*>(m)[k];
        a[4 * k] = w.x;
        a[4 * k + 1] = w.y;
        a[4 * k + 2] = w.z;
        a[4 * k + 3] = w.w;
      } else {
        const double2 w = reinterpret_cast<const double2*>(m)[k];
        a[2 * k] = w.x;
        a[2 * k + 1] = w.y;
      }
    }
  }
  __device__ __forceinline__ Real operator()(int j, int i) const { return a[j * N + i]; }
};

// One pass along axis A over the batch: the CTA's threads form EB groups of blockDim / EB, group
// b runs the lines of element b with the element's matrix held in registers.
//   FIRST: W <- M U (times the element factor when escale is given)
//   ACC:   Y += M W            otherwise: W <- M W in place
template <int D, int N, int A, bool FIRST, bool ACC, typename Real>
__device__ __forceinline__ void nd_pass(Real* base, int ne, int eb, int slot, const Real* escale) {
  using S = KronNDShape<D, N>;
  constexpr int INNER = kpow(N, A);
  const int tpe = blockDim.x / eb;
  const int b = threadIdx.x / tpe;
  if (b >= ne) return;
  Real* el = base + (size_t)b * S::PER_ELEM;
  const Real* in = FIRST ? el : el + S::ND;
  Real* out = ACC ? el + 2 * S::ND : el + S::ND;
  const SlotMat<N, Real> m(el + S::MOFF + slot * S::MATP);
  const Real f = (FIRST && escale) ? escale[b] : Real(1);
  for (int r = threadIdx.x - b * tpe; r < S::NL; r += tpe) {
    const int o = r / INNER;
    const int t = r - o * INNER;
    const int off = o * N * INNER + t;
    Real v[N];
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = in[off + i * INNER];
#pragma unroll
    for (int j = 0; j < N; ++j) {
      Real s = m(j, 0) * v[0];
#pragma unroll
      for (int i = 1; i < N; ++i) s += m(j, i) * v[i];
      if (ACC) out[off + j * INNER] += s;
      else out[off + j * INNER] = (FIRST && escale) ? s * f : s;
    }
  }
}

// Face record of face fi = a * 2 + s of element e (one thread per face): rec[2 fi] is the
// own-trace (corner) coefficient, rec[2 fi + 1] the neighbour / inflow coefficient, and the
// face's flag byte: 1 corner, 2 neighbour trace, 4 inflow value.  Follows the upwind rule of
// advectionoperator.hpp:379-386 / 422-428 per element, as the 3D kernel does.
template <int D, typename Real>
__device__ __forceinline__ void nd_face_record(const KronNDParams<Real>& P, int64_t e, const int* c, int fi, Real* rec,
                                               uint8_t* flag) {
  const bool transpose = (P.flags & kTranspose) != 0;
  const int a = fi >> 1, s = fi & 1;
  Real tsign = Real(1);
#pragma unroll
  for (int k = 0; k < D; ++k)
    if (k != a) tsign *= (Real)P.sgn[a][k][c[k]];
  const Real el = P.elem[a] ? P.elem[a][e] : Real(1);
  const int64_t n = P.sizes[a];
  const int64_t ca = c[a];
  const bool interior = s == 0 ? (ca > 0 || P.periodic[a]) : (ca + 1 < n || P.periodic[a]);
  const bool active = interior ? (P.flags & kFaceInt) : (P.flags & kFaceBnd);
  const Real phi = P.phi[a][ca * 2 + s];
  Real coef = Real(0);
  uint32_t bits = 0;
  if (active) {
    if (phi * tsign * el > Real(0)) bits |= 1u;
    if (!transpose) {
      if (!(phi * tsign * el > Real(0))) {
        coef = phi * el;
        bits |= interior ? 2u : 4u;
      }
    } else if (interior) {
      // transposed coupling: the neighbour's row, taken when its face 1 - s is inflow for it
      const int64_t cn = s ? (ca + 1 == n ? 0 : ca + 1) : (ca == 0 ? n - 1 : ca - 1);
      const int64_t en = e + (cn - ca) * P.estride[a];
      const Real phin = P.phi[a][cn * 2 + (1 - s)];
      const Real eln = P.elem[a] ? P.elem[a][en] : Real(1);
      if (!(phin * tsign * eln > Real(0))) {
        coef = phin * eln;
        bits |= 2u;
      }
    }
  }
  rec[2 * fi] = phi * el;
  rec[2 * fi + 1] = coef;
  *flag = (uint8_t)bits;
}

// Face terms of axis A added to W (= D_A U) on the two slices of that axis.  One thread takes a
// tangential point and both sides (for N = 1 the two slices are the same point).
template <int D, int N, int A, typename Real>
__device__ __forceinline__ void nd_faces(const KronNDParams<Real>& P, Real* base, int ne, int64_t e0,
                                         const int (*ecoord)[kMaxDim]) {
  using S = KronNDShape<D, N>;
  constexpr int INNER = kpow(N, A);
  const int total = ne * S::NL;
  for (int l = threadIdx.x; l < total; l += blockDim.x) {
    const int b = l / S::NL;
    const int p = l - b * S::NL;  // point of the slice: (o, t) with the axis index removed
    const int o = p / INNER, t = p - o * INNER;
    Real* el = base + (size_t)b * S::PER_ELEM;
    const Real* rec = el + S::ROFF;
    const uint8_t* fb = reinterpret_cast<const uint8_t*>(rec + 4 * D);
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const int fi = A * 2 + s;
      const uint32_t f = fb[fi];
      if (!f) continue;
      const int sl = s ? N - 1 : 0;
      const int idx = o * N * INNER + sl * INNER + t;
      Real add = Real(0);
      if (f & 1u) add += rec[2 * (A * 2 + s)] * el[idx];  // own trace
      if (f & 2u) {
        // the neighbour's opposite slice at the same tangential point
        const int64_t e = e0 + b;
        const int64_t n = P.sizes[A];
        const int64_t ca = ecoord[b][A];
        const int64_t cn = s ? (ca + 1 == n ? 0 : ca + 1) : (ca == 0 ? n - 1 : ca - 1);
        const int64_t en = e + (cn - ca) * P.estride[A];
        const int nidx = o * N * INNER + (N - 1 - sl) * INNER + t;
        add += rec[2 * (A * 2 + s) + 1] * P.x[en * S::ND + nidx];
      } else if (f & 4u) {
        add += rec[2 * (A * 2 + s) + 1] * P.g;
      }
      el[S::ND + idx] += add;
    }
  }
}

// How the last step of a term writes its block into the accumulator Y: bit 0 set, the term is the
// first to reach Y and stores (Y is not zeroed beforehand); bit 1 set, the term is the last and
// writes y = alpha (Y + block) + beta y to global memory instead of Y (no separate output pass).
enum : int { kYAdd = 0, kYStore = 1, kYOut = 2 };
// alpha and beta_y come in registers: the persistent batch kernel reads its parameters from a
// global table, which the compiler would load again after every store to y.
template <typename Real>
__device__ __forceinline__ void nd_y_write(Real alpha, Real beta_y, int ymode, Real* yl, Real* yg, Real v) {
  const Real t = (ymode & kYStore) ? v : *yl + v;
  if (ymode & kYOut) *yg = (beta_y == Real(0)) ? alpha * t : alpha * t + beta_y * *yg;
  else *yl = t;
}

// Shared-memory setup of one batch of ne elements starting at e0: U (the input), Y = 0, the
// element coordinates, every element's slot matrices and face records.
template <int D, int N, typename Real>
__device__ __forceinline__ void nd_setup(const KronNDParams<Real>& P, const Real* __restrict__ xin, int64_t e0, int ne,
                                         Real* base, int (*ecoord)[kMaxDim], bool zero_y = true) {
  using S = KronNDShape<D, N>;
  const bool adv = P.has_adv != 0;
  __syncthreads();
  // input, accumulator
  for (int l = threadIdx.x; l < ne * S::ND; l += blockDim.x) {
    const int b = l / S::ND, i = l - b * S::ND;
    Real* el = base + (size_t)b * S::PER_ELEM;
    el[i] = xin[e0 * S::ND + l];
    if (zero_y) el[2 * S::ND + i] = Real(0);
  }
  if (threadIdx.x < ne) {
    const int64_t e = e0 + threadIdx.x;
#pragma unroll
    for (int k = 0; k < D; ++k) ecoord[threadIdx.x][k] = (int)((e / P.estride[k]) % P.sizes[k]);
  }
  __syncthreads();
  // per element: slot matrices and face records
  for (int l = threadIdx.x; l < ne * S::NS * S::MAT; l += blockDim.x) {
    const int b = l / (S::NS * S::MAT);
    const int r = l - b * (S::NS * S::MAT);
    const int sl = r / S::MAT, q = r - sl * S::MAT;
    const int a = sl / D, k = sl - a * D;  // a == D: the mass term
    const KronMat m = a < D ? P.slot[a][k] : P.mslot[k];
    Real v = Real(0);
    if (m.off >= 0) v = P.mats[m.off + (int64_t)ecoord[b][k] * m.stride + q];
    base[(size_t)b * S::PER_ELEM + S::MOFF + sl * S::MATP + q] = v;
  }
  if (adv) {
    for (int l = threadIdx.x; l < ne * 2 * D; l += blockDim.x) {
      const int b = l / (2 * D), fi = l - b * (2 * D);
      Real* rec = base + (size_t)b * S::PER_ELEM + S::ROFF;
      nd_face_record<D>(P, e0 + b, ecoord[b], fi, rec, reinterpret_cast<uint8_t*>(rec + 4 * D) + fi);
    }
  }
  __syncthreads();
}

// y = alpha Y + beta_y y for the batch.
template <int D, int N, typename Real>
__device__ __forceinline__ void nd_output(const KronNDParams<Real>& P, Real* __restrict__ yout, int64_t e0, int ne,
                                          const Real* base) {
  using S = KronNDShape<D, N>;
  for (int l = threadIdx.x; l < ne * S::ND; l += blockDim.x) {
    const int b = l / S::ND, i = l - b * S::ND;
    const Real v = base[(size_t)b * S::PER_ELEM + 2 * S::ND + i];
    Real* dst = yout + e0 * S::ND + l;
    *dst = (P.beta_y == Real(0)) ? P.alpha * v : P.alpha * v + P.beta_y * *dst;
  }
}

// One batch of ne elements starting at e0 (the CTA's shared memory holds them); x / y are the
// instance's vectors.
template <int D, int N, typename Real>
__device__ __forceinline__ void kronnd_block(const KronNDParams<Real>& P, const Real* __restrict__ xin,
                                             Real* __restrict__ yout, int64_t e0, int ne, int EB, Real* base,
                                             Real* escale, int (*ecoord)[kMaxDim]) {
  using S = KronNDShape<D, N>;
  const bool adv = P.has_adv != 0;
  nd_setup<D, N>(P, xin, e0, ne, base, ecoord);
  if (adv) {
    static_for<0, D>([&](auto ac) {
      constexpr int a = decltype(ac)::value;
      if (P.elem[a]) {
        if (threadIdx.x < ne) escale[threadIdx.x] = P.elem[a][e0 + threadIdx.x];
        __syncthreads();
      }
      nd_pass<D, N, a, true, false>(base, ne, EB, a * D + a, P.elem[a] ? escale : (const Real*)nullptr);
      __syncthreads();
      nd_faces<D, N, a>(P, base, ne, e0, ecoord);
      __syncthreads();
      // tangential passes in increasing axis order; the last accumulates into Y
      static_for<0, D>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        if constexpr (k != a) {
          constexpr int lastk = (a == D - 1) ? D - 2 : D - 1;
          nd_pass<D, N, k, false, k == lastk>(base, ne, EB, a * D + k, (const Real*)nullptr);
          __syncthreads();
        }
      });
      if constexpr (D == 1) {
        // no tangential pass: the term goes straight to Y
        for (int l = threadIdx.x; l < ne * S::ND; l += blockDim.x) {
          const int b = l / S::ND, i = l - b * S::ND;
          Real* el = base + (size_t)b * S::PER_ELEM;
          el[2 * S::ND + i] += el[S::ND + i];
        }
        __syncthreads();
      }
    });
  }
  if (P.has_mass && !(adv && P.mass_merged)) {
    // separate mass term: along the last axis (scaled), then the others
    if (P.elem_mass) {
      if (threadIdx.x < ne) escale[threadIdx.x] = P.elem_mass[e0 + threadIdx.x];
      __syncthreads();
    }
    nd_pass<D, N, D - 1, true, false>(base, ne, EB, D * D + D - 1, P.elem_mass ? escale : (const Real*)nullptr);
    __syncthreads();
    static_for<0, D - 1>([&](auto kc) {
      constexpr int k = decltype(kc)::value;
      nd_pass<D, N, k, false, k == D - 2>(base, ne, EB, D * D + k, (const Real*)nullptr);
      __syncthreads();
    });
    if constexpr (D == 1) {
      for (int l = threadIdx.x; l < ne * S::ND; l += blockDim.x) {
        const int b = l / S::ND, i = l - b * S::ND;
        Real* el = base + (size_t)b * S::PER_ELEM;
        el[2 * S::ND + i] += el[S::ND + i];
      }
      __syncthreads();
    }
  }
  nd_output<D, N>(P, yout, e0, ne, base);
}

template <int D, int N, typename Real>
__global__ void __launch_bounds__(kKronNDThreads) kronnd_kernel(const __grid_constant__ KronNDParams<Real> P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Real* base = reinterpret_cast<Real*>(smem_raw);
  __shared__ Real escale[64];          // per-element factor of the pass being run (EB <= 64)
  __shared__ int ecoord[64][kMaxDim];  // element coordinates
  if (P.skip && *P.skip) return;
  const int EB = P.eb;
  for (int64_t e0 = P.e_begin + (int64_t)blockIdx.x * EB; e0 < P.nelem; e0 += (int64_t)gridDim.x * EB) {
    const int ne = (int)((P.nelem - e0) < EB ? (P.nelem - e0) : EB);
    kronnd_block<D, N>(P, P.x, P.y, e0, ne, EB, base, escale, ecoord);
  }
}

// ------------------------------------------------------------------------------------------
// Grouped variant: the axes are cut into groups of G consecutive axes, and one thread takes a
// block of the element that spans one group (N^G values with the other axes fixed), runs the
// group's passes in registers and writes the block back once.  A term costs one shared-memory
// round trip per group instead of one per axis: for D = 6, N = 3 and G = 3, two round trips of
// 27-value blocks instead of six of 3-value lines.  The term's own axis (D_a scaled by the element
// factor, then the face terms of that axis) is in the first group a term runs; the other groups
// follow in increasing order and the last one accumulates into Y.  Same shared-memory layout and
// setup as the per-axis kernel above; the tangential passes run in another order, so the results
// agree with it to rounding (the passes along different axes commute exactly in real arithmetic).
// ------------------------------------------------------------------------------------------
template <int D, int N, int G>
struct KronGroups {
  static constexpr int NG = (D + G - 1) / G;
  static constexpr int lo(int g) { return g * G; }
  static constexpr int hi(int g) { return (g + 1) * G < D ? (g + 1) * G : D; }
  static constexpr int size(int g) { return kpow(N, hi(g) - lo(g)); }
  static constexpr int inner(int g) { return kpow(N, lo(g)); }
  // step st of a term whose first pass is along AX: AX's group first, then the others in order
  static constexpr int group(int AX, int st) { return st == 0 ? AX / G : (st <= AX / G ? st - 1 : st); }
  // the kk-th axis a step of group g runs: AX first in the term's first step (its face terms need
  // the input values), the group's other axes in increasing order
  static constexpr int axis(int g, int kk, bool first, int AX) {
    return !first ? lo(g) + kk : (kk == 0 ? AX : (lo(g) + kk - 1 < AX ? lo(g) + kk - 1 : lo(g) + kk));
  }
};

// Step ST of term TERM (TERM == D: the separate mass term, first pass along axis 0) over the blocks
// of its group, for the ne elements of the batch.
template <int D, int N, int G, int TERM, int ST, typename Real>
__device__ __forceinline__ void nd_group_step(const KronNDParams<Real>& P, const Real* __restrict__ xin, Real* base,
                                              int ne, int64_t e0, const int (*ecoord)[kMaxDim], int ymode = kYAdd,
                                              Real* __restrict__ yout = nullptr) {
  using S = KronNDShape<D, N>;
  using GR = KronGroups<D, N, G>;
  constexpr bool MASS = TERM == D;
  constexpr int AX = MASS ? 0 : TERM;
  constexpr int g = GR::group(AX, ST);
  constexpr int LO = GR::lo(g), HI = GR::hi(g), GSZ = GR::size(g), INNER = GR::inner(g);
  constexpr int IPE = S::ND / GSZ;  // blocks per element
  constexpr bool FIRST = ST == 0, LAST = ST == GR::NG - 1;
  const Real alpha = P.alpha, beta_y = P.beta_y;
  const int total = ne * IPE;
  for (int it = threadIdx.x; it < total; it += blockDim.x) {
    const int b = it / IPE;
    const int loc = it - b * IPE;
    const int o = loc / INNER, t = loc - o * INNER;
    const int off = o * GSZ * INNER + t;  // block value j sits at off + j * INNER
    Real* el = base + (size_t)b * S::PER_ELEM;
    const Real* src = FIRST ? el : el + S::ND;
    Real v[GSZ];
#pragma unroll
    for (int j = 0; j < GSZ; ++j) v[j] = src[off + j * INNER];
    static_for<0, HI - LO>([&](auto kc) {
      constexpr int k = GR::axis(g, decltype(kc)::value, FIRST, AX);
      constexpr int SK = kpow(N, k - LO);  // stride of axis k inside the block
      constexpr bool OWN = FIRST && k == AX;
      const SlotMat<N, Real> m(el + S::MOFF + (MASS ? D * D + k : TERM * D + k) * S::MATP);
      Real scale = Real(1);
      if constexpr (OWN) {
        const Real* ef = MASS ? P.elem_mass : P.elem[AX];
        if (ef) scale = ef[e0 + b];
      }
#pragma unroll
      for (int ln = 0; ln < GSZ / N; ++ln) {
        const int p0 = (ln / SK) * SK * N + (ln % SK);
        Real w[N];
#pragma unroll
        for (int j = 0; j < N; ++j) {
          Real s = m(j, 0) * v[p0];
#pragma unroll
          for (int i = 1; i < N; ++i) s += m(j, i) * v[p0 + i * SK];
          w[j] = s;
        }
        if constexpr (OWN) {
          if (MASS ? P.elem_mass != nullptr : P.elem[AX] != nullptr) {
#pragma unroll
            for (int j = 0; j < N; ++j) w[j] *= scale;
          }
          if constexpr (!MASS) {
            // face terms of axis AX on the line's two ends (GLL: the trace is the end value)
            const Real* rec = el + S::ROFF;
            const uint8_t* fb = reinterpret_cast<const uint8_t*>(rec + 4 * D);
#pragma unroll
            for (int sd = 0; sd < 2; ++sd) {
              const int fi = AX * 2 + sd;
              const uint32_t f = fb[fi];
              if (!f) continue;
              const int sl = sd ? N - 1 : 0;
              Real add = Real(0);
              if (f & 1u) add += rec[2 * fi] * v[p0 + sl * SK];
              if (f & 2u) {
                const int64_t n = P.sizes[AX];
                const int64_t ca = ecoord[b][AX];
                const int64_t cn = sd ? (ca + 1 == n ? 0 : ca + 1) : (ca == 0 ? n - 1 : ca - 1);
                const int64_t en = e0 + b + (cn - ca) * P.estride[AX];
                add += rec[2 * fi + 1] * xin[en * S::ND + off + (p0 + (N - 1 - sl) * SK) * INNER];
              } else if (f & 4u) {
                add += rec[2 * fi + 1] * P.g;
              }
              w[sl] += add;
            }
          }
        }
#pragma unroll
        for (int j = 0; j < N; ++j) v[p0 + j * SK] = w[j];
      }
    });
    Real* dst = el + (LAST ? 2 : 1) * S::ND;
#pragma unroll
    for (int j = 0; j < GSZ; ++j) {
      if constexpr (LAST)
        nd_y_write(alpha, beta_y, ymode, dst + off + j * INNER, yout + (e0 + b) * S::ND + off + j * INNER, v[j]);
      else dst[off + j * INNER] = v[j];
    }
  }
}

// One batch of ne elements starting at e0 with the grouped passes.
template <int D, int N, int G, typename Real>
__device__ __forceinline__ void kronnd_grouped_block(const KronNDParams<Real>& P, const Real* __restrict__ xin,
                                                     Real* __restrict__ yout, int64_t e0, int ne, Real* base,
                                                     int (*ecoord)[kMaxDim]) {
  using GR = KronGroups<D, N, G>;
  // The terms run from D - 1 down to 0, then the separate mass term: the first to reach Y stores
  // its block (Y is not zeroed).  The last term (0, or the mass term; both start along axis 0)
  // ends on the highest group, whose blocks put INNER consecutive threads on consecutive values:
  // when that run is a 32-byte sector or more it writes y itself (nd_y_write), otherwise it
  // accumulates into Y and the coalesced output pass writes y.
  constexpr bool YOUT = GR::NG >= 2 && GR::inner(GR::NG - 1) * sizeof(Real) >= 32;
  const bool sep_mass = P.has_mass && !(P.has_adv && P.mass_merged);
  nd_setup<D, N>(P, xin, e0, ne, base, ecoord, false);
  if (P.has_adv) {
    static_for<0, D>([&](auto ac) {
      constexpr int a = D - 1 - decltype(ac)::value;
      const int ymode = (a == D - 1 ? kYStore : kYAdd) | ((YOUT && a == 0 && !sep_mass) ? kYOut : kYAdd);
      static_for<0, GR::NG>([&](auto sc) {
        nd_group_step<D, N, G, a, decltype(sc)::value>(P, xin, base, ne, e0, ecoord, ymode, yout);
        __syncthreads();
      });
    });
  }
  if (sep_mass) {
    const int ymode = (P.has_adv ? kYAdd : kYStore) | (YOUT ? kYOut : kYAdd);
    static_for<0, GR::NG>([&](auto sc) {
      nd_group_step<D, N, G, D, decltype(sc)::value>(P, xin, base, ne, e0, ecoord, ymode, yout);
      __syncthreads();
    });
  }
  if constexpr (!YOUT) nd_output<D, N>(P, yout, e0, ne, base);
}

template <int D, int N, int G, typename Real>
__global__ void __launch_bounds__(kKronNDThreads)
    kronnd_grouped_kernel(const __grid_constant__ KronNDParams<Real> P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Real* base = reinterpret_cast<Real*>(smem_raw);
  __shared__ int ecoord[64][kMaxDim];
  if (P.skip && *P.skip) return;
  const int EB = P.eb;
  for (int64_t e0 = P.e_begin + (int64_t)blockIdx.x * EB; e0 < P.nelem; e0 += (int64_t)gridDim.x * EB) {
    const int ne = (int)((P.nelem - e0) < EB ? (P.nelem - e0) : EB);
    kronnd_grouped_block<D, N, G>(P, P.x, P.y, e0, ne, base, ecoord);
  }
}

// ------------------------------------------------------------------------------------------
// Paired variant (even D, H = D / 2): axis a is grouped with axis a + H, and the two terms whose
// own axes form a pair run together.  Valid when their factors on the other D - 2 axes are the
// same matrices (the planner checks the tables: phase-space advection beta = (v, -x + 0.5) has
// terms a and a + H weighted only along the pair) and, for a separate mass term, when its factors
// outside the last pair equal that pair's terms' (it then runs with them).  Term pair g makes one
// shared-memory round trip per pair: the own step on the (g, g + H) blocks sums
//   (D_g (+ faces) then T_{g, g+H})  +  (D_{g+H} (+ faces) then T_{g+H, g})  [+ MD then MT_g]
// in registers, and the other pairs' steps apply the shared factors, the last accumulating into
// Y: D / 2 round trips per pair instead of D / G per term.  Results agree with the other variants
// to rounding (the terms are summed before, not after, their common factors).
// ------------------------------------------------------------------------------------------
template <int D, int N, int PG, int ST, typename Real>
__device__ __forceinline__ void nd_pair_step(const KronNDParams<Real>& P, const Real* __restrict__ xin, Real* base,
                                             int ne, int64_t e0, const int (*ecoord)[kMaxDim], int ymode = kYAdd,
                                             Real* __restrict__ yout = nullptr) {
  using S = KronNDShape<D, N>;
  constexpr int H = D / 2;
  constexpr int g = ST == 0 ? PG : (ST - 1 < PG ? ST - 1 : ST);  // the pair this step runs on
  constexpr int A = g, B = g + H;
  constexpr int SA = kpow(N, A), SB = kpow(N, B);
  constexpr int IPE = S::ND / (N * N);  // blocks per element
  constexpr bool OWN = ST == 0, LAST = ST == H - 1;
  constexpr bool WITH_MASS = PG == H - 1;  // the separate mass term runs with pair H - 1
  const bool mass = WITH_MASS && P.has_mass && !(P.has_adv && P.mass_merged);
  const Real alpha = P.alpha, beta_y = P.beta_y;
  const int t0 = P.has_adv ? PG : D;  // factors of the other pairs' steps (the mass term alone: its own)
  const int total = ne * IPE;
  for (int it = threadIdx.x; it < total; it += blockDim.x) {
    const int b = it / IPE;
    int r = it - b * IPE;
    // offset of the block: the other axes' indices, in increasing axis order
    int off = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) {
      if (k == A || k == B) continue;
      const int q = r / N;
      off += (r - q * N) * kpow(N, k);
      r = q;
    }
    Real* el = base + (size_t)b * S::PER_ELEM;
    const Real* mats = el + S::MOFF;
    const Real* src = OWN ? el : el + S::ND;
    Real v[N][N];  // v[i][j]: index i along A, j along B
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
      for (int j = 0; j < N; ++j) v[i][j] = src[off + i * SA + j * SB];
    Real acc[N][N];
    if constexpr (OWN) {
#pragma unroll
      for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) acc[i][j] = Real(0);
      const Real* rec = el + S::ROFF;
      const uint8_t* fb = reinterpret_cast<const uint8_t*>(rec + 4 * D);
      // own term of axis X (X == A: along the first index) then its factor along the other
      auto own_term = [&](auto xc) {
        constexpr int X = decltype(xc)::value;
        constexpr bool FIRST = X == A;
        constexpr int Y = FIRST ? B : A;
        const SlotMat<N, Real> dm(mats + (X * D + X) * S::MATP);
        const SlotMat<N, Real> tm(mats + (X * D + Y) * S::MATP);
        const Real scale = P.elem[X] ? P.elem[X][e0 + b] : Real(1);
        Real w[N][N];
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
          for (int j = 0; j < N; ++j) {
            Real s = Real(0);
#pragma unroll
            for (int k = 0; k < N; ++k) s += FIRST ? dm(i, k) * v[k][j] : dm(j, k) * v[i][k];
            w[i][j] = P.elem[X] ? s * scale : s;
          }
        if (P.has_adv) {
#pragma unroll
          for (int sd = 0; sd < 2; ++sd) {
            const int fi = X * 2 + sd;
            const uint32_t f = fb[fi];
            if (!f) continue;
            const int sl = sd ? N - 1 : 0;
            int64_t en = 0;
            if (f & 2u) {
              const int64_t n = P.sizes[X];
              const int64_t ca = ecoord[b][X];
              const int64_t cn = sd ? (ca + 1 == n ? 0 : ca + 1) : (ca == 0 ? n - 1 : ca - 1);
              en = e0 + b + (cn - ca) * P.estride[X];
            }
#pragma unroll
            for (int t = 0; t < N; ++t) {
              Real add = Real(0);
              const Real own = FIRST ? v[sl][t] : v[t][sl];
              if (f & 1u) add += rec[2 * fi] * own;
              if (f & 2u) {
                const int nidx = FIRST ? off + (N - 1 - sl) * SA + t * SB : off + t * SA + (N - 1 - sl) * SB;
                add += rec[2 * fi + 1] * xin[en * S::ND + nidx];
              } else if (f & 4u) {
                add += rec[2 * fi + 1] * P.g;
              }
              if (FIRST) w[sl][t] += add;
              else w[t][sl] += add;
            }
          }
        }
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
          for (int j = 0; j < N; ++j) {
            Real s = Real(0);
#pragma unroll
            for (int k = 0; k < N; ++k) s += FIRST ? tm(j, k) * w[i][k] : tm(i, k) * w[k][j];
            acc[i][j] += s;
          }
      };
      if (P.has_adv) {
        own_term(std::integral_constant<int, A>{});
        own_term(std::integral_constant<int, B>{});
      }
      if (mass) {
        // MD along the last axis (B of the last pair, scaled), then MT along A
        const SlotMat<N, Real> md(mats + (D * D + B) * S::MATP);
        const SlotMat<N, Real> mt(mats + (D * D + A) * S::MATP);
        const Real scale = P.elem_mass ? P.elem_mass[e0 + b] : Real(1);
        Real w[N][N];
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
          for (int j = 0; j < N; ++j) {
            Real s = Real(0);
#pragma unroll
            for (int k = 0; k < N; ++k) s += md(j, k) * v[i][k];
            w[i][j] = P.elem_mass ? s * scale : s;
          }
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
          for (int j = 0; j < N; ++j) {
            Real s = Real(0);
#pragma unroll
            for (int k = 0; k < N; ++k) s += mt(i, k) * w[k][j];
            acc[i][j] += s;
          }
      }
    } else {
      // the pair's shared factors along A and B (term PG's; equal to term PG + H's)
      const SlotMat<N, Real> fa(mats + (t0 < D ? t0 * D + A : D * D + A) * S::MATP);
      const SlotMat<N, Real> fbm(mats + (t0 < D ? t0 * D + B : D * D + B) * S::MATP);
      Real w[N][N];
#pragma unroll
      for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) {
          Real s = Real(0);
#pragma unroll
          for (int k = 0; k < N; ++k) s += fa(i, k) * v[k][j];
          w[i][j] = s;
        }
#pragma unroll
      for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) {
          Real s = Real(0);
#pragma unroll
          for (int k = 0; k < N; ++k) s += fbm(j, k) * w[i][k];
          acc[i][j] = s;
        }
    }
    Real* dst = el + (LAST ? 2 : 1) * S::ND;
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
      for (int j = 0; j < N; ++j) {
        const int q = off + i * SA + j * SB;
        if constexpr (LAST) nd_y_write(alpha, beta_y, ymode, dst + q, yout + (e0 + b) * S::ND + q, acc[i][j]);
        else dst[q] = acc[i][j];
      }
  }
}

// One batch of ne elements starting at e0 with the paired steps.
template <int D, int N, typename Real>
__device__ __forceinline__ void kronnd_paired_block(const KronNDParams<Real>& P, const Real* __restrict__ xin,
                                                    Real* __restrict__ yout, int64_t e0, int ne, Real* base,
                                                    int (*ecoord)[kMaxDim]) {
  constexpr int H = D / 2;
  // The pairs run from H - 1 down to 0: pair H - 1 (with the mass term) reaches Y first and stores
  // its blocks (Y is not zeroed).  The last step of pair PG runs on pair glast(PG), whose blocks
  // put N^glast consecutive threads on consecutive values (the axes below the pair): when that run
  // is a 32-byte sector or more the last pair writes y itself (nd_y_write), otherwise it
  // accumulates into Y and the coalesced output pass writes y.
  constexpr int GLAST_ADV = H == 1 ? 0 : H - 1;   // glast(0): pair 0 runs last
  constexpr int GLAST_MASS = H == 1 ? 0 : H - 2;  // glast(H - 1): the mass term alone
  constexpr bool YOUT_ADV = kpow(N, GLAST_ADV) * sizeof(Real) >= 32;
  constexpr bool YOUT_MASS = kpow(N, GLAST_MASS) * sizeof(Real) >= 32;
  const bool yout_ok = P.has_adv ? YOUT_ADV : YOUT_MASS;
  nd_setup<D, N>(P, xin, e0, ne, base, ecoord, false);
  static_for<0, H>([&](auto pc) {
    constexpr int PG = H - 1 - decltype(pc)::value;
    // a pair runs when it has advection terms, or the mass term alone (operators without
    // advection: the last pair carries it)
    if (P.has_adv || (PG == H - 1 && P.has_mass)) {
      const bool last = PG == 0 || !P.has_adv;
      const int ymode = (PG == H - 1 ? kYStore : kYAdd) | ((last && yout_ok) ? kYOut : kYAdd);
      static_for<0, H>([&](auto sc) {
        nd_pair_step<D, N, PG, decltype(sc)::value>(P, xin, base, ne, e0, ecoord, ymode, yout);
        __syncthreads();
      });
    }
  });
  if (!yout_ok) nd_output<D, N>(P, yout, e0, ne, base);
}

template <int D, int N, typename Real>
__global__ void __launch_bounds__(kKronNDThreads, 3)
    kronnd_paired_kernel(const __grid_constant__ KronNDParams<Real> P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Real* base = reinterpret_cast<Real*>(smem_raw);
  __shared__ int ecoord[64][kMaxDim];
  if (P.skip && *P.skip) return;
  const int EB = P.eb;
  for (int64_t e0 = P.e_begin + (int64_t)blockIdx.x * EB; e0 < P.nelem; e0 += (int64_t)gridDim.x * EB) {
    const int ne = (int)((P.nelem - e0) < EB ? (P.nelem - e0) : EB);
    kronnd_paired_block<D, N>(P, P.x, P.y, e0, ne, base, ecoord);
  }
}

// ------------------------------------------------------------------------------------------
// Mass-only variant (operators without advection terms: the mass operator, the mass inverse):
// the element's values are passed in place in ONE shared-memory array, next to the D mass
// matrices, so an element needs about a third of the layout above (6.4 instead of 21.7 KB at 6D
// p = 2 in FP64) and the SM keeps more elements resident.  The passes run group by group from
// axis 0 (scaled by the element factor) up; blocks of one step are disjoint, so each thread
// writes its block back where it read it, and the last step writes its block straight to y
// (its values lie INNER = N^(first axis of the group) apart, so consecutive threads write
// consecutive addresses).
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void cp_async_16(void* dst, const void* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

// Values of Real by which an element's first value lies past a 16-byte boundary in global memory;
// the element's slot in shared memory starts that many values into its (16-byte aligned) area, so
// the two copies have the same 16-byte phase and whole chunks move by 16-byte copies.
template <typename Real>
__device__ __forceinline__ int nd_phase(const Real* p) {
  return (int)((reinterpret_cast<uintptr_t>(p) / sizeof(Real)) & (16 / sizeof(Real) - 1));
}

template <int D, int N>
struct KronNDMassShape {
  using S = KronNDShape<D, N>;
  // the element's values (starting up to 3 values in, see nd_phase), then the D mass matrices
  // (16-byte aligned)
  static constexpr int MOFF = (S::ND + 6) / 4 * 4;
  static constexpr int PER_ELEM = MOFF + D * S::MATP;
};

template <int D, int N, int G, int ST, typename Real>
__device__ __forceinline__ void nd_mass_step(const KronNDParams<Real>& P, Real* base, int ne, int64_t e0,
                                             const Real* cm) {
  using S = KronNDShape<D, N>;
  using M = KronNDMassShape<D, N>;
  using GR = KronGroups<D, N, G>;
  constexpr int AX = 0;
  constexpr int g = GR::group(AX, ST);
  constexpr int LO = GR::lo(g), HI = GR::hi(g), GSZ = GR::size(g), INNER = GR::inner(g);
  constexpr int IPE = S::ND / GSZ;  // blocks per element
  constexpr bool FIRST = ST == 0, LAST = ST == GR::NG - 1;
  const int total = ne * IPE;
  for (int it = threadIdx.x; it < total; it += blockDim.x) {
    const int b = it / IPE;
    const int loc = it - b * IPE;
    const int o = loc / INNER, t = loc - o * INNER;
    const int off = o * GSZ * INNER + t;
    Real* el = base + (size_t)b * M::PER_ELEM;
    Real* u = el + nd_phase(P.x + (e0 + b) * S::ND);  // the element's values (see nd_phase)
    Real v[GSZ];
#pragma unroll
    for (int j = 0; j < GSZ; ++j) v[j] = u[off + j * INNER];
    static_for<0, HI - LO>([&](auto kc) {
      constexpr int k = GR::axis(g, decltype(kc)::value, FIRST, AX);
      constexpr int SK = kpow(N, k - LO);
      constexpr bool OWN = FIRST && k == AX;
      const SlotMat<N, Real> m((cm ? cm : el + M::MOFF) + k * S::MATP);
      Real scale = Real(1);
      if constexpr (OWN) {
        if (P.elem_mass) scale = P.elem_mass[e0 + b];
      }
#pragma unroll
      for (int ln = 0; ln < GSZ / N; ++ln) {
        const int p0 = (ln / SK) * SK * N + (ln % SK);
        Real w[N];
#pragma unroll
        for (int j = 0; j < N; ++j) {
          Real s = m(j, 0) * v[p0];
#pragma unroll
          for (int i = 1; i < N; ++i) s += m(j, i) * v[p0 + i * SK];
          w[j] = s;
        }
        if constexpr (OWN) {
          if (P.elem_mass) {
#pragma unroll
            for (int j = 0; j < N; ++j) w[j] *= scale;
          }
        }
#pragma unroll
        for (int j = 0; j < N; ++j) v[p0 + j * SK] = w[j];
      }
    });
    if constexpr (LAST) {
      Real* dst = P.y + (e0 + b) * S::ND + off;
#pragma unroll
      for (int j = 0; j < GSZ; ++j)
        dst[j * INNER] = (P.beta_y == Real(0)) ? P.alpha * v[j] : P.alpha * v[j] + P.beta_y * dst[j * INNER];
    } else {
#pragma unroll
      for (int j = 0; j < GSZ; ++j) u[off + j * INNER] = v[j];
    }
  }
}

// Asynchronous copy of one value from global to shared memory (4 or 8 bytes).
template <typename Real>
__device__ __forceinline__ void cp_async_value(Real* dst, const Real* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(Real) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}

// The CTA's batches alternate between two buffers of EB elements: while a batch computes in one,
// the next batch's input arrives in the other by asynchronous copies (issued at the start of the
// batch, one commit group per batch, awaited at the start of the next), so the input loads of a
// batch overlap the previous batch's passes.  The kernel is bound by registers, not shared
// memory, so the second buffer costs no resident warps.
template <int D, int N, int G, typename Real>
__global__ void __launch_bounds__(kKronNDThreads) kronnd_mass_kernel(const __grid_constant__ KronNDParams<Real> P) {
  using S = KronNDShape<D, N>;
  using M = KronNDMassShape<D, N>;
  using GR = KronGroups<D, N, G>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Real* base = reinterpret_cast<Real*>(smem_raw);
  __shared__ int ecoord[64][kMaxDim];
  if (P.skip && *P.skip) return;
  const int EB = P.eb;
  const int64_t stride = (int64_t)gridDim.x * EB;
  // input of the batch starting at e0 into buffer buf (one commit group, possibly empty)
  // element b's values occupy [a, a + ND) of its area (a = nd_phase); the area's 16-byte chunks
  // inside that range are whole 16-byte copies, the two partial ones value by value
  constexpr int R = 16 / (int)sizeof(Real);
  constexpr int NC = (S::ND + 2 * (R - 1)) / R + 1;  // chunks per element area, at most
  static_assert(M::MOFF >= S::ND + R - 1, "the values and their phase fit before the matrices");
  auto stage = [&](int64_t e0, int buf) {
    if (e0 < P.nelem) {
      const int ne = (int)((P.nelem - e0) < EB ? (P.nelem - e0) : EB);
      Real* dst = base + (size_t)buf * EB * M::PER_ELEM;
      for (int l = threadIdx.x; l < ne * NC; l += blockDim.x) {
        const int b = l / NC, k = l - b * NC;
        const Real* src = P.x + (e0 + b) * S::ND;  // the element's first value
        const int a = nd_phase(src);
        const int lo = k * R, hi = lo + R;  // the chunk, in values of the area
        if (hi <= a || lo >= a + S::ND) continue;
        Real* d = dst + (size_t)b * M::PER_ELEM;
        if (lo >= a && hi <= a + S::ND) {
          cp_async_16(d + lo, src + (lo - a));
        } else {
          for (int i = lo; i < hi; ++i)
            if (i >= a && i < a + S::ND) cp_async_value(d + i, src + (i - a));
        }
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  // mass matrices that are the same for every element (constant coefficient, the usual case):
  // one copy per CTA after the two buffers, instead of one per element and batch
  bool shared_mats = true;
#pragma unroll
  for (int kk = 0; kk < D; ++kk) shared_mats = shared_mats && (P.mslot[kk].off < 0 || P.mslot[kk].stride == 0);
  Real* cm = shared_mats ? base + (size_t)2 * EB * M::PER_ELEM : nullptr;
  if (shared_mats) {
    for (int l = threadIdx.x; l < D * S::MAT; l += blockDim.x) {
      const int kk = l / S::MAT, q = l - kk * S::MAT;
      const KronMat mk = P.mslot[kk];
      cm[kk * S::MATP + q] = mk.off >= 0 ? P.mats[mk.off + q] : Real(0);
    }
  }
  int64_t e0 = P.e_begin + (int64_t)blockIdx.x * EB;
  stage(e0, 0);
  for (int k = 0; e0 < P.nelem; e0 += stride, ++k) {
    const int ne = (int)((P.nelem - e0) < EB ? (P.nelem - e0) : EB);
    Real* cur = base + (size_t)(k & 1) * EB * M::PER_ELEM;
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");  // this batch's copies (this thread's)
    __syncthreads();  // every thread's copies landed; the previous batch is done with the other buffer
    stage(e0 + stride, (k + 1) & 1);
    if (!shared_mats) {
      if (threadIdx.x < ne) {
        const int64_t e = e0 + threadIdx.x;
#pragma unroll
        for (int kk = 0; kk < D; ++kk) ecoord[threadIdx.x][kk] = (int)((e / P.estride[kk]) % P.sizes[kk]);
      }
      __syncthreads();
      for (int l = threadIdx.x; l < ne * D * S::MAT; l += blockDim.x) {
        const int b = l / (D * S::MAT);
        const int r = l - b * (D * S::MAT);
        const int kk = r / S::MAT, q = r - kk * S::MAT;
        const KronMat mk = P.mslot[kk];
        Real v = Real(0);
        if (mk.off >= 0) v = P.mats[mk.off + (int64_t)ecoord[b][kk] * mk.stride + q];
        cur[(size_t)b * M::PER_ELEM + M::MOFF + kk * S::MATP + q] = v;
      }
      __syncthreads();
    }
    // the last step writes y; the barrier after it (or the next batch's first one) frees `cur`
    static_for<0, GR::NG>([&](auto sc) {
      nd_mass_step<D, N, G, decltype(sc)::value>(P, cur, ne, e0, cm);
      if constexpr (decltype(sc)::value + 1 < GR::NG) __syncthreads();
    });
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");  // no copy outlives the kernel
}

// Many operators of one (D, N) and kernel variant V (0: one pass per axis, 1 / 2: groups of 2 / 3
// axes, 3: paired axes) in one persistent launch: table[i] holds instance i's parameters (forward operator, x / y
// set per apply), its element batches are the global batch indices [first[i], first[i + 1]);
// every CTA walks the global batches.  Register caps keep the occupancy of the single-operator
// kernels (per-axis: 4 CTAs per SM, at most 64 registers; grouped: 2, at most 128): the
// parameters read from the table, rather than from constant memory, would otherwise take the
// register count past them.
template <int D, int N, int V, typename Real>
__global__ void __launch_bounds__(kKronNDThreads, V == 0 ? 4 : ((V == 1 || V == 2) ? 2 : 1))
    kronnd_batch_kernel(const KronNDParams<Real>* __restrict__ table, const int64_t* __restrict__ first, int count,
                        int EB) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Real* base = reinterpret_cast<Real*>(smem_raw);
  __shared__ Real escale[64];
  __shared__ int ecoord[64][kMaxDim];
  const int64_t total = first[count];
  for (int64_t gb = blockIdx.x; gb < total; gb += gridDim.x) {
    int lo = 0, hi = count;  // instance: the last i with first[i] <= gb
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (first[mid] <= gb) lo = mid;
      else hi = mid;
    }
    const KronNDParams<Real>& P = table[lo];
    const int64_t e0 = (gb - first[lo]) * EB;
    const int ne = (int)((P.nelem - e0) < EB ? (P.nelem - e0) : EB);
    if constexpr (V == 0) kronnd_block<D, N>(P, P.x, P.y, e0, ne, EB, base, escale, ecoord);
    else if constexpr (V == 3) kronnd_paired_block<D, N>(P, P.x, P.y, e0, ne, base, ecoord);
    else kronnd_grouped_block<D, N, V + 1>(P, P.x, P.y, e0, ne, base, ecoord);
  }
}

}  // namespace dgop
