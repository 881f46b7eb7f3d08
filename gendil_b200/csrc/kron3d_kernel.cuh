// Register-resident Kronecker-form DG operator kernel for 3D hexahedra, N = p + 1 <= 5.
//
// N consecutive lanes own one element; lane t holds an N x N plane of it in registers:
//   layout Z: plane z = t, values [x][y]      layout Y: plane y = t, values [x][z]
// Operators along x and y run in layout Z, along x and z in layout Y.  Schedule per element
// (9 n x n passes, 4 layout exchanges):
//
//   Z: px = Dx u + x-faces ; qx = Txy px ; py = Dy u + y-faces             exchange qx, py -> Y
//   Y: out = Txz qx + Tyx Tyz py ; pz = Dz u + z-faces (mass merged) ; qz = Tzx pz
//                                                                           exchange qz, out -> Z
//   Z: out += Tzy qz ; y = alpha out + beta y
//
// The upwind neighbour trace of every inflow face is added to the face slice of the D-pass
// output, so the tangential passes that follow apply the face's tangential operator to it.
//
// Memory: each warp loops over groups of 32/N consecutive elements (persistent grid).  The
// group's DoFs, the neighbour traces its inflow faces need and a per-element record of its face
// decisions are staged into padded shared memory one group ahead (double buffered, coalesced
// cp.async copies), so loads of the next group overlap the arithmetic of this one; results leave
// through the same buffer with coalesced stores.  Constant 1D matrices are read from
// kernel-parameter space, only element-dependent ones from global memory.  For even N the layout
// exchanges are register butterflies (shfl_xor within the element's lanes); odd N exchange
// through a shared tile.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "dgop_params.h"
#include "kron.h"

namespace dgop {

template <int N, typename Real>
struct Kron3DShape {
  static constexpr int EPW = 32 / N;  // elements per warp group
  static constexpr int NN = N * N, NNN = N * N * N;
  // staging copy granule (bytes): 16 when a plane is a whole number of 16-byte chunks
  static constexpr int CB = (NN * (int)sizeof(Real)) % 16 == 0 ? 16 : ((NN * (int)sizeof(Real)) % 8 == 0 ? 8 : 4);
  static constexpr int CR = CB / (int)sizeof(Real);  // Reals per chunk
  static constexpr int pad_for(int p) { return ((NN + p) * (int)sizeof(Real)) % CB == 0 ? p : pad_for(p + 1); }
  // vector width (Reals) of shared-memory accesses along x: 16 bytes when N allows it
  static constexpr int V = (N % (16 / (int)sizeof(Real)) == 0) ? 16 / (int)sizeof(Real) : 1;
  // Shared-memory bank model: accesses of G bytes are served 128 bytes at a time (8, 16 or 32
  // lanes together); two lanes of one such phase conflict when their G-byte granules fall in the
  // same bank group.  `distinct` checks one access pattern: offset(le, t) in Reals.
  template <typename F>
  static constexpr bool distinct(int vreals, F offset) {
    const int G = vreals * (int)sizeof(Real);
    const int L = G >= 16 ? 8 : (G == 8 ? 16 : 32);
    const int CH = 128 / (G >= 16 ? 16 : G);
    for (int ph = 0; ph < 32 / L; ++ph) {
      unsigned long long seen = 0;
      for (int l = ph * L; l < ph * L + L; ++l) {
        const int le = l / N, t = l - le * N;
        if (le >= EPW) continue;
        const int c = (offset(le, t) / vreals) % CH;
        if ((seen >> c) & 1ull) return false;
        seen |= 1ull << c;
      }
    }
    return true;
  }
  // Staged element layout: (x, y, z) at z * SP + y * N + x, element stride SE.  The smallest
  // strides (keeping the copy granule's alignment) for which the layout-Z and layout-Y plane
  // accesses are conflict-free; fallback: the dense plane padded to the copy granule.
  struct Staged {
    int SP, SE;
  };
  static constexpr Staged staged_geom() {
    // a conflict-free layout more than 25 % larger than the dense one costs more shared memory
    // (warps per SM) than its conflicts cost
    const int dense = N * (NN + pad_for(1));
    for (int se = N * NN; se <= dense + dense / 4; ++se) {
      if ((se * (int)sizeof(Real)) % CB || se % V) continue;
      for (int sp = NN; N * sp <= se; ++sp) {
        if ((sp * (int)sizeof(Real)) % CB || sp % V) continue;
        if (distinct(V, [&](int le, int t) { return le * se + t * sp; }) &&
            distinct(V, [&](int le, int t) { return le * se + t * N; }))
          return {sp, se};
      }
    }
    return {NN + pad_for(1), N * (NN + pad_for(1))};
  }
  static constexpr int SP = staged_geom().SP;  // staged plane stride (Reals)
  static constexpr int SE = staged_geom().SE;  // staged element stride
  // neighbour traces: one slot per axis (N rows of N), used by the first face of that axis that
  // needs a neighbour trace; a second one on the same axis (rare) is read from global memory.
  // Rows are read V-wide; the element stride TE is the smallest conflict-free one.
  static constexpr int RB = (N * (int)sizeof(Real)) % 16 == 0 ? 16 : ((N * (int)sizeof(Real)) % 8 == 0 ? 8 : 4);
  static constexpr int TR = N;                // trace row stride
  static constexpr int TS = N * TR;           // trace slot stride
  static constexpr int trace_stride() {
    for (int te = 3 * TS; te <= 3 * TS + 64; ++te) {
      if ((te * (int)sizeof(Real)) % RB || te % V) continue;
      if (distinct(V, [&](int le, int t) { return le * te + t * TR; })) return te;
    }
    return 3 * TS;
  }
  static constexpr int TE = trace_stride();   // traces per element
  // face record per element: 12 coefficients (axis, side, {corner, neighbour/inflow}) + flag word
  static constexpr int RE = 12 + (16 / (int)sizeof(Real));
  static constexpr int STAGE = EPW * (SE + TE + RE);  // one pipeline stage: DoFs, traces, records
  static constexpr bool BUTTERFLY = (N == 2 || N == 4);  // shuffle exchanges possible
  // Exchange tile per element, layout [y][z][x]: value (x, y, z) at y * TA + z * N + x, element
  // stride TSE.  Both sides of an exchange access V consecutive x values; TA and TSE are the
  // smallest strides for which neither side has a shared-memory bank conflict (tile_geom).
  struct Geom {
    int A, TSE;
  };
  static constexpr Geom tile_geom() {
    const int G = V * (int)sizeof(Real);  // bytes per access
    const int limit = (NNN + 1) + (NNN + 1) / 4;  // at most 25 % above the dense tile
    const int L = G == 16 ? 8 : (G == 8 ? 16 : 32);  // lanes served together
    const int CH = 128 / G;                          // access granules per 128 bytes
    for (int tse = NNN; tse <= limit; ++tse) {
      if (tse % V) continue;
      for (int a = NN; N == 1 || (N - 1) * a + NN <= tse; ++a) {
        if (a % V) continue;
        bool ok = true;
        for (int ph = 0; ph < 32 / L && ok; ++ph) {
          unsigned put = 0, get = 0;
          for (int l = ph * L; l < ph * L + L && ok; ++l) {
            const int le = l / N, t = l - le * N;
            if (le >= EPW) continue;
            const int cp = ((le * tse + t * N) / V) % CH, cg = ((le * tse + t * a) / V) % CH;
            if ((put >> cp) & 1u || (get >> cg) & 1u) ok = false;
            put |= 1u << cp;
            get |= 1u << cg;
          }
        }
        if (ok) return {a, tse};
        if (N == 1) break;
      }
    }
    return {NN, NNN};  // dense (bank conflicts accepted)
  }
  static constexpr int TA = tile_geom().A;
  static constexpr int TSE = tile_geom().TSE;
  static constexpr int TILE = EPW * TSE;
  // shared memory per warp (Reals): STAGES pipeline stages (+ the exchange tile unless shuffles)
  static constexpr int warp_smem(int stages, bool shfl) {
    return stages * STAGE + ((shfl && BUTTERFLY) ? 0 : ((TILE + 3) / 4) * 4);
  }
};

// V consecutive Reals as one shared or global access (V = 1, 2 or 4; 16-byte aligned addresses
// when V > 1), moved component-wise into register arrays.
template <typename Real, int V>
struct Vec16 {};
template <>
struct Vec16<double, 2> {
  using T = double2;
};
template <>
struct Vec16<float, 2> {
  using T = float2;
};
template <>
struct Vec16<float, 4> {
  using T = float4;
};

template <typename Real, int V>
__device__ __forceinline__ void vload(const Real* p, Real (&v)[V]) {
  if constexpr (V == 1) {
    v[0] = p[0];
  } else if constexpr (V == 2) {
    const auto w = *reinterpret_cast<const typename Vec16<Real, 2>::T*>(p);
    v[0] = w.x;
    v[1] = w.y;
  } else {
    static_assert(V == 4 && sizeof(Real) == 4, "unsupported vector width");
    const float4 w = *reinterpret_cast<const float4*>(p);
    v[0] = w.x;
    v[1] = w.y;
    v[2] = w.z;
    v[3] = w.w;
  }
}
template <typename Real, int V>
__device__ __forceinline__ void vstore(Real* p, const Real (&v)[V]) {
  if constexpr (V == 1) {
    p[0] = v[0];
  } else if constexpr (V == 2) {
    using T = typename Vec16<Real, 2>::T;
    T w;
    w.x = v[0];
    w.y = v[1];
    *reinterpret_cast<T*>(p) = w;
  } else {
    static_assert(V == 4 && sizeof(Real) == 4, "unsupported vector width");
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  }
}
template <typename Real, int V>
__device__ __forceinline__ void vldg(const Real* p, Real (&v)[V]) {
  if constexpr (V == 1) {
    v[0] = __ldg(p);
  } else if constexpr (V == 2) {
    const auto w = __ldg(reinterpret_cast<const typename Vec16<Real, 2>::T*>(p));
    v[0] = w.x;
    v[1] = w.y;
  } else {
    static_assert(V == 4 && sizeof(Real) == 4, "unsupported vector width");
    const float4 w = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = w.x;
    v[1] = w.y;
    v[2] = w.z;
    v[3] = w.w;
  }
}

// Y[i][j] = sum_r A(i, r) X[r][j]      (operator along the first plane index)
template <int N, typename Real, typename Mat>
__device__ __forceinline__ void apply_first(const Mat& A, const Real (&X)[N][N], Real (&Y)[N][N]) {
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) {
      Real s = A(i, 0) * X[0][j];
#pragma unroll
      for (int r = 1; r < N; ++r) s += A(i, r) * X[r][j];
      Y[i][j] = s;
    }
}

// Y[i][j] = sum_r A(j, r) X[i][r]      (operator along the second plane index)
template <int N, typename Real, typename Mat>
__device__ __forceinline__ void apply_second(const Mat& A, const Real (&X)[N][N], Real (&Y)[N][N]) {
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) {
      Real s = A(j, 0) * X[i][0];
#pragma unroll
      for (int r = 1; r < N; ++r) s += A(j, r) * X[i][r];
      Y[i][j] = s;
    }
}

template <int N, typename Real>
struct RegMat {
  Real a[N][N];
  __device__ __forceinline__ Real operator()(int i, int j) const { return a[i][j]; }
};

template <int N, typename Real, int SLOT>
struct ParamMat {
  const KronParams<Real>& P;
  __device__ __forceinline__ Real operator()(int i, int j) const { return P.cm[SLOT][i * N + j]; }
};

// Apply slot SLOT's matrix (for element coordinate `coord` along its axis) along the first or
// second plane index: constant matrices come from kernel-parameter space.  VM: the slot mask the
// kernel is compiled for (kron.h).
template <int N, typename Real, int SLOT, bool FIRST, uint32_t VM = kVaryRuntime>
__device__ __forceinline__ void kron_apply(const KronParams<Real>& P, uint32_t coord, const Real (&X)[N][N],
                                           Real (&Y)[N][N]) {
  bool vary;
  if constexpr (VM == kVaryRuntime) vary = P.vary[SLOT] != 0;
  else vary = ((VM >> SLOT) & 1u) != 0;
  if (vary) {
    RegMat<N, Real> A;
    const Real* p = P.mats + P.vm[SLOT].off + (int64_t)coord * P.vm[SLOT].stride;
    // N x N blocks at offsets that are multiples of the vector width (checked at setup)
    constexpr int V = Kron3DShape<N, Real>::V;
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
      for (int j = 0; j < N; j += V) {
        Real v[V];
        vldg<Real, V>(p + i * N + j, v);
#pragma unroll
        for (int q = 0; q < V; ++q) A.a[i][j + q] = v[q];
      }
    if (FIRST) apply_first<N>(A, X, Y);
    else apply_second<N>(A, X, Y);
  } else {
    ParamMat<N, Real, SLOT> A{P};
    if (FIRST) apply_first<N>(A, X, Y);
    else apply_second<N>(A, X, Y);
  }
}

// Layout exchange between the N lanes of an element: X[i][j] held by lane t (plane index t of
// the third axis) becomes Y[i][k] = X_k[i][t].  Even N: shfl_xor butterflies on the lane bits;
// at the stage on bit b each lane keeps the column of each pair (j, j|m) whose bit b matches its
// own and trades the other with lane t ^ m.
template <int N, typename Real>
__device__ __forceinline__ void exchange_butterfly(int t, Real (&X)[N][N]) {
#pragma unroll
  for (int b = 0; (1 << b) < N; ++b) {
    const int m = 1 << b;
    const bool hi = (t & m) != 0;
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
      for (int j = 0; j < N; ++j) {
        if (j & m) continue;
        const Real send = hi ? X[i][j] : X[i][j | m];
        const Real recv = __shfl_xor_sync(0xffffffffu, send, m);
        if (hi) X[i][j] = recv;
        else X[i][j | m] = recv;
      }
  }
}

// Plane of an element in layout Z (values [x][y] of plane z = t) from the staged layout, where
// (x, y, z) sits at z * SP + y * N + x: V-wide loads along x.
template <int N, typename Real>
__device__ __forceinline__ void load_plane_z(const Real* ub, int t, bool active, Real (&u)[N][N]) {
  using S = Kron3DShape<N, Real>;
  constexpr int V = S::V;
#pragma unroll
  for (int j = 0; j < N; ++j)
#pragma unroll
    for (int i = 0; i < N; i += V) {
      Real v[V];
      if (active) vload<Real, V>(ub + t * S::SP + N * j + i, v);
#pragma unroll
      for (int q = 0; q < V; ++q) u[i + q][j] = active ? v[q] : Real(0);
    }
}

// Plane of an element in layout Y (values [x][z] of plane y = t) from the staged layout.
template <int N, typename Real>
__device__ __forceinline__ void load_plane_y(const Real* ub, int t, bool active, Real (&u)[N][N]) {
  using S = Kron3DShape<N, Real>;
  constexpr int V = S::V;
#pragma unroll
  for (int k = 0; k < N; ++k)
#pragma unroll
    for (int i = 0; i < N; i += V) {
      Real v[V];
      if (active) vload<Real, V>(ub + k * S::SP + N * t + i, v);
#pragma unroll
      for (int q = 0; q < V; ++q) u[i + q][k] = active ? v[q] : Real(0);
    }
}

// Layout exchange through the warp's shared tile.  z_to_y: lane t holds X[i][j] = (x=i, y=j, z=t)
// and receives X[i][k] = (x=i, y=t, z=k); otherwise the reverse.  Tile layout [y][z][x].
template <int N, typename Real>
__device__ __forceinline__ void exchange_tile(Real* tile, int le, int t, bool slot, bool z_to_y, Real (&X)[N][N]) {
  using S = Kron3DShape<N, Real>;
  constexpr int V = S::V;
  Real* b = tile + le * S::TSE;
  // layout Z side: lane t = z owns (x, y = j) at j * TA + t * N + x;
  // layout Y side: lane t = y owns (x, z = k) at t * TA + k * N + x
  auto z_side = [&](int j, int i) { return b + j * S::TA + t * N + i; };
  auto y_side = [&](int k, int i) { return b + t * S::TA + k * N + i; };
  if (slot) {
#pragma unroll
    for (int j = 0; j < N; ++j)
#pragma unroll
      for (int i = 0; i < N; i += V) {
        Real v[V];
#pragma unroll
        for (int q = 0; q < V; ++q) v[q] = X[i + q][j];
        vstore<Real, V>(z_to_y ? z_side(j, i) : y_side(j, i), v);
      }
  }
  __syncwarp();
  if (slot) {
#pragma unroll
    for (int j = 0; j < N; ++j)
#pragma unroll
      for (int i = 0; i < N; i += V) {
        Real v[V];
        vload<Real, V>(z_to_y ? y_side(j, i) : z_side(j, i), v);
#pragma unroll
        for (int q = 0; q < V; ++q) X[i + q][j] = v[q];
      }
  }
  __syncwarp();  // the tile is free again
}

// Element coordinates (x fastest).
template <typename Real>
__device__ __forceinline__ void kron_coords(const KronParams<Real>& P, uint32_t e, uint32_t (&c)[3]) {
  uint32_t q;
  P.fdx.divmod(e, q, c[0]);
  P.fdy.divmod(q, c[2], c[1]);
}

// Upwind decision for face (a, s) of element e (cartesianndmesh.hpp:109-198 for the neighbour,
// advectionoperator.hpp:379-386 / 422-428 for the flux):
//   corner: add phi * el * u[slice]              (outflow face, own trace)
//   use_nb: add coef * neighbour trace            (inflow face, or the transposed coupling)
//   use_g:  add coef * g                          (inflow boundary face with inflow value g)
struct FaceDecision {
  bool corner, use_nb, use_g;
  int64_t d;  // neighbour offset
};

template <typename Real>
__device__ __forceinline__ FaceDecision face_decide(const KronParams<Real>& P, int a, int s, const uint32_t (&c)[3],
                                                    int64_t e, Real tsign, Real el_self, Real& phi, Real& coef) {
  FaceDecision f{false, false, false, 0};
  const int64_t n = P.sizes[a];
  const int64_t st = a == 0 ? 1 : (a == 1 ? P.sizes[0] : P.sizes[0] * P.sizes[1]);
  bool interior;
  if (s == 0) {
    interior = c[a] > 0 || P.periodic[a];
    f.d = c[a] > 0 ? -st : (n - 1) * st;
  } else {
    interior = (int64_t)c[a] + 1 < n || P.periodic[a];
    f.d = (int64_t)c[a] + 1 < n ? st : -(n - 1) * st;
  }
  const bool active = interior ? (P.flags & kFaceInt) : (P.flags & kFaceBnd);
  phi = P.phi[a][c[a] * 2 + s];
  coef = Real(0);
  if (!active) return f;
  const bool outflow = phi * tsign * el_self > Real(0);
  f.corner = outflow;
  if (!(P.flags & kTranspose)) {
    if (!outflow) {
      coef = phi * el_self;
      f.use_nb = interior;
      f.use_g = !interior;
    }
  } else if (interior) {
    // transposed coupling: the neighbour's row, taken when its face (1-s) is inflow for it
    const uint32_t cn = s ? ((int64_t)c[a] + 1 == n ? 0 : c[a] + 1) : (c[a] == 0 ? (uint32_t)(n - 1) : c[a] - 1);
    const Real phin = P.phi[a][cn * 2 + (1 - s)];
    const Real eln = P.elem[a] ? P.elem[a][e + f.d] : Real(1);
    if (!(phin * tsign * eln > Real(0))) {
      coef = phin * eln;
      f.use_nb = true;
    }
  }
  return f;
}

template <typename Real>
__device__ __forceinline__ Real tan_sign(const KronParams<Real>& P, int a, const uint32_t (&c)[3]) {
  Real s = Real(1);
#pragma unroll
  for (int k = 0; k < 3; ++k)
    if (k != a) s *= (Real)P.sgn[a][k][c[k]];
  return s;
}

// Is the x neighbour on side s the adjacent element of the same staged group?
__device__ __forceinline__ bool x_in_group(int s, int le, int ne, uint32_t cx, int64_t nx) {
  const int rl = le + (s ? 1 : -1);
  return rl >= 0 && rl < ne && (s ? (int64_t)cx + 1 < nx : cx > 0);
}

enum TraceSrc { kTraceLocal = 0, kTraceSlot = 1, kTraceGlobal = 2 };
// Face record bits (5 per face f = axis * 2 + side): corner, neighbour trace, inflow value g,
// and the trace source (TraceSrc) in bits 3-4.
enum : uint32_t { kRecCorner = 1u, kRecNb = 2u, kRecG = 4u };

template <typename Real>
__device__ __forceinline__ int64_t neighbour_offset(const KronParams<Real>& P, int a, int s, uint32_t ca) {
  const int64_t n = P.sizes[a];
  const int64_t st = a == 0 ? 1 : (a == 1 ? P.sizes[0] : P.sizes[0] * P.sizes[1]);
  if (s == 0) return ca > 0 ? -st : (n - 1) * st;
  return (int64_t)ca + 1 < n ? st : -(n - 1) * st;
}

// One staged neighbour-trace row (N Reals), V-wide.
template <int N, typename Real>
__device__ __forceinline__ void trace_row(const Real* p, Real (&v)[N]) {
  constexpr int V = Kron3DShape<N, Real>::V;
#pragma unroll
  for (int r = 0; r < N; r += V) {
    Real w[V];
    vload<Real, V>(p + r, w);
#pragma unroll
    for (int q = 0; q < V; ++q) v[r + q] = w[q];
  }
}

// Face terms of axis a added to a D-pass output Pm (plane [first][second]; the face slice is along
// the first index when FIRST), from the element's face record (see stage_group).  nbrow(side, src,
// e_nb, v) reads this lane's row of the neighbour trace of that side from the group's staged DoFs
// (x only), the axis' staged trace slot (V-wide), or global memory.
template <int N, typename Real, bool FIRST, typename NbRow>
__device__ __forceinline__ void kron_faces(const KronParams<Real>& P, int a, const uint32_t (&c)[3], int64_t e,
                                           uint32_t flags, const Real* rec, const Real (&U)[N][N], Real (&Pm)[N][N],
                                           NbRow nbrow) {
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const int sl = s ? N - 1 : 0;
    const uint32_t f = (flags >> (5 * (a * 2 + s))) & 31u;
    if (f & kRecCorner) {
      const Real k = rec[(a * 2 + s) * 2];
#pragma unroll
      for (int r = 0; r < N; ++r) {
        if (FIRST) Pm[sl][r] += k * U[sl][r];
        else Pm[r][sl] += k * U[r][sl];
      }
    }
    if (f & (kRecNb | kRecG)) {
      const Real k = rec[(a * 2 + s) * 2 + 1];
      if (f & kRecNb) {
        const int src = (int)(f >> 3);
        const int64_t en = src == kTraceGlobal ? e + neighbour_offset(P, a, s, c[a]) : e;
        Real v[N];
        nbrow(s, src, en, v);
#pragma unroll
        for (int r = 0; r < N; ++r) {
          if (FIRST) Pm[sl][r] += k * v[r];
          else Pm[r][sl] += k * v[r];
        }
      } else {
#pragma unroll
        for (int r = 0; r < N; ++r) {
          if (FIRST) Pm[sl][r] += k * P.g;
          else Pm[r][sl] += k * P.g;
        }
      }
    }
  }
}

template <int CB>
__device__ __forceinline__ void cp_async(void* smem_dst, const void* gsrc) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  if constexpr (CB == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gsrc));
  else asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(gsrc), "n"(CB));
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int K>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(K)); }

__device__ __forceinline__ int group_size(int epw, int64_t remaining) {
  return remaining < epw ? (int)remaining : epw;
}

// Copy N contiguous Reals (a trace row) from global to shared memory.
template <int N, typename Real>
__device__ __forceinline__ void copy_row(Real* dst, const Real* src) {
  using S = Kron3DShape<N, Real>;
  constexpr int R = S::RB / (int)sizeof(Real);
#pragma unroll
  for (int i = 0; i < N; i += R) cp_async<S::RB>(dst + i, src + i);
}

// Stage the DoFs of elements [e0, e0 + ne) into `buf` (padded layout, coalesced); for advection,
// also each element's face record and the neighbour traces its faces will read (lane t copies
// row t of each trace).
template <int N, typename Real>
__device__ __forceinline__ void stage_group(const KronParams<Real>& P, int64_t e0, int ne, Real* buf, int lane,
                                            int le, int t, bool adv) {
  using S = Kron3DShape<N, Real>;
  const int nchunks = ne * S::NNN / S::CR;
  const Real* src = P.x + e0 * S::NNN;
  for (int ch = lane; ch < nchunks; ch += 32) {
    const int d = ch * S::CR;
    const int r = d / S::NNN, o = d - r * S::NNN;
    const int z = o / S::NN, w = o - z * S::NN;
    cp_async<S::CB>(buf + r * S::SE + z * S::SP + w, src + d);
  }
  if (!adv || le >= ne) return;
  const int64_t e = e0 + le;
  uint32_t c[3];
  kron_coords(P, (uint32_t)e, c);
  Real* tb = buf + S::EPW * S::SE + le * S::TE;
  Real* rb = buf + S::EPW * (S::SE + S::TE) + le * S::RE;
  uint32_t flags = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const Real tsign = tan_sign(P, a, c);
    const Real el = P.elem[a] ? P.elem[a][e] : Real(1);
    bool slot_taken = false;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      Real phi, coef;
      const FaceDecision f = face_decide(P, a, s, c, e, tsign, el, phi, coef);
      uint32_t bits = 0;
      if (f.corner) bits |= kRecCorner;
      if (f.use_g) bits |= kRecG;
      int src = kTraceLocal;
      if (f.use_nb) {
        bits |= kRecNb;
        if (!(a == 0 && x_in_group(s, le, ne, c[0], P.sizes[0]))) src = slot_taken ? kTraceGlobal : kTraceSlot;
      }
      bits |= (uint32_t)src << 3;
      flags |= bits << (5 * (a * 2 + s));
      if (t == 0) {
        rb[(a * 2 + s) * 2] = phi * el;
        rb[(a * 2 + s) * 2 + 1] = coef;
      }
      if (src != kTraceSlot) continue;  // staged DoFs (x neighbours in the group) or global memory
      slot_taken = true;
      const Real* un = P.x + (e + f.d) * S::NNN;
      const int sl = s ? 0 : N - 1;  // the neighbour's opposite slice
      Real* dst = tb + a * S::TS + t * S::TR;
      if (a == 0) {
#pragma unroll
        for (int r = 0; r < N; ++r) cp_async<(int)sizeof(Real)>(dst + r, un + sl + N * r + S::NN * t);
      } else if (a == 1) {
        copy_row<N>(dst, un + N * sl + S::NN * t);
      } else {
        copy_row<N>(dst, un + N * t + S::NN * sl);
      }
    }
  }
  if (t == 0) *reinterpret_cast<uint32_t*>(rb + 12) = flags;
}

constexpr int kron_max_warps = 4;  // warps per CTA of kron3d_kernel (128 threads)

// Kernel variants (chosen per operator by the autotuner):
//   STAGES 2: the next group is staged while this one computes; 1: no overlap inside the warp,
//   less shared memory per warp and so more warps per SM
//   SHFL:    layout exchanges by shuffle butterflies (even N) instead of the shared tile
//   DOT:     the inner-product epilogue (P.dot_partials; FP64 solvers) is compiled in
//   VM:      the slot mask the kernel is compiled for (kVaryRuntime: read P.vary)
template <int N, typename Real, bool SEP, int STAGES, bool SHFL, bool DOT, uint32_t VM>
__device__ __forceinline__ void kron3d_body(const KronParams<Real>& P) {
  using S = Kron3DShape<N, Real>;
  constexpr int NN = S::NN, NNN = S::NNN, EPW = S::EPW;
  constexpr bool BFLY = SHFL && S::BUTTERFLY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int le = lane / N, t = lane - le * N;
  Real* wbase = reinterpret_cast<Real*>(smem_raw) + (size_t)warp * S::warp_smem(STAGES, SHFL);
  [[maybe_unused]] Real* tile = wbase + STAGES * S::STAGE;
  const int64_t ngroups = (P.nelem - P.e_begin + EPW - 1) / EPW;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const bool adv = P.has_adv != 0;
  const bool slot = le < EPW;
  if (P.skip && *P.skip) return;  // a finished solve: nothing to do
  [[maybe_unused]] double dot_acc = 0.0;

  int64_t g = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
  if constexpr (STAGES == 2) {
    if (g < ngroups) stage_group<N>(P, P.e_begin + g * EPW, group_size(EPW, P.nelem - P.e_begin - g * EPW), wbase, lane, le, t, adv);
    cp_async_commit();
  }
  for (int it = 0; g < ngroups; g += nwarps, ++it) {
    Real* buf = wbase + (STAGES == 2 ? (it & 1) * S::STAGE : 0);
    if constexpr (STAGES == 2) {
      const int64_t gn = g + nwarps;
      if (gn < ngroups)
        stage_group<N>(P, P.e_begin + gn * EPW, group_size(EPW, P.nelem - P.e_begin - gn * EPW), wbase + ((it + 1) & 1) * S::STAGE, lane, le,
                       t, adv);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      stage_group<N>(P, P.e_begin + g * EPW, group_size(EPW, P.nelem - P.e_begin - g * EPW), buf, lane, le, t, adv);
      cp_async_commit();
      cp_async_wait<0>();
    }
    __syncwarp();
    const int64_t e0 = P.e_begin + g * EPW;
    const int ne = group_size(EPW, P.nelem - e0);
    const int64_t e = e0 + le;
    const bool active = slot && le < ne;
    uint32_t c[3] = {0, 0, 0};
    if (active) kron_coords(P, (uint32_t)e, c);
    const Real* ub = buf + (slot ? le : 0) * S::SE;
    const Real* tb = buf + EPW * S::SE + (slot ? le : 0) * S::TE;
    const Real* rec = buf + EPW * (S::SE + S::TE) + (slot ? le : 0) * S::RE;
    const uint32_t fflags = (adv && active) ? *reinterpret_cast<const uint32_t*>(rec + 12) : 0u;
    Real qx[N][N], py[N][N];

    // ------------------------------------------------------------ layout Z (plane z = t)
    if (adv) {
      Real u[N][N];
      load_plane_z<N>(ub, t, active, u);
      {
        Real px[N][N];
        kron_apply<N, Real, kSlotDX, true, VM>(P, c[0], u, px);
        if (P.elem[0]) {
          const Real elx = active ? P.elem[0][e] : Real(1);
#pragma unroll
          for (int i = 0; i < N; ++i)
#pragma unroll
            for (int j = 0; j < N; ++j) px[i][j] *= elx;
        }
        if (active)
          kron_faces<N, Real, true>(P, 0, c, e, fflags, rec, u, px, [&](int s, int src, int64_t en, Real(&v)[N]) {
            const int sl = s ? 0 : N - 1;  // the neighbour's opposite slice
            if (src == kTraceSlot) {
              trace_row<N>(tb + 0 * S::TS + t * S::TR, v);
            } else {
#pragma unroll
              for (int r = 0; r < N; ++r)
                v[r] = src == kTraceLocal ? ub[(s ? 1 : -1) * S::SE + t * S::SP + sl + N * r]
                                          : P.x[en * NNN + sl + N * r + NN * t];
            }
          });
        kron_apply<N, Real, kSlotTXY, false, VM>(P, c[1], px, qx);
      }
      kron_apply<N, Real, kSlotDY, false, VM>(P, c[1], u, py);
      if (P.elem[1]) {
        const Real ely = active ? P.elem[1][e] : Real(1);
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
          for (int j = 0; j < N; ++j) py[i][j] *= ely;
      }
      if (active)
        kron_faces<N, Real, false>(P, 1, c, e, fflags, rec, u, py, [&](int s, int src, int64_t en, Real(&v)[N]) {
          if (src == kTraceSlot) {
            trace_row<N>(tb + 1 * S::TS + t * S::TR, v);
          } else {
#pragma unroll
            for (int r = 0; r < N; ++r) v[r] = P.x[en * NNN + r + N * (s ? 0 : N - 1) + NN * t];
          }
        });
      if constexpr (BFLY) {
        exchange_butterfly<N>(t, qx);
        exchange_butterfly<N>(t, py);
      } else {
        exchange_tile<N>(tile, le, t, slot, true, qx);
        exchange_tile<N>(tile, le, t, slot, true, py);
      }
    }

    // ------------------------------------------------------------ layout Y (plane y = t)
    Real out[N][N], qz[N][N];
    [[maybe_unused]] Real qm[N][N];
    {
      // x and y terms first, so their inputs die before u is loaded
      if (adv) {
        kron_apply<N, Real, kSlotTXZ, false, VM>(P, c[2], qx, out);
        kron_apply<N, Real, kSlotTYZ, false, VM>(P, c[2], py, qx);  // qx reused as scratch
        kron_apply<N, Real, kSlotTYX, true, VM>(P, c[0], qx, py);
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
          for (int k = 0; k < N; ++k) out[i][k] += py[i][k];
      } else {
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
          for (int k = 0; k < N; ++k) out[i][k] = Real(0);
      }
      Real u[N][N], pz[N][N];
      load_plane_y<N>(ub, t, active, u);
      kron_apply<N, Real, kSlotDZ, false, VM>(P, c[2], u, pz);
      if (adv) {
        if (P.elem[2]) {
          const Real elz = active ? P.elem[2][e] : Real(1);
#pragma unroll
          for (int i = 0; i < N; ++i)
#pragma unroll
            for (int k = 0; k < N; ++k) pz[i][k] *= elz;
        }
        if (active)
          kron_faces<N, Real, false>(P, 2, c, e, fflags, rec, u, pz, [&](int s, int src, int64_t en, Real(&v)[N]) {
            if (src == kTraceSlot) {
              trace_row<N>(tb + 2 * S::TS + t * S::TR, v);
            } else {
#pragma unroll
              for (int r = 0; r < N; ++r) v[r] = P.x[en * NNN + r + N * t + NN * (s ? 0 : N - 1)];
            }
          });
      } else if (P.elem_mass) {
        const Real em = active ? P.elem_mass[e] : Real(1);
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
          for (int k = 0; k < N; ++k) pz[i][k] *= em;
      }
      kron_apply<N, Real, kSlotTZX, true, VM>(P, c[0], pz, qz);
      if constexpr (SEP) {
        kron_apply<N, Real, kSlotMD, false, VM>(P, c[2], u, pz);
        if (P.elem_mass) {
          const Real em = active ? P.elem_mass[e] : Real(1);
#pragma unroll
          for (int i = 0; i < N; ++i)
#pragma unroll
            for (int k = 0; k < N; ++k) pz[i][k] *= em;
        }
        kron_apply<N, Real, kSlotMX, true, VM>(P, c[0], pz, qm);
      }
    }
    __syncwarp();  // every lane is done reading the staged input of this group
    Real* ob = buf + le * S::SE;  // output staging: the group's DoF slots, staged layout
    if constexpr (BFLY) {
      exchange_butterfly<N>(t, qz);
      exchange_butterfly<N>(t, out);
      if constexpr (SEP) exchange_butterfly<N>(t, qm);
    } else {
      // x and y terms leave in layout Y straight to the output slots; the z term crosses to
      // layout Z through the tile and is added there
      if (slot) {
#pragma unroll
        for (int k = 0; k < N; ++k)
#pragma unroll
          for (int i = 0; i < N; i += S::V) {
            Real v[S::V];
#pragma unroll
            for (int q = 0; q < S::V; ++q) v[q] = out[i + q][k];
            vstore<Real, S::V>(ob + k * S::SP + N * t + i, v);
          }
      }
      exchange_tile<N>(tile, le, t, slot, false, qz);
      if constexpr (SEP) exchange_tile<N>(tile, le, t, slot, false, qm);
    }

    // ------------------------------------------------------------ layout Z, output
    kron_apply<N, Real, kSlotTZY, false, VM>(P, c[1], qz, py);
    if constexpr (SEP) {
      kron_apply<N, Real, kSlotMY, false, VM>(P, c[1], qm, qx);
#pragma unroll
      for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) py[i][j] += qx[i][j];
    }
    if (slot) {
      Real* op = ob + t * S::SP;
#pragma unroll
      for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = 0; i < N; i += S::V) {
          Real v[S::V];
          if constexpr (BFLY) {
#pragma unroll
            for (int q = 0; q < S::V; ++q) v[q] = out[i + q][j] + py[i + q][j];
          } else {
            vload<Real, S::V>(op + N * j + i, v);
#pragma unroll
            for (int q = 0; q < S::V; ++q) v[q] += py[i + q][j];
          }
          vstore<Real, S::V>(op + N * j + i, v);
        }
    }
    __syncwarp();
    {
      // coalesced store, in the staging granule
      const int nchunks = ne * NNN / S::CR;
      Real* dst = P.y + e0 * NNN;
      const Real alpha = P.alpha, by = P.beta_y;
      for (int ch = lane; ch < nchunks; ch += 32) {
        const int d = ch * S::CR;
        const int r = d / NNN, o = d - r * NNN;
        const int z = o / NN, w = o - z * NN;
        Real v[S::CR];
        vload<Real, S::CR>(buf + r * S::SE + z * S::SP + w, v);
        if (by == Real(0)) {
#pragma unroll
          for (int q = 0; q < S::CR; ++q) v[q] = alpha * v[q];
        } else {
          Real o[S::CR];
          vload<Real, S::CR>(dst + d, o);
#pragma unroll
          for (int q = 0; q < S::CR; ++q) v[q] = alpha * v[q] + by * o[q];
        }
        vstore<Real, S::CR>(dst + d, v);
        if constexpr (DOT) {
          Real z[S::CR];
          vldg<Real, S::CR>(P.dot_z + e0 * NNN + d, z);
#pragma unroll
          for (int q = 0; q < S::CR; ++q) dot_acc += (double)v[q] * (double)z[q];
        }
      }
    }
    __syncwarp();  // the buffer is refilled by a later prefetch
  }
  cp_async_wait<0>();
  if constexpr (DOT) {
    // fixed-order sums: lanes (tree), warps (in order), one partial per CTA; entries past the grid
    // are zeroed so a reader sums a fixed count
    __shared__ double wsum[kron_max_warps];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dot_acc += __shfl_down_sync(0xffffffffu, dot_acc, o);
    if (lane == 0) wsum[warp] = dot_acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += wsum[w];
      P.dot_partials[blockIdx.x] = s;
      for (int i = blockIdx.x + gridDim.x; i < P.dot_count; i += gridDim.x) P.dot_partials[i] = 0.0;
    }
  }
}

template <int N, typename Real, bool SEP, int STAGES, bool SHFL, bool DOT = false, uint32_t VM = kVaryRuntime>
__global__ void __launch_bounds__(128) kron3d_kernel(const __grid_constant__ KronParams<Real> P) {
  kron3d_body<N, Real, SEP, STAGES, SHFL, DOT, VM>(P);
}

// The FP64 slot-mask forms without a separate mass term, held to the run-time form's 4 CTAs per
// SM (at most 128 registers; left to itself the compiler takes 138 for kVarySheared).
template <int N, int STAGES, bool SHFL, bool DOT, uint32_t VM>
__global__ void __launch_bounds__(128, 4) kron3d_kernel_capped(const __grid_constant__ KronParams<double> P) {
  kron3d_body<N, double, false, STAGES, SHFL, DOT, VM>(P);
}

}  // namespace dgop
