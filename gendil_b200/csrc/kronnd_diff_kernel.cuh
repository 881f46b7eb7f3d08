// Interior-penalty DG diffusion (SIPDG / NIPG / IIPG) in Kronecker form, any dimension, shared
// memory.  The reference's generic weak form (README "Weak Form DSL"; the interior-facet terms of
// tests/integration/gendil/test-sipdg-coefficient-field-inputs.cpp:560-569)
//
//   integrate(cells, mu grad u . grad v)
//   + integrate(interior_facets, -{mu grad u . n}[v] + sigma [u]{mu grad v . n} + tau {mu}[u][v])
//   + integrate(boundary_facets, -mu grad u . n v + sigma u mu grad v . n + tau mu u v)   (optional)
//
// with mu constant on each element and tau = kappa / h_a (InverseFacetSize), evaluated element by
// element (jump(v) and average(grad v) keep only the element's own test functions), becomes on a
// Cartesian mesh, for each axis a,
//
//   y_e += (x)_{k != a} M_k [ A_a(e) u_e + sum_{interior s} C_as(e) u_{nb(a,s)} ]
//
// A_a(e) = mu_e Khat_a + sum_s (c1 P1_s + c2 P2_s + c3 P3_s)      (own lines along a)
// C_as(e) = -mu_nb/2 Q1_s - sigma mu_e/2 Q2_s - mubar_s Q3_s       (the neighbour's lines)
//
// Khat_a = detJ / h_a^2 G^T W G; with the face value and derivative rows b_s = l(s), d_s = l'(s)
// and nu = -1, +1 the outward sign:  P1_s = detJ/h_a nu/h_a b_s d_s^T, P2_s = detJ/h_a nu/h_a
// d_s b_s^T, P3_s = detJ/h_a kappa/h_a b_s b_s^T, Q1_s = detJ/h_a nu/h_a b_s d_{1-s}^T,
// Q2_s = detJ/h_a nu/h_a d_s b_{1-s}^T, Q3_s = detJ/h_a kappa/h_a b_s b_{1-s}^T (host planner,
// sipdg.cu).  Interior face: c1 = -mu_e/2, c2 = sigma mu_e/2, c3 = mubar_s = (mu_e + mu_nb)/2;
// boundary face with boundary terms: c1 = -mu_e, c2 = sigma mu_e, c3 = mu_e; else 0.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "kronnd_kernel.cuh"

namespace dgop {



template <int D, int N>
struct KronDiffShape {
  static constexpr int ND = kpow(N, D);
  static constexpr int NL = ND / N;
  static constexpr int MAT = N * N;
  // per element matrix slots: A_a (D), C_a0 (D), C_a1 (D), M_a (D)
  static constexpr int NS = 4 * D;
  static constexpr int MUS = 2 * D + 2;  // mu_e, the 2D neighbours' mu, pad
  static constexpr int PER_ELEM = 3 * ND + NS * MAT + MUS;
  static constexpr int slot_A(int a) { return a; }
  static constexpr int slot_C(int a, int s) { return D + 2 * a + s; }
  static constexpr int slot_M(int a) { return 3 * D + a; }
};

// In-place pass along axis A with the element's slot matrix (see nd_pass; same layout as
// KronNDShape with U at 0, W at ND, Y at 2 ND and the slots at 3 ND).
template <int D, int N, int A, bool FIRST, bool ACC, typename Real>
__device__ __forceinline__ void diff_pass(Real* base, int ne, int eb, int slot) {
  using S = KronDiffShape<D, N>;
  constexpr int INNER = kpow(N, A);
  const int tpe = blockDim.x / eb;
  const int b = threadIdx.x / tpe;
  if (b >= ne) return;
  Real* el = base + (size_t)b * S::PER_ELEM;
  const Real* in = FIRST ? el : el + S::ND;
  Real* out = ACC ? el + 2 * S::ND : el + S::ND;
  const PassMat<N, Real> m(el + 3 * S::ND + slot * S::MAT);
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
      else out[off + j * INNER] = s;
    }
  }
}

// W_line += C_as u_nb,line for the lines along A of every element, both sides (interior only).
template <int D, int N, int A, typename Real>
__device__ __forceinline__ void diff_neighbours(const KronDiffParams<Real>& P, const Real* __restrict__ xin,
                                                Real* base, int ne, int eb, int64_t e0,
                                                const int (*ecoord)[kMaxDim]) {
  using S = KronDiffShape<D, N>;
  constexpr int INNER = kpow(N, A);
  const int tpe = blockDim.x / eb;
  const int b = threadIdx.x / tpe;
  if (b >= ne) return;
  Real* el = base + (size_t)b * S::PER_ELEM;
  const int64_t e = e0 + b;
  const int64_t n = P.sizes[A];
  const int64_t ca = ecoord[b][A];
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const bool interior = s == 0 ? (ca > 0 || P.periodic[A]) : (ca + 1 < n || P.periodic[A]);
    if (!interior) continue;
    const int64_t cn = s ? (ca + 1 == n ? 0 : ca + 1) : (ca == 0 ? n - 1 : ca - 1);
    const Real* un = xin + (e + (cn - ca) * P.estride[A]) * S::ND;
    const PassMat<N, Real> m(el + 3 * S::ND + S::slot_C(A, s) * S::MAT);
    for (int r = threadIdx.x - b * tpe; r < S::NL; r += tpe) {
      const int o = r / INNER;
      const int t = r - o * INNER;
      const int off = o * N * INNER + t;
      Real v[N];
#pragma unroll
      for (int i = 0; i < N; ++i) v[i] = un[off + i * INNER];
#pragma unroll
      for (int j = 0; j < N; ++j) {
        Real sum = m(j, 0) * v[0];
#pragma unroll
        for (int i = 1; i < N; ++i) sum += m(j, i) * v[i];
        el[S::ND + off + j * INNER] += sum;
      }
    }
  }
}

template <int D, int N, typename Real>
__global__ void __launch_bounds__(kKronNDThreads) kronnd_diff_kernel(const __grid_constant__ KronDiffParams<Real> P) {
  using S = KronDiffShape<D, N>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Real* base = reinterpret_cast<Real*>(smem_raw);
  __shared__ int ecoord[64][kMaxDim];
  if (P.skip && *P.skip) return;
  const int EB = P.eb;
  for (int64_t e0 = P.e_begin + (int64_t)blockIdx.x * EB; e0 < P.nelem; e0 += (int64_t)gridDim.x * EB) {
    const int ne = (int)((P.nelem - e0) < EB ? (P.nelem - e0) : EB);
    __syncthreads();
    for (int l = threadIdx.x; l < ne * S::ND; l += blockDim.x) {
      const int b = l / S::ND, i = l - b * S::ND;
      Real* el = base + (size_t)b * S::PER_ELEM;
      el[i] = P.x[e0 * S::ND + l];
      el[2 * S::ND + i] = Real(0);
    }
    if (threadIdx.x < ne) {
      const int b = threadIdx.x;
      const int64_t e = e0 + b;
      Real* mus = base + (size_t)b * S::PER_ELEM + 3 * S::ND + S::NS * S::MAT;
      mus[0] = P.mu[e];
#pragma unroll
      for (int k = 0; k < D; ++k) {
        const int64_t ck = (e / P.estride[k]) % P.sizes[k];
        ecoord[b][k] = (int)ck;
        const int64_t n = P.sizes[k];
#pragma unroll
        for (int s = 0; s < 2; ++s) {
          const bool interior = s == 0 ? (ck > 0 || P.periodic[k]) : (ck + 1 < n || P.periodic[k]);
          const int64_t cn = s ? (ck + 1 == n ? 0 : ck + 1) : (ck == 0 ? n - 1 : ck - 1);
          mus[1 + 2 * k + s] = interior ? P.mu[e + (cn - ck) * P.estride[k]] : Real(0);
        }
      }
    }
    __syncthreads();
    // per element matrices: A_a, C_a0, C_a1 from the base matrices and the element's mu values
    for (int l = threadIdx.x; l < ne * S::NS * S::MAT; l += blockDim.x) {
      const int b = l / (S::NS * S::MAT);
      const int r = l - b * (S::NS * S::MAT);
      const int sl = r / S::MAT, q = r - sl * S::MAT;
      Real* el = base + (size_t)b * S::PER_ELEM;
      const Real* mus = el + 3 * S::ND + S::NS * S::MAT;
      const Real mue = mus[0];
      const int a = sl < D ? sl : (sl < 3 * D ? (sl - D) / 2 : sl - 3 * D);
      const Real* bm = P.mats + (size_t)a * kDiffMats * S::MAT + q;
      Real v;
      if (sl >= 3 * D) {
        v = bm[kDM * S::MAT];
      } else {
        const int64_t n = P.sizes[a];
        const int64_t ca = ecoord[b][a];
        if (sl < D) {
          v = mue * bm[kDK * S::MAT];
#pragma unroll
          for (int s = 0; s < 2; ++s) {
            const bool interior = s == 0 ? (ca > 0 || P.periodic[a]) : (ca + 1 < n || P.periodic[a]);
            Real c1 = Real(0), c2 = Real(0), c3 = Real(0);
            if (interior) {
              c1 = Real(-0.5) * mue;
              c2 = P.sigma * Real(0.5) * mue;
              c3 = Real(0.5) * (mue + mus[1 + 2 * a + s]);
            } else if (P.boundary) {
              c1 = -mue;
              c2 = P.sigma * mue;
              c3 = mue;
            }
            v += c1 * bm[(kDP1 + s) * S::MAT] + c2 * bm[(kDP2 + s) * S::MAT] + c3 * bm[(kDP3 + s) * S::MAT];
          }
        } else {
          const int s = (sl - D) & 1;
          const bool interior = s == 0 ? (ca > 0 || P.periodic[a]) : (ca + 1 < n || P.periodic[a]);
          v = Real(0);
          if (interior) {
            const Real mun = mus[1 + 2 * a + s];
            v = Real(-0.5) * mun * bm[(kDQ1 + s) * S::MAT] - P.sigma * Real(0.5) * mue * bm[(kDQ2 + s) * S::MAT] -
                Real(0.5) * (mue + mun) * bm[(kDQ3 + s) * S::MAT];
          }
        }
      }
      el[3 * S::ND + r] = v;
    }
    __syncthreads();
    static_for<0, D>([&](auto ac) {
      constexpr int a = decltype(ac)::value;
      diff_pass<D, N, a, true, false>(base, ne, EB, S::slot_A(a));
      __syncthreads();
      diff_neighbours<D, N, a>(P, P.x, base, ne, EB, e0, ecoord);
      __syncthreads();
      static_for<0, D>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        if constexpr (k != a) {
          constexpr int lastk = (a == D - 1) ? D - 2 : D - 1;
          diff_pass<D, N, k, false, k == lastk>(base, ne, EB, S::slot_M(k));
          __syncthreads();
        }
      });
      if constexpr (D == 1) {
        for (int l = threadIdx.x; l < ne * S::ND; l += blockDim.x) {
          const int b = l / S::ND, i = l - b * S::ND;
          Real* el = base + (size_t)b * S::PER_ELEM;
          el[2 * S::ND + i] += el[S::ND + i];
        }
        __syncthreads();
      }
    });
    for (int l = threadIdx.x; l < ne * S::ND; l += blockDim.x) {
      const int b = l / S::ND, i = l - b * S::ND;
      const Real v = base[(size_t)b * S::PER_ELEM + 2 * S::ND + i];
      Real* dst = P.y + e0 * S::ND + l;
      *dst = (P.beta_y == Real(0)) ? P.alpha * v : P.alpha * v + P.beta_y * *dst;
    }
  }
}

}  // namespace dgop
