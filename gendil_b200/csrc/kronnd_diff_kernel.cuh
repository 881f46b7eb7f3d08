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
// with M_k the reference 1D mass matrix and, on every line of the element along a (values v, the
// neighbour's line z across side s, face rows b_s = l(s), d_s = l'(s), outward sign nu_s = -1, +1,
// f = detJ / h_a^2):
//
//   A_a v + sum_s C_as z = mu_e Khat_a v + f sum_s ( b_s X_s + d_s Y_s )
//   interior side:  X_s = nu_s (-mu_e/2 d_s.v - mu_nb/2 l'(1-s).z) + kappa mubar (b_s.v - l(1-s).z)
//                   Y_s = nu_s sigma mu_e/2 (b_s.v - l(1-s).z)                 mubar = (mu_e + mu_nb)/2
//   boundary side (with boundary terms):  X_s = -nu_s mu_e d_s.v + kappa mu_e b_s.v,
//                                          Y_s = nu_s sigma mu_e b_s.v        (otherwise 0)
//
// Khat_a = detJ / h_a^2 G^T W G (host planner, sipdg.cu).  The face matrices are rank one, so a
// face costs four dot products and two axpys per line instead of N x N matrices.
//
// A CTA holds EB elements (any count up to 64): U, W and Y per element in shared memory, the base
// matrices Khat_a, M_a and the face rows once per CTA.  Every pass runs over the lines of all EB
// elements (one line per thread, flattened), so the CTA's threads stay busy whatever N^(D-1) is.
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
  // per CTA: Khat_a and M_a of every axis, then l(0), l(1), l'(0), l'(1)
  static constexpr int HDR = (2 * D * MAT + 4 * N + 3) / 4 * 4;
  static constexpr int PER_ELEM = 3 * ND;  // U, W, Y
};

// Along axis A over the lines of all ne elements: out_j = sum_i m(j, i) in_i (ACC: out += ...)
template <int D, int N, int A, bool ACC, typename Real>
__device__ __forceinline__ void diff_mass_pass(Real* base, int ne, int in_off, int out_off, const Real* mat) {
  using S = KronDiffShape<D, N>;
  constexpr int INNER = kpow(N, A);
  for (int r = threadIdx.x; r < ne * S::NL; r += blockDim.x) {
    const int b = r / S::NL;
    const int l = r - b * S::NL;
    const int o = l / INNER;
    const int t = l - o * INNER;
    Real* el = base + (size_t)b * S::PER_ELEM;
    const int off = o * N * INNER + t;
    Real v[N];
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = el[in_off + off + i * INNER];
#pragma unroll
    for (int j = 0; j < N; ++j) {
      Real s = mat[j * N] * v[0];
#pragma unroll
      for (int i = 1; i < N; ++i) s += mat[j * N + i] * v[i];
      if (ACC) el[out_off + off + j * INNER] += s;
      else el[out_off + off + j * INNER] = s;
    }
  }
}

// W <- A_a U + sum_s C_as u_nb along axis A, over the lines of all ne elements.
template <int D, int N, int A, typename Real>
__device__ __forceinline__ void diff_axis_pass(const KronDiffParams<Real>& P, Real* base, int ne, int64_t e0,
                                               const Real* kh, const Real* tv, const int (*ecoord)[kMaxDim],
                                               const Real (*emu)[2 * kMaxDim + 1]) {
  using S = KronDiffShape<D, N>;
  constexpr int INNER = kpow(N, A);
  const Real f = P.face_h[A];
  const int64_t n = P.sizes[A];
  const bool per = P.periodic[A] != 0;
  for (int r = threadIdx.x; r < ne * S::NL; r += blockDim.x) {
    const int b = r / S::NL;
    const int l = r - b * S::NL;
    const int o = l / INNER;
    const int t = l - o * INNER;
    Real* el = base + (size_t)b * S::PER_ELEM;
    const int off = o * N * INNER + t;
    Real v[N];
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = el[off + i * INNER];
    const Real mue = emu[b][0];
    const int64_t ca = ecoord[b][A];
    Real X[2], Y[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const Real* bs = tv + s * N;
      const Real* ds = tv + (2 + s) * N;
      Real tb = bs[0] * v[0], td = ds[0] * v[0];
#pragma unroll
      for (int i = 1; i < N; ++i) {
        tb += bs[i] * v[i];
        td += ds[i] * v[i];
      }
      const Real nu = s ? Real(1) : Real(-1);
      const bool interior = s == 0 ? (ca > 0 || per) : (ca + 1 < n || per);
      if (interior) {
        const int64_t cn = s ? (ca + 1 == n ? 0 : ca + 1) : (ca == 0 ? n - 1 : ca - 1);
        const Real* z = P.x + (e0 + b + (cn - ca) * P.estride[A]) * S::ND + off;
        const Real* bo = tv + (1 - s) * N;
        const Real* dn = tv + (3 - s) * N;
        Real nb = Real(0), nd = Real(0);
#pragma unroll
        for (int i = 0; i < N; ++i) {
          const Real zi = z[i * INNER];
          nb += bo[i] * zi;
          nd += dn[i] * zi;
        }
        const Real mun = emu[b][1 + 2 * A + s];
        const Real jump = tb - nb;
        X[s] = nu * (Real(-0.5) * mue * td - Real(0.5) * mun * nd) + P.kappa * Real(0.5) * (mue + mun) * jump;
        Y[s] = nu * P.sigma * Real(0.5) * mue * jump;
      } else if (P.boundary) {
        X[s] = -nu * mue * td + P.kappa * mue * tb;
        Y[s] = nu * P.sigma * mue * tb;
      } else {
        X[s] = Real(0);
        Y[s] = Real(0);
      }
      X[s] *= f;
      Y[s] *= f;
    }
#pragma unroll
    for (int j = 0; j < N; ++j) {
      Real s = kh[j * N] * v[0];
#pragma unroll
      for (int i = 1; i < N; ++i) s += kh[j * N + i] * v[i];
      s *= mue;
      s += tv[j] * X[0] + tv[N + j] * X[1] + tv[2 * N + j] * Y[0] + tv[3 * N + j] * Y[1];
      el[S::ND + off + j * INNER] = s;
    }
  }
}

template <int D, int N, typename Real>
__global__ void __launch_bounds__(kKronNDThreads) kronnd_diff_kernel(const __grid_constant__ KronDiffParams<Real> P) {
  using S = KronDiffShape<D, N>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Real* hdr = reinterpret_cast<Real*>(smem_raw);
  Real* base = hdr + S::HDR;
  __shared__ int ecoord[kDiffMaxEB][kMaxDim];
  __shared__ Real emu[kDiffMaxEB][2 * kMaxDim + 1];
  if (P.skip && *P.skip) return;
  for (int i = threadIdx.x; i < D * S::MAT; i += blockDim.x) {
    const int a = i / S::MAT, q = i - a * S::MAT;
    hdr[i] = P.mats[(a * kDiffMats + kDK) * S::MAT + q];
    hdr[D * S::MAT + i] = P.mats[(a * kDiffMats + kDM) * S::MAT + q];
  }
  for (int i = threadIdx.x; i < 4 * N; i += blockDim.x) hdr[2 * D * S::MAT + i] = P.mats[D * kDiffMats * S::MAT + i];
  const Real* tv = hdr + 2 * D * S::MAT;
  const int EB = P.eb;
  for (int64_t e0 = P.e_begin + (int64_t)blockIdx.x * EB; e0 < P.nelem; e0 += (int64_t)gridDim.x * EB) {
    const int ne = (int)((P.nelem - e0) < EB ? (P.nelem - e0) : EB);
    __syncthreads();
    for (int l = threadIdx.x; l < ne * S::ND; l += blockDim.x) {
      const int b = l / S::ND, i = l - b * S::ND;
      base[(size_t)b * S::PER_ELEM + i] = P.x[e0 * S::ND + l];
    }
    if (threadIdx.x < ne) {
      const int b = threadIdx.x;
      const int64_t e = e0 + b;
      emu[b][0] = P.mu[e];
#pragma unroll
      for (int k = 0; k < D; ++k) {
        const int64_t n = P.sizes[k];
        const int64_t ck = (e / P.estride[k]) % n;
        ecoord[b][k] = (int)ck;
#pragma unroll
        for (int s = 0; s < 2; ++s) {
          const bool interior = s == 0 ? (ck > 0 || P.periodic[k]) : (ck + 1 < n || P.periodic[k]);
          const int64_t cn = s ? (ck + 1 == n ? 0 : ck + 1) : (ck == 0 ? n - 1 : ck - 1);
          emu[b][1 + 2 * k + s] = interior ? P.mu[e + (cn - ck) * P.estride[k]] : Real(0);
        }
      }
    }
    __syncthreads();
    static_for<0, D>([&](auto ac) {
      constexpr int a = decltype(ac)::value;
      diff_axis_pass<D, N, a>(P, base, ne, e0, hdr + a * S::MAT, tv, ecoord, emu);
      __syncthreads();
      if constexpr (D == 1) {
        for (int l = threadIdx.x; l < ne * S::ND; l += blockDim.x) {
          const int b = l / S::ND, i = l - b * S::ND;
          base[(size_t)b * S::PER_ELEM + 2 * S::ND + i] = base[(size_t)b * S::PER_ELEM + S::ND + i];
        }
        __syncthreads();
      } else {
        constexpr int lastk = (a == D - 1) ? D - 2 : D - 1;
        static_for<0, D>([&](auto kc) {
          constexpr int k = decltype(kc)::value;
          if constexpr (k != a) {
            if constexpr (k == lastk) {
              // the first axis writes Y, the others accumulate into it
              diff_mass_pass<D, N, k, (a > 0)>(base, ne, S::ND, 2 * S::ND, hdr + (D + k) * S::MAT);
            } else {
              diff_mass_pass<D, N, k, false>(base, ne, S::ND, S::ND, hdr + (D + k) * S::MAT);
            }
            __syncthreads();
          }
        });
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
