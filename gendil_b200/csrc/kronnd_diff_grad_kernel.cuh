// Coefficient gradient of the interior-penalty DG diffusion operator (kronnd_diff_kernel.cuh):
//
//   gout[e] = gscale[e] * lam^T (dA/dmu_e) u          (gscale NULL: 1)
//
// A(mu) is linear in the per-element diffusivity.  mu_e enters element e's rows (its cell term
// mu_e Khat, its own face terms and its half of every face's {mu}) and the rows of its face
// neighbours (their {mu grad u . n} average and {mu}).  Summing the two rows of an interior face
// between e (side s along axis a, outward sign nu = -1, +1 for s = 0, 1) and its neighbour nb,
// with value / derivative traces U = l(s)^T u_e, U' = l'(s)^T u_e, L, L' likewise of lam_e and
// U_nb = l(1-s)^T u_nb, L_nb = l(1-s)^T lam_nb on the face, and <p, q> = p^T (x)_{k != a} M_k q,
//
//   detJ/h_a^2 [ <L - L_nb, -nu/2 U' + kappa/2 (U - U_nb)> + <L', sigma nu/2 (U - U_nb)> ],
//
// and on a boundary face with boundary terms detJ/h_a^2 [ <L, -nu U' + kappa U> + <L', sigma nu U> ].
// The cell term is sum_a lam_e^T ((x)_{k != a} M_k (x) Khat_a) u_e.  One thread group per element
// (EB per CTA, as the operator kernel): the cell term by D in-place line passes per axis, each
// face by its traces and D - 1 tangential mass passes over the face arrays, and a fixed-order sum
// of the group's partial products (deterministic).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "kronnd_kernel.cuh"

namespace dgop {

template <int D, int N>
struct KronDiffGradShape {
  static constexpr int ND = kpow(N, D);
  static constexpr int NL = ND / N;  // lines along one axis = DoFs of one face array
  static constexpr int MAT = N * N;
  // per CTA: Khat_a and M_a of every axis, the trace rows l(0), l(1), l'(0), l'(1)
  static constexpr int HDR = (2 * D * MAT + 4 * N + 3) / 4 * 4;
  // per element: U (u_e), L (lam_e), W (work), the face arrays alpha, f, beta, g
  static constexpr int PER_ELEM = 3 * ND + 4 * NL;
};

// out_j = sum_i m(j, i) in_i along the lines of stride INNER of an array of NL_ * N entries
// (in == out allowed: every line is read before it is written).
template <int N, int INNER, int LINES, typename Real>
__device__ __forceinline__ void grad_line_pass(const Real* in, Real* out, const Real* mat, int lt, int tpe) {
  const PassMat<N, Real> m(mat);
  for (int r = lt; r < LINES; r += tpe) {
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
      out[off + j * INNER] = s;
    }
  }
}

template <int D, int N, typename Real>
__global__ void __launch_bounds__(kKronNDThreads) kronnd_diff_grad_kernel(const __grid_constant__ KronDiffParams<Real> P) {
  using S = KronDiffGradShape<D, N>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Real* hdr = reinterpret_cast<Real*>(smem_raw);
  Real* base = hdr + S::HDR;
  __shared__ Real red[kKronNDThreads];
  __shared__ int ecoord[64][kMaxDim];
  if (P.skip && *P.skip) return;
  for (int i = threadIdx.x; i < D * S::MAT; i += blockDim.x) {
    const int a = i / S::MAT, q = i - a * S::MAT;
    hdr[i] = P.mats[(a * kDiffMats + kDK) * S::MAT + q];
    hdr[D * S::MAT + i] = P.mats[(a * kDiffMats + kDM) * S::MAT + q];
  }
  for (int i = threadIdx.x; i < 4 * N; i += blockDim.x) hdr[2 * D * S::MAT + i] = P.mats[D * kDiffMats * S::MAT + i];
  const Real* tv = hdr + 2 * D * S::MAT;  // l(0), l(1), l'(0), l'(1)
  const int EB = P.eb;
  const int tpe = blockDim.x / EB;
  const int b = threadIdx.x / tpe;
  const int lt = threadIdx.x - b * tpe;
  for (int64_t e0 = P.e_begin + (int64_t)blockIdx.x * EB; e0 < P.nelem; e0 += (int64_t)gridDim.x * EB) {
    const int ne = (int)((P.nelem - e0) < EB ? (P.nelem - e0) : EB);
    const bool active = b < ne;
    __syncthreads();
    for (int l = threadIdx.x; l < ne * S::ND; l += blockDim.x) {
      const int bb = l / S::ND, i = l - bb * S::ND;
      Real* el = base + (size_t)bb * S::PER_ELEM;
      el[i] = P.x[e0 * S::ND + l];
      el[S::ND + i] = P.lam[e0 * S::ND + l];
    }
    if (threadIdx.x < ne) {
      const int64_t e = e0 + threadIdx.x;
#pragma unroll
      for (int k = 0; k < D; ++k) ecoord[threadIdx.x][k] = (int)((e / P.estride[k]) % P.sizes[k]);
    }
    __syncthreads();
    Real* el = base + (size_t)(active ? b : 0) * S::PER_ELEM;
    Real* U = el;
    Real* L = el + S::ND;
    Real* W = el + 2 * S::ND;
    Real* fa = el + 3 * S::ND;  // alpha
    Real* ff = fa + S::NL;      // f
    Real* fb = ff + S::NL;      // beta
    Real* fg = fb + S::NL;      // g
    Real part = Real(0);
    // cell: sum_a L . ((x)_{k != a} M_k (x) Khat_a) U
    static_for<0, D>([&](auto ac) {
      constexpr int a = decltype(ac)::value;
      if (active) grad_line_pass<N, kpow(N, a), S::NL>(U, W, hdr + a * S::MAT, lt, tpe);
      __syncthreads();
      static_for<0, D>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        if constexpr (k != a) {
          if (active) grad_line_pass<N, kpow(N, k), S::NL>(W, W, hdr + (D + k) * S::MAT, lt, tpe);
          __syncthreads();
        }
      });
      if (active)
        for (int i = lt; i < S::ND; i += tpe) part += L[i] * W[i];
      __syncthreads();
    });
    // faces
    static_for<0, D>([&](auto ac) {
      constexpr int a = decltype(ac)::value;
      constexpr int INNER = kpow(N, a);
      for (int s = 0; s < 2; ++s) {
        if (active) {
          const int64_t n = P.sizes[a];
          const int64_t ca = ecoord[b][a];
          const bool interior = s == 0 ? (ca > 0 || P.periodic[a]) : (ca + 1 < n || P.periodic[a]);
          const Real nu = s ? Real(1) : Real(-1);
          const Real* bs = tv + s * N;
          const Real* bo = tv + (1 - s) * N;
          const Real* ds = tv + (2 + s) * N;
          const Real* un = P.x;
          const Real* ln = P.lam;
          if (interior) {
            const int64_t cn = s ? (ca + 1 == n ? 0 : ca + 1) : (ca == 0 ? n - 1 : ca - 1);
            const int64_t enb = e0 + b + (cn - ca) * P.estride[a];
            un += enb * S::ND;
            ln += enb * S::ND;
          }
          for (int r = lt; r < S::NL; r += tpe) {
            const int o = r / INNER;
            const int t = r - o * INNER;
            const int off = o * N * INNER + t;
            Real ue = Real(0), ud = Real(0), le = Real(0), ld = Real(0);
#pragma unroll
            for (int i = 0; i < N; ++i) {
              const Real u = U[off + i * INNER], lv = L[off + i * INNER];
              ue += bs[i] * u;
              ud += ds[i] * u;
              le += bs[i] * lv;
              ld += ds[i] * lv;
            }
            Real alpha = Real(0), f = Real(0), beta = Real(0), gg = Real(0);
            if (interior) {
              Real unb = Real(0), lnb = Real(0);
#pragma unroll
              for (int i = 0; i < N; ++i) {
                unb += bo[i] * un[off + i * INNER];
                lnb += bo[i] * ln[off + i * INNER];
              }
              const Real du = ue - unb;
              alpha = le - lnb;
              f = Real(-0.5) * nu * ud + Real(0.5) * P.kappa * du;
              beta = ld;
              gg = Real(0.5) * P.sigma * nu * du;
            } else if (P.boundary) {
              alpha = le;
              f = -nu * ud + P.kappa * ue;
              beta = ld;
              gg = P.sigma * nu * ue;
            }
            fa[r] = alpha;
            ff[r] = f;
            fb[r] = beta;
            fg[r] = gg;
          }
        }
        __syncthreads();
        // tangential mass on f and g: axis k of the face array has stride N^k (k < a) or N^(k-1)
        static_for<0, D>([&](auto kc) {
          constexpr int k = decltype(kc)::value;
          if constexpr (k != a) {
            constexpr int SK = k < a ? kpow(N, k) : kpow(N, k - 1);
            if (active) {
              grad_line_pass<N, SK, S::NL / N>(ff, ff, hdr + (D + k) * S::MAT, lt, tpe);
              grad_line_pass<N, SK, S::NL / N>(fg, fg, hdr + (D + k) * S::MAT, lt, tpe);
            }
            __syncthreads();
          }
        });
        if (active) {
          Real fs = Real(0);
          for (int r = lt; r < S::NL; r += tpe) fs += fa[r] * ff[r] + fb[r] * fg[r];
          part += P.face_h[a] * fs;
        }
        __syncthreads();
      }
    });
    red[threadIdx.x] = part;
    __syncthreads();
    if (active && lt == 0) {
      Real sum = Real(0);
      for (int j = 0; j < tpe; ++j) sum += red[b * tpe + j];
      const int64_t e = e0 + b;
      P.gout[e] = (P.gscale ? P.gscale[e] : Real(1)) * sum;
    }
  }
}

}  // namespace dgop
