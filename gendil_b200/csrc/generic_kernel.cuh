// Generic sum-factorized DG element kernel: mass, upwind advection (cell + interior/boundary
// faces), their sum, and the transposed operator, for any dimension D <= 6, N = p + 1 <= 8 and
// Q <= 8 Gauss points.  This is the coverage path: every (D, N, Q) runs here with the
// reference's own algorithm (advectionoperator.hpp:269-441, massoperator.hpp:39-89):
//
//   u = x[e] ; Bu = (B x ... x B) u                        -- D 1D contraction passes
//   q-function at every quadrature point                   -- coefficients from 1D tables
//   sum_i Dq_i^T (collocated gradient), then B^T            -- D + D passes
//   for each axis, both faces: own trace + neighbour trace (GLL: exact face selection),
//   tangential B, upwind flux, tangential B^T, add into the element result
//   y[e] = alpha * result + beta_y * y[e]
//
// A CTA processes `eb` elements at a time; every contraction pass is one sweep of "lines"
// (1D fibres) over all of them, one line per thread, between __syncthreads().  Element work
// buffers live in shared memory, or in a per-CTA global workspace when an element is too large.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "dgop_params.h"

namespace dgop {

__host__ __device__ constexpr int ipow(int b, int e) {
  int r = 1;
  for (int i = 0; i < e; ++i) r *= b;
  return r;
}

template <int I, int E, typename F>
__host__ __device__ __forceinline__ void static_for(F&& f) {
  if constexpr (I < E) {
    f(std::integral_constant<int, I>{});
    static_for<I + 1, E>(f);
  }
}

// m(j, i) = a[j * LD + i]
template <typename Real, int LD>
struct RowMat {
  const Real* a;
  __device__ __forceinline__ Real operator()(int j, int i) const { return a[j * LD + i]; }
};
// m(j, i) = a[i * LD + j]
template <typename Real, int LD>
struct ColMat {
  const Real* a;
  __device__ __forceinline__ Real operator()(int j, int i) const { return a[i * LD + j]; }
};

// out[b][o][j][t] (+)= sum_i m(j, i) in[b][o][i][t] over `nbatch` tensors, t < INNER, o < OUTER.
template <int NIN, int NOUT, int INNER, int OUTER, bool ADD, typename Real, typename Mat>
__device__ __forceinline__ void contract_pass(const Mat& m, const Real* in, int sin, Real* out, int sout, int nbatch) {
  constexpr int LINES = INNER * OUTER;
  const int total = nbatch * LINES;
  for (int l = threadIdx.x; l < total; l += blockDim.x) {
    const int b = l / LINES;
    const int r = l - b * LINES;
    const int o = r / INNER;
    const int t = r - o * INNER;
    const Real* src = in + (int64_t)b * sin + o * NIN * INNER + t;
    Real v[NIN];
#pragma unroll
    for (int i = 0; i < NIN; ++i) v[i] = src[i * INNER];
    Real* dst = out + (int64_t)b * sout + o * NOUT * INNER + t;
#pragma unroll
    for (int j = 0; j < NOUT; ++j) {
      Real s = Real(0);
#pragma unroll
      for (int i = 0; i < NIN; ++i) s += m(j, i) * v[i];
      if constexpr (ADD) dst[j * INNER] += s;
      else dst[j * INNER] = s;
    }
  }
}

// c(X) at a point whose per-axis table index is j[k] (see CoefDev).
template <int D, typename Real>
__device__ __forceinline__ Real coef_eval(const CoefDev<Real>& c, const Real* __restrict__ tab, int ld,
                                          const int* eidx, const int* j, int64_t e) {
  Real v = c.constant;
  for (int t = 0; t < c.nterms; ++t) {
    Real p = Real(1);
    bool first = true;
#pragma unroll
    for (int k = 0; k < D; ++k) {
      const int64_t off = c.off[t][k];
      if (off >= 0) {
        const Real f = tab[off + (int64_t)eidx[k] * ld + j[k]];
        p = first ? f : p * f;
        first = false;
      }
    }
    v += p;
  }
  if (c.elem) v *= c.elem[e];
  return v;
}

template <int D, int N, int Q>
struct GenericShape {
  static constexpr int M = N > Q ? N : Q;
  static constexpr int ND = ipow(N, D), QD = ipow(Q, D), MD = ipow(M, D);
  static constexpr int NF = ipow(N, D - 1), QF = ipow(Q, D - 1), MF = ipow(M, D - 1);
  static constexpr int CELLR = 2 * MD + (D + 2) * QD;  // w1, w2, Bu, D components, accumulator
  static constexpr int FACER = 8 * MF;                  // 2 sides x (own, neighbour) x ping-pong
  static constexpr int REG = CELLR > FACER ? CELLR : FACER;
  static constexpr int PER_ELEM = 2 * ND + REG;         // u, y, region
  static constexpr int MATS = (Q * N + Q * Q + 2 * N + Q + 1) & ~1;
};

// Shared memory bytes for the fixed part (tables + indices) and per element.
template <int D, int N, int Q, typename Real>
__host__ __device__ constexpr int generic_fixed_bytes(int eb) {
  return GenericShape<D, N, Q>::MATS * (int)sizeof(Real) + ((eb * D + 1) & ~1) * 4 + eb * 2 * D * 8;
}

template <int D, int N, int Q, typename Real>
__global__ void __launch_bounds__(256) generic_kernel(const __grid_constant__ OpParams<Real> P) {
  using S = GenericShape<D, N, Q>;
  constexpr int ND = S::ND, QD = S::QD, MD = S::MD, NF = S::NF, QF = S::QF, MF = S::MF;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (P.skip && *P.skip) return;  // a finished solve: nothing to do
  const int EB = P.eb;
  Real* sB = reinterpret_cast<Real*>(smem_raw);
  Real* sDq = sB + Q * N;
  Real* sBf = sDq + Q * Q;
  Real* sW = sBf + 2 * N;
  int* sidx = reinterpret_cast<int*>(sB + S::MATS);
  int64_t* snb = reinterpret_cast<int64_t*>(sidx + ((EB * D + 1) & ~1));
  Real* work = P.scratch ? P.scratch + (int64_t)blockIdx.x * P.scratch_per_cta
                         : reinterpret_cast<Real*>(snb + EB * 2 * D);
  Real* su = work;
  Real* sy = su + (int64_t)EB * ND;
  Real* reg = sy + (int64_t)EB * ND;
  // cell-phase views of the region
  Real* w1 = reg;
  Real* w2 = w1 + (int64_t)EB * MD;
  Real* sq = w2 + (int64_t)EB * MD;
  Real* comp = sq + (int64_t)EB * QD;           // D x EB x QD
  Real* sacc = comp + (int64_t)D * EB * QD;
  // face-phase view: F[s][t][buf] blocks of EB x MF, s = side, t = own/neighbour
  auto F = [&](int s, int t, int buf) { return reg + (int64_t)((s * 2 + t) * 2 + buf) * EB * MF; };

  const int tid = threadIdx.x, nth = blockDim.x;
  for (int i = tid; i < Q * N; i += nth) sB[i] = P.B[i];
  for (int i = tid; i < Q * Q; i += nth) sDq[i] = P.Dq[i];
  for (int i = tid; i < 2 * N; i += nth) sBf[i] = P.Bf[i / N][i % N];
  for (int i = tid; i < Q; i += nth) sW[i] = P.wq[i];

  const bool transpose = (P.flags & kTranspose) != 0;
  const bool do_mass = (P.flags & kMass) != 0;
  const bool do_adv = (P.flags & kAdvCell) != 0;
  const bool do_fint = (P.flags & kFaceInt) != 0;
  const bool do_fbnd = (P.flags & kFaceBnd) != 0;
  const Real detJ = P.detJ;
  const bool GLL = P.gll != 0;

  for (int64_t e0 = P.e_begin + (int64_t)blockIdx.x * EB; e0 < P.nelem; e0 += (int64_t)gridDim.x * EB) {
    const int ne = (int)((P.nelem - e0) < EB ? (P.nelem - e0) : EB);
    __syncthreads();
    // element coordinates and neighbours (cartesianndmesh.hpp:95-198)
    for (int l = tid; l < ne * D; l += nth) {
      const int b = l / D, k = l - b * D;
      sidx[l] = (int)(((e0 + b) / P.estride[k]) % P.sizes[k]);
    }
    for (int l = tid; l < ne * 2 * D; l += nth) {
      const int b = l / (2 * D), f = l - b * 2 * D;
      const int a = f % D;
      const int64_t e = e0 + b;
      const int64_t ia = (e / P.estride[a]) % P.sizes[a];
      const int64_t n = P.sizes[a];
      int64_t nb;
      if (f < D) {
        if (ia > 0) nb = e - P.estride[a];
        else nb = P.periodic[a] ? e + (n - 1) * P.estride[a] : -1;
      } else {
        if (ia < n - 1) nb = e + P.estride[a];
        else nb = P.periodic[a] ? e - (n - 1) * P.estride[a] : -1;
      }
      snb[l] = nb;
    }
    // own DoFs: one contiguous chunk of ne * N^D values
    {
      const Real* xs = P.x + e0 * ND;
      for (int i = tid; i < ne * ND; i += nth) su[i] = xs[i];
    }
    __syncthreads();

    // ------------------------------------------------------------------ cell terms
    if (do_mass || do_adv) {
      // interpolation B along axes 0..D-1: su -> w1/w2 -> sq
      static_for<0, D>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        const Real* src = (k == 0) ? su : ((k & 1) ? w1 : w2);
        const int ss = (k == 0) ? ND : MD;
        Real* dst = (k == D - 1) ? sq : ((k & 1) ? w2 : w1);
        const int ds = (k == D - 1) ? QD : MD;
        contract_pass<N, Q, ipow(Q, k), ipow(N, D - 1 - k), false>(RowMat<Real, N>{sB}, src, ss, dst, ds, ne);
        __syncthreads();
      });
      if (transpose && do_adv) {
        // gradient at the quadrature points along each axis: comp[i] = Dq_i Bu
        static_for<0, D>([&](auto ic) {
          constexpr int i = decltype(ic)::value;
          contract_pass<Q, Q, ipow(Q, i), ipow(Q, D - 1 - i), false>(RowMat<Real, Q>{sDq}, sq, QD,
                                                                      comp + (int64_t)i * EB * QD, QD, ne);
        });
        __syncthreads();
      }
      // q-function
      for (int l = tid; l < ne * QD; l += nth) {
        const int b = l / QD, qi = l - b * QD;
        int j[D];
        int r = qi;
        Real weight = Real(1);
#pragma unroll
        for (int k = 0; k < D; ++k) {
          j[k] = r % Q;
          r /= Q;
          weight = (k == 0) ? sW[j[k]] : weight * sW[j[k]];
        }
        const int* eidx = sidx + b * D;
        const int64_t e = e0 + b;
        const Real bu = sq[l];
        Real acc = Real(0);
        if (do_mass) {
          const Real sig = coef_eval<D>(P.sigma, P.tab, P.tab_ld, eidx, j, e);
          acc = do_adv ? weight * detJ * (sig * bu) : weight * detJ * sig * bu;
        }
        if (do_adv) {
          const Real wv = -weight * detJ;
          if (!transpose) {
            const Real w = wv * bu;
#pragma unroll
            for (int i = 0; i < D; ++i) {
              const Real bi = coef_eval<D>(P.beta[i], P.tab, P.tab_ld, eidx, j, e);
              comp[(int64_t)i * EB * QD + l] = w * (bi * P.invh[i]);
            }
          } else {
            Real s = Real(0);
#pragma unroll
            for (int i = 0; i < D; ++i) {
              const Real bi = coef_eval<D>(P.beta[i], P.tab, P.tab_ld, eidx, j, e);
              s += wv * (bi * P.invh[i]) * comp[(int64_t)i * EB * QD + l];
            }
            acc += s;
          }
        }
        sacc[l] = (do_adv && !transpose) ? Real(0) : acc;
        if (do_adv && !transpose && do_mass) w1[l] = acc;  // mass term added after G^T
      }
      __syncthreads();
      if (do_adv && !transpose) {
        // collocated G^T at quadrature points (applygradienttestfunctionsthreaded.hpp:164-261)
        static_for<0, D>([&](auto ic) {
          constexpr int i = decltype(ic)::value;
          contract_pass<Q, Q, ipow(Q, i), ipow(Q, D - 1 - i), true>(ColMat<Real, Q>{sDq}, comp + (int64_t)i * EB * QD,
                                                                    QD, sacc, QD, ne);
          __syncthreads();
        });
        if (do_mass) {
          for (int l = tid; l < ne * QD; l += nth) sacc[l] += w1[l];
          __syncthreads();
        }
      }
      // B^T along axes 0..D-1: sacc -> w1/w2 -> sy
      static_for<0, D>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        const Real* src = (k == 0) ? sacc : ((k & 1) ? w1 : w2);
        const int ss = (k == 0) ? QD : MD;
        Real* dst = (k == D - 1) ? sy : ((k & 1) ? w2 : w1);
        const int ds = (k == D - 1) ? ND : MD;
        contract_pass<Q, N, ipow(N, k), ipow(Q, D - 1 - k), false>(ColMat<Real, N>{sB}, src, ss, dst, ds, ne);
        __syncthreads();
      });
    } else {
      for (int i = tid; i < ne * ND; i += nth) sy[i] = Real(0);
      __syncthreads();
    }

    // ------------------------------------------------------------------ faces
    if (do_fint || do_fbnd) {
      static_for<0, D>([&](auto ac) {
        constexpr int a = decltype(ac)::value;
        constexpr int SA = ipow(N, a);  // element stride of axis a
        // traces: own (both sides) and neighbour (interior sides)
        for (int l = tid; l < ne * 2 * NF; l += nth) {
          const int b = l / (2 * NF);
          const int r = l - b * 2 * NF;
          const int s = r / NF;
          const int f = r - s * NF;
          const int base = (f % SA) + (f / SA) * SA * N;  // element index with i_a = 0
          const Real* ue = su + (int64_t)b * ND;
          Real own, nbv = Real(0);
          const int64_t nb = snb[b * 2 * D + a + s * D];
          if (GLL) {
            own = ue[base + (s ? N - 1 : 0) * SA];
            if (nb >= 0) nbv = P.x[nb * ND + base + (s ? 0 : N - 1) * SA];
          } else {
            own = Real(0);
#pragma unroll
            for (int i = 0; i < N; ++i) own += sBf[s * N + i] * ue[base + i * SA];
            if (nb >= 0) {
              const Real* un = P.x + nb * ND;
#pragma unroll
              for (int i = 0; i < N; ++i) nbv += sBf[(1 - s) * N + i] * un[base + i * SA];
            }
          }
          F(s, 0, 0)[(int64_t)b * MF + f] = own;
          F(s, 1, 0)[(int64_t)b * MF + f] = nbv;
        }
        __syncthreads();
        // tangential interpolation (D-1 passes) on 4 * ne face tensors, buffers alternate 0/1.
        // F(s,t,buf) blocks are laid out so that (s,t) tensors of the same buf are EB*MF*2 apart.
        static_for<0, D - 1>([&](auto mc) {
          constexpr int m = decltype(mc)::value;
          const int bin = m & 1, bout = bin ^ 1;
#pragma unroll
          for (int st = 0; st < 4; ++st) {
            const int s = st >> 1, t = st & 1;
            contract_pass<N, Q, ipow(Q, m), ipow(N, D - 2 - m), false>(RowMat<Real, N>{sB}, F(s, t, bin), MF,
                                                                      F(s, t, bout), MF, ne);
          }
          __syncthreads();
        });
        constexpr int FB = (D - 1) & 1;  // buffer holding the interpolated traces
        // upwind flux at the face quadrature points
        for (int l = tid; l < ne * 2 * QF; l += nth) {
          const int b = l / (2 * QF);
          const int r = l - b * 2 * QF;
          const int s = r / QF;
          const int fq = r - s * QF;
          const int64_t e = e0 + b;
          const int64_t nb = snb[b * 2 * D + a + s * D];
          const bool interior = nb >= 0;
          Real* own_p = F(s, 0, FB) + (int64_t)b * MF + fq;
          const bool active = interior ? do_fint : do_fbnd;
          if (!active) {
            *own_p = Real(0);
            continue;
          }
          int j[D];
          int rr = fq;
          Real weight = Real(1);
          bool firstw = true;
#pragma unroll
          for (int k = 0; k < D; ++k) {
            if (k == a) {
              j[k] = Q + s;
              continue;
            }
            j[k] = rr % Q;
            rr /= Q;
            weight = firstw ? sW[j[k]] : weight * sW[j[k]];
            firstw = false;
          }
          const Real ba = coef_eval<D>(P.beta[a], P.tab, P.tab_ld, sidx + b * D, j, e);
          const Real nrm = s ? P.invh[a] : -P.invh[a];
          const Real dot = ba * nrm;
          const Real own = *own_p;
          const Real other = interior ? F(s, 1, FB)[(int64_t)b * MF + fq] : P.g;
          Real up;
          if (!transpose) {
            up = (dot > Real(0)) ? dot * own : dot * other;
          } else {
            // row e of A^T on this face: e's own outflow term, plus the neighbour's inflow term
            // when the neighbour takes e's trace, with the neighbour's velocity (its own
            // coefficient and per-element factor; equal to -dot for a continuous field)
            up = (dot > Real(0)) ? dot * own : Real(0);
            if (interior) {
              int cn[D], jn[D];
#pragma unroll
              for (int k = 0; k < D; ++k) {
                cn[k] = sidx[b * D + k];
                jn[k] = j[k];
              }
              const int na = (int)P.sizes[a];
              cn[a] = s ? (cn[a] + 1 == na ? 0 : cn[a] + 1) : (cn[a] == 0 ? na - 1 : cn[a] - 1);
              jn[a] = Q + 1 - s;
              const Real dot_nb = -coef_eval<D>(P.beta[a], P.tab, P.tab_ld, cn, jn, nb) * nrm;
              if (!(dot_nb > Real(0))) up += dot_nb * other;
            }
          }
          *own_p = (D == 1 ? detJ : weight * detJ) * up;
        }
        __syncthreads();
        // tangential B^T (D-1 passes) on the 2 * ne own-side tensors
        static_for<0, D - 1>([&](auto mc) {
          constexpr int m = decltype(mc)::value;
          const int bin = (FB + m) & 1, bout = bin ^ 1;
#pragma unroll
          for (int s = 0; s < 2; ++s)
            contract_pass<Q, N, ipow(N, m), ipow(Q, D - 2 - m), false>(ColMat<Real, N>{sB}, F(s, 0, bin), MF,
                                                                      F(s, 0, bout), MF, ne);
          __syncthreads();
        });
        constexpr int RB = (FB + D - 1) & 1;
        // add both faces of this axis into the element result
        for (int l = tid; l < ne * ND; l += nth) {
          const int b = l / ND;
          const int i = l - b * ND;
          const int ia = (i / SA) % N;
          const int f = (i % SA) + (i / (SA * N)) * SA;
          const Real r0 = F(0, 0, RB)[(int64_t)b * MF + f];
          const Real r1 = F(1, 0, RB)[(int64_t)b * MF + f];
          Real add;
          if (GLL) {
            add = Real(0);
            if (ia == 0) add += r0;
            if (ia == N - 1) add += r1;
          } else {
            add = sBf[ia] * r0 + sBf[N + ia] * r1;
          }
          sy[l] += add;
        }
        __syncthreads();
      });
    }

    // ------------------------------------------------------------------ write
    {
      Real* ys = P.y + e0 * ND;
      const Real alpha = P.alpha, by = P.beta_y;
      if (by == Real(0)) {
        for (int i = tid; i < ne * ND; i += nth) ys[i] = alpha * sy[i];
      } else {
        for (int i = tid; i < ne * ND; i += nth) ys[i] = alpha * sy[i] + by * ys[i];
      }
    }
  }
}

}  // namespace dgop
