// Kronecker-form DG operator with BF16 tensor-core contractions, FP32 accumulation and per-element
// max-abs scaling (the low-precision inner operator of the refinement solvers).
//
// For an even dimension D the element's axes split into a fast half (axes 0 .. D/2 - 1, stride
// < F = N^(D/2)) and a slow half, so the element's values form an F x F matrix U[s][f] (element
// index f + F s).  A term of the operator (kronnd_kernel.cuh: the pass along its own axis a with
// D_a, the face terms of axis a, then the tangential passes) becomes
//
//   W   = D_a along a applied to U, plus the face terms      (FP32, CUDA cores, one pass)
//   T^T = K_F W^T,  Y += K_S T                                (two BF16 tensor-core GEMMs)
//
// with K_F = (x)_{k fast} T_k and K_S = (x)_{k slow} T_k the Kronecker products of the term's
// tangential matrices (the identity on axis a).  W, K_F, the intermediate T = W K_F^T and K_S are
// each rounded to BF16 after division by their largest magnitude; the products accumulate in FP32
// (mma.sync m16n8k16) and the four scales multiply the term's contribution to the FP32
// accumulator Y (registers, in the GEMMs' fragment layout).  K_F and K_S depend on the element
// only through its coordinates along the
// half's axes whose matrices vary, so they are built once per operator on the host (padded BF16
// tiles with their scales, tc_tiles) and read by the GEMMs straight from global memory (L2).  One
// warp per element: its input, W (FP32), own-axis matrices and face records in shared memory and
// one BF16 tile padded to P x P (P = 16 or 32, row stride P + 8 so that the 32-bit fragment
// loads hit distinct banks) for W, then T^T; its padding is zeroed once and stays zero (W and
// T^T only write their F x F parts and the zero padding of W and K_F makes T^T's padding zero).
// No CTA-wide synchronisation.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "kronnd_kernel.cuh"

namespace dgop {

template <int D, int N>
struct KronTCShape {
  static constexpr int H = D / 2;          // fast axes 0 .. H - 1, slow axes H .. D - 1
  static constexpr int F = kpow(N, H);     // U is F x F
  static constexpr int P = F <= 16 ? 16 : 32;
  static constexpr int LD = P + 8;         // BF16 row stride of a tile
  static constexpr int MT = P / 16, NT = P / 8, KS = P / 16;
  static constexpr int ND = kpow(N, D);
  static constexpr int NL = ND / N;
  static constexpr int LPL = (NL + 31) / 32;  // lines per lane in the own-axis pass
  using NDS = KronNDShape<D, N>;
  static constexpr int MAT = N * N;
  // U, W, the own-axis matrix of each term (D advection terms and the mass term), face records
  static constexpr int FLOATS = 2 * ND + (D + 1) * MAT + NDS::REC;
  static constexpr int FLOAT_BYTES = (FLOATS * 4 + 15) / 16 * 16;
  static constexpr int TILE = P * LD;  // BF16 values per tile
  static constexpr int WARP_BYTES = FLOAT_BYTES + TILE * 2;
  static constexpr bool OK = (D % 2 == 0) && D >= 2 && F <= 32 && N >= 2;
};

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ uint32_t ld_b32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// C[mt][nt] = A B^T over the padded tiles: A row-major [m][k] (stride LD), Bt row-major [n][k].
// Fragment layouts of mma.m16n8k16 (PTX ISA): g = lane / 4, t = lane % 4; A holds rows g, g + 8
// and columns 2t, 2t + 1, 2t + 8, 2t + 9 of its 16 x 16 block; B columns (n) g and rows (k) 2t,
// 2t + 1, 2t + 8, 2t + 9; C rows g, g + 8 and columns 2t, 2t + 1.
template <int D, int N>
__device__ __forceinline__ void tc_gemm(const __nv_bfloat16* A, const __nv_bfloat16* Bt,
                                        float (&C)[KronTCShape<D, N>::MT][KronTCShape<D, N>::NT][4], int lane) {
  using S = KronTCShape<D, N>;
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mt = 0; mt < S::MT; ++mt)
#pragma unroll
    for (int nt = 0; nt < S::NT; ++nt)
#pragma unroll
      for (int i = 0; i < 4; ++i) C[mt][nt][i] = 0.0f;
#pragma unroll
  for (int ks = 0; ks < S::KS; ++ks) {
    uint32_t b[S::NT][2];
#pragma unroll
    for (int nt = 0; nt < S::NT; ++nt) {
      const __nv_bfloat16* q = Bt + (nt * 8 + g) * S::LD + ks * 16 + 2 * t;
      b[nt][0] = ld_b32(q);
      b[nt][1] = ld_b32(q + 8);
    }
#pragma unroll
    for (int mt = 0; mt < S::MT; ++mt) {
      const __nv_bfloat16* p = A + (mt * 16 + g) * S::LD + ks * 16 + 2 * t;
      const uint32_t a[4] = {ld_b32(p), ld_b32(p + 8 * S::LD), ld_b32(p + 8), ld_b32(p + 8 * S::LD + 8)};
#pragma unroll
      for (int nt = 0; nt < S::NT; ++nt) mma_bf16_16816(C[mt][nt], a, b[nt]);
    }
  }
}

// W along the lines of axis AX: out[j] for line l (the own-axis pass of the term times the element
// factor, plus the face terms of AX); `off` receives the line's first element-local index.
template <int D, int N, int TERM>
__device__ __forceinline__ void tc_w_line(const KronNDParams<float>& P, int64_t e, const int* ec, const float* U,
                                          const float* m, float scale, bool scaled, const float* rec, int l,
                                          float (&out)[N], int& off) {
  constexpr bool MASS = TERM == D;
  constexpr int AX = MASS ? D - 1 : TERM;
  constexpr int INNER = kpow(N, AX);
  constexpr int ND = kpow(N, D);
  const int o = l / INNER, t = l - o * INNER;
  off = o * N * INNER + t;
  float v[N];
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = U[off + i * INNER];
#pragma unroll
  for (int j = 0; j < N; ++j) {
    float s = m[j * N] * v[0];
#pragma unroll
    for (int i = 1; i < N; ++i) s += m[j * N + i] * v[i];
    out[j] = scaled ? s * scale : s;
  }
  if constexpr (!MASS) {
    const uint8_t* fb = reinterpret_cast<const uint8_t*>(rec + 4 * D);
#pragma unroll
    for (int sd = 0; sd < 2; ++sd) {
      const int fi = AX * 2 + sd;
      const uint32_t f = fb[fi];
      if (!f) continue;
      const int sl = sd ? N - 1 : 0;
      float add = 0.0f;
      if (f & 1u) add += rec[2 * fi] * v[sl];
      if (f & 2u) {
        const int64_t n = P.sizes[AX];
        const int64_t ca = ec[AX];
        const int64_t cn = sd ? (ca + 1 == n ? 0 : ca + 1) : (ca == 0 ? n - 1 : ca - 1);
        const int64_t en = e + (cn - ca) * P.estride[AX];
        add += rec[2 * fi + 1] * P.x[en * ND + off + (N - 1 - sl) * INNER];
      } else if (f & 4u) {
        add += rec[2 * fi + 1] * P.g;
      }
      out[sl] += add;
    }
  }
}

// One term (TERM == D: the separate mass term, first pass along D - 1) of element e added to the
// shared accumulator Y (element layout).
template <int D, int N, int TERM>
__device__ __forceinline__ void tc_term(const KronNDParams<float>& P, int64_t e, const int* ec, const float* U,
                                        float (&Y)[KronTCShape<D, N>::MT][KronTCShape<D, N>::NT][4], float* Wf,
                                        const float* own, const float* rec, __nv_bfloat16* T0, int lane) {
  using S = KronTCShape<D, N>;
  constexpr bool MASS = TERM == D;
  constexpr int AX = MASS ? D - 1 : TERM;
  constexpr int INNER = kpow(N, AX);
  const float* m = own + TERM * N * N;
  const float* ef = MASS ? P.elem_mass : P.elem[AX];
  const float scale = ef ? ef[e] : 1.0f;
  // W (FP32, element layout) and its largest magnitude
  float wmax = 0.0f;
  for (int l = lane; l < S::NL; l += 32) {
    float w[N];
    int off;
    tc_w_line<D, N, TERM>(P, e, ec, U, m, scale, ef != nullptr, rec, l, w, off);
#pragma unroll
    for (int j = 0; j < N; ++j) {
      Wf[off + j * INNER] = w[j];
      wmax = fmaxf(wmax, fabsf(w[j]));
    }
  }
  wmax = warp_max(wmax);
  if (wmax == 0.0f) return;  // uniform over the warp
  // the term's Kronecker tiles (global memory) and their scales
  const __nv_bfloat16* tiles = reinterpret_cast<const __nv_bfloat16*>(P.tc_tiles);
  int64_t t0 = P.tc_base[TERM][0], t1 = P.tc_base[TERM][1];
#pragma unroll
  for (int k = 0; k < D; ++k) {
    if (k < S::H) t0 += (int64_t)ec[k] * P.tc_mult[TERM][k];
    else t1 += (int64_t)ec[k] * P.tc_mult[TERM][k];
  }
  const __nv_bfloat16* KF = tiles + t0 * S::TILE;
  const __nv_bfloat16* KS = tiles + t1 * S::TILE;
  const float sf = P.tc_scale[t0], ss = P.tc_scale[t1];
  // W / wmax into the tile ([s][f]; the padding stays zero): lane s converts row s, two columns
  // per 32-bit store (row stride F floats in Wf: distinct banks for odd F)
  __syncwarp();
  const float winv = 1.0f / wmax;
  for (int r = lane; r < S::F; r += 32) {
    const float* src = Wf + r * S::F;
    __nv_bfloat16* dst = T0 + r * S::LD;
#pragma unroll
    for (int c = 0; c + 1 < S::F; c += 2)
      *reinterpret_cast<__nv_bfloat162*>(dst + c) = __floats2bfloat162_rn(src[c] * winv, src[c + 1] * winv);
    if constexpr (S::F % 2) dst[S::F - 1] = __float2bfloat16_rn(src[S::F - 1] * winv);
  }
  __syncwarp();
  float C[S::MT][S::NT][4];
  tc_gemm<D, N>(KF, T0, C, lane);  // T^T = K_F W^T  (rows f', columns s)
  float tmax = 0.0f;
#pragma unroll
  for (int mt = 0; mt < S::MT; ++mt)
#pragma unroll
    for (int nt = 0; nt < S::NT; ++nt)
#pragma unroll
      for (int i = 0; i < 4; ++i) tmax = fmaxf(tmax, fabsf(C[mt][nt][i]));
  tmax = warp_max(tmax);
  __syncwarp();
  if (tmax == 0.0f) return;
  // T^T into the tile ([f'][s]): each lane's pairs of adjacent columns as one 32-bit store
  const float tinv = 1.0f / tmax;
  const int g = lane >> 2, tq = lane & 3;
#pragma unroll
  for (int mt = 0; mt < S::MT; ++mt)
#pragma unroll
    for (int nt = 0; nt < S::NT; ++nt)
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const int r = mt * 16 + g + hh * 8;  // f'
        const int c = nt * 8 + 2 * tq;       // s
        *reinterpret_cast<__nv_bfloat162*>(T0 + r * S::LD + c) =
            __floats2bfloat162_rn(C[mt][nt][2 * hh] * tinv, C[mt][nt][2 * hh + 1] * tinv);
      }
  __syncwarp();
  tc_gemm<D, N>(KS, T0, C, lane);  // K_S T  (rows s', columns f')
  const float f = wmax * sf * tmax * ss;
#pragma unroll
  for (int mt = 0; mt < S::MT; ++mt)
#pragma unroll
    for (int nt = 0; nt < S::NT; ++nt)
#pragma unroll
      for (int i = 0; i < 4; ++i) Y[mt][nt][i] += f * C[mt][nt][i];
  __syncwarp();
}

template <int D, int N>
__global__ void __launch_bounds__(kKronTCThreads, 4) kronnd_tc_kernel(const __grid_constant__ KronNDParams<float> P) {
  using S = KronTCShape<D, N>;
  using NDS = KronNDShape<D, N>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* mine = smem_raw + (size_t)warp * S::WARP_BYTES;
  float* U = reinterpret_cast<float*>(mine);
  float* Wf = U + S::ND;
  float* own = Wf + S::ND;  // own-axis matrix of term t at own + t N^2 (t = D: the mass term)
  float* rec = own + (D + 1) * S::MAT;
  __nv_bfloat16* T0 = reinterpret_cast<__nv_bfloat16*>(mine + S::FLOAT_BYTES);
  if (P.skip && *P.skip) return;
  {
    uint4* z = reinterpret_cast<uint4*>(T0);
    for (int q = lane; q < S::TILE * 2 / 16; q += 32) z[q] = make_uint4(0u, 0u, 0u, 0u);
  }
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t e = P.e_begin + (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5); e < P.nelem; e += nw) {
    __syncwarp();
    int ec[kMaxDim];
#pragma unroll
    for (int k = 0; k < D; ++k) ec[k] = (int)((e / P.estride[k]) % P.sizes[k]);
    for (int i = lane; i < S::ND; i += 32) U[i] = P.x[e * S::ND + i];
    for (int l = lane; l < (D + 1) * S::MAT; l += 32) {
      const int t = l / S::MAT, q = l - t * S::MAT;
      const int k = t < D ? t : D - 1;
      const KronMat mm = t < D ? P.slot[t][t] : P.mslot[D - 1];
      own[l] = mm.off >= 0 ? P.mats[mm.off + (int64_t)ec[k] * mm.stride + q] : 0.0f;
    }
    if (P.has_adv)
      for (int fi = lane; fi < 2 * D; fi += 32)
        nd_face_record<D>(P, e, ec, fi, rec, reinterpret_cast<uint8_t*>(rec + 4 * D) + fi);
    __syncwarp();
    float Y[S::MT][S::NT][4];
#pragma unroll
    for (int mt = 0; mt < S::MT; ++mt)
#pragma unroll
      for (int nt = 0; nt < S::NT; ++nt)
#pragma unroll
        for (int i = 0; i < 4; ++i) Y[mt][nt][i] = 0.0f;
    if (P.has_adv) {
      static_for<0, D>([&](auto ac) {
        tc_term<D, N, decltype(ac)::value>(P, e, ec, U, Y, Wf, own, rec, T0, lane);
      });
    }
    if (P.has_mass && !(P.has_adv && P.mass_merged)) tc_term<D, N, D>(P, e, ec, U, Y, Wf, own, rec, T0, lane);
    // y = alpha Y + beta_y y (Y rows s', columns f': element index f' + F s')
    const int g = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int mt = 0; mt < S::MT; ++mt)
#pragma unroll
      for (int nt = 0; nt < S::NT; ++nt)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int r = mt * 16 + g + (i >> 1) * 8;
          const int c = nt * 8 + 2 * tq + (i & 1);
          if (r < S::F && c < S::F) {
            float* dst = P.y + e * S::ND + c + S::F * r;
            *dst = (P.beta_y == 0.0f) ? P.alpha * Y[mt][nt][i] : P.alpha * Y[mt][nt][i] + P.beta_y * *dst;
          }
        }
  }
}

}  // namespace dgop
