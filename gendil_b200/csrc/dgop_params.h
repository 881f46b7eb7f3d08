// Device-side parameter blocks shared by the operator kernels and the host dispatcher.
#pragma once

#include <cstdint>

namespace dgop {

constexpr int kMaxDim = 6;
constexpr int kMaxN = 8;      // 1D basis size p + 1 (orders 0..7)
constexpr int kMaxQ = 8;      // 1D Gauss-Legendre points
constexpr int kMaxTerms = 4;  // separable product terms per scalar coefficient

// Operator content flags.
enum OpFlags : int {
  kMass = 1 << 0,       // sigma * u * v                        (massoperator.hpp:65-83)
  kAdvCell = 1 << 1,    // -u beta . grad v                      (advectionoperator.hpp:293-331)
  kFaceInt = 1 << 2,    // upwind flux on interior faces         (advectionoperator.hpp:339-389)
  kFaceBnd = 1 << 3,    // upwind flux on boundary faces, inflow value g (advectionoperator.hpp:391-438)
  kTranspose = 1 << 4,  // apply the transposed (adjoint) operator
  kLinear = 1 << 5,     // host-side launch option: inflow value taken as 0 (the linear part)
  kInvMass = 1 << 6,    // operator is the inverse of the element mass matrices (Kronecker kernels only)
  kDiffusion = 1 << 7,  // interior-penalty diffusion operator (dgop_sipdg_create)
};

// A scalar coefficient c(X) = constant + sum_t prod_k T_{t,k}(X_k), optionally multiplied by a
// per-element factor.  T_{t,k} is tabulated per element index e_k along axis k at the points
// j = 0..q-1 (Gauss points), j = q (element face at 0) and j = q+1 (face at 1), i.e. at
// X_k = (origin_k + h_k e_k) + h_k xhat_j, the coordinate the reference computes at every
// quadrature point (hypercubecell.hpp:41-52).
template <typename Real>
struct CoefDev {
  Real constant;
  int nterms;
  int64_t off[kMaxTerms][kMaxDim];  // offset into the table buffer, -1 for a factor of 1
  const Real* elem;                 // per-element multiplier or nullptr
};

template <typename Real>
struct OpParams {
  int64_t nelem;    // the launch processes elements [e_begin, nelem)
  int64_t e_begin;
  int64_t sizes[kMaxDim];
  int64_t estride[kMaxDim];  // element linear index = sum_k e_k * estride[k], x fastest
  int periodic[kMaxDim];
  Real invh[kMaxDim];
  Real detJ;
  Real B[kMaxQ * kMaxN];    // B[q * N + j] = l_j(x_q)
  Real Dq[kMaxQ * kMaxQ];   // Dq[i * Q + j] = l^GL_j'(x_i) (collocated, doftoquad.hpp:142-150)
  Real Bf[2][kMaxN];        // basis values at the faces xhat = 0 and 1
  Real wq[kMaxQ];           // Gauss weights on [0,1]
  int tab_ld;               // q + 2
  const Real* tab;          // coefficient tables
  CoefDev<Real> sigma;
  CoefDev<Real> beta[kMaxDim];
  Real g;                   // inflow value on boundary faces
  int flags;
  int gll;                  // 1: basis nodes include both faces (exact trace selection)
  Real alpha;               // y = alpha * Op(x) + beta_y * y
  Real beta_y;
  const Real* x;
  Real* y;
  int eb;                   // elements per CTA
  Real* scratch;            // global workspace when the element does not fit in shared memory
  int64_t scratch_per_cta;  // in Real elements
  const int* skip;          // device word; the launch does nothing when it is non-zero (solvers)
};

}  // namespace dgop
