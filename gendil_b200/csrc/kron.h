// Kronecker ("1D matrix") form of the DG operators on Cartesian meshes.
//
// With every coefficient separable per axis -- beta_a(X) = c_a * prod_k f_ak(X_k) and
// sigma(X) = c_s * prod_k g_k(X_k) -- and GLL nodes (face trace = face slice), each term of the
// reference's sum-factorized operator (advectionoperator.hpp:269-441, massoperator.hpp:39-89)
// collapses to a tensor product of per-axis n x n matrices that depend only on the element's
// coordinate along that axis:
//
//   M_k^f[e]  = B^T W f B            (mass-type, symmetric)
//   G_k^f[e]  = B^T Dq^T W f B       (collocated gradient along the component's own axis)
//
//   y_e = sum_a  T_a [ D_a u_e + sum_{inflow faces s} phi_s(e) e_s (x) trace_{1-s}(u_nb) ]
//   T_a = (x)_{k != a} M_k^{f_ak}[e_k],   D_a = s_a G_a^{f_aa}[e_a] + sum_{outflow s} phi_s e_s e_s^T
//
// s_a = -c_a detJ / h_a, phi_s(e_a) = detJ c_a f_aa(face s) (+-1/h_a).  The upwind choice needs
// the sign of beta . n to be uniform over each face, i.e. each tangential factor keeps one sign
// on each element's Gauss points; the planner checks this and otherwise leaves the operator on
// the generic sum-factorized kernel.  The mass term merges into the z term when its x and y
// factors equal the z velocity's.
#pragma once

#include <cstdint>
#include <vector>

#include "dgop_params.h"
#include "fastdiv.h"

namespace dgop {

constexpr int kKronMaxN = 5;

// A per-axis matrix table: matrix for element coordinate e at off + e * stride (stride 0: one
// matrix for all elements).  Offsets are into the plan's matrix buffer.
struct KronMat {
  int64_t off = -1;
  int64_t stride = 0;
};

// Matrix slots of the 3D kernel (see kron3d_kernel.cuh); the axis each slot acts along is fixed.
enum KronSlot : int {
  kSlotDX = 0,   // x term, along x (forward or transposed D)
  kSlotDY = 1,   // y term, along y
  kSlotDZ = 2,   // z term (mass merged) or the mass term alone, along z
  kSlotTXY = 3,  // x term, y tangential
  kSlotTXZ = 4,  // x term, z tangential
  kSlotTYZ = 5,  // y term, z tangential
  kSlotTYX = 6,  // y term, x tangential
  kSlotTZX = 7,  // z term, x tangential
  kSlotTZY = 8,  // z term, y tangential
  kSlotMD = 9,   // separate mass term, along z
  kSlotMX = 10,  // separate mass term, x tangential
  kSlotMY = 11,  // separate mass term, y tangential
  kNumSlots = 12
};

template <typename Real>
struct KronParams {
  int64_t nelem;      // < 2^32 (checked by the planner); the launch processes [e_begin, nelem)
  int64_t e_begin;
  FastDiv fdx, fdy;   // element index -> (x, y, z) coordinates
  int64_t sizes[3];
  int periodic[3];
  int flags;          // kAdvCell / kFaceInt / kFaceBnd / kMass / kTranspose as in OpFlags
  int has_adv;        // advection terms present
  int has_mass;       // mass term present
  int mass_merged;    // mass folded into the z term's D matrix
  Real g;             // inflow value
  Real alpha, beta_y;
  const Real* x;
  Real* y;
  const Real* mats;                          // element-dependent matrix tables (device)
  int vary[kNumSlots];                       // slot depends on the element coordinate
  KronMat vm[kNumSlots];                     // table of a varying slot
  Real cm[kNumSlots][kKronMaxN * kKronMaxN]; // matrix of a constant slot (kernel-parameter space)
  const Real* phi[3];            // phi[a][e_a * 2 + s]
  const signed char* sgn[3][3];  // sgn[a][k][e_k] in {-1, 0, 1} (k != a)
  const Real* elem[3];           // per-element beta_a factor or nullptr
  const Real* elem_mass;         // per-element sigma factor or nullptr
  const int* skip;               // device word; the launch does nothing when it is non-zero
  // optional epilogue: dot_partials[b] = sum over CTA b's outputs of dot_z . y (fixed order),
  // entries b >= gridDim.x of the first dot_count zeroed (dot_partials null: no epilogue)
  const Real* dot_z;
  double* dot_partials;
  int dot_count;
};

// Which slots have element-dependent matrices: a compile-time mask of the 3D kernels (bit k:
// slot k varies) or kVaryRuntime (read P.vary).  A kernel compiled for one mask carries one code
// path per pass instead of two, half the instructions to fetch (the run-time form of the
// bulk-tensor kernel measured 7 % slower on the 64^3 p=3 advection apply); the launchers take
// such a kernel only for operators whose mask matches.  kVarySheared: beta_x depends on y and
// beta_y on z (beta_z constant).  kron_mask_index: 0 for kVaryNone, 1 for kVarySheared, -1 else.
constexpr uint32_t kVaryRuntime = 0xFFFFFFFFu;
constexpr uint32_t kVaryNone = 0u;
constexpr uint32_t kVarySheared = (1u << kSlotTXY) | (1u << kSlotTYZ);

template <typename Real>
inline uint32_t kron_vary_mask(const KronParams<Real>& k) {
  uint32_t m = 0;
  for (int i = 0; i < kNumSlots; ++i)
    if (k.vary[i]) m |= 1u << i;
  return m;
}
template <typename Real>
inline int kron_mask_index(const KronParams<Real>& k) {
  const uint32_t m = kron_vary_mask(k);
  return m == kVaryNone ? 0 : (m == kVarySheared ? 1 : -1);
}

// Launch parameters of the any-dimension kernel (kronnd_kernel.cuh).
template <typename Real>
struct KronNDParams {
  int64_t nelem;    // the launch processes elements [e_begin, nelem)
  int64_t e_begin;
  int64_t sizes[kMaxDim];
  int64_t estride[kMaxDim];  // element index = sum_k c_k estride[k]
  int periodic[kMaxDim];
  int flags;        // OpFlags
  int has_adv, has_mass, mass_merged;
  int eb;           // elements per CTA
  Real g, alpha, beta_y;
  const Real* x;
  Real* y;
  const Real* mats;              // matrix tables (device)
  KronMat slot[kMaxDim][kMaxDim];  // [a][k]: term a's matrix along k (k == a: D, or D^T when transposed)
  KronMat mslot[kMaxDim];          // separate mass term: matrix along k
  const Real* phi[kMaxDim];        // phi[a][e_a * 2 + s]
  const signed char* sgn[kMaxDim][kMaxDim];
  const Real* elem[kMaxDim];
  const Real* elem_mass;
  const int* skip;
  // tensor-core variant (kronnd_tc_kernel.cuh, FP32 operators): BF16 Kronecker products of every
  // term's tangential matrices over the fast half (h = 0) and the slow half (h = 1) of the axes,
  // padded tiles; the tile of term t, half h for an element with coordinates c is number
  // tc_base[t][h] + sum_k c_k tc_mult[t][k] (over the half's axes), its scale tc_scale[that]
  const void* tc_tiles;
  const float* tc_scale;
  int tc_base[kMaxDim + 1][2];
  int tc_mult[kMaxDim + 1][kMaxDim];
};

// Interior-penalty diffusion (kronnd_diff_kernel.cuh, sipdg.cu).
// Base matrix k of axis a in the table: mats[(a * kDiffMats + k) * N * N]
enum DiffMat : int {
  kDK = 0,    // Khat
  kDP1 = 1,   // P1_0, P1_1
  kDP2 = 3,   // P2_0, P2_1
  kDP3 = 5,   // P3_0, P3_1
  kDQ1 = 7,   // Q1_0, Q1_1
  kDQ2 = 9,   // Q2_0, Q2_1
  kDQ3 = 11,  // Q3_0, Q3_1
  kDM = 13,   // reference mass M_a (tangential factor)
  kDiffMats = 14
};

constexpr int kDiffMaxEB = 64;  // elements per CTA of the diffusion kernels, at most

template <typename Real>
struct KronDiffParams {
  int64_t nelem, e_begin;
  int64_t sizes[kMaxDim];
  int64_t estride[kMaxDim];
  int periodic[kMaxDim];
  int boundary;  // Dirichlet-0 boundary terms
  int eb;        // elements per CTA
  Real sigma;    // -1 SIPG, +1 NIPG, 0 IIPG
  Real alpha, beta_y;
  const Real* x;
  Real* y;
  const Real* mu;    // per element (device)
  const Real* mats;  // D x kDiffMats base matrices, N x N each (device), then the trace rows
                     // l(0), l(1), l'(0), l'(1) (N each)
  const int* skip;
  // coefficient gradient (kronnd_diff_grad_kernel): gout[e] = gscale[e] lam^T (dA/dmu_e) x
  const Real* lam;
  Real* gout;
  const Real* gscale;
  Real kappa;
  Real face_h[kMaxDim];  // detJ / h_a^2
};

struct KronPlanHost {
  bool ok = false;
  const char* why = "";
  int N = 0, dim = 0;
  std::vector<double> mats;               // all matrices, row-major N x N each
  std::vector<double> phi[kMaxDim];       // per axis, e * 2 + s
  std::vector<signed char> sgn[kMaxDim][kMaxDim];
  // term a: D[a] (Dt[a] transposed) along a, T[a][k] along k != a; a separate mass term: MD along
  // the last axis, MT[k] along the others
  KronMat D[kMaxDim], Dt[kMaxDim], T[kMaxDim][kMaxDim], MD, MT[kMaxDim];
  int has_adv = 0, has_mass = 0, mass_merged = 0;
};

// Host-side description of one scalar coefficient: c * prod_k table_k (table_k may be null).
struct SepCoef {
  bool separable = false;   // constant, or one product term with no constant
  double c = 1.0;
  const double* tab[kMaxDim] = {};  // host tables, n_k * (q + 2)
  bool has_elem = false;
};

}  // namespace dgop
