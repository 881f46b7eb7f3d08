// Host planner for the Kronecker form (see kron.h): eligibility and per-axis matrix tables.
#include "kron_plan.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace dgop {

namespace {

// f(e, point j): table value or 1.
inline double fval(const double* tab, int ld, int64_t e, int j) { return tab ? tab[e * ld + j] : 1.0; }

// Append one N x N mass-type matrix per element coordinate (a single one when tab == nullptr).
KronMat add_mass(std::vector<double>& mats, const KronInputs& in, int axis, const double* tab, double scale) {
  const int N = in.N, Q = in.Q, ld = Q + 2;
  const int64_t count = tab ? in.sizes[axis] : 1;
  KronMat m;
  m.off = (int64_t)mats.size();
  m.stride = tab ? N * N : 0;
  for (int64_t e = 0; e < count; ++e)
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) {
        double s = 0.0;
        for (int q = 0; q < Q; ++q) s += in.B[q * N + i] * (in.wq[q] * fval(tab, ld, e, q)) * in.B[q * N + j];
        mats.push_back(scale * s);
      }
  return m;
}

// G[j][m] = sum_p (sum_q B[q][j] Dq[p][q]) w_p f_p B[p][m], scaled; optionally plus a scaled
// mass-type matrix (the merged mass term), optionally transposed.
KronMat add_grad(std::vector<double>& mats, const KronInputs& in, int axis, const double* tab, double scale,
                 bool transpose, const double* mtab, double mscale, bool with_mass) {
  const int N = in.N, Q = in.Q, ld = Q + 2;
  const bool varies = tab || (with_mass && mtab);
  const int64_t count = varies ? in.sizes[axis] : 1;
  KronMat m;
  m.off = (int64_t)mats.size();
  m.stride = varies ? N * N : 0;
  for (int64_t e = 0; e < count; ++e) {
    double G[kMaxN][kMaxN];
    for (int j = 0; j < N; ++j)
      for (int c = 0; c < N; ++c) {
        double s = 0.0;
        for (int p = 0; p < Q; ++p) {
          double bd = 0.0;
          for (int q = 0; q < Q; ++q) bd += in.B[q * N + j] * in.Dq[p * Q + q];
          s += bd * (in.wq[p] * fval(tab, ld, e, p)) * in.B[p * N + c];
        }
        G[j][c] = scale * s;
        if (with_mass) {
          double ms = 0.0;
          for (int q = 0; q < Q; ++q) ms += in.B[q * N + j] * (in.wq[q] * fval(mtab, ld, e, q)) * in.B[q * N + c];
          G[j][c] += mscale * ms;
        }
      }
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) mats.push_back(transpose ? G[j][i] : G[i][j]);
  }
  return m;
}

// Sign of f over each element's Gauss points: +1 / -1 / 0 (all zero); false if mixed.
bool sign_table(const KronInputs& in, int axis, const double* tab, std::vector<signed char>& out) {
  const int Q = in.Q, ld = Q + 2;
  out.assign(in.sizes[axis], 1);
  if (!tab) return true;
  for (int64_t e = 0; e < in.sizes[axis]; ++e) {
    bool pos = false, neg = false;
    for (int q = 0; q < Q; ++q) {
      const double v = tab[e * ld + q];
      if (!std::isfinite(v)) return false;
      if (v > 0) pos = true;
      if (v < 0) neg = true;
    }
    if (pos && neg) return false;
    out[e] = pos ? 1 : (neg ? -1 : 0);
  }
  return true;
}

// In-place inverse of one N x N block (Gauss-Jordan with partial pivoting); false if singular.
bool invert_block(double* a, int N) {
  double inv[kMaxN * kMaxN];
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) inv[i * N + j] = i == j ? 1.0 : 0.0;
  for (int c = 0; c < N; ++c) {
    int piv = c;
    for (int r = c + 1; r < N; ++r)
      if (std::fabs(a[r * N + c]) > std::fabs(a[piv * N + c])) piv = r;
    if (!(std::fabs(a[piv * N + c]) > 0.0)) return false;
    if (piv != c)
      for (int j = 0; j < N; ++j) {
        std::swap(a[c * N + j], a[piv * N + j]);
        std::swap(inv[c * N + j], inv[piv * N + j]);
      }
    const double d = 1.0 / a[c * N + c];
    for (int j = 0; j < N; ++j) {
      a[c * N + j] *= d;
      inv[c * N + j] *= d;
    }
    for (int r = 0; r < N; ++r) {
      if (r == c) continue;
      const double f = a[r * N + c];
      if (f == 0.0) continue;
      for (int j = 0; j < N; ++j) {
        a[r * N + j] -= f * a[c * N + j];
        inv[r * N + j] -= f * inv[c * N + j];
      }
    }
  }
  for (int i = 0; i < N * N; ++i) a[i] = inv[i];
  return true;
}

// Invert every block of a matrix table in place.
bool invert_table(std::vector<double>& mats, const KronMat& m, int64_t count, int N) {
  for (int64_t e = 0; e < count; ++e)
    if (!invert_block(mats.data() + m.off + e * m.stride, N)) return false;
  return true;
}

}  // namespace

// The Kronecker form for any dimension (see kron.h): eligibility of the coefficients and the
// per-axis matrix tables.  Dimension- and size-specific limits are the callers'.
KronPlanHost plan_kron(const KronInputs& in) {
  KronPlanHost p;
  p.N = in.N;
  p.dim = in.D;
  const int Dm = in.D;
  if (!in.gll) {
    p.why = "basis is not GLL";
    return p;
  }
  const bool adv = (in.flags & kAdvCell) != 0;
  const bool mass = (in.flags & kMass) != 0;
  if (!adv && !mass) {
    p.why = "empty operator";
    return p;
  }
  if (in.inverse_mass && (adv || !mass || in.sigma.has_elem)) {
    p.why = "the mass inverse takes a density without per-element factor and no advection";
    return p;
  }
  if (adv)
    for (int a = 0; a < Dm; ++a)
      if (!in.beta[a].separable) {
        p.why = "velocity component is not a single separable product";
        return p;
      }
  if (mass && !in.sigma.separable) {
    p.why = "density is not a single separable product";
    return p;
  }
  double detJ = 1.0;
  for (int k = 0; k < Dm; ++k) detJ *= in.h[k];
  p.has_adv = adv;
  p.has_mass = mass;
  auto& M = p.mats;
  const int last = Dm - 1;
  if (adv) {
    // the mass term merges into the last axis' term when its other factors equal that term's
    const SepCoef& bl = in.beta[last];
    bool same = mass && !in.sigma.has_elem && !bl.has_elem;
    for (int k = 0; k < last && same; ++k) same = in.sigma.tab[k] == bl.tab[k];
    p.mass_merged = same;
    for (int a = 0; a < Dm; ++a) {
      const SepCoef& b = in.beta[a];
      const double invh = 1.0 / in.h[a];
      const double s_a = -b.c * detJ * invh;
      const bool merge = p.mass_merged && a == last;
      const double s_m = in.sigma.c * detJ;
      p.D[a] = add_grad(M, in, a, b.tab[a], s_a, false, in.sigma.tab[last], s_m, merge);
      p.Dt[a] = add_grad(M, in, a, b.tab[a], s_a, true, in.sigma.tab[last], s_m, merge);
      for (int k = 0; k < Dm; ++k) {
        if (k == a) continue;
        p.T[a][k] = add_mass(M, in, k, b.tab[k], 1.0);
        if (!sign_table(in, k, b.tab[k], p.sgn[a][k])) {
          p.why = "upwind direction changes sign inside an element face";
          return p;
        }
      }
      // phi_s(e_a) = detJ c_a f_aa(face s) (+-1/h_a); face s = 0 at xhat = 0 (index Q), 1 at xhat = 1
      const int ld = in.Q + 2;
      p.phi[a].resize(2 * in.sizes[a]);
      for (int64_t e = 0; e < in.sizes[a]; ++e)
        for (int s = 0; s < 2; ++s) {
          const double f = b.tab[a] ? b.tab[a][e * ld + in.Q + s] : 1.0;
          p.phi[a][2 * e + s] = detJ * b.c * f * (s ? invh : -invh);
        }
    }
  }
  if (mass && !p.mass_merged) {
    const double s_m = in.sigma.c * detJ;
    p.MD = add_mass(M, in, last, in.sigma.tab[last], s_m);
    for (int k = 0; k < last; ++k) p.MT[k] = add_mass(M, in, k, in.sigma.tab[k], 1.0);
    if (in.inverse_mass) {
      // (x)_k A_k is inverted factor by factor: every block of every table
      bool ok = invert_table(M, p.MD, p.MD.stride ? in.sizes[last] : 1, in.N);
      for (int k = 0; k < last && ok; ++k) ok = invert_table(M, p.MT[k], p.MT[k].stride ? in.sizes[k] : 1, in.N);
      if (!ok) {
        p.why = "singular element mass matrix";
        return p;
      }
    }
  }
  p.ok = true;
  return p;
}

KronPlanHost plan_kron3d(const KronInputs& in) {
  KronPlanHost p;
  p.N = in.N;
  if (in.D != 3) {
    p.why = "dimension != 3";
    return p;
  }
  if (in.N > 4) {  // the FP64 register kernel spills above N = 4
    p.why = "order above 3 (register kernel limit)";
    return p;
  }
  if ((uint64_t)in.sizes[0] * in.sizes[1] * in.sizes[2] >= (uint64_t(1) << 32)) {
    p.why = "more than 2^32 elements";
    return p;
  }
  return plan_kron(in);
}

}  // namespace dgop
