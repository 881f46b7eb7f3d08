/* Test infrastructure only: the CPU oracle (see dg_oracle.h).  Never linked by the product.
 *
 * Plain-C restatement of the GenDiL reference algorithms for the matrix-free DG mass and upwind
 * advection path, written for clarity rather than speed: each element is processed exactly as
 * the reference's element kernels do it (read DoFs, B contractions axis by axis, q-function,
 * collocated G^T and B^T contractions, then the 2*D faces), with runtime sizes.
 */
#include "dg_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MAXD 6
#define MAXN 8

/* ------------------------------------------------------------------------------------------ */
/* 1D nodes and weights on [0,1].  The reference hard-codes these tables                         */
/* (NumericalIntegration/QuadraturePoints/GLpoints.hpp:17-240, GLLpoints.hpp:17-241); here they  */
/* are recomputed by Newton's method on the Legendre polynomials in long double.                 */
/* ------------------------------------------------------------------------------------------ */

static void legendre_eval(int n, long double x, long double *pn, long double *pnm1)
{
   long double p0 = 1.0L, p1 = x;
   if (n == 0) { *pn = 1.0L; *pnm1 = 0.0L; return; }
   for (int k = 2; k <= n; ++k)
   {
      long double p2 = ((2.0L * k - 1.0L) * x * p1 - (k - 1.0L) * p0) / (long double)k;
      p0 = p1;
      p1 = p2;
   }
   *pn = p1;
   *pnm1 = p0;
}

static int cmp_ld(const void *a, const void *b)
{
   long double x = *(const long double *)a, y = *(const long double *)b;
   return (x > y) - (x < y);
}

int dgo_points(int kind, int npts, double *coords, double *weights)
{
   if (npts < 1 || npts > MAXN) return -1;
   long double x[MAXN], w[MAXN];
   if (npts == 1)
   {
      coords[0] = 0.5; /* GLLpoints.hpp:17-43 and GLpoints.hpp: single node at the centre */
      weights[0] = 1.0;
      return 0;
   }
   const long double pi = 3.141592653589793238462643383279502884L;
   if (kind == 1)
   {
      /* Gauss-Legendre: roots of P_n, w = 2 / ((1 - x^2) P_n'(x)^2). */
      const int n = npts;
      for (int i = 0; i < n; ++i)
      {
         long double r = cosl(pi * (i + 0.75L) / (n + 0.5L));
         for (int it = 0; it < 100; ++it)
         {
            long double p, pm1;
            legendre_eval(n, r, &p, &pm1);
            long double dp = n * (r * p - pm1) / (r * r - 1.0L);
            long double dr = p / dp;
            r -= dr;
            if (fabsl(dr) < 1e-30L) break;
         }
         long double p, pm1;
         legendre_eval(n, r, &p, &pm1);
         long double dp = n * (r * p - pm1) / (r * r - 1.0L);
         x[i] = r;
         w[i] = 2.0L / ((1.0L - r * r) * dp * dp);
      }
   }
   else
   {
      /* Gauss-Lobatto-Legendre: +-1 and the roots of P_{n-1}', w = 2 / (n (n-1) P_{n-1}(x)^2). */
      const int n = npts, m = npts - 1;
      x[0] = -1.0L;
      x[n - 1] = 1.0L;
      for (int i = 1; i < n - 1; ++i)
      {
         long double r = -cosl(pi * i / (long double)m);
         for (int it = 0; it < 100; ++it)
         {
            long double p, pm1;
            legendre_eval(m, r, &p, &pm1);
            long double dp = m * (r * p - pm1) / (r * r - 1.0L);               /* P_m'  */
            long double ddp = (2.0L * r * dp - m * (m + 1.0L) * p) / (1.0L - r * r); /* P_m'' */
            long double dr = dp / ddp;
            r -= dr;
            if (fabsl(dr) < 1e-30L) break;
         }
         x[i] = r;
      }
      for (int i = 0; i < n; ++i)
      {
         long double p, pm1;
         legendre_eval(m, x[i], &p, &pm1);
         w[i] = 2.0L / ((long double)n * m * p * p);
      }
   }
   /* map to [0,1], ascending */
   long double pairs[MAXN][2];
   for (int i = 0; i < npts; ++i) { pairs[i][0] = 0.5L * (x[i] + 1.0L); pairs[i][1] = 0.5L * w[i]; }
   qsort(pairs, (size_t)npts, sizeof(pairs[0]), cmp_ld);
   for (int i = 0; i < npts; ++i) { coords[i] = (double)pairs[i][0]; weights[i] = (double)pairs[i][1]; }
   if (kind == 0) { coords[0] = 0.0; coords[npts - 1] = 1.0; }
   return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* FillRandom (Algebra/vector.hpp:632-647): std::mt19937(seed) feeding libstdc++'s             */
/* uniform_real_distribution<double>, whose canonical draw takes two 32-bit outputs:           */
/* r = (g0 + g1 * 2^32) / 2^64 (clamped below 1), value = r * (hi - lo) + lo.                   */
/* ------------------------------------------------------------------------------------------ */

typedef struct { uint32_t s[624]; int i; } mt_state;

static void mt_seed(mt_state *m, uint32_t seed)
{
   m->s[0] = seed;
   for (int i = 1; i < 624; ++i) m->s[i] = 1812433253u * (m->s[i - 1] ^ (m->s[i - 1] >> 30)) + (uint32_t)i;
   m->i = 624;
}

static uint32_t mt_next(mt_state *m)
{
   if (m->i >= 624)
   {
      for (int k = 0; k < 624; ++k)
      {
         uint32_t y = (m->s[k] & 0x80000000u) | (m->s[(k + 1) % 624] & 0x7fffffffu);
         uint32_t v = m->s[(k + 397) % 624] ^ (y >> 1);
         if (y & 1u) v ^= 0x9908b0dfu;
         m->s[k] = v;
      }
      m->i = 0;
   }
   uint32_t y = m->s[m->i++];
   y ^= y >> 11;
   y ^= (y << 7) & 0x9d2c5680u;
   y ^= (y << 15) & 0xefc60000u;
   y ^= y >> 18;
   return y;
}

void dgo_fill_random(double *out, long n, unsigned seed, double lo, double hi)
{
   mt_state m;
   mt_seed(&m, seed);
   for (long i = 0; i < n; ++i)
   {
      double sum = (double)mt_next(&m);
      sum += (double)mt_next(&m) * 4294967296.0;
      double r = sum / 18446744073709551616.0;
      if (r >= 1.0) r = nextafter(1.0, 0.0);
      out[i] = r * (hi - lo) + lo;
   }
}

/* ------------------------------------------------------------------------------------------ */
/* Space: Cartesian mesh (cartesianndmesh.hpp:16), tensor Lagrange element and GL rule.        */
/* ------------------------------------------------------------------------------------------ */

typedef struct
{
   int D, n, q, basis;
   long sizes[MAXD];
   double h[MAXD], origin[MAXD];
   int periodic[MAXD];
   long nelem, nd, nq;
   double xq[MAXN], wq[MAXN];     /* GL quadrature on [0,1] */
   double xn[MAXN];               /* basis nodes */
   double B[MAXN][MAXN];          /* B[qp][dof] = l_dof(x_qp)           doftoquad.hpp:133-137 */
   double Dq[MAXN][MAXN];         /* Dq[i][j] = l^GL_j'(x_i), collocated doftoquad.hpp:142-150 */
   double Bf[2][MAXN];            /* basis values at 0 and 1 (face rules, zeropoint/onepoint) */
} space_t;

/* lagrangeshapefunctions.hpp:37 */
static double lagrange_value(const double *nodes, int n, int j, double x)
{
   double num = 1.0, den = 1.0;
   for (int i = 0; i < n; ++i)
      if (i != j) { num *= (x - nodes[i]); den *= (nodes[j] - nodes[i]); }
   return num / den;
}

/* lagrangeshapefunctions.hpp:60 */
static double lagrange_grad(const double *nodes, int n, int j, double x)
{
   double sum = 0.0;
   for (int i = 0; i < n; ++i)
   {
      if (i == j) continue;
      double num = 1.0, den = nodes[j] - nodes[i];
      for (int k = 0; k < n; ++k)
         if (k != i && k != j) { num *= (x - nodes[k]); den *= (nodes[j] - nodes[k]); }
      sum += num / den;
   }
   return sum;
}

static int space_init(space_t *s, int D, int P, int Q, int basis, const long *sizes, const double *h,
                      const double *origin, const int *periodic)
{
   if (D < 1 || D > MAXD || P < 0 || P + 1 > MAXN || Q < 1 || Q > MAXN || (basis != 0 && basis != 1)) return -1;
   memset(s, 0, sizeof(*s));
   s->D = D; s->n = P + 1; s->q = Q; s->basis = basis;
   s->nelem = 1; s->nd = 1; s->nq = 1;
   for (int a = 0; a < D; ++a)
   {
      if (sizes[a] < 1) return -1;
      s->sizes[a] = sizes[a]; s->h[a] = h[a]; s->origin[a] = origin[a];
      s->periodic[a] = periodic ? periodic[a] : 0;
      s->nelem *= sizes[a]; s->nd *= s->n; s->nq *= Q;
   }
   double wn[MAXN];
   dgo_points(1, Q, s->xq, s->wq);
   dgo_points(basis == 0 ? 0 : 1, s->n, s->xn, wn);
   for (int qq = 0; qq < Q; ++qq)
      for (int j = 0; j < s->n; ++j) s->B[qq][j] = lagrange_value(s->xn, s->n, j, s->xq[qq]);
   for (int i = 0; i < Q; ++i)
      for (int j = 0; j < Q; ++j) s->Dq[i][j] = lagrange_grad(s->xq, Q, j, s->xq[i]);
   for (int j = 0; j < s->n; ++j)
   {
      s->Bf[0][j] = lagrange_value(s->xn, s->n, j, 0.0);
      s->Bf[1][j] = lagrange_value(s->xn, s->n, j, 1.0);
   }
   return 0;
}

static void element_index(const space_t *s, long e, long *idx)
{
   for (int a = 0; a < s->D; ++a) { idx[a] = e % s->sizes[a]; e /= s->sizes[a]; }
}

static long linear_index(const space_t *s, const long *idx)
{
   long e = 0;
   for (int a = s->D - 1; a >= 0; --a) e = e * s->sizes[a] + idx[a];
   return e;
}

/* Neighbour across face f (cartesianndmesh.hpp:109-198); returns -1 on a boundary face. */
static long neighbour(const space_t *s, long e, int f)
{
   long idx[MAXD];
   element_index(s, e, idx);
   const int a = f % s->D, sign = f < s->D ? -1 : 1;
   const long n = s->sizes[a];
   if (n == 1) { if (!s->periodic[a]) return -1; idx[a] = 0; }
   else if (sign < 0) { if (idx[a] == 0) { if (!s->periodic[a]) return -1; idx[a] = n - 1; } else idx[a]--; }
   else { if (idx[a] == n - 1) { if (!s->periodic[a]) return -1; idx[a] = 0; } else idx[a]++; }
   return linear_index(s, idx);
}

/* ------------------------------------------------------------------------------------------ */
/* Tensor contractions (interpolatevaluesserial.hpp:25-158, applytestfunctionsserial.hpp:26-56, */
/* applygradienttestfunctionsthreaded.hpp:20-100).  Tensors are FIFO, axis 0 fastest.          */
/* ------------------------------------------------------------------------------------------ */

/* out(.., j, ..) = sum_i M[j*ldm + i] in(.., i, ..) along axis k; dims updated in place. */
static void contract(int D, int *dims, int k, int mout, const double *M, int ldm, const double *in, double *out)
{
   long inner = 1, outer = 1;
   for (int a = 0; a < k; ++a) inner *= dims[a];
   for (int a = k + 1; a < D; ++a) outer *= dims[a];
   const int nin = dims[k];
   for (long o = 0; o < outer; ++o)
      for (int j = 0; j < mout; ++j)
         for (long t = 0; t < inner; ++t)
         {
            double sum = 0.0;
            for (int i = 0; i < nin; ++i) sum += M[j * ldm + i] * in[(o * nin + i) * inner + t];
            out[(o * mout + j) * inner + t] = sum;
         }
   dims[k] = mout;
}

typedef struct { double fwd[MAXN * MAXN]; double adj[MAXN * MAXN]; } mats_t;

/* Per axis: forward (q x n) and adjoint (n x q) matrices for a given row set. */
static void cell_mats(const space_t *s, mats_t *m)
{
   for (int qq = 0; qq < s->q; ++qq)
      for (int j = 0; j < s->n; ++j) { m->fwd[qq * s->n + j] = s->B[qq][j]; m->adj[j * s->q + qq] = s->B[qq][j]; }
}

/* B along every axis: nodal n^D -> q^D (or face: axis `fa` evaluated at the end `fend`). */
static void interpolate(const space_t *s, int fa, int fend, const double *u, double *out, double *w1, double *w2)
{
   int dims[MAXD];
   for (int a = 0; a < s->D; ++a) dims[a] = s->n;
   const double *src = u;
   double *bufs[2] = { w1, w2 };
   int which = 0;
   mats_t m;
   cell_mats(s, &m);
   for (int a = 0; a < s->D; ++a)
   {
      double *dst = (a == s->D - 1) ? out : bufs[which];
      if (a == fa) contract(s->D, dims, a, 1, s->Bf[fend], s->n, src, dst);
      else contract(s->D, dims, a, s->q, m.fwd, s->n, src, dst);
      src = dst;
      which ^= 1;
   }
}

/* B^T along every axis: q^D (or face shape) -> n^D, added into y. */
static void apply_test_add(const space_t *s, int fa, int fend, const double *in, double *y, double *w1, double *w2)
{
   int dims[MAXD];
   for (int a = 0; a < s->D; ++a) dims[a] = (a == fa) ? 1 : s->q;
   const double *src = in;
   double *bufs[2] = { w1, w2 };
   int which = 0;
   mats_t m;
   cell_mats(s, &m);
   double bft[MAXN];
   if (fa >= 0) for (int j = 0; j < s->n; ++j) bft[j] = s->Bf[fend][j];
   for (int a = 0; a < s->D; ++a)
   {
      double *dst = bufs[which];
      if (a == fa) contract(s->D, dims, a, s->n, bft, 1, src, dst);
      else contract(s->D, dims, a, s->n, m.adj, s->q, src, dst);
      src = dst;
      which ^= 1;
   }
   for (long i = 0; i < s->nd; ++i) y[i] += src[i];
}

/* ------------------------------------------------------------------------------------------ */
/* Coefficient presets, evaluated pointwise like the reference's lambdas.                      */
/* ------------------------------------------------------------------------------------------ */

static double sigma_eval(int D, int kind, double c, const double *X)
{
   if (kind == DGO_SIGMA_CONST) return c;
   if (kind == DGO_SIGMA_SEP) return (1.0 + 0.5 * X[0]) * (1.0 + X[1 % D] * X[1 % D]) * (2.0 - X[2 % D]);
   return 1.0 + X[0] * X[1 % D] + X[D - 1] * X[D - 1];
}

static void beta_eval(int D, int kind, const double *c, const double *X, double *v)
{
   for (int i = 0; i < D; ++i)
   {
      if (kind == DGO_BETA_CONST) v[i] = c[i];
      else if (kind == DGO_BETA_BUBBLE) v[i] = -X[i] * (1.0 - X[i]);
      else if (kind == DGO_BETA_SINCOS)
      {
         if (i == 0) v[i] = 1.0 + 0.5 * sin(2.0 * M_PI * X[1 % D]);
         else if (i == 1) v[i] = 0.5 + 0.25 * cos(2.0 * M_PI * X[2 % D]);
         else v[i] = 0.25;
      }
      else
      {
         const int H = D / 2;
         v[i] = (i < H) ? X[i + H] : -X[i - H] + 0.5;
      }
   }
}

/* multi-index of a flat FIFO index with all extents = ext except axis fa (extent 1) */
static void unflatten(int D, long flat, int ext, int fa, int *qi)
{
   for (int a = 0; a < D; ++a)
   {
      if (a == fa) { qi[a] = 0; continue; }
      qi[a] = (int)(flat % ext);
      flat /= ext;
   }
}

/* ------------------------------------------------------------------------------------------ */
/* Operators                                                                                    */
/* ------------------------------------------------------------------------------------------ */

typedef struct
{
   double *u, *bu, *tmp1, *tmp2, *acc, *grad[MAXD], *gt, *nb, *fu, *fnb;
} work_t;

static int work_alloc(const space_t *s, work_t *w)
{
   long big = s->nd > s->nq ? s->nd : s->nq;
   /* intermediate shapes mix n and q extents: bound by max(n,q)^D */
   long m = 1;
   int e = s->n > s->q ? s->n : s->q;
   for (int a = 0; a < s->D; ++a) m *= e;
   if (m > big) big = m;
   double *pool = (double *)calloc((size_t)big * (8 + MAXD), sizeof(double));
   if (!pool) return -1;
   w->u = pool; w->bu = pool + big; w->tmp1 = pool + 2 * big; w->tmp2 = pool + 3 * big;
   w->acc = pool + 4 * big; w->gt = pool + 5 * big; w->nb = pool + 6 * big; w->fu = pool + 7 * big;
   for (int a = 0; a < MAXD; ++a) w->grad[a] = pool + (8 + a) * big;
   w->fnb = w->tmp1; /* reused after face interpolation of own trace is consumed */
   return 0;
}

static void work_free(work_t *w) { free(w->u); }

static double det_j(const space_t *s)
{
   double d = 1.0;
   for (int a = 0; a < s->D; ++a) d *= s->h[a];
   return d;
}

/* Cell mass contribution y_e = B^T (w detJ sigma B u)  (massoperator.hpp:53-88). */
static void mass_cell(const space_t *s, long e, const long *idx, int sigma_kind, double sigma_c,
                      const double *u, double *ye, work_t *w)
{
   interpolate(s, -1, 0, u, w->bu, w->tmp1, w->tmp2);
   const double detJ = det_j(s);
   int qi[MAXD];
   double X[MAXD];
   for (long t = 0; t < s->nq; ++t)
   {
      unflatten(s->D, t, s->q, -1, qi);
      double weight = 1.0;
      for (int a = 0; a < s->D; ++a)
      {
         X[a] = (s->origin[a] + s->h[a] * (double)idx[a]) + s->h[a] * s->xq[qi[a]];
         weight *= s->wq[qi[a]];
      }
      w->bu[t] = weight * detJ * sigma_eval(s->D, sigma_kind, sigma_c, X) * w->bu[t];
   }
   (void)e;
   apply_test_add(s, -1, 0, w->bu, ye, w->tmp1, w->tmp2);
}

/* Cell advection term y_e += B^T sum_i Dq_i^T (-w detJ (J^-T beta)_i B u)  (advectionoperator.hpp:125-166). */
static void advection_cell(const space_t *s, const long *idx, int beta_kind, const double *beta_c,
                           int sigma_kind, double sigma_c, int with_mass, const double *u, double *ye, work_t *w)
{
   interpolate(s, -1, 0, u, w->bu, w->tmp1, w->tmp2);
   const double detJ = det_j(s);
   int qi[MAXD];
   double X[MAXD], b[MAXD];
   for (long t = 0; t < s->nq; ++t)
   {
      unflatten(s->D, t, s->q, -1, qi);
      double weight = 1.0;
      for (int a = 0; a < s->D; ++a)
      {
         X[a] = (s->origin[a] + s->h[a] * (double)idx[a]) + s->h[a] * s->xq[qi[a]];
         weight *= s->wq[qi[a]];
      }
      beta_eval(s->D, beta_kind, beta_c, X, b);
      const double buq = w->bu[t];
      const double wq = -weight * detJ * buq;
      for (int a = 0; a < s->D; ++a) w->grad[a][t] = wq * (b[a] * (1.0 / s->h[a]));
      /* massadvectionoperator.hpp: Du_q_w = weight * detJ * (sigma * Bu_q) */
      w->acc[t] = with_mass ? weight * detJ * (sigma_eval(s->D, sigma_kind, sigma_c, X) * buq) : 0.0;
   }
   /* collocated G^T at quadrature points, summed over components */
   for (long t = 0; t < s->nq; ++t) w->gt[t] = 0.0;
   double dqt[MAXN * MAXN];
   for (int qq = 0; qq < s->q; ++qq)
      for (int p = 0; p < s->q; ++p) dqt[qq * s->q + p] = s->Dq[p][qq];
   for (int a = 0; a < s->D; ++a)
   {
      int dims[MAXD];
      for (int k = 0; k < s->D; ++k) dims[k] = s->q;
      contract(s->D, dims, a, s->q, dqt, s->q, w->grad[a], w->tmp1);
      for (long t = 0; t < s->nq; ++t) w->gt[t] += w->tmp1[t];
   }
   if (with_mass)
      for (long t = 0; t < s->nq; ++t) w->gt[t] += w->acc[t];
   apply_test_add(s, -1, 0, w->gt, ye, w->tmp1, w->tmp2);
}

/* Face f of element e (advectionoperator.hpp:339-438): upwind flux with the neighbour trace, or
 * with the inflow value g on a boundary face. */
static void advection_face(const space_t *s, const long *idx, int f, const double *u, const double *unb,
                           int beta_kind, const double *beta_c, double g, double *ye, work_t *w)
{
   const int D = s->D, a = f % D, sign = f < D ? -1 : 1;
   const int own_end = sign < 0 ? 0 : 1;
   interpolate(s, a, own_end, u, w->fu, w->tmp1, w->tmp2);
   long nfq = 1;
   for (int k = 0; k < D; ++k) if (k != a) nfq *= s->q;
   if (unb) interpolate(s, a, 1 - own_end, unb, w->nb, w->tmp1, w->tmp2);
   const double detJ = det_j(s);
   int qi[MAXD];
   double X[MAXD], b[MAXD];
   for (long t = 0; t < nfq; ++t)
   {
      unflatten(D, t, s->q, a, qi);
      double weight = 1.0;
      for (int k = 0; k < D; ++k)
      {
         const double xh = (k == a) ? (double)own_end : s->xq[qi[k]];
         X[k] = (s->origin[k] + s->h[k] * (double)idx[k]) + s->h[k] * xh;
         if (k != a) weight *= s->wq[qi[k]];
      }
      beta_eval(D, beta_kind, beta_c, X, b);
      const double dot = b[a] * ((double)sign * (1.0 / s->h[a]));
      const double other = unb ? w->nb[t] : g;
      const double upwind = dot > 0.0 ? dot * w->fu[t] : dot * other;
      w->fu[t] = weight * detJ * upwind;
   }
   apply_test_add(s, a, own_end, w->fu, ye, w->tmp1, w->tmp2);
}

int dgo_mass_apply(int D, int P, int Q, int basis, const long *sizes, const double *h,
                   const double *origin, const int *periodic, int sigma_kind, double sigma_c,
                   const double *x, double *y)
{
   space_t s;
   if (space_init(&s, D, P, Q, basis, sizes, h, origin, periodic)) return -1;
   work_t w;
   if (work_alloc(&s, &w)) return -2;
   long idx[MAXD];
   for (long e = 0; e < s.nelem; ++e)
   {
      element_index(&s, e, idx);
      double *ye = y + e * s.nd;
      memset(ye, 0, sizeof(double) * (size_t)s.nd);
      mass_cell(&s, e, idx, sigma_kind, sigma_c, x + e * s.nd, ye, &w);
   }
   work_free(&w);
   return 0;
}

int dgo_advection_apply(int D, int P, int Q, int basis, const long *sizes, const double *h,
                        const double *origin, const int *periodic, int mode, int beta_kind,
                        const double *beta_c, double g, int sigma_kind, double sigma_c,
                        const double *x, double *y)
{
   space_t s;
   if (space_init(&s, D, P, Q, basis, sizes, h, origin, periodic)) return -1;
   work_t w;
   if (work_alloc(&s, &w)) return -2;
   long idx[MAXD];
   for (long e = 0; e < s.nelem; ++e)
   {
      element_index(&s, e, idx);
      double *ye = y + e * s.nd;
      const double *ue = x + e * s.nd;
      memset(ye, 0, sizeof(double) * (size_t)s.nd);
      advection_cell(&s, idx, beta_kind, beta_c, sigma_kind, sigma_c, mode == DGO_MASS_ADV, ue, ye, &w);
      for (int f = 0; f < 2 * D; ++f)
      {
         const long nb = neighbour(&s, e, f);
         if (nb < 0 && mode != DGO_ADV_INFLOW) continue;
         advection_face(&s, idx, f, ue, nb >= 0 ? x + nb * s.nd : NULL, beta_kind, beta_c, g, ye, &w);
      }
   }
   work_free(&w);
   return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* Krylov solvers                                                                               */
/* ------------------------------------------------------------------------------------------ */

static double vdot(long n, const double *a, const double *b)
{
   double s = 0.0;
   for (long i = 0; i < n; ++i) s += a[i] * b[i];
   return s;
}

static void vaxpy(long n, double a, const double *x, double *y)
{
   for (long i = 0; i < n; ++i) y[i] = y[i] + a * x[i];
}

int dgo_mass_cg(int D, int P, int Q, int basis, const long *sizes, const double *h,
                const double *origin, const int *periodic, int sigma_kind, double sigma_c,
                const double *b, double *x, int max_iters, double tol, int *iters, double *rel,
                int *success)
{
   space_t s;
   if (space_init(&s, D, P, Q, basis, sizes, h, origin, periodic)) return -1;
   const long n = s.nelem * s.nd;
   double *tmp = (double *)malloc(sizeof(double) * (size_t)n * 3);
   if (!tmp) return -2;
   double *r = tmp + n, *p = tmp + 2 * n;
#define APPLY(in, out) dgo_mass_apply(D, P, Q, basis, sizes, h, origin, periodic, sigma_kind, sigma_c, in, out)
   /* conjugategradient.hpp:143-149: the "rhs norm" is the norm of the initial residual */
   APPLY(x, tmp);
   for (long i = 0; i < n; ++i) r[i] = b[i] - tmp[i];
   const double rhs_n = sqrt(vdot(n, r, r));
   if (rhs_n == 0.0 || rhs_n < 1e-30)
   {
      memset(x, 0, sizeof(double) * (size_t)n);
      *iters = 0; *rel = 0.0; *success = 1;
      free(tmp);
      return 0;
   }
   double r_n = sqrt(vdot(n, r, r));
   if (r_n < tol * rhs_n) { *iters = 0; *rel = sqrt(r_n / rhs_n); *success = 1; free(tmp); return 0; }
   memcpy(p, r, sizeof(double) * (size_t)n);
   double abs_new = vdot(n, r, p);
   int iter = 0;
   while (iter < max_iters)
   {
      APPLY(p, tmp);
      const double alpha = abs_new / vdot(n, p, tmp);
      vaxpy(n, alpha, p, x);
      vaxpy(n, -alpha, tmp, r);
      r_n = sqrt(vdot(n, r, r));
      if (r_n < tol * rhs_n)
      {
         /* conjugategradient.hpp:188: iterations = iter + 1, error = sqrt(|r| / |r0|) */
         *iters = iter + 1; *rel = sqrt(r_n / rhs_n); *success = 1;
         free(tmp);
         return 0;
      }
      const double abs_old = abs_new;
      abs_new = vdot(n, r, r);
      const double beta = abs_new / abs_old;
      for (long i = 0; i < n; ++i) p[i] = p[i] * beta + r[i];
      ++iter;
   }
#undef APPLY
   *iters = iter; *rel = sqrt(r_n / rhs_n); *success = 0;
   free(tmp);
   return 0;
}

typedef struct
{
   int D, P, Q, basis;
   const long *sizes;
   const double *h, *origin;
   const int *periodic;
   double sigma_c;
   int beta_kind;
   const double *beta_c;
   double g;
   double *tmp;
} sys_t;

static void sys_apply(const sys_t *S, const double *in, double *out, long n)
{
   dgo_mass_apply(S->D, S->P, S->Q, S->basis, S->sizes, S->h, S->origin, S->periodic, DGO_SIGMA_CONST, S->sigma_c, in, out);
   dgo_advection_apply(S->D, S->P, S->Q, S->basis, S->sizes, S->h, S->origin, S->periodic, DGO_ADV_INFLOW,
                       S->beta_kind, S->beta_c, S->g, DGO_SIGMA_CONST, 0.0, in, S->tmp);
   for (long i = 0; i < n; ++i) out[i] += S->tmp[i];
}

int dgo_system_gmres(int D, int P, int Q, int basis, const long *sizes, const double *h,
                     const double *origin, const int *periodic, double sigma_c, int beta_kind,
                     const double *beta_c, double g, const double *b, double *x, int max_iters,
                     int restart, double tol, int *iters, double *rel, int *success)
{
   space_t s;
   if (space_init(&s, D, P, Q, basis, sizes, h, origin, periodic)) return -1;
   const long n = s.nelem * s.nd;
   const int m = restart;
   double *pool = (double *)malloc(sizeof(double) * (size_t)n * (size_t)(m + 3));
   double *H = (double *)calloc((size_t)(m + 1) * (size_t)(m > 0 ? m : 1), sizeof(double));
   double *cs = (double *)calloc((size_t)m + 1, sizeof(double)), *sn = (double *)calloc((size_t)m + 1, sizeof(double));
   double *e1 = (double *)calloc((size_t)m + 2, sizeof(double)), *yv = (double *)calloc((size_t)m + 1, sizeof(double));
   if (!pool || !H || !cs || !sn || !e1 || !yv) return -2;
   double *w = pool, *tmp = pool + n, *V = pool + 2 * n;
   sys_t S = { D, P, Q, basis, sizes, h, origin, periodic, sigma_c, beta_kind, beta_c, g, tmp };
   const double eps = 2.220446049250313e-16;
#define HH(i, j) H[(j) * (m + 1) + (i)]
#define VV(i) (V + (long)(i) * n)
   /* gmres.hpp:96-104 */
#define RESIDUAL_IN_V0() (sys_apply(&S, x, w, n), memcpy(VV(0), b, sizeof(double) * (size_t)n), \
                          vaxpy(n, -1.0, w, VV(0)), sqrt(vdot(n, VV(0), VV(0))))
   int rc_iters = 0, rc_success = 0;
   double rc_rel = 0.0;
   const double norm_rhs = sqrt(vdot(n, b, b));
   const double denom = norm_rhs > 0.0 ? norm_rhs : 1.0;
   if (max_iters <= 0 || m <= 0)
   {
      double rn = RESIDUAL_IN_V0();
      rc_success = rn / denom <= tol; rc_iters = 0; rc_rel = rn / denom;
      goto done;
   }
   {
      double beta = RESIDUAL_IN_V0();
      double rel_res = beta / denom;
      if (rel_res <= tol) { rc_success = 1; rc_iters = 0; rc_rel = rel_res; goto done; }
      int total = 0;
      while (total < max_iters)
      {
         for (long i = 0; i < n; ++i) VV(0)[i] *= (1.0 / beta);
         for (int i = 0; i < m; ++i) { cs[i] = 1.0; sn[i] = 0.0; yv[i] = 0.0; }
         for (int i = 0; i <= m; ++i) e1[i] = 0.0;
         e1[0] = beta;
         int k = 0;
         for (int j = 0; j < m && total < max_iters; ++j)
         {
            ++total;
            sys_apply(&S, VV(j), w, n);
            for (int i = 0; i <= j; ++i)
            {
               const double hij = vdot(n, VV(i), w);
               HH(i, j) = hij;
               vaxpy(n, -hij, VV(i), w);
            }
            const double h_next = sqrt(vdot(n, w, w));
            HH(j + 1, j) = h_next;
            for (int i = 0; i < j; ++i)
            {
               const double him = HH(i, j), hip = HH(i + 1, j);
               HH(i, j) = cs[i] * him + sn[i] * hip;
               HH(i + 1, j) = -sn[i] * him + cs[i] * hip;
            }
            const double hmm = HH(j, j), hm1 = HH(j + 1, j);
            const double rho = sqrt(hmm * hmm + hm1 * hm1);
            if (rho <= eps * beta) { HH(j, j) = 0.0; HH(j + 1, j) = 0.0; k = j; break; }
            cs[j] = hmm / rho;
            sn[j] = hm1 / rho;
            HH(j, j) = rho;
            HH(j + 1, j) = 0.0;
            const double gm = e1[j], gm1 = e1[j + 1];
            e1[j] = cs[j] * gm + sn[j] * gm1;
            e1[j + 1] = -sn[j] * gm + cs[j] * gm1;
            k = j + 1;
            const double rel_est = fabs(e1[j + 1]) / denom;
            const int happy = h_next <= eps * beta;
            if (happy || rel_est <= tol) break;
            for (long i = 0; i < n; ++i) VV(j + 1)[i] = w[i] * (1.0 / h_next);
         }
         if (k == 0)
         {
            double rn = RESIDUAL_IN_V0();
            rc_success = rn / denom <= tol; rc_iters = total; rc_rel = rn / denom;
            goto done;
         }
         for (int i = k; i-- > 0;)
         {
            double sum = e1[i];
            for (int j = i + 1; j < k; ++j) sum -= HH(i, j) * yv[j];
            const double diag = HH(i, i);
            yv[i] = (fabs(diag) <= eps * beta) ? 0.0 : sum / diag;
         }
         for (int i = 0; i < k; ++i) vaxpy(n, yv[i], VV(i), x);
         beta = RESIDUAL_IN_V0();
         rel_res = beta / denom;
         if (rel_res <= tol) { rc_success = 1; rc_iters = total; rc_rel = rel_res; goto done; }
         if (total >= max_iters) { rc_success = 0; rc_iters = total; rc_rel = rel_res; goto done; }
      }
      {
         double rn = RESIDUAL_IN_V0();
         rc_success = rn / denom <= tol; rc_iters = total; rc_rel = rn / denom;
      }
   }
done:
#undef HH
#undef VV
#undef RESIDUAL_IN_V0
   *iters = rc_iters; *rel = rc_rel; *success = rc_success;
   free(pool); free(H); free(cs); free(sn); free(e1); free(yv);
   return 0;
}
