/* Test infrastructure only: the CPU oracle.  Nothing in the product links or calls this.
 *
 * A plain-C restatement of the GenDiL reference algorithms for the matrix-free DG mass and
 * upwind advection path, with the dimension, order and quadrature size as runtime values.
 * Each function cites the reference file:line it restates.  It is pinned against the
 * reference itself (oracle/_ref/libgendil_ref.so, built from the reference headers) by the
 * golden fixtures under tests/golden.
 *
 * Conventions (all as in the reference):
 *  - elements are numbered x-fastest (cartesianndmesh.hpp:95, getstructuredsubindex.hpp);
 *  - the DoF vector is element-major, each element block FIFO with axis 0 fastest
 *    (elementtensorview.hpp:42-48, L2Restriction restriction.hpp:38);
 *  - basis 0 = Gauss-Lobatto-Legendre nodes (MakeLobattoFiniteElement, finiteelement.hpp:109),
 *    basis 1 = Gauss-Legendre nodes (MakeLegendreFiniteElement, finiteelement.hpp:103);
 *    quadrature is always Gauss-Legendre (MakeIntegrationRule, integrationrule.hpp:80);
 *  - coefficient presets are evaluated pointwise, like the reference's user lambdas.
 */
#ifndef DG_ORACLE_H
#define DG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { DGO_SIGMA_CONST = 0, DGO_SIGMA_POLY = 1, DGO_SIGMA_SEP = 2 };
enum { DGO_BETA_CONST = 0, DGO_BETA_BUBBLE = 1, DGO_BETA_SINCOS = 2, DGO_BETA_PHASE = 3 };
enum { DGO_ADV_NO_BC = 0, DGO_ADV_INFLOW = 1, DGO_MASS_ADV = 2 };

/* 1D nodes/weights on [0,1]: kind 0 = GLL, kind 1 = GL, npts in 1..8. */
int dgo_points(int kind, int npts, double *coords, double *weights);

/* FillRandom (Algebra/vector.hpp:632): std::mt19937(seed) + uniform_real_distribution(lo, hi). */
void dgo_fill_random(double *out, long n, unsigned seed, double lo, double hi);

/* y = M_sigma x  (massoperator.hpp:39-89, :209). */
int dgo_mass_apply(int D, int P, int Q, int basis, const long *sizes, const double *h,
                   const double *origin, const int *periodic, int sigma_kind, double sigma_c,
                   const double *x, double *y);

/* y = A x: mode 0 = AdvectionFusedOperatorWithoutBC (advectionoperator.hpp:106),
 * 1 = AdvectionFusedOperatorWithBC with inflow value g (:269), 2 = MassAdvectionOperator
 * (massadvectionoperator.hpp:44,153). */
int dgo_advection_apply(int D, int P, int Q, int basis, const long *sizes, const double *h,
                        const double *origin, const int *periodic, int mode, int beta_kind,
                        const double *beta_c, double g, int sigma_kind, double sigma_c,
                        const double *x, double *y);

/* ConjugateGradient, scratch overload (conjugategradient.hpp:125-209) on the mass operator. */
int dgo_mass_cg(int D, int P, int Q, int basis, const long *sizes, const double *h,
                const double *origin, const int *periodic, int sigma_kind, double sigma_c,
                const double *b, double *x, int max_iters, double tol, int *iters, double *rel,
                int *success);

/* GMRES_no_alloc (gmres.hpp:74-289) on sigma*M + A(inflow g). */
int dgo_system_gmres(int D, int P, int Q, int basis, const long *sizes, const double *h,
                     const double *origin, const int *periodic, double sigma_c, int beta_kind,
                     const double *beta_c, double g, const double *b, double *x, int max_iters,
                     int restart, double tol, int *iters, double *rel, int *success);

#ifdef __cplusplus
}
#endif

#endif
