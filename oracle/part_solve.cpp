// Test infrastructure only (CPU oracle): reference Krylov solves on reference operators.
#include "ref_impl.hpp"
#include "ref_lists.hpp"

extern "C" int gref_mass_cg( int D, int P, int Q, int basis, const long * sizes, const double * h,
                             const double * origin, const int * periodic, int sigma_kind, double sigma_c,
                             const double * b, double * x, int max_iters, double tol, int * iters,
                             double * rel, int * success )
{
   gref::MeshArgs m{ sizes, h, origin, periodic };
#define X( d, p, q, bb ) \
   if ( D == d && P == p && Q == q && basis == bb ) { gref::MassCG< d, p, q, bb >( m, sigma_kind, sigma_c, b, x, max_iters, tol, iters, rel, success ); return 0; }
   GREF_CG_LIST( X )
#undef X
   return gref::GREF_UNSUPPORTED;
}

extern "C" int gref_system_gmres( int D, int P, int Q, int basis, const long * sizes, const double * h,
                                  const double * origin, const int * periodic, double sigma_c, int beta_kind,
                                  const double * beta_c, double g, const double * b, double * x, int max_iters,
                                  int restart, double tol, int * iters, double * rel, int * success )
{
   gref::MeshArgs m{ sizes, h, origin, periodic };
#define X( d, p, q, bb ) \
   if ( D == d && P == p && Q == q && basis == bb ) { gref::SystemGMRES< d, p, q, bb >( m, sigma_c, beta_kind, beta_c, g, b, x, max_iters, restart, tol, iters, rel, success ); return 0; }
   GREF_GMRES_LIST( X )
#undef X
   return gref::GREF_UNSUPPORTED;
}
