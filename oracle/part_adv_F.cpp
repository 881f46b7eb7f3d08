// Test infrastructure only (CPU oracle): reference advection-operator instantiations, list F.
#include "ref_impl.hpp"
#include "ref_lists.hpp"

extern "C" int gref_adv_part_F( int D, int P, int Q, int basis, const long * sizes, const double * h,
                                   const double * origin, const int * periodic, int mode, int beta_kind,
                                   const double * beta_c, double g, int sigma_kind, double sigma_c,
                                   const double * x, double * y )
{
   gref::MeshArgs m{ sizes, h, origin, periodic };
#define X( d, p, q, b ) \
   if ( D == d && P == p && Q == q && basis == b ) { gref::AdvectionApply< d, p, q, b >( m, mode, beta_kind, beta_c, g, sigma_kind, sigma_c, x, y ); return 0; }
   GREF_ADV_LIST_F( X )
#undef X
   return gref::GREF_UNSUPPORTED;
}
