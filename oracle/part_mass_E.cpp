// Test infrastructure only (CPU oracle): reference mass-operator instantiations, list E.
#include "ref_impl.hpp"
#include "ref_lists.hpp"

extern "C" int gref_mass_part_E( int D, int P, int Q, int basis, const long * sizes, const double * h,
                                    const double * origin, const int * periodic, int sigma_kind,
                                    double sigma_c, const double * x, double * y )
{
   gref::MeshArgs m{ sizes, h, origin, periodic };
#define X( d, p, q, b ) \
   if ( D == d && P == p && Q == q && basis == b ) { gref::MassApply< d, p, q, b >( m, sigma_kind, sigma_c, x, y ); return 0; }
   GREF_MASS_LIST_E( X )
#undef X
   return gref::GREF_UNSUPPORTED;
}
