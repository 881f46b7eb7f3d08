// Test infrastructure only (CPU oracle): the C entry points of the reference-compiled library
// (libgendil_ref.so).  They dispatch to the instantiation lists in the part files and expose the
// reference's input generator and quadrature tables, so golden vectors come from the reference.
#include "ref_impl.hpp"

#include <omp.h>

extern "C" {

int gref_mass_part_A( int, int, int, int, const long *, const double *, const double *, const int *, int, double, const double *, double * );
int gref_mass_part_B( int, int, int, int, const long *, const double *, const double *, const int *, int, double, const double *, double * );
int gref_mass_part_C( int, int, int, int, const long *, const double *, const double *, const int *, int, double, const double *, double * );
int gref_mass_part_D( int, int, int, int, const long *, const double *, const double *, const int *, int, double, const double *, double * );
int gref_mass_part_E( int, int, int, int, const long *, const double *, const double *, const int *, int, double, const double *, double * );
#define GREF_ADV_DECL( P ) \
   int gref_adv_part_##P( int, int, int, int, const long *, const double *, const double *, const int *, int, int, const double *, double, int, double, const double *, double * );
GREF_ADV_DECL( A )
GREF_ADV_DECL( B )
GREF_ADV_DECL( C )
GREF_ADV_DECL( D )
GREF_ADV_DECL( E )
GREF_ADV_DECL( F )
GREF_ADV_DECL( G )
GREF_ADV_DECL( H )

int gref_mass_apply( int D, int P, int Q, int basis, const long * sizes, const double * h,
                     const double * origin, const int * periodic, int sigma_kind, double sigma_c,
                     const double * x, double * y )
{
   int rc = gref_mass_part_A( D, P, Q, basis, sizes, h, origin, periodic, sigma_kind, sigma_c, x, y );
   if ( rc != gref::GREF_UNSUPPORTED ) return rc;
   rc = gref_mass_part_B( D, P, Q, basis, sizes, h, origin, periodic, sigma_kind, sigma_c, x, y );
   if ( rc != gref::GREF_UNSUPPORTED ) return rc;
   rc = gref_mass_part_C( D, P, Q, basis, sizes, h, origin, periodic, sigma_kind, sigma_c, x, y );
   if ( rc != gref::GREF_UNSUPPORTED ) return rc;
   rc = gref_mass_part_D( D, P, Q, basis, sizes, h, origin, periodic, sigma_kind, sigma_c, x, y );
   if ( rc != gref::GREF_UNSUPPORTED ) return rc;
   return gref_mass_part_E( D, P, Q, basis, sizes, h, origin, periodic, sigma_kind, sigma_c, x, y );
}

// mode: 0 advection without boundary faces, 1 advection with inflow value g, 2 mass + advection.
int gref_advection_apply( int D, int P, int Q, int basis, const long * sizes, const double * h,
                          const double * origin, const int * periodic, int mode, int beta_kind,
                          const double * beta_c, double g, int sigma_kind, double sigma_c,
                          const double * x, double * y )
{
   int ( *parts[] )( int, int, int, int, const long *, const double *, const double *, const int *, int, int,
                     const double *, double, int, double, const double *, double * ) = {
      gref_adv_part_A, gref_adv_part_B, gref_adv_part_C, gref_adv_part_D, gref_adv_part_E,
      gref_adv_part_F, gref_adv_part_G, gref_adv_part_H };
   for ( auto part : parts )
   {
      const int rc = part( D, P, Q, basis, sizes, h, origin, periodic, mode, beta_kind, beta_c, g, sigma_kind, sigma_c, x, y );
      if ( rc != gref::GREF_UNSUPPORTED ) return rc;
   }
   return gref::GREF_UNSUPPORTED;
}

// Wall time per apply (seconds) of the reference advection operator with inflow value g,
// measured as in benchmarks/include/benchmark-common.hpp:278-298: warm-up, then op(x,y); op(y,x)
// pairs, mean per apply.  x and y are caller buffers of the space's size (x is overwritten).
double gref_time_advection( int D, int P, int Q, int basis, const long * sizes, const double * h,
                            const double * origin, int beta_kind, const double * beta_c, double g,
                            int pairs, double * x, double * y )
{
   double seconds = -1.0;
   auto run = [&]( auto dp, auto pp, auto qp )
   {
      constexpr int Dd = decltype( dp )::value, Pp = decltype( pp )::value, Qq = decltype( qp )::value;
      gref::MeshArgs m{ sizes, h, origin, nullptr };
      gref::WithSpace< Dd, Pp, Qq, 0 >( m, [&]( auto & fes, auto & ir )
      {
         auto beta = gref::MakeBeta< Dd >( beta_kind, beta_c );
         gref::BoundaryFn< Dd > bc{ g };
         auto op = gendil::MakeAdvectionOperator< gendil::SerialKernelConfiguration >( fes, ir, beta, bc );
         const size_t n = fes.GetNumberOfFiniteElementDofs();
         gendil::Vector vx( n ), vy( n );
         gref::CopyIn( vx, x );
         op( vx, vy );  // warm-up
         op( vy, vx );
         const double t0 = omp_get_wtime();
         for ( int k = 0; k < pairs; ++k )
         {
            op( vx, vy );
            op( vy, vx );
         }
         const double t1 = omp_get_wtime();
         seconds = ( t1 - t0 ) / ( 2.0 * pairs );
         gref::CopyOut( vy, y );
      } );
   };
   if ( basis != 0 ) return -1.0;
   if ( D == 3 && P == 3 && Q == 4 ) run( std::integral_constant< int, 3 >{}, std::integral_constant< int, 3 >{}, std::integral_constant< int, 4 >{} );
   // the 6D phase-space configuration (p = 2, q = 3)
   if ( D == 6 && P == 2 && Q == 3 ) run( std::integral_constant< int, 6 >{}, std::integral_constant< int, 2 >{}, std::integral_constant< int, 3 >{} );
   return seconds;
}

int gref_num_threads( void )
{
   return omp_get_max_threads();
}

// FillRandom (Algebra/vector.hpp:632) into a caller buffer.
void gref_fill_random( double * out, long n, unsigned seed, double lo, double hi )
{
   gendil::Vector v( (size_t)n );
   gendil::FillRandom( v, seed, lo, hi );
   gref::CopyOut( v, out );
}

// The reference's hard-coded 1D node/weight tables: kind 0 = Gauss-Lobatto-Legendre,
// kind 1 = Gauss-Legendre, both on [0,1] (NumericalIntegration/QuadraturePoints/GL*points.hpp).
int gref_points( int kind, int npts, double * coords, double * weights )
{
   using namespace gendil;
   auto fill = [&]( auto pts )
   {
      using T = decltype( pts );
      for ( int i = 0; i < npts; ++i )
      {
         coords[ i ] = T::GetCoord( i );
         weights[ i ] = T::GetWeight( i );
      }
   };
#define GREF_PTS( K ) \
   if ( npts == K ) { if ( kind == 0 ) fill( GaussLobattoLegendrePoints< K >{} ); else fill( GaussLegendrePoints< K >{} ); return 0; }
   GREF_PTS( 1 ) GREF_PTS( 2 ) GREF_PTS( 3 ) GREF_PTS( 4 ) GREF_PTS( 5 ) GREF_PTS( 6 ) GREF_PTS( 7 ) GREF_PTS( 8 )
#undef GREF_PTS
   return gref::GREF_UNSUPPORTED;
}

}  // extern "C"
