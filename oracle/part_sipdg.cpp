// Test infrastructure only (CPU oracle): the reference's generic SIPDG diffusion weak form
// (README.md "Weak Form DSL", tests/integration/gendil/test-sipdg-coefficient-field-inputs.cpp:
// 547-575): mu a finite-element field (here constant on each element: every node of element e
// holds mu_e), tau = kappa * InverseFacetSize, sigma = -1 (SIPG), +1 (NIPG) or 0 (IIPG), and
// optionally the Dirichlet-0 boundary terms of the README form with the same sigma.
#include "ref_impl.hpp"

namespace gref {

template < int D, int P, int Q, int Basis >
void SipdgApply( const MeshArgs & m, const double * mu_elem, double sigma, double kappa, int boundary,
                 const double * x, double * y )
{
   WithSpace< D, P, Q, Basis >( m, [&]( auto & fes, auto & ir )
   {
      const size_t n = fes.GetNumberOfFiniteElementDofs();
      const size_t ne = fes.GetNumberOfFiniteElements();
      const size_t nd = n / ne;
      Vector vx( n ), vy( n ), vmu( n );
      CopyIn( vx, x );
      Real * md = vmu.WriteHostData();
      for ( size_t e = 0; e < ne; ++e )
         for ( size_t i = 0; i < nd; ++i ) md[ e * nd + i ] = mu_elem[ e ];
      auto mu_view = MakeReadOnlyElementTensorView< SerialKernelConfiguration >( fes, vmu );
      TrialSpace< "u" > u;
      TestSpace< "u" > v;
      Cells< "mesh" > cells;
      InteriorFacets< "mesh" > interior_facets;
      BoundaryFacets< "mesh" > boundary_facets;
      auto mu = MakeCoefficient< "diffusivity", FieldValue< "mu" > >(
         [] GENDIL_HOST_DEVICE ( const Real mu_q ) -> Real { return mu_q; } );
      auto tau = MakeCoefficient< "penalty", InverseFacetSize >(
         [=] GENDIL_HOST_DEVICE ( const Real h_inv ) -> Real { return kappa * h_inv; } );
      auto interior = integrate( cells, mu * dot( grad( u ), grad( v ) ) ) +
                      integrate( interior_facets,
                                 - average( mu * dot( grad( u ), Normal{} ) ) * jump( v )
                                 + sigma * jump( u ) * average( mu * dot( grad( v ), Normal{} ) )
                                 + tau * average( mu ) * jump( u ) * jump( v ) );
      auto ctx = MakeWeakFormContext( MakeTrialField< "u" >( fes ), MakeFiniteElementField< "mu" >( fes, mu_view ),
                                      MakeIntegrationDomain< "mesh" >( fes ) );
      vy = 0.0;
      if ( boundary )
      {
         auto form = interior + integrate( boundary_facets,
                                           - mu * dot( grad( u ), Normal{} ) * v
                                           + sigma * u * mu * dot( grad( v ), Normal{} )
                                           + tau * mu * u * v );
         auto op = MakeGenericOperator< SerialKernelConfiguration >( form, ctx, ir );
         op( vx, vy );
      }
      else
      {
         auto op = MakeGenericOperator< SerialKernelConfiguration >( interior, ctx, ir );
         op( vx, vy );
      }
      CopyOut( vy, y );
   } );
}

// The reference's legacy SIPDG operator, MakeDiffusionOperator<KP>(fes, ir, velocity, sigma, kappa)
// (FiniteElementMethod/MatrixFreeOperators/diffusionoperator.hpp:554): cell term, interior faces
// and boundary faces, with a constant diffusivity `d` as the `velocity` function of X.
template < int D, int P, int Q, int Basis >
void DiffusionLegacyApply( const MeshArgs & m, double d, double sigma, double kappa, const double * x, double * y )
{
   WithSpace< D, P, Q, Basis >( m, [&]( auto & fes, auto & ir )
   {
      const size_t n = fes.GetNumberOfFiniteElementDofs();
      Vector vx( n ), vy( n );
      CopyIn( vx, x );
      auto diffusivity = [=] GENDIL_HOST_DEVICE ( std::array< Real, D > const & ) -> Real { return d; };
      auto op = MakeDiffusionOperator< SerialKernelConfiguration >( fes, ir, diffusivity, sigma, kappa );
      vy = 0.0;
      op( vx, vy );
      CopyOut( vy, y );
   } );
}

}  // namespace gref

// (dimension, order, points, basis: 0 GLL, 1 GL)
#define GREF_SIPDG_LIST( X )                                                                          \
   X( 1, 1, 4, 0 ) X( 2, 1, 3, 0 ) X( 2, 2, 4, 0 ) X( 3, 1, 3, 0 ) X( 3, 2, 4, 0 ) X( 3, 3, 5, 0 ) \
   X( 3, 4, 6, 0 ) X( 2, 2, 4, 1 ) X( 3, 2, 4, 1 ) X( 4, 1, 3, 0 )

extern "C" int gref_sipdg_apply( int D, int P, int Q, int basis, const long * sizes, const double * h,
                                 const double * origin, const int * periodic, const double * mu_elem, double sigma,
                                 double kappa, int boundary, const double * x, double * y )
{
   gref::MeshArgs m{ sizes, h, origin, periodic };
#define X( d, p, q, b )                                                                         \
   if ( D == d && P == p && Q == q && basis == b )                                              \
   {                                                                                           \
      gref::SipdgApply< d, p, q, b >( m, mu_elem, sigma, kappa, boundary, x, y );              \
      return 0;                                                                                \
   }
   GREF_SIPDG_LIST( X )
#undef X
   return gref::GREF_UNSUPPORTED;
}

extern "C" int gref_diffusion_legacy_apply( int D, int P, int Q, int basis, const long * sizes, const double * h,
                                            const double * origin, const int * periodic, double d, double sigma,
                                            double kappa, const double * x, double * y )
{
   gref::MeshArgs m{ sizes, h, origin, periodic };
#define X( dd, p, q, b )                                                                        \
   if ( D == dd && P == p && Q == q && basis == b )                                             \
   {                                                                                           \
      gref::DiffusionLegacyApply< dd, p, q, b >( m, d, sigma, kappa, x, y );                   \
      return 0;                                                                                \
   }
   GREF_SIPDG_LIST( X )
#undef X
   return gref::GREF_UNSUPPORTED;
}
