// Test infrastructure only: this file is part of the CPU oracle, never of the product.
//
// Drives the GenDiL reference operators, compiled from the reference's own headers, so that
// the tests and the CPU baseline can call them through plain C functions.  Nothing here
// re-implements the reference: every result comes from the reference's own templates
//   MakeMassFiniteElementOperator   FiniteElementMethod/MatrixFreeOperators/massoperator.hpp:270
//   MakeAdvectionOperator           FiniteElementMethod/MatrixFreeOperators/advectionoperator.hpp:1416,1481
//   MassAdvectionOperator           FiniteElementMethod/MatrixFreeOperators/massadvectionoperator.hpp:329
//   ConjugateGradient (scratch)     Solvers/conjugategradient.hpp:125
//   GMRES_no_alloc                  Solvers/gmres.hpp:74
//   FillRandom                      Algebra/vector.hpp:632
// Every (dimension, order, quadrature points, basis) is a compile-time instantiation in the
// reference, so each part file instantiates a fixed list and reports -1 for anything else.
#pragma once

#include <gendil/gendil.hpp>

#include <array>
#include <cmath>
#include <cstring>
#include <utility>

namespace gref {

using namespace gendil;

enum { GREF_UNSUPPORTED = -1 };

// Coefficient presets.  The same formulas are tabulated for the B200 library by the tests, so
// the reference evaluates them pointwise exactly as a GenDiL user lambda would.
enum SigmaKind { SIGMA_CONST = 0, SIGMA_POLY = 1, SIGMA_SEP = 2 };
enum BetaKind { BETA_CONST = 0, BETA_BUBBLE = 1, BETA_SINCOS = 2, BETA_PHASE = 3 };

template < int D >
struct SigmaFn
{
   int kind;
   double c;
   GENDIL_HOST_DEVICE Real operator()( const std::array< Real, D > & X ) const
   {
      if ( kind == SIGMA_CONST ) return c;
      if ( kind == SIGMA_SEP ) return ( 1.0 + 0.5 * X[ 0 ] ) * ( 1.0 + X[ 1 % D ] * X[ 1 % D ] ) * ( 2.0 - X[ 2 % D ] );
      // test-mass-3d-generic.cpp:114-120 uses 1 + x*y + z*z in 3D.
      return 1.0 + X[ 0 ] * X[ 1 % D ] + X[ D - 1 ] * X[ D - 1 ];
   }
};

template < int D >
struct BetaFn
{
   int kind;
   double c[ 8 ];
   GENDIL_HOST_DEVICE void operator()( const std::array< Real, D > & X, Real ( &v )[ D ] ) const
   {
      for ( int i = 0; i < D; ++i )
      {
         if ( kind == BETA_CONST )
         {
            v[ i ] = c[ i ];
         }
         else if ( kind == BETA_BUBBLE )
         {
            // test-advection-3d-generic.cpp: beta_i = -x_i (1 - x_i)
            v[ i ] = -X[ i ] * ( 1.0 - X[ i ] );
         }
         else if ( kind == BETA_SINCOS )
         {
            if ( i == 0 ) v[ i ] = 1.0 + 0.5 * std::sin( 2.0 * M_PI * X[ 1 % D ] );
            else if ( i == 1 ) v[ i ] = 0.5 + 0.25 * std::cos( 2.0 * M_PI * X[ 2 % D ] );
            else v[ i ] = 0.25;
         }
         else
         {
            // phase space (x, v): beta = (v, -x + 0.5)
            constexpr int H = D / 2;
            if ( i < H ) v[ i ] = X[ i + H ];
            else v[ i ] = -X[ i - H ] + 0.5;
         }
      }
   }
};

template < int D >
struct BoundaryFn
{
   double g;
   GENDIL_HOST_DEVICE Real operator()( const std::array< Real, D > & ) const { return g; }
};

struct MeshArgs
{
   const long * sizes;
   const double * h;
   const double * origin;
   const int * periodic;
};

template < int D, int P, size_t... I >
auto MakeOrders( std::index_sequence< I... > )
{
   return FiniteElementOrders< ( (void)I, (Integer)P )... >{};
}

template < int D, int Q, size_t... I >
auto MakeNumPoints( std::index_sequence< I... > )
{
   return IntegrationRuleNumPoints< ( (void)I, Q )... >{};
}

template < int D >
CartesianMesh< D > MakeMesh( const MeshArgs & m )
{
   std::array< GlobalIndex, D > sizes;
   std::array< Real, D > h;
   Point< D > origin;
   std::array< int, D > periodic;
   for ( int i = 0; i < D; ++i )
   {
      sizes[ i ] = (GlobalIndex)m.sizes[ i ];
      h[ i ] = m.h[ i ];
      origin[ i ] = m.origin[ i ];
      periodic[ i ] = m.periodic ? m.periodic[ i ] : 0;
   }
   return CartesianMesh< D >( sizes, h, origin, periodic );
}

// Builds the reference space/rule for (D, P, Q, basis) and hands them to `body`.
template < int D, int P, int Q, int Basis, typename Body >
void WithSpace( const MeshArgs & margs, Body && body )
{
   auto mesh = MakeMesh< D >( margs );
   auto orders = MakeOrders< D, P >( std::make_index_sequence< D >{} );
   auto num_quads = MakeNumPoints< D, Q >( std::make_index_sequence< D >{} );
   auto integration_rule = MakeIntegrationRule( num_quads );
   if constexpr ( Basis == 0 )
   {
      auto fe = MakeLobattoFiniteElement( orders );
      auto fes = MakeFiniteElementSpace( mesh, fe );
      body( fes, integration_rule );
   }
   else
   {
      auto fe = MakeLegendreFiniteElement( orders );
      auto fes = MakeFiniteElementSpace( mesh, fe );
      body( fes, integration_rule );
   }
}

inline void CopyIn( Vector & v, const double * x )
{
   Real * d = v.WriteHostData();
   std::memcpy( d, x, sizeof( double ) * v.Size() );
}

inline void CopyOut( const Vector & v, double * y )
{
   const Real * d = v.ReadHostData();
   std::memcpy( y, d, sizeof( double ) * v.Size() );
}

template < int D, int P, int Q, int Basis >
void MassApply( const MeshArgs & m, int sigma_kind, double sigma_c, const double * x, double * y )
{
   WithSpace< D, P, Q, Basis >( m, [&]( auto & fes, auto & ir )
   {
      SigmaFn< D > sigma{ sigma_kind, sigma_c };
      auto op = MakeMassFiniteElementOperator< SerialKernelConfiguration >( fes, ir, sigma );
      const size_t n = fes.GetNumberOfFiniteElementDofs();
      Vector vx( n ), vy( n );
      CopyIn( vx, x );
      vy = 0.0;
      op( vx, vy );
      CopyOut( vy, y );
   } );
}

template < int D >
BetaFn< D > MakeBeta( int kind, const double * c )
{
   BetaFn< D > b{};
   b.kind = kind;
   for ( int i = 0; i < D; ++i ) b.c[ i ] = c ? c[ i ] : 0.0;
   return b;
}

// mode: 0 = advection without boundary terms, 1 = advection with inflow value `g`,
//       2 = mass(sigma) + advection (interior faces only).
template < int D, int P, int Q, int Basis >
void AdvectionApply( const MeshArgs & m, int mode, int beta_kind, const double * beta_c, double g,
                     int sigma_kind, double sigma_c, const double * x, double * y )
{
   WithSpace< D, P, Q, Basis >( m, [&]( auto & fes, auto & ir )
   {
      const size_t n = fes.GetNumberOfFiniteElementDofs();
      Vector vx( n ), vy( n );
      CopyIn( vx, x );
      vy = 0.0;
      auto beta = MakeBeta< D >( beta_kind, beta_c );
      if ( mode == 0 )
      {
         auto op = MakeAdvectionOperator< SerialKernelConfiguration >( fes, ir, beta );
         op( vx, vy );
      }
      else if ( mode == 1 )
      {
         BoundaryFn< D > bc{ g };
         auto op = MakeAdvectionOperator< SerialKernelConfiguration >( fes, ir, beta, bc );
         op( vx, vy );
      }
      else
      {
         SigmaFn< D > sigma{ sigma_kind, sigma_c };
         auto op = MakeMassAdvectionOperator< SerialKernelConfiguration >( fes, ir, beta, sigma );
         op( vx, vy );
      }
      CopyOut( vy, y );
   } );
}

inline Real HostDot( const Vector & a, const Vector & b )
{
   return Dot( a, b );
}

// CG on the mass operator, scratch overload (conjugategradient.hpp:125).
template < int D, int P, int Q, int Basis >
void MassCG( const MeshArgs & m, int sigma_kind, double sigma_c, const double * b, double * x,
             int max_iters, double tol, int * iters, double * rel, int * success )
{
   WithSpace< D, P, Q, Basis >( m, [&]( auto & fes, auto & ir )
   {
      SigmaFn< D > sigma{ sigma_kind, sigma_c };
      auto op = MakeMassFiniteElementOperator< SerialKernelConfiguration >( fes, ir, sigma );
      const size_t n = fes.GetNumberOfFiniteElementDofs();
      Vector vb( n ), vx( n ), tmp( n ), z( n ), r( n ), p( n );
      CopyIn( vb, b );
      CopyIn( vx, x );
      auto dot = []( const Vector & a, const Vector & c ) { return HostDot( a, c ); };
      auto res = ConjugateGradient( op, vb, dot, (Integer)max_iters, tol, vx, tmp, z, r, p );
      CopyOut( vx, x );
      *iters = (int)res.iterations;
      *rel = res.relative_error;
      *success = res.success ? 1 : 0;
   } );
}

// GMRES(restart) on sigma*M + A (A with inflow value g), gmres.hpp:74.
template < int D, int P, int Q, int Basis >
void SystemGMRES( const MeshArgs & m, double sigma_c, int beta_kind, const double * beta_c, double g,
                  const double * b, double * x, int max_iters, int restart, double tol,
                  int * iters, double * rel, int * success )
{
   WithSpace< D, P, Q, Basis >( m, [&]( auto & fes, auto & ir )
   {
      SigmaFn< D > sigma{ SIGMA_CONST, sigma_c };
      auto beta = MakeBeta< D >( beta_kind, beta_c );
      BoundaryFn< D > bc{ g };
      auto mass = MakeMassFiniteElementOperator< SerialKernelConfiguration >( fes, ir, sigma );
      auto adv = MakeAdvectionOperator< SerialKernelConfiguration >( fes, ir, beta, bc );
      const size_t n = fes.GetNumberOfFiniteElementDofs();
      Vector tmp( n );
      auto A = [&]( const Vector & in, Vector & out )
      {
         mass( in, out );
         adv( in, tmp );
         out += tmp;
      };
      Vector vb( n ), vx( n ), w( n );
      CopyIn( vb, b );
      CopyIn( vx, x );
      std::vector< Vector > V;
      V.reserve( restart + 1 );
      for ( int i = 0; i <= restart; ++i ) V.emplace_back( n );
      std::vector< Real > H( ( restart + 1 ) * restart ), cs( restart ), sn( restart ), e1( restart + 1 ), yv( restart );
      auto dot = []( const Vector & a, const Vector & c ) { return HostDot( a, c ); };
      auto res = GMRES_no_alloc( A, vb, dot, (Integer)max_iters, (Integer)restart, tol, vx, V, w, H, cs, sn, e1, yv );
      CopyOut( vx, x );
      *iters = (int)res.iterations;
      *rel = res.relative_error;
      *success = res.success ? 1 : 0;
   } );
}

} // namespace gref
