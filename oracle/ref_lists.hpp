// Test infrastructure only (CPU oracle): the (dimension, order, quadrature points, basis)
// instantiations of the reference operators that the parity tests use.  basis 0 = GLL
// (MakeLobattoFiniteElement), 1 = GL (MakeLegendreFiniteElement).
#pragma once

#define GREF_MASS_LIST_A(X) \
   X(1,0,1,0) X(1,3,5,0) X(1,7,8,0) X(2,0,1,0) X(2,2,4,0) X(2,4,3,0) X(2,2,3,1)
#define GREF_MASS_LIST_B(X) \
   X(3,1,4,0) X(3,3,4,0) X(3,3,6,0) X(3,2,2,1) X(3,7,8,0) X(3,1,2,0) X(3,4,5,0)
#define GREF_MASS_LIST_C(X) \
   X(4,2,3,0) X(5,1,2,0) X(6,1,2,0) X(6,2,3,0)

#define GREF_ADV_LIST_A(X) \
   X(1,0,1,0) X(1,2,4,0) X(2,1,2,1) X(2,2,3,0) X(2,4,3,0)
#define GREF_ADV_LIST_B(X) \
   X(3,0,2,0) X(3,1,3,0) X(3,3,4,0) X(3,2,2,1)
#define GREF_ADV_LIST_C(X) \
   X(3,5,6,0) X(3,7,8,0) X(3,2,3,0) X(3,4,5,0) X(3,3,3,0)
#define GREF_ADV_LIST_D(X) \
   X(4,1,2,0) X(5,1,2,0)
#define GREF_ADV_LIST_E(X) \
   X(6,2,3,0)

#define GREF_CG_LIST(X) X(3,3,4,0) X(2,2,3,0) X(1,3,5,0)
#define GREF_GMRES_LIST(X) X(3,3,4,0) X(2,2,3,0) X(1,2,4,0)

// the shapes of the batched uneven instances (dimension 2..4, order 1..5, q = p + 2), mass and
// advection; shapes already in the lists above are left out
#define GREF_MASS_LIST_D(X) \
   X(2,1,3,0) X(2,3,5,0) X(2,4,6,0) X(2,5,7,0) X(3,1,3,0) X(3,2,4,0) X(3,5,7,0)
#define GREF_MASS_LIST_E(X) \
   X(4,1,3,0) X(4,2,4,0) X(4,3,5,0) X(4,4,6,0) X(4,5,7,0) X(3,3,5,0) X(3,4,6,0)
#define GREF_ADV_LIST_F(X) \
   X(2,1,3,0) X(2,2,4,0) X(2,3,5,0) X(2,4,6,0) X(2,5,7,0) X(3,2,4,0) X(3,3,5,0)
#define GREF_ADV_LIST_G(X) \
   X(4,1,3,0) X(4,2,4,0) X(4,3,5,0) X(3,4,6,0) X(3,5,7,0)
#define GREF_ADV_LIST_H(X) \
   X(4,4,6,0) X(4,5,7,0)
