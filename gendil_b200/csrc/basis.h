// 1D bases and Gauss rules on [0, 1] (host).
#pragma once

namespace dgop {

// Nodes and weights on [0,1], ascending.  kind 0: Gauss-Lobatto-Legendre (n = 1 is the single
// node 0.5 with weight 1, as GLLpoints.hpp:17-43), kind 1: Gauss-Legendre.  n in 1..8.
// Computed by Newton iteration on the Legendre polynomials in long double; the reference
// hard-codes the same nodes to about 15 significant digits (GLpoints.hpp, GLLpoints.hpp).
bool gauss_points(int kind, int n, double* x, double* w);

// Lagrange basis on `nodes` (product formulas of lagrangeshapefunctions.hpp:37,60).
double lagrange_value(const double* nodes, int n, int j, double x);
double lagrange_grad(const double* nodes, int n, int j, double x);

}  // namespace dgop
