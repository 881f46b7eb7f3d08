"""Gradients of solve-based losses with respect to per-element coefficient factors.

The system is the implicit-Euler DG operator with per-element factors on the velocity and the
mass term,

    S(theta, rho) u = b,    S = M_{sigma rho} + A(theta beta0)      (sigma, beta0, bc, g fixed),

where element e's velocity is theta_e * beta0(X) and its mass density sigma(X) * rho_e.  Every
row block of S (the test functions of one element) uses only that element's coefficients: the
cell term and the element's own face fluxes, whose upwind side is decided by its own beta . n.
Hence, with the adjoint state lambda solving S^T lambda = dJ/du,

    dJ/dtheta_e = -lambda_e . (dS/dtheta_e u)_e = -s_e lambda_e . (A(s beta0) u)_e,   s_e = sign(theta_e)
    dJ/drho_e   = -lambda_e . (M_sigma u)_e
    dJ/db       =  lambda

(A(s beta0) u: the advection part, inflow value included, with element factors s, whose upwind
decisions are those of theta).  Forward and adjoint solves are device GMRES (the adjoint one with
the transposed operator); the per-element products are one kernel (dgop_element_dot).  Nothing
of the forward Krylov iteration is stored: the backward pass needs u and the operators only.
No reference counterpart; the checks are central finite differences and an FP64 discrete adjoint
assembled from operator applies (tests/test_adjoint_gpu.py).
"""
from __future__ import annotations

import copy

import torch

import gendil_b200 as g
from gendil_b200 import coefficients as C


class AdvectionSystem:
    """S(theta, rho) = M_{sigma rho} + A(theta beta0) on `space` with quadrature q; FP64 GMRES."""

    def __init__(self, space, q, beta, sigma=1.0, bc=g.BC_INFLOW, g_in=0.0, restart=30, tol=1e-12,
                 max_iters=20000):
        self.space, self.q = space, q
        self.beta = [C.as_coefficient(c, space.dim) for c in g._components(beta, space.dim)]
        self.sigma = C.as_coefficient(sigma, space.dim)
        self.bc, self.g_in = bc, g_in
        self.restart, self.tol, self.max_iters = restart, tol, max_iters
        self.last_info = None

    def _with_factor(self, coef, factor):
        c = copy.copy(coef)
        c.element_factor = factor
        return c

    def operator(self, theta, rho=None):
        beta = [self._with_factor(c, theta) for c in self.beta]
        return g.SystemOperator(self.space, self.q, beta, sigma=self._with_factor(self.sigma, rho), bc=self.bc,
                                g=self.g_in)

    def _solve(self, op, rhs, transpose=False):
        x = torch.zeros_like(rhs)
        solver = g.GMRESSolver(op, self.restart)
        if transpose:
            solver.transpose()
        info = solver.solve(rhs, x, self.max_iters, self.tol)
        solver.close()
        if not info["success"]:
            raise RuntimeError(f"GMRES did not converge: {info}")
        self.last_info = info
        return x

    def solve(self, theta, b, rho=None):
        """u = S(theta, rho)^{-1} b."""
        op = self.operator(theta, rho)
        u = self._solve(op, b)
        op.close()
        return u

    def adjoint(self, theta, grad_u, rho=None):
        """lambda = S(theta, rho)^{-T} grad_u."""
        op = self.operator(theta, rho)
        lam = self._solve(op, grad_u, transpose=True)
        op.close()
        return lam

    def grad_theta(self, theta, u, lam):
        """dJ/dtheta_e = -s_e lambda_e . (A(s beta0) u)_e."""
        s = torch.where(theta < 0, -torch.ones_like(theta), torch.ones_like(theta))
        adv = g.AdvectionOperator(self.space, self.q, [self._with_factor(c, s) for c in self.beta], bc=self.bc,
                                  g=self.g_in)
        w = torch.empty_like(u)
        adv(u, w)
        out = g.element_dot(adv, lam, w, scale=s)
        adv.close()
        return -out

    def grad_rho(self, u, lam):
        """dJ/drho_e = -lambda_e . (M_sigma u)_e."""
        mass = g.MassOperator(self.space, self.q, self.sigma)
        w = torch.empty_like(u)
        mass(u, w)
        out = g.element_dot(mass, lam, w)
        mass.close()
        return -out


class _SolveFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, rho, b, system):
        theta = theta.detach().contiguous()
        rho = None if rho is None else rho.detach().contiguous()
        u = system.solve(theta, b.detach().contiguous(), rho)
        ctx.system = system
        ctx.has_rho = rho is not None
        ctx.save_for_backward(theta, u, *([rho] if rho is not None else []))
        return u

    @staticmethod
    def backward(ctx, grad_u):
        system = ctx.system
        theta, u = ctx.saved_tensors[0], ctx.saved_tensors[1]
        rho = ctx.saved_tensors[2] if ctx.has_rho else None
        lam = system.adjoint(theta, grad_u.contiguous(), rho)
        g_theta = system.grad_theta(theta, u, lam) if ctx.needs_input_grad[0] else None
        g_rho = system.grad_rho(u, lam) if (ctx.has_rho and ctx.needs_input_grad[1]) else None
        g_b = lam if ctx.needs_input_grad[2] else None
        return g_theta, g_rho, g_b, None


def solve(system, theta, b, rho=None):
    """u = S(theta, rho)^{-1} b, differentiable in theta, rho and b (torch.autograd)."""
    return _SolveFunction.apply(theta, rho, b, system)


class DiffusionSystem:
    """A(mu) u = f for the symmetric interior-penalty DG diffusion operator (SIPG, sigma = -1) with
    one diffusivity mu_e per element; FP64 CG (A is symmetric positive definite for kappa large
    enough).  With J(u) and lambda = A^{-1} dJ/du (A^T = A),

        dJ/dmu_e = -lambda^T (dA/dmu_e) u     (dgop_sipdg_gradient, one kernel)
        dJ/df    =  lambda

    and dJ/dz_e = mu_e dJ/dmu_e for mu = exp(z) follows by the chain rule (torch.autograd).
    No reference counterpart; the checks are central finite differences and the reference
    operator's one-hot derivative (tests/test_sipdg_gpu.py)."""

    def __init__(self, space, q, kappa=None, boundary=True, tol=1e-12, max_iters=50000):
        self.space, self.q = space, q
        self.kappa = 10.0 * (space.order + 1) ** 2 if kappa is None else kappa
        self.boundary = boundary
        self.tol, self.max_iters = tol, max_iters
        self.last_info = None

    def operator(self, mu):
        return g.SIPDGOperator(self.space, self.q, mu.detach().contiguous(), sigma=-1.0, kappa=self.kappa,
                               boundary=self.boundary)

    def _solve(self, op, rhs):
        x = torch.zeros_like(rhs)
        solver = g.CGSolver(op)
        info = solver.solve(rhs, x, self.max_iters, self.tol)
        solver.close()
        if not info["success"]:
            raise RuntimeError(f"CG did not converge: {info}")
        self.last_info = info
        return x

    def solve(self, mu, f):
        """u = A(mu)^{-1} f."""
        op = self.operator(mu)
        u = self._solve(op, f)
        op.close()
        return u

    def adjoint(self, mu, grad_u):
        """lambda = A(mu)^{-T} grad_u (= A(mu)^{-1} grad_u: the form is symmetric)."""
        return self.solve(mu, grad_u)

    def grad_mu(self, mu, u, lam):
        """dJ/dmu_e = -lambda^T (dA/dmu_e) u."""
        op = self.operator(mu)
        out = op.coefficient_gradient(u, lam)
        op.close()
        return -out


class _DiffusionSolveFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, mu, f, system):
        mu = mu.detach().contiguous()
        u = system.solve(mu, f.detach().contiguous())
        ctx.system = system
        ctx.save_for_backward(mu, u)
        return u

    @staticmethod
    def backward(ctx, grad_u):
        system = ctx.system
        mu, u = ctx.saved_tensors
        lam = system.adjoint(mu, grad_u.contiguous())
        g_mu = system.grad_mu(mu, u, lam) if ctx.needs_input_grad[0] else None
        g_f = lam if ctx.needs_input_grad[1] else None
        return g_mu, g_f, None


def solve_diffusion(system, mu, f):
    """u = A(mu)^{-1} f, differentiable in mu and f (torch.autograd)."""
    return _DiffusionSolveFunction.apply(mu, f, system)
