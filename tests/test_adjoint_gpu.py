"""GPU: adjoint gradients of a solve-based loss with respect to per-element velocity and mass
factors (gendil_b200.adjoint), checked by central finite differences through the forward solve and
against an FP64 discrete adjoint assembled from operator applies."""
import numpy as np
import pytest
import torch

import gendil_b200 as g
from gendil_b200 import adjoint
from gendil_b200 import coefficients as C
from helpers import make_space, oracle

pytestmark = pytest.mark.gpu


def _case(D, n, P, Q):
    sizes = n if isinstance(n, list) else [n] * D
    return {"D": D, "P": P, "Q": Q, "basis": 0, "sizes": sizes, "h": [1.0 / s for s in sizes], "origin": [0.0] * D,
            "periodic": [0] * D}


def _loss(u, target):
    return 0.5 * torch.sum((u - target) ** 2)


@pytest.mark.parametrize("negative", [False, True], ids=["forward_flow", "reversed_flow"])
def test_gradients_match_central_differences(negative):
    case = _case(3, [4, 3, 3], 2, 3)
    sp = make_space(case)
    system = adjoint.AdvectionSystem(sp, 3, C.velocity_sincos(3), sigma=20.0, g_in=0.3, tol=1e-14)
    ne, nd = sp.num_elements, sp.num_dofs
    rng = np.random.default_rng(4)
    th = rng.uniform(0.5, 1.5, ne)
    if negative:
        # reversed flow everywhere: every upwind decision and inflow boundary flips (the sign
        # factors s_e = -1 of the gradient).  Signs that differ between neighbours would make
        # both elements of a face take the other's trace, which is not a well-posed scheme.
        th = -th
    theta = torch.tensor(th, device="cuda", requires_grad=True)
    rho = torch.tensor(rng.uniform(0.5, 1.5, ne), device="cuda", requires_grad=True)
    b = torch.tensor(oracle().fill_random(nd, 5), device="cuda", requires_grad=True)
    target = torch.tensor(oracle().fill_random(nd, 6), device="cuda")
    J = _loss(adjoint.solve(system, theta, b, rho), target)
    J.backward()
    eps = 1e-6

    def J_at(th_, rho_, b_):
        with torch.no_grad():
            return _loss(system.solve(th_, b_, rho_), target).item()

    with torch.no_grad():
        for which, grad in (("theta", theta.grad), ("rho", rho.grad), ("b", b.grad)):
            scale = grad.abs().max().item()
            idx = rng.choice(nd if which == "b" else ne, 6, replace=False)
            for i in idx:
                args = {"theta": theta.detach().clone(), "rho": rho.detach().clone(), "b": b.detach().clone()}
                plus = {k: v.clone() for k, v in args.items()}
                minus = {k: v.clone() for k, v in args.items()}
                plus[which][i] += eps
                minus[which][i] -= eps
                fd = (J_at(plus["theta"], plus["rho"], plus["b"]) - J_at(minus["theta"], minus["rho"], minus["b"])) / (
                    2 * eps)
                assert abs(fd - grad[i].item()) <= 1e-6 * scale, (which, int(i), fd, grad[i].item())


def test_gradient_matches_dense_discrete_adjoint():
    """FP64 discrete adjoint from the assembled matrix: S and dS/dtheta_e built column by column
    from operator applies, u and lambda from dense solves, g_e = -lambda^T (dS/dtheta_e) u."""
    case = _case(2, [3, 2], 1, 2)
    sp = make_space(case)
    system = adjoint.AdvectionSystem(sp, 2, C.velocity_constant([0.8, -0.5]), sigma=5.0, g_in=0.0, tol=1e-14)
    ne, nd = sp.num_elements, sp.num_dofs
    rng = np.random.default_rng(7)
    th = torch.tensor(rng.uniform(0.5, 1.5, ne), device="cuda")

    def dense(theta):
        op = system.operator(theta)
        cols = []
        for j in range(nd):
            e = torch.zeros(nd, dtype=torch.float64, device="cuda")
            e[j] = 1.0
            y = torch.empty_like(e)
            op(e, y)
            cols.append(y.cpu().numpy())
        op.close()
        return np.stack(cols, axis=1)

    S = dense(th)
    b = oracle().fill_random(nd, 5)
    target = oracle().fill_random(nd, 6)
    u = np.linalg.solve(S, b)
    lam = np.linalg.solve(S.T, u - target)
    want = np.empty(ne)
    for e in range(ne):
        t2 = th.clone()
        t2[e] += 1.0  # S is affine in theta_e while its sign is kept
        want[e] = -lam @ ((dense(t2) - S) @ u)
    theta = th.clone().requires_grad_(True)
    J = _loss(adjoint.solve(system, theta, torch.tensor(b, device="cuda")), torch.tensor(target, device="cuda"))
    J.backward()
    got = theta.grad.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max()


def test_transposed_solve_solves_the_adjoint_system():
    case = _case(3, [5, 4, 3], 3, 4)
    sp = make_space(case)
    op = g.SystemOperator(sp, 4, C.velocity_sincos(3), sigma=100.0, bc=g.BC_INFLOW, g=0.0)
    b = torch.tensor(oracle().fill_random(sp.num_dofs, 9), device="cuda")
    x = torch.zeros_like(b)
    info = g.GMRESSolver(op, 30).transpose().solve(b, x, 5000, 1e-12)
    assert info["success"]
    r = torch.empty_like(x)
    op.apply_transpose(x, r)
    assert (torch.linalg.vector_norm(b - r) / torch.linalg.vector_norm(b)).item() <= 1.01e-12


def test_element_dot():
    case = _case(3, [3, 2, 2], 2, 3)
    sp = make_space(case)
    op = g.MassOperator(sp, 3, 1.0)
    a = torch.tensor(oracle().fill_random(sp.num_dofs, 1), device="cuda")
    b = torch.tensor(oracle().fill_random(sp.num_dofs, 2), device="cuda")
    s = torch.arange(sp.num_elements, dtype=torch.float64, device="cuda") - 3.0
    got = g.element_dot(op, a, b, scale=s).cpu().numpy()
    nd = sp.dofs_per_element
    want = s.cpu().numpy() * (a.cpu().numpy() * b.cpu().numpy()).reshape(-1, nd).sum(axis=1)
    assert np.allclose(got, want, rtol=1e-14, atol=1e-14)
