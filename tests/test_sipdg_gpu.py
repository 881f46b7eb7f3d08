"""GPU: the interior-penalty DG diffusion operator (dgop_sipdg_create) against the reference's own
generic SIPDG weak form (golden fixtures from oracle/part_sipdg.cpp), its symmetry, FP32 apply
and a CG solve of the symmetric form."""
import numpy as np
import pytest
import torch

import gendil_b200 as g
from helpers import APPLY_TOL, golden, inputs, make_space, oracle, rel_max

pytestmark = pytest.mark.gpu
CASES, ARR = golden()


def _op(case, mu=None):
    sp = make_space(case)
    if mu is None:
        mu = torch.tensor(ARR[f"{case['id']}_mu"], device="cuda")
    return g.SIPDGOperator(sp, case["Q"], mu, sigma=case["sigma"], kappa=case["kappa"],
                           boundary=bool(case["boundary"]))


@pytest.mark.parametrize("case", CASES["sipdg"], ids=lambda c: c["id"])
def test_sipdg_vs_reference_golden(case):
    op = _op(case)
    assert op.kernel == "diffusion"
    x = torch.tensor(inputs(case), device="cuda")
    y = torch.empty_like(x)
    op(x, y)
    assert rel_max(y.cpu().numpy(), ARR[f"{case['id']}_y"]) <= APPLY_TOL
    y32 = torch.empty(x.numel(), dtype=torch.float32, device="cuda")
    op.apply_f32(x.float(), y32)
    assert rel_max(y32.double().cpu().numpy(), ARR[f"{case['id']}_y"]) <= 1e-5


@pytest.mark.parametrize("case", [c for c in CASES["sipdg"] if c["sigma"] == -1.0], ids=lambda c: c["id"])
def test_sipg_is_symmetric(case):
    op = _op(case)
    x = torch.tensor(inputs(case, seed=6), device="cuda")
    z = torch.tensor(inputs(case, seed=7), device="cuda")
    ax, az, atx = torch.empty_like(x), torch.empty_like(z), torch.empty_like(x)
    op(x, ax)
    op(z, az)
    op.apply_transpose(x, atx)
    assert torch.equal(ax, atx)
    lhs, rhs = float(ax @ z), float(x @ az)
    assert abs(lhs - rhs) <= 1e-12 * float(ax.abs().sum() * z.abs().max())


def test_sipg_cg_solve():
    """Configuration 4's discretisation at 6^3 (p = 4, q = 6, mu = exp(z), z ~ N(0, 0.5^2) seed 4,
    kappa = 10 (p+1)^2, Dirichlet 0): CG to 1e-12 on the symmetric positive definite system."""
    case = {"D": 3, "P": 4, "Q": 6, "basis": 0, "sizes": [6] * 3, "h": [1 / 6] * 3, "origin": [0.0] * 3,
            "periodic": [0] * 3}
    sp = make_space(case)
    mu = torch.tensor(np.exp(np.random.default_rng(4).normal(0.0, 0.5, sp.num_elements)), device="cuda")
    op = g.SIPDGOperator(sp, 6, mu, sigma=-1.0, kappa=250.0, boundary=True)
    f = torch.tensor(oracle().fill_random(sp.num_dofs, 5), device="cuda")
    u = torch.zeros_like(f)
    info = g.CGSolver(op).solve(f, u, 20000, 1e-12)
    assert info["success"], info
    r = torch.empty_like(u)
    op(u, r)
    # the CG convention: |r| / |r0| below 1e-12 (r0 = f for u0 = 0)
    assert (torch.linalg.vector_norm(f - r) / torch.linalg.vector_norm(f)).item() <= 2e-12


@pytest.mark.parametrize("case", CASES["sipdg"], ids=lambda c: c["id"])
def test_coefficient_gradient_vs_reference_golden(case):
    """lam^T (dA/dmu_e) u against the reference operator's one-hot derivative (A is linear in mu)."""
    op = _op(case)
    u = torch.tensor(inputs(case), device="cuda")
    lam = torch.tensor(inputs(case, seed=case["grad_seed"]), device="cuda")
    out = op.coefficient_gradient(u, lam)
    ref = ARR[f"{case['id']}_grad"]
    assert rel_max(out.cpu().numpy(), ref) <= 1e-12
    scale = torch.linspace(0.5, 2.0, out.numel(), dtype=torch.float64, device="cuda")
    out2 = op.coefficient_gradient(u, lam, scale=scale)
    assert torch.equal(out2, scale * out)
    again = op.coefficient_gradient(u, lam)
    assert torch.equal(again, out)  # deterministic


def test_coefficient_gradient_matches_directional_derivative():
    """sum_e dmu_e out_e = lam^T A(dmu) u for a random direction (linearity in mu), 5^3 p = 3."""
    case = {"D": 3, "P": 3, "Q": 5, "basis": 0, "sizes": [5, 4, 3], "h": [0.2, 0.25, 1 / 3], "origin": [0.0] * 3,
            "periodic": [0, 1, 0]}
    sp = make_space(case)
    rng = np.random.default_rng(9)
    mu = torch.tensor(np.exp(rng.normal(0, 0.5, sp.num_elements)), device="cuda")
    dmu = torch.tensor(rng.normal(0, 1, sp.num_elements), device="cuda")
    u = torch.tensor(rng.uniform(-1, 1, sp.num_dofs), device="cuda")
    lam = torch.tensor(rng.uniform(-1, 1, sp.num_dofs), device="cuda")
    op = g.SIPDGOperator(sp, 5, mu, sigma=1.0, kappa=160.0, boundary=True)
    out = op.coefficient_gradient(u, lam)
    opd = g.SIPDGOperator(sp, 5, dmu, sigma=1.0, kappa=160.0, boundary=True)
    w = torch.empty_like(u)
    opd(u, w)
    lhs, rhs = float(dmu @ out), float(lam @ w)
    assert abs(lhs - rhs) <= 1e-12 * float((dmu.abs() * out.abs()).sum())


def test_loss_gradient_vs_central_differences():
    """Configuration 4's gradient at 4^3, p = 4: J = 1/2 |u - u*|^2, A(exp z) u = f, dJ/dz by the
    adjoint solve and the coefficient-gradient kernel against central differences (eps = 1e-6)
    on 8 random elements, <= 1e-6 relative per element (measured on a B200: about 1.4e-8).

    Every solve is CG from x0 = 0 to 1e-13, and the difference quotient is formed without
    cancellation: J(z+) - J(z-) = 1/2 (u+ - u-) . (u+ + u- - 2 u*)."""
    from gendil_b200 import adjoint
    case = {"D": 3, "P": 4, "Q": 6, "basis": 0, "sizes": [4] * 3, "h": [0.25] * 3, "origin": [0.0] * 3,
            "periodic": [0] * 3}
    sp = make_space(case)
    system = adjoint.DiffusionSystem(sp, 6, tol=1e-13)
    z = torch.tensor(np.random.default_rng(4).normal(0.0, 0.5, sp.num_elements), device="cuda", requires_grad=True)
    f = torch.tensor(oracle().fill_random(sp.num_dofs, 5), device="cuda")
    ustar = torch.tensor(oracle().fill_random(sp.num_dofs, 6), device="cuda")

    u = adjoint.solve_diffusion(system, torch.exp(z), f)
    J = 0.5 * torch.sum((u - ustar) ** 2)
    J.backward()
    grad = z.grad.clone()
    eps = 1e-6

    def perturbed(e, sgn):
        zp = z.detach().clone()
        zp[e] += sgn * eps
        return system.solve(torch.exp(zp), f)

    rel = []
    for e in np.random.default_rng(8).choice(sp.num_elements, 8, replace=False):
        up, um = perturbed(int(e), 1.0), perturbed(int(e), -1.0)
        fd = 0.5 * torch.sum((up - um) * (up + um - 2.0 * ustar)).item() / (2 * eps)
        rel.append(abs(fd - grad[e].item()) / abs(grad[e].item()))
    assert max(rel) <= 1e-6, rel


@pytest.mark.parametrize("case", CASES["diffusion"], ids=lambda c: c["id"])
def test_legacy_diffusion_operator_vs_reference_golden(case):
    """DiffusionOperator against the reference's legacy MakeDiffusionOperator (constant diffusivity,
    interior and boundary faces), including the two-element periodic 1D mesh of the reference's
    symmetry test and sigma = 1, 0, -1."""
    sp = make_space(case)
    op = g.DiffusionOperator(sp, case["Q"], case["diffusivity"], case["sigma"], case["kappa"])
    x = torch.tensor(inputs(case), device="cuda")
    y = torch.empty_like(x)
    op(x, y)
    assert rel_max(y.cpu().numpy(), ARR[f"{case['id']}_y"]) <= APPLY_TOL
    if case["sigma"] == -1.0:
        yt = torch.empty_like(x)
        op.apply_transpose(x, yt)
        assert torch.equal(yt, y)
