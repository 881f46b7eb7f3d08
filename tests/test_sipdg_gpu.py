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
