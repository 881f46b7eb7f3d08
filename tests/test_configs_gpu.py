"""GPU: the benchmark configurations at their stated sizes against the GenDiL reference.

Fixtures come from ``tests/golden/make_golden.py --only configs`` (the reference compiled from
its own headers, oracle/_ref).  Large reference outputs are stored as strided samples plus their
max-norm and 2-norm; the GPU result is compared at the same indices, relative to the reference's
max-norm.

* C1 -- 3D mass, 16^3, p = 3, q = 4: the apply (<= 1e-13) and the CG trace of M x = M u from
  x0 = 0 (Solvers/conjugategradient.hpp:125).  The reference's own CG on this system amplifies
  rounding from about 8 iterations on: its iterates at 1 and 3 OpenMP threads differ by 3e-14
  after 5 iterations, 1.4e-11 after 8 and 4e-3 after 20 (the residual is not even monotone after
  12).  So the 5- and 8-iteration iterates are pinned tightly (1e-12, 1e-9) and the 20-iteration
  one within the reference's own spread (iterations, relative error within a factor 2, iterate
  within 2e-2).
* C2 -- 3D implicit system sigma M + A, 64^3, p = 3, sigma = 1/dt = 1e3, sin/cos velocity:
  GMRES(30) to 1e-10 from x0 = 0 against GMRES_no_alloc (Solvers/gmres.hpp:74): iteration count
  within 1 % (the reference's Dot is an OpenMP reduction), solution within 1e-8.
* C3 -- 6D phase-space advection (p = 2, q = 3, beta = (v, -x + 0.5), inflow 0) on a 4^6 mesh,
  which has interior faces on every axis: the apply <= 1e-13 at the stored samples and against
  the plain-C oracle (itself pinned to the reference) on the whole vector.
* C5 -- every element shape of the batched instances (dimension 2..4, order 1..5, q = p + 2,
  constant velocity): the mass and inflow-advection applies and the one-launch implicit system
  sigma M + A, full outputs, <= 1e-13.
"""
import numpy as np
import pytest
import torch

import gendil_b200 as g
from gendil_b200 import coefficients as C
from helpers import APPLY_TOL, golden, make_operator, make_space, oracle

pytestmark = pytest.mark.gpu
CASES, ARR = golden()
CFG = {c["id"]: c for c in CASES.get("configs", [])}
C5 = [c for c in CASES.get("configs", []) if c["id"].startswith("c5_")]


def _sample_err(v, key, stride):
    """Largest deviation at the stored sample indices, relative to the reference's max-norm."""
    s = ARR[f"{key}_sample"]
    stats = ARR[f"{key}_stats"]
    got = np.asarray(v)[::stride]
    assert got.shape == s.shape
    return float(np.abs(got - s).max() / stats[0])


def _system(case, space):
    beta = C.beta_preset(case.get("beta_kind", 0), case["D"], case.get("beta_c"))
    return g.SystemOperator(space, case["Q"], beta, sigma=case["sigma_c"], bc=g.BC_INFLOW, g=case.get("g", 0.0))


def _kernels(op):
    """The operator's own kernel plus the generic sum-factorized one, when they differ."""
    return [op.kernel] + (["generic"] if op.kernel != "generic" else [])


def test_c1_mass_apply_full_size():
    case = CFG["c1"]
    sp = make_space(case)
    op = make_operator(case, "mass", space=sp)
    for kernel in _kernels(op):
        if kernel != op.kernel:
            op.select_kernel(kernel)
        x = torch.from_numpy(oracle().fill_random(sp.num_dofs, 0)).cuda()
        y = torch.empty_like(x)
        op(x, y)
        err = _sample_err(y.cpu().numpy(), "c1_y", case["stride"])
        assert err <= APPLY_TOL, (kernel, err)


@pytest.mark.parametrize("kernel", ["default", "generic"])
def test_c1_cg_trace(kernel):
    case = CFG["c1"]
    sp = make_space(case)
    op = make_operator(case, "mass", space=sp)
    if kernel == "generic" and op.kernel != "generic":
        op.select_kernel("generic")
    u = torch.from_numpy(oracle().fill_random(sp.num_dofs, 0)).cuda()
    b = torch.empty_like(u)
    op(u, b)
    solver = g.CGSolver(op)
    bars = {5: 1e-12, 8: 1e-9}
    for k, bar in bars.items():
        x = torch.zeros_like(b)
        info = solver.solve(b, x, k, case["cg_tol"])
        ref = case["traces"][str(k)]
        assert info["iterations"] == ref["iterations"] and info["success"] == ref["success"], (k, info, ref)
        assert abs(info["relative_error"] - ref["relative_error"]) <= 1e-6 * ref["relative_error"], (k, info, ref)
        err = _sample_err(x.cpu().numpy(), f"c1_x{k}", case["stride"])
        assert err <= bar, (k, err)
    k = case["cg_iters"]
    x = torch.zeros_like(b)
    info = solver.solve(b, x, k, case["cg_tol"])
    ref = case["traces"][str(k)]
    assert info["iterations"] == ref["iterations"] == k and not info["success"]
    assert 0.5 * ref["relative_error"] <= info["relative_error"] <= 2.0 * ref["relative_error"], (info, ref)
    assert _sample_err(x.cpu().numpy(), f"c1_x{k}", case["stride"]) <= 2e-2


def test_c2_gmres30_full_size():
    case = CFG["c2"]
    sp = make_space(case)
    op = _system(case, sp)
    b = torch.from_numpy(oracle().fill_random(sp.num_dofs, case["seed"])).cuda()
    x = torch.zeros_like(b)
    info = g.GMRESSolver(op, case["restart"]).solve(b, x, case["max_iters"], case["tol"])
    assert info["success"] and info["relative_error"] <= case["tol"], info
    assert abs(info["iterations"] - case["iterations"]) <= max(1, case["iterations"] // 100), (info, case["iterations"])
    # the reported residual is recomputed from x: check it against an independent apply
    ax = torch.empty_like(x)
    op(x, ax)
    true_rel = (torch.linalg.vector_norm(b - ax) / torch.linalg.vector_norm(b)).item()
    assert true_rel <= case["tol"] and abs(true_rel - info["relative_error"]) <= 1e-3 * case["tol"]
    assert _sample_err(x.cpu().numpy(), "c2_x", case["stride"]) <= 1e-8
    norm_ref = ARR["c2_x_stats"][1]
    assert abs(torch.linalg.vector_norm(x).item() - norm_ref) <= 1e-8 * norm_ref


def test_c3_6d_apply_interior_faces_every_axis():
    case = CFG["c3"]
    sp = make_space(case)
    op = make_operator(case, "adv", mode=1, space=sp)
    x_np = oracle().fill_random(sp.num_dofs, case["seed"])
    want = oracle().advection_apply(case, x_np, 1)
    for kernel in _kernels(op):
        if kernel != op.kernel:
            op.select_kernel(kernel)
        x = torch.from_numpy(x_np).cuda()
        y = torch.empty_like(x)
        op(x, y)
        got = y.cpu().numpy()
        assert _sample_err(got, "c3_y", case["stride"]) <= APPLY_TOL, kernel
        assert float(np.abs(got - want).max() / np.abs(want).max()) <= APPLY_TOL, kernel


@pytest.mark.parametrize("case", C5, ids=lambda c: c["id"])
def test_c5_shapes(case):
    sp = make_space(case)
    x_np = oracle().fill_random(sp.num_dofs, case["seed"])
    x = torch.from_numpy(x_np).cuda()
    y = torch.empty_like(x)
    mass_ref, adv_ref = ARR[f"{case['id']}_mass_y"], ARR[f"{case['id']}_adv_y"]
    sys_ref = mass_ref + adv_ref
    for kind, ref in (("mass", mass_ref), ("adv", adv_ref), ("system", sys_ref)):
        op = _system(case, sp) if kind == "system" else make_operator(case, kind, mode=1, space=sp)
        for kernel in _kernels(op):
            if kernel != op.kernel:
                op.select_kernel(kernel)
            op(x, y)
            err = float(np.abs(y.cpu().numpy() - ref).max() / np.abs(ref).max())
            assert err <= APPLY_TOL, (kind, kernel, err)
        op.close()
