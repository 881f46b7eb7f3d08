"""GPU: CG through dgop_cg_solve_static, the entry point that allocates nothing.

It exists for callers that cannot let a library allocate device memory (a host framework that
owns all device memory through its own pool, or a latency-critical loop where cudaMalloc would
synchronize the device).  Its results must equal those of the allocating path
(dgop_cg_create + dgop_solver_solve) to the parity tolerance, on consecutive calls that reuse the
library's one static workspace.  This file is collected last on purpose."""
import ctypes

import pytest
import torch

import gendil_b200 as g
from helpers import APPLY_TOL, make_space, oracle, rel_max

pytestmark = pytest.mark.gpu

MAX_DOFS = 262144  # DGOP_STATIC_CG_MAX_DOFS in include/dgop.h


def _static_solve(op, b, x, max_iters, tol):
    L = g.lib()
    L.dgop_cg_solve_static.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                       ctypes.c_double, ctypes.POINTER(g._SolveResult), ctypes.c_void_p]
    res = g._SolveResult()
    rc = L.dgop_cg_solve_static(op.handle, b.data_ptr(), x.data_ptr(), max_iters, tol, ctypes.byref(res),
                                torch.cuda.current_stream().cuda_stream)
    return rc, {"success": bool(res.success), "iterations": res.iterations, "relative_error": res.relative_error}


def _mass_case(n, order=3, q=4, sigma_kind=0):
    return {"D": 3, "P": order, "Q": q, "basis": 0, "sizes": [n] * 3, "h": [1.0 / n] * 3, "origin": [0.0] * 3,
            "periodic": [0] * 3, "sigma_kind": sigma_kind, "sigma_c": 1.0}


@pytest.mark.parametrize("sigma_kind", [0, 1])
def test_static_cg_matches_allocating_cg_on_two_calls(sigma_kind):
    from gendil_b200 import coefficients as C
    case = _mass_case(16, sigma_kind=sigma_kind)  # 262,144 DoFs: exactly the static limit
    sp = make_space(case)
    assert sp.num_dofs == MAX_DOFS
    op = g.MassOperator(sp, 4, C.sigma_preset(sigma_kind, 3, 1.0))
    solver = g.CGSolver(op)
    for seed, iters, tol in ((0, 20, 1e-6), (1, 200, 1e-10)):  # two calls in a row, different data
        u = oracle().fill_random(sp.num_dofs, seed)
        b = torch.from_numpy(oracle().mass_apply(case, u)).cuda()
        x_ref = torch.zeros_like(b)
        info_ref = solver.solve(b, x_ref, iters, tol)
        x = torch.zeros_like(b)
        rc, info = _static_solve(op, b, x, iters, tol)
        assert rc == 0, g.lib().dgop_last_error()
        assert info["iterations"] == info_ref["iterations"] and info["success"] == info_ref["success"]
        assert abs(info["relative_error"] - info_ref["relative_error"]) <= APPLY_TOL * info_ref["relative_error"]
        assert rel_max(x.cpu().numpy(), x_ref.cpu().numpy()) <= APPLY_TOL


def test_static_cg_rejects_operators_above_the_limit():
    sp = make_space(_mass_case(17))  # 314,432 DoFs
    op = g.MassOperator(sp, 4, 1.0)
    b = torch.ones(sp.num_dofs, dtype=torch.float64, device="cuda")
    rc, _ = _static_solve(op, b, torch.zeros_like(b), 5, 1e-6)
    assert rc == -1
    assert b"static workspace limit" in g.lib().dgop_last_error()
