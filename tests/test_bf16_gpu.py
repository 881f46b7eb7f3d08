"""GPU: the BF16 tensor-core operator (dgop_apply_bf16: Kronecker products of the tangential
matrices as mma.sync BF16 GEMMs with FP32 accumulation and per-element max-abs scaling) and the
refinement solver with BF16 inner applies (DGOP_BF16).

BF16 keeps 8 significant bits, so the apply is compared with the reference's FP64 outputs at a
stated tolerance, BF16_TOL = 2e-2 of the largest output magnitude (each of the four BF16
operands of a term is rounded to 2^-9 relative of its largest entry; the sums over up to 27
products add cancellation); the solver's answer meets the FP64 stopping test exactly as with
FP32 inner applies."""
import numpy as np
import pytest
import torch

import gendil_b200 as g
from gendil_b200 import coefficients as C
from helpers import cuda_apply, golden, inputs, make_operator

pytestmark = pytest.mark.gpu
CASES, ARR = golden()
BF16_TOL = 2e-2

EVEN = [(f"{c['id']}_mode{m}", c, "adv", m) for c in CASES["advection"] if c["D"] % 2 == 0 for m in (0, 1, 2)] + \
       [(c["id"], c, "mass", 1) for c in CASES["mass"] if c["D"] % 2 == 0]


def _bf16(op, x, transpose=False):
    xt = torch.from_numpy(np.asarray(x)).to(device="cuda", dtype=torch.float32)
    y = torch.full_like(xt, float("nan"))
    op.apply_bf16(xt, y, transpose=transpose)
    torch.cuda.synchronize()
    return y.double().cpu().numpy()


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("cid,case,kind,mode", EVEN, ids=[c[0] for c in EVEN])
def test_bf16_apply_vs_reference_golden(cid, case, kind, mode):
    op = make_operator(case, kind, mode)
    try:
        op.select_kernel("kronnd")
    except g.DGOPError as exc:
        pytest.skip(f"not on the any-dimension Kronecker kernel: {exc}")
    x = inputs(case)
    want = ARR[f"{case['id']}_mode{mode}_y"] if kind == "adv" else ARR[f"{case['id']}_y"]
    try:
        got = _bf16(op, x)
    except g.DGOPError as exc:
        assert case["P"] == 0 or (case["P"] + 1) ** (case["D"] // 2) > 32, exc
        pytest.skip(str(exc))
    assert np.isfinite(got).all()
    assert _rel(got, want) <= BF16_TOL
    # the transposed operator against the FP64 transposed apply
    want_t = cuda_apply(op, x, transpose=True)
    assert _rel(_bf16(op, x, transpose=True), want_t) <= BF16_TOL


@pytest.mark.parametrize("D,n,p", [(4, 3, 2), (4, 2, 4), (6, 2, 2), (2, 6, 7)])
def test_bf16_apply_vs_fp64_on_larger_meshes(D, n, p):
    """Mass + advection with a per-axis velocity and inflow boundary (the configuration-3 kind of
    operator) on meshes with interior elements in every direction."""
    h = [1.0 / n] * D
    sp = g.Space(D, [n] * D, h, [0.0] * D, None, p)
    beta = C.velocity_constant([0.6, -0.4, 0.3, -0.2, 0.5, -0.7][:D])
    op = g.SystemOperator(sp, p + 1, beta, sigma=50.0, bc=g.BC_INFLOW, g=0.0)
    assert op.kernel in ("kronnd", "generic")
    op.select_kernel("kronnd")
    x = np.random.default_rng(D * 10 + p).uniform(-1, 1, sp.num_dofs)
    want = cuda_apply(op, x)
    assert _rel(_bf16(op, x), want) <= BF16_TOL


@pytest.mark.parametrize("D,n,p", [(4, 4, 2), (6, 4, 2)])
def test_refinement_with_bf16_inner_applies(D, n, p):
    """GMRES(20) with BF16 inner applies and the element mass inverse as preconditioner reaches
    1e-10 on the implicit-Euler system of configuration 3's kind, and its answer matches FP64
    GMRES's."""
    sizes = [n] * D
    h = [1.0 / n] * (D // 2) + [2.0 / n] * (D // 2)
    origin = [0.0] * (D // 2) + [-1.0] * (D // 2)
    sp = g.Space(D, sizes, h, origin, None, p)
    beta = C.velocity_phase_space(D) if D == 6 else C.velocity_constant([0.7, -0.3, 0.5, 0.2])
    dt = 5e-3
    A = g.SystemOperator(sp, p + 1, beta, sigma=1.0 / dt, bc=g.BC_INFLOW, g=0.0)
    A.select_kernel("kronnd")
    P = g.MassInverseOperator(sp, p + 1, 1.0 / dt)
    b = torch.from_numpy(g.fill_random(sp.num_dofs, 3)).cuda()
    sols = {}
    for inner in ("fp64", "bf16"):
        s = (g.GMRESSolver(A, 20) if inner == "fp64" else g.GMRESIRSolver(A, 20, inner="bf16")).precondition(P)
        x = torch.zeros_like(b)
        info = s.solve(b, x, 2000, 1e-10)
        assert info["success"], (inner, info)
        ax = torch.empty_like(x)
        A(x, ax)
        assert (torch.linalg.vector_norm(b - ax) / torch.linalg.vector_norm(b)).item() <= 1e-10
        sols[inner] = x
        s.close()
    d = (sols["bf16"] - sols["fp64"]).abs().max() / sols["fp64"].abs().max()
    assert d.item() < 1e-7
