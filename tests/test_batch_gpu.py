"""GPU: batches of independent operators (dgop_batch_apply): one persistent launch per
(dimension, order, kernel variant) group on the any-dimension Kronecker kernel, the rest one launch each; results
bit-identical to each operator's own apply."""
import numpy as np
import pytest
import torch

import gendil_b200 as g
from gendil_b200 import coefficients as C

pytestmark = pytest.mark.gpu


def _space(D, n, p, basis=g.GLL):
    sizes = n if isinstance(n, list) else [n] * D
    return g.Space(D, sizes, [1.0 / s for s in sizes], [0.0] * D, None, p, basis)


def _batched(o):
    """Whether the persistent batch kernel serves this operator's variant: every any-dimension
    variant but the mass-only one, with blocks of at most 27 values (N = order + 1; grouped by 2
    axes up to N = 5, by 3 up to N = 3, paired up to N = 5)."""
    if o.kernel != "kronnd":
        return False
    n = o.space.order + 1
    return {"nd-passes": True, "nd-grouped2": n * n <= 27, "nd-grouped3": n ** 3 <= 27,
            "nd-paired": n * n <= 27}.get(o.variant, False)


def test_batch_apply_equals_individual_applies():
    rng = np.random.default_rng(7)
    ops = []
    for D, n, p in [(2, [9, 7], 3), (2, [5, 11], 3), (3, [4, 3, 5], 4), (4, [3, 2, 4, 3], 1), (2, [6, 6], 1),
                    (3, [3, 3, 3], 4), (4, [2, 3, 2, 2], 2), (3, [5, 4, 3], 2), (2, [7, 5], 5)]:
        sp = _space(D, n, p)
        beta = C.velocity_constant(list(rng.uniform(-1, 1, D)))
        ops.append(g.SystemOperator(sp, p + 2, beta, sigma=1e3, bc=g.BC_INFLOW, g=0.0))
    ops.append(g.SystemOperator(_space(2, [4, 5], 2, g.GL), 4, C.velocity_constant([0.3, -0.7]), sigma=1e3))
    kinds = [o.kernel for o in ops]
    assert "kronnd" in kinds and "kron" in kinds and "generic" in kinds
    xs = [torch.rand(o.space.num_dofs, dtype=torch.float64, device="cuda") - 0.5 for o in ops]
    want = []
    for o, x in zip(ops, xs):
        y = torch.empty_like(x)
        o(x, y)
        want.append(y)
    batch = g.Batch(ops)
    assert batch.groups == len({(o.space.dim, o.space.order, o.variant) for o in ops if _batched(o)})
    for _ in range(2):  # twice: the parameter upload of the previous apply is reused safely
        ys = [torch.full_like(x, float("nan")) for x in xs]
        batch.apply(xs, ys)
        torch.cuda.synchronize()
        for y, w in zip(ys, want):
            assert torch.equal(y, w)
    batch.close()


def test_batch_large_instance_keeps_its_own_launch():
    """An instance whose element batches fill every CTA slot of the GPU twice over (here 10^6
    elements) is applied by its own launch, outside the groups; the small instances of the same
    (dimension, order) still form a group, and every result is bit-identical to its own apply."""
    rng = np.random.default_rng(11)
    specs = [(2, [1000, 1000], 1), (2, [9, 7], 1), (2, [5, 11], 1)]
    ops = []
    for D, n, p in specs:
        beta = C.velocity_constant(list(rng.uniform(-1, 1, D)))
        ops.append(g.SystemOperator(_space(D, n, p), p + 2, beta, sigma=1e3, bc=g.BC_INFLOW, g=0.0))
    for o in ops[1:]:
        o.set_variant(ops[0].variant)  # one (dimension, order, variant) key for all three
    assert all(o.kernel == "kronnd" for o in ops)
    xs = [torch.rand(o.space.num_dofs, dtype=torch.float64, device="cuda") - 0.5 for o in ops]
    want = []
    for o, x in zip(ops, xs):
        y = torch.empty_like(x)
        o(x, y)
        want.append(y)
    batch = g.Batch(ops)
    assert batch.groups == 1
    ys = [torch.full_like(x, float("nan")) for x in xs]
    batch.apply(xs, ys)
    torch.cuda.synchronize()
    for y, w in zip(ys, want):
        assert torch.equal(y, w)
    batch.close()


def test_batch_unbatched_variant_runs_one_launch_each():
    """Operators whose variant has no persistent batch kernel (2D p = 5 on 36-value blocks of 2
    axes) form no group and are applied one launch each, bit-identical to their own applies."""
    rng = np.random.default_rng(5)
    ops = []
    for n in ([7, 5], [6, 9]):
        beta = C.velocity_constant(list(rng.uniform(-1, 1, 2)))
        o = g.SystemOperator(_space(2, n, 5), 7, beta, sigma=1e3, bc=g.BC_INFLOW, g=0.0)
        o.set_variant("nd-grouped2")
        ops.append(o)
    assert not any(_batched(o) for o in ops)
    xs = [torch.rand(o.space.num_dofs, dtype=torch.float64, device="cuda") - 0.5 for o in ops]
    want = []
    for o, x in zip(ops, xs):
        y = torch.empty_like(x)
        o(x, y)
        want.append(y)
    batch = g.Batch(ops)
    assert batch.groups == 0
    ys = [torch.full_like(x, float("nan")) for x in xs]
    batch.apply(xs, ys)
    torch.cuda.synchronize()
    for y, w in zip(ys, want):
        assert torch.equal(y, w)
    batch.close()


def _systems(specs, seed=7):
    rng = np.random.default_rng(seed)
    ops, precs, bs = [], [], []
    for D, n, p in specs:
        sp = _space(D, n, p)
        beta = C.velocity_constant(list(rng.uniform(-1, 1, D)))
        ops.append(g.SystemOperator(sp, p + 2, beta, sigma=1e3, bc=g.BC_INFLOW, g=0.0))
        precs.append(g.MassInverseOperator(sp, p + 2, 1e3))
        bs.append(torch.tensor(rng.uniform(-1, 1, sp.num_dofs), device="cuda"))
    return ops, precs, bs


SOLVE_SPECS = [(2, [40, 33], 3), (3, [12, 10, 9], 2), (4, [6, 5, 4, 5], 1), (3, [16, 8, 8], 3), (2, [25, 30], 5),
               (4, [4, 4, 3, 3], 3), (3, [7, 9, 8], 4)]


@pytest.mark.parametrize("inner", ["fp32", "fp64"])
def test_batch_solver_matches_single_system_solves(inner):
    """The lockstep batched refinement GMRES(20) reaches the same 1e-10 FP64 residual as the
    single-system solver on every system, in the same number of iterations within one (their
    inner products sum in different fixed orders), with solutions equal to rounding; the reported
    residual is the true one."""
    ops, precs, bs = _systems(SOLVE_SPECS)
    batch = g.BatchSolver(ops, precs, restart=20, inner=inner)
    xs = [torch.zeros_like(b) for b in bs]
    res, secs = batch.solve(bs, xs, 2000, 1e-10)
    for A, P, b, x, r, t in zip(ops, precs, bs, xs, res, secs):
        assert r["success"] and r["relative_error"] <= 1e-10, r
        ax = torch.empty_like(x)
        A(x, ax)
        true_rel = (torch.linalg.vector_norm(b - ax) / torch.linalg.vector_norm(b)).item()
        assert abs(true_rel - r["relative_error"]) <= 1e-3 * r["relative_error"] + 1e-15
        x1 = torch.zeros_like(b)
        one = g.GMRESIRSolver(A, 20, inner=inner).precondition(P).solve(b, x1, 2000, 1e-10)
        assert abs(one["iterations"] - r["iterations"]) <= 1, (one, r)
        assert ((x - x1).abs().max() / x1.abs().max()).item() <= 1e-8
        assert t > 0.0


def test_batch_solver_waves_are_independent():
    """Cutting the systems into several waves (a small workspace budget) changes nothing: every
    system's computation depends on its own vectors and partial sums only (bit-identical)."""
    ops, precs, bs = _systems(SOLVE_SPECS, seed=9)
    one = g.BatchSolver(ops, precs, restart=20, inner="fp32")
    many = g.BatchSolver(ops, precs, restart=20, inner="fp32", workspace_bytes=8e6)
    assert one.waves == 1 and many.waves >= 3
    xa = [torch.zeros_like(b) for b in bs]
    xb = [torch.zeros_like(b) for b in bs]
    ra, _ = one.solve(bs, xa, 2000, 1e-10)
    rb, _ = many.solve(bs, xb, 2000, 1e-10)
    assert ra == rb
    for a, b in zip(xa, xb):
        assert torch.equal(a, b)
    # a second solve from the found solutions: the true residual is already below tol
    rc, _ = one.solve(bs, xa, 2000, 1e-10)
    assert all(r["success"] and r["iterations"] == 0 for r in rc)


def test_batch_solver_reports_unconverged_systems():
    ops, precs, bs = _systems(SOLVE_SPECS[:3], seed=11)
    batch = g.BatchSolver(ops, precs, restart=5, inner="fp32")
    xs = [torch.zeros_like(b) for b in bs]
    res, _ = batch.solve(bs, xs, 3, 1e-14)
    assert all(not r["success"] and r["iterations"] == 3 and r["relative_error"] > 1e-14 for r in res)
