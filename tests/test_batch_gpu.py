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
    assert batch.groups == len({(o.space.dim, o.space.order, o.variant) for o in ops if o.kernel == "kronnd"})
    for _ in range(2):  # twice: the parameter upload of the previous apply is reused safely
        ys = [torch.full_like(x, float("nan")) for x in xs]
        batch.apply(xs, ys)
        torch.cuda.synchronize()
        for y, w in zip(ys, want):
            assert torch.equal(y, w)
    batch.close()
