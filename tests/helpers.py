"""Shared test helpers: golden fixtures, oracle access, operator construction from case dicts."""
from __future__ import annotations

import json
import os

import numpy as np

from oracle.bindings import Oracle, Reference, have_oracle, have_reference, num_dofs  # noqa: F401

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# FP64 apply parity bar: relative error in max norm, per apply.
APPLY_TOL = 1e-13


def golden():
    with open(os.path.join(GOLDEN_DIR, "cases.json")) as f:
        cases = json.load(f)
    arrays = np.load(os.path.join(GOLDEN_DIR, "golden.npz"))
    return cases, arrays


def rel_max(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))


_oracle = None


def oracle():
    global _oracle
    if _oracle is None:
        _oracle = Oracle()
    return _oracle


def inputs(case, seed=None):
    return oracle().fill_random(num_dofs(case), case["seed"] if seed is None else seed)


def make_space(case):
    import gendil_b200 as g
    return g.Space(case["D"], case["sizes"], case["h"], case.get("origin"), case.get("periodic"), case["P"],
                   case["basis"])


def make_operator(case, kind, mode=1, space=None):
    """kind: 'mass' or 'adv'; mode (adv): 0 no boundary faces, 1 inflow g, 2 mass + advection."""
    import gendil_b200 as g
    from gendil_b200 import coefficients as C
    sp = space or make_space(case)
    D, Q = case["D"], case["Q"]
    sigma = C.sigma_preset(case.get("sigma_kind", 0), D, case.get("sigma_c", 1.0))
    if kind == "mass":
        return g.MassOperator(sp, Q, sigma)
    beta = C.beta_preset(case.get("beta_kind", 0), D, case.get("beta_c"))
    if mode == 0:
        return g.AdvectionOperator(sp, Q, beta, bc=g.BC_NONE)
    if mode == 1:
        return g.AdvectionOperator(sp, Q, beta, bc=g.BC_INFLOW, g=case.get("g", 0.0))
    return g.MassAdvectionOperator(sp, Q, beta, sigma)


def cuda_apply(op, x_np, transpose=False, f32=False):
    import torch
    dt = torch.float32 if f32 else torch.float64
    x = torch.from_numpy(np.asarray(x_np)).to(device="cuda", dtype=dt)
    y = torch.empty_like(x)
    if transpose:
        op.apply_transpose(x, y)
    elif f32:
        op.apply_f32(x, y)
    else:
        op(x, y)
    torch.cuda.synchronize()
    return y.double().cpu().numpy()
