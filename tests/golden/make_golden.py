"""Generate the golden fixtures from the GenDiL reference itself.

Run in a container that holds the reference source (it builds ``oracle/_ref`` first with
``make -C oracle ref``):

    python tests/golden/make_golden.py

It writes ``tests/golden/cases.json`` (case descriptions) and ``tests/golden/golden.npz``
(reference outputs).  Inputs are not stored: they are ``FillRandom(seed)`` draws
(Algebra/vector.hpp:632), which the fixtures also pin (``rng_seed<k>`` prefixes), so the
tests regenerate them bit-exactly.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.bindings import Reference, num_dofs  # noqa: E402


def cube(D, n, P, Q, basis=0, h=None, origin=None, periodic=None, sizes=None):
    sizes = list(sizes) if sizes is not None else [n] * D
    h = list(h) if h is not None else [1.0 / s for s in sizes]
    return {"D": D, "P": P, "Q": Q, "basis": basis, "sizes": sizes, "h": h,
            "origin": list(origin) if origin is not None else [0.0] * D,
            "periodic": list(periodic) if periodic is not None else [0] * D}


def mass_cases():
    c = []
    c.append(("m1", dict(cube(1, 5, 0, 1), sigma_kind=0, sigma_c=1.0)))
    c.append(("m2", dict(cube(1, 7, 3, 5, origin=[0.5]), sigma_kind=1)))
    c.append(("m3", dict(cube(1, 4, 7, 8), sigma_kind=1)))
    c.append(("m4", dict(cube(2, 0, 0, 1, sizes=[3, 4]), sigma_kind=0, sigma_c=2.5)))
    c.append(("m5", dict(cube(2, 0, 2, 4, sizes=[4, 3], h=[0.25, 1 / 3], origin=[-1.0, 0.5]), sigma_kind=1)))
    c.append(("m6", dict(cube(2, 3, 4, 3), sigma_kind=1)))
    c.append(("m7", dict(cube(2, 0, 2, 3, basis=1, sizes=[3, 2]), sigma_kind=1)))
    c.append(("m8", dict(cube(3, 0, 1, 4, sizes=[3, 2, 2]), sigma_kind=1)))
    c.append(("m9", dict(cube(3, 4, 3, 4), sigma_kind=0, sigma_c=1.0)))
    c.append(("m10", dict(cube(3, 3, 3, 6), sigma_kind=1)))
    c.append(("m11", dict(cube(3, 0, 2, 2, basis=1, sizes=[2, 3, 2]), sigma_kind=1)))
    c.append(("m12", dict(cube(3, 2, 7, 8), sigma_kind=1)))
    c.append(("m13", dict(cube(4, 2, 2, 3), sigma_kind=1)))
    c.append(("m14", dict(cube(5, 2, 1, 2), sigma_kind=1)))
    c.append(("m15", dict(cube(6, 2, 1, 2), sigma_kind=1)))
    c.append(("m16", dict(cube(6, 0, 2, 3, sizes=[2, 1, 2, 1, 2, 1]), sigma_kind=1)))
    # single separable products: these also run on the Kronecker-form kernel
    c.append(("m17", dict(cube(3, 0, 3, 4, sizes=[4, 3, 5], h=[0.25, 0.5, 0.2], origin=[-0.5, 0.0, 0.25]),
                          sigma_kind=2)))
    c.append(("m18", dict(cube(3, 0, 1, 2, sizes=[9, 2, 3]), sigma_kind=2)))
    c.append(("m19", dict(cube(3, 0, 4, 5, sizes=[3, 2, 2]), sigma_kind=2)))
    c.append(("m20", dict(cube(3, 0, 3, 4, sizes=[7, 3, 2]), sigma_kind=0, sigma_c=3.5)))
    return c


def adv_cases():
    c = []
    c.append(("a1", dict(cube(1, 6, 0, 1), beta_kind=0, beta_c=[0.7], g=0.3, sigma_kind=0, sigma_c=2.0)))
    c.append(("a2", dict(cube(1, 5, 2, 4), beta_kind=1, g=0.3, sigma_kind=1)))
    c.append(("a2s", dict(cube(1, 5, 2, 4), beta_kind=2, g=0.0, sigma_kind=1)))
    c.append(("a2p", dict(cube(1, 5, 2, 4, periodic=[1]), beta_kind=2, g=0.0, sigma_kind=0, sigma_c=1.0)))
    c.append(("a3", dict(cube(2, 3, 1, 2, basis=1), beta_kind=0, beta_c=[0.7, -0.3], g=0.3, sigma_kind=0, sigma_c=3.0)))
    c.append(("a4", dict(cube(2, 0, 2, 3, sizes=[4, 3], h=[0.25, 1 / 3], origin=[-1.0, 0.5]), beta_kind=2, g=0.3,
                         sigma_kind=1)))
    c.append(("a4b", dict(cube(2, 0, 2, 3, sizes=[4, 3]), beta_kind=1, g=0.0, sigma_kind=1)))
    c.append(("a4p", dict(cube(2, 0, 2, 3, sizes=[4, 3], origin=[-0.5, -0.5]), beta_kind=3, g=0.2, sigma_kind=0,
                          sigma_c=1.0)))
    c.append(("a4per", dict(cube(2, 0, 2, 3, sizes=[4, 3], periodic=[1, 0]), beta_kind=2, g=0.1, sigma_kind=0,
                            sigma_c=1.0)))
    c.append(("a5", dict(cube(2, 3, 4, 3), beta_kind=0, beta_c=[-0.4, 0.9], g=0.5, sigma_kind=0, sigma_c=1.0)))
    c.append(("a6", dict(cube(3, 3, 0, 2), beta_kind=0, beta_c=[0.7, -0.3, 0.4], g=0.3, sigma_kind=0, sigma_c=1.0)))
    c.append(("a7", dict(cube(3, 0, 1, 3, sizes=[3, 2, 4]), beta_kind=1, g=0.0, sigma_kind=1)))
    c.append(("a8", dict(cube(3, 4, 3, 4), beta_kind=2, g=0.0, sigma_kind=0, sigma_c=1000.0)))
    c.append(("a8g", dict(cube(3, 4, 3, 4), beta_kind=2, g=0.3, sigma_kind=1)))
    c.append(("a8per", dict(cube(3, 4, 3, 4, periodic=[1, 0, 1]), beta_kind=2, g=0.0, sigma_kind=0, sigma_c=1.0)))
    c.append(("a9", dict(cube(3, 0, 2, 2, basis=1, sizes=[2, 2, 3]), beta_kind=0, beta_c=[-0.5, 0.25, 0.8], g=0.3,
                         sigma_kind=0, sigma_c=1.0)))
    c.append(("a10", dict(cube(3, 2, 5, 6), beta_kind=2, g=0.0, sigma_kind=1)))
    c.append(("a11", dict(cube(3, 0, 7, 8, sizes=[2, 2, 1]), beta_kind=0, beta_c=[0.3, -0.6, 0.2], g=0.1,
                          sigma_kind=0, sigma_c=1.0)))
    c.append(("a12", dict(cube(4, 0, 1, 2, sizes=[2, 3, 2, 2], origin=[0, 0, -1, -1], h=[0.5, 1 / 3, 1, 1]),
                          beta_kind=3, g=0.0, sigma_kind=1)))
    c.append(("a13", dict(cube(5, 2, 1, 2), beta_kind=0, beta_c=[0.5, -0.5, 0.3, -0.2, 0.1], g=0.2, sigma_kind=0,
                          sigma_c=1.0)))
    c.append(("a14", dict(cube(6, 0, 2, 3, sizes=[2, 2, 1, 2, 1, 2], h=[0.5, 0.5, 1.0, 1.0, 2.0, 1.0],
                          origin=[0, 0, 0, -1, -1, -1]),
                          beta_kind=3, g=0.0, sigma_kind=0, sigma_c=200.0)))
    # 3D shapes that also run on the Kronecker-form kernel (separable velocity and density)
    c.append(("a15", dict(cube(3, 0, 2, 3, sizes=[5, 3, 4], h=[0.2, 1 / 3, 0.25], origin=[0.1, -0.2, 0.0]),
                          beta_kind=2, g=0.2, sigma_kind=2)))
    c.append(("a16", dict(cube(3, 0, 3, 4, sizes=[3, 4, 2]), beta_kind=1, g=0.0, sigma_kind=0, sigma_c=50.0)))
    c.append(("a17", dict(cube(3, 0, 4, 5, sizes=[3, 2, 3]), beta_kind=2, g=0.4, sigma_kind=0, sigma_c=2.0)))
    c.append(("a18", dict(cube(3, 0, 3, 4, sizes=[6, 5, 3]), beta_kind=0, beta_c=[-0.7, 0.3, -0.4], g=0.3,
                          sigma_kind=2)))
    c.append(("a19", dict(cube(3, 0, 3, 3, sizes=[4, 4, 4], periodic=[0, 1, 0]), beta_kind=2, g=0.0, sigma_kind=0,
                          sigma_c=1.0)))
    c.append(("a20", dict(cube(3, 0, 3, 4, sizes=[10, 3, 3]), beta_kind=0, beta_c=[0.0, 0.5, -0.25], g=0.1,
                          sigma_kind=0, sigma_c=1.0)))
    return c


def sipdg_cases():
    """The reference's generic SIPDG form (oracle/part_sipdg.cpp): mu_e = exp(z_e), z_e normal
    with standard deviation 0.5 from numpy seed 4 (configuration 4's field), kappa = 10 (p+1)^2."""
    c = []
    c.append(("s1", dict(cube(2, 0, 1, 3, sizes=[5, 4]), sigma=-1.0, boundary=1)))
    c.append(("s2", dict(cube(2, 0, 2, 4, sizes=[3, 4], periodic=[1, 0]), sigma=-1.0, boundary=1)))
    c.append(("s3", dict(cube(3, 0, 1, 3, sizes=[4, 3, 3]), sigma=-1.0, boundary=1)))
    c.append(("s4", dict(cube(3, 0, 2, 4, sizes=[3, 3, 2]), sigma=-1.0, boundary=0)))
    c.append(("s5", dict(cube(3, 0, 3, 5, sizes=[3, 2, 2]), sigma=1.0, boundary=1)))
    c.append(("s6", dict(cube(3, 0, 4, 6, sizes=[2, 3, 2]), sigma=-1.0, boundary=1)))
    c.append(("s7", dict(cube(3, 0, 4, 6, sizes=[3, 2, 2], h=[0.2, 0.5, 0.25]), sigma=0.0, boundary=1)))
    # Gauss-Legendre nodes (the traces are full contractions, not end values) and a 4D mesh
    c.append(("s8", dict(cube(2, 0, 2, 4, basis=1, sizes=[4, 3]), sigma=-1.0, boundary=1)))
    c.append(("s9", dict(cube(3, 0, 2, 4, basis=1, sizes=[3, 2, 3], periodic=[0, 1, 0]), sigma=1.0, boundary=1)))
    c.append(("s10", dict(cube(4, 0, 1, 3, sizes=[3, 2, 3, 2], periodic=[0, 0, 1, 0]), sigma=-1.0, boundary=1)))
    return c


def diffusion_cases():
    """The reference's legacy MakeDiffusionOperator (oracle/part_sipdg.cpp): constant diffusivity,
    interior and boundary faces; the 1D case is the two-element periodic mesh of the reference's
    tests/integration/gendil/test-diffusion-symmetry-1d-minimal.cpp (sigma = 1, kappa = 0)."""
    c = []
    c.append(("d1", dict(cube(1, 0, 1, 4, sizes=[2], periodic=[1]), diffusivity=1.0, sigma=1.0, kappa=0.0)))
    c.append(("d2", dict(cube(1, 0, 1, 4, sizes=[7]), diffusivity=0.8, sigma=-1.0, kappa=40.0)))
    c.append(("d3", dict(cube(2, 0, 1, 3, sizes=[5, 4]), diffusivity=1.0, sigma=1.0, kappa=0.0)))
    c.append(("d4", dict(cube(3, 0, 2, 4, sizes=[3, 3, 3], periodic=[1, 1, 1]), diffusivity=2.5, sigma=-1.0,
                         kappa=90.0)))
    c.append(("d5", dict(cube(3, 0, 3, 5, sizes=[3, 2, 2]), diffusivity=0.7, sigma=0.0, kappa=160.0)))
    c.append(("d6", dict(cube(3, 0, 4, 6, sizes=[2, 3, 2], h=[0.5, 0.25, 1 / 3]), diffusivity=1.3, sigma=-1.0,
                         kappa=250.0)))
    c.append(("d7", dict(cube(3, 0, 2, 4, basis=1, sizes=[3, 3, 2]), diffusivity=0.9, sigma=-1.0, kappa=90.0)))
    return c


def c5_shapes():
    """The element shapes of the batched uneven instances: dimension 2..4, order 1..5, q = p + 2,
    constant velocity with components uniform in [-1, 1] (numpy seed 7), sigma = 1/dt = 1e3."""
    rng = np.random.default_rng(7)
    sizes = {2: [5, 4], 3: [3, 2, 3], 4: [2, 2, 2, 2]}
    out = []
    for D in (2, 3, 4):
        for P in range(1, 6):
            sz = [3, 2, 2, 2] if (D == 4 and P <= 2) else sizes[D]
            beta = [float(v) for v in rng.uniform(-1.0, 1.0, D)]
            out.append((f"c5_d{D}p{P}", dict(cube(D, 0, P, P + 2, sizes=sz), beta_kind=0, beta_c=beta, g=0.0,
                                             sigma_kind=0, sigma_c=1e3)))
    return out


def sampled(arrays, key, v, stride):
    """Every `stride`-th value of a large reference output and its max-norm, 2-norm and sum."""
    arrays[f"{key}_sample"] = np.ascontiguousarray(v[::stride])
    arrays[f"{key}_stats"] = np.array([np.abs(v).max(), np.linalg.norm(v), v.sum()])


def config_fixtures(ref, cases, arrays):
    """The benchmark configurations at their stated sizes, pinned against the reference:
    C1 (16^3 mass, p = 3, q = 4: the apply and 20 CG iterations of M x = M u from x0 = 0),
    C2 (64^3 implicit system sigma M + A, sigma = 1/dt = 1e3: GMRES(30) to 1e-10 from x0 = 0,
    b = FillRandom(2); about 15 minutes on 8 cores), C3 (the 6D phase-space operator on a 4^6 mesh:
    interior faces on every axis) and the shapes of C5 (full outputs).  Large outputs are stored as
    strided samples plus norms."""
    c1 = dict(cube(3, 16, 3, 4), sigma_kind=0, sigma_c=1.0, seed=0, cg_iters=20, cg_tol=0.0, stride=61)
    u = ref.fill_random(num_dofs(c1), 0)
    y = ref.mass_apply(c1, u)
    sampled(arrays, "c1_y", y, c1["stride"])
    # the reference's CG on this system amplifies rounding from about 8 iterations on (its own
    # iterates at 1 and 3 OpenMP threads differ by 3e-14 after 5 iterations, 1.4e-11 after 8 and
    # 4e-3 after 20), so the trace is stored at 5 and 8 iterations as well as at 20
    traces = {}
    for k in (5, 8, c1["cg_iters"]):
        x, info = ref.mass_cg(c1, y, np.zeros_like(y), k, c1["cg_tol"])
        sampled(arrays, f"c1_x{k}", x, c1["stride"])
        traces[str(k)] = info
    cases["configs"].append({"id": "c1", "kind": "mass_cg", **c1, "traces": traces})
    print("c1", traces, flush=True)

    c3 = dict(cube(6, 4, 2, 3, h=[0.25] * 3 + [0.5] * 3, origin=[0.0] * 3 + [-1.0] * 3), beta_kind=3, g=0.0,
              seed=1, stride=97)
    x3 = ref.fill_random(num_dofs(c3), 1)
    sampled(arrays, "c3_y", ref.advection_apply(c3, x3, 1), c3["stride"])
    cases["configs"].append({"id": "c3", "kind": "advection_apply", "mode": 1, **c3})
    print("c3 done", flush=True)

    for cid, case in c5_shapes():
        case = dict(case, seed=1)
        xc = ref.fill_random(num_dofs(case), 1)
        arrays[f"{cid}_mass_y"] = ref.mass_apply(case, xc)
        arrays[f"{cid}_adv_y"] = ref.advection_apply(case, xc, 1)
        cases["configs"].append({"id": cid, "kind": "system_parts", **case})
    print("c5 done", flush=True)

    c2 = dict(cube(3, 64, 3, 4), beta_kind=2, g=0.0, sigma_c=1e3, seed=2, restart=30, tol=1e-10, max_iters=5000,
              stride=4099)
    b = ref.fill_random(num_dofs(c2), 2)
    x2, info = ref.system_gmres(c2, b, np.zeros_like(b), c2["max_iters"], c2["restart"], c2["tol"])
    sampled(arrays, "c2_x", x2, c2["stride"])
    cases["configs"].append({"id": "c2", "kind": "system_gmres", **c2, **info, "threads": ref.num_threads()})
    print("c2", info, flush=True)


def main(only=None):
    """Write cases.json and golden.npz.  With `only` (a case kind), regenerate that kind alone and
    keep every other stored case and array as it is (the OpenMP reference solvers' last bits
    depend on the thread schedule, so regenerating them all would churn the fixtures)."""
    if only is not None:
        with open(os.path.join(HERE, "cases.json")) as f:
            old_cases = json.load(f)
        with np.load(os.path.join(HERE, "golden.npz")) as z:
            old_arrays = {k: z[k] for k in z.files}
        old_cases.setdefault("configs", [])
        new_cases, new_arrays = build(only)
        kinds = [only] + (["diffusion"] if only == "sipdg" else [])
        ids = {c["id"] for k in kinds for c in new_cases[k]}
        for k in kinds:
            old_cases[k] = new_cases[k]
        for k in list(old_arrays):
            if k.split("_")[0] in ids:
                del old_arrays[k]
        old_arrays.update(new_arrays)
        write(old_cases, old_arrays)
        return
    write(*build(None))


def write(cases, arrays):
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(cases, f, indent=1)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **arrays)
    total = sum(a.nbytes for a in arrays.values())
    print(f"wrote {len(arrays)} arrays ({total / 1e6:.2f} MB raw)")


def build(only):
    ref = Reference()
    cases = {"mass": [], "advection": [], "cg": [], "gmres": [], "sipdg": [], "diffusion": [], "configs": []}
    arrays = {}
    if only == "sipdg":
        sipdg_fixtures(ref, cases, arrays)
        return cases, arrays
    if only == "configs":
        config_fixtures(ref, cases, arrays)
        return cases, arrays
    for seed in (0, 1, 2, 3, 12345):
        arrays[f"rng_seed{seed}"] = ref.fill_random(256, seed)
    for kind in (0, 1):
        for n in range(1, 9):
            c, w = ref.points(kind, n)
            arrays[f"points_{kind}_{n}_x"] = c
            arrays[f"points_{kind}_{n}_w"] = w
    for cid, case in mass_cases():
        case = dict(case, seed=0)
        x = ref.fill_random(num_dofs(case), case["seed"])
        arrays[f"{cid}_y"] = ref.mass_apply(case, x)
        cases["mass"].append({"id": cid, **case})
    for cid, case in adv_cases():
        case = dict(case, seed=1)
        x = ref.fill_random(num_dofs(case), case["seed"])
        for mode in (0, 1, 2):
            arrays[f"{cid}_mode{mode}_y"] = ref.advection_apply(case, x, mode)
        cases["advection"].append({"id": cid, **case})
    sipdg_fixtures(ref, cases, arrays)
    config_fixtures(ref, cases, arrays)
    # CG on the mass operator: b = M u (u from seed 0), x0 = 0 (conjugategradient.hpp:125)
    for cid, case, iters, tol in (("cg1", dict(cube(3, 4, 3, 4), sigma_kind=0, sigma_c=1.0), 20, 1e-6),
                                  ("cg2", dict(cube(3, 4, 3, 4), sigma_kind=1), 500, 1e-12),
                                  ("cg3", dict(cube(1, 10, 3, 5), sigma_kind=0, sigma_c=1.0), 500, 1e-12)):
        u = ref.fill_random(num_dofs(case), 0)
        try:
            b = ref.mass_apply(case, u)
            x, info = ref.mass_cg(case, b, np.zeros_like(b), iters, tol)
        except NotImplementedError:
            continue
        arrays[f"{cid}_x"] = x
        cases["cg"].append({"id": cid, **case, "max_iters": iters, "tol": tol, **info})
    # GMRES(30) on sigma M + A, b from seed 2 (gmres.hpp:74)
    for cid, case, dt in (("gm1", dict(cube(3, 4, 3, 4), beta_kind=2, g=0.0), 1e-3),
                          ("gm2", dict(cube(2, 8, 2, 3), beta_kind=2, g=0.0), 1e-3),
                          ("gm3", dict(cube(1, 16, 2, 4), beta_kind=1, g=0.0), 1e-2)):
        case = dict(case, sigma_c=1.0 / dt)
        b = ref.fill_random(num_dofs(case), 2)
        x, info = ref.system_gmres(case, b, np.zeros_like(b), 5000, 30, 1e-10)
        arrays[f"{cid}_x"] = x
        cases["gmres"].append({"id": cid, **case, "restart": 30, "tol": 1e-10, "max_iters": 5000, **info})
    return cases, arrays


def sipdg_fixtures(ref, cases, arrays):
    for cid, case in sipdg_cases():
        ne = int(np.prod(case["sizes"]))
        mu = np.exp(np.random.default_rng(4).normal(0.0, 0.5, ne))
        kappa = 10.0 * (case["P"] + 1) ** 2
        case = dict(case, seed=5, kappa=kappa)
        x = ref.fill_random(num_dofs(case), case["seed"])
        arrays[f"{cid}_mu"] = mu
        arrays[f"{cid}_y"] = ref.sipdg_apply(case, mu, case["sigma"], kappa, case["boundary"], x)
        # coefficient gradient lam^T (dA/dmu_e) x, lam from seed 6: A is linear in mu, so the
        # derivative is the reference operator with the one-hot diffusivity of element e
        lam = ref.fill_random(num_dofs(case), 6)
        grad = np.empty(ne)
        for e in range(ne):
            onehot = np.zeros(ne)
            onehot[e] = 1.0
            grad[e] = lam @ ref.sipdg_apply(case, onehot, case["sigma"], kappa, case["boundary"], x)
        arrays[f"{cid}_grad"] = grad
        cases["sipdg"].append({"id": cid, **case, "grad_seed": 6})
    for cid, case in diffusion_cases():
        case = dict(case, seed=5)
        x = ref.fill_random(num_dofs(case), case["seed"])
        arrays[f"{cid}_y"] = ref.diffusion_legacy_apply(case, case["diffusivity"], case["sigma"], case["kappa"], x)
        cases["diffusion"].append({"id": cid, **case})


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=["sipdg", "configs"], help="regenerate one case kind, keep the rest")
    main(ap.parse_args().only)
