"""The C++20 facade (include/gendil_b200/gendil.hpp): GenDiL's names and call shapes over the C ABI.

tests/cpp/facade_cases.cpp is compiled here with g++ -std=c++20 against libdgop.so.  Its `plan`
mode runs on the host (weak-form recognition, coefficient separation, rejection of forms and
coefficients outside the hot path); its `run` mode applies legacy-factory and weak-form operators
and runs the Krylov drivers on the GPU, and every vector is checked against the oracle."""
import os
import struct
import subprocess

import numpy as np
import pytest

from helpers import APPLY_TOL, golden, oracle, rel_max

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def facade_bin(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("facade") / "facade_cases")
    lib = os.path.join(ROOT, "gendil_b200")
    cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", "facade_cases.cpp"), "-o", out,
           "-L" + lib, "-ldgop", "-L" + os.path.join(CUDA, "lib64"), "-lcudart",
           "-Wl,-rpath," + lib + ":" + os.path.join(CUDA, "lib64")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_facade_recognises_hot_path_forms_and_rejects_others(facade_bin):
    r = subprocess.run([facade_bin, "plan"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = {}
    for line in r.stdout.splitlines():
        kind, name, rest = line.split(" ", 2)
        lines[name.rstrip(":")] = rest if kind in ("plan", "separated") else "rejected " + rest
    assert lines["mass"] == "mass sigma=const*1"
    assert lines["mass_coef"] == "mass sigma=sigma*1"
    assert lines["mass_scaled"] == "mass sigma=const*1000"
    assert lines["advection"] == "cell+interior beta=beta"
    assert lines["advection_outflow"] == "cell+interior+boundary beta=beta"
    assert lines["system"] == "mass+cell+interior+boundary sigma=const*1000 beta=beta"
    for bad in ("reject_cell_only", "reject_wrong_sign", "reject_grad_grad", "reject_average", "reject_two_mass"):
        assert lines[bad].startswith("rejected"), lines[bad]
    # constant, one axis, 1 + x y + z^2 (two terms), a three-factor product, a sum over three axes
    assert lines["const"] == "terms=0"
    assert lines["one_axis"] == "terms=1"
    assert lines["poly"] == "terms=2"
    assert lines["sep"] == "terms=1"
    assert lines["additive"] == "terms=3"
    assert "not a sum of products" in lines["reject_nonsep"]


def _read_records(path):
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos < len(data):
        (ln,) = struct.unpack_from("<I", data, pos)
        pos += 4
        name = data[pos:pos + ln].decode()
        pos += ln
        (n,) = struct.unpack_from("<Q", data, pos)
        pos += 8
        out[name] = np.frombuffer(data, dtype=np.float64, count=n, offset=pos).copy()
        pos += 8 * n
    return out


def _cube(D, n, P, Q, **kw):
    sizes = kw.pop("sizes", [n] * D)
    return {"D": D, "P": P, "Q": Q, "basis": 0, "sizes": sizes, "h": [1.0 / s for s in sizes], "origin": [0.0] * D,
            "periodic": [0] * D, **kw}


@pytest.mark.gpu
def test_facade_operators_and_solvers_match_the_oracle(facade_bin, tmp_path):
    out = str(tmp_path / "vectors.bin")
    r = subprocess.run([facade_bin, "run", out], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    vec = _read_records(out)
    solves, checks = {}, {}
    for line in r.stdout.splitlines():
        if line.startswith("solve "):
            _, name, ok, it, rel = line.split()
            solves[name] = {"success": ok == "1", "iterations": int(it), "relative_error": float(rel)}
        elif line.startswith("check "):
            _, name, val = line.split()
            checks[name] = float(val)
    o = oracle()
    fr = lambda case, seed: o.fill_random(int(np.prod(case["sizes"])) * (case["P"] + 1) ** case["D"], seed)

    a = _cube(3, 8, 3, 4, sigma_kind=1)
    ya = o.mass_apply(a, fr(a, 0))
    assert rel_max(vec["A_legacy"], ya) <= APPLY_TOL
    assert rel_max(vec["A_generic"], ya) <= APPLY_TOL

    b = _cube(3, 6, 2, 3, sigma_kind=2)
    assert rel_max(vec["B_legacy"], o.mass_apply(b, fr(b, 0))) <= APPLY_TOL

    c = _cube(3, 8, 3, 4, beta_kind=2, g=0.0)
    xc = fr(c, 1)
    y_bc, y_nobc = o.advection_apply(c, xc, 1), o.advection_apply(c, xc, 0)
    for name in ("C_legacy_bc", "C_generic_bc"):
        assert rel_max(vec[name], y_bc) <= APPLY_TOL, name
    for name in ("C_legacy_nobc", "C_generic_nobc"):
        assert rel_max(vec[name], y_nobc) <= APPLY_TOL, name

    d = _cube(3, 6, 2, 3, beta_kind=1, sigma_kind=0, sigma_c=10.0)
    assert rel_max(vec["D_legacy"], o.advection_apply(d, fr(d, 1), 2)) <= APPLY_TOL

    e = _cube(2, 0, 4, 5, sizes=[7, 9], beta_kind=0, beta_c=[0.7, -0.4], g=0.75)
    assert rel_max(vec["E_legacy_bc"], o.advection_apply(e, fr(e, 1), 1)) <= APPLY_TOL

    f = _cube(3, 16, 3, 4, sigma_kind=0, sigma_c=1.0)
    bf = o.mass_apply(f, fr(f, 0))
    xf, info = o.mass_cg(f, bf, np.zeros_like(bf), 20, 1e-6)
    assert solves["F_cg"]["success"] == info["success"]
    assert abs(solves["F_cg"]["iterations"] - info["iterations"]) <= 1
    if info["success"]:
        assert rel_max(vec["F_cg_x"], xf) < 1e-6
    else:
        # an unconverged CG iterate is rounding-sensitive (the reference's own moves with its
        # OpenMP thread count): compare the size of the reported error only
        assert 0.5 * info["relative_error"] < solves["F_cg"]["relative_error"] < 2.0 * info["relative_error"]

    cases, arr = golden()
    gm1 = next(cs for cs in cases["gmres"] if cs["id"] == "gm1")
    assert solves["G_gmres"]["success"] and abs(solves["G_gmres"]["iterations"] - gm1["iterations"]) <= 1
    assert rel_max(vec["G_gmres_x"], arr["gm1_x"]) < 1e-8
    assert solves["G_refined"]["success"] and solves["G_refined"]["relative_error"] <= 1e-10
    assert rel_max(vec["G_refined_x"], arr["gm1_x"]) < 1e-8

    # adjoint gradient (AdvectionSolveFunction) against central differences
    assert solves["H_forward"]["success"] and solves["H_adjoint"]["success"]
    assert checks["H_fd"] <= 1e-6

    # diffusion coefficient gradient (DiffusionSolveFunction) against central differences, every
    # element, relative to the element's own gradient
    assert solves["K_forward"]["success"] and solves["K_adjoint"]["success"]
    assert checks["K_fd_rel"] <= 1e-6

    # legacy diffusion operator (MakeDiffusionOperator) against the reference's own output
    assert rel_max(vec["I_diffusion"], arr["d4_y"]) <= APPLY_TOL
    assert checks["I_kernel_is_diffusion"] == 1 and checks["I_rejects_varying"] == 1
    assert checks["J_copy_exact"] == 1
