"""GPU: the sm_100a operators against the reference's golden outputs and the oracle.

FP64 applies must match to APPLY_TOL = 1e-13 relative in max norm per apply.  Every case runs on
the generic sum-factorized kernel and, where eligible, on the Kronecker-form kernels (the 3D
register kernel and the any-dimension shared-memory kernel)."""
import numpy as np
import pytest

from helpers import APPLY_TOL, cuda_apply, golden, inputs, make_operator, oracle, rel_max

pytestmark = pytest.mark.gpu
CASES, ARR = golden()
KERNELS = ["generic", "kron", "kronnd"]


def _select(op, kernel):
    if kernel == "kron" and op.kernel != "kron":
        pytest.skip(f"not eligible for the Kronecker kernel: {op.kernel_note}")
    if kernel == "kronnd" and op.kernel != "kronnd":
        import gendil_b200 as g
        try:
            op.select_kernel("kronnd")
        except g.DGOPError as exc:
            pytest.skip(f"not eligible for the any-dimension Kronecker kernel: {exc}")
    if kernel == "generic" and op.kernel != "generic":
        import gendil_b200 as g
        try:
            op.select_kernel("generic")
        except g.DGOPError as exc:
            pytest.skip(f"generic kernel not built for this shape: {exc}")
    return op


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("case", CASES["mass"], ids=lambda c: c["id"])
def test_mass_vs_reference_golden(case, kernel):
    op = _select(make_operator(case, "mass"), kernel)
    y = cuda_apply(op, inputs(case))
    assert rel_max(y, ARR[f"{case['id']}_y"]) <= APPLY_TOL


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("case", CASES["advection"], ids=lambda c: c["id"])
def test_advection_vs_reference_golden(case, mode, kernel):
    op = _select(make_operator(case, "adv", mode), kernel)
    y = cuda_apply(op, inputs(case))
    assert rel_max(y, ARR[f"{case['id']}_mode{mode}_y"]) <= APPLY_TOL


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("case", CASES["advection"], ids=lambda c: c["id"])
def test_transpose_adjoint_identity(case, mode, kernel):
    """<A x, z> = <x, A^T z> for the linear part (inflow value 0)."""
    case = dict(case, g=0.0)
    op = _select(make_operator(case, "adv", mode), kernel)
    x = inputs(case, seed=5)
    z = inputs(case, seed=6)
    ax = cuda_apply(op, x)
    atz = cuda_apply(op, z, transpose=True)
    lhs, rhs = float(ax @ z), float(x @ atz)
    assert abs(lhs - rhs) <= 1e-12 * (np.abs(ax).sum() * np.abs(z).max() + 1e-300)


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("case", CASES["advection"], ids=lambda c: c["id"])
def test_transpose_kronnd_agrees_with_generic(case, mode):
    """The any-dimension Kronecker kernel and the generic kernel give the same A^T x."""
    import gendil_b200 as g
    case = dict(case, g=0.0)
    op = make_operator(case, "adv", mode)
    try:
        op.select_kernel("kronnd")
    except g.DGOPError:
        pytest.skip("not eligible for the any-dimension Kronecker kernel")
    x = inputs(case, seed=7)
    yk = cuda_apply(op, x, transpose=True)
    try:
        op.select_kernel("generic")
    except g.DGOPError:
        pytest.skip("generic kernel not built for this shape")
    yg = cuda_apply(op, x, transpose=True)
    assert rel_max(yk, yg) <= APPLY_TOL


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("case", [c for c in CASES["advection"] if c["D"] == 3], ids=lambda c: c["id"])
def test_transpose_kernels_agree(case, mode):
    """Both kernel families give the same A^T x."""
    case = dict(case, g=0.0)
    op = make_operator(case, "adv", mode)
    if op.kernel != "kron":
        pytest.skip("not eligible for the Kronecker kernel")
    x = inputs(case, seed=7)
    yk = cuda_apply(op, x, transpose=True)
    _select(op, "generic")
    yg = cuda_apply(op, x, transpose=True)
    assert rel_max(yk, yg) <= APPLY_TOL


def _c1():
    return {"D": 3, "P": 3, "Q": 4, "basis": 0, "sizes": [16] * 3, "h": [1 / 16] * 3, "origin": [0.0] * 3,
            "periodic": [0] * 3, "sigma_kind": 0, "sigma_c": 1.0, "seed": 0}


def _c2(n=64):
    return {"D": 3, "P": 3, "Q": 4, "basis": 0, "sizes": [n] * 3, "h": [1 / n] * 3, "origin": [0.0] * 3,
            "periodic": [0] * 3, "beta_kind": 2, "g": 0.0, "seed": 1}


@pytest.mark.parametrize("kernel", KERNELS)
def test_config1_mass_full_size_vs_oracle(kernel):
    case = _c1()
    x = inputs(case)
    op = _select(make_operator(case, "mass"), kernel)
    y = cuda_apply(op, x)
    assert rel_max(y, oracle().mass_apply(case, x)) <= APPLY_TOL


@pytest.mark.parametrize("kernel", KERNELS)
def test_config2_advection_full_size_vs_oracle(kernel):
    case = _c2(64)
    x = inputs(case)
    op = _select(make_operator(case, "adv", 1), kernel)
    y = cuda_apply(op, x)
    assert rel_max(y, oracle().advection_apply(case, x, 1)) <= APPLY_TOL


def test_config2_uses_kronecker_kernel():
    op = make_operator(_c2(8), "adv", 1)
    assert op.kernel == "kron", op.kernel_note


@pytest.mark.parametrize("kernel", KERNELS)
def test_fp32_apply_error_bound(kernel):
    case = _c2(16)
    op = _select(make_operator(case, "adv", 1), kernel)
    x = inputs(case)
    y64 = cuda_apply(op, x)
    y32 = cuda_apply(op, x, f32=True)
    assert rel_max(y32, y64) < 1e-5


@pytest.mark.parametrize("kernel", KERNELS)
def test_apply_ex_alpha_beta(kernel):
    import torch
    case = _c2(8)
    op = _select(make_operator(case, "adv", 1), kernel)
    x = torch.from_numpy(inputs(case)).cuda()
    y0 = torch.from_numpy(inputs(case, seed=9)).cuda()
    ax = torch.empty_like(x)
    op(x, ax)
    y = y0.clone()
    op.apply(x, y, alpha=2.5, beta=-0.5)
    ref = 2.5 * ax - 0.5 * y0
    assert float((y - ref).abs().max() / ref.abs().max()) < 1e-14


VARIANT_CASES = [
    # (id, case, kind, mode): advection with inflow, mass + advection with a separate mass term,
    # odd order, FP64 and FP32
    ("adv_p3_sincos", {"D": 3, "P": 3, "Q": 4, "basis": 0, "sizes": [9, 6, 5], "h": [1 / 9, 1 / 6, 0.2],
                       "origin": [0.0] * 3, "periodic": [0] * 3, "beta_kind": 2, "g": 0.5}, "adv", 1),
    ("sys_p2_bubble", {"D": 3, "P": 2, "Q": 3, "basis": 0, "sizes": [7, 5, 6], "h": [1 / 7, 0.2, 1 / 6],
                       "origin": [0.0] * 3, "periodic": [0] * 3, "beta_kind": 1, "sigma_kind": 2, "g": 0.0}, "adv", 2),
    ("mass_p1", {"D": 3, "P": 1, "Q": 2, "basis": 0, "sizes": [11, 3, 4], "h": [1 / 11, 1 / 3, 0.25],
                 "origin": [0.0] * 3, "periodic": [0, 1, 0], "sigma_kind": 1}, "mass", 1),
    # p = 3 with the x extent a multiple of 8: the bulk-tensor (TMA) variants run too.  Inflow
    # faces on both sides of every axis (the bubble velocity changes sign), periodic axes (wrapped
    # neighbours come from global memory), a separate mass term, the mass operator alone, several
    # x-rows per mesh
    ("tma_adv_sincos", {"D": 3, "P": 3, "Q": 4, "basis": 0, "sizes": [16, 3, 5], "h": [1 / 16, 1 / 3, 0.2],
                        "origin": [0.0] * 3, "periodic": [0] * 3, "beta_kind": 2, "g": 0.5}, "adv", 1),
    ("tma_adv_bubble_noBC", {"D": 3, "P": 3, "Q": 4, "basis": 0, "sizes": [8, 6, 4], "h": [1 / 8, 1 / 6, 0.25],
                             "origin": [0.0] * 3, "periodic": [0] * 3, "beta_kind": 1, "g": 0.0}, "adv", 0),
    ("tma_adv_periodic", {"D": 3, "P": 3, "Q": 4, "basis": 0, "sizes": [8, 4, 3], "h": [1 / 8, 0.25, 1 / 3],
                          "origin": [-0.5, 0.0, 0.0], "periodic": [1, 1, 1], "beta_kind": 0,
                          "beta_c": [-0.7, 0.4, -0.3], "g": 0.0}, "adv", 1),
    ("tma_sys_sep", {"D": 3, "P": 3, "Q": 4, "basis": 0, "sizes": [24, 2, 3], "h": [1 / 24, 0.5, 1 / 3],
                     "origin": [0.0] * 3, "periodic": [0] * 3, "beta_kind": 1, "sigma_kind": 2, "g": 0.0}, "adv", 2),
    ("tma_mass", {"D": 3, "P": 3, "Q": 4, "basis": 0, "sizes": [8, 5, 2], "h": [1 / 8, 0.2, 0.5],
                  "origin": [0.0] * 3, "periodic": [0] * 3, "sigma_kind": 2}, "mass", 1),
]

TMA_VARIANTS = ("tma1-tile", "tma2-shfl", "tma2-tile")


@pytest.mark.parametrize("cid,case,kind,mode", VARIANT_CASES, ids=[c[0] for c in VARIANT_CASES])
def test_kron_variants_are_bit_identical(cid, case, kind, mode):
    """Every Kronecker-kernel variant the autotuner can pick computes the same bits as the others
    of its family (forward, transposed and FP32 applies): the staged variants among themselves and
    the bulk-tensor variants among themselves; the two families agree to a few ulps (the
    bulk-tensor variants accumulate each term's last pass onto the sum), and every forward apply
    meets the parity bar."""
    op = make_operator(case, kind, mode)
    if op.kernel != "kron":
        pytest.skip(op.kernel_note)
    assert op.variant in op.VARIANTS
    x = inputs(dict(case, seed=1))
    ref = {}
    for name in op.VARIANTS:
        try:
            op.set_variant(name)
        except RuntimeError:
            # shuffles need an even N = P + 1; the bulk-tensor variants p = 3 and an x extent
            # that is a multiple of 8
            assert (name == "stage2-shfl" and case["P"] % 2 == 0) or \
                (name in TMA_VARIANTS and (case["P"] != 3 or case["sizes"][0] % 8))
            continue
        if name in TMA_VARIANTS:
            assert case["P"] == 3 and case["sizes"][0] % 8 == 0
        got = (cuda_apply(op, x), cuda_apply(op, x, transpose=True), cuda_apply(op, x, f32=True))
        assert op.device_error() == 0, name
        fam = name in TMA_VARIANTS
        want = oracle().mass_apply(case, x) if kind == "mass" else oracle().advection_apply(case, x, mode)
        assert rel_max(got[0], want) <= APPLY_TOL, name
        if fam not in ref:
            ref[fam] = got
        else:
            for a, b in zip(got, ref[fam]):
                assert np.array_equal(a, b), name
    if len(ref) == 2:
        for a, b in zip(ref[True][:2], ref[False][:2]):
            assert rel_max(a, b) <= 1e-15
    op.set_variant(None)  # the autotuner again
    assert op.variant in op.VARIANTS


HOSTIO_CASES = [
    ("adv_kron", {"D": 3, "P": 3, "Q": 4, "basis": 0, "sizes": [6, 5, 7], "h": [1 / 6, 0.2, 1 / 7],
                  "origin": [0.0] * 3, "periodic": [0] * 3, "beta_kind": 2, "g": 0.5}, "adv", 1, 3),
    ("adv_periodic_z", {"D": 3, "P": 2, "Q": 3, "basis": 0, "sizes": [4, 3, 9], "h": [0.25, 1 / 3, 1 / 9],
                        "origin": [0.0] * 3, "periodic": [0, 0, 1], "beta_kind": 0, "beta_c": [0.3, -0.2, 0.7],
                        "g": 0.0}, "adv", 1, 4),
    ("mass_2d", {"D": 2, "P": 4, "Q": 5, "basis": 0, "sizes": [7, 9], "h": [1 / 7, 1 / 9], "origin": [0.0] * 2,
                 "periodic": [0] * 2, "sigma_kind": 1}, "mass", 1, 5),
    ("sys_generic_1d", {"D": 1, "P": 5, "Q": 6, "basis": 1, "sizes": [33], "h": [1 / 33], "origin": [0.0],
                        "periodic": [1], "beta_kind": 0, "beta_c": [-0.8], "sigma_kind": 0, "sigma_c": 3.0}, "adv", 2, 8),
]


@pytest.mark.parametrize("cid,case,kind,mode,slabs", HOSTIO_CASES, ids=[c[0] for c in HOSTIO_CASES])
def test_host_io_apply_equals_device_apply(cid, case, kind, mode, slabs):
    """dgop_host_io_apply (upload, per-slab applies and download pipelined) gives the bits of the
    device apply, including periodic last axes and more slabs than planes."""
    import torch
    import gendil_b200 as g
    op = make_operator(case, kind, mode)
    x = inputs(dict(case, seed=1))
    want = cuda_apply(op, x)
    for s in (1, slabs, 64):
        io = g.HostIO(op, slabs=s)
        xh = torch.from_numpy(x).pin_memory()
        yh = torch.full_like(xh, float("nan")).pin_memory()
        io.apply(xh, yh)
        assert np.array_equal(yh.numpy(), want), s
        y2 = np.full_like(x, np.nan)  # pageable host memory
        io.apply(x, y2)
        assert np.array_equal(y2, want), s
        io.close()


@pytest.mark.parametrize("variant", TMA_VARIANTS)
def test_host_io_slabs_on_bulk_tensor_variants(variant):
    """Host-vector applies run the operator on slabs of z planes; with an x extent that is a
    multiple of 8 every slab is a whole number of 8-element groups, so the bulk-tensor variants
    run on element ranges (neighbour slices of other slabs, a periodic last axis).  Every slab
    count gives the bits of the device apply with the same variant."""
    import torch
    import gendil_b200 as g
    case = {"D": 3, "P": 3, "Q": 4, "basis": 0, "sizes": [8, 3, 6], "h": [1 / 8, 1 / 3, 1 / 6],
            "origin": [0.0] * 3, "periodic": [0, 0, 1], "beta_kind": 2, "g": 0.5}
    op = make_operator(case, "adv", 1)
    assert op.kernel == "kron"
    op.set_variant(variant)
    x = inputs(dict(case, seed=1))
    want = cuda_apply(op, x)
    assert op.device_error() == 0
    assert rel_max(want, oracle().advection_apply(case, x, 1)) <= APPLY_TOL
    for s in (1, 2, 4, 64):
        io = g.HostIO(op, slabs=s)
        xh = torch.from_numpy(x).pin_memory()
        yh = torch.full_like(xh, float("nan")).pin_memory()
        io.apply(xh, yh)
        assert np.array_equal(yh.numpy(), want), s
        io.close()
    assert op.device_error() == 0


ND_VARIANT_CASES = [(f"{c['id']}_mode{m}", c, "adv", m) for c in CASES["advection"] for m in (0, 1, 2)] + \
                   [(c["id"], c, "mass", 1) for c in CASES["mass"]]


@pytest.mark.parametrize("cid,case,kind,mode", ND_VARIANT_CASES, ids=[c[0] for c in ND_VARIANT_CASES])
def test_kronnd_variants(cid, case, kind, mode):
    """Every variant of the any-dimension kernel (one pass per axis; groups of 2 or 3 axes per
    register block; axes a and a + D/2 paired where the terms share their other factors) meets the
    parity bar against the reference's golden outputs, forward, transposed and FP32, and agrees
    with the per-axis variant to rounding."""
    import torch
    import gendil_b200 as g
    op = make_operator(case, kind, mode)
    try:
        op.select_kernel("kronnd")
    except g.DGOPError as exc:
        pytest.skip(f"not eligible for the any-dimension Kronecker kernel: {exc}")
    x = inputs(case)
    want = ARR[f"{case['id']}_mode{mode}_y"] if kind == "adv" else ARR[f"{case['id']}_y"]
    ref = None
    tried = 0
    for name in op.ND_VARIANTS:
        try:
            op.set_variant(name)
        except g.DGOPError:
            continue
        assert op.variant == name
        tried += 1
        got = (cuda_apply(op, x), cuda_apply(op, x, transpose=True), cuda_apply(op, x, f32=True))
        assert rel_max(got[0], want) <= APPLY_TOL, name
        # y = alpha A x + beta y (the last step of the grouped and paired variants writes y itself)
        y0 = inputs(case, seed=9)
        yb = torch.from_numpy(y0).cuda()
        op.apply(torch.from_numpy(x).cuda(), yb, alpha=2.5, beta=-0.5)
        ab = 2.5 * got[0] - 0.5 * y0
        assert np.abs(yb.cpu().numpy() - ab).max() <= 1e-14 * max(np.abs(ab).max(), 1e-300), name
        if ref is None:
            ref = got
        else:
            assert rel_max(got[0], ref[0]) <= 1e-14, name
            assert rel_max(got[1], ref[1]) <= 1e-14, name
            assert rel_max(got[2], ref[2]) <= 1e-5, name
    assert tried >= 1
    op.set_variant(None)
    assert op.variant in op.ND_VARIANTS


def test_speed_of_light_operator_copies_exactly():
    """SpeedOfLightOperator: y = x bit for bit (16-byte vectors and the unaligned scalar path),
    alpha / beta, FP32 and the host-vector path."""
    import torch
    import gendil_b200 as g
    sp = g.Space(3, [5, 4, 3], order=2)
    op = g.SpeedOfLightOperator(sp, 3)
    assert op.kernel == "copy"
    n = sp.num_dofs
    base = torch.rand(n + 3, dtype=torch.float64, device="cuda")
    for off in (0, 1):
        x = base[off:off + n]
        y = torch.full((n + 3,), float("nan"), dtype=torch.float64, device="cuda")[off:off + n]
        op(x, y)
        assert torch.equal(x, y), off
    x = base[:n].contiguous()
    y0 = torch.rand(n, dtype=torch.float64, device="cuda")
    y = y0.clone()
    op.apply(x, y, alpha=2.0, beta=-0.5)
    assert torch.equal(y, 2.0 * x - 0.5 * y0)
    x32, y32 = x.float(), torch.empty(n, dtype=torch.float32, device="cuda")
    op.apply_f32(x32, y32)
    assert torch.equal(x32, y32)
    io = g.HostIO(op, slabs=3)
    xh = x.cpu().pin_memory()
    yh = torch.empty_like(xh).pin_memory()
    io.apply(xh, yh)
    assert torch.equal(xh, yh)
    io.close()


@pytest.mark.parametrize("cid,case,kind,mode,slabs", HOSTIO_CASES[:2], ids=[c[0] for c in HOSTIO_CASES[:2]])
def test_host_io_async_applies_overlap_and_chain(cid, case, kind, mode, slabs):
    """dgop_host_io_apply_async: several queued applies on distinct host vectors (alternating
    device pairs) and a chain y1 = A x, y2 = A y1, y3 = A y2 through host memory give the bits of
    the device applies once dgop_host_io_wait has run."""
    import torch
    import gendil_b200 as g
    op = make_operator(case, kind, mode)
    io = g.HostIO(op, slabs=slabs)
    stream = torch.cuda.current_stream()
    xs = [torch.from_numpy(inputs(dict(case, seed=s))).pin_memory() for s in (1, 2, 3, 4, 5)]
    ys = [torch.full_like(x, float("nan")).pin_memory() for x in xs]
    for x, y in zip(xs, ys):
        io.apply_async(x, y, stream)
    chain = [torch.full_like(xs[0], float("nan")).pin_memory() for _ in range(3)]
    io.apply_async(xs[0], chain[0], stream)
    io.apply_async(chain[0], chain[1], stream)
    io.apply_async(chain[1], chain[2], stream)
    io.wait(stream)
    stream.synchronize()
    for x, y in zip(xs, ys):
        assert np.array_equal(y.numpy(), cuda_apply(op, x.numpy()))
    want = xs[0].numpy()
    for c in chain:
        want = cuda_apply(op, want)
        assert np.array_equal(c.numpy(), want)
    io.close()
