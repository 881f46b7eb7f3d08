"""gendil_b200 -- B200-native matrix-free DG mass / upwind-advection operators.

Python host binding over the C ABI of ``libdgop.so`` (``include/dgop.h``).  Device memory and
streams come from PyTorch; every operator apply runs the library's own sm_100a kernels.  There
is no CPU fallback: importing this package on a machine without the built library raises.

The objects mirror GenDiL's operator API for this path:

* :class:`Space`  -- ``CartesianMesh<D>`` + ``MakeLobattoFiniteElement`` / ``MakeLegendreFiniteElement``
  + ``MakeFiniteElementSpace`` (Meshes/MeshDataStructures/CartesianMesh/cartesianndmesh.hpp:44,
  FiniteElementMethod/finiteelement.hpp:103,109, finiteelementspace.hpp:84);
* :class:`MassOperator`, :class:`AdvectionOperator`, :class:`MassAdvectionOperator`,
  :class:`SystemOperator` -- ``MakeMassFiniteElementOperator`` (massoperator.hpp:270),
  ``MakeAdvectionOperator`` (advectionoperator.hpp:1416,1481), ``MassAdvectionOperator``
  (massadvectionoperator.hpp:329); calling ``op(x, y)`` overwrites ``y`` like the reference's
  ``operator()(const Vector&, Vector&)``.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .coefficients import Coefficient, as_coefficient

__all__ = ["Space", "MassOperator", "AdvectionOperator", "MassAdvectionOperator", "SystemOperator",
           "SIPDGOperator", "DiffusionOperator", "MassInverseOperator", "SpeedOfLightOperator", "CGSolver", "GMRESSolver", "GMRESIRSolver",
           "Batch", "BatchSolver", "HostIO", "element_dot", "Coefficient", "DGOPError", "lib", "fill_random", "GLL", "GL",
           "BC_NONE", "BC_INFLOW"]

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libdgop.so")

GLL, GL = 0, 1
BC_NONE, BC_INFLOW = 0, 1
MAX_TERMS, MAX_DIM = 4, 6
MAX_VARIANTS = 6  # DGOP_MAX_VARIANTS


class DGOPError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"dgop error {code}: {msg}")
        self.code = code


class _Coef(ctypes.Structure):
    _fields_ = [("constant", ctypes.c_double), ("nterms", ctypes.c_int),
                ("tables", (ctypes.c_void_p * MAX_DIM) * MAX_TERMS), ("element_factor", ctypes.c_void_p)]


class _SolveResult(ctypes.Structure):
    _fields_ = [("success", ctypes.c_int), ("iterations", ctypes.c_int), ("relative_error", ctypes.c_double)]


_lib = None


def lib():
    """The loaded ``libdgop.so`` (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m gendil_b200.build` (no CPU fallback exists)")
        L = ctypes.CDLL(LIB_PATH)
        vp, i64, d, i = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int
        L.dgop_last_error.restype = ctypes.c_char_p
        L.dgop_version.restype = ctypes.c_char_p
        L.dgop_space_create.argtypes = [i, vp, vp, vp, vp, i, i, ctypes.POINTER(vp)]
        L.dgop_space_destroy.argtypes = [vp]
        L.dgop_space_num_dofs.argtypes = [vp]
        L.dgop_space_num_dofs.restype = i64
        L.dgop_space_num_elements.argtypes = [vp]
        L.dgop_space_num_elements.restype = i64
        L.dgop_space_coordinates.argtypes = [vp, i, i, vp]
        L.dgop_mass_create.argtypes = [vp, i, vp, ctypes.POINTER(vp)]
        L.dgop_advection_create.argtypes = [vp, i, vp, i, d, ctypes.POINTER(vp)]
        L.dgop_mass_advection_create.argtypes = [vp, i, vp, vp, ctypes.POINTER(vp)]
        L.dgop_system_create.argtypes = [vp, i, vp, vp, i, d, ctypes.POINTER(vp)]
        L.dgop_operator_destroy.argtypes = [vp]
        L.dgop_apply.argtypes = [vp, vp, vp, vp]
        L.dgop_apply_ex.argtypes = [vp, d, vp, d, vp, vp]
        L.dgop_apply_transpose.argtypes = [vp, vp, vp, vp]
        L.dgop_apply_f32.argtypes = [vp, vp, vp, vp]
        L.dgop_apply_bf16.argtypes = [vp, vp, vp, i, vp]
        L.dgop_fill_random.argtypes = [vp, i64, ctypes.c_uint, d, d]
        L.dgop_operator_kernel.argtypes = [vp]
        L.dgop_operator_kernel_note.argtypes = [vp]
        L.dgop_operator_kernel_note.restype = ctypes.c_char_p
        L.dgop_operator_select_kernel.argtypes = [vp, i]
        L.dgop_operator_variant.argtypes = [vp]
        L.dgop_operator_variant_name.argtypes = [vp]
        L.dgop_operator_variant_name.restype = ctypes.c_char_p
        L.dgop_operator_set_variant.argtypes = [vp, i]
        L.dgop_operator_variant_time.argtypes = [vp, i, ctypes.POINTER(ctypes.c_float)]
        L.dgop_operator_variant_f32.argtypes = [vp, ctypes.POINTER(i), ctypes.POINTER(ctypes.c_float)]
        L.dgop_operator_device_error.argtypes = [vp, ctypes.POINTER(i)]
        L.dgop_cg_create.argtypes = [vp, ctypes.POINTER(vp)]
        L.dgop_gmres_create.argtypes = [vp, i, ctypes.POINTER(vp)]
        L.dgop_gmres_ir_create.argtypes = [vp, i, i, ctypes.POINTER(vp)]
        L.dgop_solver_set_graphs.argtypes = [vp, i]
        L.dgop_solver_set_transpose.argtypes = [vp, i]
        L.dgop_solver_set_fused_dot.argtypes = [vp, i]
        L.dgop_solver_set_preconditioner.argtypes = [vp, vp]
        L.dgop_sipdg_create.argtypes = [vp, i, vp, ctypes.c_double, ctypes.c_double, i, ctypes.POINTER(vp)]
        L.dgop_mass_inverse_create.argtypes = [vp, i, vp, ctypes.POINTER(vp)]
        L.dgop_element_dot.argtypes = [vp, vp, vp, vp, vp, vp]
        L.dgop_sipdg_gradient.argtypes = [vp, vp, vp, vp, vp, vp]
        L.dgop_speed_of_light_create.argtypes = [vp, i, ctypes.POINTER(vp)]
        L.dgop_host_io_create.argtypes = [vp, i, ctypes.POINTER(vp)]
        L.dgop_host_io_apply_async.argtypes = [vp, vp, vp, vp]
        L.dgop_host_io_wait.argtypes = [vp, vp]
        L.dgop_batch_create.argtypes = [ctypes.POINTER(vp), i, ctypes.POINTER(vp)]
        L.dgop_batch_groups.argtypes = [vp]
        L.dgop_batch_apply.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), vp]
        L.dgop_batch_destroy.argtypes = [vp]
        L.dgop_batch_solver_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(vp), i, i, i, d, ctypes.POINTER(vp)]
        L.dgop_batch_solver_waves.argtypes = [vp]
        L.dgop_batch_solver_solve.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), i, d,
                                              ctypes.POINTER(_SolveResult), ctypes.POINTER(d), vp]
        L.dgop_batch_solver_destroy.argtypes = [vp]
        L.dgop_host_io_apply.argtypes = [vp, vp, vp, vp]
        L.dgop_host_io_destroy.argtypes = [vp]
        L.dgop_solver_solve.argtypes = [vp, vp, vp, i, d, ctypes.POINTER(_SolveResult), vp]
        L.dgop_solver_destroy.argtypes = [vp]
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        raise DGOPError(rc, lib().dgop_last_error().decode())
    return rc


def _ptr(t):
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return t.data_ptr()


_TORCH_DTYPES = {}


def _dvec(t, n, dtype="float64", name="vector"):
    """Device address of a contiguous CUDA tensor of exactly `n` values of `dtype`.  The kernels
    read and write `n` values through this address, so a CPU tensor, another dtype, a strided view
    or a short tensor is rejected here instead of becoming an out-of-bounds access on the device.
    A plain integer is taken as a raw device address whose size the caller vouches for."""
    if isinstance(t, int):
        return t
    want = _TORCH_DTYPES.get(dtype)
    if want is None:
        import torch
        want = _TORCH_DTYPES[dtype] = getattr(torch, dtype)
    try:
        if t.is_cuda and t.dtype is want and t.numel() == n and t.is_contiguous():
            return t.data_ptr()
    except AttributeError:
        pass
    if not getattr(t, "is_cuda", False):
        raise ValueError(f"{name}: a CUDA tensor is required")
    if str(t.dtype) != f"torch.{dtype}":
        raise ValueError(f"{name}: dtype {dtype} required, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name}: a contiguous tensor is required")
    if t.numel() != n:
        raise ValueError(f"{name}: {n} values required, got {t.numel()}")
    return t.data_ptr()


def _stream(stream):
    if stream is None:
        try:
            import torch
            return torch.cuda.current_stream().cuda_stream
        except Exception:  # pragma: no cover - torch always present in this package's use
            return 0
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


class Space:
    """A DG L2 space on a Cartesian hypercube mesh of dimension 1..6, order 0..7."""

    def __init__(self, dim, n_elem, h=None, origin=None, periodic=None, order=1, basis=GLL):
        n_elem = [int(v) for v in (n_elem if np.ndim(n_elem) else [n_elem] * dim)]
        if h is None:
            h = [1.0 / v for v in n_elem]
        h = [float(v) for v in (h if np.ndim(h) else [h] * dim)]
        origin = [0.0] * dim if origin is None else [float(v) for v in origin]
        periodic = [0] * dim if periodic is None else [int(bool(v)) for v in periodic]
        self.dim, self.order, self.basis = dim, order, basis
        self.n_elem, self.h, self.origin, self.periodic = n_elem, h, origin, periodic
        self._a = [np.ascontiguousarray(n_elem + [1] * (MAX_DIM - dim), dtype=np.int64),
                   np.ascontiguousarray(h + [1.0] * (MAX_DIM - dim), dtype=np.float64),
                   np.ascontiguousarray(origin + [0.0] * (MAX_DIM - dim), dtype=np.float64),
                   np.ascontiguousarray(periodic + [0] * (MAX_DIM - dim), dtype=np.int32)]
        handle = ctypes.c_void_p()
        check(lib().dgop_space_create(dim, *(a.ctypes.data for a in self._a), order, basis, ctypes.byref(handle)))
        self.handle = handle

    @property
    def num_dofs(self):
        return int(lib().dgop_space_num_dofs(self.handle))

    @property
    def num_elements(self):
        return int(lib().dgop_space_num_elements(self.handle))

    @property
    def dofs_per_element(self):
        return (self.order + 1) ** self.dim

    def coordinates(self, q, axis):
        """Coordinates at which coefficient tables are sampled along ``axis`` (n_elem x (q+2))."""
        out = np.empty(self.n_elem[axis] * (q + 2), dtype=np.float64)
        check(lib().dgop_space_coordinates(self.handle, q, axis, out.ctypes.data))
        return out

    def close(self):
        if getattr(self, "handle", None):
            lib().dgop_space_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Operator:
    def __init__(self, space, q):
        self.space, self.q = space, q
        self.handle = None
        self._keep = []

    def _coef(self, c):
        """Tabulate a coefficient into the ctypes struct (tables kept alive on self)."""
        if c is None:
            return None
        c = as_coefficient(c, self.space.dim)
        st = _Coef()
        st.constant = float(c.constant)
        st.nterms = len(c.terms)
        for t, term in enumerate(c.terms):
            for axis, fn in term.items():
                tab = np.ascontiguousarray(c.tabulate(fn, self.space.coordinates(self.q, axis)), dtype=np.float64)
                self._keep.append(tab)
                st.tables[t][axis] = tab.ctypes.data
        if c.element_factor is not None:
            self._keep.append(c.element_factor)
            st.element_factor = _ptr(c.element_factor)
        self._keep.append(st)
        return st

    def _vec(self, coefs):
        arr = (_Coef * self.space.dim)(*coefs)
        self._keep.append(arr)
        return arr

    def __call__(self, x, y, stream=None):
        """y = A x (overwrites y), FP64 device tensors."""
        n = self.space.num_dofs
        check(lib().dgop_apply(self.handle, _dvec(x, n, name="x"), _dvec(y, n, name="y"), _stream(stream)))
        return y

    def apply(self, x, y, alpha=1.0, beta=0.0, stream=None):
        """y = alpha A x + beta y."""
        n = self.space.num_dofs
        check(lib().dgop_apply_ex(self.handle, float(alpha), _dvec(x, n, name="x"), float(beta), _dvec(y, n, name="y"),
                                  _stream(stream)))
        return y

    def apply_transpose(self, x, y, stream=None):
        n = self.space.num_dofs
        check(lib().dgop_apply_transpose(self.handle, _dvec(x, n, name="x"), _dvec(y, n, name="y"), _stream(stream)))
        return y

    def apply_f32(self, x, y, stream=None):
        n = self.space.num_dofs
        check(lib().dgop_apply_f32(self.handle, _dvec(x, n, "float32", "x"), _dvec(y, n, "float32", "y"),
                                   _stream(stream)))
        return y

    def apply_bf16(self, x, y, transpose=False, stream=None):
        """y = A x (A^T x) for FP32 tensors with BF16 tensor-core contractions, FP32 accumulation and
        per-element max-abs scaling (dgop_apply_bf16; even dimensions, (p+1)^(D/2) <= 32)."""
        n = self.space.num_dofs
        check(lib().dgop_apply_bf16(self.handle, _dvec(x, n, "float32", "x"), _dvec(y, n, "float32", "y"),
                                    1 if transpose else 0, _stream(stream)))
        return y

    @property
    def num_dofs(self):
        return self.space.num_dofs

    @property
    def kernel(self):
        """'generic' (sum-factorized), 'kron' (register-resident 3D Kronecker form) or 'kronnd'
        (shared-memory Kronecker form, any dimension)."""
        return ("generic", "kron", "kronnd", "diffusion", "copy")[lib().dgop_operator_kernel(self.handle)]

    @property
    def kernel_note(self):
        return lib().dgop_operator_kernel_note(self.handle).decode()

    def select_kernel(self, name):
        check(lib().dgop_operator_select_kernel(self.handle, {"generic": 0, "kron": 1, "kronnd": 2}[name]))

    VARIANTS = ("stage2-tile", "stage1-tile", "stage2-shfl", "tma1-tile", "tma2-shfl", "tma2-tile")  # 3D ("kron")
    ND_VARIANTS = ("nd-passes", "nd-grouped2", "nd-grouped3", "nd-paired", "nd-mass")  # any-dimension kernel

    def _variants(self):
        return self.ND_VARIANTS if self.kernel == "kronnd" else self.VARIANTS

    @property
    def variant(self):
        """Kronecker-kernel variant picked by the autotuner (None without a Kronecker kernel)."""
        v = lib().dgop_operator_variant(self.handle)
        return None if v < 0 else self._variants()[v]

    def set_variant(self, name):
        """Force a Kronecker-kernel variant by name, or None to re-run the autotuner."""
        check(lib().dgop_operator_set_variant(self.handle, -1 if name is None else self._variants().index(name)))

    def variant_f32(self):
        """(variant name, {name: autotuner ms or -1 when unusable}) of the FP32 kernel configuration."""
        v = ctypes.c_int()
        ms = (ctypes.c_float * MAX_VARIANTS)()
        check(lib().dgop_operator_variant_f32(self.handle, ctypes.byref(v), ms))
        names = self._variants()
        return (None if v.value < 0 else names[v.value]), {n: ms[i] for i, n in enumerate(names)}

    def device_error(self):
        """Read and clear the operator's device error word (non-zero: a kernel's bounded wait for
        an asynchronous copy ran out and that launch's results are invalid)."""
        err = ctypes.c_int()
        check(lib().dgop_operator_device_error(self.handle, ctypes.byref(err)))
        return err.value

    def variant_times(self):
        """Autotuner time per launch (ms) of every variant (0.0: not available or not timed; the
        any-dimension kernel's variants are timed on the first 16,384 elements)."""
        out = {}
        for k, name in enumerate(self._variants()):
            ms = ctypes.c_float()
            check(lib().dgop_operator_variant_time(self.handle, k, ctypes.byref(ms)))
            out[name] = ms.value
        return out

    def close(self):
        if self.handle:
            lib().dgop_operator_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MassOperator(_Operator):
    """y = M_sigma x (MassFiniteElementOperator, massoperator.hpp:169)."""

    def __init__(self, space, q, sigma=1.0):
        super().__init__(space, q)
        h = ctypes.c_void_p()
        check(lib().dgop_mass_create(space.handle, q, ctypes.byref(self._coef(sigma)), ctypes.byref(h)))
        self.handle = h


class SIPDGOperator(_Operator):
    """Interior-penalty DG diffusion (the reference's SIPDG weak form): mu one diffusivity per
    element (FP64 device tensor, kept alive here), tau = kappa / h, sigma = -1 symmetric (SIPG),
    +1 NIPG, 0 IIPG; Dirichlet-0 boundary terms when `boundary`."""

    def __init__(self, space, q, mu, sigma=-1.0, kappa=None, boundary=True):
        super().__init__(space, q)
        if kappa is None:
            kappa = 10.0 * (space.order + 1) ** 2
        if str(mu.dtype) != "torch.float64" or not mu.is_cuda or not mu.is_contiguous() or mu.numel() != space.num_elements:
            raise ValueError("mu: one FP64 value per element, a contiguous CUDA tensor")
        self.mu = mu
        h = ctypes.c_void_p()
        check(lib().dgop_sipdg_create(space.handle, q, _ptr(mu), float(sigma), float(kappa), 1 if boundary else 0,
                                      ctypes.byref(h)))
        self.handle = h

    def coefficient_gradient(self, u, lam, scale=None, out=None, stream=None):
        """out[e] = scale[e] * lam^T (dA/dmu_e) u (one kernel; FP64 device tensors).  With lam the
        adjoint state (A^T lam = dJ/du) of A u = f, dJ/dmu_e = -out[e]."""
        import torch
        if out is None:
            out = torch.empty(self.space.num_elements, dtype=torch.float64, device=u.device)
        n, ne = self.space.num_dofs, self.space.num_elements
        check(lib().dgop_sipdg_gradient(self.handle, _dvec(u, n, name="u"), _dvec(lam, n, name="lam"),
                                        None if scale is None else _dvec(scale, ne, name="scale"),
                                        _dvec(out, ne, name="out"), _stream(stream)))
        return out


class DiffusionOperator(SIPDGOperator):
    """MakeDiffusionOperator<KP>(fes, ir, velocity, sigma, kappa), the reference's legacy SIPDG
    operator (FiniteElementMethod/MatrixFreeOperators/diffusionoperator.hpp:554): cell term,
    interior and boundary faces, penalty kappa / h.  `diffusivity` is a constant (the reference
    evaluates a function of X; constants are what its tests use) or one value per element."""

    def __init__(self, space, q, diffusivity, sigma, kappa):
        import torch
        if isinstance(diffusivity, (int, float)):
            mu = torch.full((space.num_elements,), float(diffusivity), dtype=torch.float64, device="cuda")
        else:
            mu = diffusivity
        super().__init__(space, q, mu, sigma=sigma, kappa=kappa, boundary=True)


class SpeedOfLightOperator(_Operator):
    """y = x element by element (MakeSpeedOfLightOperator, speedoflightoperator.hpp:198): the
    bandwidth reference of an apply (16 B/DoF in FP64)."""

    def __init__(self, space, q=1):
        super().__init__(space, q)
        h = ctypes.c_void_p()
        check(lib().dgop_speed_of_light_create(space.handle, q, ctypes.byref(h)))
        self.handle = h


class MassInverseOperator(_Operator):
    """y = M_sigma^{-1} x (inverse of the block-diagonal DG mass matrix; Kronecker kernels only)."""

    def __init__(self, space, q, sigma=1.0):
        super().__init__(space, q)
        h = ctypes.c_void_p()
        check(lib().dgop_mass_inverse_create(space.handle, q, ctypes.byref(self._coef(sigma)), ctypes.byref(h)))
        self.handle = h


class AdvectionOperator(_Operator):
    """y = A x, upwind DG advection (AdvectionOperator, advectionoperator.hpp:1005).

    ``bc=BC_NONE`` skips boundary faces (WithoutBC, :106); ``BC_INFLOW`` uses the constant inflow
    value ``g`` (WithBC, :269)."""

    def __init__(self, space, q, beta, bc=BC_INFLOW, g=0.0):
        super().__init__(space, q)
        h = ctypes.c_void_p()
        coefs = [self._coef(c) for c in _components(beta, space.dim)]
        check(lib().dgop_advection_create(space.handle, q, self._vec(coefs), bc, float(g), ctypes.byref(h)))
        self.handle = h


class MassAdvectionOperator(_Operator):
    """y = (M_sigma + A_interior) x (MassAdvectionOperator, massadvectionoperator.hpp:329)."""

    def __init__(self, space, q, beta, sigma=1.0):
        super().__init__(space, q)
        h = ctypes.c_void_p()
        coefs = [self._coef(c) for c in _components(beta, space.dim)]
        check(lib().dgop_mass_advection_create(space.handle, q, ctypes.byref(self._coef(sigma)), self._vec(coefs),
                                               ctypes.byref(h)))
        self.handle = h


class SystemOperator(_Operator):
    """y = (M_sigma + A) x in one launch: the implicit-Euler operator M/dt + A."""

    def __init__(self, space, q, beta, sigma=1.0, bc=BC_INFLOW, g=0.0):
        super().__init__(space, q)
        h = ctypes.c_void_p()
        coefs = [self._coef(c) for c in _components(beta, space.dim)]
        check(lib().dgop_system_create(space.handle, q, ctypes.byref(self._coef(sigma)), self._vec(coefs), bc,
                                       float(g), ctypes.byref(h)))
        self.handle = h


class _Solver:
    def __init__(self, op):
        self.op = op
        self.handle = None

    def solve(self, b, x, max_iters, tol, stream=None):
        """Solve A x = b on the device; x holds the initial guess and receives the solution.

        Returns {"success", "iterations", "relative_error"} with the reference's conventions
        (IterativeSolverResult, Solvers/iterativesolverresult.hpp:41)."""
        res = _SolveResult()
        n = self.op.space.num_dofs
        check(lib().dgop_solver_solve(self.handle, _dvec(b, n, name="b"), _dvec(x, n, name="x"), int(max_iters),
                                      float(tol), ctypes.byref(res),
                                      _stream(stream)))
        return {"success": bool(res.success), "iterations": res.iterations, "relative_error": res.relative_error}

    def precondition(self, prec):
        """Right preconditioner P (an operator on the same space, e.g. MassInverseOperator), or None."""
        check(lib().dgop_solver_set_preconditioner(self.handle, None if prec is None else prec.handle))
        self._prec = prec  # keep it alive while the solver uses it
        return self

    def transpose(self, enable=True):
        """Solve with the transposed operator A^T (adjoint solves)."""
        check(lib().dgop_solver_set_transpose(self.handle, 1 if enable else 0))
        return self

    def fused_dot(self, enable=True):
        """Form the first inner product of every iteration in the operator kernel's epilogue
        (default; 3D Kronecker-form operators) or in a separate pass."""
        check(lib().dgop_solver_set_fused_dot(self.handle, 1 if enable else 0))
        return self

    def use_graphs(self, enable=True):
        """Replay solver segments from CUDA graphs (True, the default), run the whole solve as one
        graph launch with a conditional WHILE node ("whole"), or launch every kernel directly
        (False).  All three give the same results bit for bit."""
        mode = 2 if enable == "whole" else (1 if enable else 0)
        check(lib().dgop_solver_set_graphs(self.handle, mode))
        return self

    def close(self):
        if self.handle:
            lib().dgop_solver_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CGSolver(_Solver):
    """ConjugateGradient (Solvers/conjugategradient.hpp:125), device resident."""

    def __init__(self, op):
        super().__init__(op)
        h = ctypes.c_void_p()
        check(lib().dgop_cg_create(op.handle, ctypes.byref(h)))
        self.handle = h


class GMRESSolver(_Solver):
    """GMRES_no_alloc(restart) (Solvers/gmres.hpp:74), device resident."""

    def __init__(self, op, restart=30):
        super().__init__(op)
        h = ctypes.c_void_p()
        check(lib().dgop_gmres_create(op.handle, int(restart), ctypes.byref(h)))
        self.handle = h


class GMRESIRSolver(_Solver):
    """GMRES(restart) with iterative refinement: restart cycles solve the correction equation
    with operator applies and a Krylov basis in `inner` precision ("fp32", "fp64", or "bf16": an
    FP32 basis with the operator's BF16 tensor-core applies), the residual and the solution are
    updated in FP64.  Same solve() contract and stopping test as GMRESSolver; no reference
    counterpart."""

    def __init__(self, op, restart=30, inner="fp32"):
        super().__init__(op)
        prec = {"fp32": 1, "fp64": 0, "bf16": 2}[inner]
        h = ctypes.c_void_p()
        check(lib().dgop_gmres_ir_create(op.handle, int(restart), prec, ctypes.byref(h)))
        self.handle = h


class Batch:
    """Independent operators applied together: one persistent launch per (dimension, order,
    variant) group of any-dimension Kronecker operators, one launch each for the rest (other
    kernels, variants without a persistent form, operators that fill the GPU on their own)
    (dgop_batch_apply)."""

    def __init__(self, ops):
        self.ops = list(ops)
        arr = (ctypes.c_void_p * len(self.ops))(*[o.handle for o in self.ops])
        h = ctypes.c_void_p()
        check(lib().dgop_batch_create(arr, len(self.ops), ctypes.byref(h)))
        self.handle = h

    @property
    def groups(self):
        return int(lib().dgop_batch_groups(self.handle))

    def apply(self, xs, ys, stream=None):
        xs, ys = list(xs), list(ys)
        if not (len(xs) == len(ys) == len(self.ops)):
            raise ValueError(f"Batch.apply: {len(self.ops)} operators need as many inputs and outputs "
                             f"(got {len(xs)} and {len(ys)})")
        xa = (ctypes.c_void_p * len(xs))(*[_dvec(x, o.space.num_dofs, name=f"xs[{i}]")
                                           for i, (x, o) in enumerate(zip(xs, self.ops))])
        ya = (ctypes.c_void_p * len(ys))(*[_dvec(y, o.space.num_dofs, name=f"ys[{i}]")
                                           for i, (y, o) in enumerate(zip(ys, self.ops))])
        check(lib().dgop_batch_apply(self.handle, xa, ya, _stream(stream)))

    def close(self):
        if self.handle:
            lib().dgop_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchSolver:
    """Many independent systems A_i x_i = b_i solved together (dgop_batch_solver_*): restarted
    GMRES(restart) with iterative refinement, inner cycles in `inner` precision ("fp32" or
    "fp64"), FP64 residual and solution, right preconditioners `precs` (all or none), every
    system's iterations in lockstep (one launch per vector operation over all systems, one apply
    per system, restart cycles replayed from a CUDA graph), systems cut into waves whose workspace
    fits `workspace_bytes` (0: half the free device memory).  No reference counterpart."""

    def __init__(self, ops, precs=None, restart=20, inner="fp32", workspace_bytes=0):
        self.ops = list(ops)
        self.precs = list(precs) if precs is not None else None
        if self.precs is not None and len(self.precs) != len(self.ops):
            raise ValueError("BatchSolver: one preconditioner per operator")
        n = len(self.ops)
        oa = (ctypes.c_void_p * n)(*[o.handle for o in self.ops])
        pa = None if self.precs is None else (ctypes.c_void_p * n)(*[p.handle for p in self.precs])
        h = ctypes.c_void_p()
        prec = {"fp32": 1, "fp64": 0}[inner]
        check(lib().dgop_batch_solver_create(oa, pa, n, int(restart), prec, float(workspace_bytes), ctypes.byref(h)))
        self.handle = h

    @property
    def waves(self):
        return int(lib().dgop_batch_solver_waves(self.handle))

    def solve(self, bs, xs, max_iters, tol, stream=None):
        """Solve every system (x holds the initial guesses).  Returns (results, seconds): a
        result dict per system as Solver.solve, and per system the time from the start of the call
        until the end of the restart cycle after which it was found finished."""
        bs, xs = list(bs), list(xs)
        n = len(self.ops)
        if not (len(bs) == len(xs) == n):
            raise ValueError(f"BatchSolver.solve: {n} systems need as many right-hand sides and solutions")
        ba = (ctypes.c_void_p * n)(*[_dvec(b, o.space.num_dofs, name=f"bs[{i}]") for i, (b, o) in enumerate(zip(bs, self.ops))])
        xa = (ctypes.c_void_p * n)(*[_dvec(x, o.space.num_dofs, name=f"xs[{i}]") for i, (x, o) in enumerate(zip(xs, self.ops))])
        res = (_SolveResult * n)()
        sec = (ctypes.c_double * n)()
        check(lib().dgop_batch_solver_solve(self.handle, ba, xa, int(max_iters), float(tol), res, sec, _stream(stream)))
        return ([{"success": bool(r.success), "iterations": r.iterations, "relative_error": r.relative_error} for r in res],
                list(sec))

    def close(self):
        if self.handle:
            lib().dgop_batch_solver_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HostIO:
    """y = A x for vectors in host memory (numpy arrays or CPU tensors, float64, contiguous):
    upload, apply and download pipelined over slabs of element planes (dgop_host_io_apply)."""

    def __init__(self, op, slabs=8):
        self.op = op
        h = ctypes.c_void_p()
        check(lib().dgop_host_io_create(op.handle, int(slabs), ctypes.byref(h)))
        self.handle = h

    @staticmethod
    def _host_ptr(a):
        if isinstance(a, np.ndarray):
            assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
            return a.ctypes.data
        assert a.device.type == "cpu" and a.is_contiguous() and str(a.dtype) == "torch.float64"
        return a.data_ptr()

    def apply(self, x, y, stream=None):
        check(lib().dgop_host_io_apply(self.handle, self._host_ptr(x), self._host_ptr(y), _stream(stream)))

    def apply_async(self, x, y, stream=None):
        """Queue y = A x and return (dgop_host_io_apply_async): consecutive calls overlap one
        apply's uploads with the previous one's downloads.  x and y must stay alive and untouched
        until wait() has been called and the stream synchronized."""
        check(lib().dgop_host_io_apply_async(self.handle, self._host_ptr(x), self._host_ptr(y), _stream(stream)))

    def wait(self, stream=None):
        """Make `stream` wait for every queued asynchronous apply (dgop_host_io_wait)."""
        check(lib().dgop_host_io_wait(self.handle, _stream(stream)))

    def close(self):
        if self.handle:
            lib().dgop_host_io_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def element_dot(op, a, b, scale=None, out=None, stream=None):
    """out[e] = scale[e] * sum over the DoFs of element e of a * b (FP64 device tensors)."""
    import torch
    if out is None:
        out = torch.empty(op.space.num_elements, dtype=torch.float64, device=a.device)
    n, ne = op.space.num_dofs, op.space.num_elements
    check(lib().dgop_element_dot(op.handle, _dvec(a, n, name="a"), _dvec(b, n, name="b"),
                                 None if scale is None else _dvec(scale, ne, name="scale"), _dvec(out, ne, name="out"),
                                 _stream(stream)))
    return out


def fill_random(n, seed=12345, lo=-1.0, hi=1.0):
    """FillRandom (Algebra/vector.hpp:632) into a new float64 numpy array."""
    out = np.empty(int(n), dtype=np.float64)
    check(lib().dgop_fill_random(out.ctypes.data, int(n), int(seed), float(lo), float(hi)))
    return out


def _components(beta, dim):
    if isinstance(beta, (list, tuple)) and len(beta) == dim:
        return list(beta)
    if np.ndim(beta) == 1 and len(beta) == dim:
        return [float(b) for b in beta]
    raise ValueError(f"velocity must have {dim} components")
