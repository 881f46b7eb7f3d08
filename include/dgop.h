/* dgop -- B200-native matrix-free DG operators (mass, upwind advection) behind a C ABI.
 *
 * All vectors are caller-owned DEVICE pointers in the reference's L2 layout: element-major,
 * elements numbered x-fastest, each element block FIFO with axis 0 fastest
 * (GenDiL FiniteElementMethod/MatrixFreeOperators/KernelOperators/DoFIO/elementtensorview.hpp:42-48).
 * Every entry point returns DGOP_OK (0) or a negative error code and never aborts; the message
 * of the last error on the calling thread is returned by dgop_last_error().  Applies take an
 * explicit cudaStream_t (passed as void*), allocate nothing and do not synchronize.
 */
#ifndef DGOP_H
#define DGOP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum dgop_status {
  DGOP_OK = 0,
  DGOP_ERR_ARG = -1,         /* invalid argument (sizes, null pointers, unsupported order) */
  DGOP_ERR_CUDA = -2,        /* a CUDA call failed */
  DGOP_ERR_ALLOC = -3,       /* device or host allocation failed */
  DGOP_ERR_UNSUPPORTED = -4, /* no kernel for this (dimension, order, quadrature) */
  DGOP_ERR_NOT_CONVERGED = -5,
  DGOP_ERR_TIMEOUT = -6
};

enum dgop_basis { DGOP_BASIS_GLL = 0, DGOP_BASIS_GL = 1 };
enum dgop_bc { DGOP_BC_NONE = 0, DGOP_BC_INFLOW = 1 };
enum dgop_precision { DGOP_FP64 = 0, DGOP_FP32 = 1, DGOP_BF16 = 2 };

typedef struct dgop_space dgop_space;
typedef struct dgop_operator dgop_operator;

/* A scalar coefficient c(X) = constant + sum_{t < nterms} prod_k T_{t,k}(X_k), times an optional
 * per-element factor.  tables[t][k] is a HOST array of n_elem[k] * (q + 2) samples of T_{t,k}
 * at the coordinates returned by dgop_space_coordinates (NULL = factor 1);
 * element_factor is a DEVICE array of num_elements values (NULL = 1).  This is the closed set of
 * coefficients the reference's user lambdas reduce to on Cartesian meshes: constants, functions
 * of one coordinate per factor (massoperator.hpp:78, advectionoperator.hpp:317), sums of such
 * products, and piecewise-constant element fields. */
#define DGOP_MAX_TERMS 4
#define DGOP_MAX_DIM 6
typedef struct {
  double constant;
  int nterms;
  const double* tables[DGOP_MAX_TERMS][DGOP_MAX_DIM];
  const double* element_factor;
} dgop_coef;

/* ---- spaces (CartesianMesh<D> + MakeLobatto/LegendreFiniteElement + MakeFiniteElementSpace:
 *      Meshes/MeshDataStructures/CartesianMesh/cartesianndmesh.hpp:44, finiteelement.hpp:103,109,
 *      finiteelementspace.hpp:84) */
int dgop_space_create(int dim, const int64_t* n_elem, const double* h, const double* origin,
                      const int* periodic, int order, int basis, dgop_space** out);
int dgop_space_destroy(dgop_space* space);
int64_t dgop_space_num_dofs(const dgop_space* space);
int64_t dgop_space_num_elements(const dgop_space* space);
/* The n_elem[axis] * (q + 2) coordinates at which coefficient tables are sampled: element e,
 * point j < q is Gauss point j, j = q is the element's lower face, j = q + 1 its upper face. */
int dgop_space_coordinates(const dgop_space* space, int q, int axis, double* coords);

/* ---- operators
 * mass:            y = M_sigma x                   (MakeMassFiniteElementOperator, massoperator.hpp:270)
 * advection:       y = A x, bc NONE skips boundary faces (advectionoperator.hpp:1416),
 *                  INFLOW uses the constant inflow value bc_value (advectionoperator.hpp:1481)
 * mass_advection:  y = (M_sigma + A_interior) x   (MassAdvectionOperator, massadvectionoperator.hpp:329)
 * system:          y = (M_sigma + A) x with the given boundary treatment, one fused launch
 *                  (the (M/dt + A) implicit-Euler operator the reference composes from the two). */
int dgop_mass_create(const dgop_space* space, int q, const dgop_coef* sigma, dgop_operator** out);
int dgop_advection_create(const dgop_space* space, int q, const dgop_coef* beta, int bc, double bc_value,
                          dgop_operator** out);
int dgop_mass_advection_create(const dgop_space* space, int q, const dgop_coef* sigma, const dgop_coef* beta,
                               dgop_operator** out);
int dgop_system_create(const dgop_space* space, int q, const dgop_coef* sigma, const dgop_coef* beta, int bc,
                       double bc_value, dgop_operator** out);
/* mass_inverse:    y = M_sigma^{-1} x, the inverse of the block-diagonal DG mass matrix, applied as
 *                  the tensor product of inverted per-axis factors (no reference counterpart; the
 *                  preconditioner of dgop_solver_set_preconditioner).  Needs the Kronecker form:
 *                  GLL basis, a density that is one separable product, no per-element factor. */
int dgop_mass_inverse_create(const dgop_space* space, int q, const dgop_coef* sigma, dgop_operator** out);
/* sipdg:           y = A x for the interior-penalty DG diffusion form of the reference's weak-form
 *                  DSL (README "Weak Form DSL"; test-sipdg-coefficient-field-inputs.cpp:560-569):
 *                  integrate(cells, mu grad u . grad v) + integrate(interior_facets,
 *                  -{mu grad u . n}[v] + sigma [u]{mu grad v . n} + tau {mu}[u][v]) and, when
 *                  `boundary`, integrate(boundary_facets, -mu grad u . n v + sigma u mu grad v . n
 *                  + tau mu u v) (Dirichlet 0).  mu: DEVICE array, one diffusivity per element (kept,
 *                  not copied); tau = kappa / h on each face (InverseFacetSize); sigma = -1 gives the
 *                  symmetric form (SIPG), +1 NIPG, 0 IIPG.  Any dimension, any basis; the element must
 *                  fit in shared memory (kernel DGOP_KERNEL_DIFF). */
int dgop_sipdg_create(const dgop_space* space, int q, const double* mu, double sigma, double kappa, int boundary,
                      dgop_operator** out);
/* sipdg_gradient:  out[e] = scale[e] * lambda^T (dA/dmu_e) u for an operator of dgop_sipdg_create
 *                  (scale NULL: 1; FP64 device vectors, out one value per element).  With lambda the
 *                  adjoint state of A(mu) u = f (A^T lambda = dJ/du) the gradient of J is
 *                  dJ/dmu_e = -out[e].  One launch, deterministic.  No reference counterpart. */
int dgop_sipdg_gradient(const dgop_operator* op, const double* u, const double* lambda, const double* scale,
                        double* out, void* stream);
/* speed_of_light:  y = x read and written element by element (SpeedOfLightOperator,
 *                  MakeSpeedOfLightOperator, FiniteElementMethod/MatrixFreeOperators/
 *                  speedoflightoperator.hpp:198): the bandwidth reference of an apply, 16 B/DoF in
 *                  FP64; 128-bit loads and stores, a grid of a multiple of the SM count (kernel
 *                  DGOP_KERNEL_COPY; transpose and FP32 the same copy; q is not used). */
int dgop_speed_of_light_create(const dgop_space* space, int q, dgop_operator** out);
int dgop_operator_destroy(dgop_operator* op);
int64_t dgop_operator_num_dofs(const dgop_operator* op);

/* Kernel family used by an operator (no reference counterpart; diagnostics and testing):
 * DGOP_KERNEL_GENERIC is the sum-factorized kernel that follows the reference's element
 * algorithm for every shape; DGOP_KERNEL_KRON is the register-resident Kronecker-form kernel
 * (3D, GLL, orders 0..3, separable coefficients), chosen automatically when eligible;
 * DGOP_KERNEL_KRONND is the shared-memory Kronecker-form kernel for any dimension and order
 * (GLL, separable coefficients, element within shared memory), chosen when the register kernel
 * does not apply.
 * dgop_operator_kernel_note() says why the Kronecker form was not chosen. */
enum dgop_kernel {
  DGOP_KERNEL_GENERIC = 0,
  DGOP_KERNEL_KRON = 1,
  DGOP_KERNEL_KRONND = 2,
  DGOP_KERNEL_DIFF = 3,
  DGOP_KERNEL_COPY = 4
};
int dgop_operator_kernel(const dgop_operator* op);
const char* dgop_operator_kernel_note(const dgop_operator* op);
int dgop_operator_select_kernel(dgop_operator* op, int kernel);
/* Kronecker-kernel variants (no reference counterpart): 0 "stage2-tile" (next element group staged
 * while this one computes, layout exchanges through shared memory), 1 "stage1-tile" (one staging
 * buffer, more warps per SM), 2 "stage2-shfl" (exchanges by warp shuffles; even orders), and for
 * p = 3 FP64 operators whose x extent is a multiple of 8, element groups moved by the Tensor
 * Memory Accelerator: 3 "tma1-tile", 4 "tma2-shfl", 5 "tma2-tile".  At
 * creation the autotuner times every variant on scratch vectors (operators of at most 2^26 DoFs)
 * and keeps the fastest; operators of the same kernel shape (dimension, order, quadrature,
 * precision, terms, element count within a factor 8) reuse the first one's choice.  Variants 0-2
 * give bit-identical results, and so do variants 3-5; the two
 * families differ in the last bits (3-5 accumulate each term's last pass onto the sum).  dgop_operator_variant returns
 * the FP64 variant in use (-1 without a Kronecker kernel); dgop_operator_set_variant forces one
 * (-1 times the variants of this operator again and makes its choice the shape's);
 * dgop_operator_variant_time gives the autotuner's time per launch in ms (0 when not timed). */
int dgop_operator_variant(const dgop_operator* op);
const char* dgop_operator_variant_name(const dgop_operator* op);
int dgop_operator_set_variant(dgop_operator* op, int variant);
int dgop_operator_variant_time(const dgop_operator* op, int variant, float* ms);
/* The FP32 kernel configuration's variant and its autotuner times (ms[v]; -1: variant not usable;
 * ms holds DGOP_MAX_VARIANTS entries); variant -1 without a Kronecker kernel. */
#define DGOP_MAX_VARIANTS 6
int dgop_operator_variant_f32(const dgop_operator* op, int* variant, float* ms);
/* Reads and clears the operator's device error word: non-zero when a kernel gave up waiting for
 * an asynchronous copy (its bounded waits ran out; the results of that launch are invalid).
 * Synchronizes the device.  No reference counterpart. */
int dgop_operator_device_error(const dgop_operator* op, int* error);

/* y = alpha * A x + beta * y (beta == 0: y is not read).  FP64 device pointers, aligned to their
 * element size; the Kronecker-form kernel runs on 16-byte aligned vectors (any cudaMalloc'd or
 * torch-allocated tensor), other alignments take the generic kernel.
 * (MassFiniteElementOperator::operator() massoperator.hpp:209, AdvectionOperator::operator()
 * advectionoperator.hpp:1070: both overwrite y.) */
int dgop_apply(dgop_operator* op, const double* x, double* y, void* stream);
int dgop_apply_ex(dgop_operator* op, double alpha, const double* x, double beta, double* y, void* stream);
/* y = A^T x: the adjoint of the linear part (inflow value treated as 0); no reference counterpart. */
/* apply_bf16:      y = A x (transpose: A^T x) for FP32 vectors with BF16 tensor-core contractions,
 *                  FP32 accumulation and per-element max-abs scaling (the low-precision inner
 *                  operator of the refinement solver, DGOP_BF16): operators on the any-dimension
 *                  Kronecker form with an even dimension and (p+1)^(D/2) <= 32 (6D p <= 2, 4D
 *                  p <= 4, 2D any order).  Relative error about 1e-2 of |A| |x|.  No reference
 *                  counterpart. */
int dgop_apply_bf16(dgop_operator* op, const float* x, float* y, int transpose, void* stream);
int dgop_apply_transpose(dgop_operator* op, const double* x, double* y, void* stream);
/* FP32 apply of the same operator (tables rounded to FP32); no reference counterpart. */
int dgop_apply_f32(dgop_operator* op, const float* x, float* y, void* stream);

/* Batches of independent operators (no reference counterpart; configuration 5 of the benchmark
 * plan): operators on the any-dimension Kronecker kernel are grouped by (dimension, order, kernel
 * variant) and each group is applied by ONE persistent launch over all its operators' elements;
 * the others (other kernels, variants without a persistent form, and operators large enough to
 * fill every CTA slot of the GPU twice on their own) are applied one launch each.
 * y[i] = A_i x[i] (device pointers), bit-identical to dgop_apply.  The operators must outlive the
 * batch.  dgop_batch_groups gives the number of grouped launches. */
typedef struct dgop_batch dgop_batch;
int dgop_batch_create(dgop_operator* const* ops, int count, dgop_batch** out);
int dgop_batch_groups(const dgop_batch* batch);
int dgop_batch_apply(dgop_batch* batch, const double* const* x, double* const* y, void* stream);
int dgop_batch_destroy(dgop_batch* batch);


/* Applies on HOST vectors (the reference's operator() on a host-resident Vector,
 * massoperator.hpp:209, advectionoperator.hpp:1070, where the data lives in host memory):
 * y_host = A x_host.  The host-to-device copy, the apply and the device-to-host copy are pipelined
 * over `slabs` ranges of element planes of the last axis (slabs <= 0: 8), so upload and download
 * overlap.  The handle owns two pairs of device vectors and three streams (allocated at
 * creation).  dgop_host_io_apply starts after the work queued on `stream`, makes `stream` wait for
 * its end and returns when y_host is written.  dgop_host_io_apply_async queues the same work and
 * returns at once: consecutive asynchronous applies alternate between the two device pairs, so
 * one apply's uploads run while the previous one's downloads finish (an input that overlaps an
 * earlier call's result waits for that result).  Its results are complete once
 * dgop_host_io_wait(io, stream) has made `stream` wait for them (then synchronize the stream) or
 * after a later dgop_host_io_apply returns.  Pinned host memory (cudaMallocHost /
 * cudaHostRegister) copies at full link speed; pageable memory works, more slowly. */
typedef struct dgop_host_io dgop_host_io;
int dgop_host_io_create(dgop_operator* op, int slabs, dgop_host_io** out);
int dgop_host_io_apply(dgop_host_io* io, const double* x_host, double* y_host, void* stream);
int dgop_host_io_apply_async(dgop_host_io* io, const double* x_host, double* y_host, void* stream);
int dgop_host_io_wait(dgop_host_io* io, void* stream);
int dgop_host_io_destroy(dgop_host_io* io);

/* ---- Krylov solvers, device resident (workspaces allocated at create time).
 * CG: the reference's ConjugateGradient scratch overload (Solvers/conjugategradient.hpp:125-209),
 *   including its conventions: the tolerance is relative to the norm of the INITIAL residual
 *   b - A x0, `iterations` counts the iteration that converged, and `relative_error` is
 *   sqrt(|r| / |r0|).
 * GMRES(restart): GMRES_no_alloc (Solvers/gmres.hpp:74-289): modified Gram-Schmidt Arnoldi,
 *   Givens rotations, breakdown test rho <= eps * beta, the true residual recomputed after every
 *   cycle; `relative_error` = |b - A x| / |b|.
 * x holds the initial guess on entry and the solution on return.  dgop_solver_solve enqueues on
 * `stream` and synchronizes it before returning the result; it reads the solver's done flag once
 * per segment, one segment behind the work already enqueued. */
typedef struct {
  int success;
  int iterations;
  double relative_error;
} dgop_solve_result;
typedef struct dgop_solver dgop_solver;
int dgop_cg_create(dgop_operator* op, dgop_solver** out);
int dgop_gmres_create(dgop_operator* op, int restart, dgop_solver** out);
/* GMRES(restart) with iterative refinement (no reference counterpart; it replaces
 * GMRES_no_alloc, Solvers/gmres.hpp:74, where inner-precision throughput is wanted): each restart
 * cycle runs the Arnoldi process on the correction equation A d = r with operator applies and a
 * Krylov basis in `inner_precision` (DGOP_FP32 or DGOP_FP64; inner products, Hessenberg matrix and
 * rotations always FP64, Gram-Schmidt in classical form fused into two vector passes), then
 * x += d and the residual r = b - A x are formed with the FP64 operator.  The stopping test,
 * iteration count and `relative_error` are those of dgop_gmres_create's solver, and the attainable
 * accuracy is the FP64 one because the refinement uses the FP64 residual.  The inner applies use
 * the linear part of the operator (inflow value 0).  DGOP_FP32 needs an FP32 kernel for `op`. */
int dgop_gmres_ir_create(dgop_operator* op, int restart, int inner_precision, dgop_solver** out);
int dgop_solver_solve(dgop_solver* solver, const double* b, double* x, int max_iters, double tol,
                      dgop_solve_result* result, void* stream);
int dgop_solver_destroy(dgop_solver* solver);
/* How a solve is launched (no reference counterpart; the three give the same results, bit for
 * bit):
 *   DGOP_GRAPHS_SEGMENTS (1, the default): each segment (a chunk of CG iterations, a GMRES
 *     restart cycle) is captured once as a CUDA graph and replayed, the host reading the done
 *     word one segment behind the queued work;
 *   DGOP_GRAPHS_WHOLE (2): the whole solve is ONE graph launch, a conditional WHILE node that
 *     replays the segment until the solve is done or max_iters is exhausted, with no host round
 *     trip between segments (the loop is bounded by the segment count max_iters allows);
 *   DGOP_GRAPHS_OFF (0): every kernel is launched directly.
 * Graphs are re-captured when b, x or the operator's kernel selection change (tolerance and
 * iteration limit live in device memory). */
#define DGOP_GRAPHS_OFF 0
#define DGOP_GRAPHS_SEGMENTS 1
#define DGOP_GRAPHS_WHOLE 2
int dgop_solver_set_graphs(dgop_solver* solver, int enable);
/* transpose != 0: the solver solves A^T x = b (the adjoint of the operator's linear part, inflow
 * value 0; dgop_apply_transpose) with the same algorithm; used by adjoint solves.  No reference
 * counterpart. */
int dgop_solver_set_transpose(dgop_solver* solver, int transpose);
/* enable != 0 (the default): the first inner product of every iteration (CG: p . A p; GMRES:
 * V_0 . w) is formed in the operator kernel's epilogue when the operator's kernel provides one
 * (3D Kronecker form), saving a pass over two vectors; 0: a separate pass, as in the reference
 * (conjugategradient.hpp:176-179, gmres.hpp:157-165).  The two sum the same products in different
 * fixed orders, so iterates agree to rounding.  No reference counterpart. */
int dgop_solver_set_fused_dot(dgop_solver* solver, int enable);
/* Right preconditioning of a GMRES or refinement-GMRES solver: it solves A P z = b and returns
 * x = P z, so the stopping test and `relative_error` stay those of the unpreconditioned system
 * (|b - A x| / |b|).  P is an operator on the same space, typically dgop_mass_inverse_create's
 * (for mass-dominated implicit systems, whose tensor-product mass matrix conditions badly in high
 * dimension).  NULL removes it.  The workspace (two vectors) is allocated here.  No reference
 * counterpart. */
int dgop_solver_set_preconditioner(dgop_solver* solver, dgop_operator* prec);

/* Per-element inner products: out[e] = scale[e] * sum over the DoFs i of element e of a_i b_i
 * (scale NULL: 1), for the vectors of op's space (device pointers).  With a the adjoint state and
 * b = (dA/dc_e) u this is the gradient of a solve-based loss with respect to per-element
 * coefficient factors c_e.  No reference counterpart. */
int dgop_element_dot(const dgop_operator* op, const double* a, const double* b, const double* scale, double* out,
                     void* stream);

/* CG without any allocation at call time (no counterpart in the reference).  For callers that
 * must not let a library allocate device memory: a host framework that owns all device memory
 * through its own pool, or a latency-critical loop where cudaMalloc/cudaFree would synchronize the
 * device.  Same algorithm, kernels and results as dgop_cg_create + dgop_solver_solve, but the work
 * vectors, partial sums and solver state live in one fixed device array inside the library
 * (about 6.3 MB, held on every GPU that loads the library until the process exits).
 *  - Operators with more than DGOP_STATIC_CG_MAX_DOFS DoFs are rejected with DGOP_ERR_ARG.
 *  - The operator's device must be the current device (DGOP_ERR_ARG otherwise).
 *  - The first call on a device looks the array's device address up (cudaGetSymbolAddress) and
 *    keeps it for as long as the same CUDA context stays current; after a device reset or in a new
 *    context the next call looks it up again.  Make the first call in a context before any
 *    stream capture on that device.
 *  - Every call shares the one array: calls whose GPU work overlaps (other streams, other host
 *    threads on the same device) race and corrupt each other's results; serialize them.
 *  - Synchronizes `stream` before returning, like dgop_solver_solve. */
#define DGOP_STATIC_CG_MAX_DOFS 262144
int dgop_cg_solve_static(dgop_operator* op, const double* b, double* x, int max_iters, double tol,
                         dgop_solve_result* result, void* stream);

/* Many independent systems A_i x_i = b_i solved together (no reference counterpart; the
 * reference solves one system per GMRES_no_alloc call, Solvers/gmres.hpp:74).  Restarted
 * GMRES(restart) with iterative refinement: inner Krylov cycles with operator applies and basis in
 * `inner_precision` (DGOP_FP32 or DGOP_FP64), the residual and the solution in FP64, right
 * preconditioning by precs[i] (NULL array: none; otherwise every system has one), the stopping
 * test and reported quantities of dgop_gmres_create's solver.  All systems advance in lockstep:
 * each Krylov step is one apply per system plus one launch per vector operation over all of them,
 * a restart cycle of all of them is replayed from one CUDA graph, and systems that finished stay
 * idle.  The systems are cut, in the given order, into waves whose workspace fits
 * `workspace_bytes` (<= 0: half the free device memory at creation); the workspace of the largest
 * wave is allocated here.  The operators must outlive the solver. */
typedef struct dgop_batch_solver dgop_batch_solver;
int dgop_batch_solver_create(dgop_operator* const* ops, dgop_operator* const* precs, int count, int restart,
                             int inner_precision, double workspace_bytes, dgop_batch_solver** out);
/* Number of waves the systems were cut into. */
int dgop_batch_solver_waves(const dgop_batch_solver* solver);
/* Solve every system: b[i], x[i] device pointers (x[i] 16-byte aligned, the initial guess on
 * entry); results[i] per system; seconds (NULL or count entries): per system, the time from the
 * start of the call until the end of the restart cycle after which it was found finished.
 * Synchronizes `stream`. */
int dgop_batch_solver_solve(dgop_batch_solver* solver, const double* const* b, double* const* x, int max_iters,
                            double tol, dgop_solve_result* results, double* seconds, void* stream);
int dgop_batch_solver_destroy(dgop_batch_solver* solver);

/* FillRandom (Algebra/vector.hpp:632): out[i] = std::uniform_real_distribution<double>(lo, hi)
 * draws from std::mt19937(seed), in order, into a HOST buffer of n values. */
int dgop_fill_random(double* out, int64_t n, unsigned seed, double lo, double hi);

const char* dgop_last_error(void);
const char* dgop_version(void);

#ifdef __cplusplus
}
#endif

#endif /* DGOP_H */
