/*
 * flowgpu — B200 (sm_100a) implementation of FlowPro's DG residual and
 * implicit-solve hot path behind a plain C ABI.
 *
 * Every entry point returns an int status (FP_OK = 0); the message of the last
 * failure on a context is available from fp_last_error().  No call throws, no
 * device code traps: device-side failures (non-finite values, singular blocks,
 * exhausted waits) are reported through these status codes.
 *
 * Layouts on the host side of the ABI follow FlowPro's Java arrays:
 *   state / residual:  element-major, W[e * (nEqs*nBasis) + m*nBasis + j]
 *                      (Element.W, flowpro/core/element/Element.java:119-121)
 *   vertices:          [nVertices][dim], elements: [nElements][dim+1] (0-based),
 *   neighbors:         [nElements][dim+1], neighbour index or negative boundary
 *                      code (neighbors.txt, FlowProMain.java:523-531)
 *   element blocks:    Jacobian blocks in the reference's transposed storage,
 *                      ADiag[perturbed dof][residual dof] (Implicit.java:14-15).
 *
 * One context = one mesh resident on one GPU, one CUDA stream.  Calls on one
 * context are not re-entrant; separate contexts may be used concurrently.
 */
#ifndef FLOWGPU_H
#define FLOWGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
enum {
    FP_OK = 0,
    FP_ERR_ARG = 1,             /* invalid argument / size */
    FP_ERR_CUDA = 2,            /* CUDA runtime failure */
    FP_ERR_UNSUPPORTED = 3,     /* model / order / element type not built */
    FP_ERR_STATE = 4,           /* call out of order (e.g. no mesh uploaded) */
    FP_ERR_NOT_CONVERGED = 5,   /* GMRES did not reach its tolerance */
    FP_ERR_NONFINITE = 6,       /* NaN / Inf in a solution (LinearSolver.java:304-309) */
    FP_ERR_SINGULAR = 7,        /* zero pivot in a block factorisation */
    FP_ERR_TIMEOUT = 8          /* a bounded device wait gave up */
};

/* physical models (flowpro.user.equation.<model>) */
enum {
    FP_MODEL_NAVIER_STOKES = 1,   /* NavierStokes.java (Euler when is_diffusive = 0) */
    FP_MODEL_SPALART_ALLMARAS = 2,/* SpalartAllmaras.java */
    FP_MODEL_SCALAR_TEST = 3,     /* TestScalarEquation.java of the reference tests */
    FP_MODEL_ADIABATIC_EULERS = 4 /* AdiabaticEulers.java: isentropic Euler, n_eqs = dim + 1 */
};

/* preconditioners (Preconditioner.PreconditionerType, Preconditioner.java:19-21).  FP_PREC_ILU0
 * (ILU0.java:34-96, scalar ILU(0) on the CRS matrix) is the same factorisation as block ILU(0)
 * here: the element blocks are dense, so the scalar fill pattern is the block pattern and the
 * two coincide in exact arithmetic; it runs on the block ILU(0) kernels. */
enum { FP_PREC_NONE = 0, FP_PREC_BLOCKJACOBI = 1, FP_PREC_BLOCKILU0 = 2, FP_PREC_ILU0 = 3 };
/* precision of the preconditioner factorisation and application */
enum { FP_PREC_FP64 = 0, FP_PREC_FP32 = 1 };
/* Jacobian used by the Newton-GMRES operator: finite-difference blocks (the reference's),
 * the exact tangent applied matrix-free, or blocks assembled from the exact tangent */
enum { FP_JAC_ASSEMBLED = 0, FP_JAC_MATRIXFREE = 1, FP_JAC_ASSEMBLED_EXACT = 2 };
/* functionals of interest (FunctionalsOfInterest module) */
enum { FP_FUNCTIONAL_LIFT = 1, FP_FUNCTIONAL_DRAG = 2 };

/* Model parameters after Equation.init: the POD a Java caller fills from the
 * initialised Equation object (Aerodynamics.java:119-312, SpalartAllmaras.java:35-60,
 * TestScalarEquation.java).  fp_model_from_properties() derives it from a
 * parameters.txt-style string the same way. */
typedef struct {
    int model;
    int dim;
    int n_eqs;
    int is_diffusive;
    int inlet_supersonic;
    int has_attack_angle;
    int numerical_flux;          /* 0 Lax-Friedrichs ("default"), 1 vanLeer */
    int reserved;
    double kappa, Re, Pr;
    double p_out, p_in0, rho_in0;
    double attack_angle[2];
    double w_in[8];
    /* Spalart-Allmaras */
    double vt_in, sigma, cb1, cb2, ka, cw1, cw2, cw3, cv1, prt;
    /* TestScalarEquation */
    double a[3], k_diff, lambda;
} fp_model_params;

/* Numerical parameters of the spatial discretisation (Parameters.java, DGpure.initMethod) */
typedef struct {
    int order;                   /* FlowPro "order" = p + 1 */
    int positivity_limiter;      /* Element.positivityLimiter on/off */
    int implicit_time;           /* 1: BDF (time-step factor 1), 0: RK (1/(2p+1)) */
    int element_ordering;        /* 0 none, 1 rcm (ElementOrdering.java) */
    double penalty, beta0, damp_tol, damp_const;
    double fd_step;              /* Parameters.h = 1e-8 (finite-difference Jacobian) */
    int gcl;                     /* Parameters.gcl: discrete GCL mass matrix on a moving mesh */
} fp_num_params;

typedef struct {
    int dim;                     /* 2 (triangles) or 3 (tetrahedra) */
    int n_vertices;
    int n_elements;
    int reserved;
    const double* vertices;      /* [n_vertices][dim] */
    const int* elements;         /* [n_elements][dim+1] */
    const int* neighbors;        /* [n_elements][dim+1] */
    const double* wall_distance; /* [n_vertices] or NULL */
    const double* mesh_velocity; /* [n_vertices][dim] (ALE) or NULL */
} fp_mesh_desc;

typedef struct fp_ctx fp_ctx;

/* ---- context ------------------------------------------------------------ */
/* Replaces: the per-run set-up of FlowProMain.solverFactory (FlowProMain.java:486-730). */
int fp_ctx_create(int device, fp_ctx** out);
int fp_ctx_destroy(fp_ctx* ctx);
const char* fp_last_error(const fp_ctx* ctx);
/* Run all work of this context on an external stream (cudaStream_t as uintptr_t; 0 = own stream). */
int fp_ctx_set_stream(fp_ctx* ctx, uintptr_t stream);

/* ---- set-up (host) ------------------------------------------------------ */
/* Replaces Equation.init + Parameters for the hot-path keys: parses "key = value" entries
 * separated by ';' or line breaks (the text of a parameters.txt, '%' comments as
 * FlowProProperties strips them) with FlowPro's parameter names (Aerodynamics.java:119-312,
 * Parameters.java:160-280). */
int fp_model_from_properties(const char* props, fp_model_params* model, fp_num_params* num);
/* Replaces FlowProMain.createNeighborMatrix (FlowProMain.java:772-873). */
int fp_create_neighbor_matrix(int dim, int n_elements, const int* elements, int n_boundary,
                              const int* boundary, int* neighbors);
/* Replaces ElementOrdering.order (ElementOrdering.java:35-46): element indexes in DOF order;
 * ordering 0 = none, 1 = reverse Cuthill-McKee. Host only. */
int fp_element_ordering(int dim, int n_elements, const int* neighbors, int ordering, int* order);
/* Replaces FlowProMain.generateDistanceFunction (FlowProMain.java:962-1018): distance of every
 * vertex to the vertices of the faces with neighbour code source_bc (e.g. -1, walls), measured
 * along element edges (shortest paths; the reference relaxes Bellman-Ford sweeps to the same
 * path sums).  Vertices that no path reaches get 1e30, as in the reference.  Host only. */
int fp_wall_distance(int dim, int n_vertices, const double* vertices, int n_elements, const int* elements,
                     const int* neighbors, int source_bc, double* distance);
/* Replaces Mesh(...) + Mesh.init (Mesh.java:69-224): builds quadrature/basis tables,
 * affine geometry, DOF ordering, and uploads everything once. */
int fp_mesh_upload(fp_ctx* ctx, const fp_mesh_desc* mesh, const fp_model_params* model,
                   const fp_num_params* num);
int fp_mesh_info(const fp_ctx* ctx, int* n_elements, int* n_basis, int* n_eqs, int* n_faces);
/* element position in the DOF numbering (Element.gIndex / ElementOrdering) */
int fp_dof_order(const fp_ctx* ctx, int* block_position);
/* per-element geometry: area, elemSize, Xs[dim] (Element.computeGeometry, Element.java:516-567) */
int fp_geometry(const fp_ctx* ctx, double* area, double* elem_size, double* xs);
/* per-element mass matrix mass[e][i][j] = Element.M and basis weights basis_weights[e][i] =
 * Element.Is (DGpure.computeMassMatrixAndBasisWeights, DGpure.java:546-573), summed in the
 * reference's order; either pointer may be NULL */
int fp_mass_matrix(const fp_ctx* ctx, double* mass, double* basis_weights);

/* ---- state -------------------------------------------------------------- */
/* which: 0 = W, 1 = Wo, 2 = Wo2 (Element.W/Wo/Wo2).  Host arrays, element-major. */
int fp_state_set(fp_ctx* ctx, int which, const double* w);
int fp_state_get(fp_ctx* ctx, int which, double* w);
/* W = Wo = Wo2 = the model's constant initial state (DGpure.initCondition, DGpure.java:74-105) */
int fp_state_init_const(fp_ctx* ctx);

/* ---- residual ------------------------------------------------------------ */
/* Replaces DGpure.limiter for all elements (DGpure.java:358-400): artificial viscosity eps, c_IP. */
int fp_limiter(fp_ctx* ctx);
int fp_limiter_get(const fp_ctx* ctx, double* eps, double* c_ip);
/* Replaces Element.residuum(V = 0) over all elements (DGpure.java:108-355).
 * w: host state to upload first (NULL = resident state); r: host output (NULL = keep on device).
 * With both w and r the upload, the passes and the download overlap chunk by chunk (results
 * identical to the unchunked passes); pinned host buffers give the best overlap, and a call
 * with the same pinned buffers as the previous call replays the whole sequence as one CUDA
 * graph.  Returns after the residual is in r. */
int fp_residual(fp_ctx* ctx, const double* w, double* r);
/* n back-to-back evaluations of the resident residual (device only, for timing). */
int fp_residual_repeat(fp_ctx* ctx, int n);
/* fp_residual_repeat with CUDA events around its two kernels (face pass, element pass) on the
 * context's stream; *ms_face / *ms_elem receive their summed device times (milliseconds). */
int fp_residual_timed(fp_ctx* ctx, int n, double* ms_face, double* ms_elem);
/* Tangent of the residual: dr = (dR/dW) v at the resident state (hand-written forward mode). */
int fp_jvp(fp_ctx* ctx, const double* v, double* dr);
/* Adjoint of the residual: g = (dR/dW)^T lambda at the resident state (replaces the product
 * with the transposed assembled Jacobian that OptimisationToolExport writes,
 * OptimisationToolExport.java:38-260).  No Jacobian is stored: each element column is formed
 * in registers by the exact tangent of the element residual (quadrature states recomputed) and
 * contracted with lambda at once; stored blocks, if any, are left as they are. */
int fp_vjp(fp_ctx* ctx, const double* lambda, double* g);
/* Positivity limiter (Element.positivityLimiter, Element.java:385-476); returns #limited in *n. */
int fp_positivity_limiter(fp_ctx* ctx, int* n_limited);
/* L2 norms of R per equation (MasterSolver.residuumNorms, MasterSolver.java:113-137)
 * of the last spatial residual. */
int fp_residuum_norms(fp_ctx* ctx, double* norms);
/* Allocation-free variant of the residual norms, for callers that must not call cudaMalloc or
 * cudaFree themselves (device memory owned by a foreign pool or arena, e.g. a Java host handing
 * over device pointers).  No counterpart in the reference: it computes what
 * Element.l2NormsSquared + MasterSolver.residuumNorms compute, from caller-owned device arrays
 * r [n_elements][n_eqs*n_basis] (element-major) and mass [n_elements][n_basis][n_basis], into
 * norms [n_eqs] (device).  Scratch is a fixed 256 KiB file-scope device array: at most
 * 1,048,576 elements, n_basis <= 10, n_eqs <= 8 (else FP_ERR_ARG); overlapping calls race.
 * Every element passed is summed: pass only the elements inside the computational domain (the
 * reference sums those with insideComputeDomain).  The first call on a device resolves the
 * array's address in the device's primary context (the context the CUDA runtime uses) and
 * caches it per device: make it before any stream capture; a caller that makes a context of
 * its own current (cuCtxCreate) is not supported. */
int fp_l2_norms_noalloc(int n_elements, int n_basis, int n_eqs, const double* r, const double* mass, double* norms,
                        uintptr_t stream);
/* dt = cfl * min_e elemSize/lambda_e / factor (State.getTimeStep, State.java:177-193); *min_h_over_lambda */
int fp_time_step_bound(fp_ctx* ctx, double* min_h_over_lambda);

/* ---- explicit --------------------------------------------------------------- */
/* One SSP-RK3 step of size dt (RK3.computeExplicitStep stages 1-6, RK3.java:44-86, with the
 * limiter / positivity phases of LocalExplicitSolver.java:248-289). */
int fp_rk3_step(fp_ctx* ctx, double dt);
/* W -> Wo -> Wo2 shift (Element.copyW2Wo) and Wo -> W (copyWo2W) */
int fp_copy_w2wo(fp_ctx* ctx);
int fp_copy_wo2w(fp_ctx* ctx);

/* ---- implicit -------------------------------------------------------------- */
/* Replaces JacobiAssembler.assemble (JacobiAssembler.java:28-38) with BDFk.assembleJacobiMatrix
 * (BDF2.java:320-379): RHS and finite-difference element blocks (+ a1 M).  bdf_order 1 or 2.
 * dt <= 0: the steady operator (blocks of dR/dW without the mass term, RHS = R), as
 * Element.exportLocalJacobiMatrix / exportLocalR build for the optimisation export
 * (Element.java:737-786). */
int fp_assemble(fp_ctx* ctx, int bdf_order, double dt, double dto);
/* RHS only (Implicit.assembleResiduum, BDF2.java:310-317); *rhs_norm = ||RHS||_2; dt <= 0: RHS = R */
int fp_assemble_residuum(fp_ctx* ctx, int bdf_order, double dt, double dto, double* rhs_norm);
/* Blocks / RHS back to the host in the reference's storage (for checks and export). */
int fp_blocks_get(fp_ctx* ctx, double* diag, double* neigh, double* rhs);
/* Replaces LinearSolver.solve (LinearSolver.java:291-311) with GMRES(restart) (Gmres.java:42-122).
 * jacobian: FP_JAC_ASSEMBLED (BSR matrix from fp_assemble) or FP_JAC_MATRIXFREE (a1 M - JVP).
 * x: host solution in element-major order (may be NULL: kept on device as the Newton update). */
int fp_linear_solve(fp_ctx* ctx, int jacobian, int preconditioner, int precision, int restart,
                    int max_restarts, double tol, double* x, int* iterations, double* rel_residual);
/* W += x (Element.updateW) with the last linear-solve update */
int fp_update_w(fp_ctx* ctx);

/* Local implicit solver loop (LocalImplicitSolver.solve, LocalImplicitSolver.java:107-285) on the
 * device: steps of BDF(bdf_order) with Newton-GMRES, CFL control and retries.
 * out[0..6] = t, residuum, CFL, dt, steps, newton iterations, linear iterations. */
typedef struct {
    int bdf_order, newton_iters, jacobian, preconditioner, precision, restart, max_restarts, steps;
    double newton_tol, linear_tol, cfl, max_cfl, fixed_dt, target_residuum;
    int vary_cfl;
    /* Re-run the finite-difference element blocks and refactorise the preconditioner every
     * jac_lag Newton iterations (<= 1: every iteration, as the reference).  In between, the
     * RHS is fresh, the preconditioner of the last assembly is reused and, with
     * FP_JAC_ASSEMBLED, the stored operator is moved to the current a1
     * (A_diag += (a1 - a1_old) M); with FP_JAC_MATRIXFREE the operator is always exact. */
    int jac_lag;
} fp_implicit_params;
int fp_solve_implicit(fp_ctx* ctx, const fp_implicit_params* p, double* out);
/* Moving mesh (ALE), the step Deformation.recalculateMesh + newMeshPositionAndVelocity perform
 * in the reference (Deformation.java:44-62, LocalImplicitSolver.java:176-187): new vertex
 * positions [n_vertices][dim] and mesh velocities [n_vertices][dim] (NULL: at rest) rebuild the
 * affine geometry of every element and the current level's mass matrix.  From the first call on,
 * the context keeps element mass matrices of three time levels (Element.M / Mo / Mo2, all equal to
 * the mass matrix of the mesh as uploaded at first); the BDF right-hand side uses
 * M a1 W + Mo a2 Wo + Mo2 a3 Wo2 and the blocks a1 M.  With gcl set in the numerical parameters
 * the assembly replaces M by the discrete-GCL mass matrix (Element.applyGCLMassMatrix,
 * Element.java:568-630).  The residual norms keep the geometric mass matrix. */
int fp_mesh_move(fp_ctx* ctx, const double* vertices, const double* velocity);
/* Shift of the mass-matrix time levels after a finished step: Mo2 = Mo, Mo = M
 * (Element.nextTimeLevelMassMatrixes, Element.java:632-639); no-op on a static mesh. */
int fp_mass_next_level(fp_ctx* ctx);
/* Solver files of fp_solve_implicit / fp_solve_explicit, as MasterSolver and the local solvers
 * write them into the simulation directory (MasterSolver.java:60-111, LocalImplicitSolver.java:
 * 244-275 and 326-344, State.java:113-136): a residuum.txt row per finished step; state.txt,
 * W.txt, We.txt and artificialViscosity.txt every save_rate steps (save_rate <= 0: only at the
 * end) and when the loop ends (FlowProMain.java:261-268 saves after solve); a file named STOP in
 * the directory stops the loop after the current step and is deleted.  append = 0 empties
 * residuum.txt first (a new computation, FlowProMain.java:691-700).  dir NULL or "": no files. */
int fp_solver_output(fp_ctx* ctx, const char* dir, int save_rate, int append);
/* The number format of those files, Java's Double.toString (shortest round-trip digits, plain
 * for 1e-3 <= |x| < 1e7, else d.dddE<n>), into buf of n bytes. */
int fp_java_double(double x, char* buf, int n);
/* Batched serving: n independent contexts (cases of any size and order) solved with the same
 * parameters by `threads` host workers, each case on its own stream; out[7*i..] as
 * fp_solve_implicit, status[i] its return code (both may be NULL).  Block Jacobi or no
 * preconditioner.  Replaces running LocalImplicitSolver once per case. */
int fp_batch_solve_implicit(fp_ctx** ctxs, int n, const fp_implicit_params* p, int threads, double* out, int* status);
/* Batched serving on one context: n independent cases of one model and one order (any sizes;
 * the model parameters may differ only in the outlet pressure) merged into one mesh
 * (element ranges in case order, fp_batch_info), each initialised to its own free stream.
 * Replaces running LocalImplicitSolver once per case. */
int fp_batch_upload(fp_ctx* ctx, int n, const fp_mesh_desc* descs, const fp_model_params* models, const fp_num_params* num);
int fp_batch_info(const fp_ctx* ctx, int* n_cases, int* case_e0);
/* Steady solve of every case of the batch (LocalImplicitSolver.solve per case,
 * LocalImplicitSolver.java:107-285): pseudo-time steps with one Newton iteration, each case with
 * its own time step and CFL control (State, CFLSetup) and its own residuum; every kernel covers
 * all cases in one launch (matrix-free exact tangent, exact blocks factorised in the block
 * ILU(0) storage of the merged mesh, refreshed every jac_lag steps); GMRES(restart) per case in
 * lockstep (inner products, norms and Givens rotations per case).  A case stops at
 * target_residuum; a failed linear solve returns that case to its last state with the CFL
 * reduced.  out[7*i..] as fp_solve_implicit per case; status[i]: FP_OK, FP_ERR_NOT_CONVERGED
 * (the CFL reduction became hopeless) or FP_ERR_NONFINITE.  Takes jacobian = FP_JAC_MATRIXFREE,
 * preconditioner = FP_PREC_BLOCKILU0, newton_iters = 1 and CFL control (no fixed dt). */
int fp_batch_solve(fp_ctx* ctx, const fp_implicit_params* p, double* out, int* status);
/* State level `which` (0 W, 1 Wo) of case i, element-major [n_elements(i)][n_eqs*n_basis]. */
int fp_batch_case_state(fp_ctx* ctx, int i, int which, double* w);
/* Local explicit solver loop (LocalExplicitSolver.solve, LocalExplicitSolver.java:115-195). */
int fp_solve_explicit(fp_ctx* ctx, int steps, double cfl, double target_residuum, double* out);

/* Device time per phase of the implicit solver (no counterpart in the reference; its
 * AT / ST columns time assembly and solve on the host): CUDA events around the launches of
 * each phase on the context's stream.  Phases: 0 residual and BDF right-hand side, 1 element
 * Jacobian blocks, 2 preconditioner factorisation, 3 operator products (block SpMV or the
 * matrix-free tangent), 4 preconditioner applications, 5 Krylov vector work (Gram-Schmidt,
 * norms, updates), 6 other (limiter, norms, time step).  ms[8] / counts[8] (may be NULL)
 * receive the totals since the last reset; enable = 1 resets and starts, 0 resets and stops,
 * -1 only reads. */
int fp_profile(fp_ctx* ctx, int enable, double* ms, long long* counts);
/* Kernel of the block ILU(0) application (no counterpart in the reference; the same
 * factorisation applied): 0 (default) the factor blocks staged in shared memory by bulk
 * asynchronous copies several elements ahead, with NG elements in flight per thread block (NG a
 * power of two up to 16 for nc <= 16 unknowns per element, 8 for nc <= 32, else 4, chosen by
 * timing the candidates on the first application; every NG gives the same values), where
 * nc * nc * element size is a multiple of 16 bytes, else as 1; 1 one element per block with the
 * factor entries loaded into registers one element ahead (equal to rounding); 2 .. 6 the staged
 * kernel with NG = 1, 2, 4, 8, 16 (FP_ERR_UNSUPPORTED above the limit for nc or the slots). */
int fp_set_ilu_sweep(fp_ctx* ctx, int variant);
/* Test hook (no counterpart in the reference): poll limit of every dependency wait in the block
 * ILU(0) kernels of this context (default 524288; 0 makes each wait give up at once, so the
 * factorisation or linear solve returns FP_ERR_TIMEOUT and the context stays usable). */
int fp_set_wait_limit(fp_ctx* ctx, int polls);

/* ---- functionals and adjoint ---------------------------------------------- */
/* Force on the boundary faces with code bc: F[dim] = -sum over those faces of the integrated
 * stress vector (Equation.stressVector, NavierStokes.java:39-83; the face integral and sign
 * of Deformation2DRigid.calculateForces, Deformation2DRigid.java:81-105). */
int fp_forces(fp_ctx* ctx, int bc, double* force);
/* Functional of interest at the resident state (Element.computeFunctional, Element.java:789-862,
 * with LiftCoefficient.java:31-49 / DragCoefficient.java:30-48: p n_y / p n_x on wall faces,
 * two-dimensional models).  dI_dW (may be NULL, element-major): its exact gradient, which
 * replaces the finite differences of Element.exportLocalFunctionalDerivative (Element.java:723-734). */
int fp_functional(fp_ctx* ctx, int kind, double* value, double* dI_dW);
/* fp_assemble with the element blocks from the exact tangent instead of finite differences;
 * dt <= 0 assembles the steady operator -dR/dW (a1 = a2 = a3 = 0, RHS = R). */
int fp_assemble_exact(fp_ctx* ctx, int bdf_order, double dt, double dto);
/* Preconditioner of the matrix-free Newton operator (the role BDF2.assembleJacobiMatrix +
 * Preconditioner.factor play for LinearSolver.solve, BDF2.java:320-379, BlockILU0.java:98-185):
 * RHS, then the exact element blocks (a1 M - dR/dW) written straight into the factor storage
 * of `preconditioner` in `precision` and factorised there.  With FP_PREC_BLOCKILU0 / ILU0 no
 * copy of the operator's blocks is kept (FP32: the factorisation itself runs in FP32), so a
 * following fp_linear_solve takes FP_JAC_MATRIXFREE only; FP_PREC_BLOCKJACOBI goes through
 * fp_assemble_exact; FP_PREC_NONE assembles the RHS only. */
int fp_assemble_preconditioner(fp_ctx* ctx, int bdf_order, double dt, double dto, int preconditioner, int precision);
/* Linear solve with the blocks of the last assembly and any right-hand side: A x = rhs
 * (transpose = 0; any preconditioner) or A^T x = rhs (transpose = 1; none or block Jacobi).
 * rhs and x are element-major host arrays (forward and adjoint sensitivity solves). */
int fp_block_solve(fp_ctx* ctx, int transpose, const double* rhs, int preconditioner, int precision, int restart,
                   int max_restarts, double tol, double* x, int* iterations, double* rel_residual);
/* Adjoint linear solve A^T psi = rhs with the blocks of the last assembly (the discrete adjoint
 * of a functional: rhs = dI/dW with the steady blocks gives psi = -(dR/dW)^-T dI/dW).
 * preconditioner: FP_PREC_NONE or FP_PREC_BLOCKJACOBI (transposed block inverses).
 * rhs and psi are element-major host arrays. */
int fp_adjoint_solve(fp_ctx* ctx, const double* rhs, int preconditioner, int precision, int restart, int max_restarts,
                     double tol, double* psi, int* iterations, double* rel_residual);

#ifdef __cplusplus
}
#endif
#endif /* FLOWGPU_H */
