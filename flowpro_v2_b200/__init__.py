"""flowpro_v2_b200 — B200 implementation of FlowPro's DG residual and implicit-solve
hot path behind a C ABI (include/flowgpu.h, libflowgpu.so).

This module is the host-side binding used by the tests and the benchmark.  It
mirrors the reference's solver-facing objects:

    GpuMesh            ~ flowpro.core.Mesh + the Element[] residual methods
                         (Element.residuum / limiter / positivityLimiter)
    JacobiAssembler    ~ flowpro.core.solver.JacobiAssembler (assemble, assembleResiduum)
    LinearSolver       ~ flowpro.core.LinearSolvers.LinearSolver (GMRES + preconditioner)
    GpuImplicitSolver  ~ flowpro.core.solver.LocalImplicitSolver
    GpuExplicitSolver  ~ flowpro.core.solver.LocalExplicitSolver

There is no CPU fallback: if libflowgpu.so is missing or no GPU is present the
calls raise.
"""
import ctypes
import os

import numpy as np

__all__ = ["lib", "FlowGpuError", "model_from_properties", "create_neighbor_matrix", "GpuMesh", "JacobiAssembler",
           "LinearSolver", "GpuImplicitSolver", "GpuExplicitSolver", "ModelParams", "NumParams", "ImplicitParams"]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libflowgpu.so")

FP_OK, FP_ERR_ARG, FP_ERR_CUDA, FP_ERR_UNSUPPORTED, FP_ERR_STATE, FP_ERR_NOT_CONVERGED, FP_ERR_NONFINITE, \
    FP_ERR_SINGULAR, FP_ERR_TIMEOUT = range(9)
MODEL_NAVIER_STOKES, MODEL_SPALART_ALLMARAS, MODEL_SCALAR_TEST, MODEL_ADIABATIC_EULERS = 1, 2, 3, 4
PREC_NONE, PREC_BLOCKJACOBI, PREC_BLOCKILU0, PREC_ILU0 = 0, 1, 2, 3
FP64, FP32 = 0, 1
JAC_ASSEMBLED, JAC_MATRIXFREE, JAC_ASSEMBLED_EXACT = 0, 1, 2
FUNCTIONAL_LIFT, FUNCTIONAL_DRAG = 1, 2
_PREC_NAMES = {"none": PREC_NONE, "blockjacobi": PREC_BLOCKJACOBI, "blockilu0": PREC_BLOCKILU0, "ilu0": PREC_ILU0}


class FlowGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"flowgpu error {code}: {msg}")
        self.code = code


class ModelParams(ctypes.Structure):
    _fields_ = [("model", ctypes.c_int), ("dim", ctypes.c_int), ("n_eqs", ctypes.c_int), ("is_diffusive", ctypes.c_int),
                ("inlet_supersonic", ctypes.c_int), ("has_attack_angle", ctypes.c_int), ("numerical_flux", ctypes.c_int),
                ("reserved", ctypes.c_int), ("kappa", ctypes.c_double), ("Re", ctypes.c_double), ("Pr", ctypes.c_double),
                ("p_out", ctypes.c_double), ("p_in0", ctypes.c_double), ("rho_in0", ctypes.c_double),
                ("attack_angle", ctypes.c_double * 2), ("w_in", ctypes.c_double * 8), ("vt_in", ctypes.c_double),
                ("sigma", ctypes.c_double), ("cb1", ctypes.c_double), ("cb2", ctypes.c_double), ("ka", ctypes.c_double),
                ("cw1", ctypes.c_double), ("cw2", ctypes.c_double), ("cw3", ctypes.c_double), ("cv1", ctypes.c_double),
                ("prt", ctypes.c_double), ("a", ctypes.c_double * 3), ("k_diff", ctypes.c_double),
                ("lambda_", ctypes.c_double)]


class NumParams(ctypes.Structure):
    _fields_ = [("order", ctypes.c_int), ("positivity_limiter", ctypes.c_int), ("implicit_time", ctypes.c_int),
                ("element_ordering", ctypes.c_int), ("penalty", ctypes.c_double), ("beta0", ctypes.c_double),
                ("damp_tol", ctypes.c_double), ("damp_const", ctypes.c_double), ("fd_step", ctypes.c_double),
                ("gcl", ctypes.c_int)]


class MeshDesc(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("n_vertices", ctypes.c_int), ("n_elements", ctypes.c_int), ("reserved", ctypes.c_int),
                ("vertices", ctypes.POINTER(ctypes.c_double)), ("elements", ctypes.POINTER(ctypes.c_int)),
                ("neighbors", ctypes.POINTER(ctypes.c_int)), ("wall_distance", ctypes.POINTER(ctypes.c_double)),
                ("mesh_velocity", ctypes.POINTER(ctypes.c_double))]


class ImplicitParams(ctypes.Structure):
    _fields_ = [("bdf_order", ctypes.c_int), ("newton_iters", ctypes.c_int), ("jacobian", ctypes.c_int),
                ("preconditioner", ctypes.c_int), ("precision", ctypes.c_int), ("restart", ctypes.c_int),
                ("max_restarts", ctypes.c_int), ("steps", ctypes.c_int), ("newton_tol", ctypes.c_double),
                ("linear_tol", ctypes.c_double), ("cfl", ctypes.c_double), ("max_cfl", ctypes.c_double),
                ("fixed_dt", ctypes.c_double), ("target_residuum", ctypes.c_double), ("vary_cfl", ctypes.c_int),
                ("jac_lag", ctypes.c_int)]


_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_lib = None

_SIGS = {
    "fp_ctx_create": [ctypes.c_int, ctypes.POINTER(_vp)],
    "fp_ctx_destroy": [_vp],
    "fp_ctx_set_stream": [_vp, ctypes.c_size_t],
    "fp_model_from_properties": [ctypes.c_char_p, ctypes.POINTER(ModelParams), ctypes.POINTER(NumParams)],
    "fp_create_neighbor_matrix": [ctypes.c_int, ctypes.c_int, _i, ctypes.c_int, _i, _i],
    "fp_element_ordering": [ctypes.c_int, ctypes.c_int, _i, ctypes.c_int, _i],
    "fp_mesh_upload": [_vp, ctypes.POINTER(MeshDesc), ctypes.POINTER(ModelParams), ctypes.POINTER(NumParams)],
    "fp_mesh_info": [_vp, _i, _i, _i, _i],
    "fp_dof_order": [_vp, _i],
    "fp_geometry": [_vp, _d, _d, _d],
    "fp_mass_matrix": [_vp, _d, _d],
    "fp_state_set": [_vp, ctypes.c_int, _d],
    "fp_state_get": [_vp, ctypes.c_int, _d],
    "fp_state_init_const": [_vp],
    "fp_limiter": [_vp],
    "fp_limiter_get": [_vp, _d, _d],
    "fp_residual": [_vp, _d, _d],
    "fp_residual_repeat": [_vp, ctypes.c_int],
    "fp_residual_timed": [_vp, ctypes.c_int, _d, _d],
    "fp_jvp": [_vp, _d, _d],
    "fp_vjp": [_vp, _d, _d],
    "fp_positivity_limiter": [_vp, _i],
    "fp_residuum_norms": [_vp, _d],
    "fp_time_step_bound": [_vp, _d],
    "fp_rk3_step": [_vp, ctypes.c_double],
    "fp_copy_w2wo": [_vp],
    "fp_copy_wo2w": [_vp],
    "fp_assemble": [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double],
    "fp_assemble_residuum": [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, _d],
    "fp_blocks_get": [_vp, _d, _d, _d],
    "fp_linear_solve": [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _d, _i, _d],
    "fp_update_w": [_vp],
    "fp_solve_implicit": [_vp, ctypes.POINTER(ImplicitParams), _d],
    "fp_solve_explicit": [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, _d],
    "fp_forces": [_vp, ctypes.c_int, _d],
    "fp_wall_distance": [ctypes.c_int, ctypes.c_int, _d, ctypes.c_int, _i, _i, ctypes.c_int, _d],
    "fp_block_solve": [_vp, ctypes.c_int, _d, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _d,
                       _i, _d],
    "fp_batch_solve_implicit": [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_void_p, ctypes.c_int, _d, _i],
    "fp_functional": [_vp, ctypes.c_int, _d, _d],
    "fp_assemble_exact": [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double],
    "fp_assemble_preconditioner": [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int],
    "fp_set_wait_limit": [_vp, ctypes.c_int],
    "fp_batch_upload": [_vp, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(NumParams)],
    "fp_batch_info": [_vp, _i, _i],
    "fp_batch_solve": [_vp, ctypes.POINTER(ImplicitParams), _d, _i],
    "fp_batch_case_state": [_vp, ctypes.c_int, ctypes.c_int, _d],
    "fp_set_ilu_sweep": [_vp, ctypes.c_int],
    "fp_mesh_move": [_vp, _d, _d],
    "fp_mass_next_level": [_vp],
    "fp_solver_output": [_vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_int],
    "fp_java_double": [ctypes.c_double, ctypes.c_char_p, ctypes.c_int],
    "fp_profile": [_vp, ctypes.c_int, _d, ctypes.POINTER(ctypes.c_longlong)],
    "fp_adjoint_solve": [_vp, _d, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _d, _i, _d],
    "fp_l2_norms_noalloc": [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_size_t],
}


def lib():
    """Load libflowgpu.so; raises if it is missing (there is no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FlowGpuError(FP_ERR_STATE, f"{LIB_PATH} not built (python -m flowpro_v2_b200.build)")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        L.fp_last_error.argtypes = [_vp]
        L.fp_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def java_double(x):
    """Java's Double.toString as the library's solver files write it"""
    buf = ctypes.create_string_buffer(64)
    rc = lib().fp_java_double(float(x), buf, 64)
    if rc:
        raise FlowGpuError(rc, "fp_java_double")
    return buf.value.decode()


def exported_symbols():
    return sorted(_SIGS) + ["fp_last_error"]


def _dp(a):
    return a.ctypes.data_as(_d) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(_i) if a is not None else None


def model_from_properties(props):
    """Model and numerical parameters from FlowPro parameter keys (dict or 'k = v; ...')."""
    if isinstance(props, dict):
        props = ";".join(f"{k}={v}" for k, v in props.items())
    m, n = ModelParams(), NumParams()
    rc = lib().fp_model_from_properties(props.encode(), ctypes.byref(m), ctypes.byref(n))
    if rc:
        raise FlowGpuError(rc, "bad model parameters")
    return m, n


def create_neighbor_matrix(dim, elements, boundary):
    """FlowProMain.createNeighborMatrix on the host (integer, bit-exact)."""
    el = np.ascontiguousarray(elements, dtype=np.int32)
    bd = np.ascontiguousarray(boundary, dtype=np.int32)
    tt = np.zeros((el.shape[0], dim + 1), dtype=np.int32)
    rc = lib().fp_create_neighbor_matrix(dim, el.shape[0], _ip(el), bd.shape[0], _ip(bd), _ip(tt))
    if rc:
        raise FlowGpuError(rc, "createNeighborMatrix failed")
    return tt


def wall_distance(vertices, elements, neighbors, source_bc=-1):
    """edge-path distance of every vertex to the faces with neighbour code source_bc"""
    v = np.ascontiguousarray(vertices, dtype=np.float64)
    el = np.ascontiguousarray(elements, dtype=np.int32)
    tt = np.ascontiguousarray(neighbors, dtype=np.int32)
    out = np.zeros(v.shape[0])
    rc = lib().fp_wall_distance(v.shape[1], v.shape[0], _dp(v), el.shape[0], el.ctypes.data_as(_i),
                                tt.ctypes.data_as(_i), source_bc, _dp(out))
    if rc:
        raise FlowGpuError(rc, "fp_wall_distance failed")
    return out


def element_ordering(neighbors, rcm=True):
    """ElementOrdering.order: element indexes in the order of their DOF numbering."""
    tt = np.ascontiguousarray(neighbors, dtype=np.int32)
    out = np.zeros(tt.shape[0], dtype=np.int32)
    rc = lib().fp_element_ordering(tt.shape[1] - 1, tt.shape[0], _ip(tt), 1 if rcm else 0, _ip(out))
    if rc:
        raise FlowGpuError(rc, "element ordering failed")
    return out


class GpuMesh:
    """One FlowPro mesh with its solution resident on one GPU (a flowgpu context)."""

    def __init__(self, props, vertices, elements, neighbors, wall_distance=None, mesh_velocity=None, device=0):
        L = lib()
        self.model, self.num = model_from_properties(props)
        self.ctx = _vp()
        rc = L.fp_ctx_create(device, ctypes.byref(self.ctx))
        if rc:
            raise FlowGpuError(rc, "fp_ctx_create failed (no CUDA device?)")
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float64)
        self.elements = np.ascontiguousarray(elements, dtype=np.int32)
        self.neighbors = np.ascontiguousarray(neighbors, dtype=np.int32)
        self.wall_distance = None if wall_distance is None else np.ascontiguousarray(wall_distance, dtype=np.float64)
        self.mesh_velocity = None if mesh_velocity is None else np.ascontiguousarray(mesh_velocity, dtype=np.float64)
        self.dim = self.vertices.shape[1]
        desc = MeshDesc(self.dim, self.vertices.shape[0], self.elements.shape[0], 0, _dp(self.vertices),
                        _ip(self.elements), _ip(self.neighbors), _dp(self.wall_distance), _dp(self.mesh_velocity))
        self._check(L.fp_mesh_upload(self.ctx, ctypes.byref(desc), ctypes.byref(self.model), ctypes.byref(self.num)))
        ne, nb, neq, nf = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(L.fp_mesh_info(self.ctx, ctypes.byref(ne), ctypes.byref(nb), ctypes.byref(neq), ctypes.byref(nf)))
        self.n_elem, self.n_basis, self.n_eqs, self.n_faces = ne.value, nb.value, neq.value, nf.value
        self.nb = self.n_basis * self.n_eqs

    def _check(self, rc):
        if rc:
            msg = lib().fp_last_error(self.ctx)
            raise FlowGpuError(rc, msg.decode() if msg else "")
        return rc

    def close(self):
        if getattr(self, "ctx", None):
            lib().fp_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    PHASES = ("rhs", "blocks", "factor", "operator", "preconditioner", "krylov", "other")

    def profile(self, enable=-1):
        """device ms and launch counts per solver phase since the last reset (fp_profile);
        enable 1 resets and starts, 0 resets and stops, -1 only reads"""
        ms = np.zeros(8)
        n = np.zeros(8, dtype=np.int64)
        self._check(lib().fp_profile(self.ctx, enable, _dp(ms), n.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(self.PHASES)}

    def solver_output(self, directory, save_rate=0, append=False):
        """write residuum.txt / state.txt / W.txt / We.txt / artificialViscosity.txt of the
        following solver calls into directory (None: no files); a STOP file there ends a run"""
        d = None if directory is None else os.fsencode(directory)
        self._check(lib().fp_solver_output(self.ctx, d, save_rate, 1 if append else 0))

    def mesh_move(self, vertices, velocity=None):
        """new vertex positions and mesh velocities [n_vertices, dim] (fp_mesh_move)"""
        v = np.ascontiguousarray(vertices, dtype=np.float64)
        u = None if velocity is None else np.ascontiguousarray(velocity, dtype=np.float64)
        self._check(lib().fp_mesh_move(self.ctx, _dp(v), _dp(u)))

    def mass_next_level(self):
        self._check(lib().fp_mass_next_level(self.ctx))

    def update_w(self):
        """W += the last linear-solve update (fp_update_w)"""
        self._check(lib().fp_update_w(self.ctx))

    def copy_wo2w(self):
        self._check(lib().fp_copy_wo2w(self.ctx))

    def set_ilu_sweep(self, variant):
        """block ILU(0) application kernel: 0 bulk-copy staged, autotuned (default), 1 register,
        2 / 3 / 4 bulk-copy staged with 1 / 2 / 4 elements in flight per block"""
        self._check(lib().fp_set_ilu_sweep(self.ctx, variant))

    def set_wait_limit(self, polls):
        """test hook: poll limit of the block ILU(0) dependency waits (0: every wait gives up)"""
        self._check(lib().fp_set_wait_limit(self.ctx, polls))

    def set_stream(self, stream_handle):
        self._check(lib().fp_ctx_set_stream(self.ctx, int(stream_handle)))

    # ---- state (Element.W / Wo / Wo2), element-major [nElem, nEqs*nBasis]
    def set_state(self, W, which=0):
        W = np.ascontiguousarray(W, dtype=np.float64).reshape(-1)
        if W.size != self.n_elem * self.nb:
            raise ValueError("state has the wrong size")
        self._check(lib().fp_state_set(self.ctx, which, _dp(W)))

    def get_state(self, which=0):
        W = np.zeros(self.n_elem * self.nb)
        self._check(lib().fp_state_get(self.ctx, which, _dp(W)))
        return W.reshape(self.n_elem, self.nb)

    def init_condition(self):
        self._check(lib().fp_state_init_const(self.ctx))

    def dof_order(self):
        pos = np.zeros(self.n_elem, dtype=np.int32)
        self._check(lib().fp_dof_order(self.ctx, _ip(pos)))
        return pos

    def geometry(self):
        area, size = np.zeros(self.n_elem), np.zeros(self.n_elem)
        xs = np.zeros(self.n_elem * self.dim)
        self._check(lib().fp_geometry(self.ctx, _dp(area), _dp(size), _dp(xs)))
        return area, size, xs.reshape(-1, self.dim)

    def mass_matrices(self):
        """Element.M [e][i][j] and Element.Is [e][i] (DGpure.computeMassMatrixAndBasisWeights)"""
        M = np.zeros(self.n_elem * self.n_basis * self.n_basis)
        Is = np.zeros(self.n_elem * self.n_basis)
        self._check(lib().fp_mass_matrix(self.ctx, _dp(M), _dp(Is)))
        return M.reshape(self.n_elem, self.n_basis, self.n_basis), Is.reshape(self.n_elem, self.n_basis)

    # ---- residual (DGpure.residuum / limiter)
    def limiter(self):
        self._check(lib().fp_limiter(self.ctx))

    def limiter_values(self):
        eps, cip = np.zeros(self.n_elem), np.zeros(self.n_elem)
        self._check(lib().fp_limiter_get(self.ctx, _dp(eps), _dp(cip)))
        return eps, cip

    def residuum(self, W=None):
        """R(W) of all elements (Element.residuum with V = 0); W = None uses the resident state."""
        R = np.zeros(self.n_elem * self.nb)
        Wc = None if W is None else np.ascontiguousarray(W, dtype=np.float64).reshape(-1)
        self._check(lib().fp_residual(self.ctx, _dp(Wc), _dp(R)))
        return R.reshape(self.n_elem, self.nb)

    def residuum_repeat(self, n):
        self._check(lib().fp_residual_repeat(self.ctx, n))

    def residuum_timed(self, n=1):
        """n residual passes; returns the device times (ms) of the face and the element kernels."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(lib().fp_residual_timed(self.ctx, n, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def jvp(self, V):
        V = np.ascontiguousarray(V, dtype=np.float64).reshape(-1)
        out = np.zeros_like(V)
        self._check(lib().fp_jvp(self.ctx, _dp(V), _dp(out)))
        return out.reshape(self.n_elem, self.nb)

    def vjp(self, lam):
        """(dR/dW)^T lam at the resident state (overwrites the stored blocks with -dR/dW)"""
        lam = np.ascontiguousarray(lam, dtype=np.float64).reshape(-1)
        out = np.zeros_like(lam)
        self._check(lib().fp_vjp(self.ctx, _dp(lam), _dp(out)))
        return out.reshape(self.n_elem, self.nb)

    def forces(self, bc=-1):
        """force on the faces of boundary code bc"""
        F = np.zeros(self.dim)
        self._check(lib().fp_forces(self.ctx, bc, _dp(F)))
        return F

    def functional(self, kind, gradient=True):
        """lift (FUNCTIONAL_LIFT) or drag (FUNCTIONAL_DRAG) coefficient and its exact gradient"""
        v = ctypes.c_double()
        g = np.zeros(self.n_elem * self.nb) if gradient else None
        self._check(lib().fp_functional(self.ctx, kind, ctypes.byref(v), _dp(g) if gradient else None))
        return v.value, (g.reshape(self.n_elem, self.nb) if gradient else None)

    def block_solve(self, rhs, transpose=False, preconditioner="blockjacobi", precision=FP64, restart=30, max_restarts=10,
                    tol=1e-10):
        """solve A x = rhs (or A^T x = rhs) with the blocks of the last assembly; (converged, x, iterations)"""
        rhs = np.ascontiguousarray(rhs, dtype=np.float64).reshape(-1)
        x = np.zeros_like(rhs)
        it, rel = ctypes.c_int(), ctypes.c_double()
        prec = _PREC_NAMES[preconditioner] if isinstance(preconditioner, str) else preconditioner
        rc = lib().fp_block_solve(self.ctx, 1 if transpose else 0, _dp(rhs), prec, precision, restart, max_restarts, tol,
                                  _dp(x), ctypes.byref(it), ctypes.byref(rel))
        if rc not in (FP_OK, FP_ERR_NOT_CONVERGED):
            self._check(rc)
        return rc == FP_OK, x.reshape(self.n_elem, self.nb), it.value

    def adjoint_solve(self, rhs, preconditioner="blockjacobi", precision=FP64, restart=30, max_restarts=10, tol=1e-10):
        """solve A^T psi = rhs with the blocks of the last assembly; returns (converged, psi, iterations)"""
        rhs = np.ascontiguousarray(rhs, dtype=np.float64).reshape(-1)
        psi = np.zeros_like(rhs)
        it, rel = ctypes.c_int(), ctypes.c_double()
        prec = _PREC_NAMES[preconditioner] if isinstance(preconditioner, str) else preconditioner
        rc = lib().fp_adjoint_solve(self.ctx, _dp(rhs), prec, precision, restart, max_restarts, tol, _dp(psi),
                                    ctypes.byref(it), ctypes.byref(rel))
        if rc not in (FP_OK, FP_ERR_NOT_CONVERGED):
            self._check(rc)
        return rc == FP_OK, psi.reshape(self.n_elem, self.nb), it.value

    def positivity_limiter(self):
        n = ctypes.c_int()
        self._check(lib().fp_positivity_limiter(self.ctx, ctypes.byref(n)))
        return n.value

    def residuum_norms(self):
        out = np.zeros(self.n_eqs)
        self._check(lib().fp_residuum_norms(self.ctx, _dp(out)))
        return out

    def time_step_bound(self):
        v = ctypes.c_double()
        self._check(lib().fp_time_step_bound(self.ctx, ctypes.byref(v)))
        return v.value

    def rk3_step(self, dt):
        self._check(lib().fp_rk3_step(self.ctx, dt))

    def copy_w2wo(self):
        self._check(lib().fp_copy_w2wo(self.ctx))


class JacobiAssembler:
    """JacobiAssembler.assemble / assembleResiduum (finite-difference element blocks)."""

    def __init__(self, mesh, bdf_order=1):
        self.mesh, self.bdf_order = mesh, bdf_order

    def assemble(self, dt, dto):
        self.mesh._check(lib().fp_assemble(self.mesh.ctx, self.bdf_order, dt, dto))

    def assemble_exact(self, dt, dto):
        """blocks from the exact tangent; dt <= 0: steady operator -dR/dW"""
        self.mesh._check(lib().fp_assemble_exact(self.mesh.ctx, self.bdf_order, dt, dto))

    def assemble_preconditioner(self, dt, dto, preconditioner="blockilu0", precision=FP32):
        """exact blocks straight into the preconditioner's storage, factorised there (matrix-free path)"""
        prec = _PREC_NAMES[preconditioner] if isinstance(preconditioner, str) else preconditioner
        self.mesh._check(lib().fp_assemble_preconditioner(self.mesh.ctx, self.bdf_order, dt, dto, prec, precision))

    def assemble_residuum(self, dt, dto):
        v = ctypes.c_double()
        self.mesh._check(lib().fp_assemble_residuum(self.mesh.ctx, self.bdf_order, dt, dto, ctypes.byref(v)))
        return v.value

    def blocks(self):
        m = self.mesh
        diag = np.zeros((m.n_elem, m.nb, m.nb))
        neigh = np.zeros((m.n_elem, m.n_faces, m.nb, m.nb))
        rhs = np.zeros(m.n_elem * m.nb)
        m._check(lib().fp_blocks_get(m.ctx, _dp(diag), _dp(neigh), _dp(rhs)))
        return diag, neigh, rhs.reshape(m.n_elem, m.nb)


class LinearSolver:
    """GMRES(restart) with a block preconditioner (LinearSolver.solve / Gmres.solve)."""

    def __init__(self, mesh, preconditioner="blockjacobi", precision=FP64, jacobian=JAC_ASSEMBLED, restart=30,
                 max_restarts=5, tol=1e-2):
        self.mesh = mesh
        self.prec = _PREC_NAMES[preconditioner] if isinstance(preconditioner, str) else preconditioner
        self.precision, self.jacobian, self.restart, self.max_restarts, self.tol = precision, jacobian, restart, max_restarts, tol
        self.iterations, self.rel_residual = 0, 0.0

    def solve(self):
        """returns (converged, x) with x element-major; raises on errors other than non-convergence."""
        m = self.mesh
        x = np.zeros(m.n_elem * m.nb)
        it, rel = ctypes.c_int(), ctypes.c_double()
        rc = lib().fp_linear_solve(m.ctx, self.jacobian, self.prec, self.precision, self.restart, self.max_restarts,
                                   self.tol, _dp(x), ctypes.byref(it), ctypes.byref(rel))
        self.iterations, self.rel_residual = it.value, rel.value
        if rc not in (FP_OK, FP_ERR_NOT_CONVERGED, FP_ERR_SINGULAR):
            m._check(rc)
        return rc == FP_OK, x.reshape(m.n_elem, m.nb)


class GpuImplicitSolver:
    """LocalImplicitSolver on the device; returns (t, residuum, CFL, dt, steps, newton its, linear its)."""

    def __init__(self, mesh, **kw):
        self.mesh = mesh
        p = ImplicitParams()
        p.bdf_order, p.newton_iters, p.jacobian = kw.get("bdf_order", 1), kw.get("newton_iters", 1), kw.get("jacobian", 0)
        prec = kw.get("preconditioner", "blockjacobi")
        p.preconditioner = _PREC_NAMES[prec] if isinstance(prec, str) else prec
        p.precision, p.restart, p.max_restarts = kw.get("precision", FP64), kw.get("restart", 30), kw.get("max_restarts", 5)
        p.steps, p.newton_tol, p.linear_tol = kw.get("steps", 1), kw.get("newton_tol", 1e-4), kw.get("linear_tol", 1e-2)
        p.cfl, p.max_cfl, p.fixed_dt = kw.get("cfl", 1.0), kw.get("max_cfl", 1e4), kw.get("dt", 0.0)
        p.target_residuum, p.vary_cfl = kw.get("target_residuum", 0.0), kw.get("vary_cfl", 0)
        p.jac_lag = kw.get("jac_lag", 1)
        self.params = p

    def solve(self):
        out = np.zeros(7)
        self.mesh._check(lib().fp_solve_implicit(self.mesh.ctx, ctypes.byref(self.params), _dp(out)))
        return out


class GpuBatch:
    """Independent cases of one model and one order merged into one mesh on one context
    (fp_batch_upload) and solved together (fp_batch_solve).  cases: sequence of
    (props, vertices, elements, neighbors, wall_distance or None); the props may differ only in
    the outlet pressure."""

    def __init__(self, cases, device=0):
        L = lib()
        n = len(cases)
        self.ctx = _vp()
        rc = L.fp_ctx_create(device, ctypes.byref(self.ctx))
        if rc:
            raise FlowGpuError(rc, "fp_ctx_create failed (no CUDA device?)")
        self._keep = []
        models = (ModelParams * n)()
        descs = (MeshDesc * n)()
        num0 = None
        for i, (props, v, el, tt, wd) in enumerate(cases):
            m, num = model_from_properties(props)
            models[i] = m
            num0 = num if num0 is None else num0
            v = np.ascontiguousarray(v, dtype=np.float64)
            el = np.ascontiguousarray(el, dtype=np.int32)
            tt = np.ascontiguousarray(tt, dtype=np.int32)
            wd = None if wd is None else np.ascontiguousarray(wd, dtype=np.float64)
            self._keep += [v, el, tt, wd]
            descs[i] = MeshDesc(v.shape[1], v.shape[0], el.shape[0], 0, _dp(v), _ip(el), _ip(tt), _dp(wd), None)
        self._check(L.fp_batch_upload(self.ctx, n, ctypes.cast(descs, ctypes.c_void_p), ctypes.cast(models, ctypes.c_void_p),
                                      ctypes.byref(num0)))
        ne, nb, neq, nf = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(L.fp_mesh_info(self.ctx, ctypes.byref(ne), ctypes.byref(nb), ctypes.byref(neq), ctypes.byref(nf)))
        self.n_elem, self.n_basis, self.n_eqs = ne.value, nb.value, neq.value
        self.nb = self.n_basis * self.n_eqs
        self.n_cases = n
        e0 = np.zeros(n + 1, dtype=np.int32)
        self._check(L.fp_batch_info(self.ctx, None, _ip(e0)))
        self.case_e0 = e0

    def _check(self, rc):
        if rc:
            msg = lib().fp_last_error(self.ctx)
            raise FlowGpuError(rc, msg.decode() if msg else "")

    def solve(self, **kw):
        """returns (out [n, 7] as GpuImplicitSolver per case, status [n])"""
        p = GpuImplicitSolver(self, **kw).params
        out = np.zeros((self.n_cases, 7))
        status = np.zeros(self.n_cases, dtype=np.int32)
        self._check(lib().fp_batch_solve(self.ctx, ctypes.byref(p), _dp(out), status.ctypes.data_as(_i)))
        return out, status

    def case_state(self, i, which=0):
        n = int(self.case_e0[i + 1] - self.case_e0[i])
        W = np.zeros((n, self.nb))
        self._check(lib().fp_batch_case_state(self.ctx, i, which, _dp(W)))
        return W

    def set_stream(self, stream_handle):
        self._check(lib().fp_ctx_set_stream(self.ctx, stream_handle))

    PHASES = GpuMesh.PHASES

    def profile(self, enable=-1):
        return GpuMesh.profile(self, enable)

    def close(self):
        if getattr(self, "ctx", None) and self.ctx.value:
            lib().fp_ctx_destroy(self.ctx)
            self.ctx = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_solve_implicit(meshes, threads=8, **kw):
    """fp_batch_solve_implicit over GpuMesh objects (same solver parameters as
    GpuImplicitSolver); returns (out [n, 7], status [n])."""
    n = len(meshes)
    params = GpuImplicitSolver(meshes[0], **kw).params
    arr = (ctypes.c_void_p * n)(*[m.ctx.value for m in meshes])
    out = np.zeros((n, 7))
    status = np.zeros(n, dtype=np.int32)
    rc = lib().fp_batch_solve_implicit(arr, n, ctypes.cast(ctypes.byref(params), ctypes.c_void_p), threads, _dp(out),
                                       status.ctypes.data_as(_i))
    if rc != FP_OK and not np.any(status):
        meshes[0]._check(rc)
    return out, status


class GpuExplicitSolver:
    """LocalExplicitSolver (SSP-RK3) on the device; returns (t, residuum, CFL, dt, steps)."""

    def __init__(self, mesh, steps, cfl, target_residuum=0.0):
        self.mesh, self.steps, self.cfl, self.target = mesh, steps, cfl, target_residuum

    def solve(self):
        out = np.zeros(5)
        self.mesh._check(lib().fp_solve_explicit(self.mesh.ctx, self.steps, self.cfl, self.target, _dp(out)))
        return out
