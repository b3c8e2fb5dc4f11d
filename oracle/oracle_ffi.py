"""ctypes binding of the CPU oracle (test infrastructure only).

Imported by tests/, bench.py (cpu_baseline and --impl reference) and
__graft_entry__.smoke() to check the CUDA path; the product package never
imports it.  The library is built by oracle/Makefile.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "build", "liboracle.so")
_FLOPS_PATH = os.path.join(_HERE, "build", "liboracle_flops.so")
_lib = None
_flops_lib = None

_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = _bind(ctypes.CDLL(_LIB_PATH))
    return _lib


def flops_lib():
    """the oracle built with the operation-counting floating-point type (oracle_flops.cpp)"""
    global _flops_lib
    if _flops_lib is None:
        if not os.path.exists(_FLOPS_PATH):
            build()
        L = _bind(ctypes.CDLL(_FLOPS_PATH))
        L.or_flops_reset.argtypes = []
        L.or_flops_get.argtypes = [ctypes.POINTER(ctypes.c_ulonglong)]
        _flops_lib = L
    return _flops_lib


def _bind(L):
        L.or_last_error.restype = ctypes.c_char_p
        L.or_create.restype = ctypes.c_void_p
        L.or_create.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _d, ctypes.c_int, _i, _i, _d, _d]
        for name in ["or_destroy", "or_nbasis", "or_neqs", "or_dofs", "or_positivity"]:
            getattr(L, name).argtypes = [ctypes.c_void_p]
        L.or_create_neighbor_matrix.argtypes = [ctypes.c_int, ctypes.c_int, _i, ctypes.c_int, _i, _i]
        L.or_set_state.argtypes = [ctypes.c_void_p, ctypes.c_int, _d]
        L.or_get_state.argtypes = [ctypes.c_void_p, ctypes.c_int, _d]
        L.or_limiter.argtypes = [ctypes.c_void_p, _d, _d]
        L.or_residual.argtypes = [ctypes.c_void_p, _d]
        L.or_geometry.argtypes = [ctypes.c_void_p, _d, _d, _d, _i]
        L.or_mass_matrices.argtypes = [ctypes.c_void_p, _d]
        L.or_basis_weights.argtypes = [ctypes.c_void_p, _d]
        L.or_assemble.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        L.or_assemble_residuum.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        L.or_get_blocks.argtypes = [ctypes.c_void_p, _d, _d, _d]
        L.or_linear_solve.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_double, _d, _i, _d]
        L.or_matrix_nnz.argtypes = [ctypes.c_void_p]
        L.or_matrix.argtypes = [ctypes.c_void_p, _i, _i, _d, _d]
        L.or_rk3_stage.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.or_time_step.argtypes = [ctypes.c_void_p]
        L.or_time_step.restype = ctypes.c_double
        L.or_update_cfl.argtypes = [ctypes.c_void_p]
        L.or_residuum_norms.argtypes = [ctypes.c_void_p, _d]
        L.or_run_explicit.argtypes = [ctypes.c_void_p, ctypes.c_int, _d]
        L.or_run_implicit.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _d]
        L.or_l2_error_scalar.argtypes = [ctypes.c_void_p]
        L.or_l2_error_scalar.restype = ctypes.c_double
        L.or_java_random.argtypes = [ctypes.c_longlong, ctypes.c_int, _d]
        L.or_get_gindex.argtypes = [ctypes.c_void_p, _i]
        L.or_set_threads.argtypes = [ctypes.c_int]
        L.or_forces.argtypes = [ctypes.c_void_p, ctypes.c_int, _d]
        L.or_wall_distance.argtypes = [ctypes.c_int, ctypes.c_int, _d, ctypes.c_int, _i, _i, ctypes.c_int, _d]
        L.or_functional.argtypes = [ctypes.c_void_p, ctypes.c_int, _d, _d]
        return L


def _dp(a):
    return a.ctypes.data_as(_d)


def _ip(a):
    return a.ctypes.data_as(_i)


def java_random(seed, n):
    out = np.zeros(n)
    lib().or_java_random(seed, n, _dp(out))
    return out


def create_neighbor_matrix(elem_type, elements, boundary):
    elements = np.ascontiguousarray(elements, dtype=np.int32)
    boundary = np.ascontiguousarray(boundary, dtype=np.int32)
    nf = 3 if elem_type == 3 else 4
    tt = np.zeros((elements.shape[0], nf), dtype=np.int32)
    rc = lib().or_create_neighbor_matrix(elem_type, elements.shape[0], _ip(elements), boundary.shape[0],
                                         _ip(boundary), _ip(tt))
    if rc != 0:
        raise RuntimeError(lib().or_last_error().decode())
    return tt


def wall_distance(vertices, elements, neighbors, source_bc=-1):
    """FlowProMain.generateDistanceFunction: edge-path distance to the faces of type source_bc"""
    v = np.ascontiguousarray(vertices, dtype=np.float64)
    el = np.ascontiguousarray(elements, dtype=np.int32)
    tt = np.ascontiguousarray(neighbors, dtype=np.int32)
    out = np.zeros(v.shape[0])
    lib().or_wall_distance(v.shape[1], v.shape[0], _dp(v), el.shape[0], _ip(el), _ip(tt), source_bc, _dp(out))
    return out


def props_string(props):
    return ";".join(f"{k}={v}" for k, v in props.items())


class Oracle:
    """One FlowPro mesh + solver state restated on the CPU."""

    def __init__(self, props, vertices, elements, neighbors, wall_distance=None, mesh_velocity=None, counting=False):
        L = flops_lib() if counting else lib()
        self.L = L
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float64)
        self.elements = np.ascontiguousarray(elements, dtype=np.int32)
        self.neighbors = np.ascontiguousarray(neighbors, dtype=np.int32)
        self.dim = self.vertices.shape[1]
        wd = None if wall_distance is None else np.ascontiguousarray(wall_distance, dtype=np.float64)
        uxy = None if mesh_velocity is None else np.ascontiguousarray(mesh_velocity, dtype=np.float64)
        self.h = L.or_create(props_string(props).encode(), self.dim, self.vertices.shape[0], _dp(self.vertices),
                             self.elements.shape[0], _ip(self.elements), _ip(self.neighbors),
                             _dp(wd) if wd is not None else None, _dp(uxy) if uxy is not None else None)
        if not self.h:
            raise RuntimeError(L.or_last_error().decode())
        self.n_elem = self.elements.shape[0]
        self.n_basis = L.or_nbasis(self.h)
        self.n_eqs = L.or_neqs(self.h)
        self.nb = self.n_basis * self.n_eqs

    def __del__(self):
        if getattr(self, "h", None):
            self.L.or_destroy(self.h)
            self.h = None

    def set_state(self, W, which=0):
        W = np.ascontiguousarray(W, dtype=np.float64).reshape(-1)
        assert W.size == self.n_elem * self.nb
        self.L.or_set_state(self.h, which, _dp(W))

    def get_state(self, which=0):
        W = np.zeros(self.n_elem * self.nb)
        self.L.or_get_state(self.h, which, _dp(W))
        return W.reshape(self.n_elem, self.nb)

    def limiter(self):
        eps = np.zeros(self.n_elem)
        cip = np.zeros(self.n_elem)
        self.L.or_limiter(self.h, _dp(eps), _dp(cip))
        return eps, cip

    def residual(self):
        R = np.zeros(self.n_elem * self.nb)
        self.L.or_residual(self.h, _dp(R))
        return R.reshape(self.n_elem, self.nb)

    def geometry(self):
        area = np.zeros(self.n_elem)
        size = np.zeros(self.n_elem)
        xs = np.zeros(self.n_elem * self.dim)
        ok = np.zeros(self.n_elem, dtype=np.int32)
        self.L.or_geometry(self.h, _dp(area), _dp(size), _dp(xs), _ip(ok))
        return area, size, xs.reshape(-1, self.dim), ok

    def mass_matrices(self):
        M = np.zeros(self.n_elem * self.n_basis * self.n_basis)
        self.L.or_mass_matrices(self.h, _dp(M))
        return M.reshape(self.n_elem, self.n_basis, self.n_basis)

    def basis_weights(self):
        Is = np.zeros(self.n_elem * self.n_basis)
        self.L.or_basis_weights(self.h, _dp(Is))
        return Is.reshape(self.n_elem, self.n_basis)

    def assemble(self, dt, dto):
        self.L.or_assemble(self.h, dt, dto)

    def assemble_residuum(self, dt, dto):
        self.L.or_assemble_residuum(self.h, dt, dto)

    def blocks(self):
        nf = self.dim + 1
        diag = np.zeros(self.n_elem * self.nb * self.nb)
        neigh = np.zeros(self.n_elem * nf * self.nb * self.nb)
        rhs = np.zeros(self.n_elem * self.nb)
        self.L.or_get_blocks(self.h, _dp(diag), _dp(neigh), _dp(rhs))
        return (diag.reshape(self.n_elem, self.nb, self.nb), neigh.reshape(self.n_elem, nf, self.nb, self.nb),
                rhs.reshape(self.n_elem, self.nb))

    def gindex(self):
        """block position of each element in the DOF numbering (RCM by default)."""
        g = np.zeros(self.n_elem, dtype=np.int32)
        self.L.or_get_gindex(self.h, _ip(g))
        return g

    def linear_solve(self, prec, tol):
        x = np.zeros(self.n_elem * self.nb)
        it = ctypes.c_int(0)
        err = ctypes.c_double(0)
        ok = self.L.or_linear_solve(self.h, prec.encode(), tol, _dp(x), ctypes.byref(it), ctypes.byref(err))
        return bool(ok), x, it.value, err.value

    def matrix(self):
        nnz = self.L.or_matrix_nnz(self.h)
        n = self.n_elem * self.nb
        I = np.zeros(n + 1, dtype=np.int32)
        J = np.zeros(nnz, dtype=np.int32)
        H = np.zeros(nnz)
        b = np.zeros(n)
        self.L.or_matrix(self.h, _ip(I), _ip(J), _dp(H), _dp(b))
        return I, J, H, b

    def rk3_stage(self, step, dt):
        self.L.or_rk3_stage(self.h, step, dt)

    def time_step(self):
        return self.L.or_time_step(self.h)

    def update_cfl(self):
        self.L.or_update_cfl(self.h)

    def residuum_norms(self):
        n = np.zeros(self.n_eqs)
        self.L.or_residuum_norms(self.h, _dp(n))
        return n

    def run_explicit(self, steps):
        st = np.zeros(4)
        self.L.or_run_explicit(self.h, steps, _dp(st))
        return st

    def run_implicit(self, steps, target=0.0):
        st = np.zeros(6)
        rc = self.L.or_run_implicit(self.h, steps, target, _dp(st))
        if rc != 0:
            raise RuntimeError(self.L.or_last_error().decode())
        return st

    def forces(self, bc=-1):
        """force on the faces of boundary type bc (Deformation2DRigid.calculateForces)"""
        F = np.zeros(self.dim)
        self.L.or_forces(self.h, bc, _dp(F))
        return F

    def functional(self, kind, gradient=True):
        """lift (kind 0) / drag (kind 1) coefficient and its finite-difference derivative"""
        I = np.zeros(1)
        g = np.zeros(self.n_elem * self.nb) if gradient else None
        if self.L.or_functional(self.h, kind, _dp(I), _dp(g) if gradient else None) != 0:
            raise RuntimeError(self.L.or_last_error().decode())
        return I[0], (g.reshape(self.n_elem, self.nb) if gradient else None)

    def positivity(self):
        return self.L.or_positivity(self.h)

    def l2_error_scalar(self):
        return self.L.or_l2_error_scalar(self.h)


def count_residual_flops(props, vertices, elements, neighbors, W, wall_distance=None):
    """Operations of one residual evaluation (DGpure.residuum over every element) of the
    restated reference algorithm at state W, from the counting build: a dict of the counts per
    phase ("volume", "interior_faces", "boundary_faces"; each with add, mul, div, sqrt, fn,
    trivial), the residual itself (bit-identical to the plain build's), and "flops" = the
    non-trivial +, -, *, /, sqrt with every interior face counted once (the reference evaluates
    it from both sides; the two evaluations do the same operations)."""
    o = Oracle(props, vertices, elements, neighbors, wall_distance, counting=True)
    o.set_state(W)
    o.limiter()
    L = flops_lib()
    L.or_flops_reset()
    R = o.residual()
    c = (ctypes.c_ulonglong * 18)()
    L.or_flops_get(c)
    keys = ("add", "mul", "div", "sqrt", "fn", "trivial")
    phases = {}
    for p, name in enumerate(("volume", "interior_faces", "boundary_faces")):
        phases[name] = {k: int(c[6 * p + i]) for i, k in enumerate(keys)}
    ops = lambda d: d["add"] + d["mul"] + d["div"] + d["sqrt"]  # noqa: E731
    flops = ops(phases["volume"]) + ops(phases["boundary_faces"]) + ops(phases["interior_faces"]) // 2
    return {"phases": phases, "flops": int(flops), "residual": R}


def set_threads(n):
    lib().or_set_threads(n)
