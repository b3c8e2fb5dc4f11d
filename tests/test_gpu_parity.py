"""GPU path (through the C ABI) against the CPU oracle on the same seeded inputs.

Tolerances:
  * residual, limiter, RK3 stages: normwise per equation, 1e-12 relative (FP64);
  * finite-difference element blocks (h = 1e-8, BDF2.java:349-378) and the tangent:
    1e-6 relative (FD truncation/rounding of the reference's own Jacobian);
  * linear solves: 1e-8 relative max-norm against a dense direct solve
    (LinearSolverTest.java:59).
"""
import os

import numpy as np
import pytest

import flowpro_v2_b200 as fg
from flowpro_v2_b200 import meshgen
from oracle import oracle_ffi as of
from tests import cases

pytestmark = pytest.mark.gpu


def make_pair(props, m, tt, seed=7, amp=0.02):
    o = of.Oracle(props, m.vertices, m.elements, tt, m.wall_distance)
    g = fg.GpuMesh(props, m.vertices, m.elements, tt, m.wall_distance)
    assert (g.n_basis, g.n_eqs) == (o.n_basis, o.n_eqs)
    rng = np.random.default_rng(seed)
    W = cases.perturbed(o.get_state(0), o.n_basis, o.n_eqs, rng, amp)
    for which in (0, 1, 2):
        o.set_state(W, which)
        g.set_state(W, which)
    return o, g, W


RESIDUAL_CASES = [
    ("euler", 2), ("euler", 3), ("euler", 4), ("ns", 2), ("ns", 3), ("ns", 4), ("sa", 3), ("sa", 2),
    ("scalar", 1), ("scalar", 2), ("scalar", 3), ("scalar", 4), ("scalar_diff", 3),
]


def props_for(kind, order):
    if kind == "euler":
        return cases.euler_props(order)
    if kind == "ns":
        return cases.ns_props(order, reynolds=500.0)
    if kind == "sa":
        return cases.sa_props(order)
    if kind == "scalar":
        return cases.scalar_props(order)
    return cases.scalar_props(order, 0.1)


@pytest.mark.parametrize("kind,order", RESIDUAL_CASES)
def test_residual_matches_oracle(kind, order):
    wall = meshgen.WALL if kind in ("ns", "sa") else meshgen.INVISCID_WALL
    m, tt = cases.channel(10, 5, seed=order, wall=wall)
    if kind == "sa":
        m.wall_distance[:] = np.maximum(m.wall_distance, 1e-3)
    o, g, W = make_pair(props_for(kind, order), m, tt)
    o.limiter()
    g.limiter()
    Ro = o.residual()
    Rg = g.residuum()
    err = cases.rel_err_per_component(Rg, Ro, o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-12), err


@pytest.mark.parametrize("order", [2, 3, 4])
def test_limiter_and_artificial_viscosity(order):
    props = cases.euler_props(order)
    props["dampTol"] = 3.0
    m, tt = cases.channel(10, 5, seed=11)
    o, g, W = make_pair(props, m, tt, amp=0.2)
    eo, co = o.limiter()
    g.limiter()
    eg, cg = g.limiter_values()
    assert np.max(np.abs(eo)) > 0
    assert np.max(np.abs(eg - eo)) <= 1e-12 * np.max(np.abs(eo))
    err = cases.rel_err_per_component(g.residuum(), o.residual(), o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-12), err


def test_van_leer_flux():
    m, tt = cases.channel(10, 5, seed=2)
    o, g, W = make_pair(cases.euler_props(3, flux="vanLeer"), m, tt)
    o.limiter()
    g.limiter()
    err = cases.rel_err_per_component(g.residuum(), o.residual(), o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-12), err


@pytest.mark.parametrize("kind,order", [("euler3", 2), ("euler3", 3), ("ns3", 2), ("ns3", 3)])
def test_residual_3d_matches_oracle(kind, order):
    """tetrahedra: Euler with inviscid walls, Navier-Stokes with no-slip walls"""
    if kind == "euler3":
        m, tt = cases.box(4, 3, 3, seed=order)
        props = cases.euler3_props(order)
    else:
        m, tt = cases.box(4, 3, 3, seed=order, wall=meshgen.WALL)
        props = cases.ns3_props(order)
    o, g, W = make_pair(props, m, tt)
    o.limiter()
    g.limiter()
    Ro = o.residual()
    assert np.all(np.isfinite(Ro))
    err = cases.rel_err_per_component(g.residuum(), Ro, o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-12), err


def test_rk3_3d_and_fd_blocks_3d():
    props = cases.ns3_props(2)
    props["timeMethod"] = "RK"
    m, tt = cases.box(4, 3, 3, seed=4, wall=meshgen.WALL)
    o, g, W = make_pair(props, m, tt)
    dt = 0.2 * g.time_step_bound()
    o.limiter()
    for st in range(1, 7):
        o.rk3_stage(st, dt)
    g.rk3_step(dt)
    err = cases.rel_err_per_component(g.get_state(0), o.get_state(0), o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-12), err
    props["timeMethod"] = "BDF"
    o, g, W = make_pair(props, m, tt, seed=9)
    o.limiter()
    g.limiter()
    o.assemble(0.05, 0.05)
    asm = fg.JacobiAssembler(g, bdf_order=1)
    asm.assemble(0.05, 0.05)
    Do, No, ro = o.blocks()
    Dg, Ng, rg = asm.blocks()
    scale = np.max(np.abs(Do))
    assert np.max(np.abs(Dg - Do)) <= 1e-6 * scale
    assert np.max(np.abs(Ng - No)) <= 1e-6 * scale


@pytest.mark.parametrize("order", [2, 3])
def test_rk3_step_matches_oracle(order):
    props = cases.euler_props(order)
    props["timeMethod"] = "RK"
    m, tt = cases.channel(10, 5, seed=5)
    o, g, W = make_pair(props, m, tt)
    dt = 0.2 * g.time_step_bound()
    o.limiter()
    R0 = o.residual()  # R(W) at the beginning of the step (spatialResiduum of stage 1)
    for st in range(1, 7):
        o.rk3_stage(st, dt)
    g.rk3_step(dt)
    err = cases.rel_err_per_component(g.get_state(0), o.get_state(0), o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-12), err
    err_r = cases.rel_err_per_component(g.get_state(3), R0, o.n_basis, o.n_eqs)
    assert np.all(err_r <= 1e-12), err_r


def test_time_step_bound_matches_oracle():
    props = cases.euler_props(3)
    props["CFL"] = 1.0
    m, tt = cases.channel(10, 5, seed=5)
    o, g, W = make_pair(props, m, tt)
    o.update_cfl()  # CFL ramp: 1/20 in the first step
    dto = o.time_step()
    assert abs(g.time_step_bound() / 20.0 - dto) <= 1e-13 * dto


@pytest.mark.parametrize("kind,order", [("euler", 2), ("euler", 3), ("ns", 3), ("scalar_diff", 2)])
def test_fd_element_blocks_match_oracle(kind, order):
    props = props_for(kind, order)
    props["timeOrder"] = 2
    wall = meshgen.WALL if kind == "ns" else meshgen.INVISCID_WALL
    m, tt = cases.channel(8, 4, seed=3, wall=wall)
    o, g, W = make_pair(props, m, tt)
    o.limiter()
    g.limiter()
    o.assemble(0.05, 0.04)
    asm = fg.JacobiAssembler(g, bdf_order=2)
    asm.assemble(0.05, 0.04)
    Do, No, ro = o.blocks()
    Dg, Ng, rg = asm.blocks()
    scale = np.max(np.abs(Do))
    assert np.max(np.abs(Dg - Do)) <= 1e-6 * scale
    assert np.max(np.abs(Ng - No)) <= 1e-6 * scale
    err = cases.rel_err_per_component(rg, ro, o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-12), err


@pytest.mark.parametrize("kind,order", [("euler", 3), ("ns", 3), ("sa", 3)])
def test_jvp_against_finite_differences(kind, order):
    wall = meshgen.WALL if kind in ("ns", "sa") else meshgen.INVISCID_WALL
    m, tt = cases.channel(8, 4, seed=9, wall=wall)
    if kind == "sa":
        m.wall_distance[:] = np.maximum(m.wall_distance, 1e-3)
    props = props_for(kind, order)
    o, g, W = make_pair(props, m, tt)
    g.limiter()
    rng = np.random.default_rng(20)
    for _ in range(3):
        V = rng.standard_normal(W.shape) * np.abs(W).mean(axis=0)
        Jv = g.jvp(V)
        h = 1e-7
        Rp = g.residuum(W + h * V)
        Rm = g.residuum(W - h * V)
        g.set_state(W)
        fd = (Rp - Rm) / (2 * h)
        assert np.max(np.abs(Jv - fd)) <= 1e-6 * np.max(np.abs(fd))


def _dense_from_blocks(diag, neigh, tt):
    """global matrix (element order) from blocks in the reference's transposed storage"""
    ne, nb = diag.shape[0], diag.shape[1]
    A = np.zeros((ne * nb, ne * nb))
    for e in range(ne):
        A[e * nb:(e + 1) * nb, e * nb:(e + 1) * nb] = diag[e].T
        for k in range(tt.shape[1]):
            n = tt[e, k]
            if n > -1:
                A[e * nb:(e + 1) * nb, n * nb:(n + 1) * nb] = neigh[e, k].T
    return A


@pytest.mark.parametrize("precision", [fg.FP64, fg.FP32])
@pytest.mark.parametrize("jacobian", [fg.JAC_ASSEMBLED, fg.JAC_MATRIXFREE])
def test_linear_solver_matches_direct(precision, jacobian):
    # LinearSolverTest: 4x4 square, p = 1, diffusion 0.1, W from java.util.Random(2), BDF1
    # assemble(0.05, -1); GMRES + block Jacobi to 1e-12 against a dense direct solve of the
    # same assembled system (< 1e-8).  The matrix-free operator is the exact Jacobian, the
    # assembled one its finite-difference approximation (h = 1e-8): they agree to ~1e-6.
    m = meshgen.square_mesh(4, 1.0, meshgen.INLET)
    tt = of.create_neighbor_matrix(3, m.elements, m.boundary)
    props = cases.scalar_props(2, 0.1)
    g = fg.GpuMesh(props, m.vertices, m.elements, tt, m.wall_distance)
    W = of.java_random(2, g.n_elem * g.nb)
    g.set_state(W)
    g.limiter()
    asm = fg.JacobiAssembler(g, bdf_order=1)
    asm.assemble(0.05, -1)
    diag, neigh, rhs = asm.blocks()
    xr = np.linalg.solve(_dense_from_blocks(diag, neigh, tt), rhs.reshape(-1)).reshape(-1, g.nb)
    ok, x = fg.LinearSolver(g, "blockjacobi", precision=precision, jacobian=jacobian, tol=1e-12, max_restarts=10).solve()
    assert ok
    tol = 1e-8 if jacobian == fg.JAC_ASSEMBLED else 1e-6
    assert np.max(np.abs(x - xr)) / np.max(np.abs(xr)) < tol


@pytest.mark.parametrize("ordering", ["rcm", "none"])
@pytest.mark.parametrize("precision", [fg.FP64, fg.FP32])
def test_block_ilu0_matches_direct_and_oracle(precision, ordering):
    """BlockILU0 (BlockILU0.java:22-243) as GMRES preconditioner on an implicit NS p = 2
    system: the solution equals a dense direct solve of the same blocks (1e-8), and with
    FP64 factors GMRES needs the oracle's iteration count (+-1) on the oracle's blocks."""
    props = cases.ns_props(2, reynolds=500.0)
    props["elementOrdering"] = ordering
    m, tt = cases.channel(10, 5, seed=3, wall=meshgen.WALL)
    o, g, W = make_pair(props, m, tt, amp=0.01)
    o.limiter()
    g.limiter()
    dt = 20.0 * g.time_step_bound()  # CFL 20: block Jacobi needs many more iterations
    o.assemble(dt, -1)
    asm = fg.JacobiAssembler(g, bdf_order=1)
    asm.assemble(dt, -1)
    diag, neigh, rhs = asm.blocks()
    xr = np.linalg.solve(_dense_from_blocks(diag, neigh, tt), rhs.reshape(-1)).reshape(-1, g.nb)
    ok, x = fg.LinearSolver(g, "blockilu0", precision=precision, tol=1e-12, max_restarts=20).solve()
    assert ok
    assert np.max(np.abs(x - xr)) / np.max(np.abs(xr)) < 1e-8
    ls = fg.LinearSolver(g, "blockilu0", precision=precision, tol=1e-8, max_restarts=5)
    ok, _ = ls.solve()
    assert ok
    ok_o, _, it_o, _ = o.linear_solve("blockilu0", 1e-8)
    assert ok_o
    if precision == fg.FP64:
        assert abs(ls.iterations - it_o) <= 1, (ls.iterations, it_o)
    ok_j, _, it_j, _ = o.linear_solve("blockjacobi", 1e-8)
    assert it_o < it_j


def test_block_ilu0_3d_converges_faster_than_block_jacobi():
    props = cases.euler3_props(2)
    m, tt = cases.box(6, 3, 3, seed=5)
    o, g, W = make_pair(props, m, tt, amp=0.01)
    g.limiter()
    dt = 50.0 * g.time_step_bound()
    asm = fg.JacobiAssembler(g, bdf_order=1)
    asm.assemble(dt, -1)
    diag, neigh, rhs = asm.blocks()
    xr = np.linalg.solve(_dense_from_blocks(diag, neigh, tt), rhs.reshape(-1)).reshape(-1, g.nb)
    its = {}
    for prec in ("blockilu0", "blockjacobi"):
        ls = fg.LinearSolver(g, prec, tol=1e-10, max_restarts=40)
        ok, x = ls.solve()
        assert ok, prec
        assert np.max(np.abs(x - xr)) / np.max(np.abs(xr)) < 1e-7, prec
        its[prec] = ls.iterations
    assert its["blockilu0"] < its["blockjacobi"], its


def test_assembled_system_matches_oracle():
    m = meshgen.square_mesh(4, 1.0, meshgen.INLET)
    tt = of.create_neighbor_matrix(3, m.elements, m.boundary)
    props = cases.scalar_props(2, 0.1)
    o = of.Oracle(props, m.vertices, m.elements, tt, m.wall_distance)
    g = fg.GpuMesh(props, m.vertices, m.elements, tt, m.wall_distance)
    W = of.java_random(2, o.n_elem * o.nb)
    o.set_state(W)
    g.set_state(W)
    o.limiter()
    g.limiter()
    o.assemble(0.05, -1)
    asm = fg.JacobiAssembler(g, bdf_order=1)
    asm.assemble(0.05, -1)
    Do, No, ro = o.blocks()
    Dg, Ng, rg = asm.blocks()
    assert np.max(np.abs(Dg - Do)) <= 1e-6 * np.max(np.abs(Do))
    assert np.max(np.abs(Ng - No)) <= 1e-6 * np.max(np.abs(Do))
    assert np.max(np.abs(rg - ro)) <= 1e-12 * np.max(np.abs(ro))


@pytest.mark.parametrize("p", [0, 1, 2, 3])
def test_convergence_order_on_gpu(p):
    errs = []
    for n in (4, 8, 16):
        m = meshgen.square_mesh(n, 1.0, meshgen.INLET)
        tt = fg.create_neighbor_matrix(2, m.elements, m.boundary)
        g = fg.GpuMesh(cases.scalar_props(p + 1), m.vertices, m.elements, tt, m.wall_distance)
        fg.GpuImplicitSolver(g, steps=4, dt=1e8, linear_tol=1e-13, max_restarts=20).solve()
        o = of.Oracle(cases.scalar_props(p + 1), m.vertices, m.elements, tt, m.wall_distance)
        o.set_state(g.get_state(0))
        errs.append(o.l2_error_scalar())
    rate = np.log(errs[-2] / errs[-1]) / np.log(2)
    assert rate > p + 0.7


def test_implicit_steps_match_oracle():
    props = cases.ns_props(3, reynolds=500.0)
    props.update(timeOrder=2, CFL=2.0, newtonIters=2, iterativeSolverTol=1e-12, preconditioner="blockjacobi")
    m, tt = cases.channel(8, 4, seed=4, wall=meshgen.WALL)
    o, g, W = make_pair(props, m, tt, amp=0.01)
    so = o.run_implicit(3)
    sg = fg.GpuImplicitSolver(g, bdf_order=2, newton_iters=2, steps=3, cfl=2.0, linear_tol=1e-12,
                              max_restarts=20).solve()
    assert abs(sg[0] - so[0]) <= 1e-10 * so[0]  # physical time
    err = cases.rel_err_per_component(g.get_state(0), o.get_state(0), o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-6), err


@pytest.mark.parametrize("order", [2, 3])
@pytest.mark.parametrize("mode", ["assembled_fp64", "matrixfree_fp32_lagged"])
def test_steady_state_matches_oracle(mode, order):
    """3D Euler p = 1 and p = 2 over the bump box driven to a 1e-11 residual by the oracle (FP64
    assembled Newton-GMRES, block ILU(0), CFL ramp) and by the device loop, either the same
    configuration or the mixed-precision one (matrix-free exact operator, exact blocks
    factorised in FP32 block ILU(0) storage, refreshed every 10 Newton iterations): the
    converged states and their wall forces agree to 1e-8 since both solve the same discrete
    equations."""
    props = cases.euler3_props(order)
    props.update(CFL=0, maxCFL=1e5, iterativeSolverTol=1e-3, preconditioner="blockilu0")
    m, tt = cases.box(6, 2, 2, seed=1)
    o, g, W = make_pair(props, m, tt, amp=0.0)
    so = o.run_implicit(200, 1e-11)
    assert so[1] <= 1e-11
    kw = dict(steps=200, cfl=0.0, vary_cfl=1, max_cfl=1e5, linear_tol=1e-3, preconditioner="blockilu0",
              target_residuum=1e-11)
    if mode == "assembled_fp64":
        kw.update(jacobian=fg.JAC_ASSEMBLED, precision=fg.FP64, jac_lag=1)
    else:
        kw.update(jacobian=fg.JAC_MATRIXFREE, precision=fg.FP32, jac_lag=10)
    sg = fg.GpuImplicitSolver(g, **kw).solve()
    assert sg[1] <= 1e-11, sg
    err = cases.rel_err_per_component(g.get_state(0), o.get_state(0), o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-8), err
    # the wall force of the converged states (the quantity the configuration reports)
    fo, fgpu = o.forces(meshgen.INVISCID_WALL), g.forces(meshgen.INVISCID_WALL)
    assert np.linalg.norm(fgpu - fo) <= 1e-8 * np.linalg.norm(fo), (fgpu, fo)


def test_explicit_solver_matches_oracle():
    props = cases.euler_props(2)
    props.update(timeMethod="RK", timeOrder=3, CFL=0.5)
    m, tt = cases.channel(10, 5, seed=6)
    o, g, W = make_pair(props, m, tt)
    so = o.run_explicit(5)
    sg = fg.GpuExplicitSolver(g, steps=5, cfl=0.5).solve()
    assert abs(sg[0] - so[0]) <= 1e-12 * so[0]
    err = cases.rel_err_per_component(g.get_state(0), o.get_state(0), o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-11), err
    assert abs(sg[1] - so[1]) <= 1e-9 * abs(so[1])


def test_positivity_limiter_matches_oracle():
    props = cases.euler_props(3)
    m, tt = cases.channel(8, 4, seed=8)
    o, g, W = make_pair(props, m, tt)
    W2 = W.copy()
    nb = o.n_basis
    W2[::3, 1] = -0.05  # a negative density node in every third element
    o.set_state(W2)
    g.set_state(W2)
    n_o = o.positivity()
    n_g = g.positivity_limiter()
    assert n_o == n_g and n_o > 0
    assert np.max(np.abs(g.get_state(0) - o.get_state(0))) <= 1e-12 * np.max(np.abs(W2))


def test_config1_full_size_residual_and_rk3():
    """2D Euler p = 1 on the 150 x 50 x 2 = 15,000-triangle bump channel (the explicit
    configuration): residual, then 3 SSP-RK3 steps with local CFL, against the oracle."""
    props = cases.euler_props(2)
    props.update(timeMethod="RK", timeOrder=3, CFL=0.5)
    m, tt = cases.channel(150, 50, seed=1)
    o, g, W = make_pair(props, m, tt, amp=0.01)
    o.limiter()
    g.limiter()
    err = cases.rel_err_per_component(g.residuum(), o.residual(), o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-12), err
    so = o.run_explicit(3)
    sg = fg.GpuExplicitSolver(g, steps=3, cfl=0.5).solve()
    assert abs(sg[0] - so[0]) <= 1e-12 * so[0]
    err = cases.rel_err_per_component(g.get_state(0), o.get_state(0), o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-11), err


def test_config2_full_size_residual():
    """2D Navier-Stokes p = 2 on the 548 x 183 x 2 = 200,568-triangle channel (the bench
    workload) with no-slip walls: one residual against the oracle, normwise per equation."""
    m, tt = cases.channel(548, 183, seed=1, wall=meshgen.WALL)
    o, g, W = make_pair(cases.ns_props(3, reynolds=5000.0), m, tt, amp=0.01)
    o.limiter()
    g.limiter()
    err = cases.rel_err_per_component(g.residuum(), o.residual(), o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-12), err


@pytest.mark.parametrize("dim,order", [(2, 1), (2, 2), (2, 3), (2, 4), (3, 2), (3, 3)])
def test_adiabatic_eulers_residual_matches_oracle(dim, order):
    """AdiabaticEulers (isentropic, p = rho^kappa, dim + 1 equations): residual with inlet,
    outlet and slip walls, then one SSP-RK3 step."""
    props = cases.adiabatic_props(order, dim)
    m, tt = cases.channel(10, 5, seed=order) if dim == 2 else cases.box(4, 3, 3, seed=order)
    o, g, W = make_pair(props, m, tt)
    assert o.n_eqs == dim + 1
    o.limiter()
    g.limiter()
    err = cases.rel_err_per_component(g.residuum(), o.residual(), o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-12), err
    props["timeMethod"] = "RK"
    o, g, W = make_pair(props, m, tt, seed=3)
    dt = 0.2 * g.time_step_bound()
    o.limiter()
    for st in range(1, 7):
        o.rk3_stage(st, dt)
    g.rk3_step(dt)
    err = cases.rel_err_per_component(g.get_state(0), o.get_state(0), o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-12), err


def test_adiabatic_eulers_implicit_steps_match_oracle():
    props = cases.adiabatic_props(2)
    props.update(CFL=5.0, newtonIters=2, iterativeSolverTol=1e-12, preconditioner="blockjacobi")
    m, tt = cases.channel(10, 5, seed=4)
    o, g, W = make_pair(props, m, tt, amp=0.01)
    so = o.run_implicit(3)
    sg = fg.GpuImplicitSolver(g, bdf_order=1, newton_iters=2, steps=3, cfl=5.0, linear_tol=1e-12,
                              max_restarts=20).solve()
    assert abs(sg[0] - so[0]) <= 1e-10 * so[0]
    err = cases.rel_err_per_component(g.get_state(0), o.get_state(0), o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-6), err


def _parameters_dict(text):
    """keys with values of a parameters.txt ('%' starts a comment)"""
    d = {}
    for line in text.splitlines():
        line = line.split("%", 1)[0]
        if "=" in line:
            k, v = line.split("=", 1)
            if k.strip() and v.strip():
                d[k.strip()] = v.strip()
    return d


def test_gamm_example_case_implicit_steps_match_oracle():
    """The reference's shipped GAMM example as it is set up (its 627-triangle mesh, wall
    distance and parameters.txt: AdiabaticEulers, p = 1, BDF1, CFL 5, artificial viscosity with
    dampTol 3, penalty 1, ilu0): three implicit steps from the free stream, GPU against oracle."""
    g0 = np.load(os.path.join(os.path.dirname(__file__), "golden", "gamm_mesh.npz"))
    props = _parameters_dict(str(g0["parameters"]))
    props.update(newtonIters=2, iterativeSolverTol=1e-12)
    o = of.Oracle(props, g0["vertices"], g0["elements"], g0["neighbors"], g0["wall_distance"])
    g = fg.GpuMesh(props, g0["vertices"], g0["elements"], g0["neighbors"], g0["wall_distance"])
    try:
        assert np.array_equal(g.get_state(0), o.get_state(0))
        so = o.run_implicit(3)
        sg = fg.GpuImplicitSolver(g, bdf_order=1, newton_iters=2, steps=3, cfl=5.0, linear_tol=1e-12, max_restarts=20,
                                  preconditioner="ilu0").solve()
        assert abs(sg[0] - so[0]) <= 1e-10 * so[0]
        err = cases.rel_err_per_component(g.get_state(0), o.get_state(0), o.n_basis, o.n_eqs)
        assert np.all(err <= 1e-6), err
    finally:
        g.close()


def test_ilu0_preconditioner_matches_oracle_iterations():
    """'ilu0' runs on the block ILU(0) kernels; GMRES needs the oracle's ILU0 iteration count."""
    props = cases.ns_props(2, reynolds=500.0)
    m, tt = cases.channel(10, 5, seed=3, wall=meshgen.WALL)
    o, g, W = make_pair(props, m, tt, amp=0.01)
    o.limiter()
    g.limiter()
    o.assemble(0.5, -1)
    fg.JacobiAssembler(g, bdf_order=1).assemble(0.5, -1)
    ls = fg.LinearSolver(g, "ilu0", tol=1e-8, max_restarts=5)
    ok, _ = ls.solve()
    ok_o, _, it_o, _ = o.linear_solve("ilu0", 1e-8)
    assert ok and ok_o
    assert abs(ls.iterations - it_o) <= 1, (ls.iterations, it_o)


@pytest.mark.parametrize("kind,order", [("euler", 3), ("ns", 3), ("ns3", 2), ("sa", 2)])
def test_residual_with_mesh_velocity_matches_oracle(kind, order):
    """ALE terms: a seeded smooth mesh velocity at the vertices enters the face fluxes
    (u . n), the moving-wall flux and the volume term -u W (DGpure.java:116-353,
    Element.java:299-332)."""
    if kind == "ns3":
        m, tt = cases.box(4, 3, 3, seed=2, wall=meshgen.WALL)
        props = cases.ns3_props(order)
    else:
        wall = meshgen.INVISCID_WALL if kind == "euler" else meshgen.WALL
        m, tt = cases.channel(10, 5, seed=order, wall=wall)
        if kind == "sa":
            m.wall_distance[:] = np.maximum(m.wall_distance, 1e-3)
        props = props_for(kind, order)
    x = m.vertices
    u = np.stack([0.05 * np.sin(2 * x[:, 0] + x[:, 1]), 0.03 * np.cos(x[:, 0] - 2 * x[:, 1])] +
                 ([0.02 * np.sin(x[:, 2] + x[:, 0])] if m.dim == 3 else []), axis=1)
    o = of.Oracle(props, m.vertices, m.elements, tt, m.wall_distance, mesh_velocity=u)
    g = fg.GpuMesh(props, m.vertices, m.elements, tt, m.wall_distance, mesh_velocity=u)
    W = cases.perturbed(o.get_state(0), o.n_basis, o.n_eqs, np.random.default_rng(3), 0.02)
    o.set_state(W)
    g.set_state(W)
    o.limiter()
    g.limiter()
    err = cases.rel_err_per_component(g.residuum(), o.residual(), o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-12), err


@pytest.mark.parametrize("dim", [2, 3])
def test_residual_with_host_buffers_equals_resident_residual(dim):
    """fp_residual with host input and output overlaps the state upload, the passes and the
    residual download chunk by chunk (2D: 49,868 triangles in 3 chunks; 3D: 18,000
    tetrahedra in 2 chunks).  Its result must equal, bit for bit, the residual of the same
    state evaluated on the device in one pass, on consecutive calls with different states,
    through fresh buffers and through the same pinned buffers (the captured graph)."""
    if dim == 2:
        m, tt = cases.channel(274, 91, seed=1, wall=meshgen.WALL)
        props = cases.ns_props(3, reynolds=5000.0)
    else:
        m, tt = cases.box(30, 10, 10, seed=1)
        props = cases.euler3_props(3)
    g = fg.GpuMesh(props, m.vertices, m.elements, tt, m.wall_distance)
    try:
        rng = np.random.default_rng(5)
        W0 = g.get_state(0)
        g.limiter()
        prev = None
        for _ in range(2):
            W = cases.perturbed(W0, g.n_basis, g.n_eqs, rng, 0.01)
            chunked = g.residuum(W)
            resident = g.residuum()
            assert np.array_equal(chunked, resident)
            assert np.all(np.isfinite(chunked))
            if prev is not None:
                assert not np.array_equal(chunked, prev)
            prev = chunked
        # the same pinned host buffers three times: the direct sequence, then its captured
        # CUDA graph (captured on the second call, replayed on the third)
        import torch
        Wh = torch.empty((g.n_elem, g.n_basis * g.n_eqs), dtype=torch.float64, pin_memory=True).numpy()
        Rh = torch.empty((g.n_elem, g.n_basis * g.n_eqs), dtype=torch.float64, pin_memory=True).numpy()
        for _ in range(3):
            Wh[:] = cases.perturbed(W0, g.n_basis, g.n_eqs, rng, 0.01)
            Rh[:] = np.nan
            assert fg.lib().fp_residual(g.ctx, fg._dp(Wh), fg._dp(Rh)) == 0
            resident = g.residuum()
            assert np.array_equal(Rh, resident)
            assert not np.array_equal(resident, prev)
            prev = resident
    finally:
        g.close()


def test_bdf2_temporal_order_on_gamm():
    """BDF2 temporal order on the reference's GAMM example, the check its author records
    (ZMENY_V2.md:45: fixed dt, t = 0.1, Newton to 1e-11, ratio of the differences of successive
    solutions when dt is halved 3.88 / 3.99 / 4.00; the dt sequence is not recorded).  Here the
    GAMM mesh and parameters with BDF2, no artificial viscosity (dampTol 0: the limiter's eps,
    evaluated once per step, adds a first-order term), dt = 0.1 / N for N = 20 ... 320: the
    oracle's and the GPU's ratios agree to 1e-3, are within 0.06 of the recorded ones, and the
    GPU's solutions equal the oracle's to 1e-8 per equation."""
    g0 = np.load(os.path.join(os.path.dirname(__file__), "golden", "gamm_mesh.npz"))
    props = {k: v for k, v in _parameters_dict(str(g0["parameters"])).items() if k != "CFL"}
    props.update(dampTol=0, timeOrder=2, newtonIters=30, newtonIterTol=1e-11, iterativeSolverTol=1e-13)
    Ns = (20, 40, 80, 160, 320)
    sol_o, sol_g = [], []
    for N in Ns:
        p = dict(props, dt=0.1 / N)
        o = of.Oracle(p, g0["vertices"], g0["elements"], g0["neighbors"], g0["wall_distance"])
        so = o.run_implicit(N)
        g = fg.GpuMesh(p, g0["vertices"], g0["elements"], g0["neighbors"], g0["wall_distance"])
        sg = fg.GpuImplicitSolver(g, bdf_order=2, newton_iters=30, newton_tol=1e-11, steps=N, dt=0.1 / N,
                                  linear_tol=1e-13, restart=30, max_restarts=20, preconditioner="ilu0").solve()
        assert sg[4] == so[4] == N
        assert abs(sg[0] - 0.1) <= 1e-12 and abs(so[0] - 0.1) <= 1e-12
        sol_o.append(o.get_state(0))
        sol_g.append(g.get_state(0))
        err = cases.rel_err_per_component(sol_g[-1], sol_o[-1], o.n_basis, o.n_eqs)
        assert np.all(err <= 1e-8), (N, err)
        g.close()

    def ratios(sols):
        d = [np.linalg.norm(sols[i] - sols[i + 1]) for i in range(len(sols) - 1)]
        return np.array([d[i] / d[i + 1] for i in range(len(d) - 1)])

    ro, rg = ratios(sol_o), ratios(sol_g)
    assert np.all(np.abs(rg - ro) <= 1e-3), (rg, ro)
    assert np.all(np.abs(ro - np.array([3.88, 3.99, 4.00])) <= 0.06), ro
