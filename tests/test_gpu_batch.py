"""Batched serving: independent bump-channel cases of uneven size, order, inlet Mach and
bump height (meshgen.serving_cases, scaled down) solved concurrently by
fp_batch_solve_implicit with FP32 block-Jacobi factors under FP64 GMRES.  Each case ends as
its own sequential solve does (bit for bit), reaches the 1e-10 residual target, and its wall
force agrees with the FP64 oracle's converged solution to 1e-8."""
import numpy as np
import pytest

import flowpro_v2_b200 as fg
from flowpro_v2_b200 import meshgen
from oracle import oracle_ffi as of

pytestmark = pytest.mark.gpu

SOLVER = dict(steps=300, cfl=0.0, vary_cfl=1, max_cfl=1e5, linear_tol=1e-3, preconditioner="blockjacobi",
              restart=40, max_restarts=5, target_residuum=1e-10)


def case_mesh_props(c):
    m = meshgen.bump_channel(nx=c["nx"], ny=c["ny"], height=c["height"], seed=c["seed"], wall=meshgen.INVISCID_WALL)
    tt = fg.create_neighbor_matrix(2, m.elements, m.boundary)
    props = dict(model="NavierStokes", dimension=2, kappa=1.4, cv=1, isFlowViscous="false", pIn0=1, rhoIn0=1,
                 pOut=c["pOut"], order=c["order"], penalty=0, dampTol=0, dampConst=0)
    return m, tt, props


def test_batched_cases_match_sequential_solves_and_oracle():
    cases = meshgen.serving_cases(4, seed=5, min_elements=150, max_elements=500)
    built = [case_mesh_props(c) for c in cases]
    meshes = [fg.GpuMesh(p, m.vertices, m.elements, tt) for m, tt, p in built]
    out, status = fg.batch_solve_implicit(meshes, threads=4, precision=fg.FP32, **SOLVER)
    assert np.all(status == 0), status
    assert np.all(out[:, 1] <= 1e-10), out[:, 1]
    for i, (m, tt, props) in enumerate(built):
        # the same case alone on the device: identical result
        g = fg.GpuMesh(props, m.vertices, m.elements, tt)
        st = fg.GpuImplicitSolver(g, precision=fg.FP32, **SOLVER).solve()
        assert np.array_equal(g.get_state(0), meshes[i].get_state(0))
        assert st[4] == out[i, 4]
        # the FP64 oracle's converged solution: same wall force
        o = of.Oracle(dict(props, CFL=0, maxCFL=1e5, iterativeSolverTol=1e-3, preconditioner="blockjacobi"),
                      m.vertices, m.elements, tt)
        so = o.run_implicit(300, 1e-10)
        assert so[1] <= 1e-10
        Fo = o.forces(meshgen.INVISCID_WALL)
        Fg = meshes[i].forces(meshgen.INVISCID_WALL)
        assert np.max(np.abs(Fg - Fo)) <= 1e-8 * np.max(np.abs(Fo)), (i, Fg, Fo)


def test_batch_rejects_block_ilu0():
    c = meshgen.serving_cases(1, seed=1, min_elements=100, max_elements=120)[0]
    m, tt, props = case_mesh_props(c)
    g = fg.GpuMesh(props, m.vertices, m.elements, tt)
    with pytest.raises(fg.FlowGpuError):
        fg.batch_solve_implicit([g], threads=1, **dict(SOLVER, preconditioner="blockilu0"))


BATCH_SOLVER = dict(steps=300, cfl=0.0, vary_cfl=1, max_cfl=1e5, linear_tol=1e-3, preconditioner="blockilu0",
                    jacobian=fg.JAC_MATRIXFREE, precision=fg.FP32, jac_lag=5, restart=40, max_restarts=5,
                    target_residuum=1e-10)


@pytest.mark.parametrize("order", [2, 3, 4])
def test_merged_batch_matches_single_solves_and_oracle(order):
    """fp_batch_upload / fp_batch_solve: cases of one order merged into one mesh, every kernel of
    a step one launch over all of them, GMRES per case in lockstep.  Each case reaches 1e-10, its
    state equals the same case solved alone (single-case matrix-free loop) to 1e-8 (both converge
    to the case's discrete steady state, by different iterates), and its wall force agrees with
    the FP64 oracle's converged solution to 1e-8."""
    cases = [dict(c, order=order) for c in meshgen.serving_cases(3, seed=7, min_elements=150, max_elements=400)]
    built = [case_mesh_props(c) for c in cases]
    b = fg.GpuBatch([(p, m.vertices, m.elements, tt, None) for m, tt, p in built])
    assert list(np.diff(b.case_e0)) == [m.elements.shape[0] for m, _, _ in built]
    out, status = b.solve(**BATCH_SOLVER)
    assert np.all(status == 0), status
    assert np.all(out[:, 1] <= 1e-10), out[:, 1]
    for i, (m, tt, props) in enumerate(built):
        Wb = b.case_state(i)
        g = fg.GpuMesh(props, m.vertices, m.elements, tt)
        st = fg.GpuImplicitSolver(g, **BATCH_SOLVER).solve()
        assert st[1] <= 1e-10
        Ws = g.get_state(0)
        assert np.max(np.abs(Wb - Ws)) <= 1e-8 * np.max(np.abs(Ws)), i
        g.set_state(Wb)
        Fb = g.forces(meshgen.INVISCID_WALL)
        g.close()
        o = of.Oracle(dict(props, CFL=0, maxCFL=1e5, iterativeSolverTol=1e-3, preconditioner="blockilu0"),
                      m.vertices, m.elements, tt)
        so = o.run_implicit(300, 1e-10)
        assert so[1] <= 1e-10
        Fo = o.forces(meshgen.INVISCID_WALL)
        assert np.max(np.abs(Fb - Fo)) <= 1e-8 * np.max(np.abs(Fo)), (i, Fb, Fo)
    b.close()
