"""The CPU oracle against the reference's own pins (FlowPro/src/test/java/flowpro/core/*).

* neighbors.txt of the shipped GAMM mesh (createNeighborMatrix, bit-exact)
* ConvergenceOrderTest: L2 error rates of DGpure for the manufactured solution
  (ConvergenceOrderTest.java:47-61: advection rate > p + 0.7; advection-diffusion
  rate > p + 0.7 for odd p, > p - 0.3 for even p)
* LinearSolverTest: GMRES + {ilu0, blockilu0, blockjacobi, none} against a direct
  solve of the assembled system, rel. max-norm < 1e-8 (LinearSolverTest.java:27-60)
"""
import os

import numpy as np
import pytest

from flowpro_v2_b200 import meshgen
from oracle import oracle_ffi as of
from tests import cases

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "gamm_mesh.npz")


def test_gamm_neighbors_bit_exact():
    g = np.load(GOLDEN)
    tt = of.create_neighbor_matrix(3, g["elements"], g["boundary"])
    assert np.array_equal(tt, g["neighbors"])


def test_java_random_lcg():
    # java.util.Random(1).nextDouble() known first values
    r = of.java_random(1, 2)
    assert abs(r[0] - 0.7308781907032909) < 1e-16 and abs(r[1] - 0.41008081149220166) < 1e-16


def _rate(p, k):
    errs = []
    for n in (4, 8, 16):
        m = meshgen.square_mesh(n, 1.0, meshgen.INLET)
        tt = of.create_neighbor_matrix(3, m.elements, m.boundary)
        o = of.Oracle(cases.scalar_props(p + 1, k), m.vertices, m.elements, tt, m.wall_distance)
        o.run_implicit(4)
        errs.append(o.l2_error_scalar())
    return np.log(errs[-2] / errs[-1]) / np.log(2)


@pytest.mark.parametrize("p", [0, 1, 2, 3])
def test_convergence_order_advection(p):
    assert _rate(p, 0.0) > p + 0.7


@pytest.mark.parametrize("p", [1, 2, 3])
def test_convergence_order_advection_diffusion(p):
    assert _rate(p, 0.1) > p + (0.7 if p % 2 == 1 else -0.3)


def _direct(I, J, H, b):
    n = b.size
    A = np.zeros((n, n))
    for i in range(n):
        A[i, J[I[i]:I[i + 1]]] += H[I[i]:I[i + 1]]
    return np.linalg.solve(A, b)


@pytest.mark.parametrize("ordering", ["rcm", "none"])
def test_linear_solver_matches_direct(ordering):
    m = meshgen.square_mesh(4, 1.0, meshgen.INLET)
    tt = of.create_neighbor_matrix(3, m.elements, m.boundary)
    props = cases.scalar_props(2, 0.1)
    props["elementOrdering"] = ordering
    o = of.Oracle(props, m.vertices, m.elements, tt, m.wall_distance)
    W = of.java_random(2, o.n_elem * o.nb)
    o.set_state(W)
    o.limiter()
    o.assemble(0.05, -1)
    for prec in ("ilu0", "blockilu0", "blockjacobi", "none"):
        ok, x, it, err = o.linear_solve(prec, 1e-12)
        I, J, H, b = o.matrix()
        xr = _direct(I, J, H, b)
        assert ok, prec
        assert np.max(np.abs(x - xr)) / np.max(np.abs(xr)) < 1e-8, prec


@pytest.mark.parametrize("order", [1, 2])
def test_wall_integrals_vanish_for_uniform_pressure(order):
    """Forces and the lift / drag functionals integrate p n over the channel walls; for the
    free stream (uniform p, zero velocity gradient) the walls' projected lengths cancel, so
    every component vanishes to rounding."""
    m, tt = cases.channel(12, 5, seed=2, wall=meshgen.WALL)
    o = of.Oracle(cases.ns_props(order), m.vertices, m.elements, tt, m.wall_distance)
    W = o.get_state(0)
    o.set_state(W)
    F = o.forces(meshgen.WALL)
    lift, glift = o.functional(0)
    drag, _ = o.functional(1, gradient=False)
    p_scale = 3.0 * 0.8430 / 0.4  # wall length x a pressure scale
    assert np.max(np.abs(F)) <= 1e-12 * p_scale
    assert abs(lift) <= 1e-12 * p_scale and abs(drag) <= 1e-12 * p_scale
    assert np.max(np.abs(glift)) > 0


@pytest.mark.parametrize("kind", ["scalar", "ns"])
def test_scalar_ilu0_equals_block_ilu0(kind):
    """ILU0 (ILU0.java:34-96) on the CRS matrix of dense element blocks has the block fill
    pattern, so it is BlockILU0 (BlockILU0.java:47-243): same GMRES iterations, same solution."""
    if kind == "scalar":
        m = meshgen.square_mesh(4, 1.0, meshgen.INLET)
        tt = of.create_neighbor_matrix(3, m.elements, m.boundary)
        props = cases.scalar_props(2, 0.1)
    else:
        m, tt = cases.channel(10, 5, seed=3, wall=meshgen.WALL)
        props = cases.ns_props(2, reynolds=500.0)
    o = of.Oracle(props, m.vertices, m.elements, tt, m.wall_distance)
    W = cases.perturbed(o.get_state(0), o.n_basis, o.n_eqs, np.random.default_rng(7), 0.01)
    o.set_state(W)
    o.limiter()
    o.assemble(0.5, -1)
    ok1, x1, it1, _ = o.linear_solve("ilu0", 1e-10)
    ok2, x2, it2, _ = o.linear_solve("blockilu0", 1e-10)
    assert ok1 and ok2 and it1 == it2
    assert np.max(np.abs(x1 - x2)) <= 1e-12 * np.max(np.abs(x2))


@pytest.mark.parametrize("time_order", [1, 2])
def test_free_stream_preservation_on_deforming_mesh(time_order):
    """FreeStreamPreservationTest.gasAtRestOnDeformingMesh (FlowPro/src/test/java/flowpro/core/
    FreeStreamPreservationTest.java:24-61) on the oracle: gas at rest in the closed 10 x 10
    square (8 x 8 cells, inviscid walls), the Test2D deformation, dt 0.25, 20 BDF steps with two
    Newton iterations; with the discrete GCL the state stays at rest (< 1e-10), without it not
    (> 1e-4)."""
    m = meshgen.square_mesh(8, 10.0, meshgen.INVISCID_WALL)
    tt = of.create_neighbor_matrix(3, m.elements, m.boundary)
    rest = np.array([1.0, 0.0, 0.0, 2.5])  # rho, rho u, rho v, E = p / (kappa - 1)
    deviation = {}
    for gcl in ("true", "false"):
        props = dict(model="NavierStokes", dimension=2, isFlowViscous="false", cv=1, kappa=1.4,
                     isInletSupersonic="false", attackAngle=0, pIn0=1, rhoIn0=1, pOut=1, movingMesh="true",
                     meshDeformationType="Test2D", gcl=gcl, timeMethod="BDF", timeOrder=time_order,
                     preconditioner="ilu0", iterativeSolverTol=1e-12, order=2, dt=0.25, newtonIters=2,
                     newtonIterTol=1e-12, penalty=0, dampTol=0, dampConst=0)
        o = of.Oracle(props, m.vertices, m.elements, tt)
        o.run_implicit(20)
        W = o.get_state(0)
        deviation[gcl] = np.max(np.abs(W - np.repeat(rest, o.n_basis)[None, :]))
    assert deviation["true"] < 1e-10, deviation
    assert deviation["false"] > 1e-4, deviation
