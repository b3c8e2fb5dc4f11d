"""Forces, functionals, exact Jacobian blocks, VJP and the discrete adjoint on the GPU.

Tolerances:
  * forces and functional values: 1e-12 relative (same quadrature, FP64);
  * functional gradient against the reference's finite differences (h = 1e-8,
    Element.exportLocalFunctionalDerivative): 1e-6 relative;
  * exact tangent blocks against the finite-difference blocks (GPU and oracle): 1e-6;
  * VJP: the dot-product identity <lam, J v> = <J^T lam, v> to 1e-12 (exact derivatives on
    both sides), and against the oracle's finite-difference Jacobian transposed to 1e-6;
  * adjoint sensitivity of the lift to the outlet pressure against central differences of
    converged solutions: 1e-5 relative.
"""
import numpy as np
import pytest

import flowpro_v2_b200 as fg
from flowpro_v2_b200 import meshgen
from oracle import oracle_ffi as of
from tests import cases
from tests.test_gpu_parity import _dense_from_blocks, make_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,order", [("ns", 2), ("ns", 3), ("euler", 3), ("sa", 3), ("ns3", 2)])
def test_forces_match_oracle(kind, order):
    if kind == "ns3":
        m, tt = cases.box(4, 3, 3, seed=3, wall=meshgen.WALL)
        props, bc = cases.ns3_props(order), meshgen.WALL
    else:
        wall = meshgen.INVISCID_WALL if kind == "euler" else meshgen.WALL
        m, tt = cases.channel(10, 5, seed=order, wall=wall)
        if kind == "sa":
            m.wall_distance[:] = np.maximum(m.wall_distance, 1e-3)
        props = {"ns": cases.ns_props(order, reynolds=500.0), "euler": cases.euler_props(order),
                 "sa": cases.sa_props(order)}[kind]
        bc = wall
    o, g, W = make_pair(props, m, tt)
    Fo = o.forces(bc)
    Fg = g.forces(bc)
    assert np.max(np.abs(Fo)) > 0
    assert np.max(np.abs(Fg - Fo)) <= 1e-12 * np.max(np.abs(Fo)), (Fg, Fo)


@pytest.mark.parametrize("functional", [fg.FUNCTIONAL_LIFT, fg.FUNCTIONAL_DRAG])
@pytest.mark.parametrize("order", [2, 3])
def test_functional_and_gradient_match_oracle(functional, order):
    m, tt = cases.channel(10, 5, seed=4, wall=meshgen.WALL)
    o, g, W = make_pair(cases.ns_props(order, reynolds=500.0), m, tt)
    Io, go = o.functional(0 if functional == fg.FUNCTIONAL_LIFT else 1)
    Ig, gg = g.functional(functional)
    assert abs(Ig - Io) <= 1e-12 * abs(Io)
    assert np.max(np.abs(go)) > 0
    assert np.max(np.abs(gg - go)) <= 1e-6 * np.max(np.abs(go))


@pytest.mark.parametrize("kind,order", [("euler", 3), ("ns", 2), ("ns3", 2)])
def test_exact_blocks_match_finite_differences(kind, order):
    if kind == "ns3":
        m, tt = cases.box(4, 3, 3, seed=2, wall=meshgen.WALL)
        props = cases.ns3_props(order)
    else:
        wall = meshgen.WALL if kind == "ns" else meshgen.INVISCID_WALL
        m, tt = cases.channel(8, 4, seed=3, wall=wall)
        props = cases.euler_props(order) if kind == "euler" else cases.ns_props(order, reynolds=500.0)
    o, g, W = make_pair(props, m, tt)
    o.limiter()
    g.limiter()
    asm = fg.JacobiAssembler(g, bdf_order=1)
    asm.assemble(0.05, -1)
    Dfd, Nfd, rfd = asm.blocks()
    asm.assemble_exact(0.05, -1)
    Dex, Nex, rex = asm.blocks()
    o.assemble(0.05, -1)
    Do, No, ro = o.blocks()
    scale = np.max(np.abs(Do))
    assert np.max(np.abs(Dex - Dfd)) <= 1e-6 * scale
    assert np.max(np.abs(Nex - Nfd)) <= 1e-6 * scale
    assert np.max(np.abs(Dex - Do)) <= 1e-6 * scale
    assert np.max(np.abs(Nex - No)) <= 1e-6 * scale
    assert np.max(np.abs(rex - rfd)) <= 1e-14 * np.max(np.abs(rfd))


@pytest.mark.parametrize("kind", ["ns", "euler"])
def test_vjp_dot_product_and_oracle(kind):
    wall = meshgen.WALL if kind == "ns" else meshgen.INVISCID_WALL
    m, tt = cases.channel(8, 4, seed=5, wall=wall)
    props = cases.ns_props(2, reynolds=500.0) if kind == "ns" else cases.euler_props(3)
    o, g, W = make_pair(props, m, tt)
    o.limiter()
    g.limiter()
    rng = np.random.default_rng(3)
    lam = rng.standard_normal(W.shape)
    v = rng.standard_normal(W.shape)
    Jv = g.jvp(v)
    JTl = g.vjp(lam)
    lhs, rhs = np.sum(lam * Jv), np.sum(JTl * v)
    assert abs(lhs - rhs) <= 1e-12 * np.sqrt(np.sum(lam * lam) * np.sum(Jv * Jv))
    # the VJP kernel stores no Jacobian; it equals the product with the exact steady blocks
    # (-dR/dW, assembled afterwards) transposed to rounding
    asm = fg.JacobiAssembler(g)
    asm.assemble_exact(0.0, -1.0)
    De, Ne, _ = asm.blocks()
    ref_ex = -(_dense_from_blocks(De, Ne, tt).T @ lam.reshape(-1)).reshape(W.shape)
    assert np.max(np.abs(JTl - ref_ex)) <= 1e-12 * np.max(np.abs(ref_ex))
    # the oracle's finite-difference Jacobian (a1 M - dR/dW with a1 = 1e-12) transposed
    o.assemble(1e12, -1)
    Do, No, _ = o.blocks()
    A = _dense_from_blocks(Do, No, tt)
    ref = -(A.T @ lam.reshape(-1)).reshape(W.shape)
    assert np.max(np.abs(JTl - ref)) <= 1e-6 * np.max(np.abs(ref))


def test_adjoint_lift_sensitivity_to_outlet_pressure():
    """dI/dpOut of the lift of a converged laminar channel flow: adjoint (exact steady
    blocks, transposed GMRES) against central differences of converged solutions."""
    m, tt = cases.channel(10, 4, seed=6, wall=meshgen.WALL)
    base = cases.ns_props(2, reynolds=200.0)

    def solve(pout, W0=None, steps=200):
        props = dict(base, pOut=pout)
        g = fg.GpuMesh(props, m.vertices, m.elements, tt, m.wall_distance)
        if W0 is not None:
            for which in (0, 1, 2):
                g.set_state(W0, which)
        st = fg.GpuImplicitSolver(g, steps=steps, cfl=0.0, vary_cfl=1, max_cfl=1e6, linear_tol=1e-8,
                                  preconditioner="blockjacobi", max_restarts=20, restart=40,
                                  target_residuum=1e-13).solve()
        return g, st

    p0, eps = base["pOut"], 1e-4
    g0, st = solve(p0)
    assert st[1] < 1e-9, st
    W0 = g0.get_state(0)
    # tighten from the converged state
    g0, _ = solve(p0, W0, steps=20)
    W0 = g0.get_state(0)
    I0, dIdW = g0.functional(fg.FUNCTIONAL_LIFT)
    asm = fg.JacobiAssembler(g0, bdf_order=1)
    asm.assemble_exact(0.0, -1.0)
    ok, psi, its = g0.adjoint_solve(dIdW, "blockjacobi", tol=1e-13, restart=60, max_restarts=40)
    assert ok, its
    # dR/dpOut at fixed W by central differences of the residual
    R = []
    for s in (+1, -1):
        gp = fg.GpuMesh(dict(base, pOut=p0 + s * eps), m.vertices, m.elements, tt, m.wall_distance)
        gp.set_state(W0)
        gp.limiter()
        R.append(gp.residuum())
    dRdp = (R[0] - R[1]) / (2 * eps)
    dI_adj = np.sum(psi * dRdp)
    # central differences of the converged functional
    Ival = []
    for s in (+1, -1):
        gs, _ = solve(p0 + s * eps, W0, steps=60)
        Ival.append(gs.functional(fg.FUNCTIONAL_LIFT, gradient=False)[0])
    dI_fd = (Ival[0] - Ival[1]) / (2 * eps)
    assert abs(dI_fd) > 0
    assert abs(dI_adj - dI_fd) <= 1e-5 * abs(dI_fd), (dI_adj, dI_fd)


@pytest.mark.parametrize("p,k", [(1, 0.0), (1, 0.1), (2, 0.0), (2, 0.1)])
def test_jacobian_test_restated(p, k):
    """JacobianTest.analyticMatchesFiniteDifferences (FlowPro/src/test/java/flowpro/core/
    JacobianTest.java:26-108) on the exact element blocks: TestScalarEquation (a = (1, 0.5),
    diffusion k) on the 3 x 1 square (writeSquareMesh(3, 1, -2)), W from java.util.Random(1)
    element by element; every block entry, own and neighbour, against -(R(W + h e_i) - R(W)) / h
    with h = 1e-6, max |exact - FD| / max |FD| < 1e-6 (the equation is linear)."""
    m = meshgen.square_mesh(3, 1.0, meshgen.INLET)
    tt = fg.create_neighbor_matrix(2, m.elements, m.boundary)
    g = fg.GpuMesh(cases.scalar_props(p + 1, k), m.vertices, m.elements, tt, m.wall_distance)
    try:
        nE, n = g.n_elem, g.nb
        W = of.java_random(1, nE * n).reshape(nE, n)
        g.set_state(W)
        g.limiter()
        asm = fg.JacobiAssembler(g, bdf_order=1)
        asm.assemble_exact(0.0, 0.0)  # steady: -dR/dW, A[perturbed][residual]
        D, N, _ = asm.blocks()
        h = 1e-6
        R0 = g.residuum(W)
        max_diff = max_entry = 0.0
        for r in range(nE):
            for i in range(n):
                Wh = W.copy()
                Wh[r, i] += h
                fd = -(g.residuum(Wh) - R0) / h  # column (r, i) of -dR/dW for every element
                max_diff = max(max_diff, np.max(np.abs(fd[r] - D[r, i])))
                max_entry = max(max_entry, np.max(np.abs(fd[r])))
                for e in range(nE):
                    for face in range(tt.shape[1]):
                        if tt[e, face] == r:
                            max_diff = max(max_diff, np.max(np.abs(fd[e] - N[e, face, i])))
                            max_entry = max(max_entry, np.max(np.abs(fd[e])))
        assert max_entry > 0
        assert max_diff / max_entry < 1e-6, max_diff / max_entry
    finally:
        g.close()
