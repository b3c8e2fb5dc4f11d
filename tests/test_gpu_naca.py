"""The RANS configuration on a (coarsened) NACA 0012 O-mesh: Spalart-Allmaras at M = 0.3,
alpha = 4 deg, Re = 3e6, wall distance from the edge-path distance.  Residual, forces and
functionals against the oracle; the exact tangent and its transpose (JVP / VJP) by the
dot-product identity and central differences, and against the oracle's finite-difference
Jacobian transposed; adjoint sensitivities of the lift to a flow parameter and to 50 seeded
surface-normal vertex perturbations (amplitude 1e-6) against tangent (direct) solves on the
same operator, with the parameter and geometry derivatives of the residual by central
differences.  The parameter is the outlet pressure: FlowPro's subsonic inlet prescribes total
pressure and density with the inflow normal to the boundary, so the angle of attack enters
the initial state only and dR/dalpha = 0 at a fixed state."""
import numpy as np
import pytest

import flowpro_v2_b200 as fg
from flowpro_v2_b200 import meshgen
from oracle import oracle_ffi as of
from tests import cases
from tests.test_gpu_parity import _dense_from_blocks

pytestmark = pytest.mark.gpu


def naca_case(order):
    m = meshgen.naca0012_o_mesh(n_around=64, first_height=1e-3, growth=1.3, radius=20.0)
    tt = fg.create_neighbor_matrix(2, m.elements, m.boundary)
    return m, tt, cases.sa_props(order)


def pair(order, seed=7, amp=0.01):
    m, tt, props = naca_case(order)
    o = of.Oracle(props, m.vertices, m.elements, tt, m.wall_distance)
    g = fg.GpuMesh(props, m.vertices, m.elements, tt, m.wall_distance)
    W = cases.perturbed(o.get_state(0), o.n_basis, o.n_eqs, np.random.default_rng(seed), amp)
    for which in (0, 1, 2):
        o.set_state(W, which)
        g.set_state(W, which)
    return m, tt, props, o, g, W


@pytest.mark.parametrize("order", [2, 3])
def test_sa_naca_residual_forces_functionals(order):
    m, tt, props, o, g, W = pair(order)
    o.limiter()
    g.limiter()
    err = cases.rel_err_per_component(g.residuum(), o.residual(), o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-12), err
    Fo, Fg = o.forces(meshgen.WALL), g.forces(meshgen.WALL)
    assert np.max(np.abs(Fg - Fo)) <= 1e-12 * np.max(np.abs(Fo))
    for kind, fk in ((0, fg.FUNCTIONAL_LIFT), (1, fg.FUNCTIONAL_DRAG)):
        Io, go = o.functional(kind)
        Ig, gg = g.functional(fk)
        assert abs(Ig - Io) <= 1e-12 * abs(Io)
        assert np.max(np.abs(gg - go)) <= 1e-6 * np.max(np.abs(go))


def test_sa_naca_vjp_against_oracle_jacobian_transpose():
    m, tt, props, o, g, W = pair(2)
    o.limiter()
    g.limiter()
    rng = np.random.default_rng(4)
    lam = rng.standard_normal(W.shape)
    v = rng.standard_normal(W.shape) * np.abs(W).mean(axis=0)
    JTl = g.vjp(lam)
    Jv = g.jvp(v)
    # exact tangent and transpose agree
    assert abs(np.sum(lam * Jv) - np.sum(JTl * v)) <= 1e-12 * np.linalg.norm(lam) * np.linalg.norm(Jv)
    # the tangent against central differences: the SA terms are not smooth everywhere (max(0, .),
    # the vorticity magnitude near zero vorticity of this near-free-stream state), so a few
    # quotients straddle a kink; the bulk agrees to 1e-6, the whole to 1e-4 in L2
    h = 1e-7
    fd = (g.residuum(W + h * v) - g.residuum(W - h * v)) / (2 * h)
    g.set_state(W)
    e_fd = np.abs(Jv - fd) / np.max(np.abs(fd))
    assert np.quantile(e_fd, 0.99) <= 1e-6, np.quantile(e_fd, 0.99)
    assert np.linalg.norm(Jv - fd) <= 1e-4 * np.linalg.norm(fd)
    # the reference's forward-difference Jacobian (h = 1e-8) transposed: its truncation error
    # is large where the SA source grows like 1/d^2 next to the wall; the bulk agrees to 1e-6
    o.assemble(1e12, -1)
    Do, No, _ = o.blocks()
    ref = -(_dense_from_blocks(Do, No, tt).T @ lam.reshape(-1)).reshape(W.shape)
    err = np.abs(JTl - ref) / np.max(np.abs(ref))
    assert np.quantile(err, 0.99) <= 1e-6, np.quantile(err, 0.99)


def test_sa_naca_adjoint_sensitivities_match_tangent_solves():
    m, tt, props, o, g, W = pair(2, amp=0.0)
    # a few pseudo-time steps from the free stream: a non-trivial state around the airfoil
    fg.GpuImplicitSolver(g, steps=5, cfl=2.0, linear_tol=1e-6, max_restarts=20, preconditioner="blockjacobi").solve()
    W = g.get_state(0)
    g.limiter()
    I0, dIdW = g.functional(fg.FUNCTIONAL_LIFT)
    dt = 1e-4  # the operator a1 M - dR/dW of a pseudo-time step, solved both ways
    asm = fg.JacobiAssembler(g, bdf_order=1)
    asm.assemble_exact(dt, -1.0)
    ok, psi, its = g.block_solve(dIdW, transpose=True, tol=1e-12, restart=60, max_restarts=40)
    assert ok, its

    def residual_at(vertices=None, pout=None):
        pr = dict(props) if pout is None else dict(props, pOut=pout)
        V = m.vertices if vertices is None else vertices
        wd = m.wall_distance if vertices is None else fg.wall_distance(V, m.elements, tt, meshgen.WALL)
        gp = fg.GpuMesh(pr, V, m.elements, tt, wd)
        gp.set_state(W)
        gp.limiter()
        R = gp.residuum()
        I = gp.functional(fg.FUNCTIONAL_LIFT, gradient=False)[0]
        gp.close()
        return R, I

    def check(bR, dI_explicit):
        ok, x, _ = g.block_solve(bR, transpose=False, preconditioner="blockjacobi", tol=1e-12, restart=60,
                                 max_restarts=40)
        assert ok
        adj = dI_explicit + np.sum(psi * bR)
        tan = dI_explicit + np.sum(dIdW * x)
        return adj, tan

    # outlet pressure
    p0, ep = props["pOut"], 1e-6
    Rp, _ = residual_at(pout=p0 + ep)
    Rm, _ = residual_at(pout=p0 - ep)
    bR = (Rp - Rm) / (2 * ep)
    assert np.max(np.abs(bR)) > 0
    adj, tan = check(bR, 0.0)
    assert abs(adj - tan) <= 1e-8 * abs(tan), (adj, tan)
    # 50 seeded surface-normal perturbations of wall vertices
    rng = np.random.default_rng(50)
    wall_v = np.unique(m.boundary[m.boundary[:, 0] == meshgen.WALL][:, 1:])
    picks = rng.choice(wall_v, size=50, replace=False)
    eps = 1e-6
    worst = 0.0
    for v in picks:
        # outward normal from the neighbouring wall vertices (they share a wall edge with v)
        edges = m.boundary[(m.boundary[:, 0] == meshgen.WALL) & np.any(m.boundary[:, 1:] == v, axis=1)][:, 1:]
        nbrs = [e[0] if e[1] == v else e[1] for e in edges]
        t = m.vertices[nbrs[1]] - m.vertices[nbrs[0]]
        nrm = np.array([t[1], -t[0]]) / np.linalg.norm(t)
        if np.dot(nrm, m.vertices[v] - np.array([0.5, 0.0])) < 0:
            nrm = -nrm
        Vp, Vm = m.vertices.copy(), m.vertices.copy()
        Vp[v] += eps * nrm
        Vm[v] -= eps * nrm
        (Rp, Ip), (Rm, Im) = residual_at(vertices=Vp), residual_at(vertices=Vm)
        adj, tan = check((Rp - Rm) / (2 * eps), (Ip - Im) / (2 * eps))
        worst = max(worst, abs(adj - tan) / max(abs(tan), 1e-12))
    assert worst <= 1e-8, worst
