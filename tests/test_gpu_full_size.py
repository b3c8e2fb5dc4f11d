"""The configurations at their full sizes.

3D Euler p = 2 on the 100 x 34 x 34 x 6 = 693,600-tetrahedron bump box (6.9 M DOF): the
oracle's element tables take about 225 KB per element (157 GB at this size), so it evaluates a
seeded sample instead: 4,000 random elements plus 500 boundary elements, each with its face
neighbours (an element's residual depends only on its own and its neighbours' coefficients and
geometry, so the sampled elements' residuals in the patch equal their residuals in the whole
mesh; the patch's cut faces only touch the halo, which is not compared).  GPU residual of the
whole mesh against the oracle on the sample, per equation 1e-12.  Size-independent properties
besides: the residual of the seeded free stream is finite, and the JVP agrees with central
finite differences (step 1e-7) on 20 seeded random directions: 99.99 % of the entries within
1e-6 of the largest difference quotient and the relative L2 error below 1e-5.

2D RANS Spalart-Allmaras p = 2 on the full 99,328-triangle NACA 0012 O-grid (first cell 1e-5,
growth 1.15, far field at 50 chords): GPU residual against the oracle on the whole mesh, per
equation 1e-12.  (Not every entry: among the 10 M face points a few have
Lax-Friedrichs' max(lambda_L, lambda_R) switch branch inside the finite-difference step, where
the flux is not differentiable and the difference quotient, not the tangent, is off.)"""
import numpy as np
import pytest

import flowpro_v2_b200 as fg
from flowpro_v2_b200 import meshgen
from oracle import oracle_ffi as of
from tests import cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def box3d():
    m = meshgen.bump_box(100, 34, 34, seed=1)
    tt = fg.create_neighbor_matrix(3, m.elements, m.boundary)
    g = fg.GpuMesh(cases.euler3_props(3), m.vertices, m.elements, tt, m.wall_distance)
    rng = np.random.default_rng(11)
    W = cases.perturbed(g.get_state(0), g.n_basis, g.n_eqs, rng, 0.01)
    g.set_state(W)
    g.limiter()
    yield g, W, m, tt
    g.close()


def _patch(vertices, elements, tt, sample):
    """sample elements plus their face neighbours as a mesh of its own: (vertices, elements,
    neighbour matrix, patch element ids, positions of the sample in the patch); faces that
    leave the patch become inviscid walls (they belong to halo elements only)"""
    S = np.unique(sample)
    nb = tt[S]
    P = np.unique(np.concatenate([S, nb[nb >= 0]]))
    loc = -np.ones(elements.shape[0], dtype=np.int64)
    loc[P] = np.arange(P.size)
    el = elements[P]
    used, inv = np.unique(el.ravel(), return_inverse=True)
    ttp = tt[P].copy()
    inner = ttp >= 0
    mapped = np.where(inner, loc[np.where(inner, ttp, 0)], ttp)
    mapped = np.where(inner & (mapped < 0), meshgen.INVISCID_WALL, mapped)
    return (vertices[used], inv.reshape(el.shape).astype(np.int32), mapped.astype(np.int32), P,
            loc[S].astype(np.int64))


def test_config3_residual_matches_oracle_on_a_sample(box3d):
    g, W, m, tt = box3d
    rng = np.random.default_rng(31)
    boundary_el = np.flatnonzero((tt < 0).any(axis=1))
    sample = np.concatenate([rng.choice(g.n_elem, 4000, replace=False), rng.choice(boundary_el, 500, replace=False)])
    v, el, ttp, P, pos = _patch(m.vertices, m.elements, tt, sample)
    o = of.Oracle(cases.euler3_props(3), v, el, ttp, None)
    o.set_state(W[P])
    o.limiter()
    Ro = o.residual().reshape(-1, o.nb)[pos]
    Rg = g.residuum().reshape(-1, g.nb)[np.unique(sample)]
    err = cases.rel_err_per_component(Rg, Ro, o.n_basis, o.n_eqs)
    assert np.all(err <= 1e-12), err


def test_config4_full_naca_residual_matches_oracle():
    m = meshgen.naca0012_o_mesh()
    tt = of.create_neighbor_matrix(3, m.elements, m.boundary)
    assert m.elements.shape[0] == 99328
    props = cases.sa_props(3)
    g = fg.GpuMesh(props, m.vertices, m.elements, tt, m.wall_distance)
    o = of.Oracle(props, m.vertices, m.elements, tt, m.wall_distance)
    rng = np.random.default_rng(41)
    W = cases.perturbed(o.get_state(0), o.n_basis, o.n_eqs, rng, 0.01)
    o.set_state(W)
    g.set_state(W)
    o.limiter()
    g.limiter()
    err = cases.rel_err_per_component(g.residuum(), o.residual(), o.n_basis, o.n_eqs)
    g.close()
    assert np.all(err <= 1e-12), err


def test_config3_residual_finite(box3d):
    g, W, m, tt = box3d
    assert g.n_elem == 693600 and g.n_basis == 10 and g.n_eqs == 5
    R = g.residuum()
    assert np.all(np.isfinite(R))
    assert np.max(np.abs(R)) > 0


def test_config3_jvp_against_finite_differences(box3d):
    g, W, m, tt = box3d
    rng = np.random.default_rng(20)
    scale = np.abs(W).mean(axis=0)
    h = 1e-7
    worst_q, worst_l2 = 0.0, 0.0
    for _ in range(20):
        V = rng.standard_normal(W.shape) * scale
        Jv = g.jvp(V)
        Rp = g.residuum(W + h * V)
        Rm = g.residuum(W - h * V)
        fd = (Rp - Rm) / (2 * h)
        err = np.abs(Jv - fd)
        worst_q = max(worst_q, np.quantile(err, 0.9999) / np.max(np.abs(fd)))
        worst_l2 = max(worst_l2, np.linalg.norm(Jv - fd) / np.linalg.norm(fd))
    g.set_state(W)
    assert worst_q <= 1e-6, worst_q
    assert worst_l2 <= 1e-5, worst_l2
