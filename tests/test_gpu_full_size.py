"""The 3D configuration at its full size: 3D Euler p = 2 on the 100 x 34 x 34 x 6 =
693,600-tetrahedron bump box (6.9 M DOF).  The oracle cannot evaluate this size in a test,
so the checks are size-independent properties: the residual of the seeded free stream is
finite, and the JVP agrees with central finite differences (step 1e-7) on 20 seeded random
directions: 99.99 % of the entries within 1e-6 of the largest difference quotient and the
relative L2 error below 1e-5.  (Not every entry: among the 10 M face points a few have
Lax-Friedrichs' max(lambda_L, lambda_R) switch branch inside the finite-difference step, where
the flux is not differentiable and the difference quotient, not the tangent, is off.)"""
import numpy as np
import pytest

import flowpro_v2_b200 as fg
from flowpro_v2_b200 import meshgen
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
    return g, W


def test_config3_residual_finite(box3d):
    g, W = box3d
    assert g.n_elem == 693600 and g.n_basis == 10 and g.n_eqs == 5
    R = g.residuum()
    assert np.all(np.isfinite(R))
    assert np.max(np.abs(R)) > 0


def test_config3_jvp_against_finite_differences(box3d):
    g, W = box3d
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
