"""The optimisation-toolbox export (OptimisationToolExport.export, mode "allmass") from the GPU
against the same files written from the oracle's values: functional, steady residual and
Jacobian blocks, functional derivative, mass matrices and basis weights, on the base mesh and
on one perturbed mesh."""
import os

import numpy as np
import pytest

import flowpro_v2_b200 as fg
from flowpro_v2_b200 import meshgen, optexport
from oracle import oracle_ffi as of
from tests import cases
from tests.test_optexport import _triplets, _values

pytestmark = pytest.mark.gpu


def _oracle_files(directory, props, m, tt, W, V1):
    os.makedirs(directory, exist_ok=True)
    o = of.Oracle(props, m.vertices, m.elements, tt, m.wall_distance)
    for which in (0, 1, 2):
        o.set_state(W, which)
    o.limiter()
    I0, dIdw = o.functional(0)
    o.assemble(0.0, 0.0)
    diag, neigh, _ = o.blocks()
    gpos = o.gindex()
    optexport.write_functional(directory, 0, I0)
    optexport.write_jacobian(directory, diag, neigh, tt, gpos)
    optexport.write_mass(directory, 0, o.mass_matrices(), gpos, o.n_eqs)
    optexport.write_residual(directory, 0, o.residual())
    optexport.write_functional_derivative(directory, dIdw)
    o1 = of.Oracle(props, V1, m.elements, tt, m.wall_distance)
    o1.set_state(W, 0)
    o1.limiter()
    optexport.write_mass(directory, 1, o1.mass_matrices(), gpos, o.n_eqs)
    optexport.write_functional(directory, 1, o1.functional(0, gradient=False)[0])
    optexport.write_residual(directory, 1, o1.residual())
    optexport.write_print_matrix(directory, o.basis_weights(), gpos, o.n_eqs)


def _close_values(a, b, rtol):
    assert a.shape == b.shape
    assert np.max(np.abs(a - b)) <= rtol * np.max(np.abs(b))


def _close_triplets(a, b, rtol):
    assert a.keys() == b.keys()
    keys = list(b)
    va = np.array([a[k] for k in keys])
    vb = np.array([b[k] for k in keys])
    assert np.max(np.abs(va - vb)) <= rtol * np.max(np.abs(vb))


def test_export_matches_oracle(tmp_path):
    m, tt = cases.channel(8, 4, seed=4, wall=meshgen.WALL)
    props = cases.ns_props(3, reynolds=500.0)
    rng = np.random.default_rng(7)
    g = fg.GpuMesh(props, m.vertices, m.elements, tt, m.wall_distance)
    try:
        W = cases.perturbed(g.get_state(0), g.n_basis, g.n_eqs, rng, 0.02)
        for which in (0, 1, 2):
            g.set_state(W, which)
        g.limiter()
        V1 = m.vertices + 1e-3 * (2 * rng.random(m.vertices.shape) - 1)
        written = optexport.export(g, tmp_path / "gpu", fg.FUNCTIONAL_LIFT, mode="allmass", perturbed_vertices=[V1],
                                   make_mesh=lambda v: fg.GpuMesh(props, v, m.elements, tt, m.wall_distance))
    finally:
        g.close()
    _oracle_files(tmp_path / "oracle", props, m, tt, W, V1)
    assert sorted(written) == sorted(os.listdir(tmp_path / "oracle"))
    gp, op = tmp_path / "gpu", tmp_path / "oracle"
    for name in ("I0.txt", "I1.txt", "R0.txt", "R1.txt"):
        _close_values(_values(gp / name), _values(op / name), 1e-12)
    _close_values(_values(gp / "dIdw.txt"), _values(op / "dIdw.txt"), 1e-6)  # exact against finite differences
    _close_triplets(_triplets(gp / "J.txt"), _triplets(op / "J.txt"), 1e-6)  # both finite differences
    for name in ("M0.txt", "M1.txt", "printMatrix.txt"):
        _close_triplets(_triplets(gp / name), _triplets(op / name), 1e-14)
