"""Host-side parts of the C-ABI library, no GPU needed: the library loads and exports
every entry point declared in include/flowgpu.h, and the integer set-up
(neighbour matrix, DOF ordering) is bit-exact against the reference's fixture and
the oracle's restatement of ElementOrdering.reverseCuthillMcKee."""
import os
import re

import numpy as np
import pytest

import flowpro_v2_b200 as fg
from flowpro_v2_b200 import meshgen
from oracle import oracle_ffi as of
from tests import cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "gamm_mesh.npz")


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "flowgpu.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(fp_[a-z0-9_]+)\s*\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    L = fg.lib()
    syms = header_symbols()
    assert len(syms) > 30
    for s in syms:
        assert hasattr(L, s), s
    # the Python binding covers the same set
    assert set(syms) == set(fg.exported_symbols())


@pytest.mark.parametrize("fixture", ["gamm_mesh.npz", "gammgen_mesh.npz"])
def test_neighbor_matrix_gamm_bit_exact(fixture):
    """The reference's own neighbors.txt of the two shipped example meshes (GAMM, 627
    triangles; GAMMgenerated, 1,600 triangles), from the library and from the oracle."""
    g = np.load(os.path.join(os.path.dirname(GOLDEN), fixture))
    tt = fg.create_neighbor_matrix(2, g["elements"], g["boundary"])
    assert np.array_equal(tt, g["neighbors"])
    assert np.array_equal(of.create_neighbor_matrix(3, g["elements"], g["boundary"]), g["neighbors"])


@pytest.mark.parametrize("nx,ny", [(12, 6), (40, 17)])
def test_neighbor_matrix_channel_matches_oracle(nx, ny):
    m = meshgen.bump_channel(nx=nx, ny=ny, seed=3)
    assert np.array_equal(fg.create_neighbor_matrix(2, m.elements, m.boundary),
                          of.create_neighbor_matrix(3, m.elements, m.boundary))


@pytest.mark.parametrize("mesh", ["gamm", "square", "channel"])
def test_rcm_ordering_matches_oracle(mesh):
    if mesh == "gamm":
        g = np.load(GOLDEN)
        v, el, tt = g["vertices"], g["elements"], g["neighbors"]
    elif mesh == "square":
        m = meshgen.square_mesh(8, 1.0, meshgen.INLET)
        v, el, tt = m.vertices, m.elements, of.create_neighbor_matrix(3, m.elements, m.boundary)
    else:
        m, tt = cases.channel(30, 11)
        v, el = m.vertices, m.elements
    order = fg.element_ordering(tt, rcm=True)
    o = of.Oracle(cases.euler_props(2), v, el, tt)
    rank = o.gindex()
    assert np.array_equal(np.argsort(rank), order)


def test_model_parameters_follow_aerodynamics_init():
    m, n = fg.model_from_properties(cases.ns_props(3, reynolds=5000.0))
    kap, pout = 1.4, 0.8430
    mach = np.sqrt(2 / (kap - 1) * ((1 / pout) ** ((kap - 1) / kap) - 1))
    rho_inf = 1 / (1 + (kap - 1) / 2 * mach ** 2) ** (1 / (kap - 1))
    p_inf = 1 / (1 + (kap - 1) / 2 * mach ** 2) ** (kap / (kap - 1))
    u_inf = mach * np.sqrt(kap * p_inf / rho_inf)
    assert m.model == fg.MODEL_NAVIER_STOKES and m.n_eqs == 4 and m.is_diffusive == 1
    assert abs(m.Re - 5000.0 / (rho_inf * u_inf)) < 1e-9 * m.Re
    assert abs(m.p_out - pout) < 1e-15 and n.order == 3 and n.beta0 == 2 and n.fd_step == 1e-8
    with pytest.raises(fg.FlowGpuError):
        fg.model_from_properties({"model": "KOmega", "dimension": 2})


def test_tetra_box_mesh_is_conforming_and_outward():
    """Kuhn-split box: the product's and the oracle's neighbour matrices agree, every
    element passes the oracle's geometry check (outward normals, faces summing to
    zero) and the volumes add up to the box minus the piecewise-linear bump."""
    m = meshgen.bump_box(nx=4, ny=3, nz=3, seed=2)
    tt = fg.create_neighbor_matrix(3, m.elements, m.boundary)
    assert np.array_equal(tt, of.create_neighbor_matrix(5, m.elements, m.boundary))
    assert np.count_nonzero(tt < 0) == m.boundary.shape[0]
    o = of.Oracle(cases.euler3_props(2), m.vertices, m.elements, tt)
    area, size, xs, ok = o.geometry()
    assert ok.all()
    assert np.all(area > 0)
    assert abs(area.sum() - (3.0 - 0.5 * 1.5 * 0.1)) < 1e-10


def test_adiabatic_eulers_parameters_and_initial_state():
    """AdiabaticEulers: dim + 1 equations, inviscid, and the constant initial state of
    AdiabaticEulers.constInitCondition (density and momentum, no energy)"""
    m = fg.model_from_properties(cases.adiabatic_props(2))[0]
    assert m.n_eqs == 3 and m.model == fg.MODEL_ADIABATIC_EULERS and m.is_diffusive == 0
    mesh, tt = cases.channel(6, 3)
    o = of.Oracle(cases.adiabatic_props(2), mesh.vertices, mesh.elements, tt)
    W = o.get_state(0)
    kapa, pOut = 1.4, 0.8430
    machIn = np.sqrt(2 / (kapa - 1) * ((1 / pOut) ** ((kapa - 1) / kapa) - 1))
    rhoIn = (1 + (kapa - 1) / 2 * machIn ** 2) ** (1 / (1 - kapa))
    VIn = machIn * np.sqrt(kapa * pOut / rhoIn)
    nb = o.n_basis
    assert abs(W[0, 0] - rhoIn) < 1e-14 and abs(W[0, nb] - rhoIn * VIn) < 1e-14 and abs(W[0, 2 * nb]) < 1e-14
    with pytest.raises(Exception):
        fg.model_from_properties(dict(cases.adiabatic_props(2), isInletSupersonic="true", pIn=1, rhoIn=1, vIn=2))


@pytest.mark.parametrize("fixture", ["gamm_mesh.npz", "gammgen_mesh.npz"])
def test_example_parameters_file_parses(fixture):
    """The examples' parameters.txt, as FlowPro reads it (one "key = value" per line, '%'
    comments, keys with empty values): AdiabaticEulers in 2D, kappa 1.4, pOut 0.737, order 2,
    BDF, penalty 1, dampTol 3."""
    g = np.load(os.path.join(os.path.dirname(GOLDEN), fixture))
    m, n = fg.model_from_properties(str(g["parameters"]))
    assert (m.model, m.dim, m.n_eqs, m.is_diffusive, m.inlet_supersonic) == (fg.MODEL_ADIABATIC_EULERS, 2, 3, 0, 0)
    assert (m.kappa, m.p_out, m.p_in0, m.rho_in0) == (1.4, 0.737, 1.0, 1.0)
    assert (n.order, n.implicit_time, n.penalty, n.damp_tol, n.element_ordering) == (2, 1, 1.0, 3.0, 1)


def test_wall_distance_matches_reference_file_gamm():
    """The GAMM example ships the wall distance the reference computed for it
    (simulations/examples/GAMM/mesh/wallDistance.txt, FlowProMain.generateDistanceFunction from
    the faces with code -1): fp_wall_distance and the oracle reproduce it bit for bit."""
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "gamm_mesh.npz"))
    V, E, N, ref = g["vertices"], g["elements"], g["neighbors"], g["wall_distance"]
    assert np.count_nonzero(ref == 0) > 0
    assert np.array_equal(fg.wall_distance(V, E, N, -1), ref)
    assert np.array_equal(of.wall_distance(V, E, N, -1), ref)


@pytest.mark.parametrize("mesh", ["naca", "channel"])
def test_wall_distance_matches_oracle_bit_exact(mesh):
    """fp_wall_distance (shortest edge paths) against the oracle's restatement of
    FlowProMain.generateDistanceFunction (Bellman-Ford sweeps): the same path sums."""
    if mesh == "naca":
        m = meshgen.naca0012_o_mesh(n_around=64, first_height=1e-3, growth=1.3, radius=20.0)
        tt, bc = fg.create_neighbor_matrix(2, m.elements, m.boundary), meshgen.WALL
    else:
        m, tt = cases.channel(20, 8, seed=3)
        bc = meshgen.INVISCID_WALL
    wp = fg.wall_distance(m.vertices, m.elements, tt, bc)
    wo = of.wall_distance(m.vertices, m.elements, tt, bc)
    assert np.array_equal(wp, wo)
    assert np.count_nonzero(wp == 0) > 0 and np.all(np.isfinite(wp))


def test_host_entry_points_report_bad_arguments():
    """The C ABI returns status codes for bad input instead of failing (no exceptions cross the
    ABI): out-of-range vertex indices, unsupported dimensions, null arrays."""
    m = meshgen.square_mesh(2, 1.0, meshgen.INLET)
    tt = fg.create_neighbor_matrix(2, m.elements, m.boundary)
    V = np.ascontiguousarray(m.vertices)
    bad = np.ascontiguousarray(m.elements, dtype=np.int32).copy()
    bad[0, 0] = V.shape[0]  # one past the last vertex
    out = np.zeros(V.shape[0])
    tt32 = np.ascontiguousarray(tt, dtype=np.int32)
    L = fg.lib()
    assert L.fp_wall_distance(2, V.shape[0], fg._dp(V), bad.shape[0], fg._ip(bad), fg._ip(tt32), -2,
                              fg._dp(out)) == fg.FP_ERR_ARG
    assert L.fp_wall_distance(4, V.shape[0], fg._dp(V), bad.shape[0], fg._ip(bad), fg._ip(tt32), -2,
                              fg._dp(out)) == fg.FP_ERR_ARG
    order = np.zeros(tt.shape[0], dtype=np.int32)
    assert L.fp_element_ordering(5, tt.shape[0], fg._ip(tt32), 1, fg._ip(order)) == fg.FP_ERR_ARG
    assert L.fp_element_ordering(2, tt.shape[0], None, 1, fg._ip(order)) == fg.FP_ERR_ARG
    el = np.ascontiguousarray(m.elements, dtype=np.int32)
    nb = np.zeros_like(tt32)
    assert L.fp_create_neighbor_matrix(7, el.shape[0], fg._ip(el), 0, None, fg._ip(nb)) == fg.FP_ERR_ARG
    with pytest.raises(fg.FlowGpuError) as e:
        fg.model_from_properties({"model": "KOmega", "dimension": 2})
    assert e.value.code != fg.FP_OK
