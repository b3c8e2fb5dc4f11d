"""The optimisation-toolbox export (OptimisationToolExport.java): Java's number format and the
file layouts, written from the oracle's values (CPU)."""
import numpy as np
import pytest

from flowpro_v2_b200 import meshgen, optexport
from oracle import oracle_ffi as of
from tests import cases

# Double.toString outputs (java.lang.Double's documented format: decimal notation for
# 1e-3 <= |x| < 1e7, computerized scientific notation otherwise, shortest digits)
JAVA_STRINGS = [
    (1.0, "1.0"), (100.0, "100.0"), (0.001, "0.001"), (0.0001, "1.0E-4"), (1e7, "1.0E7"),
    (9999999.0, "9999999.0"), (12345678.9, "1.23456789E7"), (-0.5, "-0.5"), (0.1, "0.1"),
    (1.0 / 3.0, "0.3333333333333333"), (2.0 / 3.0, "0.6666666666666666"), (1e21, "1.0E21"),
    (1.5e-7, "1.5E-7"), (4.9e-324, "4.9E-324"), (1.7976931348623157e308, "1.7976931348623157E308"),
    (0.0, "0.0"), (-0.0, "-0.0"), (123456.789, "123456.789"), (0.00099, "9.9E-4"), (-2.5e-10, "-2.5E-10"),
    (1234567.0, "1234567.0"), (0.0123, "0.0123"), (float("nan"), "NaN"), (float("inf"), "Infinity"),
    (float("-inf"), "-Infinity"),
]


@pytest.mark.parametrize("x,s", JAVA_STRINGS)
def test_java_double_format(x, s):
    assert optexport.java_double(x) == s


def test_java_double_reads_back_exactly():
    rng = np.random.default_rng(3)
    xs = np.concatenate([rng.standard_normal(2000) * 10.0 ** rng.integers(-12, 12, 2000),
                         rng.random(200) * 1e-3, rng.random(200) * 1e7])
    for x in xs:
        assert float(optexport.java_double(x).replace("E", "e")) == x


def _triplets(path):
    d = {}
    with open(path) as f:
        for line in f:
            a, b, v = line.split()
            d[(int(a), int(b))] = float(v.replace("E", "e"))
    return d


def _values(path):
    with open(path) as f:
        lines = f.read().splitlines()
    assert all(l.endswith(" ") for l in lines)
    return np.array([float(l.strip().replace("E", "e")) for l in lines])


def oracle_export_values(props, m, tt, seed=7):
    o = of.Oracle(props, m.vertices, m.elements, tt, m.wall_distance)
    rng = np.random.default_rng(seed)
    W = cases.perturbed(o.get_state(0), o.n_basis, o.n_eqs, rng, 0.02)
    for which in (0, 1, 2):
        o.set_state(W, which)
    o.limiter()
    I, dIdw = o.functional(0)
    o.assemble(0.0, 0.0)  # steady operator (Element.exportLocalJacobiMatrix)
    diag, neigh, rhs = o.blocks()
    return dict(o=o, W=W, I=I, dIdw=dIdw, diag=diag, neigh=neigh, rhs=rhs, R=o.residual(), M=o.mass_matrices(),
                Is=o.basis_weights(), gpos=o.gindex())


def test_export_layouts_from_oracle_values(tmp_path):
    m, tt = cases.channel(8, 4, seed=4, wall=meshgen.WALL)
    v = oracle_export_values(cases.ns_props(3, reynolds=500.0), m, tt)
    o = v["o"]
    n, nb, ne = o.nb, o.n_basis, o.n_eqs
    # the steady RHS is the residual (Element.exportLocalR)
    assert np.array_equal(v["rhs"], v["R"])
    optexport.write_functional(tmp_path, 0, v["I"])
    optexport.write_residual(tmp_path, 0, v["R"])
    optexport.write_functional_derivative(tmp_path, v["dIdw"])
    optexport.write_jacobian(tmp_path, v["diag"], v["neigh"], tt, v["gpos"])
    optexport.write_mass(tmp_path, 0, v["M"], v["gpos"], ne)
    optexport.write_print_matrix(tmp_path, v["Is"], v["gpos"], ne)
    assert np.array_equal(_values(tmp_path / "I0.txt"), [v["I"]])
    assert np.array_equal(_values(tmp_path / "R0.txt"), v["R"].reshape(-1))
    assert np.array_equal(_values(tmp_path / "dIdw.txt"), v["dIdw"].reshape(-1))
    g = v["gpos"][:, None] * n + np.arange(n)[None, :]
    J = _triplets(tmp_path / "J.txt")
    n_interior = int(np.sum(tt > -1))
    assert len(J) == m.elements.shape[0] * n * n + n_interior * n * n
    for k in range(m.elements.shape[0]):
        for i in range(n):
            for j in range(n):
                assert J[(g[k, i], g[k, j])] == v["diag"][k, j, i]
        for face in range(tt.shape[1]):
            r = tt[k, face]
            if r > -1:
                for i in range(n):
                    for j in range(n):
                        assert J[(g[k, i], g[r, j])] == v["neigh"][k, face, j, i]
    M = _triplets(tmp_path / "M0.txt")
    assert len(M) == m.elements.shape[0] * ne * nb * nb
    for k in range(m.elements.shape[0]):
        for q in range(ne):
            for i in range(nb):
                for j in range(nb):
                    assert M[(g[k, nb * q + i], g[k, nb * q + j])] == v["M"][k, i, j]
    P = _triplets(tmp_path / "printMatrix.txt")
    for k in range(m.elements.shape[0]):
        for i in range(nb):
            for q in range(ne):
                assert P[(k * ne + q, g[k, q * nb + i])] == v["Is"][k, i]
    # the basis weights are the means of the basis functions (they sum to one)
    assert np.allclose(v["Is"].sum(axis=1), 1.0, rtol=0, atol=1e-13)
