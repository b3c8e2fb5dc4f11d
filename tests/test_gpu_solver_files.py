"""Solver files of the device loops (fp_solver_output) against the reference's formats and
semantics: residuum.txt rows (MasterSolver.appendResiduum, MasterSolver.java:94-111), state.txt
(State.save, State.java:113-136), W.txt / We.txt / artificialViscosity.txt (saveData,
LocalImplicitSolver.java:326-344) and the STOP file (MasterSolver.isStopRequested,
MasterSolver.java:60-67)."""
import os

import numpy as np
import pytest

import flowpro_v2_b200 as fg
from tests import cases

pytestmark = pytest.mark.gpu


def _case():
    m, tt = cases.channel(10, 5, seed=4)
    g = fg.GpuMesh(cases.euler_props(2), m.vertices, m.elements, tt, m.wall_distance)
    return g


def _rows(path):
    with open(path) as f:
        return [[float(v.replace("E", "e")) for v in line.split()] for line in f if line.strip()]


def _props(path):
    out = {}
    with open(path) as f:
        for line in f:
            if line.startswith("#") or "=" not in line:
                continue
            k, v = line.rstrip("\n").split("=", 1)
            out[k] = v
    return out


def test_implicit_solver_files(tmp_path):
    g = _case()
    d = str(tmp_path)
    with open(os.path.join(d, "residuum.txt"), "w") as f:
        f.write("stale row\n")
    g.solver_output(d, save_rate=2)
    out = fg.GpuImplicitSolver(g, steps=7, cfl=5.0, vary_cfl=1, max_cfl=100, linear_tol=1e-3, restart=30,
                               max_restarts=5, preconditioner="blockjacobi").solve()
    assert out[4] == 7
    res = _rows(os.path.join(d, "residuum.txt"))
    assert len(res) == 7 and all(len(r) == 3 + g.n_eqs for r in res)
    assert res[-1][0] == out[1] and res[-1][1] == out[0]
    assert all(b[1] > a[1] for a, b in zip(res, res[1:]))  # time grows
    assert all(r[0] == max(r[3:]) for r in res)  # residuum = max of the equations' relative residua
    We = np.array(_rows(os.path.join(d, "We.txt")))
    assert np.array_equal(We, g.get_state(0))  # Java's shortest digits read back exactly
    _, bw = g.mass_matrices()
    Wavg = np.array(_rows(os.path.join(d, "W.txt")))
    ref = (g.get_state(0).reshape(g.n_elem, g.n_eqs, g.n_basis) * bw[:, None, :]).sum(axis=2)
    assert np.max(np.abs(Wavg - ref)) <= 1e-13 * np.max(np.abs(ref))
    st = _props(os.path.join(d, "state.txt"))
    assert int(st["steps"]) == 7 and float(st["t"].replace("E", "e")) == out[0]
    assert float(st["residuum"].replace("E", "e")) == out[1] and float(st["CFL"].replace("E", "e")) == out[2]
    assert len(st["residuumNormalisation"].split(",")) == g.n_eqs and int(st["order"]) == 2
    av = np.array(_rows(os.path.join(d, "artificialViscosity.txt")))
    assert av.shape == (g.n_elem, g.n_eqs)
    # STOP: the loop ends after the step in which it is seen, and the file is removed
    open(os.path.join(d, "STOP"), "w").close()
    g.solver_output(d, save_rate=0, append=True)
    out2 = fg.GpuImplicitSolver(g, steps=10, cfl=5.0, vary_cfl=1, max_cfl=100, linear_tol=1e-3, restart=30,
                                max_restarts=5, preconditioner="blockjacobi").solve()
    assert out2[4] == 1 and not os.path.exists(os.path.join(d, "STOP"))
    assert len(_rows(os.path.join(d, "residuum.txt"))) == 8
    g.solver_output(None)
    g.close()


def test_explicit_solver_files(tmp_path):
    g = _case()
    d = str(tmp_path)
    g.solver_output(d, save_rate=3)
    out = fg.GpuExplicitSolver(g, steps=5, cfl=0.5).solve()
    res = _rows(os.path.join(d, "residuum.txt"))
    assert len(res) == 5 and res[-1][0] == out[1] and res[-1][1] == out[0]
    assert np.array_equal(np.array(_rows(os.path.join(d, "We.txt"))), g.get_state(0))
    assert int(_props(os.path.join(d, "state.txt"))["steps"]) == 5
    g.close()
