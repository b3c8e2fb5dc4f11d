"""Failure paths of the device solver loop, injected on the host (no GPU fault): the
reference's retry semantics of LocalImplicitSolver.solve (LocalImplicitSolver.java:177-225):
a linear solve that fails restores W from Wo (copyWo2W), reduces the CFL number by 1.5 (or
halves a fixed time step, State.reduceCFL, State.java:222-228) and repeats the step; the run
ends when the reduction is hopeless (CFL < CFL0 / 20, dt < dt0 / 1024; State.java:234-240) or
when the residuum is not a number (the loop condition residuum > target fails)."""
import numpy as np
import pytest

import flowpro_v2_b200 as fg
from tests import cases

pytestmark = pytest.mark.gpu


def _case(seed=5):
    m, tt = cases.channel(10, 5, seed=seed)
    g = fg.GpuMesh(cases.euler_props(2), m.vertices, m.elements, tt, m.wall_distance)
    rng = np.random.default_rng(seed)
    W = cases.perturbed(g.get_state(0), g.n_basis, g.n_eqs, rng, 0.01)
    for which in (0, 1, 2):
        g.set_state(W, which)
    return g, W


@pytest.mark.parametrize("prec", ["blockjacobi", "blockilu0"])
def test_gmres_failure_reduces_cfl_until_hopeless(prec):
    g, W0 = _case()
    cfl = 8.0
    # one GMRES iteration to a tolerance no iterate reaches: every linear solve fails
    out = fg.GpuImplicitSolver(g, steps=5, cfl=cfl, vary_cfl=1, max_cfl=100, linear_tol=1e-30, restart=1,
                               max_restarts=1, preconditioner=prec).solve()
    k = 8  # first k with cfl / 1.5^k < cfl / 20
    assert out[4] == 0  # no step finished
    assert out[2] == pytest.approx(cfl / 1.5 ** k, rel=1e-15)
    assert out[5] == k and out[6] == k  # k Newton iterations of one GMRES iteration each
    assert np.array_equal(g.get_state(0), W0)  # W restored from Wo after every failure
    g.close()


def test_gmres_failure_halves_fixed_time_step():
    g, W0 = _case()
    dt0 = 0.01
    out = fg.GpuImplicitSolver(g, steps=5, dt=dt0, linear_tol=1e-30, restart=1, max_restarts=1,
                               preconditioner="blockjacobi").solve()
    assert out[4] == 0
    assert out[3] == dt0 / 2 ** 11  # first halving below dt0 / 1024
    assert out[5] == 11
    assert np.array_equal(g.get_state(0), W0)
    g.close()


@pytest.mark.parametrize("prec", ["blockjacobi", "blockilu0"])
def test_nan_state_is_rejected_and_restored(prec):
    g, W0 = _case()
    Wbad = W0.copy()
    Wbad[7, 0] = np.nan
    g.set_state(Wbad, 0)  # Wo stays the clean state
    g.limiter()
    # the linear solver reports the singular (non-finite) block instead of solving
    asm = fg.JacobiAssembler(g)
    asm.assemble(0.01, -1)
    ok, _ = fg.LinearSolver(g, prec, tol=1e-6).solve()
    assert not ok
    out = fg.GpuImplicitSolver(g, steps=5, cfl=5.0, vary_cfl=1, max_cfl=100, linear_tol=1e-3, restart=30,
                               max_restarts=5, preconditioner=prec).solve()
    assert np.isnan(out[1]) and out[4] == 0
    assert out[2] == pytest.approx(5.0 / 1.5, rel=1e-15)  # one reduction, then the NaN residuum ends the loop
    assert np.array_equal(g.get_state(0), W0)  # copyWo2W restored the last good state
    g.close()
