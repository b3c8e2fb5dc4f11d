"""Block ILU(0) preconditioner of the matrix-free path and its failure handling (GPU).

* fp_assemble_preconditioner writes the exact element blocks straight into the factor
  storage and factorises them in place (FP32: the factorisation runs in FP32; no copy of the
  operator's blocks).  The same blocks gathered from fp_assemble_exact give bit-identical
  factors, so the two routes must give the same GMRES iterates (BlockILU0.java:98-185 is the
  factorisation both follow).
* The application with the factor blocks staged in shared memory by bulk asynchronous copies
  (the default) and the one with register-resident factor entries: the same preconditioner to
  rounding; the staged kernel gives identical values for any number of elements in flight.
* A dependency wait of the persistent ILU kernels that runs out sets a status word; the host
  reports FP_ERR_TIMEOUT and clears the words, and the next factorisation and solve on the same
  context succeed.  The test makes the waits run out by giving them a poll limit of zero (no
  fault, no hang: every wait returns at once).
"""
import numpy as np
import pytest

import flowpro_v2_b200 as fg
from tests import cases

pytestmark = pytest.mark.gpu


def _mesh(seed=3, two_d=False):
    if two_d:  # 2D Euler p=1: 12 unknowns per element, up to 16 elements in flight per block
        props = cases.euler_props(2)
        m, tt = cases.channel(16, 8, seed=seed)
    else:  # 3D Euler p=2: 50 unknowns per element, up to 4 in flight
        props = cases.euler3_props(3)
        m, tt = cases.box(4, 3, 2, seed=seed)
    g = fg.GpuMesh(props, m.vertices, m.elements, tt, m.wall_distance)
    rng = np.random.default_rng(seed)
    W = cases.perturbed(g.get_state(0), g.n_basis, g.n_eqs, rng, 0.02)
    for which in (0, 1, 2):
        g.set_state(W, which)
    g.limiter()
    return g


def _solve(g, precision, direct, dt):
    asm = fg.JacobiAssembler(g, bdf_order=1)
    if direct:
        asm.assemble_preconditioner(dt, -1, "blockilu0", precision)
    else:
        asm.assemble_exact(dt, -1)
    ls = fg.LinearSolver(g, "blockilu0", precision=precision, jacobian=fg.JAC_MATRIXFREE, restart=30, max_restarts=5,
                         tol=1e-10)
    ok, x = ls.solve()
    return ok, x, ls.iterations


@pytest.mark.parametrize("precision", [fg.FP64, fg.FP32])
def test_direct_preconditioner_equals_gathered(precision):
    g1, g2 = _mesh(), _mesh()
    dt = 10.0 * g1.time_step_bound()
    ok1, x1, it1 = _solve(g1, precision, False, dt)
    ok2, x2, it2 = _solve(g2, precision, True, dt)
    assert ok1 and ok2
    assert it1 == it2
    assert np.array_equal(x1, x2)
    # the FP32 factorisation under FP64 GMRES reaches the FP64 solution of the same system
    g3 = _mesh()
    ok3, x3, _ = _solve(g3, fg.FP64, True, dt)
    assert ok3
    assert np.max(np.abs(x2 - x3)) <= 1e-8 * np.max(np.abs(x3))
    for g in (g1, g2, g3):
        g.close()


def test_direct_preconditioner_keeps_no_operator_blocks():
    g = _mesh()
    dt = 10.0 * g.time_step_bound()
    fg.JacobiAssembler(g).assemble_preconditioner(dt, -1, "blockilu0", fg.FP32)
    with pytest.raises(fg.FlowGpuError):
        fg.LinearSolver(g, "blockilu0", precision=fg.FP32, jacobian=fg.JAC_ASSEMBLED).solve()
    with pytest.raises(fg.FlowGpuError):
        fg.JacobiAssembler(g).blocks()
    g.close()


@pytest.mark.parametrize("precision", [fg.FP64, fg.FP32])
def test_ilu_wait_timeout_is_reported_and_recovers(precision):
    g = _mesh()
    dt = 10.0 * g.time_step_bound()
    ok, x_ref, _ = _solve(g, precision, True, dt)
    assert ok
    # factorisation waits run out
    g.set_wait_limit(0)
    with pytest.raises(fg.FlowGpuError) as ei:
        fg.JacobiAssembler(g).assemble_preconditioner(dt, -1, "blockilu0", precision)
    assert "flowgpu error 8" in str(ei.value)  # FP_ERR_TIMEOUT
    g.set_wait_limit(1 << 19)
    ok, x, _ = _solve(g, precision, True, dt)
    assert ok and np.array_equal(x, x_ref)
    # sweep waits run out (factorised with the normal limit first)
    fg.JacobiAssembler(g).assemble_preconditioner(dt, -1, "blockilu0", precision)
    g.set_wait_limit(0)
    ls = fg.LinearSolver(g, "blockilu0", precision=precision, jacobian=fg.JAC_MATRIXFREE, restart=30, max_restarts=5,
                         tol=1e-10)
    with pytest.raises(fg.FlowGpuError) as ei:
        ls.solve()
    assert "flowgpu error 8" in str(ei.value)
    g.set_wait_limit(1 << 19)
    ok, x, _ = _solve(g, precision, True, dt)
    assert ok and np.array_equal(x, x_ref)
    g.close()


@pytest.mark.parametrize("two_d", [False, True])
@pytest.mark.parametrize("precision", [fg.FP64, fg.FP32])
def test_bulk_copy_sweeps_match_register_sweeps(precision, two_d):
    """the staged kernel splits each row over fewer lanes than the register kernel: the same
    preconditioner to rounding, so GMRES needs the same iterations (+-1) and reaches the same
    solution; and its results do not depend on the number of elements in flight per block
    (every group count the block size and the slots allow: 1, 2 for 50 unknowns per element
    (two FP64 slots of five 20 KB blocks), up to 16 for 12); a group count above the limit is
    refused"""
    variants = (2, 3, 4, 5, 6) if two_d else (2, 3)
    gs = [_mesh(two_d=two_d) for _ in range(2 + len(variants))]
    gs[1].set_ilu_sweep(1)
    for g, v in zip(gs[2:], variants):
        g.set_ilu_sweep(v)
    dt = 10.0 * gs[0].time_step_bound()
    res = [_solve(g, precision, True, dt) for g in gs]
    assert all(r[0] for r in res)
    (_, x0, it0), (_, x1, it1) = res[0], res[1]
    assert abs(it0 - it1) <= 1
    assert np.max(np.abs(x0 - x1)) <= 1e-9 * np.max(np.abs(x1))
    for _, x, it in res[2:]:
        assert it == it0 and np.array_equal(x, x0)
    for g in gs:
        g.close()
    if not two_d:
        g = _mesh()
        g.set_ilu_sweep(5)  # 8 groups of 64 threads: too few for 50 rows of 2 lanes
        with pytest.raises(fg.FlowGpuError):
            _solve(g, precision, True, dt)
        g.close()
