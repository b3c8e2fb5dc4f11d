"""Shared parity cases: FlowPro parameter sets, seeded meshes and states.

The parameter keys are FlowPro's (parameters.txt); the same dictionary configures
the CPU oracle and the GPU library.
"""
import numpy as np

from flowpro_v2_b200 import meshgen
from oracle import oracle_ffi


def euler_props(order, flux="default"):
    return dict(model="NavierStokes", dimension=2, kappa=1.4, cv=1, isFlowViscous="false", pIn0=1, rhoIn0=1,
                pOut=0.8430, order=order, penalty=0, dampTol=0, dampConst=0, numericalFlux=flux)


def ns_props(order, reynolds=5000.0, penalty=1.0):
    return dict(model="NavierStokes", dimension=2, kappa=1.4, cv=1, isFlowViscous="true", pIn0=1, rhoIn0=1,
                pOut=0.8430, reynolds=reynolds, prandtl=0.72, order=order, penalty=penalty, dampTol=0, dampConst=0)


def sa_props(order, penalty=1.0):
    return dict(model="SpalartAllmaras", dimension=2, kappa=1.4, cv=1, pIn0=1, rhoIn0=1, pOut=0.9395, reynolds=3e6,
                prandtl=0.72, attackAngle=0.0698131700797732, vtIn=3, sigma=0.6667, cb1=0.1355, cb2=0.622, ka=0.41,
                cw2=0.3, cw3=2, cv1=7.1, Prt=0.9, order=order, penalty=penalty, dampTol=0, dampConst=0)


def euler3_props(order):
    return dict(model="NavierStokes", dimension=3, kappa=1.4, cv=1, isFlowViscous="false", pIn0=1, rhoIn0=1,
                pOut=0.7840, order=order, penalty=0, dampTol=0, dampConst=0)


def ns3_props(order, reynolds=500.0, penalty=1.0):
    return dict(model="NavierStokes", dimension=3, kappa=1.4, cv=1, isFlowViscous="true", pIn0=1, rhoIn0=1,
                pOut=0.7840, reynolds=reynolds, prandtl=0.72, order=order, penalty=penalty, dampTol=0, dampConst=0)


def adiabatic_props(order, dimension=2):
    return dict(model="AdiabaticEulers", dimension=dimension, kappa=1.4, cv=1, pIn0=1, rhoIn0=1, pOut=0.8430,
                order=order, penalty=0, dampTol=0, dampConst=0)


def scalar_props(order, k=0.0):
    p = dict(model="TestScalarEquation", dimension=2, a="1, 0.5", order=order, penalty=0, dampTol=0, dampConst=0,
             timeMethod="BDF", timeOrder=1, dt=1e8, iterativeSolverTol=1e-13, newtonIters=1, preconditioner="ilu0")
    if k > 0:
        p["k"] = k
    return p


def channel(nx=12, ny=6, seed=1, wall=meshgen.INVISCID_WALL):
    m = meshgen.bump_channel(nx=nx, ny=ny, seed=seed, wall=wall)
    tt = oracle_ffi.create_neighbor_matrix(3, m.elements, m.boundary)
    return m, tt


def box(nx=4, ny=3, nz=3, seed=2, wall=meshgen.INVISCID_WALL):
    m = meshgen.bump_box(nx=nx, ny=ny, nz=nz, seed=seed, wall=wall)
    tt = oracle_ffi.create_neighbor_matrix(5, m.elements, m.boundary)
    return m, tt


def free_stream(n_elem, n_basis, w0):
    W = np.zeros((n_elem, len(w0) * n_basis))
    for m, v in enumerate(w0):
        W[:, m * n_basis:(m + 1) * n_basis] = v
    return W


def perturbed(W, n_basis, n_eqs, rng, amp=0.01):
    """free-stream state with seeded relative noise on every coefficient."""
    noise = 1.0 + amp * (2 * rng.random(W.shape) - 1)
    return W * noise + amp * 0.1 * (2 * rng.random(W.shape) - 1)


def rel_err_per_component(a, b, n_basis, n_eqs):
    """max_e,j |a - b| / max_e,j |b| per equation m (normwise per component)."""
    a = a.reshape(-1, n_eqs, n_basis)
    b = b.reshape(-1, n_eqs, n_basis)
    out = []
    for m in range(n_eqs):
        den = np.max(np.abs(b[:, m, :]))
        out.append(np.max(np.abs(a[:, m, :] - b[:, m, :])) / (den if den > 0 else 1.0))
    return np.array(out)
