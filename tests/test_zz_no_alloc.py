"""fp_l2_norms_noalloc: the residual norms for callers that cannot allocate device memory
themselves (their device buffers come from a pool or arena they do not control, e.g. a Java
host passing device pointers through FFM/JNI).  The entry point takes caller-owned device
arrays only and keeps its scratch in a fixed file-scope device array.

Checked through the C ABI against the context-based entry point fp_residuum_norms on the
same residual, 1e-12 relative, on two calls in a row (the second call reuses the scratch
the first one left behind).  This file is collected last so that a run stopping at the first
failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

import flowpro_v2_b200 as fg
from oracle import oracle_ffi as of
from tests import cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["channel_p2", "channel_p2_many_blocks", "box_p2_3d"])
def test_l2_norms_noalloc_matches_context_entry_point(kind):
    """one thread block (168 triangles), many blocks (2,400 triangles: the final sum runs over
    several blocks' partials) and 3D p = 2 (10 basis functions, the largest supported)"""
    import torch

    if kind == "channel_p2":
        m, tt = cases.channel(14, 6, seed=12)
        props = cases.euler_props(3)
    elif kind == "channel_p2_many_blocks":
        m, tt = cases.channel(60, 20, seed=12)
        props = cases.euler_props(3)
    else:
        m, tt = cases.box(8, 3, 3, seed=12)
        props = cases.euler3_props(3)
    g = fg.GpuMesh(props, m.vertices, m.elements, tt, m.wall_distance)
    o = of.Oracle(props, m.vertices, m.elements, tt, m.wall_distance)
    rng = np.random.default_rng(3)
    W = cases.perturbed(g.get_state(0), g.n_basis, g.n_eqs, rng, 0.05)
    g.set_state(W)
    g.limiter()
    R = g.residuum()                      # resident residual, element-major on the host
    ref = g.residuum_norms()              # context-based entry point
    mass = o.mass_matrices()              # Element.M of every element (reference storage)
    torch.cuda.set_device(0)
    r_d = torch.from_numpy(np.ascontiguousarray(R)).cuda()
    m_d = torch.from_numpy(np.ascontiguousarray(mass)).cuda()
    stream = torch.cuda.current_stream()
    for _ in range(2):
        out = torch.full((g.n_eqs,), float("nan"), dtype=torch.float64, device="cuda")
        rc = fg.lib().fp_l2_norms_noalloc(g.n_elem, g.n_basis, g.n_eqs, ctypes.c_void_p(r_d.data_ptr()),
                                          ctypes.c_void_p(m_d.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                          stream.cuda_stream)
        assert rc == fg.FP_OK
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.abs(got - ref) <= 1e-12 * np.abs(ref)), (got, ref)


def test_l2_norms_noalloc_rejects_oversized_input():
    big = 4096 * 256 + 1
    rc = fg.lib().fp_l2_norms_noalloc(big, 3, 4, ctypes.c_void_p(8), ctypes.c_void_p(8), ctypes.c_void_p(8), 0)
    assert rc == fg.FP_ERR_ARG
