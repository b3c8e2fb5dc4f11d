"""The oracle's operation-counting build (oracle/oracle_flops.cpp, flop_real.hpp): the same
arithmetic as the plain build, so its residual is bit-identical (the counts belong to the same
algorithm), the counters reset between evaluations, and the committed counts of the bench
workloads (tests/golden/residual_flops.json, tests/golden/make_flops.py) describe the bench's
meshes."""
import json
import os

import numpy as np

import bench
from flowpro_v2_b200 import meshgen
from oracle import oracle_ffi as of
from tests import cases

HERE = os.path.dirname(os.path.abspath(__file__))


def _check(props, m, tt, W, wd=None):
    o = of.Oracle(props, m.vertices, m.elements, tt, wd)
    o.set_state(W)
    o.limiter()
    R = o.residual()
    c1 = of.count_residual_flops(props, m.vertices, m.elements, tt, W, wd)
    c2 = of.count_residual_flops(props, m.vertices, m.elements, tt, W, wd)
    assert np.array_equal(c1["residual"], R)
    assert c1["phases"] == c2["phases"] and c1["flops"] == c2["flops"] > 0
    return c1


def test_counting_build_ns2_p2():
    m = meshgen.bump_channel(nx=12, ny=5, seed=1, wall=meshgen.WALL)
    tt = of.create_neighbor_matrix(3, m.elements, m.boundary)
    o = of.Oracle(bench.PROPS, m.vertices, m.elements, tt)
    W = bench.initial_state(o.n_elem, o.n_basis, o.get_state(0)[0][::o.n_basis])
    c = _check(bench.PROPS, m, tt, W)
    ph = c["phases"]
    assert ph["interior_faces"]["mul"] > 0 and ph["boundary_faces"]["mul"] > 0 and ph["volume"]["mul"] > 0


def test_counting_build_euler3_p2():
    m, tt = cases.box(3, 2, 2, seed=4)
    props = cases.euler3_props(3)
    o = of.Oracle(props, m.vertices, m.elements, tt, m.wall_distance)
    rng = np.random.default_rng(1)
    W = o.get_state(0) + 1e-3 * (2 * rng.random((o.n_elem, o.nb)) - 1)
    _check(props, m, tt, W, m.wall_distance)


def test_committed_counts_match_bench_workloads():
    d = json.load(open(os.path.join(HERE, "golden", "residual_flops.json")))
    c2 = d["ns2_p2"]
    assert c2["workload"] == bench.WORKLOAD and c2["elements"] == 2 * bench.NX * bench.NY
    assert 3000 < c2["flops"] / c2["elements"] < 20000
    c3 = d["euler3_p2"]
    assert c3["elements"] == 6 * 100 * 34 * 34
    assert c3["units"]["elements"] == c3["elements"]


def test_committed_2d_count_reproduces():
    """the bench workload's committed count is what the counting build gives today"""
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_flops
    d = json.load(open(os.path.join(HERE, "golden", "residual_flops.json")))
    c = make_flops.count_2d()
    assert c["flops"] == d["ns2_p2"]["flops"] and c["phases"] == d["ns2_p2"]["phases"]
