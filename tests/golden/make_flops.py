"""Count the algorithmic FP64 operations of one residual evaluation of the bench workloads with
the oracle's counting build (oracle/oracle_flops.cpp) and write tests/golden/residual_flops.json.

The count is that of the restated reference algorithm (DGpure.residuum with residuumWall,
DGpure.java:108-356) at the bench's state, with every interior face counted once (the
reference evaluates it from both sides with the same operations) and operations with an exact
zero operand left out (oracle_ffi.count_residual_flops).  bench.py divides it by the measured
pass time for the FP64 side of the residual roofline.

usage: python tests/golden/make_flops.py [--quick]   (--quick: the 2D case only)
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

import bench  # noqa: E402
from flowpro_v2_b200 import meshgen  # noqa: E402
from oracle import oracle_ffi as of  # noqa: E402

OUT = os.path.join(HERE, "residual_flops.json")


def count_2d():
    m = meshgen.bump_channel(nx=bench.NX, ny=bench.NY, seed=1, wall=meshgen.WALL)
    tt = of.create_neighbor_matrix(3, m.elements, m.boundary)
    o = of.Oracle(bench.PROPS, m.vertices, m.elements, tt)
    W = bench.initial_state(o.n_elem, o.n_basis, o.get_state(0)[0][::o.n_basis])
    del o
    c = of.count_residual_flops(bench.PROPS, m.vertices, m.elements, tt, W)
    return {"workload": bench.WORKLOAD, "elements": int(m.elements.shape[0]), "props": bench.PROPS,
            "state": "bench.initial_state (free stream, 1% seeded density noise), limiter applied",
            "flops": c["flops"], "phases": c["phases"]}


def _generic(W, seed=3):
    """the free stream with seeded noise of 1e-3 on every coefficient: no exact zero of the
    state (the free stream's transverse momenta) makes operations trivial in some elements
    and not in others"""
    import numpy as np
    rng = np.random.default_rng(seed)
    return W + 1e-3 * (2 * rng.random(W.shape) - 1)


def _units(tt):
    """elements, interior face sides (each interior face appears twice) and boundary faces"""
    inner = int((tt > -1).sum())
    return tt.shape[0], inner, int(tt.size - inner)


def count_3d(box=(100, 34, 34), samples=((30, 10, 10), (50, 17, 17))):
    """The full box's residual would need more host memory than the oracle's per-element
    structures allow, so the operations are counted on smaller boxes of the same construction
    and a generic state, per element, per interior face side and per boundary face, and the
    full box's count is the largest sample's per-unit counts times its units.  Elements and
    faces near the box's walls have axis-aligned geometry whose exact zeros make some products
    trivial, so the per-unit counts grow slightly with the box (the samples' figures are
    recorded): the scaled figure is a lower bound of the full box's."""
    per, rec = None, []
    for b in samples:
        m = meshgen.bump_box(*b, seed=1)
        tt = of.create_neighbor_matrix(5, m.elements, m.boundary)
        o = of.Oracle(bench.SOLVE_PROPS, m.vertices, m.elements, tt, m.wall_distance)
        W = _generic(o.get_state(0))
        del o
        c = of.count_residual_flops(bench.SOLVE_PROPS, m.vertices, m.elements, tt, W, m.wall_distance)
        ne, ni, nb = _units(tt)
        ops = lambda d: d["add"] + d["mul"] + d["div"] + d["sqrt"]  # noqa: E731
        per = (ops(c["phases"]["volume"]) / ne, ops(c["phases"]["interior_faces"]) / ni,
               ops(c["phases"]["boundary_faces"]) / nb)
        rec.append({"box": list(b), "elements": ne, "per_element": per[0], "per_interior_face_side": per[1],
                    "per_boundary_face": per[2], "phases": c["phases"]})
        print("  sample", b, per, flush=True)
    m = meshgen.bump_box(*box, seed=1)
    from flowpro_v2_b200 import create_neighbor_matrix
    tt = create_neighbor_matrix(3, m.elements, m.boundary)
    ne, ni, nb = _units(tt)
    flops = per[0] * ne + per[1] * ni / 2 + per[2] * nb
    return {"workload": f"3D Euler DG p=2 residual, bump box {box[0]}x{box[1]}x{box[2]}x6 tetrahedra",
            "elements": ne, "props": bench.SOLVE_PROPS,
            "state": "free stream + 1e-3 seeded noise on every coefficient",
            "flops": int(round(flops)), "scaled_from": samples[-1],
            "units": {"elements": ne, "interior_faces": ni // 2, "boundary_faces": nb}, "samples": rec}


def main(quick=False):
    out = {"what": "non-trivial FP64 +, -, *, /, sqrt of one residual evaluation of the restated reference "
                   "algorithm, each interior face once (tests/golden/make_flops.py)"}
    t = time.time()
    out["ns2_p2"] = count_2d()
    print("2D", out["ns2_p2"]["flops"], time.time() - t, flush=True)
    if not quick:
        t = time.time()
        out["euler3_p2"] = count_3d()
        print("3D", out["euler3_p2"]["flops"], time.time() - t, flush=True)
    elif os.path.exists(OUT):
        old = json.load(open(OUT))
        if "euler3_p2" in old:
            out["euler3_p2"] = old["euler3_p2"]
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print(OUT)


if __name__ == "__main__":
    main("--quick" in sys.argv)
