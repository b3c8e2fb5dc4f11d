"""Generate the committed golden fixtures from the FlowPro checkout.

gamm_mesh.npz: the shipped example mesh FlowPro/simulations/examples/GAMM/mesh
(627 triangles): vertices, elements, boundaryType rows and the reference's own
neighbors.txt (the output of FlowProMain.createNeighborMatrix, FlowProMain.java:772-873),
used to pin the neighbour-matrix construction bit-exactly, and its wallDistance.txt
(FlowProMain.generateDistanceFunction, FlowProMain.java:962-1018).
gammgen_mesh.npz: the second shipped example, FlowPro/simulations/examples/GAMMgenerated/mesh
(1,600 triangles), with its neighbors.txt.
Both also hold the example's default/parameters.txt as text (the case set-up a user hands to
fp_model_from_properties).

usage: python tests/golden/make_golden.py /path/to/FlowPro_v2
"""
import os
import sys

import numpy as np


def main(ref):
    g = os.path.join(ref, "FlowPro", "simulations", "examples", "GAMM", "mesh")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "gamm_mesh.npz")
    np.savez_compressed(out,
                        vertices=np.loadtxt(os.path.join(g, "vertices.txt")),
                        elements=np.loadtxt(os.path.join(g, "elements.txt"), dtype=np.int32),
                        boundary=np.loadtxt(os.path.join(g, "boundaryType.txt"), dtype=np.int32),
                        neighbors=np.loadtxt(os.path.join(g, "neighbors.txt"), dtype=np.int32),
                        wall_distance=np.loadtxt(os.path.join(g, "wallDistance.txt")),
                        parameters=np.array(open(os.path.join(g, "..", "default", "parameters.txt")).read()))
    print(out)
    g = os.path.join(ref, "FlowPro", "simulations", "examples", "GAMMgenerated", "mesh")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "gammgen_mesh.npz")
    np.savez_compressed(out,
                        vertices=np.loadtxt(os.path.join(g, "vertices.txt")),
                        elements=np.loadtxt(os.path.join(g, "elements.txt"), dtype=np.int32),
                        boundary=np.loadtxt(os.path.join(g, "boundaryType.txt"), dtype=np.int32),
                        neighbors=np.loadtxt(os.path.join(g, "neighbors.txt"), dtype=np.int32),
                        parameters=np.array(open(os.path.join(g, "..", "default", "parameters.txt")).read()))
    print(out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the FlowPro_v2 checkout>")
    main(sys.argv[1])
