"""Generate gauss_rules.h from FlowPro's quadrature rule files.

The DG residual must integrate with exactly the rules FlowPro reads at start-up
(FlowPro/gaussRules/{gauss,gaussTri,gaussTetra}/<n>.txt, loaded by
flowpro/core/quadrature/QuadratureCentral.java:33-91), so the point/weight
tables are carried over as data.  This script parses those text files the way
QuadratureLine/QuadratureTriangle/QuadratureTetra do (count, points, weights;
triangle points given in barycentric coordinates and mapped to (xi, eta) by
QuadratureTriangle.setCoords) and writes a C header.  It is run once by a
developer with the FlowPro checkout at hand; the generated header is committed.

usage: python gen_gauss_rules.py <FlowPro/gaussRules dir> > gauss_rules.h
"""
import os
import sys


def parse(path, kind):
    with open(path) as f:
        lines = [ln.strip() for ln in f if ln.strip()]
    n = int(lines[0])
    pts = []
    for i in range(n):
        tok = [float(t) for t in lines[1 + i].split()]
        if kind == "line":
            pts.append((tok[0],))
        elif kind == "tri":
            # barycentric (b0, b1, b2) on vertices (0,0), (1,0), (0,1)
            x = 0.0 * tok[0] + 1.0 * tok[1] + 0.0 * tok[2]
            y = 0.0 * tok[0] + 0.0 * tok[1] + 1.0 * tok[2]
            pts.append((x, y))
        else:
            pts.append(tuple(tok[:3]))
    w = [float(lines[1 + n + i]) for i in range(n)]
    return pts, w


def main():
    root = sys.argv[1]
    out = []
    out.append("// Generated by gen_gauss_rules.py from FlowPro/gaussRules (data tables).")
    out.append("// Quadrature rules as loaded by FlowPro's QuadratureCentral: line rules")
    out.append("// indexed by point count, triangle/tetrahedron rules by exact degree.")
    out.append("#pragma once")
    out.append("namespace fpr {")
    out.append("struct RuleEntry { int kind; int key; int n; const double* pts; const double* w; };")
    entries = []
    specs = [("line", "gauss", range(1, 11), 1), ("tri", "gaussTri", range(1, 16), 2),
             ("tet", "gaussTetra", range(1, 16), 3)]
    for kind, sub, keys, dim in specs:
        for k in keys:
            p = os.path.join(root, sub, f"{k}.txt")
            if not os.path.exists(p):
                continue
            pts, w = parse(p, kind)
            name = f"{kind}_{k}"
            flat = [c for pt in pts for c in pt]
            out.append(f"static const double {name}_pts[{len(flat)}] = {{" +
                       ", ".join(repr(v) for v in flat) + "};")
            out.append(f"static const double {name}_w[{len(w)}] = {{" +
                       ", ".join(repr(v) for v in w) + "};")
            entries.append(f"  {{{dim}, {k}, {len(w)}, {name}_pts, {name}_w}}")
    out.append("static const RuleEntry kRules[] = {")
    out.append(",\n".join(entries))
    out.append("};")
    out.append(f"static const int kNumRules = {len(entries)};")
    out.append("}  // namespace fpr")
    print("\n".join(out))


if __name__ == "__main__":
    main()
