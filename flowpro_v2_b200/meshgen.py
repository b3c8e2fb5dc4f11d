"""Seeded synthetic meshes in FlowPro's mesh format.

FlowPro reads a mesh from vertices.txt (coordinates), elements.txt (0-based
vertex indexes, triangles counter-clockwise), elementType.txt (3 = triangle,
5 = tetrahedron), boundaryType.txt (rows "type v0 v1 [v2]") and builds
neighbors.txt from them (FlowProMain.createNeighborMatrix,
FlowPro/src/main/java/flowpro/core/FlowProMain.java:772-873).  The functions here
return the same arrays in memory:

    Mesh(vertices [nV, dim] f64, elements [nE, dim+1] i32, boundary [nB, dim+1] i32,
         wall_distance [nV] f64, elem_type int)

Boundary codes follow Aerodynamics.BoundaryType (Aerodynamics.java:11-18):
-1 wall (no-slip when viscous), -2 inlet, -3 outlet, -4 inviscid wall.
"""
from dataclasses import dataclass

import numpy as np

WALL, INLET, OUTLET, INVISCID_WALL = -1, -2, -3, -4


@dataclass
class Mesh:
    vertices: np.ndarray
    elements: np.ndarray
    boundary: np.ndarray
    wall_distance: np.ndarray
    elem_type: int

    @property
    def dim(self):
        return self.vertices.shape[1]

    @property
    def n_elem(self):
        return self.elements.shape[0]


def square_mesh(n, size=1.0, boundary_type=INLET):
    """TestSimulation.writeSquareMesh (FlowPro/src/test/java/flowpro/core/TestSimulation.java:28-80):
    [0, size]^2 in n x n cells, each split into two triangles with alternating
    diagonals, every boundary edge of type boundary_type."""
    h = size / n
    j, i = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    vertices = np.stack([i.ravel() * h, j.ravel() * h], axis=1).astype(np.float64)

    def vtx(ii, jj):
        return jj * (n + 1) + ii

    elems = []
    for jj in range(n):
        for ii in range(n):
            a, b, c, d = vtx(ii, jj), vtx(ii + 1, jj), vtx(ii + 1, jj + 1), vtx(ii, jj + 1)
            if (ii + jj) % 2 == 0:
                elems += [(a, b, c), (a, c, d)]
            else:
                elems += [(a, b, d), (b, c, d)]
    bnd = []
    for ii in range(n):
        bnd.append((boundary_type, vtx(ii, 0), vtx(ii + 1, 0)))
        bnd.append((boundary_type, vtx(n, ii), vtx(n, ii + 1)))
        bnd.append((boundary_type, vtx(ii + 1, n), vtx(ii, n)))
        bnd.append((boundary_type, vtx(0, ii + 1), vtx(0, ii)))
    wd = np.minimum(np.minimum(i, j), np.minimum(n - i, n - j)).ravel() * h
    return Mesh(vertices, np.array(elems, dtype=np.int32), np.array(bnd, dtype=np.int32),
                wd.astype(np.float64), 3)


def _bump_lower(x, height, x0=1.0, x1=2.0):
    """Lower wall y(x) of the channel: a circular arc of the given height over [x0, x1]."""
    c = x1 - x0
    r = (c * c / 4 + height * height) / (2 * height)
    xm = 0.5 * (x0 + x1)
    y = np.zeros_like(x)
    inside = (x > x0) & (x < x1)
    y[inside] = np.sqrt(np.maximum(r * r - (x[inside] - xm) ** 2, 0.0)) - (r - height)
    return y


def bump_channel(nx=150, ny=50, height=0.1, length=3.0, jitter=0.1, seed=1, inlet=INLET, outlet=OUTLET,
                 wall=INVISCID_WALL):
    """Channel [0, length] x [0, 1] with a circular-arc bump of the given height on
    x in [1, 2] of the lower wall; nx x ny quadrilaterals, each split into two
    counter-clockwise triangles; interior vertices jittered by up to `jitter` of
    the local spacing (seeded).  Left boundary inlet, right outlet, top and bottom
    walls.  Wall distance: distance to the nearest of the two walls, measured
    vertically."""
    rng = np.random.default_rng(seed)
    s = np.linspace(0.0, length, nx + 1)
    t = np.linspace(0.0, 1.0, ny + 1)
    S, T = np.meshgrid(s, t, indexing="ij")  # [nx+1, ny+1]
    yl = _bump_lower(S, height)
    X = S.copy()
    Y = yl + T * (1.0 - yl)
    hx = length / nx
    hy = (1.0 - yl) / ny
    dx = (rng.random(X.shape) * 2 - 1) * jitter * hx
    dy = (rng.random(X.shape) * 2 - 1) * jitter * hy
    interior = np.zeros(X.shape, dtype=bool)
    interior[1:-1, 1:-1] = True
    X = X + np.where(interior, dx, 0.0)
    Y = Y + np.where(interior, dy, 0.0)
    # keep the lower-wall vertices on the arc (x moved only in the interior)
    vertices = np.stack([X.ravel(), Y.ravel()], axis=1)

    def vid(i, j):
        return i * (ny + 1) + j

    I, J = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    a = vid(I, J)
    b = vid(I + 1, J)
    c = vid(I + 1, J + 1)
    d = vid(I, J + 1)
    alt = ((I + J) % 2 == 0)
    t1 = np.where(alt[..., None], np.stack([a, b, c], -1), np.stack([a, b, d], -1))
    t2 = np.where(alt[..., None], np.stack([a, c, d], -1), np.stack([b, c, d], -1))
    elems = np.stack([t1, t2], axis=2).reshape(-1, 3).astype(np.int32)
    bnd = []
    jj = np.arange(ny)
    bnd.append(np.stack([np.full(ny, inlet), vid(0, jj + 1), vid(0, jj)], 1))
    bnd.append(np.stack([np.full(ny, outlet), vid(nx, jj), vid(nx, jj + 1)], 1))
    ii = np.arange(nx)
    bnd.append(np.stack([np.full(nx, wall), vid(ii, 0), vid(ii + 1, 0)], 1))
    bnd.append(np.stack([np.full(nx, wall), vid(ii + 1, ny), vid(ii, ny)], 1))
    boundary = np.concatenate(bnd).astype(np.int32)
    yv = vertices[:, 1]
    ylow = _bump_lower(vertices[:, 0].copy(), height)
    wd = np.minimum(np.abs(yv - ylow), np.abs(1.0 - yv))
    return Mesh(vertices.astype(np.float64), elems, boundary, wd.astype(np.float64), 3)


def refined_channel_counts(refine=3.65, nx=150, ny=50):
    """Cell counts of the bump channel refined `refine` times per direction."""
    return int(round(nx * refine)), int(round(ny * refine))


def bump_box(nx=30, ny=10, nz=10, height=0.1, length=3.0, depth=1.0, jitter=0.08, seed=1, inlet=INLET,
             outlet=OUTLET, wall=INVISCID_WALL):
    """3D channel [0, length] x [0, 1] x [0, depth] with the bump of bump_channel on the
    lower y wall (extruded in z); nx x ny x nz hexahedra, each split into the six
    tetrahedra of the Kuhn split along its main diagonal (conforming across cells);
    interior vertices jittered (seeded).  Tetrahedra are emitted with
    det(x1 - x0, x2 - x0, x3 - x0) < 0, the orientation for which FlowPro's face normals
    (faceTransformation3Dtriangle.java:85-91) point outward.  Inlet at x = 0, outlet at
    x = length, walls elsewhere; wall distance measured vertically to the y walls."""
    rng = np.random.default_rng(seed)
    s = np.linspace(0.0, length, nx + 1)
    t = np.linspace(0.0, 1.0, ny + 1)
    r = np.linspace(0.0, depth, nz + 1)
    S, T, R = np.meshgrid(s, t, r, indexing="ij")
    yl = _bump_lower(S, height)
    X = S.copy()
    Y = yl + T * (1.0 - yl)
    Z = R.copy()
    interior = np.zeros(X.shape, dtype=bool)
    interior[1:-1, 1:-1, 1:-1] = True
    X = X + np.where(interior, (rng.random(X.shape) * 2 - 1) * jitter * length / nx, 0.0)
    Y = Y + np.where(interior, (rng.random(X.shape) * 2 - 1) * jitter * (1.0 - yl) / ny, 0.0)
    Z = Z + np.where(interior, (rng.random(X.shape) * 2 - 1) * jitter * depth / nz, 0.0)
    vertices = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1).astype(np.float64)

    def vid(i, j, k):
        return (i * (ny + 1) + j) * (nz + 1) + k

    I, J, K = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    unit = np.eye(3, dtype=np.int64)
    tets = []
    for perm in ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)):
        p = np.zeros((I.size, 3), dtype=np.int64)
        corners = [vid(I, J, K)]
        for ax in perm:
            p = p + unit[ax]
            corners.append(vid(I + p[:, 0], J + p[:, 1], K + p[:, 2]))
        tets.append(np.stack(corners, axis=1))
    elems = np.concatenate(tets).astype(np.int32)
    x = vertices[elems]
    det = np.einsum("ij,ij->i", np.cross(x[:, 1] - x[:, 0], x[:, 2] - x[:, 0]), x[:, 3] - x[:, 0])
    swap = det > 0
    elems[swap, 1], elems[swap, 2] = elems[swap, 2].copy(), elems[swap, 1].copy()
    # boundary faces: the faces that belong to one tetrahedron only
    faces = np.concatenate([elems[:, [0, 1, 2]], elems[:, [0, 1, 3]], elems[:, [1, 2, 3]], elems[:, [0, 2, 3]]])
    key = np.sort(faces, axis=1)
    uniq, inv, cnt = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    bfaces = uniq[cnt == 1]
    xc = vertices[bfaces][:, :, 0].mean(axis=1)
    tol = 1e-9 * length
    code = np.where(xc < tol, inlet, np.where(xc > length - tol, outlet, wall))
    boundary = np.concatenate([code[:, None], bfaces], axis=1).astype(np.int32)
    yv = vertices[:, 1]
    ylow = _bump_lower(vertices[:, 0].copy(), height)
    wd = np.minimum(np.abs(yv - ylow), np.abs(1.0 - yv))
    return Mesh(vertices, elems, boundary, wd.astype(np.float64), 5)


def serving_cases(n_cases=256, seed=1, min_elements=2000, max_elements=60000, kappa=1.4):
    """The batched-serving set: n_cases bump channels of uneven size and order, all from one
    seed.  Element counts log-uniform in [min_elements, max_elements] (nx = 3 ny, two
    triangles per cell), polynomial degree p uniform in {1, 2, 3} (FlowPro order p + 1),
    inlet Mach uniform in [0.3, 0.7] (outlet pressure pOut = (1 + (kappa-1)/2 M^2)^(-kappa/(kappa-1))
    relative to the inlet stagnation pressure), bump height uniform in [0.05, 0.12]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_cases):
        n_el = float(np.exp(rng.uniform(np.log(min_elements), np.log(max_elements))))
        ny = max(2, int(round(np.sqrt(n_el / 6.0))))
        nx = 3 * ny
        p = int(rng.integers(1, 4))
        mach = float(rng.uniform(0.3, 0.7))
        height = float(rng.uniform(0.05, 0.12))
        pout = (1 + (kappa - 1) / 2 * mach * mach) ** (-kappa / (kappa - 1))
        out.append(dict(case=i, nx=nx, ny=ny, order=p + 1, mach=mach, height=height, pOut=pout,
                        seed=int(rng.integers(1, 2 ** 31 - 1))))
    return out


def naca0012_thickness(x, t=0.12):
    """Half thickness of the NACA 0012 with the closed (sharp) trailing edge coefficient."""
    return 5 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 - 0.1036 * x ** 4)


def naca0012_o_mesh(n_around=512, first_height=1e-5, growth=1.15, radius=50.0, seed=1, jitter=0.0):
    """O-grid around the NACA 0012 (chord [0, 1], closed-form thickness, sharp trailing edge)
    in a circular far field of the given radius about (0.5, 0).  n_around surface points with
    cosine clustering towards both edges; grid lines are rays from (0.5, 0) through the surface
    points (so they never cross), with geometric stretching from first_height at the wall
    (growth ratio per layer) until the far field.  Quads split into two counter-clockwise
    triangles.  Boundary codes: -1 wall (airfoil), -2 inlet (far field upstream, x < 0.5),
    -3 outlet (downstream).  Interior vertices optionally jittered (fraction of the local
    layer height, seeded).  Wall distance per vertex by the edge-path distance of
    FlowProMain.generateDistanceFunction."""
    rng = np.random.default_rng(seed)
    half = n_around // 2
    beta = np.linspace(0.0, np.pi, half + 1)
    xs = 0.5 * (1 + np.cos(beta))  # 1 (TE) -> 0 (LE)
    yt = naca0012_thickness(xs)
    # counter-clockwise around the centre: TE, upper surface to LE, lower surface back to TE
    upper = np.stack([xs, yt], 1)                # TE -> LE over the top
    lower = np.stack([xs[::-1], -yt[::-1]], 1)   # LE -> TE along the bottom
    surf = np.concatenate([upper[:-1], lower[:-1]])  # n_around points, TE first
    n_i = surf.shape[0]
    centre = np.array([0.5, 0.0])
    ang = np.arctan2(surf[:, 1] - centre[1], surf[:, 0] - centre[0])
    far = centre + radius * np.stack([np.cos(ang), np.sin(ang)], 1)
    # layer distances along each ray, normalised so that the last layer reaches the far field
    s = [0.0]
    h = first_height
    while s[-1] < radius:
        s.append(s[-1] + h)
        h *= growth
    s = np.array(s)
    n_j = len(s) - 1
    P = np.zeros((n_i, n_j + 1, 2))
    for i in range(n_i):
        frac = s / s[-1]
        P[i] = surf[i] + frac[:, None] * (far[i] - surf[i])
    if jitter > 0:
        dj = np.diff(s)
        for j in range(1, n_j):
            amp = jitter * min(dj[j - 1], dj[j]) / s[-1]
            d = (rng.random((n_i, 2)) * 2 - 1) * amp * np.linalg.norm(far - surf, axis=1)[:, None]
            P[:, j] += d
    vertices = P.reshape(-1, 2)

    def vid(i, j):
        return (i % n_i) * (n_j + 1) + j

    I, J = np.meshgrid(np.arange(n_i), np.arange(n_j), indexing="ij")
    a, b, c, d = vid(I, J), vid(I + 1, J), vid(I + 1, J + 1), vid(I, J + 1)
    t1 = np.stack([a, b, c], -1).reshape(-1, 3)
    t2 = np.stack([a, c, d], -1).reshape(-1, 3)
    elems = np.concatenate([t1, t2]).astype(np.int32)
    x = vertices[elems]
    area = (x[:, 1, 0] - x[:, 0, 0]) * (x[:, 2, 1] - x[:, 0, 1]) - (x[:, 2, 0] - x[:, 0, 0]) * (x[:, 1, 1] - x[:, 0, 1])
    flip = area < 0
    elems[flip, 1], elems[flip, 2] = elems[flip, 2].copy(), elems[flip, 1].copy()
    ii = np.arange(n_i)
    wall = np.stack([np.full(n_i, WALL), vid(ii, 0), vid(ii + 1, 0)], 1)
    fx = 0.5 * (far[ii, 0] + far[(ii + 1) % n_i, 0])
    code = np.where(fx < centre[0], INLET, OUTLET)
    outer = np.stack([code, vid(ii + 1, n_j), vid(ii, n_j)], 1)
    boundary = np.concatenate([wall, outer]).astype(np.int32)
    from flowpro_v2_b200 import create_neighbor_matrix, wall_distance  # host functions of the library
    tt = create_neighbor_matrix(2, elems, boundary)
    wd = wall_distance(vertices, elems, tt, WALL)
    return Mesh(vertices.astype(np.float64), elems, boundary, wd, 3)
