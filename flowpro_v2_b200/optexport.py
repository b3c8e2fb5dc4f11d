"""Export for FlowPro's optimisation toolbox (OptimisationToolExport.export,
flowpro/core/OptimisationToolExport.java:40-131): the files the MATLAB toolbox reads from
<simulation>/optimisation/, written from the GPU solution in the reference's text formats.

  I<a>.txt        the functional of interest for mesh a (exportFunctional, :204-220)
  R<a>.txt        the steady residual R(W) per element and unknown (exportResiduum, :161-175,
                  Element.exportLocalR, Element.java:737-747)
  J.txt           the steady element Jacobian blocks as (row, column, value) triplets in the
                  global DOF numbering (exportJacobiTranspose, :133-159,
                  Element.exportLocalJacobiMatrix, Element.java:750-786)
  dIdw.txt        the derivative of the functional by every unknown (exportFunctionalDerivative,
                  :177-202)
  M<a>.txt        the element mass matrices as triplets (exportMassMatrix, :222-240; mode "allmass")
  printMatrix.txt (element equation, unknown, basis weight) triplets (exportPrintMatrix, :242-256)

Mode "all" writes I0, J, R0, dIdw, then I<a>, R<a> for every perturbed mesh a = 1..n, then
printMatrix; "allmass" adds M0 and M<a>; any other mode writes I0 only (the reference's
branches).  Numbers are written as Java's Double.toString writes them (shortest round-trip
digits; decimal notation for 1e-3 <= |x| < 1e7, else d.dddE<n>), one value and a space per
line where the reference writes `x + " "`.  The digits are those of Java 19 and later (shortest
decimal); the Java 17 runtime the reference targets (sourceCompatibility 17) prints one or two
extra digits for some values (2.82879384806159008E17 where Java 19 prints 2.82879384806159E17),
so such numbers can differ from a Java 17 file in their last digits, never in value.

Deviation: dIdw holds the exact derivative of the functional (forward mode on the device)
instead of the reference's one-sided finite difference with step Parameters.h.
"""
import math
import os
from decimal import Decimal

import numpy as np


def java_double(x):
    """Double.toString(x): shortest digits that read back to x, in Java's layout."""
    x = float(x)
    if x != x:
        return "NaN"
    if x == math.inf:
        return "Infinity"
    if x == -math.inf:
        return "-Infinity"
    if x == 0.0:
        return "-0.0" if math.copysign(1.0, x) < 0 else "0.0"
    sign = "-" if x < 0 else ""
    r = repr(abs(x))  # the shortest round-trip digits, e.g. '0.001', '1e-05', '1.25e+20'
    mant, _, e = r.partition("e")
    ip, _, fp = mant.partition(".")
    all_digits = ip + fp
    stripped = all_digits.lstrip("0")
    # abs(x) = 0.d1 d2 ... x 10^point
    point = len(ip) - (len(all_digits) - len(stripped)) + (int(e) if e else 0)
    digits = stripped.rstrip("0") or "0"
    if len(digits) == 1:
        # one significant digit: Java takes the two-digit decimal closest to x among those
        # that read back to x (Double.MIN_VALUE prints as 4.9E-324, 1.0 as 1.0)
        exact = Decimal(abs(x))
        best = None
        for D in range(10, 100):
            cand = Decimal(D).scaleb(point - 2)
            if float(cand) == abs(x) and (best is None or abs(cand - exact) < abs(best[1] - exact)):
                best = (D, cand)
        if best is not None:
            digits = str(best[0]).rstrip("0")
    if 1e-3 <= abs(x) < 1e7:
        if point <= 0:
            return sign + "0." + "0" * (-point) + digits
        if point >= len(digits):
            return sign + digits + "0" * (point - len(digits)) + ".0"
        return sign + digits[:point] + "." + digits[point:]
    return sign + digits[0] + "." + (digits[1:] or "0") + "E" + str(point - 1)


def _lines(values):
    return "".join(java_double(v) + " \n" for v in values)


def write_functional(directory, alpha, value):
    with open(os.path.join(directory, f"I{alpha}.txt"), "w") as f:
        f.write(java_double(value) + " \n")


def write_residual(directory, alpha, R):
    """R: [elements][n] in element order (Element.exportLocalR's RHS_loc of every element)."""
    with open(os.path.join(directory, f"R{alpha}.txt"), "w") as f:
        f.write(_lines(np.asarray(R, dtype=np.float64).reshape(-1)))


def write_functional_derivative(directory, dIdw):
    with open(os.path.join(directory, "dIdw.txt"), "w") as f:
        f.write(_lines(np.asarray(dIdw, dtype=np.float64).reshape(-1)))


def _gindex(block_position, n):
    """Element.gIndex of every element: n consecutive numbers per element in the DOF order
    (Element.setGlobalIndex, Element.java:241-248, called in ElementOrdering order, Mesh.java:181-184)."""
    return np.asarray(block_position, dtype=np.int64)[:, None] * n + np.arange(n)[None, :]


def write_jacobian(directory, diag, neigh, neighbors, block_position):
    """diag[e][i][j] = ADiag[i][j], neigh[e][k][i][j] = ANeighs[k].A[i][j] (the reference's
    transposed storage, element e, face k), neighbors[e][k] the neighbour or a negative code."""
    diag = np.asarray(diag, dtype=np.float64)
    neigh = np.asarray(neigh, dtype=np.float64)
    nE, n = diag.shape[0], diag.shape[1]
    g = _gindex(block_position, n)
    rows = []
    for k in range(nE):
        gi = g[k]
        # (gIndex[i], gIndex[j], ADiag[j][i]) for i, j in 0..n-1
        A = diag[k].T
        for i in range(n):
            rows.append("".join(f"{gi[i]} {gi[j]} {java_double(A[i, j])}\n" for j in range(n)))
        for face in range(neigh.shape[1]):
            nb = int(neighbors[k][face])
            if nb > -1:
                gr = g[nb]
                B = neigh[k, face].T  # (gIndex[i], gIndexR[j], ANeighs[face].A[j][i])
                for i in range(n):
                    rows.append("".join(f"{gi[i]} {gr[j]} {java_double(B[i, j])}\n" for j in range(n)))
    with open(os.path.join(directory, "J.txt"), "w") as f:
        f.write("".join(rows))


def write_mass(directory, alpha, M, block_position, n_eqs):
    """M[e][i][j] = Element.M; triplets (gIndex[nb m + i], gIndex[nb m + j], M[i][j]) per equation."""
    M = np.asarray(M, dtype=np.float64)
    nE, nb = M.shape[0], M.shape[1]
    g = _gindex(block_position, nb * n_eqs)
    out = []
    for k in range(nE):
        for m in range(n_eqs):
            for i in range(nb):
                out.append("".join(f"{g[k][nb * m + i]} {g[k][nb * m + j]} {java_double(M[k, i, j])}\n" for j in range(nb)))
    with open(os.path.join(directory, f"M{alpha}.txt"), "w") as f:
        f.write("".join(out))


def write_print_matrix(directory, Is, block_position, n_eqs):
    """Is[e][i] = Element.Is; triplets (k nEqs + j, gIndex[j nBasis + i], Is[i])."""
    Is = np.asarray(Is, dtype=np.float64)
    nE, nb = Is.shape
    g = _gindex(block_position, nb * n_eqs)
    out = []
    for k in range(nE):
        for i in range(nb):
            out.append("".join(f"{k * n_eqs + j} {g[k][j * nb + i]} {java_double(Is[k, i])}\n" for j in range(n_eqs)))
    with open(os.path.join(directory, "printMatrix.txt"), "w") as f:
        f.write("".join(out))


def export(mesh, directory, functional, mode="all", perturbed_vertices=(), make_mesh=None):
    """OptimisationToolExport.export from a GpuMesh holding the converged state.

    functional: FUNCTIONAL_LIFT or FUNCTIONAL_DRAG; perturbed_vertices: vertex arrays of the
    meshes a = 1, 2, ... (the reference reads optimisation/vertices<a>.txt); make_mesh(vertices)
    builds a GpuMesh of the same elements on them (the state is copied over).  Returns the
    names of the files written."""
    from . import JacobiAssembler
    os.makedirs(directory, exist_ok=True)
    written = []

    def emit(name):
        written.append(name)

    value, dIdw = mesh.functional(functional)
    write_functional(directory, 0, value)
    emit("I0.txt")
    if mode.lower() not in ("all", "allmass"):
        return written
    block_position = mesh.dof_order()
    asm = JacobiAssembler(mesh, bdf_order=1)
    asm.assemble(0.0, 0.0)  # steady operator: dR/dW blocks, RHS = R(W)
    diag, neigh, rhs = asm.blocks()
    write_jacobian(directory, diag, neigh, mesh.neighbors, block_position)
    emit("J.txt")
    if mode.lower() == "allmass":
        M, _ = mesh.mass_matrices()
        write_mass(directory, 0, M, block_position, mesh.n_eqs)
        emit("M0.txt")
    write_residual(directory, 0, rhs)
    emit("R0.txt")
    write_functional_derivative(directory, dIdw)
    emit("dIdw.txt")
    W = mesh.get_state(0)
    for a, verts in enumerate(perturbed_vertices, start=1):
        g = make_mesh(np.asarray(verts, dtype=np.float64))
        try:
            g.set_state(W)
            g.limiter()
            if mode.lower() == "allmass":
                M, _ = g.mass_matrices()
                write_mass(directory, a, M, block_position, mesh.n_eqs)
                emit(f"M{a}.txt")
            write_functional(directory, a, g.functional(functional, gradient=False)[0])
            emit(f"I{a}.txt")
            write_residual(directory, a, g.residuum())
            emit(f"R{a}.txt")
        finally:
            g.close()
    _, Is = mesh.mass_matrices()
    write_print_matrix(directory, Is, block_position, mesh.n_eqs)
    emit("printMatrix.txt")
    return written
