// Host set-up: reference-element tables, affine element geometry, neighbour
// matrix, DOF ordering and model parameters.  Runs once per mesh upload; the
// results are copied to the device by fp_api.cu.
//
// What has to agree with FlowPro for parity (and is therefore built the same way):
//   * Lagrange nodes and their order (basis2Dtriangle.barycentr,
//     flowpro/core/basis/basis2Dtriangle.java:64-86; tetrahedra: vertices, then for
//     p = 2 the edge midpoints 01, 02, 03, 12, 13, 23, because the reference's
//     basis3Dtetra.barycentr lists only the vertices there, basis3Dtetra.java:50-62);
//   * quadrature rules (QuadratureCentral.java:46-91) from gauss_rules.h;
//   * face vertex conventions (triangleElement.java:52-54, tetrahedralElement.java:52-68)
//     and the orientation of normals (faceTransformation2Dline.java:55-59,
//     faceTransformation3Dtriangle.java:85-91);
//   * the element centre Xs (transformation2Dtriangle.getXs).  Tetrahedra use the
//     centroid x(1/4, 1/4, 1/4): the reference's literal {0.25, 0.25, 0, 25}
//     (transformation3Dtetra.java:116) lands on face 0 and makes its DDG distance zero;
//   * the reverse Cuthill-McKee ordering (ElementOrdering.java:52-142).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <deque>
#include <map>
#include <sstream>
#include <unordered_map>

#include "fp_mesh.h"
#include "gauss_rules.h"

namespace fp {

namespace {

struct Rule {
    int n = 0, dim = 0;
    std::vector<double> pts, w;
};

bool find_rule(int kind, int key, Rule& r) {
    for (int i = 0; i < fpr::kNumRules; i++) {
        const auto& e = fpr::kRules[i];
        if (e.kind == kind && e.key == key) {
            r.n = e.n;
            r.dim = kind;
            r.pts.assign(e.pts, e.pts + e.n * kind);
            r.w.assign(e.w, e.w + e.n);
            return true;
        }
    }
    return false;
}

// rule of FlowPro order `order` for a simplex of dimension sdim (1 line, 2 triangle, 3 tetrahedron)
bool simplex_rule(int sdim, int order, Rule& r) {
    if (sdim == 1) return find_rule(1, order, r);
    if (sdim == 2) {
        if (!find_rule(2, 2 * order - 1, r)) return false;
        for (double w : r.w)
            if (w < 0) return find_rule(2, 2 * order, r);
        return true;
    }
    return find_rule(3, 2 * order - 1, r);
}

// small dense inverse, Gauss-Jordan with partial pivoting
bool invert(std::vector<double> A, int n, std::vector<double>& X) {
    X.assign(n * n, 0.0);
    for (int i = 0; i < n; i++) X[i * n + i] = 1;
    for (int c = 0; c < n; c++) {
        int p = c;
        for (int r = c + 1; r < n; r++)
            if (std::fabs(A[r * n + c]) > std::fabs(A[p * n + c])) p = r;
        if (A[p * n + c] == 0) return false;
        if (p != c)
            for (int j = 0; j < n; j++) {
                std::swap(A[p * n + j], A[c * n + j]);
                std::swap(X[p * n + j], X[c * n + j]);
            }
        double inv = 1.0 / A[c * n + c];
        for (int j = 0; j < n; j++) {
            A[c * n + j] *= inv;
            X[c * n + j] *= inv;
        }
        for (int r = 0; r < n; r++)
            if (r != c) {
                double f = A[r * n + c];
                if (f != 0)
                    for (int j = 0; j < n; j++) {
                        A[r * n + j] -= f * A[c * n + j];
                        X[r * n + j] -= f * X[c * n + j];
                    }
            }
    }
    return true;
}

// Lagrange basis on the reference simplex: nodes, monomial exponents, coefficients
struct Lagrange {
    int dim, order, nb;
    std::vector<std::array<int, 3>> ex;  // exponents of the complete polynomial space
    std::vector<double> C;               // C[i][m]: coefficient of monomial i in basis m

    Lagrange(int dim_, int order_) : dim(dim_), order(order_), nb(nbasis_of(dim_, order_)) {
        int p = order - 1;
        for (int t = 0; t <= p; t++)
            for (int a = t; a >= 0; a--)
                if (dim == 2) {
                    ex.push_back({a, t - a, 0});
                } else {
                    for (int b = t - a; b >= 0; b--) ex.push_back({a, b, t - a - b});
                }
        std::vector<std::array<double, 3>> nodes = lagrange_nodes();
        std::vector<double> V(nb * nb);
        for (int i = 0; i < nb; i++)
            for (int j = 0; j < nb; j++) V[i * nb + j] = mono(j, nodes[i].data());
        std::vector<double> Vi;
        invert(V, nb, Vi);
        C = Vi;  // sum_i C[i][m] mono_i(node_k) = delta_km
    }

    // node sets: triangles as basis2Dtriangle.barycentr (nodes X = (b1, b2)), tetrahedra:
    // vertices (0,0,0), (1,0,0), (0,1,0), (0,0,1) and for order 3 the edge midpoints
    std::vector<std::array<double, 3>> lagrange_nodes() const {
        std::vector<std::array<double, 3>> nd;
        if (order == 1) {
            nd.push_back(dim == 2 ? std::array<double, 3>{1.0 / 3, 1.0 / 3, 0} : std::array<double, 3>{0.25, 0.25, 0.25});
            return nd;
        }
        if (dim == 2) {
            auto lin = [](double a, double b, int n) {
                std::vector<double> x(n);
                if (n == 1) {
                    x[0] = (a + b) / 2;
                } else {
                    for (int i = 0; i < n; i++) {
                        double xi = (double)i / (n - 1);
                        x[i] = (1 - xi) * a + xi * b;
                    }
                }
                return x;
            };
            std::vector<double> x = lin(0, 1, order);
            for (int i = 0; i < order; i++) {
                std::vector<double> y = lin(0, x[i], i + 1);
                for (int j = 0; j < i + 1; j++) nd.push_back({y[j], x[i] - y[j], 0});
            }
        } else {
            double v[4][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
            for (auto& p : v) nd.push_back({p[0], p[1], p[2]});
            if (order == 3) {
                int e[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
                for (auto& ed : e)
                    nd.push_back({0.5 * (v[ed[0]][0] + v[ed[1]][0]), 0.5 * (v[ed[0]][1] + v[ed[1]][1]),
                                  0.5 * (v[ed[0]][2] + v[ed[1]][2])});
            }
        }
        return nd;
    }
    static double ipow(double x, int k) {
        double r = 1;
        for (int i = 0; i < k; i++) r *= x;
        return r;
    }
    double mono(int i, const double* X) const {
        double r = ipow(X[0], ex[i][0]) * ipow(X[1], ex[i][1]);
        if (dim == 3) r *= ipow(X[2], ex[i][2]);
        return r;
    }
    double dmono(int i, const double* X, int d) const {
        int e = ex[i][d];
        if (e == 0) return 0;
        double r = e;
        for (int c = 0; c < dim; c++) r *= ipow(X[c], c == d ? ex[i][c] - 1 : ex[i][c]);
        return r;
    }
    double phi(int m, const double* X) const {
        double v = 0;
        for (int i = 0; i < nb; i++) v += C[i * nb + m] * mono(i, X);
        return v;
    }
    double dphi(int m, const double* X, int d) const {
        double v = 0;
        for (int i = 0; i < nb; i++) v += C[i * nb + m] * dmono(i, X, d);
        return v;
    }
};

const double kRefVert2[3][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}};
const double kRefVert3[4][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};

void face_vertices(int dim, int k, int* fi) {
    if (dim == 2) {
        fi[0] = k;
        fi[1] = (k + 1) % 3;
        return;
    }
    static const int F[4][3] = {{0, 2, 1}, {0, 1, 3}, {1, 2, 3}, {2, 0, 3}};
    for (int i = 0; i < 3; i++) fi[i] = F[k][i];
}

// permutations of the face vertices: right face vertex j = left face vertex perm[j]
const int kPerm2[2][3] = {{0, 1, 0}, {1, 0, 0}};
const int kPerm3[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

const double* ref_vertex(int dim, int v) { return dim == 2 ? kRefVert2[v] : kRefVert3[v]; }

// barycentric weights of the face vertices at face quadrature point p
void face_lambda(int dim, const Rule& fr, int p, double* lam) {
    if (dim == 2) {
        double s = fr.pts[p];
        lam[0] = (1 - s) / 2;
        lam[1] = (1 + s) / 2;
    } else {
        double a = fr.pts[p * 2], b = fr.pts[p * 2 + 1];
        lam[0] = 1 - a - b;
        lam[1] = a;
        lam[2] = b;
    }
}

}  // namespace

int build_ref_tables(int dim, int order, RefTables& t, std::string& err) {
    if (dim != 2 && dim != 3) {
        err = "dimension must be 2 or 3";
        return FP_ERR_UNSUPPORTED;
    }
    if (order < 1 || (dim == 2 && order > 4) || (dim == 3 && order > 3)) {
        err = "unsupported order " + std::to_string(order) + " for dimension " + std::to_string(dim);
        return FP_ERR_UNSUPPORTED;
    }
    Rule vr, fr;
    if (!simplex_rule(dim, order, vr) || !simplex_rule(dim - 1, order, fr)) {
        err = "quadrature rule not available";
        return FP_ERR_UNSUPPORTED;
    }
    Lagrange L(dim, order);
    t.dim = dim;
    t.order = order;
    t.nb = L.nb;
    t.nqv = vr.n;
    t.nqf = fr.n;
    t.nf = dim + 1;
    t.nv = dim + 1;
    t.nvf = dim;
    t.nperm = nperm_of(dim);
    if (t.nqv != nqv_of(dim, order) || t.nqf != nqf_of(dim, order) || t.nb != nbasis_of(dim, order)) {
        err = "internal: table sizes disagree with the compiled configuration";
        return FP_ERR_UNSUPPORTED;
    }
    std::vector<double>& D = t.data;
    D.clear();
    auto alloc = [&](int n) {
        int o = (int)D.size();
        D.resize(D.size() + n, 0.0);
        return o;
    };
    int nb = t.nb, nqv = t.nqv, nqf = t.nqf, nf = t.nf, nv = t.nv, nvf = t.nvf, np = t.nperm;
    t.o_w = alloc(nqv);
    t.o_phi = alloc(nqv * nb);
    t.o_dphi = alloc(nqv * nb * dim);
    t.o_interp = alloc(nqv * nv);
    t.o_xi = alloc(nqv * dim);
    for (int q = 0; q < nqv; q++) {
        const double* X = &vr.pts[q * dim];
        D[t.o_w + q] = vr.w[q];
        for (int j = 0; j < nb; j++) {
            D[t.o_phi + q * nb + j] = L.phi(j, X);
            for (int d = 0; d < dim; d++) D[t.o_dphi + (q * nb + j) * dim + d] = L.dphi(j, X, d);
        }
        double s = 0;
        for (int d = 0; d < dim; d++) s += X[d];
        D[t.o_interp + q * nv + 0] = 1 - s;
        for (int d = 0; d < dim; d++) D[t.o_interp + q * nv + 1 + d] = X[d];
        for (int d = 0; d < dim; d++) D[t.o_xi + q * dim + d] = X[d];
    }
    t.o_wf = alloc(nqf);
    t.o_phiL = alloc(nf * nqf * nb);
    t.o_dphiL = alloc(nf * nqf * nb * dim);
    t.o_finterp = alloc(nqf * nvf);
    t.o_xiL = alloc(nf * nqf * dim);
    for (int p = 0; p < nqf; p++) {
        D[t.o_wf + p] = fr.w[p];
        double lam[3];
        face_lambda(dim, fr, p, lam);
        for (int i = 0; i < nvf; i++) D[t.o_finterp + p * nvf + i] = lam[i];
    }
    for (int k = 0; k < nf; k++) {
        int fi[3];
        face_vertices(dim, k, fi);
        for (int p = 0; p < nqf; p++) {
            double lam[3], X[3] = {0, 0, 0};
            face_lambda(dim, fr, p, lam);
            for (int i = 0; i < nvf; i++)
                for (int d = 0; d < dim; d++) X[d] += lam[i] * ref_vertex(dim, fi[i])[d];
            for (int d = 0; d < dim; d++) D[t.o_xiL + (k * nqf + p) * dim + d] = X[d];
            for (int j = 0; j < nb; j++) {
                D[t.o_phiL + (k * nqf + p) * nb + j] = L.phi(j, X);
                for (int d = 0; d < dim; d++) D[t.o_dphiL + ((k * nqf + p) * nb + j) * dim + d] = L.dphi(j, X, d);
            }
        }
    }
    t.o_phiR = alloc(nf * np * nqf * nb);
    t.o_dphiR = alloc(nf * np * nqf * nb * dim);
    for (int k = 0; k < nf; k++) {
        int fi[3];
        face_vertices(dim, k, fi);
        for (int pm = 0; pm < np; pm++) {
            const int* perm = dim == 2 ? kPerm2[pm] : kPerm3[pm];
            for (int p = 0; p < nqf; p++) {
                double lam[3], X[3] = {0, 0, 0};
                face_lambda(dim, fr, p, lam);
                for (int j = 0; j < nvf; j++)
                    for (int d = 0; d < dim; d++) X[d] += lam[perm[j]] * ref_vertex(dim, fi[j])[d];
                int base = (k * np + pm) * nqf + p;
                for (int j = 0; j < nb; j++) {
                    D[t.o_phiR + base * nb + j] = L.phi(j, X);
                    for (int d = 0; d < dim; d++) D[t.o_dphiR + (base * nb + j) * dim + d] = L.dphi(j, X, d);
                }
            }
        }
    }
    t.o_Is = alloc(nb);
    t.o_Mref = alloc(nb * nb);
    t.o_MinvRef = alloc(nb * nb);
    t.o_one = alloc(nb);
    double wsum = 0;
    for (int q = 0; q < nqv; q++) wsum += vr.w[q];
    std::vector<double> Mr(nb * nb, 0.0), ints(nb, 0.0);
    for (int j = 0; j < nb; j++) {
        double s = 0;
        for (int q = 0; q < nqv; q++) s += vr.w[q] * D[t.o_phi + q * nb + j];
        D[t.o_Is + j] = s / wsum;
        ints[j] = s;
        for (int i = 0; i < nb; i++) {
            double m = 0;
            for (int q = 0; q < nqv; q++) m += vr.w[q] * D[t.o_phi + q * nb + i] * D[t.o_phi + q * nb + j];
            Mr[i * nb + j] = m;
        }
    }
    std::vector<double> Mi;
    if (!invert(Mr, nb, Mi)) {
        err = "singular reference mass matrix";
        return FP_ERR_UNSUPPORTED;
    }
    for (int i = 0; i < nb * nb; i++) {
        D[t.o_Mref + i] = Mr[i];
        D[t.o_MinvRef + i] = Mi[i];
    }
    // coefficients of the constant function 1 (Element.positivityLimiter, Element.java:406-419)
    for (int i = 0; i < nb; i++) {
        double s = 0;
        for (int j = 0; j < nb; j++) s += Mi[i * nb + j] * ints[j];
        D[t.o_one + i] = s;
    }
    // truncation to linear order (DGpure.computeOrderTruncationMatrix, DGpure.java:595-627):
    // TrunOrd = M^-1 T^T Mhat^-1 T with the Taylor basis (1, xi - xi_s) of the reference
    // element; the L2 projection onto linear functions is invariant under the affine map.
    t.o_trun = alloc(nb * nb);
    {
        int nl = 1 + dim;
        double xs[3] = {dim == 2 ? 1.0 / 3 : 0.25, dim == 2 ? 1.0 / 3 : 0.25, 0.0};
        std::vector<double> Mh(nl * nl, 0.0), T(nl * nb, 0.0);
        auto tay = [&](int i, const double* X) { return i > 0 ? X[i - 1] - xs[i - 1] : 1.0; };
        for (int q = 0; q < nqv; q++) {
            const double* X = &vr.pts[q * dim];
            for (int i = 0; i < nl; i++) {
                for (int j = 0; j < nl; j++) Mh[i * nl + j] += vr.w[q] * tay(i, X) * tay(j, X);
                for (int j = 0; j < nb; j++) T[i * nb + j] += vr.w[q] * tay(i, X) * D[t.o_phi + q * nb + j];
            }
        }
        std::vector<double> Mhi;
        if (nb > 1 && invert(Mh, nl, Mhi)) {
            std::vector<double> A(nl * nb, 0.0), B(nb * nb, 0.0);
            for (int i = 0; i < nl; i++)
                for (int j = 0; j < nb; j++)
                    for (int k = 0; k < nl; k++) A[i * nb + j] += Mhi[i * nl + k] * T[k * nb + j];
            for (int i = 0; i < nb; i++)
                for (int j = 0; j < nb; j++)
                    for (int k = 0; k < nl; k++) B[i * nb + j] += T[k * nb + i] * A[k * nb + j];
            for (int i = 0; i < nb; i++)
                for (int j = 0; j < nb; j++) {
                    double s = 0;
                    for (int k = 0; k < nb; k++) s += Mi[i * nb + k] * B[k * nb + j];
                    D[t.o_trun + i * nb + j] = s;
                }
        }
    }
    return FP_OK;
}

// ---------------------------------------------------------------------------- geometry
int build_host_mesh(const fp_mesh_desc& desc, const fp_model_params& model, const fp_num_params& num, HostMesh& hm,
                    std::string& err) {
    int dim = desc.dim;
    if (dim != model.dim) {
        err = "mesh dimension differs from the model dimension";
        return FP_ERR_ARG;
    }
    if (desc.n_elements <= 0 || desc.n_vertices <= 0 || !desc.vertices || !desc.elements || !desc.neighbors) {
        err = "empty mesh";
        return FP_ERR_ARG;
    }
    int rc = build_ref_tables(dim, num.order, hm.tab, err);
    if (rc) return rc;
    hm.dim = dim;
    hm.nElem = desc.n_elements;
    hm.nVert = desc.n_vertices;
    hm.nf = dim + 1;
    hm.nv = dim + 1;
    hm.ld = (hm.nElem + 127) / 128 * 128;
    hm.model = model;
    hm.num = num;
    int nE = hm.nElem, nf = hm.nf, nv = hm.nv, ld = hm.ld;
    const int NFIELDS = dim == 2 ? GeoLayout<2>::NFIELDS : GeoLayout<3>::NFIELDS;
    const int JINV = 0, JAC = dim * dim, NRM = JAC + 1, JF = NRM + nf * dim, DL = JF + nf, X0 = DL + nf, JM = X0 + dim,
              SZ = JM + dim * dim, AR = SZ + 1;
    hm.geo.assign((size_t)NFIELDS * ld, 0.0);
    hm.tt.assign((size_t)nf * ld, -1);
    hm.fcode.assign((size_t)nf * ld, 0);
    hm.vwd.assign((size_t)nv * ld, 0.0);
    if (desc.mesh_velocity) hm.vu.assign((size_t)nv * dim * ld, 0.0);
    hm.area.assign(nE, 0);
    hm.elemSize.assign(nE, 0);
    hm.xs.assign((size_t)nE * dim, 0);
    const RefTables& t = hm.tab;
    double wsum = 0, wfsum = 0;
    for (int q = 0; q < t.nqv; q++) wsum += t.data[t.o_w + q];
    for (int p = 0; p < t.nqf; p++) wfsum += t.data[t.o_wf + p];
    auto G = [&](int f, int e) -> double& { return hm.geo[(size_t)f * ld + e]; };
    std::vector<double> Xes((size_t)nE * nf * dim);
    // pass 1: per element affine map, normals, centres
    for (int e = 0; e < nE; e++) {
        const int* tp = desc.elements + (size_t)e * nv;
        for (int v = 0; v < nv; v++)
            if (tp[v] < 0 || tp[v] >= desc.n_vertices) {
                err = "element vertex index out of range";
                return FP_ERR_ARG;
            }
        const double* x0 = desc.vertices + (size_t)tp[0] * dim;
        double J[9] = {0}, Ji[9] = {0};
        for (int i = 0; i < dim; i++)
            for (int j = 0; j < dim; j++) J[i * dim + j] = desc.vertices[(size_t)tp[j + 1] * dim + i] - x0[i];
        double det, jac;
        if (dim == 2) {
            det = J[0] * J[3] - J[1] * J[2];
            jac = std::fabs(det) / 2;
            Ji[0] = J[3] / det;
            Ji[1] = -J[1] / det;
            Ji[2] = -J[2] / det;
            Ji[3] = J[0] / det;
        } else {
            // |det| as transformation3Dtetra.jacobian (A = first row, B second, C third)
            const double *A = &J[0], *B = &J[3], *C = &J[6];
            det = A[0] * B[1] * C[2] + A[1] * B[2] * C[0] + A[2] * B[0] * C[1] - A[2] * B[1] * C[0] - A[1] * B[0] * C[2] -
                  A[0] * B[2] * C[1];
            jac = std::fabs(det);
            Ji[0] = (J[4] * J[8] - J[5] * J[7]) / det;
            Ji[1] = (J[2] * J[7] - J[1] * J[8]) / det;
            Ji[2] = (J[1] * J[5] - J[2] * J[4]) / det;
            Ji[3] = (J[5] * J[6] - J[3] * J[8]) / det;
            Ji[4] = (J[0] * J[8] - J[2] * J[6]) / det;
            Ji[5] = (J[2] * J[3] - J[0] * J[5]) / det;
            Ji[6] = (J[3] * J[7] - J[4] * J[6]) / det;
            Ji[7] = (J[1] * J[6] - J[0] * J[7]) / det;
            Ji[8] = (J[0] * J[4] - J[1] * J[3]) / det;
        }
        if (det == 0 || !std::isfinite(det)) {
            err = "degenerate element " + std::to_string(e);
            return FP_ERR_ARG;
        }
        // Jinv[d'][d] = (J^-1)[d'][d]: dphi/dx_d = sum_d' (J^-1)[d'][d] dphi/dxi_d' (Transformation.transformBasis)
        for (int i = 0; i < dim * dim; i++) G(JINV + i, e) = Ji[i];
        G(JAC, e) = jac;
        for (int i = 0; i < dim; i++) G(X0 + i, e) = x0[i];
        for (int i = 0; i < dim * dim; i++) G(JM + i, e) = J[i];
        auto getX = [&](const double* xi, double* X) {
            for (int i = 0; i < dim; i++) {
                double s = 0;
                for (int j = 0; j < dim; j++) s += J[i * dim + j] * xi[j];
                X[i] = s + x0[i];
            }
        };
        double xsr[3] = {dim == 2 ? 1.0 / 3 : 0.25, dim == 2 ? 1.0 / 3 : 0.25, dim == 2 ? 0.0 : 0.25};
        double Xs[3];
        getX(xsr, Xs);
        for (int d = 0; d < dim; d++) hm.xs[(size_t)e * dim + d] = Xs[d];
        double area = jac * wsum, Ssum = 0;
        for (int k = 0; k < nf; k++) {
            int fi[3];
            face_vertices(dim, k, fi);
            double nrm[3], jf;
            if (dim == 2) {
                double s[2] = {ref_vertex(2, fi[1])[0] - ref_vertex(2, fi[0])[0], ref_vertex(2, fi[1])[1] - ref_vertex(2, fi[0])[1]};
                double Js[2] = {J[0] * s[0] + J[1] * s[1], J[2] * s[0] + J[3] * s[1]};
                double L = std::sqrt(Js[0] * Js[0] + Js[1] * Js[1]);
                nrm[0] = Js[1] / L;
                nrm[1] = -Js[0] / L;
                jf = L / 2;
            } else {
                double s1[3], s2[3], J1[3], J2[3];
                for (int d = 0; d < 3; d++) {
                    s1[d] = ref_vertex(3, fi[1])[d] - ref_vertex(3, fi[0])[d];
                    s2[d] = ref_vertex(3, fi[2])[d] - ref_vertex(3, fi[0])[d];
                }
                for (int i = 0; i < 3; i++) {
                    J1[i] = J[i * 3] * s1[0] + J[i * 3 + 1] * s1[1] + J[i * 3 + 2] * s1[2];
                    J2[i] = J[i * 3] * s2[0] + J[i * 3 + 1] * s2[1] + J[i * 3 + 2] * s2[2];
                }
                double c[3] = {J2[1] * J1[2] - J2[2] * J1[1], J2[2] * J1[0] - J2[0] * J1[2], J2[0] * J1[1] - J2[1] * J1[0]};
                double L = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
                for (int d = 0; d < 3; d++) nrm[d] = c[d] / L;
                jf = L / 2;
            }
            for (int d = 0; d < dim; d++) G(NRM + k * dim + d, e) = nrm[d];
            G(JF + k, e) = jf;
            Ssum += jf * wfsum;
            // face centre (FaceTransformation.getXs)
            double xc[3] = {0, 0, 0};
            for (int i = 0; i < dim; i++)
                for (int d = 0; d < dim; d++) xc[d] += ref_vertex(dim, fi[i])[d] / dim;
            double Xe[3];
            getX(xc, Xe);
            for (int d = 0; d < dim; d++) Xes[((size_t)e * nf + k) * dim + d] = Xe[d];
        }
        G(SZ, e) = nf * area / Ssum;
        G(AR, e) = area;
        hm.area[e] = area;
        hm.elemSize[e] = nf * area / Ssum;
        for (int v = 0; v < nv; v++) {
            hm.vwd[(size_t)v * ld + e] = desc.wall_distance ? desc.wall_distance[tp[v]] : 0.0;
            if (desc.mesh_velocity)
                for (int d = 0; d < dim; d++) hm.vu[((size_t)v * dim + d) * ld + e] = desc.mesh_velocity[(size_t)tp[v] * dim + d];
        }
    }
    // pass 2: neighbours, face orientation codes, DDG distances
    for (int e = 0; e < nE; e++) {
        const int* tp = desc.elements + (size_t)e * nv;
        for (int k = 0; k < nf; k++) {
            int nb = desc.neighbors[(size_t)e * nf + k];
            hm.tt[(size_t)k * ld + e] = nb;
            double dl = 0;
            if (nb > -1) {
                if (nb >= nE || nb == e) {
                    err = "neighbour index out of range";
                    return FP_ERR_ARG;
                }
                int kr = -1;
                for (int s = 0; s < nf; s++)
                    if (desc.neighbors[(size_t)nb * nf + s] == e) {
                        kr = s;
                        break;
                    }
                if (kr < 0) {
                    err = "neighbour relation is not symmetric at element " + std::to_string(e);
                    return FP_ERR_ARG;
                }
                int fiL[3], fiR[3], gL[3], gR[3];
                face_vertices(dim, k, fiL);
                face_vertices(dim, kr, fiR);
                const int* tpr = desc.elements + (size_t)nb * nv;
                for (int i = 0; i < dim; i++) {
                    gL[i] = tp[fiL[i]];
                    gR[i] = tpr[fiR[i]];
                }
                int perm[3], pm = -1;
                bool okp = true;
                for (int j = 0; j < dim; j++) {
                    perm[j] = -1;
                    for (int i = 0; i < dim; i++)
                        if (gR[j] == gL[i]) perm[j] = i;
                    if (perm[j] < 0) okp = false;
                }
                if (okp)
                    for (int c = 0; c < nperm_of(dim); c++) {
                        const int* P = dim == 2 ? kPerm2[c] : kPerm3[c];
                        bool eq = true;
                        for (int j = 0; j < dim; j++) eq = eq && P[j] == perm[j];
                        if (eq) pm = c;
                    }
                if (pm < 0) {
                    err = "non-conforming face between elements " + std::to_string(e) + " and " + std::to_string(nb);
                    return FP_ERR_ARG;
                }
                hm.fcode[(size_t)k * ld + e] = kr * nperm_of(dim) + pm;
                for (int d = 0; d < dim; d++) dl += (hm.xs[(size_t)e * dim + d] - hm.xs[(size_t)nb * dim + d]) * G(NRM + k * dim + d, e);
            } else {
                for (int d = 0; d < dim; d++)
                    dl += (hm.xs[(size_t)e * dim + d] - Xes[((size_t)e * nf + k) * dim + d]) * G(NRM + k * dim + d, e);
            }
            G(DL + k, e) = std::fabs(dl);
        }
    }
    // face list of the face-based residual.  qmap[pm][p] is the neighbour's own face
    // quadrature point that coincides with the owner's point p when the neighbour's face
    // vertices are the owner's permuted by kPerm[pm] (symmetric rules always match).
    {
        Rule fr;
        simplex_rule(dim - 1, num.order, fr);
        const int np = nperm_of(dim), nqf = (int)fr.w.size();
        hm.qmap.assign((size_t)np * nqf, -1);
        hm.faceMode = true;
        for (int pm = 0; pm < np; pm++) {
            const int* perm = dim == 2 ? kPerm2[pm] : kPerm3[pm];
            for (int p = 0; p < nqf; p++) {
                double lp[3], lq[3];
                face_lambda(dim, fr, p, lp);
                for (int q = 0; q < nqf && hm.qmap[(size_t)pm * nqf + p] < 0; q++) {
                    face_lambda(dim, fr, q, lq);
                    bool same = std::fabs(fr.w[q] - fr.w[p]) < 1e-14;
                    for (int j = 0; j < dim; j++) same = same && std::fabs(lq[j] - lp[perm[j]]) < 1e-12;
                    if (same) hm.qmap[(size_t)pm * nqf + p] = q;
                }
                if (hm.qmap[(size_t)pm * nqf + p] < 0) hm.faceMode = false;
            }
        }
        hm.efc.assign((size_t)nf * ld, 0);
        hm.fl.clear();
        hm.fk.clear();
        hm.fr.clear();
        hm.fc.clear();
        for (int e = 0; e < nE; e++)
            for (int k = 0; k < nf; k++) {
                const int nb = desc.neighbors[(size_t)e * nf + k];
                if (nb > -1 && nb <= e) continue;  // owned by the lower-indexed element
                const int f = (int)hm.fl.size();
                const int code = nb > -1 ? hm.fcode[(size_t)k * ld + e] : 0;
                hm.fl.push_back(e);
                hm.fk.push_back(k);
                hm.fr.push_back(nb);
                hm.fc.push_back(code);
                hm.efc[(size_t)k * ld + e] = f << 1;
                if (nb > -1) hm.efc[(size_t)(code / np) * ld + nb] = (f << 1) | 1;
            }
        hm.nFaces = (int)hm.fl.size();
        hm.ldf = (hm.nFaces + 127) / 128 * 128;
        hm.fl.resize(hm.ldf, 0);
        hm.fk.resize(hm.ldf, 0);
        hm.fr.resize(hm.ldf, -1);
        hm.fc.resize(hm.ldf, 0);
    }
    // DOF ordering
    if (num.element_ordering == 1) {
        std::vector<int> ttE((size_t)nE * nf);
        for (int e = 0; e < nE; e++)
            for (int k = 0; k < nf; k++) ttE[(size_t)e * nf + k] = desc.neighbors[(size_t)e * nf + k];
        hm.order = reverse_cuthill_mckee(nE, nf, ttE.data());
    } else {
        hm.order.resize(nE);
        for (int i = 0; i < nE; i++) hm.order[i] = i;
    }
    hm.rank.assign(nE, 0);
    for (int r = 0; r < nE; r++) hm.rank[hm.order[r]] = r;
    return FP_OK;
}

// ---------------------------------------------------------------------------- ordering
// Reverse Cuthill-McKee of the face-neighbour graph; every connected component starts
// from a pseudo-peripheral element, neighbours visited by increasing degree (the same
// rules and tie-breaks as ElementOrdering.java:52-142, so the DOF numbering agrees).
std::vector<int> reverse_cuthill_mckee(int n, int nf, const int* tt) {
    std::vector<std::vector<int>> adj(n);
    std::vector<int> degree(n);
    for (int i = 0; i < n; i++) {
        for (int k = 0; k < nf; k++) {
            int t = tt[(size_t)i * nf + k];
            if (t > -1 && t != i && std::find(adj[i].begin(), adj[i].end(), t) == adj[i].end()) adj[i].push_back(t);
        }
        degree[i] = (int)adj[i].size();
    }
    for (int i = 0; i < n; i++)
        std::stable_sort(adj[i].begin(), adj[i].end(), [&](int a, int b) { return degree[a] < degree[b]; });
    auto peripheral = [&](const std::vector<char>& excluded, int start) {
        int node = start, ecc = -1;
        std::vector<int> level(n);
        for (int iter = 0; iter < 10; iter++) {
            std::fill(level.begin(), level.end(), -1);
            std::deque<int> q{node};
            level[node] = 0;
            int last = node;
            while (!q.empty()) {
                int e = q.front();
                q.pop_front();
                for (int t : adj[e])
                    if (!excluded[t] && level[t] == -1) {
                        level[t] = level[e] + 1;
                        q.push_back(t);
                        if (level[t] > level[last] || (level[t] == level[last] && adj[t].size() < adj[last].size())) last = t;
                    }
            }
            if (level[last] <= ecc) break;
            ecc = level[last];
            node = last;
        }
        return node;
    };
    std::vector<int> order(n);
    std::vector<char> visited(n, 0);
    int count = 0;
    while (count < n) {
        int start = -1;
        for (int i = 0; i < n; i++)
            if (!visited[i] && (start == -1 || degree[i] < degree[start])) start = i;
        start = peripheral(visited, start);
        std::deque<int> q{start};
        visited[start] = 1;
        while (!q.empty()) {
            int e = q.front();
            q.pop_front();
            order[count++] = e;
            for (int t : adj[e])
                if (!visited[t]) {
                    visited[t] = 1;
                    q.push_back(t);
                }
        }
    }
    std::reverse(order.begin(), order.end());
    return order;
}

// ---------------------------------------------------------------------------- neighbours
// Neighbour matrix from elements and boundary rows: two elements sharing a face (same
// vertex set) are neighbours; a face found in the boundary list takes its code, any other
// unmatched face -1 (FlowProMain.createNeighborMatrix, FlowProMain.java:772-873).
int create_neighbor_matrix(int dim, int nElem, const int* elements, int nBound, const int* boundary, int* tt) {
    int nv = dim + 1, nf = dim + 1, nvf = dim;
    struct Key {
        int v[3];
        bool operator==(const Key& o) const { return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2]; }
    };
    struct H {
        size_t operator()(const Key& k) const {
            uint64_t h = 1469598103934665603ULL;
            for (int i = 0; i < 3; i++) {
                h ^= (uint64_t)(uint32_t)k.v[i];
                h *= 1099511628211ULL;
            }
            return (size_t)h;
        }
    };
    auto key = [&](const int* vs) {
        Key k{{-1, -1, -1}};
        for (int i = 0; i < nvf; i++) k.v[i] = vs[i];
        std::sort(k.v, k.v + nvf);
        return k;
    };
    std::unordered_map<Key, std::pair<int, int>, H> faces;
    faces.reserve((size_t)nElem * nf);
    for (int i = 0; i < nElem; i++)
        for (int k = 0; k < nf; k++) {
            int fi[3], vs[3];
            face_vertices(dim, k, fi);
            for (int j = 0; j < nvf; j++) vs[j] = elements[(size_t)i * nv + fi[j]];
            auto it = faces.find(key(vs));
            if (it == faces.end())
                faces.emplace(key(vs), std::make_pair(i, -1000));
            else
                it->second.second = i;
        }
    std::unordered_map<Key, int, H> bnd;
    for (int b = 0; b < nBound; b++) bnd[key(boundary + (size_t)b * (nvf + 1) + 1)] = boundary[(size_t)b * (nvf + 1)];
    for (int i = 0; i < nElem; i++)
        for (int k = 0; k < nf; k++) {
            int fi[3], vs[3];
            face_vertices(dim, k, fi);
            for (int j = 0; j < nvf; j++) vs[j] = elements[(size_t)i * nv + fi[j]];
            Key kk = key(vs);
            auto& f = faces[kk];
            int r = -1000;
            if (f.first == i) {
                if (f.second != -1000) r = f.second;
            } else {
                r = f.first;
            }
            if (r == -1000) {
                auto it = bnd.find(kk);
                r = it != bnd.end() ? it->second : -1;
            }
            tt[(size_t)i * nf + k] = r;
        }
    return FP_OK;
}

// ---------------------------------------------------------------------------- model parameters
namespace {
using Props = std::map<std::string, std::string>;
// "key = value" entries separated by ';' or by line breaks (a parameters.txt file as
// java.util.Properties reads it, FlowProProperties.load, FlowProProperties.java:49-60); a value
// loses everything from '%' on (FlowProProperties.loseComments), so "%key = ..." lines and
// comment lines define no key, and "key =  % comment" defines key with an empty value
Props parse(const char* s) {
    Props p;
    std::string text(s ? s : "");
    for (char& c : text)
        if (c == '\n' || c == '\r') c = ';';
    std::stringstream ss(text);
    std::string item;
    auto trim = [](std::string x) {
        size_t a = x.find_first_not_of(" \t\r\n"), b = x.find_last_not_of(" \t\r\n");
        return a == std::string::npos ? std::string() : x.substr(a, b - a + 1);
    };
    while (std::getline(ss, item, ';')) {
        auto c = item.find('%');  // parameters.txt comments
        if (c != std::string::npos) item = item.substr(0, c);
        auto eq = item.find('=');
        if (eq == std::string::npos) continue;
        p[trim(item.substr(0, eq))] = trim(item.substr(eq + 1));
    }
    return p;
}
bool has(const Props& p, const char* k) { return p.count(k) > 0; }
double D(const Props& p, const char* k) { return std::atof(p.at(k).c_str()); }
bool B(const Props& p, const char* k) { return p.at(k) == "true" || p.at(k) == "1"; }
std::vector<double> DA(const Props& p, const char* k) {
    std::string s = p.at(k);
    for (char& c : s)
        if (c == ',') c = ' ';
    std::istringstream is(s);
    std::vector<double> v;
    double x;
    while (is >> x) v.push_back(x);
    return v;
}
double ssp_ratio(double kapa, double mach) { return std::pow(1 + (kapa - 1) / 2 * mach * mach, kapa / (kapa - 1)); }
double ssd_ratio(double kapa, double mach) { return std::pow(1 + (kapa - 1) / 2 * mach * mach, 1 / (kapa - 1)); }
}  // namespace

// Aerodynamics.init (Aerodynamics.java:119-312), NavierStokes.init, SpalartAllmaras.init
// (SpalartAllmaras.java:35-60), TestScalarEquation.init, and the hot-path keys of
// Parameters (Parameters.java:160-280).
int model_from_properties(const char* props, fp_model_params& m, fp_num_params& n, std::string& err) {
    try {
        Props p = parse(props);
        m = fp_model_params{};
        n = fp_num_params{};
        std::string model = has(p, "model") ? p.at("model") : "";
        m.dim = has(p, "dimension") ? (int)D(p, "dimension") : 2;
        n.order = has(p, "order") ? (int)D(p, "order") : 2;
        n.penalty = has(p, "penalty") ? D(p, "penalty") : 0;
        n.beta0 = has(p, "beta0") ? D(p, "beta0") : 2;
        n.damp_tol = has(p, "dampTol") ? D(p, "dampTol") : 0;
        n.damp_const = has(p, "dampConst") ? D(p, "dampConst") : 0;
        n.positivity_limiter = has(p, "positivityLimiter") ? (B(p, "positivityLimiter") ? 1 : 0) : 1;
        n.implicit_time = has(p, "timeMethod") && p.at("timeMethod") == "RK" ? 0 : 1;
        n.element_ordering = has(p, "elementOrdering") && p.at("elementOrdering") == "none" ? 0 : 1;
        n.fd_step = 1e-8;
        n.gcl = has(p, "gcl") && B(p, "gcl") ? 1 : 0;
        if (model == "TestScalarEquation") {
            m.model = FP_MODEL_SCALAR_TEST;
            m.n_eqs = 1;
            std::vector<double> a = DA(p, "a");
            double s = 0;
            for (size_t i = 0; i < a.size() && i < 3; i++) {
                m.a[i] = a[i];
                s += a[i] * a[i];
            }
            m.lambda = std::sqrt(s);
            m.k_diff = has(p, "k") ? D(p, "k") : 0;
            m.is_diffusive = m.k_diff > 0;
        } else if (model == "NavierStokes" || model == "SpalartAllmaras" || model == "AdiabaticEulers") {
            bool sa = model == "SpalartAllmaras", ad = model == "AdiabaticEulers";
            m.model = sa ? FP_MODEL_SPALART_ALLMARAS : (ad ? FP_MODEL_ADIABATIC_EULERS : FP_MODEL_NAVIER_STOKES);
            m.n_eqs = m.dim + (sa ? 3 : (ad ? 1 : 2));
            m.is_diffusive = sa ? 1 : (ad ? 0 : (B(p, "isFlowViscous") ? 1 : 0));
            double kapa, cp, cv;
            if (has(p, "kappa") && has(p, "cv") && !has(p, "cp")) {
                kapa = D(p, "kappa");
                cv = D(p, "cv");
                cp = cv * kapa;
            } else if (has(p, "kappa") && has(p, "cp") && !has(p, "cv")) {
                kapa = D(p, "kappa");
                cp = D(p, "cp");
                cv = cp / kapa;
            } else if (has(p, "cv") && has(p, "cp") && !has(p, "kappa")) {
                cp = D(p, "cp");
                cv = D(p, "cv");
                kapa = cp / cv;
            } else {
                err = "exactly two out of the three following parameters must be defined: kappa, cp, cv";
                return FP_ERR_ARG;
            }
            m.kappa = kapa;
            m.p_in0 = 1;
            m.rho_in0 = 1;
            m.inlet_supersonic = has(p, "isInletSupersonic") && B(p, "isInletSupersonic");
            if (ad && m.inlet_supersonic) {
                // Aerodynamics.init writes the energy of the inlet state (index dim + 1), which
                // the dim + 1 equations of AdiabaticEulers do not have
                err = "AdiabaticEulers with a supersonic inlet is not supported";
                return FP_ERR_UNSUPPORTED;
            }
            double pRef, rhoRef;
            if (m.inlet_supersonic) {
                pRef = D(p, "pIn");
                rhoRef = has(p, "rhoIn") ? D(p, "rhoIn") : pRef / (cv * (kapa - 1) * D(p, "TIn"));
            } else {
                bool ff = has(p, "pInf") && has(p, "machInf") && (has(p, "TInf") != has(p, "rhoInf"));
                bool st = has(p, "pIn0") && has(p, "pOut") && (has(p, "TIn0") != has(p, "rhoIn0"));
                if (ff && !st) {
                    double pInf = D(p, "pInf"), machInf = D(p, "machInf");
                    double rhoInf = has(p, "rhoInf") ? D(p, "rhoInf") : pInf / (cv * (kapa - 1) * D(p, "TInf"));
                    pRef = pInf * ssp_ratio(kapa, machInf);
                    rhoRef = rhoInf * ssd_ratio(kapa, machInf);
                    m.p_out = m.p_in0 / ssp_ratio(kapa, machInf);
                } else if (st && !ff) {
                    pRef = D(p, "pIn0");
                    rhoRef = has(p, "rhoIn0") ? D(p, "rhoIn0") : pRef / (cv * (kapa - 1) * D(p, "TIn0"));
                    m.p_out = D(p, "pOut") / pRef;
                } else {
                    err = "either stagnation (pOut, pIn0 and rhoIn0 or TIn0) or far-field (machInf, pInf and rhoInf or TInf) boundary conditions must be prescribed";
                    return FP_ERR_ARG;
                }
            }
            double velocityRef = std::sqrt(pRef / rhoRef);
            if (has(p, "attackAngle")) {
                std::vector<double> a = DA(p, "attackAngle");
                if ((int)a.size() != m.dim - 1) {
                    err = "variable attackAngle must be a vector of dimension - 1 entries";
                    return FP_ERR_ARG;
                }
                m.has_attack_angle = 1;
                for (size_t i = 0; i < a.size(); i++) m.attack_angle[i] = a[i];
            }
            if (m.inlet_supersonic) {
                double vIn = D(p, "vIn") / velocityRef;
                double v[3] = {0, 0, 0};
                if (m.dim == 2) {
                    v[0] = vIn * std::cos(m.attack_angle[0]);
                    v[1] = vIn * std::sin(m.attack_angle[0]);
                }
                m.w_in[0] = 1;
                for (int d = 0; d < m.dim; d++) m.w_in[d + 1] = v[d];
                double v2 = 0;
                for (int d = 0; d < m.dim; d++) v2 += v[d] * v[d];
                m.w_in[3] = 1 / (kapa - 1) + 0.5 * v2;  // Aerodynamics.java:250-257 writes index 3
            } else {
                m.w_in[0] = -1;
            }
            if (m.is_diffusive) {
                double machInf = std::sqrt(2 / (kapa - 1) * (std::pow((m.p_in0 / m.p_out), (kapa - 1) / kapa) - 1));
                double rhoInf = rhoRef / ssd_ratio(kapa, machInf);
                double pInf = pRef / ssp_ratio(kapa, machInf);
                double uInf = machInf * std::sqrt(kapa * pInf / rhoInf);
                if (has(p, "reynolds") && has(p, "prandtl") && !has(p, "viscosity") && !has(p, "conductivity")) {
                    m.Re = D(p, "reynolds") * (rhoRef * velocityRef) / (rhoInf * uInf);
                    m.Pr = D(p, "prandtl");
                } else if (has(p, "viscosity") && has(p, "conductivity")) {
                    double mu = D(p, "viscosity");
                    m.Pr = cp * mu / D(p, "conductivity");
                    double lRef = has(p, "lRef") ? D(p, "lRef") : 1;
                    m.Re = rhoRef * velocityRef * lRef / mu;
                } else {
                    err = "either the Prandtl and Reynolds numbers, or dynamic viscosity and thermal conductivity must be specified";
                    return FP_ERR_ARG;
                }
            } else {
                m.Re = -1;
                m.Pr = -1;
            }
            m.numerical_flux = has(p, "numericalFlux") && p.at("numericalFlux") == "vanLeer" ? 1 : 0;
            if (sa) {
                m.vt_in = D(p, "vtIn");
                if (m.inlet_supersonic) m.w_in[m.dim + 2] = m.vt_in;
                m.sigma = D(p, "sigma");
                m.cb1 = D(p, "cb1");
                m.cb2 = D(p, "cb2");
                m.ka = D(p, "ka");
                m.cw1 = m.cb1 / (m.ka * m.ka) + (1 + m.cb2) / m.sigma;
                m.cw2 = D(p, "cw2");
                m.cw3 = D(p, "cw3");
                m.cv1 = D(p, "cv1");
                m.prt = D(p, "Prt");
            }
        } else {
            err = "unsupported model '" + model +
                  "' (no CPU fallback): NavierStokes, SpalartAllmaras, AdiabaticEulers, TestScalarEquation";
            return FP_ERR_UNSUPPORTED;
        }
    } catch (std::exception& ex) {
        err = std::string("bad parameter: ") + ex.what();
        return FP_ERR_ARG;
    }
    return FP_OK;
}

// constInitCondition (NavierStokes.java:98-139, SpalartAllmaras.java:88-127,
// AdiabaticEulers.java:97-133, TestScalarEquation: 0)
void const_init_condition(const fp_model_params& m, double* W) {
    int dim = m.dim;
    for (int i = 0; i < m.n_eqs; i++) W[i] = 0;
    if (m.model == FP_MODEL_SCALAR_TEST) return;
    if (m.inlet_supersonic) {
        for (int i = 0; i < m.n_eqs; i++) W[i] = m.w_in[i];
        return;
    }
    double kapa = m.kappa, pOut = m.p_out;
    double machIn = std::sqrt(2 / (kapa - 1) * (std::pow((1 / pOut), (kapa - 1) / kapa) - 1));
    if (m.model == FP_MODEL_ADIABATIC_EULERS) {
        // AdiabaticEulers.constInitCondition, AdiabaticEulers.java:97-133
        double rhoIn = std::pow(1 + ((kapa - 1) / 2) * machIn * machIn, 1 / (1 - kapa));
        double VIn = machIn * std::sqrt((kapa * pOut) / rhoIn);
        double alpha = m.has_attack_angle ? m.attack_angle[0] : 0, beta = (m.has_attack_angle && dim == 3) ? m.attack_angle[1] : 0;
        double v[3] = {0, 0, 0};
        if (dim == 2) {
            v[0] = VIn * std::cos(alpha);
            v[1] = VIn * std::sin(alpha);
        } else {
            v[0] = VIn * std::cos(alpha) * std::cos(beta);
            v[1] = VIn * std::sin(alpha) * std::cos(beta);
            v[2] = VIn * std::sin(beta);
        }
        W[0] = rhoIn;
        for (int d = 0; d < dim; d++) W[d + 1] = rhoIn * v[d];
        return;
    }
    double rhoIn = std::pow(1 + ((kapa - 1) / 2) * machIn * machIn, 1 / (1 - kapa));
    double VIn = machIn * std::sqrt((kapa * pOut) / rhoIn);
    double alpha = m.has_attack_angle ? m.attack_angle[0] : 0, beta = (m.has_attack_angle && dim == 3) ? m.attack_angle[1] : 0;
    double v[3] = {0, 0, 0};
    if (dim == 2) {
        v[0] = VIn * std::cos(alpha);
        v[1] = VIn * std::sin(alpha);
    } else {
        v[0] = VIn * std::cos(alpha) * std::cos(beta);
        v[1] = VIn * std::sin(alpha) * std::cos(beta);
        v[2] = VIn * std::sin(beta);
    }
    W[0] = rhoIn;
    for (int d = 0; d < dim; d++) W[d + 1] = rhoIn * v[d];
    W[dim + 1] = pOut / (kapa - 1) + 0.5 * rhoIn * VIn * VIn;
    if (m.model == FP_MODEL_SPALART_ALLMARAS) W[dim + 2] = rhoIn * m.vt_in;
}

}  // namespace fp
