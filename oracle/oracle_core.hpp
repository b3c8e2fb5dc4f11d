// CPU ORACLE — test infrastructure only (never linked into the product library).
//
// A line-faithful C++ restatement of FlowPro's DG residual and implicit-solve
// hot path, written from the Java sources of ondrabublik/FlowPro_v2.  Every
// function cites the Java file:line it follows (paths relative to the FlowPro
// checkout).  It is compiled with -O2 -ffp-contract=off (Java does not contract
// FMAs) and is used by tests/, bench.py (cpu_baseline / --impl reference) and
// __graft_entry__.smoke() as the checker.
//
// Parity pins (what ties this restatement to the reference itself):
//   * createNeighborMatrix is checked bit-exactly against the shipped
//     FlowPro/simulations/examples/GAMM/mesh/neighbors.txt (tests/golden);
//   * the reference's own ConvergenceOrderTest, LinearSolverTest and
//     JacobianTest (FlowPro/src/test/java/flowpro/core/*) are re-run against
//     this oracle with the same meshes, seeds (java.util.Random LCG) and
//     tolerances;
//   * the quadrature tables are FlowPro's gaussRules files.
// There are no golden residual vectors for the Euler/NS/SA models in the
// reference (its tests do not cover them) and no JDK here to run the Java, so
// per-model residual values are "parity unpinned" beyond those checks.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <limits>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../flowpro_v2_b200/csrc/gauss_rules.h"

namespace orc {

using Vec = std::vector<double>;
using Mat2 = std::vector<Vec>;
using IVec = std::vector<int>;

static inline Mat2 zeros(int m, int n) { return Mat2(m, Vec(n, 0.0)); }

// ---------------------------------------------------------------- Mat (FlowProAPI/src/main/java/flowpro/api/Mat.java)
// Mat.linspace, Mat.java:42-53
static Vec linspace(double a, double b, int n) {
    Vec x(n);
    if (n == 1) {
        x[0] = (a + b) / 2;
    } else {
        for (int i = 0; i < n; i++) {
            double xi = (double)i / (n - 1);
            x[i] = (1 - xi) * a + xi * b;
        }
    }
    return x;
}

// Mat.gaussian, Mat.java:502-556 (scaled partial pivoting, in place)
static IVec gaussian(Mat2& A) {
    int n = (int)A.size();
    IVec index(n);
    Vec c(n);
    for (int i = 0; i < n; ++i) index[i] = i;
    for (int i = 0; i < n; ++i) {
        double c1 = 0;
        for (int j = 0; j < n; ++j) {
            double c0 = std::fabs(A[i][j]);
            if (c0 > c1) c1 = c0;
        }
        c[i] = c1;
    }
    for (int j = 0; j < n - 1; ++j) {
        int k = j;
        double pi1 = 0;
        for (int i = j; i < n; ++i) {
            double pi0 = std::fabs(A[index[i]][j]);
            pi0 /= c[index[i]];
            if (pi0 > pi1) {
                pi1 = pi0;
                k = i;
            }
        }
        int itmp = index[j];
        index[j] = index[k];
        index[k] = itmp;
        for (int i = j + 1; i < n; ++i) {
            double pj = A[index[i]][j] / A[index[j]][j];
            A[index[i]][j] = pj;
            for (int l = j + 1; l < n; ++l) A[index[i]][l] -= pj * A[index[j]][l];
        }
    }
    return index;
}

// Mat.invert, Mat.java:605-642
static Mat2 invert(const Mat2& A) {
    int n = (int)A.size();
    Mat2 invA = A;
    Mat2 x = zeros(n, n), b = zeros(n, n);
    for (int i = 0; i < n; ++i) b[i][i] = 1;
    IVec index = gaussian(invA);
    for (int i = 0; i < n - 1; ++i)
        for (int j = i + 1; j < n; ++j)
            for (int k = 0; k < n; ++k) b[index[j]][k] -= invA[index[j]][i] * b[index[i]][k];
    for (int i = 0; i < n; ++i) {
        x[n - 1][i] = b[index[n - 1]][i] / invA[index[n - 1]][n - 1];
        for (int j = n - 2; j >= 0; --j) {
            x[j][i] = b[index[j]][i];
            for (int k = j + 1; k < n; ++k) x[j][i] -= invA[index[j]][k] * x[k][i];
            x[j][i] /= invA[index[j]][j];
        }
    }
    return x;
}

static Vec times(const Mat2& A, const Vec& x) {
    Vec y(A.size(), 0.0);
    for (size_t i = 0; i < A.size(); i++)
        for (size_t j = 0; j < x.size(); j++) y[i] += A[i][j] * x[j];
    return y;
}

static Mat2 times(const Mat2& A, const Mat2& B) {
    int m = (int)A.size(), n = (int)B[0].size(), K = (int)B.size();
    Mat2 C = zeros(m, n);
    for (int i = 0; i < m; i++)
        for (int j = 0; j < n; j++)
            for (int k = 0; k < K; k++) C[i][j] += A[i][k] * B[k][j];
    return C;
}

static Mat2 transpose(const Mat2& A) {
    int m = (int)A.size(), n = (int)A[0].size();
    Mat2 B = zeros(n, m);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < m; ++j) B[i][j] = A[j][i];
    return B;
}

static double L2Norm(const Vec& v) {
    double s = 0;
    for (double x : v) s += x * x;
    return std::sqrt(s);
}

static Vec normVector(const Vec& v) {
    double nrm = L2Norm(v);
    Vec s(v.size());
    for (size_t i = 0; i < v.size(); i++) s[i] = v[i] / nrm;
    return s;
}

static Vec cross(const Vec& a, const Vec& b) {
    return Vec{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}

// Mat.lsolveT, Mat.java:1307-1329 — Gaussian elimination (no pivoting) of A^T,
// overwrites A (the in-place quirk used by blockJacobi).
static Vec lsolveT(Mat2& A, Vec& b) {
    int n = (int)b.size();
    for (int p = 0; p < n; p++)
        for (int i = p + 1; i < n; i++) {
            double alpha = A[p][i] / A[p][p];
            b[i] -= alpha * b[p];
            for (int j = p; j < n; j++) A[j][i] -= alpha * A[j][p];
        }
    Vec x(n);
    for (int i = n - 1; i >= 0; i--) {
        double sum = 0.0;
        for (int j = i + 1; j < n; j++) sum += A[j][i] * x[j];
        x[i] = (b[i] - sum) / A[i][i];
    }
    return x;
}

// java.util.Random (LCG, nextDouble) — used by the reference tests for seeded states.
struct JavaRandom {
    uint64_t seed;
    explicit JavaRandom(int64_t s) { seed = ((uint64_t)s ^ 0x5DEECE66DULL) & ((1ULL << 48) - 1); }
    int next(int bits) {
        seed = (seed * 0x5DEECE66DULL + 0xBULL) & ((1ULL << 48) - 1);
        return (int)(int64_t)(seed >> (48 - bits));
    }
    double nextDouble() { return (double)(((int64_t)next(26) << 27) + next(27)) * (1.0 / (double)(1ULL << 53)); }
};

// ---------------------------------------------------------------- quadrature
// flowpro/core/quadrature/Quadrature*.java: coords and weights
struct Quadrature {
    int nPoints = 0;
    Mat2 coords;
    Vec weights;
};

static Quadrature loadRule(int kind, int key) {
    for (int r = 0; r < fpr::kNumRules; r++) {
        const auto& e = fpr::kRules[r];
        if (e.kind == kind && e.key == key) {
            Quadrature q;
            q.nPoints = e.n;
            q.weights.assign(e.w, e.w + e.n);
            q.coords = zeros(e.n, kind);
            for (int i = 0; i < e.n; i++)
                for (int d = 0; d < kind; d++) q.coords[i][d] = e.pts[i * kind + d];
            return q;
        }
    }
    throw std::runtime_error("quadrature rule not available");
}

// QuadratureCentral.java:46-91 (line: k points; triangle/tetra: degree 2k-1, triangle
// bumped to 2k when the rule of degree 2k-1 has a negative weight)
struct QuadratureCentral {
    Quadrature line(int order) const { return loadRule(1, order); }
    Quadrature tri(int order) const {
        Quadrature q = loadRule(2, 2 * order - 1);
        for (double w : q.weights)
            if (w < 0) return loadRule(2, 2 * order);
        return q;
    }
    Quadrature tet(int order) const { return loadRule(3, 2 * order - 1); }
};

// ---------------------------------------------------------------- bases
struct Basis {
    int nBasis = 0;
    virtual ~Basis() {}
    virtual double basisFun(int m, const Vec& Xi) const = 0;
    virtual double derBasis(int m, const Vec& Xi, int d) const = 0;
    // Basis.getBasisXi / getDerBasisXi, basis/Basis.java:19-41
    Mat2 getBasisXi(const Mat2& c) const {
        Mat2 b = zeros((int)c.size(), nBasis);
        for (size_t p = 0; p < c.size(); p++)
            for (int m = 0; m < nBasis; m++) b[p][m] = basisFun(m, c[p]);
        return b;
    }
    std::vector<Mat2> getDerBasisXi(const Mat2& c, int dim) const {
        std::vector<Mat2> db(c.size(), zeros(nBasis, dim));
        for (int d = 0; d < dim; d++)
            for (size_t p = 0; p < c.size(); p++)
                for (int m = 0; m < nBasis; m++) db[p][m][d] = derBasis(m, c[p], d);
        return db;
    }
};

// basis/basis2Dtriangle.java:22-119
struct Basis2DTri : Basis {
    int order;
    IVec xExp, yExp;
    Mat2 coeffs;
    explicit Basis2DTri(int order_) : order(order_) {
        nBasis = order * (1 + order) / 2;
        xExp.assign(order * order, 0);
        yExp.assign(order * order, 0);
        int s = 0;
        for (int i = 0; i < order; i++)
            for (int j = 0; j <= i; j++) {
                xExp[s] = i - j;
                yExp[s] = j;
                ++s;
            }
        for (int i = order - 1; i > 0; i--)
            for (int j = 0; j < i; j++) {
                xExp[s] = order - 1 - j;
                yExp[s] = order - i + j;
                ++s;
            }
        calculateCoefficients();
    }
    Mat2 barycentr(int rad, int ne) const {
        Mat2 b;
        if (rad == 1) {
            b = Mat2{{1.0 / 3, 1.0 / 3, 1.0 / 3}};
        } else {
            Vec x = linspace(0, 1, rad);
            b = zeros(ne, 3);
            int s = 0;
            for (int i = 0; i < rad; i++) {
                Vec y = linspace(0, x[i], i + 1);
                for (int j = 0; j < i + 1; j++) {
                    b[s][0] = 1 - x[i];
                    b[s][1] = y[j];
                    b[s][2] = x[i] - y[j];
                    s++;
                }
            }
        }
        return b;
    }
    void calculateCoefficients() {
        if (order == 1) {
            coeffs = Mat2{{1.0}};
        } else {
            Mat2 b = barycentr(order, nBasis);
            Mat2 V = zeros(nBasis, nBasis);
            for (int i = 0; i < nBasis; i++) {
                double X0 = b[i][1], X1 = b[i][2];
                for (int j = 0; j < nBasis; j++) V[i][j] = std::pow(X0, xExp[j]) * std::pow(X1, yExp[j]);
            }
            coeffs = invert(V);
        }
    }
    double basisFun(int m, const Vec& Xi) const override {
        double val = 0;
        for (int i = 0; i < nBasis; i++)
            val = val + coeffs[i][m] * std::pow(Xi[0], xExp[i]) * std::pow(Xi[1], yExp[i]);
        return val;
    }
    double derBasis(int m, const Vec& Xi, int dim) const override {
        double der = 0;
        if (dim == 0) {
            for (int i = 0; i < nBasis; i++)
                if (xExp[i] > 0)
                    der = der + coeffs[i][m] * xExp[i] * std::pow(Xi[0], xExp[i] - 1) * std::pow(Xi[1], yExp[i]);
        } else {
            for (int i = 0; i < nBasis; i++)
                if (yExp[i] > 0)
                    der = der + coeffs[i][m] * yExp[i] * std::pow(Xi[0], xExp[i]) * std::pow(Xi[1], yExp[i] - 1);
        }
        return der;
    }
};

// basis/basis3Dtetra.java:23-108.  Deviation: for order 3 (p = 2) the Java
// barycentr() returns only the 4 vertices (basis3Dtetra.java:50-62) and the
// Vandermonde build then indexes past them; this restatement completes the P2
// Lagrange node set with the 6 edge midpoints (01, 02, 03, 12, 13, 23).
struct Basis3DTet : Basis {
    int order;
    IVec xExp{0, 1, 0, 0, 1, 1, 0, 2, 0, 0, 2, 2, 1, 0, 1, 0, 3, 0, 0};
    IVec yExp{0, 0, 1, 0, 1, 0, 1, 0, 2, 0, 1, 0, 2, 2, 0, 1, 0, 3, 0};
    IVec zExp{0, 0, 0, 1, 0, 1, 1, 0, 0, 2, 0, 1, 0, 1, 2, 2, 0, 0, 3};
    Mat2 coeffs;
    explicit Basis3DTet(int order_) : order(order_) {
        nBasis = (3 * (order - 1) * order + 2) / 2;
        if (order > 3) throw std::runtime_error("tetrahedral basis supports order <= 3");
        if (order == 1) {
            coeffs = Mat2{{1.0}};
        } else {
            Mat2 b{{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}};
            if (order == 3) {
                int e[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
                for (auto& ed : e) {
                    Vec r(4, 0.0);
                    r[ed[0]] = 0.5;
                    r[ed[1]] = 0.5;
                    b.push_back(r);
                }
            }
            Mat2 V = zeros(nBasis, nBasis);
            for (int i = 0; i < nBasis; i++) {
                double X0 = b[i][1], X1 = b[i][2], X2 = b[i][3];
                for (int j = 0; j < nBasis; j++)
                    V[i][j] = std::pow(X0, xExp[j]) * std::pow(X1, yExp[j]) * std::pow(X2, zExp[j]);
            }
            coeffs = invert(V);
        }
    }
    double basisFun(int m, const Vec& Xi) const override {
        double val = 0;
        for (int i = 0; i < nBasis; i++)
            val = val + coeffs[i][m] * std::pow(Xi[0], xExp[i]) * std::pow(Xi[1], yExp[i]) * std::pow(Xi[2], zExp[i]);
        return val;
    }
    double derBasis(int m, const Vec& Xi, int dim) const override {
        double r = 0;
        for (int i = 0; i < nBasis; i++) {
            int ex[3] = {xExp[i], yExp[i], zExp[i]};
            if (ex[dim] > 0) {
                double t = coeffs[i][m] * ex[dim];
                for (int d = 0; d < 3; d++) t = t * std::pow(Xi[d], d == dim ? ex[d] - 1 : ex[d]);
                r = r + t;
            }
        }
        return r;
    }
};

// ---------------------------------------------------------------- transformations
struct Transformation {
    Mat2 coordsX, coordsXi;
    virtual ~Transformation() {}
    virtual Vec getX(const Vec& Xi) const = 0;
    virtual Vec getXi(const Vec& X) const = 0;
    virtual double getDX(const Vec& Xi, int top, int bottom) const = 0;
    virtual double jacobian(const Vec& Xi) const = 0;
    virtual Mat2 getInterpolant(const Quadrature& q) const = 0;
    virtual Vec getXs() const = 0;
    // Transformation.jacobiMatrix / jacobian(quad) / jacobianMatrixDirection / transformBasis,
    // transformation/Transformation.java:235-283
    Mat2 jacobiMatrix(const Vec& Xi) const {
        int dim = (int)Xi.size();
        Mat2 J = zeros(dim, dim);
        for (int i = 0; i < dim; i++)
            for (int j = 0; j < dim; j++) J[i][j] = getDX(Xi, i, j);
        return J;
    }
    Vec jacobian(const Quadrature& q) const {
        Vec J(q.nPoints);
        for (int i = 0; i < q.nPoints; i++) J[i] = jacobian(q.coords[i]);
        return J;
    }
    Vec jacobianMatrixDirection(const Vec& Xi, const Vec& s) const {
        Mat2 J = jacobiMatrix(Xi);
        Vec Js(Xi.size(), 0.0);
        for (size_t i = 0; i < Xi.size(); i++)
            for (size_t j = 0; j < Xi.size(); j++) Js[i] += J[i][j] * s[j];
        return Js;
    }
    std::vector<Mat2> transformBasis(const Mat2& cXi, const std::vector<Mat2>& dXi) const {
        int nP = (int)dXi.size(), nB = (int)dXi[0].size(), dim = (int)dXi[0][0].size();
        std::vector<Mat2> dX(nP, zeros(nB, dim));
        for (int p = 0; p < nP; p++) {
            Mat2 iT = invert(jacobiMatrix(cXi[p]));
            for (int m = 0; m < nB; m++)
                for (int i = 0; i < dim; i++)
                    for (int j = 0; j < dim; j++) dX[p][m][i] += iT[j][i] * dXi[p][m][j];
        }
        return dX;
    }
    Mat2 getX(const Mat2& Xi) const {
        Mat2 X;
        for (auto& x : Xi) X.push_back(getX(x));
        return X;
    }
    Mat2 getXi(const Mat2& X) const {
        Mat2 Xi;
        for (auto& x : X) Xi.push_back(getXi(x));
        return Xi;
    }
};

// transformation/transformation2Dtriangle.java:14-119
struct Transformation2DTri : Transformation {
    Vec A, B, iA, iB;
    Mat2 invV, invVi;
    explicit Transformation2DTri(const Mat2& vertices) {
        coordsXi = Mat2{{0, 0}, {1, 0}, {0, 1}};
        coordsX = vertices;
        Mat2 V = zeros(3, 3);
        for (int i = 0; i < 3; i++) {
            V[i][0] = coordsXi[i][0];
            V[i][1] = coordsXi[i][1];
            V[i][2] = 1;
        }
        invV = invert(V);
        Mat2 Vi = zeros(3, 3);
        for (int i = 0; i < 3; i++) {
            Vi[i][0] = coordsX[i][0];
            Vi[i][1] = coordsX[i][1];
            Vi[i][2] = 1;
        }
        invVi = invert(Vi);
        Vec aux(3);
        for (int i = 0; i < 3; i++) aux[i] = coordsX[i][0];
        A = times(invV, aux);
        for (int i = 0; i < 3; i++) aux[i] = coordsX[i][1];
        B = times(invV, aux);
        for (int i = 0; i < 3; i++) aux[i] = coordsXi[i][0];
        iA = times(invVi, aux);
        for (int i = 0; i < 3; i++) aux[i] = coordsXi[i][1];
        iB = times(invVi, aux);
    }
    Vec getX(const Vec& Xi) const override { return Vec{A[0] * Xi[0] + A[1] * Xi[1] + A[2], B[0] * Xi[0] + B[1] * Xi[1] + B[2]}; }
    Vec getXi(const Vec& X) const override { return Vec{iA[0] * X[0] + iA[1] * X[1] + iA[2], iB[0] * X[0] + iB[1] * X[1] + iB[2]}; }
    double getDX(const Vec&, int top, int bottom) const override {
        if (top == 0) return bottom == 0 ? A[0] : A[1];
        return bottom == 0 ? B[0] : B[1];
    }
    double jacobian(const Vec& Xi) const override {
        double dxdxi = getDX(Xi, 0, 0), dxdeta = getDX(Xi, 0, 1), dydxi = getDX(Xi, 1, 0), dydeta = getDX(Xi, 1, 1);
        return std::fabs(dxdxi * dydeta - dxdeta * dydxi) / 2;
    }
    Mat2 getInterpolant(const Quadrature& q) const override {
        Mat2 I = zeros(q.nPoints, 3);
        for (int p = 0; p < q.nPoints; p++) {
            double xi = q.coords[p][0], eta = q.coords[p][1];
            I[p][0] = 1 - xi - eta;
            I[p][1] = xi;
            I[p][2] = eta;
        }
        return I;
    }
    Vec getXs() const override { return getX(Vec{1.0 / 3, 1.0 / 3}); }
};

// transformation/transformation3Dtetra.java:14-118.  Deviation: getXs returns the
// centroid x(1/4, 1/4, 1/4).  The reference's literal {0.25, 0.25, 0, 25}
// (transformation3Dtetra.java:116) evaluates x(1/4, 1/4, 0), a point on face 0, so the
// DDG distance of that face is zero and every 3D viscous residual with a boundary on
// face 0 is NaN.
struct Transformation3DTet : Transformation {
    Vec A, B, C, iA, iB, iC;
    Mat2 invV, invVi;
    explicit Transformation3DTet(const Mat2& vertices) {
        coordsXi = Mat2{{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        coordsX = vertices;
        Mat2 V = zeros(4, 4);
        for (int i = 0; i < 4; i++) {
            V[i][0] = coordsXi[i][0];
            V[i][1] = coordsXi[i][1];
            V[i][2] = coordsXi[i][2];
            V[i][3] = 1;
        }
        invV = invert(V);
        for (int i = 0; i < 4; i++) {
            V[i][0] = coordsX[i][0];
            V[i][1] = coordsX[i][1];
            V[i][2] = coordsX[i][2];
            V[i][3] = 1;
        }
        invVi = invert(V);
        Vec aux(4);
        for (int i = 0; i < 4; i++) aux[i] = coordsX[i][0];
        A = times(invV, aux);
        for (int i = 0; i < 4; i++) aux[i] = coordsX[i][1];
        B = times(invV, aux);
        for (int i = 0; i < 4; i++) aux[i] = coordsX[i][2];
        C = times(invV, aux);
        for (int i = 0; i < 4; i++) aux[i] = coordsXi[i][0];
        iA = times(invVi, aux);
        for (int i = 0; i < 4; i++) aux[i] = coordsXi[i][1];
        iB = times(invVi, aux);
        for (int i = 0; i < 4; i++) aux[i] = coordsXi[i][2];
        iC = times(invVi, aux);
    }
    Vec getX(const Vec& Xi) const override {
        return Vec{A[0] * Xi[0] + A[1] * Xi[1] + A[2] * Xi[2] + A[3], B[0] * Xi[0] + B[1] * Xi[1] + B[2] * Xi[2] + B[3],
                   C[0] * Xi[0] + C[1] * Xi[1] + C[2] * Xi[2] + C[3]};
    }
    Vec getXi(const Vec& X) const override {
        return Vec{iA[0] * X[0] + iA[1] * X[1] + iA[2] * X[2] + iA[3], iB[0] * X[0] + iB[1] * X[1] + iB[2] * X[2] + iB[3],
                   iC[0] * X[0] + iC[1] * X[1] + iC[2] * X[2] + iC[3]};
    }
    double getDX(const Vec&, int top, int bottom) const override {
        if (top == 0) return A[bottom];
        if (top == 1) return B[bottom];
        return C[bottom];
    }
    double jacobian(const Vec&) const override {
        return std::fabs(A[0] * B[1] * C[2] + A[1] * B[2] * C[0] + A[2] * B[0] * C[1] - A[2] * B[1] * C[0] -
                         A[1] * B[0] * C[2] - A[0] * B[2] * C[1]);
    }
    Mat2 getInterpolant(const Quadrature& q) const override {
        Mat2 I = zeros(q.nPoints, 4);
        for (int p = 0; p < q.nPoints; p++) {
            double xi = q.coords[p][0], eta = q.coords[p][1], zeta = q.coords[p][2];
            I[p][0] = 1 - xi - eta - zeta;
            I[p][1] = xi;
            I[p][2] = eta;
            I[p][3] = zeta;
        }
        return I;
    }
    Vec getXs() const override { return getX(Vec{0.25, 0.25, 0.25}); }
};

struct FaceTransformation {
    const Transformation* transform = nullptr;
    virtual ~FaceTransformation() {}
    virtual Vec getXiRef(const Vec& Xi) const = 0;
    virtual double jacobian(const Vec& Xi) const = 0;
    virtual Mat2 getInterpolant(const Quadrature& q) const = 0;
    virtual Vec getNormal(const Vec& Xi) const = 0;
    Vec getX(const Vec& Xi) const { return transform->getX(getXiRef(Xi)); }
    Mat2 getXiRef(const Mat2& Xi) const {
        Mat2 r;
        for (auto& x : Xi) r.push_back(getXiRef(x));
        return r;
    }
    Mat2 getX(const Mat2& Xi) const {
        Mat2 r;
        for (auto& x : Xi) r.push_back(getX(x));
        return r;
    }
    Vec jacobian(const Quadrature& q) const {
        Vec J(q.nPoints);
        for (int i = 0; i < q.nPoints; i++) J[i] = jacobian(q.coords[i]);
        return J;
    }
    virtual Vec getXs() const = 0;
};

// transformation/faceTransformation2Dline.java:12-65
struct FaceTransformation2DLine : FaceTransformation {
    Mat2 coordsXiRef;
    FaceTransformation2DLine(const Transformation* t, const IVec& fi) {
        transform = t;
        coordsXiRef = zeros(2, 2);
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++) coordsXiRef[i][j] = t->coordsXi[fi[i]][j];
    }
    Vec getXiRef(const Vec& Xi) const override {
        Vec r(2);
        r[0] = (1 + Xi[0]) / 2 * coordsXiRef[1][0] + (1 - Xi[0]) / 2 * coordsXiRef[0][0];
        r[1] = (1 + Xi[0]) / 2 * coordsXiRef[1][1] + (1 - Xi[0]) / 2 * coordsXiRef[0][1];
        return r;
    }
    double jacobian(const Vec& Xi) const override {
        Vec s{coordsXiRef[1][0] - coordsXiRef[0][0], coordsXiRef[1][1] - coordsXiRef[0][1]};
        Vec Js = transform->jacobianMatrixDirection(getXiRef(Xi), s);
        return L2Norm(Js) / 2;
    }
    Mat2 getInterpolant(const Quadrature& q) const override {
        Mat2 I = zeros(q.nPoints, 2);
        for (int p = 0; p < q.nPoints; p++) {
            double xi = q.coords[p][0];
            I[p][0] = (1 - xi) / 2;
            I[p][1] = (1 + xi) / 2;
        }
        return I;
    }
    Vec getNormal(const Vec& Xi) const override {
        Vec s{coordsXiRef[1][0] - coordsXiRef[0][0], coordsXiRef[1][1] - coordsXiRef[0][1]};
        Vec Js = transform->jacobianMatrixDirection(getXiRef(Xi), s);
        return normVector(Vec{Js[1], -Js[0]});
    }
    Vec getXs() const override { return getX(Vec{0.0}); }
};

// transformation/faceTransformation3Dtriangle.java:22-96
struct FaceTransformation3DTri : FaceTransformation {
    Mat2 coordsXiRef;
    Vec A, B, C;
    FaceTransformation3DTri(const Transformation* t, const IVec& fi) {
        transform = t;
        coordsXiRef = zeros(3, 3);
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) coordsXiRef[i][j] = t->coordsXi[fi[i]][j];
        Mat2 cxi{{0, 0}, {1, 0}, {0, 1}};
        Mat2 V = zeros(3, 3);
        for (int i = 0; i < 3; i++) {
            V[i][0] = cxi[i][0];
            V[i][1] = cxi[i][1];
            V[i][2] = 1;
        }
        Mat2 invV = invert(V);
        Vec aux(3);
        for (int i = 0; i < 3; i++) aux[i] = coordsXiRef[i][0];
        A = times(invV, aux);
        for (int i = 0; i < 3; i++) aux[i] = coordsXiRef[i][1];
        B = times(invV, aux);
        for (int i = 0; i < 3; i++) aux[i] = coordsXiRef[i][2];
        C = times(invV, aux);
    }
    Vec getXiRef(const Vec& Xi) const override {
        return Vec{A[0] * Xi[0] + A[1] * Xi[1] + A[2], B[0] * Xi[0] + B[1] * Xi[1] + B[2], C[0] * Xi[0] + C[1] * Xi[1] + C[2]};
    }
    double jacobian(const Vec& Xi) const override {
        Vec s1{A[0], B[0], C[0]}, s2{A[1], B[1], C[1]};
        Vec Js1 = transform->jacobianMatrixDirection(getXiRef(Xi), s1);
        Vec Js2 = transform->jacobianMatrixDirection(getXiRef(Xi), s2);
        return L2Norm(cross(Js1, Js2)) / 2;
    }
    Mat2 getInterpolant(const Quadrature& q) const override {
        Mat2 I = zeros(q.nPoints, 3);
        for (int p = 0; p < q.nPoints; p++) {
            double xi = q.coords[p][0], eta = q.coords[p][1];
            I[p][0] = 1 - xi - eta;
            I[p][1] = xi;
            I[p][2] = eta;
        }
        return I;
    }
    Vec getNormal(const Vec& Xi) const override {
        Vec s1{A[0], B[0], C[0]}, s2{A[1], B[1], C[1]};
        Vec Js1 = transform->jacobianMatrixDirection(getXiRef(Xi), s1);
        Vec Js2 = transform->jacobianMatrixDirection(getXiRef(Xi), s2);
        return normVector(cross(Js2, Js1));
    }
    Vec getXs() const override { return getX(Vec{1.0 / 3, 1.0 / 3}); }
};

// ---------------------------------------------------------------- element types
// elementType/triangleElement.java:52-54, tetrahedralElement.java:52-68
static IVec getFaceIndexes(int type, int k) {
    if (type == 3) return IVec{k, (k + 1) % 3};
    switch (k) {
        case 0: return IVec{0, 2, 1};
        case 1: return IVec{0, 1, 3};
        case 2: return IVec{1, 2, 3};
        default: return IVec{2, 0, 3};
    }
}
static int numberOfFaces(int type) { return type == 3 ? 3 : 4; }
static int numberOfPoints(int type) { return type == 3 ? 3 : 4; }

// FlowProMain.createNeighborMatrix, FlowProMain.java:772-873
static std::vector<IVec> createNeighborMatrix(const IVec& type, const std::vector<IVec>& TP,
                                              const std::vector<IVec>& boundary) {
    struct FI {
        int i1, i2;
    };
    std::map<std::string, FI> map;
    int nRows = (int)TP.size();
    auto keyOf = [](IVec f) {
        std::sort(f.begin(), f.end());
        std::string key;
        for (int v : f) key += std::to_string(v) + "$";
        return key;
    };
    for (int i = 0; i < nRows; i++) {
        int nF = numberOfFaces(type[i]);
        for (int k = 0; k < nF; k++) {
            IVec fi = getFaceIndexes(type[i], k);
            for (auto& v : fi) v = TP[i][v];
            std::string key = keyOf(fi);
            auto it = map.find(key);
            if (it == map.end())
                map[key] = FI{i, -1000};
            else
                it->second.i2 = i;
        }
    }
    std::vector<IVec> TT(nRows);
    for (int i = 0; i < nRows; i++) {
        int nF = numberOfFaces(type[i]);
        TT[i].assign(nF, -1000);
        for (int k = 0; k < nF; k++) {
            IVec fi = getFaceIndexes(type[i], k);
            for (auto& v : fi) v = TP[i][v];
            FI& f = map[keyOf(fi)];
            if (f.i1 == i) {
                if (f.i2 != -1000) TT[i][k] = f.i2;
            } else {
                TT[i][k] = f.i1;
            }
        }
    }
    std::map<std::string, int> bound;
    for (auto& row : boundary) {
        IVec fi(row.begin() + 1, row.end());
        bound[keyOf(fi)] = row[0];
    }
    for (int i = 0; i < nRows; i++)
        for (size_t k = 0; k < TT[i].size(); k++)
            if (TT[i][k] == -1000) {
                IVec fi = getFaceIndexes(type[i], (int)k);
                for (auto& v : fi) v = TP[i][v];
                auto it = bound.find(keyOf(fi));
                TT[i][k] = it != bound.end() ? it->second : -1;
            }
    return TT;
}

// ---------------------------------------------------------------- equations (plugins)
// flowpro/api/ElementData.java:9-26
struct ElementData {
    Vec currentX, meshVelocity;
    double currentWallDistance = 0, currentT = 0;
    int elemIndex = 0;
};

using Props = std::map<std::string, std::string>;
static bool has(const Props& p, const std::string& k) { return p.count(k) > 0; }
static double getD(const Props& p, const std::string& k) {
    auto it = p.find(k);
    if (it == p.end()) throw std::runtime_error("missing parameter " + k);
    return std::atof(it->second.c_str());
}
static Vec getDA(const Props& p, const std::string& k) {
    Vec v;
    std::string s = p.at(k);
    for (char& c : s)
        if (c == ',') c = ' ';
    std::istringstream is(s);
    double x;
    while (is >> x) v.push_back(x);
    return v;
}
static bool getB(const Props& p, const std::string& k) {
    std::string s = p.at(k);
    return s == "true" || s == "1";
}

// flowpro/api/Equation.java:5-128
struct Equation {
    virtual ~Equation() {}
    virtual int dim() const = 0;
    virtual int nEqs() const = 0;
    virtual bool isConvective() const { return true; }
    virtual bool isDiffusive() const = 0;
    virtual bool isSourcePresent() const = 0;
    virtual Vec boundaryValue(Vec& WL, const Vec& n, int TT, ElementData& e) = 0;
    virtual Vec numericalConvectiveFlux(Vec& WL, Vec& WR, const Vec& n, int TT, ElementData& e) = 0;
    virtual Vec convectiveFlux(Vec& W, const Vec& n, ElementData& e) = 0;
    virtual Vec diffusiveFlux(Vec& W, const Vec& dW, const Vec& n, ElementData& e) = 0;
    virtual Vec numericalDiffusiveFlux(Vec& Wc, const Vec& dWc, const Vec& n, int TT, ElementData& e) = 0;
    virtual Vec sourceTerm(Vec& W, const Vec& dW, ElementData& e) = 0;
    virtual double maxEigenvalue(Vec& W, ElementData* e) = 0;
    virtual bool isIPFace(int TT) const = 0;
    virtual bool isAdmissible(const Vec& W) const = 0;
    virtual Vec combineShockSensors(Vec s) const = 0;
    virtual Vec constInitCondition() = 0;
    virtual double pressure(Vec& W) = 0;
    virtual Vec stressVector(Vec& W, const Vec& dW, const Vec& n) = 0;
};

// ModuleProjects/Equations/Aerodynamics/.../Aerodynamics.java
struct Aerodynamics : Equation {
    static constexpr int WALL = -1, INLET = -2, OUTLET = -3, INVISCID_WALL = -4;
    static constexpr double RHO_TOL = 1e-2;
    static constexpr double ADMISSIBLE_TOL = 1e-10;
    int dim_ = 2, nEqs_ = 4;
    bool isDiffusive_ = false;
    double kapa = 1.4, Re = -1, Pr = -1, lRef = 1, pRef = 1, rhoRef = 1, velocityRef = 1, tRef = 1, cp = 0, cv = 0;
    bool isInletSupersonic = false;
    const double pIn0 = 1, rhoIn0 = 1;
    bool hasAttack = false;
    Vec attackAngle;
    Vec WIn;
    double pOut = 0;
    std::string numericalFluxType = "default";

    int dim() const override { return dim_; }
    int nEqs() const override { return nEqs_; }
    bool isDiffusive() const override { return isDiffusive_; }

    double stagnationStaticPressureRatio(double mach) const {
        return std::pow(1 + (kapa - 1) / 2 * mach * mach, kapa / (kapa - 1));
    }
    double stagnationStaticDensityRatio(double mach) const {
        return std::pow(1 + (kapa - 1) / 2 * mach * mach, 1 / (kapa - 1));
    }
    // Aerodynamics.init, Aerodynamics.java:119-312
    void initAero(const Props& props, int dim, int nEqs, bool isDiff) {
        nEqs_ = nEqs;
        dim_ = dim;
        isDiffusive_ = isDiff;
        if (has(props, "kappa") && has(props, "cv") && !has(props, "cp")) {
            kapa = getD(props, "kappa");
            cv = getD(props, "cv");
            cp = cv * kapa;
        } else if (has(props, "kappa") && has(props, "cp") && !has(props, "cv")) {
            kapa = getD(props, "kappa");
            cp = getD(props, "cp");
            cv = cp / kapa;
        } else if (has(props, "cv") && has(props, "cp") && !has(props, "kappa")) {
            cp = getD(props, "cp");
            cv = getD(props, "cv");
            kapa = cp / cv;
        } else {
            throw std::runtime_error("exactly two out of kappa, cp, cv");
        }
        isInletSupersonic = has(props, "isInletSupersonic") && getB(props, "isInletSupersonic");
        if (isInletSupersonic) {
            pRef = getD(props, "pIn");
            if (has(props, "rhoIn"))
                rhoRef = getD(props, "rhoIn");
            else
                rhoRef = pRef / (cv * (kapa - 1) * getD(props, "TIn"));
        } else {
            bool farField = has(props, "pInf") && has(props, "machInf") && (has(props, "TInf") != has(props, "rhoInf"));
            bool stagnation = has(props, "pIn0") && has(props, "pOut") && (has(props, "TIn0") != has(props, "rhoIn0"));
            if (farField && !stagnation) {
                double pInf = getD(props, "pInf"), machInf = getD(props, "machInf");
                double rhoInf = has(props, "rhoInf") ? getD(props, "rhoInf")
                                                     : pInf / (cv * (kapa - 1) * getD(props, "TInf"));
                pRef = pInf * stagnationStaticPressureRatio(machInf);
                rhoRef = rhoInf * stagnationStaticDensityRatio(machInf);
                pOut = pIn0 / stagnationStaticPressureRatio(machInf);
            } else if (stagnation && !farField) {
                pRef = getD(props, "pIn0");
                if (has(props, "rhoIn0"))
                    rhoRef = getD(props, "rhoIn0");
                else
                    rhoRef = pRef / (cv * (kapa - 1) * getD(props, "TIn0"));
                pOut = getD(props, "pOut") / pRef;
            } else {
                throw std::runtime_error("stagnation or far-field boundary conditions required");
            }
        }
        lRef = has(props, "lRef") ? getD(props, "lRef") : 1;
        velocityRef = std::sqrt(pRef / rhoRef);
        tRef = lRef / velocityRef;
        hasAttack = false;
        if (has(props, "attackAngle")) {
            attackAngle = getDA(props, "attackAngle");
            hasAttack = true;
            if ((int)attackAngle.size() != dim - 1) throw std::runtime_error("attackAngle must have dim-1 entries");
        }
        WIn.assign(nEqs, 0.0);
        if (isInletSupersonic) {
            double velocityIn = getD(props, "vIn") / velocityRef;
            Vec vIn(dim, 0.0);
            if (dim == 1) vIn[0] = velocityIn;
            if (dim == 2) {
                vIn[0] = velocityIn * std::cos(attackAngle[0]);
                vIn[1] = velocityIn * std::sin(attackAngle[0]);
            }
            WIn[0] = 1;
            for (int d = 0; d < dim; ++d) WIn[d + 1] = vIn[d];
            if (nEqs > dim + 1) {
                double v2 = 0;
                for (int d = 0; d < dim; ++d) v2 += vIn[d] * vIn[d];
                WIn[3] = 1 / (kapa - 1) + 0.5 * v2;
            }
        } else {
            WIn[0] = -1;
        }
        if (isDiffusive_) {
            double machInf = std::sqrt(2 / (kapa - 1) * (std::pow((pIn0 / pOut), (kapa - 1) / kapa) - 1));
            double rhoInf = rhoRef / stagnationStaticDensityRatio(machInf);
            double pInf = pRef / stagnationStaticPressureRatio(machInf);
            double aInf = std::sqrt(kapa * pInf / rhoInf);
            double uInf = machInf * aInf;
            if (has(props, "reynolds") && has(props, "prandtl") && !has(props, "viscosity") && !has(props, "conductivity")) {
                double trueRe = getD(props, "reynolds");
                Re = trueRe * (rhoRef * velocityRef) / (rhoInf * uInf);
                Pr = getD(props, "prandtl");
            } else if (has(props, "viscosity") && has(props, "conductivity")) {
                double viscosity = getD(props, "viscosity");
                double conductivity = getD(props, "conductivity");
                Pr = cp * viscosity / conductivity;
                Re = rhoRef * velocityRef * lRef / viscosity;
            } else {
                throw std::runtime_error("Prandtl and Reynolds or viscosity and conductivity required");
            }
        } else {
            Re = -1;
            Pr = -1;
        }
        numericalFluxType = has(props, "numericalFlux") ? props.at("numericalFlux") : "default";
    }
    double limiteRho(double rho) const {
        if (rho < RHO_TOL) return RHO_TOL * std::exp((rho - RHO_TOL) / RHO_TOL);
        return rho;
    }
    // Aerodynamics.maxEigenvalue, Aerodynamics.java:322-337
    double maxEigenvalue(Vec& W, ElementData* elem) override {
        W[0] = limiteRho(W[0]);
        double p = pressure(W);
        double a = std::sqrt(kapa * p / W[0]);
        double v = .0;
        for (int d = 0; d < dim_; ++d) {
            double vRel = W[d + 1] / W[0] - (elem == nullptr ? 0 : elem->meshVelocity[d]);
            v += vRel * vRel;
        }
        v = std::sqrt(v);
        return v + a;
    }
    // Aerodynamics.isAdmissible, Aerodynamics.java:347-357
    bool isAdmissible(const Vec& W) const override {
        if (!(W[0] > ADMISSIBLE_TOL)) return false;
        double m2 = .0;
        for (int d = 0; d < dim_; ++d) m2 += W[d + 1] * W[d + 1];
        return W[dim_ + 1] - m2 / (2 * W[0]) > ADMISSIBLE_TOL;
    }
    bool isIPFace(int TT) const override { return TT == WALL; }
    Vec combineShockSensors(Vec s) const override {
        for (int m = 1; m < nEqs_; m++) s[m] = s[0];
        return s;
    }
    Vec stressVector(Vec& W, const Vec&, const Vec& n) override {
        double p = pressure(W);
        Vec sv(dim_, 0.0);
        for (int d = 0; d < dim_; ++d) sv[d] -= p * n[d];
        return sv;
    }
};

// ModuleProjects/Equations/Aerodynamics/.../NavierStokes.java
struct NavierStokes : Aerodynamics {
    static constexpr double P_TOL = 1e-2;
    void init(const Props& props) {
        int dimension = (int)getD(props, "dimension");
        initAero(props, dimension, dimension + 2, getB(props, "isFlowViscous"));
    }
    bool isSourcePresent() const override { return false; }
    // NavierStokes.pressure, NavierStokes.java:23-37
    double pressure(Vec& W) override {
        W[0] = limiteRho(W[0]);
        double m2 = .0;
        for (int d = 0; d < dim_; ++d) m2 += W[d + 1] * W[d + 1];
        double p = (kapa - 1) * (W[dim_ + 1] - m2 / (2 * W[0]));
        if (p < P_TOL) p = P_TOL * std::exp((p - P_TOL) / P_TOL);
        return p;
    }
    // NavierStokes.constInitCondition, NavierStokes.java:98-139
    Vec constInitCondition() override {
        if (isInletSupersonic) return WIn;
        double machIn = std::sqrt(2 / (kapa - 1) * (std::pow((1 / pOut), (kapa - 1) / kapa) - 1));
        double rhoIn = std::pow(1 + ((kapa - 1) / 2) * machIn * machIn, 1 / (1 - kapa));
        double VIn = machIn * std::sqrt((kapa * pOut) / rhoIn);
        Vec vIn(dim_, 0.0);
        double alpha = 0, beta = 0;
        if (hasAttack) {
            alpha = attackAngle[0];
            if (dim_ == 3) beta = attackAngle[1];
        }
        if (dim_ == 1) vIn[0] = VIn;
        if (dim_ == 2) {
            vIn[0] = VIn * std::cos(alpha);
            vIn[1] = VIn * std::sin(alpha);
        }
        if (dim_ == 3) {
            vIn[0] = VIn * std::cos(alpha) * std::cos(beta);
            vIn[1] = VIn * std::sin(alpha) * std::cos(beta);
            vIn[2] = VIn * std::sin(beta);
        }
        Vec W(nEqs_, 0.0);
        W[0] = rhoIn;
        for (int d = 0; d < dim_; ++d) W[d + 1] = rhoIn * vIn[d];
        W[dim_ + 1] = pOut / (kapa - 1) + 0.5 * rhoIn * VIn * VIn;
        return W;
    }
    Vec fplus(const Vec& W, double p, const Vec& n) const {
        Vec f(nEqs_, 0.0), velocity(dim_);
        double Vn = 0, q2 = 0;
        for (int d = 0; d < dim_; ++d) {
            velocity[d] = W[d + 1] / W[0];
            Vn += velocity[d] * n[d];
            q2 += velocity[d] * velocity[d];
        }
        double a = std::sqrt(kapa * p / W[0]);
        double M = Vn / a;
        if (std::fabs(M) < 1) {
            double fm = W[0] * a * ((M + 1) * (M + 1)) / 4;
            f[0] = fm;
            for (int d = 0; d < dim_; ++d) f[d + 1] = fm * (velocity[d] + (-Vn + 2 * a) / kapa * n[d]);
            f[dim_ + 1] = fm * ((q2 - Vn * Vn) / 2 + (((kapa - 1) * Vn + 2 * a)) * (((kapa - 1) * Vn + 2 * a)) / (2 * (kapa * kapa - 1)));
        } else if (M >= 1) {
            f[0] = W[0] * Vn;
            for (int d = 0; d < dim_; ++d) f[d + 1] = W[d + 1] * Vn + p * n[d];
            f[dim_ + 1] = (W[dim_ + 1] + p) * Vn;
        }
        return f;
    }
    Vec fminus(const Vec& W, double p, const Vec& n) const {
        Vec f(nEqs_, 0.0), velocity(dim_);
        double Vn = 0, q2 = 0;
        for (int d = 0; d < dim_; ++d) {
            velocity[d] = W[d + 1] / W[0];
            Vn += velocity[d] * n[d];
            q2 += velocity[d] * velocity[d];
        }
        double a = std::sqrt(kapa * p / W[0]);
        double M = Vn / a;
        if (std::fabs(M) < 1) {
            double fm = -W[0] * a * ((M - 1) * (M - 1)) / 4;
            f[0] = fm;
            for (int d = 0; d < dim_; ++d) f[d + 1] = fm * (velocity[d] + (-Vn - 2 * a) / kapa * n[d]);
            f[dim_ + 1] = fm * ((q2 - Vn * Vn) / 2 + (((kapa - 1) * Vn - 2 * a) * ((kapa - 1) * Vn - 2 * a)) / (2 * (kapa * kapa - 1)));
        } else if (M <= -1) {
            f[0] = W[0] * Vn;
            for (int d = 0; d < dim_; ++d) f[d + 1] = W[d + 1] * Vn + p * n[d];
            f[dim_ + 1] = (W[dim_ + 1] + p) * Vn;
        }
        return f;
    }
    // NavierStokes.numericalConvectiveFlux, NavierStokes.java:141-192
    Vec numericalConvectiveFlux(Vec& WL, Vec& WR, const Vec& n, int TT, ElementData& elem) override {
        WL[0] = limiteRho(WL[0]);
        WR[0] = limiteRho(WR[0]);
        Vec f(nEqs_, 0.0);
        switch (TT) {
            case WALL:
            case INVISCID_WALL: {
                double p = pressure(WL);
                f[0] = 0;
                double V = .0;
                for (int d = 0; d < dim_; ++d) {
                    f[d + 1] = p * n[d];
                    V += elem.meshVelocity[d] * n[d];
                }
                f[dim_ + 1] = p * V;
                for (int j = 0; j < nEqs_; j++) f[j] += V * WR[j];
                break;
            }
            case INLET:
            case OUTLET:
                f = convectiveFlux(WR, n, elem);
                break;
            default:
                if (numericalFluxType == "vanLeer") {
                    double pL = pressure(WL);
                    Vec fp = fplus(WL, pL, n);
                    double pR = pressure(WR);
                    Vec fm = fminus(WR, pR, n);
                    for (int j = 0; j < nEqs_; j++) f[j] = fp[j] + fm[j];
                } else {
                    Vec fL = convectiveFlux(WL, n, elem);
                    Vec fR = convectiveFlux(WR, n, elem);
                    double lL = maxEigenvalue(WL, &elem);
                    double lR = maxEigenvalue(WR, &elem);
                    double maxEigenValue = std::max(lL, lR);
                    for (int j = 0; j < nEqs_; j++) f[j] = (fL[j] + fR[j] - maxEigenValue * (WR[j] - WL[j])) / 2;
                }
        }
        return f;
    }
    // NavierStokes.convectiveFlux, NavierStokes.java:194-214
    Vec convectiveFlux(Vec& W, const Vec& n, ElementData&) override {
        W[0] = limiteRho(W[0]);
        Vec f(nEqs_, 0.0);
        double V = .0;
        for (int d = 0; d < dim_; ++d) V += W[d + 1] * n[d];
        V /= W[0];
        double p = pressure(W);
        f[0] = W[0] * V;
        for (int d = 0; d < dim_; ++d) f[d + 1] = W[d + 1] * V + p * n[d];
        f[dim_ + 1] = (W[dim_ + 1] + p) * V;
        return f;
    }
    // NavierStokes.boundaryValue, NavierStokes.java:216-315
    Vec boundaryValue(Vec& WL, const Vec& n, int TT, ElementData& elem) override {
        WL[0] = limiteRho(WL[0]);
        Vec WR(nEqs_, 0.0);
        double p = pressure(WL);
        switch (TT) {
            case WALL:
                if (isDiffusive_) {
                    const Vec& u = elem.meshVelocity;
                    double a2 = .0;
                    for (int d = 0; d < dim_; ++d) a2 += u[d] * u[d];
                    WR[0] = WL[0];
                    for (int d = 0; d < dim_; ++d) WR[d + 1] = WR[0] * u[d];
                    WR[dim_ + 1] = p / (kapa - 1) + WR[0] * a2 / 2;
                } else {
                    WR = WL;
                    double nu = 0;
                    for (int d = 0; d < dim_; ++d) nu += WL[d + 1] * n[d];
                    for (int d = 0; d < dim_; ++d) WR[d + 1] = WL[d + 1] - n[d] * nu;
                }
                break;
            case INVISCID_WALL: {
                WR = WL;
                double nu = 0;
                for (int d = 0; d < dim_; ++d) nu += WL[d + 1] * n[d];
                for (int d = 0; d < dim_; ++d) WR[d + 1] = WL[d + 1] - n[d] * nu;
                break;
            }
            case INLET:
                if (!isInletSupersonic) {
                    double mach;
                    if (p > pIn0)
                        mach = 0;
                    else
                        mach = std::sqrt((2 / (kapa - 1)) * (-1 + std::pow(pIn0 / p, (kapa - 1) / kapa)));
                    double rhoIn = rhoIn0 * std::pow((1 + ((kapa - 1) / 2) * mach * mach), 1 / (1 - kapa));
                    double inletVelocity = mach * std::sqrt((kapa * p) / rhoIn);
                    double E = p / (kapa - 1) + 0.5 * rhoIn * inletVelocity * inletVelocity;
                    WR[0] = rhoIn;
                    if (!hasAttack) {
                        for (int d = 0; d < dim_; ++d) WR[d + 1] = -rhoIn * inletVelocity * n[d];
                    } else {
                        Vec dir;
                        if (dim_ == 2)
                            dir = Vec{std::cos(attackAngle[0]), std::sin(attackAngle[0])};
                        else
                            dir = Vec{std::cos(attackAngle[0]) * std::cos(attackAngle[1]),
                                      std::sin(attackAngle[0]) * std::cos(attackAngle[1]), std::sin(attackAngle[1])};
                        for (int d = 0; d < dim_; ++d) WR[d + 1] = rhoIn * inletVelocity * dir[d];
                    }
                    WR[dim_ + 1] = E;
                } else {
                    WR = WIn;
                }
                break;
            case OUTLET: {
                double rhoOut = WL[0];
                double a2 = .0;
                for (int d = 0; d < dim_; ++d) a2 += WL[d + 1] * WL[d + 1];
                a2 /= rhoOut * rhoOut;
                double a = std::sqrt(kapa * pressure(WL) / WL[0]);
                double mach = std::sqrt(a2) / a;
                if (mach < 1) {
                    WR[0] = rhoOut;
                    for (int d = 0; d < dim_; ++d) WR[d + 1] = rhoOut * WL[d + 1] / WL[0];
                    WR[dim_ + 1] = pOut / (kapa - 1) + rhoOut * a2 / 2;
                } else {
                    WR = WL;
                }
                break;
            }
            default:
                break;
        }
        return WR;
    }
    // NavierStokes.diffusiveFlux, NavierStokes.java:317-374
    Vec diffusiveFlux(Vec& W, const Vec& dW, const Vec& n, ElementData&) override {
        W[0] = limiteRho(W[0]);
        double rho = W[0];
        double lam = -2. / 3;
        int dim = dim_;
        Vec velocity(dim);
        double velocity2 = .0;
        for (int d = 0; d < dim; ++d) {
            velocity[d] = W[d + 1] / rho;
            velocity2 += velocity[d] * velocity[d];
        }
        Vec vJ(dim * dim);
        for (int d = 0; d < dim; ++d)
            for (int f = 0; f < dim; ++f) vJ[dim * d + f] = (dW[f * nEqs_ + d + 1] - dW[f * nEqs_] * velocity[d]) / rho;
        double p = pressure(W);
        Vec pOverRhoDer(dim);
        for (int d = 0; d < dim; ++d) {
            double temp = .0;
            for (int f = 0; f < dim; ++f) temp += velocity[f] * vJ[dim * f + d];
            double pDer = (kapa - 1) * (dW[d * nEqs_ + dim + 1] - dW[d * nEqs_] * velocity2 / 2 - rho * temp);
            pOverRhoDer[d] = (rho * pDer - p * dW[d * nEqs_]) / (rho * rho);
        }
        Vec stress(dim * dim);
        double trace = .0;
        for (int d = 0; d < dim; ++d) {
            trace += vJ[dim * d + d];
            for (int f = 0; f < dim; ++f) stress[dim * d + f] = vJ[dim * d + f] + vJ[dim * f + d];
        }
        for (int d = 0; d < dim; ++d) stress[dim * d + d] += lam * trace;
        double constant = kapa / (kapa - 1) / Pr;
        Vec flux(nEqs_, 0.0);
        flux[0] = 0;
        for (int d = 0; d < dim; ++d) {
            double tmp = .0;
            for (int f = 0; f < dim; ++f) {
                flux[f + 1] += stress[dim * d + f] * n[d] / Re;
                tmp += velocity[f] * stress[dim * d + f];
            }
            flux[dim + 1] += (tmp + constant * pOverRhoDer[d]) * n[d] / Re;
        }
        return flux;
    }
    // NavierStokes.numericalDiffusiveFlux, NavierStokes.java:376-395
    Vec numericalDiffusiveFlux(Vec& Wc, const Vec& dWc, const Vec& n, int TT, ElementData& elem) override {
        Wc[0] = limiteRho(Wc[0]);
        Vec flux = diffusiveFlux(Wc, dWc, n, elem);
        if (TT < 0) {
            if (TT == WALL) {
                double work = .0;
                for (int d = 0; d < dim_; ++d) work += elem.meshVelocity[d] * flux[d + 1];
                flux[dim_ + 1] = work;
            } else {
                std::fill(flux.begin(), flux.end(), 0.0);
            }
        }
        return flux;
    }
    Vec sourceTerm(Vec&, const Vec&, ElementData&) override { throw std::runtime_error("source is not present"); }
    // NavierStokes.stressVector, NavierStokes.java:39-83
    Vec stressVector(Vec& W, const Vec& dW, const Vec& normal) override {
        if (!isDiffusive_) return Aerodynamics::stressVector(W, dW, normal);
        int dim = dim_;
        double rho = W[0];
        Vec velocity(dim);
        for (int d = 0; d < dim; ++d) velocity[d] = W[d + 1] / rho;
        Vec vJ(dim * dim);
        for (int d = 0; d < dim; ++d)
            for (int f = 0; f < dim; ++f) vJ[dim * d + f] = (dW[f * nEqs_ + d + 1] - dW[f * nEqs_] * velocity[d]) / rho;
        Vec stress(dim * dim);
        double trace = .0;
        for (int d = 0; d < dim; ++d) {
            trace += vJ[dim * d + d];
            for (int f = 0; f < dim; ++f) stress[dim * d + f] = vJ[dim * d + f] + vJ[dim * f + d];
        }
        double lam = -2. / 3;
        for (int d = 0; d < dim; ++d) stress[dim * d + d] += lam * trace;
        double p = pressure(W);
        Vec sv(dim, 0.0);
        for (int d = 0; d < dim; ++d) {
            sv[d] -= p * normal[d];
            for (int f = 0; f < dim; ++f) sv[d] += 1 / Re * stress[dim * d + f] * normal[f];
        }
        return sv;
    }
};

// ModuleProjects/Equations/Aerodynamics/.../SpalartAllmaras.java
struct SpalartAllmaras : Aerodynamics {
    static constexpr double P_TOL = 1e-1;
    double vtIn = 0, sigma = 0, cb1 = 0, cb2 = 0, ka = 0, cw1 = 0, cw2 = 0, cw3 = 0, cv1 = 0, Prt = 0;
    void init(const Props& props) {
        int dimension = (int)getD(props, "dimension");
        initAero(props, dimension, dimension + 3, true);
        vtIn = getD(props, "vtIn");
        if (isInletSupersonic) WIn[dimension + 2] = vtIn;
        sigma = getD(props, "sigma");
        cb1 = getD(props, "cb1");
        cb2 = getD(props, "cb2");
        ka = getD(props, "ka");
        cw1 = cb1 / (ka * ka) + (1 + cb2) / sigma;
        cw2 = getD(props, "cw2");
        cw3 = getD(props, "cw3");
        cv1 = getD(props, "cv1");
        Prt = getD(props, "Prt");
    }
    // SpalartAllmaras.stressVector, SpalartAllmaras.java:510-553 (the laminar stress only)
    Vec stressVector(Vec& W, const Vec& dW, const Vec& normal) override {
        int dim = dim_;
        double rho = W[0];
        Vec velocity(dim);
        for (int d = 0; d < dim; ++d) velocity[d] = W[d + 1] / rho;
        Vec vJ(dim * dim);
        for (int d = 0; d < dim; ++d)
            for (int f = 0; f < dim; ++f) vJ[dim * d + f] = (dW[f * nEqs_ + d + 1] - dW[f * nEqs_] * velocity[d]) / rho;
        Vec stress(dim * dim);
        double trace = .0;
        for (int d = 0; d < dim; ++d) {
            trace += vJ[dim * d + d];
            for (int f = 0; f < dim; ++f) stress[dim * d + f] = vJ[dim * d + f] + vJ[dim * f + d];
        }
        double lam = -2. / 3;
        for (int d = 0; d < dim; ++d) stress[dim * d + d] += lam * trace;
        double p = pressure(W);
        Vec sv(dim, 0.0);
        for (int d = 0; d < dim; ++d) {
            sv[d] -= p * normal[d];
            for (int f = 0; f < dim; ++f) sv[d] += 1 / Re * stress[dim * d + f] * normal[f];
        }
        return sv;
    }
    bool isSourcePresent() const override { return true; }
    double pressure(Vec& W) override {
        W[0] = limiteRho(W[0]);
        double m2 = .0;
        for (int d = 0; d < dim_; ++d) m2 += W[d + 1] * W[d + 1];
        double p = (kapa - 1) * (W[dim_ + 1] - m2 / (2 * W[0]));
        if (p < P_TOL) p = P_TOL * std::exp((p - P_TOL) / P_TOL);
        return p;
    }
    Vec constInitCondition() override {
        if (isInletSupersonic) return WIn;
        double machIn = std::sqrt(2 / (kapa - 1) * (std::pow((1 / pOut), (kapa - 1) / kapa) - 1));
        double rhoIn = std::pow(1 + ((kapa - 1) / 2) * machIn * machIn, 1 / (1 - kapa));
        double VIn = machIn * std::sqrt((kapa * pOut) / rhoIn);
        Vec vIn(dim_, 0.0);
        double alpha = 0, beta = 0;
        if (hasAttack) {
            alpha = attackAngle[0];
            if (dim_ == 3) beta = attackAngle[1];
        }
        if (dim_ == 2) {
            vIn[0] = VIn * std::cos(alpha);
            vIn[1] = VIn * std::sin(alpha);
        }
        if (dim_ == 3) {
            vIn[0] = VIn * std::cos(alpha) * std::cos(beta);
            vIn[1] = VIn * std::sin(alpha) * std::cos(beta);
            vIn[2] = VIn * std::sin(beta);
        }
        Vec W(nEqs_, 0.0);
        W[0] = rhoIn;
        for (int d = 0; d < dim_; ++d) W[d + 1] = rhoIn * vIn[d];
        W[dim_ + 1] = pOut / (kapa - 1) + 0.5 * rhoIn * VIn * VIn;
        W[dim_ + 2] = rhoIn * vtIn;
        return W;
    }
    // SpalartAllmaras.numericalConvectiveFlux, SpalartAllmaras.java:130-172
    Vec numericalConvectiveFlux(Vec& WL, Vec& WR, const Vec& n, int TT, ElementData& elem) override {
        WL[0] = limiteRho(WL[0]);
        WR[0] = limiteRho(WR[0]);
        Vec f(nEqs_, 0.0);
        switch (TT) {
            case WALL:
            case INVISCID_WALL: {
                double p = pressure(WR);
                f[0] = 0;
                double V = .0;
                for (int d = 0; d < dim_; ++d) {
                    f[d + 1] = p * n[d];
                    V += elem.meshVelocity[d] * n[d];
                }
                f[dim_ + 1] = p * V;
                for (int j = 0; j < nEqs_; j++) f[j] += V * WR[j];
                break;
            }
            case INLET:
            case OUTLET:
                f = convectiveFlux(WR, n, elem);
                break;
            default: {
                Vec fL = convectiveFlux(WL, n, elem);
                Vec fR = convectiveFlux(WR, n, elem);
                double lL = maxEigenvalue(WL, &elem);
                double lR = maxEigenvalue(WR, &elem);
                double mx = std::max(lL, lR);
                for (int j = 0; j < nEqs_; j++) f[j] = (fL[j] + fR[j] - mx * (WR[j] - WL[j])) / 2;
            }
        }
        return f;
    }
    // SpalartAllmaras.convectiveFlux, SpalartAllmaras.java:174-195
    Vec convectiveFlux(Vec& W, const Vec& n, ElementData&) override {
        W[0] = limiteRho(W[0]);
        Vec f(nEqs_, 0.0);
        double V = .0;
        for (int d = 0; d < dim_; ++d) V += W[d + 1] * n[d];
        V /= W[0];
        double p = pressure(W);
        f[0] = W[0] * V;
        for (int d = 0; d < dim_; ++d) f[d + 1] = W[d + 1] * V + p * n[d];
        f[dim_ + 1] = (W[dim_ + 1] + p) * V;
        f[dim_ + 2] = W[dim_ + 2] * V;
        return f;
    }
    // SpalartAllmaras.boundaryValue, SpalartAllmaras.java:200-292
    Vec boundaryValue(Vec& WL, const Vec& n, int TT, ElementData& elem) override {
        WL[0] = limiteRho(WL[0]);
        Vec WR(nEqs_, 0.0);
        double p = pressure(WL);
        switch (TT) {
            case WALL: {
                const Vec& u = elem.meshVelocity;
                double a2 = .0;
                for (int d = 0; d < dim_; ++d) a2 += u[d] * u[d];
                WR[0] = WL[0];
                for (int d = 0; d < dim_; ++d) WR[d + 1] = WR[0] * u[d];
                WR[dim_ + 1] = p / (kapa - 1) + WR[0] * a2 / 2;
                WR[dim_ + 2] = 0;
                break;
            }
            case INVISCID_WALL: {
                WR = WL;
                double nu = 0;
                for (int d = 0; d < dim_; ++d) nu += WL[d + 1] * n[d];
                for (int d = 0; d < dim_; ++d) WR[d + 1] = WL[d + 1] + n[d] * nu;
                break;
            }
            case INLET:
                if (!isInletSupersonic) {
                    double mach;
                    if (p > pIn0)
                        mach = 0;
                    else
                        mach = std::sqrt((2 / (kapa - 1)) * (-1 + std::pow(pIn0 / p, (kapa - 1) / kapa)));
                    double rhoIn = rhoIn0 * std::pow((1 + ((kapa - 1) / 2) * mach * mach), 1 / (1 - kapa));
                    double inletVelocity = mach * std::sqrt((kapa * p) / rhoIn);
                    double E = p / (kapa - 1) + 0.5 * rhoIn * inletVelocity * inletVelocity;
                    WR[0] = rhoIn;
                    if (!hasAttack) {
                        for (int d = 0; d < dim_; ++d) WR[d + 1] = -rhoIn * inletVelocity * n[d];
                    } else {
                        Vec dir;
                        if (dim_ == 2)
                            dir = Vec{std::cos(attackAngle[0]), std::sin(attackAngle[0])};
                        else
                            dir = Vec{std::cos(attackAngle[0]) * std::cos(attackAngle[1]),
                                      std::sin(attackAngle[0]) * std::cos(attackAngle[1]), std::sin(attackAngle[1])};
                        for (int d = 0; d < dim_; ++d) WR[d + 1] = rhoIn * inletVelocity * dir[d];
                    }
                    WR[dim_ + 1] = E;
                    WR[dim_ + 2] = rhoIn * vtIn;
                } else {
                    WR = WIn;
                }
                break;
            case OUTLET: {
                double rhoOut = WL[0];
                double a2 = .0;
                for (int d = 0; d < dim_; ++d) a2 += WL[d + 1] * WL[d + 1];
                a2 /= rhoOut * rhoOut;
                double a = std::sqrt(kapa * pressure(WL) / WL[0]);
                double mach = std::sqrt(a2) / a;
                if (mach < 1) {
                    WR[0] = rhoOut;
                    for (int d = 0; d < dim_; ++d) WR[d + 1] = rhoOut * WL[d + 1] / WL[0];
                    WR[dim_ + 1] = pOut / (kapa - 1) + rhoOut * a2 / 2;
                    WR[dim_ + 2] = WL[dim_ + 2];
                } else {
                    WR = WL;
                }
                break;
            }
            default:
                break;
        }
        return WR;
    }
    static double mx(double a, double b) { return a > b ? a : b; }
    // SpalartAllmaras.diffusiveFlux, SpalartAllmaras.java:295-362
    Vec diffusiveFlux(Vec& W, const Vec& dW, const Vec& n, ElementData&) override {
        W[0] = limiteRho(W[0]);
        double rho = W[0];
        double lam = -2. / 3;
        int dim = dim_;
        Vec velocity(dim);
        double velocity2 = .0;
        for (int d = 0; d < dim; ++d) {
            velocity[d] = W[d + 1] / rho;
            velocity2 += velocity[d] * velocity[d];
        }
        Vec vJ(dim * dim);
        for (int d = 0; d < dim; ++d)
            for (int f = 0; f < dim; ++f) vJ[dim * d + f] = (dW[f * nEqs_ + d + 1] - dW[f * nEqs_] * velocity[d]) / rho;
        double p = pressure(W);
        Vec pOverRhoDer(dim);
        for (int d = 0; d < dim; ++d) {
            double temp = .0;
            for (int f = 0; f < dim; ++f) temp += velocity[f] * vJ[dim * f + d];
            double pDer = (kapa - 1) * (dW[d * nEqs_ + dim + 1] - dW[d * nEqs_] * velocity2 / 2 - rho * temp);
            pOverRhoDer[d] = (rho * pDer - p * dW[d * nEqs_]) / (rho * rho);
        }
        Vec stress(dim * dim);
        double trace = .0;
        for (int d = 0; d < dim; ++d) {
            trace += vJ[dim * d + d];
            for (int f = 0; f < dim; ++f) stress[dim * d + f] = vJ[dim * d + f] + vJ[dim * f + d];
        }
        for (int d = 0; d < dim; ++d) stress[dim * d + d] += lam * trace;
        double vt = mx(0, W[dim + 2] / rho);
        Vec vtDer(dim);
        for (int d = 0; d < dim; ++d) vtDer[d] = 1 / rho * (dW[d * nEqs_ + dim + 2] - dW[d * nEqs_] * vt);
        double xi = rho * vt;
        double fv1 = xi * xi * xi / (xi * xi * xi + cv1 * cv1 * cv1);
        double mut = rho * vt * fv1;
        double constant = kapa / (kapa - 1) * (1 / Pr + mut / Prt);
        Vec flux(nEqs_, 0.0);
        for (int d = 0; d < dim; ++d) {
            double tmp = .0;
            for (int f = 0; f < dim; ++f) {
                flux[f + 1] += (1 + mut) * stress[dim * d + f] * n[d] / Re;
                tmp += velocity[f] * (1 + mut) * stress[dim * d + f];
            }
            flux[dim + 1] += (tmp + constant * pOverRhoDer[d]) * n[d] / Re;
            flux[dim + 2] += 1 / (Re * sigma) * (1 + rho * vt) * vtDer[d] * n[d];
        }
        return flux;
    }
    Vec numericalDiffusiveFlux(Vec& Wc, const Vec& dWc, const Vec& n, int TT, ElementData& elem) override {
        Wc[0] = limiteRho(Wc[0]);
        Vec flux = diffusiveFlux(Wc, dWc, n, elem);
        if (TT < 0) {
            if (TT == WALL) {
                double work = .0;
                for (int d = 0; d < dim_; ++d) work += elem.meshVelocity[d] * flux[d + 1];
                flux[dim_ + 1] = work;
            } else {
                std::fill(flux.begin(), flux.end(), 0.0);
            }
        }
        return flux;
    }
    // SpalartAllmaras.sourceTerm, SpalartAllmaras.java:391-451
    Vec sourceTerm(Vec& W, const Vec& dW, ElementData& elem) override {
        W[0] = limiteRho(W[0]);
        double rho = W[0];
        double lam = -2. / 3;
        int dim = dim_;
        Vec velocity(dim);
        for (int d = 0; d < dim; ++d) velocity[d] = W[d + 1] / rho;
        Vec vJ(dim * dim);
        for (int d = 0; d < dim; ++d)
            for (int f = 0; f < dim; ++f) vJ[dim * d + f] = (dW[f * nEqs_ + d + 1] - dW[f * nEqs_] * velocity[d]) / rho;
        Vec stress(dim * dim);
        double trace = .0;
        for (int d = 0; d < dim; ++d) {
            trace += vJ[dim * d + d];
            for (int f = 0; f < dim; ++f) stress[dim * d + f] = vJ[dim * d + f] + vJ[dim * f + d];
        }
        for (int d = 0; d < dim; ++d) stress[dim * d + d] += lam * trace;
        double vt = mx(0, W[dim + 2] / rho);
        double vtDerMag = 0;
        for (int d = 0; d < dim; ++d) {
            double vtDer = 1 / rho * (dW[d * nEqs_ + dim + 2] - dW[d * nEqs_] * vt);
            vtDerMag += vtDer * vtDer;
        }
        if (vt < 0) vt = 0;
        double D = elem.currentWallDistance;
        double xi = rho * vt;
        double ft2 = 0;
        double fv1 = xi * xi * xi / (xi * xi * xi + cv1 * cv1 * cv1);
        double fv2 = 1 - xi / (1 + xi * fv1);
        double Om = 0;
        if (dim * dim == 4)
            Om = std::fabs(vJ[1] - vJ[2]);
        else if (dim * dim == 9)
            Om = std::sqrt((vJ[0 * dim + 1] - vJ[1 * dim + 0]) * (vJ[0 * dim + 1] - vJ[1 * dim + 0]) +
                           (vJ[0 * dim + 2] - vJ[2 * dim + 0]) * (vJ[0 * dim + 2] - vJ[2 * dim + 0]) +
                           (vJ[2 * dim + 1] - vJ[1 * dim + 2]) * (vJ[2 * dim + 1] - vJ[1 * dim + 2]));
        double S = Om + 1 / Re * vt / (ka * ka * D * D) * fv2;
        double rt = std::min(vt / (Re * S * ka * ka * D * D), 10.0);
        double g = rt + cw2 * (std::pow(rt, 6.0) - rt);
        double fw = g * std::pow((1 + std::pow(cw3, 6.0)) / (std::pow(g, 6.0) + std::pow(cw3, 6.0)), 1.0 / 6);
        Vec source(nEqs_, 0.0);
        double d = 1 / Re * rho * cb2 * vtDerMag + cb1 * (1 - ft2) * rho * S * vt -
                   1 / Re * (cw1 * fw - cb1 / (ka * ka) * ft2) / rho * (rho * vt / D) * (rho * vt / D);
        if (d < -100) d = -100;
        source[dim + 2] = d;
        return source;
    }
};

// FlowPro/src/test/java/flowpro/user/equation/TestScalarEquation.java (the reference
// tests' manufactured-solution equation, u = sin(2x + y))
struct TestScalarEquation : Equation {
    int dim_ = 2;
    Vec a;
    double k = 0, lambda = 0;
    void init(const Props& props) {
        dim_ = (int)getD(props, "dimension");
        a = getDA(props, "a");
        k = has(props, "k") ? getD(props, "k") : 0;
        double nrm = 0;
        for (double ad : a) nrm += ad * ad;
        lambda = std::sqrt(nrm);
    }
    static double exact(const Vec& x) { return std::sin(2 * x[0] + x[1]); }
    int dim() const override { return dim_; }
    int nEqs() const override { return 1; }
    bool isDiffusive() const override { return k > 0; }
    bool isSourcePresent() const override { return true; }
    Vec boundaryValue(Vec&, const Vec&, int, ElementData& e) override { return Vec{exact(e.currentX)}; }
    Vec convectiveFlux(Vec& W, const Vec& n, ElementData&) override {
        double an = 0;
        for (int d = 0; d < dim_; d++) an += a[d] * n[d];
        return Vec{an * W[0]};
    }
    Vec numericalConvectiveFlux(Vec& WL, Vec& WR, const Vec& n, int, ElementData& e) override {
        double fL = convectiveFlux(WL, n, e)[0];
        double fR = convectiveFlux(WR, n, e)[0];
        return Vec{(fL + fR) / 2 - lambda * (WR[0] - WL[0]) / 2};
    }
    Vec diffusiveFlux(Vec&, const Vec& dW, const Vec& n, ElementData&) override {
        double flux = 0;
        for (int d = 0; d < dim_; d++) flux += k * dW[d] * n[d];
        return Vec{flux};
    }
    Vec numericalDiffusiveFlux(Vec& W, const Vec& dW, const Vec& n, int, ElementData& e) override {
        return diffusiveFlux(W, dW, n, e);
    }
    Vec sourceTerm(Vec&, const Vec&, ElementData& e) override {
        double phase = 2 * e.currentX[0] + e.currentX[1];
        return Vec{(2 * a[0] + a[1]) * std::cos(phase) + 5 * k * std::sin(phase)};
    }
    double maxEigenvalue(Vec&, ElementData*) override { return lambda; }
    bool isIPFace(int) const override { return true; }
    bool isAdmissible(const Vec&) const override { return true; }
    Vec combineShockSensors(Vec s) const override { return s; }
    Vec constInitCondition() override { return Vec{0}; }
    double pressure(Vec&) override { return 0; }
    Vec stressVector(Vec&, const Vec&, const Vec&) override { return Vec(dim_, 0.0); }
};

// ModuleProjects/Equations/Aerodynamics/.../AdiabaticEulers.java: isentropic Euler,
// nEqs = dim + 1, p = rho^kappa
struct AdiabaticEulers : Aerodynamics {
    static constexpr double P_TOL = 1e-1;  // AdiabaticEulers.java:10
    void init(const Props& props) {
        int dimension = (int)getD(props, "dimension");
        if (props.count("isInletSupersonic") && getB(props, "isInletSupersonic"))
            throw std::runtime_error("AdiabaticEulers with a supersonic inlet: Aerodynamics.init writes WIn[dim + 1]");
        initAero(props, dimension, dimension + 1, false);
    }
    bool isSourcePresent() const override { return false; }
    // AdiabaticEulers.java:19-22
    bool isAdmissible(const Vec& W) const override { return W[0] > ADMISSIBLE_TOL; }
    // AdiabaticEulers.java:24-33
    double pressure(Vec& W) override {
        W[0] = limiteRho(W[0]);
        double p = std::pow(W[0], kapa);
        if (p < P_TOL) p = P_TOL * std::exp((p - P_TOL) / P_TOL);
        return p;
    }
    // AdiabaticEulers.java:35-95
    Vec boundaryValue(Vec& WL, const Vec& n, int TT, ElementData&) override {
        WL[0] = limiteRho(WL[0]);
        Vec WR(nEqs_, 0.0);
        int dim = dim_;
        switch (TT) {
            case WALL:
            case INVISCID_WALL: {
                WR = WL;
                double nu = 0;
                for (int d = 0; d < dim; ++d) nu += WL[d + 1] * n[d];
                for (int d = 0; d < dim; ++d) WR[d + 1] = WL[d + 1] + n[d] * nu;
                break;
            }
            case INLET: {
                double p = pressure(WL);
                double mach;
                if (p > pIn0)
                    mach = 0;
                else
                    mach = std::sqrt((2 / (kapa - 1)) * (-1 + std::pow(pIn0 / p, (kapa - 1) / kapa)));
                double rhoIn = rhoIn0 * std::pow((1 + ((kapa - 1) / 2) * mach * mach), 1 / (1 - kapa));
                double normalVelocity = mach * std::sqrt((kapa * p) / rhoIn);
                WR[0] = rhoIn;
                for (int d = 0; d < dim; ++d) WR[d + 1] = -rhoIn * normalVelocity * n[d];
                break;
            }
            case OUTLET: {
                double absVelocity = .0;
                for (int d = 0; d < dim; ++d) absVelocity += WL[d + 1] * WL[d + 1];
                absVelocity = std::sqrt(absVelocity) / WL[0];
                double p = pressure(WL);
                double a = std::sqrt(kapa * p / WL[0]);
                double mach = absVelocity / a;
                if (mach < 1) {
                    double rhoOut = std::pow(pOut, 1. / kapa);
                    WR[0] = rhoOut;
                    for (int d = 0; d < dim; ++d) WR[d + 1] = rhoOut * WL[d + 1] / WL[0];
                } else {
                    WR = WL;
                }
                break;
            }
        }
        return WR;
    }
    // AdiabaticEulers.java:97-133
    Vec constInitCondition() override {
        double machIn = std::sqrt(2 / (kapa - 1) * (std::pow((1 / pOut), (kapa - 1) / kapa) - 1));
        double rhoIn = std::pow(1 + ((kapa - 1) / 2) * machIn * machIn, 1 / (1 - kapa));
        double VIn = machIn * std::sqrt((kapa * pOut) / rhoIn);
        Vec vIn(dim_, 0.0);
        double a0 = hasAttack ? attackAngle[0] : 0, a1 = (hasAttack && dim_ == 3) ? attackAngle[1] : 0;
        if (dim_ == 2) {
            vIn[0] = VIn * std::cos(a0);
            vIn[1] = VIn * std::sin(a0);
        } else {
            vIn[0] = VIn * std::cos(a0) * std::cos(a1);
            vIn[1] = VIn * std::sin(a0) * std::cos(a1);
            vIn[2] = VIn * std::sin(a1);
        }
        Vec W(nEqs_, 0.0);
        W[0] = rhoIn;
        for (int d = 0; d < dim_; ++d) W[d + 1] = rhoIn * vIn[d];
        return W;
    }
    // AdiabaticEulers.java:136-176
    Vec numericalConvectiveFlux(Vec& WL, Vec& WR, const Vec& n, int TT, ElementData& elem) override {
        WL[0] = limiteRho(WL[0]);
        WR[0] = limiteRho(WR[0]);
        Vec f(nEqs_, 0.0);
        switch (TT) {
            case WALL:
            case INVISCID_WALL: {
                double p = pressure(WR);
                f[0] = 0;
                double V = .0;
                for (int d = 0; d < dim_; ++d) {
                    f[d + 1] = p * n[d];
                    V += elem.meshVelocity[d] * n[d];
                }
                for (int j = 0; j < nEqs_; j++) f[j] += V * WR[j];
                break;
            }
            case INLET:
            case OUTLET:
                f = convectiveFlux(WR, n, elem);
                break;
            default: {
                Vec fL = convectiveFlux(WL, n, elem);
                Vec fR = convectiveFlux(WR, n, elem);
                double lL = maxEigenvalue(WL, &elem);
                double lR = maxEigenvalue(WR, &elem);
                double maxEigenValue = std::max(lL, lR);
                for (int j = 0; j < nEqs_; j++) f[j] = (fL[j] + fR[j] - maxEigenValue * (WR[j] - WL[j])) / 2;
                break;
            }
        }
        return f;
    }
    // AdiabaticEulers.java:178-195
    Vec convectiveFlux(Vec& W, const Vec& n, ElementData&) override {
        W[0] = limiteRho(W[0]);
        double V = 0.;
        for (int d = 0; d < dim_; ++d) V += W[d + 1] * n[d];
        V /= W[0];
        double p = pressure(W);
        Vec f(nEqs_, 0.0);
        f[0] = W[0] * V;
        for (int d = 0; d < dim_; ++d) f[d + 1] = W[d + 1] * V + p * n[d];
        return f;
    }
    Vec diffusiveFlux(Vec&, const Vec&, const Vec&, ElementData&) override {
        throw std::runtime_error("operation not supported");
    }
    Vec numericalDiffusiveFlux(Vec&, const Vec&, const Vec&, int, ElementData&) override {
        throw std::runtime_error("operation not supported");
    }
    Vec sourceTerm(Vec&, const Vec&, ElementData&) override { throw std::runtime_error("operation not supported"); }
};

static std::unique_ptr<Equation> makeEquation(const Props& props) {
    std::string model = props.at("model");
    if (model == "NavierStokes") {
        auto e = std::make_unique<NavierStokes>();
        e->init(props);
        return e;
    }
    if (model == "SpalartAllmaras") {
        auto e = std::make_unique<SpalartAllmaras>();
        e->init(props);
        return e;
    }
    if (model == "AdiabaticEulers") {
        auto e = std::make_unique<AdiabaticEulers>();
        e->init(props);
        return e;
    }
    if (model == "TestScalarEquation") {
        auto e = std::make_unique<TestScalarEquation>();
        e->init(props);
        return e;
    }
    throw std::runtime_error("unsupported model " + model);
}

}  // namespace orc
