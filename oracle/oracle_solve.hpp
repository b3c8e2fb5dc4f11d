// CPU ORACLE (test infrastructure) — time integration, sparse matrix, GMRES,
// preconditioners and the local solver loops of FlowPro_v2:
// flowpro/core/element/{BDF1,BDF2,RK3}.java, flowpro/core/LinearSolvers/*,
// flowpro/core/{State,solver/CFLSetup,solver/LocalImplicitSolver,solver/LocalExplicitSolver,
// solver/MasterSolver}.java
#pragma once
#include "oracle_dg.hpp"
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// BDF2.coefficients, BDF2.java:298-308 (dto <= 0: first step is BDF1); dt <= 0: the steady
// operator of the optimisation export (no mass term, Element.exportLocalJacobiMatrix,
// Element.java:750-786)
static Vec bdfCoefficients(int order, double dt, double dto) {
    if (!(dt > 0)) return Vec{0, 0, 0};
    if (order == 2 && dto > 0)
        return Vec{(2 * dt + dto) / (dt * (dt + dto)), -(dt + dto) / (dt * dto), dt / (dto * (dt + dto))};
    return Vec{1 / dt, -1 / dt, 0};
}

// Deformation2DTest (meshDeformation/Deformation2DTest.java:26-73): a prescribed deformation
// x = x0 + A sin(2 pi t / t0) sin(2 pi x0 / L) sin(2 pi y0 / L) in both components, the
// vertex velocity by the BDF difference of the positions.  Its time advances by dt at every
// call, i.e. at every Newton iteration, as in the reference.
struct Deformation2DTest {
    double t = 0;
    void newMeshPositionAndVelocity(std::vector<Element>& elems, int timeOrder, double dt, double dto) {
        if (dt > 1000) dt = 0;
        double a1 = 1.0 / dt, a2 = -1.0 / dt, a3 = 0;
        if (timeOrder > 1 && dto > 0) {
            a1 = (2 * dt + dto) / (dt * (dt + dto));
            a2 = -(dt + dto) / (dt * dto);
            a3 = dt / (dto * (dt + dto));
        }
        t = t + dt;
        const double L = 20, t0 = 10, A = 2;
        const double pi = 3.14159265358979323846;  // Math.PI
        for (auto& e : elems)
            for (int j = 0; j < e.nVertices; j++) {
                const double s = A * std::sin(2 * pi * t / t0) * std::sin(2 * pi * e.vertices0[j][0] / L) *
                                 std::sin(2 * pi * e.vertices0[j][1] / L);
                e.vertices[j][0] = e.vertices0[j][0] + s;
                e.vertices[j][1] = e.vertices0[j][1] + s;
                for (int d = 0; d < e.dim; d++)
                    e.U[j][d] = a1 * e.vertices[j][d] + a2 * e.verticesOld[j][d] + a3 * e.verticesOld2[j][d];
            }
    }
    void nextTimeLevel(std::vector<Element>& elems) {
        for (auto& e : elems) {
            e.verticesOld2 = e.verticesOld;
            e.verticesOld = e.vertices;
        }
    }
    // Deformation.relaxFirstIteration, Deformation.java:64-76
    void relaxFirstIteration(std::vector<Element>& elems, double dt) {
        for (auto& e : elems)
            for (int j = 0; j < e.nVertices; j++)
                for (int d = 0; d < e.dim; d++) {
                    e.verticesOld2[j][d] = e.vertices[j][d] - 2 * dt * e.Uinit[j][d];
                    e.verticesOld[j][d] = e.vertices[j][d] - dt * e.Uinit[j][d];
                    e.U[j][d] = e.Uinit[j][d];
                }
    }
};

struct Solver {
    Mesh& mesh;
    Deformation2DTest dfm;
    std::vector<Element>& elems;
    explicit Solver(Mesh& m) : mesh(m), elems(m.elems) {}

    // ---------------------------------------------------------- residual
    // Implicit.assembleResiduum (BDF1.java:178-184, BDF2.java:310-317) -> spatialResiduum, RHS_loc
    void assembleRHS(Element& e, const Vec& Rw, double a1, double a2, double a3) {
        e.RHS_loc = Rw;
        e.spatialResiduum = Rw;
        int nB = e.nBasis;
        for (int m = 0; m < e.nEqs; m++)
            for (int i = 0; i < nB; i++)
                for (int j = 0; j < nB; j++)
                    e.RHS_loc[nB * m + i] -= e.M[i][j] * a1 * e.W[m * nB + j] + e.Mo[i][j] * a2 * e.Wo[m * nB + j] +
                                             e.Mo2[i][j] * a3 * e.Wo2[m * nB + j];
    }

    void assembleResiduum(double dt, double dto) {
        Vec a = bdfCoefficients(mesh.par.timeOrder, dt, dto);
#pragma omp parallel for schedule(dynamic, 64)
        for (int i = 0; i < (int)elems.size(); i++) {
            Element& e = elems[i];
            int nb = e.nEqs * e.nBasis;
            Vec Rw(nb, 0.0), V(nb, 0.0);
            std::vector<Vec*> KR(e.nFaces, nullptr);
            e.residuum(V, Rw, KR);
            if (mesh.par.movingMesh && mesh.par.gcl) e.applyGCLMassMatrix(a[0], a[1], a[2]);  // Implicit.applyGCL
            assembleRHS(e, Rw, a[0], a[1], a[2]);
        }
    }

    // spatial residuum R(W) only (V = 0), element-major layout [e][m*nB+j]
    void spatialResidual(Vec& out) {
        int nb = elems[0].nEqs * elems[0].nBasis;
        out.assign(elems.size() * nb, 0.0);
#pragma omp parallel for schedule(dynamic, 64)
        for (int i = 0; i < (int)elems.size(); i++) {
            Element& e = elems[i];
            Vec Rw(nb, 0.0), V(nb, 0.0);
            std::vector<Vec*> KR(e.nFaces, nullptr);
            e.residuum(V, Rw, KR);
            std::copy(Rw.begin(), Rw.end(), out.begin() + (size_t)i * nb);
        }
    }

    // BDF2.assembleJacobiMatrix (finite differences), BDF2.java:320-379
    void assemble(double dt, double dto) {
        Vec a = bdfCoefficients(mesh.par.timeOrder, dt, dto);
        double a1 = a[0];
#pragma omp parallel for schedule(dynamic, 16)
        for (int ei = 0; ei < (int)elems.size(); ei++) {
            Element& e = elems[ei];
            int nb = e.nEqs * e.nBasis;
            Vec V(nb, 0.0), Rw(nb, 0.0);
            std::vector<Vec> RwNeigh(e.nFaces), RwNeighH(e.nFaces);
            std::vector<Vec*> KR(e.nFaces, nullptr), KRH(e.nFaces, nullptr);
            for (int k = 0; k < e.nFaces; k++)
                if (e.TT[k] > -1) {
                    RwNeigh[k].assign(elems[e.TT[k]].nBasis * e.nEqs, 0.0);
                    RwNeighH[k].assign(elems[e.TT[k]].nBasis * e.nEqs, 0.0);
                    KR[k] = &RwNeigh[k];
                    KRH[k] = &RwNeighH[k];
                }
            e.residuum(V, Rw, KR);
            if (mesh.par.movingMesh && mesh.par.gcl) e.applyGCLMassMatrix(a[0], a[1], a[2]);  // Implicit.applyGCL
            assembleRHS(e, Rw, a[0], a[1], a[2]);
            double h = mesh.par.h;
            for (int i = 0; i < nb; i++) {
                for (int j = 0; j < nb; j++) e.ADiag[i][j] = -Rw[j];
                V[i] = h;
                e.residuum(V, e.ADiag[i], KRH);
                V[i] = 0;
                for (int k = 0; k < e.nFaces; k++)
                    if (e.TT[k] > -1) {
                        // neighbour block of element TT[k] (its face faceIndexReverse[k]); each
                        // element writes only rows i of its own perturbations -> no race
                        Mat2& Aaux = elems[e.TT[k]].ANeighs[e.faceIndexReverse[k]];
                        for (size_t j = 0; j < RwNeighH[k].size(); j++) Aaux[i][j] = (RwNeighH[k][j] - RwNeigh[k][j]) / h;
                    }
            }
            for (auto& row : e.ADiag)
                for (auto& v : row) v /= -h;
            int nB = e.nBasis;
            for (int m = 0; m < e.nEqs; m++)
                for (int i = 0; i < nB; i++)
                    for (int j = 0; j < nB; j++) e.ADiag[nB * m + i][nB * m + j] += a1 * e.M[i][j];
        }
    }

    // ---------------------------------------------------------- sparse matrix (SparseMatrix.java)
    int dofs = 0;
    IVec Icrs, Jcrs, diagind;
    Vec H;
    void buildMatrix() {
        dofs = mesh.dofs;
        std::vector<std::pair<long long, double>> coo;
        for (auto& e : elems) {
            int n = e.nEqs * e.nBasis;
            for (int i = 0; i < n; i++)
                for (int j = 0; j < n; j++) coo.push_back({(long long)e.gIndex[i] * dofs + e.gIndex[j], e.ADiag[j][i]});
            for (int k = 0; k < e.nFaces; k++)
                if (e.TT[k] > -1) {
                    Element& nb = elems[e.TT[k]];
                    int ne = e.nEqs * nb.nBasis;
                    for (int i = 0; i < n; i++)
                        for (int j = 0; j < ne; j++)
                            coo.push_back({(long long)e.gIndex[i] * dofs + nb.gIndex[j], e.ANeighs[k][j][i]});
                }
        }
        std::sort(coo.begin(), coo.end(), [](auto& a, auto& b) { return a.first < b.first; });
        size_t nnz = coo.size();
        Icrs.assign(dofs + 1, 0);
        Jcrs.resize(nnz);
        H.resize(nnz);
        for (size_t s = 0; s < nnz; s++) {
            int r = (int)(coo[s].first / dofs);
            Jcrs[s] = (int)(coo[s].first % dofs);
            H[s] = coo[s].second;
            Icrs[r + 1]++;
        }
        for (int r = 0; r < dofs; r++) Icrs[r + 1] += Icrs[r];
        diagind.assign(dofs, 0);
        for (int r = 0; r < dofs; r++)
            for (int s = Icrs[r]; s < Icrs[r + 1]; s++)
                if (Jcrs[s] == r) diagind[r] = s;
    }
    void updateB(Vec& b) {
        b.assign(dofs, 0.0);
        for (auto& e : elems)
            for (size_t i = 0; i < e.gIndex.size(); i++) b[e.gIndex[i]] = e.RHS_loc[i];
    }
    void Mult(Vec& y, const Vec& x) const {
#pragma omp parallel for
        for (int i = 0; i < dofs; i++) {
            double sum = 0;
            for (int j = Icrs[i]; j < Icrs[i + 1]; j++) sum += H[j] * x[Jcrs[j]];
            y[i] = sum;
        }
    }
    void SubstrMult(Vec& y, const Vec& b, const Vec& x) const {
#pragma omp parallel for
        for (int i = 0; i < dofs; i++) {
            double sum = b[i];
            for (int j = Icrs[i]; j < Icrs[i + 1]; j++) sum -= H[j] * x[Jcrs[j]];
            y[i] = sum;
        }
    }

    // ---------------------------------------------------------- preconditioners
    std::string precKind;
    std::vector<Mat2> blockLU;  // per element: LU (no pivoting) of the untransposed diagonal block
    std::vector<Mat2> diagInv;  // BlockJacobiInversion
    Vec ilu;
    // BlockILU0 state (BlockILU0.java:22-243)
    IVec bRankElem, bRank;
    std::vector<IVec> bCols;
    IVec bDiag;
    std::vector<std::vector<Mat2>> bBlocks;
    std::vector<Mat2> bDiagInv;

    bool factor() {
        if (precKind == "blockjacobi") {
            // blockJacobi.apply solves ADiag^T y = b by Gaussian elimination without pivoting
            // (Mat.lsolveT).  Here the elimination is done once per factor(), i.e. every apply
            // uses the full LU; with blockJacobiQuirk the in-place reuse of Mat.lsolveT
            // (later applies see only U, Mat.java:1307-1329) is reproduced instead.
            blockLU.assign(elems.size(), Mat2());
            for (size_t i = 0; i < elems.size(); i++) {
                Element& e = elems[i];
                int n = (int)e.ADiag.size();
                Mat2 A = zeros(n, n);  // A[row][col] = ADiag[col][row]
                for (int r = 0; r < n; r++)
                    for (int c = 0; c < n; c++) A[r][c] = e.ADiag[c][r];
                if (mesh.par.blockJacobiQuirk) {
                    blockLU[i] = e.ADiag;  // kept transposed, eliminated lazily in apply
                    continue;
                }
                for (int p = 0; p < n; p++) {
                    if (A[p][p] == 0) return false;
                    for (int r = p + 1; r < n; r++) {
                        double alpha = A[r][p] / A[p][p];
                        A[r][p] = alpha;
                        for (int c = p + 1; c < n; c++) A[r][c] -= alpha * A[p][c];
                    }
                }
                blockLU[i] = A;
            }
        } else if (precKind == "blockjacobiinversion") {
            diagInv.assign(elems.size(), Mat2());
            for (size_t i = 0; i < elems.size(); i++) diagInv[i] = invert(elems[i].ADiag);
        } else if (precKind == "ilu0") {
            // ILU0.factor, ILU0.java:34-68
            ilu = H;
            for (int k = 1; k < dofs; ++k)
                for (int i = Icrs[k]; i < diagind[k]; ++i) {
                    int index = Jcrs[i];
                    double LUii = ilu[diagind[index]];
                    if (LUii == 0) return false;
                    double LUki = (ilu[i] /= LUii);
                    for (int j = diagind[index] + 1, l = Icrs[k] + 1; j < Icrs[index + 1]; ++j) {
                        while (l < Icrs[k + 1] && Jcrs[l] < Jcrs[j]) l++;
                        if (l < Icrs[k + 1] && Jcrs[l] == Jcrs[j]) ilu[l] -= LUki * ilu[j];
                    }
                }
        } else if (precKind == "blockilu0") {
            return factorBlockILU0();
        }
        return true;
    }

    bool factorBlockILU0() {
        int nElem = (int)elems.size();
        IVec byDofs(nElem);
        for (int i = 0; i < nElem; i++) byDofs[i] = i;
        std::stable_sort(byDofs.begin(), byDofs.end(), [&](int a, int b) { return elems[a].gIndex[0] < elems[b].gIndex[0]; });
        bRankElem = byDofs;
        bRank.assign(nElem, 0);
        for (int r = 0; r < nElem; r++) bRank[byDofs[r]] = r;
        bCols.assign(nElem, IVec());
        bDiag.assign(nElem, 0);
        bBlocks.assign(nElem, std::vector<Mat2>());
        bDiagInv.assign(nElem, Mat2());
        for (int i = 0; i < nElem; i++) {
            Element& e = elems[bRankElem[i]];
            IVec row{i};
            for (int k = 0; k < e.nFaces; k++) {
                int t = e.TT[k];
                if (t > -1 && std::find(row.begin(), row.end(), bRank[t]) == row.end()) row.push_back(bRank[t]);
            }
            std::sort(row.begin(), row.end());
            bCols[i] = row;
            bDiag[i] = (int)(std::lower_bound(row.begin(), row.end(), i) - row.begin());
            int n = e.nEqs * e.nBasis;
            bBlocks[i].assign(row.size(), Mat2());
            for (size_t k = 0; k < row.size(); k++) {
                Element& c = elems[bRankElem[row[k]]];
                bBlocks[i][k] = zeros(n, c.nEqs * c.nBasis);
            }
            // copyBlocks: blocks hold untransposed values
            auto addT = [](Mat2& B, const Mat2& At) {
                for (size_t r = 0; r < B.size(); r++)
                    for (size_t c = 0; c < B[r].size(); c++) B[r][c] += At[c][r];
            };
            addT(bBlocks[i][bDiag[i]], e.ADiag);
            for (int k = 0; k < e.nFaces; k++) {
                int t = e.TT[k];
                if (t > -1) {
                    int kk = (int)(std::lower_bound(row.begin(), row.end(), bRank[t]) - row.begin());
                    addT(bBlocks[i][kk], e.ANeighs[k]);
                }
            }
        }
        for (int i = 0; i < nElem; i++) {
            IVec& row = bCols[i];
            for (int kk = 0; kk < bDiag[i]; kk++) {
                int k = row[kk];
                Mat2 L = times(bBlocks[i][kk], bDiagInv[k]);
                bBlocks[i][kk] = L;
                for (size_t jj = kk + 1; jj < row.size(); jj++) {
                    auto it = std::lower_bound(bCols[k].begin(), bCols[k].end(), row[jj]);
                    if (it != bCols[k].end() && *it == row[jj]) {
                        int kj = (int)(it - bCols[k].begin());
                        Mat2& C = bBlocks[i][jj];
                        const Mat2& B = bBlocks[k][kj];
                        for (size_t r = 0; r < C.size(); r++)
                            for (size_t m = 0; m < B.size(); m++) {
                                double a = L[r][m];
                                if (a != 0)
                                    for (size_t c = 0; c < C[r].size(); c++) C[r][c] -= a * B[m][c];
                            }
                    }
                }
            }
            bDiagInv[i] = invert(bBlocks[i][bDiag[i]]);
            for (auto& r : bDiagInv[i])
                for (double v : r)
                    if (!std::isfinite(v)) return false;
        }
        return true;
    }

    void apply(Vec& x, const Vec& b) {
        if (precKind == "none") {
            x = b;
        } else if (precKind == "blockjacobi") {
#pragma omp parallel for
            for (int i = 0; i < (int)elems.size(); i++) {
                Element& e = elems[i];
                int n = (int)e.gIndex.size();
                Vec bp(n);
                for (int j = 0; j < n; j++) bp[j] = b[e.gIndex[j]];
                Vec y;
                if (mesh.par.blockJacobiQuirk) {
                    y = lsolveT(blockLU[i], bp);
                } else {
                    Mat2& A = blockLU[i];
                    for (int r = 1; r < n; r++)
                        for (int c = 0; c < r; c++) bp[r] -= A[r][c] * bp[c];
                    y.assign(n, 0.0);
                    for (int r = n - 1; r >= 0; r--) {
                        double s = 0;
                        for (int c = r + 1; c < n; c++) s += A[r][c] * y[c];
                        y[r] = (bp[r] - s) / A[r][r];
                    }
                }
                for (int j = 0; j < n; j++) x[e.gIndex[j]] = y[j];
            }
        } else if (precKind == "blockjacobiinversion") {
            for (size_t i = 0; i < elems.size(); i++) {
                Element& e = elems[i];
                int n = (int)e.gIndex.size();
                for (int j = 0; j < n; j++) {
                    double s = 0;
                    for (int k = 0; k < n; k++) s += diagInv[i][k][j] * b[e.gIndex[k]];
                    x[e.gIndex[j]] = s;
                }
            }
        } else if (precKind == "ilu0") {
            // ILU0.apply, ILU0.java:70-96
            Vec y(dofs, 0.0);
            std::fill(x.begin(), x.end(), 0.0);
            for (int i = 0; i < dofs; i++) {
                double sum = 0;
                for (int j = Icrs[i]; j < diagind[i]; j++) sum = sum + ilu[j] * y[Jcrs[j]];
                y[i] = b[i] - sum;
            }
            for (int i = dofs - 1; i >= 0; i--) {
                double sum = 0;
                for (int j = diagind[i] + 1; j < Icrs[i + 1]; j++) sum = sum + ilu[j] * x[Jcrs[j]];
                x[i] = (y[i] - sum) / ilu[diagind[i]];
            }
        } else if (precKind == "blockilu0") {
            // BlockILU0.apply, BlockILU0.java:131-185
            int nElem = (int)elems.size();
            std::vector<Vec> y(nElem);
            for (int i = 0; i < nElem; i++) {
                IVec& row = bCols[i];
                Element& e = elems[bRankElem[i]];
                Vec yi(e.gIndex.size());
                for (size_t r = 0; r < yi.size(); r++) yi[r] = b[e.gIndex[r]];
                for (int kk = 0; kk < bDiag[i]; kk++) {
                    Mat2& L = bBlocks[i][kk];
                    Vec& yk = y[row[kk]];
                    for (size_t r = 0; r < yi.size(); r++) {
                        double s = 0;
                        for (size_t c = 0; c < yk.size(); c++) s += L[r][c] * yk[c];
                        yi[r] -= s;
                    }
                }
                y[i] = yi;
            }
            for (int i = nElem - 1; i >= 0; i--) {
                IVec& row = bCols[i];
                Vec rhs = y[i];
                for (size_t jj = bDiag[i] + 1; jj < row.size(); jj++) {
                    Mat2& Um = bBlocks[i][jj];
                    IVec& gj = elems[bRankElem[row[jj]]].gIndex;
                    for (size_t r = 0; r < rhs.size(); r++) {
                        double s = 0;
                        for (size_t c = 0; c < gj.size(); c++) s += Um[r][c] * x[gj[c]];
                        rhs[r] -= s;
                    }
                }
                Mat2& iU = bDiagInv[i];
                IVec& gi = elems[bRankElem[i]].gIndex;
                for (size_t r = 0; r < rhs.size(); r++) {
                    double s = 0;
                    for (size_t c = 0; c < rhs.size(); c++) s += iU[r][c] * rhs[c];
                    x[gi[r]] = s;
                }
            }
        }
    }

    // ---------------------------------------------------------- GMRES (Gmres.java:42-199)
    int lastIters = 0;
    double lastError = 0;
    static double norm(const Vec& a) {
        double s = 0;
        for (double v : a) s += v * v;
        return std::sqrt(s);
    }
    static double dot(const Vec& a, const Vec& b) {
        double s = 0;
        for (size_t i = 0; i < a.size(); i++) s += a[i] * b[i];
        return s;
    }
    static void rotmat(double a, double b, double& c, double& s) {
        if (b == 0) {
            c = 1;
            s = 0;
        } else if (std::fabs(b) > std::fabs(a)) {
            double t = a / b;
            s = 1 / std::sqrt(1 + t * t);
            c = t * s;
        } else {
            double t = b / a;
            c = 1 / std::sqrt(1 + t * t);
            s = t * c;
        }
    }
    static Vec lsolve(Mat2& A, Vec& b, int N) {
        for (int p = 0; p < N; p++)
            for (int i = p + 1; i < N; i++) {
                double alpha = A[i][p] / A[p][p];
                b[i] -= alpha * b[p];
                for (int j = p; j < N; j++) A[i][j] -= alpha * A[p][j];
            }
        Vec x(N);
        for (int i = N - 1; i >= 0; i--) {
            double sum = 0.0;
            for (int j = i + 1; j < N; j++) sum += A[i][j] * x[j];
            x[i] = (b[i] - sum) / A[i][i];
        }
        return x;
    }
    bool gmres(Vec& x, const Vec& b, int m, int iterationLimit, double tol) {
        int n = dofs;
        Mat2 V(m + 1, Vec(n, 0.0)), Hh = zeros(m + 1, m);
        Vec cs(m), sn(m), e1(m + 1, 0.0), w(n), r(n), aux(n), s;
        apply(r, b);
        double bnrm2 = norm(r);
        if (bnrm2 == 0) bnrm2 = 1;
        SubstrMult(aux, b, x);
        apply(r, aux);
        double error = norm(r) / bnrm2;
        lastIters = 0;
        if (error < tol) {
            lastError = error;
            return true;
        }
        e1[0] = 1;
        for (int iter = 0; iter < iterationLimit; iter++) {
            double norm_r = norm(r);
            for (int j = 0; j < n; j++) V[0][j] = r[j] / norm_r;
            s.assign(std::max(n, m + 1), 0.0);
            for (int i = 0; i <= m; i++) s[i] = e1[i] * norm_r;
            for (int i = 0; i < m; i++) {
                lastIters++;
                Mult(aux, V[i]);
                apply(w, aux);
                for (int k = 0; k <= i; k++) {
                    Hh[k][i] = dot(w, V[k]);
                    for (int j = 0; j < n; j++) w[j] = w[j] - V[k][j] * Hh[k][i];
                }
                Hh[i + 1][i] = norm(w);
                double hNorm = Hh[i + 1][i];
                for (int j = 0; j < n; j++) V[i + 1][j] = hNorm > 0 ? w[j] / hNorm : 0;
                for (int k = 0; k <= i - 1; k++) {
                    double temp = cs[k] * Hh[k][i] + sn[k] * Hh[k + 1][i];
                    Hh[k + 1][i] = -sn[k] * Hh[k][i] + cs[k] * Hh[k + 1][i];
                    Hh[k][i] = temp;
                }
                rotmat(Hh[i][i], Hh[i + 1][i], cs[i], sn[i]);
                double temp = cs[i] * s[i];
                s[i + 1] = -sn[i] * s[i];
                s[i] = temp;
                Hh[i][i] = cs[i] * Hh[i][i] + sn[i] * Hh[i + 1][i];
                Hh[i + 1][i] = 0;
                error = std::fabs(s[i + 1]) / bnrm2;
                if (error <= tol) {
                    Vec y = lsolve(Hh, s, i + 1);
                    for (int j = 0; j < n; j++)
                        for (int k = 0; k <= i; k++) x[j] += V[k][j] * y[k];
                    break;
                }
            }
            if (error <= tol) break;
            Vec y = lsolve(Hh, s, m);
            for (int j = 0; j < n; j++)
                for (int k = 0; k <= m - 1; k++) x[j] += V[k][j] * y[k];
            SubstrMult(aux, b, x);
            apply(r, aux);
            s[m] = norm(r);
            error = s[m] / bnrm2;
            if (error <= tol) break;
        }
        lastError = error;
        return error <= tol;
    }

    // LinearSolver.solve, LinearSolver.java:291-311 (matrix from the element blocks)
    bool linearSolve(Vec& x, const std::string& prec, double tol) {
        buildMatrix();
        Vec b;
        updateB(b);
        precKind = prec;
        if (!factor()) return false;
        x.assign(dofs, 0.0);
        bool flag = gmres(x, b, mesh.par.gmresRestart, mesh.par.gmresRestarts, tol);
        for (double v : x)
            if (!std::isfinite(v)) return false;
        return flag;
    }

    // ---------------------------------------------------------- state / CFL
    // State.java + CFLSetup.java
    struct State {
        int steps = 0;
        double t = 0, currentCFL = 0, residuum = std::numeric_limits<double>::max(), dt = 0, dt0 = 0;
        Vec equationResiduum, residuumNormalisation;
        int nNorm = 0;
        double cfl = 1, maxCFL = 1, resOld = -1;
        bool varyCFL = false, fixed = false;
        double getCFL(double actual, double res) {
            if (!varyCFL) return std::min(actual + cfl / 20, cfl);
            bool known = res > 0 && res < std::numeric_limits<double>::max();
            if (actual <= 0) {
                resOld = known ? res : -1;
                return cfl;
            }
            double factor = 1;
            const double MAX_FACTOR = 2;
            if (known && resOld > 0) factor = std::max(1 / MAX_FACTOR, std::min(resOld / res, MAX_FACTOR));
            resOld = known ? res : -1;
            double lower = std::min(actual, cfl);
            return std::max(lower, std::min(actual * factor, maxCFL));
        }
        void updateCFL() {
            if (fixed)
                dt = std::min(2 * dt, dt0);
            else
                currentCFL = getCFL(currentCFL, residuum);
        }
        void reduceCFL() {
            if (fixed)
                dt /= 2;
            else {
                resOld = -1;
                currentCFL = currentCFL / 1.5;
            }
        }
        bool hopeless() const { return fixed ? dt < dt0 / 1024 : (currentCFL > 0 && currentCFL < cfl / 20); }
        void setResiduum(const Vec& norms) {
            int nE = (int)norms.size();
            if ((int)residuumNormalisation.size() != nE) {
                residuumNormalisation.assign(nE, 0.0);
                nNorm = 0;
            }
            if (nNorm < 5) {
                for (int m = 0; m < nE; m++) residuumNormalisation[m] = std::max(residuumNormalisation[m], norms[m]);
                nNorm++;
            }
            double mxn = 0;
            for (double r : residuumNormalisation) mxn = std::max(mxn, r);
            equationResiduum.assign(nE, 0.0);
            residuum = 0;
            for (int m = 0; m < nE; m++) {
                double nrm = residuumNormalisation[m] > 0 ? residuumNormalisation[m] : mxn;
                equationResiduum[m] = nrm > 0 ? norms[m] / nrm : norms[m];
                if (std::isnan(equationResiduum[m]))
                    residuum = NAN;
                else if (!std::isnan(residuum))
                    residuum = std::max(residuum, equationResiduum[m]);
            }
        }
    };
    State state;

    void initState() {
        state = State();
        state.cfl = mesh.par.cfl;
        state.maxCFL = mesh.par.maxCFL;
        state.varyCFL = mesh.par.varyCFL;
        state.fixed = mesh.par.isTimeStepFixed;
        state.dt0 = mesh.par.dt;
        if (state.fixed) state.dt = state.dt0;
    }

    // State.getTimeStep, State.java:177-193
    double getTimeStep() {
        double temp = std::numeric_limits<double>::max();
        for (auto& e : elems) {
            double lam = e.calculateMaxEigenvalue();
            if (lam > 0) temp = std::min(temp, e.elemSize / lam / e.timeStepOrderFactor());
        }
        if (state.fixed)
            state.currentCFL = state.dt / temp;
        else
            state.dt = state.currentCFL * temp;
        return state.dt;
    }

    // MasterSolver.residuumNorms, MasterSolver.java:113-137
    Vec residuumNorms() {
        int nE = elems[0].nEqs;
        Vec norms(nE, 0.0);
        for (auto& e : elems) {
            Vec en = e.l2NormsSquared(e.spatialResiduum);
            for (int m = 0; m < nE; m++) norms[m] += en[m];
        }
        for (auto& v : norms) v = std::sqrt(v);
        return norms;
    }

    void limiterAll() {
#pragma omp parallel for
        for (int i = 0; i < (int)elems.size(); i++) elems[i].limiter();
    }
    int positivityAll() {
        if (!mesh.par.positivityLimiter) return 0;
        int n = 0;
#pragma omp parallel for reduction(+ : n)
        for (int i = 0; i < (int)elems.size(); i++) n += elems[i].positivityLimiter() ? 1 : 0;
        return n;
    }

    // ---------------------------------------------------------- RK3 (RK3.java:44-86, LocalExplicitSolver.java:248-289)
    void computeInvertMassMatrices() {
        for (auto& e : elems) e.computeInvertMassMatrix();
    }
    void rk3Stage(int step, double dt) {
        if (step % 2 == 1) limiterAll();
#pragma omp parallel for schedule(dynamic, 64)
        for (int i = 0; i < (int)elems.size(); i++) {
            Element& e = elems[i];
            int nb = e.nEqs * e.nBasis;
            Vec V(nb, 0.0), Rw(nb, 0.0);
            std::vector<Vec*> KR(e.nFaces, nullptr);
            switch (step) {
                case 1:
                    e.residuum(V, Rw, KR);
                    e.spatialResiduum = Rw;
                    Rw = times(e.iM, Rw);
                    for (int j = 0; j < nb; j++) e.W1[j] = e.Wo[j] + dt * Rw[j];
                    break;
                case 2: e.W = e.W1; break;
                case 3:
                    e.residuum(V, Rw, KR);
                    Rw = times(e.iM, Rw);
                    for (int j = 0; j < nb; j++) e.W2[j] = 0.75 * e.Wo[j] + 0.25 * (e.W1[j] + dt * Rw[j]);
                    break;
                case 4: e.W = e.W2; break;
                case 5:
                    e.residuum(V, Rw, KR);
                    Rw = times(e.iM, Rw);
                    for (int j = 0; j < nb; j++) e.Wn[j] = 1.0 / 3 * e.Wo[j] + 2.0 / 3 * (e.W2[j] + dt * Rw[j]);
                    break;
                case 6: e.W = e.Wn; break;
            }
        }
        if (step % 2 == 0) positivityAll();
    }

    // LocalExplicitSolver.solve, LocalExplicitSolver.java:115-195 (steps only, no files)
    void runExplicit(int nSteps) {
        computeInvertMassMatrices();
        for (int s = 0; s < nSteps; s++) {
            state.steps++;
            state.updateCFL();
            double dt = getTimeStep();
            for (int st = 1; st <= 6; st++) rk3Stage(st, dt);
            state.setResiduum(residuumNorms());
            state.t += dt;
            for (auto& e : elems) {
                e.Wo2 = e.Wo;
                e.Wo = e.W;
            }
        }
    }

    // LocalImplicitSolver.solve, LocalImplicitSolver.java:107-285 (no files); on a moving mesh
    // (Deformation2DTest) the mesh moves at every Newton iteration and the mass matrices of
    // the time levels shift after every step (LocalImplicitSolver.java:176-187, 246-255)
    int newtonIterationsTotal = 0;
    double rhsNorm() {
        double s = 0;
        for (auto& e : elems)
            for (double v : e.RHS_loc) s += v * v;
        return std::sqrt(s);
    }
    void runImplicit(int nSteps, double targetResiduum) {
        double dto = -1;
        bool converges = true;
        Vec x;
        int total = state.steps + nSteps;
        bool isFirstIter = true;
        for (++state.steps; state.steps <= total && state.residuum > targetResiduum; ++state.steps) {
            if (converges) state.updateCFL();
            if (state.hopeless()) break;
            double dt = getTimeStep();
            limiterAll();
            double rhsNorm0 = 0;
            bool restart = false;
            for (int s = 0; s < mesh.par.newtonIters; s++) {
                if (mesh.par.movingMesh) {
                    dfm.newMeshPositionAndVelocity(elems, mesh.par.timeOrder, dt, dto);
                    if (isFirstIter) dfm.relaxFirstIteration(elems, dt);
                    mesh.recalculateMesh();
                }
                if (s > 0) {
                    assembleResiduum(dt, dto);
                    double rel = rhsNorm0 > 0 ? rhsNorm() / rhsNorm0 : 0;
                    if (rel < mesh.par.newtonIterTol) break;
                }
                assemble(dt, dto);
                if (s == 0) {
                    state.setResiduum(residuumNorms());
                    rhsNorm0 = rhsNorm();
                }
                converges = linearSolve(x, mesh.par.preconditioner, mesh.par.iterativeSolverTol);
                newtonIterationsTotal++;
                if (!converges) {
                    for (auto& e : elems) e.W = e.Wo;
                    state.reduceCFL();
                    --state.steps;
                    restart = true;
                    break;
                }
                for (auto& e : elems)
                    for (size_t i = 0; i < e.W.size(); i++) e.W[i] += x[e.gIndex[i]];
                positivityAll();
            }
            if (restart) continue;
            if (!std::isfinite(state.residuum)) break;
            state.t += dt;
            dto = dt;
            for (auto& e : elems) {
                e.Wo2 = e.Wo;
                e.Wo = e.W;
            }
            if (mesh.par.movingMesh) {
                dfm.nextTimeLevel(elems);
                for (auto& e : elems) e.nextTimeLevelMassMatrixes();
            }
            isFirstIter = false;
        }
        --state.steps;
    }
};

}  // namespace orc
