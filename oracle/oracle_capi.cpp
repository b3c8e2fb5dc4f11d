// CPU ORACLE (test infrastructure) — C entry points used by tests/ and bench.py
// through ctypes.  The product library never links this file.
//
// Parameters are passed as one "key = value; key = value" string with the keys of
// FlowPro's parameters.txt (model, dimension, kappa, cv, pIn0, rhoIn0, pOut,
// isFlowViscous, reynolds, prandtl, attackAngle, order, penalty, beta0, dampTol,
// dampConst, timeMethod, timeOrder, CFL, maxCFL, dt, newtonIters, newtonIterTol,
// iterativeSolverTol, preconditioner, elementOrdering, positivityLimiter, ...).
#include <limits>
#include "oracle_solve.hpp"

using namespace orc;

namespace {

Props parseProps(const char* s) {
    Props p;
    std::string str(s ? s : "");
    std::stringstream ss(str);
    std::string item;
    while (std::getline(ss, item, ';')) {
        auto eq = item.find('=');
        if (eq == std::string::npos) continue;
        auto trim = [](std::string x) {
            size_t a = x.find_first_not_of(" \t\n"), b = x.find_last_not_of(" \t\n");
            return a == std::string::npos ? std::string() : x.substr(a, b - a + 1);
        };
        p[trim(item.substr(0, eq))] = trim(item.substr(eq + 1));
    }
    return p;
}

Params makeParams(const Props& p) {
    Params q;
    q.order = has(p, "order") ? (int)getD(p, "order") : 2;
    q.penalty = has(p, "penalty") ? getD(p, "penalty") : 0;
    q.beta0 = has(p, "beta0") ? getD(p, "beta0") : 2;
    q.dampTol = has(p, "dampTol") ? getD(p, "dampTol") : 0;
    q.dampConst = has(p, "dampConst") ? getD(p, "dampConst") : 0;
    q.positivityLimiter = has(p, "positivityLimiter") ? getB(p, "positivityLimiter") : true;
    q.implicitTime = !(has(p, "timeMethod") && p.at("timeMethod") == "RK");
    q.timeOrder = has(p, "timeOrder") ? (int)getD(p, "timeOrder") : 1;
    q.elementOrdering = has(p, "elementOrdering") ? p.at("elementOrdering") : "rcm";
    q.preconditioner = has(p, "preconditioner") ? p.at("preconditioner") : "blockjacobi";
    q.iterativeSolverTol = has(p, "iterativeSolverTol") ? getD(p, "iterativeSolverTol") : 1e-2;
    q.newtonIters = has(p, "newtonIters") ? (int)getD(p, "newtonIters") : 1;
    q.newtonIterTol = has(p, "newtonIterTol") ? getD(p, "newtonIterTol") : 1e-4;
    if (has(p, "CFL")) {
        q.isTimeStepFixed = false;
        q.cfl = getD(p, "CFL");
        if (q.cfl <= 0) {
            q.varyCFL = true;
            q.cfl = 1;
        }
        q.maxCFL = has(p, "maxCFL") ? getD(p, "maxCFL") : 1e4;
    } else if (has(p, "dt")) {
        q.isTimeStepFixed = true;
        q.dt = getD(p, "dt");
    }
    q.blockJacobiQuirk = has(p, "blockJacobiQuirk") && getB(p, "blockJacobiQuirk");
    q.movingMesh = has(p, "movingMesh") && getB(p, "movingMesh");
    q.gcl = has(p, "gcl") && getB(p, "gcl");
    q.meshDeformationType = has(p, "meshDeformationType") ? p.at("meshDeformationType") : "";
    if (q.movingMesh && q.meshDeformationType != "Test2D")
        throw std::runtime_error("moving mesh: only the Test2D deformation is restated");
    return q;
}

struct Handle {
    Mesh mesh;
    std::unique_ptr<Solver> solver;
    std::string err;
};

thread_local std::string g_err;

}  // namespace

extern "C" {

const char* or_last_error() { return g_err.c_str(); }

void or_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int or_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// FlowProMain.createNeighborMatrix: TT (nElem x nFaces) from elements and boundaryType rows
int or_create_neighbor_matrix(int elemType, int nElem, const int* TP, int nBound, const int* boundary, int* TT) {
    try {
        int nV = numberOfPoints(elemType), nF = numberOfFaces(elemType);
        int nBV = elemType == 3 ? 2 : 3;
        IVec type(nElem, elemType);
        std::vector<IVec> tp(nElem, IVec(nV)), bnd(nBound, IVec(nBV + 1));
        for (int i = 0; i < nElem; i++)
            for (int j = 0; j < nV; j++) tp[i][j] = TP[i * nV + j];
        for (int i = 0; i < nBound; i++)
            for (int j = 0; j <= nBV; j++) bnd[i][j] = boundary[i * (nBV + 1) + j];
        auto tt = createNeighborMatrix(type, tp, bnd);
        for (int i = 0; i < nElem; i++)
            for (int k = 0; k < nF; k++) TT[i * nF + k] = tt[i][k];
        return 0;
    } catch (std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

void* or_create(const char* props, int dim, int nVert, const double* PXY, int nElem, const int* TP, const int* TT,
                const double* wallDistance, const double* UXY) {
    try {
        Props p = parseProps(props);
        auto* h = new Handle();
        int nV = dim + 1, nF = dim + 1;
        Mat2 pxy(nVert, Vec(dim));
        for (int i = 0; i < nVert; i++)
            for (int d = 0; d < dim; d++) pxy[i][d] = PXY[i * dim + d];
        std::vector<IVec> tp(nElem, IVec(nV)), tt(nElem, IVec(nF));
        for (int i = 0; i < nElem; i++) {
            for (int j = 0; j < nV; j++) tp[i][j] = TP[i * nV + j];
            for (int k = 0; k < nF; k++) tt[i][k] = TT[i * nF + k];
        }
        Vec wd;
        if (wallDistance) wd.assign(wallDistance, wallDistance + nVert);
        Mat2 uxy;
        if (UXY) {
            uxy.assign(nVert, Vec(dim));
            for (int i = 0; i < nVert; i++)
                for (int d = 0; d < dim; d++) uxy[i][d] = UXY[i * dim + d];
        }
        h->mesh.build(p, makeParams(p), pxy, tp, tt, wd, UXY ? &uxy : nullptr);
        // initial condition: Element.initCondition with the model's constant state (DGpure.java:74-105)
        Vec w0 = h->mesh.eqn->constInitCondition();
        for (auto& e : h->mesh.elems) {
            int nb = e.nEqs * e.nBasis;
            e.W.assign(nb, 0.0);
            for (int i = 0; i < e.nBasis; i++)
                for (int j = 0; j < e.nEqs; j++) e.W[j * e.nBasis + i] = w0[j];
            e.Wo = e.W;
            e.Wo2 = e.W;
        }
        h->solver = std::make_unique<Solver>(h->mesh);
        h->solver->initState();
        return h;
    } catch (std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void or_destroy(void* hp) { delete (Handle*)hp; }

int or_nbasis(void* hp) { return ((Handle*)hp)->mesh.elems[0].nBasis; }
int or_neqs(void* hp) { return ((Handle*)hp)->mesh.elems[0].nEqs; }
int or_dofs(void* hp) { return ((Handle*)hp)->mesh.dofs; }

void or_get_gindex(void* hp, int* g) {
    auto& el = ((Handle*)hp)->mesh.elems;
    size_t s = 0;
    for (auto& e : el) {
        g[s++] = e.gIndex[0] / (int)e.gIndex.size();
    }
}

// element-major flat state W[e * nE*nB + m*nB + j]; which: 0 = W, 1 = Wo, 2 = Wo2
void or_set_state(void* hp, int which, const double* W) {
    auto& el = ((Handle*)hp)->mesh.elems;
    size_t s = 0;
    for (auto& e : el) {
        Vec& t = which == 0 ? e.W : which == 1 ? e.Wo : e.Wo2;
        for (auto& v : t) v = W[s++];
    }
}
void or_get_state(void* hp, int which, double* W) {
    auto& el = ((Handle*)hp)->mesh.elems;
    size_t s = 0;
    for (auto& e : el) {
        Vec& t = which == 0 ? e.W : which == 1 ? e.Wo : e.Wo2;
        for (auto v : t) W[s++] = v;
    }
}

// per-element eps and c_IP after the limiter
void or_limiter(void* hp, double* eps, double* cip) {
    auto* h = (Handle*)hp;
    h->solver->limiterAll();
    size_t i = 0;
    for (auto& e : h->mesh.elems) {
        if (eps) eps[i] = e.eps;
        if (cip) cip[i] = e.c_IP;
        i++;
    }
}

void or_residual(void* hp, double* R) {
    auto* h = (Handle*)hp;
    Vec out;
    h->solver->spatialResidual(out);
    std::copy(out.begin(), out.end(), R);
}

// element geometry for cross-checks: area, elemSize, Xs[dim], S[nF], faceIndexReverse[nF]
void or_geometry(void* hp, double* area, double* elemSize, double* Xs, int* ok) {
    auto& el = ((Handle*)hp)->mesh.elems;
    int dim = el[0].dim;
    for (size_t i = 0; i < el.size(); i++) {
        area[i] = el[i].area;
        elemSize[i] = el[i].elemSize;
        for (int d = 0; d < dim; d++) Xs[i * dim + d] = el[i].Xs[d];
        ok[i] = el[i].geometryCheck() ? 1 : 0;
    }
}

void or_mass_matrices(void* hp, double* M) {
    auto& el = ((Handle*)hp)->mesh.elems;
    size_t s = 0;
    for (auto& e : el)
        for (auto& r : e.M)
            for (double v : r) M[s++] = v;
}

void or_basis_weights(void* hp, double* Is) {
    auto& el = ((Handle*)hp)->mesh.elems;
    size_t s = 0;
    for (auto& e : el)
        for (double v : e.Is) Is[s++] = v;
}

// Implicit: assemble RHS and FD element Jacobians for (dt, dto)
void or_assemble(void* hp, double dt, double dto) { ((Handle*)hp)->solver->assemble(dt, dto); }
void or_assemble_residuum(void* hp, double dt, double dto) { ((Handle*)hp)->solver->assembleResiduum(dt, dto); }

// blocks in the reference's transposed storage: diag[e][i][j] = ADiag[i][j],
// neigh[e][k][i][j] = ANeighs[k].A[i][j] (zero for boundary faces); rhs[e][i]
void or_get_blocks(void* hp, double* diag, double* neigh, double* rhs) {
    auto& el = ((Handle*)hp)->mesh.elems;
    size_t sd = 0, sn = 0, sr = 0;
    for (auto& e : el) {
        int nb = e.nEqs * e.nBasis;
        if (diag)
            for (int i = 0; i < nb; i++)
                for (int j = 0; j < nb; j++) diag[sd++] = e.ADiag[i][j];
        if (neigh)
            for (int k = 0; k < e.nFaces; k++)
                for (int i = 0; i < nb; i++)
                    for (int j = 0; j < nb; j++) neigh[sn++] = e.TT[k] > -1 ? e.ANeighs[k][i][j] : 0.0;
        if (rhs)
            for (int i = 0; i < nb; i++) rhs[sr++] = e.RHS_loc[i];
    }
}

// LinearSolver.solve with the current blocks; x in global (gIndex) numbering
int or_linear_solve(void* hp, const char* prec, double tol, double* x, int* iters, double* err) {
    auto* h = (Handle*)hp;
    Vec xv;
    bool ok = h->solver->linearSolve(xv, prec, tol);
    std::copy(xv.begin(), xv.end(), x);
    if (iters) *iters = h->solver->lastIters;
    if (err) *err = h->solver->lastError;
    return ok ? 1 : 0;
}

// CRS matrix of the last linear solve (rows in gIndex numbering)
int or_matrix_nnz(void* hp) { return (int)((Handle*)hp)->solver->H.size(); }
void or_matrix(void* hp, int* I, int* J, double* H, double* b) {
    auto* s = ((Handle*)hp)->solver.get();
    std::copy(s->Icrs.begin(), s->Icrs.end(), I);
    std::copy(s->Jcrs.begin(), s->Jcrs.end(), J);
    std::copy(s->H.begin(), s->H.end(), H);
    Vec bv;
    s->updateB(bv);
    std::copy(bv.begin(), bv.end(), b);
}

// FlowProMain.generateDistanceFunction (FlowPro/src/main/java/flowpro/core/FlowProMain.java:962-1018):
// Bellman-Ford relaxation along element edges from the vertices of the faces with TT == sourceBc.
int or_wall_distance(int dim, int nVert, const double* PXY, int nElem, const int* TP, const int* TT, int sourceBc,
                     double* distance) {
    const int nv = dim + 1, nf = dim + 1;
    static const int F3[4][3] = {{0, 2, 1}, {0, 1, 3}, {1, 2, 3}, {2, 0, 3}};
    std::vector<double> d(nVert, std::numeric_limits<double>::infinity());
    for (int i = 0; i < nElem; i++)
        for (int k = 0; k < nf; k++)
            if (TT[(size_t)i * nf + k] == sourceBc)
                for (int q = 0; q < dim; q++) {
                    int fv = dim == 2 ? (q == 0 ? k : (k + 1) % 3) : F3[k][q];
                    d[TP[(size_t)i * nv + fv]] = 0;
                }
    bool changed = true;
    for (int iter = 0; changed && iter <= nVert; iter++) {
        changed = false;
        for (int i = 0; i < nElem; i++)
            for (int j = 0; j < nv; j++) {
                int pj = TP[(size_t)i * nv + j];
                for (int k = 0; k < nv; k++) {
                    int pk = TP[(size_t)i * nv + k];
                    if (j != k && d[pk] < d[pj]) {
                        double L = 0;
                        for (int c = 0; c < dim; c++)
                            L += (PXY[(size_t)pj * dim + c] - PXY[(size_t)pk * dim + c]) * (PXY[(size_t)pj * dim + c] - PXY[(size_t)pk * dim + c]);
                        double y = d[pk] + std::sqrt(L);
                        if (y < d[pj]) {
                            d[pj] = y;
                            changed = true;
                        }
                    }
                }
            }
    }
    bool inf = false;
    for (double v : d) inf = inf || std::isinf(v);
    for (int i = 0; i < nVert; i++) distance[i] = inf ? 1e30 : d[i];
    return 0;
}

// Force on the faces of boundary type bc: Deformation2DRigid.calculateForces
// (FlowPro/src/main/java/flowpro/core/meshDeformation/Deformation2DRigid.java:81-105) with the
// faces selected by TT == bc, i.e. F = -sum over faces of Integration.Face.integrateLeft
// (Integration.java:199-211) of Equation.stressVector (NavierStokes.java:39-83).
void or_forces(void* hp, int bc, double* F) {
    auto* h = (Handle*)hp;
    int dim = h->mesh.eqn->dim();
    Vec force(dim, 0.0);
    for (auto& e : h->mesh.elems)
        for (int k = 0; k < e.nFaces; k++) {
            if (e.TT[k] != bc) continue;
            Face& f = e.Int.faces[k];
            Vec r(dim, 0.0);
            for (int p = 0; p < f.nIntEdge; p++) {
                Vec w(e.nEqs, 0.0), dw(e.nEqs * dim, 0.0);
                for (int m = 0; m < e.nEqs; m++)
                    for (int i = 0; i < e.nBasis; i++) {
                        w[m] += e.W[m * e.nBasis + i] * f.basisFaceLeft[p][i];
                        for (int d = 0; d < dim; d++) dw[e.nEqs * d + m] += e.W[m * e.nBasis + i] * f.dXbasisFaceLeft[p][i][d];
                    }
                Vec val = e.eqn->stressVector(w, dw, e.n[k][p]);
                for (int d = 0; d < dim; d++) r[d] += f.JacobianFace[p] * f.weightsFace[p] * val[d];
            }
            for (int d = 0; d < dim; d++) force[d] -= r[d];
        }
    for (int d = 0; d < dim; d++) F[d] = force[d];
}

// Lift (kind 0) / drag (kind 1) coefficient functionals of the FunctionalsOfInterest module
// (LiftCoefficient.java:31-49, DragCoefficient.java:30-48): boundaryValue = p n[1] (lift) or
// p n[0] (drag) on faces with TT == -1, p = (kappa - 1)(W[3] - |m|^2 / (2 W[0])) with dim = 2,
// insideValue = 0; summed over elements as Element.computeFunctional (Element.java:789-862).
// dIdW (optional, element-major) is the reference's finite-difference derivative
// Element.exportLocalFunctionalDerivative (Element.java:723-734) with step par.h.
static double functional_element(const Element& e, const Vec& Wc, int kind, double kapa) {
    double I = 0;
    for (int k = 0; k < e.nFaces; k++) {
        if (e.TT[k] != -1) continue;
        const Face& f = e.Int.faces[k];
        for (int p = 0; p < f.nIntEdge; p++) {
            Vec w(e.nEqs, 0.0);
            for (int m = 0; m < e.nEqs; m++)
                for (int j = 0; j < e.nBasis; j++) w[m] += Wc[m * e.nBasis + j] * f.basisFaceLeft[p][j];
            double momentum2 = 0;
            for (int d = 0; d < 2; ++d) momentum2 += w[d + 1] * w[d + 1];
            double pr = (kapa - 1) * (w[2 + 1] - momentum2 / (2 * w[0]));
            I += f.JacobianFace[p] * f.weightsFace[p] * pr * e.n[k][p][kind == 0 ? 1 : 0];
        }
    }
    return I;
}

int or_functional(void* hp, int kind, double* I, double* dIdW) {
    auto* h = (Handle*)hp;
    if (h->mesh.eqn->dim() != 2) {
        g_err = "the lift / drag functionals are two-dimensional";
        return -1;
    }
    double kapa = 1.4;
    if (auto* a = dynamic_cast<Aerodynamics*>(h->mesh.eqn.get())) kapa = a->kapa;
    double total = 0;
    size_t off = 0;
    for (auto& e : h->mesh.elems) {
        double Ie = functional_element(e, e.W, kind, kapa);
        total += Ie;
        int nb = e.nEqs * e.nBasis;
        if (dIdW) {
            Vec Wh = e.W;
            for (int i = 0; i < nb; i++) {
                Wh[i] = e.W[i] + e.par->h;
                dIdW[off + i] = (functional_element(e, Wh, kind, kapa) - Ie) / e.par->h;
                Wh[i] = e.W[i];
            }
        }
        off += nb;
    }
    *I = total;
    return 0;
}

void or_rk3_stage(void* hp, int step, double dt) {
    auto* h = (Handle*)hp;
    if (step == 1 && h->mesh.elems[0].iM.empty()) h->solver->computeInvertMassMatrices();
    h->solver->rk3Stage(step, dt);
}

double or_time_step(void* hp) { return ((Handle*)hp)->solver->getTimeStep(); }

void or_update_cfl(void* hp) { ((Handle*)hp)->solver->state.updateCFL(); }

// norms of the spatial residuum stored in the elements (MasterSolver.residuumNorms)
void or_residuum_norms(void* hp, double* norms) {
    Vec n = ((Handle*)hp)->solver->residuumNorms();
    std::copy(n.begin(), n.end(), norms);
}

void or_run_explicit(void* hp, int steps, double* stateOut) {
    auto* h = (Handle*)hp;
    h->solver->runExplicit(steps);
    if (stateOut) {
        stateOut[0] = h->solver->state.t;
        stateOut[1] = h->solver->state.residuum;
        stateOut[2] = h->solver->state.currentCFL;
        stateOut[3] = h->solver->state.dt;
    }
}

int or_run_implicit(void* hp, int steps, double targetResiduum, double* stateOut) {
    auto* h = (Handle*)hp;
    try {
        h->solver->runImplicit(steps, targetResiduum);
    } catch (std::exception& e) {
        g_err = e.what();
        return -1;
    }
    if (stateOut) {
        stateOut[0] = h->solver->state.t;
        stateOut[1] = h->solver->state.residuum;
        stateOut[2] = h->solver->state.currentCFL;
        stateOut[3] = h->solver->state.dt;
        stateOut[4] = h->solver->state.steps;
        stateOut[5] = h->solver->newtonIterationsTotal;
    }
    return 0;
}

int or_positivity(void* hp) { return ((Handle*)hp)->solver->positivityAll(); }

// L2 error against TestScalarEquation.exact (TestSimulation.l2Error, TestSimulation.java:134-150)
double or_l2_error_scalar(void* hp) {
    auto& el = ((Handle*)hp)->mesh.elems;
    double error = 0;
    for (auto& e : el) {
        Mat2 x = e.transform->getX(e.Int.quadVolume.coords);
        for (int p = 0; p < e.Int.nIntVolume; p++) {
            double u = 0;
            for (int j = 0; j < e.nBasis; j++) u += e.W[j] * e.Int.basisVolume[p][j];
            double diff = u - TestScalarEquation::exact(x[p]);
            error += e.Int.JacobianVolume[p] * e.Int.weightsVolume[p] * diff * diff;
        }
    }
    return std::sqrt(error);
}

// java.util.Random(seed).nextDouble() sequence
void or_java_random(long long seed, int n, double* out) {
    JavaRandom r(seed);
    for (int i = 0; i < n; i++) out[i] = r.nextDouble();
}

}  // extern "C"
