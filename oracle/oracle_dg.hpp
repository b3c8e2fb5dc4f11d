// CPU ORACLE (test infrastructure) — DG elements, mesh set-up, element ordering.
// Restates flowpro/core/{Integration,Mesh,ElementOrdering}.java and
// flowpro/core/element/{Element,DGpure}.java of FlowPro_v2.
#pragma once
#include "oracle_core.hpp"

#ifndef ORC_FACE_PHASE
#define ORC_FACE_PHASE(interior) ((void)0)
#define ORC_VOLUME_PHASE() ((void)0)
#endif

namespace orc {

// Numerical parameters used on the hot path (flowpro/core/Parameters.java)
struct Params {
    int order = 2;  // p + 1
    double penalty = 0, beta0 = 2, dampTol = 0, dampConst = 0, dampInnerTol = 0;
    bool positivityLimiter = true;
    double h = 1e-8;  // Parameters.java:22
    bool implicitTime = true;
    int timeOrder = 1;
    std::string elementOrdering = "rcm";
    std::string preconditioner = "blockjacobi";
    double iterativeSolverTol = 1e-2;
    int newtonIters = 1;
    double newtonIterTol = 1e-4;
    double cfl = 1, maxCFL = 1;
    bool varyCFL = false;
    bool isTimeStepFixed = false;
    double dt = 0;
    int gmresRestart = 30, gmresRestarts = 5;
    bool blockJacobiQuirk = false;  // reproduce Mat.lsolveT's in-place elimination
    // moving mesh (Parameters.movingMesh / meshDeformationType / gcl)
    bool movingMesh = false, gcl = false;
    std::string meshDeformationType;
};

struct Element;

// Integration.java:16-217
struct Face {
    Quadrature quadFace;
    int nIntEdge = 0, TT = -1, nVerticesEdge = 0;
    IVec faceIndexes;
    Vec JacobianFace, weightsFace;
    Mat2 coordinatesFace, coordinatesFaceXiRef, coordinatesFaceXiRight;
    Mat2 basisFaceLeft, basisFaceRight;
    std::vector<Mat2> dXibasisFaceLeft, dXibasisFaceRight, dXbasisFaceLeft, dXbasisFaceRight;
    Mat2 interpolantFace;
    std::unique_ptr<FaceTransformation> faceTransform;
};

struct Integration {
    Quadrature quadVolume;
    int nIntVolume = 0;
    Vec JacobianVolume, weightsVolume;
    Mat2 basisVolume, interpolantVolume;
    std::vector<Mat2> dXibasisVolume, dXbasisVolume;
    std::vector<Face> faces;
};

struct Element {
    // mesh
    int index = 0, type = 3, dim = 2, nEqs = 4, nFaces = 3, nVertices = 3, nBasis = 1, order = 1;
    Equation* eqn = nullptr;
    const Params* par = nullptr;
    std::vector<Element>* elems = nullptr;
    const QuadratureCentral* qRules = nullptr;
    double c_IP = 0, eps = 0;
    IVec TT;
    Mat2 vertices, U;
    Mat2 vertices0, verticesOld, verticesOld2, Uinit;  // moving mesh (Element.java:71-78)
    Vec wallDistance;
    std::vector<Mat2> n;
    Vec S;
    double area = 0;
    Vec Xs;
    Mat2 Xes;
    double elemSize = 0;
    bool insideComputeDomain = true;
    IVec faceIndexReverse;
    std::unique_ptr<Transformation> transform;
    std::unique_ptr<Basis> basis;
    Integration Int;
    Vec Is;
    Mat2 M, Mo, Mo2, iM, TrunOrd;
    Vec dampInner, innerIndicatorOld;
    ElementData elemData;
    Vec centreVolumeInterpolant;
    IVec gIndex;
    Vec W, Wo, Wo2;
    // time integration element state (Implicit / RK3)
    Mat2 ADiag;
    std::vector<Mat2> ANeighs;  // per face, [neighbour dof][own dof]
    Vec RHS_loc, spatialResiduum;
    Vec W1, W2, Wn;

    // Element.set, Element.java:133-184
    void set(int idx, const Mat2& verts, const Mat2& Uv, const Vec& wd, const IVec& tt, int typ, int ord, Equation* e,
             const Params* p, std::vector<Element>* all, const QuadratureCentral* q) {
        eqn = e;
        dim = e->dim();
        nEqs = e->nEqs();
        par = p;
        qRules = q;
        elems = all;
        index = idx;
        TT = tt;
        vertices = verts;
        wallDistance = wd;
        type = typ;
        order = ord;
        nFaces = numberOfFaces(typ);
        nVertices = (int)verts.size();
        U = Uv;
        vertices0 = verticesOld = verticesOld2 = verts;
        Uinit = Uv;
        elemData.currentX.assign(dim, 0.0);
        elemData.meshVelocity.assign(dim, 0.0);
        centreVolumeInterpolant.assign(nVertices, 1.0 / nVertices);
        dampInner.assign(nEqs, 0.0);
        innerIndicatorOld.assign(nEqs, 0.0);
    }

    // Element.initBasis, Element.java:227-235
    void initBasis() {
        if (type == 3) {
            transform = std::make_unique<Transformation2DTri>(vertices);
            basis = std::make_unique<Basis2DTri>(order);
        } else {
            transform = std::make_unique<Transformation3DTet>(vertices);
            basis = std::make_unique<Basis3DTet>(order);
        }
        nBasis = basis->nBasis;
        M = zeros(nBasis, nBasis);
        Mo = zeros(nBasis, nBasis);
        Mo2 = zeros(nBasis, nBasis);
        Is.assign(nBasis, 0.0);
    }

    // Transformation.computeTransform on the current vertices (Deformation.recalculateMesh,
    // Deformation.java:44-62); the basis is unchanged
    void recomputeTransform() {
        if (type == 3)
            transform = std::make_unique<Transformation2DTri>(vertices);
        else
            transform = std::make_unique<Transformation3DTet>(vertices);
    }

    // DGpure.recalculateMassMatrix, DGpure.java:575-593
    void recalculateMassMatrix() {
        const Mat2& base = Int.basisVolume;
        for (int i = 0; i < nBasis; i++) {
            for (int j = 0; j < nBasis; j++) {
                M[i][j] = 0;
                for (int p = 0; p < Int.nIntVolume; p++)
                    M[i][j] = M[i][j] + Int.JacobianVolume[p] * Int.weightsVolume[p] * base[p][i] * base[p][j];
            }
            Is[i] = 0;
            for (int p = 0; p < Int.nIntVolume; p++)
                Is[i] = Is[i] + Int.JacobianVolume[p] * Int.weightsVolume[p] * base[p][i] / area;
        }
    }

    // Element.applyGCLMassMatrix, Element.java:568-630: the mass matrix of the time derivative
    // from the discrete geometric conservation law, M = (B - a2 Mo - a3 Mo2) / a1 with
    // B_ij = int_dK (u.n) phi_i phi_j ds - int_K u . grad(phi_i phi_j) dx
    void applyGCLMassMatrix(double a1, double a2, double a3) {
        Mat2 B = zeros(nBasis, nBasis);
        for (int k = 0; k < nFaces; k++) {
            Face& face = Int.faces[k];
            const IVec& edgeIndex = face.faceIndexes;
            for (int p = 0; p < face.nIntEdge; p++) {
                const Vec& interpolant = face.interpolantFace[p];
                double un = 0;
                for (int d = 0; d < dim; d++) {
                    double ud = 0;
                    for (int j = 0; j < face.nVerticesEdge; j++) ud += interpolant[j] * U[edgeIndex[j]][d];
                    un += ud * n[k][p][d];
                }
                const Vec& base = face.basisFaceLeft[p];
                double jw = face.JacobianFace[p] * face.weightsFace[p] * un;
                for (int i = 0; i < nBasis; i++)
                    for (int j = 0; j < nBasis; j++) B[i][j] += jw * base[i] * base[j];
            }
        }
        for (int p = 0; p < Int.nIntVolume; p++) {
            const Vec& interpolant = Int.interpolantVolume[p];
            Vec u(dim, 0.0);
            for (int j = 0; j < nVertices; j++)
                for (int d = 0; d < dim; d++) u[d] += interpolant[j] * U[j][d];
            const Vec& base = Int.basisVolume[p];
            const Mat2& dBase = Int.dXbasisVolume[p];
            double jw = Int.JacobianVolume[p] * Int.weightsVolume[p];
            for (int i = 0; i < nBasis; i++) {
                double uGradI = 0;
                for (int d = 0; d < dim; d++) uGradI += u[d] * dBase[i][d];
                for (int j = 0; j < nBasis; j++) {
                    double uGradJ = 0;
                    for (int d = 0; d < dim; d++) uGradJ += u[d] * dBase[j][d];
                    B[i][j] -= jw * (uGradI * base[j] + base[i] * uGradJ);
                }
            }
        }
        for (int i = 0; i < nBasis; i++)
            for (int j = 0; j < nBasis; j++) M[i][j] = (B[i][j] - a2 * Mo[i][j] - a3 * Mo2[i][j]) / a1;
    }

    // Element.nextTimeLevelMassMatrixes, Element.java:632-639
    void nextTimeLevelMassMatrixes() {
        Mo2 = Mo;
        Mo = M;
    }

    // Integration constructor, Integration.java:40-60 (volume quadrature order = element order)
    void initIntegration() {
        Int.quadVolume = type == 3 ? qRules->tri(order) : qRules->tet(order);
        Int.nIntVolume = Int.quadVolume.nPoints;
        Int.weightsVolume = Int.quadVolume.weights;
        Int.JacobianVolume = transform->jacobian(Int.quadVolume);
        Int.interpolantVolume = transform->getInterpolant(Int.quadVolume);
        Int.basisVolume = basis->getBasisXi(Int.quadVolume.coords);
        Int.dXibasisVolume = basis->getDerBasisXi(Int.quadVolume.coords, dim);
        Int.dXbasisVolume = transform->transformBasis(Int.quadVolume.coords, Int.dXibasisVolume);
        Int.faces.clear();
        Int.faces.resize(nFaces);
    }

    // Integration.initNeighbours + Face constructor, Integration.java:77-153
    void initNeighbours() {
        for (int k = 0; k < nFaces; k++) {
            Face& f = Int.faces[k];
            f.TT = TT[k];
            Element* right = TT[k] > -1 ? &(*elems)[TT[k]] : nullptr;
            f.faceIndexes = getFaceIndexes(type, k);
            int faceOrder = order;
            if (right != nullptr) faceOrder = std::max(order, right->order);
            f.nVerticesEdge = (int)f.faceIndexes.size();
            f.quadFace = type == 3 ? qRules->line(faceOrder) : qRules->tri(faceOrder);
            if (type == 3)
                f.faceTransform = std::make_unique<FaceTransformation2DLine>(transform.get(), f.faceIndexes);
            else
                f.faceTransform = std::make_unique<FaceTransformation3DTri>(transform.get(), f.faceIndexes);
            f.coordinatesFace = f.faceTransform->getX(f.quadFace.coords);
            f.nIntEdge = f.quadFace.nPoints;
            f.weightsFace = f.quadFace.weights;
            f.JacobianFace = f.faceTransform->jacobian(f.quadFace);
            f.coordinatesFaceXiRef = f.faceTransform->getXiRef(f.quadFace.coords);
            f.basisFaceLeft = basis->getBasisXi(f.coordinatesFaceXiRef);
            f.interpolantFace = f.faceTransform->getInterpolant(f.quadFace);
            f.dXibasisFaceLeft = basis->getDerBasisXi(f.coordinatesFaceXiRef, dim);
            f.dXbasisFaceLeft = transform->transformBasis(f.coordinatesFaceXiRef, f.dXibasisFaceLeft);
            if (TT[k] > -1) {
                f.coordinatesFaceXiRight = right->transform->getXi(f.coordinatesFace);
                f.basisFaceRight = right->basis->getBasisXi(f.coordinatesFaceXiRight);
                f.dXibasisFaceRight = right->basis->getDerBasisXi(f.coordinatesFaceXiRight, dim);
                f.dXbasisFaceRight = right->transform->transformBasis(f.coordinatesFaceXiRight, f.dXibasisFaceRight);
            }
        }
    }

    // Element.computeGeometry, Element.java:516-567
    void computeGeometry() {
        Xes.assign(nFaces, Vec());
        for (int k = 0; k < nFaces; k++) Xes[k] = Int.faces[k].faceTransform->getXs();
        S.assign(nFaces, 0.0);
        for (int k = 0; k < nFaces; k++)
            for (int i = 0; i < Int.faces[k].nIntEdge; i++)
                S[k] = S[k] + Int.faces[k].JacobianFace[i] * Int.faces[k].weightsFace[i];
        n.assign(nFaces, Mat2());
        for (int k = 0; k < nFaces; k++) {
            n[k].assign(Int.faces[k].nIntEdge, Vec());
            for (int p = 0; p < Int.faces[k].nIntEdge; p++)
                n[k][p] = Int.faces[k].faceTransform->getNormal(Int.faces[k].quadFace.coords[p]);
        }
        Xs = transform->getXs();
        area = 0;
        for (int i = 0; i < Int.nIntVolume; i++) area = area + Int.JacobianVolume[i] * Int.weightsVolume[i];
        elemSize = 0;
        for (int k = 0; k < nFaces; k++) elemSize += S[k];
        elemSize = nFaces * area / elemSize;
        faceIndexReverse.assign(nFaces, 0);
        for (int k = 0; k < nFaces; k++)
            if (TT[k] > -1) {
                Element& nb = (*elems)[TT[k]];
                for (int s = 0; s < nb.nFaces; s++)
                    if (nb.TT[s] == index) {
                        faceIndexReverse[k] = s;
                        break;
                    }
            }
    }

    // DGpure.computeMassMatrixAndBasisWeights, DGpure.java:546-573
    void computeMassMatrixAndBasisWeights() {
        const Mat2& base = Int.basisVolume;
        for (int i = 0; i < nBasis; i++) {
            for (int j = 0; j < nBasis; j++)
                for (int p = 0; p < Int.nIntVolume; p++)
                    M[i][j] = M[i][j] + Int.JacobianVolume[p] * Int.weightsVolume[p] * base[p][i] * base[p][j];
            for (int p = 0; p < Int.nIntVolume; p++)
                Is[i] = Is[i] + Int.JacobianVolume[p] * Int.weightsVolume[p] * base[p][i] / area;
        }
        Mo = M;
        Mo2 = M;
    }

    double taylorBase(int i, const Vec& X) const { return i > 0 ? (X[i - 1] - Xs[i - 1]) : 1; }

    // DGpure.computeOrderTruncationMatrix, DGpure.java:595-627
    void computeOrderTruncationMatrix() {
        if (order > 2) {
            Mat2 Xcoord = transform->getX(Int.quadVolume.coords);
            int nL = 1 + dim;
            Mat2 Mhat = zeros(nL, nL), T = zeros(nL, nBasis);
            for (int i = 0; i < nL; i++) {
                for (int j = 0; j < nL; j++)
                    for (int p = 0; p < Int.nIntVolume; p++)
                        Mhat[i][j] += Int.JacobianVolume[p] * Int.weightsVolume[p] * taylorBase(i, Xcoord[p]) * taylorBase(j, Xcoord[p]);
                for (int j = 0; j < nBasis; j++)
                    for (int p = 0; p < Int.nIntVolume; p++)
                        T[i][j] += Int.JacobianVolume[p] * Int.weightsVolume[p] * taylorBase(i, Xcoord[p]) * Int.basisVolume[p][j];
            }
            TrunOrd = times(invert(Mhat), T);
            TrunOrd = times(transpose(T), TrunOrd);
            TrunOrd = times(invert(M), TrunOrd);
        }
    }

    // Element.computeInvertMassMatrix, Element.java:250-261
    void computeInvertMassMatrix() {
        Mat2 invM = invert(M);
        iM = zeros(nEqs * nBasis, nEqs * nBasis);
        for (int m = 0; m < nEqs; m++)
            for (int i = 0; i < nBasis; i++)
                for (int j = 0; j < nBasis; j++) iM[m * nBasis + i][m * nBasis + j] = invM[i][j];
    }

    void initTimeIntegration() {
        int nb = nEqs * nBasis;
        ADiag = zeros(nb, nb);
        RHS_loc.assign(nb, 0.0);
        spatialResiduum.assign(nb, 0.0);
        ANeighs.assign(nFaces, Mat2());
        for (int k = 0; k < nFaces; k++)
            if (TT[k] > -1) ANeighs[k] = zeros((*elems)[TT[k]].nBasis * nEqs, nb);
        W1.assign(nb, 0.0);
        W2.assign(nb, 0.0);
        Wn.assign(nb, 0.0);
    }

    // Element.interpolateVelocityAndFillElementDataObjectOnVolume, Element.java:263-297
    Vec interpolateVolume(const Vec& interp) {
        Vec u(dim, 0.0), cXi(dim, 0.0);
        elemData.currentWallDistance = 0;
        for (int j = 0; j < nVertices; j++) {
            for (int d = 0; d < dim; d++) {
                u[d] += interp[j] * U[j][d];
                cXi[d] += interp[j] * transform->coordsXi[j][d];
            }
            elemData.currentWallDistance += interp[j] * wallDistance[j];
        }
        elemData.currentX = transform->getX(cXi);
        for (int d = 0; d < dim; d++) elemData.meshVelocity[d] = u[d];
        elemData.elemIndex = index;
        return u;
    }

    // Element.interpolateVelocityAndFillElementDataObjectOnFace, Element.java:299-332
    Vec interpolateFace(int k, const Vec& interp, const IVec& edgeIndex) {
        Vec u(dim, 0.0), cXi(dim, 0.0);
        elemData.currentWallDistance = 0;
        for (int j = 0; j < Int.faces[k].nVerticesEdge; j++) {
            for (int d = 0; d < dim; d++) {
                u[d] += interp[j] * U[edgeIndex[j]][d];
                elemData.meshVelocity[d] = u[d];
                cXi[d] += interp[j] * transform->coordsXi[edgeIndex[j]][d];
            }
            elemData.currentWallDistance += interp[j] * wallDistance[edgeIndex[j]];
        }
        elemData.currentX = transform->getX(cXi);
        elemData.elemIndex = index;
        return u;
    }

    // Element.calculateAvgW, Element.java:647-655
    Vec calculateAvgW() const {
        Vec Ws(nEqs, 0.0);
        for (int j = 0; j < nEqs; j++)
            for (int m = 0; m < nBasis; m++) Ws[j] = Ws[j] + W[j * nBasis + m] * Is[m];
        return Ws;
    }

    // DGpure.residuum, DGpure.java:108-192 (the phase hooks only tag the operation counters of the
    // counting build, oracle_flops.cpp; they are empty otherwise)
    void residuum(const Vec& V, Vec& K, std::vector<Vec*>& KR) {
        for (int k = 0; k < nFaces; k++) {
            ORC_FACE_PHASE(TT[k] > -1);
            residuumWall(k, V, K, KR[k]);
        }
        ORC_VOLUME_PHASE();
        bool volumeFluxes = order > 1;
        if (volumeFluxes || eqn->isSourcePresent()) {
            Vec nor(dim, 0.0);
            std::vector<Vec> f, fv;
            Vec product;
            for (int p = 0; p < Int.nIntVolume; p++) {
                const Vec& base = Int.basisVolume[p];
                const Mat2& dBase = Int.dXbasisVolume[p];
                double Jac = Int.JacobianVolume[p];
                double weight = Int.weightsVolume[p];
                Vec u = interpolateVolume(Int.interpolantVolume[p]);
                Vec WInt(nEqs, 0.0), dWInt(dim * nEqs, 0.0);
                for (int m = 0; m < nEqs; m++)
                    for (int j = 0; j < nBasis; j++) {
                        WInt[m] += (W[m * nBasis + j] + V[m * nBasis + j]) * base[j];
                        for (int d = 0; d < dim; d++)
                            dWInt[nEqs * d + m] += (W[m * nBasis + j] + V[m * nBasis + j]) * dBase[j][d];
                    }
                if (volumeFluxes && eqn->isConvective()) {
                    f.assign(dim, Vec());
                    for (int d = 0; d < dim; d++) {
                        nor[d] = 1;
                        f[d] = eqn->convectiveFlux(WInt, nor, elemData);
                        nor[d] = 0;
                    }
                }
                if (volumeFluxes && eqn->isDiffusive()) {
                    fv.assign(dim, Vec());
                    for (int d = 0; d < dim; d++) {
                        nor[d] = 1;
                        fv[d] = eqn->diffusiveFlux(WInt, dWInt, nor, elemData);
                        nor[d] = 0;
                    }
                }
                if (eqn->isSourcePresent()) product = eqn->sourceTerm(WInt, dWInt, elemData);
                for (int m = 0; m < nEqs; m++)
                    for (int j = 0; j < nBasis; j++) {
                        if (volumeFluxes && eqn->isConvective()) {
                            double fsum = 0, dWsum = 0;
                            for (int d = 0; d < dim; d++) {
                                fsum += (f[d][m] - u[d] * WInt[m]) * dBase[j][d];
                                dWsum += dWInt[nEqs * d + m] * dBase[j][d];
                            }
                            K[nBasis * m + j] += Jac * weight * fsum - (eps + par->dampConst + dampInner[m]) * Jac * weight * dWsum;
                        }
                        if (volumeFluxes && eqn->isDiffusive()) {
                            double fvsum = 0;
                            for (int d = 0; d < dim; d++) fvsum += fv[d][m] * dBase[j][d];
                            K[nBasis * m + j] -= Jac * weight * fvsum;
                        }
                        if (eqn->isSourcePresent()) K[nBasis * m + j] += Jac * weight * product[m] * base[j];
                    }
            }
        }
    }

    // DGpure.residuumWall, DGpure.java:195-355
    void residuumWall(int k, const Vec& V, Vec& K, Vec* KR) {
        if (KR != nullptr) std::fill(KR->begin(), KR->end(), 0.0);
        Vec fn, fvn;
        Face& F = Int.faces[k];
        const IVec& edgeIndex = F.faceIndexes;
        double beta0 = beta0Current();
        for (int p = 0; p < F.nIntEdge; p++) {
            const Vec& innerInterpolant = F.interpolantFace[p];
            const Vec& baseLeft = F.basisFaceLeft[p];
            const Mat2& dBaseLeft = F.dXbasisFaceLeft[p];
            double Jac = F.JacobianFace[p];
            double weight = F.weightsFace[p];
            const Vec* baseRight = nullptr;
            const Mat2* dBaseRight = nullptr;
            if (TT[k] > -1) {
                baseRight = &F.basisFaceRight[p];
                dBaseRight = &F.dXbasisFaceRight[p];
            }
            double dL = 0;
            for (int d = 0; d < dim; d++) {
                if (TT[k] > -1) {
                    if ((*elems)[TT[k]].insideComputeDomain)
                        dL += (Xs[d] - (*elems)[TT[k]].Xs[d]) * n[k][p][d];
                    else
                        dL += 2 * (Xs[d] - Xes[k][d]) * n[k][p][d];
                } else {
                    dL += (Xs[d] - Xes[k][d]) * n[k][p][d];
                }
            }
            dL = std::fabs(dL);
            Vec u = interpolateFace(k, innerInterpolant, edgeIndex);
            Vec WL(nEqs, 0.0), WR(nEqs, 0.0), dWL(dim * nEqs, 0.0), dWR(dim * nEqs, 0.0);
            for (int m = 0; m < nEqs; m++)
                for (int j = 0; j < nBasis; j++) {
                    WL[m] += (W[m * nBasis + j] + V[m * nBasis + j]) * baseLeft[j];
                    for (int d = 0; d < dim; d++) dWL[nEqs * d + m] += (W[m * nBasis + j] + V[m * nBasis + j]) * dBaseLeft[j][d];
                }
            if (TT[k] > -1) {
                const Element& R = (*elems)[TT[k]];
                const Vec& WRp = R.W;
                for (int m = 0; m < nEqs; m++) {
                    int nRB = R.nBasis;
                    for (int j = 0; j < nRB; j++) {
                        WR[m] += WRp[m * nRB + j] * (*baseRight)[j];
                        for (int d = 0; d < dim; d++) dWR[nEqs * d + m] += WRp[m * nRB + j] * (*dBaseRight)[j][d];
                    }
                }
            } else {
                WR = eqn->boundaryValue(WL, n[k][p], TT[k], elemData);
                dWR = dWL;
            }
            double vn = 0;
            Vec Wale(nEqs, 0.0);
            if (eqn->isConvective()) {
                for (int d = 0; d < dim; d++) vn = vn + u[d] * n[k][p][d];
                if (TT[k] > -1)
                    for (int j = 0; j < nEqs; j++) Wale[j] = (WL[j] + WR[j]) / 2;
                else
                    Wale = WR;
                fn = eqn->numericalConvectiveFlux(WL, WR, n[k][p], TT[k], elemData);
            }
            if (eqn->isDiffusive()) {
                Vec Wc(nEqs, 0.0), dWc(nEqs * dim, 0.0);
                for (int m = 0; m < nEqs; m++) {
                    if (TT[k] > -1)
                        Wc[m] = (WL[m] + WR[m]) / 2;
                    else
                        Wc[m] = WR[m];
                    for (int d = 0; d < dim; d++)
                        dWc[nEqs * d + m] = (dWL[nEqs * d + m] + dWR[nEqs * d + m]) / 2 + beta0 * (WR[m] - WL[m]) / dL * n[k][p][d];
                }
                fvn = eqn->numericalDiffusiveFlux(Wc, dWc, n[k][p], TT[k], elemData);
            }
            for (int m = 0; m < nEqs; m++) {
                double dWsum = 0;
                if (TT[k] > -1)
                    for (int d = 0; d < dim; d++) dWsum += (dWL[nEqs * d + m] + dWR[nEqs * d + m]) / 2 * n[k][p][d];
                double avFlux = 0;
                if (TT[k] > -1) {
                    const Element& R = (*elems)[TT[k]];
                    double epsFace = 0.5 * (eps + R.eps) + par->dampConst + 0.5 * (dampInner[m] + R.dampInner[m]);
                    avFlux = epsFace * (dWsum + beta0 * (WR[m] - WL[m]) / dL);
                }
                for (int j = 0; j < nBasis; j++) {
                    double jwb = Jac * weight * baseLeft[j];
                    if (eqn->isConvective()) {
                        K[nBasis * m + j] -= jwb * (fn[m] - vn * Wale[m]);
                        if (TT[k] > -1) K[nBasis * m + j] += avFlux * jwb;
                    }
                    if (eqn->isDiffusive()) {
                        K[nBasis * m + j] += jwb * fvn[m];
                        if (TT[k] > -1)
                            K[nBasis * m + j] -= c_IP * jwb * (WL[m] - WR[m]);
                        else if (eqn->isIPFace(TT[k]))
                            K[nBasis * m + j] -= c_IP * jwb * (WL[m] - WR[m]);
                    }
                }
                if (KR != nullptr) {
                    int nRB = (*elems)[TT[k]].nBasis;
                    for (int j = 0; j < nRB; j++) {
                        double jwb = Jac * weight * (*baseRight)[j];
                        if (eqn->isConvective()) {
                            (*KR)[nRB * m + j] -= jwb * (fn[m] - vn * Wale[m]);
                            (*KR)[nRB * m + j] += avFlux * jwb;
                        }
                        if (eqn->isDiffusive()) {
                            (*KR)[nRB * m + j] += jwb * fvn[m];
                            (*KR)[nRB * m + j] -= c_IP * jwb * (WL[m] - WR[m]);
                        }
                    }
                }
            }
        }
    }

    // DGpure.residuumWall sets the field beta0 = 0 when the global order is 1
    // (DGpure.java:287-289); the value is then kept, so it is resolved once here.
    double beta0Current() const { return (eqn->isDiffusive() && par->order == 1) ? 0.0 : par->beta0; }

    // DGpure.limiter, DGpure.java:358-400 (dampInnerTol > 0 branch not used on the hot path)
    void limiter() {
        eps = 0;
        c_IP = 0;
        if (order > 1) {
            Vec avg = calculateAvgW();
            double lam = eqn->maxEigenvalue(avg, &elemData);
            if (par->dampTol > 0) {
                double g = shock_senzor(par->dampTol);
                eps = lam * elemSize / order * g;
            }
            if (eqn->isDiffusive()) c_IP = par->penalty;
        }
    }

    // DGpure.shock_senzor, DGpure.java:402-452
    double shock_senzor(double kap) const {
        double Se = 0, pod = 0;
        Vec rhoTrunCoef(nBasis, 0.0);
        if (order > 2) {
            for (int i = 0; i < nBasis; i++)
                for (int j = 0; j < nBasis; j++) rhoTrunCoef[i] += TrunOrd[i][j] * W[j];
        } else {
            Vec Ws = calculateAvgW();
            std::fill(rhoTrunCoef.begin(), rhoTrunCoef.end(), Ws[0]);
        }
        for (int p = 0; p < Int.nIntVolume; p++) {
            double rhoInt = 0, rhoTrun = 0;
            for (int m = 0; m < nBasis; m++) {
                rhoInt += W[m] * Int.basisVolume[p][m];
                rhoTrun += rhoTrunCoef[m] * Int.basisVolume[p][m];
            }
            Se += Int.JacobianVolume[p] * Int.weightsVolume[p] * (rhoInt - rhoTrun) * (rhoInt - rhoTrun);
            pod += Int.JacobianVolume[p] * Int.weightsVolume[p] * rhoInt * rhoInt;
        }
        Se = std::log10(std::fabs(Se / pod));
        double S0 = std::log10(1. / std::pow(order - 1, 4.0));
        double shock = 0.5 * (1 + std::sin(M_PI * (Se - S0) / (2 * kap)));
        if (Se < S0 - kap) shock = 0;
        if (Se > S0 + kap) shock = 1;
        if (std::isnan(shock)) return 0;
        return shock;
    }

    // Element.l2NormsSquared, Element.java:357-373
    Vec l2NormsSquared(const Vec& R) const {
        Mat2 invM = invert(M);
        Vec norms(nEqs, 0.0);
        for (int m = 0; m < nEqs; m++) {
            int s = m * nBasis;
            double sum = 0;
            for (int i = 0; i < nBasis; i++) {
                double r = 0;
                for (int j = 0; j < nBasis; j++) r += invM[i][j] * R[s + j];
                sum += R[s + i] * r;
            }
            norms[m] = sum;
        }
        return norms;
    }

    // Element.positivityLimiter / admissibleTheta, Element.java:385-476
    double admissibleTheta(const Vec& Wavg, const Vec& base) const {
        Vec Wx(nEqs, 0.0);
        for (int m = 0; m < nEqs; m++)
            for (int j = 0; j < nBasis; j++) Wx[m] += W[m * nBasis + j] * base[j];
        if (eqn->isAdmissible(Wx)) return 1;
        double lo = 0, hi = 1;
        Vec Wt(nEqs);
        for (int iter = 0; iter < 30; iter++) {
            double mid = 0.5 * (lo + hi);
            for (int m = 0; m < nEqs; m++) Wt[m] = Wavg[m] + mid * (Wx[m] - Wavg[m]);
            if (eqn->isAdmissible(Wt))
                lo = mid;
            else
                hi = mid;
        }
        return lo;
    }
    bool positivityLimiter() {
        if (nBasis == 1) return false;
        Vec Wavg = calculateAvgW();
        if (!eqn->isAdmissible(Wavg)) return false;
        double theta = 1;
        for (int p = 0; p < Int.nIntVolume; p++) theta = std::min(theta, admissibleTheta(Wavg, Int.basisVolume[p]));
        for (int k = 0; k < nFaces; k++)
            for (int p = 0; p < Int.faces[k].nIntEdge; p++)
                theta = std::min(theta, admissibleTheta(Wavg, Int.faces[k].basisFaceLeft[p]));
        if (theta >= 1) return false;
        Mat2 Mgeom = zeros(nBasis, nBasis);
        Vec integrals(nBasis, 0.0);
        for (int p = 0; p < Int.nIntVolume; p++) {
            double jw = Int.JacobianVolume[p] * Int.weightsVolume[p];
            const Vec& base = Int.basisVolume[p];
            for (int i = 0; i < nBasis; i++) {
                integrals[i] += jw * base[i];
                for (int j = 0; j < nBasis; j++) Mgeom[i][j] += jw * base[i] * base[j];
            }
        }
        Vec one = times(invert(Mgeom), integrals);
        for (int m = 0; m < nEqs; m++)
            for (int i = 0; i < nBasis; i++) {
                double mean = one[i] * Wavg[m];
                W[m * nBasis + i] = mean + theta * (W[m * nBasis + i] - mean);
            }
        return true;
    }

    // Element.delta_t helpers, Element.java:490-513
    double timeStepOrderFactor() const { return par->implicitTime ? 1 : 2 * (order - 1) + 1; }
    double calculateMaxEigenvalue() {
        interpolateVolume(centreVolumeInterpolant);
        Vec avg = calculateAvgW();
        return eqn->maxEigenvalue(avg, &elemData);
    }

    // Element.geometryCheck, Element.java:665-720
    bool geometryCheck() const {
        bool ok = true;
        Vec t1(dim, 0.0), t2(dim, 0.0);
        double s1 = 0, s2 = 0;
        for (int k = 0; k < nFaces; k++) {
            const Face& f = Int.faces[k];
            for (int p = 0; p < f.nIntEdge; p++) {
                Vec X = f.faceTransform->getX(f.quadFace.coords[p]);
                for (int d = 0; d < dim; d++) {
                    t1[d] += f.weightsFace[p] * f.JacobianFace[p] * n[k][p][d];
                    t2[d] += X[d] * f.weightsFace[p] * f.JacobianFace[p] * n[k][p][d];
                }
            }
        }
        for (int d = 0; d < dim; d++) {
            s1 += t1[d];
            s2 += t2[d] / dim;
            if (t2[d] < 0) ok = false;
        }
        double tol2 = order == 1 ? 1e-4 : 1e-11;
        if (std::fabs(s1) > 1e-11 || std::fabs(s2 - area) > tol2 || s2 < 0) ok = false;
        return ok;
    }
};

// ElementOrdering.reverseCuthillMcKee, ElementOrdering.java:52-142
static int pseudoPeripheral(const std::vector<IVec>& adj, const std::vector<char>& excluded, int start) {
    int node = start, ecc = -1;
    for (int iter = 0; iter < 10; iter++) {
        IVec level(adj.size(), -1);
        std::deque<int> q;
        q.push_back(node);
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
}

static IVec reverseCuthillMcKee(const std::vector<IVec>& TT) {
    int n = (int)TT.size();
    std::vector<IVec> adj(n);
    IVec degree(n);
    for (int i = 0; i < n; i++) {
        for (int t : TT[i])
            if (t > -1 && t != i && std::find(adj[i].begin(), adj[i].end(), t) == adj[i].end()) adj[i].push_back(t);
        degree[i] = (int)adj[i].size();
    }
    for (int i = 0; i < n; i++)
        std::stable_sort(adj[i].begin(), adj[i].end(), [&](int a, int b) { return degree[a] < degree[b]; });
    IVec order(n);
    std::vector<char> visited(n, 0);
    int count = 0;
    while (count < n) {
        int start = -1;
        for (int i = 0; i < n; i++)
            if (!visited[i] && (start == -1 || degree[i] < degree[start])) start = i;
        start = pseudoPeripheral(adj, visited, start);
        std::deque<int> q;
        q.push_back(start);
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
    for (int i = 0; i < n / 2; i++) std::swap(order[i], order[n - 1 - i]);
    return order;
}

// Mesh constructor + Mesh.init, Mesh.java:69-224 (single domain, all elements inside)
struct Mesh {
    std::unique_ptr<Equation> eqn;
    Params par;
    QuadratureCentral qRules;
    std::vector<Element> elems;
    int dofs = 0;
    int dim = 2, type = 3;

    void build(const Props& props, const Params& p, const Mat2& PXY, const std::vector<IVec>& TP, const std::vector<IVec>& TT,
               const Vec& wallDistance, const Mat2* UXY) {
        eqn = makeEquation(props);
        par = p;
        dim = eqn->dim();
        type = dim == 2 ? 3 : 5;
        int nE = (int)TP.size();
        elems.clear();
        elems.resize(nE);
        for (int i = 0; i < nE; i++) {
            int nV = (int)TP[i].size();
            Mat2 verts(nV, Vec(dim)), mv(nV, Vec(dim, 0.0));
            Vec wd(nV);
            for (int j = 0; j < nV; j++) {
                for (int d = 0; d < dim; d++) verts[j][d] = PXY[TP[i][j]][d];
                wd[j] = wallDistance.empty() ? 0.0 : wallDistance[TP[i][j]];
                if (UXY)
                    for (int d = 0; d < dim; d++) mv[j][d] = (*UXY)[TP[i][j]][d];
            }
            elems[i].set(i, verts, mv, wd, TT[i], type, par.order, eqn.get(), &par, &elems, &qRules);
        }
        for (auto& e : elems) e.initBasis();
        for (auto& e : elems) e.initIntegration();
        IVec ord;
        if (par.elementOrdering == "rcm") {
            std::vector<IVec> tt(nE);
            for (int i = 0; i < nE; i++) tt[i] = elems[i].TT;
            ord = reverseCuthillMcKee(tt);
        } else {
            ord.resize(nE);
            for (int i = 0; i < nE; i++) ord[i] = i;
        }
        int s = 0;
        for (int i : ord) {
            Element& e = elems[i];
            e.gIndex.resize(e.nEqs * e.nBasis);
            for (int k = 0; k < e.nEqs * e.nBasis; k++) e.gIndex[k] = s++;
        }
        for (auto& e : elems) {
            e.initNeighbours();
            e.computeGeometry();
            e.computeMassMatrixAndBasisWeights();
            e.computeOrderTruncationMatrix();
        }
        for (auto& e : elems) e.initTimeIntegration();
        dofs = s;
    }

    // Deformation.recalculateMesh, Deformation.java:44-62: transformations, then volume
    // integrals, then face integrals, geometry and mass matrices on the moved vertices
    void recalculateMesh() {
        for (auto& e : elems) e.recomputeTransform();
        for (auto& e : elems) e.initIntegration();
        for (auto& e : elems) {
            e.initNeighbours();
            e.computeGeometry();
            e.recalculateMassMatrix();
        }
    }
};

}  // namespace orc
