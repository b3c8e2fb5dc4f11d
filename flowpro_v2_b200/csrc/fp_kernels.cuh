// DG element residual on the device (one element per thread, element-major SoA
// layout), restating DGpure.residuum / residuumWall
// (flowpro/core/element/DGpure.java:108-355) for affine simplices.
//
// Layout (all arrays field-major with leading dimension ld >= nElem):
//   state  W[c * ld + e],   c = m * NB + j  (Java: W[m * nBasis + j] of element e)
//   geometry geo[f * ld + e] (GeoLayout), neighbours tt[k * ld + e], face codes fcode[k * ld + e]
// Reference-element tables (basis values/gradients at volume and face quadrature
// points, both face orientations) are read through the read-only cache; their
// accesses are warp-uniform except the neighbour-side face tables.
#pragma once
#include "fp_mesh.h"
#include "fp_physics.cuh"

namespace fp {

// Compile-time offsets of the packed reference tables (same packing as build_ref_tables)
template <int DIM, int ORDER>
struct Tab {
    static constexpr int NB = nbasis_of(DIM, ORDER), NQV = nqv_of(DIM, ORDER), NQF = nqf_of(DIM, ORDER);
    static constexpr int NF = DIM + 1, NV = DIM + 1, NVF = DIM, NP = nperm_of(DIM);
    static constexpr int o_w = 0, o_phi = o_w + NQV, o_dphi = o_phi + NQV * NB, o_interp = o_dphi + NQV * NB * DIM,
                         o_xi = o_interp + NQV * NV;
    static constexpr int o_wf = o_xi + NQV * DIM, o_phiL = o_wf + NQF, o_dphiL = o_phiL + NF * NQF * NB,
                         o_finterp = o_dphiL + NF * NQF * NB * DIM, o_xiL = o_finterp + NQF * NVF;
    static constexpr int o_phiR = o_xiL + NF * NQF * DIM, o_dphiR = o_phiR + NF * NP * NQF * NB;
    static constexpr int o_Is = o_dphiR + NF * NP * NQF * NB * DIM, o_Mref = o_Is + NB, o_MinvRef = o_Mref + NB * NB,
                         o_one = o_MinvRef + NB * NB, o_trun = o_one + NB, total = o_trun + NB * NB;
};

// face vertex indexes (triangleElement.getFaceIndexes / tetrahedralElement.getFaceIndexes)
template <int DIM>
FP_HD int face_vertex(int k, int i) {
    if (DIM == 2) return i == 0 ? k : (k + 1) % 3;
    const int F[4][3] = {{0, 2, 1}, {0, 1, 3}, {1, 2, 3}, {2, 0, 3}};
    return F[k][i];
}

// Face list of the face-based residual: every face once, both sides' contributions
struct DevFaces {
    int nFaces, ldf;
    const int* __restrict__ fl;    // owner element
    const int* __restrict__ fk;    // owner's face index
    const int* __restrict__ fr;    // neighbour element, or the boundary code (< 0)
    const int* __restrict__ fc;    // neighbour's face index * NP + permutation
    const int* __restrict__ qmap;  // [NP][NQF] neighbour-side quadrature index of owner point p
    const int* __restrict__ efc;   // [NF][ld] (face << 1) | side
    double* __restrict__ G;        // [2][NQF][NE][ldf] face contributions jw * g (side 0 owner, 1 neighbour)
};

struct DevMesh {
    int nElem, ld;
    const double* __restrict__ geo;
    const int* __restrict__ tt;
    const int* __restrict__ fcode;
    const double* __restrict__ vwd;
    const double* __restrict__ vu;  // nullptr: static mesh
    const double* __restrict__ tab;
    const double* __restrict__ eps;  // artificial viscosity per element
    const double* __restrict__ cip;  // interior penalty per element
    // moving mesh: element mass matrices of the time levels [3][NB*NB][ld] (level 0 current,
    // 1 previous, 2 the one before; Element.M / Mo / Mo2), nullptr on a static mesh, where
    // every level is jac * Mref
    const double* __restrict__ mass;
    // a batch of independent cases merged into one mesh: case of each element, and per case the
    // BDF coefficients of its current step [3][ncases] and its outlet pressure (nullptr: one case)
    const int* __restrict__ case_of;
    const double* __restrict__ case_a;
    const double* __restrict__ case_pout;
    // [ncases] 0: the matrix-free operator skips the case's faces and elements, leaving its
    // output untouched (nullptr: no case is skipped)
    const int* __restrict__ case_live;
    int ncases;
    double dampConst, beta0;
    fp_model_params P;
    DevFaces F;
};

__device__ __forceinline__ double ldg(const double* p) { return __ldg(p); }

// the BDF coefficients of element e's step: its case's in a batch, else the launch's
__device__ __forceinline__ void case_coefficients(const DevMesh& M, int e, double& a1, double& a2, double& a3) {
    if (!M.case_a) return;
    const int cs = M.case_of[e];
    a1 = ldg(M.case_a + cs);
    a2 = ldg(M.case_a + M.ncases + cs);
    a3 = ldg(M.case_a + 2 * M.ncases + cs);
}
__device__ __forceinline__ void case_coefficients(const DevMesh& M, int e, double& a1) {
    if (M.case_a) a1 = ldg(M.case_a + M.case_of[e]);
}

// entry (i, j) of element e's mass matrix of time level lev
template <int DIM, int ORDER>
__device__ __forceinline__ double mass_entry(const DevMesh& M, int e, int lev, int i, int j, double jac) {
    using TB = Tab<DIM, ORDER>;
    if (M.mass) return ldg(M.mass + ((size_t)(lev * TB::NB + i) * TB::NB + j) * M.ld + e);
    return ldg(M.tab + TB::o_Mref + i * TB::NB + j) * jac;
}

// Loads of neighbour coefficients: plain state, or state + tangent (JVP)
struct NbPlain {
    const double* W;
    int ld;
    __device__ double operator()(int c, int nb) const { return ldg(W + (size_t)c * ld + nb); }
};
template <int N>
struct NbDual {
    const double* W;
    const double* V;  // tangent direction, same layout
    int ld;
    __device__ Dual<N> operator()(int c, int nb) const {
        Dual<N> r(ldg(W + (size_t)c * ld + nb));
        r.d[0] = ldg(V + (size_t)c * ld + nb);
        return r;
    }
};

struct NoKR {
    static constexpr bool enabled = false;
    template <class T>
    __device__ void begin(int) {}
    template <class T>
    __device__ void add(int, int, const T&) {}
    __device__ void end(int, int, int) {}
};

template <class Mdl, int DIM, int ORDER>
struct Element {
    using TB = Tab<DIM, ORDER>;
    using GL = GeoLayout<DIM>;
    static constexpr int NB = TB::NB, NQV = TB::NQV, NQF = TB::NQF, NF = TB::NF, NV = TB::NV, NVF = TB::NVF, NP = TB::NP;
    static constexpr int NE = Mdl::NE, NC = NE * NB;

    // One face quadrature point of DGpure.residuumWall (DGpure.java:204-353) seen from element
    // e (owner side): C = -(fn - vn Wale) + avFlux + fvn and Jmp = WL - WR (after the flux
    // calls have limited the densities in place, as Java's arrays are), so that the element's
    // integrand is C - c_IP Jmp (interior faces and IP walls) and the neighbour's -C + c_IP' Jmp.
    // w: the owner's coefficients, a register array or an accessor reading them from memory
    template <class T, class OwnL, class NbL>
    static __device__ __forceinline__ void face_point(const DevMesh& M, int e, int k, int p, int TT, const double* n,
                                                      double dL, const double* Jinv, const double* JinvR, int kr_face,
                                                      int pm, double eps_e, double eps_nb, const OwnL& w, const NbL& nbl,
                                                      T* C, T* Jmp) {
        const int ld = M.ld;
        const double* geo = M.geo;
        const double* tab = M.tab;
        const fp_model_params& P = M.P;
        const bool interior = TT > -1;
        const double* phiL = tab + TB::o_phiL + (k * NQF + p) * NB;
        const double* dphiL = tab + TB::o_dphiL + (k * NQF + p) * NB * DIM;
        // mesh velocity and position at the face point (Element.java:299-332)
        double u[DIM];
#pragma unroll
        for (int d = 0; d < DIM; d++) u[d] = 0;
        if (M.vu != nullptr) {
#pragma unroll
            for (int i = 0; i < NVF; i++) {
                const double li = ldg(tab + TB::o_finterp + p * NVF + i);
                const int v = face_vertex<DIM>(k, i);
#pragma unroll
                for (int d = 0; d < DIM; d++) u[d] += li * ldg(M.vu + (size_t)(v * DIM + d) * ld + e);
            }
        }
        double X[DIM];
        if (Mdl::NE == 1) {  // only the scalar test equation's boundary values use the position
            const double* xi = tab + TB::o_xiL + (k * NQF + p) * DIM;
#pragma unroll
            for (int i = 0; i < DIM; i++) {
                double s = 0;
#pragma unroll
                for (int j = 0; j < DIM; j++) s += ldg(geo + (size_t)(GL::JM + i * DIM + j) * ld + e) * ldg(xi + j);
                X[i] = s + ldg(geo + (size_t)(GL::X0 + i) * ld + e);
            }
        }
        // traces (DGpure.java:239-264)
        T WL[NE], WR[NE], dWL[DIM * NE], dWR[DIM * NE];
        {
            T g[DIM * NE];
#pragma unroll
            for (int m = 0; m < NE; m++) {
                WL[m] = 0.0;
#pragma unroll
                for (int d = 0; d < DIM; d++) g[d * NE + m] = 0.0;
#pragma unroll
                for (int j = 0; j < NB; j++) {
                    const T& c = w[m * NB + j];
                    WL[m] += c * ldg(phiL + j);
#pragma unroll
                    for (int d = 0; d < DIM; d++) g[d * NE + m] += c * ldg(dphiL + j * DIM + d);
                }
            }
#pragma unroll
            for (int m = 0; m < NE; m++)
#pragma unroll
                for (int d = 0; d < DIM; d++) {
                    T s = 0.0;
#pragma unroll
                    for (int q = 0; q < DIM; q++) s += Jinv[q * DIM + d] * g[q * NE + m];
                    dWL[d * NE + m] = s;
                }
        }
        if (interior) {
            const double* phiR = tab + TB::o_phiR + ((kr_face * NP + pm) * NQF + p) * NB;
            const double* dphiR = tab + TB::o_dphiR + ((kr_face * NP + pm) * NQF + p) * NB * DIM;
            T g[DIM * NE];
#pragma unroll
            for (int m = 0; m < NE; m++) {
                WR[m] = 0.0;
#pragma unroll
                for (int d = 0; d < DIM; d++) g[d * NE + m] = 0.0;
#pragma unroll
                for (int j = 0; j < NB; j++) {
                    const T c = nbl(m * NB + j, TT);
                    WR[m] += c * ldg(phiR + j);
#pragma unroll
                    for (int d = 0; d < DIM; d++) g[d * NE + m] += c * ldg(dphiR + j * DIM + d);
                }
            }
#pragma unroll
            for (int m = 0; m < NE; m++)
#pragma unroll
                for (int d = 0; d < DIM; d++) {
                    T s = 0.0;
#pragma unroll
                    for (int q = 0; q < DIM; q++) s += JinvR[q * DIM + d] * g[q * NE + m];
                    dWR[d * NE + m] = s;
                }
        } else {
            // the outlet pressure of the element's case in a batch of cases, else the model's
            Mdl::boundaryValue(WL, n, TT, u, X, WR, P, M.case_pout ? ldg(M.case_pout + M.case_of[e]) : P.p_out);
#pragma unroll
            for (int i = 0; i < DIM * NE; i++) dWR[i] = dWL[i];
        }
        // inviscid flux (DGpure.java:266-281)
        double vn = 0;
#pragma unroll
        for (int d = 0; d < DIM; d++) vn += u[d] * n[d];
        T Wale[NE], fn[NE];
#pragma unroll
        for (int j = 0; j < NE; j++) Wale[j] = interior ? (WL[j] + WR[j]) / 2.0 : WR[j];
        // interior faces with both densities >= RHO_TOL: the division-light formulation
        bool fast = false;
        if constexpr (Mdl::kFastFace)
            fast = interior && P.numerical_flux != 1 && val(WL[0]) >= RHO_TOL && val(WR[0]) >= RHO_TOL;
        if constexpr (Mdl::kFastFace) {
            if (fast)
                Mdl::laxFriedrichsFast(WL, WR, n, u, fn, P);
            else
                Mdl::numericalConvectiveFlux(WL, WR, n, TT, u, fn, P);
        } else {
            Mdl::numericalConvectiveFlux(WL, WR, n, TT, u, fn, P);
        }
        const double idL = 1.0 / dL;
        // DDG viscous flux (DGpure.java:283-303)
        T fvn[NE];
        if (Mdl::kViscous) {
            T Wc[NE], dWc[NE * DIM];
#pragma unroll
            for (int m = 0; m < NE; m++) {
                Wc[m] = interior ? (WL[m] + WR[m]) / 2.0 : WR[m];
                const T jump = M.beta0 * (WR[m] - WL[m]) * idL;
#pragma unroll
                for (int d = 0; d < DIM; d++) dWc[NE * d + m] = (dWL[NE * d + m] + dWR[NE * d + m]) / 2.0 + jump * n[d];
            }
            if constexpr (Mdl::kFastFace) {
                if (fast)
                    Mdl::diffusiveFluxFast(Wc, dWc, n, fvn, P);
                else
                    Mdl::numericalDiffusiveFlux(Wc, dWc, n, TT, u, fvn, P);
            } else {
                Mdl::numericalDiffusiveFlux(Wc, dWc, n, TT, u, fvn, P);
            }
        }
        // integrand (DGpure.java:305-338)
#pragma unroll
        for (int m = 0; m < NE; m++) {
            T g = -(fn[m] - vn * Wale[m]);
            if (interior) {
                T dWsum = 0.0;
#pragma unroll
                for (int d = 0; d < DIM; d++) dWsum += (dWL[NE * d + m] + dWR[NE * d + m]) / 2.0 * n[d];
                const double epsFace = 0.5 * (eps_e + eps_nb) + M.dampConst;
                g += epsFace * (dWsum + M.beta0 * (WR[m] - WL[m]) * idL);
            }
            if (Mdl::kViscous) g += fvn[m];
            C[m] = g;
            Jmp[m] = WL[m] - WR[m];
        }
    }

    // face geometry of element e, face k
    static __device__ __forceinline__ void face_geo(const DevMesh& M, int e, int k, double* n, double& jac, double& dL) {
#pragma unroll
        for (int d = 0; d < DIM; d++) n[d] = ldg(M.geo + (size_t)(GL::NRM + k * DIM + d) * M.ld + e);
        jac = ldg(M.geo + (size_t)(GL::JF + k) * M.ld + e);
        dL = ldg(M.geo + (size_t)(GL::DL + k) * M.ld + e);
    }

    // DGpure.residuum (faces then volume), element e, own coefficients w (already W + V).
    // nbl(c, nb) returns the coefficients of a neighbour; kr receives the contribution of
    // this element's face integrals to the neighbour's residual (DGpure.residuumWall's KR).
    // w: a register array or an accessor reading the coefficients from memory
    template <class T, class WA, class NbL, class KR>
    static __device__ void residual(const DevMesh& M, int e, const WA& w, const NbL& nbl, T* K, KR& kr) {
        const int ld = M.ld;
        double Jinv[DIM * DIM];
#pragma unroll
        for (int i = 0; i < DIM * DIM; i++) Jinv[i] = ldg(M.geo + (size_t)(GL::JINV + i) * ld + e);
        const double eps_e = ldg(M.eps + e);
        const double cip_e = ldg(M.cip + e);
#pragma unroll
        for (int c = 0; c < NC; c++) K[c] = 0.0;
#pragma unroll 1
        for (int k = 0; k < NF; k++) {
            const int TT = M.tt[(size_t)k * ld + e];
            double n[DIM], Jac, dL;
            face_geo(M, e, k, n, Jac, dL);
            const bool interior = TT > -1;
            int kr_face = 0, pm = 0;
            double JinvR[DIM * DIM];
            double eps_nb = 0;
            if (interior) {
                const int fc = M.fcode[(size_t)k * ld + e];
                kr_face = fc / NP;
                pm = fc - kr_face * NP;
#pragma unroll
                for (int i = 0; i < DIM * DIM; i++) JinvR[i] = ldg(M.geo + (size_t)(GL::JINV + i) * ld + TT);
                eps_nb = ldg(M.eps + TT);
            }
            const bool ip = Mdl::kViscous && (interior || Mdl::isIPFace(TT));
            if (KR::enabled && interior) kr.template begin<T>(k);
#pragma unroll 1
            for (int p = 0; p < NQF; p++) {
                T C[NE], Jm[NE];
                face_point(M, e, k, p, TT, n, dL, Jinv, JinvR, kr_face, pm, eps_e, eps_nb, w, nbl, C, Jm);
                const double jw = Jac * ldg(M.tab + TB::o_wf + p);
                const double* phiL = M.tab + TB::o_phiL + (k * NQF + p) * NB;
#pragma unroll
                for (int m = 0; m < NE; m++) {
                    T g = C[m];
                    if (ip) g -= cip_e * Jm[m];
                    const T gw = jw * g;
#pragma unroll
                    for (int j = 0; j < NB; j++) K[m * NB + j] += gw * ldg(phiL + j);
                    if (KR::enabled && interior) {
                        const double* phiR = M.tab + TB::o_phiR + ((kr_face * NP + pm) * NQF + p) * NB;
#pragma unroll
                        for (int j = 0; j < NB; j++) kr.add(k, m * NB + j, gw * ldg(phiR + j));
                    }
                }
            }
            if (KR::enabled && interior) kr.end(k, TT, kr_face);
        }
        volume(M, e, w, Jinv, eps_e, K);
    }

    // Face-based form: K gathers the face contributions computed once per face (k_face) and
    // adds the volume integral.
    // w: the element's coefficients, a register array or an accessor reading them from memory
    template <class T, class WA>
    static __device__ void residual_from_faces(const DevMesh& M, const DevFaces& F, int e, const WA& w, T* K) {
        const int ld = M.ld;
        double Jinv[DIM * DIM];
#pragma unroll
        for (int i = 0; i < DIM * DIM; i++) Jinv[i] = ldg(M.geo + (size_t)(GL::JINV + i) * ld + e);
        const double eps_e = ldg(M.eps + e);
#pragma unroll
        for (int c = 0; c < NC; c++) K[c] = 0.0;
#pragma unroll 1
        for (int k = 0; k < NF; k++) {
            const int code = F.efc[(size_t)k * ld + e];
            const int f = code >> 1, side = code & 1;
            const double* G = F.G + (size_t)side * NQF * NE * F.ldf + f;
#pragma unroll
            for (int q = 0; q < NQF; q++) {
                const double* phi = M.tab + TB::o_phiL + (k * NQF + q) * NB;
#pragma unroll
                for (int m = 0; m < NE; m++) {
                    const double g = ldg(G + (size_t)(q * NE + m) * F.ldf);
#pragma unroll
                    for (int j = 0; j < NB; j++) K[m * NB + j] += g * ldg(phi + j);
                }
            }
        }
        volume(M, e, w, Jinv, eps_e, K);
    }

    // volume integral of DGpure.residuum (DGpure.java:116-191)
    template <class T, class WA>
    static __device__ __forceinline__ void volume(const DevMesh& M, int e, const WA& w, const double* Jinv, double eps_e,
                                                  T* K) {
        const int ld = M.ld;
        const double* geo = M.geo;
        const double* tab = M.tab;
        const fp_model_params& P = M.P;
        const bool volumeFluxes = ORDER > 1;
        if (!(volumeFluxes || Mdl::kSource)) return;
        const double jac = ldg(geo + (size_t)GL::JAC * ld + e);
        const double avc = eps_e + M.dampConst;
#pragma unroll 1
        for (int q = 0; q < NQV; q++) {
            const double weight = ldg(tab + TB::o_w + q);
            const double* phi = tab + TB::o_phi + q * NB;
            const double* dphi = tab + TB::o_dphi + q * NB * DIM;
            double u[DIM];
#pragma unroll
            for (int d = 0; d < DIM; d++) u[d] = 0;
            double D = 0, X[DIM];
            if (M.vu != nullptr) {
#pragma unroll
                for (int v = 0; v < NV; v++) {
                    const double li = ldg(tab + TB::o_interp + q * NV + v);
#pragma unroll
                    for (int d = 0; d < DIM; d++) u[d] += li * ldg(M.vu + (size_t)(v * DIM + d) * ld + e);
                }
            }
            if (Mdl::kSource) {
#pragma unroll
                for (int v = 0; v < NV; v++) D += ldg(tab + TB::o_interp + q * NV + v) * ldg(M.vwd + (size_t)v * ld + e);
                const double* xi = tab + TB::o_xi + q * DIM;
#pragma unroll
                for (int i = 0; i < DIM; i++) {
                    double s = 0;
#pragma unroll
                    for (int j = 0; j < DIM; j++) s += ldg(geo + (size_t)(GL::JM + i * DIM + j) * ld + e) * ldg(xi + j);
                    X[i] = s + ldg(geo + (size_t)(GL::X0 + i) * ld + e);
                }
            }
            T WI[NE], dWI[DIM * NE];
            {
                T g[DIM * NE];
#pragma unroll
                for (int m = 0; m < NE; m++) {
                    WI[m] = 0.0;
#pragma unroll
                    for (int d = 0; d < DIM; d++) g[d * NE + m] = 0.0;
#pragma unroll
                    for (int j = 0; j < NB; j++) {
                        const T& c = w[m * NB + j];
                        WI[m] += c * ldg(phi + j);
#pragma unroll
                        for (int d = 0; d < DIM; d++) g[d * NE + m] += c * ldg(dphi + j * DIM + d);
                    }
                }
#pragma unroll
                for (int m = 0; m < NE; m++)
#pragma unroll
                    for (int d = 0; d < DIM; d++) {
                        T s = 0.0;
#pragma unroll
                        for (int qq = 0; qq < DIM; qq++) s += Jinv[qq * DIM + d] * g[qq * NE + m];
                        dWI[d * NE + m] = s;
                    }
            }
            const double jw = jac * weight;
            // G[d][m]: coefficient of d(phi_j)/dx_d, then mapped to the reference gradient
            T G[DIM * NE];
#pragma unroll
            for (int i = 0; i < DIM * NE; i++) G[i] = 0.0;
            // fast path when no density limiting can occur (bit-identical to the per-axis calls)
            const bool unlimited = val(WI[0]) >= RHO_TOL;
            if (volumeFluxes && Mdl::kConvective) {
                if (unlimited) {
                    Mdl::convectiveFluxAll(WI, G, P);
                } else {
#pragma unroll
                    for (int d = 0; d < DIM; d++) {
                        T f[NE];
                        Mdl::convectiveFluxAxis(WI, d, f, P);
#pragma unroll
                        for (int m = 0; m < NE; m++) G[d * NE + m] = f[m];
                    }
                }
            }
            if (volumeFluxes && Mdl::kViscous) {
                T fv[DIM * NE];
                if (unlimited) {
                    Mdl::diffusiveFluxAll(WI, dWI, fv, P);
                } else {
#pragma unroll
                    for (int d = 0; d < DIM; d++) Mdl::diffusiveFlux(WI, dWI, (const double*)nullptr, d, fv + d * NE, P);
                }
#pragma unroll
                for (int i = 0; i < DIM * NE; i++) G[i] -= fv[i];
            }
            T s[NE];
            if (Mdl::kSource) Mdl::sourceTerm(WI, dWI, D, X, s, P);
            if (volumeFluxes) {
#pragma unroll
                for (int d = 0; d < DIM; d++)
#pragma unroll
                    for (int m = 0; m < NE; m++) G[d * NE + m] = jw * (G[d * NE + m] - u[d] * WI[m] - avc * dWI[d * NE + m]);
#pragma unroll
                for (int m = 0; m < NE; m++) {
                    T Gr[DIM];
#pragma unroll
                    for (int dp = 0; dp < DIM; dp++) {
                        T t = 0.0;
#pragma unroll
                        for (int d = 0; d < DIM; d++) t += Jinv[dp * DIM + d] * G[d * NE + m];
                        Gr[dp] = t;
                    }
#pragma unroll
                    for (int j = 0; j < NB; j++) {
                        T a = K[m * NB + j];
#pragma unroll
                        for (int dp = 0; dp < DIM; dp++) a += Gr[dp] * ldg(dphi + j * DIM + dp);
                        K[m * NB + j] = a;
                    }
                }
            }
            if (Mdl::kSource) {
#pragma unroll
                for (int m = 0; m < NE; m++) {
                    const T sw = jw * s[m];
#pragma unroll
                    for (int j = 0; j < NB; j++) K[m * NB + j] += sw * ldg(phi + j);
                }
            }
        }
    }
};

}  // namespace fp
