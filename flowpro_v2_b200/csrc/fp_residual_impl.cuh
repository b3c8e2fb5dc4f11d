// Residual-side kernel templates (instantiated per model in fp_res_*.cu): residual, SSP-RK3 stages, limiter (artificial viscosity),
// positivity limiter, residual norms, time-step bound, finite-difference element
// Jacobian, tangent (JVP).  One element per thread; per-element data in the
// field-major SoA layout of fp_kernels.cuh.
#pragma once
#include <atomic>
#include <cstdio>
#include <type_traits>

#include "fp_ctx.h"
#include "fp_dispatch.cuh"
#include "fp_launch.h"

namespace fp {

constexpr int kBlock = 128;

// Minimum resident CTAs per SM requested from ptxas for the face and element kernels
// (caps registers at 65536 / (128 * MINB)).  Four CTAs (128 registers) pay off for the
// face kernel up to ~24 unknowns per element; the element kernels (residual, RK stage,
// BDF right-hand side) of 13-24 unknowns run faster with three (168 registers, fewer
// spills: 2D Navier-Stokes p = 2, 0.078 -> 0.070 ms on 200,568 triangles); larger
// elements spill too much under either cap.
template <class Mdl, int DIM, int ORDER>
struct MinBlocks {
    static constexpr int NC = Mdl::NE * nbasis_of(DIM, ORDER);
#ifdef FP_MINB_FACE
    static constexpr int face = FP_MINB_FACE;
#else
    static constexpr int face = NC <= 24 ? 4 : 2;
#endif
#ifdef FP_MINB_ELEM
    static constexpr int elem = FP_MINB_ELEM;
#else
    static constexpr int elem = NC <= 12 ? 4 : NC <= 24 ? 3 : 2;
#endif
};

template <class Mdl, int DIM, int ORDER>
using E = Element<Mdl, DIM, ORDER>;

// coefficient c of the face's neighbour, staged by the calling thread in a shared array laid
// out [c][thread] (BLOCK threads); the neighbour index is the face's own
template <int BLOCK>
struct NbShared {
    const double* p;
    __device__ double operator()(int c, int) const { return p[c * BLOCK]; }
};

// coefficient c of the calling thread in a shared array laid out [c][thread] (BLOCK threads)
template <int BLOCK>
struct OwnShared {
    const double* p;
    __device__ double operator[](int c) const { return p[c * BLOCK]; }
};

// The element's own coefficients in the face and element kernels stay in shared memory,
// one column per thread ([c][thread]), instead of NC registers: that keeps the kernels'
// per-point state in registers instead of spilling it.  Up to kShNC unknowns the array is
// static; larger elements take it from the dynamic shared memory of the launch
// (own_smem_bytes, set up by the launchers).
constexpr int kShNC = 24;
extern __shared__ __align__(16) double fp_dyn_smem[];
template <int NC>
constexpr size_t own_smem_bytes() {
    return NC > kShNC ? (size_t)NC * kBlock * sizeof(double) : 0;
}
template <class Mdl, int DIM, int ORDER>
__device__ __forceinline__ OwnShared<kBlock> own_coeffs(const double* __restrict__ W, int ld, int e, double* wsh) {
    constexpr int NC = Element<Mdl, DIM, ORDER>::NC;
#pragma unroll
    for (int c = 0; c < NC; c++) wsh[c * kBlock + threadIdx.x] = ldg(W + (size_t)c * ld + e);
    return OwnShared<kBlock>{wsh + threadIdx.x};
}
// the tangent kernel's coefficients and direction, [c][thread] each, in dynamic shared
// memory when two CTAs of it fit an SM (up to 53 unknowns), else registers
template <int NC>
constexpr size_t matfree_smem_bytes() {
    return 2 * (size_t)NC * kBlock * sizeof(double) <= 106 * 1024 ? 2 * (size_t)NC * kBlock * sizeof(double) : 0;
}
template <int BLOCK>
struct OwnDualShared {
    const double* v;
    const double* d;
    __device__ Dual<1> operator[](int c) const {
        Dual<1> x;
        x.v = v[c * BLOCK];
        x.d[0] = d[c * BLOCK];
        return x;
    }
};
// the finite-difference kernels' coefficients, [c][thread], in dynamic shared memory
template <int NC>
constexpr size_t fd_smem_bytes() {
    return (size_t)NC * kBlock * sizeof(double);
}
// coefficient c of W + V with V = h e_i (the perturbed column of the finite-difference Jacobian)
template <int BLOCK>
struct OwnPerturbed {
    const double* p;
    int i;
    double h;
    __device__ double operator[](int c) const {
        const double v = p[c * BLOCK];
        return c == i ? v + h : v;
    }
};
#define FP_OWN_COEFFS(NC_)                                                   \
    __shared__ double own_wsh_static[(NC_) <= kShNC ? (NC_) * kBlock : 1]; \
    double* own_wsh = (NC_) <= kShNC ? own_wsh_static : fp_dyn_smem

template <class Mdl, int DIM, int ORDER>
__device__ __forceinline__ void load_w(const double* __restrict__ W, int ld, int e, double* w) {
#pragma unroll
    for (int c = 0; c < E<Mdl, DIM, ORDER>::NC; c++) w[c] = ldg(W + (size_t)c * ld + e);
}

// ---------------------------------------------------------------------------- residual
// Face pass of the face-based residual: one thread per face computes the integrand of
// DGpure.residuumWall (DGpure.java:204-353) once and stores both sides' weighted
// contributions, G[0][p] = jw (C - cIP_e Jmp) for the owner and G[1][q] = jw (-C + cIP_nb Jmp)
// for the neighbour at its own quadrature point q = qmap[perm][p] (every term of the face
// integrand is odd in the normal, and the neighbour's normal is the negated one).
template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock, (MinBlocks<Mdl, DIM, ORDER>::face))
    k_face(DevMesh M, const double* __restrict__ W, int f0, int f1) {
    using El = E<Mdl, DIM, ORDER>;
    using GL = GeoLayout<DIM>;
    constexpr int NC = El::NC, NE = El::NE, NQF = El::NQF, NP = El::NP;
    const int f = f0 + blockIdx.x * blockDim.x + threadIdx.x;  // faces f0 .. f1 - 1
    const DevFaces& F = M.F;
    if (f >= f1) return;
    const int ld = M.ld, ldf = F.ldf;
    const int e = F.fl[f], k = F.fk[f], TT = F.fr[f];
    FP_OWN_COEFFS(NC);
    const auto w = own_coeffs<Mdl, DIM, ORDER>(W, ld, e, own_wsh);
    double Jinv[DIM * DIM];
#pragma unroll
    for (int i = 0; i < DIM * DIM; i++) Jinv[i] = ldg(M.geo + (size_t)(GL::JINV + i) * ld + e);
    double n[DIM], Jac, dL;
    El::face_geo(M, e, k, n, Jac, dL);
    const bool interior = TT > -1;
    int kr_face = 0, pm = 0;
    double JinvR[DIM * DIM];
    double eps_nb = 0, cip_nb = 0;
    if (interior) {
        const int fc = F.fc[f];
        kr_face = fc / NP;
        pm = fc - kr_face * NP;
#pragma unroll
        for (int i = 0; i < DIM * DIM; i++) JinvR[i] = ldg(M.geo + (size_t)(GL::JINV + i) * ld + TT);
        eps_nb = ldg(M.eps + TT);
        cip_nb = ldg(M.cip + TT);
    }
    const double eps_e = ldg(M.eps + e);
    const double cip_e = ldg(M.cip + e);
    const bool ip = Mdl::kViscous && (interior || Mdl::isIPFace(TT));
    double* G0 = F.G + f;
    double* G1 = F.G + (size_t)NQF * NE * ldf + f;
    // the neighbour's coefficients, read at every quadrature point: up to kShNC unknowns
    // they are staged once per face in shared memory beside the owner's (48 KB per CTA)
    constexpr bool kShNb = NC <= kShNC;
    __shared__ double nb_wsh[kShNb ? NC * kBlock : 1];
    if constexpr (kShNb) {
        if (interior) {
#pragma unroll
            for (int c = 0; c < NC; c++) nb_wsh[c * kBlock + threadIdx.x] = ldg(W + (size_t)c * ld + TT);
        }
    }
    using NbA = std::conditional_t<kShNb, NbShared<kBlock>, NbPlain>;
    NbA nbl;
    if constexpr (kShNb)
        nbl = NbShared<kBlock>{nb_wsh + threadIdx.x};
    else
        nbl = NbPlain{W, ld};
#pragma unroll 1
    for (int p = 0; p < NQF; p++) {
        double C[NE], Jm[NE];
        El::face_point(M, e, k, p, TT, n, dL, Jinv, JinvR, kr_face, pm, eps_e, eps_nb, w, nbl, C, Jm);
        const double jw = Jac * ldg(M.tab + Tab<DIM, ORDER>::o_wf + p);
        const int q = interior ? F.qmap[pm * NQF + p] : 0;
#pragma unroll
        for (int m = 0; m < NE; m++) {
            G0[(size_t)(p * NE + m) * ldf] = jw * (ip ? C[m] - cip_e * Jm[m] : C[m]);
            if (interior) G1[(size_t)(q * NE + m) * ldf] = jw * (ip ? -C[m] + cip_nb * Jm[m] : -C[m]);
        }
    }
}

template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock, (MinBlocks<Mdl, DIM, ORDER>::elem))
    k_residual(DevMesh M, const double* __restrict__ W, double* __restrict__ R, int e0, int e1) {
    using El = E<Mdl, DIM, ORDER>;
    const int e = e0 + blockIdx.x * blockDim.x + threadIdx.x;  // elements e0 .. e1 - 1
    if (e >= e1) return;
    FP_OWN_COEFFS(El::NC);
    const auto w = own_coeffs<Mdl, DIM, ORDER>(W, M.ld, e, own_wsh);
    double K[El::NC];
    El::residual_from_faces(M, M.F, e, w, K);
#pragma unroll
    for (int c = 0; c < El::NC; c++) R[(size_t)c * M.ld + e] = K[c];
}

// SSP-RK3 stage (RK3.computeExplicitStep, RK3.java:44-86):
// Wout = alpha Wo + beta (Wb + dt M^-1 R(W)); Rsave (optional) = R(W)
template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock, (MinBlocks<Mdl, DIM, ORDER>::elem))
    k_rk_stage(DevMesh M, const double* __restrict__ W, const double* __restrict__ Wo, const double* __restrict__ Wb,
               double alpha, double beta, double dt, double* __restrict__ Wout, double* __restrict__ Rsave) {
    using El = E<Mdl, DIM, ORDER>;
    using TB = Tab<DIM, ORDER>;
    constexpr int NB = El::NB, NE = El::NE, NC = El::NC;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M.nElem) return;
    const int ld = M.ld;
    FP_OWN_COEFFS(NC);
    const auto w = own_coeffs<Mdl, DIM, ORDER>(W, ld, e, own_wsh);
    double K[NC];
    El::residual_from_faces(M, M.F, e, w, K);
    if (Rsave) {
#pragma unroll
        for (int c = 0; c < NC; c++) Rsave[(size_t)c * ld + e] = K[c];
    }
    const double ijac = 1.0 / ldg(M.geo + (size_t)GeoLayout<DIM>::JAC * ld + e);
#pragma unroll
    for (int m = 0; m < NE; m++)
#pragma unroll
        for (int i = 0; i < NB; i++) {
            double s = 0;
#pragma unroll
            for (int j = 0; j < NB; j++) s += ldg(M.tab + TB::o_MinvRef + i * NB + j) * K[m * NB + j];
            const size_t c = (size_t)(m * NB + i) * ld + e;
            const double wo = alpha != 0.0 ? ldg(Wo + c) : 0.0;
            Wout[c] = alpha * wo + beta * (ldg(Wb + c) + dt * (s * ijac));
        }
}

// Matrix-free Newton operator y = a1 M v - (dR/dW) v (the FD-assembled block matrix
// a1 M - dR/dW of BDF2.assembleJacobiMatrix, applied through the tangent of the residual)
template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock)
    k_matfree(DevMesh M, const double* __restrict__ W, const double* __restrict__ V, double a1, double* __restrict__ Y) {
    using El = E<Mdl, DIM, ORDER>;
    using TB = Tab<DIM, ORDER>;
    constexpr int NC = El::NC, NB = El::NB, NE = El::NE;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M.nElem) return;
    case_coefficients(M, e, a1);
    const int ld = M.ld;
    // the element's coefficients and tangent in dynamic shared memory ([c][thread] each)
    // when two CTAs' worth fit an SM, else in registers
    constexpr bool kSh = matfree_smem_bytes<NC>() > 0;
    Dual<1> wr[kSh ? 1 : NC];
    double* shv = fp_dyn_smem;
    double* shd = fp_dyn_smem + NC * kBlock;
    if constexpr (kSh) {
#pragma unroll
        for (int c = 0; c < NC; c++) {
            shv[c * kBlock + threadIdx.x] = ldg(W + (size_t)c * ld + e);
            shd[c * kBlock + threadIdx.x] = ldg(V + (size_t)c * ld + e);
        }
    } else {
#pragma unroll
        for (int c = 0; c < NC; c++) {
            wr[c].v = ldg(W + (size_t)c * ld + e);
            wr[c].d[0] = ldg(V + (size_t)c * ld + e);
        }
    }
    using Own = std::conditional_t<kSh, OwnDualShared<kBlock>, const Dual<1>*>;
    Own w;
    if constexpr (kSh)
        w = OwnDualShared<kBlock>{shv + threadIdx.x, shd + threadIdx.x};
    else
        w = wr;
    Dual<1> K[NC];
    NoKR kr;
    El::residual(M, e, w, NbDual<1>{W, V, ld}, K, kr);
    const double jac = ldg(M.geo + (size_t)GeoLayout<DIM>::JAC * ld + e);
#pragma unroll
    for (int m = 0; m < NE; m++)
#pragma unroll
        for (int i = 0; i < NB; i++) {
            double s = 0;
#pragma unroll
            for (int j = 0; j < NB; j++) s += mass_entry<DIM, ORDER>(M, e, 0, i, j, jac) * w[m * NB + j].d[0];
            Y[(size_t)(m * NB + i) * ld + e] = a1 * s - K[m * NB + i].d[0];
        }
}

// Two-pass form of the same operator: the tangent of each face integrand once per face
// (k_face_tan, both sides' weighted contributions into the face buffer G, as k_face does for
// the residual), then per element the gathered face tangents plus the tangent of the volume
// integral (k_matfree_elem).  The element-gather form above evaluates every interior face
// twice, once from each side.  The limiter's eps and c_IP are constants of the step here as
// there (BDF2.assembleJacobiMatrix differentiates the residual at fixed limiter values).
template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock, 2) k_face_tan(DevMesh M, const double* __restrict__ W, const double* __restrict__ V) {
    using El = E<Mdl, DIM, ORDER>;
    using GL = GeoLayout<DIM>;
    constexpr int NC = El::NC, NE = El::NE, NQF = El::NQF, NP = El::NP;
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    const DevFaces& F = M.F;
    if (f >= F.nFaces) return;
    const int ld = M.ld, ldf = F.ldf;
    const int e = F.fl[f], k = F.fk[f], TT = F.fr[f];
    if (M.case_live && !__ldg(M.case_live + M.case_of[e])) return;
    // the owner's coefficients and tangent in dynamic shared memory ([c][thread] each) when two
    // CTAs' worth fit an SM, else in registers
    constexpr bool kSh = matfree_smem_bytes<NC>() > 0;
    Dual<1> wr[kSh ? 1 : NC];
    double* shv = fp_dyn_smem;
    double* shd = fp_dyn_smem + NC * kBlock;
    if constexpr (kSh) {
#pragma unroll
        for (int c = 0; c < NC; c++) {
            shv[c * kBlock + threadIdx.x] = ldg(W + (size_t)c * ld + e);
            shd[c * kBlock + threadIdx.x] = ldg(V + (size_t)c * ld + e);
        }
    } else {
#pragma unroll
        for (int c = 0; c < NC; c++) {
            wr[c].v = ldg(W + (size_t)c * ld + e);
            wr[c].d[0] = ldg(V + (size_t)c * ld + e);
        }
    }
    using Own = std::conditional_t<kSh, OwnDualShared<kBlock>, const Dual<1>*>;
    Own w;
    if constexpr (kSh)
        w = OwnDualShared<kBlock>{shv + threadIdx.x, shd + threadIdx.x};
    else
        w = wr;
    double Jinv[DIM * DIM];
#pragma unroll
    for (int i = 0; i < DIM * DIM; i++) Jinv[i] = ldg(M.geo + (size_t)(GL::JINV + i) * ld + e);
    double n[DIM], Jac, dL;
    El::face_geo(M, e, k, n, Jac, dL);
    const bool interior = TT > -1;
    int kr_face = 0, pm = 0;
    double JinvR[DIM * DIM];
    double eps_nb = 0, cip_nb = 0;
    if (interior) {
        const int fc = F.fc[f];
        kr_face = fc / NP;
        pm = fc - kr_face * NP;
#pragma unroll
        for (int i = 0; i < DIM * DIM; i++) JinvR[i] = ldg(M.geo + (size_t)(GL::JINV + i) * ld + TT);
        eps_nb = ldg(M.eps + TT);
        cip_nb = ldg(M.cip + TT);
    }
    const double eps_e = ldg(M.eps + e);
    const double cip_e = ldg(M.cip + e);
    const bool ip = Mdl::kViscous && (interior || Mdl::isIPFace(TT));
    double* G0 = F.G + f;
    double* G1 = F.G + (size_t)NQF * NE * ldf + f;
    const NbDual<1> nbl{W, V, ld};
#pragma unroll 1
    for (int p = 0; p < NQF; p++) {
        Dual<1> C[NE], Jm[NE];
        El::face_point(M, e, k, p, TT, n, dL, Jinv, JinvR, kr_face, pm, eps_e, eps_nb, w, nbl, C, Jm);
        const double jw = Jac * ldg(M.tab + Tab<DIM, ORDER>::o_wf + p);
        const int q = interior ? F.qmap[pm * NQF + p] : 0;
#pragma unroll
        for (int m = 0; m < NE; m++) {
            const double c = C[m].d[0], j = Jm[m].d[0];
            G0[(size_t)(p * NE + m) * ldf] = jw * (ip ? c - cip_e * j : c);
            if (interior) G1[(size_t)(q * NE + m) * ldf] = jw * (ip ? -c + cip_nb * j : -c);
        }
    }
}

template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock, 2)
    k_matfree_elem(DevMesh M, const double* __restrict__ W, const double* __restrict__ V, double a1, double* __restrict__ Y) {
    using El = E<Mdl, DIM, ORDER>;
    using TB = Tab<DIM, ORDER>;
    using GL = GeoLayout<DIM>;
    constexpr int NC = El::NC, NB = El::NB, NE = El::NE, NQF = El::NQF, NF = El::NF;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M.nElem) return;
    if (M.case_live && !__ldg(M.case_live + M.case_of[e])) return;
    case_coefficients(M, e, a1);
    const int ld = M.ld;
    constexpr bool kSh = matfree_smem_bytes<NC>() > 0;
    Dual<1> wr[kSh ? 1 : NC];
    double* shv = fp_dyn_smem;
    double* shd = fp_dyn_smem + NC * kBlock;
    if constexpr (kSh) {
#pragma unroll
        for (int c = 0; c < NC; c++) {
            shv[c * kBlock + threadIdx.x] = ldg(W + (size_t)c * ld + e);
            shd[c * kBlock + threadIdx.x] = ldg(V + (size_t)c * ld + e);
        }
    } else {
#pragma unroll
        for (int c = 0; c < NC; c++) {
            wr[c].v = ldg(W + (size_t)c * ld + e);
            wr[c].d[0] = ldg(V + (size_t)c * ld + e);
        }
    }
    using Own = std::conditional_t<kSh, OwnDualShared<kBlock>, const Dual<1>*>;
    Own w;
    if constexpr (kSh)
        w = OwnDualShared<kBlock>{shv + threadIdx.x, shd + threadIdx.x};
    else
        w = wr;
    Dual<1> K[NC];
    // gathered face tangents (their values are not needed: only K.d is used)
    const DevFaces& F = M.F;
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
                for (int j = 0; j < NB; j++) K[m * NB + j].d[0] += g * ldg(phi + j);
            }
        }
    }
    double Jinv[DIM * DIM];
#pragma unroll
    for (int i = 0; i < DIM * DIM; i++) Jinv[i] = ldg(M.geo + (size_t)(GL::JINV + i) * ld + e);
    El::volume(M, e, w, Jinv, ldg(M.eps + e), K);
    const double jac = ldg(M.geo + (size_t)GL::JAC * ld + e);
#pragma unroll
    for (int m = 0; m < NE; m++)
#pragma unroll
        for (int i = 0; i < NB; i++) {
            double s = 0;
#pragma unroll
            for (int j = 0; j < NB; j++) s += mass_entry<DIM, ORDER>(M, e, 0, i, j, jac) * w[m * NB + j].d[0];
            Y[(size_t)(m * NB + i) * ld + e] = a1 * s - K[m * NB + i].d[0];
        }
}

// ---------------------------------------------------------------------------- limiter
// DGpure.limiter + shock_senzor (DGpure.java:358-452): eps = lambda h / order * sensor,
// c_IP = penalty for diffusive models; both zero for piecewise constants.
template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock)
    k_limiter(DevMesh M, const double* __restrict__ W, double dampTol, double penalty, const double* __restrict__ trun,
              double* __restrict__ eps, double* __restrict__ cip) {
    using TB = Tab<DIM, ORDER>;
    constexpr int NB = TB::NB, NE = Mdl::NE, NQV = TB::NQV;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M.nElem) return;
    const int ld = M.ld;
    double ep = 0, ci = 0;
    if (ORDER > 1) {
        double Ws[NE];
#pragma unroll
        for (int m = 0; m < NE; m++) {
            double s = 0;
#pragma unroll
            for (int j = 0; j < NB; j++) s = s + ldg(W + (size_t)(m * NB + j) * ld + e) * ldg(M.tab + TB::o_Is + j);
            Ws[m] = s;
        }
        double u[DIM];
#pragma unroll
        for (int d = 0; d < DIM; d++) u[d] = 0;
        const double lam = val(Mdl::maxEigenvalue(Ws, u, M.P));
        if (dampTol > 0) {
            double rho[NB], tr[NB];
#pragma unroll
            for (int j = 0; j < NB; j++) rho[j] = ldg(W + (size_t)j * ld + e);
            if (ORDER > 2) {
#pragma unroll
                for (int i = 0; i < NB; i++) {
                    double s = 0;
#pragma unroll
                    for (int j = 0; j < NB; j++) s += ldg(trun + i * NB + j) * rho[j];
                    tr[i] = s;
                }
            } else {
                double avg = 0;
#pragma unroll
                for (int j = 0; j < NB; j++) avg = avg + rho[j] * ldg(M.tab + TB::o_Is + j);
#pragma unroll
                for (int i = 0; i < NB; i++) tr[i] = avg;
            }
            const double jac = ldg(M.geo + (size_t)GeoLayout<DIM>::JAC * ld + e);
            double Se = 0, pod = 0;
#pragma unroll 1
            for (int q = 0; q < NQV; q++) {
                double ri = 0, rt = 0;
#pragma unroll
                for (int j = 0; j < NB; j++) {
                    const double ph = ldg(M.tab + TB::o_phi + q * NB + j);
                    ri += rho[j] * ph;
                    rt += tr[j] * ph;
                }
                const double jw = jac * ldg(M.tab + TB::o_w + q);
                Se += jw * (ri - rt) * (ri - rt);
                pod += jw * ri * ri;
            }
            Se = log10(fabs(Se / pod));
            const double S0 = log10(1. / pow((double)(ORDER - 1), 4.0));
            double shock = 0.5 * (1 + sin(M_PI * (Se - S0) / (2 * dampTol)));
            if (Se < S0 - dampTol) shock = 0;
            if (Se > S0 + dampTol) shock = 1;
            if (isnan(shock)) shock = 0;
            ep = lam * ldg(M.geo + (size_t)GeoLayout<DIM>::SIZE * ld + e) / ORDER * shock;
        }
        if (Mdl::kViscous) ci = penalty;
    }
    eps[e] = ep;
    cip[e] = ci;
}

// ---------------------------------------------------------------------------- positivity limiter
// Element.positivityLimiter (Element.java:385-476): largest theta in [0,1] (30 bisection
// steps per point) that makes Wavg + theta (W(x) - Wavg) admissible in all volume and
// face quadrature points; W = mean + theta (W - mean).
template <class Mdl, int DIM, int ORDER>
__device__ double admissible_theta(const double* w, const double* Wavg, const double* phi) {
    constexpr int NB = nbasis_of(DIM, ORDER), NE = Mdl::NE;
    double Wx[NE];
#pragma unroll
    for (int m = 0; m < NE; m++) {
        double s = 0;
#pragma unroll
        for (int j = 0; j < NB; j++) s += w[m * NB + j] * ldg(phi + j);
        Wx[m] = s;
    }
    if (Mdl::isAdmissible(Wx)) return 1;
    double lo = 0, hi = 1, Wt[NE];
    for (int it = 0; it < 30; it++) {
        double mid = 0.5 * (lo + hi);
#pragma unroll
        for (int m = 0; m < NE; m++) Wt[m] = Wavg[m] + mid * (Wx[m] - Wavg[m]);
        if (Mdl::isAdmissible(Wt))
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock) k_positivity(DevMesh M, double* __restrict__ W, int* __restrict__ count) {
    using TB = Tab<DIM, ORDER>;
    constexpr int NB = TB::NB, NE = Mdl::NE, NC = NE * NB;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M.nElem || NB == 1) return;
    const int ld = M.ld;
    double w[NC];
    load_w<Mdl, DIM, ORDER>(W, ld, e, w);
    double Wavg[NE];
#pragma unroll
    for (int m = 0; m < NE; m++) {
        double s = 0;
#pragma unroll
        for (int j = 0; j < NB; j++) s = s + w[m * NB + j] * ldg(M.tab + TB::o_Is + j);
        Wavg[m] = s;
    }
    if (!Mdl::isAdmissible(Wavg)) return;
    double theta = 1;
    for (int q = 0; q < TB::NQV; q++) theta = fmin(theta, admissible_theta<Mdl, DIM, ORDER>(w, Wavg, M.tab + TB::o_phi + q * NB));
    for (int k = 0; k < TB::NF; k++)
        for (int p = 0; p < TB::NQF; p++)
            theta = fmin(theta, admissible_theta<Mdl, DIM, ORDER>(w, Wavg, M.tab + TB::o_phiL + (k * TB::NQF + p) * NB));
    if (theta >= 1) return;
#pragma unroll
    for (int m = 0; m < NE; m++)
#pragma unroll
        for (int i = 0; i < NB; i++) {
            const double mean = ldg(M.tab + TB::o_one + i) * Wavg[m];
            W[(size_t)(m * NB + i) * ld + e] = mean + theta * (w[m * NB + i] - mean);
        }
    atomicAdd(count, 1);
}

// ---------------------------------------------------------------------------- reductions
// per-block partial sums of the element norms R_m^T M^-1 R_m (Element.l2NormsSquared)
template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock) k_norms(DevMesh M, const double* __restrict__ R, double* __restrict__ part) {
    using TB = Tab<DIM, ORDER>;
    constexpr int NB = TB::NB, NE = Mdl::NE;
    __shared__ double sh[kBlock][NE];
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double nrm[NE];
#pragma unroll
    for (int m = 0; m < NE; m++) nrm[m] = 0;
    if (e < M.nElem) {
        const int ld = M.ld;
        const double ijac = 1.0 / ldg(M.geo + (size_t)GeoLayout<DIM>::JAC * ld + e);
#pragma unroll
        for (int m = 0; m < NE; m++) {
            double r[NB];
#pragma unroll
            for (int j = 0; j < NB; j++) r[j] = ldg(R + (size_t)(m * NB + j) * ld + e);
            double sum = 0;
#pragma unroll
            for (int i = 0; i < NB; i++) {
                double t = 0;
#pragma unroll
                for (int j = 0; j < NB; j++) t += ldg(M.tab + TB::o_MinvRef + i * NB + j) * ijac * r[j];
                sum += r[i] * t;
            }
            nrm[m] = sum;
        }
    }
#pragma unroll
    for (int m = 0; m < NE; m++) sh[threadIdx.x][m] = nrm[m];
    __syncthreads();
    for (int s = kBlock / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
#pragma unroll
            for (int m = 0; m < NE; m++) sh[threadIdx.x][m] += sh[threadIdx.x + s][m];
        __syncthreads();
    }
    if (threadIdx.x == 0)
#pragma unroll
        for (int m = 0; m < NE; m++) part[(size_t)blockIdx.x * NE + m] = sh[0][m];
}

// per-block minimum of elemSize / lambda (State.getTimeStep, Element.delta_t)
template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock) k_dtbound(DevMesh M, const double* __restrict__ W, double factor, double* __restrict__ part) {
    using TB = Tab<DIM, ORDER>;
    constexpr int NB = TB::NB, NE = Mdl::NE;
    __shared__ double sh[kBlock];
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 1.0e300;
    if (e < M.nElem) {
        const int ld = M.ld;
        double Ws[NE];
#pragma unroll
        for (int m = 0; m < NE; m++) {
            double s = 0;
#pragma unroll
            for (int j = 0; j < NB; j++) s = s + ldg(W + (size_t)(m * NB + j) * ld + e) * ldg(M.tab + TB::o_Is + j);
            Ws[m] = s;
        }
        double u[DIM];
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            u[d] = 0;
            if (M.vu)
                for (int v2 = 0; v2 < DIM + 1; v2++) u[d] += ldg(M.vu + (size_t)(v2 * DIM + d) * ld + e) / (DIM + 1);
        }
        const double lam = val(Mdl::maxEigenvalue(Ws, u, M.P));
        if (lam > 0) v = ldg(M.geo + (size_t)GeoLayout<DIM>::SIZE * ld + e) / lam / factor;
    }
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = kBlock / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] = fmin(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// per-element forms of the two reductions above, for a batch of cases (summed or minimised
// per case afterwards): out[m][e] = R_m^T M^-1 R_m of element e, out[e] = elemSize / lambda / factor
template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock) k_norms_elem(DevMesh M, const double* __restrict__ R, double* __restrict__ out) {
    using TB = Tab<DIM, ORDER>;
    constexpr int NB = TB::NB, NE = Mdl::NE;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M.nElem) return;
    const int ld = M.ld;
    const double ijac = 1.0 / ldg(M.geo + (size_t)GeoLayout<DIM>::JAC * ld + e);
#pragma unroll
    for (int m = 0; m < NE; m++) {
        double r[NB];
#pragma unroll
        for (int j = 0; j < NB; j++) r[j] = ldg(R + (size_t)(m * NB + j) * ld + e);
        double sum = 0;
#pragma unroll
        for (int i = 0; i < NB; i++) {
            double t = 0;
#pragma unroll
            for (int j = 0; j < NB; j++) t += ldg(M.tab + TB::o_MinvRef + i * NB + j) * ijac * r[j];
            sum += r[i] * t;
        }
        out[(size_t)m * ld + e] = sum;
    }
}

template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock)
    k_dtbound_elem(DevMesh M, const double* __restrict__ W, double factor, double* __restrict__ out) {
    using TB = Tab<DIM, ORDER>;
    constexpr int NB = TB::NB, NE = Mdl::NE;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M.nElem) return;
    const int ld = M.ld;
    double v = 1.0e300;
    double Ws[NE];
#pragma unroll
    for (int m = 0; m < NE; m++) {
        double s = 0;
#pragma unroll
        for (int j = 0; j < NB; j++) s = s + ldg(W + (size_t)(m * NB + j) * ld + e) * ldg(M.tab + TB::o_Is + j);
        Ws[m] = s;
    }
    double u[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        u[d] = 0;
        if (M.vu)
            for (int v2 = 0; v2 < DIM + 1; v2++) u[d] += ldg(M.vu + (size_t)(v2 * DIM + d) * ld + e) / (DIM + 1);
    }
    const double lam = val(Mdl::maxEigenvalue(Ws, u, M.P));
    if (lam > 0) v = ldg(M.geo + (size_t)GeoLayout<DIM>::SIZE * ld + e) / lam / factor;
    out[e] = v;
}

// ---------------------------------------------------------------------------- implicit RHS
// Implicit.assembleResiduum (BDF2.java:279-317): R(W), RHS = R - M (a1 W + a2 Wo + a3 Wo2),
// per-block partial sums of |RHS|^2.
template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock, (MinBlocks<Mdl, DIM, ORDER>::elem))
    k_rhs(DevMesh M, const double* __restrict__ W, const double* __restrict__ Wo, const double* __restrict__ Wo2, double a1,
          double a2, double a3, double* __restrict__ R, double* __restrict__ rhs, double* __restrict__ part) {
    using El = E<Mdl, DIM, ORDER>;
    using TB = Tab<DIM, ORDER>;
    constexpr int NB = El::NB, NE = El::NE, NC = El::NC;
    __shared__ double sh[kBlock];
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double loc = 0;
    FP_OWN_COEFFS(NC);
    if (e < M.nElem) {
        case_coefficients(M, e, a1, a2, a3);
        const int ld = M.ld;
        const auto w = own_coeffs<Mdl, DIM, ORDER>(W, ld, e, own_wsh);
        double K[NC];
        El::residual_from_faces(M, M.F, e, w, K);
        const double jac = ldg(M.geo + (size_t)GeoLayout<DIM>::JAC * ld + e);
#pragma unroll
        for (int m = 0; m < NE; m++) {
            double y[NB], yo[NB], yo2[NB];
#pragma unroll
            for (int j = 0; j < NB; j++) {
                const size_t c = (size_t)(m * NB + j) * ld + e;
                y[j] = a1 * w[m * NB + j] + a2 * ldg(Wo + c) + (a3 != 0.0 ? a3 * ldg(Wo2 + c) : 0.0);
                if (M.mass) {  // moving mesh: M a1 W + Mo a2 Wo + Mo2 a3 Wo2 (BDF2.assembleRHS)
                    y[j] = a1 * w[m * NB + j];
                    yo[j] = a2 * ldg(Wo + c);
                    yo2[j] = a3 * ldg(Wo2 + c);
                }
            }
#pragma unroll
            for (int i = 0; i < NB; i++) {
                double s = 0;
                if (M.mass) {
#pragma unroll
                    for (int j = 0; j < NB; j++)
                        s += mass_entry<DIM, ORDER>(M, e, 0, i, j, jac) * y[j] + mass_entry<DIM, ORDER>(M, e, 1, i, j, jac) * yo[j] +
                             mass_entry<DIM, ORDER>(M, e, 2, i, j, jac) * yo2[j];
                } else {
#pragma unroll
                    for (int j = 0; j < NB; j++) s += ldg(M.tab + TB::o_Mref + i * NB + j) * jac * y[j];
                }
                const double v = K[m * NB + i] - s;
                rhs[(size_t)(m * NB + i) * ld + e] = v;
                R[(size_t)(m * NB + i) * ld + e] = K[m * NB + i];
                loc += v * v;
            }
        }
    }
    sh[threadIdx.x] = loc;
    __syncthreads();
    for (int s = kBlock / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// ---------------------------------------------------------------------------- FD Jacobian
// BDF2.assembleJacobiMatrix finite differences (BDF2.java:349-378): per element, the
// residual with W + h e_i for every own unknown i; the diagonal block column
// A[r][i] = -(R_i[r] - R[r]) / h + a1 M, and the block of each face neighbour
// A_nb[r][i] = (KR_i[r] - KR[r]) / h from this element's face integrals.
template <int NC>
struct KRBase {
    static constexpr bool enabled = true;
    double acc[NC];
    double* KR0;
    int ld, e;
    template <class T>
    __device__ void begin(int) {
#pragma unroll
        for (int c = 0; c < NC; c++) acc[c] = 0;
    }
    __device__ void add(int, int c, double v) { acc[c] += v; }
    __device__ void end(int k, int, int) {
#pragma unroll
        for (int c = 0; c < NC; c++) KR0[((size_t)k * NC + c) * ld + e] = acc[c];
    }
};

template <int NC>
struct KRCol {
    static constexpr bool enabled = true;
    double acc[NC];
    const double* KR0;
    double* Aneigh;
    int ld, e, i;
    double invh;
    template <class T>
    __device__ void begin(int) {
#pragma unroll
        for (int c = 0; c < NC; c++) acc[c] = 0;
    }
    __device__ void add(int, int c, double v) { acc[c] += v; }
    __device__ void end(int k, int nb, int kr) {
        // block of element nb for its face kr, column i (this element's unknown i)
        double* A = Aneigh + (size_t)kr * NC * NC * ld;
#pragma unroll
        for (int r = 0; r < NC; r++)
            A[((size_t)r * NC + i) * ld + nb] = (acc[r] - ldg(KR0 + ((size_t)k * NC + r) * ld + e)) * invh;
    }
};

template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock)
    k_fd_base(DevMesh M, const double* __restrict__ W, double* __restrict__ K0, double* __restrict__ KR0) {
    using El = E<Mdl, DIM, ORDER>;
    constexpr int NC = El::NC;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M.nElem) return;
    double* wsh = fp_dyn_smem;
#pragma unroll
    for (int c = 0; c < NC; c++) wsh[c * kBlock + threadIdx.x] = ldg(W + (size_t)c * M.ld + e);
    const OwnShared<kBlock> w{wsh + threadIdx.x};
    double K[NC];
    KRBase<NC> kr;
    kr.KR0 = KR0;
    kr.ld = M.ld;
    kr.e = e;
    El::residual(M, e, w, NbPlain{W, M.ld}, K, kr);
#pragma unroll
    for (int c = 0; c < NC; c++) K0[(size_t)c * M.ld + e] = K[c];
}

template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock)
    k_fd_col(DevMesh M, const double* __restrict__ W, const double* __restrict__ K0, const double* __restrict__ KR0, double h,
             double a1, double* __restrict__ Adiag, double* __restrict__ Aneigh) {
    using El = E<Mdl, DIM, ORDER>;
    using TB = Tab<DIM, ORDER>;
    constexpr int NC = El::NC, NB = El::NB;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int e = (int)(t % M.nElem);
    const int i = (int)(t / M.nElem);
    if (i >= NC) return;
    case_coefficients(M, e, a1);
    const int ld = M.ld;
    double* wsh = fp_dyn_smem;
#pragma unroll
    for (int c = 0; c < NC; c++) wsh[c * kBlock + threadIdx.x] = ldg(W + (size_t)c * ld + e);
    const OwnPerturbed<kBlock> w{wsh + threadIdx.x, i, h};  // W + V with V[i] = h (DGpure.residuum)
    double K[NC];
    KRCol<NC> kr;
    kr.KR0 = KR0;
    kr.Aneigh = Aneigh;
    kr.ld = ld;
    kr.e = e;
    kr.i = i;
    kr.invh = 1.0 / h;
    El::residual(M, e, w, NbPlain{W, ld}, K, kr);
    const double jac = ldg(M.geo + (size_t)GeoLayout<DIM>::JAC * ld + e);
    const int mi = i / NB, bi = i - mi * NB;
#pragma unroll
    for (int r = 0; r < NC; r++) {
        double a = (K[r] - ldg(K0 + (size_t)r * ld + e)) / (-h);
        const int mr = r / NB, br = r - mr * NB;
        if (mr == mi) a += a1 * mass_entry<DIM, ORDER>(M, e, 0, br, bi, jac);
        Adiag[((size_t)r * NC + i) * ld + e] = a;
    }
}

// ---------------------------------------------------------------------------- exact element Jacobian
// The FD assembly above with the finite difference replaced by the exact tangent: column i
// of the blocks is the Dual<1> derivative of the element residual (and of this element's
// face contributions to its neighbours) along e_i.  Same storage and signs as k_fd_col.
template <int N>
struct NbConst {
    const double* W;
    int ld;
    __device__ Dual<N> operator()(int c, int nb) const { return Dual<N>(ldg(W + (size_t)c * ld + nb)); }
};

template <int NC>
struct KRColExact {
    static constexpr bool enabled = true;
    double acc[NC];
    double* Aneigh;
    int ld, i;
    template <class T>
    __device__ void begin(int) {
#pragma unroll
        for (int c = 0; c < NC; c++) acc[c] = 0;
    }
    __device__ void add(int, int c, const Dual<1>& v) { acc[c] += v.d[0]; }
    __device__ void end(int, int nb, int kr) {
        double* A = Aneigh + (size_t)kr * NC * NC * ld;
#pragma unroll
        for (int r = 0; r < NC; r++) A[((size_t)r * NC + i) * ld + nb] = acc[r];
    }
};

template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock)
    k_jac_exact(DevMesh M, const double* __restrict__ W, double a1, double* __restrict__ Adiag, double* __restrict__ Aneigh) {
    using El = E<Mdl, DIM, ORDER>;
    using TB = Tab<DIM, ORDER>;
    constexpr int NC = El::NC, NB = El::NB;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int e = (int)(t % M.nElem);
    const int i = (int)(t / M.nElem);
    if (i >= NC) return;
    case_coefficients(M, e, a1);
    const int ld = M.ld;
    Dual<1> w[NC], K[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) {
        w[c].v = ldg(W + (size_t)c * ld + e);
        w[c].d[0] = c == i ? 1.0 : 0.0;
    }
    KRColExact<NC> kr;
    kr.Aneigh = Aneigh;
    kr.ld = ld;
    kr.i = i;
    El::residual(M, e, w, NbConst<1>{W, ld}, K, kr);
    const double jac = ldg(M.geo + (size_t)GeoLayout<DIM>::JAC * ld + e);
    const int mi = i / NB, bi = i - mi * NB;
#pragma unroll
    for (int r = 0; r < NC; r++) {
        double a = -K[r].d[0];
        const int mr = r / NB, br = r - mr * NB;
        if (mr == mi) a += a1 * mass_entry<DIM, ORDER>(M, e, 0, br, bi, jac);
        Adiag[((size_t)r * NC + i) * ld + e] = a;
    }
}

// The exact blocks written straight into the block ILU(0) factor storage (element-major,
// column-major blocks F[e][s][c][r] in T = float or double; s = 0 the diagonal block, s = 1 + k
// the block coupling the row element with its neighbour over face k), so the matrix-free
// Newton path keeps no copy of the operator's blocks: column i of element e's diagonal block
// and column i of each neighbour's block toward e, each a contiguous run of NC values.
template <int NC, int NF, class T>
struct KRColFactor {
    static constexpr bool enabled = true;
    double acc[NC];
    T* F;
    int i;
    template <class U>
    __device__ void begin(int) {
#pragma unroll
        for (int c = 0; c < NC; c++) acc[c] = 0;
    }
    __device__ void add(int, int c, const Dual<1>& v) { acc[c] += v.d[0]; }
    __device__ void end(int, int nb, int kr) {
        T* A = F + (((size_t)nb * (1 + NF) + 1 + kr) * NC + i) * NC;
#pragma unroll
        for (int r = 0; r < NC; r++) A[r] = (T)acc[r];
    }
};

template <class Mdl, int DIM, int ORDER, class T>
__global__ void __launch_bounds__(kBlock)
    k_jac_exact_factor(DevMesh M, const double* __restrict__ W, double a1, T* __restrict__ F) {
    using El = E<Mdl, DIM, ORDER>;
    using TB = Tab<DIM, ORDER>;
    constexpr int NC = El::NC, NB = El::NB, NF = El::NF;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int e = (int)(t % M.nElem);
    const int i = (int)(t / M.nElem);
    if (i >= NC) return;
    case_coefficients(M, e, a1);
    const int ld = M.ld;
    Dual<1> w[NC], K[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) {
        w[c].v = ldg(W + (size_t)c * ld + e);
        w[c].d[0] = c == i ? 1.0 : 0.0;
    }
    KRColFactor<NC, NF, T> kr;
    kr.F = F;
    kr.i = i;
    El::residual(M, e, w, NbConst<1>{W, ld}, K, kr);
    const double jac = ldg(M.geo + (size_t)GeoLayout<DIM>::JAC * ld + e);
    const int mi = i / NB, bi = i - mi * NB;
    T* A = F + ((size_t)e * (1 + NF) * NC + i) * NC;
#pragma unroll
    for (int r = 0; r < NC; r++) {
        double a = -K[r].d[0];
        const int mr = r / NB, br = r - mr * NB;
        if (mr == mi) a += a1 * mass_entry<DIM, ORDER>(M, e, 0, br, bi, jac);
        A[r] = (T)a;
    }
}

// ---------------------------------------------------------------------------- moving mesh
// Mass matrix of time level lev from the current geometry (DGpure.recalculateMassMatrix,
// DGpure.java:575-593): M_ij = sum_p jac w_p phi_i(p) phi_j(p), in the reference's order.
template <int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock) k_mass_geo(DevMesh M, int lev, double* __restrict__ mass) {
    using TB = Tab<DIM, ORDER>;
    constexpr int NB = TB::NB, NQV = TB::NQV;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M.nElem) return;
    const int ld = M.ld;
    const double jac = ldg(M.geo + (size_t)GeoLayout<DIM>::JAC * ld + e);
    for (int i = 0; i < NB; i++)
        for (int j = 0; j < NB; j++) {
            double m = 0;
            for (int q = 0; q < NQV; q++)
                m = m + jac * ldg(M.tab + TB::o_w + q) * ldg(M.tab + TB::o_phi + q * NB + i) * ldg(M.tab + TB::o_phi + q * NB + j);
            mass[((size_t)(lev * NB + i) * NB + j) * ld + e] = m;
        }
}

// Discrete geometric conservation law (Element.applyGCLMassMatrix, Element.java:568-630): the
// current level's mass matrix becomes M = (B - a2 Mo - a3 Mo2) / a1 with
// B_ij = sum_faces int (u.n) phi_i phi_j ds - int u . grad(phi_i phi_j) dx, u the mesh velocity
// interpolated from the element's vertices, so that a uniform state satisfies the BDF update
// exactly on the moving mesh.
template <int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock) k_gcl_mass(DevMesh M, double a1, double a2, double a3, double* __restrict__ mass) {
    using TB = Tab<DIM, ORDER>;
    using GL = GeoLayout<DIM>;
    constexpr int NB = TB::NB, NQV = TB::NQV, NQF = TB::NQF, NF = TB::NF, NV = TB::NV, NVF = TB::NVF;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M.nElem || !M.vu) return;
    const int ld = M.ld;
    double B[NB][NB];
#pragma unroll
    for (int i = 0; i < NB; i++)
#pragma unroll
        for (int j = 0; j < NB; j++) B[i][j] = 0;
    for (int k = 0; k < NF; k++) {
        double n[DIM];
#pragma unroll
        for (int d = 0; d < DIM; d++) n[d] = ldg(M.geo + (size_t)(GL::NRM + k * DIM + d) * ld + e);
        const double jf = ldg(M.geo + (size_t)(GL::JF + k) * ld + e);
        for (int p = 0; p < NQF; p++) {
            double un = 0;
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                double ud = 0;
#pragma unroll
                for (int v = 0; v < NVF; v++)
                    ud += ldg(M.tab + TB::o_finterp + p * NVF + v) * ldg(M.vu + (size_t)(face_vertex<DIM>(k, v) * DIM + d) * ld + e);
                un += ud * n[d];
            }
            const double* base = M.tab + TB::o_phiL + (k * NQF + p) * NB;
            const double jw = jf * ldg(M.tab + TB::o_wf + p) * un;
#pragma unroll
            for (int i = 0; i < NB; i++)
#pragma unroll
                for (int j = 0; j < NB; j++) B[i][j] += jw * ldg(base + i) * ldg(base + j);
        }
    }
    double Jinv[DIM * DIM];
#pragma unroll
    for (int i = 0; i < DIM * DIM; i++) Jinv[i] = ldg(M.geo + (size_t)(GL::JINV + i) * ld + e);
    const double jac = ldg(M.geo + (size_t)GL::JAC * ld + e);
    for (int q = 0; q < NQV; q++) {
        double u[DIM];
#pragma unroll
        for (int d = 0; d < DIM; d++) u[d] = 0;
#pragma unroll
        for (int v = 0; v < NV; v++)
#pragma unroll
            for (int d = 0; d < DIM; d++) u[d] += ldg(M.tab + TB::o_interp + q * NV + v) * ldg(M.vu + (size_t)(v * DIM + d) * ld + e);
        const double* base = M.tab + TB::o_phi + q * NB;
        const double* dphi = M.tab + TB::o_dphi + q * NB * DIM;
        const double jw = jac * ldg(M.tab + TB::o_w + q);
        double ug[NB];  // u . grad phi_i (physical gradients J^-T grad_xi phi_i)
#pragma unroll
        for (int i = 0; i < NB; i++) {
            double s = 0;
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                double gd = 0;
#pragma unroll
                for (int qq = 0; qq < DIM; qq++) gd += Jinv[qq * DIM + d] * ldg(dphi + i * DIM + qq);
                s += u[d] * gd;
            }
            ug[i] = s;
        }
#pragma unroll
        for (int i = 0; i < NB; i++)
#pragma unroll
            for (int j = 0; j < NB; j++) B[i][j] -= jw * (ug[i] * ldg(base + j) + ldg(base + i) * ug[j]);
    }
#pragma unroll
    for (int i = 0; i < NB; i++)
#pragma unroll
        for (int j = 0; j < NB; j++) {
            const size_t o = (size_t)(i * NB + j) * ld + e, lv = (size_t)NB * NB * ld;
            mass[o] = (B[i][j] - a2 * mass[o + lv] - a3 * mass[o + 2 * lv]) / a1;
        }
}

// ---------------------------------------------------------------------------- VJP
// g = (dR/dW)^T lambda without a stored Jacobian: thread (e, i) forms column i of its
// element's blocks in registers (the Dual<1> tangent of the element residual along e_i,
// quadrature states recomputed, as k_jac_exact does) and contracts it at once with the
// adjoint weights it multiplies: lambda_e for the element's own rows and lambda_nb for the rows
// of each face neighbour its face integrals feed (the KR terms of DGpure.residuumWall), so
// g[i][e] = sum_r dR_e[r]/dW_e,i lambda_e[r] + sum_nb sum_r dR_nb[r]/dW_e,i lambda_nb[r].
// The neighbour terms carry the sign of the assembled neighbour blocks (A = a1 M - dR/dW).
struct KRColVjp {
    static constexpr bool enabled = true;
    const int* tt;
    const double* lam;
    int ld, e, nb;
    double s;
    template <class U>
    __device__ void begin(int k) {
        nb = tt[(size_t)k * ld + e];
    }
    __device__ void add(int, int c, const Dual<1>& v) { s += v.d[0] * ldg(lam + (size_t)c * ld + nb); }
    __device__ void end(int, int, int) {}
};

template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock)
    k_vjp_cols(DevMesh M, const double* __restrict__ W, const double* __restrict__ lam, double* __restrict__ g) {
    using El = E<Mdl, DIM, ORDER>;
    constexpr int NC = El::NC;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int e = (int)(t % M.nElem);
    const int i = (int)(t / M.nElem);
    if (i >= NC) return;
    const int ld = M.ld;
    Dual<1> w[NC], K[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) {
        w[c].v = ldg(W + (size_t)c * ld + e);
        w[c].d[0] = c == i ? 1.0 : 0.0;
    }
    KRColVjp kr;
    kr.tt = M.tt;
    kr.lam = lam;
    kr.ld = ld;
    kr.e = e;
    kr.nb = -1;
    kr.s = 0.0;
    El::residual(M, e, w, NbConst<1>{W, ld}, K, kr);
    double own = 0.0;
#pragma unroll
    for (int r = 0; r < NC; r++) own += K[r].d[0] * ldg(lam + (size_t)r * ld + e);
    g[(size_t)i * ld + e] = own - kr.s;
}

// ---------------------------------------------------------------------------- surface integrals
// kind 0: force on the faces of boundary type bc, F = -sum int stressVector ds
//         (Deformation2DRigid.calculateForces, Deformation2DRigid.java:81-105);
// kind 1 / 2: lift / drag coefficient functional, int p n_y (n_x) ds on faces of type bc
//         (LiftCoefficient.java:31-49, DragCoefficient.java:30-48, summed as
//         Element.computeFunctional, Element.java:789-862), and optionally its exact
//         gradient dI/dW (forward mode over the trace state, state layout).
// Per-block partial sums part[block * 4 + v] (deterministic order on the host).
template <class Mdl, int DIM, int ORDER>
__global__ void __launch_bounds__(kBlock)
    k_surface(DevMesh M, const double* __restrict__ W, int kind, int bc, double* __restrict__ part, double* __restrict__ dIdW) {
    using El = E<Mdl, DIM, ORDER>;
    using TB = Tab<DIM, ORDER>;
    using GL = GeoLayout<DIM>;
    constexpr int NB = El::NB, NE = El::NE, NQF = El::NQF, NF = El::NF, NC = El::NC;
    __shared__ double sh[kBlock][4];
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (e < M.nElem) {
        const int ld = M.ld;
        bool any = false;
#pragma unroll
        for (int k = 0; k < NF; k++) any = any || M.tt[(size_t)k * ld + e] == bc;
        const bool grad = dIdW != nullptr && kind > 0;
        double g[NC];
#pragma unroll
        for (int c = 0; c < NC; c++) g[c] = 0.0;
        if (any) {
            double w[NC];
            load_w<Mdl, DIM, ORDER>(W, ld, e, w);
            double Jinv[DIM * DIM];
#pragma unroll
            for (int q = 0; q < DIM * DIM; q++) Jinv[q] = ldg(M.geo + (size_t)(GL::JINV + q) * ld + e);
#pragma unroll 1
            for (int k = 0; k < NF; k++) {
                if (M.tt[(size_t)k * ld + e] != bc) continue;
                double n[DIM], Jac, dL;
                El::face_geo(M, e, k, n, Jac, dL);
#pragma unroll 1
                for (int p = 0; p < NQF; p++) {
                    const double* phi = M.tab + TB::o_phiL + (k * NQF + p) * NB;
                    const double* dphi = M.tab + TB::o_dphiL + (k * NQF + p) * NB * DIM;
                    double WL[NE], dWL[DIM * NE], gr[DIM * NE];
#pragma unroll
                    for (int m = 0; m < NE; m++) {
                        WL[m] = 0.0;
#pragma unroll
                        for (int d = 0; d < DIM; d++) gr[d * NE + m] = 0.0;
#pragma unroll
                        for (int j = 0; j < NB; j++) {
                            WL[m] += w[m * NB + j] * ldg(phi + j);
#pragma unroll
                            for (int d = 0; d < DIM; d++) gr[d * NE + m] += w[m * NB + j] * ldg(dphi + j * DIM + d);
                        }
                    }
#pragma unroll
                    for (int m = 0; m < NE; m++)
#pragma unroll
                        for (int d = 0; d < DIM; d++) {
                            double s = 0.0;
#pragma unroll
                            for (int q = 0; q < DIM; q++) s += Jinv[q * DIM + d] * gr[q * NE + m];
                            dWL[d * NE + m] = s;
                        }
                    const double jw = Jac * ldg(M.tab + TB::o_wf + p);
                    if (kind == 0) {
                        double sv[DIM];
                        Mdl::stressVector(WL, dWL, n, sv, M.P);
#pragma unroll
                        for (int d = 0; d < DIM; d++) acc[d] -= jw * sv[d];
                    } else {
                        Dual<NE> Wd[NE];
#pragma unroll
                        for (int m = 0; m < NE; m++) {
                            Wd[m] = Dual<NE>(WL[m]);
                            Wd[m].d[m] = 1.0;
                        }
                        const Dual<NE> val = Mdl::functionalPressure(Wd, M.P) * n[kind == 1 ? 1 : 0];
                        acc[0] += jw * val.v;
                        if (grad) {
#pragma unroll
                            for (int m = 0; m < NE; m++) {
                                const double gm = jw * val.d[m];
#pragma unroll
                                for (int j = 0; j < NB; j++) g[m * NB + j] += gm * ldg(phi + j);
                            }
                        }
                    }
                }
            }
        }
        if (grad) {
#pragma unroll
            for (int c = 0; c < NC; c++) dIdW[(size_t)c * ld + e] = g[c];
        }
    }
#pragma unroll
    for (int v = 0; v < 4; v++) sh[threadIdx.x][v] = acc[v];
    __syncthreads();
    for (int s2 = kBlock / 2; s2 > 0; s2 >>= 1) {
        if ((int)threadIdx.x < s2)
#pragma unroll
            for (int v = 0; v < 4; v++) sh[threadIdx.x][v] += sh[threadIdx.x + s2][v];
        __syncthreads();
    }
    if (threadIdx.x == 0)
#pragma unroll
        for (int v = 0; v < 4; v++) part[(size_t)blockIdx.x * 4 + v] = sh[0][v];
}

// ---------------------------------------------------------------------------- launch table
inline unsigned grid_of(int n) { return (unsigned)((n + kBlock - 1) / kBlock); }

template <class Mdl, int DIM, int ORDER>
struct Launch {
    // dynamic shared memory of the face and element kernels (the element's coefficients when
    // they do not fit the static array), allowed once per kernel before its first launch
    static constexpr size_t kDyn = own_smem_bytes<Element<Mdl, DIM, ORDER>::NC>();
    template <class K>
    static void allow_dyn(K* kernel) {
        if (kDyn > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDyn);
    }
    // the attribute belongs to the current device: set once per device (the first 64 devices
    // are remembered; beyond them it is set on every call, which is harmless)
    static void prepare() {
        static std::atomic<unsigned long long> done{0};
        int dev = 0;
        cudaGetDevice(&dev);
        const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
        if (bit && (done.load(std::memory_order_acquire) & bit)) return;
        allow_dyn(k_face<Mdl, DIM, ORDER>);
        allow_dyn(k_residual<Mdl, DIM, ORDER>);
        allow_dyn(k_rk_stage<Mdl, DIM, ORDER>);
        allow_dyn(k_rhs<Mdl, DIM, ORDER>);
        constexpr size_t mf = matfree_smem_bytes<Element<Mdl, DIM, ORDER>::NC>();
        if (mf > 48 * 1024) {
            cudaFuncSetAttribute(k_matfree<Mdl, DIM, ORDER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mf);
            cudaFuncSetAttribute(k_face_tan<Mdl, DIM, ORDER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mf);
            cudaFuncSetAttribute(k_matfree_elem<Mdl, DIM, ORDER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mf);
        }
        constexpr size_t fd = fd_smem_bytes<Element<Mdl, DIM, ORDER>::NC>();
        if (fd > 48 * 1024) {
            cudaFuncSetAttribute(k_fd_base<Mdl, DIM, ORDER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fd);
            cudaFuncSetAttribute(k_fd_col<Mdl, DIM, ORDER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fd);
        }
        done.fetch_or(bit, std::memory_order_release);
    }
    static void faces(const DevMesh& M, cudaStream_t s, const double* W) {
        prepare();
        k_face<Mdl, DIM, ORDER><<<grid_of(M.F.nFaces), kBlock, kDyn, s>>>(M, W, 0, M.F.nFaces);
    }
    static void elements(const DevMesh& M, cudaStream_t s, const double* W, double* R) {
        prepare();
        k_residual<Mdl, DIM, ORDER><<<grid_of(M.nElem), kBlock, kDyn, s>>>(M, W, R, 0, M.nElem);
    }
    static void faces_range(const DevMesh& M, cudaStream_t s, const double* W, int f0, int f1) {
        prepare();
        if (f1 > f0) k_face<Mdl, DIM, ORDER><<<grid_of(f1 - f0), kBlock, kDyn, s>>>(M, W, f0, f1);
    }
    static void elements_range(const DevMesh& M, cudaStream_t s, const double* W, double* R, int e0, int e1) {
        prepare();
        if (e1 > e0) k_residual<Mdl, DIM, ORDER><<<grid_of(e1 - e0), kBlock, kDyn, s>>>(M, W, R, e0, e1);
    }
    static void residual(const DevMesh& M, cudaStream_t s, const double* W, double* R) {
        faces(M, s, W);
        elements(M, s, W, R);
    }
    static void rk_stage(const DevMesh& M, cudaStream_t s, const double* W, const double* Wo, const double* Wb, double a,
                         double b, double dt, double* Wout, double* Rsave) {
        faces(M, s, W);
        k_rk_stage<Mdl, DIM, ORDER><<<grid_of(M.nElem), kBlock, kDyn, s>>>(M, W, Wo, Wb, a, b, dt, Wout, Rsave);
    }
    // the matrix-free operator: tangent face pass (face buffer G as scratch) + element pass
    static void matfree(const DevMesh& M, cudaStream_t s, const double* W, const double* V, double a1, double* Y) {
        prepare();
        constexpr size_t sm = matfree_smem_bytes<Element<Mdl, DIM, ORDER>::NC>();
        k_face_tan<Mdl, DIM, ORDER><<<grid_of(M.F.nFaces), kBlock, sm, s>>>(M, W, V);
        k_matfree_elem<Mdl, DIM, ORDER><<<grid_of(M.nElem), kBlock, sm, s>>>(M, W, V, a1, Y);
    }
    // the element-gather form (both sides of every face), kept for comparison
    static void matfree_gather(const DevMesh& M, cudaStream_t s, const double* W, const double* V, double a1, double* Y) {
        prepare();
        k_matfree<Mdl, DIM, ORDER><<<grid_of(M.nElem), kBlock, matfree_smem_bytes<Element<Mdl, DIM, ORDER>::NC>(), s>>>(
            M, W, V, a1, Y);
    }
    static void limiter(const DevMesh& M, cudaStream_t s, const double* W, double dampTol, double penalty, const double* trun,
                        double* eps, double* cip) {
        k_limiter<Mdl, DIM, ORDER><<<grid_of(M.nElem), kBlock, 0, s>>>(M, W, dampTol, penalty, trun, eps, cip);
    }
    static void positivity(const DevMesh& M, cudaStream_t s, double* W, int* count) {
        k_positivity<Mdl, DIM, ORDER><<<grid_of(M.nElem), kBlock, 0, s>>>(M, W, count);
    }
    static void norms(const DevMesh& M, cudaStream_t s, const double* R, double* part) {
        k_norms<Mdl, DIM, ORDER><<<grid_of(M.nElem), kBlock, 0, s>>>(M, R, part);
    }
    static void dtbound(const DevMesh& M, cudaStream_t s, const double* W, double factor, double* part) {
        k_dtbound<Mdl, DIM, ORDER><<<grid_of(M.nElem), kBlock, 0, s>>>(M, W, factor, part);
    }
    static void rhs(const DevMesh& M, cudaStream_t s, const double* W, const double* Wo, const double* Wo2, double a1,
                    double a2, double a3, double* R, double* rhs, double* part) {
        faces(M, s, W);
        k_rhs<Mdl, DIM, ORDER><<<grid_of(M.nElem), kBlock, kDyn, s>>>(M, W, Wo, Wo2, a1, a2, a3, R, rhs, part);
    }
    static void fd(const DevMesh& M, cudaStream_t s, const double* W, double* K0, double* KR0, double h, double a1,
                   double* Adiag, double* Aneigh) {
        constexpr int NC = Element<Mdl, DIM, ORDER>::NC;
        prepare();
        constexpr size_t sm = fd_smem_bytes<NC>();
        k_fd_base<Mdl, DIM, ORDER><<<grid_of(M.nElem), kBlock, sm, s>>>(M, W, K0, KR0);
        long long nt = (long long)M.nElem * NC;
        k_fd_col<Mdl, DIM, ORDER><<<(unsigned)((nt + kBlock - 1) / kBlock), kBlock, sm, s>>>(M, W, K0, KR0, h, a1, Adiag, Aneigh);
    }
    static void jac_exact(const DevMesh& M, cudaStream_t s, const double* W, double a1, double* Adiag, double* Aneigh) {
        constexpr int NC = Element<Mdl, DIM, ORDER>::NC;
        long long nt = (long long)M.nElem * NC;
        k_jac_exact<Mdl, DIM, ORDER><<<(unsigned)((nt + kBlock - 1) / kBlock), kBlock, 0, s>>>(M, W, a1, Adiag, Aneigh);
    }
    static void jac_exact_factor(const DevMesh& M, cudaStream_t s, const double* W, double a1, void* F, int fp32) {
        constexpr int NC = Element<Mdl, DIM, ORDER>::NC;
        long long nt = (long long)M.nElem * NC;
        const unsigned g = (unsigned)((nt + kBlock - 1) / kBlock);
        if (fp32)
            k_jac_exact_factor<Mdl, DIM, ORDER, float><<<g, kBlock, 0, s>>>(M, W, a1, (float*)F);
        else
            k_jac_exact_factor<Mdl, DIM, ORDER, double><<<g, kBlock, 0, s>>>(M, W, a1, (double*)F);
    }
    static void norms_elem(const DevMesh& M, cudaStream_t s, const double* R, double* out) {
        k_norms_elem<Mdl, DIM, ORDER><<<grid_of(M.nElem), kBlock, 0, s>>>(M, R, out);
    }
    static void dtbound_elem(const DevMesh& M, cudaStream_t s, const double* W, double factor, double* out) {
        k_dtbound_elem<Mdl, DIM, ORDER><<<grid_of(M.nElem), kBlock, 0, s>>>(M, W, factor, out);
    }
    static void mass_geo(const DevMesh& M, cudaStream_t s, int lev, double* mass) {
        k_mass_geo<DIM, ORDER><<<grid_of(M.nElem), kBlock, 0, s>>>(M, lev, mass);
    }
    static void gcl_mass(const DevMesh& M, cudaStream_t s, double a1, double a2, double a3, double* mass) {
        k_gcl_mass<DIM, ORDER><<<grid_of(M.nElem), kBlock, 0, s>>>(M, a1, a2, a3, mass);
    }
    static void vjp(const DevMesh& M, cudaStream_t s, const double* W, const double* lam, double* g) {
        constexpr int NC = Element<Mdl, DIM, ORDER>::NC;
        long long nt = (long long)M.nElem * NC;
        k_vjp_cols<Mdl, DIM, ORDER><<<(unsigned)((nt + kBlock - 1) / kBlock), kBlock, 0, s>>>(M, W, lam, g);
    }
    static void surface(const DevMesh& M, cudaStream_t s, const double* W, int kind, int bc, double* part, double* dIdW) {
        k_surface<Mdl, DIM, ORDER><<<grid_of(M.nElem), kBlock, 0, s>>>(M, W, kind, bc, part, dIdW);
    }
    static Launchers table() {
        Launchers t;
        t.nc = Element<Mdl, DIM, ORDER>::NC;
        t.ntrun = Tab<DIM, ORDER>::NB * Tab<DIM, ORDER>::NB;
        t.residual = residual;
        t.faces = faces;
        t.elements = elements;
        t.faces_range = faces_range;
        t.elements_range = elements_range;
        t.rk_stage = rk_stage;
        t.matfree = matfree;
        t.matfree_gather = matfree_gather;
        t.limiter = limiter;
        t.positivity = positivity;
        t.norms = norms;
        t.dtbound = dtbound;
        t.rhs = rhs;
        t.fd = fd;
        t.jac_exact = jac_exact;
        t.jac_exact_factor = jac_exact_factor;
        t.vjp = vjp;
        t.mass_geo = mass_geo;
        t.norms_elem = norms_elem;
        t.dtbound_elem = dtbound_elem;
        t.gcl_mass = gcl_mass;
        t.surface = surface;
        return t;
    }
};

}  // namespace fp
