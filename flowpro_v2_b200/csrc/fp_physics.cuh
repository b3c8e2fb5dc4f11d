// Device flux functions of the bundled FlowPro models, templated on the scalar
// type T (double, or Dual<N> for tangents) and on the dimension.
//
// They restate the Java plugin methods line by line, including the reference's
// in-place limiting of the density argument (every flux call does
// W[0] = limiteRho(W[0]), NavierStokes.java:196, 218, 319, ...): a state array
// passed to these functions is modified exactly as the Java array is.
//
// Models:
//   NS<DIM, VISC>   NavierStokes.java (+ Aerodynamics.java), Euler when VISC == false
//   SA<DIM>         SpalartAllmaras.java
//   Scalar<DIM>     TestScalarEquation.java (the reference tests' manufactured solution)
#pragma once
#include "fp_common.cuh"

namespace fp {

constexpr int BC_WALL = -1, BC_INLET = -2, BC_OUTLET = -3, BC_INVISCID_WALL = -4;
constexpr double RHO_TOL = 1e-2;        // Aerodynamics.java:21
constexpr double ADMISSIBLE_TOL = 1e-10; // Aerodynamics.java:340

// Aerodynamics.limiteRho, Aerodynamics.java:359-365
template <class T>
FP_HD T limiteRho(const T& rho) {
    if (val(rho) < RHO_TOL) return RHO_TOL * dexp((rho - RHO_TOL) / RHO_TOL);
    return rho;
}

// ============================================================================ compressible flow
// Shared by NavierStokes and SpalartAllmaras (the SA state carries rho*nu~ last).
template <int DIM, int NEQ, bool VISC, bool SA_MODEL>
struct Aero {
    static constexpr int NE = NEQ;
    static constexpr bool kViscous = VISC;
    static constexpr bool kSource = SA_MODEL;
    static constexpr bool kConvective = true;
    static constexpr double P_TOL = SA_MODEL ? 1e-1 : 1e-2;  // NavierStokes.java:15, SpalartAllmaras.java:12

    // pressure(), NavierStokes.java:23-37 / SpalartAllmaras.java:63-75
    template <class T>
    static FP_HD T pressure(T* W, const fp_model_params& P) {
        W[0] = limiteRho(W[0]);
        T m2 = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) m2 += W[d + 1] * W[d + 1];
        T p = (P.kappa - 1) * (W[DIM + 1] - m2 / (2.0 * W[0]));
        if (val(p) < P_TOL) p = P_TOL * dexp((p - P_TOL) / P_TOL);
        return p;
    }

    // Aerodynamics.maxEigenvalue, Aerodynamics.java:322-337
    template <class T>
    static FP_HD T maxEigenvalue(T* W, const double* u, const fp_model_params& P) {
        W[0] = limiteRho(W[0]);
        T p = pressure(W, P);
        T a = dsqrt(P.kappa * p / W[0]);
        T v = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            T vRel = W[d + 1] / W[0] - u[d];
            v += vRel * vRel;
        }
        v = dsqrt(v);
        return v + a;
    }

    // convectiveFlux, NavierStokes.java:194-214 / SpalartAllmaras.java:174-195
    template <class T>
    static FP_HD void convectiveFlux(T* W, const double* n, T* f, const fp_model_params& P) {
        W[0] = limiteRho(W[0]);
        T V = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) V += W[d + 1] * n[d];
        V /= W[0];
        T p = pressure(W, P);
        f[0] = W[0] * V;
#pragma unroll
        for (int d = 0; d < DIM; ++d) f[d + 1] = W[d + 1] * V + p * n[d];
        f[DIM + 1] = (W[DIM + 1] + p) * V;
        if (SA_MODEL) f[DIM + 2] = W[DIM + 2] * V;
    }

    // convectiveFlux along coordinate axis `ax` (unit normal e_ax): the terms with a
    // zero normal component vanish exactly, so this equals convectiveFlux(W, e_ax).
    template <class T>
    static FP_HD void convectiveFluxAxis(T* W, int ax, T* f, const fp_model_params& P) {
        W[0] = limiteRho(W[0]);
        T V = W[ax + 1] / W[0];
        T p = pressure(W, P);
        f[0] = W[0] * V;
#pragma unroll
        for (int d = 0; d < DIM; ++d) f[d + 1] = (d == ax) ? W[d + 1] * V + p : W[d + 1] * V;
        f[DIM + 1] = (W[DIM + 1] + p) * V;
        if (SA_MODEL) f[DIM + 2] = W[DIM + 2] * V;
    }

    // convectiveFluxAxis for every axis at once, f[ax * NE + m], with one reciprocal of the
    // density.  Only valid when W[0] >= RHO_TOL (no limiting), where it gives the per-axis
    // values up to rounding.
    template <class T>
    static FP_HD void convectiveFluxAll(T* W, T* f, const fp_model_params& P) {
        const T r = 1.0 / W[0];
        T m2 = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) m2 += W[d + 1] * W[d + 1];
        T p = (P.kappa - 1) * (W[DIM + 1] - 0.5 * m2 * r);
        if (val(p) < P_TOL) p = P_TOL * dexp((p - P_TOL) / P_TOL);
#pragma unroll
        for (int ax = 0; ax < DIM; ++ax) {
            T* fa = f + ax * NE;
            T V = W[ax + 1] * r;
            fa[0] = W[ax + 1];
#pragma unroll
            for (int d = 0; d < DIM; ++d) fa[d + 1] = (d == ax) ? W[d + 1] * V + p : W[d + 1] * V;
            fa[DIM + 1] = (W[DIM + 1] + p) * V;
            if (SA_MODEL) fa[DIM + 2] = W[DIM + 2] * V;
        }
    }

    // van Leer splitting, NavierStokes.java:407-465
    template <class T>
    static FP_HD void fsplit(const T* W, const T& p, const double* n, T* f, bool plus, const fp_model_params& P) {
        double kapa = P.kappa;
        T vel[DIM];
        T Vn = 0.0, q2 = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            vel[d] = W[d + 1] / W[0];
            Vn += vel[d] * n[d];
            q2 += vel[d] * vel[d];
        }
        T a = dsqrt(kapa * p / W[0]);
        T M = Vn / a;
#pragma unroll
        for (int j = 0; j < NE; j++) f[j] = 0.0;
        if (dfabs(val(M)) < 1) {
            if (plus) {
                T fm = W[0] * a * ((M + 1.0) * (M + 1.0)) / 4.0;
                f[0] = fm;
#pragma unroll
                for (int d = 0; d < DIM; ++d) f[d + 1] = fm * (vel[d] + (-Vn + 2.0 * a) / kapa * n[d]);
                f[DIM + 1] = fm * ((q2 - Vn * Vn) / 2.0 + (((kapa - 1) * Vn + 2.0 * a)) * (((kapa - 1) * Vn + 2.0 * a)) / (2 * (kapa * kapa - 1)));
            } else {
                T fm = -W[0] * a * ((M - 1.0) * (M - 1.0)) / 4.0;
                f[0] = fm;
#pragma unroll
                for (int d = 0; d < DIM; ++d) f[d + 1] = fm * (vel[d] + (-Vn - 2.0 * a) / kapa * n[d]);
                f[DIM + 1] = fm * ((q2 - Vn * Vn) / 2.0 + (((kapa - 1) * Vn - 2.0 * a) * ((kapa - 1) * Vn - 2.0 * a)) / (2 * (kapa * kapa - 1)));
            }
        } else if ((plus && val(M) >= 1) || (!plus && val(M) <= -1)) {
            f[0] = W[0] * Vn;
#pragma unroll
            for (int d = 0; d < DIM; ++d) f[d + 1] = W[d + 1] * Vn + p * n[d];
            f[DIM + 1] = (W[DIM + 1] + p) * Vn;
        }
    }

    // numericalConvectiveFlux, NavierStokes.java:141-192 / SpalartAllmaras.java:130-172
    template <class T>
    static FP_HD void numericalConvectiveFlux(T* WL, T* WR, const double* n, int TT, const double* u, T* f,
                                              const fp_model_params& P) {
        WL[0] = limiteRho(WL[0]);
        WR[0] = limiteRho(WR[0]);
        if (TT == BC_WALL || TT == BC_INVISCID_WALL) {
            // NavierStokes uses pressure(WL), SpalartAllmaras pressure(WR)
            T p = SA_MODEL ? pressure(WR, P) : pressure(WL, P);
            f[0] = 0.0;
            double V = 0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                f[d + 1] = p * n[d];
                V += u[d] * n[d];
            }
            f[DIM + 1] = p * V;
            if (SA_MODEL) f[DIM + 2] = 0.0;
#pragma unroll
            for (int j = 0; j < NE; j++) f[j] += V * WR[j];
        } else if (TT == BC_INLET || TT == BC_OUTLET) {
            convectiveFlux(WR, n, f, P);
        } else if (P.numerical_flux == 1 && !SA_MODEL) {
            T pL = pressure(WL, P);
            T fp[NE];
            fsplit(WL, pL, n, fp, true, P);
            T pR = pressure(WR, P);
            T fm[NE];
            fsplit(WR, pR, n, fm, false, P);
#pragma unroll
            for (int j = 0; j < NE; j++) f[j] = fp[j] + fm[j];
        } else {
            T fL[NE], fR[NE];
            convectiveFlux(WL, n, fL, P);
            convectiveFlux(WR, n, fR, P);
            T lL = maxEigenvalue(WL, u, P);
            T lR = maxEigenvalue(WR, u, P);
            T lam = dmax(lL, lR);
#pragma unroll
            for (int j = 0; j < NE; j++) f[j] = (fL[j] + fR[j] - lam * (WR[j] - WL[j])) / 2.0;
        }
    }

    // boundaryValue, NavierStokes.java:216-315 / SpalartAllmaras.java:200-292
    template <class T>
    static FP_HD void boundaryValue(T* WL, const double* n, int TT, const double* u, const double* X, T* WR,
                                    const fp_model_params& P, double p_out) {
        (void)X;
        WL[0] = limiteRho(WL[0]);
        double kapa = P.kappa;
#pragma unroll
        for (int j = 0; j < NE; j++) WR[j] = 0.0;
        T p = pressure(WL, P);
        if (TT == BC_WALL && (VISC || SA_MODEL)) {
            double a2 = 0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) a2 += u[d] * u[d];
            WR[0] = WL[0];
#pragma unroll
            for (int d = 0; d < DIM; ++d) WR[d + 1] = WR[0] * u[d];
            WR[DIM + 1] = p / (kapa - 1) + WR[0] * a2 / 2.0;
            if (SA_MODEL) WR[DIM + 2] = 0.0;
        } else if (TT == BC_WALL || TT == BC_INVISCID_WALL) {
#pragma unroll
            for (int j = 0; j < NE; j++) WR[j] = WL[j];
            T nu = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) nu += WL[d + 1] * n[d];
            // NavierStokes subtracts the normal momentum, SpalartAllmaras adds it
            // (SpalartAllmaras.java:228: WR[d + 1] = WL[d + 1] + n[d] * nu)
#pragma unroll
            for (int d = 0; d < DIM; ++d) WR[d + 1] = SA_MODEL ? WL[d + 1] + n[d] * nu : WL[d + 1] - n[d] * nu;
        } else if (TT == BC_INLET) {
            if (!P.inlet_supersonic) {
                T mach;
                if (val(p) > P.p_in0)
                    mach = 0.0;
                else
                    mach = dsqrt((2 / (kapa - 1)) * (-1.0 + dpow(P.p_in0 / p, (kapa - 1) / kapa)));
                T rhoIn = P.rho_in0 * dpow((1.0 + ((kapa - 1) / 2) * mach * mach), 1 / (1 - kapa));
                T inletVelocity = mach * dsqrt((kapa * p) / rhoIn);
                T E = p / (kapa - 1) + 0.5 * rhoIn * inletVelocity * inletVelocity;
                WR[0] = rhoIn;
                if (!P.has_attack_angle) {
#pragma unroll
                    for (int d = 0; d < DIM; ++d) WR[d + 1] = -rhoIn * inletVelocity * n[d];
                } else {
                    double dir[3];
                    if (DIM == 2) {
                        dir[0] = cos(P.attack_angle[0]);
                        dir[1] = sin(P.attack_angle[0]);
                    } else {
                        dir[0] = cos(P.attack_angle[0]) * cos(P.attack_angle[1]);
                        dir[1] = sin(P.attack_angle[0]) * cos(P.attack_angle[1]);
                        dir[2] = sin(P.attack_angle[1]);
                    }
#pragma unroll
                    for (int d = 0; d < DIM; ++d) WR[d + 1] = rhoIn * inletVelocity * dir[d];
                }
                WR[DIM + 1] = E;
                if (SA_MODEL) WR[DIM + 2] = rhoIn * P.vt_in;
            } else {
#pragma unroll
                for (int j = 0; j < NE; j++) WR[j] = P.w_in[j];
            }
        } else if (TT == BC_OUTLET) {
            T rhoOut = WL[0];
            T a2 = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) a2 += WL[d + 1] * WL[d + 1];
            a2 /= rhoOut * rhoOut;
            T pp = pressure(WL, P);
            T a = dsqrt(kapa * pp / WL[0]);
            T mach = dsqrt(a2) / a;
            if (val(mach) < 1) {
                WR[0] = rhoOut;
#pragma unroll
                for (int d = 0; d < DIM; ++d) WR[d + 1] = rhoOut * WL[d + 1] / WL[0];
                WR[DIM + 1] = p_out / (kapa - 1) + rhoOut * a2 / 2.0;
                if (SA_MODEL) WR[DIM + 2] = WL[DIM + 2];
            } else {
#pragma unroll
                for (int j = 0; j < NE; j++) WR[j] = WL[j];
            }
        }
    }

    // velocity gradient, stress tensor and d(p/rho)/dx shared by diffusiveFlux / sourceTerm
    // (NavierStokes.java:320-360, SpalartAllmaras.java:296-340)
    template <class T>
    static FP_HD void viscousTerms(T* W, const T& rho, const T* dW, T* vel, T& vel2, T* vJ, T* stress,
                                   T* pOverRhoDer, const fp_model_params& P) {
        vel2 = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            vel[d] = W[d + 1] / rho;
            vel2 += vel[d] * vel[d];
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d)
#pragma unroll
            for (int f = 0; f < DIM; ++f) vJ[DIM * d + f] = (dW[f * NE + d + 1] - dW[f * NE] * vel[d]) / rho;
        T p = pressure(W, P);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            T temp = 0.0;
#pragma unroll
            for (int f = 0; f < DIM; ++f) temp += vel[f] * vJ[DIM * f + d];
            T pDer = (P.kappa - 1) * (dW[d * NE + DIM + 1] - dW[d * NE] * vel2 / 2.0 - rho * temp);
            pOverRhoDer[d] = (rho * pDer - p * dW[d * NE]) / (rho * rho);
        }
        T trace = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            trace += vJ[DIM * d + d];
#pragma unroll
            for (int f = 0; f < DIM; ++f) stress[DIM * d + f] = vJ[DIM * d + f] + vJ[DIM * f + d];
        }
        const double lam = -2. / 3;
#pragma unroll
        for (int d = 0; d < DIM; ++d) stress[DIM * d + d] += lam * trace;
    }

    // diffusiveFlux, NavierStokes.java:317-374 / SpalartAllmaras.java:295-362.
    // n == nullptr: unit normal e_ax (volume fluxes, same values as Java's nor[d] = 1).
    template <class T>
    static FP_HD void diffusiveFlux(T* W, const T* dW, const double* n, int ax, T* flux, const fp_model_params& P) {
        W[0] = limiteRho(W[0]);
        const T rho = W[0];  // captured before pressure() limits W[0] again (NavierStokes.java:319-320)
        T vel[DIM], vJ[DIM * DIM], stress[DIM * DIM], pOverRhoDer[DIM], vel2;
        viscousTerms(W, rho, dW, vel, vel2, vJ, stress, pOverRhoDer, P);
        double kapa = P.kappa, Re = P.Re;
        T mut = 0.0, vt = 0.0;
        T vtDer[DIM];
        if (SA_MODEL) {
            vt = dmax(T(0.0), W[DIM + 2] / rho);
#pragma unroll
            for (int d = 0; d < DIM; ++d) vtDer[d] = 1.0 / rho * (dW[d * NE + DIM + 2] - dW[d * NE] * vt);
            T xi = rho * vt;
            T fv1 = xi * xi * xi / (xi * xi * xi + P.cv1 * P.cv1 * P.cv1);
            mut = rho * vt * fv1;
        }
        T constant;
        if (SA_MODEL)
            constant = kapa / (kapa - 1) * (1 / P.Pr + mut / P.prt);
        else
            constant = T(kapa / (kapa - 1) / P.Pr);
#pragma unroll
        for (int j = 0; j < NE; j++) flux[j] = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            if (n == nullptr && d != ax) continue;
            double nd = n == nullptr ? 1.0 : n[d];
            T tmp = 0.0;
#pragma unroll
            for (int f = 0; f < DIM; ++f) {
                if (SA_MODEL) {
                    flux[f + 1] += (1.0 + mut) * stress[DIM * d + f] * nd / Re;
                    tmp += vel[f] * (1.0 + mut) * stress[DIM * d + f];
                } else {
                    flux[f + 1] += stress[DIM * d + f] * nd / Re;
                    tmp += vel[f] * stress[DIM * d + f];
                }
            }
            flux[DIM + 1] += (tmp + constant * pOverRhoDer[d]) * nd / Re;
            if (SA_MODEL) flux[DIM + 2] += 1.0 / (Re * P.sigma) * (1.0 + rho * vt) * vtDer[d] * nd;
        }
    }

    // diffusiveFlux along every axis at once (fv[ax * NE + m]) with one reciprocal of the
    // density and of Re.  Only valid when W[0] >= RHO_TOL (no limiting); then each axis equals
    // diffusiveFlux(..., ax) up to rounding.
    template <class T>
    static FP_HD void diffusiveFluxAll(T* W, const T* dW, T* fv, const fp_model_params& P) {
        const T rho = W[0];
        const T r = 1.0 / rho;
        const double invRe = 1.0 / P.Re;
        T vel[DIM], vJ[DIM * DIM], stress[DIM * DIM], pOverRhoDer[DIM], vel2 = 0.0, m2 = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            vel[d] = W[d + 1] * r;
            vel2 += vel[d] * vel[d];
            m2 += W[d + 1] * W[d + 1];
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d)
#pragma unroll
            for (int f = 0; f < DIM; ++f) vJ[DIM * d + f] = (dW[f * NE + d + 1] - dW[f * NE] * vel[d]) * r;
        T p = (P.kappa - 1) * (W[DIM + 1] - 0.5 * m2 * r);
        if (val(p) < P_TOL) p = P_TOL * dexp((p - P_TOL) / P_TOL);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            T temp = 0.0;
#pragma unroll
            for (int f = 0; f < DIM; ++f) temp += vel[f] * vJ[DIM * f + d];
            const T pDer = (P.kappa - 1) * (dW[d * NE + DIM + 1] - dW[d * NE] * vel2 / 2.0 - rho * temp);
            pOverRhoDer[d] = (rho * pDer - p * dW[d * NE]) * (r * r);
        }
        T trace = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            trace += vJ[DIM * d + d];
#pragma unroll
            for (int f = 0; f < DIM; ++f) stress[DIM * d + f] = vJ[DIM * d + f] + vJ[DIM * f + d];
        }
        const double lam = -2. / 3;
#pragma unroll
        for (int d = 0; d < DIM; ++d) stress[DIM * d + d] += lam * trace;
        double kapa = P.kappa;
        T mut = 0.0, vt = 0.0;
        T vtDer[DIM];
        if (SA_MODEL) {
            vt = dmax(T(0.0), W[DIM + 2] * r);
#pragma unroll
            for (int d = 0; d < DIM; ++d) vtDer[d] = r * (dW[d * NE + DIM + 2] - dW[d * NE] * vt);
            T xi = rho * vt;
            T fv1 = xi * xi * xi / (xi * xi * xi + P.cv1 * P.cv1 * P.cv1);
            mut = rho * vt * fv1;
        }
        T constant;
        if (SA_MODEL)
            constant = kapa / (kapa - 1) * (1 / P.Pr + mut / P.prt);
        else
            constant = T(kapa / (kapa - 1) / P.Pr);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            T* fa = fv + d * NE;
            fa[0] = 0.0;
            T tmp = 0.0;
#pragma unroll
            for (int f = 0; f < DIM; ++f) {
                if (SA_MODEL) {
                    fa[f + 1] = (1.0 + mut) * stress[DIM * d + f] * invRe;
                    tmp += vel[f] * (1.0 + mut) * stress[DIM * d + f];
                } else {
                    fa[f + 1] = stress[DIM * d + f] * invRe;
                    tmp += vel[f] * stress[DIM * d + f];
                }
            }
            fa[DIM + 1] = (tmp + constant * pOverRhoDer[d]) * invRe;
            if (SA_MODEL) fa[DIM + 2] = (1.0 + rho * vt) * vtDer[d] * (invRe / P.sigma);
        }
    }

    // stressVector (force density on a surface with unit normal n): NavierStokes.java:39-83 and
    // SpalartAllmaras.java:510-553 (viscous: -p n + tau n / Re, rho taken before pressure()
    // limits W[0]), Aerodynamics.java:108-117 (inviscid: -p n)
    template <class T>
    static FP_HD void stressVector(T* W, const T* dW, const double* n, T* sv, const fp_model_params& P) {
        if (VISC) {
            const T rho = W[0];
            T vel[DIM], vJ[DIM * DIM], stress[DIM * DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) vel[d] = W[d + 1] / rho;
#pragma unroll
            for (int d = 0; d < DIM; ++d)
#pragma unroll
                for (int f = 0; f < DIM; ++f) vJ[DIM * d + f] = (dW[f * NE + d + 1] - dW[f * NE] * vel[d]) / rho;
            T trace = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                trace += vJ[DIM * d + d];
#pragma unroll
                for (int f = 0; f < DIM; ++f) stress[DIM * d + f] = vJ[DIM * d + f] + vJ[DIM * f + d];
            }
            const double lam = -2. / 3;
#pragma unroll
            for (int d = 0; d < DIM; ++d) stress[DIM * d + d] += lam * trace;
            T p = pressure(W, P);
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                sv[d] = 0.0;
                sv[d] -= p * n[d];
#pragma unroll
                for (int f = 0; f < DIM; ++f) sv[d] += 1 / P.Re * stress[DIM * d + f] * n[f];
            }
        } else {
            T p = pressure(W, P);
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                sv[d] = 0.0;
                sv[d] -= p * n[d];
            }
        }
    }

    // pressure of the lift / drag functionals, LiftCoefficient.java:40-49 (no clipping, dim 2)
    template <class T>
    static FP_HD T functionalPressure(const T* W, const fp_model_params& P) {
        T momentum2 = 0.0;
#pragma unroll
        for (int d = 0; d < 2; ++d) momentum2 += W[d + 1] * W[d + 1];
        return (P.kappa - 1) * (W[2 + 1] - momentum2 / (2 * W[0]));
    }

    // numericalDiffusiveFlux, NavierStokes.java:376-395 (adiabatic wall: only the work
    // of the viscous stress of a moving wall)
    template <class T>
    static FP_HD void numericalDiffusiveFlux(T* Wc, const T* dWc, const double* n, int TT, const double* u, T* flux,
                                             const fp_model_params& P) {
        Wc[0] = limiteRho(Wc[0]);
        diffusiveFlux(Wc, dWc, n, 0, flux, P);
        if (TT < 0) {
            if (TT == BC_WALL) {
                T work = 0.0;
#pragma unroll
                for (int d = 0; d < DIM; ++d) work += u[d] * flux[d + 1];
                flux[DIM + 1] = work;
            } else {
#pragma unroll
                for (int j = 0; j < NE; j++) flux[j] = 0.0;
            }
        }
    }

    // ---- interior-face fast path (Lax-Friedrichs, DDG) ---------------------------------
    // Valid when both densities are >= RHO_TOL: limiteRho is then the identity, so the
    // reference's repeated in-place limiting changes nothing and the same quantities can be
    // formed with one reciprocal of the density per state (the reference divides at every
    // use).  The results differ from the per-use divisions only by rounding.
    static constexpr bool kFastFace = true;

    // pressure from the reciprocal density (pressure() without the limiting)
    template <class T>
    static FP_HD T pressureRcp(const T* W, const T& r, const fp_model_params& P) {
        T m2 = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) m2 += W[d + 1] * W[d + 1];
        T p = (P.kappa - 1) * (W[DIM + 1] - 0.5 * m2 * r);
        if (val(p) < P_TOL) p = P_TOL * dexp((p - P_TOL) / P_TOL);
        return p;
    }

    // numericalConvectiveFlux of an interior face, Lax-Friedrichs branch
    template <class T>
    static FP_HD void laxFriedrichsFast(const T* WL, const T* WR, const double* n, const double* u, T* f,
                                        const fp_model_params& P) {
        T fL[NE], fR[NE];
        T lam[2];
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const T* W = s == 0 ? WL : WR;
            T* fs = s == 0 ? fL : fR;
            const T r = 1.0 / W[0];
            const T p = pressureRcp(W, r, P);
            T Vn = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) Vn += W[d + 1] * n[d];
            Vn = Vn * r;
            fs[0] = W[0] * Vn;
#pragma unroll
            for (int d = 0; d < DIM; ++d) fs[d + 1] = W[d + 1] * Vn + p * n[d];
            fs[DIM + 1] = (W[DIM + 1] + p) * Vn;
            if (SA_MODEL) fs[DIM + 2] = W[DIM + 2] * Vn;
            T v2 = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                const T vRel = W[d + 1] * r - u[d];
                v2 += vRel * vRel;
            }
            lam[s] = dsqrt(v2) + dsqrt(P.kappa * p * r);
        }
        const T l = dmax(lam[0], lam[1]);
#pragma unroll
        for (int j = 0; j < NE; j++) f[j] = (fL[j] + fR[j] - l * (WR[j] - WL[j])) / 2.0;
    }

    // diffusiveFlux(W, dW, n) of an interior face
    template <class T>
    static FP_HD void diffusiveFluxFast(const T* W, const T* dW, const double* n, T* flux, const fp_model_params& P) {
        const T rho = W[0];
        const T r = 1.0 / rho;
        const double invRe = 1.0 / P.Re;
        T vel[DIM], vJ[DIM * DIM], stress[DIM * DIM], pOverRhoDer[DIM], vel2 = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            vel[d] = W[d + 1] * r;
            vel2 += vel[d] * vel[d];
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d)
#pragma unroll
            for (int f = 0; f < DIM; ++f) vJ[DIM * d + f] = (dW[f * NE + d + 1] - dW[f * NE] * vel[d]) * r;
        const T p = pressureRcp(W, r, P);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            T temp = 0.0;
#pragma unroll
            for (int f = 0; f < DIM; ++f) temp += vel[f] * vJ[DIM * f + d];
            const T pDer = (P.kappa - 1) * (dW[d * NE + DIM + 1] - dW[d * NE] * vel2 / 2.0 - rho * temp);
            pOverRhoDer[d] = (rho * pDer - p * dW[d * NE]) * (r * r);
        }
        T trace = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            trace += vJ[DIM * d + d];
#pragma unroll
            for (int f = 0; f < DIM; ++f) stress[DIM * d + f] = vJ[DIM * d + f] + vJ[DIM * f + d];
        }
        const double lam = -2. / 3;
#pragma unroll
        for (int d = 0; d < DIM; ++d) stress[DIM * d + d] += lam * trace;
        const double kapa = P.kappa;
        T mut = 0.0, vt = 0.0;
        T vtDer[DIM];
        if (SA_MODEL) {
            vt = dmax(T(0.0), W[DIM + 2] * r);
#pragma unroll
            for (int d = 0; d < DIM; ++d) vtDer[d] = r * (dW[d * NE + DIM + 2] - dW[d * NE] * vt);
            T xi = rho * vt;
            T fv1 = xi * xi * xi / (xi * xi * xi + P.cv1 * P.cv1 * P.cv1);
            mut = rho * vt * fv1;
        }
        T constant;
        if (SA_MODEL)
            constant = kapa / (kapa - 1) * (1 / P.Pr + mut / P.prt);
        else
            constant = T(kapa / (kapa - 1) / P.Pr);
#pragma unroll
        for (int j = 0; j < NE; j++) flux[j] = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const double nd = n[d] * invRe;
            T tmp = 0.0;
#pragma unroll
            for (int f = 0; f < DIM; ++f) {
                if (SA_MODEL) {
                    flux[f + 1] += (1.0 + mut) * stress[DIM * d + f] * nd;
                    tmp += vel[f] * (1.0 + mut) * stress[DIM * d + f];
                } else {
                    flux[f + 1] += stress[DIM * d + f] * nd;
                    tmp += vel[f] * stress[DIM * d + f];
                }
            }
            flux[DIM + 1] += (tmp + constant * pOverRhoDer[d]) * nd;
            if (SA_MODEL) flux[DIM + 2] += (1.0 + rho * vt) * vtDer[d] * (nd / P.sigma);
        }
    }

    // SpalartAllmaras.sourceTerm, SpalartAllmaras.java:391-451
    template <class T>
    static FP_HD void sourceTerm(T* W, const T* dW, double D, const double* X, T* s, const fp_model_params& P) {
        (void)X;
#pragma unroll
        for (int j = 0; j < NE; j++) s[j] = 0.0;
        if (!SA_MODEL) return;
        W[0] = limiteRho(W[0]);
        const T rho = W[0];
        T vel[DIM], vJ[DIM * DIM], stress[DIM * DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) vel[d] = W[d + 1] / rho;
#pragma unroll
        for (int d = 0; d < DIM; ++d)
#pragma unroll
            for (int f = 0; f < DIM; ++f) vJ[DIM * d + f] = (dW[f * NE + d + 1] - dW[f * NE] * vel[d]) / rho;
        (void)stress;
        T vt = dmax(T(0.0), W[DIM + 2] / rho);
        T vtDerMag = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            T vtDer = 1.0 / rho * (dW[d * NE + DIM + 2] - dW[d * NE] * vt);
            vtDerMag += vtDer * vtDer;
        }
        if (val(vt) < 0) vt = 0.0;
        double Re = P.Re, ka = P.ka;
        T xi = rho * vt;
        const double ft2 = 0;
        T fv1 = xi * xi * xi / (xi * xi * xi + P.cv1 * P.cv1 * P.cv1);
        T fv2 = 1.0 - xi / (1.0 + xi * fv1);
        T Om;
        if (DIM == 2) {
            Om = dfabs(vJ[1] - vJ[2]);
        } else {
            T a = vJ[0 * DIM + 1] - vJ[1 * DIM + 0];
            T b = vJ[0 * DIM + 2] - vJ[2 * DIM + 0];
            T c = vJ[2 * DIM + 1] - vJ[1 * DIM + 2];
            Om = dsqrt(a * a + b * b + c * c);
        }
        T S = Om + 1 / Re * vt / (ka * ka * D * D) * fv2;
        T rt = dmin(vt / (Re * S * ka * ka * D * D), T(10.0));
        T g = rt + P.cw2 * (dpow(rt, 6.0) - rt);
        double cw36 = pow(P.cw3, 6.0);
        T fw = g * dpow((1 + cw36) / (dpow(g, 6.0) + cw36), 1.0 / 6);
        T d = 1 / Re * rho * P.cb2 * vtDerMag + P.cb1 * (1 - ft2) * rho * S * vt -
              1 / Re * (P.cw1 * fw - P.cb1 / (ka * ka) * ft2) / rho * (rho * vt / D) * (rho * vt / D);
        if (val(d) < -100) d = -100.0;
        s[DIM + 2] = d;
    }

    static FP_HD bool isIPFace(int TT) { return TT == BC_WALL; }

    // Aerodynamics.isAdmissible, Aerodynamics.java:347-357
    static FP_HD bool isAdmissible(const double* W) {
        if (!(W[0] > ADMISSIBLE_TOL)) return false;
        double m2 = 0;
        for (int d = 0; d < DIM; ++d) m2 += W[d + 1] * W[d + 1];
        return W[DIM + 1] - m2 / (2 * W[0]) > ADMISSIBLE_TOL;
    }
};

template <int DIM, bool VISC>
using NS = Aero<DIM, DIM + 2, VISC, false>;
template <int DIM>
using SA = Aero<DIM, DIM + 3, true, true>;

// ============================================================================ isentropic Euler
// AdiabaticEulers.java (ModuleProjects/Equations/Aerodynamics): nEqs = dim + 1 (no energy
// equation), p = rho^kappa with the smooth clip at P_TOL = 0.1, Lax-Friedrichs interior flux,
// slip walls by the reference's reflected state.  Inviscid, no source.
template <int DIM>
struct Adiabatic {
    static constexpr int NE = DIM + 1;
    static constexpr bool kFastFace = false;
    static constexpr bool kViscous = false;
    static constexpr bool kSource = false;
    static constexpr bool kConvective = true;
    static constexpr double P_TOL = 1e-1;  // AdiabaticEulers.java:10

    // AdiabaticEulers.pressure, AdiabaticEulers.java:24-33
    template <class T>
    static FP_HD T pressure(T* W, const fp_model_params& P) {
        W[0] = limiteRho(W[0]);
        T p = dpow(W[0], P.kappa);
        if (val(p) < P_TOL) p = P_TOL * dexp((p - P_TOL) / P_TOL);
        return p;
    }

    // Aerodynamics.maxEigenvalue (Aerodynamics.java:322-337) with this model's pressure
    template <class T>
    static FP_HD T maxEigenvalue(T* W, const double* u, const fp_model_params& P) {
        W[0] = limiteRho(W[0]);
        T p = pressure(W, P);
        T a = dsqrt(P.kappa * p / W[0]);
        T v = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            T vRel = W[d + 1] / W[0] - u[d];
            v += vRel * vRel;
        }
        v = dsqrt(v);
        return v + a;
    }

    // AdiabaticEulers.convectiveFlux, AdiabaticEulers.java:178-195
    template <class T>
    static FP_HD void convectiveFlux(T* W, const double* n, T* f, const fp_model_params& P) {
        W[0] = limiteRho(W[0]);
        T V = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) V += W[d + 1] * n[d];
        V /= W[0];
        T p = pressure(W, P);
        f[0] = W[0] * V;
#pragma unroll
        for (int d = 0; d < DIM; ++d) f[d + 1] = W[d + 1] * V + p * n[d];
    }
    template <class T>
    static FP_HD void convectiveFluxAxis(T* W, int ax, T* f, const fp_model_params& P) {
        W[0] = limiteRho(W[0]);
        T V = W[ax + 1] / W[0];
        T p = pressure(W, P);
        f[0] = W[0] * V;
#pragma unroll
        for (int d = 0; d < DIM; ++d) f[d + 1] = (d == ax) ? W[d + 1] * V + p : W[d + 1] * V;
    }
    // all axes at once; only valid when W[0] >= RHO_TOL (no limiting)
    template <class T>
    static FP_HD void convectiveFluxAll(T* W, T* f, const fp_model_params& P) {
        T p = pressure(W, P);
#pragma unroll
        for (int ax = 0; ax < DIM; ++ax) {
            T* fa = f + ax * NE;
            T V = W[ax + 1] / W[0];
            fa[0] = W[0] * V;
#pragma unroll
            for (int d = 0; d < DIM; ++d) fa[d + 1] = (d == ax) ? W[d + 1] * V + p : W[d + 1] * V;
        }
    }

    // AdiabaticEulers.numericalConvectiveFlux, AdiabaticEulers.java:136-176
    template <class T>
    static FP_HD void numericalConvectiveFlux(T* WL, T* WR, const double* n, int TT, const double* u, T* f,
                                              const fp_model_params& P) {
        WL[0] = limiteRho(WL[0]);
        WR[0] = limiteRho(WR[0]);
        if (TT == BC_WALL || TT == BC_INVISCID_WALL) {
            T p = pressure(WR, P);
            f[0] = 0.0;
            double V = 0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                f[d + 1] = p * n[d];
                V += u[d] * n[d];
            }
#pragma unroll
            for (int j = 0; j < NE; j++) f[j] += V * WR[j];
        } else if (TT == BC_INLET || TT == BC_OUTLET) {
            convectiveFlux(WR, n, f, P);
        } else {
            T fL[NE], fR[NE];
            convectiveFlux(WL, n, fL, P);
            convectiveFlux(WR, n, fR, P);
            T lL = maxEigenvalue(WL, u, P);
            T lR = maxEigenvalue(WR, u, P);
            T lam = dmax(lL, lR);
#pragma unroll
            for (int j = 0; j < NE; j++) f[j] = (fL[j] + fR[j] - lam * (WR[j] - WL[j])) / 2.0;
        }
    }

    // AdiabaticEulers.boundaryValue, AdiabaticEulers.java:35-95
    template <class T>
    static FP_HD void boundaryValue(T* WL, const double* n, int TT, const double*, const double*, T* WR,
                                    const fp_model_params& P, double p_out) {
        WL[0] = limiteRho(WL[0]);
#pragma unroll
        for (int j = 0; j < NE; j++) WR[j] = 0.0;
        const double kapa = P.kappa;
        if (TT == BC_WALL || TT == BC_INVISCID_WALL) {
#pragma unroll
            for (int j = 0; j < NE; j++) WR[j] = WL[j];
            T nu = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) nu += WL[d + 1] * n[d];
#pragma unroll
            for (int d = 0; d < DIM; ++d) WR[d + 1] = WL[d + 1] + n[d] * nu;
        } else if (TT == BC_INLET) {
            // subsonic inlet (a supersonic inlet is rejected at set-up)
            T p = pressure(WL, P);
            T mach;
            if (val(p) > P.p_in0)
                mach = 0.0;
            else
                mach = dsqrt((2 / (kapa - 1)) * (-1.0 + dpow(P.p_in0 / p, (kapa - 1) / kapa)));
            T rhoIn = P.rho_in0 * dpow((1.0 + ((kapa - 1) / 2) * mach * mach), 1 / (1 - kapa));
            T normalVelocity = mach * dsqrt((kapa * p) / rhoIn);
            WR[0] = rhoIn;
#pragma unroll
            for (int d = 0; d < DIM; ++d) WR[d + 1] = -rhoIn * normalVelocity * n[d];
        } else if (TT == BC_OUTLET) {
            T absVelocity = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) absVelocity += WL[d + 1] * WL[d + 1];
            absVelocity = dsqrt(absVelocity) / WL[0];
            T p = pressure(WL, P);  // Java evaluates kapa * pressure(WL) before reading WL[0]
            T a = dsqrt(kapa * p / WL[0]);
            T mach = absVelocity / a;
            if (val(mach) < 1) {
                const double rhoOut = pow(p_out, 1. / kapa);
                WR[0] = rhoOut;
#pragma unroll
                for (int d = 0; d < DIM; ++d) WR[d + 1] = rhoOut * WL[d + 1] / WL[0];
            } else {
#pragma unroll
                for (int j = 0; j < NE; j++) WR[j] = WL[j];
            }
        }
    }

    // inviscid, no source: never called (kViscous / kSource are false)
    template <class T>
    static FP_HD void diffusiveFlux(T*, const T*, const double*, int, T* flux, const fp_model_params&) {
        for (int j = 0; j < NE; j++) flux[j] = 0.0;
    }
    template <class T>
    static FP_HD void diffusiveFluxAll(T*, const T*, T* fv, const fp_model_params&) {
        for (int j = 0; j < DIM * NE; j++) fv[j] = 0.0;
    }
    template <class T>
    static FP_HD void numericalDiffusiveFlux(T*, const T*, const double*, int, const double*, T* flux,
                                             const fp_model_params&) {
        for (int j = 0; j < NE; j++) flux[j] = 0.0;
    }
    template <class T>
    static FP_HD void sourceTerm(T*, const T*, double, const double*, T* s, const fp_model_params&) {
        for (int j = 0; j < NE; j++) s[j] = 0.0;
    }
    // Aerodynamics.stressVector: -p n
    template <class T>
    static FP_HD void stressVector(T* W, const T*, const double* n, T* sv, const fp_model_params& P) {
        T p = pressure(W, P);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            sv[d] = 0.0;
            sv[d] -= p * n[d];
        }
    }
    template <class T>
    static FP_HD T functionalPressure(const T*, const fp_model_params&) {
        return T(0.0);
    }
    static FP_HD bool isIPFace(int TT) { return TT == BC_WALL; }
    // AdiabaticEulers.isAdmissible, AdiabaticEulers.java:19-22
    static FP_HD bool isAdmissible(const double* W) { return W[0] > ADMISSIBLE_TOL; }
};

// ============================================================================ scalar test equation
// TestScalarEquation.java (FlowPro/src/test/java/flowpro/user/equation)
template <int DIM, bool VISC>
struct Scalar {
    static constexpr int NE = 1;
    static constexpr bool kFastFace = false;
    static constexpr bool kViscous = VISC;
    static constexpr bool kSource = true;
    static constexpr bool kConvective = true;

    static FP_HD double exact(const double* x) { return sin(2 * x[0] + x[1]); }

    template <class T>
    static FP_HD T maxEigenvalue(T*, const double*, const fp_model_params& P) { return T(P.lambda); }
    template <class T>
    static FP_HD void convectiveFlux(T* W, const double* n, T* f, const fp_model_params& P) {
        double an = 0;
        for (int d = 0; d < DIM; d++) an += P.a[d] * n[d];
        f[0] = an * W[0];
    }
    template <class T>
    static FP_HD void convectiveFluxAxis(T* W, int ax, T* f, const fp_model_params& P) {
        double n[DIM];
        for (int d = 0; d < DIM; d++) n[d] = d == ax ? 1.0 : 0.0;
        convectiveFlux(W, n, f, P);
    }
    template <class T>
    static FP_HD void numericalConvectiveFlux(T* WL, T* WR, const double* n, int, const double*, T* f,
                                              const fp_model_params& P) {
        T fL, fR;
        convectiveFlux(WL, n, &fL, P);
        convectiveFlux(WR, n, &fR, P);
        f[0] = (fL + fR) / 2.0 - P.lambda * (WR[0] - WL[0]) / 2.0;
    }
    template <class T>
    static FP_HD void boundaryValue(T*, const double*, int, const double*, const double* X, T* WR,
                                    const fp_model_params&, double) {
        WR[0] = exact(X);
    }
    template <class T>
    static FP_HD void diffusiveFlux(T*, const T* dW, const double* n, int ax, T* flux, const fp_model_params& P) {
        T f = 0.0;
        for (int d = 0; d < DIM; d++) {
            double nd = n == nullptr ? (d == ax ? 1.0 : 0.0) : n[d];
            f += P.k_diff * dW[d] * nd;
        }
        flux[0] = f;
    }
    template <class T>
    static FP_HD void numericalDiffusiveFlux(T* Wc, const T* dWc, const double* n, int, const double*, T* flux,
                                             const fp_model_params& P) {
        diffusiveFlux(Wc, dWc, n, 0, flux, P);
    }
    template <class T>
    static FP_HD void convectiveFluxAll(T* W, T* f, const fp_model_params& P) {
        for (int d = 0; d < DIM; d++) convectiveFluxAxis(W, d, f + d, P);
    }
    template <class T>
    static FP_HD void diffusiveFluxAll(T* W, const T* dW, T* fv, const fp_model_params& P) {
        for (int d = 0; d < DIM; d++) diffusiveFlux(W, dW, (const double*)nullptr, d, fv + d, P);
    }
    template <class T>
    static FP_HD void sourceTerm(T*, const T*, double, const double* X, T* s, const fp_model_params& P) {
        double phase = 2 * X[0] + X[1];
        s[0] = (2 * P.a[0] + P.a[1]) * cos(phase) + 5 * P.k_diff * sin(phase);
    }
    template <class T>
    static FP_HD void stressVector(T*, const T*, const double*, T* sv, const fp_model_params&) {
        for (int d = 0; d < DIM; d++) sv[d] = 0.0;
    }
    template <class T>
    static FP_HD T functionalPressure(const T*, const fp_model_params&) {
        return T(0.0);
    }
    static FP_HD bool isIPFace(int) { return true; }
    static FP_HD bool isAdmissible(const double*) { return true; }
};

}  // namespace fp
