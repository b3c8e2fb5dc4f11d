// Table of the kernel launchers of one compiled configuration (model x dimension x
// order).  Each fp_res_*.cu translation unit instantiates the kernels of one model
// family and returns its tables, so the configurations compile in parallel.
#pragma once
#include <cuda_runtime.h>

#include "fp_kernels.cuh"

namespace fp {

struct Launchers {
    int nc = 0;     // unknowns per element
    int ntrun = 0;  // size of the truncation matrix at the end of the reference tables
    void (*residual)(const DevMesh&, cudaStream_t, const double* W, double* R) = nullptr;
    // the two passes of residual(), separately (per-kernel timing)
    void (*faces)(const DevMesh&, cudaStream_t, const double* W) = nullptr;
    void (*elements)(const DevMesh&, cudaStream_t, const double* W, double* R) = nullptr;
    // the passes over a range of faces (f0 .. f1 - 1) or elements (e0 .. e1 - 1)
    void (*faces_range)(const DevMesh&, cudaStream_t, const double* W, int f0, int f1) = nullptr;
    void (*elements_range)(const DevMesh&, cudaStream_t, const double* W, double* R, int e0, int e1) = nullptr;
    void (*rk_stage)(const DevMesh&, cudaStream_t, const double* W, const double* Wo, const double* Wb, double a, double b,
                     double dt, double* Wout, double* Rsave) = nullptr;
    void (*matfree)(const DevMesh&, cudaStream_t, const double* W, const double* V, double a1, double* Y) = nullptr;
    void (*matfree_gather)(const DevMesh&, cudaStream_t, const double* W, const double* V, double a1, double* Y) = nullptr;
    void (*limiter)(const DevMesh&, cudaStream_t, const double* W, double dampTol, double penalty, const double* trun,
                    double* eps, double* cip) = nullptr;
    void (*positivity)(const DevMesh&, cudaStream_t, double* W, int* count) = nullptr;
    void (*norms)(const DevMesh&, cudaStream_t, const double* R, double* part) = nullptr;
    void (*dtbound)(const DevMesh&, cudaStream_t, const double* W, double factor, double* part) = nullptr;
    void (*rhs)(const DevMesh&, cudaStream_t, const double* W, const double* Wo, const double* Wo2, double a1, double a2,
                double a3, double* R, double* rhs, double* part) = nullptr;
    void (*fd)(const DevMesh&, cudaStream_t, const double* W, double* K0, double* KR0, double h, double a1, double* Adiag,
               double* Aneigh) = nullptr;
    void (*jac_exact)(const DevMesh&, cudaStream_t, const double* W, double a1, double* Adiag, double* Aneigh) = nullptr;
    // exact blocks into the block ILU(0) factor storage (float when fp32, else double)
    void (*jac_exact_factor)(const DevMesh&, cudaStream_t, const double* W, double a1, void* F, int fp32) = nullptr;
    // per-element norms R_m^T M^-1 R_m [NE][ld] and time-step bounds [ld] (batches of cases)
    void (*norms_elem)(const DevMesh&, cudaStream_t, const double* R, double* out) = nullptr;
    void (*dtbound_elem)(const DevMesh&, cudaStream_t, const double* W, double factor, double* out) = nullptr;
    // moving mesh: mass matrix of time level lev from the geometry; discrete-GCL mass matrix of level 0
    void (*mass_geo)(const DevMesh&, cudaStream_t, int lev, double* mass) = nullptr;
    void (*gcl_mass)(const DevMesh&, cudaStream_t, double a1, double a2, double a3, double* mass) = nullptr;
    // g = (dR/dW)^T lambda, no stored Jacobian
    void (*vjp)(const DevMesh&, cudaStream_t, const double* W, const double* lam, double* g) = nullptr;
    void (*surface)(const DevMesh&, cudaStream_t, const double* W, int kind, int bc, double* part, double* dIdW) = nullptr;
};

// per model family (fp_res_*.cu); nullptr when the order is not built
const Launchers* launchers_ns2(int viscous, int order);
const Launchers* launchers_ns3(int viscous, int order);
const Launchers* launchers_sa2(int order);
const Launchers* launchers_scalar2(int viscous, int order);
const Launchers* launchers_adiabatic(int dim, int order);

// the table for a model configuration, nullptr when it is not built
inline const Launchers* find_launchers(const fp_model_params& P, int order) {
    if (P.dim == 2 && P.model == FP_MODEL_NAVIER_STOKES) return launchers_ns2(P.is_diffusive, order);
    if (P.dim == 3 && P.model == FP_MODEL_NAVIER_STOKES) return launchers_ns3(P.is_diffusive, order);
    if (P.dim == 2 && P.model == FP_MODEL_SPALART_ALLMARAS) return launchers_sa2(order);
    if (P.dim == 2 && P.model == FP_MODEL_SCALAR_TEST) return launchers_scalar2(P.is_diffusive, order);
    if (P.model == FP_MODEL_ADIABATIC_EULERS) return launchers_adiabatic(P.dim, order);
    return nullptr;
}

}  // namespace fp
