// Linear algebra on the element-block matrix: block SpMV, matrix-free operator,
// batched inversion of the diagonal blocks (FP64 or FP32) for block Jacobi,
// deterministic reductions and restarted left-preconditioned GMRES with
// modified Gram-Schmidt (flowpro/core/LinearSolvers/Gmres.java:42-199).
//
// Vectors are state-shaped: x[c * ld + e] (c = unknown of the element).  The
// matrix is stored untransposed per element block, A[r][c] at (r*nc + c)*ld + e
// (field-major, coalesced over elements); FlowPro keeps the same blocks transposed
// (Implicit.ADiag[column][row], SparseMatrix.updateData transposes them back).
#include <algorithm>
#include <cmath>
#include <vector>

#include "fp_ctx.h"
#include "fp_dispatch.cuh"

namespace fp {

namespace {
constexpr int kRedBlocks = 592;  // 4 x 148 SMs
constexpr int kRedThreads = 256;

// y[r][e] = sum_c A_diag[r][c] x[c][e] + sum_k sum_c A_k[r][c] x[c][nb_k(e)]
__global__ void __launch_bounds__(128)
    k_spmv(int nElem, int ld, int nc, int nf, const double* __restrict__ Ad, const double* __restrict__ An,
           const int* __restrict__ tt, const double* __restrict__ x, double* __restrict__ y) {
    const int e = blockIdx.y * blockDim.x + threadIdx.x;  // rows of one element range in consecutive blocks:
    const int r = blockIdx.x;                             // the vector entries they read stay in cache
    if (e >= nElem) return;
    const size_t blk = (size_t)nc * nc * ld;
    const double* A = Ad + (size_t)r * nc * ld + e;
    double s = 0;
    for (int c = 0; c < nc; c++) s += __ldg(A + (size_t)c * ld) * __ldg(x + (size_t)c * ld + e);
    for (int k = 0; k < nf; k++) {
        const int nb = __ldg(tt + (size_t)k * ld + e);
        if (nb < 0) continue;
        const double* B = An + k * blk + (size_t)r * nc * ld + e;
        for (int c = 0; c < nc; c++) s += __ldg(B + (size_t)c * ld) * __ldg(x + (size_t)c * ld + nb);
    }
    y[(size_t)r * ld + e] = s;
}

// y = A^T x: y[c][e] = sum_r A_diag(e)[r][c] x[r][e] + sum_k sum_r A_kr(nb)[r][c] x[r][nb],
// nb = neighbour over face k, kr = nb's face toward e (the block of row nb, column e)
__global__ void __launch_bounds__(128)
    k_spmv_t(int nElem, int ld, int nc, int nf, int nperm, const double* __restrict__ Ad, const double* __restrict__ An,
             const int* __restrict__ tt, const int* __restrict__ fcode, const double* __restrict__ x, double* __restrict__ y) {
    const int e = blockIdx.y * blockDim.x + threadIdx.x;
    const int c = blockIdx.x;
    if (e >= nElem) return;
    const size_t blk = (size_t)nc * nc * ld;
    double s = 0;
    for (int r = 0; r < nc; r++) s += __ldg(Ad + ((size_t)r * nc + c) * ld + e) * __ldg(x + (size_t)r * ld + e);
    for (int k = 0; k < nf; k++) {
        const int nb = __ldg(tt + (size_t)k * ld + e);
        if (nb < 0) continue;
        const int kr = __ldg(fcode + (size_t)k * ld + e) / nperm;
        const double* B = An + kr * blk;
        for (int r = 0; r < nc; r++) s += __ldg(B + ((size_t)r * nc + c) * ld + nb) * __ldg(x + (size_t)r * ld + nb);
    }
    y[(size_t)c * ld + e] = s;
}

// y[r][e] = sum_c P[c][r] x[c][e]  (transposed inverse diagonal block, adjoint solves)
template <class Real>
__global__ void __launch_bounds__(128)
    k_block_apply_t(int nElem, int ld, int nc, const Real* __restrict__ P, const double* __restrict__ x, double* __restrict__ y) {
    const int e = blockIdx.y * blockDim.x + threadIdx.x;  // rows of one element range in consecutive blocks:
    const int r = blockIdx.x;                             // the vector entries they read stay in cache
    if (e >= nElem) return;
    Real s = 0;
    for (int c = 0; c < nc; c++) s += P[((size_t)c * nc + r) * ld + e] * (Real)__ldg(x + (size_t)c * ld + e);
    y[(size_t)r * ld + e] = (double)s;
}

// y[r][e] = sum_c P[r][c] x[c][e]  (P: inverse diagonal block)
template <class Real>
__global__ void __launch_bounds__(128)
    k_block_apply(int nElem, int ld, int nc, const Real* __restrict__ P, const double* __restrict__ x, double* __restrict__ y) {
    const int e = blockIdx.y * blockDim.x + threadIdx.x;  // rows of one element range in consecutive blocks:
    const int r = blockIdx.x;                             // the vector entries they read stay in cache
    if (e >= nElem) return;
    const Real* A = P + (size_t)r * nc * ld + e;
    Real s = 0;
    for (int c = 0; c < nc; c++) s += A[(size_t)c * ld] * (Real)__ldg(x + (size_t)c * ld + e);
    y[(size_t)r * ld + e] = (double)s;
}

// Inverse of each diagonal block by Gauss-Jordan elimination with partial pivoting in
// shared memory, one thread block per element; the result is stored in FP64 or FP32.
template <class Real>
__global__ void __launch_bounds__(128)
    k_block_invert(int nElem, int ld, int nc, const double* __restrict__ Ad, Real* __restrict__ P, unsigned* status) {
    extern __shared__ double sm[];
    const int e = blockIdx.x;
    if (e >= nElem) return;
    const int n2 = 2 * nc;
    double* a = sm;              // [nc][2nc]
    __shared__ int piv;
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    for (int t = threadIdx.x; t < nc * nc; t += blockDim.x) {
        int r = t / nc, c = t - r * nc;
        a[r * n2 + c] = Ad[(size_t)t * ld + e];
        a[r * n2 + nc + c] = (r == c) ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int p = 0; p < nc; p++) {
        if (threadIdx.x == 0) {
            int best = p;
            double bv = fabs(a[p * n2 + p]);
            for (int r = p + 1; r < nc; r++) {
                double v = fabs(a[r * n2 + p]);
                if (v > bv) {
                    bv = v;
                    best = r;
                }
            }
            piv = best;
            if (!(bv > 0) || !isfinite(bv)) bad = 1;
        }
        __syncthreads();
        if (bad) break;
        if (piv != p)
            for (int c = threadIdx.x; c < n2; c += blockDim.x) {
                double t = a[p * n2 + c];
                a[p * n2 + c] = a[piv * n2 + c];
                a[piv * n2 + c] = t;
            }
        __syncthreads();
        const double inv = 1.0 / a[p * n2 + p];
        __syncthreads();
        for (int c = threadIdx.x; c < n2; c += blockDim.x) a[p * n2 + c] *= inv;
        __syncthreads();
        for (int t = threadIdx.x; t < nc * n2; t += blockDim.x) {
            int r = t / n2, c = t - r * n2;
            if (r != p && c != p) a[r * n2 + c] -= a[r * n2 + p] * a[p * n2 + c];
        }
        __syncthreads();
        for (int r = threadIdx.x; r < nc; r += blockDim.x)
            if (r != p) a[r * n2 + p] = 0.0;
        __syncthreads();
    }
    if (bad) {
        if (threadIdx.x == 0) atomicOr(status, (unsigned)FP_DEV_SINGULAR);
        return;
    }
    for (int t = threadIdx.x; t < nc * nc; t += blockDim.x) {
        int r = t / nc, c = t - r * nc;
        P[(size_t)t * ld + e] = (Real)a[r * n2 + nc + c];
    }
}

__global__ void k_dot_part(size_t n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ part) {
    __shared__ double sh[kRedThreads];
    double s = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        s += a[i] * b[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int k = kRedThreads / 2; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_dot_final(const double* __restrict__ part, int n, double* __restrict__ out) {
    __shared__ double sh[kRedThreads];
    double s = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int k = kRedThreads / 2; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

// Classical Gram-Schmidt pass of the Arnoldi step, fused: h[k] = <w, V_k> for k < kc
// (k_mdot_part over a grid of kRedBlocks x ceil(kc / kDotVecs) blocks, each reading w once for
// its kDotVecs basis vectors, then k_mdot_final, both in a fixed order), then
// w -= sum_k h[k] V_k (k_mdaxpy, one pass over the basis).
constexpr int kDotVecs = 8;
__global__ void __launch_bounds__(kRedThreads) k_mdot_part(size_t n, int kc, const double* __restrict__ w,
                                                           const double* __restrict__ V, size_t stride,
                                                           double* __restrict__ part) {
    __shared__ double sh[kDotVecs][kRedThreads / 32];
    const int k0 = blockIdx.y * kDotVecs;
    const int nk = min(kDotVecs, kc - k0);
    const double* V0 = V + (size_t)k0 * stride;
    double s[kDotVecs];
#pragma unroll
    for (int k = 0; k < kDotVecs; k++) s[k] = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double wi = w[i];
#pragma unroll
        for (int k = 0; k < kDotVecs; k++)
            if (k < nk) s[k] += wi * V0[(size_t)k * stride + i];
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kDotVecs; k++) {
        double v = s[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[k][wid] = v;
    }
    __syncthreads();
    if ((int)threadIdx.x < nk) {
        double v = 0.0;
        for (int q = 0; q < kRedThreads / 32; q++) v += sh[threadIdx.x][q];
        part[(size_t)(k0 + threadIdx.x) * gridDim.x + blockIdx.x] = v;
    }
}

__global__ void k_mdot_final(const double* __restrict__ part, int nblk, double* __restrict__ out) {
    __shared__ double sh[kRedThreads];
    const double* p = part + (size_t)blockIdx.x * nblk;
    double s = 0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) s += p[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int k = kRedThreads / 2; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

__global__ void k_mdaxpy(size_t n, int kc, double* __restrict__ w, const double* __restrict__ V, size_t stride,
                         const double* __restrict__ h) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double s = 0;
        for (int k = 0; k < kc; k++) s += h[k] * V[(size_t)k * stride + i];
        w[i] -= s;
    }
}

// y -= h[0] * x, h on the device
__global__ void k_axpy_dev(size_t n, double* __restrict__ y, const double* __restrict__ x, const double* __restrict__ h) {
    const double a = *h;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) y[i] -= a * x[i];
}
// y = x / sqrt(h[0]) (0 when h[0] == 0: happy breakdown, Gmres.java:80-84)
__global__ void k_scale_norm(size_t n, double* __restrict__ y, const double* __restrict__ x, const double* __restrict__ h2) {
    const double nrm = sqrt(*h2);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = nrm > 0 ? x[i] / nrm : 0.0;
}
__global__ void k_axpby(size_t n, double* __restrict__ y, double a, const double* __restrict__ x, double b) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = a * x[i] + b * y[i];
}
// x += sum_k V_k y_k (y on the device)
__global__ void k_update_x(size_t n, int kmax, double* __restrict__ x, const double* __restrict__ V, size_t stride,
                           const double* __restrict__ y) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double s = x[i];
        for (int k = 0; k < kmax; k++) s += V[k * stride + i] * y[k];
        x[i] = s;
    }
}
// y = b - y
__global__ void k_bminus(size_t n, double* __restrict__ y, const double* __restrict__ b) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) y[i] = b[i] - y[i];
}

inline unsigned vgrid(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16); }
}  // namespace

int dot(fp_ctx* c, const double* a, const double* b, double* dev_out) {
    k_dot_part<<<kRedBlocks, kRedThreads, 0, c->stream>>>(c->nvec, a, b, c->d_part);
    k_dot_final<<<1, kRedThreads, 0, c->stream>>>(c->d_part, kRedBlocks, dev_out);
    return cuda_check(c, cudaGetLastError(), "dot");
}

int vec_copy(fp_ctx* c, double* y, const double* x) {
    return cuda_check(c, cudaMemcpyAsync(y, x, c->nvec * sizeof(double), cudaMemcpyDeviceToDevice, c->stream), "copy");
}

int vec_axpby(fp_ctx* c, double* y, double a, const double* x, double b) {
    k_axpby<<<vgrid(c->nvec), 256, 0, c->stream>>>(c->nvec, y, a, x, b);
    return cuda_check(c, cudaGetLastError(), "axpby");
}

int vec_add_scaled(fp_ctx* c, double* y, const double* x, double s) { return vec_axpby(c, y, s, x, 1.0); }

int spmv(fp_ctx* c, const double* x, double* y) {
    const int nE = c->hm.nElem;
    dim3 g(c->nc, (nE + 127) / 128);
    k_spmv<<<g, 128, 0, c->stream>>>(nE, c->hm.ld, c->nc, c->hm.nf, c->d_Adiag, c->d_Aneigh, c->d_tt, x, y);
    return cuda_check(c, cudaGetLastError(), "spmv");
}

// A_diag += delta * (mass matrix of the element): moves assembled blocks a1 M - dR/dW to a
// new BDF coefficient a1 without re-running the finite differences (lagged Jacobian).  The
// factorised preconditioner is left as it is (the caller decides when to refactorise).
__global__ void __launch_bounds__(128) k_mass_shift(int nElem, int ld, int nc, int nb, const double* __restrict__ Mref,
                                                    const double* __restrict__ jac, const double* __restrict__ mass,
                                                    double delta, double* __restrict__ Adiag) {
    const int e = blockIdx.y * blockDim.x + threadIdx.x;  // rows of one element range in consecutive blocks:
    const int r = blockIdx.x;                             // the vector entries they read stay in cache
    if (e >= nElem) return;
    const int m = r / nb, br = r - m * nb;
    if (mass) {  // moving mesh: the current level's element mass matrix
        for (int bc = 0; bc < nb; bc++)
            Adiag[((size_t)r * nc + m * nb + bc) * ld + e] += delta * mass[((size_t)br * nb + bc) * ld + e];
        return;
    }
    const double s = delta * jac[e];
    for (int bc = 0; bc < nb; bc++) Adiag[((size_t)r * nc + m * nb + bc) * ld + e] += s * Mref[br * nb + bc];
}

int mass_shift(fp_ctx* c, double delta) {
    if (delta == 0.0) return FP_OK;
    const int nE = c->hm.nElem;
    dim3 g(c->nc, (nE + 127) / 128);
    const double* jac = c->d_geo + (size_t)(c->hm.dim * c->hm.dim) * c->hm.ld;
    k_mass_shift<<<g, 128, 0, c->stream>>>(nE, c->hm.ld, c->nc, c->hm.tab.nb, c->d_tab + c->hm.tab.o_Mref, jac, c->d_mass,
                                           delta, c->d_Adiag);
    return cuda_check(c, cudaGetLastError(), "mass shift");
}

int spmv_t(fp_ctx* c, const double* x, double* y) {
    const int nE = c->hm.nElem;
    dim3 g(c->nc, (nE + 127) / 128);
    k_spmv_t<<<g, 128, 0, c->stream>>>(nE, c->hm.ld, c->nc, c->hm.nf, c->hm.tab.nperm, c->d_Adiag, c->d_Aneigh, c->d_tt,
                                       c->d_fcode, x, y);
    return cuda_check(c, cudaGetLastError(), "spmv_t");
}

static int prec_factor_impl(fp_ctx* c, int kind, int precision);

int prec_factor(fp_ctx* c, int kind, int precision) {
    prof_begin(c, PH_FACTOR);
    const int rc = prec_factor_impl(c, kind, precision);
    prof_end(c);
    return rc;
}

static int prec_factor_impl(fp_ctx* c, int kind, int precision) {
    if (kind == FP_PREC_NONE) {
        c->prec_kind = kind;
        c->prec_ready = precision;
        return FP_OK;
    }
    if (kind == FP_PREC_BLOCKILU0) {
        int rc = ilu_factor(c, precision);
        if (rc) return rc;
        c->prec_kind = kind;
        c->prec_ready = precision;
        return FP_OK;
    }
    if (kind != FP_PREC_BLOCKJACOBI) return set_err(c, FP_ERR_UNSUPPORTED, "preconditioner not available");
    if (!c->d_Adiag) return set_err(c, FP_ERR_STATE, "block Jacobi: no assembled blocks");
    const int nE = c->hm.nElem, nc = c->nc, ld = c->hm.ld;
    size_t smem = (size_t)nc * 2 * nc * sizeof(double);
    // the inverse diagonal blocks of the precision in use, allocated on first use
    void** pp = precision == FP_PREC_FP32 ? (void**)&c->d_P32 : (void**)&c->d_P64;
    if (!*pp) {
        const size_t bytes = (size_t)nc * nc * ld * (precision == FP_PREC_FP32 ? sizeof(float) : sizeof(double));
        void* q = nullptr;
        int arc = cuda_check(c, cudaMalloc(&q, bytes), "cudaMalloc (block Jacobi)");
        if (arc) return arc;
        c->allocs.push_back((double*)q);
        *pp = q;
    }
    int rc = cuda_check(c, cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->stream), "memset");
    if (rc) return rc;
    if (precision == FP_PREC_FP32) {
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(k_block_invert<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_block_invert<float><<<nE, 128, smem, c->stream>>>(nE, ld, nc, c->d_Adiag, c->d_P32, c->d_status);
    } else {
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(k_block_invert<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_block_invert<double><<<nE, 128, smem, c->stream>>>(nE, ld, nc, c->d_Adiag, c->d_P64, c->d_status);
    }
    rc = cuda_check(c, cudaGetLastError(), "block invert");
    if (rc) return rc;
    unsigned st = 0;
    rc = cuda_check(c, cudaMemcpyAsync(&st, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream), "copy");
    if (rc) return rc;
    rc = cuda_check(c, cudaStreamSynchronize(c->stream), "sync");
    if (rc) return rc;
    if (st & FP_DEV_SINGULAR) return set_err(c, FP_ERR_SINGULAR, "singular diagonal block in block Jacobi factorisation");
    c->prec_kind = kind;
    c->prec_ready = precision;
    return FP_OK;
}

int prec_apply(fp_ctx* c, int kind, const double* x, double* y) {
    if (kind == FP_PREC_NONE) return vec_copy(c, y, x);
    if (kind == FP_PREC_BLOCKILU0) {
        if (c->kry_transposed) return set_err(c, FP_ERR_UNSUPPORTED, "block ILU(0) is not available for adjoint solves");
        return ilu_apply(c, x, y);
    }
    const int nE = c->hm.nElem;
    dim3 g(c->nc, (nE + 127) / 128);
    if (c->kry_transposed) {
        if (c->prec_ready == FP_PREC_FP32)
            k_block_apply_t<float><<<g, 128, 0, c->stream>>>(nE, c->hm.ld, c->nc, c->d_P32, x, y);
        else
            k_block_apply_t<double><<<g, 128, 0, c->stream>>>(nE, c->hm.ld, c->nc, c->d_P64, x, y);
        return cuda_check(c, cudaGetLastError(), "block apply");
    }
    if (c->prec_ready == FP_PREC_FP32)
        k_block_apply<float><<<g, 128, 0, c->stream>>>(nE, c->hm.ld, c->nc, c->d_P32, x, y);
    else
        k_block_apply<double><<<g, 128, 0, c->stream>>>(nE, c->hm.ld, c->nc, c->d_P64, x, y);
    return cuda_check(c, cudaGetLastError(), "block apply");
}

int matfree_apply(fp_ctx* c, const double* x, double* y);  // fp_residual.cu

static int apply_A(fp_ctx* c, int jacobian, const double* x, double* y) {
    prof_begin(c, PH_OPERATOR);
    const int rc = c->kry_transposed ? spmv_t(c, x, y) : jacobian == FP_JAC_MATRIXFREE ? matfree_apply(c, x, y) : spmv(c, x, y);
    prof_end(c);
    return rc;
}

static int apply_M(fp_ctx* c, int kind, const double* x, double* y) {
    prof_begin(c, PH_PREC);
    const int rc = prec_apply(c, kind, x, y);
    prof_end(c);
    return rc;
}

// Gmres.rotmat, Gmres.java:132-148
static void rotmat(double a, double b, double& cs, double& sn) {
    if (b == 0) {
        cs = 1;
        sn = 0;
    } else if (std::fabs(b) > std::fabs(a)) {
        double t = a / b;
        sn = 1 / std::sqrt(1 + t * t);
        cs = t * sn;
    } else {
        double t = b / a;
        cs = 1 / std::sqrt(1 + t * t);
        sn = t * cs;
    }
}

// Gmres.lsolve, Gmres.java:176-199 (Gaussian elimination of the rotated Hessenberg matrix)
static std::vector<double> lsolve(std::vector<std::vector<double>> A, std::vector<double> b, int N) {
    for (int p = 0; p < N; p++)
        for (int i = p + 1; i < N; i++) {
            double alpha = A[i][p] / A[p][p];
            b[i] -= alpha * b[p];
            for (int j = p; j < N; j++) A[i][j] -= alpha * A[p][j];
        }
    std::vector<double> x(N);
    for (int i = N - 1; i >= 0; i--) {
        double sum = 0.0;
        for (int j = i + 1; j < N; j++) sum += A[i][j] * x[j];
        x[i] = (b[i] - sum) / A[i][i];
    }
    return x;
}

static int fetch(fp_ctx* c, int n, double* host) {
    int rc = cuda_check(c, cudaMemcpyAsync(host, c->d_scal, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "copy");
    if (rc) return rc;
    rc = cuda_check(c, cudaStreamSynchronize(c->stream), "sync");
    prof_resolve(c);
    return rc;
}

// Restarted left-preconditioned GMRES(m) on (A, b = d_b) from x = d_x (Gmres.solve,
// Gmres.java:42-122): tolerance relative to ||M^-1 b||, MGS orthogonalisation, Givens
// rotations, at most max_restarts cycles.
int gmres(fp_ctx* c, int jacobian, int kind, int m, int max_restarts, double tol, int* iters, double* rel) {
    int rc;
    const size_t n = c->nvec;
    double* V = c->d_V;
    double *w = c->d_w, *aux = c->d_aux, *r = c->d_r, *x = c->d_x, *b = c->d_b;
    double* hs = c->h_scal;
    int total = 0;
    // M.apply(r, b); bnrm2 = ||r||
    if ((rc = apply_M(c, kind, b, r)) || (rc = dot(c, r, r, c->d_scal)) || (rc = fetch(c, 1, hs))) return rc;
    double bnrm2 = std::sqrt(hs[0]);
    if (bnrm2 == 0) bnrm2 = 1;
    // r = M (b - A x)
    if ((rc = apply_A(c, jacobian, x, aux))) return rc;
    k_bminus<<<vgrid(n), 256, 0, c->stream>>>(n, aux, b);
    if ((rc = apply_M(c, kind, aux, r)) || (rc = dot(c, r, r, c->d_scal)) || (rc = fetch(c, 1, hs))) return rc;
    double error = std::sqrt(hs[0]) / bnrm2;
    if (iters) *iters = 0;
    if (rel) *rel = error;
    if (error < tol) return FP_OK;
    std::vector<std::vector<double>> H(m + 1, std::vector<double>(m, 0.0));
    std::vector<double> cs(m, 0.0), sn(m, 0.0), s(m + 1, 0.0);
    for (int iter = 0; iter < max_restarts; iter++) {
        if ((rc = dot(c, r, r, c->d_scal)) || (rc = fetch(c, 1, hs))) return rc;
        double norm_r = std::sqrt(hs[0]);
        k_scale_norm<<<vgrid(n), 256, 0, c->stream>>>(n, V, r, c->d_scal);
        std::fill(s.begin(), s.end(), 0.0);
        s[0] = norm_r;
        bool done = false;
        for (int i = 0; i < m; i++) {
            total++;
            double* Vi = V + (size_t)i * n;
            if ((rc = apply_A(c, jacobian, Vi, aux)) || (rc = apply_M(c, kind, aux, w))) return rc;
            // orthogonalise w against V_0..V_i: two fused classical Gram-Schmidt passes (CGS2,
            // as stable as the modified Gram-Schmidt of Gmres.java:62-70 in a few launches)
            const int kc = i + 1;
            prof_begin(c, PH_KRYLOV);
            double* h1 = c->d_scal;        // first pass coefficients [0, 256)
            double* h2 = c->d_scal + 256;  // second pass [256, 512); |w|^2 at 512
            for (double* h : {h1, h2}) {
                k_mdot_part<<<dim3(kRedBlocks, (kc + kDotVecs - 1) / kDotVecs), kRedThreads, 0, c->stream>>>(n, kc, w, V, n,
                                                                                                             c->d_part);
                k_mdot_final<<<kc, kRedThreads, 0, c->stream>>>(c->d_part, kRedBlocks, h);
                k_mdaxpy<<<vgrid(n), 256, 0, c->stream>>>(n, kc, w, V, n, h);
            }
            if ((rc = dot(c, w, w, c->d_scal + 512))) return rc;
            k_scale_norm<<<vgrid(n), 256, 0, c->stream>>>(n, V + (size_t)(i + 1) * n, w, c->d_scal + 512);
            prof_end(c);
            if ((rc = fetch(c, 513, hs))) return rc;
            for (int k = 0; k <= i; k++) H[k][i] = hs[k] + hs[256 + k];
            H[i + 1][i] = std::sqrt(hs[512]);
            for (int k = 0; k <= i - 1; k++) {
                double temp = cs[k] * H[k][i] + sn[k] * H[k + 1][i];
                H[k + 1][i] = -sn[k] * H[k][i] + cs[k] * H[k + 1][i];
                H[k][i] = temp;
            }
            rotmat(H[i][i], H[i + 1][i], cs[i], sn[i]);
            double temp = cs[i] * s[i];
            s[i + 1] = -sn[i] * s[i];
            s[i] = temp;
            H[i][i] = cs[i] * H[i][i] + sn[i] * H[i + 1][i];
            H[i + 1][i] = 0;
            error = std::fabs(s[i + 1]) / bnrm2;
            if (error <= tol) {
                std::vector<double> y = lsolve(H, s, i + 1);
                rc = cuda_check(c, cudaMemcpyAsync(c->d_scal, y.data(), (i + 1) * sizeof(double), cudaMemcpyHostToDevice, c->stream), "copy");
                if (rc) return rc;
                k_update_x<<<vgrid(n), 256, 0, c->stream>>>(n, i + 1, x, V, n, c->d_scal);
                done = true;
                break;
            }
        }
        if (!done) {
            std::vector<double> y = lsolve(H, s, m);
            rc = cuda_check(c, cudaMemcpyAsync(c->d_scal, y.data(), m * sizeof(double), cudaMemcpyHostToDevice, c->stream), "copy");
            if (rc) return rc;
            k_update_x<<<vgrid(n), 256, 0, c->stream>>>(n, m, x, V, n, c->d_scal);
        }
        // true preconditioned residual r = M (b - A x).  Gmres.java trusts the Arnoldi
        // estimate when it drops below tol; with an FP32 preconditioner the estimate can
        // run ahead of the true residual, so convergence is accepted on the true one (for
        // an FP64 preconditioner both agree to rounding and the iteration count is Java's).
        if ((rc = apply_A(c, jacobian, x, aux))) return rc;
        k_bminus<<<vgrid(n), 256, 0, c->stream>>>(n, aux, b);
        if ((rc = apply_M(c, kind, aux, r)) || (rc = dot(c, r, r, c->d_scal)) || (rc = fetch(c, 1, hs))) return rc;
        error = std::sqrt(hs[0]) / bnrm2;
        if (error <= tol) break;
    }
    if (iters) *iters = total;
    if (rel) *rel = error;
    rc = cuda_check(c, cudaStreamSynchronize(c->stream), "sync");
    if (rc) return rc;
    if (!(error <= tol)) return set_err(c, FP_ERR_NOT_CONVERGED, "GMRES did not converge");
    return FP_OK;
}

}  // namespace fp
