// fp_l2_norms_noalloc: the per-equation L2 norms of a residual, sqrt(sum_e R_m^T M_e^-1 R_m),
// computed without allocating any memory.
//
// Who needs it: a caller that must not call cudaMalloc/cudaFree itself — for example a
// Java host whose device memory comes from an arena or pool owned by someone else (the
// JVM side hands over device pointers through FFM/JNI and forbids raw CUDA allocation),
// or a thread that has to avoid the device-wide synchronisation a cudaFree implies.  The
// context-based fp_residuum_norms allocates its reduction buffers when the mesh is
// uploaded; this variant keeps its only scratch (per-block partial sums) in a file-scope
// device array instead, so a call touches nothing but the caller's buffers and that array.
//
// Limits and sharing rules:
//   * at most kMaxElements elements (4096 blocks of 256 threads), n_basis <= 10,
//     n_eqs <= 8; larger sizes are rejected with FP_ERR_ARG;
//   * every GPU that loads the library holds the 256 KiB scratch array until exit;
//   * all calls share the array: calls that overlap on the GPU (different streams or
//     threads without ordering between them) race and give wrong norms;
//   * each call writes every partial it later reads, so nothing needs clearing between
//     calls; the array keeps the last call's partials;
//   * the first call on a device resolves the array's device address (cudaGetSymbolAddress,
//     with that device current) and caches it: make that first call before any stream
//     capture on that device.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/flowgpu.h"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 4096;
constexpr int kMaxElements = kMaxBlocks * kThreads;
constexpr int kMaxEqs = 8;
constexpr int kMaxBasis = 10;
constexpr int kMaxDevices = 64;

// the only scratch: partial sums [block][equation]
static __device__ __align__(256) double g_norm_partials[kMaxBlocks * kMaxEqs];

std::mutex g_mutex;
double* g_partials_addr[kMaxDevices] = {nullptr};

// per element: R_m^T M^-1 R_m = |L^-1 R_m|^2 with M = L L^T (Cholesky), summed per block
__global__ void __launch_bounds__(kThreads)
    k_l2_partials(int n_elem, int nb, int neq, const double* __restrict__ R, const double* __restrict__ M,
                  double* __restrict__ partials) {
    __shared__ double sh[kThreads];
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double nrm[kMaxEqs];
    for (int m = 0; m < kMaxEqs; m++) nrm[m] = 0.0;
    if (e < n_elem) {
        double L[kMaxBasis * kMaxBasis];
        const double* Me = M + (size_t)e * nb * nb;
        for (int i = 0; i < nb; i++)
            for (int j = 0; j <= i; j++) {
                double s = Me[i * nb + j];
                for (int k = 0; k < j; k++) s -= L[i * kMaxBasis + k] * L[j * kMaxBasis + k];
                L[i * kMaxBasis + j] = (i == j) ? sqrt(s) : s / L[j * kMaxBasis + j];
            }
        const double* Re = R + (size_t)e * nb * neq;
        for (int m = 0; m < neq; m++) {
            double z[kMaxBasis], s2 = 0.0;
            for (int i = 0; i < nb; i++) {
                double s = Re[m * nb + i];
                for (int k = 0; k < i; k++) s -= L[i * kMaxBasis + k] * z[k];
                z[i] = s / L[i * kMaxBasis + i];
                s2 += z[i] * z[i];
            }
            nrm[m] = s2;
        }
    }
    for (int m = 0; m < neq; m++) {
        sh[threadIdx.x] = nrm[m];
        __syncthreads();
        for (int s = kThreads / 2; s > 0; s >>= 1) {
            if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) partials[(size_t)blockIdx.x * kMaxEqs + m] = sh[0];
        __syncthreads();
    }
}

// fixed-order sum of the block partials, one thread per equation
__global__ void k_l2_final(int nblocks, int neq, const double* __restrict__ partials, double* __restrict__ norms) {
    const int m = threadIdx.x;
    if (m >= neq) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; b++) s += partials[(size_t)b * kMaxEqs + m];
    norms[m] = sqrt(s);
}

int partials_address(double** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return FP_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_partials_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_norm_partials) != cudaSuccess || !p) return FP_ERR_CUDA;
        g_partials_addr[dev] = static_cast<double*>(p);
    }
    *out = g_partials_addr[dev];
    return FP_OK;
}

}  // namespace

extern "C" int fp_l2_norms_noalloc(int n_elements, int n_basis, int n_eqs, const double* r, const double* mass,
                                   double* norms, uintptr_t stream) {
    if (n_elements <= 0 || n_elements > kMaxElements || n_basis <= 0 || n_basis > kMaxBasis || n_eqs <= 0 ||
        n_eqs > kMaxEqs || !r || !mass || !norms)
        return FP_ERR_ARG;
    double* partials = nullptr;
    int rc = partials_address(&partials);
    if (rc) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int nblocks = (n_elements + kThreads - 1) / kThreads;
    k_l2_partials<<<nblocks, kThreads, 0, s>>>(n_elements, n_basis, n_eqs, r, mass, partials);
    k_l2_final<<<1, 32, 0, s>>>(nblocks, n_eqs, partials, norms);
    return cudaGetLastError() == cudaSuccess ? FP_OK : FP_ERR_CUDA;
}
