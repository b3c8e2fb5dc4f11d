// Block ILU(0) preconditioner on the element-block matrix (BlockILU0.factor / apply,
// flowpro/core/LinearSolvers/preconditioners/BlockILU0.java:22-243).
//
// Rows are taken in the DOF (RCM) order.  Row i of the factor is
//   for each lower neighbour k (rank[k] < rank[i]) in rank order:
//       L_ik = A_ik * inv(U_kk);  A_ij -= L_ik * U_kj  for every column j > k of row i that row k has
//   inv(U_ii) = inverse of the updated A_ii
// which is BlockILU0's loop; the only fill-in-free columns a row k can share with row
// i are i itself and (around a vertex or an edge of valence 3) a common neighbour, both
// handled by the per-element program built on the host.
//
// Device side:
//   * factor values in element-major storage, F[e][s][c][r] (column-major blocks):
//     s = 0 holds inv(U_ee), s = 1 + k the block coupling e with its neighbour over face
//     k (L or U);
//   * rows whose lower neighbours are all finished form a level.  The factorisation
//     runs one launch per level, one 512-thread block per row in shared memory
//     (register-tiled block products, Gauss-Jordan with implicit partial pivoting);
//   * an application (forward L sweep, backward U sweep) is ONE persistent cooperative
//     kernel: thread blocks stride over the elements of a level and meet at a grid
//     barrier between levels.  Each element's factor blocks are loaded into registers
//     before the (L2-coherent) loads of the neighbours' sweep values they multiply;
//   * the factorisation always runs in FP64; the FP32 variant stores a rounded copy
//     for the sweeps (mixed-precision GMRES).
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "fp_ctx.h"

namespace cg = cooperative_groups;

namespace fp {

namespace {

constexpr int kFactorThreads = 512;
constexpr int kSweepThreads = 512;
constexpr int kMaxNc = 64;   // unknowns per element
constexpr int kMaxF = 4;     // faces per element
constexpr int kMaxJ = 8;     // columns per thread and block in the sweeps: ceil(nc / (512 / nc)) <= 8 for nc <= 64

template <class T>
int ialloc(fp_ctx* c, T** p, size_t n) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) return cuda_check(c, e, "cudaMalloc (ILU)");
    c->allocs.push_back((double*)q);
    *p = (T*)q;
    return FP_OK;
}

// F[e][s] <- A_s(e) transposed into column-major blocks; tiles of 32 elements x 32
// block entries through shared memory so both the field-major read and the
// element-major write are coalesced.  Boundary faces get zero blocks.
__global__ void __launch_bounds__(256) k_ilu_gather(int nElem, int ld, int nc, int nf, const double* __restrict__ Ad,
                                                    const double* __restrict__ An, const int* __restrict__ tt,
                                                    double* __restrict__ F) {
    __shared__ double tile[32][33];
    const int nc2 = nc * nc;
    const int s = blockIdx.y;  // 0 diagonal, 1 + k face k
    const int e0 = blockIdx.x * 32;
    const int lane = threadIdx.x & 31, wy = threadIdx.x >> 5;  // 8 warps
    const double* A = s == 0 ? Ad : An + (size_t)(s - 1) * nc2 * ld;
    for (int o0 = 0; o0 < nc2; o0 += 32) {
        // load: warp row = output entry o, lanes along elements
        for (int j = wy; j < 32; j += 8) {
            const int o = o0 + j, e = e0 + lane;
            double v = 0.0;
            if (o < nc2 && e < nElem) {
                const int cc = o / nc, r = o - cc * nc;  // output (r, cc) column-major
                const bool interior = s == 0 || tt[(size_t)(s - 1) * ld + e] > -1;
                if (interior) v = A[(size_t)(r * nc + cc) * ld + e];
            }
            tile[j][lane] = v;
        }
        __syncthreads();
        // store: warp row = element, lanes along output entries
        for (int j = wy; j < 32; j += 8) {
            const int e = e0 + j, o = o0 + lane;
            if (e < nElem && o < nc2) F[((size_t)e * (1 + nf) + s) * nc2 + o] = tile[lane][j];
        }
        __syncthreads();
    }
}

// C (-)= X * Y for nc x nc column-major blocks in shared memory (nc <= 64, 512 threads):
// thread (r = t % 64, cb = t / 64) accumulates row r of the columns cb, cb + 8, ...;
// X is read conflict-free, Y as a warp broadcast.
__device__ __forceinline__ void block_mul(int nc, const double* X, const double* Y, double* C, bool subtract) {
    const int r = threadIdx.x & 63, cb = threadIdx.x >> 6;
    if (r >= nc) return;
    double acc[8];
#pragma unroll
    for (int j = 0; j < 8; j++) acc[j] = 0.0;
#pragma unroll 2
    for (int m = 0; m < nc; m++) {
        const double x = X[m * nc + r];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int cc = cb + 8 * j;
            if (cc < nc) acc[j] += x * Y[cc * nc + m];
        }
    }
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int cc = cb + 8 * j;
        if (cc < nc) {
            if (subtract)
                C[cc * nc + r] -= acc[j];
            else
                C[cc * nc + r] = acc[j];
        }
    }
}

// one level of the factorisation: one thread block per element row
__global__ void __launch_bounds__(kFactorThreads) k_ilu_factor(int nc, int nf, const int* __restrict__ lvl, int offset,
                                                               const int* __restrict__ opPtr, const int4* __restrict__ ops,
                                                               double* __restrict__ F, unsigned* status) {
    extern __shared__ double sm[];
    const int nc2 = nc * nc, ns = 1 + nf, n2 = 2 * nc;
    const int i = lvl[offset + blockIdx.x];
    const int t = threadIdx.x;
    double* R = sm;               // [ns][nc2] the row's blocks
    double* Lb = R + ns * nc2;    // current L block
    double* aug = Lb + nc2;       // [nc][2nc] Gauss-Jordan; before that, staging of row k's block
    __shared__ double fcol[kMaxNc];     // multipliers of the current pivot column
    __shared__ double prow[2 * kMaxNc]; // scaled pivot row
    __shared__ int used[kMaxNc], perm[kMaxNc];
    __shared__ int piv, bad;
    double* Fi = F + (size_t)i * ns * nc2;
    for (int q = t; q < ns * nc2; q += blockDim.x) R[q] = Fi[q];
    if (t == 0) bad = 0;
    if (t < kMaxNc) used[t] = 0;
    for (int q = opPtr[i]; q < opPtr[i + 1]; q++) {
        const int4 op = ops[q];
        // block of row k: inv(U_kk) for an L step, U_kj for an update
        const double* Y = F + ((size_t)op.z * ns + (op.x == 0 ? 0 : 1 + op.w)) * nc2;
        __syncthreads();
        for (int u = t; u < nc2; u += blockDim.x) aug[u] = __ldg(Y + u);
        __syncthreads();
        if (op.x == 0) {
            // L = A_ik * inv(U_kk)
            block_mul(nc, R + (size_t)(1 + op.y) * nc2, aug, Lb, false);
            __syncthreads();
            for (int u = t; u < nc2; u += blockDim.x) R[(size_t)(1 + op.y) * nc2 + u] = Lb[u];
        } else {
            // A_ij -= L * U_kj
            block_mul(nc, Lb, aug, R + (size_t)op.y * nc2, true);
        }
    }
    __syncthreads();
    // inverse of the updated diagonal block: Gauss-Jordan on [A | I] with implicit partial
    // pivoting (the pivot of column p is the largest unused row; rows stay in place).
    // Thread (column cc = t % 128, row group rg = t / 128) owns rows rg, rg + 4, ...
    const int cc = t & 127, rg = t >> 7;
    for (int u = t; u < nc2; u += blockDim.x) {
        const int c0 = u / nc, r0 = u - c0 * nc;
        aug[r0 * n2 + c0] = R[u];
        aug[r0 * n2 + nc + c0] = r0 == c0 ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int p = 0; p < nc; p++) {
        if (t < 32) {
            double bv = -1.0;
            int br = nc;
            for (int r = t; r < nc; r += 32) {
                const double v = used[r] ? -1.0 : fabs(aug[r * n2 + p]);
                if (v > bv) {
                    bv = v;
                    br = r;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
                const int orow = __shfl_xor_sync(0xffffffffu, br, o);
                if (ov > bv || (ov == bv && orow < br)) {
                    bv = ov;
                    br = orow;
                }
            }
            if (!(bv > 0) || !isfinite(bv) || br >= nc) {
                if (t == 0) bad = 1;
            } else {
                const double inv = 1.0 / aug[br * n2 + p];
                for (int c2 = t; c2 < n2; c2 += 32) prow[c2] = c2 == p ? 1.0 : aug[br * n2 + c2] * inv;
                for (int r = t; r < nc; r += 32) fcol[r] = r == br ? 0.0 : aug[r * n2 + p];
                if (t == 0) {
                    piv = br;
                    used[br] = 1;
                    perm[p] = br;
                }
            }
        }
        __syncthreads();
        if (bad) break;
        if (cc < n2) {
            const int pr = piv;
            const double a = prow[cc];
            for (int r = rg; r < nc; r += 4) {
                if (r == pr)
                    aug[r * n2 + cc] = a;
                else
                    aug[r * n2 + cc] = cc == p ? 0.0 : aug[r * n2 + cc] - fcol[r] * a;
            }
        }
        __syncthreads();
    }
    if (bad) {
        if (t == 0) atomicOr(status, (unsigned)FP_DEV_SINGULAR);
        return;
    }
    // inverse row r = right half of row perm[r]; stored column-major
    for (int u = t; u < nc2; u += blockDim.x) {
        const int c0 = u / nc, r0 = u - c0 * nc;
        Fi[u] = aug[perm[r0] * n2 + nc + c0];
    }
    for (int u = nc2 + t; u < ns * nc2; u += blockDim.x) Fi[u] = R[u];
}

__global__ void k_to_f32(size_t n, const double* __restrict__ a, float* __restrict__ b) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) b[t] = (float)a[t];
}

// One element of a sweep: out_i = in_i - sum_f B_f v_f over the faces in nb (B_f = block
// 1 + f of F[i], v_f the sweep value of neighbour nb.f), then, when D is set, out_i =
// D (that), D = block 0 (inv(U_ii)).  Thread t = g * nc + r (g < G = 512 / nc) handles
// row r of the columns c = g + G j; the G partial sums of a row meet in shared memory.
// v and in are read through L2 (ld.global.cg): other blocks wrote them in this kernel.
template <class T>
__device__ __forceinline__ void sweep_element(int nc, int nf, int ld, int i, int4 nb, const T* __restrict__ F, bool withD,
                                              const double* in, const double* v, double* out, double* vs, double* part,
                                              double* tv) {
    const int t = threadIdx.x, nc2 = nc * nc, G = kSweepThreads / nc;
    const int g = t / nc, r = t - g * nc;
    const T* Fi = F + (size_t)i * (1 + nf) * nc2;
    const int nbs[kMaxF] = {nb.x, nb.y, nb.z, nb.w};
    // factor entries first (independent of the sweep values)
    T fv[kMaxF][kMaxJ], dv[kMaxJ];
    if (g < G) {
#pragma unroll
        for (int f = 0; f < kMaxF; f++)
#pragma unroll
            for (int j = 0; j < kMaxJ; j++) {
                const int c = g + G * j;
                fv[f][j] = (f < nf && nbs[f] >= 0 && c < nc) ? Fi[(size_t)(1 + f) * nc2 + (size_t)c * nc + r] : T(0);
            }
        if (withD) {
#pragma unroll
            for (int j = 0; j < kMaxJ; j++) {
                const int c = g + G * j;
                dv[j] = c < nc ? Fi[(size_t)c * nc + r] : T(0);
            }
        }
    }
    // neighbours' sweep values: thread (f = t / 64, c = t % 64)
    if (t < kMaxF * 64) {
        const int f = t >> 6, c = t & 63;
        vs[t] = (f < nf && nbs[f] >= 0 && c < nc) ? __ldcg(v + (size_t)c * ld + nbs[f]) : 0.0;
    }
    __syncthreads();
    double s = 0.0;
    if (g < G) {
#pragma unroll
        for (int f = 0; f < kMaxF; f++)
#pragma unroll
            for (int j = 0; j < kMaxJ; j++) {
                const int c = g + G * j;
                if (c < nc) s += (double)fv[f][j] * vs[f * 64 + c];
            }
    }
    part[t] = s;
    __syncthreads();
    if (t < nc) {
        double a = __ldcg(in + (size_t)t * ld + i);
        for (int q = 0; q < G; q++) a -= part[q * nc + t];
        if (withD)
            tv[t] = a;
        else
            out[(size_t)t * ld + i] = a;
    }
    if (withD) {
        __syncthreads();
        double d = 0.0;
        if (g < G) {
#pragma unroll
            for (int j = 0; j < kMaxJ; j++) {
                const int c = g + G * j;
                if (c < nc) d += (double)dv[j] * tv[c];
            }
        }
        part[t] = d;
        __syncthreads();
        if (t < nc) {
            double a = 0.0;
            for (int q = 0; q < G; q++) a += part[q * nc + t];
            out[(size_t)t * ld + i] = a;
        }
    }
    __syncthreads();  // shared buffers are reused by the next element
}

// the whole application: forward levels (y = L^-1 b), then backward levels (x = U^-1 y)
template <class T>
__global__ void __launch_bounds__(kSweepThreads)
    k_ilu_sweeps(int nc, int nf, int ld, const int* __restrict__ lvlF, const int* __restrict__ ptrF, int nlF,
                 const int* __restrict__ lvlB, const int* __restrict__ ptrB, int nlB, const int4* __restrict__ nbLow,
                 const int4* __restrict__ nbUp, const T* __restrict__ F, const double* b, double* y, double* x) {
    __shared__ double vs[kMaxF * 64];
    __shared__ double part[kSweepThreads];
    __shared__ double tv[kMaxNc];
    cg::grid_group grid = cg::this_grid();
    for (int l = 0; l < nlF; l++) {
        const int q1 = ptrF[l + 1];
        for (int q = ptrF[l] + blockIdx.x; q < q1; q += gridDim.x) {
            const int i = lvlF[q];
            sweep_element<T>(nc, nf, ld, i, nbLow[i], F, false, b, y, y, vs, part, tv);
        }
        grid.sync();
    }
    for (int l = 0; l < nlB; l++) {
        const int q1 = ptrB[l + 1];
        for (int q = ptrB[l] + blockIdx.x; q < q1; q += gridDim.x) {
            const int i = lvlB[q];
            sweep_element<T>(nc, nf, ld, i, nbUp[i], F, true, y, x, x, vs, part, tv);
        }
        if (l + 1 < nlB) grid.sync();
    }
}

// levels, neighbour sets and the per-element factorisation program (host, once per mesh)
int ilu_build(fp_ctx* c) {
    const HostMesh& h = c->hm;
    const int nE = h.nElem, nf = h.nf, ld = h.ld;
    const std::vector<int>& rank = h.rank;
    auto nb = [&](int e, int k) { return h.tt[(size_t)k * ld + e]; };
    std::vector<int> levF(nE, 0), levB(nE, 0);
    for (int r = 0; r < nE; r++) {
        const int i = h.order[r];
        for (int k = 0; k < nf; k++) {
            const int j = nb(i, k);
            if (j > -1 && rank[j] < r) levF[i] = std::max(levF[i], levF[j] + 1);
        }
    }
    for (int r = nE - 1; r >= 0; r--) {
        const int i = h.order[r];
        for (int k = 0; k < nf; k++) {
            const int j = nb(i, k);
            if (j > -1 && rank[j] > r) levB[i] = std::max(levB[i], levB[j] + 1);
        }
    }
    auto group = [&](const std::vector<int>& lev, std::vector<int>& el, std::vector<int>& ptr) {
        const int nl = nE ? *std::max_element(lev.begin(), lev.end()) + 1 : 0;
        ptr.assign(nl + 1, 0);
        for (int e = 0; e < nE; e++) ptr[lev[e] + 1]++;
        for (int l = 0; l < nl; l++) ptr[l + 1] += ptr[l];
        el.assign(nE, 0);
        std::vector<int> pos(ptr.begin(), ptr.end() - 1);
        for (int r = 0; r < nE; r++) el[pos[lev[h.order[r]]]++] = h.order[r];
    };
    std::vector<int> elF, elB;
    group(levF, elF, c->lvlF_ptr);
    group(levB, elB, c->lvlB_ptr);
    std::vector<int4> nbLow(nE), nbUp(nE);
    for (int i = 0; i < nE; i++) {
        int lo[4] = {-1, -1, -1, -1}, up[4] = {-1, -1, -1, -1};
        for (int f = 0; f < nf; f++) {
            const int j = nb(i, f);
            if (j > -1 && rank[j] < rank[i]) lo[f] = j;
            if (j > -1 && rank[j] > rank[i]) up[f] = j;
        }
        nbLow[i] = make_int4(lo[0], lo[1], lo[2], lo[3]);
        nbUp[i] = make_int4(up[0], up[1], up[2], up[3]);
    }
    // factorisation program: per lower neighbour k in rank order an L step, then the
    // updates of every column j > k of row i that row k also has (j = i always)
    std::vector<int> opPtr(nE + 1, 0);
    std::vector<int4> ops;
    for (int i = 0; i < nE; i++) {
        opPtr[i] = (int)ops.size();
        std::vector<std::pair<int, int>> lower;  // (rank, face)
        for (int f = 0; f < nf; f++) {
            const int k = nb(i, f);
            if (k > -1 && rank[k] < rank[i]) lower.push_back({rank[k], f});
        }
        std::sort(lower.begin(), lower.end());
        for (auto& lf : lower) {
            const int f = lf.second, k = nb(i, f);
            ops.push_back(make_int4(0, f, k, 0));
            // columns of row i right of k, in rank order: i itself and its other neighbours
            std::vector<std::pair<int, int>> cols;  // (rank, slot)
            cols.push_back({rank[i], 0});
            for (int g = 0; g < nf; g++) {
                const int j = nb(i, g);
                if (j > -1 && rank[j] > rank[k]) cols.push_back({rank[j], 1 + g});
            }
            std::sort(cols.begin(), cols.end());
            for (auto& cs : cols) {
                const int j = cs.second == 0 ? i : nb(i, cs.second - 1);
                for (int hk = 0; hk < nf; hk++)
                    if (nb(k, hk) == j) {
                        ops.push_back(make_int4(1, cs.second, k, hk));
                        break;
                    }
            }
        }
    }
    opPtr[nE] = (int)ops.size();
    const int nlF = (int)c->lvlF_ptr.size() - 1, nlB = (int)c->lvlB_ptr.size() - 1;
    int rc;
    if ((rc = ialloc(c, &c->d_rank, nE)) || (rc = ialloc(c, &c->d_lvlF, nE)) || (rc = ialloc(c, &c->d_lvlB, nE)) ||
        (rc = ialloc(c, &c->d_opPtr, nE + 1)) || (rc = ialloc(c, &c->d_ops, ops.size())) ||
        (rc = ialloc(c, &c->d_nbLow, nE)) || (rc = ialloc(c, &c->d_nbUp, nE)) || (rc = ialloc(c, &c->d_ptrF, nlF + 1)) ||
        (rc = ialloc(c, &c->d_ptrB, nlB + 1)))
        return rc;
    cudaStream_t s = c->stream;
    auto up = [&](void* d, const void* hsrc, size_t bytes) {
        return cuda_check(c, cudaMemcpyAsync(d, hsrc, bytes, cudaMemcpyHostToDevice, s), "upload");
    };
    if ((rc = up(c->d_rank, rank.data(), nE * sizeof(int))) || (rc = up(c->d_lvlF, elF.data(), nE * sizeof(int))) ||
        (rc = up(c->d_lvlB, elB.data(), nE * sizeof(int))) || (rc = up(c->d_opPtr, opPtr.data(), (nE + 1) * sizeof(int))) ||
        (rc = up(c->d_ops, ops.data(), ops.size() * sizeof(int4))) || (rc = up(c->d_nbLow, nbLow.data(), nE * sizeof(int4))) ||
        (rc = up(c->d_nbUp, nbUp.data(), nE * sizeof(int4))) ||
        (rc = up(c->d_ptrF, c->lvlF_ptr.data(), (nlF + 1) * sizeof(int))) ||
        (rc = up(c->d_ptrB, c->lvlB_ptr.data(), (nlB + 1) * sizeof(int))) ||
        (rc = cuda_check(c, cudaStreamSynchronize(s), "sync")))
        return rc;
    const size_t nF = (size_t)nE * (1 + nf) * c->nc * c->nc;
    if ((rc = ialloc(c, &c->d_iluF64, nF)) || (rc = ialloc(c, &c->d_ilu_y, c->nvec))) return rc;
    if ((rc = cuda_check(c, cudaMemsetAsync(c->d_ilu_y, 0, c->nvec * sizeof(double), s), "memset"))) return rc;
    // persistent sweep grid: every block co-resident (cooperative launch), no more
    // blocks than the widest level
    int dev = 0, nsm = 0, perSm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if ((rc = cuda_check(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_ilu_sweeps<double>, kSweepThreads, 0),
                         "occupancy")))
        return rc;
    int perSm32 = 0;
    if ((rc = cuda_check(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm32, k_ilu_sweeps<float>, kSweepThreads, 0),
                         "occupancy")))
        return rc;
    int widest = 1;
    for (int l = 0; l < nlF; l++) widest = std::max(widest, c->lvlF_ptr[l + 1] - c->lvlF_ptr[l]);
    for (int l = 0; l < nlB; l++) widest = std::max(widest, c->lvlB_ptr[l + 1] - c->lvlB_ptr[l]);
    c->sweep_grid = std::max(1, std::min(widest, nsm * std::min(perSm, perSm32)));
    c->ilu_built = true;
    return FP_OK;
}

}  // namespace

void ilu_release(fp_ctx* c) {
    c->ilu_built = false;
    c->ilu_prec = -1;
    c->d_iluF64 = nullptr;
    c->d_iluF32 = nullptr;
    c->d_rank = c->d_lvlF = c->d_lvlB = c->d_opPtr = c->d_ptrF = c->d_ptrB = nullptr;
    c->d_ops = c->d_nbLow = c->d_nbUp = nullptr;
    c->d_ilu_y = nullptr;
    c->sweep_grid = 0;
    c->lvlF_ptr.clear();
    c->lvlB_ptr.clear();
}

int ilu_factor(fp_ctx* c, int precision) {
    int rc;
    const int nc = c->nc, nf = c->hm.nf, nE = c->hm.nElem, ld = c->hm.ld;
    if (nc > kMaxNc || nf > kMaxF) return set_err(c, FP_ERR_UNSUPPORTED, "block ILU(0): more than 64 unknowns per element");
    const size_t nc2 = (size_t)nc * nc;
    const size_t smem = ((size_t)(1 + nf) * nc2 + nc2 + 2 * nc2) * sizeof(double);
    if (smem > 227 * 1024) return set_err(c, FP_ERR_UNSUPPORTED, "block ILU(0): element blocks exceed shared memory");
    if (!c->ilu_built && (rc = ilu_build(c))) return rc;
    if ((rc = cuda_check(c, cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->stream), "memset"))) return rc;
    dim3 gg((nE + 31) / 32, 1 + nf);
    k_ilu_gather<<<gg, 256, 0, c->stream>>>(nE, ld, nc, nf, c->d_Adiag, c->d_Aneigh, c->d_tt, c->d_iluF64);
    if ((rc = cuda_check(c, cudaGetLastError(), "ILU gather"))) return rc;
    if (smem > 48 * 1024 &&
        (rc = cuda_check(c, cudaFuncSetAttribute(k_ilu_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem")))
        return rc;
    for (size_t l = 0; l + 1 < c->lvlF_ptr.size(); l++) {
        const int n = c->lvlF_ptr[l + 1] - c->lvlF_ptr[l];
        k_ilu_factor<<<n, kFactorThreads, smem, c->stream>>>(nc, nf, c->d_lvlF, c->lvlF_ptr[l], c->d_opPtr, c->d_ops,
                                                            c->d_iluF64, c->d_status);
    }
    if ((rc = cuda_check(c, cudaGetLastError(), "ILU factor"))) return rc;
    if (precision == FP_PREC_FP32) {
        const size_t n = (size_t)nE * (1 + nf) * nc2;
        if (!c->d_iluF32 && (rc = ialloc(c, &c->d_iluF32, n))) return rc;
        k_to_f32<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(n, c->d_iluF64, c->d_iluF32);
        if ((rc = cuda_check(c, cudaGetLastError(), "ILU convert"))) return rc;
    }
    unsigned st = 0;
    if ((rc = cuda_check(c, cudaMemcpyAsync(&st, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream), "copy")) ||
        (rc = cuda_check(c, cudaStreamSynchronize(c->stream), "sync")))
        return rc;
    if (st & FP_DEV_SINGULAR) return set_err(c, FP_ERR_SINGULAR, "singular pivot block in block ILU(0)");
    c->ilu_prec = precision;
    return FP_OK;
}

int ilu_apply(fp_ctx* c, const double* x, double* y) {
    int nc = c->nc, nf = c->hm.nf, ld = c->hm.ld;
    int nlF = (int)c->lvlF_ptr.size() - 1, nlB = (int)c->lvlB_ptr.size() - 1;
    const double* b = x;
    double* yy = c->d_ilu_y;
    double* xx = y;
    cudaError_t e;
    if (c->ilu_prec == FP_PREC_FP32) {
        const float* F = c->d_iluF32;
        void* args[] = {&nc, &nf, &ld, &c->d_lvlF, &c->d_ptrF, &nlF, &c->d_lvlB, &c->d_ptrB, &nlB, &c->d_nbLow, &c->d_nbUp,
                        (void*)&F, (void*)&b, &yy, &xx};
        e = cudaLaunchCooperativeKernel((const void*)k_ilu_sweeps<float>, dim3(c->sweep_grid), dim3(kSweepThreads), args, 0,
                                        c->stream);
    } else {
        const double* F = c->d_iluF64;
        void* args[] = {&nc, &nf, &ld, &c->d_lvlF, &c->d_ptrF, &nlF, &c->d_lvlB, &c->d_ptrB, &nlB, &c->d_nbLow, &c->d_nbUp,
                        (void*)&F, (void*)&b, &yy, &xx};
        e = cudaLaunchCooperativeKernel((const void*)k_ilu_sweeps<double>, dim3(c->sweep_grid), dim3(kSweepThreads), args, 0,
                                        c->stream);
    }
    return cuda_check(c, e, "ILU sweeps");
}

}  // namespace fp
