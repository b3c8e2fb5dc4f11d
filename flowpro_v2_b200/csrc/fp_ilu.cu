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
//   * rows whose lower neighbours are all finished form a level.  The factorisation is
//     ONE persistent cooperative kernel, one 512-thread block per row in shared memory
//     (register-tiled block products, register-resident Gauss-Jordan with implicit
//     partial pivoting); thread blocks take the rows in level order and each row waits
//     (bounded) only for the completion flags of its lower neighbours;
//   * an application (forward L sweep, backward U sweep) is ONE persistent cooperative
//     kernel: thread blocks take the elements in level order, and each element waits
//     (bounded) only for the values of the neighbours it multiplies, which are published
//     with the epoch of the application in every word, so levels overlap and no flag or
//     fence stands between a value and its consumer.  Each element's factor blocks are
//     loaded into registers before the values they multiply arrive;
//   * the factorisation runs in the precision of the factors: FP64, or FP32 for the
//     mixed-precision GMRES, where the blocks are either gathered from the assembled
//     operator (rounded) or written straight into the FP32 factor storage by the exact
//     Jacobian kernel (no FP64 copy of the blocks exists then), and factorised in place.
#include <cuda_pipeline.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "fp_ctx.h"

namespace fp {

namespace {

constexpr int kFactorThreads = 512;
constexpr int kSweepThreads = 512;
constexpr int kMaxNc = 64;   // unknowns per element
constexpr int kMaxF = 4;     // faces per element
constexpr int kMaxJ = 8;     // columns per thread and block in the sweeps: ceil(nc / sweep_group(nc)) <= 8 for nc <= 64

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
template <class T>
__global__ void __launch_bounds__(256) k_ilu_gather(int nElem, int ld, int nc, int nf, const double* __restrict__ Ad,
                                                    const double* __restrict__ An, const int* __restrict__ tt,
                                                    T* __restrict__ F) {
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
            if (e < nElem && o < nc2) F[((size_t)e * (1 + nf) + s) * nc2 + o] = (T)tile[lane][j];
        }
        __syncthreads();
    }
}

// C (-)= X * Y for nc x nc column-major blocks in shared memory (nc <= 64): thread t
// computes the 4 x 4 tile (rows 4 (t % 16) .., columns 4 (t / 16) ..), so each value read
// from shared memory feeds four multiply-adds (the products are bound by shared-memory
// wavefronts, not by the FP64 pipe).
template <class T>
__device__ __forceinline__ void block_mul(int nc, const T* X, const T* Y, T* C, bool subtract) {
    const int t = threadIdx.x;
    const int r0 = 4 * (t & 15), c0 = 4 * (t >> 4);
    if (r0 >= nc || c0 >= nc) return;
    T acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = T(0);
    for (int m = 0; m < nc; m++) {
        T x[4], y[4];
#pragma unroll
        for (int a = 0; a < 4; a++) x[a] = r0 + a < nc ? X[m * nc + r0 + a] : T(0);
#pragma unroll
        for (int b = 0; b < 4; b++) y[b] = c0 + b < nc ? Y[(c0 + b) * nc + m] : T(0);
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int b = 0; b < 4; b++) acc[a][b] += x[a] * y[b];
    }
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
        for (int a = 0; a < 4; a++)
            if (r0 + a < nc && c0 + b < nc) {
                T* cp = C + (c0 + b) * nc + r0 + a;
                if (subtract)
                    *cp -= acc[a][b];
                else
                    *cp = acc[a][b];
            }
}

// Inverse of the nc x nc column-major block A (shared memory) into out (column-major,
// global memory) by Gauss-Jordan on [A | I] with implicit partial pivoting and unscaled
// pivot rows.  Thread (row r = t % 64, column group cg = t / 64) keeps a_r,c for
// c = cg + 8 (k + k0) (k < 16) in registers, where k0 = p / 8 counts the register shifts
// made so far (every 8 steps the array moves down by one, dropping a left-half column
// that is no longer read, so the pivot column always sits in a[0] and no register is
// indexed at run time).  Step p: the owners of column p publish it, every warp finds the
// pivot row br (the unused row with the largest |a_rp|, compared in single precision)
// itself, the owners of row br publish it, and each
// thread updates a_rc -= (a_rp / a_br,p) a_br,c for its c > p.  The published column and
// row are double-buffered, so two barriers per step suffice; columns <= p of the left
// half are left stale.  At the end row stepOfRow^-1(p) holds d_p e_p on the left and d_p
// times row p of inv(A) on the right, d_p its pivot.  512 threads.  A singular block sets
// FP_DEV_SINGULAR in *status and returns false.  T is the arithmetic type (the factors').
template <class T>
__device__ __forceinline__ bool gj_inverse(int nc, const T* A, T* colbuf, T* rowbuf, int* stepOfRow, T* pivOfRow, T* out,
                                           unsigned* status) {
    __shared__ T pivInv[2];
    const int t = threadIdx.x, n2 = 2 * nc;
    const int r = t & 63, cg = t >> 6, lane = t & 31;
    T a[16];
#pragma unroll
    for (int k = 0; k < 16; k++) {
        const int c = cg + 8 * k;
        a[k] = T(0);
        if (r < nc && c < nc) a[k] = A[c * nc + r];
        if (r < nc && c >= nc && c < n2) a[k] = (c - nc == r) ? T(1) : T(0);
    }
    unsigned long long usedMask = 0ull;
    bool singular = false;
    int k0 = 0;
    for (int p = 0; p < nc; p++) {
        T* colp = colbuf + (p & 1) * 64;
        T* rowp = rowbuf + (p & 1) * 128;
        if (cg == (p & 7) && r < nc) colp[r] = a[0];
        __syncthreads();
        // pivot key: the bits of (float)|a_rp| (ordered like unsigned integers for
        // non-negative floats) with the low 6 bits replaced by 63 - r, reduced by one
        // warp-wide unsigned max; ties in the leading 18 bits go to the lowest row
        unsigned key = 0u;
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int rr = lane + 32 * k;
            if (rr < nc && !((usedMask >> rr) & 1ull)) {
                const T v = fabs(colp[rr]);
                unsigned kb = __float_as_uint((float)v) & ~63u;
                if (kb == 0u && v > T(0)) kb = 64u;  // below float range: still a candidate
                if (!isfinite(v)) kb = 0xffffffc0u;
                key = max(key, kb | (unsigned)(63 - rr));
            }
        }
        key = __reduce_max_sync(0xffffffffu, key);
        const int br = 63 - (int)(key & 63u);
        const T bv = br < nc ? fabs(colp[br]) : T(0);
        if (key < 64u || !(bv > T(0)) || !isfinite(bv)) {  // the same decision in every warp
            singular = true;
            break;
        }
        usedMask |= 1ull << br;
        if (r == br) {
#pragma unroll
            for (int k = 0; k < 16; k++) {
                const int c = cg + 8 * (k + k0);
                if (c < n2) rowp[c] = a[k];
            }
        }
        if (t == 0) {
            stepOfRow[br] = p;
            pivOfRow[br] = colp[br];
            pivInv[p & 1] = T(1) / colp[br];
        }
        __syncthreads();
        if (r < nc && r != br) {
            const T m = colp[r] * pivInv[p & 1];
#pragma unroll
            for (int k = 0; k < 16; k++) {
                const int c = cg + 8 * (k + k0);
                if (c > p && c < n2) a[k] -= m * rowp[c];
            }
        }
        if ((p & 7) == 7) {
#pragma unroll
            for (int k = 0; k < 15; k++) a[k] = a[k + 1];
            a[15] = T(0);
            k0++;
        }
    }
    if (singular) {
        if (t == 0) atomicOr(status, (unsigned)FP_DEV_SINGULAR);
        return false;
    }
    __syncthreads();
    // row r holds d times row stepOfRow[r] of the inverse in its right half
    if (r < nc) {
        const int pr = stepOfRow[r];
        const T d = pivOfRow[r];
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const int c = cg + 8 * (k + k0);
            if (c >= nc && c < n2) out[(c - nc) * nc + pr] = a[k] / d;
        }
    }
    return true;
}

// completion flags of the factorisation rows: release by the producer, acquire by the consumers
__device__ __forceinline__ unsigned flag_load(const unsigned* f) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(f) : "memory");
    return v;
}
__device__ __forceinline__ void flag_store(unsigned* f, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(f), "r"(v) : "memory");
}

constexpr int kSpinPolls = 1 << 12;  // polled back to back first (a dependency is usually microseconds away)
// then with 64 ns sleeps up to the context's limit (default 2^19 polls: a wait gives up well
// within a second; a context may lower it, down to 0, so that tests can make a wait run out)

// Bounded wait until *f == epoch.  A wait that runs out sets FP_DEV_TIMEOUT and the abort
// word, which ends every other wait of the launch at once; the results are then garbage
// and the host reports the timeout.
__device__ __forceinline__ void flag_wait(const unsigned* f, unsigned epoch, unsigned* abortw, unsigned* status,
                                          int maxPolls) {
    for (int it = 0; it < maxPolls; it++) {
        if (flag_load(f) == epoch) return;
        if ((it & 31) == 31 && *(volatile unsigned*)abortw) return;
        if (it >= kSpinPolls) __nanosleep(64);
    }
    atomicOr(status, (unsigned)FP_DEV_TIMEOUT);
    atomicExch(abortw, 1u);
}

// The factorisation in one persistent launch: thread block g takes the rows g, g +
// gridDim.x, ... in forward-level order, one 512-thread block per row in shared memory.
// A row's own blocks are requested first (only the row itself changes them); then it
// waits (bounded) for the completion flags of its lower neighbours, whose finished
// blocks it reads, so consecutive levels overlap.  Every dependency lies in an earlier
// level, every block walks its rows in level order and all blocks are co-resident
// (cooperative launch), so each wait ends.  A singular diagonal block sets
// FP_DEV_SINGULAR and still completes its row, so no dependent waits for it.  T: the
// factors' type, in which the factorisation also computes.
template <class T>
__global__ void __launch_bounds__(kFactorThreads)
    k_ilu_factor(int nc, int nf, int nE, const int* __restrict__ lvl, const int4* __restrict__ nbLow,
                 const int* __restrict__ opPtr, const int4* __restrict__ ops, T* F, unsigned* done, unsigned epoch,
                 unsigned* abortw, unsigned* status, int maxPolls, unsigned* sing) {
    extern __shared__ __align__(16) unsigned char ilu_smem[];
    T* sm = reinterpret_cast<T*>(ilu_smem);
    const int nc2 = nc * nc, ns = 1 + nf;
    const int t = threadIdx.x;
    T* R = sm;             // [ns][nc2] the row's blocks
    T* Lb = R + ns * nc2;  // current L block
    T* Yb = Lb + nc2;      // staging of row k's block
    __shared__ T colbuf[2 * kMaxNc], rowbuf[4 * kMaxNc], pivOfRow[kMaxNc];
    __shared__ int stepOfRow[kMaxNc];
    for (int q0 = blockIdx.x; q0 < nE; q0 += gridDim.x) {
        const int i = lvl[q0];
        T* Fi = F + (size_t)i * ns * nc2;
        // global -> shared copies as asynchronous element copies: all of a thread's copies
        // are in flight together instead of one DRAM round trip per loop iteration
        for (int q = t; q < ns * nc2; q += blockDim.x) __pipeline_memcpy_async(R + q, Fi + q, sizeof(T));
        __pipeline_commit();
        if (t < nf) {
            const int4 nb = nbLow[i];
            const int k = t == 0 ? nb.x : t == 1 ? nb.y : t == 2 ? nb.z : nb.w;
            if (k >= 0) flag_wait(done + k, epoch, abortw, status, maxPolls);
        }
        for (int q = opPtr[i]; q < opPtr[i + 1]; q++) {
            const int4 op = ops[q];
            // block of row k: inv(U_kk) for an L step, U_kj for an update
            const T* Y = F + ((size_t)op.z * ns + (op.x == 0 ? 0 : 1 + op.w)) * nc2;
            __syncthreads();
            for (int u = t; u < nc2; u += blockDim.x) __pipeline_memcpy_async(Yb + u, Y + u, sizeof(T));
            __pipeline_commit();
            __pipeline_wait_prior(0);
            __syncthreads();
            if (op.x == 0) {
                // L = A_ik * inv(U_kk)
                block_mul(nc, R + (size_t)(1 + op.y) * nc2, Yb, Lb, false);
                __syncthreads();
                for (int u = t; u < nc2; u += blockDim.x) R[(size_t)(1 + op.y) * nc2 + u] = Lb[u];
            } else {
                // A_ij -= L * U_kj
                block_mul(nc, Lb, Yb, R + (size_t)op.y * nc2, true);
            }
        }
        __pipeline_wait_prior(0);
        __syncthreads();
        // inverse of the updated diagonal block
        if (!gj_inverse(nc, R, colbuf, rowbuf, stepOfRow, pivOfRow, Fi, status) && t == 0) sing[i] = 1u;  // the row's mark
        for (int u = nc2 + t; u < ns * nc2; u += blockDim.x) Fi[u] = R[u];
        __syncthreads();  // the row is written (and the shared buffers are free again)
        if (t == 0) flag_store(done + i, epoch);
    }
}

// Lanes per row in the sweeps: the largest power of two G <= 32 with G nc <= 512, so a
// row's G lanes are adjacent in one warp and meet by shuffles.
__host__ __device__ __forceinline__ int sweep_group(int nc) {
    int G = 32;
    while (G > 1 && G * nc > kSweepThreads) G >>= 1;
    return G;
}

// Factor entries of one sweep element held in registers.  Thread t = G r + g (g < G)
// handles row r of the columns c = g + G j.
template <class T>
struct SweepRegs {
    T fv[kMaxF][kMaxJ];  // blocks 1 + f (L or U)
    T dv[kMaxJ];         // block 0, inv(U_ii) (backward sweep)
    int4 nb;             // neighbours taking part (-1: none)
    int i;               // element, -1: nothing loaded
};

// issue the loads of element i's factor entries (they do not depend on the sweep values,
// so they are in flight while the element waits for its neighbours)
template <class T>
__device__ __forceinline__ void sweep_load(int nc, int nf, int G, const T* __restrict__ F, int i, int4 nbi, bool withD,
                                           SweepRegs<T>& R) {
    const int t = threadIdx.x, nc2 = nc * nc;
    const int r = t / G, g = t - r * G;
    R.i = i;
    R.nb = nbi;
    const int nb[kMaxF] = {R.nb.x, R.nb.y, R.nb.z, R.nb.w};
    const T* Fi = F + (size_t)i * (1 + nf) * nc2;
#pragma unroll
    for (int f = 0; f < kMaxF; f++)
#pragma unroll
        for (int j = 0; j < kMaxJ; j++) {
            const int c = g + G * j;
            R.fv[f][j] = (r < nc && f < nf && nb[f] >= 0 && c < nc) ? Fi[(size_t)(1 + f) * nc2 + (size_t)c * nc + r] : T(0);
        }
    if (withD) {
#pragma unroll
        for (int j = 0; j < kMaxJ; j++) {
            const int c = g + G * j;
            R.dv[j] = (r < nc && c < nc) ? Fi[(size_t)c * nc + r] : T(0);
        }
    }
}

// sum over the G adjacent lanes of a row (every lane of the warp takes part)
__device__ __forceinline__ double group_sum(double v, int G) {
    for (int o = G >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sweep values are published element-major with the epoch of the application: word
// (i, c, h) holds half h (0 low, 1 high) of value c of element i in its low 32 bits and
// the epoch in its high 32 bits.  A consumer polls the words themselves, so a value is
// usable as soon as its own word is, with no completion flag and no release fence (an
// aligned 64-bit store is seen whole or not at all).
__device__ __forceinline__ unsigned long long pub_load(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void pub_store(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Bounded wait for one published word of this epoch; returns its payload.  A wait that
// runs out sets FP_DEV_TIMEOUT and the abort word, which ends every other wait of the
// launch at once; the sweep values are then garbage and the host reports the timeout.
__device__ __forceinline__ unsigned pub_wait(const unsigned long long* p, unsigned epoch, unsigned* abortw,
                                             unsigned* status, int maxPolls) {
    for (int it = 0; it < maxPolls; it++) {
        const unsigned long long v = pub_load(p);
        if ((unsigned)(v >> 32) == epoch) return (unsigned)v;
        if ((it & 31) == 31 && *(volatile unsigned*)abortw) return 0u;
        if (it >= kSpinPolls) __nanosleep(64);
    }
    atomicOr(status, (unsigned)FP_DEV_TIMEOUT);
    atomicExch(abortw, 1u);
    return 0u;
}

// The whole application in one persistent launch over the sweep program: position v <
// nE is the forward sweep (y = L^-1 b) in forward-level order, v >= nE the backward sweep
// (x = U^-1 y) in backward-level order; swEl[v] is the element at position v and swNb[v]
// the neighbours it multiplies (lower, then upper; -1 none).  Thread block g takes the
// positions g, g + gridDim.x, ... of each sweep.  An element waits only for the published
// values it multiplies (the neighbours' and, in the backward sweep, its own forward
// value), so consecutive levels overlap.  Every dependency lies in an earlier level,
// every block walks its positions in level order and all blocks are co-resident
// (cooperative launch), so each wait ends.  The block's next element is known one element
// ahead, so its factor entries are requested right after the current values are published.
//
// One element: thread t = 128 f + 2 c + h fetches half h of value c of the neighbour over
// face f into shared memory; thread t = G r + g forms the partial sums of row r over the
// columns g + G j (one per face, so the chains are short), the G lanes of the row add
// them by shuffles and out_i = in_i - sum_f B_f v_f, then, backward, out_i = inv(U_ii)
// (that).  The shared buffers alternate between consecutive elements, so one barrier
// (two backward) per element suffices.
__device__ __forceinline__ int sweep_next(int v, int nE) {
    const int w = v + (int)gridDim.x;
    if (v < nE) return w < nE ? w : nE + (int)blockIdx.x;  // the first backward position after the last forward one
    return w;
}

template <class T>
__global__ void __launch_bounds__(kSweepThreads)
    k_ilu_sweeps(int nc, int nf, int ld, int nE, const int* __restrict__ swEl, const int4* __restrict__ swNb,
                 const T* __restrict__ F, const double* __restrict__ b, double* __restrict__ x, unsigned long long* pubF,
                 unsigned long long* pubB, unsigned epoch, unsigned* abortw, unsigned* status, int maxPolls) {
    __shared__ double vsb[2][kMaxF * 64];  // the neighbours' values
    __shared__ double yob[2][kMaxNc];      // backward: the element's forward value
    __shared__ double tvb[2][kMaxNc];      // backward: value before inv(U_ii)
    const int t = threadIdx.x, G = sweep_group(nc);
    const int r = t / G, g = t - r * G;
    const int nV = 2 * nE;
    SweepRegs<T> R;
    int v = blockIdx.x;
    if (v >= nE) return;
    sweep_load<T>(nc, nf, G, F, swEl[v], swNb[v], false, R);
    int v1 = sweep_next(v, nE);
    int i1 = v1 < nV ? swEl[v1] : -1;
    int4 nb1 = v1 < nV ? swNb[v1] : make_int4(-1, -1, -1, -1);
    int par = 0;
    while (v < nV) {
        const bool bwd = v >= nE;
        unsigned long long* pub = bwd ? pubB : pubF;  // the neighbours' values and this element's
        double* vs = vsb[par];
        double* yo = yob[par];
        double* tv = tvb[par];
        const int i = R.i;
        const double a_in = (!bwd && g < 2 && r < nc) ? __ldcg(b + (size_t)r * ld + i) : 0.0;  // the two publishing lanes
        // factor entries in double before the wait (a no-op for FP64 factors)
        double fv[kMaxF][kMaxJ], dv[kMaxJ];
#pragma unroll
        for (int f = 0; f < kMaxF; f++)
#pragma unroll
            for (int j = 0; j < kMaxJ; j++) fv[f][j] = (double)R.fv[f][j];
#pragma unroll
        for (int j = 0; j < kMaxJ; j++) dv[j] = bwd ? (double)R.dv[j] : 0.0;
        {
            const int f = t >> 7, c = (t >> 1) & 63, h = t & 1;
            const int n = f == 0 ? R.nb.x : f == 1 ? R.nb.y : f == 2 ? R.nb.z : R.nb.w;
            unsigned w = 0u;
            if (f < nf && n >= 0 && c < nc) w = pub_wait(pub + ((size_t)n * nc + c) * 2 + h, epoch, abortw, status, maxPolls);
            reinterpret_cast<unsigned*>(vs)[t] = w;
        }
        if (bwd && t < 2 * nc)
            reinterpret_cast<unsigned*>(yo)[t] = pub_wait(pubF + (size_t)i * nc * 2 + t, epoch, abortw, status, maxPolls);
        __syncthreads();
        double sf[kMaxF];
#pragma unroll
        for (int f = 0; f < kMaxF; f++) {
            sf[f] = 0.0;
#pragma unroll
            for (int j = 0; j < kMaxJ; j++) {
                const int c = g + G * j;
                if (c < nc) sf[f] += fv[f][j] * vs[f * 64 + c];
            }
        }
        const double s = group_sum((sf[0] + sf[1]) + (sf[2] + sf[3]), G);
        double a;
        if (!bwd) {
            a = a_in - s;
        } else {
            if (g == 0 && r < nc) tv[r] = yo[r] - s;
            __syncthreads();
            double d = 0.0;
#pragma unroll
            for (int j = 0; j < kMaxJ; j++) {
                const int c = g + G * j;
                if (c < nc) d += dv[j] * tv[c];
            }
            a = group_sum(d, G);
            if (g == 0 && r < nc) x[(size_t)r * ld + i] = a;
        }
        if (g < 2 && r < nc) {
            const unsigned long long e = (unsigned long long)epoch << 32;
            pub_store(pub + ((size_t)i * nc + r) * 2 + g, e | (unsigned)(g == 0 ? __double2loint(a) : __double2hiint(a)));
        }
        // the next element's factor entries, then the element after it
        if (v1 < nV) sweep_load<T>(nc, nf, G, F, i1, nb1, v1 >= nE, R);
        v = v1;
        v1 = v < nV ? sweep_next(v, nE) : nV;
        if (v1 < nV) {
            i1 = swEl[v1];
            nb1 = swNb[v1];
        }
        par ^= 1;
    }
}

// ---------------------------------------------------------------------------- bulk-copy sweeps
// The same application with the factor blocks staged in shared memory by bulk asynchronous
// copies (the TMA engine's cp.async.bulk, one instruction per block, completion counted in
// bytes on an mbarrier) up to S positions ahead.  An element's blocks are contiguous in the
// element-major factor storage (F[e][s], nc * nc values each), so thread 0 requests exactly the
// blocks the position multiplies (forward: the lower neighbours' L blocks; backward: the upper
// neighbours' U blocks and inv(U_ii)) into slot k % S and the block's threads read them from
// shared memory when the position's turn comes.  A slot is refilled as soon as the barrier of
// the next position shows every thread done with it, and the program entries are loaded a
// position ahead, so one barrier per forward position (two backward) is on the path.  One block per SM holds S slots of (1 + nf)
// blocks; the per-position arithmetic is the register kernel's, in the same order, so both give
// identical results.  Needs nc * nc * sizeof(T) to be a multiple of 16 bytes (bulk-copy size and
// address alignment).
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// global -> shared bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned),
// completing on bar; no cluster multicast
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

constexpr int kBulkPolls = 1 << 22;  // a bulk copy from device memory completes within microseconds

// Bounded wait for phase `parity` of bar.  A wait that runs out sets FP_DEV_TIMEOUT and the
// abort word and returns false.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, unsigned* abortw, unsigned* status) {
    for (int it = 0; it < kBulkPolls; it++)
        if (mbar_try_wait(bar, parity)) return true;
    atomicOr(status, (unsigned)FP_DEV_TIMEOUT);
    atomicExch(abortw, 1u);
    return false;
}

// thread 0: request the blocks the position of element i with neighbours nbv multiplies into
// slot (forward: the neighbours' blocks 1 + f; backward: those and block 0)
// (skip: an arrival without bytes, which completes the slot's phase at once)
template <class T>
__device__ __forceinline__ void sweep_request(bool bwd, int i, int4 nbv, int nc2, int nf, const T* __restrict__ F, T* slot,
                                              unsigned long long* bar, bool skip) {
    if (skip) {
        mbar_expect_tx(bar, 0u);
        return;
    }
    const int nb[kMaxF] = {nbv.x, nbv.y, nbv.z, nbv.w};
    const unsigned bb = (unsigned)(nc2 * sizeof(T));
    unsigned bytes = bwd ? bb : 0u;
    for (int f = 0; f < nf; f++)
        if (nb[f] >= 0) bytes += bb;
    mbar_expect_tx(bar, bytes);
    const T* src = F + (size_t)i * (1 + nf) * nc2;
    if (bwd) bulk_load(slot, src, bb, bar);
    for (int f = 0; f < nf; f++)
        if (nb[f] >= 0) bulk_load(slot + (size_t)(1 + f) * nc2, src + (size_t)(1 + f) * nc2, bb, bar);
}

// barrier of the threads of group grp: a warp-wide sync for one-warp groups, else named
// barrier 1 + grp (ids 1 .. 8; 0 is __syncthreads)
__device__ __forceinline__ void group_sync(int grp, int nthreads) {
    if (nthreads == 32)
        __syncwarp();
    else
        asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "r"(nthreads) : "memory");
}

// Most groups per block of the staged sweep for nc unknowns per element (16 one-warp groups
// for nc <= 16, 8 for nc <= 32, else 4), and the lanes per row that go with it: a power of two,
// adjacent in one warp, such that a row set fits a group of the most groups.  The lane split
// depends on nc alone, so the sums, and the results, do not depend on the group count.  It is
// at least 2 for every nc up to kMaxNc: lanes 0 and 1 of a row publish the two halves of its
// value.
constexpr __host__ __device__ int sweep_max_groups(int nc) { return nc <= 16 ? 16 : nc <= 32 ? 8 : 4; }
constexpr __host__ __device__ int sweep_row_lanes(int nc) {
    const int lim = kSweepThreads / sweep_max_groups(nc);
    int G = 32;
    while (G > 1 && G * nc > lim) G >>= 1;
    return G;
}
constexpr bool sweep_lanes_publish(int nc) { return nc > kMaxNc || (sweep_row_lanes(nc) >= 2 && sweep_lanes_publish(nc + 1)); }
static_assert(sweep_lanes_publish(1), "every row of the staged sweep needs two lanes up to kMaxNc unknowns");

// k-th position of this block's sequence: forward b, b + GB, ... (< nE), then backward
// nE + b, nE + b + GB, ... (GB = gridDim.x); nV past the end
__device__ __forceinline__ int block_position(int k, int nE) {
    const int b = (int)blockIdx.x, GB = (int)gridDim.x;
    const int Jf = b < nE ? (nE - 1 - b) / GB + 1 : 0;
    if (k < Jf) return b + k * GB;
    const int v = nE + b + (k - Jf) * GB;
    return v < 2 * nE ? v : 2 * nE;
}

// The block's 512 threads form NG groups of 512 / NG threads; group g takes the positions
// k = g, g + NG, ... of the block's sequence, so NG positions are in flight per block, each
// group synchronising on its own barrier.  Slot k % S holds position k's factor blocks;
// S is a multiple of NG, so a slot always serves the same group, whose leader refills it with
// position k + S as soon as the group is done with position k.  With live flags (batched cases:
// caseOf, live non-null), the positions of a case whose flag is 0 only keep the slot rotation
// (no copy, no wait on neighbours, no value published); no position of another case depends on
// them.  Dynamic shared memory: the
// S slots, their S mbarriers, then per group (of sweep_max_groups(nc)) the neighbours' values
// (nf * nc), the element's forward value and its value before inv(U_ii) (nc each).
template <class T>
__global__ void __launch_bounds__(kSweepThreads, 2)
    k_ilu_sweeps_bulk(int nc, int nf, int ld, int nE, int S, int NG, const int* __restrict__ swEl,
                      const int4* __restrict__ swNb, const T* __restrict__ F, const double* __restrict__ b,
                      double* __restrict__ x, unsigned long long* pubF, unsigned long long* pubB, unsigned epoch,
                      unsigned* abortw, unsigned* status, int maxPolls, const int* __restrict__ caseOf,
                      const int* __restrict__ live) {
    extern __shared__ __align__(128) unsigned char sweep_smem[];
    const int nc2 = nc * nc, ns = 1 + nf;
    T* slots = reinterpret_cast<T*>(sweep_smem);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(sweep_smem + (size_t)S * ns * nc2 * sizeof(T));
    __shared__ int failed[16];
    const int GT = kSweepThreads / NG;  // threads of a group
    const int grp = threadIdx.x / GT, t = threadIdx.x - grp * GT;
    const int G = sweep_row_lanes(nc);
    const int r = t / G, g = t - r * G;
    const int nV = 2 * nE;
    if ((int)blockIdx.x >= nE) return;
    if (threadIdx.x == 0) {
        for (int q = 0; q < S; q++) mbar_init(bars + q, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (t == 0) failed[grp] = 0;
    __syncthreads();
    double* vs = reinterpret_cast<double*>(bars + S) + (size_t)grp * (nf + 2) * nc;  // [nf][nc]
    double* yo = vs + (size_t)nf * nc;
    double* tv = yo + nc;
    // the group leader requests its positions grp, grp + NG, ... below S
    int kq = grp;  // next sequence index to request (leader)
    if (t == 0) {
        for (; kq < S; kq += NG) {
            const int vq = block_position(kq, nE);
            if (vq >= nV) break;
            const int iq = swEl[vq];
            sweep_request<T>(vq >= nE, iq, swNb[vq], nc2, nf, F, slots + (size_t)(kq % S) * ns * nc2, bars + kq % S,
                             live && !live[caseOf[iq]]);
        }
    }
    int k = grp;
    int v = block_position(k, nE);
    int i_cur = v < nV ? swEl[v] : 0;
    int4 nb_cur = v < nV ? swNb[v] : make_int4(-1, -1, -1, -1);
    while (v < nV) {
        const int q = k % S;
        const bool bwd = v >= nE;
        const T* Fs = slots + (size_t)q * ns * nc2;
        const int i = i_cur;
        const int4 nbv = nb_cur;
        const int vn = block_position(k + NG, nE);
        if (vn < nV) {  // the group's next program entry, in flight during this position
            i_cur = swEl[vn];
            nb_cur = swNb[vn];
        }
        unsigned long long* pub = bwd ? pubB : pubF;  // the neighbours' values and this element's
        const bool skip = live && !live[caseOf[i]];  // the same for the whole group
        const double a_in = (!skip && !bwd && g < 2 && r < nc) ? __ldcg(b + (size_t)r * ld + i) : 0.0;  // the two publishing lanes
        // word u: half u & 1 of value (u / 2) mod nc of neighbour f = u / (2 nc); each thread's
        // words go four at a time, their first loads in flight together, and only a word not
        // yet of this epoch is polled again
        const int nw = skip ? 0 : nf * nc * 2;
        for (int u0 = t; u0 < nw; u0 += 4 * GT) {
            const unsigned long long* pp[4];
            unsigned long long pv[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int u = u0 + q * GT;
                pp[q] = nullptr;
                if (u < nw) {
                    const int f = u / (2 * nc), cw = u - f * 2 * nc;
                    const int n = f == 0 ? nbv.x : f == 1 ? nbv.y : f == 2 ? nbv.z : nbv.w;
                    if (n >= 0) pp[q] = pub + (size_t)n * nc * 2 + cw;
                }
            }
#pragma unroll
            for (int q = 0; q < 4; q++) pv[q] = pp[q] ? pub_load(pp[q]) : 0ull;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int u = u0 + q * GT;
                if (u < nw) {
                    unsigned w = 0u;
                    if (pp[q])
                        w = (unsigned)(pv[q] >> 32) == epoch ? (unsigned)pv[q] : pub_wait(pp[q], epoch, abortw, status, maxPolls);
                    reinterpret_cast<unsigned*>(vs)[u] = w;
                }
            }
        }
        if (bwd && !skip)
            for (int u = t; u < 2 * nc; u += GT)
                reinterpret_cast<unsigned*>(yo)[u] = pub_wait(pubF + (size_t)i * nc * 2 + u, epoch, abortw, status, maxPolls);
        // the position's factor blocks have arrived in slot q
        if (!mbar_wait(bars + q, (unsigned)((k / S) & 1), abortw, status)) failed[grp] = 1;
        group_sync(grp, GT);
        if (failed[grp]) break;
        if (!skip) {
            const int nb[kMaxF] = {nbv.x, nbv.y, nbv.z, nbv.w};
            double sf[kMaxF];
#pragma unroll
            for (int f = 0; f < kMaxF; f++) {
                sf[f] = 0.0;
                if (f < nf && nb[f] >= 0 && r < nc) {
                    const T* Bf = Fs + (size_t)(1 + f) * nc2;
                    for (int c = g; c < nc; c += G) sf[f] += (double)Bf[c * nc + r] * vs[f * nc + c];
                }
            }
            const double s = group_sum((sf[0] + sf[1]) + (sf[2] + sf[3]), G);
            double a;
            if (!bwd) {
                a = a_in - s;
            } else {
                if (g == 0 && r < nc) tv[r] = yo[r] - s;
                group_sync(grp, GT);
                double d = 0.0;
                if (r < nc)
                    for (int c = g; c < nc; c += G) d += (double)Fs[c * nc + r] * tv[c];
                a = group_sum(d, G);
                if (g == 0 && r < nc) x[(size_t)r * ld + i] = a;
            }
            if (g < 2 && r < nc) {
                const unsigned long long e = (unsigned long long)epoch << 32;
                pub_store(pub + ((size_t)i * nc + r) * 2 + g, e | (unsigned)(g == 0 ? __double2loint(a) : __double2hiint(a)));
            }
        }
        // the group is done with slot q: it takes the group's position S ahead
        group_sync(grp, GT);
        if (t == 0) {
            const int vq = block_position(kq, nE);
            if (vq < nV) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                const int iq = swEl[vq];
                sweep_request<T>(vq >= nE, iq, swNb[vq], nc2, nf, F, slots + (size_t)q * ns * nc2, bars + q,
                                 live && !live[caseOf[iq]]);
                kq += NG;
            }
        }
        v = vn;
        k += NG;
    }
    // after a failed copy wait: let the group's copies still in flight land before the block exits
    if (t == 0 && failed[grp]) {
        for (int kk = k; kk < kq; kk += NG) {
            unsigned long long* bar = bars + kk % S;
            for (int it = 0; it < kBulkPolls && !mbar_try_wait(bar, (unsigned)((kk / S) & 1)); it++) {
            }
        }
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
    // sweep program: forward positions, then backward positions
    std::vector<int> swEl(2 * (size_t)nE);
    std::vector<int4> swNb(2 * (size_t)nE);
    for (int q = 0; q < nE; q++) {
        swEl[q] = elF[q];
        swNb[q] = nbLow[elF[q]];
        swEl[nE + q] = elB[q];
        swNb[nE + q] = nbUp[elB[q]];
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
    int rc;
    if ((rc = ialloc(c, &c->d_rank, nE)) || (rc = ialloc(c, &c->d_lvlF, nE)) ||
        (rc = ialloc(c, &c->d_opPtr, nE + 1)) || (rc = ialloc(c, &c->d_ops, ops.size())) ||
        (rc = ialloc(c, &c->d_nbLow, nE)) || (rc = ialloc(c, &c->d_swEl, 2 * (size_t)nE)) ||
        (rc = ialloc(c, &c->d_swNb, 2 * (size_t)nE)) ||
        (rc = ialloc(c, &c->d_iluFlags, 2 + (size_t)nE)) || (rc = ialloc(c, &c->d_ilu_pub, 4 * (size_t)nE * c->nc)) ||
        (rc = ialloc(c, &c->d_ilu_sing, (size_t)nE)))
        return rc;
    cudaStream_t s = c->stream;
    auto up = [&](void* d, const void* hsrc, size_t bytes) {
        return cuda_check(c, cudaMemcpyAsync(d, hsrc, bytes, cudaMemcpyHostToDevice, s), "upload");
    };
    if ((rc = up(c->d_rank, rank.data(), nE * sizeof(int))) || (rc = up(c->d_lvlF, elF.data(), nE * sizeof(int))) ||
        (rc = up(c->d_opPtr, opPtr.data(), (nE + 1) * sizeof(int))) ||
        (rc = up(c->d_ops, ops.data(), ops.size() * sizeof(int4))) || (rc = up(c->d_nbLow, nbLow.data(), nE * sizeof(int4))) ||
        (rc = up(c->d_swEl, swEl.data(), 2 * (size_t)nE * sizeof(int))) ||
        (rc = up(c->d_swNb, swNb.data(), 2 * (size_t)nE * sizeof(int4))) ||
        (rc = cuda_check(c, cudaMemsetAsync(c->d_iluFlags, 0, (2 + (size_t)nE) * sizeof(unsigned), s), "memset")) ||
        (rc = cuda_check(c, cudaMemsetAsync(c->d_ilu_pub, 0, 4 * (size_t)nE * c->nc * sizeof(unsigned long long), s),
                         "memset")) ||
        (rc = cuda_check(c, cudaStreamSynchronize(s), "sync")))
        return rc;
    // persistent sweep grid: every block co-resident (cooperative launch)
    int dev = 0, nsm = 0, perSm = 0, perSm32 = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if ((rc = cuda_check(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_ilu_sweeps<double>, kSweepThreads, 0),
                         "occupancy")) ||
        (rc = cuda_check(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm32, k_ilu_sweeps<float>, kSweepThreads, 0),
                         "occupancy")))
        return rc;
    c->sweep_grid = std::max(1, std::min(nE, nsm * std::max(1, std::min(perSm, perSm32))));
    c->ilu_epoch = 0;
    c->ilu_fepoch = 0;
    c->ilu_built = true;
    return FP_OK;
}

// factor storage of one precision, allocated on first use (the full 3D p = 2 case holds
// 69 GB of FP64 or 35 GB of FP32 factors, so only the precision in use exists)
template <class T>
int ilu_storage(fp_ctx* c, T** out);
template <>
int ilu_storage<double>(fp_ctx* c, double** out) {
    int rc;
    if (!c->d_iluF64 && (rc = ialloc(c, &c->d_iluF64, (size_t)c->hm.nElem * (1 + c->hm.nf) * c->nc * c->nc))) return rc;
    *out = c->d_iluF64;
    return FP_OK;
}
template <>
int ilu_storage<float>(fp_ctx* c, float** out) {
    int rc;
    if (!c->d_iluF32 && (rc = ialloc(c, &c->d_iluF32, (size_t)c->hm.nElem * (1 + c->hm.nf) * c->nc * c->nc))) return rc;
    *out = c->d_iluF32;
    return FP_OK;
}

int ilu_check_sizes(fp_ctx* c) {
    if (c->nc > kMaxNc || c->hm.nf > kMaxF)
        return set_err(c, FP_ERR_UNSUPPORTED, "block ILU(0): more than 64 unknowns per element");
    const size_t nc2 = (size_t)c->nc * c->nc;
    if (((size_t)(1 + c->hm.nf) * nc2 + 2 * nc2) * sizeof(double) > 227 * 1024)
        return set_err(c, FP_ERR_UNSUPPORTED, "block ILU(0): element blocks exceed shared memory");
    return FP_OK;
}

// the persistent factorisation of the blocks already in F (T precision), in place
template <class T>
int ilu_factor_run(fp_ctx* c, T* F) {
    int rc;
    const int nc = c->nc, nf = c->hm.nf, nE = c->hm.nElem;
    const size_t nc2 = (size_t)nc * nc;
    const size_t smem = ((size_t)(1 + nf) * nc2 + 2 * nc2) * sizeof(T);
    if ((rc = cuda_check(c, cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->stream), "memset"))) return rc;
    if (smem > 48 * 1024 &&
        (rc = cuda_check(c, cudaFuncSetAttribute(k_ilu_factor<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                         "smem")))
        return rc;
    // persistent factorisation grid: every block co-resident (cooperative launch)
    int dev = 0, nsm = 0, perSm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if ((rc = cuda_check(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_ilu_factor<T>, kFactorThreads, smem),
                         "occupancy")))
        return rc;
    if (perSm < 1) return set_err(c, FP_ERR_UNSUPPORTED, "block ILU(0): factorisation block does not fit an SM");
    unsigned* abortw = c->d_iluFlags;
    unsigned* done = c->d_iluFlags + 2;
    unsigned epoch = ++c->ilu_fepoch;
    if (epoch == 0) {  // wrapped: clear the row flags and start again
        if ((rc = cuda_check(c, cudaMemsetAsync(done, 0, (size_t)nE * sizeof(unsigned), c->stream), "memset"))) return rc;
        epoch = c->ilu_fepoch = 1;
    }
    int nEl = nE, ncl = nc, nfl = nf, polls = c->ilu_max_polls;
    unsigned* status = c->d_status;
    unsigned* sing = c->d_ilu_sing;
    if ((rc = cuda_check(c, cudaMemsetAsync(sing, 0, (size_t)nE * sizeof(unsigned), c->stream), "memset"))) return rc;
    void* args[] = {&ncl, &nfl, &nEl, &c->d_lvlF, &c->d_nbLow, &c->d_opPtr, &c->d_ops, &F, &done, &epoch, &abortw,
                    &status, &polls, &sing};
    const int grid = std::max(1, std::min(nE, nsm * perSm));
    if ((rc = cuda_check(c,
                         cudaLaunchCooperativeKernel((const void*)k_ilu_factor<T>, dim3(grid), dim3(kFactorThreads), args,
                                                     smem, c->stream),
                         "ILU factor")))
        return rc;
    unsigned st = 0;
    if ((rc = cuda_check(c, cudaMemcpyAsync(&st, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream), "copy")) ||
        (rc = cuda_check(c, cudaStreamSynchronize(c->stream), "sync")))
        return rc;
    if (st & FP_DEV_TIMEOUT) {
        cudaMemsetAsync(abortw, 0, sizeof(unsigned), c->stream);
        c->ilu_prec = -1;
        return set_err(c, FP_ERR_TIMEOUT, "block ILU(0) factorisation: a dependency wait gave up");
    }
    if (st & FP_DEV_SINGULAR) {
        c->ilu_prec = -1;
        return set_err(c, FP_ERR_SINGULAR, "singular pivot block in block ILU(0)");
    }
    return FP_OK;
}

template <class T>
int ilu_factor_t(fp_ctx* c, bool gather) {
    int rc;
    T* F = nullptr;
    if ((rc = ilu_storage<T>(c, &F))) return rc;
    if (gather) {
        if (!c->d_Adiag) return set_err(c, FP_ERR_STATE, "block ILU(0): no assembled blocks");
        const int nc = c->nc, nf = c->hm.nf, nE = c->hm.nElem, ld = c->hm.ld;
        dim3 gg((nE + 31) / 32, 1 + nf);
        k_ilu_gather<T><<<gg, 256, 0, c->stream>>>(nE, ld, nc, nf, c->d_Adiag, c->d_Aneigh, c->d_tt, F);
        if ((rc = cuda_check(c, cudaGetLastError(), "ILU gather"))) return rc;
    }
    return ilu_factor_run<T>(c, F);
}

}  // namespace

void ilu_release(fp_ctx* c) {
    c->ilu_built = false;
    c->ilu_prec = -1;
    c->d_iluF64 = nullptr;
    c->d_iluF32 = nullptr;
    c->d_rank = c->d_lvlF = c->d_opPtr = nullptr;
    c->d_iluFlags = nullptr;
    c->d_ilu_sing = nullptr;
    c->ilu_epoch = 0;
    c->ilu_fepoch = 0;
    c->d_ops = c->d_nbLow = c->d_swNb = nullptr;
    c->d_swEl = nullptr;
    c->d_ilu_pub = nullptr;
    c->sweep_grid = 0;
    c->sweep_bulk_grid[0] = c->sweep_bulk_grid[1] = -1;

    c->lvlF_ptr.clear();
    c->lvlB_ptr.clear();
}


int ilu_factor(fp_ctx* c, int precision) {
    int rc;
    if ((rc = ilu_check_sizes(c))) return rc;
    if (!c->ilu_built && (rc = ilu_build(c))) return rc;
    rc = precision == FP_PREC_FP32 ? ilu_factor_t<float>(c, true) : ilu_factor_t<double>(c, true);
    if (rc) return rc;
    c->ilu_prec = precision;
    return FP_OK;
}

int ilu_prepare_direct(fp_ctx* c, int precision, void** F) {
    int rc;
    if ((rc = ilu_check_sizes(c))) return rc;
    if (!c->ilu_built && (rc = ilu_build(c))) return rc;
    c->ilu_prec = -1;  // the storage is about to be overwritten
    if (precision == FP_PREC_FP32) {
        float* p = nullptr;
        rc = ilu_storage<float>(c, &p);
        *F = p;
    } else {
        double* p = nullptr;
        rc = ilu_storage<double>(c, &p);
        *F = p;
    }
    return rc;
}

int ilu_factor_direct(fp_ctx* c, int precision) {
    int rc = precision == FP_PREC_FP32 ? ilu_factor_run<float>(c, c->d_iluF32) : ilu_factor_run<double>(c, c->d_iluF64);
    if (rc) return rc;
    c->ilu_prec = precision;
    return FP_OK;
}

// bulk-copy sweep configuration of factor type T: slots per block, grid, dynamic shared
// memory (grid 0: the register kernel is used)
// slots per block, grid and dynamic shared memory of the bulk-copy sweep for factor type T
// (grid 0: the register kernel is used)
template <class T>
int bulk_sweep_config(fp_ctx* c, int* S_out, int* grid_out, size_t* smem_out) {
    const size_t nc2 = (size_t)c->nc * c->nc, ns = 1 + c->hm.nf;
    *grid_out = 0;
    if ((nc2 * sizeof(T)) % 16 != 0 || c->nc > kSweepThreads / 4) return FP_OK;
    if (sweep_row_lanes(c->nc) < 2) return FP_OK;  // a row's value is published by two lanes
    const size_t slot = ns * nc2 * sizeof(T);
    // slot budget: 208 KB (one block per SM) for large blocks, 100 KB (two blocks per SM, the
    // register limit of __launch_bounds__) for nc <= 32
    const size_t budget = (c->nc > 32 ? 208 : 100) * 1024;
    int S = (int)std::min<size_t>(32, budget / slot);
    if (S < 2) return FP_OK;
    int p = 2;  // S: a multiple of the largest power of two up to the group limit that fits
    while (2 * p <= std::min(S, sweep_max_groups(c->nc))) p *= 2;
    S -= S % p;
    const size_t smem = (size_t)S * slot + (size_t)S * sizeof(unsigned long long) +
                        (size_t)sweep_max_groups(c->nc) * (ns + 1) * c->nc * sizeof(double);
    int rc;
    if ((rc = cuda_check(c, cudaFuncSetAttribute(k_ilu_sweeps_bulk<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                         "smem")))
        return rc;
    int dev = 0, nsm = 0, perSm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if ((rc = cuda_check(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_ilu_sweeps_bulk<T>, kSweepThreads, smem),
                         "occupancy")))
        return rc;
    if (perSm < 1) return FP_OK;
    *S_out = S;
    *grid_out = std::max(1, std::min(c->hm.nElem, nsm * perSm));
    *smem_out = smem;
    return FP_OK;
}

template <class T>
int launch_sweeps(fp_ctx* c, const T* F, const double* b, double* xx, unsigned epoch) {
    int nc = c->nc, nf = c->hm.nf, ld = c->hm.ld, nE = c->hm.nElem;
    unsigned long long* pubF = c->d_ilu_pub;
    unsigned long long* pubB = c->d_ilu_pub + 2 * (size_t)nE * nc;
    unsigned* abortw = c->d_iluFlags;
    unsigned* status = abortw + 1;
    int polls = c->ilu_max_polls;
    const int pi = sizeof(T) == sizeof(float) ? 1 : 0;
    if (c->sweep_bulk_grid[pi] < 0) {
        int S = 0, grid = 0;
        size_t smem = 0;
        int rc = bulk_sweep_config<T>(c, &S, &grid, &smem);
        if (rc) return rc;
        c->sweep_bulk_S[pi] = S;
        c->sweep_bulk_NG[pi] = 0;  // groups per block: chosen by timing at the first application
        c->sweep_bulk_grid[pi] = grid;
        c->sweep_bulk_smem[pi] = smem;
    }
    auto launch_bulk = [&](int NG) {
        int S = c->sweep_bulk_S[pi];
        const int* caseOf = c->batch_mask ? c->d_case_of : nullptr;
        const int* live = c->batch_mask ? c->d_blive : nullptr;
        void* args[] = {&nc, &nf, &ld, &nE, &S, &NG, &c->d_swEl, &c->d_swNb, (void*)&F, (void*)&b, &xx, &pubF, &pubB,
                        &epoch, &abortw, &status, &polls, (void*)&caseOf, (void*)&live};
        return cudaLaunchCooperativeKernel((const void*)k_ilu_sweeps_bulk<T>, dim3(c->sweep_bulk_grid[pi]),
                                           dim3(kSweepThreads), args, c->sweep_bulk_smem[pi], c->stream);
    };
    if (c->sweep_variant >= 2 && c->sweep_bulk_grid[pi] > 0) {  // a fixed group count: 2 .. 6 -> 1 .. 16
        const int NG = 1 << (c->sweep_variant - 2);
        if (c->sweep_bulk_S[pi] % NG != 0 || NG > sweep_max_groups(nc))
            return set_err(c, FP_ERR_UNSUPPORTED, "ILU sweeps: group count above the slots or the block size allows");
        return cuda_check(c, launch_bulk(NG), "ILU sweeps");
    }
    if (c->sweep_variant == 0 && c->sweep_bulk_grid[pi] > 0 && c->sweep_bulk_NG[pi] == 0) {
        // autotuning: every group count NG whose slots divide evenly is timed on this application
        // (each candidate computes the same values, so the choice never changes a result) and the
        // fastest is kept for the context and precision
        float best = 1e30f;
        int bestNG = 1;
        cudaEvent_t ev[2];
        int rc = cuda_check(c, cudaEventCreate(&ev[0]), "event");
        if (!rc) rc = cuda_check(c, cudaEventCreate(&ev[1]), "event");
        if (rc) return rc;
        for (int NG = 1; NG <= sweep_max_groups(nc) && !rc; NG *= 2) {
            if (c->sweep_bulk_S[pi] % NG != 0) continue;
            if (NG > 1) {  // a fresh epoch for every further candidate
                epoch = ++c->ilu_epoch;
                if (epoch == 0) {
                    rc = cuda_check(c, cudaMemsetAsync(c->d_ilu_pub, 0, 4 * (size_t)nE * nc * sizeof(unsigned long long),
                                                       c->stream), "memset");
                    epoch = c->ilu_epoch = 1;
                }
            }
            cudaEventRecord(ev[0], c->stream);
            if (!rc) rc = cuda_check(c, launch_bulk(NG), "ILU sweeps");
            cudaEventRecord(ev[1], c->stream);
            float ms = 0;
            if (!rc) rc = cuda_check(c, cudaEventSynchronize(ev[1]), "sync");
            if (!rc) cudaEventElapsedTime(&ms, ev[0], ev[1]);
            if (!rc && ms < best) {
                best = ms;
                bestNG = NG;
            }
        }
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
        if (rc) return rc;
        c->sweep_bulk_NG[pi] = bestNG;
        return FP_OK;
    }
    cudaError_t e;
    if (c->sweep_variant == 0 && c->sweep_bulk_grid[pi] > 0) {
        e = launch_bulk(c->sweep_bulk_NG[pi]);
    } else {
        void* args[] = {&nc, &nf, &ld, &nE, &c->d_swEl, &c->d_swNb, (void*)&F, (void*)&b, &xx, &pubF, &pubB, &epoch,
                        &abortw, &status, &polls};
        e = cudaLaunchCooperativeKernel((const void*)k_ilu_sweeps<T>, dim3(c->sweep_grid), dim3(kSweepThreads), args, 0,
                                        c->stream);
    }
    return cuda_check(c, e, "ILU sweeps");
}

int ilu_apply(fp_ctx* c, const double* x, double* y) {
    const int nc = c->nc, nE = c->hm.nElem;
    if (c->ilu_prec != FP_PREC_FP32 && c->ilu_prec != FP_PREC_FP64) return set_err(c, FP_ERR_STATE, "block ILU(0): not factorised");
    unsigned epoch = ++c->ilu_epoch;
    if (epoch == 0) {  // wrapped: clear the published words and start again
        int rc = cuda_check(
            c, cudaMemsetAsync(c->d_ilu_pub, 0, 4 * (size_t)nE * nc * sizeof(unsigned long long), c->stream), "memset");
        if (rc) return rc;
        epoch = c->ilu_epoch = 1;
    }
    if (c->ilu_prec == FP_PREC_FP32) return launch_sweeps<float>(c, c->d_iluF32, x, y, epoch);
    return launch_sweeps<double>(c, c->d_iluF64, x, y, epoch);
}

int ilu_check(fp_ctx* c) {
    if (!c->ilu_built) return FP_OK;
    unsigned* words = c->d_iluFlags;
    unsigned h[2] = {0, 0};
    int rc;
    if ((rc = cuda_check(c, cudaMemcpyAsync(h, words, sizeof(h), cudaMemcpyDeviceToHost, c->stream), "copy")) ||
        (rc = cuda_check(c, cudaStreamSynchronize(c->stream), "sync")))
        return rc;
    if (h[0] || h[1]) {
        cudaMemsetAsync(words, 0, sizeof(h), c->stream);
        return set_err(c, FP_ERR_TIMEOUT, "block ILU(0) sweep: a dependency wait gave up");
    }
    return FP_OK;
}

}  // namespace fp
