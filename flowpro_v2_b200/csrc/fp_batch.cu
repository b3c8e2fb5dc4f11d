// Batched serving: independent cases of one model and one polynomial order (any mesh sizes,
// their own outlet pressures) merged into one mesh on one context and driven to their steady
// states together.  Every kernel of a pseudo-time step covers all cases in one launch: the
// residual and its tangent read each element's case for the outlet pressure and the BDF
// coefficients of the case's own time step; the block ILU(0) preconditioner of the merged mesh
// is block-diagonal over the cases (no face couples two cases), so one factorisation and one
// application serve all of them.  What belongs to one case is kept per case: the time step and
// CFL control (State / CFLSetup), the residual norms, and GMRES, whose inner products, norms
// and Givens rotations are taken per case (segmented reductions over the cases' element ranges,
// deterministic order) while the Krylov vectors of all cases advance in lockstep.  A case that
// reaches the target residuum is frozen (its coefficients no longer change); a case whose linear
// solve fails returns to its last state with a reduced CFL, as LocalImplicitSolver does.
//
// It replaces running LocalImplicitSolver (LocalImplicitSolver.java:107-285) once per case.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "fp_ctx.h"
#include "fp_launch.h"
#include "fp_state.h"

namespace fp {

namespace {

constexpr int kChunk = 2048;  // elements per chunk of the segmented reductions
constexpr int kRT = 256;

inline unsigned vgrid_of(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16); }

constexpr int kKB = 8;  // Krylov vectors per block of the chunk dot products

// part[k][ch] = sum over the chunk's elements e and components q < K of a[q ld + e] * b_k[q ld + e]
// for the kKB vectors k = blockIdx.y * kKB, ... below kc (b_k = V + k stride; V == nullptr: a
// itself, one vector), components outer, elements inner, each value of a read once for the
// block's vectors.  Chunks of a case whose live flag is 0 are skipped (their partials stay stale).
__global__ void __launch_bounds__(kRT) k_chunk_dots(int nchunks, const int* __restrict__ ch_e0, const int* __restrict__ ch_e1,
                                                  const int* __restrict__ case_of, const int* __restrict__ live, int K,
                                                  int ld, int kc, const double* __restrict__ a, const double* __restrict__ V,
                                                  size_t stride, double* __restrict__ part) {
    const int ch = blockIdx.x, k0 = blockIdx.y * kKB;
    const int e0 = ch_e0[ch], n = ch_e1[ch] - e0;
    if (live && !live[case_of[e0]]) return;
    const int nk = V ? min(kKB, kc - k0) : 1;
    double s[kKB];
#pragma unroll
    for (int k = 0; k < kKB; k++) s[k] = 0.0;
    for (int q = 0; q < K; q++) {
        const size_t base = (size_t)q * ld + e0;
        for (int e = threadIdx.x; e < n; e += kRT) {
            const double av = a[base + e];
            if (!V) {
                s[0] += av * av;
                continue;
            }
#pragma unroll
            for (int k = 0; k < kKB; k++)
                if (k < nk) s[k] += av * V[(size_t)(k0 + k) * stride + base + e];
        }
    }
    __shared__ double sh[kKB][kRT / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kKB; k++) {
        double v = s[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[k][wid] = v;
    }
    __syncthreads();
    if ((int)threadIdx.x < nk) {
        double v = 0.0;
        for (int w = 0; w < kRT / 32; w++) v += sh[threadIdx.x][w];
        part[(size_t)(k0 + threadIdx.x) * nchunks + ch] = v;
    }
}

// per-component sums of per-element values in[q][e] (q < K) over each chunk: part[q][ch]
__global__ void __launch_bounds__(kRT) k_chunk_sums(int nchunks, const int* __restrict__ ch_e0, const int* __restrict__ ch_e1,
                                                  int ld, const double* __restrict__ in, double* __restrict__ part) {
    const int ch = blockIdx.x, q = blockIdx.y;
    const int e0 = ch_e0[ch], e1 = ch_e1[ch];
    double s = 0;
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) s += in[(size_t)q * ld + e];
    __shared__ double sh[kRT];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = kRT / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[(size_t)q * nchunks + ch] = sh[0];
}

__global__ void __launch_bounds__(kRT) k_chunk_min(int nchunks, const int* __restrict__ ch_e0, const int* __restrict__ ch_e1,
                                                 const double* __restrict__ in, double* __restrict__ part) {
    const int ch = blockIdx.x;
    double s = 1.0e300;
    for (int e = ch_e0[ch] + threadIdx.x; e < ch_e1[ch]; e += blockDim.x) s = fmin(s, in[e]);
    __shared__ double sh[kRT];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = kRT / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] = fmin(sh[threadIdx.x], sh[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[ch] = sh[0];
}

// out[k][case] = the case's chunk partials combined in chunk order (sum, or min when mn)
__global__ void k_case_combine(int ncases, const int* __restrict__ cptr, int nchunks, int K, const double* __restrict__ part,
                               double* __restrict__ out, int mn) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= K * ncases) return;
    const int k = t / ncases, cs = t - k * ncases;
    double s = mn ? 1.0e300 : 0.0;
    for (int ch = cptr[cs]; ch < cptr[cs + 1]; ch++) s = mn ? fmin(s, part[(size_t)k * nchunks + ch]) : s + part[(size_t)k * nchunks + ch];
    out[(size_t)k * ncases + cs] = s;
}

// Element-parallel vector kernels over the merged mesh: thread e handles the K components of
// element e, reads its case once, and skips the element when the case's live flag is 0 (live ==
// nullptr: every case), leaving its values untouched.

// w[q ld + e] += sgn * sum_{k < kc(case)} h[k][case] V_k[q ld + e] (kcs: per-case counts,
// nullptr: kc for every case)
__global__ void k_case_maxpy(int nElem, int ld, int K, int kc, int ncases, const int* __restrict__ case_of,
                             const int* __restrict__ live, const int* __restrict__ kcs, double sgn, double* __restrict__ w,
                             const double* __restrict__ V, size_t stride, const double* __restrict__ h) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nElem; e += gridDim.x * blockDim.x) {
        const int cs = case_of[e];
        if (live && !live[cs]) continue;
        const int kn = kcs ? kcs[cs] : kc;
        for (int q = 0; q < K; q++) {
            const size_t i = (size_t)q * ld + e;
            double s = 0;
#pragma unroll 4
            for (int k = 0; k < kn; k++) s += h[(size_t)k * ncases + cs] * V[(size_t)k * stride + i];
            w[i] += sgn * s;
        }
    }
}

// y = x / sqrt(nrm2[case]) (0 for a zero norm)
__global__ void k_case_normalise(int nElem, int ld, int K, const int* __restrict__ case_of, const int* __restrict__ live,
                                 const double* __restrict__ nrm2, const double* __restrict__ x, double* __restrict__ y) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nElem; e += gridDim.x * blockDim.x) {
        const int cs = case_of[e];
        if (live && !live[cs]) continue;
        const double s = nrm2[cs];
        const double r = s > 0 ? sqrt(s) : 0.0;
        for (int q = 0; q < K; q++) {
            const size_t i = (size_t)q * ld + e;
            y[i] = s > 0 ? x[i] / r : 0.0;
        }
    }
}

// cases with mask[case] != 0: mode 0 y = x, mode 1 y += x
__global__ void k_case_masked(int nElem, int ld, int K, const int* __restrict__ case_of, const int* __restrict__ mask, int mode,
                              const double* __restrict__ x, double* __restrict__ y) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nElem; e += gridDim.x * blockDim.x) {
        if (!mask[case_of[e]]) continue;
        for (int q = 0; q < K; q++) {
            const size_t i = (size_t)q * ld + e;
            if (mode == 0)
                y[i] = x[i];
            else
                y[i] += x[i];
        }
    }
}

__global__ void k_bminus_all(size_t n, double* __restrict__ y, const double* __restrict__ b) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) y[i] = b[i] - y[i];
}

// Gmres.rotmat, Gmres.java:132-148
void rotmat(double a, double b, double& cs, double& sn) {
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

// Gmres.lsolve, Gmres.java:176-199
std::vector<double> lsolve(std::vector<std::vector<double>> A, std::vector<double> b, int N) {
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

struct Batch {
    fp_ctx* c;
    int n = 0, nch = 0;
    size_t nvec = 0;
    int *d_ch0 = nullptr, *d_ch1 = nullptr, *d_cptr = nullptr;
    double* part = nullptr;  // [K][nch]
    double* cbuf = nullptr;  // [K][n] per-case results
    int* d_mask = nullptr;
    std::vector<double> h;   // host mirror of cbuf
};

// the chunk table of the cases' element ranges and the reduction buffers (on first use)
int batch_prepare(fp_ctx* c, int kmax) {
    const int n = c->n_cases;
    if (c->batch_ready && c->batch_kmax >= kmax) return FP_OK;
    std::vector<int> e0, e1, cptr(n + 1, 0);
    for (int cs = 0; cs < n; cs++) {
        cptr[cs] = (int)e0.size();
        for (int a = c->case_e0[cs]; a < c->case_e0[cs + 1]; a += kChunk) {
            e0.push_back(a);
            e1.push_back(std::min(a + kChunk, c->case_e0[cs + 1]));
        }
    }
    cptr[n] = (int)e0.size();
    const int nch = (int)e0.size();
    const int K = std::max(kmax, c->hm.model.n_eqs) + 1;
    int rc;
    if ((rc = dalloc(c, &c->d_bch0, (size_t)nch, false)) || (rc = dalloc(c, &c->d_bch1, (size_t)nch, false)) ||
        (rc = dalloc(c, &c->d_bcptr, (size_t)n + 1, false)) || (rc = dalloc(c, &c->d_bpart, (size_t)K * nch)) ||
        (rc = dalloc(c, &c->d_bcase, (size_t)3 * K * n)) || (rc = dalloc(c, &c->d_bmask, (size_t)n)) ||
        (rc = dalloc(c, &c->d_blive, (size_t)n)) || (rc = dalloc(c, &c->d_bkc, (size_t)n)))
        return rc;
    if ((rc = upload(c, c->d_bch0, e0.data(), nch)) || (rc = upload(c, c->d_bch1, e1.data(), nch)) ||
        (rc = upload(c, c->d_bcptr, cptr.data(), n + 1)))
        return rc;
    c->batch_nch = nch;
    c->batch_kmax = kmax;
    c->batch_ready = true;
    return FP_OK;
}

// per-case values of K per-element components in[q][e] (sum) into c->d_bcase + off, and on the host
int case_sums(fp_ctx* c, const double* in, int K, std::vector<double>& host) {
    const int n = c->n_cases, nch = c->batch_nch;
    k_chunk_sums<<<dim3(nch, K), kRT, 0, c->stream>>>(nch, c->d_bch0, c->d_bch1, c->hm.ld, in, c->d_bpart);
    k_case_combine<<<(K * n + 127) / 128, 128, 0, c->stream>>>(n, c->d_bcptr, nch, K, c->d_bpart, c->d_bcase, 0);
    host.resize((size_t)K * n);
    int rc = cuda_check(c, cudaMemcpyAsync(host.data(), c->d_bcase, host.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                           c->stream), "copy");
    if (rc) return rc;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "sync");
}

// per-case dots: out[k][case] = <a, V_k>_case for k < kc (V == nullptr: <a, a>), left on the device
// (cases whose live flag is 0 are skipped while c->batch_mask is set; their values are stale)
void case_dots(fp_ctx* c, const double* a, const double* V, int kc, double* out) {
    const int n = c->n_cases, nch = c->batch_nch;
    const int* live = c->batch_mask ? c->d_blive : nullptr;
    const int ky = V ? (kc + kKB - 1) / kKB : 1;
    k_chunk_dots<<<dim3(nch, ky), kRT, 0, c->stream>>>(nch, c->d_bch0, c->d_bch1, c->d_case_of, live, c->nc, c->hm.ld, kc, a,
                                                        V, c->nvec, c->d_bpart);
    k_case_combine<<<(kc * n + 127) / 128, 128, 0, c->stream>>>(n, c->d_bcptr, nch, kc, c->d_bpart, out, 0);
}

int fetch_dev(fp_ctx* c, const double* d, size_t n, double* h) {
    int rc = cuda_check(c, cudaMemcpyAsync(h, d, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "copy");
    if (rc) return rc;
    rc = cuda_check(c, cudaStreamSynchronize(c->stream), "sync");
    prof_resolve(c);
    return rc;
}

// cases marked in `mark` back to the free stream they started from (W = Wo = Wo2 = W0)
int batch_reset(fp_ctx* c, const std::vector<int>& mark) {
    bool any = false;
    for (int m : mark) any = any || m;
    if (!any) return FP_OK;
    int rc = upload(c, c->d_bmask, mark.data(), mark.size());
    if (rc) return rc;
    const unsigned G = vgrid_of(c->hm.nElem);
    for (double* d : {c->d_W, c->d_Wo, c->d_Wo2})
        k_case_masked<<<G, 256, 0, c->stream>>>(c->hm.nElem, c->hm.ld, c->nc, c->d_case_of, c->d_bmask, 0, c->d_case_W0, d);
    return cuda_check(c, cudaGetLastError(), "reset");
}

// Batched left-preconditioned GMRES(m) on (A, b = d_rhs) from x = 0 (Gmres.solve per case,
// Gmres.java:42-122): per-case tolerance relative to ||M^-1 b||_case, CGS2 orthogonalisation per
// case, Givens rotations per case on the host; convergence accepted on the true preconditioned
// residual.  ok[cs] = converged, its[cs] = iterations the case took.
int batch_gmres(fp_ctx* c, const std::vector<int>& want, int kind, int m, int max_restarts, double tol, std::vector<int>& ok,
                std::vector<int>& its) {
    const int n = c->n_cases;
    const size_t N = c->nvec;
    const int ld = c->hm.ld, nE = c->hm.nElem;
    double *V = c->d_V, *w = c->d_w, *aux = c->d_aux, *r = c->d_r, *x = c->d_x, *b = c->d_rhs;
    double* h1 = c->d_bcase;                        // [m+1][n]
    double* h2 = c->d_bcase + (size_t)(m + 1) * n;  // [m+1][n]
    double* nr = c->d_bcase + (size_t)2 * (m + 1) * n;
    const int* case_of = c->d_case_of;
    const unsigned G = vgrid_of(nE);
    const int K = c->nc;
    int rc;
    if ((rc = cuda_check(c, cudaMemsetAsync(x, 0, N * sizeof(double), c->stream), "memset"))) return rc;
    // the kernels skip the elements of cases that are not iterating (live flags on the device,
    // uploaded when the set changes); the operator and the block ILU(0) sweeps read the same flags
    std::vector<int> flags(n, 0);
    bool uploaded = false;
    auto set_live = [&](const std::vector<char>& on) -> int {
        bool same = uploaded;
        for (int cs = 0; cs < n; cs++) same = same && flags[cs] == (int)on[cs];
        if (same) return FP_OK;
        for (int cs = 0; cs < n; cs++) flags[cs] = on[cs];
        uploaded = true;
        return upload(c, c->d_blive, flags.data(), (size_t)n);
    };
    struct MaskScope {  // the flags apply while batch_gmres runs
        fp_ctx* c;
        ~MaskScope() { c->batch_mask = false; }
    } scope{c};
    if ((rc = set_live(std::vector<char>(want.begin(), want.end())))) return rc;
    c->batch_mask = true;
    // ||M^-1 b||_case
    if ((rc = prec_apply(c, kind, b, r))) return rc;
    case_dots(c, r, nullptr, 1, nr);
    std::vector<double> hh((size_t)3 * (m + 1) * n), bn(n), err(n), s((size_t)n * (m + 1)), csv((size_t)n * m), snv((size_t)n * m);
    if ((rc = fetch_dev(c, nr, n, hh.data()))) return rc;
    std::vector<char> active(n, 0);
    for (int cs = 0; cs < n; cs++) {
        bn[cs] = std::sqrt(hh[cs]);
        if (bn[cs] == 0) bn[cs] = 1;
        err[cs] = std::sqrt(hh[cs]) / bn[cs];  // x = 0: r = M^-1 b
        active[cs] = want[cs] && err[cs] >= tol;
        its[cs] = 0;
    }
    std::vector<std::vector<std::vector<double>>> H(n);
    std::vector<int> used(n, 0);
    for (int cycle = 0; cycle < max_restarts; cycle++) {
        bool any = false;
        for (int cs = 0; cs < n; cs++) any = any || active[cs];
        if (!any) break;
        // V_0 = r / ||r||_case
        if ((rc = set_live(active))) return rc;
        case_dots(c, r, nullptr, 1, nr);
        k_case_normalise<<<G, 256, 0, c->stream>>>(nE, ld, K, case_of, c->d_blive, nr, r, V);
        if ((rc = fetch_dev(c, nr, n, hh.data()))) return rc;
        std::vector<char> live(active);
        for (int cs = 0; cs < n; cs++) {
            H[cs].assign(m + 1, std::vector<double>(m, 0.0));
            std::fill(s.begin() + (size_t)cs * (m + 1), s.begin() + (size_t)(cs + 1) * (m + 1), 0.0);
            s[(size_t)cs * (m + 1)] = std::sqrt(hh[cs]);
            used[cs] = 0;
        }
        for (int i = 0; i < m; i++) {
            bool anyl = false;
            for (int cs = 0; cs < n; cs++) anyl = anyl || live[cs];
            if (!anyl) break;
            double* Vi = V + (size_t)i * N;
            if ((rc = set_live(live))) return rc;
            prof_begin(c, PH_OPERATOR);
            rc = matfree_apply(c, Vi, aux);
            prof_end(c);
            if (rc) return rc;
            prof_begin(c, PH_PREC);
            rc = prec_apply(c, kind, aux, w);
            prof_end(c);
            if (rc) return rc;
            const int kc = i + 1;
            prof_begin(c, PH_KRYLOV);
            for (double* hk : {h1, h2}) {  // two classical Gram-Schmidt passes per case
                case_dots(c, w, V, kc, hk);
                k_case_maxpy<<<G, 256, 0, c->stream>>>(nE, ld, K, kc, n, case_of, c->d_blive, nullptr, -1.0, w, V, N, hk);
            }
            case_dots(c, w, nullptr, 1, nr);
            k_case_normalise<<<G, 256, 0, c->stream>>>(nE, ld, K, case_of, c->d_blive, nr, w, V + (size_t)(i + 1) * N);
            prof_end(c);
            if ((rc = fetch_dev(c, c->d_bcase, (size_t)3 * (m + 1) * n, hh.data()))) return rc;
            for (int cs = 0; cs < n; cs++) {
                if (!live[cs]) continue;
                its[cs]++;
                auto& Hc = H[cs];
                double* sc = s.data() + (size_t)cs * (m + 1);
                double* cc = csv.data() + (size_t)cs * m;
                double* sn = snv.data() + (size_t)cs * m;
                for (int k = 0; k <= i; k++) Hc[k][i] = hh[(size_t)k * n + cs] + hh[(size_t)(m + 1) * n + (size_t)k * n + cs];
                Hc[i + 1][i] = std::sqrt(hh[(size_t)2 * (m + 1) * n + cs]);
                for (int k = 0; k <= i - 1; k++) {
                    double temp = cc[k] * Hc[k][i] + sn[k] * Hc[k + 1][i];
                    Hc[k + 1][i] = -sn[k] * Hc[k][i] + cc[k] * Hc[k + 1][i];
                    Hc[k][i] = temp;
                }
                rotmat(Hc[i][i], Hc[i + 1][i], cc[i], sn[i]);
                double temp = cc[i] * sc[i];
                sc[i + 1] = -sn[i] * sc[i];
                sc[i] = temp;
                Hc[i][i] = cc[i] * Hc[i][i] + sn[i] * Hc[i + 1][i];
                Hc[i + 1][i] = 0;
                used[cs] = i + 1;
                err[cs] = std::fabs(sc[i + 1]) / bn[cs];
                if (err[cs] <= tol || !std::isfinite(err[cs])) live[cs] = 0;
            }
        }
        // x += V y per case (cases that were not active take no update); the true residual of
        // every case active in this cycle
        if ((rc = set_live(active))) return rc;
        int kmax = 0;
        std::vector<int> kcs(n, 0);
        for (int cs = 0; cs < n; cs++) {
            kcs[cs] = active[cs] ? used[cs] : 0;
            kmax = std::max(kmax, kcs[cs]);
        }
        std::vector<double> y((size_t)std::max(kmax, 1) * n, 0.0);
        for (int cs = 0; cs < n; cs++) {
            if (!active[cs] || used[cs] == 0) continue;
            std::vector<double> sc(s.begin() + (size_t)cs * (m + 1), s.begin() + (size_t)(cs + 1) * (m + 1));
            std::vector<double> yc = lsolve(H[cs], sc, used[cs]);
            for (int k = 0; k < used[cs]; k++) y[(size_t)k * n + cs] = yc[k];
        }
        if (kmax > 0) {
            if ((rc = cuda_check(c, cudaMemcpyAsync(h1, y.data(), y.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream),
                                 "copy")))
                return rc;
            if ((rc = upload(c, c->d_bkc, kcs.data(), (size_t)n))) return rc;
            // each case's own Krylov vectors only (those past its count may be stale)
            k_case_maxpy<<<G, 256, 0, c->stream>>>(nE, ld, K, kmax, n, case_of, c->d_blive, c->d_bkc, 1.0, x, V, N, h1);
        }
        // true preconditioned residual per case
        prof_begin(c, PH_OPERATOR);
        rc = matfree_apply(c, x, aux);
        prof_end(c);
        if (rc) return rc;
        k_bminus_all<<<G, 256, 0, c->stream>>>(N, aux, b);
        if ((rc = prec_apply(c, kind, aux, r))) return rc;
        case_dots(c, r, nullptr, 1, nr);
        if ((rc = fetch_dev(c, nr, n, hh.data()))) return rc;
        for (int cs = 0; cs < n; cs++) {
            if (!active[cs]) continue;
            err[cs] = std::sqrt(hh[cs]) / bn[cs];
            if (err[cs] <= tol) active[cs] = 0;
        }
    }
    for (int cs = 0; cs < n; cs++) ok[cs] = want[cs] && err[cs] <= tol;
    return FP_OK;
}

}  // namespace
}  // namespace fp

using namespace fp;

extern "C" {

int fp_batch_upload(fp_ctx* c, int n, const fp_mesh_desc* descs, const fp_model_params* models, const fp_num_params* num) {
    if (!c || n <= 0 || !descs || !models || !num) return FP_ERR_ARG;
    const fp_model_params& m0 = models[0];
    size_t nv = 0, ne = 0;
    bool wd = true;
    for (int i = 0; i < n; i++) {
        const fp_model_params& mi = models[i];
        if (mi.model != m0.model || mi.dim != m0.dim || mi.n_eqs != m0.n_eqs || mi.is_diffusive != m0.is_diffusive ||
            mi.kappa != m0.kappa || descs[i].dim != m0.dim)
            return set_err(c, FP_ERR_ARG, "a batch takes cases of one model; only the outlet pressure may differ");
        if (descs[i].n_vertices <= 0 || descs[i].n_elements <= 0) return set_err(c, FP_ERR_ARG, "empty case");
        nv += descs[i].n_vertices;
        ne += descs[i].n_elements;
        wd = wd && descs[i].wall_distance;
    }
    if (ne > (size_t)1 << 30) return set_err(c, FP_ERR_ARG, "batch too large");
    const int dim = m0.dim, nvx = dim + 1;
    std::vector<double> V(nv * dim), WD(wd ? nv : 0);
    std::vector<int> E(ne * nvx), T(ne * nvx), e0(n + 1, 0);
    size_t vo = 0, eo = 0;
    for (int i = 0; i < n; i++) {
        const fp_mesh_desc& d = descs[i];
        std::copy(d.vertices, d.vertices + (size_t)d.n_vertices * dim, V.begin() + vo * dim);
        if (wd) std::copy(d.wall_distance, d.wall_distance + d.n_vertices, WD.begin() + vo);
        for (size_t k = 0; k < (size_t)d.n_elements * nvx; k++) {
            E[eo * nvx + k] = d.elements[k] + (int)vo;
            const int t = d.neighbors[k];
            T[eo * nvx + k] = t >= 0 ? t + (int)eo : t;
        }
        e0[i] = (int)eo;
        vo += d.n_vertices;
        eo += d.n_elements;
    }
    e0[n] = (int)eo;
    fp_mesh_desc md{};
    md.dim = dim;
    md.n_vertices = (int)nv;
    md.n_elements = (int)ne;
    md.vertices = V.data();
    md.elements = E.data();
    md.neighbors = T.data();
    md.wall_distance = wd ? WD.data() : nullptr;
    int rc = fp_mesh_upload(c, &md, &m0, num);
    if (rc) return rc;
    // the cases' element ranges, their outlet pressures and free-stream states
    c->n_cases = n;
    c->case_e0 = e0;
    std::vector<double> pout(n);
    for (int i = 0; i < n; i++) pout[i] = models[i].p_out;
    std::vector<int> cof(c->hm.ld, 0);
    for (int i = 0; i < n; i++)
        for (int e = e0[i]; e < e0[i + 1]; e++) cof[e] = i;
    if ((rc = dalloc(c, &c->d_case_of, (size_t)c->hm.ld, false)) || (rc = upload(c, c->d_case_of, cof.data(), cof.size())) ||
        (rc = dalloc(c, &c->d_case_pout, (size_t)n, false)) || (rc = upload(c, c->d_case_pout, pout.data(), (size_t)n)) ||
        (rc = dalloc(c, &c->d_case_a, (size_t)3 * n)))
        return rc;
    const int nb = c->hm.tab.nb, neq = c->hm.model.n_eqs, nc = c->nc;
    std::vector<double> W(ne * (size_t)nc);
    for (int i = 0; i < n; i++) {
        double w0[8];
        const_init_condition(models[i], w0);
        for (int e = e0[i]; e < e0[i + 1]; e++)
            for (int q = 0; q < neq; q++)
                for (int j = 0; j < nb; j++) W[(size_t)e * nc + q * nb + j] = w0[q];
    }
    for (int which = 0; which < 3; which++)
        if ((rc = fp_state_set(c, which, W.data()))) return rc;
    // the free streams, kept for cases whose state stops being finite
    if ((rc = dalloc(c, &c->d_case_W0, c->nvec, false)) ||
        (rc = cuda_check(c, cudaMemcpyAsync(c->d_case_W0, c->d_W, c->nvec * sizeof(double), cudaMemcpyDeviceToDevice, c->stream),
                         "copy")))
        return rc;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "sync");
}

int fp_batch_info(const fp_ctx* c, int* n_cases, int* case_e0) {
    if (!c || !c->has_mesh) return FP_ERR_STATE;
    if (n_cases) *n_cases = c->n_cases;
    if (case_e0 && c->n_cases > 0) std::copy(c->case_e0.begin(), c->case_e0.end(), case_e0);
    return FP_OK;
}

int fp_batch_solve(fp_ctx* c, const fp_implicit_params* pin, double* out, int* status) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if (c->n_cases <= 0) return set_err(c, FP_ERR_STATE, "no batch uploaded (fp_batch_upload)");
    if (!pin) return set_err(c, FP_ERR_ARG, "null parameters");
    fp_implicit_params P = *pin;
    if (P.preconditioner == FP_PREC_ILU0) P.preconditioner = FP_PREC_BLOCKILU0;
    if (P.jacobian != FP_JAC_MATRIXFREE || P.preconditioner != FP_PREC_BLOCKILU0 || P.newton_iters != 1 || P.fixed_dt > 0)
        return set_err(c, FP_ERR_UNSUPPORTED,
                       "batched solves take the matrix-free operator with block ILU(0), one Newton iteration per step "
                       "and CFL control");
    if (P.restart < 1 || P.restart > 200 || P.max_restarts < 1) return set_err(c, FP_ERR_ARG, "bad GMRES sizes");
    const Launchers* t = find_launchers(c->hm.model, c->hm.num.order);
    if (!t) return set_err(c, FP_ERR_UNSUPPORTED, "model / order not built");
    const int n = c->n_cases, neq = c->hm.model.n_eqs;
    if ((rc = ensure_rhs(c)) || (rc = ensure_krylov(c, P.restart, P.precision)) || (rc = batch_prepare(c, P.restart + 1)))
        return rc;
    double* elem = c->d_Wst[0];  // per-element scratch [NE][ld] (the RK stage states are idle here)
    std::vector<State> st(n);
    for (auto& s : st) {
        s.cfl = P.cfl > 0 ? P.cfl : 1;
        s.vary = P.vary_cfl != 0 || P.cfl <= 0;
        s.maxCFL = P.max_cfl > 0 ? P.max_cfl : 1e4;
    }
    enum { RUNNING = 0, DONE = 1, HOPELESS = 2, NONFINITE = 3 };
    std::vector<int> state(n, RUNNING), converges(n, 1), newton(n, 0), linear(n, 0), ok(n), its(n), want(n);
    std::vector<double> dto(n, -1.0), dt(n, 0.0), a((size_t)3 * n, 0.0), hbuf;
    const int lag = P.jac_lag > 1 ? P.jac_lag : 1;
    int since = 1 << 30;
    const double factor = c->hm.num.implicit_time ? 1.0 : 2.0 * (c->hm.num.order - 1) + 1;
    DevMesh base = dev_mesh(c);
    for (int step = 0; step < P.steps; step++) {
        bool any = false;
        for (int cs = 0; cs < n; cs++) {
            if (state[cs] != RUNNING) continue;
            if (converges[cs]) st[cs].updateCFL();
            if (st[cs].hopeless()) state[cs] = HOPELESS;
            any = any || state[cs] == RUNNING;
        }
        if (!any) break;
        // the time step of every running case (State.getTimeStep per case)
        t->dtbound_elem(base, c->stream, c->d_W, factor, elem);
        {
            const int nch = c->batch_nch;
            k_chunk_min<<<nch, kRT, 0, c->stream>>>(nch, c->d_bch0, c->d_bch1, elem, c->d_bpart);
            k_case_combine<<<(n + 127) / 128, 128, 0, c->stream>>>(n, c->d_bcptr, nch, 1, c->d_bpart, c->d_bcase, 1);
            hbuf.resize(n);
            if ((rc = fetch_dev(c, c->d_bcase, n, hbuf.data()))) return rc;
        }
        for (int cs = 0; cs < n; cs++) {
            if (state[cs] != RUNNING) continue;  // frozen cases keep their last coefficients
            dt[cs] = st[cs].currentCFL * hbuf[cs];
            st[cs].dt = dt[cs];
            double ac[3];
            bdf_coef(P.bdf_order, dt[cs], dto[cs], ac);
            for (int k = 0; k < 3; k++) a[(size_t)k * n + cs] = ac[k];
        }
        if ((rc = upload(c, c->d_case_a, a.data(), a.size()))) return rc;
        if ((rc = launch_limiter(c))) return rc;
        // right-hand side and residual norms of every case (MasterSolver.residuumNorms,
        // State.setResiduum); a case whose state is no longer finite stops, and it and any frozen
        // case in that condition return to their free stream so the shared factorisation stays
        // regular
        double nrm = 0;
        if ((rc = fp_assemble_residuum(c, P.bdf_order, 1.0, -1.0, &nrm))) return rc;
        t->norms_elem(base, c->stream, c->d_R, elem);
        if ((rc = case_sums(c, elem, neq, hbuf))) return rc;
        std::vector<int> reset(n, 0);
        bool any_reset = false;
        for (int cs = 0; cs < n; cs++) {
            std::vector<double> norms(neq);
            bool finite = true;
            for (int q = 0; q < neq; q++) {
                norms[q] = std::sqrt(hbuf[(size_t)q * n + cs]);
                finite = finite && std::isfinite(norms[q]);
            }
            if (!finite) {
                reset[cs] = 1;
                any_reset = true;
                if (state[cs] == RUNNING) state[cs] = NONFINITE;
                continue;
            }
            if (state[cs] == RUNNING) st[cs].setResiduum(norms);
        }
        if (any_reset) {
            if ((rc = batch_reset(c, reset))) return rc;
            if ((rc = fp_assemble_residuum(c, P.bdf_order, 1.0, -1.0, &nrm))) return rc;
        }
        // the preconditioner when it is due; a singular block sends its case back to its last
        // state with a reduced CFL (LinearSolver.solve returning false), and the step is retried
        if (since >= lag - 1) {
            rc = fp_assemble_preconditioner(c, P.bdf_order, 1.0, -1.0, P.preconditioner, P.precision);
            if (rc == FP_ERR_SINGULAR) {
                std::vector<unsigned> sg(c->hm.nElem);
                if ((rc = cuda_check(c, cudaMemcpyAsync(sg.data(), c->d_ilu_sing, sg.size() * sizeof(unsigned),
                                                        cudaMemcpyDeviceToHost, c->stream), "copy")) ||
                    (rc = cuda_check(c, cudaStreamSynchronize(c->stream), "sync")))
                    return rc;
                std::vector<int> back(n, 0), frozen(n, 0);
                for (int cs = 0; cs < n; cs++)
                    for (int e = c->case_e0[cs]; e < c->case_e0[cs + 1]; e++)
                        if (sg[e]) {
                            (state[cs] == RUNNING ? back : frozen)[cs] = 1;
                            break;
                        }
                for (int cs = 0; cs < n; cs++)
                    if (back[cs]) {
                        st[cs].reduceCFL();
                        converges[cs] = 0;
                    }
                const unsigned G = vgrid_of(c->hm.nElem);
                if ((rc = upload(c, c->d_bmask, back.data(), (size_t)n))) return rc;
                k_case_masked<<<G, 256, 0, c->stream>>>(c->hm.nElem, c->hm.ld, c->nc, c->d_case_of, c->d_bmask, 0, c->d_Wo,
                                                         c->d_W);
                if ((rc = batch_reset(c, frozen))) return rc;
                since = 1 << 30;
                continue;
            }
            if (rc) return rc;
            since = 0;
        } else {
            since++;
        }
        for (int cs = 0; cs < n; cs++) want[cs] = state[cs] == RUNNING;
        if ((rc = batch_gmres(c, want, P.preconditioner, P.restart, P.max_restarts, P.linear_tol, ok, its))) return rc;
        if ((rc = ilu_check(c))) return rc;
        // the cases' outcomes: update, or back to the last state with a smaller CFL
        std::vector<int> upd(n, 0), back(n, 0);
        for (int cs = 0; cs < n; cs++) {
            if (state[cs] != RUNNING) continue;
            newton[cs]++;
            linear[cs] += its[cs];
            converges[cs] = ok[cs];
            if (ok[cs]) {
                upd[cs] = 1;
            } else {
                back[cs] = 1;
                st[cs].reduceCFL();
                since = 1 << 30;  // the retry starts from a fresh preconditioner
            }
        }
        const unsigned G = vgrid_of(c->hm.nElem);
        if ((rc = upload(c, c->d_bmask, upd.data(), (size_t)n))) return rc;
        k_case_masked<<<G, 256, 0, c->stream>>>(c->hm.nElem, c->hm.ld, c->nc, c->d_case_of, c->d_bmask, 1, c->d_x, c->d_W);
        if ((rc = upload(c, c->d_bmask, back.data(), (size_t)n))) return rc;
        k_case_masked<<<G, 256, 0, c->stream>>>(c->hm.nElem, c->hm.ld, c->nc, c->d_case_of, c->d_bmask, 0, c->d_Wo, c->d_W);
        if (c->hm.num.positivity_limiter && (rc = launch_positivity(c, c->d_W, nullptr))) return rc;
        if ((rc = fp_copy_w2wo(c))) return rc;
        for (int cs = 0; cs < n; cs++) {
            if (!upd[cs]) continue;
            if (!std::isfinite(st[cs].residuum)) {
                state[cs] = NONFINITE;
                continue;
            }
            st[cs].steps++;
            st[cs].t += dt[cs];
            dto[cs] = dt[cs];
            if (st[cs].residuum <= P.target_residuum) state[cs] = DONE;
        }
    }
    if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "sync"))) return rc;
    for (int cs = 0; cs < n; cs++) {
        if (out) {
            double* o = out + 7 * (size_t)cs;
            o[0] = st[cs].t;
            o[1] = st[cs].residuum;
            o[2] = st[cs].currentCFL;
            o[3] = st[cs].dt;
            o[4] = st[cs].steps;
            o[5] = newton[cs];
            o[6] = linear[cs];
        }
        if (status) status[cs] = state[cs] == HOPELESS ? FP_ERR_NOT_CONVERGED : state[cs] == NONFINITE ? FP_ERR_NONFINITE : FP_OK;
    }
    return FP_OK;
}

int fp_batch_case_state(fp_ctx* c, int cs, int which, double* w) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if (cs < 0 || cs >= c->n_cases || !w) return set_err(c, FP_ERR_ARG, "bad case");
    std::vector<double> all((size_t)c->hm.nElem * c->nc);
    if ((rc = fp_state_get(c, which, all.data()))) return rc;
    std::copy(all.begin() + (size_t)c->case_e0[cs] * c->nc, all.begin() + (size_t)c->case_e0[cs + 1] * c->nc, w);
    return FP_OK;
}

}  // extern "C"
