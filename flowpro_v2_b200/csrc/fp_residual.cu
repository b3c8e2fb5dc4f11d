// Host wrappers of the residual-side kernels: pick the launch table of the mesh's
// configuration, launch on the context stream, finish the block reductions on the
// host in a fixed order (deterministic results).
#include <algorithm>
#include <cmath>
#include <vector>

#include "fp_ctx.h"
#include "fp_launch.h"

namespace fp {

namespace {
constexpr int kBlk = 128;
inline int nblocks(int n) { return (n + kBlk - 1) / kBlk; }

const Launchers* L(fp_ctx* c, int& rc) {
    const Launchers* t = find_launchers(c->hm.model, c->hm.num.order);
    rc = t ? FP_OK : set_err(c, FP_ERR_UNSUPPORTED, "model / dimension / order combination is not built");
    return t;
}

int read_parts(fp_ctx* c, size_t n, std::vector<double>& h) {
    h.resize(n);
    int rc = cuda_check(c, cudaMemcpyAsync(h.data(), c->d_part, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "copy");
    if (rc) return rc;
    rc = cuda_check(c, cudaStreamSynchronize(c->stream), "sync");
    prof_resolve(c);
    return rc;
}
}  // namespace

int launch_residual(fp_ctx* c, const double* W, double* R) {
    int rc;
    const Launchers* t = L(c, rc);
    if (!t) return rc;
    t->residual(dev_mesh(c), c->stream, W, R);
    return cuda_check(c, cudaGetLastError(), "residual");
}

int launch_residual_timed(fp_ctx* c, const double* W, double* R, cudaEvent_t ev[3]) {
    int rc;
    const Launchers* t = L(c, rc);
    if (!t) return rc;
    const DevMesh M = dev_mesh(c);
    cudaEventRecord(ev[0], c->stream);
    t->faces(M, c->stream, W);
    cudaEventRecord(ev[1], c->stream);
    t->elements(M, c->stream, W, R);
    cudaEventRecord(ev[2], c->stream);
    return cuda_check(c, cudaGetLastError(), "residual");
}

namespace {
// chunks of the pipelined host-buffer residual (elements): a small first chunk starts the
// downloads early; middle chunks of about one wave of the face pass (148 SMs x 4 CTAs x 128
// threads = 75,776 faces, ~1.5 per element in 2D), since a pass over fewer faces still
// takes a wave's time; a small last chunk shortens what follows the last upload
constexpr int kPipeHead = 8192;
constexpr int kPipeBody = 49152;
constexpr int kPipeTail = 8192;

// element-major host layout <-> field-major device layout, elements e0 .. e1 - 1
__global__ void k_to_soa_range(int e0, int e1, int ld, int nc, const double* __restrict__ in, double* __restrict__ out) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)(e1 - e0) * nc) return;
    const size_t g = (size_t)e0 * nc + t;
    const int e = (int)(g / nc), cc = (int)(g - (size_t)e * nc);
    out[(size_t)cc * ld + e] = in[g];
}
__global__ void k_from_soa_range(int e0, int e1, int ld, int nc, const double* __restrict__ in, double* __restrict__ out) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)(e1 - e0) * nc) return;
    const size_t g = (size_t)e0 * nc + t;
    const int e = (int)(g / nc), cc = (int)(g - (size_t)e * nc);
    out[g] = in[(size_t)cc * ld + e];
}
inline unsigned grid256(size_t n) { return (unsigned)((n + 255) / 256); }

// Chunk plan: chunk k holds the elements pipe_e[k] .. pipe_e[k+1] - 1 and the faces they
// own, pipe_f[k] .. pipe_f[k+1] - 1 (the face list is in owner order, every face owned by
// its lower-indexed element, so every face of a chunk's elements belongs to that chunk or
// an earlier one); the face pass of chunk k reads the state of elements below pipe_need[k]
// (its own elements and their neighbours), a non-decreasing bound.
void pipe_plan(fp_ctx* c) {
    const HostMesh& h = c->hm;
    const int nE = h.nElem;
    std::vector<int>& b = c->pipe_e;
    b.assign(1, 0);
    if (nE > kPipeHead + kPipeTail) b.push_back(kPipeHead);
    while (nE - b.back() > kPipeBody + kPipeTail) b.push_back(b.back() + kPipeBody);
    if (nE - b.back() > 2 * kPipeTail) b.push_back(nE - kPipeTail);
    b.push_back(nE);
    const int K = (int)b.size() - 1;
    c->pipe_f.assign(K + 1, 0);
    c->pipe_need.assign(K, 0);
    int f = 0, need = 0;
    for (int k = 0; k < K; k++) {
        c->pipe_f[k] = f;
        need = std::max(need, c->pipe_e[k + 1]);
        for (; f < h.nFaces && h.fl[f] < c->pipe_e[k + 1]; f++)
            if (h.fr[f] >= 0) need = std::max(need, h.fr[f] + 1);
        c->pipe_need[k] = need;
    }
    c->pipe_f[K] = h.nFaces;
}
}  // namespace

namespace {
// Queue the chunked residual on the context stream and the two copy streams (fork and
// join through events, so the sequence can also be captured into a CUDA graph).
int pipe_enqueue(fp_ctx* c, const Launchers* t, const double* w, double* r) {
    int rc;
    const int K = (int)c->pipe_e.size() - 1;
    const int ld = c->hm.ld, nc = c->nc;
    cudaEvent_t evStart = c->pipe_ev[0], evEnd = c->pipe_ev[1];
    const DevMesh M = dev_mesh(c);
    cudaStream_t s = c->stream;
    // the copy streams start after the work already queued on the context stream
    cudaEventRecord(evStart, s);
    cudaStreamWaitEvent(c->s_h2d, evStart, 0);
    cudaStreamWaitEvent(c->s_d2h, evStart, 0);
    // every upload is queued first, so the upload stream never waits for the host
    int uploaded = 0;
    for (int k = 0; k < K; k++) {
        const int need = c->pipe_need[k];
        if (need > uploaded &&
            (rc = cuda_check(c,
                             cudaMemcpyAsync(c->d_io + (size_t)uploaded * nc, w + (size_t)uploaded * nc,
                                             (size_t)(need - uploaded) * nc * sizeof(double), cudaMemcpyHostToDevice, c->s_h2d),
                             "upload")))
            return rc;
        uploaded = std::max(uploaded, need);
        cudaEventRecord(c->pipe_ev[2 + k], c->s_h2d);
    }
    // face passes on the context stream, element passes on a second stream: the face pass
    // of a chunk runs beside the element pass of the one before (an element pass needs
    // the face passes of its own chunk and the earlier ones)
    int converted = 0;
    cudaStream_t se = c->s_elem;
    for (int k = 0; k < K; k++) {
        cudaEvent_t evFace = c->pipe_ev[3 + 2 * K + k], evDone = c->pipe_ev[2 + K + k];
        const int need = c->pipe_need[k], e0 = c->pipe_e[k], e1 = c->pipe_e[k + 1];
        cudaStreamWaitEvent(s, c->pipe_ev[2 + k], 0);
        if (need > converted) {
            k_to_soa_range<<<grid256((size_t)(need - converted) * nc), 256, 0, s>>>(converted, need, ld, nc, c->d_io, c->d_W);
            converted = need;
        }
        t->faces_range(M, s, c->d_W, c->pipe_f[k], c->pipe_f[k + 1]);
        cudaEventRecord(evFace, s);
        cudaStreamWaitEvent(se, evFace, 0);
        t->elements_range(M, se, c->d_W, c->d_R, e0, e1);
        k_from_soa_range<<<grid256((size_t)(e1 - e0) * nc), 256, 0, se>>>(e0, e1, ld, nc, c->d_R, c->d_io2);
        cudaEventRecord(evDone, se);
        cudaStreamWaitEvent(c->s_d2h, evDone, 0);
        if ((rc = cuda_check(c,
                             cudaMemcpyAsync(r + (size_t)e0 * nc, c->d_io2 + (size_t)e0 * nc,
                                             (size_t)(e1 - e0) * nc * sizeof(double), cudaMemcpyDeviceToHost, c->s_d2h),
                             "download")))
            return rc;
    }
    cudaEventRecord(c->pipe_ev[2 + 3 * K], se);
    cudaStreamWaitEvent(s, c->pipe_ev[2 + 3 * K], 0);
    cudaEventRecord(evEnd, c->s_d2h);
    cudaStreamWaitEvent(s, evEnd, 0);
    return cuda_check(c, cudaGetLastError(), "residual");
}

bool pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}
}  // namespace

void pipe_release(fp_ctx* c) {
    if (c->pipe_exec) cudaGraphExecDestroy(c->pipe_exec);
    c->pipe_exec = nullptr;
    c->pipe_w = nullptr;
    c->pipe_r = nullptr;
}

// fp_residual with host input and output.  The state goes up chunk by chunk on one copy
// stream; each chunk's face pass runs as soon as the state it reads has arrived and its
// element pass right after (on a second compute stream, beside the next face pass), and
// its residual goes down on a second copy stream while later chunks go up, so the two
// PCIe directions overlap each other and the passes.
// The results are those of the unchunked passes (the same kernels over index ranges).
// A call with the same pinned host buffers as the previous call replays the sequence as
// one CUDA graph (captured on that second call), which takes the ~160 launches and copy
// calls of the sequence off the host.
int launch_residual_pipelined(fp_ctx* c, const double* w, double* r) {
    int rc;
    const Launchers* t = L(c, rc);
    if (!t) return rc;
    if (c->pipe_e.empty()) pipe_plan(c);
    const int K = (int)c->pipe_e.size() - 1;
    if (!c->d_io2) {
        void* q = nullptr;
        if ((rc = cuda_check(c, cudaMalloc(&q, (size_t)c->hm.nElem * c->nc * sizeof(double) + 256), "cudaMalloc"))) return rc;
        c->allocs.push_back((double*)q);
        c->d_io2 = (double*)q;
    }
    if (!c->s_h2d && ((rc = cuda_check(c, cudaStreamCreateWithFlags(&c->s_h2d, cudaStreamNonBlocking), "stream")) ||
                      (rc = cuda_check(c, cudaStreamCreateWithFlags(&c->s_d2h, cudaStreamNonBlocking), "stream")) ||
                      (rc = cuda_check(c, cudaStreamCreateWithFlags(&c->s_elem, cudaStreamNonBlocking), "stream"))))
        return rc;
    // events: start, end, K uploads, K chunk results, the element stream's end, K face passes
    while ((int)c->pipe_ev.size() < 3 * K + 3) {
        cudaEvent_t e;
        if ((rc = cuda_check(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event"))) return rc;
        c->pipe_ev.push_back(e);
    }
    cudaStream_t s = c->stream;
    const bool repeat = w == c->pipe_w && r == c->pipe_r;
    if (!repeat) pipe_release(c);
    if (repeat && !c->pipe_exec && c->pipe_graph_ok && pinned(w) && pinned(r)) {
        cudaGraph_t g = nullptr;
        cudaStreamCaptureStatus cs;
        bool ok = cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone &&
                  cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            rc = pipe_enqueue(c, t, w, r);
            ok = cudaStreamEndCapture(s, &g) == cudaSuccess && rc == FP_OK && g &&
                 cudaGraphInstantiate(&c->pipe_exec, g, 0) == cudaSuccess;
            if (g) cudaGraphDestroy(g);
        }
        if (!ok) {  // capture unavailable here: stay on the direct path for this context
            cudaGetLastError();
            c->pipe_exec = nullptr;
            c->pipe_graph_ok = false;
            c->err.clear();
        }
    }
    if (c->pipe_exec) {
        if ((rc = cuda_check(c, cudaGraphLaunch(c->pipe_exec, s), "graph launch"))) return rc;
    } else {
        if ((rc = pipe_enqueue(c, t, w, r))) return rc;
        c->pipe_w = w;
        c->pipe_r = r;
    }
    return cuda_check(c, cudaStreamSynchronize(s), "sync");
}

int launch_rk_stage(fp_ctx* c, const double* Wcur, const double* Wo, const double* Wb, double alpha, double beta, double dt,
                    double* Wout, double* Rsave) {
    int rc;
    const Launchers* t = L(c, rc);
    if (!t) return rc;
    t->rk_stage(dev_mesh(c), c->stream, Wcur, Wo, Wb, alpha, beta, dt, Wout, Rsave);
    return cuda_check(c, cudaGetLastError(), "rk stage");
}

int matfree_apply(fp_ctx* c, const double* x, double* y) {
    int rc;
    const Launchers* t = L(c, rc);
    if (!t) return rc;
    t->matfree(dev_mesh(c), c->stream, c->d_W, x, c->a_coef[0], y);
    return cuda_check(c, cudaGetLastError(), "matrix-free operator");
}

int launch_jvp(fp_ctx* c, const double* V, double* JV, double*) {
    // JV = -(0 * M V - (dR/dW) V) is returned negated by the caller
    int rc;
    const Launchers* t = L(c, rc);
    if (!t) return rc;
    t->matfree(dev_mesh(c), c->stream, c->d_W, V, 0.0, JV);
    return cuda_check(c, cudaGetLastError(), "jvp");
}

int launch_limiter(fp_ctx* c) {
    int rc;
    const Launchers* t = L(c, rc);
    if (!t) return rc;
    const double* trun = c->d_tab + c->hm.tab.data.size() - (size_t)t->ntrun;
    t->limiter(dev_mesh(c), c->stream, c->d_W, c->hm.num.damp_tol, c->hm.num.penalty, trun, c->d_eps, c->d_cip);
    return cuda_check(c, cudaGetLastError(), "limiter");
}

int launch_positivity(fp_ctx* c, double* W, int* n_limited) {
    int rc;
    const Launchers* t = L(c, rc);
    if (!t) return rc;
    int* d_count = reinterpret_cast<int*>(c->d_status) + 1;
    if ((rc = cuda_check(c, cudaMemsetAsync(d_count, 0, sizeof(int), c->stream), "memset"))) return rc;
    t->positivity(dev_mesh(c), c->stream, W, d_count);
    if ((rc = cuda_check(c, cudaGetLastError(), "positivity"))) return rc;
    if (!n_limited) return FP_OK;
    int h = 0;
    if ((rc = cuda_check(c, cudaMemcpyAsync(&h, d_count, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "copy"))) return rc;
    rc = cuda_check(c, cudaStreamSynchronize(c->stream), "sync");
    *n_limited = h;
    return rc;
}

int launch_norms(fp_ctx* c, const double* R, double* norms) {
    int rc;
    const Launchers* t = L(c, rc);
    if (!t) return rc;
    t->norms(dev_mesh(c), c->stream, R, c->d_part);
    if ((rc = cuda_check(c, cudaGetLastError(), "norms"))) return rc;
    const int nb = nblocks(c->hm.nElem), ne = c->hm.model.n_eqs;
    std::vector<double> h;
    if ((rc = read_parts(c, (size_t)nb * ne, h))) return rc;
    for (int m = 0; m < ne; m++) {
        double s = 0;
        for (int b = 0; b < nb; b++) s += h[(size_t)b * ne + m];
        norms[m] = std::sqrt(s);
    }
    return FP_OK;
}

int launch_dt_bound(fp_ctx* c, double* out) {
    int rc;
    const Launchers* t = L(c, rc);
    if (!t) return rc;
    const double factor = c->hm.num.implicit_time ? 1.0 : 2.0 * (c->hm.num.order - 1) + 1;
    t->dtbound(dev_mesh(c), c->stream, c->d_W, factor, c->d_part);
    if ((rc = cuda_check(c, cudaGetLastError(), "dt bound"))) return rc;
    std::vector<double> h;
    if ((rc = read_parts(c, nblocks(c->hm.nElem), h))) return rc;
    double m = 1.0e300;
    for (double v : h) m = std::min(m, v);
    *out = m;
    return FP_OK;
}

int launch_rhs(fp_ctx* c, double a1, double a2, double a3, double* rhs_norm) {
    int rc;
    const Launchers* t = L(c, rc);
    if (!t) return rc;
    prof_begin(c, PH_RHS);
    // moving mesh with the discrete GCL: the current level's mass matrix of this time step
    // (Implicit.applyGCL before the right-hand side and the blocks)
    if (c->d_mass && c->hm.num.gcl && a1 != 0.0) t->gcl_mass(dev_mesh(c), c->stream, a1, a2, a3, c->d_mass);
    t->rhs(dev_mesh(c), c->stream, c->d_W, c->d_Wo, c->d_Wo2, a1, a2, a3, c->d_R, c->d_rhs, c->d_part);
    prof_end(c);
    if ((rc = cuda_check(c, cudaGetLastError(), "rhs"))) return rc;
    if (!rhs_norm) return FP_OK;
    std::vector<double> h;
    if ((rc = read_parts(c, nblocks(c->hm.nElem), h))) return rc;
    double s = 0;
    for (double v : h) s += v;
    *rhs_norm = std::sqrt(s);
    return FP_OK;
}

int launch_fd_jacobian(fp_ctx* c, double a1, double a2, double a3, double* rhs_norm) {
    int rc = launch_rhs(c, a1, a2, a3, rhs_norm);
    if (rc) return rc;
    const Launchers* t = L(c, rc);
    if (!t) return rc;
    prof_begin(c, PH_BLOCKS);
    t->fd(dev_mesh(c), c->stream, c->d_W, c->d_K0, c->d_KR0, c->hm.num.fd_step, a1, c->d_Adiag, c->d_Aneigh);
    prof_end(c);
    return cuda_check(c, cudaGetLastError(), "fd jacobian");
}

int launch_jac_exact(fp_ctx* c, double a1, double a2, double a3, double* rhs_norm) {
    int rc = launch_rhs(c, a1, a2, a3, rhs_norm);
    if (rc) return rc;
    const Launchers* t = L(c, rc);
    if (!t) return rc;
    prof_begin(c, PH_BLOCKS);
    t->jac_exact(dev_mesh(c), c->stream, c->d_W, a1, c->d_Adiag, c->d_Aneigh);
    prof_end(c);
    return cuda_check(c, cudaGetLastError(), "exact jacobian");
}

int launch_jac_exact_factor(fp_ctx* c, double a1, double a2, double a3, double* rhs_norm, void* F, int fp32) {
    int rc = launch_rhs(c, a1, a2, a3, rhs_norm);
    if (rc) return rc;
    const Launchers* t = L(c, rc);
    if (!t) return rc;
    prof_begin(c, PH_BLOCKS);
    t->jac_exact_factor(dev_mesh(c), c->stream, c->d_W, a1, F, fp32);
    prof_end(c);
    return cuda_check(c, cudaGetLastError(), "exact jacobian (factor storage)");
}

int launch_vjp(fp_ctx* c, const double* lam, double* g) {
    int rc;
    const Launchers* t = L(c, rc);
    if (!t) return rc;
    t->vjp(dev_mesh(c), c->stream, c->d_W, lam, g);
    return cuda_check(c, cudaGetLastError(), "vjp");
}

int launch_surface(fp_ctx* c, int kind, int bc, double* out4, double* dIdW) {
    int rc;
    const Launchers* t = L(c, rc);
    if (!t) return rc;
    t->surface(dev_mesh(c), c->stream, c->d_W, kind, bc, c->d_part, dIdW);
    if ((rc = cuda_check(c, cudaGetLastError(), "surface integral"))) return rc;
    const int nb = nblocks(c->hm.nElem);
    std::vector<double> h;
    if ((rc = read_parts(c, (size_t)nb * 4, h))) return rc;
    for (int v = 0; v < 4; v++) {
        double s = 0;
        for (int b = 0; b < nb; b++) s += h[(size_t)b * 4 + v];
        out4[v] = s;
    }
    return FP_OK;
}

}  // namespace fp
