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
    return cuda_check(c, cudaStreamSynchronize(c->stream), "sync");
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
    t->rhs(dev_mesh(c), c->stream, c->d_W, c->d_Wo, c->d_Wo2, a1, a2, a3, c->d_R, c->d_rhs, c->d_part);
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
    t->fd(dev_mesh(c), c->stream, c->d_W, c->d_K0, c->d_KR0, c->hm.num.fd_step, a1, c->d_Adiag, c->d_Aneigh);
    return cuda_check(c, cudaGetLastError(), "fd jacobian");
}

int launch_jac_exact(fp_ctx* c, double a1, double a2, double a3, double* rhs_norm) {
    int rc = launch_rhs(c, a1, a2, a3, rhs_norm);
    if (rc) return rc;
    const Launchers* t = L(c, rc);
    if (!t) return rc;
    t->jac_exact(dev_mesh(c), c->stream, c->d_W, a1, c->d_Adiag, c->d_Aneigh);
    return cuda_check(c, cudaGetLastError(), "exact jacobian");
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
