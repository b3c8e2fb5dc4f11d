// C-ABI entry points (include/flowgpu.h): context, mesh upload, state transfer,
// and the host-side drivers that mirror FlowPro's solver loops
// (LocalExplicitSolver / LocalImplicitSolver, State, CFLSetup) on top of the
// device kernels.  No entry point throws; every failure is a status code with a
// message in fp_last_error().
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <new>
#include <string>
#include <atomic>
#include <chrono>
#include <cmath>
#include <queue>
#include <thread>
#include <vector>

#include "fp_ctx.h"
#include "fp_launch.h"
#include "fp_state.h"

namespace fp {

int set_err(fp_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_check(fp_ctx* c, cudaError_t e, const char* where) {
    if (e == cudaSuccess) return FP_OK;
    return set_err(c, FP_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

void prof_begin(fp_ctx* c, int phase) {
    if (!c->prof_on || c->prof_open) return;
    if ((size_t)(2 * c->prof_used + 2) > c->prof_ev.size()) {
        if (c->prof_ev.size() >= 8192) {  // pool full: settle the recorded intervals first
            cudaStreamSynchronize(c->stream);
            prof_resolve(c);
        } else {
            for (int i = 0; i < 256; i++) {
                cudaEvent_t e;
                if (cudaEventCreate(&e) != cudaSuccess) return;
                c->prof_ev.push_back(e);
            }
            c->prof_ph.resize(c->prof_ev.size() / 2);
        }
    }
    cudaEventRecord(c->prof_ev[2 * c->prof_used], c->stream);
    c->prof_ph[c->prof_used] = phase;
    c->prof_open = true;
}

void prof_end(fp_ctx* c) {
    if (!c->prof_on || !c->prof_open) return;
    cudaEventRecord(c->prof_ev[2 * c->prof_used + 1], c->stream);
    c->prof_used++;
    c->prof_open = false;
}

void prof_resolve(fp_ctx* c) {
    if (!c->prof_on) return;
    for (int k = 0; k < c->prof_used; k++) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, c->prof_ev[2 * k], c->prof_ev[2 * k + 1]) == cudaSuccess) {
            c->prof_ms[c->prof_ph[k]] += ms;
            c->prof_n[c->prof_ph[k]]++;
        }
    }
    c->prof_used = 0;
}

DevMesh dev_mesh(const fp_ctx* c) {
    DevMesh M;
    M.nElem = c->hm.nElem;
    M.ld = c->hm.ld;
    M.geo = c->d_geo;
    M.tt = c->d_tt;
    M.fcode = c->d_fcode;
    M.vwd = c->d_vwd;
    M.vu = c->d_vu;
    M.tab = c->d_tab;
    M.eps = c->d_eps;
    M.cip = c->d_cip;
    M.mass = c->d_mass;
    M.case_of = c->d_case_of;
    M.case_a = c->n_cases > 0 ? c->d_case_a : nullptr;
    M.case_pout = c->n_cases > 0 ? c->d_case_pout : nullptr;
    M.ncases = c->n_cases;
    M.case_live = (c->n_cases > 0 && c->batch_mask) ? c->d_blive : nullptr;
    M.dampConst = c->hm.num.damp_const;
    // DGpure.residuumWall sets beta0 = 0 for a global order 1 with a diffusive model (DGpure.java:287-289)
    M.beta0 = (c->hm.model.is_diffusive && c->hm.num.order == 1) ? 0.0 : c->hm.num.beta0;
    M.P = c->hm.model;
    M.F.nFaces = c->hm.nFaces;
    M.F.ldf = c->hm.ldf;
    M.F.fl = c->d_fl;
    M.F.fk = c->d_fk;
    M.F.fr = c->d_fr;
    M.F.fc = c->d_fc;
    M.F.qmap = c->d_qmap;
    M.F.efc = c->d_efc;
    M.F.G = c->d_G;
    return M;
}

void free_all(fp_ctx* c) {
    for (double* p : c->allocs) cudaFree(p);
    c->allocs.clear();
    if (c->h_scal) cudaFreeHost(c->h_scal);
    c->h_scal = nullptr;
    c->d_Adiag = c->d_Aneigh = c->d_rhs = c->d_K0 = c->d_KR0 = c->d_P64 = nullptr;
    c->d_mass = nullptr;
    c->d_vu = nullptr;
    c->n_cases = 0;
    c->case_e0.clear();
    c->d_case_of = nullptr;
    c->d_case_pout = c->d_case_a = c->d_case_W0 = nullptr;
    c->batch_ready = false;
    c->batch_kmax = c->batch_nch = 0;
    c->d_bch0 = c->d_bch1 = c->d_bcptr = c->d_bmask = nullptr;
    c->d_blive = c->d_bkc = nullptr;
    c->batch_mask = false;
    c->d_bpart = c->d_bcase = nullptr;
    c->d_P32 = nullptr;
    c->d_V = nullptr;
    c->kry_m = 0;
    c->blocks_ready = false;
    c->rhs_ready = false;
    c->prec_ready = -1;
    c->prec_kind = -1;
    c->d_w = c->d_aux = c->d_r = c->d_x = c->d_b = c->d_tmp = nullptr;
    c->d_io2 = nullptr;
    pipe_release(c);
    c->pipe_e.clear();
    c->pipe_f.clear();
    c->pipe_need.clear();
    ilu_release(c);
}

// element-major host layout  <->  field-major device layout
__global__ void k_to_soa(int nElem, int ld, int nc, const double* __restrict__ in, double* __restrict__ out) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)nElem * nc) return;
    const int e = (int)(t / nc), cc = (int)(t - (size_t)e * nc);
    out[(size_t)cc * ld + e] = in[t];
}
__global__ void k_from_soa(int nElem, int ld, int nc, const double* __restrict__ in, double* __restrict__ out) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)nElem * nc) return;
    const int e = (int)(t / nc), cc = (int)(t - (size_t)e * nc);
    out[t] = in[(size_t)cc * ld + e];
}

int host_to_soa(fp_ctx* c, const double* h, double* d) {
    size_t n = (size_t)c->hm.nElem * c->nc;
    int rc = upload(c, c->d_io, h, n);
    if (rc) return rc;
    k_to_soa<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->hm.nElem, c->hm.ld, c->nc, c->d_io, d);
    return cuda_check(c, cudaGetLastError(), "to soa");
}

int soa_to_host(fp_ctx* c, const double* d, double* h) {
    size_t n = (size_t)c->hm.nElem * c->nc;
    k_from_soa<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->hm.nElem, c->hm.ld, c->nc, d, c->d_io);
    int rc = cuda_check(c, cudaGetLastError(), "from soa");
    if (rc) return rc;
    rc = cuda_check(c, cudaMemcpyAsync(h, c->d_io, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "download");
    if (rc) return rc;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "sync");
}

int need_mesh(fp_ctx* c) {
    if (!c) return FP_ERR_ARG;
    if (!c->has_mesh) return set_err(c, FP_ERR_STATE, "no mesh uploaded");
    return cudaSetDevice(c->device) == cudaSuccess ? FP_OK : set_err(c, FP_ERR_CUDA, "cudaSetDevice");
}

// the right-hand side of the implicit step (every implicit path)
int ensure_rhs(fp_ctx* c) {
    if (c->d_rhs) return FP_OK;
    return dalloc(c, &c->d_rhs, (size_t)c->nc * c->hm.ld);
}

// the operator's element blocks (assembled paths; 69 GB in FP64 for 693,600 tetrahedra of
// 50 unknowns, so the matrix-free path never allocates them)
int ensure_implicit(fp_ctx* c) {
    int rc;
    if ((rc = ensure_rhs(c))) return rc;
    if (c->d_Adiag) return FP_OK;
    const size_t ld = c->hm.ld, nc = c->nc, nf = c->hm.nf;
    if ((rc = dalloc(c, &c->d_Adiag, nc * nc * ld)) || (rc = dalloc(c, &c->d_Aneigh, nf * nc * nc * ld)) ||
        (rc = dalloc(c, &c->d_K0, nc * ld)) || (rc = dalloc(c, &c->d_KR0, nf * nc * ld)))
        return rc;
    return FP_OK;
}

// Krylov basis and work vectors (the block-Jacobi inverses are allocated by the
// factorisation that needs them)
int ensure_krylov(fp_ctx* c, int m, int) {
    int rc;
    if (m > c->kry_m) {
        if ((rc = dalloc(c, &c->d_V, (size_t)(m + 1) * c->nvec))) return rc;
        c->kry_m = m;
    }
    if (!c->d_w) {
        if ((rc = dalloc(c, &c->d_w, c->nvec)) || (rc = dalloc(c, &c->d_aux, c->nvec)) || (rc = dalloc(c, &c->d_r, c->nvec)) ||
            (rc = dalloc(c, &c->d_x, c->nvec)) || (rc = dalloc(c, &c->d_b, c->nvec)) || (rc = dalloc(c, &c->d_tmp, c->nvec)))
            return rc;
    }
    return FP_OK;
}

long long ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count();
}

// LocalImplicitSolver.saveData / LocalExplicitSolver.saveData (LocalImplicitSolver.java:326-344):
// state.txt, W.txt (integral averages), We.txt (coefficients), artificialViscosity.txt
int save_data(fp_ctx* c, const State& st, long long cpu_ms) {
    if (c->io_dir.empty()) return FP_OK;
    const HostMesh& h = c->hm;
    const int nE = h.nElem, nb = h.tab.nb, ne = h.model.n_eqs, nc = c->nc;
    std::vector<double> W((size_t)nE * nc), eps(nE), avg((size_t)nE * ne), av((size_t)nE * ne);
    int rc = soa_to_host(c, c->d_W, W.data());
    if (rc) return rc;
    if ((rc = cuda_check(c, cudaMemcpyAsync(eps.data(), c->d_eps, nE * sizeof(double), cudaMemcpyDeviceToHost, c->stream),
                         "copy")) ||
        (rc = cuda_check(c, cudaStreamSynchronize(c->stream), "sync")))
        return rc;
    const double* Is = h.tab.data.data() + h.tab.o_Is;
    for (int e = 0; e < nE; e++)
        for (int m = 0; m < ne; m++) {
            double v = 0;
            for (int j = 0; j < nb; j++) v = v + W[(size_t)e * nc + m * nb + j] * Is[j];
            avg[(size_t)e * ne + m] = v;
            av[(size_t)e * ne + m] = eps[e];  // + dampInner[m], zero without the inner damping
        }
    IoState s;
    s.t = st.t;
    s.steps = st.steps;
    s.cpu_ms = cpu_ms;
    s.residuum = st.residuum;
    s.cfl = st.currentCFL;
    s.dt = st.dt;
    if (st.nNorm >= 5) s.normalisation = st.normalisation;
    s.order = h.num.order;
    if (io_save_state(c->io_dir, s) || io_save_rows(c->io_dir, "W.txt", avg.data(), nE, ne) ||
        io_save_rows(c->io_dir, "We.txt", W.data(), nE, nc) ||
        io_save_rows(c->io_dir, "artificialViscosity.txt", av.data(), nE, ne))
        return set_err(c, FP_ERR_ARG, "cannot write the solver files into " + c->io_dir);
    return FP_OK;
}

// per finished step: residuum.txt row, saveData every save_rate steps, STOP request
// (LocalImplicitSolver.java:244-275); returns true when a stop was requested
bool step_output(fp_ctx* c, const State& st, long long cpu_ms, int* rc) {
    *rc = FP_OK;
    if (c->io_dir.empty()) return false;
    if (io_append_residuum(c->io_dir, st.residuum, st.t, (double)cpu_ms, st.equationResiduum)) {
        *rc = set_err(c, FP_ERR_ARG, "cannot append to residuum.txt in " + c->io_dir);
        return false;
    }
    if (c->io_save_rate > 0 && st.steps % c->io_save_rate == 0 && (*rc = save_data(c, st, cpu_ms))) return false;
    return io_stop_requested(c->io_dir);
}

}  // namespace fp

using namespace fp;

extern "C" {

int fp_ctx_create(int device, fp_ctx** out) {
    if (!out) return FP_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return FP_ERR_CUDA;
    if (device < 0 || device >= n) return FP_ERR_ARG;
    fp_ctx* c = new (std::nothrow) fp_ctx();
    if (!c) return FP_ERR_ARG;
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return FP_ERR_CUDA;
    }
    *out = c;
    return FP_OK;
}

int fp_ctx_destroy(fp_ctx* c) {
    if (!c) return FP_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_all(c);
    for (cudaEvent_t e : c->pipe_ev) cudaEventDestroy(e);
    for (cudaEvent_t e : c->prof_ev) cudaEventDestroy(e);
    if (c->s_h2d) cudaStreamDestroy(c->s_h2d);
    if (c->s_d2h) cudaStreamDestroy(c->s_d2h);
    if (c->s_elem) cudaStreamDestroy(c->s_elem);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return FP_OK;
}

const char* fp_last_error(const fp_ctx* c) { return c ? c->err.c_str() : "null context"; }

int fp_ctx_set_stream(fp_ctx* c, uintptr_t stream) {
    if (!c) return FP_ERR_ARG;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    if (stream == 0) {
        c->own_stream = true;
        return cuda_check(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream");
    }
    c->own_stream = false;
    c->stream = reinterpret_cast<cudaStream_t>(stream);
    return FP_OK;
}

int fp_model_from_properties(const char* props, fp_model_params* model, fp_num_params* num) {
    if (!model || !num) return FP_ERR_ARG;
    std::string err;
    return model_from_properties(props, *model, *num, err);
}

int fp_create_neighbor_matrix(int dim, int n_elements, const int* elements, int n_boundary, const int* boundary,
                              int* neighbors) {
    if ((dim != 2 && dim != 3) || n_elements <= 0 || !elements || !neighbors || (n_boundary > 0 && !boundary)) return FP_ERR_ARG;
    return create_neighbor_matrix(dim, n_elements, elements, n_boundary, boundary, neighbors);
}

int fp_wall_distance(int dim, int n_vertices, const double* vertices, int n_elements, const int* elements,
                     const int* neighbors, int source_bc, double* distance) {
    if ((dim != 2 && dim != 3) || n_vertices <= 0 || n_elements <= 0 || !vertices || !elements || !neighbors || !distance)
        return FP_ERR_ARG;
    const int nv = dim + 1, nf = dim + 1;
    static const int F3[4][3] = {{0, 2, 1}, {0, 1, 3}, {1, 2, 3}, {2, 0, 3}};
    std::vector<double> d(n_vertices, HUGE_VAL);
    // vertex adjacency through element edges
    std::vector<std::vector<int>> adj(n_vertices);
    for (int e = 0; e < n_elements; e++)
        for (int a = 0; a < nv; a++)
            for (int b = 0; b < nv; b++)
                if (a != b) {
                    const int pa = elements[(size_t)e * nv + a], pb = elements[(size_t)e * nv + b];
                    if (pa < 0 || pa >= n_vertices || pb < 0 || pb >= n_vertices) return FP_ERR_ARG;
                    adj[pa].push_back(pb);
                }
    using QE = std::pair<double, int>;
    std::priority_queue<QE, std::vector<QE>, std::greater<QE>> q;
    for (int e = 0; e < n_elements; e++)
        for (int k = 0; k < nf; k++) {
            if (neighbors[(size_t)e * nf + k] != source_bc) continue;
            for (int i = 0; i < dim; i++) {
                const int fv = dim == 2 ? (i == 0 ? k : (k + 1) % 3) : F3[k][i];
                const int v = elements[(size_t)e * nv + fv];
                if (d[v] != 0.0) {
                    d[v] = 0.0;
                    q.push({0.0, v});
                }
            }
        }
    while (!q.empty()) {
        const QE top = q.top();
        q.pop();
        const int v = top.second;
        if (top.first > d[v]) continue;
        for (int w : adj[v]) {
            double L = 0;
            for (int c = 0; c < dim; c++) {
                const double t = vertices[(size_t)w * dim + c] - vertices[(size_t)v * dim + c];
                L += t * t;
            }
            const double y = d[v] + std::sqrt(L);
            if (y < d[w]) {
                d[w] = y;
                q.push({y, w});
            }
        }
    }
    bool unreached = false;
    for (int i = 0; i < n_vertices; i++) unreached = unreached || std::isinf(d[i]);
    for (int i = 0; i < n_vertices; i++) distance[i] = unreached ? 1e30 : d[i];
    return FP_OK;
}

int fp_element_ordering(int dim, int n_elements, const int* neighbors, int ordering, int* order) {
    if ((dim != 2 && dim != 3) || n_elements <= 0 || !neighbors || !order) return FP_ERR_ARG;
    if (ordering == 1) {
        std::vector<int> o = reverse_cuthill_mckee(n_elements, dim + 1, neighbors);
        std::copy(o.begin(), o.end(), order);
    } else {
        for (int i = 0; i < n_elements; i++) order[i] = i;
    }
    return FP_OK;
}

int fp_mesh_upload(fp_ctx* c, const fp_mesh_desc* desc, const fp_model_params* model, const fp_num_params* num) {
    if (!c || !desc || !model || !num) return FP_ERR_ARG;
    if (cudaSetDevice(c->device) != cudaSuccess) return set_err(c, FP_ERR_CUDA, "cudaSetDevice");
    cudaStreamSynchronize(c->stream);
    free_all(c);
    c->has_mesh = false;
    HostMesh hm;
    int rc = build_host_mesh(*desc, *model, *num, hm, c->err);
    if (rc) return rc;
    const int n_eqs = model->model == FP_MODEL_SCALAR_TEST         ? 1
                      : model->model == FP_MODEL_SPALART_ALLMARAS   ? model->dim + 3
                      : model->model == FP_MODEL_ADIABATIC_EULERS   ? model->dim + 1
                                                                    : model->dim + 2;
    if (model->n_eqs != n_eqs)
        return set_err(c, FP_ERR_ARG, "n_eqs does not match the model");
    c->hm = std::move(hm);
    const HostMesh& h = c->hm;
    c->h_elements.assign(desc->elements, desc->elements + (size_t)desc->n_elements * (desc->dim + 1));
    c->h_neighbors.assign(desc->neighbors, desc->neighbors + (size_t)desc->n_elements * (desc->dim + 1));
    if (desc->wall_distance)
        c->h_wd.assign(desc->wall_distance, desc->wall_distance + desc->n_vertices);
    else
        c->h_wd.clear();
    c->nc = h.tab.nb * model->n_eqs;
    c->nvec = (size_t)c->nc * h.ld;
    const size_t ld = h.ld;
    if ((rc = dalloc(c, &c->d_geo, h.geo.size(), false)) || (rc = upload(c, c->d_geo, h.geo.data(), h.geo.size()))) return rc;
    std::vector<double> tab = h.tab.data;
    if ((rc = dalloc(c, &c->d_tab, tab.size(), false)) || (rc = upload(c, c->d_tab, tab.data(), tab.size()))) return rc;
    if ((rc = dalloc(c, &c->d_vwd, h.vwd.size(), false)) || (rc = upload(c, c->d_vwd, h.vwd.data(), h.vwd.size()))) return rc;
    if (!h.vu.empty()) {
        if ((rc = dalloc(c, &c->d_vu, h.vu.size(), false)) || (rc = upload(c, c->d_vu, h.vu.data(), h.vu.size()))) return rc;
    }
    if ((rc = dalloc(c, &c->d_tt, h.tt.size(), false)) || (rc = upload(c, c->d_tt, h.tt.data(), h.tt.size()))) return rc;
    if ((rc = dalloc(c, &c->d_fcode, h.fcode.size(), false)) || (rc = upload(c, c->d_fcode, h.fcode.data(), h.fcode.size())))
        return rc;
    if ((rc = dalloc(c, &c->d_order, h.order.size(), false)) || (rc = upload(c, c->d_order, h.order.data(), h.order.size())))
        return rc;
    if (!h.faceMode) return set_err(c, FP_ERR_UNSUPPORTED, "face quadrature rule is not symmetric under vertex permutations");
    if ((rc = dalloc(c, &c->d_fl, h.fl.size(), false)) || (rc = upload(c, c->d_fl, h.fl.data(), h.fl.size())) ||
        (rc = dalloc(c, &c->d_fk, h.fk.size(), false)) || (rc = upload(c, c->d_fk, h.fk.data(), h.fk.size())) ||
        (rc = dalloc(c, &c->d_fr, h.fr.size(), false)) || (rc = upload(c, c->d_fr, h.fr.data(), h.fr.size())) ||
        (rc = dalloc(c, &c->d_fc, h.fc.size(), false)) || (rc = upload(c, c->d_fc, h.fc.data(), h.fc.size())) ||
        (rc = dalloc(c, &c->d_qmap, h.qmap.size(), false)) || (rc = upload(c, c->d_qmap, h.qmap.data(), h.qmap.size())) ||
        (rc = dalloc(c, &c->d_efc, h.efc.size(), false)) || (rc = upload(c, c->d_efc, h.efc.data(), h.efc.size())) ||
        (rc = dalloc(c, &c->d_G, (size_t)2 * h.tab.nqf * model->n_eqs * h.ldf)))
        return rc;
    if ((rc = dalloc(c, &c->d_eps, ld)) || (rc = dalloc(c, &c->d_cip, ld))) return rc;
    if ((rc = dalloc(c, &c->d_W, c->nvec)) || (rc = dalloc(c, &c->d_Wo, c->nvec)) || (rc = dalloc(c, &c->d_Wo2, c->nvec)) ||
        (rc = dalloc(c, &c->d_R, c->nvec)) || (rc = dalloc(c, &c->d_io, c->nvec)))
        return rc;
    for (int i = 0; i < 3; i++)
        if ((rc = dalloc(c, &c->d_Wst[i], c->nvec))) return rc;
    // partial sums: per-block reductions of the element kernels (8 per block of 128) and the
    // fused Gram-Schmidt dots (592 blocks x up to 201 basis vectors)
    size_t npart = std::max<size_t>((size_t)((h.nElem + 127) / 128) * 8, (size_t)592 * 201);
    if ((rc = dalloc(c, &c->d_part, npart)) || (rc = dalloc(c, &c->d_scal, 1024)) || (rc = dalloc(c, &c->d_status, 4)))
        return rc;
    if (cudaMallocHost(&c->h_scal, 1024 * sizeof(double)) != cudaSuccess) return set_err(c, FP_ERR_CUDA, "cudaMallocHost");
    rc = cuda_check(c, cudaStreamSynchronize(c->stream), "upload sync");
    if (rc) return rc;
    c->has_mesh = true;
    return fp_state_init_const(c);
}

int fp_mesh_info(const fp_ctx* c, int* n_elements, int* n_basis, int* n_eqs, int* n_faces) {
    if (!c || !c->has_mesh) return FP_ERR_STATE;
    if (n_elements) *n_elements = c->hm.nElem;
    if (n_basis) *n_basis = c->hm.tab.nb;
    if (n_eqs) *n_eqs = c->hm.model.n_eqs;
    if (n_faces) *n_faces = c->hm.nf;
    return FP_OK;
}

int fp_dof_order(const fp_ctx* c, int* pos) {
    if (!c || !c->has_mesh || !pos) return FP_ERR_STATE;
    for (int e = 0; e < c->hm.nElem; e++) pos[e] = c->hm.rank[e];
    return FP_OK;
}

int fp_geometry(const fp_ctx* c, double* area, double* elem_size, double* xs) {
    if (!c || !c->has_mesh) return FP_ERR_STATE;
    const HostMesh& h = c->hm;
    if (area) std::copy(h.area.begin(), h.area.end(), area);
    if (elem_size) std::copy(h.elemSize.begin(), h.elemSize.end(), elem_size);
    if (xs) std::copy(h.xs.begin(), h.xs.end(), xs);
    return FP_OK;
}

int fp_mass_matrix(const fp_ctx* c, double* mass, double* basis_weights) {
    if (!c || !c->has_mesh) return FP_ERR_STATE;
    const HostMesh& h = c->hm;
    const RefTables& t = h.tab;
    const int nb = t.nb, nq = t.nqv, JAC = h.dim * h.dim;
    const double* w = t.data.data() + t.o_w;
    const double* phi = t.data.data() + t.o_phi;  // [q][j]
    for (int e = 0; e < h.nElem; e++) {
        const double jac = h.geo[(size_t)JAC * h.ld + e];  // affine: Int.JacobianVolume[p] at every p
        for (int i = 0; i < nb; i++) {
            if (mass)
                for (int j = 0; j < nb; j++) {
                    double m = 0;
                    for (int p = 0; p < nq; p++) m = m + jac * w[p] * phi[p * nb + i] * phi[p * nb + j];
                    mass[((size_t)e * nb + i) * nb + j] = m;
                }
            if (basis_weights) {
                double s = 0;
                for (int p = 0; p < nq; p++) s = s + jac * w[p] * phi[p * nb + i] / h.area[e];
                basis_weights[(size_t)e * nb + i] = s;
            }
        }
    }
    return FP_OK;
}

static double* state_ptr(fp_ctx* c, int which) { return which == 0 ? c->d_W : which == 1 ? c->d_Wo : which == 2 ? c->d_Wo2 : nullptr; }

int fp_state_set(fp_ctx* c, int which, const double* w) {
    int rc = need_mesh(c);
    if (rc) return rc;
    double* d = state_ptr(c, which);
    if (!d || !w) return set_err(c, FP_ERR_ARG, "bad state index or null array");
    rc = host_to_soa(c, w, d);
    if (rc) return rc;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "sync");
}

int fp_state_get(fp_ctx* c, int which, double* w) {
    int rc = need_mesh(c);
    if (rc) return rc;
    double* d = which == 3 ? c->d_R : state_ptr(c, which);
    if (!d || !w) return set_err(c, FP_ERR_ARG, "bad state index or null array");
    return soa_to_host(c, d, w);
}

int fp_state_init_const(fp_ctx* c) {
    int rc = need_mesh(c);
    if (rc) return rc;
    double w0[8];
    const_init_condition(c->hm.model, w0);
    const int nb = c->hm.tab.nb, ne = c->hm.model.n_eqs;
    std::vector<double> h((size_t)c->hm.nElem * c->nc);
    for (int e = 0; e < c->hm.nElem; e++)
        for (int m = 0; m < ne; m++)
            for (int j = 0; j < nb; j++) h[(size_t)e * c->nc + m * nb + j] = w0[m];
    for (int which = 0; which < 3; which++)
        if ((rc = host_to_soa(c, h.data(), state_ptr(c, which)))) return rc;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "sync");
}

int fp_limiter(fp_ctx* c) {
    int rc = need_mesh(c);
    if (rc) return rc;
    return launch_limiter(c);
}

int fp_limiter_get(const fp_ctx* cc, double* eps, double* c_ip) {
    fp_ctx* c = const_cast<fp_ctx*>(cc);
    int rc = need_mesh(c);
    if (rc) return rc;
    size_t n = c->hm.nElem;
    if (eps && (rc = cuda_check(c, cudaMemcpyAsync(eps, c->d_eps, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "copy")))
        return rc;
    if (c_ip && (rc = cuda_check(c, cudaMemcpyAsync(c_ip, c->d_cip, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "copy")))
        return rc;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "sync");
}

int fp_residual(fp_ctx* c, const double* w, double* r) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if (w && r) return launch_residual_pipelined(c, w, r);
    if (w && (rc = host_to_soa(c, w, c->d_W))) return rc;
    if ((rc = launch_residual(c, c->d_W, c->d_R))) return rc;
    if (r) return soa_to_host(c, c->d_R, r);
    return FP_OK;
}

int fp_residual_repeat(fp_ctx* c, int n) {
    int rc = need_mesh(c);
    if (rc) return rc;
    for (int i = 0; i < n; i++)
        if ((rc = launch_residual(c, c->d_W, c->d_R))) return rc;
    return FP_OK;
}

int fp_residual_timed(fp_ctx* c, int n, double* ms_face, double* ms_elem) {
    int rc = need_mesh(c);
    if (rc) return rc;
    cudaEvent_t ev[3];
    for (int i = 0; i < 3; i++)
        if ((rc = cuda_check(c, cudaEventCreate(&ev[i]), "event"))) return rc;
    double tf = 0, te = 0;
    for (int i = 0; i < n && !rc; i++) {
        rc = launch_residual_timed(c, c->d_W, c->d_R, ev);
        if (!rc) rc = cuda_check(c, cudaEventSynchronize(ev[2]), "event sync");
        float a = 0, b = 0;
        if (!rc) rc = cuda_check(c, cudaEventElapsedTime(&a, ev[0], ev[1]), "event time");
        if (!rc) rc = cuda_check(c, cudaEventElapsedTime(&b, ev[1], ev[2]), "event time");
        tf += a;
        te += b;
    }
    for (int i = 0; i < 3; i++) cudaEventDestroy(ev[i]);
    if (ms_face) *ms_face = tf;
    if (ms_elem) *ms_elem = te;
    return rc;
}

int fp_jvp(fp_ctx* c, const double* v, double* dr) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if (!v || !dr) return set_err(c, FP_ERR_ARG, "null array");
    if ((rc = ensure_krylov(c, 1, -1))) return rc;
    if ((rc = host_to_soa(c, v, c->d_tmp)) || (rc = launch_jvp(c, c->d_tmp, c->d_aux, nullptr))) return rc;
    if ((rc = vec_axpby(c, c->d_aux, 0.0, c->d_aux, -1.0))) return rc;  // the operator returns -(dR/dW) v
    return soa_to_host(c, c->d_aux, dr);
}

int fp_assemble_exact(fp_ctx* c, int bdf_order, double dt, double dto) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if ((rc = ensure_implicit(c))) return rc;
    if (dt > 0) {
        bdf_coef(bdf_order, dt, dto, c->a_coef);
    } else {
        c->a_coef[0] = c->a_coef[1] = c->a_coef[2] = 0.0;
    }
    c->bdf_order = bdf_order;
    if ((rc = launch_jac_exact(c, c->a_coef[0], c->a_coef[1], c->a_coef[2], &c->last_rhs_norm))) return rc;
    c->blocks_ready = true;
    c->rhs_ready = true;
    c->prec_ready = -1;
    return FP_OK;
}

int fp_assemble_preconditioner(fp_ctx* c, int bdf_order, double dt, double dto, int preconditioner, int precision) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if (preconditioner == FP_PREC_ILU0) preconditioner = FP_PREC_BLOCKILU0;
    if (precision != FP_PREC_FP32 && precision != FP_PREC_FP64) return set_err(c, FP_ERR_ARG, "bad precision");
    if (preconditioner == FP_PREC_BLOCKJACOBI) {
        if ((rc = fp_assemble_exact(c, bdf_order, dt, dto)) || (rc = prec_factor(c, preconditioner, precision))) return rc;
        return FP_OK;
    }
    if ((rc = ensure_rhs(c))) return rc;
    if (dt > 0) {
        bdf_coef(bdf_order, dt, dto, c->a_coef);
    } else {
        c->a_coef[0] = c->a_coef[1] = c->a_coef[2] = 0.0;
    }
    c->bdf_order = bdf_order;
    c->prec_ready = -1;
    c->blocks_ready = false;  // stored operator blocks, if any, belong to an earlier state
    if (preconditioner == FP_PREC_NONE) {
        if ((rc = launch_rhs(c, c->a_coef[0], c->a_coef[1], c->a_coef[2], &c->last_rhs_norm))) return rc;
    } else if (preconditioner == FP_PREC_BLOCKILU0) {
        void* F = nullptr;
        if ((rc = ilu_prepare_direct(c, precision, &F)) ||
            (rc = launch_jac_exact_factor(c, c->a_coef[0], c->a_coef[1], c->a_coef[2], &c->last_rhs_norm, F,
                                          precision == FP_PREC_FP32)) ||
            (rc = [&] {
                prof_begin(c, PH_FACTOR);
                const int r = ilu_factor_direct(c, precision);
                prof_end(c);
                return r;
            }()))
            return rc;
    } else {
        return set_err(c, FP_ERR_UNSUPPORTED, "preconditioner not available");
    }
    c->rhs_ready = true;
    c->prec_kind = preconditioner;
    c->prec_ready = precision;
    return FP_OK;
}

int fp_vjp(fp_ctx* c, const double* lambda, double* g) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if (!lambda || !g) return set_err(c, FP_ERR_ARG, "null array");
    if ((rc = ensure_krylov(c, 1, -1))) return rc;
    if ((rc = host_to_soa(c, lambda, c->d_tmp)) || (rc = launch_vjp(c, c->d_tmp, c->d_aux))) return rc;
    return soa_to_host(c, c->d_aux, g);
}

int fp_positivity_limiter(fp_ctx* c, int* n_limited) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if (!c->hm.num.positivity_limiter) {
        if (n_limited) *n_limited = 0;
        return FP_OK;
    }
    return launch_positivity(c, c->d_W, n_limited);
}

int fp_residuum_norms(fp_ctx* c, double* norms) {
    int rc = need_mesh(c);
    if (rc) return rc;
    return launch_norms(c, c->d_R, norms);
}

int fp_time_step_bound(fp_ctx* c, double* v) {
    int rc = need_mesh(c);
    if (rc) return rc;
    return launch_dt_bound(c, v);
}

// RK3 stages 1-6 with the limiter before the residual stages and the positivity limiter
// after the copy stages (LocalExplicitSolver.LocalTimeStepIterator.iterate, :267-288)
int fp_rk3_step(fp_ctx* c, double dt) {
    int rc = need_mesh(c);
    if (rc) return rc;
    const size_t bytes = c->nvec * sizeof(double);
    double *W1 = c->d_Wst[0], *W2 = c->d_Wst[1], *Wn = c->d_Wst[2];
    const bool pos = c->hm.num.positivity_limiter != 0;
    // stage 1: W1 = Wo + dt M^-1 R(W), spatial residual kept
    if ((rc = launch_limiter(c)) || (rc = launch_rk_stage(c, c->d_W, c->d_Wo, c->d_Wo, 0.0, 1.0, dt, W1, c->d_R))) return rc;
    // stage 2: W = W1
    if ((rc = cuda_check(c, cudaMemcpyAsync(c->d_W, W1, bytes, cudaMemcpyDeviceToDevice, c->stream), "copy"))) return rc;
    if (pos && (rc = launch_positivity(c, c->d_W, nullptr))) return rc;
    // stage 3: W2 = 3/4 Wo + 1/4 (W1 + dt M^-1 R(W))
    if ((rc = launch_limiter(c)) || (rc = launch_rk_stage(c, c->d_W, c->d_Wo, W1, 0.75, 0.25, dt, W2, nullptr))) return rc;
    if ((rc = cuda_check(c, cudaMemcpyAsync(c->d_W, W2, bytes, cudaMemcpyDeviceToDevice, c->stream), "copy"))) return rc;
    if (pos && (rc = launch_positivity(c, c->d_W, nullptr))) return rc;
    // stage 5: Wn = 1/3 Wo + 2/3 (W2 + dt M^-1 R(W))
    if ((rc = launch_limiter(c)) || (rc = launch_rk_stage(c, c->d_W, c->d_Wo, W2, 1.0 / 3, 2.0 / 3, dt, Wn, nullptr))) return rc;
    if ((rc = cuda_check(c, cudaMemcpyAsync(c->d_W, Wn, bytes, cudaMemcpyDeviceToDevice, c->stream), "copy"))) return rc;
    if (pos && (rc = launch_positivity(c, c->d_W, nullptr))) return rc;
    return FP_OK;
}

int fp_copy_w2wo(fp_ctx* c) {
    int rc = need_mesh(c);
    if (rc) return rc;
    const size_t bytes = c->nvec * sizeof(double);
    if ((rc = cuda_check(c, cudaMemcpyAsync(c->d_Wo2, c->d_Wo, bytes, cudaMemcpyDeviceToDevice, c->stream), "copy"))) return rc;
    return cuda_check(c, cudaMemcpyAsync(c->d_Wo, c->d_W, bytes, cudaMemcpyDeviceToDevice, c->stream), "copy");
}

int fp_copy_wo2w(fp_ctx* c) {
    int rc = need_mesh(c);
    if (rc) return rc;
    return cuda_check(c, cudaMemcpyAsync(c->d_W, c->d_Wo, c->nvec * sizeof(double), cudaMemcpyDeviceToDevice, c->stream), "copy");
}

int fp_assemble(fp_ctx* c, int bdf_order, double dt, double dto) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if ((rc = ensure_implicit(c))) return rc;
    if (dt > 0) {
        bdf_coef(bdf_order, dt, dto, c->a_coef);
    } else {  // steady operator (Element.exportLocalJacobiMatrix / exportLocalR)
        c->a_coef[0] = c->a_coef[1] = c->a_coef[2] = 0.0;
    }
    c->bdf_order = bdf_order;
    if ((rc = launch_fd_jacobian(c, c->a_coef[0], c->a_coef[1], c->a_coef[2], &c->last_rhs_norm))) return rc;
    c->blocks_ready = true;
    c->rhs_ready = true;
    c->prec_ready = -1;
    return FP_OK;
}

int fp_assemble_residuum(fp_ctx* c, int bdf_order, double dt, double dto, double* rhs_norm) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if ((rc = ensure_rhs(c))) return rc;
    if (dt > 0) {
        bdf_coef(bdf_order, dt, dto, c->a_coef);
    } else {  // steady operator (Element.exportLocalJacobiMatrix / exportLocalR)
        c->a_coef[0] = c->a_coef[1] = c->a_coef[2] = 0.0;
    }
    c->bdf_order = bdf_order;
    double nrm = 0;
    if ((rc = launch_rhs(c, c->a_coef[0], c->a_coef[1], c->a_coef[2], &nrm))) return rc;
    c->rhs_ready = true;
    if (rhs_norm) *rhs_norm = nrm;
    return FP_OK;
}

int fp_blocks_get(fp_ctx* c, double* diag, double* neigh, double* rhs) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if (!c->blocks_ready) return set_err(c, FP_ERR_STATE, "no assembled blocks");
    const int nE = c->hm.nElem, nc = c->nc, nf = c->hm.nf;
    const size_t ld = c->hm.ld, nb = (size_t)nc * nc * ld;
    std::vector<double> A(nb), B(nf * nb);
    if ((rc = cuda_check(c, cudaMemcpyAsync(A.data(), c->d_Adiag, nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "copy")) ||
        (rc = cuda_check(c, cudaMemcpyAsync(B.data(), c->d_Aneigh, nf * nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "copy")) ||
        (rc = cuda_check(c, cudaStreamSynchronize(c->stream), "sync")))
        return rc;
    // reference storage: ADiag[i = perturbed][j = residual] = A[j][i]
    for (int e = 0; e < nE; e++)
        for (int i = 0; i < nc; i++)
            for (int j = 0; j < nc; j++) {
                if (diag) diag[((size_t)e * nc + i) * nc + j] = A[((size_t)j * nc + i) * ld + e];
                if (neigh)
                    for (int k = 0; k < nf; k++)
                        neigh[(((size_t)e * nf + k) * nc + i) * nc + j] =
                            c->hm.tt[(size_t)k * ld + e] > -1 ? B[(size_t)k * nb + ((size_t)j * nc + i) * ld + e] : 0.0;
            }
    if (rhs) return soa_to_host(c, c->d_rhs, rhs);
    return FP_OK;
}

int fp_linear_solve(fp_ctx* c, int jacobian, int preconditioner, int precision, int restart, int max_restarts, double tol,
                    double* x, int* iterations, double* rel_residual) {
    if (preconditioner == FP_PREC_ILU0) preconditioner = FP_PREC_BLOCKILU0;  // same factorisation (header)
    int rc = need_mesh(c);
    if (rc) return rc;
    if (jacobian == FP_JAC_MATRIXFREE ? !c->rhs_ready : !c->blocks_ready)
        return set_err(c, FP_ERR_STATE, "call fp_assemble first");
    if (restart < 1 || max_restarts < 1 || restart > 200) return set_err(c, FP_ERR_ARG, "bad GMRES sizes");
    if ((rc = ensure_krylov(c, restart, precision))) return rc;
    if (c->prec_ready != precision || c->prec_kind != preconditioner) {
        if (preconditioner != FP_PREC_NONE && !c->blocks_ready)
            return set_err(c, FP_ERR_STATE, "no assembled blocks to factorise (fp_assemble or fp_assemble_preconditioner)");
        if ((rc = prec_factor(c, preconditioner, precision))) return rc;
    }
    if ((rc = vec_copy(c, c->d_b, c->d_rhs))) return rc;
    if ((rc = cuda_check(c, cudaMemsetAsync(c->d_x, 0, c->nvec * sizeof(double), c->stream), "memset"))) return rc;
    int it = 0;
    double rel = 0;
    int grc = gmres(c, jacobian, preconditioner, restart, max_restarts, tol, &it, &rel);
    if (preconditioner == FP_PREC_BLOCKILU0 && (grc == FP_OK || grc == FP_ERR_NOT_CONVERGED) && (rc = ilu_check(c)))
        return rc;
    if (iterations) *iterations = it;
    if (rel_residual) *rel_residual = rel;
    if (grc && grc != FP_ERR_NOT_CONVERGED) return grc;
    if (x && (rc = soa_to_host(c, c->d_x, x))) return rc;
    return grc;
}

int fp_update_w(fp_ctx* c) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if (!c->d_x) return set_err(c, FP_ERR_STATE, "no linear-solve update");
    return vec_add_scaled(c, c->d_W, c->d_x, 1.0);
}

// LocalExplicitSolver.solve (LocalExplicitSolver.java:115-195); solver files when fp_solver_output names a directory
int fp_solve_explicit(fp_ctx* c, int steps, double cfl, double target, double* out) {
    int rc = need_mesh(c);
    if (rc) return rc;
    State st;
    st.cfl = cfl > 0 ? cfl : 1;
    st.vary = cfl <= 0;
    std::vector<double> norms(c->hm.model.n_eqs);
    const auto t_start = std::chrono::steady_clock::now();
    for (int s = 0; s < steps && st.residuum > target; s++) {
        st.steps++;
        st.updateCFL();
        double bound = 0;
        if ((rc = launch_dt_bound(c, &bound))) return rc;
        double dt = st.currentCFL * bound;
        if ((rc = fp_rk3_step(c, dt)) || (rc = launch_norms(c, c->d_R, norms.data()))) return rc;
        st.setResiduum(norms);
        st.t += dt;
        st.dt = dt;
        if ((rc = fp_copy_w2wo(c))) return rc;
        const bool stop = step_output(c, st, ms_since(t_start), &rc);
        if (rc) return rc;
        if (stop) break;
    }
    if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "sync"))) return rc;
    if ((rc = save_data(c, st, ms_since(t_start)))) return rc;
    if (out) {
        out[0] = st.t;
        out[1] = st.residuum;
        out[2] = st.currentCFL;
        out[3] = st.dt;
        out[4] = st.steps;
    }
    return FP_OK;
}

// LocalImplicitSolver.solve (LocalImplicitSolver.java:107-285); solver files when fp_solver_output names a directory
int fp_solve_implicit(fp_ctx* c, const fp_implicit_params* pin, double* out) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if (!pin) return set_err(c, FP_ERR_ARG, "null parameters");
    fp_implicit_params pcopy = *pin;
    if (pcopy.preconditioner == FP_PREC_ILU0) pcopy.preconditioner = FP_PREC_BLOCKILU0;
    const fp_implicit_params* p = &pcopy;
    State st;
    if (p->fixed_dt > 0) {
        st.fixed = true;
        st.dt0 = st.dt = p->fixed_dt;
    } else {
        st.cfl = p->cfl > 0 ? p->cfl : 1;
        st.vary = p->vary_cfl != 0 || p->cfl <= 0;
        st.maxCFL = p->max_cfl > 0 ? p->max_cfl : 1e4;
    }
    double dto = -1;
    bool converges = true;
    long newton = 0, linear = 0;
    std::vector<double> norms(c->hm.model.n_eqs);
    const int lag = p->jac_lag > 1 ? p->jac_lag : 1;
    int since_assembly = 1 << 30;  // Newton iterations since the last finite-difference assembly
    double blocks_a1 = 0;          // a1 the stored diagonal blocks were built (or shifted) with
    int total = st.steps + p->steps;
    const auto t_start = std::chrono::steady_clock::now();
    for (++st.steps; st.steps <= total && st.residuum > p->target_residuum; ++st.steps) {
        if (converges) st.updateCFL();
        if (st.hopeless()) break;
        double bound = 0;
        if ((rc = launch_dt_bound(c, &bound))) return rc;
        double dt;
        if (st.fixed) {
            st.currentCFL = st.dt / bound;
            dt = st.dt;
        } else {
            dt = st.currentCFL * bound;
            st.dt = dt;
        }
        if ((rc = launch_limiter(c))) return rc;
        double rhs0 = 0;
        bool restart = false;
        for (int s = 0; s < p->newton_iters; s++) {
            if (s > 0) {
                double nrm = 0;
                if ((rc = fp_assemble_residuum(c, p->bdf_order, dt, dto, &nrm))) return rc;
                double rel = rhs0 > 0 ? nrm / rhs0 : 0;
                if (rel < p->newton_tol) break;
            }
            const bool have_ops = p->jacobian == FP_JAC_MATRIXFREE
                                      ? c->prec_ready == p->precision && c->prec_kind == p->preconditioner
                                      : c->blocks_ready;
            if (p->jacobian == FP_JAC_MATRIXFREE && p->preconditioner == FP_PREC_NONE) {
                double nrm = 0;
                if ((rc = fp_assemble_residuum(c, p->bdf_order, dt, dto, &nrm))) return rc;
                if (s == 0) rhs0 = nrm;
            } else if (since_assembly >= lag - 1 || !have_ops) {
                // matrix-free: exact blocks straight into the preconditioner (no operator
                // blocks); assembled: the operator's blocks (finite differences or exact)
                rc = p->jacobian == FP_JAC_MATRIXFREE
                         ? fp_assemble_preconditioner(c, p->bdf_order, dt, dto, p->preconditioner, p->precision)
                     : p->jacobian == FP_JAC_ASSEMBLED_EXACT ? fp_assemble_exact(c, p->bdf_order, dt, dto)
                                                             : fp_assemble(c, p->bdf_order, dt, dto);
                if (rc == FP_ERR_SINGULAR) {
                    // the matrix-free path factorises at assembly: a singular block there is the
                    // failed linear solve of LinearSolver.solve (copyWo2W, reduceCFL, retry)
                    converges = false;
                    since_assembly = 1 << 30;
                    if ((rc = fp_copy_wo2w(c))) return rc;
                    st.reduceCFL();
                    --st.steps;
                    restart = true;
                    break;
                }
                if (rc) return rc;
                if (s == 0) rhs0 = c->last_rhs_norm;
                since_assembly = 0;
                blocks_a1 = c->a_coef[0];
            } else {
                // lagged Jacobian: fresh RHS; the assembled operator is moved to the current
                // a1, the preconditioner of the last assembly is kept
                double nrm = 0;
                if ((rc = fp_assemble_residuum(c, p->bdf_order, dt, dto, &nrm))) return rc;
                if (s == 0) rhs0 = nrm;
                if (p->jacobian != FP_JAC_MATRIXFREE && (rc = mass_shift(c, c->a_coef[0] - blocks_a1))) return rc;
                blocks_a1 = c->a_coef[0];
                since_assembly++;
            }
            if (s == 0) {
                if ((rc = launch_norms(c, c->d_R, norms.data()))) return rc;
                st.setResiduum(norms);
            }
            int it = 0;
            double rel = 0;
            int lrc = fp_linear_solve(c, p->jacobian, p->preconditioner, p->precision, p->restart, p->max_restarts,
                                      p->linear_tol, nullptr, &it, &rel);
            linear += it;
            newton++;
            bool ok = lrc == FP_OK;
            if (lrc != FP_OK && lrc != FP_ERR_NOT_CONVERGED && lrc != FP_ERR_SINGULAR) return lrc;
            converges = ok;
            if (!converges) {
                since_assembly = 1 << 30;  // the retry starts from fresh blocks
                if ((rc = fp_copy_wo2w(c))) return rc;
                st.reduceCFL();
                --st.steps;
                restart = true;
                break;
            }
            if ((rc = fp_update_w(c))) return rc;
            if (c->hm.num.positivity_limiter && (rc = launch_positivity(c, c->d_W, nullptr))) return rc;
        }
        if (restart) continue;
        if (!std::isfinite(st.residuum)) break;
        st.t += dt;
        dto = dt;
        if ((rc = fp_copy_w2wo(c))) return rc;
        const bool stop = step_output(c, st, ms_since(t_start), &rc);
        if (rc) return rc;
        if (stop) {
            ++st.steps;
            break;
        }
    }
    --st.steps;
    if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "sync"))) return rc;
    if ((rc = save_data(c, st, ms_since(t_start)))) return rc;
    if (out) {
        out[0] = st.t;
        out[1] = st.residuum;
        out[2] = st.currentCFL;
        out[3] = st.dt;
        out[4] = st.steps;
        out[5] = (double)newton;
        out[6] = (double)linear;
    }
    return FP_OK;
}

// Independent cases solved concurrently: worker threads take the contexts in order and run
// the implicit solver loop on each (every context has its own stream, so the kernels of
// different cases overlap on the device).  The block ILU(0) sweep is excluded: its
// persistent launch relies on co-residency, which concurrent kernels of other cases do not
// give.
int fp_batch_solve_implicit(fp_ctx** ctxs, int n, const fp_implicit_params* p, int threads, double* out, int* status) {
    if (!ctxs || n <= 0 || !p) return FP_ERR_ARG;
    for (int i = 0; i < n; i++)
        if (!ctxs[i]) return FP_ERR_ARG;
    if (p->preconditioner == FP_PREC_BLOCKILU0 || p->preconditioner == FP_PREC_ILU0)
        return set_err(ctxs[0], FP_ERR_UNSUPPORTED, "batched solves take block Jacobi or no preconditioner");
    threads = std::max(1, std::min(threads, n));
    std::atomic<int> next(0);
    std::vector<int> rcs(n, FP_OK);
    auto work = [&]() {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n) break;
            cudaSetDevice(ctxs[i]->device);
            rcs[i] = fp_solve_implicit(ctxs[i], p, out ? out + 7 * (size_t)i : nullptr);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++) pool.emplace_back(work);
    for (auto& th : pool) th.join();
    int rc = FP_OK;
    for (int i = 0; i < n; i++) {
        if (status) status[i] = rcs[i];
        if (rc == FP_OK && rcs[i] != FP_OK) rc = rcs[i];
    }
    return rc;
}

int fp_profile(fp_ctx* c, int enable, double* ms, long long* counts) {
    if (!c) return FP_ERR_ARG;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->prof_open) prof_end(c);
    prof_resolve(c);
    for (int i = 0; i < 8; i++) {
        if (ms) ms[i] = c->prof_ms[i];
        if (counts) counts[i] = c->prof_n[i];
    }
    if (enable >= 0) {
        for (int i = 0; i < 8; i++) {
            c->prof_ms[i] = 0;
            c->prof_n[i] = 0;
        }
        c->prof_on = enable > 0;
    }
    return FP_OK;
}

int fp_mesh_move(fp_ctx* c, const double* vertices, const double* velocity) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if (!vertices) return set_err(c, FP_ERR_ARG, "null vertices");
    HostMesh& h = c->hm;
    fp_mesh_desc d{};
    d.dim = h.dim;
    d.n_vertices = h.nVert;
    d.n_elements = h.nElem;
    d.vertices = vertices;
    d.elements = c->h_elements.data();
    d.neighbors = c->h_neighbors.data();
    d.wall_distance = c->h_wd.empty() ? nullptr : c->h_wd.data();
    d.mesh_velocity = velocity;
    HostMesh moved;
    if ((rc = build_host_mesh(d, h.model, h.num, moved, c->err))) return rc;
    if (moved.nFaces != h.nFaces || moved.geo.size() != h.geo.size())
        return set_err(c, FP_ERR_ARG, "moved mesh does not match the uploaded one");
    const Launchers* t = find_launchers(h.model, h.num.order);
    if (!t) return set_err(c, FP_ERR_UNSUPPORTED, "model / order not built");
    const size_t nb2 = (size_t)h.tab.nb * h.tab.nb;
    if (!c->d_mass) {
        // the time levels start from the mass matrix of the mesh as it was (Element init: Mo = Mo2 = M)
        if ((rc = dalloc(c, &c->d_mass, 3 * nb2 * h.ld))) return rc;
        for (int lev = 0; lev < 3; lev++) t->mass_geo(dev_mesh(c), c->stream, lev, c->d_mass);
        if ((rc = cuda_check(c, cudaGetLastError(), "mass levels"))) return rc;
    }
    h.geo = std::move(moved.geo);
    h.area = std::move(moved.area);
    h.elemSize = std::move(moved.elemSize);
    h.xs = std::move(moved.xs);
    if ((rc = upload(c, c->d_geo, h.geo.data(), h.geo.size()))) return rc;
    if (velocity) {
        h.vu = std::move(moved.vu);
        if (!c->d_vu && (rc = dalloc(c, &c->d_vu, h.vu.size(), false))) return rc;
        if ((rc = upload(c, c->d_vu, h.vu.data(), h.vu.size()))) return rc;
    } else if (c->d_vu) {
        std::fill(h.vu.begin(), h.vu.end(), 0.0);
        if ((rc = cuda_check(c, cudaMemsetAsync(c->d_vu, 0, h.vu.size() * sizeof(double), c->stream), "memset"))) return rc;
    }
    // the current level's mass matrix on the moved geometry (Deformation.recalculateMesh ->
    // DGpure.recalculateMassMatrix); the discrete-GCL one replaces it at assembly when gcl is on
    t->mass_geo(dev_mesh(c), c->stream, 0, c->d_mass);
    if ((rc = cuda_check(c, cudaGetLastError(), "mass"))) return rc;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "sync");
}

int fp_mass_next_level(fp_ctx* c) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if (!c->d_mass) return FP_OK;
    const size_t lv = (size_t)c->hm.tab.nb * c->hm.tab.nb * c->hm.ld;
    if ((rc = cuda_check(c, cudaMemcpyAsync(c->d_mass + 2 * lv, c->d_mass + lv, lv * sizeof(double), cudaMemcpyDeviceToDevice,
                                            c->stream), "copy")))
        return rc;
    return cuda_check(c, cudaMemcpyAsync(c->d_mass + lv, c->d_mass, lv * sizeof(double), cudaMemcpyDeviceToDevice, c->stream),
                      "copy");
}

int fp_solver_output(fp_ctx* c, const char* dir, int save_rate, int append) {
    if (!c) return FP_ERR_ARG;
    c->io_dir = dir ? dir : "";
    c->io_save_rate = save_rate;
    if (!c->io_dir.empty() && !append && io_reset_residuum(c->io_dir))
        return set_err(c, FP_ERR_ARG, "cannot create residuum.txt in " + c->io_dir);
    return FP_OK;
}

int fp_set_ilu_sweep(fp_ctx* c, int variant) {
    if (!c || variant < 0 || variant > 6) return FP_ERR_ARG;
    c->sweep_variant = variant;
    return FP_OK;
}

int fp_set_wait_limit(fp_ctx* c, int polls) {
    if (!c || polls < 0) return FP_ERR_ARG;
    c->ilu_max_polls = polls;
    return FP_OK;
}

int fp_forces(fp_ctx* c, int bc, double* force) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if (!force) return set_err(c, FP_ERR_ARG, "null array");
    if (bc >= 0) return set_err(c, FP_ERR_ARG, "boundary codes are negative");
    double out[4];
    if ((rc = launch_surface(c, 0, bc, out, nullptr))) return rc;
    for (int d = 0; d < c->hm.dim; d++) force[d] = out[d];
    return FP_OK;
}

int fp_functional(fp_ctx* c, int kind, double* value, double* dI_dW) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if (!value) return set_err(c, FP_ERR_ARG, "null value");
    if (kind != FP_FUNCTIONAL_LIFT && kind != FP_FUNCTIONAL_DRAG) return set_err(c, FP_ERR_ARG, "unknown functional");
    if (c->hm.dim != 2 || c->hm.model.model == FP_MODEL_SCALAR_TEST || c->hm.model.model == FP_MODEL_ADIABATIC_EULERS)
        return set_err(c, FP_ERR_UNSUPPORTED, "the lift / drag functionals are two-dimensional flow functionals");
    if (dI_dW && (rc = ensure_krylov(c, 1, -1))) return rc;
    double out[4];
    if ((rc = launch_surface(c, kind, BC_WALL, out, dI_dW ? c->d_tmp : nullptr))) return rc;
    *value = out[0];
    if (dI_dW) return soa_to_host(c, c->d_tmp, dI_dW);
    return FP_OK;
}

int fp_adjoint_solve(fp_ctx* c, const double* rhs, int preconditioner, int precision, int restart, int max_restarts,
                     double tol, double* psi, int* iterations, double* rel_residual) {
    return fp_block_solve(c, 1, rhs, preconditioner, precision, restart, max_restarts, tol, psi, iterations, rel_residual);
}

int fp_block_solve(fp_ctx* c, int transpose, const double* rhs, int preconditioner, int precision, int restart,
                   int max_restarts, double tol, double* psi, int* iterations, double* rel_residual) {
    int rc = need_mesh(c);
    if (rc) return rc;
    if (!rhs) return set_err(c, FP_ERR_ARG, "null rhs");
    if (!c->blocks_ready) return set_err(c, FP_ERR_STATE, "call fp_assemble or fp_assemble_exact first");
    if (preconditioner == FP_PREC_ILU0) preconditioner = FP_PREC_BLOCKILU0;
    if (transpose && preconditioner == FP_PREC_BLOCKILU0)
        return set_err(c, FP_ERR_UNSUPPORTED, "block ILU(0) is not available for transposed solves");
    if (restart < 1 || max_restarts < 1 || restart > 200) return set_err(c, FP_ERR_ARG, "bad GMRES sizes");
    if ((rc = ensure_krylov(c, restart, precision))) return rc;
    if ((c->prec_ready != precision || c->prec_kind != preconditioner) && (rc = prec_factor(c, preconditioner, precision)))
        return rc;
    if ((rc = host_to_soa(c, rhs, c->d_b))) return rc;
    if ((rc = cuda_check(c, cudaMemsetAsync(c->d_x, 0, c->nvec * sizeof(double), c->stream), "memset"))) return rc;
    int it = 0;
    double rel = 0;
    c->kry_transposed = transpose != 0;
    int grc = gmres(c, FP_JAC_ASSEMBLED, preconditioner, restart, max_restarts, tol, &it, &rel);
    c->kry_transposed = false;
    if (preconditioner == FP_PREC_BLOCKILU0 && (grc == FP_OK || grc == FP_ERR_NOT_CONVERGED) && (rc = ilu_check(c)))
        return rc;
    if (iterations) *iterations = it;
    if (rel_residual) *rel_residual = rel;
    if (grc && grc != FP_ERR_NOT_CONVERGED) return grc;
    if (psi && (rc = soa_to_host(c, c->d_x, psi))) return rc;
    return grc;
}

}  // extern "C"
