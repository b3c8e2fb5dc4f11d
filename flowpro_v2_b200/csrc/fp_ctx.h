// Context of one resident mesh: host set-up data, device buffers, stream.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "fp_kernels.cuh"
#include "fp_mesh.h"

struct fp_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    std::string err;
    bool has_mesh = false;
    fp::HostMesh hm;
    int nc = 0;            // unknowns per element (nEqs * nBasis)
    size_t nvec = 0;       // nc * ld: length of a state-shaped device vector
    // mesh and tables
    double* d_geo = nullptr;
    double* d_tab = nullptr;
    double* d_vwd = nullptr;
    double* d_vu = nullptr;
    int* d_tt = nullptr;
    int* d_fcode = nullptr;
    int* d_order = nullptr;   // DOF order (RCM)
    double* d_eps = nullptr;
    // moving mesh (fp_mesh_move): element mass matrices of the time levels [3][nb*nb][ld], and
    // the mesh arrays the geometry is rebuilt from
    double* d_mass = nullptr;
    // a batch of independent cases merged into this context's mesh (fp_batch_upload)
    int n_cases = 0;
    std::vector<int> case_e0;         // [n_cases + 1] element ranges
    int* d_case_of = nullptr;         // [ld] case of each element
    double* d_case_pout = nullptr;    // [n_cases] outlet pressures
    double* d_case_a = nullptr;       // [3][n_cases] BDF coefficients of each case's step
    double* d_case_W0 = nullptr;      // the cases' free-stream states (field-major, all cases)
    bool batch_ready = false;         // chunk table and reduction buffers of the batched solver
    int batch_kmax = 0, batch_nch = 0;
    int *d_bch0 = nullptr, *d_bch1 = nullptr, *d_bcptr = nullptr, *d_bmask = nullptr;
    double *d_bpart = nullptr, *d_bcase = nullptr;
    // [n_cases] live flags of the batched GMRES and per-case vector counts; while batch_mask is
    // set, the matrix-free operator, the staged block ILU(0) sweeps and the Krylov kernels skip the
    // elements of cases whose flag is 0
    int *d_blive = nullptr, *d_bkc = nullptr;
    bool batch_mask = false;
    std::vector<int> h_elements, h_neighbors;
    std::vector<double> h_wd;
    double* d_cip = nullptr;
    // face list of the face-based residual
    int* d_fl = nullptr;
    int* d_fk = nullptr;
    int* d_fr = nullptr;
    int* d_fc = nullptr;
    int* d_qmap = nullptr;
    int* d_efc = nullptr;
    double* d_G = nullptr;     // [2][nqf][n_eqs][ldf] face contributions
    // state and residual
    double* d_W = nullptr;
    double* d_Wo = nullptr;
    double* d_Wo2 = nullptr;
    double* d_R = nullptr;     // last spatial residual R(W)
    double* d_Wst[3] = {nullptr, nullptr, nullptr};  // RK3 stage states W1, W2, Wn
    double* d_io = nullptr;    // staging for host <-> device layout conversion
    // fp_residual with host input and output: the copies overlap the passes chunk by chunk
    // (plan, staging of the result, copy streams and events; made on first use)
    double* d_io2 = nullptr;
    std::vector<int> pipe_e, pipe_f, pipe_need;
    cudaStream_t s_h2d = nullptr, s_d2h = nullptr, s_elem = nullptr;
    std::vector<cudaEvent_t> pipe_ev;
    cudaGraphExec_t pipe_exec = nullptr;  // the sequence for the host buffers pipe_w / pipe_r
    const double* pipe_w = nullptr;
    double* pipe_r = nullptr;
    bool pipe_graph_ok = true;
    // implicit
    double* d_Adiag = nullptr; // [nc*nc][ld]  untransposed: A[r][c] at (r*nc + c)*ld + e
    double* d_Aneigh = nullptr;// [nf][nc*nc][ld]
    double* d_rhs = nullptr;   // [nc][ld]
    double* d_K0 = nullptr;    // FD base residual [nc][ld]
    double* d_KR0 = nullptr;   // FD base face contributions [nf][nc][ld]
    double* d_P64 = nullptr;   // inverse diagonal blocks, FP64 [nc*nc][ld]
    float* d_P32 = nullptr;    // inverse diagonal blocks, FP32
    int prec_ready = -1;       // precision of the factorised preconditioner, -1 none
    bool blocks_ready = false; // d_Adiag / d_Aneigh hold the blocks of the last assembly
    bool rhs_ready = false;    // d_rhs holds the right-hand side of the last assembly
    int prec_kind = -1;        // preconditioner kind of the factorisation
    // block ILU(0): factor rows in DOF (RCM) order, element-major, blocks column-major:
    // F[e][s][c][r], s = 0 inverse of the factored diagonal block, s = 1 + k the block
    // coupling e with its neighbour over face k (L for lower-ranked, U for higher-ranked)
    double* d_iluF64 = nullptr;
    float* d_iluF32 = nullptr;
    int* d_rank = nullptr;        // DOF position of each element
    int* d_lvlF = nullptr;        // elements grouped by forward level (lower neighbours first)
    int* d_opPtr = nullptr;       // factorisation program per element
    int4* d_ops = nullptr;
    std::vector<int> lvlF_ptr, lvlB_ptr;
    bool ilu_built = false;
    int ilu_prec = -1;
    int4* d_nbLow = nullptr;      // per element: neighbour over face f if it is lower-ranked, else -1
    int* d_swEl = nullptr;        // sweep program: element at position v (forward levels, then backward levels)
    int4* d_swNb = nullptr;       // sweep program: neighbours multiplied at position v (lower, then upper; -1 none)
    unsigned* d_iluFlags = nullptr;  // abort word, sweep status word, then [nElem] factorisation row flags
    unsigned* d_ilu_sing = nullptr;  // [nElem] 1 where the last factorisation met a singular diagonal block
    unsigned ilu_epoch = 0;          // epoch of the last application
    unsigned ilu_fepoch = 0;         // epoch of the last factorisation
    int ilu_max_polls = 1 << 19;     // poll limit of every dependency wait of the ILU kernels
    unsigned long long* d_ilu_pub = nullptr;  // [2][nElem][nc][2] published sweep values (forward, backward)
    int sweep_grid = 0;           // thread blocks of the persistent sweep kernel
    // bulk-copy sweep kernel per factor precision [FP64, FP32]: slots, grid (-1 unknown, 0 not
    // applicable), dynamic shared memory
    int sweep_bulk_S[2] = {0, 0};
    int sweep_bulk_NG[2] = {0, 0};   // positions in flight per block (0: not tuned yet)
    int sweep_bulk_grid[2] = {-1, -1};
    size_t sweep_bulk_smem[2] = {0, 0};
    int sweep_variant = 0;           // 0 bulk-copy staged (autotuned groups), 1 register, 2-6 bulk with 1-16 groups
    // Krylov
    int kry_m = 0;
    bool kry_transposed = false;  // GMRES on A^T (adjoint solves)
    double* d_V = nullptr;     // (m+1) vectors
    double* d_w = nullptr;
    double* d_aux = nullptr;
    double* d_r = nullptr;
    double* d_x = nullptr;
    double* d_b = nullptr;
    double* d_tmp = nullptr;
    double* d_part = nullptr;  // reduction partials
    double* d_scal = nullptr;  // device scalars
    double* h_scal = nullptr;  // pinned host mirror
    unsigned* d_status = nullptr;
    // bookkeeping
    double last_dt = 0;
    double last_rhs_norm = 0;
    int bdf_order = 1;
    double a_coef[3] = {0, 0, 0};
    std::vector<double*> allocs;
    // solver output files (fp_solver_output): directory ("" = none) and save rate in steps
    std::string io_dir;
    int io_save_rate = 0;
    // device time per solver phase (fp_profile): CUDA events around the launches of each
    // phase on the context's stream, resolved after the stream synchronisations the solver
    // makes anyway
    bool prof_on = false;
    double prof_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    long long prof_n[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    std::vector<cudaEvent_t> prof_ev;
    std::vector<int> prof_ph;
    int prof_used = 0;
    bool prof_open = false;
};

namespace fp {

int set_err(fp_ctx* c, int code, const std::string& msg);
int cuda_check(fp_ctx* c, cudaError_t e, const char* where);
DevMesh dev_mesh(const fp_ctx* c);

// device allocation owned by the context (released with it), optionally zeroed
template <class T>
inline int dalloc(fp_ctx* c, T** p, size_t n, bool zero = true) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) return cuda_check(c, e, "cudaMalloc");
    c->allocs.push_back((double*)q);
    *p = (T*)q;
    if (zero) {
        e = cudaMemsetAsync(q, 0, std::max<size_t>(n, 1) * sizeof(T), c->stream);
        if (e != cudaSuccess) return cuda_check(c, e, "cudaMemset");
    }
    return FP_OK;
}

template <class T>
inline int upload(fp_ctx* c, T* d, const T* h, size_t n) {
    return cuda_check(c, cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, c->stream), "upload");
}

int host_to_soa(fp_ctx* c, const double* h, double* d);  // element-major host -> field-major device
int soa_to_host(fp_ctx* c, const double* d, double* h);  // and back (synchronises)
int need_mesh(fp_ctx* c);
int ensure_rhs(fp_ctx* c);
int ensure_krylov(fp_ctx* c, int m, int precision);
void free_all(fp_ctx* c);

// solver output files (fp_io.cpp)
struct IoState {
    double t = 0, residuum = 0, cfl = 0, dt = 0;
    long long steps = 0, cpu_ms = 0;
    std::vector<double> normalisation;  // empty until the normalisation steps are done
    int order = 1;
};
std::string java_double(double x);
int io_reset_residuum(const std::string& dir);
int io_append_residuum(const std::string& dir, double residuum, double t, double cpu, const std::vector<double>& eq);
int io_save_rows(const std::string& dir, const char* name, const double* a, size_t rows, size_t cols);
int io_save_state(const std::string& dir, const IoState& s);
bool io_stop_requested(const std::string& dir);

// solver phases timed by fp_profile
enum { PH_RHS = 0, PH_BLOCKS = 1, PH_FACTOR = 2, PH_OPERATOR = 3, PH_PREC = 4, PH_KRYLOV = 5, PH_OTHER = 6 };
void prof_begin(fp_ctx* c, int phase);  // no-op unless profiling; phases do not nest
void prof_end(fp_ctx* c);
void prof_resolve(fp_ctx* c);           // after a stream synchronisation: add the finished intervals

// kernels (fp_residual.cu)
int launch_residual(fp_ctx* c, const double* W, double* R);
int launch_residual_timed(fp_ctx* c, const double* W, double* R, cudaEvent_t ev[3]);  // events around both passes
int launch_residual_pipelined(fp_ctx* c, const double* w_host, double* r_host);       // host buffers, chunked copies
void pipe_release(fp_ctx* c);                                                        // drop the captured sequence
int launch_rk_stage(fp_ctx* c, const double* Wcur, const double* Wo, const double* Wb, double alpha, double beta, double dt,
                    double* Wout, double* Rsave);
int launch_limiter(fp_ctx* c);
int launch_positivity(fp_ctx* c, double* W, int* n_limited);
int launch_norms(fp_ctx* c, const double* R, double* norms_host);
int launch_dt_bound(fp_ctx* c, double* out_host);
int launch_fd_jacobian(fp_ctx* c, double a1, double a2, double a3, double* rhs_norm_host);
int launch_rhs(fp_ctx* c, double a1, double a2, double a3, double* rhs_norm_host);
int launch_jvp(fp_ctx* c, const double* V, double* JV, double* R);
int launch_jac_exact(fp_ctx* c, double a1, double a2, double a3, double* rhs_norm_host);  // exact tangent blocks
// RHS and exact blocks written straight into block ILU(0) factor storage F (float when fp32)
int launch_jac_exact_factor(fp_ctx* c, double a1, double a2, double a3, double* rhs_norm_host, void* F, int fp32);
int launch_surface(fp_ctx* c, int kind, int bc, double* out4_host, double* dIdW_dev);     // forces / functionals
int launch_vjp(fp_ctx* c, const double* lam, double* g);  // g = (dR/dW)^T lam, no stored Jacobian

// linear algebra (fp_linalg.cu)
int spmv(fp_ctx* c, const double* x, double* y);                 // y = A x (assembled blocks)
int spmv_t(fp_ctx* c, const double* x, double* y);               // y = A^T x
int matfree_apply(fp_ctx* c, const double* x, double* y);        // y = a1 M x - (dR/dW) x
int mass_shift(fp_ctx* c, double delta);                         // A_diag += delta * M
int prec_factor(fp_ctx* c, int kind, int precision);
int prec_apply(fp_ctx* c, int kind, const double* x, double* y);
int ilu_factor(fp_ctx* c, int precision);                        // block ILU(0) of the assembled blocks (fp_ilu.cu)
int ilu_prepare_direct(fp_ctx* c, int precision, void** F);      // factor storage for blocks written in place
int ilu_factor_direct(fp_ctx* c, int precision);                 // factorise the blocks written in place
int ilu_apply(fp_ctx* c, const double* x, double* y);
int ilu_check(fp_ctx* c);                                        // FP_ERR_TIMEOUT if a sweep wait gave up
void ilu_release(fp_ctx* c);
int gmres(fp_ctx* c, int jacobian, int kind, int restart, int max_restarts, double tol, int* iters, double* rel);
int dot(fp_ctx* c, const double* a, const double* b, double* dev_out);
int vec_copy(fp_ctx* c, double* y, const double* x);
int vec_axpby(fp_ctx* c, double* y, double a, const double* x, double b);  // y = a x + b y
int vec_add_scaled(fp_ctx* c, double* y, const double* x, double s);       // y += s x

}  // namespace fp
