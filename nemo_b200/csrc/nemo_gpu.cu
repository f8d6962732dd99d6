// nemo_gpu.cu -- host side of the C-ABI in include/nemo_gpu.h.
//
// Owns the device memory, the CUDA stream and the captured step graphs; builds the
// Gauss-Lobatto operators (the same construction as the reference's kernel_share_mod init,
// source/kernel/dgsem/weakform/2d/kernel_share_mod.f90:56-151, on Gauss-Lobatto nodes);
// converts the reference's side connectivity into per-element face-neighbour tables.
// Compiled with -ffp-contract=off so that the operator matrices are bit-identical to every
// other IEEE-exact construction of them.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.h"

using namespace nemo;

namespace {

// ---- operator construction ------------------------------------------------------------------

// Gauss-Lobatto nodes/weights by Newton on q = L_{N+1} - L_{N-1}, as LegendreGaussLobattoNodesAndWeights
// (source/utils/interpol_mod.f90:513-582) with its qAndLEvaluation helper.
void gl_qeval(int N, double x, double& q, double& dq, double& LN) {
    double a2 = 1.0, a1 = x, d2 = 0.0, d1 = 1.0, dd = 0.0;
    LN = 0.0;
    for (int k = 2; k <= N; ++k) {
        LN = (2.0 * k - 1.0) / k * x * a1 - (k - 1.0) / k * a2;
        dd = d2 + (2.0 * k - 1.0) * a1;
        a2 = a1; a1 = LN; d2 = d1; d1 = dd;
    }
    const int k = N + 1;
    const double Lk = (2.0 * k - 1.0) / k * x * LN - (k - 1.0) / k * a2;
    const double dLk = d2 + (2.0 * k - 1.0) * a1;
    q = Lk - a2;
    dq = dLk - d2;
}

void gl_nodes(int N, double* x, double* w) {
    const double pi = 4.0 * std::atan(1.0);
    x[0] = -1.0; w[0] = 2.0 / (N * (N + 1.0)); x[N] = 1.0; w[N] = w[0];
    double q, dq, LN;
    for (int j = 1; j <= (N + 1) / 2 - 1; ++j) {
        x[j] = -std::cos(((j + 0.25) * pi) / N - (3.0 / (8.0 * N * pi)) * (1.0 / (j + 0.25)));
        for (int it = 0; it <= 4; ++it) {
            gl_qeval(N, x[j], q, dq, LN);
            const double step = -q / dq;
            x[j] = x[j] + step;
            if (std::fabs(step) <= 4.0e-16 * std::fabs(x[j])) break;
        }
        gl_qeval(N, x[j], q, dq, LN);
        x[N - j] = -x[j];
        w[j] = 2.0 / (N * (N + 1.0) * (LN * LN));
        w[N - j] = w[j];
    }
    if (N % 2 == 0) {
        gl_qeval(N, 0.0, q, dq, LN);
        x[N / 2] = 0.0;
        w[N / 2] = 2.0 / (N * (N + 1.0) * (LN * LN));
    }
}

// Barycentric differentiation matrix (source/utils/interpol_mod.f90:38-81), D[i*n+m] = l_m'(x_i).
void bary_diff(int n, const double* x, double* D) {
    double wb[NN];
    for (int i = 0; i < n; ++i) wb[i] = 1.0;
    for (int i = 1; i < n; ++i)
        for (int j = 0; j < i; ++j) {
            wb[j] = wb[j] * (x[j] - x[i]);
            wb[i] = wb[i] * (x[i] - x[j]);
        }
    for (int i = 0; i < n; ++i) wb[i] = 1.0 / wb[i];
    for (int i = 0; i < n * n; ++i) D[i] = 0.0;
    for (int l = 0; l < n; ++l)
        for (int g = 0; g < n; ++g)
            if (l != g) {
                D[g * n + l] = wb[l] / (wb[g] * (x[g] - x[l]));
                D[g * n + g] = D[g * n + g] - D[g * n + l];
            }
}

// Normalised Legendre polynomial (source/utils/interpol_mod.f90:274-311).
double leg_norm(int N, double x) {
    double L;
    if (N == 0) L = 1.0;
    else if (N == 1) L = x;
    else {
        double m2 = 1.0, m1 = x;
        L = 0.0;
        for (int i = 2; i <= N; ++i) {
            L = ((2 * i - 1) * x * m1 - (i - 1) * m2) / i;
            m2 = m1; m1 = L;
        }
    }
    return L * std::sqrt(N + 0.5);
}

// Inverse by Doolittle LU without pivoting (source/utils/linalg_mod.f90:123-201).
void lu_inverse(int n, const double* A, double* C) {
    double a[NN * NN], L[NN * NN], U[NN * NN], b[NN], d[NN], xx[NN];
    std::memcpy(a, A, sizeof(double) * n * n);
    std::fill(L, L + n * n, 0.0);
    std::fill(U, U + n * n, 0.0);
    for (int k = 0; k < n - 1; ++k)
        for (int i = k + 1; i < n; ++i) {
            const double coeff = a[i * n + k] / a[k * n + k];
            L[i * n + k] = coeff;
            for (int j = k + 1; j < n; ++j) a[i * n + j] = a[i * n + j] - coeff * a[k * n + j];
        }
    for (int i = 0; i < n; ++i) L[i * n + i] = 1.0;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i <= j; ++i) U[i * n + j] = a[i * n + j];
    for (int col = 0; col < n; ++col) {
        for (int i = 0; i < n; ++i) b[i] = 0.0;
        b[col] = 1.0;
        d[0] = b[0];
        for (int i = 1; i < n; ++i) {
            d[i] = b[i];
            for (int j = 0; j < i; ++j) d[i] = d[i] - L[i * n + j] * d[j];
        }
        xx[n - 1] = d[n - 1] / U[(n - 1) * n + n - 1];
        for (int i = n - 2; i >= 0; --i) {
            xx[i] = d[i];
            for (int j = n - 1; j > i; --j) xx[i] = xx[i] - U[i * n + j] * xx[j];
            xx[i] = xx[i] / U[i * n + i];
        }
        for (int i = 0; i < n; ++i) C[i * n + col] = xx[i];
    }
}

struct HostOps {
    double x[NN], w[NN], D[NN * NN], S[NN * NN], V[NN * NN], Vinv[NN * NN];
    double pro[2][NN * NN], prj[2][NN * NN];
};

// Lagrange basis polynomial j of the nodes x at xi
double lagrange_at(int n, const double* x, int j, double xi) {
    double l = 1.0;
    for (int m = 0; m < n; ++m)
        if (m != j) l = l * ((xi - x[m]) / (x[j] - x[m]));
    return l;
}

void build_host_ops(HostOps& h) {
    gl_nodes(NN - 1, h.x, h.w);
    bary_diff(NN, h.x, h.D);
    // split-form matrix S = 2D - W^-1 B (Gassner-Winters-Kopriva 2016); zero diagonal on LGL nodes
    for (int i = 0; i < NN; ++i)
        for (int m = 0; m < NN; ++m) h.S[i * NN + m] = i == m ? 0.0 : 2.0 * h.D[i * NN + m];
    for (int i = 0; i < NN; ++i)
        for (int j = 0; j < NN; ++j) h.V[i * NN + j] = leg_norm(j, h.x[i]);
    lu_inverse(NN, h.V, h.Vinv);
    // 2:1 mortar matrices with Q = 2 sub-faces (kernel_operators_interpolationMatrix and
    // _projectionMatrix, source/kernel/dgsem/weakform/2d/kernel_operators_mod.f90:1010-1100):
    // pro[s][i][j] = l_j(mu_s + x_i/2), prj[s][a][i] = l_a(mu_s + x_i/2) w_i / w_a / 2, mu = -+1/2
    for (int s = 0; s < 2; ++s) {
        const double mu = s ? 0.5 : -0.5;
        for (int i = 0; i < NN; ++i)
            for (int j = 0; j < NN; ++j) {
                h.pro[s][i * NN + j] = lagrange_at(NN, h.x, j, mu + h.x[i] / 2.0);
                h.prj[s][j * NN + i] = lagrange_at(NN, h.x, j, mu + h.x[i] / 2.0) * h.w[i] / h.w[j] / 2.0;
            }
    }
}

// ---- library state ----------------------------------------------------------------------------

struct Lib {
    bool inited = false;
    nemo_cfg cfg{};
    HostOps hops{};
    OpConsts ops{};
    cudaStream_t stream = nullptr;
    char err[512] = "";

    int64_t E = 0;
    int64_t E_own = 0;            // elements advanced by this process; [E_own, E) are ghost copies
    int64_t n_interior = 0;       // owned elements [0, n_interior) read no ghost data (0: no split)
    bool split_open = false;      // a stage's interior part is enqueued, its boundary part not yet
    unsigned long long nbad_mark = 0;  // repair-failure count before the open split stage (host copy)
    int V = 5;
    bool has_mesh = false, has_state = false;
    int ngroups = 1;

    double* u[2] = {nullptr, nullptr};
    double* reg = nullptr;
    double* stagebuf = nullptr;   // AoS staging for upload/download
    double* alpha[2] = {nullptr, nullptr};
    double* alpha_used = nullptr;
    int32_t* nbr = nullptr;
    int64_t nm = 0;               // 2:1 mortars
    int32_t* mortar = nullptr;    // [nm][6]
    double* mflux = nullptr;      // [5 nm][V][16]
    uint32_t* mflag = nullptr;    // [nm] persistent FP32 stage: epoch of each mortar's rows

    // stage schedule of the FP32 Euler form (nemo_gpu_autotune): 0 = one CTA per tile plus the
    // mortar kernel, 1 = persistent CTAs (tune_ctas of them) taking mortar and tile tasks
    int tune_mode = 0;
    int tune_ctas = 0;
    double* cdel = nullptr;
    double* delta = nullptr;
    int32_t* group = nullptr;
    Control* ctrl = nullptr;
    double* part = nullptr;       // totals partials [V][E]
    double* tot = nullptr;        // totals [10]
    int cur = 0;                  // u[cur] holds the state, alpha[cur] its raw indicator
    bool prepared = false;        // alpha[cur] and the CFL bound in ctrl are valid for u[cur]
    bool reg_valid = false;

    cudaGraphExec_t graph[2] = {nullptr, nullptr};

    // learned indicator: BF16-rounded weights + input bounds, as FP32 and FP64 arrays
    float* mlp32 = nullptr;
    double* mlp64 = nullptr;
    bool mlp_ready = false;
    float* feat_dev = nullptr;     // [E][12] features of nemo_gpu_features

    bool timing = false;
    double t_stage_ms = 0.0, t_total_ms = 0.0;
    int64_t n_stage = 0, n_total = 0;

    // checkpoint staging: an AoS copy of the state (and of t, steps) taken in stream order, copied
    // to the host on its own stream while the library stream computes on
    double* ckpt = nullptr;
    int64_t ckpt_bytes = 0;
    double* ckpt_meta = nullptr;       // device [2]: t of group 0, steps (bits)
    double* ckpt_meta_host = nullptr;  // pinned [2]
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ckpt_ready = nullptr, ckpt_done = nullptr;
    bool ckpt_pending = false;

    // asynchronous uploads (nemo_gpu_upload_state_async): two AoS staging slots filled on their
    // own stream, consumed in stream order by the library stream; per slot a pinned control block
    cudaStream_t in_stream = nullptr;
    double* in_stage[2] = {nullptr, nullptr};
    int64_t in_bytes = 0;
    cudaEvent_t in_done[2] = {nullptr, nullptr};   // host->device copy of the slot finished
    cudaEvent_t in_free[2] = {nullptr, nullptr};   // the library stream has consumed the slot
    bool in_used[2] = {false, false};
    int in_next = 0;
    Control* in_ctrl = nullptr;                    // pinned [2]

    // asynchronous downloads (nemo_gpu_download_state_async): two AoS staging slots filled in stream
    // order by the library stream, copied to the host on their own stream
    cudaStream_t out_stream = nullptr;
    double* out_stage[2] = {nullptr, nullptr};
    int64_t out_bytes = 0;
    cudaEvent_t out_ready[2] = {nullptr, nullptr};  // the slot holds the snapshot
    cudaEvent_t out_done[2] = {nullptr, nullptr};   // its device->host copy finished
    bool out_used[2] = {false, false};
    int out_next = 0;
};

Lib g;

int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g.err, sizeof g.err, fmt, ap);
    va_end(ap);
    return code;
}

#define CK(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) return fail(NEMO_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

void free_dev(void* p) {
    if (p) cudaFree(p);
}

void release_graphs() {
    for (auto& ge : g.graph)
        if (ge) {
            cudaGraphExecDestroy(ge);
            ge = nullptr;
        }
}

void release_checkpoint() {
    if (g.ckpt_pending) cudaEventSynchronize(g.ckpt_done);
    g.ckpt_pending = false;
    free_dev(g.ckpt);
    g.ckpt = nullptr;
    g.ckpt_bytes = 0;
}

void release_downloads() {
    for (int i = 0; i < 2; ++i) {
        if (g.out_used[i]) cudaEventSynchronize(g.out_done[i]);
        g.out_used[i] = false;
        free_dev(g.out_stage[i]);
        g.out_stage[i] = nullptr;
    }
    g.out_bytes = 0;
}

void release_uploads() {
    for (int i = 0; i < 2; ++i) {
        if (g.in_used[i]) cudaEventSynchronize(g.in_free[i]);
        g.in_used[i] = false;
        free_dev(g.in_stage[i]);
        g.in_stage[i] = nullptr;
    }
    g.in_bytes = 0;
}

void release_mesh() {
    release_checkpoint();
    release_uploads();
    release_downloads();
    release_graphs();
    free_dev(g.u[0]); free_dev(g.u[1]); free_dev(g.reg); free_dev(g.stagebuf);
    free_dev(g.alpha[0]); free_dev(g.alpha[1]); free_dev(g.alpha_used);
    free_dev(g.nbr); free_dev(g.cdel); free_dev(g.delta); free_dev(g.group);
    free_dev(g.mortar); free_dev(g.mflux); free_dev(g.mflag);
    g.mortar = nullptr; g.mflux = nullptr; g.mflag = nullptr; g.nm = 0;
    g.tune_mode = 0;
    g.tune_ctas = 0;
    free_dev(g.part);
    free_dev(g.feat_dev);
    g.feat_dev = nullptr;
    g.u[0] = g.u[1] = g.reg = g.stagebuf = nullptr;
    g.alpha[0] = g.alpha[1] = g.alpha_used = nullptr;
    g.nbr = nullptr; g.cdel = g.delta = nullptr; g.group = nullptr; g.part = nullptr;
    g.has_mesh = g.has_state = false;
    g.prepared = false;
}

bool blended() { return g.cfg.indicator != NEMO_IND_NONE; }

// float offset of the transposed weights in g.mlp32 (16-byte aligned)
int mlp_t_offset() { return (MLP_NPACK + 3) / 4 * 4; }

StageArgs stage_args(int st, bool rhs_only) {
    StageArgs a{};
    a.E = g.E;
    a.E_begin = 0;
    a.E_own = g.E_own;
    a.tick = 1;
    a.u_in = g.u[g.cur];
    a.u_out = g.u[g.cur ^ 1];
    a.reg = g.reg;
    a.nbr = g.nbr;
    a.cdel = g.cdel;
    a.delta = g.delta;
    a.alpha_in = blended() ? g.alpha[g.cur] : nullptr;
    a.alpha_out = (blended() && !rhs_only) ? g.alpha[g.cur ^ 1] : nullptr;
    a.alpha_used = blended() ? g.alpha_used : nullptr;
    a.group = g.ngroups > 1 ? g.group : nullptr;
    a.ctrl = g.ctrl;
    a.rhs_out = nullptr;
    a.stage = st;
    a.epi_dt = (st == 4 && !rhs_only) ? 1 : 0;
    a.smooth = g.cfg.alpha_smoothing;
    a.positivity = g.cfg.positivity;
    a.surface_flux = g.cfg.surface_flux;
    a.volume_flux = g.cfg.volume_flux;
    a.prep_only = 0;
    const bool learned = g.cfg.indicator == NEMO_IND_LEARNED && g.mlp_ready;
    a.mlp64 = learned ? g.mlp64 : nullptr;
    a.mlp32 = learned ? g.mlp32 : nullptr;
    a.mlp32t = learned ? g.mlp32 + mlp_t_offset() : nullptr;
    a.feat_out = nullptr;
    a.alpha_modal_out = nullptr;
    a.mflux = g.mflux;
    a.mflag = g.mflag;
    return a;
}

bool is_mhd() { return g.cfg.eqn == NEMO_EQN_MHD; }

MortarArgs mortar_args(const StageArgs& a, bool rhs_only) {
    MortarArgs m{};
    m.E = a.E;
    m.nm = g.nm;
    m.u_in = a.u_in;
    m.mortar = g.mortar;
    m.mflux = g.mflux;
    m.ctrl = g.ctrl;
    m.mhd = is_mhd() ? 1 : 0;
    m.surface_flux = g.cfg.surface_flux;
    m.skip_if_done = rhs_only ? 0 : 1;
    return m;
}

bool persistent_stage(const StageArgs& a, bool rhs_only) {
    return g.tune_mode == 1 && !rhs_only && !a.prep_only && !is_mhd() && g.cfg.precision == NEMO_PREC_FP32;
}

cudaError_t launch_stage_any(const StageArgs& a, bool rhs_only, cudaStream_t s) {
    if (persistent_stage(a, rhs_only)) {
        MortarArgs m = mortar_args(a, rhs_only);
        m.mflag = g.mflag;
        return launch_stage_euler32p(a, m, blended(), g.tune_ctas, s);
    }
    if (g.nm > 0 && !a.prep_only) {  // fluxes of the 2:1 faces of u_in first
        MortarArgs m{};
        m.E = a.E;
        m.nm = g.nm;
        m.u_in = a.u_in;
        m.mortar = g.mortar;
        m.mflux = g.mflux;
        m.ctrl = g.ctrl;
        m.mhd = is_mhd() ? 1 : 0;
        m.surface_flux = g.cfg.surface_flux;
        m.skip_if_done = rhs_only ? 0 : 1;
        cudaError_t e = launch_mortar(m, s);
        if (e != cudaSuccess) return e;
    }
    if (is_mhd()) {
        if (g.cfg.precision == NEMO_PREC_FP32) return launch_stage_mhd32(a, blended(), rhs_only, s);
        return launch_stage_mhd64(a, blended(), rhs_only, s);
    }
    if (g.cfg.precision == NEMO_PREC_FP32)
        return launch_stage_euler32(a, blended(), rhs_only, s, g.tune_mode == 2 ? 4 : (g.tune_mode == 3 ? 16 : 8));
    return launch_stage_euler64(a, blended(), blended(), rhs_only, s);
}

cudaError_t launch_stage(int st, cudaStream_t s) {
    StageArgs a = stage_args(st, false);
    cudaError_t e = launch_stage_any(a, false, s);
    g.cur ^= 1;
    return e;
}

// One part of a stage over owned elements [begin, end) of u[cur] (u[cur] stays current: the caller
// toggles after the last part).  The mortar rows are recomputed for every part: a part that follows
// a ghost refresh sees the fresh traces, and the rows the earlier part used are rewritten with the
// same values where they read no ghost.  tick: this part advances t and the step counter.
cudaError_t launch_stage_part(int st, int64_t begin, int64_t end, bool tick, cudaStream_t s) {
    StageArgs a = stage_args(st, false);
    a.E_begin = begin;
    a.E_own = end;
    a.tick = tick ? 1 : 0;
    if (end <= begin && g.nm == 0) return cudaSuccess;
    return launch_stage_any(a, false, s);
}

// Indicator (and, if dt_cand, the CFL bound) of the state in u[cur]: the stage kernel's epilogue
// on the loaded state.
cudaError_t launch_prepare(bool dt_cand, cudaStream_t s, float* feat = nullptr, double* alpha_modal = nullptr) {
    StageArgs a = stage_args(0, true);
    a.prep_only = 1;
    a.alpha_out = blended() ? g.alpha[g.cur] : (feat ? g.alpha_used : nullptr);
    a.epi_dt = dt_cand ? 1 : 0;
    a.feat_out = feat;
    a.alpha_modal_out = alpha_modal;
    if (feat) return launch_stage_euler32(a, blended(), false, s);
    return launch_stage_any(a, false, s);
}

int ensure_ready() {
    if (!g.inited) return fail(NEMO_ERR_STATE, "nemo_gpu_init has not been called");
    if (!g.has_mesh) return fail(NEMO_ERR_STATE, "no mesh (nemo_gpu_set_mesh)");
    if (!g.has_state) return fail(NEMO_ERR_STATE, "no state (nemo_gpu_upload_state)");
    return NEMO_OK;
}

// Make alpha[cur] and the CFL bounds in ctrl valid for u[cur].
int prepare_if_needed() {
    if (g.prepared) return NEMO_OK;
    CK(launch_ctrl_reset(g.ctrl, g.stream));
    CK(launch_prepare(true, g.stream));
    g.prepared = true;
    return NEMO_OK;
}

int check_ctrl_error() {
    int32_t err = 0;
    CK(cudaMemcpyAsync(&err, &g.ctrl->error, sizeof err, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    if (err & 1) return fail(NEMO_ERR_CUDA, "a bounded device wait expired (TMA copy did not complete)");
    if (err & 2) return fail(NEMO_ERR_NONFINITE, "non-finite or negative time step");
    if (err & 4) return fail(NEMO_ERR_CUDA, "a bounded wait on a mortar flag expired");
    return NEMO_OK;
}

int build_graph(int start) {
    // [ctrl step, stage 1..5] starting from u[start]
    const int saved = g.cur;
    g.cur = start;
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(g.stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = launch_ctrl_step(g.ctrl, g.stream);
    for (int st = 0; st < 5 && e == cudaSuccess; ++st) e = launch_stage(st, g.stream);
    cudaError_t e2 = cudaStreamEndCapture(g.stream, &graph);
    g.cur = saved;
    if (e != cudaSuccess) return fail(NEMO_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    if (e2 != cudaSuccess) return fail(NEMO_ERR_CUDA, "graph capture end: %s", cudaGetErrorString(e2));
    cudaError_t e3 = cudaGraphInstantiate(&g.graph[start], graph, 0);
    cudaGraphDestroy(graph);
    if (e3 != cudaSuccess) return fail(NEMO_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e3));
    return NEMO_OK;
}

// The control block of a new run (time 0, counters reset, the configuration's GLM values).
Control fresh_control() {
    Control c{};
    c.ngroups = g.ngroups;
    c.dt_factor = 0.25 * g.cfg.cfl / (double)(2 * NN - 1);
    c.glm_ch = g.cfg.glm_ch;
    c.glm_alpha = g.cfg.glm_alpha;
    c.mhd = is_mhd() ? 1 : 0;
    return c;
}

}  // namespace

namespace nemo {
void set_last_error(const char* msg) { std::snprintf(g.err, sizeof g.err, "%s", msg); }
}  // namespace nemo

// ================================================================================================
extern "C" {

int nemo_gpu_default_cfg(nemo_cfg* cfg) {
    if (!cfg) return fail(NEMO_ERR_ARG, "cfg is NULL");
    std::memset(cfg, 0, sizeof *cfg);
    cfg->n_nodes = NN;
    cfg->n_vars = 5;
    cfg->eqn = NEMO_EQN_EULER;
    cfg->volume_flux = NEMO_VOLFLUX_CHANDRASHEKAR;
    cfg->surface_flux = NEMO_SURFFLUX_HLLC;
    cfg->precision = NEMO_PREC_FP64;
    cfg->indicator = NEMO_IND_NONE;
    cfg->alpha_smoothing = 1;
    cfg->positivity = 0;
    cfg->kappa = 1.4;
    cfg->mu0 = 1.0;
    cfg->cfl = 0.5;
    cfg->alpha_max = 0.5;
    cfg->alpha_min = 0.001;
    cfg->repair_decr = 0.01;
    return NEMO_OK;
}

int nemo_gpu_mortar_operators(int32_t n, double* prolong, double* project) {
    if (n != NN) return fail(NEMO_ERR_ARG, "only n = %d Gauss-Lobatto nodes are compiled (got %d)", NN, n);
    HostOps h;
    build_host_ops(h);
    if (prolong) std::memcpy(prolong, h.pro, sizeof h.pro);
    if (project) std::memcpy(project, h.prj, sizeof h.prj);
    return NEMO_OK;
}

int nemo_gpu_amr_operators(int32_t n, int32_t qmax, double* refine, double* coarsen) {
    if (n != NN) return fail(NEMO_ERR_ARG, "only n = %d Gauss-Lobatto nodes are compiled (got %d)", NN, n);
    if (qmax < 0 || qmax > NN - 1) return fail(NEMO_ERR_ARG, "qmax must be in [0, %d] (got %d)", NN - 1, qmax);
    HostOps h;
    build_host_ops(h);
    for (int q = 0; q <= qmax; ++q) {
        // nodal filter to the Legendre modes 0..q of one direction: P = V diag(m <= q) Vinv
        double P[NN * NN];
        for (int i = 0; i < NN; ++i)
            for (int j = 0; j < NN; ++j) {
                double acc = 0.0;
                for (int m = 0; m <= q; ++m) acc = acc + h.V[i * NN + m] * h.Vinv[m * NN + j];
                P[i * NN + j] = acc;
            }
        for (int f = 0; f < 8; ++f)
            for (int d = 0; d < 3; ++d) {
                const int s = (f >> d) & 1;   // child f = cx + 2 cy + 4 cz: its half in direction d
                for (int i = 0; i < NN; ++i)
                    for (int j = 0; j < NN; ++j) {
                        double r = 0.0, c = 0.0;
                        for (int m = 0; m < NN; ++m) {
                            r = r + h.pro[s][i * NN + m] * P[m * NN + j];
                            c = c + P[i * NN + m] * h.prj[s][m * NN + j];
                        }
                        // Fortran layout (N, N, 3, 8, 0:qmax), first index fastest
                        const size_t o = (size_t)i + NN * ((size_t)j + NN * ((size_t)d + 3 * ((size_t)f + 8 * (size_t)q)));
                        if (refine) refine[o] = r;
                        if (coarsen) coarsen[o] = c;
                    }
            }
    }
    return NEMO_OK;
}

int nemo_gpu_repair_states(double* host, int64_t n, int64_t stride, int32_t* ok_host) {
    if (!g.inited) return fail(NEMO_ERR_STATE, "call nemo_gpu_init first");
    if (n < 0 || (n > 0 && (!host || !ok_host))) return fail(NEMO_ERR_ARG, "bad repair arguments");
    if (n == 0) return NEMO_OK;
    const size_t row = sizeof(double) * (size_t)g.V * NP;
    if (stride < (int64_t)row) return fail(NEMO_ERR_ARG, "element stride %lld < %zu bytes", (long long)stride, row);
    double* dst = nullptr;
    int32_t* dok = nullptr;
    cudaError_t err = cudaMalloc(&dst, row * (size_t)n);
    if (err == cudaSuccess) err = cudaMalloc(&dok, sizeof(int32_t) * (size_t)n);
    if (err == cudaSuccess)
        err = cudaMemcpy2DAsync(dst, row, host, (size_t)stride, row, (size_t)n, cudaMemcpyHostToDevice, g.stream);
    if (err == cudaSuccess) err = launch_repair_states64(dst, n, g.V, is_mhd() ? 1 : 0, dok, g.stream);
    if (err == cudaSuccess)
        err = cudaMemcpy2DAsync(host, (size_t)stride, dst, row, row, (size_t)n, cudaMemcpyDeviceToHost, g.stream);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(ok_host, dok, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, g.stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(g.stream);
    if (dst) cudaFree(dst);
    if (dok) cudaFree(dok);
    if (err != cudaSuccess) return fail(NEMO_ERR_CUDA, "%s", cudaGetErrorString(err));
    int64_t nbad = 0;
    for (int64_t e = 0; e < n; ++e) nbad += ok_host[e] ? 0 : 1;
    if (nbad) return fail(NEMO_ERR_REPAIR, "%lld of %lld elements stay inadmissible after the repair", (long long)nbad,
                          (long long)n);
    return NEMO_OK;
}

int nemo_gpu_operators(int32_t n, double* nodes, double* weights, double* dmat, double* smat, double* vinv) {
    if (n != NN) return fail(NEMO_ERR_ARG, "only n = %d Gauss-Lobatto nodes are compiled (got %d)", NN, n);
    HostOps h;
    build_host_ops(h);
    if (nodes) std::memcpy(nodes, h.x, sizeof h.x);
    if (weights) std::memcpy(weights, h.w, sizeof h.w);
    if (dmat) std::memcpy(dmat, h.D, sizeof h.D);
    if (smat) std::memcpy(smat, h.S, sizeof h.S);
    if (vinv) std::memcpy(vinv, h.Vinv, sizeof h.Vinv);
    return NEMO_OK;
}

int nemo_gpu_init(const nemo_cfg* cfg) {
    if (!cfg) return fail(NEMO_ERR_ARG, "cfg is NULL");
    if (cfg->n_nodes != NN) return fail(NEMO_ERR_ARG, "n_nodes must be %d", NN);
    if (cfg->eqn == NEMO_EQN_EULER) {
        if (cfg->n_vars != 5) return fail(NEMO_ERR_ARG, "the Euler equations have n_vars 5");
        if (cfg->volume_flux != NEMO_VOLFLUX_CHANDRASHEKAR && cfg->volume_flux != NEMO_VOLFLUX_CENTRAL)
            return fail(NEMO_ERR_ARG, "unsupported Euler volume flux %d", cfg->volume_flux);
        if (cfg->surface_flux != NEMO_SURFFLUX_HLLC && cfg->surface_flux != NEMO_SURFFLUX_RUSANOV)
            return fail(NEMO_ERR_ARG, "unsupported Euler surface flux %d", cfg->surface_flux);
    } else if (cfg->eqn == NEMO_EQN_MHD) {
        if (cfg->n_vars != 9) return fail(NEMO_ERR_ARG, "GLM-MHD has n_vars 9");
        if (cfg->volume_flux != NEMO_VOLFLUX_EC_MHD && cfg->volume_flux != NEMO_VOLFLUX_CENTRAL)
            return fail(NEMO_ERR_ARG, "unsupported MHD volume flux %d", cfg->volume_flux);
        if (cfg->surface_flux != NEMO_SURFFLUX_RUSANOV && cfg->surface_flux != NEMO_SURFFLUX_HLLD)
            return fail(NEMO_ERR_ARG, "unsupported MHD surface flux %d (Rusanov or HLLD)", cfg->surface_flux);
        if (!(cfg->mu0 > 0.0)) return fail(NEMO_ERR_ARG, "mu0 must be positive");
        // the HLLD star states assume mu0 = 1 (source/equations/mhd/riemann/hlld/riemann_mod.f90:13)
        if (cfg->surface_flux == NEMO_SURFFLUX_HLLD && cfg->mu0 != 1.0)
            return fail(NEMO_ERR_ARG, "the HLLD surface flux requires mu0 = 1 (got %g)", cfg->mu0);
    } else {
        return fail(NEMO_ERR_ARG, "unknown equation system %d", cfg->eqn);
    }
    if (cfg->precision != NEMO_PREC_FP64 && cfg->precision != NEMO_PREC_FP32)
        return fail(NEMO_ERR_ARG, "unsupported precision %d", cfg->precision);
    if (cfg->indicator != NEMO_IND_NONE && cfg->indicator != NEMO_IND_MODAL && cfg->indicator != NEMO_IND_LEARNED)
        return fail(NEMO_ERR_ARG, "unsupported indicator %d", cfg->indicator);
    if (!(cfg->kappa > 1.0)) return fail(NEMO_ERR_ARG, "kappa must be > 1");
    if (cfg->source != NEMO_SOURCE_NONE && cfg->source != NEMO_SOURCE_BAROTROPIC_COOLING)
        return fail(NEMO_ERR_ARG, "unknown source term %d", cfg->source);
    if (cfg->source == NEMO_SOURCE_BAROTROPIC_COOLING) {
        if (cfg->eqn != NEMO_EQN_EULER) return fail(NEMO_ERR_ARG, "barotropic cooling is an Euler source term");
        if (!(cfg->dens_critical > 0.0) || !(cfg->k_isothermal > 0.0) || !(cfg->k_adiabatic > 0.0))
            return fail(NEMO_ERR_ARG, "barotropic cooling needs dens_critical, k_isothermal, k_adiabatic > 0");
    }
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (ndev < 1) return fail(NEMO_ERR_CUDA, "no CUDA device");
    if (g.inited) nemo_gpu_finalize();
    g.cfg = *cfg;
    g.V = cfg->n_vars;
    build_host_ops(g.hops);
    OpConsts& o = g.ops;
    std::memcpy(o.S, g.hops.S, sizeof o.S);
    for (int i = 0; i < NN; ++i) o.winv[i] = 1.0 / g.hops.w[i];
    std::memcpy(o.Vinv, g.hops.Vinv, sizeof o.Vinv);
    for (int i = 0; i < NN; ++i) o.wt[i] = 0.5 * g.hops.w[i];
    o.kappa = cfg->kappa;
    o.km1 = cfg->kappa - 1.0;
    o.c_enth = 0.5 / (cfg->kappa - 1.0);
    o.hllc_beta = std::sqrt(0.5 * (cfg->kappa - 1) / cfg->kappa);
    o.ind_T = 0.5 * std::pow(10.0, -1.8 * std::pow((double)NN, 0.25));
    const double s = std::log((1.0 - 0.0001) / 0.0001);
    o.ind_k = -s / o.ind_T;
    o.alpha_min = cfg->alpha_min;
    o.alpha_max = cfg->alpha_max;
    o.one_m_alpha_min = 1.0 - cfg->alpha_min;
    o.repair_decr = cfg->repair_decr;
    o.mu0 = cfg->mu0;
    o.cool = cfg->source == NEMO_SOURCE_BAROTROPIC_COOLING ? 1 : 0;
    o.cool_rho = cfg->dens_critical;
    o.cool_ci = cfg->k_isothermal / (cfg->kappa - 1.0);
    o.cool_ca = cfg->k_adiabatic / (cfg->kappa - 1.0);
    std::memcpy(o.x, g.hops.x, sizeof o.x);
    std::memcpy(o.w, g.hops.w, sizeof o.w);
    std::memcpy(o.pro, g.hops.pro, sizeof o.pro);
    std::memcpy(o.prj, g.hops.prj, sizeof o.prj);
    for (int i = 0; i < NN * NN; ++i) {
        o.S32[i] = (float)o.S[i];
        o.Vinv32[i] = (float)o.Vinv[i];
    }
    for (int i = 0; i < NN; ++i) o.winv32[i] = (float)o.winv[i];
    o.kappa32 = (float)o.kappa;
    o.km1_32 = (float)o.km1;
    o.ikm1_32 = (float)(1.0 / o.km1);
    o.c_enth32 = (float)o.c_enth;
    o.hllc_beta32 = (float)o.hllc_beta;
    o.ind_k32 = (float)o.ind_k;
    o.ind_T32 = (float)o.ind_T;
    o.alpha_min32 = (float)o.alpha_min;
    o.alpha_max32 = (float)o.alpha_max;
    o.one_m_alpha_min32 = (float)o.one_m_alpha_min;
    CK(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
    CK(setup_stage_euler64(o));
    CK(setup_stage_euler32(o));
    CK(setup_stage_mhd64());
    CK(setup_stage_mhd32());
    CK(setup_mortar(o));
    CK(cudaMalloc(&g.ctrl, sizeof(Control)));
    CK(cudaMemset(g.ctrl, 0, sizeof(Control)));
    CK(cudaMalloc(&g.tot, 16 * sizeof(double)));
    CK(cudaMalloc(&g.mlp32, sizeof(float) * (MLP_NPACK + 8 + MLP_NT)));
    CK(cudaMalloc(&g.mlp64, sizeof(double) * MLP_NPACK));
    g.mlp_ready = false;
    g.inited = true;
    g.ngroups = 1;
    return NEMO_OK;
}

int nemo_gpu_set_mesh(int64_t nelems, const double* delta, const double* center, int64_t nsides,
                      const int32_t* side_quads, const int8_t* side_faceid, const int8_t* side_nquads,
                      const int32_t* boundary) {
    if (!g.inited) return fail(NEMO_ERR_STATE, "nemo_gpu_init has not been called");
    if (nelems <= 0 || nsides <= 0) return fail(NEMO_ERR_ARG, "nelems and nsides must be positive");
    if (!delta || !side_quads || !side_faceid || !side_nquads || !boundary)
        return fail(NEMO_ERR_ARG, "NULL mesh array");
    (void)center;
    const int64_t E = nelems;
    constexpr int32_t UNSET = INT32_MIN;
    std::vector<int32_t> nbr(E * 6, UNSET);
    std::vector<int32_t> mort;
    for (int64_t s = 0; s < nsides; ++s) {
        const int n0 = side_nquads[s * 2 + 0], n1 = side_nquads[s * 2 + 1];
        const int f0 = side_faceid[s * 2 + 0], f1 = side_faceid[s * 2 + 1];
        const int32_t* q0 = side_quads + s * 8;
        const int32_t* q1 = side_quads + s * 8 + 4;
        auto bad_quad = [&](int32_t q, int f) { return f < 0 || f > 5 || q < 0 || q >= E; };
        if (n0 == 4 || n1 == 4) {  // 2:1 mortar: one coarse quad, four fine quads
            if (!((n0 == 1 && n1 == 4) || (n0 == 4 && n1 == 1)) || boundary[s] > 0)
                return fail(NEMO_ERR_ARG, "side %lld: a mortar side joins 1 and 4 quads in the interior", (long long)s);
            const bool c0 = n0 == 1;
            const int32_t* qc = c0 ? q0 : q1;
            const int32_t* qf = c0 ? q1 : q0;
            const int fc = c0 ? f0 : f1, ff = c0 ? f1 : f0;
            if ((fc >> 1) != (ff >> 1) || fc == ff)
                return fail(NEMO_ERR_ARG, "side %lld: faces %d/%d are not opposite faces of one direction", (long long)s, fc, ff);
            if (bad_quad(qc[0], fc)) return fail(NEMO_ERR_ARG, "side %lld: bad coarse quad", (long long)s);
            const int32_t m = (int32_t)(mort.size() / 6);
            if ((int64_t)m * 5 + 5 > (int64_t)INT32_MAX - 2) return fail(NEMO_ERR_ARG, "too many mortars");
            mort.push_back(qc[0]);
            mort.push_back(fc);
            nbr[qc[0] * 6 + fc] = -2 - 5 * m;
            for (int k = 0; k < 4; ++k) {
                if (bad_quad(qf[k], ff)) return fail(NEMO_ERR_ARG, "side %lld: bad fine quad %d", (long long)s, k);
                mort.push_back(qf[k]);
                nbr[qf[k] * 6 + ff] = -2 - (5 * m + 1 + k);
            }
            continue;
        }
        if (n0 != 1) return fail(NEMO_ERR_ARG, "side %lld: first half must hold one element", (long long)s);
        if (bad_quad(q0[0], f0)) return fail(NEMO_ERR_ARG, "side %lld: bad element/face", (long long)s);
        if (n1 == 0 || boundary[s] > 0) {
            nbr[q0[0] * 6 + f0] = -1;
        } else {
            if (n1 != 1 || bad_quad(q1[0], f1)) return fail(NEMO_ERR_ARG, "side %lld: bad element/face", (long long)s);
            if ((f0 >> 1) != (f1 >> 1) || f0 == f1)
                return fail(NEMO_ERR_ARG, "side %lld: faces %d/%d are not opposite faces of one direction", (long long)s, f0, f1);
            nbr[q0[0] * 6 + f0] = q1[0];
            nbr[q1[0] * 6 + f1] = q0[0];
        }
    }
    for (int64_t i = 0; i < E * 6; ++i)
        if (nbr[i] == UNSET) return fail(NEMO_ERR_ARG, "element %lld face %d has no side", (long long)(i / 6), (int)(i % 6));
    const int64_t nm = (int64_t)(mort.size() / 6);
    std::vector<double> cd(E * 3);
    for (int64_t i = 0; i < E * 3; ++i) {
        if (!(delta[i] > 0.0)) return fail(NEMO_ERR_ARG, "element %lld has non-positive size", (long long)(i / 3));
        cd[i] = 2.0 / delta[i];
    }
    release_mesh();
    g.E = E;
    g.E_own = E;
    const size_t bytes = sizeof(double) * (size_t)g.V * E * NP;
    CK(cudaMalloc(&g.u[0], bytes));
    CK(cudaMalloc(&g.u[1], bytes));
    CK(cudaMalloc(&g.reg, bytes));
    CK(cudaMalloc(&g.stagebuf, bytes));
    CK(cudaMalloc(&g.alpha[0], sizeof(double) * E));
    CK(cudaMalloc(&g.alpha[1], sizeof(double) * E));
    CK(cudaMalloc(&g.alpha_used, sizeof(double) * E));
    CK(cudaMemset(g.alpha[0], 0, sizeof(double) * E));
    CK(cudaMemset(g.alpha[1], 0, sizeof(double) * E));
    CK(cudaMemset(g.alpha_used, 0, sizeof(double) * E));
    CK(cudaMalloc(&g.nbr, sizeof(int32_t) * E * 6));
    CK(cudaMalloc(&g.cdel, sizeof(double) * E * 3));
    CK(cudaMalloc(&g.delta, sizeof(double) * E * 3));
    CK(cudaMalloc(&g.part, sizeof(double) * (size_t)g.V * E));
    CK(cudaMemcpy(g.nbr, nbr.data(), sizeof(int32_t) * E * 6, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(g.cdel, cd.data(), sizeof(double) * E * 3, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(g.delta, delta, sizeof(double) * E * 3, cudaMemcpyHostToDevice));
    g.nm = nm;
    if (nm > 0) {
        CK(cudaMalloc(&g.mortar, sizeof(int32_t) * 6 * nm));
        CK(cudaMemcpy(g.mortar, mort.data(), sizeof(int32_t) * 6 * nm, cudaMemcpyHostToDevice));
        CK(cudaMalloc(&g.mflux, sizeof(double) * 5 * nm * g.V * NF));
        CK(cudaMemset(g.mflux, 0, sizeof(double) * 5 * nm * g.V * NF));
        CK(cudaMalloc(&g.mflag, sizeof(uint32_t) * nm));
        CK(cudaMemset(g.mflag, 0, sizeof(uint32_t) * nm));
    }
    g.ngroups = 1;
    Control c{};
    c.ngroups = 1;
    c.dt_factor = 0.25 * g.cfg.cfl / (double)(2 * NN - 1);
    c.glm_ch = g.cfg.glm_ch;
    c.glm_alpha = g.cfg.glm_alpha;
    c.mhd = is_mhd() ? 1 : 0;
    c.epoch = 1u;   // mortar flags start at 0: never equal to a launch's epoch before it sets them
    CK(cudaMemcpy(g.ctrl, &c, sizeof c, cudaMemcpyHostToDevice));
    g.has_mesh = true;
    return NEMO_OK;
}

int nemo_gpu_adapt(int64_t nelems, const double* delta, const double* center, int64_t nsides,
                   const int32_t* side_quads, const int8_t* side_faceid, const int8_t* side_nquads,
                   const int32_t* boundary, const int32_t* remap) {
    int st = ensure_ready();
    if (st) return st;
    if (nelems <= 0 || !remap) return fail(NEMO_ERR_ARG, "adapt needs nelems > 0 and a remap table");
    if (g.ngroups > 1 || g.E_own != g.E)
        return fail(NEMO_ERR_STATE, "adapt supports one run on one process (no groups, no ghost elements)");
    const int64_t Eo = g.E;
    for (int64_t e = 0; e < nelems; ++e) {
        const int32_t* r = remap + 4 * e;
        const int kind = r[0];
        const int64_t src = r[1];
        bool ok = kind >= 0 && kind <= 2 && src >= 0;
        if (kind == 0) ok = ok && src < Eo;
        if (kind == 1) {
            const int d = r[2], o = r[3];
            ok = ok && src < Eo && d >= 1 && d <= 7 && (o & 0xff) < (1 << d) && ((o >> 8) & 0xff) < (1 << d) &&
                 ((o >> 16) & 0xff) < (1 << d) && (o >> 24) == 0;
        }
        if (kind == 2) ok = ok && src + 8 <= Eo;
        if (!ok) return fail(NEMO_ERR_ARG, "remap row %lld is invalid", (long long)e);
    }
    // the new state from the old one, before the mesh (and its buffers) is replaced
    const size_t bytes = sizeof(double) * (size_t)g.V * nelems * NP;
    double* tmp = nullptr;
    int32_t* rm = nullptr;
    CK(cudaMalloc(&tmp, bytes));
    // remap rows, then one flag per old element and per new element for the admissibility fallback
    cudaError_t e1 = cudaMalloc(&rm, sizeof(int32_t) * (4 * nelems + Eo + nelems));
    if (e1 == cudaSuccess) e1 = cudaMemcpy(rm, remap, sizeof(int32_t) * 4 * nelems, cudaMemcpyHostToDevice);
    if (e1 == cudaSuccess) e1 = launch_remap(g.u[g.cur], Eo, tmp, nelems, rm, g.V, rm + 4 * nelems, g.stream);
    if (e1 == cudaSuccess) e1 = cudaStreamSynchronize(g.stream);
    double t0 = 0.0;
    unsigned long long steps = 0;
    if (e1 == cudaSuccess) e1 = cudaMemcpy(&t0, &g.ctrl->t[0], sizeof t0, cudaMemcpyDeviceToHost);
    if (e1 == cudaSuccess) e1 = cudaMemcpy(&steps, &g.ctrl->steps, sizeof steps, cudaMemcpyDeviceToHost);
    cudaFree(rm);
    if (e1 != cudaSuccess) {
        cudaFree(tmp);
        return fail(NEMO_ERR_CUDA, "adapt: %s", cudaGetErrorString(e1));
    }
    st = nemo_gpu_set_mesh(nelems, delta, center, nsides, side_quads, side_faceid, side_nquads, boundary);
    if (st) {
        cudaFree(tmp);
        return st;
    }
    e1 = cudaMemcpy(g.u[0], tmp, bytes, cudaMemcpyDeviceToDevice);
    cudaFree(tmp);
    if (e1 != cudaSuccess) return fail(NEMO_ERR_CUDA, "adapt: %s", cudaGetErrorString(e1));
    CK(cudaMemset(g.reg, 0, bytes));
    CK(cudaMemcpy(&g.ctrl->t[0], &t0, sizeof t0, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(&g.ctrl->steps, &steps, sizeof steps, cudaMemcpyHostToDevice));
    g.cur = 0;
    g.has_state = true;
    g.prepared = false;
    return NEMO_OK;
}

int nemo_gpu_amr_flags(double refine_threshold, double coarsen_threshold, int32_t* flags) {
    int st = ensure_ready();
    if (st) return st;
    if (!flags) return fail(NEMO_ERR_ARG, "flags is NULL");
    int32_t* d = nullptr;
    CK(cudaMalloc(&d, sizeof(int32_t) * g.E));
    cudaError_t e1 = launch_amr_flags(g.u[g.cur], g.E, refine_threshold, coarsen_threshold, d, g.stream);
    if (e1 == cudaSuccess) e1 = cudaMemcpyAsync(flags, d, sizeof(int32_t) * g.E, cudaMemcpyDeviceToHost, g.stream);
    if (e1 == cudaSuccess) e1 = cudaStreamSynchronize(g.stream);
    cudaFree(d);
    if (e1 != cudaSuccess) return fail(NEMO_ERR_CUDA, "amr_flags: %s", cudaGetErrorString(e1));
    return NEMO_OK;
}

int nemo_gpu_set_owned(int64_t n_owned) {
    if (!g.has_mesh) return fail(NEMO_ERR_STATE, "set the mesh first");
    if (n_owned < 1 || n_owned > g.E) return fail(NEMO_ERR_ARG, "n_owned must be in [1, %lld]", (long long)g.E);
    g.E_own = n_owned;
    g.n_interior = 0;
    release_graphs();
    g.prepared = false;
    return NEMO_OK;
}

int nemo_gpu_pack_elements(const int32_t* idx_dev, int64_t n, double* buf_dev) {
    int st = ensure_ready();
    if (st) return st;
    if (n < 0 || (n > 0 && (!idx_dev || !buf_dev))) return fail(NEMO_ERR_ARG, "bad pack arguments");
    if ((st = prepare_if_needed())) return st;
    CK(launch_pack(g.u[g.cur], blended() ? g.alpha[g.cur] : nullptr, idx_dev, n, g.E, g.V, buf_dev, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    return NEMO_OK;
}

int nemo_gpu_unpack_elements(const int32_t* idx_dev, int64_t n, const double* buf_dev) {
    int st = ensure_ready();
    if (st) return st;
    if (n < 0 || (n > 0 && (!idx_dev || !buf_dev))) return fail(NEMO_ERR_ARG, "bad unpack arguments");
    if ((st = prepare_if_needed())) return st;
    CK(launch_unpack(g.u[g.cur], blended() ? g.alpha[g.cur] : nullptr, idx_dev, n, g.E, g.V, buf_dev, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    return NEMO_OK;
}

int nemo_gpu_pack_faces(const int32_t* idx_dev, const int32_t* face_dev, int64_t n, double* buf_dev) {
    int st = ensure_ready();
    if (st) return st;
    if (n < 0 || (n > 0 && (!idx_dev || !face_dev || !buf_dev))) return fail(NEMO_ERR_ARG, "bad pack arguments");
    if ((st = prepare_if_needed())) return st;
    CK(launch_pack_faces(g.u[g.cur], blended() ? g.alpha[g.cur] : nullptr, idx_dev, face_dev, n, g.E, g.V, buf_dev,
                         g.stream));
    CK(cudaStreamSynchronize(g.stream));
    return NEMO_OK;
}

int nemo_gpu_unpack_faces(const int32_t* idx_dev, const int32_t* face_dev, int64_t n, const double* buf_dev) {
    int st = ensure_ready();
    if (st) return st;
    if (n < 0 || (n > 0 && (!idx_dev || !face_dev || !buf_dev))) return fail(NEMO_ERR_ARG, "bad unpack arguments");
    if ((st = prepare_if_needed())) return st;
    CK(launch_unpack_faces(g.u[g.cur], blended() ? g.alpha[g.cur] : nullptr, idx_dev, face_dev, n, g.E, g.V, buf_dev,
                           g.stream));
    CK(cudaStreamSynchronize(g.stream));
    return NEMO_OK;
}

int nemo_gpu_set_groups(int32_t ngroups, const int32_t* group_of_elem) {
    if (!g.has_mesh) return fail(NEMO_ERR_STATE, "set the mesh first");
    if (ngroups < 1 || ngroups > MAX_GROUPS) return fail(NEMO_ERR_ARG, "ngroups must be in [1, %d]", MAX_GROUPS);
    if (ngroups > 1 && !group_of_elem) return fail(NEMO_ERR_ARG, "group_of_elem is NULL");
    if (ngroups > 1) {
        for (int64_t e = 0; e < g.E; ++e)
            if (group_of_elem[e] < 0 || group_of_elem[e] >= ngroups)
                return fail(NEMO_ERR_ARG, "element %lld has group %d outside [0,%d)", (long long)e, group_of_elem[e], ngroups);
        if (!g.group) CK(cudaMalloc(&g.group, sizeof(int32_t) * g.E));
        CK(cudaMemcpy(g.group, group_of_elem, sizeof(int32_t) * g.E, cudaMemcpyHostToDevice));
    }
    release_graphs();
    g.ngroups = ngroups;
    CK(cudaMemcpy(&g.ctrl->ngroups, &ngroups, sizeof(int32_t), cudaMemcpyHostToDevice));
    g.prepared = false;
    return NEMO_OK;
}

int nemo_gpu_upload_state(const double* host, int64_t stride) {
    if (!g.has_mesh) return fail(NEMO_ERR_STATE, "set the mesh first");
    if (!host) return fail(NEMO_ERR_ARG, "host is NULL");
    const size_t row = sizeof(double) * (size_t)g.V * NP;
    if (stride < (int64_t)row) return fail(NEMO_ERR_ARG, "element stride %lld < %zu bytes", (long long)stride, row);
    if (stride == (int64_t)row) CK(cudaMemcpyAsync(g.stagebuf, host, row * g.E, cudaMemcpyHostToDevice, g.stream));
    else CK(cudaMemcpy2DAsync(g.stagebuf, row, host, (size_t)stride, row, (size_t)g.E, cudaMemcpyHostToDevice, g.stream));
    g.cur = 0;
    CK(launch_aos_to_soa(g.stagebuf, g.u[0], g.E, g.V, g.stream));
    CK(cudaMemsetAsync(g.reg, 0, row * g.E, g.stream));
    // reset the simulation time and counters
    const Control c = fresh_control();
    CK(cudaMemcpyAsync(g.ctrl, &c, sizeof c, cudaMemcpyHostToDevice, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    g.has_state = true;
    g.prepared = false;
    return NEMO_OK;
}

int nemo_gpu_upload_state_async(const double* host, int64_t stride) {
    if (!g.has_mesh) return fail(NEMO_ERR_STATE, "set the mesh first");
    if (!host) return fail(NEMO_ERR_ARG, "host is NULL");
    const size_t row = sizeof(double) * (size_t)g.V * NP;
    if (stride < (int64_t)row) return fail(NEMO_ERR_ARG, "element stride %lld < %zu bytes", (long long)stride, row);
    // first call: stream, events, pinned control blocks (each piece on its own, so that a failed
    // set-up is completed by the next call)
    if (!g.in_stream) CK(cudaStreamCreateWithFlags(&g.in_stream, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i) {
        if (!g.in_done[i]) CK(cudaEventCreateWithFlags(&g.in_done[i], cudaEventDisableTiming));
        if (!g.in_free[i]) CK(cudaEventCreateWithFlags(&g.in_free[i], cudaEventDisableTiming));
    }
    if (!g.in_ctrl) CK(cudaHostAlloc((void**)&g.in_ctrl, 2 * sizeof(Control), cudaHostAllocDefault));
    const int64_t bytes = (int64_t)row * g.E;
    if (g.in_bytes != bytes) {
        release_uploads();
        for (int i = 0; i < 2; ++i) CK(cudaMalloc(&g.in_stage[i], (size_t)bytes));
        g.in_bytes = bytes;
    }
    const int s = g.in_next;
    // the slot's previous upload must have been consumed before its staging buffer and control
    // block are written again (two uploads ago: in a pipelined loop this has long happened)
    if (g.in_used[s]) CK(cudaEventSynchronize(g.in_free[s]));
    g.in_ctrl[s] = fresh_control();
    if (stride == (int64_t)row)
        CK(cudaMemcpyAsync(g.in_stage[s], host, (size_t)bytes, cudaMemcpyHostToDevice, g.in_stream));
    else
        CK(cudaMemcpy2DAsync(g.in_stage[s], row, host, (size_t)stride, row, (size_t)g.E, cudaMemcpyHostToDevice,
                             g.in_stream));
    CK(cudaEventRecord(g.in_done[s], g.in_stream));
    // consumed in stream order by the library stream: the work enqueued so far still sees the old
    // state, the work enqueued after this call sees the new one
    CK(cudaStreamWaitEvent(g.stream, g.in_done[s], 0));
    g.cur = 0;
    CK(launch_aos_to_soa(g.in_stage[s], g.u[0], g.E, g.V, g.stream));
    CK(cudaMemsetAsync(g.reg, 0, row * g.E, g.stream));
    CK(cudaMemcpyAsync(g.ctrl, &g.in_ctrl[s], sizeof(Control), cudaMemcpyHostToDevice, g.stream));
    CK(cudaEventRecord(g.in_free[s], g.stream));
    g.in_used[s] = true;
    g.in_next = s ^ 1;
    g.has_state = true;
    g.prepared = false;
    return NEMO_OK;
}

int nemo_gpu_download_state_async(double* host, int64_t stride) {
    int st = ensure_ready();
    if (st) return st;
    if (!host) return fail(NEMO_ERR_ARG, "host is NULL");
    const size_t row = sizeof(double) * (size_t)g.V * NP;
    if (stride < (int64_t)row) return fail(NEMO_ERR_ARG, "element stride %lld < %zu bytes", (long long)stride, row);
    if (!g.out_stream) CK(cudaStreamCreateWithFlags(&g.out_stream, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i) {
        if (!g.out_ready[i]) CK(cudaEventCreateWithFlags(&g.out_ready[i], cudaEventDisableTiming));
        if (!g.out_done[i]) CK(cudaEventCreateWithFlags(&g.out_done[i], cudaEventDisableTiming));
    }
    const int64_t bytes = (int64_t)row * g.E;
    if (g.out_bytes != bytes) {
        release_downloads();
        for (int i = 0; i < 2; ++i) CK(cudaMalloc(&g.out_stage[i], (size_t)bytes));
        g.out_bytes = bytes;
    }
    const int s = g.out_next;
    // the slot's previous copy must have left the staging buffer (two downloads ago)
    if (g.out_used[s]) CK(cudaEventSynchronize(g.out_done[s]));
    CK(launch_soa_to_aos(g.u[g.cur], g.out_stage[s], g.E, g.V, g.stream));
    CK(cudaEventRecord(g.out_ready[s], g.stream));
    CK(cudaStreamWaitEvent(g.out_stream, g.out_ready[s], 0));
    if (stride == (int64_t)row)
        CK(cudaMemcpyAsync(host, g.out_stage[s], (size_t)bytes, cudaMemcpyDeviceToHost, g.out_stream));
    else
        CK(cudaMemcpy2DAsync(host, (size_t)stride, g.out_stage[s], row, row, (size_t)g.E, cudaMemcpyDeviceToHost,
                             g.out_stream));
    CK(cudaEventRecord(g.out_done[s], g.out_stream));
    g.out_used[s] = true;
    g.out_next = s ^ 1;
    return NEMO_OK;
}

int nemo_gpu_upload_wait(void) {
    for (int i = 0; i < 2; ++i)
        if (g.in_used[i]) CK(cudaEventSynchronize(g.in_done[i]));
    return NEMO_OK;
}

int nemo_gpu_download_state(double* host, int64_t stride) {
    int st = ensure_ready();
    if (st) return st;
    if (!host) return fail(NEMO_ERR_ARG, "host is NULL");
    const size_t row = sizeof(double) * (size_t)g.V * NP;
    if (stride < (int64_t)row) return fail(NEMO_ERR_ARG, "element stride %lld < %zu bytes", (long long)stride, row);
    CK(launch_soa_to_aos(g.u[g.cur], g.stagebuf, g.E, g.V, g.stream));
    if (stride == (int64_t)row) CK(cudaMemcpyAsync(host, g.stagebuf, row * g.E, cudaMemcpyDeviceToHost, g.stream));
    else CK(cudaMemcpy2DAsync(host, (size_t)stride, g.stagebuf, row, row, (size_t)g.E, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    return NEMO_OK;
}

int nemo_gpu_checkpoint_begin(double* host, int64_t stride, double* alpha_host) {
    int st = ensure_ready();
    if (st) return st;
    if (!host) return fail(NEMO_ERR_ARG, "host is NULL");
    const size_t row = sizeof(double) * (size_t)g.V * NP;
    if (stride < (int64_t)row) return fail(NEMO_ERR_ARG, "element stride %lld < %zu bytes", (long long)stride, row);
    if (g.ckpt_pending) {  // the staging buffer is reused: the previous copy must have left it
        CK(cudaEventSynchronize(g.ckpt_done));
        g.ckpt_pending = false;
    }
    // first call: the copy stream, its events and the time/step staging (each piece on its own, so a
    // failed set-up is completed by the next call)
    if (!g.copy_stream) CK(cudaStreamCreateWithFlags(&g.copy_stream, cudaStreamNonBlocking));
    if (!g.ckpt_ready) CK(cudaEventCreateWithFlags(&g.ckpt_ready, cudaEventDisableTiming));
    if (!g.ckpt_done) CK(cudaEventCreateWithFlags(&g.ckpt_done, cudaEventDisableTiming));
    if (!g.ckpt_meta) CK(cudaMalloc(&g.ckpt_meta, 2 * sizeof(double)));
    if (!g.ckpt_meta_host) CK(cudaHostAlloc(&g.ckpt_meta_host, 2 * sizeof(double), cudaHostAllocDefault));
    const int64_t bytes = (int64_t)row * g.E;
    const int64_t abytes = (int64_t)sizeof(double) * g.E;   // blending coefficients after the state
    if (g.ckpt_bytes != bytes + abytes) {
        free_dev(g.ckpt);
        g.ckpt = nullptr;
        g.ckpt_bytes = 0;
        CK(cudaMalloc(&g.ckpt, (size_t)(bytes + abytes)));
        g.ckpt_bytes = bytes + abytes;
    }
    double* ckpt_alpha = g.ckpt + (size_t)g.V * NP * g.E;
    if (alpha_host && !blended()) std::fill(alpha_host, alpha_host + g.E, 0.0);
    // in stream order: the snapshot is the state after everything enqueued so far
    CK(launch_soa_to_aos(g.u[g.cur], g.ckpt, g.E, g.V, g.stream));
    CK(cudaMemcpyAsync(g.ckpt_meta, &g.ctrl->t[0], sizeof(double), cudaMemcpyDeviceToDevice, g.stream));
    CK(cudaMemcpyAsync(g.ckpt_meta + 1, &g.ctrl->steps, sizeof(double), cudaMemcpyDeviceToDevice, g.stream));
    if (alpha_host && blended())
        CK(cudaMemcpyAsync(ckpt_alpha, g.alpha_used, (size_t)abytes, cudaMemcpyDeviceToDevice, g.stream));
    CK(cudaEventRecord(g.ckpt_ready, g.stream));
    CK(cudaStreamWaitEvent(g.copy_stream, g.ckpt_ready, 0));
    if (stride == (int64_t)row) CK(cudaMemcpyAsync(host, g.ckpt, (size_t)bytes, cudaMemcpyDeviceToHost, g.copy_stream));
    else CK(cudaMemcpy2DAsync(host, (size_t)stride, g.ckpt, row, row, (size_t)g.E, cudaMemcpyDeviceToHost, g.copy_stream));
    if (alpha_host && blended())
        CK(cudaMemcpyAsync(alpha_host, ckpt_alpha, (size_t)abytes, cudaMemcpyDeviceToHost, g.copy_stream));
    CK(cudaMemcpyAsync(g.ckpt_meta_host, g.ckpt_meta, 2 * sizeof(double), cudaMemcpyDeviceToHost, g.copy_stream));
    CK(cudaEventRecord(g.ckpt_done, g.copy_stream));
    g.ckpt_pending = true;
    return NEMO_OK;
}

int nemo_gpu_checkpoint_wait(double* t_out, int64_t* steps_out) {
    if (!g.ckpt_pending) return fail(NEMO_ERR_STATE, "no checkpoint copy in flight (nemo_gpu_checkpoint_begin)");
    CK(cudaEventSynchronize(g.ckpt_done));
    g.ckpt_pending = false;
    if (t_out) *t_out = g.ckpt_meta_host[0];
    if (steps_out) {
        unsigned long long s = 0;
        std::memcpy(&s, &g.ckpt_meta_host[1], sizeof s);
        *steps_out = (int64_t)s;
    }
    return NEMO_OK;
}

int nemo_gpu_set_time(double t, int64_t steps) {
    int st = ensure_ready();
    if (st) return st;
    if (!(t >= 0.0) || !std::isfinite(t) || steps < 0) return fail(NEMO_ERR_ARG, "need a finite t >= 0 and steps >= 0");
    double ts[MAX_GROUPS];
    for (int i = 0; i < MAX_GROUPS; ++i) ts[i] = t;
    const unsigned long long s = (unsigned long long)steps;
    CK(cudaMemcpyAsync(g.ctrl->t, ts, sizeof(double) * g.ngroups, cudaMemcpyHostToDevice, g.stream));
    CK(cudaMemcpyAsync(&g.ctrl->steps, &s, sizeof s, cudaMemcpyHostToDevice, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    return NEMO_OK;
}

int nemo_gpu_calc_timestep(double cfl, double* dt_out, double* lmax_out) {
    int st = ensure_ready();
    if (st) return st;
    if (!(cfl > 0.0)) return fail(NEMO_ERR_ARG, "cfl must be positive");
    CK(launch_ctrl_reset(g.ctrl, g.stream));
    CK(launch_prepare(true, g.stream));
    unsigned long long bits[2];
    CK(cudaMemcpyAsync(&bits[0], &g.ctrl->dtmin_bits[0], 8, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaMemcpyAsync(&bits[1], &g.ctrl->lmax_bits[0], 8, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    double dtmin, lmax;
    std::memcpy(&dtmin, &bits[0], 8);
    std::memcpy(&lmax, &bits[1], 8);
    const double dt = 0.25 * cfl / (double)(2 * NN - 1) * dtmin;
    if (!std::isfinite(dt) || !(dt > 0.0)) return fail(NEMO_ERR_NONFINITE, "time step %g is not positive and finite", dt);
    if (is_mhd()) {  // GLM cleaning speed and damping for the coming step (kernel_timestep_mod.f90:338-344)
        unsigned long long vb = 0;
        CK(cudaMemcpy(&vb, &g.ctrl->vmax_bits, 8, cudaMemcpyDeviceToHost));
        double vmax;
        std::memcpy(&vmax, &vb, 8);
        const double gch = 2.0 * std::fabs(lmax - vmax);
        const double gal = gch / 0.18;
        CK(cudaMemcpy(&g.ctrl->glm_ch, &gch, 8, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(&g.ctrl->glm_alpha, &gal, 8, cudaMemcpyHostToDevice));
    }
    if (dt_out) *dt_out = dt;
    if (lmax_out) *lmax_out = lmax;
    g.prepared = true;
    return NEMO_OK;
}

int nemo_gpu_stage(int32_t stage, double dt, double t_stage, int32_t* nbad_out) {
    int st = ensure_ready();
    if (st) return st;
    (void)t_stage;
    if (stage < 1 || stage > 5) return fail(NEMO_ERR_ARG, "stage must be 1..5");
    if (!(dt >= 0.0) || !std::isfinite(dt)) return fail(NEMO_ERR_ARG, "dt must be finite and >= 0");
    unsigned long long nb0 = 0, nb1 = 0;
    CK(cudaMemcpyAsync(&nb0, &g.ctrl->nbad, 8, cudaMemcpyDeviceToHost, g.stream));
    if ((st = prepare_if_needed())) return st;
    CK(launch_ctrl_set_dt(g.ctrl, dt, g.stream));
    CK(launch_stage(stage - 1, g.stream));
    CK(cudaMemcpyAsync(&nb1, &g.ctrl->nbad, 8, cudaMemcpyDeviceToHost, g.stream));
    if ((st = check_ctrl_error())) return st;
    if (nbad_out) *nbad_out = (int32_t)(nb1 - nb0);
    if (nb1 > nb0) return fail(NEMO_ERR_REPAIR, "positivity repair failed on %llu elements", nb1 - nb0);
    return NEMO_OK;
}

int nemo_gpu_step(double dt) {
    int st = ensure_ready();
    if (st) return st;
    if (!(dt >= 0.0) || !std::isfinite(dt)) return fail(NEMO_ERR_ARG, "dt must be finite and >= 0");
    if ((st = prepare_if_needed())) return st;
    CK(launch_ctrl_set_dt(g.ctrl, dt, g.stream));
    for (int s = 0; s < 5; ++s) CK(launch_stage(s, g.stream));
    return check_ctrl_error();
}

int nemo_gpu_set_interior(int64_t n_interior) {
    if (!g.has_mesh) return fail(NEMO_ERR_STATE, "set the mesh first");
    if (n_interior < 0 || n_interior > g.E_own)
        return fail(NEMO_ERR_ARG, "n_interior must be in [0, %lld]", (long long)g.E_own);
    g.n_interior = n_interior;
    return NEMO_OK;
}

int nemo_gpu_stage_interior(int32_t stage, double dt) {
    int st = ensure_ready();
    if (st) return st;
    if (stage < 1 || stage > 5) return fail(NEMO_ERR_ARG, "stage must be 1..5");
    if (!(dt >= 0.0) || !std::isfinite(dt)) return fail(NEMO_ERR_ARG, "dt must be finite and >= 0");
    if (g.tune_mode == 1) return fail(NEMO_ERR_STATE, "split stages need the grid schedule (nemo_gpu_set_schedule 0)");
    if ((st = prepare_if_needed())) return st;
    CK(cudaMemcpyAsync(&g.nbad_mark, &g.ctrl->nbad, 8, cudaMemcpyDeviceToHost, g.stream));
    CK(launch_ctrl_set_dt(g.ctrl, dt, g.stream));
    // the interior part advances the clock only when there is no boundary part
    CK(launch_stage_part(stage - 1, 0, g.n_interior, g.n_interior == g.E_own, g.stream));
    g.split_open = true;
    return NEMO_OK;
}

int nemo_gpu_stage_boundary(int32_t stage, double dt, int32_t* nbad_out) {
    int st = ensure_ready();
    if (st) return st;
    (void)dt;
    if (!g.split_open) return fail(NEMO_ERR_STATE, "nemo_gpu_stage_interior of this stage first");
    g.split_open = false;
    if (g.E_own > g.n_interior) CK(launch_stage_part(stage - 1, g.n_interior, g.E_own, true, g.stream));
    g.cur ^= 1;
    unsigned long long nb1 = 0;
    CK(cudaMemcpyAsync(&nb1, &g.ctrl->nbad, 8, cudaMemcpyDeviceToHost, g.stream));
    if ((st = check_ctrl_error())) return st;
    if (nbad_out) *nbad_out = (int32_t)(nb1 - g.nbad_mark);
    if (nb1 > g.nbad_mark) return fail(NEMO_ERR_REPAIR, "positivity repair failed on %llu elements", nb1 - g.nbad_mark);
    return NEMO_OK;
}

int nemo_gpu_glm_speeds(double* lmax_out, double* vmax_out) {
    int st = ensure_ready();
    if (st) return st;
    unsigned long long b[2] = {0, 0};
    CK(cudaMemcpyAsync(&b[0], &g.ctrl->lmax_bits[0], 8, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaMemcpyAsync(&b[1], &g.ctrl->vmax_bits, 8, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    if (lmax_out) std::memcpy(lmax_out, &b[0], 8);
    if (vmax_out) std::memcpy(vmax_out, &b[1], 8);
    return NEMO_OK;
}

int nemo_gpu_set_glm(double ch, double alpha) {
    int st = ensure_ready();
    if (st) return st;
    if (!is_mhd()) return fail(NEMO_ERR_STATE, "GLM cleaning needs the MHD equations");
    if (!std::isfinite(ch) || ch < 0.0 || !std::isfinite(alpha) || alpha < 0.0)
        return fail(NEMO_ERR_ARG, "GLM speed and damping must be finite and >= 0");
    const double v[2] = {ch, alpha};
    CK(cudaMemcpyAsync(&g.ctrl->glm_ch, &v[0], 8, cudaMemcpyHostToDevice, g.stream));
    CK(cudaMemcpyAsync(&g.ctrl->glm_alpha, &v[1], 8, cudaMemcpyHostToDevice, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    return NEMO_OK;
}

int nemo_gpu_run_async(int64_t nsteps) {
    int st = ensure_ready();
    if (st) return st;
    if (nsteps <= 0) return fail(NEMO_ERR_ARG, "nsteps must be > 0");
    if (g.timing) return fail(NEMO_ERR_STATE, "timing mode runs synchronously (nemo_gpu_run)");
    g.prepared = false;  // the CFL bound must belong to the current state
    if ((st = prepare_if_needed())) return st;
    // no end time (t_end = 0.0 is all-zero bits), not done
    CK(cudaMemsetAsync(&g.ctrl->t_end, 0, sizeof(double), g.stream));
    CK(cudaMemsetAsync(&g.ctrl->done, 0, sizeof(int32_t), g.stream));
    for (int s = 0; s < 2; ++s)
        if (!g.graph[s] && (st = build_graph(s))) return st;
    for (int64_t i = 0; i < nsteps; ++i) {
        CK(cudaGraphLaunch(g.graph[g.cur], g.stream));
        g.cur ^= 1;
    }
    return NEMO_OK;
}

int nemo_gpu_sync(void) {
    if (!g.inited) return fail(NEMO_ERR_STATE, "nemo_gpu_init has not been called");
    if (g.in_stream) CK(cudaStreamSynchronize(g.in_stream));
    if (g.out_stream) CK(cudaStreamSynchronize(g.out_stream));
    if (g.copy_stream) CK(cudaStreamSynchronize(g.copy_stream));
    CK(cudaStreamSynchronize(g.stream));
    if (g.has_mesh) return check_ctrl_error();
    return NEMO_OK;
}

int nemo_gpu_run(int64_t nsteps, double t_end, double* t_out, int64_t* steps_out) {
    int st = ensure_ready();
    if (st) return st;
    if (nsteps <= 0 && !(t_end > 0.0)) return fail(NEMO_ERR_ARG, "give nsteps > 0 or t_end > 0");
    g.prepared = false;  // the CFL bound must belong to the current state
    if ((st = prepare_if_needed())) return st;
    const int64_t prep_launches = 2;
    CK(cudaMemcpyAsync(&g.ctrl->t_end, &t_end, sizeof(double), cudaMemcpyHostToDevice, g.stream));
    const int32_t zero = 0;
    CK(cudaMemcpyAsync(&g.ctrl->done, &zero, sizeof zero, cudaMemcpyHostToDevice, g.stream));
    unsigned long long steps0 = 0, steps1 = 0;
    CK(cudaMemcpyAsync(&steps0, &g.ctrl->steps, 8, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    const int start_cur = g.cur;
    int64_t issued = 0;
    const int64_t limit = nsteps > 0 ? nsteps : INT64_MAX;
    std::vector<cudaEvent_t> evs;
    if (g.timing) {
        // one event before the first kernel and one after every kernel; read after the run
        const int64_t nk = 6 * (nsteps > 0 ? nsteps : 0);
        if (nk <= 0 || nk > 600000) return fail(NEMO_ERR_ARG, "timing mode needs 0 < nsteps <= 100000");
        evs.resize(nk + 1);
        for (auto& ev : evs) CK(cudaEventCreate(&ev));
        g.t_stage_ms = g.t_total_ms = 0.0;
        g.n_stage = 0;
        g.n_total = prep_launches;  // counted, not timed
        CK(cudaEventRecord(evs[0], g.stream));
        int64_t k = 1;
        for (int64_t i = 0; i < nsteps; ++i) {
            CK(launch_ctrl_step(g.ctrl, g.stream));
            CK(cudaEventRecord(evs[k++], g.stream));
            for (int s = 0; s < 5; ++s) {
                CK(launch_stage(s, g.stream));
                CK(cudaEventRecord(evs[k++], g.stream));
            }
        }
        CK(cudaEventSynchronize(evs[nk]));
        for (int64_t j = 0; j < nk; ++j) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, evs[j], evs[j + 1]));
            g.t_total_ms += ms;
            if (j % 6 != 0) {  // stage kernels; j % 6 == 0 is the control kernel
                g.t_stage_ms += ms;
                g.n_stage += 1;
            }
            g.n_total += 1;
        }
        for (auto& ev : evs) cudaEventDestroy(ev);
        const bool fused = g.tune_mode == 1 && !is_mhd() && g.cfg.precision == NEMO_PREC_FP32;
        if (g.nm > 0 && !fused) g.n_total += 5 * nsteps;  // mortar launches, timed inside their stage interval
        issued = nsteps;
    } else {
        for (int s = 0; s < 2; ++s)
            if (!g.graph[s] && (st = build_graph(s))) return st;
    }
    while (!g.timing && issued < limit) {
        const int64_t chunk = std::min<int64_t>(limit - issued, t_end > 0.0 ? 16 : limit);
        for (int64_t i = 0; i < chunk; ++i) {
            CK(cudaGraphLaunch(g.graph[g.cur], g.stream));
            g.cur ^= 1;
        }
        issued += chunk;
        if (t_end > 0.0) {
            int32_t done = 0;
            CK(cudaMemcpyAsync(&done, &g.ctrl->done, sizeof done, cudaMemcpyDeviceToHost, g.stream));
            CK(cudaStreamSynchronize(g.stream));
            if (done) break;
        }
    }
    CK(cudaMemcpyAsync(&steps1, &g.ctrl->steps, 8, cudaMemcpyDeviceToHost, g.stream));
    double t0 = 0.0;
    CK(cudaMemcpyAsync(&t0, &g.ctrl->t[0], 8, cudaMemcpyDeviceToHost, g.stream));
    if ((st = check_ctrl_error())) return st;
    const int64_t done_steps = (int64_t)(steps1 - steps0);
    g.cur = start_cur ^ (int)(done_steps & 1);
    if (t_out) *t_out = t0;
    if (steps_out) *steps_out = done_steps;
    return NEMO_OK;
}

int nemo_gpu_rhs(double* rhs_host) {
    int st = ensure_ready();
    if (st) return st;
    if (!rhs_host) return fail(NEMO_ERR_ARG, "rhs_host is NULL");
    if ((st = prepare_if_needed())) return st;
    StageArgs a = stage_args(0, true);
    a.rhs_out = g.stagebuf;
    a.alpha_out = nullptr;
    CK(launch_stage_any(a, true, g.stream));
    // rhs is in SoA order in stagebuf: convert to AoS via the second state buffer as scratch
    double* scratch = g.u[g.cur ^ 1];
    CK(launch_soa_to_aos(g.stagebuf, scratch, g.E, g.V, g.stream));
    CK(cudaMemcpyAsync(rhs_host, scratch, sizeof(double) * (size_t)g.V * g.E * NP, cudaMemcpyDeviceToHost, g.stream));
    return check_ctrl_error();
}

int nemo_gpu_alpha(double* alpha_host) {
    int st = ensure_ready();
    if (st) return st;
    if (!alpha_host) return fail(NEMO_ERR_ARG, "alpha_host is NULL");
    if (!blended()) {
        for (int64_t e = 0; e < g.E; ++e) alpha_host[e] = 0.0;
        return NEMO_OK;
    }
    if ((st = prepare_if_needed())) return st;
    // smoothed alpha as the next stage would use it: run a throw-away rhs launch that records it
    StageArgs a = stage_args(0, true);
    a.rhs_out = g.stagebuf;
    a.alpha_out = nullptr;
    CK(launch_stage_any(a, true, g.stream));
    CK(cudaMemcpyAsync(alpha_host, g.alpha_used, sizeof(double) * g.E, cudaMemcpyDeviceToHost, g.stream));
    return check_ctrl_error();
}

int nemo_gpu_totals(double* out) {
    int st = ensure_ready();
    if (st) return st;
    if (!out) return fail(NEMO_ERR_ARG, "out is NULL");
    CK(launch_totals64(g.u[g.cur], g.delta, g.E, g.E_own, g.V, g.part, g.tot, g.stream));
    double tmp[16] = {0};
    CK(cudaMemcpyAsync(tmp, g.tot, sizeof(double) * g.V, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    for (int v = 0; v < 10; ++v) out[v] = v < g.V ? tmp[v] : 0.0;
    return NEMO_OK;
}

int nemo_gpu_status(double* t_out, int64_t* nbad_out) {
    int st = ensure_ready();
    if (st) return st;
    double t = 0;
    unsigned long long nb = 0;
    CK(cudaMemcpyAsync(&t, &g.ctrl->t[0], 8, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaMemcpyAsync(&nb, &g.ctrl->nbad, 8, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    if (t_out) *t_out = t;
    if (nbad_out) *nbad_out = (int64_t)nb;
    return NEMO_OK;
}

int nemo_gpu_autotune(int32_t nsteps, int32_t* mode_out, int32_t* ctas_out, double* ms_out) {
    int st = ensure_ready();
    if (st) return st;
    if (nsteps < 1 || nsteps > 1000) return fail(NEMO_ERR_ARG, "nsteps must be in [1, 1000]");
    if (ms_out)
        for (int i = 0; i < 8; ++i) ms_out[i] = -1.0;
    const bool tunable = !is_mhd() && g.cfg.precision == NEMO_PREC_FP32;
    if (!tunable) {  // the other forms have a single schedule
        g.tune_mode = 0;
        if (mode_out) *mode_out = 0;
        if (ctas_out) *ctas_out = 0;
        return NEMO_OK;
    }
    if ((st = prepare_if_needed())) return st;
    int nsm = 0, dev = 0, occ = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    CK(stage32p_max_ctas_per_sm(blended(), &occ));
    if (occ < 1) return fail(NEMO_ERR_CUDA, "the persistent stage kernel does not fit on an SM");
    // snapshot of everything a step changes: state, register, indicator, control block
    const size_t bytes = sizeof(double) * (size_t)g.V * g.E * NP;
    double* reg_snap = nullptr;
    double* alpha_snap = nullptr;
    CK(cudaMalloc(&reg_snap, bytes));
    CK(cudaMalloc(&alpha_snap, sizeof(double) * g.E));
    Control* csnap = new Control;   // the control block as found
    Control* ctrial = new Control;  // the same without an end time: the trial steps always run
    Control* cnow = new Control;
    auto cleanup = [&]() {
        cudaFree(reg_snap);
        cudaFree(alpha_snap);
        delete csnap;
        delete ctrial;
        delete cnow;
    };
    const int cur0 = g.cur;
    const bool regv = g.reg_valid;
    auto save_or_restore = [&](bool save, Control* src) -> cudaError_t {
        cudaError_t e;
        if (save) {
            if ((e = cudaMemcpyAsync(g.stagebuf, g.u[cur0], bytes, cudaMemcpyDeviceToDevice, g.stream))) return e;
            if ((e = cudaMemcpyAsync(reg_snap, g.reg, bytes, cudaMemcpyDeviceToDevice, g.stream))) return e;
            if ((e = cudaMemcpyAsync(alpha_snap, g.alpha[cur0], sizeof(double) * g.E, cudaMemcpyDeviceToDevice, g.stream))) return e;
            if ((e = cudaMemcpyAsync(csnap, g.ctrl, sizeof(Control), cudaMemcpyDeviceToHost, g.stream))) return e;
            if ((e = cudaStreamSynchronize(g.stream))) return e;
            *ctrial = *csnap;
            ctrial->t_end = 0.0;
            ctrial->done = 0;
            return cudaSuccess;
        }
        // keep the epoch monotonic: mortar flags may carry the epochs of the trial launches
        if ((e = cudaMemcpyAsync(cnow, g.ctrl, sizeof(Control), cudaMemcpyDeviceToHost, g.stream))) return e;
        if ((e = cudaStreamSynchronize(g.stream))) return e;
        src->epoch = cnow->epoch;
        src->work = 0u;
        src->exit_count = 0u;
        if ((e = cudaMemcpyAsync(g.u[cur0], g.stagebuf, bytes, cudaMemcpyDeviceToDevice, g.stream))) return e;
        if ((e = cudaMemcpyAsync(g.reg, reg_snap, bytes, cudaMemcpyDeviceToDevice, g.stream))) return e;
        if ((e = cudaMemcpyAsync(g.alpha[cur0], alpha_snap, sizeof(double) * g.E, cudaMemcpyDeviceToDevice, g.stream))) return e;
        if ((e = cudaMemcpyAsync(g.ctrl, src, sizeof(Control), cudaMemcpyHostToDevice, g.stream))) return e;
        if ((e = cudaStreamSynchronize(g.stream))) return e;
        g.cur = cur0;
        g.reg_valid = regv;
        return cudaSuccess;
    };
    cudaError_t e = save_or_restore(true, nullptr);
    if (e == cudaSuccess) e = save_or_restore(false, ctrial);
    double best = 1e300;
    int best_mode = 0, best_ctas = 0;
    // candidates (mode, CTAs, slot of ms_out): the grid schedule at 8, 4 and 16 elements per CTA, the
    // persistent kernel at 1..4 CTAs per SM (as many as fit)
    struct Cand { int mode, ctas, slot; };
    Cand cand[8];
    int ncand = 0;
    cand[ncand++] = {0, 0, 0};
    for (int c = 1; c <= std::min(occ, 4); ++c) cand[ncand++] = {1, nsm * c, c};
    cand[ncand++] = {2, 0, 5};
    cand[ncand++] = {3, 0, 6};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    for (int ci = 0; ci < ncand && e == cudaSuccess; ++ci) {
        g.tune_mode = cand[ci].mode;
        g.tune_ctas = cand[ci].ctas;
        const int c = cand[ci].slot;
        // one untimed step (first-launch costs), then nsteps timed steps, from the same state
        for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {
            const int n = rep == 0 ? 1 : nsteps;
            if ((e = cudaEventRecord(e0, g.stream))) break;
            for (int i = 0; i < n && e == cudaSuccess; ++i) {
                e = launch_ctrl_step(g.ctrl, g.stream);
                for (int s2 = 0; s2 < 5 && e == cudaSuccess; ++s2) e = launch_stage(s2, g.stream);
            }
            if (e == cudaSuccess) e = cudaEventRecord(e1, g.stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            if (e == cudaSuccess && rep == 1) {
                float ms = 0.f;
                e = cudaEventElapsedTime(&ms, e0, e1);
                const double per = ms / nsteps;
                if (ms_out) ms_out[c] = per;
                if (per < best) {
                    best = per;
                    best_mode = g.tune_mode;
                    best_ctas = g.tune_ctas;
                }
            }
            if (e == cudaSuccess) e = save_or_restore(false, ctrial);
        }
    }
    if (e == cudaSuccess) e = save_or_restore(false, csnap);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cleanup();
    if (e != cudaSuccess) {
        g.tune_mode = 0;
        return fail(NEMO_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
    }
    if ((st = check_ctrl_error())) return st;
    g.tune_mode = best_mode;
    g.tune_ctas = best_ctas;
    release_graphs();   // rebuilt with the chosen schedule
    if (mode_out) *mode_out = best_mode;
    if (ctas_out) *ctas_out = best_ctas;
    return NEMO_OK;
}

int nemo_gpu_set_schedule(int32_t mode, int32_t ctas) {
    if (!g.inited) return fail(NEMO_ERR_STATE, "nemo_gpu_init has not been called");
    if (mode < 0 || mode > 3)
        return fail(NEMO_ERR_ARG, "mode must be 0 (grid, 8 elements per CTA), 1 (persistent), 2 (grid, 4) or 3 (grid, 16)");
    if (mode == 1) {
        int nsm = 0, dev = 0, occ = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        CK(stage32p_max_ctas_per_sm(blended(), &occ));
        if (ctas < 1 || ctas > nsm * occ)
            return fail(NEMO_ERR_ARG, "persistent CTAs must be in [1, %d] (SMs x resident CTAs)", nsm * occ);
    }
    g.tune_mode = mode;
    g.tune_ctas = mode == 1 ? ctas : 0;
    release_graphs();
    return NEMO_OK;
}

int nemo_gpu_set_timing(int32_t on) {
    g.timing = on != 0;
    return NEMO_OK;
}

int nemo_gpu_kernel_timing(double* stage_ms, int64_t* stage_launches, double* total_ms, int64_t* total_launches) {
    if (stage_ms) *stage_ms = g.t_stage_ms;
    if (stage_launches) *stage_launches = g.n_stage;
    if (total_ms) *total_ms = g.t_total_ms;
    if (total_launches) *total_launches = g.n_total;
    return NEMO_OK;
}

int nemo_gpu_stream(uint64_t* out) {
    if (!g.inited) return fail(NEMO_ERR_STATE, "nemo_gpu_init has not been called");
    if (out) *out = (uint64_t)(uintptr_t)g.stream;
    return NEMO_OK;
}

int nemo_gpu_set_mlp(const float* weights, int32_t nweights, const float* lo, const float* hi) {
    if (!g.inited) return fail(NEMO_ERR_STATE, "nemo_gpu_init has not been called");
    if (!weights || !lo || !hi) return fail(NEMO_ERR_ARG, "NULL weights or bounds");
    if (nweights != MLP_NW) return fail(NEMO_ERR_ARG, "the indicator MLP has %d weights (got %d)", MLP_NW, nweights);
    std::vector<float> w32(MLP_NPACK);
    std::vector<double> w64(MLP_NPACK);
    for (int i = 0; i < MLP_NW; ++i) {
        // round to BF16 (nearest, ties to even): the network is stored and evaluated from BF16 weights
        uint32_t b;
        std::memcpy(&b, &weights[i], 4);
        if ((b & 0x7f800000u) != 0x7f800000u) b = (b + 0x7fffu + ((b >> 16) & 1u)) & 0xffff0000u;
        else b &= 0xffff0000u;
        float r;
        std::memcpy(&r, &b, 4);
        w32[i] = r;
        w64[i] = (double)r;
    }
    for (int i = 0; i < 12; ++i) {
        w32[MLP_NW + i] = lo[i];
        w32[MLP_NW + 12 + i] = hi[i];
        w64[MLP_NW + i] = (double)lo[i];
        w64[MLP_NW + 12 + i] = (double)hi[i];
    }
    // transposed copy for the FP32 stage: W1T[i][j] = W1[j][i], W2T[i][j] = W2[j][i]
    std::vector<float> wt(MLP_NT, 0.0f);
    for (int i = 0; i < MLP_NW; ++i) {
        float v;
        if (i < 12 * 32) v = w32[(i % 32) * 12 + i / 32];
        else if (i < 12 * 32 + 32) v = w32[i];
        else if (i < 12 * 32 + 32 + 32 * 32) {
            const int r = i - (12 * 32 + 32);
            v = w32[12 * 32 + 32 + (r % 32) * 32 + r / 32];
        } else v = w32[i];
        wt[i] = v;
    }
    for (int i = MLP_NW; i < MLP_NPACK; ++i) wt[i] = w32[i];   // input bounds
    CK(cudaMemcpy(g.mlp32, w32.data(), sizeof(float) * MLP_NPACK, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(g.mlp32 + mlp_t_offset(), wt.data(), sizeof(float) * MLP_NT, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(g.mlp64, w64.data(), sizeof(double) * MLP_NPACK, cudaMemcpyHostToDevice));
    g.mlp_ready = true;
    release_graphs();
    g.prepared = false;
    return NEMO_OK;
}

int nemo_gpu_features(float* feat_host, double* alpha_modal_host) {
    int st = ensure_ready();
    if (st) return st;
    if (!feat_host) return fail(NEMO_ERR_ARG, "feat_host is NULL");
    if (!g.feat_dev) CK(cudaMalloc(&g.feat_dev, sizeof(float) * 12 * g.E));
    double* am = g.part;  // [E] scratch (the totals partials are not live here)
    CK(launch_ctrl_reset(g.ctrl, g.stream));
    CK(launch_prepare(false, g.stream, g.feat_dev, am));
    CK(cudaMemcpyAsync(feat_host, g.feat_dev, sizeof(float) * 12 * g.E, cudaMemcpyDeviceToHost, g.stream));
    if (alpha_modal_host) CK(cudaMemcpyAsync(alpha_modal_host, am, sizeof(double) * g.E, cudaMemcpyDeviceToHost, g.stream));
    g.prepared = false;
    return check_ctrl_error();
}

int nemo_gpu_indicator_stats(int64_t* fallback_out, int64_t* judged_out, double* judge_mae_out) {
    int st = ensure_ready();
    if (st) return st;
    unsigned long long fb = 0, jn = 0;
    double js = 0.0;
    CK(cudaMemcpyAsync(&fb, &g.ctrl->fallback, 8, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaMemcpyAsync(&jn, &g.ctrl->judge_n, 8, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaMemcpyAsync(&js, &g.ctrl->judge_sum, 8, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    if (fallback_out) *fallback_out = (int64_t)fb;
    if (judged_out) *judged_out = (int64_t)jn;
    if (judge_mae_out) *judge_mae_out = jn ? js / (double)jn : 0.0;
    return NEMO_OK;
}

// ---- training (independent of init: own buffers, default stream) -------------------------------

namespace {
struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};
}  // namespace

int nemo_gpu_mlp_grad(const float* feat, const float* target, int64_t nsamp, const float* weights, float amax,
                      float* loss_out, float* grad_out) {
    if (!feat || !target || !weights || nsamp <= 0) return fail(NEMO_ERR_ARG, "bad training arguments");
    DevBuf f, t, w, gr, l;
    CK(cudaMalloc(&f.p, sizeof(float) * 12 * nsamp));
    CK(cudaMalloc(&t.p, sizeof(float) * nsamp));
    CK(cudaMalloc(&w.p, sizeof(float) * MLP_NW));
    CK(cudaMalloc(&gr.p, sizeof(float) * MLP_NW));
    CK(cudaMalloc(&l.p, sizeof(float)));
    CK(cudaMemcpy(f.p, feat, sizeof(float) * 12 * nsamp, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(t.p, target, sizeof(float) * nsamp, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(w.p, weights, sizeof(float) * MLP_NW, cudaMemcpyHostToDevice));
    CK(cudaMemset(gr.p, 0, sizeof(float) * MLP_NW));
    CK(cudaMemset(l.p, 0, sizeof(float)));
    CK(mlp_grad_launch((const float*)f.p, (const float*)t.p, nullptr, nsamp, (const float*)w.p, amax, (float*)gr.p,
                       (float*)l.p, 0));
    CK(cudaDeviceSynchronize());
    if (loss_out) CK(cudaMemcpy(loss_out, l.p, sizeof(float), cudaMemcpyDeviceToHost));
    if (grad_out) CK(cudaMemcpy(grad_out, gr.p, sizeof(float) * MLP_NW, cudaMemcpyDeviceToHost));
    return NEMO_OK;
}

int nemo_gpu_mlp_forward(const float* feat, int64_t nsamp, const float* weights, float amax, float* alpha_out) {
    if (!feat || !weights || !alpha_out || nsamp <= 0) return fail(NEMO_ERR_ARG, "bad forward arguments");
    DevBuf f, w, o;
    CK(cudaMalloc(&f.p, sizeof(float) * 12 * nsamp));
    CK(cudaMalloc(&w.p, sizeof(float) * MLP_NW));
    CK(cudaMalloc(&o.p, sizeof(float) * nsamp));
    CK(cudaMemcpy(f.p, feat, sizeof(float) * 12 * nsamp, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(w.p, weights, sizeof(float) * MLP_NW, cudaMemcpyHostToDevice));
    CK(mlp_forward_launch((const float*)f.p, nsamp, (const float*)w.p, amax, (float*)o.p, 0));
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(alpha_out, o.p, sizeof(float) * nsamp, cudaMemcpyDeviceToHost));
    return NEMO_OK;
}

int nemo_gpu_mlp_train(const float* feat, const float* target, int64_t nsamp, float* weights, float amax,
                       int32_t epochs, int32_t batch, float lr, uint64_t seed, float* loss_out) {
    if (!feat || !target || !weights || nsamp <= 0 || epochs <= 0 || batch <= 0 || !(lr > 0.f))
        return fail(NEMO_ERR_ARG, "bad training arguments");
    if (nsamp > INT32_MAX) return fail(NEMO_ERR_ARG, "at most 2^31-1 samples");
    DevBuf f, t, w, gr, m, v, l, ix;
    CK(cudaMalloc(&f.p, sizeof(float) * 12 * nsamp));
    CK(cudaMalloc(&t.p, sizeof(float) * nsamp));
    CK(cudaMalloc(&w.p, sizeof(float) * MLP_NW));
    CK(cudaMalloc(&gr.p, sizeof(float) * MLP_NW));
    CK(cudaMalloc(&m.p, sizeof(float) * MLP_NW));
    CK(cudaMalloc(&v.p, sizeof(float) * MLP_NW));
    CK(cudaMalloc(&l.p, sizeof(float)));
    CK(cudaMalloc(&ix.p, sizeof(int32_t) * nsamp));
    CK(cudaMemcpy(f.p, feat, sizeof(float) * 12 * nsamp, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(t.p, target, sizeof(float) * nsamp, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(w.p, weights, sizeof(float) * MLP_NW, cudaMemcpyHostToDevice));
    CK(cudaMemset(m.p, 0, sizeof(float) * MLP_NW));
    CK(cudaMemset(v.p, 0, sizeof(float) * MLP_NW));
    std::vector<int32_t> perm(nsamp);
    for (int64_t i = 0; i < nsamp; ++i) perm[i] = (int32_t)i;
    uint64_t state = seed ? seed : 0x9E3779B97F4A7C15ull;
    int step = 0;
    for (int ep = 0; ep < epochs; ++ep) {
        for (int64_t i = nsamp - 1; i > 0; --i) {  // Fisher-Yates with a splitmix64 stream
            state += 0x9E3779B97F4A7C15ull;
            uint64_t z = state;
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            z ^= z >> 31;
            const int64_t j = (int64_t)(z % (uint64_t)(i + 1));
            std::swap(perm[i], perm[j]);
        }
        CK(cudaMemcpy(ix.p, perm.data(), sizeof(int32_t) * nsamp, cudaMemcpyHostToDevice));
        CK(cudaMemset(l.p, 0, sizeof(float)));
        int64_t nb = 0;
        for (int64_t b0 = 0; b0 < nsamp; b0 += batch) {
            const int64_t nbat = std::min<int64_t>(batch, nsamp - b0);
            CK(cudaMemsetAsync(gr.p, 0, sizeof(float) * MLP_NW, 0));
            CK(mlp_grad_launch((const float*)f.p, (const float*)t.p, (const int32_t*)ix.p + b0, nbat,
                               (const float*)w.p, amax, (float*)gr.p, (float*)l.p, 0));
            CK(mlp_adam_launch((float*)w.p, (const float*)gr.p, (float*)m.p, (float*)v.p, ++step, lr, 0));
            ++nb;
        }
        float ls = 0.f;
        CK(cudaMemcpy(&ls, l.p, sizeof(float), cudaMemcpyDeviceToHost));
        if (loss_out) loss_out[ep] = ls / (float)nb;
    }
    CK(cudaMemcpy(weights, w.p, sizeof(float) * MLP_NW, cudaMemcpyDeviceToHost));
    return NEMO_OK;
}

int nemo_gpu_finalize(void) {
    if (!g.inited) return NEMO_OK;
    cudaStreamSynchronize(g.stream);
    release_mesh();
    free_dev(g.ctrl);
    free_dev(g.tot);
    free_dev(g.mlp32);
    free_dev(g.mlp64);
    free_dev(g.ckpt_meta);
    if (g.ckpt_meta_host) cudaFreeHost(g.ckpt_meta_host);
    if (g.ckpt_ready) cudaEventDestroy(g.ckpt_ready);
    if (g.ckpt_done) cudaEventDestroy(g.ckpt_done);
    if (g.copy_stream) cudaStreamDestroy(g.copy_stream);
    g.ckpt_meta = g.ckpt_meta_host = nullptr;
    g.ckpt_ready = g.ckpt_done = nullptr;
    g.copy_stream = nullptr;
    for (int i = 0; i < 2; ++i) {   // release_mesh released the staging slots
        if (g.in_done[i]) cudaEventDestroy(g.in_done[i]);
        if (g.in_free[i]) cudaEventDestroy(g.in_free[i]);
        g.in_done[i] = g.in_free[i] = nullptr;
    }
    if (g.in_ctrl) cudaFreeHost(g.in_ctrl);
    if (g.in_stream) cudaStreamDestroy(g.in_stream);
    g.in_ctrl = nullptr;
    g.in_stream = nullptr;
    g.in_next = 0;
    for (int i = 0; i < 2; ++i) {   // release_mesh released the staging slots
        if (g.out_ready[i]) cudaEventDestroy(g.out_ready[i]);
        if (g.out_done[i]) cudaEventDestroy(g.out_done[i]);
        g.out_ready[i] = g.out_done[i] = nullptr;
    }
    if (g.out_stream) cudaStreamDestroy(g.out_stream);
    g.out_stream = nullptr;
    g.out_next = 0;
    g.ctrl = nullptr;
    g.tot = nullptr;
    g.mlp32 = nullptr;
    g.mlp64 = nullptr;
    g.mlp_ready = false;
    cudaStreamDestroy(g.stream);
    g.stream = nullptr;
    g.inited = false;
    return NEMO_OK;
}

int nemo_gpu_last_error(char* buf, int32_t len) {
    if (!buf || len <= 0) return NEMO_ERR_ARG;
    std::snprintf(buf, (size_t)len, "%s", g.err);
    return NEMO_OK;
}

}  // extern "C"
