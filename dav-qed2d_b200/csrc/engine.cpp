// engine.cpp -- the C ABI of libqed2d (include/qed2d.h): context and workspace,
// argument checks, the reference's operators, observables, solvers, RHMC
// helpers, integrators and HMC steps, built from the kernel launchers in
// kernels.cu and the solvers in cg.cu.  Work is enqueued asynchronously on the
// context stream; the host synchronises only where a host scalar is returned
// (observables, iteration counts, the Metropolis decision).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "graph.h"
#include "internal.h"

struct qed2d_ctx {
    qed2d::Ctx c;
};

namespace qed2d {

// ---------------------------------------------------------------------------
// errors
static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
int cuda_status(cudaError_t e, const char* what) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return QED2D_ERR_CUDA;
}
static int bad_arg(const std::string& msg) {
    set_error(msg);
    return QED2D_ERR_BAD_ARG;
}

void* Ctx::buf(const std::string& name, size_t bytes) {
    auto it = ws.find(name);
    if (it != ws.end() && it->second.second >= bytes) return it->second.first;
    if (it != ws.end()) {
        cudaStreamSynchronize(stream);
        cudaFree(it->second.first);
        ws.erase(it);
        ws_gen++;   // a captured graph holding the old address is stale
    }
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_error("workspace allocation of " + std::to_string(bytes) + " bytes failed (" + name + ")");
        return nullptr;
    }
    ws[name] = {p, bytes};
    return p;
}

// ---------------------------------------------------------------------------
// helpers
static inline double2* C2(double* p) { return reinterpret_cast<double2*>(p); }
static inline const double2* C2(const double* p) { return reinterpret_cast<const double2*>(p); }
static inline size_t field_bytes(const Ctx& c) { return sizeof(double2) * 2 * (size_t)c.g.V; }
static inline size_t real_bytes(const Ctx& c) { return sizeof(double) * 2 * (size_t)c.g.V; }

static int check_ptr(const void* p, const char* name) {
    if (!p) return bad_arg(std::string(name) + " is NULL");
    if (reinterpret_cast<uintptr_t>(p) % 16 != 0) return bad_arg(std::string(name) + " is not 16-byte aligned");
    return QED2D_OK;
}
static bool overlap(const void* a, size_t na, const void* b, size_t nb) {
    const char *pa = (const char*)a, *pb = (const char*)b;
    return pa < pb + nb && pb < pa + na;
}
static int check_out(const Ctx& c, const void* out, const void* in, const char* what) {
    if (overlap(out, field_bytes(c), in, field_bytes(c)))
        return bad_arg(std::string(what) + ": output aliases an input (stencil operators run out of place)");
    return QED2D_OK;
}
#define QCTX(ctx)                                                 \
    if (!(ctx)) return ::qed2d::bad_arg("context is NULL");      \
    ::qed2d::Ctx& c = (ctx)->c;                                   \
    (void)c
#define QPTR(p) QTRY(::qed2d::check_ptr((p), #p))

static int fetch_scal(Ctx& c, int slot, int n, double* out) {
    QCHECK(cudaMemcpyAsync(out, &c.ctl->scal[slot], sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream));
    QCHECK(cudaStreamSynchronize(c.stream));
    return QED2D_OK;
}
static int reset_seq(Ctx& c) {
    QCHECK(cudaMemsetAsync(&c.ctl->status, 0, sizeof(int), c.stream));
    QCHECK(cudaMemsetAsync(&c.ctl->iters_total, 0, sizeof(long long), c.stream));
    return QED2D_OK;
}
static int finish_seq(Ctx& c, int64_t* iters_acc) {
    const int st = read_ctl(c, false);
    if (iters_acc) *iters_acc += c.ctl_host->iters_total;
    if (st != QED2D_OK && g_last_error.empty()) set_error(qed2d_status_string(st));
    return st;
}

static int op_sqr(Ctx& c, double2* so, const double2* U, const double2* si, double am0, double mu) {
    double2* tmp = c.spinor("op_tmp");
    if (!tmp) return QED2D_ERR_NO_MEMORY;
    QTRY(launch_g5dw(c, tmp, U, si, am0, nullptr, make_double2(0, 0), false));
    return launch_g5dw(c, so, U, tmp, am0, mu != 0.0 ? si : nullptr, make_double2(mu * mu, 0), false);
}

static int solve(Ctx& c, double2* x, const double2* U, const double2* b, double am0, double mu, int maxiter,
                 double eps, bool guess, double2* g5x, const float4* U32 = nullptr) {
    SolveArgs a;
    a.U = U;
    a.U32 = U32;
    a.b = b;
    a.x = x;
    a.am0 = am0;
    a.mu2 = mu * mu;
    a.maxiter = maxiter;
    a.eps = eps;
    a.guess = guess;
    a.g5x = g5x;
    return cg_solve(c, a, c.precision);
}

// ---------------------------------------------------------------------------
// RHMC building blocks (no host synchronisation)
static int multi_cg_core(Ctx& c, double2* so, const double2* U, const double2* si, double am0, int maxiter,
                         double eps, const qed2d_rhmc_params* r, bool apply_R) {
    const int n = r->n;
    const long long N = 2 * c.g.V;
    std::vector<double2*> xs(n);
    std::vector<double> mu2(n);
    for (int i = 0; i < n; i++) {
        xs[i] = c.spinor("mcg_x_" + std::to_string(i));
        if (!xs[i]) return QED2D_ERR_NO_MEMORY;
        mu2[i] = r->mu[i] * r->mu[i];
    }
    if (c.precision == QED2D_PREC_PLAIN) {
        for (int i = 0; i < n; i++) QTRY(solve(c, xs[i], U, si, am0, r->mu[i], maxiter, eps, false, nullptr));
    } else {
        QTRY(multishift_solve(c, U, si, xs.data(), mu2.data(), n, am0, maxiter, eps));
    }
    // so = si + sum rho_j x_j   (MultiCG, src/QED2dRHMC.jl:283-287)
    QTRY(launch_copy(c, so, si, sizeof(double2) * N));
    for (int i = 0; i < n; i++)
        QTRY(launch_zaxpby(c, so, make_double2(1, 0), so, make_double2(r->rho[i], 0), xs[i], N));
    if (apply_R) {   // R: so = r_b^-1 A so   (src/QED2dRHMC.jl:268)
        const double s = std::pow(r->r_b, -1.0) * r->A;
        QTRY(launch_zaxpby(c, so, make_double2(s, 0), so, make_double2(0, 0), nullptr, N));
    }
    return QED2D_OK;
}

static int pf_generate_core(Ctx& c, double2* F, const double2* U, const double2* X, double am0, int maxiter,
                            double tol, const qed2d_rhmc_params* r) {
    const long long N = 2 * c.g.V;
    double2* aux = c.spinor("pf_aux");
    if (!aux) return QED2D_ERR_NO_MEMORY;
    QTRY(launch_copy(c, F, X, sizeof(double2) * N));
    for (int i = 0; i < r->n; i++) {
        // F = g5Dw F + i mu F ; F = (A + nu^2)^-1 F ; F = g5Dw F - i nu F  (src/QED2dRHMC.jl:302-318)
        QTRY(launch_copy(c, aux, F, sizeof(double2) * N));
        QTRY(launch_g5dw(c, F, U, aux, am0, aux, make_double2(0, r->mu[i]), false));
        QTRY(launch_copy(c, aux, F, sizeof(double2) * N));
        QTRY(solve(c, F, U, aux, am0, r->nu[i], maxiter, tol, false, nullptr));
        QTRY(launch_copy(c, aux, F, sizeof(double2) * N));
        QTRY(launch_g5dw(c, F, U, aux, am0, aux, make_double2(0, -r->nu[i]), false));
    }
    return QED2D_OK;
}

static int luscher_z_core(Ctx& c, double2* Z, const double2* U, const double2* Xin, double am0, int maxiter,
                          double tol, const qed2d_rhmc_params* r) {
    const long long N = 2 * c.g.V;
    double2* tmp = c.spinor("lz_tmp");
    double2* tmp2 = c.spinor("lz_tmp2");
    if (!tmp || !tmp2) return QED2D_ERR_NO_MEMORY;
    QTRY(multi_cg_core(c, tmp, U, Xin, am0, maxiter, tol, r, true));
    QTRY(multi_cg_core(c, tmp2, U, tmp, am0, maxiter, tol, r, true));
    QTRY(launch_g5dw(c, tmp, U, tmp2, am0, nullptr, make_double2(0, 0), false));
    // Z = g5Dw tmp - Xin   (src/QED2dRHMC.jl:180-184)
    return launch_g5dw(c, Z, U, tmp, am0, Xin, make_double2(-1, 0), false);
}

// ---------------------------------------------------------------------------
// molecular dynamics (no host synchronisation; status collected in ctl)
static constexpr double R1 = 0.08398315262876693, R2 = 0.2539785108410595, R3 = 0.6822365335719091,
                        R4 = -0.03230286765269967;   // src/QED2dHMC.jl:241-246

struct MDState {
    float4* U32 = nullptr;   // FP32 copy of U maintained for the mixed solver
};

static int md_prepare(Ctx& c, const double2* U, MDState& s) {
    if (c.precision == QED2D_PREC_MIXED) {
        s.U32 = c.spinor32("md_u32");
        if (!s.U32) return QED2D_ERR_NO_MEMORY;
        QTRY(launch_pack_links(c, s.U32, U));
    }
    return QED2D_OK;
}

static int md_links(Ctx& c, double2* U, const double* mom, double eps, MDState& s) {
    return launch_updt_fld(c, U, mom, eps, s.U32);
}

static int md_kick_gauge(Ctx& c, double* mom, const double2* U, double eps) {
    return launch_mom_kick(c, mom, U, eps, nullptr, nullptr, nullptr);
}

// update_momenta! Nf=2 (src/QED2dHMC.jl:452-481): X = ((g5Dw)^2)^-1 F with g5Dw X
// produced by the solver's last phase, then one fused kick with both forces
static int md_kick_nf2(Ctx& c, double* mom, const double2* U, double2* X, const double2* F, double2* g5DX,
                       double am0, double eps, int maxiter, double tol, MDState& s) {
    QTRY(solve(c, X, U, F, am0, 0.0, maxiter, tol, false, g5DX, s.U32));
    return launch_mom_kick(c, mom, U, eps, X, g5DX, nullptr);
}

// update_momenta! RHMC (src/QED2dHMC.jl:516-557): all poles of a flavour in one
// multi-shift solve; force = sum_j sum_i rho_i tr_dQwdU(X_i)
static int md_kick_rhmc(Ctx& c, double* mom, const double2* U, double2* X, const double* const* F, double2* g5DX,
                        int nf, const double* am0, double eps, int maxiter, double tol, const qed2d_rhmc_params* r) {
    double* frc = c.real2("rhmc_frc");
    if (!frc) return QED2D_ERR_NO_MEMORY;
    bool first = true;
    for (int j = 0; j < nf; j++) {
        const int n = r[j].n;
        std::vector<double2*> xs(n);
        std::vector<double> mu2(n);
        for (int i = 0; i < n; i++) {
            xs[i] = c.spinor("mcg_x_" + std::to_string(i));
            if (!xs[i]) return QED2D_ERR_NO_MEMORY;
            mu2[i] = r[j].mu[i] * r[j].mu[i];
        }
        if (c.precision == QED2D_PREC_PLAIN) {
            // the reference's sequence: warm start from the previous pole's solution
            for (int i = 0; i < n; i++) {
                if (i > 0) QTRY(launch_copy(c, xs[i], xs[i - 1], field_bytes(c)));
                QTRY(solve(c, xs[i], U, C2(F[j]), am0[j], r[j].mu[i], maxiter, tol, i > 0, nullptr));
            }
        } else {
            QTRY(multishift_solve(c, U, C2(F[j]), xs.data(), mu2.data(), n, am0[j], maxiter, tol));
        }
        if (c.precision == QED2D_PREC_PLAIN) {   // the reference's sequence: two launches per pole
            for (int i = 0; i < n; i++) {
                QTRY(launch_g5dw(c, g5DX, U, xs[i], am0[j], nullptr, make_double2(0, 0), false));
                QTRY(launch_force_accum(c, frc, U, xs[i], g5DX, r[j].rho[i], !first));
                first = false;
            }
        } else if (n > 0) {   // all poles in two launches
            std::vector<double2*> gs(n);
            for (int i = 0; i < n; i++) {
                gs[i] = c.spinor("mcg_g_" + std::to_string(i));
                if (!gs[i]) return QED2D_ERR_NO_MEMORY;
            }
            QTRY(launch_force_poles(c, frc, U, xs.data(), gs.data(), r[j].rho, n, am0[j], !first));
            first = false;
            if (j == nf - 1) QTRY(launch_copy(c, g5DX, gs[n - 1], field_bytes(c)));   // g5Dw X of the last pole
        }
        if (j == nf - 1 && n > 0) QTRY(launch_copy(c, X, xs[n - 1], field_bytes(c)));
    }
    return launch_mom_kick(c, mom, U, eps, nullptr, nullptr, first ? nullptr : frc);
}

// Pure-gauge MD whose link updates are each followed by a kick: every such pair
// runs as one k_updt_kick pass that reads one (links, momenta) buffer pair and
// writes the other (the caller's arrays and a workspace pair, alternating), the
// other kicks in place on the current pair; the caller's arrays hold the result
// at the end (one copy when the pass count is odd).  Same operations in the same
// order as separate updates and kicks; the compiler contracts them into FMAs
// differently in the fused kernel, so results agree to rounding (1e-14 on links
// after OMF4 trajectories), not bit for bit.  Lattices of whole 32 x 8 tiles
// (kernel requirement) without an FP32 link copy to refresh.  Measured per
// OMF4 step: up to 256^2 44.5 -> 34.9 us (fewer launches), 512^2 67.1 -> 49.5,
// 2048^2 555 -> 516, 4096^2 2082 -> 1942, 8192^2 8274 -> 8179; but 1024^2
// 112.8 -> 143.4 us, where the separate kernels' links and momenta (48 B/site)
// stay in the 126 MB L2 and the two buffer pairs (96 B/site) do not -- so not
// for 2^19 < V <= 2^21 sites.
struct GaugePingPong {
    Ctx& c;
    double2* U[2];
    double* mom[2];
    int cur = 0;
    bool on = false;
    GaugePingPong(Ctx& c_, double2* U0, double* m0, const MDState& s) : c(c_) {
        U[0] = U0;
        mom[0] = m0;
        U[1] = nullptr;
        mom[1] = nullptr;
        if (s.U32 || !updt_kick_fits(c) || (c.g.V > (1LL << 19) && c.g.V <= (1LL << 21))) return;
        U[1] = c.spinor("md_u_alt");
        mom[1] = c.real2("md_mom_alt");
        on = U[1] && mom[1];
    }
    int kick(double eps) { return md_kick_gauge(c, mom[cur], U[cur], eps); }
    int links_then_kick(double eu, double ek, MDState& s) {
        if (!on) {
            QTRY(md_links(c, U[cur], mom[cur], eu, s));
            return md_kick_gauge(c, mom[cur], U[cur], ek);
        }
        QTRY(launch_updt_kick(c, U[cur ^ 1], U[cur], mom[cur ^ 1], mom[cur], eu, ek));
        cur ^= 1;
        return QED2D_OK;
    }
    int finish() {   // the result into the caller's arrays
        if (cur == 0) return QED2D_OK;
        QTRY(launch_copy(c, U[0], U[1], field_bytes(c)));
        QTRY(launch_copy(c, mom[0], mom[1], sizeof(double) * 2 * (size_t)c.g.V));
        cur = 0;
        return QED2D_OK;
    }
};

static int md_omf4_gauge(Ctx& c, double* mom, double2* U, double eps, int ns, MDState& s) {
    const double r5 = 0.5 - R1 - R3, r6 = 1.0 - 2.0 * (R2 + R4);
    const double cm[6] = {R1, R3, r5, r5, R3, R1};
    const double cu[5] = {R2, R4, r6, R4, R2};
    GaugePingPong pp(c, U, mom, s);
    for (int i = 0; i < ns; i++) {
        QTRY(pp.kick(cm[0] * eps));
        for (int k = 0; k < 5; k++) QTRY(pp.links_then_kick(eps * cu[k], cm[k + 1] * eps, s));
    }
    return pp.finish();
}

static int md_leapfrog_gauge(Ctx& c, double* mom, double2* U, double eps, int ns, MDState& s) {
    GaugePingPong pp(c, U, mom, s);
    QTRY(pp.kick(0.5 * eps));
    for (int i = 0; i < ns - 1; i++) QTRY(pp.links_then_kick(eps, eps, s));
    QTRY(pp.links_then_kick(eps, 0.5 * eps, s));
    return pp.finish();
}

static int md_leapfrog_nf2(Ctx& c, double* mom, double2* U, double2* X, const double2* F, double2* g5DX,
                           double am0, double eps, int ns, int maxiter, double tol, MDState& s) {
    QTRY(md_kick_nf2(c, mom, U, X, F, g5DX, am0, 0.5 * eps, maxiter, tol, s));
    for (int i = 0; i < ns - 1; i++) {
        QTRY(md_links(c, U, mom, eps, s));
        QTRY(md_kick_nf2(c, mom, U, X, F, g5DX, am0, eps, maxiter, tol, s));
    }
    QTRY(md_links(c, U, mom, eps, s));
    return md_kick_nf2(c, mom, U, X, F, g5DX, am0, 0.5 * eps, maxiter, tol, s);
}

static int md_omf4_nf2(Ctx& c, double* mom, double2* U, double2* X, const double2* F, double2* g5DX, double am0,
                       double eps, int ns, int maxiter, double tol, MDState& s) {
    const double r5 = 0.5 - R1 - R3, r6 = 1.0 - 2.0 * (R2 + R4);
    const double cm[6] = {R1, R3, r5, r5, R3, R1};
    const double cu[5] = {R2, R4, r6, R4, R2};
    for (int i = 0; i < ns; i++)
        for (int k = 0; k < 6; k++) {
            QTRY(md_kick_nf2(c, mom, U, X, F, g5DX, am0, cm[k] * eps, maxiter, tol, s));
            if (k < 5) QTRY(md_links(c, U, mom, eps * cu[k], s));
        }
    return QED2D_OK;
}

static int md_leapfrog_rhmc(Ctx& c, double* mom, double2* U, double2* X, const double* const* F, double2* g5DX,
                            int nf, const double* am0, double eps, int ns, int maxiter, double tol,
                            const qed2d_rhmc_params* r, MDState& s) {
    QTRY(md_kick_rhmc(c, mom, U, X, F, g5DX, nf, am0, 0.5 * eps, maxiter, tol, r));
    for (int i = 0; i < ns - 1; i++) {
        QTRY(md_links(c, U, mom, eps, s));
        QTRY(md_kick_rhmc(c, mom, U, X, F, g5DX, nf, am0, eps, maxiter, tol, r));
    }
    QTRY(md_links(c, U, mom, eps, s));
    return md_kick_rhmc(c, mom, U, X, F, g5DX, nf, am0, 0.5 * eps, maxiter, tol, r);
}

// Metropolis with the Qzero veto (src/QED2dHMC.jl:31-51)
static int metropolis(double hini, double hfin, double q, int qzero, double u) {
    double pacc;
    if (qzero && std::fabs(q) > 0.1) pacc = 0.0;
    else pacc = std::exp(-(hfin - hini));
    if (pacc < 1.0) return pacc > u ? 1 : 0;
    return 1;
}

}  // namespace qed2d

using namespace qed2d;

// ===========================================================================
// C ABI
extern "C" {

const char* qed2d_status_string(int s) {
    switch (s) {
        case QED2D_OK: return "ok";
        case QED2D_ERR_NOT_CONVERGED: return "CG not converged";
        case QED2D_ERR_TIMEOUT: return "grid barrier timed out";
        case QED2D_ERR_BAD_ARG: return "bad argument";
        case QED2D_ERR_CUDA: return "CUDA error";
        case QED2D_ERR_NO_MEMORY: return "out of device memory";
        case QED2D_ERR_UNSUPPORTED: return "unsupported";
        default: return "unknown status";
    }
}

const char* qed2d_last_error(void) { return g_last_error.c_str(); }
int64_t qed2d_launch_count(void) { return launches(); }

int qed2d_ctx_create(int L1, int L2, double beta, qed2d_ctx** out) {
    if (!out) return bad_arg("out is NULL");
    *out = nullptr;
    if (L1 < 2 || L2 < 2) return bad_arg("lattice extents must be >= 2");
    if ((long long)L1 * L2 > (1LL << 30)) return bad_arg("lattice volume above 2^30 sites");
    auto* h = new qed2d_ctx();
    Ctx& c = h->c;
    c.g.L1 = L1;
    c.g.L2 = L2;
    c.g.V = (long long)L1 * L2;
    c.beta = beta;
    cudaError_t e = cudaGetDevice(&c.device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, c.device);
    if (e == cudaSuccess) e = cudaMalloc(&c.ctl, sizeof(DevCtl));
    if (e == cudaSuccess) e = cudaMalloc(&c.part, sizeof(double) * kMaxPartVals * kMaxPartBlocks);
    if (e == cudaSuccess) e = cudaMallocHost(&c.ctl_host, sizeof(DevCtl));
    if (e == cudaSuccess) e = cudaMemset(c.ctl, 0, sizeof(DevCtl));
    if (e != cudaSuccess) {
        const int st = cuda_status(e, "qed2d_ctx_create");
        qed2d_ctx_destroy(h);
        return st;
    }
    std::memset(c.ctl_host, 0, sizeof(DevCtl));
    *out = h;
    return QED2D_OK;
}

int qed2d_ctx_destroy(qed2d_ctx* ctx) {
    if (!ctx) return QED2D_OK;
    Ctx& c = ctx->c;
    if (c.stream) cudaStreamSynchronize(c.stream);
    else cudaDeviceSynchronize();
    c.md_graph.release();
    for (auto& kv : c.ws) cudaFree(kv.second.first);
    if (c.ctl) cudaFree(c.ctl);
    if (c.part) cudaFree(c.part);
    if (c.ctl_host) cudaFreeHost(c.ctl_host);
    delete ctx;
    return QED2D_OK;
}

int qed2d_ctx_set_beta(qed2d_ctx* ctx, double beta) {
    QCTX(ctx);
    c.beta = beta;
    return QED2D_OK;
}

int qed2d_ctx_set_stream(qed2d_ctx* ctx, void* stream) {
    QCTX(ctx);
    c.stream = (cudaStream_t)stream;
    return QED2D_OK;
}

int qed2d_ctx_set_precision(qed2d_ctx* ctx, int precision) {
    QCTX(ctx);
    if (precision < QED2D_PREC_F64 || precision > QED2D_PREC_PLAIN) return bad_arg("unknown precision");
    c.precision = precision;
    return QED2D_OK;
}

int qed2d_ctx_get_dims(const qed2d_ctx* ctx, int* L1, int* L2) {
    if (!ctx) return bad_arg("context is NULL");
    if (L1) *L1 = ctx->c.g.L1;
    if (L2) *L2 = ctx->c.g.L2;
    return QED2D_OK;
}

// the Ctx::sched slot of a solver selector, -1 for none
static int sched_slot(int solver) {
    switch (solver) {
        case QED2D_PREC_F64: return 0;
        case QED2D_PREC_MIXED: return 1;
        case QED2D_MULTISHIFT: return 2;
        default: return -1;
    }
}

int qed2d_ctx_set_schedule(qed2d_ctx* ctx, int precision, int schedule) {
    QCTX(ctx);
    const int slot = sched_slot(precision);
    if (slot < 0) return bad_arg("schedule: QED2D_PREC_F64, QED2D_PREC_MIXED or QED2D_MULTISHIFT only");
    // the multishift solver also has its FP32-inner form (3), the mixed CG its RL form (4, 5, 6)
    const bool ok = schedule >= -1 && (schedule <= 2 || (slot == 2 && schedule == 3) ||
                                       (slot == 1 && schedule >= 4 && schedule <= 6));
    if (!ok)
        return bad_arg(slot == 2   ? "multishift schedule must be -1, 0, 1, 2 or 3"
                       : slot == 1 ? "mixed CG schedule must be -1, 0, 1, 2, 4, 5 or 6"
                                   : "schedule must be -1, 0, 1 or 2");
    c.sched[slot] = schedule;
    return QED2D_OK;
}

int qed2d_ctx_get_schedule(const qed2d_ctx* ctx, int precision, int* schedule) {
    if (!ctx || !schedule) return bad_arg("context or schedule is NULL");
    const int slot = sched_slot(precision);
    if (slot < 0) return bad_arg("schedule: QED2D_PREC_F64, QED2D_PREC_MIXED or QED2D_MULTISHIFT only");
    *schedule = ctx->c.sched[slot];
    return QED2D_OK;
}

int qed2d_ctx_set_multishift_layout(qed2d_ctx* ctx, int layout) {
    QCTX(ctx);
    if (layout < -1 || layout >= kMsLayoutCount) return bad_arg("multishift layout must be -1, 0, 1, 2 or 3");
    c.ms_layout = layout;
    if (layout < 0 && c.sched[2] >= 0 && c.sched[2] != 3) c.sched[2] = -1;   // tune both on the next solve
    return QED2D_OK;
}

int qed2d_ctx_get_multishift_layout(const qed2d_ctx* ctx, int* layout) {
    if (!ctx || !layout) return bad_arg("context or layout is NULL");
    *layout = ctx->c.ms_layout;
    return QED2D_OK;
}

int qed2d_ctx_set_graphs(qed2d_ctx* ctx, int on) {
    QCTX(ctx);
    c.md_graph.drop();
    c.md_graph.on = on != 0;
    return QED2D_OK;
}

int qed2d_ctx_graph_stats(const qed2d_ctx* ctx, int* on, int64_t* captures, int64_t* replays, int64_t* failures) {
    if (!ctx) return bad_arg("context is NULL");
    const GraphCache& g = ctx->c.md_graph;
    if (on) *on = g.on ? 1 : 0;
    if (captures) *captures = g.captures;
    if (replays) *replays = g.replays;
    if (failures) *failures = g.failures;
    return QED2D_OK;
}

int qed2d_selftest_barrier_timeout(qed2d_ctx* ctx, int64_t polls) {
    QCTX(ctx);
    if (polls < 1 || polls > (1LL << 26)) return bad_arg("polls must be in [1, 2^26]");
    QTRY(reset_seq(c));
    QTRY(barrier_timeout_probe(c, (long long)polls));
    return finish_seq(c, nullptr);
}

int qed2d_last_solve(const qed2d_ctx* ctx, int64_t* iterations, double* rel, int64_t* reliable_updates) {
    if (!ctx) return bad_arg("context is NULL");
    if (iterations) *iterations = ctx->c.last_iters;
    if (rel) *rel = ctx->c.last_relres;
    if (reliable_updates) *reliable_updates = ctx->c.last_updates;
    return QED2D_OK;
}

// ---- gauge kernels ----
int qed2d_plaquette_field(qed2d_ctx* ctx, double* plx, const double* U) {
    QCTX(ctx);
    QPTR(plx);
    QPTR(U);
    return launch_plaq_field(c, plx, C2(U), 0);
}

int qed2d_qtop_field(qed2d_ctx* ctx, double* plx, const double* U) {
    QCTX(ctx);
    QPTR(plx);
    QPTR(U);
    return launch_plaq_field(c, plx, C2(U), 1);
}

int qed2d_krnl_force(qed2d_ctx* ctx, double* frc1, double* frc2, const double* U) {
    QCTX(ctx);
    QPTR(frc1);
    QPTR(frc2);
    QPTR(U);
    return launch_krnl_force(c, frc1, frc2, C2(U));
}

int qed2d_updt_fld(qed2d_ctx* ctx, double* U, const double* mom, double eps) {
    QCTX(ctx);
    QPTR(U);
    QPTR(mom);
    return launch_updt_fld(c, C2(U), mom, eps, nullptr);
}

// ---- Dirac operator ----
int qed2d_gamm5dw(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0) {
    QCTX(ctx);
    QPTR(so);
    QPTR(U);
    QPTR(si);
    QTRY(check_out(c, so, si, "gamm5Dw"));
    QTRY(check_out(c, so, U, "gamm5Dw"));
    return launch_g5dw(c, C2(so), C2(U), C2(si), am0, nullptr, make_double2(0, 0), false);
}

int qed2d_gamm5dw_c64(qed2d_ctx* ctx, float* so, const float* U, const float* si, double am0) {
    QCTX(ctx);
    QPTR(so);
    QPTR(U);
    QPTR(si);
    const size_t nb = sizeof(float2) * 2 * (size_t)c.g.V;
    if (overlap(so, nb, si, nb) || overlap(so, nb, U, nb))
        return bad_arg("gamm5Dw (complex64): output aliases an input");
    return launch_g5dw_c64(c, reinterpret_cast<float2*>(so), reinterpret_cast<const float2*>(U),
                           reinterpret_cast<const float2*>(si), am0);
}

int qed2d_gamm5(qed2d_ctx* ctx, double* so, const double* si) {
    QCTX(ctx);
    QPTR(so);
    QPTR(si);
    return launch_g5(c, C2(so), C2(si));
}

int qed2d_dw(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0) {
    QCTX(ctx);
    QPTR(so);
    QPTR(U);
    QPTR(si);
    QTRY(check_out(c, so, si, "Dw"));
    QTRY(check_out(c, so, U, "Dw"));
    return launch_g5dw(c, C2(so), C2(U), C2(si), am0, nullptr, make_double2(0, 0), true);
}

int qed2d_gamm5dw_sqr(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0) {
    QCTX(ctx);
    QPTR(so);
    QPTR(U);
    QPTR(si);
    QTRY(check_out(c, so, si, "gamm5Dw_sqr"));
    QTRY(check_out(c, so, U, "gamm5Dw_sqr"));
    return op_sqr(c, C2(so), C2(U), C2(si), am0, 0.0);
}

int qed2d_gamm5dw_sqr_musq(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0, double mu) {
    QCTX(ctx);
    QPTR(so);
    QPTR(U);
    QPTR(si);
    QTRY(check_out(c, so, si, "gamm5Dw_sqr_musq"));
    QTRY(check_out(c, so, U, "gamm5Dw_sqr_musq"));
    return op_sqr(c, C2(so), C2(U), C2(si), am0, mu);
}

int qed2d_gamm5dw_sqr_sqr(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0) {
    QCTX(ctx);
    QPTR(so);
    QPTR(U);
    QPTR(si);
    QTRY(check_out(c, so, si, "gamm5Dw_sqr_sqr"));
    QTRY(check_out(c, so, U, "gamm5Dw_sqr_sqr"));
    double2* t = c.spinor("op_t2");
    if (!t) return QED2D_ERR_NO_MEMORY;
    QTRY(op_sqr(c, t, C2(U), C2(si), am0, 0.0));
    return op_sqr(c, C2(so), C2(U), t, am0, 0.0);
}

int qed2d_gamm5dw_sqr_sqr_musq(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0,
                               double mu) {
    QCTX(ctx);
    QPTR(so);
    QPTR(U);
    QPTR(si);
    QTRY(check_out(c, so, si, "gamm5Dw_sqr_sqr_musq"));
    QTRY(check_out(c, so, U, "gamm5Dw_sqr_sqr_musq"));
    double2* t = c.spinor("op_t2");
    double2* t3 = c.spinor("op_t3");
    if (!t || !t3) return QED2D_ERR_NO_MEMORY;
    QTRY(op_sqr(c, t, C2(U), C2(si), am0, 0.0));
    QTRY(launch_g5dw(c, t3, C2(U), t, am0, nullptr, make_double2(0, 0), false));
    return launch_g5dw(c, C2(so), C2(U), t3, am0, C2(si), make_double2(mu * mu, 0), false);
}

int qed2d_tr_dqwdu(qed2d_ctx* ctx, double* frc, const double* U, const double* X, const double* g5DwX) {
    QCTX(ctx);
    QPTR(frc);
    QPTR(U);
    QPTR(X);
    QPTR(g5DwX);
    return launch_tr_dqwdu(c, frc, C2(U), C2(X), C2(g5DwX));
}

int qed2d_unfold(qed2d_ctx* ctx, double* Uout, const double* Uin, int reflect) {
    QCTX(ctx);
    QPTR(Uout);
    QPTR(Uin);
    if (overlap(Uout, 4 * field_bytes(c), Uin, field_bytes(c))) return bad_arg("unfold: Uout aliases Uin");
    return launch_unfold(c, C2(Uout), C2(Uin), reflect);
}

int qed2d_plwv(qed2d_ctx* ctx, double* so, double k1, double k2) {
    QCTX(ctx);
    QPTR(so);
    return launch_plwv(c, C2(so), k1, k2);
}

int qed2d_random_normal(qed2d_ctx* ctx, double* out, int64_t n, uint64_t seed, uint32_t stream, uint32_t counter) {
    QCTX(ctx);
    QPTR(out);
    if (n < 0) return bad_arg("n < 0");
    return launch_random_normal(c, out, n, seed, stream, counter, 1.0);
}

double qed2d_random_uniform(uint64_t seed, uint32_t stream, uint32_t counter) {
    // Philox4x32-10 on the host (same rounds as the device version in device.cuh)
    uint32_t x[4] = {0u, 0u, stream, counter};
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    for (int r = 0; r < 10; r++) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * x[0], p1 = (uint64_t)0xCD9E8D57u * x[2];
        const uint32_t o0 = (uint32_t)(p1 >> 32) ^ x[1] ^ k0, o2 = (uint32_t)(p0 >> 32) ^ x[3] ^ k1;
        x[0] = o0;
        x[1] = (uint32_t)p1;
        x[2] = o2;
        x[3] = (uint32_t)p0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    const uint64_t a = ((((uint64_t)x[0]) << 32) | x[1]) >> 11;
    return ((double)a + 0.5) * 0x1.0p-53;
}

// ---- observables ----
int qed2d_action(qed2d_ctx* ctx, const double* U, double* S) {
    QCTX(ctx);
    QPTR(U);
    if (!S) return bad_arg("S is NULL");
    double h[3];
    QTRY(launch_reduce_gauge(c, C2(U), nullptr, 0));
    QTRY(fetch_scal(c, 0, 3, h));
    *S = c.beta * ((double)c.g.V - h[0]);
    return QED2D_OK;
}

int qed2d_plaquette(qed2d_ctx* ctx, const double* U, double* P) {
    QCTX(ctx);
    QPTR(U);
    if (!P) return bad_arg("P is NULL");
    double h[3];
    QTRY(launch_reduce_gauge(c, C2(U), nullptr, 0));
    QTRY(fetch_scal(c, 0, 3, h));
    *P = h[0] / (double)c.g.V;
    return QED2D_OK;
}

int qed2d_qtop(qed2d_ctx* ctx, const double* U, double* Q, int64_t* q_round) {
    QCTX(ctx);
    QPTR(U);
    double h[3];
    QTRY(launch_reduce_gauge(c, C2(U), nullptr, 0));
    QTRY(fetch_scal(c, 0, 3, h));
    const double q = h[1] / (2.0 * M_PI);
    if (Q) *Q = q;
    if (q_round) *q_round = (int64_t)std::llround(q);
    return QED2D_OK;
}

int qed2d_hamiltonian(qed2d_ctx* ctx, const double* mom, const double* U, double* H) {
    QCTX(ctx);
    QPTR(mom);
    QPTR(U);
    if (!H) return bad_arg("H is NULL");
    double h[3];
    QTRY(launch_reduce_gauge(c, C2(U), mom, 0));
    QTRY(fetch_scal(c, 0, 3, h));
    *H = h[2] / 2.0 + c.beta * ((double)c.g.V - h[0]);
    return QED2D_OK;
}

// ---- solvers ----
int qed2d_cg(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0, int maxiter, double eps,
             int* iterations) {
    QCTX(ctx);
    QPTR(so);
    QPTR(U);
    QPTR(si);
    QTRY(check_out(c, so, si, "CG"));
    QTRY(check_out(c, so, U, "CG"));
    if (maxiter < 0) return bad_arg("maxiter < 0");
    QTRY(reset_seq(c));
    QTRY(solve(c, C2(so), C2(U), C2(si), am0, 0.0, maxiter, eps, false, nullptr));
    const int st = finish_seq(c, nullptr);
    if (iterations) *iterations = (int)c.last_iters;
    return st;
}

int qed2d_cg_shift(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0, double mu,
                   int maxiter, double eps, int so_as_guess, int* iterations) {
    QCTX(ctx);
    QPTR(so);
    QPTR(U);
    QPTR(si);
    QTRY(check_out(c, so, si, "CG"));
    QTRY(check_out(c, so, U, "CG"));
    if (maxiter < 0) return bad_arg("maxiter < 0");
    QTRY(reset_seq(c));
    QTRY(solve(c, C2(so), C2(U), C2(si), am0, mu, maxiter, eps, so_as_guess != 0, nullptr));
    const int st = finish_seq(c, nullptr);
    if (iterations) *iterations = (int)c.last_iters;
    return st;
}

int qed2d_multishift_cg(qed2d_ctx* ctx, double* const* so, const double* U, const double* si, double am0,
                        const double* mu, int n, int maxiter, double eps, int* iterations) {
    QCTX(ctx);
    QPTR(U);
    QPTR(si);
    if (!so || !mu || n < 1 || n > QED2D_MAXPOLES) return bad_arg("multishift: bad shift list");
    std::vector<double2*> xs(n);
    std::vector<double> mu2(n);
    for (int i = 0; i < n; i++) {
        QTRY(check_ptr(so[i], "so[i]"));
        QTRY(check_out(c, so[i], si, "multishift CG"));
        QTRY(check_out(c, so[i], U, "multishift CG"));
        xs[i] = C2(so[i]);
        mu2[i] = mu[i] * mu[i];
    }
    QTRY(reset_seq(c));
    QTRY(multishift_solve(c, C2(U), C2(si), xs.data(), mu2.data(), n, am0, maxiter, eps));
    const int st = finish_seq(c, nullptr);
    if (iterations) *iterations = (int)c.last_iters;
    return st;
}

// ---- RHMC ----
int qed2d_get_rhmc_params(int n, double r_a, double r_b, qed2d_rhmc_params* out) {
    const int st = zolotarev_params(n, r_a, r_b, out);
    if (st != QED2D_OK) set_error("get_rhmc_params: need 1 <= n <= 32 and 0 < r_a < r_b");
    return st;
}

static int check_rhmc(const qed2d_rhmc_params* r) {
    if (!r || r->n < 1 || r->n > QED2D_MAXPOLES) return bad_arg("RHMC parameters: n out of range");
    return QED2D_OK;
}

int qed2d_multi_cg(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0, int maxiter,
                   double eps, const qed2d_rhmc_params* rprm, int* iterations) {
    QCTX(ctx);
    QPTR(so);
    QPTR(U);
    QPTR(si);
    QTRY(check_rhmc(rprm));
    QTRY(check_out(c, so, si, "MultiCG"));
    QTRY(check_out(c, so, U, "MultiCG"));
    QTRY(reset_seq(c));
    QTRY(multi_cg_core(c, C2(so), C2(U), C2(si), am0, maxiter, eps, rprm, false));
    int64_t it = 0;
    const int st = finish_seq(c, &it);
    if (iterations) *iterations = (int)it;
    return st;
}

int qed2d_rational(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0, int maxiter,
                   double eps, const qed2d_rhmc_params* rprm, int* iterations) {
    QCTX(ctx);
    QPTR(so);
    QPTR(U);
    QPTR(si);
    QTRY(check_rhmc(rprm));
    QTRY(check_out(c, so, si, "R"));
    QTRY(check_out(c, so, U, "R"));
    QTRY(reset_seq(c));
    QTRY(multi_cg_core(c, C2(so), C2(U), C2(si), am0, maxiter, eps, rprm, true));
    int64_t it = 0;
    const int st = finish_seq(c, &it);
    if (iterations) *iterations = (int)it;
    return st;
}

int qed2d_generate_pseudofermion(qed2d_ctx* ctx, double* F, const double* U, const double* X, double am0,
                                 int maxiter, double tol, const qed2d_rhmc_params* rprm, int* iterations) {
    QCTX(ctx);
    QPTR(F);
    QPTR(U);
    QPTR(X);
    QTRY(check_rhmc(rprm));
    QTRY(check_out(c, F, X, "generate_pseudofermion!"));
    QTRY(check_out(c, F, U, "generate_pseudofermion!"));
    QTRY(reset_seq(c));
    QTRY(pf_generate_core(c, C2(F), C2(U), C2(X), am0, maxiter, tol, rprm));
    int64_t it = 0;
    const int st = finish_seq(c, &it);
    if (iterations) *iterations = (int)it;
    return st;
}

int qed2d_power_method(qed2d_ctx* ctx, const double* U, double am0, int iter, uint64_t seed, uint32_t counter,
                       double* lambda_min, double* lambda_max) {
    QCTX(ctx);
    QPTR(U);
    if (iter < 0) return bad_arg("iter < 0");
    const long long N = 2 * c.g.V;
    double2* b = c.spinor("pm_b");
    double2* b2 = c.spinor("pm_b2");
    double2* tmp = c.spinor("pm_tmp");
    if (!b || !b2 || !tmp) return QED2D_ERR_NO_MEMORY;
    const double shift = 2.0;   // src/QED2dRHMC.jl:139
    const double2 z0 = make_double2(0, 0);
    // b = (randn + i randn)/sqrt(2)  (:137)
    QTRY(launch_random_normal(c, (double*)b, 2 * N, seed, QED2D_STREAM_POWER, counter, 1.0 / std::sqrt(2.0)));
    // b <- ((g5Dw)^2 b + shift b) / <.,.>  (:144-149)
    for (int it = 0; it < iter; it++) {
        QTRY(launch_g5dw(c, tmp, C2(U), b, am0, nullptr, z0, false));
        QTRY(launch_g5dw(c, b2, C2(U), tmp, am0, b, make_double2(shift, 0), false));
        QTRY(launch_reduce_vec(c, 0, b2, nullptr, N, 0));
        QTRY(launch_scale_inv(c, b, b2, N, 0));
    }
    // lambda_max = <b, A b + shift b> / <b, b> - shift  (:150-153)
    double h[4];
    QTRY(launch_g5dw(c, tmp, C2(U), b, am0, nullptr, z0, false));
    QTRY(launch_g5dw(c, b2, C2(U), tmp, am0, b, make_double2(shift, 0), false));
    QTRY(launch_reduce_vec(c, 1, b, b2, N, 0));
    QTRY(launch_reduce_vec(c, 1, b, b, N, 2));
    QTRY(fetch_scal(c, 0, 4, h));
    auto cdiv = [](double ar, double ai, double br, double bi) {
        if (std::fabs(br) >= std::fabs(bi)) {
            const double r = bi / br, den = br + bi * r;
            return std::pair<double, double>((ar + ai * r) / den, (ai - ar * r) / den);
        }
        const double r = br / bi, den = bi + br * r;
        return std::pair<double, double>((ar * r + ai) / den, (ai * r - ar) / den);
    };
    auto lmax = cdiv(h[0], h[1], h[2], h[3]);
    lmax.first -= shift;
    // b <- ((g5Dw)^2 b - lambda_max b) / <.,.>, applied out of place  (:157-162)
    const double2 ml = make_double2(-lmax.first, -lmax.second);
    for (int it = 0; it < iter; it++) {
        QTRY(launch_g5dw(c, tmp, C2(U), b, am0, nullptr, z0, false));
        QTRY(launch_g5dw(c, b2, C2(U), tmp, am0, b, ml, false));
        QTRY(launch_reduce_vec(c, 0, b2, nullptr, N, 0));
        QTRY(launch_scale_inv(c, b, b2, N, 0));
    }
    QTRY(launch_g5dw(c, tmp, C2(U), b, am0, nullptr, z0, false));
    QTRY(launch_g5dw(c, b2, C2(U), tmp, am0, b, ml, false));
    QTRY(launch_reduce_vec(c, 1, b, b2, N, 0));
    QTRY(launch_reduce_vec(c, 1, b, b, N, 2));
    QTRY(fetch_scal(c, 0, 4, h));
    auto lmin = cdiv(h[0], h[1], h[2], h[3]);
    if (lambda_max) *lambda_max = lmax.first;
    if (lambda_min) *lambda_min = lmin.first + lmax.first;
    return QED2D_OK;
}

int qed2d_luscher_z(qed2d_ctx* ctx, double* Z, const double* U, const double* Xin, double am0, int maxiter,
                    double tol, const qed2d_rhmc_params* rprm) {
    QCTX(ctx);
    QPTR(Z);
    QPTR(U);
    QPTR(Xin);
    QTRY(check_rhmc(rprm));
    QTRY(check_out(c, Z, Xin, "LuscherZ"));
    QTRY(check_out(c, Z, U, "LuscherZ"));
    QTRY(reset_seq(c));
    QTRY(luscher_z_core(c, C2(Z), C2(U), C2(Xin), am0, maxiter, tol, rprm));
    return finish_seq(c, nullptr);
}

int qed2d_reweighting_factor(qed2d_ctx* ctx, const double* U, double am0, int maxiter, double tol,
                             const qed2d_rhmc_params* rprm, uint64_t seed, uint32_t counter, double* W) {
    QCTX(ctx);
    QPTR(U);
    QTRY(check_rhmc(rprm));
    if (!W) return bad_arg("W is NULL");
    const long long N = 2 * c.g.V;
    double2* X = c.spinor("rw_X");
    double2* Z = c.spinor("rw_Z");
    double2* tmp = c.spinor("rw_tmp");
    if (!X || !Z || !tmp) return QED2D_ERR_NO_MEMORY;
    QTRY(reset_seq(c));
    double WN = 0.0;
    for (int j = 0; j < rprm->reweighting_N; j++) {
        double argexp = 0.0, Tfactor = 0.5, fact_i = 1.0;
        QTRY(launch_random_normal(c, (double*)X, 2 * N, seed, QED2D_STREAM_REWEIGHT + (uint32_t)j, counter,
                                  1.0 / std::sqrt(2.0)));
        QTRY(launch_copy(c, tmp, X, sizeof(double2) * N));
        for (int i = 1; i <= rprm->reweighting_Taylor; i++) {
            QTRY(luscher_z_core(c, Z, C2(U), tmp, am0, maxiter, tol, rprm));
            double h[2];
            QTRY(launch_reduce_vec(c, 1, X, Z, N, 0));
            QTRY(fetch_scal(c, 0, 2, h));
            argexp += Tfactor * h[0];
            const double fact_ip1 = fact_i * (double)(i + 1);   // (src/QED2dRHMC.jl:224)
            Tfactor *= (double)(-(2 * i + 1)) / 2.0 / fact_ip1 * fact_i;
            fact_i = fact_ip1;
            QTRY(launch_copy(c, tmp, Z, sizeof(double2) * N));
        }
        WN += std::exp(argexp) / (double)rprm->reweighting_N;
    }
    *W = WN;
    return finish_seq(c, nullptr);
}

// ---- molecular dynamics ----
int qed2d_omf4_gauge(qed2d_ctx* ctx, double* mom, double* U, double eps, int ns) {
    QCTX(ctx);
    QPTR(mom);
    QPTR(U);
    MDState s;
    return md_omf4_gauge(c, mom, C2(U), eps, ns, s);
}

int qed2d_update_momenta_nf2(qed2d_ctx* ctx, double* mom, const double* U, double* X, const double* F,
                             double* g5DX, double am0, double eps, int maxiter, double tol, int64_t* iterations) {
    QCTX(ctx);
    QPTR(mom);
    QPTR(U);
    QPTR(X);
    QPTR(F);
    QPTR(g5DX);
    QTRY(reset_seq(c));
    MDState s;
    QTRY(md_prepare(c, C2(U), s));
    QTRY(md_kick_nf2(c, mom, C2(U), C2(X), C2(F), C2(g5DX), am0, eps, maxiter, tol, s));
    return finish_seq(c, iterations);
}

int qed2d_leapfrog_nf2(qed2d_ctx* ctx, double* mom, double* U, double* X, const double* F, double* g5DX,
                       double am0, double eps, int ns, int maxiter, double tol, int64_t* iterations) {
    QCTX(ctx);
    QPTR(mom);
    QPTR(U);
    QPTR(X);
    QPTR(F);
    QPTR(g5DX);
    QTRY(reset_seq(c));
    MDState s;
    QTRY(md_prepare(c, C2(U), s));
    QTRY(md_leapfrog_nf2(c, mom, C2(U), C2(X), C2(F), C2(g5DX), am0, eps, ns, maxiter, tol, s));
    return finish_seq(c, iterations);
}

int qed2d_omf4_nf2(qed2d_ctx* ctx, double* mom, double* U, double* X, const double* F, double* g5DX, double am0,
                   double eps, int ns, int maxiter, double tol, int64_t* iterations) {
    QCTX(ctx);
    QPTR(mom);
    QPTR(U);
    QPTR(X);
    QPTR(F);
    QPTR(g5DX);
    QTRY(reset_seq(c));
    MDState s;
    QTRY(md_prepare(c, C2(U), s));
    QTRY(md_omf4_nf2(c, mom, C2(U), C2(X), C2(F), C2(g5DX), am0, eps, ns, maxiter, tol, s));
    return finish_seq(c, iterations);
}

int qed2d_update_momenta_rhmc(qed2d_ctx* ctx, double* mom, const double* U, double* X, const double* const* F,
                              double* g5DX, int nf, const double* am0, double eps, int maxiter, double tol,
                              const qed2d_rhmc_params* rprm, int64_t* iterations) {
    QCTX(ctx);
    QPTR(mom);
    QPTR(U);
    QPTR(X);
    QPTR(g5DX);
    if (!F || !am0 || !rprm || nf < 1) return bad_arg("update_momenta! RHMC: bad flavour arrays");
    for (int j = 0; j < nf; j++) {
        QTRY(check_ptr(F[j], "F[j]"));
        QTRY(check_rhmc(&rprm[j]));
    }
    QTRY(reset_seq(c));
    QTRY(md_kick_rhmc(c, mom, C2(U), C2(X), F, C2(g5DX), nf, am0, eps, maxiter, tol, rprm));
    return finish_seq(c, iterations);
}

int qed2d_leapfrog_rhmc(qed2d_ctx* ctx, double* mom, double* U, double* X, const double* const* F, double* g5DX,
                        int nf, const double* am0, double eps, int ns, int maxiter, double tol,
                        const qed2d_rhmc_params* rprm, int64_t* iterations) {
    QCTX(ctx);
    QPTR(mom);
    QPTR(U);
    QPTR(X);
    QPTR(g5DX);
    if (!F || !am0 || !rprm || nf < 1) return bad_arg("leapfrog! RHMC: bad flavour arrays");
    for (int j = 0; j < nf; j++) {
        QTRY(check_ptr(F[j], "F[j]"));
        QTRY(check_rhmc(&rprm[j]));
    }
    QTRY(reset_seq(c));
    MDState s;
    QTRY(md_prepare(c, C2(U), s));
    QTRY(md_leapfrog_rhmc(c, mom, C2(U), C2(X), F, C2(g5DX), nf, am0, eps, ns, maxiter, tol, rprm, s));
    return finish_seq(c, iterations);
}

// ---- HMC steps ----
// Slots of ctl->scal: [0..2] sums at the start (Re P, arg P, mom^2), [3] |X|^2,
// [4..6] sums at the end, [8..9] <X, F> at the end, [10..11] scratch.
static void fill_result(qed2d_hmc_result* res, int acc, double hi, double hf, double q, int64_t it) {
    if (!res) return;
    res->accepted = acc;
    res->hini = hi;
    res->hfin = hf;
    res->dH = hf - hi;
    res->qtop = q;
    res->cg_iterations = it;
}

int qed2d_hmc_gauge(qed2d_ctx* ctx, double* U, double eps, int ns, int integrator, int qzero, uint64_t seed,
                    uint32_t counter, qed2d_hmc_result* res) {
    QCTX(ctx);
    QPTR(U);
    double2* Ucp = c.spinor("hmc_Ucp");
    double* mom = c.real2("hmc_mom");
    if (!Ucp || !mom) return QED2D_ERR_NO_MEMORY;
    QTRY(reset_seq(c));
    QTRY(launch_copy(c, Ucp, U, field_bytes(c)));
    QTRY(launch_random_normal(c, mom, 2 * c.g.V, seed, QED2D_STREAM_MOMENTA, counter, 1.0));
    QTRY(launch_reduce_gauge(c, C2(U), mom, 0));
    GraphKey k;
    k.i(1).p(U).p(mom).d(eps).i(ns).i(integrator).d(c.beta).i((long long)c.ws_gen);
    QTRY(run_graphed(c.md_graph, c.stream, k.s, [&]() -> int {
        MDState s;
        if (integrator == QED2D_OMF4) return md_omf4_gauge(c, mom, C2(U), eps, ns, s);
        return md_leapfrog_gauge(c, mom, C2(U), eps, ns, s);
    }));
    QTRY(launch_reduce_gauge(c, C2(U), mom, 4));
    double h[8];
    QTRY(fetch_scal(c, 0, 8, h));
    const double V = (double)c.g.V;
    const double hini = h[2] / 2.0 + c.beta * (V - h[0]);
    const double hfin = h[6] / 2.0 + c.beta * (V - h[4]);
    const double qf = h[5] / (2.0 * M_PI);
    const int acc = metropolis(hini, hfin, qf, qzero, qed2d_random_uniform(seed, QED2D_STREAM_METROPOLIS, counter));
    if (!acc) QTRY(launch_copy(c, U, Ucp, field_bytes(c)));
    fill_result(res, acc, hini, hfin, acc ? qf : h[1] / (2.0 * M_PI), 0);
    const int st = finish_seq(c, nullptr);
    return st;
}

int qed2d_hmc_nf2(qed2d_ctx* ctx, double* U, double am0, double eps, int ns, int integrator, int maxiter,
                  double tol, int qzero, uint64_t seed, uint32_t counter, qed2d_hmc_result* res) {
    QCTX(ctx);
    QPTR(U);
    const long long N = 2 * c.g.V;
    double2* Ucp = c.spinor("hmc_Ucp");
    double* mom = c.real2("hmc_mom");
    double2* X = c.spinor("hmc_X");
    double2* F = c.spinor("hmc_F");
    double2* g5DX = c.spinor("hmc_g5DX");
    if (!Ucp || !mom || !X || !F || !g5DX) return QED2D_ERR_NO_MEMORY;
    QTRY(reset_seq(c));
    QTRY(launch_copy(c, Ucp, U, field_bytes(c)));
    // momenta and X = (randn + i randn)/sqrt(2)   (src/QED2dHMC.jl:69-70)
    QTRY(launch_random_normal(c, mom, N, seed, QED2D_STREAM_MOMENTA, counter, 1.0));
    QTRY(launch_random_normal(c, (double*)X, 2 * N, seed, QED2D_STREAM_NOISE, counter, 1.0 / std::sqrt(2.0)));
    QTRY(launch_reduce_gauge(c, C2(U), mom, 0));
    QTRY(launch_reduce_vec(c, 0, X, nullptr, N, 3));
    // F = g5Dw X  (:76-78)
    QTRY(launch_g5dw(c, F, C2(U), X, am0, nullptr, make_double2(0, 0), false));
    auto md = [&]() -> int {
        MDState s;
        QTRY(md_prepare(c, C2(U), s));
        if (integrator == QED2D_OMF4) return md_omf4_nf2(c, mom, C2(U), X, F, g5DX, am0, eps, ns, maxiter, tol, s);
        return md_leapfrog_nf2(c, mom, C2(U), X, F, g5DX, am0, eps, ns, maxiter, tol, s);
    };
    if (c.precision == QED2D_PREC_PLAIN) {   // host-synchronised solver: not capturable
        QTRY(md());
    } else {
        GraphKey k;
        k.i(2).p(U).p(mom).p(X).p(F).p(g5DX).d(am0).d(eps).i(ns).i(integrator).i(maxiter).d(tol).d(c.beta);
        k.i(c.precision).i(c.sched[0]).i(c.sched[1]).i((long long)c.ws_gen);
        QTRY(run_graphed(c.md_graph, c.stream, k.s, md));
    }
    QTRY(launch_reduce_gauge(c, C2(U), mom, 4));
    QTRY(launch_reduce_vec(c, 1, X, F, N, 8));
    double h[10];
    QTRY(fetch_scal(c, 0, 10, h));
    const int st = read_ctl(c, false);
    const int64_t iters = c.ctl_host->iters_total;
    const double V = (double)c.g.V;
    const double hini = h[2] / 2.0 + c.beta * (V - h[0]) + h[3];
    const double hfin = h[6] / 2.0 + c.beta * (V - h[4]) + h[8];
    const double qf = h[5] / (2.0 * M_PI);
    int acc = 0;
    if (st == QED2D_OK)
        acc = metropolis(hini, hfin, qf, qzero, qed2d_random_uniform(seed, QED2D_STREAM_METROPOLIS, counter));
    if (!acc) QTRY(launch_copy(c, U, Ucp, field_bytes(c)));
    fill_result(res, acc, hini, hfin, acc ? qf : h[1] / (2.0 * M_PI), iters);
    if (!acc) QCHECK(cudaStreamSynchronize(c.stream));
    if (st != QED2D_OK) set_error(std::string("HMC! Nf=2: ") + qed2d_status_string(st));
    return st;
}

int qed2d_hmc_rhmc(qed2d_ctx* ctx, double* U, int nf, const double* am0, double eps, int ns, int maxiter,
                   double tol, const qed2d_rhmc_params* rprm, int qzero, int reversibility, uint64_t seed,
                   uint32_t counter, qed2d_hmc_result* res) {
    QCTX(ctx);
    QPTR(U);
    if (nf < 1 || !am0 || !rprm) return bad_arg("HMC! RHMC: bad flavour arrays");
    for (int j = 0; j < nf; j++) QTRY(check_rhmc(&rprm[j]));
    const long long N = 2 * c.g.V;
    double2* Ucp = c.spinor("hmc_Ucp");
    double* mom = c.real2("hmc_mom");
    double2* X = c.spinor("hmc_X");
    double2* g5DX = c.spinor("hmc_g5DX");
    std::vector<double*> F(nf);
    for (int j = 0; j < nf; j++) F[j] = (double*)c.spinor("hmc_F_" + std::to_string(j));
    if (!Ucp || !mom || !X || !g5DX) return QED2D_ERR_NO_MEMORY;
    for (int j = 0; j < nf; j++)
        if (!F[j]) return QED2D_ERR_NO_MEMORY;
    QTRY(reset_seq(c));
    QTRY(launch_copy(c, Ucp, U, field_bytes(c)));
    QTRY(launch_random_normal(c, mom, N, seed, QED2D_STREAM_MOMENTA, counter, 1.0));
    QTRY(launch_reduce_gauge(c, C2(U), mom, 0));
    double h[12];
    QTRY(fetch_scal(c, 0, 3, h));
    const double V = (double)c.g.V;
    double hini = h[2] / 2.0 + c.beta * (V - h[0]);
    const double q_ini = h[1] / (2.0 * M_PI);
    // pseudofermions (src/QED2dHMC.jl:136-144)
    for (int j = 0; j < nf; j++) {
        QTRY(launch_random_normal(c, (double*)X, 2 * N, seed, QED2D_STREAM_NOISE + (uint32_t)j, counter,
                                  1.0 / std::sqrt(2.0)));
        QTRY(launch_reduce_vec(c, 0, X, nullptr, N, 3));
        QTRY(fetch_scal(c, 3, 1, &h[3]));
        hini += h[3];
        QTRY(pf_generate_core(c, C2(F[j]), C2(U), X, am0[j], maxiter, tol, &rprm[j]));
    }
    MDState s;
    auto md = [&]() -> int {
        QTRY(md_prepare(c, C2(U), s));
        return md_leapfrog_rhmc(c, mom, C2(U), X, F.data(), g5DX, nf, am0, eps, ns, maxiter, tol, rprm, s);
    };
    if (c.precision == QED2D_PREC_PLAIN) {   // host-synchronised solver: not capturable
        QTRY(md());
    } else {
        GraphKey k;
        k.i(3).p(U).p(mom).p(X).p(g5DX).i(nf).d(eps).i(ns).i(maxiter).d(tol).d(c.beta);
        k.i(c.precision).i(c.sched[0]).i(c.sched[1]).i(c.sched[2]).i(c.ms_layout).i((long long)c.ws_gen);
        for (int j = 0; j < nf; j++) {
            k.p(F[j]).d(am0[j]).i(rprm[j].n);
            for (int i = 0; i < rprm[j].n; i++) k.d(rprm[j].mu[i]).d(rprm[j].rho[i]);
        }
        QTRY(run_graphed(c.md_graph, c.stream, k.s, md));
        s.U32 = c.precision == QED2D_PREC_MIXED ? c.spinor32("md_u32") : nullptr;   // as md_prepare leaves it
    }
    QTRY(launch_reduce_gauge(c, C2(U), mom, 4));
    QTRY(fetch_scal(c, 4, 3, &h[4]));
    double hfin = h[6] / 2.0 + c.beta * (V - h[4]);
    const double qf = h[5] / (2.0 * M_PI);
    // final pseudofermion action with MultiCG (:150-156)
    for (int j = 0; j < nf; j++) {
        QTRY(multi_cg_core(c, X, C2(U), C2(F[j]), am0[j], maxiter, tol, &rprm[j], false));
        QTRY(launch_reduce_vec(c, 1, X, C2(F[j]), N, 8));
        QTRY(fetch_scal(c, 8, 2, &h[8]));
        hfin += h[8];
    }
    int acc = 1;
    if (reversibility) {   // (:159-164): negate momenta, integrate back, keep U
        QTRY(launch_zaxpby(c, (double2*)mom, make_double2(-1, 0), (const double2*)mom, make_double2(0, 0), nullptr,
                           c.g.V));
        QTRY(md_leapfrog_rhmc(c, mom, C2(U), X, F.data(), g5DX, nf, am0, eps, ns, maxiter, tol, rprm, s));
    }
    const int st = read_ctl(c, false);
    const int64_t iters = c.ctl_host->iters_total;
    if (!reversibility) {
        acc = st == QED2D_OK
                  ? metropolis(hini, hfin, qf, qzero, qed2d_random_uniform(seed, QED2D_STREAM_METROPOLIS, counter))
                  : 0;
        if (!acc) QTRY(launch_copy(c, U, Ucp, field_bytes(c)));
    }
    fill_result(res, acc, hini, hfin, acc ? qf : q_ini, iters);
    QCHECK(cudaStreamSynchronize(c.stream));
    if (st != QED2D_OK) set_error(std::string("HMC! RHMC: ") + qed2d_status_string(st));
    return st;
}

}  // extern "C"
