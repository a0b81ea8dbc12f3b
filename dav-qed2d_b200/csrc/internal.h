// internal.h -- host-side internals of libqed2d: the context (lattice geometry,
// stream, workspace, device control block) and the kernel launchers that the
// C ABI (api.cpp) and the solvers/integrators (engine.cpp) are built from.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <vector>

#include "qed2d.h"   // include/ (on the include path)

namespace qed2d {

struct Lat {
    int L1, L2;
    long long V;
};

// Device control block shared by the kernels of one context.
struct DevCtl {
    unsigned long long bar;   // grid-barrier arrivals, zeroed before each persistent launch
    unsigned long long gen;   // grid-barrier release generation, zeroed likewise
    int err;                  // barrier timeout flag, zeroed likewise
    int status;               // sticky: first failing status of the current sequence
    long long iters_total;    // CG iterations accumulated since the last reset
    int last_iters;           // iterations of the most recent solve
    int last_conv;            // 1 if the most recent solve converged
    double last_relres;       // |r|^2 / |b|^2 at the end of the most recent solve
    unsigned ticket;          // completion ticket of single-launch reductions
    int last_updates;         // reliable updates of the most recent (mixed) solve
    double scal[32];          // results of reductions
    double red[8];            // grid-reduction results of persistent kernels (double buffered)
};

constexpr int kMaxPartBlocks = 2048;   // partial-sum slots per reduced quantity
constexpr int kMsLayoutCount = 4;      // layouts of the multishift kernel (tile rows, threads per site)
constexpr int kMaxPartVals = 8;        // quantities reduced together

// CUDA graph of the MD part of a trajectory, replayed per trajectory (graph.h)
struct GraphCache {
    bool on = true;
    std::string key;    // key of exec
    std::string warm;   // key of the last direct run
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap = nullptr;   // private capture stream
    int64_t nlaunch = 0;          // library launches inside the graph
    int64_t captures = 0, replays = 0, failures = 0;

    void drop() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        key.clear();
        warm.clear();
    }
    void release() {
        drop();
        if (cap) cudaStreamDestroy(cap);
        cap = nullptr;
    }
};

struct Ctx {
    Lat g;
    double beta = 0.0;
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    int precision = QED2D_PREC_F64;
    DevCtl* ctl = nullptr;       // device
    DevCtl* ctl_host = nullptr;  // pinned mirror for read-back
    double* part = nullptr;      // device partials [kMaxPartVals][kMaxPartBlocks]
    std::map<std::string, std::pair<void*, size_t>> ws;   // named device workspace
    int64_t last_iters = 0;
    int64_t last_updates = 0;
    double last_relres = 0.0;
    int sched[3] = {-1, -1, -1};   // reduction schedule of the F64 / MIXED / multishift solvers (-1: not tuned yet)
    int ms_layout = -1;            // layout of the multishift kernel (kMsLayouts; -1: tuned with the schedule)
    GraphCache md_graph;           // MD integration of the HMC trajectories (graph.h)
    uint64_t ws_gen = 0;           // bumped whenever a workspace buffer is reallocated

    void* buf(const std::string& name, size_t bytes);   // grow-only named workspace
    double2* spinor(const std::string& name) { return (double2*)buf(name, sizeof(double2) * 2 * g.V); }
    double* real2(const std::string& name) { return (double*)buf(name, sizeof(double) * 2 * g.V); }
    float4* spinor32(const std::string& name) { return (float4*)buf(name, sizeof(float4) * g.V); }
};

// error plumbing ------------------------------------------------------------
void set_error(const std::string& msg);
int cuda_status(cudaError_t e, const char* what);
#define QCHECK(call)                                                   \
    do {                                                               \
        cudaError_t e_ = (call);                                       \
        if (e_ != cudaSuccess) return ::qed2d::cuda_status(e_, #call); \
    } while (0)
#define QTRY(call)                          \
    do {                                    \
        int s_ = (call);                    \
        if (s_ != QED2D_OK) return s_;      \
    } while (0)

void count_launch(int n = 1);
// Reliable-update threshold of the mixed solvers: the FP32 residual is replaced
// by the FP64 true residual once |r|^2 has dropped by kReliableDelta^2 since the
// last update (or looks converged).  Convergence is decided on the FP64 true
// residual whatever the value, so it sets only how often the update runs.
// Measured on B200 (batched 4 x 512^2 Nf=2 trajectory): 0.05 -> 0.01 takes the
// updates per solve from 10 to 6 with the same iteration counts (302-312),
// 23.4 -> 24.0 traj/s; on a well-conditioned 512^2 system the mixed and FP64
// solvers need the same iterations (122) at 0.02 and 0.05 alike.
constexpr double kReliableDelta = 0.01;

// launches the bounded-wait self-test kernel (cg.cu); the status lands in ctl->status
int barrier_timeout_probe(Ctx& c, long long polls);

bool tuning_enabled();   // QED2D_TUNE=0 in the environment turns schedule tuning off
int64_t launches();

// kernel launchers (kernels.cu) --------------------------------------------
// All complex fields are double2 planes in the reference layout.
int launch_g5dw_c64(Ctx& c, float2* so, const float2* U, const float2* si, double am0);
int launch_g5dw(Ctx& c, double2* so, const double2* U, const double2* si, double am0, const double2* addv,
                double2 addc, bool g5_out);
int launch_g5(Ctx& c, double2* so, const double2* si);
int launch_tr_dqwdu(Ctx& c, double* frc, const double2* U, const double2* X, const double2* G);
int launch_plaq_field(Ctx& c, double* plx, const double2* U, int mode);
int launch_krnl_force(Ctx& c, double* frc1, double* frc2, const double2* U);
int launch_updt_fld(Ctx& c, double2* U, const double* mom, double eps, float4* U32);
int launch_pack_links(Ctx& c, float4* U32, const double2* U);
int launch_unfold(Ctx& c, double2* Uout, const double2* Uin, int reflect);
int launch_plwv(Ctx& c, double2* so, double k1, double k2);
int launch_random_normal(Ctx& c, double* out, int64_t n, uint64_t seed, uint32_t stream, uint32_t counter,
                         double scale);
// Uout = e^{i eu mom_in} Uin, then mom_out = mom_in + ek * gauge force(Uout): a
// link update and the pure-gauge kick after it in one pass (distinct in/out
// buffers); QED2D_ERR_UNSUPPORTED unless the lattice is whole 32 x 8 tiles
int launch_updt_kick(Ctx& c, double2* Uout, const double2* Uin, double* mom_out, const double* mom_in, double eu,
                     double ek);
bool updt_kick_fits(const Ctx& c);   // the lattice is whole tiles of launch_updt_kick
// mom += eps * (gauge force + fermion force), the fermion force either from
// (X, G = g5Dw X) or precomputed in frc (either may be null)
int launch_mom_kick(Ctx& c, double* mom, const double2* U, double eps, const double2* X, const double2* G,
                    const double* frc);
// frc (+)= rho * tr_dQwdU(U, X, G)
int launch_force_poles(Ctx& c, double* frc, const double2* U, const double2* const* X, double2* const* G,
                       const double* rho, int n, double am0, bool accumulate);
int launch_force_accum(Ctx& c, double* frc, const double2* U, const double2* X, const double2* G, double rho,
                       bool accumulate);
// BLAS-1 on complex planes of n = 2V elements (alpha given on host)
int launch_zaxpby(Ctx& c, double2* y, double2 a, const double2* x, double2 b, const double2* z, long long n);
int launch_copy(Ctx& c, void* dst, const void* src, size_t bytes);
int launch_zero(Ctx& c, void* dst, size_t bytes);
// dot / norms into ctl->scal[slot..]: kind 0 = |x|^2 (1 value), 1 = <x,y> (2 values)
int launch_reduce_vec(Ctx& c, int kind, const double2* x, const double2* y, long long n, int slot);
// lattice sums into ctl->scal[slot..]: (sum Re P, sum arg P, sum mom^2) -- mom may be null
int launch_reduce_gauge(Ctx& c, const double2* U, const double* mom, int slot);
int launch_copy_scalar(Ctx& c, int dst_slot, int src_slot);
int launch_scale_inv(Ctx& c, double2* y, const double2* x, long long n, int slot);

// solvers (cg.cu) -----------------------------------------------------------
struct SolveArgs {
    const double2* U = nullptr;   // links (planes)
    const float4* U32 = nullptr;  // packed FP32 links (mixed path); built if null
    const double2* b = nullptr;
    double2* x = nullptr;         // solution (planes); input guess if guess
    double am0 = 0.0;
    double mu2 = 0.0;             // shift mu^2
    int maxiter = 10000;
    double eps = 1e-24;           // stop when |r|^2 < eps |b|^2
    bool guess = false;
    double2* g5x = nullptr;       // optional output: g5Dw x of the final solution
};
int cg_solve(Ctx& c, const SolveArgs& a, int precision);
int multishift_solve(Ctx& c, const double2* U, const double2* b, double2* const* x, const double* mu2, int n,
                     double am0, int maxiter, double eps);
// read back the control block (synchronises the stream); status of the sequence
int read_ctl(Ctx& c, bool reset_sequence);

// host-side Zolotarev (zolotarev.cpp)
int zolotarev_params(int n, double r_a, double r_b, qed2d_rhmc_params* out);

}  // namespace qed2d
