/*
 * qed2d.h -- C ABI of libqed2d, the B200 (sm_100a) engine for the simulation hot
 * path of the QED2d Julia package (dalbandea/Dav-QED2d): 2D compact U(1) gauge
 * theory with two-spin Wilson fermions, HMC and RHMC.
 *
 * Each entry point replaces one function of the reference's exported API
 * (src/QED2d.jl:27-54); the comment above it gives the reference file:line.
 * Paths are relative to the reference project root.
 *
 * Conventions
 *  - Arrays are caller-owned DEVICE pointers in the reference's layout: the
 *    Julia column-major arrays
 *        U    :: CuArray{ComplexF64}(L1, L2, 2)   links, direction last
 *        s    :: CuArray{ComplexF64}(L1, L2, 2)   spinors, spin last
 *        mom  :: CuArray{Float64}(L1, L2, 2)      momenta / forces
 *        plx  :: CuArray{Float64}(L1, L2)         per-site fields
 *    i.e. element (i1, i2, k) (0-based) at offset i1 + L1*(i2 + L2*k).  A complex
 *    array is passed as `double*` to interleaved (re, im) pairs.  Pointers must be
 *    16-byte aligned; stencil operators reject an output that aliases an input.
 *  - Every function returns a qed2d_status.  Work is issued on the context's
 *    stream (default: the legacy default stream).  Functions that return host
 *    scalars (observables, iteration counts, HMC results) synchronise that
 *    stream; the others are asynchronous.
 *  - A context is not thread-safe; use one context per host thread.
 *  - CG tolerance: as in the reference (src/QED2dSolver.jl:13-29) a solve stops
 *    when |r|^2 < eps * |b|^2, so eps = 1e-24 means a relative residual of 1e-12.
 *  - Random numbers (momenta, pseudofermion noise, power-method start vectors,
 *    reweighting noise, the Metropolis uniform) come from Philox4x32-10 keyed by
 *    (seed, stream, counter); qed2d_random_normal() reproduces any stream.
 */
#ifndef QED2D_H
#define QED2D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    QED2D_OK = 0,
    QED2D_ERR_NOT_CONVERGED = 1, /* CG hit maxiter (reference: error(), src/QED2dSolver.jl:39-43,98-102) */
    QED2D_ERR_TIMEOUT = 2,       /* a grid barrier inside a persistent kernel gave up waiting */
    QED2D_ERR_BAD_ARG = 3,       /* bad size, NULL, misaligned or aliased pointer */
    QED2D_ERR_CUDA = 4,          /* a CUDA runtime call failed (qed2d_last_error() has the text) */
    QED2D_ERR_NO_MEMORY = 5,
    QED2D_ERR_UNSUPPORTED = 6
} qed2d_status;

/* solver precision used by every CG inside the library */
typedef enum {
    QED2D_PREC_F64 = 0,   /* FP64 persistent fused CG; the reference's arithmetic and stop rule */
    QED2D_PREC_MIXED = 1, /* FP32 inner CG with FP64 reliable updates; stops on the FP64 true residual */
    QED2D_PREC_PLAIN = 2  /* reference-structured FP64: unfused kernels, host-synchronised CG loop */
} qed2d_precision;

typedef enum { QED2D_LEAPFROG = 0, QED2D_OMF4 = 1 } qed2d_integrator;   /* src/integrators/integrators.jl:1-3 */

#define QED2D_MAXPOLES 32

/* RHMCParm -- src/QED2d.jl:15-26 */
typedef struct {
    double r_b;
    int32_t n;
    double eps;
    double A;
    double rho[QED2D_MAXPOLES];
    double mu[QED2D_MAXPOLES];
    double nu[QED2D_MAXPOLES];
    double delta;
    int32_t reweighting_N;
    int32_t reweighting_Taylor;
} qed2d_rhmc_params;

/* outcome of one HMC trajectory (the reference logs these, src/QED2dHMC.jl:53-57) */
typedef struct {
    int32_t accepted;
    double hini;
    double hfin;
    double dH;
    double qtop;            /* Qtop(U) of the final (accepted or restored) field */
    int64_t cg_iterations;  /* summed over every solve of the trajectory */
} qed2d_hmc_result;

/* Philox streams used by the HMC entry points (counter = the trajectory counter) */
#define QED2D_STREAM_MOMENTA 1u
#define QED2D_STREAM_METROPOLIS 3u
#define QED2D_STREAM_POWER 4u
#define QED2D_STREAM_NOISE 16u      /* + flavour index j: pseudofermion noise X_j */
#define QED2D_STREAM_REWEIGHT 64u   /* + sample index j: reweighting noise */

typedef struct qed2d_ctx qed2d_ctx;

/* ---- context: LattParm(iL, beta) -- src/QED2d.jl:5-8.  KernelParm (:10-13) has no
 * counterpart: launch geometry is chosen by the library. ---- */
int qed2d_ctx_create(int L1, int L2, double beta, qed2d_ctx** out);
int qed2d_ctx_destroy(qed2d_ctx* ctx);
int qed2d_ctx_set_beta(qed2d_ctx* ctx, double beta);
int qed2d_ctx_set_stream(qed2d_ctx* ctx, void* cuda_stream);
int qed2d_ctx_set_precision(qed2d_ctx* ctx, int precision);
int qed2d_ctx_get_dims(const qed2d_ctx* ctx, int* L1, int* L2);
/* Reduction schedule of a persistent solver, selected by `precision`:
 * QED2D_PREC_F64 or QED2D_PREC_MIXED (qed2d_cg and the HMC solves), or
 * QED2D_MULTISHIFT (qed2d_multishift_cg and the RHMC solves).  0 = the last
 * block to reach a grid barrier sums the partials and publishes them, 1 = every
 * block sums them itself, 2 = the whole solve in one thread-block cluster with
 * the hardware cluster barrier (lattices of at most 128 tiles of 32x8 sites).
 * 0 and 1 give the same bits; 2 uses fewer blocks, so its sums are grouped
 * differently.  The first solve of each kind on a context times the candidates
 * and keeps the fastest (a host synchronisation; QED2D_TUNE=0 in the
 * environment selects a fixed size rule instead).  set: 0, 1 or 2 to fix it
 * (2 falls back to 1 where no cluster fits), -1 to tune again on the next
 * solve; get: -1 while untuned.  The multishift solver has a fourth form, 3 =
 * the shared Krylov space in FP32 (to a relative residual of 1e-6), then every
 * shift refined by the mixed CG from that start to the FP64 stop rule; it is the
 * first solve's choice on lattices of 2^22 sites and more (measured faster there,
 * slower below), and is otherwise chosen only when set.  The mixed CG has a
 * second form under each reduction schedule, 4, 5, 6 = 0, 1, 2 with the first
 * phase's stencil applied to r (t = g5Dw r + beta t_old) and the FP32 links of
 * every block's tiles staged once per solve in shared memory; it agrees with
 * the first form to the solver's accuracy, is a candidate of the first solve's
 * timing, and is refused (QED2D_ERR_UNSUPPORTED) where the staged links do not
 * fit beside co-resident blocks (large lattices). */
#define QED2D_MULTISHIFT 3   /* schedule selector of the multishift solver (FP64) */
int qed2d_ctx_set_schedule(qed2d_ctx* ctx, int precision, int schedule);
int qed2d_ctx_get_schedule(const qed2d_ctx* ctx, int precision, int* schedule);
/* Layout of the FP64 multishift kernel (schedules 0-2; no reference
 * counterpart: it takes the role of KernelParm's launch geometry for the RHMC
 * solves).  0 = tiles of 32 x 8 sites, one thread per site; 1 = 32 x 8 tiles,
 * two threads per site; 2 = 32 x 4 tiles, four threads per site; 3 = 32 x 4
 * tiles, two threads per site.  The extra threads of a site take a share of the
 * shift updates (each shift's x and p), the first runs the stencil and the base
 * system as well, so the lattice spreads over more SMs and warps.  Layouts
 * that split the lattice into the same blocks (same tile height, as many
 * blocks as tiles) give the same bits; the others agree to rounding.  -1 =
 * tune it with the schedule on the next multishift solve (get: -1 while
 * untuned).  Measured per iteration with 12 poles, grid schedule 1: 64^2 9.50
 * (layout 0) -> 7.85 us (layout 2); 128^2 9.54 -> 8.30 us (layout 2); 256^2
 * and 512^2 layout 0 fastest (12.7 and 42.9 us). */
int qed2d_ctx_set_multishift_layout(qed2d_ctx* ctx, int layout);
int qed2d_ctx_get_multishift_layout(const qed2d_ctx* ctx, int* layout);

/* No counterpart in the reference (CUDA.jl enqueues and synchronises every
 * launch from the host).  CUDA-graph replay of the MD integration inside
 * qed2d_hmc_gauge, qed2d_hmc_nf2 and qed2d_hmc_rhmc (not in the PLAIN
 * precision, whose solver reads scalars back every iteration; not the RHMC
 * reversibility pass): the first trajectory with a given set of arguments runs
 * directly (it tunes the solvers and allocates the workspace), the second
 * captures its MD launches -- every force evaluation's persistent solver
 * launch, the kicks and the link updates -- into a graph, and later ones replay
 * it with one cudaGraphLaunch.  Any change of arguments, field pointers,
 * precision, schedule, beta or workspace starts over.  Results are bitwise
 * those of the direct launches.  On by default; a capture the driver refuses
 * turns it off for the context (failures counts those).  set: 0 off, 1 on
 * (drops a captured graph).  stats: on, graphs captured, graph launches,
 * failed captures (any pointer may be NULL). */
int qed2d_ctx_set_graphs(qed2d_ctx* ctx, int on);
int qed2d_ctx_graph_stats(const qed2d_ctx* ctx, int* on, int64_t* captures, int64_t* replays, int64_t* failures);
/* Self-test of failure detection (no counterpart in the reference): runs one
 * kernel whose grid-barrier wait can never complete, with the wait bounded to
 * `polls` polls (1..2^26, rounded up to a multiple of 8: the limit is checked
 * every 8th poll) instead of the solvers' 2^26.  The wait gives up as a
 * solver's barrier does when a block never arrives, and the call returns
 * QED2D_ERR_TIMEOUT; the context stays usable for the next call. */
int qed2d_selftest_barrier_timeout(qed2d_ctx* ctx, int64_t polls);
/* iterations, final |r|^2/|b|^2 and (QED2D_PREC_MIXED) FP64 reliable updates of
 * the most recent solve on this context; any pointer may be NULL */
int qed2d_last_solve(const qed2d_ctx* ctx, int64_t* iterations, double* rel_residual_sq,
                     int64_t* reliable_updates);
const char* qed2d_status_string(int status);
const char* qed2d_last_error(void);
/* kernels launched by this process so far (all contexts) */
int64_t qed2d_launch_count(void);

/* ---- gauge kernels: src/QED2dAction.jl ---- */
/* plaquette! -- src/QED2dAction.jl:2-16: plx = Re U1(x)U2(x+1)conj(U1(x+2)U2(x)) */
int qed2d_plaquette_field(qed2d_ctx* ctx, double* plx, const double* U);
/* qtop! -- src/QED2dAction.jl:18-32: plx = arg of the plaquette */
int qed2d_qtop_field(qed2d_ctx* ctx, double* plx, const double* U);
/* krnl_force! -- src/QED2dAction.jl:34-53 (two buffers, every element written) */
int qed2d_krnl_force(qed2d_ctx* ctx, double* frc1, double* frc2, const double* U);
/* updt_fld! -- src/QED2dAction.jl:55-65: U <- exp(i eps mom) U */
int qed2d_updt_fld(qed2d_ctx* ctx, double* U, const double* mom, double eps);

/* ---- Dirac operator: src/QED2dDirac.jl ---- */
/* gamm5Dw -- src/QED2dDirac.jl:2-33 */
int qed2d_gamm5dw(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0);
/* gamm5Dw on complex64 fields in the same layout (FP32 arithmetic): the
 * single-precision apply of the mixed solver, for complex64 callers */
int qed2d_gamm5dw_c64(qed2d_ctx* ctx, float* so, const float* U, const float* si, double am0);
/* gamm5 -- src/QED2dDirac.jl:130-146 */
int qed2d_gamm5(qed2d_ctx* ctx, double* so, const double* si);
/* Dw -- src/QED2dDirac.jl:157-169 */
int qed2d_dw(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0);
/* gamm5Dw_sqr -- src/QED2dDirac.jl:35-46; also gamm5Dw_sqr_msq (:69-81), which adds no mass term */
int qed2d_gamm5dw_sqr(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0);
/* gamm5Dw_sqr_sqr -- src/QED2dDirac.jl:48-67 */
int qed2d_gamm5dw_sqr_sqr(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0);
/* gamm5Dw_sqr_musq -- src/QED2dDirac.jl:83-95: so = (g5Dw)^2 si + mu^2 si */
int qed2d_gamm5dw_sqr_musq(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0, double mu);
/* gamm5Dw_sqr_sqr_musq -- src/QED2dDirac.jl:97-117 */
int qed2d_gamm5dw_sqr_sqr_musq(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0,
                               double mu);
/* tr_dQwdU -- src/QED2dDirac.jl:172-199 */
int qed2d_tr_dqwdu(qed2d_ctx* ctx, double* frc, const double* U, const double* X, const double* g5DwX);

/* ---- fields and utilities ---- */
/* unfold_fld! / unfold_reflect! -- src/QED2dFields.jl:2-50.  ctx describes the
 * OLD (L1 x L2) lattice; Uout is a caller-owned (2 L1) x (2 L2) link array. */
int qed2d_unfold(qed2d_ctx* ctx, double* Uout, const double* Uin, int reflect);
/* plwv -- src/QED2dUtils.jl:2-11 */
int qed2d_plwv(qed2d_ctx* ctx, double* so, double k1, double k2);
/* n N(0,1) numbers of stream `stream` at counter `counter` (CUDA.randn's role) */
int qed2d_random_normal(qed2d_ctx* ctx, double* out, int64_t n, uint64_t seed, uint32_t stream,
                        uint32_t counter);
/* the Metropolis uniform of trajectory `counter` (Julia rand()'s role), host only */
double qed2d_random_uniform(uint64_t seed, uint32_t stream, uint32_t counter);

/* ---- observables: src/QED2dHMC.jl:198-237 ---- */
int qed2d_action(qed2d_ctx* ctx, const double* U, double* S);            /* Action   :206-215 */
int qed2d_plaquette(qed2d_ctx* ctx, const double* U, double* P);         /* Plaquette :217-226 */
/* Qtop :228-237 (unrounded, as the reference); q_round (may be NULL) = round(Q) */
int qed2d_qtop(qed2d_ctx* ctx, const double* U, double* Q, int64_t* q_round);
int qed2d_hamiltonian(qed2d_ctx* ctx, const double* mom, const double* U, double* H); /* :198-203 */

/* ---- solvers: src/QED2dSolver.jl ---- */
/* CG method 1 (:3-46) on gamm5Dw_sqr_msq: so = ((g5Dw)^2)^-1 si */
int qed2d_cg(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0, int maxiter,
             double eps, int* iterations);
/* CG method 2 (:49-105) on gamm5Dw_sqr_musq: so = ((g5Dw)^2 + mu^2)^-1 si; so_as_guess != 0 warm-starts */
int qed2d_cg_shift(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0, double mu,
                   int maxiter, double eps, int so_as_guess, int* iterations);
/* all n shifted systems ((g5Dw)^2 + mu_i^2) so[i] = si in one Krylov space.  No
 * single reference counterpart: it replaces the n sequential CG calls of
 * MultiCG (src/QED2dRHMC.jl:284-287) and update_momenta! (src/QED2dHMC.jl:529-544). */
int qed2d_multishift_cg(qed2d_ctx* ctx, double* const* so, const double* U, const double* si, double am0,
                        const double* mu, int n, int maxiter, double eps, int* iterations);

/* No counterpart in the reference.  CG method 1 exactly as qed2d_cg, for callers
 * that cannot allocate device memory while they run (a loop whose device memory
 * is owned by its own pool allocator, or one that cannot afford the implicit
 * device synchronisation of cudaMalloc): it needs no context and allocates
 * nothing.  Its scratch is one static device array, held by every GPU that loads
 * the library, sized for at most QED2D_NOALLOC_MAX_SITES = L1*L2 sites (larger
 * lattices are rejected with QED2D_ERR_BAD_ARG).  The first call on a device looks
 * up that array's address (make it before any stream capture) and keeps it for
 * the process: after a cudaDeviceReset of that device, do not call this entry
 * point on it again.  All calls share the array: calls that overlap on the GPU
 * race.  so must not overlap si or U.  Work runs on `stream` (NULL: the legacy
 * default stream); the call synchronises it. */
#define QED2D_NOALLOC_MAX_SITES 16384
int qed2d_cg_noalloc(int L1, int L2, double* so, const double* U, const double* si, double am0, int maxiter,
                     double eps, void* stream, int* iterations);

/* ---- RHMC: src/QED2dRHMC.jl ---- */
/* get_rhmc_params -- :93-110 (host; Zolotarev coefficients) */
int qed2d_get_rhmc_params(int n, double r_a, double r_b, qed2d_rhmc_params* out);
/* Elliptic.K(m) and Jacobi.sn(u, m), Jacobi.cn(u, m) of Elliptic.jl -- the
 * functions the reference's Zolotarev helpers k, v, a_r, c_r, mu, nu, rho_mu, d,
 * A, delta are written on (src/QED2dRHMC.jl:2-89; calls at :3-5), with the
 * parameter m = k^2, 0 <= m < 1.  Host only (no device work). */
int qed2d_ellip_K(double m, double* K);
int qed2d_ellip_sncn(double u, double m, double* sn, double* cn);
/* MultiCG -- :281-290: so = (1 + sum_j rho_j ((g5Dw)^2 + mu_j^2)^-1) si */
int qed2d_multi_cg(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0, int maxiter,
                   double eps, const qed2d_rhmc_params* rprm, int* iterations);
/* R -- :261-271: so = (A / r_b) MultiCG(si) ~ ((g5Dw)^2)^-1/2 si */
int qed2d_rational(qed2d_ctx* ctx, double* so, const double* U, const double* si, double am0, int maxiter,
                   double eps, const qed2d_rhmc_params* rprm, int* iterations);
/* generate_pseudofermion! -- :298-319 */
int qed2d_generate_pseudofermion(qed2d_ctx* ctx, double* F, const double* U, const double* X, double am0,
                                 int maxiter, double tol, const qed2d_rhmc_params* rprm, int* iterations);
/* power_method -- :135-170 (start vector: stream QED2D_STREAM_POWER at `counter`;
 * the second loop is applied out of place, see the reference's :159) */
int qed2d_power_method(qed2d_ctx* ctx, const double* U, double am0, int iter, uint64_t seed, uint32_t counter,
                       double* lambda_min, double* lambda_max);
/* LuscherZ -- :174-186: Z = ((g5Dw)^2 R^2 - 1) Xin */
int qed2d_luscher_z(qed2d_ctx* ctx, double* Z, const double* U, const double* Xin, double am0, int maxiter,
                    double tol, const qed2d_rhmc_params* rprm);
/* reweighting_factor -- :210-239 (noise: stream QED2D_STREAM_REWEIGHT + j at `counter`) */
int qed2d_reweighting_factor(qed2d_ctx* ctx, const double* U, double am0, int maxiter, double tol,
                             const qed2d_rhmc_params* rprm, uint64_t seed, uint32_t counter, double* W);

/* ---- molecular dynamics: src/QED2dHMC.jl ---- */
/* OMF4! pure gauge -- :239-305 */
int qed2d_omf4_gauge(qed2d_ctx* ctx, double* mom, double* U, double eps, int ns);
/* update_momenta! Nf=2 -- :452-481 (iterations may be NULL; accumulates otherwise) */
int qed2d_update_momenta_nf2(qed2d_ctx* ctx, double* mom, const double* U, double* X, const double* F,
                             double* g5DX, double am0, double eps, int maxiter, double tol, int64_t* iterations);
/* leapfrog! Nf=2 -- :426-449 */
int qed2d_leapfrog_nf2(qed2d_ctx* ctx, double* mom, double* U, double* X, const double* F, double* g5DX,
                       double am0, double eps, int ns, int maxiter, double tol, int64_t* iterations);
/* OMF4! Nf=2 -- :307-422 */
int qed2d_omf4_nf2(qed2d_ctx* ctx, double* mom, double* U, double* X, const double* F, double* g5DX,
                   double am0, double eps, int ns, int maxiter, double tol, int64_t* iterations);
/* update_momenta! RHMC -- :516-557 (F: nf pseudofermion fields) */
int qed2d_update_momenta_rhmc(qed2d_ctx* ctx, double* mom, const double* U, double* X, const double* const* F,
                              double* g5DX, int nf, const double* am0, double eps, int maxiter, double tol,
                              const qed2d_rhmc_params* rprm, int64_t* iterations);
/* leapfrog! RHMC -- :485-513 */
int qed2d_leapfrog_rhmc(qed2d_ctx* ctx, double* mom, double* U, double* X, const double* const* F,
                        double* g5DX, int nf, const double* am0, double eps, int ns, int maxiter, double tol,
                        const qed2d_rhmc_params* rprm, int64_t* iterations);

/* ---- HMC steps (U updated in place; restored on rejection) ---- */
/* HMC! pure gauge -- :19-60 (integrator: OMF4 as the reference; LEAPFROG is an extension) */
int qed2d_hmc_gauge(qed2d_ctx* ctx, double* U, double eps, int ns, int integrator, int qzero, uint64_t seed,
                    uint32_t counter, qed2d_hmc_result* res);
/* HMC! Nf=2 -- :64-113 */
int qed2d_hmc_nf2(qed2d_ctx* ctx, double* U, double am0, double eps, int ns, int integrator, int maxiter,
                  double tol, int qzero, uint64_t seed, uint32_t counter, qed2d_hmc_result* res);
/* HMC! RHMC -- :116-195 (reversibility != 0: the reference's reversibility_test mode) */
int qed2d_hmc_rhmc(qed2d_ctx* ctx, double* U, int nf, const double* am0, double eps, int ns, int maxiter,
                   double tol, const qed2d_rhmc_params* rprm, int qzero, int reversibility, uint64_t seed,
                   uint32_t counter, qed2d_hmc_result* res);

/* ---- batched replicas (no single reference counterpart: the reference runs one
 * chain per process; this runs nrep independent chains together, of equal or
 * uneven lattice sizes, each following HMC! Nf=2 with leapfrog,
 * src/QED2dHMC.jl:64-113,426-481).  A batch field is replica-major: replica r's
 * field is an ordinary reference-layout array ([L1_r, L2_r, 2]) starting at
 * complex element 2*off_r (real fields: real element 2*off_r), where off_r is
 * the number of sites of replicas 0..r-1 (qed2d_batch_layout).  Solves use the
 * mixed FP32/FP64 solver.  At most 1024 replicas and 2^30 sites per batch. ---- */
typedef struct qed2d_batch qed2d_batch;
/* nrep replicas of L1 x L2 sites; beta[nrep] */
int qed2d_batch_create(int nrep, int L1, int L2, const double* beta, qed2d_batch** out);
/* nrep replicas of L1[r] x L2[r] sites; beta[nrep] */
int qed2d_batch_create_ragged(int nrep, const int* L1, const int* L2, const double* beta, qed2d_batch** out);
/* site_offsets[nrep+1]: off_r of every replica, then the total number of sites */
int qed2d_batch_layout(const qed2d_batch* batch, int64_t* site_offsets);
int qed2d_batch_destroy(qed2d_batch* batch);
int qed2d_batch_set_stream(qed2d_batch* batch, void* cuda_stream);
/* the batched solver's schedule.  Equal-size batches of at most 64 replicas: 0/1
 * as qed2d_ctx_set_schedule, 4 = independent replicas (each replica's blocks
 * have a barrier of their own and leave when it has converged), 5 = the same
 * with a leaner reduction (two block barriers per grid reduction instead of
 * seven), 7 = schedule 5 with the stencil operands of each tile staged into
 * shared memory by TMA one tile ahead (replicas of whole tiles only: L1 a
 * multiple of 32, L2 of the tile height 8 or 16; QED2D_ERR_UNSUPPORTED
 * otherwise); 0, 1, 4, 5 and 7 give the same bits.  8 = schedule 5 with the
 * first phase's stencil applied to r (t = g5Dw r + beta t_old; p formed at the
 * site only): the same recurrences with t rounded along its own recurrence, so
 * results agree with 5 to the solver's accuracy (FP64 stop rule unchanged);
 * faster where the FP32 working set stays in L2 (4 x 512^2: 26.5 -> 24.5 us per
 * iteration).  9 = schedule 8 with the FP32 links of each block's tiles staged
 * once per solve in shared memory (where they fit beside co-resident blocks;
 * QED2D_ERR_UNSUPPORTED otherwise); agrees with 8 to rounding.  Other batches:
 * 2 = one launch over all replicas with grid
 * barriers, 3 = one thread-block cluster per replica (no grid barrier; replicas
 * stream through the GPU, largest first), 6 = 3 with the first phase's stencil
 * on r (as 8); these group their sums differently.
 * The first solve times the candidates and keeps the fastest; a schedule set
 * here is kept (for equal sizes the first solve then tunes the tile height
 * only); -1 = tune again on the next solve (get: -1 while untuned). */
int qed2d_batch_set_schedule(qed2d_batch* batch, int schedule);
int qed2d_batch_get_schedule(const qed2d_batch* batch, int* schedule);
/* Tile height of the equal-size batched solver: tiles of 32 x rows sites, rows =
 * 4, 8 or 16 (blocks of 128, 256 or 512 threads, so more or fewer blocks share a
 * replica's tiles and barriers).  It takes the role of the reference's
 * KernelParm launch geometry (src/QED2d.jl:10-13), which the library chooses:
 * the first solve tunes it together with the schedule; set: fix it (-1 = tune
 * again); get: -1 while untuned.  Heights group the sums differently: results
 * agree to rounding, not bit for bit.  Other batches: BAD_ARG. */
int qed2d_batch_set_tile_rows(qed2d_batch* batch, int rows);
int qed2d_batch_get_tile_rows(const qed2d_batch* batch, int* rows);
/* No counterpart in the reference.  CUDA-graph replay of the leapfrog inside
 * qed2d_batch_hmc_nf2 (the FP32 link copy, every force evaluation's batched
 * solver launch, the kicks and link updates), with the protocol and stats of
 * qed2d_ctx_set_graphs / qed2d_ctx_graph_stats: direct on the first trajectory
 * with given arguments (masses, eps, ns, tolerances, field pointers,
 * schedules), captured on the second, replayed after.  On by default. */
int qed2d_batch_set_graphs(qed2d_batch* batch, int on);
int qed2d_batch_graph_stats(const qed2d_batch* batch, int* on, int64_t* captures, int64_t* replays,
                            int64_t* failures);
/* every replica's CG method 1 (src/QED2dSolver.jl:3-46) in one launch:
 * x_r = ((g5Dw)^2)^-1 b_r with mass am0[r]; iterations[nrep] and updates[nrep]
 * (FP64 reliable updates) may be NULL */
int qed2d_batch_cg(qed2d_batch* batch, double* x, const double* U, const double* b, const double* am0, int maxiter,
                   double eps, int* iterations, int* updates);
/* one trajectory of every replica: am0[nrep], seeds[nrep] (replica r draws as a
 * single-lattice qed2d_hmc_nf2 with seed seeds[r] and the same counter); res[nrep] */
int qed2d_batch_hmc_nf2(qed2d_batch* batch, double* U, const double* am0, double eps, int ns, int maxiter,
                        double tol, int qzero, const uint64_t* seeds, uint32_t counter, qed2d_hmc_result* res);

#ifdef __cplusplus
}
#endif
#endif /* QED2D_H */
