/*
 * qed2d_oracle.h -- CPU restatement of the QED2d (dalbandea/Dav-QED2d) simulation
 * hot path, used ONLY as test infrastructure: the checker that the CUDA library's
 * results are compared against, and the timed CPU baseline.  Nothing in the
 * product (libqed2d) links or calls this code.
 *
 * Parity status: the reference is Julia/CUDA.jl and cannot run in this
 * environment (no Julia, no CPU path in the reference).  This restatement is
 * pinned against
 *   - the reference's own known-answer test: the free-field plane-wave eigenvalue
 *     of D_W (tests/Dw-eigenvalues.jl:15-35 with src/QED2dUtils.jl:2-11), turned
 *     into a hard assertion;
 *   - the reference's property assertions (test/rhmc_pf_generation.jl:56-57,
 *     test/rhmc_pf_forcetest.jl:92-93, test/rhmc_hmc_reversibility.jl:46-50,
 *     test/rhmc_zolovarev_bound.jl:42,65,84) and force-vs-finite-difference
 *     checks (tests/gauge_forcetest.jl, tests/fermion_forcetest.jl);
 *   - golden vectors from an independent NumPy restatement plus dense linear
 *     algebra, and Zolotarev coefficients evaluated with mpmath at 50 digits
 *     (tests/golden/make_golden.py).
 * No output of the reference itself exists to pin against ("parity pinned by the
 * reference's tests, not by reference outputs").
 *
 * Layout (identical to the reference's Julia column-major arrays):
 *   gauge links  U[i1,i2,mu]  -> complex double at i1 + L1*(i2 + L2*mu)
 *   spinors      s[i1,i2,sp]  -> complex double at i1 + L1*(i2 + L2*sp)
 *   momenta / forces mom[i1,i2,mu] -> double at i1 + L1*(i2 + L2*mu)
 *   per-site fields plx[i1,i2] -> double at i1 + L1*i2
 * All indices here are 0-based; the reference's are 1-based.
 */
#ifndef QED2D_ORACLE_H
#define QED2D_ORACLE_H

#include <complex.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double _Complex ocplx;

#define O_MAXPOLES 32

/* LattParm (src/QED2d.jl:5-8) */
typedef struct {
    int L1, L2;
    double beta;
} o_latt;

/* RHMCParm (src/QED2d.jl:15-26) */
typedef struct {
    double r_b;
    int n;
    double eps;
    double A;
    double rho[O_MAXPOLES];
    double mu[O_MAXPOLES];
    double nu[O_MAXPOLES];
    double delta;
    int reweighting_N;
    int reweighting_Taylor;
} o_rhmc;

enum { O_OK = 0, O_NOT_CONVERGED = 1, O_BAD_ARG = 3 };
enum { O_OP_SQR = 0, O_OP_SQR_MUSQ = 1 };   /* gamm5Dw_sqr_msq, gamm5Dw_sqr_musq */
enum { O_LEAPFROG = 0, O_OMF4 = 1 };

/* ---- random numbers shared with the CUDA library (Philox4x32-10 + Box-Muller) ---- */
void o_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void o_fill_normal(double* out, int64_t n, uint64_t seed, uint32_t stream, uint32_t counter);
double o_uniform(uint64_t seed, uint32_t stream, uint32_t counter);

/* ---- site kernels (src/QED2dAction.jl, src/QED2dDirac.jl, src/QED2dFields.jl, src/QED2dUtils.jl) ---- */
void o_plaquette_field(const o_latt* p, double* plx, const ocplx* U);
void o_qtop_field(const o_latt* p, double* plx, const ocplx* U);
void o_gauge_force(const o_latt* p, double* frc1, double* frc2, const ocplx* U);
void o_update_links(const o_latt* p, ocplx* U, const double* mom, double eps);
void o_g5dw(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0);
void o_g5(const o_latt* p, ocplx* so, const ocplx* si);
void o_dw(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0);
void o_g5dw_sqr(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0);
void o_g5dw_sqr_sqr(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0);
void o_g5dw_sqr_musq(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0, double mu);
void o_g5dw_sqr_sqr_musq(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0, double mu);
void o_fermion_force(const o_latt* p, double* frc, const ocplx* U, const ocplx* X, const ocplx* g5X);
void o_unfold(int L1old, int L2old, ocplx* Uout, const ocplx* Uin, int reflect);
void o_plane_wave(const o_latt* p, ocplx* so, double k1, double k2);

/* ---- reductions (src/QED2dHMC.jl:198-237) ---- */
double o_action(const o_latt* p, const ocplx* U);
double o_plaquette(const o_latt* p, const ocplx* U);
double o_qtop(const o_latt* p, const ocplx* U);
double o_hamiltonian(const o_latt* p, const double* mom, const ocplx* U);
ocplx o_dot(int64_t n, const ocplx* a, const ocplx* b);   /* sum conj(a)*b */
double o_norm2(int64_t n, const ocplx* a);

/* ---- solvers (src/QED2dSolver.jl) ---- */
int o_cg(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0,
         double mu, int op, int maxiter, double eps, int so_as_guess, int* iters, double* final_err);
int o_multi_cg(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0,
               int maxiter, double eps, const o_rhmc* r, int* iters);
int o_rational(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0,
               int maxiter, double eps, const o_rhmc* r, int* iters);

/* ---- RHMC (src/QED2dRHMC.jl) ---- */
double o_ellip_K(double m);
void o_ellip_sncn(double u, double m, double* sn, double* cn);
int o_zolotarev(int n, double r_a, double r_b, o_rhmc* out);
int o_pf_generate(const o_latt* p, ocplx* F, const ocplx* U, const ocplx* X, double am0,
                  int maxiter, double tol, const o_rhmc* r, int* iters);
void o_power_method(const o_latt* p, const ocplx* U, double am0, int iter, const ocplx* b0,
                    double* lmin, double* lmax);
int o_luscher_z(const o_latt* p, ocplx* Z, const ocplx* U, const ocplx* Xin, double am0,
                int maxiter, double tol, const o_rhmc* r);
int o_reweighting_factor(const o_latt* p, const ocplx* U, double am0, int maxiter, double tol,
                         const o_rhmc* r, const ocplx* noise, double* W);

/* ---- integrators and HMC (src/QED2dHMC.jl) ---- */
void o_omf4_gauge(const o_latt* p, double* mom, ocplx* U, double eps, int ns);
int o_update_momenta_nf2(const o_latt* p, double* mom, const ocplx* U, ocplx* X, const ocplx* F,
                         ocplx* g5DX, double am0, double eps, int maxiter, double tol, int* iters);
int o_leapfrog_nf2(const o_latt* p, double* mom, ocplx* U, ocplx* X, const ocplx* F, ocplx* g5DX,
                   double am0, double eps, int ns, int maxiter, double tol, int* iters);
int o_omf4_nf2(const o_latt* p, double* mom, ocplx* U, ocplx* X, const ocplx* F, ocplx* g5DX,
               double am0, double eps, int ns, int maxiter, double tol, int* iters);
int o_update_momenta_rhmc(const o_latt* p, double* mom, const ocplx* U, ocplx* X, ocplx* const* F,
                          ocplx* g5DX, int nf, const double* am0, double eps, int maxiter, double tol,
                          const o_rhmc* r, int* iters);
int o_leapfrog_rhmc(const o_latt* p, double* mom, ocplx* U, ocplx* X, ocplx* const* F, ocplx* g5DX,
                    int nf, const double* am0, double eps, int ns, int maxiter, double tol,
                    const o_rhmc* r, int* iters);

/* HMC steps.  Random inputs are injected (momenta, noise, Metropolis uniform) so
 * that the CUDA library's draws can be replayed here exactly. */
int o_hmc_gauge(const o_latt* p, ocplx* U, double eps, int ns, int integrator, int qzero,
                const double* mom0, double r_unif, int* accepted, double* hini, double* hfin);
int o_hmc_nf2(const o_latt* p, ocplx* U, double am0, double eps, int ns, int integrator,
              int maxiter, double tol, int qzero, const double* mom0, const ocplx* noise,
              double r_unif, int* accepted, double* hini, double* hfin, int* iters);
int o_hmc_rhmc(const o_latt* p, ocplx* U, int nf, const double* am0, double eps, int ns,
               int maxiter, double tol, const o_rhmc* r, int qzero, int reversibility,
               const double* mom0, const ocplx* noise, double r_unif,
               int* accepted, double* hini, double* hfin, int* iters);

int o_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
