/*
 * qed2d_oracle.c -- CPU restatement (C99 + OpenMP, FP64) of the simulation hot
 * path of the QED2d Julia package (dalbandea/Dav-QED2d).  TEST INFRASTRUCTURE
 * ONLY: the parity checker for the CUDA library and the timed CPU baseline.
 * The product library never links, loads or calls this file.
 *
 * Every function cites the reference lines it restates (paths relative to the
 * reference project root).  Array layout and parity status: see qed2d_oracle.h.
 *
 * Documented deviations from the reference (each also applies to the CUDA path):
 *   - o_cg with an all-zero source returns the zero solution after 0 iterations
 *     (the reference divides 0/0 and returns NaNs, src/QED2dSolver.jl:15-21);
 *   - o_power_method applies (g5 Dw)^2 out of place in its second loop; the
 *     reference passes the same array as input and output (src/QED2dRHMC.jl:159),
 *     a read/write race on the GPU whose result depends on launch order.
 */
#include "qed2d_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define CHUNK 4096

static inline ocplx mul_i(ocplx z) { return CMPLX(-cimag(z), creal(z)); }

/* a / b by Smith's scaled algorithm (R. L. Smith, CACM 5(8), 1962).  The plain
 * formula a*conj(b)/|b|^2 underflows once |b| ~ 1e-160, which the powers Z^p X
 * of the reweighting test reach; Julia's complex division is scaled as well. */
static inline ocplx cdiv(ocplx a, ocplx b) {
    const double ar = creal(a), ai = cimag(a), br = creal(b), bi = cimag(b);
    if (fabs(br) >= fabs(bi)) {
        const double r = bi / br, den = br + bi * r;
        return CMPLX((ar + ai * r) / den, (ai - ar * r) / den);
    } else {
        const double r = br / bi, den = bi + br * r;
        return CMPLX((ar * r + ai) / den, (ai * r - ar) / den);
    }
}

int o_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------- */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
 * as 1, 2, 3", SC'11) and the Box-Muller transform.  The CUDA library uses the
 * same counter layout, so a trajectory's random inputs can be replayed here. */
static inline void philox_round(uint32_t c[4], const uint32_t k[2]) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t o0 = hi1 ^ c[1] ^ k[0];
    uint32_t o1 = lo1;
    uint32_t o2 = hi0 ^ c[3] ^ k[1];
    uint32_t o3 = lo0;
    c[0] = o0; c[1] = o1; c[2] = o2; c[3] = o3;
}

void o_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    uint32_t k[2] = {key[0], key[1]};
    for (int r = 0; r < 10; r++) {
        philox_round(c, k);
        if (r < 9) { k[0] += 0x9E3779B9u; k[1] += 0xBB67AE85u; }
    }
    memcpy(out, c, sizeof(c));
}

/* pair j of stream `stream` at trajectory `counter`: two N(0,1) numbers */
static inline void normal_pair(uint64_t seed, uint32_t stream, uint32_t counter, uint64_t j,
                               double* z0, double* z1) {
    const uint32_t ctr[4] = {(uint32_t)j, (uint32_t)(j >> 32), stream, counter};
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t x[4];
    o_philox4x32_10(ctr, key, x);
    const uint64_t a = (((uint64_t)x[0] << 32) | x[1]) >> 11;
    const uint64_t b = (((uint64_t)x[2] << 32) | x[3]) >> 11;
    const double u1 = ((double)a + 0.5) * 0x1.0p-53;   /* (0,1) */
    const double u2 = (double)b * 0x1.0p-53;           /* [0,1) */
    const double rad = sqrt(-2.0 * log(u1));
    const double th = 6.283185307179586 * u2;
    *z0 = rad * cos(th);
    *z1 = rad * sin(th);
}

void o_fill_normal(double* out, int64_t n, uint64_t seed, uint32_t stream, uint32_t counter) {
    const int64_t npair = (n + 1) / 2;
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < npair; j++) {
        double z0, z1;
        normal_pair(seed, stream, counter, (uint64_t)j, &z0, &z1);
        out[2 * j] = z0;
        if (2 * j + 1 < n) out[2 * j + 1] = z1;
    }
}

double o_uniform(uint64_t seed, uint32_t stream, uint32_t counter) {
    const uint32_t ctr[4] = {0u, 0u, stream, counter};
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t x[4];
    o_philox4x32_10(ctr, key, x);
    const uint64_t a = (((uint64_t)x[0] << 32) | x[1]) >> 11;
    return ((double)a + 0.5) * 0x1.0p-53;
}

/* ------------------------------------------------------------------------- */
/* Reductions in a fixed order (chunks of CHUNK elements, then the chunk sums in
 * order), so results do not depend on the thread count. */
double o_norm2(int64_t n, const ocplx* a) {
    const int64_t nc = (n + CHUNK - 1) / CHUNK;
    double* part = (double*)malloc(sizeof(double) * (size_t)(nc > 0 ? nc : 1));
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nc; c++) {
        const int64_t e = (c + 1) * CHUNK < n ? (c + 1) * CHUNK : n;
        double s = 0.0;
        for (int64_t i = c * CHUNK; i < e; i++) s += creal(a[i]) * creal(a[i]) + cimag(a[i]) * cimag(a[i]);
        part[c] = s;
    }
    double s = 0.0;
    for (int64_t c = 0; c < nc; c++) s += part[c];
    free(part);
    return s;
}

ocplx o_dot(int64_t n, const ocplx* a, const ocplx* b) {
    const int64_t nc = (n + CHUNK - 1) / CHUNK;
    ocplx* part = (ocplx*)malloc(sizeof(ocplx) * (size_t)(nc > 0 ? nc : 1));
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nc; c++) {
        const int64_t e = (c + 1) * CHUNK < n ? (c + 1) * CHUNK : n;
        double sr = 0.0, si = 0.0;
        for (int64_t i = c * CHUNK; i < e; i++) {
            const double ar = creal(a[i]), ai = cimag(a[i]), br = creal(b[i]), bi = cimag(b[i]);
            sr += ar * br + ai * bi;
            si += ar * bi - ai * br;
        }
        part[c] = CMPLX(sr, si);
    }
    ocplx s = 0.0;
    for (int64_t c = 0; c < nc; c++) s += part[c];
    free(part);
    return s;
}

static double sum_real(int64_t n, const double* a) {
    const int64_t nc = (n + CHUNK - 1) / CHUNK;
    double* part = (double*)malloc(sizeof(double) * (size_t)(nc > 0 ? nc : 1));
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nc; c++) {
        const int64_t e = (c + 1) * CHUNK < n ? (c + 1) * CHUNK : n;
        double s = 0.0;
        for (int64_t i = c * CHUNK; i < e; i++) s += a[i];
        part[c] = s;
    }
    double s = 0.0;
    for (int64_t c = 0; c < nc; c++) s += part[c];
    free(part);
    return s;
}

static double sum_sq_real(int64_t n, const double* a) {
    const int64_t nc = (n + CHUNK - 1) / CHUNK;
    double* part = (double*)malloc(sizeof(double) * (size_t)(nc > 0 ? nc : 1));
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nc; c++) {
        const int64_t e = (c + 1) * CHUNK < n ? (c + 1) * CHUNK : n;
        double s = 0.0;
        for (int64_t i = c * CHUNK; i < e; i++) s += a[i] * a[i];
        part[c] = s;
    }
    double s = 0.0;
    for (int64_t c = 0; c < nc; c++) s += part[c];
    free(part);
    return s;
}

static inline int64_t vol(const o_latt* p) { return (int64_t)p->L1 * p->L2; }

static ocplx* cnew(int64_t n) { return (ocplx*)calloc((size_t)n, sizeof(ocplx)); }
static double* dnew(int64_t n) { return (double*)calloc((size_t)n, sizeof(double)); }

/* ------------------------------------------------------------------------- */
/* Gauge kernels: src/QED2dAction.jl */

/* plaquette P(x) = U1(x) U2(x+1) conj(U1(x+2) U2(x)) -- src/QED2dAction.jl:8-11 */
static inline ocplx plaq_at(const ocplx* U, int L1, int L2, int i1, int i2) {
    const int64_t V = (int64_t)L1 * L2;
    const int iu1 = (i1 + 1) % L1, iu2 = (i2 + 1) % L2;
    return U[i1 + (int64_t)L1 * i2] * U[V + iu1 + (int64_t)L1 * i2] *
           conj(U[i1 + (int64_t)L1 * iu2] * U[V + i1 + (int64_t)L1 * i2]);
}

/* plaquette! -- src/QED2dAction.jl:2-16 */
void o_plaquette_field(const o_latt* p, double* plx, const ocplx* U) {
#pragma omp parallel for schedule(static)
    for (int i2 = 0; i2 < p->L2; i2++)
        for (int i1 = 0; i1 < p->L1; i1++)
            plx[i1 + (int64_t)p->L1 * i2] = creal(plaq_at(U, p->L1, p->L2, i1, i2));
}

/* qtop! -- src/QED2dAction.jl:18-32 (CUDA.angle == carg) */
void o_qtop_field(const o_latt* p, double* plx, const ocplx* U) {
#pragma omp parallel for schedule(static)
    for (int i2 = 0; i2 < p->L2; i2++)
        for (int i1 = 0; i1 < p->L1; i1++)
            plx[i1 + (int64_t)p->L1 * i2] = carg(plaq_at(U, p->L1, p->L2, i1, i2));
}

/* krnl_force! -- src/QED2dAction.jl:34-53.  Two output buffers: every element of
 * frc1 and of frc2 is written exactly once. */
void o_gauge_force(const o_latt* p, double* frc1, double* frc2, const ocplx* U) {
    const int L1 = p->L1, L2 = p->L2;
    const int64_t V = vol(p);
#pragma omp parallel for schedule(static)
    for (int i2 = 0; i2 < L2; i2++)
        for (int i1 = 0; i1 < L1; i1++) {
            const int iu1 = (i1 + 1) % L1, iu2 = (i2 + 1) % L2;
            const double v = p->beta * cimag(plaq_at(U, L1, L2, i1, i2));
            frc1[i1 + (int64_t)L1 * i2] = -v;
            frc1[V + i1 + (int64_t)L1 * i2] = v;
            frc2[V + iu1 + (int64_t)L1 * i2] = -v;
            frc2[i1 + (int64_t)L1 * iu2] = v;
        }
}

/* updt_fld! -- src/QED2dAction.jl:55-65 */
void o_update_links(const o_latt* p, ocplx* U, const double* mom, double eps) {
    const int64_t n = 2 * vol(p);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        const double a = eps * mom[i];
        U[i] = CMPLX(cos(a), sin(a)) * U[i];
    }
}

/* ------------------------------------------------------------------------- */
/* Dirac operator: src/QED2dDirac.jl */

/* gamm5Dw -- src/QED2dDirac.jl:2-33, periodic in both directions (:7-11) */
void o_g5dw(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0) {
    const int L1 = p->L1, L2 = p->L2;
    const int64_t V = vol(p);
    const ocplx *U1 = U, *U2 = U + V, *s1 = si, *s2 = si + V;
#pragma omp parallel for schedule(static)
    for (int i2 = 0; i2 < L2; i2++) {
        const int iu2 = (i2 + 1) % L2, id2 = (i2 + L2 - 1) % L2;
        for (int i1 = 0; i1 < L1; i1++) {
            const int iu1 = (i1 + 1) % L1, id1 = (i1 + L1 - 1) % L1;
            const int64_t x = i1 + (int64_t)L1 * i2;
            const int64_t xp1 = iu1 + (int64_t)L1 * i2, xm1 = id1 + (int64_t)L1 * i2;
            const int64_t xp2 = i1 + (int64_t)L1 * iu2, xm2 = i1 + (int64_t)L1 * id2;
            const ocplx A = 0.5 * (U1[x] * (s1[xp1] - s2[xp1]) + conj(U1[xm1]) * (s1[xm1] + s2[xm1]));
            const ocplx B = 0.5 * (U2[x] * (s1[xp2] + mul_i(s2[xp2])) +
                                   conj(U2[xm2]) * (s1[xm2] - mul_i(s2[xm2])));
            const ocplx A2 = 0.5 * (U1[x] * (s1[xp1] - s2[xp1]) - conj(U1[xm1]) * (s1[xm1] + s2[xm1]));
            const ocplx B2 = 0.5 * (U2[x] * (-s2[xp2] + mul_i(s1[xp2])) -
                                    conj(U2[xm2]) * (s2[xm2] + mul_i(s1[xm2])));
            so[x] = (2.0 + am0) * s1[x] - A - B;
            so[V + x] = -(2.0 + am0) * s2[x] - A2 - B2;
        }
    }
}

/* gamm5 -- src/QED2dDirac.jl:130-146 */
void o_g5(const o_latt* p, ocplx* so, const ocplx* si) {
    const int64_t V = vol(p);
    for (int64_t x = 0; x < V; x++) {
        so[x] = si[x];
        so[V + x] = -si[V + x];
    }
}

/* Dw = g5 (g5 Dw) -- src/QED2dDirac.jl:157-169 */
void o_dw(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0) {
    const int64_t V = vol(p);
    ocplx* tmp = cnew(2 * V);
    o_g5dw(p, so, U, si, am0);
    memcpy(tmp, so, sizeof(ocplx) * 2 * V);
    o_g5(p, so, tmp);
    free(tmp);
}

/* gamm5Dw_sqr -- src/QED2dDirac.jl:35-46 (also gamm5Dw_sqr_msq, :69-81, which
 * despite its name adds no mass term) */
void o_g5dw_sqr(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0) {
    const int64_t V = vol(p);
    ocplx* tmp = cnew(2 * V);
    o_g5dw(p, tmp, U, si, am0);
    o_g5dw(p, so, U, tmp, am0);
    free(tmp);
}

/* gamm5Dw_sqr_sqr -- src/QED2dDirac.jl:48-67 */
void o_g5dw_sqr_sqr(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0) {
    const int64_t V = vol(p);
    ocplx* t1 = cnew(2 * V);
    ocplx* t2 = cnew(2 * V);
    o_g5dw(p, t1, U, si, am0);
    o_g5dw(p, t2, U, t1, am0);
    o_g5dw(p, t1, U, t2, am0);
    o_g5dw(p, so, U, t1, am0);
    free(t1);
    free(t2);
}

/* gamm5Dw_sqr_musq -- src/QED2dDirac.jl:83-95: so = (g5Dw)^2 si + mu^2 si */
void o_g5dw_sqr_musq(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0, double mu) {
    const int64_t n = 2 * vol(p);
    o_g5dw_sqr(p, so, U, si, am0);
    const double m2 = mu * mu;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) so[i] = so[i] + m2 * si[i];
}

/* gamm5Dw_sqr_sqr_musq -- src/QED2dDirac.jl:97-117 */
void o_g5dw_sqr_sqr_musq(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0, double mu) {
    const int64_t n = 2 * vol(p);
    o_g5dw_sqr_sqr(p, so, U, si, am0);
    const double m2 = mu * mu;
    for (int64_t i = 0; i < n; i++) so[i] = so[i] + m2 * si[i];
}

/* tr_dQwdU -- src/QED2dDirac.jl:172-199 */
void o_fermion_force(const o_latt* p, double* frc, const ocplx* U, const ocplx* X, const ocplx* G) {
    const int L1 = p->L1, L2 = p->L2;
    const int64_t V = vol(p);
    const ocplx *U1 = U, *U2 = U + V, *X1 = X, *X2 = X + V, *G1 = G, *G2 = G + V;
#pragma omp parallel for schedule(static)
    for (int i2 = 0; i2 < L2; i2++) {
        const int iu2 = (i2 + 1) % L2;
        for (int i1 = 0; i1 < L1; i1++) {
            const int iu1 = (i1 + 1) % L1;
            const int64_t x = i1 + (int64_t)L1 * i2;
            const int64_t xp1 = iu1 + (int64_t)L1 * i2, xp2 = i1 + (int64_t)L1 * iu2;
            const ocplx z1 =
                conj(U1[x]) * (conj(X1[xp1]) * (G1[x] + G2[x]) - conj(X2[xp1]) * (G1[x] + G2[x])) -
                U1[x] * (conj(X1[x]) * (G1[xp1] - G2[xp1]) + conj(X2[x]) * (G1[xp1] - G2[xp1]));
            const ocplx z2 =
                conj(U2[x]) * (conj(X1[xp2]) * (G1[x] - mul_i(G2[x])) - conj(X2[xp2]) * (mul_i(G1[x]) + G2[x])) -
                U2[x] * (conj(X1[x]) * (G1[xp2] + mul_i(G2[xp2])) + conj(X2[x]) * (mul_i(G1[xp2]) - G2[xp2]));
            frc[x] = creal(mul_i(z1));
            frc[V + x] = creal(mul_i(z2));
        }
    }
}

/* krnl_unfold! / krnl_reflect! -- src/QED2dFields.jl:2-50.  Uout is 2L1 x 2L2. */
void o_unfold(int L1old, int L2old, ocplx* Uout, const ocplx* Uin, int reflect) {
    const int64_t Vin = (int64_t)L1old * L2old;
    const int L1n = 2 * L1old, L2n = 2 * L2old;
    const int64_t Vout = (int64_t)L1n * L2n;
    for (int mu = 0; mu < 2; mu++)
        for (int i2 = 0; i2 < L2old; i2++)
            for (int i1 = 0; i1 < L1old; i1++) {
                const ocplx u = Uin[i1 + (int64_t)L1old * i2 + Vin * mu];
                const ocplx uc = reflect ? conj(u) : u;
                Uout[i1 + (int64_t)L1n * i2 + Vout * mu] = u;
                Uout[i1 + L1old + (int64_t)L1n * i2 + Vout * mu] = uc;
                Uout[i1 + (int64_t)L1n * (i2 + L2old) + Vout * mu] = uc;
                Uout[i1 + L1old + (int64_t)L1n * (i2 + L2old) + Vout * mu] = u;
            }
}

/* plwv -- src/QED2dUtils.jl:2-11 (i1-1, i2-1 there are the 0-based i1, i2 here) */
void o_plane_wave(const o_latt* p, ocplx* so, double k1, double k2) {
    const int64_t V = vol(p);
    const double s1 = sin(k1), s2 = sin(k2);
    const ocplx root = csqrt(CMPLX(-s1 * s1 - s2 * s2, 0.0));
    const ocplx pref = cdiv(mul_i(root), CMPLX(s1, s2));
    for (int i2 = 0; i2 < p->L2; i2++)
        for (int i1 = 0; i1 < p->L1; i1++) {
            const double ph = k1 * i1 + k2 * i2;
            const ocplx e = cexp(CMPLX(0.0, ph));
            so[i1 + (int64_t)p->L1 * i2] = pref * e;
            so[V + i1 + (int64_t)p->L1 * i2] = e;
        }
}

/* ------------------------------------------------------------------------- */
/* Observables: src/QED2dHMC.jl:198-237 */

double o_action(const o_latt* p, const ocplx* U) {
    const int64_t V = vol(p);
    double* plx = dnew(V);
    o_plaquette_field(p, plx, U);
    const double s = p->beta * ((double)V - sum_real(V, plx));
    free(plx);
    return s;
}

double o_plaquette(const o_latt* p, const ocplx* U) {
    const int64_t V = vol(p);
    double* plx = dnew(V);
    o_plaquette_field(p, plx, U);
    const double s = sum_real(V, plx) / (double)V;
    free(plx);
    return s;
}

double o_qtop(const o_latt* p, const ocplx* U) {
    const int64_t V = vol(p);
    double* plx = dnew(V);
    o_qtop_field(p, plx, U);
    const double s = sum_real(V, plx) / (2.0 * M_PI);
    free(plx);
    return s;
}

double o_hamiltonian(const o_latt* p, const double* mom, const ocplx* U) {
    return sum_sq_real(2 * vol(p), mom) / 2.0 + o_action(p, U);
}

/* ------------------------------------------------------------------------- */
/* CG: src/QED2dSolver.jl.  op == O_OP_SQR is method 1 (:3-46) with the operator
 * gamm5Dw_sqr_msq; op == O_OP_SQR_MUSQ is method 2 (:49-105) with
 * gamm5Dw_sqr_musq and shift mu, optionally warm-started from `so`. */
static void apply_op(const o_latt* p, int op, ocplx* so, const ocplx* U, const ocplx* si, double am0, double mu) {
    if (op == O_OP_SQR) o_g5dw_sqr(p, so, U, si, am0);
    else o_g5dw_sqr_musq(p, so, U, si, am0, mu);
}

int o_cg(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0, double mu, int op,
         int maxiter, double eps, int so_as_guess, int* iters, double* final_err) {
    const int64_t n = 2 * vol(p);
    if (iters) *iters = 0;
    const double bb = o_norm2(n, si);
    if (bb == 0.0) {   /* documented deviation: zero source -> zero solution */
        memset(so, 0, sizeof(ocplx) * n);
        if (final_err) *final_err = 0.0;
        return O_OK;
    }
    ocplx* r = cnew(n);
    ocplx* pp = cnew(n);
    ocplx* Ap = cnew(n);
    double tol = eps * bb, norm;
    if (!(so_as_guess && op == O_OP_SQR_MUSQ)) {
        memset(so, 0, sizeof(ocplx) * n);
        memcpy(r, si, sizeof(ocplx) * n);
        memcpy(pp, si, sizeof(ocplx) * n);
        norm = bb;
    } else {
        apply_op(p, op, Ap, U, so, am0, mu);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; i++) { r[i] = si[i] - Ap[i]; pp[i] = r[i]; }
        norm = o_norm2(n, r);
        if (norm < tol) {
            if (final_err) *final_err = norm;
            free(r); free(pp); free(Ap);
            return O_OK;
        }
    }
    double err = 0.0;
    int iterations = 0;
    for (int it = 1; it <= maxiter; it++) {
        apply_op(p, op, Ap, U, pp, am0, mu);
        const ocplx prod = o_dot(n, pp, Ap);
        const ocplx alpha = cdiv(norm, prod);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; i++) {
            so[i] = so[i] + alpha * pp[i];
            r[i] = r[i] - alpha * Ap[i];
        }
        err = o_norm2(n, r);
        if (err < tol) { iterations = it; break; }
        const double beta = err / norm;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; i++) pp[i] = r[i] + beta * pp[i];
        norm = err;
    }
    free(r); free(pp); free(Ap);
    if (final_err) *final_err = err;
    if (err > tol) { if (iters) *iters = maxiter; return O_NOT_CONVERGED; }
    if (iters) *iters = iterations;
    return O_OK;
}

/* MultiCG -- src/QED2dRHMC.jl:281-290 */
int o_multi_cg(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0,
               int maxiter, double eps, const o_rhmc* r, int* iters) {
    const int64_t n = 2 * vol(p);
    ocplx* aux = cnew(n);
    memcpy(so, si, sizeof(ocplx) * n);
    int total = 0, st = O_OK;
    for (int j = 0; j < r->n && st == O_OK; j++) {
        int it = 0;
        st = o_cg(p, aux, U, si, am0, r->mu[j], O_OP_SQR_MUSQ, maxiter, eps, 0, &it, NULL);
        total += it;
        for (int64_t i = 0; i < n; i++) so[i] = so[i] + r->rho[j] * aux[i];
    }
    free(aux);
    if (iters) *iters = total;
    return st;
}

/* R -- src/QED2dRHMC.jl:261-271 */
int o_rational(const o_latt* p, ocplx* so, const ocplx* U, const ocplx* si, double am0,
               int maxiter, double eps, const o_rhmc* r, int* iters) {
    const int64_t n = 2 * vol(p);
    const int st = o_multi_cg(p, so, U, si, am0, maxiter, eps, r, iters);
    const double c = pow(r->r_b, -1.0) * r->A;
    for (int64_t i = 0; i < n; i++) so[i] = c * so[i];
    return st;
}

/* ------------------------------------------------------------------------- */
/* Zolotarev coefficients: src/QED2dRHMC.jl:1-121.  The reference evaluates K, sn
 * and cn with Elliptic.jl 1.0.1 (parameter convention m = k^2).  Restated here
 * from the arithmetic-geometric mean: K(m) = pi / (2 AGM(1, sqrt(1-m))), and sn,
 * cn by the descending Landen / AGM scheme of Abramowitz & Stegun 16.4. */
double o_ellip_K(double m) {
    double a = 1.0, b = sqrt(1.0 - m);
    for (int i = 0; i < 64 && fabs(a - b) > 1e-17 * a; i++) {
        const double an = 0.5 * (a + b);
        b = sqrt(a * b);
        a = an;
    }
    return M_PI / (a + b);
}

void o_ellip_sncn(double u, double m, double* sn, double* cn) {
    double a[64], c[64];
    double aa = 1.0, bb = sqrt(1.0 - m), cc = sqrt(m);
    int N = 0;
    a[0] = aa; c[0] = cc;
    while (fabs(cc) > 1e-17 * aa && N < 62) {
        const double an = 0.5 * (aa + bb);
        const double bn = sqrt(aa * bb);
        cc = 0.5 * (aa - bb);
        aa = an; bb = bn;
        N++;
        a[N] = aa; c[N] = cc;
    }
    double phi = ldexp(a[N] * u, N);
    for (int k = N; k >= 1; k--) phi = 0.5 * (phi + asin(c[k] / a[k] * sin(phi)));
    *sn = sin(phi);
    *cn = cos(phi);
}

static double zk(double eps) { return sqrt(1.0 - eps); }                              /* :2 */
static double zv(int n, double eps) { const double k = zk(eps); return o_ellip_K(k * k) / (2.0 * n + 1.0); } /* :3 */
static double za_r(int r, int n, double eps) {                                         /* :4 */
    const double k = zk(eps);
    double s, c;
    o_ellip_sncn(r * zv(n, eps), k * k, &s, &c);
    return (c * c) / (s * s);
}
static double zc_r(int r, int n, double eps) {                                         /* :5 */
    const double k = zk(eps);
    double s, c;
    o_ellip_sncn(r * zv(n, eps), k * k, &s, &c);
    return s * s;
}
static double zmu(int j, int n, double eps, double r_b) { return r_b * sqrt(za_r(2 * j, n, eps)); }     /* :8 */
static double znu(int j, int n, double eps, double r_b) { return r_b * sqrt(za_r(2 * j - 1, n, eps)); } /* :9 */
static double zrho_mu(int j, int n, double eps, double r_b) {                          /* :11-25 */
    const double muj = zmu(j, n, eps, r_b), nuj = znu(j, n, eps, r_b);
    double res = nuj * nuj - muj * muj;
    for (int m = 1; m <= n; m++)
        if (m != j) {
            const double num = znu(m, n, eps, r_b), mum = zmu(m, n, eps, r_b);
            res *= (num * num - muj * muj) / (mum * mum - muj * muj);
        }
    return res;
}
static double zd(int n, double eps) {                                                  /* :60-68 */
    double res = pow(zk(eps), 2 * n + 1);
    for (int i = 1; i <= 2 * n + 1; i += 2) { const double c = zc_r(i, n, eps); res *= c * c; }
    return res;
}
static double zdelta(int n, double eps) {                                              /* :70 */
    const double d = zd(n, eps);
    const double den = 1.0 + sqrt(1.0 - d * d);
    return d * d / (den * den);
}
static double zA(int n, double eps) {                                                  /* :72-84 */
    const double d = zd(n, eps);
    double res = 2.0 / (1.0 + sqrt(1.0 - d * d));
    for (int i = 1; i <= 2 * n - 1; i += 2) res *= zc_r(i, n, eps);
    for (int i = 2; i <= 2 * n; i += 2) res *= 1.0 / zc_r(i, n, eps);
    return res;
}

/* get_rhmc_params (scalar method) -- src/QED2dRHMC.jl:93-110 */
int o_zolotarev(int n, double r_a, double r_b, o_rhmc* out) {
    if (n < 1 || n > O_MAXPOLES || !(r_a > 0.0) || !(r_b > r_a)) return O_BAD_ARG;
    memset(out, 0, sizeof(*out));
    const double eps = (r_a / r_b) * (r_a / r_b);
    out->r_b = r_b;
    out->n = n;
    out->eps = eps;
    out->A = zA(n, eps);
    out->delta = zdelta(n, eps);
    for (int j = 1; j <= n; j++) {
        out->mu[j - 1] = zmu(j, n, eps, r_b);
        out->nu[j - 1] = znu(j, n, eps, r_b);
        out->rho[j - 1] = zrho_mu(j, n, eps, r_b);
    }
    out->reweighting_N = 1;
    out->reweighting_Taylor = 5;
    return O_OK;
}

/* generate_pseudofermion! -- src/QED2dRHMC.jl:298-319 */
int o_pf_generate(const o_latt* p, ocplx* F, const ocplx* U, const ocplx* X, double am0,
                  int maxiter, double tol, const o_rhmc* r, int* iters) {
    const int64_t n = 2 * vol(p);
    ocplx* aux = cnew(n);
    memcpy(F, X, sizeof(ocplx) * n);
    int total = 0, st = O_OK;
    for (int i = 0; i < r->n && st == O_OK; i++) {
        memcpy(aux, F, sizeof(ocplx) * n);
        o_g5dw(p, F, U, aux, am0);
        for (int64_t k = 0; k < n; k++) F[k] = F[k] + CMPLX(0.0, r->mu[i]) * aux[k];
        memcpy(aux, F, sizeof(ocplx) * n);
        int it = 0;
        st = o_cg(p, F, U, aux, am0, r->nu[i], O_OP_SQR_MUSQ, maxiter, tol, 0, &it, NULL);
        total += it;
        memcpy(aux, F, sizeof(ocplx) * n);
        o_g5dw(p, F, U, aux, am0);
        for (int64_t k = 0; k < n; k++) F[k] = F[k] - CMPLX(0.0, r->nu[i]) * aux[k];
    }
    free(aux);
    if (iters) *iters = total;
    return st;
}

/* power_method -- src/QED2dRHMC.jl:135-170 (start vector b0 injected; second
 * loop applied out of place, see the header comment) */
void o_power_method(const o_latt* p, const ocplx* U, double am0, int iter, const ocplx* b0,
                    double* lmin, double* lmax) {
    const int64_t n = 2 * vol(p);
    ocplx* b = cnew(n);
    ocplx* aux = cnew(n);
    ocplx* bl = cnew(n);
    const double shift = 2.0;
    memcpy(b, b0, sizeof(ocplx) * n);
    for (int it = 0; it < iter; it++) {
        o_g5dw_sqr(p, aux, U, b, am0);
        for (int64_t i = 0; i < n; i++) aux[i] = aux[i] + shift * b[i];
        const double nn = creal(o_dot(n, aux, aux));
        for (int64_t i = 0; i < n; i++) b[i] = aux[i] / nn;
    }
    o_g5dw_sqr(p, aux, U, b, am0);
    for (int64_t i = 0; i < n; i++) aux[i] = aux[i] + shift * b[i];
    const ocplx lmx = cdiv(o_dot(n, b, aux), o_dot(n, b, b)) - shift;
    for (int it = 0; it < iter; it++) {
        memcpy(bl, b, sizeof(ocplx) * n);
        o_g5dw_sqr(p, b, U, bl, am0);
        for (int64_t i = 0; i < n; i++) b[i] = b[i] - lmx * bl[i];
        const double nn = creal(o_dot(n, b, b));
        for (int64_t i = 0; i < n; i++) b[i] = b[i] / nn;
    }
    o_g5dw_sqr(p, aux, U, b, am0);
    for (int64_t i = 0; i < n; i++) aux[i] = aux[i] - lmx * b[i];
    const ocplx lmn = cdiv(o_dot(n, b, aux), o_dot(n, b, b)) + lmx;
    *lmax = creal(lmx);
    *lmin = creal(lmn);
    free(b); free(aux); free(bl);
}

/* LuscherZ -- src/QED2dRHMC.jl:174-186: Z = ((g5Dw)^2 R^2 - 1) Xin */
int o_luscher_z(const o_latt* p, ocplx* Z, const ocplx* U, const ocplx* Xin, double am0,
                int maxiter, double tol, const o_rhmc* r) {
    const int64_t n = 2 * vol(p);
    ocplx* tmp = cnew(n);
    int st = o_rational(p, Z, U, Xin, am0, maxiter, tol, r, NULL);
    memcpy(tmp, Z, sizeof(ocplx) * n);
    if (st == O_OK) st = o_rational(p, Z, U, tmp, am0, maxiter, tol, r, NULL);
    memcpy(tmp, Z, sizeof(ocplx) * n);
    o_g5dw(p, Z, U, tmp, am0);
    memcpy(tmp, Z, sizeof(ocplx) * n);
    o_g5dw(p, Z, U, tmp, am0);
    for (int64_t i = 0; i < n; i++) Z[i] = Z[i] - Xin[i];
    free(tmp);
    return st;
}

/* reweighting_factor -- src/QED2dRHMC.jl:210-239.  `noise` holds
 * r->reweighting_N complex fields (the reference's X draws, :218). */
int o_reweighting_factor(const o_latt* p, const ocplx* U, double am0, int maxiter, double tol,
                         const o_rhmc* r, const ocplx* noise, double* W) {
    const int64_t n = 2 * vol(p);
    ocplx* Z = cnew(n);
    ocplx* tmp = cnew(n);
    double WN = 0.0;
    int st = O_OK;
    for (int j = 0; j < r->reweighting_N && st == O_OK; j++) {
        const ocplx* X = noise + (int64_t)j * n;
        double argexp = 0.0, Tfactor = 0.5;
        memcpy(tmp, X, sizeof(ocplx) * n);
        double fact_i = 1.0;   /* i! */
        for (int i = 1; i <= r->reweighting_Taylor && st == O_OK; i++) {
            st = o_luscher_z(p, Z, U, tmp, am0, maxiter, tol, r);
            argexp += Tfactor * creal(o_dot(n, X, Z));
            const double fact_ip1 = fact_i * (double)(i + 1);
            Tfactor *= (double)(-(2 * i + 1)) / 2.0 / fact_ip1 * fact_i;
            fact_i = fact_ip1;
            memcpy(tmp, Z, sizeof(ocplx) * n);
        }
        WN += exp(argexp) / (double)r->reweighting_N;
    }
    free(Z); free(tmp);
    *W = WN;
    return st;
}

/* ------------------------------------------------------------------------- */
/* Integrators: src/QED2dHMC.jl */

static const double OMF4_R1 = 0.08398315262876693;
static const double OMF4_R2 = 0.2539785108410595;
static const double OMF4_R3 = 0.6822365335719091;
static const double OMF4_R4 = -0.03230286765269967;

/* mom += c * (frc1 + frc2 [+ frc]) */
static void mom_add(int64_t n, double* mom, double c, const double* f1, const double* f2, const double* f) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) mom[i] = mom[i] + c * (f ? (f1[i] + f2[i]) + f[i] : f1[i] + f2[i]);
}

/* OMF4! pure gauge -- src/QED2dHMC.jl:239-305 */
void o_omf4_gauge(const o_latt* p, double* mom, ocplx* U, double eps, int ns) {
    const int64_t n = 2 * vol(p);
    const double r1 = OMF4_R1, r2 = OMF4_R2, r3 = OMF4_R3, r4 = OMF4_R4;
    const double r5 = 0.5 - r1 - r3, r6 = 1.0 - 2.0 * (r2 + r4);
    double* f1 = dnew(n);
    double* f2 = dnew(n);
    const double cm[6] = {r1, r3, r5, r5, r3, r1};
    const double cu[5] = {r2, r4, r6, r4, r2};
    for (int i = 0; i < ns; i++)
        for (int s = 0; s < 6; s++) {
            o_gauge_force(p, f1, f2, U);
            mom_add(n, mom, cm[s] * eps, f1, f2, NULL);
            if (s < 5) o_update_links(p, U, mom, eps * cu[s]);
        }
    free(f1); free(f2);
}

/* leapfrog for pure gauge: the reference defines MD!(Leapfrog, ...) only with
 * fermions (src/QED2dHMC.jl:5-16); this is the same kick-drift-kick scheme with
 * the gauge force alone (src/QED2dHMC.jl:426-449 without the CG). */
static void o_leapfrog_gauge(const o_latt* p, double* mom, ocplx* U, double eps, int ns) {
    const int64_t n = 2 * vol(p);
    double* f1 = dnew(n);
    double* f2 = dnew(n);
    o_gauge_force(p, f1, f2, U);
    mom_add(n, mom, 0.5 * eps, f1, f2, NULL);
    for (int i = 0; i < ns - 1; i++) {
        o_update_links(p, U, mom, eps);
        o_gauge_force(p, f1, f2, U);
        mom_add(n, mom, eps, f1, f2, NULL);
    }
    o_update_links(p, U, mom, eps);
    o_gauge_force(p, f1, f2, U);
    mom_add(n, mom, 0.5 * eps, f1, f2, NULL);
    free(f1); free(f2);
}

/* fermion + gauge force and momentum kick for Nf=2 -- src/QED2dHMC.jl:452-481 */
int o_update_momenta_nf2(const o_latt* p, double* mom, const ocplx* U, ocplx* X, const ocplx* F,
                         ocplx* g5DX, double am0, double eps, int maxiter, double tol, int* iters) {
    const int64_t n = 2 * vol(p);
    double* f1 = dnew(n);
    double* f2 = dnew(n);
    double* f = dnew(n);
    int it = 0;
    const int st = o_cg(p, X, U, F, am0, 0.0, O_OP_SQR, maxiter, tol, 0, &it, NULL);
    if (iters) *iters += it;
    o_g5dw(p, g5DX, U, X, am0);
    o_fermion_force(p, f, U, X, g5DX);
    o_gauge_force(p, f1, f2, U);
    mom_add(n, mom, eps, f1, f2, f);
    free(f1); free(f2); free(f);
    return st;
}

/* leapfrog! Nf=2 -- src/QED2dHMC.jl:426-449 */
int o_leapfrog_nf2(const o_latt* p, double* mom, ocplx* U, ocplx* X, const ocplx* F, ocplx* g5DX,
                   double am0, double eps, int ns, int maxiter, double tol, int* iters) {
    int st = o_update_momenta_nf2(p, mom, U, X, F, g5DX, am0, 0.5 * eps, maxiter, tol, iters);
    for (int i = 0; i < ns - 1 && st == O_OK; i++) {
        o_update_links(p, U, mom, eps);
        st = o_update_momenta_nf2(p, mom, U, X, F, g5DX, am0, eps, maxiter, tol, iters);
    }
    if (st != O_OK) return st;
    o_update_links(p, U, mom, eps);
    return o_update_momenta_nf2(p, mom, U, X, F, g5DX, am0, 0.5 * eps, maxiter, tol, iters);
}

/* OMF4! Nf=2 -- src/QED2dHMC.jl:307-422 */
int o_omf4_nf2(const o_latt* p, double* mom, ocplx* U, ocplx* X, const ocplx* F, ocplx* g5DX,
               double am0, double eps, int ns, int maxiter, double tol, int* iters) {
    const double r1 = OMF4_R1, r2 = OMF4_R2, r3 = OMF4_R3, r4 = OMF4_R4;
    const double r5 = 0.5 - r1 - r3, r6 = 1.0 - 2.0 * (r2 + r4);
    const double cm[6] = {r1, r3, r5, r5, r3, r1};
    const double cu[5] = {r2, r4, r6, r4, r2};
    int st = O_OK;
    for (int i = 0; i < ns && st == O_OK; i++)
        for (int s = 0; s < 6 && st == O_OK; s++) {
            st = o_update_momenta_nf2(p, mom, U, X, F, g5DX, am0, cm[s] * eps, maxiter, tol, iters);
            if (s < 5) o_update_links(p, U, mom, eps * cu[s]);
        }
    return st;
}

/* update_momenta! RHMC -- src/QED2dHMC.jl:516-557 */
int o_update_momenta_rhmc(const o_latt* p, double* mom, const ocplx* U, ocplx* X, ocplx* const* F,
                          ocplx* g5DX, int nf, const double* am0, double eps, int maxiter, double tol,
                          const o_rhmc* r, int* iters) {
    const int64_t n = 2 * vol(p);
    double* f1 = dnew(n);
    double* f2 = dnew(n);
    double* fi = dnew(n);
    double* f = dnew(n);
    int st = O_OK, guess = 0;
    for (int j = 0; j < nf && st == O_OK; j++) {
        for (int i = 0; i < r[j].n && st == O_OK; i++) {
            int it = 0;
            st = o_cg(p, X, U, F[j], am0[j], r[j].mu[i], O_OP_SQR_MUSQ, maxiter, tol, guess, &it, NULL);
            if (iters) *iters += it;
            guess = 1;
            o_g5dw(p, g5DX, U, X, am0[j]);
            o_fermion_force(p, fi, U, X, g5DX);
            for (int64_t k = 0; k < n; k++) f[k] = f[k] + r[j].rho[i] * fi[k];
        }
        guess = 0;
    }
    o_gauge_force(p, f1, f2, U);
    mom_add(n, mom, eps, f1, f2, f);
    free(f1); free(f2); free(fi); free(f);
    return st;
}

/* leapfrog! RHMC -- src/QED2dHMC.jl:485-513 */
int o_leapfrog_rhmc(const o_latt* p, double* mom, ocplx* U, ocplx* X, ocplx* const* F, ocplx* g5DX,
                    int nf, const double* am0, double eps, int ns, int maxiter, double tol,
                    const o_rhmc* r, int* iters) {
    int st = o_update_momenta_rhmc(p, mom, U, X, F, g5DX, nf, am0, 0.5 * eps, maxiter, tol, r, iters);
    for (int i = 0; i < ns - 1 && st == O_OK; i++) {
        o_update_links(p, U, mom, eps);
        st = o_update_momenta_rhmc(p, mom, U, X, F, g5DX, nf, am0, eps, maxiter, tol, r, iters);
    }
    if (st != O_OK) return st;
    o_update_links(p, U, mom, eps);
    return o_update_momenta_rhmc(p, mom, U, X, F, g5DX, nf, am0, 0.5 * eps, maxiter, tol, r, iters);
}

/* ------------------------------------------------------------------------- */
/* HMC steps: src/QED2dHMC.jl:19-195.  Metropolis as in :31-51. */
static int metropolis(const o_latt* p, const ocplx* U, int qzero, double hini, double hfin, double r_unif) {
    double pacc;
    if (qzero && fabs(o_qtop(p, U)) > 0.1) pacc = 0.0;
    else pacc = exp(-(hfin - hini));
    if (pacc < 1.0) return pacc > r_unif ? 1 : 0;
    return 1;
}

int o_hmc_gauge(const o_latt* p, ocplx* U, double eps, int ns, int integrator, int qzero,
                const double* mom0, double r_unif, int* accepted, double* hini, double* hfin) {
    const int64_t n = 2 * vol(p);
    ocplx* Ucp = cnew(n);
    double* mom = dnew(n);
    memcpy(Ucp, U, sizeof(ocplx) * n);
    memcpy(mom, mom0, sizeof(double) * n);
    *hini = o_hamiltonian(p, mom, U);
    if (integrator == O_OMF4) o_omf4_gauge(p, mom, U, eps, ns);
    else o_leapfrog_gauge(p, mom, U, eps, ns);
    *hfin = o_hamiltonian(p, mom, U);
    *accepted = metropolis(p, U, qzero, *hini, *hfin, r_unif);
    if (!*accepted) memcpy(U, Ucp, sizeof(ocplx) * n);
    free(Ucp); free(mom);
    return O_OK;
}

int o_hmc_nf2(const o_latt* p, ocplx* U, double am0, double eps, int ns, int integrator,
              int maxiter, double tol, int qzero, const double* mom0, const ocplx* noise,
              double r_unif, int* accepted, double* hini, double* hfin, int* iters) {
    const int64_t n = 2 * vol(p);
    ocplx* Ucp = cnew(n);
    double* mom = dnew(n);
    ocplx* X = cnew(n);
    ocplx* F = cnew(n);
    ocplx* g5DX = cnew(n);
    memcpy(Ucp, U, sizeof(ocplx) * n);
    memcpy(mom, mom0, sizeof(double) * n);
    memcpy(X, noise, sizeof(ocplx) * n);
    if (iters) *iters = 0;
    *hini = creal(o_hamiltonian(p, mom, U) + o_dot(n, X, X));
    o_g5dw(p, F, U, X, am0);
    int st;
    if (integrator == O_OMF4) st = o_omf4_nf2(p, mom, U, X, F, g5DX, am0, eps, ns, maxiter, tol, iters);
    else st = o_leapfrog_nf2(p, mom, U, X, F, g5DX, am0, eps, ns, maxiter, tol, iters);
    *hfin = creal(o_hamiltonian(p, mom, U) + o_dot(n, X, F));
    if (st == O_OK) *accepted = metropolis(p, U, qzero, *hini, *hfin, r_unif);
    else *accepted = 0;
    if (!*accepted) memcpy(U, Ucp, sizeof(ocplx) * n);
    free(Ucp); free(mom); free(X); free(F); free(g5DX);
    return st;
}

int o_hmc_rhmc(const o_latt* p, ocplx* U, int nf, const double* am0, double eps, int ns,
               int maxiter, double tol, const o_rhmc* r, int qzero, int reversibility,
               const double* mom0, const ocplx* noise, double r_unif,
               int* accepted, double* hini, double* hfin, int* iters) {
    const int64_t n = 2 * vol(p);
    ocplx* Ucp = cnew(n);
    double* mom = dnew(n);
    ocplx* X = cnew(n);
    ocplx* g5DX = cnew(n);
    ocplx** F = (ocplx**)malloc(sizeof(ocplx*) * (size_t)nf);
    memcpy(Ucp, U, sizeof(ocplx) * n);
    memcpy(mom, mom0, sizeof(double) * n);
    if (iters) *iters = 0;
    *hini = o_hamiltonian(p, mom, U);
    int st = O_OK;
    for (int j = 0; j < nf; j++) {
        memcpy(X, noise + (int64_t)j * n, sizeof(ocplx) * n);
        *hini += o_norm2(n, X);
        F[j] = cnew(n);
        int it = 0;
        if (st == O_OK) st = o_pf_generate(p, F[j], U, X, am0[j], maxiter, tol, &r[j], &it);
        if (iters) *iters += it;
    }
    if (st == O_OK) st = o_leapfrog_rhmc(p, mom, U, X, F, g5DX, nf, am0, eps, ns, maxiter, tol, r, iters);
    *hfin = o_hamiltonian(p, mom, U);
    for (int j = 0; j < nf && st == O_OK; j++) {
        int it = 0;
        st = o_multi_cg(p, X, U, F[j], am0[j], maxiter, tol, &r[j], &it);
        if (iters) *iters += it;
        *hfin += creal(o_dot(n, X, F[j]));
    }
    if (reversibility) {
        for (int64_t i = 0; i < n; i++) mom[i] = -mom[i];
        if (st == O_OK) st = o_leapfrog_rhmc(p, mom, U, X, F, g5DX, nf, am0, eps, ns, maxiter, tol, r, iters);
        *accepted = 1;
    } else {
        if (st == O_OK) *accepted = metropolis(p, U, qzero, *hini, *hfin, r_unif);
        else *accepted = 0;
        if (!*accepted) memcpy(U, Ucp, sizeof(ocplx) * n);
    }
    for (int j = 0; j < nf; j++) free(F[j]);
    free(F); free(Ucp); free(mom); free(X); free(g5DX);
    return st;
}
