// cg.cu -- conjugate-gradient solvers of libqed2d on the Hermitian positive
// operator A + mu^2, A = (g5 Dw)^2 (gamm5Dw_sqr_msq / gamm5Dw_sqr_musq of
// src/QED2dDirac.jl:69-95).
//
// QED2D_PREC_F64 and QED2D_PREC_MIXED run a whole solve as ONE persistent
// cooperative launch: every block owns a fixed set of 32x8 tiles, the two
// reductions of an iteration go through per-block partials summed in a fixed
// order by every block (deterministic, no host round trip), and phases are
// separated by a bounded grid barrier.  Per iteration:
//   phase A:  p = r + beta p_old (evaluated on load, at the 5 stencil points),
//             t = g5Dw p, store p and t,  partial <p,Ap> = |t|^2 + mu^2 |p|^2
//   phase B:  Ap = g5Dw t + mu^2 p, x += alpha p, r -= alpha Ap, partial |r|^2
// (g5Dw is Hermitian, so <p, (g5Dw)^2 p> = |g5Dw p|^2.)  The stop rule is the
// reference's: |r|^2 < eps |b|^2 (src/QED2dSolver.jl:13-29).
//
// QED2D_PREC_MIXED runs phases A/B in FP32 on packed float4 fields with FP64
// partial sums, and replaces the residual by the FP64 true residual
// b - (A + mu^2) x (reliable update) whenever the FP32 residual has dropped by
// delta^2 since the last update, or looks converged; it stops only when the FP64
// true residual meets the reference's tolerance.  FP32 fields are kept at unit
// norm (rescaled at every update), so tiny right-hand sides cannot underflow.
//
// QED2D_PREC_PLAIN mirrors the reference's own structure (src/QED2dSolver.jl):
// unfused kernels and two device-to-host reads per iteration.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "stencil.cuh"

namespace qed2d {

constexpr int kMaxShifts = QED2D_MAXPOLES;

struct CGP {
    Lat g;
    const double2* U;
    const float4* U32;
    const double2* b;
    double2* x;
    double2* r;      // FP64 residual (planes)
    double2* p0;     // FP64 search directions (double buffer)
    double2* p1;
    double2* t;      // FP64 g5Dw p  (mixed: g5Dw x at reliable updates)
    float4* r32;
    float4* q0;      // FP32 search directions (double buffer)
    float4* q1;
    float4* t32;
    float4* x32;
    double2* g5x;    // optional output g5Dw x (F64 path)
    double m2;       // 2 + m0
    double mu2;
    double eps;
    double delta2;   // reliable-update threshold delta^2 (mixed)
    int maxiter;
    int guess;
    int per_block;   // tiles per block (a contiguous range)
    DevCtl* ctl;
    double* part;
};

__device__ __forceinline__ void write_partials(double* part, const double* v, int nv) {
    if (threadIdx.x == 0)
        for (int k = 0; k < nv; k++) part[(size_t)k * kMaxPartBlocks + blockIdx.x] = v[k];
}

// RS = 2: the whole solve runs in ONE thread-block cluster (at most 16 blocks,
// small lattices).  The hardware cluster barrier (barrier.cluster arrive with
// release, wait with acquire) orders the blocks' memory accesses at cluster
// scope, so no atomics, polling or error flag are needed.  Every block computes
// the same reductions from the same partials in the same order, so all blocks
// take the same path and reach the same barriers.
struct ClusterSync {
    int nred = 0;
    __device__ __forceinline__ bool sync() {
        cooperative_groups::this_cluster().sync();
        return true;
    }
};
template <int RS>
struct SyncOf {
    using type = GridSync;
};
template <>
struct SyncOf<2> {
    using type = ClusterSync;
};
template <int RS>
__device__ __forceinline__ typename SyncOf<RS>::type make_sync(DevCtl* c) {
    if constexpr (RS == 2) return ClusterSync{};
    else return GridSync{&c->bar, &c->gen, &c->err};
}

// Grid-wide sum of NV values (NV <= 4), deterministic: every block writes its
// partials and arrives at a bounded grid barrier; the partials are summed in a
// fixed order (thread t takes partials t, t+blockDim, ..., then a fixed-shape
// tree).  Two schedules give the same bits:
//   RS = 0: the last block to arrive sums them, publishes the sums in red[]
//           and releases; every block then reads red[] (one more round trip);
//   RS = 1: counter barrier, then every block sums all partials itself (no
//           second round trip, more L2 reads).
// Which one is faster depends on the lattice size; the context tunes it.
// Partials and sums alternate between two buffers: reduction n+2 overwrites
// buffer n's only after every block has passed barrier n+1, i.e. has read the
// results of n.  (The error flag is read once per barrier: a status kept in
// shared memory instead made these kernels spill, 7% slower at 2048^2.)
template <int NV, int RS, class S>
__device__ __forceinline__ bool reduce_sync(S& gs, double (&v)[NV], double* part_base, double* red_base,
                                            double* smem) {
    static_assert(NV <= kMaxPartVals / 2, "too many values for the double-buffered partials");
    __shared__ int s_last;
    const int buf = gs.nred++ & 1;
    double* part = part_base + (size_t)buf * (kMaxPartVals / 2) * kMaxPartBlocks;
    block_sum<NV>(v, smem);
    write_partials(part, v, NV);
    if constexpr (RS == 2) {   // cluster barrier, then every block sums the partials (as RS = 1)
        gs.sync();
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double s = 0.0;
            for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x)
                s += __ldcg(part + (size_t)k * kMaxPartBlocks + i);
            v[k] = s;
        }
        block_sum<NV>(v, smem);
        __shared__ double s_v2[4];
        if (threadIdx.x == 0)
#pragma unroll
            for (int k = 0; k < NV; k++) s_v2[k] = v[k];
        __syncthreads();
#pragma unroll
        for (int k = 0; k < NV; k++) v[k] = s_v2[k];
        return true;
    } else if constexpr (RS == 0) {
        const bool last = gs.arrive(&s_last);
        double* red = red_base + buf * 4;
        if (last) {
            double w[NV];
#pragma unroll
            for (int k = 0; k < NV; k++) {
                double s = 0.0;
                for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x)
                    s += __ldcg(part + (size_t)k * kMaxPartBlocks + i);
                w[k] = s;
            }
            block_sum<NV>(w, smem);
            if (threadIdx.x == 0) {
#pragma unroll
                for (int k = 0; k < NV; k++) red[k] = w[k];
                gs.release();
            }
        } else if (threadIdx.x == 0) {
            gs.wait();
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < NV; k++) v[k] = __ldcg(red + k);
        return ld_volatile_int(gs.err) == 0;
    } else {
        gs.count_sync();
        const bool ok = ld_volatile_int(gs.err) == 0;   // issued together with the partial loads
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double s = 0.0;
            for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x)
                s += __ldcg(part + (size_t)k * kMaxPartBlocks + i);
            v[k] = s;
        }
        block_sum<NV>(v, smem);
        __shared__ double s_v[4];
        if (threadIdx.x == 0)
#pragma unroll
            for (int k = 0; k < NV; k++) s_v[k] = v[k];
        __syncthreads();
#pragma unroll
        for (int k = 0; k < NV; k++) v[k] = s_v[k];
        return ok;
    }
}

__device__ __forceinline__ void finish_solve(const CGP& P, int iters, bool conv, double rr, double bb,
                                             int updates = 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        DevCtl* c = P.ctl;
        const int err = ld_volatile_int(&c->err);
        c->last_iters = iters;
        c->last_updates = updates;
        c->last_conv = conv && !err;
        c->last_relres = bb > 0.0 ? rr / bb : 0.0;
        c->iters_total += iters;
        if (c->status == 0) {
            if (err) c->status = QED2D_ERR_TIMEOUT;
            else if (!conv) c->status = QED2D_ERR_NOT_CONVERGED;
        }
    }
}

#define FOR_TILES(q) FOR_RANGE(q, P.g, TR)

// ---------------------------------------------------------------------------
// FP64 persistent CG
template <int RS>
__global__ void __launch_bounds__(TILE, 3) k_cg_f64(const CGP P) {
    __shared__ double smem[32 * 2];
    auto gs = make_sync<RS>(P.ctl);
    const long long ntiles = num_tiles(P.g), V = P.g.V;
    const TileRange TR = tile_range(ntiles, (P.g.L1 + TX - 1) / TX, P.per_block, blockIdx.x);
    const LkD L{P.U, V};
    const double m2 = P.m2, mu2 = P.mu2;
    int k = 0;
    bool conv = false;
    double rr = 0.0, bb = 0.0;

    // setup: |b|^2, and x = 0 / r = b, or t = g5Dw x for a warm start
    {
        double v[1] = {0.0};
        FOR_TILES(q) {
            const Pair<double> bv{__ldg(P.b + q.x), __ldg(P.b + q.x + V)};
            v[0] += norm2(bv.a) + norm2(bv.b);
            if (!P.guess) {
                st_d(P.x, V, q.x, Pair<double>{make_double2(0, 0), make_double2(0, 0)});
                st_d(P.r, V, q.x, bv);
            } else {
                st_d(P.t, V, q.x, g5dw_at<double>(SpD{P.x, V}, L, q, m2));
            }
        }
        if (!reduce_sync<1, RS>(gs, v, P.part, P.ctl->red, smem)) goto done;
        bb = v[0];
    }
    if (bb == 0.0) {   // zero source: zero solution
        if (P.guess) FOR_TILES(q) st_d(P.x, V, q.x, Pair<double>{make_double2(0, 0), make_double2(0, 0)});
        conv = true;
        if (!gs.sync()) goto done;
        goto epilogue;
    }
    {
        const double tol = P.eps * bb;
        if (P.guess) {
            double v[1] = {0.0};
            FOR_TILES(q) {
                const Pair<double> xc = SpD{P.x, V}.ld(q.x);
                const Pair<double> a = g5dw_at<double>(SpD{P.t, V}, L, q, m2);
                Pair<double> r;
                r.a = __ldg(P.b + q.x) - (a.a + mu2 * xc.a);
                r.b = __ldg(P.b + q.x + V) - (a.b + mu2 * xc.b);
                st_d(P.r, V, q.x, r);
                v[0] += norm2(r.a) + norm2(r.b);
            }
            if (!reduce_sync<1, RS>(gs, v, P.part, P.ctl->red, smem)) goto done;
            rr = v[0];
            if (rr < tol) { conv = true; goto epilogue; }
        } else {
            rr = bb;
        }
        double beta = 0.0;
        // x += alpha p every second iteration, for two directions at once (the
        // same operations in the same order, so the same bits); an update still
        // waiting when the loop ends is added after it.  Grid schedules only, as
        // in the mixed solver.
        constexpr bool kPair = RS != 2;
        bool pend = false;
        double apend = 0.0;
        const double2* plast = nullptr;   // the direction of the waiting update
        for (k = 1; k <= P.maxiter; k++) {
            double2* pn = (k & 1) ? P.p0 : P.p1;
            const double2* po = (k & 1) ? P.p1 : P.p0;
            const SpAxpy<double, SpD> Q{SpD{P.r, V}, SpD{po, V}, beta, k > 1};
            double v[1] = {0.0};
            FOR_TILES(q) {
                const Pair<double> c = Q.ld(q.x);
                const Pair<double> tt = g5dw_at_c<double>(Q, c, L, q, m2);
                st_d(pn, V, q.x, c);
                st_d(P.t, V, q.x, tt);
                v[0] += norm2(tt.a) + norm2(tt.b) + mu2 * (norm2(c.a) + norm2(c.b));
            }
            if (!reduce_sync<1, RS>(gs, v, P.part, P.ctl->red, smem)) goto done;
            const double alpha = rr / v[0];
            v[0] = 0.0;
            if (!kPair || pend) {
                FOR_TILES(q) {
                    const Pair<double> pc = SpD{pn, V}.ld(q.x);
                    const Pair<double> a = g5dw_at<double>(SpD{P.t, V}, L, q, m2);
                    Pair<double> xv = SpD{P.x, V}.ld(q.x), r = SpD{P.r, V}.ld(q.x);
                    if (kPair) {   // the previous iteration's update first
                        const Pair<double> pp = SpD{po, V}.ld(q.x);
                        xv.a = xv.a + apend * pp.a;
                        xv.b = xv.b + apend * pp.b;
                    }
                    xv.a = xv.a + alpha * pc.a;
                    xv.b = xv.b + alpha * pc.b;
                    r.a = r.a - alpha * (a.a + mu2 * pc.a);
                    r.b = r.b - alpha * (a.b + mu2 * pc.b);
                    st_d(P.x, V, q.x, xv);
                    st_d(P.r, V, q.x, r);
                    v[0] += norm2(r.a) + norm2(r.b);
                }
            } else {
                FOR_TILES(q) {   // x's update waits for the next iteration
                    const Pair<double> pc = SpD{pn, V}.ld(q.x);
                    const Pair<double> a = g5dw_at<double>(SpD{P.t, V}, L, q, m2);
                    Pair<double> r = SpD{P.r, V}.ld(q.x);
                    r.a = r.a - alpha * (a.a + mu2 * pc.a);
                    r.b = r.b - alpha * (a.b + mu2 * pc.b);
                    st_d(P.r, V, q.x, r);
                    v[0] += norm2(r.a) + norm2(r.b);
                }
            }
            apend = alpha;
            plast = pn;
            pend = kPair && !pend;
            if (!reduce_sync<1, RS>(gs, v, P.part, P.ctl->red, smem)) goto done;
            const double rn = v[0];
            if (rn < tol) { rr = rn; conv = true; break; }
            beta = rn / rr;
            rr = rn;
        }
        if (!conv) k = P.maxiter;
        if (pend) {   // the update still waiting (each block its own sites)
            FOR_TILES(q) {
                const Pair<double> pc = SpD{plast, V}.ld(q.x);
                Pair<double> xv = SpD{P.x, V}.ld(q.x);
                xv.a = xv.a + apend * pc.a;
                xv.b = xv.b + apend * pc.b;
                st_d(P.x, V, q.x, xv);
            }
            if (P.g5x && !gs.sync()) goto done;   // the epilogue's stencil reads other blocks' x
        }
    }
epilogue:
    if (P.g5x) FOR_TILES(q) st_d(P.g5x, V, q.x, g5dw_at<double>(SpD{P.x, V}, L, q, m2));
done:
    finish_solve(P, k, conv, rr, bb);
}

// ---------------------------------------------------------------------------
// mixed FP32/FP64 reliable-update CG.  RL (schedules 4, 5, 6 = 0, 1, 2 with it):
// the first phase applies the stencil to r and carries t = g5Dw r + beta t_old
// (g5Dw is linear, so t = g5Dw p; p is formed at the site only), and the FP32
// links of the block's tiles are staged once per solve in shared memory
// (ULsm<TY>; dynamic shared memory of per_block tiles).  The same recurrences,
// with t rounded along its own recurrence, so results agree with the plain form
// to the solver's accuracy.
template <int RS, bool RL = false>
__global__ void __launch_bounds__(TILE, 4) k_cg_mixed(const CGP P) {
    extern __shared__ float2 lsm_dyn[];   // RL: ULsm<TY>::bytes(P.per_block)
    __shared__ double smem[32 * 2];
    auto gs = make_sync<RS>(P.ctl);
    const long long ntiles = num_tiles(P.g), V = P.g.V;
    const TileRange TR = tile_range(ntiles, (P.g.L1 + TX - 1) / TX, P.per_block, blockIdx.x);
    const LkD L{P.U, V};
    const LkF Lf{P.U32, P.g.V};
    const double m2 = P.m2, mu2 = P.mu2;
    const float m2f = (float)m2, mu2f = (float)mu2;
    double2* t64 = P.g5x ? P.g5x : P.t;
    int k = 0, nupd = 0;
    bool conv = false;
    double rr64 = 0.0, bb = 0.0;
    // the FP32 stencil of accessor S around site q of the block's tile j (centre c given)
    auto sten = [&](const auto& S, const Pair<float>& c, const Site& q, int j) -> Pair<float> {
        if constexpr (RL) return ULsm<TY>::stencil(lsm_dyn, j, S, c, q, m2f);
        else return g5dw_at_c<float>(S, c, Lf, q, m2f);
    };
    if constexpr (RL) {   // stage the links of the block's tiles
        FOR_TILES(q) ULsm<TY>::stage(lsm_dyn, tt_ - TR.lo, Lf, q);
        __syncthreads();
    }

    {
        double v[1] = {0.0};
        FOR_TILES(q) {
            const Pair<double> bv{__ldg(P.b + q.x), __ldg(P.b + q.x + V)};
            v[0] += norm2(bv.a) + norm2(bv.b);
            if (!P.guess) st_d(P.x, V, q.x, Pair<double>{make_double2(0, 0), make_double2(0, 0)});
            else st_d(t64, V, q.x, g5dw_at<double>(SpD{P.x, V}, L, q, m2));
        }
        if (!reduce_sync<1, RS>(gs, v, P.part, P.ctl->red, smem)) goto done;
        bb = v[0];
    }
    if (bb == 0.0) {
        FOR_TILES(q) {
            st_d(P.x, V, q.x, Pair<double>{make_double2(0, 0), make_double2(0, 0)});
            if (P.g5x) st_d(P.g5x, V, q.x, Pair<double>{make_double2(0, 0), make_double2(0, 0)});
        }
        conv = true;
        goto done;
    }
    {
        const double tol = P.eps * bb;
        if (P.guess) {
            double v[1] = {0.0};
            FOR_TILES(q) {
                const Pair<double> xc = SpD{P.x, V}.ld(q.x);
                const Pair<double> a = g5dw_at<double>(SpD{t64, V}, L, q, m2);
                Pair<double> r;
                r.a = __ldg(P.b + q.x) - (a.a + mu2 * xc.a);
                r.b = __ldg(P.b + q.x + V) - (a.b + mu2 * xc.b);
                st_d(P.r, V, q.x, r);
                v[0] += norm2(r.a) + norm2(r.b);
            }
            if (!reduce_sync<1, RS>(gs, v, P.part, P.ctl->red, smem)) goto done;
            rr64 = v[0];
            if (rr64 < tol) { conv = true; goto done; }
        } else {
            rr64 = bb;
        }
        const double2* rsrc = P.guess ? P.r : P.b;
        double s = 1.0 / sqrt(rr64);
        double rr;   // |r32|^2 at the start of the current iteration
        {
            double v[1] = {0.0};
            FOR_TILES(q) {
                const double2 a = rsrc[q.x], b2 = rsrc[q.x + V];
                const Pair<float> r32{to_f(s * a), to_f(s * b2)};
                st_f(P.r32, q.x, r32);
                st_f(P.x32, q.x, Pair<float>{make_float2(0, 0), make_float2(0, 0)});
                v[0] += (double)norm2(r32.a) + (double)norm2(r32.b);
            }
            if (!reduce_sync<1, RS>(gs, v, P.part, P.ctl->red, smem)) goto done;
            rr = v[0];
        }
        double maxrr = rr, beta = 0.0;
        bool first = true;
        int cur = 0;
        // x32 += alpha p every second iteration, for two directions at once (the
        // same operations in the same order, so the same bits): while `pend`, the
        // previous iteration's update (alpha apend, direction in qo) waits.  Grid
        // schedules only: per iteration 2048^2 161.9 -> 147.6 us, 512^2 equal,
        // while the one-cluster schedule (<= 128 tiles) lost 4% at 64^2.
        constexpr bool kPair = RS != 2;
        bool pend = false;
        float apend = 0.f;
        const bool shifted = mu2f != 0.f;   // without a shift, skipped iterations need no p
        for (k = 1; k <= P.maxiter; k++) {
            float4* qn = cur ? P.q1 : P.q0;
            const float4* qo = cur ? P.q0 : P.q1;
            float ft = 0.f, fc = 0.f;   // per-thread sums in FP32: one conversion per phase
            if constexpr (RL) {
                const float bf = (float)beta;
                FOR_TILES(q) {
                    const Pair<float> rc = SpF{P.r32}.ld(q.x);
                    Pair<float> tt = sten(SpF{P.r32}, rc, q, tt_ - TR.lo), c = rc;
                    if (!first) {   // p = r + beta p_old, t = g5Dw r + beta t_old
                        const Pair<float> po = SpF{qo}.ld(q.x), to = SpF{P.t32}.ld(q.x);
                        c.a = c.a + bf * po.a;
                        c.b = c.b + bf * po.b;
                        tt.a = tt.a + bf * to.a;
                        tt.b = tt.b + bf * to.b;
                    }
                    st_f(qn, q.x, c);
                    st_f(P.t32, q.x, tt);
                    ft += norm2(tt.a) + norm2(tt.b);
                    fc += norm2(c.a) + norm2(c.b);
                }
            } else {
                const SpAxpy<float, SpF> Q{SpF{P.r32}, SpF{qo}, (float)beta, !first};
                FOR_TILES(q) {
                    const Pair<float> c = Q.ld(q.x);
                    const Pair<float> tt = g5dw_at_c<float>(Q, c, Lf, q, m2f);
                    st_f(qn, q.x, c);
                    st_f(P.t32, q.x, tt);
                    ft += norm2(tt.a) + norm2(tt.b);
                    fc += norm2(c.a) + norm2(c.b);
                }
            }
            double v[1] = {(double)ft + mu2 * (double)fc};
            if (!reduce_sync<1, RS>(gs, v, P.part, P.ctl->red, smem)) goto done;
            const float alpha = (float)(rr / v[0]);
            float fr = 0.f;
            if (!kPair) {
                FOR_TILES(q) {
                    const Pair<float> pc = SpF{qn}.ld(q.x);
                    const Pair<float> a = sten(SpF{P.t32}, SpF{P.t32}.ld(q.x), q, tt_ - TR.lo);
                    Pair<float> xv = SpF{P.x32}.ld(q.x), r = SpF{P.r32}.ld(q.x);
                    xv.a = xv.a + alpha * pc.a;
                    xv.b = xv.b + alpha * pc.b;
                    r.a = r.a - alpha * (a.a + mu2f * pc.a);
                    r.b = r.b - alpha * (a.b + mu2f * pc.b);
                    st_f(P.x32, q.x, xv);
                    st_f(P.r32, q.x, r);
                    fr += norm2(r.a) + norm2(r.b);
                }
            } else if (pend) {
                FOR_TILES(q) {   // x += apend p_old, then x += alpha p
                    const Pair<float> po = SpF{qo}.ld(q.x), pc = SpF{qn}.ld(q.x);
                    const Pair<float> a = sten(SpF{P.t32}, SpF{P.t32}.ld(q.x), q, tt_ - TR.lo);
                    Pair<float> xv = SpF{P.x32}.ld(q.x), r = SpF{P.r32}.ld(q.x);
                    xv.a = xv.a + apend * po.a;
                    xv.b = xv.b + apend * po.b;
                    xv.a = xv.a + alpha * pc.a;
                    xv.b = xv.b + alpha * pc.b;
                    r.a = r.a - alpha * (a.a + mu2f * pc.a);
                    r.b = r.b - alpha * (a.b + mu2f * pc.b);
                    st_f(P.x32, q.x, xv);
                    st_f(P.r32, q.x, r);
                    fr += norm2(r.a) + norm2(r.b);
                }
            } else if (shifted) {
                FOR_TILES(q) {   // x's update waits for the next iteration
                    const Pair<float> pc = SpF{qn}.ld(q.x);
                    const Pair<float> a = sten(SpF{P.t32}, SpF{P.t32}.ld(q.x), q, tt_ - TR.lo);
                    Pair<float> r = SpF{P.r32}.ld(q.x);
                    r.a = r.a - alpha * (a.a + mu2f * pc.a);
                    r.b = r.b - alpha * (a.b + mu2f * pc.b);
                    st_f(P.r32, q.x, r);
                    fr += norm2(r.a) + norm2(r.b);
                }
            } else {
                FOR_TILES(q) {   // the same without a shift (a + 0 p = a exactly)
                    const Pair<float> a = sten(SpF{P.t32}, SpF{P.t32}.ld(q.x), q, tt_ - TR.lo);
                    Pair<float> r = SpF{P.r32}.ld(q.x);
                    r.a = r.a - alpha * a.a;
                    r.b = r.b - alpha * a.b;
                    st_f(P.r32, q.x, r);
                    fr += norm2(r.a) + norm2(r.b);
                }
            }
            apend = alpha;
            pend = kPair && !pend;
            v[0] = (double)fr;
            if (!reduce_sync<1, RS>(gs, v, P.part, P.ctl->red, smem)) goto done;
            const double rn = v[0];
            maxrr = fmax(maxrr, rn);
            const bool cand = rn < tol * s * s;
            if (rn < P.delta2 * maxrr || cand || k == P.maxiter) {
                // reliable update: x += x32 / s, then the FP64 true residual
                nupd++;
                const double inv_s = 1.0 / s;
                FOR_TILES(q) {   // with this iteration's x32 update if it waits
                    Pair<float> d = SpF{P.x32}.ld(q.x);
                    if (pend) {
                        const Pair<float> pc = SpF{qn}.ld(q.x);
                        d.a = d.a + apend * pc.a;
                        d.b = d.b + apend * pc.b;
                    }
                    Pair<double> xv = SpD{P.x, V}.ld(q.x);
                    xv.a = xv.a + inv_s * to_d(d.a);
                    xv.b = xv.b + inv_s * to_d(d.b);
                    st_d(P.x, V, q.x, xv);
                    st_f(P.x32, q.x, Pair<float>{make_float2(0, 0), make_float2(0, 0)});
                }
                pend = false;
                if (!gs.sync()) goto done;
                FOR_TILES(q) st_d(t64, V, q.x, g5dw_at<double>(SpD{P.x, V}, L, q, m2));
                if (!gs.sync()) goto done;
                double w[1] = {0.0};
                FOR_TILES(q) {
                    const Pair<double> xc = SpD{P.x, V}.ld(q.x);
                    const Pair<double> a = g5dw_at<double>(SpD{t64, V}, L, q, m2);
                    Pair<double> r;
                    r.a = __ldg(P.b + q.x) - (a.a + mu2 * xc.a);
                    r.b = __ldg(P.b + q.x + V) - (a.b + mu2 * xc.b);
                    st_d(P.r, V, q.x, r);
                    w[0] += norm2(r.a) + norm2(r.b);
                }
                if (!reduce_sync<1, RS>(gs, w, P.part, P.ctl->red, smem)) goto done;
                const double rrt = w[0];
                rr64 = rrt;
                if (rrt < tol) { conv = true; break; }
                if (k == P.maxiter) break;
                const double s_new = 1.0 / sqrt(rrt);
                w[0] = 0.0;
                FOR_TILES(q) {
                    const Pair<float> r32{to_f(s_new * P.r[q.x]), to_f(s_new * P.r[q.x + V])};
                    st_f(P.r32, q.x, r32);
                    w[0] += (double)(norm2(r32.a) + norm2(r32.b));
                }
                if (!reduce_sync<1, RS>(gs, w, P.part, P.ctl->red, smem)) goto done;
                beta = (rrt * s * s / rr) * (s_new / s);
                s = s_new;
                rr = w[0];
                maxrr = rr;
            } else {
                beta = rn / rr;
                rr = rn;
                rr64 = rn / (s * s);
            }
            first = false;
            cur ^= 1;
        }
        if (!conv) k = P.maxiter;
    }
done:
    finish_solve(P, k, conv, rr64, bb, nupd);
}

// ---------------------------------------------------------------------------
// FP64 multi-shift CG (one Krylov space for all shifts).  The base system is
// the smallest shift; shift i uses the collinear-residual recurrences
//   z_{k+1} = z_k z_{k-1} a_{k-1} / (a_k b_{k-1} (z_{k-1} - z_k) + z_{k-1} a_{k-1} (1 + d_i a_k))
//   a^i_k = a_k z_{k+1}/z_k,  b^i_k = b_k (z_{k+1}/z_k)^2,
//   x_i += a^i_k p_i,  p_i <- z_{k+1} r_{k+1} + b^i_k p_i
// (B. Jegerlehner, "Krylov space solvers for shifted linear systems",
// hep-lat/9612014), d_i = mu_i^2 - mu_base^2.  Shift i is frozen once
// |z|^2 |r|^2 < eps |b|^2; the x_i update of step k is applied in phase A of
// step k+1, before p_i is overwritten.
struct MSP {
    Lat g;
    const double2* U;
    const double2* b;
    double2* r;
    double2* p0;
    double2* p1;
    double2* t;
    double2* x[kMaxShifts];
    double2* ps[kMaxShifts];
    double d[kMaxShifts];
    int n;
    int base;
    double m2;
    double mu2b;
    double eps;
    int maxiter;
    int per_block;
    DevCtl* ctl;
    double* part;
};


// RS: the reduction schedules of reduce_sync (tuned per context as for cg_solve).
// Layout: tiles of 32 x TYv sites, S threads per site.  Group 0 of a block (its
// first 32 * TYv threads, one per site) runs the stencil phases and the base
// system; the shift updates of phase A, which read and write only the site's
// own values, are dealt over the groups: non-base shift j goes to group
// (j + 1) % S, so group 0, which also runs the stencil, gets the fewest (leaving
// it none measured slower with four groups: 128^2 8.30 -> 8.50 us per
// iteration).  With S = 1 and TYv = 8 this is one thread per site of a 32 x 8
// tile.  Layouts that
// split the lattice into the same blocks give the same bits (the extra groups
// add zeros to the block sums); otherwise the partial sums group differently.
template <int RS, int TYv, int S>
__global__ void __launch_bounds__(32 * TYv * S, TYv * S <= 8 ? 3 : 1) k_cg_multishift(const MSP P) {
    constexpr int TPB = 32 * TYv;   // threads of one group: one per site of a tile
    __shared__ double smem[32 * 2];
    __shared__ double z[kMaxShifts], zp[kMaxShifts], ai[kMaxShifts], bi[kMaxShifts];
    __shared__ int upd[kMaxShifts], act[kMaxShifts];
    auto gs = make_sync<RS>(P.ctl);
    const int nt1 = (P.g.L1 + TX - 1) / TX;
    const long long ntiles = (long long)nt1 * ((P.g.L2 + TYv - 1) / TYv), V = P.g.V;
    const TileRange TR = tile_range(ntiles, nt1, P.per_block, blockIdx.x);
    const int st = S == 1 ? (int)threadIdx.x : (int)threadIdx.x % TPB;
    const int grp = S == 1 ? 0 : (int)threadIdx.x / TPB;
    const int j0 = (grp + S - 1) % S;   // this group's first non-base shift
    const LkD L{P.U, V};
    const double m2 = P.m2, mu2 = P.mu2b;
    int k = 0;
    bool conv = false;
    double rr = 0.0, bb = 0.0;
#define FOR_MS_TILES(q)                                                                       \
    for (int tt_ = TR.lo, t1_ = TR.s1, t2_ = TR.s2; tt_ < TR.hi;                              \
         ++tt_, (++t1_ == TR.nt1 ? (t1_ = 0, ++t2_) : 0))                                       \
        if (const Site q = site_at_t<TYv>(P.g, t1_, t2_, st); q.ok)
#define FOR_MY_SHIFTS(i)                                                                      \
    for (int j_ = j0, i = j0 < P.base ? j0 : j0 + 1; j_ < P.n - 1;                            \
         j_ += S, i = j_ < P.base ? j_ : j_ + 1)
    if (threadIdx.x < kMaxShifts) {
        z[threadIdx.x] = 1.0; zp[threadIdx.x] = 1.0; ai[threadIdx.x] = 0.0; bi[threadIdx.x] = 0.0;
        upd[threadIdx.x] = 0; act[threadIdx.x] = threadIdx.x < P.n;
    }
    {
        double v[1] = {0.0};
        const Pair<double> zz{make_double2(0, 0), make_double2(0, 0)};
        FOR_MS_TILES(q) {
            if (grp == 0) {
                const Pair<double> bv{__ldg(P.b + q.x), __ldg(P.b + q.x + V)};
                v[0] += norm2(bv.a) + norm2(bv.b);
                st_d(P.r, V, q.x, bv);
                st_d(P.x[P.base], V, q.x, zz);
            }
            FOR_MY_SHIFTS(i) st_d(P.x[i], V, q.x, zz);
        }
        if (!reduce_sync<1, RS>(gs, v, P.part, P.ctl->red, smem)) goto done;
        bb = v[0];
    }
    if (bb == 0.0) { conv = true; goto done; }
    {
        const double tol = P.eps * bb;
        rr = bb;
        double beta = 0.0, alpha_prev = 1.0;
        for (k = 1; k <= P.maxiter; k++) {
            double2* pn = (k & 1) ? P.p0 : P.p1;
            const double2* po = (k & 1) ? P.p1 : P.p0;
            const SpAxpy<double, SpD> Q{SpD{P.r, V}, SpD{po, V}, beta, k > 1};
            double v[1] = {0.0};
            FOR_MS_TILES(q) {
                if (grp == 0) {
                    const Pair<double> c = Q.ld(q.x);
                    const Pair<double> tt = g5dw_at_c<double>(Q, c, L, q, m2);
                    st_d(pn, V, q.x, c);
                    st_d(P.t, V, q.x, tt);
                    v[0] += norm2(tt.a) + norm2(tt.b) + mu2 * (norm2(c.a) + norm2(c.b));
                }
                const Pair<double> rc = SpD{P.r, V}.ld(q.x);
                FOR_MY_SHIFTS(i) {
                    if (upd[i]) {   // x_i += a^i_{k-1} p_i^{k-1}
                        const Pair<double> pi = SpD{P.ps[i], V}.ld(q.x);
                        Pair<double> xi = SpD{P.x[i], V}.ld(q.x);
                        xi.a = xi.a + ai[i] * pi.a;
                        xi.b = xi.b + ai[i] * pi.b;
                        st_d(P.x[i], V, q.x, xi);
                        if (act[i]) {
                            Pair<double> pnew;
                            pnew.a = z[i] * rc.a + bi[i] * pi.a;
                            pnew.b = z[i] * rc.b + bi[i] * pi.b;
                            st_d(P.ps[i], V, q.x, pnew);
                        }
                    } else if (k == 1) {
                        st_d(P.ps[i], V, q.x, rc);
                    }
                }
            }
            if (!reduce_sync<1, RS>(gs, v, P.part, P.ctl->red, smem)) goto done;
            const double alpha = rr / v[0];
            v[0] = 0.0;
            if (grp == 0) FOR_MS_TILES(q) {
                    const Pair<double> pc = SpD{pn, V}.ld(q.x);
                    const Pair<double> a = g5dw_at<double>(SpD{P.t, V}, L, q, m2);
                    Pair<double> xb = SpD{P.x[P.base], V}.ld(q.x), r = SpD{P.r, V}.ld(q.x);
                    xb.a = xb.a + alpha * pc.a;
                    xb.b = xb.b + alpha * pc.b;
                    r.a = r.a - alpha * (a.a + mu2 * pc.a);
                    r.b = r.b - alpha * (a.b + mu2 * pc.b);
                    st_d(P.x[P.base], V, q.x, xb);
                    st_d(P.r, V, q.x, r);
                    v[0] += norm2(r.a) + norm2(r.b);
                }
            if (!reduce_sync<1, RS>(gs, v, P.part, P.ctl->red, smem)) goto done;
            const double rn = v[0];
            const double beta_new = rn / rr;
            // shift scalars (identical in every block)
            if (threadIdx.x < P.n && threadIdx.x != P.base) {
                const int i = threadIdx.x;
                if (act[i]) {
                    const double zk = z[i], zkm = zp[i];
                    const double znew = zk * zkm * alpha_prev /
                                        (alpha * beta * (zkm - zk) + zkm * alpha_prev * (1.0 + P.d[i] * alpha));
                    ai[i] = alpha * znew / zk;
                    bi[i] = beta_new * (znew / zk) * (znew / zk);
                    zp[i] = zk;
                    z[i] = znew;
                    upd[i] = 1;
                    if (znew * znew * rn < tol) act[i] = 0;
                } else {
                    upd[i] = 0;
                }
            }
            __syncthreads();
            alpha_prev = alpha;
            beta = beta_new;
            rr = rn;
            if (rn < tol) { conv = true; break; }
        }
        if (!conv) k = P.maxiter;
        // final x_i updates of the last step
        if (!gs.sync()) goto done;
        FOR_MS_TILES(q) {
            FOR_MY_SHIFTS(i) {
                if (!upd[i]) continue;
                const Pair<double> pi = SpD{P.ps[i], V}.ld(q.x);
                Pair<double> xi = SpD{P.x[i], V}.ld(q.x);
                xi.a = xi.a + ai[i] * pi.a;
                xi.b = xi.b + ai[i] * pi.b;
                st_d(P.x[i], V, q.x, xi);
            }
        }
    }
#undef FOR_MS_TILES
#undef FOR_MY_SHIFTS
done:
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        DevCtl* c = P.ctl;
        const int err = ld_volatile_int(&c->err);
        c->last_iters = k;
        c->last_updates = 0;
        c->last_conv = conv && !err;
        c->last_relres = bb > 0.0 ? rr / bb : 0.0;
        c->iters_total += k;
        if (c->status == 0) {
            if (err) c->status = QED2D_ERR_TIMEOUT;
            else if (!conv) c->status = QED2D_ERR_NOT_CONVERGED;
        }
    }
}

// ---------------------------------------------------------------------------
// FP32-inner multi-shift CG: the recurrences of k_cg_multishift (same shift
// scalars, computed in FP64) on FP32 vectors -- r, p, t, every shift's x and p
// packed as float4 per site, links in FP32 -- for a source normalised to unit
// norm.  It stops when |r|^2 < eps32 (relative to |b|^2), a residual FP32 can
// reach, and writes every shift's solution in FP64 planes, scaled back by |b|;
// the host then refines each shift with the mixed CG (warm start) to the
// caller's FP64 stop rule, so every shift meets the same bound as with the FP64
// multi-shift.
struct MSP32 {
    Lat g;
    const float4* U32;
    const double2* b;
    float4* r;
    float4* p0;
    float4* p1;
    float4* t;
    float4* x[kMaxShifts];
    float4* ps[kMaxShifts];
    double2* x64[kMaxShifts];
    double d[kMaxShifts];
    int n;
    int base;
    double m2;
    double mu2b;
    double eps32;
    int maxiter;
    int per_block;
    DevCtl* ctl;
    double* part;
};

template <int RS>
__global__ void __launch_bounds__(TILE, 3) k_cg_multishift32(const MSP32 P) {
    __shared__ double smem[32 * 2];
    __shared__ double z[kMaxShifts], zp[kMaxShifts], ai[kMaxShifts], bi[kMaxShifts];
    __shared__ int upd[kMaxShifts], act[kMaxShifts];
    auto gs = make_sync<RS>(P.ctl);
    const long long ntiles = num_tiles(P.g), V = P.g.V;
    const TileRange TR = tile_range(ntiles, (P.g.L1 + TX - 1) / TX, P.per_block, blockIdx.x);
    const LkF Lf{P.U32, P.g.V};
    const float m2f = (float)P.m2, mu2f = (float)P.mu2b;
    const Pair<float> zf{make_float2(0, 0), make_float2(0, 0)};
    int k = 0;
    bool conv = false;
    double rr = 0.0, bb = 0.0, scale = 1.0;
    if (threadIdx.x < kMaxShifts) {
        z[threadIdx.x] = 1.0; zp[threadIdx.x] = 1.0; ai[threadIdx.x] = 0.0; bi[threadIdx.x] = 0.0;
        upd[threadIdx.x] = 0; act[threadIdx.x] = threadIdx.x < P.n;
    }
    {   // |b|^2
        double v[1] = {0.0};
        FOR_TILES(q) {
            const Pair<double> bv{__ldg(P.b + q.x), __ldg(P.b + q.x + V)};
            v[0] += norm2(bv.a) + norm2(bv.b);
        }
        if (!reduce_sync<1, RS>(gs, v, P.part, P.ctl->red, smem)) goto done;
        bb = v[0];
    }
    if (bb == 0.0) {   // zero source: zero solutions
        FOR_TILES(q) for (int i = 0; i < P.n; i++) st_d(P.x64[i], V, q.x, Pair<double>{make_double2(0, 0), make_double2(0, 0)});
        conv = true;
        goto done;
    }
    {   // r = b / |b|, x_i = 0
        scale = 1.0 / sqrt(bb);
        double v[1] = {0.0};
        FOR_TILES(q) {
            const Pair<float> r{to_f(scale * __ldg(P.b + q.x)), to_f(scale * __ldg(P.b + q.x + V))};
            st_f(P.r, q.x, r);
            v[0] += (double)(norm2(r.a) + norm2(r.b));
            for (int i = 0; i < P.n; i++) st_f(P.x[i], q.x, zf);
        }
        if (!reduce_sync<1, RS>(gs, v, P.part, P.ctl->red, smem)) goto done;
        rr = v[0];
    }
    {
        const double tol = P.eps32 * rr;
        double beta = 0.0, alpha_prev = 1.0;
        for (k = 1; k <= P.maxiter; k++) {
            float4* pn = (k & 1) ? P.p0 : P.p1;
            const float4* po = (k & 1) ? P.p1 : P.p0;
            const SpAxpy<float, SpF> Q{SpF{P.r}, SpF{po}, (float)beta, k > 1};
            double v[1] = {0.0};
            FOR_TILES(q) {
                const Pair<float> c = Q.ld(q.x);
                const Pair<float> tt = g5dw_at_c<float>(Q, c, Lf, q, m2f);
                st_f(pn, q.x, c);
                st_f(P.t, q.x, tt);
                v[0] += (double)(norm2(tt.a) + norm2(tt.b) + mu2f * (norm2(c.a) + norm2(c.b)));
                const Pair<float> rc = SpF{P.r}.ld(q.x);
                for (int i = 0; i < P.n; i++) {
                    if (i == P.base) continue;
                    if (upd[i]) {   // x_i += a^i_{k-1} p_i^{k-1}
                        const Pair<float> pi = SpF{P.ps[i]}.ld(q.x);
                        Pair<float> xi = SpF{P.x[i]}.ld(q.x);
                        const float a = (float)ai[i];
                        xi.a = xi.a + a * pi.a;
                        xi.b = xi.b + a * pi.b;
                        st_f(P.x[i], q.x, xi);
                        if (act[i]) {
                            const float zi = (float)z[i], bs = (float)bi[i];
                            Pair<float> pnew;
                            pnew.a = zi * rc.a + bs * pi.a;
                            pnew.b = zi * rc.b + bs * pi.b;
                            st_f(P.ps[i], q.x, pnew);
                        }
                    } else if (k == 1) {
                        st_f(P.ps[i], q.x, rc);
                    }
                }
            }
            if (!reduce_sync<1, RS>(gs, v, P.part, P.ctl->red, smem)) goto done;
            const double alpha = rr / v[0];
            const float af = (float)alpha;
            v[0] = 0.0;
            FOR_TILES(q) {
                const Pair<float> pc = SpF{pn}.ld(q.x);
                const Pair<float> a = g5dw_at<float>(SpF{P.t}, Lf, q, m2f);
                Pair<float> xb = SpF{P.x[P.base]}.ld(q.x), r = SpF{P.r}.ld(q.x);
                xb.a = xb.a + af * pc.a;
                xb.b = xb.b + af * pc.b;
                r.a = r.a - af * (a.a + mu2f * pc.a);
                r.b = r.b - af * (a.b + mu2f * pc.b);
                st_f(P.x[P.base], q.x, xb);
                st_f(P.r, q.x, r);
                v[0] += (double)(norm2(r.a) + norm2(r.b));
            }
            if (!reduce_sync<1, RS>(gs, v, P.part, P.ctl->red, smem)) goto done;
            const double rn = v[0];
            const double beta_new = rn / rr;
            if (threadIdx.x < P.n && threadIdx.x != P.base) {
                const int i = threadIdx.x;
                if (act[i]) {
                    const double zk = z[i], zkm = zp[i];
                    const double znew = zk * zkm * alpha_prev /
                                        (alpha * beta * (zkm - zk) + zkm * alpha_prev * (1.0 + P.d[i] * alpha));
                    ai[i] = alpha * znew / zk;
                    bi[i] = beta_new * (znew / zk) * (znew / zk);
                    zp[i] = zk;
                    z[i] = znew;
                    upd[i] = 1;
                    if (znew * znew * rn < tol) act[i] = 0;
                } else {
                    upd[i] = 0;
                }
            }
            __syncthreads();
            alpha_prev = alpha;
            beta = beta_new;
            rr = rn;
            if (rn < tol) { conv = true; break; }
        }
        if (!conv) k = P.maxiter;
        if (!gs.sync()) goto done;
        // the last x_i updates, then every solution to FP64, scaled back by |b|
        const double inv = 1.0 / scale;
        FOR_TILES(q) {
            for (int i = 0; i < P.n; i++) {
                Pair<float> xi = SpF{P.x[i]}.ld(q.x);
                if (i != P.base && upd[i]) {
                    const Pair<float> pi = SpF{P.ps[i]}.ld(q.x);
                    const float a = (float)ai[i];
                    xi.a = xi.a + a * pi.a;
                    xi.b = xi.b + a * pi.b;
                }
                st_d(P.x64[i], V, q.x, Pair<double>{make_double2(inv * xi.a.x, inv * xi.a.y),
                                                     make_double2(inv * xi.b.x, inv * xi.b.y)});
            }
        }
    }
done:
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        DevCtl* c = P.ctl;
        const int err = ld_volatile_int(&c->err);
        c->last_iters = k;
        c->last_updates = 0;
        c->last_conv = conv && !err;
        c->last_relres = rr;
        c->iters_total += k;
        if (c->status == 0 && err) c->status = QED2D_ERR_TIMEOUT;
    }
}

// ---------------------------------------------------------------------------
// host side
static_assert(offsetof(DevCtl, gen) == sizeof(unsigned long long) &&
                  offsetof(DevCtl, err) == 2 * sizeof(unsigned long long),
              "reset_barrier zeroes bar, gen and err as one range");

// Cooperative grid: at most the co-resident limit, then as few blocks as give
// every block the same number of tiles (fewer arrivals per barrier, no tail).
template <class K>
static int coop_grid(Ctx& c, K kernel, int* grid, int threads = TILE, long long nt = -1) {
    if (nt < 0) nt = num_tiles(c.g);
    int per_sm = 0;
    QCHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0));
    if (per_sm < 1) return QED2D_ERR_UNSUPPORTED;
    long long g = (long long)per_sm * c.num_sms;
    if (g > kMaxPartBlocks) g = kMaxPartBlocks;
    const long long per_block = (nt + g - 1) / g;
    g = (nt + per_block - 1) / per_block;
    *grid = (int)g;
    return QED2D_OK;
}

static int reset_barrier(Ctx& c) {   // bar, gen and err are contiguous
    QCHECK(cudaMemsetAsync(&c.ctl->bar, 0, 2 * sizeof(unsigned long long) + sizeof(int), c.stream));
    return QED2D_OK;
}

// Self-test of the bounded barrier wait: thread 0 of a one-block launch arrives
// at a barrier of two members whose second never comes and polls with the
// caller's (small) limit, so the wait gives up exactly as a persistent kernel's
// barrier does when a block never arrives: QED2D_ERR_TIMEOUT in err and status.
__global__ void k_barrier_timeout_probe(DevCtl* c, unsigned long long limit) {
    if (threadIdx.x != 0) return;
    GridSync gs{&c->bar, &c->gen, &c->err, 2u};
    gs.target = 2;
    red_release_add_u64(gs.arrivals, 1ULL);
    if (!gs.poll(gs.arrivals, limit) && c->status == 0)
        c->status = ld_volatile_int(&c->err) ? QED2D_ERR_TIMEOUT : QED2D_ERR_CUDA;
}

int barrier_timeout_probe(Ctx& c, long long polls) {
    QTRY(reset_barrier(c));
    k_barrier_timeout_probe<<<1, 32, 0, c.stream>>>(c.ctl, (unsigned long long)polls);
    count_launch();
    QCHECK(cudaGetLastError());
    return QED2D_OK;
}

template <class K, class Par>
static int launch_coop(Ctx& c, K kernel, Par P, int threads = TILE, long long nt = -1) {
    if (nt < 0) nt = num_tiles(c.g);
    int grid = 0;
    QTRY(coop_grid(c, kernel, &grid, threads, nt));
    P.per_block = (int)((nt + grid - 1) / grid);
    QTRY(reset_barrier(c));
    void* args[] = {(void*)&P};
    QCHECK(cudaLaunchCooperativeKernel((const void*)kernel, dim3(grid), dim3(threads), args, 0, c.stream));
    count_launch();
    return QED2D_OK;
}

static int solve_plain(Ctx& c, const SolveArgs& a);

// One-cluster launch (RS = 2): grid = cluster = min(tiles, 16) blocks, each a
// contiguous range of tiles.  Only for lattices of at most kClusterTiles tiles;
// returns QED2D_ERR_UNSUPPORTED when no such cluster fits on the device.
constexpr int kClusterTiles = 128;

// (threads: block size; nt: the lattice's tiles in the kernel's tile shape)
template <class K>
static int cluster_grid(Ctx& c, K kernel, int* grid, int threads = TILE, long long nt = -1) {
    if (nt < 0) nt = num_tiles(c.g);
    if (nt > kClusterTiles) return QED2D_ERR_UNSUPPORTED;
    int g = (int)std::min<long long>(nt, 16);
    if (g > 8 && cudaFuncSetAttribute((const void*)kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                     cudaSuccess) {
        cudaGetLastError();
        g = 8;
    }
    for (; g >= 1; g /= 2) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(g);
        cfg.blockDim = dim3(threads);
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = g;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, (const void*)kernel, &cfg) == cudaSuccess && n >= 1) {
            *grid = g;
            return QED2D_OK;
        }
        cudaGetLastError();
        if (g == 1) break;
    }
    return QED2D_ERR_UNSUPPORTED;
}

template <class Par>
static int launch_cluster(Ctx& c, void (*kernel)(Par), Par P, int threads = TILE, long long nt = -1) {
    if (nt < 0) nt = num_tiles(c.g);
    int grid = 0;
    QTRY(cluster_grid(c, kernel, &grid, threads, nt));
    P.per_block = (int)((nt + grid - 1) / grid);
    grid = (int)((nt + P.per_block - 1) / P.per_block);   // no block without tiles
    QTRY(reset_barrier(c));   // no barrier here, but the epilogue reads err: clear one a timeout left
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(threads);
    cfg.stream = c.stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = grid;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    QCHECK(cudaLaunchKernelEx(&cfg, kernel, P));
    count_launch();
    return QED2D_OK;
}

// The mixed solver's RL form (schedules 4, 5, 6): the reduction schedule rs =
// 0, 1 (cooperative grid) or 2 (one cluster) with the links of every block's
// tiles in dynamic shared memory.  The geometry is the plain form's; the launch
// is refused (QED2D_ERR_UNSUPPORTED, nothing enqueued) when the blocks of that
// geometry are not co-resident with the staged links.
static int launch_mixed_rl(Ctx& c, const CGP& P0, int rs) {
    void (*kern)(CGP) = rs == 2 ? k_cg_mixed<2, true> : rs ? k_cg_mixed<1, true> : k_cg_mixed<0, true>;
    const long long nt = num_tiles(c.g);
    int grid = 0;
    if (rs == 2) QTRY(cluster_grid(c, kern, &grid));
    else QTRY(coop_grid(c, kern, &grid));
    CGP P = P0;
    P.per_block = (int)((nt + grid - 1) / grid);
    grid = (int)((nt + P.per_block - 1) / P.per_block);
    const size_t sm = ULsm<TY>::bytes(P.per_block);
    int optin = 0;
    cudaFuncAttributes fa{};
    QCHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.device));
    QCHECK(cudaFuncGetAttributes(&fa, (const void*)kern));
    if (sm + fa.sharedSizeBytes > (size_t)optin) return QED2D_ERR_UNSUPPORTED;
    QCHECK(cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                optin - (int)fa.sharedSizeBytes));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(TILE);
    cfg.dynamicSmemBytes = sm;
    cfg.stream = c.stream;
    cudaLaunchAttribute at[1];
    if (rs == 2) {
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = grid;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        int n = 0;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        if (cudaOccupancyMaxActiveClusters(&n, (const void*)kern, &cfg) != cudaSuccess || n < 1) {
            cudaGetLastError();
            return QED2D_ERR_UNSUPPORTED;
        }
    } else {
        int n = 0;
        QCHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, (const void*)kern, TILE, sm));
        if ((long long)n * c.num_sms < grid) return QED2D_ERR_UNSUPPORTED;
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
    }
    QTRY(reset_barrier(c));
    QCHECK(cudaLaunchKernelEx(&cfg, kern, P));
    count_launch();
    return QED2D_OK;
}

// the solver of precision slot (0 = F64, 1 = MIXED) under schedule rs (the
// mixed solver's 4, 5, 6: its RL form under 0, 1, 2)
static int launch_cg(Ctx& c, const CGP& P, int slot, int rs) {
    if (slot == 0) {
        if (rs == 2) return launch_cluster(c, k_cg_f64<2>, P);
        return launch_coop(c, rs ? k_cg_f64<1> : k_cg_f64<0>, P);
    }
    if (rs >= 4) return launch_mixed_rl(c, P, rs - 4);
    if (rs == 2) return launch_cluster(c, k_cg_mixed<2>, P);
    return launch_coop(c, rs ? k_cg_mixed<1> : k_cg_mixed<0>, P);
}

static bool cluster_possible(Ctx& c, int slot) {
    int g = 0;
    return (slot == 0 ? cluster_grid(c, k_cg_f64<2>, &g) : cluster_grid(c, k_cg_mixed<2>, &g)) == QED2D_OK;
}

// Schedule tuning.  The grid reduction schedules RS = 0 and RS = 1 give the same
// bits.  RS = 2 (one cluster, tried only for lattices that fit one) runs fewer
// blocks than the cooperative grid, so its partial sums are grouped differently
// and its results agree with the others only to the solver's accuracy; exact-bit
// comparisons must fix the schedule.  The first solve of each
// precision on a context times both on the caller's operator and source,
// capped at kTuneIters iterations, into scratch outputs, and keeps the faster;
// the device control block is saved before and restored after, so counters and
// status are those of the caller's solves alone.  With QED2D_TUNE=0 in the
// environment the choice is the size rule measured on B200 instead: every
// block sums (RS = 1) up to 2^20 sites, the last block publishes beyond.
constexpr int kTuneIters = 24;
constexpr long long kMs32Sites = 1LL << 22;   // lattices from 2048^2 on: FP32-inner multishift (schedule 3)

bool tuning_enabled() {
    const char* e = std::getenv("QED2D_TUNE");
    return !(e && e[0] == '0');
}

// Times every candidate schedule (3 rounds, the first warms up) and returns the
// fastest in *best; a candidate whose launch is refused with
// QED2D_ERR_UNSUPPORTED (a cluster or staged links that do not fit) is dropped.
template <class Launch>
static int time_schedules(Ctx& c, Launch launch, const std::vector<int>& cand, int* best) {
    cudaEvent_t e0, e1;
    QCHECK(cudaEventCreate(&e0));
    QCHECK(cudaEventCreate(&e1));
    std::vector<float> tbest(cand.size(), 1e30f);
    int st = QED2D_OK;
    for (int rep = 0; rep < 3 && st == QED2D_OK; rep++)
        for (size_t i = 0; i < cand.size() && st == QED2D_OK; i++) {
            if (tbest[i] >= 2e30f) continue;
            cudaEventRecord(e0, c.stream);
            const int lst = launch(cand[i]);
            cudaEventRecord(e1, c.stream);
            if (lst == QED2D_ERR_UNSUPPORTED) {   // refused before anything was enqueued: drop it
                cudaGetLastError();
                tbest[i] = 3e30f;
                continue;
            }
            st = lst;
            if (cudaEventSynchronize(e1) != cudaSuccess) st = cuda_status(cudaGetLastError(), "schedule tuning");
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) tbest[i] = std::min(tbest[i], ms);
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    size_t b = 0;
    for (size_t i = 1; i < cand.size(); i++)
        if (tbest[i] <= tbest[b]) b = i;
    *best = cand[b];
    return st;
}

static int tune_cg(Ctx& c, const CGP& P, int slot) {
    if (!tuning_enabled()) {
        c.sched[slot] = c.g.V <= (1LL << 20) ? 1 : 0;
        return QED2D_OK;
    }
    DevCtl saved;
    QCHECK(cudaMemcpyAsync(&saved, c.ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, c.stream));
    QCHECK(cudaStreamSynchronize(c.stream));
    CGP T = P;
    T.x = c.spinor("tune_x");
    if (T.g5x) T.g5x = c.spinor("tune_g5x");
    if (!T.x || (P.g5x && !T.g5x)) return QED2D_ERR_NO_MEMORY;
    T.maxiter = std::min(P.maxiter, kTuneIters);
    const size_t fb = sizeof(double2) * 2 * (size_t)c.g.V;
    std::vector<int> cand = {0, 1};
    if (cluster_possible(c, slot)) cand.push_back(2);
    if (slot == 1) {   // the RL form under each reduction schedule
        const size_t n = cand.size();
        for (size_t i = 0; i < n; i++) cand.push_back(cand[i] + 4);
    }
    int best = 1;
    const int st = time_schedules(
        c,
        [&](int rs) -> int {
            if (P.guess) QCHECK(cudaMemcpyAsync(T.x, P.x, fb, cudaMemcpyDeviceToDevice, c.stream));
            return launch_cg(c, T, slot, rs);
        },
        cand, &best);
    QCHECK(cudaMemcpyAsync(c.ctl, &saved, sizeof(DevCtl), cudaMemcpyHostToDevice, c.stream));
    QCHECK(cudaStreamSynchronize(c.stream));
    if (st != QED2D_OK) return st;
    c.sched[slot] = best;
    return QED2D_OK;
}

int cg_solve(Ctx& c, const SolveArgs& a, int precision) {
    if (precision == QED2D_PREC_PLAIN) return solve_plain(c, a);
    CGP P{};
    P.g = c.g;
    P.U = a.U;
    P.b = a.b;
    P.x = a.x;
    P.r = c.spinor("cg_r");
    P.t = c.spinor("cg_t");
    P.g5x = a.g5x;
    P.m2 = 2.0 + a.am0;
    P.mu2 = a.mu2;
    P.eps = a.eps;
    P.maxiter = a.maxiter;
    P.guess = a.guess ? 1 : 0;
    P.ctl = c.ctl;
    P.part = c.part;
    P.delta2 = kReliableDelta * kReliableDelta;
    if (precision == QED2D_PREC_F64) {
        P.p0 = c.spinor("cg_p0");
        P.p1 = c.spinor("cg_p1");
        if (c.sched[0] < 0) QTRY(tune_cg(c, P, 0));
        if (c.sched[0] == 2 && !cluster_possible(c, 0)) c.sched[0] = 1;
        return launch_cg(c, P, 0, c.sched[0]);
    }
    P.r32 = c.spinor32("cg_r32");
    P.q0 = c.spinor32("cg_q0");
    P.q1 = c.spinor32("cg_q1");
    P.t32 = c.spinor32("cg_t32");
    P.x32 = c.spinor32("cg_x32");
    if (a.U32) {
        P.U32 = a.U32;
    } else {
        float4* u32 = c.spinor32("cg_u32");
        QTRY(launch_pack_links(c, u32, a.U));
        P.U32 = u32;
    }
    if (c.sched[1] < 0) QTRY(tune_cg(c, P, 1));
    if ((c.sched[1] & 3) == 2 && !cluster_possible(c, 1)) c.sched[1] -= 1;
    return launch_cg(c, P, 1, c.sched[1]);
}

// layouts of k_cg_multishift: tile rows and threads per site (shift groups)
struct MsLayout {
    int ty, s;
};
constexpr MsLayout kMsLayouts[kMsLayoutCount] = {{8, 1}, {8, 2}, {4, 4}, {4, 2}};

template <int RS>
static void (*ms_kernel(int layout))(MSP) {
    switch (layout) {
        case 1: return k_cg_multishift<RS, 8, 2>;
        case 2: return k_cg_multishift<RS, 4, 4>;
        case 3: return k_cg_multishift<RS, 4, 2>;
        default: return k_cg_multishift<RS, 8, 1>;
    }
}

static long long ms_tiles(const Ctx& c, int ty) {
    return (long long)((c.g.L1 + TX - 1) / TX) * ((c.g.L2 + ty - 1) / ty);
}

static int launch_multishift(Ctx& c, const MSP& P, int rs, int layout) {
    const MsLayout& l = kMsLayouts[layout];
    const int threads = TX * l.ty * l.s;
    const long long nt = ms_tiles(c, l.ty);
    if (rs == 2) return launch_cluster(c, ms_kernel<2>(layout), P, threads, nt);
    return launch_coop(c, rs ? ms_kernel<1>(layout) : ms_kernel<0>(layout), P, threads, nt);
}

static bool multishift_cluster_possible(Ctx& c, int layout) {
    int g = 0;
    const MsLayout& l = kMsLayouts[layout];
    return cluster_grid(c, ms_kernel<2>(layout), &g, TX * l.ty * l.s, ms_tiles(c, l.ty)) == QED2D_OK;
}

// As tune_cg: the first multishift solve of a context times the schedules and
// layouts on the caller's operator and source, capped at kTuneIters
// iterations, into scratch solutions (one per shift), and keeps the fastest.
// The single cluster wins on the smallest lattices (one barrier round trip less
// than the grid, a few tiles per block); the grid wins once a cluster's blocks
// walk many tiles each, the shift updates growing with them.  A layout fixed by
// the caller is kept.
static int tune_multishift(Ctx& c, const MSP& P) {
    if (c.g.V >= kMs32Sites) {   // the FP32-inner form, measured faster from 2048^2 on
        c.sched[2] = 3;
        return QED2D_OK;
    }
    if (!tuning_enabled()) {   // measured: 32 x 4 tiles with four threads per site up to 128^2
        c.sched[2] = 1;
        if (c.ms_layout < 0) c.ms_layout = c.g.V <= (1LL << 14) ? 2 : 0;
        return QED2D_OK;
    }
    DevCtl saved;
    QCHECK(cudaMemcpyAsync(&saved, c.ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, c.stream));
    QCHECK(cudaStreamSynchronize(c.stream));
    MSP T = P;
    for (int i = 0; i < P.n; i++) {
        T.x[i] = c.spinor("tune_ms_x_" + std::to_string(i));
        if (!T.x[i]) return QED2D_ERR_NO_MEMORY;
    }
    T.maxiter = std::min(P.maxiter, kTuneIters);
    std::vector<std::pair<int, int>> cand;   // (schedule, layout)
    const int l_lo = c.ms_layout >= 0 ? c.ms_layout : 0, l_hi = c.ms_layout >= 0 ? c.ms_layout + 1 : kMsLayoutCount;
    for (int l = l_lo; l < l_hi; l++) {
        cand.push_back({0, l});
        cand.push_back({1, l});
        if (multishift_cluster_possible(c, l)) cand.push_back({2, l});
    }
    cudaEvent_t e0, e1;
    QCHECK(cudaEventCreate(&e0));
    QCHECK(cudaEventCreate(&e1));
    std::vector<float> tbest(cand.size(), 1e30f);
    int st = QED2D_OK;
    for (int rep = 0; rep < 3 && st == QED2D_OK; rep++)
        for (size_t i = 0; i < cand.size() && st == QED2D_OK; i++) {
            cudaEventRecord(e0, c.stream);
            st = launch_multishift(c, T, cand[i].first, cand[i].second);
            cudaEventRecord(e1, c.stream);
            if (cudaEventSynchronize(e1) != cudaSuccess) st = cuda_status(cudaGetLastError(), "schedule tuning");
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) tbest[i] = std::min(tbest[i], ms);   // the first repetition warms up
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    QCHECK(cudaMemcpyAsync(c.ctl, &saved, sizeof(DevCtl), cudaMemcpyHostToDevice, c.stream));
    QCHECK(cudaStreamSynchronize(c.stream));
    if (st != QED2D_OK) return st;
    size_t best = 0;
    for (size_t i = 1; i < cand.size(); i++)
        if (tbest[i] < tbest[best]) best = i;
    c.sched[2] = cand[best].first;
    c.ms_layout = cand[best].second;
    return QED2D_OK;
}

// Multishift schedule 3: the FP32 shared Krylov space (k_cg_multishift32, grid
// reductions) to the relative residual sqrt(kMs32Eps), then every shift refined
// by the mixed CG from that start to the caller's eps.  The refinement of a
// shift stops on the FP64 true residual of that shift's system, as every solve
// of the library does.  Measured on B200, 12 Zolotarev poles, eps = 1e-24 (the
// FP64 multi-shift first): 128^2 2.32 -> 5.16 ms, 512^2 9.68 -> 11.53 ms,
// 2048^2 157.7 -> 141.5 ms.  Below 2048^2 the twelve refinement solves cost more
// than the halved bytes of the shared Krylov space save (the solver is
// latency-bound there); the untuned choice is this form from kMs32Sites on.
constexpr double kMs32Eps = 1e-12;

static int multishift32_solve(Ctx& c, const double2* U, const double2* b, double2* const* x, const double* mu2,
                              int n, double am0, int maxiter, double eps) {
    MSP32 P{};
    P.g = c.g;
    float4* u32 = c.spinor32("ms32_u");
    if (!u32) return QED2D_ERR_NO_MEMORY;
    QTRY(launch_pack_links(c, u32, U));
    P.U32 = u32;
    P.b = b;
    P.r = c.spinor32("ms32_r");
    P.p0 = c.spinor32("ms32_p0");
    P.p1 = c.spinor32("ms32_p1");
    P.t = c.spinor32("ms32_t");
    int base = 0;
    for (int i = 1; i < n; i++)
        if (mu2[i] < mu2[base]) base = i;
    for (int i = 0; i < n; i++) {
        P.x[i] = c.spinor32("ms32_x_" + std::to_string(i));
        P.ps[i] = i == base ? nullptr : c.spinor32("ms32_ps_" + std::to_string(i));
        P.x64[i] = x[i];
        P.d[i] = mu2[i] - mu2[base];
        if (!P.x[i] || (i != base && !P.ps[i])) return QED2D_ERR_NO_MEMORY;
    }
    if (!P.r || !P.p0 || !P.p1 || !P.t) return QED2D_ERR_NO_MEMORY;
    P.n = n;
    P.base = base;
    P.m2 = 2.0 + am0;
    P.mu2b = mu2[base];
    P.eps32 = std::max(eps, kMs32Eps);
    P.maxiter = maxiter;
    P.ctl = c.ctl;
    P.part = c.part;
    QTRY(launch_coop(c, k_cg_multishift32<1>, P));
    for (int i = 0; i < n; i++) {   // refine each shift to the FP64 stop rule
        SolveArgs a;
        a.U = U;
        a.U32 = u32;
        a.b = b;
        a.x = x[i];
        a.am0 = am0;
        a.mu2 = mu2[i];
        a.maxiter = maxiter;
        a.eps = eps;
        a.guess = true;
        QTRY(cg_solve(c, a, QED2D_PREC_MIXED));
    }
    return QED2D_OK;
}

int multishift_solve(Ctx& c, const double2* U, const double2* b, double2* const* x, const double* mu2, int n,
                     double am0, int maxiter, double eps) {
    if (n < 1 || n > kMaxShifts) return QED2D_ERR_BAD_ARG;
    if (c.sched[2] == 3) return multishift32_solve(c, U, b, x, mu2, n, am0, maxiter, eps);
    MSP P{};
    P.g = c.g;
    P.U = U;
    P.b = b;
    P.r = c.spinor("ms_r");
    P.p0 = c.spinor("ms_p0");
    P.p1 = c.spinor("ms_p1");
    P.t = c.spinor("ms_t");
    int base = 0;
    for (int i = 1; i < n; i++)
        if (mu2[i] < mu2[base]) base = i;
    for (int i = 0; i < n; i++) {
        P.x[i] = x[i];
        P.ps[i] = i == base ? nullptr : c.spinor("ms_p_" + std::to_string(i));
        P.d[i] = mu2[i] - mu2[base];
    }
    P.n = n;
    P.base = base;
    P.m2 = 2.0 + am0;
    P.mu2b = mu2[base];
    P.eps = eps;
    P.maxiter = maxiter;
    P.ctl = c.ctl;
    P.part = c.part;
    if (c.sched[2] < 0) QTRY(tune_multishift(c, P));
    const int layout = c.ms_layout < 0 ? 0 : c.ms_layout;
    if (c.sched[2] == 2 && !multishift_cluster_possible(c, layout)) c.sched[2] = 1;
    return launch_multishift(c, P, c.sched[2], layout);
}

// ---------------------------------------------------------------------------
// QED2D_PREC_PLAIN: the reference's CG loop structure (src/QED2dSolver.jl:49-105)
// on the GPU -- operator as two gamm5Dw launches, BLAS-1 launches, and the host
// reading <p,Ap> and |r|^2 back every iteration.
static int read_scal(Ctx& c, int slot, int n, double* out) {
    QCHECK(cudaMemcpyAsync(out, &c.ctl->scal[slot], sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream));
    QCHECK(cudaStreamSynchronize(c.stream));
    return QED2D_OK;
}

static int plain_op(Ctx& c, double2* Ap, double2* tmp, const double2* U, const double2* p, double am0, double mu2) {
    QTRY(launch_g5dw(c, tmp, U, p, am0, nullptr, make_double2(0, 0), false));
    return launch_g5dw(c, Ap, U, tmp, am0, mu2 != 0.0 ? p : nullptr, make_double2(mu2, 0), false);
}

static int solve_plain(Ctx& c, const SolveArgs& a) {
    const long long n = 2 * c.g.V;
    double2* r = c.spinor("pl_r");
    double2* p = c.spinor("pl_p");
    double2* Ap = c.spinor("pl_Ap");
    double2* tmp = c.spinor("pl_tmp");
    const double2 one = make_double2(1, 0), zero = make_double2(0, 0);
    double h[2];
    QTRY(launch_reduce_vec(c, 0, a.b, nullptr, n, 0));
    QTRY(read_scal(c, 0, 1, h));
    const double bb = h[0], tol = a.eps * bb;
    int iters = 0;
    bool conv = false;
    double err = 0.0, norm, final_rr = 0.0;
    if (bb == 0.0) {
        QTRY(launch_zero(c, a.x, sizeof(double2) * n));
        conv = true;
        norm = 0.0;
    } else if (!a.guess) {
        QTRY(launch_zero(c, a.x, sizeof(double2) * n));
        QTRY(launch_copy(c, r, a.b, sizeof(double2) * n));
        QTRY(launch_copy(c, p, a.b, sizeof(double2) * n));
        norm = bb;
    } else {
        QTRY(plain_op(c, Ap, tmp, a.U, a.x, a.am0, a.mu2));
        QTRY(launch_zaxpby(c, r, one, a.b, make_double2(-1, 0), Ap, n));
        QTRY(launch_copy(c, p, r, sizeof(double2) * n));
        QTRY(launch_reduce_vec(c, 0, r, nullptr, n, 0));
        QTRY(read_scal(c, 0, 1, h));
        norm = h[0];
        final_rr = norm;
        if (norm < tol) conv = true;
    }
    if (!conv) {
        for (int i = 1; i <= a.maxiter; i++) {
            QTRY(plain_op(c, Ap, tmp, a.U, p, a.am0, a.mu2));
            QTRY(launch_reduce_vec(c, 1, p, Ap, n, 0));
            QTRY(read_scal(c, 0, 2, h));
            // alpha = norm / prod (complex), Smith's division
            double2 alpha;
            {
                const double br = h[0], bi = h[1];
                if (fabs(br) >= fabs(bi)) {
                    const double t = bi / br, den = br + bi * t;
                    alpha = make_double2(norm / den, (-norm * t) / den);
                } else {
                    const double t = br / bi, den = bi + br * t;
                    alpha = make_double2((norm * t) / den, -norm / den);
                }
            }
            QTRY(launch_zaxpby(c, a.x, one, a.x, alpha, p, n));
            QTRY(launch_zaxpby(c, r, one, r, make_double2(-alpha.x, -alpha.y), Ap, n));
            QTRY(launch_reduce_vec(c, 0, r, nullptr, n, 0));
            QTRY(read_scal(c, 0, 1, h));
            err = h[0];
            final_rr = err;
            if (err < tol) { iters = i; conv = true; break; }
            const double beta = err / norm;
            QTRY(launch_zaxpby(c, p, one, r, make_double2(beta, 0), p, n));
            norm = err;
        }
        if (!conv) iters = a.maxiter;
    }
    if (a.g5x) QTRY(launch_g5dw(c, a.g5x, a.U, a.x, a.am0, nullptr, make_double2(0, 0), false));
    // record in the control block like the persistent solvers do
    QTRY(read_ctl(c, false));
    c.ctl_host->last_iters = iters;
    c.ctl_host->last_updates = 0;
    c.ctl_host->last_conv = conv;
    c.ctl_host->last_relres = bb > 0 ? final_rr / bb : 0.0;
    c.ctl_host->iters_total += iters;
    if (c.ctl_host->status == 0 && !conv) c.ctl_host->status = QED2D_ERR_NOT_CONVERGED;
    QCHECK(cudaMemcpyAsync(c.ctl, c.ctl_host, sizeof(DevCtl), cudaMemcpyHostToDevice, c.stream));
    QCHECK(cudaStreamSynchronize(c.stream));
    return QED2D_OK;
}

int read_ctl(Ctx& c, bool reset_sequence) {
    QCHECK(cudaMemcpyAsync(c.ctl_host, c.ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, c.stream));
    QCHECK(cudaStreamSynchronize(c.stream));
    const int st = c.ctl_host->status;
    c.last_iters = c.ctl_host->last_iters;
    c.last_updates = c.ctl_host->last_updates;
    c.last_relres = c.ctl_host->last_relres;
    if (reset_sequence) {
        QCHECK(cudaMemsetAsync(&c.ctl->status, 0, sizeof(int), c.stream));
        QCHECK(cudaMemsetAsync(&c.ctl->iters_total, 0, sizeof(long long), c.stream));
    }
    return st;
}

}  // namespace qed2d

namespace qed2d {

// ---------------------------------------------------------------------------
// Allocation-free CG (qed2d_cg_noalloc).  Some callers must not allocate device
// memory once they are running: a host loop that has handed all device memory
// to its own pool allocator up front (CUDA.jl's or PyTorch's caching allocator
// would see an out-of-band cudaMalloc as lost capacity), or a latency-bound loop
// in which the implicit device synchronisation of cudaMalloc/cudaFree would stall
// the pipeline.  This entry point runs the same persistent FP64 CG kernel as
// qed2d_cg (method 1) without a context: its scratch -- the control block, the
// reduction partials and the four solver vectors r, p (x2), t -- is one
// file-scope device array, sized for at most QED2D_NOALLOC_MAX_SITES sites, that
// every GPU which loads this library holds until the process exits.
//
// Set-up: the first call on a device looks up the array's device address with
// cudaGetSymbolAddress (this can also load the library's device code) and caches
// it per device; make that first call before any stream capture.  The cached
// address belongs to the device context it was looked up in: a caller that ends
// that context with cudaDeviceReset must not call this entry point on that
// device again in the same process (the address would be stale).  Every call
// shares the one array, so calls that overlap on the GPU (two streams, two host
// threads) race; serialise them.  Each call synchronises its stream before it
// returns.  The control block is zeroed by each call; the vectors are always
// written before they are read.
namespace {
constexpr size_t kNaCtlBytes = 512;
constexpr size_t kNaPartBytes = sizeof(double) * kMaxPartVals * kMaxPartBlocks;
constexpr size_t kNaFieldBytes = sizeof(double2) * 2 * (size_t)QED2D_NOALLOC_MAX_SITES;
constexpr size_t kNaBytes = kNaCtlBytes + kNaPartBytes + 4 * kNaFieldBytes;
static_assert(sizeof(DevCtl) <= kNaCtlBytes, "control block does not fit its slot");
static_assert(kNaPartBytes % 256 == 0 && kNaFieldBytes % 256 == 0, "scratch slices must stay 256-byte aligned");
constexpr int kNaMaxDevices = 64;
std::mutex g_na_mutex;
void* g_na_base[kNaMaxDevices] = {};
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

// device address of g_noalloc_scratch on the current device (looked up once per device)
static int noalloc_scratch(void** base) {
    int dev = 0;
    QCHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNaMaxDevices) {
        set_error("qed2d_cg_noalloc: device ordinal out of range");
        return QED2D_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_base[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_na_base[dev] = p;
    }
    *base = g_na_base[dev];
    return QED2D_OK;
}

}  // namespace qed2d

extern "C" int qed2d_cg_noalloc(int L1, int L2, double* so, const double* U, const double* si, double am0,
                                int maxiter, double eps, void* stream, int* iterations) {
    using namespace qed2d;
    if (L1 < 2 || L2 < 2) {
        set_error("qed2d_cg_noalloc: lattice extents must be >= 2");
        return QED2D_ERR_BAD_ARG;
    }
    const long long V = (long long)L1 * L2;
    if (V > QED2D_NOALLOC_MAX_SITES) {
        set_error("qed2d_cg_noalloc: " + std::to_string(L1) + "x" + std::to_string(L2) + " = " + std::to_string(V) +
                  " sites exceeds the static scratch limit of " + std::to_string(QED2D_NOALLOC_MAX_SITES) +
                  " sites; use qed2d_cg");
        return QED2D_ERR_BAD_ARG;
    }
    if (!so || !U || !si || maxiter < 0 || (reinterpret_cast<uintptr_t>(so) | reinterpret_cast<uintptr_t>(U) |
                                            reinterpret_cast<uintptr_t>(si)) % 16 != 0) {
        set_error("qed2d_cg_noalloc: NULL or misaligned array, or maxiter < 0");
        return QED2D_ERR_BAD_ARG;
    }
    const size_t fb = sizeof(double2) * 2 * (size_t)V;
    const char *a = (const char*)so, *b = (const char*)si, *u = (const char*)U;
    if ((a < b + fb && b < a + fb) || (a < u + fb && u < a + fb)) {
        set_error("qed2d_cg_noalloc: so aliases si or U");
        return QED2D_ERR_BAD_ARG;
    }
    void* base = nullptr;
    QTRY(noalloc_scratch(&base));
    char* p = (char*)base;
    DevCtl* ctl = (DevCtl*)p;
    double* part = (double*)(p + kNaCtlBytes);
    double2* fields = (double2*)(p + kNaCtlBytes + kNaPartBytes);
    cudaStream_t s = (cudaStream_t)stream;

    CGP P{};
    P.g.L1 = L1;
    P.g.L2 = L2;
    P.g.V = V;
    P.U = (const double2*)U;
    P.b = (const double2*)si;
    P.x = (double2*)so;
    P.r = fields;
    P.p0 = fields + 2 * QED2D_NOALLOC_MAX_SITES;
    P.p1 = fields + 4 * QED2D_NOALLOC_MAX_SITES;
    P.t = fields + 6 * QED2D_NOALLOC_MAX_SITES;
    P.g5x = nullptr;
    P.m2 = 2.0 + am0;
    P.mu2 = 0.0;
    P.eps = eps;
    P.maxiter = maxiter;
    P.guess = 0;
    P.ctl = ctl;
    P.part = part;

    int dev = 0, sms = 0, per_sm = 0;
    QCHECK(cudaGetDevice(&dev));
    QCHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    QCHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cg_f64<0>, TILE, 0));
    if (per_sm < 1) return QED2D_ERR_UNSUPPORTED;
    long long grid = (long long)per_sm * sms;
    if (grid > kMaxPartBlocks) grid = kMaxPartBlocks;
    const long long nt = num_tiles(P.g);
    const long long per_block = (nt + grid - 1) / grid;
    grid = (nt + per_block - 1) / per_block;
    P.per_block = (int)per_block;

    QCHECK(cudaMemsetAsync(ctl, 0, sizeof(DevCtl), s));
    void* args[] = {(void*)&P};
    QCHECK(cudaLaunchCooperativeKernel((const void*)k_cg_f64<0>, dim3((unsigned)grid), dim3(TILE), args, 0, s));
    count_launch();
    DevCtl h;
    QCHECK(cudaMemcpyAsync(&h, ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, s));
    QCHECK(cudaStreamSynchronize(s));
    if (iterations) *iterations = h.last_iters;
    if (h.status != QED2D_OK) set_error(std::string("qed2d_cg_noalloc: ") + qed2d_status_string(h.status));
    return h.status;
}
