// batch_cg_cluster.cuh -- the batched mixed CG with one thread-block cluster
// per replica: the alternative to k_r_cg_mixed for batches of uneven lattices.
//
// Cluster c (CS blocks) solves replica order[c] alone: its blocks split the
// replica's tiles, reduce over distributed shared memory and synchronise with
// the hardware cluster barrier, and there is no grid-wide barrier at all.  A
// replica that converges frees its SMs for clusters still waiting to start, so
// the replicas stream through the GPU (largest first), and while one is being
// solved its few MB of vectors stay in L2.  The CG recurrences are those of
// the single-lattice mixed solver (rep_step); every block of a cluster computes
// them from the same sums in the same order, so all blocks take the same path.
// Layout as batch.cu (replica-major).
#pragma once

#include <cooperative_groups.h>

namespace qed2d {

struct CCGP {
    const RepInfo* reps;
    const int* order;   // cluster c solves replica order[c]
    const double* m2;   // 2 + m0 per replica
    const double2* U;
    const float4* U32;   // FP32 link planes of vtot sites
    long long vtot;
    const double2* b;
    double2* x;
    double2* r64;
    double2* t64;   // g5Dw x of the solution (the force needs it)
    float4 *r32, *q0, *q1, *t32, *x32;
    double eps, delta2;
    int maxiter;
    RepState* st_out;   // [nrep] final records
};

// Sum of v over the cluster: a block sum into this block's shared slot
// (alternating between two), the cluster barrier, then lane i reads rank i's
// slot over distributed shared memory and a fixed shuffle tree adds them; every
// block gets the same bits.
template <int CS>
__device__ __forceinline__ double cluster_sum(double v, double* smem, double* s_slot, int& nred) {
    namespace cgr = cooperative_groups;
    __shared__ double s_tot;
    double vv[1] = {v};
    block_sum<1>(vv, smem);
    const int buf = nred++ & 1;
    if (threadIdx.x == 0) s_slot[buf] = vv[0];
    cgr::cluster_group cl = cgr::this_cluster();
    cl.sync();
    if (threadIdx.x < 32) {
        double s = threadIdx.x < CS ? *cl.map_shared_rank(s_slot + buf, threadIdx.x) : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) s_tot = s;
    }
    __syncthreads();
    return s_tot;
}

// thread 0 advances the replica's record for reduction `kind`; all threads see it after
__device__ __forceinline__ void cluster_step(RepState* S, int kind, double s, int k, const CCGP& P) {
    if (threadIdx.x == 0) {
        RepState st = *S;
        int fl[FL_N] = {0, 0, 0};
        rep_step(st, kind, s, k, P.eps, P.delta2, P.maxiter, fl);
        *S = st;
    }
    __syncthreads();
}

// RSTEN: the first phase's stencil on r, t = g5Dw r + beta t_old (as schedule 8
// of the equal-size solver)
template <int CS, bool RSTEN = false>
__device__ __forceinline__ void c_body(const CCGP& P, int r, int& k, double* smem, double* s_slot, RepState* S) {
    namespace cgr = cooperative_groups;
    const int rank = (int)cgr::this_cluster().block_rank();
    const RepInfo R = P.reps[r];
    const Lat g = lat_of(R);
    const TileRange TR = tile_range(R.nt, R.nt1, (R.nt + CS - 1) / CS, rank);
    const long long V = R.V, o2 = 2 * R.off, o1 = R.off;
    const double2* bb = P.b + o2;
    double2* xx = P.x + o2;
    double2* r64 = P.r64 + o2;
    double2* t64 = P.t64 + o2;
    float4* r32 = P.r32 + o1;
    float4* x32 = P.x32 + o1;
    float4* t32 = P.t32 + o1;
    float4* q0 = P.q0 + o1;
    float4* q1 = P.q1 + o1;
    const LkD L{P.U + o2, V};
    const LkF Lf{P.U32, P.vtot, o1};
    const double m2 = P.m2[r];
    const float m2f = (float)m2;
    const Pair<double> z{make_double2(0, 0), make_double2(0, 0)};
    const Pair<float> zf{make_float2(0, 0), make_float2(0, 0)};
    int cur = 0, nred = 0;
    bool pend = false;   // x32 += alpha p every second iteration, as in k_u_cg_mixed (same bits)
    float apend = 0.f;
#define FOR_MY_CTILES(q) FOR_RANGE(q, g, TR)
    {   // |b|^2; x = 0
        double v = 0.0;
        FOR_MY_CTILES(q) {
            const Pair<double> bv{__ldg(bb + q.x), __ldg(bb + q.x + V)};
            v += norm2(bv.a) + norm2(bv.b);
            st_d(xx, V, q.x, z);
        }
        cluster_step(S, RED_BB, cluster_sum<CS>(v, smem, s_slot, nred), 0, P);
    }
    {   // r32 = s b, x32 = 0 (a zero source keeps x = 0 and g5Dw x = 0)
        double v = 0.0;
        const RepState st = *S;
        FOR_MY_CTILES(q) {
            if (st.act) {
                const Pair<float> rv{to_f(st.s * __ldg(bb + q.x)), to_f(st.s * __ldg(bb + q.x + V))};
                st_f(r32, q.x, rv);
                st_f(x32, q.x, zf);
                v += (double)(norm2(rv.a) + norm2(rv.b));
            } else {
                st_d(t64, V, q.x, z);
            }
        }
        cluster_step(S, RED_RR0, cluster_sum<CS>(v, smem, s_slot, nred), 0, P);
    }
    for (k = 1; k <= P.maxiter; k++) {
        if (!S->act) break;
        float4* qn = cur ? q1 : q0;
        const float4* qo = cur ? q0 : q1;
        {   // p = r + beta p_old, t = g5Dw p, <p, A p> = |t|^2
            float f = 0.f;
            const RepState st = *S;
            if constexpr (RSTEN) {
                const float beta = (float)st.beta;
                const bool use_p = !st.first;
                FOR_MY_CTILES(q) {
                    const Pair<float> rc = SpF{r32}.ld(q.x);
                    Pair<float> tt = g5dw_at_c<float>(SpF{r32}, rc, Lf, q, m2f), c = rc;
                    if (use_p) {   // p = r + beta p_old, t = g5Dw r + beta t_old
                        const Pair<float> po = SpF{qo}.ld(q.x), to = SpF{t32}.ld(q.x);
                        c.a = c.a + beta * po.a;
                        c.b = c.b + beta * po.b;
                        tt.a = tt.a + beta * to.a;
                        tt.b = tt.b + beta * to.b;
                    }
                    st_f(qn, q.x, c);
                    st_f(t32, q.x, tt);
                    f += norm2(tt.a) + norm2(tt.b);
                }
            } else {
                const SpAxpy<float, SpF> Q{SpF{r32}, SpF{qo}, (float)st.beta, !st.first};
                FOR_MY_CTILES(q) {
                    const Pair<float> c = Q.ld(q.x);
                    const Pair<float> tt = g5dw_at_c<float>(Q, c, Lf, q, m2f);
                    st_f(qn, q.x, c);
                    st_f(t32, q.x, tt);
                    f += norm2(tt.a) + norm2(tt.b);
                }
            }
            cluster_step(S, RED_PAP, cluster_sum<CS>((double)f, smem, s_slot, nred), k, P);
        }
        {   // x += alpha p (every second iteration, for two directions), r -= alpha g5Dw t
            float f = 0.f;
            const float alpha = (float)S->alpha;
            if (pend) {
                FOR_MY_CTILES(q) {
                    const Pair<float> po = SpF{qo}.ld(q.x), pc = SpF{qn}.ld(q.x);
                    const Pair<float> a = g5dw_at<float>(SpF{t32}, Lf, q, m2f);
                    Pair<float> xv = SpF{x32}.ld(q.x), rv = SpF{r32}.ld(q.x);
                    xv.a = xv.a + apend * po.a;
                    xv.b = xv.b + apend * po.b;
                    xv.a = xv.a + alpha * pc.a;
                    xv.b = xv.b + alpha * pc.b;
                    rv.a = rv.a - alpha * a.a;
                    rv.b = rv.b - alpha * a.b;
                    st_f(x32, q.x, xv);
                    st_f(r32, q.x, rv);
                    f += norm2(rv.a) + norm2(rv.b);
                }
            } else {
                FOR_MY_CTILES(q) {
                    const Pair<float> a = g5dw_at<float>(SpF{t32}, Lf, q, m2f);
                    Pair<float> rv = SpF{r32}.ld(q.x);
                    rv.a = rv.a - alpha * a.a;
                    rv.b = rv.b - alpha * a.b;
                    st_f(r32, q.x, rv);
                    f += norm2(rv.a) + norm2(rv.b);
                }
            }
            apend = alpha;
            pend = !pend;
            cluster_step(S, RED_RN, cluster_sum<CS>((double)f, smem, s_slot, nred), k, P);
        }
        if (S->upd) {   // FP64 reliable update
            const double inv_s = 1.0 / S->s;
            FOR_MY_CTILES(q) {   // x += x32 / s, with this iteration's x32 update if it waits
                Pair<float> d = SpF{x32}.ld(q.x);
                if (pend) {
                    const Pair<float> pc = SpF{qn}.ld(q.x);
                    d.a = d.a + apend * pc.a;
                    d.b = d.b + apend * pc.b;
                }
                Pair<double> xv = SpD{xx, V}.ld(q.x);
                xv.a = xv.a + inv_s * to_d(d.a);
                xv.b = xv.b + inv_s * to_d(d.b);
                st_d(xx, V, q.x, xv);
                st_f(x32, q.x, zf);
            }
            pend = false;
            cgr::this_cluster().sync();
            FOR_MY_CTILES(q) st_d(t64, V, q.x, g5dw_at<double>(SpD{xx, V}, L, q, m2));
            cgr::this_cluster().sync();
            double w = 0.0;
            FOR_MY_CTILES(q) {   // r64 = b - A x
                const Pair<double> a = g5dw_at<double>(SpD{t64, V}, L, q, m2);
                Pair<double> rv;
                rv.a = __ldg(bb + q.x) - a.a;
                rv.b = __ldg(bb + q.x + V) - a.b;
                st_d(r64, V, q.x, rv);
                w += norm2(rv.a) + norm2(rv.b);
            }
            cluster_step(S, RED_TRUE, cluster_sum<CS>(w, smem, s_slot, nred), k, P);
            if (S->r4) {
                double v = 0.0;
                const double sn = S->snew;
                FOR_MY_CTILES(q) {   // r32 = s_new r64
                    const Pair<float> rv{to_f(sn * r64[q.x]), to_f(sn * r64[q.x + V])};
                    st_f(r32, q.x, rv);
                    v += (double)(norm2(rv.a) + norm2(rv.b));
                }
                cluster_step(S, RED_R4, cluster_sum<CS>(v, smem, s_slot, nred), k, P);
            }
        }
        cur ^= 1;
    }
#undef FOR_MY_CTILES
}

template <int CS, bool RSTEN = false>
__global__ void __launch_bounds__(TILE, 4) k_rc_cg_mixed(const CCGP P) {
    namespace cgr = cooperative_groups;
    __shared__ double smem[32];
    __shared__ double s_slot[2];
    __shared__ RepState s_st;
    const int r = P.order[blockIdx.x / CS];
    int k = 0;
    c_body<CS, RSTEN>(P, r, k, smem, s_slot, &s_st);
    if (cgr::this_cluster().block_rank() == 0 && threadIdx.x == 0) P.st_out[r] = s_st;
    cgr::this_cluster().sync();   // no block leaves while another may still read its slots
}

}  // namespace qed2d
