// batch_cg_uniform.cuh -- the batched mixed CG for batches of equal-size
// replicas (at most kUniformReps of them): the fast path of batch.cu.
//
// Block b serves replica b / bpr only, and a contiguous range of that
// replica's tiles, so every block's geometry, masses and pointers are kernel
// constants and a phase starts without any loads.  Each replica's partials are
// summed in a fixed order (deterministic) under one of three schedules
// (ureduce), and the blocks run the per-replica CG scalar recurrences
// themselves in shared memory.  Under the grid schedules (RS = 0, 1) all
// replicas pass the same barriers, and replicas that have converged stop
// working but keep joining them until all are done; under RS = 2 each replica
// has its own barrier, so one replica's wait overlaps another's work on the
// same SMs, and a converged replica's blocks leave.  The
// recurrences are those of the ragged kernel (rep_step) and of the
// single-lattice mixed solver.
//
// Layout as batch.cu (replica-major): replica r's FP32 packed site x (global,
// r*V + local) and its FP64 planes at 2*r*V + local and 2*r*V + V + local, read
// through the replica-shifted base pointer base + r*V with the global site
// index.
#pragma once

namespace qed2d {

constexpr int kUniformReps = 64;

struct UGeom {
    int L1, L2, B, nt1;
    long long V;     // sites per replica
    long long ntr;   // tiles per replica
};

struct UCGP {
    UGeom g;
    const double2* U;
    const float4* U32;
    const double2* b;
    double2* x;
    double2* r64;
    double2* t64;   // g5Dw x of the solution (the force needs it)
    float4 *r32, *q0, *q1, *t32, *x32;
    double m2[kUniformReps];
    double eps, delta2;
    int maxiter, bpr, per_block;
    DevCtl* ctl;
    double* part;       // [2][bpr * B] block partials (alternating)
    double* red;        // [2][B] published per-replica sums (RS = 0)
    unsigned long long* rbar;   // [B][16] per-replica barrier counters, one 128-byte line each (RS = 2)
    RepState* st_out;   // [B] final records
};

// site of thread t in tile (t1, t2) of replica r, tiles of 32 x TYv sites (a
// block of 32 * TYv threads, one site each): global FP32 index, neighbours
// wrapping inside the replica (no division)
template <int TYv>
__device__ __forceinline__ Site usite_at(const UGeom& g, int r, int t1, int t2, int t) {
    Site s;
    s.i1 = t1 * TX + (t & (TX - 1));
    s.i2 = t2 * TYv + (t >> 5);
    s.ok = s.i1 < g.L1 && s.i2 < g.L2;
    s.x = s.i1 + g.L1 * (r * g.L2 + s.i2);   // 32-bit: the batch holds < 2^30 sites
    s.xp1 = (s.i1 + 1 == g.L1) ? s.x - (g.L1 - 1) : s.x + 1;
    s.xm1 = (s.i1 == 0) ? s.x + (g.L1 - 1) : s.x - 1;
    s.xp2 = (s.i2 + 1 == g.L2) ? s.x - (long long)(g.L2 - 1) * g.L1 : s.x + g.L1;
    s.xm2 = (s.i2 == 0) ? s.x + (long long)(g.L2 - 1) * g.L1 : s.x - g.L1;
    return s;
}

// Barrier with one sum per replica (one warp per replica over its blocks'
// partials, fixed order).  Three schedules give the same bits: RS = 0, the last
// block to arrive sums and publishes red[] before releasing and every block
// reads red[]; RS = 1, a counter barrier, then every block sums the partials
// itself; then every block runs every replica's recurrences for reduction
// `kind` on its shared records and flags.  RS = 2 (independent replicas): gs is
// the barrier of this block's replica alone (its own counter, its bpr blocks),
// the block sums its replica's partials and runs that replica's recurrences
// only, and its flags are that replica's.  A failed or timed-out wait is passed
// on through shared memory.
template <int RS>
__device__ __forceinline__ bool ureduce(GridSync& gs, double v, const UCGP& P, double* smem, RepState* s_st,
                                        int* s_fl, int kind, int k) {
    __shared__ int s_last, s_bits, s_ok;
    __shared__ double s_red[kUniformReps];
    const int myr = RS >= 2 ? blockIdx.x / P.bpr : 0;
    const int buf = gs.nred++ & 1;
    double* part = P.part + (size_t)buf * P.bpr * P.g.B;
    double* red = P.red + (size_t)buf * P.g.B;
    if constexpr (RS == 3) {
        // Independent replicas, lean: the same additions in the same order as
        // RS = 2 (so the same bits), with two block barriers instead of seven.
        // Every warp reduces its value by shuffles; after one __syncthreads
        // (which orders the block's stores before thread 0's release-add) warp 0
        // sums the warp values, publishes the block partial and arrives, polls,
        // sums the replica's partials, and thread 0 steps the replica's
        // recurrences and sets the flags; one more __syncthreads releases the
        // block.
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) smem[warp] = v;
        __syncthreads();
        gs.target += gs.n();
        if (warp == 0) {
            double s = lane < nw ? smem[lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            int ok = 1;
            if (lane == 0) {
                part[blockIdx.x] = s;
                red_release_add_u64(gs.arrivals, 1ULL);
                gs.poll(gs.arrivals);
                ok = ld_volatile_int(gs.err) == 0;
            }
            __syncwarp();   // orders lane 0's acquire before the other lanes' partial loads
            ok = __shfl_sync(0xffffffffu, ok, 0);
            double t = 0.0;
            for (int i = lane; i < P.bpr; i += 32) t += __ldcg(part + (size_t)myr * P.bpr + i);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (lane == 0) {
                int fl[FL_N] = {0, 0, 0};
                RepState st = s_st[myr];
                rep_step(st, kind, t, k, P.eps, P.delta2, P.maxiter, fl);
                s_st[myr] = st;
                clear_flags(kind, s_fl);
                s_fl[FL_ACT] |= fl[FL_ACT];
                s_fl[FL_UPD] |= fl[FL_UPD];
                s_fl[FL_R4] |= fl[FL_R4];
                s_ok = ok;
            }
        }
        __syncthreads();
        return s_ok != 0;
    }
    double vv[1] = {v};
    block_sum<1>(vv, smem);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = vv[0];
        s_bits = 0;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    // the replicas whose sums this block needs: all of them, or (RS = 2) its own.
    // RS = 2 goes through the same loop shapes as RS = 1 on purpose: a
    // single-replica copy of them (warp 0 sums, thread myr steps) compiled to
    // code whose barrier waits took 50% longer (one replica of 512^2: 25.0
    // against 16.9 us per iteration, same arithmetic).
    const int r0 = RS == 2 ? myr : 0, r1 = RS == 2 ? myr + 1 : P.g.B;
    auto sum_partials = [&](double* out) {
        for (int r = r0 + warp; r < r1; r += nw) {
            double s = 0.0;
            for (int i = lane; i < P.bpr; i += 32) s += __ldcg(part + (size_t)r * P.bpr + i);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) out[r] = s;
        }
    };
    if constexpr (RS == 0) {
        if (gs.arrive(&s_last)) {
            sum_partials(red);
            __syncthreads();
            if (threadIdx.x == 0) {
                gs.release();
                s_ok = 1;
            }
        } else if (threadIdx.x == 0) {
            s_ok = gs.wait();
        }
        __syncthreads();
        if (threadIdx.x < P.g.B) s_red[threadIdx.x] = __ldcg(red + threadIdx.x);
    } else {
        gs.count_sync();
        if (threadIdx.x == 0) s_ok = ld_volatile_int(gs.err) == 0;
        sum_partials(s_red);
    }
    __syncthreads();
    int fl[FL_N] = {0, 0, 0};
    if ((int)threadIdx.x >= r0 && (int)threadIdx.x < r1) {
        RepState st = s_st[threadIdx.x];
        rep_step(st, kind, s_red[threadIdx.x], k, P.eps, P.delta2, P.maxiter, fl);
        s_st[threadIdx.x] = st;
    }
    const int bits = __reduce_or_sync(0xffffffffu, fl[FL_ACT] | fl[FL_UPD] << 1 | fl[FL_R4] << 2);
    if ((threadIdx.x & 31) == 0 && bits) atomicOr(&s_bits, bits);
    __syncthreads();
    if (threadIdx.x == 0) {
        clear_flags(kind, s_fl);
        s_fl[FL_ACT] |= s_bits & 1;
        s_fl[FL_UPD] |= (s_bits >> 1) & 1;
        s_fl[FL_R4] |= (s_bits >> 2) & 1;
    }
    __syncthreads();
    return s_ok != 0;
}

// this block's contiguous range of its replica's tiles, walked without division
#define FOR_MY_UTILES(q)                                                                       \
    for (int tt_ = TR.lo, t1_ = TR.s1, t2_ = TR.s2; tt_ < TR.hi;                              \
         ++tt_, (++t1_ == TR.nt1 ? (t1_ = 0, ++t2_) : 0))                                       \
        if (const Site q = usite_at<TYv>(P.g, myr, t1_, t2_, threadIdx.x); q.ok)

template <int RS, int TYv>
__device__ __forceinline__ bool u_body(const UCGP& P, GridSync& gs, int& k, double* smem, RepState* s_st,
                                       int* s_fl) {
    const int myr = blockIdx.x / P.bpr, lb = blockIdx.x - myr * P.bpr;
    const TileRange TR = tile_range(P.g.ntr, P.g.nt1, P.per_block, lb);
    const long long V = P.g.V, sh = (long long)myr * V;   // FP64 planes of replica myr: base + sh, stride V
    const double2* bb = P.b + sh;
    double2* xx = P.x + sh;
    double2* r64 = P.r64 + sh;
    double2* t64 = P.t64 + sh;
    const LkD L{P.U + sh, V};
    const LkF Lf{P.U32, P.g.V * P.g.B};
    const double m2 = P.m2[myr];
    const float m2f = (float)m2;
    const Pair<double> z{make_double2(0, 0), make_double2(0, 0)};
    const Pair<float> zf{make_float2(0, 0), make_float2(0, 0)};
    int cur = 0;
    // x32 += alpha p is applied every second iteration, for two directions at
    // once: while `pend`, the update of the previous iteration (alpha `apend`,
    // direction in the buffer that the next phase A reads as p_old) is still to
    // be added.  Same operations in the same order as one update per iteration,
    // so the same bits; x32 and one direction are read and x32 written half as
    // often (192 -> 176 algorithmic bytes per site-iteration).
    bool pend = false;
    float apend = 0.f;

    {   // |b|^2 per replica; x = 0
        double v = 0.0;
        FOR_MY_UTILES(q) {
            const Pair<double> bv{__ldg(bb + q.x), __ldg(bb + q.x + V)};
            v += norm2(bv.a) + norm2(bv.b);
            st_d(xx, V, q.x, z);
        }
        if (!ureduce<RS>(gs, v, P, smem, s_st, s_fl, RED_BB, 0)) return false;
    }
    {   // r32 = s b, x32 = 0 (a zero source keeps x = 0 and g5Dw x = 0)
        double v = 0.0;
        const RepState st = s_st[myr];
        FOR_MY_UTILES(q) {
            if (st.act) {
                const Pair<float> r32{to_f(st.s * __ldg(bb + q.x)), to_f(st.s * __ldg(bb + q.x + V))};
                st_f(P.r32, q.x, r32);
                st_f(P.x32, q.x, zf);
                v += (double)(norm2(r32.a) + norm2(r32.b));
            } else {
                st_d(t64, V, q.x, z);
            }
        }
        if (!ureduce<RS>(gs, v, P, smem, s_st, s_fl, RED_RR0, 0)) return false;
    }
    for (k = 1; k <= P.maxiter; k++) {
        if (!s_fl[FL_ACT]) break;
        float4* qn = cur ? P.q1 : P.q0;
        const float4* qo = cur ? P.q0 : P.q1;
        {   // p = r + beta p_old, t = g5Dw p, <p, A p> = |t|^2
            float f = 0.f;   // per-thread sum in FP32, one conversion per phase
            const RepState st = s_st[myr];
            if (st.act) {
                const SpAxpy<float, SpF> Q{SpF{P.r32}, SpF{qo}, (float)st.beta, !st.first};
                FOR_MY_UTILES(q) {
                    const Pair<float> c = Q.ld(q.x);
                    const Pair<float> tt = g5dw_at_c<float>(Q, c, Lf, q, m2f);
                    st_f(qn, q.x, c);
                    st_f(P.t32, q.x, tt);
                    f += norm2(tt.a) + norm2(tt.b);
                }
            }
            if (!ureduce<RS>(gs, (double)f, P, smem, s_st, s_fl, RED_PAP, k)) return false;
        }
        {   // x += alpha p, r -= alpha g5Dw t
            float f = 0.f;
            const RepState st = s_st[myr];
            if (st.act) {
                const float alpha = (float)st.alpha;
                if (pend) {
                    FOR_MY_UTILES(q) {   // x += apend p_old, then x += alpha p
                        const Pair<float> po = SpF{qo}.ld(q.x), pc = SpF{qn}.ld(q.x);
                        const Pair<float> a = g5dw_at<float>(SpF{P.t32}, Lf, q, m2f);
                        Pair<float> xv = SpF{P.x32}.ld(q.x), r = SpF{P.r32}.ld(q.x);
                        xv.a = xv.a + apend * po.a;
                        xv.b = xv.b + apend * po.b;
                        xv.a = xv.a + alpha * pc.a;
                        xv.b = xv.b + alpha * pc.b;
                        r.a = r.a - alpha * a.a;
                        r.b = r.b - alpha * a.b;
                        st_f(P.x32, q.x, xv);
                        st_f(P.r32, q.x, r);
                        f += norm2(r.a) + norm2(r.b);
                    }
                } else {
                    FOR_MY_UTILES(q) {   // x's update waits for the next iteration
                        const Pair<float> a = g5dw_at<float>(SpF{P.t32}, Lf, q, m2f);
                        Pair<float> r = SpF{P.r32}.ld(q.x);
                        r.a = r.a - alpha * a.a;
                        r.b = r.b - alpha * a.b;
                        st_f(P.r32, q.x, r);
                        f += norm2(r.a) + norm2(r.b);
                    }
                }
                apend = alpha;
                pend = !pend;
            }
            if (!ureduce<RS>(gs, (double)f, P, smem, s_st, s_fl, RED_RN, k)) return false;
        }
        if (s_fl[FL_UPD]) {   // FP64 reliable update of the replicas that asked for one
            const RepState st = s_st[myr];
            const double inv_s = 1.0 / st.s;
            if (st.upd) FOR_MY_UTILES(q) {   // x += x32 / s, with this iteration's x32 update if it waits
                    Pair<float> d = SpF{P.x32}.ld(q.x);
                    if (pend) {
                        const Pair<float> pc = SpF{qn}.ld(q.x);
                        d.a = d.a + apend * pc.a;
                        d.b = d.b + apend * pc.b;
                    }
                    Pair<double> xv = SpD{xx, V}.ld(q.x);
                    xv.a = xv.a + inv_s * to_d(d.a);
                    xv.b = xv.b + inv_s * to_d(d.b);
                    st_d(xx, V, q.x, xv);
                    st_f(P.x32, q.x, zf);
                }
            if (st.upd) pend = false;
            if (!gs.sync()) return false;
            if (st.upd) FOR_MY_UTILES(q) st_d(t64, V, q.x, g5dw_at<double>(SpD{xx, V}, L, q, m2));
            if (!gs.sync()) return false;
            double w = 0.0;
            if (st.upd) FOR_MY_UTILES(q) {   // r64 = b - A x
                    const Pair<double> a = g5dw_at<double>(SpD{t64, V}, L, q, m2);
                    Pair<double> r;
                    r.a = __ldg(bb + q.x) - a.a;
                    r.b = __ldg(bb + q.x + V) - a.b;
                    st_d(r64, V, q.x, r);
                    w += norm2(r.a) + norm2(r.b);
                }
            if (!ureduce<RS>(gs, w, P, smem, s_st, s_fl, RED_TRUE, k)) return false;
            if (s_fl[FL_R4]) {
                double v = 0.0;
                const RepState st4 = s_st[myr];
                if (st4.r4) FOR_MY_UTILES(q) {   // r32 = s_new r64
                        const Pair<float> r32{to_f(st4.snew * r64[q.x]), to_f(st4.snew * r64[q.x + V])};
                        st_f(P.r32, q.x, r32);
                        v += (double)(norm2(r32.a) + norm2(r32.b));
                    }
                if (!ureduce<RS>(gs, v, P, smem, s_st, s_fl, RED_R4, k)) return false;
            }
        }
        cur ^= 1;
    }
    return true;
}
#undef FOR_MY_UTILES

// Tiles of 32 x TYv sites, TYv = 4, 8 or 16 (blocks of 128, 256 or 512 threads):
// the tile height sets how many blocks share a replica's tiles (and its
// barriers) and how many tiles each block walks; the register budget (64 per
// thread) is the same for all three.  Different heights group the partial sums
// differently, so they agree to rounding, not bit for bit.
template <int RS, int TYv>
__global__ void __launch_bounds__(32 * TYv, 32 / TYv) k_u_cg_mixed(const UCGP P) {
    __shared__ double smem[32];
    __shared__ RepState s_st[kUniformReps];
    __shared__ int s_fl[FL_N];
    if (threadIdx.x < FL_N) s_fl[threadIdx.x] = 0;
    __syncthreads();
    int k = 0;
    if constexpr (RS >= 2) {   // independent replicas: a barrier per replica; its blocks leave when it is done
        const int myr = blockIdx.x / P.bpr;
        GridSync gs{P.rbar + 16 * myr, &P.ctl->gen, &P.ctl->err, (unsigned)P.bpr};
        const bool ok = u_body<RS, TYv>(P, gs, k, smem, s_st, s_fl);
        if (blockIdx.x == myr * P.bpr && threadIdx.x == 0) {   // the replica's first block
            if (ok) P.st_out[myr] = s_st[myr];
            DevCtl* c = P.ctl;
            if (myr == 0) c->last_iters = k;
            if (ld_volatile_int(&c->err) || !ok) atomicCAS(&c->status, 0, QED2D_ERR_TIMEOUT);
        }
        return;
    }
    GridSync gs{&P.ctl->bar, &P.ctl->gen, &P.ctl->err};
    const bool ok = u_body<RS, TYv>(P, gs, k, smem, s_st, s_fl);
    if (blockIdx.x == 0) {
        if (ok)   // every block holds the same records: block 0 stores them
            for (int r = threadIdx.x; r < P.g.B; r += blockDim.x) P.st_out[r] = s_st[r];
        if (threadIdx.x == 0) {
            DevCtl* c = P.ctl;
            c->last_iters = k;
            if (c->status == 0 && (ld_volatile_int(&c->err) || !ok)) c->status = QED2D_ERR_TIMEOUT;
        }
    }
}

}  // namespace qed2d
