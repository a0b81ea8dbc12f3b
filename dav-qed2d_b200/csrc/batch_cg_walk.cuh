// batch_cg_walk.cuh -- the column-walk form of the equal-size batched mixed CG
// (k_u_cg_mixed<RS, TYv, true>).
//
// Same recurrences, reductions, barriers and memory layout as u_body
// (batch_cg_uniform.cuh); only the mapping of sites to threads differs.  A
// block's tiles (32 x TYv sites) are dealt to its 8 warps, and a warp walks its
// tile down the rows: lane l holds column t1*32 + l, and step j of the walk
// computes row j.  In the two FP32 stencil phases of an iteration the rows above
// and below a site are the walk's previous and next steps, kept in registers,
// and the columns left and right are the neighbouring lanes (warp shuffles), so
// each site's spinor is read from memory once per phase instead of five times,
// p = r + beta p_old is formed once per site instead of five times, and the
// links of x - 1 come from the lane to the left.  Lanes 0 and 31 (and the lane
// whose right neighbour wraps around the lattice) load their missing
// neighbour.  Rows are prefetched through a per-warp ring in shared memory.
//
// Every site's FP32 values (p, g5Dw p, the r and x updates) are computed by the
// same operations as in u_body, so they are bitwise the same for the same
// alpha and beta; the per-thread partial sums run over other sites, so the
// reductions -- and hence alpha, beta and the iteration path -- agree with
// u_body to rounding, not bit for bit.  The FP64 phases (set-up and reliable
// updates) visit the same sites with the walk's mapping and per-site code.
#pragma once

namespace qed2d {

constexpr int kWalkWarps = 8;   // warps per block of the walk kernels (256 threads)

__device__ __forceinline__ float4 shfl_down4(float4 v) {
    return make_float4(__shfl_down_sync(0xffffffffu, v.x, 1), __shfl_down_sync(0xffffffffu, v.y, 1),
                       __shfl_down_sync(0xffffffffu, v.z, 1), __shfl_down_sync(0xffffffffu, v.w, 1));
}
__device__ __forceinline__ float4 shfl_up4(float4 v) {
    return make_float4(__shfl_up_sync(0xffffffffu, v.x, 1), __shfl_up_sync(0xffffffffu, v.y, 1),
                       __shfl_up_sync(0xffffffffu, v.z, 1), __shfl_up_sync(0xffffffffu, v.w, 1));
}
__device__ __forceinline__ float4 pk(const Pair<float>& p) { return make_float4(p.a.x, p.a.y, p.b.x, p.b.y); }
__device__ __forceinline__ Pair<float> upk(float4 q) { return {make_float2(q.x, q.y), make_float2(q.z, q.w)}; }

// the walk geometry of one tile held by a warp: columns (clamped for loads),
// the neighbouring columns with the periodic wrap, and the rows
struct WalkCol {
    int c1, p1c, m1c, r0, nrow, rowbase;
    bool ok, edge_p, edge_m;
};
__device__ __forceinline__ WalkCol walk_col(const UGeom& g, int r, int t1, int t2, int tyv, int lane) {
    WalkCol w;
    const int i1 = t1 * TX + lane;
    w.ok = i1 < g.L1;
    w.c1 = w.ok ? i1 : g.L1 - 1;
    w.p1c = (w.c1 + 1 == g.L1) ? 0 : w.c1 + 1;
    w.m1c = (w.c1 == 0) ? g.L1 - 1 : w.c1 - 1;
    w.edge_p = lane == TX - 1 || w.c1 + 1 >= g.L1;   // x + 1 is not lane + 1's site
    w.edge_m = lane == 0;                            // tiles start at multiples of 32
    w.r0 = t2 * tyv;
    w.nrow = min(tyv, g.L2 - w.r0);
    w.rowbase = r * g.L2;   // first row of replica r in the global row numbering
    return w;
}
// site index of (column c, row i2) of the walk's replica
__device__ __forceinline__ int wx(const UGeom& g, const WalkCol& w, int c, int i2) {
    return c + g.L1 * (w.rowbase + i2);
}

// Row prefetch: each warp streams its tile's rows (the row above the tile, its
// rows, the row below) through a ring of kWalkDepth stages in shared memory with
// cp.async (16 bytes per lane per array, through L2), so rows are requested
// kWalkDepth - 1 steps before they are used without holding registers.  A lane
// reads back only the slots it copied itself, so the ring needs no barrier: the
// lane's cp.async.wait_group is enough.  A stage is refilled one step after it
// was read, once every value taken from it has been used.  Per stage and warp:
// three 32-lane arrays (phase A: r, p_old, links; phase B: t, r, links) and five
// edge slots (lane 0: the spinor arrays and links of column x - 1; the lane
// whose right neighbour is not lane + 1: the spinor arrays of column x + 1).
constexpr int kWalkDepth = 4;
constexpr int kRingStage = 3 * 32 + 5;   // float4 slots per stage and warp
constexpr size_t kWalkSmem = sizeof(float4) * kWalkWarps * kWalkDepth * kRingStage;

__device__ __forceinline__ void cp16(float4* dst, const float4* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Phase A: p = r + beta p_old, t = g5Dw p; returns this thread's sum of |t|^2.
template <int TYv>
__device__ __forceinline__ float walk_phase_a(const UCGP& P, int myr, const TileRange& TR, float4* qn,
                                              const float4* qo, float beta, bool use_p, float m2f, float4* ring) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const UGeom& g = P.g;
    float4* wr = ring + warp * (kWalkDepth * kRingStage);
    float f = 0.f;
    auto form = [&](float4 r, float4 po) -> Pair<float> {   // as SpAxpy::ld
        Pair<float> v = upk(r);
        if (use_p) {
            const Pair<float> w = upk(po);
            v.a = v.a + beta * w.a;
            v.b = v.b + beta * w.b;
        }
        return v;
    };
    for (int tt = TR.lo + warp; tt < TR.hi; tt += kWalkWarps) {
        const int t2 = tt / TR.nt1, t1 = tt - t2 * TR.nt1;
        const WalkCol w = walk_col(g, myr, t1, t2, TYv, lane);
        const int nstream = w.nrow + 2;   // the row above, the tile's rows, the row below
        const bool iss_p = w.edge_p && w.ok;
        auto row_of = [&](int k) {   // stream position k -> lattice row (periodic)
            int i2 = w.r0 - 1 + k;
            return i2 < 0 ? i2 + g.L2 : (i2 >= g.L2 ? i2 - g.L2 : i2);
        };
        auto issue = [&](int k) {
            if (k < nstream) {
                float4* st = wr + (k % kWalkDepth) * kRingStage;
                const int xr = wx(g, w, 0, row_of(k));
                cp16(st + lane, P.r32 + xr + w.c1);
                if (use_p) cp16(st + 32 + lane, qo + xr + w.c1);
                cp16(st + 64 + lane, P.U32 + xr + w.c1);
                if (w.edge_m) {
                    cp16(st + 96, P.r32 + xr + w.m1c);
                    if (use_p) cp16(st + 97, qo + xr + w.m1c);
                    cp16(st + 98, P.U32 + xr + w.m1c);
                }
                if (iss_p) {
                    cp16(st + 99, P.r32 + xr + w.p1c);
                    if (use_p) cp16(st + 100, qo + xr + w.p1c);
                }
            }
            cp_commit();
        };
        for (int k = 0; k < kWalkDepth; k++) issue(k);
        Pair<float> pm{}, pc{};
        float2 u2m{};
        float4 uc{};
        Pair<float> em{}, ep{};
        float2 eu{};
        for (int k = 0; k < nstream; k++) {
            cp_wait<kWalkDepth - 2>();
            const float4* st = wr + (k % kWalkDepth) * kRingStage;
            const Pair<float> pk_ = form(st[lane], use_p ? st[32 + lane] : make_float4(0, 0, 0, 0));
            const float4 uk = st[64 + lane];
            Pair<float> emk{}, epk{};
            float2 euk{};
            if (w.edge_m) {
                emk = form(st[96], use_p ? st[97] : make_float4(0, 0, 0, 0));
                const float4 q = st[98];
                euk = make_float2(q.x, q.y);
            }
            if (w.edge_p) epk = form(st[99], use_p ? st[100] : make_float4(0, 0, 0, 0));
            if (k >= 2) {   // row k - 1 of the stream = tile row k - 2
                const int x = wx(g, w, w.c1, w.r0 + k - 2);
                Pair<float> p1 = upk(shfl_down4(pk(pc))), m1 = upk(shfl_up4(pk(pc)));
                float2 u1m = make_float2(__shfl_up_sync(0xffffffffu, uc.x, 1), __shfl_up_sync(0xffffffffu, uc.y, 1));
                if (w.edge_p) p1 = ep;
                if (w.edge_m) {
                    m1 = em;
                    u1m = eu;
                }
                Pair<float> t;
                g5dw_site<float>(pc.a, pc.b, p1.a, p1.b, m1.a, m1.b, pk_.a, pk_.b, pm.a, pm.b,
                                 make_float2(uc.x, uc.y), make_float2(uc.z, uc.w), u1m, u2m, m2f, t.a, t.b);
                if (w.ok) {
                    st_f(qn, x, pc);
                    st_f(P.t32, x, t);
                    f += norm2(t.a) + norm2(t.b);
                }
            }
            if (k >= 1) issue(k - 1 + kWalkDepth);   // stage of row k - 1: all its values are used
            if (k >= 1) u2m = make_float2(uc.z, uc.w);
            pm = pc;
            pc = pk_;
            uc = uk;
            em = emk;
            ep = epk;
            eu = euk;
        }
        cp_wait<0>();
    }
    return f;
}

// Phase B: r -= alpha g5Dw t, with the x update (two directions when `pend`);
// returns this thread's sum of |r|^2.
template <int TYv, bool PEND>
__device__ __forceinline__ float walk_phase_b(const UCGP& P, int myr, const TileRange& TR, const float4* qn,
                                              const float4* qo, float alpha, float apend, float m2f, float4* ring) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const UGeom& g = P.g;
    float4* wr = ring + warp * (kWalkDepth * kRingStage);
    float f = 0.f;
    for (int tt = TR.lo + warp; tt < TR.hi; tt += kWalkWarps) {
        const int t2 = tt / TR.nt1, t1 = tt - t2 * TR.nt1;
        const WalkCol w = walk_col(g, myr, t1, t2, TYv, lane);
        const int nstream = w.nrow + 2;
        const bool iss_p = w.edge_p && w.ok;
        auto row_of = [&](int k) {
            int i2 = w.r0 - 1 + k;
            return i2 < 0 ? i2 + g.L2 : (i2 >= g.L2 ? i2 - g.L2 : i2);
        };
        auto issue = [&](int k) {
            if (k < nstream) {
                float4* st = wr + (k % kWalkDepth) * kRingStage;
                const int xr = wx(g, w, 0, row_of(k));
                cp16(st + lane, P.t32 + xr + w.c1);
                cp16(st + 32 + lane, P.r32 + xr + w.c1);
                cp16(st + 64 + lane, P.U32 + xr + w.c1);
                if (w.edge_m) {
                    cp16(st + 96, P.t32 + xr + w.m1c);
                    cp16(st + 98, P.U32 + xr + w.m1c);
                }
                if (iss_p) cp16(st + 99, P.t32 + xr + w.p1c);
            }
            cp_commit();
        };
        for (int k = 0; k < kWalkDepth; k++) issue(k);
        float4 tm{}, tc{}, uc{}, rc{};
        float2 u2m{}, eu{};
        Pair<float> em{}, ep{};
        for (int k = 0; k < nstream; k++) {
            cp_wait<kWalkDepth - 2>();
            const float4* st = wr + (k % kWalkDepth) * kRingStage;
            const float4 tk = st[lane], rk = st[32 + lane], uk = st[64 + lane];
            Pair<float> emk{}, epk{};
            float2 euk{};
            if (w.edge_m) {
                emk = upk(st[96]);
                const float4 q = st[98];
                euk = make_float2(q.x, q.y);
            }
            if (w.edge_p) epk = upk(st[99]);
            if (k >= 2) {   // tile row k - 2
                const int x = wx(g, w, w.c1, w.r0 + k - 2);
                Pair<float> xv, pc, po;
                if constexpr (PEND) {
                    xv = SpF{P.x32}.ld(x);
                    pc = SpF{qn}.ld(x);
                    po = SpF{qo}.ld(x);
                }
                Pair<float> t1p = upk(shfl_down4(tc)), t1m = upk(shfl_up4(tc));
                float2 u1m = make_float2(__shfl_up_sync(0xffffffffu, uc.x, 1), __shfl_up_sync(0xffffffffu, uc.y, 1));
                if (w.edge_p) t1p = ep;
                if (w.edge_m) {
                    t1m = em;
                    u1m = eu;
                }
                const Pair<float> c = upk(tc), tpn = upk(tk), tmm = upk(tm);
                Pair<float> a;
                g5dw_site<float>(c.a, c.b, t1p.a, t1p.b, t1m.a, t1m.b, tpn.a, tpn.b, tmm.a, tmm.b,
                                 make_float2(uc.x, uc.y), make_float2(uc.z, uc.w), u1m, u2m, m2f, a.a, a.b);
                if (w.ok) {
                    if constexpr (PEND) {   // x += apend p_old, then x += alpha p
                        xv.a = xv.a + apend * po.a;
                        xv.b = xv.b + apend * po.b;
                        xv.a = xv.a + alpha * pc.a;
                        xv.b = xv.b + alpha * pc.b;
                        st_f(P.x32, x, xv);
                    }
                    Pair<float> r = upk(rc);
                    r.a = r.a - alpha * a.a;
                    r.b = r.b - alpha * a.b;
                    st_f(P.r32, x, r);
                    f += norm2(r.a) + norm2(r.b);
                }
            }
            if (k >= 1) issue(k - 1 + kWalkDepth);
            if (k >= 1) u2m = make_float2(uc.z, uc.w);
            tm = tc;
            tc = tk;
            rc = rk;
            uc = uk;
            em = emk;
            ep = epk;
            eu = euk;
        }
        cp_wait<0>();
    }
    return f;
}

// every site of this block, visited with the walk's mapping (warp w: tiles
// lo + w, lo + w + 8, ...; row j of the tile at step j)
#define FOR_MY_WSITES(q)                                                                                  \
    for (int tt_ = TR.lo + (threadIdx.x >> 5); tt_ < TR.hi; tt_ += kWalkWarps)                           \
        for (int j_ = 0, t2_ = tt_ / TR.nt1, t1_ = tt_ - t2_ * TR.nt1; j_ < TYv; ++j_)                   \
            if (const Site q = usite_at<TYv>(P.g, myr, t1_, t2_, (j_ << 5) | (threadIdx.x & 31)); q.ok)

template <int RS, int TYv>
__device__ __forceinline__ bool w_body(const UCGP& P, GridSync& gs, int& k, double* smem, RepState* s_st,
                                       int* s_fl) {
    extern __shared__ float4 ring[];   // kWalkSmem bytes: the warps' row rings
    const int myr = blockIdx.x / P.bpr, lb = blockIdx.x - myr * P.bpr;
    const TileRange TR = tile_range(P.g.ntr, P.g.nt1, P.per_block, lb);
    const long long V = P.g.V, sh = (long long)myr * V;
    const double2* bb = P.b + sh;
    double2* xx = P.x + sh;
    double2* r64 = P.r64 + sh;
    double2* t64 = P.t64 + sh;
    const LkD L{P.U + sh, V};
    const double m2 = P.m2[myr];
    const float m2f = (float)m2;
    const Pair<double> z{make_double2(0, 0), make_double2(0, 0)};
    const Pair<float> zf{make_float2(0, 0), make_float2(0, 0)};
    int cur = 0;
    bool pend = false;   // as u_body: x32 += alpha p every second iteration, two directions at once
    float apend = 0.f;

    {   // |b|^2 per replica; x = 0
        double v = 0.0;
        FOR_MY_WSITES(q) {
            const Pair<double> bv{__ldg(bb + q.x), __ldg(bb + q.x + V)};
            v += norm2(bv.a) + norm2(bv.b);
            st_d(xx, V, q.x, z);
        }
        if (!ureduce<RS>(gs, v, P, smem, s_st, s_fl, RED_BB, 0)) return false;
    }
    {   // r32 = s b, x32 = 0
        double v = 0.0;
        const RepState st = s_st[myr];
        FOR_MY_WSITES(q) {
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
            float f = 0.f;
            const RepState st = s_st[myr];
            if (st.act) f = walk_phase_a<TYv>(P, myr, TR, qn, qo, (float)st.beta, !st.first, m2f, ring);
            if (!ureduce<RS>(gs, (double)f, P, smem, s_st, s_fl, RED_PAP, k)) return false;
        }
        {   // x += alpha p, r -= alpha g5Dw t
            float f = 0.f;
            const RepState st = s_st[myr];
            if (st.act) {
                const float alpha = (float)st.alpha;
                f = pend ? walk_phase_b<TYv, true>(P, myr, TR, qn, qo, alpha, apend, m2f, ring)
                         : walk_phase_b<TYv, false>(P, myr, TR, qn, qo, alpha, apend, m2f, ring);
                apend = alpha;
                pend = !pend;
            }
            if (!ureduce<RS>(gs, (double)f, P, smem, s_st, s_fl, RED_RN, k)) return false;
        }
        if (s_fl[FL_UPD]) {   // FP64 reliable update of the replicas that asked for one
            const RepState st = s_st[myr];
            const double inv_s = 1.0 / st.s;
            if (st.upd) FOR_MY_WSITES(q) {
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
            if (st.upd) FOR_MY_WSITES(q) st_d(t64, V, q.x, g5dw_at<double>(SpD{xx, V}, L, q, m2));
            if (!gs.sync()) return false;
            double w = 0.0;
            if (st.upd) FOR_MY_WSITES(q) {   // r64 = b - A x
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
                if (st4.r4) FOR_MY_WSITES(q) {   // r32 = s_new r64
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
#undef FOR_MY_WSITES

}  // namespace qed2d
