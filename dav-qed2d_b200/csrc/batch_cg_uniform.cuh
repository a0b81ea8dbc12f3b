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

#include "tma.cuh"

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

// ---------------------------------------------------------------------------
// TMA staging of the stencil operands (schedule 7; lattices of whole 32 x TYv
// tiles, L1 a multiple of 32).  The FP32 spinor fields are 2D float32 tensors of
// (4 L1) x (B L2) elements (a replica's rows follow the previous replica's), the
// link planes (2 L1) x (B L2).  For a tile, one box of the tile itself and four
// one-wide boxes of its neighbours (the columns left and right, the rows below
// and above), each at explicitly wrapped coordinates inside its own replica, so
// no box leaves the tensor and every x coordinate is a multiple of 16 bytes
// (4 floats; the link planes' left column is loaded two sites wide from i1 - 2).
struct UTma {
    // per spinor field (r32, q0, q1, t32): tile box, column box, row box
    CUtensorMap fc[4], fk[4], fw[4];
    CUtensorMap u1c, u1l, u2c, u2b;   // link planes: tile boxes, u1's left columns, u2's lower row
};
enum { TF_R = 0, TF_Q0 = 1, TF_Q1 = 2, TF_T = 3 };
constexpr int kTmaStages = 2;   // stages per block: tiles staged one ahead (three measured slower)

// one stage: a spinor field's five boxes (tile [TYv][32], left and right
// columns [TYv], lower and upper rows [32]), float4 each, at 128-byte aligned
// offsets; two spinor slots, then the link boxes
template <int TYv>
struct UStage {
    static constexpr int C = TYv * 32 * 16, K = TYv * 16, W = 32 * 16;
    static constexpr int FIELD = C + 2 * K + 2 * W;               // one spinor field's boxes
    static constexpr int U1C = 2 * FIELD, U1L = U1C + TYv * 32 * 8;
    static constexpr int U2C = U1L + TYv * 16, U2B = U2C + TYv * 32 * 8;
    static constexpr int BYTES = U2B + 32 * 8;
    static constexpr int LINKS = BYTES - U1C;
    static_assert(TYv < 8 || (C % 128 == 0 && K % 128 == 0 && FIELD % 128 == 0 && U1L % 128 == 0 &&
                              U2C % 128 == 0 && U2B % 128 == 0),
                  "TMA destinations must be 128-byte aligned (tile heights of 8 rows and more)");
};

// The five values of a spinor field around site (lx, ly) of the tile staged at
// `f` (pointer selects, so edge lanes take the halo without diverging).
template <int TYv>
__device__ __forceinline__ void tma_ld5(const char* f, int lx, int ly, Pair<float>& c, Pair<float>& p1,
                                        Pair<float>& m1, Pair<float>& p2, Pair<float>& mm2) {
    using S = UStage<TYv>;
    const float4* C = reinterpret_cast<const float4*>(f);
    const float4* K0 = reinterpret_cast<const float4*>(f + S::C);
    const float4* K1 = reinterpret_cast<const float4*>(f + S::C + S::K);
    const float4* W0 = reinterpret_cast<const float4*>(f + S::C + 2 * S::K);
    const float4* W1 = reinterpret_cast<const float4*>(f + S::C + 2 * S::K + S::W);
    const int o = ly * 32 + lx;
    const float4 vc = C[o];
    const float4 vp1 = *(lx < 31 ? C + o + 1 : K1 + ly);
    const float4 vm1 = *(lx > 0 ? C + o - 1 : K0 + ly);
    const float4 vp2 = *(ly < TYv - 1 ? C + o + 32 : W1 + lx);
    const float4 vm2 = *(ly > 0 ? C + o - 32 : W0 + lx);
    c = {make_float2(vc.x, vc.y), make_float2(vc.z, vc.w)};
    p1 = {make_float2(vp1.x, vp1.y), make_float2(vp1.z, vp1.w)};
    m1 = {make_float2(vm1.x, vm1.y), make_float2(vm1.z, vm1.w)};
    p2 = {make_float2(vp2.x, vp2.y), make_float2(vp2.z, vp2.w)};
    mm2 = {make_float2(vm2.x, vm2.y), make_float2(vm2.z, vm2.w)};
}

// the four links of site (lx, ly)'s stencil from the staged link boxes
template <int TYv>
__device__ __forceinline__ void tma_links(const char* st, int lx, int ly, float2& u1x, float2& u2x, float2& u1m1,
                                          float2& u2m2) {
    using S = UStage<TYv>;
    const float2* U1 = reinterpret_cast<const float2*>(st + S::U1C);
    const float2* U1L = reinterpret_cast<const float2*>(st + S::U1L);
    const float2* U2 = reinterpret_cast<const float2*>(st + S::U2C);
    const float2* U2B = reinterpret_cast<const float2*>(st + S::U2B);
    const int o = ly * 32 + lx;
    u1x = U1[o];
    u2x = U2[o];
    u1m1 = *(lx > 0 ? U1 + o - 1 : U1L + 2 * ly + 1);   // the left box holds sites i1 - 2 and i1 - 1
    u2m2 = *(ly > 0 ? U2 + o - 32 : U2B + lx);
}

// Thread 0: the boxes of tile (t1, t2) of replica r into stage `st`, completing
// on `bar`: spinor fields f0 (and f1 when f1 >= 0) and the links.
template <int TYv>
__device__ __forceinline__ void tma_issue(const UTma& T, const UGeom& g, char* st, uint64_t* bar, int r, int t1,
                                          int t2, int f0, int f1) {
    using S = UStage<TYv>;
    const int L1 = g.L1, L2 = g.L2;
    const int y = r * L2 + t2 * TYv;
    const int ylo = r * L2 + (t2 == 0 ? L2 - 1 : t2 * TYv - 1);
    const int yhi = r * L2 + ((t2 + 1) * TYv == L2 ? 0 : (t2 + 1) * TYv);
    const int xl = t1 == 0 ? L1 - 1 : 32 * t1 - 1, xr = (32 * t1 + 32) % L1;
    const int nf = f1 >= 0 ? 2 : 1;
    mbar_arrive_expect_tx(bar, nf * S::FIELD + S::LINKS);
    for (int j = 0; j < nf; j++) {
        const int f = j ? f1 : f0;
        char* d = st + j * S::FIELD;
        tma_load_2d(d, &T.fc[f], 128 * t1, y, bar);
        tma_load_2d(d + S::C, &T.fk[f], 4 * xl, y, bar);
        tma_load_2d(d + S::C + S::K, &T.fk[f], 4 * xr, y, bar);
        tma_load_2d(d + S::C + 2 * S::K, &T.fw[f], 128 * t1, ylo, bar);
        tma_load_2d(d + S::C + 2 * S::K + S::W, &T.fw[f], 128 * t1, yhi, bar);
    }
    tma_load_2d(st + S::U1C, &T.u1c, 64 * t1, y, bar);
    tma_load_2d(st + S::U1L, &T.u1l, 2 * (t1 == 0 ? L1 - 2 : 32 * t1 - 2), y, bar);
    tma_load_2d(st + S::U2C, &T.u2c, 64 * t1, y, bar);
    tma_load_2d(st + S::U2B, &T.u2b, 64 * t1, ylo, bar);
}

// TMA: the stencil operands of phases A and B come through shared memory
// (T: the tensor maps; stg: kTmaStages stages; bar: their mbarriers), staged up
// to kTmaStages - 1 tiles ahead.
// RSTEN (schedule 8): phase A applies the stencil to r instead of p, t = g5Dw r
// + beta t_old (g5Dw is linear, so t = g5Dw p as before), and forms p only at
// the thread's own site: 7 float4 loads per site instead of 10 and no p at the
// four neighbours.  Same recurrences; t carries the rounding of its own
// recurrence (the Chronopoulos-Gear form of the direction update), so the bits
// differ from the other schedules while the FP64 stop rule is unchanged.  After
// a reliable update the rescaled beta of RED_R4 keeps t = g5Dw p, as it keeps p.
// LSM (schedule 9 with RSTEN): the FP32 links of the block's tiles staged once
// per solve in shared memory (ULsm, stencil.cuh).  The links do not change
// during a solve, and the values are those of the global planes.

template <int RS, int TYv, bool TMA = false, bool RSTEN = false, bool LSM = false>
__device__ __forceinline__ bool u_body(const UCGP& P, const UTma* T, char* stg, uint64_t* bar, GridSync& gs, int& k,
                                       double* smem, RepState* s_st, int* s_fl, const float2* lsm = nullptr) {
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
    // TMA staging: kTmaStages stages, the next to compute (sg), the mbarrier phase
    // parities, this thread's site in the tile
    constexpr int SB = UStage<TYv>::BYTES, NS = kTmaStages;
    int sg = 0;
    unsigned par = 0u;   // bit s: the phase parity stage s waits for next
    const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
    // Runs fn(stage, t1, t2) over the block's tiles with fields f0 (and f1) and
    // the links of each tile staged, NS - 1 tiles ahead; a block barrier after
    // each tile frees its stage for the next copy.  False (with no copy in
    // flight) when a stage's copies did not complete.  (Per-stage "read"
    // mbarriers with one arrival per warp instead of the block barrier measured
    // slower: 4x512^2 33.5 -> 35.4 us per iteration.)
    auto staged = [&](int f0, int f1, auto&& fn) -> bool {
        const int n = TR.hi - TR.lo;
        int t1 = TR.s1, t2 = TR.s2, i1 = TR.s1, i2 = TR.s2, issued = 0, si = sg;
        if (threadIdx.x == 0) fence_proxy_async_global();   // the phase reads what the last one wrote
        auto issue = [&]() {
            if (threadIdx.x == 0) {
                fence_proxy_async_shared();
                tma_issue<TYv>(*T, P.g, stg + si * SB, bar + si, myr, i1, i2, f0, f1);
            }
            if (++i1 == TR.nt1) i1 = 0, ++i2;
            si = si + 1 == NS ? 0 : si + 1;
            ++issued;
        };
        while (issued < n && issued < NS - 1) issue();
        for (int k = 0; k < n; k++) {
            if (issued < n) issue();   // into the stage tile k - 1 released
            const bool ok = mbar_wait(bar + sg, (par >> sg) & 1u, gs.err);
            par ^= 1u << sg;
            fn((const char*)(stg + sg * SB), t1, t2);
            if (++t1 == TR.nt1) t1 = 0, ++t2;
            sg = sg + 1 == NS ? 0 : sg + 1;
            if (!__syncthreads_and(ok)) {   // drain the copies still in flight, then give up
                for (int j = k + 1, s2 = sg; j < issued; j++, s2 = s2 + 1 == NS ? 0 : s2 + 1)
                    mbar_wait(bar + s2, (par >> s2) & 1u, gs.err);
                return false;
            }
        }
        return true;
    };

    // the FP32 stencil of spinor accessor S around site q of the block's tile j
    // (centre value c given), links from shared memory (LSM) or the planes
    auto sten = [&](const auto& S, const Pair<float>& c, const Site& q, int j) -> Pair<float> {
        if constexpr (LSM) return ULsm<TYv>::stencil(lsm, j, S, c, q, m2f);
        else return g5dw_at_c<float>(S, c, Lf, q, m2f);
    };
    if constexpr (LSM) {   // stage the links of the block's tiles
        FOR_MY_UTILES(q) ULsm<TYv>::stage(const_cast<float2*>(lsm), tt_ - TR.lo, Lf, q);
        __syncthreads();
    }
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
            if constexpr (TMA) {
                if (st.act) {   // r and p_old of the tile and its halo staged in shared memory
                    const float beta = (float)st.beta;
                    const bool use_p = !st.first;
                    const bool ok = staged(TF_R, cur ? TF_Q0 : TF_Q1, [&](const char* sb, int t1, int t2) {
                        Pair<float> c, p1, m1, p2, mm2;
                        tma_ld5<TYv>(sb, lx, ly, c, p1, m1, p2, mm2);
                        if (use_p) {
                            Pair<float> w, w1, wm1, w2, wm2;
                            tma_ld5<TYv>(sb + UStage<TYv>::FIELD, lx, ly, w, w1, wm1, w2, wm2);
                            c.a = c.a + beta * w.a;
                            c.b = c.b + beta * w.b;
                            p1.a = p1.a + beta * w1.a;
                            p1.b = p1.b + beta * w1.b;
                            m1.a = m1.a + beta * wm1.a;
                            m1.b = m1.b + beta * wm1.b;
                            p2.a = p2.a + beta * w2.a;
                            p2.b = p2.b + beta * w2.b;
                            mm2.a = mm2.a + beta * wm2.a;
                            mm2.b = mm2.b + beta * wm2.b;
                        }
                        float2 u1x, u2x, u1m1, u2m2;
                        tma_links<TYv>(sb, lx, ly, u1x, u2x, u1m1, u2m2);
                        Pair<float> tt_;
                        g5dw_site<float>(c.a, c.b, p1.a, p1.b, m1.a, m1.b, p2.a, p2.b, mm2.a, mm2.b, u1x, u2x, u1m1,
                                         u2m2, m2f, tt_.a, tt_.b);
                        const Site q = usite_at<TYv>(P.g, myr, t1, t2, threadIdx.x);
                        st_f(qn, q.x, c);
                        st_f(P.t32, q.x, tt_);
                        f += norm2(tt_.a) + norm2(tt_.b);
                    });
                    if (!ok) return false;
                }
            } else if (RSTEN && st.act) {
                const float beta = (float)st.beta;
                const bool use_p = !st.first;
                FOR_MY_UTILES(q) {
                    const Pair<float> rc = SpF{P.r32}.ld(q.x);
                    Pair<float> tt = sten(SpF{P.r32}, rc, q, tt_ - TR.lo), c = rc;
                    if (use_p) {   // p = r + beta p_old, t = g5Dw r + beta t_old
                        const Pair<float> po = SpF{qo}.ld(q.x), to = SpF{P.t32}.ld(q.x);
                        c.a = c.a + beta * po.a;
                        c.b = c.b + beta * po.b;
                        tt.a = tt.a + beta * to.a;
                        tt.b = tt.b + beta * to.b;
                    }
                    st_f(qn, q.x, c);
                    st_f(P.t32, q.x, tt);
                    f += norm2(tt.a) + norm2(tt.b);
                }
            } else if (st.act) {
                const SpAxpy<float, SpF> Q{SpF{P.r32}, SpF{qo}, (float)st.beta, !st.first};
                FOR_MY_UTILES(q) {
                    const Pair<float> c = Q.ld(q.x);
                    const Pair<float> tt = sten(Q, c, q, tt_ - TR.lo);
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
            if (TMA && st.act) {   // t of the tile and its halo staged in shared memory
                const float alpha = (float)st.alpha;
                const bool ok = staged(TF_T, -1, [&](const char* sb, int t1, int t2) {
                    const Site q = usite_at<TYv>(P.g, myr, t1, t2, threadIdx.x);
                    Pair<float> c, p1, m1, p2, mm2, a;
                    tma_ld5<TYv>(sb, lx, ly, c, p1, m1, p2, mm2);
                    float2 u1x, u2x, u1m1, u2m2;
                    tma_links<TYv>(sb, lx, ly, u1x, u2x, u1m1, u2m2);
                    g5dw_site<float>(c.a, c.b, p1.a, p1.b, m1.a, m1.b, p2.a, p2.b, mm2.a, mm2.b, u1x, u2x, u1m1, u2m2,
                                     m2f, a.a, a.b);
                    Pair<float> r = SpF{P.r32}.ld(q.x);
                    if (pend) {   // x += apend p_old, then x += alpha p
                        const Pair<float> po = SpF{qo}.ld(q.x), pc = SpF{qn}.ld(q.x);
                        Pair<float> xv = SpF{P.x32}.ld(q.x);
                        xv.a = xv.a + apend * po.a;
                        xv.b = xv.b + apend * po.b;
                        xv.a = xv.a + alpha * pc.a;
                        xv.b = xv.b + alpha * pc.b;
                        st_f(P.x32, q.x, xv);
                    }
                    r.a = r.a - alpha * a.a;
                    r.b = r.b - alpha * a.b;
                    st_f(P.r32, q.x, r);
                    f += norm2(r.a) + norm2(r.b);
                });
                if (!ok) return false;
                apend = alpha;
                pend = !pend;
            } else if (st.act) {
                const float alpha = (float)st.alpha;
                if (pend) {
                    FOR_MY_UTILES(q) {   // x += apend p_old, then x += alpha p
                        const Pair<float> po = SpF{qo}.ld(q.x), pc = SpF{qn}.ld(q.x);
                        const Pair<float> a = sten(SpF{P.t32}, SpF{P.t32}.ld(q.x), q, tt_ - TR.lo);
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
                        const Pair<float> a = sten(SpF{P.t32}, SpF{P.t32}.ld(q.x), q, tt_ - TR.lo);
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
template <int RS, int TYv, bool RSTEN = false, bool LSM = false>
__global__ void __launch_bounds__(32 * TYv, 32 / TYv) k_u_cg_mixed(const UCGP P) {
    extern __shared__ float2 lsm_dyn[];   // LSM: ULsm<TYv>::bytes(P.per_block)
    __shared__ double smem[32];
    __shared__ RepState s_st[kUniformReps];
    __shared__ int s_fl[FL_N];
    if (threadIdx.x < FL_N) s_fl[threadIdx.x] = 0;
    __syncthreads();
    int k = 0;
    if constexpr (RS >= 2) {   // independent replicas: a barrier per replica; its blocks leave when it is done
        const int myr = blockIdx.x / P.bpr;
        GridSync gs{P.rbar + 16 * myr, &P.ctl->gen, &P.ctl->err, (unsigned)P.bpr};
        const bool ok =
            u_body<RS, TYv, false, RSTEN, LSM>(P, nullptr, nullptr, nullptr, gs, k, smem, s_st, s_fl, lsm_dyn);
        if (blockIdx.x == myr * P.bpr && threadIdx.x == 0) {   // the replica's first block
            if (ok) P.st_out[myr] = s_st[myr];
            DevCtl* c = P.ctl;
            if (myr == 0) c->last_iters = k;
            if (ld_volatile_int(&c->err) || !ok) atomicCAS(&c->status, 0, QED2D_ERR_TIMEOUT);
        }
        return;
    }
    GridSync gs{&P.ctl->bar, &P.ctl->gen, &P.ctl->err};
    const bool ok = u_body<RS, TYv>(P, nullptr, nullptr, nullptr, gs, k, smem, s_st, s_fl);
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

// Schedule 7: schedule 5 (independent replicas, lean reduction) with the
// stencil operands of both CG phases staged by TMA one tile ahead (UTma).
// Lattices of whole tiles only (L1 % 32 == 0, L2 % TYv == 0).  The arithmetic,
// its order and the reductions are those of schedule 5, so the bits are too.
// Dynamic shared memory: kTmaStages stages plus 128 bytes of alignment slack.
template <int TYv>
__global__ void __launch_bounds__(32 * TYv, 32 / TYv)
    k_u_cg_mixed_tma(const __grid_constant__ UCGP P, const __grid_constant__ UTma T) {
    extern __shared__ char dyn[];
    __shared__ double smem[32];
    __shared__ RepState s_st[kUniformReps];
    __shared__ int s_fl[FL_N];
    __shared__ __align__(8) uint64_t s_bar[kTmaStages];   // stage filled
    char* stg = dyn + ((128u - (smem_addr(dyn) & 127u)) & 127u);
    if (threadIdx.x < FL_N) s_fl[threadIdx.x] = 0;
    if (threadIdx.x == 0) {
        for (int i = 0; i < kTmaStages; i++) mbar_init(&s_bar[i], 1);
        fence_mbar_init();
    }
    __syncthreads();
    int k = 0;
    const int myr = blockIdx.x / P.bpr;
    GridSync gs{P.rbar + 16 * myr, &P.ctl->gen, &P.ctl->err, (unsigned)P.bpr};
    const bool ok = u_body<3, TYv, true>(P, &T, stg, s_bar, gs, k, smem, s_st, s_fl);
    if (blockIdx.x == myr * P.bpr && threadIdx.x == 0) {   // the replica's first block
        if (ok) P.st_out[myr] = s_st[myr];
        DevCtl* c = P.ctl;
        if (myr == 0) c->last_iters = k;
        if (ld_volatile_int(&c->err) || !ok) atomicCAS(&c->status, 0, QED2D_ERR_TIMEOUT);
    }
}

}  // namespace qed2d
