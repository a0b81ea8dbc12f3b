// batch.cu -- batches of independent replica lattices, of equal or uneven sizes,
// advanced together (ensemble generation: many Markov chains per GPU).  Every
// kernel of an Nf=2 trajectory covers all replicas, and every force evaluation
// is ONE persistent mixed-precision CG launch that solves all replicas' systems
// at once, so the grid barriers and launch latencies of a solve are paid once
// for the whole batch.  Each replica follows exactly the algorithm of HMC! Nf=2
// (src/QED2dHMC.jl:64-113) with leapfrog (:426-481).
//
// Layout (replica-major): replica r's field is an ordinary reference-layout
// array ([L1_r, L2_r, 2], i1 fastest) starting at complex element 2*off_r, with
// off_r the number of sites of the replicas before r; real fields (momenta)
// start at real element 2*off_r.  Random draws of replica r use its own seed
// and the single-lattice element order, so replica r reproduces a
// single-lattice run with that seed.
//
// Work decomposition of the persistent solver: every replica's 32x8 tiles are
// cut into chunks, the chunks dealt round-robin over the replicas, and each
// block owns a contiguous range of that order, so one replica's work (its FP64
// reliable updates run while the others wait) is spread over many blocks.  A
// run of one replica's tiles inside a block is a "segment" with one partial
// sum (fixed order inside), so per-replica sums are deterministic.  The block
// arriving last at a barrier sums each replica's partials and either publishes
// the sums (at most 64 replicas: every block keeps all replicas' CG records in
// shared memory and updates them itself) or updates the records in global
// memory.  Standalone kernels (forces, link updates, sums) run one block per
// tile of a replica-major tile table.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <type_traits>
#include <vector>

#include "graph.h"
#include "stencil.cuh"

namespace qed2d {

constexpr int kMaxReplicas = 1024;
constexpr int kClusterSizes[3] = {4, 8, 16};   // blocks per cluster tried by the cluster solver's tuner

struct RepInfo {
    int L1, L2, nt1, nt;   // extents, tiles along i1, tiles of the replica
    long long V, off;      // sites, first site of the replica in the batch
    int tile0, pad;        // first entry of the replica in the tile table
};

__host__ __device__ __forceinline__ Lat lat_of(const RepInfo& R) { return Lat{R.L1, R.L2, R.V}; }

struct TileView {
    const RepInfo* reps;
    const int4* tiles;   // (replica, t1, t2, 0)
    long long vtot;      // sites of the batch (the stride of the FP32 link planes)
};

// ---------------------------------------------------------------------------
// standalone kernels: one block per entry of the tile table
__global__ void __launch_bounds__(TILE) k_r_g5dw(double2* __restrict__ so, const double2* __restrict__ U,
                                                 const double2* __restrict__ si, TileView tv,
                                                 const double* __restrict__ m2) {
    const int4 T = __ldg(tv.tiles + blockIdx.x);
    const RepInfo R = tv.reps[T.x];
    const Site q = site_at(lat_of(R), T.y, T.z, threadIdx.x);
    if (!q.ok) return;
    const long long o = 2 * R.off;
    st_d(so + o, R.V, q.x, g5dw_at<double>(SpDro{si + o, R.V}, LkD{U + o, R.V}, q, m2[T.x]));
}

// mom += eps (gauge force with beta_r + fermion force from (X, G = g5Dw X));
// gauge part as krnl_force! (src/QED2dAction.jl:25-52)
__global__ void __launch_bounds__(TILE) k_r_mom_kick(double* __restrict__ mom, const double2* __restrict__ U,
                                                     TileView tv, const double* __restrict__ beta, double eps,
                                                     const double2* __restrict__ X, const double2* __restrict__ G) {
    const int4 T = __ldg(tv.tiles + blockIdx.x);
    const RepInfo R = tv.reps[T.x];
    const Lat g = lat_of(R);
    const Site q = site_at(g, T.y, T.z, threadIdx.x);
    if (!q.ok) return;
    const long long o = 2 * R.off;
    double* m = mom + o;
    const double mo1 = m[q.x], mo2 = m[q.x + g.V];   // issued with the link loads
    double F1, F2;
    gauge_force_at(U + o, g, q, beta[T.x], F1, F2);
    if (X) {
        double f1, f2;
        fermion_force_at(U + o, X + o, G + o, g.V, q, f1, f2);
        F1 = F1 + f1;
        F2 = F2 + f2;
    }
    m[q.x] = mo1 + eps * F1;
    m[q.x + g.V] = mo2 + eps * F2;
}

// U <- exp(i eps mom) U (updt_fld!, src/QED2dAction.jl:55-65) and the packed FP32
// copy of the links; eps == 0 only packs
__global__ void __launch_bounds__(TILE) k_r_updt(double2* __restrict__ U, const double* __restrict__ mom, double eps,
                                                 float4* __restrict__ U32, TileView tv) {
    const int4 T = __ldg(tv.tiles + blockIdx.x);
    const RepInfo R = tv.reps[T.x];
    const Site q = site_at(lat_of(R), T.y, T.z, threadIdx.x);
    if (!q.ok) return;
    double2* u = U + 2 * R.off;
    double2 u1 = u[q.x], u2 = u[q.x + R.V];
    if (eps != 0.0) {
        const double* m = mom + 2 * R.off;
        double s1, c1, s2, c2;
        sincos(eps * m[q.x], &s1, &c1);
        sincos(eps * m[q.x + R.V], &s2, &c2);
        u1 = cmul(make_double2(c1, s1), u1);
        u2 = cmul(make_double2(c2, s2), u2);
        u[q.x] = u1;
        u[q.x + R.V] = u2;
    }
    st_links32(U32, tv.vtot, R.off + q.x, u1, u2);
}

// N(0,1) doubles: one thread per pair of doubles of the batch array; the replica
// is found by binary search over the replicas' first doubles dbase[0..nrep], and
// the pair index inside the replica is the single-lattice one
__global__ void k_r_random_normal(double* __restrict__ out, const long long* __restrict__ dbase, int nrep,
                                  long long npairs, const uint64_t* __restrict__ seeds, uint32_t stream,
                                  uint32_t counter, double scale) {
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const long long d = 2 * p;
    int lo = 0, hi = nrep;   // find dbase[lo] <= d < dbase[lo + 1]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(dbase + mid) <= d) lo = mid;
        else hi = mid;
    }
    double z0, z1;
    normal_pair(seeds[lo], stream, counter, (uint64_t)((d - __ldg(dbase + lo)) >> 1), z0, z1);
    out[d] = scale * z0;
    out[d + 1] = scale * z1;
}

// per-tile compensated sums (Re P, arg P, mom^2, |X|^2, Re<X,F>) ->
// part[tile*10 + 2k] (hi), part[tile*10 + 2k + 1] (lo)
__global__ void __launch_bounds__(TILE) k_r_reduce_tiles(const double2* __restrict__ U, const double* __restrict__ mom,
                                                         const double2* __restrict__ X, const double2* __restrict__ F,
                                                         TileView tv, double* __restrict__ part) {
    const int4 T = __ldg(tv.tiles + blockIdx.x);
    const RepInfo R = tv.reps[T.x];
    const Lat g = lat_of(R);
    const Site q = site_at(g, T.y, T.z, threadIdx.x);
    const long long o = 2 * R.off;
    DSum v[5] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}};
    if (q.ok) {
        const double2* u = U + o;
        const double2 p = plaquette_of(__ldg(u + q.x), __ldg(u + g.V + q.xp1), __ldg(u + q.xp2), __ldg(u + g.V + q.x));
        v[0].hi = p.x;
        v[1].hi = atan2(p.y, p.x);
        if (mom) v[2].hi = mom[o + q.x] * mom[o + q.x] + mom[o + q.x + g.V] * mom[o + q.x + g.V];
        if (X) {
            const double2 a = X[o + q.x], b = X[o + q.x + g.V];
            v[3].hi = norm2(a) + norm2(b);
            if (F) v[4].hi = cjmul(a, F[o + q.x]).x + cjmul(b, F[o + q.x + g.V]).x;
        }
    }
    __shared__ double smem[64 * 5];
    block_dsum<5>(v, smem);
    if (threadIdx.x == 0)
        for (int k = 0; k < 5; k++) {
            part[(size_t)blockIdx.x * 10 + 2 * k] = v[k].hi;
            part[(size_t)blockIdx.x * 10 + 2 * k + 1] = v[k].lo;
        }
}

// per-replica sums of the per-tile partials (one warp per replica, fixed order)
__global__ void k_r_reduce_final(const double* __restrict__ part, const RepInfo* __restrict__ reps, int nrep,
                                 double* __restrict__ out) {
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (r >= nrep) return;   // whole warps leave together
    const RepInfo R = reps[r];
    DSum s[5] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}};
    for (int t = lane; t < R.nt; t += 32)
#pragma unroll
        for (int k = 0; k < 5; k++) {
            const double* pp = part + (size_t)(R.tile0 + t) * 10 + 2 * k;
            dsum_merge(s[k], DSum{pp[0], pp[1]});
        }
#pragma unroll
    for (int k = 0; k < 5; k++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const DSum t{__shfl_xor_sync(0xffffffffu, s[k].hi, o), __shfl_xor_sync(0xffffffffu, s[k].lo, o)};
            dsum_merge(s[k], t);
        }
        if (lane == 0) out[(size_t)r * 5 + k] = s[k].hi + s[k].lo;
    }
}

// ---------------------------------------------------------------------------
// The persistent batched mixed CG: per replica, CG method 1 on (g5Dw)^2 + 0
// (src/QED2dSolver.jl:3-46) with FP32 iterations on unit-norm rescaled vectors,
// FP64 reliable updates, and the reference's FP64 stop rule |r|^2 < eps |b|^2.

// Per-replica solver state: one 96-byte record per replica.  With at most
// kSharedReps replicas every block keeps all records in shared memory and runs
// the recurrences itself on the per-replica sums published by the block that
// arrives last at a barrier (one L2 round trip per barrier).  Larger batches
// keep the records in global memory; the last block updates them (one record =
// six 16-byte loads issued together) and publishes the flags.
constexpr int kSharedReps = 64;

struct __align__(16) RepState {
    double tol, rr, maxrr, s, beta, alpha, rr64, snew;
    int act, conv, it, upd, r4, first, nupd, pad;
};
static_assert(sizeof(RepState) == 96, "RepState is six 16-byte words");

// one record = four double2 + two int4 words, loaded and stored field-wise
__device__ __forceinline__ RepState ld_state(const RepState* p) {
    const double2* d = reinterpret_cast<const double2*>(p);
    const int4* w = reinterpret_cast<const int4*>(p) + 4;
    const double2 a = __ldcg(d), b = __ldcg(d + 1), c = __ldcg(d + 2), e = __ldcg(d + 3);
    const int4 f = __ldcg(w), g = __ldcg(w + 1);
    return RepState{a.x, a.y, b.x, b.y, c.x, c.y, e.x, e.y, f.x, f.y, f.z, f.w, g.x, g.y, g.z, g.w};
}
__device__ __forceinline__ void st_state(RepState* p, const RepState& s) {
    double2* d = reinterpret_cast<double2*>(p);
    int4* w = reinterpret_cast<int4*>(p) + 4;
    d[0] = make_double2(s.tol, s.rr);
    d[1] = make_double2(s.maxrr, s.s);
    d[2] = make_double2(s.beta, s.alpha);
    d[3] = make_double2(s.rr64, s.snew);
    w[0] = make_int4(s.act, s.conv, s.it, s.upd);
    w[1] = make_int4(s.r4, s.first, s.nupd, s.pad);
}

enum { FL_ACT, FL_UPD, FL_R4, FL_N };   // any replica active / updating / rescaling
enum { RED_BB, RED_RR0, RED_PAP, RED_RN, RED_TRUE, RED_R4 };
enum { PH_SETUP, PH_START, PH_A, PH_B, PH_R1, PH_R2, PH_R3, PH_R4 };

// One segment of the solver's work: n tiles of replica r starting at tile
// (t1, t2), walked row by row; its partial sum goes to part[slot].  Slots are
// numbered replica by replica, so replica r's partials are the contiguous
// range rep_seg[r] .. rep_seg[r+1]-1.
struct SegDesc {
    int r, t1, t2, n, slot, pad0, pad1, pad2;
};

struct RCGP {
    int nrep;
    const RepInfo* reps;
    const SegDesc* segs;  // segments, block after block
    const int* seg0;      // [grid+1] segments of block b: seg0[b] .. seg0[b+1]-1
    const int* rep_seg;   // [nrep+1] partial slots of replica r
    const double* m2;     // 2 + m0 per replica
    const double2* U;
    const float4* U32;    // FP32 link planes of vtot sites
    long long vtot;
    const double2* b;
    double2* x;
    double2* r64;
    double2* t64;   // g5Dw x of the solution (the force needs it)
    float4 *r32, *q0, *q1, *t32, *x32;
    double eps, delta2;
    int maxiter;
    RepState* st;   // [nrep] (final state in both modes)
    int* flags;     // [FL_N] (global-state mode)
    int* flag_acc;  // OR of the flags raised by the replicas finished at a barrier (global-state mode)
    int* cnt;       // [nrep] segments of each replica reduced so far at the current barrier
    double* red;    // [2][nrep] per-replica sums (shared-state mode, alternating)
    double* part;   // one partial per segment
    DevCtl* ctl;
};

// where a block finds the records: shared memory or global memory
template <bool SH>
struct StateView {
    RepState* sh;
    const RepState* gl;
    __device__ __forceinline__ RepState get(int r) const { return SH ? sh[r] : ld_state(gl + r); }
};

template <int PH>
using acc_t = typename std::conditional<PH == PH_A || PH == PH_B, float, double>::type;

// a replica's scalars for one phase (loaded once per segment)
struct RepVals {
    bool work, act, first;
    double s, beta, alpha, snew, m2;
};

template <int PH, bool SH>
__device__ __forceinline__ RepVals rep_vals(const StateView<SH>& sv, int r, double m2) {
    RepVals v{};
    v.m2 = m2;
    if constexpr (PH == PH_SETUP) {
        v.work = true;
    } else {
        const RepState st = sv.get(r);
        v.act = st.act;
        v.first = st.first;
        v.s = st.s;
        v.beta = st.beta;
        v.alpha = st.alpha;
        v.snew = st.snew;
        if constexpr (PH == PH_START) v.work = true;
        else if constexpr (PH == PH_A || PH == PH_B) v.work = st.act;
        else if constexpr (PH == PH_R4) v.work = st.r4;
        else v.work = st.upd;   // R1, R2, R3
    }
    return v;
}

// the work of phase PH on this thread's site of tile (t1, t2) of replica R;
// returns the site's contribution to the phase's per-replica sum
template <int PH>
__device__ __forceinline__ acc_t<PH> tile_work(const RCGP& P, const RepVals& v, const RepInfo& R, int t1, int t2,
                                               int cur) {
    const Lat g = lat_of(R);
    const Site q = site_at(g, t1, t2, threadIdx.x);
    if (!q.ok) return 0;
    const long long o2 = 2 * R.off, o1 = R.off, V = R.V;
    const Pair<double> z{make_double2(0, 0), make_double2(0, 0)};
    const Pair<float> zf{make_float2(0, 0), make_float2(0, 0)};
    if constexpr (PH == PH_SETUP) {   // |b|^2, x = 0
        const Pair<double> bv{__ldg(P.b + o2 + q.x), __ldg(P.b + o2 + q.x + V)};
        st_d(P.x + o2, V, q.x, z);
        return norm2(bv.a) + norm2(bv.b);
    } else if constexpr (PH == PH_START) {   // r32 = s b, x32 = 0; a zero source keeps x = 0 and g5Dw x = 0
        if (!v.act) {
            st_d(P.t64 + o2, V, q.x, z);
            return 0;
        }
        const Pair<float> r32{to_f(v.s * __ldg(P.b + o2 + q.x)), to_f(v.s * __ldg(P.b + o2 + q.x + V))};
        st_f(P.r32 + o1, q.x, r32);
        st_f(P.x32 + o1, q.x, zf);
        return (double)(norm2(r32.a) + norm2(r32.b));
    } else if constexpr (PH == PH_A) {   // p = r + beta p_old, t = g5Dw p, |t|^2 = <p, (g5Dw)^2 p>
        float4* qn = cur ? P.q1 : P.q0;
        const float4* qo = cur ? P.q0 : P.q1;
        const SpAxpy<float, SpF> Q{SpF{P.r32 + o1}, SpF{qo + o1}, (float)v.beta, !v.first};
        const Pair<float> c = Q.ld(q.x);
        const Pair<float> tt = g5dw_at_c<float>(Q, c, LkF{P.U32, P.vtot, o1}, q, (float)v.m2);
        st_f(qn + o1, q.x, c);
        st_f(P.t32 + o1, q.x, tt);
        return norm2(tt.a) + norm2(tt.b);
    } else if constexpr (PH == PH_B) {   // x += alpha p, r -= alpha g5Dw t
        const float4* qn = cur ? P.q1 : P.q0;
        const float alpha = (float)v.alpha;
        const Pair<float> pc = SpF{qn + o1}.ld(q.x);
        const Pair<float> a = g5dw_at<float>(SpF{P.t32 + o1}, LkF{P.U32, P.vtot, o1}, q, (float)v.m2);
        Pair<float> xv = SpF{P.x32 + o1}.ld(q.x), rv = SpF{P.r32 + o1}.ld(q.x);
        xv.a = xv.a + alpha * pc.a;
        xv.b = xv.b + alpha * pc.b;
        rv.a = rv.a - alpha * a.a;
        rv.b = rv.b - alpha * a.b;
        st_f(P.x32 + o1, q.x, xv);
        st_f(P.r32 + o1, q.x, rv);
        return norm2(rv.a) + norm2(rv.b);
    } else if constexpr (PH == PH_R1) {   // x += x32 / s, x32 = 0
        const double inv_s = 1.0 / v.s;
        const Pair<float> d = SpF{P.x32 + o1}.ld(q.x);
        Pair<double> xv = SpD{P.x + o2, V}.ld(q.x);
        xv.a = xv.a + inv_s * to_d(d.a);
        xv.b = xv.b + inv_s * to_d(d.b);
        st_d(P.x + o2, V, q.x, xv);
        st_f(P.x32 + o1, q.x, zf);
        return 0;
    } else if constexpr (PH == PH_R2) {   // t64 = g5Dw x
        st_d(P.t64 + o2, V, q.x, g5dw_at<double>(SpD{P.x + o2, V}, LkD{P.U + o2, V}, q, v.m2));
        return 0;
    } else if constexpr (PH == PH_R3) {   // r64 = b - g5Dw t64, |r64|^2
        const Pair<double> a = g5dw_at<double>(SpD{P.t64 + o2, V}, LkD{P.U + o2, V}, q, v.m2);
        Pair<double> rv;
        rv.a = __ldg(P.b + o2 + q.x) - a.a;
        rv.b = __ldg(P.b + o2 + q.x + V) - a.b;
        st_d(P.r64 + o2, V, q.x, rv);
        return norm2(rv.a) + norm2(rv.b);
    } else {   // PH_R4: r32 = s_new r64
        const Pair<float> r32{to_f(v.snew * P.r64[o2 + q.x]), to_f(v.snew * P.r64[o2 + q.x + V])};
        st_f(P.r32 + o1, q.x, r32);
        return (double)(norm2(r32.a) + norm2(r32.b));
    }
}

// A block's place in the tile table (set once per launch, kept in shared
// memory) and the records of its first kSegCache replicas, so that a phase
// starts without global loads.
constexpr int kSegCache = 64;
struct BlockCtx {
    int seg, nsb;   // first segment, segments of this block
};
struct SegInfo {
    SegDesc d;
    RepInfo R;
    double m2;
    int rs0, rs1;   // the replica's partial slots
};
// per-block shared scratch of a phase: the segments' scalars and per-warp partials
struct PhaseScratch {
    RepVals vals[kSegCache];
    double wsum[kSegCache][TILE / 32];
};

__device__ __forceinline__ void block_ctx_init(const RCGP& P, BlockCtx& bc, SegInfo* seg) {
    if (threadIdx.x == 0) {
        const int s0 = P.seg0[blockIdx.x];
        bc = BlockCtx{s0, P.seg0[blockIdx.x + 1] - s0};
    }
    __syncthreads();
    for (int i = threadIdx.x; i < min(bc.nsb, kSegCache); i += blockDim.x) {
        const SegDesc d = P.segs[bc.seg + i];
        seg[i].d = d;
        seg[i].R = P.reps[d.r];
        seg[i].m2 = P.m2[d.r];
        seg[i].rs0 = P.rep_seg[d.r];
        seg[i].rs1 = P.rep_seg[d.r + 1];
    }
    __syncthreads();
}

// One phase over the block's segments (phases R1 and R2 sum nothing).  The
// scalars of the block's first kSegCache segments are fetched together at the
// start (one round trip), and a segment's partial is a warp sum per warp,
// summed over the warps in a fixed order at the end of the phase; further
// segments fetch their scalars and reduce one by one.
template <int PH, bool SH>
__device__ __forceinline__ void run_phase(const RCGP& P, const StateView<SH>& sv, int cur, const BlockCtx& bcs,
                                          const SegInfo* segs, PhaseScratch& ps, double* smem) {
    constexpr bool kSum = PH != PH_R1 && PH != PH_R2;
    const int nsb = bcs.nsb, ncache = min(nsb, kSegCache);
    if (threadIdx.x < ncache) ps.vals[threadIdx.x] = rep_vals<PH, SH>(sv, segs[threadIdx.x].d.r, segs[threadIdx.x].m2);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = 0; i < nsb; i++) {
        const bool cached = i < kSegCache;
        const SegDesc d = cached ? segs[i].d : P.segs[bcs.seg + i];
        const RepInfo R = cached ? segs[i].R : P.reps[d.r];
        const RepVals v = cached ? ps.vals[i] : rep_vals<PH, SH>(sv, d.r, __ldg(P.m2 + d.r));
        acc_t<PH> acc = 0;
        if (v.work)
            for (int j = 0, t1 = d.t1, t2 = d.t2; j < d.n; j++) {
                acc += tile_work<PH>(P, v, R, t1, t2, cur);
                if (++t1 == R.nt1) {
                    t1 = 0;
                    ++t2;
                }
            }
        if constexpr (kSum) {
            if (cached) {
                double w = (double)acc;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
                if (lane == 0) ps.wsum[i][warp] = w;
            } else {
                double red[1] = {(double)acc};
                block_sum<1>(red, smem);
                if (threadIdx.x == 0) {
                    P.part[d.slot] = red[0];
                    __threadfence();
                }
            }
        }
    }
    if constexpr (kSum) {
        __syncthreads();
        if (threadIdx.x < ncache) {
            double s = 0.0;
#pragma unroll
            for (int w = 0; w < TILE / 32; w++) s += ps.wsum[threadIdx.x][w];
            P.part[segs[threadIdx.x].d.slot] = s;
            __threadfence();
        }
    }
}

// the CG scalar recurrences of one replica after reduction `kind` gave sum s
// (the scalar steps of the single-lattice mixed solver)
__device__ __forceinline__ void rep_step(RepState& st, int kind, double s, int k, double eps, double delta2,
                                         int maxiter, int* fl) {
    switch (kind) {
        case RED_BB:
            st.tol = eps * s;
            st.act = s > 0.0;
            st.conv = s == 0.0;
            st.it = 0;
            st.first = 1;
            st.nupd = 0;
            st.upd = 0;
            st.r4 = 0;
            st.rr64 = s;
            st.s = s > 0.0 ? 1.0 / sqrt(s) : 0.0;
            st.beta = 0.0;
            fl[FL_ACT] |= st.act;
            break;
        case RED_RR0:
            st.rr = s;
            st.maxrr = s;
            fl[FL_ACT] |= st.act;
            break;
        case RED_PAP:
            if (st.act) st.alpha = st.rr / s;
            break;
        case RED_RN:
            st.upd = 0;
            if (st.act) {
                st.maxrr = fmax(st.maxrr, s);
                const bool cand = s < st.tol * st.s * st.s;
                if (s < delta2 * st.maxrr || cand || k == maxiter) {
                    st.upd = 1;
                    st.nupd += 1;
                    fl[FL_UPD] = 1;
                } else {
                    st.beta = s / st.rr;
                    st.rr = s;
                    st.rr64 = s / (st.s * st.s);
                }
                st.first = 0;
            }
            break;
        case RED_TRUE:
            st.r4 = 0;
            if (st.upd) {
                st.rr64 = s;
                if (s < st.tol) {
                    st.act = 0;
                    st.conv = 1;
                    st.it = k;
                } else if (k == maxiter) {
                    st.act = 0;
                    st.it = k;
                } else {
                    st.r4 = 1;
                    st.snew = 1.0 / sqrt(s);
                    fl[FL_R4] = 1;
                }
            }
            fl[FL_ACT] |= st.act;
            break;
        case RED_R4:
            if (st.r4) {
                st.beta = (st.rr64 * st.s * st.s / st.rr) * (st.snew / st.s);
                st.s = st.snew;
                st.rr = s;
                st.maxrr = s;
            }
            fl[FL_ACT] |= st.act;
            break;
    }
}

// which flags reduction `kind` recomputes
__device__ __forceinline__ void clear_flags(int kind, int* fl) {
    if (kind == RED_BB || kind == RED_RR0 || kind == RED_TRUE || kind == RED_R4) fl[FL_ACT] = 0;
    if (kind == RED_RN) fl[FL_UPD] = 0;
    if (kind == RED_TRUE) fl[FL_R4] = 0;
}

// Per-replica completion at a barrier, before the block arrives: each segment
// of this block counts itself into its replica's counter; the block whose
// segment completes a replica finishes it -- one warp sums the replica's
// partials (lanes over the slots in a fixed order, then a fixed shuffle tree,
// so the result does not depend on which block finishes) and either publishes
// the sum (SH) or runs the replica's recurrences on its global record and ORs
// the flags it raises into flag_acc.  The per-replica work is thus spread over
// the blocks instead of serialised in the block that arrives last.
template <bool SH>
__device__ __forceinline__ void finish_replica(const RCGP& P, int r, int rs0, int rs1, int kind, int k,
                                               double* red) {
    const int lane = threadIdx.x & 31;
    __threadfence();
    double s = 0.0;
    for (int i = rs0 + lane; i < rs1; i += 32) s += __ldcg(P.part + i);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        if (SH) {
            red[r] = s;
        } else {
            RepState st = ld_state(P.st + r);
            int fl[FL_N] = {0, 0, 0};
            rep_step(st, kind, s, k, P.eps, P.delta2, P.maxiter, fl);
            st_state(P.st + r, st);
            const int bits = fl[FL_ACT] | fl[FL_UPD] << 1 | fl[FL_R4] << 2;
            if (bits) atomicOr(P.flag_acc, bits);
        }
        __threadfence();
    }
}

template <bool SH>
__device__ __forceinline__ void complete_replicas(const RCGP& P, const BlockCtx& bcs, const SegInfo* segs, int kind,
                                                  int k, double* red) {
    __shared__ int s_ntask, s_task[kSegCache][3];
    if (threadIdx.x == 0) s_ntask = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < bcs.nsb; i += blockDim.x) {
        int r, rs0, rs1;
        if (i < kSegCache) {
            r = segs[i].d.r;
            rs0 = segs[i].rs0;
            rs1 = segs[i].rs1;
        } else {
            r = P.segs[bcs.seg + i].r;
            rs0 = __ldg(P.rep_seg + r);
            rs1 = __ldg(P.rep_seg + r + 1);
        }
        if (atomicAdd(P.cnt + r, 1) == rs1 - rs0 - 1) {   // this block completes replica r
            P.cnt[r] = 0;
            const int t = atomicAdd(&s_ntask, 1);
            if (t < kSegCache) {
                s_task[t][0] = r;
                s_task[t][1] = rs0;
                s_task[t][2] = rs1;
            } else {   // more completions than task slots: this thread finishes it alone
                __threadfence();
                double s = 0.0;
                for (int j = rs0; j < rs1; j++) s += __ldcg(P.part + j);
                if (SH) {
                    red[r] = s;
                } else {
                    RepState st = ld_state(P.st + r);
                    int fl[FL_N] = {0, 0, 0};
                    rep_step(st, kind, s, k, P.eps, P.delta2, P.maxiter, fl);
                    st_state(P.st + r, st);
                    const int bits = fl[FL_ACT] | fl[FL_UPD] << 1 | fl[FL_R4] << 2;
                    if (bits) atomicOr(P.flag_acc, bits);
                }
                __threadfence();
            }
        }
    }
    __syncthreads();
    const int nt = min(s_ntask, kSegCache), warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int t = warp; t < nt; t += nw) finish_replica<SH>(P, s_task[t][0], s_task[t][1], s_task[t][2], kind, k, red);
}

// Grid barrier after a reduction: the replicas are completed by the blocks
// (complete_replicas), the last block to arrive merges the flags (global
// records) and releases; with shared records every block then runs every
// replica's recurrences on the published sums.  s_fl (shared) holds the flags
// afterwards in every block.
template <bool SH>
__device__ __forceinline__ bool rbarrier(GridSync& gs, const RCGP& P, RepState* s_st, int* s_fl, const BlockCtx& bcs,
                                         const SegInfo* segs, int kind, int k) {
    __shared__ int s_last, s_bits;
    double* red = P.red + (size_t)(gs.nred++ & 1) * P.nrep;   // alternate: a slow block may still read the last
    complete_replicas<SH>(P, bcs, segs, kind, k, red);
    if (threadIdx.x == 0) s_bits = 0;   // arrive() begins with __syncthreads
    const bool last = gs.arrive(&s_last);
    if (threadIdx.x == 0) {
        if (last) {
            if (!SH) {
                __threadfence();
                const int bits = atomicExch(P.flag_acc, 0);
                int g[FL_N] = {s_fl[FL_ACT], s_fl[FL_UPD], s_fl[FL_R4]};
                clear_flags(kind, g);
                g[FL_ACT] |= bits & 1;
                g[FL_UPD] |= (bits >> 1) & 1;
                g[FL_R4] |= (bits >> 2) & 1;
                for (int i = 0; i < FL_N; i++) {
                    s_fl[i] = g[i];
                    P.flags[i] = g[i];
                }
            }
            gs.release();
        } else {
            gs.wait();
            if (!SH)
                for (int i = 0; i < FL_N; i++) s_fl[i] = __ldcg(P.flags + i);
        }
    }
    __syncthreads();
    if (SH) {   // every block: the recurrences of every replica on the published sums
        int fl[FL_N] = {0, 0, 0};
        if (threadIdx.x < P.nrep) {   // nrep <= kSharedReps <= blockDim.x
            const int r = threadIdx.x;
            RepState st = s_st[r];
            rep_step(st, kind, __ldcg(red + r), k, P.eps, P.delta2, P.maxiter, fl);
            s_st[r] = st;
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
    }
    return ld_volatile_int(gs.err) == 0;
}

// the solve; false when a barrier gave up
template <bool SH>
__device__ __forceinline__ bool r_body(const RCGP& P, GridSync& gs, int& k, double* smem, RepState* s_st, int* s_fl,
                                       const BlockCtx& bc, const SegInfo* segs, PhaseScratch& ps) {
    const StateView<SH> sv{s_st, P.st};
    int cur = 0;
    run_phase<PH_SETUP, SH>(P, sv, cur, bc, segs, ps, smem);
    if (!rbarrier<SH>(gs, P, s_st, s_fl, bc, segs, RED_BB, 0)) return false;
    run_phase<PH_START, SH>(P, sv, cur, bc, segs, ps, smem);
    if (!rbarrier<SH>(gs, P, s_st, s_fl, bc, segs, RED_RR0, 0)) return false;
    for (k = 1; k <= P.maxiter; k++) {
        if (!s_fl[FL_ACT]) break;
        run_phase<PH_A, SH>(P, sv, cur, bc, segs, ps, smem);
        if (!rbarrier<SH>(gs, P, s_st, s_fl, bc, segs, RED_PAP, k)) return false;
        run_phase<PH_B, SH>(P, sv, cur, bc, segs, ps, smem);
        if (!rbarrier<SH>(gs, P, s_st, s_fl, bc, segs, RED_RN, k)) return false;
        if (s_fl[FL_UPD]) {
            run_phase<PH_R1, SH>(P, sv, cur, bc, segs, ps, smem);
            if (!gs.sync()) return false;
            run_phase<PH_R2, SH>(P, sv, cur, bc, segs, ps, smem);
            if (!gs.sync()) return false;
            run_phase<PH_R3, SH>(P, sv, cur, bc, segs, ps, smem);
            if (!rbarrier<SH>(gs, P, s_st, s_fl, bc, segs, RED_TRUE, k)) return false;
            if (s_fl[FL_R4]) {
                run_phase<PH_R4, SH>(P, sv, cur, bc, segs, ps, smem);
                if (!rbarrier<SH>(gs, P, s_st, s_fl, bc, segs, RED_R4, k)) return false;
            }
        }
        cur ^= 1;
    }
    return true;
}

template <bool SH>
__global__ void __launch_bounds__(TILE, 4) k_r_cg_mixed(const RCGP P) {
    __shared__ double smem[32];
    __shared__ RepState s_st[SH ? kSharedReps : 1];
    __shared__ int s_fl[FL_N];
    __shared__ BlockCtx s_bc;
    __shared__ SegInfo s_seg[kSegCache];
    __shared__ PhaseScratch s_ps;
    if (threadIdx.x < FL_N) s_fl[threadIdx.x] = 0;
    block_ctx_init(P, s_bc, s_seg);
    GridSync gs{&P.ctl->bar, &P.ctl->gen, &P.ctl->err};
    int k = 0;
    const bool ok = r_body<SH>(P, gs, k, smem, s_st, s_fl, s_bc, s_seg, s_ps);
    if (blockIdx.x == 0) {
        if (SH && ok)   // every block holds the same records: block 0 stores them
            for (int r = threadIdx.x; r < P.nrep; r += blockDim.x) P.st[r] = s_st[r];
        if (threadIdx.x == 0) {
            DevCtl* c = P.ctl;
            c->last_iters = k;
            if (c->status == 0 && (ld_volatile_int(&c->err) || !ok)) c->status = QED2D_ERR_TIMEOUT;
        }
    }
}

// per-replica outputs of a solve: iterations, reliable updates; accumulated
// iterations; status NOT_CONVERGED when a replica did not converge
__global__ void k_r_finish(const RepState* __restrict__ st, int nrep, int maxiter, int* __restrict__ it_out,
                           int* __restrict__ upd_out, long long* __restrict__ acc, DevCtl* ctl) {
    if (ctl->status != 0) return;   // a solve that gave up leaves no per-replica results
    int bad = 0;
    for (int r = threadIdx.x; r < nrep; r += blockDim.x) {
        const RepState s = st[r];
        const int its = s.conv ? s.it : (s.it ? s.it : maxiter);
        it_out[r] = its;
        upd_out[r] = s.nupd;
        acc[r] += its;
        bad |= !s.conv;
    }
    bad = __syncthreads_or(bad);
    if (threadIdx.x == 0 && bad) ctl->status = QED2D_ERR_NOT_CONVERGED;
}

}  // namespace qed2d

#include "batch_cg_uniform.cuh"
#include "batch_cg_cluster.cuh"

namespace qed2d {
// tile heights of k_u_cg_mixed (rows of 32 sites per tile = warps per block);
// the first is the default when the tuner is off
constexpr int kUTileRows[3] = {8, 16, 4};

template <int RS, bool RSTEN = false, bool LSM = false>
static const void* uniform_kernel_rs(int rows) {
    return rows == 4    ? (const void*)k_u_cg_mixed<RS, 4, RSTEN, LSM>
           : rows == 16 ? (const void*)k_u_cg_mixed<RS, 16, RSTEN, LSM>
                        : (const void*)k_u_cg_mixed<RS, 8, RSTEN, LSM>;
}
// shared memory of schedule 9's staged links for a tile height and tiles per block
static size_t uniform_lsm_bytes(int rows, int per_block) {
    return rows == 4 ? ULsm<4>::bytes(per_block) : rows == 16 ? ULsm<16>::bytes(per_block) : ULsm<8>::bytes(per_block);
}

// host: cuTensorMapEncodeTiled through the runtime's driver entry point
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int encode_map_2d(CUtensorMap* map, const void* base, unsigned long long nx, unsigned long long ny,
                  unsigned long long pitch, unsigned bx, unsigned by) {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !p) {
            cudaGetLastError();
            set_error("cuTensorMapEncodeTiled is not available from the driver");
            return QED2D_ERR_UNSUPPORTED;
        }
        fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    if (reinterpret_cast<uintptr_t>(base) % 16 || pitch % 16 || (4ull * bx) % 16 || bx > 256 || by > 256 || bx > nx ||
        by > ny) {
        set_error("tensor map: unaligned base or pitch, or box outside the tensor");
        return QED2D_ERR_BAD_ARG;
    }
    const cuuint64_t dims[2] = {nx, ny};
    const cuuint64_t strides[1] = {pitch};
    const cuuint32_t box[2] = {bx, by};
    const cuuint32_t es[2] = {1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(base), dims, strides, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed");
        return QED2D_ERR_CUDA;
    }
    return QED2D_OK;
}

// the TMA-staged solver (schedule 7) for a tile height, or null where it has no instance
static const void* uniform_kernel_tma(int rows) {
    return rows == 16 ? (const void*)k_u_cg_mixed_tma<16> : rows == 8 ? (const void*)k_u_cg_mixed_tma<8> : nullptr;
}
static size_t uniform_tma_smem(int rows) {
    return (size_t)kTmaStages * (rows == 16 ? UStage<16>::BYTES : UStage<8>::BYTES) + 128;
}

// the equal-size solver for schedule 0/1 (grid reductions), 4 (a barrier per
// replica), 5 (the same, lean reduction), 8 (5 with the phase-A stencil on r) or
// 9 (8 with the links staged in shared memory) and a tile height
static const void* uniform_kernel(int sched, int rows) {
    switch (sched) {
        case 0: return uniform_kernel_rs<0>(rows);
        case 1: return uniform_kernel_rs<1>(rows);
        case 4: return uniform_kernel_rs<2>(rows);
        case 8: return uniform_kernel_rs<3, true>(rows);
        case 9: return uniform_kernel_rs<3, true, true>(rows);
        default: return uniform_kernel_rs<3>(rows);
    }
}
}  // namespace qed2d

// ===========================================================================
// host side
using namespace qed2d;

struct qed2d_batch {
    int nrep = 0, ntiles = 0;
    long long Vtot = 0;
    std::vector<RepInfo> reps;
    std::vector<double> beta, m2;
    int device = 0, num_sms = 148;
    cudaStream_t stream = nullptr;
    int grid = 0, per_block = 0, nseg = 0;   // persistent CG geometry
    RepInfo* d_reps = nullptr;
    int4* d_tiles = nullptr;
    int* d_seg0 = nullptr;
    SegDesc* d_segs = nullptr;
    int* d_rep_seg = nullptr;
    long long* d_dbase_c = nullptr;   // first double of each replica: complex fields [nrep+1]
    long long* d_dbase_r = nullptr;   // the same for real fields
    double* d_m2 = nullptr;
    double* d_beta = nullptr;
    uint64_t* d_seed = nullptr;
    RepState* d_st = nullptr;       // [nrep] solver records
    int* d_flags = nullptr;         // [FL_N]
    double* d_red = nullptr;        // [2][nrep]
    int* d_cnt = nullptr;           // [nrep + 1]: per-replica counters, then the flag accumulator
    bool shared_state = false;      // records in shared memory (nrep <= kSharedReps)
    bool uniform = false;           // equal sizes, nrep <= kUniformReps: k_u_cg_mixed
    int usched = -1;                // its schedule: 0, 1 (grid reductions), 4, 5, 8 (independent replicas); -1 untuned
    int rsched = -1;                // uneven batches: 2 grid solver, 3 one cluster per replica, 6 the same with
                                    // the first phase's stencil on r (-1: not tuned)
    int rcs = 8;                    // blocks per cluster of the cluster solver (tuned)
    int* d_order = nullptr;         // [nrep] replicas by decreasing size (cluster solver)
    // k_u_cg_mixed geometry per tile height (kUTileRows): tiles per replica,
    // tiles per block, blocks per replica, grid
    struct UVar {
        int rows = 0, per_block = 0, bpr = 0, grid = 0;
        long long ntr = 0;
        bool tma = false;   // schedule 7 possible: whole tiles, an instance, co-resident with its shared memory
        size_t lsm = 0;     // schedule 9's dynamic shared memory; 0: not co-resident with it
    } uv[3];
    int nuv = 0;                    // heights whose kernels fit (co-resident grid)
    int utile = -1;                 // index into uv of the tile height in use; -1 untuned
    bool utile_fixed = false;       // set by qed2d_batch_set_tile_rows: the tuner keeps it
    bool usched_fixed = false;      // set by qed2d_batch_set_schedule: the tuner keeps it (tunes the height only)
    UGeom ug{};
    double* d_upart = nullptr;      // [2][max grid over uv]
    double* d_ured = nullptr;       // [2][nrep]
    unsigned long long* d_ubar = nullptr;   // [nrep][16] per-replica barrier counters (schedule 4)
    int* d_out = nullptr;           // [2][nrep]: iterations, reliable updates of the last solve
    long long* d_iters = nullptr;   // [nrep] iterations accumulated over a trajectory
    double* d_sums = nullptr;       // [2][nrep][5] start / end sums of a trajectory
    double* d_tpart = nullptr;      // [ntiles][5][hi, lo]
    double* d_part = nullptr;       // [nseg]
    DevCtl* ctl = nullptr;
    DevCtl* ctl_host = nullptr;
    std::map<std::string, std::pair<void*, size_t>> ws;
    uint64_t ws_gen = 0;            // bumped whenever a workspace buffer is reallocated
    GraphCache md_graph;            // MD integration of qed2d_batch_hmc_nf2 (graph.h)

    void* buf(const std::string& name, size_t bytes) {
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
            set_error("batch workspace allocation failed (" + name + ")");
            return nullptr;
        }
        ws[name] = {p, bytes};
        return p;
    }
    double2* field(const char* n) { return (double2*)buf(n, sizeof(double2) * 2 * Vtot); }
    double* real2(const char* n) { return (double*)buf(n, sizeof(double) * 2 * Vtot); }
    float4* field32(const char* n) { return (float4*)buf(n, sizeof(float4) * Vtot); }
    TileView tv() const { return TileView{d_reps, d_tiles, Vtot}; }
};

namespace {

int r_post(const char* name) {
    count_launch();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QED2D_OK : cuda_status(e, name);
}

int r_fill(qed2d_batch* h, double* out, bool complex_field, uint32_t stream, uint32_t counter, double scale) {
    const long long npairs = complex_field ? 2 * h->Vtot : h->Vtot;   // pairs of doubles
    k_r_random_normal<<<(unsigned)((npairs + 255) / 256), 256, 0, h->stream>>>(
        out, complex_field ? h->d_dbase_c : h->d_dbase_r, h->nrep, npairs, h->d_seed, stream, counter, scale);
    return r_post("k_r_random_normal");
}

int r_sums(qed2d_batch* h, const double2* U, const double* mom, const double2* X, const double2* F, int slot) {
    k_r_reduce_tiles<<<h->ntiles, TILE, 0, h->stream>>>(U, mom, X, F, h->tv(), h->d_tpart);
    QTRY(r_post("k_r_reduce_tiles"));
    k_r_reduce_final<<<(h->nrep + 7) / 8, 256, 0, h->stream>>>(h->d_tpart, h->d_reps, h->nrep,
                                                                h->d_sums + (size_t)slot * h->nrep * 5);
    return r_post("k_r_reduce_final");
}

int r_pack(qed2d_batch* h, double2* U, const double* mom, double eps, float4* U32) {
    k_r_updt<<<h->ntiles, TILE, 0, h->stream>>>(U, mom, eps, U32, h->tv());
    return r_post("k_r_updt");
}

// First solve of an equal-size batch: time the schedules of k_u_cg_mixed
// (same bits) on the caller's operator and sources, capped at 24 iterations,
// into scratch outputs, and keep the fastest; the device control block is saved
// and restored around it.  Independent replicas (4) are a candidate from two
// replicas up (with one they are schedule 1).  QED2D_TUNE=0: the size rule
// measured on B200 instead -- independent replicas with the lean reduction from
// two replicas up (schedule 1 -> 4 per iteration: 2 x 512^2 23.1 -> 20.2 us,
// 4 x 512^2 39.1 -> 30.8 us, 32 x 64^2 28.8 -> 9.8 us; 4 -> 5: 16 x 128^2
// 11.9 -> 11.3 us, 8 x 256^2 16.9 -> 16.6 us, 4 x 512^2 within 4% either way
// over runs), every block sums for one; with the phase-A stencil on r
// (schedule 8) while the batch's FP32 working set stays in L2 (at most 2^20
// sites: 4 x 512^2 26.5 -> 24.5 us per iteration, same iteration counts), where
// its three fewer float4 loads per site count; beyond, phase A's extra read of
// t_old (16 B per site from DRAM) does; and with the links staged in shared
// memory (schedule 9) where they fit beside co-resident blocks (4 x 512^2
// 27.4 -> 25.3 us per iteration; the tuner picked 9 at every equal-size batch
// measured from 32 x 64^2 to 4 x 512^2); tiles of 16 rows for replicas of 2^18
// sites and more (the tuner's choice at 4 x 512^2), else 8.
template <class Launch>
int tune_uniform(qed2d_batch* h, const UCGP& Q, int maxiter, Launch launch) {
    if (!tuning_enabled()) {
        if (!h->utile_fixed) {
            h->utile = 0;
            if (h->Vtot / h->nrep >= (1LL << 18))
                for (int t = 0; t < h->nuv; t++)
                    if (h->uv[t].rows == 16) h->utile = t;
        }
        if (!h->usched_fixed)
            h->usched = h->nrep >= 2 ? (h->Vtot <= (1LL << 20) ? (h->uv[h->utile].lsm ? 9 : 8) : 5) : 1;
        return QED2D_OK;
    }
    // candidates: (schedule, tile height); the height only when it is not fixed,
    // the schedule only when the caller has not fixed it
    // (schedule 7, the TMA-staged solver, is not a candidate: it gives the same
    // bits as 5 and measured slower everywhere, e.g. 4 x 512^2 28.1 -> 33.5 us per
    // iteration; callers can select it)
    constexpr int scheds[6] = {0, 1, 4, 5, 8, 9};
    const int nsched = h->nrep >= 2 ? 6 : 2;
    const int t_lo = h->utile_fixed ? h->utile : 0, t_hi = h->utile_fixed ? h->utile + 1 : h->nuv;
    auto fits = [&](int s, int t) { return (s != 9 || h->uv[t].lsm) && (s != 7 || h->uv[t].tma); };
    std::vector<std::pair<int, int>> cand;
    for (int t = t_lo; t < t_hi; t++) {
        if (h->usched_fixed) {
            if (fits(h->usched, t)) cand.push_back({h->usched, t});
            continue;
        }
        for (int rs = 0; rs < nsched; rs++)
            if (fits(scheds[rs], t)) cand.push_back({scheds[rs], t});
    }
    if (cand.empty()) {
        set_error("batch schedule " + std::to_string(h->usched) + ": no tile height fits it");
        return QED2D_ERR_UNSUPPORTED;
    }
    DevCtl saved;
    QCHECK(cudaMemcpyAsync(&saved, h->ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, h->stream));
    QCHECK(cudaStreamSynchronize(h->stream));
    UCGP T = Q;
    T.x = h->field("tune_x");
    T.t64 = h->field("tune_g5x");
    T.maxiter = std::min(maxiter, 24);
    if (!T.x || !T.t64) return QED2D_ERR_NO_MEMORY;
    cudaEvent_t e0, e1;
    QCHECK(cudaEventCreate(&e0));
    QCHECK(cudaEventCreate(&e1));
    std::vector<float> tbest(cand.size(), 1e30f);
    int st = QED2D_OK;
    for (int rep = 0; rep < 3 && st == QED2D_OK; rep++)
        for (size_t c = 0; c < cand.size() && st == QED2D_OK; c++) {
            cudaEventRecord(e0, h->stream);
            st = launch(cand[c].first, cand[c].second, T);
            cudaEventRecord(e1, h->stream);
            if (cudaEventSynchronize(e1) != cudaSuccess) st = cuda_status(cudaGetLastError(), "schedule tuning");
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) tbest[c] = std::min(tbest[c], ms);   // the first round warms up
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    QCHECK(cudaMemcpyAsync(h->ctl, &saved, sizeof(DevCtl), cudaMemcpyHostToDevice, h->stream));
    QCHECK(cudaStreamSynchronize(h->stream));
    if (st != QED2D_OK) return st;
    size_t best = 0;
    for (size_t c = 1; c < cand.size(); c++)
        if (tbest[c] < tbest[best]) best = c;
    h->usched = cand[best].first;
    h->utile = cand[best].second;
    return QED2D_OK;
}

// One cluster of cs blocks per replica (k_rc_cg_mixed<cs>).
static bool cluster_fits(int cs, const void* kern) {
    if (cs > 8 && cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(TILE);
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess || n < 1) {
        cudaGetLastError();
        return false;
    }
    return true;
}

static const void* replica_cluster_kernel(int cs, bool rsten = false) {
    if (rsten)
        return cs == 4    ? (const void*)k_rc_cg_mixed<4, true>
               : cs == 16 ? (const void*)k_rc_cg_mixed<16, true>
                          : (const void*)k_rc_cg_mixed<8, true>;
    return cs == 4 ? (const void*)k_rc_cg_mixed<4> : cs == 16 ? (const void*)k_rc_cg_mixed<16> : (const void*)k_rc_cg_mixed<8>;
}

// rsten: the first phase's stencil on r (schedule 6)
int launch_replica_clusters(qed2d_batch* h, const CCGP& cc, int cs, bool rsten) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(h->nrep * cs));
    cfg.blockDim = dim3(TILE);
    cfg.stream = h->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (rsten) {
        if (cs == 4) QCHECK(cudaLaunchKernelEx(&cfg, k_rc_cg_mixed<4, true>, cc));
        else if (cs == 16) QCHECK(cudaLaunchKernelEx(&cfg, k_rc_cg_mixed<16, true>, cc));
        else QCHECK(cudaLaunchKernelEx(&cfg, k_rc_cg_mixed<8, true>, cc));
    } else {
        if (cs == 4) QCHECK(cudaLaunchKernelEx(&cfg, k_rc_cg_mixed<4>, cc));
        else if (cs == 16) QCHECK(cudaLaunchKernelEx(&cfg, k_rc_cg_mixed<16>, cc));
        else QCHECK(cudaLaunchKernelEx(&cfg, k_rc_cg_mixed<8>, cc));
    }
    return QED2D_OK;
}

// First solve of an uneven batch: time the grid solver (k_r_cg_mixed, one
// launch over all replicas with grid barriers) and the cluster solver
// (k_rc_cg_mixed, one cluster of 4, 8 or 16 blocks per replica), capped at 24
// iterations into scratch outputs, and keep the fastest; the control block is
// saved and restored.  QED2D_TUNE=0: the size rule measured on B200 instead --
// clusters of 8 blocks where they fit (grid -> clusters per solve: 6 replicas of
// 8..96 x 4..40 sites 1.83 -> 0.49 ms, 32 of 32^2..128^2 4.30 -> 1.40 ms, 128 of
// 32^2..256^2 19.7 -> 11.9 ms, the 512-replica ensemble 46.1 -> 30.3 ms), else
// the grid solver.  The solvers group their sums differently (same accuracy, not
// the same bits).  The cluster solver runs in two forms, both candidates: the
// plain phase A (schedule 3) and the stencil on r (schedule 6, as schedule 8 of
// the equal-size solver; results agree to the solver's accuracy).
template <class Launch>
int tune_ragged(qed2d_batch* h, const RCGP& P, const CCGP& C, int maxiter, Launch launch) {
    h->rsched = 2;
    std::vector<std::pair<int, int>> cand = {{2, 0}};   // (schedule, blocks per cluster)
    for (int cs : kClusterSizes)
        if (cluster_fits(cs, replica_cluster_kernel(cs))) {
            cand.push_back({3, cs});
            if (cluster_fits(cs, replica_cluster_kernel(cs, true))) cand.push_back({6, cs});
        }
    if (!tuning_enabled()) {
        for (const auto& c : cand)
            if (c.first == 3 && c.second == 8) {
                h->rsched = 3;
                h->rcs = 8;
            }
        return QED2D_OK;
    }
    if (cand.size() == 1) return QED2D_OK;
    DevCtl saved;
    QCHECK(cudaMemcpyAsync(&saved, h->ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, h->stream));
    QCHECK(cudaStreamSynchronize(h->stream));
    RCGP TP = P;
    CCGP TC = C;
    TP.x = TC.x = h->field("tune_x");
    TP.t64 = TC.t64 = h->field("tune_g5x");
    TP.maxiter = TC.maxiter = std::min(maxiter, 24);
    if (!TP.x || !TP.t64) return QED2D_ERR_NO_MEMORY;
    cudaEvent_t e0, e1;
    QCHECK(cudaEventCreate(&e0));
    QCHECK(cudaEventCreate(&e1));
    std::vector<float> tbest(cand.size(), 1e30f);
    int st = QED2D_OK;
    for (int rep = 0; rep < 3 && st == QED2D_OK; rep++)
        for (size_t c = 0; c < cand.size() && st == QED2D_OK; c++) {
            cudaEventRecord(e0, h->stream);
            st = launch(cand[c].first, TP, TC, cand[c].second);
            cudaEventRecord(e1, h->stream);
            if (cudaEventSynchronize(e1) != cudaSuccess) st = cuda_status(cudaGetLastError(), "schedule tuning");
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) tbest[c] = std::min(tbest[c], ms);
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    QCHECK(cudaMemcpyAsync(h->ctl, &saved, sizeof(DevCtl), cudaMemcpyHostToDevice, h->stream));
    QCHECK(cudaStreamSynchronize(h->stream));
    if (st != QED2D_OK) return st;
    size_t best = 0;
    for (size_t c = 1; c < cand.size(); c++)
        if (tbest[c] < tbest[best]) best = c;
    h->rsched = cand[best].first;
    if (cand[best].second) h->rcs = cand[best].second;
    return QED2D_OK;
}

int r_solve(qed2d_batch* h, const double2* U, const float4* U32, const double2* b, double2* x, double2* g5x,
            int maxiter, double eps) {
    RCGP P{};
    P.nrep = h->nrep;
    P.reps = h->d_reps;
    P.segs = h->d_segs;
    P.seg0 = h->d_seg0;
    P.rep_seg = h->d_rep_seg;
    P.m2 = h->d_m2;
    P.U = U;
    P.U32 = U32;
    P.vtot = h->Vtot;
    P.b = b;
    P.x = x;
    P.t64 = g5x;
    P.r64 = h->field("b_r64");
    P.r32 = h->field32("b_r32");
    P.q0 = h->field32("b_q0");
    P.q1 = h->field32("b_q1");
    P.t32 = h->field32("b_t32");
    P.x32 = h->field32("b_x32");
    if (!P.r64 || !P.r32 || !P.q0 || !P.q1 || !P.t32 || !P.x32) return QED2D_ERR_NO_MEMORY;
    P.eps = eps;
    P.delta2 = kReliableDelta * kReliableDelta;
    P.maxiter = maxiter;
    P.st = h->d_st;
    P.flags = h->d_flags;
    P.red = h->d_red;
    P.cnt = h->d_cnt;
    P.flag_acc = h->d_cnt + h->nrep;
    P.part = h->d_part;
    P.ctl = h->ctl;
    if (h->uniform) {
        UCGP Q{};
        Q.g = h->ug;
        Q.U = U;
        Q.U32 = U32;
        Q.b = b;
        Q.x = x;
        Q.t64 = g5x;
        Q.r64 = P.r64;
        Q.r32 = P.r32;
        Q.q0 = P.q0;
        Q.q1 = P.q1;
        Q.t32 = P.t32;
        Q.x32 = P.x32;
        for (int r = 0; r < h->nrep; r++) Q.m2[r] = h->m2[r];
        Q.eps = eps;
        Q.delta2 = P.delta2;
        Q.maxiter = maxiter;
        Q.ctl = h->ctl;
        Q.part = h->d_upart;
        Q.red = h->d_ured;
        Q.rbar = h->d_ubar;
        Q.st_out = h->d_st;
        auto launch = [&](int sched, int tile, const UCGP& q0) -> int {
            const qed2d_batch::UVar& v = h->uv[tile];
            UCGP q = q0;
            q.g.ntr = v.ntr;
            q.bpr = v.bpr;
            q.per_block = v.per_block;
            QCHECK(cudaMemsetAsync(&h->ctl->bar, 0, 2 * sizeof(unsigned long long) + sizeof(int), h->stream));
            if (sched >= 4) QCHECK(cudaMemsetAsync(h->d_ubar, 0, sizeof(unsigned long long) * 16 * h->nrep, h->stream));
            if (sched == 7) {
                if (!v.tma) {
                    set_error("batch schedule 7 needs whole 32-site-wide tiles and co-resident blocks at this height");
                    return QED2D_ERR_UNSUPPORTED;
                }
                UTma tm;
                const unsigned long long L1 = (unsigned long long)q.g.L1, ny = (unsigned long long)q.g.L2 * q.g.B;
                const unsigned rows = (unsigned)v.rows;
                const float4* fld[4] = {q.r32, q.q0, q.q1, q.t32};
                for (int f = 0; f < 4; f++) {
                    QTRY(encode_map_2d(&tm.fc[f], fld[f], 4 * L1, ny, 16 * L1, 128, rows));
                    QTRY(encode_map_2d(&tm.fk[f], fld[f], 4 * L1, ny, 16 * L1, 4, rows));
                    QTRY(encode_map_2d(&tm.fw[f], fld[f], 4 * L1, ny, 16 * L1, 128, 1));
                }
                const float2* u1 = reinterpret_cast<const float2*>(q.U32);
                const float2* u2 = u1 + h->Vtot;   // the second link plane
                QTRY(encode_map_2d(&tm.u1c, u1, 2 * L1, ny, 8 * L1, 64, rows));
                QTRY(encode_map_2d(&tm.u1l, u1, 2 * L1, ny, 8 * L1, 4, rows));
                QTRY(encode_map_2d(&tm.u2c, u2, 2 * L1, ny, 8 * L1, 64, rows));
                QTRY(encode_map_2d(&tm.u2b, u2, 2 * L1, ny, 8 * L1, 64, 1));
                void* targs[] = {(void*)&q, (void*)&tm};
                QCHECK(cudaLaunchCooperativeKernel(uniform_kernel_tma(v.rows), dim3((unsigned)v.grid),
                                                   dim3((unsigned)(TX * v.rows)), targs, uniform_tma_smem(v.rows),
                                                   h->stream));
                count_launch();
                return QED2D_OK;
            }
            if (sched == 9 && !v.lsm) {
                set_error("batch schedule 9: the staged links do not fit co-resident at this tile height");
                return QED2D_ERR_UNSUPPORTED;
            }
            void* uargs[] = {(void*)&q};
            QCHECK(cudaLaunchCooperativeKernel(uniform_kernel(sched, v.rows), dim3((unsigned)v.grid),
                                               dim3((unsigned)(TX * v.rows)), uargs, sched == 9 ? v.lsm : 0,
                                               h->stream));
            count_launch();
            return QED2D_OK;
        };
        if (h->usched < 0 || h->utile < 0) QTRY(tune_uniform(h, Q, maxiter, launch));
        QTRY(launch(h->usched, h->utile, Q));
        k_r_finish<<<1, 256, 0, h->stream>>>(h->d_st, h->nrep, maxiter, h->d_out, h->d_out + h->nrep, h->d_iters,
                                              h->ctl);
        return r_post("k_r_finish");
    } else {
        CCGP C{};
        C.reps = h->d_reps;
        C.order = h->d_order;
        C.m2 = h->d_m2;
        C.U = U;
        C.U32 = U32;
        C.vtot = h->Vtot;
        C.b = b;
        C.x = x;
        C.t64 = g5x;
        C.r64 = P.r64;
        C.r32 = P.r32;
        C.q0 = P.q0;
        C.q1 = P.q1;
        C.t32 = P.t32;
        C.x32 = P.x32;
        C.eps = eps;
        C.delta2 = P.delta2;
        C.maxiter = maxiter;
        C.st_out = h->d_st;
        auto launch = [&](int sched, const RCGP& p, const CCGP& cc, int cs) -> int {
            if (sched == 3 || sched == 6) {
                QTRY(launch_replica_clusters(h, cc, cs, sched == 6));
            } else {
                QCHECK(cudaMemsetAsync(&h->ctl->bar, 0, 2 * sizeof(unsigned long long) + sizeof(int), h->stream));
                QCHECK(cudaMemsetAsync(h->d_cnt, 0, sizeof(int) * (h->nrep + 1), h->stream));   // counters at zero
                void* rargs[] = {(void*)&p};
                const void* kern =
                    h->shared_state ? (const void*)k_r_cg_mixed<true> : (const void*)k_r_cg_mixed<false>;
                QCHECK(cudaLaunchCooperativeKernel(kern, dim3((unsigned)h->grid), dim3(TILE), rargs, 0, h->stream));
            }
            count_launch();
            return QED2D_OK;
        };
        if (h->rsched < 0) QTRY(tune_ragged(h, P, C, maxiter, launch));
        QTRY(launch(h->rsched, P, C, h->rcs));
    }
    k_r_finish<<<1, 256, 0, h->stream>>>(h->d_st, h->nrep, maxiter, h->d_out, h->d_out + h->nrep, h->d_iters, h->ctl);
    return r_post("k_r_finish");
}

int r_kick(qed2d_batch* h, double* mom, const double2* U, const float4* U32, double2* X, const double2* F, double2* G,
           double eps, int maxiter, double tol) {
    QTRY(r_solve(h, U, U32, F, X, G, maxiter, tol));
    k_r_mom_kick<<<h->ntiles, TILE, 0, h->stream>>>(mom, U, h->tv(), h->d_beta, eps, X, G);
    return r_post("k_r_mom_kick");
}

template <class T>
int upload(T** d, const std::vector<T>& v) {
    QCHECK(cudaMalloc(d, sizeof(T) * std::max<size_t>(v.size(), 1)));
    QCHECK(cudaMemcpy(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    return QED2D_OK;
}

// replica table, tile table, persistent-grid geometry and (block, replica) segments
int batch_setup(qed2d_batch* h, const int* L1, const int* L2, const double* beta) {
    const int B = h->nrep;
    std::vector<int4> tiles;
    long long off = 0;
    for (int r = 0; r < B; r++) {
        RepInfo R{};
        R.L1 = L1[r];
        R.L2 = L2[r];
        R.nt1 = (L1[r] + TX - 1) / TX;
        const int nt2 = (L2[r] + TY - 1) / TY;
        R.nt = R.nt1 * nt2;
        R.V = (long long)L1[r] * L2[r];
        R.off = off;
        R.tile0 = (int)tiles.size();
        for (int t2 = 0; t2 < nt2; t2++)
            for (int t1 = 0; t1 < R.nt1; t1++) tiles.push_back(make_int4(r, t1, t2, 0));
        off += R.V;
        h->reps.push_back(R);
    }
    h->Vtot = off;
    h->ntiles = (int)tiles.size();
    h->beta.assign(beta, beta + B);
    h->m2.assign(B, 2.0);
    QCHECK(cudaGetDevice(&h->device));
    QCHECK(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device));
    int per_sm = 0;
    h->shared_state = B <= kSharedReps;
    if (h->shared_state) QCHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_r_cg_mixed<true>, TILE, 0));
    else QCHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_r_cg_mixed<false>, TILE, 0));
    if (per_sm < 1) {
        set_error("batch: the persistent solver does not fit on an SM");
        return QED2D_ERR_UNSUPPORTED;
    }
    const long long maxg = std::min<long long>((long long)per_sm * h->num_sms, kMaxPartBlocks);
    // Work order of the persistent solver: every replica's tiles cut into chunks
    // of `chunk` tiles, the chunks dealt round-robin over the replicas, so the
    // work of any one replica is spread over many blocks (a replica's FP64
    // reliable updates run while the others wait); blocks take contiguous
    // ranges of this order, and each run of consecutive tiles of one replica
    // inside a block is a segment with its own partial sum.
    const int chunk = std::max(8, (h->ntiles + 4095) / 4096);
    std::vector<int2> order;   // (replica, tile index inside the replica)
    order.reserve(h->ntiles);
    int maxch = 0;
    for (int r = 0; r < B; r++) maxch = std::max(maxch, (h->reps[r].nt + chunk - 1) / chunk);
    for (int k = 0; k < maxch; k++)
        for (int r = 0; r < B; r++)
            for (int lt = k * chunk; lt < std::min((k + 1) * chunk, h->reps[r].nt); lt++) order.push_back(make_int2(r, lt));
    h->per_block = (int)((h->ntiles + maxg - 1) / maxg);
    h->grid = (h->ntiles + h->per_block - 1) / h->per_block;
    std::vector<int> seg0(h->grid + 1);
    std::vector<SegDesc> segs;
    std::vector<std::vector<int>> rep_segs(B);   // segments of each replica, in block order
    for (int b = 0; b < h->grid; b++) {
        seg0[b] = (int)segs.size();
        const int lo = b * h->per_block, hi = std::min(lo + h->per_block, h->ntiles);
        for (int t = lo; t < hi; t++) {
            const int2 o = order[t];
            if (t > lo && o.x == order[t - 1].x && o.y == order[t - 1].y + 1) {
                segs.back().n++;
                continue;
            }
            const RepInfo& R = h->reps[o.x];
            rep_segs[o.x].push_back((int)segs.size());
            segs.push_back(SegDesc{o.x, o.y % R.nt1, o.y / R.nt1, 1, 0, 0, 0, 0});
        }
    }
    seg0[h->grid] = (int)segs.size();
    h->nseg = (int)segs.size();
    std::vector<int> rep_seg(B + 1, 0);   // partial slots: replica by replica
    for (int r = 0, slot = 0; r < B; r++) {
        rep_seg[r] = slot;
        for (int i : rep_segs[r]) segs[i].slot = slot++;
        rep_seg[r + 1] = slot;
    }
    // equal sizes and few replicas: the uniform kernel, whole blocks per replica
    bool same = B <= kUniformReps;
    for (int r = 1; r < B && same; r++) same = L1[r] == L1[0] && L2[r] == L2[0];
    if (same) {
        // one geometry per tile height: as many blocks per replica as stay
        // co-resident (cooperative launch), tiles dealt in contiguous ranges
        const RepInfo& R0 = h->reps[0];
        for (int rows : kUTileRows) {
            int per_smu = 1 << 30;
            for (int sched : {0, 1, 4, 5, 8}) {
                int n = 0;
                QCHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, uniform_kernel(sched, rows), TX * rows, 0));
                per_smu = std::min(per_smu, n);
            }
            const long long maxgu = std::min<long long>((long long)per_smu * h->num_sms, kMaxPartBlocks);
            if (per_smu < 1 || maxgu / B < 1) continue;
            qed2d_batch::UVar v;
            v.rows = rows;
            v.ntr = (long long)R0.nt1 * ((R0.L2 + rows - 1) / rows);
            const long long bpr = maxgu / B;
            v.per_block = (int)((v.ntr + bpr - 1) / bpr);
            v.bpr = (int)((v.ntr + v.per_block - 1) / v.per_block);
            v.grid = v.bpr * B;
            if (const void* kt = uniform_kernel_tma(rows); kt && R0.L1 % TX == 0 && R0.L2 % rows == 0) {
                const size_t sm = uniform_tma_smem(rows);
                int n7 = 0;
                if (cudaFuncSetAttribute(kt, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) == cudaSuccess &&
                    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n7, kt, TX * rows, sm) == cudaSuccess)
                    v.tma = (long long)n7 * h->num_sms >= v.grid;
                cudaGetLastError();
            }
            {   // schedule 9: the grid stays co-resident with the staged links
                // (the attribute is set to what the device allows beside the
                // kernel's static shared memory, so batches of other sizes keep
                // launching the same kernel)
                const size_t sm = uniform_lsm_bytes(rows, v.per_block);
                const void* k9 = uniform_kernel(9, rows);
                int n9 = 0, optin = 0;
                cudaFuncAttributes fa{};
                if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device) == cudaSuccess &&
                    cudaFuncGetAttributes(&fa, k9) == cudaSuccess && sm + fa.sharedSizeBytes <= (size_t)optin &&
                    cudaFuncSetAttribute(k9, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         optin - (int)fa.sharedSizeBytes) == cudaSuccess &&
                    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n9, k9, TX * rows, sm) == cudaSuccess &&
                    (long long)n9 * h->num_sms >= v.grid)
                    v.lsm = sm;
                cudaGetLastError();
            }
            h->uv[h->nuv++] = v;
        }
        if (h->nuv > 0) {
            h->uniform = true;
            h->ug = UGeom{R0.L1, R0.L2, B, R0.nt1, R0.V, 0};
        }
    }
    std::vector<long long> dbc(B + 1), dbr(B + 1);
    for (int r = 0; r <= B; r++) {
        const long long o = r < B ? h->reps[r].off : h->Vtot;
        dbc[r] = 4 * o;   // complex fields: 2 planes x 2 doubles per site
        dbr[r] = 2 * o;   // real fields: 2 planes
    }
    QTRY(upload(&h->d_reps, h->reps));
    QTRY(upload(&h->d_tiles, tiles));
    QTRY(upload(&h->d_seg0, seg0));
    QTRY(upload(&h->d_segs, segs));
    {   // cluster solver: largest replicas first (they take longest)
        std::vector<int> order(B);
        for (int r = 0; r < B; r++) order[r] = r;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b2) { return h->reps[a].nt > h->reps[b2].nt; });
        QTRY(upload(&h->d_order, order));
    }
    QTRY(upload(&h->d_rep_seg, rep_seg));
    QTRY(upload(&h->d_dbase_c, dbc));
    QTRY(upload(&h->d_dbase_r, dbr));
    QTRY(upload(&h->d_beta, h->beta));
    QTRY(upload(&h->d_m2, h->m2));
    QCHECK(cudaMalloc(&h->d_seed, sizeof(uint64_t) * B));
    QCHECK(cudaMalloc(&h->d_st, sizeof(RepState) * B));
    QCHECK(cudaMalloc(&h->d_flags, sizeof(int) * FL_N));
    QCHECK(cudaMalloc(&h->d_red, sizeof(double) * 2 * B));
    QCHECK(cudaMalloc(&h->d_cnt, sizeof(int) * (B + 1)));
    if (h->uniform) {
        int gmax = 0;
        for (int t = 0; t < h->nuv; t++) gmax = std::max(gmax, h->uv[t].grid);
        QCHECK(cudaMalloc(&h->d_upart, sizeof(double) * 2 * (size_t)gmax));
        QCHECK(cudaMalloc(&h->d_ured, sizeof(double) * 2 * B));
        QCHECK(cudaMalloc(&h->d_ubar, sizeof(unsigned long long) * 16 * B));
    }
    QCHECK(cudaMalloc(&h->d_out, sizeof(int) * 2 * B));
    QCHECK(cudaMalloc(&h->d_iters, sizeof(long long) * B));
    QCHECK(cudaMalloc(&h->d_sums, sizeof(double) * 2 * 5 * B));
    QCHECK(cudaMalloc(&h->d_tpart, sizeof(double) * 10 * h->ntiles));
    QCHECK(cudaMalloc(&h->d_part, sizeof(double) * h->nseg));
    QCHECK(cudaMalloc(&h->ctl, sizeof(DevCtl)));
    QCHECK(cudaMallocHost(&h->ctl_host, sizeof(DevCtl)));
    QCHECK(cudaMemset(h->ctl, 0, sizeof(DevCtl)));
    return QED2D_OK;
}

int set_masses(qed2d_batch* h, const double* am0) {
    for (int r = 0; r < h->nrep; r++) h->m2[r] = 2.0 + am0[r];
    QCHECK(cudaMemcpyAsync(h->d_m2, h->m2.data(), sizeof(double) * h->nrep, cudaMemcpyHostToDevice, h->stream));
    return QED2D_OK;
}

}  // namespace

extern "C" {

int qed2d_batch_create_ragged(int nrep, const int* L1, const int* L2, const double* beta, qed2d_batch** out) {
    if (!out) return QED2D_ERR_BAD_ARG;
    *out = nullptr;
    if (nrep < 1 || nrep > kMaxReplicas || !L1 || !L2 || !beta) {
        set_error("qed2d_batch_create_ragged: need 1 <= nrep <= 1024 and L1, L2, beta for every replica");
        return QED2D_ERR_BAD_ARG;
    }
    long long V = 0;
    for (int r = 0; r < nrep; r++) {
        if (L1[r] < 2 || L2[r] < 2 || L1[r] > (1 << 20) || L2[r] > (1 << 20)) {
            set_error("qed2d_batch_create_ragged: lattice extents must lie in [2, 2^20]");
            return QED2D_ERR_BAD_ARG;
        }
        V += (long long)L1[r] * L2[r];
        if (V > (1LL << 30)) {
            set_error("qed2d_batch_create_ragged: more than 2^30 sites in the batch");
            return QED2D_ERR_BAD_ARG;
        }
    }
    auto* h = new qed2d_batch();
    h->nrep = nrep;
    const int st = batch_setup(h, L1, L2, beta);
    if (st != QED2D_OK) {
        qed2d_batch_destroy(h);
        return st;
    }
    *out = h;
    return QED2D_OK;
}

int qed2d_batch_create(int nrep, int L1, int L2, const double* beta, qed2d_batch** out) {
    if (!out) return QED2D_ERR_BAD_ARG;
    *out = nullptr;
    if (nrep < 1 || nrep > kMaxReplicas) {
        set_error("qed2d_batch_create: need 1 <= nrep <= 1024");
        return QED2D_ERR_BAD_ARG;
    }
    const std::vector<int> a(nrep, L1), b(nrep, L2);
    return qed2d_batch_create_ragged(nrep, a.data(), b.data(), beta, out);
}

int qed2d_batch_destroy(qed2d_batch* h) {
    if (!h) return QED2D_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    else cudaDeviceSynchronize();
    h->md_graph.release();
    for (auto& kv : h->ws) cudaFree(kv.second.first);
    void* dev[] = {h->d_reps,  h->d_tiles, h->d_seg0,  h->d_segs,  h->d_order, h->d_rep_seg, h->d_dbase_c,
                   h->d_dbase_r, h->d_m2,  h->d_beta,  h->d_seed,  h->d_st,    h->d_flags,   h->d_red,
                   h->d_cnt,   h->d_upart, h->d_ured,  h->d_ubar,  h->d_out,   h->d_iters,   h->d_sums,
                   h->d_tpart, h->d_part,  h->ctl};
    for (void* p : dev)
        if (p) cudaFree(p);
    if (h->ctl_host) cudaFreeHost(h->ctl_host);
    delete h;
    return QED2D_OK;
}

int qed2d_batch_set_graphs(qed2d_batch* h, int on) {
    if (!h) return QED2D_ERR_BAD_ARG;
    h->md_graph.drop();
    h->md_graph.on = on != 0;
    return QED2D_OK;
}

int qed2d_batch_graph_stats(const qed2d_batch* h, int* on, int64_t* captures, int64_t* replays, int64_t* failures) {
    if (!h) return QED2D_ERR_BAD_ARG;
    const GraphCache& g = h->md_graph;
    if (on) *on = g.on ? 1 : 0;
    if (captures) *captures = g.captures;
    if (replays) *replays = g.replays;
    if (failures) *failures = g.failures;
    return QED2D_OK;
}

int qed2d_batch_set_stream(qed2d_batch* h, void* stream) {
    if (!h) return QED2D_ERR_BAD_ARG;
    h->stream = (cudaStream_t)stream;
    return QED2D_OK;
}

int qed2d_batch_set_schedule(qed2d_batch* h, int schedule) {
    const bool ok = h && (schedule == -1 || (h->uniform ? (schedule == 0 || schedule == 1 || schedule == 4 ||
                                                          schedule == 5 || schedule == 7 || schedule == 8 ||
                                                          schedule == 9)
                                                         : (schedule == 2 || schedule == 3 || schedule == 6)));
    if (!ok) {
        set_error(
            "qed2d_batch_set_schedule: -1, or 0/1/4/5/7/8/9 (equal sizes, at most 64 replicas), or 2/3/6 (otherwise)");
        return QED2D_ERR_BAD_ARG;
    }
    if (h->uniform) {
        h->usched = schedule;
        h->usched_fixed = schedule >= 0;
    } else {
        h->rsched = schedule;
    }
    return QED2D_OK;
}

int qed2d_batch_get_schedule(const qed2d_batch* h, int* schedule) {
    if (!h || !schedule) return QED2D_ERR_BAD_ARG;
    *schedule = h->uniform ? h->usched : h->rsched;
    return QED2D_OK;
}

int qed2d_batch_set_tile_rows(qed2d_batch* h, int rows) {
    if (!h || !h->uniform) {
        set_error("qed2d_batch_set_tile_rows: only equal-size batches of at most 64 replicas have tile heights");
        return QED2D_ERR_BAD_ARG;
    }
    if (rows == -1) {
        h->utile_fixed = false;
        h->utile = -1;
        return QED2D_OK;
    }
    for (int t = 0; t < h->nuv; t++)
        if (h->uv[t].rows == rows) {
            h->utile = t;
            h->utile_fixed = true;
            return QED2D_OK;
        }
    set_error("qed2d_batch_set_tile_rows: rows must be -1 or one of 4, 8, 16 (with co-resident blocks)");
    return QED2D_ERR_BAD_ARG;
}

int qed2d_batch_get_tile_rows(const qed2d_batch* h, int* rows) {
    if (!h || !rows) return QED2D_ERR_BAD_ARG;
    *rows = (h->uniform && h->utile >= 0) ? h->uv[h->utile].rows : -1;
    return QED2D_OK;
}

int qed2d_batch_layout(const qed2d_batch* h, int64_t* site_offsets) {
    if (!h || !site_offsets) return QED2D_ERR_BAD_ARG;
    for (int r = 0; r < h->nrep; r++) site_offsets[r] = h->reps[r].off;
    site_offsets[h->nrep] = h->Vtot;
    return QED2D_OK;
}

int qed2d_batch_cg(qed2d_batch* h, double* x, const double* U, const double* b, const double* am0, int maxiter,
                   double eps, int* iterations, int* updates) {
    if (!h || !x || !U || !b || !am0 || maxiter < 0 ||
        ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(U) | reinterpret_cast<uintptr_t>(b)) % 16)) {
        set_error("qed2d_batch_cg: bad argument");
        return QED2D_ERR_BAD_ARG;
    }
    const size_t fb = sizeof(double2) * 2 * (size_t)h->Vtot;
    if ((const char*)x < (const char*)b + fb && (const char*)b < (const char*)x + fb) {
        set_error("qed2d_batch_cg: x aliases b");
        return QED2D_ERR_BAD_ARG;
    }
    cudaStream_t s = h->stream;
    float4* U32 = h->field32("b_U32");
    double2* G = h->field("b_G");
    if (!U32 || !G) return QED2D_ERR_NO_MEMORY;
    QTRY(set_masses(h, am0));
    QCHECK(cudaMemsetAsync(&h->ctl->status, 0, sizeof(int), s));
    QCHECK(cudaMemsetAsync(h->d_iters, 0, sizeof(long long) * h->nrep, s));
    QTRY(r_pack(h, const_cast<double2*>((const double2*)U), nullptr, 0.0, U32));   // eps = 0: U is only read
    QTRY(r_solve(h, (const double2*)U, U32, (const double2*)b, (double2*)x, G, maxiter, eps));
    std::vector<int> out(2 * h->nrep);
    QCHECK(cudaMemcpyAsync(out.data(), h->d_out, sizeof(int) * out.size(), cudaMemcpyDeviceToHost, s));
    QCHECK(cudaMemcpyAsync(h->ctl_host, h->ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, s));
    QCHECK(cudaStreamSynchronize(s));
    for (int r = 0; r < h->nrep; r++) {
        if (iterations) iterations[r] = out[r];
        if (updates) updates[r] = out[h->nrep + r];
    }
    const int st = h->ctl_host->status;
    if (st != QED2D_OK) set_error(std::string("qed2d_batch_cg: ") + qed2d_status_string(st));
    return st;
}

int qed2d_batch_hmc_nf2(qed2d_batch* h, double* Ud, const double* am0, double eps, int ns, int maxiter, double tol,
                        int qzero, const uint64_t* seeds, uint32_t counter, qed2d_hmc_result* res) {
    if (!h || !Ud || !am0 || !seeds || ns < 1 || maxiter < 0 || (reinterpret_cast<uintptr_t>(Ud) % 16)) {
        set_error("qed2d_batch_hmc_nf2: bad argument");
        return QED2D_ERR_BAD_ARG;
    }
    const int B = h->nrep;
    double2* U = (double2*)Ud;
    double2* Ucp = h->field("b_Ucp");
    double* mom = h->real2("b_mom");
    double2* X = h->field("b_X");
    double2* F = h->field("b_F");
    double2* G = h->field("b_G");
    float4* U32 = h->field32("b_U32");
    if (!Ucp || !mom || !X || !F || !G || !U32) return QED2D_ERR_NO_MEMORY;
    cudaStream_t s = h->stream;
    QTRY(set_masses(h, am0));
    QCHECK(cudaMemcpyAsync(h->d_seed, seeds, sizeof(uint64_t) * B, cudaMemcpyHostToDevice, s));
    QCHECK(cudaMemsetAsync(h->d_iters, 0, sizeof(long long) * B, s));
    QCHECK(cudaMemsetAsync(&h->ctl->status, 0, sizeof(int), s));
    QCHECK(cudaMemcpyAsync(Ucp, U, sizeof(double2) * 2 * h->Vtot, cudaMemcpyDeviceToDevice, s));
    // draws (src/QED2dHMC.jl:69-70), H_ini, F = g5Dw X (:74-78)
    QTRY(r_fill(h, mom, false, QED2D_STREAM_MOMENTA, counter, 1.0));
    QTRY(r_fill(h, (double*)X, true, QED2D_STREAM_NOISE, counter, 1.0 / std::sqrt(2.0)));
    QTRY(r_sums(h, U, mom, X, nullptr, 0));
    k_r_g5dw<<<h->ntiles, TILE, 0, s>>>(F, U, X, h->tv(), h->d_m2);
    QTRY(r_post("k_r_g5dw"));
    // FP32 links, then leapfrog (src/QED2dHMC.jl:426-449): replayed from a CUDA
    // graph from the third trajectory with the same arguments on (graph.h)
    GraphKey k;
    k.p(U).p(mom).p(X).p(F).p(G).p(U32).d(eps).i(ns).i(maxiter).d(tol);
    k.i(h->usched).i(h->utile).i(h->rsched).i(h->rcs).i((long long)h->ws_gen);
    for (int r = 0; r < B; r++) k.d(h->m2[r]);
    QTRY(run_graphed(h->md_graph, h->stream, k.s, [&]() -> int {
        QTRY(r_pack(h, U, mom, 0.0, U32));
        QTRY(r_kick(h, mom, U, U32, X, F, G, 0.5 * eps, maxiter, tol));
        for (int i = 0; i < ns - 1; i++) {
            QTRY(r_pack(h, U, mom, eps, U32));
            QTRY(r_kick(h, mom, U, U32, X, F, G, eps, maxiter, tol));
        }
        QTRY(r_pack(h, U, mom, eps, U32));
        return r_kick(h, mom, U, U32, X, F, G, 0.5 * eps, maxiter, tol);
    }));
    // H_fin with <X, F> (:82)
    QTRY(r_sums(h, U, mom, X, F, 1));
    std::vector<double> sc(2 * 5 * (size_t)B);
    std::vector<long long> its(B);
    QCHECK(cudaMemcpyAsync(sc.data(), h->d_sums, sizeof(double) * sc.size(), cudaMemcpyDeviceToHost, s));
    QCHECK(cudaMemcpyAsync(its.data(), h->d_iters, sizeof(long long) * B, cudaMemcpyDeviceToHost, s));
    QCHECK(cudaMemcpyAsync(h->ctl_host, h->ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, s));
    QCHECK(cudaStreamSynchronize(s));
    const int st = h->ctl_host->status;
    for (int r = 0; r < B; r++) {
        const RepInfo& R = h->reps[r];
        const double* a = &sc[(size_t)r * 5];
        const double* f = &sc[(size_t)(B + r) * 5];
        const double hini = a[2] / 2.0 + h->beta[r] * ((double)R.V - a[0]) + a[3];
        const double hfin = f[2] / 2.0 + h->beta[r] * ((double)R.V - f[0]) + f[4];
        const double qf = f[1] / (2.0 * M_PI);
        const double pacc = (qzero && std::fabs(qf) > 0.1) ? 0.0 : std::exp(-(hfin - hini));
        int acc = 1;
        if (st != QED2D_OK) acc = 0;
        else if (pacc < 1.0) acc = pacc > qed2d_random_uniform(seeds[r], QED2D_STREAM_METROPOLIS, counter);
        if (!acc)   // restore the replica's links: one contiguous block
            QCHECK(cudaMemcpyAsync(U + 2 * R.off, Ucp + 2 * R.off, sizeof(double2) * 2 * R.V, cudaMemcpyDeviceToDevice,
                                   s));
        if (res) {
            res[r].accepted = acc;
            res[r].hini = hini;
            res[r].hfin = hfin;
            res[r].dH = hfin - hini;
            res[r].qtop = acc ? qf : a[1] / (2.0 * M_PI);
            res[r].cg_iterations = its[r];
        }
    }
    QCHECK(cudaStreamSynchronize(s));
    if (st != QED2D_OK) set_error(std::string("batch HMC! Nf=2: ") + qed2d_status_string(st));
    return st;
}

}  // extern "C"
