// batch.cu -- batched replicas: B independent lattices of the same size advanced
// together.  Every kernel of an Nf=2 trajectory covers all replicas, and every
// force evaluation is ONE persistent mixed-precision CG launch that solves the B
// systems at once (per-replica scalars, convergence and reliable updates), so
// the grid barriers and launch latencies of a solve are paid once for B
// lattices.  This is the batching of independent Markov chains (ensemble
// generation); every replica follows exactly the algorithm of HMC! Nf=2
// (src/QED2dHMC.jl:64-113) with leapfrog (:426-481).
//
// Layout: a batch field is the reference layout of an L1 x (B*L2) lattice,
//   element (i1, i2, replica r, plane k) at  i1 + L1*(i2 + L2*(r + B*k)),
// so plane k of replica r is one contiguous reference-layout block of L1*L2
// elements at offset (r + B*k)*L1*L2.  Neighbours in direction 2 wrap inside each
// replica.  Random draws of replica r use its own seed and the element index of
// a single lattice, so replica r reproduces a single-lattice run with seed r.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "stencil.cuh"

namespace qed2d {

constexpr int kMaxBatch = 64;

struct BLat {
    int L1, L2r, B;
    long long Vr, V;   // sites per replica, total
    int nt1;           // tiles along i1
    long long ntr;     // tiles per replica
};

static BLat make_blat(int B, int L1, int L2) {
    BLat g;
    g.L1 = L1;
    g.L2r = L2;
    g.B = B;
    g.Vr = (long long)L1 * L2;
    g.V = g.Vr * B;
    g.nt1 = (L1 + TX - 1) / TX;
    g.ntr = (long long)g.nt1 * ((L2 + TY - 1) / TY);
    return g;
}

// site of thread t in local tile lt of replica r; neighbours wrap inside the replica
__device__ __forceinline__ Site bsite(const BLat& g, int r, long long lt, int t) {
    const int t2 = (int)(lt / g.nt1), t1 = (int)(lt - (long long)t2 * g.nt1);
    Site s;
    s.i1 = t1 * TX + (t & (TX - 1));
    s.i2 = t2 * TY + (t >> 5);
    s.ok = s.i1 < g.L1 && s.i2 < g.L2r;
    s.x = s.i1 + (long long)g.L1 * ((long long)r * g.L2r + s.i2);
    s.xp1 = (s.i1 + 1 == g.L1) ? s.x - (g.L1 - 1) : s.x + 1;
    s.xm1 = (s.i1 == 0) ? s.x + (g.L1 - 1) : s.x - 1;
    s.xp2 = (s.i2 + 1 == g.L2r) ? s.x - (long long)(g.L2r - 1) * g.L1 : s.x + g.L1;
    s.xm2 = (s.i2 == 0) ? s.x + (long long)(g.L2r - 1) * g.L1 : s.x - g.L1;
    return s;
}

// the same without division: tile (t1, t2) of replica r
__device__ __forceinline__ Site bsite_at(const BLat& g, int r, int t1, int t2, int t) {
    Site s;
    s.i1 = t1 * TX + (t & (TX - 1));
    s.i2 = t2 * TY + (t >> 5);
    s.ok = s.i1 < g.L1 && s.i2 < g.L2r;
    s.x = s.i1 + g.L1 * (r * g.L2r + s.i2);   // 32-bit: V < 2^30 is checked at creation
    s.xp1 = (s.i1 + 1 == g.L1) ? s.x - (g.L1 - 1) : s.x + 1;
    s.xm1 = (s.i1 == 0) ? s.x + (g.L1 - 1) : s.x - 1;
    s.xp2 = (s.i2 + 1 == g.L2r) ? s.x - (long long)(g.L2r - 1) * g.L1 : s.x + g.L1;
    s.xm2 = (s.i2 == 0) ? s.x + (long long)(g.L2r - 1) * g.L1 : s.x - g.L1;
    return s;
}

// ---------------------------------------------------------------------------
// standalone batched kernels: grid = (tiles per replica, B)
__global__ void __launch_bounds__(TILE) k_b_g5dw(double2* __restrict__ so, const double2* __restrict__ U,
                                                 const double2* __restrict__ si, BLat g, const double* __restrict__ m2) {
    const int r = blockIdx.y;
    const Site q = bsite(g, r, blockIdx.x, threadIdx.x);
    if (!q.ok) return;
    st_d(so, g.V, q.x, g5dw_at<double>(SpDro{si, g.V}, LkD{U, g.V}, q, m2[r]));
}

__device__ __forceinline__ double b_im_plaq(const double2* U, const BLat& g, int r, int i1, int i2) {
    const int iu1 = (i1 + 1 == g.L1) ? 0 : i1 + 1;
    const int iu2 = (i2 + 1 == g.L2r) ? 0 : i2 + 1;
    const long long row = (long long)r * g.L2r;
    const long long x = i1 + (long long)g.L1 * (row + i2);
    const double2 p = plaquette_of(__ldg(U + x), __ldg(U + g.V + iu1 + (long long)g.L1 * (row + i2)),
                                   __ldg(U + i1 + (long long)g.L1 * (row + iu2)), __ldg(U + g.V + x));
    return p.y;
}

// mom += eps (gauge force with beta_r + fermion force from (X, G)) -- k_mom_kick per replica
__global__ void __launch_bounds__(TILE) k_b_mom_kick(double* __restrict__ mom, const double2* __restrict__ U,
                                                     BLat g, const double* __restrict__ beta, double eps,
                                                     const double2* __restrict__ X, const double2* __restrict__ G) {
    const int r = blockIdx.y;
    const Site q = bsite(g, r, blockIdx.x, threadIdx.x);
    if (!q.ok) return;
    const int im1 = (q.i1 == 0) ? g.L1 - 1 : q.i1 - 1;
    const int im2 = (q.i2 == 0) ? g.L2r - 1 : q.i2 - 1;
    const double b = beta[r];
    const double v = b * b_im_plaq(U, g, r, q.i1, q.i2);
    const double vm2 = b * b_im_plaq(U, g, r, q.i1, im2);
    const double vm1 = b * b_im_plaq(U, g, r, im1, q.i2);
    double F1 = -v + vm2, F2 = v - vm1;
    if (X) {
        double f1, f2;
        fermion_force_at(U, X, G, g.V, q, f1, f2);
        F1 = F1 + f1;
        F2 = F2 + f2;
    }
    mom[q.x] = mom[q.x] + eps * F1;
    mom[q.x + g.V] = mom[q.x + g.V] + eps * F2;
}

// N(0,1) fields of every replica: replica r draws with seed seeds[r] the doubles of
// a single-lattice array of 2 Vr elements of dbl_per_elem doubles each (1: real
// momenta, 2: complex noise), in the single-lattice order, and stores them in the
// batch layout
__global__ void k_b_random_normal(double* __restrict__ out, BLat g, int dbl_per_elem, const uint64_t* __restrict__ seeds,
                                  uint32_t stream, uint32_t counter, double scale) {
    // one thread per pair of doubles of one replica's single-lattice array
    const int r = blockIdx.y;
    const long long n = 2 * g.Vr * dbl_per_elem;   // doubles of one replica
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (2 * j >= n) return;
    double z0, z1;
    normal_pair(seeds[r], stream, counter, (uint64_t)j, z0, z1);
    // double index d of the single-lattice array -> (plane, site, component)
    for (int h = 0; h < 2; h++) {
        const long long d = 2 * j + h;
        if (d >= n) break;
        const long long e = d / dbl_per_elem, comp = d - e * dbl_per_elem;
        const long long k = e / g.Vr, x = e - k * g.Vr;
        out[((k * g.B + r) * g.Vr + x) * dbl_per_elem + comp] = scale * (h ? z1 : z0);
    }
}

// per-replica sums: (Re P, arg P, mom^2, |X|^2, Re<X,F>) -- grid = (nb, B)
constexpr int RBB = 256;
__global__ void __launch_bounds__(RBB) k_b_reduce(const double2* __restrict__ U, const double* __restrict__ mom,
                                                  const double2* __restrict__ X, const double2* __restrict__ F,
                                                  BLat g, double* __restrict__ part, double* __restrict__ out) {
    const int r = blockIdx.y;
    double v[5] = {0, 0, 0, 0, 0};
    const long long row0 = (long long)r * g.L2r;
    for (long long s = blockIdx.x * (long long)RBB + threadIdx.x; s < g.Vr; s += (long long)gridDim.x * RBB) {
        const int i2 = (int)(s / g.L1), i1 = (int)(s - (long long)i2 * g.L1);
        const long long x = i1 + (long long)g.L1 * (row0 + i2);
        if (U) {
            const int iu1 = (i1 + 1 == g.L1) ? 0 : i1 + 1, iu2 = (i2 + 1 == g.L2r) ? 0 : i2 + 1;
            const double2 p = plaquette_of(__ldg(U + x), __ldg(U + g.V + iu1 + (long long)g.L1 * (row0 + i2)),
                                           __ldg(U + i1 + (long long)g.L1 * (row0 + iu2)), __ldg(U + g.V + x));
            v[0] += p.x;
            v[1] += atan2(p.y, p.x);
        }
        if (mom) v[2] += mom[x] * mom[x] + mom[x + g.V] * mom[x + g.V];
        if (X) {
            const double2 a = X[x], b = X[x + g.V];
            v[3] += norm2(a) + norm2(b);
            if (F) v[4] += cjmul(a, F[x]).x + cjmul(b, F[x + g.V]).x;
        }
    }
    __shared__ double smem[32 * 5];
    block_sum<5>(v, smem);
    if (threadIdx.x == 0)
        for (int k = 0; k < 5; k++) part[((size_t)r * 5 + k) * gridDim.x + blockIdx.x] = v[k];
}

// fixed-order final sums of k_b_reduce's partials: out[r*5 + k]
__global__ void k_b_reduce_final(const double* __restrict__ part, int nb, int B, double* __restrict__ out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int rk = warp; rk < B * 5; rk += nw) {
        double s = 0.0;
        for (int i = lane; i < nb; i += 32) s += part[(size_t)rk * nb + i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) out[rk] = s;
    }
}

// ---------------------------------------------------------------------------
// Batched persistent mixed CG.  Block b serves replica b / bpr and that
// replica's tiles lb, lb + bpr, ... (lb = b % bpr); its partial sums belong to
// one replica, and the last block at a barrier sums each replica's partials in
// a fixed order (deterministic).  Per-replica scalars live in shared memory,
// computed identically in every block.  Replicas that have converged stop
// working but keep joining the barriers until all are done.
struct BCGP {
    BLat g;
    const double2* U;
    const float4* U32;
    const double2* b;
    double2* x;
    double2* r64;
    double2* t64;   // g5Dw x of the solution (the force needs it)
    float4* r32;
    float4* q0;
    float4* q1;
    float4* t32;
    float4* x32;
    double m2[kMaxBatch];
    double eps, delta2;
    int maxiter, bpr, per_block;
    DevCtl* ctl;
    double* part;
    int* out_iters;   // [B] iterations of this solve
    int* out_conv;    // [B]
    int* out_upd;     // [B] FP64 reliable updates
};

__device__ __forceinline__ bool breduce(GridSync& gs, double v, const BCGP& P, double* smem, double* out) {
    __shared__ int s_last;
    const int buf = gs.nred++ & 1;
    double* part = P.part + (size_t)buf * (kMaxPartVals / 2) * kMaxPartBlocks;
    double* red = part + kMaxPartBlocks;
    double vv[1] = {v};
    block_sum<1>(vv, smem);
    if (threadIdx.x == 0) part[blockIdx.x] = vv[0];
    const bool last = gs.arrive(&s_last);
    if (last) {
        __threadfence();
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
        for (int r = warp; r < P.g.B; r += nw) {
            double s = 0.0;
            for (int i = lane; i < P.bpr; i += 32) s += __ldcg(part + (size_t)r * P.bpr + i);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) red[r] = s;
        }
        __syncthreads();
        if (threadIdx.x == 0) gs.release();
    } else if (threadIdx.x == 0) {
        gs.wait();
    }
    __syncthreads();
    for (int r = threadIdx.x; r < P.g.B; r += blockDim.x) out[r] = __ldcg(red + r);
    __syncthreads();
    return ld_volatile_int(gs.err) == 0;
}

// this block's contiguous range of its replica's tiles, walked without division
#define FOR_MY_TILES(q)                                                                            \
    for (int tt_ = TR.lo, t1_ = TR.s1, t2_ = TR.s2; tt_ < TR.hi;                                 \
         ++tt_, (++t1_ == TR.nt1 ? (t1_ = 0, ++t2_) : 0))                                          \
        if (const Site q = bsite_at(P.g, myr, t1_, t2_, threadIdx.x); q.ok)

__global__ void __launch_bounds__(TILE, 4) k_b_cg_mixed(const BCGP P) {
    __shared__ double smem[64];
    __shared__ double s_bb[kMaxBatch], s_tol[kMaxBatch], s_rr[kMaxBatch], s_maxrr[kMaxBatch], s_s[kMaxBatch],
        s_beta[kMaxBatch], s_alpha[kMaxBatch], s_rr64[kMaxBatch], s_tmp[kMaxBatch], s_snew[kMaxBatch];
    __shared__ int s_act[kMaxBatch], s_it[kMaxBatch], s_conv[kMaxBatch], s_upd[kMaxBatch], s_r4[kMaxBatch],
        s_first[kMaxBatch], s_nupd[kMaxBatch], s_any[2];
    GridSync gs{&P.ctl->bar, &P.ctl->gen, &P.ctl->err};
    const int B = P.g.B;
    const int myr = blockIdx.x / P.bpr, lb = blockIdx.x % P.bpr;
    const TileRange TR = tile_range(P.g.ntr, P.g.nt1, P.per_block, lb);
    const long long V = P.g.V;
    const LkD L{P.U, V};
    const LkF Lf{P.U32};
    const double m2 = P.m2[myr];
    const float m2f = (float)m2;
    const Pair<double> z{make_double2(0, 0), make_double2(0, 0)};
    bool ok = true;
    int k = 0, cur = 0;

    // |b|^2 per replica; x = 0
    {
        double v = 0.0;
        FOR_MY_TILES(q) {
            const Pair<double> bv{__ldg(P.b + q.x), __ldg(P.b + q.x + V)};
            v += norm2(bv.a) + norm2(bv.b);
            st_d(P.x, V, q.x, z);
        }
        if (!breduce(gs, v, P, smem, s_bb)) { ok = false; goto done; }
    }
    for (int r = threadIdx.x; r < B; r += blockDim.x) {
        s_tol[r] = P.eps * s_bb[r];
        s_act[r] = s_bb[r] > 0.0;
        s_conv[r] = s_bb[r] == 0.0;
        s_it[r] = 0;
        s_rr64[r] = s_bb[r];
        s_s[r] = s_bb[r] > 0.0 ? 1.0 / sqrt(s_bb[r]) : 0.0;
        s_first[r] = 1;
        s_beta[r] = 0.0;
        s_nupd[r] = 0;
    }
    __syncthreads();
    // r32 = s b, x32 = 0 (and g5Dw x = 0 for a zero source)
    {
        double v = 0.0;
        const double s = s_s[myr];
        const bool act = s_act[myr];
        FOR_MY_TILES(q) {
            if (act) {
                const Pair<float> r32{to_f(s * __ldg(P.b + q.x)), to_f(s * __ldg(P.b + q.x + V))};
                st_f(P.r32, q.x, r32);
                st_f(P.x32, q.x, Pair<float>{make_float2(0, 0), make_float2(0, 0)});
                v += (double)(norm2(r32.a) + norm2(r32.b));
            } else {
                st_d(P.t64, V, q.x, z);
            }
        }
        if (!breduce(gs, v, P, smem, s_rr)) { ok = false; goto done; }
    }
    for (int r = threadIdx.x; r < B; r += blockDim.x) s_maxrr[r] = s_rr[r];
    __syncthreads();

    for (k = 1; k <= P.maxiter; k++) {
        if (threadIdx.x == 0) {
            int any = 0;
            for (int r = 0; r < B; r++) any |= s_act[r];
            s_any[0] = any;
        }
        __syncthreads();
        if (!s_any[0]) break;
        float4* qn = cur ? P.q1 : P.q0;
        const float4* qo = cur ? P.q0 : P.q1;
        const bool act = s_act[myr];
        // phase A: p = r + beta p_old, t = g5Dw p, <p,Ap>
        {
            float f = 0.f;   // per-thread sum in FP32, one conversion per phase
            if (act) {
                const SpAxpy<float, SpF> Q{SpF{P.r32}, SpF{qo}, (float)s_beta[myr], !s_first[myr]};
                FOR_MY_TILES(q) {
                    const Pair<float> c = Q.ld(q.x);
                    const Pair<float> tt = g5dw_at_c<float>(Q, c, Lf, q, m2f);
                    st_f(qn, q.x, c);
                    st_f(P.t32, q.x, tt);
                    f += norm2(tt.a) + norm2(tt.b);
                }
            }
            if (!breduce(gs, (double)f, P, smem, s_tmp)) { ok = false; goto done; }
        }
        for (int r = threadIdx.x; r < B; r += blockDim.x)
            if (s_act[r]) s_alpha[r] = s_rr[r] / s_tmp[r];
        __syncthreads();
        // phase B: x += alpha p, r -= alpha g5Dw t
        {
            float f = 0.f;
            if (act) {
                const float alpha = (float)s_alpha[myr];
                FOR_MY_TILES(q) {
                    const Pair<float> pc = SpF{qn}.ld(q.x);
                    const Pair<float> a = g5dw_at<float>(SpF{P.t32}, Lf, q, m2f);
                    Pair<float> xv = SpF{P.x32}.ld(q.x), r = SpF{P.r32}.ld(q.x);
                    xv.a = xv.a + alpha * pc.a;
                    xv.b = xv.b + alpha * pc.b;
                    r.a = r.a - alpha * a.a;
                    r.b = r.b - alpha * a.b;
                    st_f(P.x32, q.x, xv);
                    st_f(P.r32, q.x, r);
                    f += norm2(r.a) + norm2(r.b);
                }
            }
            if (!breduce(gs, (double)f, P, smem, s_tmp)) { ok = false; goto done; }
        }
        // per-replica reliable-update decisions (identical in every block)
        if (threadIdx.x == 0) {
            int any = 0;
            for (int r = 0; r < B; r++) {
                s_upd[r] = 0;
                if (!s_act[r]) continue;
                const double rn = s_tmp[r];
                s_maxrr[r] = fmax(s_maxrr[r], rn);
                const bool cand = rn < s_tol[r] * s_s[r] * s_s[r];
                if (rn < P.delta2 * s_maxrr[r] || cand || k == P.maxiter) {
                    s_upd[r] = 1;
                    s_nupd[r]++;
                    any = 1;
                } else {
                    s_beta[r] = rn / s_rr[r];
                    s_rr[r] = rn;
                    s_rr64[r] = rn / (s_s[r] * s_s[r]);
                }
                s_first[r] = 0;
            }
            s_any[1] = any;
        }
        __syncthreads();
        if (s_any[1]) {
            const bool upd = s_upd[myr];
            const double inv_s = 1.0 / s_s[myr];
            if (upd) FOR_MY_TILES(q) {   // x += x32 / s
                    const Pair<float> d = SpF{P.x32}.ld(q.x);
                    Pair<double> xv = SpD{P.x, V}.ld(q.x);
                    xv.a = xv.a + inv_s * to_d(d.a);
                    xv.b = xv.b + inv_s * to_d(d.b);
                    st_d(P.x, V, q.x, xv);
                    st_f(P.x32, q.x, Pair<float>{make_float2(0, 0), make_float2(0, 0)});
                }
            if (!gs.sync()) { ok = false; goto done; }
            if (upd) FOR_MY_TILES(q) st_d(P.t64, V, q.x, g5dw_at<double>(SpD{P.x, V}, L, q, m2));
            if (!gs.sync()) { ok = false; goto done; }
            double w = 0.0;
            if (upd) FOR_MY_TILES(q) {   // r64 = b - A x
                    const Pair<double> a = g5dw_at<double>(SpD{P.t64, V}, L, q, m2);
                    Pair<double> r;
                    r.a = __ldg(P.b + q.x) - a.a;
                    r.b = __ldg(P.b + q.x + V) - a.b;
                    st_d(P.r64, V, q.x, r);
                    w += norm2(r.a) + norm2(r.b);
                }
            if (!breduce(gs, w, P, smem, s_tmp)) { ok = false; goto done; }
            if (threadIdx.x == 0) {
                int any = 0;
                for (int r = 0; r < B; r++) {
                    s_r4[r] = 0;
                    if (!s_upd[r]) continue;
                    const double rrt = s_tmp[r];
                    s_rr64[r] = rrt;
                    if (rrt < s_tol[r]) {
                        s_act[r] = 0;
                        s_conv[r] = 1;
                        s_it[r] = k;
                    } else if (k == P.maxiter) {
                        s_act[r] = 0;
                        s_it[r] = k;
                    } else {
                        s_r4[r] = 1;
                        s_snew[r] = 1.0 / sqrt(rrt);
                        any = 1;
                    }
                }
                s_any[1] = any;
            }
            __syncthreads();
            if (s_any[1]) {
                double v = 0.0;
                if (s_r4[myr]) {
                    const double sn = s_snew[myr];
                    FOR_MY_TILES(q) {   // r32 = s_new r64
                        const Pair<float> r32{to_f(sn * P.r64[q.x]), to_f(sn * P.r64[q.x + V])};
                        st_f(P.r32, q.x, r32);
                        v += (double)(norm2(r32.a) + norm2(r32.b));
                    }
                }
                if (!breduce(gs, v, P, smem, s_tmp)) { ok = false; goto done; }
                for (int r = threadIdx.x; r < B; r += blockDim.x)
                    if (s_r4[r]) {
                        const double s = s_s[r], sn = s_snew[r];
                        s_beta[r] = (s_rr64[r] * s * s / s_rr[r]) * (sn / s);
                        s_s[r] = sn;
                        s_rr[r] = s_tmp[r];
                        s_maxrr[r] = s_tmp[r];
                    }
                __syncthreads();
            }
        }
        cur ^= 1;
    }
done:
    if (blockIdx.x == 0) {
        DevCtl* c = P.ctl;
        for (int r = threadIdx.x; r < B; r += blockDim.x) {
            P.out_iters[r] = s_conv[r] ? s_it[r] : (s_it[r] ? s_it[r] : P.maxiter);
            P.out_conv[r] = ok && s_conv[r];
            P.out_upd[r] = s_nupd[r];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const int err = ld_volatile_int(&c->err);
            int all = ok;
            long long tot = 0;
            for (int r = 0; r < B; r++) {
                all &= s_conv[r];
                tot += P.out_iters[r];
            }
            c->last_iters = k;
            c->iters_total += tot;
            if (c->status == 0) {
                if (err || !ok) c->status = QED2D_ERR_TIMEOUT;
                else if (!all) c->status = QED2D_ERR_NOT_CONVERGED;
            }
        }
    }
}

}  // namespace qed2d

// ===========================================================================
// host side
using namespace qed2d;

struct qed2d_batch {
    BLat g;
    int device = 0, num_sms = 148;
    cudaStream_t stream = nullptr;
    std::vector<double> beta;
    std::vector<double> m2;     // 2 + m0 per replica, set by each trajectory
    DevCtl* ctl = nullptr;
    DevCtl* ctl_host = nullptr;
    double* part = nullptr;
    double* dscal = nullptr;    // [kMaxBatch*5 * 2] per-replica sums (start, end)
    double* dpar = nullptr;     // [kMaxBatch * 2]: m2 (2+m0), beta
    uint64_t* dseed = nullptr;  // [kMaxBatch]
    int* dint = nullptr;        // [kMaxBatch * 3]: iterations, converged, reliable updates of the last solve
    long long* diters = nullptr;   // [kMaxBatch] accumulated iterations
    std::map<std::string, std::pair<void*, size_t>> ws;
    void* buf(const std::string& name, size_t bytes) {
        auto it = ws.find(name);
        if (it != ws.end() && it->second.second >= bytes) return it->second.first;
        if (it != ws.end()) {
            cudaFree(it->second.first);
            ws.erase(it);
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
    double2* field(const char* n) { return (double2*)buf(n, sizeof(double2) * 2 * g.V); }
    double* real2(const char* n) { return (double*)buf(n, sizeof(double) * 2 * g.V); }
    float4* field32(const char* n) { return (float4*)buf(n, sizeof(float4) * g.V); }
};

namespace {

int b_post(const char* name) {
    count_launch();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QED2D_OK : cuda_status(e, name);
}

dim3 b_tiles(const qed2d_batch* h) { return dim3((unsigned)h->g.ntr, (unsigned)h->g.B); }

// accumulate this solve's per-replica iterations
__global__ void k_b_acc_iters(long long* acc, const int* it, int B) {
    const int r = threadIdx.x;
    if (r < B) acc[r] += it[r];
}

int b_solve(qed2d_batch* h, const double2* U, const float4* U32, const double2* b, double2* x, double2* g5x,
            int maxiter, double eps) {
    BCGP P{};
    P.g = h->g;
    P.U = U;
    P.U32 = U32;
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
    for (int r = 0; r < h->g.B; r++) P.m2[r] = h->m2[r];
    P.eps = eps;
    P.delta2 = 0.05 * 0.05;
    P.maxiter = maxiter;
    P.ctl = h->ctl;
    P.part = h->part;
    P.out_iters = h->dint;
    P.out_conv = h->dint + kMaxBatch;
    P.out_upd = h->dint + 2 * kMaxBatch;
    int per_sm = 0;
    QCHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_b_cg_mixed, TILE, 0));
    if (per_sm < 1) return QED2D_ERR_UNSUPPORTED;
    long long maxg = (long long)per_sm * h->num_sms;
    if (maxg > kMaxPartBlocks) maxg = kMaxPartBlocks;
    long long bpr = maxg / h->g.B;
    if (bpr < 1) return QED2D_ERR_UNSUPPORTED;
    const long long per_block = (h->g.ntr + bpr - 1) / bpr;
    bpr = (h->g.ntr + per_block - 1) / per_block;
    P.bpr = (int)bpr;
    P.per_block = (int)per_block;
    QCHECK(cudaMemsetAsync(&h->ctl->bar, 0, 2 * sizeof(unsigned long long) + sizeof(int), h->stream));
    void* args[] = {(void*)&P};
    QCHECK(cudaLaunchCooperativeKernel((const void*)k_b_cg_mixed, dim3((unsigned)(bpr * h->g.B)), dim3(TILE), args, 0,
                                       h->stream));
    count_launch();
    k_b_acc_iters<<<1, kMaxBatch, 0, h->stream>>>(h->diters, h->dint, h->g.B);
    return b_post("k_b_acc_iters");
}

int b_reduce(qed2d_batch* h, const double2* U, const double* mom, const double2* X, const double2* F, int slot) {
    long long nb = (h->g.Vr + RBB - 1) / RBB;
    const long long cap = (long long)(kMaxPartVals * kMaxPartBlocks) / (5LL * h->g.B);
    if (nb > 64) nb = 64;
    if (nb > cap) nb = cap;
    k_b_reduce<<<dim3((unsigned)nb, (unsigned)h->g.B), RBB, 0, h->stream>>>(U, mom, X, F, h->g, h->part,
                                                                             h->dscal + slot * kMaxBatch * 5);
    QTRY(b_post("k_b_reduce"));
    k_b_reduce_final<<<1, 256, 0, h->stream>>>(h->part, (int)nb, h->g.B, h->dscal + slot * kMaxBatch * 5);
    return b_post("k_b_reduce_final");
}

int b_fill(qed2d_batch* h, double* out, int dbl_per_elem, uint32_t stream, uint32_t counter, double scale) {
    const long long pairs = h->g.Vr * dbl_per_elem;   // 2 Vr dbl_per_elem doubles per replica
    k_b_random_normal<<<dim3((unsigned)((pairs + 255) / 256), (unsigned)h->g.B), 256, 0, h->stream>>>(
        out, h->g, dbl_per_elem, h->dseed, stream, counter, scale);
    return b_post("k_b_random_normal");
}

int b_kick(qed2d_batch* h, double* mom, const double2* U, const float4* U32, double2* X, const double2* F,
           double2* G, double eps, int maxiter, double tol) {
    QTRY(b_solve(h, U, U32, F, X, G, maxiter, tol));
    k_b_mom_kick<<<b_tiles(h), TILE, 0, h->stream>>>(mom, U, h->g, h->dpar + kMaxBatch, eps, X, G);
    return b_post("k_b_mom_kick");
}

}  // namespace

extern "C" {

int qed2d_batch_create(int nrep, int L1, int L2, const double* beta, qed2d_batch** out) {
    if (!out) return QED2D_ERR_BAD_ARG;
    *out = nullptr;
    if (nrep < 1 || nrep > kMaxBatch || L1 < 2 || L2 < 2 || !beta ||
        (long long)nrep * L1 * L2 > (1LL << 30)) {
        set_error("qed2d_batch_create: need 1 <= nrep <= 64, L1, L2 >= 2, nrep*L1*L2 <= 2^30 and a beta per replica");
        return QED2D_ERR_BAD_ARG;
    }
    auto* h = new qed2d_batch();
    h->g = make_blat(nrep, L1, L2);
    h->beta.assign(beta, beta + nrep);
    cudaError_t e = cudaGetDevice(&h->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
    if (e == cudaSuccess) e = cudaMalloc(&h->ctl, sizeof(DevCtl));
    if (e == cudaSuccess) e = cudaMallocHost(&h->ctl_host, sizeof(DevCtl));
    if (e == cudaSuccess) e = cudaMalloc(&h->part, sizeof(double) * kMaxPartVals * kMaxPartBlocks);
    if (e == cudaSuccess) e = cudaMalloc(&h->dscal, sizeof(double) * kMaxBatch * 5 * 2);
    if (e == cudaSuccess) e = cudaMalloc(&h->dpar, sizeof(double) * kMaxBatch * 2);
    if (e == cudaSuccess) e = cudaMalloc(&h->dseed, sizeof(uint64_t) * kMaxBatch);
    if (e == cudaSuccess) e = cudaMalloc(&h->dint, sizeof(int) * kMaxBatch * 3);
    if (e == cudaSuccess) e = cudaMalloc(&h->diters, sizeof(long long) * kMaxBatch);
    if (e == cudaSuccess) e = cudaMemset(h->ctl, 0, sizeof(DevCtl));
    if (e == cudaSuccess) e = cudaMemcpy(h->dpar + kMaxBatch, beta, sizeof(double) * nrep, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        const int st = cuda_status(e, "qed2d_batch_create");
        qed2d_batch_destroy(h);
        return st;
    }
    *out = h;
    return QED2D_OK;
}

int qed2d_batch_destroy(qed2d_batch* h) {
    if (!h) return QED2D_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    else cudaDeviceSynchronize();
    for (auto& kv : h->ws) cudaFree(kv.second.first);
    cudaFree(h->ctl);
    cudaFreeHost(h->ctl_host);
    cudaFree(h->part);
    cudaFree(h->dscal);
    cudaFree(h->dpar);
    cudaFree(h->dseed);
    cudaFree(h->dint);
    cudaFree(h->diters);
    delete h;
    return QED2D_OK;
}

int qed2d_batch_set_stream(qed2d_batch* h, void* stream) {
    if (!h) return QED2D_ERR_BAD_ARG;
    h->stream = (cudaStream_t)stream;
    return QED2D_OK;
}

int qed2d_batch_cg(qed2d_batch* h, double* x, const double* U, const double* b, const double* am0, int maxiter,
                   double eps, int* iterations, int* updates) {
    if (!h || !x || !U || !b || !am0 || maxiter < 0 ||
        ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(U) | reinterpret_cast<uintptr_t>(b)) % 16)) {
        set_error("qed2d_batch_cg: bad argument");
        return QED2D_ERR_BAD_ARG;
    }
    const int B = h->g.B;
    const size_t fb = sizeof(double2) * 2 * (size_t)h->g.V;
    if ((const char*)x < (const char*)b + fb && (const char*)b < (const char*)x + fb) {
        set_error("qed2d_batch_cg: x aliases b");
        return QED2D_ERR_BAD_ARG;
    }
    cudaStream_t s = h->stream;
    float4* U32 = h->field32("b_U32");
    double2* G = h->field("b_G");
    if (!U32 || !G) return QED2D_ERR_NO_MEMORY;
    h->m2.assign(B, 0.0);
    for (int r = 0; r < B; r++) h->m2[r] = 2.0 + am0[r];
    QCHECK(cudaMemsetAsync(&h->ctl->status, 0, sizeof(int), s));
    QCHECK(cudaMemsetAsync(h->diters, 0, sizeof(long long) * B, s));
    Ctx tmp;
    tmp.g.L1 = h->g.L1;
    tmp.g.L2 = h->g.L2r * B;
    tmp.g.V = h->g.V;
    tmp.stream = s;
    QTRY(launch_pack_links(tmp, U32, (const double2*)U));
    QTRY(b_solve(h, (const double2*)U, U32, (const double2*)b, (double2*)x, G, maxiter, eps));
    int hi[3 * kMaxBatch];
    QCHECK(cudaMemcpyAsync(hi, h->dint, sizeof(hi), cudaMemcpyDeviceToHost, s));
    QCHECK(cudaMemcpyAsync(h->ctl_host, h->ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, s));
    QCHECK(cudaStreamSynchronize(s));
    for (int r = 0; r < B; r++) {
        if (iterations) iterations[r] = hi[r];
        if (updates) updates[r] = hi[2 * kMaxBatch + r];
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
    const int B = h->g.B;
    const long long V = h->g.V, Vr = h->g.Vr;
    double2* U = (double2*)Ud;
    double2* Ucp = h->field("b_Ucp");
    double* mom = h->real2("b_mom");
    double2* X = h->field("b_X");
    double2* F = h->field("b_F");
    double2* G = h->field("b_G");
    float4* U32 = h->field32("b_U32");
    if (!Ucp || !mom || !X || !F || !G || !U32) return QED2D_ERR_NO_MEMORY;
    cudaStream_t s = h->stream;
    // per-replica parameters
    h->m2.assign(B, 0.0);
    for (int r = 0; r < B; r++) h->m2[r] = 2.0 + am0[r];
    QCHECK(cudaMemcpyAsync(h->dpar, h->m2.data(), sizeof(double) * B, cudaMemcpyHostToDevice, s));
    QCHECK(cudaMemcpyAsync(h->dseed, seeds, sizeof(uint64_t) * B, cudaMemcpyHostToDevice, s));
    QCHECK(cudaMemsetAsync(h->diters, 0, sizeof(long long) * B, s));
    QCHECK(cudaMemsetAsync(&h->ctl->status, 0, sizeof(int), s));
    QCHECK(cudaMemcpyAsync(Ucp, U, sizeof(double2) * 2 * V, cudaMemcpyDeviceToDevice, s));
    // draws (src/QED2dHMC.jl:69-70), H_ini, F = g5Dw X (:74-78)
    QTRY(b_fill(h, mom, 1, QED2D_STREAM_MOMENTA, counter, 1.0));
    QTRY(b_fill(h, (double*)X, 2, QED2D_STREAM_NOISE, counter, 1.0 / std::sqrt(2.0)));
    QTRY(b_reduce(h, U, mom, X, nullptr, 0));
    k_b_g5dw<<<b_tiles(h), TILE, 0, s>>>(F, U, X, h->g, h->dpar);
    QTRY(b_post("k_b_g5dw"));
    {
        Ctx tmp;
        tmp.g.L1 = h->g.L1;
        tmp.g.L2 = h->g.L2r * B;
        tmp.g.V = V;
        tmp.stream = s;
        QTRY(launch_pack_links(tmp, U32, U));
        // leapfrog (src/QED2dHMC.jl:426-449)
        QTRY(b_kick(h, mom, U, U32, X, F, G, 0.5 * eps, maxiter, tol));
        for (int i = 0; i < ns - 1; i++) {
            QTRY(launch_updt_fld(tmp, U, mom, eps, U32));
            QTRY(b_kick(h, mom, U, U32, X, F, G, eps, maxiter, tol));
        }
        QTRY(launch_updt_fld(tmp, U, mom, eps, U32));
        QTRY(b_kick(h, mom, U, U32, X, F, G, 0.5 * eps, maxiter, tol));
    }
    // H_fin with <X, F> (:82)
    QTRY(b_reduce(h, U, mom, X, F, 1));
    double sc[2][kMaxBatch * 5];
    long long its[kMaxBatch];
    QCHECK(cudaMemcpyAsync(sc, h->dscal, sizeof(sc), cudaMemcpyDeviceToHost, s));
    QCHECK(cudaMemcpyAsync(its, h->diters, sizeof(long long) * B, cudaMemcpyDeviceToHost, s));
    QCHECK(cudaMemcpyAsync(h->ctl_host, h->ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, s));
    QCHECK(cudaStreamSynchronize(s));
    const int st = h->ctl_host->status;
    for (int r = 0; r < B; r++) {
        const double* a = &sc[0][r * 5];
        const double* f = &sc[1][r * 5];
        const double beta = h->beta[r];
        const double hini = a[2] / 2.0 + beta * ((double)Vr - a[0]) + a[3];
        const double hfin = f[2] / 2.0 + beta * ((double)Vr - f[0]) + f[4];
        const double qf = f[1] / (2.0 * M_PI);
        double pacc = (qzero && std::fabs(qf) > 0.1) ? 0.0 : std::exp(-(hfin - hini));
        int acc = 1;
        if (st != QED2D_OK) acc = 0;
        else if (pacc < 1.0) acc = pacc > qed2d_random_uniform(seeds[r], QED2D_STREAM_METROPOLIS, counter);
        if (!acc)   // restore the replica's two planes
            for (int k2 = 0; k2 < 2; k2++)
                QCHECK(cudaMemcpyAsync(U + (k2 * B + r) * Vr, Ucp + (k2 * B + r) * Vr, sizeof(double2) * Vr,
                                       cudaMemcpyDeviceToDevice, s));
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
