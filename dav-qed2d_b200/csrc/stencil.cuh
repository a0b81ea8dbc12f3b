// stencil.cuh -- lattice geometry, field accessors and the stencil/force
// evaluators used by both the standalone kernels and the persistent solvers.
//
// Sites are visited in tiles of TX x TY = 32 x 8 (i1 fastest): a warp covers 32
// consecutive i1 of one row, so every plane load of a warp is one contiguous
// 512-byte segment, and the rows i2 +- 1 of a tile are read by the same block.
#pragma once

#include "device.cuh"
#include "internal.h"

namespace qed2d {

constexpr int TX = 32;
constexpr int TY = 8;
constexpr int TILE = TX * TY;

struct Site {
    int i1, i2;
    long long x, xp1, xm1, xp2, xm2;
    bool ok;
};

// neighbours with periodic wrap (src/QED2dDirac.jl:7-11)
__device__ __forceinline__ Site site_of_tile(const Lat& g, long long tile, int t) {
    const int nt1 = (g.L1 + TX - 1) / TX;
    const long long t2 = tile / nt1;
    const int t1 = (int)(tile - t2 * nt1);
    Site s;
    s.i1 = t1 * TX + (t & (TX - 1));
    s.i2 = (int)t2 * TY + (t >> 5);
    s.ok = s.i1 < g.L1 && s.i2 < g.L2;
    s.x = s.i1 + (long long)g.L1 * s.i2;
    s.xp1 = (s.i1 + 1 == g.L1) ? s.x - (g.L1 - 1) : s.x + 1;
    s.xm1 = (s.i1 == 0) ? s.x + (g.L1 - 1) : s.x - 1;
    s.xp2 = (s.i2 + 1 == g.L2) ? (long long)s.i1 : s.x + g.L1;
    s.xm2 = (s.i2 == 0) ? s.x + (g.V - g.L1) : s.x - g.L1;
    return s;
}

__host__ __device__ __forceinline__ long long num_tiles(const Lat& g) {
    return (long long)((g.L1 + TX - 1) / TX) * ((g.L2 + TY - 1) / TY);
}

// site of thread t in tile (t1, t2) of 32 x TYv sites -- no division; the
// persistent solvers walk a block's contiguous tile range and advance (t1, t2)
// incrementally
template <int TYv>
__device__ __forceinline__ Site site_at_t(const Lat& g, int t1, int t2, int t) {
    Site s;
    s.i1 = t1 * TX + (t & (TX - 1));
    s.i2 = t2 * TYv + (t >> 5);
    s.ok = s.i1 < g.L1 && s.i2 < g.L2;
    s.x = s.i1 + g.L1 * s.i2;   // 32-bit arithmetic: 2*V < 2^31 is checked at context creation
    s.xp1 = (s.i1 + 1 == g.L1) ? s.x - (g.L1 - 1) : s.x + 1;
    s.xm1 = (s.i1 == 0) ? s.x + (g.L1 - 1) : s.x - 1;
    s.xp2 = (s.i2 + 1 == g.L2) ? (long long)s.i1 : s.x + g.L1;
    s.xm2 = (s.i2 == 0) ? s.x + (g.V - g.L1) : s.x - g.L1;
    return s;
}
__device__ __forceinline__ Site site_at(const Lat& g, int t1, int t2, int t) {
    Site s;
    s.i1 = t1 * TX + (t & (TX - 1));
    s.i2 = t2 * TY + (t >> 5);
    s.ok = s.i1 < g.L1 && s.i2 < g.L2;
    s.x = s.i1 + g.L1 * s.i2;   // 32-bit arithmetic: 2*V < 2^31 is checked at context creation
    s.xp1 = (s.i1 + 1 == g.L1) ? s.x - (g.L1 - 1) : s.x + 1;
    s.xm1 = (s.i1 == 0) ? s.x + (g.L1 - 1) : s.x - 1;
    s.xp2 = (s.i2 + 1 == g.L2) ? (long long)s.i1 : s.x + g.L1;
    s.xm2 = (s.i2 == 0) ? s.x + (g.V - g.L1) : s.x - g.L1;
    return s;
}

// the block's contiguous tile range [lo, hi) and the coordinates of tile lo
struct TileRange {
    int lo, hi, s1, s2, nt1;
};
__device__ __forceinline__ TileRange tile_range(long long ntiles, int nt1, int per_block, int b) {
    TileRange r;
    r.lo = b * per_block;
    r.hi = (int)min((long long)r.lo + per_block, ntiles);
    r.s2 = r.lo / nt1;
    r.s1 = r.lo - r.s2 * nt1;
    r.nt1 = nt1;
    return r;
}
#define FOR_RANGE(q, G, R)                                                                                    \
    for (int tt_ = (R).lo, t1_ = (R).s1, t2_ = (R).s2; tt_ < (R).hi;                                        \
         ++tt_, (++t1_ == (R).nt1 ? (t1_ = 0, ++t2_) : 0))                                                    \
        if (const Site q = site_at((G), t1_, t2_, threadIdx.x); q.ok)

// the same for a BX x BY tile visited by BX*BY threads (thread t -> (t % BX, t / BX))
template <int BX, int BY>
__device__ __forceinline__ Site site_of_tile_t(const Lat& g, long long tile, int t) {
    const int nt1 = (g.L1 + BX - 1) / BX;
    const long long t2 = tile / nt1;
    const int t1 = (int)(tile - t2 * nt1);
    Site s;
    s.i1 = t1 * BX + (t % BX);
    s.i2 = (int)t2 * BY + (t / BX);
    s.ok = s.i1 < g.L1 && s.i2 < g.L2;
    s.x = s.i1 + (long long)g.L1 * s.i2;
    s.xp1 = (s.i1 + 1 == g.L1) ? s.x - (g.L1 - 1) : s.x + 1;
    s.xm1 = (s.i1 == 0) ? s.x + (g.L1 - 1) : s.x - 1;
    s.xp2 = (s.i2 + 1 == g.L2) ? (long long)s.i1 : s.x + g.L1;
    s.xm2 = (s.i2 == 0) ? s.x + (g.V - g.L1) : s.x - g.L1;
    return s;
}
template <int BX, int BY>
__host__ __device__ __forceinline__ long long num_tiles_t(const Lat& g) {
    return (long long)((g.L1 + BX - 1) / BX) * ((g.L2 + BY - 1) / BY);
}

// ---------------------------------------------------------------------------
// spinor accessors
struct SpD {   // FP64 planes (reference layout): spin k of site x at p[x + k V]
    const double2* p;
    long long V;
    __device__ __forceinline__ Pair<double> ld(long long x) const { return {p[x], p[x + V]}; }
};
struct SpDro {   // read-only for the kernel's lifetime: non-coherent path
    const double2* p;
    long long V;
    __device__ __forceinline__ Pair<double> ld(long long x) const { return {__ldg(p + x), __ldg(p + x + V)}; }
};
__device__ __forceinline__ void st_d(double2* p, long long V, long long x, const Pair<double>& v) {
    p[x] = v.a;
    p[x + V] = v.b;
}
struct SpF {   // FP32 packed: (s1, s2) of site x in one float4
    const float4* p;
    __device__ __forceinline__ Pair<float> ld(long long x) const {
        const float4 q = p[x];
        return {make_float2(q.x, q.y), make_float2(q.z, q.w)};
    }
};
__device__ __forceinline__ void st_f(float4* p, long long x, const Pair<float>& v) {
    p[x] = make_float4(v.a.x, v.a.y, v.b.x, v.b.y);
}
// q = r + beta p, evaluated on load (p skipped when beta == 0)
template <typename R, class A>
struct SpAxpy {
    A r, p;
    R beta;
    bool use_p;
    __device__ __forceinline__ Pair<R> ld(long long x) const {
        Pair<R> v = r.ld(x);
        if (use_p) {
            const Pair<R> w = p.ld(x);
            v.a = v.a + beta * w.a;
            v.b = v.b + beta * w.b;
        }
        return v;
    }
};

struct SpF2 {   // complex64 planes (reference layout in single precision): p[x + k V]
    const float2* p;
    long long V;
    __device__ __forceinline__ Pair<float> ld(long long x) const { return {__ldg(p + x), __ldg(p + x + V)}; }
};

// link accessors
struct LkD {
    const double2* U;
    long long V;
    __device__ __forceinline__ double2 u1(long long x) const { return __ldg(U + x); }
    __device__ __forceinline__ double2 u2(long long x) const { return __ldg(U + V + x); }
};
// packed FP32 links of the mixed solvers: two float2 planes (u1, u2) of
// `stride` sites each, stored in a float4 array of `stride` elements; a link
// load reads only the direction it needs (8 bytes, not the site's 16)
struct LkF {
    const float2* U;
    long long stride;
    __device__ __forceinline__ LkF(const float4* base, long long stride_, long long off = 0)
        : U(reinterpret_cast<const float2*>(base) + off), stride(stride_) {}
    __device__ __forceinline__ float2 u1(long long x) const { return __ldg(U + x); }
    __device__ __forceinline__ float2 u2(long long x) const { return __ldg(U + stride + x); }
};
// store the FP32 links of site x into the planes of `stride` sites
__device__ __forceinline__ void st_links32(float4* base, long long stride, long long x, double2 u1, double2 u2) {
    float2* u = reinterpret_cast<float2*>(base);
    u[x] = make_float2((float)u1.x, (float)u1.y);
    u[stride + x] = make_float2((float)u2.x, (float)u2.y);
}

struct LkF2 {   // complex64 link planes
    const float2* U;
    long long V;
    __device__ __forceinline__ float2 u1(long long x) const { return __ldg(U + x); }
    __device__ __forceinline__ float2 u2(long long x) const { return __ldg(U + V + x); }
};

// gamma5 Dw applied at one site
template <typename R, class S, class L>
__device__ __forceinline__ Pair<R> g5dw_at(const S& s, const L& U, const Site& q, R m2) {
    const Pair<R> c = s.ld(q.x), p1 = s.ld(q.xp1), m1 = s.ld(q.xm1), p2 = s.ld(q.xp2), mm2 = s.ld(q.xm2);
    Pair<R> o;
    g5dw_site<R>(c.a, c.b, p1.a, p1.b, m1.a, m1.b, p2.a, p2.b, mm2.a, mm2.b, U.u1(q.x), U.u2(q.x), U.u1(q.xm1),
                 U.u2(q.xm2), m2, o.a, o.b);
    return o;
}

// gamma5 Dw at one site with the centre value already known (saves a load)
template <typename R, class S, class L>
__device__ __forceinline__ Pair<R> g5dw_at_c(const S& s, const Pair<R>& c, const L& U, const Site& q, R m2) {
    const Pair<R> p1 = s.ld(q.xp1), m1 = s.ld(q.xm1), p2 = s.ld(q.xp2), mm2 = s.ld(q.xm2);
    Pair<R> o;
    g5dw_site<R>(c.a, c.b, p1.a, p1.b, m1.a, m1.b, p2.a, p2.b, mm2.a, mm2.b, U.u1(q.x), U.u2(q.x), U.u1(q.xm1),
                 U.u2(q.xm2), m2, o.a, o.b);
    return o;
}

// gamma5 Dw at one site with the centre value and the four links given
template <typename R, class S, typename LT>
__device__ __forceinline__ Pair<R> g5dw_at_cl(const S& s, const Pair<R>& c, const Site& q, LT u1x, LT u2x, LT u1m1,
                                              LT u2m2, R m2) {
    const Pair<R> p1 = s.ld(q.xp1), m1 = s.ld(q.xm1), p2 = s.ld(q.xp2), mm2 = s.ld(q.xm2);
    Pair<R> o;
    g5dw_site<R>(c.a, c.b, p1.a, p1.b, m1.a, m1.b, p2.a, p2.b, mm2.a, mm2.b, u1x, u2x, u1m1, u2m2, m2, o.a, o.b);
    return o;
}

// FP32 links of a block's tiles staged in shared memory for the length of a
// solve (they do not change during one): per tile of 32 x TYv sites a box of u1
// over the tile's rows and the column left of it (TYv x 33) and a box of u2 over
// the tile's columns and the row below it ((TYv + 1) x 32), so a site reads
// u1(x), u1(x - 1), u2(x) and u2(x - 2) without a branch.  j is the tile's index
// in the block's range; thread t of the tile is site (t % 32, t / 32).
template <int TYv>
struct ULsm {
    static constexpr int B1 = TYv * 33, TS = TYv * 33 + (TYv + 1) * 32;   // float2 per tile
    static __host__ __device__ constexpr size_t bytes(int per_block) { return sizeof(float2) * TS * (size_t)per_block; }
    static __device__ __forceinline__ void stage(float2* s, int j, const LkF& Lf, const Site& q) {
        const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
        float2* b1 = s + j * TS + ly * 33 + lx;
        float2* b2 = s + j * TS + B1 + ly * 32 + lx;
        b1[1] = Lf.u1(q.x);
        b2[32] = Lf.u2(q.x);
        if (lx == 0) b1[0] = Lf.u1(q.xm1);
        if (ly == 0) b2[0] = Lf.u2(q.xm2);
    }
    template <class S>
    static __device__ __forceinline__ Pair<float> stencil(const float2* s, int j, const S& sp, const Pair<float>& c,
                                                          const Site& q, float m2) {
        const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
        const float2* b1 = s + j * TS + ly * 33 + lx;
        const float2* b2 = s + j * TS + B1 + ly * 32 + lx;
        return g5dw_at_cl<float>(sp, c, q, b1[1], b2[32], b1[0], b2[0], m2);
    }
};

// total gauge force on the two links of site y: frc1+frc2 of krnl_force!
//   F1(y) = -v(y) + v(y-2),  F2(y) = v(y) - v(y-1)
// The three plaquettes share links: the 10 distinct links are addressed from
// the site's neighbour indices and all loaded before any arithmetic, so a
// thread waits for memory once (the diagonal neighbours y-1+2 and y+1-2 are
// the row neighbours shifted by the same i1 offset).
__device__ __forceinline__ void gauge_force_at(const double2* U, const Lat& g, const Site& q, double beta,
                                               double& F1, double& F2) {
    const long long V = g.V;
    const long long xm1p2 = q.xp2 + (q.xm1 - q.x), xp1m2 = q.xm2 + (q.xp1 - q.x);
    const double2 u1x = __ldg(U + q.x), u2x = __ldg(U + V + q.x);
    const double2 u2xp1 = __ldg(U + V + q.xp1), u1xp2 = __ldg(U + q.xp2);
    const double2 u1xm2 = __ldg(U + q.xm2), u2xm2 = __ldg(U + V + q.xm2), u2xp1m2 = __ldg(U + V + xp1m2);
    const double2 u1xm1 = __ldg(U + q.xm1), u2xm1 = __ldg(U + V + q.xm1), u1xm1p2 = __ldg(U + xm1p2);
    const double v = beta * plaquette_of(u1x, u2xp1, u1xp2, u2x).y;
    const double vm2 = beta * plaquette_of(u1xm2, u2xp1m2, u1x, u2xm2).y;
    const double vm1 = beta * plaquette_of(u1xm1, u2x, u1xm1p2, u2xm1).y;
    F1 = -v + vm2;
    F2 = v - vm1;
}

// fermion force at one site from (X, G) planes
__device__ __forceinline__ void fermion_force_at(const double2* U, const double2* X, const double2* G,
                                                 long long V, const Site& q, double& f1, double& f2) {
    force_site<double>(__ldg(U + q.x), __ldg(U + V + q.x), X[q.x], X[q.x + V], G[q.x], G[q.x + V], X[q.xp1],
                       X[q.xp1 + V], G[q.xp1], G[q.xp1 + V], X[q.xp2], X[q.xp2 + V], G[q.xp2], G[q.xp2 + V], f1,
                       f2);
}

}  // namespace qed2d
