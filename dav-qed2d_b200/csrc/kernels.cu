// kernels.cu -- standalone (one tile per block) kernels of libqed2d and their
// launchers: the reference's device kernels (gamm5Dw, gamm5, tr_dQwdU,
// plaquette!, qtop!, krnl_force!, updt_fld!, unfold, plwv), the fused momentum
// kick, random fields, BLAS-1 and deterministic single-launch reductions.
#include <atomic>

#include "stencil.cuh"

namespace qed2d {

static std::atomic<int64_t> g_launches{0};
void count_launch(int n) { g_launches += n; }
int64_t launches() { return g_launches.load(); }

static inline unsigned tiles_grid(const Lat& g) { return (unsigned)num_tiles(g); }

// Tile kernels run on a 2D grid of tiles (x along i1, y along i2), so a thread
// finds its site without an index division; lattices taller than 65535 tiles
// fall back to a 1D grid.
static inline dim3 tiles_grid2(const Lat& g) {
    const unsigned nt1 = (unsigned)((g.L1 + TX - 1) / TX), nt2 = (unsigned)((g.L2 + TY - 1) / TY);
    return nt2 <= 65535 ? dim3(nt1, nt2) : dim3(tiles_grid(g));
}
__device__ __forceinline__ Site tile_site(const Lat& g) {
    return gridDim.y > 1 || g.L2 <= TY ? site_at(g, blockIdx.x, blockIdx.y, threadIdx.x)
                                       : site_of_tile(g, blockIdx.x, threadIdx.x);
}

// ---------------------------------------------------------------------------
// gamm5Dw (src/QED2dDirac.jl:2-33); optionally  so += addc * addv  with complex
// addc (the mu^2 si term of gamm5Dw_sqr_musq, :92, and the +-i mu terms of
// generate_pseudofermion!, src/QED2dRHMC.jl:308,317) and optionally so2 *= -1
// (Dw = g5 (g5 Dw), :157-169)
__global__ void __launch_bounds__(TILE) k_g5dw(double2* __restrict__ so, const double2* __restrict__ U,
                                               const double2* __restrict__ si, double m2, Lat g,
                                               const double2* __restrict__ addv, double2 addc, int g5_out) {
    const Site q = tile_site(g);
    if (!q.ok) return;
    Pair<double> o = g5dw_at<double>(SpDro{si, g.V}, LkD{U, g.V}, q, m2);
    if (addv) {
        o.a = o.a + cmul(addc, __ldg(addv + q.x));
        o.b = o.b + cmul(addc, __ldg(addv + q.x + g.V));
    }
    if (g5_out) o.b = -o.b;
    st_d(so, g.V, q.x, o);
}

// gamm5Dw on complex64 fields in the reference layout: the FP32 arithmetic of
// the mixed solver's inner iterations on complex64 spinors and links
__global__ void __launch_bounds__(TILE) k_g5dw_c64(float2* __restrict__ so, const float2* __restrict__ U,
                                                   const float2* __restrict__ si, float m2, Lat g) {
    const Site q = tile_site(g);
    if (!q.ok) return;
    const Pair<float> o = g5dw_at<float>(SpF2{si, g.V}, LkF2{U, g.V}, q, m2);
    so[q.x] = o.a;
    so[q.x + g.V] = o.b;
}

// gamm5 (src/QED2dDirac.jl:130-146)
__global__ void k_g5(double2* __restrict__ so, const double2* __restrict__ si, long long V) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= V) return;
    so[x] = si[x];
    so[x + V] = -si[x + V];
}

// tr_dQwdU (src/QED2dDirac.jl:172-199); frc = [accumulate ? frc : 0] + rho * force
__global__ void __launch_bounds__(TILE) k_force(double* __restrict__ frc, const double2* __restrict__ U,
                                                const double2* __restrict__ X, const double2* __restrict__ G,
                                                Lat g, double rho, int accumulate) {
    const Site q = tile_site(g);
    if (!q.ok) return;
    double f1, f2;
    fermion_force_at(U, X, G, g.V, q, f1, f2);
    if (accumulate) {
        frc[q.x] += rho * f1;
        frc[q.x + g.V] += rho * f2;
    } else {
        frc[q.x] = rho * f1;
        frc[q.x + g.V] = rho * f2;
    }
}

// The RHMC force of all poles of a flavour in two launches instead of two per
// pole (src/QED2dHMC.jl:528-545): k_g5dw_poles applies gamm5Dw to every pole's
// solution (blockIdx.z = pole), k_force_poles sums rho_i tr_dQwdU(X_i, g5Dw X_i)
// over the poles in pole order, each term as k_force computes it (the same bits
// as one k_force launch per pole).
struct Poles {
    const double2* X[QED2D_MAXPOLES];
    double2* G[QED2D_MAXPOLES];
    double rho[QED2D_MAXPOLES];
    int n;
};
__global__ void __launch_bounds__(TILE) k_g5dw_poles(const double2* __restrict__ U, const Poles P, double m2, Lat g) {
    const Site q = tile_site(g);
    if (!q.ok) return;
    const int i = blockIdx.z;
    st_d(P.G[i], g.V, q.x, g5dw_at<double>(SpDro{P.X[i], g.V}, LkD{U, g.V}, q, m2));
}
__global__ void __launch_bounds__(TILE) k_force_poles(double* __restrict__ frc, const double2* __restrict__ U,
                                                      const Poles P, Lat g, int accumulate) {
    const Site q = tile_site(g);
    if (!q.ok) return;
    double a1 = 0.0, a2 = 0.0;
    for (int i = 0; i < P.n; i++) {
        double f1, f2;
        fermion_force_at(U, P.X[i], P.G[i], g.V, q, f1, f2);
        if (i == 0 && !accumulate) {
            a1 = P.rho[0] * f1;
            a2 = P.rho[0] * f2;
        } else {
            if (i == 0) {
                a1 = frc[q.x];
                a2 = frc[q.x + g.V];
            }
            a1 += P.rho[i] * f1;
            a2 += P.rho[i] * f2;
        }
    }
    frc[q.x] = a1;
    frc[q.x + g.V] = a2;
}

// plaquette! (mode 0, Re P) and qtop! (mode 1, arg P) -- src/QED2dAction.jl:2-32
__global__ void __launch_bounds__(TILE) k_plaq_field(double* __restrict__ plx, const double2* __restrict__ U, Lat g,
                                                     int mode) {
    const Site q = tile_site(g);
    if (!q.ok) return;
    const double2 p = plaquette_of(__ldg(U + q.x), __ldg(U + g.V + q.xp1), __ldg(U + q.xp2), __ldg(U + g.V + q.x));
    plx[q.x] = mode == 0 ? p.x : atan2(p.y, p.x);
}

// krnl_force! -- src/QED2dAction.jl:34-53: every element of frc1 and frc2 written once
__global__ void __launch_bounds__(TILE) k_krnl_force(double* __restrict__ frc1, double* __restrict__ frc2,
                                                     const double2* __restrict__ U, Lat g, double beta) {
    const Site q = tile_site(g);
    if (!q.ok) return;
    const double2 p = plaquette_of(__ldg(U + q.x), __ldg(U + g.V + q.xp1), __ldg(U + q.xp2), __ldg(U + g.V + q.x));
    const double v = beta * p.y;
    frc1[q.x] = -v;
    frc1[q.x + g.V] = v;
    frc2[q.xp1 + g.V] = -v;
    frc2[q.xp2] = v;
}

// updt_fld! -- src/QED2dAction.jl:55-65; also refreshes the packed FP32 copy
__global__ void k_updt_fld(double2* __restrict__ U, const double* __restrict__ mom, double eps, long long V,
                           float4* __restrict__ U32) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= V) return;
    double s1, c1, s2, c2;
    sincos(eps * mom[x], &s1, &c1);
    sincos(eps * mom[x + V], &s2, &c2);
    const double2 u1 = cmul(make_double2(c1, s1), U[x]);
    const double2 u2 = cmul(make_double2(c2, s2), U[x + V]);
    U[x] = u1;
    U[x + V] = u2;
    if (U32) st_links32(U32, V, x, u1, u2);
}

__global__ void k_pack_links(float4* __restrict__ U32, const double2* __restrict__ U, long long V) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= V) return;
    const double2 u1 = U[x], u2 = U[x + V];
    st_links32(U32, V, x, u1, u2);
}

// krnl_unfold! / krnl_reflect! -- src/QED2dFields.jl:12-25,37-50
__global__ void k_unfold(double2* __restrict__ Uout, const double2* __restrict__ Uin, Lat g, int reflect) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= 2 * g.V) return;
    const int mu = x >= g.V;
    const long long s = x - mu * g.V;
    const int i2 = (int)(s / g.L1), i1 = (int)(s - (long long)i2 * g.L1);
    const long long L1n = 2LL * g.L1, Vout = 4 * g.V;
    const double2 u = Uin[x];
    const double2 uc = reflect ? conj(u) : u;
    double2* o = Uout + mu * Vout;
    o[i1 + L1n * i2] = u;
    o[i1 + g.L1 + L1n * i2] = uc;
    o[i1 + L1n * (i2 + g.L2)] = uc;
    o[i1 + g.L1 + L1n * (i2 + g.L2)] = u;
}

// plwv -- src/QED2dUtils.jl:2-11; pref = i sqrt(-sin^2 k1 - sin^2 k2) / (sin k1 + i sin k2)
__global__ void k_plwv(double2* __restrict__ so, Lat g, double k1, double k2, double2 pref) {
    const long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x >= g.V) return;
    const int i2 = (int)(x / g.L1), i1 = (int)(x - (long long)i2 * g.L1);
    double s, c;
    sincos(k1 * i1 + k2 * i2, &s, &c);
    const double2 e = make_double2(c, s);
    so[x] = cmul(pref, e);
    so[x + g.V] = e;
}

// n N(0,1) numbers of (seed, stream, counter), times scale
__global__ void k_random_normal(double* __restrict__ out, long long n, uint64_t seed, uint32_t stream,
                                uint32_t counter, double scale) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (2 * j >= n) return;
    double z0, z1;
    normal_pair(seed, stream, counter, (uint64_t)j, z0, z1);
    out[2 * j] = scale * z0;
    if (2 * j + 1 < n) out[2 * j + 1] = scale * z1;
}

// mom += eps * (frc1 + frc2 [+ fermion force]) -- the kick of OMF4!/update_momenta!
// (src/QED2dHMC.jl:256,478,554) with krnl_force!'s two scattered buffers gathered
// per link, so no force arrays are stored.  The total gauge force on the links
// of site x is F1 = -v(x) + v(x - 2), F2 = v(x) - v(x - 1) with v = beta Im P
// (gauge_force_at).  Each thread computes the plaquette of its own site once
// into shared memory; the last warp also computes the row below the tile and
// the second-last warp's first TY lanes the column left of it (the tile's halo;
// two warps with two plaquettes each, the others one); every thread reads its
// neighbours' values from there: 4 link loads per site instead of 10, the same
// plaquette arithmetic, so the same bits.  FERM: add the fermion force of
// (X, G = g5Dw X); FRC: add frc.  The kicks without the fermion force fit in 40
// registers (6 blocks per SM on this streaming kernel), the fermion ones in 64.
template <bool FERM, bool FRC>
__global__ void __launch_bounds__(TILE, FERM ? 4 : 6) k_mom_kick(double* __restrict__ mom, const double2* __restrict__ U, Lat g,
                                                   double beta, double eps, const double2* __restrict__ X,
                                                   const double2* __restrict__ G, const double* __restrict__ frc) {
    __shared__ double sv[TY + 1][TX + 1];   // [1 + row][1 + column]; row 0 / column 0: the halo
    int t1, t2;
    if (gridDim.y > 1 || g.L2 <= TY) {
        t1 = blockIdx.x;
        t2 = blockIdx.y;
    } else {
        const int nt1 = (g.L1 + TX - 1) / TX;
        t2 = blockIdx.x / nt1;
        t1 = blockIdx.x - t2 * nt1;
    }
    const Site q = site_at(g, t1, t2, threadIdx.x);
    const int lx = threadIdx.x & (TX - 1), ly = threadIdx.x >> 5;
    const long long V = g.V;
    double mo1 = 0.0, mo2 = 0.0;
    if (q.ok) {
        mo1 = mom[q.x];   // issued with the link loads
        mo2 = mom[q.x + V];
        const double2 u1x = __ldg(U + q.x), u2x = __ldg(U + V + q.x);
        const double2 u2xp1 = __ldg(U + V + q.xp1), u1xp2 = __ldg(U + q.xp2);
        sv[ly + 1][lx + 1] = beta * plaquette_of(u1x, u2xp1, u1xp2, u2x).y;
    }
    if (ly == TY - 1) {   // v(y - 2) for y in the tile's first row: links of y - 2, y - 2 + 1 and y
        const Site y = site_at(g, t1, t2, lx);
        if (y.ok) {
            const long long xp1m2 = y.xm2 + (y.xp1 - y.x);
            sv[0][lx + 1] = beta * plaquette_of(__ldg(U + y.xm2), __ldg(U + V + xp1m2), __ldg(U + y.x),
                                                __ldg(U + V + y.xm2)).y;
        }
    } else if (ly == TY - 2 && lx < TY) {   // v(y - 1) for y in the tile's first column: links of y - 1, y, y - 1 + 2
        const Site y = site_at(g, t1, t2, TX * lx);
        if (y.ok) {
            const long long xm1p2 = y.xp2 + (y.xm1 - y.x);
            sv[lx + 1][0] = beta * plaquette_of(__ldg(U + y.xm1), __ldg(U + V + y.x), __ldg(U + xm1p2),
                                                __ldg(U + V + y.xm1)).y;
        }
    }
    __syncthreads();
    if (!q.ok) return;
    const double v = sv[ly + 1][lx + 1];
    double F1 = -v + sv[ly][lx + 1];
    double F2 = v - sv[ly + 1][lx];
    if constexpr (FERM) {
        double f1, f2;
        fermion_force_at(U, X, G, V, q, f1, f2);
        F1 = F1 + f1;
        F2 = F2 + f2;
    }
    if constexpr (FRC) {
        F1 = F1 + frc[q.x];
        F2 = F2 + frc[q.x + V];
    }
    mom[q.x] = mo1 + eps * F1;
    mom[q.x + V] = mo2 + eps * F2;
}

// updt_fld! followed by the pure-gauge kick, in one pass (OMF4! and leapfrog
// pure gauge alternate the two, src/QED2dHMC.jl:248-305): Uout = e^{i eu mom_in} Uin,
// mom_out = mom_in + ek F(Uout).  The tile's updated links and the halo the force
// needs (U1 on rows -1..TY of columns -1..31, U2 on rows -1..TY-1 of columns
// -1..32) are computed into shared memory, each with the operations of
// updt_fld!; then the plaquettes of the tile, of the row below and of the
// column to its left; then the kick with those of k_mom_kick.  Reads Uin and mom_in,
// writes Uout and mom_out (distinct buffers: neighbours read the old momenta).  Lattices
// of whole 32 x TY tiles only.  Per site: links in 32 + out 32, momenta in 16 +
// out 16 (96 B) instead of 80 + 64 B for the two kernels.
__global__ void __launch_bounds__(TILE) k_updt_kick(double2* __restrict__ Uout, const double2* __restrict__ Uin,
                                                    double* __restrict__ mom_out, const double* __restrict__ mom_in, Lat g,
                                                    double beta, double eu, double ek) {
    constexpr int R1 = TY + 2, C1 = TX + 1;   // U1: rows -1..TY, columns -1..31
    constexpr int R2 = TY + 1, C2 = TX + 2;   // U2: rows -1..TY-1, columns -1..32
    __shared__ double2 s1[R1 * C1], s2[R2 * C2];
    __shared__ double sv[(TY + 1) * (TX + 1)];   // v on rows -1..TY-1, columns -1..31
    int t1, t2;
    if (gridDim.y > 1 || g.L2 <= TY) {
        t1 = blockIdx.x;
        t2 = blockIdx.y;
    } else {
        const int nt1 = g.L1 / TX;
        t2 = blockIdx.x / nt1;
        t1 = blockIdx.x - t2 * nt1;
    }
    const long long V = g.V;
    const int i10 = t1 * TX, i20 = t2 * TY;
    // the updated link of direction mu at tile position (row, col), periodic
    auto upd = [&](int mu, int row, int col, bool own) {
        int i1 = i10 + col, i2 = i20 + row;
        i1 = i1 < 0 ? i1 + g.L1 : (i1 >= g.L1 ? i1 - g.L1 : i1);
        i2 = i2 < 0 ? i2 + g.L2 : (i2 >= g.L2 ? i2 - g.L2 : i2);
        const long long x = i1 + (long long)g.L1 * i2 + (mu ? V : 0);
        double s, c;
        sincos(eu * mom_in[x], &s, &c);
        const double2 u = cmul(make_double2(c, s), Uin[x]);
        if (own) Uout[x] = u;
        return u;
    };
    for (int e = threadIdx.x; e < R1 * C1; e += TILE) {
        const int row = e / C1 - 1, col = e % C1 - 1;
        s1[e] = upd(0, row, col, row >= 0 && row < TY && col >= 0);
    }
    for (int e = threadIdx.x; e < R2 * C2; e += TILE) {
        const int row = e / C2 - 1, col = e % C2 - 1;
        s2[e] = upd(1, row, col, row >= 0 && col >= 0 && col < TX);
    }
    __syncthreads();
    // v(y) = beta Im P(y) from U1(y), U2(y + 1), U1(y + 2), U2(y)
    for (int e = threadIdx.x; e < (TY + 1) * (TX + 1); e += TILE) {
        const int row = e / (TX + 1) - 1, col = e % (TX + 1) - 1;
        if (row >= 0 && col >= 0 || row < 0 && col >= 0 || row >= 0 && col < 0) {   // not the corner
            const double2 u1y = s1[(row + 1) * C1 + col + 1], u1yp2 = s1[(row + 2) * C1 + col + 1];
            const double2 u2y = s2[(row + 1) * C2 + col + 1], u2yp1 = s2[(row + 1) * C2 + col + 2];
            sv[e] = beta * plaquette_of(u1y, u2yp1, u1yp2, u2y).y;
        }
    }
    __syncthreads();
    const int lx = threadIdx.x & (TX - 1), ly = threadIdx.x >> 5;
    const long long x = (i10 + lx) + (long long)g.L1 * (i20 + ly);
    const double v = sv[(ly + 1) * (TX + 1) + lx + 1];
    const double F1 = -v + sv[ly * (TX + 1) + lx + 1];
    const double F2 = v - sv[(ly + 1) * (TX + 1) + lx];
    mom_out[x] = mom_in[x] + ek * F1;
    mom_out[x + V] = mom_in[x + V] + ek * F2;
}

// y = a x + b z (complex scalars; z may alias y)
__global__ void k_zaxpby(double2* y, double2 a, const double2* x, double2 b, const double2* z,
                         long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double2 v = cmul(a, x[i]);
    if (z) v = v + cmul(b, z[i]);
    y[i] = v;
}

// ---------------------------------------------------------------------------
// single-launch deterministic reductions: per-block compensated sums to part[]
// (hi, lo pairs), the last block to finish merges part[] in a fixed order into
// ctl->scal[slot..] (hi + lo)
constexpr int RB = 256;

template <int NV>
__device__ __forceinline__ void finish_reduce(DSum (&v)[NV], double* part, DevCtl* ctl, int slot) {
    static_assert(2 * NV <= kMaxPartVals, "partials hold (hi, lo) pairs");
    __shared__ double smem[64 * NV];
    __shared__ bool last;
    block_dsum<NV>(v, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            part[(size_t)(2 * k) * kMaxPartBlocks + blockIdx.x] = v[k].hi;
            part[(size_t)(2 * k + 1) * kMaxPartBlocks + blockIdx.x] = v[k].lo;
        }
        __threadfence();
        last = atomicAdd(&ctl->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < 32) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            DSum s{0.0, 0.0};
            for (int i = threadIdx.x; i < (int)gridDim.x; i += 32)
                dsum_merge(s, DSum{__ldcg(part + (size_t)(2 * k) * kMaxPartBlocks + i),
                                   __ldcg(part + (size_t)(2 * k + 1) * kMaxPartBlocks + i)});
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const DSum t{__shfl_xor_sync(0xffffffffu, s.hi, o), __shfl_xor_sync(0xffffffffu, s.lo, o)};
                dsum_merge(s, t);
            }
            if (threadIdx.x == 0) ctl->scal[slot + k] = s.hi + s.lo;
        }
        if (threadIdx.x == 0) ctl->ticket = 0;
    }
}

// |x|^2 (kind 0) or <x, y> (kind 1), compensated
__global__ void __launch_bounds__(RB) k_reduce_vec(int kind, const double2* __restrict__ x,
                                                   const double2* __restrict__ y, long long n, double* part,
                                                   DevCtl* ctl, int slot) {
    DSum v[2] = {{0.0, 0.0}, {0.0, 0.0}};
    for (long long i = blockIdx.x * (long long)RB + threadIdx.x; i < n; i += (long long)gridDim.x * RB) {
        const double2 a = x[i];
        if (kind == 0) {
            dsum_add(v[0], norm2(a));
        } else {
            const double2 d = cjmul(a, y[i]);
            dsum_add(v[0], d.x);
            dsum_add(v[1], d.y);
        }
    }
    finish_reduce<2>(v, part, ctl, slot);
}

// (sum Re P, sum arg P, sum mom^2), compensated -- Action/Plaquette/Qtop/Hamiltonian
// (src/QED2dHMC.jl:198-237)
__global__ void __launch_bounds__(RB) k_reduce_gauge(const double2* __restrict__ U, const double* __restrict__ mom,
                                                     Lat g, double* part, DevCtl* ctl, int slot) {
    DSum v[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    for (long long x = blockIdx.x * (long long)RB + threadIdx.x; x < g.V; x += (long long)gridDim.x * RB) {
        const int i2 = (int)(x / g.L1), i1 = (int)(x - (long long)i2 * g.L1);
        const long long xp1 = (i1 + 1 == g.L1) ? x - (g.L1 - 1) : x + 1;
        const long long xp2 = (i2 + 1 == g.L2) ? (long long)i1 : x + g.L1;
        const double2 p = plaquette_of(__ldg(U + x), __ldg(U + g.V + xp1), __ldg(U + xp2), __ldg(U + g.V + x));
        dsum_add(v[0], p.x);
        dsum_add(v[1], atan2(p.y, p.x));
        if (mom) dsum_add(v[2], mom[x] * mom[x] + mom[x + g.V] * mom[x + g.V]);
    }
    finish_reduce<3>(v, part, ctl, slot);
}

__global__ void k_copy_scalar(DevCtl* ctl, int dst, int src) { ctl->scal[dst] = ctl->scal[src]; }

// y = x / ctl->scal[slot] (the power method's normalisation, kept on the device)
__global__ void k_scale_inv(double2* y, const double2* x, long long n, const DevCtl* __restrict__ ctl, int slot) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double d = ctl->scal[slot];
    y[i] = make_double2(x[i].x / d, x[i].y / d);
}

// ---------------------------------------------------------------------------
// launchers
static int post_launch(const char* name) {
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, name);
    return QED2D_OK;
}

static unsigned blocks_for(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

static unsigned reduce_grid(long long n) {
    long long b = (n + RB - 1) / RB;
    if (b > 4 * 148) b = 4 * 148;
    if (b < 1) b = 1;
    return (unsigned)b;
}

int launch_g5dw_c64(Ctx& c, float2* so, const float2* U, const float2* si, double am0) {
    k_g5dw_c64<<<tiles_grid2(c.g), TILE, 0, c.stream>>>(so, U, si, (float)(2.0 + am0), c.g);
    return post_launch("k_g5dw_c64");
}

int launch_g5dw(Ctx& c, double2* so, const double2* U, const double2* si, double am0, const double2* addv,
                double2 addc, bool g5_out) {
    k_g5dw<<<tiles_grid2(c.g), TILE, 0, c.stream>>>(so, U, si, 2.0 + am0, c.g, addv, addc, g5_out ? 1 : 0);
    return post_launch("k_g5dw");
}

int launch_g5(Ctx& c, double2* so, const double2* si) {
    k_g5<<<blocks_for(c.g.V, 256), 256, 0, c.stream>>>(so, si, c.g.V);
    return post_launch("k_g5");
}

int launch_tr_dqwdu(Ctx& c, double* frc, const double2* U, const double2* X, const double2* G) {
    k_force<<<tiles_grid2(c.g), TILE, 0, c.stream>>>(frc, U, X, G, c.g, 1.0, 0);
    return post_launch("k_force");
}

int launch_force_accum(Ctx& c, double* frc, const double2* U, const double2* X, const double2* G, double rho,
                       bool accumulate) {
    k_force<<<tiles_grid2(c.g), TILE, 0, c.stream>>>(frc, U, X, G, c.g, rho, accumulate ? 1 : 0);
    return post_launch("k_force");
}

int launch_force_poles(Ctx& c, double* frc, const double2* U, const double2* const* X, double2* const* G,
                       const double* rho, int n, double am0, bool accumulate) {
    if (n < 1 || n > QED2D_MAXPOLES) return QED2D_ERR_BAD_ARG;
    Poles P{};
    for (int i = 0; i < n; i++) {
        P.X[i] = X[i];
        P.G[i] = G[i];
        P.rho[i] = rho[i];
    }
    P.n = n;
    dim3 grid = tiles_grid2(c.g);
    grid.z = (unsigned)n;
    k_g5dw_poles<<<grid, TILE, 0, c.stream>>>(U, P, 2.0 + am0, c.g);
    QTRY(post_launch("k_g5dw_poles"));
    k_force_poles<<<tiles_grid2(c.g), TILE, 0, c.stream>>>(frc, U, P, c.g, accumulate ? 1 : 0);
    return post_launch("k_force_poles");
}

int launch_plaq_field(Ctx& c, double* plx, const double2* U, int mode) {
    k_plaq_field<<<tiles_grid2(c.g), TILE, 0, c.stream>>>(plx, U, c.g, mode);
    return post_launch("k_plaq_field");
}

int launch_krnl_force(Ctx& c, double* frc1, double* frc2, const double2* U) {
    k_krnl_force<<<tiles_grid2(c.g), TILE, 0, c.stream>>>(frc1, frc2, U, c.g, c.beta);
    return post_launch("k_krnl_force");
}

int launch_updt_fld(Ctx& c, double2* U, const double* mom, double eps, float4* U32) {
    k_updt_fld<<<blocks_for(c.g.V, 256), 256, 0, c.stream>>>(U, mom, eps, c.g.V, U32);
    return post_launch("k_updt_fld");
}

int launch_pack_links(Ctx& c, float4* U32, const double2* U) {
    k_pack_links<<<blocks_for(c.g.V, 256), 256, 0, c.stream>>>(U32, U, c.g.V);
    return post_launch("k_pack_links");
}

int launch_unfold(Ctx& c, double2* Uout, const double2* Uin, int reflect) {
    k_unfold<<<blocks_for(2 * c.g.V, 256), 256, 0, c.stream>>>(Uout, Uin, c.g, reflect);
    return post_launch("k_unfold");
}

int launch_plwv(Ctx& c, double2* so, double k1, double k2) {
    // pref = i * sqrt(complex(-s1^2 - s2^2)) / (s1 + i s2); sqrt of a non-positive
    // real is i*sqrt(|.|), so pref = -sqrt(s1^2 + s2^2) / (s1 + i s2)
    const double s1 = sin(k1), s2 = sin(k2);
    const double r = sqrt(s1 * s1 + s2 * s2);
    double2 pref;
    // -r / (s1 + i s2) by Smith's scaled division
    if (fabs(s1) >= fabs(s2)) {
        const double t = s2 / s1, den = s1 + s2 * t;
        pref = make_double2(-r / den, (r * t) / den);
    } else {
        const double t = s1 / s2, den = s2 + s1 * t;
        pref = make_double2((-r * t) / den, r / den);
    }
    k_plwv<<<blocks_for(c.g.V, 256), 256, 0, c.stream>>>(so, c.g, k1, k2, pref);
    return post_launch("k_plwv");
}

int launch_random_normal(Ctx& c, double* out, int64_t n, uint64_t seed, uint32_t stream, uint32_t counter,
                         double scale) {
    if (n <= 0) return QED2D_OK;
    k_random_normal<<<blocks_for((n + 1) / 2, 256), 256, 0, c.stream>>>(out, n, seed, stream, counter, scale);
    return post_launch("k_random_normal");
}

bool updt_kick_fits(const Ctx& c) { return c.g.L1 % TX == 0 && c.g.L2 % TY == 0; }

int launch_updt_kick(Ctx& c, double2* Uout, const double2* Uin, double* mom_out, const double* mom_in, double eu,
                     double ek) {
    if (!updt_kick_fits(c)) return QED2D_ERR_UNSUPPORTED;
    k_updt_kick<<<tiles_grid2(c.g), TILE, 0, c.stream>>>(Uout, Uin, mom_out, mom_in, c.g, c.beta, eu, ek);
    return post_launch("k_updt_kick");
}

int launch_mom_kick(Ctx& c, double* mom, const double2* U, double eps, const double2* X, const double2* G,
                    const double* frc) {
    const dim3 grid = tiles_grid2(c.g);
    if (X && frc) k_mom_kick<true, true><<<grid, TILE, 0, c.stream>>>(mom, U, c.g, c.beta, eps, X, G, frc);
    else if (X) k_mom_kick<true, false><<<grid, TILE, 0, c.stream>>>(mom, U, c.g, c.beta, eps, X, G, frc);
    else if (frc) k_mom_kick<false, true><<<grid, TILE, 0, c.stream>>>(mom, U, c.g, c.beta, eps, X, G, frc);
    else k_mom_kick<false, false><<<grid, TILE, 0, c.stream>>>(mom, U, c.g, c.beta, eps, X, G, frc);
    return post_launch("k_mom_kick");
}

int launch_zaxpby(Ctx& c, double2* y, double2 a, const double2* x, double2 b, const double2* z, long long n) {
    k_zaxpby<<<blocks_for(n, 256), 256, 0, c.stream>>>(y, a, x, b, z, n);
    return post_launch("k_zaxpby");
}

int launch_copy(Ctx& c, void* dst, const void* src, size_t bytes) {
    if (dst == src || bytes == 0) return QED2D_OK;
    QCHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, c.stream));
    return QED2D_OK;
}

int launch_zero(Ctx& c, void* dst, size_t bytes) {
    QCHECK(cudaMemsetAsync(dst, 0, bytes, c.stream));
    return QED2D_OK;
}

int launch_reduce_vec(Ctx& c, int kind, const double2* x, const double2* y, long long n, int slot) {
    k_reduce_vec<<<reduce_grid(n), RB, 0, c.stream>>>(kind, x, y, n, c.part, c.ctl, slot);
    return post_launch("k_reduce_vec");
}

int launch_reduce_gauge(Ctx& c, const double2* U, const double* mom, int slot) {
    k_reduce_gauge<<<reduce_grid(c.g.V), RB, 0, c.stream>>>(U, mom, c.g, c.part, c.ctl, slot);
    return post_launch("k_reduce_gauge");
}

int launch_scale_inv(Ctx& c, double2* y, const double2* x, long long n, int slot) {
    k_scale_inv<<<blocks_for(n, 256), 256, 0, c.stream>>>(y, x, n, c.ctl, slot);
    return post_launch("k_scale_inv");
}

int launch_copy_scalar(Ctx& c, int dst_slot, int src_slot) {
    k_copy_scalar<<<1, 1, 0, c.stream>>>(c.ctl, dst_slot, src_slot);
    return post_launch("k_copy_scalar");
}

}  // namespace qed2d
