// device.cuh -- device-side building blocks shared by every kernel of libqed2d:
// complex arithmetic on double2/float2, the gamma5-Wilson site stencil, the
// fermion-force site formula, Philox4x32-10, a bounded grid barrier and block
// reductions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace qed2d {

// ---------------------------------------------------------------------------
// complex arithmetic on CUDA vector types
template <typename R> struct cplx_of;
template <> struct cplx_of<double> { using type = double2; };
template <> struct cplx_of<float> { using type = float2; };

__device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }

#define QED2D_CPLX_OPS(C, R)                                                                        \
    __device__ __forceinline__ C operator+(C a, C b) { return mk(a.x + b.x, a.y + b.y); }          \
    __device__ __forceinline__ C operator-(C a, C b) { return mk(a.x - b.x, a.y - b.y); }          \
    __device__ __forceinline__ C operator-(C a) { return mk(-a.x, -a.y); }                          \
    __device__ __forceinline__ C operator*(R s, C a) { return mk(s * a.x, s * a.y); }               \
    __device__ __forceinline__ C cmul(C a, C b) { return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); } \
    /* conj(a) * b */                                                                               \
    __device__ __forceinline__ C cjmul(C a, C b) { return mk(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x); } \
    __device__ __forceinline__ C conj(C a) { return mk(a.x, -a.y); }                                \
    __device__ __forceinline__ C mul_i(C a) { return mk(-a.y, a.x); }                               \
    __device__ __forceinline__ R norm2(C a) { return a.x * a.x + a.y * a.y; }

QED2D_CPLX_OPS(double2, double)
QED2D_CPLX_OPS(float2, float)
#undef QED2D_CPLX_OPS

__device__ __forceinline__ float2 to_f(double2 a) { return make_float2((float)a.x, (float)a.y); }
__device__ __forceinline__ double2 to_d(float2 a) { return make_double2((double)a.x, (double)a.y); }

// ---------------------------------------------------------------------------
// A two-spin value at one site (spinor) or the two links at one site.
template <typename R> struct Pair {
    using C = typename cplx_of<R>::type;
    C a, b;
};

// gamma5-Wilson operator at one site -- the formula of gamm5Dw
// (src/QED2dDirac.jl:13-29), written with the two hopping products shared:
//   f1 = U1(x) (s1 - s2)(x+1),  b1 = conj(U1(x-1)) (s1 + s2)(x-1)
//   f2 = U2(x) (s1 + i s2)(x+2), b2 = conj(U2(x-2)) (s1 - i s2)(x-2)
//   A = (f1+b1)/2, A2 = (f1-b1)/2, B = (f2+b2)/2, B2 = i (f2-b2)/2
//   so1 = (2+m0) s1 - A - B,  so2 = -(2+m0) s2 - A2 - B2
template <typename R, typename C = typename cplx_of<R>::type>
__device__ __forceinline__ void g5dw_site(C s1, C s2, C p1s1, C p1s2, C m1s1, C m1s2, C p2s1, C p2s2, C m2s1,
                                          C m2s2, C u1, C u2, C u1m, C u2m, R m2, C& o1, C& o2) {
    const C f1 = cmul(u1, p1s1 - p1s2);
    const C b1 = cjmul(u1m, m1s1 + m1s2);
    const C f2 = cmul(u2, p2s1 + mul_i(p2s2));
    const C b2 = cjmul(u2m, m2s1 - mul_i(m2s2));
    const R h = R(0.5);
    const C A = h * (f1 + b1), A2 = h * (f1 - b1);
    const C B = h * (f2 + b2), B2 = mul_i(h * (f2 - b2));
    o1 = m2 * s1 - A - B;
    o2 = -(m2 * s2) - A2 - B2;
}

// tr_dQwdU at one site (src/QED2dDirac.jl:180-196): returns (frc1, frc2).
//   z1 = conj(U1)(conj(X1(x+1)) - conj(X2(x+1)))(G1+G2) - U1 (conj(X1)+conj(X2)) (G1(x+1)-G2(x+1))
//   z2 = conj(U2)(conj(X1(x+2)) - i conj(X2(x+2)))(G1 - i G2) - U2 (conj(X1) + i conj(X2)) (G1(x+2) + i G2(x+2))
//   frc = Re(i z) = -Im z
template <typename R, typename C = typename cplx_of<R>::type>
__device__ __forceinline__ void force_site(C u1, C u2, C x1, C x2, C g1, C g2, C x1p1, C x2p1, C g1p1, C g2p1,
                                           C x1p2, C x2p2, C g1p2, C g2p2, R& f1, R& f2) {
    const C z1 = cjmul(u1, cmul(conj(x1p1) - conj(x2p1), g1 + g2)) - cmul(u1, cmul(conj(x1) + conj(x2), g1p1 - g2p1));
    const C z2 = cjmul(u2, cmul(conj(x1p2) - mul_i(conj(x2p2)), g1 - mul_i(g2))) -
                 cmul(u2, cmul(conj(x1) + mul_i(conj(x2)), g1p2 + mul_i(g2p2)));
    f1 = -z1.y;
    f2 = -z2.y;
}

// plaquette U1(x) U2(x+1) conj(U1(x+2) U2(x)) (src/QED2dAction.jl:8-11)
__device__ __forceinline__ double2 plaquette_of(double2 u1x, double2 u2xp1, double2 u1xp2, double2 u2x) {
    return cmul(cmul(u1x, u2xp1), conj(cmul(u1xp2, u2x)));
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11) -- the same stream layout as the host
// restatement, so a trajectory's draws can be replayed on the CPU.
__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
        const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
        const uint32_t o0 = hi1 ^ c[1] ^ k0, o2 = hi0 ^ c[3] ^ k1;
        c[0] = o0; c[1] = lo1; c[2] = o2; c[3] = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
}

// pair j of (seed, stream, counter): two N(0,1) numbers by Box-Muller
__device__ __forceinline__ void normal_pair(uint64_t seed, uint32_t stream, uint32_t counter, uint64_t j, double& z0,
                                            double& z1) {
    uint32_t c[4] = {(uint32_t)j, (uint32_t)(j >> 32), stream, counter};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t a = ((((uint64_t)c[0]) << 32) | c[1]) >> 11;
    const uint64_t b = ((((uint64_t)c[2]) << 32) | c[3]) >> 11;
    const double u1 = ((double)a + 0.5) * 0x1.0p-53;
    const double u2 = (double)b * 0x1.0p-53;
    const double rad = sqrt(-2.0 * log(u1));
    double s, co;
    sincos(6.283185307179586 * u2, &s, &co);
    z0 = rad * co;
    z1 = rad * s;
}

// ---------------------------------------------------------------------------
// Grid-wide barriers for persistent kernels launched cooperatively (all blocks
// co-resident).  Every block's thread 0 adds one arrival to `arrivals` after a
// __syncthreads, with release semantics: the block's earlier writes, by any of
// its threads, are ordered before its arrival.  Two ways to leave:
//  * count_sync: thread 0 polls `arrivals` with acquire loads until it reaches
//    the barrier's target (n() per barrier so far), then the block
//    follows through a __syncthreads.  One fire-and-forget add and one poll per
//    block: the short path;
//  * arrive / release / wait: the block whose add sees target-1 arrived last; it
//    does the barrier's completion work (e.g. the final sum of a reduction) and
//    publishes the barrier's generation in `gen` (release), the others poll
//    `gen` (acquire).
// A group of the grid (e.g. the blocks of one replica) can have a barrier of its
// own: its own counter, and `members` = its number of blocks.
// The adds of all blocks form one chain of atomic updates of `arrivals`, so an
// acquire that sees the final count is ordered after every block's release.
// No sequentially-consistent fence (__threadfence) is needed on either path.
// Both counters only grow within a launch and are zeroed before it; the two
// kinds of barrier can follow each other in one kernel.  Waits are bounded:
// after ~2^26 polls (seconds) a block records QED2D_ERR_TIMEOUT in *err and
// leaves, and every block stops at its next check of *err.
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" : : "l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void red_release_add_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" : : "l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long atom_acq_rel_add_u64(unsigned long long* p, unsigned long long v) {
    unsigned long long old;
    asm volatile("atom.acq_rel.gpu.global.add.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
    return old;
}
__device__ __forceinline__ int ld_volatile_int(const int* p) {
    return *reinterpret_cast<const volatile int*>(p);
}

struct GridSync {
    unsigned long long* arrivals;
    unsigned long long* gen;
    int* err;
    unsigned members = 0;   // blocks taking part (a group of the grid with its own counter); 0: the grid
    unsigned long long target = 0;
    int nred = 0;   // reductions done so far: selects the double-buffered partials/results

    __device__ __forceinline__ unsigned n() const { return members ? members : gridDim.x; }

    // Poll *c (acquire) until it reaches target, about `limit` times at most
    // (checked every 8th poll).  False when the wait ended on the error flag or
    // timed out.  The error flag is read every 8th poll only: each read is an
    // L2 round trip that would otherwise sit between two polls of the counter.
    __device__ __forceinline__ bool poll(const unsigned long long* c, unsigned long long limit = 1ULL << 26) {
        unsigned long long polls = 0;
        while (ld_acquire_u64(c) < target) {
            if ((++polls & 7) == 0) {
                if (ld_volatile_int(err) != 0) return false;
                if (polls > limit) {
                    atomicExch(err, 2 /* QED2D_ERR_TIMEOUT */);
                    return false;
                }
            }
            __nanosleep(32);
        }
        return true;
    }
    // Counter barrier (all threads).  No status: a failed wait has set *err,
    // which the caller reads.
    __device__ __forceinline__ void count_sync() {
        __syncthreads();
        target += n();
        if (threadIdx.x == 0) {
            red_release_add_u64(arrivals, 1ULL);
            poll(arrivals);
        }
        __syncthreads();
    }
    // Arrive (all threads; thread 0 adds).  Returns true in the last-arriving
    // block, whose threads are then ordered after every block's arrival.
    __device__ __forceinline__ bool arrive(int* s_last) {
        __syncthreads();
        target += n();
        if (threadIdx.x == 0) {
            const unsigned long long old = atom_acq_rel_add_u64(arrivals, 1ULL);
            *s_last = old == target - 1;
        }
        __syncthreads();
        return *s_last != 0;
    }
    // Release (thread 0 of the last block, after its completion work and a
    // __syncthreads if other threads took part in it).
    __device__ __forceinline__ void release() { st_release_u64(gen, target); }
    // Wait for the release (thread 0 of the other blocks), bounded.
    __device__ __forceinline__ bool wait() { return poll(gen); }
    // Plain grid barrier; false once any block has given up.
    __device__ __forceinline__ bool sync() {
        count_sync();
        return ld_volatile_int(err) == 0;
    }
};

// ---------------------------------------------------------------------------
// block reductions (FP64): warp shuffles, then one value per warp in shared
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* smem /* >= 32*NV */) {
#pragma unroll
    for (int k = 0; k < NV; k++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) smem[k * 32 + warp] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double s = lane < nw ? smem[k * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            v[k] = s;
        }
    }
}

// Compensated (double-double) sums for the energies that Metropolis compares:
// TwoSum (Knuth; Moller) yields the exact rounding error of each addition, and
// the errors are summed separately (Ogita, Rump & Oishi's Sum2), so a sum of
// 10^8 site terms is as accurate as one in twice the working precision.
struct DSum {
    double hi, lo;
};
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
    s = a + b;
    const double bp = s - a;
    e = (a - (s - bp)) + (b - bp);
}
__device__ __forceinline__ void dsum_add(DSum& d, double x) {
    double s, e;
    two_sum(d.hi, x, s, e);
    d.hi = s;
    d.lo += e;
}
__device__ __forceinline__ void dsum_merge(DSum& d, const DSum& o) {
    double s, e;
    two_sum(d.hi, o.hi, s, e);
    d.hi = s;
    d.lo += e + o.lo;
}
// block reduction of NV compensated sums; the result is valid in thread 0
template <int NV>
__device__ __forceinline__ void block_dsum(DSum (&v)[NV], double* smem /* >= 64*NV */) {
#pragma unroll
    for (int k = 0; k < NV; k++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const DSum t{__shfl_xor_sync(0xffffffffu, v[k].hi, o), __shfl_xor_sync(0xffffffffu, v[k].lo, o)};
            dsum_merge(v[k], t);
        }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) {
            smem[(2 * k) * 32 + warp] = v[k].hi;
            smem[(2 * k + 1) * 32 + warp] = v[k].lo;
        }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            DSum s{lane < nw ? smem[(2 * k) * 32 + lane] : 0.0, lane < nw ? smem[(2 * k + 1) * 32 + lane] : 0.0};
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const DSum t{__shfl_xor_sync(0xffffffffu, s.hi, o), __shfl_xor_sync(0xffffffffu, s.lo, o)};
                dsum_merge(s, t);
            }
            v[k] = s;
        }
    }
}

// Sum part[0..n) in a fixed order, identically in every block (warp 0 does it;
// result broadcast through shared memory).  Deterministic across launches.
template <int NV>
__device__ __forceinline__ void sum_partials(const double* part, int n, double (&out)[NV], double* smem) {
    __syncthreads();
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double s = 0.0;
            for (int i = lane; i < n; i += 32) s += __ldcg(part + (size_t)k * n + i);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) smem[k] = s;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) out[k] = smem[k];
    __syncthreads();
}

}  // namespace qed2d
