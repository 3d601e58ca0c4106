// D3Q19 lattice constants and the collision operators, device side.
//
// Velocity order, weights and opposite pairs follow LMB3d/lbm3d-perm.cpp:94-110:
//   k = 0 rest; 1,2 = +-x; 3,4 = +-y; 5,6 = +-z; 7-10 = xy diagonals;
//   11-14 = xz diagonals; 15-18 = yz diagonals; opp(k) pairs (1,2),(3,4),...
// Everything is a constexpr function so that, with the k loops fully
// unrolled, every velocity component folds to an immediate.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace lbm {

constexpr int Q3 = 19;

__host__ __device__ constexpr int ex3(int k)
{
    return (k == 1 || k == 7 || k == 9 || k == 11 || k == 13) ? 1
         : (k == 2 || k == 8 || k == 10 || k == 12 || k == 14) ? -1 : 0;
}
__host__ __device__ constexpr int ey3(int k)
{
    return (k == 3 || k == 7 || k == 10 || k == 15 || k == 17) ? 1
         : (k == 4 || k == 8 || k == 9 || k == 16 || k == 18) ? -1 : 0;
}
__host__ __device__ constexpr int ez3(int k)
{
    return (k == 5 || k == 11 || k == 14 || k == 15 || k == 18) ? 1
         : (k == 6 || k == 12 || k == 13 || k == 16 || k == 17) ? -1 : 0;
}
__host__ __device__ constexpr int opp3(int k) { return k == 0 ? 0 : ((k & 1) ? k + 1 : k - 1); }
__host__ __device__ constexpr double w3(int k) { return k == 0 ? 1.0 / 3.0 : (k <= 6 ? 1.0 / 18.0 : 1.0 / 36.0); }
__host__ __device__ constexpr float w3f(int k) { return k == 0 ? 1.0f / 3.0f : (k <= 6 ? 1.0f / 18.0f : 1.0f / 36.0f); }

// Per-solve physical constants, prepared on the host.
struct Phys3 {
    double F[3];      // body force
    double tau;       // relaxation time
    double pref;      // 1 - 1/(2 tau), Guo prefactor (LMB3d/lbm3d-perm.cpp:233)
    float Ff[3];
    float omega;      // 1/tau
    float preff;
};

// ---------------------------------------------------------------------------
// FP64 operator in the reference's evaluation order (LMB3d/lbm3d-perm.cpp:218-245).
// Compiled in a translation unit with -fmad=false so that each product and sum
// rounds exactly as the CPU oracle's; terms whose velocity component is zero
// are skipped, which leaves every rounded value unchanged (x + 0 == x, x*1 == x).
// g holds the pre-collision values on entry and the post-collision ones on exit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void collide_ref64(double (&g)[Q3], const Phys3 &P,
                                              double &ux, double &uy, double &uz)
{
    double r = 0.0, jx = 0.0, jy = 0.0, jz = 0.0;
#pragma unroll
    for (int k = 0; k < Q3; ++k) {
        r = r + g[k];
        if (ex3(k) == 1) jx = jx + g[k]; else if (ex3(k) == -1) jx = jx - g[k];
        if (ey3(k) == 1) jy = jy + g[k]; else if (ey3(k) == -1) jy = jy - g[k];
        if (ez3(k) == 1) jz = jz + g[k]; else if (ez3(k) == -1) jz = jz - g[k];
    }
    const double Fx = P.F[0], Fy = P.F[1], Fz = P.F[2];
    ux = (jx + 0.5 * Fx) / r;
    uy = (jy + 0.5 * Fy) / r;
    uz = (jz + 0.5 * Fz) / r;
    const double u2 = (ux * ux + uy * uy) + uz * uz;
    const double tau = P.tau, pref = P.pref;
    // (e_c - u_c) * F_c for e_c in {-1, 0, +1}; the three candidates per axis
    const double ax[3] = {(-1.0 - ux) * Fx, (0.0 - ux) * Fx, (1.0 - ux) * Fx};
    const double ay[3] = {(-1.0 - uy) * Fy, (0.0 - uy) * Fy, (1.0 - uy) * Fy};
    const double az[3] = {(-1.0 - uz) * Fz, (0.0 - uz) * Fz, (1.0 - uz) * Fz};
#pragma unroll
    for (int k = 0; k < Q3; ++k) {
        const int cx = ex3(k), cy = ey3(k), cz = ez3(k);
        // eu = ex*ux + ey*uy + ez*uz with the zero products dropped
        double eu;
        if (cx != 0 && cy != 0)      eu = (cx > 0 ? ux : -ux) + (cy > 0 ? uy : -uy);
        else if (cx != 0 && cz != 0) eu = (cx > 0 ? ux : -ux) + (cz > 0 ? uz : -uz);
        else if (cy != 0 && cz != 0) eu = (cy > 0 ? uy : -uy) + (cz > 0 ? uz : -uz);
        else if (cx != 0)            eu = cx > 0 ? ux : -ux;
        else if (cy != 0)            eu = cy > 0 ? uy : -uy;
        else if (cz != 0)            eu = cz > 0 ? uz : -uz;
        else                         eu = 0.0;
        const double feq = (w3(k) * r) * (((1.0 + 3.0 * eu) + (4.5 * eu) * eu) - 1.5 * u2);
        const double A = (ax[cx + 1] + ay[cy + 1]) + az[cz + 1];
        // e_k . F = (ex Fx + ey Fy) + ez Fz: products with 0 and +-1 are exact
        double eF = 0.0;
        if (cx != 0) eF = cx > 0 ? Fx : -Fx;
        if (cy != 0) eF = (cx != 0) ? eF + (cy > 0 ? Fy : -Fy) : (cy > 0 ? Fy : -Fy);
        if (cz != 0) eF = (cx != 0 || cy != 0) ? eF + (cz > 0 ? Fz : -Fz) : (cz > 0 ? Fz : -Fz);
        const double sk = (w3(k) * pref) * (3.0 * A + (9.0 * eu) * eF);
        g[k] = g[k] + ((feq - g[k]) / tau + sk);
    }
}

// ---------------------------------------------------------------------------
// FP32 operator on shifted populations h_k = s (f_k - w_k) (rho0 = 1, s the
// storage scale: a power of two for FP16, 1 otherwise), the form every
// reduced-precision storage uses.  It is the same BGK + Guo operator:
//   rho = 1 + sum h / s,  j = sum h e / s (sum w e = 0),
//   h_eq = s w (drho + rho (3 eu + 4.5 eu^2 - 1.5 u^2)),
//   S_k  = s w (1 - 1/2tau) [3 e.F - 3 u.F + 9 (e.u)(e.F)],
//   h   <- h + (h_eq - h)/tau + S_k,
// evaluated per opposite pair (k, opp k): e.u and e.F change sign, so each
// pair shares one symmetric and one antisymmetric part and costs about half
// of two separate directions.  Keeping the O(u) deviations instead of O(1)
// populations removes the cancellation that makes raw FP32 storage drift by
// ~1e-2 in k; working in scaled units leaves FP16 loads and stores a bare
// conversion.  W1: tau == 1, where h drops out of the update.
// ---------------------------------------------------------------------------
//
// Every operation is written out with its rounding (no contraction left to
// the compiler), and the operator is a template over the arithmetic: F32x1
// evaluates one voxel, F32x2 two voxels at once with the sm_100 packed FP32
// instructions (one issue slot per pair of lanes).  Both round each value
// identically, so a kernel that collides voxel pairs gives the same bits as
// one that collides them one at a time.
struct F32x1 {
    using V = float;
    __device__ static __forceinline__ V add(V a, V b) { return __fadd_rn(a, b); }
    __device__ static __forceinline__ V sub(V a, V b) { return __fsub_rn(a, b); }
    __device__ static __forceinline__ V mul(V a, V b) { return __fmul_rn(a, b); }
    __device__ static __forceinline__ V fma(V a, V b, V c) { return __fmaf_rn(a, b, c); }
    __device__ static __forceinline__ V neg(V a) { return -a; }
    __device__ static __forceinline__ V splat(float x) { return x; }
    __device__ static __forceinline__ V recip(V a) { return __frcp_rn(a); }
};
struct F32x2 {
    using V = float2;
    __device__ static __forceinline__ V add(V a, V b) { return __fadd2_rn(a, b); }
    // a - b as b * (-1) + a: the product is exact, so one rounding, as __fsub_rn
    __device__ static __forceinline__ V sub(V a, V b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
    __device__ static __forceinline__ V mul(V a, V b) { return __fmul2_rn(a, b); }
    __device__ static __forceinline__ V fma(V a, V b, V c) { return __ffma2_rn(a, b, c); }
    __device__ static __forceinline__ V neg(V a) { return make_float2(-a.x, -a.y); }
    __device__ static __forceinline__ V splat(float x) { return make_float2(x, x); }
    __device__ static __forceinline__ V recip(V a) { return make_float2(__frcp_rn(a.x), __frcp_rn(a.y)); }
};

// sign * v accumulated into acc; `first` starts the sum with the term itself
template <class O>
__device__ __forceinline__ void signed_acc(typename O::V &acc, bool &first, int sign, typename O::V v)
{
    if (!sign) return;
    if (first) acc = sign > 0 ? v : O::neg(v);
    else acc = sign > 0 ? O::add(acc, v) : O::sub(acc, v);
    first = false;
}

__device__ __forceinline__ float signed_sum3(int cx, int cy, int cz, float x, float y, float z)
{
    float r = 0.0f;
    bool first = true;
    signed_acc<F32x1>(r, first, cx, x);
    signed_acc<F32x1>(r, first, cy, y);
    signed_acc<F32x1>(r, first, cz, z);
    return r;
}

template <bool W1, class O>
__device__ __forceinline__ void collide_pairs(typename O::V (&h)[Q3], const Phys3 &P, float s, float is,
                                              typename O::V &ux, typename O::V &uy, typename O::V &uz)
{
    using V = typename O::V;
    // pair sums and differences; the odd member k of each pair is the "+" one
    V sm[9], df[9];
#pragma unroll
    for (int p = 0; p < 9; ++p) {
        sm[p] = O::add(h[2 * p + 1], h[2 * p + 2]);
        df[p] = O::sub(h[2 * p + 1], h[2 * p + 2]);
    }
    V drs = h[0];
#pragma unroll
    for (int p = 0; p < 9; ++p) drs = O::add(drs, sm[p]);
    V jx = O::splat(0.0f), jy = O::splat(0.0f), jz = O::splat(0.0f);
    bool fx = true, fy = true, fz = true;
#pragma unroll
    for (int p = 0; p < 9; ++p) {
        const int k = 2 * p + 1;
        signed_acc<O>(jx, fx, ex3(k), df[p]);
        signed_acc<O>(jy, fy, ey3(k), df[p]);
        signed_acc<O>(jz, fz, ez3(k), df[p]);
    }
    // per-solve scalars (the same for every voxel)
    const float Fx = P.Ff[0], Fy = P.Ff[1], Fz = P.Ff[2];
    const float spr = __fmul_rn(s, P.preff);
    const float p9 = __fmul_rn(9.0f, spr), p3 = __fmul_rn(3.0f, spr);
    const float om = P.omega;
    const V rho = O::add(O::splat(1.0f), O::mul(drs, O::splat(is)));
    const V ir = O::recip(rho);
    ux = O::mul(O::fma(jx, O::splat(is), O::splat(0.5f * Fx)), ir);
    uy = O::mul(O::fma(jy, O::splat(is), O::splat(0.5f * Fy)), ir);
    uz = O::mul(O::fma(jz, O::splat(is), O::splat(0.5f * Fz)), ir);
    const V u2 = O::fma(uz, uz, O::fma(uy, uy, O::mul(ux, ux)));
    const V uF = O::fma(uz, O::splat(Fz), O::fma(uy, O::splat(Fy), O::mul(ux, O::splat(Fx))));
    const V srho = O::mul(O::splat(s), rho);
    // symmetric, eu = eF = 0 part: drs - 1.5 s rho u^2 - 3 s pr uF
    const V c1 = O::fma(O::splat(-p3), uF, O::fma(O::mul(O::splat(-1.5f), srho), u2, drs));
    const V r45 = O::mul(O::splat(4.5f), srho), r3 = O::mul(O::splat(3.0f), srho);
    V c1p, p3uF;
    if constexpr (W1) {
        // rest population: h_eq + S = w0 c1
        h[0] = O::mul(O::splat(w3f(0)), c1);
    } else {
        c1p = O::fma(O::splat(p3), uF, c1);      // equilibrium part of c1
        p3uF = O::mul(O::splat(p3), uF);
        h[0] = O::sub(O::fma(O::splat(om), O::fma(O::splat(w3f(0)), c1p, O::neg(h[0])), h[0]),
                      O::mul(O::splat(w3f(0)), p3uF));
    }
#pragma unroll
    for (int p = 0; p < 9; ++p) {
        const int k = 2 * p + 1;
        const int cx = ex3(k), cy = ey3(k), cz = ez3(k);
        V eu = O::splat(0.0f);
        bool fe = true;
        signed_acc<O>(eu, fe, cx, ux);
        signed_acc<O>(eu, fe, cy, uy);
        signed_acc<O>(eu, fe, cz, uz);
        const float eF = signed_sum3(cx, cy, cz, Fx, Fy, Fz);
        const float w = w3f(k);
        const float p9eF = __fmul_rn(p9, eF), p3eF = __fmul_rn(p3, eF);
        if constexpr (W1) {
            // (h_eq + S)_k = sym + anti, (h_eq + S)_opp = sym - anti
            const V sym = O::mul(O::splat(w), O::fma(O::fma(r45, eu, O::splat(p9eF)), eu, c1));
            const V anti = O::mul(O::splat(w), O::fma(r3, eu, O::splat(p3eF)));
            h[k] = O::add(sym, anti);
            h[k + 1] = O::sub(sym, anti);
        } else {
            // equilibrium and source split: E = Es +- Ea, S = Ss +- Sa
            const V Es = O::mul(O::splat(w), O::fma(O::mul(r45, eu), eu, c1p));
            const V Ea = O::mul(O::mul(O::splat(w), r3), eu);
            const V Ss = O::mul(O::splat(w), O::fma(O::splat(p9eF), eu, O::neg(p3uF)));
            const V Sa = O::splat(__fmul_rn(w, p3eF));
            h[k] = O::add(O::fma(O::splat(om), O::sub(O::add(Es, Ea), h[k]), h[k]), O::add(Ss, Sa));
            h[k + 1] = O::add(O::fma(O::splat(om), O::sub(O::sub(Es, Ea), h[k + 1]), h[k + 1]), O::sub(Ss, Sa));
        }
    }
}

// ---------------------------------------------------------------------------
// Storage formats: element type, compute type, whether the stored value is
// the (scaled) shifted population, and plain load/store conversions.
// ---------------------------------------------------------------------------
// W: the word cp.async stages for one population (cp.async copies 4, 8 or 16
// bytes, so a 2-byte population travels in the aligned 4-byte word that
// holds it, and `unword` picks its half).
struct StoreF64 {
    using T = double; using C = double; using W = double;
    __device__ static __forceinline__ const W *word(const T *p) { return p; }
    __device__ static __forceinline__ C unword(W w, unsigned) { return w; }
    static constexpr bool shifted = false;
    static constexpr bool stochastic = false;
    static constexpr int code = 0;
    __device__ static __forceinline__ C ld(const T *p) { return __ldcs(p); }
    __device__ static __forceinline__ void st(T *p, C v) { __stcs(p, v); }
    __host__ __device__ static constexpr double init(int k) { return w3(k); }
};
struct StoreF32 {
    using T = float; using C = float; using W = float;
    __device__ static __forceinline__ const W *word(const T *p) { return p; }
    __device__ static __forceinline__ C unword(W w, unsigned) { return w; }
    static constexpr bool shifted = true;
    static constexpr bool stochastic = false;
    static constexpr int code = 1;
    __device__ static __forceinline__ C ld(const T *p) { return __ldcs(p); }
    __device__ static __forceinline__ void st(T *p, C v) { __stcs(p, v); }
    __host__ __device__ static constexpr double init(int) { return 0.0; }
    // two adjacent slots (p 8-byte aligned) in one access
    __device__ static __forceinline__ void ld2(const T *p, C &lo, C &hi)
    {
        const float2 v = __ldcs(reinterpret_cast<const float2 *>(p));
        lo = v.x; hi = v.y;
    }
    // the same pair from a shared-memory copy of the slots
    __device__ static __forceinline__ void lds2(const T *p, C &lo, C &hi)
    {
        const float2 v = *reinterpret_cast<const float2 *>(p);
        lo = v.x; hi = v.y;
    }
    __device__ static __forceinline__ void st2(T *p, C lo, C hi, uint32_t, uint32_t)
    {
        __stcs(reinterpret_cast<float2 *>(p), make_float2(lo, hi));
    }
};
struct StoreF16 {
    using T = __half; using C = float; using W = uint32_t;
    __device__ static __forceinline__ const W *word(const T *p)
    {
        return reinterpret_cast<const W *>(reinterpret_cast<uintptr_t>(p) & ~uintptr_t(3));
    }
    __device__ static __forceinline__ C unword(W w, unsigned idx)
    {
        return __half2float(__ushort_as_half((unsigned short)(w >> ((idx & 1u) * 16))));
    }
    static constexpr bool shifted = true;
    static constexpr int code = 2;
    __device__ static __forceinline__ C ld(const T *p) { return __half2float(__ldcs(p)); }
    __device__ static __forceinline__ void st(T *p, C v) { __stcs(p, __float2half_rn(v)); }
    // stochastic rounding (sm_100a cvt.rs with random bits; the product bits
    // in `rnd` are rotated so that its well-mixed high half is used): rounds up
    // with probability equal to the distance from the lower half, unbiased, so
    // increments smaller than half an ulp accumulate instead of being rounded
    // away every step
    static constexpr bool stochastic = true;
    __device__ static __forceinline__ void st_sr(T *p, C v, uint32_t rnd)
    {
        uint32_t d;
        asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(0.0f), "f"(v), "r"(__funnelshift_l(rnd, rnd, 16)));
        __stcs(p, __ushort_as_half((unsigned short)(d & 0xffffu)));
    }
    // two adjacent slots (p 4-byte aligned) in one access; the pair store
    // rounds each half with the random bits st_sr would give it (the low 16
    // of its rotated bits), so results equal two single stores
    __device__ static __forceinline__ void ld2(const T *p, C &lo, C &hi)
    {
        const uint32_t w = __ldcs(reinterpret_cast<const unsigned int *>(p));
        lo = __half2float(__ushort_as_half((unsigned short)(w & 0xffffu)));
        hi = __half2float(__ushort_as_half((unsigned short)(w >> 16)));
    }
    __device__ static __forceinline__ void lds2(const T *p, C &lo, C &hi)
    {
        const uint32_t w = *reinterpret_cast<const unsigned int *>(p);
        lo = __half2float(__ushort_as_half((unsigned short)(w & 0xffffu)));
        hi = __half2float(__ushort_as_half((unsigned short)(w >> 16)));
    }
    __device__ static __forceinline__ void st2(T *p, C lo, C hi, uint32_t rlo, uint32_t rhi)
    {
        const uint32_t rb = __byte_perm(rlo, rhi, 0x7632);   // high halves: rhi above, rlo below
        uint32_t d;
        asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rb));
        __stcs(reinterpret_cast<unsigned int *>(p), d);
    }
    __host__ __device__ static constexpr double init(int) { return 0.0; }
};
struct StoreBF16 {
    using T = __nv_bfloat16; using C = float; using W = uint32_t;
    __device__ static __forceinline__ const W *word(const T *p)
    {
        return reinterpret_cast<const W *>(reinterpret_cast<uintptr_t>(p) & ~uintptr_t(3));
    }
    __device__ static __forceinline__ C unword(W w, unsigned idx)
    {
        return __bfloat162float(__ushort_as_bfloat16((unsigned short)(w >> ((idx & 1u) * 16))));
    }
    static constexpr bool shifted = true;
    static constexpr int code = 3;
    __device__ static __forceinline__ C ld(const T *p) { return __bfloat162float(__ldcs(p)); }
    __device__ static __forceinline__ void st(T *p, C v) { __stcs(p, __float2bfloat16_rn(v)); }
    // stochastic rounding (as StoreF16)
    static constexpr bool stochastic = true;
    __device__ static __forceinline__ void st_sr(T *p, C v, uint32_t rnd)
    {
        uint32_t d;
        asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(0.0f), "f"(v), "r"(__funnelshift_l(rnd, rnd, 16)));
        __stcs(p, __ushort_as_bfloat16((unsigned short)(d & 0xffffu)));
    }
    __device__ static __forceinline__ void ld2(const T *p, C &lo, C &hi)
    {
        const uint32_t w = __ldcs(reinterpret_cast<const unsigned int *>(p));
        lo = __bfloat162float(__ushort_as_bfloat16((unsigned short)(w & 0xffffu)));
        hi = __bfloat162float(__ushort_as_bfloat16((unsigned short)(w >> 16)));
    }
    __device__ static __forceinline__ void lds2(const T *p, C &lo, C &hi)
    {
        const uint32_t w = *reinterpret_cast<const unsigned int *>(p);
        lo = __bfloat162float(__ushort_as_bfloat16((unsigned short)(w & 0xffffu)));
        hi = __bfloat162float(__ushort_as_bfloat16((unsigned short)(w >> 16)));
    }
    __device__ static __forceinline__ void st2(T *p, C lo, C hi, uint32_t rlo, uint32_t rhi)
    {
        const uint32_t rb = __byte_perm(rlo, rhi, 0x7632);   // high halves: rhi above, rlo below
        uint32_t d;
        asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rb));
        __stcs(reinterpret_cast<unsigned int *>(p), d);
    }
    __host__ __device__ static constexpr double init(int) { return 0.0; }
};

}  // namespace lbm
