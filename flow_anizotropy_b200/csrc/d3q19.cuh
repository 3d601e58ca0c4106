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
// FP32 operator on shifted populations h_k = f_k - w_k (rho0 = 1), the form
// every reduced-precision storage uses.  Mathematically the same BGK + Guo
// operator: rho = 1 + sum h, j = sum h e (sum w e = 0),
//   h_eq = w (drho + rho (3 eu + 4.5 eu^2 - 1.5 u^2)),
//   S_k  = w (1 - 1/2tau) [3 e.F - 3 u.F + 9 (e.u)(e.F)],
//   h   <- h + (h_eq - h)/tau + S_k.
// Keeping the O(u) deviations instead of O(1) populations removes the
// cancellation that makes raw FP32 storage drift by ~1e-2 in k.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void collide_shift32(float (&h)[Q3], const Phys3 &P,
                                                float &ux, float &uy, float &uz)
{
    float dr = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int k = 0; k < Q3; ++k) {
        dr += h[k];
        if (ex3(k) == 1) jx += h[k]; else if (ex3(k) == -1) jx -= h[k];
        if (ey3(k) == 1) jy += h[k]; else if (ey3(k) == -1) jy -= h[k];
        if (ez3(k) == 1) jz += h[k]; else if (ez3(k) == -1) jz -= h[k];
    }
    const float rho = 1.0f + dr;
    const float ir = 1.0f / rho;
    ux = (jx + 0.5f * P.Ff[0]) * ir;
    uy = (jy + 0.5f * P.Ff[1]) * ir;
    uz = (jz + 0.5f * P.Ff[2]) * ir;
    const float u2 = ux * ux + uy * uy + uz * uz;
    const float uF = ux * P.Ff[0] + uy * P.Ff[1] + uz * P.Ff[2];
    const float base = -1.5f * u2;
    const float om = P.omega, pr = P.preff;
    const float Fx = P.Ff[0], Fy = P.Ff[1], Fz = P.Ff[2];
#pragma unroll
    for (int k = 0; k < Q3; ++k) {
        const int cx = ex3(k), cy = ey3(k), cz = ez3(k);
        float eu = 0.f, eF = 0.f;
        if (cx) { eu += cx > 0 ? ux : -ux; eF += cx > 0 ? Fx : -Fx; }
        if (cy) { eu += cy > 0 ? uy : -uy; eF += cy > 0 ? Fy : -Fy; }
        if (cz) { eu += cz > 0 ? uz : -uz; eF += cz > 0 ? Fz : -Fz; }
        const float w = w3f(k);
        const float heq = w * (dr + rho * (eu * (3.0f + 4.5f * eu) + base));
        const float sk = (w * pr) * (3.0f * eF * (1.0f + 3.0f * eu) - 3.0f * uF);
        h[k] = h[k] + om * (heq - h[k]) + sk;
    }
}

// ---------------------------------------------------------------------------
// Storage formats.  Each exposes the element type, whether the stored value is
// shifted (f - w), and load/store to the compute type.
// ---------------------------------------------------------------------------
struct StoreF64 {
    using T = double; using C = double;
    static constexpr bool shifted = false;
    static constexpr int code = 0;
    __device__ static __forceinline__ C ld(const T *p, float) { return *p; }
    __device__ static __forceinline__ void st(T *p, C v, float) { *p = v; }
    __host__ __device__ static constexpr double init(int k) { return w3(k); }
};
struct StoreF32 {
    using T = float; using C = float;
    static constexpr bool shifted = true;
    static constexpr int code = 1;
    __device__ static __forceinline__ C ld(const T *p, float) { return *p; }
    __device__ static __forceinline__ void st(T *p, C v, float) { *p = v; }
    __host__ __device__ static constexpr double init(int) { return 0.0; }
};
struct StoreF16 {
    using T = __half; using C = float;
    static constexpr bool shifted = true;
    static constexpr int code = 2;
    // stored value = h * scale, scale a power of two chosen per solve
    __device__ static __forceinline__ C ld(const T *p, float inv_scale) { return __half2float(*p) * inv_scale; }
    __device__ static __forceinline__ void st(T *p, C v, float scale) { *p = __float2half_rn(v * scale); }
    __host__ __device__ static constexpr double init(int) { return 0.0; }
};
struct StoreBF16 {
    using T = __nv_bfloat16; using C = float;
    static constexpr bool shifted = true;
    static constexpr int code = 3;
    __device__ static __forceinline__ C ld(const T *p, float) { return __bfloat162float(*p); }
    __device__ static __forceinline__ void st(T *p, C v, float) { *p = __float2bfloat16_rn(v); }
    __host__ __device__ static constexpr double init(int) { return 0.0; }
};

}  // namespace lbm
