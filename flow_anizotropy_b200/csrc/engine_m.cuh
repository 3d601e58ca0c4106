// Moment-projected D3Q19 step for tau = 1.
//
// With tau = 1 the BGK update f* = g + (feq - g)/tau + S loses g: the
// post-collision populations of a voxel are feq_k(rho, u) + S_k(u), a function
// of its four moments (rho, u) alone (u the Guo velocity (j + F/2)/rho that the
// reference stores in U, V, W, LMB3d/lbm3d-perm.cpp:226-230).  A step of the
// reference is then exactly: for every pore voxel x, pull g_k(x) = f*_k(x - e_k)
// (or f*_opp(k)(x) across a solid link), evaluated from the moments of the
// source voxel, and sum the new moments.  The state is 4 numbers per pore voxel
// in two ping-pong buffers (step n writes buffer n & 1) instead of 19
// populations: 2 x 16 B per voxel-step in FP32 against 2 x 76 B.  Same
// operator, same boundary rule, same step sequence (step 1 is the moments of
// the initial state f = w: rho = 1, u = F/2); only the rounding differs, at
// the level of the storage precision.
#pragma once
#include "engine3d.cuh"

namespace lbm {

// State per pore voxel, written by the voxel's own update and read by its
// up to 19 receivers: (c1, d3, ux, uy, uz) with
//   c1 = drho - 1.5 rho u^2 - 3 pr u.F   (the direction-independent part),
//   d3 = 3 drho                          (3 rho - 3, kept shifted for precision),
// so a receiver evaluates a post-collision population without recomputing
// per-source invariants:
//   f*_k - w_k = w_k [c1 + eu (r3 + 1.5 r3 eu) + pr eF_k (3 + 9 eu)],
//   r3 = 3 + d3, eu = e_k . u, eF_k = e_k . F.
// A buffer holds `slots` records: a float4/double2x2 part (c1, ux, uy, uz)
// followed by the d3 part.
struct MomF32 {
    using C = float;
    static constexpr int code = 4;
    static constexpr size_t rec_bytes = 20;
    __device__ static __forceinline__ void ld(const void *buf, long long slots, unsigned i, C &c1, C &d3, C &x, C &y, C &z)
    {
        const float4 v = __ldg(static_cast<const float4 *>(buf) + i);
        c1 = v.x; x = v.y; y = v.z; z = v.w;
        d3 = __ldg(reinterpret_cast<const float *>(static_cast<const float4 *>(buf) + slots) + i);
    }
    __device__ static __forceinline__ void st(void *buf, long long slots, unsigned i, C c1, C d3, C x, C y, C z)
    {
        static_cast<float4 *>(buf)[i] = make_float4(c1, x, y, z);
        reinterpret_cast<float *>(static_cast<float4 *>(buf) + slots)[i] = d3;
    }
};

struct MomF64 {
    using C = double;
    static constexpr int code = 5;
    static constexpr size_t rec_bytes = 40;
    __device__ static __forceinline__ void ld(const void *buf, long long slots, unsigned i, C &c1, C &d3, C &x, C &y, C &z)
    {
        const double2 *b = static_cast<const double2 *>(buf);
        const double2 a = __ldg(b + 2 * (size_t)i), c = __ldg(b + 2 * (size_t)i + 1);
        c1 = a.x; x = a.y; y = c.x; z = c.y;
        d3 = __ldg(reinterpret_cast<const double *>(b + 2 * slots) + i);
    }
    __device__ static __forceinline__ void st(void *buf, long long slots, unsigned i, C c1, C d3, C x, C y, C z)
    {
        double2 *b = static_cast<double2 *>(buf);
        b[2 * (size_t)i] = make_double2(c1, x);
        b[2 * (size_t)i + 1] = make_double2(y, z);
        reinterpret_cast<double *>(b + 2 * slots)[i] = d3;
    }
};

// Record slots per buffer (padded so both parts stay 128-byte aligned).
inline long long mom_slots(long long nfluid) { return (nfluid + 31) / 32 * 32; }
inline long long mom_buffer_bytes(int prec, long long nfluid)
{
    return mom_slots(nfluid) * (prec == MomF32::code ? (long long)MomF32::rec_bytes : (long long)MomF64::rec_bytes);
}

// The record of a voxel with moments (drho, u).
template <class C>
__device__ __forceinline__ void make_record(C dr, C x, C y, C z, C Fx, C Fy, C Fz, C pr, C &c1, C &d3)
{
    const C rho = C(1) + dr;
    const C u2 = x * x + y * y + z * z;
    const C uF = x * Fx + y * Fy + z * Fz;
    c1 = dr - C(1.5) * rho * u2 - C(3) * pr * uF;
    d3 = C(3) * dr;
}

// f*_k - w_k of a source with record (c1, d3, u); sgn = -1 evaluates the
// opposite direction (bounce-back: f*_opp(k) of the receiving voxel itself).
template <int K, class C>
__device__ __forceinline__ C pop_rec(C c1, C d3, C ux, C uy, C uz, C sgn, C pr, C Fx, C Fy, C Fz)
{
    constexpr int cx = ex3(K), cy = ey3(K), cz = ez3(K);
    C eu = C(0), eF = C(0);
    if (cx) { eu += cx > 0 ? ux : -ux; eF += cx > 0 ? Fx : -Fx; }
    if (cy) { eu += cy > 0 ? uy : -uy; eF += cy > 0 ? Fy : -Fy; }
    if (cz) { eu += cz > 0 ? uz : -uz; eF += cz > 0 ? Fz : -Fz; }
    const C w = (C)w3(K);
    if constexpr (K == 0) return w * c1;
    eu *= sgn;
    eF *= sgn;
    const C r3 = C(3) + d3;
    return w * (c1 + eu * (r3 + C(1.5) * r3 * eu) + pr * eF * (C(3) + C(9) * eu));
}

template <int K, class MT>
__device__ __forceinline__ void gather_rec(const void *src, long long slots, unsigned i, const CNb &nb,
                                           typename MT::C pr, typename MT::C Fx, typename MT::C Fy,
                                           typename MT::C Fz, typename MT::C (&acc)[4])
{
    using C = typename MT::C;
    constexpr int o = opp3(K);
    // pull f*_k(x - e_k), or across a solid link f*_opp(k)(x): the same
    // formula on the voxel's own record with the direction reversed
    const bool bb = (nb.solid >> o) & 1u;
    const unsigned from = bb ? i : nb.idx[o];
    C c1, d3, x, y, z;
    MT::ld(src, slots, from, c1, d3, x, y, z);
    const C g = pop_rec<K, C>(c1, d3, x, y, z, bb ? C(-1) : C(1), pr, Fx, Fy, Fz);
    acc[0] += g;
    if (ex3(K)) acc[1] += ex3(K) > 0 ? g : -g;
    if (ey3(K)) acc[2] += ey3(K) > 0 ? g : -g;
    if (ez3(K)) acc[3] += ez3(K) > 0 ? g : -g;
}

template <class MT, int K>
struct GatherRec {
    __device__ __forceinline__ static void run(const void *src, long long slots, unsigned i, const CNb &nb,
                                               typename MT::C pr, typename MT::C Fx, typename MT::C Fy,
                                               typename MT::C Fz, typename MT::C (&acc)[4])
    {
        gather_rec<K, MT>(src, slots, i, nb, pr, Fx, Fy, Fz, acc);
        GatherRec<MT, K + 1>::run(src, slots, i, nb, pr, Fx, Fy, Fz, acc);
    }
};
template <class MT>
struct GatherRec<MT, Q3> {
    __device__ __forceinline__ static void run(const void *, long long, unsigned, const CNb &, typename MT::C,
                                               typename MT::C, typename MT::C, typename MT::C, typename MT::C (&)[4]) {}
};

template <class MT, int MINB>
__global__ void __launch_bounds__(TPB, MINB) stepm_kernel(const StepArgs a)
{
    using C = typename MT::C;
    __shared__ double sh[TPB / 32][3];
    const int nwork = a.nwork_dev ? *a.nwork_dev : a.nwork;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 item = a.work[w];
        const Solve3 &S = a.solves[item.x];
        const int phase = S.st->phase;
        if (phase >= PH_DONE) continue;
        const long long n = S.st->s_base + a.step + 1;
        const bool red = step_reduces(a, S.c, phase, n);
        char *base = static_cast<char *>(S.A);
        const long long slots = S.plane;
        const long long bytes = slots * (long long)MT::rec_bytes;
        void *dst = base + (n & 1ll) * bytes;
        const void *src = base + ((n + 1) & 1ll) * bytes;
        const C Fx = (C)S.P.F[0], Fy = (C)S.P.F[1], Fz = (C)S.P.F[2];
        const C pr = (C)S.P.pref;
        double acc3[3] = {0.0, 0.0, 0.0};
        const unsigned i = (unsigned)(item.y * TPB + threadIdx.x);
        if (i < (unsigned)S.nfluid) {
            C dr, ux, uy, uz;
            if (n == 1) {
                // moments of the initial state f = w: rho = 1, j = 0
                dr = C(0); ux = C(0.5) * Fx; uy = C(0.5) * Fy; uz = C(0.5) * Fz;
            } else {
                CNb nb;
                if (S.meta) {
                    meta_nbrs(S, i, __ldg(S.meta + i), __ldg(S.meta2 + i), nb);
                } else {
                    int x, y, z;
                    coords3(S, __ldg(S.fnode + i), x, y, z);
                    compact_nbrs(S, i, x, y, z, nb);
                }
                C c1, d3, ox, oy, oz;
                MT::ld(src, slots, i, c1, d3, ox, oy, oz);
                C acc[4] = {pop_rec<0, C>(c1, d3, ox, oy, oz, C(1), pr, Fx, Fy, Fz), C(0), C(0), C(0)};
                GatherRec<MT, 1>::run(src, slots, i, nb, pr, Fx, Fy, Fz, acc);
                dr = acc[0];
                const C rho = C(1) + dr;
                ux = (acc[1] + C(0.5) * Fx) / rho;
                uy = (acc[2] + C(0.5) * Fy) / rho;
                uz = (acc[3] + C(0.5) * Fz) / rho;
            }
            C c1n, d3n;
            make_record<C>(dr, ux, uy, uz, Fx, Fy, Fz, pr, c1n, d3n);
            MT::st(dst, slots, i, c1n, d3n, ux, uy, uz);
            acc3[0] = (double)ux; acc3[1] = (double)uy; acc3[2] = (double)uz;
        }
        if (red) finish_tile(S, item.y, n, acc3, sh, defer_slot(a));
    }
}

// Dense outputs from the records of step `done`: velocity (the reference's U,
// V, W) and/or the canonical post-collision populations f*_k = w_k + h_k.
template <class MT>
__global__ void canonm_kernel(const Solve3 S, long long done, double *f_out, float *u_out)
{
    using C = typename MT::C;
    const char *base = static_cast<const char *>(S.A);
    const long long slots = S.plane;
    const void *cur = base + (done & 1ll) * slots * (long long)MT::rec_bytes;
    const C Fx = (C)S.P.F[0], Fy = (C)S.P.F[1], Fz = (C)S.P.F[2];
    const C pr = (C)S.P.pref;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < (unsigned)S.nfluid;
         i += gridDim.x * blockDim.x) {
        const unsigned node = S.fnode[i];
        if (done == 0) {
            if (u_out) {
                u_out[3 * (size_t)node] = (float)(C(0.5) * Fx);
                u_out[3 * (size_t)node + 1] = (float)(C(0.5) * Fy);
                u_out[3 * (size_t)node + 2] = (float)(C(0.5) * Fz);
            }
            if (f_out)
                for (int k = 0; k < Q3; ++k) f_out[(size_t)node * Q3 + k] = w3(k);
            continue;
        }
        C c1, d3, x, y, z;
        MT::ld(cur, slots, i, c1, d3, x, y, z);
        if (u_out) {
            u_out[3 * (size_t)node] = (float)x;
            u_out[3 * (size_t)node + 1] = (float)y;
            u_out[3 * (size_t)node + 2] = (float)z;
        }
        if (f_out) {
            double f[Q3];
#define LBM_POP(K) f[K] = w3(K) + (double)pop_rec<K, C>(c1, d3, x, y, z, C(1), pr, Fx, Fy, Fz);
            LBM_POP(0) LBM_POP(1) LBM_POP(2) LBM_POP(3) LBM_POP(4) LBM_POP(5) LBM_POP(6) LBM_POP(7) LBM_POP(8)
            LBM_POP(9) LBM_POP(10) LBM_POP(11) LBM_POP(12) LBM_POP(13) LBM_POP(14) LBM_POP(15) LBM_POP(16)
            LBM_POP(17) LBM_POP(18)
#undef LBM_POP
            for (int k = 0; k < Q3; ++k) f_out[(size_t)node * Q3 + k] = f[k];
        }
    }
}

constexpr int NVAR_M = 3;
__host__ __device__ constexpr int variant_m_minb(int v) { return v == 0 ? 3 : v == 1 ? 4 : 2; }

cudaError_t launch_stepm(int prec, int variant, dim3 grid, cudaStream_t s, const StepArgs &a);
cudaError_t launch_canonm(int prec, const Solve3 &S, long long done, double *f, float *u, cudaStream_t s);
int max_blocks_stepm(int prec, int variant);

}  // namespace lbm
