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

struct MomF32 {
    using T = float4;
    using C = float;
    static constexpr int code = 4;
    __device__ static __forceinline__ void ld(const T *b, unsigned i, C &d, C &x, C &y, C &z)
    {
        const float4 v = __ldg(b + i);
        d = v.x; x = v.y; y = v.z; z = v.w;
    }
    __device__ static __forceinline__ void st(T *b, unsigned i, C d, C x, C y, C z)
    {
        b[i] = make_float4(d, x, y, z);
    }
};

struct MomF64 {
    using T = double2;       // two double2 per voxel: (drho, ux), (uy, uz)
    using C = double;
    static constexpr int code = 5;
    __device__ static __forceinline__ void ld(const T *b, unsigned i, C &d, C &x, C &y, C &z)
    {
        const double2 a = __ldg(b + 2 * (size_t)i), c = __ldg(b + 2 * (size_t)i + 1);
        d = a.x; x = a.y; y = c.x; z = c.y;
    }
    __device__ static __forceinline__ void st(T *b, unsigned i, C d, C x, C y, C z)
    {
        b[2 * (size_t)i] = make_double2(d, x);
        b[2 * (size_t)i + 1] = make_double2(y, z);
    }
};

// Elements of T per buffer (padded to 128 B); the two buffers are contiguous.
inline long long mom_buffer_elems(int prec, long long nfluid)
{
    const long long per = prec == MomF32::code ? 1 : 2;
    return (nfluid * per + 7) / 8 * 8;
}

// Post-collision shifted population k (f*_k - w_k) of a voxel with moments
// (dr, u): w_k [c1 + eu (3 rho + 4.5 rho eu) + pr eF_k (3 + 9 eu)], with
// c1 = dr - 1.5 rho u^2 - 3 pr u.F.  Accumulated straight into the moments of
// the receiving voxel.
template <class C>
struct SrcM {
    C c1, r3, r45, ux, uy, uz;
    __device__ __forceinline__ void set(C dr, C x, C y, C z, C Fx, C Fy, C Fz, C pr)
    {
        const C rho = C(1) + dr;
        const C u2 = x * x + y * y + z * z;
        const C uF = x * Fx + y * Fy + z * Fz;
        c1 = dr - C(1.5) * rho * u2 - C(3) * pr * uF;
        r3 = C(3) * rho;
        r45 = C(4.5) * rho;
        ux = x; uy = y; uz = z;
    }
};

template <int K, class C>
__device__ __forceinline__ C pop_from(const SrcM<C> &s, C pr, C Fx, C Fy, C Fz)
{
    constexpr int cx = ex3(K), cy = ey3(K), cz = ez3(K);
    C eu = C(0), eF = C(0);
    if (cx) { eu += cx > 0 ? s.ux : -s.ux; eF += cx > 0 ? Fx : -Fx; }
    if (cy) { eu += cy > 0 ? s.uy : -s.uy; eF += cy > 0 ? Fy : -Fy; }
    if (cz) { eu += cz > 0 ? s.uz : -s.uz; eF += cz > 0 ? Fz : -Fz; }
    const C w = (C)w3(K);
    if constexpr (K == 0) return w * s.c1;
    return w * (s.c1 + eu * (s.r3 + s.r45 * eu) + pr * eF * (C(3) + C(9) * eu));
}

template <int K, class MT>
__device__ __forceinline__ void gather_one(const typename MT::T *__restrict__ src, unsigned i, const CNb &nb,
                                           const SrcM<typename MT::C> &own, typename MT::C pr,
                                           typename MT::C Fx, typename MT::C Fy, typename MT::C Fz,
                                           typename MT::C (&acc)[4])
{
    using C = typename MT::C;
    constexpr int o = opp3(K);
    C g;
    if ((nb.solid >> o) & 1u) {
        g = pop_from<o, C>(own, pr, Fx, Fy, Fz);      // bounce back: f*_opp(k)(x)
    } else {
        C d, x, y, z;
        MT::ld(src, nb.idx[o], d, x, y, z);
        SrcM<C> s;
        s.set(d, x, y, z, Fx, Fy, Fz, pr);
        g = pop_from<K, C>(s, pr, Fx, Fy, Fz);        // pull f*_k(x - e_k)
    }
    acc[0] += g;
    if (ex3(K)) acc[1] += ex3(K) > 0 ? g : -g;
    if (ey3(K)) acc[2] += ey3(K) > 0 ? g : -g;
    if (ez3(K)) acc[3] += ez3(K) > 0 ? g : -g;
}

template <class MT, int K>
struct GatherAll {
    __device__ __forceinline__ static void run(const typename MT::T *src, unsigned i, const CNb &nb,
                                               const SrcM<typename MT::C> &own, typename MT::C pr,
                                               typename MT::C Fx, typename MT::C Fy, typename MT::C Fz,
                                               typename MT::C (&acc)[4])
    {
        gather_one<K, MT>(src, i, nb, own, pr, Fx, Fy, Fz, acc);
        GatherAll<MT, K + 1>::run(src, i, nb, own, pr, Fx, Fy, Fz, acc);
    }
};
template <class MT>
struct GatherAll<MT, Q3> {
    __device__ __forceinline__ static void run(const typename MT::T *, unsigned, const CNb &,
                                               const SrcM<typename MT::C> &, typename MT::C, typename MT::C,
                                               typename MT::C, typename MT::C, typename MT::C (&)[4]) {}
};

template <class MT, int MINB>
__global__ void __launch_bounds__(TPB, MINB) stepm_kernel(const StepArgs a)
{
    using T = typename MT::T;
    using C = typename MT::C;
    __shared__ double sh[TPB / 32][3];
    const int nwork = a.nwork_dev ? *a.nwork_dev : a.nwork;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 item = a.work[w];
        const Solve3 &S = a.solves[item.x];
        const int phase = S.st->phase;
        if (phase >= PH_DONE) continue;
        const long long n = S.st->s_base + a.step + 1;
        const bool red = needs_reduction(S.c, phase, n);
        T *base = static_cast<T *>(S.A);
        const long long per = S.plane;                 // elements of T per buffer
        T *dst = base + (n & 1ll) * per;
        const T *src = base + ((n + 1) & 1ll) * per;
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
                C od, ox, oy, oz;
                MT::ld(src, i, od, ox, oy, oz);
                SrcM<C> own;
                own.set(od, ox, oy, oz, Fx, Fy, Fz, pr);
                C acc[4] = {C(0), C(0), C(0), C(0)};
                acc[0] = pop_from<0, C>(own, pr, Fx, Fy, Fz);
                GatherAll<MT, 1>::run(src, i, nb, own, pr, Fx, Fy, Fz, acc);
                dr = acc[0];
                const C rho = C(1) + dr;
                ux = (acc[1] + C(0.5) * Fx) / rho;
                uy = (acc[2] + C(0.5) * Fy) / rho;
                uz = (acc[3] + C(0.5) * Fz) / rho;
            }
            MT::st(dst, i, dr, ux, uy, uz);
            acc3[0] = (double)ux; acc3[1] = (double)uy; acc3[2] = (double)uz;
        }
        if (red) finish_tile(S, item.y, n, acc3, sh);
    }
}

// Dense outputs from the moments of step `done`: velocity (the reference's U,
// V, W) and/or the canonical post-collision populations f*_k = w_k + h_k.
template <class MT>
__global__ void canonm_kernel(const Solve3 S, long long done, double *f_out, float *u_out)
{
    using T = typename MT::T;
    using C = typename MT::C;
    const T *base = static_cast<const T *>(S.A);
    const T *cur = base + (done & 1ll) * S.plane;
    const C Fx = (C)S.P.F[0], Fy = (C)S.P.F[1], Fz = (C)S.P.F[2];
    const C pr = (C)S.P.pref;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < (unsigned)S.nfluid;
         i += gridDim.x * blockDim.x) {
        const unsigned node = S.fnode[i];
        C d, x, y, z;
        if (done == 0) { d = C(0); x = C(0); y = C(0); z = C(0); }
        else MT::ld(cur, i, d, x, y, z);
        if (u_out) {
            u_out[3 * (size_t)node] = (float)(done == 0 ? C(0.5) * Fx : x);
            u_out[3 * (size_t)node + 1] = (float)(done == 0 ? C(0.5) * Fy : y);
            u_out[3 * (size_t)node + 2] = (float)(done == 0 ? C(0.5) * Fz : z);
        }
        if (f_out) {
            if (done == 0) {
                for (int k = 0; k < Q3; ++k) f_out[(size_t)node * Q3 + k] = w3(k);
                continue;
            }
            SrcM<C> s;
            s.set(d, x, y, z, Fx, Fy, Fz, pr);
            double f[Q3];
            f[0] = w3(0) + (double)pop_from<0, C>(s, pr, Fx, Fy, Fz);
            f[1] = w3(1) + (double)pop_from<1, C>(s, pr, Fx, Fy, Fz);
            f[2] = w3(2) + (double)pop_from<2, C>(s, pr, Fx, Fy, Fz);
            f[3] = w3(3) + (double)pop_from<3, C>(s, pr, Fx, Fy, Fz);
            f[4] = w3(4) + (double)pop_from<4, C>(s, pr, Fx, Fy, Fz);
            f[5] = w3(5) + (double)pop_from<5, C>(s, pr, Fx, Fy, Fz);
            f[6] = w3(6) + (double)pop_from<6, C>(s, pr, Fx, Fy, Fz);
            f[7] = w3(7) + (double)pop_from<7, C>(s, pr, Fx, Fy, Fz);
            f[8] = w3(8) + (double)pop_from<8, C>(s, pr, Fx, Fy, Fz);
            f[9] = w3(9) + (double)pop_from<9, C>(s, pr, Fx, Fy, Fz);
            f[10] = w3(10) + (double)pop_from<10, C>(s, pr, Fx, Fy, Fz);
            f[11] = w3(11) + (double)pop_from<11, C>(s, pr, Fx, Fy, Fz);
            f[12] = w3(12) + (double)pop_from<12, C>(s, pr, Fx, Fy, Fz);
            f[13] = w3(13) + (double)pop_from<13, C>(s, pr, Fx, Fy, Fz);
            f[14] = w3(14) + (double)pop_from<14, C>(s, pr, Fx, Fy, Fz);
            f[15] = w3(15) + (double)pop_from<15, C>(s, pr, Fx, Fy, Fz);
            f[16] = w3(16) + (double)pop_from<16, C>(s, pr, Fx, Fy, Fz);
            f[17] = w3(17) + (double)pop_from<17, C>(s, pr, Fx, Fy, Fz);
            f[18] = w3(18) + (double)pop_from<18, C>(s, pr, Fx, Fy, Fz);
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
