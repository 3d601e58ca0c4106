// D2Q9 permeability solve on the device (the 2D reference solver,
// LMB2d/lbm.cpp:563-632 and LMB2d/main.cpp:99-235, at a runtime cell size).
//
// Same in-place AA layout as the D3Q19 engine: A[k][n], n = y*nx + x.  The
// reference's df[2][LX][LY][9] double buffer with push streaming and its
// parity flip (LMB2d/lbm.cpp:712-726) become one buffer: odd steps read and
// write a node's own slots, even steps pull from and push to the neighbours.
// Populations are raw FP32 as in the reference; the operator is compiled
// without FMA contraction and keeps the reference's operation order, so each
// step is bit-identical to it.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "engine3d.cuh"

namespace lbm {

constexpr int Q2 = 9;
// LMB2d/lbm.cpp:67-70
__host__ __device__ constexpr int ex2(int k) { return (k == 1 || k == 5 || k == 8) ? 1 : (k == 3 || k == 6 || k == 7) ? -1 : 0; }
__host__ __device__ constexpr int ey2(int k) { return (k == 2 || k == 5 || k == 6) ? 1 : (k == 4 || k == 7 || k == 8) ? -1 : 0; }
__host__ __device__ constexpr int inv2(int k) { return k == 0 ? 0 : (k <= 4 ? ((k + 1) & 3) + 1 : ((k - 3) & 3) + 5); }
__host__ __device__ constexpr float w2(int k) { return k == 0 ? 4.0f / 9.0f : (k <= 4 ? 1.0f / 9.0f : 1.0f / 36.0f); }

struct Ctl2 {              // LMB2d/main.cpp:64-79
    double eps, qfloor, ksigma;
    long long lag, min_steps, max_steps, avg_steps, avg_sample;
    int hold;
};

struct State2 {
    long long s_base;
    int phase, hold, have_prev, converged, status;
    unsigned counter;
    double pm[2], pse[2];
    double bs[2], bss[2];
    long long bn;
    long long avg_start;   // step at which phase 1 ended
    double sum[2], sumsq[2];
    long long n_avg;
    double q[2], se[2];
    long long steps;
    int snap_valid;        // U/V of the phase-1 end are in `snap`
};

struct Solve2 {
    float *A;
    unsigned plane;
    const uint32_t *mask;
    const uint16_t *nbm;   // per cell: bit k set if the cell at offset e_k is solid (k = 0: itself)
    int nx, ny, wpr;
    int nn;
    int ntiles;
    FastDiv dvx;
    float fx, fy, tau;     // as the reference's float globals (LMB2d/lbm.cpp:82-86)
    Ctl2 c;
    double *partials;      // ntiles * 2
    State2 *st;
    float *snap;           // nn * 2: U,V written on candidate phase-1 end steps
    float *last;           // nn * 2: U,V of the final step
};

struct StepArgs2 {
    const Solve2 *solves;
    const int2 *work;
    int nwork;
    long long step;
};

// Steps on which the flux is reduced, and on which the U,V field is kept.
__device__ __forceinline__ bool reduce2(const Ctl2 &c, const State2 &st, long long n)
{
    if (st.phase == PH_RUN)
        return n % c.avg_sample == 0 || n % c.lag == 0 || n == c.max_steps;
    const long long t = n - st.avg_start;
    return t % c.avg_sample == 0 || t == c.avg_steps;
}
__device__ __forceinline__ bool snap2(const Ctl2 &c, const State2 &st, long long n)
{
    return st.phase == PH_RUN && (n % c.lag == 0 || n == c.max_steps);
}
__device__ __forceinline__ bool last2(const Ctl2 &c, const State2 &st, long long n)
{
    if (st.phase == PH_RUN) return c.avg_steps <= 0 && (n % c.lag == 0 || n == c.max_steps);
    return n - st.avg_start == c.avg_steps;
}

// LMB2d/main.cpp:99-235, driven by the flux of step n (valid only when
// reduce2() held for step n).
__device__ inline void controller2(const Ctl2 &c, State2 &st, long long n, const double q[2])
{
    if (st.phase == PH_RUN) {
        if (n % c.avg_sample == 0) {
            if (!isfinite(q[0]) || !isfinite(q[1])) { st.status = 2; st.phase = PH_ERR; st.steps = n; return; }
            st.bs[0] += q[0]; st.bss[0] += q[0] * q[0];
            st.bs[1] += q[1]; st.bss[1] += q[1] * q[1];
            st.bn++;
        }
        bool stop = false;
        if (n % c.lag == 0 && st.bn >= 2) {
            const double bn = (double)st.bn;
            const double mx = st.bs[0] / bn, my = st.bs[1] / bn;
            const double vx = (st.bss[0] - bn * mx * mx) / (bn - 1);
            const double vy = (st.bss[1] - bn * my * my) / (bn - 1);
            const double sex = sqrt(fmax(vx, 0.0) / bn);
            const double sey = sqrt(fmax(vy, 0.0) / bn);
            if (st.have_prev) {
                const double qmag = sqrt(mx * mx + my * my);
                const double flo = c.qfloor * qmag;
                const double dx = fabs(mx - st.pm[0]), dy = fabs(my - st.pm[1]);
                const double tolx = fmax(c.eps * fmax(fabs(mx), flo), c.ksigma * sqrt(sex * sex + st.pse[0] * st.pse[0]));
                const double toly = fmax(c.eps * fmax(fabs(my), flo), c.ksigma * sqrt(sey * sey + st.pse[1] * st.pse[1]));
                if (n >= c.min_steps && dx < tolx && dy < toly) st.hold++;
                else st.hold = 0;
            }
            st.pm[0] = mx; st.pm[1] = my; st.pse[0] = sex; st.pse[1] = sey; st.have_prev = 1;
            st.bs[0] = st.bs[1] = st.bss[0] = st.bss[1] = 0.0;
            st.bn = 0;
            stop = st.hold >= c.hold;
        }
        if (stop || n >= c.max_steps) {
            st.converged = st.hold >= c.hold ? 1 : 0;
            st.avg_start = n;
            st.snap_valid = 1;
            if (c.avg_steps < c.avg_sample) {
                // no sample will be taken: q is the volume average of the last step
                if (c.avg_steps <= 0) {
                    st.q[0] = q[0]; st.q[1] = q[1]; st.se[0] = st.se[1] = 0.0;
                    st.steps = n; st.phase = PH_DONE;
                    return;
                }
            }
            st.phase = PH_AVG;
        }
        return;
    }
    if (st.phase == PH_AVG) {
        const long long t = n - st.avg_start;
        if (t % c.avg_sample == 0) {
            if (!isfinite(q[0]) || !isfinite(q[1])) { st.status = 2; st.phase = PH_ERR; st.steps = n; return; }
            st.sum[0] += q[0]; st.sumsq[0] += q[0] * q[0];
            st.sum[1] += q[1]; st.sumsq[1] += q[1] * q[1];
            st.n_avg++;
        }
        if (t == c.avg_steps) {
            if (st.n_avg == 0) {
                st.q[0] = q[0]; st.q[1] = q[1]; st.se[0] = st.se[1] = 0.0;
            } else {
                const double nn = (double)st.n_avg;
                for (int k = 0; k < 2; ++k) {
                    st.q[k] = st.sum[k] / nn;
                    st.se[k] = 0.0;
                    if (st.n_avg > 1) {
                        const double v = (st.sumsq[k] - nn * st.q[k] * st.q[k]) / (nn - 1);
                        st.se[k] = sqrt(fmax(v, 0.0) / nn);
                    }
                }
            }
            st.steps = n;
            st.phase = PH_DONE;
        }
    }
}

__device__ __forceinline__ void block_sum2(double (&v)[2], double (*sh)[3])
{
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { sh[wid][0] = v[0]; sh[wid][1] = v[1]; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a0 = 0.0, a1 = 0.0;
        for (int w = 0; w < TPB / 32; ++w) { a0 += sh[w][0]; a1 += sh[w][1]; }
        v[0] = a0; v[1] = a1;
    }
    __syncthreads();
}

__device__ __forceinline__ void finish_tile2(const Solve2 &S, int tile, long long n,
                                             double (&acc)[2], double (*sh)[3])
{
    __shared__ int s_last;
    block_sum2(acc, sh);
    if (threadIdx.x == 0) {
        double *p = S.partials + 2ll * tile;
        p[0] = acc[0]; p[1] = acc[1];
        __threadfence();
        const unsigned prev = atomicAdd(&S.st->counter, 1u);
        s_last = (prev == (unsigned)S.ntiles - 1u);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double v[2] = {0.0, 0.0};
    for (int t = threadIdx.x; t < S.ntiles; t += TPB) {
        v[0] += __ldcg(S.partials + 2ll * t);
        v[1] += __ldcg(S.partials + 2ll * t + 1);
    }
    block_sum2(v, sh);
    if (threadIdx.x == 0) {
        State2 &st = *S.st;
        st.counter = 0u;
        // LMB2d/lbm.cpp:188-199: q_i = sum(u_i) / (L * L0^2), L0 = 4
        const double q[2] = {v[0] / ((double)S.nx * 4.0 * 4.0), v[1] / ((double)S.ny * 4.0 * 4.0)};
        controller2(S.c, st, n, q);
    }
}

// macro + collision of one fluid node (LMB2d/lbm.cpp:563-612), in place on g;
// returns the raw-moment velocity the reference stores in U, V.
__device__ __forceinline__ void collide2(float (&g)[Q2], float fx, float fy, float tau,
                                         float &U, float &V)
{
    float rho = 0.0f;
#pragma unroll
    for (int k = 0; k < Q2; ++k) rho = rho + g[k];
    float ux = 0.0f, uy = 0.0f;
#pragma unroll
    for (int k = 0; k < Q2; ++k) {
        if (ex2(k) == 1) ux = ux + g[k]; else if (ex2(k) == -1) ux = ux - g[k];
        if (ey2(k) == 1) uy = uy + g[k]; else if (ey2(k) == -1) uy = uy - g[k];
    }
    ux = ux / rho;
    uy = uy / rho;
    U = ux; V = uy;
    ux = ux + fx * tau / rho;
    uy = uy + fy * tau / rho;
    const float usq = ux * ux + uy * uy;
    const float itau = 1.0f / tau;
#pragma unroll
    for (int k = 0; k < Q2; ++k) {
        const float eu = (float)ex2(k) * ux + (float)ey2(k) * uy;
        const float feq = (w2(k) * rho) * (((1.0f - 1.5f * usq) + 3.0f * eu) + (4.5f * eu) * eu);
        g[k] = g[k] - itau * (g[k] - feq);
    }
}

__global__ void __launch_bounds__(TPB, 4) step2d_kernel(const StepArgs2 a);
__global__ void init2d_kernel(float *A, unsigned plane, int nn);
// Neighbour solid bits of every cell (Solve2::nbm) from the bit mask.
__global__ void nbmask2d_kernel(const uint32_t *mask, int nx, int ny, int wpr, uint16_t *nbm);
__global__ void canon2d_kernel(const Solve2 S, long long done, float *f_out);
__global__ void fieldres2d_kernel(const float *snap, const float *last, int nn, double *out);

cudaError_t launch_step2d(dim3 grid, cudaStream_t s, const StepArgs2 &a);
cudaError_t launch_advance2d(const Solve2 *solves, int nsolves, long long steps, cudaStream_t s);
cudaError_t launch_nbmask2d(const uint32_t *mask, int nx, int ny, uint16_t *nbm, cudaStream_t s);

}  // namespace lbm
