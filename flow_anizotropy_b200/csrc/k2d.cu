// D2Q9 kernels.  Compiled with -fmad=false: every float operation of the
// collision rounds as in the reference build (plain -O3, no FMA), so a step
// is bit-identical to LMB2d/lbm.cpp:563-632.
#include "engine2d.cuh"

namespace lbm {

__global__ void __launch_bounds__(TPB, 4) step2d_kernel(const StepArgs2 a)
{
    __shared__ double sh[TPB / 32][3];
    for (int w = blockIdx.x; w < a.nwork; w += gridDim.x) {
        const int2 item = a.work[w];
        const Solve2 &S = a.solves[item.x];
        State2 &st = *S.st;
        if (st.phase >= PH_DONE) continue;
        const long long n = st.s_base + a.step + 1;
        const bool neighbour = (n & 1ll) == 0;
        const bool red = reduce2(S.c, st, n);
        const bool wsnap = snap2(S.c, st, n);
        const bool wlast = last2(S.c, st, n);
        float *__restrict__ A = S.A;
        const unsigned P = S.plane;
        double acc[2] = {0.0, 0.0};
        const int nd = item.y * TPB + threadIdx.x;
        if (nd < S.nn) {
            const int y = S.dvx.div(nd);
            const int x = nd - y * S.nx;
            const int nx = S.nx, ny = S.ny;
            const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
            const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
            const int X[3] = {xm, x, xp};
            const int Yr[3] = {ym, y, yp};
            const uint32_t sol = S.nbm[nd];
            int idx[Q2];
#pragma unroll
            for (int k = 0; k < Q2; ++k) idx[k] = Yr[ey2(k) + 1] * nx + X[ex2(k) + 1];
            float U = 0.0f, V = 0.0f;
            if (!(sol & 1u)) {
                float g[Q2];
                if (!neighbour) {
#pragma unroll
                    for (int k = 0; k < Q2; ++k) g[k] = A[k * P + (unsigned)nd];
                } else {
                    g[0] = A[(unsigned)nd];
#pragma unroll
                    for (int k = 1; k < Q2; ++k) {
                        const int o = inv2(k);
                        g[k] = ((sol >> o) & 1u) ? A[k * P + (unsigned)nd] : A[o * P + (unsigned)idx[o]];
                    }
                }
                collide2(g, S.fx, S.fy, S.tau, U, V);
                if (!neighbour) {
#pragma unroll
                    for (int k = 0; k < Q2; ++k) A[inv2(k) * P + (unsigned)nd] = g[k];
                } else {
                    A[(unsigned)nd] = g[0];
#pragma unroll
                    for (int k = 1; k < Q2; ++k) {
                        if ((sol >> k) & 1u) A[inv2(k) * P + (unsigned)nd] = g[k];
                        else A[k * P + (unsigned)idx[k]] = g[k];
                    }
                }
                acc[0] = (double)U; acc[1] = (double)V;
            }
            if (wsnap) { S.snap[2 * nd] = U; S.snap[2 * nd + 1] = V; }
            if (wlast) { S.last[2 * nd] = U; S.last[2 * nd + 1] = V; }
        }
        if (red) finish_tile2(S, item.y, n, acc, sh);
    }
}

__global__ void nbmask2d_kernel(const uint32_t *mask, int nx, int ny, int wpr, uint16_t *nbm)
{
    const int nn = nx * ny;
    for (int nd = blockIdx.x * blockDim.x + threadIdx.x; nd < nn; nd += gridDim.x * blockDim.x) {
        const int y = nd / nx, x = nd - y * nx;
        const int X[3] = {x == 0 ? nx - 1 : x - 1, x, x == nx - 1 ? 0 : x + 1};
        const int Yr[3] = {y == 0 ? ny - 1 : y - 1, y, y == ny - 1 ? 0 : y + 1};
        uint32_t sol = 0;
#pragma unroll
        for (int k = 0; k < Q2; ++k) {
            const int yy = Yr[ey2(k) + 1], xx = X[ex2(k) + 1];
            sol |= (uint32_t)mbit(mask + (size_t)yy * wpr, xx) << k;
        }
        nbm[nd] = (uint16_t)sol;
    }
}

cudaError_t launch_nbmask2d(const uint32_t *mask, int nx, int ny, uint16_t *nbm, cudaStream_t s)
{
    const int nn = nx * ny;
    nbmask2d_kernel<<<(nn + 255) / 256 < 1184 ? (nn + 255) / 256 : 1184, 256, 0, s>>>(mask, nx, ny, (nx + 31) / 32, nbm);
    return cudaGetLastError();
}

__global__ void init2d_kernel(float *A, unsigned plane, int nn)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < Q2; ++k) A[k * plane + (unsigned)i] = w2(k);
}

// Populations the next step will read, in the reference's pre-collision
// (post-transport) form: after a local step A[opp k][x] holds f*_k(x), which
// streams to x + e_k; after a neighbour step A[k][x] already holds them.
__global__ void canon2d_kernel(const Solve2 S, long long done, float *f_out)
{
    for (int nd = blockIdx.x * blockDim.x + threadIdx.x; nd < S.nn; nd += gridDim.x * blockDim.x) {
        const int y = S.dvx.div(nd);
        const int x = nd - y * S.nx;
        if (mbit(S.mask + (size_t)y * S.wpr, x)) {
            for (int k = 0; k < Q2; ++k) f_out[nd * Q2 + k] = 0.0f;
            continue;
        }
        for (int k = 0; k < Q2; ++k) {
            float v;
            if (!(done & 1ll)) {
                v = S.A[k * S.plane + (unsigned)nd];
            } else {
                // pre-collision f_k(x) = f*_k(x - e_k), or f*_inv(k)(x) if x - e_k is solid
                const int sx = (x - ex2(k) + S.nx) % S.nx, sy = (y - ey2(k) + S.ny) % S.ny;
                const int o = inv2(k);
                if (mbit(S.mask + (size_t)sy * S.wpr, sx)) v = S.A[k * S.plane + (unsigned)nd];
                else v = S.A[o * S.plane + (unsigned)(sy * S.nx + sx)];
            }
            f_out[nd * Q2 + k] = v;
        }
    }
}

// field_residual (LMB2d/lbm.cpp:217-229): out[0] = sum (du^2 + dv^2), out[1] = sum (u^2 + v^2)
__global__ void fieldres2d_kernel(const float *snap, const float *last, int nn, double *out)
{
    __shared__ double sh[TPB / 32][3];
    double v[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        const float u = last[2 * i], w = last[2 * i + 1];
        const double du = u - snap[2 * i];
        const double dv = w - snap[2 * i + 1];
        v[0] += du * du + dv * dv;
        v[1] += (double)u * u + (double)w * w;
    }
    block_sum2(v, sh);
    if (threadIdx.x == 0) { atomicAdd(out, v[0]); atomicAdd(out + 1, v[1]); }
}

// s_base += steps for every solve of a launch list (the step numbers of a
// replayed chunk of step launches are relative to s_base)
__global__ void advance2d_kernel(const Solve2 *solves, int nsolves, long long steps)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < nsolves) solves[j].st->s_base += steps;
}

cudaError_t launch_advance2d(const Solve2 *solves, int nsolves, long long steps, cudaStream_t s)
{
    advance2d_kernel<<<(nsolves + 127) / 128, 128, 0, s>>>(solves, nsolves, steps);
    return cudaGetLastError();
}

cudaError_t launch_step2d(dim3 grid, cudaStream_t s, const StepArgs2 &a)
{
    step2d_kernel<<<grid, TPB, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace lbm
