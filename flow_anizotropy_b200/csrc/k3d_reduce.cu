// Deferred flux reduction of the 3D step kernels (StepArgs::defer): after a
// run of launches, one block per (solve, launch) sums the tile partials a
// reduction step left in its slot, in the order the last tile of an
// immediate reduction uses (thread t takes tiles t, t + TPB, ..., then the
// fixed-order block sum), and one thread per solve runs the controller over
// the steps in order.  So a deferred solve takes the same decisions and
// reports the same bits as one reduced at every step; only the work moves
// out of the step kernels (LMB3d/lbm3d-perm.cpp:298-303 is the reduction,
// :320-398 the controller).
#include "engine3d.cuh"

namespace lbm {

__global__ void __launch_bounds__(TPB) reduce3d_kernel(const Solve3 *solves, long long step0, double *qbuf)
{
    __shared__ double sh[TPB / 32][3];
    const int j = blockIdx.x, r = blockIdx.y;
    const Solve3 &S = solves[j];
    double *out = qbuf + 4ll * ((long long)j * DEFER_SLOTS + r);
    const int phase = S.st->phase;
    const long long rel = step0 + r;
    const long long n = S.st->s_base + rel + 1;
    if (phase >= PH_DONE || !needs_reduction(S.c, phase, n)) {
        if (threadIdx.x == 0) out[3] = 0.0;
        return;
    }
    const double *p = S.partials + 3ll * (long long)(rel & (DEFER_SLOTS - 1)) * S.ntiles;
    double v[3] = {0.0, 0.0, 0.0};
    for (int t = threadIdx.x; t < S.ntiles; t += TPB) {
        v[0] += p[3ll * t];
        v[1] += p[3ll * t + 1];
        v[2] += p[3ll * t + 2];
    }
    block_sum3<TPB>(v, sh);
    if (threadIdx.x == 0) {
        const double inv = (double)S.nn;
        out[0] = v[0] / inv;
        out[1] = v[1] / inv;
        out[2] = v[2] / inv;
        out[3] = 1.0;
    }
}

__global__ void control3d_kernel(const Solve3 *solves, int nsolves, long long step0, int nsteps, const double *qbuf)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nsolves) return;
    const Solve3 &S = solves[j];
    State3 &st = *S.st;
    for (int r = 0; r < nsteps; ++r) {
        const double *q = qbuf + 4ll * ((long long)j * DEFER_SLOTS + r);
        if (q[3] == 0.0) continue;
        if (st.phase >= PH_DONE) break;
        controller3(S.c, st, st.s_base + step0 + r + 1, q);
    }
}

cudaError_t launch_deferred3d(const Solve3 *solves, int nsolves, long long step0, int nsteps, double *qbuf,
                              cudaStream_t s)
{
    if (nsolves <= 0 || nsteps <= 0) return cudaSuccess;
    if (nsteps > DEFER_SLOTS) return cudaErrorInvalidValue;
    reduce3d_kernel<<<dim3(nsolves, nsteps), TPB, 0, s>>>(solves, step0, qbuf);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    control3d_kernel<<<(nsolves + 127) / 128, 128, 0, s>>>(solves, nsolves, step0, nsteps, qbuf);
    return cudaGetLastError();
}

}  // namespace lbm
