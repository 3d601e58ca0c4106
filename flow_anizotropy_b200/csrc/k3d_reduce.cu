// Deferred flux reduction of the 3D step kernels (StepArgs::defer): after a
// run of at most DEFER_SLOTS launches, one block per (solve, launch) sums the
// tile partials a reduction step left in its slot, in the order the last
// tile of an immediate reduction uses (thread t takes tiles t, t + TPB, ...,
// then the fixed-order block sum), and one block per solve runs the
// controller over the steps in order.  So a deferred solve takes the same
// decisions and reports the same bits as one reduced at every step; only the
// work moves out of the step kernels (LMB3d/lbm3d-perm.cpp:298-303 is the
// reduction, :320-398 the controller).
#include "engine3d.cuh"

namespace lbm {

// mode 1: the solves keep their phase through the pass (the single-solve
// loop splits runs where the controller can act); mode 2: a phase can change
// inside the pass, and every step the step kernels may have reduced is summed
// (deferred_reduces).
__global__ void __launch_bounds__(TPB) reduce3d_kernel(const Solve3 *solves, long long step0, double *qbuf, int mode)
{
    __shared__ double sh[TPB / 32][3];
    const int j = blockIdx.x, r = blockIdx.y;
    const Solve3 &S = solves[j];
    double *out = qbuf + 4ll * ((long long)j * DEFER_SLOTS + r);
    const int phase = S.st->phase;
    const long long rel = step0 + r;
    const long long s_base = S.st->s_base;
    const long long n = s_base + rel + 1;
    const long long pass_start = s_base + (step0 & ~(long long)(DEFER_SLOTS - 1));
    if (phase >= PH_DONE || !deferred_reduces(S.c, phase, n, pass_start, mode)) {
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

// One block per solve: the pass's fluxes come to shared memory together,
// then one thread runs the controller over the steps in order on a shared
// copy of the state (the controller acts on a step when the phase it has
// reached by then needs that step).
__global__ void __launch_bounds__(DEFER_SLOTS) control3d_kernel(const Solve3 *solves, long long step0, int nsteps,
                                                                  const double *qbuf)
{
    __shared__ double q[DEFER_SLOTS][4];
    __shared__ State3 st;
    const int j = blockIdx.x;
    const Solve3 &S = solves[j];
    for (int r = threadIdx.x; r < nsteps; r += blockDim.x)
        for (int c = 0; c < 4; ++c) q[r][c] = qbuf[4ll * ((long long)j * DEFER_SLOTS + r) + c];
    if (threadIdx.x == 0) st = *S.st;
    __syncthreads();
    if (threadIdx.x != 0 || st.phase >= PH_DONE) return;
    for (int r = 0; r < nsteps; ++r) {
        if (st.phase >= PH_DONE) break;
        const long long n = st.s_base + step0 + r + 1;
        if (!needs_reduction(S.c, st.phase, n)) continue;
        if (q[r][3] == 0.0) {            // a needed step without partials: cannot happen by construction
            st.status = STATUS_WAIT_TIMEOUT;
            st.phase = PH_ERR;
            st.steps = n;
            break;
        }
        controller3(S.c, st, n, q[r]);
    }
    *S.st = st;
}

cudaError_t launch_deferred3d(const Solve3 *solves, int nsolves, long long step0, int nsteps, double *qbuf,
                              int mode, cudaStream_t s)
{
    if (nsolves <= 0 || nsteps <= 0) return cudaSuccess;
    if (nsteps > DEFER_SLOTS) return cudaErrorInvalidValue;
    reduce3d_kernel<<<dim3(nsolves, nsteps), TPB, 0, s>>>(solves, step0, qbuf, mode);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    control3d_kernel<<<nsolves, DEFER_SLOTS, 0, s>>>(solves, step0, nsteps, qbuf);
    return cudaGetLastError();
}

}  // namespace lbm
