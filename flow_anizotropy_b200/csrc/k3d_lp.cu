// Reduced-precision D3Q19 kernels: shifted populations stored as FP32, FP16
// (power-of-two scaled) or BF16, collision in FP32, flux reduced in FP64.
#include "engine3d.cuh"

namespace lbm {

cudaError_t launch_init3d_f64(void *A, long long plane, long long nn, cudaStream_t s);
cudaError_t launch_canon3d_f64(const Solve3 &S, long long done, double *f, float *u, cudaStream_t s);
int max_blocks_f64(int npt);

template <class ST>
static cudaError_t launch_lp(int npt, dim3 grid, cudaStream_t s, const StepArgs &a)
{
    switch (npt) {
    case 1: step3d_kernel<ST, 1><<<grid, TPB, 0, s>>>(a); break;
    case 2: step3d_kernel<ST, 2><<<grid, TPB, 0, s>>>(a); break;
    case 4: step3d_kernel<ST, 4><<<grid, TPB, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_step3d_lp(int prec, int npt, dim3 grid, cudaStream_t s, const StepArgs &a)
{
    switch (prec) {
    case 1: return launch_lp<StoreF32>(npt, grid, s, a);
    case 2: return launch_lp<StoreF16>(npt, grid, s, a);
    case 3: return launch_lp<StoreBF16>(npt, grid, s, a);
    default: return cudaErrorInvalidValue;
    }
}

template <class ST>
static int occ(int npt)
{
    int nb = 0;
    if (npt == 1) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, step3d_kernel<ST, 1>, TPB, 0);
    else if (npt == 2) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, step3d_kernel<ST, 2>, TPB, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, step3d_kernel<ST, 4>, TPB, 0);
    return nb;
}

int max_blocks_step3d(int prec, int npt)
{
    switch (prec) {
    case 0: return max_blocks_f64(npt);
    case 1: return occ<StoreF32>(npt);
    case 2: return occ<StoreF16>(npt);
    case 3: return occ<StoreBF16>(npt);
    default: return 0;
    }
}

cudaError_t launch_init3d(int prec, void *A, long long plane, long long nn, cudaStream_t s)
{
    switch (prec) {
    case 0: return launch_init3d_f64(A, plane, nn, s);
    case 1: init3d_kernel<StoreF32><<<1184, 256, 0, s>>>(A, plane, nn); break;
    case 2: init3d_kernel<StoreF16><<<1184, 256, 0, s>>>(A, plane, nn); break;
    case 3: init3d_kernel<StoreBF16><<<1184, 256, 0, s>>>(A, plane, nn); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_canon3d(int prec, const Solve3 &S, long long done, double *f, float *u, cudaStream_t s)
{
    switch (prec) {
    case 0: return launch_canon3d_f64(S, done, f, u, s);
    case 1: canon3d_kernel<StoreF32><<<1184, 256, 0, s>>>(S, done, f, u); break;
    case 2: canon3d_kernel<StoreF16><<<1184, 256, 0, s>>>(S, done, f, u); break;
    case 3: canon3d_kernel<StoreBF16><<<1184, 256, 0, s>>>(S, done, f, u); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

__global__ void advance3d_kernel(Solve3 *solves, int nsolves, long long steps)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nsolves && solves[i].st->phase < PH_DONE) solves[i].st->s_base += steps;
}

}  // namespace lbm
