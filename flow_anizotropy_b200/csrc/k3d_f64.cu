// FP64 D3Q19 kernels.  This translation unit is compiled with -fmad=false:
// the collision keeps the reference's rounding step by step
// (LMB3d/lbm3d-perm.cpp:218-245), so one step matches the CPU oracle bit for bit.
#include "engine3d.cuh"

namespace lbm {

cudaError_t launch_step3d_f64(int npt, dim3 grid, cudaStream_t s, const StepArgs &a)
{
    switch (npt) {
    case 1: step3d_kernel<StoreF64, 1><<<grid, TPB, 0, s>>>(a); break;
    case 2: step3d_kernel<StoreF64, 2><<<grid, TPB, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int max_blocks_f64(int npt)
{
    int nb = 0;
    if (npt == 1) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, step3d_kernel<StoreF64, 1>, TPB, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, step3d_kernel<StoreF64, 2>, TPB, 0);
    return nb;
}

cudaError_t launch_init3d_f64(void *A, long long plane, long long nn, cudaStream_t s)
{
    init3d_kernel<StoreF64><<<1184, 256, 0, s>>>(A, plane, nn);
    return cudaGetLastError();
}

cudaError_t launch_canon3d_f64(const Solve3 &S, long long done, double *f, float *u, cudaStream_t s)
{
    canon3d_kernel<StoreF64><<<1184, 256, 0, s>>>(S, done, f, u);
    return cudaGetLastError();
}

}  // namespace lbm
