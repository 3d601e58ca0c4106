// FP64 D3Q19 kernels.  This translation unit is compiled with -fmad=false:
// the collision keeps the reference's rounding step by step
// (LMB3d/lbm3d-perm.cpp:218-245), so one step matches the CPU oracle bit for bit.
#include "engine3d.cuh"

namespace lbm {

#define LBM_F64(V) step3d_kernel<StoreF64, variant_f64(V).npt, variant_f64(V).minb, false>

cudaError_t launch_step3d_f64(int variant, dim3 grid, cudaStream_t s, const StepArgs &a)
{
    switch (variant) {
    case 0: LBM_F64(0)<<<grid, TPB, 0, s>>>(a); break;
    case 1: LBM_F64(1)<<<grid, TPB, 0, s>>>(a); break;
    case 2: LBM_F64(2)<<<grid, TPB, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int max_blocks_f64(int variant)
{
    const void *k = variant == 0 ? (const void *)LBM_F64(0) : variant == 1 ? (const void *)LBM_F64(1)
                                                                           : (const void *)LBM_F64(2);
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, TPB, 0);
    return nb;
}

cudaError_t launch_init3d_f64(void *A, long long plane, long long n, cudaStream_t s)
{
    init3d_kernel<StoreF64><<<1184, 256, 0, s>>>(A, plane, n);
    return cudaGetLastError();
}

cudaError_t launch_canon3d_f64(const Solve3 &S, long long done, double *f, float *u, cudaStream_t s)
{
    canon3d_kernel<StoreF64><<<1184, 256, 0, s>>>(S, done, f, u);
    return cudaGetLastError();
}

}  // namespace lbm
