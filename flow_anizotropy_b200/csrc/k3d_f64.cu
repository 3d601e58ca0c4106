// FP64 D3Q19 kernels.  This translation unit is compiled with -fmad=false:
// the collision keeps the reference's rounding step by step
// (LMB3d/lbm3d-perm.cpp:218-245), so one step matches the CPU oracle bit for bit.
#include "engine3d.cuh"

namespace lbm {

#define LBM_ODD(V) step3d_odd_kernel<StoreF64, odd_f64(V).npt, odd_f64(V).minb, false>
#define LBM_EVEN(V) step3d_even_kernel<StoreF64, even_f64(V).minb, false, even_meta(V)>

cudaError_t launch_step3d_f64(int variant, bool odd, dim3 grid, cudaStream_t s, const StepArgs &a)
{
    if (variant < 0 || variant >= 2 * NVAR_F64) return cudaErrorInvalidValue;
    variant = kernel_variant(0, variant);        // the two-lattice AA form runs the in-place kernels
    const int vo = variant / NVAR_EVEN, ve = variant % NVAR_EVEN;
    if (odd) {
        switch (vo) {
        case 0: LBM_ODD(0)<<<grid, TPB, 0, s>>>(a); break;
        case 1: LBM_ODD(1)<<<grid, TPB, 0, s>>>(a); break;
        default: LBM_ODD(2)<<<grid, TPB, 0, s>>>(a); break;
        }
    } else {
        switch (ve) {
        case 0: LBM_EVEN(0)<<<grid, TPB, 0, s>>>(a); break;
        case 1: LBM_EVEN(1)<<<grid, TPB, 0, s>>>(a); break;
        case 2: LBM_EVEN(2)<<<grid, TPB, 0, s>>>(a); break;
        case 3: LBM_EVEN(3)<<<grid, TPB, 0, s>>>(a); break;
        // FP64 staging would exceed the static shared-memory limit: variants
        // 4-5 run the register-staged kernel with the same record reads
        case 4: LBM_EVEN(0)<<<grid, TPB, 0, s>>>(a); break;
        default: LBM_EVEN(1)<<<grid, TPB, 0, s>>>(a); break;
        }
    }
    return cudaGetLastError();
}

int max_blocks_f64(int variant, bool odd)
{
    variant = kernel_variant(0, variant);
    const int vo = variant / NVAR_EVEN, ve = variant % NVAR_EVEN;
    const void *k = odd ? (vo == 0 ? (const void *)LBM_ODD(0) : vo == 1 ? (const void *)LBM_ODD(1) : (const void *)LBM_ODD(2))
                        : (ve == 0 ? (const void *)LBM_EVEN(0) : ve == 1 ? (const void *)LBM_EVEN(1)
                           : ve == 2 ? (const void *)LBM_EVEN(2) : ve == 3 ? (const void *)LBM_EVEN(3)
                           : ve == 4 ? (const void *)LBM_EVEN(0) : (const void *)LBM_EVEN(1));
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
