// Moment-projected (tau = 1) D3Q19 kernels, FP32 and FP64 moments.
#include "engine_m.cuh"

namespace lbm {

#define LBM_M(MT, V) stepm_kernel<MT, variant_m_minb(V)>

template <class MT>
static cudaError_t launch_m(int v, dim3 grid, cudaStream_t s, const StepArgs &a)
{
    switch (v) {
    case 0: LBM_M(MT, 0)<<<grid, TPB, 0, s>>>(a); break;
    case 1: LBM_M(MT, 1)<<<grid, TPB, 0, s>>>(a); break;
    case 2: LBM_M(MT, 2)<<<grid, TPB, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_stepm(int prec, int variant, dim3 grid, cudaStream_t s, const StepArgs &a)
{
    if (prec == MomF32::code) return launch_m<MomF32>(variant, grid, s, a);
    if (prec == MomF64::code) return launch_m<MomF64>(variant, grid, s, a);
    return cudaErrorInvalidValue;
}

template <class MT>
static int occ_m(int v)
{
    const void *k = v == 0 ? (const void *)LBM_M(MT, 0) : v == 1 ? (const void *)LBM_M(MT, 1)
                                                                 : (const void *)LBM_M(MT, 2);
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, TPB, 0);
    return nb;
}

int max_blocks_stepm(int prec, int variant)
{
    return prec == MomF32::code ? occ_m<MomF32>(variant) : occ_m<MomF64>(variant);
}

cudaError_t launch_canonm(int prec, const Solve3 &S, long long done, double *f, float *u, cudaStream_t s)
{
    if (prec == MomF32::code) canonm_kernel<MomF32><<<1184, 256, 0, s>>>(S, done, f, u);
    else canonm_kernel<MomF64><<<1184, 256, 0, s>>>(S, done, f, u);
    return cudaGetLastError();
}

}  // namespace lbm
