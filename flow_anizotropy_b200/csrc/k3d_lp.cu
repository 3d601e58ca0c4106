// Reduced-precision D3Q19 kernels: shifted populations stored as FP32, FP16
// (power-of-two scaled) or BF16, collision in FP32, flux reduced in FP64.
#include "engine3d.cuh"

namespace lbm {

cudaError_t launch_init3d_f64(void *A, long long plane, long long n, cudaStream_t s);
cudaError_t launch_canon3d_f64(const Solve3 &S, long long done, double *f, float *u, cudaStream_t s);
int max_blocks_f64(int variant);

#define LBM_LP(ST, V, W) step3d_kernel<ST, variant_lp(V).npt, variant_lp(V).minb, W>

template <class ST, bool W>
static cudaError_t launch_lp(int v, dim3 grid, cudaStream_t s, const StepArgs &a)
{
    switch (v) {
    case 0: LBM_LP(ST, 0, W)<<<grid, TPB, 0, s>>>(a); break;
    case 1: LBM_LP(ST, 1, W)<<<grid, TPB, 0, s>>>(a); break;
    case 2: LBM_LP(ST, 2, W)<<<grid, TPB, 0, s>>>(a); break;
    case 3: LBM_LP(ST, 3, W)<<<grid, TPB, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_step3d_lp(int prec, int variant, bool w1, dim3 grid, cudaStream_t s, const StepArgs &a)
{
    switch (prec) {
    case 1: return w1 ? launch_lp<StoreF32, true>(variant, grid, s, a) : launch_lp<StoreF32, false>(variant, grid, s, a);
    case 2: return w1 ? launch_lp<StoreF16, true>(variant, grid, s, a) : launch_lp<StoreF16, false>(variant, grid, s, a);
    case 3: return w1 ? launch_lp<StoreBF16, true>(variant, grid, s, a) : launch_lp<StoreBF16, false>(variant, grid, s, a);
    default: return cudaErrorInvalidValue;
    }
}

template <class ST>
static int occ(int v)
{
    const void *k = v == 0 ? (const void *)LBM_LP(ST, 0, false) : v == 1 ? (const void *)LBM_LP(ST, 1, false)
                  : v == 2 ? (const void *)LBM_LP(ST, 2, false) : (const void *)LBM_LP(ST, 3, false);
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, TPB, 0);
    return nb;
}

int max_blocks_step3d(int prec, int variant)
{
    switch (prec) {
    case 0: return max_blocks_f64(variant);
    case 1: return occ<StoreF32>(variant);
    case 2: return occ<StoreF16>(variant);
    case 3: return occ<StoreBF16>(variant);
    default: return 0;
    }
}

cudaError_t launch_init3d(int prec, void *A, long long plane, long long n, cudaStream_t s)
{
    switch (prec) {
    case 0: return launch_init3d_f64(A, plane, n, s);
    case 1: init3d_kernel<StoreF32><<<1184, 256, 0, s>>>(A, plane, n); break;
    case 2: init3d_kernel<StoreF16><<<1184, 256, 0, s>>>(A, plane, n); break;
    case 3: init3d_kernel<StoreBF16><<<1184, 256, 0, s>>>(A, plane, n); break;
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

// Pore voxels per block of SCAN_WORDS mask words.
__global__ void word_sums_kernel(const uint32_t *mask, long long nwords, unsigned *bsum)
{
    __shared__ unsigned sh[TPB / 32];
    unsigned c = 0;
    for (int q = threadIdx.x; q < SCAN_WORDS; q += TPB) {
        const long long w = (long long)blockIdx.x * SCAN_WORDS + q;
        if (w < nwords) c += __popc(~mask[w]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t = 0;
        for (int i = 0; i < TPB / 32; ++i) t += sh[i];
        bsum[blockIdx.x] = t;
    }
}

// wpre[w] = pore voxels before word w (exclusive scan), from per-block offsets.
__global__ void word_scan_kernel(const uint32_t *mask, long long nwords, const unsigned *boff, uint32_t *wpre)
{
    constexpr int PER = SCAN_WORDS / TPB;       // consecutive words per thread
    __shared__ unsigned sh[TPB / 32];
    const long long w0 = (long long)blockIdx.x * SCAN_WORDS + (long long)threadIdx.x * PER;
    unsigned c[PER], t = 0;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        c[q] = (w0 + q < nwords) ? __popc(~mask[w0 + q]) : 0u;
        t += c[q];
    }
    // exclusive scan of t across the block
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned incl = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) sh[wid] = incl;
    __syncthreads();
    unsigned wbase = 0;
    for (int i = 0; i < wid; ++i) wbase += sh[i];
    unsigned run = boff[blockIdx.x] + wbase + incl - t;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        if (w0 + q < nwords) wpre[w0 + q] = run;
        run += c[q];
    }
}

// fnode[rank] = linear index of every pore voxel.
__global__ void scatter_fnode_kernel(const uint32_t *mask, const uint32_t *wpre, long long nwords, int wpr,
                                     int nx, uint32_t *fnode)
{
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < nwords;
         w += (long long)gridDim.x * blockDim.x) {
        uint32_t f = ~mask[w];
        unsigned at = wpre[w];
        const long long row = w / wpr;
        const int x0 = (int)(w - row * wpr) * 32;
        while (f) {
            const int b = __ffs(f) - 1;
            f &= f - 1u;
            fnode[at++] = (uint32_t)(row * nx + x0 + b);
        }
    }
}

__global__ void advance3d_kernel(Solve3 *solves, int nsolves, long long steps)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nsolves && solves[i].st->phase < PH_DONE) solves[i].st->s_base += steps;
}

}  // namespace lbm
