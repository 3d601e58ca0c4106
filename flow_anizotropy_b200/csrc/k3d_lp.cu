// Reduced-precision D3Q19 kernels: shifted populations stored as FP32, FP16
// (power-of-two scaled) or BF16, collision in FP32, flux reduced in FP64.
#include <algorithm>

#include "engine3d.cuh"

namespace lbm {

cudaError_t launch_init3d_f64(void *A, long long plane, long long n, cudaStream_t s);
cudaError_t launch_canon3d_f64(const Solve3 &S, long long done, double *f, float *u, cudaStream_t s);
int max_blocks_f64(int variant, bool odd);

#define LBM_ODD(ST, V, W) step3d_odd_kernel<ST, odd_lp(V).npt, odd_lp(V).minb, W>
#define LBM_ODDP(ST, W) step3d_odd_pair_kernel<ST, odd_lp(3).minb, W>
#define LBM_EVEN(ST, V, W) step3d_even_kernel<ST, even_lp(V).minb, W, even_meta(V)>
#define LBM_EVENA(ST, V, W) step3d_even_async_kernel<ST, even_lp(V).minb, W>
#define LBM_EVENG(ST, V, W) step3d_even_group_kernel<ST, even_lp(V).minb, W, even_meta(V)>
#define LBM_EVENL(ST, V, W) step3d_even_links_kernel<ST, even_lp(V).minb, W, even_meta(V), even_pair(V)>
#define LBM_EVENW(ST, V, W) step3d_even_links1_kernel<ST, even_lp(V).minb, W, even_meta(V)>
#define LBM_ODDB(ST, W) step3d_odd_bulk_kernel<ST, odd_lp(4).minb, W>
#define LBM_PULL(ST, Q, W) step3d_pull_kernel<ST, pull_minb(Q), W, pull_meta(Q)>
#define LBM_PULL1(ST, Q, W) step3d_pull1_kernel<ST, pull_minb(Q), W, pull_meta(Q)>
#define LBM_PULLG(ST, Q, W) step3d_pull_group_kernel<ST, pull_minb(Q), W, pull_meta(Q)>

// Pull-form kernel of pull variant q (any step parity).
template <class ST, bool W>
static const void *pull_kernel(int q)
{
    switch (q) {
    case 0: return (const void *)LBM_PULL(ST, 0, W);
    case 1: return (const void *)LBM_PULL(ST, 1, W);
    case 2: return (const void *)LBM_PULL(ST, 2, W);
    case 3: return (const void *)LBM_PULL1(ST, 3, W);
    case 4: return (const void *)LBM_PULLG(ST, 4, W);
    default: return (const void *)LBM_PULLG(ST, 5, W);
    }
}

// Persistent CTAs of the bulk-staged odd kernel per (storage, tau = 1, device),
// set by prepare_bulk once its shared-memory ring has been allowed.
static int g_bulk_ctas[3][2][64];

template <class ST, bool W>
static int prepare_bulk(int dev)
{
    using T = typename ST::T;
    const void *k = (const void *)LBM_ODDB(ST, W);
    const unsigned smem = odd_bulk_smem<T>();
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    int nb = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, ODD_BULK_THREADS, smem) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    g_bulk_ctas[ST::code - 1][W ? 1 : 0][dev] = nb * sms;
    return nb;
}

cudaError_t prepare_step3d_lp(int dev)
{
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    const bool ok = prepare_bulk<StoreF32, true>(dev) > 0 && prepare_bulk<StoreF32, false>(dev) > 0
                 && prepare_bulk<StoreF16, true>(dev) > 0 && prepare_bulk<StoreF16, false>(dev) > 0
                 && prepare_bulk<StoreBF16, true>(dev) > 0 && prepare_bulk<StoreBF16, false>(dev) > 0;
    return ok ? cudaSuccess : cudaErrorInvalidConfiguration;
}

template <class ST, bool W>
static cudaError_t launch_bulk(dim3 grid, cudaStream_t s, const StepArgs &a)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const int ctas = (dev >= 0 && dev < 64) ? g_bulk_ctas[ST::code - 1][W ? 1 : 0][dev] : 0;
    if (ctas <= 0) return cudaErrorInvalidConfiguration;   // prepare_step3d_lp not run on this device
    grid.x = std::min<unsigned>(grid.x, (unsigned)ctas);
    LBM_ODDB(ST, W)<<<grid, ODD_BULK_THREADS, odd_bulk_smem<typename ST::T>(), s>>>(a);
    return cudaSuccess;
}

template <class ST, bool W>
static cudaError_t launch_lp(int v, bool odd, dim3 grid, cudaStream_t s, const StepArgs &a)
{
    if (v < 0 || v >= NVAR_LP + NVAR_PULL) return cudaErrorInvalidValue;
    if (v >= NVAR_LP) {
        switch (v - NVAR_LP) {
        case 0: LBM_PULL(ST, 0, W)<<<grid, TPB, 0, s>>>(a); break;
        case 1: LBM_PULL(ST, 1, W)<<<grid, TPB, 0, s>>>(a); break;
        case 2: LBM_PULL(ST, 2, W)<<<grid, TPB, 0, s>>>(a); break;
        case 3: LBM_PULL1(ST, 3, W)<<<grid, TPB, 0, s>>>(a); break;
        case 4: LBM_PULLG(ST, 4, W)<<<grid, TPB, 0, s>>>(a); break;
        default: LBM_PULLG(ST, 5, W)<<<grid, TPB, 0, s>>>(a); break;
        }
        return cudaGetLastError();
    }
    const int vo = v / NVAR_EVEN_LP, ve = v % NVAR_EVEN_LP;
    if (odd) {
        switch (vo) {
        case 0: LBM_ODD(ST, 0, W)<<<grid, TPB, 0, s>>>(a); break;
        case 1: LBM_ODD(ST, 1, W)<<<grid, TPB, 0, s>>>(a); break;
        case 2: LBM_ODD(ST, 2, W)<<<grid, TPB, 0, s>>>(a); break;
        case 3: LBM_ODDP(ST, W)<<<grid, TPB, 0, s>>>(a); break;
        default: {
            const cudaError_t e = launch_bulk<ST, W>(grid, s, a);
            if (e != cudaSuccess) return e;
        } break;
        }
    } else {
        switch (ve) {
        case 0: LBM_EVEN(ST, 0, W)<<<grid, TPB, 0, s>>>(a); break;
        case 1: LBM_EVEN(ST, 1, W)<<<grid, TPB, 0, s>>>(a); break;
        case 2: LBM_EVEN(ST, 2, W)<<<grid, TPB, 0, s>>>(a); break;
        case 3: LBM_EVEN(ST, 3, W)<<<grid, TPB, 0, s>>>(a); break;
        case 4: LBM_EVENA(ST, 4, W)<<<grid, TPB, 0, s>>>(a); break;
        case 5: LBM_EVENA(ST, 5, W)<<<grid, TPB, 0, s>>>(a); break;
        case 6: LBM_EVENG(ST, 6, W)<<<grid, TPB, 0, s>>>(a); break;
        case 7: LBM_EVENG(ST, 7, W)<<<grid, TPB, 0, s>>>(a); break;
        case 8: LBM_EVENL(ST, 8, W)<<<grid, TPB, 0, s>>>(a); break;
        case 9: LBM_EVENL(ST, 9, W)<<<grid, TPB, 0, s>>>(a); break;
        case 10: LBM_EVENL(ST, 10, W)<<<grid, TPB, 0, s>>>(a); break;
        case 11: LBM_EVENL(ST, 11, W)<<<grid, TPB, 0, s>>>(a); break;
        case 12: LBM_EVENL(ST, 12, W)<<<grid, TPB, 0, s>>>(a); break;
        case 13: LBM_EVENW(ST, 13, W)<<<grid, 2 * TPB, 0, s>>>(a); break;
        default: LBM_EVENW(ST, 14, W)<<<grid, 2 * TPB, 0, s>>>(a); break;
        }
    }
    return cudaGetLastError();
}

cudaError_t launch_step3d_lp(int prec, int variant, bool w1, bool odd, dim3 grid, cudaStream_t s, const StepArgs &a)
{
    variant = kernel_variant(prec, variant);     // the two-lattice AA form runs the in-place kernels
    switch (prec) {
    case 1: return w1 ? launch_lp<StoreF32, true>(variant, odd, grid, s, a) : launch_lp<StoreF32, false>(variant, odd, grid, s, a);
    case 2: return w1 ? launch_lp<StoreF16, true>(variant, odd, grid, s, a) : launch_lp<StoreF16, false>(variant, odd, grid, s, a);
    case 3: return w1 ? launch_lp<StoreBF16, true>(variant, odd, grid, s, a) : launch_lp<StoreBF16, false>(variant, odd, grid, s, a);
    default: return cudaErrorInvalidValue;
    }
}

template <class ST>
static int occ(int v, bool odd)
{
    if (v >= NVAR_LP) {
        int nb = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, pull_kernel<ST, true>(v - NVAR_LP), TPB, 0);
        return nb;
    }
    const int vo = v / NVAR_EVEN_LP, ve = v % NVAR_EVEN_LP;
    if (odd && vo == 4) {
        int dev = 0;
        cudaGetDevice(&dev);
        return prepare_bulk<ST, true>(dev);
    }
    const void *k = odd ? (vo == 0 ? (const void *)LBM_ODD(ST, 0, true) : vo == 1 ? (const void *)LBM_ODD(ST, 1, true)
                           : vo == 2 ? (const void *)LBM_ODD(ST, 2, true) : (const void *)LBM_ODDP(ST, true))
                        : (ve == 0 ? (const void *)LBM_EVEN(ST, 0, true) : ve == 1 ? (const void *)LBM_EVEN(ST, 1, true)
                           : ve == 2 ? (const void *)LBM_EVEN(ST, 2, true) : ve == 3 ? (const void *)LBM_EVEN(ST, 3, true)
                           : ve == 4 ? (const void *)LBM_EVENA(ST, 4, true) : ve == 5 ? (const void *)LBM_EVENA(ST, 5, true)
                           : ve == 6 ? (const void *)LBM_EVENG(ST, 6, true) : ve == 7 ? (const void *)LBM_EVENG(ST, 7, true)
                           : ve == 8 ? (const void *)LBM_EVENL(ST, 8, true) : ve == 9 ? (const void *)LBM_EVENL(ST, 9, true)
                           : ve == 10 ? (const void *)LBM_EVENL(ST, 10, true) : ve == 11 ? (const void *)LBM_EVENL(ST, 11, true)
                           : ve == 12 ? (const void *)LBM_EVENL(ST, 12, true) : ve == 13 ? (const void *)LBM_EVENW(ST, 13, true)
                           : (const void *)LBM_EVENW(ST, 14, true));
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, (!odd && even_wide(ve)) ? 2 * TPB : TPB, 0);
    return nb;
}

int max_blocks_step3d(int prec, int variant, bool odd)
{
    variant = kernel_variant(prec, variant);
    switch (prec) {
    case 0: return max_blocks_f64(variant, odd);
    case 1: return occ<StoreF32>(variant, odd);
    case 2: return occ<StoreF16>(variant, odd);
    case 3: return occ<StoreBF16>(variant, odd);
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

// Neighbour records of every pore voxel (see meta_nbrs).
__global__ void build_meta_kernel(Solve3 S, uint4 *meta, uint2 *meta2)
{
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < (unsigned)S.nfluid;
         i += gridDim.x * blockDim.x) {
        int x, y, z;
        coords3(S, S.fnode[i], x, y, z);
        CNb nb;
        compact_nbrs(S, i, x, y, z, nb);
        const int ny = S.ny, nz = S.nz, wpr = S.wpr;
        const int row = z * ny + y;
        const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
        const int zm = z == 0 ? nz - 1 : z - 1, zp = z == nz - 1 ? 0 : z + 1;
        auto off = [&](int yy, int zz, int k) -> unsigned {
            return nb.idx[k] - S.wpre[(unsigned)(zz * ny + yy) * wpr];
        };
        unsigned link = nb.solid & 0x7ffffu;
        link |= (x == 0 ? LK_XLO : 0u) | (x == S.nx - 1 ? LK_XHI : 0u) | (y == 0 ? LK_YLO : 0u) |
                (y == ny - 1 ? LK_YHI : 0u) | (z == 0 ? LK_ZLO : 0u) | (z == nz - 1 ? LK_ZHI : 0u);
        meta[i] = make_uint4((unsigned)row, link,
                             off(ym, z, k_of(0, -1, 0)) | (off(yp, z, k_of(0, 1, 0)) << 16),
                             off(y, zm, k_of(0, 0, -1)) | (off(y, zp, k_of(0, 0, 1)) << 16));
        meta2[i] = make_uint2(off(ym, zm, k_of(0, -1, -1)) | (off(yp, zm, k_of(0, 1, -1)) << 16),
                              off(ym, zp, k_of(0, -1, 1)) | (off(yp, zp, k_of(0, 1, 1)) << 16));
    }
}

__global__ void advance3d_kernel(Solve3 *solves, int nsolves, long long steps)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nsolves && solves[i].st->phase < PH_DONE) solves[i].st->s_base += steps;
}

}  // namespace lbm
