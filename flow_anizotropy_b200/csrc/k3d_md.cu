// Dense moment-form (LBM_MD32) kernels, launchers and tensor maps.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "engine_md.cuh"

namespace lbm {

__global__ void canonmd_kernel(const Solve3 S, long long done, double *f_out, float *u_out)
{
    const int nx = S.nx, ny = S.ny, nyp = ny + 2, xp = S.md.xp;
    const long long vol = S.md.vol;
    const float *cur = reinterpret_cast<const float *>(static_cast<const char *>(S.A) + MD_MAPS_BYTES) +
                       (done & 1ll) * (MD_NC * vol);
    const float Fx = (float)S.P.F[0], Fy = (float)S.P.F[1], Fz = (float)S.P.F[2];
    const float pr = (float)S.P.pref;
    for (long long node = blockIdx.x * (long long)blockDim.x + threadIdx.x; node < S.nn;
         node += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(node % nx);
        const long long r = node / nx;
        const int y = (int)(r % ny), z = (int)(r / ny);
        if (mbit(S.mask + ((size_t)z * ny + y) * S.wpr, x)) continue;
        float c1, d3, ux, uy, uz;
        if (done == 0) {
            ux = 0.5f * Fx; uy = 0.5f * Fy; uz = 0.5f * Fz;
            if (u_out) {
                u_out[3 * node] = ux; u_out[3 * node + 1] = uy; u_out[3 * node + 2] = uz;
            }
            if (f_out)
                for (int k = 0; k < Q3; ++k) f_out[node * Q3 + k] = w3(k);
            continue;
        }
        const long long o = ((long long)(z + 1) * nyp + (y + 1)) * xp + (x + 1);
        c1 = cur[o]; ux = cur[o + vol]; uy = cur[o + 2 * vol]; uz = cur[o + 3 * vol]; d3 = cur[o + 4 * vol];
        if (u_out) {
            u_out[3 * node] = ux; u_out[3 * node + 1] = uy; u_out[3 * node + 2] = uz;
        }
        if (f_out) {
            double f[Q3];
#define LBM_POP(K) f[K] = w3(K) + (double)pop_rec<K, float>(c1, d3, ux, uy, uz, 1.0f, pr, Fx, Fy, Fz);
            LBM_POP(0) LBM_POP(1) LBM_POP(2) LBM_POP(3) LBM_POP(4) LBM_POP(5) LBM_POP(6) LBM_POP(7) LBM_POP(8)
            LBM_POP(9) LBM_POP(10) LBM_POP(11) LBM_POP(12) LBM_POP(13) LBM_POP(14) LBM_POP(15) LBM_POP(16)
            LBM_POP(17) LBM_POP(18)
#undef LBM_POP
            for (int k = 0; k < Q3; ++k) f_out[node * Q3 + k] = f[k];
        }
    }
}

__global__ void padmask_kernel(const uint32_t *mask, int nx, int ny, int nz, int wpr, int xpm, uint8_t *pm)
{
    const long long total = (long long)xpm * (ny + 2) * (nz + 2);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(i % xpm);
        const long long r = i / xpm;
        const int py = (int)(r % (ny + 2)), pz = (int)(r / (ny + 2));
        uint8_t v = 1;                                   // past the ghost column: solid
        if (p <= nx + 1) {
            const int x = (p + nx - 1) % nx, y = (py + ny - 1) % ny, z = (pz + nz - 1) % nz;
            v = (uint8_t)mbit(mask + ((size_t)z * ny + y) * wpr, x);
        }
        pm[i] = v;
    }
}

#define LBM_MD(V) stepmd_kernel<md_ns(V), md_minb(V)>

static const void *md_kernel(int v)
{
    switch (v) {
    case 0: return (const void *)LBM_MD(0);
    case 1: return (const void *)LBM_MD(1);
    case 2: return (const void *)LBM_MD(2);
    case 3: return (const void *)LBM_MD(3);
    default: return nullptr;
    }
}

cudaError_t launch_stepmd(int v, dim3 grid, cudaStream_t s, const StepArgs &a)
{
    const size_t smem = md_smem_bytes(v);
    switch (v) {
    case 0: LBM_MD(0)<<<grid, MD_TPB, smem, s>>>(a); break;
    case 1: LBM_MD(1)<<<grid, MD_TPB, smem, s>>>(a); break;
    case 2: LBM_MD(2)<<<grid, MD_TPB, smem, s>>>(a); break;
    case 3: LBM_MD(3)<<<grid, MD_TPB, smem, s>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int max_blocks_stepmd(int v)
{
    const void *k = md_kernel(v);
    int nb = 0;
    if (k) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, MD_TPB, md_smem_bytes(v));
    return nb;
}

cudaError_t launch_canonmd(const Solve3 &S, long long done, double *f, float *u, cudaStream_t s)
{
    canonmd_kernel<<<1184, 256, 0, s>>>(S, done, f, u);
    return cudaGetLastError();
}

cudaError_t launch_padmask(const Solve3 &S, cudaStream_t s)
{
    padmask_kernel<<<1184, 256, 0, s>>>(S.mask, S.nx, S.ny, S.nz, S.wpr, S.md.xpm, const_cast<uint8_t *>(S.md.pmask));
    return cudaGetLastError();
}

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Maps: [0] records of buffer 0, [1] records of buffer 1 (4D: x, y, z,
// component; box 36 x 10 x 1 x 5), [2] padded mask (3D bytes; box 48 x 10 x 1).
cudaError_t init_md_lattice(const Solve3 &S, cudaStream_t s)
{
    static_assert(sizeof(CUtensorMap) == 128, "tensor map size");
    auto enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    const MDGeom &g = S.md;
    char *lat = static_cast<char *>(S.A);
    float *rec = reinterpret_cast<float *>(lat + MD_MAPS_BYTES);
    alignas(64) CUtensorMap maps[3];
    const cuuint64_t ny2 = (cuuint64_t)S.ny + 2, nz2 = (cuuint64_t)S.nz + 2;
    for (int b = 0; b < 2; ++b) {
        const cuuint64_t dims[4] = {(cuuint64_t)g.xp, ny2, nz2, (cuuint64_t)MD_NC};
        const cuuint64_t strides[3] = {(cuuint64_t)g.xp * 4, (cuuint64_t)g.xp * ny2 * 4, (cuuint64_t)g.vol * 4};
        const cuuint32_t box[4] = {MD_HX, MD_HY, 1, MD_NC};
        const cuuint32_t es[4] = {1, 1, 1, 1};
        if (enc(&maps[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, rec + (size_t)b * MD_NC * g.vol, dims, strides, box,
                es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorInvalidValue;
    }
    {
        const cuuint64_t dims[3] = {(cuuint64_t)g.xpm, ny2, nz2};
        const cuuint64_t strides[2] = {(cuuint64_t)g.xpm, (cuuint64_t)g.xpm * ny2};
        const cuuint32_t box[3] = {MD_MX, MD_HY, 1};
        const cuuint32_t es[3] = {1, 1, 1};
        if (enc(&maps[2], CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<uint8_t *>(g.pmask), dims, strides, box, es,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorInvalidValue;
    }
    // pageable source: staged before the call returns
    cudaError_t e = cudaMemcpyAsync(lat, maps, sizeof(maps), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    return cudaMemsetAsync(rec, 0, (size_t)2 * MD_NC * g.vol * 4, s);
}

}  // namespace lbm
