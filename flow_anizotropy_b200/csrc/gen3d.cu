// On-device structure generation for scripts/gen_aniso_structures3d.py
// datasets: the random trigonometric field, its porosity quantile and the
// 6-connected percolation test on the 3 x 3 x 3 tiling.
//
// The host draws every random number (wavevectors, phases) with the
// reference's own generator calls; the device does the work that scales with
// the voxel count:
//
//  * field (gen_aniso_structures3d.py:154-176): S = scale * sum_i
//    cos(((2 pi qz_i) z + (2 pi qy_i) y) + (2 pi qx_i) x + phi_i), the terms
//    formed and summed in the reference's order and rounding (this unit is
//    compiled without FMA contraction), modes accumulated in order;
//  * threshold (:179-181): the two order statistics around numpy's linear
//    quantile index, found by an 8-pass radix selection over the sortable
//    bit patterns of the doubles (the interpolation itself is done on the
//    host, in numpy's arithmetic); solid where S > t;
//  * percolation (:184-205): connected components of the pore phase of the
//    3 x 3 x 3 tiling (6-connectivity, no wrap) by union-find with atomic
//    minimum links, then whether a component touches both faces of each axis.
//
// Every loop over labels is bounded; exceeding the bound reports an error
// instead of spinning.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "../../include/lbm.h"
#include "engine_host.h"

namespace {

constexpr int GTPB = 256;

__global__ void trig_field_kernel(int size, int n_modes, const int *__restrict__ q, const double *__restrict__ phases,
                                  const double *__restrict__ pts, double scale, double *__restrict__ field)
{
    const double twopi = 2.0 * 3.141592653589793;
    const long long n = (long long)size * size * size;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % size);
        const long long r = i / size;
        const int y = (int)(r % size), z = (int)(r / size);
        const double px = pts[x], py = pts[y], pz = pts[z];
        double acc = 0.0;
        for (int m = 0; m < n_modes; ++m) {
            const double cz = twopi * (double)q[3 * m + 2], cy = twopi * (double)q[3 * m + 1],
                         cx = twopi * (double)q[3 * m];
            double phase = (cz * pz + cy * py) + cx * px;
            phase = phase + phases[m];
            acc = acc + cos(phase);
        }
        field[i] = scale * acc;
    }
}

// order-preserving map of a double's bits to an unsigned key
__device__ __forceinline__ unsigned long long sort_key(double v)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__global__ void select_hist_kernel(const double *__restrict__ field, long long n, unsigned long long prefix,
                                   unsigned long long pmask, int shift, unsigned *__restrict__ hist)
{
    __shared__ unsigned sh[256];
    for (int b = threadIdx.x; b < 256; b += blockDim.x) sh[b] = 0;
    __syncthreads();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = sort_key(field[i]);
        if ((k & pmask) == prefix) atomicAdd(&sh[(k >> shift) & 255u], 1u);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < 256; b += blockDim.x)
        if (sh[b]) atomicAdd(&hist[b], sh[b]);
}

__global__ void threshold_kernel(const double *__restrict__ field, long long n, double t, uint8_t *__restrict__ solid)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        solid[i] = field[i] > t ? 1 : 0;
}

// ---------------------------------------------------------------- union-find
struct Tile {
    int nx, ny, nz;     // cell
    int X, Y, Z;        // tiling = 3 x cell
};

__device__ __forceinline__ bool tile_pore(const uint8_t *solid, const Tile &t, long long i)
{
    const int X = (int)(i % t.X);
    const long long r = i / t.X;
    const int Y = (int)(r % t.Y), Z = (int)(r / t.Y);
    return solid[((long long)(Z % t.nz) * t.ny + (Y % t.ny)) * t.nx + (X % t.nx)] == 0;
}

__global__ void uf_init_kernel(const uint8_t *solid, Tile t, long long n, int *lab)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        lab[i] = tile_pore(solid, t, i) ? (int)i : -1;
}

// root of i: labels only ever point to smaller indices, so a chain is at most
// n long; `limit` guards the walk anyway
__device__ __forceinline__ int uf_find(const int *lab, int i, long long limit, unsigned *err)
{
    for (long long it = 0; it < limit; ++it) {
        const int p = __ldcg(lab + i);
        if (p == i) return i;
        i = p;
    }
    atomicOr(err, 1u);
    return i;
}

__device__ void uf_union(int *lab, int a, int b, long long limit, unsigned *err)
{
    for (int it = 0; it < (1 << 20); ++it) {
        a = uf_find(lab, a, limit, err);
        b = uf_find(lab, b, limit, err);
        if (a == b) return;
        if (a > b) { const int s = a; a = b; b = s; }
        // link the larger root under the smaller; retry if another thread
        // linked it first (its label then decreased, so progress is made)
        const int old = atomicMin(lab + b, a);
        if (old == b) return;
        b = old;
    }
    atomicOr(err, 2u);
}

__global__ void uf_merge_kernel(Tile t, long long n, int *lab, unsigned *err)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (__ldcg(lab + i) < 0) continue;
        const int X = (int)(i % t.X);
        const long long r = i / t.X;
        const int Y = (int)(r % t.Y), Z = (int)(r / t.Y);
        if (X > 0 && __ldcg(lab + i - 1) >= 0) uf_union(lab, (int)i, (int)(i - 1), n, err);
        if (Y > 0 && __ldcg(lab + i - t.X) >= 0) uf_union(lab, (int)i, (int)(i - t.X), n, err);
        if (Z > 0 && __ldcg(lab + i - (long long)t.X * t.Y) >= 0)
            uf_union(lab, (int)i, (int)(i - (long long)t.X * t.Y), n, err);
    }
}

__global__ void uf_flatten_kernel(long long n, int *lab, unsigned *err)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (lab[i] >= 0) lab[i] = uf_find(lab, (int)i, n, err);
}

// face voxel j of axis a (0 = x, 1 = y, 2 = z) on side hi (0/1) of the tiling
__device__ __forceinline__ long long face_index(const Tile &t, int a, int hi, long long j)
{
    long long u, v;
    if (a == 0) { u = j % t.Y; v = j / t.Y; return (v * t.Y + u) * t.X + (hi ? t.X - 1 : 0); }
    if (a == 1) { u = j % t.X; v = j / t.X; return (v * t.Y + (hi ? t.Y - 1 : 0)) * t.X + u; }
    u = j % t.X; v = j / t.X; return ((long long)(hi ? t.Z - 1 : 0) * t.Y + v) * t.X + u;
}

__device__ __forceinline__ long long face_count(const Tile &t, int a)
{
    return a == 0 ? (long long)t.Y * t.Z : a == 1 ? (long long)t.X * t.Z : (long long)t.X * t.Y;
}

// mark the roots that touch the high face of each axis (bit a of mark[root])
__global__ void face_mark_kernel(Tile t, const int *lab, uint8_t *mark)
{
    for (int a = 0; a < 3; ++a) {
        const long long m = face_count(t, a);
        for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < m; j += (long long)gridDim.x * blockDim.x) {
            const int l = lab[face_index(t, a, 1, j)];
            if (l >= 0) atomicOr(reinterpret_cast<unsigned *>(mark + (l & ~3)), 1u << (8 * (l & 3) + a));
        }
    }
}

// a root on the low face that also touches the high face: the axis percolates
__global__ void face_check_kernel(Tile t, const int *lab, const uint8_t *mark, unsigned *perc)
{
    for (int a = 0; a < 3; ++a) {
        const long long m = face_count(t, a);
        for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < m; j += (long long)gridDim.x * blockDim.x) {
            const int l = lab[face_index(t, a, 0, j)];
            if (l >= 0 && ((mark[l] >> a) & 1u)) atomicOr(perc, 1u << a);
        }
    }
}

int grid_for(long long n) { return (int)std::min<long long>((n + GTPB - 1) / GTPB, 148ll * 16); }

}  // namespace

extern "C" int lbm_trig_structure3d(lbm_ctx *ctx, int size, int n_modes, const int32_t *q, const double *phases,
                                    const double *pts, double scale, double porosity, uint8_t *solid_out,
                                    double *threshold)
{
    if (!ctx) return LBM_EINPUT;
    if (!q || !phases || !pts || !solid_out || !threshold) return lbm_fail_input(ctx, "null argument");
    if (size <= 0 || size > 1024 || n_modes <= 0) return lbm_fail_input(ctx, "bad size or mode count");
    if (!(porosity >= 0.0 && porosity <= 1.0)) return lbm_fail_input(ctx, "porosity must lie in [0, 1]");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const long long n = (long long)size * size * size;
    DevMem d_q(s), d_ph(s), d_pts(s), d_field(s), d_hist(s), d_solid(s);
    CK(d_q.alloc(sizeof(int) * 3 * (size_t)n_modes));
    CK(d_ph.alloc(sizeof(double) * (size_t)n_modes));
    CK(d_pts.alloc(sizeof(double) * (size_t)size));
    CK(d_field.alloc(sizeof(double) * (size_t)n));
    CK(d_hist.alloc(sizeof(unsigned) * 256));
    CK(cudaMemcpyAsync(d_q.p, q, sizeof(int) * 3 * (size_t)n_modes, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_ph.p, phases, sizeof(double) * (size_t)n_modes, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_pts.p, pts, sizeof(double) * (size_t)size, cudaMemcpyHostToDevice, s));
    auto *field = static_cast<double *>(d_field.p);
    trig_field_kernel<<<grid_for(n), GTPB, 0, s>>>(size, n_modes, static_cast<const int *>(d_q.p),
                                                   static_cast<const double *>(d_ph.p),
                                                   static_cast<const double *>(d_pts.p), scale, field);
    CK(cudaGetLastError());

    // numpy's linear quantile: virtual index (n - 1) q, its floor and the next
    const double vi = (double)(n - 1) * porosity;
    const long long lo = (long long)std::floor(vi);
    const long long hi = std::min(lo + 1, n - 1);
    double ord[2];
    const long long want[2] = {lo, hi};
    for (int w = 0; w < 2; ++w) {
        unsigned long long prefix = 0, pmask = 0;
        unsigned long long k = (unsigned long long)want[w];       // rank among the matching keys
        for (int shift = 56; shift >= 0; shift -= 8) {
            CK(cudaMemsetAsync(d_hist.p, 0, sizeof(unsigned) * 256, s));
            select_hist_kernel<<<grid_for(n), GTPB, 0, s>>>(field, n, prefix, pmask, shift,
                                                            static_cast<unsigned *>(d_hist.p));
            CK(cudaGetLastError());
            unsigned h[256];
            CK(cudaMemcpyAsync(h, d_hist.p, sizeof(h), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            int b = 0;
            while (b < 255 && k >= h[b]) { k -= h[b]; ++b; }
            prefix |= (unsigned long long)b << shift;
            pmask |= 255ull << shift;
        }
        const unsigned long long bits = (prefix >> 63) ? (prefix & 0x7fffffffffffffffull) : ~prefix;
        std::memcpy(&ord[w], &bits, sizeof(double));
    }
    const double gamma = vi - (double)lo;
    const double diff = ord[1] - ord[0];
    double t = ord[0] + diff * gamma;
    if (gamma >= 0.5) t = ord[1] - diff * (1.0 - gamma);
    *threshold = t;

    uint8_t *dst = solid_out;
    const bool dev = lbm_is_device_ptr(solid_out);
    if (!dev) {
        CK(d_solid.alloc((size_t)n));
        dst = static_cast<uint8_t *>(d_solid.p);
    }
    threshold_kernel<<<grid_for(n), GTPB, 0, s>>>(field, n, t, dst);
    CK(cudaGetLastError());
    if (!dev) CK(cudaMemcpyAsync(solid_out, dst, (size_t)n, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return LBM_OK;
}

extern "C" int lbm_percolates3d(lbm_ctx *ctx, const uint8_t *solid, int nx, int ny, int nz, int perc[3])
{
    if (!ctx) return LBM_EINPUT;
    if (!solid || !perc) return lbm_fail_input(ctx, "null argument");
    if (nx <= 0 || ny <= 0 || nz <= 0) return lbm_fail_input(ctx, "bad dimensions");
    const long long n = 27ll * nx * ny * nz;
    if (n >= (1ll << 31)) return lbm_fail_input(ctx, "3x3x3 tiling exceeds 2^31 voxels");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const long long cell = (long long)nx * ny * nz;
    DevMem d_solid(s), d_lab(s), d_mark(s), d_flags(s);
    const uint8_t *src = solid;
    if (!lbm_is_device_ptr(solid)) {
        CK(d_solid.alloc((size_t)cell));
        CK(cudaMemcpyAsync(d_solid.p, solid, (size_t)cell, cudaMemcpyHostToDevice, s));
        src = static_cast<const uint8_t *>(d_solid.p);
    }
    CK(d_lab.alloc(sizeof(int) * (size_t)n));
    CK(d_mark.alloc((size_t)(n + 3) / 4 * 4));
    CK(d_flags.alloc(sizeof(unsigned) * 2));
    CK(cudaMemsetAsync(d_mark.p, 0, (size_t)(n + 3) / 4 * 4, s));
    CK(cudaMemsetAsync(d_flags.p, 0, sizeof(unsigned) * 2, s));
    Tile t{nx, ny, nz, 3 * nx, 3 * ny, 3 * nz};
    auto *lab = static_cast<int *>(d_lab.p);
    auto *flags = static_cast<unsigned *>(d_flags.p);   // [0] percolation bits, [1] error bits
    uf_init_kernel<<<grid_for(n), GTPB, 0, s>>>(src, t, n, lab);
    CK(cudaGetLastError());
    uf_merge_kernel<<<grid_for(n), GTPB, 0, s>>>(t, n, lab, flags + 1);
    CK(cudaGetLastError());
    uf_flatten_kernel<<<grid_for(n), GTPB, 0, s>>>(n, lab, flags + 1);
    CK(cudaGetLastError());
    const long long fmax = std::max({(long long)t.Y * t.Z, (long long)t.X * t.Z, (long long)t.X * t.Y});
    face_mark_kernel<<<grid_for(fmax), GTPB, 0, s>>>(t, lab, static_cast<uint8_t *>(d_mark.p));
    CK(cudaGetLastError());
    face_check_kernel<<<grid_for(fmax), GTPB, 0, s>>>(t, lab, static_cast<const uint8_t *>(d_mark.p), flags);
    CK(cudaGetLastError());
    unsigned h[2] = {0, 0};
    CK(cudaMemcpyAsync(h, flags, sizeof(h), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (h[1]) return lbm_fail_input(ctx, "percolation labelling did not settle (iteration bound reached)");
    for (int a = 0; a < 3; ++a) perc[a] = (h[0] >> a) & 1u;
    return LBM_OK;
}
