// Dense moment-form D3Q19 step for tau = 1 (LBM_MD32), with TMA-staged
// z-planes in shared memory.
//
// The operator is the moment-projected step of engine_m.cuh (a voxel's state
// is its record (c1, ux, uy, uz, d3); a step pulls f*_k(x - e_k) from the
// neighbour's record, or f*_opp(k)(x) from its own record across a solid
// link, and sums the new moments), with the same arithmetic in the same
// order.  What changes is the data path:
//
//  * records of every voxel (solids included, never read) live in a dense
//    padded volume with one ghost layer per face holding the periodic image,
//    so every neighbour of a tile is at a fixed offset and no rank tables are
//    read; rows are padded to 16 bytes;
//  * a CTA of 128 threads owns a 32 x 8 column of voxels and marches along z
//    through a segment of lz planes.  Each z-plane of the column with its halo
//    (36 x 10 cells x 5 components, plus 48 x 10 mask bytes) arrives by two
//    TMA tiled loads into a ring of shared-memory slots, completing on an
//    mbarrier; a plane is loaded once and serves three consecutive output
//    planes, so global reads are one record per voxel plus halo overlap that
//    neighbouring CTAs read at the same time (L2 hits);
//  * per plane, one warp compacts the pore cells of the staged mask into a
//    shared list (ballots), and the threads take pore voxels from the list,
//    so no lane idles on a solid voxel; the 19-point gather runs out of shared
//    memory; the new record is stored with row-ordered (mostly coalesced)
//    stores, plus the ghost copies of face voxels.
//
// Global traffic per voxel-step: 20 B read (every voxel) + 20 B written (pore
// voxels) + 1 B of mask, against 152 B per pore voxel for FP32 populations.
//
// Every wait on a TMA completion is bounded (1 s); a CTA that gives up waits
// (bounded) for its own loads in flight, marks the solve failed
// (status MD_STATUS_TIMEOUT, phase ERR) and returns.
#pragma once
#include "engine_m.cuh"
#include "tma.cuh"

namespace lbm {

constexpr int MD_TPB = 128;                                 // threads per CTA
constexpr int MD_BX = 32;                                   // tile width (x)
constexpr int MD_BY = 8;                                    // tile height (y)
constexpr int MD_CELLS = MD_BX * MD_BY;                     // voxels of a tile plane
constexpr int MD_HX = 36;                                   // record box width: x0-1 .. x0+34 (144 B)
constexpr int MD_HY = MD_BY + 2;
constexpr int MD_MX = 48;                                   // mask box width (48 B)
constexpr int MD_NC = 5;                                    // components: c1, ux, uy, uz, d3
constexpr int MD_PLANE = MD_HX * MD_HY;                     // cells per component in a slot
constexpr int MD_REC_BYTES = MD_NC * MD_PLANE * 4;
constexpr int MD_MASK_OFF = (MD_REC_BYTES + 127) / 128 * 128;
constexpr int MD_MASK_BYTES = MD_MX * MD_HY;
constexpr int MD_SLOT = (MD_MASK_OFF + MD_MASK_BYTES + 127) / 128 * 128;
constexpr unsigned MD_TX = MD_REC_BYTES + MD_MASK_BYTES;    // bytes per plane (both loads)
constexpr int MD_MAPS_BYTES = 512;                          // tensor maps at the head of a lattice
constexpr unsigned long long MD_WAIT_NS = WAIT_NS;
constexpr int MD_STATUS_TIMEOUT = STATUS_WAIT_TIMEOUT;

// ring depth and register budget per variant (z-segment length: md_lz)
__host__ __device__ constexpr int md_ns(int v) { return v == 3 ? 6 : 4; }
__host__ __device__ constexpr int md_minb(int v) { return v == 3 ? 5 : 7; }
inline size_t md_smem_bytes(int v) { return (size_t)md_ns(v) * MD_SLOT + 128; }

inline long long md_lattice_bytes(const MDGeom &g) { return MD_MAPS_BYTES + 2ll * MD_NC * g.vol * 4; }
inline long long md_pmask_bytes(const MDGeom &g, int ny, int nz) { return (long long)g.xpm * (ny + 2) * (nz + 2); }

// Geometry of a solve's dense volume and tile list for variant v.
inline void md_fill_geom(MDGeom &g, int nx, int ny, int nz, int v, int &ntiles)
{
    g.xp = (nx + 2 + 3) / 4 * 4;
    g.xpm = (nx + 2 + 15) / 16 * 16;
    g.vol = (long long)g.xp * (ny + 2) * (nz + 2);
    g.nxt = (nx + MD_BX - 1) / MD_BX;
    g.nyt = (ny + MD_BY - 1) / MD_BY;
    g.lz = md_lz(v);
    g.nzs = (nz + g.lz - 1) / g.lz;
    ntiles = g.nxt * g.nyt * g.nzs;
}

// Store a record at padded offset o of component-stride vol.
__device__ __forceinline__ void md_st5(float *dst, long long o, long long vol, float c1, float ux, float uy,
                                       float uz, float d3)
{
    dst[o] = c1;
    dst[o + vol] = ux;
    dst[o + 2 * vol] = uy;
    dst[o + 3 * vol] = uz;
    dst[o + 4 * vol] = d3;
}

// The new record of voxel (x, y, z) into its cell and the ghost cells that
// hold its periodic images.
__device__ __forceinline__ void md_store(float *dst, const Solve3 &S, int x, int y, int z, float c1, float ux,
                                         float uy, float uz, float d3)
{
    const int nx = S.nx, ny = S.ny, nz = S.nz, xp = S.md.xp, nyp = ny + 2;
    const long long vol = S.md.vol;
    md_st5(dst, ((long long)(z + 1) * nyp + (y + 1)) * xp + (x + 1), vol, c1, ux, uy, uz, d3);
    if (x != 0 && x != nx - 1 && y != 0 && y != ny - 1 && z != 0 && z != nz - 1) return;
#pragma unroll
    for (int iz = 0; iz < 3; ++iz) {
        const int pz = iz == 0 ? z + 1 : iz == 1 ? (z == 0 ? nz + 1 : -1) : (z == nz - 1 ? 0 : -1);
        if (pz < 0) continue;
#pragma unroll
        for (int iy = 0; iy < 3; ++iy) {
            const int py = iy == 0 ? y + 1 : iy == 1 ? (y == 0 ? ny + 1 : -1) : (y == ny - 1 ? 0 : -1);
            if (py < 0) continue;
#pragma unroll
            for (int ix = 0; ix < 3; ++ix) {
                if (ix == 0 && iy == 0 && iz == 0) continue;
                const int px = ix == 0 ? x + 1 : ix == 1 ? (x == 0 ? nx + 1 : -1) : (x == nx - 1 ? 0 : -1);
                if (px < 0) continue;
                md_st5(dst, ((long long)pz * nyp + py) * xp + px, vol, c1, ux, uy, uz, d3);
            }
        }
    }
}

// pull f*_k(x - e_k) from the staged planes (R[0] = z-1, R[1] = z, R[2] = z+1),
// or f*_opp(k)(x) from the own record across a solid link
template <int K>
__device__ __forceinline__ void md_gather(const float *const (&R)[3], const uint8_t *const (&M)[3], int c, int cm,
                                          const float *own, float pr, float Fx, float Fy, float Fz,
                                          float (&acc)[4])
{
    constexpr int ex = ex3(K), ey = ey3(K), ez = ez3(K);
    const bool bb = M[1 - ez][cm - ey * MD_MX - ex] != 0;
    const float *src = bb ? own : R[1 - ez] + (c - ey * MD_HX - ex);
    const float g = pop_rec<K, float>(src[0], src[4 * MD_PLANE], src[MD_PLANE], src[2 * MD_PLANE],
                                      src[3 * MD_PLANE], bb ? -1.0f : 1.0f, pr, Fx, Fy, Fz);
    acc[0] += g;
    if (ex) acc[1] += ex > 0 ? g : -g;
    if (ey) acc[2] += ey > 0 ? g : -g;
    if (ez) acc[3] += ez > 0 ? g : -g;
}

template <int K>
struct MDGather {
    __device__ __forceinline__ static void run(const float *const (&R)[3], const uint8_t *const (&M)[3], int c,
                                               int cm, const float *own, float pr, float Fx, float Fy, float Fz,
                                               float (&acc)[4])
    {
        md_gather<K>(R, M, c, cm, own, pr, Fx, Fy, Fz, acc);
        MDGather<K + 1>::run(R, M, c, cm, own, pr, Fx, Fy, Fz, acc);
    }
};
template <>
struct MDGather<Q3> {
    __device__ __forceinline__ static void run(const float *const (&)[3], const uint8_t *const (&)[3], int, int,
                                               const float *, float, float, float, float, float (&)[4]) {}
};

template <int NS, int MINB>
__global__ void __launch_bounds__(MD_TPB, MINB) stepmd_kernel(const StepArgs a)
{
    extern __shared__ unsigned char md_raw[];
    __shared__ uint64_t bars[NS];
    __shared__ double sh[MD_TPB / 32][3];
    __shared__ unsigned char list[MD_CELLS];                // pore cells of the current plane
    __shared__ int list_n;
    unsigned char *sm = md_raw + ((128u - (smem_u32(md_raw) & 127u)) & 127u);
    const int tid = threadIdx.x, lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < NS; ++s) mbar_init(&bars[s], 1);
        mbar_init_fence();
    }
    __syncthreads();
    unsigned parity = 0;   // bit s: parity of the next completion of slot s
    unsigned pend = 0;     // thread 0: slots with a load in flight not yet seen complete
    const int nwork = a.nwork_dev ? *a.nwork_dev : a.nwork;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 item = a.work[w];
        const Solve3 &S = a.solves[item.x];
        const int phase = S.st->phase;
        if (phase >= PH_DONE) continue;
        const long long n = S.st->s_base + a.step + 1;
        const bool red = needs_reduction(S.c, phase, n);
        const MDGeom &G = S.md;
        int t = item.y;
        const int txi = t % G.nxt;
        t /= G.nxt;
        const int tyi = t % G.nyt;
        const int zs = (t / G.nyt) * G.lz;
        const int ze = min(zs + G.lz, S.nz);
        const int x0 = txi * MD_BX, y0 = tyi * MD_BY;
        char *lat = static_cast<char *>(S.A);
        float *dst = reinterpret_cast<float *>(lat + MD_MAPS_BYTES) + (n & 1ll) * (MD_NC * G.vol);
        const float Fx = (float)S.P.F[0], Fy = (float)S.P.F[1], Fz = (float)S.P.F[2];
        const float pr = (float)S.P.pref;
        double acc3[3] = {0.0, 0.0, 0.0};
        if (n == 1) {
            // moments of the initial state f = w: rho = 1, j = 0
            for (int z = zs; z < ze; ++z)
                for (int cell = tid; cell < MD_CELLS; cell += MD_TPB) {
                    const int x = x0 + (cell & (MD_BX - 1)), y = y0 + cell / MD_BX;
                    if (x >= S.nx || y >= S.ny) continue;
                    if (mbit(S.mask + ((size_t)z * S.ny + y) * S.wpr, x)) continue;
                    const float ux = 0.5f * Fx, uy = 0.5f * Fy, uz = 0.5f * Fz;
                    float c1n, d3n;
                    make_record<float>(0.0f, ux, uy, uz, Fx, Fy, Fz, pr, c1n, d3n);
                    md_store(dst, S, x, y, z, c1n, ux, uy, uz, d3n);
                    acc3[0] += (double)ux; acc3[1] += (double)uy; acc3[2] += (double)uz;
                }
        } else {
            const void *rmap = lat + ((n + 1) & 1ll) * 128;   // records of step n - 1
            const void *mmap = lat + 256;
            const int np = ze - zs + 2;                      // padded planes zs .. ze + 1
            auto issue = [&](int j) {
                const int s = j % NS;
                unsigned char *slot = sm + s * MD_SLOT;
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(&bars[s], MD_TX);
                tma_load_4d(slot, rmap, x0, y0, zs + j, 0, &bars[s]);
                tma_load_3d(slot + MD_MASK_OFF, mmap, x0, y0, zs + j, &bars[s]);
                pend |= 1u << s;
            };
            if (tid == 0) {
                tensormap_acquire(rmap);
                tensormap_acquire(mmap);
                for (int j = 0; j < min(NS, np); ++j) issue(j);
            }
            int waited = 0;
            bool bad = false;
            const int xlim = S.nx - x0, ylim = S.ny - y0;   // valid cells: tx < xlim, ty < ylim
            for (int z = zs; z < ze; ++z) {
                const int j = z - zs + 1;                    // slot index of plane z
                while (waited <= j + 1) {
                    const int s = waited % NS;
                    if (!bad) {
                        if (mbar_wait_bounded(&bars[s], (parity >> s) & 1u, MD_WAIT_NS)) {
                            parity ^= 1u << s;
                            if (tid == 0) pend &= ~(1u << s);
                        } else {
                            bad = true;
                        }
                    }
                    ++waited;
                }
                const float *R[3] = {reinterpret_cast<const float *>(sm + ((j - 1) % NS) * MD_SLOT),
                                     reinterpret_cast<const float *>(sm + (j % NS) * MD_SLOT),
                                     reinterpret_cast<const float *>(sm + ((j + 1) % NS) * MD_SLOT)};
                const uint8_t *M[3] = {sm + ((j - 1) % NS) * MD_SLOT + MD_MASK_OFF,
                                       sm + (j % NS) * MD_SLOT + MD_MASK_OFF,
                                       sm + ((j + 1) % NS) * MD_SLOT + MD_MASK_OFF};
                // warp 0 compacts the pore cells of plane z, row by row
                if (tid < 32) {
                    int cnt = 0;
#pragma unroll
                    for (int r = 0; r < MD_BY; ++r) {
                        const bool pore = lane < xlim && r < ylim && !M[1][(r + 1) * MD_MX + lane + 1];
                        const unsigned b = __ballot_sync(0xffffffffu, pore);
                        if (pore) list[cnt + __popc(b & ((1u << lane) - 1u))] = (unsigned char)(r * MD_BX + lane);
                        cnt += __popc(b);
                    }
                    if (lane == 0) list_n = cnt;
                }
                __syncthreads();
                const int npz = bad ? 0 : list_n;
                for (int q = tid; q < npz; q += MD_TPB) {
                    const int cell = list[q];
                    const int tx = cell & (MD_BX - 1), ty = cell / MD_BX;
                    const int c = (ty + 1) * MD_HX + (tx + 1);
                    const int cm = (ty + 1) * MD_MX + (tx + 1);
                    const float *own = R[1] + c;
                    float acc[4] = {pop_rec<0, float>(own[0], own[4 * MD_PLANE], own[MD_PLANE], own[2 * MD_PLANE],
                                                      own[3 * MD_PLANE], 1.0f, pr, Fx, Fy, Fz),
                                    0.0f, 0.0f, 0.0f};
                    MDGather<1>::run(R, M, c, cm, own, pr, Fx, Fy, Fz, acc);
                    const float dr = acc[0];
                    const float rho = 1.0f + dr;
                    const float ux = (acc[1] + 0.5f * Fx) / rho;
                    const float uy = (acc[2] + 0.5f * Fy) / rho;
                    const float uz = (acc[3] + 0.5f * Fz) / rho;
                    float c1n, d3n;
                    make_record<float>(dr, ux, uy, uz, Fx, Fy, Fz, pr, c1n, d3n);
                    md_store(dst, S, x0 + tx, y0 + ty, z, c1n, ux, uy, uz, d3n);
                    acc3[0] += (double)ux; acc3[1] += (double)uy; acc3[2] += (double)uz;
                }
                if (__syncthreads_or(bad)) {
                    if (tid == 0) {
                        for (int s = 0; s < NS; ++s)
                            if ((pend >> s) & 1u) mbar_wait_bounded(&bars[s], (parity >> s) & 1u, MD_WAIT_NS);
                        S.st->status = MD_STATUS_TIMEOUT;
                        S.st->phase = PH_ERR;
                        __threadfence();
                    }
                    return;
                }
                if (tid == 0 && j - 1 + NS < np) issue(j - 1 + NS);
            }
        }
        if (red) finish_tile<MD_TPB>(S, item.y, n, acc3, sh);
    }
}

// Dense outputs from the records of step `done` (see canonm_kernel).
__global__ void canonmd_kernel(const Solve3 S, long long done, double *f_out, float *u_out);
// Padded byte mask with periodic ghost layers from the bit mask.
__global__ void padmask_kernel(const uint32_t *mask, int nx, int ny, int nz, int wpr, int xpm, uint8_t *pm);

cudaError_t launch_stepmd(int variant, dim3 grid, cudaStream_t s, const StepArgs &a);
cudaError_t launch_canonmd(const Solve3 &S, long long done, double *f, float *u, cudaStream_t s);
// Build the padded mask of a structure (S.md.pmask must point to its buffer).
cudaError_t launch_padmask(const Solve3 &S, cudaStream_t s);
// Tensor maps (head of S.A) and zeroed records of one direction.
cudaError_t init_md_lattice(const Solve3 &S, cudaStream_t s);
int max_blocks_stepmd(int variant);

}  // namespace lbm
