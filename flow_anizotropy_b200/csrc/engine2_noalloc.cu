// lbm_solve2d_noalloc: the D2Q9 solve of lbm_solve2d (LMB2d/main.cpp:99-235)
// with every device buffer carved out of one statically sized device array,
// so that the call itself allocates no device memory.
//
// Who needs it: a caller whose device memory is already owned by another
// allocator (a framework's caching pool that has reserved most of the GPU,
// where a cudaMalloc of a few MB can fail or fragment the pool), and a
// latency-bound caller that cannot take the device-wide synchronisation that
// cudaFree implies or the first-touch cost of a fresh allocation.  The 2D
// reference solver is itself built this way: its lattice, velocity and mask
// arrays are static globals of a fixed 256 x 256 cell (LMB2d/lbm.cpp:18-28,
// LMB2d/lbm.h:24-26); this entry point keeps that property on the device.
//
// Limits: nx * ny <= LBM_NOALLOC2D_MAX_CELLS (the reference's 256 x 256 cell)
// and ndir <= LBM_NOALLOC2D_MAX_DIRS (its two forcing directions); anything
// larger returns LBM_EINPUT naming the limit.  The array is one per device
// and process, so two calls that overlapped on one device would race on it:
// calls are serialised by a per-device lock that is held until the call's
// work on its stream has finished.
//
// Setup: every call takes the array's address with cudaGetSymbolAddress
// (with the context's device current; cheap once the module is loaded, and
// never stale, even if the caller reset the device in between).  On a
// device's first call this may make the CUDA runtime load this library's
// device code there, so that first call belongs before any stream capture
// starts.  The call synchronises its own stream, so it is not meant to be
// captured at all.
//
// Cost: the time loop launches one kernel per step from the host (about
// 8.6 us per step on a 256 x 256 cell, against 6.8 us for lbm_solve2d, which
// replays 100-step chunks from a CUDA graph); the results are the same.
//
// Kernels and arithmetic are those of lbm_solve2d (same work list, same
// fixed-order reductions), so the results equal lbm_solve2d's bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/lbm.h"
#include "engine2_host.h"
#include "engine2d.cuh"
#include "engine_host.h"

using namespace lbm;

// Defined in engine.cu: packs a byte mask into rows of 32-bit words, counts
// the pore cells and flags values other than 0/1.
__global__ void pack_mask_kernel(const uint8_t *__restrict__ solid, int nx, long long rows, int wpr,
                                 uint32_t *__restrict__ mask, unsigned long long *npore, unsigned *bad);

namespace {

constexpr long long kCells = LBM_NOALLOC2D_MAX_CELLS;
constexpr int kDirs = LBM_NOALLOC2D_MAX_DIRS;
constexpr long long kTiles = (kCells + TPB - 1) / TPB;
static_assert(kCells % 64 == 0, "the lattice plane (cells rounded up to 64) must fit kCells");

constexpr size_t al256(size_t n) { return (n + 255) / 256 * 256; }

// Byte layout of the scratch array.  Per direction: the AA lattice (9 planes),
// the U,V snapshot and last fields, the per-tile flux partials.  Shared: the
// bit mask (ceil(nx/32) * ny <= nx * ny words), the byte mask staged from
// host memory, the neighbour solid bits (one 16-bit word per cell), controller states, solve records, the work list, and the
// small sums (fieldres numerator/denominator per direction, pore count and
// the non-binary flag of the mask packing).
constexpr size_t kLatBytes = al256(sizeof(float) * Q2 * kCells);
constexpr size_t kFieldBytes = al256(sizeof(float) * 2 * kCells);
constexpr size_t kPartBytes = al256(sizeof(double) * 2 * kTiles);
constexpr size_t kDirBytes = kLatBytes + 2 * kFieldBytes + kPartBytes;
constexpr size_t kMaskOff = kDirs * kDirBytes;
constexpr size_t kSolidOff = kMaskOff + al256(sizeof(uint32_t) * kCells);
constexpr size_t kNbmOff = kSolidOff + al256((size_t)kCells);
constexpr size_t kStateOff = kNbmOff + al256(sizeof(uint16_t) * kCells);
constexpr size_t kSolveOff = kStateOff + al256(sizeof(State2) * kDirs);
constexpr size_t kWorkOff = kSolveOff + al256(sizeof(Solve2) * kDirs);
constexpr size_t kSmallOff = kWorkOff + al256(sizeof(int2) * kDirs * kTiles);
constexpr size_t kSmallBytes = al256(sizeof(double) * 2 * kDirs + 16);
constexpr size_t kScratchBytes = kSmallOff + kSmallBytes;   // about 7 MB

}  // namespace

// The scratch: one copy per device (per CUDA context) of this library.
static __device__ __align__(256) unsigned char g_scratch2d[kScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_lock[kMaxDevices];

// Holds the device's lock for the whole call and, before releasing it, waits
// for everything the call queued on its stream (also on error returns), so
// the next caller never meets work of this one in flight.
struct ScratchLock {
    lbm_ctx *ctx;
    std::lock_guard<std::mutex> guard;
    explicit ScratchLock(lbm_ctx *c) : ctx(c), guard(g_lock[c->device]) {}
    ~ScratchLock() { cudaStreamSynchronize(ctx->stream); }
};

}  // namespace

extern "C" int lbm_solve2d_noalloc(lbm_ctx *ctx, const uint8_t *solid, int nx, int ny,
                                   int ndir, const double *forces, const lbm_params2d *params,
                                   lbm_result2d *results, float *vel_out)
{
    if (!ctx) return LBM_EINPUT;
    if (!solid || !forces || !params || !results || ndir <= 0) return lbm_fail_input(ctx, "null argument");
    if (nx <= 0 || ny <= 0) return lbm_fail_input(ctx, "bad dimensions");
    if ((long long)nx * ny > kCells)
        return lbm_fail_input(ctx, "lbm_solve2d_noalloc: nx*ny = " + std::to_string((long long)nx * ny) +
                                       " exceeds LBM_NOALLOC2D_MAX_CELLS = " + std::to_string(kCells) +
                                       " (use lbm_solve2d)");
    if (ndir > kDirs)
        return lbm_fail_input(ctx, "lbm_solve2d_noalloc: ndir = " + std::to_string(ndir) +
                                       " exceeds LBM_NOALLOC2D_MAX_DIRS = " + std::to_string(kDirs));
    if (ctx->device < 0 || ctx->device >= kMaxDevices) return lbm_fail_input(ctx, "device ordinal out of range");
    const lbm_params2d p = *params;
    int rc = check_params2d(ctx, p);
    if (rc) return rc;
    CK(cudaSetDevice(ctx->device));
    ScratchLock lock(ctx);
    void *ptr = nullptr;
    CK(cudaGetSymbolAddress(&ptr, g_scratch2d));
    unsigned char *base = static_cast<unsigned char *>(ptr);
    cudaStream_t st = ctx->stream;

    // mask: stage host bytes in the scratch (device input is read in place)
    const long long nn = (long long)nx * ny;
    const int wpr = (nx + 31) / 32;
    const uint8_t *src = solid;
    if (!lbm_is_device_ptr(solid)) {
        CK(cudaMemcpyAsync(base + kSolidOff, solid, (size_t)nn, cudaMemcpyHostToDevice, st));
        src = base + kSolidOff;
    }
    auto *mask = reinterpret_cast<uint32_t *>(base + kMaskOff);
    auto *small = reinterpret_cast<double *>(base + kSmallOff);     // fieldres sums, 2 per direction
    auto *cnt = reinterpret_cast<unsigned long long *>(small + 2 * kDirs);
    auto *bad = reinterpret_cast<unsigned *>(cnt + 1);
    CK(cudaMemsetAsync(small, 0, kSmallBytes, st));
    const int blocks = (int)((nn / 32 + ny + 255) / 256);
    pack_mask_kernel<<<blocks, 256, 0, st>>>(src, nx, ny, wpr, mask, cnt, bad);
    CK(cudaGetLastError());
    unsigned long long h[2] = {0, 0};
    CK(cudaMemcpyAsync(h, cnt, 16, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if ((unsigned)h[1]) return lbm_fail_input(ctx, "non-binary voxel");
    if (h[0] == 0) return lbm_fail_input(ctx, "structure has no pore space");
    auto *nbm = reinterpret_cast<uint16_t *>(base + kNbmOff);
    CK(launch_nbmask2d(mask, nx, ny, nbm, st));

    // per-direction solve records on the scratch
    auto *d_states = reinterpret_cast<State2 *>(base + kStateOff);
    auto *d_solves = reinterpret_cast<Solve2 *>(base + kSolveOff);
    auto *d_work = reinterpret_cast<int2 *>(base + kWorkOff);
    Solve2 hs[kDirs];
    State2 hst[kDirs];
    int2 work[kDirs * kTiles];
    int nwork = 0;
    for (int j = 0; j < ndir; ++j) {
        Solve2 &S = hs[j];
        fill_solve2(S, nx, ny, forces + 2 * j, p);
        unsigned char *d = base + j * kDirBytes;
        S.A = reinterpret_cast<float *>(d);
        S.snap = reinterpret_cast<float *>(d + kLatBytes);
        S.last = reinterpret_cast<float *>(d + kLatBytes + kFieldBytes);
        S.partials = reinterpret_cast<double *>(d + kLatBytes + 2 * kFieldBytes);
        S.mask = mask;
        S.nbm = nbm;
        S.st = d_states + j;
        // the fields are read back for cells a step never writes (solids), so
        // they start at zero as in lbm_solve2d; lattice and partials are
        // written before they are read
        CK(cudaMemsetAsync(S.snap, 0, sizeof(float) * 2 * (size_t)nn, st));
        CK(cudaMemsetAsync(S.last, 0, sizeof(float) * 2 * (size_t)nn, st));
        init_state2(hst[j], S.c);      // zero flux counter, phase RUN
        init2d_kernel<<<256, 256, 0, st>>>(S.A, S.plane, S.nn);
        CK(cudaGetLastError());
        for (int t = 0; t < S.ntiles; ++t) work[nwork++] = make_int2(j, t);
    }
    CK(cudaMemcpyAsync(d_solves, hs, sizeof(Solve2) * ndir, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_work, work, sizeof(int2) * nwork, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_states, hst, sizeof(State2) * ndir, cudaMemcpyHostToDevice, st));

    // the host loop of lbm_solve2d: launch up to the next step at which some
    // direction's controller can change phase, then read the states back
    StepArgs2 a;
    a.solves = d_solves; a.work = d_work; a.nwork = nwork;
    for (long long s = 0;;) {
        CK(cudaMemcpyAsync(hst, d_states, sizeof(State2) * ndir, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        long long target = LLONG_MAX;
        for (int j = 0; j < ndir; ++j) {
            const Ctl2 &c = hs[j].c;
            if (hst[j].phase == PH_RUN) {
                long long nxt = (s / c.lag + 1) * c.lag;
                if (c.max_steps > s) nxt = std::min(nxt, c.max_steps);
                target = std::min(target, nxt);
            } else if (hst[j].phase == PH_AVG) {
                target = std::min(target, hst[j].avg_start + c.avg_steps);
            }
        }
        if (target == LLONG_MAX) break;
        for (; s < target; ++s) {
            a.step = s;
            CK(launch_step2d(dim3(nwork), st, a));
        }
    }

    for (int j = 0; j < ndir; ++j) {
        fieldres2d_kernel<<<64, TPB, 0, st>>>(hs[j].snap, hs[j].last, hs[j].nn, small + 2 * j);
        CK(cudaGetLastError());
    }
    double frh[2 * kDirs];
    CK(cudaMemcpyAsync(frh, small, sizeof(double) * 2 * ndir, cudaMemcpyDeviceToHost, st));
    if (vel_out)
        for (int j = 0; j < ndir; ++j)
            CK(cudaMemcpyAsync(vel_out + 2 * nn * j, hs[j].last, sizeof(float) * 2 * nn, cudaMemcpyDefault, st));
    CK(cudaStreamSynchronize(st));

    int out = LBM_OK;
    for (int j = 0; j < ndir; ++j) {
        const State2 &s2 = hst[j];
        lbm_result2d &r = results[j];
        r.q[0] = s2.q[0]; r.q[1] = s2.q[1];
        r.se[0] = s2.se[0]; r.se[1] = s2.se[1];
        r.steps = s2.steps;
        r.converged = s2.converged;
        r.status = s2.status;
        const double num = frh[2 * j], den = frh[2 * j + 1];
        r.fieldres = den > 0.0 ? (double)(float)std::sqrt(num / den) : 10.0;
        if (s2.status) {
            ctx->err = "non-finite flux in run " + std::to_string(j) + " at step " + std::to_string(s2.steps);
            out = LBM_EINPUT;
        } else if (!s2.converged && out == LBM_OK) {
            out = LBM_NOT_CONVERGED;
        }
    }
    return out;
}
