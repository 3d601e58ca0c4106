// D3Q19 permeability solve on the device: data layout, the AA-pattern
// stream-collide kernel with its fused flux reduction, and the convergence
// controller that replaces the host loop of LMB3d/lbm3d-perm.cpp:320-398.
//
// Layout in HBM (one lattice per forcing direction):
//   A[k][i]   19 planes over the PORE voxels only, i = rank of the voxel among
//             the pore voxels in x-fastest order (solids are never read by the
//             reference, LMB3d/lbm3d-perm.cpp:261-265, so they get no storage);
//             plane stride padded to 128 B.  One in-place buffer: the AA access
//             pattern (Bailey et al. 2009) alternates
//               odd steps  (local):     read A[k][i],           write A[opp k][i]
//               even steps (neighbour): read A[opp k][i(x-e_k)], write A[k][i(x+e_k)]
//             so each location is read and then rewritten by the same thread
//             and a step needs no second buffer.  Halfway bounce-back folds
//             into the neighbour step: a link whose far end is solid reads
//             A[k][i] and writes A[opp k][i] instead.  Step 1 of a solve is a
//             local step on the initial state, which is exactly the reference's
//             collide_only priming (LMB3d/lbm3d-perm.cpp:249-253,291-295).
//   mask      1 bit per voxel, 1 = solid, rows of ceil(nx/32) words (bits past
//             nx in a row's last word set, i.e. solid).
//   wpre      per mask word, the number of pore voxels before it (plus one
//             final entry = pore count): the rank of voxel x in row r is
//             wpre[r*wpr + x/32] + popc(~mask word & bits below x).
//   fnode     linear index of each pore voxel (neighbour steps need x, y, z).
//   partials  one double3 per tile, written only on reduction steps.
//
// Work is a list of (solve, tile) items; a tile is TPB*NPT consecutive pore
// voxels of one lattice.  One launch advances every listed solve by one step,
// each at its own step number, so solves admitted at different times share a
// launch.
#pragma once
#include <cuda_pipeline.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "d3q19.cuh"
#include "tma.cuh"

namespace lbm {

constexpr int TPB = 256;     // threads per block of the step kernels

// Unsigned division by a runtime constant via multiply-high (valid for
// dividends < 2^31): q = umulhi(n, m) >> s.
struct FastDiv {
    int d;
    unsigned m;
    unsigned s;
    void init(int div)
    {
        d = div;
        if (div == 1) { m = 0; s = 0; return; }
        unsigned l = 0;
        while ((1u << l) < (unsigned)div) ++l;          // ceil(log2 d)
        const unsigned long long p = 31ull + l;
        m = (unsigned)(((1ull << p) + (unsigned)div - 1) / (unsigned)div);
        s = (unsigned)(p - 32);
    }
    __device__ __forceinline__ int div(int n) const
    {
        return d == 1 ? n : (int)(__umulhi((unsigned)n, m) >> s);
    }
};

// Convergence controller parameters (LMB3d/lbm3d-perm.cpp:118-130), plus the
// optional block-mean criterion of the 2D reference (LMB2d/main.cpp:99-178)
// for reduced-precision storage.
struct Ctl3 {
    double eps;
    long long lag, min_steps, max_steps, avg_steps;
    int hold;
    int criterion;        // 0: instantaneous drift (reference); 1: block means; 2: block means, batch-means SE
    long long sample;     // criteria 1-2: flux sample interval
    double ksigma;        // criteria 1-2: k-sigma acceptance
};

enum { PH_RUN = 1, PH_AVG = 2, PH_DONE = 3, PH_ERR = 4 };

// Every wait of a step kernel on its own asynchronous copies is bounded by
// WAIT_NS; a kernel that gives up marks the solve with this status and PH_ERR.
constexpr int STATUS_WAIT_TIMEOUT = 5;
constexpr unsigned long long WAIT_NS = 1000000000ull;

// Mutable per-solve state, device resident, written only by the controller.
struct State3 {
    long long s_base;     // steps completed before the current launch chunk
    int phase;
    int hold, have_prev;
    int converged, status;
    unsigned counter;     // tiles finished on the current reduction step
    double qprev[3];
    double bs[3], bss[3], pse[3];
    long long bn;
    double ws[3];         // criterion 2: sum of the current sub-block's samples
    long long wn;
    double sum[3], sumsq[3];
    long long n_avg;
    double q[3], se[3];
    long long steps;
    double qlast[3];
    long long avg_start;  // step at which phase 1 ended
};

// Geometry of the dense moment form (LBM_MD32): a record for every voxel in
// a padded volume with one ghost layer per face (periodic images), rows
// padded to 16 bytes so that TMA boxes start on aligned addresses.
struct MDGeom {
    const uint8_t *pmask;  // padded byte mask (1 = solid), xpm x (ny+2) x (nz+2)
    long long vol;         // cells of one record component: xp * (ny+2) * (nz+2)
    int xp, xpm;           // padded row lengths: records (floats), mask (bytes)
    int nxt, nyt, nzs, lz; // tiles along x and y, z segments of lz planes
};

struct Solve3 {
    void *A;
    void *B;                 // pull form: the second lattice (else null)
    long long plane;         // elements per plane (>= nfluid)
    const uint32_t *mask;
    const uint32_t *wpre;    // pore voxels before each mask word (+ final total)
    const uint32_t *fnode;   // pore voxels, ascending linear index
    const uint4 *meta;       // per pore voxel: neighbour record (see NbMeta), or null
    const uint2 *meta2;
    int nfluid;
    int prec;                // LBM_FP64 .. LBM_M64
    int nx, ny, nz, wpr;
    long long nn;
    int ntiles;              // tiles of TPB*NPT pore voxels
    FastDiv dvx, dvy;
    float scale, inv_scale;
    Phys3 P;
    Ctl3 c;
    double *partials;     // ntiles * 3
    State3 *st;
    MDGeom md;            // dense moment form only
    int group;            // grouped even step: directions in the group led by this record (else 0)
    int pull;             // two-lattice pull form (step3d_pull_kernel): A and B alternate
    int aa2;              // two-lattice AA form: the even step scatters into the other lattice (aa_buf)
};

struct StepArgs {
    const Solve3 *solves;
    const int2 *work;     // (solve index, tile index)
    const int *nwork_dev; // if non-null, the item count is read here
    int nwork;
    long long step;       // steps completed = st->s_base + step
    unsigned long long wait_ns = 0;   // bulk-staged kernels: wait limit (0: WAIT_NS)
    int starve = 0;                   // test only: the bulk producer issues nothing
    int defer = 0;                    // flux partials to deferred slots (see finish_tile)
};

// Deferred reduction: with StepArgs::defer set, a reduction step leaves each
// tile's flux partial in slot (step & (DEFER_SLOTS - 1)) of the solve's
// partials (DEFER_SLOTS x ntiles x 3 doubles), and reduce3d_kernel /
// control3d_kernel sum and control those steps, in step order, after at most
// DEFER_SLOTS launches.  The host launches them before the controller's phase
// can matter again (every lag multiple, every phase end), so the step kernels
// of a reduction step need no fence, ticket or last-tile pass.
constexpr int DEFER_SLOTS = 64;

// Lattice buffer m of a solve (A = 0, B = 1).  The in-place AA form uses A
// for every step.  The two-lattice AA form (Solve3::aa2) runs step n with
// source buffer ((n - 1) >> 1) & 1 and destination buffer (n >> 1) & 1: the
// odd (local) step stays in place, and the even step gathers from one lattice
// and scatters into the other, so no slot is read and rewritten in one
// launch (the in-place even step's stores drop lines from the SM's L1 cache
// that other warps' gathers still need; on the 128^3 workload's access
// pattern alone, 119 -> 83 us per 2-byte launch and 152 -> 120 us per
// 4-byte one).  The slots within a buffer are those of the in-place form, so
// the kernels, their arithmetic and their bits are unchanged.  In the
// in-place form the even kernels' source and destination pointers are the
// same lattice: every slot belongs to one (thread, voxel, link), which loads
// it and later stores a value computed from that load, so no load and store
// of one address are unordered by data dependence, and loads of a thread's
// next voxel may move above its previous voxel's stores (disjoint slots).
template <class T>
__device__ __forceinline__ T *aa_buf(const Solve3 &S, long long m)
{
    return static_cast<T *>((S.aa2 && (m & 1)) ? S.B : S.A);
}
template <class T>
__device__ __forceinline__ T *aa_src(const Solve3 &S, long long n) { return aa_buf<T>(S, (n - 1) >> 1); }
template <class T>
__device__ __forceinline__ T *aa_dst(const Solve3 &S, long long n) { return aa_buf<T>(S, n >> 1); }

// ----------------------------------------------------------------- helpers --
__device__ __forceinline__ int mbit(const uint32_t *row, int x)
{
    return (int)((__ldg(row + (x >> 5)) >> (x & 31)) & 1u);
}

__device__ __forceinline__ bool needs_reduction(const Ctl3 &c, int phase, long long n)
{
    if (phase == PH_AVG) return true;
    if (n == c.max_steps) return true;
    if (n % c.lag == 0) return true;
    return c.criterion != 0 && (n % c.sample == 0);
}

// Controller step, run by one thread once the flux q of step n is known.
// Phase 1 is LMB3d/lbm3d-perm.cpp:332-364 (criterion 0), or the block-mean
// test of LMB2d/main.cpp:123-178 on 3D flux vectors (criterion 1); phase 2 is
// the averaging of :370-390.  Every FP64 operation is written with its
// rounding (no contraction left to the compiler), so the controller gives
// the same bits in every translation unit that runs it: in the step kernels
// of any precision and in the deferred reduction kernel.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double dnorm3(const double v[3])
{
    return __dsqrt_rn(dadd(dadd(dmul(v[0], v[0]), dmul(v[1], v[1])), dmul(v[2], v[2])));
}

__device__ inline void controller3(const Ctl3 &c, State3 &st, long long n, const double q[3])
{
    if (st.phase == PH_RUN) {
        st.qlast[0] = q[0]; st.qlast[1] = q[1]; st.qlast[2] = q[2];
        if (c.criterion == 0) {
            if (n % c.lag == 0) {
                for (int k = 0; k < 3; ++k)
                    if (!isfinite(q[k])) { st.status = 2; st.phase = PH_ERR; st.steps = n; return; }
                const double norm = dnorm3(q);
                double drift = 0.0;
                for (int k = 0; k < 3; ++k) drift = fmax(drift, fabs(dsub(q[k], st.qprev[k])));
                if (st.have_prev && n >= c.min_steps && drift < dmul(c.eps, norm)) st.hold++;
                else st.hold = 0;
                for (int k = 0; k < 3; ++k) st.qprev[k] = q[k];
                st.have_prev = 1;
            }
        } else {
            if (n % c.sample == 0) {
                for (int k = 0; k < 3; ++k)
                    if (!isfinite(q[k])) { st.status = 2; st.phase = PH_ERR; st.steps = n; return; }
                if (c.criterion == 1) {
                    for (int k = 0; k < 3; ++k) { st.bs[k] = dadd(st.bs[k], q[k]); st.bss[k] = dadd(st.bss[k], dmul(q[k], q[k])); }
                    st.bn++;
                } else {
                    // batch means: a block's SE from the means of its 10 sub-blocks
                    const long long per = c.lag / c.sample / 10 > 0 ? c.lag / c.sample / 10 : 1;
                    for (int k = 0; k < 3; ++k) st.ws[k] = dadd(st.ws[k], q[k]);
                    if (++st.wn == per) {
                        for (int k = 0; k < 3; ++k) {
                            const double mb = ddiv(st.ws[k], (double)per);
                            st.bs[k] = dadd(st.bs[k], mb); st.bss[k] = dadd(st.bss[k], dmul(mb, mb)); st.ws[k] = 0.0;
                        }
                        st.wn = 0;
                        st.bn++;
                    }
                }
            }
            if (n % c.lag == 0 && st.bn >= 2) {
                const double bn = (double)st.bn;
                double m[3], se[3];
                for (int k = 0; k < 3; ++k) {
                    m[k] = ddiv(st.bs[k], bn);
                    const double v = ddiv(dsub(st.bss[k], dmul(dmul(bn, m[k]), m[k])), dsub(bn, 1.0));
                    se[k] = __dsqrt_rn(ddiv(fmax(v, 0.0), bn));
                }
                if (st.have_prev) {
                    const double norm = dnorm3(m);
                    bool pass = n >= c.min_steps;
                    for (int k = 0; k < 3; ++k) {
                        const double tol = fmax(dmul(c.eps, norm),
                                                dmul(c.ksigma, __dsqrt_rn(dadd(dmul(se[k], se[k]), dmul(st.pse[k], st.pse[k])))));
                        pass = pass && fabs(dsub(m[k], st.qprev[k])) < tol;
                    }
                    if (pass) st.hold++; else st.hold = 0;
                }
                for (int k = 0; k < 3; ++k) {
                    st.qprev[k] = m[k]; st.pse[k] = se[k];
                    st.bs[k] = 0.0; st.bss[k] = 0.0; st.ws[k] = 0.0;
                }
                st.bn = 0;
                st.wn = 0;
                st.have_prev = 1;
            }
        }
        const bool conv = st.hold >= c.hold;
        if (conv || n >= c.max_steps) {
            st.converged = conv ? 1 : 0;
            if (c.avg_steps <= 0) {
                for (int k = 0; k < 3; ++k) { st.q[k] = q[k]; st.se[k] = 0.0; }
                st.steps = n;
                st.phase = PH_DONE;
            } else {
                st.phase = PH_AVG;
                st.avg_start = n;
            }
        }
        return;
    }
    if (st.phase == PH_AVG) {
        for (int k = 0; k < 3; ++k) { st.sum[k] = dadd(st.sum[k], q[k]); st.sumsq[k] = dadd(st.sumsq[k], dmul(q[k], q[k])); }
        st.n_avg++;
        if (st.n_avg >= c.avg_steps) {
            const double nn = (double)st.n_avg;
            for (int k = 0; k < 3; ++k) {
                st.q[k] = ddiv(st.sum[k], nn);
                st.se[k] = 0.0;
                if (st.n_avg > 1) {
                    const double var = ddiv(dsub(st.sumsq[k], dmul(dmul(nn, st.q[k]), st.q[k])), dsub(nn, 1.0));
                    st.se[k] = __dsqrt_rn(ddiv(fmax(var, 0.0), nn));
                }
            }
            st.steps = n;
            st.phase = PH_DONE;
        }
    }
}

// Barrier over the first NT threads of the block: __syncthreads (BAR 0), or
// the named barrier BAR when other warps of the block do other work.
template <int NT, int BAR>
__device__ __forceinline__ void cta_sync()
{
    if constexpr (BAR == 0) __syncthreads();
    else asm volatile("bar.sync %0, %1;" ::"n"(BAR), "n"(NT) : "memory");
}

// Block-wide fixed-order sum of three doubles; result valid in thread 0.
// TRAIL = false leaves out the closing barrier: the caller then has one
// before any thread can write `sh` again.
template <int NT = TPB, int BAR = 0, bool TRAIL = true>
__device__ __forceinline__ void block_sum3(double (&v)[3], double (*sh)[3])
{
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { sh[wid][0] = v[0]; sh[wid][1] = v[1]; sh[wid][2] = v[2]; }
    cta_sync<NT, BAR>();
    if (threadIdx.x == 0) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (int w = 0; w < NT / 32; ++w) { a0 += sh[w][0]; a1 += sh[w][1]; a2 += sh[w][2]; }
        v[0] = a0; v[1] = a1; v[2] = a2;
    }
    if constexpr (TRAIL) cta_sync<NT, BAR>();
}

__device__ __forceinline__ int defer_slot(const StepArgs &a)
{
    return a.defer ? (int)(a.step & (DEFER_SLOTS - 1)) : -1;
}

// Does a deferred step write (and the reduction pass sum) its flux partials?
// The steps the controller needs at the phase of the run (`pass_start`:
// steps done before the current reduction pass), and, with mode 2 (runs in
// which a solve's phase can change between passes, as in a batch whose
// solves sit at different step counts), every step after a lag multiple or
// max_steps since the pass started: the controller may have left phase 1
// there and then needs every step.
__device__ __forceinline__ bool deferred_reduces(const Ctl3 &c, int phase, long long n, long long pass_start, int mode)
{
    if (needs_reduction(c, phase, n)) return true;
    if (mode != 2 || phase != PH_RUN) return false;
    return (n - 1) / c.lag > pass_start / c.lag || (c.max_steps > pass_start && c.max_steps < n);
}

// Reduction flag of step n (= s_base + a.step + 1) of a solve in a launch.
__device__ __forceinline__ bool step_reduces(const StepArgs &a, const Ctl3 &c, int phase, long long n)
{
    if (a.defer != 2) return needs_reduction(c, phase, n);
    const long long s_base = n - a.step - 1;
    return deferred_reduces(c, phase, n, s_base + (a.step & ~(long long)(DEFER_SLOTS - 1)), 2);
}

// Tile finished on a reduction step: publish the tile's flux partial; the
// last tile of the solve to finish sums all partials in a fixed order (the
// result does not depend on which blocks ran which tiles, or on what else is
// in the batch) and runs the controller.  With slot >= 0 the partial goes to
// that deferred slot instead, and reduce3d_kernel does the rest later with
// the same sums in the same order, so the results are the same bits.
template <int NT = TPB, int BAR = 0>
__device__ __forceinline__ void finish_tile(const Solve3 &S, int tile, long long n,
                                            double (&acc)[3], double (*sh)[3], int slot = -1)
{
    __shared__ int s_last;
    if (slot >= 0) {
        block_sum3<NT, BAR, true>(acc, sh);
        if (threadIdx.x == 0) {
            double *p = S.partials + 3ll * ((long long)slot * S.ntiles + tile);
            p[0] = acc[0]; p[1] = acc[1]; p[2] = acc[2];
        }
        return;
    }
    block_sum3<NT, BAR, false>(acc, sh);    // the s_last barrier below closes it
    if (threadIdx.x == 0) {
        double *p = S.partials + 3ll * tile;
        p[0] = acc[0]; p[1] = acc[1]; p[2] = acc[2];
        __threadfence();
        const unsigned prev = atomicAdd(&S.st->counter, 1u);
        s_last = (prev == (unsigned)S.ntiles - 1u);
    }
    cta_sync<NT, BAR>();
    if (!s_last) return;
    __threadfence();
    double v[3] = {0.0, 0.0, 0.0};
    for (int t = threadIdx.x; t < S.ntiles; t += NT) {
        v[0] += __ldcg(S.partials + 3ll * t);
        v[1] += __ldcg(S.partials + 3ll * t + 1);
        v[2] += __ldcg(S.partials + 3ll * t + 2);
    }
    block_sum3<NT, BAR>(v, sh);
    if (threadIdx.x == 0) {
        State3 &st = *S.st;
        st.counter = 0u;
        const double inv = (double)S.nn;
        const double q[3] = {v[0] / inv, v[1] / inv, v[2] / inv};
        controller3(S.c, st, n, q);
    }
}

// Compact indices and solid bits of the 18 neighbours x + e_k of pore voxel
// i at (x, y, z): bit k of `solid` is set if x + e_k is solid, idx[k] is the
// pore rank of x + e_k (meaningful only when it is a pore).  Reads only the
// mask and the word-prefix table, both small enough to stay in L1/L2.
struct CNb {
    unsigned idx[Q3];
    unsigned solid;
};

__host__ __device__ constexpr int k_of(int dx, int dy, int dz)
{
    for (int k = 0; k < Q3; ++k)
        if (ex3(k) == dx && ey3(k) == dy && ez3(k) == dz) return k;
    return -1;
}

__device__ __forceinline__ void compact_nbrs(const Solve3 &S, unsigned i, int x, int y, int z, CNb &nb)
{
    const int nx = S.nx, ny = S.ny, nz = S.nz, wpr = S.wpr;
    const uint32_t *__restrict__ mask = S.mask;
    const uint32_t *__restrict__ wpre = S.wpre;
    const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
    const int zm = z == 0 ? nz - 1 : z - 1, zp = z == nz - 1 ? 0 : z + 1;
    const int yr[3] = {ym, y, yp};
    const int zr[3] = {zm * ny, z * ny, zp * ny};
    const int b = x & 31, wx = x >> 5;
    const unsigned below = (1u << b) - 1u;
    // words and bits of x - 1 and x + 1 within a row (periodic), and whether
    // they leave the word of x: every lane takes the same instructions, the
    // extra words are predicated loads (no divergent branches)
    const bool xlo = x == 0, xhi = x == nx - 1;
    const int xm = xlo ? nx - 1 : x - 1, xp = xhi ? 0 : x + 1;
    const int wm = xm >> 5, bm = xm & 31, wp = xp >> 5, bp = xp & 31;
    const bool om = wm != wx, op = wp != wx;
    unsigned bits = 0;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy) {
            const unsigned rb = (unsigned)((zr[dz + 1] + yr[dy + 1]) * wpr);
            const uint32_t m = __ldg(mask + rb + wx);
            const unsigned s0 = (m >> b) & 1u;
            const bool own = dy == 0 && dz == 0;
            const unsigned A = own ? i : __ldg(wpre + rb + wx) + __popc(~m & below);
            if (!own) {
                nb.idx[k_of(0, dy, dz)] = A;
                bits |= s0 << k_of(0, dy, dz);
            }
            if (dy == 0 || dz == 0) {
                const int km = k_of(-1, dy, dz), kp = k_of(1, dy, dz);
                const uint32_t mmw = om ? __ldg(mask + rb + wm) : m;
                const uint32_t mpw = op ? __ldg(mask + rb + wp) : m;
                const unsigned sm = (mmw >> bm) & 1u, sp = (mpw >> bp) & 1u;
                // rank of x - 1: A - 1, or the row's last pore across the wrap;
                // rank of x + 1: A + (x is a pore), or the row's first pore
                const unsigned im = xlo ? __ldg(wpre + rb + wpr) - 1u : A - 1u;
                const unsigned ip = xhi ? __ldg(wpre + rb) : A + 1u - s0;
                nb.idx[km] = im;
                nb.idx[kp] = ip;
                bits |= (sm << km) | (sp << kp);
            }
        }
    nb.solid = bits;
}

__device__ __forceinline__ void coords3(const Solve3 &S, unsigned node, int &x, int &y, int &z)
{
    const int r = S.dvx.div((int)node);
    x = (int)node - r * S.nx;
    z = S.dvy.div(r);
    y = r - z * S.ny;
}

// Per-pore-voxel neighbour record, built once per structure, so that the even
// step gets its 18 neighbour ranks from 24 bytes and a few table reads
// instead of the mask arithmetic of compact_nbrs:
//   meta.x  row index r = z*ny + y of the voxel
//   meta.y  bits 0-18: x + e_k solid; 19/20: x == 0 / nx-1; 21/22: y == 0 /
//           ny-1; 23/24: z == 0 / nz-1
//   meta.z  pores before x in rows (y-1, z) | (y+1, z) << 16
//   meta.w  pores before x in rows (y, z-1) | (y, z+1) << 16
//   meta2.x pores before x in rows (y-1, z-1) | (y+1, z-1) << 16
//   meta2.y pores before x in rows (y-1, z+1) | (y+1, z+1) << 16
// The rank of (x, row') is rowstart(row') + offset with rowstart(r) =
// wpre[r * wpr]; x +- 1 ranks follow from the row's rank at x and the solid
// bits, or across the periodic x wrap from the row's first / last pore.
constexpr unsigned LK_XLO = 1u << 19, LK_XHI = 1u << 20, LK_YLO = 1u << 21, LK_YHI = 1u << 22,
                   LK_ZLO = 1u << 23, LK_ZHI = 1u << 24;

__device__ __forceinline__ void meta_nbrs(const Solve3 &S, unsigned i, const uint4 m, const uint2 m2, CNb &nb)
{
    const int ny = S.ny, nz = S.nz, wpr = S.wpr;
    const uint32_t *__restrict__ wpre = S.wpre;
    const int row = (int)m.x;
    const unsigned link = m.y;
    const bool xlo = link & LK_XLO, xhi = link & LK_XHI;
    const int dym = (link & LK_YLO) ? ny - 1 : -1, dyp = (link & LK_YHI) ? 1 - ny : 1;
    const int dzm = (link & LK_ZLO) ? (nz - 1) * ny : -ny, dzp = (link & LK_ZHI) ? -(nz - 1) * ny : ny;
    const int rows[3][3] = {{row + dzm + dym, row + dym, row + dzp + dym},
                            {row + dzm, row, row + dzp},
                            {row + dzm + dyp, row + dyp, row + dzp + dyp}};   // [dy+1][dz+1]
    const unsigned offs[3][3] = {{m2.x & 0xffffu, m.z & 0xffffu, m2.y & 0xffffu},
                                 {m.w & 0xffffu, 0u, m.w >> 16},
                                 {m2.x >> 16, m.z >> 16, m2.y >> 16}};
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy) {
            const bool own = dy == 0 && dz == 0;
            const int r = rows[dy + 1][dz + 1];
            const bool face = dy == 0 || dz == 0;
            const unsigned rs = (!own || xhi) ? __ldg(wpre + (unsigned)r * wpr) : 0u;
            const unsigned A = own ? i : rs + offs[dy + 1][dz + 1];
            if (!own) nb.idx[k_of(0, dy, dz)] = A;
            if (face) {
                const unsigned s0 = own ? 0u : (link >> k_of(0, dy, dz)) & 1u;
                nb.idx[k_of(-1, dy, dz)] = xlo ? __ldg(wpre + (unsigned)(r + 1) * wpr) - 1u : A - 1u;
                nb.idx[k_of(1, dy, dz)] = xhi ? rs : A + 1u - s0;
            }
        }
    nb.solid = link & 0x7ffffu;
}

// Step-kernel variants.  The two AA steps are separate kernels with separate
// register budgets: the odd (local) step is pure streaming and wants many
// loads in flight (several voxels per thread, high occupancy); the even
// (neighbour) step carries the neighbour-rank arithmetic.  A variant index
// v selects odd variant v / NVAR_EVEN and even variant v % NVAR_EVEN
// (NVAR_EVEN_LP for the reduced-precision storage, which adds the grouped
// even kernels); lbm_tune3d times them on the actual structure.
struct Variant { int npt, minb; };
constexpr int NVAR_ODD = 3, NVAR_ODD_LP = 5, NVAR_EVEN = 6, NVAR_EVEN_LP = 15;
constexpr int NVAR_LP = NVAR_ODD_LP * NVAR_EVEN_LP, NVAR_F64 = NVAR_ODD * NVAR_EVEN;
constexpr int MAX_GROUP = 3;    // directions per grouped even step
inline int nvar_even(int prec) { return prec == 0 ? NVAR_EVEN : NVAR_EVEN_LP; }
// odd variants: 0-1 one voxel per thread, 2 two voxels a tile-half apart, 3
// two adjacent voxels per thread with paired (vector) slot accesses, 4 the
// same collision fed from a shared-memory ring filled by bulk copies
__host__ __device__ constexpr Variant odd_lp(int v)
{
    return v == 0 ? Variant{1, 4} : v == 1 ? Variant{1, 5} : Variant{2, 2};
}
// even variants: 0-1 read the neighbour record (META), 2-3 compute ranks from
// the mask, 4-5 read the record and stage their gathers with cp.async, 6-7
// are grouped (one rank computation for all directions of a structure; 6
// from the mask, 7 from the record), 8-12 are grouped with the link slots
// kept in shared memory and the directions stepped one at a time (8-9 from
// the record, 10 from the mask, 11-12 from the record with a thread's two
// voxels collided together in packed FP32, 13-14 one voxel per thread in
// blocks of 2 * TPB threads, 13 from the record, 14 from the mask)
__host__ __device__ constexpr Variant even_lp(int v)
{
    return v == 0 ? Variant{1, 3} : v == 1 ? Variant{1, 4} : v == 2 ? Variant{1, 3} : v == 3 ? Variant{1, 4}
         : v == 4 ? Variant{1, 4} : v == 5 ? Variant{1, 3} : v <= 7 ? Variant{1, 2}
         : v == 8 ? Variant{1, 3} : v == 9 ? Variant{1, 4} : v == 10 ? Variant{1, 3}
         : v == 11 ? Variant{2, 3} : v == 12 ? Variant{2, 2} : Variant{1, 2};
}
__host__ __device__ constexpr bool even_meta(int v)
{
    return v < 2 || v == 4 || v == 5 || v == 7 || v == 8 || v == 9 || v == 11 || v == 12 || v == 13;
}
__host__ __device__ constexpr bool even_async(int v) { return v == 4 || v == 5; }
__host__ __device__ constexpr bool even_grouped(int v) { return v >= 6; }
__host__ __device__ constexpr bool even_links(int v) { return v >= 8; }
__host__ __device__ constexpr bool even_pair(int v) { return v == 11 || v == 12; }
__host__ __device__ constexpr bool even_wide(int v) { return v >= 13; }   // blocks of 2 * TPB threads
__host__ __device__ constexpr Variant odd_f64(int v) { return v == 0 ? Variant{1, 2} : v == 1 ? Variant{2, 1} : Variant{1, 1}; }
__host__ __device__ constexpr Variant even_f64(int v)
{
    return v == 0 ? Variant{1, 2} : v == 1 ? Variant{1, 1} : v == 2 ? Variant{1, 2} : v == 3 ? Variant{1, 1}
         : v == 4 ? Variant{1, 2} : Variant{1, 3};
}
// Pull-form variants (two lattices, one kernel for every step; see
// step3d_pull_kernel) are the reduced-precision indices NVAR_LP ..
// NVAR_LP + NVAR_PULL - 1; with p = v - NVAR_LP: 0-1 per direction, source
// ranks from the neighbour record, 2 or 3 blocks per SM; 2 per direction,
// ranks from the mask; 3 one voxel per thread at a time (voxels t and
// t + TPB of a tile, one-voxel collision and stores), 4 blocks per SM; 4-5 a
// structure's directions in one work item with the source slots found once
// into shared memory (ranks from the record), 2 or 3 blocks per SM.  All but
// 3 step a thread's two adjacent voxels together.
constexpr int NVAR_PULL = 6;
__host__ __device__ constexpr bool is_pull_variant(int prec, int v)
{
    return prec >= 1 && prec <= 3 && v >= NVAR_LP && v < NVAR_LP + NVAR_PULL;
}
__host__ __device__ constexpr int pull_minb(int p) { return p == 3 ? 4 : (p == 0 || p == 2 || p == 4) ? 2 : 3; }
__host__ __device__ constexpr bool pull_meta(int p) { return p != 2; }
__host__ __device__ constexpr bool pull_grouped(int p) { return p >= 4; }
// Two-lattice AA variants (Solve3::aa2) follow: the in-place variant v runs
// as NVAR_LP + NVAR_PULL + v (FP32, FP16, BF16) or NVAR_F64 + v (FP64), the
// same kernels with the even step scattering into the other lattice.
constexpr int AA2_BASE_LP = NVAR_LP + NVAR_PULL;
__host__ __device__ constexpr int aa2_base(int prec) { return prec == 0 ? NVAR_F64 : AA2_BASE_LP; }
__host__ __device__ constexpr bool is_aa2_variant(int prec, int v) { return prec >= 0 && prec <= 3 && v >= aa2_base(prec); }
// the in-place variant whose kernels a variant runs
__host__ __device__ constexpr int kernel_variant(int prec, int v) { return is_aa2_variant(prec, v) ? v - aa2_base(prec) : v; }
// pore voxels per tile: the odd and even kernels of one solve share the tile
// list (and its partials), so both use TPB * TILE_NPT voxels per tile
constexpr int TILE_NPT = 2;

// Store of population k of pore voxel i at lattice slot `slot` in step n: the
// 16-bit storage types round stochastically, the others to nearest.  The
// random bits are a per-(voxel, step) hash times an odd per-direction
// constant (its high bits are used), so each store draws fresh bits for one
// multiply, and a solve gives the same bits alone or in a batch.
__device__ __forceinline__ uint32_t sr_voxel(unsigned i, long long n)
{
    uint32_t h = i * 0x9e3779b1u ^ (uint32_t)n * 0x85ebca77u ^ (uint32_t)(n >> 32) * 0xc2b2ae3du;
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    h *= 0x846ca68bu;
    h ^= h >> 16;
    return h;
}

// random bits of store k of a voxel with per-(voxel, step) hash hv
__device__ __forceinline__ uint32_t dir_bits(uint32_t hv, int k) { return hv * (0x9e3779b1u * (2u * (uint32_t)k + 1u)); }

template <class ST>
__device__ __forceinline__ void store_pop(typename ST::T *A, unsigned slot, typename ST::C v, uint32_t hv, int k)
{
    if constexpr (ST::stochastic) ST::st_sr(A + slot, v, dir_bits(hv, k));
    else ST::st(A + slot, v);
}

template <class ST>
__device__ __forceinline__ uint32_t voxel_bits(unsigned i, long long n)
{
    if constexpr (ST::stochastic) return sr_voxel(i, n);
    else return 0u;
}

// Collision dispatch: FP64 keeps the reference's arithmetic; reduced-precision
// storage uses the pair-symmetric FP32 operator, specialised for tau = 1.
template <class ST, bool W1, class Cp>
__device__ __forceinline__ void collide3(Cp (&g)[Q3], const Solve3 &S, Cp &ux, Cp &uy, Cp &uz)
{
    if constexpr (ST::shifted) collide_pairs<W1, F32x1>(g, S.P, S.scale, S.inv_scale, ux, uy, uz);
    else collide_ref64(g, S.P, ux, uy, uz);
}

// Two voxels' populations collided together (packed FP32, the same bits per
// voxel as collide3 on each); u receives both velocities.
template <class ST, bool W1>
__device__ __forceinline__ void collide3x2(float2 (&g)[Q3], const Solve3 &S, float2 (&u)[3])
{
    static_assert(ST::shifted, "the packed operator is the reduced-precision one");
    collide_pairs<W1, F32x2>(g, S.P, S.scale, S.inv_scale, u[0], u[1], u[2]);
}

// Odd (local) step: read A[k][i], collide, write A[opp k][i].  The NPT voxels
// of a thread have all their loads issued before any store, so NPT x 19 loads
// are in flight per thread.  One tile = TPB * TILE_NPT voxels.
template <class ST, int NPT, int MINB, bool W1>
__global__ void __launch_bounds__(TPB, MINB) step3d_odd_kernel(const StepArgs a)
{
    using T = typename ST::T;
    using Cp = typename ST::C;
    static_assert(TILE_NPT % NPT == 0, "tile must split evenly");
    __shared__ double sh[TPB / 32][3];
    const int nwork = a.nwork_dev ? *a.nwork_dev : a.nwork;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 item = a.work[w];
        const Solve3 &S = a.solves[item.x];
        const int phase = S.st->phase;
        if (phase >= PH_DONE) continue;
        const long long n = S.st->s_base + a.step + 1;
        const bool red = step_reduces(a, S.c, phase, n);
        T *__restrict__ A = aa_src<T>(S, n);          // odd steps run in place
        const unsigned P = (unsigned)S.plane;
        double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
        for (int r = 0; r < TILE_NPT / NPT; ++r) {
            unsigned iv[NPT];
            bool vv[NPT];
            Cp g[NPT][Q3];
#pragma unroll
            for (int j = 0; j < NPT; ++j) {
                iv[j] = (unsigned)(item.y * (TPB * TILE_NPT) + (r * NPT + j) * TPB + threadIdx.x);
                vv[j] = iv[j] < (unsigned)S.nfluid;
#pragma unroll
                for (int k = 0; k < Q3; ++k) g[j][k] = vv[j] ? ST::ld(A + (k * P + iv[j])) : Cp(0);
            }
            if constexpr (NPT == 2 && ST::shifted) {
                // both voxels collide together (packed); an invalid one
                // computes on zeros and is neither stored nor summed
                float2 gp[Q3], u[3];
#pragma unroll
                for (int k = 0; k < Q3; ++k) gp[k] = make_float2(g[0][k], g[1][k]);
                collide3x2<ST, W1>(gp, S, u);
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    if (!vv[j]) continue;
                    const uint32_t hv = voxel_bits<ST>(iv[j], n);
#pragma unroll
                    for (int k = 0; k < Q3; ++k)
                        store_pop<ST>(A, opp3(k) * P + iv[j], j ? gp[k].y : gp[k].x, hv, k);
                    acc[0] += (double)(j ? u[0].y : u[0].x);
                    acc[1] += (double)(j ? u[1].y : u[1].x);
                    acc[2] += (double)(j ? u[2].y : u[2].x);
                }
            } else {
#pragma unroll
                for (int j = 0; j < NPT; ++j) {
                    if (!vv[j]) continue;
                    Cp ux, uy, uz;
                    collide3<ST, W1>(g[j], S, ux, uy, uz);
                    {
                        const uint32_t hv = voxel_bits<ST>(iv[j], n);
#pragma unroll
                        for (int k = 0; k < Q3; ++k) store_pop<ST>(A, opp3(k) * P + iv[j], g[j][k], hv, k);
                    }
                    acc[0] += (double)ux; acc[1] += (double)uy; acc[2] += (double)uz;
                }
            }
        }
        if (red) finish_tile(S, item.y, n, acc, sh, defer_slot(a));
    }
}

// Flux partial of a thread in the canonical order of a tile (thread t sums
// voxel t, then voxel t + TPB, as the one-voxel kernels do), for kernels
// whose threads own the adjacent voxels (2t, 2t + 1): the velocities are
// exchanged through shared memory, so every kernel variant reduces the same
// values in the same order and the fluxes agree bit for bit.  Called by all
// NT threads of the barrier group on reduction steps.
template <int NT, int BAR>
__device__ __forceinline__ void canonical_acc(float (*su)[TPB * TILE_NPT], const float2 (&u)[3], unsigned tid,
                                              unsigned tile_start, unsigned nfluid, double (&acc)[3])
{
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        su[c][2 * tid] = u[c].x;
        su[c][2 * tid + 1] = u[c].y;
    }
    cta_sync<NT, BAR>();
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        acc[c] = 0.0;
        if (tile_start + tid < nfluid) acc[c] += (double)su[c][tid];
        if (tile_start + tid + TPB < nfluid) acc[c] += (double)su[c][tid + TPB];
    }
}

// Odd (local) step with two adjacent pore voxels (i, i + 1), i even, per
// thread: every slot pair of a plane is one aligned 8-byte (FP32) or 4-byte
// (16-bit) access, the two voxels collide together in packed FP32, and the
// 16-bit types round both values with one cvt.rs fed with the bits each would
// get alone, so the populations equal those of step3d_odd_kernel, and the
// flux partials are summed in its order (canonical_acc).  The
// partner of the last voxel of an odd-sized lattice is a padding slot (the
// plane stride is a multiple of 64); it is read and written but never used.
template <class ST, int MINB, bool W1>
__global__ void __launch_bounds__(TPB, MINB) step3d_odd_pair_kernel(const StepArgs a)
{
    using T = typename ST::T;
    static_assert(TILE_NPT == 2, "a tile is one voxel pair per thread");
    __shared__ double sh[TPB / 32][3];
    __shared__ float su[3][TPB * TILE_NPT];
    const int nwork = a.nwork_dev ? *a.nwork_dev : a.nwork;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 item = a.work[w];
        const Solve3 &S = a.solves[item.x];
        const int phase = S.st->phase;
        if (phase >= PH_DONE) continue;
        const long long n = S.st->s_base + a.step + 1;
        const bool red = step_reduces(a, S.c, phase, n);
        T *__restrict__ A = aa_src<T>(S, n);          // odd steps run in place
        const unsigned P = (unsigned)S.plane;
        double acc[3] = {0.0, 0.0, 0.0};
        const unsigned ts = (unsigned)item.y * (TPB * TILE_NPT);
        const unsigned i0 = ts + 2u * threadIdx.x;
        float2 u[3] = {};
        if (i0 < (unsigned)S.nfluid) {
            float2 g[Q3];
#pragma unroll
            for (int k = 0; k < Q3; ++k) ST::ld2(A + (k * P + i0), g[k].x, g[k].y);
            collide3x2<ST, W1>(g, S, u);
            const uint32_t h0 = voxel_bits<ST>(i0, n), h1 = voxel_bits<ST>(i0 + 1u, n);
#pragma unroll
            for (int k = 0; k < Q3; ++k)
                ST::st2(A + (opp3(k) * P + i0), g[k].x, g[k].y, dir_bits(h0, k), dir_bits(h1, k));
        }
        if (red) {
            canonical_acc<TPB, 0>(su, u, threadIdx.x, ts, (unsigned)S.nfluid, acc);
            finish_tile(S, item.y, n, acc, sh, defer_slot(a));
        }
    }
}

// What a consumer of the bulk-staged odd step needs to know about its tile,
// written to shared memory by the producer with the tile's copies, so that
// the consumers read no global memory before their stores: the item, the
// solve, its lattice, the step number and reduction flag of this step, and
// the collision constants.
struct BulkTile {
    void *A;
    long long n;
    int item, solve, red;
    unsigned tile_start;     // rank of the tile's first voxel
    unsigned P, nfluid;
    float scale, inv_scale;
    Phys3 phys;
};

// Odd (local) step staged through shared memory by the copy engine.  A
// producer warp (the block's last 32 threads; one lane works) walks the work
// list (persistent grid, stride gridDim.x), skips items of finished solves,
// and for each tile (TPB * TILE_NPT voxels) issues 19 untiled bulk copies,
// one per plane run, into a ring of ODD_BULK_STAGES tile buffers; each
// buffer carries its tile descriptor (BulkTile).  The TPB consumer threads collide a tile
// out of shared memory (two adjacent voxels per thread, packed, as the pair
// kernel), store it straight to global memory and release the buffer.  So
// the loads of the next tiles are in flight while a tile is collided, and
// the producer's work-list reads never stall the consumers.  Populations and
// fluxes equal those of step3d_odd_pair_kernel bit for bit.  Every wait is
// bounded: consumers that give up mark the solve and leave, and the producer
// waits (bounded) for its copies in flight before it returns.
constexpr int ODD_BULK_STAGES_16 = 4, ODD_BULK_STAGES_32 = 2;
constexpr int ODD_BULK_THREADS = TPB + 32;
template <class T>
__host__ __device__ constexpr int odd_bulk_stages() { return sizeof(T) == 4 ? ODD_BULK_STAGES_32 : ODD_BULK_STAGES_16; }
template <class T>
__host__ __device__ constexpr unsigned odd_bulk_smem()
{
    return (unsigned)odd_bulk_stages<T>() * Q3 * TPB * TILE_NPT * (unsigned)sizeof(T);
}

template <class ST, int MINB, bool W1>
__global__ void __launch_bounds__(ODD_BULK_THREADS, MINB) step3d_odd_bulk_kernel(const StepArgs a)
{
    using T = typename ST::T;
    static_assert(TILE_NPT == 2, "a tile is one voxel pair per thread");
    constexpr int NS = odd_bulk_stages<T>();
    constexpr unsigned TV = TPB * TILE_NPT;              // voxels of a tile
    constexpr unsigned RUN = TV * (unsigned)sizeof(T);   // bytes of one plane run
    constexpr int BAR = 1;                               // consumers' named barrier
    extern __shared__ __align__(128) unsigned char ring[];
    __shared__ uint64_t full[NS], empty[NS];
    __shared__ BulkTile slot[NS];
    __shared__ double sh[TPB / 32][3];
    __shared__ float su[3][TPB * TILE_NPT];
    const int nwork = a.nwork_dev ? *a.nwork_dev : a.nwork;
    const int tid = threadIdx.x;
    const unsigned long long wait_ns = a.wait_ns ? a.wait_ns : WAIT_NS;
    if (tid == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(&full[s], 1u);
            mbar_init(&empty[s], (unsigned)TPB);
            slot[s].item = -1;
        }
        mbar_init_fence();
    }
    __syncthreads();

    if (tid >= TPB) {
        // ------------------------------------------------------ producer --
        // lane 0 walks the work list, waits for free buffers and fills the
        // tile descriptors; lanes 0..18 then issue one plane run each
        if (a.starve) return;
        const unsigned lane = (unsigned)tid & 31u;
        int next = blockIdx.x;
        unsigned eparity = 0u, fparity = 0u, copies = 0u;   // copies: buffers with bytes issued
        // the fields of the last solve seen (items of one solve come in runs;
        // nothing a tile needs changes during a launch once the solve is seen)
        int cx = -1, cphase = PH_DONE, cred = 0;
        BulkTile c{};
        bool gave_up = false;
        for (int t = 0;; ++t) {
            const int s = t % NS;
            bool more = false;
            unsigned bytes = 0u, P = 0u;
            const T *src = nullptr;
            if (lane == 0) {
                if (t >= NS) {
                    // the consumers' release of this buffer's previous tile
                    if (!mbar_wait_bounded(&empty[s], (eparity >> s) & 1u, wait_ns)) {
                        gave_up = true;
                    } else {
                        eparity ^= 1u << s;
                        copies &= ~(1u << s);
                    }
                }
                if (!gave_up) {
                    int w = next;
                    BulkTile &d = slot[s];
                    for (; w < nwork; w += gridDim.x) {
                        const int2 it = a.work[w];
                        if (it.x != cx) {
                            const Solve3 &S = a.solves[it.x];
                            cx = it.x;
                            cphase = S.st->phase;
                            c.n = S.st->s_base + a.step + 1;
                            c.A = aa_src<T>(S, c.n);          // odd steps run in place
                            c.P = (unsigned)S.plane;
                            c.nfluid = (unsigned)S.nfluid;
                            c.scale = S.scale;
                            c.inv_scale = S.inv_scale;
                            c.phys = S.P;
                            cred = cphase < PH_DONE && step_reduces(a, S.c, cphase, c.n) ? 1 : 0;
                            if (cphase < PH_DONE && ((reinterpret_cast<uintptr_t>(c.A) | (uintptr_t)c.P * sizeof(T)) & 15u)) {
                                // not a legal bulk copy (lattices are allocated
                                // aligned and planes padded to 64 slots, so this
                                // does not happen): the solve is failed instead
                                S.st->status = STATUS_WAIT_TIMEOUT;
                                S.st->phase = PH_ERR;
                                cphase = PH_ERR;
                            }
                        }
                        if (cphase >= PH_DONE) continue;
                        const unsigned i0 = (unsigned)it.y * TV;
                        P = c.P;
                        src = static_cast<const T *>(c.A) + i0;
                        bytes = ((unsigned)min(TV, c.nfluid - i0) * (unsigned)sizeof(T) + 15u) & ~15u;
                        d.A = c.A;
                        d.n = c.n;
                        d.tile_start = i0;
                        d.solve = it.x;
                        d.red = cred;
                        d.P = P;
                        d.nfluid = c.nfluid;
                        d.scale = c.scale;
                        d.inv_scale = c.inv_scale;
                        d.phys = c.phys;
                        break;
                    }
                    more = w < nwork;
                    next = more ? w + gridDim.x : w;
                    d.item = more ? w : -1;
                    if (more && bytes) {
                        fence_proxy_async_smem();
                        mbar_arrive_expect_tx(&full[s], Q3 * bytes);
                        copies |= 1u << s;
                    } else {
                        mbar_arrive(&full[s]);   // end of the list, or an item without voxels
                    }
                    fparity ^= 1u << s;
                }
            }
            // lane 0's decisions to the warp
            gave_up = __shfl_sync(0xffffffffu, gave_up ? 1 : 0, 0) != 0;
            if (gave_up) break;
            more = __shfl_sync(0xffffffffu, more ? 1 : 0, 0) != 0;
            bytes = __shfl_sync(0xffffffffu, bytes, 0);
            P = __shfl_sync(0xffffffffu, P, 0);
            src = reinterpret_cast<const T *>(__shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(src), 0));
            if (more && bytes && lane < (unsigned)Q3) {
                unsigned char *buf = ring + s * (Q3 * RUN);
                fence_proxy_async_smem();
                bulk_load(buf + lane * RUN, src + (size_t)lane * P, bytes, &full[s]);
            }
            if (!more) return;           // the consumers stop at this buffer
        }
        // gave up on a release: wait for the copies still in flight, then leave
        if (lane == 0)
            for (int r = 0; r < NS; ++r)
                if ((copies >> r) & 1u) mbar_wait_bounded(&full[r], ((fparity >> r) & 1u) ^ 1u, wait_ns);
        return;
    }

    // -------------------------------------------------------- consumers --
    unsigned parity = 0u;
    for (int t = 0;; ++t) {
        const int s = t % NS;
        const bool ok = mbar_wait_bounded(&full[s], (parity >> s) & 1u, wait_ns);
        int bad;
        asm volatile("{\n\t.reg .pred p, q;\n\t"
                     "setp.ne.u32 p, %1, 0;\n\t"
                     "bar.red.or.pred q, %2, %3, p;\n\t"
                     "selp.u32 %0, 1, 0, q;\n\t}"
                     : "=r"(bad)
                     : "r"((unsigned)!ok), "n"(BAR), "n"(TPB)
                     : "memory");
        if (bad) {
            if (tid == 0) {
                // the item index is written before the buffer's copies are
                // issued, so it is there even if they never completed; with
                // none, the CTA's first item names the solve
                int w = *static_cast<volatile int *>(&slot[s].item);
                if (w < 0 && (int)blockIdx.x < nwork) w = blockIdx.x;
                if (w >= 0) {
                    const Solve3 &S = a.solves[a.work[w].x];
                    S.st->status = STATUS_WAIT_TIMEOUT;
                    S.st->phase = PH_ERR;
                    __threadfence();
                }
            }
            return;
        }
        parity ^= 1u << s;
        const BulkTile &d = slot[s];
        const int w = d.item;
        if (w < 0) break;
        const long long n = d.n;
        const bool red = d.red != 0;
        T *__restrict__ A = static_cast<T *>(d.A);
        const unsigned P = d.P, nf = d.nfluid;
        const T *buf = reinterpret_cast<const T *>(ring + s * (Q3 * RUN));
        double acc[3] = {0.0, 0.0, 0.0};
        float2 g[Q3], u[3] = {};
#pragma unroll
        for (int k = 0; k < Q3; ++k) ST::lds2(buf + (k * TV + 2u * tid), g[k].x, g[k].y);
        const float sc = d.scale, isc = d.inv_scale;
        const Phys3 phys = d.phys;
        const int solve = d.solve;
        const unsigned tstart = d.tile_start;
        mbar_arrive(&empty[s]);    // this thread is done with buffer s (and its descriptor)
        const unsigned i0 = tstart + 2u * tid;
        if (i0 < nf) {
            collide_pairs<W1, F32x2>(g, phys, sc, isc, u[0], u[1], u[2]);
            const uint32_t h0 = voxel_bits<ST>(i0, n), h1 = voxel_bits<ST>(i0 + 1u, n);
#pragma unroll
            for (int k = 0; k < Q3; ++k)
                ST::st2(A + (opp3(k) * P + i0), g[k].x, g[k].y, dir_bits(h0, k), dir_bits(h1, k));
        }
        if (red) {
            const Solve3 &S = a.solves[solve];
            canonical_acc<TPB, BAR>(su, u, tid, tstart, nf, acc);
            finish_tile<TPB, BAR>(S, (int)(tstart / TV), n, acc, sh, defer_slot(a));
        }
    }
}

// Even (neighbour) step: pull A[opp k][rank(x - e_k)] (A[k][i] across a solid
// link), collide, push to A[k][rank(x + e_k)] (A[opp k][i] across a solid
// link).  One voxel per thread at a time; a tile is TPB * TILE_NPT voxels.
template <class ST, int MINB, bool W1, bool META>
__global__ void __launch_bounds__(TPB, MINB) step3d_even_kernel(const StepArgs a)
{
    using T = typename ST::T;
    using Cp = typename ST::C;
    __shared__ double sh[TPB / 32][3];
    const int nwork = a.nwork_dev ? *a.nwork_dev : a.nwork;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 item = a.work[w];
        const Solve3 &S = a.solves[item.x];
        const int phase = S.st->phase;
        if (phase >= PH_DONE) continue;
        const long long n = S.st->s_base + a.step + 1;
        const bool red = step_reduces(a, S.c, phase, n);
        const T *__restrict__ R = aa_src<T>(S, n);   // gathers
        T *__restrict__ W = aa_dst<T>(S, n);         // scatters
        const unsigned P = (unsigned)S.plane;
        double acc[3] = {0.0, 0.0, 0.0};
        // the records of all of this thread's voxels are requested up front:
        // each voxel's chain (record -> row starts -> populations) then starts
        // with its first DRAM trip already under way
        uint4 mr[TILE_NPT];
        uint2 mr2[TILE_NPT];
        if constexpr (META) {
#pragma unroll
            for (int j = 0; j < TILE_NPT; ++j) {
                const unsigned i = (unsigned)(item.y * (TPB * TILE_NPT) + j * TPB + threadIdx.x);
                const bool v = i < (unsigned)S.nfluid;
                mr[j] = v ? __ldg(S.meta + i) : make_uint4(0, 0, 0, 0);
                mr2[j] = v ? __ldg(S.meta2 + i) : make_uint2(0, 0);
            }
        }
#pragma unroll
        for (int j = 0; j < TILE_NPT; ++j) {
            const unsigned i = (unsigned)(item.y * (TPB * TILE_NPT) + j * TPB + threadIdx.x);
            if (i >= (unsigned)S.nfluid) continue;
            CNb nb;
            if constexpr (META) {
                meta_nbrs(S, i, mr[j], mr2[j], nb);
            } else {
                int x, y, z;
                coords3(S, __ldg(S.fnode + i), x, y, z);
                compact_nbrs(S, i, x, y, z, nb);
            }
            Cp g[Q3];
            g[0] = ST::ld(R + i);
#pragma unroll
            for (int k = 1; k < Q3; ++k) {
                const int o = opp3(k);
                const unsigned src = ((nb.solid >> o) & 1u) ? (k * P + i) : (o * P + nb.idx[o]);
                g[k] = ST::ld(R + src);
            }
            Cp ux, uy, uz;
            collide3<ST, W1>(g, S, ux, uy, uz);
            const uint32_t hv = voxel_bits<ST>(i, n);
            store_pop<ST>(W, i, g[0], hv, 0);
#pragma unroll
            for (int k = 1; k < Q3; ++k) {
                const unsigned dst = ((nb.solid >> k) & 1u) ? (opp3(k) * P + i) : (k * P + nb.idx[k]);
                store_pop<ST>(W, dst, g[k], hv, k);
            }
            acc[0] += (double)ux; acc[1] += (double)uy; acc[2] += (double)uz;
        }
        if (red) finish_tile(S, item.y, n, acc, sh, defer_slot(a));
    }
}

// Even step of a group of directions that share one structure (consecutive
// solve records; the first holds the group size in `group`): the neighbour
// ranks of a pore voxel are found once and serve every direction's lattice,
// and the gathers of one direction overlap the rank work of the next voxel.
// Per-direction phases, step counts and reductions are those of
// step3d_even_kernel, with the flux partials summed in the same order, so the
// results are bit-identical to it.
template <class ST, int MINB, bool W1, bool META>
__global__ void __launch_bounds__(TPB, MINB) step3d_even_group_kernel(const StepArgs a)
{
    using T = typename ST::T;
    using Cp = typename ST::C;
    __shared__ double sh[TPB / 32][3];
    __shared__ double sacc[MAX_GROUP][3][TPB];
    const int nwork = a.nwork_dev ? *a.nwork_dev : a.nwork;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 item = a.work[w];
        const Solve3 &S0 = a.solves[item.x];
        const int ng = min(S0.group, MAX_GROUP);
        unsigned live = 0, redm = 0;
#pragma unroll
        for (int d = 0; d < MAX_GROUP; ++d) {
            if (d >= ng) break;
            const Solve3 &S = a.solves[item.x + d];
            const int phase = S.st->phase;
            if (phase >= PH_DONE) continue;
            live |= 1u << d;
            if (step_reduces(a, S.c, phase, S.st->s_base + a.step + 1)) {
                redm |= 1u << d;
                sacc[d][0][threadIdx.x] = 0.0;
                sacc[d][1][threadIdx.x] = 0.0;
                sacc[d][2][threadIdx.x] = 0.0;
            }
        }
        if (!live) continue;
        const unsigned P = (unsigned)S0.plane;
#pragma unroll 1
        for (int j = 0; j < TILE_NPT; ++j) {
            const unsigned i = (unsigned)(item.y * (TPB * TILE_NPT) + j * TPB + threadIdx.x);
            if (i >= (unsigned)S0.nfluid) continue;
            CNb nb;
            if constexpr (META) {
                meta_nbrs(S0, i, __ldg(S0.meta + i), __ldg(S0.meta2 + i), nb);
            } else {
                int x, y, z;
                coords3(S0, __ldg(S0.fnode + i), x, y, z);
                compact_nbrs(S0, i, x, y, z, nb);
            }
            // every direction's pulls are issued before the first collision:
            // one memory round trip serves all the directions of the voxel
            Cp g[MAX_GROUP][Q3];
#pragma unroll
            for (int d = 0; d < MAX_GROUP; ++d) {
                if (!((live >> d) & 1u)) continue;
                const T *__restrict__ A = aa_src<const T>(a.solves[item.x + d], a.solves[item.x + d].st->s_base + a.step + 1);
                g[d][0] = ST::ld(A + i);
#pragma unroll
                for (int k = 1; k < Q3; ++k) {
                    const int o = opp3(k);
                    const unsigned src = ((nb.solid >> o) & 1u) ? (k * P + i) : (o * P + nb.idx[o]);
                    g[d][k] = ST::ld(A + src);
                }
            }
#pragma unroll
            for (int d = 0; d < MAX_GROUP; ++d) {
                if (!((live >> d) & 1u)) continue;
                const Solve3 &S = a.solves[item.x + d];
                T *__restrict__ A = aa_dst<T>(S, S.st->s_base + a.step + 1);
                Cp ux, uy, uz;
                collide3<ST, W1>(g[d], S, ux, uy, uz);
                const uint32_t hv = voxel_bits<ST>(i, S.st->s_base + a.step + 1);
                store_pop<ST>(A, i, g[d][0], hv, 0);
#pragma unroll
                for (int k = 1; k < Q3; ++k) {
                    const unsigned dst = ((nb.solid >> k) & 1u) ? (opp3(k) * P + i) : (k * P + nb.idx[k]);
                    store_pop<ST>(A, dst, g[d][k], hv, k);
                }
                if ((redm >> d) & 1u) {
                    sacc[d][0][threadIdx.x] += (double)ux;
                    sacc[d][1][threadIdx.x] += (double)uy;
                    sacc[d][2][threadIdx.x] += (double)uz;
                }
            }
        }
#pragma unroll 1
        for (int d = 0; d < ng; ++d) {
            if (!((redm >> d) & 1u)) continue;
            const Solve3 &S = a.solves[item.x + d];
            double acc[3] = {sacc[d][0][threadIdx.x], sacc[d][1][threadIdx.x], sacc[d][2][threadIdx.x]};
            finish_tile(S, item.y, S.st->s_base + a.step + 1, acc, sh, defer_slot(a));
        }
    }
}

// Even step of a group of directions that share one structure, with each
// voxel's 18 link slots found once per step and reused by every direction.
// The AA even step reads and writes the same slot per link: population k is
// pulled from slot(o) = A[k][i] across a solid link, else A[o][rank(x - e_k)]
// (o = opp k), and the post-collision population o is pushed back to that
// slot.  The slots of the tile's voxels go to shared memory (each thread
// reads back only its own, so no barrier), then the directions are stepped
// one after another: a direction costs one shared-memory read and one
// address computation per access instead of the rank arithmetic and the
// solid selects, and only one direction's populations are held at a time.
// Per direction, voxel, step and tile the arithmetic, the random bits and
// the flux order are those of step3d_even_kernel, so the results are
// bit-identical to it.  PAIR: a thread's two voxels (t, t + TPB) are pulled
// together and collided in packed FP32 (the same bits per voxel); a missing
// second voxel collides zeros and is neither stored nor summed.
template <class ST, int MINB, bool W1, bool META, bool PAIR>
__global__ void __launch_bounds__(TPB, MINB) step3d_even_links_kernel(const StepArgs a)
{
    static_assert(!PAIR || (ST::shifted && TILE_NPT == 2), "pairs are collided by the packed FP32 operator");
    using T = typename ST::T;
    using Cp = typename ST::C;
    constexpr unsigned TV = TPB * TILE_NPT;
    __shared__ double sh[TPB / 32][3];
    __shared__ unsigned sl[Q3 - 1][TV];          // slot of link k (k = 1..18) of each voxel of the tile
    const int nwork = a.nwork_dev ? *a.nwork_dev : a.nwork;
    const unsigned tid = threadIdx.x;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 item = a.work[w];
        const Solve3 &S0 = a.solves[item.x];
        const int ng = min(S0.group, MAX_GROUP);
        unsigned live = 0;
#pragma unroll
        for (int d = 0; d < MAX_GROUP; ++d)
            if (d < ng && a.solves[item.x + d].st->phase < PH_DONE) live |= 1u << d;
        if (!live) continue;
        const unsigned P = (unsigned)S0.plane;
        const unsigned nf = (unsigned)S0.nfluid;
        const unsigned i0 = (unsigned)item.y * TV;
#pragma unroll
        for (int j = 0; j < TILE_NPT; ++j) {
            const unsigned i = i0 + j * TPB + tid;
            if (i >= nf) continue;
            CNb nb;
            if constexpr (META) {
                meta_nbrs(S0, i, __ldg(S0.meta + i), __ldg(S0.meta2 + i), nb);
            } else {
                int x, y, z;
                coords3(S0, __ldg(S0.fnode + i), x, y, z);
                compact_nbrs(S0, i, x, y, z, nb);
            }
#pragma unroll
            for (int k = 1; k < Q3; ++k) {
                const int o = opp3(k);
                sl[k - 1][j * TPB + tid] = ((nb.solid >> o) & 1u) ? (k * P + i) : (o * P + nb.idx[o]);
            }
        }
#pragma unroll 1
        for (int d = 0; d < ng; ++d) {
            if (!((live >> d) & 1u)) continue;
            const Solve3 &S = a.solves[item.x + d];
            const long long n = S.st->s_base + a.step + 1;
            const bool red = step_reduces(a, S.c, S.st->phase, n);
            const T *__restrict__ R = aa_src<T>(S, n);   // gathers
            T *__restrict__ W = aa_dst<T>(S, n);         // scatters
            double acc[3] = {0.0, 0.0, 0.0};
            if constexpr (PAIR) {
                const unsigned ia = i0 + tid, ib = i0 + TPB + tid;
                const bool va = ia < nf, vb = ib < nf;
                float2 g[Q3], u[3];
                g[0].x = va ? ST::ld(R + ia) : 0.0f;
                g[0].y = vb ? ST::ld(R + ib) : 0.0f;
#pragma unroll
                for (int k = 1; k < Q3; ++k) {
                    g[k].x = va ? ST::ld(R + sl[k - 1][tid]) : 0.0f;
                    g[k].y = vb ? ST::ld(R + sl[k - 1][TPB + tid]) : 0.0f;
                }
                collide3x2<ST, W1>(g, S, u);
                if (va) {
                    const uint32_t hv = voxel_bits<ST>(ia, n);
                    store_pop<ST>(W, ia, g[0].x, hv, 0);
#pragma unroll
                    for (int k = 1; k < Q3; ++k) store_pop<ST>(W, sl[opp3(k) - 1][tid], g[k].x, hv, k);
                    acc[0] += (double)u[0].x; acc[1] += (double)u[1].x; acc[2] += (double)u[2].x;
                }
                if (vb) {
                    const uint32_t hv = voxel_bits<ST>(ib, n);
                    store_pop<ST>(W, ib, g[0].y, hv, 0);
#pragma unroll
                    for (int k = 1; k < Q3; ++k) store_pop<ST>(W, sl[opp3(k) - 1][TPB + tid], g[k].y, hv, k);
                    acc[0] += (double)u[0].y; acc[1] += (double)u[1].y; acc[2] += (double)u[2].y;
                }
            } else {
#pragma unroll
                for (int j = 0; j < TILE_NPT; ++j) {
                    const unsigned i = i0 + j * TPB + tid;
                    if (i >= nf) continue;
                    Cp g[Q3];
                    g[0] = ST::ld(R + i);
#pragma unroll
                    for (int k = 1; k < Q3; ++k) g[k] = ST::ld(R + sl[k - 1][j * TPB + tid]);
                    Cp ux, uy, uz;
                    collide3<ST, W1>(g, S, ux, uy, uz);
                    const uint32_t hv = voxel_bits<ST>(i, n);
                    store_pop<ST>(W, i, g[0], hv, 0);
#pragma unroll
                    for (int k = 1; k < Q3; ++k) store_pop<ST>(W, sl[opp3(k) - 1][j * TPB + tid], g[k], hv, k);
                    acc[0] += (double)ux; acc[1] += (double)uy; acc[2] += (double)uz;
                }
            }
            if (red) finish_tile(S, item.y, n, acc, sh, defer_slot(a));
        }
    }
}

// The link-slot even step with one voxel per thread: blocks of 2 * TPB
// threads, thread t stepping voxel t of the tile.  A tile's directions take
// half as long per block as with two voxels per thread, so the grouped work
// list (a third as many items as the per-direction one) spreads over the
// SMs in more, shorter waves.  On reduction steps the velocities pass
// through shared memory so that thread t < TPB sums voxel t, then voxel
// t + TPB, as the other kernels do (the same flux bits); threads t >= TPB
// take no part in the block sum (named barrier 1 over the first TPB threads).
template <class ST, int MINB, bool W1, bool META>
__global__ void __launch_bounds__(2 * TPB, MINB) step3d_even_links1_kernel(const StepArgs a)
{
    using T = typename ST::T;
    using Cp = typename ST::C;
    static_assert(TILE_NPT == 2, "a tile is one voxel per thread of a 2 * TPB block");
    constexpr unsigned TV = TPB * TILE_NPT;
    __shared__ double sh[TPB / 32][3];
    __shared__ unsigned sl[Q3 - 1][TV];
    __shared__ float su[3][TV];
    const int nwork = a.nwork_dev ? *a.nwork_dev : a.nwork;
    const unsigned tid = threadIdx.x;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 item = a.work[w];
        const Solve3 &S0 = a.solves[item.x];
        const int ng = min(S0.group, MAX_GROUP);
        unsigned live = 0;
#pragma unroll
        for (int d = 0; d < MAX_GROUP; ++d)
            if (d < ng && a.solves[item.x + d].st->phase < PH_DONE) live |= 1u << d;
        if (!live) continue;
        const unsigned P = (unsigned)S0.plane;
        const unsigned nf = (unsigned)S0.nfluid;
        const unsigned i0 = (unsigned)item.y * TV;
        const unsigned i = i0 + tid;
        const bool v = i < nf;
        if (v) {
            CNb nb;
            if constexpr (META) {
                meta_nbrs(S0, i, __ldg(S0.meta + i), __ldg(S0.meta2 + i), nb);
            } else {
                int x, y, z;
                coords3(S0, __ldg(S0.fnode + i), x, y, z);
                compact_nbrs(S0, i, x, y, z, nb);
            }
#pragma unroll
            for (int k = 1; k < Q3; ++k) {
                const int o = opp3(k);
                sl[k - 1][tid] = ((nb.solid >> o) & 1u) ? (k * P + i) : (o * P + nb.idx[o]);
            }
        }
#pragma unroll 1
        for (int d = 0; d < ng; ++d) {
            if (!((live >> d) & 1u)) continue;
            const Solve3 &S = a.solves[item.x + d];
            const long long n = S.st->s_base + a.step + 1;
            const bool red = step_reduces(a, S.c, S.st->phase, n);
            const T *__restrict__ R = aa_src<T>(S, n);   // gathers
            T *__restrict__ W = aa_dst<T>(S, n);         // scatters
            Cp ux = Cp(0), uy = Cp(0), uz = Cp(0);
            if (v) {
                Cp g[Q3];
                g[0] = ST::ld(R + i);
#pragma unroll
                for (int k = 1; k < Q3; ++k) g[k] = ST::ld(R + sl[k - 1][tid]);
                collide3<ST, W1>(g, S, ux, uy, uz);
                const uint32_t hv = voxel_bits<ST>(i, n);
                store_pop<ST>(W, i, g[0], hv, 0);
#pragma unroll
                for (int k = 1; k < Q3; ++k) store_pop<ST>(W, sl[opp3(k) - 1][tid], g[k], hv, k);
            }
            if (red) {
                su[0][tid] = (float)ux; su[1][tid] = (float)uy; su[2][tid] = (float)uz;
                __syncthreads();
                if (tid < TPB) {
                    double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        if (i < nf) acc[c] += (double)su[c][tid];
                        if (i + TPB < nf) acc[c] += (double)su[c][tid + TPB];
                    }
                    finish_tile<TPB, 1>(S, item.y, n, acc, sh, defer_slot(a));
                }
                __syncthreads();      // su and sh are reused by the next direction
            }
        }
    }
}

// Even step with its gathers staged in shared memory by cp.async: the pulls
// of all TILE_NPT voxels of a thread are issued (address from the neighbour
// record, copy straight to shared memory, no register held) before the first
// voxel is collided, so twice the loads are in flight per thread and the
// register budget stays small enough for high occupancy.  Stores go straight
// to global memory; their addresses are decoded again from the record.
template <class ST, int MINB, bool W1>
__global__ void __launch_bounds__(TPB, MINB) step3d_even_async_kernel(const StepArgs a)
{
    using T = typename ST::T;
    using Cp = typename ST::C;
    using Wd = typename ST::W;
    __shared__ double sh[TPB / 32][3];
    __shared__ Wd stage[TILE_NPT][Q3][TPB];
    const int nwork = a.nwork_dev ? *a.nwork_dev : a.nwork;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 item = a.work[w];
        const Solve3 &S = a.solves[item.x];
        const int phase = S.st->phase;
        if (phase >= PH_DONE) continue;
        const long long n = S.st->s_base + a.step + 1;
        const bool red = step_reduces(a, S.c, phase, n);
        const T *__restrict__ R = aa_src<T>(S, n);   // gathers
        T *__restrict__ W = aa_dst<T>(S, n);         // scatters
        const unsigned P = (unsigned)S.plane;
        double acc[3] = {0.0, 0.0, 0.0};
        uint4 mr[TILE_NPT];
        uint2 mr2[TILE_NPT];
        unsigned par[TILE_NPT];          // bit k: parity of the pulled element (2-byte storage)
#pragma unroll
        for (int j = 0; j < TILE_NPT; ++j) {
            const unsigned i = (unsigned)(item.y * (TPB * TILE_NPT) + j * TPB + threadIdx.x);
            const bool v = i < (unsigned)S.nfluid;
            mr[j] = v ? __ldg(S.meta + i) : make_uint4(0, 0, 0, 0);
            mr2[j] = v ? __ldg(S.meta2 + i) : make_uint2(0, 0);
        }
#pragma unroll
        for (int j = 0; j < TILE_NPT; ++j) {
            const unsigned i = (unsigned)(item.y * (TPB * TILE_NPT) + j * TPB + threadIdx.x);
            par[j] = 0;
            if (i < (unsigned)S.nfluid) {
                CNb nb;
                meta_nbrs(S, i, mr[j], mr2[j], nb);
#pragma unroll
                for (int k = 0; k < Q3; ++k) {
                    const int o = opp3(k);
                    const unsigned src = k == 0 ? i : (((nb.solid >> o) & 1u) ? (k * P + i) : (o * P + nb.idx[o]));
                    par[j] |= (src & 1u) << k;
                    __pipeline_memcpy_async(&stage[j][k][threadIdx.x], ST::word(R + src), sizeof(Wd));
                }
            }
            __pipeline_commit();
        }
#pragma unroll
        for (int j = 0; j < TILE_NPT; ++j) {
            __pipeline_wait_prior(TILE_NPT - 1 - j);
            const unsigned i = (unsigned)(item.y * (TPB * TILE_NPT) + j * TPB + threadIdx.x);
            if (i >= (unsigned)S.nfluid) continue;
            Cp g[Q3];
#pragma unroll
            for (int k = 0; k < Q3; ++k) g[k] = ST::unword(stage[j][k][threadIdx.x], (par[j] >> k) & 1u);
            Cp ux, uy, uz;
            collide3<ST, W1>(g, S, ux, uy, uz);
            CNb nb;
            meta_nbrs(S, i, mr[j], mr2[j], nb);
            const uint32_t hv = voxel_bits<ST>(i, n);
            store_pop<ST>(W, i, g[0], hv, 0);
#pragma unroll
            for (int k = 1; k < Q3; ++k) {
                const unsigned dst = ((nb.solid >> k) & 1u) ? (opp3(k) * P + i) : (k * P + nb.idx[k]);
                store_pop<ST>(W, dst, g[k], hv, k);
            }
            acc[0] += (double)ux; acc[1] += (double)uy; acc[2] += (double)uz;
        }
        if (red) finish_tile(S, item.y, n, acc, sh, defer_slot(a));
    }
}

// ------------------------------------------------------------ pull form ----
// Two-lattice ("pull") storage of the reduced-precision forms: a direction
// keeps two lattices of 19 planes (A = buffer 0, B = buffer 1), and step n
// reads buffer (n - 1) & 1 and writes buffer n & 1.  After step n a buffer
// holds the post-collision populations in natural slots, f*_k(x_i) at
// [k][i].  Step n pulls population k of voxel x from [k][rank(x - e_k)], or
// across a solid link (x - e_k solid) the bounced [opp k][i], collides, and
// writes all 19 values to its own slots [k][i]: the gathers are the only
// scattered accesses, the stores are coalesced, and no slot is both read and
// written in one step (the in-place even step reads and rewrites the same
// scattered slots).  The initial state is uniform (h = 0), which streaming
// leaves unchanged, so step 1 (the reference's collide_only priming,
// LMB3d/lbm3d-perm.cpp:249-253) is an ordinary pull step on it.  The
// collision, the random bits of every store (voxel, step, direction) and the
// flux order are those of the in-place kernels, so populations, fluxes and
// step counts are bit-identical to theirs; the second lattice doubles the
// memory of a solve.
//
// Source slots of the 19 populations of pore voxel i (src[0] = i).
template <bool META>
__device__ __forceinline__ void pull_sources(const Solve3 &S, unsigned i, unsigned P, unsigned (&src)[Q3])
{
    CNb nb;
    if constexpr (META) {
        meta_nbrs(S, i, __ldg(S.meta + i), __ldg(S.meta2 + i), nb);
    } else {
        int x, y, z;
        coords3(S, __ldg(S.fnode + i), x, y, z);
        compact_nbrs(S, i, x, y, z, nb);
    }
    src[0] = i;
#pragma unroll
    for (int k = 1; k < Q3; ++k) {
        const int o = opp3(k);
        src[k] = ((nb.solid >> o) & 1u) ? (o * P + i) : (k * P + nb.idx[o]);
    }
}

// Buffers of step n of a pull-form solve.
template <class T>
__device__ __forceinline__ const T *pull_src(const Solve3 &S, long long n)
{
    return static_cast<const T *>((n & 1) ? S.A : S.B);
}
template <class T>
__device__ __forceinline__ T *pull_dst(const Solve3 &S, long long n)
{
    return static_cast<T *>((n & 1) ? S.B : S.A);
}

// One step of a pull-form solve: thread t steps the adjacent voxels (2t,
// 2t + 1) of its tile, gathers both voxels' populations, collides them
// together in packed FP32 and stores both with paired (4- or 8-byte)
// coalesced stores.  The partner of the last voxel of an odd-sized lattice is
// a padding slot of plane stride (read and written, never used).
template <class ST, int MINB, bool W1, bool META>
__global__ void __launch_bounds__(TPB, MINB) step3d_pull_kernel(const StepArgs a)
{
    using T = typename ST::T;
    static_assert(ST::shifted && TILE_NPT == 2, "the pull form is a reduced-precision voxel-pair kernel");
    constexpr unsigned TV = TPB * TILE_NPT;
    __shared__ double sh[TPB / 32][3];
    __shared__ float su[3][TV];
    const int nwork = a.nwork_dev ? *a.nwork_dev : a.nwork;
    const unsigned tid = threadIdx.x;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 item = a.work[w];
        const Solve3 &S = a.solves[item.x];
        const int phase = S.st->phase;
        if (phase >= PH_DONE) continue;
        const long long n = S.st->s_base + a.step + 1;
        const bool red = step_reduces(a, S.c, phase, n);
        const T *__restrict__ R = pull_src<T>(S, n);
        T *__restrict__ W = pull_dst<T>(S, n);
        const unsigned P = (unsigned)S.plane, nf = (unsigned)S.nfluid;
        const unsigned ts = (unsigned)item.y * TV;
        const unsigned i0 = ts + 2u * tid;
        float2 u[3] = {};
        if (i0 < nf) {
            unsigned sa[Q3], sb[Q3];
            pull_sources<META>(S, i0, P, sa);
            if (i0 + 1u < nf) {
                pull_sources<META>(S, i0 + 1u, P, sb);
            } else {
#pragma unroll
                for (int k = 0; k < Q3; ++k) sb[k] = k * P + i0 + 1u;
            }
            float2 g[Q3];
            ST::ld2(R + i0, g[0].x, g[0].y);
#pragma unroll
            for (int k = 1; k < Q3; ++k) {
                g[k].x = ST::ld(R + sa[k]);
                g[k].y = ST::ld(R + sb[k]);
            }
            collide3x2<ST, W1>(g, S, u);
            const uint32_t h0 = voxel_bits<ST>(i0, n), h1 = voxel_bits<ST>(i0 + 1u, n);
#pragma unroll
            for (int k = 0; k < Q3; ++k)
                ST::st2(W + (k * P + i0), g[k].x, g[k].y, dir_bits(h0, k), dir_bits(h1, k));
        }
        if (red) {
            double acc[3];
            canonical_acc<TPB, 0>(su, u, tid, ts, nf, acc);
            finish_tile(S, item.y, n, acc, sh, defer_slot(a));
        }
    }
}

// Pull step with one voxel per thread at a time: thread t steps voxels t and
// t + TPB of its tile one after the other (the flux order of the in-place
// one-voxel kernels), each with 2- or 4-byte coalesced stores.
template <class ST, int MINB, bool W1, bool META>
__global__ void __launch_bounds__(TPB, MINB) step3d_pull1_kernel(const StepArgs a)
{
    using T = typename ST::T;
    using Cp = typename ST::C;
    static_assert(ST::shifted, "the pull form is a reduced-precision kernel");
    __shared__ double sh[TPB / 32][3];
    const int nwork = a.nwork_dev ? *a.nwork_dev : a.nwork;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 item = a.work[w];
        const Solve3 &S = a.solves[item.x];
        const int phase = S.st->phase;
        if (phase >= PH_DONE) continue;
        const long long n = S.st->s_base + a.step + 1;
        const bool red = step_reduces(a, S.c, phase, n);
        const T *__restrict__ R = pull_src<T>(S, n);
        T *__restrict__ W = pull_dst<T>(S, n);
        const unsigned P = (unsigned)S.plane, nf = (unsigned)S.nfluid;
        double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
        for (int j = 0; j < TILE_NPT; ++j) {
            const unsigned i = (unsigned)(item.y * (TPB * TILE_NPT) + j * TPB + threadIdx.x);
            if (i >= nf) continue;
            unsigned src[Q3];
            pull_sources<META>(S, i, P, src);
            Cp g[Q3];
#pragma unroll
            for (int k = 0; k < Q3; ++k) g[k] = ST::ld(R + src[k]);
            Cp ux, uy, uz;
            collide3<ST, W1>(g, S, ux, uy, uz);
            const uint32_t hv = voxel_bits<ST>(i, n);
#pragma unroll
            for (int k = 0; k < Q3; ++k) store_pop<ST>(W, k * P + i, g[k], hv, k);
            acc[0] += (double)ux; acc[1] += (double)uy; acc[2] += (double)uz;
        }
        if (red) finish_tile(S, item.y, n, acc, sh, defer_slot(a));
    }
}

// Pull step of a group of directions that share one structure (the grouped
// work list of the in-place link-slot kernels): the source slots of the
// tile's voxels are found once into shared memory (each thread reads back
// only its own, so no barrier) and serve every direction's gathers.  Per
// direction the arithmetic, random bits and flux order are those of
// step3d_pull_kernel.
template <class ST, int MINB, bool W1, bool META>
__global__ void __launch_bounds__(TPB, MINB) step3d_pull_group_kernel(const StepArgs a)
{
    using T = typename ST::T;
    static_assert(ST::shifted && TILE_NPT == 2, "the pull form is a reduced-precision voxel-pair kernel");
    constexpr unsigned TV = TPB * TILE_NPT;
    __shared__ double sh[TPB / 32][3];
    __shared__ float su[3][TV];
    __shared__ uint2 sl[Q3 - 1][TPB];            // source slots of population k (1..18) of the thread's pair
    const int nwork = a.nwork_dev ? *a.nwork_dev : a.nwork;
    const unsigned tid = threadIdx.x;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 item = a.work[w];
        const Solve3 &S0 = a.solves[item.x];
        const int ng = min(S0.group, MAX_GROUP);
        unsigned live = 0;
#pragma unroll
        for (int d = 0; d < MAX_GROUP; ++d)
            if (d < ng && a.solves[item.x + d].st->phase < PH_DONE) live |= 1u << d;
        if (!live) continue;
        const unsigned P = (unsigned)S0.plane, nf = (unsigned)S0.nfluid;
        const unsigned ts = (unsigned)item.y * TV;
        const unsigned i0 = ts + 2u * tid;
        if (i0 < nf) {
            unsigned sa[Q3], sb[Q3];
            pull_sources<META>(S0, i0, P, sa);
            if (i0 + 1u < nf) {
                pull_sources<META>(S0, i0 + 1u, P, sb);
            } else {
#pragma unroll
                for (int k = 0; k < Q3; ++k) sb[k] = k * P + i0 + 1u;
            }
#pragma unroll
            for (int k = 1; k < Q3; ++k) sl[k - 1][tid] = make_uint2(sa[k], sb[k]);
        }
#pragma unroll 1
        for (int d = 0; d < ng; ++d) {
            if (!((live >> d) & 1u)) continue;
            const Solve3 &S = a.solves[item.x + d];
            const long long n = S.st->s_base + a.step + 1;
            const bool red = step_reduces(a, S.c, S.st->phase, n);
            const T *__restrict__ R = pull_src<T>(S, n);
            T *__restrict__ W = pull_dst<T>(S, n);
            float2 u[3] = {};
            if (i0 < nf) {
                float2 g[Q3];
                ST::ld2(R + i0, g[0].x, g[0].y);
#pragma unroll
                for (int k = 1; k < Q3; ++k) {
                    const uint2 s = sl[k - 1][tid];
                    g[k].x = ST::ld(R + s.x);
                    g[k].y = ST::ld(R + s.y);
                }
                collide3x2<ST, W1>(g, S, u);
                const uint32_t h0 = voxel_bits<ST>(i0, n), h1 = voxel_bits<ST>(i0 + 1u, n);
#pragma unroll
                for (int k = 0; k < Q3; ++k)
                    ST::st2(W + (k * P + i0), g[k].x, g[k].y, dir_bits(h0, k), dir_bits(h1, k));
            }
            if (red) {
                double acc[3];
                canonical_acc<TPB, 0>(su, u, tid, ts, nf, acc);
                finish_tile(S, item.y, n, acc, sh, defer_slot(a));
            }
        }
    }
}

// Pore-rank tables (once per structure).
constexpr int SCAN_WORDS = 1024;    // mask words per block of the scan kernels
__global__ void word_sums_kernel(const uint32_t *mask, long long nwords, unsigned *bsum);
__global__ void word_scan_kernel(const uint32_t *mask, long long nwords, const unsigned *boff, uint32_t *wpre);
__global__ void scatter_fnode_kernel(const uint32_t *mask, const uint32_t *wpre, long long nwords, int wpr,
                                     int nx, uint32_t *fnode);
__global__ void build_meta_kernel(Solve3 S, uint4 *meta, uint2 *meta2);

// After a chunk of `steps` launches, solves still running have advanced by it.
__global__ void advance3d_kernel(Solve3 *solves, int nsolves, long long steps);

// Deferred reduction of the launches with relative steps step0 .. step0 +
// nsteps - 1 (nsteps <= DEFER_SLOTS, within one block of DEFER_SLOTS): the
// fluxes (qbuf: per solve and step, q[3] and a flag), then the controllers
// in step order.  mode: StepArgs::defer of those launches.
cudaError_t launch_deferred3d(const Solve3 *solves, int nsolves, long long step0, int nsteps, double *qbuf,
                              int mode, cudaStream_t s);

// Initial state: every population at rest (f = w, or h = 0 when shifted).
template <class ST>
__global__ void init3d_kernel(void *A, long long plane, long long n)
{
    using T = typename ST::T;
    T *a = static_cast<T *>(A);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < Q3; ++k) {
            if constexpr (ST::shifted) a[k * plane + i] = T(0.0f);
            else a[k * plane + i] = (T)ST::init(k);
        }
}

// Post-collision populations f*_k(x) of the last completed step `done`
// (canonical, as the reference's f0 holds them) into the dense AoS f_out, and/or
// the velocity of that step recovered from them: Guo forcing gives
// j* = j + F, so u = (j* - F/2) / rho.  Solid voxels are left untouched
// (the caller zeroes the outputs).
template <class ST>
__global__ void canon3d_kernel(const Solve3 S, long long done, double *f_out, float *u_out)
{
    using T = typename ST::T;
    const T *A = static_cast<const T *>(S.A);
    const unsigned P = (unsigned)S.plane;
    const double isc = (double)S.inv_scale;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < (unsigned)S.nfluid;
         i += gridDim.x * blockDim.x) {
        const unsigned node = S.fnode[i];
        int x, y, z;
        coords3(S, node, x, y, z);
        CNb nb;
        compact_nbrs(S, i, x, y, z, nb);
        double f[Q3];
        // pull form: the buffer step `done` wrote holds f*_k at [k][i] (the
        // initial state, done = 0, sits in A); two-lattice AA form: the
        // in-place slots, in the buffer step `done` wrote (aa_dst)
        const T *Ab = S.pull ? static_cast<const T *>((done & 1ll) ? S.B : S.A)
                    : S.aa2 ? aa_buf<const T>(S, done >> 1) : A;
#pragma unroll
        for (int k = 0; k < Q3; ++k) {
            const int o = opp3(k);
            unsigned at;
            if (done == 0 || S.pull) at = k * P + i;                // initial, pre-collision / pull form
            else if (done & 1ll) at = o * P + i;                    // after a local step
            else if (k == 0) at = i;
            else if ((nb.solid >> k) & 1u) at = o * P + i;
            else at = k * P + nb.idx[k];
            const double v = (double)ST::ld(Ab + at);
            f[k] = ST::shifted ? v * isc + w3(k) : v;
        }
        if (f_out)
            for (int k = 0; k < Q3; ++k) f_out[(size_t)node * Q3 + k] = f[k];
        if (u_out) {
            double rho = 0.0, jx = 0.0, jy = 0.0, jz = 0.0;
            for (int k = 0; k < Q3; ++k) {
                rho += f[k]; jx += f[k] * ex3(k); jy += f[k] * ey3(k); jz += f[k] * ez3(k);
            }
            const double sh = done == 0 ? 0.5 : -0.5;   // pre-collision state needs +F/2
            u_out[3 * (size_t)node] = (float)((jx + sh * S.P.F[0]) / rho);
            u_out[3 * (size_t)node + 1] = (float)((jy + sh * S.P.F[1]) / rho);
            u_out[3 * (size_t)node + 2] = (float)((jz + sh * S.P.F[2]) / rho);
        }
    }
}

// Host-side launchers, one per translation unit (FP64 is compiled without FMA
// contraction to keep the reference's rounding).
// `odd`: launch the odd-step (local) kernel, else the even-step one; every
// solve in the launch must be at a step of that parity.
cudaError_t launch_step3d_f64(int variant, bool odd, dim3 grid, cudaStream_t s, const StepArgs &a);
cudaError_t launch_step3d_lp(int prec, int variant, bool w1, bool odd, dim3 grid, cudaStream_t s, const StepArgs &a);
cudaError_t launch_init3d(int prec, void *A, long long plane, long long n, cudaStream_t s);
// Allow the bulk-staged odd kernels their shared-memory ring on device `dev`
// (once per device, before any launch or capture).
cudaError_t prepare_step3d_lp(int dev);
cudaError_t launch_canon3d(int prec, const Solve3 &S, long long done, double *f, float *u, cudaStream_t s);
int max_blocks_step3d(int prec, int variant, bool odd);
inline bool is_moment(int prec) { return prec == 4 || prec == 5; }
inline bool is_dense_m(int prec) { return prec == 6; }
// Dense moment form variants: z-segment length (planes per tile) x
// shared-memory ring depth x register budget.
constexpr int NVAR_MD = 4;
__host__ __device__ constexpr int md_lz(int v) { return v == 1 ? 32 : v == 2 ? 8 : 16; }
inline int variant_count(int prec) { return prec == 0 ? 2 * NVAR_F64 : prec == 6 ? NVAR_MD : (prec >= 4 ? 3 : AA2_BASE_LP + NVAR_LP); }
// pore voxels per tile (in units of TPB) of a solve's tile list
inline int variant_npt(int prec, int) { return prec >= 4 ? 1 : TILE_NPT; }

}  // namespace lbm
