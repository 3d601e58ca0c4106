// liblbm host engine: contexts, structure upload and bit packing, the plain
// solve loops (one launch per step, on-device convergence controller, one
// host synchronisation per convergence check), velocity export and the
// diagnostic entry points.  The C ABI is declared in include/lbm.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lbm.h"
#include "engine2d.cuh"
#include "engine_host.h"
#include "engine_m.cuh"
#include "engine_md.cuh"

using namespace lbm;

// ------------------------------------------------------------- utilities ----
int lbm_fail_cuda(lbm_ctx *ctx, cudaError_t e, const char *what, int line)
{
    if (ctx)
        ctx->err = std::string("CUDA error: ") + cudaGetErrorString(e) + " in " + what +
                   " (engine line " + std::to_string(line) + ")";
    return LBM_ECUDA;
}

int lbm_fail_input(lbm_ctx *ctx, const std::string &msg)
{
    if (ctx) ctx->err = msg;
    return LBM_EINPUT;
}

bool lbm_is_device_ptr(const void *p)
{
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Pack a byte mask (x fastest, 1 = solid) into rows of 32-bit words, count
// the pore voxels and flag any value other than 0/1 (LMB3d/lbm3d-perm.cpp:190-192).
__global__ void pack_mask_kernel(const uint8_t *__restrict__ solid, int nx, long long rows, int wpr,
                                 uint32_t *__restrict__ mask, unsigned long long *npore, unsigned *bad)
{
    const long long total = rows * wpr;
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < total;
         w += (long long)gridDim.x * blockDim.x) {
        const long long r = w / wpr;
        const int c = (int)(w - r * wpr);
        const int x0 = c * 32;
        const uint8_t *row = solid + r * nx;
        uint32_t bits = 0;
        unsigned cnt = 0, b = 0;
        for (int i = 0; i < 32; ++i) {
            if (x0 + i >= nx) { bits |= 1u << i; continue; }   // past the row end: solid
            const uint8_t v = row[x0 + i];
            b |= v > 1;
            if (v) bits |= 1u << i; else ++cnt;
        }
        mask[w] = bits;
        if (cnt) atomicAdd(npore, (unsigned long long)cnt);
        if (b) atomicOr(bad, 1u);
    }
}

int lbm_upload_mask(lbm_ctx *ctx, const uint8_t *solid, int nx, long long rows, DevMem &mask,
                    long long &npore)
{
    const long long nn = (long long)nx * rows;
    const int wpr = (nx + 31) / 32;
    DevMem staging(ctx->stream), scratch(ctx->stream);
    const uint8_t *src = solid;
    if (!lbm_is_device_ptr(solid)) {
        CK(staging.alloc((size_t)nn));
        CK(cudaMemcpyAsync(staging.p, solid, (size_t)nn, cudaMemcpyHostToDevice, ctx->stream));
        src = static_cast<const uint8_t *>(staging.p);
    }
    CK(mask.alloc(sizeof(uint32_t) * (size_t)rows * wpr));
    CK(scratch.alloc(16));
    CK(cudaMemsetAsync(scratch.p, 0, 16, ctx->stream));
    auto *cnt = static_cast<unsigned long long *>(scratch.p);
    auto *bad = reinterpret_cast<unsigned *>(cnt + 1);
    const long long words = rows * wpr;
    const int blocks = (int)std::min<long long>((words + 255) / 256, 4L * 1184);
    pack_mask_kernel<<<blocks, 256, 0, ctx->stream>>>(src, nx, rows, wpr, static_cast<uint32_t *>(mask.p), cnt, bad);
    CK(cudaGetLastError());
    unsigned long long h[2] = {0, 0};
    CK(cudaMemcpyAsync(h, scratch.p, 16, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if ((unsigned)h[1]) return lbm_fail_input(ctx, "non-binary voxel");
    npore = (long long)h[0];
    if (npore == 0) return lbm_fail_input(ctx, "structure has no pore space");
    return LBM_OK;
}

// ------------------------------------------------------------- context ------
extern "C" int lbm_version(void) { return LBM_API_VERSION; }

extern "C" int lbm_create(lbm_ctx **out, int device)
{
    if (!out) return LBM_EINPUT;
    *out = nullptr;
    lbm_ctx *ctx = new lbm_ctx();
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = prepare_step3d_lp(device);
    if (e == cudaSuccess) {
        // keep up to 4 GiB of freed lattices in the device's stream-ordered
        // pool between solves instead of returning them to the driver at
        // every synchronisation (repeated solves then reuse mapped memory)
        cudaMemPool_t pool = nullptr;
        e = cudaDeviceGetDefaultMemPool(&pool, device);
        unsigned long long keep = 4ull << 30;
        if (e == cudaSuccess) e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e != cudaSuccess) {
        lbm_last_error_global() = std::string("CUDA error: ") + cudaGetErrorString(e);
        delete ctx;
        return LBM_ECUDA;
    }
    *out = ctx;
    return LBM_OK;
}

extern "C" void lbm_destroy(lbm_ctx *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

std::string &lbm_last_error_global()
{
    static std::string s;
    return s;
}

extern "C" void *lbm_stream(const lbm_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

extern "C" const char *lbm_last_error(const lbm_ctx *ctx)
{
    return ctx ? ctx->err.c_str() : lbm_last_error_global().c_str();
}

// --------------------------------------------------------------- 3D ---------
int lbm_check_params3d(lbm_ctx *ctx, const lbm_params3d &p)
{
    if (!(p.tau > 0.5)) return lbm_fail_input(ctx, "tau must exceed 0.5");
    if (p.lag <= 0) return lbm_fail_input(ctx, "--lag must be positive");
    if (p.precision < LBM_FP64 || p.precision > LBM_MD32) return lbm_fail_input(ctx, "unknown precision");
    if ((is_moment(p.precision) || is_dense_m(p.precision)) && p.tau != 1.0)
        return lbm_fail_input(ctx, "moment-projected storage needs tau = 1");
    if (p.criterion != LBM_CRIT_DRIFT && p.criterion != LBM_CRIT_BLOCK && p.criterion != LBM_CRIT_BATCH)
        return lbm_fail_input(ctx, "unknown criterion");
    if (p.criterion != LBM_CRIT_DRIFT && (p.sample <= 0 || p.lag % p.sample != 0))
        return lbm_fail_input(ctx, "block criterion needs sample > 0 dividing lag");
    if (p.variant != LBM_VARIANT_DEFAULT && (p.variant < 0 || p.variant >= variant_count(p.precision)))
        return lbm_fail_input(ctx, "unknown step-kernel variant");
    return LBM_OK;
}

// The autotuner's pick on the 128^3 tensor workload: FP32 the pull form
// (voxel pairs, ranks from the neighbour record, 3 blocks per SM); 16-bit
// the two-lattice AA form of the bulk-staged odd step + the grouped even
// step with the link slots shared by the directions (4 blocks per SM).
int lbm_default_variant(int prec)
{
    if (prec == LBM_FP32) return NVAR_LP + 1;
    if (prec == LBM_FP16 || prec == LBM_BF16) return AA2_BASE_LP + 4 * NVAR_EVEN_LP + 9;
    return 0;
}

// The batch's default: the solve default (its 16-bit pick has a grouped even
// step, which the batch runs over runs of a structure's consecutive slots).
int lbm_default_batch_variant(int prec)
{
    return lbm_default_variant(prec);
}

static lbm_params3d lbm_resolve_variant(lbm_params3d p)
{
    if (p.variant == LBM_VARIANT_DEFAULT) p.variant = lbm_default_variant(p.precision);
    return p;
}

static size_t elem_size(int prec) { return prec == LBM_FP64 ? 8 : (prec == LBM_FP32 ? 4 : 2); }

long long lbm_plane_elems(long long nn) { return (nn + 63) / 64 * 64; }

// Lattice bytes of one direction over n pore voxels.
long long lbm_lattice_bytes3d(long long n, int prec)
{
    if (is_moment(prec)) return 2ll * mom_buffer_bytes(prec, n);
    return (long long)Q3 * lbm_plane_elems(n) * (long long)elem_size(prec);
}

// Lattice bytes of one direction of a filled solve record (both lattices of
// the pull and two-lattice AA forms).
long long lbm_lattice_bytes(const Solve3 &S)
{
    if (is_dense_m(S.prec)) return md_lattice_bytes(S.md);
    return lbm_lattice_bytes3d(S.nfluid, S.prec) * ((S.pull || S.aa2) ? 2 : 1);
}

// Point a solve record at its lattice memory (lbm_lattice_bytes(S) bytes);
// the second lattice of the two-lattice forms follows the first.
void lbm_attach_lattice(Solve3 &S, void *p)
{
    S.A = p;
    S.B = (S.pull || S.aa2) ? static_cast<char *>(p) + lbm_lattice_bytes3d(S.nfluid, S.prec) : nullptr;
}

// Plane stride (populations) or record slots per buffer (moments).
long long lbm_plane_for(int prec, long long n)
{
    return is_moment(prec) ? mom_slots(n) : lbm_plane_elems(n);
}

// A variant whose even kernel reads neighbour records needs them built.
int lbm_effective_variant(int prec, int variant, bool have_meta)
{
    if (is_moment(prec) || is_dense_m(prec) || have_meta) return variant;
    if (is_aa2_variant(prec, variant))
        return aa2_base(prec) + lbm_effective_variant(prec, kernel_variant(prec, variant), false);
    if (is_pull_variant(prec, variant))
        return pull_meta(variant - NVAR_LP) ? NVAR_LP + 2 : variant;   // pull, ranks from the mask
    const int ve = variant % nvar_even(prec);
    if (!even_meta(ve)) return variant;
    if (even_wide(ve)) return variant - ve + 14;        // link slots, one voxel per thread, ranks from the mask
    if (even_links(ve)) return variant - ve + 10;       // grouped link slots (one voxel at a time), ranks from the mask
    if (even_grouped(ve)) return variant - ve + 6;      // grouped, ranks from the mask
    return variant - ve + (ve & 1) + 2;                 // same budget, ranks from the mask
}

// Does this (effective) variant run the grouped even kernel?
bool lbm_grouped_variant(int prec, int variant)
{
    if (is_pull_variant(prec, variant)) return pull_grouped(variant - NVAR_LP);
    variant = kernel_variant(prec, variant);
    return prec >= LBM_FP32 && prec <= LBM_BF16 && even_grouped(variant % NVAR_EVEN_LP);
}

// Do all launches (not only the even ones) of this variant take the grouped work list?
bool lbm_grouped_all(int prec, int variant)
{
    return is_pull_variant(prec, variant) && pull_grouped(variant - NVAR_LP);
}

// Work list of the grouped even step over solves that share one structure:
// runs of up to MAX_GROUP consecutive records, led by the first of each run.
static void lbm_group_items(std::vector<Solve3> &hs, std::vector<int2> &items)
{
    const int n = (int)hs.size();
    for (auto &S : hs) S.group = 0;
    for (int j = 0; j < n; j += MAX_GROUP) {
        hs[j].group = std::min(MAX_GROUP, n - j);
        for (int t = 0; t < hs[j].ntiles; ++t) items.push_back(make_int2(j, t));
    }
}

cudaError_t lbm_launch_step(int prec, int variant, bool w1, bool odd, dim3 grid, cudaStream_t s, const StepArgs &a)
{
    if (prec == LBM_FP64) return launch_step3d_f64(variant, odd, grid, s, a);
    if (is_dense_m(prec)) return launch_stepmd(variant, grid, s, a);
    if (is_moment(prec)) return launch_stepm(prec, variant, grid, s, a);
    return launch_step3d_lp(prec, variant, w1, odd, grid, s, a);
}

int lbm_max_blocks(int prec, int variant, bool odd)
{
    if (is_dense_m(prec)) return max_blocks_stepmd(variant);
    return is_moment(prec) ? max_blocks_stepm(prec, variant) : max_blocks_step3d(prec, variant, odd);
}

cudaError_t lbm_init_lattice(int prec, const Solve3 &S, cudaStream_t s)
{
    if (is_dense_m(prec)) return init_md_lattice(S, s);   // tensor maps; step 1 writes the records
    if (is_moment(prec)) return cudaSuccess;        // step 1 writes the moments from scratch
    return launch_init3d(prec, S.A, S.plane, S.nfluid, s);
}

cudaError_t lbm_canon(int prec, const Solve3 &S, long long done, double *f, float *u, cudaStream_t s)
{
    if (is_dense_m(prec)) return launch_canonmd(S, done, f, u, s);
    if (is_moment(prec)) return launch_canonm(prec, S, done, f, u, s);
    return launch_canon3d(prec, S, done, f, u, s);
}

void lbm_fill_solve3(Solve3 &S, int nx, int ny, int nz, const double F[3], const lbm_params3d &p, int npt)
{
    memset(&S, 0, sizeof(S));
    S.prec = p.precision;
    S.pull = is_pull_variant(p.precision, p.variant) ? 1 : 0;
    S.aa2 = is_aa2_variant(p.precision, p.variant) ? 1 : 0;
    S.nx = nx; S.ny = ny; S.nz = nz;
    S.wpr = (nx + 31) / 32;
    S.nn = (long long)nx * ny * nz;
    S.plane = lbm_plane_elems(S.nn);
    S.ntiles = (int)((S.nn + TPB * npt - 1) / (TPB * npt));
    if (is_dense_m(p.precision)) md_fill_geom(S.md, nx, ny, nz, p.variant, S.ntiles);
    S.dvx.init(nx);
    S.dvy.init(ny);
    Phys3 &P = S.P;
    for (int c = 0; c < 3; ++c) { P.F[c] = F[c]; P.Ff[c] = (float)F[c]; }
    P.tau = p.tau;
    P.pref = 1.0 - 0.5 / p.tau;
    P.omega = (float)(1.0 / p.tau);
    P.preff = (float)P.pref;
    // FP16 keeps h * scale; scale puts the largest plausible deviation
    // (Poiseuille peak |F| L^2 / 8 nu over the longest axis) near 2^12, far
    // from both the overflow at 65504 and the subnormal range.
    double scale = 1.0;
    if (p.precision == LBM_FP16) {
        const double nu = (p.tau - 0.5) / 3.0;
        const double L = (double)std::max(nx, std::max(ny, nz));
        const double fmag = std::sqrt(F[0] * F[0] + F[1] * F[1] + F[2] * F[2]);
        const double uest = fmag * L * L / (8.0 * nu);
        scale = uest > 0 ? std::exp2(std::round(std::log2(4096.0 / uest))) : 1.0;
        scale = std::min(std::max(scale, 1.0), std::exp2(40.0));
    }
    S.scale = (float)scale;
    S.inv_scale = (float)(1.0 / scale);
    Ctl3 &c = S.c;
    c.eps = p.eps; c.lag = p.lag; c.min_steps = p.min_steps; c.max_steps = p.max_steps;
    c.avg_steps = p.avg_steps; c.hold = p.hold; c.criterion = p.criterion;
    c.sample = p.sample > 0 ? p.sample : 1; c.ksigma = p.ksigma;
}

void lbm_init_state3(State3 &st, const Ctl3 &c)
{
    memset(&st, 0, sizeof(st));
    st.phase = PH_RUN;
    if (c.max_steps <= 0) {
        // no run-in steps: converged iff hold <= 0 (LMB3d/lbm3d-perm.cpp:362)
        st.converged = 0 >= c.hold ? 1 : 0;
        if (c.avg_steps <= 0) { st.phase = PH_DONE; st.steps = 0; }
        else { st.phase = PH_AVG; st.avg_start = 0; }
    }
}

int lbm_pick_npt(const lbm_params3d &p) { return variant_npt(p.precision, p.variant); }

int lbm_build_pores(lbm_ctx *ctx, Solve3 &S, int npt, DevMem &wpre, DevMem &fnode, DevMem &meta, DevMem &meta2)
{
    const long long nwords = (long long)S.wpr * S.ny * S.nz;
    const int blocks = (int)((nwords + SCAN_WORDS - 1) / SCAN_WORDS);
    DevMem bsum(ctx->stream), boff(ctx->stream);
    CK(bsum.alloc(sizeof(unsigned) * (size_t)blocks));
    CK(boff.alloc(sizeof(unsigned) * (size_t)blocks));
    CK(wpre.alloc(sizeof(uint32_t) * (size_t)(nwords + 1)));
    word_sums_kernel<<<blocks, TPB, 0, ctx->stream>>>(S.mask, nwords, static_cast<unsigned *>(bsum.p));
    CK(cudaGetLastError());
    std::vector<unsigned> h(blocks);
    CK(cudaMemcpyAsync(h.data(), bsum.p, sizeof(unsigned) * blocks, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    unsigned long long total = 0;
    for (int b = 0; b < blocks; ++b) { const unsigned c = h[b]; h[b] = (unsigned)total; total += c; }
    const uint32_t tot32 = (uint32_t)total;
    CK(cudaMemcpyAsync(boff.p, h.data(), sizeof(unsigned) * blocks, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(static_cast<uint32_t *>(wpre.p) + nwords, &tot32, sizeof(uint32_t),
                       cudaMemcpyHostToDevice, ctx->stream));
    word_scan_kernel<<<blocks, TPB, 0, ctx->stream>>>(S.mask, nwords, static_cast<const unsigned *>(boff.p),
                                                      static_cast<uint32_t *>(wpre.p));
    CK(cudaGetLastError());
    CK(fnode.alloc(sizeof(uint32_t) * (size_t)std::max<unsigned long long>(total, 1)));
    const int sb = (int)std::min<long long>((nwords + 255) / 256, 8L * 1184);
    scatter_fnode_kernel<<<sb, 256, 0, ctx->stream>>>(S.mask, static_cast<const uint32_t *>(wpre.p), nwords,
                                                      S.wpr, S.nx, static_cast<uint32_t *>(fnode.p));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));   // host staging must outlive the copies
    S.wpre = static_cast<const uint32_t *>(wpre.p);
    S.fnode = static_cast<const uint32_t *>(fnode.p);
    S.nfluid = (int)total;
    if (is_dense_m(S.prec)) {
        // dense moment form: tiles cover the box; the padded byte mask
        // replaces the neighbour records
        S.meta = nullptr;
        S.meta2 = nullptr;
        CK(meta.alloc((size_t)md_pmask_bytes(S.md, S.ny, S.nz)));
        S.md.pmask = static_cast<const uint8_t *>(meta.p);
        CK(launch_padmask(S, ctx->stream));
        return LBM_OK;
    }
    S.plane = lbm_plane_for(S.prec, (long long)total);
    S.ntiles = (int)((total + (unsigned long long)TPB * npt - 1) / ((unsigned long long)TPB * npt));
    if (S.ntiles == 0) S.ntiles = 1;
    S.meta = nullptr;
    S.meta2 = nullptr;
    // neighbour records (24 B per pore voxel) for the even-step kernels that
    // read them; in-row offsets are 16-bit, so rows up to 65535 voxels
    if (S.nx <= 65535 && total > 0) {
        CK(meta.alloc(sizeof(uint4) * (size_t)total));
        CK(meta2.alloc(sizeof(uint2) * (size_t)total));
        const int mb = (int)std::min<unsigned long long>((total + 255) / 256, 8ull * 1184);
        build_meta_kernel<<<mb, 256, 0, ctx->stream>>>(S, static_cast<uint4 *>(meta.p), static_cast<uint2 *>(meta2.p));
        CK(cudaGetLastError());
        S.meta = static_cast<const uint4 *>(meta.p);
        S.meta2 = static_cast<const uint2 *>(meta2.p);
    }
    return LBM_OK;
}

void lbm_copy_pores(Solve3 &dst, const Solve3 &src)
{
    dst.wpre = src.wpre; dst.fnode = src.fnode; dst.nfluid = src.nfluid;
    dst.meta = src.meta; dst.meta2 = src.meta2;
    dst.plane = src.plane; dst.ntiles = src.ntiles;
    dst.md.pmask = src.md.pmask;
}

// Run a set of 3D solves sharing one mask to completion, one launch per step.
// The host synchronises only where the controller can change phase: on lag
// multiples and max_steps in phase 1, at the end of the averaging phase.  In
// between, whole chunks of kGraphSteps3 launches (an even count, starting on
// an even step, plus the s_base advance) are replayed from a CUDA graph, which
// removes the per-launch overhead that dominates small structures; the step
// numbers and kernels are those of single launches.
constexpr int kGraphSteps3 = 64;

// Does a solve of this precision reduce its flux through deferred slots (its
// partials buffer then holds DEFER_SLOTS x ntiles x 3 doubles)?  The dense
// moment form keeps the immediate reduction (its tiles have their own block
// size).
bool lbm_defers(int prec) { return !is_dense_m(prec); }

long long lbm_partial_doubles(int prec, int ntiles)
{
    return 3ll * ntiles * (lbm_defers(prec) ? DEFER_SLOTS : 1);
}

static int run_plain3d(lbm_ctx *ctx, std::vector<Solve3> &hs, Solve3 *d_solves, State3 *d_states,
                       const int2 *d_work, int nwork, int prec, int variant, std::vector<State3> &hst)
{
    const int n = (int)hs.size();
    bool w1 = true;
    for (const Solve3 &S : hs) w1 = w1 && S.P.tau == 1.0;
    variant = lbm_effective_variant(prec, variant, hs.empty() || hs[0].meta != nullptr);
    long long s = 0, base = 0;        // steps done; s_base of the unfinished solves (host copy)
    const bool defer = lbm_defers(prec);
    DevMem qbuf(ctx->stream);
    if (defer) CK(qbuf.alloc(sizeof(double) * 4 * DEFER_SLOTS * (size_t)std::max(1, n)));
    double *qb = static_cast<double *>(qbuf.p);
    long long pend0 = 0;              // deferred single launches not yet reduced: [pend0, pend0 + pending)
    int pending = 0;
    StepArgs a;
    a.solves = d_solves; a.work = d_work; a.nwork_dev = nullptr; a.nwork = nwork;
    a.defer = defer ? 1 : 0;
    StepArgs ae = a;                  // even steps (grouped work list for grouped variants)
    DevMem gwork(ctx->stream);
    if (lbm_grouped_variant(prec, variant)) {
        std::vector<int2> items;
        lbm_group_items(hs, items);
        CK(gwork.alloc(sizeof(int2) * items.size()));
        CK(cudaMemcpyAsync(gwork.p, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(d_solves, hs.data(), sizeof(Solve3) * n, cudaMemcpyHostToDevice, ctx->stream));
        ae.work = static_cast<const int2 *>(gwork.p);
        ae.nwork = (int)items.size();
    }
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    struct GraphGuard {
        cudaGraph_t &g; cudaGraphExec_t &e;
        ~GraphGuard() { if (e) cudaGraphExecDestroy(e); if (g) cudaGraphDestroy(g); }
    } guard{graph, exec};
    a.wait_ns = ctx->test_wait_ns;
    a.starve = ctx->test_starve;
    ae.wait_ns = a.wait_ns;
    ae.starve = a.starve;
    const bool gall = lbm_grouped_all(prec, variant);
    auto launch = [&](long long rel, bool odd) {
        StepArgs x = (odd && !gall) ? a : ae;
        x.step = rel;
        return lbm_launch_step(prec, variant, w1, odd, dim3(x.nwork), ctx->stream, x);
    };
    // reduce and control the deferred single launches (before s_base moves,
    // before a chunk reuses their slots, and before the states are read)
    auto flush = [&]() -> cudaError_t {
        if (!pending) return cudaSuccess;
        const cudaError_t e = launch_deferred3d(d_solves, n, pend0, pending, qb, 1, ctx->stream);
        pending = 0;
        return e;
    };
    for (;;) {
        CK(cudaMemcpyAsync(hst.data(), d_states, sizeof(State3) * n, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        long long target = LLONG_MAX;
        for (int j = 0; j < n; ++j) {
            const State3 &st = hst[j];
            const Ctl3 &c = hs[j].c;
            if (st.phase == PH_RUN) {
                long long nx = (s / c.lag + 1) * c.lag;
                if (c.max_steps > s) nx = std::min(nx, c.max_steps);
                target = std::min(target, nx);
            } else if (st.phase == PH_AVG) {
                target = std::min(target, st.avg_start + c.avg_steps);
            }
        }
        if (target == LLONG_MAX) break;
        if (!exec && target - s >= 2 * kGraphSteps3) {
            CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t e = cudaSuccess;
            // launch i of a chunk runs step i + 1 after s_base (s_base even)
            for (int i = 0; i < kGraphSteps3 && e == cudaSuccess; ++i) e = launch(i, ((i + 1) & 1) == 1);
            if (e == cudaSuccess && defer) e = launch_deferred3d(d_solves, n, 0, kGraphSteps3, qb, 1, ctx->stream);
            if (e == cudaSuccess) {
                advance3d_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(d_solves, n, kGraphSteps3);
                e = cudaGetLastError();
            }
            const cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &graph);
            CK(e);
            CK(e2);
            CK(cudaGraphInstantiate(&exec, graph, 0));
        }
        while (s < target) {
            if (exec && (s & 1) == 0 && target - s >= kGraphSteps3) {
                CK(flush());
                if (base != s) {
                    // a chunk numbers its steps from s_base: catch up with the single steps
                    advance3d_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(d_solves, n, s - base);
                    CK(cudaGetLastError());
                    base = s;
                }
                CK(cudaGraphLaunch(exec, ctx->stream));
                s += kGraphSteps3;
                base += kGraphSteps3;
            } else {
                // every unfinished solve of the call is at step s + 1 (they start together)
                CK(launch(s - base, ((s + 1) & 1) == 1));
                if (defer) {
                    if (!pending) pend0 = s - base;
                    if (++pending == DEFER_SLOTS) CK(flush());
                }
                ++s;
            }
        }
        CK(flush());
    }
    return LBM_OK;
}

extern "C" int lbm_solve3d(lbm_ctx *ctx, const uint8_t *solid, int nx, int ny, int nz,
                           int ndir, const double *forces, const lbm_params3d *params,
                           lbm_result3d *results, float *vel_out)
{
    if (!ctx) return LBM_EINPUT;
    if (!solid || !forces || !params || !results || ndir <= 0)
        return lbm_fail_input(ctx, "null argument");
    CK(cudaSetDevice(ctx->device));
    if (nx <= 0 || ny <= 0 || nz <= 0) return lbm_fail_input(ctx, "bad dimensions");
    const long long nn = (long long)nx * ny * nz;
    if (nn >= (1ll << 31) || (long long)Q3 * lbm_plane_elems(nn) >= (1ll << 32))
        return lbm_fail_input(ctx, "lattice too large (19 x nodes must stay below 2^32)");
    int rc = lbm_check_params3d(ctx, *params);
    if (rc) return rc;
    const lbm_params3d p = lbm_resolve_variant(*params);
    const int prec = p.precision, npt = lbm_pick_npt(p);

    DevMem mask(ctx->stream);
    long long npore = 0;
    rc = lbm_upload_mask(ctx, solid, nx, (long long)ny * nz, mask, npore);
    if (rc) return rc;

    std::vector<Solve3> hs(ndir);
    std::vector<State3> hst(ndir);
    std::vector<DevMem> lat, part;
    lat.reserve(ndir); part.reserve(ndir);
    DevMem d_states(ctx->stream), d_solves(ctx->stream), d_work(ctx->stream);
    DevMem wpre(ctx->stream), fnode(ctx->stream), meta(ctx->stream), meta2(ctx->stream);
    Solve3 proto;
    lbm_fill_solve3(proto, nx, ny, nz, forces, p, npt);
    proto.mask = static_cast<const uint32_t *>(mask.p);
    rc = lbm_build_pores(ctx, proto, npt, wpre, fnode, meta, meta2);
    if (rc) return rc;
    CK(d_states.alloc(sizeof(State3) * ndir));
    for (int j = 0; j < ndir; ++j) {
        Solve3 &S = hs[j];
        lbm_fill_solve3(S, nx, ny, nz, forces + 3 * j, p, npt);
        lbm_copy_pores(S, proto);
        lat.emplace_back(ctx->stream);
        part.emplace_back(ctx->stream);
        CK(lat.back().alloc((size_t)lbm_lattice_bytes(S)));
        CK(part.back().alloc(sizeof(double) * (size_t)lbm_partial_doubles(prec, S.ntiles)));
        lbm_attach_lattice(S, lat.back().p);
        S.mask = static_cast<const uint32_t *>(mask.p);
        S.partials = static_cast<double *>(part.back().p);
        S.st = static_cast<State3 *>(d_states.p) + j;
        lbm_init_state3(hst[j], S.c);
        CK(lbm_init_lattice(prec, S, ctx->stream));
    }
    std::vector<int2> work;
    for (int j = 0; j < ndir; ++j)
        for (int t = 0; t < hs[j].ntiles; ++t) work.push_back(make_int2(j, t));
    CK(d_solves.alloc(sizeof(Solve3) * ndir));
    CK(d_work.alloc(sizeof(int2) * work.size()));
    CK(cudaMemcpyAsync(d_solves.p, hs.data(), sizeof(Solve3) * ndir, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_work.p, work.data(), sizeof(int2) * work.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_states.p, hst.data(), sizeof(State3) * ndir, cudaMemcpyHostToDevice, ctx->stream));

    rc = run_plain3d(ctx, hs, static_cast<Solve3 *>(d_solves.p), static_cast<State3 *>(d_states.p),
                     static_cast<const int2 *>(d_work.p), (int)work.size(), prec, p.variant, hst);
    if (rc) return rc;

    if (vel_out) {
        const bool dev = lbm_is_device_ptr(vel_out);
        DevMem vbuf(ctx->stream);
        if (!dev) CK(vbuf.alloc(sizeof(float) * 3 * (size_t)nn));
        for (int j = 0; j < ndir; ++j) {
            float *dst = dev ? vel_out + 3 * nn * j : static_cast<float *>(vbuf.p);
            CK(cudaMemsetAsync(dst, 0, sizeof(float) * 3 * (size_t)nn, ctx->stream));   // solids: u = 0
            CK(lbm_canon(prec, hs[j], hst[j].steps, nullptr, dst, ctx->stream));
            if (!dev)
                CK(cudaMemcpyAsync(vel_out + 3 * nn * j, vbuf.p, sizeof(float) * 3 * nn,
                                   cudaMemcpyDeviceToHost, ctx->stream));
        }
        CK(cudaStreamSynchronize(ctx->stream));
    }

    int out = LBM_OK;
    for (int j = 0; j < ndir; ++j) {
        const State3 &st = hst[j];
        lbm_result3d &r = results[j];
        for (int c = 0; c < 3; ++c) { r.q[c] = st.q[c]; r.se[c] = st.se[c]; }
        r.steps = st.steps;
        r.converged = st.converged;
        r.status = st.status;
        if (st.status == STATUS_WAIT_TIMEOUT) {
            ctx->err = "run " + std::to_string(j) + ": a step kernel gave up waiting for its shared-memory copies";
            out = LBM_ECUDA;
        } else if (st.status) {
            ctx->err = "non-finite flux in run " + std::to_string(j) + " at step " + std::to_string(st.steps);
            out = LBM_EINPUT;
        } else if (!st.converged && out == LBM_OK) {
            out = LBM_NOT_CONVERGED;
        }
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return out;
}

extern "C" int lbm_debug_bulk_wait(lbm_ctx *ctx, unsigned long long wait_ns, int starve)
{
    if (!ctx) return LBM_EINPUT;
    ctx->test_wait_ns = wait_ns;
    ctx->test_starve = starve ? 1 : 0;
    return LBM_OK;
}

extern "C" int lbm_debug_steps3d(lbm_ctx *ctx, const uint8_t *solid, int nx, int ny, int nz,
                                 const double force[3], double tau, int precision, int variant,
                                 long long nsteps, double *f_out, float *u_out, double q_out[3])
{
    if (!ctx) return LBM_EINPUT;
    CK(cudaSetDevice(ctx->device));
    if (nx <= 0 || ny <= 0 || nz <= 0) return lbm_fail_input(ctx, "bad dimensions");
    const long long nn = (long long)nx * ny * nz;
    if (nn >= (1ll << 31) || (long long)Q3 * lbm_plane_elems(nn) >= (1ll << 32))
        return lbm_fail_input(ctx, "lattice too large");
    lbm_params3d p;
    memset(&p, 0, sizeof(p));
    p.tau = tau; p.eps = 0.0; p.lag = LLONG_MAX / 4; p.hold = 1 << 30;
    p.min_steps = 0; p.max_steps = nsteps; p.avg_steps = 0;
    p.precision = precision; p.criterion = LBM_CRIT_DRIFT; p.variant = variant; p.sample = 1;
    int rc = lbm_check_params3d(ctx, p);
    if (rc) return rc;
    p = lbm_resolve_variant(p);
    variant = p.variant;
    const int npt = lbm_pick_npt(p);
    DevMem mask(ctx->stream);
    long long npore = 0;
    rc = lbm_upload_mask(ctx, solid, nx, (long long)ny * nz, mask, npore);
    if (rc) return rc;
    std::vector<Solve3> hs(1);
    std::vector<State3> hst(1);
    Solve3 &S = hs[0];
    lbm_fill_solve3(S, nx, ny, nz, force, p, npt);
    DevMem lat(ctx->stream), part(ctx->stream), d_states(ctx->stream), d_solves(ctx->stream), d_work(ctx->stream);
    DevMem wpre(ctx->stream), fnode(ctx->stream), meta(ctx->stream), meta2(ctx->stream);
    S.mask = static_cast<const uint32_t *>(mask.p);
    rc = lbm_build_pores(ctx, S, npt, wpre, fnode, meta, meta2);
    if (rc) return rc;
    CK(lat.alloc((size_t)lbm_lattice_bytes(S)));
    CK(part.alloc(sizeof(double) * (size_t)lbm_partial_doubles(precision, S.ntiles)));
    CK(d_states.alloc(sizeof(State3)));
    lbm_attach_lattice(S, lat.p);
    S.mask = static_cast<const uint32_t *>(mask.p);
    S.partials = static_cast<double *>(part.p); S.st = static_cast<State3 *>(d_states.p);
    lbm_init_state3(hst[0], S.c);
    CK(lbm_init_lattice(precision, S, ctx->stream));
    std::vector<int2> work;
    for (int t = 0; t < S.ntiles; ++t) work.push_back(make_int2(0, t));
    CK(d_solves.alloc(sizeof(Solve3)));
    CK(d_work.alloc(sizeof(int2) * work.size()));
    CK(cudaMemcpyAsync(d_solves.p, &S, sizeof(Solve3), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_work.p, work.data(), sizeof(int2) * work.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_states.p, hst.data(), sizeof(State3), cudaMemcpyHostToDevice, ctx->stream));
    rc = run_plain3d(ctx, hs, static_cast<Solve3 *>(d_solves.p), static_cast<State3 *>(d_states.p),
                     static_cast<const int2 *>(d_work.p), (int)work.size(), precision, variant, hst);
    if (rc) return rc;
    DevMem fb(ctx->stream), ub(ctx->stream);
    if (f_out) {
        CK(fb.alloc(sizeof(double) * Q3 * (size_t)nn));
        CK(cudaMemsetAsync(fb.p, 0, sizeof(double) * Q3 * (size_t)nn, ctx->stream));
    }
    if (u_out) {
        CK(ub.alloc(sizeof(float) * 3 * (size_t)nn));
        CK(cudaMemsetAsync(ub.p, 0, sizeof(float) * 3 * (size_t)nn, ctx->stream));
    }
    CK(lbm_canon(precision, S, nsteps, static_cast<double *>(fb.p), static_cast<float *>(ub.p), ctx->stream));
    if (f_out) CK(cudaMemcpyAsync(f_out, fb.p, sizeof(double) * Q3 * nn, cudaMemcpyDeviceToHost, ctx->stream));
    if (u_out) CK(cudaMemcpyAsync(u_out, ub.p, sizeof(float) * 3 * nn, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (q_out) for (int c = 0; c < 3; ++c) q_out[c] = hst[0].q[c];
    return LBM_OK;
}

extern "C" int lbm_variant_count(int precision)
{
    return (precision >= LBM_FP64 && precision <= LBM_MD32) ? variant_count(precision) : 0;
}

// Autotuner: every variant runs the same fixed number of steps on the same
// resident lattices (directions as a batch, like a tensor solve), timed with
// CUDA events on the launch stream.
extern "C" int lbm_tune3d(lbm_ctx *ctx, const uint8_t *solid, int nx, int ny, int nz, int ndir,
                          int precision, int nsteps, double *ms_per_step, int *best)
{
    if (!ctx) return LBM_EINPUT;
    CK(cudaSetDevice(ctx->device));
    if (nx <= 0 || ny <= 0 || nz <= 0 || ndir <= 0 || nsteps <= 0) return lbm_fail_input(ctx, "bad arguments");
    if (precision < LBM_FP64 || precision > LBM_MD32) return lbm_fail_input(ctx, "unknown precision");
    const long long nn = (long long)nx * ny * nz;
    if (nn >= (1ll << 31) || (long long)Q3 * lbm_plane_elems(nn) >= (1ll << 32))
        return lbm_fail_input(ctx, "lattice too large");
    DevMem mask(ctx->stream);
    long long npore = 0;
    int rc = lbm_upload_mask(ctx, solid, nx, (long long)ny * nz, mask, npore);
    if (rc) return rc;
    const int nv = variant_count(precision);
    // lattice bytes and tile count bounds over the variants
    long long lat_bytes = 0, max_tiles = (nn + TPB - 1) / TPB + 1;
    for (int v = 0; v < nv; ++v) {
        lbm_params3d pv;
        memset(&pv, 0, sizeof(pv));
        pv.tau = 1.0; pv.precision = precision; pv.variant = v;
        Solve3 g;
        const double F0[3] = {0, 0, 0};
        lbm_fill_solve3(g, nx, ny, nz, F0, pv, variant_npt(precision, v));
        g.nfluid = (int)npore;
        lat_bytes = std::max(lat_bytes, lbm_lattice_bytes(g));
        max_tiles = std::max<long long>(max_tiles, g.ntiles);
    }
    std::vector<DevMem> lat;
    lat.reserve(ndir);
    for (int j = 0; j < ndir; ++j) {
        lat.emplace_back(ctx->stream);
        CK(lat.back().alloc((size_t)lat_bytes));
    }
    DevMem d_states(ctx->stream), d_solves(ctx->stream), d_work(ctx->stream), part(ctx->stream);
    CK(d_states.alloc(sizeof(State3) * ndir));
    CK(d_solves.alloc(sizeof(Solve3) * ndir));
    CK(part.alloc(sizeof(double) * 3 * (size_t)max_tiles * ndir));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    double best_ms = 1e300;
    int best_v = 0;
    for (int v = 0; v < nv; ++v) {
        lbm_params3d p;
        memset(&p, 0, sizeof(p));
        p.tau = 1.0; p.lag = LLONG_MAX / 4; p.hold = 1 << 30; p.max_steps = LLONG_MAX / 4;
        p.precision = precision; p.variant = v; p.sample = 1;
        const int npt = variant_npt(precision, v);
        DevMem wpre(ctx->stream), fnode(ctx->stream), meta(ctx->stream), meta2(ctx->stream);
        Solve3 proto;
        const double F0[3] = {1e-6, 0, 0};
        lbm_fill_solve3(proto, nx, ny, nz, F0, p, npt);
        proto.mask = static_cast<const uint32_t *>(mask.p);
        rc = lbm_build_pores(ctx, proto, npt, wpre, fnode, meta, meta2);
        if (rc) break;
        std::vector<Solve3> hs(ndir);
        std::vector<State3> hst(ndir);
        std::vector<int2> work;
        for (int j = 0; j < ndir; ++j) {
            double F[3] = {0, 0, 0};
            F[j % 3] = 1e-6;
            lbm_fill_solve3(hs[j], nx, ny, nz, F, p, npt);
            lbm_copy_pores(hs[j], proto);
            lbm_attach_lattice(hs[j], lat[j].p);
            hs[j].mask = proto.mask;
            hs[j].partials = static_cast<double *>(part.p) + 3ll * j * max_tiles;
            hs[j].st = static_cast<State3 *>(d_states.p) + j;
            lbm_init_state3(hst[j], hs[j].c);
            CK(lbm_init_lattice(precision, hs[j], ctx->stream));
            for (int t = 0; t < hs[j].ntiles; ++t) work.push_back(make_int2(j, t));
        }
        DevMem w(ctx->stream);
        CK(w.alloc(sizeof(int2) * work.size()));
        CK(cudaMemcpyAsync(w.p, work.data(), sizeof(int2) * work.size(), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(d_solves.p, hs.data(), sizeof(Solve3) * ndir, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(d_states.p, hst.data(), sizeof(State3) * ndir, cudaMemcpyHostToDevice, ctx->stream));
        StepArgs a;
        a.solves = static_cast<const Solve3 *>(d_solves.p);
        a.work = static_cast<const int2 *>(w.p);
        a.nwork_dev = nullptr;
        a.nwork = (int)work.size();
        const int ev = lbm_effective_variant(precision, v, proto.meta != nullptr);
        StepArgs ae = a;
        DevMem gw(ctx->stream);
        if (lbm_grouped_variant(precision, ev)) {
            std::vector<int2> items;
            lbm_group_items(hs, items);
            CK(gw.alloc(sizeof(int2) * items.size()));
            CK(cudaMemcpyAsync(gw.p, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice, ctx->stream));
            CK(cudaMemcpyAsync(d_solves.p, hs.data(), sizeof(Solve3) * ndir, cudaMemcpyHostToDevice, ctx->stream));
            ae.work = static_cast<const int2 *>(gw.p);
            ae.nwork = (int)items.size();
        }
        const bool gall = lbm_grouped_all(precision, ev);
        auto launch = [&](long long s) {
            const bool odd = ((s + 1) & 1) == 1;
            StepArgs &x = (odd && !gall) ? a : ae;
            x.step = s;
            return lbm_launch_step(precision, ev, true, odd, dim3(x.nwork), ctx->stream, x);
        };
        long long s = 0;
        for (int i = 0; i < std::max(2, nsteps / 4); ++i) CK(launch(s++));
        CK(cudaEventRecord(e0, ctx->stream));
        for (int i = 0; i < nsteps; ++i) CK(launch(s++));
        CK(cudaEventRecord(e1, ctx->stream));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        const double per = (double)ms / nsteps;
        if (ms_per_step) ms_per_step[v] = per;
        if (per < best_ms) { best_ms = per; best_v = v; }
        CK(cudaStreamSynchronize(ctx->stream));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (best) *best = best_v;
    return LBM_OK;
}
