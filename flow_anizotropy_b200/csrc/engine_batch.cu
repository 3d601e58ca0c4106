// liblbm batch engine: many resident 3D solves of one storage precision,
// advanced together.  One step kernel per time step covers a device work list
// of (solve, tile) items of every unfinished solve, each at its own step
// count, one block per item (the hardware block scheduler balances tiles of
// uneven cost, and blocks running at the same time touch neighbouring
// tiles); a chunk of steps is one CUDA graph launch.  When the work list
// changes, the graph's launch sizes are updated in place.  Solves retire on
// the device (the controller marks them done; their blocks exit at once) and
// are reclaimed by lbm_batch_poll; new structures can be admitted between
// chunks, which is what the serving loop uses for continuous batching.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/lbm.h"
#include "engine3d.cuh"
#include "engine_md.cuh"
#include "engine_host.h"

using namespace lbm;

namespace {

struct Slot {
    bool used = false;
    bool retired = false;
    long long tag = 0;
    int dir = 0;
    Solve3 S{};
    std::shared_ptr<DevMem> mask;     // shared by the directions of one structure
    std::shared_ptr<DevMem> wpre, fnode, meta, meta2;
    DevMem lattice{nullptr};
    DevMem partials{nullptr};
    long long bytes = 0;
    long long tables = 0;     // mask + rank tables of the structure
    int lead = -1;            // grouped variants: first slot of this direction's group
};

}  // namespace

struct lbm_batch {
    lbm_ctx *ctx = nullptr;
    int precision = LBM_FP32;
    int variant = 0;
    bool w1 = true;
    int npt = 1;
    int chunk = 64;
    long long budget = 0;
    long long resident = 0;
    int cap_slots = 0;
    int cap_work = 0;
    int nwork = 0;         // items in the device work list (= blocks per step launch)
    int graph_nwork = -1;  // launch size the graph holds
    // grouped even-step variants: the even launches take a second work list of
    // (group leader slot, tile) items; a group's slots are consecutive
    bool grouped = false;
    int ngwork = 0, graph_ngwork = -1, cap_gwork = 0;
    DevMem d_gwork{nullptr}, d_ngwork{nullptr};
    int slot_hi = 0;       // slots below this index hold every resident solve
    int graph_slot_hi = -1;
    DevMem d_qbuf{nullptr};   // deferred reduction: q and flag per slot and step
    std::vector<Slot> slots;
    DevMem d_solves{nullptr}, d_states{nullptr}, d_work{nullptr}, d_nwork{nullptr};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<State3> hst;
};

static void destroy_graph(lbm_batch *b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

// One graph = `chunk` step launches (step index 0..chunk-1 relative to each
// solve's s_base) followed by the s_base advance.  An existing executable
// graph is updated in place when only launch sizes changed.
static int capture(lbm_batch *b)
{
    lbm_ctx *ctx = b->ctx;
    StepArgs a;
    a.solves = static_cast<const Solve3 *>(b->d_solves.p);
    a.work = static_cast<const int2 *>(b->d_work.p);
    a.nwork_dev = static_cast<const int *>(b->d_nwork.p);
    a.nwork = 0;
    const dim3 grid(std::max(1, b->nwork));
    const bool defer = lbm_defers(b->precision);
    a.defer = defer ? 2 : 0;
    StepArgs ae = a;                 // even launches: the grouped work list when grouped
    dim3 grid_e = grid;
    if (b->grouped) {
        ae.work = static_cast<const int2 *>(b->d_gwork.p);
        ae.nwork_dev = static_cast<const int *>(b->d_ngwork.p);
        grid_e = dim3(std::max(1, b->ngwork));
    }
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    // chunks are even and solves join at chunk boundaries (s_base even), so
    // launch i runs step i + 1 of every solve: odd launches use the local kernel.
    // Deferred reduction: a pass after every DEFER_SLOTS launches and at the
    // chunk's end; solves sit at different step counts, so their phases can
    // change inside a pass (mode 2)
    for (int i = 0; i < b->chunk && e == cudaSuccess; ++i) {
        a.step = i;
        ae.step = i;
        const bool odd = ((i + 1) & 1) == 1;
        e = lbm_launch_step(b->precision, b->variant, b->w1, odd, odd ? grid : grid_e, ctx->stream, odd ? a : ae);
        const bool pass_end = ((i + 1) % DEFER_SLOTS) == 0 || i + 1 == b->chunk;
        if (e == cudaSuccess && defer && pass_end) {
            const int first = i - (i % DEFER_SLOTS);
            e = launch_deferred3d(static_cast<const Solve3 *>(b->d_solves.p), std::max(1, b->slot_hi), first,
                                  i + 1 - first, static_cast<double *>(b->d_qbuf.p), 2, ctx->stream);
        }
    }
    if (e == cudaSuccess) {
        advance3d_kernel<<<(b->cap_slots + 255) / 256, 256, 0, ctx->stream>>>(
            static_cast<Solve3 *>(b->d_solves.p), b->cap_slots, b->chunk);
        e = cudaGetLastError();
    }
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &g);
    if (e != cudaSuccess) { if (g) cudaGraphDestroy(g); return lbm_fail_cuda(ctx, e, "graph capture", __LINE__); }
    CK(e2);
    if (b->exec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(b->exec, g, &info) == cudaSuccess) {
            if (b->graph) cudaGraphDestroy(b->graph);
            b->graph = g;
            b->graph_nwork = b->nwork;
            b->graph_ngwork = b->ngwork;
            b->graph_slot_hi = b->slot_hi;
            return LBM_OK;
        }
        cudaGetLastError();            // not updatable (kernels changed): instantiate anew
    }
    destroy_graph(b);
    b->graph = g;
    CK(cudaGraphInstantiate(&b->exec, g, 0));
    b->graph_nwork = b->nwork;
    b->graph_ngwork = b->ngwork;
    b->graph_slot_hi = b->slot_hi;
    return LBM_OK;
}

// Upload descriptors and the work list of every unfinished solve.
static int sync_work(lbm_batch *b)
{
    lbm_ctx *ctx = b->ctx;
    std::vector<Solve3> desc(b->cap_slots);
    std::vector<int2> work;
    int hi = 0;
    for (int i = 0; i < b->cap_slots; ++i)
        if (b->slots[i].used) hi = i + 1;
    b->slot_hi = hi;
    for (int i = 0; i < b->cap_slots; ++i) {
        const Slot &s = b->slots[i];
        if (!s.used) {
            // an empty slot: a descriptor whose state pointer marks it finished
            desc[i] = Solve3{};
            desc[i].st = static_cast<State3 *>(b->d_states.p) + i;
            continue;
        }
        desc[i] = s.S;
        if (!s.retired)
            for (int t = 0; t < s.S.ntiles; ++t) work.push_back(make_int2(i, t));
    }
    // grouped even steps: one item per tile of every group with a direction
    // still running (its slots stay resident until the whole group is done)
    std::vector<int2> gwork;
    if (b->grouped)
        for (int i = 0; i < b->cap_slots; ++i) {
            const Slot &s = b->slots[i];
            if (!s.used || s.lead != i) continue;
            bool live = false;
            for (int d = 0; d < s.S.group; ++d) live = live || !b->slots[i + d].retired;
            if (live)
                for (int t = 0; t < s.S.ntiles; ++t) gwork.push_back(make_int2(i, t));
        }
    const int nwork = (int)work.size(), ngwork = (int)gwork.size();
    bool recapture = nwork != b->graph_nwork || b->slot_hi != b->graph_slot_hi || ngwork != b->graph_ngwork;
    if (nwork > b->cap_work) {
        b->cap_work = std::max<int>(nwork, 2 * b->cap_work);
        CK(b->d_work.alloc(sizeof(int2) * (size_t)b->cap_work));
        recapture = true;
    }
    if (ngwork > b->cap_gwork) {
        b->cap_gwork = std::max<int>(ngwork, 2 * b->cap_gwork);
        CK(b->d_gwork.alloc(sizeof(int2) * (size_t)b->cap_gwork));
        recapture = true;
    }
    b->nwork = nwork;
    b->ngwork = ngwork;
    if (recapture) {
        int rc = capture(b);
        if (rc) return rc;
    }
    CK(cudaMemcpyAsync(b->d_solves.p, desc.data(), sizeof(Solve3) * b->cap_slots, cudaMemcpyHostToDevice, ctx->stream));
    if (nwork)
        CK(cudaMemcpyAsync(b->d_work.p, work.data(), sizeof(int2) * work.size(), cudaMemcpyHostToDevice, ctx->stream));
    if (ngwork)
        CK(cudaMemcpyAsync(b->d_gwork.p, gwork.data(), sizeof(int2) * gwork.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(b->d_ngwork.p, &ngwork, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    // pageable source: the copy is staged before the call returns
    CK(cudaMemcpyAsync(b->d_nwork.p, &nwork, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return LBM_OK;
}

extern "C" long long lbm_batch_bytes3d(int nx, int ny, int nz, int ndir, int precision)
{
    const long long nn = (long long)nx * ny * nz;
    // upper bound: every voxel a pore (the batch charges the exact size on admission)
    const long long tables = 4ll * ((nx + 31) / 32) * (long long)ny * nz * 2 + 28ll * nn + 8;
    if (is_dense_m(precision)) {
        MDGeom g{};
        int tiles = 0;
        md_fill_geom(g, nx, ny, nz, 0, tiles);
        return tables + md_pmask_bytes(g, ny, nz) + (long long)ndir * (md_lattice_bytes(g) + 24ll * tiles);
    }
    const long long tiles = (nn + TPB - 1) / TPB;
    // the two lattices of the pull and two-lattice AA forms, for the
    // precisions that have them
    const long long lat = lbm_lattice_bytes3d(nn, precision) * (precision >= LBM_FP64 && precision <= LBM_BF16 ? 2 : 1);
    return tables + (long long)ndir * (lat + 8 * lbm_partial_doubles(precision, (int)tiles));
}

extern "C" int lbm_batch_create(lbm_ctx *ctx, lbm_batch **out, int precision, long long hbm_budget, int chunk)
{
    if (!ctx || !out) return LBM_EINPUT;
    *out = nullptr;
    CK(cudaSetDevice(ctx->device));
    if (precision < LBM_FP64 || precision > LBM_MD32) return lbm_fail_input(ctx, "unknown precision");
    if (chunk <= 0 || chunk > 4096) return lbm_fail_input(ctx, "chunk must be in 1..4096");
    chunk += chunk & 1;                  // even: every solve keeps the launch's parity
    if (hbm_budget <= 0) return lbm_fail_input(ctx, "budget must be positive");
    std::unique_ptr<lbm_batch> b(new lbm_batch());
    b->ctx = ctx;
    b->precision = precision;
    b->chunk = chunk;
    b->budget = hbm_budget;
    b->variant = lbm_default_batch_variant(precision);
    b->npt = variant_npt(precision, b->variant);
    b->cap_slots = 4096;
    b->cap_work = 1 << 16;
    b->slots.resize(b->cap_slots);
    b->hst.resize(b->cap_slots);
    b->d_solves = DevMem(ctx->stream);
    b->d_states = DevMem(ctx->stream);
    b->d_work = DevMem(ctx->stream);
    b->d_nwork = DevMem(ctx->stream);
    for (auto &s : b->slots) { s.lattice = DevMem(ctx->stream); s.partials = DevMem(ctx->stream); }
    CK(b->d_solves.alloc(sizeof(Solve3) * b->cap_slots));
    CK(b->d_states.alloc(sizeof(State3) * b->cap_slots));
    CK(b->d_work.alloc(sizeof(int2) * b->cap_work));
    CK(b->d_nwork.alloc(sizeof(int)));
    b->d_gwork = DevMem(ctx->stream);
    b->d_ngwork = DevMem(ctx->stream);
    b->cap_gwork = 1 << 14;
    CK(b->d_gwork.alloc(sizeof(int2) * b->cap_gwork));
    CK(b->d_ngwork.alloc(sizeof(int)));
    b->grouped = lbm_grouped_variant(precision, b->variant);
    b->d_qbuf = DevMem(ctx->stream);
    CK(b->d_qbuf.alloc(sizeof(double) * 4 * DEFER_SLOTS * (size_t)b->cap_slots));
    std::vector<State3> done(b->cap_slots);
    for (auto &st : done) { memset(&st, 0, sizeof(st)); st.phase = PH_DONE; }
    CK(cudaMemcpyAsync(b->d_states.p, done.data(), sizeof(State3) * b->cap_slots, cudaMemcpyHostToDevice, ctx->stream));
    int rc = sync_work(b.get());
    if (rc) return rc;
    *out = b.release();
    return LBM_OK;
}

extern "C" int lbm_batch_set_variant(lbm_batch *b, int variant)
{
    if (!b) return LBM_EINPUT;
    lbm_ctx *ctx = b->ctx;
    if (variant == LBM_VARIANT_DEFAULT) variant = lbm_default_batch_variant(b->precision);
    if (variant < 0 || variant >= variant_count(b->precision))
        return lbm_fail_input(ctx, "unknown step-kernel variant");
    for (const Slot &s : b->slots)
        if (s.used) return lbm_fail_input(ctx, "the batch has resident solves");
    if (variant_npt(b->precision, variant) != b->npt) return lbm_fail_input(ctx, "variant changes the tile size");
    if (lbm_grouped_all(b->precision, variant))
        return lbm_fail_input(ctx, "grouped pull variants step every launch by structure; the batch steps its "
                                   "odd launches per direction");
    b->variant = variant;
    b->grouped = lbm_grouped_variant(b->precision, variant);
    b->graph_nwork = -1;      // recapture with the new kernels at the next change
    b->graph_ngwork = -1;
    return LBM_OK;
}

extern "C" void lbm_batch_destroy(lbm_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    destroy_graph(b);
    delete b;
}

extern "C" int lbm_batch_submit3d(lbm_batch *b, const uint8_t *solid, int nx, int ny, int nz,
                                  int ndir, const double *forces, const lbm_params3d *params, long long tag)
{
    if (!b) return LBM_EINPUT;
    lbm_ctx *ctx = b->ctx;
    if (!solid || !forces || !params || ndir <= 0) return lbm_fail_input(ctx, "null argument");
    CK(cudaSetDevice(ctx->device));
    if (nx <= 0 || ny <= 0 || nz <= 0) return lbm_fail_input(ctx, "bad dimensions");
    const long long nn = (long long)nx * ny * nz;
    if (nn >= (1ll << 31) || (long long)Q3 * lbm_plane_elems(nn) >= (1ll << 32))
        return lbm_fail_input(ctx, "lattice too large");
    lbm_params3d p = *params;
    if (p.precision != b->precision) return lbm_fail_input(ctx, "precision differs from the batch's");
    p.variant = b->variant;
    int rc = lbm_check_params3d(ctx, p);
    if (rc) return rc;
    std::vector<int> free_slots;
    if (b->grouped) {
        // a structure's directions take consecutive slots (one group of up
        // to MAX_GROUP per run), so the grouped even kernel finds them at
        // leader + d
        for (int i = 0; i + ndir <= b->cap_slots && (int)free_slots.size() < ndir; ++i) {
            int run = 0;
            while (run < ndir && !b->slots[i + run].used) ++run;
            if (run == ndir) for (int d = 0; d < ndir; ++d) free_slots.push_back(i + d);
            else i += run;
        }
    } else {
        for (int i = 0; i < b->cap_slots && (int)free_slots.size() < ndir; ++i)
            if (!b->slots[i].used) free_slots.push_back(i);
    }
    if ((int)free_slots.size() < ndir) { ctx->err = "batch slots exhausted"; return LBM_EBUSY; }

    auto mask = std::make_shared<DevMem>(ctx->stream);
    long long npore = 0;
    rc = lbm_upload_mask(ctx, solid, nx, (long long)ny * nz, *mask, npore);
    if (rc) return rc;
    auto wpre = std::make_shared<DevMem>(ctx->stream), fnode = std::make_shared<DevMem>(ctx->stream);
    auto meta = std::make_shared<DevMem>(ctx->stream), meta2 = std::make_shared<DevMem>(ctx->stream);
    Solve3 proto;
    lbm_fill_solve3(proto, nx, ny, nz, forces, p, b->npt);
    proto.mask = static_cast<const uint32_t *>(mask->p);
    rc = lbm_build_pores(ctx, proto, b->npt, *wpre, *fnode, *meta, *meta2);
    if (rc) return rc;
    if (!proto.meta && lbm_effective_variant(b->precision, b->variant, false) != b->variant) {
        // a structure too wide for neighbour records: the batch computes ranks
        // (the mask-rank counterpart of a grouped variant is grouped too, so
        // the resident groups keep their layout)
        b->variant = lbm_effective_variant(b->precision, b->variant, false);
        b->grouped = lbm_grouped_variant(b->precision, b->variant);
        rc = capture(b);
        if (rc) return rc;
    }
    const long long tables = 4ll * ((nx + 31) / 32) * (long long)ny * nz * 2 + 4ll * proto.nfluid + 8 +
                             (proto.meta ? 24ll * proto.nfluid : 0) +
                             (is_dense_m(b->precision) ? md_pmask_bytes(proto.md, ny, nz) : 0);
    const long long part_bytes = 8ll * lbm_partial_doubles(b->precision, proto.ntiles);
    const long long exact = tables + (long long)ndir * (lbm_lattice_bytes(proto) + part_bytes);
    if (b->resident + exact > b->budget) {
        ctx->err = "batch budget exhausted";
        return LBM_EBUSY;
    }
    if (p.tau != 1.0 && b->w1) {
        // a relaxation time other than 1 needs the general collision kernel
        b->w1 = false;
        rc = capture(b);
        if (rc) return rc;
    }
    std::vector<State3> init(ndir);
    for (int j = 0; j < ndir; ++j) {
        Slot &s = b->slots[free_slots[j]];
        lbm_fill_solve3(s.S, nx, ny, nz, forces + 3 * j, p, b->npt);
        lbm_copy_pores(s.S, proto);
        // group leader of direction j: the first of its run of MAX_GROUP
        const int j0 = j - j % MAX_GROUP;
        s.lead = b->grouped ? free_slots[j0] : -1;
        if (b->grouped && j == j0) s.S.group = std::min(MAX_GROUP, ndir - j0);
        s.wpre = wpre; s.fnode = fnode; s.meta = meta; s.meta2 = meta2;
        s.tables = tables;
        CK(s.lattice.alloc((size_t)lbm_lattice_bytes(s.S)));
        CK(s.partials.alloc(sizeof(double) * (size_t)lbm_partial_doubles(b->precision, s.S.ntiles)));
        lbm_attach_lattice(s.S, s.lattice.p);
        s.S.mask = static_cast<const uint32_t *>(mask->p);
        s.S.partials = static_cast<double *>(s.partials.p);
        s.S.st = static_cast<State3 *>(b->d_states.p) + free_slots[j];
        s.mask = mask;
        s.tag = tag;
        s.dir = j;
        s.used = true;
        s.retired = false;
        s.bytes = lbm_lattice_bytes(s.S) + part_bytes;
        lbm_init_state3(init[j], s.S.c);
        CK(lbm_init_lattice(b->precision, s.S, ctx->stream));
        CK(cudaMemcpyAsync(s.S.st, &init[j], sizeof(State3), cudaMemcpyHostToDevice, ctx->stream));
    }
    b->resident += exact;
    return sync_work(b);
}

extern "C" int lbm_batch_run(lbm_batch *b, int chunks)
{
    if (!b) return LBM_EINPUT;
    lbm_ctx *ctx = b->ctx;
    CK(cudaSetDevice(ctx->device));
    for (int i = 0; i < chunks; ++i) CK(cudaGraphLaunch(b->exec, ctx->stream));
    return LBM_OK;
}

// Free a finished solve's slot: its lattice, partials and, with the
// structure's last direction, the mask and rank tables.
static void release_slot(lbm_batch *b, Slot &s)
{
    s.used = false;
    s.lead = -1;
    s.lattice.release();
    s.partials.release();
    b->resident -= s.bytes;
    // the structure's mask goes with its last direction
    const bool last = s.mask.use_count() == 1;
    if (last) b->resident -= s.tables;
    s.mask.reset();
    s.wpre.reset();
    s.fnode.reset();
    s.meta.reset();
    s.meta2.reset();
}

extern "C" int lbm_batch_poll(lbm_batch *b, long long *tags, int *dirs, lbm_result3d *results, int max, int *n)
{
    if (!b || !n) return LBM_EINPUT;
    lbm_ctx *ctx = b->ctx;
    *n = 0;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(b->hst.data(), b->d_states.p, sizeof(State3) * b->cap_slots, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    bool changed = false;
    for (int i = 0; i < b->cap_slots && *n < max; ++i) {
        Slot &s = b->slots[i];
        if (!s.used || s.retired) continue;
        const State3 &st = b->hst[i];
        if (st.phase < PH_DONE) continue;
        lbm_result3d &r = results[*n];
        for (int c = 0; c < 3; ++c) { r.q[c] = st.q[c]; r.se[c] = st.se[c]; }
        r.steps = st.steps;
        r.converged = st.converged;
        r.status = st.status;
        tags[*n] = s.tag;
        dirs[*n] = s.dir;
        ++*n;
        s.retired = true;
        changed = true;
        if (s.lead < 0) {
            release_slot(b, s);
            continue;
        }
        // grouped: the group's slots stay resident (the grouped even kernel
        // reads its leader's record) until every direction of it is done
        const int lead = s.lead, ng = b->slots[lead].S.group;
        bool all = true;
        for (int d = 0; d < ng; ++d) all = all && b->slots[lead + d].retired;
        if (all)
            for (int d = 0; d < ng; ++d) release_slot(b, b->slots[lead + d]);
    }
    if (changed) return sync_work(b);
    return LBM_OK;
}

extern "C" int lbm_batch_active(const lbm_batch *b)
{
    if (!b) return 0;
    int n = 0;
    for (const auto &s : b->slots) n += s.used && !s.retired;
    return n;
}

extern "C" long long lbm_batch_resident_bytes(const lbm_batch *b) { return b ? b->resident : 0; }
