// liblbm host engine, D2Q9: the plain solve loop of LMB2d/main.cpp:99-235 on
// the device controller, and the 2D diagnostic entry point.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lbm.h"
#include "engine2d.cuh"
#include "engine2_host.h"
#include "engine_host.h"

using namespace lbm;

int check_params2d(lbm_ctx *ctx, const lbm_params2d &p)
{
    if (!(p.tau > 0.5)) return lbm_fail_input(ctx, "tau must exceed 0.5");
    // LMB2d/main.cpp:304
    if (p.lag <= 0 || p.avg_sample <= 0) return lbm_fail_input(ctx, "--lag and --avg-sample must be positive");
    return LBM_OK;
}

void fill_solve2(Solve2 &S, int nx, int ny, const double F[2], const lbm_params2d &p)
{
    memset(&S, 0, sizeof(S));
    S.nx = nx; S.ny = ny; S.wpr = (nx + 31) / 32;
    S.nn = nx * ny;
    S.plane = (unsigned)lbm_plane_elems(S.nn);
    S.ntiles = (S.nn + TPB - 1) / TPB;
    S.dvx.init(nx);
    // the reference stores fx, fy and tau in float globals (LMB2d/lbm.cpp:82-86,
    // LMB2d/main.cpp:104-106)
    S.fx = (float)F[0]; S.fy = (float)F[1]; S.tau = (float)p.tau;
    Ctl2 &c = S.c;
    c.eps = p.eps; c.qfloor = p.qfloor; c.ksigma = p.ksigma;
    c.lag = p.lag; c.min_steps = p.min_steps; c.max_steps = p.max_steps;
    c.avg_steps = p.avg_steps; c.avg_sample = p.avg_sample; c.hold = p.hold;
}

void init_state2(State2 &st, const Ctl2 &c)
{
    memset(&st, 0, sizeof(st));
    st.phase = PH_RUN;
    if (c.max_steps <= 0) {
        st.converged = 0 >= c.hold ? 1 : 0;
        st.avg_start = 0;
        st.snap_valid = 1;           // snapshot of the rest state: U = V = 0
        if (c.avg_steps <= 0) { st.phase = PH_DONE; st.steps = 0; }
        else st.phase = PH_AVG;
    }
}

// The host loop of LMB2d/main.cpp:99-235 with the controller on the device:
// launch up to the next step at which some direction's controller can change
// phase, then read the states back.  The launches in between are replayed
// from a CUDA graph of kGraphSteps step launches (plus the s_base advance),
// which removes most of the per-launch overhead of this small, launch-bound
// lattice; the step numbers and kernels are the same as single launches.
constexpr int kGraphSteps = 100;

static int run_plain2d(lbm_ctx *ctx, std::vector<Solve2> &hs, Solve2 *d_solves, State2 *d_states,
                       const int2 *d_work, int nwork, std::vector<State2> &hst)
{
    const int n = (int)hs.size();
    long long s = 0, base = 0;        // steps done; s_base of every solve (host copy)
    StepArgs2 a;
    a.solves = d_solves; a.work = d_work; a.nwork = nwork;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    struct GraphGuard {
        cudaGraph_t &g; cudaGraphExec_t &e;
        ~GraphGuard() { if (e) cudaGraphExecDestroy(e); if (g) cudaGraphDestroy(g); }
    } guard{graph, exec};
    for (;;) {
        CK(cudaMemcpyAsync(hst.data(), d_states, sizeof(State2) * n, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        long long target = LLONG_MAX;
        for (int j = 0; j < n; ++j) {
            const State2 &st = hst[j];
            const Ctl2 &c = hs[j].c;
            if (st.phase == PH_RUN) {
                long long nx = (s / c.lag + 1) * c.lag;
                if (c.max_steps > s) nx = std::min(nx, c.max_steps);
                target = std::min(target, nx);
            } else if (st.phase == PH_AVG) {
                target = std::min(target, st.avg_start + c.avg_steps);
            }
        }
        if (target == LLONG_MAX) break;
        if (!exec && target - s >= kGraphSteps) {
            CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t e = cudaSuccess;
            for (int i = 0; i < kGraphSteps && e == cudaSuccess; ++i) {
                StepArgs2 g = a;
                g.step = i;
                e = launch_step2d(dim3(nwork), ctx->stream, g);
            }
            if (e == cudaSuccess) e = launch_advance2d(d_solves, n, kGraphSteps, ctx->stream);
            const cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &graph);
            CK(e);
            CK(e2);
            CK(cudaGraphInstantiate(&exec, graph, 0));
        }
        while (s < target) {
            if (exec && target - s >= kGraphSteps) {
                if (base != s) {
                    // a chunk numbers its steps from s_base: catch up with the single steps
                    CK(launch_advance2d(d_solves, n, s - base, ctx->stream));
                    base = s;
                }
                CK(cudaGraphLaunch(exec, ctx->stream));
                s += kGraphSteps;
                base += kGraphSteps;
            } else {
                a.step = s - base;
                CK(launch_step2d(dim3(nwork), ctx->stream, a));
                ++s;
            }
        }
    }
    return LBM_OK;
}

struct Set2 {
    std::vector<Solve2> hs;
    std::vector<State2> hst;
    std::vector<DevMem> bufs;
};

static int setup2d(lbm_ctx *ctx, const uint8_t *solid, int nx, int ny, int ndir, const double *forces,
                   const lbm_params2d &p, DevMem &mask, Set2 &set, DevMem &d_states, DevMem &d_solves,
                   DevMem &d_work, int &nwork)
{
    long long npore = 0;
    int rc = lbm_upload_mask(ctx, solid, nx, ny, mask, npore);
    if (rc) return rc;
    set.hs.resize(ndir);
    set.hst.resize(ndir);
    set.bufs.reserve(4 * ndir + 1);
    set.bufs.emplace_back(ctx->stream);                 // neighbour solid bits, shared by the directions
    DevMem &nbm = set.bufs.back();
    CK(nbm.alloc(sizeof(uint16_t) * (size_t)nx * ny));
    CK(launch_nbmask2d(static_cast<const uint32_t *>(mask.p), nx, ny, static_cast<uint16_t *>(nbm.p), ctx->stream));
    const uint16_t *nbm_p = static_cast<const uint16_t *>(nbm.p);
    CK(d_states.alloc(sizeof(State2) * ndir));
    for (int j = 0; j < ndir; ++j) {
        Solve2 &S = set.hs[j];
        fill_solve2(S, nx, ny, forces + 2 * j, p);
        for (int b = 0; b < 4; ++b) set.bufs.emplace_back(ctx->stream);
        DevMem *B = &set.bufs[1 + 4 * j];
        CK(B[0].alloc(sizeof(float) * Q2 * (size_t)S.plane));
        CK(B[1].alloc(sizeof(double) * 2 * (size_t)S.ntiles));
        CK(B[2].alloc(sizeof(float) * 2 * (size_t)S.nn));
        CK(B[3].alloc(sizeof(float) * 2 * (size_t)S.nn));
        CK(cudaMemsetAsync(B[2].p, 0, sizeof(float) * 2 * (size_t)S.nn, ctx->stream));
        CK(cudaMemsetAsync(B[3].p, 0, sizeof(float) * 2 * (size_t)S.nn, ctx->stream));
        S.A = static_cast<float *>(B[0].p);
        S.partials = static_cast<double *>(B[1].p);
        S.snap = static_cast<float *>(B[2].p);
        S.last = static_cast<float *>(B[3].p);
        S.mask = static_cast<const uint32_t *>(mask.p);
        S.nbm = nbm_p;
        S.st = static_cast<State2 *>(d_states.p) + j;
        init_state2(set.hst[j], S.c);
        init2d_kernel<<<256, 256, 0, ctx->stream>>>(S.A, S.plane, S.nn);
        CK(cudaGetLastError());
    }
    std::vector<int2> work;
    for (int j = 0; j < ndir; ++j)
        for (int t = 0; t < set.hs[j].ntiles; ++t) work.push_back(make_int2(j, t));
    nwork = (int)work.size();
    CK(d_solves.alloc(sizeof(Solve2) * ndir));
    CK(d_work.alloc(sizeof(int2) * work.size()));
    CK(cudaMemcpyAsync(d_solves.p, set.hs.data(), sizeof(Solve2) * ndir, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_work.p, work.data(), sizeof(int2) * work.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_states.p, set.hst.data(), sizeof(State2) * ndir, cudaMemcpyHostToDevice, ctx->stream));
    return LBM_OK;
}

extern "C" int lbm_solve2d(lbm_ctx *ctx, const uint8_t *solid, int nx, int ny,
                           int ndir, const double *forces, const lbm_params2d *params,
                           lbm_result2d *results, float *vel_out)
{
    if (!ctx) return LBM_EINPUT;
    if (!solid || !forces || !params || !results || ndir <= 0) return lbm_fail_input(ctx, "null argument");
    CK(cudaSetDevice(ctx->device));
    if (nx <= 0 || ny <= 0) return lbm_fail_input(ctx, "bad dimensions");
    if ((long long)nx * ny >= (1ll << 27)) return lbm_fail_input(ctx, "2D lattice too large");
    const lbm_params2d p = *params;
    int rc = check_params2d(ctx, p);
    if (rc) return rc;
    DevMem mask(ctx->stream), d_states(ctx->stream), d_solves(ctx->stream), d_work(ctx->stream);
    Set2 set;
    int nwork = 0;
    rc = setup2d(ctx, solid, nx, ny, ndir, forces, p, mask, set, d_states, d_solves, d_work, nwork);
    if (rc) return rc;
    rc = run_plain2d(ctx, set.hs, static_cast<Solve2 *>(d_solves.p), static_cast<State2 *>(d_states.p),
                     static_cast<const int2 *>(d_work.p), nwork, set.hst);
    if (rc) return rc;

    DevMem fr(ctx->stream);
    CK(fr.alloc(sizeof(double) * 2 * ndir));
    CK(cudaMemsetAsync(fr.p, 0, sizeof(double) * 2 * ndir, ctx->stream));
    for (int j = 0; j < ndir; ++j) {
        const Solve2 &S = set.hs[j];
        fieldres2d_kernel<<<64, TPB, 0, ctx->stream>>>(S.snap, S.last, S.nn, static_cast<double *>(fr.p) + 2 * j);
        CK(cudaGetLastError());
    }
    std::vector<double> frh(2 * ndir);
    CK(cudaMemcpyAsync(frh.data(), fr.p, sizeof(double) * 2 * ndir, cudaMemcpyDeviceToHost, ctx->stream));
    if (vel_out) {
        const long long nn = (long long)nx * ny;
        for (int j = 0; j < ndir; ++j)
            CK(cudaMemcpyAsync(vel_out + 2 * nn * j, set.hs[j].last, sizeof(float) * 2 * nn,
                               cudaMemcpyDefault, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));

    int out = LBM_OK;
    for (int j = 0; j < ndir; ++j) {
        const State2 &st = set.hst[j];
        lbm_result2d &r = results[j];
        r.q[0] = st.q[0]; r.q[1] = st.q[1];
        r.se[0] = st.se[0]; r.se[1] = st.se[1];
        r.steps = st.steps;
        r.converged = st.converged;
        r.status = st.status;
        const double num = frh[2 * j], den = frh[2 * j + 1];
        r.fieldres = den > 0.0 ? (double)(float)std::sqrt(num / den) : 10.0;
        if (st.status) {
            ctx->err = "non-finite flux in run " + std::to_string(j) + " at step " + std::to_string(st.steps);
            out = LBM_EINPUT;
        } else if (!st.converged && out == LBM_OK) {
            out = LBM_NOT_CONVERGED;
        }
    }
    return out;
}

// Several structures of one cell size, each with the same forcing directions,
// advanced by one launch per step: the work list covers every (structure,
// direction) solve, each with its own mask, controller and flux partials, so
// every result equals the structure solved alone.
extern "C" int lbm_solve2d_many(lbm_ctx *ctx, int nstruct, const uint8_t *solids, int nx, int ny, int ndir,
                                const double *forces, const lbm_params2d *params, lbm_result2d *results)
{
    if (!ctx) return LBM_EINPUT;
    if (!solids || !forces || !params || !results || ndir <= 0 || nstruct <= 0)
        return lbm_fail_input(ctx, "null argument");
    CK(cudaSetDevice(ctx->device));
    if (nx <= 0 || ny <= 0) return lbm_fail_input(ctx, "bad dimensions");
    const long long nn = (long long)nx * ny;
    if (nn >= (1ll << 27)) return lbm_fail_input(ctx, "2D lattice too large");
    const lbm_params2d p = *params;
    int rc = check_params2d(ctx, p);
    if (rc) return rc;
    const int nsolve = nstruct * ndir;
    std::vector<DevMem> masks, nbms;
    masks.reserve(nstruct);
    nbms.reserve(nstruct);
    std::vector<Solve2> hs(nsolve);
    std::vector<State2> hst(nsolve);
    std::vector<DevMem> bufs;
    bufs.reserve(4 * (size_t)nsolve);
    DevMem d_states(ctx->stream), d_solves(ctx->stream), d_work(ctx->stream), fr(ctx->stream);
    CK(d_states.alloc(sizeof(State2) * nsolve));
    for (int k = 0; k < nstruct; ++k) {
        masks.emplace_back(ctx->stream);
        long long npore = 0;
        rc = lbm_upload_mask(ctx, solids + nn * k, nx, ny, masks.back(), npore);
        if (rc) {
            ctx->err = "structure " + std::to_string(k) + ": " + ctx->err;
            return rc;
        }
        nbms.emplace_back(ctx->stream);
        CK(nbms.back().alloc(sizeof(uint16_t) * (size_t)nn));
        CK(launch_nbmask2d(static_cast<const uint32_t *>(masks.back().p), nx, ny,
                           static_cast<uint16_t *>(nbms.back().p), ctx->stream));
        for (int j = 0; j < ndir; ++j) {
            const int id = k * ndir + j;
            Solve2 &S = hs[id];
            fill_solve2(S, nx, ny, forces + 2 * j, p);
            for (int b = 0; b < 4; ++b) bufs.emplace_back(ctx->stream);
            DevMem *B = &bufs[4 * (size_t)id];
            CK(B[0].alloc(sizeof(float) * Q2 * (size_t)S.plane));
            CK(B[1].alloc(sizeof(double) * 2 * (size_t)S.ntiles));
            CK(B[2].alloc(sizeof(float) * 2 * (size_t)nn));
            CK(B[3].alloc(sizeof(float) * 2 * (size_t)nn));
            CK(cudaMemsetAsync(B[2].p, 0, sizeof(float) * 2 * (size_t)nn, ctx->stream));
            CK(cudaMemsetAsync(B[3].p, 0, sizeof(float) * 2 * (size_t)nn, ctx->stream));
            S.A = static_cast<float *>(B[0].p);
            S.partials = static_cast<double *>(B[1].p);
            S.snap = static_cast<float *>(B[2].p);
            S.last = static_cast<float *>(B[3].p);
            S.mask = static_cast<const uint32_t *>(masks.back().p);
            S.nbm = static_cast<const uint16_t *>(nbms.back().p);
            S.st = static_cast<State2 *>(d_states.p) + id;
            init_state2(hst[id], S.c);
            init2d_kernel<<<256, 256, 0, ctx->stream>>>(S.A, S.plane, S.nn);
            CK(cudaGetLastError());
        }
    }
    std::vector<int2> work;
    for (int id = 0; id < nsolve; ++id)
        for (int t = 0; t < hs[id].ntiles; ++t) work.push_back(make_int2(id, t));
    CK(d_solves.alloc(sizeof(Solve2) * nsolve));
    CK(d_work.alloc(sizeof(int2) * work.size()));
    CK(cudaMemcpyAsync(d_solves.p, hs.data(), sizeof(Solve2) * nsolve, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_work.p, work.data(), sizeof(int2) * work.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_states.p, hst.data(), sizeof(State2) * nsolve, cudaMemcpyHostToDevice, ctx->stream));
    rc = run_plain2d(ctx, hs, static_cast<Solve2 *>(d_solves.p), static_cast<State2 *>(d_states.p),
                     static_cast<const int2 *>(d_work.p), (int)work.size(), hst);
    if (rc) return rc;
    CK(fr.alloc(sizeof(double) * 2 * nsolve));
    CK(cudaMemsetAsync(fr.p, 0, sizeof(double) * 2 * nsolve, ctx->stream));
    for (int id = 0; id < nsolve; ++id) {
        fieldres2d_kernel<<<64, TPB, 0, ctx->stream>>>(hs[id].snap, hs[id].last, hs[id].nn,
                                                       static_cast<double *>(fr.p) + 2 * id);
        CK(cudaGetLastError());
    }
    std::vector<double> frh(2 * (size_t)nsolve);
    CK(cudaMemcpyAsync(frh.data(), fr.p, sizeof(double) * 2 * nsolve, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    int out = LBM_OK;
    for (int id = 0; id < nsolve; ++id) {
        const State2 &st = hst[id];
        lbm_result2d &r = results[id];
        r.q[0] = st.q[0]; r.q[1] = st.q[1];
        r.se[0] = st.se[0]; r.se[1] = st.se[1];
        r.steps = st.steps;
        r.converged = st.converged;
        r.status = st.status;
        const double num = frh[2 * id], den = frh[2 * id + 1];
        r.fieldres = den > 0.0 ? (double)(float)std::sqrt(num / den) : 10.0;
        if (st.status) {
            ctx->err = "non-finite flux in structure " + std::to_string(id / ndir) + " run " +
                       std::to_string(id % ndir) + " at step " + std::to_string(st.steps);
            out = LBM_EINPUT;
        } else if (!st.converged && out == LBM_OK) {
            out = LBM_NOT_CONVERGED;
        }
    }
    return out;
}

extern "C" int lbm_debug_steps2d(lbm_ctx *ctx, const uint8_t *solid, int nx, int ny,
                                 const double force[2], double tau, long long nsteps,
                                 float *f_out, float *u_out, double q_out[2])
{
    if (!ctx) return LBM_EINPUT;
    CK(cudaSetDevice(ctx->device));
    if (nx <= 0 || ny <= 0) return lbm_fail_input(ctx, "bad dimensions");
    if ((long long)nx * ny >= (1ll << 27)) return lbm_fail_input(ctx, "2D lattice too large");
    lbm_params2d p;
    memset(&p, 0, sizeof(p));
    p.tau = tau; p.lag = LLONG_MAX / 4; p.hold = 1 << 30; p.max_steps = nsteps;
    p.avg_steps = 0; p.avg_sample = LLONG_MAX / 4; p.eps = 0.0; p.ksigma = 0.0;
    int rc = check_params2d(ctx, p);
    if (rc) return rc;
    DevMem mask(ctx->stream), d_states(ctx->stream), d_solves(ctx->stream), d_work(ctx->stream);
    Set2 set;
    int nwork = 0;
    rc = setup2d(ctx, solid, nx, ny, 1, force, p, mask, set, d_states, d_solves, d_work, nwork);
    if (rc) return rc;
    rc = run_plain2d(ctx, set.hs, static_cast<Solve2 *>(d_solves.p), static_cast<State2 *>(d_states.p),
                     static_cast<const int2 *>(d_work.p), nwork, set.hst);
    if (rc) return rc;
    const Solve2 &S = set.hs[0];
    if (f_out) {
        DevMem fb(ctx->stream);
        CK(fb.alloc(sizeof(float) * Q2 * (size_t)S.nn));
        canon2d_kernel<<<256, 256, 0, ctx->stream>>>(S, nsteps, static_cast<float *>(fb.p));
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(f_out, fb.p, sizeof(float) * Q2 * S.nn, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    if (u_out) CK(cudaMemcpyAsync(u_out, S.last, sizeof(float) * 2 * S.nn, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (q_out) { q_out[0] = set.hst[0].q[0]; q_out[1] = set.hst[0].q[1]; }
    return LBM_OK;
}
