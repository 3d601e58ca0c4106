/*
 * liblbm — B200 lattice-Boltzmann permeability solver, C ABI.
 *
 * The reference has no library interface: its solvers are processes
 * (LMB3d/lbm3d-perm.cpp:478-631, LMB2d/main.cpp:237-427) driven through
 * subprocess by scripts/solve_permeability3d.py:113-146 and
 * scripts/solve_permeability.py:29-46.  These entry points replace the
 * in-process pieces of those binaries; the argv / CSV / exit-code surface is
 * kept by the Python host (flow_anizotropy_b200.cli3d / cli2d), which calls
 * this ABI through ctypes.
 *
 * Conventions
 *   - Plain pointers and sizes only.  `solid` and `vel_out` may be host or
 *     device pointers (detected with cudaPointerGetAttributes); results are
 *     host structs.
 *   - Voxel order is x fastest, then y, then z (the .raw payload order,
 *     scripts/structure_io3d.py:13-18); 1 = solid, 0 = pore.
 *   - Return codes: LBM_OK (0) = all solves converged; LBM_NOT_CONVERGED (3)
 *     = results valid but some `converged` flag is 0 (the reference's exit 3);
 *     LBM_EINPUT (2) = bad input or non-finite flux (the reference's exit 2,
 *     LMB3d/lbm3d-perm.cpp:140-144,339-341); LBM_EBUSY (4) = a batch has no
 *     room; LBM_ECUDA (-1) = CUDA error.  Nothing here calls exit() or traps.
 *     lbm_last_error() returns the message of the last failing call.
 *   - One context per process and device; calls on one context are serialised
 *     by the caller.  The library owns its lattice allocations.
 */
#ifndef LBM_H
#define LBM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_API_VERSION 1

#define LBM_OK             0
#define LBM_EINPUT         2
#define LBM_NOT_CONVERGED  3
#define LBM_EBUSY          4
#define LBM_ECUDA        (-1)

/* lbm_params3d.variant: the library's default for the precision (the
 * variant the autotuner picks on the 128^3 tensor workload: FP32 76, FP16 and
 * BF16 150, 0 otherwise; a batch takes the same defaults).  Every variant of
 * a precision gives the same
 * bits.  For FP32, FP16 and BF16, variants v < 75 are the in-place (AA)
 * lattice, odd-step kernel v / 15 and even-step kernel v % 15; v = 75..80
 * are the two-lattice pull form (one kernel for every step); v = 81..155 are
 * the two-lattice AA form of in-place variant v - 81 (the same kernels, the
 * even step scattering into the other lattice).  FP64: odd-step kernel v / 6
 * and even-step kernel v % 6 for v < 18, the two-lattice AA form of v - 18
 * for v = 18..35.  The two-lattice forms take twice the lattice memory. */
#define LBM_VARIANT_DEFAULT (-1)

/* Population storage (collision arithmetic is FP64 for LBM_FP64, else FP32;
 * flux reductions, convergence test and averaging are FP64 in every mode). */
#define LBM_FP64  0   /* f_k as double, the reference's own arithmetic           */
#define LBM_FP32  1   /* shifted populations f_k - w_k as float                  */
#define LBM_FP16  2   /* shifted populations, power-of-two scaled, IEEE half     */
#define LBM_BF16  3   /* shifted populations as bfloat16                         */
/* tau = 1 only: the post-collision populations are a function of a voxel's
 * moments, so the state is (rho - 1, u) per pore voxel (exact reformulation;
 * rounding at the storage precision). */
#define LBM_M32   4   /* moments as float, FP32 arithmetic                       */
#define LBM_M64   5   /* moments as double, FP64 arithmetic                      */
#define LBM_MD32  6   /* moments as float over the dense voxel box, z-planes    */
                      /* staged in shared memory by TMA                          */

/* Phase-1 convergence criterion */
#define LBM_CRIT_DRIFT  0  /* every lag steps: max_c |q_c - qprev_c| < eps ||q||
                              (LMB3d/lbm3d-perm.cpp:332-360)                     */
#define LBM_CRIT_BLOCK  1  /* block means over lag steps sampled every `sample`
                              steps, accepted within max(eps ||m||, ksigma * SE)
                              (the 2D reference's test, LMB2d/main.cpp:123-178) */
#define LBM_CRIT_BATCH  2  /* LBM_CRIT_BLOCK with the SE of a block taken from
                              the means of its 10 sub-blocks (batch means), so
                              noise correlated over many steps (stochastic
                              rounding of 16-bit storage) is not underrated   */

typedef struct lbm_ctx lbm_ctx;

/* Solver knobs of LMB3d/lbm3d-perm.cpp:118-130 plus tau (a compile-time
 * constant there, :112), storage precision and criterion. */
typedef struct {
    double    tau;
    double    eps;
    long long lag;
    long long min_steps;
    long long max_steps;
    long long avg_steps;
    int       hold;
    int       precision;
    int       criterion;
    int       variant;      /* step-kernel variant (see lbm_tune3d), or LBM_VARIANT_DEFAULT */
    long long sample;       /* LBM_CRIT_BLOCK sample interval                 */
    double    ksigma;       /* LBM_CRIT_BLOCK acceptance                      */
} lbm_params3d;

/* Per-direction result: struct Solve of LMB3d/lbm3d-perm.cpp:132-138. */
typedef struct {
    double    q[3];         /* Darcy flux mean(u) over ALL nodes              */
    double    se[3];        /* standard error over the averaging phase        */
    long long steps;
    int       converged;
    int       status;       /* 0; 2 non-finite flux; 5 a copy wait ran out    */
} lbm_result3d;

/* D2Q9 knobs of LMB2d/main.cpp:64-79 plus tau (LMB2d/lbm.cpp:86). */
typedef struct {
    double    tau;
    double    eps;
    long long lag;
    long long min_steps;
    long long max_steps;
    long long avg_steps;
    long long avg_sample;
    double    qfloor;
    double    ksigma;
    int       hold;
    int       reserved;
} lbm_params2d;

/* struct Solve of LMB2d/main.cpp:81-89 */
typedef struct {
    double    q[2];
    double    se[2];
    long long steps;
    int       converged;
    int       status;
    double    fieldres;
} lbm_result2d;

/* ---- context ---------------------------------------------------------- */
int         lbm_version(void);
int         lbm_create(lbm_ctx **ctx, int device);
void        lbm_destroy(lbm_ctx *ctx);
const char *lbm_last_error(const lbm_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t), on which every kernel of the
 * context is launched: for timing with CUDA events from the caller. */
void       *lbm_stream(const lbm_ctx *ctx);

/* ---- plain solves ----------------------------------------------------- */

/* ndir forcing directions of one structure, each to convergence, concurrently
 * (one lattice per direction, one launch per step for all of them).
 * Replaces the three sequential solve() calls of LMB3d/lbm3d-perm.cpp:518-520
 * (and the fourth, --validate, :558) together with read_structure (:174-193).
 * forces: ndir x 3 doubles.  results: ndir.  vel_out: NULL or
 * ndir x nx*ny*nz x 3 floats, the export_velocity field (:305-317) of each
 * direction. */
int lbm_solve3d(lbm_ctx *ctx, const uint8_t *solid, int nx, int ny, int nz,
                int ndir, const double *forces, const lbm_params3d *params,
                lbm_result3d *results, float *vel_out);

/* D2Q9: solve() of LMB2d/main.cpp:99-235 with macro/collision/transport of
 * LMB2d/lbm.cpp:563-632, for a runtime nx x ny cell (the reference is fixed
 * at 256 x 256, LMB2d/lbm.h:24-25).  solid is ny x nx, x fastest.
 * vel_out: NULL or ndir x nx*ny x 2 floats (U, V of the last step). */
int lbm_solve2d(lbm_ctx *ctx, const uint8_t *solid, int nx, int ny,
                int ndir, const double *forces, const lbm_params2d *params,
                lbm_result2d *results, float *vel_out);

/* nstruct structures of one nx x ny cell (solids: nstruct x ny x nx), each
 * solved along the same ndir forcing directions, all advanced by one launch
 * per step; results: nstruct x ndir, structure-major, each equal to
 * lbm_solve2d of that structure alone.  Replaces nstruct lbm2d-perm processes
 * of scripts/solve_permeability.py:29-46 (LMB2d/main.cpp:99-235 each). */
int lbm_solve2d_many(lbm_ctx *ctx, int nstruct, const uint8_t *solids, int nx, int ny, int ndir,
                     const double *forces, const lbm_params2d *params, lbm_result2d *results);

/* Largest input of lbm_solve2d_noalloc: the reference's fixed 256 x 256 cell
 * (LMB2d/lbm.h:24-26) and its two forcing directions (LMB2d/main.cpp:323-324). */
#define LBM_NOALLOC2D_MAX_CELLS 65536
#define LBM_NOALLOC2D_MAX_DIRS  2

/* lbm_solve2d that allocates no device memory.  No counterpart in the
 * reference (whose 2D solver keeps its lattice in static arrays,
 * LMB2d/lbm.cpp:18-28; this entry point keeps that property on the device).
 * Same arguments, codes and results (bit for bit) as lbm_solve2d, for callers
 * that must not allocate: device memory already owned by another allocator,
 * or a loop that cannot take the synchronisation of cudaFree.  Lattices, mask
 * and controller state live in one static device array of this library
 * (about 7 MB per device, reserved when the library's device code is loaded).
 *   nx * ny > LBM_NOALLOC2D_MAX_CELLS or ndir > LBM_NOALLOC2D_MAX_DIRS:
 * LBM_EINPUT, with lbm_last_error naming the limit.
 *   Every call looks up the array (cudaGetSymbolAddress, so a device reset
 * between calls is harmless); a device's first call may load the library's
 * device code there: make it before any stream capture.  The call
 * synchronises its stream and is not capturable.
 *   One array per device and process: overlapping calls on one device would
 * race on it, so they are serialised by a per-device lock.
 *   The time loop launches one step at a time from the host (about 8.6 us per
 * step on 256 x 256 against 6.8 us for lbm_solve2d's graph chunks). */
int lbm_solve2d_noalloc(lbm_ctx *ctx, const uint8_t *solid, int nx, int ny,
                        int ndir, const double *forces, const lbm_params2d *params,
                        lbm_result2d *results, float *vel_out);

/* ---- batched / served solves ------------------------------------------ */
typedef struct lbm_batch lbm_batch;

/* A resident set of 3D solves of one storage precision advanced together:
 * each CUDA-graph launch runs `chunk` steps of every unfinished solve, each at
 * its own step count; solves finish (retire) independently.  hbm_budget is
 * the device memory the batch may hold for lattices, in bytes. */
int  lbm_batch_create(lbm_ctx *ctx, lbm_batch **batch, int precision,
                      long long hbm_budget, int chunk);

/* Step-kernel variant of every launch of an empty batch (default
 * LBM_VARIANT_DEFAULT, the variant lbm_tune3d picks on the 128^3 tensor
 * workload; mixes of small structures may prefer another).  Results do not
 * depend on it.  With a grouped even-step variant a structure's directions
 * take consecutive slots and stay resident until all of them are done.
 * LBM_EINPUT while solves are resident, and for the grouped pull variants
 * (79-80: every launch by structure; the batch steps its odd launches per
 * direction). */
int  lbm_batch_set_variant(lbm_batch *batch, int variant);
void lbm_batch_destroy(lbm_batch *batch);

/* Upper bound on the device bytes one structure with ndir directions
 * occupies in a batch (as if every voxel were a pore, and with the pull
 * form's two lattices for FP32, FP16 and BF16; lattices hold pore voxels
 * only, and admission charges the exact size of the batch's variant). */
long long lbm_batch_bytes3d(int nx, int ny, int nz, int ndir, int precision);

/* Admit one structure with ndir directions (results are reported per
 * direction under (tag, dir)).  LBM_EBUSY if it does not fit the budget now. */
int  lbm_batch_submit3d(lbm_batch *batch, const uint8_t *solid, int nx, int ny, int nz,
                        int ndir, const double *forces, const lbm_params3d *params,
                        long long tag);

/* Advance every resident solve by `chunks` graph launches. */
int  lbm_batch_run(lbm_batch *batch, int chunks);

/* Retire finished solves: up to `max` (tag, dir, result) triples; *n gets
 * the count.  Their memory returns to the budget. */
int  lbm_batch_poll(lbm_batch *batch, long long *tags, int *dirs,
                    lbm_result3d *results, int max, int *n);

/* Unfinished solves in the batch, and the lattice bytes it holds now. */
int       lbm_batch_active(const lbm_batch *batch);
long long lbm_batch_resident_bytes(const lbm_batch *batch);

/* ---- structure generation (scripts/gen_aniso_structures3d.py datasets) - */

/* The random trigonometric field of gen_aniso_structures3d.py:154-176 over a
 * size^3 periodic cell, S = scale * sum_m cos(((2 pi qz_m) z + (2 pi qy_m) y)
 * + (2 pi qx_m) x + phases[m]) at the coordinates pts[0..size) of each axis,
 * in the reference's operation order; *threshold = numpy's linear quantile of
 * S at `porosity` (:179-181) and solid_out = S > *threshold (size^3 bytes,
 * x fastest; host or device pointer).  q: n_modes x 3 int32 (qx, qy, qz). */
int lbm_trig_structure3d(lbm_ctx *ctx, int size, int n_modes, const int32_t *q, const double *phases,
                         const double *pts, double scale, double porosity, uint8_t *solid_out,
                         double *threshold);

/* Percolation of the pore phase (solid = 0) of gen_aniso_structures3d.py:184-205:
 * 6-connected components of the 3 x 3 x 3 tiling; perc[a] = 1 if a component
 * touches both faces of axis a (x, y, z).  27 nx ny nz < 2^31. */
int lbm_percolates3d(lbm_ctx *ctx, const uint8_t *solid, int nx, int ny, int nz, int perc[3]);

/* ---- autotuning ------------------------------------------------------ */

/* Number of step-kernel variants (pore voxels per thread x register budget)
 * for a storage precision. */
int lbm_variant_count(int precision);

/* Time every step-kernel variant on this structure (ndir directions resident,
 * `nsteps` timed steps each after a warm-up) with CUDA events; ms_per_step
 * (may be NULL) receives lbm_variant_count(precision) values and *best the
 * fastest variant.  No counterpart in the reference, which has one loop. */
int lbm_tune3d(lbm_ctx *ctx, const uint8_t *solid, int nx, int ny, int nz, int ndir,
               int precision, int nsteps, double *ms_per_step, int *best);

/* ---- diagnostics (used by the parity tests) --------------------------- */

/* Run exactly nsteps steps of one 3D solve and return the post-collision
 * populations f*_k(x) in the reference's AoS order (N x 19 doubles; pores
 * only, solids 0), the velocity of the last step (N x 3 floats) and the flux
 * of the last step from the fused reduction.  Any output may be NULL. */
int lbm_debug_steps3d(lbm_ctx *ctx, const uint8_t *solid, int nx, int ny, int nz,
                      const double force[3], double tau, int precision, int variant,
                      long long nsteps, double *f_out, float *u_out, double q_out[3]);

/* Test knobs of the bulk-staged odd step (odd variant 4) in this context:
 * wait_ns replaces the 1 s limit of its waits on shared-memory copies (0
 * restores it), and starve != 0 makes its producer issue nothing, so the
 * waits run out: the solve then ends with status 5 and the call returns
 * LBM_ECUDA, the context staying usable.  No counterpart in the reference. */
int lbm_debug_bulk_wait(lbm_ctx *ctx, unsigned long long wait_ns, int starve);

/* 2D counterpart: populations of the buffer the next step reads, ny x nx x 9
 * floats, the U,V of the last step (ny x nx x 2) and its flux. */
int lbm_debug_steps2d(lbm_ctx *ctx, const uint8_t *solid, int nx, int ny,
                      const double force[2], double tau, long long nsteps,
                      float *f_out, float *u_out, double q_out[2]);

#ifdef __cplusplus
}
#endif
#endif /* LBM_H */
