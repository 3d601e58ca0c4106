/*
 * CPU oracle for the lattice-Boltzmann permeability solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * solvers, used by tests/, by __graft_entry__.smoke() and by bench.py's
 * cpu_baseline leg as the checker.  The product path (the CUDA library
 * liblbm.so and the Python host above it) never links, loads or calls it.
 *
 *   D3Q19, FP64  : LMB3d/lbm3d-perm.cpp:93-398   (operator, pull stream, solve())
 *   D2Q9,  FP32  : LMB2d/lbm.cpp:188-199,247-258,563-632,712-726 and
 *                  LMB2d/main.cpp:99-235          (macro/collision/transport, solve())
 *
 * Arithmetic follows the reference's operation order term by term.  The file
 * is compiled with -ffp-contract=off so that the CUDA FP64 (3D) and FP32 (2D)
 * kernels, which are compiled without FMA contraction for the same reason,
 * can be compared with it bit for bit per step.  The reference 3D build uses
 * -ffast-math, so against the reference binary itself parity is a tolerance
 * (pinned by the golden fixtures in tests/golden/), not bit identity.
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    double tau;        /* relaxation time (reference: static const 1.0)      */
    double eps;        /* drift tolerance relative to ||q||                  */
    long   lag;        /* steps between checks                               */
    int    hold;       /* consecutive passing checks required                */
    long   min_steps;
    long   max_steps;
    long   avg_steps;
} or3d_params;

typedef struct {
    double q[3];
    double se[3];
    long   steps;
    int    converged;
    int    status;     /* 0 ok, 2 non-finite flux (reference: die(), exit 2) */
} or3d_result;

/* Opaque 3D state (two AoS FP64 buffers, as LMB3d/lbm3d-perm.cpp:147-154). */
typedef struct or3d_state or3d_state;

or3d_state *or3d_new(const uint8_t *solid, int nx, int ny, int nz, double tau);
void   or3d_free(or3d_state *st);
void   or3d_reset(or3d_state *st, double fx, double fy, double fz);
void   or3d_step(or3d_state *st);
void   or3d_volumeavg(const or3d_state *st, double q[3]);
/* f*_k(x) after the last step, AoS [node][19]; U,V,W of the last collision. */
const double *or3d_f(const or3d_state *st);
void   or3d_velocity(const or3d_state *st, double *u /* 3*N, x fastest, interleaved */);

/* Whole solve of one forcing direction (LMB3d/lbm3d-perm.cpp:320-398).
 * vel_out (nullable): N*3 float32, x fastest, the field export_velocity writes. */
int or3d_solve(const uint8_t *solid, int nx, int ny, int nz,
               const double force[3], const or3d_params *p,
               or3d_result *r, float *vel_out);

/* ---- D2Q9 ---------------------------------------------------------------- */
typedef struct {
    double tau;
    double eps;
    long   lag;
    int    hold;
    long   min_steps;
    long   max_steps;
    long   avg_steps;
    long   avg_sample;
    double qfloor;
    double ksigma;
} or2d_params;

typedef struct {
    double q[2];
    double se[2];
    long   steps;
    int    converged;
    int    status;
    double fieldres;
} or2d_result;

typedef struct or2d_state or2d_state;

/* solid is indexed [y][x] (x fastest), 1 = solid, as the host reader returns it. */
or2d_state *or2d_new(const uint8_t *solid, int nx, int ny, float tau);
void   or2d_free(or2d_state *st);
void   or2d_reset(or2d_state *st, float fx, float fy);
void   or2d_step(or2d_state *st);
void   or2d_volumeavg(const or2d_state *st, double *qx, double *qy);
/* distributions of the buffer the next step will read, as [y][x][9] */
void   or2d_f(const or2d_state *st, float *out);
void   or2d_velocity(const or2d_state *st, float *u /* [y][x][2] */);

int or2d_solve(const uint8_t *solid, int nx, int ny, const double force[2],
               const or2d_params *p, or2d_result *r, float *vel_out);

#ifdef __cplusplus
}
#endif
#endif
