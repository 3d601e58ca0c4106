/*
 * D3Q19 FP64 oracle — TEST INFRASTRUCTURE ONLY (never on the product path).
 *
 * Restates the reference solver LMB3d/lbm3d-perm.cpp for use as a checker:
 *   velocity set, weights, opposite table ........ :94-110
 *   TAU / CS2 / MU (tau is a parameter here) ..... :112-114
 *   reset to w_k, U=V=W=0 ........................ :203-212
 *   collide_node (BGK + Guo forcing) ............. :218-245
 *   collide_only (first step) .................... :249-253
 *   stream_collide (pull + halfway bounce-back) .. :270-289
 *   volumeavg (mean over ALL nodes) .............. :298-303
 *   solve() convergence + averaging .............. :320-398
 *
 * Two AoS buffers f0/f1 ([node][19]) exactly like the reference, so this file
 * also documents, by contrast, the in-place AA layout the CUDA kernels use.
 * Compiled with -ffp-contract=off; every expression keeps the reference's
 * evaluation order.
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define Q3 19

/* LMB3d/lbm3d-perm.cpp:95-102 */
static const int EX[Q3] = {0, 1,-1, 0, 0, 0, 0, 1,-1, 1,-1, 1,-1, 1,-1, 0, 0, 0, 0};
static const int EY[Q3] = {0, 0, 0, 1,-1, 0, 0, 1,-1,-1, 1, 0, 0, 0, 0, 1,-1, 1,-1};
static const int EZ[Q3] = {0, 0, 0, 0, 0, 1,-1, 0, 0, 0, 0, 1,-1,-1, 1, 1,-1,-1, 1};
static const double WQ[Q3] = {
    1.0/3.0,
    1.0/18.0, 1.0/18.0, 1.0/18.0, 1.0/18.0, 1.0/18.0, 1.0/18.0,
    1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0,
    1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0};

struct or3d_state {
    int nx, ny, nz;
    long nn;
    uint8_t *solid;
    double *f0, *f1;
    double *U, *V, *W, *RHO;
    double F[3];
    double tau;
    int primed;
    int opp[Q3];
};

static long wrap(long a, long n) { return ((a % n) + n) % n; }

or3d_state *or3d_new(const uint8_t *solid, int nx, int ny, int nz, double tau)
{
    or3d_state *st = (or3d_state *)calloc(1, sizeof(*st));
    st->nx = nx; st->ny = ny; st->nz = nz;
    st->nn = (long)nx * ny * nz;
    st->tau = tau;
    st->solid = (uint8_t *)malloc((size_t)st->nn);
    memcpy(st->solid, solid, (size_t)st->nn);
    st->f0 = (double *)malloc(sizeof(double) * (size_t)st->nn * Q3);
    st->f1 = (double *)malloc(sizeof(double) * (size_t)st->nn * Q3);
    st->U = (double *)calloc((size_t)st->nn, sizeof(double));
    st->V = (double *)calloc((size_t)st->nn, sizeof(double));
    st->W = (double *)calloc((size_t)st->nn, sizeof(double));
    st->RHO = (double *)calloc((size_t)st->nn, sizeof(double));
    for (int k = 0; k < Q3; k++)
        for (int m = 0; m < Q3; m++)
            if (EX[m] == -EX[k] && EY[m] == -EY[k] && EZ[m] == -EZ[k]) { st->opp[k] = m; break; }
    or3d_reset(st, 0.0, 0.0, 0.0);
    return st;
}

void or3d_free(or3d_state *st)
{
    if (!st) return;
    free(st->solid); free(st->f0); free(st->f1);
    free(st->U); free(st->V); free(st->W); free(st->RHO);
    free(st);
}

/* LMB3d/lbm3d-perm.cpp:203-212 plus the force assignment of solve() :324 */
void or3d_reset(or3d_state *st, double fx, double fy, double fz)
{
    for (long i = 0; i < st->nn; i++) {
        for (int k = 0; k < Q3; k++) st->f0[i * Q3 + k] = st->f1[i * Q3 + k] = WQ[k];
        st->U[i] = st->V[i] = st->W[i] = 0.0;
        st->RHO[i] = 1.0;
    }
    st->F[0] = fx; st->F[1] = fy; st->F[2] = fz;
    st->primed = 0;
}

/* LMB3d/lbm3d-perm.cpp:218-245: moments, Guo half-force velocity, BGK with
 * the Guo source term.  g and out may alias. */
static void collide_node(or3d_state *st, long i, const double *g, double *out)
{
    const double Fx = st->F[0], Fy = st->F[1], Fz = st->F[2];
    const double tau = st->tau;
    double r = 0, ux = 0, uy = 0, uz = 0;
    for (int k = 0; k < Q3; k++) {
        r += g[k];
        ux += g[k] * EX[k]; uy += g[k] * EY[k]; uz += g[k] * EZ[k];
    }
    st->RHO[i] = r;
    ux = st->U[i] = (ux + 0.5 * Fx) / r;
    uy = st->V[i] = (uy + 0.5 * Fy) / r;
    uz = st->W[i] = (uz + 0.5 * Fz) / r;

    const double u2 = ux * ux + uy * uy + uz * uz;
    const double pref = 1.0 - 0.5 / tau;
    double res[Q3];
    for (int k = 0; k < Q3; k++) {
        const double eu = EX[k] * ux + EY[k] * uy + EZ[k] * uz;
        const double feq = WQ[k] * r * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * u2);
        const double sk = WQ[k] * pref *
            (3.0 * ((EX[k] - ux) * Fx + (EY[k] - uy) * Fy + (EZ[k] - uz) * Fz)
             + 9.0 * eu * (EX[k] * Fx + EY[k] * Fy + EZ[k] * Fz));
        res[k] = g[k] + ((feq - g[k]) / tau + sk);
    }
    memcpy(out, res, sizeof(res));
}

/* LMB3d/lbm3d-perm.cpp:249-253, :270-295 */
void or3d_step(or3d_state *st)
{
    const int nx = st->nx, ny = st->ny, nz = st->nz;
    if (!st->primed) {
        for (long i = 0; i < st->nn; i++)
            if (!st->solid[i]) collide_node(st, i, &st->f0[i * Q3], &st->f0[i * Q3]);
        st->primed = 1;
        return;
    }
    double g[Q3];
    for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
    for (int x = 0; x < nx; x++) {
        const long i = ((long)z * ny + y) * nx + x;
        if (st->solid[i]) continue;
        for (int k = 0; k < Q3; k++) {
            const long px = wrap(x - EX[k], nx), py = wrap(y - EY[k], ny), pz = wrap(z - EZ[k], nz);
            const long p = (pz * ny + py) * nx + px;
            g[k] = st->solid[p] ? st->f0[i * Q3 + st->opp[k]] : st->f0[p * Q3 + k];
        }
        collide_node(st, i, g, &st->f1[i * Q3]);
    }
    double *t = st->f0; st->f0 = st->f1; st->f1 = t;
}

/* LMB3d/lbm3d-perm.cpp:298-303: sequential sum over all nodes, / N */
void or3d_volumeavg(const or3d_state *st, double q[3])
{
    double su = 0, sv = 0, sw = 0;
    for (long i = 0; i < st->nn; i++) { su += st->U[i]; sv += st->V[i]; sw += st->W[i]; }
    q[0] = su / (double)st->nn; q[1] = sv / (double)st->nn; q[2] = sw / (double)st->nn;
}

const double *or3d_f(const or3d_state *st) { return st->f0; }

void or3d_velocity(const or3d_state *st, double *u)
{
    for (long i = 0; i < st->nn; i++) {
        u[3 * i] = st->U[i]; u[3 * i + 1] = st->V[i]; u[3 * i + 2] = st->W[i];
    }
}

/* LMB3d/lbm3d-perm.cpp:320-398 */
int or3d_solve(const uint8_t *solid, int nx, int ny, int nz,
               const double force[3], const or3d_params *p,
               or3d_result *r, float *vel_out)
{
    memset(r, 0, sizeof(*r));
    or3d_state *st = or3d_new(solid, nx, ny, nz, p->tau);
    or3d_reset(st, force[0], force[1], force[2]);

    long s = 0;
    int hold = 0, have_prev = 0;
    double qprev[3] = {0, 0, 0};

    while (s < p->max_steps) {
        or3d_step(st); s++;
        if (s % p->lag) continue;
        double q[3];
        or3d_volumeavg(st, q);
        for (int c = 0; c < 3; c++)
            if (!isfinite(q[c])) { r->status = 2; r->steps = s; or3d_free(st); return 2; }
        const double norm = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
        double drift = 0.0;
        for (int c = 0; c < 3; c++) drift = fmax(drift, fabs(q[c] - qprev[c]));
        if (have_prev && s >= p->min_steps && drift < p->eps * norm) hold++;
        else hold = 0;
        for (int c = 0; c < 3; c++) qprev[c] = q[c];
        have_prev = 1;
        if (hold >= p->hold) break;
    }
    r->converged = (hold >= p->hold) ? 1 : 0;

    double sum[3] = {0, 0, 0}, sumsq[3] = {0, 0, 0};
    long n = 0;
    for (long i = 0; i < p->avg_steps; i++) {
        or3d_step(st); s++;
        double q[3];
        or3d_volumeavg(st, q);
        for (int c = 0; c < 3; c++) { sum[c] += q[c]; sumsq[c] += q[c] * q[c]; }
        n++;
    }
    if (n == 0) or3d_volumeavg(st, r->q);
    else
        for (int c = 0; c < 3; c++) {
            r->q[c] = sum[c] / n;
            if (n > 1) {
                const double var = (sumsq[c] - n * r->q[c] * r->q[c]) / (n - 1);
                r->se[c] = sqrt(fmax(var, 0.0) / n);
            }
        }
    r->steps = s;
    if (vel_out)
        for (long i = 0; i < st->nn; i++) {
            vel_out[3 * i] = (float)st->U[i];
            vel_out[3 * i + 1] = (float)st->V[i];
            vel_out[3 * i + 2] = (float)st->W[i];
        }
    or3d_free(st);
    return 0;
}
