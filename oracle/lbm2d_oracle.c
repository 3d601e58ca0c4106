/*
 * D2Q9 FP32 oracle — TEST INFRASTRUCTURE ONLY (never on the product path).
 *
 * Restates the reference 2D solver with a runtime lattice size:
 *   velocity set, inverse table, weights ......... LMB2d/lbm.cpp:67-70
 *   tau = 1, mu = 0.33 (tau - 1/2) ................ LMB2d/lbm.cpp:86-87
 *   volumeavg, q = sum(u) / (L * L0^2), L0 = 4 .... LMB2d/lbm.cpp:188-199, lbm.h:26-28
 *   snapshot_field / field_residual ............... LMB2d/lbm.cpp:207-229
 *   resetdistributions ............................ LMB2d/lbm.cpp:247-258
 *   macro / collision / transport ................. LMB2d/lbm.cpp:563-632
 *   lbm() parity flip ............................. LMB2d/lbm.cpp:712-726
 *   solve() block-mean k-sigma controller ......... LMB2d/main.cpp:99-235
 *
 * The reference 2D build is plain -O3 (no -ffast-math, no FMA on the default
 * x86-64 target), i.e. strict IEEE float in source order; this file keeps that
 * order and is compiled with -ffp-contract=off, so per step it is bit-identical
 * to the reference and to the CUDA D2Q9 kernel.
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define Q2 9
#define L0_2D 4.0          /* LMB2d/lbm.h:26 (legacy normalisation length) */

static const int EX2[Q2] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
static const int EY2[Q2] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
static const int INV2[Q2] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
static const float W2[Q2] = {4.0f/9.0f, 1.0f/9.0f, 1.0f/9.0f, 1.0f/9.0f, 1.0f/9.0f,
                             1.0f/36.0f, 1.0f/36.0f, 1.0f/36.0f, 1.0f/36.0f};

struct or2d_state {
    int nx, ny;            /* LX, LY */
    uint8_t *F;            /* F[x][y] as the reference: index x*ny + y */
    float *df;             /* df[2][x][y][9] */
    float *U, *V, *R;      /* [x][y] */
    float *US, *VS;        /* snapshot */
    float fx, fy, tau;
    int c;                 /* lbm_c */
};

#define DF(st, c, i, j, k) (st)->df[((((size_t)(c) * (st)->nx + (i)) * (st)->ny + (j)) * Q2) + (k)]
#define AT(st, a, i, j) (st)->a[(size_t)(i) * (st)->ny + (j)]

or2d_state *or2d_new(const uint8_t *solid, int nx, int ny, float tau)
{
    or2d_state *st = (or2d_state *)calloc(1, sizeof(*st));
    st->nx = nx; st->ny = ny; st->tau = tau;
    const size_t nn = (size_t)nx * ny;
    st->F = (uint8_t *)malloc(nn);
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            st->F[(size_t)i * ny + j] = solid[(size_t)j * nx + i] ? 1 : 0;
    st->df = (float *)malloc(sizeof(float) * nn * 2 * Q2);
    st->U = (float *)calloc(nn, sizeof(float));
    st->V = (float *)calloc(nn, sizeof(float));
    st->R = (float *)calloc(nn, sizeof(float));
    st->US = (float *)calloc(nn, sizeof(float));
    st->VS = (float *)calloc(nn, sizeof(float));
    or2d_reset(st, 0.0f, 0.0f);
    return st;
}

void or2d_free(or2d_state *st)
{
    if (!st) return;
    free(st->F); free(st->df); free(st->U); free(st->V); free(st->R);
    free(st->US); free(st->VS); free(st);
}

/* LMB2d/lbm.cpp:247-258 (+ the fx/fy assignment of main.cpp:104-106) */
void or2d_reset(or2d_state *st, float fx, float fy)
{
    for (int i = 0; i < st->nx; i++)
        for (int j = 0; j < st->ny; j++) {
            for (int k = 0; k < Q2; k++) DF(st, 0, i, j, k) = DF(st, 1, i, j, k) = W2[k];
            AT(st, U, i, j) = AT(st, V, i, j) = 0.0f;
            AT(st, R, i, j) = 1.0f;
        }
    st->c = 1;
    st->fx = fx; st->fy = fy;
}

static void macro(or2d_state *st, int c)
{
    for (int i = 0; i < st->nx; i++)
        for (int j = 0; j < st->ny; j++)
            if (AT(st, F, i, j) == 0) {
                float rho = 0, ux = 0, uy = 0;
                for (int k = 0; k < Q2; k++) {
                    rho = rho + DF(st, c, i, j, k);
                    ux = ux + DF(st, c, i, j, k) * EX2[k];
                    uy = uy + DF(st, c, i, j, k) * EY2[k];
                }
                ux /= rho;
                uy /= rho;
                AT(st, U, i, j) = ux;
                AT(st, V, i, j) = uy;
                AT(st, R, i, j) = rho;
            }
}

static void collision(or2d_state *st, int c)
{
    const float fx = st->fx, fy = st->fy, tau = st->tau;
    for (int i = 0; i < st->nx; i++)
        for (int j = 0; j < st->ny; j++)
            if (AT(st, F, i, j) == 0) {
                float ux = AT(st, U, i, j), uy = AT(st, V, i, j), rho = AT(st, R, i, j);
                ux = ux + fx * tau / rho;
                uy = uy + fy * tau / rho;
                for (int k = 0; k < Q2; k++) {
                    const float feq = W2[k] * rho * (1.0f - (3.0f / 2.0f) * (ux * ux + uy * uy)
                        + 3.0f * (EX2[k] * ux + EY2[k] * uy)
                        + (9.0f / 2.0f) * (EX2[k] * ux + EY2[k] * uy) * (EX2[k] * ux + EY2[k] * uy));
                    DF(st, c, i, j, k) = DF(st, c, i, j, k) - (1 / tau) * (DF(st, c, i, j, k) - feq);
                }
            }
}

static void transport(or2d_state *st, int c)
{
    const int nx = st->nx, ny = st->ny;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            if (AT(st, F, i, j) == 0)
                for (int k = 0; k < Q2; k++) {
                    const int ip = (i + EX2[k] + nx) % nx;
                    const int jp = (j + EY2[k] + ny) % ny;
                    if (AT(st, F, ip, jp) == 1)
                        DF(st, 1 - c, i, j, INV2[k]) = DF(st, c, i, j, k);
                    else
                        DF(st, 1 - c, ip, jp, k) = DF(st, c, i, j, k);
                }
}

void or2d_step(or2d_state *st)
{
    st->c = 1 - st->c;
    macro(st, st->c);
    collision(st, st->c);
    transport(st, st->c);
}

void or2d_volumeavg(const or2d_state *st, double *qx, double *qy)
{
    double su = 0.0, sv = 0.0;
    for (int i = 0; i < st->nx; i++)
        for (int j = 0; j < st->ny; j++) {
            su += AT(st, U, i, j);
            sv += AT(st, V, i, j);
        }
    *qx = su / ((double)st->nx * L0_2D * L0_2D);
    *qy = sv / ((double)st->ny * L0_2D * L0_2D);
}

void or2d_f(const or2d_state *st, float *out)
{
    const int cn = 1 - st->c;     /* the buffer the next step's macro() reads */
    for (int j = 0; j < st->ny; j++)
        for (int i = 0; i < st->nx; i++)
            for (int k = 0; k < Q2; k++)
                out[((size_t)j * st->nx + i) * Q2 + k] = DF(st, cn, i, j, k);
}

void or2d_velocity(const or2d_state *st, float *u)
{
    for (int j = 0; j < st->ny; j++)
        for (int i = 0; i < st->nx; i++) {
            u[((size_t)j * st->nx + i) * 2] = AT(st, U, i, j);
            u[((size_t)j * st->nx + i) * 2 + 1] = AT(st, V, i, j);
        }
}

static void snapshot(or2d_state *st)
{
    const size_t nn = (size_t)st->nx * st->ny;
    memcpy(st->US, st->U, nn * sizeof(float));
    memcpy(st->VS, st->V, nn * sizeof(float));
}

static float field_residual(const or2d_state *st)
{
    double num = 0.0, den = 0.0;
    for (int i = 0; i < st->nx; i++)
        for (int j = 0; j < st->ny; j++) {
            const double du = AT(st, U, i, j) - AT(st, US, i, j);
            const double dv = AT(st, V, i, j) - AT(st, VS, i, j);
            num += du * du + dv * dv;
            den += (double)AT(st, U, i, j) * AT(st, U, i, j) + (double)AT(st, V, i, j) * AT(st, V, i, j);
        }
    return den > 0.0 ? (float)sqrt(num / den) : 10.0f;
}

/* LMB2d/main.cpp:99-235 */
int or2d_solve(const uint8_t *solid, int nx, int ny, const double force[2],
               const or2d_params *p, or2d_result *r, float *vel_out)
{
    memset(r, 0, sizeof(*r));
    or2d_state *st = or2d_new(solid, nx, ny, (float)p->tau);
    or2d_reset(st, (float)force[0], (float)force[1]);

    long s = 0;
    int hold = 0, have_prev = 0;
    double pm_x = 0, pm_y = 0, pse_x = 0, pse_y = 0;
    double bsx = 0, bsy = 0, bsxx = 0, bsyy = 0;
    long bn = 0;

    while (s < p->max_steps) {
        or2d_step(st);
        s++;
        if (s % p->avg_sample == 0) {
            double qx, qy;
            or2d_volumeavg(st, &qx, &qy);
            if (!isfinite(qx) || !isfinite(qy)) { r->status = 2; r->steps = s; or2d_free(st); return 2; }
            bsx += qx; bsxx += qx * qx;
            bsy += qy; bsyy += qy * qy;
            bn++;
        }
        if (s % p->lag || bn < 2) continue;

        const double mx = bsx / bn, my = bsy / bn;
        const double vx = (bsxx - bn * mx * mx) / (bn - 1);
        const double vy = (bsyy - bn * my * my) / (bn - 1);
        const double sex = sqrt(fmax(vx, 0.0) / bn);
        const double sey = sqrt(fmax(vy, 0.0) / bn);
        if (have_prev) {
            const double qmag = sqrt(mx * mx + my * my);
            const double flo = p->qfloor * qmag;
            const double dx = fabs(mx - pm_x), dy = fabs(my - pm_y);
            const double tolx = fmax(p->eps * fmax(fabs(mx), flo), p->ksigma * sqrt(sex * sex + pse_x * pse_x));
            const double toly = fmax(p->eps * fmax(fabs(my), flo), p->ksigma * sqrt(sey * sey + pse_y * pse_y));
            if (s >= p->min_steps && dx < tolx && dy < toly) hold++;
            else hold = 0;
        }
        pm_x = mx; pm_y = my; pse_x = sex; pse_y = sey; have_prev = 1;
        bsx = bsy = bsxx = bsyy = 0.0; bn = 0;
        if (hold >= p->hold) break;
    }
    r->converged = (hold >= p->hold) ? 1 : 0;

    snapshot(st);
    double sx = 0, sy = 0, sxx = 0, syy = 0;
    long n = 0;
    for (long t = 1; t <= p->avg_steps; t++) {
        or2d_step(st);
        s++;
        if (t % p->avg_sample) continue;
        double qx, qy;
        or2d_volumeavg(st, &qx, &qy);
        if (!isfinite(qx) || !isfinite(qy)) { r->status = 2; r->steps = s; or2d_free(st); return 2; }
        sx += qx; sxx += qx * qx;
        sy += qy; syy += qy * qy;
        n++;
    }
    if (n == 0) {
        or2d_volumeavg(st, &r->q[0], &r->q[1]);
    } else {
        r->q[0] = sx / n;
        r->q[1] = sy / n;
        if (n > 1) {
            const double vx = (sxx - n * r->q[0] * r->q[0]) / (n - 1);
            const double vy = (syy - n * r->q[1] * r->q[1]) / (n - 1);
            r->se[0] = sqrt(fmax(vx, 0.0) / n);
            r->se[1] = sqrt(fmax(vy, 0.0) / n);
        }
    }
    r->steps = s;
    r->fieldres = field_residual(st);
    if (vel_out) or2d_velocity(st, vel_out);
    or2d_free(st);
    return 0;
}
