/*
 * oracle.c -- serial FP64 CPU restatement of the iceMPM hot path.
 * TEST INFRASTRUCTURE (see oracle.h): used only as the checker.
 *
 * Matrices are held as named scalars or row-major arrays m[r*2+c]; each
 * expression keeps the reference's evaluation order (citations inline).
 */
#include "oracle.h"

#include <math.h>
#include <stdint.h>
#include <string.h>

static const double PI = 3.14159265358979323846;   /* SimParams::pi */
static const double COEFF1 = 1.4142135623730950;   /* kernels.cuh:10 */
static const double COEFF1_INV = 0.7071067811865475;/* kernels.cuh:11 */

static long long as_ll(double d) { long long v; memcpy(&v, &d, 8); return v; }
static double as_d(long long v) { double d; memcpy(&d, &v, 8); return d; }

long oracle_grid_nodes(const icy_sim_params *p)
{
    return (long)p->GridY * (p->GridXTotal + 2 * p->GridHaloSize);
}

/* quadratic B-spline weights, kernels.cuh:99-103 */
static void weights(double f, double w[3])
{
    double a0 = 1.5 - f, a1 = f - 1.0, a2 = f - 0.5;
    w[0] = (0.5 * a0) * a0;
    w[1] = 0.75 - a1 * a1;
    w[2] = (0.5 * a2) * a2;
}

/* base node (truncation) and fractional offset, kernels.cuh:90-92 */
static void base_of(double x, double hinv, int *b, double *f)
{
    *b = (int)(x * hinv - 0.5);
    *f = x * hinv - (double)(*b);
}

/* dev(F F^T) as the reference forms it (kernels.cuh:31, 591-594) */
static void dev_bbt(const double F[4], double d[4])
{
    /* b(r,c) = F(r,0)F(c,0) + F(r,1)F(c,1) */
    double b00 = F[0] * F[0] + F[1] * F[1];
    double b01 = F[0] * F[2] + F[1] * F[3];
    double b10 = F[2] * F[0] + F[3] * F[1];
    double b11 = F[2] * F[2] + F[3] * F[3];
    double h = (b00 + b11) / 2;
    d[0] = b00 - h * 1.0;
    d[1] = b01 - h * 0.0;
    d[2] = b10 - h * 0.0;
    d[3] = b11 - h * 1.0;
}

static double det2(const double F[4]) { return F[0] * F[3] - F[2] * F[1]; }

void oracle_kirchhoff(const icy_sim_params *p, const double F[4], double tau[4])
{
    /* kernels.cuh:30-33 */
    double Je = det2(F);
    double d[4];
    dev_bbt(F, d);
    double s1 = p->mu * (1.0 / Je);
    double s2 = (p->kappa * 0.5) * (Je * Je - 1.0);
    tau[0] = s1 * d[0] + s2 * 1.0;
    tau[1] = s1 * d[1] + s2 * 0.0;
    tau[2] = s1 * d[2] + s2 * 0.0;
    tau[3] = s1 * d[3] + s2 * 1.0;
}

static void water(const icy_sim_params *p, double J, double tau[4])
{
    /* kernels.cuh:37-44 */
    double s = p->kappa * (1. - pow(J, -5.0));
    tau[0] = s * 1.0; tau[1] = s * 0.0; tau[2] = s * 0.0; tau[3] = s * 1.0;
}

void oracle_pq(const icy_sim_params *p, const double F[4], double *ptr, double *qtr, double *Je)
{
    /* kernels.cuh:547-557; norm() sums squares in column-major order */
    double J = det2(F);
    *Je = J;
    *ptr = (-(p->kappa / 2.)) * (J * J - 1.);
    double d[4];
    dev_bbt(F, d);
    double sq = ((d[0] * d[0] + d[2] * d[2]) + d[1] * d[1]) + d[3] * d[3];
    *qtr = ((COEFF1 * p->mu) * (1. / J)) * sqrt(sq);
}

void oracle_svd(const double F[4], double U[4], double sigma[2], double V[4])
{
    /* column-major copy of F, helper_math.cuh:88 */
    double a[4] = {F[0], F[2], F[1], F[3]};
    /* polar decomposition, helper_math.cuh:27-46 */
    double x0 = a[0] + a[3], x1 = a[1] - a[2];
    double den = sqrt(x0 * x0 + x1 * x1);
    double uc = 1, us = 0;
    if (den != 0) { uc = x0 / den; us = -x1 / den; }
    double s[4];
    for (int d = 0; d < 2; d++) {          /* givens.cuh:120-128 */
        double t1 = a[0 + 2 * d], t2 = a[1 + 2 * d];
        s[0 + 2 * d] = uc * t1 - us * t2;
        s[1 + 2 * d] = us * t1 + uc * t2;
    }
    /* symmetric 2x2 eigen-solve, helper_math.cuh:90-126 */
    double x = s[0], y = s[2], z = s[3];
    double y2 = y * y, cosine, sine, s0, s1;
    if (y2 == 0) {
        cosine = 1; sine = 0; s0 = x; s1 = z;
    } else {
        double tau = 0.5 * (x - z);
        double w = sqrt(tau * tau + y2);
        double t = (tau > 0) ? y / (tau + w) : y / (tau - w);
        cosine = 1.0 / sqrt(t * t + 1.0);
        sine = -t * cosine;
        double c2 = cosine * cosine, csy = 2 * cosine * sine * y, s2 = sine * sine;
        s0 = c2 * x - csy + s2 * z;
        s1 = s2 * x + csy + c2 * z;
    }
    double vc, vs;
    if (s0 < s1) { double tmp = s0; s0 = s1; s1 = tmp; vc = -sine; vs = cosine; }
    else { vc = cosine; vs = sine; }
    /* u *= v, givens.cuh:161-166 */
    double nc = uc * vc - us * vs, ns = us * vc + uc * vs;
    uc = nc; us = ns;
    /* fill<2> then row-wise comma init, kernels.cuh:521-538, givens.cuh:99-111 */
    U[0] = uc; U[1] = us; U[2] = -us; U[3] = uc;
    V[0] = vc; V[1] = vs; V[2] = -vs; V[3] = vc;
    sigma[0] = s0; sigma[1] = s1;
}

int oracle_failure(const icy_sim_params *p, int grain, double ptr, double qtr)
{
    /* GetParametersForGrain, kernels.cuh:560-576 */
    double var2 = 1.0 + p->GrainVariability * 0.033 * (double)(-15 + (grain + 3) % 30);
    double var3 = 1.0 + p->GrainVariability * 0.1 * (double)(-10 + (grain + 4) % 11);
    double pmax = p->IceCompressiveStrength;
    double pmin = -p->IceTensileStrength;
    double qmax = p->IceShearStrength * var3;
    double pmin2 = -p->IceTensileStrength2 * var2;
    double beta = p->NACC_beta;
    double mSq = (4 * qmax * qmax * (1 + 2 * beta)) / ((pmax - pmin) * (pmax - pmin));
    /* CheckIfPointIsInsideFailureSurface, kernels.cuh:598-619 */
    if (ptr < 0) {
        if (ptr < pmin2) return 1;
        double q0 = 2 * sqrt(-pmax * pmin) * qmax / (pmax - pmin);
        double k = -q0 / pmin2;
        double q_limit = k * (ptr - pmin2);
        if (qtr > q_limit) return 1;
    } else {
        double yv = (1. + 2. * beta) * qtr * qtr + mSq * (ptr + beta * pmax) * (ptr - pmax);
        if (yv > 0) return 1;
    }
    return 0;
}

/* Fe = U diag(s) V^T, evaluated as (U*D)*V^T (kernels.cuh:642,671) */
static void usv(const double U[4], const double s[2], const double V[4], double F[4])
{
    double ud00 = U[0] * s[0], ud01 = U[1] * s[1], ud10 = U[2] * s[0], ud11 = U[3] * s[1];
    /* (V^T)(k,c) = V(c,k) */
    F[0] = ud00 * V[0] + ud01 * V[1];
    F[1] = ud00 * V[2] + ud01 * V[3];
    F[2] = ud10 * V[0] + ud11 * V[1];
    F[3] = ud10 * V[2] + ud11 * V[3];
}

void oracle_return_map(const icy_sim_params *p, double F[4], double *Jp,
                       double ptr, double qtr, double Je)
{
    /* ComputeSVD, kernels.cuh:540-545 */
    double U[4], V[4], sg[2];
    oracle_svd(F, U, sg, V);
    double sq0 = sg[0] * sg[0], sq1 = sg[1] * sg[1];
    double hs = (sq0 + sq1) / 2;
    double f = p->mu / Je;
    double vsh0 = f * (sq0 - hs * 1.), vsh1 = f * (sq1 - hs * 1.);
    /* Wolper_Drucker_Prager, kernels.cuh:623-674 */
    double kappa = p->kappa, mu = p->mu;
    double pmax = p->IceCompressiveStrength, qmax = p->IceShearStrength;
    if (ptr < -p->DP_threshold_p || *Jp < 1) {
        double p_new = -p->DP_threshold_p;
        double Je_new = sqrt(-2. * p_new / kappa + 1.);
        double sj = sqrt(Je_new);
        double sn[2] = {sj, sj};
        usv(U, sn, V, F);
        *Jp = *Jp * (Je_new / Je);
    } else {
        double q_n_1;
        if (ptr > pmax) {
            q_n_1 = 0;
        } else {
            double q_from_dp = (ptr + p->DP_threshold_p) * p->DP_tan_phi;
            double pmin = -p->IceTensileStrength;
            double q_from_fs = 2 * sqrt((pmax - ptr) * (ptr - pmin)) * qmax / (pmax - pmin);
            q_n_1 = fmin(q_from_fs, q_from_dp);
        }
        if (qtr >= q_n_1) {
            double snorm = q_n_1 * COEFF1_INV;
            double z = vsh0 * vsh0 + vsh1 * vsh1;
            double n0 = vsh0, n1 = vsh1;
            if (z > 0) { double r = sqrt(z); n0 = vsh0 / r; n1 = vsh1 / r; }
            double k = snorm * (Je / mu);
            double tr = 1. * ((sq0 + sq1) / 2.);
            double sn[2] = {sqrt(k * n0 + tr), sqrt(k * n1 + tr)};
            usv(U, sn, V, F);
        }
    }
}

/* stencil base check, kernels.cuh:94-97 (gridX_offset = 0) */
static int base_error(const icy_sim_params *p, int bx, int by)
{
    int e = 0, halo = p->GridHaloSize;
    if (bx < -halo) e = ICY_ERR_OUT_OF_GRID_XLO;
    if (by < 0) e = ICY_ERR_OUT_OF_GRID_YLO;
    if (bx > p->GridXTotal + halo - 3) e = ICY_ERR_OUT_OF_GRID_XHI;
    if (by > p->GridY - 3) e = ICY_ERR_OUT_OF_GRID_YHI;
    return e;
}

int oracle_p2g(const icy_sim_params *p, const double *soa, unsigned pitch, unsigned n,
               double *gm, double *gpx, double *gpy)
{
    const double h = p->cellsize, hinv = p->cellsize_inv;
    const int gy = p->GridY, off = p->GridY * p->GridHaloSize;
    int err = 0;
    for (unsigned i = 0; i < n; i++) {
        long long util = as_ll(soa[i]);
        if (util & ICY_STATUS_DISABLED) continue;
        int liquid = (int)((util & ICY_STATUS_LIQUID) >> 18);
        double mass = liquid ? p->WaterParticleMass : p->ParticleMass;
        double x = soa[i + (size_t)pitch * ICY_POSX], y = soa[i + (size_t)pitch * (ICY_POSX + 1)];
        double vx = soa[i + (size_t)pitch * ICY_VELX], vy = soa[i + (size_t)pitch * (ICY_VELX + 1)];
        double F[4], B[4], P[4];
        for (int k = 0; k < 4; k++) {
            F[k] = soa[i + (size_t)pitch * (ICY_FE00 + k)];
            B[k] = soa[i + (size_t)pitch * (ICY_BP00 + k)];
        }
        if (liquid) water(p, soa[i + (size_t)pitch * ICY_IDX_JP_INV], P);
        else oracle_kirchhoff(p, F, P);
        double S[4];                                    /* kernels.cuh:88 */
        for (int k = 0; k < 4; k++) S[k] = mass * B[k] - p->dt_vol_Dpinv * P[k];
        int bx, by;
        double fx, fy;
        base_of(x, hinv, &bx, &fx);
        base_of(y, hinv, &by, &fy);
        int e = base_error(p, bx, by);
        if (e) { err = e; continue; }
        double wx[3], wy[3];
        weights(fx, wx);
        weights(fy, wy);
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {                /* kernels.cuh:105-121 */
                double W = wx[a] * wy[b];
                double d0 = ((double)a - fx) * h, d1 = ((double)b - fy) * h;
                double iv0 = W * (vx * mass + (S[0] * d0 + S[1] * d1));
                double iv1 = W * (vy * mass + (S[2] * d0 + S[3] * d1));
                double im = W * mass;
                long idx = (long)(by + b) + (long)(bx + a) * gy + off;
                gm[idx] += im;
                gpx[idx] += iv0;
                gpy[idx] += iv1;
            }
    }
    return err;
}

void oracle_update(const icy_sim_params *p, double *gm, double *gpx, double *gpy,
                   double ind_x, double ind_y, double *bins)
{
    const int gy = p->GridY, halo = p->GridHaloSize, nsub = p->n_indenter_subdivisions;
    const long nn = oracle_grid_nodes(p);
    const double dt = p->InitialTimeStep, vco = p->IndVelocity;
    for (long idx = 0; idx < nn; idx++) {
        double mass = gm[idx];
        double vx = gpx[idx], vy = gpy[idx];
        if (mass == 0) continue;                          /* kernels.cuh:178 */
        int gix = (int)(idx / gy) - halo, giy = (int)(idx % gy);
        double gnx = (double)gix * p->cellsize, gny = (double)giy * p->cellsize;
        vx = vx / mass; vy = vy / mass;                   /* :194-196 */
        vy = vy - p->dt_Gravity;
        if (vx * vx + vy * vy > p->vmax_squared) {        /* :261 */
            double r = sqrt(vx * vx + vy * vy);
            vx = (vx / r) * p->vmax; vy = (vy / r) * p->vmax;
        }
        double nx = gnx - ind_x, ny = gny - ind_y;        /* :264-287 */
        if (nx * nx + ny * ny < p->IndRSq) {
            double vrx = vx - vco, vry = vy - 0.0;
            double z = nx * nx + ny * ny;
            if (z > 0) { double r = sqrt(z); nx = nx / r; ny = ny / r; }
            double vn = vrx * nx + vry * ny;
            if (vn < 0) {
                double vtx = vrx - nx * vn, vty = vry - ny * vn;
                double pvx = vx, pvy = vy;
                vx = vco + vtx; vy = 0.0 + vty;
                double fx = (pvx - vx) * mass / dt, fy = (pvy - vy) * mass / dt;
                float angle = atan2f((float)nx, (float)ny);
                angle += PI;
                angle *= nsub / (2 * PI);
                int index = (int)angle;
                if (index < 0) index = 0;
                if (index > nsub - 1) index = nsub - 1;
                if (bins) { bins[2 * index] += fx; bins[2 * index + 1] += fy; }
            }
        }
        if (giy <= 2) { vx = 0; vy = 0; }                 /* :290-294 */
        if (giy >= gy - 3 && vy > 0) vy = 0;
        if (gix <= 2 && vx < 0) vx = 0;
        else if (gix >= p->GridXTotal - 3 && vx > 0) vx = 0;
        gpx[idx] = vx;
        gpy[idx] = vy;
    }
}

int oracle_g2p(const icy_sim_params *p, double *soa, unsigned pitch, unsigned n,
               const double *gvx, const double *gvy, int recordPQ)
{
    const double hinv = p->cellsize_inv, dt = p->InitialTimeStep;
    const int gy = p->GridY, off = p->GridY * p->GridHaloSize;
    int err = 0;
    for (unsigned i = 0; i < n; i++) {
        double *L[16];
        for (int k = 0; k < 16; k++) L[k] = soa + (size_t)pitch * k + i;
        long long util = as_ll(*L[0]);
        if (util & ICY_STATUS_DISABLED) continue;         /* kernels.cuh:320 */
        int liquid = (util & ICY_STATUS_LIQUID) != 0;
        double x = *L[ICY_POSX], y = *L[ICY_POSX + 1];
        double F[4] = {*L[ICY_FE00], *L[ICY_FE00 + 1], *L[ICY_FE00 + 2], *L[ICY_FE00 + 3]};
        double Jp = *L[ICY_IDX_JP_INV];
        int grain = (short)util;
        int bx, by;
        double fx, fy;
        base_of(x, hinv, &bx, &fx);
        base_of(y, hinv, &by, &fy);
        int e = base_error(p, bx, by);
        if (e) { err = e; continue; }
        double wx[3], wy[3];
        weights(fx, wx);
        weights(fy, wy);
        double vx = 0, vy = 0, B[4] = {0, 0, 0, 0};
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {                 /* :357-372 */
                double d0 = (double)a - fx, d1 = (double)b - fy;
                double w = wx[a] * wy[b];
                long idx = (long)(by + b) + (long)(bx + a) * gy + off;
                double nvx = gvx[idx], nvy = gvy[idx];
                vx = vx + w * nvx;
                vy = vy + w * nvy;
                double s = (4. * hinv) * w;
                double snx = s * nvx, sny = s * nvy;
                B[0] = B[0] + snx * d0; B[1] = B[1] + snx * d1;
                B[2] = B[2] + sny * d0; B[3] = B[3] + sny * d1;
            }
        x = x + vx * dt;                                   /* :375-376 */
        y = y + vy * dt;
        double A[4] = {1.0 + dt * B[0], 0.0 + dt * B[1], 0.0 + dt * B[2], 1.0 + dt * B[3]};
        double Fn[4] = {A[0] * F[0] + A[1] * F[2], A[0] * F[1] + A[1] * F[3],
                        A[2] * F[0] + A[3] * F[2], A[2] * F[1] + A[3] * F[3]};
        double ptr = 0, qtr = 0;
        if (liquid) {
            Jp = Jp * (A[0] * A[3] - A[2] * A[1]);        /* :380 */
        } else {
            double Je;
            oracle_pq(p, Fn, &ptr, &qtr, &Je);            /* :384-390 */
            if (!(util & ICY_STATUS_CRUSHED))
                if (oracle_failure(p, grain, ptr, qtr)) util |= ICY_STATUS_CRUSHED;
            if (util & ICY_STATUS_CRUSHED) oracle_return_map(p, Fn, &Jp, ptr, qtr, Je);
        }
        *L[ICY_POSX] = x; *L[ICY_POSX + 1] = y;             /* :395-407 */
        *L[ICY_VELX] = vx; *L[ICY_VELX + 1] = vy;
        for (int k = 0; k < 4; k++) { *L[ICY_FE00 + k] = Fn[k]; *L[ICY_BP00 + k] = B[k]; }
        *L[ICY_IDX_JP_INV] = Jp;
        *L[0] = as_d(util);
        if (recordPQ) { *L[ICY_IDX_P] = ptr; *L[ICY_IDX_Q] = qtr; }   /* :410-414 */
    }
    return err;
}

#include <stdlib.h>

int oracle_run(const icy_sim_params *p, double *soa, unsigned pitch, unsigned n,
               int step0, int nsteps, double *sim_time, double *bins)
{
    long nn = oracle_grid_nodes(p);
    double *g = (double *)malloc(sizeof(double) * 3 * nn);
    if (!g) return ICY_ERR_OUT_OF_MEMORY;
    double t = *sim_time;
    int err = 0;
    for (int k = 0; k < nsteps && !err; k++) {
        t += p->InitialTimeStep;                           /* model.cpp:40-41 */
        double ind_x = p->indenter_x_initial + t * p->IndVelocity;
        memset(g, 0, sizeof(double) * 3 * nn);
        err = oracle_p2g(p, soa, pitch, n, g, g + nn, g + 2 * nn);
        if (err) break;
        oracle_update(p, g, g + nn, g + 2 * nn, ind_x, p->indenter_y, bins);
        int rec = ((step0 + k) % p->UpdateEveryNthStep) == 0;   /* model.cpp:47 */
        err = oracle_g2p(p, soa, pitch, n, g + nn, g + 2 * nn, rec);
    }
    *sim_time = t;
    free(g);
    return err;
}
