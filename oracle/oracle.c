/*
 * oracle.c -- FP64 CPU restatement of sma-dft's time-step loop (TEST INFRASTRUCTURE ONLY).
 * See oracle.h.  Every block cites the reference lines it restates; the operation order
 * follows the reference so that FP64 results agree to rounding.
 */
#include "oracle.h"
#include "r2r.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define T10 ORC_REDFT10
#define T01 ORC_REDFT01
#define S10 ORC_RODFT10
#define S01 ORC_RODFT01

struct orc_ctx {
    orc_params p;
    int nx, ny, nz;
    long n;
    double Lx, Ly, Lz, dx, dy, dz, scale;
    double rho_m, lambda;
    /* DCT wavenumbers q_i = pi i / L and DST wavenumbers s_i = pi (i+1) / L */
    double *qx, *qy, *qz, *sx, *sy, *sz;
    double *aLin, *C1, *C2, *mq2;
    double *CM1x, *CM1y, *CM1z, *CM2x, *CM2y, *CM2z;
    double *psi, *psiq, *psiNew, *Nr, *Nq, *NqPast;
    /* advection */
    double *gx, *gy, *gz, *sp2, *Sx, *Sy, *Sz, *vx, *vy, *vz;
    /* quasi */
    double *psiq_old, *psi_old, *rho, *rhoq, *rho_old, *p_, *divv, *mu, *energy, *dfd, *lap;
    double *rdx, *rdy, *rdz;
    /* compressible */
    double *amp, *fgrad, *ampd, *frho, *virx, *viry, *virz, *fxs, *fys, *fzs;
    double amp_c, kp_c;         /* compressible/compressible.cpp:265-267 */
    /* surface diagnostics of one step (orc_step_surface) */
    int surf_pending;
    double *dTpsi, *psiDxx, *psiDyy, *psiDzz, *fgx, *fgy, *fgz;
    int *s_idx;
    double *s_vel, *s_H, *s_K;
    long nloop;
    double L1, mass, en;
    int have_psi;
};

#define IDX(c, i, j, k) (((long)(i) * (c)->ny + (j)) * (c)->nz + (k))

static double *dal(long n) { return (double *)calloc((size_t)n, sizeof(double)); }

void orc_r2r_3d_kinds(const double *in, double *out, int nx, int ny, int nz, int kx, int ky, int kz)
{
    orc_r2r_3d(in, out, nx, ny, nz, kx, ky, kz);
}

static void r3(orc_ctx *c, const double *in, double *out, int kx, int ky, int kz)
{
    orc_r2r_3d(in, out, c->nx, c->ny, c->nz, kx, ky, kz);
}

orc_ctx *orc_create(const orc_params *p)
{
    if (p->nx < 2 || p->ny < 2 || p->nz < 2) return NULL;
    if (p->conserved && (p->model == ORC_QUASI || p->model == ORC_COMP)) return NULL;   /* none in the reference */
    orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx));
    c->p = *p;
    c->nx = p->nx; c->ny = p->ny; c->nz = p->nz;
    c->n = (long)c->nx * c->ny * c->nz;
    /* box and grid: no-adv/cosNoAdvTrackSing.cpp:160-172 */
    c->Lx = c->nx * 2.0 * M_PI / (p->q0 * p->nw);
    c->Ly = c->ny * 2.0 * M_PI / (p->q0 * p->nw);
    c->Lz = c->nz * 2.0 * M_PI / (p->q0 * p->nw);
    c->dx = c->Lx / c->nx; c->dy = c->Ly / c->ny; c->dz = c->Lz / c->nz;
    c->scale = 0.125 / ((double)c->nx * c->ny * c->nz);
    /* quasi constants: quasi/quasi.cpp:237-246 */
    double rho_s = p->kp * p->amp + p->rho0;
    c->rho_m = rho_s / 2;
    c->lambda = -2 * p->nu / 3;
    if (p->model == ORC_COMP) {
        /* compressible/compressible.cpp:265-271: Amp of the one-mode smectic at eps, kp such
         * that rho_s = kp Amp + rho_0 = 1, rho_m = rho_s / 2, lambda = nu */
        c->amp_c = sqrt((3 * p->beta + sqrt(9 * p->beta * p->beta + 40 * p->eps * p->gamma)) / 5);
        c->kp_c = (1 - p->rho0) / c->amp_c;
        rho_s = c->kp_c * c->amp_c + p->rho0;
        c->rho_m = rho_s / 2;
        c->lambda = p->nu;
    }
    /* wavenumbers: no-adv/cosNoAdvTrackSing.cpp:309-324 (DCT), adv/cosAdvTrackMult.cpp:386-401 (DST) */
    c->qx = dal(c->nx); c->sx = dal(c->nx);
    c->qy = dal(c->ny); c->sy = dal(c->ny);
    c->qz = dal(c->nz); c->sz = dal(c->nz);
    for (int i = 0; i < c->nx; i++) { c->qx[i] = 1.0 * M_PI * i / (c->dx * c->nx); c->sx[i] = 1.0 * M_PI * (i + 1) / (c->dx * c->nx); }
    for (int j = 0; j < c->ny; j++) { c->qy[j] = M_PI * (j) / (c->dy * c->ny); c->sy[j] = M_PI * (j + 1) / (c->dy * c->ny); }
    for (int k = 0; k < c->nz; k++) { c->qz[k] = M_PI * (k) / (c->dz * c->nz); c->sz[k] = M_PI * (k + 1) / (c->dz * c->nz); }
    long n = c->n;
    c->aLin = dal(n); c->C1 = dal(n); c->C2 = dal(n); c->mq2 = dal(n);
    c->psi = dal(n); c->psiq = dal(n); c->psiNew = dal(n); c->Nr = dal(n); c->Nq = dal(n); c->NqPast = dal(n);
    if (p->model != ORC_NOADV) {
        c->CM1x = dal(n); c->CM1y = dal(n); c->CM1z = dal(n);
        c->CM2x = dal(n); c->CM2y = dal(n); c->CM2z = dal(n);
        c->gx = dal(n); c->gy = dal(n); c->gz = dal(n); c->sp2 = dal(n);
        c->Sx = dal(n); c->Sy = dal(n); c->Sz = dal(n);
        c->vx = dal(n); c->vy = dal(n); c->vz = dal(n);
    }
    if (p->model == ORC_COMP) {
        c->amp = dal(n); c->fgrad = dal(n); c->ampd = dal(n); c->frho = dal(n);
        c->virx = dal(n); c->viry = dal(n); c->virz = dal(n);
        c->fxs = dal(n); c->fys = dal(n); c->fzs = dal(n);
    }
    if (p->model == ORC_QUASI || p->model == ORC_COMP) {
        c->psiq_old = dal(n); c->psi_old = dal(n); c->rho = dal(n); c->rhoq = dal(n);
        c->rho_old = dal(n); c->p_ = dal(n); c->divv = dal(n); c->mu = dal(n); c->energy = dal(n);
        c->dfd = dal(n); c->lap = dal(n); c->rdx = dal(n); c->rdy = dal(n); c->rdz = dal(n);
    }
    /* linear operator and Stokes coefficients:
     * noadv  no-adv/cosNoAdvTrackSing.cpp:594-602
     * adv    adv/cosAdvTrackMult.cpp:729-751
     * quasi  quasi/quasi.cpp:963-985 (C1 = 2 - dt rho_m L, C2 = 1.5 - dt rho_m L) */
    const double dtd2 = p->dt / 2;
    for (int i = 0; i < c->nx; i++)
        for (int j = 0; j < c->ny; j++)
            for (int k = 0; k < c->nz; k++) {
                long idx = IDX(c, i, j, k);
                double mq2 = pow(c->qx[i], 2) + pow(c->qy[j], 2) + pow(c->qz[k], 2);
                c->mq2[idx] = mq2;
                double q02 = p->q0 * p->q0;
                if (p->model == ORC_QUASI || p->model == ORC_COMP) {
                    double opSH = p->alpha * pow(q02 - mq2, 2);
                    c->aLin[idx] = p->eps - opSH;
                    c->C1[idx] = (2.0 - p->dt * c->rho_m * c->aLin[idx]);
                    c->C2[idx] = (1.5 - p->dt * c->rho_m * c->aLin[idx]);
                } else if (p->conserved && p->model == ORC_NOADV) {
                    /* q^2-weighted operator in aLin itself: no-adv/cosNoAdvConserv.cpp:646-650 */
                    double opSH = p->alpha * pow(mq2 - q02, 2);
                    c->aLin[idx] = mq2 * (p->eps - opSH);
                    c->C1[idx] = (1.0 + dtd2 * c->aLin[idx]);
                    c->C2[idx] = (1.0 - dtd2 * c->aLin[idx]);
                } else if (p->conserved) {
                    /* aLin stays L (it also builds Sp2); only C1, C2 carry q^2:
                     * adv/cosAdvConSingle.cpp:738-742 */
                    double opSH = p->alpha * pow(mq2 - q02, 2);
                    c->aLin[idx] = p->eps - opSH;
                    c->C1[idx] = (1.0 + dtd2 * mq2 * c->aLin[idx]);
                    c->C2[idx] = (1.0 - dtd2 * mq2 * c->aLin[idx]);
                } else {
                    double opSH = p->alpha * pow(mq2 - q02, 2);
                    c->aLin[idx] = p->eps - opSH;
                    c->C1[idx] = (1.0 + dtd2 * c->aLin[idx]);
                    c->C2[idx] = (1.0 - dtd2 * c->aLin[idx]);
                }
                if (p->model == ORC_COMP) {
                    /* compressible/compressible.cpp:1136-1145: CM1 = scale/|q_s|^2 (nu applied later) */
                    double m2 = pow(c->sx[i], 2) + pow(c->qy[j], 2) + pow(c->qz[k], 2);
                    c->CM1x[idx] = c->scale / (m2);
                    c->CM2x[idx] = c->sx[i] / m2;
                    m2 = pow(c->qx[i], 2) + pow(c->sy[j], 2) + pow(c->qz[k], 2);
                    c->CM1y[idx] = c->scale / (m2);
                    c->CM2y[idx] = c->sy[j] / m2;
                    m2 = pow(c->qx[i], 2) + pow(c->qy[j], 2) + pow(c->sz[k], 2);
                    c->CM1z[idx] = c->scale / (m2);
                    c->CM2z[idx] = c->sz[k] / m2;
                } else if (p->model != ORC_NOADV) {
                    double m2 = pow(c->sx[i], 2) + pow(c->qy[j], 2) + pow(c->qz[k], 2);
                    c->CM1x[idx] = c->scale / (p->nu * m2);
                    c->CM2x[idx] = c->sx[i] / m2;
                    m2 = pow(c->qx[i], 2) + pow(c->sy[j], 2) + pow(c->qz[k], 2);
                    c->CM1y[idx] = c->scale / (p->nu * m2);
                    c->CM2y[idx] = c->sy[j] / m2;
                    m2 = pow(c->qx[i], 2) + pow(c->qy[j], 2) + pow(c->sz[k], 2);
                    c->CM1z[idx] = c->scale / (p->nu * m2);
                    c->CM2z[idx] = c->sz[k] / m2;
                }
            }
    return c;
}

void orc_destroy(orc_ctx *c)
{
    if (!c) return;
    double **ptrs[] = {&c->qx, &c->qy, &c->qz, &c->sx, &c->sy, &c->sz, &c->aLin, &c->C1, &c->C2,
                       &c->mq2, &c->CM1x, &c->CM1y, &c->CM1z, &c->CM2x, &c->CM2y, &c->CM2z,
                       &c->psi, &c->psiq, &c->psiNew, &c->Nr, &c->Nq, &c->NqPast, &c->gx, &c->gy,
                       &c->gz, &c->sp2, &c->Sx, &c->Sy, &c->Sz, &c->vx, &c->vy, &c->vz,
                       &c->psiq_old, &c->psi_old, &c->rho, &c->rhoq, &c->rho_old, &c->p_,
                       &c->divv, &c->mu, &c->energy, &c->dfd, &c->lap, &c->rdx, &c->rdy, &c->rdz,
                       &c->amp, &c->fgrad, &c->ampd, &c->frho, &c->virx, &c->viry, &c->virz,
                       &c->fxs, &c->fys, &c->fzs};
    for (size_t q = 0; q < sizeof(ptrs) / sizeof(ptrs[0]); q++) free(*ptrs[q]);
    free(c->dTpsi); free(c->psiDxx); free(c->psiDyy); free(c->psiDzz);
    free(c->fgx); free(c->fgy); free(c->fgz);
    free(c);
}

/* N = beta psi^3 - gamma psi^5, no-adv/cosNoAdvTrackSing.cpp:713-723 */
static void nonlin(orc_ctx *c, const double *psi, double *out)
{
    const double b = c->p.beta, g = c->p.gamma;
    for (long q = 0; q < c->n; q++) out[q] = b * pow(psi[q], 3) - g * pow(psi[q], 5);
}

int orc_set_psi(orc_ctx *c, const double *psi0)
{
    long n = c->n;
    memcpy(c->psi, psi0, sizeof(double) * n);
    c->nloop = 0;
    c->L1 = c->mass = c->en = 0.0;
    if (c->p.model == ORC_COMP) {
        /* compressible/compressible.cpp:1150-1194: psiq = s CT(psi), psi = iCT(psiq), N^0
         * (unused: the first step sets Nl_old = Nl), psiq_old, psi_old; rho and its rate start
         * at zero (load != 1, :612) */
        r3(c, c->psi, c->psiq, T10, T10, T10);
        for (long q = 0; q < n; q++) c->psiq[q] = c->scale * c->psiq[q];
        r3(c, c->psiq, c->psi, T01, T01, T01);
        nonlin(c, c->psi, c->Nr);
        memcpy(c->psiq_old, c->psiq, sizeof(double) * n);
        r3(c, c->Nr, c->Nq, T10, T10, T10);
        memcpy(c->psi_old, c->psi, sizeof(double) * n);
        memset(c->rho, 0, sizeof(double) * n);
        memset(c->frho, 0, sizeof(double) * n);
    } else if (c->p.model == ORC_QUASI) {
        /* quasi/quasi.cpp:990-1034: psiq = scale CT(psi), psi = iCT(psiq), N^0, psiq_old, psi_old */
        r3(c, c->psi, c->psiq, T10, T10, T10);
        for (long q = 0; q < n; q++) c->psiq[q] = c->scale * c->psiq[q];
        r3(c, c->psiq, c->psi, T01, T01, T01);
        nonlin(c, c->psi, c->Nr);
        memcpy(c->psiq_old, c->psiq, sizeof(double) * n);
        r3(c, c->Nr, c->Nq, T10, T10, T10);
        memcpy(c->psi_old, c->psi, sizeof(double) * n);
        memset(c->divv, 0, sizeof(double) * n);
        memset(c->rhoq, 0, sizeof(double) * n);
        memset(c->rho_old, 0, sizeof(double) * n);
        memset(c->vx, 0, sizeof(double) * n);
        memset(c->vy, 0, sizeof(double) * n);
        memset(c->vz, 0, sizeof(double) * n);
    } else {
        /* pre-loop N^0 (no advection term): no-adv/cosNoAdvTrackSing.cpp:618-635,
         * adv/cosAdvTrackMult.cpp:760-777.  The wall potential has sigma = 0 (:75-82). */
        nonlin(c, c->psi, c->Nr);
        r3(c, c->Nr, c->Nq, T10, T10, T10);
        /* conserved noadv weights the pre-loop N by q^2 (no-adv/cosNoAdvConserv.cpp:688-701);
         * conserved adv keeps it unweighted (adv/cosAdvConSingle.cpp:762-780) */
        if (c->p.conserved && c->p.model == ORC_NOADV)
            for (long q = 0; q < n; q++) c->Nq[q] = c->mq2[q] * c->Nq[q];
        if (c->p.model == ORC_NOADV) {
            /* psiq is recomputed every step; keep the scaled transform for orc_get */
            r3(c, c->psi, c->psiq, T10, T10, T10);
            for (long q = 0; q < n; q++) c->psiq[q] *= c->scale;
        } else {
            r3(c, c->psi, c->psiq, T10, T10, T10);
            for (long q = 0; q < n; q++) c->psiq[q] *= c->scale;
        }
    }
    c->have_psi = 1;
    return 0;
}

/* L1 = sum|new - old| / (dt sum|new|): no-adv/cosNoAdvTrackSing.cpp:775-789 */
static double l1_measure(const orc_ctx *c, const double *newv, const double *oldv)
{
    double a = 0.0, b = 0.0;
    for (long q = 0; q < c->n; q++) {
        a = a + fabs(newv[q] - oldv[q]);
        b = b + fabs(newv[q]);
    }
    return a / (c->p.dt * b);
}

/* Spectral second derivatives and the time derivative of psi for the surface diagnostics,
 * from the spectrum psiq (times `sc`) and the nonlinear spectrum Nq of the same step:
 *   dTpsi = iCT(sc (L psiq) + sN Nq), psiDaa = iCT(-sc q_a^2 psiq)
 * noadv (psiq unscaled, sc = sN = scale): no-adv/cosNoAdvTrackSing.cpp:737-750,760-764;
 * adv (psiq scaled, sc = 1, sN = scale): adv/cosAdvTrackMult.cpp:1311-1347. */
static void surface_spectra(orc_ctx *c, double sc, double sN)
{
    const long n = c->n;
    if (!c->dTpsi) {
        c->dTpsi = dal(n); c->psiDxx = dal(n); c->psiDyy = dal(n); c->psiDzz = dal(n);
    }
    for (int i = 0; i < c->nx; i++)
        for (int j = 0; j < c->ny; j++)
            for (int k = 0; k < c->nz; k++) {
                long q = IDX(c, i, j, k);
                c->dTpsi[q] = sc == 1.0 ? (c->aLin[q] * c->psiq[q] + sN * c->Nq[q])
                                        : sc * (c->aLin[q] * c->psiq[q] + c->Nq[q]);
                c->psiDxx[q] = -sc * c->qx[i] * c->qx[i] * c->psiq[q];
                c->psiDyy[q] = -sc * c->qy[j] * c->qy[j] * c->psiq[q];
                c->psiDzz[q] = -sc * c->qz[k] * c->qz[k] * c->psiq[q];
            }
    r3(c, c->dTpsi, c->dTpsi, T01, T01, T01);
    r3(c, c->psiDxx, c->psiDxx, T01, T01, T01);
    r3(c, c->psiDyy, c->psiDyy, T01, T01, T01);
    r3(c, c->psiDzz, c->psiDzz, T01, T01, T01);
}

/* Finite-difference gradient of psi, centred inside and one-sided (2 (a - b) / 2dx) at the
 * walls: no-adv/cosNoAdvTrackSing.cpp:819-878. */
static void fd_gradient(orc_ctx *c, const double *psi)
{
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    const double tdx = 2 * c->dx, tdy = 2 * c->dy, tdz = 2 * c->dz;
    if (!c->fgx) { c->fgx = dal(c->n); c->fgy = dal(c->n); c->fgz = dal(c->n); }
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                long q = IDX(c, i, j, k);
                if (i > 0 && i < nx - 1) c->fgx[q] = (psi[IDX(c, i + 1, j, k)] - psi[IDX(c, i - 1, j, k)]) / tdx;
                else if (i == 0) c->fgx[q] = 2 * (psi[IDX(c, 1, j, k)] - psi[q]) / tdx;
                else c->fgx[q] = 2 * (psi[q] - psi[IDX(c, i - 1, j, k)]) / tdx;
                if (j != 0 && j != ny - 1) c->fgy[q] = (psi[IDX(c, i, j + 1, k)] - psi[IDX(c, i, j - 1, k)]) / tdy;
                else if (j == 0) c->fgy[q] = 2 * (psi[IDX(c, i, j + 1, k)] - psi[q]) / tdy;
                else c->fgy[q] = 2 * (psi[q] - psi[IDX(c, i, j - 1, k)]) / tdy;
                if (k != 0 && k != nz - 1) c->fgz[q] = (psi[q + 1] - psi[q - 1]) / tdz;
                else if (k == 0) c->fgz[q] = 2 * (psi[q + 1] - psi[q]) / tdz;
                else c->fgz[q] = 2 * (psi[q] - psi[q - 1]) / tdz;
            }
}

/* Interface per (i, j) column, scanning z downward (first psi > 0.7, then first psi < 0,
 * the nearer of k, k+1), with the normal velocity dTpsi/|grad psi| and the curvatures 2H, K
 * (Megrabov's divergence forms) there: no-adv/cosNoAdvTrackSing.cpp:880-964,
 * adv/cosAdvTrackMult.cpp:1417-1515.  Mixed derivatives are differences of the gradient
 * fields: along y at the chosen index k2, along z around that index with the branch taken
 * on k (as the reference does).  An element past the end of the array reads 0. */
static void surface_eval(orc_ctx *c, const double *psi, const double *gx, const double *gy, const double *gz)
{
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    const double tdy = 2 * c->dy, tdz = 2 * c->dz;
    const long n = c->n;
#define GAT(f, q) ((q) < n ? (f)[q] : 0.0)
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            const long col = (long)i * ny + j;
            c->s_idx[col] = -1;
            c->s_vel[col] = c->s_H[col] = c->s_K[col] = NAN;
            int track = 0;
            for (int k = nz - 1; k > -1; k--) {
                long index = IDX(c, i, j, k);
                if (psi[index] > 0.7 && track == 0) track = 1;
                if (psi[index] < 0.0 && track == 1) {
                    int k2 = k;
                    if (fabs(psi[index]) > fabs(psi[index + 1])) { index = index + 1; k2 = k + 1; }
                    c->s_idx[col] = k2;
                    const double gxv = gx[index], gyv = gy[index], gzv = gz[index];
                    const double gradVal = sqrt(gxv * gxv + gyv * gyv + gzv * gzv);
                    c->s_vel[col] = c->dTpsi[index] / gradVal;
                    double Dxy = 0, Dxz = 0, Dyz = 0;
                    if (j > 0 && j < ny - 1) Dxy = (gx[IDX(c, i, j + 1, k2)] - gx[IDX(c, i, j - 1, k2)]) / tdy;
                    if (j == 0) Dxy = 2 * (gx[IDX(c, i, 1, k2)] - gx[IDX(c, i, 0, k2)]) / tdy;
                    if (j == ny - 1) Dxy = 2 * (gx[IDX(c, i, j, k2)] - gx[IDX(c, i, j - 1, k2)]) / tdy;
                    if (k > 0 && k < nz - 1) {
                        Dxz = (GAT(gx, index + 1) - gx[index - 1]) / tdz;
                        Dyz = (GAT(gy, index + 1) - gy[index - 1]) / tdz;
                    }
                    if (k == 0) {
                        Dxz = 2 * (GAT(gx, index + 1) - gx[index]) / tdz;
                        Dyz = 2 * (GAT(gy, index + 1) - gy[index]) / tdz;
                    }
                    const double Dxx = c->psiDxx[index], Dyy = c->psiDyy[index], Dzz = c->psiDzz[index];
                    c->s_H[col] = ((gyv * gyv + gzv * gzv) * Dxx + (gxv * gxv + gzv * gzv) * Dyy +
                                   (gxv * gxv + gyv * gyv) * Dzz -
                                   2 * (gxv * gyv * Dxy + gxv * gzv * Dxz + gyv * gzv * Dyz)) /
                                  pow(gradVal, 3);
                    c->s_K[col] = (gzv * gzv * (Dxx * Dyy - Dxy * Dxy) + gxv * gxv * (Dyy * Dzz - Dyz * Dyz) +
                                   gyv * gyv * (Dxx * Dzz - Dxz * Dxz) +
                                   2 * (gyv * Dxy * (gzv * Dxz - gxv * Dzz) + gxv * Dxz * (gyv * Dyz - gzv * Dyy) +
                                        gzv * Dyz * (gxv * Dxy - gyv * Dxx))) /
                                  pow(gradVal, 4);
                    track = 2;
                }
            }
        }
#undef GAT
}

/* ---------------- noadv: no-adv/cosNoAdvTrackSing.cpp:681-764,1072 ---------------- */
static void step_noadv(orc_ctx *c)
{
    const long n = c->n;
    const double dtd2 = c->p.dt / 2;
    memcpy(c->NqPast, c->Nq, sizeof(double) * n);                 /* :688 */
    nonlin(c, c->psi, c->Nr);                                      /* :713-723 */
    r3(c, c->Nr, c->Nq, T10, T10, T10);                            /* :727 */
    r3(c, c->psi, c->psiq, T10, T10, T10);                         /* :731 */
    if (c->surf_pending) surface_spectra(c, c->scale, c->scale);   /* :737-750 */
    if (c->p.conserved)                                            /* cosNoAdvConserv.cpp:809 */
        for (long q = 0; q < n; q++) c->Nq[q] = c->mq2[q] * c->Nq[q];
    for (long q = 0; q < n; q++)                                   /* :752-753 */
        c->psiq[q] = c->scale * (c->C1[q] * c->psiq[q] + dtd2 * (3.0 * c->Nq[q] - c->NqPast[q])) / c->C2[q];
    r3(c, c->psiq, c->psiNew, T01, T01, T01);                      /* :758 */
    c->L1 = l1_measure(c, c->psiNew, c->psi);                      /* :769-789 */
    if (c->surf_pending) {                                         /* :808-964, on psi^n */
        fd_gradient(c, c->psi);
        surface_eval(c, c->psi, c->fgx, c->fgy, c->fgz);
    }
    memcpy(c->psi, c->psiNew, sizeof(double) * n);                 /* :1072 */
}

/* Stokes velocity from the force spectra (adv/cosAdvTrackMult.cpp:1103-1274 on one rank;
 * quasi adds the irrotational part, quasi/quasi.cpp:1704-2109).  Truncations: v_x at
 * i = nx-1 is 0; v_y, v_z at j = ny-1 or k = nz-1 are 0; the shifted neighbours at
 * index -1 are 0 (the single-rank halo planes stay zero-filled, adv :1157, quasi :1841). */
static void stokes(orc_ctx *c, int with_divv)
{
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    const double nu = c->p.nu;
    memset(c->vx, 0, sizeof(double) * c->n);
    memset(c->vy, 0, sizeof(double) * c->n);
    memset(c->vz, 0, sizeof(double) * c->n);
    for (int i = 0; i < nx - 1; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                long idx = IDX(c, i, j, k);
                double Sy = (j != 0) ? c->Sy[IDX(c, i + 1, j - 1, k)] : 0.0;
                double Sz = (k != 0) ? c->Sz[IDX(c, i + 1, j, k - 1)] : 0.0;
                double dot = c->sx[i] * c->Sx[idx] + c->qy[j] * Sy + c->qz[k] * Sz;
                double v = c->CM1x[idx] * (c->Sx[idx] - c->CM2x[idx] * dot);
                if (with_divv) v = v + c->CM1x[idx] * (nu * c->sx[i] * c->divv[IDX(c, i + 1, j, k)]);
                c->vx[idx] = v;
            }
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny - 1; j++)
            for (int k = 0; k < nz - 1; k++) {
                long idx = IDX(c, i, j, k);
                double Sx = (i != 0) ? c->Sx[IDX(c, i - 1, j + 1, k)] : 0.0;
                double Sz = (k != 0) ? c->Sz[IDX(c, i, j + 1, k - 1)] : 0.0;
                double dot = c->qx[i] * Sx + c->sy[j] * c->Sy[idx] + c->qz[k] * Sz;
                double v = c->CM1y[idx] * (c->Sy[idx] - c->CM2y[idx] * dot);
                if (with_divv) v = v + c->CM1y[idx] * (nu * c->sy[j] * c->divv[IDX(c, i, j + 1, k)]);
                c->vy[idx] = v;

                Sx = (i != 0) ? c->Sx[IDX(c, i - 1, j, k + 1)] : 0.0;
                double Sy = (j != 0) ? c->Sy[IDX(c, i, j - 1, k + 1)] : 0.0;
                dot = c->qx[i] * Sx + c->qy[j] * Sy + c->sz[k] * c->Sz[idx];
                v = c->CM1z[idx] * (c->Sz[idx] - c->CM2z[idx] * dot);
                if (with_divv) v = v + c->CM1z[idx] * (nu * c->sz[k] * c->divv[IDX(c, i, j, k + 1)]);
                c->vz[idx] = v;
            }
}

/* Gradient spectra by index shift (adv/cosAdvTrackMult.cpp:904-959): G_x[i] = -s_i f[i+1],
 * last index along the shifted axis left 0. */
static void shift_grad(orc_ctx *c, const double *f, double *gxo, double *gyo, double *gzo)
{
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    memset(gxo, 0, sizeof(double) * c->n);
    memset(gyo, 0, sizeof(double) * c->n);
    memset(gzo, 0, sizeof(double) * c->n);
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                long idx = IDX(c, i, j, k);
                if (i < nx - 1) gxo[idx] = -c->sx[i] * f[IDX(c, i + 1, j, k)];
                if (j < ny - 1) gyo[idx] = -c->sy[j] * f[IDX(c, i, j + 1, k)];
                if (k < nz - 1) gzo[idx] = -c->sz[k] * f[IDX(c, i, j, k + 1)];
            }
}

/* ---------------- adv: adv/cosAdvTrackMult.cpp:824-1369,1742 ---------------- */
static void step_adv(orc_ctx *c)
{
    const long n = c->n;
    const double dtd2 = c->p.dt / 2, b = c->p.beta, g = c->p.gamma;
    memcpy(c->NqPast, c->Nq, sizeof(double) * n);                  /* :842 */
    r3(c, c->psi, c->psiq, T10, T10, T10);                          /* :847 */
    for (long q = 0; q < n; q++) c->psiq[q] = c->scale * c->psiq[q]; /* :849-860 */
    shift_grad(c, c->psiq, c->gx, c->gy, c->gz);                    /* :864-959 */
    r3(c, c->psiq, c->psi, T01, T01, T01);                          /* :961-963 */
    r3(c, c->gx, c->gx, S01, T01, T01);                             /* :965-975 */
    r3(c, c->gy, c->gy, T01, S01, T01);
    r3(c, c->gz, c->gz, T01, T01, S01);
    for (long q = 0; q < n; q++) c->sp2[q] = -c->aLin[q] * c->psiq[q]; /* :980-986 */
    r3(c, c->sp2, c->sp2, T01, T01, T01);                           /* :988-990 */
    for (long q = 0; q < n; q++) {                                  /* :994-1015 */
        double m = (c->sp2[q] - b * pow(c->psi[q], 3) + g * pow(c->psi[q], 5));
        c->Sx[q] = m * c->gx[q];
        c->Sy[q] = m * c->gy[q];
        c->Sz[q] = m * c->gz[q];
    }
    r3(c, c->Sx, c->Sx, S10, T10, T10);                             /* :1017-1027 */
    r3(c, c->Sy, c->Sy, T10, S10, T10);
    r3(c, c->Sz, c->Sz, T10, T10, S10);
    stokes(c, 0);                                                   /* :1030-1274 */
    r3(c, c->vx, c->vx, S01, T01, T01);                             /* :1276-1286 */
    r3(c, c->vy, c->vy, T01, S01, T01);
    r3(c, c->vz, c->vz, T01, T01, S01);
    if (c->p.conserved) {
        /* conserved: N = q^2 CT(beta psi^3 - gamma psi^5) - CT(v . grad psi), the advection
         * unweighted (adv/cosAdvConSingle.cpp:1296-1310,1369); Sx is free after stokes() */
        for (long q = 0; q < n; q++) {
            c->Nr[q] = b * pow(c->psi[q], 3) - g * pow(c->psi[q], 5);
            c->Sx[q] = c->vx[q] * c->gx[q] + c->vy[q] * c->gy[q] + c->vz[q] * c->gz[q];
        }
        r3(c, c->Nr, c->Nq, T10, T10, T10);
        r3(c, c->Sx, c->Sx, T10, T10, T10);
        for (long q = 0; q < n; q++) c->Nq[q] = c->mq2[q] * c->Nq[q] - c->Sx[q];
    } else {
        for (long q = 0; q < n; q++)                                /* :1290-1303 */
            c->Nr[q] = b * pow(c->psi[q], 3) - g * pow(c->psi[q], 5) - c->vx[q] * c->gx[q] -
                       c->vy[q] * c->gy[q] - c->vz[q] * c->gz[q];
        r3(c, c->Nr, c->Nq, T10, T10, T10);                         /* :1307 */
    }
    if (c->surf_pending) surface_spectra(c, 1.0, c->scale);         /* :1311-1347 */
    for (long q = 0; q < n; q++)                                    /* :1355-1365 */
        c->psiq[q] = (c->C1[q] * c->psiq[q] + dtd2 * c->scale * (3.0 * c->Nq[q] - c->NqPast[q])) / c->C2[q];
    r3(c, c->psiq, c->psiNew, T01, T01, T01);                       /* :1369 */
    c->L1 = l1_measure(c, c->psiNew, c->psi);                       /* :1374-1396 */
    if (c->surf_pending) surface_eval(c, c->psi, c->gx, c->gy, c->gz); /* :1417-1515, psi^n */
    memcpy(c->psi, c->psiNew, sizeof(double) * n);                  /* :1742 */
}

/* ---------------- quasi: quasi/quasi.cpp:1099-2255 ---------------- */
static void step_quasi(orc_ctx *c)
{
    const long n = c->n;
    const orc_params *P = &c->p;
    const double dtd2 = P->dt / 2, b = P->beta, g = P->gamma, ep = P->eps, al = P->alpha;
    const double q02 = P->q0 * P->q0;
    c->nloop++;                                                     /* :1103 */
    memcpy(c->NqPast, c->Nq, sizeof(double) * n);                   /* :1117 (Nl_old = Nl) */
    for (long q = 0; q < n; q++) c->dfd[q] = al * (q02 - c->mq2[q]) * c->psiq[q]; /* :1121-1131 */
    r3(c, c->dfd, c->dfd, T01, T01, T01);                           /* :1135-1137 */
    shift_grad(c, c->psiq, c->gx, c->gy, c->gz);                    /* :1147-1256 */
    shift_grad(c, c->rhoq, c->rdx, c->rdy, c->rdz);
    r3(c, c->gx, c->gx, S01, T01, T01);                             /* :1280-1290 */
    r3(c, c->gy, c->gy, T01, S01, T01);
    r3(c, c->gz, c->gz, T01, T01, S01);
    r3(c, c->rdx, c->rdx, S01, T01, T01);                           /* :1294-1304 */
    r3(c, c->rdy, c->rdy, T01, S01, T01);
    r3(c, c->rdz, c->rdz, T01, T01, S01);
    for (long q = 0; q < n; q++)                                    /* :1322-1336 */
        c->rho[q] = P->kp * sqrt(q02 * pow(c->psi[q], 2) + pow(c->gx[q], 2) + pow(c->gy[q], 2) +
                                 pow(c->gz[q], 2)) + P->rho0;
    r3(c, c->rho, c->rhoq, T10, T10, T10);                          /* :1338-1340 */
    for (long q = 0; q < n; q++)                                    /* :1342-1351 */
        c->rhoq[q] = c->scale * c->rhoq[q] * exp(-1.57 * 1.57 * c->mq2[q] * 2);
    r3(c, c->rhoq, c->rho, T01, T01, T01);                          /* :1355-1357 */
    if (P->loaded && c->nloop == 1) memcpy(c->rho_old, c->rho, sizeof(double) * n); /* :1362-1364 */
    if (c->nloop > P->divv_switch || P->loaded) {                   /* :1366-1406 */
        for (long q = 0; q < n; q++) {
            c->divv[q] = -((c->rho[q] - c->rho_old[q]) / P->dt + c->vx[q] * c->rdx[q] +
                           c->vy[q] * c->rdy[q] + c->vz[q] * c->rdz[q]) /
                         (0.5 * (c->rho[q] + c->rho_old[q]));
            c->lap[q] = c->rho[q] * c->dfd[q];
        }
        r3(c, c->lap, c->lap, T10, T10, T10);
        for (long q = 0; q < n; q++) c->lap[q] = -c->scale * c->mq2[q] * c->lap[q];
        r3(c, c->lap, c->lap, T01, T01, T01);
    } else {                                                        /* :1410-1437 */
        for (long q = 0; q < n; q++) c->lap[q] = -c->mq2[q] * al * (q02 - c->mq2[q]) * c->psiq[q];
        r3(c, c->lap, c->lap, T01, T01, T01);
        for (long q = 0; q < n; q++) c->lap[q] = c->rho[q] * c->lap[q];
    }
    memcpy(c->rho_old, c->rho, sizeof(double) * n);                 /* :1439 */
    r3(c, c->divv, c->divv, T10, T10, T10);                         /* :1441-1443 */
    for (long q = 0; q < n; q++) {                                  /* :1448-1490 */
        double ps = c->psi[q];
        c->energy[q] = -0.5 * ep * pow(ps, 2) + 0.5 * pow(c->dfd[q], 2) - 0.25 * b * pow(ps, 4) +
                       (g / 6) * pow(ps, 6);
        c->mu[q] = c->lap[q] + c->rho[q] * (c->dfd[q] - ep * ps - b * pow(ps, 3) + g * pow(ps, 5));
        c->Sx[q] = c->mu[q] * c->gx[q] + c->energy[q] * c->rdx[q];
        c->Sy[q] = c->mu[q] * c->gy[q] + c->energy[q] * c->rdy[q];
        c->Sz[q] = c->mu[q] * c->gz[q] + c->energy[q] * c->rdz[q];
    }
    r3(c, c->Sx, c->Sx, S10, T10, T10);                             /* :1494-1504 */
    r3(c, c->Sy, c->Sy, T10, S10, T10);
    r3(c, c->Sz, c->Sz, T10, T10, S10);
    /* pressure, quasi/quasi.cpp:1548-1592 (single rank: the back plane is zero, :1546-1550) */
    for (int i = 0; i < c->nx; i++)
        for (int j = 0; j < c->ny; j++)
            for (int k = 0; k < c->nz; k++) {
                long idx = IDX(c, i, j, k);
                double Sx = (i > 0) ? c->Sx[IDX(c, i - 1, j, k)] : 0.0;
                double Sy = (j > 0) ? c->Sy[IDX(c, i, j - 1, k)] : 0.0;
                double Sz = (k > 0) ? c->Sz[idx - 1] : 0.0;
                if (i + j + k != 0)
                    c->p_[idx] = c->scale * (-(c->qx[i] * Sx + c->qy[j] * Sy + c->qz[k] * Sz) / c->mq2[idx] +
                                             (c->lambda + 2 * P->nu) * c->divv[idx]);
                else
                    c->p_[idx] = 0;
            }
    r3(c, c->p_, c->p_, T01, T01, T01);                             /* :1590-1592 */
    stokes(c, 1);                                                   /* :1599-2109 */
    r3(c, c->vx, c->vx, S01, T01, T01);                             /* :2113-2123 */
    r3(c, c->vy, c->vy, T01, S01, T01);
    r3(c, c->vz, c->vz, T01, T01, S01);
    for (long q = 0; q < n; q++) {                                  /* :2128-2154 */
        double v = -c->mu[q] - c->vx[q] * c->gx[q] - c->vy[q] * c->gy[q] - c->vz[q] * c->gz[q];
        if (c->nloop > P->divv_switch + 1)
            v += (c->p_[q] + c->rho[q] * c->energy[q]) * P->kp *
                 sqrt(pow(c->rdx[q], 2) + pow(c->rdy[q], 2) + pow(c->rdz[q], 2)) / pow(c->rho[q], 2);
        c->Nr[q] = v;
    }
    r3(c, c->Nr, c->Nq, T10, T10, T10);                             /* :2158-2160 */
    if (c->nloop == 1) memcpy(c->NqPast, c->Nq, sizeof(double) * n); /* :2162-2164 */
    for (long q = 0; q < n; q++) {                                  /* :2169-2182 */
        double old = c->psiq[q];
        c->psiq[q] = (c->C1[q] * c->psiq[q] - 0.5 * c->psiq_old[q] +
                      dtd2 * c->scale * (3.0 * c->Nq[q] - c->NqPast[q])) / c->C2[q];
        c->psiq_old[q] = old;
    }
    memcpy(c->psi_old, c->psi, sizeof(double) * n);                 /* :2186 */
    r3(c, c->psiq, c->psi, T01, T01, T01);                          /* :2188-2190 */
    /* diagnostics, quasi/quasi.cpp:2194-2251 */
    c->L1 = l1_measure(c, c->psi, c->psi_old);
    double rs = 0.0, es = 0.0;
    for (long q = 0; q < n; q++) { rs = rs + c->rho[q]; es = es + c->energy[q]; }
    c->mass = rs * c->dx * c->dx * c->dx;
    c->en = es * c->dx * c->dx * c->dx;
}

/* ---------------- compressible: compressible/compressible.cpp:1265-2720 ----------------
 * Single-rank semantics: the halo planes read as zero, so the last x-plane of the shifted
 * spectra and of v_x stay zero and the i = 0 neighbours of the y, z velocities and of the
 * divergence are zero.  Each expression keeps the reference's operand order. */
static void step_comp(orc_ctx *c)
{
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    const long n = c->n, nyz = (long)ny * nz;
    const orc_params *P = &c->p;
    const double scale = c->scale, dt = P->dt, dtd2 = P->dt / 2;
    const double beta = P->beta, gamma = P->gamma, alpha = P->alpha, ep = P->eps;
    const double q02 = P->q0 * P->q0, nu = P->nu, lambda = c->lambda, zeta = P->zeta;
    const double rho_0 = P->rho0, kp = c->kp_c, Amp = c->amp_c;
    c->nloop++;                                                      /* :1269 */
    const long nLoop = c->nloop;
    memcpy(c->NqPast, c->Nq, sizeof(double) * n);                    /* :1287 Nl_old = Nl */
    r3(c, c->rho, c->rhoq, T10, T10, T10);                           /* :1292-1294 */
    /* shifted gradient spectra of psi and rho (:1296-1431) */
    memset(c->gx, 0, sizeof(double) * n); memset(c->gy, 0, sizeof(double) * n); memset(c->gz, 0, sizeof(double) * n);
    memset(c->rdx, 0, sizeof(double) * n); memset(c->rdy, 0, sizeof(double) * n); memset(c->rdz, 0, sizeof(double) * n);
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                const long q = IDX(c, i, j, k);
                if (i < nx - 1) {
                    c->gx[q] = -c->sx[i] * c->psiq[q + nyz];
                    c->rdx[q] = -scale * c->sx[i] * c->rhoq[q + nyz];
                }
                if (j < ny - 1) {
                    c->gy[q] = -c->sy[j] * c->psiq[q + nz];
                    c->rdy[q] = -scale * c->sy[j] * c->rhoq[q + nz];
                }
                if (k < nz - 1) {
                    c->gz[q] = -c->sz[k] * c->psiq[q + 1];
                    c->rdz[q] = -scale * c->sz[k] * c->rhoq[q + 1];
                }
            }
    r3(c, c->gx, c->gx, S01, T01, T01);                              /* :1433-1455 */
    r3(c, c->gy, c->gy, T01, S01, T01);
    r3(c, c->gz, c->gz, T01, T01, S01);
    r3(c, c->rdx, c->rdx, S01, T01, T01);
    r3(c, c->rdy, c->rdy, T01, S01, T01);
    r3(c, c->rdz, c->rdz, T01, T01, S01);
    /* amplitude, Gaussian-filtered (:1478-1515) */
    for (long q = 0; q < n; q++)
        c->amp[q] = sqrt(q02 * pow(c->psi[q], 2) + pow(c->gx[q], 2) + pow(c->gy[q], 2) + pow(c->gz[q], 2));
    r3(c, c->amp, c->amp, T10, T10, T10);
    for (long q = 0; q < n; q++) c->amp[q] = scale * c->amp[q] * exp(-1.57 * 1.57 * c->mq2[q] * 2);
    r3(c, c->amp, c->amp, T01, T01, T01);
    /* dF/d(lap psi) (:1520-1534) */
    for (long q = 0; q < n; q++) c->dfd[q] = alpha * (q02 - c->mq2[q]) * c->psiq[q];
    r3(c, c->dfd, c->dfd, T01, T01, T01);
    /* lap(rho dF/dlap psi) (:1542-1630): after the relaxation steps rho is independent;
     * during them rho follows the amplitude, shifted up by rho_up planes */
    if (nLoop > P->divv_switch || P->loaded) {
        for (long q = 0; q < n; q++) c->lap[q] = c->rho[q] * c->dfd[q];
        r3(c, c->lap, c->lap, T10, T10, T10);
        for (long q = 0; q < n; q++) c->lap[q] = -scale * c->mq2[q] * c->lap[q];
        r3(c, c->lap, c->lap, T01, T01, T01);
    } else {
        for (long q = 0; q < n; q++) c->lap[q] = -c->mq2[q] * alpha * (q02 - c->mq2[q]) * c->psiq[q];
        r3(c, c->lap, c->lap, T01, T01, T01);
        for (long q = 0; q < n; q++) {
            const double rho_1 = rho_0;
            c->rho[q] = rho_1 + ((1 - rho_1) / Amp) * c->amp[q];
            c->lap[q] = c->rho[q] * c->lap[q];
        }
        if (P->rho_up > 0) {
            const int up = P->rho_up;
            for (int i = 0; i < nx; i++)
                for (int j = 0; j < ny; j++) {
                    const long col = IDX(c, i, j, 0);
                    for (int k = nz - 1; k > up - 1; k--) {
                        c->rho[col + k] = c->rho[col + k - up];
                        c->lap[col + k] = c->rho[col + k] * c->lap[col + k];
                    }
                    for (int k = 0; k < up && k < nz; k++) {
                        c->rho[col + k] = 1;
                        c->lap[col + k] = c->rho[col + k] * c->lap[col + k];
                    }
                }
        }
    }
    /* forces, chemical potential, density penalty (:1636-1678) */
    for (long q = 0; q < n; q++) {
        c->energy[q] = 0.5 * pow(c->dfd[q], 2);
        c->fgrad[q] = 0.5 * zeta * (pow(c->rho[q], 2) - pow(rho_0 + kp * c->amp[q], 2));
        c->mu[q] = c->lap[q] + c->rho[q] * (c->dfd[q]);
        c->Sx[q] = c->mu[q] * c->gx[q] + c->energy[q] * c->rdx[q];
        c->Sy[q] = c->mu[q] * c->gy[q] + c->energy[q] * c->rdy[q];
        c->Sz[q] = c->mu[q] * c->gz[q] + c->energy[q] * c->rdz[q];
        c->mu[q] = c->lap[q] + c->rho[q] * (c->dfd[q] - ep * c->psi[q] - beta * pow(c->psi[q], 3) +
                                            gamma * pow(c->psi[q], 5));
        c->energy[q] = c->rho[q] * c->energy[q];
        const double fx = kp * zeta * (c->rho[q] - rho_0 - kp * c->amp[q]) / (c->amp[q] + 0.001);
        c->fxs[q] = fx * c->gx[q];
        c->fys[q] = fx * c->gy[q];
        c->fzs[q] = fx * c->gz[q];
    }
    r3(c, c->fgrad, c->fgrad, T10, T10, T10);                        /* :1681-1711 */
    r3(c, c->energy, c->energy, T10, T10, T10);
    r3(c, c->Sx, c->Sx, S10, T10, T10);
    r3(c, c->Sy, c->Sy, T10, S10, T10);
    r3(c, c->Sz, c->Sz, T10, T10, S10);
    r3(c, c->fxs, c->fxs, S10, T10, T10);
    r3(c, c->fys, c->fys, T10, S10, T10);
    r3(c, c->fzs, c->fzs, T10, T10, S10);
    for (long q = 0; q < n; q++) c->fgrad[q] = c->fgrad[q] + c->energy[q] * exp(-1.57 * 1.57 * c->mq2[q] * 2); /* :1826-1835 */
    /* solenoidal and irrotational velocity spectra (:1838-2410) */
    memset(c->vx, 0, sizeof(double) * n); memset(c->vy, 0, sizeof(double) * n); memset(c->vz, 0, sizeof(double) * n);
    memset(c->virx, 0, sizeof(double) * n); memset(c->viry, 0, sizeof(double) * n); memset(c->virz, 0, sizeof(double) * n);
    const double l2n = lambda + 2 * nu;
    for (int i = 0; i < nx - 1; i++)                                 /* :1966-2085 */
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                const long q = IDX(c, i, j, k);
                const double Sy = (j != 0) ? c->Sy[IDX(c, i + 1, j - 1, k)] : 0.0;
                const double Sz = (k != 0) ? c->Sz[IDX(c, i + 1, j, k - 1)] : 0.0;
                const double dot = c->sx[i] * c->Sx[q] + c->qy[j] * Sy + c->qz[k] * Sz;
                c->vx[q] = (c->CM1x[q] / nu) * (c->Sx[q] - c->CM2x[q] * dot);
                c->virx[q] = (c->CM1x[q] / l2n) *
                             (c->sx[i] * c->fgrad[q + nyz] + c->CM2x[q] * dot * exp(-1.57 * 1.57 * 2 * scale / c->CM1x[q]));
            }
    for (int i = 0; i < nx; i++)                                     /* :2135-2410 */
        for (int j = 0; j < ny - 1; j++)
            for (int k = 0; k < nz - 1; k++) {
                const long q = IDX(c, i, j, k);
                double Sx = (i != 0) ? c->Sx[IDX(c, i - 1, j + 1, k)] : 0.0;
                const double Sz = (k != 0) ? c->Sz[IDX(c, i, j + 1, k - 1)] : 0.0;
                double dot = c->qx[i] * Sx + c->sy[j] * c->Sy[q] + c->qz[k] * Sz;
                c->vy[q] = (c->CM1y[q] / nu) * (c->Sy[q] - c->CM2y[q] * dot);
                c->viry[q] = (c->CM1y[q] / l2n) *
                             (c->sy[j] * c->fgrad[q + nz] + c->CM2y[q] * dot * exp(-1.57 * 1.57 * 2 * scale / c->CM1y[q]));
                Sx = (i != 0) ? c->Sx[IDX(c, i - 1, j, k + 1)] : 0.0;
                const double Sy = (j != 0) ? c->Sy[IDX(c, i, j - 1, k + 1)] : 0.0;
                dot = c->qx[i] * Sx + c->qy[j] * Sy + c->sz[k] * c->Sz[q];
                c->vz[q] = (c->CM1z[q] / nu) * (c->Sz[q] - c->CM2z[q] * dot);
                /* the k = 0 branch for i >= 1, 0 < j < ny-1 filters with CM1y (:2348-2350) */
                const double cmf = (i >= 1 && k == 0 && j >= 1) ? c->CM1y[q] : c->CM1z[q];
                c->virz[q] = (c->CM1z[q] / l2n) *
                             (c->sz[k] * c->fgrad[q + 1] + c->CM2z[q] * dot * exp(-1.57 * 1.57 * 2 * scale / cmf));
            }
    /* divergence of the irrotational part and the penalty force term (:2478-2527) */
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                const long q = IDX(c, i, j, k);
                const double Sx = i > 0 ? c->virx[q - nyz] : 0.0, fx = i > 0 ? c->fxs[q - nyz] : 0.0;
                const double Sy = j > 0 ? c->viry[q - nz] : 0.0, fy = j > 0 ? c->fys[q - nz] : 0.0;
                const double Sz = k > 0 ? c->virz[q - 1] : 0.0, fz = k > 0 ? c->fzs[q - 1] : 0.0;
                c->divv[q] = c->qx[i] * Sx + c->qy[j] * Sy + c->qz[k] * Sz;
                c->ampd[q] = scale * (c->qx[i] * fx + c->qy[j] * fy + c->qz[k] * fz);
            }
    r3(c, c->divv, c->divv, T01, T01, T01);
    r3(c, c->ampd, c->ampd, T01, T01, T01);
    r3(c, c->vx, c->vx, S01, T01, T01);                              /* :2529-2552 */
    r3(c, c->vy, c->vy, T01, S01, T01);
    r3(c, c->vz, c->vz, T01, T01, S01);
    r3(c, c->virx, c->virx, S01, T01, T01);
    r3(c, c->viry, c->viry, T01, S01, T01);
    r3(c, c->virz, c->virz, T01, T01, S01);
    /* mass balance, AB2 in real space (:2555-2573) */
    for (long q = 0; q < n; q++) {
        const double S = -(c->vx[q] + c->virx[q]) * c->rdx[q] - (c->vy[q] + c->viry[q]) * c->rdy[q] -
                         (c->vz[q] + c->virz[q]) * c->rdz[q] - c->rho[q] * c->divv[q];
        c->rho[q] = c->rho[q] + dt * (1.5 * S - 0.5 * c->frho[q]);
        c->frho[q] = S;
    }
    /* N (:2578-2612) */
    for (long q = 0; q < n; q++)
        c->Nr[q] = -c->mu[q] + (kp * zeta / (c->amp[q] + 0.001)) * (c->rho[q] - rho_0 - kp * c->amp[q]) * c->psi[q] -
                   c->ampd[q] - (c->vx[q] + c->virx[q]) * c->gx[q] - (c->vy[q] + c->viry[q]) * c->gy[q] -
                   (c->vz[q] + c->virz[q]) * c->gz[q];
    r3(c, c->Nr, c->Nq, T10, T10, T10);                              /* :2613 */
    if (nLoop == 1) memcpy(c->NqPast, c->Nq, sizeof(double) * n);    /* :2615-2617 */
    for (long q = 0; q < n; q++) {                                   /* :2619-2635 */
        const double old = c->psiq[q];
        c->psiq[q] = (c->C1[q] * c->psiq[q] - 0.5 * c->psiq_old[q] +
                      dtd2 * scale * (3.0 * c->Nq[q] - c->NqPast[q])) / c->C2[q];
        c->psiq_old[q] = old;
    }
    memcpy(c->psi_old, c->psi, sizeof(double) * n);                  /* :2639 */
    r3(c, c->psiq, c->psi, T01, T01, T01);                           /* :2641-2643 */
    /* diagnostics (:2647-2690), every step here */
    c->L1 = l1_measure(c, c->psi, c->psi_old);
    double rs = 0.0, es = 0.0;
    for (long q = 0; q < n; q++) {
        rs = rs + c->rho[q];
        const double e = -0.5 * ep * pow(c->psi[q], 2) + 0.5 * pow(c->dfd[q], 2) - 0.25 * beta * pow(c->psi[q], 4) +
                         (gamma / 6) * pow(c->psi[q], 6);
        c->energy[q] = e;
        es = es + c->rho[q] * e + 0.5 * zeta * pow(c->rho[q] - rho_0 - kp * c->amp[q], 2);
    }
    c->mass = rs * c->dx * c->dx * c->dx;
    c->en = es * c->dx * c->dx * c->dx;
}

int orc_step(orc_ctx *c, int nsteps)
{
    if (!c || !c->have_psi) return -1;
    for (int s = 0; s < nsteps; s++) {
        if (c->p.model == ORC_NOADV) { step_noadv(c); c->nloop++; }
        else if (c->p.model == ORC_ADV) { step_adv(c); c->nloop++; }
        else if (c->p.model == ORC_COMP) step_comp(c);
        else step_quasi(c);
    }
    return 0;
}

int orc_step_surface(orc_ctx *c, int *surf, double *vel, double *curvH, double *curvK)
{
    /* conserved runs have no reference surface output to follow: adv/cosAdvConSingle.cpp
     * comments it out (:1316-1352,1454-1524) and no-adv/cosNoAdvConserv.cpp evaluates its
     * spectra from the updated, already scaled psihat with one more scale factor (:816-847) */
    if (!c || !c->have_psi || c->p.model >= ORC_QUASI || c->p.conserved || !surf || !vel || !curvH || !curvK)
        return -1;
    c->s_idx = surf; c->s_vel = vel; c->s_H = curvH; c->s_K = curvK;
    c->surf_pending = 1;
    int rc = orc_step(c, 1);
    c->surf_pending = 0;
    c->s_idx = NULL; c->s_vel = c->s_H = c->s_K = NULL;
    return rc;
}

int orc_get(const orc_ctx *c, int field, double *out)
{
    const double *src = NULL;
    switch (field) {
    case ORC_F_PSI: src = c->psi; break;
    case ORC_F_PSIHAT: src = c->psiq; break;
    case ORC_F_VX: src = c->vx; break;
    case ORC_F_VY: src = c->vy; break;
    case ORC_F_VZ: src = c->vz; break;
    case ORC_F_GX: src = c->gx; break;
    case ORC_F_GY: src = c->gy; break;
    case ORC_F_GZ: src = c->gz; break;
    case ORC_F_RHO: src = c->rho; break;
    case ORC_F_P: src = c->p_; break;
    case ORC_F_DIVV: src = c->divv; break;
    case ORC_F_MU: src = c->mu; break;
    case ORC_F_ENERGY: src = c->energy; break;
    case ORC_F_NHAT: src = c->Nq; break;
    case ORC_F_AMP: src = c->amp; break;
    case ORC_F_VSOLX: src = c->p.model == ORC_COMP ? c->vx : NULL; break;
    case ORC_F_VSOLY: src = c->p.model == ORC_COMP ? c->vy : NULL; break;
    case ORC_F_VSOLZ: src = c->p.model == ORC_COMP ? c->vz : NULL; break;
    case ORC_F_VIRRX: src = c->virx; break;
    case ORC_F_VIRRY: src = c->viry; break;
    case ORC_F_VIRRZ: src = c->virz; break;
    case ORC_F_FRHO: src = c->frho; break;
    default: return -1;
    }
    if (!src) return -1;
    memcpy(out, src, sizeof(double) * c->n);
    return 0;
}

int orc_diag(const orc_ctx *c, double *d)
{
    double s = 0.0;
    for (long q = 0; q < c->n; q++) s += c->psi[q];
    d[0] = c->L1;
    d[1] = c->mass;
    d[2] = c->en;
    d[3] = s / (double)c->n;
    d[4] = (double)c->nloop;
    return 0;
}

double orc_free_energy(orc_ctx *c)
{
    const long n = c->n;
    const orc_params *P = &c->p;
    const double q02 = P->q0 * P->q0;
    double *ph = dal(n), *f = dal(n);
    r3(c, c->psi, ph, T10, T10, T10);
    for (long q = 0; q < n; q++) f[q] = P->alpha * (q02 - c->mq2[q]) * c->scale * ph[q];
    r3(c, f, f, T01, T01, T01);
    double es = 0.0;
    for (long q = 0; q < n; q++) {
        double ps = c->psi[q];
        es = es + (-0.5 * P->eps * pow(ps, 2) + 0.5 * pow(f[q], 2) - 0.25 * P->beta * pow(ps, 4) +
                   (P->gamma / 6) * pow(ps, 6));
    }
    free(ph);
    free(f);
    return es * c->dx * c->dx * c->dx;
}

/* Interface trackers:
 *   mode 0 (flat):  no-adv/cosNoAdvTrackSing.cpp:880-913, adv/cosAdvTrackMult.cpp:1417-1441
 *   mode 1 (bump):  no-adv/cosNoAdvTrackBump.cpp:936-970 (the upward walk stops at the last
 *                   index; the reference reads past the end there)
 *   mode 2 (level): quasi/quasi.cpp:2264-2280 (first value above hi from the top)
 * The scan runs from the last index of `axis` downwards, as the reference scans k. */
int orc_track(const orc_ctx *c, int field, int axis, int mode, double hi, double lo, int *idxo,
              double *poso)
{
    const double *f = (field == ORC_F_RHO) ? c->rho : c->psi;
    if (!f) return -1;
    int na, nb, nl;
    long sa, sb, sl;
    if (axis == 2) { na = c->nx; nb = c->ny; nl = c->nz; sa = (long)c->ny * c->nz; sb = c->nz; sl = 1; }
    else if (axis == 1) { na = c->nx; nb = c->nz; nl = c->ny; sa = (long)c->ny * c->nz; sb = 1; sl = c->nz; }
    else { na = c->ny; nb = c->nz; nl = c->nx; sa = c->nz; sb = 1; sl = (long)c->ny * c->nz; }
    for (int a = 0; a < na; a++)
        for (int bb = 0; bb < nb; bb++) {
            const double *col = f + a * sa + bb * sb;
#define V(t) col[(long)(t) * sl]
            int found = -1;
            double pos = NAN;
            if (mode == 0) {
                int track = 0;
                for (int t = nl - 1; t >= 0; t--) {
                    if (V(t) > hi && track == 0) track = 1;
                    if (V(t) < lo && track == 1) {
                        if (t + 1 >= nl) break;
                        int k2 = t;
                        if (fabs(V(t)) > fabs(V(t + 1))) k2 = t + 1;
                        found = k2;
                        double f0 = V(t), f1 = V(t + 1);
                        pos = t + (lo - f0) / (f1 - f0);
                        track = 2;
                        break;
                    }
                }
            } else if (mode == 1) {
                for (int t = nl - 1; t >= 0; t--) {
                    if (fabs(V(t)) > hi) {
                        int t3 = t;
                        while (t3 < nl - 1 && fabs(V(t3)) > lo) t3++;
                        int k2 = t3;
                        if (t3 + 1 < nl && fabs(V(t3)) > fabs(V(t3 + 1))) k2 = t3 + 1;
                        found = k2;
                        if (t3 > t) {
                            double f0 = fabs(V(t3 - 1)), f1 = fabs(V(t3));
                            pos = (t3 - 1) + (f0 - lo) / (f0 - f1);
                        } else {
                            pos = (double)t3;
                        }
                        break;
                    }
                }
            } else {
                for (int t = nl - 1; t >= 0; t--) {
                    if (V(t) > hi) {
                        found = t;
                        if (t + 1 < nl) {
                            double f0 = V(t), f1 = V(t + 1);
                            pos = t + (f0 - hi) / (f0 - f1);
                        } else {
                            pos = (double)t;
                        }
                        break;
                    }
                }
            }
#undef V
            idxo[(long)a * nb + bb] = found;
            poso[(long)a * nb + bb] = pos;
        }
    return 0;
}
