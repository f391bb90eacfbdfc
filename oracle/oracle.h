/*
 * oracle.h -- FP64 CPU restatement of sma-dft's time-step loop (TEST INFRASTRUCTURE ONLY).
 *
 * This library is the parity checker for the CUDA path: only tests/, the smoke check and
 * the CPU-baseline leg of bench.py load it.  The product library never links or calls it.
 *
 * Models (one per reference directory):
 *   ORC_NOADV  no-adv/cosNoAdvTrackSing.cpp:584-1074   (diffusive, CN/AB2)
 *   ORC_ADV    adv/cosAdvTrackMult.cpp:717-1744          (advected, Stokes projection)
 *   ORC_QUASI  quasi/quasi.cpp:951-2498                  (quasi-incompressible, BDF2-like)
 *   ORC_COMP   compressible/compressible.cpp:1122-2720   (independent density, amplitude field)
 *
 * Parity is pinned two ways (tests/test_oracle_pin.py): against the reference's own
 * sources compiled here with a single-rank MPI shim and an FFTW-r2r shim (oracle/_ref,
 * built by oracle/build_ref.sh), and against the committed golden vectors in
 * tests/golden/ that were produced by that build.
 */
#ifndef SMADFT_ORACLE_H
#define SMADFT_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_NOADV = 0, ORC_ADV = 1, ORC_QUASI = 2, ORC_COMP = 3 };

typedef struct {
    int model;
    int nx, ny, nz;
    double nw;          /* points per wavelength: L_c = N_c 2 pi / (q0 nw) */
    double dt;
    double alpha, beta, gamma, eps, q0;
    double nu;          /* viscosity (adv, quasi) */
    double rho0, kp, amp; /* quasi density law: rho = kp sqrt(q0^2 psi^2 + |grad psi|^2) + rho0 */
    int divv_switch;    /* quasi: steps before div v comes from the mass balance (ref: 200) */
    int loaded;         /* quasi: the reference's load==1 branch semantics */
    int conserved;      /* noadv, adv: conserved dynamics d psi/dt = -q^2 (dF/dpsi)^,
                         * no-adv/cosNoAdvConserv.cpp, adv/cosAdvConSingle.cpp */
    double zeta;        /* comp: density penalty (ref 0.001); rho0 is the comp rho_0 (ref 0.01) */
    int rho_up;         /* comp: z shift of rho in the relaxation steps (ref 16) */
} orc_params;

typedef struct orc_ctx orc_ctx;

/* Field ids for orc_get. */
enum {
    ORC_F_PSI = 0,      /* real-space psi (current state) */
    ORC_F_PSIHAT = 1,   /* scaled spectral psi: scale * REDFT10^3(psi) */
    ORC_F_VX = 2, ORC_F_VY = 3, ORC_F_VZ = 4,      /* real-space velocity of the last step */
    ORC_F_GX = 5, ORC_F_GY = 6, ORC_F_GZ = 7,      /* real-space grad psi of the last step */
    ORC_F_RHO = 8, ORC_F_P = 9, ORC_F_DIVV = 10,   /* quasi: filtered rho, pressure, div v (spectral) */
    ORC_F_MU = 11, ORC_F_ENERGY = 12,              /* quasi: chemical potential, energy density */
    ORC_F_NHAT = 13,                               /* unscaled REDFT10^3 of the nonlinear term */
    ORC_F_AMP = 14,                                /* comp: filtered amplitude */
    ORC_F_VSOLX = 15, ORC_F_VSOLY = 16, ORC_F_VSOLZ = 17,   /* comp: solenoidal velocity */
    ORC_F_VIRRX = 18, ORC_F_VIRRY = 19, ORC_F_VIRRZ = 20,   /* comp: irrotational velocity */
    ORC_F_FRHO = 21,                               /* comp: the density rate of the last step */
    ORC_F_COUNT = 22
};

orc_ctx *orc_create(const orc_params *p);
void orc_destroy(orc_ctx *c);
/* Sets the initial condition and runs the model's pre-loop block. */
int orc_set_psi(orc_ctx *c, const double *psi);
/* Advances nsteps time steps (the reference's loop body). */
int orc_step(orc_ctx *c, int nsteps);
/* One time step that also evaluates the surface diagnostics the reference writes every
 * 1000 steps (noadv, adv): per (i, j) column (nx*ny entries) the flat-tracked interface
 * index along z (-1: none), the normal velocity dTpsi/|grad psi| and the curvatures 2H and
 * K there (NaN: none), all at the step's starting state psi^n: noadv
 * no-adv/cosNoAdvTrackSing.cpp:737-964 (finite-difference gradient), adv
 * adv/cosAdvTrackMult.cpp:1311-1347,1417-1515 (the step's spectral gradient). */
int orc_step_surface(orc_ctx *c, int *surf, double *vel, double *curvH, double *curvK);
/* Copies one field (nx*ny*nz doubles) out. */
int orc_get(const orc_ctx *c, int field, double *out);
/* diag[0]=L1 of the last step (ref definition), diag[1]=mass (quasi), diag[2]=energy of the
 * last step (quasi), diag[3]=mean psi, diag[4]=steps taken. */
int orc_diag(const orc_ctx *c, double *diag);
/* Free energy of the current psi: sum over cells of
 * -eps/2 psi^2 + 1/2 f'^2 - beta/4 psi^4 + gamma/6 psi^6 times dx^3, f' = alpha (q0^2 + lap) psi
 * (the quasi energy density, quasi/quasi.cpp:1470-1473, applied to any model). */
double orc_free_energy(orc_ctx *c);

/* Interface tracker (reference-compatible integer index and FP64 sub-grid position).
 * axis: 0=x, 1=y, 2=z (the reference scans z).  mode: 0 flat (psi>hi then psi<lo),
 * 1 bump (|psi|>hi then walk while |psi|>lo), 2 threshold (first value > hi, quasi rho).
 * field: ORC_F_PSI or ORC_F_RHO.  idx/pos are arrays over the two other axes in index
 * order; not found -> idx=-1, pos=NaN. */
int orc_track(const orc_ctx *c, int field, int axis, int mode, double hi, double lo, int *idx,
              double *pos);

/* Stand-alone pieces, exposed for unit tests. */
void orc_r2r_3d_kinds(const double *in, double *out, int nx, int ny, int nz, int kx, int ky, int kz);

#ifdef __cplusplus
}
#endif
#endif
