/*
 * smadft.h -- C ABI of the B200 time-step library for sma-dft's smectic-A / isotropic
 * Swift-Hohenberg solvers (diffusive "noadv", advected "adv", quasi-incompressible "quasi").
 *
 * The reference has no library API: each model is one monolithic main() whose time loop
 * body is the "per-step call" this ABI replaces.  The host driver keeps the reference's
 * parameter block, initial-condition builders and output files, and calls:
 *
 *     smadft_create(&params, &ctx);     // replaces the FFTW plan + aLin/C1/C2/CM* setup
 *     smadft_set_psi(ctx, psi0, n);     // replaces the IC upload + pre-loop N^0 block
 *     loop: smadft_step(ctx, 99);       // the loop body, 99 times
 *           smadft_step_diag(ctx, &d);  // one more step with the FP64 L1/mass/energy sums
 *           smadft_track(...);          // interface tracker on save steps
 *     smadft_get_psi(ctx, psi, n);      // final / checkpoint gather
 *
 * Conventions: plain C types only; every function returns SMADFT_OK (0) or a negative
 * SMADFT_ERR_* code and never exits or throws.  Host arrays use the reference layout
 * idx = (i*ny + j)*nz + k (x slowest, z contiguous) and are copied; the caller keeps
 * ownership.  A context owns its device memory and CUDA stream; one context is not
 * thread-safe, distinct contexts may be driven from different threads.
 */
#ifndef SMADFT_H
#define SMADFT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SMADFT_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------------------ */
#define SMADFT_OK 0
#define SMADFT_ERR_INVALID -1      /* bad argument / parameter block                       */
#define SMADFT_ERR_CUDA -2         /* a CUDA runtime call failed                            */
#define SMADFT_ERR_NOMEM -3        /* device or host allocation failed                      */
#define SMADFT_ERR_NONFINITE -4    /* psi became NaN/Inf (the reference's L1 test would
                                      silently stop: adv/cosAdvTrackMult.cpp:824)           */
#define SMADFT_ERR_TIMEOUT -5      /* a bounded device wait ran out                         */
#define SMADFT_ERR_UNSUPPORTED -6  /* grid length with a prime factor other than 2, 3, 5,
                                    * or a call the run's model does not have             */
#define SMADFT_ERR_IO -7           /* checkpoint file could not be read or written          */
#define SMADFT_ERR_STATE -8        /* call out of order (e.g. step before set_psi)          */
#define SMADFT_ERR_NODEVICE -9     /* no CUDA device / extension not usable                 */
#define SMADFT_ERR_TOO_LARGE -10   /* grid exceeds the fixed scratch of smadft_r2r3d_noalloc */

/* ---- models, precisions, fields -------------------------------------------------------- */
#define SMADFT_MODEL_NOADV 0  /* no-adv/cosNoAdvTrackSing.cpp */
#define SMADFT_MODEL_ADV 1    /* adv/cosAdvTrackMult.cpp      */
#define SMADFT_MODEL_QUASI 2  /* quasi/quasi.cpp              */
#define SMADFT_MODEL_COMP 3   /* compressible/compressible.cpp (independent density, amplitude field) */

#define SMADFT_FP64 0  /* every field and transform in double (the reference's arithmetic) */
#define SMADFT_FP32 1  /* fields and transforms in float; FP64 reductions                 */

#define SMADFT_FIELD_PSI 0       /* real-space psi                                              */
#define SMADFT_FIELD_PSIHAT 1    /* scaled spectral psi, psi = REDFT01^3(psihat)                */
#define SMADFT_FIELD_VX 2        /* real-space velocity of the last step (adv, quasi; comp: its
                                    solenoidal part)                                             */
#define SMADFT_FIELD_VY 3
#define SMADFT_FIELD_VZ 4
#define SMADFT_FIELD_GX 5        /* real-space grad psi of the last step (adv, quasi)           */
#define SMADFT_FIELD_GY 6
#define SMADFT_FIELD_GZ 7
#define SMADFT_FIELD_RHO 8       /* quasi: filtered density of the last step; comp: the density  */
#define SMADFT_FIELD_P 9         /* quasi: pressure of the last step                            */
#define SMADFT_FIELD_DIVV 10     /* quasi: REDFT10^3 of div v (the reference keeps it spectral);
                                    comp: div v in real space                                    */
#define SMADFT_FIELD_MU 11       /* quasi: chemical potential of the last step                  */
#define SMADFT_FIELD_ENERGY 12   /* quasi: energy density of the last step (not comp)           */
#define SMADFT_FIELD_NHAT 13     /* unscaled REDFT10^3 of the last nonlinear term               */
#define SMADFT_FIELD_AMP 14      /* comp: Gaussian-filtered amplitude of the last step          */
#define SMADFT_FIELD_VIRRX 15    /* comp: irrotational velocity of the last step                */
#define SMADFT_FIELD_VIRRY 16
#define SMADFT_FIELD_VIRRZ 17
#define SMADFT_FIELD_FRHO 18     /* comp: density rate of the last step (its AB2 history)       */
#define SMADFT_FIELD_DIVV_REAL 19 /* quasi: div v of the last step in real space, scale REDFT01^3
                                    of SMADFT_FIELD_DIVV (what the reference's save iteration
                                    writes to divv.dat, quasi/quasi.cpp:2417-2427,2468-2471)      */

/* Interface tracker modes (reference trackers; the scan runs from the last index down) */
#define SMADFT_TRACK_FLAT 0   /* psi > hi then psi < lo: no-adv/cosNoAdvTrackSing.cpp:880-913  */
#define SMADFT_TRACK_BUMP 1   /* |psi| > hi, walk up while |psi| > lo:
                                 no-adv/cosNoAdvTrackBump.cpp:936-970                          */
#define SMADFT_TRACK_LEVEL 2  /* first value > hi: quasi/quasi.cpp:2264-2280 (rho)           */

/* Parameter block.  Mirrors the reference's compile-time constants and argv:
 * no-adv/cosNoAdvTrackSing.cpp:130-172, adv/cosAdvTrackMult.cpp:149-198,
 * quasi/quasi.cpp:203-268, compressible/compressible.cpp:224-290. */
typedef struct {
    int model;          /* SMADFT_MODEL_*                                             */
    int precision;      /* SMADFT_FP64 or SMADFT_FP32                                  */
    int nx, ny, nz;     /* grid; each length even with prime factors 2, 3, 5 only     */
    double nw;          /* points per wavelength: L = N 2 pi / (q0 nw), dx = L / N     */
    double dt;          /* time step                                                  */
    double alpha, beta, gamma, eps, q0;  /* SH free energy                            */
    double nu;          /* viscosity (adv, quasi)                                     */
    double rho0, kp, amp;  /* quasi density law and rho_s = kp amp + rho0             */
    int divv_switch;    /* quasi: steps before div v comes from mass balance (ref 200) */
    int loaded;         /* quasi: the reference's load==1 branch (restart semantics)   */
    int device;         /* CUDA device ordinal                                        */
    int conserved;      /* noadv, adv: 1 = conserved dynamics, the reference's
                         * no-adv/cosNoAdvConserv.cpp (L and N weighted by q^2) and
                         * adv/cosAdvConSingle.cpp (C1, C2 and the SH part of N weighted by
                         * q^2, the advection v.grad psi not); 0 = the non-conserved models */
    int rho_up;         /* comp: planes rho is shifted up by in the relaxation steps (ref 16),
                         * 0 <= rho_up < nz; comp uses rho0 as its rho_0 (ref 0.01), divv_switch
                         * as the relaxation length, and derives Amp and kp from eps, beta, gamma */
    int reserved[3];
    double zeta;        /* comp: density penalty (ref 0.001)                                */
    double reserved_d[3];
} smadft_params;

/* FP64 diagnostics of one step (no-adv/cosNoAdvTrackSing.cpp:769-801,
 * adv/cosAdvTrackMult.cpp:1374-1408, quasi/quasi.cpp:2194-2255). */
typedef struct {
    double l1;        /* sum|psi_new - psi_old| / (dt sum|psi_new|)                     */
    double mass;      /* quasi: sum(rho) dx^3 of the step                               */
    double energy;    /* quasi: sum(e) dx^3 of the step; 0 for noadv/adv                 */
    double mean;      /* mean of psi_new (FP64 sum)                                     */
    long long steps;  /* steps taken since smadft_set_psi                               */
    int nonfinite;    /* 1 if psi_new holds NaN/Inf                                     */
    int reserved;
} smadft_diag;

typedef struct smadft_ctx smadft_ctx;

/* Library / error helpers */
int smadft_abi_version(void);
const char *smadft_error_string(int code);
/* Fills a parameter block with the configs' defaults for `model` (dx = lambda0/8,
 * alpha=1, beta=2, gamma=1, eps=-0.75, q0=1, nu=1, dt = 0.05 noadv / 0.02 adv, quasi). */
void smadft_params_init(smadft_params *p, int model);
/* Validates a parameter block without touching a device. */
int smadft_params_check(const smadft_params *p);

/* Replaces the FFTW plan creation and the aLin/C1/C2/CM* tables
 * (no-adv/cosNoAdvTrackSing.cpp:342-375,587-612; adv/cosAdvTrackMult.cpp:419-467,717-751;
 *  quasi/quasi.cpp:519-565,951-985). */
int smadft_create(const smadft_params *p, smadft_ctx **out);
int smadft_destroy(smadft_ctx *ctx);
const char *smadft_last_error(const smadft_ctx *ctx);

/* Initial condition upload + the pre-loop block (N^0 etc.):
 * no-adv/cosNoAdvTrackSing.cpp:614-635, adv/cosAdvTrackMult.cpp:755-777,
 * quasi/quasi.cpp:990-1062.  n must equal nx*ny*nz. */
int smadft_set_psi(smadft_ctx *ctx, const double *host_psi, size_t n);
int smadft_get_psi(smadft_ctx *ctx, double *host_psi, size_t n);
int smadft_get_field(smadft_ctx *ctx, int field, double *host, size_t n);

/* nsteps iterations of the loop body, asynchronous on the context stream:
 * no-adv/cosNoAdvTrackSing.cpp:681-764,1072; adv/cosAdvTrackMult.cpp:824-1369,1742;
 * quasi/quasi.cpp:1099-2190. */
int smadft_step(smadft_ctx *ctx, int nsteps);
/* One loop iteration with the FP64 diagnostic reductions; synchronises. */
int smadft_step_diag(smadft_ctx *ctx, smadft_diag *out);
int smadft_sync(smadft_ctx *ctx);

/* Interface tracker on the current psi (or rho for quasi with field SMADFT_FIELD_RHO).
 * axis: 0=x, 1=y, 2=z (the reference scans z).  idx (int) and pos (FP64 sub-grid
 * position, linear interpolation of the threshold crossing) are arrays over the two other
 * axes in index order; not found -> idx = -1, pos = NaN.  Replaces
 * no-adv/cosNoAdvTrackSing.cpp:880-913, no-adv/cosNoAdvTrackBump.cpp:936-970,
 * adv/cosAdvTrackMult.cpp:1417-1441, quasi/quasi.cpp:2264-2280. */
int smadft_track(smadft_ctx *ctx, int field, int axis, int mode, double hi, double lo,
                 int *idx, double *pos);
/* One loop body that also evaluates the interface diagnostics the reference writes every
 * 1000 steps (surfPsi, velSurf, curvH, curvK): per (i, j) column (nx*ny entries, index
 * i*ny + j) the flat-tracked interface index along z (-1: none), the normal velocity
 * dTpsi/|grad psi| and the curvatures 2H and K (Megrabov's divergence forms) there (NaN:
 * none), all at the step's starting state; noadv uses the finite-difference gradient of
 * psi, adv the step's spectral gradient.  diag (may be NULL) receives the step's FP64
 * diagnostics as smadft_step_diag gives them, since the reference computes both on the same
 * iteration.  Replaces no-adv/cosNoAdvTrackSing.cpp:737-764,808-1021 and
 * adv/cosAdvTrackMult.cpp:1311-1347,1417-1585.  Non-conserved noadv and adv only
 * (SMADFT_ERR_UNSUPPORTED for quasi and conserved runs: adv/cosAdvConSingle.cpp has these
 * outputs commented out, :1316-1352,1454-1524, and no-adv/cosNoAdvConserv.cpp:816-847 takes
 * its spectra from the updated, already normalised psihat with a second scale factor, so its
 * files do not hold the physical quantities).  Synchronises. */
int smadft_step_surface(smadft_ctx *ctx, int *surf_idx, double *vel, double *curvH, double *curvK,
                        smadft_diag *diag);
/* Free energy of the current psi, sum(e) dx^3 with the quasi energy density
 * (quasi/quasi.cpp:1470-1473) for any model; FP64 reduction. */
int smadft_free_energy(smadft_ctx *ctx, double *out);

/* Binary checkpoint (params, step counter, spectral state incl. the AB2/BDF2 history):
 * replaces the per-rank text save/load, adv/cosAdvTrackMult.cpp:606-631,1546-1557. */
int smadft_save_checkpoint(smadft_ctx *ctx, const char *path);
int smadft_load_checkpoint(smadft_ctx *ctx, const char *path);

/* Drop-in for the reference's per-step call with psi in HOST memory, as the reference
 * keeps it (its loop re-transforms psi every step: no-adv/cosNoAdvTrackSing.cpp:731,
 * adv/cosAdvTrackMult.cpp:847).  Uploads psi (n doubles), sets psihat = scale REDFT10^3 psi,
 * runs nsteps loop bodies, and writes psi back.  The AB2/BDF2 history stays on the device
 * (set it up once with smadft_set_psi).  Synchronises. */
int smadft_step_host(smadft_ctx *ctx, double *host_psi, size_t n, int nsteps);

/* The context's CUDA stream (a cudaStream_t) so callers can order or time work on it. */
int smadft_get_stream(smadft_ctx *ctx, void **stream);
/* Number of kernels this context has launched since creation. */
int smadft_launch_count(const smadft_ctx *ctx, long long *count);

/* Bounds-check build (`make -C sma-dft_b200 check` -> libsmadft_check.so, compiled with
 * SMADFT_CHECK_BOUNDS): every element index the axis-pass kernels hand to their loaders and
 * storers is checked against the field size, and an index outside it sets a device word
 * instead of touching memory.  *bad = 1 if that happened since the context was created
 * (synchronises).  The normal library returns SMADFT_ERR_UNSUPPORTED. */
int smadft_bounds_status(smadft_ctx *ctx, int *bad);

/* One axis pass of a 3-D r2r transform on device buffers (axis 0=x, 1=y, 2=z; kind as
 * below); in may equal out; both 16-byte aligned.  Exposed for tuning and for per-kernel roofline timing. */
int smadft_r2r_pass_device(smadft_ctx *ctx, const void *in, void *out, int axis, int kind);

/* Stand-alone 3-D r2r transform on device buffers (what fftw_execute does for one plan,
 * e.g. no-adv/cosNoAdvTrackSing.cpp:727).  kinds: 0 REDFT10, 1 REDFT01, 2 RODFT10,
 * 3 RODFT01 per axis; in may equal out; both 16-byte aligned.  precision SMADFT_FP64 (double*) or SMADFT_FP32
 * (float*).  Uses the context's stream and scratch field; the context's grid must match. */
int smadft_r2r3d_device(smadft_ctx *ctx, const void *in, void *out, int kx, int ky, int kz);

/* The same 3-D r2r transform for callers that cannot allocate device memory.  No
 * counterpart in the reference: FFTW plans own their buffers there.  Some callers cannot
 * call cudaMalloc: code whose device memory is fully reserved up front by another allocator
 * (a caching pool, an MPI+CUDA code that carved HBM at start-up), where cudaMalloc fails, and
 * fixed-latency loops where cudaMalloc's implicit device synchronisation is not acceptable.
 * This entry point needs no context and allocates nothing: the intermediate field lives in
 * a fixed file-scope device array of SMADFT_NOALLOC_MAX_BYTES that every GPU loading the
 * library holds until exit, and the twiddle tables in another (48 KiB), filled by a small
 * kernel on `stream` (no host copies).  It is an ordinary CUDA host call (it queries the
 * device and launches kernels): not for stream callbacks or cudaLaunchHostFunc functions,
 * where CUDA calls are not allowed.  Limits: nx*ny*nz*element_size <=
 * SMADFT_NOALLOC_MAX_BYTES (else SMADFT_ERR_TOO_LARGE), lengths even, <= 512, factors 2, 3, 5
 * (else SMADFT_ERR_UNSUPPORTED).  in/out 16-byte aligned device buffers (double* for
 * SMADFT_FP64, float* for SMADFT_FP32); in may equal out.  The work is queued on `stream` (a
 * cudaStream_t, NULL = legacy default stream).  All calls share the scratch array and the
 * twiddle tables, so calls that overlap on the GPU race; a call needs nothing from earlier
 * calls (it writes every element it reads).  The first call on a device looks the arrays up
 * for that device and sets kernel attributes; it should come before any stream capture. */
#define SMADFT_NOALLOC_MAX_BYTES (16u << 20)
int smadft_r2r3d_noalloc(const void *in, void *out, int nx, int ny, int nz, int kx, int ky, int kz,
                         int precision, void *stream);

/* ---- batches: independent runs advanced by one captured step ---------------------------
 * The batched parameter sweep of the north star (many runs of uneven grids and parameters):
 * the reference runs each as its own MPI job.  A batch owns n contexts (any model, grid,
 * precision and parameters; one device); smadft_batch_step advances every member by nsteps
 * loop bodies, each body one CUDA graph that runs all members' kernels concurrently.
 * Members of the same model (noadv or adv, non-conserved), grid and precision form a group:
 * their fields share one allocation per field, and each plain axis pass of the group runs as
 * one launch over all of them (the passes that carry a member's parameters run per member);
 * SMADFT_BATCH_GROUP=0 in the environment turns grouping off.
 * Members are ordinary contexts for everything else (smadft_batch_member): set their
 * initial conditions, read fields, track, checkpoint.  A batch is not thread-safe. */
typedef struct smadft_batch smadft_batch;
int smadft_batch_create(const smadft_params *params, int n, smadft_batch **out);
int smadft_batch_destroy(smadft_batch *batch);
int smadft_batch_size(const smadft_batch *batch, int *n);
int smadft_batch_member(smadft_batch *batch, int i, smadft_ctx **ctx);
int smadft_batch_step(smadft_batch *batch, int nsteps);
int smadft_batch_sync(smadft_batch *batch);
/* The batch's CUDA stream (a cudaStream_t): every batch step is ordered on it, so callers can
 * time or order work around smadft_batch_step. */
int smadft_batch_get_stream(smadft_batch *batch, void **stream);
/* Number of member groups advanced with pooled fields (see above). */
int smadft_batch_groups(const smadft_batch *batch, int *groups);
const char *smadft_batch_last_error(const smadft_batch *batch);

/* ---- adjoint (diffusive and advected models) -------------------------------------------
 * Gradients of an interface loss with respect to eps, alpha, beta, gamma (adv: and nu) and
 * the initial psi, by a hand-written adjoint of the semi-implicit step (transposed
 * transforms, linearised nonlinearity, transposed Stokes projection; the reference has no
 * counterpart).  The run must be at its
 * initial condition (right after smadft_set_psi).  smadft_adjoint advances it `steps`
 * loop bodies, keeping psihat and the AB2 history every `checkpoint_every` steps, takes
 * loss = mean sub-grid interface position (in lambda0) over the columns the tracker
 * (axis, mode, hi, lo as smadft_track; SMADFT_TRACK_FLAT or SMADFT_TRACK_BUMP) finds on the
 * final psi, then runs the reverse sweep, re-running each segment from its checkpoint.  The
 * found set and crossing cells are held fixed (as a small central difference sees them).
 * d_psi0 (may be NULL) receives dloss/dpsi_0 (nx*ny*nz doubles).  The run continues from
 * the final state.  Non-conserved noadv and adv (SMADFT_ERR_UNSUPPORTED for quasi and
 * conserved runs).  Synchronises. */
typedef struct {
    int steps;              /* loop bodies                                   */
    int checkpoint_every;   /* K: psihat / Nhat_prev kept every K steps       */
    int axis, mode;         /* interface tracker                             */
    double hi, lo;
} smadft_adj_opts;
typedef struct {
    double loss;            /* mean interface position, lambda0 units        */
    int found;              /* columns in the loss                           */
    double d_eps, d_alpha, d_beta, d_gamma;
    double d_nu;            /* adv: dloss/dnu (noadv: 0)                      */
} smadft_grads;
int smadft_adjoint(smadft_ctx *ctx, const smadft_adj_opts *opts, smadft_grads *out, double *d_psi0);

/* ---- kernel-path autotuner ---------------------------------------------------------------
 * Times `steps` loop bodies of each applicable kernel-path configuration on this context
 * (register-direct or staged passes, fused plane kernel, grouped y passes, forked chains)
 * and keeps the fastest; the run's state is restored after every trial, so stepping
 * continues exactly as without the call.  ms[i] = time per body of configuration i (-1:
 * not applicable to this grid), named by smadft_tune_config_name(i).  Synchronises. */
#define SMADFT_TUNE_MAX 8
typedef struct {
    int configs;                  /* configurations timed                    */
    int chosen;                   /* index of the one kept                   */
    double ms[SMADFT_TUNE_MAX];   /* milliseconds per loop body, -1 = skipped */
} smadft_tune_report;
int smadft_autotune(smadft_ctx *ctx, int steps, smadft_tune_report *out);
const char *smadft_tune_config_name(int i);

/* ---- initial-condition builders (host only, no device) --------------------------------
 * All write nx*ny*nz doubles in the reference layout; grid spacing dx = 2 pi/(q0 nw). */
/* Flat x-normal interface: A cos(q0 z) 1/2 (1 - tanh((x - x0)/(2 lambda0))) + U(+-noise),
 * x0 = L/2 + bump_amp sin(2 pi y / Ly) (bump_amp = 0: flat).  Noise from a counter-based
 * SplitMix64 stream keyed by (seed, idx). */
int smadft_ic_interface(const smadft_params *p, double A, double bump_amp, double noise,
                        unsigned long long seed, double *psi);
/* Single focal conic (torus cyclide), the reference's builder
 * no-adv/cosNoAdvTrackSing.cpp:403-449 / adv/cosAdvTrackMult.cpp:496-542 /
 * quasi/quasi.cpp:675-721: amplitude A, radii aE = bE = radius (grid units). */
int smadft_ic_focal_conic(const smadft_params *p, double A, double radius, double *psi);
/* Smectic layers A cos(q0 z) in the lower half (k < nz/2) with `count` focal-conic-like
 * radial perturbations (radius in [rmin, rmax] wavelengths, centres uniform in the
 * smectic half), seeded; plus U(+-noise). */
int smadft_ic_conics(const smadft_params *p, double A, int count, double rmin, double rmax,
                     double noise, unsigned long long seed, double *psi);

#ifdef __cplusplus
}
#endif
#endif /* SMADFT_H */
