// smadft.cu -- C ABI implementation: context set-up, the per-model loop bodies, FP64
// diagnostics, interface tracker and checkpoints.  See include/smadft.h for the contract.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "ctx.cuh"
#include "reduce.cuh"
#include "smadft.h"
#include "steps.h"

using namespace smadft;

// A captured loop body.  noadv/adv steps are all alike; quasi steps differ by the step
// counter (first step, before/after the div v switch, the extra N term), so each variant
// gets its own graph.
struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    long long launches = 0;   // kernels per replay
};

struct smadft_ctx {
    Ctx c;
    std::map<int, StepGraph> graphs;
    bool use_graphs = true;
    SurfaceScratch surf;
};

// One NVTX range per ABI call, named after the call: profilers (nsys, ncu --nvtx) group the
// call's kernels under it; without a tool attached a range costs a few nanoseconds.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

namespace {

int fail(Ctx &c, int code, const std::string &msg)
{
    c.err = msg;
    return code;
}

// After a synchronisation: SMADFT_ERR_TIMEOUT when a GEMM-form pass gave up one of its
// bounded waits (the error word is cleared again, so the context stays usable).
int gemm_wait_status(Ctx &c)
{
    if (!c.gz_err) return SMADFT_OK;
    int e = 0;
    if (cudaMemcpy(&e, c.gz_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, SMADFT_ERR_CUDA, "reading the GEMM-form pass status");
    }
    if (!e) return SMADFT_OK;
    cudaMemset(c.gz_err, 0, sizeof(int));
    return fail(c, SMADFT_ERR_TIMEOUT, "GEMM-form z pass: a bounded wait ran out (role " + std::to_string(e) + ")");
}

bool factor_ok(int n)
{
    if (n < 2 || (n & 1)) return false;
    while (n % 2 == 0) n /= 2;
    while (n % 3 == 0) n /= 3;
    while (n % 5 == 0) n /= 5;
    return n == 1;
}

// radix sequence: 4s, then a 2, then 3s and 5s (same factor order as the oracle)
void make_radices(int n, PlanDev &pd)
{
    int m = n, s = 0;
    while (m % 4 == 0) { pd.radix[s++] = 4; m /= 4; }
    while (m % 2 == 0) { pd.radix[s++] = 2; m /= 2; }
    while (m % 3 == 0) { pd.radix[s++] = 3; m /= 3; }
    while (m % 5 == 0) { pd.radix[s++] = 5; m /= 5; }
    pd.nst = s;
    for (; s < kMaxStages; s++) pd.radix[s] = 1;
}

// FFTW's r2r kinds of length n as dense matrices, Y = M x (unnormalised): REDFT10, REDFT01,
// RODFT10, RODFT01 in their published definitions.  Angles are reduced exactly in integers
// (pi a / (2n) with a taken mod 4n) before the FP64 cosine / sine.
double r2r_matrix_entry(int kind, int n, int k, int m)
{
    auto cs = [n](long long a) { return std::cos(M_PI * (double)(a % (4LL * n)) / (2.0 * n)); };
    auto sn = [n](long long a) { return std::sin(M_PI * (double)(a % (4LL * n)) / (2.0 * n)); };
    switch (kind) {
    case K_DCT2: return 2.0 * cs((long long)(2 * m + 1) * k);                      // 2 cos(pi (2m+1) k / 2n)
    case K_DCT3: return m == 0 ? 1.0 : 2.0 * cs((long long)m * (2 * k + 1));          // x_0 + 2 cos(pi m (2k+1) / 2n)
    case K_DST2: return 2.0 * sn((long long)(2 * m + 1) * (k + 1));                // 2 sin(pi (2m+1)(k+1) / 2n)
    default:                                                                          // (-1)^k x_{n-1} + 2 sin(...)
        return m == n - 1 ? ((k & 1) ? -1.0 : 1.0) : 2.0 * sn((long long)(m + 1) * (2 * k + 1));
    }
}

// The GEMM-form z pass's block matrices (r2r_gemm.cuh) of the four kinds, FP16 hi/lo of the
// entries scaled by 2^12: per kind, NB blocks x {hi, lo} x 128 x 128, row = output index.
// n = 256 splits each kind by its mirror symmetry: forward kinds take the even / odd output
// rows over the first 128 inputs (E[k][m] = M[2k][m], O[k][m] = M[2k+1][m]); inverse kinds
// the even / odd input columns of the first 128 outputs (P[k][j] = M[k][2j],
// Q[k][j] = M[k][2j+1]).  n = 128 keeps the whole matrix as one block.
std::vector<__half> gemm_z_matrices(int n)
{
    const int nb = n / 128;
    const size_t per_kind = (size_t)nb * 2 * 128 * 128;
    std::vector<__half> out(4 * per_kind);
    for (int kind = 0; kind < 4; kind++) {
        const bool fwd = kind == K_DCT2 || kind == K_DST2;
        for (int b = 0; b < nb; b++)
            for (int r = 0; r < 128; r++)
                for (int q = 0; q < 128; q++) {
                    int k = r, m = q;
                    if (nb == 2) {
                        if (fwd) k = 2 * r + b;
                        else m = 2 * q + b;
                    }
                    const double v = kGzMatScale * r2r_matrix_entry(kind, n, k, m);
                    const __half hi = __double2half(v);
                    const __half lo = __double2half(v - (double)__half2float(hi));
                    const size_t base = (size_t)kind * per_kind + ((size_t)(2 * b) * 128 + r) * 128 + q;
                    out[base] = hi;
                    out[base + 128 * 128] = lo;
                }
    }
    return out;
}

template <typename T>
int upload_plan(Ctx &c, int n)
{
    if (c.plans.count(n)) return SMADFT_OK;
    PlanDev pd{};
    make_radices(n, pd);
    std::vector<cpx<T>> w(n), h(n);
    for (int m = 0; m < n; m++) {
        double a = 2.0 * M_PI * (double)m / (double)n;
        w[m] = {T(std::cos(a)), T(-std::sin(a))};
        double b = M_PI * (double)m / (2.0 * (double)n);
        h[m] = {T(std::cos(b)), T(std::sin(b))};
    }
    SMADFT_CUDA(cudaMalloc(&pd.w, sizeof(cpx<T>) * n));
    SMADFT_CUDA(cudaMalloc(&pd.h, sizeof(cpx<T>) * n));
    SMADFT_CUDA(cudaMemcpy(pd.w, w.data(), sizeof(cpx<T>) * n, cudaMemcpyHostToDevice));
    SMADFT_CUDA(cudaMemcpy(pd.h, h.data(), sizeof(cpx<T>) * n, cudaMemcpyHostToDevice));
    if (sizeof(T) == 4 && (n == 128 || n == 256)) {
        const std::vector<__half> m = gemm_z_matrices(n);
        SMADFT_CUDA(cudaMalloc(&pd.gz, m.size() * sizeof(__half)));
        SMADFT_CUDA(cudaMemcpy(pd.gz, m.data(), m.size() * sizeof(__half), cudaMemcpyHostToDevice));
    }
    c.plans[n] = pd;
    return SMADFT_OK;
}

// Wavenumber tables exactly as the reference forms them (no-adv/cosNoAdvTrackSing.cpp:
// 309-324, adv/cosAdvTrackMult.cpp:386-401), then converted to the compute type.
template <typename T>
int upload_tables(Ctx &c)
{
    const int nx = c.g.nx, ny = c.g.ny, nz = c.g.nz;
    std::vector<double> qx(nx), qy(ny), qz(nz), sx(nx), sy(ny), sz(nz), ex(nx), ey(ny), ez(nz);
    std::vector<double> esx(nx), esy(ny), esz(nz);
    for (int i = 0; i < nx; i++) { qx[i] = 1.0 * M_PI * i / (c.dx * nx); sx[i] = 1.0 * M_PI * (i + 1) / (c.dx * nx); }
    for (int j = 0; j < ny; j++) { qy[j] = M_PI * (j) / (c.dy * ny); sy[j] = M_PI * (j + 1) / (c.dy * ny); }
    for (int k = 0; k < nz; k++) { qz[k] = M_PI * (k) / (c.dz * nz); sz[k] = M_PI * (k + 1) / (c.dz * nz); }
    // quasi Gaussian filter exp(-1.57^2 q^2 2) (quasi/quasi.cpp:1349), separable per axis
    const double fk = 1.57 * 1.57 * 2;
    for (int i = 0; i < nx; i++) ex[i] = std::exp(-fk * qx[i] * qx[i]);
    for (int j = 0; j < ny; j++) ey[j] = std::exp(-fk * qy[j] * qy[j]);
    for (int k = 0; k < nz; k++) ez[k] = std::exp(-fk * qz[k] * qz[k]);
    // the same factor on the DST wavenumbers: the compressible model's irrotational-velocity
    // filter exp(-2 1.57^2 |q_s|^2) (compressible/compressible.cpp:1985), separable per axis
    for (int i = 0; i < nx; i++) esx[i] = std::exp(-fk * sx[i] * sx[i]);
    for (int j = 0; j < ny; j++) esy[j] = std::exp(-fk * sy[j] * sy[j]);
    for (int k = 0; k < nz; k++) esz[k] = std::exp(-fk * sz[k] * sz[k]);
    const std::vector<double> *t[12] = {&qx, &qy, &qz, &sx, &sy, &sz, &ex, &ey, &ez, &esx, &esy, &esz};
    std::vector<T> all;
    for (int q = 0; q < 12; q++) {
        c.off[q] = all.size() * sizeof(T);
        for (double v : *t[q]) all.push_back(T(v));
    }
    SMADFT_CUDA(cudaMalloc(&c.tables, all.size() * sizeof(T)));
    SMADFT_CUDA(cudaMemcpy(c.tables, all.data(), all.size() * sizeof(T), cudaMemcpyHostToDevice));
    if (sizeof(T) == 8) {
        c.tables64 = c.tables;
        for (int q = 0; q < 12; q++) c.off64[q] = c.off[q];
    } else {
        std::vector<double> all64;
        for (int q = 0; q < 12; q++) {
            c.off64[q] = all64.size() * sizeof(double);
            for (double v : *t[q]) all64.push_back(v);
        }
        SMADFT_CUDA(cudaMalloc(&c.tables64, all64.size() * sizeof(double)));
        SMADFT_CUDA(cudaMemcpy(c.tables64, all64.data(), all64.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    return SMADFT_OK;
}

std::vector<int> slots_for(int model)
{
    std::vector<int> s = {S_PSI, S_PSI2, S_PSIH, S_NP, S_TMP};
    if (model != SMADFT_MODEL_NOADV) {
        for (int q : {S_GX, S_GY, S_GZ, S_SP2, S_SX, S_SY, S_SZ, S_VX, S_VY, S_VZ}) s.push_back(q);
    }
    if (model == SMADFT_MODEL_QUASI) {
        for (int q : {S_PSIH_OLD, S_RHO, S_RHO_OLD, S_RHOQ, S_DFD, S_RDX, S_RDY, S_RDZ, S_LAP,
                      S_DIVV, S_P, S_MU, S_EN})
            s.push_back(q);
    }
    if (model == SMADFT_MODEL_COMP) {
        for (int q : {S_PSIH_OLD, S_RHO, S_RHOQ, S_DFD, S_RDX, S_RDY, S_RDZ, S_LAP, S_DIVV, S_MU, S_EN,
                      S_AMP, S_FRHO, S_FGRAD, S_FX, S_FY, S_FZ, S_VIRX, S_VIRY, S_VIRZ, S_AMPD})
            s.push_back(q);
    }
    return s;
}

// Graph variant of the next loop body (see StepGraph).
int step_variant(const Ctx &c)
{
    if (c.p.model != SMADFT_MODEL_QUASI && c.p.model != SMADFT_MODEL_COMP) return 0;
    const long long nloop = c.steps + 1;
    if (c.p.model == SMADFT_MODEL_COMP)
        return (nloop == 1) | ((nloop > c.p.divv_switch || c.p.loaded) ? 2 : 0);
    const int first = nloop == 1;
    const int divv = (nloop > c.p.divv_switch || c.p.loaded) ? 1 : 0;
    const int extra = nloop > c.p.divv_switch + 1;
    return first | (divv << 1) | (extra << 2) | ((first && c.p.loaded) << 3);
}

template <typename T>
int one_step(Ctx &c, bool keep_old)
{
    int rc;
    switch (c.p.model) {
    case SMADFT_MODEL_NOADV: rc = noadv_step<T>(c, keep_old); break;
    case SMADFT_MODEL_ADV: rc = adv_step<T>(c); break;
    case SMADFT_MODEL_COMP: rc = comp_step<T>(c, c.steps + 1, keep_old); break;
    default: rc = quasi_step<T>(c, c.steps + 1, keep_old); break;
    }
    return rc;
}

// psi of the current state into S_PSI (adv keeps only psihat between steps)
template <typename T>
int ensure_psi(Ctx &c)
{
    if (c.p.model == SMADFT_MODEL_ADV && !c.psi_current) {
        int rc = refresh_psi<T>(c, c.f<T>(S_PSI));
        if (rc) return rc;
        c.psi_current = true;
    }
    return SMADFT_OK;
}

template <typename T>
int finish_diag(Ctx &c, smadft_diag *out);

template <typename T>
int step_diag_t(Ctx &c, smadft_diag *out)
{
    int rc;
    // psi_old must hold psi at the start of the step
    if ((rc = ensure_psi<T>(c))) return rc;
    if (c.p.model == SMADFT_MODEL_ADV) {
        if ((rc = adv_step<T>(c))) return rc;
        // adv compares with the round-tripped psi of the step (adv/cosAdvTrackMult.cpp:961-963)
        if ((rc = refresh_psi<T>(c, c.f<T>(S_PSI2)))) return rc;
    } else {
        if ((rc = one_step<T>(c, true))) return rc;
    }
    return finish_diag<T>(c, out);
}

// After a loop body that left psi^n in S_PSI and psi^{n+1} in S_PSI2: FP64 L1 / mean (and
// quasi's mass and energy) of the step, then psi^{n+1} -> S_PSI.
template <typename T>
int finish_diag(Ctx &c, smadft_diag *out)
{
    int rc;
    c.steps++;
    double sums[4];
    const T *nw = c.f<T>(S_PSI2), *od = c.f<T>(S_PSI);
    if ((rc = reduce_l1<T>(c, nw, od, sums))) return rc;
    double ms[2] = {0, 0};
    if (c.p.model == SMADFT_MODEL_QUASI) {
        if ((rc = reduce_mass_energy<T>(c, ms))) return rc;
    } else if (c.p.model == SMADFT_MODEL_COMP) {
        if ((rc = reduce_comp_mass_energy<T>(c, nw, ms))) return rc;
    }
    // psi_new -> S_PSI by copy: captured step graphs hold the slot pointers
    SMADFT_CUDA(cudaMemcpyAsync(c.slot[S_PSI], c.slot[S_PSI2], c.esize * c.n, cudaMemcpyDeviceToDevice, c.stream));
    c.psi_current = true;
    out->l1 = sums[0] / (c.p.dt * sums[1]);
    out->mean = sums[2] / (double)c.n;
    out->nonfinite = (sums[3] != 0.0 || !std::isfinite(sums[1])) ? 1 : 0;
    const double dx3 = c.dx * c.dx * c.dx;
    out->mass = ms[0] * dx3;
    out->energy = ms[1] * dx3;
    out->steps = c.steps;
    if ((rc = gemm_wait_status(c))) return rc;
    return out->nonfinite ? fail(c, SMADFT_ERR_NONFINITE, "psi is not finite") : SMADFT_OK;
}

// the surface body, then the step's L1 diagnostics (psi^{n+1} -> S_PSI as in step_diag)
template <typename T>
int step_surface_t(Ctx &c, SurfaceScratch &sc, smadft_diag *d)
{
    int rc = surface_step<T>(c, sc);
    if (rc) return rc;
    if (c.p.model == SMADFT_MODEL_ADV && (rc = refresh_psi<T>(c, c.f<T>(S_PSI2)))) return rc;
    return finish_diag<T>(c, d);
}

template <typename T>
int free_energy_t(Ctx &c, double *out)
{
    int rc;
    if ((rc = ensure_psi<T>(c))) return rc;
    T *fp = c.f<T>(S_PSI2);
    // f' = REDFT01^3(alpha (q0^2 - q^2) psihat)  (quasi/quasi.cpp:1121-1137)
    if ((rc = dfd_field<T>(c, fp))) return rc;
    double e;
    if ((rc = reduce_energy<T>(c, c.f<T>(S_PSI), fp, &e))) return rc;
    *out = e * c.dx * c.dx * c.dx;
    return SMADFT_OK;
}

template <typename T>
int set_psi_t(Ctx &c, const double *h)
{
    std::vector<T> tmp(c.n);
    for (long long q = 0; q < c.n; q++) tmp[q] = T(h[q]);
    SMADFT_CUDA(cudaMemcpyAsync(c.slot[S_PSI], tmp.data(), sizeof(T) * c.n, cudaMemcpyHostToDevice,
                                c.stream));
    int rc = pre_loop<T>(c);
    if (rc) return rc;
    SMADFT_CUDA(cudaStreamSynchronize(c.stream));
    return SMADFT_OK;
}

template <typename T>
int get_slot_t(Ctx &c, int slot, double *h)
{
    std::vector<T> tmp(c.n);
    SMADFT_CUDA(cudaMemcpyAsync(tmp.data(), c.slot[slot], sizeof(T) * c.n, cudaMemcpyDeviceToHost,
                                c.stream));
    SMADFT_CUDA(cudaStreamSynchronize(c.stream));
    for (long long q = 0; q < c.n; q++) h[q] = double(tmp[q]);
    return SMADFT_OK;
}

template <typename T>
int step_host_t(Ctx &c, double *host, int nsteps)
{
    if (!c.stage) SMADFT_CUDA(cudaMalloc(&c.stage, sizeof(double) * c.n));
    SMADFT_CUDA(cudaMemcpyAsync(c.stage, host, sizeof(double) * c.n, cudaMemcpyHostToDevice, c.stream));
    T *psi = c.f<T>(S_PSI);
    int rc;
    // psi from the host; psihat = scale REDFT10^3 psi (the reference's per-step planPsi)
    if ((rc = convert<double, T>(c, c.stage, psi))) return rc;
    if ((rc = psihat_from_psi<T>(c))) return rc;
    c.psi_current = true;
    for (int q = 0; q < nsteps; q++) {
        if ((rc = one_step<T>(c, false))) return rc;
        c.steps++;
        c.psi_current = (c.p.model != SMADFT_MODEL_ADV);
    }
    if ((rc = ensure_psi<T>(c))) return rc;
    if ((rc = convert<T, double>(c, psi, c.stage))) return rc;
    SMADFT_CUDA(cudaMemcpyAsync(host, c.stage, sizeof(double) * c.n, cudaMemcpyDeviceToHost, c.stream));
    SMADFT_CUDA(cudaStreamSynchronize(c.stream));
    return SMADFT_OK;
}

template <typename T>
int track_t(Ctx &c, int field, int axis, int mode, double hi, double lo, int *idx, double *pos)
{
    int rc;
    if (field == SMADFT_FIELD_PSI && (rc = ensure_psi<T>(c))) return rc;
    const T *f = c.f<T>(field == SMADFT_FIELD_RHO ? S_RHO : S_PSI);
    if (!f) return fail(c, SMADFT_ERR_INVALID, "field not available for this model");
    return track_columns<T>(c, f, axis, mode, hi, lo, idx, pos);
}

}  // namespace

// ====================================================================== C ABI ==========
extern "C" {

int smadft_abi_version(void) { return SMADFT_ABI_VERSION; }

const char *smadft_error_string(int code)
{
    switch (code) {
    case SMADFT_OK: return "ok";
    case SMADFT_ERR_INVALID: return "invalid argument";
    case SMADFT_ERR_CUDA: return "CUDA error";
    case SMADFT_ERR_NOMEM: return "out of memory";
    case SMADFT_ERR_NONFINITE: return "non-finite field";
    case SMADFT_ERR_TIMEOUT: return "device wait timed out";
    case SMADFT_ERR_UNSUPPORTED: return "unsupported grid length or model feature";
    case SMADFT_ERR_IO: return "checkpoint I/O error";
    case SMADFT_ERR_STATE: return "call out of order";
    case SMADFT_ERR_NODEVICE: return "no CUDA device";
    case SMADFT_ERR_TOO_LARGE: return "grid exceeds the no-alloc scratch maximum";
    default: return "unknown error";
    }
}

void smadft_params_init(smadft_params *p, int model)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->model = model;
    p->precision = SMADFT_FP64;
    p->nx = p->ny = p->nz = 64;
    p->nw = 8.0;
    p->dt = (model == SMADFT_MODEL_NOADV) ? 0.05 : 0.02;
    p->alpha = 1.0; p->beta = 2.0; p->gamma = 1.0; p->eps = -0.75; p->q0 = 1.0;
    p->nu = 1.0;
    p->rho0 = 1.0; p->kp = 0.0; p->amp = 1.34164;   // quasi/quasi.cpp:241-243
    p->divv_switch = 200;                            // quasi/quasi.cpp:206, compressible/compressible.cpp:228
    if (model == SMADFT_MODEL_COMP) {                // compressible/compressible.cpp:229,266,272,277
        p->dt = 0.001;
        p->rho0 = 0.01;
        p->zeta = 0.001;
        p->rho_up = 16;
    }
    p->loaded = 0;
    p->device = 0;
}

int smadft_params_check(const smadft_params *p)
{
    if (!p) return SMADFT_ERR_INVALID;
    if (p->model < 0 || p->model > 3) return SMADFT_ERR_INVALID;
    if (p->precision != SMADFT_FP64 && p->precision != SMADFT_FP32) return SMADFT_ERR_INVALID;
    if (p->nx < 4 || p->ny < 4 || p->nz < 4) return SMADFT_ERR_INVALID;
    if (p->nx > 1024 || p->ny > 1024 || p->nz > 1024) return SMADFT_ERR_UNSUPPORTED;
    if (!factor_ok(p->nx) || !factor_ok(p->ny) || !factor_ok(p->nz)) return SMADFT_ERR_UNSUPPORTED;
    if (!(p->nw > 0) || !(p->dt > 0) || !(p->q0 > 0)) return SMADFT_ERR_INVALID;
    if (p->model != SMADFT_MODEL_NOADV && !(p->nu > 0)) return SMADFT_ERR_INVALID;
    if (p->model == SMADFT_MODEL_QUASI && !(p->rho0 > 0)) return SMADFT_ERR_INVALID;
    // the reference has conserved variants of noadv and adv only
    if (p->conserved != 0 && (p->conserved != 1 || p->model >= SMADFT_MODEL_QUASI)) return SMADFT_ERR_INVALID;
    if (p->model == SMADFT_MODEL_COMP) {
        if (!(p->rho0 >= 0 && p->rho0 < 1) || !(p->zeta >= 0) || p->rho_up < 0 || p->rho_up >= p->nz)
            return SMADFT_ERR_INVALID;
        // the reference's load == 1 branch also reads rho from files; this ABI has no rho input
        if (p->loaded) return SMADFT_ERR_UNSUPPORTED;
        if (!(9 * p->beta * p->beta + 40 * p->eps * p->gamma >= 0)) return SMADFT_ERR_INVALID;   // real Amp
    }
    return SMADFT_OK;
}

int smadft_create(const smadft_params *p, smadft_ctx **out)
{
    if (!out) return SMADFT_ERR_INVALID;
    *out = nullptr;
    int rc = smadft_params_check(p);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return SMADFT_ERR_NODEVICE;
    }
    if (p->device < 0 || p->device >= ndev) return SMADFT_ERR_INVALID;
    smadft_ctx *h = new (std::nothrow) smadft_ctx;
    if (!h) return SMADFT_ERR_NOMEM;
    Ctx &c = h->c;
    c.p = *p;
    c.f32 = p->precision == SMADFT_FP32;
    c.esize = c.f32 ? 4 : 8;
    c.dev = p->device;
    c.g.nx = p->nx; c.g.ny = p->ny; c.g.nz = p->nz;
    c.g.nyz = (long long)p->ny * p->nz;
    c.n = (long long)p->nx * p->ny * p->nz;
    // box: no-adv/cosNoAdvTrackSing.cpp:160-172
    c.Lx = p->nx * 2.0 * M_PI / (p->q0 * p->nw);
    c.Ly = p->ny * 2.0 * M_PI / (p->q0 * p->nw);
    c.Lz = p->nz * 2.0 * M_PI / (p->q0 * p->nw);
    c.dx = c.Lx / p->nx; c.dy = c.Ly / p->ny; c.dz = c.Lz / p->nz;
    c.scale = 0.125 / ((double)p->nx * p->ny * p->nz);
    // SMADFT_PLANE=1 selects the fused z + y plane kernel (r2r_plane.cuh) where ny = nz allows;
    // the separate axis passes are the default (faster in FP32 on B200)
    if (const char *e = std::getenv("SMADFT_PLANE")) c.use_plane = e[0] != '0';
    if (const char *e = std::getenv("SMADFT_RDZ")) c.use_rdz = e[0] != '0';
    if (const char *e = std::getenv("SMADFT_MULTI")) c.use_multi = e[0] != '0';
    if (const char *e = std::getenv("SMADFT_FORK")) c.use_fork = e[0] != '0';
    if (const char *e = std::getenv("SMADFT_RDZ_REV")) c.rdz_rev = e[0] != '0';
    if (const char *e = std::getenv("SMADFT_RDZ_KIND")) c.rdz_static_kind = e[0] != '0';
    if (const char *e = std::getenv("SMADFT_RD_KIND")) c.rd_static_kind = e[0] != '0';
    if (const char *e = std::getenv("SMADFT_RD_DIR")) c.rd_static_dir = e[0] != '0';
    if (const char *e = std::getenv("SMADFT_RDZ_STAGE")) c.rdz_stage = e[0] != '0';
    // SMADFT_GEMM_Z=1: FP32 plain z passes of length 128 / 256 in GEMM form on the tensor cores
    if (const char *e = std::getenv("SMADFT_GEMM_Z")) c.use_gemm_z = e[0] != '0';
    // SMADFT_TMA_PASS=1: FP32 plain strided passes fed by TMA (r2r_rdt.cuh)
    if (const char *e = std::getenv("SMADFT_TMA_PASS")) c.use_tma = e[0] != '0';
    if (const char *e = std::getenv("SMADFT_SHARE_GRAD")) c.share_grad = e[0] != '0';
    if (const char *e = std::getenv("SMADFT_STOKES_K")) c.stokes_true_k = e[0] != '0';
    auto bail = [&](int code) { smadft_destroy(h); return code; };
    if (cudaSetDevice(c.dev) != cudaSuccess) { cudaGetLastError(); delete h; return SMADFT_ERR_CUDA; }
    if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess) return bail(SMADFT_ERR_CUDA);
    for (int m = 0; m < Ctx::kMaxFork; m++) {
        if (cudaStreamCreateWithFlags(&c.aux[m], cudaStreamNonBlocking) != cudaSuccess) return bail(SMADFT_ERR_CUDA);
        if (cudaEventCreateWithFlags(&c.ev_join[m], cudaEventDisableTiming) != cudaSuccess) return bail(SMADFT_ERR_CUDA);
    }
    if (cudaEventCreateWithFlags(&c.ev_fork, cudaEventDisableTiming) != cudaSuccess) return bail(SMADFT_ERR_CUDA);
    // Host-side fault injection for the failure tests: SMADFT_FAIL_ALLOC=k makes the k-th
    // field allocation of this call report out-of-memory (nothing is allocated for it), so
    // the clean-up path runs without a real allocation failure.
    int fail_at = -1, nalloc = 0;
    if (const char *e = std::getenv("SMADFT_FAIL_ALLOC")) fail_at = std::atoi(e);
    for (int s : slots_for(p->model)) {
        const size_t bytes = (slot_is_state(s) ? sizeof(double) : c.esize) * c.n;
        if (nalloc++ == fail_at) return bail(SMADFT_ERR_NOMEM);
        if (cudaMalloc(&c.slot[s], bytes) != cudaSuccess) { cudaGetLastError(); return bail(SMADFT_ERR_NOMEM); }
        if (cudaMemset(c.slot[s], 0, bytes) != cudaSuccess) return bail(SMADFT_ERR_CUDA);
    }
    for (int n : {p->nx, p->ny, p->nz}) {
        rc = c.f32 ? upload_plan<float>(c, n) : upload_plan<double>(c, n);
        if (rc) return bail(rc);
    }
    rc = c.f32 ? upload_tables<float>(c) : upload_tables<double>(c);
    if (rc) return bail(rc);
    if (cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, c.dev) != cudaSuccess || c.num_sms <= 0) {
        cudaGetLastError();
        c.num_sms = 148;
    }
#ifdef SMADFT_CHECK_BOUNDS
    if (cudaMalloc(&c.chk, sizeof(int)) != cudaSuccess) { cudaGetLastError(); return bail(SMADFT_ERR_NOMEM); }
    if (cudaMemset(c.chk, 0, sizeof(int)) != cudaSuccess) return bail(SMADFT_ERR_CUDA);
    c.g.nelem = c.n;
    c.g.chk = c.chk;
#endif
    if (c.f32) {   // error word of the GEMM-form passes
        if (cudaMalloc(&c.gz_err, sizeof(int)) != cudaSuccess) { cudaGetLastError(); return bail(SMADFT_ERR_NOMEM); }
        if (cudaMemset(c.gz_err, 0, sizeof(int)) != cudaSuccess) return bail(SMADFT_ERR_CUDA);
    }
    if ((rc = reduce_init(c))) return bail(rc);
    *out = h;
    return SMADFT_OK;
}

int smadft_destroy(smadft_ctx *h)
{
    if (!h) return SMADFT_OK;
    Ctx &c = h->c;
    cudaSetDevice(c.dev);
    if (c.stream) cudaStreamSynchronize(c.stream);
    for (auto &kv : h->graphs) cudaGraphExecDestroy(kv.second.exec);
    for (int s = 0; s < S_COUNT; s++)
        if (c.slot[s] && !c.pooled) cudaFree(c.slot[s]);
    for (auto &kv : c.plans) {
        cudaFree(kv.second.w);
        cudaFree(kv.second.h);
        if (kv.second.gz) cudaFree(kv.second.gz);
    }
    if (c.gz_err) cudaFree(c.gz_err);
    if (c.chk) cudaFree(c.chk);
    if (c.tables64 && c.tables64 != c.tables) cudaFree(c.tables64);
    if (c.tables) cudaFree(c.tables);
    if (c.red) cudaFree(c.red);
    if (c.red_out) cudaFree(c.red_out);
    if (c.stage) cudaFree(c.stage);
    cudaFree(h->surf.psih_prev);
    cudaFree(h->surf.fields);
    cudaFree(h->surf.idx);
    cudaFree(h->surf.vel);
    cudaFree(h->surf.curvH);
    cudaFree(h->surf.curvK);
    for (int m = 0; m < Ctx::kMaxFork; m++) {
        if (c.aux[m]) cudaStreamDestroy(c.aux[m]);
        if (c.ev_join[m]) cudaEventDestroy(c.ev_join[m]);
    }
    if (c.ev_fork) cudaEventDestroy(c.ev_fork);
    if (c.stream) cudaStreamDestroy(c.stream);
    cudaGetLastError();
    delete h;
    return SMADFT_OK;
}

const char *smadft_last_error(const smadft_ctx *h)
{
    if (!h) return "null context";
    return h->c.err.c_str();
}

int smadft_set_psi(smadft_ctx *h, const double *host, size_t n)
{
    NvtxRange nvtx_("smadft_set_psi");
    if (!h || !host) return SMADFT_ERR_INVALID;
    Ctx &c = h->c;
    if ((long long)n != c.n) return fail(c, SMADFT_ERR_INVALID, "size mismatch");
    cudaSetDevice(c.dev);
    for (int s = 0; s < S_COUNT; s++)
        if (c.slot[s] && s != S_PSI) {
            if (cudaMemsetAsync(c.slot[s], 0, (slot_is_state(s) ? sizeof(double) : c.esize) * c.n, c.stream) !=
                cudaSuccess)
                return fail(c, SMADFT_ERR_CUDA, "memset");
        }
    int rc = c.f32 ? set_psi_t<float>(c, host) : set_psi_t<double>(c, host);
    if (rc) return rc;
    c.steps = 0;
    c.have_psi = true;
    c.psi_current = true;
    return SMADFT_OK;
}

int smadft_get_psi(smadft_ctx *h, double *host, size_t n)
{
    return smadft_get_field(h, SMADFT_FIELD_PSI, host, n);
}

int smadft_get_field(smadft_ctx *h, int field, double *host, size_t n)
{
    if (!h || !host) return SMADFT_ERR_INVALID;
    Ctx &c = h->c;
    if ((long long)n != c.n) return fail(c, SMADFT_ERR_INVALID, "size mismatch");
    if (!c.have_psi) return fail(c, SMADFT_ERR_STATE, "no initial condition");
    cudaSetDevice(c.dev);
    int slot;
    switch (field) {
    case SMADFT_FIELD_PSI: slot = S_PSI; break;
    case SMADFT_FIELD_PSIHAT: slot = S_PSIH; break;
    case SMADFT_FIELD_VX: slot = S_VX; break;
    case SMADFT_FIELD_VY: slot = S_VY; break;
    case SMADFT_FIELD_VZ: slot = S_VZ; break;
    case SMADFT_FIELD_GX: slot = S_GX; break;
    case SMADFT_FIELD_GY: slot = S_GY; break;
    case SMADFT_FIELD_GZ: slot = S_GZ; break;
    case SMADFT_FIELD_RHO: slot = S_RHO; break;
    case SMADFT_FIELD_P: slot = S_P; break;
    case SMADFT_FIELD_DIVV: slot = S_DIVV; break;
    case SMADFT_FIELD_MU: slot = S_MU; break;
    case SMADFT_FIELD_ENERGY: slot = S_EN; break;
    case SMADFT_FIELD_NHAT: slot = S_NP; break;
    case SMADFT_FIELD_AMP: slot = S_AMP; break;
    case SMADFT_FIELD_VIRRX: slot = S_VIRX; break;
    case SMADFT_FIELD_VIRRY: slot = S_VIRY; break;
    case SMADFT_FIELD_VIRRZ: slot = S_VIRZ; break;
    case SMADFT_FIELD_FRHO: slot = S_FRHO; break;
    case SMADFT_FIELD_DIVV_REAL: {
        // the reference's save iteration: divv = REDFT01^3(scale divv_hat) (quasi/quasi.cpp:2417-2427)
        if (c.p.model != SMADFT_MODEL_QUASI) return fail(c, SMADFT_ERR_INVALID, "field not available for this model");
        int rc = c.f32 ? plain_r2r3d<float>(c, c.f<float>(S_DIVV), c.f<float>(S_TMP), K_DCT3, K_DCT3, K_DCT3)
                       : plain_r2r3d<double>(c, c.f<double>(S_DIVV), c.f<double>(S_TMP), K_DCT3, K_DCT3, K_DCT3);
        if (rc) return rc;
        rc = c.f32 ? get_slot_t<float>(c, S_TMP, host) : get_slot_t<double>(c, S_TMP, host);
        if (rc) return rc;
        for (long long q = 0; q < c.n; q++) host[q] *= c.scale;
        return SMADFT_OK;
    }
    default: return fail(c, SMADFT_ERR_INVALID, "unknown field");
    }
    if (!c.slot[slot]) return fail(c, SMADFT_ERR_INVALID, "field not available for this model");
    int rc;
    if (slot == S_PSI) {
        rc = c.f32 ? ensure_psi<float>(c) : ensure_psi<double>(c);
        if (rc) return rc;
    }
    return (c.f32 && !slot_is_state(slot)) ? get_slot_t<float>(c, slot, host) : get_slot_t<double>(c, slot, host);
}

// Runs one loop body by replaying its captured graph (captured on first use; the very
// first body of a context runs eagerly so that kernel attributes are set outside capture).
static int graph_step(smadft_ctx *h)
{
    Ctx &c = h->c;
    const int v = step_variant(c);
    auto it = h->graphs.find(v);
    if (it == h->graphs.end()) {
        if (c.launches == 0 || !h->use_graphs) {
            return c.f32 ? one_step<float>(c, false) : one_step<double>(c, false);
        }
        StepGraph g;
        cudaGraph_t graph = nullptr;
        const long long l0 = c.launches;
        SMADFT_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
        int rc = c.f32 ? one_step<float>(c, false) : one_step<double>(c, false);
        cudaError_t ce = cudaStreamEndCapture(c.stream, &graph);
        if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
        if (ce != cudaSuccess) { c.err = cudaGetErrorString(ce); return SMADFT_ERR_CUDA; }
        ce = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) { c.err = cudaGetErrorString(ce); return SMADFT_ERR_CUDA; }
        g.launches = c.launches - l0;
        c.launches = l0;
        it = h->graphs.emplace(v, g).first;
    }
    SMADFT_CUDA(cudaGraphLaunch(it->second.exec, c.stream));
    c.launches += it->second.launches;
    return SMADFT_OK;
}

int smadft_step(smadft_ctx *h, int nsteps)
{
    NvtxRange nvtx_("smadft_step");
    if (!h || nsteps < 0) return SMADFT_ERR_INVALID;
    Ctx &c = h->c;
    if (!c.have_psi) return fail(c, SMADFT_ERR_STATE, "no initial condition");
    cudaSetDevice(c.dev);
    for (int s = 0; s < nsteps; s++) {
        int rc = graph_step(h);
        if (rc) return rc;
        c.steps++;
        c.psi_current = (c.p.model != SMADFT_MODEL_ADV);
    }
    return SMADFT_OK;
}

int smadft_step_diag(smadft_ctx *h, smadft_diag *out)
{
    NvtxRange nvtx_("smadft_step_diag");
    if (!h || !out) return SMADFT_ERR_INVALID;
    Ctx &c = h->c;
    if (!c.have_psi) return fail(c, SMADFT_ERR_STATE, "no initial condition");
    cudaSetDevice(c.dev);
    std::memset(out, 0, sizeof(*out));
    return c.f32 ? step_diag_t<float>(c, out) : step_diag_t<double>(c, out);
}

int smadft_step_surface(smadft_ctx *h, int *surf_idx, double *vel, double *curvH, double *curvK,
                        smadft_diag *diag)
{
    NvtxRange nvtx_("smadft_step_surface");
    if (!h || !surf_idx || !vel || !curvH || !curvK) return SMADFT_ERR_INVALID;
    Ctx &c = h->c;
    if (!c.have_psi) return fail(c, SMADFT_ERR_STATE, "no initial condition");
    if (c.p.model >= SMADFT_MODEL_QUASI) return fail(c, SMADFT_ERR_UNSUPPORTED, "surface diagnostics: noadv and adv");
    if (c.p.conserved) return fail(c, SMADFT_ERR_UNSUPPORTED, "surface diagnostics: non-conserved runs only");
    cudaSetDevice(c.dev);
    SurfaceScratch &sc = h->surf;
    const size_t cols = (size_t)c.g.nx * c.g.ny;
    if (!sc.psih_prev) {
        bool ok = cudaMalloc(&sc.psih_prev, sizeof(double) * c.n) == cudaSuccess &&
                  cudaMalloc(&sc.fields, 4 * c.esize * c.n) == cudaSuccess &&
                  cudaMalloc(&sc.idx, sizeof(int) * cols) == cudaSuccess &&
                  cudaMalloc(&sc.vel, sizeof(double) * cols) == cudaSuccess &&
                  cudaMalloc(&sc.curvH, sizeof(double) * cols) == cudaSuccess &&
                  cudaMalloc(&sc.curvK, sizeof(double) * cols) == cudaSuccess;
        if (!ok) {
            cudaGetLastError();
            return fail(c, SMADFT_ERR_NOMEM, "surface diagnostics scratch");
        }
    }
    smadft_diag d;
    std::memset(&d, 0, sizeof(d));
    int rc = c.f32 ? step_surface_t<float>(c, sc, &d) : step_surface_t<double>(c, sc, &d);
    if (rc && rc != SMADFT_ERR_NONFINITE) return rc;
    if (diag) *diag = d;
    SMADFT_CUDA(cudaMemcpyAsync(surf_idx, sc.idx, sizeof(int) * cols, cudaMemcpyDeviceToHost, c.stream));
    SMADFT_CUDA(cudaMemcpyAsync(vel, sc.vel, sizeof(double) * cols, cudaMemcpyDeviceToHost, c.stream));
    SMADFT_CUDA(cudaMemcpyAsync(curvH, sc.curvH, sizeof(double) * cols, cudaMemcpyDeviceToHost, c.stream));
    SMADFT_CUDA(cudaMemcpyAsync(curvK, sc.curvK, sizeof(double) * cols, cudaMemcpyDeviceToHost, c.stream));
    SMADFT_CUDA(cudaStreamSynchronize(c.stream));
    return rc;
}

int smadft_adjoint(smadft_ctx *h, const smadft_adj_opts *o, smadft_grads *out, double *d_psi0)
{
    NvtxRange nvtx_("smadft_adjoint");
    if (!h || !o || !out || o->steps <= 0 || o->checkpoint_every <= 0 || o->axis < 0 || o->axis > 2 ||
        (o->mode != SMADFT_TRACK_FLAT && o->mode != SMADFT_TRACK_BUMP))
        return SMADFT_ERR_INVALID;
    Ctx &c = h->c;
    if (!c.have_psi || c.steps != 0) return fail(c, SMADFT_ERR_STATE, "adjoint: start from the initial condition");
    if (c.p.model >= SMADFT_MODEL_QUASI || c.p.conserved)
        return fail(c, SMADFT_ERR_UNSUPPORTED, "adjoint: non-conserved noadv and adv only");
    cudaSetDevice(c.dev);
    std::memset(out, 0, sizeof(*out));
    int rc;
    if (c.p.model == SMADFT_MODEL_ADV)
        rc = c.f32 ? adv_adjoint<float>(c, *o, out, d_psi0) : adv_adjoint<double>(c, *o, out, d_psi0);
    else
        rc = c.f32 ? noadv_adjoint<float>(c, *o, out, d_psi0) : noadv_adjoint<double>(c, *o, out, d_psi0);
    if (rc) return rc;
    c.steps += o->steps;
    c.psi_current = c.p.model != SMADFT_MODEL_ADV;   // adv: S_PSI holds psi of the last step's start
    return SMADFT_OK;
}

int smadft_sync(smadft_ctx *h)
{
    if (!h) return SMADFT_ERR_INVALID;
    Ctx &c = h->c;
    cudaSetDevice(c.dev);
    SMADFT_CUDA(cudaStreamSynchronize(c.stream));
    return gemm_wait_status(c);
}

int smadft_track(smadft_ctx *h, int field, int axis, int mode, double hi, double lo, int *idx,
                 double *pos)
{
    if (!h || !idx || !pos || axis < 0 || axis > 2 || mode < 0 || mode > 2) return SMADFT_ERR_INVALID;
    if (field != SMADFT_FIELD_PSI && field != SMADFT_FIELD_RHO) return SMADFT_ERR_INVALID;
    Ctx &c = h->c;
    if (!c.have_psi) return fail(c, SMADFT_ERR_STATE, "no initial condition");
    cudaSetDevice(c.dev);
    return c.f32 ? track_t<float>(c, field, axis, mode, hi, lo, idx, pos)
                 : track_t<double>(c, field, axis, mode, hi, lo, idx, pos);
}

int smadft_free_energy(smadft_ctx *h, double *out)
{
    if (!h || !out) return SMADFT_ERR_INVALID;
    Ctx &c = h->c;
    if (!c.have_psi) return fail(c, SMADFT_ERR_STATE, "no initial condition");
    cudaSetDevice(c.dev);
    return c.f32 ? free_energy_t<float>(c, out) : free_energy_t<double>(c, out);
}

int smadft_step_host(smadft_ctx *h, double *host, size_t n, int nsteps)
{
    NvtxRange nvtx_("smadft_step_host");
    if (!h || !host || nsteps < 0) return SMADFT_ERR_INVALID;
    Ctx &c = h->c;
    if ((long long)n != c.n) return fail(c, SMADFT_ERR_INVALID, "size mismatch");
    if (!c.have_psi) return fail(c, SMADFT_ERR_STATE, "no initial condition");
    cudaSetDevice(c.dev);
    return c.f32 ? step_host_t<float>(c, host, nsteps) : step_host_t<double>(c, host, nsteps);
}

int smadft_get_stream(smadft_ctx *h, void **stream)
{
    if (!h || !stream) return SMADFT_ERR_INVALID;
    *stream = (void *)h->c.stream;
    return SMADFT_OK;
}

int smadft_launch_count(const smadft_ctx *h, long long *count)
{
    if (!h || !count) return SMADFT_ERR_INVALID;
    *count = h->c.launches;
    return SMADFT_OK;
}

int smadft_bounds_status(smadft_ctx *h, int *bad)
{
    if (!h || !bad) return SMADFT_ERR_INVALID;
    *bad = 0;
#ifdef SMADFT_CHECK_BOUNDS
    Ctx &c = h->c;
    cudaSetDevice(c.dev);
    SMADFT_CUDA(cudaStreamSynchronize(c.stream));
    SMADFT_CUDA(cudaMemcpy(bad, c.chk, sizeof(int), cudaMemcpyDeviceToHost));
    return SMADFT_OK;
#else
    return SMADFT_ERR_UNSUPPORTED;
#endif
}

int smadft_r2r_pass_device(smadft_ctx *h, const void *in, void *out, int axis, int kind)
{
    if (!h || !in || !out || axis < 0 || axis > 2 || kind < 0 || kind > 3) return SMADFT_ERR_INVALID;
    if (((uintptr_t)in | (uintptr_t)out) & 15) return fail(h->c, SMADFT_ERR_INVALID, "buffers must be 16-byte aligned");
    Ctx &c = h->c;
    cudaSetDevice(c.dev);
    if (c.f32) return plain_pass<float>(c, (const float *)in, (float *)out, axis, kind);
    return plain_pass<double>(c, (const double *)in, (double *)out, axis, kind);
}

int smadft_r2r3d_device(smadft_ctx *h, const void *in, void *out, int kx, int ky, int kz)
{
    if (!h || !in || !out) return SMADFT_ERR_INVALID;
    for (int k : {kx, ky, kz})
        if (k < 0 || k > 3) return SMADFT_ERR_INVALID;
    Ctx &c = h->c;
    if (((uintptr_t)in | (uintptr_t)out) & 15) return fail(c, SMADFT_ERR_INVALID, "buffers must be 16-byte aligned");
    cudaSetDevice(c.dev);
    if (c.f32) return plain_r2r3d<float>(c, (const float *)in, (float *)out, kx, ky, kz);
    return plain_r2r3d<double>(c, (const double *)in, (double *)out, kx, ky, kz);
}

}  // extern "C"

#include "checkpoint.inc"
#include "batch.inc"
