// ctx.cuh -- context, device buffers, per-length FFT plans and launch helpers.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <type_traits>
#include <string>
#include <vector>

#include "r2r_fast.cuh"
#include "r2r_gemm.cuh"
#include "r2r_plane.cuh"
#include "r2r_rd.cuh"
#include "r2r_rdz.cuh"
#include "r2r_rdt.cuh"
#include "r2r_pass.cuh"
#include "smadft.h"

namespace smadft {

// Kernel attributes (dynamic shared memory opt-in) are per device: launch helpers keep one
// flag per device index below this bound.
constexpr int kMaxDevices = 64;
// Distinct contexts may be driven from different host threads: the per-device attribute
// flags below are read and set under this lock (set once per kernel and device, so the lock
// is taken while a step graph is captured, not in the replayed steps).
inline std::mutex &attr_mutex()
{
    static std::mutex m;
    return m;
}

// Field slots (allocated per model; unused slots stay null).
enum Slot : int {
    S_PSI = 0, S_PSI2, S_PSIH, S_PSIH_OLD, S_NP, S_TMP,
    S_GX, S_GY, S_GZ, S_SP2, S_SX, S_SY, S_SZ, S_VX, S_VY, S_VZ,
    S_RHO, S_RHO_OLD, S_RHOQ, S_DFD, S_RDX, S_RDY, S_RDZ, S_LAP, S_DIVV, S_P, S_MU, S_EN,
    S_AMP, S_FRHO, S_FGRAD, S_FX, S_FY, S_FZ, S_VIRX, S_VIRY, S_VIRZ, S_AMPD,   // compressible
    S_COUNT
};

// The spectral state psihat (and quasi's psihat_old) is FP64 in every context: it carries
// the run from step to step, so its rounding would accumulate.  Nprev only enters the
// AB2 extrapolation and is replaced every step: it stays in the field precision.
inline bool slot_is_state(int s) { return s == S_PSIH || s == S_PSIH_OLD; }

struct PlanDev {
    int nst;
    int radix[kMaxStages];
    void *w;   // cpx<T>[n]
    void *h;   // cpx<T>[n]
    void *gz;  // FP32 contexts, n = 128 / 256: the GEMM-form block matrices of the four kinds
};

// Model constants handed to device functors by value.
template <typename T>
struct Spec {
    const T *qx, *qy, *qz, *sx, *sy, *sz;   // DCT / DST wavenumbers per axis
    const T *ex, *ey, *ez;                   // exp(-2 * 1.57^2 q^2) per axis (quasi filter)
    const T *esx, *esy, *esz;                // exp(-2 * 1.57^2 s^2) per axis (DST wavenumbers)
    T eps, alpha, beta, gamma, q02, dtd2, dt, scale, nu;
    T rho_m, lam, kp, rho0;
    T zeta, amp0;                            // compressible: density penalty, one-mode amplitude
    int nx, ny, nz;
    int nyz;
    __device__ __forceinline__ T mq2(int i, int j, int k) const
    {
        return qx[i] * qx[i] + qy[j] * qy[j] + qz[k] * qz[k];
    }
    // L(q) = eps - alpha (q^2 - q0^2)^2   (no-adv/cosNoAdvTrackSing.cpp:598-600)
    __device__ __forceinline__ T alin(int i, int j, int k) const
    {
        T d = mq2(i, j, k) - q02;
        return eps - alpha * (d * d);
    }
};

struct Ctx {
    smadft_params p;
    bool f32 = false;
    int dev = 0;
    cudaStream_t stream = nullptr;
    Geom g{};
    long long n = 0;
    double Lx = 0, Ly = 0, Lz = 0, dx = 0, dy = 0, dz = 0, scale = 0;
    std::string err;
    void *slot[S_COUNT] = {};
    size_t esize = 8;
    void *tables = nullptr;     // qx qy qz sx sy sz ex ey ez esx esy esz (T), contiguous
    size_t off[12] = {};
    void *tables64 = nullptr;   // the same in FP64 (= tables for FP64 contexts): time-update coefficients
    size_t off64[12] = {};
    std::map<int, PlanDev> plans;
    double *red = nullptr;      // reduction partials (device)
    double *red_out = nullptr;  // final sums (device)
    int red_blocks = 0;
    long long steps = 0;        // loop iterations since set_psi
    bool have_psi = false;
    bool psi_current = false;   // adv: S_PSI holds iCT(psihat) of the current state
    long long launches = 0;     // kernels launched by this context
    bool use_fast = true;       // compile-time-length pass kernels where available
    bool use_rd = true;         // register-direct kernels for plain strided passes
    bool use_rdz = true;        // register-direct z kernel for plain z passes (SMADFT_RDZ=0: staged)
    bool use_multi = true;      // one y-pass launch for the components of r2r3d_multi (SMADFT_MULTI=0: off)
    bool use_fork = true;       // independent per-component passes on forked streams (SMADFT_FORK=0: off)
    bool use_plane = false;
    bool rdz_rev = true;        // z passes walk their tiles from the last row down (SMADFT_RDZ_REV=0: up)
    bool rdz_static_kind = true;   // z passes specialised per transform kind (SMADFT_RDZ_KIND=0: not)
    bool rd_static_kind = true;    // plain strided passes specialised per kind (SMADFT_RD_KIND=0: not)
    bool rd_static_dir = true;     // grouped passes specialised per direction (SMADFT_RD_DIR=0: not)
    bool rdz_stage = true;         // inverse z passes stage their outputs in shared memory (SMADFT_RDZ_STAGE=0: not)
    bool use_gemm_z = false;       // FP32 plain z passes of length 128 / 256 on the tensor cores (SMADFT_GEMM_Z=1)
    int num_sms = 148;             // persistent grids (GEMM-form passes): one CTA per SM
    int *gz_err = nullptr;         // device word: nonzero when a GEMM-form pass gave up a bounded wait
    bool use_tma = false;          // FP32 plain strided passes fed by TMA, persistent (SMADFT_TMA_PASS=1)
    bool stokes_true_k = true;     // adv: force spectra stored by true wavenumber, aligned Stokes reads (SMADFT_STOKES_K=0: not)
    bool share_grad = true;        // adv: gradients reuse psi's y and z passes (SMADFT_SHARE_GRAD=0: not)
    int grid_y = 1;                // strided and generic passes: CTA rows (fields of a batch group, LoadArrM)
    bool pooled = false;           // field slots live in a batch group's pools (the batch frees them)
    int *chk = nullptr;            // bounds-check build: device word set by an out-of-range index
    static constexpr int kMaxFork = 5;
    cudaStream_t aux[kMaxFork] = {};   // forked streams (graph branches under capture)
    cudaEvent_t ev_fork = nullptr, ev_join[kMaxFork] = {};     // fused z + y passes (r2r_plane_kernel) where ny = nz allows
    double *stage = nullptr;    // FP64 staging field for host-psi steps (allocated on first use)

    template <typename T>
    T *f(int s) const { return reinterpret_cast<T *>(slot[s]); }
    template <typename T>
    const T *tab(int which) const
    {
        return reinterpret_cast<const T *>(reinterpret_cast<const char *>(tables) + off[which]);
    }
};

#define SMADFT_CUDA(call)                                                            \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) {                                                     \
            c.err = std::string(#call) + ": " + cudaGetErrorString(e_);              \
            return SMADFT_ERR_CUDA;                                                  \
        }                                                                            \
    } while (0)

template <typename T>
Spec<T> make_spec(const Ctx &c)
{
    Spec<T> s;
    if constexpr (sizeof(T) == 8) {
        // FP64 tables exist for every context (the time update always runs in FP64)
        auto t = [&](int w) { return reinterpret_cast<const T *>(reinterpret_cast<const char *>(c.tables64) + c.off64[w]); };
        s.qx = t(0); s.qy = t(1); s.qz = t(2); s.sx = t(3); s.sy = t(4); s.sz = t(5);
        s.ex = t(6); s.ey = t(7); s.ez = t(8);
        s.esx = t(9); s.esy = t(10); s.esz = t(11);
    } else {
        s.qx = c.tab<T>(0); s.qy = c.tab<T>(1); s.qz = c.tab<T>(2);
        s.sx = c.tab<T>(3); s.sy = c.tab<T>(4); s.sz = c.tab<T>(5);
        s.ex = c.tab<T>(6); s.ey = c.tab<T>(7); s.ez = c.tab<T>(8);
        s.esx = c.tab<T>(9); s.esy = c.tab<T>(10); s.esz = c.tab<T>(11);
    }
    const smadft_params &p = c.p;
    s.eps = T(p.eps); s.alpha = T(p.alpha); s.beta = T(p.beta); s.gamma = T(p.gamma);
    s.q02 = T(p.q0 * p.q0); s.dtd2 = T(p.dt / 2); s.dt = T(p.dt); s.scale = T(c.scale);
    s.nu = T(p.nu);
    double rho_s = p.kp * p.amp + p.rho0;       // quasi/quasi.cpp:244-245
    s.rho_m = T(rho_s / 2); s.lam = T(-2 * p.nu / 3); s.kp = T(p.kp); s.rho0 = T(p.rho0);
    s.zeta = T(p.zeta); s.amp0 = T(p.amp);
    if (p.model == SMADFT_MODEL_COMP) {
        // compressible/compressible.cpp:265-271: Amp of the one-mode smectic at eps, kp so that
        // rho_s = kp Amp + rho_0 = 1, rho_m = rho_s / 2, lambda = nu
        const double amp = std::sqrt((3 * p.beta + std::sqrt(9 * p.beta * p.beta + 40 * p.eps * p.gamma)) / 5);
        const double kp = (1 - p.rho0) / amp;
        rho_s = kp * amp + p.rho0;
        s.rho_m = T(rho_s / 2); s.lam = T(p.nu); s.kp = T(kp); s.amp0 = T(amp);
    }
    s.nx = c.g.nx; s.ny = c.g.ny; s.nz = c.g.nz; s.nyz = c.g.nyz;
    return s;
}

// Tile width: one 128-byte row segment per tile row.
template <typename T>
constexpr int tile_w() { return sizeof(T) == 4 ? 32 : 16; }

template <typename T, class LD, class ST>
int launch_generic(Ctx &c, int axis, int kind, LD ld, ST st)
{
    const int n = axis == 0 ? c.g.nx : (axis == 1 ? c.g.ny : c.g.nz);
    const PlanDev &pd = c.plans.at(n);
    PassArgs<T> a;
    a.g = c.g;
    a.axis = axis;
    a.kind = kind;
    a.W = tile_w<T>();
    a.ld = n;
    a.P.n = n;
    a.P.nst = pd.nst;
    for (int s = 0; s < kMaxStages; s++) a.P.radix[s] = pd.radix[s];
    a.P.w = reinterpret_cast<const cpx<T> *>(pd.w);
    a.P.h = reinterpret_cast<const cpx<T> *>(pd.h);
    long long tiles;
    if (axis == 2) {
        a.tiles_b = 1;
        tiles = ((long long)c.g.nx * c.g.ny + a.W - 1) / a.W;
    } else {
        a.tiles_b = (c.g.nz + a.W - 1) / a.W;
        tiles = (long long)(axis == 1 ? c.g.nx : c.g.ny) * a.tiles_b;
    }
    const size_t smem = 2 * (size_t)(a.W / 2) * a.ld * sizeof(cpx<T>);
    static size_t attr_set[kMaxDevices] = {};   // largest opt-in so far, per device and instantiation
    {
        std::lock_guard<std::mutex> lock(attr_mutex());
        if (smem > attr_set[c.dev % kMaxDevices]) {
            SMADFT_CUDA(cudaFuncSetAttribute(r2r_pass_kernel<T, LD, ST>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            attr_set[c.dev % kMaxDevices] = smem;
        }
    }
    r2r_pass_kernel<T, LD, ST><<<dim3((unsigned)tiles, (unsigned)c.grid_y), 256, smem, c.stream>>>(a, ld, st);
    SMADFT_CUDA(cudaGetLastError());
    c.launches++;
    return SMADFT_OK;
}

template <typename T, int N, int AXIS, class LD, class ST, int NC, int KIND, int DIR = -1>
int launch_rd_k(Ctx &c, const KindSet<NC> &kinds, LD ld, ST st)
{
    const PlanDev &pd = c.plans.at(N);
    const int tiles_b = (c.g.nz + 31) / 32;
    const long long tiles = (long long)(AXIS == 1 ? c.g.nx : c.g.ny) * tiles_b * NC;
    constexpr size_t smem = rd_smem_bytes<T, N>();
    static unsigned long long attr_set = 0;   // devices whose attribute is set (bit per device)
    {
        std::lock_guard<std::mutex> lock(attr_mutex());
        if (!(attr_set >> (c.dev % kMaxDevices) & 1ull)) {
            SMADFT_CUDA(cudaFuncSetAttribute(r2r_rd_kernel<T, N, AXIS, LD, ST, NC, KIND, DIR>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            attr_set |= 1ull << (c.dev % kMaxDevices);
        }
    }
    r2r_rd_kernel<T, N, AXIS, LD, ST, NC, KIND, DIR><<<dim3((unsigned)tiles, (unsigned)c.grid_y), RdInfo<N>::THREADS, smem,
                                                       c.stream>>>(
        c.g, kinds, tiles_b, ld, reinterpret_cast<const cpx<T> *>(pd.w), reinterpret_cast<const cpx<T> *>(pd.h), st);
    SMADFT_CUDA(cudaGetLastError());
    c.launches++;
    return SMADFT_OK;
}

// strided pass: one-component passes run an instantiation per transform kind
// (SMADFT_RD_KIND=0: the kind at run time): plain ones (LoadArr -> StoreArr, the bulk of a
// step) for all four kinds, passes with fused loaders or storers for the cosine kinds they
// use (their sine passes and the grouped passes take the kind at run time)
template <typename T, int N, int AXIS, class LD, class ST, int NC = 1, int DIR = -1>
int launch_rd(Ctx &c, const KindSet<NC> &kinds, LD ld, ST st)
{
    if constexpr (NC > 1 && DIR >= 0) {
        // grouped pass whose caller states the direction (SMADFT_RD_DIR=0: at run time)
        if (c.rd_static_dir) return launch_rd_k<T, N, AXIS, LD, ST, NC, -1, DIR>(c, kinds, ld, st);
    }
    if constexpr (NC == 1) {
        if (c.rd_static_kind) {
            constexpr bool plain = std::is_same<LD, LoadArr<T>>::value && std::is_same<ST, StoreArr<T>>::value;
            switch (kinds.k[0]) {
            case K_DCT2: return launch_rd_k<T, N, AXIS, LD, ST, 1, K_DCT2>(c, kinds, ld, st);
            case K_DCT3: return launch_rd_k<T, N, AXIS, LD, ST, 1, K_DCT3>(c, kinds, ld, st);
            case K_DST2:
                if constexpr (plain) return launch_rd_k<T, N, AXIS, LD, ST, 1, K_DST2>(c, kinds, ld, st);
                break;
            default:
                if constexpr (plain) return launch_rd_k<T, N, AXIS, LD, ST, 1, K_DST3>(c, kinds, ld, st);
                break;
            }
        }
    }
    return launch_rd_k<T, N, AXIS, LD, ST, NC, -1>(c, kinds, ld, st);
}

// z passes run more CTAs per SM (fewer registers); strided passes keep two
template <int AXIS>
using FastCfgFor = typename std::conditional<AXIS == 2, FastCfg<32, 256, 4, 3>, FastDefault>::type;

template <typename T, int N, int AXIS, class LD, class ST>
int launch_fast(Ctx &c, int kind, LD ld, ST st)
{
    using CFG = FastCfgFor<AXIS>;
    const PlanDev &pd = c.plans.at(N);
    const int W = CFG::W;
    int tiles_b = 1;
    long long tiles;
    if (AXIS == 2) {
        tiles = ((long long)c.g.nx * c.g.ny + W - 1) / W;
    } else {
        tiles_b = (c.g.nz + W - 1) / W;
        tiles = (long long)(AXIS == 1 ? c.g.nx : c.g.ny) * tiles_b;
    }
    constexpr size_t smem = fast_smem_bytes<T, N, CFG>();
    static unsigned long long attr_set = 0;   // devices whose attribute is set (bit per device)
    {
        std::lock_guard<std::mutex> lock(attr_mutex());
        if (!(attr_set >> (c.dev % kMaxDevices) & 1ull)) {
            SMADFT_CUDA(cudaFuncSetAttribute(r2r_fast_kernel<T, N, AXIS, LD, ST, CFG>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            attr_set |= 1ull << (c.dev % kMaxDevices);
        }
    }
    r2r_fast_kernel<T, N, AXIS, LD, ST, CFG><<<dim3((unsigned)tiles, (unsigned)c.grid_y), CFG::THREADS, smem, c.stream>>>(
        c.g, kind, tiles_b, reinterpret_cast<const cpx<T> *>(pd.w), reinterpret_cast<const cpx<T> *>(pd.h), ld, st);
    SMADFT_CUDA(cudaGetLastError());
    c.launches++;
    return SMADFT_OK;
}

// plain z pass of length N through the register-direct z kernel (in == out allowed); with
// zs, the pass of the shifted gradient spectrum along z (in != out)
template <typename T, int N, int KIND, bool STAGE = false, int ZM = kZPlain>
int launch_rdz_k(Ctx &c, int kind, const T *in, T *out, const T *zs = nullptr)
{
    const PlanDev &pd = c.plans.at(N);
    const int rows = c.g.nx * c.g.ny;
    const int tiles = (rows + 2 * kRdLines - 1) / (2 * kRdLines);
    constexpr size_t smem = rdz_smem_bytes<T, N>();
    static unsigned long long attr_set = 0;   // devices whose attribute is set (bit per device)
    {
        std::lock_guard<std::mutex> lock(attr_mutex());
        if (!(attr_set >> (c.dev % kMaxDevices) & 1ull)) {
            SMADFT_CUDA(cudaFuncSetAttribute(r2r_rdz_kernel<T, N, KIND, STAGE, ZM>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            attr_set |= 1ull << (c.dev % kMaxDevices);
        }
    }
    r2r_rdz_kernel<T, N, KIND, STAGE, ZM><<<(unsigned)tiles, RdInfo<N>::THREADS, smem, c.stream>>>(
        rows, kind, in, out, reinterpret_cast<const cpx<T> *>(pd.w), reinterpret_cast<const cpx<T> *>(pd.h),
        c.rdz_rev ? 1 : 0, zs);
    SMADFT_CUDA(cudaGetLastError());
    c.launches++;
    return SMADFT_OK;
}

// plain z pass: one instantiation per transform kind (SMADFT_RDZ_KIND=0: the kind at run time)
template <typename T, int N>
int launch_rdz(Ctx &c, int kind, const T *in, T *out)
{
    if (!c.rdz_static_kind) return launch_rdz_k<T, N, -1>(c, kind, in, out);
    // inverse kinds stage their outputs through shared memory when `out` allows 16-byte stores
    const bool stage = c.rdz_stage && ((uintptr_t)out & 15) == 0;
    switch (kind) {
    case K_DCT2: return launch_rdz_k<T, N, K_DCT2, false>(c, kind, in, out);
    case K_DCT3:
        return stage ? launch_rdz_k<T, N, K_DCT3, true>(c, kind, in, out)
                     : launch_rdz_k<T, N, K_DCT3, false>(c, kind, in, out);
    case K_DST2: return launch_rdz_k<T, N, K_DST2, false>(c, kind, in, out);
    default:
        return stage ? launch_rdz_k<T, N, K_DST3, true>(c, kind, in, out)
                     : launch_rdz_k<T, N, K_DST3, false>(c, kind, in, out);
    }
}

// z pass of the shifted gradient spectrum along z (LdGrad<T, 2, T>), inverse sine kind: the
// gradient's z transform in the psi / grad psi family
template <typename T, int N>
int launch_rdz_gradz(Ctx &c, const T *in, T *out, const T *zs)
{
    if (((uintptr_t)out & 15) == 0 && c.rdz_stage) return launch_rdz_k<T, N, K_DST3, true, kZGrad>(c, K_DST3, in, out, zs);
    return launch_rdz_k<T, N, K_DST3, false, kZGrad>(c, K_DST3, in, out, zs);
}

// inverse sine z pass of a spectrum stored by true wavenumber along z (read one index up)
template <typename T, int N>
int launch_rdz_upread(Ctx &c, const T *in, T *out)
{
    if (((uintptr_t)out & 15) == 0 && c.rdz_stage) return launch_rdz_k<T, N, K_DST3, true, kZUpRead>(c, K_DST3, in, out);
    return launch_rdz_k<T, N, K_DST3, false, kZUpRead>(c, K_DST3, in, out);
}

// forward sine z pass whose output is stored by true wavenumber along z (one index up)
template <typename T, int N>
int launch_rdz_upstore(Ctx &c, const T *in, T *out)
{
    return launch_rdz_k<T, N, K_DST2, false, kZUpStore>(c, K_DST2, in, out);
}

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime (no link
// against libcuda)
using GzEncodeFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
inline GzEncodeFn gz_encode_fn()
{
    static GzEncodeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<GzEncodeFn>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// plain FP32 strided pass of length N fed by TMA (r2r_rdt.cuh): persistent, two CTAs per SM
template <int N, int AXIS, class ST, int KIND>
int launch_rdt_k(Ctx &c, int kind, const float *in, ST st)
{
    const int tiles_b = (c.g.nz + 31) / 32;
    const int tiles = (AXIS == 1 ? c.g.nx : c.g.ny) * tiles_b;
    GzEncodeFn enc = gz_encode_fn();
    if (!enc) {
        c.err = "TMA-fed pass: cuTensorMapEncodeTiled unavailable";
        return SMADFT_ERR_CUDA;
    }
    CUtensorMap map;
    const cuuint64_t gdim[3] = {(cuuint64_t)c.g.nz, (cuuint64_t)c.g.ny, (cuuint64_t)c.g.nx};
    const cuuint64_t gstride[2] = {(cuuint64_t)c.g.nz * sizeof(float), (cuuint64_t)c.g.nyz * sizeof(float)};
    const cuuint32_t box[3] = {32, AXIS == 1 ? (cuuint32_t)N : 1u, AXIS == 0 ? (cuuint32_t)N : 1u};
    const cuuint32_t estr[3] = {1, 1, 1};
    if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(in), gdim, gstride, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
        c.err = "TMA-fed pass: tensor map rejected";
        return SMADFT_ERR_CUDA;
    }
    constexpr size_t smem = rdt_smem_bytes<float, float, N>();
    static unsigned long long attr_set = 0;
    {
        std::lock_guard<std::mutex> lock(attr_mutex());
        if (!(attr_set >> (c.dev % kMaxDevices) & 1ull)) {
            SMADFT_CUDA(cudaFuncSetAttribute(r2r_rdt_kernel<float, float, N, AXIS, ST, KIND>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            attr_set |= 1ull << (c.dev % kMaxDevices);
        }
    }
    const PlanDev &pd = c.plans.at(N);
    const int grid = tiles < 2 * c.num_sms ? tiles : 2 * c.num_sms;
    r2r_rdt_kernel<float, float, N, AXIS, ST, KIND><<<grid, RdInfo<N>::THREADS, smem, c.stream>>>(
        map, c.g, kind, tiles, tiles_b, reinterpret_cast<const cpx<float> *>(pd.w),
        reinterpret_cast<const cpx<float> *>(pd.h), st, c.gz_err);
    SMADFT_CUDA(cudaGetLastError());
    c.launches++;
    return SMADFT_OK;
}

template <int N, int AXIS, class ST>
int launch_rdt(Ctx &c, int kind, const float *in, ST st)
{
    switch (kind) {
    case K_DCT2: return launch_rdt_k<N, AXIS, ST, K_DCT2>(c, kind, in, st);
    case K_DCT3: return launch_rdt_k<N, AXIS, ST, K_DCT3>(c, kind, in, st);
    default: return launch_rdt_k<N, AXIS, ST, -1>(c, kind, in, st);
    }
}

// plain z pass of length N (FP32) in GEMM form on the tensor cores (r2r_gemm.cuh); in == out allowed
template <int N, bool FWD>
int launch_gemm_z_k(Ctx &c, int kind, const float *in, float *out)
{
    using GI = GzInfo<N>;
    const int rows = c.g.nx * c.g.ny;
    const PlanDev &pd = c.plans.at(N);
    if (!pd.gz || !c.gz_err) {
        c.err = "GEMM-form z pass: no block matrices for this length";
        return SMADFT_ERR_STATE;
    }
    GzEncodeFn enc = gz_encode_fn();
    if (!enc) {
        c.err = "GEMM-form z pass: cuTensorMapEncodeTiled unavailable";
        return SMADFT_ERR_CUDA;
    }
    CUtensorMap map;
    const cuuint64_t gdim[2] = {(cuuint64_t)N, (cuuint64_t)rows};
    const cuuint64_t gstride[1] = {(cuuint64_t)N * sizeof(float)};
    const cuuint32_t box[2] = {32, (cuuint32_t)kGzRows};
    const cuuint32_t estr[2] = {1, 1};
    if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(in), gdim, gstride, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
        c.err = "GEMM-form z pass: tensor map rejected";
        return SMADFT_ERR_CUDA;
    }
    static unsigned long long attr_set = 0;   // devices whose attribute is set (bit per device)
    {
        std::lock_guard<std::mutex> lock(attr_mutex());
        if (!(attr_set >> (c.dev % kMaxDevices) & 1ull)) {
            SMADFT_CUDA(cudaFuncSetAttribute(r2r_gemm_z_kernel<N, FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)GI::SMEM));
            attr_set |= 1ull << (c.dev % kMaxDevices);
        }
    }
    const int tiles = (rows + kGzRows - 1) / kGzRows;
    const int grid = tiles < c.num_sms ? tiles : c.num_sms;
    const __half *mats = reinterpret_cast<const __half *>(pd.gz) + (size_t)kind * GI::MAT_ELEMS;
    r2r_gemm_z_kernel<N, FWD><<<grid, kGzThreads, GI::SMEM, c.stream>>>(map, out, rows, mats, c.gz_err);
    SMADFT_CUDA(cudaGetLastError());
    c.launches++;
    return SMADFT_OK;
}

template <int N>
int launch_gemm_z(Ctx &c, int kind, const float *in, float *out)
{
    const bool fwd = kind == K_DCT2 || kind == K_DST2;
    return fwd ? launch_gemm_z_k<N, true>(c, kind, in, out) : launch_gemm_z_k<N, false>(c, kind, in, out);
}

// Line lengths with a compile-time staged kernel (the configs' grids); others use the
// generic one.  Lengths 64/128/256 run the register-direct kernels instead: strided axes
// with any loader and storer, the z axis for plain arrays.
#define SMADFT_FAST_SIZES(X) X(64) X(96) X(128) X(160) X(256)
#define SMADFT_FAST_SIZES_STRIDED(X) X(96) X(160)

template <typename T, int AXIS, class LD, class ST>
int launch_axis(Ctx &c, int kind, LD ld, ST st)
{
    const int n = AXIS == 0 ? c.g.nx : (AXIS == 1 ? c.g.ny : c.g.nz);
    if constexpr (AXIS != 2 && std::is_same<T, float>::value && std::is_same<LD, LoadArr<float>>::value) {
        // plain FP32 inputs: the TMA-fed persistent pass where enabled and the layout allows
        if (c.use_tma && c.gz_err && c.grid_y == 1 && c.g.nz % 4 == 0 && ((uintptr_t)ld.p & 15) == 0) {
            switch (n) {
            case 64: return launch_rdt<64, AXIS>(c, kind, ld.p, st);
            case 128: return launch_rdt<128, AXIS>(c, kind, ld.p, st);
            case 256: return launch_rdt<256, AXIS>(c, kind, ld.p, st);
            default: break;
            }
        }
    }
    if constexpr (AXIS != 2) {
        if (c.use_rd) {
            switch (n) {
            case 64: return launch_rd<T, 64, AXIS>(c, KindSet<1>{{kind}}, ld, st);
            case 128: return launch_rd<T, 128, AXIS>(c, KindSet<1>{{kind}}, ld, st);
            case 256: return launch_rd<T, 256, AXIS>(c, KindSet<1>{{kind}}, ld, st);
            default: break;
            }
        }
    } else if constexpr (std::is_same<LD, LoadArr<T>>::value && std::is_same<ST, StoreArr<T>>::value) {
        if constexpr (std::is_same<T, float>::value) {
            if (c.use_gemm_z && c.gz_err && (n == 128 || n == 256) && ((uintptr_t)ld.p & 15) == 0) {
                if (n == 256) return launch_gemm_z<256>(c, kind, ld.p, st.p);
                return launch_gemm_z<128>(c, kind, ld.p, st.p);
            }
        }
        if (c.use_rd && c.use_rdz) {
            switch (n) {
            case 64: return launch_rdz<T, 64>(c, kind, ld.p, st.p);
            case 128: return launch_rdz<T, 128>(c, kind, ld.p, st.p);
            case 256: return launch_rdz<T, 256>(c, kind, ld.p, st.p);
            default: break;
            }
        }
    }
    if (c.use_fast) {
#define SMADFT_CASE(N_) \
    case N_: return launch_fast<T, N_, AXIS>(c, kind, ld, st);
        if constexpr (AXIS == 2) {
            switch (n) {
                SMADFT_FAST_SIZES(SMADFT_CASE)
            default: break;
            }
        } else {
            switch (n) {
                SMADFT_FAST_SIZES_STRIDED(SMADFT_CASE)
            default: break;
            }
        }
#undef SMADFT_CASE
    }
    return launch_generic<T>(c, AXIS, kind, ld, st);
}

template <typename T, class LD, class ST>
int launch_pass(Ctx &c, int axis, int kind, LD ld, ST st)
{
    if (axis == 0) return launch_axis<T, 0>(c, kind, ld, st);
    if (axis == 1) return launch_axis<T, 1>(c, kind, ld, st);
    return launch_axis<T, 2>(c, kind, ld, st);
}

// Element-wise precision conversion (host-psi steps).
template <typename S, typename D>
__global__ void convert_kernel(const S *__restrict__ src, D *__restrict__ dst, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) dst[q] = D(src[q]);
}

template <typename S, typename D>
int convert(Ctx &c, const S *src, D *dst)
{
    convert_kernel<S, D><<<1184, 256, 0, c.stream>>>(src, dst, c.n);
    SMADFT_CUDA(cudaGetLastError());
    c.launches++;
    return SMADFT_OK;
}

// z and y passes of NC components per plane in one launch: one cluster of N / 32 CTAs per
// (plane, component)
template <typename T, int N, int NC, class LD>
int launch_plane(Ctx &c, const PlaneKinds<NC> &kinds, LD ld, const StoreMulti<T, NC> &st)
{
    const PlanDev &pd = c.plans.at(N);
    constexpr size_t smem = plane_smem_bytes<T, N>();
    using ST = StoreMulti<T, NC>;
    static unsigned long long attr_set = 0;   // devices whose attribute is set (bit per device)
    {
        std::lock_guard<std::mutex> lock(attr_mutex());
        if (!(attr_set >> (c.dev % kMaxDevices) & 1ull)) {
            SMADFT_CUDA(cudaFuncSetAttribute(r2r_plane_kernel<T, N, NC, LD, ST>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            attr_set |= 1ull << (c.dev % kMaxDevices);
        }
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)c.g.nx * NC * PlaneInfo<N>::C);
    cfg.blockDim = dim3(RdInfo<N>::THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = c.stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = PlaneInfo<N>::C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    SMADFT_CUDA(cudaLaunchKernelEx(&cfg, r2r_plane_kernel<T, N, NC, LD, ST>, c.g, kinds, ld,
                                   reinterpret_cast<const cpx<T> *>(pd.w), reinterpret_cast<const cpx<T> *>(pd.h), st));
    c.launches++;
    return SMADFT_OK;
}

template <typename T, int NC, class LD>
int launch_plane_n(Ctx &c, const PlaneKinds<NC> &kinds, LD ld, const StoreMulti<T, NC> &st)
{
    switch (c.g.nz) {
    case 64: return launch_plane<T, 64, NC>(c, kinds, ld, st);
    case 128: return launch_plane<T, 128, NC>(c, kinds, ld, st);
    default: return launch_plane<T, 256, NC>(c, kinds, ld, st);
    }
}

inline bool plane_ok(const Ctx &c)
{
    return c.use_plane && c.g.ny == c.g.nz && (c.g.nz == 64 || c.g.nz == 128 || c.g.nz == 256);
}

// 3-D transform with the custom loader in the first pass and the custom storer in the last,
// through the scratch field: for ny = nz in {64, 128, 256} the fused z + y plane kernel then
// the x pass (two sweeps over HBM), otherwise y pass -> z pass -> x pass, all in place on
// the scratch field (the z pass in between only moves the scratch field).
template <typename T, class LD, class ST>
int r2r3d(Ctx &c, int kx, int ky, int kz, LD ld, ST st)
{
    T *tmp = c.f<T>(S_TMP);
    int rc;
    if (plane_ok(c)) {
        rc = launch_plane_n<T, 1>(c, PlaneKinds<1>{{ky}, {kz}}, make_multi(ld), StoreMulti<T, 1>{{tmp}});
        if (rc) return rc;
        return launch_axis<T, 0>(c, kx, LoadArr<T>{tmp}, st);
    }
    rc = launch_axis<T, 1>(c, ky, ld, StoreArr<T>{tmp});
    if (rc) return rc;
    rc = launch_axis<T, 2>(c, kz, LoadArr<T>{tmp}, StoreArr<T>{tmp});
    if (rc) return rc;
    return launch_axis<T, 0>(c, kx, LoadArr<T>{tmp}, st);
}

// Runs fn(m) for m < n on forked streams: each branch starts after the work queued so far
// and the stream continues after all branches.  Under stream capture the branches become
// parallel paths of the graph, so the tails and launch gaps of independent passes overlap.
template <class F>
int forked(Ctx &c, int n, F fn)
{
    if (!c.use_fork || n <= 1 || !c.aux[0] || !c.ev_fork) {
        for (int m = 0; m < n; m++)
            if (int rc = fn(m)) return rc;
        return SMADFT_OK;
    }
    const cudaStream_t main = c.stream;
    cudaError_t e = cudaEventRecord(c.ev_fork, main);
    int rc = SMADFT_OK;
    for (int m = 0; m < n && e == cudaSuccess && rc == SMADFT_OK; m++) {
        const cudaStream_t s = c.aux[m % Ctx::kMaxFork];
        e = cudaStreamWaitEvent(s, c.ev_fork, 0);
        if (e != cudaSuccess) break;
        c.stream = s;
        rc = fn(m);
        c.stream = main;
        e = cudaEventRecord(c.ev_join[m % Ctx::kMaxFork], s);
    }
    // join every branch that was started (also on error, so that a capture can end)
    for (int m = 0; m < n && m < Ctx::kMaxFork; m++) {
        const cudaError_t ej = cudaStreamWaitEvent(main, c.ev_join[m], 0);
        if (e == cudaSuccess) e = ej;
    }
    if (rc) return rc;
    if (e != cudaSuccess) {
        c.err = std::string("forked streams: ") + cudaGetErrorString(e);
        return SMADFT_ERR_CUDA;
    }
    return SMADFT_OK;
}

// ---- batch groups: M members of one model and grid whose fields lie in pools (member i's
// field at the lead's pointer + i n elements).  Their plain axis passes run as one launch over
// the pool; passes with member-specific loaders or storers run per member on the lead's stream.

// `fn` on a copy of the lead context (same stream, plans and launch helpers) whose geometry
// or grid is widened to the whole pool; the copy's launches are counted on the lead
template <class F>
int on_pool_copy(Ctx &lead, F fn)
{
    Ctx pc = lead;
    const int rc = fn(pc);
    lead.launches = pc.launches;
    if (rc) lead.err = pc.err;
    return rc;
}

// one plain axis pass over the pooled fields of M members: z and y passes see the pool as one
// field of M nx planes; x passes run M CTA rows, each addressing its member's field
template <typename T, int AXIS, typename S = T>
int pooled_pass(Ctx &lead, int M, int kind, const S *in, T *out)
{
    return on_pool_copy(lead, [&](Ctx &pc) {
        if constexpr (AXIS == 0) {
            pc.grid_y = M;
            return launch_axis<T, 0>(pc, kind, LoadArrM<T, S>{in, (idx_t)lead.n}, StoreArrM<T>{out, (idx_t)lead.n});
        } else {
            pc.g.nx = lead.g.nx * M;
#ifdef SMADFT_CHECK_BOUNDS
            pc.g.nelem = lead.g.nelem * M;
#endif
            return launch_axis<T, AXIS>(pc, kind, LoadArr<T, S>{in}, StoreArr<T>{out});
        }
    });
}

// the y passes of NC components with loaders ls (one grouped launch where the length has the
// register-direct kernel, else one pass per component), outputs into out[m]
template <typename T, int NC, int DIR, class... L>
int y_pass_multi(Ctx &c, const int (&ky)[NC], T *const (&out)[NC], L... ls)
{
    static_assert(sizeof...(L) == NC, "one loader per component");
    if (c.g.ny == 64 || c.g.ny == 128 || c.g.ny == 256) {
        KindSet<NC> ks;
        StoreMulti<T, NC> sm;
        for (int m = 0; m < NC; m++) {
            ks.k[m] = ky[m];
            sm.p[m] = out[m];
        }
        using LM = decltype(make_multi(ls...));
        using SM = StoreMulti<T, NC>;
        switch (c.g.ny) {
        case 64: return launch_rd<T, 64, 1, LM, SM, NC, DIR>(c, ks, make_multi(ls...), sm);
        case 128: return launch_rd<T, 128, 1, LM, SM, NC, DIR>(c, ks, make_multi(ls...), sm);
        default: return launch_rd<T, 256, 1, LM, SM, NC, DIR>(c, ks, make_multi(ls...), sm);
        }
    }
    int rc = SMADFT_OK, m = 0;
    ((rc = rc ? rc : launch_axis<T, 1>(c, ky[m], ls, StoreArr<T>{out[m]}), m++), ...);
    return rc;
}

// runs fn(member) with the member's launches on the lead's stream
template <class F>
int on_lead_stream(Ctx &lead, Ctx &member, F fn)
{
    const cudaStream_t own = member.stream;
    member.stream = lead.stream;
    const int rc = fn(member);
    member.stream = own;
    return rc;
}

// NC 3-D transforms whose loaders share input fields: component m goes from loader ls[m]
// to field out[m] with kinds (kx[m], ky[m], kz[m]).  Plane path: one plane launch for all
// components (their shared reads meet in L2), then the x pass of each in place; otherwise
// NC separate transforms through the scratch field.
template <typename T, int NC, int DIR = -1, class... L>
int r2r3d_multi(Ctx &c, const int (&kx)[NC], const int (&ky)[NC], const int (&kz)[NC], T *const (&out)[NC], L... ls)
{
    static_assert(sizeof...(L) == NC, "one loader per component");
    if constexpr (DIR >= 0) {   // the stated direction must be every component's
        for (int m = 0; m < NC; m++) {
            const int want = DIR == 1 ? ((kx[m] == K_DCT2 || kx[m] == K_DST2) && (ky[m] == K_DCT2 || ky[m] == K_DST2) &&
                                         (kz[m] == K_DCT2 || kz[m] == K_DST2))
                                      : ((kx[m] == K_DCT3 || kx[m] == K_DST3) && (ky[m] == K_DCT3 || ky[m] == K_DST3) &&
                                         (kz[m] == K_DCT3 || kz[m] == K_DST3));
            if (!want) {
                c.err = "r2r3d_multi: component kinds do not match the stated direction";
                return SMADFT_ERR_INVALID;
            }
        }
    }
    int rc = SMADFT_OK;
    if (plane_ok(c)) {
        PlaneKinds<NC> pk;
        StoreMulti<T, NC> sm;
        for (int m = 0; m < NC; m++) {
            pk.ky[m] = ky[m];
            pk.kz[m] = kz[m];
            sm.p[m] = out[m];
        }
        if ((rc = launch_plane_n<T, NC>(c, pk, make_multi(ls...), sm))) return rc;
        return forked(c, NC, [&](int m) { return launch_axis<T, 0>(c, kx[m], LoadArr<T>{out[m]}, StoreArr<T>{out[m]}); });
    }
    if (c.use_rd && c.use_multi && (c.g.ny == 64 || c.g.ny == 128 || c.g.ny == 256)) {
        // y pass of all components in one register-direct launch (their shared reads meet
        // in L2), then the z and x passes of each in place
        KindSet<NC> ks;
        StoreMulti<T, NC> sm;
        for (int m = 0; m < NC; m++) {
            ks.k[m] = ky[m];
            sm.p[m] = out[m];
        }
        using LM = decltype(make_multi(ls...));
        using SM = StoreMulti<T, NC>;
        switch (c.g.ny) {
        case 64: rc = launch_rd<T, 64, 1, LM, SM, NC, DIR>(c, ks, make_multi(ls...), sm); break;
        case 128: rc = launch_rd<T, 128, 1, LM, SM, NC, DIR>(c, ks, make_multi(ls...), sm); break;
        default: rc = launch_rd<T, 256, 1, LM, SM, NC, DIR>(c, ks, make_multi(ls...), sm); break;
        }
        if (rc) return rc;
        return forked(c, NC, [&](int m) {
            const int r = launch_axis<T, 2>(c, kz[m], LoadArr<T>{out[m]}, StoreArr<T>{out[m]});
            return r ? r : launch_axis<T, 0>(c, kx[m], LoadArr<T>{out[m]}, StoreArr<T>{out[m]});
        });
    }
    int m = 0;
    ((rc = rc ? rc : r2r3d<T>(c, kx[m], ky[m], kz[m], ls, StoreArr<T>{out[m]}), m++), ...);
    return rc;
}

}  // namespace smadft
