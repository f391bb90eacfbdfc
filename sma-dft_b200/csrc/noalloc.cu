// noalloc.cu -- smadft_r2r3d_noalloc: the 3-D r2r transform of smadft_r2r3d_device for
// callers that cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not an option -- inside a stream
// callback or host function enqueued with cudaLaunchHostFunc (CUDA calls are not allowed
// there), in applications whose device memory is fully reserved up front by another
// allocator (a framework's caching pool, an MPI+CUDA code that carved HBM at start-up), or
// in fixed-latency loops that must not call cudaMalloc after start-up because it can
// synchronise the device and take unbounded time.  This entry point needs no context, no
// allocation of any kind (device or host heap): the intermediate field between the axis
// passes lives in a file-scope __device__ array, and so do the twiddle tables.
//
// Limits and sharing rules:
//   * nx*ny*nz*sizeof(element) <= SMADFT_NOALLOC_MAX_BYTES (16 MiB: 128^3 doubles,
//     2^22 floats); each length even, at most 512, prime factors 2, 3, 5 only.
//   * Every GPU that loads the library holds the 16 MiB array (plus 48 KiB of twiddles)
//     until the process exits.
//   * All calls share the array, which keeps the last call's contents.  Every element a
//     call reads from it was written earlier by the same call, so nothing needs clearing;
//     but calls that overlap on the GPU (different streams, or other host threads on the
//     same device) race on it.
//   * The first call on each device looks the array up with cudaGetSymbolAddress while
//     that device is current; make that first call before any stream capture.
//   * The work is queued on `stream` and the call returns without waiting for it.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>

#include "r2r_fast.cuh"
#include "r2r_pass.cuh"
#include "smadft.h"

namespace {

using namespace smadft;

constexpr int kNaMaxLine = 512;
constexpr int kNaMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[SMADFT_NOALLOC_MAX_BYTES];
// per axis: w[kNaMaxLine] then h[kNaMaxLine] complex doubles (floats use the first half)
static __device__ __align__(256) unsigned char g_noalloc_twiddles[3 * 2 * kNaMaxLine * 16];

struct NaDevice {
    bool ready = false;
    unsigned char *scratch = nullptr;
    unsigned char *twiddles = nullptr;
};
NaDevice g_na[kNaMaxDevices];
std::mutex g_na_mu;

// Device addresses of the static arrays for the current device (looked up once per device).
int na_setup(NaDevice **out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
        cudaGetLastError();
        return SMADFT_ERR_NODEVICE;
    }
    if (dev >= kNaMaxDevices) return SMADFT_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_na_mu);
    NaDevice &d = g_na[dev];
    if (!d.ready) {
        void *s = nullptr, *t = nullptr;
        if (cudaGetSymbolAddress(&s, g_noalloc_scratch) != cudaSuccess ||
            cudaGetSymbolAddress(&t, g_noalloc_twiddles) != cudaSuccess) {
            cudaGetLastError();
            return SMADFT_ERR_CUDA;
        }
        d.scratch = static_cast<unsigned char *>(s);
        d.twiddles = static_cast<unsigned char *>(t);
        d.ready = true;
    }
    *out = &d;
    return SMADFT_OK;
}

bool na_len_ok(int n)
{
    if (n < 4 || n > kNaMaxLine || (n & 1)) return false;
    while (n % 2 == 0) n /= 2;
    while (n % 3 == 0) n /= 3;
    while (n % 5 == 0) n /= 5;
    return n == 1;
}

template <typename T>
struct NaAxis {
    int n;
    LinePlan<T> plan;   // radices + device twiddle pointers into g_noalloc_twiddles
};

template <typename T>
void na_plan(int n, unsigned char *tw_dev, NaAxis<T> &ax, cpx<T> *host_w, cpx<T> *host_h)
{
    ax.n = n;
    ax.plan.n = n;
    int m = n, s = 0;
    while (m % 4 == 0) { ax.plan.radix[s++] = 4; m /= 4; }
    while (m % 2 == 0) { ax.plan.radix[s++] = 2; m /= 2; }
    while (m % 3 == 0) { ax.plan.radix[s++] = 3; m /= 3; }
    while (m % 5 == 0) { ax.plan.radix[s++] = 5; m /= 5; }
    ax.plan.nst = s;
    for (; s < kMaxStages; s++) ax.plan.radix[s] = 1;
    for (int k = 0; k < n; k++) {
        const double a = 2.0 * M_PI * (double)k / (double)n;
        host_w[k] = {T(std::cos(a)), T(-std::sin(a))};
        const double b = M_PI * (double)k / (2.0 * (double)n);
        host_h[k] = {T(std::cos(b)), T(std::sin(b))};
    }
    ax.plan.w = reinterpret_cast<const cpx<T> *>(tw_dev);
    ax.plan.h = reinterpret_cast<const cpx<T> *>(tw_dev) + kNaMaxLine;
}

template <typename T>
constexpr int na_tile_w() { return sizeof(T) == 4 ? 32 : 16; }

template <typename T, int AXIS>
cudaError_t na_pass(const Geom &g, const NaAxis<T> &ax, int kind, const T *in, T *out, cudaStream_t st)
{
    LoadArr<T> ld{in};
    StoreArr<T> sv{out};
    const int W = kFastW;
    int tiles_b = 1;
    long long tiles;
    if (AXIS == 2) tiles = ((long long)g.nx * g.ny + W - 1) / W;
    else {
        tiles_b = (g.nz + W - 1) / W;
        tiles = (long long)(AXIS == 1 ? g.nx : g.ny) * tiles_b;
    }
    switch (ax.n) {
#define SMADFT_NA_CASE(N_)                                                                          \
    case N_: {                                                                                      \
        constexpr size_t smem = fast_smem_bytes<T, N_>();                                           \
        cudaError_t e = cudaFuncSetAttribute(r2r_fast_kernel<T, N_, AXIS, LoadArr<T>, StoreArr<T>>,  \
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
        if (e != cudaSuccess) return e;                                                             \
        r2r_fast_kernel<T, N_, AXIS, LoadArr<T>, StoreArr<T>><<<(unsigned)tiles, kFastThreads, smem, st>>>( \
            g, kind, tiles_b, ax.plan.w, ax.plan.h, ld, sv);                                        \
        return cudaGetLastError();                                                                  \
    }
        SMADFT_NA_CASE(64)
        SMADFT_NA_CASE(96)
        SMADFT_NA_CASE(128)
#undef SMADFT_NA_CASE
    default: break;
    }
    PassArgs<T> a;
    a.g = g;
    a.axis = AXIS;
    a.kind = kind;
    a.W = na_tile_w<T>();
    a.ld = ax.n;
    a.P = ax.plan;
    if (AXIS == 2) {
        a.tiles_b = 1;
        tiles = ((long long)g.nx * g.ny + a.W - 1) / a.W;
    } else {
        a.tiles_b = (g.nz + a.W - 1) / a.W;
        tiles = (long long)(AXIS == 1 ? g.nx : g.ny) * a.tiles_b;
    }
    const size_t smem = 2 * (size_t)(a.W / 2) * a.ld * sizeof(cpx<T>);
    cudaError_t e = cudaFuncSetAttribute(r2r_pass_kernel<T, LoadArr<T>, StoreArr<T>>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    r2r_pass_kernel<T, LoadArr<T>, StoreArr<T>><<<(unsigned)tiles, 256, smem, st>>>(a, ld, sv);
    return cudaGetLastError();
}

template <typename T>
int na_transform(const Geom &g, const T *in, T *out, int kx, int ky, int kz, cudaStream_t st, NaDevice &d)
{
    // host twiddles on the stack (no heap), uploaded into the static device tables
    cpx<T> hw[3][kNaMaxLine], hh[3][kNaMaxLine];
    NaAxis<T> ax[3];
    const int lens[3] = {g.nx, g.ny, g.nz};
    for (int a = 0; a < 3; a++) {
        unsigned char *tw = d.twiddles + (size_t)a * 2 * kNaMaxLine * 16;
        na_plan<T>(lens[a], tw, ax[a], hw[a], hh[a]);
        if (cudaMemcpyAsync(tw, hw[a], sizeof(cpx<T>) * lens[a], cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(tw + sizeof(cpx<T>) * kNaMaxLine, hh[a], sizeof(cpx<T>) * lens[a],
                            cudaMemcpyHostToDevice, st) != cudaSuccess) {
            cudaGetLastError();
            return SMADFT_ERR_CUDA;
        }
    }
    T *tmp = reinterpret_cast<T *>(d.scratch);
    if (na_pass<T, 2>(g, ax[2], kz, in, tmp, st) != cudaSuccess ||
        na_pass<T, 1>(g, ax[1], ky, tmp, tmp, st) != cudaSuccess ||
        na_pass<T, 0>(g, ax[0], kx, tmp, out, st) != cudaSuccess) {
        cudaGetLastError();
        return SMADFT_ERR_CUDA;
    }
    // copies from pageable host memory are staged before cudaMemcpyAsync returns, so the
    // stack twiddle arrays may go out of scope while the work is still queued
    return SMADFT_OK;
}

}  // namespace

extern "C" int smadft_r2r3d_noalloc(const void *in, void *out, int nx, int ny, int nz, int kx, int ky, int kz,
                                    int precision, void *stream)
{
    if (!in || !out) return SMADFT_ERR_INVALID;
    if (precision != SMADFT_FP64 && precision != SMADFT_FP32) return SMADFT_ERR_INVALID;
    for (int k : {kx, ky, kz})
        if (k < 0 || k > 3) return SMADFT_ERR_INVALID;
    if (((uintptr_t)in | (uintptr_t)out) & 15) return SMADFT_ERR_INVALID;
    if (!na_len_ok(nx) || !na_len_ok(ny) || !na_len_ok(nz)) return SMADFT_ERR_UNSUPPORTED;
    const size_t es = precision == SMADFT_FP64 ? 8 : 4;
    if ((size_t)nx * ny * nz * es > (size_t)SMADFT_NOALLOC_MAX_BYTES) return SMADFT_ERR_TOO_LARGE;
    NaDevice *d = nullptr;
    int rc = na_setup(&d);
    if (rc) return rc;
    Geom g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.nyz = (long long)ny * nz;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precision == SMADFT_FP64)
        return na_transform<double>(g, static_cast<const double *>(in), static_cast<double *>(out), kx, ky, kz, st, *d);
    return na_transform<float>(g, static_cast<const float *>(in), static_cast<float *>(out), kx, ky, kz, st, *d);
}
