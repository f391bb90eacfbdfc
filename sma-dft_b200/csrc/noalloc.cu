// noalloc.cu -- smadft_r2r3d_noalloc: the 3-D r2r transform of smadft_r2r3d_device for
// callers that cannot allocate device memory.
//
// Who needs it: applications whose device memory is fully reserved up front by another
// allocator (a framework's caching pool, an MPI+CUDA code that carved HBM at start-up), so
// that a cudaMalloc would fail, and fixed-latency loops that must not call cudaMalloc after
// start-up because it can synchronise the device and take unbounded time.  This entry point
// needs no context and allocates nothing, on the device or on the host heap: the
// intermediate field between the axis passes lives in a file-scope __device__ array, and so
// do the twiddle tables, which a small kernel fills on the caller's stream (no host copies).
// It is still an ordinary CUDA host API call (it queries the device and launches kernels),
// so it may not be called from a stream callback or a cudaLaunchHostFunc host function,
// where CUDA calls are not allowed.
//
// Limits and sharing rules:
//   * nx*ny*nz*sizeof(element) <= SMADFT_NOALLOC_MAX_BYTES (16 MiB: 128^3 doubles,
//     2^22 floats); each length even, at most 512, prime factors 2, 3, 5 only.
//   * Every GPU that loads the library holds the 16 MiB array (plus 48 KiB of twiddles)
//     until the process exits.
//   * All calls share the scratch array and the twiddle tables, which keep the last call's
//     contents.  Every element a call reads from them was written earlier by the same call,
//     so nothing needs clearing; but calls that overlap on the GPU (different streams, or
//     other host threads on the same device) race on both.
//   * The first call on each device looks the arrays up with cudaGetSymbolAddress while
//     that device is current and sets the kernels' shared-memory attributes; make that
//     first call before any stream capture.
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
int na_setup(NaDevice **out, int *dev_out)
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
    *dev_out = dev;
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

// Twiddle tables of the three axes, computed on the device from the lengths alone:
// w[k] = exp(-2 pi i k / n), h[k] = exp(+i pi k / (2 n)) (the layout LinePlan expects).  One
// block per axis, FP64 angles through sincospi, queued on the caller's stream.
template <typename T>
__global__ void na_twiddle_kernel(unsigned char *tw, int nx, int ny, int nz)
{
    const int a = blockIdx.x;
    const int n = a == 0 ? nx : (a == 1 ? ny : nz);
    cpx<T> *w = reinterpret_cast<cpx<T> *>(tw + (size_t)a * 2 * kNaMaxLine * 16);
    cpx<T> *h = w + kNaMaxLine;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)k / (double)n, &s, &c);
        w[k] = {T(c), T(-s)};
        sincospi((double)k / (2.0 * (double)n), &s, &c);
        h[k] = {T(c), T(s)};
    }
}

// Kernel attributes (dynamic shared memory opt-in) are per device: one flag per device and
// instantiation, set on the first call under a lock.
template <class K>
cudaError_t na_smem_attr(K *kern, size_t smem, int dev, unsigned long long &mask)
{
    std::lock_guard<std::mutex> lock(g_na_mu);
    if (mask >> dev & 1ull) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) mask |= 1ull << dev;
    return e;
}

template <typename T>
void na_plan(int n, unsigned char *tw_dev, NaAxis<T> &ax)
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
    ax.plan.w = reinterpret_cast<const cpx<T> *>(tw_dev);
    ax.plan.h = reinterpret_cast<const cpx<T> *>(tw_dev) + kNaMaxLine;
}

template <typename T>
constexpr int na_tile_w() { return sizeof(T) == 4 ? 32 : 16; }

template <typename T, int AXIS>
cudaError_t na_pass(const Geom &g, const NaAxis<T> &ax, int kind, const T *in, T *out, cudaStream_t st, int dev)
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
        static unsigned long long mask_ = 0;                                                        \
        cudaError_t e = na_smem_attr(r2r_fast_kernel<T, N_, AXIS, LoadArr<T>, StoreArr<T>>, smem, dev, mask_); \
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
    // the generic kernel's opt-in is sized for the longest line (one flag per device)
    const size_t smem = 2 * (size_t)(a.W / 2) * a.ld * sizeof(cpx<T>);
    static unsigned long long mask = 0;
    cudaError_t e = na_smem_attr(r2r_pass_kernel<T, LoadArr<T>, StoreArr<T>>,
                                 2 * (size_t)(a.W / 2) * kNaMaxLine * sizeof(cpx<T>), dev, mask);
    if (e != cudaSuccess) return e;
    r2r_pass_kernel<T, LoadArr<T>, StoreArr<T>><<<(unsigned)tiles, 256, smem, st>>>(a, ld, sv);
    return cudaGetLastError();
}

template <typename T>
int na_transform(const Geom &g, const T *in, T *out, int kx, int ky, int kz, cudaStream_t st, NaDevice &d, int dev)
{
    NaAxis<T> ax[3];
    const int lens[3] = {g.nx, g.ny, g.nz};
    for (int a = 0; a < 3; a++) na_plan<T>(lens[a], d.twiddles + (size_t)a * 2 * kNaMaxLine * 16, ax[a]);
    na_twiddle_kernel<T><<<3, 256, 0, st>>>(d.twiddles, g.nx, g.ny, g.nz);
    if (cudaGetLastError() != cudaSuccess) return SMADFT_ERR_CUDA;
    T *tmp = reinterpret_cast<T *>(d.scratch);
    if (na_pass<T, 2>(g, ax[2], kz, in, tmp, st, dev) != cudaSuccess ||
        na_pass<T, 1>(g, ax[1], ky, tmp, tmp, st, dev) != cudaSuccess ||
        na_pass<T, 0>(g, ax[0], kx, tmp, out, st, dev) != cudaSuccess) {
        cudaGetLastError();
        return SMADFT_ERR_CUDA;
    }
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
    int dev = 0;
    int rc = na_setup(&d, &dev);
    if (rc) return rc;
    Geom g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.nyz = (long long)ny * nz;
#ifdef SMADFT_CHECK_BOUNDS
    g.nelem = (long long)nx * ny * nz;
#endif
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precision == SMADFT_FP64)
        return na_transform<double>(g, static_cast<const double *>(in), static_cast<double *>(out), kx, ky, kz, st, *d, dev);
    return na_transform<float>(g, static_cast<const float *>(in), static_cast<float *>(out), kx, ky, kz, st, *d, dev);
}
