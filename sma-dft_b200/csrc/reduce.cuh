// reduce.cuh -- FP64 diagnostics: deterministic two-level reductions and the interface
// tracker.
//
// Sums (L1, mass, energy, mean) accumulate in double whatever the field precision: each
// block reduces a fixed, grid-strided slice in a fixed order, writes one partial per
// value, and a single block adds the partials in index order.  The result is bit
// reproducible run to run.  Reference sums: no-adv/cosNoAdvTrackSing.cpp:775-789,
// adv/cosAdvTrackMult.cpp:1377-1404, quasi/quasi.cpp:2197-2251.
#pragma once

#include "ctx.cuh"

namespace smadft {

constexpr int kRedThreads = 256;
constexpr int kRedVals = 4;

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

template <class F>
__global__ void __launch_bounds__(kRedThreads) reduce_partials(long long n, F f, double *partials)
{
    double acc[kRedVals] = {0.0, 0.0, 0.0, 0.0};
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) f(q, acc);
    __shared__ double sh[kRedVals][kRedThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < kRedVals; v++) {
        double s = warp_sum(acc[v]);
        if (lane == 0) sh[v][wid] = s;
    }
    __syncthreads();
    if (threadIdx.x < kRedVals) {
        double s = 0.0;
        for (int w = 0; w < kRedThreads / 32; w++) s += sh[threadIdx.x][w];
        partials[(long long)blockIdx.x * kRedVals + threadIdx.x] = s;
    }
}

static __global__ void reduce_final(const double *partials, int nblocks, double *out)
{
    // one warp per value, fixed order
    const int v = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (v >= kRedVals) return;
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32) s += partials[(long long)b * kRedVals + v];
    s = warp_sum(s);
    if (lane == 0) out[v] = s;
}

inline int reduce_init(Ctx &c)
{
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.dev);
    c.red_blocks = sms * 4;
    SMADFT_CUDA(cudaMalloc(&c.red, sizeof(double) * kRedVals * c.red_blocks));
    SMADFT_CUDA(cudaMalloc(&c.red_out, sizeof(double) * kRedVals));
    return SMADFT_OK;
}

template <class F>
int run_reduce(Ctx &c, F f, double *host_out)
{
    reduce_partials<F><<<c.red_blocks, kRedThreads, 0, c.stream>>>(c.n, f, c.red);
    SMADFT_CUDA(cudaGetLastError());
    reduce_final<<<1, 32 * kRedVals, 0, c.stream>>>(c.red, c.red_blocks, c.red_out);
    SMADFT_CUDA(cudaGetLastError());
    c.launches += 2;
    SMADFT_CUDA(cudaMemcpyAsync(host_out, c.red_out, sizeof(double) * kRedVals, cudaMemcpyDeviceToHost,
                                c.stream));
    SMADFT_CUDA(cudaStreamSynchronize(c.stream));
    return SMADFT_OK;
}

// acc: sum|new-old|, sum|new|, sum new, count of non-finite new
template <typename T>
struct RedL1 {
    const T *__restrict__ nw, *__restrict__ od;
    __device__ __forceinline__ void operator()(long long q, double *acc) const
    {
        double a = (double)nw[q], b = (double)od[q];
        acc[0] += fabs(a - b);
        acc[1] += fabs(a);
        acc[2] += a;
        acc[3] += isfinite(a) ? 0.0 : 1.0;
    }
};

template <typename T>
int reduce_l1(Ctx &c, const T *nw, const T *od, double *out)
{
    return run_reduce(c, RedL1<T>{nw, od}, out);
}

// e = -eps/2 psi^2 + 1/2 f'^2 - beta/4 psi^4 + gamma/6 psi^6 (quasi/quasi.cpp:1470-1473), FP64
template <typename T>
struct RedEnergy {
    const T *__restrict__ psi, *__restrict__ fp;
    double eps, beta, gamma;
    __device__ __forceinline__ void operator()(long long q, double *acc) const
    {
        double p = (double)psi[q], f = (double)fp[q];
        double p2 = p * p;
        acc[0] += -0.5 * eps * p2 + 0.5 * f * f - 0.25 * beta * p2 * p2 + (gamma / 6) * p2 * p2 * p2;
    }
};

template <typename T>
int reduce_energy(Ctx &c, const T *psi, const T *fp, double *e)
{
    double out[kRedVals];
    int rc = run_reduce(c, RedEnergy<T>{psi, fp, c.p.eps, c.p.beta, c.p.gamma}, out);
    *e = out[0];
    return rc;
}

template <typename T>
struct RedSum2 {
    const T *__restrict__ a, *__restrict__ b;
    __device__ __forceinline__ void operator()(long long q, double *acc) const
    {
        acc[0] += (double)a[q];
        acc[1] += (double)b[q];
    }
};

// ---------------------------------------------------------------- tracker --------------
// One thread per column; the scan runs from the last index of `axis` down, as the
// reference scans k.  Modes: see SMADFT_TRACK_* in smadft.h.
template <typename T>
__global__ void track_kernel(const T *__restrict__ f, int na, int nb, int nl, long long sa, long long sb,
                             long long sl, int mode, double hi, double lo, int *idx, double *pos)
{
    const long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= (long long)na * nb) return;
    const int a = (int)(col / nb), b = (int)(col % nb);
    const T *cp = f + a * sa + b * sb;
    auto V = [&](int t) -> double { return (double)cp[(long long)t * sl]; };
    int found = -1;
    double ps = nan("");
    if (mode == SMADFT_TRACK_FLAT) {
        int track = 0;
        for (int t = nl - 1; t >= 0; t--) {
            double v = V(t);
            if (v > hi && track == 0) track = 1;
            if (v < lo && track == 1) {
                if (t + 1 >= nl) break;
                double v1 = V(t + 1);
                found = (fabs(v) > fabs(v1)) ? t + 1 : t;
                ps = t + (lo - v) / (v1 - v);
                break;
            }
        }
    } else if (mode == SMADFT_TRACK_BUMP) {
        for (int t = nl - 1; t >= 0; t--) {
            if (fabs(V(t)) > hi) {
                int t3 = t;
                while (t3 < nl - 1 && fabs(V(t3)) > lo) t3++;
                found = (t3 + 1 < nl && fabs(V(t3)) > fabs(V(t3 + 1))) ? t3 + 1 : t3;
                if (t3 > t) {
                    double f0 = fabs(V(t3 - 1)), f1 = fabs(V(t3));
                    ps = (t3 - 1) + (f0 - lo) / (f0 - f1);
                } else {
                    ps = (double)t3;
                }
                break;
            }
        }
    } else {
        for (int t = nl - 1; t >= 0; t--) {
            double v = V(t);
            if (v > hi) {
                found = t;
                if (t + 1 < nl) {
                    double v1 = V(t + 1);
                    ps = t + (v - hi) / (v - v1);
                } else {
                    ps = (double)t;
                }
                break;
            }
        }
    }
    idx[col] = found;
    pos[col] = ps;
}

template <typename T>
int track_columns(Ctx &c, const T *f, int axis, int mode, double hi, double lo, int *hidx, double *hpos)
{
    int na, nb, nl;
    long long sa, sb, sl;
    const Geom &g = c.g;
    if (axis == 2) { na = g.nx; nb = g.ny; nl = g.nz; sa = g.nyz; sb = g.nz; sl = 1; }
    else if (axis == 1) { na = g.nx; nb = g.nz; nl = g.ny; sa = g.nyz; sb = 1; sl = g.nz; }
    else { na = g.ny; nb = g.nz; nl = g.nx; sa = g.nz; sb = 1; sl = g.nyz; }
    const long long ncol = (long long)na * nb;
    int *didx = nullptr;
    double *dpos = nullptr;
    SMADFT_CUDA(cudaMallocAsync(&didx, sizeof(int) * ncol, c.stream));
    SMADFT_CUDA(cudaMallocAsync(&dpos, sizeof(double) * ncol, c.stream));
    track_kernel<T><<<(unsigned)((ncol + 255) / 256), 256, 0, c.stream>>>(f, na, nb, nl, sa, sb, sl, mode, hi,
                                                                         lo, didx, dpos);
    SMADFT_CUDA(cudaGetLastError());
    c.launches++;
    SMADFT_CUDA(cudaMemcpyAsync(hidx, didx, sizeof(int) * ncol, cudaMemcpyDeviceToHost, c.stream));
    SMADFT_CUDA(cudaMemcpyAsync(hpos, dpos, sizeof(double) * ncol, cudaMemcpyDeviceToHost, c.stream));
    SMADFT_CUDA(cudaFreeAsync(didx, c.stream));
    SMADFT_CUDA(cudaFreeAsync(dpos, c.stream));
    SMADFT_CUDA(cudaStreamSynchronize(c.stream));
    return SMADFT_OK;
}

}  // namespace smadft
