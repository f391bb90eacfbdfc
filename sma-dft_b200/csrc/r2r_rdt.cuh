// r2r_rdt.cuh -- register-direct strided axis pass (x, y) fed by TMA: a persistent CTA walks
// its tiles (32 k-columns x N points along the axis) with the next tiles' inputs already in
// flight, so the pass keeps HBM busy between the load phases of the plain r2r_rd_kernel.
//
// Tiles are the r2r_rd_kernel's: thread (c, j) owns first-stage butterfly j of complex line c
// (real k-columns 2c, 2c+1).  Here the tile's inputs arrive by cp.async.bulk.tensor into a
// two-stage shared-memory ring ([N points][32 columns], 128-byte rows), issued two tiles
// ahead by one thread on an mbarrier per stage; each thread then picks its R0 stage-0 points
// from shared memory (a half-warp reads one 128-byte row), and the transform (rd_fft) and the
// stores through the Storer are those of r2r_rd_kernel.  The loader is a plain array of the
// source type S (FP32 fields, or the FP64 spectral state read as FP32); any Storer works.
// Every wait on a stage barrier is bounded; a wait that runs out records the error word and
// the CTA stops after draining its own copies in flight.
#pragma once

#include <cuda.h>

#include "r2r_rd.cuh"

namespace smadft {

constexpr int kRdtStages = 2;
constexpr long long kRdtWaitCycles = 4000000000ll;   // about 2 s at the B200's clocks

template <typename S, int N>
constexpr size_t rdt_stage_bytes() { return (size_t)N * 32 * sizeof(S); }

// stages first (1024-byte aligned), then the exchange buffer and twiddles of r2r_rd_kernel,
// then the barriers and the abort flag
template <typename T, typename S, int N>
constexpr size_t rdt_smem_bytes()
{
    return 1024 + kRdtStages * rdt_stage_bytes<S, N>() + rd_smem_bytes<T, N>() + 64;
}

__device__ __forceinline__ uint32_t rdt_smem(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool rdt_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// tile `t` of the pass: box {32 columns, 1, N} (x) or {32, N, 1} (y) of the 3-D map
template <int AXIS>
__device__ __forceinline__ void rdt_issue(const CUtensorMap *map, uint32_t dst, uint32_t bar, uint32_t bytes, int tile,
                                          int tiles_b)
{
    const int kt = tile % tiles_b, a = tile / tiles_b;
    const int x = kt * 32, y = AXIS == 1 ? 0 : a, z = AXIS == 1 ? a : 0;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

// One plain strided pass (source type S, transform in T, kind KIND >= 0 or kind_rt) over
// `tiles` tiles of tiles_b k-blocks each; the storer gets the tile's output points.
template <typename T, typename S, int N, int AXIS, class ST, int KIND>
__global__ void __launch_bounds__(RdInfo<N>::THREADS, 2)
    r2r_rdt_kernel(const __grid_constant__ CUtensorMap map, Geom g, int kind_rt, int tiles, int tiles_b,
                   const cpx<T> *__restrict__ wt_g, const cpx<T> *__restrict__ ht_g, ST st, int *err)
{
    using RI = RdInfo<N>;
    constexpr int R0 = RI::R0, R1 = RI::R1, NT = RI::THREADS;
    constexpr int BPT = R0 / R1 > 0 ? R0 / R1 : 1;
    constexpr int NP = BPT * R1;
    constexpr uint32_t SB = (uint32_t)rdt_stage_bytes<S, N>();
    extern __shared__ __align__(16) unsigned char rdt_raw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>(((uintptr_t)rdt_raw + 1023) & ~(uintptr_t)1023);
    const S *stage = reinterpret_cast<const S *>(sm);
    cpx<T> *buf = reinterpret_cast<cpx<T> *>(sm + kRdtStages * SB);
    cpx<T> *wt = buf + kRdLines * RI::LD;
    cpx<T> *ht = wt + N;
    unsigned char *misc = reinterpret_cast<unsigned char *>(ht + N);
    const uint32_t bar0 = rdt_smem(misc);                 // kRdtStages barriers, 8 bytes each
    volatile int *abort = reinterpret_cast<volatile int *>(misc + 8 * kRdtStages);

    const int my_tiles = (tiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kRdtStages; s++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0 + 8u * s) : "memory");
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    for (int m = threadIdx.x; m < N; m += NT) {
        wt[m] = wt_g[m];
        ht[m] = ht_g[m];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int it = 0; it < kRdtStages && it < my_tiles; it++)
            rdt_issue<AXIS>(&map, rdt_smem(sm + it * SB), bar0 + 8u * it, SB, (int)blockIdx.x + it * (int)gridDim.x,
                            tiles_b);
    }

    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5, hh16 = lane >> 4;
    const int c = lane & 15;
    const int j = (wi == 0) ? (hh16 ? R1 / 2 : 0) : (hh16 ? R1 - wi : wi);
    const int kind = KIND >= 0 ? KIND : kind_rt;
    const bool fwd = (kind == K_DCT2 || kind == K_DST2);
    const bool sine = (kind == K_DST2 || kind == K_DST3);
    const RdPos<N> pos(j, fwd, sine);
    const idx_t stride = AXIS == 1 ? g.nz : g.nyz;

    int it = 0;
    for (; it < my_tiles; it++) {
        const int tile = (int)blockIdx.x + it * (int)gridDim.x;
        const int s = it % kRdtStages;
        // this tile's inputs (bounded wait; the whole CTA agrees on giving up)
        {
            const long long t0 = clock64();
            while (!rdt_try_wait(bar0 + 8u * s, (uint32_t)((it / kRdtStages) & 1))) {
                if (*abort) break;
                if (clock64() - t0 > kRdtWaitCycles) {
                    *abort = 1;
                    atomicCAS(err, 0, 16 + AXIS);
                    break;
                }
            }
        }
        const int kt = tile % tiles_b, a = tile / tiles_b;
        const int k = kt * 32 + 2 * c;
        const idx_t base = (AXIS == 1 ? a * g.nyz : a * g.nz) + k;
        const int nk = g.nz - k;
        const bool full = (kt + 1) * 32 <= g.nz;
        cpx<T> v[R0];
        const S *stg = stage + (size_t)s * (SB / sizeof(S));
#pragma unroll
        for (int q = 0; q < R0; q++) {
            // columns 2c, 2c+1 of point row src(q): a half-warp reads one 128-byte row
            if constexpr (sizeof(S) == 4) {
                const float2 e = *reinterpret_cast<const float2 *>(stg + pos.src(q) * 32 + 2 * c);
                v[q] = {T(e.x), T(e.y)};
            } else {
                const double2 e = *reinterpret_cast<const double2 *>(stg + pos.src(q) * 32 + 2 * c);
                v[q] = {T(e.x), T(e.y)};
            }
        }
        __syncthreads();   // every thread has its points: the stage may be refilled
        if (*abort) break;
        if (threadIdx.x == 0 && it + kRdtStages < my_tiles) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            rdt_issue<AXIS>(&map, rdt_smem(sm + s * SB), bar0 + 8u * s, SB,
                            (int)blockIdx.x + (it + kRdtStages) * (int)gridDim.x, tiles_b);
        }
        if (fwd && sine) {   // DST-II negates odd natural samples (the upper half in Makhoul order)
#pragma unroll
            for (int q = 0; q < R0; q++)
                if (!RdPos<N>::src_lo(q)) v[q] = {-v[q].x, -v[q].y};
        }
        cpx<T> x1[BPT][R1];
        rd_fft<T, N>(v, x1, buf + c * RI::LD, wt, ht, j, wi, fwd, sine);

        const idx_t olo = base + pos.olb * stride, dolo = pos.ols * stride;
        const idx_t ohi = base + pos.ohb * stride, dohi = pos.ohs * stride;
        auto out_idx = [&](int pnt) -> idx_t {
            constexpr int H = N / 2;
            const int C = RdPos<N>::cpos(pnt);
            return C < H ? olo + C * dolo : ohi + C * dohi;
        };
        constexpr int CH = 4;
        constexpr int PL = pre_len<ST, 2>();
        using PB = pre_t<ST, T>;
        auto put = [&](int pnt, bool edge, const PB *pre_buf) {
            const cpx<T> z = x1[pnt / R1][pnt % R1];
            const int o = pos.out(pnt);
            const idx_t q = out_idx(pnt);
            const int ii = AXIS == 1 ? a : o, jj = AXIS == 1 ? o : a;
            const T w2[2] = {z.x, z.y};
            if (!edge || nk >= 2) {
                if (idx_ok(g, q, 2)) fin_c<2>(st, 0, q, ii, jj, k, w2, pre_buf);
            } else if (nk == 1) {
                if (idx_ok(g, q)) store_c<1>(st, 0, q, ii, jj, k, w2);
            }
        };
        if (full) {
#pragma unroll
            for (int p0 = 0; p0 < NP; p0 += CH) {
                PB pre_buf[CH][PL];
#pragma unroll
                for (int u = 0; u < CH; u++) {
                    const int o = pos.out(p0 + u);
                    if (idx_ok(g, out_idx(p0 + u), 2))
                    pre_c<2>(st, 0, out_idx(p0 + u), AXIS == 1 ? a : o, AXIS == 1 ? o : a, k, pre_buf[u]);
                }
#pragma unroll
                for (int u = 0; u < CH; u++) put(p0 + u, false, pre_buf[u]);
            }
        } else {
#pragma unroll
            for (int p0 = 0; p0 < NP; p0++) {
                PB pre_buf[PL];
                const int o = pos.out(p0);
                if (nk >= 2 && idx_ok(g, out_idx(p0), 2)) pre_c<2>(st, 0, out_idx(p0), AXIS == 1 ? a : o, AXIS == 1 ? o : a, k, pre_buf);
                put(p0, true, pre_buf);
            }
        }
    }
    // drain: copies this CTA issued whose stage it did not finish (a wait gave up) land before
    // it ends (bounded); after the last tile nothing is in flight
    if (threadIdx.x == 0) {
        for (int r = it; r < my_tiles && r < it + kRdtStages; r++) {
            const long long t0 = clock64();
            while (!rdt_try_wait(bar0 + 8u * (r % kRdtStages), (uint32_t)((r / kRdtStages) & 1)) &&
                   clock64() - t0 < kRdtWaitCycles) {
            }
        }
    }
    __syncthreads();
}

}  // namespace smadft
