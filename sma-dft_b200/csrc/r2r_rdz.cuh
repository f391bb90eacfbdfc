// r2r_rdz.cuh -- register-direct axis pass along z (the contiguous axis) for the
// two-stage plans of r2r_rd.cuh (N = R0 x R1: 64 = 8x8, 128 = 16x8, 256 = 16x16).
//
// The strided kernel puts 16 lines on the lanes of a half-warp so that one access covers
// 128 contiguous bytes.  Along z a line is itself contiguous, so here the R1 lanes of a
// line group are the first-stage butterflies j of one packed complex line (real rows
// r and r + 1 as real and imaginary parts).  Butterfly j reads the positions of its
// points j + R1 q straight from global memory into registers: consecutive lanes read
// consecutive positions (inverse kinds) or every second one (the Makhoul order of the
// forward kinds, whose other half the same warp reads in another instruction), so each
// 32-byte sector a warp touches is used in full and the tile is never staged in shared
// memory.  Shared memory carries only the exchange between the two radix stages; the
// X[p] / X[N - p] pairings are lane shuffles inside the line group (rd_fft, ZMAP).
// Outputs go from registers to global memory.  Loads finish before the first barrier and
// every row belongs to one CTA, so the pass may run in place (in == out).
#pragma once

#include "r2r_rd.cuh"

namespace smadft {

template <typename T, int N>
constexpr size_t rdz_smem_bytes() { return rd_smem_bytes<T, N>() + (size_t)N * sizeof(cpx<T>); }

// rows = number of z lines (nx * ny); a CTA transforms 2 * kRdLines consecutive rows.
// rev = 1 walks the tiles from the last row down: the pass before a z pass (the y pass of the
// same transform) writes its field from x = 0 up, so the rows it wrote last, still in L2,
// are read first.  Tiles are independent, so the order does not change the result.
// KIND >= 0 fixes the transform kind at compile time (the kind checks inside the transform
// and the position maps fold away); KIND = -1 takes it from `kind_rt`.
// STAGE: the outputs go through shared memory and leave as whole rows in 16-byte stores (the
// inverse kinds' Makhoul order would otherwise scatter every warp store over every second
// element); `out` must then be 16-byte aligned.
// ZM: how the line is read or written.  kZPlain; kZGrad: the index-shifted gradient spectrum
// of `in` along z (LdGrad along z): point n takes -zs[n] in[n + 1], the last point 0;
// kZUpRead: point n takes in[n + 1], the last point 0 (a spectrum stored by true wavenumber,
// read as a sine series); kZUpStore (direct stores only): output position n goes to n + 1,
// the last one is dropped and position 0 is zero-filled (a sine-axis spectrum stored by true
// wavenumber).  Loads finish before the first barrier and a row belongs to one CTA, so every
// mode may run in place.
enum : int { kZPlain = 0, kZGrad = 1, kZUpRead = 2, kZUpStore = 3 };
template <typename T, int N, int KIND = -1, bool STAGE = false, int ZM = kZPlain>
__global__ void __launch_bounds__(RdInfo<N>::THREADS, sizeof(T) == 4 ? 3 : 2) r2r_rdz_kernel(int rows, int kind_rt, const T *in, T *out,
                                                                        const cpx<T> *__restrict__ wt_g,
                                                                        const cpx<T> *__restrict__ ht_g, int rev,
                                                                        const T *__restrict__ zs)
{
    const int kind = KIND >= 0 ? KIND : kind_rt;
    using RI = RdInfo<N>;
    constexpr int R0 = RI::R0, R1 = RI::R1, NT = RI::THREADS;
    constexpr int BPT = R0 / R1 > 0 ? R0 / R1 : 1;
    constexpr int NP = BPT * R1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T> *buf = reinterpret_cast<cpx<T> *>(smem_raw);
    cpx<T> *wt = buf + kRdLines * RI::LD;
    cpx<T> *ht = wt + N;
    cpx<T> *wz = ht + N;                            // stage-0 twiddles W_N^(j q) at q R1 + j
    for (int m = threadIdx.x; m < N; m += NT) {
        wt[m] = wt_g[m];
        ht[m] = ht_g[m];
        wz[m] = wt_g[(m % R1) * (m / R1)];
    }
    const int j = threadIdx.x % R1;                 // first-stage butterfly (lane in its group)
    const int c = threadIdx.x / R1;                 // complex line of the CTA
    const int tile = rev ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x;
    const int ra = tile * (2 * kRdLines) + 2 * c;   // real rows ra, ra + 1
    const bool oka = ra < rows, okb = ra + 1 < rows;
    const idx_t ia = (oka ? ra : 0) * N, ib = (okb ? ra + 1 : 0) * N;
    const bool fwd = (kind == K_DCT2 || kind == K_DST2);
    const bool sine = (kind == K_DST2 || kind == K_DST3);

    const RdPos<N> pos(j, fwd, sine);               // affine position maps (r2r_rd.cuh)
    const T *pa = in + ia, *pb = in + ib;
    cpx<T> v[R0];
#pragma unroll
    for (int q = 0; q < R0; q++) {
        const int n = pos.src(q);
        T a, b;
        if constexpr (ZM == kZGrad) {
            const bool inr = n < N - 1;
            const int m = inr ? n + 1 : n;
            const T sc = inr ? -zs[n] : T(0);
            a = sc * pa[m];
            b = sc * pb[m];
        } else if constexpr (ZM == kZUpRead) {
            const bool inr = n < N - 1;
            const int m = inr ? n + 1 : n;
            const T ra = pa[m], rb = pb[m];
            a = inr ? ra : T(0);
            b = inr ? rb : T(0);
        } else {
            a = pa[n];
            b = pb[n];
        }
        if (!oka) a = T(0);
        if (!okb) b = T(0);
        if (fwd && sine && !RdPos<N>::src_lo(q)) {   // DST-II negates odd natural samples
            a = -a;
            b = -b;
        }
        v[q] = {a, b};
    }
    __syncthreads();                                 // twiddle tables
    cpx<T> x1[BPT][R1];
    rd_fft<T, N, true>(v, x1, buf + c * RI::LD, wt, ht, j, threadIdx.x >> 5, fwd, sine, wz);
    static_assert(!(STAGE && ZM == kZUpStore), "shifted stores go direct");
    if constexpr (STAGE) {
        // the CTA's 2 kRdLines rows in shared memory (inside the exchange buffer), then rows
        // of N elements out with 16-byte stores; rows past `rows` are not written
        T *sb = reinterpret_cast<T *>(buf);
        __syncthreads();                                 // every warp is done with buf
        if constexpr (R1 == 16 && BPT == 1) {
            // the two half-warps of a warp write rows 2N apart (same banks) and each point
            // goes to every second element; the odd line takes its points half a turn later,
            // so in each store one half-warp writes even and the other odd elements
            const bool odd = c & 1;
#pragma unroll
            for (int pnt = 0; pnt < NP; pnt++) {
                constexpr int H = NP / 2;
                const int pt = (pnt + H) % NP;
                const cpx<T> z0 = x1[0][pnt], z1 = x1[0][pt];
                const int o = odd ? pos.out(pt) : pos.out(pnt);
                const T zx = odd ? z1.x : z0.x, zy = odd ? z1.y : z0.y;
                sb[(2 * c) * N + o] = zx;
                sb[(2 * c + 1) * N + o] = zy;
            }
        } else {
#pragma unroll
            for (int pnt = 0; pnt < NP; pnt++) {
                const cpx<T> z = x1[pnt / R1][pnt % R1];
                const int o = pos.out(pnt);
                sb[(2 * c) * N + o] = z.x;
                sb[(2 * c + 1) * N + o] = z.y;
            }
        }
        __syncthreads();
        constexpr int VEC = 16 / (int)sizeof(T);
        constexpr int PER_ROW = N / VEC;
        const int row0 = tile * (2 * kRdLines);
        for (int e = threadIdx.x; e < 2 * kRdLines * PER_ROW; e += NT) {
            const int r = e / PER_ROW, cv = e % PER_ROW;
            if (row0 + r < rows)
                *reinterpret_cast<uint4 *>(out + (idx_t)(row0 + r) * N + cv * VEC) =
                    *reinterpret_cast<const uint4 *>(sb + r * N + cv * VEC);
        }
    } else {
        T *qa = out + ia, *qb = out + ib;
#pragma unroll
        for (int pnt = 0; pnt < NP; pnt++) {
            const cpx<T> z = x1[pnt / R1][pnt % R1];
            const int o = pos.out(pnt);
            if constexpr (ZM == kZUpStore) {
                if (oka && o + 1 < N) qa[o + 1] = z.x;
                if (okb && o + 1 < N) qb[o + 1] = z.y;
                if (oka && o == 0) qa[0] = T(0);
                if (okb && o == 0) qb[0] = T(0);
            } else {
                if (oka) qa[o] = z.x;
                if (okb) qb[o] = z.y;
            }
        }
    }
}

}  // namespace smadft
