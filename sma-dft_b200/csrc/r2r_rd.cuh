// r2r_rd.cuh -- register-direct axis pass for the strided axes (x, y) with two-stage plans
// (N = R0 x R1: 64 = 8x8, 128 = 16x8, 256 = 16x16).
//
// A CTA owns 32 consecutive k-columns (16 complex lines: real lines 2c and 2c+1 travel as
// the real and imaginary parts of complex line c).  Thread (c, j) loads the R0 points of
// its first-stage butterfly straight from global memory into registers -- one 8/16-byte
// access per point covers both real lines, and the 16 threads of a half-warp cover 128
// contiguous bytes -- so the tile is never staged in shared memory on the way in.  Shared
// memory carries only the one exchange between the two radix stages (and, for the forward
// kinds, the X[k] / X[N-k] pairing of the DCT-II post-twiddle).  Outputs go straight from
// registers to global memory through the Storer, and inputs come through the Loader, so
// the fused multi-field loaders and storers of the model steps run here too.
//
// Index conventions follow r2r_fast.cuh: DIF stage 0 (radix R0, stride R1) then stage 1
// (radix R1, stride 1); position b*R1 + q then holds X[b + R0 q].  The pairings X[p] /
// X[N-p] (DCT-III pre-twiddle) and X[k] / X[N-k] (DCT-II post-twiddle) are done with one
// warp shuffle per value: butterflies j and R1 - j sit in the two halves of one warp.
#pragma once

#include <type_traits>

#include "r2r_fast.cuh"

namespace smadft {

template <int N>
struct RdPlan;
template <>
struct RdPlan<64> { static constexpr int R0 = 8, R1 = 8; };
template <>
struct RdPlan<128> { static constexpr int R0 = 16, R1 = 8; };
template <>
struct RdPlan<256> { static constexpr int R0 = 16, R1 = 16; };

constexpr int kRdLines = 16;   // complex lines per CTA (32 real k-columns)

template <int N>
struct RdInfo {
    static constexpr int R0 = RdPlan<N>::R0, R1 = RdPlan<N>::R1;
    static constexpr int THREADS = kRdLines * R1;
    static constexpr int LD = N + N / R1 + 1;              // padded complex line stride
    __device__ static __forceinline__ int phys(int p) { return p + p / R1; }
};

template <typename T, int N>
constexpr size_t rd_smem_bytes() { return ((size_t)kRdLines * RdInfo<N>::LD + 2 * N) * sizeof(cpx<T>); }

// CTAs per SM the register budget is sized for: FP32 passes fit three (80 registers; the
// fused loaders spill at most a few words there, and the extra resident CTA hides more
// load latency) unless the loader asks for two (ld_blocks); FP64 passes, and FP32 passes
// whose storer carries FP64 state reads (the spectral updates), keep two
template <typename T, class LD, class ST>
constexpr int rd_min_blocks() { return (sizeof(T) == 4 && sizeof(pre_t<ST, T>) == 4) ? ld_blocks<LD>::value : 2; }

// natural sample index whose Makhoul position is p (inverse of makhoul_pos)
template <int N>
__device__ __forceinline__ int makhoul_src(int p) { return p < N / 2 ? 2 * p : 2 * (N - 1 - p) + 1; }

// The transform of one packed complex line by thread (line c, butterfly j) of warp wi: v
// holds the R0 stage-0 points j + q R1 (Makhoul-permuted for the forward kinds, DST-II
// signs applied; natural or reversed order for the inverse kinds); x1 receives the
// output points, whose line positions rd_out_pos gives.  `line` is this thread's complex
// line in the CTA's exchange buffer.  Contains __syncthreads(): every thread of the CTA
// calls it.
//
// ZMAP selects the lane layout of r2r_rdz_kernel (lane = butterfly j of one line, see
// r2r_rdz.cuh): the pairings then go to butterfly R1 - j by an indexed shuffle, and
// butterfly 0, which pairs with itself, takes its own path after the shuffled one.
template <typename T, int N, bool ZMAP = false>
__device__ __forceinline__ void rd_fft(cpx<T> (&v)[RdInfo<N>::R0],
                                       cpx<T> (&x1)[RdInfo<N>::R0 / RdInfo<N>::R1 > 0 ? RdInfo<N>::R0 / RdInfo<N>::R1 : 1]
                                                   [RdInfo<N>::R1],
                                       cpx<T> *line, const cpx<T> *wt, const cpx<T> *ht, int j, int wi, bool fwd,
                                       bool sine, const cpx<T> *wz = nullptr)
{
    using RI = RdInfo<N>;
    constexpr int R0 = RI::R0, R1 = RI::R1;
    constexpr int BPT = R0 / R1 > 0 ? R0 / R1 : 1;
    if (!fwd) {
        // DCT-III pre-twiddle Z_p = V_A[p] + i V_B[p], V[p] = exp(+i pi p/2N)(X_p - i X_{N-p}),
        // X_N = 0; DST-III reads the line reversed.  X_{N-p} comes from the partner lane (or
        // the thread itself in warp 0); each pair of points is rewritten in place together so
        // only one array stays live.
        auto ztw = [&](int q, cpx<T> xa, cpx<T> xb) -> cpx<T> { return dct3_pre(xa, xb, ht[j + q * R1]); };
        if constexpr (ZMAP) {
            // butterfly j >= 1: partner point of q is R0 - 1 - q in butterfly R1 - j (lane pl;
            // j = R1/2 reads itself); butterfly 0 keeps its values for the path below
            const int lane = threadIdx.x & 31;
            const int pl = j == 0 ? lane : lane + R1 - 2 * j;
#pragma unroll
            for (int q = 0; q < R0 / 2; q++) {
                const int qb = R0 - 1 - q;
                cpx<T> pa, pb;
                pa.x = __shfl_sync(0xffffffffu, v[qb].x, pl);
                pa.y = __shfl_sync(0xffffffffu, v[qb].y, pl);
                pb.x = __shfl_sync(0xffffffffu, v[q].x, pl);
                pb.y = __shfl_sync(0xffffffffu, v[q].y, pl);
                const cpx<T> za = ztw(q, v[q], pa), zb = ztw(qb, v[qb], pb);
                if (j != 0) {
                    v[q] = za;
                    v[qb] = zb;
                }
            }
            if (j == 0) {
                v[0] = ztw(0, v[0], cpx<T>{T(0), T(0)});
                v[R0 / 2] = ztw(R0 / 2, v[R0 / 2], v[R0 / 2]);
#pragma unroll
                for (int q = 1; q < R0 / 2; q++) {
                    const int qb = R0 - q;
                    const cpx<T> za = ztw(q, v[q], v[qb]), zb = ztw(qb, v[qb], v[q]);
                    v[q] = za;
                    v[qb] = zb;
                }
            }
        } else if (wi != 0 || j == R1 / 2) {
            // partner point of q is R0 - 1 - q (in lane ^ 16, or here for j = R1/2)
#pragma unroll
            for (int q = 0; q < R0 / 2; q++) {
                const int qb = R0 - 1 - q;
                cpx<T> pa, pb;
                if (wi != 0) {
                    pa.x = __shfl_xor_sync(0xffffffffu, v[qb].x, 16);
                    pa.y = __shfl_xor_sync(0xffffffffu, v[qb].y, 16);
                    pb.x = __shfl_xor_sync(0xffffffffu, v[q].x, 16);
                    pb.y = __shfl_xor_sync(0xffffffffu, v[q].y, 16);
                } else {
                    pa = v[qb];
                    pb = v[q];
                }
                const cpx<T> za = ztw(q, v[q], pa), zb = ztw(qb, v[qb], pb);
                v[q] = za;
                v[qb] = zb;
            }
        } else {
            // j = 0: partner of q is R0 - q (q = 0 pairs with X_N = 0, q = R0/2 with itself)
            v[0] = ztw(0, v[0], cpx<T>{T(0), T(0)});
            v[R0 / 2] = ztw(R0 / 2, v[R0 / 2], v[R0 / 2]);
#pragma unroll
            for (int q = 1; q < R0 / 2; q++) {
                const int qb = R0 - q;
                const cpx<T> za = ztw(q, v[q], v[qb]), zb = ztw(qb, v[qb], v[q]);
                v[q] = za;
                v[qb] = zb;
            }
        }
    }

    // ---- stage 0: radix R0 over stride R1, twiddles W_N^(j q), into shared memory
    if (fwd) codelet<R0, T, false>(v);
    else codelet<R0, T, true>(v);
#pragma unroll
    for (int q = 0; q < R0; q++) {
        cpx<T> o = v[q];
        // ZMAP reads W_N^(j q) from the transposed table wz[q R1 + j] (consecutive lanes,
        // consecutive banks); the strided layout broadcasts wt[j q] over a half-warp
        const cpx<T> *wq = ZMAP ? wz : wt;
        const int e = ZMAP ? q * R1 + j : j * q;
        if (q > 0) o = fwd ? cmul(o, tw<T, false>(wq, e)) : cmul(o, tw<T, true>(wq, e));
        line[RI::phys(j + q * R1)] = o;
    }
    __syncthreads();

    // ---- stage 1: radix R1 over contiguous blocks; block b holds X[b + R0 q] afterwards
#pragma unroll
    for (int r = 0; r < BPT; r++) {
        const int b = j + r * R1;
        cpx<T> *pb = line + RI::phys(b * R1);
#pragma unroll
        for (int q = 0; q < R1; q++) x1[r][q] = pb[q];
        if (fwd) codelet<R1, T, false>(x1[r]);
        else codelet<R1, T, true>(x1[r]);
    }

    // ---- outputs: (real line A, real line B) pairs in x1
    if (!fwd) {
        // DCT-III output y[2m] = v[m], y[2m+1] = v[N-1-m]; DST-III negates odd outputs
#pragma unroll
        for (int r = 0; r < BPT; r++)
#pragma unroll
            for (int q = 0; q < R1; q++) {
                const int m = j + r * R1 + R0 * q;
                const int o = m < N / 2 ? 2 * m : 2 * (N - 1 - m) + 1;
                if (sine && (o & 1)) x1[r][q] = {-x1[r][q].x, -x1[r][q].y};
            }
    } else {
        // DCT-II post-twiddle pairs X[k] with X[N-k]
        if constexpr (BPT == 1) {
            // X[N - k] is block R1 - j at q' = R1 - 1 - q (lane ^ 16, or this thread for
            // j = R1/2), or block 0 at q' = (R1 - q) mod R1 for j = 0; each pair (q, q') is
            // rewritten in place together
            auto post = [&](int q, cpx<T> zm) -> cpx<T> { return dct2_post(x1[0][q], zm, ht[j + R0 * q]); };
            if constexpr (ZMAP) {
                const int lane = threadIdx.x & 31;
                const int pl = j == 0 ? lane : lane + R1 - 2 * j;
#pragma unroll
                for (int q = 0; q < R1 / 2; q++) {
                    const int qb = R1 - 1 - q;
                    cpx<T> pa, pb;
                    pa.x = __shfl_sync(0xffffffffu, x1[0][qb].x, pl);
                    pa.y = __shfl_sync(0xffffffffu, x1[0][qb].y, pl);
                    pb.x = __shfl_sync(0xffffffffu, x1[0][q].x, pl);
                    pb.y = __shfl_sync(0xffffffffu, x1[0][q].y, pl);
                    const cpx<T> oa = post(q, pa), ob = post(qb, pb);
                    if (j != 0) {
                        x1[0][q] = oa;
                        x1[0][qb] = ob;
                    }
                }
                if (j == 0) {
                    const cpx<T> o0 = post(0, x1[0][0]);
                    const cpx<T> oh = post(R1 / 2, x1[0][R1 / 2]);
#pragma unroll
                    for (int q = 1; q < R1 / 2; q++) {
                        const int qb = R1 - q;
                        const cpx<T> oa = post(q, x1[0][qb]), ob = post(qb, x1[0][q]);
                        x1[0][q] = oa;
                        x1[0][qb] = ob;
                    }
                    x1[0][0] = o0;
                    x1[0][R1 / 2] = oh;
                }
            } else if (wi != 0 || j == R1 / 2) {
#pragma unroll
                for (int q = 0; q < R1 / 2; q++) {
                    const int qb = R1 - 1 - q;
                    cpx<T> pa, pb;
                    if (wi != 0) {
                        pa.x = __shfl_xor_sync(0xffffffffu, x1[0][qb].x, 16);
                        pa.y = __shfl_xor_sync(0xffffffffu, x1[0][qb].y, 16);
                        pb.x = __shfl_xor_sync(0xffffffffu, x1[0][q].x, 16);
                        pb.y = __shfl_xor_sync(0xffffffffu, x1[0][q].y, 16);
                    } else {
                        pa = x1[0][qb];
                        pb = x1[0][q];
                    }
                    const cpx<T> oa = post(q, pa), ob = post(qb, pb);
                    x1[0][q] = oa;
                    x1[0][qb] = ob;
                }
            } else {
                const cpx<T> o0 = post(0, x1[0][0]);
                const cpx<T> oh = post(R1 / 2, x1[0][R1 / 2]);
#pragma unroll
                for (int q = 1; q < R1 / 2; q++) {
                    const int qb = R1 - q;
                    const cpx<T> oa = post(q, x1[0][qb]), ob = post(qb, x1[0][q]);
                    x1[0][q] = oa;
                    x1[0][qb] = ob;
                }
                x1[0][0] = o0;
                x1[0][R1 / 2] = oh;
            }
        } else {
            // through shared memory (each thread rewrites only its own blocks first)
#pragma unroll
            for (int r = 0; r < BPT; r++) {
                cpx<T> *pb = line + RI::phys((j + r * R1) * R1);
#pragma unroll
                for (int q = 0; q < R1; q++) pb[q] = x1[r][q];
            }
            __syncthreads();
#pragma unroll
            for (int r = 0; r < BPT; r++)
#pragma unroll
                for (int q = 0; q < R1; q++) {
                    const int kk = j + r * R1 + R0 * q;
                    const int km = kk == 0 ? 0 : N - kk;
                    const cpx<T> zm = line[RI::phys((km % R0) * R1 + km / R0)];
                    x1[r][q] = dct2_post(x1[r][q], zm, ht[kk]);
                }
        }
    }

}

// line position of output point pnt of butterfly j (see rd_fft)
template <int N>
__device__ __forceinline__ int rd_out_pos(int j, int pnt, bool fwd, bool sine)
{
    constexpr int R0 = RdInfo<N>::R0, R1 = RdInfo<N>::R1;
    const int kk = j + (pnt / R1) * R1 + R0 * (pnt % R1);   // X index held by point pnt
    if (fwd) return sine ? N - 1 - kk : kk;
    return kk < N / 2 ? 2 * kk : 2 * (N - 1 - kk) + 1;
}

// Line positions of butterfly j as affine maps of the (compile-time) point index.  The
// natural position read by stage-0 point q is lb + ls q when q R1 < N/2, else hb + hs q;
// the position of output point pnt is olb + ols C, else ohb + ohs C, with
// C = (pnt / R1) R1 + R0 (pnt mod R1) against N/2 (j < R1 never moves a point across N/2,
// which is a multiple of R0 and R1).  Inside the unrolled loops the branch folds and one
// multiply-add per point remains (the maps equal makhoul_src / rd_out_pos).
template <int N>
struct RdPos {
    static constexpr int R0 = RdInfo<N>::R0, R1 = RdInfo<N>::R1;
    int lb, ls, hb, hs, olb, ols, ohb, ohs;
    __device__ __forceinline__ RdPos(int j, bool fwd, bool sine)
    {
        if (fwd) {
            lb = 2 * j; ls = 2 * R1; hb = 2 * N - 1 - 2 * j; hs = -2 * R1;   // Makhoul order
            olb = ohb = sine ? N - 1 - j : j;
            ols = ohs = sine ? -1 : 1;
        } else {
            lb = hb = sine ? N - 1 - j : j;
            ls = hs = sine ? -R1 : R1;
            olb = 2 * j; ols = 2; ohb = 2 * N - 1 - 2 * j; ohs = -2;         // y[2m], y[2m+1]
        }
    }
    static constexpr bool src_lo(int q) { return q * R1 < N / 2; }
    static constexpr int cpos(int pnt) { return (pnt / R1) * R1 + R0 * (pnt % R1); }
    __device__ __forceinline__ int src(int q) const { return src_lo(q) ? lb + ls * q : hb + hs * q; }
    __device__ __forceinline__ int out(int pnt) const
    {
        return cpos(pnt) < N / 2 ? olb + ols * cpos(pnt) : ohb + ohs * cpos(pnt);
    }
};

// NC > 1: multi-component pass (LoadMulti / StoreMulti); CTA b transforms component b mod NC
// of tile b / NC, so the components' shared input reads meet in L2.
// KIND >= 0 fixes the transform kind of a one-component pass at compile time (the kind
// checks inside the transform and the position maps fold away); KIND = -1 reads `kinds`.
// DIR >= 0 fixes only the direction (1 forward kinds, 0 inverse kinds), which the components
// of a grouped pass share; the sine/cosine choice then stays per component.
template <typename T, int N, int AXIS, class LD, class ST, int NC = 1, int KIND = -1, int DIR = -1>
__global__ void __launch_bounds__(RdInfo<N>::THREADS, rd_min_blocks<T, LD, ST>()) r2r_rd_kernel(Geom g, KindSet<NC> kinds, int tiles_b, LD ld,
                                                                       const cpx<T> *__restrict__ wt_g,
                                                                       const cpx<T> *__restrict__ ht_g, ST st)
{
    using RI = RdInfo<N>;
    constexpr int R0 = RI::R0, R1 = RI::R1, NT = RI::THREADS;
    constexpr int BPT = R0 / R1 > 0 ? R0 / R1 : 1;   // last-stage blocks per thread
    constexpr int NP = BPT * R1;                      // output points per thread (= R0)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T> *buf = reinterpret_cast<cpx<T> *>(smem_raw);
    cpx<T> *wt = buf + kRdLines * RI::LD;
    cpx<T> *ht = wt + N;
    for (int m = threadIdx.x; m < N; m += NT) {
        wt[m] = wt_g[m];
        ht[m] = ht_g[m];
    }
    // Thread (c, j): c = complex line (fastest, for coalescing), j = first-stage butterfly.
    // Warp w holds the butterfly pair {j, R1 - j} (warp 0: {0, R1/2}) in its two half-warps:
    // X[N - p] for the points p of butterfly j lives in butterfly R1 - j (lane ^ 16), and the
    // same pairing holds for X[k] / X[N - k] after the last stage.
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5, hh16 = lane >> 4;
    const int c = lane & 15;
    const int j = (wi == 0) ? (hh16 ? R1 / 2 : 0) : (hh16 ? R1 - wi : wi);
    // tile: 32 k-columns starting at kt*32 along the non-transformed line coordinate `a`
    const int comp = NC > 1 ? (int)(blockIdx.x % NC) : 0;
    const int bt = NC > 1 ? (int)(blockIdx.x / NC) : (int)blockIdx.x;
    const int kind = KIND >= 0 ? KIND : kinds.k[comp];
    const int kt = bt % tiles_b;
    const int a = bt / tiles_b;
    const int k = kt * 32 + 2 * c;                 // first of the two real lines
    const idx_t stride = AXIS == 1 ? g.nz : g.nyz;
    const idx_t base = (AXIS == 1 ? a * g.nyz : a * g.nz) + k;
    const int nk = g.nz - k;                       // real lines of this pair inside the box
    const bool full = (kt + 1) * 32 <= g.nz;       // CTA-uniform: no line outside the box
    const bool fwd = DIR >= 0 ? DIR == 1 : (kind == K_DCT2 || kind == K_DST2);
    const bool sine = (kind == K_DST2 || kind == K_DST3);
    __syncthreads();

    // element indices: position t of a line point sits at base + t * stride, so the affine
    // position maps become affine index maps (one multiply-add per point)
    const RdPos<N> pos(j, fwd, sine);
    const idx_t slo = base + pos.lb * stride, dslo = pos.ls * stride;
    const idx_t shi = base + pos.hb * stride, dshi = pos.hs * stride;
    const idx_t olo = base + pos.olb * stride, dolo = pos.ols * stride;
    const idx_t ohi = base + pos.ohb * stride, dohi = pos.ohs * stride;
    auto src_idx = [&](int q) -> idx_t { return RdPos<N>::src_lo(q) ? slo + q * dslo : shi + q * dshi; };
    auto out_idx = [&](int pnt) -> idx_t {
        constexpr int H = N / 2;
        const int C = RdPos<N>::cpos(pnt);
        return C < H ? olo + C * dolo : ohi + C * dohi;
    };

    // the pair of real samples (lines k, k+1) of stage-0 point q, packed as one complex;
    // the Loader computes them from its fields (each point is loaded exactly once)
    auto load_pair = [&](const auto &l, int q, bool edge) -> cpx<T> {
        const int t = pos.src(q);
        const int ii = AXIS == 1 ? a : t, jj = AXIS == 1 ? t : a;
        T v[2] = {T(0), T(0)};
        const idx_t si = src_idx(q);
        if (!edge || nk >= 2) {
            if (idx_ok(g, si, 2)) l.template load<2>(si, ii, jj, k, v);
        } else if (nk == 1) {
            if (idx_ok(g, si)) l.template load<1>(si, ii, jj, k, v);
        }
        return {v[0], v[1]};
    };

    cpx<T> v[R0];
    // one straight-line load loop per loader (a multi-component loader is resolved once per CTA)
    visit_c(ld, comp, [&](const auto &l) {
        if (full) {
#pragma unroll
            for (int q = 0; q < R0; q++) v[q] = load_pair(l, q, false);
        } else {
#pragma unroll
            for (int q = 0; q < R0; q++) v[q] = load_pair(l, q, true);
        }
    });
    if (fwd) {
        // Makhoul-permuted input: DST-II negates odd natural samples (the odd ones are the
        // upper half, q R1 >= N/2)
        if (sine) {
#pragma unroll
            for (int q = 0; q < R0; q++)
                if (!RdPos<N>::src_lo(q)) v[q] = {-v[q].x, -v[q].y};
        }
    }
    cpx<T> x1[BPT][R1];
    rd_fft<T, N>(v, x1, buf + c * RI::LD, wt, ht, j, wi, fwd, sine);
    auto out_row = [&](int pnt) -> int { return pos.out(pnt); };

    // ---- stores: the storer's reads (pre) for a chunk of points go out before its writes
    constexpr int CH = 4;
    constexpr int PL = pre_len<ST, 2>();
    using PB = pre_t<ST, T>;
    auto put = [&](int pnt, bool edge, const PB *pre_buf) {
        const cpx<T> z = x1[pnt / R1][pnt % R1];
        const int o = out_row(pnt);
        const idx_t q = out_idx(pnt);
        const int ii = AXIS == 1 ? a : o, jj = AXIS == 1 ? o : a;
        const T w2[2] = {z.x, z.y};
        if (!edge || nk >= 2) {
            if (idx_ok(g, q, 2)) fin_c<2>(st, comp, q, ii, jj, k, w2, pre_buf);
        } else if (nk == 1) {
            if (idx_ok(g, q)) store_c<1>(st, comp, q, ii, jj, k, w2);
        }
    };
    if (full) {
#pragma unroll
        for (int p0 = 0; p0 < NP; p0 += CH) {
            PB pre_buf[CH][PL];
#pragma unroll
            for (int u = 0; u < CH; u++) {
                const int o = out_row(p0 + u);
                if (idx_ok(g, out_idx(p0 + u), 2))
                    pre_c<2>(st, comp, out_idx(p0 + u), AXIS == 1 ? a : o, AXIS == 1 ? o : a, k, pre_buf[u]);
            }
#pragma unroll
            for (int u = 0; u < CH; u++) put(p0 + u, false, pre_buf[u]);
        }
    } else {
#pragma unroll
        for (int p0 = 0; p0 < NP; p0++) {
            PB pre_buf[PL];
            const int o = out_row(p0);
            if (nk >= 2 && idx_ok(g, out_idx(p0), 2)) pre_c<2>(st, comp, out_idx(p0), AXIS == 1 ? a : o, AXIS == 1 ? o : a, k, pre_buf);
            put(p0, true, pre_buf);
        }
    }
}

}  // namespace smadft
