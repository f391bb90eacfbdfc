// r2r_fast.cuh -- compile-time-specialised axis pass (the hot kernel).
//
// Same contract as r2r_pass_kernel (r2r_pass.cuh) but for line lengths known at compile
// time, so that every index computation is shifts and constant multiplies:
//   * the tile (W = 32 lines) is staged once in shared memory as 16 complex lines
//     (two real lines per complex line, Makhoul permutation applied on the way in);
//   * the complex FFT is an in-place mixed-radix decimation-in-frequency with register
//     codelets of radix 16/10/8/6/4/2/3/5 (e.g. 256 = 16 x 16, 160 = 16 x 10, 96 = 16 x 6:
//     two passes over shared memory);
//     its output is left in digit-reversed order and read back through that map;
//   * shared-memory positions are padded (one slot per last-radix block, one per line)
//     so the stage loads/stores and the row-major global staging are bank-conflict free;
//   * tile coordinates are computed once per CTA; per element only adds remain.
#pragma once

#include "r2r_pass.cuh"

namespace smadft {

// ---- radix plans per length ----------------------------------------------------------
template <int N>
struct FastPlan;
#define SMADFT_PLAN(N_, S_, R0, R1, R2)                    \
    template <>                                            \
    struct FastPlan<N_> {                                  \
        static constexpr int S = S_;                       \
        static constexpr int R[3] = {R0, R1, R2};          \
    };
SMADFT_PLAN(16, 2, 4, 4, 1)
SMADFT_PLAN(24, 2, 8, 3, 1)
SMADFT_PLAN(32, 2, 8, 4, 1)
SMADFT_PLAN(40, 2, 8, 5, 1)
SMADFT_PLAN(48, 2, 16, 3, 1)
SMADFT_PLAN(64, 2, 8, 8, 1)
SMADFT_PLAN(80, 2, 16, 5, 1)
SMADFT_PLAN(96, 2, 16, 6, 1)
SMADFT_PLAN(128, 2, 16, 8, 1)
SMADFT_PLAN(160, 2, 16, 10, 1)
SMADFT_PLAN(192, 3, 16, 4, 3)
SMADFT_PLAN(256, 2, 16, 16, 1)
SMADFT_PLAN(320, 3, 16, 4, 5)
SMADFT_PLAN(384, 3, 16, 8, 3)
SMADFT_PLAN(512, 3, 16, 8, 4)
#undef SMADFT_PLAN

template <int N>
struct PlanInfo {
    static constexpr int S = FastPlan<N>::S;
    static constexpr int R0 = FastPlan<N>::R[0];
    static constexpr int R1 = FastPlan<N>::R[1];
    static constexpr int R2 = FastPlan<N>::R[2];
    static constexpr int RL = S == 2 ? R1 : R2;             // last radix
    static constexpr int M1 = N / R0;                       // block size after stage 0
    static constexpr int M2 = M1 / R1;                      // after stage 1
    static constexpr int LD = N + N / RL + 1;               // padded line stride (complex)
    __device__ static __forceinline__ int phys(int p) { return p + p / RL; }
    // position holding X[k] after the DIF stages (mixed-radix digit reversal)
    __device__ static __forceinline__ int pos(int k)
    {
        const int q0 = k % R0, k1 = k / R0;
        if (S == 2) return q0 * M1 + k1;
        const int q1 = k1 % R1, q2 = k1 / R1;
        return q0 * M1 + q1 * M2 + q2;
    }
};

// ---- register codelets -----------------------------------------------------------------
// Size-R DFT of v[0..R-1] in place, in-order output.  INV selects exp(+2 pi i / R).
template <typename T, bool INV>
__device__ __forceinline__ void dft4(cpx<T> &a0, cpx<T> &a1, cpx<T> &a2, cpx<T> &a3)
{
    cpx<T> s0 = cadd(a0, a2), d0 = csub(a0, a2), s1 = cadd(a1, a3), d1 = csub(a1, a3);
    cpx<T> j = INV ? mul_pi(d1) : mul_mi(d1);
    a0 = cadd(s0, s1);
    a2 = csub(s0, s1);
    a1 = cadd(d0, j);
    a3 = csub(d0, j);
}

// exp(sign 2 pi i m / 16) for m = 0..15, sign = -1 (forward) or +1 (inverse)
template <typename T, bool INV>
__device__ __forceinline__ cpx<T> w16(int m)
{
    const T c1 = T(0.92387953251128675612818318939679);  // cos(pi/8)
    const T s1 = T(0.38268343236508977172845998403040);  // sin(pi/8)
    const T h = T(0.70710678118654752440084436210485);   // cos(pi/4)
    T c, s;
    switch (m & 15) {
    case 0: c = 1; s = 0; break;
    case 1: c = c1; s = s1; break;
    case 2: c = h; s = h; break;
    case 3: c = s1; s = c1; break;
    case 4: c = 0; s = 1; break;
    case 5: c = -s1; s = c1; break;
    case 6: c = -h; s = h; break;
    case 7: c = -c1; s = s1; break;
    case 8: c = -1; s = 0; break;
    case 9: c = -c1; s = -s1; break;
    case 10: c = -h; s = -h; break;
    case 11: c = -s1; s = -c1; break;
    case 12: c = 0; s = -1; break;
    case 13: c = s1; s = -c1; break;
    case 14: c = h; s = -h; break;
    default: c = c1; s = -s1; break;
    }
    return {c, INV ? s : -s};
}

template <int R, typename T, bool INV>
__device__ __forceinline__ void codelet(cpx<T> *v)
{
    if constexpr (R == 1) {
        return;
    } else if constexpr (R == 2 || R == 3 || R == 5) {
        dft<R, T, INV>(v);
    } else if constexpr (R == 4) {
        dft4<T, INV>(v[0], v[1], v[2], v[3]);
    } else if constexpr (R == 6 || R == 10) {
        // radix-2 decimation in time over two length-R/2 DFTs (R/2 = 3 or 5):
        // X[k] = E[k] + w^k O[k], X[k + R/2] = E[k] - w^k O[k], w = exp(-+ 2 pi i / R)
        constexpr int H = R / 2;
        cpx<T> e[H], o[H];
#pragma unroll
        for (int m = 0; m < H; m++) {
            e[m] = v[2 * m];
            o[m] = v[2 * m + 1];
        }
        dft<H, T, INV>(e);
        dft<H, T, INV>(o);
#pragma unroll
        for (int k = 0; k < H; k++) {
            cpx<T> t = o[k];
            if (k > 0) {
                T c, sn;   // cos, sin of 2 pi k / R
                if constexpr (R == 6) {
                    c = k == 1 ? T(0.5) : T(-0.5);
                    sn = T(0.86602540378443864676372317075294);
                } else {
                    const T c1 = T(0.80901699437494742410229341718282), s1 = T(0.58778525229247312916870595463907);
                    const T c2 = T(0.30901699437494742410229341718282), s2 = T(0.95105651629515357211643933337938);
                    c = k == 1 ? c1 : k == 2 ? c2 : k == 3 ? -c2 : -c1;
                    sn = (k == 1 || k == 4) ? s1 : s2;
                }
                t = cmul(t, cpx<T>{c, INV ? sn : -sn});
            }
            v[k] = cadd(e[k], t);
            v[k + H] = csub(e[k], t);
        }
    } else if constexpr (R == 8) {
        // radix-2 decimation in time over two length-4 DFTs
        cpx<T> e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
        dft4<T, INV>(e[0], e[1], e[2], e[3]);
        dft4<T, INV>(o[0], o[1], o[2], o[3]);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            cpx<T> t = (k == 0) ? o[0] : cmul(o[k], w16<T, INV>(2 * k));
            v[k] = cadd(e[k], t);
            v[k + 4] = csub(e[k], t);
        }
    } else if constexpr (R == 16) {
        // 4 x 4: length-4 DFTs over x[r + 4m], twiddle w16^(r k1), length-4 DFTs over r
        cpx<T> f[4][4];
#pragma unroll
        for (int r = 0; r < 4; r++) {
            f[r][0] = v[r]; f[r][1] = v[r + 4]; f[r][2] = v[r + 8]; f[r][3] = v[r + 12];
            dft4<T, INV>(f[r][0], f[r][1], f[r][2], f[r][3]);
        }
#pragma unroll
        for (int k1 = 0; k1 < 4; k1++) {
            cpx<T> g0 = f[0][k1];
            cpx<T> g1 = (k1 == 0) ? f[1][k1] : cmul(f[1][k1], w16<T, INV>(k1));
            cpx<T> g2 = (k1 == 0) ? f[2][k1] : cmul(f[2][k1], w16<T, INV>(2 * k1));
            cpx<T> g3 = (k1 == 0) ? f[3][k1] : cmul(f[3][k1], w16<T, INV>(3 * k1));
            dft4<T, INV>(g0, g1, g2, g3);
            v[k1] = g0; v[k1 + 4] = g1; v[k1 + 8] = g2; v[k1 + 12] = g3;
        }
    }
}

// One in-place DIF stage of radix R over `nl` lines: block size M (= R * stride).
// In every plan each stage's stride is a multiple of the last radix RL (or the stage is the
// last one and its block base is), so phys(base + q STR) = phys(base) + q (STR + STR/RL).
template <typename T, int N, int R, int M, bool INV>
__device__ __forceinline__ void dif_stage(cpx<T> *__restrict__ buf, int nl, const cpx<T> *__restrict__ w)
{
    using PI = PlanInfo<N>;
    constexpr int STR = M / R;              // butterfly stride
    constexpr int PER_LINE = N / R;         // butterflies per line
    constexpr int TW = N / M;               // twiddle table step: W_M^e = W_N^(e TW)
    constexpr int DP = STR + STR / PI::RL;  // physical distance between the R points
    const int tasks = nl * PER_LINE;
    for (int t = threadIdx.x; t < tasks; t += blockDim.x) {
        const int c = t / PER_LINE;
        const int u = t - c * PER_LINE;
        const int b = u / STR;
        const int j = u - b * STR;
        cpx<T> *pt = buf + c * PI::LD + PI::phys(b * M + j);
        cpx<T> v[R];
#pragma unroll
        for (int q = 0; q < R; q++) v[q] = pt[q * DP];
        codelet<R, T, INV>(v);
        pt[0] = v[0];
        const int jt = j * TW;
#pragma unroll
        for (int q = 1; q < R; q++) {
            cpx<T> o = v[q];
            if (STR > 1) o = cmul(o, tw<T, INV>(w, jt * q));
            pt[q * DP] = o;
        }
    }
}

template <typename T, int N, bool INV>
__device__ __forceinline__ void fft_dif(cpx<T> *buf, int nl, const cpx<T> *__restrict__ w)
{
    using PI = PlanInfo<N>;
    dif_stage<T, N, PI::R0, N, INV>(buf, nl, w);
    __syncthreads();
    dif_stage<T, N, PI::R1, PI::M1, INV>(buf, nl, w);
    __syncthreads();
    if constexpr (PI::S == 3) {
        dif_stage<T, N, PI::R2, PI::M2, INV>(buf, nl, w);
        __syncthreads();
    }
}

// Tile geometry resolved once per CTA.
struct TileBase {
    long long base;   // idx of element (t = 0, w = 0)
    int i0, j0, k0;   // coordinates of that element
};

template <int AXIS>
__device__ __forceinline__ TileBase tile_base(const Geom &g, int W, int tiles_b)
{
    TileBase tb;
    if (AXIS == 2) {
        const long long line = (long long)blockIdx.x * W;
        tb.i0 = (int)(line / g.ny);
        tb.j0 = (int)(line - (long long)tb.i0 * g.ny);
        tb.k0 = 0;
        tb.base = line * g.nz;
    } else {
        const int kt = blockIdx.x % tiles_b;
        const int a = blockIdx.x / tiles_b;
        tb.k0 = kt * W;
        if (AXIS == 1) { tb.i0 = a; tb.j0 = 0; }
        else { tb.j0 = a; tb.i0 = 0; }
        tb.base = ((long long)tb.i0 * g.ny + tb.j0) * g.nz + tb.k0;
    }
    return tb;
}

// element (t along the line, w = line in tile)
template <int AXIS>
__device__ __forceinline__ ElemPos tile_elem(const Geom &g, const TileBase &tb, int t, int w)
{
    ElemPos e;
    if (AXIS == 2) {
        int i = tb.i0, j = tb.j0 + w;
        while (j >= g.ny) { j -= g.ny; i++; }
        e.i = i; e.j = j; e.k = t;
        e.valid = i < g.nx;
        e.idx = tb.base + (long long)w * g.nz + t;
    } else {
        e.k = tb.k0 + w;
        e.valid = e.k < g.nz;
        if (AXIS == 1) { e.i = tb.i0; e.j = t; e.idx = tb.base + (long long)t * g.nz + w; }
        else { e.j = tb.j0; e.i = t; e.idx = tb.base + (long long)t * g.nyz + w; }
    }
    return e;
}

// Launch shape of the pass kernel: W real lines per tile, THREADS per CTA, at most MAXB
// 16-byte loads in flight per thread, MINB CTAs per SM for the register budget.
template <int W_, int THREADS_, int MAXB_, int MINB_>
struct FastCfg {
    static constexpr int W = W_;
    static constexpr int THREADS = THREADS_;
    static constexpr int MAXB = MAXB_;
    static constexpr int MINB = MINB_;
};
using FastDefault = FastCfg<32, 256, 8, 2>;
constexpr int kFastW = FastDefault::W;        // real lines per tile
constexpr int kFastThreads = FastDefault::THREADS;

// largest divisor of `per` not above `maxb`
constexpr int batch_size(int per, int maxb = 8)
{
    for (int b = maxb; b > 1; b--)
        if (per % b == 0) return b;
    return 1;
}

template <typename T, int N, class CFG = FastDefault>
constexpr size_t fast_smem_bytes() { return ((size_t)(CFG::W / 2) * PlanInfo<N>::LD + 2 * N) * sizeof(cpx<T>); }

// Post-twiddle of a forward (DCT-II) transform: output for line part `odd` (0 = real line A,
// 1 = real line B) from Z[k] and Z[N-k] of the packed complex line (see fft_tile.cuh).
template <typename T>
__device__ __forceinline__ T dct2_out(cpx<T> zk, cpx<T> zm, cpx<T> hh, int odd)
{
    const cpx<T> o = dct2_post(zk, zm, hh);
    return odd ? o.y : o.x;
}

template <typename T, int N, int AXIS, class LD, class ST, class CFG = FastDefault>
__global__ void __launch_bounds__(CFG::THREADS, CFG::MINB) r2r_fast_kernel(Geom g, int kind, int tiles_b,
                                                                           const cpx<T> *__restrict__ wt_g,
                                                                           const cpx<T> *__restrict__ ht_g, LD ld, ST st)
{
    using PI = PlanInfo<N>;
    constexpr int W = CFG::W, NL = W / 2;
    constexpr int NT = CFG::THREADS;
    constexpr int V = 16 / sizeof(T);             // elements per 16-byte global access
    constexpr int PERV = N * W / V / NT;          // vector accesses per thread
    constexpr int BATCH = batch_size(PERV, CFG::MAXB);
    static_assert(PERV % BATCH == 0, "tile must split evenly");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T> *buf = reinterpret_cast<cpx<T> *>(smem_raw);
    cpx<T> *wt = buf + NL * PI::LD;               // FFT twiddles W_N^m
    cpx<T> *ht = wt + N;                          // Makhoul twiddles exp(i pi k / 2N)
    T *rb = reinterpret_cast<T *>(smem_raw);
    const TileBase tb = tile_base<AXIS>(g, W, tiles_b);
    const bool fwd = (kind == K_DCT2 || kind == K_DST2);
    const bool sine = (kind == K_DST2 || kind == K_DST3);
    // 16-byte accesses need V | nz (element index alignment); otherwise V = 1 accesses
    const bool vec_ok = (g.nz % V) == 0;
    for (int m = threadIdx.x; m < N; m += NT) {
        wt[m] = wt_g[m];
        ht[m] = ht_g[m];
    }

    // ---- global -> shared.  A vector access covers V consecutive k: V consecutive line
    // positions t (z axis) or V consecutive lines w (x, y axes).  Partial tiles (nz not a
    // multiple of W) fall back to V = 1 accesses through the same code.
#pragma unroll 1
    for (int e0 = 0; e0 < PERV; e0 += BATCH) {
        T vals[BATCH][V];
        int tt[BATCH], ww[BATCH];
#pragma unroll
        for (int b = 0; b < BATCH; b++) {
            const int e = (e0 + b) * NT + threadIdx.x;
            int t, w;
            if (AXIS == 2) { t = (e % (N / V)) * V; w = e / (N / V); }
            else { w = (e % (W / V)) * V; t = e / (W / V); }
            tt[b] = t;
            ww[b] = w;
            const ElemPos p = tile_elem<AXIS>(g, tb, t, w);
            if (vec_ok && (AXIS == 2 || p.k + V <= g.nz)) {
                if (p.valid && idx_ok(g, p.idx, V)) ld.template load<V>(p.idx, p.i, p.j, p.k, vals[b]);
                else {
#pragma unroll
                    for (int u = 0; u < V; u++) vals[b][u] = T(0);
                }
            } else {
#pragma unroll
                for (int u = 0; u < V; u++) {
                    if (p.k + u < g.nz && idx_ok(g, p.idx + u)) ld.template load<1>(p.idx + u, p.i, p.j, p.k + u, &vals[b][u]);
                    else vals[b][u] = T(0);
                }
            }
        }
#pragma unroll
        for (int b = 0; b < BATCH; b++) {
#pragma unroll
            for (int u = 0; u < V; u++) {
                const int t = AXIS == 2 ? tt[b] + u : tt[b];
                const int w = AXIS == 2 ? ww[b] : ww[b] + u;
                T v = vals[b][u];
                int pos;
                if (fwd) {
                    pos = makhoul_pos(t, N);
                    if (sine && (t & 1)) v = -v;
                } else {
                    pos = sine ? N - 1 - t : t;
                }
                rb[2 * ((w >> 1) * PI::LD + PI::phys(pos)) + (w & 1)] = v;
            }
        }
    }
    __syncthreads();

    if (fwd) {
        fft_dif<T, N, false>(buf, NL, wt);
    } else {
        // DCT-III pre-twiddle, in place on pairs (t, N - t): Z_t = V_A[t] + i V_B[t],
        // V[t] = exp(+i pi t / 2N) (X_t - i X_{N-t}), X_N = 0
        constexpr int HALF = N / 2 + 1;
        for (int e = threadIdx.x; e < NL * HALF; e += NT) {
            const int c = e / HALF;
            const int t = e - c * HALF;
            cpx<T> *L = buf + c * PI::LD;
            const int pa = PI::phys(t);
            const int tm = N - t;
            cpx<T> xa = L[pa];
            cpx<T> xb = (t == 0) ? cpx<T>{T(0), T(0)} : L[PI::phys(tm)];
            L[pa] = dct3_pre(xa, xb, ht[t]);
            if (t != 0 && tm != t) L[PI::phys(tm)] = dct3_pre(xb, xa, ht[tm]);
        }
        __syncthreads();
        fft_dif<T, N, true>(buf, NL, wt);
    }

    // ---- shared -> global, output permutation / post-twiddle per kind
    for (int e = threadIdx.x; e < N * W / V; e += NT) {
        int o, w;
        if (AXIS == 2) { o = (e % (N / V)) * V; w = e / (N / V); }
        else { w = (e % (W / V)) * V; o = e / (W / V); }
        const ElemPos p = tile_elem<AXIS>(g, tb, o, w);
        T v[V];
#pragma unroll
        for (int u = 0; u < V; u++) {
            const int oo = AXIS == 2 ? o + u : o;
            const int wu = AXIS == 2 ? w : w + u;
            const cpx<T> *L = buf + (wu >> 1) * PI::LD;
            if (fwd) {
                const int k = sine ? (N - 1 - oo) : oo;
                const cpx<T> zk = L[PI::phys(PI::pos(k))];
                const cpx<T> zm = L[PI::phys(PI::pos(k == 0 ? 0 : N - k))];
                v[u] = dct2_out(zk, zm, ht[k], wu & 1);
            } else {
                const cpx<T> z = L[PI::phys(PI::pos(makhoul_pos(oo, N)))];
                T r = (wu & 1) ? z.y : z.x;
                v[u] = (sine && (oo & 1)) ? -r : r;
            }
        }
        if (!p.valid) continue;
        if (vec_ok && (AXIS == 2 || p.k + V <= g.nz)) {
            if (idx_ok(g, p.idx, V)) st.template store<V>(p.idx, p.i, p.j, p.k, v);
        } else {
#pragma unroll
            for (int u = 0; u < V; u++)
                if (p.k + u < g.nz && idx_ok(g, p.idx + u)) st.template store<1>(p.idx + u, p.i, p.j, p.k + u, &v[u]);
        }
    }
}

}  // namespace smadft
