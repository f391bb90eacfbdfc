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

// natural sample index whose Makhoul position is p (inverse of makhoul_pos)
template <int N>
__device__ __forceinline__ int makhoul_src(int p) { return p < N / 2 ? 2 * p : 2 * (N - 1 - p) + 1; }

template <typename T, int N, int AXIS, class LD, class ST>
__global__ void __launch_bounds__(RdInfo<N>::THREADS, 2) r2r_rd_kernel(Geom g, int kind, int tiles_b, LD ld,
                                                                       const cpx<T> *__restrict__ wt_g,
                                                                       const cpx<T> *__restrict__ ht_g, ST st)
{
    using RI = RdInfo<N>;
    constexpr int R0 = RI::R0, R1 = RI::R1, NT = RI::THREADS;
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
    // tile: 32 k-columns starting at k0 along the non-transformed line coordinate `a`
    const int kt = blockIdx.x % tiles_b;
    const int a = blockIdx.x / tiles_b;
    const int k = kt * 32 + 2 * c;                 // first of the two real lines
    const long long stride = AXIS == 1 ? (long long)g.nz : g.nyz;
    const long long base = (AXIS == 1 ? (long long)a * g.nyz : (long long)a * g.nz) + k;
    const int nk = g.nz - k;                       // real lines of this pair inside the box
    const bool fwd = (kind == K_DCT2 || kind == K_DST2);
    const bool sine = (kind == K_DST2 || kind == K_DST3);
    __syncthreads();

    // the pair of real samples (lines k, k+1) at line position t, packed as one complex;
    // the Loader computes them from its fields (each point is loaded exactly once)
    auto load_pair = [&](int t) -> cpx<T> {
        const long long q = base + (long long)t * stride;
        const int ii = AXIS == 1 ? a : t, jj = AXIS == 1 ? t : a;
        T v[2] = {T(0), T(0)};
        if (nk >= 2) ld.template load<2>(q, ii, jj, k, v);
        else if (nk == 1) ld.template load<1>(q, ii, jj, k, v);
        return {v[0], v[1]};
    };
    cpx<T> v[R0];
    if (fwd) {
        // stage-0 points p = j + q R1 of the Makhoul-permuted sequence
#pragma unroll
        for (int q = 0; q < R0; q++) {
            const int p = j + q * R1;
            const int t = makhoul_src<N>(p);
            cpx<T> x = load_pair(t);
            if (sine && (t & 1)) x = {-x.x, -x.y};
            v[q] = x;
        }
    } else {
        // DCT-III pre-twiddle Z_p = V_A[p] + i V_B[p], V[p] = exp(+i pi p/2N)(X_p - i X_{N-p}),
        // X_N = 0; DST-III reads the line reversed.  X_{N-p} comes from the partner lane (or
        // the thread itself in warp 0); each pair of points is rewritten in place together so
        // only one array stays live.
#pragma unroll
        for (int q = 0; q < R0; q++) {
            const int p = j + q * R1;
            v[q] = load_pair(sine ? N - 1 - p : p);
        }
        auto ztw = [&](int q, cpx<T> xa, cpx<T> xb) -> cpx<T> {
            const cpx<T> hh = ht[j + q * R1];
            const T cc = hh.x, ss = hh.y;
            const T var = cc * xa.x + ss * xb.x, vai = ss * xa.x - cc * xb.x;
            const T vbr = cc * xa.y + ss * xb.y, vbi = ss * xa.y - cc * xb.y;
            return {var - vbi, vai + vbr};
        };
        if (wi != 0 || j == R1 / 2) {
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
    cpx<T> *line = buf + c * RI::LD;
    if (fwd) codelet<R0, T, false>(v);
    else codelet<R0, T, true>(v);
#pragma unroll
    for (int q = 0; q < R0; q++) {
        cpx<T> o = v[q];
        if (q > 0) o = fwd ? cmul(o, tw<T, false>(wt, j * q)) : cmul(o, tw<T, true>(wt, j * q));
        line[RI::phys(j + q * R1)] = o;
    }
    __syncthreads();

    // ---- stage 1: radix R1 over contiguous blocks; block b holds X[b + R0 q] afterwards
    constexpr int BPT = R0 / R1 > 0 ? R0 / R1 : 1;   // blocks per thread
    cpx<T> x1[BPT][R1];
#pragma unroll
    for (int r = 0; r < BPT; r++) {
        const int b = j + r * R1;
        cpx<T> *pb = line + RI::phys(b * R1);
#pragma unroll
        for (int q = 0; q < R1; q++) x1[r][q] = pb[q];
        if (fwd) codelet<R1, T, false>(x1[r]);
        else codelet<R1, T, true>(x1[r]);
    }

    auto store_pair = [&](int o, T A, T B) {
        const long long q = base + (long long)o * stride;
        const int ii = AXIS == 1 ? a : o, jj = AXIS == 1 ? o : a;
        if (nk >= 2) {
            const T w2[2] = {A, B};
            st.template store<2>(q, ii, jj, k, w2);
        } else if (nk == 1) {
            st.template store<1>(q, ii, jj, k, &A);
        }
    };

    if (!fwd) {
        // DCT-III output y[2m] = v[m], y[2m+1] = v[N-1-m]; DST-III negates odd outputs
#pragma unroll
        for (int r = 0; r < BPT; r++) {
            const int b = j + r * R1;
#pragma unroll
            for (int q = 0; q < R1; q++) {
                const int m = b + R0 * q;
                const int o = m < N / 2 ? 2 * m : 2 * (N - 1 - m) + 1;
                cpx<T> z = x1[r][q];
                if (sine && (o & 1)) z = {-z.x, -z.y};
                store_pair(o, z.x, z.y);
            }
        }
        return;
    }
    // forward: DCT-II post-twiddle pairs X[k] with X[N-k].  With one block per thread the
    // partner is lane ^ 16 (or the thread itself in warp 0); otherwise through shared memory.
    if constexpr (BPT == 1) {
        // block j holds X[j + R0 q]; X[N - k] is block R1 - j at q' = R1 - 1 - q (lane ^ 16, or
        // this thread for j = R1/2), and block 0 at q' = (R1 - q) mod R1 for j = 0
        auto emit = [&](int q, cpx<T> zm) {
            const int kk = j + R0 * q;
            const cpx<T> zk = x1[0][q];
            const cpx<T> hh = ht[kk];
            store_pair(sine ? N - 1 - kk : kk, dct2_out(zk, zm, hh, 0), dct2_out(zk, zm, hh, 1));
        };
        if (wi != 0) {
#pragma unroll
            for (int q = 0; q < R1; q++) {
                cpx<T> zm;
                zm.x = __shfl_xor_sync(0xffffffffu, x1[0][R1 - 1 - q].x, 16);
                zm.y = __shfl_xor_sync(0xffffffffu, x1[0][R1 - 1 - q].y, 16);
                emit(q, zm);
            }
        } else if (j == R1 / 2) {
#pragma unroll
            for (int q = 0; q < R1; q++) emit(q, x1[0][R1 - 1 - q]);
        } else {
#pragma unroll
            for (int q = 0; q < R1; q++) emit(q, x1[0][(R1 - q) % R1]);
        }
    } else {
        // each thread rewrites only its own blocks, so no barrier is needed before this
#pragma unroll
        for (int r = 0; r < BPT; r++) {
            const int b = j + r * R1;
            cpx<T> *pb = line + RI::phys(b * R1);
#pragma unroll
            for (int q = 0; q < R1; q++) pb[q] = x1[r][q];
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < BPT; r++) {
            const int b = j + r * R1;
#pragma unroll
            for (int q = 0; q < R1; q++) {
                const int kk = b + R0 * q;
                const int km = kk == 0 ? 0 : N - kk;
                const cpx<T> zk = x1[r][q];
                const cpx<T> zm = line[RI::phys((km % R0) * R1 + km / R0)];
                const cpx<T> hh = ht[kk];
                const T A = dct2_out(zk, zm, hh, 0), B = dct2_out(zk, zm, hh, 1);
                store_pair(sine ? N - 1 - kk : kk, A, B);
            }
        }
    }
}

}  // namespace smadft
