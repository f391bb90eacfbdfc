// fft_tile.cuh -- shared-memory building blocks of the axis-pass r2r kernels.
//
// An axis pass transforms every line of an nx*ny*nz field along one axis with one of the
// four FFTW r2r kinds the reference plans (REDFT10/01, RODFT10/01; no-adv/
// cosNoAdvTrackSing.cpp:342-375, adv/cosAdvTrackMult.cpp:419-467):
//
//   REDFT10 (DCT-II):  Y_k = 2 sum_j X_j cos(pi (j+1/2) k / n)
//   REDFT01 (DCT-III): Y_k = X_0 + 2 sum_{j>0} X_j cos(pi j (k+1/2) / n)
//   RODFT10 (DST-II):  Y_k = DCT-II[(-1)^j X_j]_{n-1-k}
//   RODFT01 (DST-III): Y_k = (-1)^k DCT-III[X_{n-1-j}]_k
//
// The cosine kinds run as an n-point complex FFT with Makhoul's reordering (IEEE TASSP
// 28(1), 1980): DCT-II permutes the input (even samples forward, odd samples backward),
// FFTs, and post-multiplies by exp(-i pi k / 2n); DCT-III pre-multiplies by
// exp(+i pi k / 2n) (X_k - i X_{n-k}), inverse-FFTs and un-permutes.  Two real lines
// travel as the real and imaginary parts of one complex line and are separated by
// Hermitian symmetry, so no arithmetic is spent on zero imaginary parts.
//
// The complex FFT is a Stockham auto-sort in shared memory with radix-4/2/3/5 stages
// (lengths 2^a 3^b 5^c; the grids here are 16..256).  Twiddles come from tables the host
// computes in FP64 and converts once to the compute type.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace smadft {

template <typename T>
struct cpx {
    T x, y;
};

enum R2RKind : int { K_DCT2 = 0, K_DCT3 = 1, K_DST2 = 2, K_DST3 = 3 };

constexpr int kMaxStages = 12;

// Per-length FFT plan (radix sequence) plus device twiddle tables.
template <typename T>
struct LinePlan {
    int n;
    int nst;
    int radix[kMaxStages];
    const cpx<T> *w;   // w[m]  = (cos 2 pi m/n, -sin 2 pi m/n)   m < n
    const cpx<T> *h;   // h[k]  = (cos pi k/2n,   sin pi k/2n)    k < n
};

template <typename T>
__device__ __forceinline__ cpx<T> cmul(cpx<T> a, cpx<T> b)
{
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}

// forward twiddle w^e or its conjugate for the inverse transform
template <typename T, bool INV>
__device__ __forceinline__ cpx<T> tw(const cpx<T> *__restrict__ w, int e)
{
    cpx<T> t = w[e];
    if (INV) t.y = -t.y;
    return t;
}

// Size-R DFT in registers.  Forward uses exp(-2 pi i/R), inverse exp(+2 pi i/R).
template <int R, typename T, bool INV>
__device__ __forceinline__ void dft(cpx<T> *v)
{
    if (R == 2) {
        cpx<T> a = v[0], b = v[1];
        v[0] = {a.x + b.x, a.y + b.y};
        v[1] = {a.x - b.x, a.y - b.y};
    } else if (R == 4) {
        cpx<T> s0 = {v[0].x + v[2].x, v[0].y + v[2].y};
        cpx<T> d0 = {v[0].x - v[2].x, v[0].y - v[2].y};
        cpx<T> s1 = {v[1].x + v[3].x, v[1].y + v[3].y};
        cpx<T> d1 = {v[1].x - v[3].x, v[1].y - v[3].y};
        // forward: X1 = d0 - i d1 ; inverse: X1 = d0 + i d1
        cpx<T> j = INV ? cpx<T>{-d1.y, d1.x} : cpx<T>{d1.y, -d1.x};
        v[0] = {s0.x + s1.x, s0.y + s1.y};
        v[2] = {s0.x - s1.x, s0.y - s1.y};
        v[1] = {d0.x + j.x, d0.y + j.y};
        v[3] = {d0.x - j.x, d0.y - j.y};
    } else if (R == 3) {
        const T h = T(0.86602540378443864676372317075294);  // sin(2 pi/3)
        cpx<T> t1 = {v[1].x + v[2].x, v[1].y + v[2].y};
        cpx<T> d = {v[1].x - v[2].x, v[1].y - v[2].y};
        cpx<T> m = {v[0].x - T(0.5) * t1.x, v[0].y - T(0.5) * t1.y};
        // forward: X1 = m - i h d ; X2 = m + i h d
        cpx<T> q = INV ? cpx<T>{-h * d.y, h * d.x} : cpx<T>{h * d.y, -h * d.x};
        v[0] = {v[0].x + t1.x, v[0].y + t1.y};
        v[1] = {m.x + q.x, m.y + q.y};
        v[2] = {m.x - q.x, m.y - q.y};
    } else if (R == 5) {
        const T c1 = T(0.30901699437494742410229341718282);   // cos(2 pi/5)
        const T c2 = T(-0.80901699437494742410229341718282);  // cos(4 pi/5)
        const T s1 = T(0.95105651629515357211643933337938);   // sin(2 pi/5)
        const T s2 = T(0.58778525229247312916870595463907);   // sin(4 pi/5)
        cpx<T> t1 = {v[1].x + v[4].x, v[1].y + v[4].y};
        cpx<T> t2 = {v[2].x + v[3].x, v[2].y + v[3].y};
        cpx<T> t3 = {v[1].x - v[4].x, v[1].y - v[4].y};
        cpx<T> t4 = {v[2].x - v[3].x, v[2].y - v[3].y};
        cpx<T> a1 = {v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y};
        cpx<T> a2 = {v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y};
        cpx<T> b1 = {s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y};
        cpx<T> b2 = {s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y};
        // forward: X1 = a1 - i b1, X4 = a1 + i b1, X2 = a2 - i b2, X3 = a2 + i b2
        cpx<T> ib1 = INV ? cpx<T>{-b1.y, b1.x} : cpx<T>{b1.y, -b1.x};
        cpx<T> ib2 = INV ? cpx<T>{-b2.y, b2.x} : cpx<T>{b2.y, -b2.x};
        v[0] = {v[0].x + t1.x + t2.x, v[0].y + t1.y + t2.y};
        v[1] = {a1.x + ib1.x, a1.y + ib1.y};
        v[4] = {a1.x - ib1.x, a1.y - ib1.y};
        v[2] = {a2.x + ib2.x, a2.y + ib2.y};
        v[3] = {a2.x - ib2.x, a2.y - ib2.y};
    }
}

// One Stockham stage of radix R over `nlines` lines of length n (line stride ld).
template <int R, typename T, bool INV>
__device__ __forceinline__ void stockham_stage(const cpx<T> *__restrict__ a, cpx<T> *__restrict__ b,
                                               int nlines, int ld, int n, int ns,
                                               const cpx<T> *__restrict__ w)
{
    const int m = n / R;
    const int tstep = n / (ns * R);
    const int tasks = nlines * m;
    for (int t = threadIdx.x; t < tasks; t += blockDim.x) {
        const int c = t / m;
        const int j = t - c * m;
        const int k = j % ns;
        const cpx<T> *src = a + c * ld;
        cpx<T> *dst = b + c * ld;
        cpx<T> v[R];
#pragma unroll
        for (int q = 0; q < R; q++) {
            cpx<T> x = src[j + q * m];
            v[q] = (q == 0 || k == 0) ? x : cmul(x, tw<T, INV>(w, k * q * tstep));
        }
        dft<R, T, INV>(v);
        const int d = (j / ns) * ns * R + k;
#pragma unroll
        for (int q = 0; q < R; q++) dst[d + q * ns] = v[q];
    }
}

// Complex FFT of `nlines` lines held in shared memory.  Data starts in *a; *b is scratch.
// Returns the buffer holding the result.  Ends with a __syncthreads().
template <typename T, bool INV>
__device__ cpx<T> *fft_lines(cpx<T> *a, cpx<T> *b, int nlines, int ld, const LinePlan<T> &P)
{
    int ns = 1;
    for (int s = 0; s < P.nst; s++) {
        const int r = P.radix[s];
        switch (r) {
        case 4: stockham_stage<4, T, INV>(a, b, nlines, ld, P.n, ns, P.w); break;
        case 2: stockham_stage<2, T, INV>(a, b, nlines, ld, P.n, ns, P.w); break;
        case 3: stockham_stage<3, T, INV>(a, b, nlines, ld, P.n, ns, P.w); break;
        default: stockham_stage<5, T, INV>(a, b, nlines, ld, P.n, ns, P.w); break;
        }
        __syncthreads();
        cpx<T> *t = a;
        a = b;
        b = t;
        ns *= r;
    }
    return a;
}

// Position of input sample t in the Makhoul-permuted sequence (also the DCT-III output map).
__device__ __forceinline__ int makhoul_pos(int t, int n) { return (t & 1) ? (n - 1 - (t >> 1)) : (t >> 1); }

}  // namespace smadft
