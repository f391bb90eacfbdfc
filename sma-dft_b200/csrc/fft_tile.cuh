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

// ---- complex arithmetic on the packed (real, imaginary) pair -----------------------------
// FP32 sums, differences and real-scalar multiply-adds of a pair run as one packed two-lane
// instruction (sm_100: add / sub / mul / fma .rn.f32x2), which rounds each lane exactly as the
// scalar instruction would; FP64 stays scalar.
template <typename T>
__device__ __forceinline__ cpx<T> mul_mi(cpx<T> a) { return {a.y, -a.x}; }   // -i a
template <typename T>
__device__ __forceinline__ cpx<T> mul_pi(cpx<T> a) { return {-a.y, a.x}; }   // +i a
template <typename T>
__device__ __forceinline__ cpx<T> cadd(cpx<T> a, cpx<T> b) { return {a.x + b.x, a.y + b.y}; }
template <typename T>
__device__ __forceinline__ cpx<T> csub(cpx<T> a, cpx<T> b) { return {a.x - b.x, a.y - b.y}; }
// a + s b, s real (one rounding per lane)
template <typename T>
__device__ __forceinline__ cpx<T> caxpy(cpx<T> a, T s, cpx<T> b) { return {fma(s, b.x, a.x), fma(s, b.y, a.y)}; }
// s b, s real
template <typename T>
__device__ __forceinline__ cpx<T> cscale(T s, cpx<T> b) { return {s * b.x, s * b.y}; }

// lane-wise product and multiply-add of two pairs (a.x b.x, a.y b.y) and (a.x b.x + c.x, ...):
// two independent real values carried as one pair (two points of a loader)
template <typename T>
__device__ __forceinline__ cpx<T> pmul(cpx<T> a, cpx<T> b) { return {a.x * b.x, a.y * b.y}; }
template <typename T>
__device__ __forceinline__ cpx<T> pfma(cpx<T> a, cpx<T> b, cpx<T> c) { return {fma(a.x, b.x, c.x), fma(a.y, b.y, c.y)}; }

__device__ __forceinline__ unsigned long long pk2(cpx<float> a)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ cpx<float> upk2(unsigned long long r)
{
    cpx<float> a;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
    return a;
}
template <>
__device__ __forceinline__ cpx<float> cadd<float>(cpx<float> a, cpx<float> b)
{
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)));
    return upk2(r);
}
template <>
__device__ __forceinline__ cpx<float> csub<float>(cpx<float> a, cpx<float> b)
{
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)));
    return upk2(r);
}
template <>
__device__ __forceinline__ cpx<float> caxpy<float>(cpx<float> a, float s, cpx<float> b)
{
    unsigned long long r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pk2(b)), "l"(pk2(cpx<float>{s, s})), "l"(pk2(a)));
    return upk2(r);
}
template <>
__device__ __forceinline__ cpx<float> cscale<float>(float s, cpx<float> b)
{
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(cpx<float>{s, s})), "l"(pk2(b)));
    return upk2(r);
}

// DCT-III pre-twiddle of a packed pair of lines (line A in the real parts, line B in the
// imaginary parts): Z_t = V_A[t] + i V_B[t] with V[t] = exp(+i pi t/2n) (X_t - i X_{n-t}).
// With xa = X_t and xb = X_{n-t} of both lines and h = exp(+i pi t/2n) this is
// Z_t = h (xa - i xb): one complex product.
template <typename T>
__device__ __forceinline__ cpx<T> dct3_pre(cpx<T> xa, cpx<T> xb, cpx<T> h)
{
    return cmul(cpx<T>{xa.x + xb.y, xa.y - xb.x}, h);
}

// DCT-II post-twiddle of a packed pair of lines: the outputs (line A, line B) at k from
// Z_k, Z_{n-k} and h = (cos, sin) of pi k/2n, with P = Z_k + Z_{n-k}, D = Z_k - Z_{n-k}:
//   A_k = h.x P.x + h.y D.y,   B_k = h.x P.y - h.y D.x
template <typename T>
__device__ __forceinline__ cpx<T> dct2_post(cpx<T> zk, cpx<T> zm, cpx<T> h)
{
    const cpx<T> p = cadd(zk, zm), d = csub(zk, zm);
    return {fma(h.y, d.y, h.x * p.x), fma(-h.y, d.x, h.x * p.y)};
}

template <>
__device__ __forceinline__ cpx<float> pmul<float>(cpx<float> a, cpx<float> b)
{
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)));
    return upk2(r);
}
template <>
__device__ __forceinline__ cpx<float> pfma<float>(cpx<float> a, cpx<float> b, cpx<float> c)
{
    unsigned long long r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)), "l"(pk2(c)));
    return upk2(r);
}

// Size-R DFT in registers.  Forward uses exp(-2 pi i/R), inverse exp(+2 pi i/R).
template <int R, typename T, bool INV>
__device__ __forceinline__ void dft(cpx<T> *v)
{
    if (R == 2) {
        const cpx<T> a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if (R == 4) {
        const cpx<T> s0 = cadd(v[0], v[2]), d0 = csub(v[0], v[2]);
        const cpx<T> s1 = cadd(v[1], v[3]), d1 = csub(v[1], v[3]);
        // forward: X1 = d0 - i d1 ; inverse: X1 = d0 + i d1
        const cpx<T> j = INV ? mul_pi(d1) : mul_mi(d1);
        v[0] = cadd(s0, s1);
        v[2] = csub(s0, s1);
        v[1] = cadd(d0, j);
        v[3] = csub(d0, j);
    } else if (R == 3) {
        const T h = T(0.86602540378443864676372317075294);  // sin(2 pi/3)
        const cpx<T> t1 = cadd(v[1], v[2]), d = csub(v[1], v[2]);
        const cpx<T> m = caxpy(v[0], T(-0.5), t1);
        // forward: X1 = m - i h d ; X2 = m + i h d
        const cpx<T> hd = cscale(h, d);
        const cpx<T> q = INV ? mul_pi(hd) : mul_mi(hd);
        v[0] = cadd(v[0], t1);
        v[1] = cadd(m, q);
        v[2] = csub(m, q);
    } else if (R == 5) {
        const T c1 = T(0.30901699437494742410229341718282);   // cos(2 pi/5)
        const T c2 = T(-0.80901699437494742410229341718282);  // cos(4 pi/5)
        const T s1 = T(0.95105651629515357211643933337938);   // sin(2 pi/5)
        const T s2 = T(0.58778525229247312916870595463907);   // sin(4 pi/5)
        const cpx<T> t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        const cpx<T> t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        const cpx<T> a1 = caxpy(caxpy(v[0], c1, t1), c2, t2);
        const cpx<T> a2 = caxpy(caxpy(v[0], c2, t1), c1, t2);
        const cpx<T> b1 = caxpy(cscale(s1, t3), s2, t4);
        const cpx<T> b2 = caxpy(cscale(s2, t3), -s1, t4);
        // forward: X1 = a1 - i b1, X4 = a1 + i b1, X2 = a2 - i b2, X3 = a2 + i b2
        const cpx<T> ib1 = INV ? mul_pi(b1) : mul_mi(b1);
        const cpx<T> ib2 = INV ? mul_pi(b2) : mul_mi(b2);
        v[0] = cadd(cadd(v[0], t1), t2);
        v[1] = cadd(a1, ib1);
        v[4] = csub(a1, ib1);
        v[2] = cadd(a2, ib2);
        v[3] = csub(a2, ib2);
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
