// adjoint.cu -- hand-written adjoints of the diffusive (noadv) and advected (adv)
// semi-implicit steps; the noadv derivation first, the adv one above adv_adjoint.
//
// Forward (scaled spectral state, no-adv/cosNoAdvTrackSing.cpp:618-635,688-764):
//   pre-loop   psihat_0 = s CT(psi_0),  Nhat_{-1} = CT f(psi_0)          (s = scale)
//   step n     Nhat_n = CT f(psi_n),  psihat_{n+1} = A psihat_n + B (3 Nhat_n - Nhat_{n-1}),
//              psi_{n+1} = iCT psihat_{n+1}     (psi_0 is the initial condition itself)
//   with A = (1 + h L)/(1 - h L), B = h s/(1 - h L), h = dt/2, L = eps - alpha (q^2 - q0^2)^2,
//   f(psi) = beta psi^3 - gamma psi^5, CT = REDFT10^3, iCT = REDFT01^3.
// Loss J: mean sub-grid interface position (in lambda0) over the columns the tracker finds
// on psi_T (the found set and crossing cells held fixed, as a central difference sees them).
// Reverse, lambda_n = dJ/dpsihat_n, mu_n = dJ/dNhat_n:
//   lambda_T = iCT^T g_T (g_T = dJ/dpsi_T);  mu_n = 3 B lambda_{n+1} - B lambda_{n+2};
//   lambda_n = A lambda_{n+1} + iCT^T (f'(psi_n) CT^T mu_n)  (n >= 1);  lambda_0 = A lambda_1;
//   dJ/dpsi_0 = s CT^T lambda_0 + f'(psi_0) CT^T (mu_0 + mu_{-1}),  mu_{-1} = -B lambda_1;
//   dJ/dbeta = sum_n <CT^T mu_n, psi_n^3>, dJ/dgamma = -sum_n <CT^T mu_n, psi_n^5>
//   (n = 0 with mu_0 + mu_{-1}); dJ/deps, dJ/dalpha = sum_n <lambda_{n+1}, dA/dL psihat_n +
//   (dB/dL / B)(psihat_{n+1} - A psihat_n)> dL/d(eps, alpha).
// Transposes: REDFT10^T = REDFT01 diag(2, 1, ..., 1) and REDFT01^T = diag(1/2, 1, ..., 1)
// REDFT10 per axis, so CT^T x = REDFT01^3(W x) and iCT^T y = U REDFT10^3(y) with the
// separable weights W = w_i w_j w_k (w_0 = 2), U = u_i u_j u_k (u_0 = 1/2).
// Memory: the forward keeps psihat and Nhat_prev every K steps; the reverse sweep re-runs
// each segment from its checkpoint and keeps that segment's psihat and psi.
#include "models.cuh"
#include "reduce.cuh"
#include "steps.h"

namespace smadft {

namespace {

__device__ __forceinline__ double wsep(int i, int j, int k, double w0)
{
    return (i == 0 ? w0 : 1.0) * (j == 0 ? w0 : 1.0) * (k == 0 ? w0 : 1.0);
}

// W (a B lambda1 + b B lambda2) (useB) or W a lambda1 (!useB): input of CT^T = REDFT01^3
template <typename T>
struct LdAdjIn {
    Spec<double> s;
    const double *__restrict__ l1, *__restrict__ l2;   // l2 may be null
    double a, b;
    int useB;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int i, int j, int k, T *out) const
    {
        double x[V], y[V];
        vld<double, V>(l1, q, x);
        if (l2) vld<double, V>(l2, q, y);
#pragma unroll
        for (int u = 0; u < V; u++) {
            double v = a * x[u] + (l2 ? b * y[u] : 0.0);
            if (useB) v *= s.dtd2 * s.scale / (1.0 - s.dtd2 * s.alin(i, j, k + u));
            out[u] = T(wsep(i, j, k + u, 2.0) * v);
        }
    }
};

// f'(psi) t, f'(psi) = 3 beta psi^2 - 5 gamma psi^4 (input of iCT^T)
template <typename T>
struct LdFprime {
    const T *__restrict__ t, *__restrict__ psi;
    T beta, gamma;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int, int, int, T *out) const
    {
        T a[V], p[V];
        vld<T, V>(t, q, a);
        vld<T, V>(psi, q, p);
#pragma unroll
        for (int u = 0; u < V; u++) {
            const T p2 = p[u] * p[u];
            out[u] = a[u] * (T(3) * beta * p2 - T(5) * gamma * p2 * p2);
        }
    }
};

// lambda_out = A lambda_in + U y (lambda_in null: U y), FP64
template <typename T>
struct StAdjLam {
    Spec<double> s;
    const double *__restrict__ lin;
    double *__restrict__ lout;
    static constexpr int PRE = 1;
    using Pre = double;
    template <int V>
    __device__ __forceinline__ void pre(idx_t q, int, int, int, double *buf) const
    {
        if (lin) vld<double, V>(lin, q, buf);
        else
#pragma unroll
            for (int u = 0; u < V; u++) buf[u] = 0.0;
    }
    template <int V>
    __device__ __forceinline__ void fin(idx_t q, int i, int j, int k, const T *v, const double *buf) const
    {
        double o[V];
#pragma unroll
        for (int u = 0; u < V; u++) {
            const double hl = s.dtd2 * s.alin(i, j, k + u);
            o[u] = (1.0 + hl) / (1.0 - hl) * buf[u] + wsep(i, j, k + u, 0.5) * double(v[u]);
        }
        vst<double, V>(lout, q, o);
    }
    template <int V>
    __device__ __forceinline__ void store(idx_t q, int i, int j, int k, const T *v) const
    {
        double buf[V];
        pre<V>(q, i, j, k, buf);
        fin<V>(q, i, j, k, v, buf);
    }
};

// sums <t, psi^3>, <t, psi^5>
template <typename T>
struct RedBetaGamma {
    const T *__restrict__ t, *__restrict__ psi;
    __device__ __forceinline__ void operator()(long long q, double *acc) const
    {
        const double a = double(t[q]), p = double(psi[q]), p3 = p * p * p;
        acc[0] += a * p3;
        acc[1] += a * p3 * p * p;
    }
};

// sums over modes of lambda1 (dA/dL ph0 + (dB/dL / B)(ph1 - A ph0)) and the same times dL/dalpha
struct RedEpsAlpha {
    Spec<double> s;
    const double *__restrict__ l1, *__restrict__ ph0, *__restrict__ ph1;
    __device__ __forceinline__ void operator()(long long q, double *acc) const
    {
        const int k = (int)(q % s.nz);
        const int j = (int)((q / s.nz) % s.ny);
        const int i = (int)(q / ((long long)s.nz * s.ny));
        const double L = s.alin(i, j, k), h = s.dtd2, den = 1.0 - h * L;
        const double A = (1.0 + h * L) / den;
        const double term = l1[q] * (2.0 * h / (den * den) * ph0[q] + h / den * (ph1[q] - A * ph0[q]));
        const double d = s.mq2(i, j, k) - s.q02;
        acc[0] += term;
        acc[1] += term * (-(d * d));
    }
};

// derivative of the mean interface position (lambda0 units) with respect to psi_T on the
// found columns: two entries per column (the tracker's linear interpolation)
template <typename T>
__global__ void interface_seed(const T *__restrict__ f, int na, int nb, int nl, long long sa, long long sb,
                               long long sl, int mode, double hi, double lo, double w, T *__restrict__ g)
{
    const long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= (long long)na * nb) return;
    const int a = (int)(col / nb), b = (int)(col % nb);
    const long long c0 = a * sa + b * sb;
    auto V = [&](int t) -> double { return (double)f[c0 + (long long)t * sl]; };
    if (mode == SMADFT_TRACK_FLAT) {
        int track = 0;
        for (int t = nl - 1; t >= 0; t--) {
            const double v = V(t);
            if (v > hi && track == 0) track = 1;
            if (v < lo && track == 1) {
                if (t + 1 >= nl) break;
                const double v1 = V(t + 1), d = v1 - v;
                g[c0 + (long long)t * sl] = T(w * (lo - v1) / (d * d));
                g[c0 + (long long)(t + 1) * sl] = T(w * (v - lo) / (d * d));
                break;
            }
        }
    } else if (mode == SMADFT_TRACK_BUMP) {
        for (int t = nl - 1; t >= 0; t--) {
            if (fabs(V(t)) > hi) {
                int t3 = t;
                while (t3 < nl - 1 && fabs(V(t3)) > lo) t3++;
                if (t3 > t) {
                    const double x0 = V(t3 - 1), x1 = V(t3);
                    const double f0 = fabs(x0), f1 = fabs(x1), d = f0 - f1;
                    g[c0 + (long long)(t3 - 1) * sl] = T(w * (x0 < 0 ? -1.0 : 1.0) * (lo - f1) / (d * d));
                    g[c0 + (long long)t3 * sl] = T(w * (x1 < 0 ? -1.0 : 1.0) * (f0 - lo) / (d * d));
                }
                break;
            }
        }
    }
}

// lambda_0 = A lambda_1
__global__ void adj_lambda0(Spec<double> s, const double *__restrict__ l1, double *__restrict__ l0, long long n)
{
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(q % s.nz), j = (int)((q / s.nz) % s.ny), i = (int)(q / ((long long)s.nz * s.ny));
        const double hl = s.dtd2 * s.alin(i, j, k);
        l0[q] = (1.0 + hl) / (1.0 - hl) * l1[q];
    }
}

// dpsi0 = s_ct + f'(psi0) t0 (FP64 out)
template <typename T>
__global__ void adj_dpsi0(const T *__restrict__ s_ct, const T *__restrict__ t0, const T *__restrict__ psi0,
                          double beta, double gamma, double *__restrict__ out, long long n)
{
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const double p = double(psi0[q]), p2 = p * p;
        out[q] = double(s_ct[q]) + (3.0 * beta * p2 - 5.0 * gamma * p2 * p2) * double(t0[q]);
    }
}

// ---- advected model (adv_adjoint) -------------------------------------------------------

// Separable end weight of a 3-D transform with its sine along axis `sine` (-1: none): w at
// index 0 of each cosine axis and at the last index of the sine axis.  The transposes are
// REDFT01^T = (1/2 at 0) REDFT10, RODFT01^T = (1/2 at n-1) RODFT10, REDFT10^T = REDFT01 (2 at
// 0) and RODFT10^T = RODFT01 (2 at n-1), per axis.
template <class S>
__device__ __forceinline__ double wend(const S &s, int i, int j, int k, int sine, double w)
{
    const double a = (sine == 0 ? i == s.nx - 1 : i == 0) ? w : 1.0;
    const double b = (sine == 1 ? j == s.ny - 1 : j == 0) ? w : 1.0;
    const double c = (sine == 2 ? k == s.nz - 1 : k == 0) ? w : 1.0;
    return a * b * c;
}

// -t g_c: the velocity adjoint in real space (N = f(psi) - v . grad psi)
template <typename T, int AX>
struct LdNegTG {
    const T *__restrict__ t, *__restrict__ g;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int, int, int, T *out) const
    {
        T a[V], b[V];
        vld<T, V>(t, q, a);
        vld<T, V>(g, q, b);
#pragma unroll
        for (int u = 0; u < V; u++) out[u] = -a[u] * b[u];
    }
};

// Transpose of the Stokes projection (adv/cosAdvTrackMult.cpp:1103-1274 on one rank, the map
// LdStokes<AX, false> applies): from the velocity-spectrum adjoints a_c = ST_c(-t g_c) (their
// end weights U_c = 1/2 applied here, at each read) to the force-spectrum adjoint of
// component AX, times the end weights W_AX = 2 of ST_AX^T = iST_AX W_AX.  The forward map
//   v_x = snu cx ((1 - s_i^2 cx) Sx - s_i cx (q_j Sy[i+1,j-1,k] + q_k Sz[i+1,j,k-1]))
// (and its y, z analogues, with their truncations) read backwards: every read below is the
// transpose of one forward read, under the same index conditions.
template <typename T, int AX>
struct LdStokesT {
    Spec<T> s;
    const T *__restrict__ ax, *__restrict__ ay, *__restrict__ az;
    __device__ __forceinline__ T cxf(int a, int b, int c) const { return T(1) / (s.sx[a] * s.sx[a] + s.qy[b] * s.qy[b] + s.qz[c] * s.qz[c]); }
    __device__ __forceinline__ T cyf(int a, int b, int c) const { return T(1) / (s.qx[a] * s.qx[a] + s.sy[b] * s.sy[b] + s.qz[c] * s.qz[c]); }
    __device__ __forceinline__ T czf(int a, int b, int c) const { return T(1) / (s.qx[a] * s.qx[a] + s.qy[b] * s.qy[b] + s.sz[c] * s.sz[c]); }
    __device__ __forceinline__ T U(int a, int b, int c, int sine) const { return T(wend(s, a, b, c, sine, 0.5)); }
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int i, int j, int k, T *out) const
    {
        const T snu = s.scale / s.nu;
        const int nx = s.nx, ny = s.ny, nz = s.nz, nyz = s.nyz;
#pragma unroll
        for (int u = 0; u < V; u++) {
            const int kk = k + u;
            const idx_t qq = q + u;
            T v = T(0);
            if (AX == 0) {
                if (i <= nx - 2) {
                    const T cx = cxf(i, j, kk);
                    v = U(i, j, kk, 0) * ax[qq] * snu * cx * (T(1) - s.sx[i] * s.sx[i] * cx);
                    if (j >= 1 && kk <= nz - 2) {       // v_y[i+1, j-1, k] read Sx[i, j, k]
                        const T cy = cyf(i + 1, j - 1, kk);
                        v += U(i + 1, j - 1, kk, 1) * ay[qq + nyz - nz] * (-snu * cy * cy * s.sy[j - 1] * s.qx[i + 1]);
                    }
                    if (j <= ny - 2 && kk >= 1) {       // v_z[i+1, j, k-1] read Sx[i, j, k]
                        const T cz = czf(i + 1, j, kk - 1);
                        v += U(i + 1, j, kk - 1, 2) * az[qq + nyz - 1] * (-snu * cz * cz * s.sz[kk - 1] * s.qx[i + 1]);
                    }
                }
            } else if (AX == 1) {
                if (j <= ny - 2 && kk <= nz - 2) {
                    const T cy = cyf(i, j, kk);
                    v = U(i, j, kk, 1) * ay[qq] * snu * cy * (T(1) - s.sy[j] * s.sy[j] * cy);
                }
                if (i >= 1 && j <= ny - 2) {            // v_x[i-1, j+1, k] read Sy[i, j, k]
                    const T cx = cxf(i - 1, j + 1, kk);
                    v += U(i - 1, j + 1, kk, 0) * ax[qq - nyz + nz] * (-snu * cx * cx * s.sx[i - 1] * s.qy[j + 1]);
                }
                if (j <= ny - 3 && kk >= 1) {           // v_z[i, j+1, k-1] read Sy[i, j, k]
                    const T cz = czf(i, j + 1, kk - 1);
                    v += U(i, j + 1, kk - 1, 2) * az[qq + nz - 1] * (-snu * cz * cz * s.sz[kk - 1] * s.qy[j + 1]);
                }
            } else {
                if (j <= ny - 2 && kk <= nz - 2) {
                    const T cz = czf(i, j, kk);
                    v = U(i, j, kk, 2) * az[qq] * snu * cz * (T(1) - s.sz[kk] * s.sz[kk] * cz);
                }
                if (i >= 1 && kk <= nz - 2) {           // v_x[i-1, j, k+1] read Sz[i, j, k]
                    const T cx = cxf(i - 1, j, kk + 1);
                    v += U(i - 1, j, kk + 1, 0) * ax[qq - nyz + 1] * (-snu * cx * cx * s.sx[i - 1] * s.qz[kk + 1]);
                }
                if (j >= 1 && kk <= nz - 3) {           // v_y[i, j-1, k+1] read Sz[i, j, k]
                    const T cy = cyf(i, j - 1, kk + 1);
                    v += U(i, j - 1, kk + 1, 1) * ay[qq - nz + 1] * (-snu * cy * cy * s.sy[j - 1] * s.qz[kk + 1]);
                }
            }
            out[u] = T(wend(s, i, j, kk, AX, 2.0)) * v;
        }
    }
};

// a_psi = f'(psi) (t - a_mu), a_mu = sum_c a_Sc g_c (psi enters N directly and mu = Sp2 - f(psi))
template <typename T>
struct LdAdjPsi {
    static constexpr int kMinBlocks = 2;
    const T *__restrict__ t, *__restrict__ sx, *__restrict__ sy, *__restrict__ sz;
    const T *__restrict__ gx, *__restrict__ gy, *__restrict__ gz, *__restrict__ psi;
    T beta, gamma;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int, int, int, T *out) const
    {
        T a[V], b[V], c[V], d[V], e[V], f[V], g[V], p[V];
        vld<T, V>(t, q, a);
        vld<T, V>(sx, q, b); vld<T, V>(gx, q, e);
        vld<T, V>(sy, q, c); vld<T, V>(gy, q, f);
        vld<T, V>(sz, q, d); vld<T, V>(gz, q, g);
        vld<T, V>(psi, q, p);
#pragma unroll
        for (int u = 0; u < V; u++) {
            const T p2 = p[u] * p[u];
            out[u] = (T(3) * beta * p2 - T(5) * gamma * p2 * p2) * (a[u] - (b[u] * e[u] + c[u] * f[u] + d[u] * g[u]));
        }
    }
};

// a_mu = sum_c a_Sc g_c (S_c = mu g_c); its spectrum enters through Sp2 = iCT(-L psihat)
template <typename T>
struct LdAdjMu {
    const T *__restrict__ sx, *__restrict__ sy, *__restrict__ sz;
    const T *__restrict__ gx, *__restrict__ gy, *__restrict__ gz;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int, int, int, T *out) const
    {
        T b[V], c[V], d[V], e[V], f[V], g[V];
        vld<T, V>(sx, q, b); vld<T, V>(gx, q, e);
        vld<T, V>(sy, q, c); vld<T, V>(gy, q, f);
        vld<T, V>(sz, q, d); vld<T, V>(gz, q, g);
#pragma unroll
        for (int u = 0; u < V; u++) out[u] = b[u] * e[u] + c[u] * f[u] + d[u] * g[u];
    }
};

// a_gc = -t v_c + a_Sc mu, mu = Sp2 - f(psi): the adjoint of the gradient component c
template <typename T, int AX>
struct LdAdjG {
    const T *__restrict__ t, *__restrict__ v, *__restrict__ as, *__restrict__ sp2, *__restrict__ psi;
    T beta, gamma;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int, int, int, T *out) const
    {
        T a[V], b[V], c[V], d[V], p[V];
        vld<T, V>(t, q, a);
        vld<T, V>(v, q, b);
        vld<T, V>(as, q, c);
        vld<T, V>(sp2, q, d);
        vld<T, V>(psi, q, p);
#pragma unroll
        for (int u = 0; u < V; u++) out[u] = -a[u] * b[u] + c[u] * (d[u] - nl3(p[u], beta, gamma));
    }
};

// lambda_n = A lambda_{n+1} + U (x1 - L x2) + sum_c shift_c^T (U_c x3_c): the transposes of
// psi = iCT psihat, Sp2 = iCT(-L psihat) and grad_c psi = iST_c G_c with the index-shifted
// G_x[i] = -s_i psihat[i+1] (i < nx-1; y, z alike), FP64
template <typename T>
__global__ void adv_adj_combine(Spec<double> s, const double *__restrict__ l1, const T *__restrict__ x1,
                                const T *__restrict__ x2, const T *__restrict__ x3x, const T *__restrict__ x3y,
                                const T *__restrict__ x3z, double *__restrict__ lout, long long n)
{
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(q % s.nz), j = (int)((q / s.nz) % s.ny), i = (int)(q / ((long long)s.nz * s.ny));
        const double L = s.alin(i, j, k), hl = s.dtd2 * L;
        double v = (1.0 + hl) / (1.0 - hl) * l1[q] + wend(s, i, j, k, -1, 0.5) * (double(x1[q]) - L * double(x2[q]));
        if (i >= 1) v -= s.sx[i - 1] * wend(s, i - 1, j, k, 0, 0.5) * double(x3x[q - s.nyz]);
        if (j >= 1) v -= s.sy[j - 1] * wend(s, i, j - 1, k, 1, 0.5) * double(x3y[q - s.nz]);
        if (k >= 1) v -= s.sz[k - 1] * wend(s, i, j, k - 1, 2, 0.5) * double(x3z[q - 1]);
        lout[q] = v;
    }
}

// sums <t - a_mu, psi^3>, <t - a_mu, psi^5> (beta, gamma) and <t, v . grad psi> (nu: v ~ 1/nu)
template <typename T>
struct RedAdvBGN {
    const T *__restrict__ t, *__restrict__ sx, *__restrict__ sy, *__restrict__ sz;
    const T *__restrict__ gx, *__restrict__ gy, *__restrict__ gz;
    const T *__restrict__ vx, *__restrict__ vy, *__restrict__ vz, *__restrict__ psi;
    __device__ __forceinline__ void operator()(long long q, double *acc) const
    {
        const double g0 = gx[q], g1 = gy[q], g2 = gz[q], tt = t[q];
        const double t2 = tt - (double(sx[q]) * g0 + double(sy[q]) * g1 + double(sz[q]) * g2);
        const double p = psi[q], p3 = p * p * p;
        acc[0] += t2 * p3;
        acc[1] += t2 * p3 * p * p;
        acc[2] += tt * (g0 * double(vx[q]) + g1 * double(vy[q]) + g2 * double(vz[q]));
    }
};

// eps, alpha: the update's A, B (as RedEpsAlpha) plus Sp2 = iCT(-L psihat): -psihat_n U x2
template <typename T>
struct RedEpsAlphaAdv {
    Spec<double> s;
    const double *__restrict__ l1, *__restrict__ ph0, *__restrict__ ph1;
    const T *__restrict__ x2;
    __device__ __forceinline__ void operator()(long long q, double *acc) const
    {
        const int k = (int)(q % s.nz);
        const int j = (int)((q / s.nz) % s.ny);
        const int i = (int)(q / ((long long)s.nz * s.ny));
        const double L = s.alin(i, j, k), h = s.dtd2, den = 1.0 - h * L;
        const double A = (1.0 + h * L) / den;
        const double term = l1[q] * (2.0 * h / (den * den) * ph0[q] + h / den * (ph1[q] - A * ph0[q])) -
                            ph0[q] * wend(s, i, j, k, -1, 0.5) * double(x2[q]);
        const double d = s.mq2(i, j, k) - s.q02;
        acc[0] += term;
        acc[1] += term * (-(d * d));
    }
};

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};

}  // namespace

template <typename T>
int noadv_adjoint(Ctx &c, const smadft_adj_opts &o, smadft_grads *out, double *dpsi0_host)
{
    const long long n = c.n;
    const int T_ = o.steps, K = o.checkpoint_every;
    const int ncp = (T_ + K - 1) / K;
    const size_t bd = sizeof(double) * n, bt = sizeof(T) * n;
    Spec<T> sT = make_spec<T>(c);
    Spec<double> sd = make_spec<double>(c);
    // device memory: checkpoints, one segment, three lambdas, two real scratch fields,
    // the initial psi, the final state
    DevBuf m_cp_ph, m_cp_np, m_seg_ph, m_seg_psi, m_lam, m_t, m_psi0, m_fin, m_dpsi;
    auto alloc = [&](DevBuf &b, size_t bytes) { return cudaMalloc(&b.p, bytes) == cudaSuccess; };
    const size_t fin_bytes = bd + 2 * bt;
    if (!alloc(m_cp_ph, bd * ncp) || !alloc(m_cp_np, bt * ncp) || !alloc(m_seg_ph, bd * (K + 1)) ||
        !alloc(m_seg_psi, bt * K) || !alloc(m_lam, 3 * bd) || !alloc(m_t, 2 * bt) || !alloc(m_psi0, bt) ||
        !alloc(m_fin, fin_bytes) || !alloc(m_dpsi, bd)) {
        cudaGetLastError();
        c.err = "adjoint: device memory";
        return SMADFT_ERR_NOMEM;
    }
    double *cp_ph = (double *)m_cp_ph.p, *seg_ph = (double *)m_seg_ph.p, *lam = (double *)m_lam.p;
    T *cp_np = (T *)m_cp_np.p, *seg_psi = (T *)m_seg_psi.p, *tA = (T *)m_t.p, *tB = tA + n, *psi0 = (T *)m_psi0.p;
    double *ph = c.f<double>(S_PSIH);
    T *np = c.f<T>(S_NP), *psi = c.f<T>(S_PSI);
    auto d2d = [&](void *dst, const void *src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, c.stream);
    };
    int rc;
    // ---- forward with checkpoints
    SMADFT_CUDA(d2d(psi0, psi, bt));
    for (int s = 0; s < T_; s++) {
        if (s % K == 0) {
            SMADFT_CUDA(d2d(cp_ph + (size_t)(s / K) * n, ph, bd));
            SMADFT_CUDA(d2d(cp_np + (size_t)(s / K) * n, np, bt));
        }
        if ((rc = noadv_step<T>(c, false))) return rc;
    }
    char *fin = (char *)m_fin.p;
    SMADFT_CUDA(d2d(fin, ph, bd));
    SMADFT_CUDA(d2d(fin + bd, np, bt));
    SMADFT_CUDA(d2d(fin + bd + bt, psi, bt));
    // ---- loss on psi_T and its seed
    const int axis = o.axis;
    int na, nb, nl;
    long long sa, sb, sl;
    const Geom &g = c.g;
    if (axis == 2) { na = g.nx; nb = g.ny; nl = g.nz; sa = g.nyz; sb = g.nz; sl = 1; }
    else if (axis == 1) { na = g.nx; nb = g.nz; nl = g.ny; sa = g.nyz; sb = 1; sl = g.nz; }
    else { na = g.ny; nb = g.nz; nl = g.nx; sa = g.nz; sb = 1; sl = g.nyz; }
    std::vector<int> hidx((size_t)na * nb);
    std::vector<double> hpos((size_t)na * nb);
    if ((rc = track_columns<T>(c, psi, axis, o.mode, o.hi, o.lo, hidx.data(), hpos.data()))) return rc;
    double sum = 0;
    int found = 0;
    for (size_t q = 0; q < hpos.size(); q++)
        if (hidx[q] >= 0 && std::isfinite(hpos[q])) { sum += hpos[q]; found++; }
    out->found = found;
    out->loss = found ? sum / found / c.p.nw : std::nan("");
    if (!found) {
        c.err = "adjoint: the tracker finds no interface on the final psi";
        return SMADFT_ERR_INVALID;
    }
    SMADFT_CUDA(cudaMemsetAsync(tA, 0, bt, c.stream));
    interface_seed<T><<<(unsigned)((na * (long long)nb + 255) / 256), 256, 0, c.stream>>>(
        psi, na, nb, nl, sa, sb, sl, o.mode, o.hi, o.lo, 1.0 / (found * c.p.nw), tA);
    SMADFT_CUDA(cudaGetLastError());
    c.launches++;
    // lambda buffers: L[0] = lambda_{n+1}, L[1] = lambda_{n+2}, L[2] = lambda_n
    double *L[3] = {lam, lam + n, lam + 2 * n};
    SMADFT_CUDA(cudaMemsetAsync(L[1], 0, bd, c.stream));
    if ((rc = r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LoadArr<T>{tA}, StAdjLam<T>{sd, nullptr, L[0]}))) return rc;
    bool have_l2 = false;     // lambda_{n+2} exists (n + 2 <= T)
    double dbeta = 0, dgamma = 0, deps = 0, dalpha = 0;
    double red[kRedVals];
    // ---- reverse sweep, one checkpoint segment at a time
    for (int sgi = ncp - 1; sgi >= 0; sgi--) {
        const int n0 = sgi * K, n1 = std::min(n0 + K, T_);
        SMADFT_CUDA(d2d(ph, cp_ph + (size_t)sgi * n, bd));
        SMADFT_CUDA(d2d(np, cp_np + (size_t)sgi * n, bt));
        if (n0 == 0) SMADFT_CUDA(d2d(psi, psi0, bt));
        else if ((rc = refresh_psi<T>(c, psi))) return rc;
        for (int s = n0; s < n1; s++) {
            SMADFT_CUDA(d2d(seg_ph + (size_t)(s - n0) * n, ph, bd));
            SMADFT_CUDA(d2d(seg_psi + (size_t)(s - n0) * n, psi, bt));
            if ((rc = noadv_step<T>(c, false))) return rc;
        }
        SMADFT_CUDA(d2d(seg_ph + (size_t)(n1 - n0) * n, ph, bd));
        for (int s = n1 - 1; s >= n0; s--) {
            const T *psin = seg_psi + (size_t)(s - n0) * n;
            const double *ph0 = seg_ph + (size_t)(s - n0) * n, *ph1 = ph0 + n;
            // t = CT^T mu_s  (s = 0: mu_0 + mu_{-1} = 2 B lambda_1 - B lambda_2)
            const double a = s == 0 ? 2.0 : 3.0;
            if ((rc = r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3,
                               LdAdjIn<T>{sd, L[0], have_l2 ? L[1] : nullptr, a, -1.0, 1}, StoreArr<T>{tA})))
                return rc;
            if ((rc = run_reduce(c, RedBetaGamma<T>{tA, psin}, red))) return rc;
            dbeta += red[0];
            dgamma -= red[1];
            if ((rc = run_reduce(c, RedEpsAlpha{sd, L[0], ph0, ph1}, red))) return rc;
            deps += red[0];
            dalpha += red[1];
            if (s >= 1) {
                if ((rc = r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LdFprime<T>{tA, psin, sT.beta, sT.gamma},
                                   StAdjLam<T>{sd, L[0], L[2]})))
                    return rc;
            } else {
                adj_lambda0<<<c.red_blocks, 256, 0, c.stream>>>(sd, L[0], L[2], n);
                SMADFT_CUDA(cudaGetLastError());
                c.launches++;
                // dpsi0 = s CT^T lambda_0 + f'(psi_0) CT^T (mu_0 + mu_{-1})
                if ((rc = r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3, LdAdjIn<T>{sd, L[2], nullptr, c.scale, 0.0, 0},
                                   StoreArr<T>{tB})))
                    return rc;
                adj_dpsi0<T><<<c.red_blocks, 256, 0, c.stream>>>(tB, tA, psin, c.p.beta, c.p.gamma,
                                                                  (double *)m_dpsi.p, n);
                SMADFT_CUDA(cudaGetLastError());
                c.launches++;
            }
            // rotate: lambda_{n+2} <- lambda_{n+1} <- lambda_n
            double *tmp = L[1];
            L[1] = L[0];
            L[0] = L[2];
            L[2] = tmp;
            have_l2 = true;
        }
    }
    // the context continues from psi_T
    SMADFT_CUDA(d2d(ph, fin, bd));
    SMADFT_CUDA(d2d(np, fin + bd, bt));
    SMADFT_CUDA(d2d(psi, fin + bd + bt, bt));
    if (dpsi0_host)
        SMADFT_CUDA(cudaMemcpyAsync(dpsi0_host, m_dpsi.p, bd, cudaMemcpyDeviceToHost, c.stream));
    SMADFT_CUDA(cudaStreamSynchronize(c.stream));
    out->d_eps = deps;
    out->d_alpha = dalpha;
    out->d_beta = dbeta;
    out->d_gamma = dgamma;
    return SMADFT_OK;
}

// Advected model (adv/cosAdvTrackMult.cpp:760-777,824-1369).  The update is the noadv one
// with N_n = Phi(psihat_n) = f(psi) - v . grad psi, all of psi, grad psi, Sp2 and v functions
// of psihat_n, and the pre-loop Nhat_{-1} = CT f(psi_0) without advection.  Per reverse step
// n, from the recomputed fields of step n (adv_fields):
//   t = CT^T mu_n, mu_n = 3 B lambda_{n+1} - B lambda_{n+2}          (dJ/dN, real space)
//   dvhat_c = ST_c(-t g_c);  a_S = iST_c(W_c P^T(U_c dvhat))            (velocity, Stokes)
//   a_mu = sum a_Sc g_c,  a_g_c = -t v_c + a_Sc mu,  a_psi = f'(psi)(t - a_mu)
//   lambda_n = A lambda_{n+1} + U CT(a_psi) - L U CT(a_mu) + sum_c shift_c^T(U_c ST_c(a_g_c))
// and at the end dJ/dpsi_0 = s CT^T lambda_0 + f'(psi_0) CT^T(-B lambda_1).  The parameter
// gradients add, per step: beta, gamma from <t - a_mu, psi^3, psi^5>; nu from
// -1/nu <-t g, v>; eps, alpha from A, B and from Sp2 (-psihat_n U CT(a_mu)).
template <typename T>
int adv_adjoint(Ctx &c, const smadft_adj_opts &o, smadft_grads *out, double *dpsi0_host)
{
    const long long n = c.n;
    const int T_ = o.steps, K = o.checkpoint_every;
    const int ncp = (T_ + K - 1) / K, kseg = std::min(K, T_);
    const size_t bd = sizeof(double) * n, bt = sizeof(T) * n;
    Spec<T> sT = make_spec<T>(c);
    Spec<double> sd = make_spec<double>(c);
    // device memory: checkpoints (psihat, Nhat_prev), one segment of them, three lambdas,
    // seven real scratch fields, the initial psi, the final state, dJ/dpsi_0
    DevBuf m_cp_ph, m_cp_np, m_seg_ph, m_seg_np, m_lam, m_t, m_psi0, m_fin, m_dpsi;
    auto alloc = [&](DevBuf &b, size_t bytes) { return cudaMalloc(&b.p, bytes) == cudaSuccess; };
    if (!alloc(m_cp_ph, bd * ncp) || !alloc(m_cp_np, bt * ncp) || !alloc(m_seg_ph, bd * (kseg + 1)) ||
        !alloc(m_seg_np, bt * kseg) || !alloc(m_lam, 3 * bd) || !alloc(m_t, 7 * bt) || !alloc(m_psi0, bt) ||
        !alloc(m_fin, 2 * bd + bt) || !alloc(m_dpsi, bd)) {
        cudaGetLastError();
        c.err = "adjoint: device memory";
        return SMADFT_ERR_NOMEM;
    }
    double *cp_ph = (double *)m_cp_ph.p, *seg_ph = (double *)m_seg_ph.p, *lam = (double *)m_lam.p;
    T *cp_np = (T *)m_cp_np.p, *seg_np = (T *)m_seg_np.p, *psi0 = (T *)m_psi0.p;
    T *tA = (T *)m_t.p, *tB = tA + n, *aSx = tA + 2 * n, *aSy = tA + 3 * n, *aSz = tA + 4 * n;
    T *x1 = tA + 5 * n, *x2 = tA + 6 * n;
    double *ph = c.f<double>(S_PSIH);
    T *np = c.f<T>(S_NP), *psi = c.f<T>(S_PSI), *sp2 = c.f<T>(S_SP2);
    T *gx = c.f<T>(S_GX), *gy = c.f<T>(S_GY), *gz = c.f<T>(S_GZ);
    T *vx = c.f<T>(S_VX), *vy = c.f<T>(S_VY), *vz = c.f<T>(S_VZ);
    T *dx = c.f<T>(S_SX), *dy = c.f<T>(S_SY), *dz = c.f<T>(S_SZ);   // S-hat slots reused backwards
    auto d2d = [&](void *dst, const void *src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, c.stream);
    };
    int rc;
    // ---- forward with checkpoints (psi holds the initial condition itself); the final state
    // keeps psihat_T, psihat_{T-1} (for the fields of the last step) and Nhat_{T-1}
    double *fin_ph = (double *)m_fin.p, *last_ph = fin_ph + n;
    T *fin_np = (T *)(fin_ph + 2 * n);
    SMADFT_CUDA(d2d(psi0, psi, bt));
    for (int st = 0; st < T_; st++) {
        if (st % K == 0) {
            SMADFT_CUDA(d2d(cp_ph + (size_t)(st / K) * n, ph, bd));
            SMADFT_CUDA(d2d(cp_np + (size_t)(st / K) * n, np, bt));
        }
        if (st == T_ - 1) SMADFT_CUDA(d2d(last_ph, ph, bd));
        if ((rc = adv_step<T>(c))) return rc;
    }
    SMADFT_CUDA(d2d(fin_ph, ph, bd));
    SMADFT_CUDA(d2d(fin_np, np, bt));
    // ---- loss on psi_T = iCT psihat_T and its seed
    if ((rc = refresh_psi<T>(c, psi))) return rc;
    const int axis = o.axis;
    int na, nb, nl;
    long long sa, sb, sl;
    const Geom &g = c.g;
    if (axis == 2) { na = g.nx; nb = g.ny; nl = g.nz; sa = g.nyz; sb = g.nz; sl = 1; }
    else if (axis == 1) { na = g.nx; nb = g.nz; nl = g.ny; sa = g.nyz; sb = 1; sl = g.nz; }
    else { na = g.ny; nb = g.nz; nl = g.nx; sa = g.nz; sb = 1; sl = g.nyz; }
    std::vector<int> hidx((size_t)na * nb);
    std::vector<double> hpos((size_t)na * nb);
    if ((rc = track_columns<T>(c, psi, axis, o.mode, o.hi, o.lo, hidx.data(), hpos.data()))) return rc;
    double sum = 0;
    int found = 0;
    for (size_t q = 0; q < hpos.size(); q++)
        if (hidx[q] >= 0 && std::isfinite(hpos[q])) { sum += hpos[q]; found++; }
    out->found = found;
    out->loss = found ? sum / found / c.p.nw : std::nan("");
    if (!found) {
        c.err = "adjoint: the tracker finds no interface on the final psi";
        return SMADFT_ERR_INVALID;
    }
    SMADFT_CUDA(cudaMemsetAsync(tA, 0, bt, c.stream));
    interface_seed<T><<<(unsigned)((na * (long long)nb + 255) / 256), 256, 0, c.stream>>>(
        psi, na, nb, nl, sa, sb, sl, o.mode, o.hi, o.lo, 1.0 / (found * c.p.nw), tA);
    SMADFT_CUDA(cudaGetLastError());
    c.launches++;
    double *L[3] = {lam, lam + n, lam + 2 * n};   // lambda_{n+1}, lambda_{n+2}, lambda_n
    SMADFT_CUDA(cudaMemsetAsync(L[1], 0, bd, c.stream));
    if ((rc = r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LoadArr<T>{tA}, StAdjLam<T>{sd, nullptr, L[0]}))) return rc;
    bool have_l2 = false;
    double dbeta = 0, dgamma = 0, deps = 0, dalpha = 0, dnu = 0;
    double red[kRedVals];
    // ---- reverse sweep, one checkpoint segment at a time
    for (int sgi = ncp - 1; sgi >= 0; sgi--) {
        const int n0 = sgi * K, n1 = std::min(n0 + K, T_);
        SMADFT_CUDA(d2d(ph, cp_ph + (size_t)sgi * n, bd));
        SMADFT_CUDA(d2d(np, cp_np + (size_t)sgi * n, bt));
        for (int st = n0; st < n1; st++) {
            SMADFT_CUDA(d2d(seg_ph + (size_t)(st - n0) * n, ph, bd));
            SMADFT_CUDA(d2d(seg_np + (size_t)(st - n0) * n, np, bt));
            if ((rc = adv_step<T>(c))) return rc;
        }
        SMADFT_CUDA(d2d(seg_ph + (size_t)(n1 - n0) * n, ph, bd));
        for (int st = n1 - 1; st >= n0; st--) {
            const double *ph0 = seg_ph + (size_t)(st - n0) * n, *ph1 = ph0 + n;
            // the fields of step st: psi, grad psi, Sp2, v
            SMADFT_CUDA(d2d(ph, ph0, bd));
            if ((rc = adv_fields<T>(c))) return rc;
            // t = CT^T mu_st
            if ((rc = r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3,
                               LdAdjIn<T>{sd, L[0], have_l2 ? L[1] : nullptr, 3.0, -1.0, 1}, StoreArr<T>{tA})))
                return rc;
            {   // velocity-spectrum adjoints ST_c(-t g_c)
                const int kx[3] = {K_DST2, K_DCT2, K_DCT2};
                const int ky[3] = {K_DCT2, K_DST2, K_DCT2};
                const int kz[3] = {K_DCT2, K_DCT2, K_DST2};
                T *const o3[3] = {dx, dy, dz};
                if ((rc = r2r3d_multi<T, 3, 1>(c, kx, ky, kz, o3, LdNegTG<T, 0>{tA, gx}, LdNegTG<T, 1>{tA, gy},
                                            LdNegTG<T, 2>{tA, gz})))
                    return rc;
            }
            {   // force adjoints a_S = iST_c(W_c P^T(U_c dvhat))
                const int kx[3] = {K_DST3, K_DCT3, K_DCT3};
                const int ky[3] = {K_DCT3, K_DST3, K_DCT3};
                const int kz[3] = {K_DCT3, K_DCT3, K_DST3};
                T *const o3[3] = {aSx, aSy, aSz};
                if ((rc = r2r3d_multi<T, 3, 0>(c, kx, ky, kz, o3, LdStokesT<T, 0>{sT, dx, dy, dz},
                                            LdStokesT<T, 1>{sT, dx, dy, dz}, LdStokesT<T, 2>{sT, dx, dy, dz})))
                    return rc;
            }
            if ((rc = run_reduce(c, RedAdvBGN<T>{tA, aSx, aSy, aSz, gx, gy, gz, vx, vy, vz, psi}, red))) return rc;
            dbeta += red[0];
            dgamma -= red[1];
            dnu += red[2];
            {   // spectra of a_psi, a_mu, a_g (the last three into the free S-hat slots)
                const int kx[5] = {K_DCT2, K_DCT2, K_DST2, K_DCT2, K_DCT2};
                const int ky[5] = {K_DCT2, K_DCT2, K_DCT2, K_DST2, K_DCT2};
                const int kz[5] = {K_DCT2, K_DCT2, K_DCT2, K_DCT2, K_DST2};
                T *const o5[5] = {x1, x2, dx, dy, dz};
                if ((rc = r2r3d_multi<T, 5, 1>(c, kx, ky, kz, o5,
                                            LdAdjPsi<T>{tA, aSx, aSy, aSz, gx, gy, gz, psi, sT.beta, sT.gamma},
                                            LdAdjMu<T>{aSx, aSy, aSz, gx, gy, gz},
                                            LdAdjG<T, 0>{tA, vx, aSx, sp2, psi, sT.beta, sT.gamma},
                                            LdAdjG<T, 1>{tA, vy, aSy, sp2, psi, sT.beta, sT.gamma},
                                            LdAdjG<T, 2>{tA, vz, aSz, sp2, psi, sT.beta, sT.gamma})))
                    return rc;
            }
            if ((rc = run_reduce(c, RedEpsAlphaAdv<T>{sd, L[0], ph0, ph1, x2}, red))) return rc;
            deps += red[0];
            dalpha += red[1];
            adv_adj_combine<T><<<c.red_blocks, 256, 0, c.stream>>>(sd, L[0], x1, x2, dx, dy, dz, L[2], n);
            SMADFT_CUDA(cudaGetLastError());
            c.launches++;
            if (st == 0) {
                // the pre-loop Nhat_{-1} = CT f(psi_0): t_{-1} = CT^T(-B lambda_1)
                if ((rc = r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3, LdAdjIn<T>{sd, L[0], nullptr, -1.0, 0.0, 1},
                                   StoreArr<T>{tA})))
                    return rc;
                if ((rc = run_reduce(c, RedBetaGamma<T>{tA, psi0}, red))) return rc;
                dbeta += red[0];
                dgamma -= red[1];
                // dpsi0 = s CT^T lambda_0 + f'(psi_0) t_{-1}
                if ((rc = r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3, LdAdjIn<T>{sd, L[2], nullptr, c.scale, 0.0, 0},
                                   StoreArr<T>{tB})))
                    return rc;
                adj_dpsi0<T><<<c.red_blocks, 256, 0, c.stream>>>(tB, tA, psi0, c.p.beta, c.p.gamma,
                                                                  (double *)m_dpsi.p, n);
                SMADFT_CUDA(cudaGetLastError());
                c.launches++;
            }
            double *tmp = L[1];
            L[1] = L[0];
            L[0] = L[2];
            L[2] = tmp;
            have_l2 = true;
        }
    }
    // the context continues from the final state, its fields (psi, grad psi, Sp2, S-hat, v)
    // those of the last step as a plain run leaves them
    SMADFT_CUDA(d2d(ph, last_ph, bd));
    if ((rc = adv_fields<T>(c))) return rc;
    SMADFT_CUDA(d2d(ph, fin_ph, bd));
    SMADFT_CUDA(d2d(np, fin_np, bt));
    if (dpsi0_host)
        SMADFT_CUDA(cudaMemcpyAsync(dpsi0_host, m_dpsi.p, bd, cudaMemcpyDeviceToHost, c.stream));
    SMADFT_CUDA(cudaStreamSynchronize(c.stream));
    out->d_eps = deps;
    out->d_alpha = dalpha;
    out->d_beta = dbeta;
    out->d_gamma = dgamma;
    out->d_nu = dnu / c.p.nu;
    return SMADFT_OK;
}

#if !defined(SMADFT_INST_DOUBLE)
template int noadv_adjoint<float>(Ctx &, const smadft_adj_opts &, smadft_grads *, double *);
template int adv_adjoint<float>(Ctx &, const smadft_adj_opts &, smadft_grads *, double *);
#endif
#if !defined(SMADFT_INST_FLOAT)
template int noadv_adjoint<double>(Ctx &, const smadft_adj_opts &, smadft_grads *, double *);
template int adv_adjoint<double>(Ctx &, const smadft_adj_opts &, smadft_grads *, double *);
#endif

}  // namespace smadft
