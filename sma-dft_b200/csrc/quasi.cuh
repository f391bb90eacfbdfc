// quasi.cuh -- the quasi-incompressible loop body (quasi/quasi.cpp:1099-2190) as fused
// r2r passes.  Density law, Gaussian filter, div v from the mass balance, pressure,
// solenoidal + irrotational velocity and the BDF2-like update all ride in the loaders and
// storers of the 21 transforms the reference runs per step.
#pragma once

#include "models.cuh"
#include "reduce.cuh"

namespace smadft {

// f' = alpha (q0^2 - q^2) psihat (quasi/quasi.cpp:1121-1131)
template <typename T>
struct LdDfd {
    Spec<T> s;
    const double *__restrict__ ph;   // spectral state (FP64)
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int i, int j, int k, T *out) const
    {
        T v[V];
        vld_as<T, V, double>(ph, q, v);
#pragma unroll
        for (int u = 0; u < V; u++) out[u] = s.alpha * (s.q02 - s.mq2(i, j, k + u)) * v[u];
    }
};

// -q^2 alpha (q0^2 - q^2) psihat (quasi/quasi.cpp:1414-1420)
template <typename T>
struct LdLapDfd {
    Spec<T> s;
    const double *__restrict__ ph;   // spectral state (FP64)
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int i, int j, int k, T *out) const
    {
        T v[V];
        vld_as<T, V, double>(ph, q, v);
#pragma unroll
        for (int u = 0; u < V; u++) {
            const T m = s.mq2(i, j, k + u);
            out[u] = -m * s.alpha * (s.q02 - m) * v[u];
        }
    }
};

// rho = kp sqrt(q0^2 psi^2 + |grad psi|^2) + rho0 (quasi/quasi.cpp:1322-1336)
template <typename T>
struct LdRhoRaw {
    const T *__restrict__ psi, *__restrict__ gx, *__restrict__ gy, *__restrict__ gz;
    T kp, rho0, q02;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int, int, int, T *out) const
    {
        T p[V], a[V], b[V], c[V];
        vld<T, V>(psi, q, p); vld<T, V>(gx, q, a); vld<T, V>(gy, q, b); vld<T, V>(gz, q, c);
#pragma unroll
        for (int u = 0; u < V; u++)
            out[u] = kp * sqrt(q02 * (p[u] * p[u]) + a[u] * a[u] + b[u] * b[u] + c[u] * c[u]) + rho0;
    }
};

// rhohat = scale REDFT10^3(rho) exp(-2 1.57^2 q^2) (quasi/quasi.cpp:1342-1351)
template <typename T>
struct StFilter {
    Spec<T> s;
    T *__restrict__ out;
    static constexpr int PRE = 0;
    template <int V>
    __device__ __forceinline__ void pre(idx_t, int, int, int, T *) const {}
    template <int V>
    __device__ __forceinline__ void fin(idx_t q, int i, int j, int k, const T *v, const T *) const
    {
        store<V>(q, i, j, k, v);
    }
    template <int V>
    __device__ __forceinline__ void store(idx_t q, int i, int j, int k, const T *v) const
    {
        T o[V];
        const T exy = s.ex[i] * s.ey[j];
#pragma unroll
        for (int u = 0; u < V; u++) o[u] = (s.scale * v[u]) * (exy * s.ez[k + u]);
        vst<T, V>(out, q, o);
    }
};

// div v = -((rho - rho_old)/dt + v . grad rho) / (0.5 (rho + rho_old)) (quasi/quasi.cpp:1370-1377)
template <typename T>
struct LdDivv {
    const T *__restrict__ rho, *__restrict__ ro, *__restrict__ vx, *__restrict__ vy, *__restrict__ vz;
    const T *__restrict__ rx, *__restrict__ ry, *__restrict__ rz;
    T dt;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int, int, int, T *out) const
    {
        T r[V], o[V], a[V], b[V], c[V], d[V], e[V], f[V];
        vld<T, V>(rho, q, r); vld<T, V>(ro, q, o);
        vld<T, V>(vx, q, a); vld<T, V>(rx, q, d);
        vld<T, V>(vy, q, b); vld<T, V>(ry, q, e);
        vld<T, V>(vz, q, c); vld<T, V>(rz, q, f);
#pragma unroll
        for (int u = 0; u < V; u++)
            out[u] = -((r[u] - o[u]) / dt + a[u] * d[u] + b[u] * e[u] + c[u] * f[u]) / (T(0.5) * (r[u] + o[u]));
    }
};

template <typename T>
struct LdMul {
    const T *__restrict__ a, *__restrict__ b;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int, int, int, T *out) const
    {
        T x[V], y[V];
        vld<T, V>(a, q, x);
        vld<T, V>(b, q, y);
#pragma unroll
        for (int u = 0; u < V; u++) out[u] = x[u] * y[u];
    }
};

// lap <- -scale q^2 REDFT10^3(rho f') (quasi/quasi.cpp:1392-1400)
template <typename T>
struct StLapSpec {
    Spec<T> s;
    T *__restrict__ out;
    static constexpr int PRE = 0;
    template <int V>
    __device__ __forceinline__ void pre(idx_t, int, int, int, T *) const {}
    template <int V>
    __device__ __forceinline__ void fin(idx_t q, int i, int j, int k, const T *v, const T *) const
    {
        store<V>(q, i, j, k, v);
    }
    template <int V>
    __device__ __forceinline__ void store(idx_t q, int i, int j, int k, const T *v) const
    {
        T o[V];
#pragma unroll
        for (int u = 0; u < V; u++) o[u] = -s.scale * s.mq2(i, j, k + u) * v[u];
        vst<T, V>(out, q, o);
    }
};

// e, mu and S_c = mu d_c psi + e d_c rho (quasi/quasi.cpp:1448-1490).  AX == 0 also stores mu
// and e; lap_rho == 1 multiplies the relaxation-branch Laplacian by rho (:1429-1435).
template <typename T, int AX>
struct LdQForce {
    const T *__restrict__ psi, *__restrict__ dfd, *__restrict__ lap, *__restrict__ rho;
    const T *__restrict__ g, *__restrict__ r;
    T *__restrict__ mu_out, *__restrict__ en_out;
    T eps, beta, gamma;
    int lap_rho;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int, int, int, T *out) const
    {
        T ps[V], f[V], lp[V], rh[V], gg[V], rr[V], mo[V], eo[V];
        vld<T, V>(psi, q, ps); vld<T, V>(dfd, q, f); vld<T, V>(lap, q, lp); vld<T, V>(rho, q, rh);
        vld<T, V>(g, q, gg); vld<T, V>(r, q, rr);
#pragma unroll
        for (int u = 0; u < V; u++) {
            const T p = ps[u], p2 = p * p, p3 = p2 * p, p4 = p2 * p2;
            const T e = T(-0.5) * eps * p2 + T(0.5) * (f[u] * f[u]) - T(0.25) * beta * p4 + (gamma / T(6)) * (p4 * p2);
            const T lv = lap_rho ? rh[u] * lp[u] : lp[u];
            const T m = lv + rh[u] * (f[u] - eps * p - beta * p3 + gamma * (p3 * p2));
            mo[u] = m;
            eo[u] = e;
            out[u] = m * gg[u] + e * rr[u];
        }
        if (AX == 0) {
            vst<T, V>(mu_out, q, mo);
            vst<T, V>(en_out, q, eo);
        }
    }
};

// p = scale(-(q . S[-1 shifts]) / q^2 + (lambda + 2 nu) divv), p(0,0,0) = 0 (quasi/quasi.cpp:1553-1588)
template <typename T>
struct LdPressure {
    Spec<T> s;
    const T *__restrict__ Sx, *__restrict__ Sy, *__restrict__ Sz, *__restrict__ dv;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int i, int j, int k, T *out) const
    {
        // branch-free: missing neighbours read a clamped address and are zeroed by selects
#pragma unroll
        for (int u = 0; u < V; u++) {
            const int kk = k + u;
            const idx_t qq = q + u;
            const T sxr = Sx[i > 0 ? qq - s.nyz : qq];
            const T syr = Sy[j > 0 ? qq - s.nz : qq];
            const T szr = Sz[kk > 0 ? qq - 1 : qq];
            const T sx = i > 0 ? sxr : T(0), sy = j > 0 ? syr : T(0), sz = kk > 0 ? szr : T(0);
            const bool origin = (i + j + kk) == 0;
            const T m2 = origin ? T(1) : s.mq2(i, j, kk);
            const T v = s.scale * (-(s.qx[i] * sx + s.qy[j] * sy + s.qz[kk] * sz) / m2 +
                                   (s.lam + T(2) * s.nu) * dv[qq]);
            out[u] = origin ? T(0) : v;
        }
    }
};

// Nl = -mu - v . grad psi [+ (p + rho e) kp |grad rho| / rho^2 after the switch]
// (quasi/quasi.cpp:2128-2154)
template <typename T>
struct LdQN {
    const T *__restrict__ mu, *__restrict__ vx, *__restrict__ vy, *__restrict__ vz;
    const T *__restrict__ gx, *__restrict__ gy, *__restrict__ gz;
    const T *__restrict__ p, *__restrict__ rho, *__restrict__ en;
    const T *__restrict__ rx, *__restrict__ ry, *__restrict__ rz;
    T kp;
    int extra;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int, int, int, T *out) const
    {
        T m[V], a[V], b[V], c[V], d[V], e[V], f[V];
        vld<T, V>(mu, q, m);
        vld<T, V>(vx, q, a); vld<T, V>(gx, q, d);
        vld<T, V>(vy, q, b); vld<T, V>(gy, q, e);
        vld<T, V>(vz, q, c); vld<T, V>(gz, q, f);
#pragma unroll
        for (int u = 0; u < V; u++) out[u] = -m[u] - a[u] * d[u] - b[u] * e[u] - c[u] * f[u];
        if (extra) {
#pragma unroll
            for (int u = 0; u < V; u++) {
                const T x = rx[q + u], y = ry[q + u], z = rz[q + u], r = rho[q + u];
                out[u] += (p[q + u] + r * en[q + u]) * kp * sqrt(x * x + y * y + z * z) / (r * r);
            }
        }
    }
};

// psihat <- (C1 psihat - psihat_old/2 + dt/2 scale (3 N - Nprev)) / C2,
// C1 = 2 - dt rho_m L, C2 = 1.5 - dt rho_m L; first step uses Nprev = N (quasi/quasi.cpp:2162-2182)
// Runs in FP64 for every field precision (see StUpdCN).
template <typename T>
struct StUpdBDF {
    Spec<double> s;
    double *__restrict__ ph, *__restrict__ pho;   // spectral state (FP64)
    T *__restrict__ np;                           // Nprev (field precision)
    int first;
    static constexpr int PRE = 3;   // psihat, psihat_old, Nprev
    using Pre = double;
    template <int V>
    __device__ __forceinline__ void pre(idx_t q, int, int, int, double *buf) const
    {
        vld<double, V>(ph, q, buf);
        vld<double, V>(pho, q, buf + V);
        vld_as<double, V, T>(np, q, buf + 2 * V);
    }
    template <int V>
    __device__ __forceinline__ void fin(idx_t q, int i, int j, int k, const T *v, const double *buf) const
    {
        double o[V];
#pragma unroll
        for (int u = 0; u < V; u++) {
            const double al = s.alin(i, j, k + u);
            const double c1 = 2.0 - s.dt * s.rho_m * al, c2 = 1.5 - s.dt * s.rho_m * al;
            const double nv = double(v[u]);
            const double npv = first ? nv : buf[2 * V + u];
            o[u] = (c1 * buf[u] - 0.5 * buf[V + u] + s.dtd2 * s.scale * (3.0 * nv - npv)) / c2;
        }
        vst<double, V>(ph, q, o);
        vst<double, V>(pho, q, buf);
        vst<T, V>(np, q, v);
    }
    template <int V>
    __device__ __forceinline__ void store(idx_t q, int i, int j, int k, const T *v) const
    {
        double buf[3 * V];
        pre<V>(q, i, j, k, buf);
        fin<V>(q, i, j, k, v, buf);
    }
};

template <typename T>
int quasi_pre_loop(Ctx &c)
{
    Spec<T> s = make_spec<T>(c);
    T *psi = c.f<T>(S_PSI);
    double *ph = c.f<double>(S_PSIH);   // spectral state (FP64)
    int rc;
    // psihat = scale CT(psi); psi = iCT(psihat); psihat_old = psihat (quasi/quasi.cpp:990-1034)
    if ((rc = r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LoadArr<T>{psi}, StScale<T>{ph, c.scale}))) return rc;
    if ((rc = r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3, LoadArr<T, double>{ph}, StoreArr<T>{psi}))) return rc;
    SMADFT_CUDA(cudaMemcpyAsync(c.slot[S_PSIH_OLD], ph, sizeof(double) * c.n, cudaMemcpyDeviceToDevice, c.stream));
    return SMADFT_OK;
}

template <typename T>
int quasi_step(Ctx &c, long long nloop, bool keep_old)
{
    Spec<T> s = make_spec<T>(c);
    const smadft_params &P = c.p;
    T *psi = c.f<T>(S_PSI);
    double *ph = c.f<double>(S_PSIH), *pho = c.f<double>(S_PSIH_OLD);   // FP64 state
    T *np = c.f<T>(S_NP);
    T *gx = c.f<T>(S_GX), *gy = c.f<T>(S_GY), *gz = c.f<T>(S_GZ);
    T *rx = c.f<T>(S_RDX), *ry = c.f<T>(S_RDY), *rz = c.f<T>(S_RDZ);
    T *rho = c.f<T>(S_RHO), *ro = c.f<T>(S_RHO_OLD), *rq = c.f<T>(S_RHOQ);
    T *dfd = c.f<T>(S_DFD), *lap = c.f<T>(S_LAP), *dv = c.f<T>(S_DIVV), *pp = c.f<T>(S_P);
    T *mu = c.f<T>(S_MU), *en = c.f<T>(S_EN);
    T *Sx = c.f<T>(S_SX), *Sy = c.f<T>(S_SY), *Sz = c.f<T>(S_SZ);
    T *vx = c.f<T>(S_VX), *vy = c.f<T>(S_VY), *vz = c.f<T>(S_VZ);
    int rc;
    // f', grad psi, grad rho (quasi/quasi.cpp:1121-1304)
    {
        const int kx[4] = {K_DCT3, K_DST3, K_DCT3, K_DCT3};
        const int ky[4] = {K_DCT3, K_DCT3, K_DST3, K_DCT3};
        const int kz[4] = {K_DCT3, K_DCT3, K_DCT3, K_DST3};
        T *const out[4] = {dfd, gx, gy, gz};
        if ((rc = r2r3d_multi<T, 4, 0>(c, kx, ky, kz, out, LdDfd<T>{s, ph}, LdGrad<T, 0, double>{s, ph},
                                    LdGrad<T, 1, double>{s, ph}, LdGrad<T, 2, double>{s, ph})))
            return rc;
    }
    {
        const int kx[3] = {K_DST3, K_DCT3, K_DCT3};
        const int ky[3] = {K_DCT3, K_DST3, K_DCT3};
        const int kz[3] = {K_DCT3, K_DCT3, K_DST3};
        T *const out[3] = {rx, ry, rz};
        if ((rc = r2r3d_multi<T, 3, 0>(c, kx, ky, kz, out, LdGrad<T, 0>{s, rq}, LdGrad<T, 1>{s, rq}, LdGrad<T, 2>{s, rq})))
            return rc;
    }
    // density law + filter (:1322-1357)
    if ((rc = r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LdRhoRaw<T>{psi, gx, gy, gz, s.kp, s.rho0, s.q02},
                       StFilter<T>{s, rq}))) return rc;
    if ((rc = r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3, LoadArr<T>{rq}, StoreArr<T>{rho}))) return rc;
    if (P.loaded && nloop == 1)
        SMADFT_CUDA(cudaMemcpyAsync(ro, rho, sizeof(T) * c.n, cudaMemcpyDeviceToDevice, c.stream));
    int lap_rho;
    if (nloop > P.divv_switch || P.loaded) {   // :1366-1406
        if ((rc = r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LdDivv<T>{rho, ro, vx, vy, vz, rx, ry, rz, s.dt},
                           StoreArr<T>{dv}))) return rc;
        if ((rc = r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LdMul<T>{rho, dfd}, StLapSpec<T>{s, lap}))) return rc;
        if ((rc = r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3, LoadArr<T>{lap}, StoreArr<T>{lap}))) return rc;
        lap_rho = 0;
    } else {                                   // :1410-1437 (div v stays 0 before the switch)
        SMADFT_CUDA(cudaMemsetAsync(dv, 0, sizeof(T) * c.n, c.stream));
        if ((rc = r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3, LdLapDfd<T>{s, ph}, StoreArr<T>{lap}))) return rc;
        lap_rho = 1;
    }
    SMADFT_CUDA(cudaMemcpyAsync(ro, rho, sizeof(T) * c.n, cudaMemcpyDeviceToDevice, c.stream));  // :1439
    // forces (:1448-1504); the x loader also stores mu and e
    {
        const int kx[3] = {K_DST2, K_DCT2, K_DCT2};
        const int ky[3] = {K_DCT2, K_DST2, K_DCT2};
        const int kz[3] = {K_DCT2, K_DCT2, K_DST2};
        T *const out[3] = {Sx, Sy, Sz};
        if ((rc = r2r3d_multi<T, 3, 1>(
                 c, kx, ky, kz, out,
                 LdQForce<T, 0>{psi, dfd, lap, rho, gx, rx, mu, en, s.eps, s.beta, s.gamma, lap_rho},
                 LdQForce<T, 1>{psi, dfd, lap, rho, gy, ry, nullptr, nullptr, s.eps, s.beta, s.gamma, lap_rho},
                 LdQForce<T, 2>{psi, dfd, lap, rho, gz, rz, nullptr, nullptr, s.eps, s.beta, s.gamma, lap_rho})))
            return rc;
    }
    // pressure (:1510-1592) and velocity = solenoidal + irrotational (:1599-2123)
    {
        const int kx[4] = {K_DCT3, K_DST3, K_DCT3, K_DCT3};
        const int ky[4] = {K_DCT3, K_DCT3, K_DST3, K_DCT3};
        const int kz[4] = {K_DCT3, K_DCT3, K_DCT3, K_DST3};
        T *const out[4] = {pp, vx, vy, vz};
        if ((rc = r2r3d_multi<T, 4, 0>(c, kx, ky, kz, out, LdPressure<T>{s, Sx, Sy, Sz, dv},
                                    LdStokes<T, 0, true>{s, Sx, Sy, Sz, dv}, LdStokes<T, 1, true>{s, Sx, Sy, Sz, dv},
                                    LdStokes<T, 2, true>{s, Sx, Sy, Sz, dv})))
            return rc;
    }
    // N and the BDF2-like update (:2128-2182)
    if ((rc = r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2,
                       LdQN<T>{mu, vx, vy, vz, gx, gy, gz, pp, rho, en, rx, ry, rz, s.kp,
                               (int)(nloop > P.divv_switch + 1)},
                       StUpdBDF<T>{make_spec<double>(c), ph, pho, np, (int)(nloop == 1)}))) return rc;
    // psi = iCT(psihat) (:2186-2190)
    T *dst = keep_old ? c.f<T>(S_PSI2) : psi;
    return r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3, LoadArr<T, double>{ph}, StoreArr<T>{dst});
}

template <typename T>
int reduce_mass_energy(Ctx &c, double *ms)
{
    double out[kRedVals];
    int rc = run_reduce(c, RedSum2<T>{c.f<T>(S_RHO), c.f<T>(S_EN)}, out);
    ms[0] = out[0];
    ms[1] = out[1];
    return rc;
}

}  // namespace smadft
