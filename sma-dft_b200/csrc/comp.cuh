// comp.cuh -- the compressible loop body (compressible/compressible.cpp:1265-2720) as fused
// r2r passes and a few pointwise kernels.  The model has an independent density rho (its own
// AB2 mass balance), an amplitude field A = filter(sqrt(q0^2 psi^2 + |grad psi|^2)) that
// penalises rho - rho_0 - kp A, and a solenoidal plus irrotational velocity.  The first
// divv_switch steps are a relaxation: rho follows A, shifted up by rho_up planes.
// Single-rank semantics: halo planes read as zero (the last x-plane of the shifted spectra
// and of v_x stay zero, the i = 0 neighbours of v_y, v_z and of div v are zero).
#pragma once

#include "quasi.cuh"

namespace smadft {

// T(scale) times a forward transform: rhohat for the gradient spectra of rho
// (compressible/compressible.cpp:1292-1431 scale the shifted rhohat by `scale`)
template <typename T>
struct StScaleT {
    T *__restrict__ out;
    T scale;
    static constexpr int PRE = 0;
    template <int V>
    __device__ __forceinline__ void pre(idx_t, int, int, int, T *) const {}
    template <int V>
    __device__ __forceinline__ void fin(idx_t q, int i, int j, int k, const T *v, const T *) const
    {
        store<V>(q, i, j, k, v);
    }
    template <int V>
    __device__ __forceinline__ void store(idx_t q, int, int, int, const T *v) const
    {
        T o[V];
#pragma unroll
        for (int u = 0; u < V; u++) o[u] = scale * v[u];
        vst<T, V>(out, q, o);
    }
};

// Relaxation steps (:1574-1630): rho = rho_0 + ((1 - rho_0)/Amp) A, lap *= rho; then rho is
// shifted up by `up` planes in z (rho = 1 below) and lap multiplied by the shifted rho once
// more, as the reference's second loop does.  Out of place in rho, in place in lap.
template <typename T>
__global__ void comp_relax_kernel(int nz, int up, long long n, T rho1, T c1, const T *__restrict__ amp,
                                  T *__restrict__ rho, T *__restrict__ lap)
{
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(q % nz);
        const T r = rho1 + c1 * amp[q];
        T lv = r * lap[q], ro = r;
        if (up > 0) {
            ro = k >= up ? rho1 + c1 * amp[q - up] : T(1);
            lv = ro * lv;
        }
        rho[q] = ro;
        lap[q] = lv;
    }
}

// The eight forward-transformed fields of :1636-1711, all from psi, f' (dfd), lap, rho, A:
//   C 0  fgrad = zeta/2 (rho^2 - (rho_0 + kp A)^2)        (also stores mu)
//   C 1  e = rho f'^2 / 2
//   C 2-4  S_c = (lap + rho f') d_c psi + f'^2/2 d_c rho   (c = C - 2)
//   C 5-7  f_c = kp zeta (rho - rho_0 - kp A)/(A + 0.001) d_c psi
// mu = lap + rho (f' - eps psi - beta psi^3 + gamma psi^5).
template <typename T, int C>
struct LdCForce {
    static constexpr int kMinBlocks = 2;
    const T *__restrict__ psi, *__restrict__ dfd, *__restrict__ lap, *__restrict__ rho, *__restrict__ amp;
    const T *__restrict__ g, *__restrict__ r;   // C >= 2: this component's grad psi (and grad rho)
    T *__restrict__ mu_out;                     // C == 0
    T eps, beta, gamma, zeta, kp, rho0;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int, int, int, T *out) const
    {
        T f[V], rh[V];
        vld<T, V>(dfd, q, f);
        vld<T, V>(rho, q, rh);
        if constexpr (C == 0) {
            T am[V], lp[V], ps[V], mo[V];
            vld<T, V>(amp, q, am); vld<T, V>(lap, q, lp); vld<T, V>(psi, q, ps);
#pragma unroll
            for (int u = 0; u < V; u++) {
                const T b = rho0 + kp * am[u], p = ps[u], p3 = p * p * p;
                out[u] = T(0.5) * zeta * (rh[u] * rh[u] - b * b);
                mo[u] = lp[u] + rh[u] * (f[u] - eps * p - beta * p3 + gamma * (p3 * p * p));
            }
            vst<T, V>(mu_out, q, mo);
        } else if constexpr (C == 1) {
#pragma unroll
            for (int u = 0; u < V; u++) out[u] = rh[u] * (T(0.5) * (f[u] * f[u]));
        } else if constexpr (C <= 4) {
            T lp[V], gg[V], rr[V];
            vld<T, V>(lap, q, lp); vld<T, V>(g, q, gg); vld<T, V>(r, q, rr);
#pragma unroll
            for (int u = 0; u < V; u++) out[u] = (lp[u] + rh[u] * f[u]) * gg[u] + (T(0.5) * (f[u] * f[u])) * rr[u];
        } else {
            T am[V], gg[V];
            vld<T, V>(amp, q, am); vld<T, V>(g, q, gg);
#pragma unroll
            for (int u = 0; u < V; u++)
                out[u] = kp * zeta * (rh[u] - rho0 - kp * am[u]) / (am[u] + T(0.001)) * gg[u];
        }
    }
};

// Solenoidal and irrotational velocity spectra (:1838-2410), one thread per mode:
//   vsol_x = CM1x/nu (Sx - CM2x dot),  virr_x = CM1x/(lambda + 2 nu) (s_i fgrad'[i+1] + CM2x dot G)
// with CM1 = scale/|q_s|^2, CM2 = s/|q_s|^2, dot the shifted-neighbour product of LdStokes,
// fgrad' = fgrad + e exp(-2 1.57^2 q^2) and G = exp(-2 1.57^2 |q_s|^2), both from the
// per-axis factor tables.  v_x for i < nx-1, v_y, v_z for j < ny-1 and k < nz-1 (zero
// elsewhere).  The reference's k = 0 branch of v_z for i >= 1, 0 < j < ny-1 takes G from
// CM1y (:2348-2350); so does this kernel.  Grid: x = k blocks, y = j, z = i.
template <typename T>
__global__ void comp_vel_kernel(Spec<T> s, const T *__restrict__ Sx, const T *__restrict__ Sy, const T *__restrict__ Sz,
                                const T *__restrict__ fg, const T *__restrict__ en, T *__restrict__ vsx,
                                T *__restrict__ vsy, T *__restrict__ vsz, T *__restrict__ vix, T *__restrict__ viy,
                                T *__restrict__ viz)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, i = blockIdx.z;
    if (k >= s.nz) return;
    const idx_t nyz = s.nyz, nz = s.nz;
    const idx_t q = (idx_t)i * nyz + (idx_t)j * nz + k;
    // one reciprocal per component: CM1 = scale/m2, CM2 = s/m2; 1/nu and 1/(lambda + 2 nu) hoisted
    const T sc = s.scale, inu = T(1) / s.nu, il2n = T(1) / (s.lam + T(2) * s.nu);
    const T qi = s.qx[i], qj = s.qy[j], qk = s.qz[k], si = s.sx[i], sj = s.sy[j], sk = s.sz[k];
    const T exi = s.ex[i], eyj = s.ey[j], ezk = s.ez[k];
    T vx = T(0), ix = T(0), vy = T(0), iy = T(0), vz = T(0), iz = T(0);
    if (i < s.nx - 1) {
        const T syv = j != 0 ? Sy[q + nyz - nz] : T(0);    // (i+1, j-1, k)
        const T szv = k != 0 ? Sz[q + nyz - 1] : T(0);     // (i+1, j, k-1)
        const T inv = T(1) / (si * si + qj * qj + qk * qk), cm1 = sc * inv, cm2 = si * inv;
        const T dot = si * Sx[q] + qj * syv + qk * szv;
        const T fgn = fg[q + nyz] + en[q + nyz] * (s.ex[i + 1] * eyj * ezk);
        vx = (cm1 * inu) * (Sx[q] - cm2 * dot);
        ix = (cm1 * il2n) * (si * fgn + cm2 * dot * (s.esx[i] * eyj * ezk));
    }
    if (j < s.ny - 1 && k < s.nz - 1) {
        T sxv = i != 0 ? Sx[q - nyz + nz] : T(0);            // (i-1, j+1, k)
        const T szv = k != 0 ? Sz[q + nz - 1] : T(0);        // (i, j+1, k-1)
        const T invy = T(1) / (qi * qi + sj * sj + qk * qk);
        T cm1 = sc * invy, cm2 = sj * invy;
        T dot = qi * sxv + sj * Sy[q] + qk * szv;
        const T gy = exi * s.esy[j] * ezk;
        const T fgy = fg[q + nz] + en[q + nz] * (exi * s.ey[j + 1] * ezk);
        vy = (cm1 * inu) * (Sy[q] - cm2 * dot);
        iy = (cm1 * il2n) * (sj * fgy + cm2 * dot * gy);
        sxv = i != 0 ? Sx[q - nyz + 1] : T(0);               // (i-1, j, k+1)
        const T syv = j != 0 ? Sy[q - nz + 1] : T(0);        // (i, j-1, k+1)
        const T invz = T(1) / (qi * qi + qj * qj + sk * sk);
        cm1 = sc * invz;
        cm2 = sk * invz;
        dot = qi * sxv + qj * syv + sk * Sz[q];
        const T fgz = fg[q + 1] + en[q + 1] * (exi * eyj * s.ez[k + 1]);
        const T gz = (i >= 1 && k == 0 && j >= 1) ? gy : exi * eyj * s.esz[k];
        vz = (cm1 * inu) * (Sz[q] - cm2 * dot);
        iz = (cm1 * il2n) * (sk * fgz + cm2 * dot * gz);
    }
    vsx[q] = vx; vsy[q] = vy; vsz[q] = vz;
    vix[q] = ix; viy[q] = iy; viz[q] = iz;
}

// div v and the penalty-force divergence from the shifted spectra (:2478-2527):
//   divv = q . virr[-1 shifts],  ampd = scale q . f[-1 shifts]  (index -1 -> 0)
// Grid as comp_vel_kernel.
template <typename T>
__global__ void comp_div_kernel(Spec<T> s, const T *__restrict__ vix, const T *__restrict__ viy, const T *__restrict__ viz,
                                const T *__restrict__ fx, const T *__restrict__ fy, const T *__restrict__ fz,
                                T *__restrict__ dv, T *__restrict__ ad)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, i = blockIdx.z;
    if (k >= s.nz) return;
    const idx_t nyz = s.nyz, nz = s.nz;
    const idx_t q = (idx_t)i * nyz + (idx_t)j * nz + k;
    const T a = i > 0 ? vix[q - nyz] : T(0), fa = i > 0 ? fx[q - nyz] : T(0);
    const T b = j > 0 ? viy[q - nz] : T(0), fb = j > 0 ? fy[q - nz] : T(0);
    const T c = k > 0 ? viz[q - 1] : T(0), fc = k > 0 ? fz[q - 1] : T(0);
    dv[q] = s.qx[i] * a + s.qy[j] * b + s.qz[k] * c;
    ad[q] = s.scale * (s.qx[i] * fa + s.qy[j] * fb + s.qz[k] * fc);
}

// Mass balance, AB2 in real space (:2555-2573):
//   S = -(vsol + virr) . grad rho - rho div v,  rho += dt (3/2 S - 1/2 S_prev),  S_prev = S
template <typename T>
__global__ void comp_rho_kernel(long long n, T dt, const T *__restrict__ vsx, const T *__restrict__ vsy,
                                const T *__restrict__ vsz, const T *__restrict__ vix, const T *__restrict__ viy,
                                const T *__restrict__ viz, const T *__restrict__ rx, const T *__restrict__ ry,
                                const T *__restrict__ rz, const T *__restrict__ dv, T *__restrict__ rho,
                                T *__restrict__ fr)
{
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const T S = -(vsx[q] + vix[q]) * rx[q] - (vsy[q] + viy[q]) * ry[q] - (vsz[q] + viz[q]) * rz[q] -
                    rho[q] * dv[q];
        rho[q] = rho[q] + dt * (T(1.5) * S - T(0.5) * fr[q]);
        fr[q] = S;
    }
}

// N = -mu + kp zeta/(A + 0.001) (rho - rho_0 - kp A) psi - ampd - (vsol + virr) . grad psi
// (:2578-2612)
template <typename T>
struct LdCN {
    static constexpr int kMinBlocks = 2;
    const T *__restrict__ mu, *__restrict__ amp, *__restrict__ rho, *__restrict__ psi, *__restrict__ ad;
    const T *__restrict__ vsx, *__restrict__ vsy, *__restrict__ vsz, *__restrict__ vix, *__restrict__ viy,
        *__restrict__ viz;
    const T *__restrict__ gx, *__restrict__ gy, *__restrict__ gz;
    T kp, zeta, rho0;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int, int, int, T *out) const
    {
        T m[V], a[V], r[V], p[V], d[V];
        vld<T, V>(mu, q, m); vld<T, V>(amp, q, a); vld<T, V>(rho, q, r); vld<T, V>(psi, q, p); vld<T, V>(ad, q, d);
#pragma unroll
        for (int u = 0; u < V; u++)
            out[u] = -m[u] + (kp * zeta / (a[u] + T(0.001))) * (r[u] - rho0 - kp * a[u]) * p[u] - d[u];
        T x[V], y[V], g[V];
        vld<T, V>(vsx, q, x); vld<T, V>(vix, q, y); vld<T, V>(gx, q, g);
#pragma unroll
        for (int u = 0; u < V; u++) out[u] -= (x[u] + y[u]) * g[u];
        vld<T, V>(vsy, q, x); vld<T, V>(viy, q, y); vld<T, V>(gy, q, g);
#pragma unroll
        for (int u = 0; u < V; u++) out[u] -= (x[u] + y[u]) * g[u];
        vld<T, V>(vsz, q, x); vld<T, V>(viz, q, y); vld<T, V>(gz, q, g);
#pragma unroll
        for (int u = 0; u < V; u++) out[u] -= (x[u] + y[u]) * g[u];
    }
};

// sums of rho and of rho e + zeta/2 (rho - rho_0 - kp A)^2 with the energy density
// e = -eps psi^2/2 + f'^2/2 - beta psi^4/4 + gamma psi^6/6 of the new psi (:2647-2690)
template <typename T>
struct RedCompME {
    const T *__restrict__ psi, *__restrict__ dfd, *__restrict__ rho, *__restrict__ amp;
    double eps, beta, gamma, zeta, kp, rho0;
    __device__ __forceinline__ void operator()(long long q, double *acc) const
    {
        const double p = psi[q], f = dfd[q], r = rho[q], a = amp[q], p2 = p * p, p4 = p2 * p2;
        const double e = -0.5 * eps * p2 + 0.5 * f * f - 0.25 * beta * p4 + (gamma / 6) * (p4 * p2);
        const double d = r - rho0 - kp * a;
        acc[0] += r;
        acc[1] += r * e + 0.5 * zeta * d * d;
    }
};

template <typename T>
int comp_pre_loop(Ctx &c)
{
    // psihat = scale CT(psi), psi = iCT(psihat), psihat_old = psihat (:1150-1194); rho and its
    // AB2 history start at zero (:612)
    int rc = quasi_pre_loop<T>(c);
    if (rc) return rc;
    SMADFT_CUDA(cudaMemsetAsync(c.slot[S_RHO], 0, c.esize * c.n, c.stream));
    SMADFT_CUDA(cudaMemsetAsync(c.slot[S_FRHO], 0, c.esize * c.n, c.stream));
    return SMADFT_OK;
}

template <typename T>
int comp_step(Ctx &c, long long nloop, bool keep_old)
{
    Spec<T> s = make_spec<T>(c);
    const smadft_params &P = c.p;
    const long long n = c.n;
    T *psi = c.f<T>(S_PSI);
    double *ph = c.f<double>(S_PSIH), *pho = c.f<double>(S_PSIH_OLD);   // FP64 state
    T *np = c.f<T>(S_NP);
    T *gx = c.f<T>(S_GX), *gy = c.f<T>(S_GY), *gz = c.f<T>(S_GZ);
    T *rx = c.f<T>(S_RDX), *ry = c.f<T>(S_RDY), *rz = c.f<T>(S_RDZ);
    T *rho = c.f<T>(S_RHO), *rq = c.f<T>(S_RHOQ), *fr = c.f<T>(S_FRHO), *amp = c.f<T>(S_AMP);
    T *dfd = c.f<T>(S_DFD), *lap = c.f<T>(S_LAP), *dv = c.f<T>(S_DIVV), *ad = c.f<T>(S_AMPD);
    T *mu = c.f<T>(S_MU), *en = c.f<T>(S_EN), *fg = c.f<T>(S_FGRAD);
    T *Sx = c.f<T>(S_SX), *Sy = c.f<T>(S_SY), *Sz = c.f<T>(S_SZ);
    T *fx = c.f<T>(S_FX), *fy = c.f<T>(S_FY), *fz = c.f<T>(S_FZ);
    T *vsx = c.f<T>(S_VX), *vsy = c.f<T>(S_VY), *vsz = c.f<T>(S_VZ);
    T *vix = c.f<T>(S_VIRX), *viy = c.f<T>(S_VIRY), *viz = c.f<T>(S_VIRZ);
    int rc;
    // scale CT(rho) (:1292-1294), then f', grad psi (from psihat) and grad rho (:1296-1534)
    if ((rc = r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LoadArr<T>{rho}, StScaleT<T>{rq, s.scale}))) return rc;
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
    // amplitude: filtered sqrt(q0^2 psi^2 + |grad psi|^2) (:1478-1515), via rq (free now)
    if ((rc = r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LdRhoRaw<T>{psi, gx, gy, gz, T(1), T(0), s.q02},
                       StFilter<T>{s, rq}))) return rc;
    if ((rc = r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3, LoadArr<T>{rq}, StoreArr<T>{amp}))) return rc;
    // lap(rho f') (:1542-1630)
    if (nloop > P.divv_switch || P.loaded) {
        if ((rc = r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2, LdMul<T>{rho, dfd}, StLapSpec<T>{s, lap}))) return rc;
        if ((rc = r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3, LoadArr<T>{lap}, StoreArr<T>{lap}))) return rc;
    } else {
        if ((rc = r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3, LdLapDfd<T>{s, ph}, StoreArr<T>{lap}))) return rc;
        const double amp0 = std::sqrt((3 * P.beta + std::sqrt(9 * P.beta * P.beta + 40 * P.eps * P.gamma)) / 5);
        comp_relax_kernel<T><<<c.red_blocks, 256, 0, c.stream>>>(c.g.nz, P.rho_up, n, T(P.rho0),
                                                                 T((1 - P.rho0) / amp0), amp, rho, lap);
        SMADFT_CUDA(cudaGetLastError());
        c.launches++;
    }
    // fgrad, e, S and the penalty force f, forward (:1636-1711); the first loader stores mu
    {
        const int kx[8] = {K_DCT2, K_DCT2, K_DST2, K_DCT2, K_DCT2, K_DST2, K_DCT2, K_DCT2};
        const int ky[8] = {K_DCT2, K_DCT2, K_DCT2, K_DST2, K_DCT2, K_DCT2, K_DST2, K_DCT2};
        const int kz[8] = {K_DCT2, K_DCT2, K_DCT2, K_DCT2, K_DST2, K_DCT2, K_DCT2, K_DST2};
        T *const out[8] = {fg, en, Sx, Sy, Sz, fx, fy, fz};
        const T e = s.eps, b = s.beta, g = s.gamma, z = s.zeta, kp = s.kp, r0 = s.rho0;
        if ((rc = r2r3d_multi<T, 8, 1>(
                 c, kx, ky, kz, out, LdCForce<T, 0>{psi, dfd, lap, rho, amp, nullptr, nullptr, mu, e, b, g, z, kp, r0},
                 LdCForce<T, 1>{psi, dfd, lap, rho, amp, nullptr, nullptr, nullptr, e, b, g, z, kp, r0},
                 LdCForce<T, 2>{psi, dfd, lap, rho, amp, gx, rx, nullptr, e, b, g, z, kp, r0},
                 LdCForce<T, 3>{psi, dfd, lap, rho, amp, gy, ry, nullptr, e, b, g, z, kp, r0},
                 LdCForce<T, 4>{psi, dfd, lap, rho, amp, gz, rz, nullptr, e, b, g, z, kp, r0},
                 LdCForce<T, 5>{psi, dfd, lap, rho, amp, gx, nullptr, nullptr, e, b, g, z, kp, r0},
                 LdCForce<T, 6>{psi, dfd, lap, rho, amp, gy, nullptr, nullptr, e, b, g, z, kp, r0},
                 LdCForce<T, 7>{psi, dfd, lap, rho, amp, gz, nullptr, nullptr, e, b, g, z, kp, r0})))
            return rc;
    }
    // velocity spectra, div v and the penalty divergence (:1826-2527)
    {
        const dim3 blk(128), grd((unsigned)((c.g.nz + 127) / 128), (unsigned)c.g.ny, (unsigned)c.g.nx);
        comp_vel_kernel<T><<<grd, blk, 0, c.stream>>>(s, Sx, Sy, Sz, fg, en, vsx, vsy, vsz, vix, viy, viz);
        SMADFT_CUDA(cudaGetLastError());
        comp_div_kernel<T><<<grd, blk, 0, c.stream>>>(s, vix, viy, viz, fx, fy, fz, dv, ad);
    }
    SMADFT_CUDA(cudaGetLastError());
    c.launches += 2;
    // all eight back to real space, in place (:2521-2552): one grouped launch for the y passes
    // where each CTA only rewrites the lines it loaded; the fused plane kernel exchanges rows
    // across a cluster, so with it each field goes through the scratch field instead
    {
        const int kx[8] = {K_DST3, K_DCT3, K_DCT3, K_DST3, K_DCT3, K_DCT3, K_DCT3, K_DCT3};
        const int ky[8] = {K_DCT3, K_DST3, K_DCT3, K_DCT3, K_DST3, K_DCT3, K_DCT3, K_DCT3};
        const int kz[8] = {K_DCT3, K_DCT3, K_DST3, K_DCT3, K_DCT3, K_DST3, K_DCT3, K_DCT3};
        T *const out[8] = {vsx, vsy, vsz, vix, viy, viz, dv, ad};
        if (plane_ok(c)) {
            for (int m = 0; m < 8; m++)
                if ((rc = r2r3d<T>(c, kx[m], ky[m], kz[m], LoadArr<T>{out[m]}, StoreArr<T>{out[m]}))) return rc;
        } else if ((rc = r2r3d_multi<T, 8, 0>(c, kx, ky, kz, out, LoadArr<T>{vsx}, LoadArr<T>{vsy}, LoadArr<T>{vsz},
                                           LoadArr<T>{vix}, LoadArr<T>{viy}, LoadArr<T>{viz}, LoadArr<T>{dv},
                                           LoadArr<T>{ad})))
            return rc;
    }
    // mass balance (:2555-2573)
    comp_rho_kernel<T><<<c.red_blocks, 256, 0, c.stream>>>(n, s.dt, vsx, vsy, vsz, vix, viy, viz, rx, ry, rz, dv,
                                                           rho, fr);
    SMADFT_CUDA(cudaGetLastError());
    c.launches++;
    // N and the BDF2-like update (:2578-2635)
    if ((rc = r2r3d<T>(c, K_DCT2, K_DCT2, K_DCT2,
                       LdCN<T>{mu, amp, rho, psi, ad, vsx, vsy, vsz, vix, viy, viz, gx, gy, gz, s.kp, s.zeta, s.rho0},
                       StUpdBDF<T>{make_spec<double>(c), ph, pho, np, (int)(nloop == 1)}))) return rc;
    // psi = iCT(psihat) (:2639-2643)
    T *dst = keep_old ? c.f<T>(S_PSI2) : psi;
    return r2r3d<T>(c, K_DCT3, K_DCT3, K_DCT3, LoadArr<T, double>{ph}, StoreArr<T>{dst});
}

template <typename T>
int reduce_comp_mass_energy(Ctx &c, const T *psi_new, double *ms)
{
    Spec<double> s = make_spec<double>(c);
    double out[kRedVals];
    int rc = run_reduce(c, RedCompME<T>{psi_new, c.f<T>(S_DFD), c.f<T>(S_RHO), c.f<T>(S_AMP), c.p.eps, c.p.beta,
                                        c.p.gamma, c.p.zeta, s.kp, c.p.rho0},
                        out);
    ms[0] = out[0];
    ms[1] = out[1];
    return rc;
}

}  // namespace smadft
