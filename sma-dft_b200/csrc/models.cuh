// models.cuh -- the per-model loop bodies as chains of fused r2r passes.
//
// Every pointwise stage of the reference loop is folded into the first pass (Loader) or
// the last pass (Storer) of the 3-D transform that consumes or produces it, so a step is
// a sequence of axis-pass kernels and nothing else.  State kept between steps:
//   psihat  scaled spectral psi (psi = REDFT01^3 psihat); the reference recomputes it from
//           psi every step (adv/cosAdvTrackMult.cpp:847-860), which is the same up to rounding
//   Nprev   unscaled REDFT10^3 of the previous nonlinear term (the AB2 history)
//   quasi: psihat_old, rho_old and the real-space velocity (div v needs them)
#pragma once

#include "ctx.cuh"

namespace smadft {

template <typename T>
__device__ __forceinline__ T nl3(T p, T beta, T gamma)   // beta psi^3 - gamma psi^5
{
    T p2 = p * p, p3 = p2 * p;
    return beta * p3 - gamma * (p3 * p2);
}

// 1 / x for x > 0.  FP32: __fdividef (hardware reciprocal, at most 2 ulp), far inside the
// FP32 path's error budget; FP64: the correctly rounded reciprocal the FP64 parity needs.
template <typename T>
__device__ __forceinline__ T recip(T x)
{
    if constexpr (sizeof(T) == 4) return __fdividef(1.0f, x);
    else return T(1) / x;
}

// ---------------------------------------------------------------- loaders -------------
// All functors follow the vector interface of r2r_pass.cuh: V consecutive elements along z
// (idx .. idx+V-1 at (i, j, k .. k+V-1)); same-index fields use 16-byte loads, index-shifted
// neighbours along z use scalar loads.

// N = beta psi^3 - gamma psi^5 (no-adv/cosNoAdvTrackSing.cpp:713-723)
template <typename T>
struct LdNonlin {
    const T *__restrict__ psi;
    T beta, gamma;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int, int, int, T *out) const
    {
        T p[V];
        vld<T, V>(psi, q, p);
#pragma unroll
        for (int u = 0; u < V; u++) out[u] = nl3(p[u], beta, gamma);
    }
};

// Index-shifted gradient spectra (adv/cosAdvTrackMult.cpp:904-959): G_c = -s_c f[+1 along c],
// zero at the last index of c.  Branch-free: out-of-range points read a clamped in-range
// address and are zeroed by a select, so the loads of all points can be issued together.
template <typename T, int AX, typename S = T>
struct LdGrad {
    Spec<T> s;
    const S *__restrict__ f;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int i, int j, int k, T *out) const
    {
        if (AX == 0 || AX == 1) {
            const bool in = AX == 0 ? (i < s.nx - 1) : (j < s.ny - 1);
            const idx_t sh = AX == 0 ? s.nyz : (idx_t)s.nz;
            T v[V];
            vld_as<T, V, S>(f, in ? q + sh : q, v);
            const T sc = in ? -(AX == 0 ? s.sx[i] : s.sy[j]) : T(0);
#pragma unroll
            for (int u = 0; u < V; u++) out[u] = sc * v[u];
        } else {
#pragma unroll
            for (int u = 0; u < V; u++) {
                const bool in = k + u < s.nz - 1;
                const T x = T(f[in ? q + u + 1 : q + u]);
                out[u] = in ? -s.sz[k + u] * x : T(0);
            }
        }
    }
};

// Inverse sine z pass of the shifted gradient spectrum of f along z (LdGrad<T, 2, T>) into out
// (out != f): the register-direct z kernel reads the shifted, scaled line itself where the
// length has it, else the loader runs in the staged z pass.
template <typename T>
int z_pass_grad(Ctx &c, const Spec<T> &s, const T *f, T *out)
{
    if (c.use_rd && c.use_rdz && f != out) {
        switch (c.g.nz) {
        case 64: return launch_rdz_gradz<T, 64>(c, f, out, s.sz);
        case 128: return launch_rdz_gradz<T, 128>(c, f, out, s.sz);
        case 256: return launch_rdz_gradz<T, 256>(c, f, out, s.sz);
        default: break;
        }
    }
    return launch_axis<T, 2>(c, K_DST3, LdGrad<T, 2, T>{s, f}, StoreArr<T>{out});
}

// sine z passes of spectra stored by true wavenumber along z (lengths with the register-direct
// z kernel): the inverse one reads one index up, the forward one stores one index up
template <typename T>
int z_pass_upread(Ctx &c, const T *in, T *out)
{
    switch (c.g.nz) {
    case 64: return launch_rdz_upread<T, 64>(c, in, out);
    case 128: return launch_rdz_upread<T, 128>(c, in, out);
    case 256: return launch_rdz_upread<T, 256>(c, in, out);
    default: c.err = "z_pass_upread: length without the register-direct z kernel"; return SMADFT_ERR_INVALID;
    }
}
template <typename T>
int z_pass_upstore(Ctx &c, const T *in, T *out)
{
    switch (c.g.nz) {
    case 64: return launch_rdz_upstore<T, 64>(c, in, out);
    case 128: return launch_rdz_upstore<T, 128>(c, in, out);
    case 256: return launch_rdz_upstore<T, 256>(c, in, out);
    default: c.err = "z_pass_upstore: length without the register-direct z kernel"; return SMADFT_ERR_INVALID;
    }
}

// -L(q) psihat (adv/cosAdvTrackMult.cpp:980-986)
template <typename T>
struct LdNegLin {
    Spec<T> s;
    const double *__restrict__ ph;   // spectral state (FP64)
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int i, int j, int k, T *out) const
    {
        T v[V];
        vld_as<T, V, double>(ph, q, v);
#pragma unroll
        for (int u = 0; u < V; u++) out[u] = -s.alin(i, j, k + u) * v[u];
    }
};

// S_c = (Sp2 - beta psi^3 + gamma psi^5) d_c psi (adv/cosAdvTrackMult.cpp:994-1015)
template <typename T>
struct LdForce {
    static constexpr int kMinBlocks = 2;   // three fields per point: memory-bound, keep registers
    const T *__restrict__ psi, *__restrict__ sp2, *__restrict__ g;
    T beta, gamma;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int, int, int, T *out) const
    {
        T a[V], b[V], c[V];
        vld<T, V>(psi, q, a);
        vld<T, V>(sp2, q, b);
        vld<T, V>(g, q, c);
        if constexpr (V == 2) {
            // the two points as one pair (lane-wise packed arithmetic)
            const cpx<T> A{a[0], a[1]};
            const cpx<T> p2 = pmul(A, A), p3 = pmul(p2, A);
            const cpx<T> nl = pfma(cpx<T>{-gamma, -gamma}, pmul(p3, p2), pmul(cpx<T>{beta, beta}, p3));
            const cpx<T> r = pmul(csub(cpx<T>{b[0], b[1]}, nl), cpx<T>{c[0], c[1]});
            out[0] = r.x;
            out[1] = r.y;
        } else {
#pragma unroll
            for (int u = 0; u < V; u++) out[u] = (b[u] - nl3(a[u], beta, gamma)) * c[u];
        }
    }
};

// Spectral Stokes projection, one velocity component (adv/cosAdvTrackMult.cpp:1103-1274 on
// one rank; with DIVV, the irrotational part of quasi/quasi.cpp:1704-2109):
//   v_x[i,j,k] = CM1x (Sx - CM2x (s_i Sx + q_j Sy[i+1,j-1,k] + q_k Sz[i+1,j,k-1])), i < nx-1
//   v_y[i,j,k] = CM1y (Sy - CM2y (q_i Sx[i-1,j+1,k] + s_j Sy + q_k Sz[i,j+1,k-1])), j<ny-1, k<nz-1
//   v_z[i,j,k] = CM1z (Sz - CM2z (q_i Sx[i-1,j,k+1] + q_j Sy[i,j-1,k+1] + s_k Sz)), j<ny-1, k<nz-1
// with CM1 = scale / (nu |q_s|^2), CM2 = s / |q_s|^2 (one reciprocal) and index -1
// neighbours = 0.
template <typename T, int AX, bool DIVV>
struct LdStokes {
    Spec<T> s;
    const T *__restrict__ Sx, *__restrict__ Sy, *__restrict__ Sz, *__restrict__ dv;
    // Branch-free: neighbours outside the box read a clamped in-range address and are
    // zeroed by selects; truncated modes are zeroed at the end.
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int i, int j, int k, T *out) const
    {
        const T snu = s.scale / s.nu;
        if (AX == 0) {
            const bool live = i < s.nx - 1;
            const idx_t qn = live ? q + s.nyz : q;         // (i+1, j, k)
            const bool jy = j != 0;
            T sx[V], sy[V], d[V];
            vld<T, V>(Sx, q, sx);
            vld<T, V>(Sy, jy ? qn - s.nz : qn, sy);             // (i+1, j-1, k)
            if (DIVV) vld<T, V>(dv, qn, d);
            const T si = s.sx[i], qj = s.qy[j];
            const T a2 = si * si + qj * qj;
#pragma unroll
            for (int u = 0; u < V; u++) {
                const int kk = k + u;
                const T qk = s.qz[kk];
                const bool kz = kk != 0;
                const T szr = Sz[kz ? qn - 1 + u : qn + u];       // (i+1, j, k-1)
                const T syv = jy ? sy[u] : T(0), sz = kz ? szr : T(0);
                const T inv = recip<T>(a2 + qk * qk);
                const T dot = si * sx[u] + qj * syv + qk * sz;
                T v = snu * inv * (sx[u] - si * inv * dot);
                if (DIVV) v = v + snu * inv * (s.nu * si * d[u]);
                out[u] = live ? v : T(0);
            }
        } else if (AX == 1) {
            const bool live = j < s.ny - 1;
            const idx_t qj1 = live ? q + s.nz : q;          // (i, j+1, k)
            const bool ix = i != 0;
            T syv[V], sx[V], d[V];
            vld<T, V>(Sy, q, syv);
            vld<T, V>(Sx, ix ? qj1 - s.nyz : qj1, sx);          // (i-1, j+1, k)
            if (DIVV) vld<T, V>(dv, qj1, d);
            const T qi = s.qx[i], sj = s.sy[j];
            const T a2 = qi * qi + sj * sj;
#pragma unroll
            for (int u = 0; u < V; u++) {
                const int kk = k + u;
                const T qk = s.qz[kk];
                const bool kz = kk != 0;
                const T szr = Sz[kz ? qj1 - 1 + u : qj1 + u];     // (i, j+1, k-1)
                const T sxv = ix ? sx[u] : T(0), sz = kz ? szr : T(0);
                const T inv = recip<T>(a2 + qk * qk);
                const T dot = qi * sxv + sj * syv[u] + qk * sz;
                T v = snu * inv * (syv[u] - sj * inv * dot);
                if (DIVV) v = v + snu * inv * (s.nu * sj * d[u]);
                out[u] = (live && kk < s.nz - 1) ? v : T(0);
            }
        } else {
            const bool live = j < s.ny - 1;
            const bool ix = i != 0, jy = j != 0;
            T szv[V];
            vld<T, V>(Sz, q, szv);
            const T qi = s.qx[i], qj = s.qy[j];
            const T a2 = qi * qi + qj * qj;
#pragma unroll
            for (int u = 0; u < V; u++) {
                const int kk = k + u;
                const bool kl = kk < s.nz - 1;
                const idx_t qk1 = kl ? q + 1 + u : q + u;    // (i, j, k+1)
                const T sk = s.sz[kk];
                const T sxr = Sx[ix ? qk1 - s.nyz : qk1];         // (i-1, j, k+1)
                const T syr = Sy[jy ? qk1 - s.nz : qk1];          // (i, j-1, k+1)
                const T sx = ix ? sxr : T(0), sy = jy ? syr : T(0);
                const T inv = recip<T>(a2 + sk * sk);
                const T dot = qi * sx + qj * sy + sk * szv[u];
                T v = snu * inv * (szv[u] - sk * inv * dot);
                if (DIVV) v = v + snu * inv * (s.nu * sk * dv[qk1]);
                out[u] = (live && kl) ? v : T(0);
            }
        }
    }
};

// The same projection from force spectra stored by true wavenumber: S~_c(I, J, K) is S_c with
// the sine index of axis c moved up by one (S~_c = 0 at wavenumber 0 of axis c), so the three
// values of one wavenumber sit at one index and every read is an aligned vector.  The
// neighbours of LdStokes become S~x[i+1,j,k], S~y[i+1,j,k], S~z[i+1,j,k] (= Sx, Sy[i+1,j-1,k],
// Sz[i+1,j,k-1]) for v_x and S~[i,j+1,k] for v_y; v_z is produced at its true wavenumber
// (index k = wavenumber K) and its sine z pass reads it one index up.  Same operands, same
// operations and truncations as LdStokes.
template <typename T, int AX>
struct LdStokesK {
    Spec<T> s;
    const T *__restrict__ Sx, *__restrict__ Sy, *__restrict__ Sz;
    // v = snu inv (own - sc inv dot), inv = 1 / (a2 + qk^2), dot = c0 x + c1 y + qk z, for the
    // two points of a pair at once (lane-wise packed arithmetic; the same operations in the
    // same order as the scalar form)
    __device__ __forceinline__ static cpx<T> proj2(T snu, T a2, T c0, T c1, T sc, cpx<T> qk, cpx<T> x, cpx<T> y,
                                                   cpx<T> z, cpx<T> own)
    {
        const cpx<T> d = pfma(qk, qk, cpx<T>{a2, a2});
        const cpx<T> inv{recip<T>(d.x), recip<T>(d.y)};
        const cpx<T> dot = pfma(qk, z, pfma(cpx<T>{c1, c1}, y, pmul(cpx<T>{c0, c0}, x)));
        const cpx<T> t = pfma(pmul(cpx<T>{-sc, -sc}, inv), dot, own);
        return pmul(pmul(cpx<T>{snu, snu}, inv), t);
    }
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int i, int j, int k, T *out) const
    {
        const T snu = s.scale / s.nu;
        if constexpr (V == 2) {
            // k even: the pair (k, k+1) of every field and table is one aligned vector
            T x[2], y[2], z[2];
            if (AX == 0) {
                const bool live = i < s.nx - 1;
                const idx_t qn = live ? q + s.nyz : q;
                vld<T, 2>(Sx, qn, x);
                vld<T, 2>(Sy, qn, y);
                vld<T, 2>(Sz, qn, z);
                const T si = s.sx[i], qj = s.qy[j];
                const cpx<T> X{x[0], x[1]};
                const cpx<T> v = proj2(snu, si * si + qj * qj, si, qj, si, cpx<T>{s.qz[k], s.qz[k + 1]}, X,
                                       cpx<T>{y[0], y[1]}, cpx<T>{z[0], z[1]}, X);
                out[0] = live ? v.x : T(0);
                out[1] = live ? v.y : T(0);
            } else if (AX == 1) {
                const bool live = j < s.ny - 1;
                const idx_t qj1 = live ? q + s.nz : q;
                vld<T, 2>(Sx, qj1, x);
                vld<T, 2>(Sy, qj1, y);
                vld<T, 2>(Sz, qj1, z);
                const T qi = s.qx[i], sj = s.sy[j];
                const cpx<T> Y{y[0], y[1]};
                const cpx<T> v = proj2(snu, qi * qi + sj * sj, qi, sj, sj, cpx<T>{s.qz[k], s.qz[k + 1]},
                                       cpx<T>{x[0], x[1]}, Y, cpx<T>{z[0], z[1]}, Y);
                out[0] = (live && k < s.nz - 1) ? v.x : T(0);
                out[1] = (live && k + 1 < s.nz - 1) ? v.y : T(0);
            } else {
                const bool live = j < s.ny - 1;
                vld<T, 2>(Sx, q, x);
                vld<T, 2>(Sy, q, y);
                vld<T, 2>(Sz, q, z);
                const T qi = s.qx[i], qj = s.qy[j];
                const bool kl = k >= 1;
                const cpx<T> sk{s.sz[kl ? k - 1 : 0], s.sz[k]};
                const cpx<T> Z{z[0], z[1]};
                // the sine wavenumber is the product's own coefficient here: dot = qi x + qj y + sk z
                const cpx<T> d = pfma(sk, sk, cpx<T>{qi * qi + qj * qj, qi * qi + qj * qj});
                const cpx<T> inv{recip<T>(d.x), recip<T>(d.y)};
                const cpx<T> dot = pfma(sk, Z, pfma(cpx<T>{qj, qj}, cpx<T>{y[0], y[1]}, pmul(cpx<T>{qi, qi}, cpx<T>{x[0], x[1]})));
                const cpx<T> t = pfma(pmul(cpx<T>{-sk.x, -sk.y}, inv), dot, Z);
                const cpx<T> v = pmul(pmul(cpx<T>{snu, snu}, inv), t);
                out[0] = (live && kl) ? v.x : T(0);
                out[1] = live ? v.y : T(0);
            }
            return;
        }
        if (AX == 0) {
            const bool live = i < s.nx - 1;
            const idx_t qn = live ? q + s.nyz : q;         // wavenumber (i+1, j, k)
            T sx[V], sy[V], sz[V];
            vld<T, V>(Sx, qn, sx);
            vld<T, V>(Sy, qn, sy);
            vld<T, V>(Sz, qn, sz);
            const T si = s.sx[i], qj = s.qy[j];
            const T a2 = si * si + qj * qj;
#pragma unroll
            for (int u = 0; u < V; u++) {
                const T qk = s.qz[k + u];
                const T inv = recip<T>(a2 + qk * qk);
                const T dot = si * sx[u] + qj * sy[u] + qk * sz[u];
                const T v = snu * inv * (sx[u] - si * inv * dot);
                out[u] = live ? v : T(0);
            }
        } else if (AX == 1) {
            const bool live = j < s.ny - 1;
            const idx_t qj1 = live ? q + s.nz : q;          // wavenumber (i, j+1, k)
            T sx[V], sy[V], sz[V];
            vld<T, V>(Sx, qj1, sx);
            vld<T, V>(Sy, qj1, sy);
            vld<T, V>(Sz, qj1, sz);
            const T qi = s.qx[i], sj = s.sy[j];
            const T a2 = qi * qi + sj * sj;
#pragma unroll
            for (int u = 0; u < V; u++) {
                const int kk = k + u;
                const T qk = s.qz[kk];
                const T inv = recip<T>(a2 + qk * qk);
                const T dot = qi * sx[u] + sj * sy[u] + qk * sz[u];
                const T v = snu * inv * (sy[u] - sj * inv * dot);
                out[u] = (live && kk < s.nz - 1) ? v : T(0);
            }
        } else {
            const bool live = j < s.ny - 1;
            T sx[V], sy[V], sz[V];
            vld<T, V>(Sx, q, sx);
            vld<T, V>(Sy, q, sy);
            vld<T, V>(Sz, q, sz);
            const T qi = s.qx[i], qj = s.qy[j];
            const T a2 = qi * qi + qj * qj;
#pragma unroll
            for (int u = 0; u < V; u++) {
                const int kk = k + u;                        // wavenumber K; sine index K - 1
                const bool kl = kk >= 1;
                const T sk = s.sz[kl ? kk - 1 : 0];
                const T inv = recip<T>(a2 + sk * sk);
                const T dot = qi * sx[u] + qj * sy[u] + sk * sz[u];
                const T v = snu * inv * (sz[u] - sk * inv * dot);
                out[u] = (live && kl) ? v : T(0);
            }
        }
    }
};

// N = beta psi^3 - gamma psi^5 - v . grad psi (adv/cosAdvTrackMult.cpp:1290-1303)
template <typename T>
struct LdAdvN {
    static constexpr int kMinBlocks = 2;   // seven fields per point: memory-bound, keep registers
    const T *__restrict__ psi, *__restrict__ vx, *__restrict__ vy, *__restrict__ vz;
    const T *__restrict__ gx, *__restrict__ gy, *__restrict__ gz;
    T beta, gamma;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int, int, int, T *out) const
    {
        T p[V], a[V], b[V], c[V], d[V], e[V], f[V];
        vld<T, V>(psi, q, p);
        vld<T, V>(vx, q, a); vld<T, V>(gx, q, d);
        vld<T, V>(vy, q, b); vld<T, V>(gy, q, e);
        vld<T, V>(vz, q, c); vld<T, V>(gz, q, f);
#pragma unroll
        for (int u = 0; u < V; u++) out[u] = nl3(p[u], beta, gamma) - a[u] * d[u] - b[u] * e[u] - c[u] * f[u];
    }
};

// v . grad psi alone, the conserved adv model's unweighted advection term
// (adv/cosAdvConSingle.cpp:1301-1303)
template <typename T>
struct LdAdvDot {
    static constexpr int kMinBlocks = 2;   // six fields per point: memory-bound, keep registers
    const T *__restrict__ vx, *__restrict__ vy, *__restrict__ vz;
    const T *__restrict__ gx, *__restrict__ gy, *__restrict__ gz;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int, int, int, T *out) const
    {
        T a[V], b[V], c[V], d[V], e[V], f[V];
        vld<T, V>(vx, q, a); vld<T, V>(gx, q, d);
        vld<T, V>(vy, q, b); vld<T, V>(gy, q, e);
        vld<T, V>(vz, q, c); vld<T, V>(gz, q, f);
#pragma unroll
        for (int u = 0; u < V; u++) out[u] = a[u] * d[u] + b[u] * e[u] + c[u] * f[u];
    }
};

// ---------------------------------------------------------------- storers -------------
// Crank-Nicolson / Adams-Bashforth update fed by the freshly transformed N
// (no-adv/cosNoAdvTrackSing.cpp:752-753, adv/cosAdvTrackMult.cpp:1362-1364):
//   psihat <- (C1 psihat + dt/2 scale (3 N - Nprev)) / C2,  C1,2 = 1 +- dt/2 L(q);  Nprev <- N
// The update runs in FP64 from FP64 wavenumbers for every field precision: C1/C2 is applied
// to psihat every step, so a rounding error in it would grow linearly with the step count.
//
// CONS selects the conserved variants (d psi/dt = -q^2 (dF/dpsi)^):
//   1  noadv: the operator in C1, C2 and N are weighted by q^2
//      (no-adv/cosNoAdvConserv.cpp:646-650,809);
//   2  adv: C1, C2 and the Swift-Hohenberg part of N are weighted by q^2, the advection
//      term is not: N = q^2 v - w with w = REDFT10^3(v . grad psi)
//      (adv/cosAdvConSingle.cpp:741-742,1296-1310,1369).
// Nprev keeps the weighted N, as the reference's NqPast does.
template <typename T, int CONS = 0>
struct StUpdCN {
    Spec<double> s;
    double *__restrict__ ph;        // spectral state (FP64 for every compute precision)
    T *__restrict__ np;             // Nprev (field precision)
    const T *__restrict__ w = nullptr;   // CONS 2: REDFT10^3(v . grad psi)
    // w is read ahead with psihat and Nprev for FP32 fields; FP64 fields read it in fin()
    // (three FP64 reads ahead spill more at the FP64 passes' 128 registers)
    static constexpr bool W_AHEAD = CONS == 2 && sizeof(T) == 4;
    static constexpr int PRE = W_AHEAD ? 3 : 2;   // psihat, Nprev (, w)
    using Pre = double;
    template <int V>
    __device__ __forceinline__ void pre(idx_t q, int, int, int, double *buf) const
    {
        vld<double, V>(ph, q, buf);
        vld_as<double, V, T>(np, q, buf + V);
        if constexpr (W_AHEAD) vld_as<double, V, T>(w, q, buf + 2 * V);
    }
    template <int V>
    __device__ __forceinline__ void fin(idx_t q, int i, int j, int k, const T *v, const double *buf) const
    {
        double o[V];
        T nw[V], wl[V];
        if constexpr (CONS == 2 && !W_AHEAD) vld<T, V>(w, q, wl);
#pragma unroll
        for (int u = 0; u < V; u++) {
            double al = s.alin(i, j, k + u);
            double nn = double(v[u]);
            if constexpr (CONS != 0) {
                const double m2 = s.mq2(i, j, k + u);
                al = m2 * al;
                nn = m2 * nn;
                if constexpr (W_AHEAD) nn -= buf[2 * V + u];
                if constexpr (CONS == 2 && !W_AHEAD) nn -= double(wl[u]);
            }
            const double c1 = 1.0 + s.dtd2 * al, c2 = 1.0 - s.dtd2 * al;
            o[u] = (c1 * buf[u] + s.dtd2 * s.scale * (3.0 * nn - buf[V + u])) / c2;
            nw[u] = T(nn);
        }
        vst<double, V>(ph, q, o);
        vst<T, V>(np, q, nw);
    }
    template <int V>
    __device__ __forceinline__ void store(idx_t q, int i, int j, int k, const T *v) const
    {
        double buf[2 * V];
        pre<V>(q, i, j, k, buf);
        fin<V>(q, i, j, k, v, buf);
    }
};

// q^2-weighted copy of a forward transform: the conserved noadv pre-loop N
// (no-adv/cosNoAdvConserv.cpp:688-701)
template <typename T>
struct StQ2 {
    Spec<double> s;
    T *__restrict__ p;
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
        for (int u = 0; u < V; u++) o[u] = T(s.mq2(i, j, k + u) * double(v[u]));
        vst<T, V>(p, q, o);
    }
};

// Scales a forward transform into psihat (pre-loop: psihat = scale REDFT10^3 psi)
template <typename T>
struct StScale {
    double *__restrict__ p;         // spectral state (FP64)
    double scale;
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
        double o[V];
#pragma unroll
        for (int u = 0; u < V; u++) o[u] = scale * double(v[u]);
        vst<double, V>(p, q, o);
    }
};

}  // namespace smadft
