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

// ---------------------------------------------------------------- loaders -------------
// N = beta psi^3 - gamma psi^5 (no-adv/cosNoAdvTrackSing.cpp:713-723)
template <typename T>
struct LdNonlin {
    const T *__restrict__ psi;
    T beta, gamma;
    __device__ __forceinline__ T operator()(long long q, int, int, int) const
    {
        return nl3(psi[q], beta, gamma);
    }
};

// Index-shifted gradient spectra (adv/cosAdvTrackMult.cpp:904-959): G_c = -s_c f[+1 along c],
// zero at the last index of c.
template <typename T, int AX>
struct LdGrad {
    Spec<T> s;
    const T *__restrict__ f;
    __device__ __forceinline__ T operator()(long long q, int i, int j, int k) const
    {
        if (AX == 0) return (i < s.nx - 1) ? -s.sx[i] * f[q + s.nyz] : T(0);
        if (AX == 1) return (j < s.ny - 1) ? -s.sy[j] * f[q + s.nz] : T(0);
        return (k < s.nz - 1) ? -s.sz[k] * f[q + 1] : T(0);
    }
};

// -L(q) psihat (adv/cosAdvTrackMult.cpp:980-986)
template <typename T>
struct LdNegLin {
    Spec<T> s;
    const T *__restrict__ ph;
    __device__ __forceinline__ T operator()(long long q, int i, int j, int k) const
    {
        return -s.alin(i, j, k) * ph[q];
    }
};

// S_c = (Sp2 - beta psi^3 + gamma psi^5) d_c psi (adv/cosAdvTrackMult.cpp:994-1015)
template <typename T>
struct LdForce {
    const T *__restrict__ psi, *__restrict__ sp2, *__restrict__ g;
    T beta, gamma;
    __device__ __forceinline__ T operator()(long long q, int, int, int) const
    {
        return (sp2[q] - nl3(psi[q], beta, gamma)) * g[q];
    }
};

// Spectral Stokes projection, one velocity component (adv/cosAdvTrackMult.cpp:1103-1274 on
// one rank; with DIVV, the irrotational part of quasi/quasi.cpp:1704-2109):
//   v_x[i,j,k] = CM1x (Sx - CM2x (s_i Sx + q_j Sy[i+1,j-1,k] + q_k Sz[i+1,j,k-1])), i < nx-1
//   v_y[i,j,k] = CM1y (Sy - CM2y (q_i Sx[i-1,j+1,k] + s_j Sy + q_k Sz[i,j+1,k-1])), j<ny-1, k<nz-1
//   v_z[i,j,k] = CM1z (Sz - CM2z (q_i Sx[i-1,j,k+1] + q_j Sy[i,j-1,k+1] + s_k Sz)), j<ny-1, k<nz-1
// with CM1 = scale / (nu |q_s|^2), CM2 = s / |q_s|^2 and index -1 neighbours = 0.
template <typename T, int AX, bool DIVV>
struct LdStokes {
    Spec<T> s;
    const T *__restrict__ Sx, *__restrict__ Sy, *__restrict__ Sz, *__restrict__ dv;
    __device__ __forceinline__ T operator()(long long q, int i, int j, int k) const
    {
        if (AX == 0) {
            if (i >= s.nx - 1) return T(0);
            const long long qn = q + s.nyz;   // (i+1, j, k)
            T sy = (j != 0) ? Sy[qn - s.nz] : T(0);
            T sz = (k != 0) ? Sz[qn - 1] : T(0);
            T m2 = s.sx[i] * s.sx[i] + s.qy[j] * s.qy[j] + s.qz[k] * s.qz[k];
            T cm1 = s.scale / (s.nu * m2), cm2 = s.sx[i] / m2;
            T sxv = Sx[q];
            T dot = s.sx[i] * sxv + s.qy[j] * sy + s.qz[k] * sz;
            T v = cm1 * (sxv - cm2 * dot);
            if (DIVV) v = v + cm1 * (s.nu * s.sx[i] * dv[qn]);
            return v;
        } else if (AX == 1) {
            if (j >= s.ny - 1 || k >= s.nz - 1) return T(0);
            T sx = (i != 0) ? Sx[q - s.nyz + s.nz] : T(0);          // (i-1, j+1, k)
            T sz = (k != 0) ? Sz[q + s.nz - 1] : T(0);              // (i, j+1, k-1)
            T m2 = s.qx[i] * s.qx[i] + s.sy[j] * s.sy[j] + s.qz[k] * s.qz[k];
            T cm1 = s.scale / (s.nu * m2), cm2 = s.sy[j] / m2;
            T syv = Sy[q];
            T dot = s.qx[i] * sx + s.sy[j] * syv + s.qz[k] * sz;
            T v = cm1 * (syv - cm2 * dot);
            if (DIVV) v = v + cm1 * (s.nu * s.sy[j] * dv[q + s.nz]);
            return v;
        } else {
            if (j >= s.ny - 1 || k >= s.nz - 1) return T(0);
            T sx = (i != 0) ? Sx[q - s.nyz + 1] : T(0);             // (i-1, j, k+1)
            T sy = (j != 0) ? Sy[q - s.nz + 1] : T(0);              // (i, j-1, k+1)
            T m2 = s.qx[i] * s.qx[i] + s.qy[j] * s.qy[j] + s.sz[k] * s.sz[k];
            T cm1 = s.scale / (s.nu * m2), cm2 = s.sz[k] / m2;
            T szv = Sz[q];
            T dot = s.qx[i] * sx + s.qy[j] * sy + s.sz[k] * szv;
            T v = cm1 * (szv - cm2 * dot);
            if (DIVV) v = v + cm1 * (s.nu * s.sz[k] * dv[q + 1]);
            return v;
        }
    }
};

// N = beta psi^3 - gamma psi^5 - v . grad psi (adv/cosAdvTrackMult.cpp:1290-1303)
template <typename T>
struct LdAdvN {
    const T *__restrict__ psi, *__restrict__ vx, *__restrict__ vy, *__restrict__ vz;
    const T *__restrict__ gx, *__restrict__ gy, *__restrict__ gz;
    T beta, gamma;
    __device__ __forceinline__ T operator()(long long q, int, int, int) const
    {
        return nl3(psi[q], beta, gamma) - vx[q] * gx[q] - vy[q] * gy[q] - vz[q] * gz[q];
    }
};

// ---------------------------------------------------------------- storers -------------
// Crank-Nicolson / Adams-Bashforth update fed by the freshly transformed N
// (no-adv/cosNoAdvTrackSing.cpp:752-753, adv/cosAdvTrackMult.cpp:1362-1364):
//   psihat <- (C1 psihat + dt/2 scale (3 N - Nprev)) / C2,  C1,2 = 1 +- dt/2 L(q);  Nprev <- N
template <typename T>
struct StUpdCN {
    Spec<T> s;
    T *__restrict__ ph;
    T *__restrict__ np;
    __device__ __forceinline__ void operator()(long long q, int i, int j, int k, T v) const
    {
        T al = s.alin(i, j, k);
        T c1 = T(1) + s.dtd2 * al, c2 = T(1) - s.dtd2 * al;
        T npv = np[q];
        ph[q] = (c1 * ph[q] + s.dtd2 * s.scale * (T(3) * v - npv)) / c2;
        np[q] = v;
    }
};

// Scales a forward transform into psihat (pre-loop: psihat = scale REDFT10^3 psi)
template <typename T>
struct StScale {
    T *__restrict__ p;
    T scale;
    __device__ __forceinline__ void operator()(long long q, int, int, int, T v) const { p[q] = scale * v; }
};

}  // namespace smadft
