// surface.cu -- one loop body with the interface diagnostics the reference writes every
// 1000 steps: per (i, j) column the flat-tracked interface along z, the normal velocity
// dTpsi/|grad psi| and the curvatures 2H and K there (Megrabov's divergence forms).
//   noadv: no-adv/cosNoAdvTrackSing.cpp:737-764 (spectra), 808-964 (interface, finite-
//          difference gradient);
//   adv:   adv/cosAdvTrackMult.cpp:1311-1347 (spectra), 1417-1515 (interface, the step's
//          spectral gradient).
// Everything is evaluated at the step's starting state psi^n, as the reference does (its
// tracker reads psi_local before psi_local = psiNew_local).
#include "models.cuh"
#include "steps.h"

namespace smadft {

// dTpsi spectrum: L(q) psihat^n + scale Nhat^n (psihat scaled, Nhat unscaled)
template <typename T>
struct LdSurfDt {
    Spec<T> s;
    const double *__restrict__ ph;   // psihat^n (FP64 state copy)
    const T *__restrict__ nq;        // Nhat^n
    T scale;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int i, int j, int k, T *out) const
    {
        T p[V], n[V];
        vld_as<T, V, double>(ph, q, p);
        vld<T, V>(nq, q, n);
#pragma unroll
        for (int u = 0; u < V; u++) out[u] = s.alin(i, j, k + u) * p[u] + scale * n[u];
    }
};

// second-derivative spectrum along AX: -q_AX^2 psihat^n
template <typename T, int AX>
struct LdSurfD2 {
    Spec<T> s;
    const double *__restrict__ ph;
    template <int V>
    __device__ __forceinline__ void load(idx_t q, int i, int j, int k, T *out) const
    {
        T p[V];
        vld_as<T, V, double>(ph, q, p);
#pragma unroll
        for (int u = 0; u < V; u++) {
            const T qa = AX == 0 ? s.qx[i] : (AX == 1 ? s.qy[j] : s.qz[k + u]);
            out[u] = -qa * qa * p[u];
        }
    }
};

struct SurfGeom {
    int nx, ny, nz;
    double dx, dy, dz;
};

// centred / one-sided (2 (a - b) / 2h at the walls) difference of psi along `axis` at (i, j, k)
template <typename T>
__device__ double fd_grad(const T *psi, const SurfGeom &g, int axis, int i, int j, int k)
{
    const long long q = ((long long)i * g.ny + j) * g.nz + k;
    const int n = axis == 0 ? g.nx : (axis == 1 ? g.ny : g.nz);
    const int t = axis == 0 ? i : (axis == 1 ? j : k);
    const long long st = axis == 0 ? (long long)g.ny * g.nz : (axis == 1 ? g.nz : 1);
    const double td = 2.0 * (axis == 0 ? g.dx : (axis == 1 ? g.dy : g.dz));
    if (t > 0 && t < n - 1) return (double(psi[q + st]) - double(psi[q - st])) / td;
    if (t == 0) return 2.0 * (double(psi[q + st]) - double(psi[q])) / td;
    return 2.0 * (double(psi[q]) - double(psi[q - st])) / td;
}

// One thread per (i, j) column (the reference's loop, FP64 arithmetic).  gx/gy/gz null: the
// gradient is the finite difference of psi (noadv), else the given fields (adv).  An
// element past the end of a gradient field reads 0.
template <typename T>
__global__ void surface_kernel(SurfGeom g, const T *__restrict__ psi, const T *__restrict__ gx,
                               const T *__restrict__ gy, const T *__restrict__ gz, const T *__restrict__ dT,
                               const T *__restrict__ dxx, const T *__restrict__ dyy, const T *__restrict__ dzz,
                               int *__restrict__ sidx, double *__restrict__ vel, double *__restrict__ cH,
                               double *__restrict__ cK)
{
    const long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= (long long)g.nx * g.ny) return;
    const int i = (int)(col / g.ny), j = (int)(col % g.ny);
    const long long n = (long long)g.nx * g.ny * g.nz;
    const bool fd = gx == nullptr;
    auto G = [&](int axis, long long q) -> double {      // gradient component at element q
        if (q >= n) return 0.0;
        if (fd) {
            const int ii = (int)(q / ((long long)g.ny * g.nz));
            const int jj = (int)((q / g.nz) % g.ny), kk = (int)(q % g.nz);
            return fd_grad(psi, g, axis, ii, jj, kk);
        }
        const T *f = axis == 0 ? gx : (axis == 1 ? gy : gz);
        return double(f[q]);
    };
    sidx[col] = -1;
    vel[col] = cH[col] = cK[col] = __longlong_as_double(0x7ff8000000000000ll);   // NaN
    const double tdy = 2.0 * g.dy, tdz = 2.0 * g.dz;
    const long long base = col * g.nz;
    int track = 0;
    for (int k = g.nz - 1; k > -1; k--) {
        long long index = base + k;
        const double pv = double(psi[index]);
        if (pv > 0.7 && track == 0) track = 1;
        if (pv < 0.0 && track == 1) {
            int k2 = k;
            if (fabs(pv) > fabs(double(psi[index + 1]))) {
                index = index + 1;
                k2 = k + 1;
            }
            sidx[col] = k2;
            const double gxv = G(0, index), gyv = G(1, index), gzv = G(2, index);
            const double gv = sqrt(gxv * gxv + gyv * gyv + gzv * gzv);
            vel[col] = double(dT[index]) / gv;
            const long long rowk2 = (long long)i * g.ny;   // (i, j', k2) = (rowk2 + j') nz + k2
            auto at = [&](int jj) { return (rowk2 + jj) * g.nz + k2; };
            double Dxy = 0, Dxz = 0, Dyz = 0;
            if (j > 0 && j < g.ny - 1) Dxy = (G(0, at(j + 1)) - G(0, at(j - 1))) / tdy;
            if (j == 0) Dxy = 2 * (G(0, at(1)) - G(0, at(0))) / tdy;
            if (j == g.ny - 1) Dxy = 2 * (G(0, at(j)) - G(0, at(j - 1))) / tdy;
            if (k > 0 && k < g.nz - 1) {
                Dxz = (G(0, index + 1) - G(0, index - 1)) / tdz;
                Dyz = (G(1, index + 1) - G(1, index - 1)) / tdz;
            }
            if (k == 0) {
                Dxz = 2 * (G(0, index + 1) - G(0, index)) / tdz;
                Dyz = 2 * (G(1, index + 1) - G(1, index)) / tdz;
            }
            const double Dxx = double(dxx[index]), Dyy = double(dyy[index]), Dzz = double(dzz[index]);
            cH[col] = ((gyv * gyv + gzv * gzv) * Dxx + (gxv * gxv + gzv * gzv) * Dyy + (gxv * gxv + gyv * gyv) * Dzz -
                       2 * (gxv * gyv * Dxy + gxv * gzv * Dxz + gyv * gzv * Dyz)) /
                      (gv * gv * gv);
            cK[col] = (gzv * gzv * (Dxx * Dyy - Dxy * Dxy) + gxv * gxv * (Dyy * Dzz - Dyz * Dyz) +
                       gyv * gyv * (Dxx * Dzz - Dxz * Dxz) +
                       2 * (gyv * Dxy * (gzv * Dxz - gxv * Dzz) + gxv * Dxz * (gyv * Dyz - gzv * Dyy) +
                            gzv * Dyz * (gxv * Dxy - gyv * Dxx))) /
                      (gv * gv * gv * gv);
            track = 2;
        }
    }
}

template <typename T>
int surface_step(Ctx &c, SurfaceScratch &sc)
{
    Spec<T> s = make_spec<T>(c);
    const size_t nb = sizeof(double) * c.n;
    SMADFT_CUDA(cudaMemcpyAsync(sc.psih_prev, c.slot[S_PSIH], nb, cudaMemcpyDeviceToDevice, c.stream));
    int rc;
    if (c.p.model == SMADFT_MODEL_NOADV) {
        if ((rc = noadv_step<T>(c, true))) return rc;   // psi^n stays in S_PSI, psi^{n+1} in S_PSI2
    } else {
        if ((rc = adv_step<T>(c))) return rc;           // S_PSI = psi^n, S_G* = grad psi^n
    }
    T *f[4];
    for (int m = 0; m < 4; m++) f[m] = reinterpret_cast<T *>(sc.fields) + (size_t)m * c.n;
    {
        const int kk[4] = {K_DCT3, K_DCT3, K_DCT3, K_DCT3};
        T *const out[4] = {f[0], f[1], f[2], f[3]};
        if ((rc = r2r3d_multi<T, 4, 0>(c, kk, kk, kk, out, LdSurfDt<T>{s, sc.psih_prev, c.f<T>(S_NP), T(c.scale)},
                                    LdSurfD2<T, 0>{s, sc.psih_prev}, LdSurfD2<T, 1>{s, sc.psih_prev},
                                    LdSurfD2<T, 2>{s, sc.psih_prev})))
            return rc;
    }
    SurfGeom g{c.g.nx, c.g.ny, c.g.nz, c.dx, c.dy, c.dz};
    const bool fd = c.p.model == SMADFT_MODEL_NOADV;
    const long long cols = (long long)c.g.nx * c.g.ny;
    surface_kernel<T><<<(unsigned)((cols + 127) / 128), 128, 0, c.stream>>>(
        g, c.f<T>(S_PSI), fd ? nullptr : c.f<T>(S_GX), fd ? nullptr : c.f<T>(S_GY), fd ? nullptr : c.f<T>(S_GZ),
        f[0], f[1], f[2], f[3], sc.idx, sc.vel, sc.curvH, sc.curvK);
    SMADFT_CUDA(cudaGetLastError());
    c.launches++;
    return SMADFT_OK;   // noadv: psi^{n+1} waits in S_PSI2 (the caller moves it to S_PSI)
}

#if !defined(SMADFT_INST_DOUBLE)
template int surface_step<float>(Ctx &, SurfaceScratch &);
#endif
#if !defined(SMADFT_INST_FLOAT)
template int surface_step<double>(Ctx &, SurfaceScratch &);
#endif

}  // namespace smadft
