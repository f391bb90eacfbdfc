// ic.cpp -- initial-condition builders (host only).  They write the reference layout
// idx = (i*ny + j)*nz + k and use node positions x_i = i dx as the reference does
// (adv/cosAdvTrackMult.cpp:500-536 writes cos(q0 k dz)).
#include <cmath>
#include <cstdint>

#include "smadft.h"

namespace {

// SplitMix64 finaliser (Steele, Lea, Flood 2014), used as a counter-based stream.
inline uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// uniform in [0, 1) from (seed, counter)
inline double uni(uint64_t seed, uint64_t ctr)
{
    uint64_t x = mix64(seed ^ mix64(ctr));
    return (double)(x >> 11) * (1.0 / 9007199254740992.0);
}

bool grid_ok(const smadft_params *p)
{
    return p && p->nx > 0 && p->ny > 0 && p->nz > 0 && p->nw > 0 && p->q0 > 0;
}

}  // namespace

extern "C" int smadft_ic_interface(const smadft_params *p, double A, double bump_amp, double noise,
                                   unsigned long long seed, double *psi)
{
    if (!grid_ok(p) || !psi) return SMADFT_ERR_INVALID;
    const double dx = 2.0 * M_PI / (p->q0 * p->nw);
    const double Lx = p->nx * dx, Ly = p->ny * dx;
    const double lam0 = 2.0 * M_PI / p->q0;
    for (int i = 0; i < p->nx; i++)
        for (int j = 0; j < p->ny; j++) {
            const double x0 = 0.5 * Lx + bump_amp * std::sin(2.0 * M_PI * (j * dx) / Ly);
            const double env = 0.5 * (1.0 - std::tanh((i * dx - x0) / (2.0 * lam0)));
            for (int k = 0; k < p->nz; k++) {
                const long long q = ((long long)i * p->ny + j) * p->nz + k;
                double v = A * std::cos(p->q0 * k * dx) * env;
                if (noise != 0.0) v += noise * (2.0 * uni(seed, (uint64_t)q) - 1.0);
                psi[q] = v;
            }
        }
    return SMADFT_OK;
}

// The reference's single focal conic (torus cyclide) IC, no-adv/cosNoAdvTrackSing.cpp:403-449,
// adv/cosAdvTrackMult.cpp:496-542, quasi/quasi.cpp:675-721 (aE = bE = radius, mid = Nx/2).
extern "C" int smadft_ic_focal_conic(const smadft_params *p, double A, double radius, double *psi)
{
    if (!grid_ok(p) || !psi || !(radius > 0)) return SMADFT_ERR_INVALID;
    const double dz = 2.0 * M_PI / (p->q0 * p->nw);
    const double mid = p->nx / 2;
    const double aE = radius, bE = radius;
    for (int i = 0; i < p->nx; i++)
        for (int j = 0; j < p->ny; j++)
            for (int k = 0; k < p->nz; k++) {
                const long long q = ((long long)i * p->ny + j) * p->nz + k;
                double v = 0.0;
                if (k < bE + 1) {
                    const double xs = i - mid, ys = j - mid, zs = k;
                    const double ds = std::sqrt(xs * xs + ys * ys);
                    if (ds < mid) {
                        if (std::sqrt(std::pow((ds - mid) / aE, 2) + std::pow(zs / bE, 2)) > 1) v = 0.0;
                        else v = A * std::cos(p->q0 * dz * std::sqrt(std::pow((bE / aE) * (ds - mid), 2) + zs * zs));
                    } else {
                        v = (std::fabs(zs) < bE) ? A * std::cos(p->q0 * zs * dz) : 0.0;
                    }
                }
                psi[q] = v;
            }
    return SMADFT_OK;
}

// Smectic layers A cos(q0 z) over the smectic half x < L/2 (x-normal interface profile of
// the flat builder) with `count` radial (onion-like) focal perturbations: inside a sphere
// of radius R around a centre the layers follow cos(q0 |r - c|), blended over one
// wavelength.  Centres are uniform in the smectic half, R uniform in [rmin, rmax] lambda0.
extern "C" int smadft_ic_conics(const smadft_params *p, double A, int count, double rmin, double rmax,
                                double noise, unsigned long long seed, double *psi)
{
    if (!grid_ok(p) || !psi || count < 0 || count > 64 || rmin < 0 || rmax < rmin) return SMADFT_ERR_INVALID;
    const double dx = 2.0 * M_PI / (p->q0 * p->nw);
    const double Lx = p->nx * dx, Ly = p->ny * dx, Lz = p->nz * dx;
    const double lam0 = 2.0 * M_PI / p->q0;
    double cx[64], cy[64], cz[64], R[64];
    for (int c = 0; c < count; c++) {
        const uint64_t base = 0x5A5A0000ull + 16ull * (uint64_t)c;
        cx[c] = uni(seed, base + 0) * 0.5 * Lx;
        cy[c] = uni(seed, base + 1) * Ly;
        cz[c] = uni(seed, base + 2) * Lz;
        R[c] = (rmin + (rmax - rmin) * uni(seed, base + 3)) * lam0;
    }
    for (int i = 0; i < p->nx; i++) {
        const double x = i * dx;
        const double env = 0.5 * (1.0 - std::tanh((x - 0.5 * Lx) / (2.0 * lam0)));
        for (int j = 0; j < p->ny; j++) {
            const double y = j * dx;
            for (int k = 0; k < p->nz; k++) {
                const double z = k * dx;
                double layer = std::cos(p->q0 * z);
                for (int c = 0; c < count; c++) {
                    const double d = std::sqrt((x - cx[c]) * (x - cx[c]) + (y - cy[c]) * (y - cy[c]) +
                                               (z - cz[c]) * (z - cz[c]));
                    const double w = 0.5 * (1.0 - std::tanh((d - R[c]) / lam0));
                    layer = w * std::cos(p->q0 * d) + (1.0 - w) * layer;
                }
                const long long q = ((long long)i * p->ny + j) * p->nz + k;
                double v = A * layer * env;
                if (noise != 0.0) v += noise * (2.0 * uni(seed, (uint64_t)q) - 1.0);
                psi[q] = v;
            }
        }
    }
    return SMADFT_OK;
}
