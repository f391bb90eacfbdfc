/*
 * r2r.h -- FP64 real-to-real transforms used by the oracle (test infrastructure only).
 *
 * The transforms follow FFTW 3.3's published r2r definitions (unnormalised), which is
 * what the reference calls through fftw_mpi_plan_r2r_3d / fftw_execute
 * (no-adv/cosNoAdvTrackSing.cpp:342-375, adv/cosAdvTrackMult.cpp:419-467,
 *  quasi/quasi.cpp:519-565).  FFTW itself is an unvendored dependency of the
 * reference (FFTW 3.3.4 in runAdv:28, 3.3.8 in runComp:23) and is not installed
 * here, so this file restates the published algorithm:
 *
 *   REDFT10 (DCT-II):  Y_k = 2 sum_{j<n} X_j cos(pi (j+1/2) k / n)
 *   REDFT01 (DCT-III): Y_k = X_0 + 2 sum_{0<j<n} X_j cos(pi j (k+1/2) / n)
 *   RODFT10 (DST-II):  Y_k = 2 sum_{j<n} X_j sin(pi (j+1/2)(k+1) / n)
 *   RODFT01 (DST-III): Y_k = (-1)^k X_{n-1} + 2 sum_{j<n-1} X_j sin(pi (j+1)(k+1/2) / n)
 *
 * computed in O(n log n) by Makhoul's reordering (J. Makhoul, IEEE TASSP 28(1), 1980)
 * over a mixed-radix Stockham complex FFT.  The sine kinds reduce to the cosine kinds:
 *   RODFT10[x]_k = REDFT10[(-1)^j x_j]_{n-1-k}
 *   RODFT01[X]_k = (-1)^k REDFT01[X_{n-1-j}]_k
 * Pinned against scipy.fft.dct/dst (types 2/3, norm=None) by tests/test_oracle_r2r.py.
 */
#ifndef SMADFT_ORACLE_R2R_H
#define SMADFT_ORACLE_R2R_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_REDFT10 = 0, ORC_REDFT01 = 1, ORC_RODFT10 = 2, ORC_RODFT01 = 3 };

/* 1-D transform of one line (in may equal out). */
void orc_r2r_1d(const double *in, double *out, int n, int kind);

/* 3-D transform of an nx*ny*nz array laid out idx = (i*ny + j)*nz + k (in may equal out).
 * kx, ky, kz are the per-axis kinds.  Uses OpenMP threads over lines. */
void orc_r2r_3d(const double *in, double *out, int nx, int ny, int nz, int kx, int ky, int kz);

/* Number of OpenMP threads the 3-D transform uses (0 = library default). */
void orc_set_threads(int nthreads);
int orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
