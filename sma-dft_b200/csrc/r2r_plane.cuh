// r2r_plane.cuh -- the z and y passes of a 3-D r2r transform in one kernel, one (y, z)
// plane per thread-block cluster (ny = nz = N in {64, 128, 256}).
//
// A separate z pass and y pass each read and write the whole field once.  Here a cluster
// of C = N / 32 CTAs holds one plane i between the two 1-D transforms, so the field
// crosses HBM once for both axes:
//
//   phase 1  CTA `rank` loads rows y = 32 rank .. 32 rank + 31 through the Loader
//            (coalesced 8-byte accesses, Makhoul permutation applied on the way into
//            shared memory; rows 2c and 2c + 1 travel as one complex line) and runs the
//            register-direct transform of rd_fft along z.  The transformed rows go to a
//            row buffer whose column index is XOR-swizzled per row pair.
//   cluster barrier
//   phase 2  CTA `rank` owns columns z = 32 rank .. 32 rank + 31 (column pairs packed as
//            complex lines): each thread reads its 16 stage-0 points straight from the
//            owning CTAs' row buffers (distributed shared memory, 8/16-byte reads).
//   cluster barrier (every remote read done: the row buffer is free again)
//            rd_fft along y in the same shared memory, outputs through the Storer.
//
// A launch may carry NC components (LoadMulti / StoreMulti): cluster q then transforms
// component q mod NC of plane q / NC, so the components that read the same input fields
// run on neighbouring clusters at the same time and share those reads in L2.
//
// The swizzle puts element (r, k) of the row buffer at r N + (k ^ 2 ((r / 2) mod 16)):
// the phase-1 writes of a half-warp (16 row pairs, one column) hit 16 different banks and
// the phase-2 reads (one row, 16 consecutive column pairs) stay in one 128-byte window.
#pragma once

#include <cooperative_groups.h>

#include "r2r_rd.cuh"

namespace smadft {

template <int N>
struct PlaneInfo {
    static constexpr int ROWS = 2 * kRdLines;   // real rows (phase 1) / columns (phase 2) per CTA
    static constexpr int C = N / ROWS;          // CTAs per cluster = one plane
};

// bytes of the exchange / row buffer (shared by both phases) and of the whole allocation
template <typename T, int N>
constexpr size_t plane_body_bytes()
{
    const size_t a = (size_t)kRdLines * RdInfo<N>::LD * sizeof(cpx<T>);
    const size_t b = (size_t)PlaneInfo<N>::ROWS * N * sizeof(T);
    return a > b ? a : b;
}
template <typename T, int N>
constexpr size_t plane_smem_bytes() { return plane_body_bytes<T, N>() + 2 * (size_t)N * sizeof(cpx<T>); }

__device__ __forceinline__ int plane_swz(int r) { return ((r >> 1) & 15) << 1; }

// one packed pair (k, k + 1) of a row; p is 2 sizeof(T)-aligned
template <typename T>
__device__ __forceinline__ cpx<T> ld_pair(const T *p)
{
    if constexpr (sizeof(T) == 4) {
        const float2 u = *reinterpret_cast<const float2 *>(p);
        return {u.x, u.y};
    } else {
        const double2 u = *reinterpret_cast<const double2 *>(p);
        return {u.x, u.y};
    }
}

template <typename T, int N, int NC, class LD, class ST>
__global__ void __launch_bounds__(RdInfo<N>::THREADS, 2) r2r_plane_kernel(Geom g, PlaneKinds<NC> kinds, LD ld,
                                                                          const cpx<T> *__restrict__ wt_g,
                                                                          const cpx<T> *__restrict__ ht_g, ST st)
{
    namespace cg = cooperative_groups;
    using RI = RdInfo<N>;
    constexpr int R0 = RI::R0, R1 = RI::R1, NT = RI::THREADS;
    constexpr int BPT = R0 / R1 > 0 ? R0 / R1 : 1;
    constexpr int NP = BPT * R1;
    constexpr int ROWS = PlaneInfo<N>::ROWS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T> *buf = reinterpret_cast<cpx<T> *>(smem_raw);
    T *rows = reinterpret_cast<T *>(smem_raw);
    cpx<T> *wt = reinterpret_cast<cpx<T> *>(smem_raw + plane_body_bytes<T, N>());
    cpx<T> *ht = wt + N;
    for (int m = threadIdx.x; m < N; m += NT) {
        wt[m] = wt_g[m];
        ht[m] = ht_g[m];
    }
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int cid = blockIdx.x / PlaneInfo<N>::C;         // cluster
    const int i = cid / NC, comp = cid % NC;              // plane (x index), component
    const int kind_y = kinds.ky[comp], kind_z = kinds.kz[comp];
    const idx_t pbase = i * g.nyz;                        // element (i, 0, 0)
    // thread (c, j) as in r2r_rd_kernel: c = complex line, j = first-stage butterfly
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5, hh16 = lane >> 4;
    const int c = lane & 15;
    const int j = (wi == 0) ? (hh16 ? R1 / 2 : 0) : (hh16 ? R1 - wi : wi);

    // ---- phase 1: z transform of rows r0 .. r0 + 31 (complex line c = rows r0 + 2c, +1)
    {
        const bool fwd = (kind_z == K_DCT2 || kind_z == K_DST2);
        const bool sine = (kind_z == K_DST2 || kind_z == K_DST3);
        const int r0 = rank * ROWS;
        constexpr int PER = kRdLines * (N / 2) / NT;      // (line, sample pair) tasks per thread
        T va[PER][2], vb[PER][2];
        ld.visit(comp, [&](const auto &l) {
#pragma unroll
            for (int e = 0; e < PER; e++) {
                const int t = e * NT + threadIdx.x;
                const int ln = t / (N / 2), n = 2 * (t % (N / 2));
                const int ja = r0 + 2 * ln;
                const idx_t qa = pbase + ja * g.nz + n;
                l.template load<2>(qa, i, ja, n, va[e]);
                l.template load<2>(qa + g.nz, i, ja + 1, n, vb[e]);
            }
        });
#pragma unroll
        for (int e = 0; e < PER; e++) {
            const int t = e * NT + threadIdx.x;
            const int ln = t / (N / 2), n = 2 * (t % (N / 2));
            cpx<T> *L = buf + ln * RI::LD;
            cpx<T> z0 = {va[e][0], vb[e][0]}, z1 = {va[e][1], vb[e][1]};
            int p0, p1;                                   // positions of samples n, n + 1
            if (fwd) {
                p0 = n / 2;                               // Makhoul: even samples first,
                p1 = N - 1 - n / 2;                       // odd ones reversed at the end
                if (sine) z1 = {-z1.x, -z1.y};            // DST-II negates odd samples
            } else if (sine) {
                p0 = N - 1 - n;                           // DST-III reads the line reversed
                p1 = N - 2 - n;
            } else {
                p0 = n;
                p1 = n + 1;
            }
            L[RI::phys(p0)] = z0;
            L[RI::phys(p1)] = z1;
        }
        __syncthreads();
        cpx<T> *line = buf + c * RI::LD;
        cpx<T> v[R0];
#pragma unroll
        for (int q = 0; q < R0; q++) v[q] = line[RI::phys(j + q * R1)];
        cpx<T> x1[BPT][R1];
        rd_fft<T, N>(v, x1, line, wt, ht, j, wi, fwd, sine);
        __syncthreads();                                  // exchange buffer reads done
        const int sw = plane_swz(2 * c);
#pragma unroll
        for (int pnt = 0; pnt < NP; pnt++) {
            const cpx<T> z = x1[pnt / R1][pnt % R1];
            const int kk = rd_out_pos<N>(j, pnt, fwd, sine) ^ sw;
            rows[(2 * c) * N + kk] = z.x;
            rows[(2 * c + 1) * N + kk] = z.y;
        }
    }
    cl.sync();

    // ---- phase 2: y transform of columns k0 .. k0 + 31 (complex line c = columns k0 + 2c, +1)
    {
        const bool fwd = (kind_y == K_DCT2 || kind_y == K_DST2);
        const bool sine = (kind_y == K_DST2 || kind_y == K_DST3);
        const int k = rank * ROWS + 2 * c;
        cpx<T> v[R0];
#pragma unroll
        for (int q = 0; q < R0; q++) {
            const int p = j + q * R1;
            const int r = fwd ? makhoul_src<N>(p) : (sine ? N - 1 - p : p);   // row (y index)
            const int lr = r % ROWS;
            const T *src = cl.map_shared_rank(rows, r / ROWS);
            v[q] = ld_pair<T>(src + lr * N + (k ^ plane_swz(lr)));
            if (fwd && sine && (r & 1)) v[q] = {-v[q].x, -v[q].y};
        }
        cl.sync();                                        // every row buffer has been read
        cpx<T> x1[BPT][R1];
        rd_fft<T, N>(v, x1, buf + c * RI::LD, wt, ht, j, wi, fwd, sine);

        // stores: the storer's reads (pre) for a chunk of points go out before its writes
        const idx_t base = pbase + k;
        constexpr int CH = 4;
        constexpr int PL = pre_len<ST, 2>();
#pragma unroll
        for (int p0 = 0; p0 < NP; p0 += CH) {
            T pre_buf[CH][PL];
#pragma unroll
            for (int u = 0; u < CH; u++) {
                const int o = rd_out_pos<N>(j, p0 + u, fwd, sine);
                st.template pre<2>(comp, base + o * g.nz, i, o, k, pre_buf[u]);
            }
#pragma unroll
            for (int u = 0; u < CH; u++) {
                const int pnt = p0 + u;
                const cpx<T> z = x1[pnt / R1][pnt % R1];
                const int o = rd_out_pos<N>(j, pnt, fwd, sine);
                const T w2[2] = {z.x, z.y};
                st.template fin<2>(comp, base + o * g.nz, i, o, k, w2, pre_buf[u]);
            }
        }
    }
}

}  // namespace smadft
