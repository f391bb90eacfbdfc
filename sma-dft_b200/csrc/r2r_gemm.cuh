// r2r_gemm.cuh -- GEMM-form r2r pass along z (the contiguous axis) on the 5th-generation
// tensor cores: tcgen05.mma with the DCT matrix resident in tensor memory, the field rows
// streamed in by TMA, FP32 accumulators in tensor memory.
//
// The four r2r kinds of length N are dense matrices Y = M x (FFTW's REDFT10 / REDFT01 /
// RODFT10 / RODFT01, unnormalised).  For N = 256 each splits by its mirror symmetry into two
// 128 x 128 blocks, halving the work:
//   * forward kinds (DCT-II, DST-II): with e_n = x_n + x_{N-1-n}, o_n = x_n - x_{N-1-n}
//     (n < N/2), the even outputs Y_{2k} = E e and the odd ones Y_{2k+1} = O o;
//   * inverse kinds (DCT-III, DST-III): with p_j = x_{2j}, q_j = x_{2j+1},
//     Y_k = (P p + Q q)_k and Y_{N-1-k} = (P p - Q q)_k for k < N/2.
// For N = 128 the whole 128 x 128 matrix is one block.
//
// Precision: a field row is scaled by a power of two s (its largest entry near 2^13) and
// split into FP16 hi + lo parts (x s = hi + lo + O(2^-22 x s)); the block matrices are
// stored scaled by 2^12 and split the same way on the host.  Three products
// (A_hi B_hi + A_lo B_hi + A_hi B_lo) accumulate in FP32, so the result carries about 22
// significant bits, the accuracy class of the FP32 FFT passes; the epilogue multiplies by
// 2^-12 / s.
//
// Work split (one persistent CTA per SM, 320 threads, tiles of kGzRows field rows):
//   warp 8      TMA producer: the tile's rows (FP32, 128-byte swizzled boxes of 32 x kGzRows)
//               into a kGzStages-deep staging ring;
//   warps 0-3   converters: per row, the butterflies (forward) or the even/odd split
//               (inverse), the row scale, the FP16 hi/lo split, written as the K-major,
//               128-byte-swizzled B operand of the MMA (N = kGzRows rows, K = 128 per
//               block), double-buffered so that a tile converts while the last one multiplies;
//   warp 9      MMA issuer: per block 8 tcgen05.mma (M = 128, N = kGzRows, K = 16) of
//               A_hi B_hi into one accumulator and 16 of A_lo B_hi + A_hi B_lo into a second
//               (A, the block matrix, read from tensor memory; both accumulators in tensor
//               memory, double-buffered), tcgen05.commit to the barriers;
//   warps 4-7   epilogue: tcgen05.ld of the accumulators (lane = output index), their sum,
//               the scale, the output order, and 8-byte (forward) or 4-byte (inverse)
//               stores: a warp writes 256 or 2 x 128 contiguous bytes of one row per
//               instruction.
// The tensor cores' FP32 accumulation does not round to nearest: it loses magnitude
// (a bias of a few 1e-7 relative per pass when all three products share one accumulator).
// Keeping the small cross products in their own accumulator, summed in FP32 in the
// epilogue, limits that loss to the hi x hi accumulation.
// Every wait on an mbarrier is bounded (clock64 deadline); a wait that runs out sets the
// error word, makes the other roles stop, waits (bounded) for the CTA's own copies and MMAs
// in flight and frees the tensor memory before returning.  Each row is read once (TMA,
// before) and written once (epilogue, after) by the same CTA, so the pass may run in place.
#pragma once

#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace smadft {

constexpr int kGzRows = 32;            // field rows per tile (the MMA's N)
constexpr int kGzStages = 3;           // staging buffers for the TMA loads
constexpr int kGzThreads = 320;        // 10 warps: 0-3 converters, 4-7 epilogue, 8 TMA, 9 MMA
constexpr int kGzK = 128;              // K (and M) of one block
constexpr double kGzMatScale = 4096.0;  // block matrices are stored scaled by 2^12
constexpr long long kGzWaitCycles = 4000000000ll;   // about 2 s at the B200's clocks

template <int N>
struct GzInfo {
    static_assert(N == 128 || N == 256, "GEMM-form z pass: N = 128 or 256");
    static constexpr int NB = N / 128;                              // 128 x 128 blocks
    static constexpr int BOXES = N / 32;                            // 128-byte boxes per row
    static constexpr uint32_t STAGE_BYTES = kGzRows * N * 4;        // one FP32 tile
    static constexpr uint32_t OP_BYTES = kGzRows * kGzK * 2;        // one FP16 operand (16 KiB)
    static constexpr uint32_t BOP_BYTES = NB * 2 * OP_BYTES;        // hi and lo per block (one buffer)
    // tensor memory: A[b][hl] at (2b + hl) * 64; accumulators D[d][b][main, corr] at
    // D_COL0 + ((d NB + b) 2 + c) kGzRows
    static constexpr uint32_t A_COL0 = 0;
    static constexpr uint32_t D_COL0 = NB * 2 * 64;
    static constexpr uint32_t COLS_USED = D_COL0 + 2 * NB * 2 * kGzRows;
    static constexpr uint32_t TMEM_COLS = COLS_USED <= 32 ? 32 : COLS_USED <= 64 ? 64 : COLS_USED <= 128 ? 128
                                        : COLS_USED <= 256 ? 256 : 512;
    static constexpr uint32_t OFF_STAGE = 0;
    static constexpr uint32_t OFF_BOP = kGzStages * STAGE_BYTES;
    static constexpr uint32_t OFF_SCALE = OFF_BOP + 2 * BOP_BYTES;  // float [4][kGzRows]
    static constexpr uint32_t OFF_BAR = OFF_SCALE + 4 * kGzRows * 4;
    // barriers: full[S] empty[S] bready[2] bfree[2] dfull[2] dempty[2], then tmem slot + abort flag
    static constexpr uint32_t NBAR = 2 * kGzStages + 8;
    static constexpr uint32_t OFF_MISC = OFF_BAR + NBAR * 8;
    static constexpr uint32_t SMEM = OFF_MISC + 16 + 1024;          // + alignment slack
    // elements of the matrix table per kind: NB blocks x {hi, lo} x 128 x 128
    static constexpr size_t MAT_ELEMS = (size_t)NB * 2 * kGzK * kGzK;
};

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t gz_smem(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void gz_bar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void gz_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void gz_arrive_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool gz_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on phase `parity` of a barrier: false when the deadline passed or another
// role gave up (the shared abort flag); the first role to give up records `code`.
__device__ __forceinline__ bool gz_wait(uint32_t bar, uint32_t parity, volatile int *abort, int *err, int code)
{
    const long long t0 = clock64();
    while (!gz_try_wait(bar, parity)) {
        if (*abort) return false;
        if (clock64() - t0 > kGzWaitCycles) {
            *abort = 1;
            atomicCAS(err, 0, code);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void gz_tma_load(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void gz_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void gz_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem d] (+)= A[tmem a] * B[smem desc], kind::f16, FP32 accumulate
__device__ __forceinline__ void gz_mma_ts(uint32_t d, uint32_t a, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d),
        "r"(a), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void gz_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// 16 consecutive 32-bit columns of this thread's lane
__device__ __forceinline__ void gz_tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}
__device__ __forceinline__ void gz_tmem_st16(uint32_t taddr, const uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
        "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}
__device__ __forceinline__ void gz_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void gz_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Shared-memory descriptor of a K-major operand in the 128-byte swizzle layout: rows of
// 128 bytes, 8-row groups 1024 bytes apart (SBO), descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t gz_desc(uint32_t addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFFu) >> 4);   // start address
    d |= (uint64_t)1u << 16;                    // leading byte offset (unused in this layout)
    d |= (uint64_t)(1024u >> 4) << 32;          // stride byte offset
    d |= (uint64_t)1u << 46;                    // version
    d |= (uint64_t)2u << 61;                    // 128-byte swizzle
    return d;
}

// Instruction descriptor: D FP32, A and B FP16, both K-major, M = 128, N = kGzRows.
__host__ __device__ constexpr uint32_t gz_idesc()
{
    return (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(kGzRows >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

// Byte offset of 16-bit element (row r, k) inside one K-major swizzled operand of kGzRows
// rows and kGzK = 128 columns (two 64-element chunks, each kGzRows x 128 bytes).
__device__ __forceinline__ uint32_t gz_bop_off(int r, int k)
{
    const int chunk = k >> 6, kk = k & 63;
    return (uint32_t)(chunk * (kGzRows * 128) + r * 128 + ((((kk >> 3) ^ (r & 7))) << 4) + (kk & 7) * 2);
}

// Power-of-two scale bringing the row maximum m into [2^13, 2^14), and its inverse times
// 2^-12 (the matrix scale) for the epilogue; rows of zeros (or below 2^-100) keep factor 0.
__device__ __forceinline__ void gz_row_scale(float m, float &s, float &back)
{
    const int eb = (int)((__float_as_uint(m) >> 23) & 0xFF);   // biased exponent of m
    if (eb < 27) {                                               // m < 2^-100 (or zero)
        s = 1.0f;
        back = 0.0f;
        return;
    }
    const int e = eb - 127;                                      // m in [2^e, 2^(e+1))
    s = __uint_as_float((uint32_t)(127 + 13 - e) << 23);         // 2^(13 - e), e >= -100
    back = __uint_as_float((uint32_t)(127 + e - 25) << 23);      // 2^(e - 13 - 12)
}

// hi/lo FP16 split of two scaled values, packed as (first, second) half2 words
__device__ __forceinline__ void gz_split2(float a, float b, uint32_t &hi, uint32_t &lo)
{
    const __half2 h = __floats2half2_rn(a, b);
    const float2 hf = __half22float2(h);
    const __half2 l = __floats2half2_rn(a - hf.x, b - hf.y);
    hi = *reinterpret_cast<const uint32_t *>(&h);
    lo = *reinterpret_cast<const uint32_t *>(&l);
}

// ---------------------------------------------------------------- the kernel
// mats: this kind's NB x {hi, lo} x 128 x 128 FP16 block matrices, row = output index,
// scaled by 2^12.  map: the field as a 2-D FP32 tensor [rows][N], boxes of 32 x kGzRows with
// the 128-byte swizzle.  FWD: forward kinds (butterflies in, interleaved out) or inverse
// kinds (even/odd split in, mirrored out); for N = 128 both are the plain block product.
template <int N, bool FWD>
__global__ void __launch_bounds__(kGzThreads, 1)
    r2r_gemm_z_kernel(const __grid_constant__ CUtensorMap map, float *out, int rows, const __half *__restrict__ mats,
                      int *err)
{
    using GI = GzInfo<N>;
    constexpr int NB = GI::NB;
    extern __shared__ __align__(1024) unsigned char gz_raw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>(((uintptr_t)gz_raw + 1023) & ~(uintptr_t)1023);
    const uint32_t sbase = gz_smem(sm);
    float *scale_back = reinterpret_cast<float *>(sm + GI::OFF_SCALE);
    const uint32_t bar0 = sbase + GI::OFF_BAR;
    constexpr uint32_t S = kGzStages;
    auto bar_full = [&](int s) { return bar0 + 8u * s; };
    auto bar_empty = [&](int s) { return bar0 + 8u * (S + s); };
    auto bar_bready = [&](int b) { return bar0 + 8u * (2 * S + b); };
    auto bar_bfree = [&](int b) { return bar0 + 8u * (2 * S + 2 + b); };
    auto bar_dfull = [&](int d) { return bar0 + 8u * (2 * S + 4 + d); };
    auto bar_dempty = [&](int d) { return bar0 + 8u * (2 * S + 6 + d); };
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(sm + GI::OFF_MISC);
    volatile int *abort = reinterpret_cast<volatile int *>(sm + GI::OFF_MISC + 4);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles = (rows + kGzRows - 1) / kGzRows;
    const int my_tiles = (int)((tiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x);

    if (threadIdx.x == 0) {
        for (int s = 0; s < kGzStages; s++) {
            gz_bar_init(bar_full(s), 1);
            gz_bar_init(bar_empty(s), 4);
        }
        for (int d = 0; d < 2; d++) {
            gz_bar_init(bar_bready(d), 4);
            gz_bar_init(bar_bfree(d), 1);
            gz_bar_init(bar_dfull(d), 1);
            gz_bar_init(bar_dempty(d), 4);
        }
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 9) {   // tensor memory for the block matrices and two accumulator sets
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(gz_smem(tmem_slot)),
                     "r"(GI::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    gz_fence_before();
    __syncthreads();
    gz_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp < 4) {
        // block matrices into tensor memory: lane (32 warp + lane) holds row k of each
        // operand, two FP16 per 32-bit column
        const int k = warp * 32 + lane;
        for (int op = 0; op < NB * 2; op++) {
            const uint4 *src = reinterpret_cast<const uint4 *>(mats + ((size_t)op * kGzK + k) * kGzK);
#pragma unroll
            for (int part = 0; part < 4; part++) {   // 4 x 16 columns = 128 FP16
                uint32_t r[16];
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    const uint4 q = src[part * 4 + v];
                    r[4 * v + 0] = q.x;
                    r[4 * v + 1] = q.y;
                    r[4 * v + 2] = q.z;
                    r[4 * v + 3] = q.w;
                }
                gz_tmem_st16(tmem + ((uint32_t)(warp * 32) << 16) + GI::A_COL0 + op * 64 + part * 16, r);
            }
        }
        gz_wait_st();
    }
    gz_fence_before();
    __syncthreads();
    gz_fence_after();

    if (warp == 8) {
        // ---------------- TMA producer
        if (lane == 0) {
            for (int i = 0; i < my_tiles; i++) {
                const int s = i % kGzStages;
                if (i >= kGzStages && !gz_wait(bar_empty(s), ((i / kGzStages) - 1) & 1, abort, err, 1)) break;
                const int row0 = ((int)blockIdx.x + i * (int)gridDim.x) * kGzRows;
                const uint32_t dst = sbase + GI::OFF_STAGE + s * GI::STAGE_BYTES;
                gz_arrive_tx(bar_full(s), GI::STAGE_BYTES);
#pragma unroll
                for (int c = 0; c < GI::BOXES; c++) gz_tma_load(dst + c * (kGzRows * 128), &map, c * 32, row0, bar_full(s));
            }
            // drain: every issued load has landed before the CTA may end (bounded)
            for (int i = (my_tiles > kGzStages ? my_tiles - kGzStages : 0); i < my_tiles; i++) {
                const long long t0 = clock64();
                while (!gz_try_wait(bar_full(i % kGzStages), (i / kGzStages) & 1) && clock64() - t0 < kGzWaitCycles) {
                }
            }
        }
    } else if (warp == 9) {
        // ---------------- MMA issuer
        if (lane == 0) {
            constexpr uint32_t idesc = gz_idesc();
            const uint32_t bop = sbase + GI::OFF_BOP;
            int issued = 0;
            for (int i = 0; i < my_tiles; i++) {
                const int d = i & 1;   // accumulator set and B operand buffer of this tile
                if (i >= 2 && !gz_wait(bar_dempty(d), ((i >> 1) - 1) & 1, abort, err, 2)) break;
                if (!gz_wait(bar_bready(d), (i >> 1) & 1, abort, err, 3)) break;
                gz_fence_after();
#pragma unroll
                for (int b = 0; b < NB; b++) {
                    const uint32_t dmain = tmem + GI::D_COL0 + (uint32_t)(((NB * d + b) * 2) * kGzRows);
                    const uint32_t dcorr = dmain + kGzRows;
                    const uint32_t a_hi = tmem + GI::A_COL0 + (uint32_t)((2 * b) * 64);
                    const uint32_t a_lo = a_hi + 64;
                    const uint32_t b_hi = bop + (uint32_t)(d * GI::BOP_BYTES + (2 * b) * GI::OP_BYTES);
                    const uint32_t b_lo = b_hi + GI::OP_BYTES;
#pragma unroll
                    for (int s = 0; s < kGzK / 16; s++) {
                        const uint32_t koff = (uint32_t)((s >> 2) * (kGzRows * 128) + (s & 3) * 32);
                        gz_mma_ts(dmain, a_hi + 8 * s, gz_desc(b_hi + koff), idesc, s > 0 ? 1u : 0u);
                        gz_mma_ts(dcorr, a_lo + 8 * s, gz_desc(b_hi + koff), idesc, s > 0 ? 1u : 0u);
                        gz_mma_ts(dcorr, a_hi + 8 * s, gz_desc(b_lo + koff), idesc, 1u);
                    }
                }
                gz_commit(bar_bfree(d));
                gz_commit(bar_dfull(d));
                issued = i + 1;
            }
            // drain: the last MMAs have completed before the tensor memory is freed
            if (issued > 0) {
                const int i = issued - 1;
                const long long t0 = clock64();
                while (!gz_try_wait(bar_dfull(i & 1), (i >> 1) & 1) && clock64() - t0 < kGzWaitCycles) {
                }
            }
        }
    } else if (warp < 4) {
        // ---------------- converters: kGzRows / 4 rows per warp per tile
        for (int i = 0; i < my_tiles; i++) {
            const int s = i % kGzStages;
            unsigned char *bop = sm + GI::OFF_BOP + (i & 1) * GI::BOP_BYTES;
            if (!gz_wait(bar_full(s), (i / kGzStages) & 1, abort, err, 4)) break;
            if (i >= 2 && !gz_wait(bar_bfree(i & 1), ((i >> 1) - 1) & 1, abort, err, 5)) break;
            const unsigned char *stg = sm + GI::OFF_STAGE + s * GI::STAGE_BYTES;
            float *sb = scale_back + (i & 3) * kGzRows;
            for (int rr = 0; rr < kGzRows / 4; rr++) {
                const int r = warp + 4 * rr;
                // lane l: elements 4l..4l+3 of the row's first 128 and (N = 256) second 128
                const int j = lane & 7;
                const float4 v1 = *reinterpret_cast<const float4 *>(stg + (lane >> 3) * (kGzRows * 128) + r * 128 +
                                                                    ((j ^ (r & 7)) << 4));
                float a[4] = {v1.x, v1.y, v1.z, v1.w};
                float b[4] = {0.f, 0.f, 0.f, 0.f};
                if constexpr (NB == 2) {
                    const float4 v2 = *reinterpret_cast<const float4 *>(stg + (4 + (lane >> 3)) * (kGzRows * 128) +
                                                                        r * 128 + ((j ^ (r & 7)) << 4));
                    if constexpr (FWD) {
                        // mirror x_{255-n} of n = 4l + t sits in lane 31 - l at element 3 - t
                        float w[4];
                        w[0] = __shfl_xor_sync(0xffffffffu, v2.x, 31);
                        w[1] = __shfl_xor_sync(0xffffffffu, v2.y, 31);
                        w[2] = __shfl_xor_sync(0xffffffffu, v2.z, 31);
                        w[3] = __shfl_xor_sync(0xffffffffu, v2.w, 31);
#pragma unroll
                        for (int t = 0; t < 4; t++) {
                            const float x = a[t], y = w[3 - t];
                            a[t] = x + y;   // e_{4l+t}
                            b[t] = x - y;   // o_{4l+t}
                        }
                    } else {
                        // p (even samples) and q (odd samples) at j = 2l, 2l+1 (first half)
                        // and 64 + 2l, 65 + 2l (second half)
                        const float p0 = v1.x, q0 = v1.y, p1 = v1.z, q1 = v1.w;
                        a[0] = p0; a[1] = p1; a[2] = v2.x; a[3] = v2.z;
                        b[0] = q0; b[1] = q1; b[2] = v2.y; b[3] = v2.w;
                    }
                }
                float m = 0.f;
#pragma unroll
                for (int t = 0; t < 4; t++) m = fmaxf(m, fmaxf(fabsf(a[t]), fabsf(b[t])));
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
                float sc, back;
                gz_row_scale(m, sc, back);
                if (lane == 0) sb[r] = back;
                uint32_t h0, l0, h1, l1;
                // block 0 (e, p, or the whole row)
                gz_split2(a[0] * sc, a[1] * sc, h0, l0);
                gz_split2(a[2] * sc, a[3] * sc, h1, l1);
                if (NB == 2 && !FWD) {
                    // K indices 2l, 2l+1 and 64 + 2l, 65 + 2l
                    *reinterpret_cast<uint32_t *>(bop + 0 * GI::OP_BYTES + gz_bop_off(r, 2 * lane)) = h0;
                    *reinterpret_cast<uint32_t *>(bop + 1 * GI::OP_BYTES + gz_bop_off(r, 2 * lane)) = l0;
                    *reinterpret_cast<uint32_t *>(bop + 0 * GI::OP_BYTES + gz_bop_off(r, 64 + 2 * lane)) = h1;
                    *reinterpret_cast<uint32_t *>(bop + 1 * GI::OP_BYTES + gz_bop_off(r, 64 + 2 * lane)) = l1;
                } else {
                    // K indices 4l .. 4l+3
                    *reinterpret_cast<uint2 *>(bop + 0 * GI::OP_BYTES + gz_bop_off(r, 4 * lane)) = make_uint2(h0, h1);
                    *reinterpret_cast<uint2 *>(bop + 1 * GI::OP_BYTES + gz_bop_off(r, 4 * lane)) = make_uint2(l0, l1);
                }
                if constexpr (NB == 2) {
                    gz_split2(b[0] * sc, b[1] * sc, h0, l0);
                    gz_split2(b[2] * sc, b[3] * sc, h1, l1);
                    if constexpr (!FWD) {
                        *reinterpret_cast<uint32_t *>(bop + 2 * GI::OP_BYTES + gz_bop_off(r, 2 * lane)) = h0;
                        *reinterpret_cast<uint32_t *>(bop + 3 * GI::OP_BYTES + gz_bop_off(r, 2 * lane)) = l0;
                        *reinterpret_cast<uint32_t *>(bop + 2 * GI::OP_BYTES + gz_bop_off(r, 64 + 2 * lane)) = h1;
                        *reinterpret_cast<uint32_t *>(bop + 3 * GI::OP_BYTES + gz_bop_off(r, 64 + 2 * lane)) = l1;
                    } else {
                        *reinterpret_cast<uint2 *>(bop + 2 * GI::OP_BYTES + gz_bop_off(r, 4 * lane)) = make_uint2(h0, h1);
                        *reinterpret_cast<uint2 *>(bop + 3 * GI::OP_BYTES + gz_bop_off(r, 4 * lane)) = make_uint2(l0, l1);
                    }
                }
            }
            // staging buffer consumed; operand written (visible to the tensor core's proxy)
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) {
                gz_arrive(bar_empty(s));
                gz_arrive(bar_bready(i & 1));
            }
        }
    } else {
        // ---------------- epilogue (warps 4-7: lane quarter q of the accumulators)
        const int q = warp & 3;
        const int kk = q * 32 + lane;   // output index within a block
        for (int i = 0; i < my_tiles; i++) {
            const int d = i & 1;
            if (!gz_wait(bar_dfull(d), (i >> 1) & 1, abort, err, 6)) break;
            gz_fence_after();
            const int row0 = ((int)blockIdx.x + i * (int)gridDim.x) * kGzRows;
            const float *sb = scale_back + (i & 3) * kGzRows;
            // block b's main and correction accumulators at dbase + 2 b kGzRows (+ kGzRows)
            const uint32_t dbase = tmem + ((uint32_t)(q * 32) << 16) + GI::D_COL0 + (uint32_t)(NB * d * 2 * kGzRows);
#pragma unroll 1
            for (int cc = 0; cc < kGzRows / 16; cc++) {
                uint32_t m0[16], c0[16], m1[16], c1[16];
                gz_tmem_ld16(dbase + cc * 16, m0);
                gz_tmem_ld16(dbase + kGzRows + cc * 16, c0);
                if constexpr (NB == 2) {
                    gz_tmem_ld16(dbase + 2 * kGzRows + cc * 16, m1);
                    gz_tmem_ld16(dbase + 3 * kGzRows + cc * 16, c1);
                }
                gz_wait_ld();
#pragma unroll
                for (int jj = 0; jj < 16; jj++) {
                    const int r = cc * 16 + jj;
                    if (row0 + r >= rows) break;
                    const float f = sb[r];
                    float *orow = out + (size_t)(row0 + r) * N;
                    const float u = (__uint_as_float(m0[jj]) + __uint_as_float(c0[jj])) * f;
                    if constexpr (NB == 1) {
                        orow[kk] = u;
                    } else {
                        const float v = (__uint_as_float(m1[jj]) + __uint_as_float(c1[jj])) * f;
                        if constexpr (FWD) {
                            *reinterpret_cast<float2 *>(orow + 2 * kk) = make_float2(u, v);
                        } else {
                            orow[kk] = u + v;
                            orow[N - 1 - kk] = u - v;
                        }
                    }
                }
            }
            gz_fence_before();
            __syncwarp();
            if (lane == 0) gz_arrive(bar_dempty(d));
        }
    }

    gz_fence_before();
    __syncthreads();
    gz_fence_after();
    if (warp == 9)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(GI::TMEM_COLS)
                     : "memory");
}

}  // namespace smadft
