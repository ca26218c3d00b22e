// gram_tc.cuh -- Gram matrix of the rows of an FP32 matrix on the tensor
// cores (tcgen05, three TF32 products per term), for ffdas_truncate_rank.
//
// The reference forms G = A A^T with one cuBLAS GEMM in FP32
// (src/truncate_rank/truncate_rank_impl.cuh:64-90, 451-480).  Here A is p x q,
// p <= 256, each row contiguous (K-major), and every CTA (one per SM) sums the
// columns [z * kchunk, (z + 1) * kchunk) into a p x p FP32 partial, stored
// column-major (entry (i, j) at j * p + i: a warp's 32 rows of one column are
// one 128-byte store); tr_gram_reduce_kernel adds the partials in double in a
// fixed order.
//
// Per CTA, a ring of S stages each holds 32 columns of all 128 * NB rows:
//  * warp 0 (one lane) loads a stage with one TMA box {32 columns, 128 * NB
//    rows} and the 128-byte swizzle, which is the K-major layout the MMA
//    reads (8-row groups 1024 bytes apart); rows past p read as zeros.  A
//    stage is p row segments of 128 bytes, each in its own DRAM page, so the
//    same lane also prefetches the boxes kPrefetch chunks ahead into L2: the
//    stage loads then wait on L2, not on DRAM;
//  * warps 2-9 split each element a into hi = tf32(a), written in place, and
//    lo = tf32(a - hi), written to the stage's second buffer at the same
//    offset (the split is elementwise, so the swizzle is kept), then make the
//    writes visible to the tensor core's proxy and arrive on the stage;
//  * warp 1 (one lane) issues, per 8-column step, tcgen05.mma kind::tf32
//        D += hi hi^T + hi lo^T + lo hi^T
//    with FP32 accumulators in tensor memory (the dropped lo lo^T term is
//    below 2^-22 of |a|^2, FP32 rounding of the products is exact: 11-bit
//    significands), then commits to the stage's empty barrier, which hands
//    the stage back to the loader.  Row block 0 (rows 0..127) against rows
//    0..n0-1 is one M = 128 product into columns 0..n0-1 of tensor memory;
//    with NB = 2, row block 1 against rows 128..128+n1-1 a second one into
//    columns 256..; the lower-left block, which the symmetric reduce never
//    reads, is not formed;
//  * after the last stage warps 2-9 read the accumulators back (warp w reads
//    tensor-memory lanes 32 (w % 4) .. +31, one row of D per thread, and
//    every other 16-column block) and store rows and columns below p.
// Every wait is bounded (about two seconds of clock): on expiry the CTA
// records FFDAS device status 1, stops issuing, waits (bounded) for its own
// copies and products in flight, releases its tensor memory and returns.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace ffdas {

// the driver's tensor-map encoder, or null (das_staged.cu)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

namespace gram_tc {

constexpr int kChunk = 32;           // columns per stage: one 128-byte row of FP32
constexpr int kThreads = 320;        // warp 0 loads, warp 1 issues products, warps 2-9 split and store
constexpr int kSplitters = 256;      // threads of warps 2-9: two per SM sub-partition, so that one
                                     // hides the other's shared-memory latency
constexpr int kRowBytes = kChunk * 4;
constexpr long long kWaitCycles = 4000000000LL;   // ~2 s at 2 GHz
constexpr int kStatusTimeout = 1;
constexpr uint32_t kBlock1Col = 256;             // tensor-memory column of row block 1's accumulator
constexpr int kPrefetch = 8;                     // chunks prefetched into L2 ahead of the stage loads

template <int NB> constexpr int stages() { return NB == 1 ? 6 : 3; }
template <int NB> constexpr uint32_t stage_bytes() { return (uint32_t)(128 * NB * kRowBytes); }
template <int NB> constexpr uint32_t tmem_cols() { return NB == 1 ? 128u : 512u; }
// operand buffers (hi and lo per stage), barriers, the tensor-memory address,
// the abort flag, and 1024 bytes to align the buffers to the swizzle atom
template <int NB> constexpr size_t smem_bytes() {
    return 1024 + 2 * (size_t)stages<NB>() * stage_bytes<NB>() + (3 * stages<NB>() + 1) * 8 + 16;
}

struct params {
    int p;              // rows of A, 1..128*NB
    int64_t q;          // columns of A
    int64_t kchunk;     // columns per CTA, a multiple of kChunk
    int n0, n1;         // product widths (multiples of 16): rows 0..n0-1 against block 0, 128..128+n1-1 against block 1
    float *part;        // gridDim.x partials of p x p, column-major
    int *status;        // device status word
};

__device__ __forceinline__ uint32_t su32(const void *p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void bar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void bar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void bar_expect(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_test(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}
// Waits for the phase of `parity`; false when the CTA aborted or the budget
// ran out (then the CTA aborts and the status word records the timeout).
__device__ __forceinline__ bool wait(uint32_t bar, uint32_t parity, volatile int *abort, int *status) {
    if (*abort) return false;
    const long long t0 = clock64();
    while (!bar_test(bar, parity)) {
        if (*abort) return false;
        if (clock64() - t0 > kWaitCycles) {
            *abort = 1;
            atomicExch(status, kStatusTimeout);
            return false;
        }
        __nanosleep(32);
    }
    return true;
}
// The same without the abort test: for work this thread itself put in flight.
__device__ __forceinline__ void settle(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!bar_test(bar, parity) && clock64() - t0 < kWaitCycles) __nanosleep(64);
}

__device__ __forceinline__ void tma_prefetch(const CUtensorMap *map, int x, int y) {
    asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];"
                 ::"l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y) : "memory");
}
__device__ __forceinline__ void tma_load(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar) : "memory");
}

// Shared-memory operand descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (stride byte offset), descriptor version 1; the leading
// byte offset is not used by swizzled K-major layouts.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t tf32_idesc(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void mma_tf32(uint32_t d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n"
        ::"r"(d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}
// The barrier receives one arrival when every product this thread issued
// before it has completed.
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Nearest TF32 value, ties away from zero: add half of the 13 dropped
// significand bits to the magnitude and clear them (integer ops at full rate;
// a carry into the exponent gives the next binade, infinities stay).
__device__ __forceinline__ float round_tf32(float a) {
    return __uint_as_float((__float_as_uint(a) + 0x1000u) & 0xFFFFE000u);
}
// a = hi + lo + O(2^-22 |a|), both parts TF32 values
__device__ __forceinline__ void split_tf32(float a, float &hi, float &lo) {
    hi = round_tf32(a);
    lo = round_tf32(a - hi);
}

// Rows r0..r0+127 of D (one per thread, warp quarter w % 4) from the
// accumulator at tensor-memory address `tmem`, 16-column blocks `half`,
// half + 2, ... of the n columns, into columns c0.. of the partial.
__device__ __forceinline__ void store_block(uint32_t tmem, int quarter, int half, int lane, int r0, int c0, int n,
                                            int p, bool zero, float *part) {
    const int i = r0 + quarter * 32 + lane;
    for (int c = 16 * half; c < n; c += 32) {
        uint32_t v[16];
        __syncwarp();    // the load below is warp-collective
        if (!zero) tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c, v);
        if (i < p) {
#pragma unroll
            for (int t = 0; t < 16; t++) {
                const int j = c0 + c + t;
                if (j < p) part[(int64_t)j * p + i] = zero ? 0.f : __uint_as_float(v[t]);
            }
        }
    }
}

template <int NB>
__global__ void __launch_bounds__(kThreads, 1) gram_tc_kernel(const __grid_constant__ CUtensorMap map, const params a) {
    constexpr int S = stages<NB>();
    constexpr uint32_t SB = stage_bytes<NB>();
    constexpr uint32_t kCols = tmem_cols<NB>();
    extern __shared__ unsigned char smem_raw[];
    const uint32_t pad = (1024u - (su32(smem_raw) & 1023u)) & 1023u;
    unsigned char *buf = smem_raw + pad;                   // hi[S] then lo[S], each SB bytes
    const uint32_t hi0 = su32(buf), lo0 = hi0 + S * SB;
    uint64_t *bars = reinterpret_cast<uint64_t *>(buf + 2 * S * SB);   // full[S], split[S], empty[S], done
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 3 * S + 1);
    int *abort_word = reinterpret_cast<int *>(tmem_slot + 1);
    volatile int *abort = abort_word;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t kbeg = (int64_t)blockIdx.x * a.kchunk;
    const int64_t kend = kbeg + a.kchunk < a.q ? kbeg + a.kchunk : a.q;
    const int nchunks = kbeg < kend ? (int)((kend - kbeg + kChunk - 1) / kChunk) : 0;
    const uint32_t done = su32(&bars[3 * S]);

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            bar_init(su32(&bars[s]), 1);
            bar_init(su32(&bars[S + s]), kSplitters / 32);
            bar_init(su32(&bars[2 * S + s]), 1);
        }
        bar_init(done, 1);
        *abort_word = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (warp >= 2) {
        // lo rows p.. are never written by the split: zero them once
        const int t = threadIdx.x - 64;
        for (int s = 0; s < S; s++) {
            float4 *l4 = reinterpret_cast<float4 *>(buf + (S + s) * SB);
            for (int e = a.p * (kRowBytes / 16) + t; e < (int)(SB / 16); e += kSplitters)
                l4[e] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            int issued = 0;
            for (int c = 0; c < nchunks && c < kPrefetch; c++)
                tma_prefetch(&map, (int)(kbeg + (int64_t)c * kChunk), 0);
            for (int c = 0; c < nchunks; c++) {
                const int s = c % S;
                if (c + kPrefetch < nchunks) tma_prefetch(&map, (int)(kbeg + (int64_t)(c + kPrefetch) * kChunk), 0);
                if (c >= S && !wait(su32(&bars[2 * S + s]), ((c / S) - 1) & 1, abort, a.status)) break;
                bar_expect(su32(&bars[s]), SB);
                tma_load(hi0 + s * SB, &map, (int)(kbeg + (int64_t)c * kChunk), 0, su32(&bars[s]));
                issued = c + 1;
            }
            // copies still in flight land before the CTA leaves
            for (int c = issued > S ? issued - S : 0; c < issued; c++) settle(su32(&bars[c % S]), (c / S) & 1);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t id0 = tf32_idesc(128, a.n0), id1 = tf32_idesc(128, a.n1);
            constexpr uint32_t kBlock1 = 128 * kRowBytes;   // byte offset of row 128
            for (int c = 0; c < nchunks; c++) {
                const int s = c % S;
                if (!wait(su32(&bars[S + s]), (c / S) & 1, abort, a.status)) break;
                fence_after_sync();
                const uint32_t hs = hi0 + s * SB, ls = lo0 + s * SB;
#pragma unroll
                for (int kk = 0; kk < kChunk / 8; kk++) {
                    const uint32_t acc = (c > 0 || kk > 0) ? 1u : 0u;
                    const uint32_t o = kk * 32;   // 8 TF32 columns
                    mma_tf32(tmem, sw128_desc(hs + o), sw128_desc(hs + o), id0, acc);
                    mma_tf32(tmem, sw128_desc(hs + o), sw128_desc(ls + o), id0, 1u);
                    mma_tf32(tmem, sw128_desc(ls + o), sw128_desc(hs + o), id0, 1u);
                    if (NB == 2) {
                        const uint32_t h1 = hs + kBlock1 + o, l1 = ls + kBlock1 + o;
                        mma_tf32(tmem + kBlock1Col, sw128_desc(h1), sw128_desc(h1), id1, acc);
                        mma_tf32(tmem + kBlock1Col, sw128_desc(h1), sw128_desc(l1), id1, 1u);
                        mma_tf32(tmem + kBlock1Col, sw128_desc(l1), sw128_desc(h1), id1, 1u);
                    }
                }
                mma_commit(su32(&bars[2 * S + s]));
            }
            mma_commit(done);   // fires when every product above has completed
        }
    } else {
        const int t = threadIdx.x - 64;
        const int n4 = a.p * (kRowBytes / 16);   // 16-byte groups of rows 0..p-1
        for (int c = 0; c < nchunks; c++) {
            const int s = c % S;
            if (!wait(su32(&bars[s]), (c / S) & 1, abort, a.status)) break;
            float4 *h4 = reinterpret_cast<float4 *>(buf + s * SB);
            float4 *l4 = reinterpret_cast<float4 *>(buf + (S + s) * SB);
#pragma unroll 4
            for (int e = t; e < n4; e += kSplitters) {
                const float4 v = h4[e];
                float4 h, l;
                split_tf32(v.x, h.x, l.x);
                split_tf32(v.y, h.y, l.y);
                split_tf32(v.z, h.z, l.z);
                split_tf32(v.w, h.w, l.w);
                h4[e] = h;
                l4[e] = l;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) bar_arrive(su32(&bars[S + s]));
        }
        if (wait(done, 0, abort, a.status)) {
            fence_after_sync();
            const int quarter = warp & 3, half = (warp - 2) >> 2;
            float *part = a.part + (int64_t)blockIdx.x * a.p * a.p;
            const bool zero = nchunks == 0;
            store_block(tmem, quarter, half, lane, 0, 0, a.n0, a.p, zero, part);
            if (NB == 2) store_block(tmem + kBlock1Col, quarter, half, lane, 128, 128, a.n1, a.p, zero, part);
        }
    }

    fence_before_sync();
    __syncthreads();
    if (warp == 1) {
        fence_after_sync();
        settle(done, 0);    // no product in flight when the columns are released
        __syncwarp();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
    }
}

}  // namespace gram_tc
}  // namespace ffdas
