// das_staged.cuh -- TMA-staged delay-and-sum kernels (sm_100a): forward and adjoint.
//
// A CTA owns a compact tile of 256 voxels (one per consumer thread) and one
// batch item.  A ninth warp is the producer: for every (channel, event) it
// bounds the sample window the whole tile can touch -- from the tile's
// bounding box and the tile's min/max delay for that event -- and stages that
// window of interpolation pairs into shared memory with one TMA tile load
// (cp.async.bulk.tensor, no multicast), running up to kStages chunks ahead of
// the consumers through a full/empty mbarrier ring.  Consumers then gather
// each tap from shared memory: per unit one packed FFMA for the delay, the
// floor/fraction split, one index clamp, one LDS and the taps/accumulates.
//
// Window slot layout: WB pairs written by TMA, followed by a permanent zero
// pair (zeroed once per CTA, never written by TMA).  A tap index is clamped to
// WB, so any index outside the window -- an out-of-record voxel, an excluded
// channel, an unused event slot -- reads exact zeros, reproducing the
// reference's validity rule (src/das/das_alg1_kernels.cuh:70-76).  TMA's
// out-of-bounds fill covers windows that straddle the ends of a pair row.
// A window wider than WB is flagged and its units read the pair rows in
// global memory instead.
//
// Every mbarrier wait is bounded by a clock budget; on expiry the CTA records
// status 1 in the handle's status word, stops issuing and computing, drains
// its own TMA copies (bounded) and exits without trapping.
//
// The adjoint kernel (das_staged_bwd_kernel) runs the same producer and
// window ring; its consumers recompute each tap and scatter the
// channel-data adjoint g*w*(1-t), g*w*t into a per-window shared gradient
// slot, which is flushed to global memory with one red.add per touched
// sample after the stage.
#pragma once

#include <cuda.h>
#include <type_traits>
#include "das_gather.cuh"

namespace ffdas {

constexpr int kStConsumers = 256;
constexpr int kStWarps = kStConsumers / 32;
constexpr int kStThreads = kStConsumers + 32;
constexpr int kStages = 4;
constexpr int kStWin = 32;                 // windows per stage (one per producer lane)
constexpr uint32_t kOvf = 0xFFFFFFFFu;     // meta value: window wider than a slot
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 2 GHz
constexpr int kStatusTimeout = 1;

struct staged_params {
    const void *P;
    int64_t npad;
    int C, S, N, n_events, B;
    int64_t V;
    int D0, D1, D2, T0, T1, T2, n0, n1;
    const float *srcpos;
    const float4 *srcdir;
    const float *dstpos, *offsets, *weights;
    float wavenum;             // complex data: phase rotation per sample of delay
    void *out;
    int64_t out_bstride;
    double beta_re, beta_im;   // beta_im: complex output only
    int beta_zero;
    int *status;
    int debug_drop_stage;  // test hook: the producer never fills the first stage
    int copy_async;        // 1: windows staged by per-lane cp.async copies instead of TMA tile loads
    int cchunk;            // forward: channels per blockIdx.z slice (0: all channels in one CTA)
    // das_sparse on the 512-voxel kernel: per-voxel lists (sparse_n, V) of events of x;
    // the passes run over x's events and each voxel takes the list entry naming the event
    const int *sparse_idx;
    int sparse_n;
    const int *gate;       // when set and *gate != 0 the kernel does nothing (a duplicate listed event)
    unsigned long long *units;   // when set, the kernel adds the units it evaluated (512-voxel kernel)
    // adjoint only
    const float *gout;
    int64_t gout_bstride;
    float *gx, *goff, *gw, *gdst, *gsrc;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}
__device__ __forceinline__ void tma_load_row(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar) : "memory");
}
// 16-byte global->shared async copy; src_bytes 0 writes 16 zero bytes.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
// The mbarrier receives one arrival when all of this thread's earlier
// cp.async copies have landed (its expected count includes that arrival).
__device__ __forceinline__ void cp_async_arrive(uint32_t bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// Box {WB pairs, 1 row, BT batch items} of the 3-D pair-row map.
__device__ __forceinline__ void tma_load_box3(uint32_t dst, const CUtensorMap *map, int x, int y, int z,
                                              uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar) : "memory");
}
__device__ __forceinline__ void consumer_sync() {
    asm volatile("bar.sync 1, %0;" ::"r"(kStConsumers) : "memory");
}

// try_wait with a suspend-time hint: the thread sleeps in the barrier until
// the phase completes or about `ns` nanoseconds pass, issuing nothing.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint32_t bar, uint32_t parity, uint32_t ns) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok) : "r"(bar), "r"(parity), "r"(ns) : "memory");
    return ok != 0;
}

// Bounded wait: false when the CTA aborted or the clock budget ran out.
// Waiting threads sleep in the barrier (suspend hint) rather than spin, so a
// warp that waits takes no issue slots from the warps that compute.
__device__ __forceinline__ bool bounded_wait(uint32_t bar, uint32_t parity, volatile int *abort, int *status) {
    if (*abort) return false;
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    for (;;) {
        if (mbar_try_wait_sleep(bar, parity, 20000u)) return true;
        if (*abort) return false;
        if (clock64() - t0 > kWaitCycles) {
            *abort = 1;
            atomicExch(status, kStatusTimeout);
            return false;
        }
    }
}

template <int K> struct staged_traits {
    using st = typename pair_traits<K>::storage;
    static constexpr int bytes = sizeof(st);
    static constexpr int align_pairs = bytes >= 16 ? 1 : 16 / bytes;   // TMA x coordinate granularity
    // TMA elements per pair: 16-byte (complex f32) pairs are two 8-byte elements
    static constexpr int tma_units = bytes == 16 ? 2 : 1;
};

template <int WB, int K> struct slot_geom {
    static constexpr int pair_bytes = staged_traits<K>::bytes;
    // WB pairs of data, then zeros up to the next 128-byte boundary (at least
    // 16 bytes): the pair at index WB is always zero.  Slots stay 128-B aligned.
    static constexpr int data_bytes = WB * pair_bytes;
    static constexpr int bytes = ((data_bytes + 16 + 127) / 128) * 128;
    static constexpr int stage_bytes = bytes * kStWin;
    static constexpr int ring_bytes = stage_bytes * kStages;
};

// Batch-tile window groups: the BT windows of one (channel, event) lie back to
// back ([BT][WB] pairs, one TMA box), groups 128-byte aligned; a stage holds
// kStWin / BT groups, so the ring is no larger than the single-item ring.
template <int WB, int K, int BT> struct group_geom {
    static constexpr int pair_bytes = staged_traits<K>::bytes;
    static constexpr int item_bytes = WB * pair_bytes;
    static constexpr int data_bytes = BT * item_bytes;
    static constexpr int bytes = ((data_bytes + 127) / 128) * 128;
    static constexpr int groups = kStWin / BT;
    static constexpr int stage_bytes = bytes * groups;
    static_assert(stage_bytes <= slot_geom<WB, K>::stage_bytes, "batch stage must fit the ring");
};

// Meta value of a window that holds no data: with it, no tap whose delay is
// finite and below 2^22 in magnitude -- and no larger or non-finite delay --
// yields an index inside the slot, so every tap reads the zero pair.
constexpr uint32_t kZeroWindow = kFloorMagicBits + 0x40000000u;

constexpr size_t kStMiscBytes = kStages * kStWin * 4      // meta
                                + kStages * 4              // overflow flags
                                + 2 * kStages * 8          // full / empty barriers
                                + 40 * 4                   // bounding box, per-event delay range
                                + 32 * 4                   // abort flag (+pad)
                                + kStWarps * 16 * 2 * 4    // reduction scratch
                                + kStages * kStWin * 2 * 16   // channel table (position, normal)
                                + kStages * kStWin * 2 * 16   // channel positions as pairs (x,x,y,y), (z,z,0,0)
                                + kStages * kStWin * 4        // window address biases (unclamped path)
                                + kStages * 4                 // stage modes
                                + 16 * 4;                     // channel box, pass flags

// Stage modes written by the 512-voxel kernel's producer (sm.mode):
//   kStageEmpty  no window of the stage holds data and none overflows: every
//                tap of the stage reads zeros, the consumers skip it;
//   kStageFast   every window of the stage is a real window or a zero window
//                whose whole tap range fits one slot, so a tap address is
//                bits(floor(tau) + 1.5 * 2^23) * pair_bytes + bias, no clamp.
enum : int { kStageEmpty = 1, kStageFast = 2 };
// Pass flags (sm.flags[2 + pass parity]), set by the consumers before a pass:
//   kPassSkip    every tap of the pass lies outside the record for every
//                voxel of the tile and every channel: the pass is skipped;
//   kPassFast    every delay of the pass is present, finite and below 2^20 in
//                magnitude, every voxel and channel position finite, the event
//                chunk full and no directivity test: stages marked kStageFast
//                may use the unclamped taps.
enum : int { kPassSkip = 1, kPassFast = 2 };
constexpr float kSaneRange = 1048576.0f;   // 2^20: tau, offsets and distances below it keep |rounding| < 1 sample

template <int WB, int K>
constexpr size_t staged_smem_bytes() {
    // ring, one zero slot (the target of zero windows on the unclamped path), misc
    return slot_geom<WB, K>::ring_bytes + slot_geom<WB, K>::bytes + kStMiscBytes + 128;
}

// The adjoints keep two copies of their fixed-point gradient bins (cx.par
// picks one per thread) to halve same-address atomics.  A copy spans `words`
// rounded up to whole bank rows plus half a row, so the copies' bins sit 16
// banks apart.
constexpr int bin_region_words(int words) { return (words + 31) / 32 * 32 + 16; }
constexpr int kBinCopies = 2;
// Words per window in the bins: samples kw .. kw + WB (WB + 1 bins) plus one
// bin that only out-of-window taps touch (always with zero), rounded up to
// whole 16-byte quads.
constexpr int bin_stride(int wb) { return (wb + 2 + 3) / 4 * 4; }

// Flush of one stage's fixed-point gradient bins: for every window, gx[kw + r]
// += (copy 0 + copy 1)[r] * finv for the nonzero bins r = 0..WB, and the bins
// are cleared.  WB / 4 lanes take a window, four bins each, with 128-bit
// shared loads and stores (a quarter warp moves 128 consecutive bytes: no bank
// conflicts); the window's first lane also takes bin WB.  row(win, kw) returns
// the gx row of the window (nullptr when it adds nothing) and its first sample.
template <int WB, int REGION, class RowFn>
__device__ __forceinline__ void flush_bins(int *bins0, int lane, int warp, float finv, RowFn &&row) {
    constexpr int GS4 = bin_stride(WB);
    constexpr int LPW = WB / 4;     // lanes per window
    constexpr int WPI = 32 / LPW;   // windows per warp and pass
    static_assert(WB % 4 == 0 && 32 % LPW == 0 && REGION % 4 == 0, "flush layout");
    const int sub = lane / LPW, q = lane % LPW;
    for (int w0 = warp * WPI; w0 < kStWin; w0 += kStWarps * WPI) {
        const int win = w0 + sub;
        int *b = bins0 + win * GS4 + 4 * q;
        const int4 u = *reinterpret_cast<const int4 *>(b);
        const int4 v = *reinterpret_cast<const int4 *>(b + REGION);
        *reinterpret_cast<int4 *>(b) = make_int4(0, 0, 0, 0);
        *reinterpret_cast<int4 *>(b + REGION) = make_int4(0, 0, 0, 0);
        int last = 0;
        if (q == 0) {
            int *e = bins0 + win * GS4 + WB;
            last = e[0] + e[REGION];
            e[0] = 0;
            e[REGION] = 0;
        }
        int kw;
        float *g = row(win, kw);
        if (g) {
            g += kw + 4 * q;
            const int s0 = u.x + v.x, s1 = u.y + v.y, s2 = u.z + v.z, s3 = u.w + v.w;
            if (s0) atomicAdd(g, (float)s0 * finv);
            if (s1) atomicAdd(g + 1, (float)s1 * finv);
            if (s2) atomicAdd(g + 2, (float)s2 * finv);
            if (s3) atomicAdd(g + 3, (float)s3 * finv);
            if (last) atomicAdd(g + WB, (float)last * finv);   // only q == 0 has one
        }
    }
}

// Adjoint extras: two copies of the fixed-point gradient slots [kStWin][WB + 2]
// int32, the per-stage channel-gradient scratch [kStWin / SC * 3][256] floats
// and a per-warp reduction scratch.
template <int WB, int K, int SC>
constexpr size_t staged_bwd_smem_bytes() {
    return staged_smem_bytes<WB, K>() + kBinCopies * bin_region_words(kStWin * bin_stride(WB)) * 4 + (kStWin / SC) * 3 * kStConsumers * 4 +
           kStWarps * 4;
}

// Shared-memory integer adds into the adjoints' gradient bins.  No "memory"
// clobber: the bins are only read after a consumer barrier (whose asm has
// one), and without it the compiler may hoist the staged-pair loads of later
// taps above these adds instead of waiting out each load in turn.
__device__ __forceinline__ void red_shared_add(uint32_t addr, int v) {
    asm volatile("red.shared.add.s32 [%0], %1;" ::"r"(addr), "r"(v));
}
// red.shared.add.s32 at addr + OFF bytes (OFF an immediate): no result
// register, and the offset folds into the instruction.
template <int OFF>
__device__ __forceinline__ void red_shared_add_at(uint32_t addr, int v) {
    asm volatile("red.shared.add.s32 [%0+%2], %1;" ::"r"(addr), "r"(v), "n"(OFF));
}

// Calls f(std::integral_constant<int, I>) for I = 0 .. N-1 (compile-time loop).
template <int I, int N, class F>
__device__ __forceinline__ void static_for(F &&f) {
    if constexpr (I < N) {
        f(std::integral_constant<int, I>{});
        static_for<I + 1, N>(f);
    }
}

// Fixed point for the adjoint's shared gradient slots: a value |v| <= 2^22
// rounds to the nearest integer as bits(v + 1.5 * 2^23) - bits(1.5 * 2^23).
constexpr float kFixRange = 4194000.0f;   // a little under 2^22
__device__ __forceinline__ int fix_round(float v) {
    return __float_as_int(v + kFloorMagic) - (int)kFloorMagicBits;
}
__device__ __forceinline__ int fix_round_fma(float a, float b) {   // round(a * b), one rounding
    return __float_as_int(__fmaf_rn(a, b, kFloorMagic)) - (int)kFloorMagicBits;
}
// round(a * b) + bits(1.5 * 2^23): differences of two such values need no
// bias correction
__device__ __forceinline__ int fix_bits_fma(float a, float b) {
    return __float_as_int(__fmaf_rn(a, b, kFloorMagic));
}

// Shared-memory layout shared by the forward and adjoint kernels.
template <int K, int WB>
struct staged_smem {
    using SG = slot_geom<WB, K>;
    unsigned char *ring;
    uint32_t *meta;        // [kStages][kStWin]
    int *ovf;              // [kStages]
    uint64_t *full, *empty;
    float *aabb;           // [6]
    float *ofs_lo, *ofs_hi;  // [16]
    volatile int *abort_flag;
    float *red;            // [warps][16][2]
    float4 *chan_pos, *chan_dir;  // [kStages][kStWin]
    float4 *chan_pair;            // [kStages][kStWin][2]: (x, x, y, y), (z, z, 0, 0)
    unsigned char *zslot;  // one slot of zeros (zeroed once per CTA, never written by TMA)
    uint32_t *bias;        // [kStages][kStWin]: tap address = bits(floor + magic) * pair_bytes + bias
    int *mode;             // [kStages]: kStageEmpty / kStageFast
    float *cbox;           // [6]: bounding box of this CTA's channels (min xyz, max xyz)
    int *flags;            // [4]: -, voxel and channel positions finite, pass flags (by pass parity)
    unsigned char *extra;  // adjoint scratch

    __device__ explicit staged_smem(unsigned char *raw) {
        ring = raw;
        zslot = ring + SG::ring_bytes;
        meta = reinterpret_cast<uint32_t *>(zslot + SG::bytes);
        ovf = reinterpret_cast<int *>(meta + kStages * kStWin);
        full = reinterpret_cast<uint64_t *>(ovf + kStages);
        empty = full + kStages;
        aabb = reinterpret_cast<float *>(empty + kStages);
        ofs_lo = aabb + 8;
        ofs_hi = ofs_lo + 16;
        abort_flag = reinterpret_cast<volatile int *>(ofs_hi + 16);
        red = const_cast<float *>(reinterpret_cast<volatile float *>(abort_flag + 32));
        chan_pos = reinterpret_cast<float4 *>(red + kStWarps * 32);
        chan_dir = chan_pos + kStages * kStWin;
        chan_pair = chan_dir + kStages * kStWin;
        bias = reinterpret_cast<uint32_t *>(chan_pair + kStages * kStWin * 2);
        mode = reinterpret_cast<int *>(bias + kStages * kStWin);
        cbox = reinterpret_cast<float *>(mode + kStages);
        flags = reinterpret_cast<int *>(cbox + 8);
        extra = reinterpret_cast<unsigned char *>(flags + 8);
    }
};

// Channel range of this CTA: the forward kernels may split the channels of a
// tile over blockIdx.z (small problems), each slice adding into the image.
__device__ __forceinline__ int chan_begin(const staged_params &p) { return p.cchunk ? (int)blockIdx.z * p.cchunk : 0; }
__device__ __forceinline__ int chan_end(const staged_params &p) {
    return p.cchunk ? min(p.C, ((int)blockIdx.z + 1) * p.cchunk) : p.C;
}

// Per-CTA state common to both kernels.
struct staged_ctx {
    int tid, warp, lane, b;
    bool producer, active;
    int64_t v;
    float vx, vy, vz;
    // checkerboard parity of the voxel in its tile (i0 + i1 + i2) & 1: the
    // adjoints' scatter copy, so that neighbouring voxels, which often hit one
    // sample, add into different copies of the gradient bins
    int par;
    // second voxel of the thread in 512-voxel tiles (tile index + 256)
    bool active2;
    int64_t v2;
    float vx2, vy2, vz2;
};

// Voxel of the thread, barrier init, zero pairs, tile bounding box.
// With spread, lane l of warp w takes the tile's voxel l * 8 + w, so a warp's
// voxels sit across the whole tile and rarely hit the same sample of a window
// (the adjoint's scatter then meets few same-address atomics).
// With vt == 2 the tile holds 512 voxels and each consumer thread also owns
// the voxel 256 places further in the tile's linear order.
template <int K, int WB>
__device__ __forceinline__ staged_ctx staged_setup(const staged_params &p, staged_smem<K, WB> &sm,
                                                   bool spread = false, int vt = 1) {
    using SG = slot_geom<WB, K>;
    staged_ctx cx;
    cx.tid = threadIdx.x;
    cx.warp = cx.tid >> 5;
    cx.lane = cx.tid & 31;
    cx.producer = (cx.warp == kStWarps);
    cx.b = blockIdx.y;
    cx.active = false;
    cx.v = 0;
    cx.vx = cx.vy = cx.vz = 0.f;
    cx.par = 0;
    cx.active2 = false;
    cx.v2 = 0;
    cx.vx2 = cx.vy2 = cx.vz2 = 0.f;
    const int tile = blockIdx.x;
    const int t0 = tile % p.n0, t1 = (tile / p.n0) % p.n1, t2 = tile / (p.n0 * p.n1);
    if (!cx.producer) {
        const int lt = spread ? (cx.lane * kStWarps + cx.warp) : cx.tid;
        const int i0 = lt % p.T0, i1 = (lt / p.T0) % p.T1, i2 = lt / (p.T0 * p.T1);
        const int g0 = t0 * p.T0 + i0, g1 = t1 * p.T1 + i1, g2 = t2 * p.T2 + i2;
        cx.par = (i0 + i1 + i2) & 1;
        cx.active = (g0 < p.D0 && g1 < p.D1 && g2 < p.D2);
        // 512-voxel tiles: a voxel past the grid stands in for the tile's
        // first voxel (always inside the grid) -- same position and delays,
        // weight 0, no output -- so every thread's taps stay inside the
        // windows the producer bounds from the tile's voxels
        const int64_t v_first = ((int64_t)(t2 * p.T2) * p.D1 + t1 * p.T1) * p.D0 + t0 * p.T0;
        if (cx.active || vt == 2) {
            cx.v = cx.active ? ((int64_t)g2 * p.D1 + g1) * p.D0 + g0 : v_first;
            cx.vx = __ldg(p.dstpos + 3 * cx.v);
            cx.vy = __ldg(p.dstpos + 3 * cx.v + 1);
            cx.vz = __ldg(p.dstpos + 3 * cx.v + 2);
        }
        if (vt == 2) {
            const int lt2 = lt + kStConsumers;
            const int j0 = lt2 % p.T0, j1 = (lt2 / p.T0) % p.T1, j2 = lt2 / (p.T0 * p.T1);
            const int h0 = t0 * p.T0 + j0, h1 = t1 * p.T1 + j1, h2 = t2 * p.T2 + j2;
            cx.active2 = (h0 < p.D0 && h1 < p.D1 && h2 < p.D2);
            cx.v2 = cx.active2 ? ((int64_t)h2 * p.D1 + h1) * p.D0 + h0 : v_first;
            cx.vx2 = __ldg(p.dstpos + 3 * cx.v2);
            cx.vy2 = __ldg(p.dstpos + 3 * cx.v2 + 1);
            cx.vz2 = __ldg(p.dstpos + 3 * cx.v2 + 2);
        }
    }
    if (cx.tid == 0) {
        for (int i = 0; i < kStages; i++) {
            // TMA: one arrival (expect_tx) by producer lane 0.  cp.async: lane 0's
            // arrival plus one completion arrival per producer lane.
            mbar_init(smem_u32(&sm.full[i]), p.copy_async ? 33u : 1u);
            mbar_init(smem_u32(&sm.empty[i]), kStWarps);
        }
        *sm.abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    {
        constexpr int zwords = (SG::bytes - SG::data_bytes) / 4;
        for (int i = cx.tid; i < kStages * kStWin * zwords; i += kStThreads) {
            const int slot = i / zwords, word = i - slot * zwords;
            reinterpret_cast<uint32_t *>(sm.ring + slot * SG::bytes + SG::data_bytes)[word] = 0u;
        }
        for (int i = cx.tid; i < SG::bytes / 4; i += kStThreads) reinterpret_cast<uint32_t *>(sm.zslot)[i] = 0u;
    }
    if (!cx.producer) {
        float mn[3] = {cx.active ? cx.vx : INFINITY, cx.active ? cx.vy : INFINITY, cx.active ? cx.vz : INFINITY};
        float mx[3] = {cx.active ? cx.vx : -INFINITY, cx.active ? cx.vy : -INFINITY, cx.active ? cx.vz : -INFINITY};
        if (cx.active2) {
            mn[0] = fminf(mn[0], cx.vx2); mn[1] = fminf(mn[1], cx.vy2); mn[2] = fminf(mn[2], cx.vz2);
            mx[0] = fmaxf(mx[0], cx.vx2); mx[1] = fmaxf(mx[1], cx.vy2); mx[2] = fmaxf(mx[2], cx.vz2);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
            for (int a = 0; a < 3; a++) {
                mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
                mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
            }
        }
        if (cx.lane == 0) {
#pragma unroll
            for (int a = 0; a < 3; a++) {
                sm.red[(cx.warp * 16 + a) * 2] = mn[a];
                sm.red[(cx.warp * 16 + a) * 2 + 1] = mx[a];
            }
        }
    }
    __syncthreads();
    if (cx.tid < 3) {
        float mn = INFINITY, mx = -INFINITY;
        for (int w = 0; w < kStWarps; w++) {
            mn = fminf(mn, sm.red[(w * 16 + cx.tid) * 2]);
            mx = fmaxf(mx, sm.red[(w * 16 + cx.tid) * 2 + 1]);
        }
        sm.aabb[cx.tid] = mn;
        sm.aabb[3 + cx.tid] = mx;
    }
    __syncthreads();
    return cx;
}

// Consumers: load this pass's delays and weights, reduce the tile's per-event
// delay range into ofs_lo / ofs_hi.  Ends with __syncthreads (all threads).
template <int K, int WB, int SC>
__device__ __forceinline__ void staged_pass_begin(const staged_params &p, staged_smem<K, WB> &sm,
                                                  const staged_ctx &cx, int e0, int sc, float (&ofs)[SC],
                                                  float (&w)[SC]) {
    if (!cx.producer) {
#pragma unroll
        for (int j = 0; j < SC; j++) {
            ofs[j] = 1e30f;
            w[j] = 0.f;
            if (cx.active && j < sc) {
                const int64_t idx = (int64_t)(e0 + j) * p.V + cx.v;
                ofs[j] = __ldg(p.offsets + idx);
                w[j] = __ldg(p.weights + idx);
            }
        }
#pragma unroll
        for (int j = 0; j < SC; j++) {
            const bool ok = cx.active && j < sc && isfinite(ofs[j]);
            float lo = ok ? ofs[j] : INFINITY, hi = ok ? ofs[j] : -INFINITY;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
            }
            if (cx.lane == 0) {
                sm.red[(cx.warp * 16 + j) * 2] = lo;
                sm.red[(cx.warp * 16 + j) * 2 + 1] = hi;
            }
        }
        consumer_sync();
        if (cx.tid < SC) {
            float lo = INFINITY, hi = -INFINITY;
            for (int ww = 0; ww < kStWarps; ww++) {
                lo = fminf(lo, sm.red[(ww * 16 + cx.tid) * 2]);
                hi = fmaxf(hi, sm.red[(ww * 16 + cx.tid) * 2 + 1]);
            }
            sm.ofs_lo[cx.tid] = lo;
            sm.ofs_hi[cx.tid] = hi;
        }
    }
    __syncthreads();
}

// Channel bounding box of this CTA's channel slice (sm.cbox), whether every
// voxel position of the tile and every channel position is finite
// (sm.flags[1]), and the number of voxels of the tile inside the grid (the
// return value, on every thread).  Called once after staged_setup.
template <int K, int WB>
__device__ __forceinline__ int staged_tile_bounds(const staged_params &p, staged_smem<K, WB> &sm,
                                                  const staged_ctx &cx) {
    bool fin = true;
    if (!cx.producer) {
        float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int c = chan_begin(p) + cx.tid; c < chan_end(p); c += kStConsumers) {
            const float q[3] = {__ldg(p.srcpos + 3 * c), __ldg(p.srcpos + 3 * c + 1), __ldg(p.srcpos + 3 * c + 2)};
#pragma unroll
            for (int a = 0; a < 3; a++) {
                fin &= isfinite(q[a]);
                mn[a] = fminf(mn[a], q[a]);
                mx[a] = fmaxf(mx[a], q[a]);
            }
        }
        fin &= isfinite(cx.vx) && isfinite(cx.vy) && isfinite(cx.vz) && isfinite(cx.vx2) && isfinite(cx.vy2) &&
               isfinite(cx.vz2);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
            for (int a = 0; a < 3; a++) {
                mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
                mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
            }
        }
        if (cx.lane == 0) {
#pragma unroll
            for (int a = 0; a < 3; a++) {
                sm.red[(cx.warp * 16 + a) * 2] = mn[a];
                sm.red[(cx.warp * 16 + a) * 2 + 1] = mx[a];
            }
        }
    }
    const int all_fin = __syncthreads_and(fin);
    const int n_active = __syncthreads_count(cx.active) + __syncthreads_count(cx.active2);
    if (cx.tid < 3) {
        float mn = INFINITY, mx = -INFINITY;
        for (int w = 0; w < kStWarps; w++) {
            mn = fminf(mn, sm.red[(w * 16 + cx.tid) * 2]);
            mx = fmaxf(mx, sm.red[(w * 16 + cx.tid) * 2 + 1]);
        }
        sm.cbox[cx.tid] = mn;
        sm.cbox[3 + cx.tid] = mx;
    }
    if (cx.tid == 0) sm.flags[1] = all_fin;
    __syncthreads();
    return n_active;
}

// Pass flags (kPassSkip, kPassFast) from the tile's per-event delay range, the
// tile's box and the channel box.  A tap's sample index is floor(tau) with
// tau = offset + |v - c|: the distance between the two boxes bounds |v - c|
// from below and above, so when every event of the pass has offset + the
// lower bound at or past N - 1 (or offset + the upper bound below 0), no tap
// of the pass lies inside the record and the pass adds exactly nothing.  The
// margin covers the FP32 rounding of tau, rsqrt included (< 1 sample below
// 2^20).
// `items`: the delays are the per-voxel list entries of the sparse item
// kernel, all present, so the fast path is open to them.
template <int K, int WB>
__device__ __forceinline__ int pass_flags(const staged_params &p, const staged_smem<K, WB> &sm, int sc, int SC,
                                          bool anybad, bool items = false) {
    float gmin = 0.f, gmax = 0.f;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float amin = sm.aabb[a], amax = sm.aabb[3 + a], cmin = sm.cbox[a], cmax = sm.cbox[3 + a];
        const float gap = fmaxf(fmaxf(cmin - amax, amin - cmax), 0.f);
        const float ext = fmaxf(fabsf(cmax - amin), fabsf(amax - cmin));
        gmin += gap * gap;
        gmax += ext * ext;
    }
    const float dmin = sqrtf(gmin), dmax = sqrtf(gmax);
    const bool boxes_ok = sm.flags[1] != 0 && dmax == dmax && dmax <= kSaneRange;
    bool skip = !anybad && boxes_ok;
    bool fast = !anybad && boxes_ok && (items || (sc == SC && !p.sparse_idx)) && !p.srcdir;
    for (int j = 0; j < sc; j++) {
        const float lo = sm.ofs_lo[j], hi = sm.ofs_hi[j];
        if (lo == INFINITY) {   // no delay of this event is present
            if (!items) fast = false;   // (item taps never name such an event)
            continue;
        }
        const float marg = 4.f + 1e-5f * (fabsf(lo) + fabsf(hi) + dmax);
        skip &= (lo + dmin - marg >= (float)(p.N - 1)) || (hi + dmax + marg < 0.f);
        fast &= fabsf(lo) <= kSaneRange && fabsf(hi) <= kSaneRange;
    }
    return (skip ? kPassSkip : 0) | (fast ? kPassFast : 0);
}

// staged_pass_begin for two voxels per thread: delays and weights as
// (voxel 1, voxel 2) pairs; the per-event delay range covers both.
template <int K, int WB, int SC>
__device__ __forceinline__ void staged_pass_begin2(const staged_params &p, staged_smem<K, WB> &sm,
                                                   const staged_ctx &cx, int e0, int sc, float2 (&ofs2)[SC],
                                                   float2 (&w2)[SC]) {
    if (!cx.producer) {
        // absent taps: delay 1e30 (its index clamps to the zero pair, its
        // fraction is 0) and weight 0, left out of the tile's delay range
        uint32_t present = 0u;   // bit 2j: voxel 1 has event e0 + j, bit 2j+1: voxel 2
#pragma unroll
        for (int j = 0; j < SC; j++) {
            ofs2[j] = make_float2(1e30f, 1e30f);
            w2[j] = make_float2(0.f, 0.f);
        }
        if (!p.sparse_idx) {
            // a voxel past the grid stands in for the tile's first voxel
            // (staged_setup): its delays, weight 0
#pragma unroll
            for (int j = 0; j < SC; j++) {
                if (j < sc) {
                    const int64_t base = (int64_t)(e0 + j) * p.V;
                    ofs2[j].x = __ldg(p.offsets + base + cx.v);
                    w2[j].x = cx.active ? __ldg(p.weights + base + cx.v) : 0.f;
                    ofs2[j].y = __ldg(p.offsets + base + cx.v2);
                    w2[j].y = cx.active2 ? __ldg(p.weights + base + cx.v2) : 0.f;
                    present |= 3u << (2 * j);
                }
            }
        } else {
            // das_sparse: each voxel's list entry that names event e0 + j
            // (zero-weight entries and events outside x add nothing, as in the
            // gather kernel; a doubly listed event never reaches this kernel)
            for (int i = 0; i < p.sparse_n; i++) {
                const int64_t base = (int64_t)i * p.V;
                if (cx.active) {
                    const uint32_t j = (uint32_t)(__ldg(p.sparse_idx + base + cx.v) - e0);
                    const float wv = __ldg(p.weights + base + cx.v);
                    if (j < (uint32_t)sc && wv != 0.f) {
                        const float ov = __ldg(p.offsets + base + cx.v);
#pragma unroll
                        for (int jj = 0; jj < SC; jj++)
                            if (j == (uint32_t)jj) { ofs2[jj].x = ov; w2[jj].x = wv; present |= 1u << (2 * jj); }
                    }
                }
                if (cx.active2) {
                    const uint32_t j = (uint32_t)(__ldg(p.sparse_idx + base + cx.v2) - e0);
                    const float wv = __ldg(p.weights + base + cx.v2);
                    if (j < (uint32_t)sc && wv != 0.f) {
                        const float ov = __ldg(p.offsets + base + cx.v2);
#pragma unroll
                        for (int jj = 0; jj < SC; jj++)
                            if (j == (uint32_t)jj) { ofs2[jj].y = ov; w2[jj].y = wv; present |= 2u << (2 * jj); }
                    }
                }
            }
        }
        bool bad = false;   // a present delay that is not finite (its tap is NaN)
#pragma unroll
        for (int j = 0; j < SC; j++) {
            const bool pa = (present >> (2 * j)) & 1u, pb = (present >> (2 * j)) & 2u;
            const bool oka = pa && isfinite(ofs2[j].x);
            const bool okb = pb && isfinite(ofs2[j].y);
            bad |= (pa && !oka) || (pb && !okb);
            float lo = fminf(oka ? ofs2[j].x : INFINITY, okb ? ofs2[j].y : INFINITY);
            float hi = fmaxf(oka ? ofs2[j].x : -INFINITY, okb ? ofs2[j].y : -INFINITY);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
            }
            if (cx.lane == 0) {
                sm.red[(cx.warp * 16 + j) * 2] = lo;
                sm.red[(cx.warp * 16 + j) * 2 + 1] = hi;
            }
        }
        bad = __any_sync(0xffffffffu, bad);
        if (cx.lane == 0) sm.red[(cx.warp * 16 + 15) * 2] = bad ? 1.f : 0.f;
        consumer_sync();
        if (cx.tid < SC) {
            float lo = INFINITY, hi = -INFINITY;
            for (int ww = 0; ww < kStWarps; ww++) {
                lo = fminf(lo, sm.red[(ww * 16 + cx.tid) * 2]);
                hi = fmaxf(hi, sm.red[(ww * 16 + cx.tid) * 2 + 1]);
            }
            sm.ofs_lo[cx.tid] = lo;
            sm.ofs_hi[cx.tid] = hi;
        }
        consumer_sync();
        if (cx.tid == 0) {
            bool anybad = false;
            for (int ww = 0; ww < kStWarps; ww++) anybad |= sm.red[(ww * 16 + 15) * 2] != 0.f;
            // two words by pass parity: a skipped pass has no barrier after
            // its threads read the flags, so the next pass writes the other word
            sm.flags[2 + ((e0 / SC) & 1)] = pass_flags(p, sm, sc, SC, anybad);
        }
    }
    __syncthreads();
}

// Producer warp: stage the windows of CC channels x SC events of one chunk.
// Publishes, with the full barrier's arrival, the window metadata, the
// overflow flag and the channel table of the stage.
//
// With FAST (the 512-voxel kernel) it also publishes each window's address
// bias and the stage's mode (kStageEmpty, kStageFast): a window whose whole
// tap range -- [lo + 1, hi - 1] at most, see below -- fits its slot gets
// bias = slot - pair_bytes * (bits(1.5 * 2^23) + k0); a zero window (no pair
// row data in range) whose tap range fits one slot points at the zero slot.
template <int K, int WB, int SC, bool FAST = false>
__device__ __forceinline__ void staged_produce(const staged_params &p, const CUtensorMap *tmap,
                                               staged_smem<K, WB> &sm, const staged_ctx &cx, int stage,
                                               uint32_t phase, int e0, int sc, int c0, bool &dead,
                                               uint32_t &issued_mask) {
    using SG = slot_geom<WB, K>;
    using st = typename pair_traits<K>::storage;
    const int cend = chan_end(p);
    const uint32_t full_bar = smem_u32(&sm.full[stage]);
    const uint32_t empty_bar = smem_u32(&sm.empty[stage]);
    unsigned char *stage_base = sm.ring + stage * SG::stage_bytes;
    const int lane = cx.lane;
    if (!dead && !bounded_wait(empty_bar, phase ^ 1u, sm.abort_flag, p.status)) dead = true;
    // Test hook: leave the very first stage unfilled (no copy, no arrival) so
    // the consumers' bounded waits must expire.
    const bool drop = p.debug_drop_stage && e0 == 0 && c0 == 0;
    if (drop) dead = true;
    bool issued = false, overflow = false, mappable = false;
    int k0w = 0;
    uint32_t bias = 0u;
    if (!dead) {
        const int cl = lane / SC, j = lane % SC;
        const int c = c0 + cl;
        const int bb = cx.b;   // batch item of the CTA
        uint32_t m = kZeroWindow;  // every tap index clamps to the zero pair
        float px = 0.f, py = 0.f, pz = 0.f;
        if (c < cend) {
            px = __ldg(p.srcpos + 3 * c);
            py = __ldg(p.srcpos + 3 * c + 1);
            pz = __ldg(p.srcpos + 3 * c + 2);
        }
        if (j == 0) {
            sm.chan_pos[stage * kStWin + cl] = make_float4(px, py, pz, 0.f);
            sm.chan_pair[(stage * kStWin + cl) * 2] = make_float4(px, px, py, py);
            sm.chan_pair[(stage * kStWin + cl) * 2 + 1] = make_float4(pz, pz, 0.f, 0.f);
            if (p.srcdir)
                sm.chan_dir[stage * kStWin + cl] = (c < cend) ? __ldg(p.srcdir + c) : make_float4(0, 0, 0, 2.f);
        }
        if (c < cend && j < sc) {
            const float *ab = sm.aabb;
            const float dx = fmaxf(fmaxf(ab[0] - px, px - ab[3]), 0.f);
            const float dy = fmaxf(fmaxf(ab[1] - py, py - ab[4]), 0.f);
            const float dz = fmaxf(fmaxf(ab[2] - pz, pz - ab[5]), 0.f);
            const float ex = fmaxf(fabsf(px - ab[0]), fabsf(px - ab[3]));
            const float ey = fmaxf(fabsf(py - ab[1]), fabsf(py - ab[4]));
            const float ez = fmaxf(fabsf(pz - ab[2]), fabsf(pz - ab[5]));
            const float rmin = sqrtf(dx * dx + dy * dy + dz * dz);
            const float rmax = sqrtf(ex * ex + ey * ey + ez * ez);
            const float lo = floorf(sm.ofs_lo[j] + rmin) - 2.f;
            const float hi = floorf(sm.ofs_hi[j] + rmax) + 2.f;
            // Every tap's floor(tau) lies in [lo + 1, hi - 1] when the delays,
            // distances and tau stay below 2^20 in magnitude (rounding < 1 sample).
            const bool sane = fabsf(lo) <= kSaneRange && fabsf(hi) <= kSaneRange && rmax <= kSaneRange;
            // a window that misses the pair row entirely stays a zero window
            if (lo == lo && hi == hi && hi >= 0.f && lo < (float)p.npad) {
                const int k0 = ((int)fmaxf(lo, -(float)WB)) & ~(staged_traits<K>::align_pairs - 1);
                const int k1 = (int)fminf(hi, (float)p.npad + WB);
                if (k1 - k0 + 1 <= WB) {
                    if (!p.copy_async) {
                        const int row = (bb * p.C + c) * p.S + (e0 + j);
                        tma_load_row(smem_u32(stage_base + lane * SG::bytes), tmap, k0 * staged_traits<K>::tma_units,
                                     row, full_bar);
                    }
                    k0w = k0;
                    m = kFloorMagicBits + (uint32_t)k0;
                    issued = true;
                    if constexpr (FAST) {
                        // the slot holds every tap only when neither end was clipped
                        mappable = sane && (float)k0 <= lo && hi <= (float)(k0 + WB - 1);
                        bias = smem_u32(stage_base + lane * SG::bytes) -
                               (uint32_t)sizeof(st) * (kFloorMagicBits + (uint32_t)k0);
                    }
                } else {
                    m = kOvf;
                    overflow = true;
                }
            } else if (FAST && sane && hi - lo + 1.f <= (float)WB) {
                // zero window: its taps read the zero slot
                mappable = true;
                bias = smem_u32(sm.zslot) - (uint32_t)sizeof(st) * (kFloorMagicBits + (uint32_t)(int)lo);
            }
        }
        sm.meta[stage * kStWin + lane] = m;
        if constexpr (FAST) sm.bias[stage * kStWin + lane] = bias;
    }
    const unsigned issued_ballot = __ballot_sync(0xffffffffu, issued);
    const unsigned ovf_ballot = __ballot_sync(0xffffffffu, overflow);
    const unsigned fast_ballot = __ballot_sync(0xffffffffu, mappable);
    if (p.copy_async && !drop) {
        // The warp copies the issued windows together, 16 bytes per lane per
        // copy: CPW lanes per window, 32 / CPW windows per round, coalesced
        // within each window.  Chunks outside the pair row are zero-filled
        // (the window start is 16-byte aligned and the row length a multiple
        // of 16 bytes, so a chunk lies wholly inside or outside the row).
        constexpr int PB = (int)sizeof(st);
        constexpr int CPW = WB * PB / 16;          // 16-byte chunks per window
        constexpr int WPR = 32 / CPW;              // windows per round
        constexpr int PPC = 16 / PB;               // pairs per chunk
        static_assert(CPW >= 1 && CPW <= 32 && 32 % CPW == 0, "window must split into lane chunks");
        const uint32_t stage_u32 = smem_u32(stage_base);
        const char *Pb = static_cast<const char *>(p.P);
        const int q = lane % CPW;
#pragma unroll 1
        for (int it = 0; it < CPW; it++) {
            const int w = it * WPR + lane / CPW;
            const int kw = __shfl_sync(0xffffffffu, k0w, w);
            if ((issued_ballot >> w) & 1u) {
                const int64_t row = ((int64_t)cx.b * p.C + c0 + w / SC) * p.S + e0 + w % SC;
                const int kp = kw + q * PPC;
                const bool in_row = kp >= 0 && (int64_t)kp < p.npad;
                const char *src = Pb + (row * p.npad + (in_row ? kp : 0)) * PB;
                cp_async16(stage_u32 + w * SG::bytes + q * 16, src, in_row ? 16u : 0u);
            }
        }
        cp_async_arrive(full_bar);
    }
    __syncwarp();
    if (lane == 0 && !drop) {
        sm.ovf[stage] = ovf_ballot != 0u;
        if constexpr (FAST)
            sm.mode[stage] = ((issued_ballot | ovf_ballot) == 0u ? kStageEmpty : 0) |
                             (fast_ballot == 0xffffffffu ? kStageFast : 0);
        // the producer's arrival also publishes meta / ovf / channel table (release)
        if (p.copy_async)
            mbar_arrive(full_bar);
        else
            mbar_arrive_expect_tx(full_bar, (uint32_t)__popc(issued_ballot) * (uint32_t)(WB * sizeof(st)));
    }
    if (!dead) issued_mask |= (1u << stage);
}

// Producer warp of the 512-voxel kernel: all stages of one pass.  Per stage
// the same windows, metadata, address biases and modes as staged_produce<FAST>,
// but the work that needs no ring slot is done before waiting for the slot:
// the channel positions are loaded one stage ahead, and each lane's window
// bounds (its event's delay range and the tile box are pass constants held in
// registers) are computed from them; only the stores, the copies and the
// arrival wait for the consumers to release the slot.  The distance bounds
// use x * rsqrt(x) (relative error a few 1e-7, far inside the windows'
// two-sample margins).
// The channel range is [cbeg, cend), the batch item cx.b.  With ITEMS (the
// sparse item kernel) a window no tap can read -- an event with no list
// entry in the tile, an event past the chunk, a channel past the slice, which
// that kernel's consumers skip -- does not hold the stage off the unclamped path.
template <int K, int WB, int SC, bool ITEMS = false>
__device__ __forceinline__ void staged_produce_pass2(const staged_params &p, const CUtensorMap *tmap,
                                                     staged_smem<K, WB> &sm, const staged_ctx &cx, int &stage,
                                                     uint32_t &phase, int e0, int sc, bool &dead,
                                                     uint32_t &issued_mask, int cbeg, int cend) {
    using SG = slot_geom<WB, K>;
    using st = typename pair_traits<K>::storage;
    constexpr int CC = kStWin / SC;
    constexpr uint32_t PB = (uint32_t)sizeof(st);
    const int lane = cx.lane, cl = lane / SC, j = lane % SC;
    const bool jv = j < sc;
    const float olo = sm.ofs_lo[j], ohi = sm.ofs_hi[j];
    const float ax0 = sm.aabb[0], ay0 = sm.aabb[1], az0 = sm.aabb[2];
    const float ax1 = sm.aabb[3], ay1 = sm.aabb[4], az1 = sm.aabb[5];
    const uint32_t zslot_u32 = smem_u32(sm.zslot);
    int c = cbeg + cl;
    float px = 0.f, py = 0.f, pz = 0.f;
    if (c < cend) {
        px = __ldg(p.srcpos + 3 * c);
        py = __ldg(p.srcpos + 3 * c + 1);
        pz = __ldg(p.srcpos + 3 * c + 2);
    }
    for (int c0 = cbeg; c0 < cend; c0 += CC) {
        // the next stage's channel position, in flight while this stage is built
        const int cn = c + CC;
        float qx = 0.f, qy = 0.f, qz = 0.f;
        if (cn < cend) {
            qx = __ldg(p.srcpos + 3 * cn);
            qy = __ldg(p.srcpos + 3 * cn + 1);
            qz = __ldg(p.srcpos + 3 * cn + 2);
        }
        // this lane's window of (channel c, event e0 + j): registers only
        uint32_t m = kZeroWindow;   // every tap index clamps to the zero pair
        bool issue = false, overflow = false, mappable = false, zero_map = false;
        int k0 = 0;
        if (ITEMS && !(c < cend && jv && olo != INFINITY)) mappable = true;   // never read
        if (c < cend && jv && !(ITEMS && olo == INFINITY)) {
            const float dx = fmaxf(fmaxf(ax0 - px, px - ax1), 0.f);
            const float dy = fmaxf(fmaxf(ay0 - py, py - ay1), 0.f);
            const float dz = fmaxf(fmaxf(az0 - pz, pz - az1), 0.f);
            const float ex = fmaxf(fabsf(px - ax0), fabsf(px - ax1));
            const float ey = fmaxf(fabsf(py - ay0), fabsf(py - ay1));
            const float ez = fmaxf(fabsf(pz - az0), fabsf(pz - az1));
            const float n2 = dx * dx + dy * dy + dz * dz, x2 = ex * ex + ey * ey + ez * ez;
            const float rmin = n2 > 0.f ? n2 * rsqrtf(n2) : 0.f;
            const float rmax = x2 > 0.f ? x2 * rsqrtf(x2) : 0.f;
            const float lo = floorf(olo + rmin) - 2.f;
            const float hi = floorf(ohi + rmax) + 2.f;
            // Every tap's floor(tau) lies in [lo + 1, hi - 1] when the delays,
            // distances and tau stay below 2^20 in magnitude (rounding < 1 sample).
            const bool sane = fabsf(lo) <= kSaneRange && fabsf(hi) <= kSaneRange && rmax <= kSaneRange;
            if (lo == lo && hi == hi && hi >= 0.f && lo < (float)p.npad) {   // the window meets the pair row
                k0 = ((int)fmaxf(lo, -(float)WB)) & ~(staged_traits<K>::align_pairs - 1);
                const int k1 = (int)fminf(hi, (float)p.npad + WB);
                if (k1 - k0 + 1 <= WB) {
                    issue = true;
                    m = kFloorMagicBits + (uint32_t)k0;
                    // the slot holds every tap only when neither end was clipped
                    mappable = sane && (float)k0 <= lo && hi <= (float)(k0 + WB - 1);
                } else {
                    m = kOvf;
                    overflow = true;
                }
            } else if (sane && hi - lo + 1.f <= (float)WB) {
                // zero window: its taps read the zero slot
                mappable = zero_map = true;
                k0 = (int)lo;
            }
        }

        const uint32_t full_bar = smem_u32(&sm.full[stage]);
        const uint32_t empty_bar = smem_u32(&sm.empty[stage]);
        unsigned char *stage_base = sm.ring + stage * SG::stage_bytes;
        if (!dead && !bounded_wait(empty_bar, phase ^ 1u, sm.abort_flag, p.status)) dead = true;
        // Test hook: leave the very first stage unfilled (no copy, no arrival) so
        // the consumers' bounded waits must expire.
        const bool drop = p.debug_drop_stage && e0 == 0 && c0 == 0;
        if (drop) dead = true;
        if (dead) issue = overflow = mappable = false;
        if (!dead) {
            if (j == 0) {
                sm.chan_pos[stage * kStWin + cl] = make_float4(px, py, pz, 0.f);
                sm.chan_pair[(stage * kStWin + cl) * 2] = make_float4(px, px, py, py);
                sm.chan_pair[(stage * kStWin + cl) * 2 + 1] = make_float4(pz, pz, 0.f, 0.f);
                if (p.srcdir)
                    sm.chan_dir[stage * kStWin + cl] = (c < cend) ? __ldg(p.srcdir + c) : make_float4(0, 0, 0, 2.f);
            }
            const uint32_t slot_u32 = smem_u32(stage_base + lane * SG::bytes);
            if (issue && !p.copy_async) {
                const int row = (cx.b * p.C + c) * p.S + (e0 + j);
                tma_load_row(slot_u32, tmap, k0 * staged_traits<K>::tma_units, row, full_bar);
            }
            sm.meta[stage * kStWin + lane] = m;
            sm.bias[stage * kStWin + lane] = (zero_map ? zslot_u32 : slot_u32) - PB * (kFloorMagicBits + (uint32_t)k0);
        }
        const unsigned issued_ballot = __ballot_sync(0xffffffffu, issue);
        const unsigned ovf_ballot = __ballot_sync(0xffffffffu, overflow);
        const unsigned fast_ballot = __ballot_sync(0xffffffffu, mappable);
        if (p.copy_async && !drop) {
            // The warp copies the issued windows together, 16 bytes per lane per
            // copy (as in staged_produce).
            constexpr int PBY = (int)sizeof(st);
            constexpr int CPW = WB * PBY / 16;
            constexpr int WPR = 32 / CPW;
            constexpr int PPC = 16 / PBY;
            static_assert(CPW >= 1 && CPW <= 32 && 32 % CPW == 0, "window must split into lane chunks");
            const uint32_t stage_u32 = smem_u32(stage_base);
            const char *Pb = static_cast<const char *>(p.P);
            const int q = lane % CPW;
#pragma unroll 1
            for (int it = 0; it < CPW; it++) {
                const int w = it * WPR + lane / CPW;
                const int kw = __shfl_sync(0xffffffffu, k0, w);
                if ((issued_ballot >> w) & 1u) {
                    const int64_t row = ((int64_t)cx.b * p.C + c0 + w / SC) * p.S + e0 + w % SC;
                    const int kp = kw + q * PPC;
                    const bool in_row = kp >= 0 && (int64_t)kp < p.npad;
                    const char *src = Pb + (row * p.npad + (in_row ? kp : 0)) * PBY;
                    cp_async16(stage_u32 + w * SG::bytes + q * 16, src, in_row ? 16u : 0u);
                }
            }
            cp_async_arrive(full_bar);
        }
        __syncwarp();
        if (lane == 0 && !drop) {
            sm.ovf[stage] = ovf_ballot != 0u;
            sm.mode[stage] = ((issued_ballot | ovf_ballot) == 0u ? kStageEmpty : 0) |
                             (fast_ballot == 0xffffffffu ? kStageFast : 0);
            // the producer's arrival also publishes meta / ovf / channel table (release)
            if (p.copy_async)
                mbar_arrive(full_bar);
            else
                mbar_arrive_expect_tx(full_bar, (uint32_t)__popc(issued_ballot) * (uint32_t)(WB * sizeof(st)));
        }
        if (!dead) issued_mask |= (1u << stage);
        if (++stage == kStages) {
            stage = 0;
            phase ^= 1u;
        }
        c = cn;
        px = qx; py = qy; pz = qz;
    }
}

// After an abort the producer waits (bounded, ignoring the abort flag) until
// every copy its CTA issued has landed, so no TMA write outlives the CTA.
template <int K, int WB>
__device__ __forceinline__ void staged_drain(staged_smem<K, WB> &sm, const staged_ctx &cx, int stage,
                                             uint32_t phase, uint32_t issued_mask) {
    cp_async_wait_all();   // no cp.async of this thread outlives the CTA (none in TMA mode)
    if (*sm.abort_flag && cx.lane == 0) {
        for (int i = 0; i < kStages; i++) {
            const int s = (stage + i) % kStages;
            if (!(issued_mask & (1u << s))) continue;
            const uint32_t par = (s < stage) ? phase : (phase ^ 1u);
            const long long t0 = clock64();
            while (!mbar_try_wait(smem_u32(&sm.full[s]), par) && clock64() - t0 < kWaitCycles) __nanosleep(64);
        }
    }
}

// Shared-memory loads on 32-bit shared-window addresses.  Volatile keeps them
// after the mbarrier wait that publishes the data (also volatile asm).
__device__ __forceinline__ uint32_t lds_u32(uint32_t a) {
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ float2 lds_f2(uint32_t a) {
    float2 v;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a));
    return v;
}
__device__ __forceinline__ uint4 lds_u4(uint32_t a) {
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
    return v;
}
__device__ __forceinline__ float4 lds_f4(uint32_t a) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
    return v;
}

// Interpolate one tap from the pair at shared address `a` (f32 result).
template <int K> __device__ __forceinline__ float tap_at(uint32_t a, float t);
template <> __device__ __forceinline__ float tap_at<ST_F32>(uint32_t a, float t) {
    const float2 p = lds_f2(a);
    return __fmaf_rn(t, p.y, p.x);
}
template <> __device__ __forceinline__ float tap_at<ST_F16>(uint32_t a, float t) {
    const uint32_t u = lds_u32(a);
    return pair_traits<ST_F16>::tap(*reinterpret_cast<const __half2 *>(&u), t);
}
template <> __device__ __forceinline__ float tap_at<ST_BF16>(uint32_t a, float t) {
    return pair_traits<ST_BF16>::tap(lds_u32(a), t);
}

// Sample x0 and slope d of the pair at shared address `a` (tap = x0 + t d).
template <int K> __device__ __forceinline__ void pair_x0_d(uint32_t a, float &x0, float &d);
template <> __device__ __forceinline__ void pair_x0_d<ST_F32>(uint32_t a, float &x0, float &d) {
    const float2 p = lds_f2(a);
    x0 = p.x;
    d = p.y;
}
template <> __device__ __forceinline__ void pair_x0_d<ST_F16>(uint32_t a, float &x0, float &d) {
    const uint32_t u = lds_u32(a);
    const float2 f = __half22float2(*reinterpret_cast<const __half2 *>(&u));
    x0 = f.x;
    d = f.y - f.x;
}
template <> __device__ __forceinline__ void pair_x0_d<ST_BF16>(uint32_t a, float &x0, float &d) {
    const uint32_t u = lds_u32(a);
    x0 = __uint_as_float(u << 16);
    d = __uint_as_float(u & 0xFFFF0000u) - x0;
}

// pair_x0_d on a shared-memory pointer (lets constant offsets fold).
template <int K> __device__ __forceinline__ void pair_x0_d_ptr(const typename pair_traits<K>::storage *q, float &x0,
                                                               float &d) {
    const typename pair_traits<K>::storage pr = *q;
    if constexpr (K == ST_F32) {
        x0 = pr.x;
        d = pr.y;
    } else {
        d = pair_traits<K>::slope(pr);
        x0 = pair_traits<K>::tap(pr, 0.f);
    }
}

// Interpolate one tap from a staged slot (f32 result).
template <int K>
__device__ __forceinline__ float staged_tap(const unsigned char *slot, uint32_t rel, float t) {
    using st = typename pair_traits<K>::storage;
    return pair_traits<K>::tap(*reinterpret_cast<const st *>(slot + rel * sizeof(st)), t);
}

// Read the SC window metadata words of channel cl of a stage.
template <int SC>
__device__ __forceinline__ void load_meta(const uint32_t *meta, int stage, int cl, uint32_t (&k0p)[SC]) {
    const uint32_t base = smem_u32(meta + stage * kStWin + cl * SC);
    if constexpr (SC >= 4) {
#pragma unroll
        for (int j = 0; j < SC; j += 4) {
            const uint4 q = lds_u4(base + 4 * j);
            k0p[j] = q.x; k0p[j + 1] = q.y; k0p[j + 2] = q.z; k0p[j + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int q = 0; q < SC; q++) k0p[q] = lds_u32(base + 4 * q);
    }
}

// ------------------------------------------------------------------ forward ---
template <int K, int SC, int WB>
__global__ void __launch_bounds__(kStThreads) das_staged_kernel(const staged_params p,
                                                                 const __grid_constant__ CUtensorMap tmap) {
    using st = typename pair_traits<K>::storage;
    using SG = slot_geom<WB, K>;
    constexpr int CC = kStWin / SC;  // channels per stage
    static_assert(kStWin % SC == 0, "SC must divide the stage");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    staged_smem<K, WB> sm(smem_raw);
    const staged_ctx cx = staged_setup<K, WB>(p, sm);

    const st *__restrict__ Pg = static_cast<const st *>(p.P);
    const uint32_t kmax_pair = (uint32_t)(p.npad - 1);
    float acc = 0.f;
    const int cbeg = chan_begin(p), cend = chan_end(p);   // this CTA's channel slice
    float2 acc2 = make_float2(0.f, 0.f);  // packed partial sums (even / odd event)
    int stage = 0;
    uint32_t phase = 0;
    bool dead = false;
    uint32_t issued_mask = 0;

    const uint32_t ring_u32 = smem_u32(sm.ring);
    const uint32_t chan_u32 = smem_u32(sm.chan_pos);

    for (int e0 = 0; e0 < p.n_events; e0 += SC) {
        const int sc = min(SC, p.n_events - e0);
        float ofs[SC], w[SC];
        staged_pass_begin<K, WB, SC>(p, sm, cx, e0, sc, ofs, w);
        // delays and weights as event pairs for the packed FP32 loop
        float2 ofs2[(SC + 1) / 2], w2[(SC + 1) / 2];
#pragma unroll
        for (int j = 0; j + 1 < SC; j += 2) {
            ofs2[j / 2] = make_float2(ofs[j], ofs[j + 1]);
            w2[j / 2] = make_float2(w[j], w[j + 1]);
        }

        for (int c0 = cbeg; c0 < cend; c0 += CC) {
            if (cx.producer) {
                staged_produce<K, WB, SC>(p, &tmap, sm, cx, stage, phase, e0, sc, c0, dead, issued_mask);
            } else {
                const uint32_t full_bar = smem_u32(&sm.full[stage]);
                const unsigned char *stage_base = sm.ring + stage * SG::stage_bytes;
                if (!dead && !bounded_wait(full_bar, phase, sm.abort_flag, p.status)) dead = true;
                if (!dead) {
                    const bool any_ovf = sm.ovf[stage] != 0;
                    const uint32_t stage_u32 = ring_u32 + stage * SG::stage_bytes;
                    // channels past C carry a zero window and a zero position: their
                    // taps read the zero pair, so the loop needs no bound check
#pragma unroll
                    for (int cl = 0; cl < CC; cl++) {
                        const int c = c0 + cl;
                        const float4 cp = lds_f4(chan_u32 + (stage * kStWin + cl) * 16);
                        recv_geom g = receive_geometry(cx.vx, cx.vy, cx.vz, cp.x, cp.y, cp.z);
                        if (p.srcdir)
                            apply_directivity(g, cx.vx, cx.vy, cx.vz, cp.x, cp.y, cp.z,
                                              sm.chan_dir[stage * kStWin + cl]);
                        uint32_t k0p[SC];
                        load_meta<SC>(sm.meta, stage, cl, k0p);
                        const uint32_t slots_u32 = stage_u32 + (cl * SC) * SG::bytes;
                        const unsigned char *slots = stage_base + (cl * SC) * SG::bytes;
                        if (!any_ovf) {
                            if constexpr (SC >= 2) {
                                // Two events per packed FP32 instruction: delay, floor
                                // split and fraction, then two taps and one packed
                                // accumulate into the two partial sums acc2.
                                const float2 rsq2 = make_float2(g.rsq, g.rsq);
                                const float2 rinv2 = make_float2(g.rinv, g.rinv);
                                const float2 magic2 = make_float2(kFloorMagic, kFloorMagic);
                                const float2 neg1 = make_float2(-1.f, -1.f);
#pragma unroll
                                for (int j = 0; j < SC; j += 2) {
                                    const float2 tau2 = __ffma2_rn(rsq2, rinv2, ofs2[j / 2]);
                                    const float2 mm2 = __fadd2_rd(tau2, magic2);
                                    const float2 nfl2 = __ffma2_rn(mm2, neg1, magic2);   // -(floor), exact
                                    const float2 t2 = __fadd2_rn(tau2, nfl2);
                                    const uint32_t ra = min(__float_as_uint(mm2.x) - k0p[j], (uint32_t)WB);
                                    const uint32_t rb = min(__float_as_uint(mm2.y) - k0p[j + 1], (uint32_t)WB);
                                    const float ta = tap_at<K>(slots_u32 + j * SG::bytes + ra * sizeof(st), t2.x);
                                    const float tb =
                                        tap_at<K>(slots_u32 + (j + 1) * SG::bytes + rb * sizeof(st), t2.y);
                                    acc2 = __ffma2_rn(w2[j / 2], make_float2(ta, tb), acc2);
                                }
                            } else {
#pragma unroll
                                for (int j = 0; j < SC; j++) {
                                    const float tau = __fmaf_rn(g.rsq, g.rinv, ofs[j]);
                                    const float mm = __fadd_rd(tau, kFloorMagic);
                                    const float t = tau - (mm - kFloorMagic);
                                    const uint32_t rel = min(__float_as_uint(mm) - k0p[j], (uint32_t)WB);
                                    acc = __fmaf_rn(w[j], tap_at<K>(slots_u32 + j * SG::bytes + rel * sizeof(st), t),
                                                    acc);
                                }
                            }
                        } else {
#pragma unroll
                            for (int j = 0; j < SC; j++) {
                                const float tau = __fmaf_rn(g.rsq, g.rinv, ofs[j]);
                                const tau_split ts = split_tau(tau);
                                st pr;
                                if (k0p[j] == kOvf) {
                                    const int64_t row = ((int64_t)cx.b * p.C + c) * p.S + (e0 + min(j, sc - 1));
                                    pr = Pg[row * p.npad + min(ts.k, kmax_pair)];
                                } else {
                                    const uint32_t rel = min(ts.k + kFloorMagicBits - k0p[j], (uint32_t)WB);
                                    pr = *reinterpret_cast<const st *>(slots + j * SG::bytes + rel * sizeof(st));
                                }
                                acc = __fmaf_rn(w[j], pair_traits<K>::tap(pr, ts.t), acc);
                            }
                        }
                    }
                }
                __syncwarp();
                if (cx.lane == 0) mbar_arrive(smem_u32(&sm.empty[stage]));
            }
            if (++stage == kStages) {
                stage = 0;
                phase ^= 1u;
            }
        }
        __syncthreads();
    }

    if (cx.producer) {
        staged_drain<K, WB>(sm, cx, stage, phase, issued_mask);
        return;
    }
    if (cx.active && !dead) {
        acc += acc2.x + acc2.y;
        float *o = static_cast<float *>(p.out) + (int64_t)cx.b * p.out_bstride + cx.v;
        if (p.cchunk) atomicAdd(o, acc);   // channel slices add into the prepared image
        else *o = p.beta_zero ? acc : __fmaf_rn((float)p.beta_re, *o, acc);
    }
}

// ------------------------------------------------- forward, 512-voxel tiles ---
// Same producer, ring and windows as das_staged_kernel, but each consumer
// thread owns two voxels of a 512-voxel tile (tile positions t and t + 256).
// A staged window then serves twice the units, which halves the producer's
// work, the channel-table and window-metadata loads and the barrier waits per
// unit.  The packed FP32 lanes carry the two voxels (not two events): the
// delay, floor split and fraction of one event for both voxels are one
// instruction each, and both taps read the same window.
//
// Work that adds nothing is not done:
//   * a pass (event chunk) whose taps all lie outside the record, for every
//     voxel of the tile and every channel, is skipped by producer and
//     consumers alike (pass_flags; deep tiles of a volume past the record);
//   * a stage whose windows all miss the pair rows (kStageEmpty) is skipped
//     by the consumers.
// On stages whose windows each hold their whole tap range (kStageFast, with
// the pass's kPassFast) a tap's shared address is one multiply-add of the
// floor bits and the window's bias, with no clamp; other stages clamp the
// index onto the slot's zero pair as before.  Every variant reads the same
// pair for every tap, so the image is bit-identical across them.
template <int K, int SC, int WB>
__global__ void __launch_bounds__(kStThreads, SC >= 8 ? 2 : 3) das_staged2_kernel(const staged_params p,
                                                                  const __grid_constant__ CUtensorMap tmap) {
    using st = typename pair_traits<K>::storage;
    using SG = slot_geom<WB, K>;
    constexpr int CC = kStWin / SC;  // channels per stage
    constexpr uint32_t PB = (uint32_t)sizeof(st);
    static_assert(kStWin % SC == 0, "SC must divide the stage");

    // a das_sparse call whose lists name an event twice runs on the gather
    // kernel instead (uniform for the whole grid, before any barrier or copy)
    if (p.gate && *(volatile const int *)p.gate) return;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    staged_smem<K, WB> sm(smem_raw);
    const staged_ctx cx = staged_setup<K, WB>(p, sm, false, 2);
    const int n_active = staged_tile_bounds<K, WB>(p, sm, cx);
    const int cbeg = chan_begin(p), cend = chan_end(p);   // this CTA's channel slice

    const st *__restrict__ Pg = static_cast<const st *>(p.P);
    const uint32_t kmax_pair = (uint32_t)(p.npad - 1);
    float2 acc2 = make_float2(0.f, 0.f);  // (voxel 1, voxel 2)
    int stage = 0;
    uint32_t phase = 0;
    bool dead = false;
    uint32_t issued_mask = 0;
    unsigned long long units = 0ull;      // units evaluated (thread 0 counts)

    const uint32_t ring_u32 = smem_u32(sm.ring);
    const uint32_t chan_u32 = smem_u32(sm.chan_pos);
    const float2 vx2 = make_float2(cx.vx, cx.vx2), vy2 = make_float2(cx.vy, cx.vy2), vz2 = make_float2(cx.vz, cx.vz2);
    const float2 nvx2 = make_float2(-cx.vx, -cx.vx2), nvy2 = make_float2(-cx.vy, -cx.vy2),
                 nvz2 = make_float2(-cx.vz, -cx.vz2);
    const uint32_t pair_u32 = smem_u32(sm.chan_pair);
    const float2 magic2 = make_float2(kFloorMagic, kFloorMagic);
    const float2 neg1 = make_float2(-1.f, -1.f);

    for (int e0 = 0; e0 < p.n_events; e0 += SC) {
        const int sc = min(SC, p.n_events - e0);
        float2 ofs2[SC], w2[SC];
        staged_pass_begin2<K, WB, SC>(p, sm, cx, e0, sc, ofs2, w2);
        const int pflags = *(volatile int *)&sm.flags[2 + ((e0 / SC) & 1)];
        if (pflags & kPassSkip) continue;   // uniform: the ring is left as it is
        const bool pass_fast = (pflags & kPassFast) != 0;

        if (cx.producer) {
            staged_produce_pass2<K, WB, SC>(p, &tmap, sm, cx, stage, phase, e0, sc, dead, issued_mask, cbeg, cend);
        } else {
        for (int c0 = cbeg; c0 < cend; c0 += CC) {
            {
                const uint32_t full_bar = smem_u32(&sm.full[stage]);
                if (!dead && !bounded_wait(full_bar, phase, sm.abort_flag, p.status)) dead = true;
                const int mode = dead ? kStageEmpty : *(volatile int *)&sm.mode[stage];
                if (!(mode & kStageEmpty)) {
                    if (cx.tid == 0) units += (unsigned long long)min(CC, cend - c0) * sc * n_active;
                    const bool any_ovf = sm.ovf[stage] != 0;
                    const uint32_t stage_u32 = ring_u32 + stage * SG::stage_bytes;
                    if (pass_fast && (mode & kStageFast)) {
                        // Every window holds its whole tap range: address =
                        // bits(floor + magic) * pair_bytes + bias, no clamp.
#pragma unroll
                        for (int cl = 0; cl < CC; cl++) {
                            const float4 qa = lds_f4(pair_u32 + (stage * kStWin + cl) * 32);
                            const float4 qb = lds_f4(pair_u32 + (stage * kStWin + cl) * 32 + 16);
                            const float2 dx = __fadd2_rn(make_float2(qa.x, qa.y), nvx2);
                            const float2 dy = __fadd2_rn(make_float2(qa.z, qa.w), nvy2);
                            const float2 dz = __fadd2_rn(make_float2(qb.x, qb.y), nvz2);
                            float2 r2 = __fmul2_rn(dx, dx);
                            r2 = __ffma2_rn(dy, dy, r2);
                            r2 = __ffma2_rn(dz, dz, r2);
                            const float2 rsq2 = make_float2(fmaxf(r2.x, 1e-7f), fmaxf(r2.y, 1e-7f));
                            const float2 rinv2 = make_float2(rsqrtf(rsq2.x), rsqrtf(rsq2.y));
                            uint32_t bias[SC];
                            load_meta<SC>(sm.bias, stage, cl, bias);
#pragma unroll
                            for (int j = 0; j < SC; j++) {
                                const float2 tau2 = __ffma2_rn(rsq2, rinv2, ofs2[j]);
                                const float2 mm2 = __fadd2_rd(tau2, magic2);
                                const float2 nfl2 = __ffma2_rn(mm2, neg1, magic2);   // -(floor), exact
                                const float2 t2 = __fadd2_rn(tau2, nfl2);
                                const float ta = tap_at<K>(__float_as_uint(mm2.x) * PB + bias[j], t2.x);
                                const float tb = tap_at<K>(__float_as_uint(mm2.y) * PB + bias[j], t2.y);
                                acc2 = __ffma2_rn(w2[j], make_float2(ta, tb), acc2);
                            }
                        }
                    } else if (!any_ovf && !p.srcdir) {
                        // No per-channel branch; tap indices are clamped onto the
                        // slot's zero pair.  The channel table's (x, x, y, y),
                        // (z, z, 0, 0) rows feed the packed geometry directly:
                        // d = c - v, the exact negative of v - c, so rsq is the
                        // same as receive_geometry's.  Channels past C carry a
                        // zero window: their taps read the zero pair.
#pragma unroll
                        for (int cl = 0; cl < CC; cl++) {
                            const float4 qa = lds_f4(pair_u32 + (stage * kStWin + cl) * 32);
                            const float4 qb = lds_f4(pair_u32 + (stage * kStWin + cl) * 32 + 16);
                            const float2 dx = __fadd2_rn(make_float2(qa.x, qa.y), nvx2);
                            const float2 dy = __fadd2_rn(make_float2(qa.z, qa.w), nvy2);
                            const float2 dz = __fadd2_rn(make_float2(qb.x, qb.y), nvz2);
                            float2 r2 = __fmul2_rn(dx, dx);
                            r2 = __ffma2_rn(dy, dy, r2);
                            r2 = __ffma2_rn(dz, dz, r2);
                            const float2 rsq2 = make_float2(fmaxf(r2.x, 1e-7f), fmaxf(r2.y, 1e-7f));
                            const float2 rinv2 = make_float2(rsqrtf(rsq2.x), rsqrtf(rsq2.y));
                            uint32_t k0p[SC];
                            load_meta<SC>(sm.meta, stage, cl, k0p);
                            const uint32_t slots_u32 = stage_u32 + (cl * SC) * SG::bytes;
#pragma unroll
                            for (int j = 0; j < SC; j++) {
                                const float2 tau2 = __ffma2_rn(rsq2, rinv2, ofs2[j]);
                                const float2 mm2 = __fadd2_rd(tau2, magic2);
                                const float2 nfl2 = __ffma2_rn(mm2, neg1, magic2);   // -(floor), exact
                                const float2 t2 = __fadd2_rn(tau2, nfl2);
                                const uint32_t ra = min(__float_as_uint(mm2.x) - k0p[j], (uint32_t)WB);
                                const uint32_t rb = min(__float_as_uint(mm2.y) - k0p[j], (uint32_t)WB);
                                const uint32_t slot = slots_u32 + j * SG::bytes;
                                const float ta = tap_at<K>(slot + ra * sizeof(st), t2.x);
                                const float tb = tap_at<K>(slot + rb * sizeof(st), t2.y);
                                acc2 = __ffma2_rn(w2[j], make_float2(ta, tb), acc2);
                            }
                        }
                    } else {
#pragma unroll 1
                    for (int cl = 0; cl < CC; cl++) {
                        const int c = c0 + cl;
                        const float4 cp = lds_f4(chan_u32 + (stage * kStWin + cl) * 16);
                        // receive geometry of both voxels, packed; the same operation
                        // sequence per lane as receive_geometry
                        const float2 cx2 = make_float2(-cp.x, -cp.x), cy2 = make_float2(-cp.y, -cp.y),
                                     cz2 = make_float2(-cp.z, -cp.z);
                        const float2 dx = __fadd2_rn(vx2, cx2), dy = __fadd2_rn(vy2, cy2), dz = __fadd2_rn(vz2, cz2);
                        float2 r2 = __fmul2_rn(dx, dx);
                        r2 = __ffma2_rn(dy, dy, r2);
                        r2 = __ffma2_rn(dz, dz, r2);
                        recv_geom ga, gb;
                        ga.rsq = fmaxf(r2.x, 1e-7f);
                        gb.rsq = fmaxf(r2.y, 1e-7f);
                        ga.rinv = rsqrtf(ga.rsq);
                        gb.rinv = rsqrtf(gb.rsq);
                        if (p.srcdir) {
                            const float4 dir = sm.chan_dir[stage * kStWin + cl];
                            apply_directivity(ga, cx.vx, cx.vy, cx.vz, cp.x, cp.y, cp.z, dir);
                            apply_directivity(gb, cx.vx2, cx.vy2, cx.vz2, cp.x, cp.y, cp.z, dir);
                        }
                        const float2 rsq2 = make_float2(ga.rsq, gb.rsq), rinv2 = make_float2(ga.rinv, gb.rinv);
                        uint32_t k0p[SC];
                        load_meta<SC>(sm.meta, stage, cl, k0p);
                        const uint32_t slots_u32 = stage_u32 + (cl * SC) * SG::bytes;
                        if (!any_ovf) {
#pragma unroll
                            for (int j = 0; j < SC; j++) {
                                const float2 tau2 = __ffma2_rn(rsq2, rinv2, ofs2[j]);
                                const float2 mm2 = __fadd2_rd(tau2, magic2);
                                const float2 nfl2 = __ffma2_rn(mm2, neg1, magic2);   // -(floor), exact
                                const float2 t2 = __fadd2_rn(tau2, nfl2);
                                const uint32_t ra = min(__float_as_uint(mm2.x) - k0p[j], (uint32_t)WB);
                                const uint32_t rb = min(__float_as_uint(mm2.y) - k0p[j], (uint32_t)WB);
                                const uint32_t slot = slots_u32 + j * SG::bytes;
                                const float ta = tap_at<K>(slot + ra * sizeof(st), t2.x);
                                const float tb = tap_at<K>(slot + rb * sizeof(st), t2.y);
                                acc2 = __ffma2_rn(w2[j], make_float2(ta, tb), acc2);
                            }
                        } else {
                            const unsigned char *slots = sm.ring + stage * SG::stage_bytes + (cl * SC) * SG::bytes;
#pragma unroll
                            for (int j = 0; j < SC; j++) {
                                float tv[2];
#pragma unroll
                                for (int h = 0; h < 2; h++) {
                                    const recv_geom &g = h ? gb : ga;
                                    const float tau = __fmaf_rn(g.rsq, g.rinv, h ? ofs2[j].y : ofs2[j].x);
                                    const tau_split ts = split_tau(tau);
                                    st pr;
                                    if (k0p[j] == kOvf) {
                                        const int64_t row = ((int64_t)cx.b * p.C + c) * p.S + (e0 + min(j, sc - 1));
                                        pr = Pg[row * p.npad + min(ts.k, kmax_pair)];
                                    } else {
                                        const uint32_t rel = min(ts.k + kFloorMagicBits - k0p[j], (uint32_t)WB);
                                        pr = *reinterpret_cast<const st *>(slots + j * SG::bytes + rel * sizeof(st));
                                    }
                                    tv[h] = pair_traits<K>::tap(pr, ts.t);
                                }
                                acc2 = __ffma2_rn(w2[j], make_float2(tv[0], tv[1]), acc2);
                            }
                        }
                    }
                    }
                }
                __syncwarp();
                if (cx.lane == 0) mbar_arrive(smem_u32(&sm.empty[stage]));
            }
            if (++stage == kStages) {
                stage = 0;
                phase ^= 1u;
            }
        }
        }
        __syncthreads();
    }

    if (cx.producer) {
        staged_drain<K, WB>(sm, cx, stage, phase, issued_mask);
        return;
    }
    if (dead) return;
    if (p.units && cx.tid == 0 && units) atomicAdd(p.units, units);
    float *o = static_cast<float *>(p.out) + (int64_t)cx.b * p.out_bstride;
    if (p.cchunk) {   // channel slices add into the prepared image
        if (cx.active) atomicAdd(o + cx.v, acc2.x);
        if (cx.active2) atomicAdd(o + cx.v2, acc2.y);
    } else {
        if (cx.active) o[cx.v] = p.beta_zero ? acc2.x : __fmaf_rn((float)p.beta_re, o[cx.v], acc2.x);
        if (cx.active2) o[cx.v2] = p.beta_zero ? acc2.y : __fmaf_rn((float)p.beta_re, o[cx.v2], acc2.y);
    }
}

// ------------------------------------------------- forward, batch tiles ---
// One CTA = one 256-voxel tile x BT batch items (frame ensembles, batched
// acquisitions).  The delays do not depend on the batch item, so the BT
// windows of one (channel, event) have the same bounds: the producer stages
// them with ONE 3-D TMA box {WB pairs, 1 row, BT items} (a stage holds
// kStWin / BT such groups, so copies per unit drop by BT), and per (voxel,
// channel, event) the consumers compute the delay, floor split, fraction and
// window index once for BT taps.  Groups are dense ([BT][WB] pairs, no zero
// pair between items): a tap outside its window (outside the record, an
// excluded channel, an unused slot) is redirected to a zeroed group instead.
template <int K, int WB, int SC, int BT>
__device__ __forceinline__ void staged_produce_batch(const staged_params &p, const CUtensorMap *tmap,
                                                     staged_smem<K, WB> &sm, const staged_ctx &cx, int stage,
                                                     uint32_t phase, int e0, int sc, int c0, bool &dead,
                                                     uint32_t &issued_mask) {
    using SG = slot_geom<WB, K>;
    using GG = group_geom<WB, K, BT>;
    const int cend = chan_end(p);
    const uint32_t full_bar = smem_u32(&sm.full[stage]);
    const uint32_t empty_bar = smem_u32(&sm.empty[stage]);
    const uint32_t stage_u32 = smem_u32(sm.ring + stage * SG::stage_bytes);
    const int lane = cx.lane;
    if (!dead && !bounded_wait(empty_bar, phase ^ 1u, sm.abort_flag, p.status)) dead = true;
    const bool drop = p.debug_drop_stage && e0 == 0 && c0 == 0;   // test hook, as in staged_produce
    if (drop) dead = true;
    bool issued = false, overflow = false;
    const bool own = lane < GG::groups;
    if (!dead && own) {
        const int cl = lane / SC, j = lane % SC;
        const int c = c0 + cl;
        uint32_t m = kZeroWindow;
        float px = 0.f, py = 0.f, pz = 0.f;
        if (c < cend) {
            px = __ldg(p.srcpos + 3 * c);
            py = __ldg(p.srcpos + 3 * c + 1);
            pz = __ldg(p.srcpos + 3 * c + 2);
        }
        if (j == 0) {
            sm.chan_pos[stage * kStWin + cl] = make_float4(px, py, pz, 0.f);
            if (p.srcdir)
                sm.chan_dir[stage * kStWin + cl] = (c < cend) ? __ldg(p.srcdir + c) : make_float4(0, 0, 0, 2.f);
        }
        if (c < cend && j < sc) {
            const float *ab = sm.aabb;
            const float dx = fmaxf(fmaxf(ab[0] - px, px - ab[3]), 0.f);
            const float dy = fmaxf(fmaxf(ab[1] - py, py - ab[4]), 0.f);
            const float dz = fmaxf(fmaxf(ab[2] - pz, pz - ab[5]), 0.f);
            const float ex = fmaxf(fabsf(px - ab[0]), fabsf(px - ab[3]));
            const float ey = fmaxf(fabsf(py - ab[1]), fabsf(py - ab[4]));
            const float ez = fmaxf(fabsf(pz - ab[2]), fabsf(pz - ab[5]));
            const float rmin = sqrtf(dx * dx + dy * dy + dz * dz);
            const float rmax = sqrtf(ex * ex + ey * ey + ez * ez);
            const float lo = floorf(sm.ofs_lo[j] + rmin) - 2.f;
            const float hi = floorf(sm.ofs_hi[j] + rmax) + 2.f;
            if (lo == lo && hi == hi && hi >= 0.f && lo < (float)p.npad) {
                const int k0 = ((int)fmaxf(lo, -(float)WB)) & ~(staged_traits<K>::align_pairs - 1);
                const int k1 = (int)fminf(hi, (float)p.npad + WB);
                if (k1 - k0 + 1 <= WB) {
                    tma_load_box3(stage_u32 + lane * GG::bytes, tmap, k0, c * p.S + e0 + j, cx.b * BT, full_bar);
                    m = kFloorMagicBits + (uint32_t)k0;
                    issued = true;
                } else {
                    m = kOvf;
                    overflow = true;
                }
            }
        }
        sm.meta[stage * kStWin + lane] = m;
    }
    const unsigned issued_ballot = __ballot_sync(0xffffffffu, issued);
    const unsigned ovf_ballot = __ballot_sync(0xffffffffu, overflow);
    __syncwarp();
    if (lane == 0 && !drop) {
        sm.ovf[stage] = ovf_ballot != 0u;
        mbar_arrive_expect_tx(full_bar, (uint32_t)__popc(issued_ballot) * (uint32_t)GG::data_bytes);
    }
    if (!dead) issued_mask |= (1u << stage);
}

template <int WB, int K, int BT>
constexpr size_t staged_batch_smem_bytes() {
    return staged_smem_bytes<WB, K>() + group_geom<WB, K, BT>::data_bytes;   // + the zero group
}

template <int K, int SC, int WB, int BT>
__global__ void __launch_bounds__(kStThreads) das_staged_batch_kernel(const staged_params p,
                                                                       const __grid_constant__ CUtensorMap tmap) {
    using st = typename pair_traits<K>::storage;
    using SG = slot_geom<WB, K>;
    using GG = group_geom<WB, K, BT>;
    constexpr int CC = GG::groups / SC;  // channels per stage
    static_assert(SC % 2 == 0 && GG::groups % SC == 0, "SC * BT must divide the stage");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    staged_smem<K, WB> sm(smem_raw);
    unsigned char *zero_group = sm.extra;
    for (int i = threadIdx.x; i < GG::data_bytes / 4; i += kStThreads) reinterpret_cast<uint32_t *>(zero_group)[i] = 0u;
    const staged_ctx cx = staged_setup<K, WB>(p, sm);   // ends with __syncthreads

    const st *__restrict__ Pg = static_cast<const st *>(p.P);
    const uint32_t kmax_pair = (uint32_t)(p.npad - 1);
    float2 acc2[BT];   // per batch item: (even events, odd events)
    const int cbeg = chan_begin(p), cend = chan_end(p);   // this CTA's channel slice
#pragma unroll
    for (int bi = 0; bi < BT; bi++) acc2[bi] = make_float2(0.f, 0.f);
    int stage = 0;
    uint32_t phase = 0;
    bool dead = false;
    uint32_t issued_mask = 0;

    const uint32_t ring_u32 = smem_u32(sm.ring);
    const uint32_t chan_u32 = smem_u32(sm.chan_pos);
    const uint32_t zero_u32 = smem_u32(zero_group);
    const float2 magic2 = make_float2(kFloorMagic, kFloorMagic);
    const float2 neg1 = make_float2(-1.f, -1.f);

    for (int e0 = 0; e0 < p.n_events; e0 += SC) {
        const int sc = min(SC, p.n_events - e0);
        float ofs[SC], w[SC];
        staged_pass_begin<K, WB, SC>(p, sm, cx, e0, sc, ofs, w);
        float2 ofs2[SC / 2], w2[SC / 2];
#pragma unroll
        for (int j = 0; j < SC; j += 2) {
            ofs2[j / 2] = make_float2(ofs[j], ofs[j + 1]);
            w2[j / 2] = make_float2(w[j], w[j + 1]);
        }

        for (int c0 = cbeg; c0 < cend; c0 += CC) {
            if (cx.producer) {
                staged_produce_batch<K, WB, SC, BT>(p, &tmap, sm, cx, stage, phase, e0, sc, c0, dead, issued_mask);
            } else {
                const uint32_t full_bar = smem_u32(&sm.full[stage]);
                if (!dead && !bounded_wait(full_bar, phase, sm.abort_flag, p.status)) dead = true;
                if (!dead) {
                    const bool any_ovf = sm.ovf[stage] != 0;
                    const uint32_t stage_u32 = ring_u32 + stage * SG::stage_bytes;
#pragma unroll 1
                    for (int cl = 0; cl < CC; cl++) {
                        const int c = c0 + cl;
                        const float4 cp = lds_f4(chan_u32 + (stage * kStWin + cl) * 16);
                        recv_geom g = receive_geometry(cx.vx, cx.vy, cx.vz, cp.x, cp.y, cp.z);
                        if (p.srcdir)
                            apply_directivity(g, cx.vx, cx.vy, cx.vz, cp.x, cp.y, cp.z,
                                              sm.chan_dir[stage * kStWin + cl]);
                        uint32_t k0p[SC];
                        load_meta<SC>(sm.meta, stage, cl, k0p);
                        const unsigned char *groups = sm.ring + stage * SG::stage_bytes + (cl * SC) * GG::bytes;
                        if (!any_ovf) {
                            const float2 rsq2 = make_float2(g.rsq, g.rsq);
                            const float2 rinv2 = make_float2(g.rinv, g.rinv);
#pragma unroll
                            for (int j = 0; j < SC; j += 2) {
                                const float2 tau2 = __ffma2_rn(rsq2, rinv2, ofs2[j / 2]);
                                const float2 mm2 = __fadd2_rd(tau2, magic2);
                                const float2 nfl2 = __ffma2_rn(mm2, neg1, magic2);   // -(floor), exact
                                const float2 t2 = __fadd2_rn(tau2, nfl2);
                                const uint32_t ra = __float_as_uint(mm2.x) - k0p[j];
                                const uint32_t rb = __float_as_uint(mm2.y) - k0p[j + 1];
                                // plain shared-memory pointers: the per-item offsets fold into
                                // the loads as immediates
                                const st *pa = ra < (uint32_t)WB
                                                   ? reinterpret_cast<const st *>(groups + j * GG::bytes) + ra
                                                   : reinterpret_cast<const st *>(zero_group);
                                const st *pb = rb < (uint32_t)WB
                                                   ? reinterpret_cast<const st *>(groups + (j + 1) * GG::bytes) + rb
                                                   : reinterpret_cast<const st *>(zero_group);
#pragma unroll
                                for (int bi = 0; bi < BT; bi++) {
                                    constexpr int IE = GG::item_bytes / (int)sizeof(st);
                                    const float ta = pair_traits<K>::tap(pa[bi * IE], t2.x);
                                    const float tb = pair_traits<K>::tap(pb[bi * IE], t2.y);
                                    acc2[bi] = __ffma2_rn(w2[j / 2], make_float2(ta, tb), acc2[bi]);
                                }
                            }
                        } else {
#pragma unroll
                            for (int j = 0; j < SC; j++) {
                                const float tau = __fmaf_rn(g.rsq, g.rinv, ofs[j]);
                                const tau_split ts = split_tau(tau);
                                const uint32_t rr = ts.k + kFloorMagicBits - k0p[j];
#pragma unroll
                                for (int bi = 0; bi < BT; bi++) {
                                    st pr;
                                    if (k0p[j] == kOvf) {
                                        const int bb = min(cx.b * BT + bi, p.B - 1);
                                        const int64_t row = ((int64_t)bb * p.C + c) * p.S + (e0 + min(j, sc - 1));
                                        pr = Pg[row * p.npad + min(ts.k, kmax_pair)];
                                    } else if (rr < (uint32_t)WB) {
                                        pr = *reinterpret_cast<const st *>(groups + j * GG::bytes + bi * GG::item_bytes +
                                                                           rr * sizeof(st));
                                    } else {
                                        pr = *reinterpret_cast<const st *>(zero_group);
                                    }
                                    const float tv = pair_traits<K>::tap(pr, ts.t);
                                    if (j & 1) acc2[bi].y = __fmaf_rn(w[j], tv, acc2[bi].y);
                                    else acc2[bi].x = __fmaf_rn(w[j], tv, acc2[bi].x);
                                }
                            }
                        }
                    }
                }
                __syncwarp();
                if (cx.lane == 0) mbar_arrive(smem_u32(&sm.empty[stage]));
            }
            if (++stage == kStages) {
                stage = 0;
                phase ^= 1u;
            }
        }
        __syncthreads();
    }

    if (cx.producer) {
        staged_drain<K, WB>(sm, cx, stage, phase, issued_mask);
        return;
    }
    if (!cx.active || dead) return;
#pragma unroll
    for (int bi = 0; bi < BT; bi++) {
        const int bb = cx.b * BT + bi;
        if (bb < p.B) {
            float *o = static_cast<float *>(p.out) + (int64_t)bb * p.out_bstride + cx.v;
            const float acc = acc2[bi].x + acc2[bi].y;
            if (p.cchunk) atomicAdd(o, acc);   // channel slices add into the prepared image
            else *o = p.beta_zero ? acc : __fmaf_rn((float)p.beta_re, *o, acc);
        }
    }
}

// ------------------------------------------------------------------ adjoint ---
// One CTA = one voxel tile x one batch item.  Per unit (v, c, e):
//   L = x0 + t d, d = slope;  g = dLoss/dout[b, v];  a = g w
//   gw[e,v] += g L;  goff[e,v] += a d;  q(v,c) += a d
//   gdst[v] += q (v - c)/r;  gsrc[c] -= q (v - c)/r
//   gx[b,c,s,k] += a (1 - t);  gx[b,c,s,k+1] += a t      (0 <= k <= N-2)
// The two-tap scatter goes into the window's shared gradient slot as fixed
// point: per event pass the CTA takes amax = max |g w| over its tile, scales
// every contribution by 2^22 / amax and adds round(a s t) and
// round(a s) - round(a s t) with native shared-memory integer adds (float adds
// to shared memory would be compare-and-swap loops).  A slot entry collects at
// most 2 x 256 contributions per stage, so it stays within 2^31; the rounding
// error per contribution is 2^-23 amax.  After all consumer warps finished a
// stage, they flush the touched entries to gx (red.global.add.f32) and zero
// them.  Taps outside a staged window (overflowing windows) and passes whose
// amax is not a positive finite number scatter with global float atomics.
// Channel-position gradients are reduced over the tile in shared memory and
// added once per channel per CTA.  Voxels are spread over the warps
// (staged_setup's spread mapping) so a warp's lanes rarely share a sample.
template <int K, int SC, int WB>
__global__ void __launch_bounds__(kStThreads, 2) das_staged_bwd_kernel(const staged_params p,
                                                                     const __grid_constant__ CUtensorMap tmap) {
    using SG = slot_geom<WB, K>;
    using st = typename pair_traits<K>::storage;
    constexpr int CC = kStWin / SC;
    constexpr int GS = bin_stride(WB);  // gradient slot stride (int32 entries)
    static_assert(kStWin % SC == 0, "SC must divide the stage");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    staged_smem<K, WB> sm(smem_raw);
    // one set of gradient slots (in two copies): a stage's slots are flushed
    // and cleared between two consumer barriers before the next stage
    // scatters into them
    constexpr int kRegion = bin_region_words(kStWin * GS);
    int *gslot = reinterpret_cast<int *>(sm.extra);                      // [kBinCopies][kRegion]
    float *cgrad = reinterpret_cast<float *>(gslot + kBinCopies * kRegion);  // [CC * 3][256]
    float *wmax = cgrad + CC * 3 * kStConsumers;                          // [kStWarps]
    for (int i = threadIdx.x; i < kBinCopies * kRegion; i += kStThreads) gslot[i] = 0;
    const staged_ctx cx = staged_setup<K, WB>(p, sm, true);   // ends with __syncthreads
    const uint32_t gslot_u32 = smem_u32(gslot) + cx.par * (kRegion * 4);   // this thread's copy

    const bool multi_b = p.B > 1 || gridDim.z > 1;   // several CTAs add into the voxel-side gradients
    const int cbeg = chan_begin(p), cend = chan_end(p);
    const float g = (cx.active) ? __ldg(p.gout + (int64_t)cx.b * p.gout_bstride + cx.v) : 0.f;
    const bool want_pos = p.gdst != nullptr || p.gsrc != nullptr;
    float gpx = 0.f, gpy = 0.f, gpz = 0.f;
    int stage = 0;
    uint32_t phase = 0;
    bool dead = false;
    uint32_t issued_mask = 0;

    for (int e0 = 0; e0 < p.n_events; e0 += SC) {
        const int sc = min(SC, p.n_events - e0);
        float ofs[SC], w[SC];
        staged_pass_begin<K, WB, SC>(p, sm, cx, e0, sc, ofs, w);
        // Per event: sums over channels of x0, d and t*d of the taps (L = x0 + t d),
        // so gw = g (sx0 + std) and goff = g w sd at the end of the pass.
        float sx0[SC], sd[SC], std_[SC];
#pragma unroll
        for (int j = 0; j < SC; j++) { sx0[j] = 0.f; sd[j] = 0.f; std_[j] = 0.f; }
        // fixed-point scale of this pass: amax = max |g w| over the tile
        float fscale = 0.f, finv = 0.f;
        bool fixed = false;
        if (!cx.producer) {
            float m = 0.f;
            bool bad = false;   // a non-finite g w (NaN fails the comparison)
#pragma unroll
            for (int j = 0; j < SC; j++) {
                const float aw = fabsf(g * w[j]);
                m = fmaxf(m, aw);
                bad |= !(aw <= 3.0e38f);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            bad = __any_sync(0xffffffffu, bad);
            if (cx.lane == 0) wmax[cx.warp] = bad ? -1.f : m;
            consumer_sync();
            float amax = 0.f;
            bool any_bad = false;
#pragma unroll
            for (int i = 0; i < kStWarps; i++) {
                const float v = wmax[i];
                any_bad |= v < 0.f;
                amax = fmaxf(amax, v);
            }
            fixed = !any_bad && amax > 0.f && amax <= 3.0e38f;
            if (fixed) {
                fscale = kFixRange / amax;
                finv = amax / kFixRange;
            }
            consumer_sync();   // wmax is rewritten by the next pass
        }
        float aw[SC], asw[SC];   // g w and its fixed-point scaling, per event
#pragma unroll
        for (int j = 0; j < SC; j++) {
            aw[j] = g * w[j];
            asw[j] = aw[j] * fscale;
        }
        const float2 magic2 = make_float2(kFloorMagic, kFloorMagic);
        const float2 neg1 = make_float2(-1.f, -1.f);

        for (int c0 = cbeg; c0 < cend; c0 += CC) {
            if (cx.producer) {
                staged_produce<K, WB, SC>(p, &tmap, sm, cx, stage, phase, e0, sc, c0, dead, issued_mask);
            } else {
                const uint32_t full_bar = smem_u32(&sm.full[stage]);
                const unsigned char *stage_base = sm.ring + stage * SG::stage_bytes;
                int *gstage = gslot;
                const uint32_t gstage_u32 = gslot_u32;
                if (!dead && !bounded_wait(full_bar, phase, sm.abort_flag, p.status)) dead = true;
                const bool any_ovf = !dead && sm.ovf[stage] != 0;
                if (!dead && !any_ovf && (fixed || !p.gx)) {
                    // Common case, branch-free per unit: every tap lies in its window
                    // (out-of-window taps are out of the record and read the zero
                    // pair), and a tap outside the record scatters a zero.
                    const uint32_t stage_u32 = smem_u32(stage_base);
                    const uint32_t nlast = (uint32_t)(p.N - 1);
                    for (int cl = 0; cl < CC; cl++) {
                        const int c = c0 + cl;
                        if (c >= cend) break;   // a channel past the slice (or a phantom one) is not this CTA's
                        const float4 cp = sm.chan_pos[stage * kStWin + cl];
                        const recv_geom gm = receive_geometry(cx.vx, cx.vy, cx.vz, cp.x, cp.y, cp.z);
                        uint32_t k0p[SC];
                        load_meta<SC>(sm.meta, stage, cl, k0p);
                        const uint32_t slots_u32 = stage_u32 + (cl * SC) * SG::bytes;
                        const uint32_t gwin_u32 = gstage_u32 + (cl * SC) * GS * 4;
                        const float2 rsq2 = make_float2(gm.rsq, gm.rsq), rinv2 = make_float2(gm.rinv, gm.rinv);
                        float q = 0.f;
#pragma unroll
                        for (int j = 0; j < SC; j += 2) {
                            const float o1 = (j + 1 < SC) ? ofs[j + 1] : 1e30f;
                            const float2 tau2 = __ffma2_rn(rsq2, rinv2, make_float2(ofs[j], o1));
                            const float2 mm2 = __fadd2_rd(tau2, magic2);
                            const float2 nfl2 = __ffma2_rn(mm2, neg1, magic2);   // -(floor), exact
                            const float2 t2 = __fadd2_rn(tau2, nfl2);
#pragma unroll
                            for (int h = 0; h < 2; h++) {
                                const int jj = j + h;
                                if (jj >= SC) break;
                                const uint32_t mb = __float_as_uint(h ? mm2.y : mm2.x);
                                const float t = h ? t2.y : t2.x;
                                const uint32_t rel = min(mb - k0p[jj], (uint32_t)WB);
                                float x0, d;
                                pair_x0_d<K>(slots_u32 + jj * SG::bytes + rel * sizeof(st), x0, d);
                                sx0[jj] += x0;
                                sd[jj] += d;
                                std_[jj] = __fmaf_rn(t, d, std_[jj]);
                                q = __fmaf_rn(aw[jj], d, q);
                                if (p.gx) {
                                    const float as = (mb - kFloorMagicBits < nlast) ? asw[jj] : 0.f;
                                    // round(a) - round(a t) to sample k, round(a t) to k + 1
                                    const int ab = __float_as_int(as + kFloorMagic), tb = fix_bits_fma(as, t);
                                    const uint32_t ga = gwin_u32 + (jj * GS + rel) * 4;
                                    red_shared_add(ga, ab - tb);
                                    red_shared_add(ga + 4, tb - (int)kFloorMagicBits);
                                }
                            }
                        }
                        if (want_pos) {
                            const float qr = q * gm.rinv;
                            const float ex = (cx.vx - cp.x) * qr, ey = (cx.vy - cp.y) * qr, ez = (cx.vz - cp.z) * qr;
                            gpx += ex; gpy += ey; gpz += ez;
                            if (p.gsrc) {
                                cgrad[(cl * 3 + 0) * kStConsumers + cx.tid] = -ex;
                                cgrad[(cl * 3 + 1) * kStConsumers + cx.tid] = -ey;
                                cgrad[(cl * 3 + 2) * kStConsumers + cx.tid] = -ez;
                            }
                        }
                    }
                } else if (!dead) {
                    for (int cl = 0; cl < CC; cl++) {
                        const int c = c0 + cl;
                        if (c >= cend) break;   // a channel past the slice (or a phantom one) is not this CTA's
                        const float4 cp = sm.chan_pos[stage * kStWin + cl];
                        const recv_geom gm = receive_geometry(cx.vx, cx.vy, cx.vz, cp.x, cp.y, cp.z);
                        uint32_t k0p[SC];
                        load_meta<SC>(sm.meta, stage, cl, k0p);
                        const unsigned char *slots = stage_base + (cl * SC) * SG::bytes;
                        float q = 0.f;
#pragma unroll
                        for (int j = 0; j < SC; j++) {
                            const float tau = __fmaf_rn(gm.rsq, gm.rinv, ofs[j]);
                            const tau_split ts = split_tau(tau);
                            st pr;
                            const bool ovfw = any_ovf && k0p[j] == kOvf;
                            uint32_t rel = WB;
                            if (ovfw) {
                                const int64_t row = ((int64_t)cx.b * p.C + c) * p.S + (e0 + min(j, sc - 1));
                                pr = static_cast<const st *>(p.P)[row * p.npad + min(ts.k, (uint32_t)(p.npad - 1))];
                            } else {
                                rel = min(ts.k + kFloorMagicBits - k0p[j], (uint32_t)WB);
                                pr = *reinterpret_cast<const st *>(slots + j * SG::bytes + rel * sizeof(st));
                            }
                            const float d = pair_traits<K>::slope(pr);
                            const float x0 = pair_traits<K>::tap(pr, 0.f);
                            const float a = aw[j];
                            sx0[j] += x0;
                            sd[j] += d;
                            std_[j] = __fmaf_rn(ts.t, d, std_[j]);
                            q = __fmaf_rn(a, d, q);
                            // channel-data adjoint: only taps inside the record
                            if (p.gx && a != 0.f && ts.k < (uint32_t)(p.N - 1)) {
                                if (fixed && !ovfw && rel < (uint32_t)WB) {
                                    const float as = asw[j];
                                    const int it = fix_round(as);
                                    const int i1 = fix_round_fma(as, ts.t);
                                    const uint32_t ga = gstage_u32 + ((cl * SC + j) * GS + rel) * 4;
                                    red_shared_add(ga, it - i1);
                                    red_shared_add(ga + 4, i1);
                                } else {
                                    const float a1 = a * ts.t;
                                    float *gr = p.gx + (((int64_t)cx.b * p.C + c) * p.S + (e0 + j)) * p.N + ts.k;
                                    atomicAdd(gr, a - a1);
                                    atomicAdd(gr + 1, a1);
                                }
                            }
                        }
                        if (want_pos) {
                            const float qr = q * gm.rinv;
                            const float ex = (cx.vx - cp.x) * qr, ey = (cx.vy - cp.y) * qr, ez = (cx.vz - cp.z) * qr;
                            gpx += ex; gpy += ey; gpz += ez;
                            if (p.gsrc) {
                                cgrad[(cl * 3 + 0) * kStConsumers + cx.tid] = -ex;
                                cgrad[(cl * 3 + 1) * kStConsumers + cx.tid] = -ey;
                                cgrad[(cl * 3 + 2) * kStConsumers + cx.tid] = -ez;
                            }
                        }
                    }
                }
                // every consumer warp finished this stage's scatter
                consumer_sync();
                if (!dead) {
                    // flush the stage's gradient slots: one red.add per touched sample
                    if (p.gx && fixed) {
                        flush_bins<WB, kRegion>(gstage, cx.lane, cx.warp, finv, [&](int win, int &kw) -> float * {
                            const int cl = win / SC, j = win % SC;
                            kw = (int)(sm.meta[stage * kStWin + win] - kFloorMagicBits);
                            if (c0 + cl >= cend) return nullptr;
                            return p.gx + (((int64_t)cx.b * p.C + (c0 + cl)) * p.S + (e0 + j)) * p.N;
                        });
                    }
                    // channel-position gradients: reduce the tile, one add per channel
                    if (p.gsrc) {
                        for (int o = cx.warp; o < CC * 3; o += kStWarps) {
                            const int cl = o / 3;
                            if (c0 + cl >= cend) continue;
                            float s = 0.f;
#pragma unroll
                            for (int i = 0; i < kStConsumers / 32; i++) s += cgrad[o * kStConsumers + cx.lane + 32 * i];
#pragma unroll
                            for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
                            if (cx.lane == 0 && s != 0.f) atomicAdd(p.gsrc + 3 * (c0 + cl) + (o % 3), s);
                        }
                    }
                }
                consumer_sync();  // scratch reused by the next stage
                __syncwarp();
                if (cx.lane == 0) mbar_arrive(smem_u32(&sm.empty[stage]));
            }
            if (++stage == kStages) {
                stage = 0;
                phase ^= 1u;
            }
        }
        if (!cx.producer && cx.active && !dead) {
#pragma unroll
            for (int j = 0; j < SC; j++) {
                if (j < sc) {
                    const int64_t idx = (int64_t)(e0 + j) * p.V + cx.v;
                    const float gwv = g * (sx0[j] + std_[j]);   // g * sum over channels of the taps
                    const float gov = aw[j] * sd[j];            // g w * sum of the slopes
                    if (multi_b) {
                        if (p.gw) atomicAdd(p.gw + idx, gwv);
                        if (p.goff) atomicAdd(p.goff + idx, gov);
                    } else {
                        if (p.gw) p.gw[idx] = gwv;
                        if (p.goff) p.goff[idx] = gov;
                    }
                }
            }
        }
        __syncthreads();
    }

    if (cx.producer) {
        staged_drain<K, WB>(sm, cx, stage, phase, issued_mask);
        return;
    }
    if (cx.active && !dead && p.gdst) {
        if (multi_b) {
            atomicAdd(p.gdst + 3 * cx.v, gpx);
            atomicAdd(p.gdst + 3 * cx.v + 1, gpy);
            atomicAdd(p.gdst + 3 * cx.v + 2, gpz);
        } else {
            p.gdst[3 * cx.v] = gpx;
            p.gdst[3 * cx.v + 1] = gpy;
            p.gdst[3 * cx.v + 2] = gpz;
        }
    }
}

// ------------------------------------------------------- adjoint, batch tiles ---
// The adjoint for BT batch items per CTA: windows staged as in
// das_staged_batch_kernel (one 3-D TMA box per channel and event), delays,
// split and window index computed once per (voxel, channel, event), then per
// item: the tap's sample and slope, g_b-weighted sums for the weight, offset
// and position gradients, and the fixed-point scatter of g_b w (1 - t), g_b w t
// into the item's gradient slot.  amax = max_b |g_b| * max_j |w_j| over the tile.
//
// The slot of a window holds one fixed-point bin per sample kw .. kw + WB:
// a tap at sample k adds round(a) - round(a t) to bin k and round(a t) to bin
// k + 1, a = g_b w scaled, and a tap outside the record adds zeros (one test
// per voxel, channel and event, shared by the BT items).  A tap outside its
// window is always outside the record and adds its zeros past the window.
template <int WB, int K, int SC, int BT>
constexpr size_t staged_bwd_batch_smem_bytes() {
    return staged_smem_bytes<WB, K>() + 2 * kBinCopies * bin_region_words(kStWin * bin_stride(WB)) * 4 +
           2 * (group_geom<WB, K, BT>::groups / SC) * 3 * kStConsumers * 4 + kStWarps * 4 + 16 +
           group_geom<WB, K, BT>::data_bytes;
}

template <int K, int SC, int WB, int BT>
__global__ void __launch_bounds__(kStThreads, 2) das_staged_bwd_batch_kernel(const staged_params p,
                                                                            const __grid_constant__ CUtensorMap tmap) {
    using SG = slot_geom<WB, K>;
    using GG = group_geom<WB, K, BT>;
    using st = typename pair_traits<K>::storage;
    constexpr int CC = GG::groups / SC;
    constexpr int GS = bin_stride(WB);  // bins per window: samples kw .. kw + WB, then zero-only ones
    static_assert(SC % 2 == 0 && GG::groups % SC == 0, "SC * BT must divide the stage");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    staged_smem<K, WB> sm(smem_raw);
    // Two sets of bins (each in two copies) and of channel-gradient scratch,
    // used by stages of alternate parity (kStages is even): a warp that has
    // flushed stage s's set scatters stage s + 1 into the other while slower
    // warps still read s's, and the barrier after stage s + 1's scatter orders
    // every flush of s's set before stage s + 2 writes it -- one consumer
    // barrier per stage.
    static_assert(kStages % 2 == 0, "stage parity must alternate around the ring");
    constexpr int kRegion = bin_region_words(kStWin * GS);
    constexpr int kSet = kBinCopies * kRegion;                           // words per set of bins
    constexpr int kCg = CC * 3 * kStConsumers;                           // floats per channel-gradient set
    int *gslot = reinterpret_cast<int *>(sm.extra);   // [2][kBinCopies][kRegion]: [kStWin][GS], window = group * BT + item
    float *cgrad0 = reinterpret_cast<float *>(gslot + 2 * kSet);        // [2][CC * 3][256]
    float *wmax = cgrad0 + 2 * kCg;                                      // [kStWarps]
    // zero group after the scratch, 16-byte aligned (offset arithmetic on the
    // shared pointer keeps its address space visible to the compiler)
    constexpr int kZeroOff = ((2 * kSet + 2 * kCg + kStWarps) * 4 + 15) & ~15;
    unsigned char *zero_group = sm.extra + kZeroOff;
    for (int i = threadIdx.x; i < 2 * kSet; i += kStThreads) gslot[i] = 0;
    for (int i = threadIdx.x; i < GG::data_bytes / 4; i += kStThreads) reinterpret_cast<uint32_t *>(zero_group)[i] = 0u;
    const staged_ctx cx = staged_setup<K, WB>(p, sm, true);   // ends with __syncthreads
    const uint32_t gslot_u32 = smem_u32(gslot) + cx.par * (kRegion * 4);   // this thread's copy
    const uint32_t zero_u32 = smem_u32(zero_group);

    const int b0 = cx.b * BT;
    const bool multi = gridDim.y > 1 || gridDim.z > 1;   // several CTAs add into the voxel-side gradients
    const int cbeg = chan_begin(p), cend = chan_end(p);
    float g[BT];
    float gmax = 0.f;
#pragma unroll
    for (int bi = 0; bi < BT; bi++) {
        g[bi] = (cx.active && b0 + bi < p.B) ? __ldg(p.gout + (int64_t)(b0 + bi) * p.gout_bstride + cx.v) : 0.f;
        gmax = fmaxf(gmax, fabsf(g[bi]));
    }
    bool gbad = false;
    float2 g2[BT];   // (g_b, g_b) for the packed sample / slope sums
#pragma unroll
    for (int bi = 0; bi < BT; bi++) {
        gbad |= !(fabsf(g[bi]) <= 3.0e38f);
        g2[bi] = make_float2(g[bi], g[bi]);
    }
    const bool want_pos = p.gdst != nullptr || p.gsrc != nullptr;
    float gpx = 0.f, gpy = 0.f, gpz = 0.f;
    int stage = 0;
    uint32_t phase = 0;
    bool dead = false;
    uint32_t issued_mask = 0;
    const float2 magic2 = make_float2(kFloorMagic, kFloorMagic);
    const float2 neg1 = make_float2(-1.f, -1.f);

    for (int e0 = 0; e0 < p.n_events; e0 += SC) {
        const int sc = min(SC, p.n_events - e0);
        float ofs[SC], w[SC];
        staged_pass_begin<K, WB, SC>(p, sm, cx, e0, sc, ofs, w);
        // per event: sum of g_b x0, of g_b d and of t g_b d over channels and items
        float sx[SC], sd[SC], std_[SC];
#pragma unroll
        for (int j = 0; j < SC; j++) { sx[j] = 0.f; sd[j] = 0.f; std_[j] = 0.f; }
        float fscale = 0.f, finv = 0.f;
        bool fixed = false;
        if (!cx.producer) {
            float wm = 0.f;
            bool bad = gbad;
#pragma unroll
            for (int j = 0; j < SC; j++) {
                wm = fmaxf(wm, fabsf(w[j]));
                bad |= !(fabsf(w[j]) <= 3.0e38f);
            }
            float m = gmax * wm;
            bad |= !(m <= 3.0e38f);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            bad = __any_sync(0xffffffffu, bad);
            if (cx.lane == 0) wmax[cx.warp] = bad ? -1.f : m;
            consumer_sync();
            float amax = 0.f;
            bool any_bad = false;
#pragma unroll
            for (int i = 0; i < kStWarps; i++) {
                const float v = wmax[i];
                any_bad |= v < 0.f;
                amax = fmaxf(amax, v);
            }
            fixed = !any_bad && amax > 0.f && amax <= 3.0e38f;
            if (fixed) {
                fscale = kFixRange / amax;
                finv = amax / kFixRange;
            }
            consumer_sync();   // wmax is rewritten by the next pass
        }
        float gsw[SC];   // w scaled to fixed point; a contribution is g_b * gsw
#pragma unroll
        for (int j = 0; j < SC; j++) gsw[j] = w[j] * fscale;

        for (int c0 = cbeg; c0 < cend; c0 += CC) {
            if (cx.producer) {
                staged_produce_batch<K, WB, SC, BT>(p, &tmap, sm, cx, stage, phase, e0, sc, c0, dead, issued_mask);
            } else {
                const uint32_t full_bar = smem_u32(&sm.full[stage]);
                const uint32_t stage_u32 = smem_u32(sm.ring + stage * SG::stage_bytes);
                int *gstage = gslot + (stage & 1) * kSet;
                const uint32_t gstage_u32 = gslot_u32 + (stage & 1) * (kSet * 4);
                float *cgrad = cgrad0 + (stage & 1) * kCg;
                if (!dead && !bounded_wait(full_bar, phase, sm.abort_flag, p.status)) dead = true;
                const bool any_ovf = !dead && sm.ovf[stage] != 0;
                if (!dead) {
                    const uint32_t nlast = (uint32_t)(p.N - 1);
                    // One channel of the stage.  FAST: every in-record tap is in its
                    // window and the scatter (SCATTER) is fixed point; POS: position
                    // gradients.  The flags are decided once per stage, so the fast
                    // path's channels unroll into one straight run (independent work
                    // for the scheduler); its phantom channels past the slice read
                    // zero windows and add exact zeros (their bins are never flushed
                    // to gx, their channel gradients never reduced).
                    auto channel = [&](const int cl, auto fast_c, auto scatter_c, auto pos_c) {
                        constexpr bool FAST = decltype(fast_c)::value;
                        constexpr bool SCATTER = decltype(scatter_c)::value;
                        constexpr bool POS = decltype(pos_c)::value;
                        (void)SCATTER;

                        const int c = c0 + cl;
                        const float4 cp = sm.chan_pos[stage * kStWin + cl];
                        const recv_geom gm = receive_geometry(cx.vx, cx.vy, cx.vz, cp.x, cp.y, cp.z);
                        uint32_t k0p[SC];
                        load_meta<SC>(sm.meta, stage, cl, k0p);
                        const uint32_t groups_u32 = stage_u32 + (cl * SC) * GG::bytes;
                        const uint32_t gwin_u32 = gstage_u32 + (cl * SC * BT) * GS * 4;
                        float q = 0.f;
                        if constexpr (FAST) {
                            const unsigned char *groups = sm.ring + stage * SG::stage_bytes + (cl * SC) * GG::bytes;
                            // common case: every in-record tap is in its window
                            const float2 rsq2 = make_float2(gm.rsq, gm.rsq), rinv2 = make_float2(gm.rinv, gm.rinv);
                            {
#pragma unroll
                                for (int j = 0; j < SC; j += 2) {
                                    const float2 tau2 = __ffma2_rn(rsq2, rinv2, make_float2(ofs[j], ofs[j + 1]));
                                    const float2 mm2 = __fadd2_rd(tau2, magic2);
                                    const float2 nfl2 = __ffma2_rn(mm2, neg1, magic2);   // -(floor), exact
                                    const float2 t2 = __fadd2_rn(tau2, nfl2);
#pragma unroll
                                    for (int h = 0; h < 2; h++) {
                                        const int jj = j + h;
                                        const uint32_t mb = __float_as_uint(h ? mm2.y : mm2.x);
                                        const float t = h ? t2.y : t2.x;
                                        const uint32_t rr = mb - k0p[jj];
                                        // plain shared-memory pointers: the per-item offsets fold
                                        // into the load / atomic instructions as immediates
                                        const st *tp = rr < (uint32_t)WB
                                                           ? reinterpret_cast<const st *>(groups + jj * GG::bytes) + rr
                                                           : reinterpret_cast<const st *>(zero_group);
                                        float2 sg = make_float2(sx[jj], 0.f);   // (sum g_b x0, sum g_b d)
                                        if constexpr (SCATTER) {
                                            const uint32_t gb = gwin_u32 + ((jj * BT) * GS + min(rr, (uint32_t)WB)) * 4;
                                            // a tap outside the record scatters zeros (into its
                                            // window's bins, or the zero-only bins past the window)
                                            const float gsin = (mb - kFloorMagicBits < nlast) ? gsw[jj] : 0.f;
                                            const float gst = gsin * t;
                                            static_for<0, BT>([&](auto bic) {
                                                constexpr int bi = decltype(bic)::value;
                                                float x0, d;
                                                pair_x0_d_ptr<K>(tp + bi * (GG::item_bytes / (int)sizeof(st)), x0, d);
                                                sg = __ffma2_rn(g2[bi], make_float2(x0, d), sg);
                                                // round(g w) - round(g w t) to sample k, round(g w t) to k + 1
                                                const int ab = fix_bits_fma(g[bi], gsin), tb = fix_bits_fma(g[bi], gst);
                                                red_shared_add_at<bi * GS * 4>(gb, ab - tb);
                                                red_shared_add_at<bi * GS * 4 + 4>(gb, tb - (int)kFloorMagicBits);
                                            });
                                        } else {
#pragma unroll
                                            for (int bi = 0; bi < BT; bi++) {
                                                float x0, d;
                                                pair_x0_d_ptr<K>(tp + bi * (GG::item_bytes / (int)sizeof(st)), x0, d);
                                                sg = __ffma2_rn(g2[bi], make_float2(x0, d), sg);
                                            }
                                        }
                                        sx[jj] = sg.x;
                                        const float gd = sg.y;
                                        sd[jj] += gd;
                                        std_[jj] = __fmaf_rn(t, gd, std_[jj]);
                                        q = __fmaf_rn(w[jj], gd, q);
                                    }
                                }
                            }
                        } else {
                            const unsigned char *groups = sm.ring + stage * SG::stage_bytes + (cl * SC) * GG::bytes;
#pragma unroll
                            for (int j = 0; j < SC; j++) {
                                const float tau = __fmaf_rn(gm.rsq, gm.rinv, ofs[j]);
                                const tau_split ts = split_tau(tau);
                                const bool ovfw = k0p[j] == kOvf;
                                const uint32_t rr = ts.k + kFloorMagicBits - k0p[j];
                                float gd = 0.f;
#pragma unroll
                                for (int bi = 0; bi < BT; bi++) {
                                    st pr;
                                    if (ovfw) {
                                        const int bb = min(b0 + bi, p.B - 1);
                                        const int64_t row = ((int64_t)bb * p.C + c) * p.S + (e0 + min(j, sc - 1));
                                        pr = static_cast<const st *>(p.P)[row * p.npad + min(ts.k, (uint32_t)(p.npad - 1))];
                                    } else if (rr < (uint32_t)WB) {
                                        pr = *reinterpret_cast<const st *>(groups + j * GG::bytes + bi * GG::item_bytes +
                                                                           rr * sizeof(st));
                                    } else {
                                        pr = *reinterpret_cast<const st *>(zero_group);
                                    }
                                    const float d = pair_traits<K>::slope(pr);
                                    const float x0 = pair_traits<K>::tap(pr, 0.f);
                                    sx[j] = __fmaf_rn(g[bi], x0, sx[j]);
                                    gd = __fmaf_rn(g[bi], d, gd);
                                    const float a = g[bi] * w[j];
                                    if (p.gx && a != 0.f && ts.k < nlast && b0 + bi < p.B) {
                                        if (fixed && !ovfw && rr < (uint32_t)WB) {
                                            const float as = g[bi] * gsw[j];
                                            const uint32_t ga = gwin_u32 + ((j * BT + bi) * GS + rr) * 4;
                                            const int it = fix_round(as), i1 = fix_round_fma(as, ts.t);
                                            red_shared_add(ga, it - i1);
                                            red_shared_add(ga + 4, i1);
                                        } else {
                                            const float a1 = a * ts.t;
                                            float *gr = p.gx + (((int64_t)(b0 + bi) * p.C + c) * p.S + (e0 + j)) * p.N + ts.k;
                                            atomicAdd(gr, a - a1);
                                            atomicAdd(gr + 1, a1);
                                        }
                                    }
                                }
                                sd[j] += gd;
                                std_[j] = __fmaf_rn(ts.t, gd, std_[j]);
                                q = __fmaf_rn(w[j], gd, q);
                            }
                        }
                        if constexpr (POS) {
                            const float qr = q * gm.rinv;
                            const float ex = (cx.vx - cp.x) * qr, ey = (cx.vy - cp.y) * qr, ez = (cx.vz - cp.z) * qr;
                            gpx += ex; gpy += ey; gpz += ez;
                            if (p.gsrc) {
                                cgrad[(cl * 3 + 0) * kStConsumers + cx.tid] = -ex;
                                cgrad[(cl * 3 + 1) * kStConsumers + cx.tid] = -ey;
                                cgrad[(cl * 3 + 2) * kStConsumers + cx.tid] = -ez;
                            }
                        }
                                        };
                    auto run = [&](auto fast_c, auto scatter_c, auto pos_c) {
                        if constexpr (decltype(fast_c)::value) {
#pragma unroll
                            for (int cl = 0; cl < CC; cl++) channel(cl, fast_c, scatter_c, pos_c);
                        } else {
                            for (int cl = 0; cl < CC; cl++) {
                                if (c0 + cl >= cend) break;   // a channel past the slice (or a phantom one)
                                channel(cl, fast_c, scatter_c, pos_c);
                            }
                        }
                    };
                    using T_ = std::true_type;
                    using F_ = std::false_type;
                    if (!any_ovf && (fixed || !p.gx)) {
                        if (p.gx) {
                            if (want_pos) run(T_{}, T_{}, T_{}); else run(T_{}, T_{}, F_{});
                        } else {
                            if (want_pos) run(T_{}, F_{}, T_{}); else run(T_{}, F_{}, F_{});
                        }
                    } else {
                        if (want_pos) run(F_{}, F_{}, T_{}); else run(F_{}, F_{}, F_{});
                    }
                }
                // every consumer warp finished this stage's scatter
                consumer_sync();
                if (!dead) {
                    if (p.gx && fixed) {
                        flush_bins<WB, kRegion>(gstage, cx.lane, cx.warp, finv, [&](int win, int &kw) -> float * {
                            const int grp = win / BT, bi = win % BT;
                            const int cl = grp / SC, j = grp % SC;
                            kw = (int)(sm.meta[stage * kStWin + grp] - kFloorMagicBits);
                            if (b0 + bi >= p.B || c0 + cl >= cend) return nullptr;
                            return p.gx + (((int64_t)(b0 + bi) * p.C + (c0 + cl)) * p.S + (e0 + j)) * p.N;
                        });
                    }
                    if (p.gsrc) {
                        for (int o = cx.warp; o < CC * 3; o += kStWarps) {
                            const int cl = o / 3;
                            if (c0 + cl >= cend) continue;
                            float s = 0.f;
#pragma unroll
                            for (int i = 0; i < kStConsumers / 32; i++) s += cgrad[o * kStConsumers + cx.lane + 32 * i];
#pragma unroll
                            for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
                            if (cx.lane == 0 && s != 0.f) atomicAdd(p.gsrc + 3 * (c0 + cl) + (o % 3), s);
                        }
                    }
                }
                // no barrier: the next stage uses the other set of scratch, and
                // the producer refills this ring stage once every warp arrived
                __syncwarp();
                if (cx.lane == 0) mbar_arrive(smem_u32(&sm.empty[stage]));
            }
            if (++stage == kStages) {
                stage = 0;
                phase ^= 1u;
            }
        }
        if (!cx.producer && cx.active && !dead) {
#pragma unroll
            for (int j = 0; j < SC; j++) {
                if (j < sc) {
                    const int64_t idx = (int64_t)(e0 + j) * p.V + cx.v;
                    const float gwv = sx[j] + std_[j];   // sum over items and channels of g_b L
                    const float gov = w[j] * sd[j];      // w * sum of g_b d
                    if (multi) {
                        if (p.gw) atomicAdd(p.gw + idx, gwv);
                        if (p.goff) atomicAdd(p.goff + idx, gov);
                    } else {
                        if (p.gw) p.gw[idx] = gwv;
                        if (p.goff) p.goff[idx] = gov;
                    }
                }
            }
        }
        __syncthreads();
    }

    if (cx.producer) {
        staged_drain<K, WB>(sm, cx, stage, phase, issued_mask);
        return;
    }
    if (cx.active && !dead && p.gdst) {
        if (multi) {
            atomicAdd(p.gdst + 3 * cx.v, gpx);
            atomicAdd(p.gdst + 3 * cx.v + 1, gpy);
            atomicAdd(p.gdst + 3 * cx.v + 2, gpz);
        } else {
            p.gdst[3 * cx.v] = gpx;
            p.gdst[3 * cx.v + 1] = gpy;
            p.gdst[3 * cx.v + 2] = gpz;
        }
    }
}

// ------------------------------------------------------- complex (IQ) data ---
// Forward for complex channel data (complex64 pairs (x0, x1 - x0), or
// complex32 pairs (x0, x1)) on the same producer and ring: one voxel per
// consumer thread, SC events per pass.  A tap adds w (cos, sin)(wavenum tau)
// x lerp with the reference's cmadd ordering (src/das/das_alg1_kernels.cuh:
// 78-98); a tap outside the record reads the zero pair and adds an exact zero,
// as in the gather kernel.  Channels, event chunks and events within a chunk
// are summed in the gather kernel's order, so with the same event chunk the
// two kernels agree bit for bit.
template <int K, int SC, int WB>
__global__ void __launch_bounds__(kStThreads) das_staged_cplx_kernel(const staged_params p,
                                                                     const __grid_constant__ CUtensorMap tmap) {
    using st = typename pair_traits<K>::storage;
    using SG = slot_geom<WB, K>;
    constexpr int CC = kStWin / SC;
    static_assert(kStWin % SC == 0, "SC must divide the stage");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    staged_smem<K, WB> sm(smem_raw);
    const staged_ctx cx = staged_setup<K, WB>(p, sm);
    const int cbeg = chan_begin(p), cend = chan_end(p);
    const st *__restrict__ Pg = static_cast<const st *>(p.P);
    const uint32_t kmax_pair = (uint32_t)(p.npad - 1);
    const uint32_t nlast = (uint32_t)(p.N - 1);
    const float wavenum = p.wavenum;
    const bool srcdir = p.srcdir != nullptr;
    float2 acc = make_float2(0.f, 0.f);
    int stage = 0;
    uint32_t phase = 0;
    bool dead = false;
    uint32_t issued_mask = 0;

    for (int e0 = 0; e0 < p.n_events; e0 += SC) {
        const int sc = min(SC, p.n_events - e0);
        float ofs[SC], w[SC];
        staged_pass_begin<K, WB, SC>(p, sm, cx, e0, sc, ofs, w);
        for (int c0 = cbeg; c0 < cend; c0 += CC) {
            if (cx.producer) {
                staged_produce<K, WB, SC>(p, &tmap, sm, cx, stage, phase, e0, sc, c0, dead, issued_mask);
            } else {
                const uint32_t full_bar = smem_u32(&sm.full[stage]);
                if (!dead && !bounded_wait(full_bar, phase, sm.abort_flag, p.status)) dead = true;
                if (!dead && cx.active) {
                    const unsigned char *stage_base = sm.ring + stage * SG::stage_bytes;
                    const bool any_ovf = sm.ovf[stage] != 0;
                    for (int cl = 0; cl < CC; cl++) {
                        const int c = c0 + cl;
                        if (c >= cend) break;
                        const float4 cp = sm.chan_pos[stage * kStWin + cl];
                        recv_geom gm = receive_geometry(cx.vx, cx.vy, cx.vz, cp.x, cp.y, cp.z);
                        if (srcdir)
                            apply_directivity(gm, cx.vx, cx.vy, cx.vz, cp.x, cp.y, cp.z, sm.chan_dir[stage * kStWin + cl]);
                        uint32_t k0p[SC];
                        load_meta<SC>(sm.meta, stage, cl, k0p);
                        const unsigned char *slots = stage_base + (cl * SC) * SG::bytes;
                        if (!any_ovf) {
                            // branch-free: a tap outside the record reads the zero pair
                            // (its window index clamps there) and adds an exact zero
#pragma unroll
                            for (int j = 0; j < SC; j++) {
                                const float tau = __fmaf_rn(gm.rsq, gm.rinv, ofs[j]);
                                const tau_split ts = split_tau(tau);
                                const uint32_t rel = min(ts.k + kFloorMagicBits - k0p[j], (uint32_t)WB);
                                const st pr = *reinterpret_cast<const st *>(slots + j * SG::bytes + rel * sizeof(st));
                                float sn, cs;
                                __sincosf(wavenum * tau, &sn, &cs);
                                acc = cfma(make_float2(cs * w[j], sn * w[j]), pair_traits<K>::tap(pr, ts.t), acc);
                            }
                        } else {
#pragma unroll
                            for (int j = 0; j < SC; j++) {
                                const float tau = __fmaf_rn(gm.rsq, gm.rinv, ofs[j]);
                                const tau_split ts = split_tau(tau);
                                if (ts.k < nlast) {
                                    st pr;
                                    if (k0p[j] == kOvf) {
                                        const int64_t row = ((int64_t)cx.b * p.C + c) * p.S + (e0 + min(j, sc - 1));
                                        pr = Pg[row * p.npad + min(ts.k, kmax_pair)];
                                    } else {
                                        const uint32_t rel = min(ts.k + kFloorMagicBits - k0p[j], (uint32_t)WB);
                                        pr = *reinterpret_cast<const st *>(slots + j * SG::bytes + rel * sizeof(st));
                                    }
                                    float sn, cs;
                                    __sincosf(wavenum * tau, &sn, &cs);
                                    acc = cfma(make_float2(cs * w[j], sn * w[j]), pair_traits<K>::tap(pr, ts.t), acc);
                                }
                            }
                        }
                    }
                }
                __syncwarp();
                if (cx.lane == 0) mbar_arrive(smem_u32(&sm.empty[stage]));
            }
            if (++stage == kStages) {
                stage = 0;
                phase ^= 1u;
            }
        }
        __syncthreads();
    }

    if (cx.producer) {
        staged_drain<K, WB>(sm, cx, stage, phase, issued_mask);
        return;
    }
    if (dead || !cx.active) return;
    float2 *o = static_cast<float2 *>(p.out) + (int64_t)cx.b * p.out_bstride + cx.v;
    *o = p.beta_zero ? acc : cfma(make_float2((float)p.beta_re, (float)p.beta_im), *o, acc);
}

// Prepares the image for channel slices that add into it: out = beta * out
// (or 0) for every batch item and voxel.
__global__ void __launch_bounds__(256) scale_image_kernel(float *out, int64_t bstride, int64_t V, int B,
                                                          float beta, int beta_zero, const int *gate) {
    if (gate && *(volatile const int *)gate) return;   // the staged call is off: the gather kernel applies beta
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V) return;
    for (int b = blockIdx.y; b < B; b += gridDim.y) {
        float *o = out + (int64_t)b * bstride + i;
        *o = beta_zero ? 0.f : beta * *o;
    }
}

}  // namespace ffdas
