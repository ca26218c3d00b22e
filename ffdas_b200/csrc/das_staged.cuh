// das_staged.cuh -- forward delay-and-sum, TMA-staged schedule (sm_100a).
//
// A CTA owns a compact tile of 256 voxels (one per consumer thread) and one
// batch item.  A ninth warp is the producer: for every (channel, event) it
// bounds the sample window the whole tile can touch -- from the tile's
// bounding box and the tile's min/max delay for that event -- and stages that
// window of interpolation pairs into shared memory with one TMA tile load
// (cp.async.bulk.tensor, no multicast), running up to kStages chunks ahead of
// the consumers through a full/empty mbarrier ring.  Consumers then gather
// each tap from shared memory: per unit one FFMA for the delay, the
// floor/fraction split, one index clamp, one 8-byte LDS and two FFMAs.
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
// FFDAS_DEVICE_STATUS_TIMEOUT in the status word, stops issuing and
// computing, drains its own TMA copies (bounded) and exits without trapping.
#pragma once

#include <cuda.h>
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
    int C, S, n_events, B;
    int64_t V;
    int D0, D1, D2, T0, T1, T2, n0, n1;
    const float *srcpos;
    const float4 *srcdir;
    const float *dstpos, *offsets, *weights;
    void *out;
    int64_t out_bstride;
    double beta_re;
    int beta_zero;
    int *status;
    int debug_drop_stage;  // test hook: the producer never fills the first stage
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

// Bounded wait: false when the CTA aborted or the clock budget ran out.
__device__ __forceinline__ bool bounded_wait(uint32_t bar, uint32_t parity, volatile int *abort, int *status) {
    if (*abort) return false;
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    for (uint32_t i = 1;; i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 31) == 0) {
            if (*abort) return false;
            if (clock64() - t0 > kWaitCycles) {
                *abort = 1;
                atomicExch(status, kStatusTimeout);
                return false;
            }
            __nanosleep(64);
        }
    }
}

template <int K> struct staged_traits {
    using st = typename pair_traits<K>::storage;
    static constexpr int bytes = sizeof(st);
    static constexpr int align_pairs = 16 / bytes;     // TMA x coordinate granularity
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

// Meta value of a window that holds no data: with it, no tap whose delay is
// finite and below 2^22 in magnitude -- and no larger or non-finite delay --
// yields an index inside the slot, so every tap reads the zero pair.
constexpr uint32_t kZeroWindow = kFloorMagicBits + 0x40000000u;

template <int WB, int K>
constexpr size_t staged_smem_bytes() {
    return slot_geom<WB, K>::ring_bytes + kStages * kStWin * 4 + kStages * 4 + 2 * kStages * 8 + 64 * 4 + 32 * 4 +
           kStWarps * 16 * 2 * 4 + kStages * kStWin * 2 * 16 + 128;
}

// Interpolate one tap from a staged slot and return it (f32 accumulation).
template <int K>
__device__ __forceinline__ float staged_tap(const unsigned char *slot, uint32_t rel, float t) {
    using st = typename pair_traits<K>::storage;
    return pair_traits<K>::tap(*reinterpret_cast<const st *>(slot + rel * sizeof(st)), t);
}

template <int K, int SC, int WB>
__global__ void __launch_bounds__(kStThreads) das_staged_kernel(const staged_params p,
                                                                 const __grid_constant__ CUtensorMap tmap) {
    using tr = pair_traits<K>;
    using st = typename tr::storage;
    using SG = slot_geom<WB, K>;
    constexpr int CC = kStWin / SC;  // channels per stage
    static_assert(kStWin % SC == 0, "SC must divide the stage");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char *ring = smem_raw;
    uint32_t *meta = reinterpret_cast<uint32_t *>(ring + SG::ring_bytes);    // [kStages][kStWin]
    int *ovf = reinterpret_cast<int *>(meta + kStages * kStWin);             // [kStages]
    uint64_t *full = reinterpret_cast<uint64_t *>(ovf + kStages);            // [kStages]
    uint64_t *empty = full + kStages;                                        // [kStages]
    float *aabb = reinterpret_cast<float *>(empty + kStages);                // [6] (+pad)
    float *ofs_lo = aabb + 8;                                                // [16]
    float *ofs_hi = ofs_lo + 16;                                             // [16]
    volatile int *abort_flag = reinterpret_cast<volatile int *>(ofs_hi + 16);
    float *red = const_cast<float *>(reinterpret_cast<volatile float *>(abort_flag + 32));  // [warps][16][2]
    float4 *chan_pos = reinterpret_cast<float4 *>(red + kStWarps * 32);                    // [kStages][kStWin]
    float4 *chan_dir = chan_pos + kStages * kStWin;                                        // [kStages][kStWin]

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const bool producer = (warp == kStWarps);
    const int b = blockIdx.y;

    // ---- voxel of this consumer thread ----
    const int tile = blockIdx.x;
    const int t0 = tile % p.n0, t1 = (tile / p.n0) % p.n1, t2 = tile / (p.n0 * p.n1);
    bool active = false;
    int64_t v = 0;
    float vx = 0.f, vy = 0.f, vz = 0.f;
    if (!producer) {
        const int i0 = tid % p.T0, i1 = (tid / p.T0) % p.T1, i2 = tid / (p.T0 * p.T1);
        const int g0 = t0 * p.T0 + i0, g1 = t1 * p.T1 + i1, g2 = t2 * p.T2 + i2;
        active = (g0 < p.D0 && g1 < p.D1 && g2 < p.D2);
        if (active) {
            v = ((int64_t)g2 * p.D1 + g1) * p.D0 + g0;
            vx = __ldg(p.dstpos + 3 * v);
            vy = __ldg(p.dstpos + 3 * v + 1);
            vz = __ldg(p.dstpos + 3 * v + 2);
        }
    }

    // ---- init: barriers, zero regions, abort flag ----
    if (tid == 0) {
        for (int i = 0; i < kStages; i++) {
            mbar_init(smem_u32(&full[i]), 1);
            mbar_init(smem_u32(&empty[i]), kStWarps);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    {
        constexpr int zwords = (SG::bytes - SG::data_bytes) / 4;
        for (int i = tid; i < kStages * kStWin * zwords; i += kStThreads) {
            const int slot = i / zwords, word = i - slot * zwords;
            reinterpret_cast<uint32_t *>(ring + slot * SG::bytes + SG::data_bytes)[word] = 0u;
        }
    }
    // ---- tile bounding box (consumers) ----
    if (!producer) {
        float mn[3] = {active ? vx : INFINITY, active ? vy : INFINITY, active ? vz : INFINITY};
        float mx[3] = {active ? vx : -INFINITY, active ? vy : -INFINITY, active ? vz : -INFINITY};
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
            for (int a = 0; a < 3; a++) {
                mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
                mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
            }
        }
        if (lane == 0) {
#pragma unroll
            for (int a = 0; a < 3; a++) {
                red[(warp * 16 + a) * 2] = mn[a];
                red[(warp * 16 + a) * 2 + 1] = mx[a];
            }
        }
    }
    __syncthreads();
    if (tid < 3) {
        float mn = INFINITY, mx = -INFINITY;
        for (int w = 0; w < kStWarps; w++) {
            mn = fminf(mn, red[(w * 16 + tid) * 2]);
            mx = fmaxf(mx, red[(w * 16 + tid) * 2 + 1]);
        }
        aabb[tid] = mn;
        aabb[3 + tid] = mx;
    }
    __syncthreads();

    const st *__restrict__ Pg = static_cast<const st *>(p.P);
    const uint32_t kmax_pair = (uint32_t)(p.npad - 1);
    float acc = 0.f;
    float2 acc2 = make_float2(0.f, 0.f);  // packed partial sums (even / odd event)
    int stage = 0;
    uint32_t phase = 0;
    bool dead = false;
    uint32_t issued_mask = 0;  // producer: stages whose copies may still be in flight

    for (int e0 = 0; e0 < p.n_events; e0 += SC) {
        const int sc = min(SC, p.n_events - e0);
        float ofs[SC], w[SC];
        // ---- per-event delay range of the tile (consumers) ----
        if (!producer) {
#pragma unroll
            for (int j = 0; j < SC; j++) {
                ofs[j] = 1e30f;
                w[j] = 0.f;
                if (active && j < sc) {
                    const int64_t idx = (int64_t)(e0 + j) * p.V + v;
                    ofs[j] = __ldg(p.offsets + idx);
                    w[j] = __ldg(p.weights + idx);
                }
            }
#pragma unroll
            for (int j = 0; j < SC; j++) {
                const bool ok = active && j < sc && isfinite(ofs[j]);
                float lo = ok ? ofs[j] : INFINITY, hi = ok ? ofs[j] : -INFINITY;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
                }
                if (lane == 0) {
                    red[(warp * 16 + j) * 2] = lo;
                    red[(warp * 16 + j) * 2 + 1] = hi;
                }
            }
            asm volatile("bar.sync 1, %0;" ::"r"(kStConsumers) : "memory");
            if (tid < SC) {
                float lo = INFINITY, hi = -INFINITY;
                for (int ww = 0; ww < kStWarps; ww++) {
                    lo = fminf(lo, red[(ww * 16 + tid) * 2]);
                    hi = fmaxf(hi, red[(ww * 16 + tid) * 2 + 1]);
                }
                ofs_lo[tid] = lo;
                ofs_hi[tid] = hi;
            }
        }
        __syncthreads();

        for (int c0 = 0; c0 < p.C; c0 += CC) {
            const uint32_t full_bar = smem_u32(&full[stage]);
            const uint32_t empty_bar = smem_u32(&empty[stage]);
            unsigned char *stage_base = ring + stage * SG::stage_bytes;
            if (producer) {
                // ---- stage the windows of CC channels x SC events ----
                if (!dead && !bounded_wait(empty_bar, phase ^ 1u, abort_flag, p.status)) dead = true;
                // Test hook: leave the very first stage unfilled (no copy, no
                // arrival) so the consumers' bounded waits must expire.
                const bool drop = p.debug_drop_stage && e0 == 0 && c0 == 0;
                if (drop) dead = true;
                bool issued = false, overflow = false;
                if (!dead) {
                    const int cl = lane / SC, j = lane % SC;
                    const int c = c0 + cl;
                    uint32_t m = kZeroWindow;  // every tap index clamps to the zero pair
                    float cx = 0.f, cy = 0.f, cz = 0.f;
                    if (c < p.C) {
                        cx = __ldg(p.srcpos + 3 * c);
                        cy = __ldg(p.srcpos + 3 * c + 1);
                        cz = __ldg(p.srcpos + 3 * c + 2);
                    }
                    if (j == 0) {
                        // channel table of the stage, read by the consumers
                        chan_pos[stage * kStWin + cl] = make_float4(cx, cy, cz, 0.f);
                        if (p.srcdir)
                            chan_dir[stage * kStWin + cl] = (c < p.C) ? __ldg(p.srcdir + c) : make_float4(0, 0, 0, 2.f);
                    }
                    if (c < p.C && j < sc) {
                        const float dx = fmaxf(fmaxf(aabb[0] - cx, cx - aabb[3]), 0.f);
                        const float dy = fmaxf(fmaxf(aabb[1] - cy, cy - aabb[4]), 0.f);
                        const float dz = fmaxf(fmaxf(aabb[2] - cz, cz - aabb[5]), 0.f);
                        const float ex = fmaxf(fabsf(cx - aabb[0]), fabsf(cx - aabb[3]));
                        const float ey = fmaxf(fabsf(cy - aabb[1]), fabsf(cy - aabb[4]));
                        const float ez = fmaxf(fabsf(cz - aabb[2]), fabsf(cz - aabb[5]));
                        const float rmin = sqrtf(dx * dx + dy * dy + dz * dz);
                        const float rmax = sqrtf(ex * ex + ey * ey + ez * ez);
                        const float lo = floorf(ofs_lo[j] + rmin) - 2.f;
                        const float hi = floorf(ofs_hi[j] + rmax) + 2.f;
                        // a window that misses the pair row entirely stays a zero window
                        if (lo == lo && hi == hi && hi >= 0.f && lo < (float)p.npad) {
                            const int k0 = ((int)fmaxf(lo, -(float)WB)) & ~(staged_traits<K>::align_pairs - 1);
                            const int k1 = (int)fminf(hi, (float)p.npad + WB);
                            if (k1 - k0 + 1 <= WB) {
                                const int row = (b * p.C + c) * p.S + (e0 + j);
                                const uint32_t dst = smem_u32(stage_base + lane * SG::bytes);
                                tma_load_row(dst, &tmap, k0, row, full_bar);
                                m = kFloorMagicBits + (uint32_t)k0;
                                issued = true;
                            } else {
                                m = kOvf;
                                overflow = true;
                            }
                        }
                    }
                    meta[stage * kStWin + lane] = m;
                }
                const unsigned issued_ballot = __ballot_sync(0xffffffffu, issued);
                const unsigned ovf_ballot = __ballot_sync(0xffffffffu, overflow);
                __syncwarp();
                if (lane == 0 && !drop) {
                    ovf[stage] = ovf_ballot != 0u;
                    // the producer's arrive also publishes meta/ovf (release)
                    mbar_arrive_expect_tx(full_bar, (uint32_t)__popc(issued_ballot) * (uint32_t)(WB * sizeof(st)));
                }
                if (!dead) issued_mask |= (1u << stage);
            } else {
                // ---- consume: CC channels x SC events from shared memory ----
                if (!dead && !bounded_wait(full_bar, phase, abort_flag, p.status)) dead = true;
                if (!dead) {
                    const bool any_ovf = ovf[stage] != 0;
                    for (int cl = 0; cl < CC; cl++) {
                        const int c = c0 + cl;
                        if (c >= p.C) break;
                        const float4 cp = chan_pos[stage * kStWin + cl];
                        recv_geom g = receive_geometry(vx, vy, vz, cp.x, cp.y, cp.z);
                        if (p.srcdir)
                            apply_directivity(g, vx, vy, vz, cp.x, cp.y, cp.z, chan_dir[stage * kStWin + cl]);
                        uint32_t k0p[SC];
#pragma unroll
                        for (int j = 0; j < SC; j += 4) {
                            if constexpr (SC >= 4) {
                                const uint4 q = *reinterpret_cast<const uint4 *>(&meta[stage * kStWin + cl * SC + j]);
                                k0p[j] = q.x; k0p[j + 1] = q.y; k0p[j + 2] = q.z; k0p[j + 3] = q.w;
                            } else {
#pragma unroll
                                for (int q = 0; q < SC; q++) k0p[q] = meta[stage * kStWin + cl * SC + q];
                            }
                        }
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
                                    const float2 tau2 = __ffma2_rn(rsq2, rinv2, make_float2(ofs[j], ofs[j + 1]));
                                    const float2 mm2 = __fadd2_rd(tau2, magic2);
                                    const float2 nfl2 = __ffma2_rn(mm2, neg1, magic2);   // -(floor), exact
                                    const float2 t2 = __fadd2_rn(tau2, nfl2);
                                    const uint32_t ra = min(__float_as_uint(mm2.x) - k0p[j], (uint32_t)WB);
                                    const uint32_t rb = min(__float_as_uint(mm2.y) - k0p[j + 1], (uint32_t)WB);
                                    const float ta = staged_tap<K>(slots + j * SG::bytes, ra, t2.x);
                                    const float tb = staged_tap<K>(slots + (j + 1) * SG::bytes, rb, t2.y);
                                    acc2 = __ffma2_rn(make_float2(w[j], w[j + 1]), make_float2(ta, tb), acc2);
                                }
                            } else {
#pragma unroll
                                for (int j = 0; j < SC; j++) {
                                    const float tau = __fmaf_rn(g.rsq, g.rinv, ofs[j]);
                                    const float mm = __fadd_rd(tau, kFloorMagic);
                                    const float t = tau - (mm - kFloorMagic);
                                    const uint32_t rel = min(__float_as_uint(mm) - k0p[j], (uint32_t)WB);
                                    acc = __fmaf_rn(w[j], staged_tap<K>(slots + j * SG::bytes, rel, t), acc);
                                }
                            }
                        } else {
#pragma unroll
                            for (int j = 0; j < SC; j++) {
                                const float tau = __fmaf_rn(g.rsq, g.rinv, ofs[j]);
                                const tau_split ts = split_tau(tau);
                                st pr;
                                if (k0p[j] == kOvf) {
                                    const int64_t row = ((int64_t)b * p.C + c) * p.S + (e0 + min(j, sc - 1));
                                    pr = Pg[row * p.npad + min(ts.k, kmax_pair)];
                                } else {
                                    const uint32_t rel = min(ts.k + kFloorMagicBits - k0p[j], (uint32_t)WB);
                                    pr = *reinterpret_cast<const st *>(slots + j * SG::bytes + rel * sizeof(st));
                                }
                                acc = __fmaf_rn(w[j], tr::tap(pr, ts.t), acc);
                            }
                        }
                    }
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(empty_bar);
            }
            if (++stage == kStages) {
                stage = 0;
                phase ^= 1u;
            }
        }
        __syncthreads();
    }

    if (producer) {
        // After an abort, wait (bounded, ignoring the abort flag) until every
        // copy this CTA issued has landed, so no TMA write outlives the CTA.
        if (*abort_flag && lane == 0) {
            for (int i = 0; i < kStages; i++) {
                const int s = (stage + i) % kStages;
                if (!(issued_mask & (1u << s))) continue;
                const uint32_t par = (s < stage) ? phase : (phase ^ 1u);
                const long long t0 = clock64();
                while (!mbar_try_wait(smem_u32(&full[s]), par) && clock64() - t0 < kWaitCycles) __nanosleep(64);
            }
        }
        return;
    }
    if (active && !dead) {
        acc += acc2.x + acc2.y;
        float *o = static_cast<float *>(p.out) + (int64_t)b * p.out_bstride + v;
        *o = p.beta_zero ? acc : __fmaf_rn((float)p.beta_re, *o, acc);
    }
}

}  // namespace ffdas
