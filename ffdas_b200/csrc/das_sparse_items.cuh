// das_sparse_items.cuh -- das_sparse as one persistent, load-balanced launch.
//
// The reference pads every voxel's event list to sparse_count and runs a flat
// grid over (voxel, padded slot) (src/das/das_alg1.cu:247-305,
// src/das/das_sparse_impl.cuh:38-45): a voxel with 2 real entries costs as
// much as one with 32.  Here the real entries drive the work:
//
//   1. sparse_bucket_kernel: per voxel, the entries with a nonzero weight and
//      an event inside x, sorted by event ([n][V] arrays), the number of them
//      before each pass of SC events ([passes + 1][V] bytes), and the tile's
//      total (its work).  A list naming one event twice sets the gate word, and
//      the call falls back to the gather kernel (launched after, idle otherwise).
//   2. sparse_order_kernel: one CTA sorts the tiles by work, longest first.
//   3. das_sparse_items_kernel: a persistent grid (CTAs resident on every SM)
//      pulls work items -- (tile, channel slice), longest tiles first -- from
//      a global counter until none is left.  Per item and pass, the 256
//      voxels of the tile are ordered by their entry count in the pass
//      (counting sort in shared memory), so a warp runs its voxels' entries up
//      to the warp's longest list and no further; each thread loads the
//      entries of the voxel it took.  The channel-sample windows of the pass's
//      events are staged into shared memory by the producer warp with TMA
//      (the ring and producer of the 512-voxel dense kernel), and a tap reads
//      its pair from there: per entry and channel one delay FFMA, the floor
//      split, one shared-memory bias load, one pair load and two FFMAs.
//
// The sum per voxel is that of the gather kernel over the same entries;
// only the order of the terms differs.
#pragma once

#include "das_staged.cuh"

namespace ffdas {

constexpr int kItemsTile = kStConsumers;   // voxels per tile, one per consumer thread
constexpr int kItemsMaxList = 64;          // longest list the bucket pass sorts

// ----------------------------------------------------------------- bucketing ---
struct bucket_params {
    const int *idx;
    const float *ofs, *w;
    int n, S, SC, passes;
    int64_t V;
    int D0, D1, T0, T1, T2, n0, n1;
    int *bs;            // [n][V] sorted events
    float *bo, *bw;     // [n][V] their delays and weights
    uint8_t *pstart;    // [passes + 1][V] entries before each pass
    int *tile_work;     // [tiles]
    int *gate;
};

__global__ void __launch_bounds__(128) sparse_bucket_kernel(const bucket_params p) {
    const int64_t v = (int64_t)blockIdx.x * 128 + threadIdx.x;
    if (v >= p.V) return;
    int ss[kItemsMaxList];
    float oo[kItemsMaxList], ww[kItemsMaxList];
    int cnt = 0;
    bool dup = false;
    for (int i = 0; i < p.n; i++) {
        const int64_t e = (int64_t)i * p.V + v;
        const int s = __ldg(p.idx + e);
        const float wt = __ldg(p.w + e);
        if ((unsigned)s >= (unsigned)p.S || wt == 0.f) continue;   // padding and events outside x add nothing
        const float o = __ldg(p.ofs + e);
        int k = cnt;   // insertion by event
        while (k > 0 && ss[k - 1] > s) {
            ss[k] = ss[k - 1];
            oo[k] = oo[k - 1];
            ww[k] = ww[k - 1];
            k--;
        }
        dup |= (k > 0 && ss[k - 1] == s);
        ss[k] = s;
        oo[k] = o;
        ww[k] = wt;
        cnt++;
    }
    for (int k = 0; k < cnt; k++) {
        p.bs[(int64_t)k * p.V + v] = ss[k];
        p.bo[(int64_t)k * p.V + v] = oo[k];
        p.bw[(int64_t)k * p.V + v] = ww[k];
    }
    int k = 0;
    for (int q = 0; q <= p.passes; q++) {
        const int lim = q * p.SC;
        while (k < cnt && ss[k] < lim) k++;
        p.pstart[(int64_t)q * p.V + v] = (uint8_t)k;
    }
    if (dup) atomicExch(p.gate, 1);
    const int g0 = (int)(v % p.D0), g1 = (int)((v / p.D0) % p.D1), g2 = (int)(v / ((int64_t)p.D0 * p.D1));
    const int tile = ((g2 / p.T2) * p.n1 + g1 / p.T1) * p.n0 + g0 / p.T0;
    if (cnt) atomicAdd(p.tile_work + tile, cnt);
}

// Tiles ordered by work, longest first: a 64-level counting sort in one CTA
// (the order within a level is whatever the atomics give; the sum of every
// voxel does not depend on it).
constexpr int kOrderLevels = 64;
__global__ void __launch_bounds__(1024) sparse_order_kernel(const int *__restrict__ work, int tiles,
                                                            int *__restrict__ order) {
    __shared__ int hist[kOrderLevels];
    __shared__ int wmax;
    const int tid = threadIdx.x;
    if (tid == 0) wmax = 0;
    if (tid < kOrderLevels) hist[tid] = 0;
    __syncthreads();
    int m = 0;
    for (int t = tid; t < tiles; t += blockDim.x) m = max(m, work[t]);
    atomicMax(&wmax, m);
    __syncthreads();
    const long long den = max(wmax, 1);
    for (int t = tid; t < tiles; t += blockDim.x)
        atomicAdd(&hist[(int)((long long)(wmax - work[t]) * (kOrderLevels - 1) / den)], 1);
    __syncthreads();
    if (tid < 32) {   // exclusive prefix over the 64 levels, two per lane
        const int a = hist[2 * tid], b = hist[2 * tid + 1];
        int incl = a + b;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (tid >= o) incl += y;
        }
        hist[2 * tid] = incl - a - b;
        hist[2 * tid + 1] = incl - b;
    }
    __syncthreads();
    for (int t = tid; t < tiles; t += blockDim.x)
        order[atomicAdd(&hist[(int)((long long)(wmax - work[t]) * (kOrderLevels - 1) / den)], 1)] = t;
}

// ------------------------------------------------------------ item kernel ---
struct items_params {
    const int *bs;
    const float *bo, *bw;
    const uint8_t *pstart;
    int n;                 // list length (entries per voxel in the bucket arrays)
    const int *order;      // tiles, longest first
    int tiles, slices;     // work items = tiles * slices
    int *queue;            // work-item counter (zeroed before the launch)
};

template <int K, int SC, int WB>
__global__ void __launch_bounds__(kStThreads, 2) das_sparse_items_kernel(const staged_params p, const items_params q,
                                                                         const __grid_constant__ CUtensorMap tmap) {
    using st = typename pair_traits<K>::storage;
    using SG = slot_geom<WB, K>;
    constexpr int CC = kStWin / SC;
    constexpr uint32_t PB = (uint32_t)sizeof(st);
    static_assert(kStWin % SC == 0 && SC <= 16, "SC must divide the stage");

    if (p.gate && *(volatile const int *)p.gate) return;   // doubly listed event: the gather kernel runs
    extern __shared__ __align__(128) unsigned char smem_raw[];
    staged_smem<K, WB> sm(smem_raw);
    // per-item scratch after the shared layout: voxel order, count histogram,
    // per-voxel sums
    short *vorder = reinterpret_cast<short *>(sm.extra);          // [256]
    int *hist = reinterpret_cast<int *>(vorder + kItemsTile);       // [SC + 1]
    float *acc_s = reinterpret_cast<float *>(hist + 32);            // [256]
    int *work = reinterpret_cast<int *>(acc_s + kItemsTile);        // [2]: current work item

    staged_ctx cx;
    cx.tid = threadIdx.x;
    cx.warp = cx.tid >> 5;
    cx.lane = cx.tid & 31;
    cx.producer = (cx.warp == kStWarps);
    cx.b = blockIdx.y;
    cx.active2 = false;
    cx.v2 = 0;
    cx.vx2 = cx.vy2 = cx.vz2 = 0.f;
    cx.par = 0;

    if (cx.tid == 0) {
        for (int i = 0; i < kStages; i++) {
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

    const st *__restrict__ Pg = static_cast<const st *>(p.P);
    const uint32_t kmax_pair = (uint32_t)(p.npad - 1);
    const uint32_t ring_u32 = smem_u32(sm.ring);
    int stage = 0;
    uint32_t phase = 0;
    bool dead = false;
    uint32_t issued_mask = 0;
    int pass_no = 0;   // passes run by this CTA (pass-flag parity)

    for (;;) {
        if (cx.tid == 0) work[0] = atomicAdd(q.queue + cx.b, 1);   // one queue per batch item
        __syncthreads();
        const int wi = work[0];
        if (wi >= q.tiles * q.slices || *sm.abort_flag) break;   // uniform: read after the barrier
        const int tile = q.order[wi / q.slices], slice = wi - (wi / q.slices) * q.slices;
        const int cbeg = p.cchunk ? slice * p.cchunk : 0;
        const int cend = p.cchunk ? min(p.C, cbeg + p.cchunk) : p.C;

        // ---- the tile: this thread's voxel, the tile box, the channel box
        const int t0 = tile % p.n0, t1 = (tile / p.n0) % p.n1, t2 = tile / (p.n0 * p.n1);
        cx.active = false;
        cx.v = 0;
        cx.vx = cx.vy = cx.vz = 0.f;
        if (!cx.producer) {
            const int i0 = cx.tid % p.T0, i1 = (cx.tid / p.T0) % p.T1, i2 = cx.tid / (p.T0 * p.T1);
            const int g0 = t0 * p.T0 + i0, g1 = t1 * p.T1 + i1, g2 = t2 * p.T2 + i2;
            cx.active = (g0 < p.D0 && g1 < p.D1 && g2 < p.D2);
            if (cx.active) {
                cx.v = ((int64_t)g2 * p.D1 + g1) * p.D0 + g0;
                cx.vx = __ldg(p.dstpos + 3 * cx.v);
                cx.vy = __ldg(p.dstpos + 3 * cx.v + 1);
                cx.vz = __ldg(p.dstpos + 3 * cx.v + 2);
            }
            acc_s[cx.tid] = 0.f;
            float mn[3] = {cx.active ? cx.vx : INFINITY, cx.active ? cx.vy : INFINITY, cx.active ? cx.vz : INFINITY};
            float mx[3] = {cx.active ? cx.vx : -INFINITY, cx.active ? cx.vy : -INFINITY, cx.active ? cx.vz : -INFINITY};
            float cmn[3] = {INFINITY, INFINITY, INFINITY}, cmx[3] = {-INFINITY, -INFINITY, -INFINITY};
            for (int c = cbeg + cx.tid; c < cend; c += kStConsumers) {
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const float pc = __ldg(p.srcpos + 3 * c + a);
                    cmn[a] = fminf(cmn[a], pc);
                    cmx[a] = fmaxf(cmx[a], pc);
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
                    mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
                    cmn[a] = fminf(cmn[a], __shfl_xor_sync(0xffffffffu, cmn[a], o));
                    cmx[a] = fmaxf(cmx[a], __shfl_xor_sync(0xffffffffu, cmx[a], o));
                }
            }
            if (cx.lane == 0) {
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    sm.red[(cx.warp * 16 + a) * 2] = mn[a];
                    sm.red[(cx.warp * 16 + a) * 2 + 1] = mx[a];
                    sm.red[(cx.warp * 16 + 3 + a) * 2] = cmn[a];
                    sm.red[(cx.warp * 16 + 3 + a) * 2 + 1] = cmx[a];
                }
            }
        }
        const bool vfin = cx.producer || !cx.active || (isfinite(cx.vx) && isfinite(cx.vy) && isfinite(cx.vz));
        const int all_vfin = __syncthreads_and(vfin);
        if (cx.tid < 6) {
            float mn = INFINITY, mx = -INFINITY;
            for (int w = 0; w < kStWarps; w++) {
                mn = fminf(mn, sm.red[(w * 16 + cx.tid) * 2]);
                mx = fmaxf(mx, sm.red[(w * 16 + cx.tid) * 2 + 1]);
            }
            if (cx.tid < 3) {
                sm.aabb[cx.tid] = mn;
                sm.aabb[3 + cx.tid] = mx;
            } else {
                sm.cbox[cx.tid - 3] = mn;
                sm.cbox[cx.tid] = mx;
            }
        }
        if (cx.tid == 0)   // channel positions finite <=> their box is (an infinite or NaN one is not)
            sm.flags[1] = all_vfin;
        __syncthreads();
        if (cx.tid == 0)
            sm.flags[1] = sm.flags[1] && isfinite(sm.cbox[0] + sm.cbox[1] + sm.cbox[2] + sm.cbox[3] + sm.cbox[4] +
                                                  sm.cbox[5]);

        for (int e0 = 0; e0 < p.S; e0 += SC) {
            const int sc = min(SC, p.S - e0);
            const int pidx = e0 / SC;
            // ---- entry counts of the pass, voxels ordered by them
            int m_own = 0;
            if (!cx.producer && cx.active)
                m_own = (int)__ldg(q.pstart + (int64_t)(pidx + 1) * p.V + cx.v) -
                        (int)__ldg(q.pstart + (int64_t)pidx * p.V + cx.v);
            if (cx.tid <= SC) hist[cx.tid] = 0;
            __syncthreads();
            int rank = 0;
            if (!cx.producer) rank = atomicAdd(&hist[m_own], 1);
            __syncthreads();
            if (cx.tid == 0) {
                int run = 0;
                for (int i = 0; i <= SC; i++) {
                    const int c = hist[i];
                    hist[i] = run;
                    run += c;
                }
            }
            __syncthreads();
            if (!cx.producer) vorder[hist[m_own] + rank] = (short)cx.tid;
            __syncthreads();

            // ---- this thread's voxel for the pass and its entries
            int m = 0, u = 0;
            int64_t vv = 0;
            float ux = 0.f, uy = 0.f, uz = 0.f;
            float eo[SC], ew[SC];
            int ej[SC];
#pragma unroll
            for (int i = 0; i < SC; i++) { eo[i] = 0.f; ew[i] = 0.f; ej[i] = 0; }
            bool bad = false;
            if (!cx.producer) {
                u = vorder[cx.tid];
                const int i0 = u % p.T0, i1 = (u / p.T0) % p.T1, i2 = u / (p.T0 * p.T1);
                const int g0 = t0 * p.T0 + i0, g1 = t1 * p.T1 + i1, g2 = t2 * p.T2 + i2;
                if (g0 < p.D0 && g1 < p.D1 && g2 < p.D2) {
                    vv = ((int64_t)g2 * p.D1 + g1) * p.D0 + g0;
                    const int k0 = __ldg(q.pstart + (int64_t)pidx * p.V + vv);
                    m = (int)__ldg(q.pstart + (int64_t)(pidx + 1) * p.V + vv) - k0;
                    ux = __ldg(p.dstpos + 3 * vv);
                    uy = __ldg(p.dstpos + 3 * vv + 1);
                    uz = __ldg(p.dstpos + 3 * vv + 2);
#pragma unroll
                    for (int i = 0; i < SC; i++) {
                        if (i < m) {
                            const int64_t e = (int64_t)(k0 + i) * p.V + vv;
                            ej[i] = __ldg(q.bs + e) - e0;
                            eo[i] = __ldg(q.bo + e);
                            ew[i] = __ldg(q.bw + e);
                            bad |= !isfinite(eo[i]);
                        }
                    }
                }
                // per-event delay range over the tile's entries of the pass
#pragma unroll
                for (int j = 0; j < SC; j++) {
                    float lo = INFINITY, hi = -INFINITY;
#pragma unroll
                    for (int i = 0; i < SC; i++) {
                        const bool ok = i < m && ej[i] == j && isfinite(eo[i]);
                        lo = fminf(lo, ok ? eo[i] : INFINITY);
                        hi = fmaxf(hi, ok ? eo[i] : -INFINITY);
                    }
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
                if (cx.lane == 0) sm.red[(cx.warp * 16 + 15) * 2 + 1] = bad ? 1.f : 0.f;
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
                    for (int ww = 0; ww < kStWarps; ww++) anybad |= sm.red[(ww * 16 + 15) * 2 + 1] != 0.f;
                    sm.flags[2 + (pass_no & 1)] = pass_flags(p, sm, sc, SC, anybad, true);
                }
            }
            __syncthreads();
            const int pflags = *(volatile int *)&sm.flags[2 + (pass_no & 1)];
            pass_no++;
            if (pflags & kPassSkip) continue;   // uniform: the ring is left as it is
            const bool pass_fast = (pflags & kPassFast) != 0;
            const int mw = __reduce_max_sync(0xffffffffu, (unsigned)m);   // the warp's longest list

            if (cx.producer) {
                staged_produce_pass2<K, WB, SC, true>(p, &tmap, sm, cx, stage, phase, e0, sc, dead, issued_mask,
                                                      cbeg, cend);
            } else {
                float acc = 0.f;
                for (int c0 = cbeg; c0 < cend; c0 += CC) {
                    const uint32_t full_bar = smem_u32(&sm.full[stage]);
                    if (!dead && !bounded_wait(full_bar, phase, sm.abort_flag, p.status)) dead = true;
                    const int mode = dead ? kStageEmpty : *(volatile int *)&sm.mode[stage];
                    if (!(mode & kStageEmpty) && mw > 0) {
                        const bool any_ovf = sm.ovf[stage] != 0;
                        const bool fast = pass_fast && (mode & kStageFast);
                        const uint32_t stage_u32 = ring_u32 + stage * SG::stage_bytes;
                        const int ncl = min(CC, cend - c0);   // channels past the slice add nothing
#pragma unroll 1
                        for (int cl = 0; cl < ncl; cl++) {
                            const float4 cp = sm.chan_pos[stage * kStWin + cl];
                            recv_geom g = receive_geometry(ux, uy, uz, cp.x, cp.y, cp.z);
                            if (p.srcdir) apply_directivity(g, ux, uy, uz, cp.x, cp.y, cp.z, sm.chan_dir[stage * kStWin + cl]);
                            const uint32_t meta_u32 = smem_u32(sm.meta + stage * kStWin + cl * SC);
                            const uint32_t bias_u32 = smem_u32(sm.bias + stage * kStWin + cl * SC);
                            if (fast) {
#pragma unroll
                                for (int i = 0; i < SC; i++) {
                                    if (i < mw) {
                                        if (i < m) {
                                            const float tau = __fmaf_rn(g.rsq, g.rinv, eo[i]);
                                            const float mm = __fadd_rd(tau, kFloorMagic);
                                            const float t = tau - (mm - kFloorMagic);
                                            const uint32_t a = __float_as_uint(mm) * PB + lds_u32(bias_u32 + 4 * ej[i]);
                                            acc = __fmaf_rn(ew[i], tap_at<K>(a, t), acc);
                                        }
                                    }
                                }
                            } else {
#pragma unroll
                                for (int i = 0; i < SC; i++) {
                                    if (i < mw && i < m) {
                                        const float tau = __fmaf_rn(g.rsq, g.rinv, eo[i]);
                                        const tau_split ts = split_tau(tau);
                                        const uint32_t k0 = lds_u32(meta_u32 + 4 * ej[i]);
                                        st pr;
                                        if (any_ovf && k0 == kOvf) {
                                            const int64_t row = ((int64_t)cx.b * p.C + c0 + cl) * p.S + (e0 + ej[i]);
                                            pr = Pg[row * p.npad + min(ts.k, kmax_pair)];
                                        } else {
                                            const uint32_t rel = min(ts.k + kFloorMagicBits - k0, (uint32_t)WB);
                                            pr = *reinterpret_cast<const st *>(
                                                sm.ring + stage * SG::stage_bytes + (cl * SC + ej[i]) * SG::bytes +
                                                rel * sizeof(st));
                                        }
                                        acc = __fmaf_rn(ew[i], pair_traits<K>::tap(pr, ts.t), acc);
                                    }
                                }
                            }
                        }
                        (void)stage_u32;
                    }
                    __syncwarp();
                    if (cx.lane == 0) mbar_arrive(smem_u32(&sm.empty[stage]));
                    if (++stage == kStages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                acc_s[u] += acc;   // the thread owns voxel u for this pass
            }
            __syncthreads();
        }

        // ---- the tile's voxels out
        if (!cx.producer && cx.active && !dead) {
            float *o = static_cast<float *>(p.out) + (int64_t)cx.b * p.out_bstride + cx.v;
            const float acc = acc_s[cx.tid];
            if (p.cchunk) atomicAdd(o, acc);   // channel slices add into the prepared image
            else *o = p.beta_zero ? acc : __fmaf_rn((float)p.beta_re, *o, acc);
        }
        __syncthreads();
    }

    if (cx.producer) staged_drain<K, WB>(sm, cx, stage, phase, issued_mask);
}

template <int K, int WB>
constexpr size_t items_smem_bytes() {
    // shared layout, voxel order (short), count histogram, per-voxel sums, work word
    return staged_smem_bytes<WB, K>() + kItemsTile * 2 + 32 * 4 + kItemsTile * 4 + 16;
}

}  // namespace ffdas
