// das_bwd.cu -- ffdas_das_backward: adjoint of the delay-and-sum forward.
//
// For each unit (b, v, c, e) the forward adds w * L with
//   L = x0 + t d,  d = x1 - x0,  t = tau - floor(tau),  tau = ofs[e,v] + r(v,c)
// so, with g = dLoss/dout[b,v]:
//   dLoss/dweights[e,v] += g L
//   dLoss/doffsets[e,v] += g w d               (slope of the interpolant)
//   dLoss/ddstpos[v]    += g w d (v - c) / r
//   dLoss/dsrcpos[c]    -= g w d (v - c) / r
//   dLoss/dx[b,c,s,k]   += g w (1 - t),  dLoss/dx[b,c,s,k+1] += g w t
// One kernel recomputes (k, t) from the same pair rows the forward reads (no
// stored indices), keeps the per-voxel gradients in registers, and scatters
// the channel-data adjoint through a shared-memory window per (channel,
// event) that is flushed to global memory with one red.add per touched
// sample.  Voxel tiles are the forward's compact tiles, so a window covers
// only the few tens of samples the tile's voxels touch.
#include <algorithm>
#include <climits>
#include <cstring>

#include "core.h"
#include "das_problem.h"
#include "das_pairs.cuh"

namespace ffdas {

struct bwd_params {
    const void *P;
    int64_t npad;
    int C, S, N, n_events, B;
    int64_t V;
    int D0, D1, D2, T0, T1, T2, n0, n1;
    const float *srcpos, *dstpos, *offsets, *weights;
    const float4 *srcdir;       // element directivity (C x 4), or null
    const int *sparse_idx;
    const float *gout;          // (B, V) with batch stride gout_bstride
    int64_t gout_bstride;
    float *gx;                  // (B, C, S, N) contiguous
    float *goff, *gw, *gdst, *gsrc;
    int cchunk;                 // channels per blockIdx.z slice (0: no split)
};

constexpr int kBwdThreads = 256;
constexpr int kBwdWin = 128;   // samples per shared window (per event, per batch item)

template <int K, int BT, int SC, bool SPARSE>
__global__ void __launch_bounds__(kBwdThreads) das_bwd_kernel(const bwd_params p) {
    using tr = pair_traits<K>;
    using st = typename tr::storage;
    __shared__ float win[SC][BT][kBwdWin];
    __shared__ int kmin_s[SC], kmax_s[SC];

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int tile = blockIdx.x;
    const int t0 = tile % p.n0, t1 = (tile / p.n0) % p.n1, t2 = tile / (p.n0 * p.n1);
    // das_sparse without the weight gradient: the CTA orders its voxels by
    // list length (as the forward gather does) and each warp runs its events
    // only up to its longest real list.  Padding entries (zero weight) add
    // nothing to the other gradients; they do have a weight gradient (the
    // tap they would read), so with gw the walk covers every entry.
    int pos = tid, n_ev = p.n_events;
    if constexpr (SPARSE) {
        if (p.gw == nullptr) {
            __shared__ int Ls[kBwdThreads];
            int L;
            const int me = sparse_balance(p, tid, t0, t1, t2, L);
            Ls[tid] = L;
            __syncthreads();
            pos = me;
            n_ev = (int)__reduce_max_sync(0xffffffffu, (unsigned)Ls[me]);
        }
    }
    const int i0 = pos % p.T0, i1 = (pos / p.T0) % p.T1, i2 = pos / (p.T0 * p.T1);
    const int g0 = t0 * p.T0 + i0, g1 = t1 * p.T1 + i1, g2 = t2 * p.T2 + i2;
    const bool active = (g0 < p.D0 && g1 < p.D1 && g2 < p.D2);
    const int64_t v = active ? ((int64_t)g2 * p.D1 + g1) * p.D0 + g0 : 0;
    const int b0 = blockIdx.y * BT;
    const bool do_gx = p.gx != nullptr;
    // When several CTAs share a voxel (batch chunks, channel slices) they add
    // the voxel-side gradients with atomics into zeroed outputs; a single CTA
    // stores them directly.
    const bool multi_chunk = gridDim.y > 1 || gridDim.z > 1;
    const int cbeg = p.cchunk ? (int)blockIdx.z * p.cchunk : 0;
    const int cend = p.cchunk ? min(p.C, cbeg + p.cchunk) : p.C;

    for (int i = tid; i < SC * BT * kBwdWin; i += kBwdThreads) (&win[0][0][0])[i] = 0.f;
    if (tid < SC) { kmin_s[tid] = INT_MAX; kmax_s[tid] = INT_MIN; }
    __syncthreads();

    float vx = 0.f, vy = 0.f, vz = 0.f;
    if (active) {
        vx = __ldg(p.dstpos + 3 * v); vy = __ldg(p.dstpos + 3 * v + 1); vz = __ldg(p.dstpos + 3 * v + 2);
    }
    float g[BT];
#pragma unroll
    for (int b = 0; b < BT; b++)
        g[b] = (active && b0 + b < p.B) ? __ldg(p.gout + (int64_t)(b0 + b) * p.gout_bstride + v) : 0.f;

    const st *__restrict__ P = static_cast<const st *>(p.P);
    const uint32_t kmax_pair = (uint32_t)(p.npad - 1);
    const int64_t row_b = (int64_t)p.C * p.S * p.npad;
    float gpx = 0.f, gpy = 0.f, gpz = 0.f;

    for (int e0 = 0; e0 < n_ev; e0 += SC) {
        const int sc = min(SC, n_ev - e0);
        float ofs[SC], w[SC], gwa[SC], goa[SC];
        int srow[SC];
#pragma unroll
        for (int j = 0; j < SC; j++) {
            gwa[j] = 0.f; goa[j] = 0.f;
            if (active && j < sc) {
                const int64_t idx = (int64_t)(e0 + j) * p.V + v;
                ofs[j] = __ldg(p.offsets + idx);
                w[j] = __ldg(p.weights + idx);
                int s = e0 + j;
                if constexpr (SPARSE) {
                    s = __ldg(p.sparse_idx + idx);
                    if ((unsigned)s >= (unsigned)p.S) { s = 0; w[j] = 0.f; ofs[j] = 1e30f; }
                }
                srow[j] = s;
            } else {
                ofs[j] = 1e30f; w[j] = 0.f; srow[j] = 0;
            }
        }

        for (int c = cbeg; c < cend; c++) {
            const float cx = __ldg(p.srcpos + 3 * c), cy = __ldg(p.srcpos + 3 * c + 1),
                        cz = __ldg(p.srcpos + 3 * c + 2);
            recv_geom gm = receive_geometry(vx, vy, vz, cx, cy, cz);
            // outside the element's directivity cone the tap leaves the
            // record, as in the forward: no contribution, no gradient
            if (p.srcdir) apply_directivity(gm, vx, vy, vz, cx, cy, cz, __ldg(p.srcdir + c));
            const st *Pc = P + (int64_t)c * p.S * p.npad;
            float q = 0.f;      // sum_j w_j sum_b g_b d_b  (for the position gradients)
            uint32_t kk[SC];
            float tt[SC];
#pragma unroll
            for (int j = 0; j < SC; j++) {
                const float tau = __fmaf_rn(gm.rsq, gm.rinv, ofs[j]);
                const tau_split ts = split_tau(tau);
                kk[j] = ts.k;
                tt[j] = ts.t;
                if (j < sc) {
                    const uint32_t k = min(ts.k, kmax_pair);
                    const st *row = Pc + (int64_t)srow[j] * p.npad + k;
                    float gl = 0.f, gd = 0.f;
#pragma unroll
                    for (int b = 0; b < BT; b++) {
                        if (b0 + b < p.B) {
                            const st pr = row[(int64_t)(b0 + b) * row_b];
                            const float L = tr::tap(pr, ts.t);
                            const float d = tr::slope(pr);
                            gl = __fmaf_rn(g[b], L, gl);
                            gd = __fmaf_rn(g[b], d, gd);
                        }
                    }
                    gwa[j] += gl;
                    goa[j] = __fmaf_rn(w[j], gd, goa[j]);
                    q = __fmaf_rn(w[j], gd, q);
                }
            }
            // position gradients: d r / d v = (v - c) / r
            const float qr = q * gm.rinv;
            const float ex = (vx - cx) * qr, ey = (vy - cy) * qr, ez = (vz - cz) * qr;
            gpx += ex; gpy += ey; gpz += ez;
            if (p.gsrc) {
                float sx = -ex, sy = -ey, sz = -ez;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    sx += __shfl_xor_sync(0xffffffffu, sx, o);
                    sy += __shfl_xor_sync(0xffffffffu, sy, o);
                    sz += __shfl_xor_sync(0xffffffffu, sz, o);
                }
                if (lane == 0 && (sx != 0.f || sy != 0.f || sz != 0.f)) {
                    atomicAdd(p.gsrc + 3 * c, sx);
                    atomicAdd(p.gsrc + 3 * c + 1, sy);
                    atomicAdd(p.gsrc + 3 * c + 2, sz);
                }
            }
            if (!do_gx) continue;

            // ---- channel-data adjoint: two-tap scatter ----
            if constexpr (SPARSE) {
                // event rows differ per voxel: scatter straight to global memory
#pragma unroll
                for (int j = 0; j < SC; j++) {
                    if (j < sc && kk[j] < (uint32_t)(p.N - 1) && w[j] != 0.f) {
#pragma unroll
                        for (int b = 0; b < BT; b++) {
                            if (b0 + b < p.B && g[b] != 0.f) {
                                float *gr = p.gx + (((int64_t)(b0 + b) * p.C + c) * p.S + srow[j]) * p.N + kk[j];
                                const float a = g[b] * w[j];
                                atomicAdd(gr, a - a * tt[j]);
                                atomicAdd(gr + 1, a * tt[j]);
                            }
                        }
                    }
                }
            } else {
#pragma unroll
                for (int j = 0; j < SC; j++) {
                    const bool valid = active && j < sc && kk[j] < (uint32_t)(p.N - 1);
                    int lo = valid ? (int)kk[j] : INT_MAX;
                    int hi = valid ? (int)kk[j] : INT_MIN;
                    lo = __reduce_min_sync(0xffffffffu, lo);
                    hi = __reduce_max_sync(0xffffffffu, hi);
                    if (lane == 0 && lo != INT_MAX) {
                        atomicMin(&kmin_s[j], lo);
                        atomicMax(&kmax_s[j], hi);
                    }
                }
                __syncthreads();
#pragma unroll
                for (int j = 0; j < SC; j++) {
                    const bool valid = active && j < sc && kk[j] < (uint32_t)(p.N - 1) && w[j] != 0.f;
                    if (!valid) continue;
                    const int base = kmin_s[j];
                    const bool fits = (kmax_s[j] - base + 2) <= kBwdWin;
                    const int rel = (int)kk[j] - base;
#pragma unroll
                    for (int b = 0; b < BT; b++) {
                        if (b0 + b < p.B) {
                            const float a = g[b] * w[j];
                            const float a1 = a * tt[j];
                            if (fits) {
                                atomicAdd(&win[j][b][rel], a - a1);
                                atomicAdd(&win[j][b][rel + 1], a1);
                            } else {
                                float *gr = p.gx + (((int64_t)(b0 + b) * p.C + c) * p.S + (e0 + j)) * p.N + kk[j];
                                atomicAdd(gr, a - a1);
                                atomicAdd(gr + 1, a1);
                            }
                        }
                    }
                }
                __syncthreads();
                // flush the windows
                for (int j = 0; j < sc; j++) {
                    const int base = kmin_s[j];
                    if (base == INT_MAX) continue;
                    const int wlen = kmax_s[j] - base + 2;
                    if (wlen > kBwdWin) continue;
                    for (int i = tid; i < BT * wlen; i += kBwdThreads) {
                        const int b = i / wlen, r = i - b * wlen;
                        const float val = win[j][b][r];
                        if (val != 0.f) {
                            win[j][b][r] = 0.f;
                            atomicAdd(p.gx + (((int64_t)(b0 + b) * p.C + c) * p.S + (e0 + j)) * p.N + base + r, val);
                        }
                    }
                }
                __syncthreads();
                if (tid < SC) { kmin_s[tid] = INT_MAX; kmax_s[tid] = INT_MIN; }
            }
        }
        if (active) {
#pragma unroll
            for (int j = 0; j < SC; j++) {
                if (j < sc) {
                    const int64_t idx = (int64_t)(e0 + j) * p.V + v;
                    if (multi_chunk) {
                        if (p.gw) atomicAdd(p.gw + idx, gwa[j]);
                        if (p.goff) atomicAdd(p.goff + idx, goa[j]);
                    } else {
                        if (p.gw) p.gw[idx] = gwa[j];
                        if (p.goff) p.goff[idx] = goa[j];
                    }
                }
            }
        }
    }
    if (active && p.gdst) {
        if (multi_chunk) {
            atomicAdd(p.gdst + 3 * v, gpx); atomicAdd(p.gdst + 3 * v + 1, gpy); atomicAdd(p.gdst + 3 * v + 2, gpz);
        } else {
            p.gdst[3 * v] = gpx; p.gdst[3 * v + 1] = gpy; p.gdst[3 * v + 2] = gpz;
        }
    }
}

template <int K, int BT, bool SPARSE>
static ffdas_error_t launch_bwd_t(ffdas_context &h, const bwd_params &bp, dim3 grid) {
    das_bwd_kernel<K, BT, 8, SPARSE><<<grid, kBwdThreads, 0, h.stream>>>(bp);
    return ffdas_launch_check(h.stream);
}

template <int K, bool SPARSE>
static ffdas_error_t launch_bwd_k(ffdas_context &h, const bwd_params &bp, int BT, dim3 grid) {
    switch (BT) {
        case 1: return launch_bwd_t<K, 1, SPARSE>(h, bp, grid);
        case 2: return launch_bwd_t<K, 2, SPARSE>(h, bp, grid);
        default: return launch_bwd_t<K, 4, SPARSE>(h, bp, grid);
    }
}

// ------------------------------------------------ complex (IQ) adjoint ---
// The forward adds, per tap, A v with A = w (cos, sin)(wavenum tau) (the
// reference's weight, src/das/das_alg1_kernels.cuh:79-86) and v = x_k + t
// (x_{k+1} - x_k).  With g the output gradient (d loss / d Re + i d loss /
// d Im, the convention of complex autograd): x_k gets (1 - t) conj(A) g and
// x_{k+1} gets t conj(A) g; the weight Re(conj(g) (cos, sin) v); the delay
// Re(conj(g) A (i wavenum v + d)), d = x_{k+1} - x_k, which the positions
// take through d tau / d v = (v - c) / r.  A thread per voxel walks its
// events and the channels of its slice (blockIdx.y; slices add the
// voxel-side gradients with atomics into zeroed outputs), as the forward
// gather does; the channel-data gradient goes to global memory with one
// float2 atomic per sample, the channel positions take a warp sum per
// channel.
template <int K>
__device__ __forceinline__ float2 pair_slope_c(const typename pair_traits<K>::storage &pr);
template <> __device__ __forceinline__ float2 pair_slope_c<ST_C32>(const float4 &pr) {
    return make_float2(pr.z, pr.w);
}
template <> __device__ __forceinline__ float2 pair_slope_c<ST_C16>(const uint2 &pr) {
    uint2 q = pr;
    const float2 a = __half22float2(*reinterpret_cast<__half2 *>(&q.x));
    const float2 b = __half22float2(*reinterpret_cast<__half2 *>(&q.y));
    return make_float2(b.x - a.x, b.y - a.y);
}

template <int K, bool SPARSE>
__global__ void __launch_bounds__(kBwdThreads) das_bwd_complex_kernel(const bwd_params p, float wavenum) {
    using tr = pair_traits<K>;
    using st = typename tr::storage;
    const int lane = threadIdx.x & 31;
    const int64_t v = (int64_t)blockIdx.x * kBwdThreads + threadIdx.x;
    const bool active = v < p.V;
    const float2 *gout = reinterpret_cast<const float2 *>(p.gout);
    float2 *gx = reinterpret_cast<float2 *>(p.gx);
    float vx = 0.f, vy = 0.f, vz = 0.f;
    if (active) {
        vx = __ldg(p.dstpos + 3 * v); vy = __ldg(p.dstpos + 3 * v + 1); vz = __ldg(p.dstpos + 3 * v + 2);
    }
    const st *__restrict__ P = static_cast<const st *>(p.P);
    const uint32_t kmax_pair = (uint32_t)(p.npad - 1);
    const int64_t row_b = (int64_t)p.C * p.S * p.npad;
    float gpx = 0.f, gpy = 0.f, gpz = 0.f;
    const bool multi = gridDim.y > 1;
    const int cbeg = p.cchunk ? (int)blockIdx.y * p.cchunk : 0;
    const int cend = p.cchunk ? min(p.C, cbeg + p.cchunk) : p.C;
    for (int e = 0; e < p.n_events; e++) {
        float ofs = 1e30f, w = 0.f;
        int s = 0;
        if (active) {
            const int64_t idx = (int64_t)e * p.V + v;
            ofs = __ldg(p.offsets + idx);
            w = __ldg(p.weights + idx);
            s = e;
            if constexpr (SPARSE) {
                s = __ldg(p.sparse_idx + idx);
                if ((unsigned)s >= (unsigned)p.S) { s = 0; w = 0.f; ofs = 1e30f; }
            }
        }
        float gwa = 0.f, goa = 0.f;
        for (int c = cbeg; c < cend; c++) {
            const float cx = __ldg(p.srcpos + 3 * c), cy = __ldg(p.srcpos + 3 * c + 1),
                        cz = __ldg(p.srcpos + 3 * c + 2);
            recv_geom gm = receive_geometry(vx, vy, vz, cx, cy, cz);
            if (p.srcdir) apply_directivity(gm, vx, vy, vz, cx, cy, cz, __ldg(p.srcdir + c));
            const float tau = __fmaf_rn(gm.rsq, gm.rinv, ofs);
            const tau_split ts = split_tau(tau);
            float sn, cs;
            __sincosf(wavenum * tau, &sn, &cs);
            const float2 A = make_float2(cs * w, sn * w);
            const st *row = P + ((int64_t)c * p.S + s) * p.npad + min(ts.k, kmax_pair);
            const bool in_record = active && ts.k < (uint32_t)(p.N - 1);
            float q = 0.f;
            for (int b = 0; b < p.B; b++) {
                const float2 g = active ? gout[(int64_t)b * p.gout_bstride + v] : make_float2(0.f, 0.f);
                const st pr = row[(int64_t)b * row_b];
                const float2 val = tr::tap(pr, ts.t);
                const float2 d = pair_slope_c<K>(pr);
                // Re(conj(g) (cos, sin) val)
                const float2 pv = make_float2(cs * val.x - sn * val.y, cs * val.y + sn * val.x);
                gwa += g.x * pv.x + g.y * pv.y;
                // Re(conj(g) A (i wavenum val + d))
                const float2 z = make_float2(d.x - wavenum * val.y, d.y + wavenum * val.x);
                const float2 Az = make_float2(A.x * z.x - A.y * z.y, A.x * z.y + A.y * z.x);
                q += g.x * Az.x + g.y * Az.y;
                if (gx && in_record && w != 0.f) {
                    // conj(A) g, split over the two samples
                    const float2 cg = make_float2(A.x * g.x + A.y * g.y, A.x * g.y - A.y * g.x);
                    float2 *gr = gx + ((int64_t)b * p.C + c) * (int64_t)p.S * p.N + (int64_t)s * p.N + ts.k;
                    // one 8-byte vector atomic per sample (global memory,
                    // compute capability 9.0 and up)
                    atomicAdd(gr, make_float2(cg.x - cg.x * ts.t, cg.y - cg.y * ts.t));
                    atomicAdd(gr + 1, make_float2(cg.x * ts.t, cg.y * ts.t));
                }
            }
            goa += q;
            const float qr = q * gm.rinv;
            const float ex = (vx - cx) * qr, ey = (vy - cy) * qr, ez = (vz - cz) * qr;
            gpx += ex; gpy += ey; gpz += ez;
            if (p.gsrc) {
                float sx = -ex, sy = -ey, sz = -ez;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    sx += __shfl_xor_sync(0xffffffffu, sx, o);
                    sy += __shfl_xor_sync(0xffffffffu, sy, o);
                    sz += __shfl_xor_sync(0xffffffffu, sz, o);
                }
                if (lane == 0 && (sx != 0.f || sy != 0.f || sz != 0.f)) {
                    atomicAdd(p.gsrc + 3 * c, sx);
                    atomicAdd(p.gsrc + 3 * c + 1, sy);
                    atomicAdd(p.gsrc + 3 * c + 2, sz);
                }
            }
        }
        if (active) {
            const int64_t idx = (int64_t)e * p.V + v;
            if (multi) {
                if (p.gw) atomicAdd(p.gw + idx, gwa);
                if (p.goff) atomicAdd(p.goff + idx, goa);
            } else {
                if (p.gw) p.gw[idx] = gwa;
                if (p.goff) p.goff[idx] = goa;
            }
        }
    }
    if (active && p.gdst) {
        if (multi) {
            atomicAdd(p.gdst + 3 * v, gpx); atomicAdd(p.gdst + 3 * v + 1, gpy); atomicAdd(p.gdst + 3 * v + 2, gpz);
        } else {
            p.gdst[3 * v] = gpx; p.gdst[3 * v + 1] = gpy; p.gdst[3 * v + 2] = gpz;
        }
    }
}

template <int K>
static ffdas_error_t launch_bwd_complex(ffdas_context &h, const bwd_params &bp, bool sparse, float wavenum,
                                       int64_t blocks, int slices) {
    const dim3 grid((unsigned)blocks, (unsigned)slices);
    if (sparse)
        das_bwd_complex_kernel<K, true><<<grid, kBwdThreads, 0, h.stream>>>(bp, wavenum);
    else
        das_bwd_complex_kernel<K, false><<<grid, kBwdThreads, 0, h.stream>>>(bp, wavenum);
    return ffdas_launch_check(h.stream);
}

// ---------------------------------------- das_sparse adjoint, sorted lists ---
// The gather adjoint above gives each lane a voxel and walks its list, so at
// a list slot the lanes of a warp name different events and the two-tap
// scatter of the channel-data gradient goes to up to 32 pair rows per warp
// reduction.  Here a lane takes one list entry instead: the CTA (a tile of
// up to 128 voxels) counts its entries per event in a shared histogram,
// scans the counts and places every entry in its event's bucket, so the
// lanes of a warp mostly share the event and their reductions land on one
// row at nearby samples.  No lane works on a padding entry (zero weight)
// unless the weight gradient is asked for, where its tap is the gradient.
// Per entry the lane sums over the channels, as the gather adjoint does per
// voxel: the weight gradient g L, the delay gradient g w d and the voxel
// position gradient g w d (v - c) / r; the channel positions take the warp's
// sum per channel.  The position gradients of a voxel's entries meet in
// shared memory.
constexpr int kBwsThreads = 256;
constexpr int kBwsMaxEvents = 4096;     // events of x (shared histogram)
constexpr int kBwsMaxSlots = 8192;      // tile voxels x list length (16-bit entry codes)
constexpr int kBwsMaxTile = 128;
constexpr size_t kBwsMaxSmem = 200 * 1024;   // dynamic shared memory the kernel may be launched with

constexpr int kBwsGroup = 8;                 // channels whose position gradients a warp sums at once
constexpr int kBwsUnroll = 4;                // channels whose pair loads are in flight together
constexpr int kBwsRed = 3 * kBwsGroup * 33;   // floats of a warp's staging tile (rows padded to 33)

size_t bws_smem_bytes(int TV, int L, int S, int CS) {   // CS: channels of one CTA
    return (size_t)TV * 16 + (size_t)TV * 4 * 2 + (size_t)TV * 12 + (size_t)(kBwsThreads / 32) * kBwsRed * 4 +
           (size_t)S * 4 + (size_t)CS * 12 + (size_t)TV * L * 2;
}

template <int K, bool POS>   // POS: voxel or channel position gradients wanted
__global__ void __launch_bounds__(kBwsThreads) das_bwd_sorted_kernel(const bwd_params p, int L) {
    using tr = pair_traits<K>;
    using st = typename tr::storage;
    extern __shared__ __align__(16) unsigned char bws_smem[];
    __shared__ int total;
    const int TV = p.T0 * p.T1 * p.T2;
    const int NE = TV * L;                                          // slot q = j * TV + vl
    float4 *vpos = reinterpret_cast<float4 *>(bws_smem);            // [TV] position, w = 1 on the grid
    int *vidx = reinterpret_cast<int *>(vpos + TV);                 // [TV] voxel index
    float *gvox = reinterpret_cast<float *>(vidx + TV);             // [TV] output gradient of the voxel
    float *gpos = gvox + TV;                                        // [TV][3] voxel position gradients
    float *gred = gpos + 3 * TV;                                    // [warps][kBwsRed] channel-gradient staging
    int *cnt = reinterpret_cast<int *>(gred + (kBwsThreads / 32) * kBwsRed);   // [S] counts, then cursors
    float *gch = reinterpret_cast<float *>(cnt + p.S);              // [CTA's channels][3] position gradients
    const int cbeg = p.cchunk ? (int)blockIdx.z * p.cchunk : 0;
    const int cend = p.cchunk ? min(p.C, cbeg + p.cchunk) : p.C;
    uint16_t *code = reinterpret_cast<uint16_t *>(gch + 3 * (cend - cbeg));   // [NE] sorted position -> slot
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int b = blockIdx.y;
    const bool multi_chunk = gridDim.y > 1 || gridDim.z > 1;
    const bool all_entries = p.gw != nullptr;   // padding entries have a weight gradient

    const int tile = blockIdx.x;
    const int t0 = tile % p.n0, t1 = (tile / p.n0) % p.n1, t2 = tile / (p.n0 * p.n1);
    for (int vl = tid; vl < TV; vl += kBwsThreads) {
        const int i0 = vl % p.T0, i1 = (vl / p.T0) % p.T1, i2 = vl / (p.T0 * p.T1);
        const int g0 = t0 * p.T0 + i0, g1 = t1 * p.T1 + i1, g2 = t2 * p.T2 + i2;
        float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
        int v = 0;
        float gv = 0.f;
        if (g0 < p.D0 && g1 < p.D1 && g2 < p.D2) {
            v = (g2 * p.D1 + g1) * p.D0 + g0;
            q = make_float4(__ldg(p.dstpos + 3 * (int64_t)v), __ldg(p.dstpos + 3 * (int64_t)v + 1),
                            __ldg(p.dstpos + 3 * (int64_t)v + 2), 1.f);
            gv = __ldg(p.gout + (int64_t)b * p.gout_bstride + v);
        }
        vpos[vl] = q;
        vidx[vl] = v;
        gvox[vl] = gv;
        gpos[3 * vl] = gpos[3 * vl + 1] = gpos[3 * vl + 2] = 0.f;
    }
    for (int e = tid; e < p.S; e += kBwsThreads) cnt[e] = 0;
    if (POS)
        for (int i = tid; i < 3 * (cend - cbeg); i += kBwsThreads) gch[i] = 0.f;
    __syncthreads();

    // entries that can have a gradient: on the grid, event in [0, S), and a
    // nonzero weight unless the weight gradient is wanted (an entry with an
    // event outside [0, S) reads the zero pair: every gradient is 0, which
    // the zeroed outputs already hold)
    auto entry = [&](int q, int &s) -> bool {
        const int j = q / TV, vl = q - j * TV;
        if (vpos[vl].w == 0.f) return false;
        const int64_t idx = (int64_t)j * p.V + vidx[vl];
        s = __ldg(p.sparse_idx + idx);
        return (unsigned)s < (unsigned)p.S && (all_entries || __ldg(p.weights + idx) != 0.f);
    };
    for (int q = tid; q < NE; q += kBwsThreads) {
        int s;
        if (entry(q, s)) atomicAdd(&cnt[s], 1);
    }
    __syncthreads();
    if (warp == 0) {   // bucket starts: each lane scans a contiguous run of events
        const int per = (p.S + 31) / 32;
        const int s0 = min(lane * per, p.S), s1 = min(s0 + per, p.S);
        int sum = 0;
        for (int e = s0; e < s1; e++) sum += cnt[e];
        int incl = sum;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += y;
        }
        int run = incl - sum;
        for (int e = s0; e < s1; e++) {
            const int c = cnt[e];
            cnt[e] = run;
            run += c;
        }
        if (lane == 31) total = incl;
    }
    __syncthreads();
    for (int q = tid; q < NE; q += kBwsThreads) {
        int s;
        if (entry(q, s)) code[atomicAdd(&cnt[s], 1)] = (uint16_t)q;
    }
    __syncthreads();

    const int E = total;
    const st *Pb = static_cast<const st *>(p.P) + (int64_t)b * p.C * p.S * p.npad;   // < 2^31 pairs per item
    const uint32_t kmax = (uint32_t)(p.npad - 1);
    const uint32_t cstride = (uint32_t)(p.S * p.npad);
    for (int e0 = warp * 32; e0 < E; e0 += kBwsThreads) {   // uniform per warp: lanes past E stay for the shuffles
        const int e = e0 + lane;
        const bool act = e < E;
        int vl = 0, s = 0;
        int64_t idx = 0;
        float ofs = 1e30f, w = 0.f, g = 0.f;
        float4 vp = make_float4(0.f, 0.f, 0.f, 0.f);
        if (act) {
            const int q = code[e];
            const int j = q / TV;
            vl = q - j * TV;
            idx = (int64_t)j * p.V + vidx[vl];
            ofs = __ldg(p.offsets + idx);
            w = __ldg(p.weights + idx);
            s = __ldg(p.sparse_idx + idx);
            g = gvox[vl];
            vp = vpos[vl];
        }
        const uint32_t row = (uint32_t)s * (uint32_t)p.npad;
        float *gxr = p.gx ? p.gx + ((int64_t)b * p.C * p.S + s) * p.N : nullptr;   // + (c S) N + k
        const float a = g * w;
        float gwa = 0.f, goa = 0.f, ex = 0.f, ey = 0.f, ez = 0.f;
        // the gradients of one channel from its pair, once loaded
        auto channel = [&](int c, float cx, float cy, float cz, float rinv, const tau_split &ts, const st &pr) {
            const float Lt = tr::tap(pr, ts.t);
            const float gd = g * tr::slope(pr);
            gwa = __fmaf_rn(g, Lt, gwa);
            goa = __fmaf_rn(w, gd, goa);
            if (POS) {
            const float qr = w * gd * rinv;
            const float dx = (vp.x - cx) * qr, dy = (vp.y - cy) * qr, dz = (vp.z - cz) * qr;
            ex += dx; ey += dy; ez += dz;
            if (p.gsrc) {
                // channel position gradients, summed over the warp's entries
                // through a staging tile: each lane writes its three terms of
                // up to 8 channels, then lane r sums row r (channel r / 3,
                // component r % 3) and adds it to the CTA's sum
                float *rw = gred + warp * kBwsRed;
                const int slot = (c - cbeg) % kBwsGroup;
                rw[(3 * slot) * 33 + lane] = -dx;
                rw[(3 * slot + 1) * 33 + lane] = -dy;
                rw[(3 * slot + 2) * 33 + lane] = -dz;
                if (slot == kBwsGroup - 1 || c == cend - 1) {   // uniform over the warp
                    __syncwarp();
                    if (lane < 3 * (slot + 1)) {
                        float sum = 0.f;
#pragma unroll 8
                        for (int i = 0; i < 32; i++) sum += rw[lane * 33 + i];
                        if (sum != 0.f) atomicAdd(gch + 3 * (c - slot - cbeg) + lane, sum);
                    }
                    __syncwarp();
                }
            }
            }
            // two-tap scatter of the channel-data gradient: the warp's lanes
            // mostly share the event, so these land in one row
            if (gxr && a != 0.f && ts.k < (uint32_t)(p.N - 1)) {
                float *gr = gxr + (int64_t)c * p.S * p.N + ts.k;
                const float a1 = a * ts.t;
                atomicAdd(gr, a - a1);
                atomicAdd(gr + 1, a1);
            }
        };
        // kBwsUnroll channels at a time: their pair loads are in flight together
        int c = cbeg;
        for (; c + kBwsUnroll <= cend; c += kBwsUnroll) {
            float cx[kBwsUnroll], cy[kBwsUnroll], cz[kBwsUnroll], ri[kBwsUnroll];
            tau_split ts[kBwsUnroll];
            st pr[kBwsUnroll];
#pragma unroll
            for (int u = 0; u < kBwsUnroll; u++) {
                cx[u] = __ldg(p.srcpos + 3 * (c + u));
                cy[u] = __ldg(p.srcpos + 3 * (c + u) + 1);
                cz[u] = __ldg(p.srcpos + 3 * (c + u) + 2);
                recv_geom gm = receive_geometry(vp.x, vp.y, vp.z, cx[u], cy[u], cz[u]);
                if (p.srcdir) apply_directivity(gm, vp.x, vp.y, vp.z, cx[u], cy[u], cz[u], __ldg(p.srcdir + c + u));
                ri[u] = gm.rinv;
                ts[u] = split_tau(__fmaf_rn(gm.rsq, gm.rinv, ofs));
                pr[u] = Pb[row + (uint32_t)(c + u) * cstride + min(ts[u].k, kmax)];
            }
#pragma unroll
            for (int u = 0; u < kBwsUnroll; u++) channel(c + u, cx[u], cy[u], cz[u], ri[u], ts[u], pr[u]);
        }
        for (; c < cend; c++) {
            const float cx = __ldg(p.srcpos + 3 * c), cy = __ldg(p.srcpos + 3 * c + 1),
                        cz = __ldg(p.srcpos + 3 * c + 2);
            recv_geom gm = receive_geometry(vp.x, vp.y, vp.z, cx, cy, cz);
            if (p.srcdir) apply_directivity(gm, vp.x, vp.y, vp.z, cx, cy, cz, __ldg(p.srcdir + c));
            const tau_split ts = split_tau(__fmaf_rn(gm.rsq, gm.rinv, ofs));
            channel(c, cx, cy, cz, gm.rinv, ts, Pb[row + (uint32_t)c * cstride + min(ts.k, kmax)]);
        }
        if (act) {
            if (multi_chunk) {
                if (p.gw) atomicAdd(p.gw + idx, gwa);
                if (p.goff) atomicAdd(p.goff + idx, goa);
            } else {
                if (p.gw) p.gw[idx] = gwa;
                if (p.goff) p.goff[idx] = goa;
            }
            if (POS && p.gdst) {
                atomicAdd(&gpos[3 * vl], ex);
                atomicAdd(&gpos[3 * vl + 1], ey);
                atomicAdd(&gpos[3 * vl + 2], ez);
            }
        }
    }
    if (POS) __syncthreads();
    if (POS && p.gsrc) {   // one global add per channel and component from each CTA
        for (int i = tid; i < 3 * (cend - cbeg); i += kBwsThreads)
            if (gch[i] != 0.f) atomicAdd(p.gsrc + 3 * cbeg + i, gch[i]);
    }
    if (POS && p.gdst) {
        for (int vl = tid; vl < TV; vl += kBwsThreads) {
            if (vpos[vl].w == 0.f) continue;
            float *o = p.gdst + 3 * (int64_t)vidx[vl];
            if (multi_chunk) {
                atomicAdd(o, gpos[3 * vl]); atomicAdd(o + 1, gpos[3 * vl + 1]); atomicAdd(o + 2, gpos[3 * vl + 2]);
            } else {
                o[0] = gpos[3 * vl]; o[1] = gpos[3 * vl + 1]; o[2] = gpos[3 * vl + 2];
            }
        }
    }
}

bool bws_supported(const das_problem &pb, int kind) {
    if (kind != ST_F32 && kind != ST_F16 && kind != ST_BF16) return false;
    const int64_t item_pairs = (int64_t)pb.C * pb.S * pair_row_length(pb.N);
    return pb.n_events >= 1 && pb.n_events <= kBwsMaxSlots / 32 && pb.S >= 1 && pb.S <= kBwsMaxEvents &&
           pb.V <= INT_MAX && (int64_t)pb.D0 * pb.D1 * pb.D2 <= INT_MAX && pb.B <= 65535 && item_pairs < INT_MAX;
}

template <int K, bool POS>
ffdas_error_t launch_bws_pos(ffdas_context &h, const bwd_params &bp, int L, dim3 grid, size_t smem) {
    if (ffdas_raise_smem_limit(reinterpret_cast<const void *>(das_bwd_sorted_kernel<K, POS>), h.device_id,
                               kBwsMaxSmem) != cudaSuccess)
        return FFDAS_ERROR_CUDA_RUNTIME;
    das_bwd_sorted_kernel<K, POS><<<grid, kBwsThreads, smem, h.stream>>>(bp, L);
    return ffdas_launch_check(h.stream);
}

template <int K>
ffdas_error_t launch_bws_t(ffdas_context &h, const bwd_params &bp, int L, dim3 grid, size_t smem) {
    return (bp.gdst || bp.gsrc) ? launch_bws_pos<K, true>(h, bp, L, grid, smem)
                                : launch_bws_pos<K, false>(h, bp, L, grid, smem);
}

// defined in das.cu
ffdas_error_t ingest_for_backward(ffdas_context &h, const das_problem &pb, ffdas_datatype_t xt, int kind,
                                  const void *x, int64_t npad, void *P);
void *reusable_pairs(const ffdas_context &h, const ffdas_tensor_desc &xd, const void *x, int kind);

ffdas_error_t das_backward(ffdas_context &h, const das_call &a, const ffdas_tensor_desc &gd,
                           const void *gout, float *gx, float *goff, float *gw, float *gdst, float *gsrc) {
    const ffdas_tensor_desc &xd = *a.x_desc;
    // real data without phase rotation, or complex data (complex64 or
    // complex32 pairs) with any wavenum and a complex64 output gradient;
    // directivity (a mask per element and voxel) is applied as in the forward
    // the adjoint of a channel-scaled forward is not provided: clear the scale
    if (h.chan_scale) return FFDAS_ERROR_INVALID_ARGUMENT;
    const bool cplx = xd.dtype == FFDAS_C_32F || xd.dtype == FFDAS_C_16F;
    if (gd.dtype != (cplx ? FFDAS_C_32F : FFDAS_R_32F)) return FFDAS_ERROR_UNSUPPORTED_TYPE;
    if (!cplx && a.wavenum != 0.f) return FFDAS_ERROR_INVALID_ARGUMENT;
    const int kind = select_storage(xd.dtype, gd.dtype, a.compute_type, xd.ndim == 4 ? (int)xd.dims[0] : 1);
    if (cplx ? (kind != ST_C32 && kind != ST_C16) : (kind != ST_F32 && kind != ST_F16 && kind != ST_BF16))
        return FFDAS_ERROR_UNSUPPORTED_TYPE;
    if (!fits_int32_indexing(xd) || !fits_int32_indexing(gd)) return FFDAS_ERROR_INVALID_DIMS;
    das_problem pb;
    FFDAS_TRY(make_problem(xd, gd, pb));
    if (a.sparse) {
        if (a.sparse_count <= 0) return FFDAS_ERROR_INVALID_ARGUMENT;
        if (!a.sparse_indices) return FFDAS_ERROR_NULL_POINTER;
        pb.n_events = a.sparse_count;
    } else {
        pb.n_events = pb.S;
    }
    if (pb.N >= (1 << 22)) return FFDAS_ERROR_DIMS_TOO_LARGE;
    if (pb.V == 0 || pb.B == 0) return FFDAS_SUCCESS;
    if (!gout || !a.dstpos || !a.offsets || !a.weights || (pb.C > 0 && !a.srcpos)) return FFDAS_ERROR_NULL_POINTER;
    if (!gx && !goff && !gw && !gdst && !gsrc) return FFDAS_SUCCESS;

    const int64_t npad = pair_row_length(pb.N);
    const int64_t rows = (int64_t)pb.B * pb.C * pb.S;
    const size_t sb = kind == ST_C32 ? 16 : (kind == ST_F32 || kind == ST_C16) ? 8 : 4;
    // the pair rows of the forward call on this x when it left them in the
    // handle's pair buffer, else built again
    workspace P(h);
    void *Pbase = reusable_pairs(h, xd, a.x, kind);
    h.last_pairs_reused = Pbase != nullptr;
    if (!Pbase) {
        FFDAS_TRY(P.alloc((size_t)std::max<int64_t>(rows, 1) * npad * sb));
        FFDAS_TRY(ingest_for_backward(h, pb, xd.dtype, kind, a.x, npad, P.get<void>()));
        Pbase = P.get<void>();
    }

    bwd_params bp;
    std::memset(&bp, 0, sizeof(bp));
    bp.P = Pbase;
    bp.npad = npad;
    bp.C = pb.C; bp.S = pb.S; bp.N = pb.N; bp.n_events = pb.n_events; bp.B = pb.B; bp.V = pb.V;
    bp.D0 = pb.D0; bp.D1 = pb.D1; bp.D2 = pb.D2;
    if (pb.D1 <= 1) { bp.T0 = 256; bp.T1 = 1; bp.T2 = 1; }
    else if (pb.D0 >= 16 && pb.D1 >= 16) { bp.T0 = 16; bp.T1 = 16; bp.T2 = 1; }
    else if (pb.D0 >= 32) { bp.T0 = 32; bp.T1 = 8; bp.T2 = 1; }
    else {
        int t = 1;
        while (t * 2 <= pb.D0) t *= 2;
        bp.T0 = t; bp.T1 = 256 / t; bp.T2 = 1;
    }
    bp.n0 = (pb.D0 + bp.T0 - 1) / bp.T0;
    bp.n1 = (pb.D1 + bp.T1 - 1) / bp.T1;
    const int n2 = (pb.D2 + bp.T2 - 1) / bp.T2;
    bp.srcpos = a.srcpos; bp.dstpos = a.dstpos; bp.offsets = a.offsets; bp.weights = a.weights;
    bp.srcdir = reinterpret_cast<const float4 *>(a.srcdir);
    bp.sparse_idx = a.sparse ? a.sparse_indices : nullptr;
    bp.gout = static_cast<const float *>(gout);
    bp.gout_bstride = pb.out_bstride;
    bp.gx = gx; bp.goff = goff; bp.gw = gw; bp.gdst = gdst; bp.gsrc = gsrc;

    pb.sparse = a.sparse;
    if (cplx) {   // complex data: the gather-form complex adjoint, one thread per voxel
        const int64_t blocks = (pb.V + kBwdThreads - 1) / kBwdThreads;
        if (blocks > INT32_MAX) return FFDAS_ERROR_DIMS_TOO_LARGE;
        // channel slices (8+ channels each) until about 8 CTAs per SM
        int slices = 1;
        while (blocks * slices * 2 <= (int64_t)std::max(h.sm_count, 1) * 8 && pb.C >= 16 * slices && slices < 64)
            slices *= 2;
        bwd_params cp = bp;
        cp.cchunk = 0;
        if (slices > 1) {
            const int chunk = (pb.C + slices - 1) / slices;
            slices = (pb.C + chunk - 1) / chunk;
            cp.cchunk = slices > 1 ? chunk : 0;
        }
        if (slices > 1) {   // the slices add into the voxel-side gradients
            const size_t ve = (size_t)pb.n_events * pb.V * sizeof(float);
            if (gw) FFDAS_CUDA(cudaMemsetAsync(gw, 0, ve, h.stream));
            if (goff) FFDAS_CUDA(cudaMemsetAsync(goff, 0, ve, h.stream));
            if (gdst) FFDAS_CUDA(cudaMemsetAsync(gdst, 0, (size_t)pb.V * 3 * sizeof(float), h.stream));
        }
        if (gsrc) FFDAS_CUDA(cudaMemsetAsync(gsrc, 0, (size_t)pb.C * 3 * sizeof(float), h.stream));
        h.last = ffdas_kernel_info_t{};
        h.last.variant = 8;
        h.last.storage = kind;
        h.last.kernels = h.last_pairs_reused ? 1 : 2;   // (ingest,) adjoint
        h.last.grid = blocks * slices;
        h.mark_start();
        const ffdas_error_t err =
            kind == ST_C32 ? launch_bwd_complex<ST_C32>(h, cp, a.sparse, a.wavenum, blocks, slices)
                           : launch_bwd_complex<ST_C16>(h, cp, a.sparse, a.wavenum, blocks, slices);
        h.mark_stop();
        return err;
    }
    // The backward kernel does not follow a forward schedule choice: only
    // variant 3 asks for the gather adjoint on dense problems.
    if (!a.sparse && !a.srcdir && staged_supported(pb, kind) && !(h.has_config && h.config.variant == 3)) {
        // Dense problems: TMA-staged adjoint, one CTA per voxel tile x batch item.
        if (h.has_config && h.config.variant == 2 && (h.config.tile_x || h.config.tile_y)) {
            const int tx = h.config.tile_x ? h.config.tile_x : 1, ty = h.config.tile_y ? h.config.tile_y : 1,
                      tz = h.config.tile_z ? h.config.tile_z : 1;
            if (tx * ty * tz == 256) {
                bp.T0 = tx; bp.T1 = ty; bp.T2 = tz;
                bp.n0 = (pb.D0 + tx - 1) / tx;
                bp.n1 = (pb.D1 + ty - 1) / ty;
            }
        } else if (pb.D0 >= 8 && pb.D1 >= 32) {
            // 8 x 32 tiles: a warp's voxels (one column of the tile under the
            // spread mapping) cover 32 rows along the second axis, so where that
            // axis is depth they meet more distinct samples -- fewer same-address
            // atomics in the scatter -- and where it is not, the cost is that of
            // 16 x 16 tiles.
            bp.T0 = 8; bp.T1 = 32; bp.T2 = 1;
            bp.n0 = (pb.D0 + 7) / 8;
            bp.n1 = (pb.D1 + 31) / 32;
        }
        const int64_t stiles = (int64_t)bp.n0 * bp.n1 * ((pb.D2 + bp.T2 - 1) / bp.T2);
        if (stiles > INT32_MAX) return FFDAS_ERROR_DIMS_TOO_LARGE;
        // batch tiles: up to 4 items per CTA share each window's delays
        const int WB = (h.has_config && h.config.window > 32) ? 64 : 32;
        const int copy = h.has_config ? h.config.copy_engine : 0;
        int BT = 1;
        while (BT * 2 <= std::min(pb.B, 4)) BT *= 2;
        if (h.has_config && h.config.variant == 2 && h.config.batch_tile) BT = std::min(h.config.batch_tile, 4);
        if (copy == 2 || !staged_batch_supported()) BT = 1;
        const int SC = BT > 1 ? 4 : (pb.n_events <= 1 ? 1 : 4);
        const int bchunks_st = (pb.B + BT - 1) / BT;
        // Channel slices over blockIdx.z (32+ channels each) while there are
        // fewer than min_blocks (default 2, the adjoint's CTAs per SM) CTAs per
        // SM, so that small problems fill the GPU.
        int csplit = 1;
        {
            const int per_sm = (h.has_config && h.config.min_blocks) ? h.config.min_blocks : 2;
            const int64_t ctas = stiles * bchunks_st;
            const int64_t want = (int64_t)std::max(h.sm_count, 1) * per_sm;
            while (ctas * csplit * 2 <= want && pb.C >= 64 * csplit && csplit < 64) csplit *= 2;
        }
        int cchunk = 0;
        if (csplit > 1) {
            cchunk = ((pb.C + csplit - 1) / csplit + 31) / 32 * 32;   // whole stages of channels
            csplit = (pb.C + cchunk - 1) / cchunk;
            if (csplit < 2) cchunk = 0;
        }
        const size_t ve0 = (size_t)pb.n_events * pb.V * sizeof(float);
        if (pb.B > 1 || csplit > 1) {  // several CTAs add into the voxel-side gradients
            if (gw) FFDAS_CUDA(cudaMemsetAsync(gw, 0, ve0, h.stream));
            if (goff) FFDAS_CUDA(cudaMemsetAsync(goff, 0, ve0, h.stream));
            if (gdst) FFDAS_CUDA(cudaMemsetAsync(gdst, 0, (size_t)pb.V * 3 * sizeof(float), h.stream));
        }
        if (gsrc) FFDAS_CUDA(cudaMemsetAsync(gsrc, 0, (size_t)pb.C * 3 * sizeof(float), h.stream));
        gather_params gp;
        std::memset(&gp, 0, sizeof(gp));
        gp.P = Pbase;
        gp.npad = npad;
        gp.C = pb.C; gp.S = pb.S; gp.n_events = pb.n_events; gp.B = pb.B; gp.V = pb.V;
        gp.D0 = pb.D0; gp.D1 = pb.D1; gp.D2 = pb.D2;
        gp.T0 = bp.T0; gp.T1 = bp.T1; gp.T2 = bp.T2; gp.n0 = bp.n0; gp.n1 = bp.n1;
        gp.srcpos = a.srcpos; gp.dstpos = a.dstpos; gp.offsets = a.offsets; gp.weights = a.weights;
        gp.beta_zero = 1;
        gp.cchunk = cchunk;
        const staged_grads gr{static_cast<const float *>(gout), pb.out_bstride, gx, goff, gw, gdst, gsrc};
        h.last = ffdas_kernel_info_t{};
        h.last.variant = 4;
        h.last.tile_x = bp.T0; h.last.tile_y = bp.T1; h.last.tile_z = bp.T2;
        h.last.batch_tile = BT; h.last.event_chunk = SC; h.last.storage = kind;
        h.last.kernels = h.last_pairs_reused ? 1 : 2;   // (ingest,) adjoint
        h.last.grid = stiles * bchunks_st * csplit;
        if (bchunks_st > 65535) return FFDAS_ERROR_DIMS_TOO_LARGE;
        h.mark_start();
        const ffdas_error_t err = launch_staged_bwd(h, pb, kind, gp, gr, SC, WB, BT, copy,
                                                    dim3((unsigned)stiles, (unsigned)bchunks_st, (unsigned)csplit));
        h.mark_stop();
        return err;
    }

    // das_sparse: the sorted-list adjoint (a lane per list entry) unless the
    // schedule asks for the gather adjoint (variant 3) or the CTA's tables
    // would not fit shared memory
    if (a.sparse && bws_supported(pb, kind) && !(h.has_config && h.config.variant == 3)) {
        bwd_params sp = bp;
        const int Ls = pb.n_events;
        int TV = kBwsMaxTile;
        while (TV > 32 && TV * Ls > kBwsMaxSlots) TV >>= 1;
        auto fit = [](int want, int dim) {   // power of two up to want, not past the first one >= dim
            int t = 1;
            while (t * 2 <= want && t < dim) t *= 2;
            return t;
        };
        sp.T0 = fit(std::min(TV, 16), pb.D0);
        sp.T1 = fit(TV / sp.T0, pb.D1);
        sp.T2 = fit(TV / (sp.T0 * sp.T1), pb.D2);
        sp.T0 = TV / (sp.T1 * sp.T2);
        sp.n0 = (pb.D0 + sp.T0 - 1) / sp.T0;
        sp.n1 = (pb.D1 + sp.T1 - 1) / sp.T1;
        const int64_t stiles = (int64_t)sp.n0 * sp.n1 * ((pb.D2 + sp.T2 - 1) / sp.T2);
        int csplit = 1;
        {
            const int per_sm = (h.has_config && h.config.min_blocks) ? h.config.min_blocks : 16;
            const int64_t want = (int64_t)std::max(h.sm_count, 1) * per_sm;
            while (stiles * pb.B * csplit * 2 <= want && pb.C >= 64 * csplit && csplit < 64) csplit *= 2;
        }
        sp.cchunk = 0;
        if (csplit > 1) {
            const int chunk = (pb.C + csplit - 1) / csplit;
            csplit = (pb.C + chunk - 1) / chunk;
            sp.cchunk = csplit > 1 ? chunk : 0;
        }
        const size_t smem = bws_smem_bytes(TV, Ls, pb.S, sp.cchunk ? sp.cchunk : pb.C);
        if (stiles <= INT32_MAX && smem <= kBwsMaxSmem) {
            // entries the kernel does not place have no gradient: zeroed outputs
            const size_t ves = (size_t)pb.n_events * pb.V * sizeof(float);
            if (gw) FFDAS_CUDA(cudaMemsetAsync(gw, 0, ves, h.stream));
            if (goff) FFDAS_CUDA(cudaMemsetAsync(goff, 0, ves, h.stream));
            if (gdst && (pb.B > 1 || csplit > 1))
                FFDAS_CUDA(cudaMemsetAsync(gdst, 0, (size_t)pb.V * 3 * sizeof(float), h.stream));
            if (gsrc) FFDAS_CUDA(cudaMemsetAsync(gsrc, 0, (size_t)pb.C * 3 * sizeof(float), h.stream));
            h.last = ffdas_kernel_info_t{};
            h.last.variant = 7;
            h.last.tile_x = sp.T0; h.last.tile_y = sp.T1; h.last.tile_z = sp.T2;
            h.last.batch_tile = 1; h.last.event_chunk = 0; h.last.storage = kind;
            h.last.kernels = h.last_pairs_reused ? 1 : 2;   // (ingest,) adjoint
            h.last.grid = stiles * pb.B * csplit;
            const dim3 grid((unsigned)stiles, (unsigned)pb.B, (unsigned)csplit);
            ffdas_error_t err;
            h.mark_start();
            switch (kind) {
                case ST_F32: err = launch_bws_t<ST_F32>(h, sp, Ls, grid, smem); break;
                case ST_F16: err = launch_bws_t<ST_F16>(h, sp, Ls, grid, smem); break;
                default: err = launch_bws_t<ST_BF16>(h, sp, Ls, grid, smem); break;
            }
            h.mark_stop();
            return err;
        }
    }

    const int BT = pb.B >= 4 ? 4 : (pb.B >= 2 ? 2 : 1);
    const int bchunks = (pb.B + BT - 1) / BT;
    const int64_t tiles = (int64_t)bp.n0 * bp.n1 * n2;
    if (tiles > INT32_MAX || bchunks > 65535) return FFDAS_ERROR_DIMS_TOO_LARGE;
    // Channel slices over blockIdx.z (32+ channels each) until there are about
    // min_blocks (default 16) CTAs per SM: at 97 registers two CTAs fit an
    // SM, and a few hundred tiles leave the last wave half empty.
    int csplit = 1;
    {
        const int per_sm = (h.has_config && h.config.min_blocks) ? h.config.min_blocks : 16;
        const int64_t want = (int64_t)std::max(h.sm_count, 1) * per_sm;
        while (tiles * bchunks * csplit * 2 <= want && pb.C >= 64 * csplit && csplit < 64) csplit *= 2;
    }
    if (csplit > 1) {
        const int chunk = (pb.C + csplit - 1) / csplit;
        csplit = (pb.C + chunk - 1) / chunk;
        bp.cchunk = csplit > 1 ? chunk : 0;
    }
    // outputs reduced with atomics must start at zero; the balanced das_sparse
    // walk (no weight gradient) stores no delay gradient for the entries past
    // a warp's longest list, which are padding: zero them too
    const size_t ve = (size_t)pb.n_events * pb.V * sizeof(float);
    const bool shared_voxels = bchunks > 1 || csplit > 1;
    if (shared_voxels || (a.sparse && !gw)) {
        if (gw) FFDAS_CUDA(cudaMemsetAsync(gw, 0, ve, h.stream));
        if (goff) FFDAS_CUDA(cudaMemsetAsync(goff, 0, ve, h.stream));
    }
    if (shared_voxels && gdst) FFDAS_CUDA(cudaMemsetAsync(gdst, 0, (size_t)pb.V * 3 * sizeof(float), h.stream));
    if (gsrc) FFDAS_CUDA(cudaMemsetAsync(gsrc, 0, (size_t)pb.C * 3 * sizeof(float), h.stream));

    dim3 grid((unsigned)tiles, (unsigned)bchunks, (unsigned)csplit);
    h.last = ffdas_kernel_info_t{};
    h.last.variant = 3;
    h.last.tile_x = bp.T0; h.last.tile_y = bp.T1; h.last.tile_z = bp.T2;
    h.last.batch_tile = BT; h.last.event_chunk = 8; h.last.storage = kind;
    h.last.kernels = h.last_pairs_reused ? 1 : 2;   // (ingest,) adjoint
    h.last.grid = tiles * bchunks * csplit;
    const bool sp = a.sparse;
    ffdas_error_t err;
    h.mark_start();
    switch (kind) {
        case ST_F32: err = sp ? launch_bwd_k<ST_F32, true>(h, bp, BT, grid) : launch_bwd_k<ST_F32, false>(h, bp, BT, grid); break;
        case ST_F16: err = sp ? launch_bwd_k<ST_F16, true>(h, bp, BT, grid) : launch_bwd_k<ST_F16, false>(h, bp, BT, grid); break;
        default: err = sp ? launch_bwd_k<ST_BF16, true>(h, bp, BT, grid) : launch_bwd_k<ST_BF16, false>(h, bp, BT, grid); break;
    }
    h.mark_stop();
    return err;
}

}  // namespace ffdas

using namespace ffdas;

extern "C" ffdas_error_t ffdas_das_backward(
    ffdas_handle_t handle, const float *srcpos, const float *srcdir, float wavenum,
    ffdas_tensor_desc_t x_desc, const void *x, const float *dstpos, const float *offsets,
    const float *weights, int sparse_count, const int *sparse_indices,
    ffdas_tensor_desc_t grad_out_desc, const void *grad_out, float *grad_x, float *grad_offsets,
    float *grad_weights, float *grad_dstpos, float *grad_srcpos) {
    if (!handle) return FFDAS_ERROR_INVALID_HANDLE;
    FFDAS_TRY(handle->check_device());
    if (!x_desc || !grad_out_desc) return FFDAS_ERROR_NULL_POINTER;
    das_call a;
    a.srcpos = srcpos; a.srcdir = srcdir; a.wavenum = wavenum; a.x_desc = x_desc; a.x = x;
    a.dstpos = dstpos; a.offsets = offsets; a.weights = weights;
    a.sparse = sparse_indices != nullptr;
    a.sparse_count = sparse_count; a.sparse_indices = sparse_indices;
    a.compute_type = FFDAS_COMPUTE_DEFAULT;
    return das_backward(*handle, a, *grad_out_desc, grad_out, grad_x, grad_offsets, grad_weights,
                        grad_dstpos, grad_srcpos);
}
