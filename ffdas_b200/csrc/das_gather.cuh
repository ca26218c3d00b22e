// das_gather.cuh -- forward delay-and-sum, L1 gather schedule.
//
// One thread = one voxel x BT batch items.  A CTA is a spatially compact tile
// of voxels (tile_x x tile_y x tile_z over the output grid), so the warps of a
// CTA read the same narrow sample window of each (channel, event) row and the
// pair loads hit in L1.  Per (voxel, channel) the receive geometry (rsq,
// rsqrt) is computed once and reused for every event and batch item; per
// (voxel, channel, event) the delay is one FFMA, the floor/fraction split is
// three FADDs, and each batch item costs one 8-byte (f32) or 4-byte (f16/bf16)
// load, one tap FFMA and one accumulate FFMA.
//
// Follows the arithmetic of das_alg1_kernel (src/das/das_alg1_kernels.cuh:
// 16-107): same tau, same floor split, same lerp and the same FFMA
// accumulation; only the order of the sum over (channel, event) differs.
#pragma once

#include <type_traits>

#include "das_pairs.cuh"

namespace ffdas {

struct gather_params {
    const void *P;            // pair rows [B][C][S][Npad]
    int64_t npad;             // pairs per row
    int C, S;                 // channels, events in x
    int n_events;             // S (dense) or sparse_count
    int B;                    // batch
    int64_t V;                // voxels
    int D0, D1, D2;           // output grid (D0 innermost)
    int T0, T1, T2;           // tile extents (T0*T1*T2 == blockDim.x)
    int n0, n1;               // tiles along D0, D1
    const float *srcpos;      // (C,3)
    const float4 *srcdir;     // (C,4) or null
    const float *dstpos;      // (V,3)
    const float *offsets;     // (n_events, V)
    const float *weights;     // (n_events, V)
    const int *sparse_idx;    // (n_events, V) or null
    float wavenum;
    void *out;
    int64_t out_bstride;      // elements between batch items of out
    double beta_re, beta_im;
    int beta_zero;
    int cchunk;               // staged forward: channels per blockIdx.z slice (0: no split)
    const int *run_if;        // when set, the kernel runs only if *run_if != 0 (das_sparse fallback)
};

template <typename A> struct acc_ops;
template <> struct acc_ops<float> {
    __device__ static float zero() { return 0.f; }
};
template <> struct acc_ops<double> {
    __device__ static double zero() { return 0.0; }
};
template <> struct acc_ops<float2> {
    __device__ static float2 zero() { return make_float2(0.f, 0.f); }
};
template <> struct acc_ops<double2> {
    __device__ static double2 zero() { return make_double2(0.0, 0.0); }
};

// cuCfmaf ordering (reference cmadd for float2, src/core/math/vector.cuh:150)
__device__ __forceinline__ float2 cfma(float2 x, float2 y, float2 z) {
    float re = __fmaf_rn(-x.y, y.y, __fmaf_rn(x.x, y.x, z.x));
    float im = __fmaf_rn(x.y, y.x, __fmaf_rn(x.x, y.y, z.y));
    return make_float2(re, im);
}
// reference cmadd for double2 (src/core/math/vector.cuh:156-160)
__device__ __forceinline__ double2 cfma(double2 x, double2 y, double2 z) {
    return make_double2(fma(x.x, y.x, z.x) - x.y * y.y, fma(x.x, y.y, z.y) + x.y * y.x);
}

// acc += w * v (real) or acc += w * exp(i wavenum tau) * v (complex)
template <int K>
__device__ __forceinline__ void accumulate(typename pair_traits<K>::acc &acc,
                                           typename pair_traits<K>::value v, float w,
                                           float wavenum, float tau) {
    if constexpr (K == ST_F32 || K == ST_F16 || K == ST_BF16) {
        acc = __fmaf_rn(w, v, acc);
    } else if constexpr (K == ST_F64) {
        acc = fma((double)w, v, acc);
    } else if constexpr (K == ST_C32 || K == ST_C16) {
        float sn, cs;
        __sincosf(wavenum * tau, &sn, &cs);
        acc = cfma(make_float2(cs * w, sn * w), v, acc);
    } else {
        float sn, cs;
        __sincosf(wavenum * tau, &sn, &cs);
        acc = cfma(make_double2((double)(cs * w), (double)(sn * w)), v, acc);
    }
}

template <typename A> __device__ __forceinline__ void store_out(A *o, A acc, const gather_params &p);
template <> __device__ __forceinline__ void store_out<float>(float *o, float acc, const gather_params &p) {
    *o = p.beta_zero ? acc : __fmaf_rn((float)p.beta_re, *o, acc);
}
template <> __device__ __forceinline__ void store_out<double>(double *o, double acc, const gather_params &p) {
    *o = p.beta_zero ? acc : fma(p.beta_re, *o, acc);
}
template <> __device__ __forceinline__ void store_out<float2>(float2 *o, float2 acc, const gather_params &p) {
    *o = p.beta_zero ? acc : cfma(make_float2((float)p.beta_re, (float)p.beta_im), *o, acc);
}
template <> __device__ __forceinline__ void store_out<double2>(double2 *o, double2 acc, const gather_params &p) {
    *o = p.beta_zero ? acc : cfma(make_double2(p.beta_re, p.beta_im), *o, acc);
}

// Sparse load balance.  A voxel's event list may end in padding (entries
// with zero weight or an out-of-range index, as the reference's callers pad
// uneven lists to sparse_count).  Each thread of a sparse CTA measures, for
// its tile position, L = 1 + the last real entry; the CTA then orders its
// voxels by L (a 64-bucket counting sort in shared memory) so that each warp
// holds voxels of similar L, and each warp runs the event loop only up to the
// largest L among its lanes.  Work then follows the real event count instead
// of sparse_count.  Returns the tile position this thread takes; L_out is the
// L of the thread's original position (the caller exchanges them through
// shared memory).
template <typename Params>   // gather_params, or the adjoint's parameters (same field names)
__device__ __forceinline__ int sparse_balance(const Params &p, int tid, int t0, int t1, int t2, int &L_out) {
    __shared__ int hist[64], base[64];
    __shared__ short order[256];
    const int i0 = tid % p.T0, i1 = (tid / p.T0) % p.T1, i2 = tid / (p.T0 * p.T1);
    const int g0 = t0 * p.T0 + i0, g1 = t1 * p.T1 + i1, g2 = t2 * p.T2 + i2;
    int L = 0;
    if (g0 < p.D0 && g1 < p.D1 && g2 < p.D2) {
        const int64_t v = ((int64_t)g2 * p.D1 + g1) * p.D0 + g0;
        for (int e = 0; e < p.n_events; e++) {
            const int64_t idx = (int64_t)e * p.V + v;
            const int s = __ldg(p.sparse_idx + idx);
            if ((unsigned)s < (unsigned)p.S && __ldg(p.weights + idx) != 0.f) L = e + 1;
        }
    }
    if (tid < 64) hist[tid] = 0;
    __syncthreads();
    const int bucket = (int)(((int64_t)L * 63) / max(p.n_events, 1));   // 0..63, monotone in L
    const int pos = atomicAdd(&hist[bucket], 1);
    __syncthreads();
    if (tid < 32) {   // exclusive prefix over the 64 buckets, two per lane
        const int a = hist[2 * tid], b = hist[2 * tid + 1];
        int incl = a + b;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (tid >= o) incl += y;
        }
        base[2 * tid] = incl - a - b;
        base[2 * tid + 1] = incl - b;
    }
    __syncthreads();
    order[base[bucket] + pos] = (short)tid;
    __syncthreads();
    L_out = L;          // L of this thread's own tile position
    return order[tid];  // the tile position this thread takes over
}

// Output element type for a storage kind and output dtype: the kernel
// accumulates in pair_traits<K>::acc and converts on store.
template <int K, typename OutT, int BT, int SC, bool SPARSE>
__global__ void __launch_bounds__(256) das_gather_kernel(const gather_params p) {
    using tr = pair_traits<K>;
    using st = typename tr::storage;
    using acc_t = typename tr::acc;
    if (p.run_if && *(volatile const int *)p.run_if == 0) return;   // uniform for the grid

    int tid = threadIdx.x;
    const int tile = blockIdx.x;
    const int t0 = tile % p.n0;
    const int t1 = (tile / p.n0) % p.n1;
    const int t2 = tile / (p.n0 * p.n1);
    int n_ev = p.n_events;
    if constexpr (SPARSE) {
        __shared__ int Ls[256];
        int L;
        const int me = sparse_balance(p, tid, t0, t1, t2, L);
        Ls[tid] = L;
        __syncthreads();
        tid = me;                      // the tile position this thread now owns
        L = Ls[me];
        n_ev = __reduce_max_sync(0xffffffffu, (unsigned)L);   // the warp's longest list
    }
    const int i0 = tid % p.T0;
    const int i1 = (tid / p.T0) % p.T1;
    const int i2 = tid / (p.T0 * p.T1);
    const int g0 = t0 * p.T0 + i0, g1 = t1 * p.T1 + i1, g2 = t2 * p.T2 + i2;
    if (g0 >= p.D0 || g1 >= p.D1 || g2 >= p.D2) return;
    const int64_t v = ((int64_t)g2 * p.D1 + g1) * p.D0 + g0;
    const int b0 = blockIdx.y * BT;

    const float vx = __ldg(p.dstpos + 3 * v + 0);
    const float vy = __ldg(p.dstpos + 3 * v + 1);
    const float vz = __ldg(p.dstpos + 3 * v + 2);

    const st *__restrict__ P = static_cast<const st *>(p.P);
    const uint32_t kmax = (uint32_t)(p.npad - 1);
    const int64_t row_stride_b = (int64_t)p.C * p.S * p.npad;  // pairs per batch item

    acc_t acc[BT];
#pragma unroll
    for (int b = 0; b < BT; b++) acc[b] = acc_ops<acc_t>::zero();

    // Batch items past B read batch item 0 (their results are discarded), so
    // the unrolled loops below carry no per-item branch.
    int64_t boff[BT];
#pragma unroll
    for (int b = 0; b < BT; b++) boff[b] = (b0 + b < p.B) ? (int64_t)(b0 + b) * row_stride_b : 0;

    for (int e0 = 0; e0 < n_ev; e0 += SC) {
        const int sc = min(SC, n_ev - e0);
        // Event slots past the end, zero-weight (padding) entries and
        // out-of-range event indices get a huge delay: their tap lands on the
        // zero pair and their weight is 0, so every slot runs the same
        // branch-free code.
        float ofs[SC], w[SC];
        uint32_t srow[SC];  // row offset of the event within a channel, in pairs
#pragma unroll
        for (int j = 0; j < SC; j++) {
            ofs[j] = 1e30f;
            w[j] = 0.f;
            srow[j] = 0;
            if (j < sc) {
                const int64_t idx = (int64_t)(e0 + j) * p.V + v;
                const float o = __ldg(p.offsets + idx);
                const float ww = __ldg(p.weights + idx);
                int s = e0 + j;
                if constexpr (SPARSE) s = __ldg(p.sparse_idx + idx);
                if ((unsigned)s < (unsigned)p.S && (!SPARSE || ww != 0.f)) {
                    ofs[j] = o;
                    w[j] = ww;
                    srow[j] = (uint32_t)s * (uint32_t)p.npad;
                }
            }
        }

        // channel slice of this CTA (blockIdx.z) when the call splits channels
        const int cbeg = p.cchunk ? (int)blockIdx.z * p.cchunk : 0;
        const int cend = p.cchunk ? min(p.C, cbeg + p.cchunk) : p.C;
        for (int c = cbeg; c < cend; c++) {
            const float cx = __ldg(p.srcpos + 3 * c + 0);
            const float cy = __ldg(p.srcpos + 3 * c + 1);
            const float cz = __ldg(p.srcpos + 3 * c + 2);
            recv_geom g = receive_geometry(vx, vy, vz, cx, cy, cz);
            if (p.srcdir) apply_directivity(g, vx, vy, vz, cx, cy, cz, __ldg(p.srcdir + c));
            const st *Pc = P + (int64_t)c * p.S * p.npad;

            // phase 1: every tap's index and load, so all loads are in flight
            st pr[SC][BT];
            float tt[SC], tau[SC];
#pragma unroll
            for (int j = 0; j < SC; j++) {
                tau[j] = __fmaf_rn(g.rsq, g.rinv, ofs[j]);
                const tau_split ts = split_tau(tau[j]);
                tt[j] = ts.t;
                // Slots past the last event must still address a row of THIS
                // channel (their tap is the zero pair), so clamp the event.
                const uint32_t rowoff =
                    SPARSE ? srow[j] : (uint32_t)min(e0 + j, p.n_events - 1) * (uint32_t)p.npad;
                const st *row = Pc + (rowoff + min(ts.k, kmax));
#pragma unroll
                for (int b = 0; b < BT; b++) pr[j][b] = row[boff[b]];
            }
            // phase 2: interpolate and accumulate
#pragma unroll
            for (int j = 0; j < SC; j++) {
#pragma unroll
                for (int b = 0; b < BT; b++)
                    accumulate<K>(acc[b], tr::tap(pr[j][b], tt[j]), w[j], p.wavenum, tau[j]);
            }
        }
    }

    OutT *out = static_cast<OutT *>(p.out);
#pragma unroll
    for (int b = 0; b < BT; b++) {
        if (BT == 1 || b0 + b < p.B) {
            OutT *o = out + (int64_t)(b0 + b) * p.out_bstride + v;
            if constexpr (std::is_same_v<OutT, float> && std::is_same_v<acc_t, float>) {
                if (p.cchunk) {   // channel slices add into the prepared image
                    atomicAdd(o, acc[b]);
                    continue;
                }
            }
            if constexpr (sizeof(OutT) == sizeof(acc_t)) {
                store_out<OutT>(o, acc[b], p);
            } else if constexpr (sizeof(OutT) == 8 && sizeof(acc_t) == 4) {
                store_out<double>(reinterpret_cast<double *>(o), (double)acc[b], p);
            } else {
                // complex float accumulation stored to complex double
                store_out<double2>(reinterpret_cast<double2 *>(o),
                                   make_double2(acc[b].x, acc[b].y), p);
            }
        }
    }
}

}  // namespace ffdas
