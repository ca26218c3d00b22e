// das_direct.cu -- delay-and-sum for small problems, straight from x.
//
// A frame of a few million units (one plane wave on a 2-D grid: 32K pixels x
// 128 channels) is over in microseconds, so the cost of a call is its launch
// chain: the pair ingest, the staged kernel's pipeline fill and the handful
// of windows each CTA stages.  This kernel is the whole call in one launch
// and no workspace: `split` consecutive lanes share a voxel and take every
// split-th channel, read x[k] and x[k+1] where the tap lands (L1/L2 gathers;
// the channel data of such a frame is a megabyte or two), and add their
// partial sums with warp shuffles.
//
// Arithmetic per (voxel, channel, event) is the reference's
// (src/das/das_alg1_kernels.cuh:60-99, lerp = fma(t, x1 - x0, x0)): the same
// delay, floor split and tap as the staged kernels' f32 pairs, so only the
// order of the sum over channels and events differs.  A tap outside the record
// (0 <= k < N - 1 fails) reads nothing and contributes fma(w, 0, acc), as a
// zero pair would.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <type_traits>

#include "core.h"
#include "das_common.cuh"
#include "das_direct.h"
#include "das_pairs.cuh"

namespace ffdas {

struct direct_params {
    const void *x;
    int bstride, cstride, sstride;   // x strides in elements (sample stride 1; x fits int32 indexing)
    int B, C, S, N;
    int64_t V;
    int split, split_log2;
    int chan_smem;                   // channel positions staged in shared memory
    const float *srcpos;
    const float4 *srcdir;
    const float *dstpos, *offsets, *weights;
    float *out;
    int64_t out_bstride;
    float beta;
    int beta_zero;
};

constexpr int kDirectThreads = 256;
constexpr int kDirectSmemChannels = 4096;   // channel positions kept in shared memory up to this count
constexpr int kDirectUnroll = 4;

template <typename Tin, int BT>
__global__ void __launch_bounds__(kDirectThreads) das_direct_kernel(const direct_params p) {
    extern __shared__ float4 chan[];   // (x, y, z, 0) per channel
    const int C = p.C, S = p.S, split = p.split;
    const int64_t V = p.V;
    if (p.chan_smem) {
        for (int i = threadIdx.x; i < C; i += kDirectThreads)
            chan[i] = make_float4(__ldg(p.srcpos + 3 * i), __ldg(p.srcpos + 3 * i + 1), __ldg(p.srcpos + 3 * i + 2), 0.f);
        __syncthreads();
    }
    const int64_t gt = (int64_t)blockIdx.x * kDirectThreads + threadIdx.x;
    const int64_t v = gt >> p.split_log2;
    const int part = (int)(gt & (split - 1));
    const bool active = v < V;
    const int b0 = (int)blockIdx.y * BT;
    float acc[BT];
#pragma unroll
    for (int bi = 0; bi < BT; bi++) acc[bi] = 0.f;
    if (active) {
        const Tin *xb[BT];
#pragma unroll
        for (int bi = 0; bi < BT; bi++)   // items past B read item B-1 and are never stored
            xb[bi] = static_cast<const Tin *>(p.x) + (int64_t)min(b0 + bi, p.B - 1) * p.bstride;
        const float vx = __ldg(p.dstpos + 3 * v), vy = __ldg(p.dstpos + 3 * v + 1), vz = __ldg(p.dstpos + 3 * v + 2);
        const uint32_t nlast = (uint32_t)(p.N - 1);
        const float *po0 = p.offsets + v, *pw0 = p.weights + v;
        const int cstride = p.cstride, sstride = p.sstride;
        const bool chan_smem = p.chan_smem;
        const float *srcpos = p.srcpos;
        const float4 *srcdir = p.srcdir;
        // kDirectUnroll channels per step: their gathers are independent, so a
        // thread keeps several L2 requests in flight instead of waiting out
        // each tap in turn.  Whole steps run without channel tests; the last,
        // partial step (CHECK) masks the channels past C.
        auto step = [&](const int c0, auto check_c) {
            constexpr bool CHECK = decltype(check_c)::value;
            recv_geom gm[kDirectUnroll];
            int row[kDirectUnroll];
            bool live[kDirectUnroll];
#pragma unroll
            for (int u = 0; u < kDirectUnroll; u++) {
                const int c = c0 + u * split;
                live[u] = !CHECK || c < C;
                const int cc = live[u] ? c : 0;
                const float4 cp = chan_smem ? chan[cc]
                                            : make_float4(__ldg(srcpos + 3 * cc), __ldg(srcpos + 3 * cc + 1),
                                                          __ldg(srcpos + 3 * cc + 2), 0.f);
                gm[u] = receive_geometry(vx, vy, vz, cp.x, cp.y, cp.z);
                if (srcdir) apply_directivity(gm[u], vx, vy, vz, cp.x, cp.y, cp.z, __ldg(srcdir + cc));
                row[u] = cc * cstride;
            }
            const float *po = po0, *pw = pw0;
            int srow = 0;
            for (int s = 0; s < S; s++, po += V, pw += V, srow += sstride) {
                const float ofs = __ldg(po), w = __ldg(pw);
                float t[kDirectUnroll];
                int e[kDirectUnroll];
                bool in[kDirectUnroll];
#pragma unroll
                for (int u = 0; u < kDirectUnroll; u++) {
                    const tau_split ts = split_tau(__fmaf_rn(gm[u].rsq, gm[u].rinv, ofs));
                    in[u] = live[u] && ts.k < nlast;
                    t[u] = ts.t;
                    e[u] = row[u] + srow + (in[u] ? (int)ts.k : 0);
                }
#pragma unroll
                for (int bi = 0; bi < BT; bi++) {
                    float x0[kDirectUnroll], x1[kDirectUnroll];
#pragma unroll
                    for (int u = 0; u < kDirectUnroll; u++) {
                        x0[u] = in[u] ? (float)sample_io<Tin>::load(xb[bi] + e[u]) : 0.f;
                        x1[u] = in[u] ? (float)sample_io<Tin>::load(xb[bi] + e[u] + 1) : 0.f;
                    }
#pragma unroll
                    for (int u = 0; u < kDirectUnroll; u++)
                        if (live[u]) acc[bi] = __fmaf_rn(w, __fmaf_rn(t[u], x1[u] - x0[u], x0[u]), acc[bi]);
                }
            }
        };
        const int stride = kDirectUnroll * split;
        int c0 = part;
        for (; c0 + (kDirectUnroll - 1) * split < C; c0 += stride) step(c0, std::false_type{});
        if (c0 < C) step(c0, std::true_type{});
    }
    // partial sums of the voxel's split lanes (consecutive lanes of one warp)
    for (int off = split >> 1; off > 0; off >>= 1) {
#pragma unroll
        for (int bi = 0; bi < BT; bi++) acc[bi] += __shfl_xor_sync(0xffffffffu, acc[bi], off);
    }
    if (!active || part != 0) return;
#pragma unroll
    for (int bi = 0; bi < BT; bi++) {
        const int b = b0 + bi;
        if (b >= p.B) break;
        float *o = p.out + (int64_t)b * p.out_bstride + v;
        *o = p.beta_zero ? acc[bi] : __fmaf_rn(p.beta, *o, acc[bi]);
    }
}

bool direct_supported(const das_problem &pb, ffdas_datatype_t xt, ffdas_datatype_t ot, int kind) {
    if (pb.sparse || kind != ST_F32 || ot != FFDAS_R_32F) return false;
    if (xt != FFDAS_R_32F && xt != FFDAS_R_16F && xt != FFDAS_R_16BF && xt != FFDAS_R_16I) return false;
    return pb.C > 0 && pb.S > 0 && pb.B <= 65535 * 4;
}

template <typename Tin, int BT>
static ffdas_error_t launch_direct_t(ffdas_context &h, const direct_params &dp) {
    const int64_t threads = dp.V << dp.split_log2;
    const int64_t blocks = (threads + kDirectThreads - 1) / kDirectThreads;
    const int64_t bchunks = (dp.B + BT - 1) / BT;
    if (blocks > INT32_MAX || bchunks > 65535) return FFDAS_ERROR_DIMS_TOO_LARGE;
    const size_t smem = dp.chan_smem ? (size_t)dp.C * sizeof(float4) : 0;
    if (smem > 48 * 1024) {   // the attribute belongs to the device: set it for each one
        static std::atomic<unsigned long long> done{0ull};
        int dev = 0;
        FFDAS_CUDA(cudaGetDevice(&dev));
        const unsigned long long bit = 1ull << (dev & 63);
        if (!(done.load(std::memory_order_acquire) & bit)) {
            FFDAS_CUDA(cudaFuncSetAttribute(das_direct_kernel<Tin, BT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)(kDirectSmemChannels * sizeof(float4))));
            done.fetch_or(bit, std::memory_order_release);
        }
    }
    das_direct_kernel<Tin, BT><<<dim3((unsigned)blocks, (unsigned)bchunks), kDirectThreads, smem, h.stream>>>(dp);
    return ffdas_launch_check(h.stream);
}

template <typename Tin>
static ffdas_error_t launch_direct_bt(ffdas_context &h, const direct_params &dp, int BT) {
    if (BT >= 4) return launch_direct_t<Tin, 4>(h, dp);
    if (BT == 2) return launch_direct_t<Tin, 2>(h, dp);
    return launch_direct_t<Tin, 1>(h, dp);
}

// Resident CTAs per SM of the kernel instance a call will launch.
static int direct_blocks_per_sm(ffdas_datatype_t xt, int batch_tile, int C) {
    const size_t smem = C <= kDirectSmemChannels ? (size_t)C * sizeof(float4) : 0;
    int n = 0;
    cudaError_t e = cudaErrorInvalidValue;
    const int bt = batch_tile >= 4 ? 4 : (batch_tile == 2 ? 2 : 1);
    switch (xt) {
        case FFDAS_R_16F:
            e = bt == 4 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, das_direct_kernel<__half, 4>, kDirectThreads, smem)
              : bt == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, das_direct_kernel<__half, 2>, kDirectThreads, smem)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, das_direct_kernel<__half, 1>, kDirectThreads, smem);
            break;
        case FFDAS_R_16I:
            e = bt == 4 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, das_direct_kernel<int16_t, 4>, kDirectThreads, smem)
              : bt == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, das_direct_kernel<int16_t, 2>, kDirectThreads, smem)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, das_direct_kernel<int16_t, 1>, kDirectThreads, smem);
            break;
        case FFDAS_R_16BF:
            e = bt == 4 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, das_direct_kernel<__nv_bfloat16, 4>, kDirectThreads, smem)
              : bt == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, das_direct_kernel<__nv_bfloat16, 2>, kDirectThreads, smem)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, das_direct_kernel<__nv_bfloat16, 1>, kDirectThreads, smem);
            break;
        default:
            e = bt == 4 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, das_direct_kernel<float, 4>, kDirectThreads, smem)
              : bt == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, das_direct_kernel<float, 2>, kDirectThreads, smem)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, das_direct_kernel<float, 1>, kDirectThreads, smem);
            break;
    }
    return (e == cudaSuccess && n > 0) ? n : 4;
}

ffdas_error_t launch_direct(ffdas_context &h, const das_problem &pb, ffdas_datatype_t xt, const void *x,
                            const float *srcpos, const float *srcdir, const float *dstpos, const float *offsets,
                            const float *weights, float *out, double beta, int beta_zero, int batch_tile,
                            int split_req) {
    int BT = batch_tile > 0 ? batch_tile : 1;
    while (BT > 1 && BT > pb.B) BT >>= 1;
    direct_params dp;
    std::memset(&dp, 0, sizeof(dp));
    dp.x = x;
    // x fits int32 indexing (checked by the caller), so element offsets are int
    dp.bstride = (int)pb.x_bstride; dp.cstride = (int)pb.x_cstride; dp.sstride = (int)pb.x_sstride;
    dp.chan_smem = pb.C <= kDirectSmemChannels;
    dp.B = pb.B; dp.C = pb.C; dp.S = pb.S; dp.N = pb.N; dp.V = pb.V;
    // lanes per voxel (power of two, at most 32 and at most the channel
    // count): the schedule's tile_x, else the most that keeps the launch
    // within two waves of resident threads (measured: the per-thread channel
    // loop is latency-bound, so more lanes pay until the second wave fills)
    int split = 1, lg = 0;
    if (split_req > 0) {
        while (split * 2 <= std::min(split_req, 32)) {
            split *= 2;
            lg++;
        }
    } else {
        const int64_t resident = (int64_t)std::max(h.sm_count, 1) * direct_blocks_per_sm(xt, BT, pb.C) *
                                 kDirectThreads;
        while (split < 32 && split * 2 <= pb.C && pb.V * split * 2 <= 2 * resident) {
            split *= 2;
            lg++;
        }
    }
    dp.split = split; dp.split_log2 = lg;
    dp.srcpos = srcpos;
    dp.srcdir = reinterpret_cast<const float4 *>(srcdir);
    dp.dstpos = dstpos; dp.offsets = offsets; dp.weights = weights;
    dp.out = out;
    dp.out_bstride = pb.out_bstride;
    dp.beta = (float)beta;
    dp.beta_zero = beta_zero;
    h.last = ffdas_kernel_info_t{};
    h.last.variant = 5;
    h.last.tile_x = split;     // lanes per voxel
    h.last.tile_y = 1; h.last.tile_z = 1;
    h.last.batch_tile = BT >= 4 ? 4 : BT;
    h.last.event_chunk = 1;
    h.last.storage = ST_F32;
    h.last.kernels = 1;
    h.last.grid = ((pb.V << lg) + kDirectThreads - 1) / kDirectThreads * ((pb.B + h.last.batch_tile - 1) / h.last.batch_tile);
    h.mark_start();
    ffdas_error_t err;
    switch (xt) {
        case FFDAS_R_32F: err = launch_direct_bt<float>(h, dp, BT); break;
        case FFDAS_R_16F: err = launch_direct_bt<__half>(h, dp, BT); break;
        case FFDAS_R_16BF: err = launch_direct_bt<__nv_bfloat16>(h, dp, BT); break;
        case FFDAS_R_16I: err = launch_direct_bt<int16_t>(h, dp, BT); break;
        default: err = FFDAS_ERROR_INTERNAL; break;
    }
    h.mark_stop();
    return err;
}

}  // namespace ffdas
