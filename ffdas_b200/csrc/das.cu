// das.cu -- ffdas_das / ffdas_das_sparse entry points and forward dispatch.
//
// Validation order and error codes follow the reference: handle, device,
// descriptors (src/das/das.cu:25-28), dtype combination (:40-82), int32
// index guard and algorithm (src/das/das_impl.cuh:34-54), problem dims
// (src/das/das_utils.h:32-69), compute-type support
// (src/das/das_alg1.cu:172-178), sparse count (das_alg1.cu:267).
// After validation every call runs: ingest (x -> pair rows) then the
// forward kernel chosen by the planner or the handle's config.
#include <cuda.h>
#include <algorithm>
#include <cstring>
#include <mutex>

#include "core.h"
#include "das_problem.h"
#include "das_direct.h"
#include "das_gather.cuh"

namespace ffdas {

bool fits_int32_indexing(const ffdas_tensor_desc &d) {
    int64_t max_off = 0;
    for (int64_t i = 0; i < d.ndim; i++)
        if (d.dims[i] > 1) max_off += (d.dims[i] - 1) * (d.strides[i] < 0 ? -d.strides[i] : d.strides[i]);
    return max_off <= INT32_MAX && d.numel() <= INT32_MAX;
}

ffdas_error_t make_problem(const ffdas_tensor_desc &x, const ffdas_tensor_desc &out, das_problem &p) {
    if (x.ndim != 3 && x.ndim != 4) return FFDAS_ERROR_INVALID_DIMS;
    if (out.ndim < 1) return FFDAS_ERROR_INVALID_DIMS;
    p.have_batch = (x.ndim == 4);
    const int o = p.have_batch ? 1 : 0;
    for (int64_t i = 0; i < x.ndim; i++)
        if (x.dims[i] < 0) return FFDAS_ERROR_INVALID_DIMS;
    for (int64_t i = 0; i < out.ndim; i++)
        if (out.dims[i] < 0) return FFDAS_ERROR_INVALID_DIMS;
    p.B = p.have_batch ? (int)x.dims[0] : 1;
    p.C = (int)x.dims[o + 0];
    p.S = (int)x.dims[o + 1];
    p.N = (int)x.dims[o + 2];
    if (p.have_batch && (out.ndim < 2 || out.dims[0] != p.B)) return FFDAS_ERROR_INVALID_DIMS;
    p.V = 1;
    for (int64_t i = o; i < out.ndim; i++) p.V *= out.dims[i];
    p.x_bstride = p.have_batch ? x.strides[0] : 0;
    p.x_cstride = x.strides[o + 0];
    p.x_sstride = x.strides[o + 1];
    if (x.strides[o + 2] != 1 && p.N > 1) return FFDAS_ERROR_INVALID_ARGUMENT;
    p.out_bstride = p.have_batch ? out.strides[0] : 0;

    // Spatial dims of out must be C-contiguous (the reference assumes it
    // without checking, das_alg1_kernels.cuh:104).
    int64_t s = 1;
    for (int64_t i = out.ndim - 1; i >= o; i--) {
        if (out.dims[i] > 1 && out.strides[i] != s) return FFDAS_ERROR_NON_CONTIGUOUS;
        s *= out.dims[i];
    }
    // Collapse spatial dims (dropping size-1 dims) into (D2, D1, D0).
    int64_t sp[FFDAS_MAX_DIMS];
    int ns = 0;
    for (int64_t i = o; i < out.ndim; i++)
        if (out.dims[i] != 1) sp[ns++] = out.dims[i];
    int64_t d0 = 1, d1 = 1, d2 = 1;
    if (ns >= 1) d0 = sp[ns - 1];
    if (ns >= 2) d1 = sp[ns - 2];
    for (int i = 0; i < ns - 2; i++) d2 *= sp[i];
    if (p.V == 0) d0 = d1 = d2 = 0;
    p.D0 = (int)d0;
    p.D1 = (int)d1;
    p.D2 = (int)d2;
    return FFDAS_SUCCESS;
}

int select_storage(ffdas_datatype_t xt, ffdas_datatype_t ot, ffdas_compute_type_t ct, int batch) {
    switch (xt) {
        // 16-bit channel data: both pair formats interpolate the 16-bit
        // samples exactly (in FP32), so the choice is speed.  For one to a few
        // items the kernels are bound by instruction issue and FP32 pairs need
        // the fewest instructions per tap; for large batches (8 items or more
        // per CTA) the per-tap arithmetic is shared and the pair bytes start
        // to count, so the data keeps its 16-bit pairs.
        case FFDAS_R_16F:
            if (ot != FFDAS_R_32F) return -1;
            // reference: a half-precision compute request on half input is
            // rejected (das_alg1.cu:172-178)
            if (ct == FFDAS_COMPUTE_16F) return -1;
            if (ct == FFDAS_COMPUTE_16BF) return ST_BF16;
            return batch >= 8 ? ST_F16 : ST_F32;   // default or FP32 compute: both formats compute in FP32
        case FFDAS_R_16BF:
            if (ot != FFDAS_R_32F) return -1;
            if (ct == FFDAS_COMPUTE_16F) return ST_F16;
            if (ct == FFDAS_COMPUTE_16BF) return ST_BF16;
            return batch >= 8 ? ST_BF16 : ST_F32;
        case FFDAS_R_32F:
            if (ot != FFDAS_R_32F) return -1;
            if (ct == FFDAS_COMPUTE_16F) return ST_F16;
            if (ct == FFDAS_COMPUTE_16BF) return ST_BF16;
            return ST_F32;
        // int16 channel data (raw ADC samples; the reference rejects the type):
        // FP32 pairs hold every int16 exactly, 16-bit pairs only when asked for
        case FFDAS_R_16I:
            if (ot != FFDAS_R_32F) return -1;
            if (ct == FFDAS_COMPUTE_16F) return ST_F16;
            if (ct == FFDAS_COMPUTE_16BF) return ST_BF16;
            return ST_F32;
        case FFDAS_C_16F:
            if (ot != FFDAS_C_32F) return -1;
            if (ct == FFDAS_COMPUTE_16F || ct == FFDAS_COMPUTE_16BF) return -1;
            return ST_C16;
        case FFDAS_C_32F:
            if (ot != FFDAS_C_32F) return -1;
            if (ct == FFDAS_COMPUTE_16F) return ST_C16;
            if (ct == FFDAS_COMPUTE_16BF) return -1;
            return ST_C32;
        case FFDAS_R_64F:
            if (ot != FFDAS_R_64F) return -1;
            if (ct == FFDAS_COMPUTE_16F || ct == FFDAS_COMPUTE_16BF) return -1;
            return ct == FFDAS_COMPUTE_32F ? ST_F32 : ST_F64;
        case FFDAS_C_64F:
            if (ot != FFDAS_C_64F) return -1;
            if (ct == FFDAS_COMPUTE_16F || ct == FFDAS_COMPUTE_16BF) return -1;
            return ct == FFDAS_COMPUTE_32F ? ST_C32 : ST_C64;
        default:
            return -1;
    }
}

static size_t storage_bytes(int kind) {
    switch (kind) {
        case ST_F32: return 8;
        case ST_F16: return 4;
        case ST_BF16: return 4;
        case ST_F64: return 16;
        case ST_C32: return 16;
        case ST_C16: return 8;
        case ST_C64: return 32;
        default: return 0;
    }
}

// ---------------------------------------------------------------- ingest ---
template <typename Tin, int K>
static ffdas_error_t launch_ingest_t(ffdas_context &h, const das_problem &pb, const void *x,
                                     int64_t npad, void *P, const float *gain, int gain_bstride) {
    const int64_t rows = (int64_t)pb.B * pb.C * pb.S;
    if (rows == 0) return FFDAS_SUCCESS;
    const int64_t bc = (int64_t)pb.B * pb.C;
    if (bc > INT32_MAX || npad % kIngestVec != 0) return FFDAS_ERROR_INTERNAL;
    const int64_t per_block = (int64_t)kIngestThreads * kIngestVec;
    dim3 grid((unsigned)((npad + per_block - 1) / per_block), (unsigned)std::min<int64_t>(pb.S, 65535),
              (unsigned)std::min<int64_t>(bc, 65535));
    ingest_pairs_kernel<Tin, K><<<grid, kIngestThreads, 0, h.stream>>>(
        static_cast<const Tin *>(x), pb.x_bstride, pb.x_cstride, pb.x_sstride, pb.C, pb.S, pb.N,
        (int)bc, npad, static_cast<typename pair_traits<K>::storage *>(P), gain, gain_bstride);
    return ffdas_launch_check(h.stream);
}

// Per-channel gain of the handle (ffdas_set_channel_scale) for a problem:
// the pointer and its batch stride, or an error when its length fits neither
// C nor B * C.
static ffdas_error_t channel_gain(const ffdas_context &h, const das_problem &pb, const float **gain, int *bstride) {
    *gain = nullptr;
    *bstride = 0;
    if (!h.chan_scale) return FFDAS_SUCCESS;
    if (h.chan_scale_count == (int64_t)pb.C) {
        *bstride = 0;
    } else if (h.chan_scale_count == (int64_t)pb.B * pb.C) {
        *bstride = pb.C;
    } else {
        return FFDAS_ERROR_INVALID_ARGUMENT;
    }
    *gain = h.chan_scale;
    return FFDAS_SUCCESS;
}

static ffdas_error_t launch_ingest(ffdas_context &h, const das_problem &pb, ffdas_datatype_t xt,
                                   int kind, const void *x, int64_t npad, void *P) {
    const float *gain = nullptr;
    int gain_bstride = 0;
    FFDAS_TRY(channel_gain(h, pb, &gain, &gain_bstride));
#define FFDAS_INGEST(Tin, K) launch_ingest_t<Tin, K>(h, pb, x, npad, P, gain, gain_bstride)
    switch (xt) {
        case FFDAS_R_32F:
            if (kind == ST_F32) return FFDAS_INGEST(float, ST_F32);
            if (kind == ST_F16) return FFDAS_INGEST(float, ST_F16);
            if (kind == ST_BF16) return FFDAS_INGEST(float, ST_BF16);
            break;
        case FFDAS_R_16F:
            if (kind == ST_F32) return FFDAS_INGEST(__half, ST_F32);
            if (kind == ST_F16) return FFDAS_INGEST(__half, ST_F16);
            if (kind == ST_BF16) return FFDAS_INGEST(__half, ST_BF16);
            break;
        case FFDAS_R_16I:
            if (kind == ST_F32) return FFDAS_INGEST(int16_t, ST_F32);
            if (kind == ST_F16) return FFDAS_INGEST(int16_t, ST_F16);
            if (kind == ST_BF16) return FFDAS_INGEST(int16_t, ST_BF16);
            break;
        case FFDAS_R_16BF:
            if (kind == ST_F32) return FFDAS_INGEST(__nv_bfloat16, ST_F32);
            if (kind == ST_BF16) return FFDAS_INGEST(__nv_bfloat16, ST_BF16);
            if (kind == ST_F16) return FFDAS_INGEST(__nv_bfloat16, ST_F16);
            break;
        case FFDAS_R_64F:
            if (kind == ST_F64) return FFDAS_INGEST(double, ST_F64);
            if (kind == ST_F32) return FFDAS_INGEST(double, ST_F32);
            break;
        case FFDAS_C_32F:
            if (kind == ST_C32) return FFDAS_INGEST(float2, ST_C32);
            if (kind == ST_C16) return FFDAS_INGEST(float2, ST_C16);
            break;
        case FFDAS_C_16F:
            if (kind == ST_C16) return FFDAS_INGEST(__half2, ST_C16);
            break;
        case FFDAS_C_64F:
            if (kind == ST_C64) return FFDAS_INGEST(double2, ST_C64);
            if (kind == ST_C32) return FFDAS_INGEST(double2, ST_C32);
            break;
        default:
            break;
    }
    return FFDAS_ERROR_INTERNAL;
#undef FFDAS_INGEST
}

// Bytes a pair buffer needs for a forward call on x (the pair rows and one
// 256-byte control block), for the default output dtype of x.
ffdas_error_t pair_buffer_bytes(const ffdas_tensor_desc &xd, ffdas_compute_type_t ct, size_t *bytes) {
    ffdas_datatype_t od;
    switch (xd.dtype) {
        case FFDAS_R_64F: od = FFDAS_R_64F; break;
        case FFDAS_C_16F: case FFDAS_C_32F: od = FFDAS_C_32F; break;
        case FFDAS_C_64F: od = FFDAS_C_64F; break;
        default: od = FFDAS_R_32F; break;
    }
    if (xd.ndim != 3 && xd.ndim != 4) return FFDAS_ERROR_INVALID_DIMS;
    const int kind = select_storage(xd.dtype, od, ct, xd.ndim == 4 ? (int)xd.dims[0] : 1);
    if (kind < 0) return FFDAS_ERROR_UNSUPPORTED_TYPE;
    const int o = xd.ndim == 4 ? 1 : 0;
    const int64_t B = xd.ndim == 4 ? xd.dims[0] : 1;
    const int64_t rows = B * xd.dims[o] * xd.dims[o + 1];
    const int64_t npad = pair_row_length((int)xd.dims[o + 2]);
    *bytes = ((((size_t)std::max<int64_t>(rows, 1) * npad * storage_bytes(kind)) + 255) & ~size_t(255)) + 256;
    return FFDAS_SUCCESS;
}

// The pair rows a forward call left in the handle's pair buffer, if they are
// those of this x (same pointer, descriptor, storage and channel scale).
void *reusable_pairs(const ffdas_context &h, const ffdas_tensor_desc &xd, const void *x, int kind) {
    const auto &g = h.pair_sig;
    if (!h.pair_buf || g.buf != h.pair_buf || g.x != x || g.kind != kind || g.scale != h.chan_scale ||
        g.scale_count != h.chan_scale_count || g.desc.ndim != xd.ndim || g.desc.dtype != xd.dtype)
        return nullptr;
    for (int64_t i = 0; i < xd.ndim; i++)
        if (g.desc.dims[i] != xd.dims[i] || g.desc.strides[i] != xd.strides[i]) return nullptr;
    return h.pair_buf;
}

ffdas_error_t ingest_for_backward(ffdas_context &h, const das_problem &pb, ffdas_datatype_t xt, int kind,
                                  const void *x, int64_t npad, void *P) {
    return launch_ingest(h, pb, xt, kind, x, npad, P);
}

// ---------------------------------------------------------------- gather ---
struct schedule {
    int variant = 1;
    int T0 = 16, T1 = 16, T2 = 1;
    int BT = 1;
    int SC = 16;
    int WB = 32;   // staged kernel: pairs per window slot
    int copy = 0;  // staged kernel: copy engine (0 default)
};

// Events per staged pass: the smallest supported chunk covering n events.
static int staged_event_chunk(int n) {
    if (n <= 1) return 1;
    if (n <= 4) return 4;
    if (n <= 8) return 8;
    return 16;
}

static int floor_pow2(int v) {
    int p = 1;
    while (p * 2 <= v) p *= 2;
    return p;
}

// staged_ok: the staged kernel can run this problem; without it a staged
// request falls back to the gather kernel.
static schedule plan_schedule(const ffdas_context &h, const das_problem &pb, int kind, bool staged_ok = false) {
    schedule s;
    const bool real = (kind == ST_F32 || kind == ST_F16 || kind == ST_BF16);
    // batch tile: amortise geometry over batch items, bounded by registers
    s.BT = real ? std::min(8, floor_pow2(std::max(1, pb.B))) : (pb.B >= 4 ? 4 : 1);
    // gather event chunk: 16 for dense lists; 8 for sparse ones (fewer registers,
    // more resident warps for the latency-bound list walk)
    s.SC = (real && pb.n_events > 4) ? ((pb.sparse && s.BT <= 4) ? 8 : 16) : 4;
    // tile: 2-D patch over the two innermost grid dims, 256 threads
    if (pb.D1 <= 1) {
        s.T0 = 256; s.T1 = 1; s.T2 = 1;
    } else if (pb.D0 >= 16 && pb.D1 >= 16) {
        s.T0 = 16; s.T1 = 16; s.T2 = 1;
    } else if (pb.D0 >= 32) {
        s.T0 = 32; s.T1 = 8; s.T2 = 1;
    } else {
        s.T0 = std::max(1, floor_pow2(pb.D0)); s.T1 = 256 / s.T0; s.T2 = 1;
    }
    // Default: the staged kernel for every dense real problem of a few
    // thousand voxels or more -- 512-voxel tiles for one batch item, batch
    // tiles of up to 4 items otherwise; the gather kernel for the rest.
    bool staged_default = false;
    if (staged_ok && pb.V >= 4096) {
        staged_default = true;
        s.variant = 2;
        if (pb.B == 1) {
            if (pb.D1 <= 1) { s.T0 = 512; s.T1 = 1; s.T2 = 1; }
            else { s.T0 = std::min(32, std::max(1, floor_pow2(pb.D0))); s.T1 = 512 / s.T0; s.T2 = 1; }
        }
    }
    if (h.has_config) {
        const ffdas_das_config_t &c = h.config;
        if (c.variant == 1 || c.variant == 2) s.variant = c.variant;   // 3 selects a backward kernel only
        if (c.tile_x || c.tile_y || c.tile_z) {
            s.T0 = c.tile_x ? c.tile_x : 1;
            s.T1 = c.tile_y ? c.tile_y : 1;
            s.T2 = c.tile_z ? c.tile_z : 1;
        }
        if (c.batch_tile) s.BT = c.batch_tile;
        if (c.event_chunk) {
            // gather kernel chunks: 4, 8 (batch tiles up to 4) or 16
            s.SC = c.event_chunk <= 4 ? 4 : ((c.event_chunk <= 8 && real && s.BT <= 4) ? 8 : 16);
        }
        if (c.window) s.WB = c.window <= 32 ? 32 : 64;
        s.copy = c.copy_engine;
    }
    if (s.variant == 2) {
        // staged kernel: event chunk from the count; batch tile from the
        // config, else up to 4 items (512-voxel tiles take one item)
        s.SC = staged_event_chunk(pb.n_events);
        if (h.has_config && h.config.event_chunk) s.SC = staged_event_chunk(h.config.event_chunk);
        int bt = (h.has_config && h.config.batch_tile) ? h.config.batch_tile
                                                        : std::min(8, floor_pow2(std::max(1, pb.B)));
        if (!staged_default && !(h.has_config && h.config.batch_tile)) bt = 1;
        // batch tiles use TMA boxes: not with an explicit cp.async request or without the encoder
        if (!staged_batch_supported() || (h.has_config && h.config.copy_engine == 2)) bt = 1;
        // batch groups of delays widen windows (frame ensembles): default 64-pair windows
        if (bt > 1 && !(h.has_config && h.config.window)) s.WB = 64;
        if (s.T0 * s.T1 * s.T2 == 512) bt = 1;
        bt = std::min(bt, 8);
        if (bt > 1) {
            // batch tiles pair events: chunks of 4 or 8, at most 32 windows per stage
            s.SC = s.SC <= 4 ? 4 : 8;
            if (s.SC * bt > 32) s.SC = 32 / bt;
        }
        s.BT = bt;
    }
    if (!real && s.BT != 1) s.BT = 4;
    if (s.variant == 2 && !staged_ok) s.variant = 1;
    const int tile_voxels = s.T0 * s.T1 * s.T2;
    // the gather kernel runs 256-voxel tiles; the staged kernel 256 or 512
    if (tile_voxels != 256 && !(s.variant == 2 && tile_voxels == 512)) {
        s.T0 = 16; s.T1 = 16; s.T2 = 1;
        if (pb.D1 <= 1) { s.T0 = 256; s.T1 = 1; }
    }
    return s;
}

template <int K, typename OutT, int BT, int SC, bool SPARSE>
static ffdas_error_t launch_gather_t(ffdas_context &h, const gather_params &gp, dim3 grid) {
    das_gather_kernel<K, OutT, BT, SC, SPARSE><<<grid, 256, 0, h.stream>>>(gp);
    return ffdas_launch_check(h.stream);
}

template <int K, typename OutT, bool SPARSE>
static ffdas_error_t launch_gather_bt(ffdas_context &h, const gather_params &gp, const schedule &s,
                                      dim3 grid) {
    constexpr bool real = (K == ST_F32 || K == ST_F16 || K == ST_BF16);
    if constexpr (real) {
        if (s.SC == 16) {
            switch (s.BT) {
                case 1: return launch_gather_t<K, OutT, 1, 16, SPARSE>(h, gp, grid);
                case 2: return launch_gather_t<K, OutT, 2, 16, SPARSE>(h, gp, grid);
                case 4: return launch_gather_t<K, OutT, 4, 16, SPARSE>(h, gp, grid);
                case 8: return launch_gather_t<K, OutT, 8, 16, SPARSE>(h, gp, grid);
                default: break;
            }
        } else if (s.SC == 8) {   // fewer registers than 16: more CTAs per SM for latency-bound lists
            switch (s.BT) {
                case 1: return launch_gather_t<K, OutT, 1, 8, SPARSE>(h, gp, grid);
                case 2: return launch_gather_t<K, OutT, 2, 8, SPARSE>(h, gp, grid);
                case 4: return launch_gather_t<K, OutT, 4, 8, SPARSE>(h, gp, grid);
                default: break;
            }
        } else {
            switch (s.BT) {
                case 1: return launch_gather_t<K, OutT, 1, 4, SPARSE>(h, gp, grid);
                case 2: return launch_gather_t<K, OutT, 2, 4, SPARSE>(h, gp, grid);
                case 4: return launch_gather_t<K, OutT, 4, 4, SPARSE>(h, gp, grid);
                case 8: return launch_gather_t<K, OutT, 8, 4, SPARSE>(h, gp, grid);
                default: break;
            }
        }
    } else {
        if (s.BT == 4) return launch_gather_t<K, OutT, 4, 4, SPARSE>(h, gp, grid);
        return launch_gather_t<K, OutT, 1, 4, SPARSE>(h, gp, grid);
    }
    return FFDAS_ERROR_INVALID_ARGUMENT;
}

template <bool SPARSE>
static ffdas_error_t launch_gather(ffdas_context &h, int kind, ffdas_datatype_t ot,
                                   const gather_params &gp, const schedule &s, dim3 grid) {
    switch (kind) {
        case ST_F32:
            if (ot == FFDAS_R_64F) return launch_gather_bt<ST_F32, double, SPARSE>(h, gp, s, grid);
            return launch_gather_bt<ST_F32, float, SPARSE>(h, gp, s, grid);
        case ST_F16: return launch_gather_bt<ST_F16, float, SPARSE>(h, gp, s, grid);
        case ST_BF16: return launch_gather_bt<ST_BF16, float, SPARSE>(h, gp, s, grid);
        case ST_F64: return launch_gather_bt<ST_F64, double, SPARSE>(h, gp, s, grid);
        case ST_C32:
            if (ot == FFDAS_C_64F) return launch_gather_bt<ST_C32, double2, SPARSE>(h, gp, s, grid);
            return launch_gather_bt<ST_C32, float2, SPARSE>(h, gp, s, grid);
        case ST_C16: return launch_gather_bt<ST_C16, float2, SPARSE>(h, gp, s, grid);
        case ST_C64: return launch_gather_bt<ST_C64, double2, SPARSE>(h, gp, s, grid);
        default: return FFDAS_ERROR_INTERNAL;
    }
}

static void read_beta(ffdas_datatype_t ot, const void *beta, double &re, double &im, int &zero) {
    re = 0.0;
    im = 0.0;
    if (beta) {
        switch (ot) {
            case FFDAS_R_32F: re = *static_cast<const float *>(beta); break;
            case FFDAS_R_64F: re = *static_cast<const double *>(beta); break;
            case FFDAS_C_32F: {
                const float *b = static_cast<const float *>(beta);
                re = b[0]; im = b[1];
                break;
            }
            case FFDAS_C_64F: {
                const double *b = static_cast<const double *>(beta);
                re = b[0]; im = b[1];
                break;
            }
            default: break;
        }
    }
    zero = (re == 0.0 && im == 0.0) ? 1 : 0;
}

ffdas_error_t das_forward(ffdas_context &h, const das_call &a) {
    const ffdas_tensor_desc &xd = *a.x_desc;
    const ffdas_tensor_desc &od = *a.out_desc;

    const int kind = select_storage(xd.dtype, od.dtype, a.compute_type, xd.ndim == 4 ? (int)xd.dims[0] : 1);
    // dtype combination first (reference das.cu:40-82); compute-type
    // rejections are reported at the same code, after the dims checks below.
    const bool combo_ok =
        (xd.dtype == FFDAS_R_16F && od.dtype == FFDAS_R_32F) ||
        (xd.dtype == FFDAS_R_16BF && od.dtype == FFDAS_R_32F) ||
        (xd.dtype == FFDAS_R_16I && od.dtype == FFDAS_R_32F) ||
        (xd.dtype == FFDAS_R_32F && od.dtype == FFDAS_R_32F) ||
        (xd.dtype == FFDAS_C_16F && od.dtype == FFDAS_C_32F) ||
        (xd.dtype == FFDAS_C_32F && od.dtype == FFDAS_C_32F) ||
        (xd.dtype == FFDAS_R_64F && od.dtype == FFDAS_R_64F) ||
        (xd.dtype == FFDAS_C_64F && od.dtype == FFDAS_C_64F);
    if (!combo_ok) return FFDAS_ERROR_UNSUPPORTED_TYPE;

    if (!fits_int32_indexing(xd) || !fits_int32_indexing(od)) return FFDAS_ERROR_INVALID_DIMS;

    const bool f64 = (od.dtype == FFDAS_R_64F || od.dtype == FFDAS_C_64F);
    if (a.sparse) {
        if (a.alg != FFDAS_ALG_DEFAULT && a.alg != FFDAS_ALG1) return FFDAS_ERROR_INVALID_ARGUMENT;
    } else {
        if (f64 && a.alg != FFDAS_ALG_DEFAULT && a.alg != FFDAS_ALG1) return FFDAS_ERROR_UNSUPPORTED_TYPE;
        if (a.alg != FFDAS_ALG_DEFAULT && a.alg != FFDAS_ALG1 && a.alg != FFDAS_ALG2 && a.alg != FFDAS_ALG4)
            return FFDAS_ERROR_INVALID_ARGUMENT;
    }

    das_problem pb;
    FFDAS_TRY(make_problem(xd, od, pb));
    if (a.sparse) {
        if (a.sparse_count <= 0) return FFDAS_ERROR_INVALID_ARGUMENT;
        pb.n_events = a.sparse_count;
        pb.sparse = true;
    } else {
        pb.n_events = pb.S;
    }
    if (kind < 0) return FFDAS_ERROR_UNSUPPORTED_TYPE;
    if (pb.N >= (1 << 22)) return FFDAS_ERROR_DIMS_TOO_LARGE;  // floor split is exact below 2^22

    if (pb.V == 0 || pb.B == 0) return FFDAS_SUCCESS;
    if (!a.out || !a.dstpos || !a.offsets || !a.weights) return FFDAS_ERROR_NULL_POINTER;
    if (pb.C > 0 && !a.srcpos) return FFDAS_ERROR_NULL_POINTER;
    if ((int64_t)pb.B * pb.C * pb.S * pb.N > 0 && !a.x) return FFDAS_ERROR_NULL_POINTER;
    if (a.sparse && !a.sparse_indices) return FFDAS_ERROR_NULL_POINTER;
    h.units_recorded = false;
    h.pair_sig = ffdas_context::pair_signature{};   // set again below if this call fills the pair buffer
    // timed calls: the kernels that count the units they evaluate add into
    // the handle's counter, cleared here, before the timed launch
    if (h.timing && h.unit_count) FFDAS_CUDA(cudaMemsetAsync(h.unit_count, 0, sizeof(unsigned long long), h.stream));

    // a channel scale of the wrong length fails before anything is launched
    {
        const float *g = nullptr;
        int gb = 0;
        FFDAS_TRY(channel_gain(h, pb, &g, &gb));
    }

    // ---- small problems: the whole call as one launch straight from x ----
    // (it reads x in place, so not with a channel scale, which the ingest applies)
    if (!h.chan_scale && direct_supported(pb, xd.dtype, od.dtype, kind)) {
        const bool asked = h.has_config && h.config.variant == 5;
        const bool planner = !h.has_config || h.config.variant == 0;
        const int64_t units = pb.V * pb.C * (int64_t)pb.S * pb.B;
        if (asked || (planner && units <= (pb.B == 1 ? kDirectUnits : kDirectUnitsBatched))) {
            double br = 0.0, bi = 0.0;
            int bz = 1;
            read_beta(od.dtype, a.beta, br, bi, bz);
            return launch_direct(h, pb, xd.dtype, a.x, a.srcpos, a.srcdir, a.dstpos, a.offsets, a.weights,
                                 static_cast<float *>(a.out), br, bz, asked ? h.config.batch_tile : 0,
                                 asked ? h.config.tile_x : 0);
        }
    }

    // ---- ingest: x -> pair rows (workspace) ----
    const int64_t npad = pair_row_length(pb.N);
    const int64_t rows = (int64_t)pb.B * pb.C * pb.S;
    workspace P(h);
    const size_t pair_bytes = ((size_t)std::max<int64_t>(rows, 1) * npad * storage_bytes(kind) + 255) & ~size_t(255);
    // the caller's pair buffer when one is set and large enough (the pair
    // rows then outlive the call, for ffdas_das_backward), else workspace
    void *Pbase = nullptr;
    if (h.pair_buf && h.pair_buf_bytes >= pair_bytes + 256) {
        Pbase = h.pair_buf;
    } else {
        FFDAS_TRY(P.alloc(pair_bytes + (a.sparse ? 256 : 0)));   // das_sparse: a gate word after the pairs
        Pbase = P.get<void>();
    }
    FFDAS_TRY(launch_ingest(h, pb, xd.dtype, kind, a.x, npad, Pbase));
    if (Pbase == h.pair_buf) {
        h.pair_sig.buf = h.pair_buf;
        h.pair_sig.x = a.x;
        h.pair_sig.desc = xd;
        h.pair_sig.kind = kind;
        h.pair_sig.scale = h.chan_scale;
        h.pair_sig.scale_count = h.chan_scale_count;
    }

    // ---- forward kernel ----
    const bool staged_ok = staged_supported(pb, kind) && od.dtype == FFDAS_R_32F;
    const schedule s = plan_schedule(h, pb, kind, staged_ok);
    gather_params gp;
    std::memset(&gp, 0, sizeof(gp));
    gp.P = Pbase;
    gp.npad = npad;
    gp.C = pb.C;
    gp.S = pb.S;
    gp.n_events = pb.n_events;
    gp.B = pb.B;
    gp.V = pb.V;
    gp.D0 = pb.D0; gp.D1 = pb.D1; gp.D2 = pb.D2;
    gp.T0 = s.T0; gp.T1 = s.T1; gp.T2 = s.T2;
    gp.n0 = (pb.D0 + s.T0 - 1) / s.T0;
    gp.n1 = (pb.D1 + s.T1 - 1) / s.T1;
    const int n2 = (pb.D2 + s.T2 - 1) / s.T2;
    gp.srcpos = a.srcpos;
    gp.srcdir = reinterpret_cast<const float4 *>(a.srcdir);
    gp.dstpos = a.dstpos;
    gp.offsets = a.offsets;
    gp.weights = a.weights;
    gp.sparse_idx = a.sparse_indices;
    gp.wavenum = a.wavenum;
    gp.out = a.out;
    gp.out_bstride = pb.out_bstride;
    read_beta(od.dtype, a.beta, gp.beta_re, gp.beta_im, gp.beta_zero);

    const int64_t tiles = (int64_t)gp.n0 * gp.n1 * n2;
    const int bchunks = (pb.B + s.BT - 1) / s.BT;
    if (tiles > INT32_MAX || bchunks > 65535) return FFDAS_ERROR_DIMS_TOO_LARGE;
    dim3 grid((unsigned)tiles, (unsigned)bchunks);

    h.last = ffdas_kernel_info_t{};
    h.last.variant = 1;
    h.last.tile_x = s.T0; h.last.tile_y = s.T1; h.last.tile_z = s.T2;
    h.last.batch_tile = s.BT;
    h.last.event_chunk = s.SC;
    h.last.storage = kind;
    h.last.kernels = 2;
    h.last.grid = tiles * bchunks;

    // Complex (IQ) data on the staged complex kernel when the schedule asks
    // for variant 2: 256-voxel tiles, the gather kernel's event chunk so that
    // both sum in the same order.  The planner keeps complex data on the
    // gather kernel: measured on B200 the two are level for single frames
    // (3-D diverging volume, 1024 channels: 146 ms staged, 152 ms gather,
    // 284 ms reference ALG1) -- both bound by the per-tap sincos and complex
    // multiply-add -- and the gather kernel's batch tiles share the phase
    // over frames (50-frame ensemble: 9.9 ms gather, 34.6 ms staged).
    if ((kind == ST_C32 || kind == ST_C16) && od.dtype == FFDAS_C_32F && !a.sparse && staged_batch_supported() &&
        npad >= 64 && rows < INT32_MAX && pb.B <= 65535 && h.has_config && h.config.variant == 2) {
        gather_params cg = gp;
        cg.cchunk = 0;
        const int SCc = (h.has_config && h.config.event_chunk >= 8) ? 8 : 4;
        h.last.variant = 2;
        h.last.event_chunk = SCc;
        h.last.batch_tile = 1;
        h.last.grid = tiles * pb.B;
        h.mark_start();
        const ffdas_error_t err = launch_staged_cplx(h, pb, kind, cg, SCc, dim3((unsigned)tiles, (unsigned)pb.B));
        h.mark_stop();
        return err;
    }

    const bool staged = s.variant == 2;
    if (staged) {
        const int bchunks_st = (pb.B + s.BT - 1) / s.BT;
        // Small problems (fewer CTAs than the target of min_blocks, default 3,
        // per SM): split each tile's channels over blockIdx.z slices of 32+
        // channels that add into the image, so every SM has work.
        int csplit = 1;
        {
            const int per_sm = (h.has_config && h.config.min_blocks) ? h.config.min_blocks : 3;
            const int64_t ctas = tiles * bchunks_st;
            const int64_t want = (int64_t)std::max(h.sm_count, 1) * per_sm;
            while (ctas * csplit * 2 <= want && pb.C >= 64 * csplit && csplit < 64) csplit *= 2;
        }
        if (csplit > 1) {
            const int chunk = ((pb.C + csplit - 1) / csplit + 31) / 32 * 32;   // whole stages of channels
            csplit = (pb.C + chunk - 1) / chunk;
            gp.cchunk = csplit > 1 ? chunk : 0;
        }
        h.last.variant = 2;
        h.last.batch_tile = s.BT;
        h.last.event_chunk = s.SC;
        h.last.grid = tiles * bchunks_st * csplit;
        h.last.kernels = csplit > 1 ? 3 : 2;   // ingest, (image preparation,) delay-and-sum
        if (bchunks_st > 65535) return FFDAS_ERROR_DIMS_TOO_LARGE;
        h.mark_start();
        const ffdas_error_t err = launch_staged(h, pb, kind, gp, s.SC, s.WB, s.BT, s.copy,
                                                dim3((unsigned)tiles, (unsigned)bchunks_st, (unsigned)csplit));
        h.mark_stop();
        return err;
    }
    // das_sparse as one persistent, load-balanced launch (schedule variant 6):
    // bucketed lists, tiles longest first, voxels ordered by their entries per
    // pass, windows staged by TMA.  A list naming an event twice sets the
    // gate and the gated gather kernel launched after computes the call.
    // Not the planner's default: a window here serves only the tile's voxels
    // that list its event, so the producer's cost per window is spread over
    // few taps; measured on B200 it is slower than the gather kernel on the
    // 128-channel focused frame (1.26 vs 0.60 ms) and than the 512-voxel
    // staged pass on a 1024-channel volume with 8 of 16 transmits per voxel
    // (17.9 vs 9.0 ms).  The tuner offers it.
    {
        const bool real_pairs_i = (kind == ST_F32 || kind == ST_F16 || kind == ST_BF16);
        const bool asked = h.has_config && h.config.variant == 6;
        if (a.sparse && real_pairs_i && od.dtype == FFDAS_R_32F && staged_batch_supported() &&
            sparse_items_supported(pb, kind) && s.T0 * s.T1 * s.T2 == 256 && asked) {
            const int SCi = (h.has_config && h.config.event_chunk && h.config.event_chunk <= 4) ? 4 : 8;
            const int WBi = (h.has_config && h.config.window && h.config.window <= 32) ? 32 : 64;
            const int copy = h.has_config ? h.config.copy_engine : 0;
            // channel slices until the work items are about 4x the CTAs the GPU holds
            int islices = 1;
            {
                const int per_sm = (h.has_config && h.config.min_blocks) ? h.config.min_blocks : 8;
                const int64_t want = (int64_t)std::max(h.sm_count, 1) * per_sm;
                while (tiles * islices * pb.B * 2 <= want && pb.C >= 64 * islices && islices < 64) islices *= 2;
            }
            gather_params ig = gp;
            ig.cchunk = 0;
            if (islices > 1) {
                const int chunk = ((pb.C + islices - 1) / islices + 31) / 32 * 32;   // whole stages of channels
                if ((pb.C + chunk - 1) / chunk > 1) ig.cchunk = chunk;
            }
            workspace IW(h);
            FFDAS_TRY(IW.alloc(sparse_items_workspace(pb, (int)tiles, SCi)));
            int *gate = reinterpret_cast<int *>(static_cast<char *>(Pbase) + pair_bytes);
            h.last.variant = 6;
            h.last.batch_tile = 1;
            h.last.event_chunk = SCi;
            h.last.kernels = ig.cchunk ? 5 : 4;   // ingest, list buckets, tile order, (image preparation,) items
            h.mark_start();
            ffdas_error_t err = launch_sparse_items(h, pb, kind, ig, SCi, WBi, copy, IW.get<void>(), gate);
            if (err == FFDAS_SUCCESS) {
                gather_params fg = gp;
                fg.run_if = gate;
                h.last.kernels += 1;   // the gated gather kernel
                err = launch_gather<true>(h, kind, od.dtype, fg, s, grid);
            }
            h.mark_stop();
            return err;
        }
    }
    // das_sparse on the 512-voxel staged kernel: each pass runs over x's
    // events and each voxel takes the list entry naming the event, so the
    // work is that of the dense call over x's S events.  The planner takes it
    // for 256+ channels and S at most 4x the list length (measured on B200:
    // 3-D volumes of 256-1024 channels 1.5-3.1x faster than the gather
    // kernel; a 128-channel 2-D frame is faster on the gather kernel, whose
    // per-voxel list walk costs less than the staged pass's list scan), or
    // when the schedule asks for variant 2.  A
    // list that names an event twice sets a device gate: the staged kernel
    // then does nothing and the gather kernel, launched after it and
    // otherwise idle, computes the call -- no host round trip, and the call
    // stays capturable in a CUDA graph.
    const bool real_pairs = (kind == ST_F32 || kind == ST_F16 || kind == ST_BF16);
    if (a.sparse && real_pairs && od.dtype == FFDAS_R_32F && staged_batch_supported() && npad >= 64 &&
        rows < INT32_MAX && !(h.has_config && h.config.variant == 1) &&
        ((h.has_config && h.config.variant == 2) ||
         (!h.has_config && pb.C >= 256 && (int64_t)pb.S <= 4 * (int64_t)pb.n_events))) {
        gather_params sg = gp;
        const ffdas_das_config_t *c = h.has_config ? &h.config : nullptr;
        int T0, T1;
        if (c && c->tile_x * (c->tile_y ? c->tile_y : 1) == 512) {
            T0 = c->tile_x; T1 = c->tile_y ? c->tile_y : 1;
        } else if (pb.D1 <= 1) {
            T0 = 512; T1 = 1;
        } else {
            T0 = std::min(32, std::max(1, floor_pow2(pb.D0))); T1 = 512 / T0;
        }
        sg.T0 = T0; sg.T1 = T1; sg.T2 = 1;
        sg.n0 = (pb.D0 + T0 - 1) / T0;
        sg.n1 = (pb.D1 + T1 - 1) / T1;
        sg.cchunk = 0;
        const int64_t stiles = (int64_t)sg.n0 * sg.n1 * pb.D2;
        // channel slices for grids that leave SMs idle, as in the dense call
        int csplit = 1;
        {
            const int per_sm = (c && c->min_blocks) ? c->min_blocks : 3;
            const int64_t want = (int64_t)std::max(h.sm_count, 1) * per_sm;
            while (stiles * pb.B * csplit * 2 <= want && pb.C >= 64 * csplit && csplit < 64) csplit *= 2;
        }
        if (csplit > 1) {
            const int chunk = ((pb.C + csplit - 1) / csplit + 31) / 32 * 32;   // whole stages of channels
            csplit = (pb.C + chunk - 1) / chunk;
            sg.cchunk = csplit > 1 ? chunk : 0;
        }
        const int SCs = (c && c->event_chunk) ? (c->event_chunk <= 1 ? 1 : (c->event_chunk <= 4 ? 4 : 8))
                                              : (pb.S <= 1 ? 1 : (pb.S <= 4 ? 4 : 8));
        const int WBs = (c && c->window > 32) ? 64 : 32;
        const int copy = c ? c->copy_engine : 0;
        if (stiles <= INT32_MAX && pb.B <= 65535) {
            int *gate = reinterpret_cast<int *>(static_cast<char *>(Pbase) + pair_bytes);
            h.last.variant = 2;
            h.last.tile_x = T0; h.last.tile_y = T1; h.last.tile_z = 1;
            h.last.batch_tile = 1;
            h.last.event_chunk = SCs;
            h.last.kernels = csplit > 1 ? 5 : 4;   // ingest, list check, (image preparation,) staged, gated gather
            h.last.grid = stiles * pb.B * csplit;
            h.mark_start();
            ffdas_error_t err = launch_staged_sparse(h, pb, kind, sg, SCs, WBs, copy,
                                                     dim3((unsigned)stiles, (unsigned)pb.B, (unsigned)csplit), gate);
            if (err == FFDAS_SUCCESS) {
                gather_params fg = gp;
                fg.run_if = gate;
                err = launch_gather<true>(h, kind, od.dtype, fg, s, grid);
            }
            h.mark_stop();
            return err;
        }
    }
    // Channel slices for the gather kernel (real data into f32): sparse calls
    // are latency-bound with a few hundred CTAs, so each tile's channels split
    // over blockIdx.z slices (8+ channels) adding into a prepared image until
    // there are about min_blocks (default 16) CTAs per SM -- measured on the
    // 128-channel focused frame: 0.88 ms unsplit with 16-event chunks, 0.60 ms
    // split with 8-event chunks; dense calls split only when the schedule
    // sets min_blocks.
    int gsplit = 1;
    if (real_pairs && od.dtype == FFDAS_R_32F && (a.sparse || (h.has_config && h.config.min_blocks))) {
        const int per_sm = (h.has_config && h.config.min_blocks) ? h.config.min_blocks : 16;
        const int64_t want = (int64_t)std::max(h.sm_count, 1) * per_sm;
        while (tiles * bchunks * gsplit * 2 <= want && pb.C >= 16 * gsplit && gsplit < 64) gsplit *= 2;
    }
    gather_params gq = gp;
    if (gsplit > 1) {
        const int chunk = (pb.C + gsplit - 1) / gsplit;
        gsplit = (pb.C + chunk - 1) / chunk;
        if (gsplit > 1) {
            gq.cchunk = chunk;
            grid.z = (unsigned)gsplit;
            h.last.grid = tiles * bchunks * gsplit;
            h.last.kernels = 3;   // ingest, image preparation, gather
            FFDAS_TRY(launch_scale_image(h, pb, static_cast<float *>(gq.out), (float)gq.beta_re, gq.beta_zero));
        }
    }
    h.mark_start();
    const ffdas_error_t err = a.sparse ? launch_gather<true>(h, kind, od.dtype, gq, s, grid)
                                       : launch_gather<false>(h, kind, od.dtype, gq, s, grid);
    h.mark_stop();
    return err;
}

}  // namespace ffdas

using namespace ffdas;

static ffdas_error_t das_entry(ffdas_handle_t handle, das_call &a) {
    if (!handle) return FFDAS_ERROR_INVALID_HANDLE;
    FFDAS_TRY(handle->check_device());
    if (!a.x_desc || !a.out_desc) return FFDAS_ERROR_NULL_POINTER;
    return das_forward(*handle, a);
}

// ------------------------------------------- host-resident channel data ---
// ffdas_das_from_host: ffdas_das on channel data in host memory.  The
// channels are cut into K chunks; the handle's upload stream copies chunk
// k + 1 (one cudaMemcpyAsync per batch item) while the handle's stream runs
// chunk k's ingest and delay-and-sum, which waits only for its own chunk's
// event; chunk 0 applies the caller's beta and every later chunk adds into
// the image (beta = 1).  So the upload of all but the first chunk hides behind
// the beamforming, where a copy followed by ffdas_das pays for both.
namespace {

constexpr int kHostChunksMax = ffdas_context::kUploadEvents - 1;

ffdas_error_t upload_resources(ffdas_context &h) {
    if (!h.upload_stream) FFDAS_CUDA(cudaStreamCreateWithFlags(&h.upload_stream, cudaStreamNonBlocking));
    for (cudaEvent_t &e : h.upload_ev)
        if (!e) FFDAS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return FFDAS_SUCCESS;
}

// Channels per run: about C / 8 when there are 1024 channels, runs of at
// least 128 channels, rounded to the 8 channels of one staged-kernel stage.
int host_chunk_channels(int64_t C, int chunks) {
    int64_t k = chunks > 0 ? chunks : std::max<int64_t>(1, std::min<int64_t>(8, C / 128));
    // at most kHostChunksMax - 1 full runs: with the half-width first run the
    // runs then fit the kHostChunksMax per-run events
    k = std::min<int64_t>(std::min<int64_t>(k, kHostChunksMax - 1), std::max<int64_t>(C, 1));
    int64_t cc = (C + k - 1) / k;
    if (k > 1) cc = (cc + 7) / 8 * 8;
    return (int)std::max<int64_t>(cc, 1);
}

ffdas_error_t das_from_host(ffdas_context &h, const das_call &a0, int chunks) {
    const ffdas_tensor_desc &xd = *a0.x_desc;
    if (xd.ndim != 3 && xd.ndim != 4) return FFDAS_ERROR_INVALID_DIMS;
    const size_t esz = ffdas_type_size(xd.dtype);
    if (esz == 0) return FFDAS_ERROR_UNSUPPORTED_TYPE;
    int64_t expect = 1;
    for (int i = (int)xd.ndim - 1; i >= 0; i--) {   // C-contiguous: chunks are runs of whole channels
        if (xd.dims[i] > 1 && xd.strides[i] != expect) return FFDAS_ERROR_NON_CONTIGUOUS;
        expect *= xd.dims[i];
    }
    const int cdim = (int)xd.ndim - 3;
    const int64_t B = xd.ndim == 4 ? xd.dims[0] : 1, C = xd.dims[cdim];
    const int64_t row = xd.dims[cdim + 1] * xd.dims[cdim + 2];          // S * N elements per channel
    const int64_t total = B * C * row;
    if (total > 0 && !a0.x) return FFDAS_ERROR_NULL_POINTER;
    if (C > 0 && !a0.srcpos) return FFDAS_ERROR_NULL_POINTER;
    // a per-item channel scale (B x C values) does not split by channel
    const bool item_scale = h.chan_scale && h.chan_scale_count != C;
    const int cc = item_scale ? (int)std::max<int64_t>(C, 1) : host_chunk_channels(C, chunks);
    // Run k covers channels [run_lo(k), run_lo(k + 1)).  The first run's
    // upload is the one copy nothing hides, so it is half a run (whole
    // stages of 8 channels) when there are several runs.
    const int64_t first = (cc >= C) ? C : std::min<int64_t>(C, std::max<int64_t>(8, (cc / 2 + 7) / 8 * 8));
    const int K = (int)(first >= C ? 1 : 1 + (C - first + cc - 1) / cc);
    auto run_lo = [&](int k) -> int64_t { return k == 0 ? 0 : std::min<int64_t>(C, first + (int64_t)(k - 1) * cc); };
    if (K > kHostChunksMax) return FFDAS_ERROR_INTERNAL;

    FFDAS_TRY(upload_resources(h));
    workspace X(h);
    FFDAS_TRY(X.alloc((size_t)std::max<int64_t>(total, 1) * esz));
    unsigned char *xdev = X.get<unsigned char>();
    const unsigned char *xh = static_cast<const unsigned char *>(a0.x);
    // the uploads start after the work already queued on the handle's stream
    // (the staging buffer's allocation among it)
    FFDAS_CUDA(cudaEventRecord(h.upload_ev[kHostChunksMax], h.stream));
    FFDAS_CUDA(cudaStreamWaitEvent(h.upload_stream, h.upload_ev[kHostChunksMax], 0));
    ffdas_error_t cerr = FFDAS_SUCCESS;
    for (int k = 0; k < K && cerr == FFDAS_SUCCESS; k++) {
        const int64_t c0 = run_lo(k), c1 = run_lo(k + 1);
        for (int64_t b = 0; b < B && cerr == FFDAS_SUCCESS; b++) {
            const size_t off = (size_t)((b * C + c0) * row) * esz;
            if (cudaMemcpyAsync(xdev + off, xh + off, (size_t)((c1 - c0) * row) * esz, cudaMemcpyHostToDevice,
                                h.upload_stream) != cudaSuccess)
                cerr = FFDAS_ERROR_CUDA_MEMCPY_FAILED;
        }
        if (cerr == FFDAS_SUCCESS && cudaEventRecord(h.upload_ev[k], h.upload_stream) != cudaSuccess)
            cerr = FFDAS_ERROR_CUDA_RUNTIME;
    }
    // The end of this call's uploads, recorded whatever happened above: the
    // handle's stream waits for it before the staging buffer is released.
    const cudaEvent_t uploads_done = h.upload_ev[kHostChunksMax];
    cudaEventRecord(uploads_done, h.upload_stream);
    if (cerr != FFDAS_SUCCESS) {
        cudaStreamWaitEvent(h.stream, uploads_done, 0);
        return cerr;
    }

    // beta = 1 of the output type, for the chunks after the first
    const float one_f[2] = {1.f, 0.f};
    const double one_d[2] = {1.0, 0.0};
    const ffdas_datatype_t ot = a0.out_desc->dtype;
    const void *one = (ot == FFDAS_R_64F || ot == FFDAS_C_64F) ? static_cast<const void *>(one_d)
                                                                : static_cast<const void *>(one_f);
    // chunks neither fill nor read the caller's pair buffer
    void *const saved_buf = h.pair_buf;
    const size_t saved_bytes = h.pair_buf_bytes;
    const float *const saved_scale = h.chan_scale;
    const int64_t saved_count = h.chan_scale_count;
    h.pair_buf = nullptr;
    h.pair_buf_bytes = 0;
    ffdas_error_t err = FFDAS_SUCCESS;
    int kernels = 0;
    for (int k = 0; k < K && err == FFDAS_SUCCESS; k++) {
        const int64_t c0 = run_lo(k), c1 = run_lo(k + 1);
        ffdas_tensor_desc dk = xd;
        dk.dims[cdim] = c1 - c0;
        das_call a = a0;
        a.x_desc = &dk;
        a.x = xdev + (size_t)(c0 * row) * esz;
        a.srcpos = a0.srcpos + 3 * c0;
        a.srcdir = a0.srcdir ? a0.srcdir + 4 * c0 : nullptr;
        a.beta = k == 0 ? a0.beta : one;
        if (saved_scale && !item_scale) {
            h.chan_scale = saved_scale + c0;
            h.chan_scale_count = c1 - c0;
        }
        err = cudaStreamWaitEvent(h.stream, h.upload_ev[k], 0) == cudaSuccess ? FFDAS_SUCCESS
                                                                                : FFDAS_ERROR_CUDA_RUNTIME;
        if (err == FFDAS_SUCCESS) err = das_forward(h, a);
        kernels += h.last.kernels;
    }
    h.pair_buf = saved_buf;
    h.pair_buf_bytes = saved_bytes;
    h.chan_scale = saved_scale;
    h.chan_scale_count = saved_count;
    h.last.kernels = kernels;
    // every upload lands before the staging buffer is released on the
    // handle's stream, whatever happened above
    if (cudaStreamWaitEvent(h.stream, uploads_done, 0) != cudaSuccess && err == FFDAS_SUCCESS)
        err = FFDAS_ERROR_CUDA_RUNTIME;
    return err;
}

}  // namespace

extern "C" {

ffdas_error_t ffdas_das_from_host(ffdas_handle_t handle, const float *srcpos, const float *srcdir, float wavenum,
                                  ffdas_tensor_desc_t x_desc, const void *x_host, const float *dstpos,
                                  const float *offsets, const float *weights, const void *beta,
                                  ffdas_tensor_desc_t out_desc, void *out, ffdas_compute_type_t compute_type,
                                  ffdas_alg_t alg, int chunks) {
    if (!handle) return FFDAS_ERROR_INVALID_HANDLE;
    FFDAS_TRY(handle->check_device());
    if (!x_desc || !out_desc) return FFDAS_ERROR_NULL_POINTER;
    if (chunks < 0) return FFDAS_ERROR_INVALID_ARGUMENT;
    das_call a;
    a.srcpos = srcpos; a.srcdir = srcdir; a.wavenum = wavenum;
    a.x_desc = x_desc; a.x = x_host; a.dstpos = dstpos; a.offsets = offsets; a.weights = weights;
    a.beta = beta; a.out_desc = out_desc; a.out = out;
    a.compute_type = compute_type; a.alg = alg; a.sparse = false;
    return das_from_host(*handle, a, chunks);
}

ffdas_error_t ffdas_das_pair_bytes(ffdas_tensor_desc_t x_desc, ffdas_compute_type_t compute_type, size_t *bytes) {
    if (!x_desc || !bytes) return FFDAS_ERROR_NULL_POINTER;
    return pair_buffer_bytes(*x_desc, compute_type, bytes);
}

ffdas_error_t ffdas_set_pair_buffer(ffdas_handle_t handle, void *buffer, size_t bytes) {
    if (!handle) return FFDAS_ERROR_INVALID_HANDLE;
    if (buffer && bytes == 0) return FFDAS_ERROR_INVALID_ARGUMENT;
    handle->pair_buf = buffer;
    handle->pair_buf_bytes = buffer ? bytes : 0;
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_das(ffdas_handle_t handle, const float *srcpos, const float *srcdir,
                        float wavenum, ffdas_tensor_desc_t x_desc, const void *x,
                        const float *dstpos, const float *offsets, const float *weights,
                        const void *beta, ffdas_tensor_desc_t out_desc, void *out,
                        ffdas_compute_type_t compute_type, ffdas_alg_t alg) {
    das_call a;
    a.srcpos = srcpos; a.srcdir = srcdir; a.wavenum = wavenum;
    a.x_desc = x_desc; a.x = x; a.dstpos = dstpos; a.offsets = offsets; a.weights = weights;
    a.beta = beta; a.out_desc = out_desc; a.out = out;
    a.compute_type = compute_type; a.alg = alg; a.sparse = false;
    return das_entry(handle, a);
}

ffdas_error_t ffdas_das_sparse(ffdas_handle_t handle, const float *srcpos, const float *srcdir,
                               float wavenum, ffdas_tensor_desc_t x_desc, const void *x,
                               const float *dstpos, const float *offsets, const float *weights,
                               int sparse_count, const int *sparse_indices, const void *beta,
                               ffdas_tensor_desc_t out_desc, void *out,
                               ffdas_compute_type_t compute_type, ffdas_alg_t alg) {
    das_call a;
    a.srcpos = srcpos; a.srcdir = srcdir; a.wavenum = wavenum;
    a.x_desc = x_desc; a.x = x; a.dstpos = dstpos; a.offsets = offsets; a.weights = weights;
    a.sparse_count = sparse_count; a.sparse_indices = sparse_indices;
    a.beta = beta; a.out_desc = out_desc; a.out = out;
    a.compute_type = compute_type; a.alg = alg; a.sparse = true;
    return das_entry(handle, a);
}

}  // extern "C"

// ------------------------------------------------- allocation-free variant ---
// ffdas_das_static: the forward delay-and-sum for callers that cannot allocate
// device memory -- a real-time thread or an embedded host that forbids
// cudaMalloc, a memory budget that is fixed before the first frame, or a caller
// with no ffdas handle (creating one allocates its workspace pool).  Instead of
// workspace from a pool, the interpolation-pair rows live in the file-scope
// array below, which every GPU that loads this library holds until exit.  The
// entry point calls no cudaMalloc/cudaFree and no allocating library routine.
namespace {

constexpr size_t kStaticPairBytes = size_t(16) << 20;   // 16 MiB per GPU
constexpr int kStaticMaxDevices = 64;
static __device__ __align__(256) unsigned char g_static_pairs[kStaticPairBytes];

std::mutex g_static_mu;

// Per-device set-up of the static entry: the array's device address and the
// device properties the planner reads.  It is tied to the CUDA context it was
// made in (by the context's unique id), so a context torn down and created
// again -- cudaDeviceReset, a primary context released by another library --
// gets a fresh lookup instead of a stale address.
struct static_device_setup {
    unsigned long long ctx_id = 0;   // 0: not set up
    void *pairs = nullptr;
    int sm_count = 0, arch_code = 0;
    size_t smem_optin = 0;
};
static_device_setup g_static_setup[kStaticMaxDevices];

using ctx_get_current_fn = CUresult (*)(CUcontext *);
using ctx_get_id_fn = CUresult (*)(CUcontext, unsigned long long *);

// Unique id of the calling thread's current context (driver entry points
// fetched through the runtime, like the tensor-map encoder).
ffdas_error_t current_context_id(unsigned long long *id) {
    static ctx_get_current_fn get_current = nullptr;
    static ctx_get_id_fn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<ctx_get_current_fn>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<ctx_get_id_fn>(p);
        cudaGetLastError();
    });
    if (!get_current || !get_id) return FFDAS_ERROR_CUDA_DRIVER;
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return FFDAS_ERROR_CUDA_DRIVER;
    if (get_id(ctx, id) != CUDA_SUCCESS) return FFDAS_ERROR_CUDA_DRIVER;
    return FFDAS_SUCCESS;
}

// Set-up for the current device: looked up once per device and context
// (host code may not use the symbol itself: its host-side name is a
// stand-in, not a device address).  The queries allocate nothing.
ffdas_error_t static_setup(int *device, static_device_setup *out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return FFDAS_ERROR_CUDA_RUNTIME;
    }
    if (dev < 0 || dev >= kStaticMaxDevices) return FFDAS_ERROR_INVALID_DEVICE;
    unsigned long long ctx_id = 0;
    if (current_context_id(&ctx_id) != FFDAS_SUCCESS) {
        // no current context yet on this thread: cudaSetDevice makes the
        // device's primary context current (it allocates no device memory)
        if (cudaSetDevice(dev) != cudaSuccess) {
            cudaGetLastError();
            return FFDAS_ERROR_CUDA_RUNTIME;
        }
        FFDAS_TRY(current_context_id(&ctx_id));
    }
    std::lock_guard<std::mutex> lock(g_static_mu);
    static_device_setup &st = g_static_setup[dev];
    if (st.ctx_id != ctx_id) {
        static_device_setup fresh;
        if (cudaGetSymbolAddress(&fresh.pairs, g_static_pairs) != cudaSuccess || !fresh.pairs) {
            cudaGetLastError();
            return FFDAS_ERROR_CUDA_RUNTIME;
        }
        int major = 0, minor = 0, optin = 0;
        if (cudaDeviceGetAttribute(&fresh.sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
            cudaGetLastError();
            return FFDAS_ERROR_CUDA_RUNTIME;
        }
        // same rules and encoding as ffdas_create
        if (major < 10) return FFDAS_ERROR_INSUFFICIENT_COMPUTE_CAPABILITY;
        if (major != 10) return FFDAS_ERROR_DEVICE_NOT_SUPPORTED;
        fresh.arch_code = major * 100 + minor * 10;
        fresh.smem_optin = (size_t)optin;
        fresh.ctx_id = ctx_id;
        st = fresh;
    }
    *device = dev;
    *out = st;
    return FFDAS_SUCCESS;
}

}  // namespace

extern "C" ffdas_error_t ffdas_das_static(uintptr_t stream, const float *srcpos, const float *srcdir,
                                          float wavenum, ffdas_tensor_desc_t x_desc, const void *x,
                                          const float *dstpos, const float *offsets, const float *weights,
                                          const void *beta, ffdas_tensor_desc_t out_desc, void *out,
                                          ffdas_compute_type_t compute_type, ffdas_alg_t alg) {
    if (!x_desc || !out_desc) return FFDAS_ERROR_NULL_POINTER;
    const ffdas_tensor_desc &xd = *x_desc;
    const ffdas_tensor_desc &od = *out_desc;
    const bool combo_ok = (xd.dtype == FFDAS_R_16F || xd.dtype == FFDAS_R_16BF || xd.dtype == FFDAS_R_32F ||
                           xd.dtype == FFDAS_R_16I) &&
                          od.dtype == FFDAS_R_32F;
    if (!combo_ok) return FFDAS_ERROR_UNSUPPORTED_TYPE;   // real channel data, float output
    if (!fits_int32_indexing(xd) || !fits_int32_indexing(od)) return FFDAS_ERROR_INVALID_DIMS;
    if (alg != FFDAS_ALG_DEFAULT && alg != FFDAS_ALG1 && alg != FFDAS_ALG2 && alg != FFDAS_ALG4)
        return FFDAS_ERROR_INVALID_ARGUMENT;
    das_problem pb;
    FFDAS_TRY(make_problem(xd, od, pb));
    pb.n_events = pb.S;
    const int kind = select_storage(xd.dtype, od.dtype, compute_type, pb.B);
    if (kind < 0) return FFDAS_ERROR_UNSUPPORTED_TYPE;
    if (pb.N >= (1 << 22)) return FFDAS_ERROR_DIMS_TOO_LARGE;
    if (pb.V == 0 || pb.B == 0) return FFDAS_SUCCESS;
    if (!out || !dstpos || !offsets || !weights) return FFDAS_ERROR_NULL_POINTER;
    if (pb.C > 0 && !srcpos) return FFDAS_ERROR_NULL_POINTER;
    if ((int64_t)pb.B * pb.C * pb.S * pb.N > 0 && !x) return FFDAS_ERROR_NULL_POINTER;

    // the pair rows must fit the static array; larger problems use ffdas_das
    const int64_t npad = pair_row_length(pb.N);
    const int64_t rows = (int64_t)pb.B * pb.C * pb.S;
    const size_t bytes = (size_t)std::max<int64_t>(rows, 1) * npad * storage_bytes(kind);
    if (bytes > kStaticPairBytes) return FFDAS_ERROR_DIMS_TOO_LARGE;
    static_device_setup st;
    int dev = -1;
    FFDAS_TRY(static_setup(&dev, &st));
    void *P = st.pairs;

    // A handle-shaped view of the caller's stream and device: no pool, no
    // status word, no events.
    ffdas_context ctx;
    ctx.stream = reinterpret_cast<cudaStream_t>(stream);
    ctx.device_id = dev;
    ctx.sm_count = st.sm_count;
    ctx.arch_code = st.arch_code;
    ctx.smem_optin = st.smem_optin;
    // Every pair of every row is rewritten by the ingest pass, so nothing left
    // in the array by an earlier call needs clearing.
    FFDAS_TRY(launch_ingest(ctx, pb, xd.dtype, kind, x, npad, P));

    const schedule s = plan_schedule(ctx, pb, kind);
    gather_params gp;
    std::memset(&gp, 0, sizeof(gp));
    gp.P = P;
    gp.npad = npad;
    gp.C = pb.C; gp.S = pb.S; gp.n_events = pb.n_events; gp.B = pb.B; gp.V = pb.V;
    gp.D0 = pb.D0; gp.D1 = pb.D1; gp.D2 = pb.D2;
    gp.T0 = s.T0; gp.T1 = s.T1; gp.T2 = s.T2;
    gp.n0 = (pb.D0 + s.T0 - 1) / s.T0;
    gp.n1 = (pb.D1 + s.T1 - 1) / s.T1;
    const int n2 = (pb.D2 + s.T2 - 1) / s.T2;
    gp.srcpos = srcpos;
    gp.srcdir = reinterpret_cast<const float4 *>(srcdir);
    gp.dstpos = dstpos; gp.offsets = offsets; gp.weights = weights;
    gp.wavenum = wavenum;
    gp.out = out;
    gp.out_bstride = pb.out_bstride;
    read_beta(od.dtype, beta, gp.beta_re, gp.beta_im, gp.beta_zero);
    const int64_t tiles = (int64_t)gp.n0 * gp.n1 * n2;
    const int bchunks = (pb.B + s.BT - 1) / s.BT;
    if (tiles > INT32_MAX || bchunks > 65535) return FFDAS_ERROR_DIMS_TOO_LARGE;
    return launch_gather<false>(ctx, kind, od.dtype, gp, s, dim3((unsigned)tiles, (unsigned)bchunks));
}
