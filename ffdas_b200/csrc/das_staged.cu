// das_staged.cu -- host side of the TMA-staged forward and adjoint kernels.
//
// Builds the 2-D tensor map over the pair rows (inner dim = pairs of a row,
// outer dim = rows; 8-byte or 4-byte elements; box = WB pairs x 1 row;
// out-of-bounds elements fill with zeros) and launches one CTA per (voxel
// tile, batch item).  cuTensorMapEncodeTiled is fetched through
// cudaGetDriverEntryPoint so the library has no link-time dependency on
// libcuda.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>

#include "core.h"
#include "das_problem.h"
#include "das_staged.cuh"
#include "das_sparse_items.cuh"

namespace ffdas {

constexpr int kDefaultCopy = 1;   // TMA tile loads

// Shared with the tensor-core Gram of truncate_rank (gram_tc.cuh).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        cudaGetLastError();
    });
    return fn;
}

bool staged_supported(const das_problem &pb, int kind) {
    if (pb.sparse) return false;
    if (kind != ST_F32 && kind != ST_F16 && kind != ST_BF16) return false;
    const int64_t rows = (int64_t)pb.B * pb.C * pb.S;
    // pair rows at least as long as the widest window (64 pairs)
    return rows > 0 && rows < INT32_MAX && pb.B <= 65535 && pair_row_length(pb.N) >= 64;
}

// Copy engine actually used: TMA needs the driver's tensor-map encoder.
static int resolve_copy(int copy) {
    if (copy == 0) copy = kDefaultCopy;
    if (copy == 1 && tensor_map_encoder() == nullptr) copy = 2;
    return copy;
}

// Tensor map over the pair rows: dims {npad, rows}, box {WB, 1}, zero OOB fill.
static int staged_pair_bytes(int kind) {
    return kind == ST_C32 ? 16 : ((kind == ST_F32 || kind == ST_C16) ? 8 : 4);
}

// 2-D map over the pair rows (one row per item, channel, event); a 16-byte
// (complex f32) pair is two 8-byte elements, so its x coordinates and box
// width count elements, not pairs.
static ffdas_error_t pair_row_map(CUtensorMap &map, const void *P, int64_t npad, int64_t rows, int kind, int WB) {
    auto encode = tensor_map_encoder();
    if (!encode) return FFDAS_ERROR_CUDA_DRIVER;
    const int pair_bytes = staged_pair_bytes(kind);
    const int units = pair_bytes == 16 ? 2 : 1;
    const cuuint64_t dims[2] = {(cuuint64_t)(npad * units), (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)npad * pair_bytes};
    const cuuint32_t box[2] = {(cuuint32_t)(WB * units), 1u};
    const cuuint32_t estr[2] = {1u, 1u};
    const CUresult r = encode(&map, pair_bytes >= 8 ? CU_TENSOR_MAP_DATA_TYPE_UINT64 : CU_TENSOR_MAP_DATA_TYPE_UINT32,
                              2, const_cast<void *>(P), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? FFDAS_SUCCESS : FFDAS_ERROR_CUDA_DRIVER;
}

// 3-D map over the same rows for batch tiles: dims {npad, C*S, B}, box
// {WB, 1, BT}; batch items past B read as zeros.
static ffdas_error_t pair_batch_map(CUtensorMap &map, const void *P, int64_t npad, int64_t cs, int64_t B, int kind,
                                    int WB, int BT) {
    auto encode = tensor_map_encoder();
    if (!encode) return FFDAS_ERROR_CUDA_DRIVER;
    const int pair_bytes = (kind == ST_F32) ? 8 : 4;
    const cuuint64_t dims[3] = {(cuuint64_t)npad, (cuuint64_t)cs, (cuuint64_t)B};
    const cuuint64_t strides[2] = {(cuuint64_t)npad * pair_bytes, (cuuint64_t)(cs * npad * pair_bytes)};
    const cuuint32_t box[3] = {(cuuint32_t)WB, 1u, (cuuint32_t)BT};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    const CUresult r = encode(&map, pair_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_UINT64 : CU_TENSOR_MAP_DATA_TYPE_UINT32,
                              3, const_cast<void *>(P), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? FFDAS_SUCCESS : FFDAS_ERROR_CUDA_DRIVER;
}

bool staged_batch_supported() { return tensor_map_encoder() != nullptr; }

template <typename Kernel>
static ffdas_error_t prepare_kernel(Kernel kernel, size_t smem) {
    FFDAS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // all of the unified L1/shared array as shared memory: several CTAs per SM
    FFDAS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    (int)cudaSharedmemCarveoutMaxShared));
    return FFDAS_SUCCESS;
}

// Kernel attributes (dynamic shared memory above 48 KB, carveout) belong to a
// device: set them once for every device the process launches the kernel on.
template <auto Kernel>
static ffdas_error_t prepare_once(size_t smem) {
    static std::atomic<unsigned long long> done{0ull};
    int dev = 0;
    FFDAS_CUDA(cudaGetDevice(&dev));
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return FFDAS_SUCCESS;
    FFDAS_TRY(prepare_kernel(Kernel, smem));
    done.fetch_or(bit, std::memory_order_release);
    return FFDAS_SUCCESS;
}

template <int K, int SC, int WB>
static ffdas_error_t launch_fwd_t(ffdas_context &h, const staged_params &sp, const CUtensorMap &map, dim3 grid) {
    constexpr size_t smem = staged_smem_bytes<WB, K>();
    FFDAS_TRY((prepare_once<das_staged_kernel<K, SC, WB>>(smem)));
    das_staged_kernel<K, SC, WB><<<grid, kStThreads, smem, h.stream>>>(sp, map);
    return ffdas_launch_check(h.stream);
}

template <int K, int SC, int WB>
static ffdas_error_t launch_fwd2_t(ffdas_context &h, const staged_params &sp, const CUtensorMap &map, dim3 grid) {
    constexpr size_t smem = staged_smem_bytes<WB, K>();
    FFDAS_TRY((prepare_once<das_staged2_kernel<K, SC, WB>>(smem)));
    das_staged2_kernel<K, SC, WB><<<grid, kStThreads, smem, h.stream>>>(sp, map);
    return ffdas_launch_check(h.stream);
}

template <int K, int SC, int WB, int BT>
static ffdas_error_t launch_fwdb_t(ffdas_context &h, const staged_params &sp, const CUtensorMap &map, dim3 grid) {
    constexpr size_t smem = staged_batch_smem_bytes<WB, K, BT>();
    FFDAS_TRY((prepare_once<das_staged_batch_kernel<K, SC, WB, BT>>(smem)));
    das_staged_batch_kernel<K, SC, WB, BT><<<grid, kStThreads, smem, h.stream>>>(sp, map);
    return ffdas_launch_check(h.stream);
}

template <int K, int WB>
static ffdas_error_t launch_fwd_batch(ffdas_context &h, const staged_params &sp, const CUtensorMap &map, int SC,
                                      int BT, dim3 grid) {
    if (BT == 2) return SC <= 4 ? launch_fwdb_t<K, 4, WB, 2>(h, sp, map, grid) : launch_fwdb_t<K, 8, WB, 2>(h, sp, map, grid);
    if (BT == 4) return SC <= 4 ? launch_fwdb_t<K, 4, WB, 4>(h, sp, map, grid) : launch_fwdb_t<K, 8, WB, 4>(h, sp, map, grid);
    return launch_fwdb_t<K, 4, WB, 8>(h, sp, map, grid);
}

template <int K, int SC, int WB>
static ffdas_error_t launch_bwd_t(ffdas_context &h, const staged_params &sp, const CUtensorMap &map, dim3 grid) {
    constexpr size_t smem = staged_bwd_smem_bytes<WB, K, SC>();
    FFDAS_TRY((prepare_once<das_staged_bwd_kernel<K, SC, WB>>(smem)));
    das_staged_bwd_kernel<K, SC, WB><<<grid, kStThreads, smem, h.stream>>>(sp, map);
    return ffdas_launch_check(h.stream);
}

template <int K, int WB>
static ffdas_error_t launch_fwd_sc(ffdas_context &h, const staged_params &sp, const CUtensorMap &map, int SC,
                                   dim3 grid) {
    if (sp.T0 * sp.T1 * sp.T2 == 2 * kStConsumers) {   // 512-voxel tiles: two voxels per thread
        h.units_recorded = sp.units != nullptr;            // this kernel counts the units it evaluates
        // event chunks of 1, 4 (three CTAs per SM) or 8 (two CTAs per SM)
        switch (SC) {
            case 1: return launch_fwd2_t<K, 1, WB>(h, sp, map, grid);
            case 4: return launch_fwd2_t<K, 4, WB>(h, sp, map, grid);
            default: return launch_fwd2_t<K, 8, WB>(h, sp, map, grid);
        }
    }
    switch (SC) {
        case 1: return launch_fwd_t<K, 1, WB>(h, sp, map, grid);
        case 4: return launch_fwd_t<K, 4, WB>(h, sp, map, grid);
        case 8: return launch_fwd_t<K, 8, WB>(h, sp, map, grid);
        default: return launch_fwd_t<K, 16, WB>(h, sp, map, grid);
    }
}

template <int K, int WB, int BT>
static ffdas_error_t launch_bwdb_t(ffdas_context &h, const staged_params &sp, const CUtensorMap &map, dim3 grid) {
    constexpr size_t smem = staged_bwd_batch_smem_bytes<WB, K, 4, BT>();
    FFDAS_TRY((prepare_once<das_staged_bwd_batch_kernel<K, 4, WB, BT>>(smem)));
    das_staged_bwd_batch_kernel<K, 4, WB, BT><<<grid, kStThreads, smem, h.stream>>>(sp, map);
    return ffdas_launch_check(h.stream);
}

// Batch tiles of 2 or 4 items (eight would spill), event chunk 4.
template <int K, int WB>
static ffdas_error_t launch_bwd_batch(ffdas_context &h, const staged_params &sp, const CUtensorMap &map, int BT,
                                      dim3 grid) {
    if (BT == 2) return launch_bwdb_t<K, WB, 2>(h, sp, map, grid);
    return launch_bwdb_t<K, WB, 4>(h, sp, map, grid);
}

template <int K, int WB>
static ffdas_error_t launch_bwd_sc(ffdas_context &h, const staged_params &sp, const CUtensorMap &map, int SC,
                                   dim3 grid) {
    // event chunks of 1 or 4: eight events per pass would spill registers
    return SC == 1 ? launch_bwd_t<K, 1, WB>(h, sp, map, grid) : launch_bwd_t<K, 4, WB>(h, sp, map, grid);
}

static staged_params base_params(ffdas_context &h, const das_problem &pb, const gather_params &gp) {
    staged_params sp;
    std::memset(&sp, 0, sizeof(sp));
    sp.P = gp.P;
    sp.npad = gp.npad;
    sp.C = gp.C; sp.S = gp.S; sp.N = pb.N; sp.n_events = gp.n_events; sp.B = gp.B; sp.V = gp.V;
    sp.D0 = gp.D0; sp.D1 = gp.D1; sp.D2 = gp.D2;
    sp.T0 = gp.T0; sp.T1 = gp.T1; sp.T2 = gp.T2; sp.n0 = gp.n0; sp.n1 = gp.n1;
    sp.srcpos = gp.srcpos; sp.srcdir = gp.srcdir; sp.dstpos = gp.dstpos;
    sp.offsets = gp.offsets; sp.weights = gp.weights;
    sp.out = gp.out; sp.out_bstride = gp.out_bstride;
    sp.beta_re = gp.beta_re; sp.beta_im = gp.beta_im; sp.beta_zero = gp.beta_zero;
    sp.wavenum = gp.wavenum;
    sp.status = h.status;
    sp.units = h.timing ? h.unit_count : nullptr;
    sp.debug_drop_stage = ffdas_take_debug_drop_stage();
    sp.cchunk = gp.cchunk;
    return sp;
}

ffdas_error_t launch_scale_image(ffdas_context &h, const das_problem &pb, float *out, float beta, int beta_zero) {
    dim3 sg((unsigned)((pb.V + 255) / 256), (unsigned)std::min(pb.B, 65535));
    scale_image_kernel<<<sg, 256, 0, h.stream>>>(out, pb.out_bstride, pb.V, pb.B, beta, beta_zero, nullptr);
    return ffdas_launch_check(h.stream);
}

ffdas_error_t launch_staged(ffdas_context &h, const das_problem &pb, int kind, const gather_params &gp, int SC,
                            int WB, int BT, int copy, dim3 grid) {
    if (gp.cchunk) {   // channel slices add into the image: prepare it (beta * out, or 0)
        if (grid.z < 2) return FFDAS_ERROR_INTERNAL;
        dim3 sg((unsigned)((pb.V + 255) / 256), (unsigned)std::min(pb.B, 65535));
        scale_image_kernel<<<sg, 256, 0, h.stream>>>(static_cast<float *>(gp.out), pb.out_bstride, pb.V, pb.B,
                                                     (float)gp.beta_re, gp.beta_zero, nullptr);
        FFDAS_TRY(ffdas_launch_check(h.stream));
    }
    if (BT > 1) copy = 1;   // batch tiles stage their windows with 3-D TMA boxes
    copy = resolve_copy(copy);
    if (BT > 1 && copy != 1) return FFDAS_ERROR_CUDA_DRIVER;
    CUtensorMap map;
    std::memset(&map, 0, sizeof(map));
    if (copy == 1 && BT > 1)
        FFDAS_TRY(pair_batch_map(map, gp.P, gp.npad, (int64_t)pb.C * pb.S, pb.B, kind, WB, BT));
    else if (copy == 1)
        FFDAS_TRY(pair_row_map(map, gp.P, gp.npad, (int64_t)pb.B * pb.C * pb.S, kind, WB));
    staged_params sp = base_params(h, pb, gp);
    sp.copy_async = copy == 2;
    h.last.copy_engine = copy;
    if (BT > 1) {
        switch (kind) {
            case ST_F32:
                return WB == 64 ? launch_fwd_batch<ST_F32, 64>(h, sp, map, SC, BT, grid)
                                : launch_fwd_batch<ST_F32, 32>(h, sp, map, SC, BT, grid);
            case ST_F16:
                return WB == 64 ? launch_fwd_batch<ST_F16, 64>(h, sp, map, SC, BT, grid)
                                : launch_fwd_batch<ST_F16, 32>(h, sp, map, SC, BT, grid);
            default:
                return WB == 64 ? launch_fwd_batch<ST_BF16, 64>(h, sp, map, SC, BT, grid)
                                : launch_fwd_batch<ST_BF16, 32>(h, sp, map, SC, BT, grid);
        }
    }
    switch (kind) {
        case ST_F32:
            return WB == 64 ? launch_fwd_sc<ST_F32, 64>(h, sp, map, SC, grid) : launch_fwd_sc<ST_F32, 32>(h, sp, map, SC, grid);
        case ST_F16:
            return WB == 64 ? launch_fwd_sc<ST_F16, 64>(h, sp, map, SC, grid) : launch_fwd_sc<ST_F16, 32>(h, sp, map, SC, grid);
        default:
            return WB == 64 ? launch_fwd_sc<ST_BF16, 64>(h, sp, map, SC, grid) : launch_fwd_sc<ST_BF16, 32>(h, sp, map, SC, grid);
    }
}

template <int K, int SC>
static ffdas_error_t launch_cplx_t(ffdas_context &h, const staged_params &sp, const CUtensorMap &map, dim3 grid) {
    constexpr size_t smem = staged_smem_bytes<32, K>();
    FFDAS_TRY((prepare_once<das_staged_cplx_kernel<K, SC, 32>>(smem)));
    das_staged_cplx_kernel<K, SC, 32><<<grid, kStThreads, smem, h.stream>>>(sp, map);
    return ffdas_launch_check(h.stream);
}

ffdas_error_t launch_staged_cplx(ffdas_context &h, const das_problem &pb, int kind, const gather_params &gp,
                                 int SC, dim3 grid) {
    if (kind != ST_C32 && kind != ST_C16) return FFDAS_ERROR_INTERNAL;
    if (gp.cchunk || gp.T0 * gp.T1 * gp.T2 != kStConsumers) return FFDAS_ERROR_INTERNAL;
    CUtensorMap map;
    std::memset(&map, 0, sizeof(map));
    FFDAS_TRY(pair_row_map(map, gp.P, gp.npad, (int64_t)pb.B * pb.C * pb.S, kind, 32));
    staged_params sp = base_params(h, pb, gp);
    h.last.copy_engine = 1;
    if (kind == ST_C32) return SC >= 8 ? launch_cplx_t<ST_C32, 8>(h, sp, map, grid) : launch_cplx_t<ST_C32, 4>(h, sp, map, grid);
    return SC >= 8 ? launch_cplx_t<ST_C16, 8>(h, sp, map, grid) : launch_cplx_t<ST_C16, 4>(h, sp, map, grid);
}

// das_sparse lists that name an event twice with nonzero weights (the staged
// pass holds one entry per voxel and event): sets *gate.  Zero-weight entries
// and events outside x are ignored, as both kernels ignore them.
__global__ void __launch_bounds__(256) sparse_duplicate_kernel(const int *__restrict__ idx,
                                                               const float *__restrict__ w, int n, int S,
                                                               int64_t V, int *gate) {
    const int64_t v = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (v >= V) return;
    bool dup = false;
    if (S <= 64) {
        unsigned long long seen = 0ull;
        for (int i = 0; i < n && !dup; i++) {
            const int s = __ldg(idx + (int64_t)i * V + v);
            if ((unsigned)s < (unsigned)S && __ldg(w + (int64_t)i * V + v) != 0.f) {
                const unsigned long long bit = 1ull << s;
                dup = (seen & bit) != 0ull;
                seen |= bit;
            }
        }
    } else {
        for (int i = 1; i < n && !dup; i++) {
            const int s = __ldg(idx + (int64_t)i * V + v);
            if ((unsigned)s >= (unsigned)S || __ldg(w + (int64_t)i * V + v) == 0.f) continue;
            for (int j = 0; j < i && !dup; j++)
                dup = __ldg(idx + (int64_t)j * V + v) == s && __ldg(w + (int64_t)j * V + v) != 0.f;
        }
    }
    if (dup) atomicExch(gate, 1);
}

ffdas_error_t launch_staged_sparse(ffdas_context &h, const das_problem &pb, int kind, const gather_params &gp,
                                   int SC, int WB, int copy, dim3 grid, int *gate) {
    if (gp.T0 * gp.T1 * gp.T2 != 2 * kStConsumers || !gp.sparse_idx) return FFDAS_ERROR_INTERNAL;
    if (gp.cchunk && grid.z < 2) return FFDAS_ERROR_INTERNAL;
    FFDAS_CUDA(cudaMemsetAsync(gate, 0, sizeof(int), h.stream));
    const int64_t vb = (pb.V + 255) / 256;
    if (vb > INT32_MAX) return FFDAS_ERROR_DIMS_TOO_LARGE;
    sparse_duplicate_kernel<<<(unsigned)vb, 256, 0, h.stream>>>(gp.sparse_idx, gp.weights, pb.n_events, pb.S, pb.V,
                                                               gate);
    FFDAS_TRY(ffdas_launch_check(h.stream));
    if (gp.cchunk) {   // channel slices add into the image: prepare it unless the call falls back
        dim3 sg((unsigned)vb, (unsigned)std::min(pb.B, 65535));
        scale_image_kernel<<<sg, 256, 0, h.stream>>>(static_cast<float *>(gp.out), pb.out_bstride, pb.V, pb.B,
                                                     (float)gp.beta_re, gp.beta_zero, gate);
        FFDAS_TRY(ffdas_launch_check(h.stream));
    }
    copy = resolve_copy(copy);
    CUtensorMap map;
    std::memset(&map, 0, sizeof(map));
    if (copy == 1) FFDAS_TRY(pair_row_map(map, gp.P, gp.npad, (int64_t)pb.B * pb.C * pb.S, kind, WB));
    staged_params sp = base_params(h, pb, gp);
    sp.copy_async = copy == 2;
    sp.n_events = pb.S;            // passes run over x's events
    sp.sparse_idx = gp.sparse_idx;
    sp.sparse_n = pb.n_events;     // list length
    sp.gate = gate;
    h.last.copy_engine = copy;
    switch (kind) {
        case ST_F32:
            return WB == 64 ? launch_fwd_sc<ST_F32, 64>(h, sp, map, SC, grid) : launch_fwd_sc<ST_F32, 32>(h, sp, map, SC, grid);
        case ST_F16:
            return WB == 64 ? launch_fwd_sc<ST_F16, 64>(h, sp, map, SC, grid) : launch_fwd_sc<ST_F16, 32>(h, sp, map, SC, grid);
        default:
            return WB == 64 ? launch_fwd_sc<ST_BF16, 64>(h, sp, map, SC, grid) : launch_fwd_sc<ST_BF16, 32>(h, sp, map, SC, grid);
    }
}

// ------------------------------------------------------ das_sparse items ---
bool sparse_items_supported(const das_problem &pb, int kind) {
    return (kind == ST_F32 || kind == ST_F16 || kind == ST_BF16) && pb.sparse && pb.n_events <= kItemsMaxList &&
           pair_row_length(pb.N) >= 64 && (int64_t)pb.B * pb.C * pb.S < INT32_MAX && pb.B <= 64 &&
           (pb.S + 3) / 4 < 255;
}

size_t sparse_items_workspace(const das_problem &pb, int n_tiles, int SC) {
    const int passes = (pb.S + SC - 1) / SC;
    size_t b = ((size_t)pb.n_events * pb.V * 12 + 255) & ~size_t(255);   // sorted lists
    b += ((size_t)(passes + 1) * pb.V + 255) & ~size_t(255);             // pass starts
    b += ((size_t)n_tiles * 8 + 255) & ~size_t(255);                     // tile work, order
    b += 256;                                                             // queues (one per batch item)
    return b;
}

template <int K, int SC, int WB>
static ffdas_error_t launch_items_t(ffdas_context &h, const staged_params &sp, const items_params &ip,
                                    const CUtensorMap &map, int batch) {
    constexpr size_t smem = items_smem_bytes<K, WB>();
    FFDAS_TRY((prepare_once<das_sparse_items_kernel<K, SC, WB>>(smem)));
    int per_sm = 0;
    FFDAS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, das_sparse_items_kernel<K, SC, WB>, kStThreads,
                                                             smem));
    per_sm = std::max(per_sm, 1);
    // a persistent grid: as many CTAs as the GPU holds at once (split over the
    // batch items, each of which pulls from its own queue)
    const int64_t items = (int64_t)ip.tiles * ip.slices;
    const int64_t resident = std::max<int64_t>(1, (int64_t)std::max(h.sm_count, 1) * per_sm / std::max(batch, 1));
    const int grid = (int)std::min(items, resident);
    h.last.grid = (int64_t)grid * batch;
    das_sparse_items_kernel<K, SC, WB><<<dim3((unsigned)grid, (unsigned)batch), kStThreads, smem, h.stream>>>(sp, ip, map);
    return ffdas_launch_check(h.stream);
}

ffdas_error_t launch_sparse_items(ffdas_context &h, const das_problem &pb, int kind, const gather_params &gp,
                                  int SC, int WB, int copy, void *ws, int *gate) {
    if (gp.T0 * gp.T1 * gp.T2 != kItemsTile || !gp.sparse_idx || !sparse_items_supported(pb, kind))
        return FFDAS_ERROR_INTERNAL;
    SC = SC <= 4 ? 4 : 8;
    const int tiles = gp.n0 * gp.n1 * ((pb.D2 + gp.T2 - 1) / gp.T2);
    const int passes = (pb.S + SC - 1) / SC;
    char *w = static_cast<char *>(ws);
    int *bs = reinterpret_cast<int *>(w);
    float *bo = reinterpret_cast<float *>(bs + (size_t)pb.n_events * pb.V);
    float *bw = bo + (size_t)pb.n_events * pb.V;
    w += ((size_t)pb.n_events * pb.V * 12 + 255) & ~size_t(255);
    uint8_t *pstart = reinterpret_cast<uint8_t *>(w);
    w += ((size_t)(passes + 1) * pb.V + 255) & ~size_t(255);
    int *tile_work = reinterpret_cast<int *>(w);
    int *order = tile_work + tiles;
    w += ((size_t)tiles * 8 + 255) & ~size_t(255);
    int *queue = reinterpret_cast<int *>(w);

    FFDAS_CUDA(cudaMemsetAsync(gate, 0, sizeof(int), h.stream));
    FFDAS_CUDA(cudaMemsetAsync(tile_work, 0, (size_t)tiles * 4, h.stream));
    FFDAS_CUDA(cudaMemsetAsync(queue, 0, 256, h.stream));
    bucket_params bp;
    bp.idx = gp.sparse_idx; bp.ofs = gp.offsets; bp.w = gp.weights;
    bp.n = pb.n_events; bp.S = pb.S; bp.SC = SC; bp.passes = passes; bp.V = pb.V;
    bp.D0 = pb.D0; bp.D1 = pb.D1; bp.T0 = gp.T0; bp.T1 = gp.T1; bp.T2 = gp.T2; bp.n0 = gp.n0; bp.n1 = gp.n1;
    bp.bs = bs; bp.bo = bo; bp.bw = bw; bp.pstart = pstart; bp.tile_work = tile_work; bp.gate = gate;
    const int64_t vb = (pb.V + 127) / 128;
    if (vb > INT32_MAX) return FFDAS_ERROR_DIMS_TOO_LARGE;
    sparse_bucket_kernel<<<(unsigned)vb, 128, 0, h.stream>>>(bp);
    FFDAS_TRY(ffdas_launch_check(h.stream));
    sparse_order_kernel<<<1, 1024, 0, h.stream>>>(tile_work, tiles, order);
    FFDAS_TRY(ffdas_launch_check(h.stream));
    if (gp.cchunk) {   // channel slices add into the image: prepare it unless the call falls back
        dim3 sg((unsigned)((pb.V + 255) / 256), (unsigned)std::min(pb.B, 65535));
        scale_image_kernel<<<sg, 256, 0, h.stream>>>(static_cast<float *>(gp.out), pb.out_bstride, pb.V, pb.B,
                                                     (float)gp.beta_re, gp.beta_zero, gate);
        FFDAS_TRY(ffdas_launch_check(h.stream));
    }
    copy = resolve_copy(copy);
    CUtensorMap map;
    std::memset(&map, 0, sizeof(map));
    if (copy == 1) FFDAS_TRY(pair_row_map(map, gp.P, gp.npad, (int64_t)pb.B * pb.C * pb.S, kind, WB));
    staged_params sp = base_params(h, pb, gp);
    sp.copy_async = copy == 2;
    sp.gate = gate;
    h.last.copy_engine = copy;
    items_params ip;
    ip.bs = bs; ip.bo = bo; ip.bw = bw; ip.pstart = pstart; ip.n = pb.n_events; ip.order = order;
    ip.tiles = tiles;
    ip.slices = gp.cchunk ? (pb.C + gp.cchunk - 1) / gp.cchunk : 1;
    ip.queue = queue;
    switch (kind) {
        case ST_F32:
            if (WB == 64) return SC <= 4 ? launch_items_t<ST_F32, 4, 64>(h, sp, ip, map, pb.B)
                                         : launch_items_t<ST_F32, 8, 64>(h, sp, ip, map, pb.B);
            return SC <= 4 ? launch_items_t<ST_F32, 4, 32>(h, sp, ip, map, pb.B)
                           : launch_items_t<ST_F32, 8, 32>(h, sp, ip, map, pb.B);
        case ST_F16:
            if (WB == 64) return SC <= 4 ? launch_items_t<ST_F16, 4, 64>(h, sp, ip, map, pb.B)
                                         : launch_items_t<ST_F16, 8, 64>(h, sp, ip, map, pb.B);
            return SC <= 4 ? launch_items_t<ST_F16, 4, 32>(h, sp, ip, map, pb.B)
                           : launch_items_t<ST_F16, 8, 32>(h, sp, ip, map, pb.B);
        default:
            if (WB == 64) return SC <= 4 ? launch_items_t<ST_BF16, 4, 64>(h, sp, ip, map, pb.B)
                                         : launch_items_t<ST_BF16, 8, 64>(h, sp, ip, map, pb.B);
            return SC <= 4 ? launch_items_t<ST_BF16, 4, 32>(h, sp, ip, map, pb.B)
                           : launch_items_t<ST_BF16, 8, 32>(h, sp, ip, map, pb.B);
    }
}

ffdas_error_t launch_staged_bwd(ffdas_context &h, const das_problem &pb, int kind, const gather_params &gp,
                                const staged_grads &gr, int SC, int WB, int BT, int copy, dim3 grid) {
    if (BT > 1) copy = 1;   // batch tiles stage their windows with 3-D TMA boxes
    copy = resolve_copy(copy);
    if (BT > 1 && copy != 1) return FFDAS_ERROR_CUDA_DRIVER;
    CUtensorMap map;
    std::memset(&map, 0, sizeof(map));
    if (copy == 1 && BT > 1)
        FFDAS_TRY(pair_batch_map(map, gp.P, gp.npad, (int64_t)pb.C * pb.S, pb.B, kind, WB, BT));
    else if (copy == 1)
        FFDAS_TRY(pair_row_map(map, gp.P, gp.npad, (int64_t)pb.B * pb.C * pb.S, kind, WB));
    staged_params sp = base_params(h, pb, gp);
    sp.copy_async = copy == 2;
    h.last.copy_engine = copy;
    sp.gout = gr.gout;
    sp.gout_bstride = gr.gout_bstride;
    sp.gx = gr.gx; sp.goff = gr.goff; sp.gw = gr.gw; sp.gdst = gr.gdst; sp.gsrc = gr.gsrc;
    if (BT > 1) {
        switch (kind) {
            case ST_F32:
                return WB == 64 ? launch_bwd_batch<ST_F32, 64>(h, sp, map, BT, grid)
                                : launch_bwd_batch<ST_F32, 32>(h, sp, map, BT, grid);
            case ST_F16:
                return WB == 64 ? launch_bwd_batch<ST_F16, 64>(h, sp, map, BT, grid)
                                : launch_bwd_batch<ST_F16, 32>(h, sp, map, BT, grid);
            default:
                return WB == 64 ? launch_bwd_batch<ST_BF16, 64>(h, sp, map, BT, grid)
                                : launch_bwd_batch<ST_BF16, 32>(h, sp, map, BT, grid);
        }
    }
    const int sc = SC > 8 ? 8 : SC;
    switch (kind) {
        case ST_F32:
            return WB == 64 ? launch_bwd_sc<ST_F32, 64>(h, sp, map, sc, grid) : launch_bwd_sc<ST_F32, 32>(h, sp, map, sc, grid);
        case ST_F16:
            return WB == 64 ? launch_bwd_sc<ST_F16, 64>(h, sp, map, sc, grid) : launch_bwd_sc<ST_F16, 32>(h, sp, map, sc, grid);
        default:
            return WB == 64 ? launch_bwd_sc<ST_BF16, 64>(h, sp, map, sc, grid) : launch_bwd_sc<ST_BF16, 32>(h, sp, map, sc, grid);
    }
}

}  // namespace ffdas

extern "C" ffdas_error_t ffdas_get_device_status(ffdas_handle_t h, int *status) {
    if (!h) return FFDAS_ERROR_INVALID_HANDLE;
    if (!status) return FFDAS_ERROR_NULL_POINTER;
    FFDAS_TRY(h->check_device());
    FFDAS_CUDA(cudaStreamSynchronize(h->stream));
    FFDAS_CUDA(cudaMemcpy(status, h->status, sizeof(int), cudaMemcpyDeviceToHost));
    FFDAS_CUDA(cudaMemset(h->status, 0, sizeof(int)));
    return FFDAS_SUCCESS;
}
