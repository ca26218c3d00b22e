/*
 * ffdas.h -- C-ABI of the B200-native delay-and-sum library (libffdas_b200.so).
 *
 * This header is the drop-in boundary for the delay-and-sum path of ffdas.
 * Every enum value and every entry point that also exists in the reference
 * header (include/ffdas.h of BrainEchoLab/ffdas) keeps its value, name,
 * argument order and meaning, so a caller built against the reference can
 * link this library instead for `das` / `das_sparse`.  Each declaration
 * cites the reference line it replaces.
 *
 * Additions (new codes and new symbols only; nothing existing is altered):
 *   - FFDAS_R_16BF: bfloat16 channel data (unused code 18).
 *   - FFDAS_R_16I channel data (the reference's code 14) into FFDAS_R_32F output:
 *     raw int16 ADC samples, interpolated in FP32 (the reference rejects the
 *     type for das with FFDAS_ERROR_UNSUPPORTED_TYPE).
 *   - ffdas_das_backward: adjoint of ffdas_das / ffdas_das_sparse.
 *   - ffdas_das_set_config / ffdas_das_get_config: kernel schedule override
 *     used by the autotuner.
 *   - ffdas_get_last_kernel_info: which kernel the last call launched.
 *   - ffdas_set_pair_buffer / ffdas_das_pair_bytes: interpolation pairs kept
 *     from a forward call for the backward on the same data.
 *   - ffdas_set_channel_scale: per-channel gain applied at the ingest.
 *   - ffdas_das_static: forward without device allocation or handle.
 *   - ffdas_das_from_host: forward on host-resident channel data, uploads
 *     overlapped with the beamforming.
 *   - ffdas_sparse_select: das_sparse index lists selected on the device.
 *   - ffdas_set_gram_engine: tensor-core or FP32-FMA Gram in truncate_rank.
 *   - ffdas_set_kernel_timing / ffdas_get_last_kernel_time /
 *     ffdas_get_last_kernel_units / ffdas_measure_fp32_peak /
 *     ffdas_get_device_status: measurement and bounded-wait status.
 *
 * Conventions (unchanged from the reference):
 *   - dims and strides are in ELEMENTS; strides == NULL means C-contiguous.
 *   - all device pointers are caller-owned; descriptors are caller-owned
 *     heap objects.
 *   - every call is asynchronous on the handle's stream and returns an
 *     ffdas_error_t; nothing throws across the ABI.
 */
#ifndef FFDAS_H_
#define FFDAS_H_

#if defined(_WIN32) || defined(_WIN64)
#  if defined(ffdas_EXPORTS)
#    define FFDAS_API __declspec(dllexport)
#  else
#    define FFDAS_API __declspec(dllimport)
#  endif
#else
#  define FFDAS_API __attribute__((visibility("default")))
#endif

#include <stdint.h>
#include <stdbool.h>
#include <stddef.h>

/* Error codes: values identical to the reference, include/ffdas.h:19-62. */
typedef enum {
    FFDAS_SUCCESS = 0,

    FFDAS_ERROR_INVALID_ARGUMENT = 1,
    FFDAS_ERROR_INVALID_DIMS = 2,
    FFDAS_ERROR_UNSUPPORTED_TYPE = 3,
    FFDAS_ERROR_NULL_POINTER = 4,
    FFDAS_ERROR_INVALID_HANDLE = 5,
    FFDAS_ERROR_NON_CONTIGUOUS = 6,
    FFDAS_ERROR_DIMS_TOO_LARGE = 7,

    FFDAS_ERROR_ALLOCATION_FAILED = 10,
    FFDAS_ERROR_DEVICE_MEMORY_INSUFFICIENT = 11,
    FFDAS_ERROR_HOST_MEMORY_INSUFFICIENT = 12,
    FFDAS_ERROR_INVALID_DEVICE = 13,

    FFDAS_ERROR_DEVICE_NOT_SUPPORTED = 20,
    FFDAS_ERROR_INSUFFICIENT_COMPUTE_CAPABILITY = 21,
    FFDAS_ERROR_DEVICE_NOT_AVAILABLE = 22,
    FFDAS_ERROR_DEVICE_MISMATCH = 23,

    FFDAS_ERROR_CUDA_DRIVER = 30,
    FFDAS_ERROR_CUDA_RUNTIME = 31,
    FFDAS_ERROR_CUDA_LAUNCH_FAILED = 32,
    FFDAS_ERROR_CUDA_SYNC_FAILED = 33,
    FFDAS_ERROR_CUDA_MEMCPY_FAILED = 34,

    FFDAS_ERROR_CUBLAS = 40,
    FFDAS_ERROR_CUSOLVER = 41,
    FFDAS_ERROR_CUFFT = 42,
    FFDAS_ERROR_NVTX = 43,

    FFDAS_ERROR_ALGORITHM_FAILED = 50,
    FFDAS_ERROR_CONVERGENCE_FAILED = 51,
    FFDAS_ERROR_NUMERICAL_INSTABILITY = 52,

    FFDAS_ERROR_NOT_INITIALIZED = 60,
    FFDAS_ERROR_ALREADY_INITIALIZED = 61,
    FFDAS_ERROR_INVALID_STATE = 62,
    FFDAS_ERROR_OUT_OF_BOUNDS_INDEX = 63,

    FFDAS_ERROR_INTERNAL = 100,
    FFDAS_ERROR_UNKNOWN = 101
} ffdas_error_t;

/* Data types: reference values include/ffdas.h:64-75, plus FFDAS_R_16BF. */
typedef enum {
    FFDAS_R_16F = 2,
    FFDAS_C_16F = 6,
    FFDAS_R_32F = 0,
    FFDAS_C_32F = 4,
    FFDAS_R_64F = 16,
    FFDAS_C_64F = 17,
    FFDAS_R_32I = 10,
    FFDAS_C_32I = 11,
    FFDAS_R_16I = 14,
    FFDAS_C_16I = 15,
    /* new: IEEE bfloat16 real channel data (2 bytes). */
    FFDAS_R_16BF = 18
} ffdas_datatype_t;

/* Compute types: include/ffdas.h:77-82.  FFDAS_COMPUTE_16F stores channel
 * data as fp16 pairs (interpolation and accumulation stay fp32).  The new
 * value FFDAS_COMPUTE_16BF stores them as bf16 pairs. */
typedef enum {
    FFDAS_COMPUTE_DEFAULT = 0,
    FFDAS_COMPUTE_16F = 1,
    FFDAS_COMPUTE_32F = 2,
    FFDAS_COMPUTE_64F = 3,
    FFDAS_COMPUTE_16BF = 4
} ffdas_compute_type_t;

/* Algorithm selector: include/ffdas.h:84-90.  Every value is accepted; all
 * of them run the B200 kernels chosen by the planner (see ffdas_das_config),
 * because the reference's ALG1/ALG2/ALG4 schedules are superseded. */
typedef enum {
    FFDAS_ALG_DEFAULT = 0,
    FFDAS_ALG1 = 1,
    FFDAS_ALG2 = 2,
    FFDAS_ALG3 = 3,
    FFDAS_ALG4 = 4
} ffdas_alg_t;

typedef enum {
    FFDAS_INTERP_NEAREST = 0,
    FFDAS_INTERP_LINEAR = 1
} ffdas_interp_mode_t;

struct ffdas_context;
typedef struct ffdas_context* ffdas_handle_t;

struct ffdas_tensor_desc;
typedef struct ffdas_tensor_desc* ffdas_tensor_desc_t;

/* Kernel schedule for the delay-and-sum kernels (new).  Zero in a field
 * means "planner default".  The autotuner sweeps these. */
typedef struct {
    int32_t variant;      /* 0 auto, 1 L1 gather kernel, 2 TMA-staged kernel (forward and adjoint),
                             3 gather adjoint in ffdas_das_backward (forward as 0),
                             5 direct kernel: one launch, no workspace, for small real problems
                               (forward; the adjoint as 0),
                             6 das_sparse: persistent staged kernel over bucketed lists, tiles
                               longest first (real data, lists of up to 64 entries;
                               min_blocks sets the channel slicing, about that many work
                               items per SM) */
    int32_t tile_x;       /* voxels per CTA along the innermost spatial dim
                             (variant 5: lanes per voxel, 1..32, 0 = from the occupancy) */
    int32_t tile_y;       /* ... along the middle spatial dim */
    int32_t tile_z;       /* ... along the outermost spatial dim */
    int32_t batch_tile;   /* batch items per thread (1,2,4,8,16) */
    int32_t event_chunk;  /* events held in registers per pass (1..16) */
    int32_t min_blocks;   /* staged kernels: target CTAs per SM; problems with fewer tiles split
                             each tile's channels over CTAs that add into the image or the
                             voxel-side gradients (default 3 forward, 2 adjoint) */
    int32_t window;       /* TMA-staged kernel: pairs per staged window (32 or 64) */
    int32_t copy_engine;  /* staged kernels: 0 auto, 1 TMA tile loads, 2 per-thread cp.async copies */
} ffdas_das_config_t;

/* What the last das/das_sparse/backward call on a handle launched (new).
 * After ffdas_truncate_rank, variant is its eigen route: 10 orthogonal
 * iteration on the device, 11 cuSOLVER syevd, 12 syevdx over one index
 * range, 13 keep-all copy; grid is the Gram kernel's CTA count and
 * copy_engine the Gram engine (1 FP32 FMA, 2 tensor cores). */
typedef struct {
    int32_t variant;
    int32_t tile_x, tile_y, tile_z;
    int32_t batch_tile;
    int32_t event_chunk;
    int32_t storage;      /* pair storage: 0 f32, 1 f16, 2 bf16, 3 f64, 4 c32, 5 c16, 6 c64 */
    int32_t kernels;      /* kernels launched by the call */
    int64_t grid;         /* CTAs of the main kernel */
    int32_t copy_engine;  /* staged kernels: 1 TMA, 2 cp.async; 0 otherwise */
} ffdas_kernel_info_t;

#if defined(__cplusplus)
extern "C" {
#endif

/* include/ffdas.h:115 */
FFDAS_API size_t ffdas_type_size(ffdas_datatype_t datatype);

/* include/ffdas.h:117 */
FFDAS_API const char* ffdas_error_string(ffdas_error_t error);

/* include/ffdas.h:119-125 (src/core/tensor.cu:9-33) */
FFDAS_API ffdas_error_t ffdas_create_tensor_desc(
    ffdas_tensor_desc_t *desc,
    int64_t ndim,
    const int64_t *dims,
    const int64_t *strides,
    ffdas_datatype_t dtype
);

/* include/ffdas.h:127-129 */
FFDAS_API ffdas_error_t ffdas_destroy_tensor_desc(ffdas_tensor_desc_t desc);

/* include/ffdas.h:131-133 (src/core/context.cu:16) */
FFDAS_API ffdas_error_t ffdas_create(ffdas_handle_t *handle);

/* include/ffdas.h:135-137 (src/core/context.cu:72) */
FFDAS_API ffdas_error_t ffdas_destroy(ffdas_handle_t handle);

/* include/ffdas.h:139-142 */
FFDAS_API ffdas_error_t ffdas_set_stream(ffdas_handle_t handle, uintptr_t stream);

/* include/ffdas.h:144-147 */
FFDAS_API ffdas_error_t ffdas_get_stream(ffdas_handle_t handle, uintptr_t *stream);

/* include/ffdas.h:149-155: strided copy with dtype cast (src/tensor_ops/
 * contiguous_copy.cu).  Supports the real/complex float types and bf16. */
FFDAS_API ffdas_error_t ffdas_contiguous_copy(
    ffdas_handle_t handle,
    ffdas_tensor_desc_t x_desc,
    const void *x,
    ffdas_tensor_desc_t out_desc,
    void *out
);

/* include/ffdas.h:188-203 (src/das/das.cu:9).
 * out[b, v] = beta * out[b, v] + sum_s sum_c w[s,v] * lerp(x[b,c,s,:], tau)
 * with tau = offsets[s,v] + |dstpos[v] - srcpos[c]|.
 * offsets/weights are indexed [s * V + v] for both 3-D and 4-D x (the
 * reference reuses event 0's row for 3-D x; see the design notes). */
FFDAS_API ffdas_error_t ffdas_das(
    ffdas_handle_t handle,
    const float *srcpos,
    const float *srcdir,
    float wavenum,
    ffdas_tensor_desc_t x_desc,
    const void* x,
    const float *dstpos,
    const float *offsets,
    const float *weights,
    const void *beta,
    ffdas_tensor_desc_t out_desc,
    void* out,
    ffdas_compute_type_t compute_type,
    ffdas_alg_t alg
);

/* include/ffdas.h:205-222 (src/das/das_sparse.cu:6).  Entries whose weight
 * is exactly zero are skipped, so uneven per-voxel subsets can be padded
 * with weight 0. */
FFDAS_API ffdas_error_t ffdas_das_sparse(
    ffdas_handle_t handle,
    const float *srcpos,
    const float *srcdir,
    float wavenum,
    ffdas_tensor_desc_t x_desc,
    const void* x,
    const float *dstpos,
    const float *offsets,
    const float *weights,
    int sparse_count,
    const int *sparse_indices,
    const void *beta,
    ffdas_tensor_desc_t out_desc,
    void* out,
    ffdas_compute_type_t compute_type,
    ffdas_alg_t alg
);

/* New: adjoint of ffdas_das (sparse_indices == NULL) or ffdas_das_sparse.
 * Real FP32/FP16/BF16 channel data with an FP32 output, or complex64 /
 * complex32 channel data with a complex64 output (any wavenum).  grad_out
 * has the layout and type of `out`.  Each grad pointer may be NULL (not
 * computed).  Shapes:
 *   grad_x       : x_desc layout, FP32 (complex data: interleaved complex64),
 *                  accumulated (+=) so the caller zeroes it
 *   grad_offsets : (S or n, V) FP32, overwritten
 *   grad_weights : (S or n, V) FP32, overwritten
 *   grad_dstpos  : (V, 3) FP32, overwritten
 *   grad_srcpos  : (C, 3) FP32, overwritten
 * Real data needs wavenum 0.  Complex data: x_k gets (1 - t) conj(A) g and
 * x_{k+1} gets t conj(A) g for the tap weight A = w (cos, sin)(wavenum tau),
 * g = d loss / d Re(out) + i d loss / d Im(out); the real inputs get the
 * real part of conj(g) times their derivative of out.  srcdir (element
 * directivity) masks taps as in the forward; the mask has no gradient, and
 * dense calls with it run the gather adjoint.
 * ffdas_get_last_kernel_info then reports variant 4 (TMA-staged adjoint,
 * dense calls), 3 (gather adjoint: dense calls under schedule variant 3 or
 * with directivity, and das_sparse under variant 3 or when the lists' tables
 * do not fit), 7 (das_sparse: a lane per list entry, entries bucketed by
 * event) or 8 (complex data: a thread per voxel). */
FFDAS_API ffdas_error_t ffdas_das_backward(
    ffdas_handle_t handle,
    const float *srcpos,
    const float *srcdir,
    float wavenum,
    ffdas_tensor_desc_t x_desc,
    const void* x,
    const float *dstpos,
    const float *offsets,
    const float *weights,
    int sparse_count,
    const int *sparse_indices,
    ffdas_tensor_desc_t grad_out_desc,
    const void *grad_out,
    float *grad_x,
    float *grad_offsets,
    float *grad_weights,
    float *grad_dstpos,
    float *grad_srcpos
);

/* New: a caller-owned device buffer for the interpolation-pair rows.  While
 * one is set (and holds ffdas_das_pair_bytes for the call), a forward call
 * builds its pair rows there instead of in workspace, and
 * ffdas_das_backward on the same x -- same pointer, descriptor, pair storage
 * and channel scale as the last forward call on this handle -- reads them
 * instead of building them again (the adjoint then launches one kernel
 * fewer).  The caller keeps the buffer and x unchanged in between (an
 * autograd forward saves both for its backward).  NULL clears the buffer. */
FFDAS_API ffdas_error_t ffdas_set_pair_buffer(ffdas_handle_t handle, void *buffer, size_t bytes);
FFDAS_API ffdas_error_t ffdas_das_pair_bytes(ffdas_tensor_desc_t x_desc, ffdas_compute_type_t compute_type,
                                             size_t *bytes);

/* New: ffdas_das on channel data in host memory (page-locked for the copies
 * to overlap; pageable memory works, serially).  Same arguments as ffdas_das
 * except that x_host is a host pointer to C-contiguous x, plus `chunks`: the
 * channels are cut into about that many runs (0: about C / 128, at most 8;
 * at most 15), the first of half the width.  The handle's own upload stream
 * copies run k + 1 while the handle's stream beamforms run k, which waits
 * only for its own run; run 0 applies beta and every later run adds into out
 * (beta = 1), so only the first run's upload is not hidden behind the
 * beamforming.  The output, positions,
 * delays and weights are device buffers as for ffdas_das.  A per-item
 * channel scale (B * C values) keeps the whole call in one run.  The sum
 * over channels is grouped by run, so the image differs from ffdas_das's in
 * rounding only.  Not for ffdas_das_backward's pair reuse (the runs do not
 * fill the pair buffer).  x_host must stay valid and unchanged until the
 * call's work on the handle's stream has completed. */
FFDAS_API ffdas_error_t ffdas_das_from_host(ffdas_handle_t handle, const float *srcpos, const float *srcdir,
                                            float wavenum, ffdas_tensor_desc_t x_desc, const void *x_host,
                                            const float *dstpos, const float *offsets, const float *weights,
                                            const void *beta, ffdas_tensor_desc_t out_desc, void *out,
                                            ffdas_compute_type_t compute_type, ffdas_alg_t alg, int chunks);

/* New: per-channel scale of the channel data, applied by the ingest of every
 * following ffdas_das / ffdas_das_sparse call on this handle (it replaces the
 * reference's caller-side cast/copy, src/tensor_ops/contiguous_copy_impl.cuh:
 * 17-57, with a scaled one): sample k of row (b, c, s) enters as
 * scale[c] * x[b,c,s,k] when count == C, or scale[b * C + c] * x[b,c,s,k]
 * when count == B * C, formed in FP32 (FP64 for FP64 data, both parts of
 * complex samples) and then rounded into the pair storage -- so FP32 or int16
 * data can be normalised per channel (scale = 1 / peak) before FP16/BF16
 * storage, or raw ADC samples given their channel gains.  `scale` is a
 * device array the caller keeps alive while it is set; NULL clears it.  A
 * call whose C or B * C does not match `count` returns
 * FFDAS_ERROR_INVALID_ARGUMENT; ffdas_das_backward returns the same while a
 * scale is set (its adjoint is not provided). */
FFDAS_API ffdas_error_t ffdas_set_channel_scale(ffdas_handle_t handle, const float *scale, int64_t count);

/* New, no counterpart in the reference: the forward delay-and-sum for callers
 * that cannot allocate device memory (a real-time or embedded host where
 * cudaMalloc is forbidden, a memory budget fixed before the first frame, or a
 * caller without an ffdas handle, whose creation allocates a workspace pool).
 * Same arguments as ffdas_das, except that it takes the CUDA stream directly
 * instead of a handle.  It allocates nothing: the interpolation-pair workspace
 * is a 16 MiB array in the library's device image (every GPU that loads the
 * library holds it until exit), so B * C * S * roundup(N, 4) * 8 bytes (4 for
 * 16-bit channel data) must not exceed 16 MiB, else FFDAS_ERROR_DIMS_TOO_LARGE.
 * Real channel data (float32, float16, bfloat16, int16) with float32 output only.
 * The first call on a device looks up the array's device address (once per
 * device and CUDA context: after cudaDeviceReset the next call looks it up
 * again); make that first call before any stream capture.  All calls share
 * the one array: calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialised by the caller. */
FFDAS_API ffdas_error_t ffdas_das_static(
    uintptr_t stream,
    const float *srcpos,
    const float *srcdir,
    float wavenum,
    ffdas_tensor_desc_t x_desc,
    const void* x,
    const float *dstpos,
    const float *offsets,
    const float *weights,
    const void *beta,
    ffdas_tensor_desc_t out_desc,
    void* out,
    ffdas_compute_type_t compute_type,
    ffdas_alg_t alg
);

/* New, no counterpart in the reference library: the event lists a
 * das_sparse call sums, chosen on the device.  Replaces the host-array step
 * of the reference's sparse-compounding example
 * (bindings/python/examples/sparse_compounding.py:141-144: argpartition of
 * the weights over the event axis, then take_along_axis of weights and
 * delays).  weights and offsets are (n_events, n_voxels) float32 rows;
 * per voxel the k events with the largest weight (NaN above every number,
 * ties to the lower event index), in that order, go to sparse_indices
 * (k, n_voxels) int32, their weights to sparse_weights and their delays to
 * sparse_offsets (both nullable; offsets may be NULL when sparse_offsets is).
 * 1 <= k <= min(n_events, 32), else FFDAS_ERROR_INVALID_ARGUMENT.
 * Asynchronous on the handle's stream; allocates nothing. */
FFDAS_API ffdas_error_t ffdas_sparse_select(
    ffdas_handle_t handle,
    const float *weights,
    const float *offsets,
    int n_events,
    int64_t n_voxels,
    int k,
    int *sparse_indices,
    float *sparse_weights,
    float *sparse_offsets
);

/* Rank filter: out = the singular components start..stop-1 of x (m, n)
 * (reference include/ffdas.h:178-186, src/truncate_rank/truncate_rank.cu:6).
 * x and out: 2-D, same dims, C-contiguous (else FFDAS_ERROR_NON_CONTIGUOUS),
 * same dtype in {R_32F, C_32F, R_64F, C_64F}; 0 <= start < stop <=
 * min(m, n), else FFDAS_ERROR_INVALID_ARGUMENT.  out may be x.  The
 * leading-subspace case (start = 0, or stop = min(m, n)) is first tried
 * with an orthogonal iteration on the device; otherwise, or if that does
 * not converge, cuSOLVER's syevd/syevdx (loaded at the first call that
 * needs it) solves the eigenproblem and reports through FFDAS_ERROR_CUSOLVER.  The call
 * waits on the host for the eigen step's status, so, like the reference's,
 * it cannot be captured in a CUDA graph.  The Gram matrix of the smaller
 * side is formed on the tensor cores (tcgen05, FP32 split into two TF32
 * parts, three products) for float32 with m <= n, m <= 256, n a multiple
 * of 4 and x 16-byte aligned, else with FP32 FMAs; see
 * ffdas_set_gram_engine. */
FFDAS_API ffdas_error_t ffdas_truncate_rank(
    ffdas_handle_t handle,
    ffdas_tensor_desc_t x_desc,
    const void *x,
    int64_t start,
    int64_t stop,
    ffdas_tensor_desc_t out_desc,
    void *out
);

/* New: engine of ffdas_truncate_rank's Gram matrix on this handle.
 * 0 (default): tensor cores where the input qualifies (see above) and
 * m * n >= 2^20, else the FP32 FMA kernel; 1: always the FP32 FMA kernel
 * (every product and sum in FP32, as the reference's cuBLAS SGEMM);
 * 2: tensor cores wherever the input qualifies.  Tensor-core Gram entries
 * carry about 2^-21 relative error per product (the dropped lo*lo term and
 * TF32 rounding of the low part) against FP32's 2^-24; both sum in FP32
 * within a CTA and in double across CTAs.  After the call,
 * ffdas_get_last_kernel_info's copy_engine is the engine used (1 FMA,
 * 2 tensor cores).  Other values: FFDAS_ERROR_INVALID_ARGUMENT. */
FFDAS_API ffdas_error_t ffdas_set_gram_engine(ffdas_handle_t handle, int32_t engine);

/* New: schedule override for the following calls on this handle
 * (NULL restores the planner default). */
FFDAS_API ffdas_error_t ffdas_das_set_config(ffdas_handle_t handle,
                                             const ffdas_das_config_t *config);
FFDAS_API ffdas_error_t ffdas_das_get_config(ffdas_handle_t handle,
                                             ffdas_das_config_t *config);

/* New: description of the kernels the last DAS call launched. */
FFDAS_API ffdas_error_t ffdas_get_last_kernel_info(ffdas_handle_t handle,
                                                   ffdas_kernel_info_t *info);

/* New: when enabled, each DAS call records CUDA events on the handle's stream
 * around its main (gather) kernel; ffdas_get_last_kernel_time waits for the
 * last call's stop event and returns that kernel's duration in ms. */
FFDAS_API ffdas_error_t ffdas_set_kernel_timing(ffdas_handle_t handle, int enable);
FFDAS_API ffdas_error_t ffdas_get_last_kernel_time(ffdas_handle_t handle, float *ms);

/* New: with kernel timing enabled, the number of voxel x channel x event x
 * batch units the last call's main kernel actually evaluated (units of
 * passes and stages it skipped because every tap lies outside the record
 * are not counted).  Waits for the handle's stream.  FFDAS_ERROR_INVALID_STATE
 * when timing is off or the last kernel does not count its units (only the
 * 512-voxel TMA-staged forward does). */
FFDAS_API ffdas_error_t ffdas_get_last_kernel_units(ffdas_handle_t handle, long long *units);

/* New: measured FP32 FMA throughput of the current device (TFLOP/s): the
 * faster of a scalar-FMA and a packed-f32x2-FMA kernel of independent chains
 * on the handle's stream (synchronous). */
FFDAS_API ffdas_error_t ffdas_measure_fp32_peak(ffdas_handle_t handle, double *tflops);

/* New: device-side status of the handle's kernels since the last query
 * (0 = ok, 1 = a bounded wait inside a staged kernel expired and the kernel
 * returned early).  Synchronises the handle's stream, then clears the word. */
FFDAS_API ffdas_error_t ffdas_get_device_status(ffdas_handle_t handle, int *status);

/* include/ffdas.h:290-300 */
FFDAS_API ffdas_error_t ffdas_device_count(int *count);
FFDAS_API ffdas_error_t ffdas_device_get(int *device);
FFDAS_API ffdas_error_t ffdas_device_set(int device);

/* include/ffdas.h:302-323 */
FFDAS_API ffdas_error_t ffdas_event_create(uintptr_t *event);
FFDAS_API ffdas_error_t ffdas_event_destroy(uintptr_t event);
FFDAS_API ffdas_error_t ffdas_event_record(ffdas_handle_t handle, uintptr_t event);
FFDAS_API ffdas_error_t ffdas_event_synchronize(uintptr_t event);
FFDAS_API ffdas_error_t ffdas_event_elapsed_time(uintptr_t start, uintptr_t stop, float *ms);

#if defined(__cplusplus)
}
#endif

#endif /* FFDAS_H_ */
