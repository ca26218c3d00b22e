// core.h -- handle, tensor descriptor and error plumbing behind include/ffdas.h.
//
// The handle mirrors the reference's ffdas_context (src/core/context.cuh:21):
// device id, arch code, stream, and a stream-ordered workspace allocator.
// No cuBLAS handle: no kernel here calls it.  The cuSOLVER state that
// ffdas_truncate_rank needs is created on that function's first call.
// Workspace comes from a per-handle CUDA memory pool
// (cudaMallocFromPoolAsync) with a high release threshold, which makes it a
// caching, graph-capturable allocator (the reference uses
// cub::CachingDeviceAllocator, src/core/context.cu:143-158).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <mutex>

#include "ffdas.h"

#define FFDAS_MAX_DIMS 16

struct ffdas_tensor_desc {
    int64_t ndim;
    int64_t dims[FFDAS_MAX_DIMS];
    int64_t strides[FFDAS_MAX_DIMS];
    ffdas_datatype_t dtype;

    int64_t numel() const {
        int64_t n = 1;
        for (int64_t i = 0; i < ndim; i++) n *= dims[i];
        return n;
    }
};

// Host hook used by tests to inject workspace-allocation failures without a
// GPU fault: when > 0, the n-th following workspace allocation fails.
extern "C" FFDAS_API void ffdas_debug_fail_alloc_after(int n);

// Test hook: the next TMA-staged launch leaves its first pipeline stage
// unfilled, so its bounded waits expire and it reports a device status of 1
// instead of completing.  One-shot.
extern "C" FFDAS_API void ffdas_debug_staged_drop_stage(int enable);
int ffdas_take_debug_drop_stage();

struct ffdas_context {
    int device_id = 0;
    int arch_code = 0;
    int sm_count = 0;
    size_t smem_optin = 0;
    cudaStream_t stream = 0;
    cudaMemPool_t pool = nullptr;
    bool has_config = false;
    ffdas_das_config_t config{};
    ffdas_kernel_info_t last{};
    int *status = nullptr;  // device word: bounded-wait timeouts of the staged kernels
    unsigned long long *unit_count = nullptr;   // device counter: units the last timed kernel evaluated
    bool timing = false;
    bool timing_recorded = false;
    bool units_recorded = false;   // the last timed kernel counted its units
    // per-channel gain applied by the ingest (ffdas_set_channel_scale): a
    // caller-owned device array of chan_scale_count floats, or null
    const float *chan_scale = nullptr;
    int64_t chan_scale_count = 0;
    // caller-owned buffer for the pair rows (ffdas_set_pair_buffer) and what
    // the last forward call on this handle wrote into it
    void *pair_buf = nullptr;
    size_t pair_buf_bytes = 0;
    struct pair_signature {
        const void *buf = nullptr;     // null: the last forward wrote no buffer
        const void *x = nullptr;
        ffdas_tensor_desc desc{};
        int kind = -1;
        const float *scale = nullptr;
        int64_t scale_count = 0;
    } pair_sig;
    bool last_pairs_reused = false;   // the last ffdas_das_backward read the pair buffer
    int gram_engine = 0;              // ffdas_set_gram_engine: 0 auto, 1 FP32 FMA, 2 tensor cores
    // ffdas_das_from_host: the stream that uploads channel chunks, and one
    // event per chunk plus one for the start (created at the first call)
    static constexpr int kUploadEvents = 17;
    cudaStream_t upload_stream = nullptr;
    cudaEvent_t upload_ev[kUploadEvents] = {};
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    // eigensolver state of ffdas_truncate_rank, created on its first call and
    // released with the handle
    void *solver = nullptr;
    void (*solver_release)(void *) = nullptr;

    // Brackets the main kernel launch with events when timing is enabled.
    void mark_start() { if (timing) cudaEventRecord(ev_start, stream); }
    void mark_stop() { if (timing) { cudaEventRecord(ev_stop, stream); timing_recorded = true; } }

    ffdas_error_t check_device() const;
    ffdas_error_t alloc(size_t bytes, void **ptr);
    void free(void *ptr);
};

namespace ffdas {

// Scoped workspace buffer, freed stream-ordered at scope exit.
class workspace {
public:
    explicit workspace(ffdas_context &ctx) : ctx_(ctx) {}
    ~workspace() { if (ptr_) ctx_.free(ptr_); }
    ffdas_error_t alloc(size_t bytes) { return ctx_.alloc(bytes, &ptr_); }
    template <typename T> T *get() const { return static_cast<T *>(ptr_); }
    workspace(const workspace &) = delete;
    workspace &operator=(const workspace &) = delete;
private:
    ffdas_context &ctx_;
    void *ptr_ = nullptr;
};

}  // namespace ffdas

#define FFDAS_TRY(call)                                   \
    do {                                                  \
        ffdas_error_t e_ = (call);                        \
        if (e_ != FFDAS_SUCCESS) return e_;               \
    } while (0)

#define FFDAS_CUDA(call)                                  \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return FFDAS_ERROR_CUDA_RUNTIME; \
    } while (0)

// Launch check: asynchronous unless FFDAS_DEBUG is set in the environment at
// handle creation (then the stream is synchronised after every launch, as the
// reference's CUDA_LAUNCH_CHECK does under FFDAS_DEBUG, error_checking.h:115).
ffdas_error_t ffdas_launch_check(cudaStream_t stream);

// Raises the dynamic shared memory limit of kernel `func` to `bytes` on
// `device` (the current device; the attribute belongs to the device's
// context), once per kernel, device and size.
cudaError_t ffdas_raise_smem_limit(const void *func, int device, size_t bytes);
