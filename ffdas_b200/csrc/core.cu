// core.cu -- handle, descriptor, stream, event, device and error entry points.
//
// Behaviour follows the reference's src/core/context.cu, tensor.cu,
// error_utils.cu and type_utils.cu: the same validation order and the same
// error codes for the same invalid inputs.
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <atomic>
#include <map>
#include <mutex>
#include <cstdlib>
#include <cstring>
#include <new>

#include "core.h"

static std::atomic<int> g_fail_alloc_after{0};
static bool g_debug_sync = false;

extern "C" FFDAS_API void ffdas_debug_fail_alloc_after(int n) {
    g_fail_alloc_after.store(n);
}

static std::atomic<int> g_drop_stage{0};

extern "C" FFDAS_API void ffdas_debug_staged_drop_stage(int enable) {
    g_drop_stage.store(enable ? 1 : 0);
}

int ffdas_take_debug_drop_stage() {
    return g_drop_stage.exchange(0);
}

cudaError_t ffdas_raise_smem_limit(const void *func, int device, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> raised;
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_pair(func, device);
    const auto it = raised.find(key);
    if (it != raised.end() && it->second >= bytes) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return e;
    }
    raised[key] = bytes;
    return cudaSuccess;
}

ffdas_error_t ffdas_launch_check(cudaStream_t stream) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return FFDAS_ERROR_CUDA_LAUNCH_FAILED;
    if (g_debug_sync) {
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return FFDAS_ERROR_CUDA_SYNC_FAILED;
    }
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_context::check_device() const {
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) return FFDAS_ERROR_CUDA_RUNTIME;
    return cur == device_id ? FFDAS_SUCCESS : FFDAS_ERROR_DEVICE_MISMATCH;
}

ffdas_error_t ffdas_context::alloc(size_t bytes, void **ptr) {
    *ptr = nullptr;
    if (bytes == 0) return FFDAS_SUCCESS;
    int n = g_fail_alloc_after.load();
    if (n > 0) {
        if (n == 1) {
            g_fail_alloc_after.store(0);
            return FFDAS_ERROR_DEVICE_MEMORY_INSUFFICIENT;
        }
        g_fail_alloc_after.store(n - 1);
    }
    cudaError_t e = cudaMallocFromPoolAsync(ptr, bytes, pool, stream);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return FFDAS_ERROR_DEVICE_MEMORY_INSUFFICIENT;
    }
    return e == cudaSuccess ? FFDAS_SUCCESS : FFDAS_ERROR_ALLOCATION_FAILED;
}

void ffdas_context::free(void *ptr) {
    if (ptr) cudaFreeAsync(ptr, stream);
}

extern "C" {

size_t ffdas_type_size(ffdas_datatype_t t) {
    switch (t) {
        case FFDAS_R_16F: return 2;
        case FFDAS_R_16BF: return 2;
        case FFDAS_C_16F: return 4;
        case FFDAS_R_32F: return 4;
        case FFDAS_C_32F: return 8;
        case FFDAS_R_64F: return 8;
        case FFDAS_C_64F: return 16;
        case FFDAS_R_32I: return 4;
        case FFDAS_C_32I: return 8;
        case FFDAS_R_16I: return 2;
        case FFDAS_C_16I: return 4;
        default: return 0;
    }
}

const char *ffdas_error_string(ffdas_error_t e) {
    switch (e) {
        case FFDAS_SUCCESS: return "Success";
        case FFDAS_ERROR_INVALID_ARGUMENT: return "Invalid argument";
        case FFDAS_ERROR_INVALID_DIMS: return "Invalid dimensions";
        case FFDAS_ERROR_UNSUPPORTED_TYPE: return "Unsupported data type";
        case FFDAS_ERROR_NULL_POINTER: return "Null pointer argument";
        case FFDAS_ERROR_INVALID_HANDLE: return "Invalid handle";
        case FFDAS_ERROR_NON_CONTIGUOUS: return "Non-contiguous tensor";
        case FFDAS_ERROR_DIMS_TOO_LARGE: return "Dimensions too large";
        case FFDAS_ERROR_ALLOCATION_FAILED: return "Memory allocation failed";
        case FFDAS_ERROR_DEVICE_MEMORY_INSUFFICIENT: return "Insufficient device memory";
        case FFDAS_ERROR_HOST_MEMORY_INSUFFICIENT: return "Insufficient host memory";
        case FFDAS_ERROR_INVALID_DEVICE: return "Invalid device";
        case FFDAS_ERROR_DEVICE_NOT_SUPPORTED: return "Device not supported";
        case FFDAS_ERROR_INSUFFICIENT_COMPUTE_CAPABILITY: return "Insufficient compute capability";
        case FFDAS_ERROR_DEVICE_NOT_AVAILABLE: return "Device not available";
        case FFDAS_ERROR_DEVICE_MISMATCH: return "Device mismatch";
        case FFDAS_ERROR_CUDA_DRIVER: return "CUDA driver error";
        case FFDAS_ERROR_CUDA_RUNTIME: return "CUDA runtime error";
        case FFDAS_ERROR_CUDA_LAUNCH_FAILED: return "CUDA kernel launch failed";
        case FFDAS_ERROR_CUDA_SYNC_FAILED: return "CUDA synchronization failed";
        case FFDAS_ERROR_CUDA_MEMCPY_FAILED: return "CUDA memory copy failed";
        case FFDAS_ERROR_CUBLAS: return "cuBLAS library error";
        case FFDAS_ERROR_CUSOLVER: return "cuSOLVER library error";
        case FFDAS_ERROR_CUFFT: return "cuFFT library error";
        case FFDAS_ERROR_NVTX: return "NVTX error";
        case FFDAS_ERROR_ALGORITHM_FAILED: return "Algorithm execution failed";
        case FFDAS_ERROR_CONVERGENCE_FAILED: return "Algorithm failed to converge";
        case FFDAS_ERROR_NUMERICAL_INSTABILITY: return "Numerical instability detected";
        case FFDAS_ERROR_NOT_INITIALIZED: return "Library not initialized";
        case FFDAS_ERROR_ALREADY_INITIALIZED: return "Library already initialized";
        case FFDAS_ERROR_INVALID_STATE: return "Invalid library state";
        case FFDAS_ERROR_OUT_OF_BOUNDS_INDEX: return "Out of bounds index";
        case FFDAS_ERROR_INTERNAL: return "Internal error";
        case FFDAS_ERROR_UNKNOWN: return "Unknown error";
        default: return "Unrecognized error code";
    }
}

ffdas_error_t ffdas_create_tensor_desc(ffdas_tensor_desc_t *desc, int64_t ndim,
                                       const int64_t *dims, const int64_t *strides,
                                       ffdas_datatype_t dtype) {
    // Same checks and order as the reference (src/core/tensor.cu:9-33), plus
    // a cap on ndim because this descriptor stores dims inline.
    if (!desc || ndim <= 0 || !dims) return FFDAS_ERROR_INVALID_ARGUMENT;
    if (ffdas_type_size(dtype) == 0) return FFDAS_ERROR_UNSUPPORTED_TYPE;
    if (ndim > FFDAS_MAX_DIMS) return FFDAS_ERROR_DIMS_TOO_LARGE;
    ffdas_tensor_desc *d = new (std::nothrow) ffdas_tensor_desc();
    if (!d) return FFDAS_ERROR_ALLOCATION_FAILED;
    d->ndim = ndim;
    d->dtype = dtype;
    for (int64_t i = 0; i < ndim; i++) d->dims[i] = dims[i];
    if (strides) {
        for (int64_t i = 0; i < ndim; i++) d->strides[i] = strides[i];
    } else {
        int64_t s = 1;
        for (int64_t i = ndim - 1; i >= 0; i--) {
            d->strides[i] = s;
            s *= dims[i];
        }
    }
    *desc = d;
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_destroy_tensor_desc(ffdas_tensor_desc_t desc) {
    delete desc;
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_create(ffdas_handle_t *handle) {
    if (!handle) return FFDAS_ERROR_NULL_POINTER;
    *handle = nullptr;
    ffdas_context *h = new (std::nothrow) ffdas_context();
    if (!h) return FFDAS_ERROR_HOST_MEMORY_INSUFFICIENT;

    ffdas_error_t err = FFDAS_SUCCESS;
    cudaDeviceProp prop;
    cudaMemPoolProps pp;
    uint64_t threshold = UINT64_MAX;
    const char *dbg = std::getenv("FFDAS_DEBUG");
    g_debug_sync = dbg && dbg[0] && dbg[0] != '0';

    if (cudaGetDevice(&h->device_id) != cudaSuccess) { err = FFDAS_ERROR_CUDA_RUNTIME; goto fail; }
    if (cudaGetDeviceProperties(&prop, h->device_id) != cudaSuccess) { err = FFDAS_ERROR_CUDA_RUNTIME; goto fail; }
    h->arch_code = prop.major * 100 + prop.minor * 10;
    // The kernels are compiled for sm_100a only.
    if (prop.major < 10) { err = FFDAS_ERROR_INSUFFICIENT_COMPUTE_CAPABILITY; goto fail; }
    if (prop.major != 10) { err = FFDAS_ERROR_DEVICE_NOT_SUPPORTED; goto fail; }
    h->sm_count = prop.multiProcessorCount;
    h->smem_optin = prop.sharedMemPerBlockOptin;

    std::memset(&pp, 0, sizeof(pp));
    pp.allocType = cudaMemAllocationTypePinned;
    pp.handleTypes = cudaMemHandleTypeNone;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = h->device_id;
    if (cudaMemPoolCreate(&h->pool, &pp) != cudaSuccess) { err = FFDAS_ERROR_CUDA_RUNTIME; goto fail; }
    cudaMemPoolSetAttribute(h->pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    // 16 device bytes: the status word, and at byte 8 the counter of units
    // evaluated that kernel timing reads (ffdas_get_last_kernel_units)
    if (cudaMalloc(reinterpret_cast<void **>(&h->status), 16) != cudaSuccess ||
        cudaMemset(h->status, 0, 16) != cudaSuccess) {
        err = FFDAS_ERROR_ALLOCATION_FAILED;
        goto fail;
    }
    h->unit_count = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(h->status) + 8);
    *handle = h;
    return FFDAS_SUCCESS;
fail:
    cudaGetLastError();
    if (h->status) cudaFree(h->status);
    if (h->pool) cudaMemPoolDestroy(h->pool);
    cudaGetLastError();
    delete h;
    return err;
}

ffdas_error_t ffdas_destroy(ffdas_handle_t h) {
    if (!h) return FFDAS_ERROR_INVALID_HANDLE;
    ffdas_error_t err = FFDAS_SUCCESS;
    if (h->pool) {
        // Pool memory freed with cudaFreeAsync is released once the stream
        // reaches the free; synchronise so the pool can be destroyed.  If
        // the context is gone (process teardown) these calls fail and the
        // OS reclaims everything, as in the reference (context.cu:72-80).
        if (cudaStreamSynchronize(h->stream) == cudaSuccess) {
            if (cudaMemPoolDestroy(h->pool) != cudaSuccess) err = FFDAS_ERROR_CUDA_RUNTIME;
        }
        cudaGetLastError();
    }
    if (h->ev_start) cudaEventDestroy(h->ev_start);
    if (h->ev_stop) cudaEventDestroy(h->ev_stop);
    for (cudaEvent_t e : h->upload_ev)
        if (e) cudaEventDestroy(e);
    if (h->upload_stream) {
        cudaStreamSynchronize(h->upload_stream);
        cudaStreamDestroy(h->upload_stream);
    }
    if (h->status) cudaFree(h->status);
    if (h->solver && h->solver_release) h->solver_release(h->solver);
    cudaGetLastError();
    delete h;
    return err;
}

ffdas_error_t ffdas_set_channel_scale(ffdas_handle_t h, const float *scale, int64_t count) {
    if (!h) return FFDAS_ERROR_INVALID_HANDLE;
    if (scale && count <= 0) return FFDAS_ERROR_INVALID_ARGUMENT;
    h->chan_scale = scale;
    h->chan_scale_count = scale ? count : 0;
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_set_gram_engine(ffdas_handle_t h, int32_t engine) {
    if (!h) return FFDAS_ERROR_INVALID_HANDLE;
    if (engine < 0 || engine > 2) return FFDAS_ERROR_INVALID_ARGUMENT;
    h->gram_engine = engine;
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_set_stream(ffdas_handle_t h, uintptr_t stream) {
    if (!h) return FFDAS_ERROR_INVALID_HANDLE;
    h->stream = reinterpret_cast<cudaStream_t>(stream);
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_get_stream(ffdas_handle_t h, uintptr_t *stream) {
    if (!h) return FFDAS_ERROR_INVALID_HANDLE;
    if (!stream) return FFDAS_ERROR_NULL_POINTER;
    *stream = reinterpret_cast<uintptr_t>(h->stream);
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_das_set_config(ffdas_handle_t h, const ffdas_das_config_t *config) {
    if (!h) return FFDAS_ERROR_INVALID_HANDLE;
    if (!config) {
        h->has_config = false;
        std::memset(&h->config, 0, sizeof(h->config));
        return FFDAS_SUCCESS;
    }
    const ffdas_das_config_t &c = *config;
    auto pow2_or_zero = [](int v, int hi) { return v == 0 || (v > 0 && v <= hi && (v & (v - 1)) == 0); };
    if (c.variant < 0 || c.variant > 6 || c.variant == 4) return FFDAS_ERROR_INVALID_ARGUMENT;
    if (!pow2_or_zero(c.tile_x, 256) || !pow2_or_zero(c.tile_y, 256) || !pow2_or_zero(c.tile_z, 256))
        return FFDAS_ERROR_INVALID_ARGUMENT;
    if (!pow2_or_zero(c.batch_tile, 16)) return FFDAS_ERROR_INVALID_ARGUMENT;
    if (c.event_chunk < 0 || c.event_chunk > 16) return FFDAS_ERROR_INVALID_ARGUMENT;
    if (c.min_blocks < 0 || c.min_blocks > 32) return FFDAS_ERROR_INVALID_ARGUMENT;
    if (c.copy_engine < 0 || c.copy_engine > 2) return FFDAS_ERROR_INVALID_ARGUMENT;
    int tx = c.tile_x ? c.tile_x : 1, ty = c.tile_y ? c.tile_y : 1, tz = c.tile_z ? c.tile_z : 1;
    // variant 5 reads tile_x as lanes per voxel (1..32)
    if (c.variant == 5 && (c.tile_x > 32 || c.tile_y > 1 || c.tile_z > 1)) return FFDAS_ERROR_INVALID_ARGUMENT;
    if (c.variant != 5 && (c.tile_x || c.tile_y || c.tile_z) && (tx * ty * tz < 32 || tx * ty * tz > 1024))
        return FFDAS_ERROR_INVALID_ARGUMENT;
    h->config = c;
    h->has_config = true;
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_das_get_config(ffdas_handle_t h, ffdas_das_config_t *config) {
    if (!h) return FFDAS_ERROR_INVALID_HANDLE;
    if (!config) return FFDAS_ERROR_NULL_POINTER;
    *config = h->config;
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_get_last_kernel_info(ffdas_handle_t h, ffdas_kernel_info_t *info) {
    if (!h) return FFDAS_ERROR_INVALID_HANDLE;
    if (!info) return FFDAS_ERROR_NULL_POINTER;
    *info = h->last;
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_device_count(int *count) {
    if (!count) return FFDAS_ERROR_NULL_POINTER;
    FFDAS_CUDA(cudaGetDeviceCount(count));
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_device_get(int *device) {
    if (!device) return FFDAS_ERROR_NULL_POINTER;
    FFDAS_CUDA(cudaGetDevice(device));
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_device_set(int device) {
    int count = 0;
    FFDAS_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return FFDAS_ERROR_INVALID_DEVICE;
    FFDAS_CUDA(cudaSetDevice(device));
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_event_create(uintptr_t *event) {
    if (!event) return FFDAS_ERROR_NULL_POINTER;
    cudaEvent_t e;
    FFDAS_CUDA(cudaEventCreate(&e));
    *event = reinterpret_cast<uintptr_t>(e);
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_event_destroy(uintptr_t event) {
    if (event == 0) return FFDAS_SUCCESS;
    FFDAS_CUDA(cudaEventDestroy(reinterpret_cast<cudaEvent_t>(event)));
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_event_record(ffdas_handle_t h, uintptr_t event) {
    if (!h) return FFDAS_ERROR_INVALID_HANDLE;
    if (event == 0) return FFDAS_ERROR_INVALID_ARGUMENT;
    FFDAS_TRY(h->check_device());
    FFDAS_CUDA(cudaEventRecord(reinterpret_cast<cudaEvent_t>(event), h->stream));
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_event_synchronize(uintptr_t event) {
    if (event == 0) return FFDAS_ERROR_INVALID_ARGUMENT;
    FFDAS_CUDA(cudaEventSynchronize(reinterpret_cast<cudaEvent_t>(event)));
    return FFDAS_SUCCESS;
}

ffdas_error_t ffdas_event_elapsed_time(uintptr_t start, uintptr_t stop, float *ms) {
    if (!ms) return FFDAS_ERROR_NULL_POINTER;
    if (start == 0 || stop == 0) return FFDAS_ERROR_INVALID_ARGUMENT;
    FFDAS_CUDA(cudaEventElapsedTime(ms, reinterpret_cast<cudaEvent_t>(start),
                                    reinterpret_cast<cudaEvent_t>(stop)));
    return FFDAS_SUCCESS;
}

}  // extern "C"
