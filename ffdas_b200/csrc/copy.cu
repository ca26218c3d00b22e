// copy.cu -- ffdas_contiguous_copy: strided -> C-contiguous copy with a cast.
//
// Same contract as the reference (src/tensor_ops/contiguous_copy.cu): dims of
// x and out must match, out must be contiguous, and the (x, out) dtype pair
// must be in the table below (the reference's pairs plus bfloat16).  Dims
// and strides travel as kernel parameters (no host-to-device copies), so the
// call can be captured in a CUDA graph.
#include <cuda_fp16.h>
#include <cuda_bf16.h>

#include "core.h"

namespace {

struct copy_shape {
    int nd;
    int64_t n;
    int64_t dims[FFDAS_MAX_DIMS];
    int64_t xstr[FFDAS_MAX_DIMS];
};

template <typename Tx, typename Ty> __device__ __forceinline__ Ty cvt(Tx v) { return static_cast<Ty>(v); }
template <> __device__ __forceinline__ __half cvt(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ float cvt(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ __half cvt(__half v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 cvt(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ float cvt(__nv_bfloat16 v) { return __bfloat162float(v); }
template <> __device__ __forceinline__ __nv_bfloat16 cvt(__nv_bfloat16 v) { return v; }
template <> __device__ __forceinline__ float cvt(short v) { return (float)v; }
template <> __device__ __forceinline__ float2 cvt(short2 v) { return make_float2((float)v.x, (float)v.y); }
template <> __device__ __forceinline__ short2 cvt(short2 v) { return v; }
template <> __device__ __forceinline__ __half2 cvt(float2 v) { return __floats2half2_rn(v.x, v.y); }
template <> __device__ __forceinline__ float2 cvt(__half2 v) { return __half22float2(v); }
template <> __device__ __forceinline__ __half2 cvt(__half2 v) { return v; }
template <> __device__ __forceinline__ float2 cvt(float2 v) { return v; }
template <> __device__ __forceinline__ double2 cvt(float2 v) { return make_double2(v.x, v.y); }
template <> __device__ __forceinline__ float2 cvt(double2 v) { return make_float2((float)v.x, (float)v.y); }
template <> __device__ __forceinline__ double2 cvt(double2 v) { return v; }

template <typename Tx, typename Ty>
__global__ void __launch_bounds__(256) strided_cast_kernel(const Tx *__restrict__ x, Ty *__restrict__ y,
                                                           copy_shape sh) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < sh.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t rem = i, off = 0;
        for (int d = sh.nd - 1; d >= 0; d--) {
            int64_t q = rem / sh.dims[d];
            off += (rem - q * sh.dims[d]) * sh.xstr[d];
            rem = q;
        }
        y[i] = cvt<Tx, Ty>(x[off]);
    }
}

template <typename Tx, typename Ty>
ffdas_error_t launch(ffdas_context &h, const copy_shape &sh, const void *x, void *y) {
    if (sh.n == 0) return FFDAS_SUCCESS;
    int64_t blocks = (sh.n + 255) / 256;
    if (blocks > (int64_t)h.sm_count * 32) blocks = (int64_t)h.sm_count * 32;
    strided_cast_kernel<Tx, Ty><<<(unsigned)blocks, 256, 0, h.stream>>>(static_cast<const Tx *>(x),
                                                                        static_cast<Ty *>(y), sh);
    return ffdas_launch_check(h.stream);
}

}  // namespace

extern "C" ffdas_error_t ffdas_contiguous_copy(ffdas_handle_t handle, ffdas_tensor_desc_t x_desc,
                                               const void *x, ffdas_tensor_desc_t out_desc, void *out) {
    if (!handle) return FFDAS_ERROR_INVALID_HANDLE;
    FFDAS_TRY(handle->check_device());
    if (!x_desc || !out_desc) return FFDAS_ERROR_NULL_POINTER;
    const ffdas_tensor_desc &xd = *x_desc, &od = *out_desc;
    if (xd.ndim != od.ndim) return FFDAS_ERROR_INVALID_DIMS;
    for (int64_t i = 0; i < xd.ndim; i++)
        if (xd.dims[i] != od.dims[i]) return FFDAS_ERROR_INVALID_DIMS;
    int64_t s = 1;
    for (int64_t i = od.ndim - 1; i >= 0; i--) {
        if (od.strides[i] != s) return FFDAS_ERROR_INVALID_DIMS;
        s *= od.dims[i];
    }
    copy_shape sh{};
    sh.nd = (int)xd.ndim;
    sh.n = xd.numel();
    for (int i = 0; i < sh.nd; i++) {
        sh.dims[i] = xd.dims[i];
        sh.xstr[i] = xd.strides[i];
    }
    if (sh.n > 0 && (!x || !out)) return FFDAS_ERROR_NULL_POINTER;
    ffdas_context &h = *handle;
#define PAIR(a, b) (((int)(a) << 8) | (int)(b))
    switch (PAIR(xd.dtype, od.dtype)) {
        case PAIR(FFDAS_R_16I, FFDAS_R_16I): return launch<short, short>(h, sh, x, out);
        case PAIR(FFDAS_R_16I, FFDAS_R_32F): return launch<short, float>(h, sh, x, out);
        case PAIR(FFDAS_R_16F, FFDAS_R_16F): return launch<__half, __half>(h, sh, x, out);
        case PAIR(FFDAS_R_16F, FFDAS_R_32F): return launch<__half, float>(h, sh, x, out);
        case PAIR(FFDAS_R_16BF, FFDAS_R_16BF): return launch<__nv_bfloat16, __nv_bfloat16>(h, sh, x, out);
        case PAIR(FFDAS_R_16BF, FFDAS_R_32F): return launch<__nv_bfloat16, float>(h, sh, x, out);
        case PAIR(FFDAS_R_32F, FFDAS_R_16F): return launch<float, __half>(h, sh, x, out);
        case PAIR(FFDAS_R_32F, FFDAS_R_16BF): return launch<float, __nv_bfloat16>(h, sh, x, out);
        case PAIR(FFDAS_R_32F, FFDAS_R_32F): return launch<float, float>(h, sh, x, out);
        case PAIR(FFDAS_R_32F, FFDAS_R_64F): return launch<float, double>(h, sh, x, out);
        case PAIR(FFDAS_C_16I, FFDAS_C_16I): return launch<short2, short2>(h, sh, x, out);
        case PAIR(FFDAS_C_16I, FFDAS_C_32F): return launch<short2, float2>(h, sh, x, out);
        case PAIR(FFDAS_C_16F, FFDAS_C_16F): return launch<__half2, __half2>(h, sh, x, out);
        case PAIR(FFDAS_C_16F, FFDAS_C_32F): return launch<__half2, float2>(h, sh, x, out);
        case PAIR(FFDAS_C_32F, FFDAS_C_16F): return launch<float2, __half2>(h, sh, x, out);
        case PAIR(FFDAS_C_32F, FFDAS_C_32F): return launch<float2, float2>(h, sh, x, out);
        case PAIR(FFDAS_C_32F, FFDAS_C_64F): return launch<float2, double2>(h, sh, x, out);
        case PAIR(FFDAS_R_64F, FFDAS_R_64F): return launch<double, double>(h, sh, x, out);
        case PAIR(FFDAS_R_64F, FFDAS_R_32F): return launch<double, float>(h, sh, x, out);
        case PAIR(FFDAS_C_64F, FFDAS_C_64F): return launch<double2, double2>(h, sh, x, out);
        case PAIR(FFDAS_C_64F, FFDAS_C_32F): return launch<double2, float2>(h, sh, x, out);
        default: break;
    }
#undef PAIR
    return FFDAS_ERROR_UNSUPPORTED_TYPE;
}
