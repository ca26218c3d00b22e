// das_pairs.cuh -- interpolation-pair storage kinds, their ingest and taps.
//
// One storage kind per (channel-data dtype, compute type) combination that
// ffdas_das accepts (the reference's dispatch table, src/das/das.cu:40-82 and
// src/das/das_alg1.cu:157-188).  Each kind says how a pair is built from two
// consecutive samples and how one tap interpolates it.
#pragma once

#include "das_common.cuh"

namespace ffdas {

enum storage_kind : int {
    ST_F32 = 0,   // float2 (x0, x1 - x0)
    ST_F16 = 1,   // half2  (x0, x1)
    ST_BF16 = 2,  // u32    bf16 x0 (low half), bf16 x1 (high half)
    ST_F64 = 3,   // double2 (x0, x1 - x0)
    ST_C32 = 4,   // float4 (x0.re, x0.im, d.re, d.im)
    ST_C16 = 5,   // uint2 = half2 x0, half2 x1
    ST_C64 = 6,   // 2 x double2 (x0, d)
};

struct __align__(16) dpair2 { double2 a, d; };

template <int K> struct pair_traits;

template <> struct pair_traits<ST_F32> {
    using storage = float2;
    using value = float;
    using acc = float;
    static constexpr bool complex = false;
    __device__ static storage make(float x0, float x1) { return make_float2(x0, x1 - x0); }
    __device__ static value tap(storage p, float t) { return __fmaf_rn(t, p.y, p.x); }
    __device__ static value slope(storage p) { return p.y; }
};

// f16 pairs hold both samples, (x0, x1): a tap interpolates the stored f16
// values exactly (in f32) -- two conversions, one FADD, one FFMA.  Storing
// the slope instead would save the FADD but add an f16 rounding of x1 - x0.
template <> struct pair_traits<ST_F16> {
    using storage = __half2;
    using value = float;
    using acc = float;
    static constexpr bool complex = false;
    __device__ static storage make(float x0, float x1) { return __floats2half2_rn(x0, x1); }
    __device__ static value tap(storage p, float t) {
        const float2 f = __half22float2(p);
        return __fmaf_rn(t, f.y - f.x, f.x);
    }
    __device__ static value slope(storage p) {
        const float2 f = __half22float2(p);
        return f.y - f.x;
    }
};

// bf16 pair word: low half = bf16(x0), high half = bf16(x1).  Both samples
// are kept as stored, so a tap interpolates the bf16 data exactly (in f32);
// a bf16 slope would add its own rounding, which on 1024-channel volumes
// doubled the image error of bf16 channel data.  Each half widens to f32
// with one integer op (shift, mask).
template <> struct pair_traits<ST_BF16> {
    using storage = uint32_t;
    using value = float;
    using acc = float;
    static constexpr bool complex = false;
    __device__ static uint32_t bits(float v) {
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        return *reinterpret_cast<const uint16_t *>(&h);
    }
    __device__ static storage make(float x0, float x1) { return (bits(x1) << 16) | bits(x0); }
    __device__ static value tap(storage p, float t) {
        const float a = __uint_as_float(p << 16), b = __uint_as_float(p & 0xFFFF0000u);
        return __fmaf_rn(t, b - a, a);
    }
    __device__ static value slope(storage p) { return __uint_as_float(p & 0xFFFF0000u) - __uint_as_float(p << 16); }
};

template <> struct pair_traits<ST_F64> {
    using storage = double2;
    using value = double;
    using acc = double;
    static constexpr bool complex = false;
    __device__ static storage make(double x0, double x1) { return make_double2(x0, x1 - x0); }
    // src/core/math/vector.cuh:63: fma((double)t, s1 - s0, s0)
    __device__ static value tap(storage p, float t) { return fma((double)t, p.y, p.x); }
};

template <> struct pair_traits<ST_C32> {
    using storage = float4;
    using value = float2;
    using acc = float2;
    static constexpr bool complex = true;
    __device__ static storage make(float2 x0, float2 x1) {
        return make_float4(x0.x, x0.y, x1.x - x0.x, x1.y - x0.y);
    }
    __device__ static value tap(storage p, float t) {
        return make_float2(__fmaf_rn(t, p.z, p.x), __fmaf_rn(t, p.w, p.y));
    }
};

template <> struct pair_traits<ST_C16> {
    using storage = uint2;
    using value = float2;
    using acc = float2;
    static constexpr bool complex = true;
    __device__ static storage make(float2 x0, float2 x1) {
        __half2 a = __floats2half2_rn(x0.x, x0.y), b = __floats2half2_rn(x1.x, x1.y);
        return make_uint2(*reinterpret_cast<uint32_t *>(&a), *reinterpret_cast<uint32_t *>(&b));
    }
    __device__ static value tap(storage p, float t) {
        float2 a = __half22float2(*reinterpret_cast<__half2 *>(&p.x));
        float2 b = __half22float2(*reinterpret_cast<__half2 *>(&p.y));
        return make_float2(__fmaf_rn(t, b.x - a.x, a.x), __fmaf_rn(t, b.y - a.y, a.y));
    }
};

template <> struct pair_traits<ST_C64> {
    using storage = dpair2;
    using value = double2;
    using acc = double2;
    static constexpr bool complex = true;
    __device__ static storage make(double2 x0, double2 x1) {
        dpair2 r;
        r.a = x0;
        r.d = make_double2(x1.x - x0.x, x1.y - x0.y);
        return r;
    }
    __device__ static value tap(storage p, float t) {
        double td = (double)t;
        return make_double2(fma(td, p.d.x, p.a.x), fma(td, p.d.y, p.a.y));
    }
};

// ---- sample loaders for the ingest pass (input dtype -> working scalar) ----
template <typename T> struct sample_io;
template <> struct sample_io<float> { using w = float; __device__ static w load(const float *p) { return __ldg(p); } };
template <> struct sample_io<double> { using w = double; __device__ static w load(const double *p) { return __ldg(p); } };
template <> struct sample_io<__half> { using w = float; __device__ static w load(const __half *p) { return __half2float(*p); } };
template <> struct sample_io<__nv_bfloat16> { using w = float; __device__ static w load(const __nv_bfloat16 *p) { return __bfloat162float(*p); } };
template <> struct sample_io<int16_t> { using w = float; __device__ static w load(const int16_t *p) { return (float)__ldg(p); } };
template <> struct sample_io<float2> { using w = float2; __device__ static w load(const float2 *p) { return __ldg(p); } };
template <> struct sample_io<double2> { using w = double2; __device__ static w load(const double2 *p) { return __ldg(p); } };
template <> struct sample_io<__half2> { using w = float2; __device__ static w load(const __half2 *p) { return __half22float2(*p); } };

// per-channel gain of the ingest, applied to a working scalar in its own
// precision (FP32, or FP64 for FP64 data; both components of complex samples)
__device__ __forceinline__ float scaled(float v, float g) { return v * g; }
__device__ __forceinline__ double scaled(double v, float g) { return v * (double)g; }
__device__ __forceinline__ float2 scaled(float2 v, float g) { return make_float2(v.x * g, v.y * g); }
__device__ __forceinline__ double2 scaled(double2 v, float g) { return make_double2(v.x * (double)g, v.y * (double)g); }

// conversion of a working scalar to the storage kind's make() argument type
__device__ __forceinline__ float2 to_c32(float2 v) { return v; }
__device__ __forceinline__ float2 to_c32(double2 v) { return make_float2((float)v.x, (float)v.y); }
__device__ __forceinline__ double2 to_c64(double2 v) { return v; }
__device__ __forceinline__ double2 to_c64(float2 v) { return make_double2(v.x, v.y); }

template <int K, typename W> struct make_pair;
template <typename W> struct make_pair<ST_F32, W> {
    __device__ static float2 go(W a, W b) { return pair_traits<ST_F32>::make((float)a, (float)b); }
};
template <typename W> struct make_pair<ST_F16, W> {
    __device__ static __half2 go(W a, W b) { return pair_traits<ST_F16>::make((float)a, (float)b); }
};
template <typename W> struct make_pair<ST_BF16, W> {
    __device__ static uint32_t go(W a, W b) { return pair_traits<ST_BF16>::make((float)a, (float)b); }
};
template <typename W> struct make_pair<ST_F64, W> {
    __device__ static double2 go(W a, W b) { return pair_traits<ST_F64>::make((double)a, (double)b); }
};
template <typename W> struct make_pair<ST_C32, W> {
    __device__ static float4 go(W a, W b) { return pair_traits<ST_C32>::make(to_c32(a), to_c32(b)); }
};
template <typename W> struct make_pair<ST_C16, W> {
    __device__ static uint2 go(W a, W b) { return pair_traits<ST_C16>::make(to_c32(a), to_c32(b)); }
};
template <typename W> struct make_pair<ST_C64, W> {
    __device__ static dpair2 go(W a, W b) { return pair_traits<ST_C64>::make(to_c64(a), to_c64(b)); }
};

// Ingest: x[b,c,s,k] (any strides, sample stride 1) -> pair rows
// P[((b*C + c)*S + s)*Npad + k].  A thread builds kIngestVec consecutive
// pairs: consecutive threads read consecutive samples (each warp load
// instruction covers a few whole cache lines), the pairs go out as 16-byte
// stores, and the row of a block comes from blockIdx.y (event) and blockIdx.z
// (batch item x channel) without 64-bit divisions.
// Replaces the reference's cast/permute pre-pass (contiguous_copy_impl,
// src/tensor_ops/contiguous_copy_impl.cuh:17-57) and folds the pair build in.
constexpr int kIngestVec = 4;
constexpr int kIngestThreads = 256;

template <typename S>
struct alignas(sizeof(S) * kIngestVec >= 16 ? 16 : sizeof(S) * kIngestVec) pair_quad {
    S v[kIngestVec];
};

// With `gain` set, sample k of row (b, c, s) enters as gain[b * gain_bstride + c]
// times its value (a per-channel scale: ADC gains, or 1 / peak to normalise
// each channel before 16-bit storage).
template <typename Tin, int K>
__global__ void __launch_bounds__(kIngestThreads) ingest_pairs_kernel(
    const Tin *__restrict__ x, int64_t bstride, int64_t cstride, int64_t sstride,
    int C, int S, int N, int BC, int64_t Npad,
    typename pair_traits<K>::storage *__restrict__ P, const float *__restrict__ gain, int gain_bstride) {
    using st = typename pair_traits<K>::storage;
    using W = typename sample_io<Tin>::w;
    static_assert(sizeof(pair_quad<st>) == kIngestVec * sizeof(st), "pair_quad packing");
    const int64_t k0 = ((int64_t)blockIdx.x * kIngestThreads + threadIdx.x) * kIngestVec;
    if (k0 >= Npad) return;   // Npad is a multiple of kIngestVec
    for (int s = blockIdx.y; s < S; s += gridDim.y) {
        for (int bc = blockIdx.z; bc < BC; bc += gridDim.z) {
            const int c = bc % C, b = bc / C;
            const Tin *xr = x + (int64_t)b * bstride + (int64_t)c * cstride + (int64_t)s * sstride;
            const float g = gain ? __ldg(gain + (int64_t)b * gain_bstride + c) : 1.f;
            pair_quad<st> q;
            if (k0 + kIngestVec < (int64_t)N) {   // every pair of the quad inside the record
                W v[kIngestVec + 1];
#pragma unroll
                for (int i = 0; i <= kIngestVec; i++) v[i] = sample_io<Tin>::load(xr + k0 + i);
                if (gain) {
#pragma unroll
                    for (int i = 0; i <= kIngestVec; i++) v[i] = scaled(v[i], g);
                }
#pragma unroll
                for (int i = 0; i < kIngestVec; i++) q.v[i] = make_pair<K, W>::go(v[i], v[i + 1]);
            } else {
#pragma unroll
                for (int i = 0; i < kIngestVec; i++) {
                    const int64_t k = k0 + i;
                    if (k < (int64_t)N - 1) {
                        W a = sample_io<Tin>::load(xr + k);
                        W bb = sample_io<Tin>::load(xr + k + 1);
                        if (gain) {
                            a = scaled(a, g);
                            bb = scaled(bb, g);
                        }
                        q.v[i] = make_pair<K, W>::go(a, bb);
                    } else {
                        memset(&q.v[i], 0, sizeof(st));
                    }
                }
            }
            *reinterpret_cast<pair_quad<st> *>(P + ((int64_t)bc * S + s) * Npad + k0) = q;
        }
    }
}

}  // namespace ffdas
