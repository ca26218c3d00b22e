// das_common.cuh -- shared device helpers for the delay-and-sum kernels.
//
// Interpolation-pair storage ("pairs"): the ingest kernel rewrites channel data
// x[b,c,s,k] into rows of pairs P[b,c,s,k] that hold everything one
// linear-interpolation tap needs, so the hot loop issues ONE load per unit and
// needs no bounds test:
//   f32 / f64 / c32 / c64 : P[k] = (x[k], x[k+1] - x[k])     for 0 <= k <= N-2
//   f16 / bf16 / c16      : P[k] = (x[k], x[k+1])            for 0 <= k <= N-2
//   all                   : P[k] = 0                         for N-1 <= k < Npad
// A sample index outside [0, Npad) is clamped to Npad-1 (a zero pair), which
// reproduces the reference's validity rule 0 <= k < N-1
// (src/das/das_alg1_kernels.cuh:70) without a compare per unit.
// For f32 the stored difference is exactly the reference's `s1 - s0`, so
// lerp = fma(t, d, x0) is bit-identical to lerp() in
// src/core/math/vector.cuh:15.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <cstdint>

namespace ffdas {

// floor(tau) and tau - floor(tau) without the quarter-rate F2I/I2F
// conversions: adding 1.5*2^23 with round-toward-minus-infinity leaves
// floor(tau) in the low mantissa bits.  Exact for |tau| < 2^22; larger or
// non-finite tau yields an index that the caller clamps to the zero pair.
// (The reference computes the same pair with __float2int_rd/__int2float_rn,
// src/das/das_device_utils.cuh:10-13.)
constexpr float kFloorMagic = 12582912.0f;       // 1.5 * 2^23
constexpr uint32_t kFloorMagicBits = 0x4B400000u;

struct tau_split {
    uint32_t k;   // sample index, wraps to a huge value when negative
    float t;      // fractional part
};

__device__ __forceinline__ tau_split split_tau(float tau) {
    float m = __fadd_rd(tau, kFloorMagic);
    float fl = m - kFloorMagic;
    tau_split r;
    r.t = tau - fl;
    r.k = __float_as_uint(m) - kFloorMagicBits;
    return r;
}

// Distance term exactly as the reference forms it
// (src/das/das_alg1_kernels.cuh:60-66): rsq = max(|d|^2, 1e-7),
// tau = fma(rsq, rsqrt(rsq), offset).  Keeping rsq and rsqrt(rsq) per
// (voxel, channel) lets each event add its offset with one FFMA and produce
// the reference's tau bit for bit.
struct recv_geom {
    float rsq;
    float rinv;
};

__device__ __forceinline__ recv_geom receive_geometry(float vx, float vy, float vz,
                                                      float cx, float cy, float cz) {
    float dx = vx - cx, dy = vy - cy, dz = vz - cz;
    // Written as the same source expression the reference uses so that, built
    // with --fmad=true, it contracts into the same FFMA chain.
    float rsq = dx * dx + dy * dy + dz * dz;
    rsq = fmaxf(rsq, 1e-7f);
    recv_geom g;
    g.rsq = rsq;
    g.rinv = rsqrtf(rsq);
    return g;
}

// Directivity test (src/das/das_alg1_kernels.cuh:72-76): a channel whose
// normal makes too large an angle with the voxel is excluded.  Excluded
// channels get rsq = 1e30, rinv = 1, so tau is finite and huge and its index
// lands on the zero pair.
__device__ __forceinline__ void apply_directivity(recv_geom &g, float vx, float vy, float vz,
                                                  float cx, float cy, float cz,
                                                  float4 dir) {
    float dx = vx - cx, dy = vy - cy, dz = vz - cz;
    float proj = (dx * dir.x + dy * dir.y + dz * dir.z) * g.rinv;
    if (!(proj > dir.w)) {
        g.rsq = 1e30f;
        g.rinv = 1.0f;
    }
}

__device__ __forceinline__ float bf16lo_to_f32(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf16hi_to_f32(uint32_t u) { return __uint_as_float(u & 0xFFFF0000u); }

}  // namespace ffdas
