// sparse_select.cu -- ffdas_sparse_select: the per-voxel event lists that a
// das_sparse call sums.
//
// The reference builds das_sparse inputs with its host array library
// (bindings/python/examples/sparse_compounding.py:141-144): per voxel the k
// events with the largest weight (argpartition over the event axis), then the
// weights and delays gathered at them (take_along_axis).  This kernel does the
// same on the device in one pass.  Up to 64 events: a CTA stages the (S, 32)
// weight and delay blocks of 32 consecutive voxels in shared memory
// (coalesced rows), each warp sorts a voxel's entries with a 64-element
// bitonic network over its lanes (two entries per lane, 64-bit keys that
// carry the order below), and the CTA writes the first k as (k, V) index,
// weight and delay rows, again coalesced.  More events: one thread per voxel
// streams the voxel's S weights (consecutive threads read consecutive
// voxels) and keeps the best KC entries, sorted, in registers with a
// branch-free compare-and-shift insertion.
//
// Order: larger weight first, NaN above every number (the host library sorts
// NaN last in ascending order, so NaN weights are among its k largest), ties
// to the lower event index.  argpartition leaves the order inside the k
// unspecified and may resolve ties differently; das_sparse sums the list, so
// only the rounding of the sum depends on the order.
#include "core.h"

namespace ffdas {

constexpr int kSelectThreads = 256;
constexpr int kSelectMaxK = 32;

// (a, ia) ranks before (b, ib); ib < 0 marks an empty slot, which every entry beats.
__device__ __forceinline__ bool select_before(float a, int ia, float b, int ib) {
    if (ib < 0) return true;
    const bool na = a != a, nb = b != b;
    if (na != nb) return na;
    if (!na && a != b) return a > b;
    return ia < ib;
}

template <int KC>
__global__ void __launch_bounds__(kSelectThreads) sparse_select_kernel(
    const float *__restrict__ w, const float *__restrict__ offs, int S, int64_t V, int k,
    int *__restrict__ idx, float *__restrict__ sw, float *__restrict__ so) {
    const int64_t v = (int64_t)blockIdx.x * kSelectThreads + threadIdx.x;
    if (v >= V) return;
    float tw[KC];
    int ti[KC];
#pragma unroll
    for (int p = 0; p < KC; p++) {
        tw[p] = 0.f;
        ti[p] = -1;
    }
    for (int s = 0; s < S; s++) {
        const float x = __ldg(w + (int64_t)s * V + v);
        // slot p takes slot p-1's entry when the new one ranks before it, the
        // new entry when it ranks before slot p's (but not slot p-1's), else
        // keeps its own; slots are updated from the last one down
#pragma unroll
        for (int p = KC - 1; p > 0; p--) {
            const bool before_prev = select_before(x, s, tw[p - 1], ti[p - 1]);
            const bool before_cur = select_before(x, s, tw[p], ti[p]);
            tw[p] = before_prev ? tw[p - 1] : (before_cur ? x : tw[p]);
            ti[p] = before_prev ? ti[p - 1] : (before_cur ? s : ti[p]);
        }
        const bool first = select_before(x, s, tw[0], ti[0]);
        tw[0] = first ? x : tw[0];
        ti[0] = first ? s : ti[0];
    }
#pragma unroll
    for (int p = 0; p < KC; p++) {
        if (p < k) {
            idx[(int64_t)p * V + v] = ti[p];
            if (sw) sw[(int64_t)p * V + v] = tw[p];
            if (so) so[(int64_t)p * V + v] = __ldg(offs + (int64_t)ti[p] * V + v);
        }
    }
}

// Sort key of an entry: larger ranks first.  High word: the weight's bits
// mapped to an order-preserving unsigned integer (-0 taken as +0, every NaN
// above +inf); low word: ~event, so the lower event ranks first among equal
// weights.  0 (below every entry) pads a list shorter than 64.
__device__ __forceinline__ unsigned long long select_key(float x, int s) {
    uint32_t u = __float_as_uint(x);
    if (u == 0x80000000u) u = 0u;
    const uint32_t hi = x != x ? 0xffffffffu : ((u & 0x80000000u) ? ~u : (u | 0x80000000u));
    return ((unsigned long long)hi << 32) | (uint32_t)~(uint32_t)s;
}

constexpr int kSelectVoxels = 32;           // voxels per CTA (one 128-byte row segment)
constexpr int kSelectWarps = 8;
constexpr int kSelectPitch = kSelectVoxels + 1;   // shared rows padded: a warp's column reads meet no conflicts

__global__ void __launch_bounds__(32 * kSelectWarps) sparse_select_warp_kernel(
    const float *__restrict__ w, const float *__restrict__ offs, int S, int64_t V, int k,
    int *__restrict__ idx, float *__restrict__ sw, float *__restrict__ so) {
    __shared__ float tw[64][kSelectPitch], to[64][kSelectPitch];
    __shared__ int oi[kSelectMaxK][kSelectPitch];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t v0 = (int64_t)blockIdx.x * kSelectVoxels;
    for (int e = tid; e < S * kSelectVoxels; e += 32 * kSelectWarps) {
        const int sv = e / kSelectVoxels, c = e % kSelectVoxels;
        const int64_t v = v0 + c;
        tw[sv][c] = v < V ? __ldg(w + (int64_t)sv * V + v) : 0.f;
        if (offs) to[sv][c] = v < V ? __ldg(offs + (int64_t)sv * V + v) : 0.f;
    }
    __syncthreads();
    for (int c = warp; c < kSelectVoxels; c += kSelectWarps) {
        if (v0 + c >= V) break;   // warp-uniform
        // entry e = lane + 32 j; ascending bitonic sort of the 64 keys
        unsigned long long key[2];
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int sv = lane + 32 * j;
            key[j] = sv < S ? select_key(tw[sv][c], sv) : 0ull;
        }
#pragma unroll
        for (int size = 2; size <= 64; size <<= 1) {
#pragma unroll
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                if (stride == 32) {   // partner: the lane's other entry (size 64: ascending)
                    const unsigned long long lo = key[0] < key[1] ? key[0] : key[1];
                    const unsigned long long hi = key[0] < key[1] ? key[1] : key[0];
                    key[0] = lo;
                    key[1] = hi;
                } else {
#pragma unroll
                    for (int j = 0; j < 2; j++) {
                        const int e = lane + 32 * j;
                        const unsigned long long other = __shfl_xor_sync(0xffffffffu, key[j], stride);
                        const bool lower = (e & stride) == 0, up = (e & size) == 0;
                        const bool keep_small = lower == up;
                        const bool other_smaller = other < key[j];
                        key[j] = (keep_small == other_smaller) ? other : key[j];
                    }
                }
            }
        }
        // rank p (0 = first) is entry 63 - p: lane 31 - p, j = 1
        const int p = 31 - lane;
        if (p < k) oi[p][c] = (int)~(uint32_t)(key[1] & 0xffffffffull);
    }
    __syncthreads();
    for (int e = tid; e < k * kSelectVoxels; e += 32 * kSelectWarps) {
        const int p = e / kSelectVoxels, c = e % kSelectVoxels;
        const int64_t v = v0 + c;
        if (v >= V) continue;
        const int sv = oi[p][c];
        idx[(int64_t)p * V + v] = sv;
        if (sw) sw[(int64_t)p * V + v] = tw[sv][c];
        if (so) so[(int64_t)p * V + v] = to[sv][c];
    }
}

template <int KC>
static ffdas_error_t launch_select(ffdas_context &h, const float *w, const float *offs, int S, int64_t V, int k,
                                   int *idx, float *sw, float *so) {
    const int64_t blocks = (V + kSelectThreads - 1) / kSelectThreads;
    if (blocks > INT32_MAX) return FFDAS_ERROR_DIMS_TOO_LARGE;
    sparse_select_kernel<KC><<<(unsigned)blocks, kSelectThreads, 0, h.stream>>>(w, offs, S, V, k, idx, sw, so);
    return ffdas_launch_check(h.stream);
}

}  // namespace ffdas

using namespace ffdas;

extern "C" ffdas_error_t ffdas_sparse_select(ffdas_handle_t handle, const float *weights, const float *offsets,
                                             int n_events, int64_t n_voxels, int k, int *sparse_indices,
                                             float *sparse_weights, float *sparse_offsets) {
    if (!handle) return FFDAS_ERROR_INVALID_HANDLE;
    FFDAS_TRY(handle->check_device());
    if (n_events <= 0 || n_voxels < 0 || k <= 0 || k > n_events || k > kSelectMaxK)
        return FFDAS_ERROR_INVALID_ARGUMENT;
    if (n_voxels == 0) return FFDAS_SUCCESS;
    if (!weights || !sparse_indices || (sparse_offsets && !offsets)) return FFDAS_ERROR_NULL_POINTER;
    ffdas_context &h = *handle;
    const float *offs = sparse_offsets ? offsets : nullptr;
    if (n_events <= 64) {
        const int64_t blocks = (n_voxels + kSelectVoxels - 1) / kSelectVoxels;
        if (blocks > INT32_MAX) return FFDAS_ERROR_DIMS_TOO_LARGE;
        sparse_select_warp_kernel<<<(unsigned)blocks, 32 * kSelectWarps, 0, h.stream>>>(
            weights, offs, n_events, n_voxels, k, sparse_indices, sparse_weights, sparse_offsets);
        return ffdas_launch_check(h.stream);
    }
    if (k <= 1) return launch_select<1>(h, weights, offs, n_events, n_voxels, k, sparse_indices, sparse_weights, sparse_offsets);
    if (k <= 2) return launch_select<2>(h, weights, offs, n_events, n_voxels, k, sparse_indices, sparse_weights, sparse_offsets);
    if (k <= 4) return launch_select<4>(h, weights, offs, n_events, n_voxels, k, sparse_indices, sparse_weights, sparse_offsets);
    if (k <= 8) return launch_select<8>(h, weights, offs, n_events, n_voxels, k, sparse_indices, sparse_weights, sparse_offsets);
    if (k <= 16) return launch_select<16>(h, weights, offs, n_events, n_voxels, k, sparse_indices, sparse_weights, sparse_offsets);
    return launch_select<32>(h, weights, offs, n_events, n_voxels, k, sparse_indices, sparse_weights, sparse_offsets);
}
