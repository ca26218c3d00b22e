// truncate_rank.cu -- ffdas_truncate_rank: keep the singular components
// [start, stop) of a 2-D matrix.  This is the slow-time clutter filter that
// follows delay-and-sum on a frame ensemble: frames x voxels, with the
// leading components (tissue) removed.
//
// Reference: src/truncate_rank/truncate_rank.cu:6-42 (entry point, dtype
// switch) and src/truncate_rank/truncate_rank_impl.cuh:426-513 (Gram matrix of
// the smaller side, eigendecomposition, projection).  The result is
//     out = U_k U_k^H A,   U_k = left singular vectors start..stop-1 of A,
// where A is x viewed as a (p, q) matrix with p = min(m, n) rows: x itself
// when m <= n, else its transpose (then the filter reads out = x V_k V_k^H
// with V the right singular vectors, the same result).
//
// Steps on the device:
//  1. G = A A^H / q, p x p, split over q into partial sums that a second
//     kernel adds in a fixed order in double.  The sum is therefore the same
//     on every run.  It is written as the column-major Hermitian matrix that
//     the solver takes.  The reference forms the full product with one
//     cuBLAS GEMM.  FP32 rows (A = x, p <= 256) run on the tensor cores
//     (gram_tc.cuh: tcgen05, each element split into two TF32 parts, three
//     products); every other case, or ffdas_set_gram_engine(1), runs a tiled
//     SIMT product over the upper-triangle tiles only.
//  2. The basis of step 3.  When it is the leading subspace (the clutter
//     filter: remove ranks 0..start-1; or keep ranks 0..stop-1) and has at
//     most 16 vectors, an orthogonal iteration in double on the device
//     (G Q, Cholesky QR twice) runs first and is accepted at a backward-
//     stable residual ||G Q - Q H|| <= 2 eps(FP32) max H_aa (45 eps for
//     FP64): the subspace is then as accurate as a dense solver's for this G.
//     Otherwise, or if it has not converged after 30 steps, the
//     eigendecomposition of G runs in cuSOLVER's syevd, as in the reference,
//     or syevdx over one index range when the basis is one contiguous run of
//     eigenvectors.  The library is loaded at the first call that needs
//     it, so the delay-and-sum path and the iteration never depend on it.  Eigenvalues come
//     back ascending, so singular rank s is eigenvector p-1-s.
//  3. Projection with the smaller basis.  With k = stop-start kept vectors
//     and c = p-k removed ones, out = U_k (U_k^H A) when k <= c, else
//     out = A - U_c (U_c^H A).  Both are exact for an orthonormal
//     eigenbasis.  The reference forms P = V_k V_k^H (SYRK) and applies it
//     with one SYMM: 2 p^2 q multiply-adds.  Here the clutter filter
//     (start = a few tissue ranks, stop = p) costs 4 c p q, and with up to 32
//     basis vectors it is one pass over A: each thread owns one column,
//     keeps U^H a in registers, and writes the filtered column.  Larger
//     bases run as two tiled products through a (r, q) workspace.
//  With k = p (keep everything) out is x, copied.
//
// A single TF32 product would not do: the filter subtracts a dominant
// component, and TF32 carries errors of about 1e-3 of |x|, the size of the
// signal that remains.  The three-product split keeps each Gram term within
// about 2^-21 of |a|^2, and the projection stays in FP32 FMAs.
#include "core.h"
#include "gram_tc.cuh"

#include <cusolverDn.h>
#include <dlfcn.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <vector>

namespace ffdas {
namespace {

// ---------------------------------------------------------------- elements

template <typename T> struct tr_elem;
template <> struct tr_elem<float> {
    using real = float;
    using acc = double;
    static constexpr cudaDataType cuda = CUDA_R_32F, cuda_real = CUDA_R_32F;
};
template <> struct tr_elem<double> {
    using real = double;
    using acc = double;
    static constexpr cudaDataType cuda = CUDA_R_64F, cuda_real = CUDA_R_64F;
};
template <> struct tr_elem<float2> {
    using real = float;
    using acc = double2;
    static constexpr cudaDataType cuda = CUDA_C_32F, cuda_real = CUDA_R_32F;
};
template <> struct tr_elem<double2> {
    using real = double;
    using acc = double2;
    static constexpr cudaDataType cuda = CUDA_C_64F, cuda_real = CUDA_R_64F;
};

template <typename T> __device__ __forceinline__ T tr_zero();
template <> __device__ __forceinline__ float tr_zero<float>() { return 0.f; }
template <> __device__ __forceinline__ double tr_zero<double>() { return 0.0; }
template <> __device__ __forceinline__ float2 tr_zero<float2>() { return make_float2(0.f, 0.f); }
template <> __device__ __forceinline__ double2 tr_zero<double2>() { return make_double2(0.0, 0.0); }

__device__ __forceinline__ float tr_conj(float a) { return a; }
__device__ __forceinline__ double tr_conj(double a) { return a; }
__device__ __forceinline__ float2 tr_conj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ double2 tr_conj(double2 a) { return make_double2(a.x, -a.y); }

// c += a * b
__device__ __forceinline__ void tr_mac(float &c, float a, float b) { c = fmaf(a, b, c); }
__device__ __forceinline__ void tr_mac(double &c, double a, double b) { c = fma(a, b, c); }
__device__ __forceinline__ void tr_mac(float2 &c, float2 a, float2 b) {
    c.x = fmaf(a.x, b.x, c.x);
    c.x = fmaf(-a.y, b.y, c.x);
    c.y = fmaf(a.x, b.y, c.y);
    c.y = fmaf(a.y, b.x, c.y);
}
__device__ __forceinline__ void tr_mac(double2 &c, double2 a, double2 b) {
    c.x = fma(a.x, b.x, c.x);
    c.x = fma(-a.y, b.y, c.x);
    c.y = fma(a.x, b.y, c.y);
    c.y = fma(a.y, b.x, c.y);
}

// a + s * b (s = +1 or -1)
__device__ __forceinline__ float tr_axpy(float a, float s, float b) { return fmaf(s, b, a); }
__device__ __forceinline__ double tr_axpy(double a, double s, double b) { return fma(s, b, a); }
__device__ __forceinline__ float2 tr_axpy(float2 a, float s, float2 b) {
    return make_float2(fmaf(s, b.x, a.x), fmaf(s, b.y, a.y));
}
__device__ __forceinline__ double2 tr_axpy(double2 a, double s, double2 b) {
    return make_double2(fma(s, b.x, a.x), fma(s, b.y, a.y));
}

// double accumulation of the Gram partials
__device__ __forceinline__ void tr_acc_add(double &c, float a) { c += (double)a; }
__device__ __forceinline__ void tr_acc_add(double &c, double a) { c += a; }
__device__ __forceinline__ void tr_acc_add(double2 &c, float2 a) { c.x += (double)a.x; c.y += (double)a.y; }
__device__ __forceinline__ void tr_acc_add(double2 &c, double2 a) { c.x += a.x; c.y += a.y; }
template <typename T> __device__ __forceinline__ typename tr_elem<T>::acc tr_acc_zero();
template <> __device__ __forceinline__ double tr_acc_zero<float>() { return 0.0; }
template <> __device__ __forceinline__ double tr_acc_zero<double>() { return 0.0; }
template <> __device__ __forceinline__ double2 tr_acc_zero<float2>() { return make_double2(0.0, 0.0); }
template <> __device__ __forceinline__ double2 tr_acc_zero<double2>() { return make_double2(0.0, 0.0); }
__device__ __forceinline__ void tr_store(float &o, double v, double s) { o = (float)(v * s); }
__device__ __forceinline__ void tr_store(double &o, double v, double s) { o = v * s; }
__device__ __forceinline__ void tr_store(float2 &o, double2 v, double s) {
    o = make_float2((float)(v.x * s), (float)(v.y * s));
}
__device__ __forceinline__ void tr_store(double2 &o, double2 v, double s) { o = make_double2(v.x * s, v.y * s); }

// ---------------------------------------------------------- tiled product

constexpr int kTrTile = 64;       // C tile edge
constexpr int kTrTileK = 32;      // host-side k granularity (a multiple of every tr_tile_k)
constexpr int kTrThreads = 256;   // 16 x 16 threads, 4 x 4 outputs each (rows 4 ty + a, columns 4 tx + b)

template <typename T>
struct tr_gemm_args {
    const T *L;          // L(i, k) = L[i * li + k * lk]
    int64_t li, lk;
    const T *R;          // R(k, j) = R[k * rk + j * rj]
    int64_t rk, rj;
    T *C;                // C(i, j) = C[z * zstride + i * ci + j * cj]
    int64_t ci, cj;
    const T *base;       // when set, C = base + sign * sum (base has C's strides)
    int64_t M, N, K;
    int64_t kchunk;      // blockIdx.z sums k in [z * kchunk, (z + 1) * kchunk), a multiple of kTrTileK
    int64_t zstride;
    int conj_l, conj_r, upper;   // conjugate an operand; skip tiles below the diagonal
    typename tr_elem<T>::real sign;
};

// four consecutive elements, read from shared memory as 16-byte vectors
template <typename T> struct __align__(16) tr_quad { T v[4]; };

// A thread's 4 x 4 accumulators.  For float they are held as pairs, so
// that a step of the tile is 8 packed FMAs (the same operations and
// rounding as 16 scalar ones, half the issue slots).
template <typename T> struct tr_accum {
    T c[4][4];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int x = 0; x < 4; x++)
#pragma unroll
            for (int y = 0; y < 4; y++) c[x][y] = tr_zero<T>();
    }
    __device__ __forceinline__ void mac(const tr_quad<T> &l, const tr_quad<T> &r) {
#pragma unroll
        for (int x = 0; x < 4; x++)
#pragma unroll
            for (int y = 0; y < 4; y++) tr_mac(c[x][y], l.v[x], r.v[y]);
    }
    __device__ __forceinline__ T get(int x, int y) const { return c[x][y]; }
};
template <> struct tr_accum<float> {
    float2 c[4][2];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int x = 0; x < 4; x++) c[x][0] = c[x][1] = make_float2(0.f, 0.f);
    }
    __device__ __forceinline__ void mac(const tr_quad<float> &l, const tr_quad<float> &r) {
        const float2 r01 = make_float2(r.v[0], r.v[1]), r23 = make_float2(r.v[2], r.v[3]);
#pragma unroll
        for (int x = 0; x < 4; x++) {
            const float2 lx = make_float2(l.v[x], l.v[x]);
            c[x][0] = __ffma2_rn(lx, r01, c[x][0]);
            c[x][1] = __ffma2_rn(lx, r23, c[x][1]);
        }
    }
    __device__ __forceinline__ float get(int x, int y) const { return (y & 1) ? c[x][y >> 1].y : c[x][y >> 1].x; }
};

// k depth staged per step: 32 for float, 16 for 8-byte and 8 for 16-byte
// elements (two stages of both operand tiles, 34 KB, within the 48 KB of
// static shared memory).  The step is deep so that each CTA keeps several KB
// of loads in flight: with 16 floats per step the FP32 Gram was bound by the
// latency of its loads (0.33 ms at 1.6 TB/s from L2 for 200 x 102400).
template <typename T> constexpr int tr_tile_k() { return sizeof(T) > 8 ? 8 : (sizeof(T) == 4 ? 32 : 16); }

// C = op(L) op(R) over a 64 x 64 tile of C per CTA.  Each operand tile is
// loaded with consecutive threads on its unit-stride index, so the loads
// coalesce whichever way the operand is laid out.  Two shared-memory stages:
// the next tiles are loaded into registers while the current ones are used,
// one barrier per step.
// resident CTAs per SM the register budget is sized for: 3 for float (79
// registers), 2 for the 8- and 16-byte elements (their 4 x 4 accumulators)
template <typename T> constexpr int tr_min_blocks() { return sizeof(T) == 4 ? 3 : 2; }

template <typename T>
__global__ void __launch_bounds__(kTrThreads, tr_min_blocks<T>()) tr_gemm_kernel(const tr_gemm_args<T> a) {
    constexpr int BK = tr_tile_k<T>();
    constexpr int U = kTrTile * BK / kTrThreads;   // elements of each operand a thread stages per step
    const int64_t bi = blockIdx.y, bj = blockIdx.x;
    if (a.upper && bi > bj) return;
    // rows padded by 4 elements: a thread's 4 consecutive entries start on a
    // 16-byte boundary and are read with 16-byte shared loads
    __shared__ __align__(16) T sL[2][BK][kTrTile + 4];
    __shared__ __align__(16) T sR[2][BK][kTrTile + 4];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int64_t i0 = bi * kTrTile, j0 = bj * kTrTile;
    const int64_t kbeg = (int64_t)blockIdx.z * a.kchunk;
    const int64_t kend = min(a.K, kbeg + a.kchunk);
    const bool l_kfast = a.lk == 1, r_kfast = a.rk == 1;
    tr_accum<T> acc;
    acc.zero();

    T rl[U], rr[U];
    auto fetch = [&](int64_t k0) {
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int e = tid + u * kTrThreads;
            int kk = l_kfast ? (e % BK) : (e / kTrTile);
            const int ii = l_kfast ? (e / BK) : (e % kTrTile);
            int64_t k = k0 + kk;
            T v = tr_zero<T>();
            if (i0 + ii < a.M && k < kend) {
                v = a.L[(i0 + ii) * a.li + k * a.lk];
                if (a.conj_l) v = tr_conj(v);
            }
            rl[u] = v;
            kk = r_kfast ? (e % BK) : (e / kTrTile);
            const int jj = r_kfast ? (e / BK) : (e % kTrTile);
            k = k0 + kk;
            T w = tr_zero<T>();
            if (j0 + jj < a.N && k < kend) {
                w = a.R[k * a.rk + (j0 + jj) * a.rj];
                if (a.conj_r) w = tr_conj(w);
            }
            rr[u] = w;
        }
    };
    auto stage = [&](int buf) {
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int e = tid + u * kTrThreads;
            sL[buf][l_kfast ? (e % BK) : (e / kTrTile)][l_kfast ? (e / BK) : (e % kTrTile)] = rl[u];
            sR[buf][r_kfast ? (e % BK) : (e / kTrTile)][r_kfast ? (e / BK) : (e % kTrTile)] = rr[u];
        }
    };

    if (kbeg < kend) {
        fetch(kbeg);
        stage(0);
    }
    __syncthreads();
    int buf = 0;
    for (int64_t k0 = kbeg; k0 < kend; k0 += BK) {
        const bool more = k0 + BK < kend;
        if (more) fetch(k0 + BK);       // in flight while this step computes
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            const tr_quad<T> l = *reinterpret_cast<const tr_quad<T> *>(&sL[buf][kk][4 * ty]);
            const tr_quad<T> r = *reinterpret_cast<const tr_quad<T> *>(&sR[buf][kk][4 * tx]);
            acc.mac(l, r);
        }
        // the other stage was last read before the previous barrier
        if (more) stage(buf ^ 1);
        __syncthreads();
        buf ^= 1;
    }
    T *C = a.C + (int64_t)blockIdx.z * a.zstride;
#pragma unroll
    for (int x = 0; x < 4; x++) {
        const int64_t i = i0 + 4 * ty + x;
        if (i >= a.M) continue;
#pragma unroll
        for (int y = 0; y < 4; y++) {
            const int64_t j = j0 + 4 * tx + y;
            if (j >= a.N) continue;
            T v = acc.get(x, y);
            if (a.base) v = tr_axpy(a.base[i * a.ci + j * a.cj], a.sign, v);
            C[i * a.ci + j * a.cj] = v;
        }
    }
}

// G (column-major, p x p, both triangles) = scale * sum over the splits of
// the partials, in double and in a fixed order: a CTA takes 32 consecutive
// elements, warp w adds splits w, w+8, ..., and the eight warp sums are added
// in warp order.  The partials are row-major (FMA kernel) or column-major
// (tensor-core kernel, `cm`); only i <= j is read: every upper-triangle
// element lies in a computed tile.
constexpr int kReduceWarps = 8;

template <typename T>
__global__ void __launch_bounds__(32 * kReduceWarps) tr_gram_reduce_kernel(const T *__restrict__ part, int splits,
                                                                          int64_t p, double scale, int cm,
                                                                          T *__restrict__ G) {
    using acc_t = typename tr_elem<T>::acc;
    __shared__ acc_t red[kReduceWarps][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t e = (int64_t)blockIdx.x * 32 + lane;
    const int64_t major = e / p, minor = e - major * p;
    const int64_t i = cm ? minor : major, j = cm ? major : minor;
    const bool use = e < p * p && i <= j;
    acc_t s = tr_acc_zero<T>();
    if (use) {
        const int64_t pp = p * p;
#pragma unroll 4
        for (int z = w; z < splits; z += kReduceWarps) tr_acc_add(s, part[(int64_t)z * pp + e]);
    }
    red[w][lane] = s;
    __syncthreads();
    if (w != 0 || !use) return;
    acc_t t = red[0][lane];
#pragma unroll
    for (int k = 1; k < kReduceWarps; k++) tr_acc_add(t, red[k][lane]);
    T v;
    tr_store(v, t, scale);
    G[i + j * p] = v;
    G[j + i * p] = tr_conj(v);
}

// U[i * r + t] = V[i + e(t) * p] (row-major p x r basis), e(t) = e0 + t for
// t < r0, else e1 + t - r0.
template <typename T>
__global__ void tr_gather_basis_kernel(const T *__restrict__ V, int64_t p, int r, int64_t e0, int r0, int64_t e1,
                                       T *__restrict__ U) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= p * r) return;
    const int64_t i = e / r;
    const int t = (int)(e - i * r);
    const int64_t col = t < r0 ? e0 + t : e1 + (t - r0);
    U[e] = V[i + col * p];
}

// One pass over A for bases of up to RMAX vectors.  A CTA takes 32
// consecutive columns (one per lane, so every row read is one coalesced
// segment) and splits the rows among its warps: warp g forms its partial
// U^H a_j over its block of rows, the partials meet in shared memory and each
// warp adds them in group order (the same order in every warp, so every warp
// holds the same w), then writes U w (or a_j - U w) over its rows.  The basis
// sits in shared memory and is read as a broadcast.  Rows are read in
// batches of kProjBatch so that several loads are in flight per thread.
// out may alias x: each element is read before it is written, by the thread
// that writes it, and all reads of phase 1 end at the barrier.
constexpr int kProjBatch = 8;
constexpr int kProjMaxGroups = 8;
constexpr size_t kSmallBasisSmem = 48 * 1024;   // dynamic shared memory without an opt-in

template <typename T, int RMAX>
__global__ void __launch_bounds__(32 * kProjMaxGroups) tr_project_small_kernel(
    const T *x, int64_t sp, int64_t sq, int64_t p, int64_t q, const T *__restrict__ U, int r, int subtract,
    T *out, const int *gate) {
    if (gate && *gate != 1) return;
    extern __shared__ __align__(16) unsigned char tr_smem[];
    T *sU = reinterpret_cast<T *>(tr_smem);      // p x r
    T *red = sU + p * r;                          // [groups][r][32]
    const int groups = blockDim.x >> 5, g = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int64_t e = threadIdx.x; e < p * r; e += blockDim.x) sU[e] = U[e];
    __syncthreads();
    const int64_t j = (int64_t)blockIdx.x * 32 + lane;
    const bool ok = j < q;
    const int64_t rows = (p + groups - 1) / groups;
    const int64_t l0 = min(p, g * rows), l1 = min(p, l0 + rows);
    const T *col = x + (ok ? j : 0) * sq;
    T w[RMAX];
#pragma unroll
    for (int t = 0; t < RMAX; t++) w[t] = tr_zero<T>();
    if (ok) {
        int64_t l = l0;
        for (; l + kProjBatch <= l1; l += kProjBatch) {
            T v[kProjBatch];
#pragma unroll
            for (int b = 0; b < kProjBatch; b++) v[b] = col[(l + b) * sp];
#pragma unroll
            for (int b = 0; b < kProjBatch; b++) {
                const T *u = sU + (l + b) * r;
#pragma unroll
                for (int t = 0; t < RMAX; t++)
                    if (t < r) tr_mac(w[t], tr_conj(u[t]), v[b]);
            }
        }
        for (; l < l1; l++) {
            const T v = col[l * sp];
            const T *u = sU + l * r;
#pragma unroll
            for (int t = 0; t < RMAX; t++)
                if (t < r) tr_mac(w[t], tr_conj(u[t]), v);
        }
    }
#pragma unroll
    for (int t = 0; t < RMAX; t++)
        if (t < r) red[((int64_t)g * r + t) * 32 + lane] = w[t];
    __syncthreads();
    if (!ok) return;
    const typename tr_elem<T>::real one = 1;
#pragma unroll
    for (int t = 0; t < RMAX; t++) {
        if (t >= r) continue;
        T s = red[(int64_t)t * 32 + lane];
        for (int k = 1; k < groups; k++) s = tr_axpy(s, one, red[((int64_t)k * r + t) * 32 + lane]);
        w[t] = s;
    }
    T *oc = out + j * sq;
    const typename tr_elem<T>::real minus = -1;
    int64_t l = l0;
    for (; l + kProjBatch <= l1; l += kProjBatch) {
        T v[kProjBatch];
        if (subtract) {
#pragma unroll
            for (int b = 0; b < kProjBatch; b++) v[b] = col[(l + b) * sp];
        }
#pragma unroll
        for (int b = 0; b < kProjBatch; b++) {
            const T *u = sU + (l + b) * r;
            T s = tr_zero<T>();
#pragma unroll
            for (int t = 0; t < RMAX; t++)
                if (t < r) tr_mac(s, u[t], w[t]);
            oc[(l + b) * sp] = subtract ? tr_axpy(v[b], minus, s) : s;
        }
    }
    for (; l < l1; l++) {
        const T *u = sU + l * r;
        T s = tr_zero<T>();
#pragma unroll
        for (int t = 0; t < RMAX; t++)
            if (t < r) tr_mac(s, u[t], w[t]);
        oc[l * sp] = subtract ? tr_axpy(col[l * sp], minus, s) : s;
    }
}

// The same pass for FP32 with unit column stride (A = x's rows), q a
// multiple of 4 and x, out and the row stride 16-byte aligned: a lane takes
// four adjacent columns and reads each row's four values as one 16-byte load
// (a warp's row read is 512 bytes), and a warp's ragged last batch of rows
// is read together with the rest of its batch, under a predicate.  Per
// column the operations and their order are those of the kernel above.
__device__ __forceinline__ void mac4(float4 &c, float a, const float4 &b) {
    c.x = fmaf(a, b.x, c.x); c.y = fmaf(a, b.y, c.y); c.z = fmaf(a, b.z, c.z); c.w = fmaf(a, b.w, c.w);
}

template <int RMAX>
__global__ void __launch_bounds__(32 * kProjMaxGroups) tr_project_small4_kernel(
    const float *x, int64_t sp, int64_t p, int64_t q, const float *__restrict__ U, int r, int subtract,
    float *out, const int *gate) {
    if (gate && *gate != 1) return;
    constexpr int B = RMAX <= 8 ? 8 : 4;   // rows a warp reads at once
    extern __shared__ __align__(16) unsigned char tr_smem[];
    float *sU = reinterpret_cast<float *>(tr_smem);                                 // p x r
    float4 *red = reinterpret_cast<float4 *>(sU + ((p * r + 3) & ~int64_t(3)));     // [groups][r][32]
    const int groups = blockDim.x >> 5, g = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int64_t e = threadIdx.x; e < p * r; e += blockDim.x) sU[e] = U[e];
    __syncthreads();
    const int64_t j = ((int64_t)blockIdx.x * 32 + lane) * 4;
    const bool ok = j < q;
    const int64_t rows = (p + groups - 1) / groups;
    const int64_t l0 = min(p, g * rows), l1 = min(p, l0 + rows);
    const float *col = x + (ok ? j : 0);
    float4 w[RMAX];
#pragma unroll
    for (int t = 0; t < RMAX; t++) w[t] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ok) {
        for (int64_t l = l0; l < l1; l += B) {
            float4 v[B];
#pragma unroll
            for (int b = 0; b < B; b++)
                if (l + b < l1) v[b] = *reinterpret_cast<const float4 *>(col + (l + b) * sp);
#pragma unroll
            for (int b = 0; b < B; b++) {
                if (l + b >= l1) continue;
                const float *u = sU + (l + b) * r;
#pragma unroll
                for (int t = 0; t < RMAX; t++)
                    if (t < r) mac4(w[t], u[t], v[b]);
            }
        }
    }
#pragma unroll
    for (int t = 0; t < RMAX; t++)
        if (t < r) red[((int64_t)g * r + t) * 32 + lane] = w[t];
    __syncthreads();
    if (!ok) return;
#pragma unroll
    for (int t = 0; t < RMAX; t++) {
        if (t >= r) continue;
        float4 s4 = red[(int64_t)t * 32 + lane];
        for (int k = 1; k < groups; k++) {
            const float4 c = red[((int64_t)k * r + t) * 32 + lane];
            s4.x = fmaf(1.f, c.x, s4.x); s4.y = fmaf(1.f, c.y, s4.y);
            s4.z = fmaf(1.f, c.z, s4.z); s4.w = fmaf(1.f, c.w, s4.w);
        }
        w[t] = s4;
    }
    float *oc = out + j;
    for (int64_t l = l0; l < l1; l += B) {
        float4 v[B];
        if (subtract) {
#pragma unroll
            for (int b = 0; b < B; b++)
                if (l + b < l1) v[b] = *reinterpret_cast<const float4 *>(col + (l + b) * sp);
        }
#pragma unroll
        for (int b = 0; b < B; b++) {
            if (l + b >= l1) continue;
            const float *u = sU + (l + b) * r;
            float4 s4 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int t = 0; t < RMAX; t++)
                if (t < r) {
                    s4.x = fmaf(u[t], w[t].x, s4.x); s4.y = fmaf(u[t], w[t].y, s4.y);
                    s4.z = fmaf(u[t], w[t].z, s4.z); s4.w = fmaf(u[t], w[t].w, s4.w);
                }
            float4 o = s4;
            if (subtract)
                o = make_float4(fmaf(-1.f, s4.x, v[b].x), fmaf(-1.f, s4.y, v[b].y), fmaf(-1.f, s4.z, v[b].z),
                                fmaf(-1.f, s4.w, v[b].w));
            *reinterpret_cast<float4 *>(oc + (l + b) * sp) = o;
        }
    }
}

// Row groups (warps) per CTA of the one-pass projection: at least 32 rows
// per warp (fewer leaves each warp too little work for the basis load and
// the barrier), at most 8, and shared memory (basis + partials) within the
// static limit; 0 when even one group does not fit.
template <typename T>
int small_groups(int64_t p, int r) {
    if (r > 32) return 0;
    int g = 1;
    while (g < kProjMaxGroups && (int64_t)(2 * g) * 32 <= p) g *= 2;
    for (; g >= 1; g /= 2)
        if ((size_t)(p * r + (int64_t)g * r * 32) * sizeof(T) <= kSmallBasisSmem) return g;
    return 0;
}

// ------------------------------------------------- leading subspace (fast)

// Double-precision helpers for the subspace iteration (real: double,
// complex: double2).
__device__ __forceinline__ double oi_conj(double a) { return a; }
__device__ __forceinline__ double2 oi_conj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double oi_mul(double a, double b) { return a * b; }
__device__ __forceinline__ double2 oi_mul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double oi_add(double a, double b) { return a + b; }
__device__ __forceinline__ double2 oi_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double oi_sub(double a, double b) { return a - b; }
__device__ __forceinline__ double2 oi_sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double oi_scale(double a, double s) { return a * s; }
__device__ __forceinline__ double2 oi_scale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double oi_abs2(double a) { return a * a; }
__device__ __forceinline__ double oi_abs2(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double oi_re(double a) { return a; }
__device__ __forceinline__ double oi_re(double2 a) { return a.x; }
__device__ __forceinline__ double oi_shfl(double a, int o) { return __shfl_xor_sync(0xffffffffu, a, o); }
__device__ __forceinline__ double2 oi_shfl(double2 a, int o) {
    return make_double2(__shfl_xor_sync(0xffffffffu, a.x, o), __shfl_xor_sync(0xffffffffu, a.y, o));
}
__device__ __forceinline__ double oi_from(float a) { return a; }
__device__ __forceinline__ double oi_from(double a) { return a; }
__device__ __forceinline__ double2 oi_from(float2 a) { return make_double2(a.x, a.y); }
__device__ __forceinline__ double2 oi_from(double2 a) { return a; }
__device__ __forceinline__ void oi_to(float &o, double a) { o = (float)a; }
__device__ __forceinline__ void oi_to(double &o, double a) { o = a; }
__device__ __forceinline__ void oi_to(float2 &o, double2 a) { o = make_float2((float)a.x, (float)a.y); }
__device__ __forceinline__ void oi_to(double2 &o, double2 a) { o = a; }
template <typename A> __device__ __forceinline__ A oi_real(double v);
template <> __device__ __forceinline__ double oi_real<double>(double v) { return v; }
template <> __device__ __forceinline__ double2 oi_real<double2>(double v) { return make_double2(v, 0.0); }
template <typename A> __device__ __forceinline__ A oi_zero();
template <> __device__ __forceinline__ double oi_zero<double>() { return 0.0; }
template <> __device__ __forceinline__ double2 oi_zero<double2>() { return make_double2(0.0, 0.0); }
// deterministic start vectors in [-1, 1)
__device__ __forceinline__ double oi_hash(uint32_t k) {
    k ^= k >> 16; k *= 0x7feb352du; k ^= k >> 15; k *= 0x846ca68bu; k ^= k >> 16;
    return (double)k * (2.0 / 4294967296.0) - 1.0;
}
__device__ __forceinline__ void oi_start(double &a, uint32_t k) { a = oi_hash(2 * k + 1); }
__device__ __forceinline__ void oi_start(double2 &a, uint32_t k) { a = make_double2(oi_hash(2 * k + 1), oi_hash(2 * k + 2)); }

// eigen route of the last call, reported through ffdas_get_last_kernel_info
// (variant): device orthogonal iteration, cuSOLVER syevd, syevdx over one
// index range, or keep-all copy
constexpr int kRouteSubspace = 10, kRouteSyevd = 11, kRouteSyevdx = 12, kRouteCopy = 13;

constexpr int kOiThreads = 512;
constexpr int kOiMaxRank = 16;
constexpr int kOiMaxIter = 30;
constexpr int kOiMaxSlices = 8;
// residual bound relative to the largest Rayleigh quotient: 2 eps for FP32
// data, about 45 eps for FP64 (the rounding floor of G Q in double)
template <typename T> constexpr double oi_tol() { return sizeof(typename tr_elem<T>::real) == 4 ? 2.4e-7 : 1e-14; }

// (a, b), a <= b, of the e-th entry of an r x r upper triangle, row by row
__device__ __forceinline__ void oi_upper(int e, int r, int &a, int &b) {
    a = 0;
    while (e >= r - a && a < r) e -= r - a, a++;
    b = a + e;
}

// Hermitian products of p x r row-major matrices, M = X^H Z, and M2 =
// X2^H Z2 when X2 is given (the products this iteration forms are Q^H Y,
// Y^H Y and Q^H Q, Hermitian in exact arithmetic): the upper triangles, one
// warp per entry, lanes over rows and a shuffle sum, mirrored into the lower
// triangles.  Ends with a barrier.
template <typename A>
__device__ void oi_hermitian(const A *X, const A *Z, A *M, const A *X2, const A *Z2, A *M2, int p, int r) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int ne = r * (r + 1) / 2, total = X2 ? 2 * ne : ne;
    for (int e = warp; e < total; e += nw) {
        const bool second = e >= ne;
        const A *x = second ? X2 : X;
        const A *z = second ? Z2 : Z;
        A *m = second ? M2 : M;
        int a, b;
        oi_upper(second ? e - ne : e, r, a, b);
        A s = oi_zero<A>();
        for (int i = lane; i < p; i += 32) s = oi_add(s, oi_mul(oi_conj(x[i * r + a]), z[i * r + b]));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s = oi_add(s, oi_shfl(s, o));
        if (lane == 0) {
            m[a * r + b] = s;
            if (a != b) m[b * r + a] = oi_conj(s);
        }
    }
    __syncthreads();
}

// Cholesky factor of the r x r Hermitian C (full storage), C = L L^H, in
// place (L in the lower triangle), by one warp: per column the pivot, then
// a lane per row of the trailing lower triangle.  With `cs`, of
// D C D for D = diag(C)^-1/2 (the Gram matrix of the columns scaled to unit
// norm; a zero column keeps scale 1), the scales stored to cs.  1 / L[j][j]
// goes to invd; *flag = 0 when a pivot is not positive.  Called by warp 0.
template <typename A>
__device__ void oi_cholesky_warp(A *C, int r, double *invd, double *cs, int *flag) {
    const int lane = threadIdx.x & 31;
    if (cs) {
        if (lane < r) {
            const double n2 = oi_re(C[lane * r + lane]);
            cs[lane] = n2 > 0.0 ? rsqrt(n2) : 1.0;
        }
        __syncwarp();
        if (lane < r)
            for (int k = 0; k < r; k++) C[lane * r + k] = oi_scale(C[lane * r + k], cs[lane] * cs[k]);
        __syncwarp();
    }
    int ok = 1;
    for (int j = 0; j < r; j++) {
        const double d = oi_re(C[j * r + j]);
        if (!(d > 0.0)) {
            ok = 0;
            break;
        }
        const double inv = rsqrt(d);
        if (lane == j) C[j * r + j] = oi_real<A>(d * inv);
        else if (lane > j && lane < r) C[lane * r + j] = oi_scale(C[lane * r + j], inv);
        if (lane == 0) invd[j] = inv;
        __syncwarp();
        if (lane > j && lane < r) {   // row `lane` of the trailing lower triangle
            const A lij = C[lane * r + j];
            for (int k = j + 1; k <= lane; k++)
                C[lane * r + k] = oi_sub(C[lane * r + k], oi_mul(lij, oi_conj(C[k * r + j])));
        }
        __syncwarp();
    }
    if (lane == 0) *flag = ok;
}

// Rows of Q = (Y D) L^-H (D = diag(cs), or none): per row the forward
// substitution z_b = ((y D)_b - sum_{a<b} z_a conj(L[b][a])) / L[b][b], in
// registers.  Y and Q may be the same array.
template <typename A, int RM>
__device__ void oi_solve_rows(const A *Y, A *Q, int p, int r, const A *Lm, const double *invd, const double *cs) {
    for (int i = threadIdx.x; i < p; i += blockDim.x) {
        A z[RM];
#pragma unroll
        for (int b = 0; b < RM; b++) {
            if (b >= r) break;
            A v = Y[i * r + b];
            if (cs) v = oi_scale(v, cs[b]);
#pragma unroll
            for (int a = 0; a < b; a++) v = oi_sub(v, oi_mul(z[a], oi_conj(Lm[b * r + a])));
            z[b] = oi_scale(v, invd[b]);
        }
#pragma unroll
        for (int b = 0; b < RM; b++)
            if (b < r) Q[i * r + b] = z[b];
    }
}

// shared memory the subspace kernel addresses past G
template <typename A>
struct oi_layout {
    A *Q, *Y, *H, *C, *P;
    double *red, *invd, *cs;
    __device__ oi_layout(unsigned char *base, int p, int r, int ks) {
        Q = reinterpret_cast<A *>(base);
        Y = Q + p * r;
        H = Y + p * r;
        C = H + r * r;
        P = C + r * r;
        red = reinterpret_cast<double *>(P + (ks - 1) * p * r);
        invd = red + 32;
        cs = invd + kOiMaxRank;
    }
};

// Q <- an orthonormal basis of span(Y), given C = Y^H Y: Cholesky QR of the
// unit-norm columns, then once more on the result unless Q^H Q is already
// within `orth` of the identity in every entry (the second pass restores
// orthogonality to rounding; one pass loses about cond(Y)^2 eps).  False (on
// every thread) when a pivot is not positive.
template <typename A, int RM>
__device__ bool oi_orthonormalize(const oi_layout<A> &s, int p, int r, int *flag, double orth) {
    const int warp = threadIdx.x >> 5;
    if (warp == 0) oi_cholesky_warp<A>(s.C, r, s.invd, s.cs, flag);
    __syncthreads();
    if (!*flag) return false;
    oi_solve_rows<A, RM>(s.Y, s.Q, p, r, s.C, s.invd, s.cs);
    __syncthreads();
    oi_hermitian<A>(s.Q, s.Q, s.C, nullptr, nullptr, nullptr, p, r);
    double dev2 = 0.0;   // largest squared deviation from I
    for (int a = 0; a < r; a++)
        for (int b = 0; b < r; b++) {
            const A c = s.C[a * r + b];
            dev2 = fmax(dev2, oi_abs2(a == b ? oi_sub(c, oi_real<A>(1.0)) : c));
        }
    if (dev2 <= orth * orth) return true;
    if (warp == 0) oi_cholesky_warp<A>(s.C, r, s.invd, nullptr, flag);
    __syncthreads();
    if (!*flag) return false;
    oi_solve_rows<A, RM>(s.Q, s.Q, p, r, s.C, s.invd, nullptr);
    __syncthreads();
    return true;
}

// Asynchronous copy of G's p columns (p elements each) into shared memory
// with leading dimension ld, issued before the start basis is built and
// waited for before the first product: 16-byte pieces when the column and
// ld byte sizes allow, else one element per copy (4, 8 or 16 bytes).
template <int BYTES>
__device__ __forceinline__ void oi_cp_async(uint32_t dst, const char *src) {
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(dst), "l"(src), "n"(BYTES) : "memory");
}
template <typename T>
__device__ void oi_copy_async(unsigned char *dst, const T *G, int p, int ld) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    const char *g = reinterpret_cast<const char *>(G);
    // (the copy fits shared memory: every offset fits 32 bits)
    const uint32_t col = (uint32_t)p * sizeof(T), dcol = (uint32_t)ld * sizeof(T);
    if (col % 16 == 0 && dcol % 16 == 0) {
        const uint32_t per = col / 16;
        for (uint32_t e = threadIdx.x; e < per * (uint32_t)p; e += blockDim.x) {
            const uint32_t k = e / per, o = (e - k * per) * 16;
            oi_cp_async<16>(d + k * dcol + o, g + (size_t)k * col + o);
        }
    } else {
        for (uint32_t e = threadIdx.x; e < (uint32_t)(p * p); e += blockDim.x) {
            const uint32_t k = e / (uint32_t)p, o = (e - k * (uint32_t)p) * (uint32_t)sizeof(T);
            oi_cp_async<sizeof(T)>(d + k * dcol + o, g + (size_t)k * col + o);
        }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void oi_copy_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Y = G Q for real data on the FP64 tensor cores (mma.m8n8k4 .f64; each of
// its products and sums is an FP64 operation).  A task is an 8-row tile of
// Y, an 8-column tile of Q and one of `parts` ranges of the inner dimension
// (steps of 4); a warp runs up to kOiTasks tasks at once, so that their
// fragment loads and products overlap (the product's latency is about six
// times its issue interval).  Part 0 goes to Y, part k to P + (k-1) p r.
// Fragments (PTX ISA, mma.m8n8k4 .f64): lane l holds A[l/4][l%4],
// B[l%4][l/4] and D[l/4][2(l%4) + 0..1].  G column-major with leading
// dimension ld; Q, Y row-major p x r.
constexpr int kOiTasks = 4;
template <typename T>
__device__ void oi_gq_dmma(const T *G, int ld, const double *Q, double *Y, double *P, int p, int r, int parts) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int mt = (p + 7) / 8, tiles = mt * ((r + 7) / 8), kt = (p + 3) / 4, steps = (kt + parts - 1) / parts;
    const int tasks = tiles * parts;
    const int g = lane >> 2, t4 = lane & 3;
    for (int base = 0; base < tasks; base += kOiTasks * nw) {
        int row[kOiTasks], col[kOiTasks], k0[kOiTasks], part[kOiTasks];
        bool on[kOiTasks];
#pragma unroll
        for (int u = 0; u < kOiTasks; u++) {
            const int task = base + warp + u * nw;
            on[u] = task < tasks;
            const int tile = on[u] ? task % tiles : 0;
            part[u] = on[u] ? task / tiles : 0;
            row[u] = (tile % mt) * 8;
            col[u] = (tile / mt) * 8;
            k0[u] = part[u] * steps * 4 + t4;
        }
        double c0[kOiTasks], c1[kOiTasks];
#pragma unroll
        for (int u = 0; u < kOiTasks; u++) c0[u] = c1[u] = 0.0;
        // every slot multiplies (an idle one zeros): no branch around the
        // warp-wide instruction
        for (int s = 0; s < steps; s++) {
            double a[kOiTasks], b[kOiTasks];
#pragma unroll
            for (int u = 0; u < kOiTasks; u++) {
                const int k = k0[u] + 4 * s, i = row[u] + g, n = col[u] + g;
                a[u] = on[u] && i < p && k < p ? oi_from(G[i + (int64_t)k * ld]) : 0.0;
                b[u] = on[u] && n < r && k < p ? Q[k * r + n] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kOiTasks; u++)
                asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                    : "+d"(c0[u]), "+d"(c1[u]) : "d"(a[u]), "d"(b[u]));
        }
#pragma unroll
        for (int u = 0; u < kOiTasks; u++) {
            if (!on[u]) continue;
            double *dst = part[u] == 0 ? Y : P + (int64_t)(part[u] - 1) * p * r;
            const int i = row[u] + g, n = col[u] + 2 * t4;
            if (i < p && n < r) dst[i * r + n] = c0[u];
            if (i < p && n + 1 < r) dst[i * r + n + 1] = c1[u];
        }
    }
}

// Orthogonal iteration for the leading r-dimensional invariant subspace of
// the Hermitian p x p matrix G (column-major, both triangles), in double:
// Y = G Q, H = Q^H Y, stop when ||Y - Q H||_F <= tol * max_a H[a][a] (a
// backward-stable residual: the subspace is then as good as a dense
// eigensolver's for this G), else Q = orth(Y).  On convergence the basis is
// written as T (row-major p x r) and *status = 1; otherwise *status = 0 and
// the caller runs the dense eigensolver.  One CTA; every loop is bounded.
// g_ld > 0: G is copied into shared memory with that leading dimension
// (padded so that the tensor-core fragments' loads meet no bank conflicts).
// Real data: G Q on the FP64 tensor cores.  Complex data: G Q split over ks
// slices of its inner dimension, so that more threads than rows share the
// product (each G element is read and widened to double once per step).
template <typename T, int RM>
__global__ void __launch_bounds__(kOiThreads) tr_leading_subspace_kernel(const T *__restrict__ G, int p, int r,
                                                                        int max_iter, double tol,
                                                                        T *__restrict__ basis,
                                                                        int *__restrict__ status, int g_ld,
                                                                        int ks) {
    using A = typename tr_elem<T>::acc;
    constexpr bool kReal = sizeof(A) == sizeof(double);
    extern __shared__ __align__(16) unsigned char oi_smem[];
    const size_t g_bytes = g_ld ? ((size_t)p * g_ld * sizeof(T) + 15) / 16 * 16 : 0;
    const oi_layout<A> s(oi_smem + g_bytes, p, r, ks);
    __shared__ int s_flag;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    if (tid == 0) *status = 0;
    const T *Gs = reinterpret_cast<const T *>(oi_smem);
    if (g_ld) oi_copy_async<T>(oi_smem, G, p, g_ld);
    for (int e = tid; e < p * r; e += nt) oi_start(s.Y[e], (uint32_t)e);
    __syncthreads();
    oi_hermitian<A>(s.Y, s.Y, s.C, nullptr, nullptr, nullptr, p, r);
    // one pass leaving Q^H Q within tol / 16 of I keeps the residual test and
    // the basis at the bound
    const double orth = tol / 16;
    const bool ok0 = oi_orthonormalize<A, RM>(s, p, r, &s_flag, orth);
    oi_copy_wait();
    __syncthreads();
    if (!ok0) return;
    const int len = (p + ks - 1) / ks;
    for (int it = 0; it < max_iter; it++) {
        if constexpr (kReal) {
            const double *Qd = reinterpret_cast<const double *>(s.Q);
            double *Yd = reinterpret_cast<double *>(s.Y), *Pd = reinterpret_cast<double *>(s.P);
            if (g_ld) oi_gq_dmma<T>(Gs, g_ld, Qd, Yd, Pd, p, r, ks);
            else oi_gq_dmma<T>(G, p, Qd, Yd, Pd, p, r, ks);
        } else {
            // Y = G Q: thread (slice, row i) sums its slice of l for all r
            // columns; consecutive threads take consecutive rows (coalesced G)
            const T *Gm = g_ld ? Gs : G;
            const int ld = g_ld ? g_ld : p;
            for (int t = tid; t < p * ks; t += nt) {
                const int sl = t / p, i = t - sl * p;
                const int l0 = min(p, sl * len), l1 = min(p, l0 + len);
                A acc[RM];
#pragma unroll
                for (int j = 0; j < RM; j++) acc[j] = oi_zero<A>();
                for (int l = l0; l < l1; l++) {
                    const A g = oi_from(Gm[i + (int64_t)l * ld]);
                    const A *qr = s.Q + l * r;
#pragma unroll
                    for (int j = 0; j < RM; j++)
                        if (j < r) acc[j] = oi_add(acc[j], oi_mul(g, qr[j]));
                }
                A *dst = sl == 0 ? s.Y : s.P + (sl - 1) * p * r;
#pragma unroll
                for (int j = 0; j < RM; j++)
                    if (j < r) dst[i * r + j] = acc[j];
            }
        }
        __syncthreads();
        if (ks > 1) {   // the parts in order
            for (int e = tid; e < p * r; e += nt) {
                A v = s.Y[e];
                for (int k = 1; k < ks; k++) v = oi_add(v, s.P[(k - 1) * p * r + e]);
                s.Y[e] = v;
            }
            __syncthreads();
        }
        // H = Q^H Y and C = Y^H Y together
        oi_hermitian<A>(s.Q, s.Y, s.H, s.Y, s.Y, s.C, p, r);
        // residual ||Y - Q H||_F^2: a row per thread, warp sums, then every
        // thread adds the warp sums in the same order (the same decision)
        double part = 0.0;
        for (int i = tid; i < p; i += nt) {
            A qi[RM];
#pragma unroll
            for (int a = 0; a < RM; a++) qi[a] = a < r ? s.Q[i * r + a] : oi_zero<A>();
#pragma unroll
            for (int b = 0; b < RM; b++) {
                if (b >= r) break;
                A v = s.Y[i * r + b];
#pragma unroll
                for (int a = 0; a < RM; a++)
                    if (a < r) v = oi_sub(v, oi_mul(qi[a], s.H[a * r + b]));
                part += oi_abs2(v);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (lane == 0) s.red[warp] = part;
        __syncthreads();
        double res2 = 0.0;
        for (int w = 0; w < nw; w++) res2 += s.red[w];
        double scale = 0.0;
        for (int a = 0; a < r; a++) scale = fmax(scale, oi_re(s.H[a * r + a]));
        if (sqrt(res2) <= tol * scale) {
            for (int e = tid; e < p * r; e += nt) oi_to(basis[e], s.Q[e]);
            if (tid == 0) *status = 1;
            return;
        }
        if (!oi_orthonormalize<A, RM>(s, p, r, &s_flag, orth)) return;
    }
}

// shared memory of the subspace kernel past G: Q, Y (p x r), H, C (r x r),
// ks - 1 slice partials (p x r), the warp sums, 1 / L[j][j] and the column
// scales
template <typename T>
size_t oi_smem_bytes(int64_t p, int r, int ks) {
    return (size_t)((2 + (int64_t)(ks - 1)) * p * r + 2 * (int64_t)r * r) * sizeof(typename tr_elem<T>::acc) +
           (32 + 2 * kOiMaxRank) * sizeof(double);
}

// ------------------------------------------------------------- cuSOLVER

struct solver_api {
    decltype(&cusolverDnCreate) create = nullptr;
    decltype(&cusolverDnDestroy) destroy = nullptr;
    decltype(&cusolverDnSetStream) set_stream = nullptr;
    decltype(&cusolverDnCreateParams) create_params = nullptr;
    decltype(&cusolverDnDestroyParams) destroy_params = nullptr;
    decltype(&cusolverDnXsyevd_bufferSize) buffer_size = nullptr;
    decltype(&cusolverDnXsyevd) syevd = nullptr;
    decltype(&cusolverDnXsyevdx_bufferSize) buffer_size_x = nullptr;   // optional
    decltype(&cusolverDnXsyevdx) syevdx = nullptr;                     // optional
    bool ok = false;
};

const solver_api &solver() {
    static const solver_api api = [] {
        solver_api s;
        void *lib = dlopen("libcusolver.so.11", RTLD_NOW | RTLD_LOCAL);
        if (!lib) lib = dlopen("libcusolver.so", RTLD_NOW | RTLD_LOCAL);
        if (!lib) return s;
        s.create = reinterpret_cast<decltype(s.create)>(dlsym(lib, "cusolverDnCreate"));
        s.destroy = reinterpret_cast<decltype(s.destroy)>(dlsym(lib, "cusolverDnDestroy"));
        s.set_stream = reinterpret_cast<decltype(s.set_stream)>(dlsym(lib, "cusolverDnSetStream"));
        s.create_params = reinterpret_cast<decltype(s.create_params)>(dlsym(lib, "cusolverDnCreateParams"));
        s.destroy_params = reinterpret_cast<decltype(s.destroy_params)>(dlsym(lib, "cusolverDnDestroyParams"));
        s.buffer_size = reinterpret_cast<decltype(s.buffer_size)>(dlsym(lib, "cusolverDnXsyevd_bufferSize"));
        s.syevd = reinterpret_cast<decltype(s.syevd)>(dlsym(lib, "cusolverDnXsyevd"));
        s.buffer_size_x = reinterpret_cast<decltype(s.buffer_size_x)>(dlsym(lib, "cusolverDnXsyevdx_bufferSize"));
        s.syevdx = reinterpret_cast<decltype(s.syevdx)>(dlsym(lib, "cusolverDnXsyevdx"));
        if (!s.buffer_size_x || !s.syevdx) s.buffer_size_x = nullptr, s.syevdx = nullptr;
        s.ok = s.create && s.destroy && s.set_stream && s.create_params && s.destroy_params && s.buffer_size &&
               s.syevd;
        return s;
    }();
    return api;
}

struct solver_state {
    cusolverDnHandle_t h = nullptr;
    cusolverDnParams_t params = nullptr;
};

void release_solver(void *p) {
    auto *s = static_cast<solver_state *>(p);
    if (solver().ok) {
        if (s->params) solver().destroy_params(s->params);
        if (s->h) solver().destroy(s->h);
    }
    delete s;
}

// The handle's solver state, created on first use (binds to the current
// device, which check_device has matched to the handle's).
ffdas_error_t get_solver(ffdas_context &ctx, solver_state **out) {
    if (!solver().ok) return FFDAS_ERROR_CUSOLVER;
    if (!ctx.solver) {
        auto *s = new solver_state;
        if (solver().create(&s->h) != CUSOLVER_STATUS_SUCCESS) {
            delete s;
            return FFDAS_ERROR_CUSOLVER;
        }
        if (solver().create_params(&s->params) != CUSOLVER_STATUS_SUCCESS) {
            solver().destroy(s->h);
            delete s;
            return FFDAS_ERROR_CUSOLVER;
        }
        ctx.solver = s;
        ctx.solver_release = release_solver;
    }
    *out = static_cast<solver_state *>(ctx.solver);
    return solver().set_stream((*out)->h, ctx.stream) == CUSOLVER_STATUS_SUCCESS ? FFDAS_SUCCESS
                                                                              : FFDAS_ERROR_CUSOLVER;
}

// ------------------------------------------------------------------ driver

// The subspace iteration for bases of up to RM vectors: G in shared memory
// when it fits the device's opt-in size less the kernel's static shared
// memory (leading dimension padded to 8 mod 32 elements where that fits),
// and for complex data as many slices of G Q (up to one thread per row and
// slice) as the threads and the shared memory allow.
template <typename T, int RM>
ffdas_error_t launch_subspace(ffdas_context &h, const T *G, int64_t p, int r, T *basis, int *status) {
    static const size_t static_smem = [] {
        cudaFuncAttributes fa{};
        const bool ok = cudaFuncGetAttributes(&fa, tr_leading_subspace_kernel<T, RM>) == cudaSuccess;
        cudaGetLastError();
        return ok ? fa.sharedSizeBytes : SIZE_MAX;
    }();
    constexpr bool real = sizeof(typename tr_elem<T>::acc) == sizeof(double);
    const size_t dyn_max = static_smem < h.smem_optin ? h.smem_optin - static_smem : 0;
    const auto g_bytes = [&](int64_t ld) { return ((size_t)(p * ld) * sizeof(T) + 15) / 16 * 16; };
    // complex: slices of rows' inner sums (one thread per row and slice);
    // real: parts of the tensor-core tasks' inner dimension, about three
    // tasks per warp and at most kOiTasks
    const int64_t warps = kOiThreads / 32, tiles = (p + 7) / 8 * ((r + 7) / 8);
    int ks = real ? (int)std::max<int64_t>(1, std::min<int64_t>({(3 * warps + tiles - 1) / tiles, kOiTasks * warps / tiles,
                                                                 (p + 3) / 4, (int64_t)kOiMaxSlices}))
                  : (int)std::max<int64_t>(1, std::min<int64_t>(kOiMaxSlices, kOiThreads / p));
    int g_ld = 0;
    const bool aligned = reinterpret_cast<uintptr_t>(G) % 16 == 0;
    for (int k = ks; k >= 1 && !g_ld && aligned; k--) {
        const int64_t padded = p + ((8 - p % 32) % 32 + 32) % 32;
        for (const int64_t ld : {padded, p})
            if (!g_ld && oi_smem_bytes<T>(p, r, k) + g_bytes(ld) <= dyn_max) g_ld = (int)ld, ks = k;
    }
    if (!g_ld)
        while (ks > 1 && oi_smem_bytes<T>(p, r, ks) > std::max(dyn_max, kSmallBasisSmem)) ks--;
    const size_t smem = oi_smem_bytes<T>(p, r, ks) + (g_ld ? g_bytes(g_ld) : 0);
    if (smem > kSmallBasisSmem &&
        ffdas_raise_smem_limit(reinterpret_cast<const void *>(tr_leading_subspace_kernel<T, RM>), h.device_id,
                               smem) != cudaSuccess)
        return FFDAS_ERROR_CUDA_RUNTIME;
    tr_leading_subspace_kernel<T, RM><<<1, kOiThreads, smem, h.stream>>>(G, (int)p, r, kOiMaxIter, oi_tol<T>(), basis,
                                                                        status, g_ld, ks);
    return ffdas_launch_check(h.stream);
}

constexpr size_t kGramPartialBytes = size_t(256) << 20;

// Row groups of the four-column FP32 pass (0: it does not apply): unit
// column stride, q and the row stride multiples of 4, x and out 16-byte
// aligned, and the basis and float4 partials of the one-column pass's group
// count within the static limit.  The group count sets the order of the
// sums, so it is never changed: aligned or not, the bits are the same.
template <typename T>
int small4_groups(const T *, int64_t, int64_t, int64_t, int64_t, int, int, const T *) { return 0; }
template <>
int small4_groups<float>(const float *x, int64_t sp, int64_t sq, int64_t p, int64_t q, int r, int groups,
                         const float *out) {
    if (sq != 1 || q % 4 != 0 || sp % 4 != 0 || reinterpret_cast<uintptr_t>(x) % 16 != 0 ||
        reinterpret_cast<uintptr_t>(out) % 16 != 0)
        return 0;
    const size_t smem = (size_t)(((p * r + 3) & ~int64_t(3)) + (int64_t)groups * r * 32 * 4) * sizeof(float);
    return smem <= kSmallBasisSmem ? groups : 0;
}

template <int RMAX, typename T>
ffdas_error_t launch_small4(ffdas_context &, const T *, int64_t, int64_t, int64_t, const T *, int, int, int, T *,
                            const int *) {
    return FFDAS_ERROR_INTERNAL;
}
template <int RMAX>
ffdas_error_t launch_small4(ffdas_context &h, const float *x, int64_t sp, int64_t p, int64_t q, const float *U, int r,
                            int groups, int subtract, float *out, const int *gate) {
    const int64_t blocks = (q / 4 + 31) / 32;
    if (blocks > INT32_MAX) return FFDAS_ERROR_DIMS_TOO_LARGE;
    const size_t smem = (size_t)(((p * r + 3) & ~int64_t(3)) + (int64_t)groups * r * 32 * 4) * sizeof(float);
    tr_project_small4_kernel<RMAX><<<(unsigned)blocks, 32 * groups, smem, h.stream>>>(x, sp, p, q, U, r, subtract,
                                                                                     out, gate);
    return ffdas_launch_check(h.stream);
}

template <typename T, int RMAX>
ffdas_error_t launch_small(ffdas_context &h, const T *x, int64_t sp, int64_t sq, int64_t p, int64_t q, const T *U,
                           int r, int groups, int subtract, T *out, const int *gate) {
    if (const int g4 = small4_groups<T>(x, sp, sq, p, q, r, groups, out))
        return launch_small4<RMAX>(h, x, sp, p, q, U, r, g4, subtract, out, gate);
    const int64_t blocks = (q + 31) / 32;
    if (blocks > INT32_MAX) return FFDAS_ERROR_DIMS_TOO_LARGE;
    const size_t smem = (size_t)(p * r + (int64_t)groups * r * 32) * sizeof(T);
    tr_project_small_kernel<T, RMAX><<<(unsigned)blocks, 32 * groups, smem, h.stream>>>(x, sp, sq, p, q, U, r,
                                                                                       subtract, out, gate);
    return ffdas_launch_check(h.stream);
}

// Tensor-core Gram (gram_tc.cuh): FP32 rows (A = x, m <= n) of at most 256,
// rows 16-byte aligned for the tensor map.  Engine 0 keeps small problems on
// the FMA kernel.
template <typename T>
bool gram_tc_usable(const ffdas_context &, const T *, bool, int64_t, int64_t, int64_t) { return false; }
template <>
bool gram_tc_usable<float>(const ffdas_context &h, const float *x, bool rows, int64_t p, int64_t q, int64_t n) {
    if (h.gram_engine == 1 || h.arch_code != 1000) return false;
    if (!rows || p < 1 || p > 256 || q < gram_tc::kChunk || q > INT32_MAX || n % 4 != 0) return false;
    if (reinterpret_cast<uintptr_t>(x) % 16 != 0) return false;
    if (h.gram_engine == 0 && p * q < (int64_t(1) << 20)) return false;
    return tensor_map_encoder() != nullptr;
}

template <int NB>
ffdas_error_t launch_gram_tc(ffdas_context &h, const CUtensorMap &map, const gram_tc::params &a, int64_t splits) {
    if (ffdas_raise_smem_limit(reinterpret_cast<const void *>(gram_tc::gram_tc_kernel<NB>), h.device_id,
                               gram_tc::smem_bytes<NB>()) != cudaSuccess)
        return FFDAS_ERROR_CUDA_RUNTIME;
    gram_tc::gram_tc_kernel<NB><<<(unsigned)splits, gram_tc::kThreads, gram_tc::smem_bytes<NB>(), h.stream>>>(map, a);
    return ffdas_launch_check(h.stream);
}

// Partials of G = A A^T over `splits` column ranges, about one CTA per SM;
// `ok` false when the tensor map cannot be encoded (the caller then uses the
// FMA kernel).
ffdas_error_t gram_tc_partials(ffdas_context &h, const float *x, int64_t p, int64_t q, int64_t n, workspace &part,
                               int64_t &splits, bool &ok) {
    using namespace gram_tc;
    ok = false;
    splits = std::min<int64_t>(h.sm_count, (q + kChunk - 1) / kChunk);
    int64_t kchunk = (q + splits - 1) / splits;
    kchunk = (kchunk + kChunk - 1) / kChunk * kChunk;
    splits = (q + kchunk - 1) / kchunk;
    const int NB = p > 128 ? 2 : 1;
    CUtensorMap map;
    const cuuint64_t dims[2] = {(cuuint64_t)q, (cuuint64_t)p};
    const cuuint64_t strides[1] = {(cuuint64_t)n * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)kChunk, (cuuint32_t)(128 * NB)};
    const cuuint32_t estr[2] = {1u, 1u};
    if (tensor_map_encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(x), dims, strides, box,
                             estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return FFDAS_SUCCESS;
    ok = true;
    FFDAS_TRY(part.alloc((size_t)(splits * p * p) * sizeof(float)));
    params a{};
    a.p = (int)p;
    a.q = q;
    a.kchunk = kchunk;
    const auto up16 = [](int64_t v) { return (int)((v + 15) / 16 * 16); };
    a.n0 = up16(p);
    a.n1 = NB == 2 ? up16(p - 128) : 16;
    a.part = part.get<float>();
    a.status = h.status;
    return NB == 2 ? launch_gram_tc<2>(h, map, a, splits) : launch_gram_tc<1>(h, map, a, splits);
}

template <typename T>
ffdas_error_t launch_gemm(ffdas_context &h, const tr_gemm_args<T> &a, int splits) {
    const int64_t gx = (a.N + kTrTile - 1) / kTrTile, gy = (a.M + kTrTile - 1) / kTrTile;
    if (gx > INT32_MAX || gy > 65535) return FFDAS_ERROR_DIMS_TOO_LARGE;
    tr_gemm_kernel<T><<<dim3((unsigned)gx, (unsigned)gy, (unsigned)splits), kTrThreads, 0, h.stream>>>(a);
    return ffdas_launch_check(h.stream);
}

// out = U (U^H A), or A - U (U^H A) when subtract: the one-pass kernel for
// bases of up to 32 vectors, else two tiled products through a (r, q)
// workspace.  gate (one-pass kernel only): a device flag; the kernel writes
// nothing unless it reads 1 (the subspace iteration's convergence status).
template <typename T>
bool project_takes_gate(int64_t p, int r) { return small_groups<T>(p, r) > 0; }

template <typename T>
ffdas_error_t project(ffdas_context &h, const T *x, int64_t sp, int64_t sq, int64_t p, int64_t q, const T *U, int r,
                      int subtract, T *out, const int *gate = nullptr) {
    using real = typename tr_elem<T>::real;
    const int groups = small_groups<T>(p, r);
    if (groups > 0) {
        if (r <= 4) FFDAS_TRY((launch_small<T, 4>(h, x, sp, sq, p, q, U, r, groups, subtract, out, gate)));
        else if (r <= 8) FFDAS_TRY((launch_small<T, 8>(h, x, sp, sq, p, q, U, r, groups, subtract, out, gate)));
        else if (r <= 16) FFDAS_TRY((launch_small<T, 16>(h, x, sp, sq, p, q, U, r, groups, subtract, out, gate)));
        else FFDAS_TRY((launch_small<T, 32>(h, x, sp, sq, p, q, U, r, groups, subtract, out, gate)));
    } else {
        workspace wbuf(h);
        FFDAS_TRY(wbuf.alloc((size_t)r * (size_t)q * sizeof(T)));
        tr_gemm_args<T> w{};          // W = U^H A  (r x q)
        w.L = U; w.li = 1; w.lk = r; w.conj_l = 1;
        w.R = x; w.rk = sp; w.rj = sq;
        w.C = wbuf.get<T>(); w.ci = q; w.cj = 1;
        w.M = r; w.N = q; w.K = p; w.kchunk = (p + kTrTileK - 1) / kTrTileK * kTrTileK; w.sign = 1;
        FFDAS_TRY(launch_gemm(h, w, 1));
        tr_gemm_args<T> o{};          // out = U W, or A - U W
        o.L = U; o.li = r; o.lk = 1;
        o.R = wbuf.get<T>(); o.rk = q; o.rj = 1;
        o.C = out; o.ci = sp; o.cj = sq;
        o.base = subtract ? x : nullptr; o.sign = subtract ? (real)-1 : (real)1;
        o.M = p; o.N = q; o.K = r; o.kchunk = ((int64_t)r + kTrTileK - 1) / kTrTileK * kTrTileK;
        FFDAS_TRY(launch_gemm(h, o, 1));
    }

    return FFDAS_SUCCESS;
}

template <typename T>
ffdas_error_t truncate_rank_t(ffdas_context &h, int64_t m, int64_t n, const T *x, T *out, int64_t start,
                              int64_t stop) {
    using real = typename tr_elem<T>::real;
    // A = x (p = m) when m <= n, else x^T (p = n): truncate_rank_impl.cuh:451-453
    const bool rows = m <= n;
    const int64_t p = rows ? m : n, q = rows ? n : m;
    const int64_t sp = rows ? n : 1, sq = rows ? 1 : n;
    const int64_t keep = stop - start, drop = p - keep;
    h.last = ffdas_kernel_info_t{};
    h.last.variant = kRouteCopy;
    if (drop == 0) {
        if (out != x) FFDAS_CUDA(cudaMemcpyAsync(out, x, (size_t)(m * n) * sizeof(T), cudaMemcpyDeviceToDevice,
                                                 h.stream));
        return FFDAS_SUCCESS;
    }

    // 1. Gram matrix split over q: on the tensor cores (FP32 rows up to 256),
    // else the FMA kernel over the upper tiles
    workspace part(h), gram(h), eig(h), info(h);
    int64_t splits = 0, gram_grid = 0;
    bool tensor = false;
    if (gram_tc_usable<T>(h, x, rows, p, q, n)) {
        FFDAS_TRY(gram_tc_partials(h, reinterpret_cast<const float *>(x), p, q, n, part, splits, tensor));
        gram_grid = splits;
    }
    if (!tensor) {
        const int64_t tiles = (p + kTrTile - 1) / kTrTile;
        const int64_t tri = tiles * (tiles + 1) / 2;
        // one wave: as many CTAs as the SMs hold at this kernel's occupancy
        int per_sm = 0;
        FFDAS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tr_gemm_kernel<T>, kTrThreads, 0));
        splits = std::max<int64_t>(1, (int64_t)std::max(per_sm, 1) * h.sm_count / tri);
        splits = std::max<int64_t>(1, std::min<int64_t>(splits, (q + kTrTileK - 1) / kTrTileK));
        splits = std::max<int64_t>(1, std::min<int64_t>(splits, (int64_t)(kGramPartialBytes / ((size_t)p * p * sizeof(T)))));
        splits = std::min<int64_t>(splits, 65535);
        int64_t kchunk = (q + splits - 1) / splits;
        kchunk = (kchunk + kTrTileK - 1) / kTrTileK * kTrTileK;
        splits = (q + kchunk - 1) / kchunk;
        FFDAS_TRY(part.alloc((size_t)(splits * p * p) * sizeof(T)));
        tr_gemm_args<T> g{};
        g.L = x; g.li = sp; g.lk = sq;
        g.R = x; g.rk = sq; g.rj = sp; g.conj_r = 1;
        g.C = part.get<T>(); g.ci = p; g.cj = 1; g.zstride = p * p;
        g.M = p; g.N = p; g.K = q; g.kchunk = kchunk; g.upper = 1; g.sign = 1;
        FFDAS_TRY(launch_gemm(h, g, (int)splits));
        gram_grid = tiles * tiles * splits;
    }
    FFDAS_TRY(gram.alloc((size_t)(p * p) * sizeof(T)));
    FFDAS_TRY(eig.alloc((size_t)p * sizeof(real)));
    FFDAS_TRY(info.alloc(2 * sizeof(int)));   // solver status, subspace-iteration status
    h.last.copy_engine = tensor ? 2 : 1;
    {
        const int64_t blocks = (p * p + 31) / 32;
        if (blocks > INT32_MAX) return FFDAS_ERROR_DIMS_TOO_LARGE;
        tr_gram_reduce_kernel<T><<<(unsigned)blocks, 32 * kReduceWarps, 0, h.stream>>>(
            part.get<T>(), (int)splits, p, 1.0 / (double)q, tensor ? 1 : 0, gram.get<T>());
        FFDAS_TRY(ffdas_launch_check(h.stream));
    }

    // 3's basis, chosen first: the smaller of the kept and the removed sets;
    // eigenvector e = p-1-rank
    const bool direct = keep <= drop;
    const int r = (int)(direct ? keep : drop);
    int64_t e0 = direct ? p - stop : 0;
    int r0 = (int)(direct ? keep : p - stop);
    const int64_t e1 = p - start;
    // When the basis is one contiguous run of eigenvectors (always for the
    // kept set; for the removed set when start = 0 or stop = p, as in the
    // clutter filter), only those r are computed (syevdx, index range): the
    // back-transform then handles r vectors instead of p.  They come back in
    // columns 0..r-1.
    int64_t lo = -1;
    if (direct) lo = p - stop;
    else if (stop == p) lo = p - start;
    else if (start == 0) lo = 0;
    bool ranged = false;
    workspace basis(h);
    FFDAS_TRY(basis.alloc((size_t)(p * r) * sizeof(T)));

    // 2a. the basis is the leading subspace (kept ranks 0..stop-1, or removed
    // ranks 0..start-1 with stop = p: the clutter filter) and small: try the
    // orthogonal iteration first; the dense solver runs only if it does not
    // reach its residual bound
    const bool leading = direct ? start == 0 : stop == p;
    if (leading && r <= kOiMaxRank && oi_smem_bytes<T>(p, r, 1) <= kSmallBasisSmem) {
        if (r <= 4) FFDAS_TRY((launch_subspace<T, 4>(h, gram.get<T>(), p, r, basis.get<T>(), info.get<int>() + 1)));
        else if (r <= 8) FFDAS_TRY((launch_subspace<T, 8>(h, gram.get<T>(), p, r, basis.get<T>(), info.get<int>() + 1)));
        else FFDAS_TRY((launch_subspace<T, 16>(h, gram.get<T>(), p, r, basis.get<T>(), info.get<int>() + 1)));
        h.last.variant = kRouteSubspace;
        h.last.grid = gram_grid;
        h.last.kernels = 4;
        // the one-pass projection is queued behind the iteration and reads
        // its status on the device (no host round trip between them); the
        // host reads the status once, at the end, for the fallback
        const bool gated = project_takes_gate<T>(p, r);
        if (gated) FFDAS_TRY(project(h, x, sp, sq, p, q, basis.get<T>(), r, direct ? 0 : 1, out, info.get<int>() + 1));
        int converged = 0;
        FFDAS_CUDA(cudaMemcpyAsync(&converged, info.get<int>() + 1, sizeof(int), cudaMemcpyDeviceToHost, h.stream));
        FFDAS_CUDA(cudaStreamSynchronize(h.stream));
        if (converged == 1) {
            if (!gated) FFDAS_TRY(project(h, x, sp, sq, p, q, basis.get<T>(), r, direct ? 0 : 1, out));
            return FFDAS_SUCCESS;
        }
    }

    // 2. eigendecomposition (truncate_rank_impl.cuh:481-500, 68-90).
    // cuSOLVER is loaded here, at the first call that needs it; the device
    // iteration above does not.
    solver_state *sv = nullptr;
    FFDAS_TRY(get_solver(h, &sv));
    ranged = lo >= 0 && solver().syevdx != nullptr;
    size_t dev_bytes = 0, host_bytes = 0;
    real vl = 0, vu = 0;
    int64_t found = 0;
    cusolverStatus_t st;
    if (ranged)
        st = solver().buffer_size_x(sv->h, sv->params, CUSOLVER_EIG_MODE_VECTOR, CUSOLVER_EIG_RANGE_I,
                                    CUBLAS_FILL_MODE_UPPER, p, tr_elem<T>::cuda, gram.get<T>(), p, &vl, &vu, lo + 1,
                                    lo + r, &found, tr_elem<T>::cuda_real, eig.get<real>(), tr_elem<T>::cuda,
                                    &dev_bytes, &host_bytes);
    else
        st = solver().buffer_size(sv->h, sv->params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, p,
                                  tr_elem<T>::cuda, gram.get<T>(), p, tr_elem<T>::cuda_real, eig.get<real>(),
                                  tr_elem<T>::cuda, &dev_bytes, &host_bytes);
    if (st != CUSOLVER_STATUS_SUCCESS) return FFDAS_ERROR_CUSOLVER;
    // The reference allocates p times the reported device workspace (its
    // note: the size is underestimated on some architectures); the same
    // margin here, bounded for large p.
    size_t margin = (size_t)p * dev_bytes;
    if (dev_bytes && margin / dev_bytes != (size_t)p) margin = SIZE_MAX;
    const size_t cap = std::max<size_t>(size_t(1) << 30, 8 * dev_bytes);
    const size_t dev_alloc = std::max<size_t>(std::min(margin, cap), dev_bytes);
    workspace sdev(h);
    FFDAS_TRY(sdev.alloc(dev_alloc));
    std::vector<unsigned char> shost(std::max<size_t>(host_bytes, 1));
    if (ranged)
        st = solver().syevdx(sv->h, sv->params, CUSOLVER_EIG_MODE_VECTOR, CUSOLVER_EIG_RANGE_I,
                             CUBLAS_FILL_MODE_UPPER, p, tr_elem<T>::cuda, gram.get<T>(), p, &vl, &vu, lo + 1, lo + r,
                             &found, tr_elem<T>::cuda_real, eig.get<real>(), tr_elem<T>::cuda, sdev.get<void>(),
                             dev_bytes, shost.data(), host_bytes, info.get<int>());
    else
        st = solver().syevd(sv->h, sv->params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, p,
                            tr_elem<T>::cuda, gram.get<T>(), p, tr_elem<T>::cuda_real, eig.get<real>(),
                            tr_elem<T>::cuda, sdev.get<void>(), dev_bytes, shost.data(), host_bytes,
                            info.get<int>());
    if (st != CUSOLVER_STATUS_SUCCESS) return FFDAS_ERROR_CUSOLVER;
    h.last.variant = ranged ? kRouteSyevdx : kRouteSyevd;
    h.last.grid = gram_grid;
    h.last.kernels = 4;
    if (ranged) {
        e0 = 0;           // the r vectors sit in columns 0..r-1
        r0 = r;
    }

    // 3. projection
    {
        const int64_t blocks = (p * r + 255) / 256;
        tr_gather_basis_kernel<T><<<(unsigned)blocks, 256, 0, h.stream>>>(gram.get<T>(), p, r, e0, r0, e1,
                                                                          basis.get<T>());
        FFDAS_TRY(ffdas_launch_check(h.stream));
    }
    FFDAS_TRY(project(h, x, sp, sq, p, q, basis.get<T>(), r, direct ? 0 : 1, out));

    // The solver's status, read once everything is queued (the reference
    // reads it before the projection, truncate_rank_impl.cuh:92-97).
    int h_info = 0;
    FFDAS_CUDA(cudaMemcpyAsync(&h_info, info.get<int>(), sizeof(int), cudaMemcpyDeviceToHost, h.stream));
    FFDAS_CUDA(cudaStreamSynchronize(h.stream));
    if (ranged && found != r) return FFDAS_ERROR_CUSOLVER;
    return h_info == 0 ? FFDAS_SUCCESS : FFDAS_ERROR_CUSOLVER;
}

bool c_contiguous_2d(const ffdas_tensor_desc &d) {
    return (d.dims[1] <= 1 || d.strides[1] == 1) && (d.dims[0] <= 1 || d.strides[0] == d.dims[1]);
}

}  // namespace
}  // namespace ffdas

using namespace ffdas;

extern "C" ffdas_error_t ffdas_truncate_rank(ffdas_handle_t handle, ffdas_tensor_desc_t x_desc, const void *x,
                                             int64_t start, int64_t stop, ffdas_tensor_desc_t out_desc,
                                             void *out) {
    // validation order: truncate_rank.cu:15-26, truncate_rank_impl.cuh:432-443
    if (!handle) return FFDAS_ERROR_INVALID_HANDLE;
    if (!x_desc || !out_desc) return FFDAS_ERROR_NULL_POINTER;
    FFDAS_TRY(handle->check_device());
    const ffdas_tensor_desc &xd = *x_desc, &od = *out_desc;
    if (xd.dtype != od.dtype) return FFDAS_ERROR_UNSUPPORTED_TYPE;
    if (xd.dtype != FFDAS_R_32F && xd.dtype != FFDAS_C_32F && xd.dtype != FFDAS_R_64F && xd.dtype != FFDAS_C_64F)
        return FFDAS_ERROR_UNSUPPORTED_TYPE;
    if (xd.ndim != 2 || od.ndim != 2) return FFDAS_ERROR_INVALID_DIMS;
    if (xd.dims[0] != od.dims[0] || xd.dims[1] != od.dims[1]) return FFDAS_ERROR_INVALID_DIMS;
    if (xd.dims[0] > INT_MAX || xd.dims[1] > INT_MAX) return FFDAS_ERROR_INVALID_DIMS;
    if (!c_contiguous_2d(xd) || !c_contiguous_2d(od)) return FFDAS_ERROR_NON_CONTIGUOUS;
    const int64_t m = xd.dims[0], n = xd.dims[1];
    const int64_t p = std::min(m, n);
    if (start < 0 || start >= p || stop <= start || stop > p) return FFDAS_ERROR_INVALID_ARGUMENT;
    if (!x || !out) return FFDAS_ERROR_NULL_POINTER;
    ffdas_context &h = *handle;
    switch (xd.dtype) {
    case FFDAS_R_32F:
        return truncate_rank_t<float>(h, m, n, static_cast<const float *>(x), static_cast<float *>(out), start, stop);
    case FFDAS_R_64F:
        return truncate_rank_t<double>(h, m, n, static_cast<const double *>(x), static_cast<double *>(out), start,
                                       stop);
    case FFDAS_C_32F:
        return truncate_rank_t<float2>(h, m, n, static_cast<const float2 *>(x), static_cast<float2 *>(out), start,
                                       stop);
    default:
        return truncate_rank_t<double2>(h, m, n, static_cast<const double2 *>(x), static_cast<double2 *>(out),
                                        start, stop);
    }
}
