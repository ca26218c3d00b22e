/*
 * das_oracle.c -- CPU restatement of ffdas delay-and-sum, for TESTS ONLY.
 *
 * This file is test infrastructure: the parity tests, the smoke check and the
 * CPU-baseline leg of bench.py call it as the checker.  No product code path
 * links or calls it.
 *
 * Two functions:
 *
 *   oracle_das_f64   FP64 restatement of the reference kernel das_alg1_kernel
 *                    (src/das/das_alg1_kernels.cuh:16-107 of BrainEchoLab/ffdas):
 *                      rsq  = max(|dst[v] - src[c]|^2, 1e-7)          (:60-64)
 *                      tau  = offsets[e,v] + sqrt(rsq)                 (:65-66)
 *                      k    = floor(tau), t = tau - k                  (das_device_utils.cuh:10-13)
 *                      valid iff 0 <= k < N-1                          (:70)
 *                            and, with srcdir, dot(d, n)/r > cos       (:72-76)
 *                      w    = weights[e,v]            real             (:88)
 *                           = weights[e,v]*exp(i*wavenum*tau) complex  (:81-86)
 *                      acc += w * (x[k] + t*(x[k+1]-x[k]))             (:92-99, math/vector.cuh:15)
 *                      out  = acc  or  beta*out + acc                  (:103-106, das_device_utils.cuh:33-39)
 *                    with exact sqrt/sin/cos and double accumulation.
 *                    Sparse: event index e -> sparse_indices[i,v]       (:48-53)
 *                    Offsets/weights are indexed [e*V + v]; with q1 != 0 and
 *                    3-D x every event uses row 0, reproducing the reference's
 *                    outstride = 0 indexing (src/das/das_utils.h:64).
 *
 *   oracle_das_f32   The same formula as a plain FP32 OpenMP loop over voxels
 *                    (real data only).  This is the timed CPU baseline; its
 *                    loop order (voxel, event chunk, channel, event) matches
 *                    the GPU kernel's.
 *
 * Layouts: x is C-contiguous (B, C, S, N) doubles (complex: interleaved
 * re/im, (B, C, S, N, 2)); out is (B, V) (complex (B, V, 2)).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void oracle_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

void oracle_das_f64(int B, int C, int S, int N, int64_t V,
                    const double *x, int complex_data,
                    const float *srcpos, const float *srcdir, float wavenum,
                    const float *dstpos, const float *offsets, const float *weights,
                    int n_events, const int *sparse_indices, int q1,
                    double beta_re, double beta_im, double *out) {
    const int ncomp = complex_data ? 2 : 1;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t v = 0; v < V; v++) {
        const double vx = dstpos[3 * v], vy = dstpos[3 * v + 1], vz = dstpos[3 * v + 2];
        for (int b = 0; b < B; b++) {
            double acc_re = 0.0, acc_im = 0.0;
            for (int i = 0; i < n_events; i++) {
                const int64_t row = q1 ? 0 : i;
                const int64_t idx = row * V + v;
                int s = i;
                if (sparse_indices) {
                    s = sparse_indices[idx];
                    if (s < 0 || s >= S) continue;
                }
                const double ofs = offsets[idx];
                const double scl = weights[idx];
                for (int c = 0; c < C; c++) {
                    const double dx = vx - srcpos[3 * c];
                    const double dy = vy - srcpos[3 * c + 1];
                    const double dz = vz - srcpos[3 * c + 2];
                    double rsq = dx * dx + dy * dy + dz * dz;
                    if (rsq < 1e-7) rsq = 1e-7;
                    const double r = sqrt(rsq);
                    const double tau = ofs + r;
                    const double kf = floor(tau);
                    if (!(kf >= 0.0 && kf < (double)(N - 1))) continue;
                    if (srcdir) {
                        const float *d = srcdir + 4 * c;
                        const double proj = (dx * d[0] + dy * d[1] + dz * d[2]) / r;
                        if (!(proj > (double)d[3])) continue;
                    }
                    const int64_t k = (int64_t)kf;
                    const double t = tau - kf;
                    const double *xr = x + ((((int64_t)b * C + c) * S + s) * N) * ncomp;
                    if (!complex_data) {
                        const double x0 = xr[k], x1 = xr[k + 1];
                        acc_re += scl * (x0 + t * (x1 - x0));
                    } else {
                        const double x0r = xr[2 * k], x0i = xr[2 * k + 1];
                        const double x1r = xr[2 * k + 2], x1i = xr[2 * k + 3];
                        const double lr = x0r + t * (x1r - x0r);
                        const double li = x0i + t * (x1i - x0i);
                        const double ph = (double)wavenum * tau;
                        const double wr = scl * cos(ph), wi = scl * sin(ph);
                        acc_re += wr * lr - wi * li;
                        acc_im += wr * li + wi * lr;
                    }
                }
            }
            double *o = out + ((int64_t)b * V + v) * ncomp;
            if (!complex_data) {
                o[0] = beta_re * o[0] + acc_re;
            } else {
                const double orr = o[0], oi = o[1];
                o[0] = beta_re * orr - beta_im * oi + acc_re;
                o[1] = beta_re * oi + beta_im * orr + acc_im;
            }
        }
    }
}

/* FP32 CPU loop, real data, dense events, beta = 0.  x is (B, C, S, N)
 * float32.  Returns nothing; out is (B, V). */
void oracle_das_f32(int B, int C, int S, int N, int64_t V, const float *x,
                    const float *srcpos, const float *dstpos,
                    const float *offsets, const float *weights, float *out) {
    enum { EC = 16 };
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t v = 0; v < V; v++) {
        const float vx = dstpos[3 * v], vy = dstpos[3 * v + 1], vz = dstpos[3 * v + 2];
        for (int b = 0; b < B; b++) {
            float acc = 0.f;
            for (int e0 = 0; e0 < S; e0 += EC) {
                const int ec = (S - e0) < EC ? (S - e0) : EC;
                float ofs[EC], w[EC];
                for (int j = 0; j < ec; j++) {
                    ofs[j] = offsets[(int64_t)(e0 + j) * V + v];
                    w[j] = weights[(int64_t)(e0 + j) * V + v];
                }
                for (int c = 0; c < C; c++) {
                    const float dx = vx - srcpos[3 * c];
                    const float dy = vy - srcpos[3 * c + 1];
                    const float dz = vz - srcpos[3 * c + 2];
                    float rsq = dx * dx + dy * dy + dz * dz;
                    if (rsq < 1e-7f) rsq = 1e-7f;
                    const float r = sqrtf(rsq);
                    const float *xc = x + (((int64_t)b * C + c) * S + e0) * N;
                    for (int j = 0; j < ec; j++) {
                        const float tau = ofs[j] + r;
                        const float kf = floorf(tau);
                        if (kf >= 0.f && kf < (float)(N - 1)) {
                            const int k = (int)kf;
                            const float t = tau - kf;
                            const float *xr = xc + (int64_t)j * N;
                            acc += w[j] * (xr[k] + t * (xr[k + 1] - xr[k]));
                        }
                    }
                }
            }
            out[(int64_t)b * V + v] = acc;
        }
    }
}
