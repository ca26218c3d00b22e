// das_problem.h -- problem description shared by the delay-and-sum entry points.
//
// Mirrors get_das_problem_params (src/das/das_utils.h:32-69): x is
// ([B,] C, S, N) with unit sample stride; out is ([B,] spatial...).  The
// spatial dims of out are collapsed into a (D2, D1, D0) grid that the tiled
// kernels walk.
#pragma once

#include <cstdint>
#include "core.h"

namespace ffdas {

struct das_problem {
    int B = 1, C = 0, S = 0, N = 0;
    bool have_batch = false;
    int64_t V = 0;
    int64_t x_bstride = 0, x_cstride = 0, x_sstride = 0;
    int64_t out_bstride = 0;
    int D0 = 1, D1 = 1, D2 = 1;
    int n_events = 0;      // S (dense) or sparse_count
    bool sparse = false;
};

struct das_call {
    const float *srcpos = nullptr;
    const float *srcdir = nullptr;
    float wavenum = 0.f;
    const ffdas_tensor_desc *x_desc = nullptr;
    const void *x = nullptr;
    const float *dstpos = nullptr;
    const float *offsets = nullptr;
    const float *weights = nullptr;
    int sparse_count = 0;
    const int *sparse_indices = nullptr;
    const void *beta = nullptr;
    const ffdas_tensor_desc *out_desc = nullptr;
    void *out = nullptr;
    ffdas_compute_type_t compute_type = FFDAS_COMPUTE_DEFAULT;
    ffdas_alg_t alg = FFDAS_ALG_DEFAULT;
    bool sparse = false;
};

// Largest element offset a descriptor can address fits in int32
// (reference: can_use_int32_indexing, src/core/tensor.cuh:99-107).
bool fits_int32_indexing(const ffdas_tensor_desc &d);

ffdas_error_t make_problem(const ffdas_tensor_desc &x, const ffdas_tensor_desc &out,
                           das_problem &p);

// Storage kind for a (x dtype, out dtype, compute type), or -1 if the
// combination is unsupported (FFDAS_ERROR_UNSUPPORTED_TYPE).
// batch: items in x (dims[0] of 4-D x, else 1); it picks the 16-bit data layout.
int select_storage(ffdas_datatype_t xt, ffdas_datatype_t ot, ffdas_compute_type_t ct, int batch);

ffdas_error_t das_forward(ffdas_context &h, const das_call &a);

// Pairs per row, rounded so every row starts 16-byte aligned for both pair
// sizes (the TMA tensor map needs 16-byte row strides).
inline int64_t pair_row_length(int N) {
    const int64_t n = (int64_t)N < 2 ? 2 : (int64_t)N;
    return (n + 3) & ~int64_t(3);
}

}  // namespace ffdas

#include "das_gather.cuh"

namespace ffdas {

bool staged_supported(const das_problem &pb, int kind);
// copy: 0 default, 1 TMA tile loads, 2 per-thread cp.async (also used when the
// driver's tensor-map encoder is unavailable).  Records it in h.last.
// Batch tiles need the TMA tensor-map encoder (3-D boxes).
bool staged_batch_supported();
// out = beta * out (or 0) for every item and voxel of an f32 image, before
// channel slices add into it.
ffdas_error_t launch_scale_image(ffdas_context &h, const das_problem &pb, float *out, float beta, int beta_zero);
// BT > 1: batch tiles of BT items per CTA (256-voxel tiles, SC * BT <= 32).
ffdas_error_t launch_staged(ffdas_context &h, const das_problem &pb, int kind, const gather_params &gp, int SC,
                            int WB, int BT, int copy, dim3 grid);

// Gradient outputs of the staged adjoint kernel (null = not computed).
struct staged_grads {
    const float *gout;
    int64_t gout_bstride;
    float *gx, *goff, *gw, *gdst, *gsrc;
};
// Complex (IQ) data on the staged kernel: 256-voxel tiles, 32-pair windows,
// TMA copies, event chunk 4 or 8.
ffdas_error_t launch_staged_cplx(ffdas_context &h, const das_problem &pb, int kind, const gather_params &gp,
                                 int SC, dim3 grid);
// das_sparse on the 512-voxel staged kernel: zeroes *gate, flags lists that
// name an event twice, then runs the kernel (which does nothing when flagged).
ffdas_error_t launch_staged_sparse(ffdas_context &h, const das_problem &pb, int kind, const gather_params &gp,
                                   int SC, int WB, int copy, dim3 grid, int *gate);
ffdas_error_t launch_staged_bwd(ffdas_context &h, const das_problem &pb, int kind, const gather_params &gp,
                                const staged_grads &gr, int SC, int WB, int BT, int copy, dim3 grid);

// das_sparse as one persistent launch over (tile, channel slice) work items,
// longest tiles first (csrc/das_sparse_items.cuh): real pair storage, f32
// output, lists of at most 64 entries.  gp holds 256-voxel tiles and the
// channel slice (cchunk); ws is sparse_items_workspace() bytes; *gate is
// zeroed, set for a list naming an event twice (the kernel then does nothing
// and the caller's gated gather kernel runs).
bool sparse_items_supported(const das_problem &pb, int kind);
size_t sparse_items_workspace(const das_problem &pb, int n_tiles, int SC);
ffdas_error_t launch_sparse_items(ffdas_context &h, const das_problem &pb, int kind, const gather_params &gp,
                                  int SC, int WB, int copy, void *ws, int *gate);

}  // namespace ffdas
