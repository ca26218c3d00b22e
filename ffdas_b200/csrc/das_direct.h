// das_direct.h -- one-launch delay-and-sum for small real problems (das_direct.cu).
#pragma once
#include "core.h"
#include "das_problem.h"

namespace ffdas {

// Problems of at most this many units (voxels x channels x events x items)
// take the direct kernel when the planner chooses: single frames up to 2^25
// units (measured on B200: 15 us against 18-27 us staged for a 4.2e6-unit
// plane-wave frame, 39 us against 49 us at 2.7e7 units), batches up to 2^22
// (the staged batch tiles share each tap's delay over the items; the direct
// kernel only shares the geometry).
constexpr int64_t kDirectUnits = int64_t(1) << 25;
constexpr int64_t kDirectUnitsBatched = int64_t(1) << 22;

// Real channel data (f32, f16, bf16) into f32 output, dense.
bool direct_supported(const das_problem &pb, ffdas_datatype_t xt, ffdas_datatype_t ot, int kind);

ffdas_error_t launch_direct(ffdas_context &h, const das_problem &pb, ffdas_datatype_t xt, const void *x,
                            const float *srcpos, const float *srcdir, const float *dstpos, const float *offsets,
                            const float *weights, float *out, double beta, int beta_zero, int batch_tile,
                            int split_req);

}  // namespace ffdas
