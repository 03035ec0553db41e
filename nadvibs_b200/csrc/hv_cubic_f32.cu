// FP32 launches of the factorised cubic H.v kernel: pencils of up to 288 threads (two CTAs per
// multiprocessor where shared memory allows); wider pencils go to hv_cubic_f32w.cu.
#include "hv_cubic_impl.h"

namespace nvb {

int cubic_launch_f32(CubPlan &cp, const float *x, float *y, const double *scale, double *alpha_part, cudaStream_t st) {
    if (cp.threads > 288) return cubic_launch_f32_wide(cp, x, y, scale, alpha_part, st);
    return cubk::launch_shape<float, 0, 320, 2>(cp, x, y, scale, alpha_part, st);
}

}  // namespace nvb
