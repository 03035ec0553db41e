// FP64 launches of the factorised cubic H.v kernel (pencils of up to 288 threads, one CTA per
// multiprocessor).
#include "hv_cubic_impl.h"

namespace nvb {

int cubic_launch_f64(CubPlan &cp, const double *x, double *y, const double *scale, double *alpha_part, cudaStream_t st) {
    return cubk::launch_shape<double, 0, 320, 1>(cp, x, y, scale, alpha_part, st);
}

}  // namespace nvb
