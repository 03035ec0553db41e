// FP32 launches of the factorised cubic H.v kernel for pencils of 320..576 threads (one CTA per
// multiprocessor); 576 threads with 3 states and 5 fast modes (the large benchmark system) get
// the pencil stride as a compile-time constant.
#include "hv_cubic_impl.h"

namespace nvb {

int cubic_launch_f32_wide(CubPlan &cp, const float *x, float *y, const double *scale, double *alpha_part,
                          cudaStream_t st) {
    if (cp.threads == 576 && cp.S == 3 && cp.nF == 5)
        return cubk::launch_c<float, 3, 5, 576, 608, 1>(cp, x, y, scale, alpha_part, st);
    return cubk::launch_shape<float, 0, 608, 1>(cp, x, y, scale, alpha_part, st);
}

}  // namespace nvb
