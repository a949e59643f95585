// diag.cu -- diagnostics entry points (no counterpart in the reference):
// element-wise access to the library's double-double math so tests can check
// it against the host libm over wide argument ranges.
#include "common.cuh"
#include <algorithm>

#include "crmath.cuh"

namespace mckl_b200 {

__global__ void k_math_f64(int fn, uint64_t n, const double *x, double *y, double *y2)
{
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const double v = x[i];
        switch (fn) {
            case 0: y[i] = dd::log(v); break;
            case 1: y[i] = dd::exp(v); break;
            default: {
                double s, c;
                dd::sincos(v, &s, &c);
                y[i] = s;
                if (y2) y2[i] = c;
            }
        }
    }
}

}  // namespace mckl_b200

using namespace mckl_b200;

extern "C" int mckl_b200_math_f64(int fn, size_t n, const double *x, double *y, double *y2, void *stream)
{
    MB_CHECK_ARG(fn >= 0 && fn <= 2, "fn must be 0 (log), 1 (exp) or 2 (sincos)");
    if (n == 0) return MCKL_B200_OK;
    MB_CHECK_ARG(x != nullptr && y != nullptr, "null pointer");
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, 4096));
    k_math_f64<<<grid, 256, 0, as_stream(stream)>>>(fn, n, x, y, y2);
    MB_LAUNCH_CHECK();
    return MCKL_B200_OK;
}
