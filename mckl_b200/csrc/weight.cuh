// weight.cuh -- device-side Weight normalisation (weight.cu), shared with the
// particle-filter drivers.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace mckl_b200 {

size_t weight_scratch_bytes(uint64_t N);

// Normalise W in place (add_log: w = log W + v; otherwise w = v).  result_dev
// (device, 4 doubles) receives {ESS, log normalising-constant ratio, accw, lmax}.
int weight_normalize_dev(uint64_t N, double *W, const double *v, int add_log, void *scratch_base,
    double *result_dev, cudaStream_t s);

}  // namespace mckl_b200
