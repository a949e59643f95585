// weight.cuh -- device-side Weight normalisation (weight.cu), shared with the
// particle-filter drivers.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace mckl_b200 {

// wcap: capacity of the exact fold's window list (0: the fold's default for N)
size_t weight_scratch_bytes(uint64_t N, uint64_t wcap = 0);

// Normalise W in place (add_log: w = log W + v; otherwise w = v).  result_dev
// (device, 4 doubles) receives {ESS, log normalising-constant ratio, accw, lmax}.
int weight_normalize_dev(uint64_t N, double *W, const double *v, int add_log, void *scratch_base,
    double *result_dev, cudaStream_t s, uint64_t wcap = 0);

}  // namespace mckl_b200
