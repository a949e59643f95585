// weight.cuh -- device-side Weight normalisation (weight.cu), shared with the
// particle-filter drivers.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace mckl_b200 {

// wcap: capacity of the exact fold's window list (0: the fold's default for N)
size_t weight_scratch_bytes(uint64_t N, uint64_t wcap = 0);

// A second stream and two events owned by the caller: with them the ESS's
// chunk dot products run on `side` while `s` runs the normaliser's fold (the
// two meet before the result is formed).  Works the same when `s` is being
// captured into a graph (the events become the graph's edges).
struct WeightFork {
    cudaStream_t side;
    cudaEvent_t fork, join;
};

// Normalise W in place (add_log: w = log W + v; otherwise w = v).  result_dev
// (device, 4 doubles) receives {ESS, log normalising-constant ratio, accw, lmax}.
// `fork` (nullable): overlap the ESS with the fold, as above.
int weight_normalize_dev(uint64_t N, double *W, const double *v, int add_log, void *scratch_base,
    double *result_dev, cudaStream_t s, uint64_t wcap = 0, const WeightFork *fork = nullptr);

}  // namespace mckl_b200
