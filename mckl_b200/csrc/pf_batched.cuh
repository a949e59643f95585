// pf_batched.cuh -- descriptors of the batched particle filter (pf_batched.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace mckl_b200 {

struct BatchedFilter {
    uint64_t n;         // particles
    uint64_t off;       // offset of this filter's particles in the work arrays
    double phi, sx, sd0, lconst, hinv, sy;
    // shadow run (FP64, follows the main run's decisions): its parameters
    double phi_s, sx_s, sd0_s, lconst_s, hinv_s;
    uint32_t mkey[2];   // model stream: Philox4x32 key
    uint32_t rkey[2];   // resampling stream: Philox4x32 key
};

struct BatchedArgs {
    BatchedFilter *filt;
    double *y;          // F x (T + 1) observations
    int T;
    double threshold;
    int fp64;           // 1: propagate in double, 0: in float
    void *xa, *xb, *lw; // particles (resampled in place; xb unused), log-weights
    uint32_t *scanS, *epos;
    double *loglik;
    uint32_t *nresampled;
    double *xsa = nullptr, *xsb = nullptr, *lws = nullptr;  // FP64 shadow (FP32 run only)
    double *loglik_shadow = nullptr;
};

int pf_batched_launch(const BatchedArgs &a, const int *order, int nf, int threads, int ctas_per_sm, int *queue,
    cudaStream_t s);

}  // namespace mckl_b200
