// resample.cuh -- device-side resampling pieces (resample.cu), shared with
// the particle-filter drivers.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "../../include/mckl_b200.h"
#include "fold.cuh"

namespace mckl_b200 {

size_t resample_scratch_bytes(uint64_t N, uint64_t M);
size_t rep_index_scratch_bytes(uint64_t N, uint64_t M);

// Uniform sequence kind (0 sorted, 1 stratified, 2 systematic) of length n.
int u01_sequence_dev(int kind, mckl_b200_engine_t &e, uint64_t n, double *u, double *tmp, FoldScratch &fs,
    cudaStream_t s);
// ResampleAlgorithm::operator()(N, M, rng, W, rep); scheme 0 multinomial,
// 1 stratified, 2 systematic, 3 residual, 4 residual-stratified,
// 5 residual-systematic.  Residual schemes synchronize (the number of
// uniforms they draw depends on the weights).  ties_dev (device, nullable):
// incremented by the number of uniforms within one representable step of a
// cumulative weight.
int resample_dev(int scheme, uint64_t N, uint64_t M, mckl_b200_engine_t &e, const double *W, uint64_t *rep,
    void *scratch_base, cudaStream_t s, unsigned long long *ties_dev = nullptr);
int rep_to_index_dev(uint64_t N, uint64_t M, const uint64_t *rep, uint64_t *idx, void *scratch_base, int *err_dev,
    cudaStream_t s);

// The pieces of resample_dev for the schemes without residuals (0, 1, 2), so
// a caller can put the engine-independent half in a CUDA graph: the uniforms
// go to rs.u (u01_sequence_dev with rs.tmp and rs.fs), then rep_counts_dev
// folds W and counts (no engine, no host synchronisation).
struct ResampleScratch {
    double *u, *tmp;
    FoldScratch fs;
};
ResampleScratch resample_scratch_carve(void *scratch_base, uint64_t N, uint64_t M);
int rep_counts_dev(uint64_t N, uint64_t M, const double *W, const double *u, uint64_t *rep, ResampleScratch &rs,
    cudaStream_t s, unsigned long long *ties_dev);
template <typename T>
int select_dev(uint64_t N, uint64_t M, uint64_t dim, const uint64_t *idx, const T *in, T *out, cudaStream_t s);

}  // namespace mckl_b200
