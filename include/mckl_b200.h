/* mckl_b200.h -- C ABI of the B200 (sm_100a) implementation of MCKL's
 * counter-based RNG, distribution and SMC hot path.
 *
 * Conventions (all entry points):
 *   - `extern "C"`, plain pointers and sizes; returns an int status
 *     (MCKL_B200_OK == 0, negative on error; mckl_b200_last_error() gives the
 *     message).  No exception crosses this boundary.
 *   - Array arguments named `*_dev` / documented as device pointers must be
 *     addressable by the device: CUDA device memory, or page-locked host
 *     memory (cudaHostAlloc / cudaHostRegister), which kernels then read and
 *     write over the host link.  Engine states and scalar results live on the
 *     host.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *     stream).  Work is enqueued on it; a call returns before the GPU finishes
 *     unless its comment says it synchronizes.
 *   - Engine state is updated on the host exactly as the reference's
 *     CounterEngine would be after the same call sequence, so states stay
 *     interchangeable with mckl::Philox4x32 / Threefry4x64 / ARS (and _64).
 *
 * Reference citations are to the MCKL source tree (zhouyan/MCKL).
 */
#ifndef MCKL_B200_H
#define MCKL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MCKL_B200_OK 0
#define MCKL_B200_ERR_ARG (-1)     /* invalid argument (size, kind, null pointer) */
#define MCKL_B200_ERR_CUDA (-2)    /* a CUDA runtime call failed */
#define MCKL_B200_ERR_NOMEM (-3)   /* device scratch could not be obtained */
#define MCKL_B200_ERR_DEVICE (-4)  /* a kernel reported an error status */

/* Engine kinds: the reference's engine aliases with 32- and 64-bit results. */
#define MCKL_B200_PHILOX4X32 1      /* mckl::Philox4x32     random/philox.hpp:216    */
#define MCKL_B200_PHILOX4X32_64 2   /* mckl::Philox4x32_64  random/philox.hpp:232    */
#define MCKL_B200_THREEFRY4X64 3    /* mckl::Threefry4x64   random/threefry.hpp:271  */
#define MCKL_B200_THREEFRY4X64_64 4 /* mckl::Threefry4x64_64 random/threefry.hpp:307 */
#define MCKL_B200_ARS 5             /* mckl::ARS            random/aes.hpp:256       */
#define MCKL_B200_ARS_64 6          /* mckl::ARS_64         random/aes.hpp:272       */

/* State of one counter-based engine: mckl::CounterEngine<ResultType, Generator>
 * (random/counter.hpp:61-288).  `ctr` is the counter of the last generated
 * block in the reference's Counter layout (Counter<u32,4> = 2 x u64 for
 * Philox4x32 and ARS, 4 x u64 for Threefry4x64; random/increment.hpp:54-104).
 * `index` counts the words of that block already returned; a value >= words
 * per block (4 or 8 u32, 2 or 4 u64) means no word is buffered.  The buffered
 * block itself is not stored: it is a pure function of (key, ctr). */
typedef struct mckl_b200_engine {
    uint64_t ctr[4];
    uint64_t key[4];   /* Philox4x32: 2 x u32; ARS: 4 x u32; Threefry4x64: 4 x u64 */
    uint64_t tweak[2]; /* Threefry4x64 tweak (ThreefryGenerator::tweak, random/threefry.hpp:126-133) */
    uint32_t index;
    uint32_t kind;     /* MCKL_B200_PHILOX4X32 ... MCKL_B200_ARS_64 */
} mckl_b200_engine_t;

const char *mckl_b200_last_error(void);
const char *mckl_b200_version(void);
/* Number of kernels this library has launched in this process (diagnostics;
 * no counterpart in the reference). */
uint64_t mckl_b200_launch_count(void);
/* Working memory.  Calls that need device working memory beyond their
 * arguments (Weight, fold, resampling, rep -> index, the plain filter, Gamma,
 * the index matrix, the weighted estimate) take it from buffers the library
 * keeps per (device, stream): calls on different streams or host threads
 * never share them, calls on one stream are ordered by it.  A buffer grows
 * (stream-ordered, without synchronising the device) when a call needs more
 * than the stream's previous calls; growing is refused with
 * MCKL_B200_ERR_NOMEM while the stream is being captured into a CUDA graph,
 * so make one call of the largest size on a stream before capturing it.
 * mckl_b200_release_stream frees the buffers held for `stream` on the current
 * device (after its queued work); call it before destroying a stream the
 * library has used.  No counterpart in the reference (its objects own their
 * buffers). */
int mckl_b200_release_stream(void *stream);

/* ---- engines (host-only state operations, no GPU work) ------------------ */

/* CounterEngine::seed(s): key = {s, 0, ...}, ctr = 0, nothing buffered
 * (random/counter.hpp:97-103, 282-287). */
int mckl_b200_engine_seed(mckl_b200_engine_t *e, uint32_t kind, uint64_t seed);
/* CounterEngine::discard(nskip) (random/counter.hpp:178-199). */
int mckl_b200_engine_discard(mckl_b200_engine_t *e, uint64_t nskip);

/* ---- generator-level block kernels --------------------------------------
 * Same contract as the reference's native kernels
 * `void mckl_<engine>_<isa>_kernel(uint64_t *ctr, size_t n, void *r, const void *)`
 * (include/mckl/mckl.h:313-341; call sites random/internal/philox_avx2_4x32.hpp:94-121
 * and random/internal/aes_aesni_ars.hpp:175-190): n whole blocks for the
 * counters ctr+1 .. ctr+n are written to r_dev and ctr is advanced by n. */
int mckl_b200_philox4x32_kernel(uint64_t ctr[2], size_t n, void *r_dev, const uint32_t key[2],
    void *stream);
int mckl_b200_threefry4x64_kernel(uint64_t ctr[4], size_t n, void *r_dev, const uint64_t key[4],
    const uint64_t tweak[2], void *stream);
int mckl_b200_ars_kernel(uint64_t ctr[2], size_t n, void *r_dev, const uint32_t key[4],
    void *stream);

/* ---- raw words: mckl::rand(rng, n, r) (random/counter.hpp:142-165, 298-303)
 * n result words (u32, or u64 for the _64 kinds) into r_dev. */
int mckl_b200_rand(mckl_b200_engine_t *e, size_t n, void *r_dev, void *stream);

/* ---- U01 distributions (random/u01_distribution.hpp:131-142 and
 * random/internal/u01_generic.hpp:48-198), reference chunking included:
 * u01_canonical_distribution / u01_cc / u01_co / u01_oc / u01_oo. */
int mckl_b200_u01_canonical_f32(mckl_b200_engine_t *e, size_t n, float *r_dev, void *stream);
int mckl_b200_u01_canonical_f64(mckl_b200_engine_t *e, size_t n, double *r_dev, void *stream);
int mckl_b200_u01_cc_f32(mckl_b200_engine_t *e, size_t n, float *r_dev, void *stream);
int mckl_b200_u01_cc_f64(mckl_b200_engine_t *e, size_t n, double *r_dev, void *stream);
int mckl_b200_u01_co_f32(mckl_b200_engine_t *e, size_t n, float *r_dev, void *stream);
int mckl_b200_u01_co_f64(mckl_b200_engine_t *e, size_t n, double *r_dev, void *stream);
int mckl_b200_u01_oc_f32(mckl_b200_engine_t *e, size_t n, float *r_dev, void *stream);
int mckl_b200_u01_oc_f64(mckl_b200_engine_t *e, size_t n, double *r_dev, void *stream);
int mckl_b200_u01_oo_f32(mckl_b200_engine_t *e, size_t n, float *r_dev, void *stream);
int mckl_b200_u01_oo_f64(mckl_b200_engine_t *e, size_t n, double *r_dev, void *stream);

/* Normal: normal_distribution (random/normal_distribution.hpp:50-101): chunks of
 * 8192 bytes, Box-Muller with the first half of each chunk's uniforms as
 * radii; an odd n redraws its last value from two further U01OC words. */
int mckl_b200_normal_f32(mckl_b200_engine_t *e, size_t n, float *r_dev, float mean, float sd,
    void *stream);
int mckl_b200_normal_f64(mckl_b200_engine_t *e, size_t n, double *r_dev, double mean, double sd,
    void *stream);

/* Exponential: exponential_distribution (random/exponential_distribution.hpp:48-60). */
int mckl_b200_exponential_f32(mckl_b200_engine_t *e, size_t n, float *r_dev, float lambda,
    void *stream);
int mckl_b200_exponential_f64(mckl_b200_engine_t *e, size_t n, double *r_dev, double lambda,
    void *stream);

/* Gamma(alpha, beta): gamma_distribution (random/gamma_distribution.hpp:57-302):
 * chunks of 8192 bytes with the T / W / N / E algorithms chosen by alpha, the
 * accepted values compacted in order, scalar fallback for the last few; the
 * engine state after the call is the reference's.  One stream, so the chunks
 * run in order on one CTA. */
int mckl_b200_gamma_f32(mckl_b200_engine_t *e, size_t n, float *r_dev, float alpha, float beta, void *stream);
int mckl_b200_gamma_f64(mckl_b200_engine_t *e, size_t n, double *r_dev, double alpha, double beta,
    void *stream);

/* Independent Gamma streams, one per block of `block` samples: block b draws
 * gamma_distribution(rng_b, block, r + b * block, alpha_host[b], beta) with
 * rng_b = *e with counter (0, b, 0, 0) and an empty buffer (the reference's
 * rng.ctr() positioning, random/counter.hpp:129-133); *e is not changed.
 * No counterpart entry point in the reference: it is the per-block loop a
 * parallel caller writes around gamma_distribution. */
int mckl_b200_gamma_blocks_f32(const mckl_b200_engine_t *e, size_t nblocks, size_t block, const double *alpha_host,
    double beta, float *r_dev, void *stream);
int mckl_b200_gamma_blocks_f64(const mckl_b200_engine_t *e, size_t nblocks, size_t block, const double *alpha_host,
    double beta, double *r_dev, void *stream);

/* ---- SMC: Weight (core/weight.hpp:64-227) --------------------------------
 * W_dev: N normalised weights, updated in place; v_dev: N log-weight
 * increments.  add_log: log W_i += v_i (Weight::add_log, :143-148); set_log:
 * log W_i = v_i (Weight::set_log, :123-128); both then normalise exactly as
 * Weight::normalize(true) does, including its sequential sums, so W matches
 * the reference's bits up to the last-place rounding of exp/log.
 * ess (host, nullable): Weight::ess().  log_nc (host, nullable): log of the
 * normalising-constant ratio, log sum_i W_i^old exp(v_i) = max + log(sum).
 * Synchronizes the stream when ess or log_nc is requested. */
int mckl_b200_weight_set_log(size_t N, double *W_dev, const double *v_dev, double *ess, double *log_nc,
    void *stream);
int mckl_b200_weight_add_log(size_t N, double *W_dev, const double *v_dev, double *ess, double *log_nc_inc,
    void *stream);

/* ---- SMC: resampling (algorithm/resample.hpp) ---------------------------
 * Uniform sequences of u01_rand_sorted / _stratified / _systematic
 * (:216-268): kind 0 sorted, 1 stratified, 2 systematic; n doubles into u_dev. */
int mckl_b200_u01_sequence(int kind, mckl_b200_engine_t *rng, size_t n, double *u_dev, void *stream);
/* ResampleAlgorithm::operator()(N, M, rng, W, rep) (:514-566): scheme 0
 * Multinomial, 1 Stratified, 2 Systematic, 3 Residual, 4 ResidualStratified,
 * 5 ResidualSystematic (:569-593).  W_dev: N normalised weights; rep_dev: N
 * replication counts (sum M).  The engine must have 32-bit results.
 * Residual schemes synchronize (their number of uniforms depends on W). */
int mckl_b200_resample(int scheme, size_t N, size_t M, mckl_b200_engine_t *rng, const double *W_dev,
    uint64_t *rep_dev, void *stream);
/* resample_trans_rep_index (:416-466): replication counts -> M parent
 * indices; occupied slots keep their own particle.  Synchronizes. */
int mckl_b200_rep_to_index(size_t N, size_t M, const uint64_t *rep_dev, uint64_t *idx_dev, void *stream);
/* StateMatrix<ColMajor>::select with n == size() (core/state_matrix.hpp:239-253),
 * in place: state_dev is N x dim column-major, row i <- row idx[i]. */
int mckl_b200_select_f64(size_t N, size_t dim, const uint64_t *idx_dev, double *state_dev, void *stream);
int mckl_b200_select_f32(size_t N, size_t dim, const uint64_t *idx_dev, float *state_dev, void *stream);

/* ---- particle filters ----------------------------------------------------
 * Plain FP64 bootstrap filter for x_0 ~ N(0, sd0^2), x_t = phi x_{t-1} +
 * sx eps_t, y_t = x_t + sy eta_t, t = 1..T (y[0] unused; y is a HOST array of
 * T + 1 values), in SMCSampler's step order (algorithm/smc.hpp:389-406):
 * iteration 0 draws x_0; iteration t propagates with a Normal(0,1) batch from
 * the model engine Philox4x32(mkey), weights with Weight::add_log, records
 * the ESS and resamples with `scheme` (as in mckl_b200_resample) from the
 * engine Philox4x32(rkey) when ESS < N * threshold.  *loglik (host) = sum over
 * t of log sum_i W_{t-1,i} p(y_t | x_{t,i}).  ess_hist / resampled (host,
 * T + 1 entries) and anc_dev ((T + 1) x N parent indices, rows written at
 * resampling steps) are optional.  x_dev, W_dev (device, N) receive the final
 * particles and weights.  Synchronizes once per step. */
int mckl_b200_pf_ar1_plain_f64(size_t N, size_t T, const double *y, double phi, double sx, double sy, double sd0,
    const uint32_t mkey[2], const uint32_t rkey[2], int scheme, double threshold, double *loglik,
    double *ess_hist, uint8_t *resampled, uint64_t *anc_dev, double *x_dev, double *W_dev, void *stream);

/* Scan ties of the calling thread's last mckl_b200_pf_ar1_plain_f64 run: the
 * number of (uniform, cumulative weight) pairs over all its resampling steps
 * whose uniform lies within one representable step of the cumulative weight
 * (prev(c_i) <= u_j <= next(c_i)).  Those are the only comparisons that a
 * cumulative weight one ulp off would decide the other way; the cumulative
 * weights here are the reference's sequential fold bit for bit, so a tie
 * changes no ancestor.  Diagnostics; no counterpart in the reference. */
int mckl_b200_pf_ar1_plain_ties(uint64_t *ties);

/* Weight::add_log without any device allocation (no counterpart in the
 * reference).  Same contract and results as mckl_b200_weight_add_log, for
 * host programs that cannot let a library call cudaMalloc: plugins whose host
 * owns all device memory through its own pool or budget, code that must not
 * synchronize the device the way an allocation can, or processes running at
 * the memory limit.  Its working memory is a fixed 128 KiB array compiled into
 * the library, held on every GPU that loads it until the process exits; N is
 * limited to 4194304 (2^22) particles and larger N is rejected with
 * MCKL_B200_ERR_ARG.  The first call on a device looks up that array's device
 * address (cudaGetSymbolAddress) with the device current; make that first
 * call before any stream capture.  All calls share the one array: calls that
 * may run at the same time on the GPU (different streams, threads or graphs
 * without an ordering between them) race and must be serialized by the
 * caller.  Synchronizes when ess or log_nc_inc is requested. */
int mckl_b200_weight_add_log_static(size_t N, double *W_dev, const double *v_dev, double *ess, double *log_nc_inc,
    void *stream);

/* Batched filters (the chosen form, no single counterpart in the reference:
 * many SMCSampler runs at once).  F independent AR(1) filters, filter f with
 * N[f] particles, parameters phi[f], sx[f], sy[f], stationary x_0 (sd0 =
 * sx / sqrt(1 - phi^2)), observations y[f * (T + 1) + t] (HOST, t = 1..T), model
 * stream Philox4x32(mkeys[2f], mkeys[2f+1]) and resampling stream
 * Philox4x32(rkeys[2f], rkeys[2f+1]) consumed exactly as the plain filter
 * consumes them, systematic resampling when ESS < N * threshold.  fp64 = 0:
 * FP32 propagation and likelihoods, FP64 normaliser / log-likelihood / scan;
 * fp64 = 1: all FP64; fp64 = 2: FP32 as for 0, plus an FP64 shadow of every
 * particle driven by the same uniforms and by the FP32 run's resampling
 * decisions and parent indices, whose log-likelihood
 * (mckl_b200_batched_shadow) measures the FP32 arithmetic error alone.
 * create uploads and allocates; run launches one
 * persistent kernel (filters pulled from a queue, largest first); run_graph
 * replays it from a CUDA graph captured on first use; results copies the F
 * log-likelihood estimates and resampling counts to the host. */
typedef struct mckl_b200_batched mckl_b200_batched_t;
int mckl_b200_batched_create(mckl_b200_batched_t **out, size_t F, const size_t *N, size_t T, const double *y,
    const double *phi, const double *sx, const double *sy, const uint32_t *mkeys, const uint32_t *rkeys,
    double threshold, int fp64);
int mckl_b200_batched_config(mckl_b200_batched_t *b, int threads, int ctas_per_sm);
int mckl_b200_batched_run(mckl_b200_batched_t *b, void *stream);
int mckl_b200_batched_run_graph(mckl_b200_batched_t *b, void *stream);
int mckl_b200_batched_results(mckl_b200_batched_t *b, double *loglik, uint32_t *nresampled, void *stream);
int mckl_b200_batched_shadow(mckl_b200_batched_t *b, double *loglik_fp64, void *stream);
/* Replace the observations (HOST array of F x (T + 1), copied on `stream`). */
/* New parameters / new keys for every filter of a handle (HOST arrays of F,
 * keys F x 2), copied on `stream`; the next run (graph replays included)
 * uses them.  For callers that rerun the same filters with other parameters
 * or fresh randomness, e.g. the PMCMC driver below. */
int mckl_b200_batched_set_params(mckl_b200_batched_t *b, const double *phi, const double *sx, const double *sy,
                                 void *stream);
int mckl_b200_batched_set_keys(mckl_b200_batched_t *b, const uint32_t *mkeys, const uint32_t *rkeys, void *stream);

/* Shadow-run parameters (handles created with fp64 = 2 or 3): the FP64 shadow
 * follows the main run's resampling decisions and parent indices with its own
 * (phi, sx, sy) per filter (host arrays of F).  With perturbed parameters it
 * evaluates the estimate at theta +- h under common random numbers and fixed
 * ancestors -- the finite differences the adjoint is checked against. */
int mckl_b200_batched_shadow_params(mckl_b200_batched_t *b, const double *phi, const double *sx, const double *sy);

/* Adjoint: the gradient of each filter's FP64 log-likelihood estimate with
 * respect to (phi, sx, sy), resampling times and ancestor indices held fixed
 * (no counterpart in the reference, which has no derivatives).  The forward
 * pass keeps a checkpoint every `checkpoint_every` steps; the backward pass
 * replays each block of steps from its checkpoint -- the noise, decisions and
 * ancestors are recomputed from the counters, not stored -- and sweeps it in
 * reverse.  Handle created with fp64 = 1.  loglik: F doubles (may be NULL),
 * grad: F x 3 doubles (d/dphi, d/dsx, d/dsy), both HOST arrays; synchronizes
 * `stream`.  Device memory: checkpoints 16 B x particles x (T / C + 1) plus
 * per-SM replay records of C x the largest N x 28 B. */
int mckl_b200_batched_adjoint(mckl_b200_batched_t *b, int checkpoint_every, double *loglik, double *grad,
                              void *stream);

/* Score estimate by the Fisher identity (no counterpart in the reference):
 * grad log p(y_1:T | theta) = E[grad log p(x_0:T, y_1:T | theta) | y_1:T],
 * estimated in the same forward pass as each filter's FP64 log-likelihood by
 * PaRIS (per-particle statistics updated from two backward draws per step, an
 * independent Metropolis-Hastings chain started at the particle's ancestor).
 * Unlike the adjoint, which differentiates the estimate with the ancestors
 * held fixed, this is a consistent estimate of the exact score: its error
 * against the Kalman gradient is Monte Carlo error that falls as N grows.
 * Handle created with fp64 = 1.  loglik: F doubles (may be NULL), score:
 * F x 3 doubles (d/dphi, d/dsx, d/dsy), HOST arrays; synchronizes `stream`.
 * Device memory: 80 B x the largest N per SM. */
int mckl_b200_batched_score(mckl_b200_batched_t *b, double *loglik, double *score, void *stream);

/* Autotuner: times the candidate block shapes (threads per CTA x resident CTAs
 * per SM, skipping shapes that do not fit) on this handle's own filters, one
 * full run each, and configures the fastest.  The first `max_trials` trials
 * are reported in threads[] / ctas_per_sm[] / ms[] (any may be NULL); the
 * number of trials in *ntrials.  The pick is kept for the process: a later
 * handle with the same workload (device, precision mode, filter count, steps,
 * threshold and particle counts) is configured from it without timing
 * (*ntrials = 0).  Synchronizes `stream` when it times. */
int mckl_b200_batched_autotune(mckl_b200_batched_t *b, int max_trials, int *threads, int *ctas_per_sm, float *ms,
                               int *ntrials, void *stream);
int mckl_b200_batched_set_y(mckl_b200_batched_t *b, const double *y, void *stream);
/* The block shape the handle runs with (set by _config or the autotuner). */
int mckl_b200_batched_get_config(const mckl_b200_batched_t *b, int *threads, int *ctas_per_sm);
int mckl_b200_batched_destroy(mckl_b200_batched_t *b);

/* Sequential left fold s_i = s_{i-1} + x_i (s_{-1} = s0) of n nonnegative
 * doubles, bit-identical to the reference's `accw += w[i]` loops
 * (algorithm/resample.hpp:395-403, core/weight.hpp:221).  prefix_dev
 * (nullable) receives every s_i; *final_value (host) the last.  Synchronizes. */
int mckl_b200_fold_f64(size_t n, const double *x_dev, double s0, double *prefix_dev, double *final_value,
    void *stream);

/* ---- Engine state in the reference's text form --------------------------
 * CounterEngine's operator<< / operator>> (random/counter.hpp:235-272): save
 * writes the text `os << eng` produces for the engine in this state
 * (buffered results, counter, generator parameters, index; an unused buffer
 * as zeros) into buf (cap bytes; *len = its length, buf == NULL only asks
 * for it); load parses such text into *e of the given kind and checks the
 * buffered results against the counter.  Host-only, no device work. */
int mckl_b200_engine_save(const mckl_b200_engine_t *e, char *buf, size_t cap, size_t *len);
int mckl_b200_engine_load(mckl_b200_engine_t *e, uint32_t kind, const char *text);

/* ---- Genealogy: ResampleIndex (algorithm/resample.hpp:597-832) ----------
 * The ancestors of the N particles of the last of R recorded iterations at
 * every one of the R iterations (ResampleIndex::read_index_matrix, :752-829):
 * index_host is a HOST array of R DEVICE pointers to uint64 parent-index
 * vectors (entry r of sizes_host entries; the last has N), oldest first;
 * out (DEVICE) is N x R, row-major (R per particle) or column-major.  One
 * thread follows each particle's line back.  A parent index outside the
 * previous vector returns MCKL_B200_ERR_ARG.  Synchronizes the stream (to
 * read the error word). */
int mckl_b200_index_matrix(size_t N, size_t R, const uint64_t *const *index_host, const size_t *sizes_host,
                           int col_major, uint64_t *out_dev, void *stream);

/* ---- Estimates: SMCEstimator::estimate (algorithm/smc.hpp:90-120) -------
 * result_j = sum_i W_i u(i, j), j < d: the reference's cblas_dgemv of the
 * evaluations with the normalised weights.  u (DEVICE) n x d, row-major (d
 * values per particle, the reference's RowMajor) or column-major; W and
 * result DEVICE.  Deterministic order: FP64 partial sums over fixed ranges of
 * particles, then the partials in a fixed tree.  d <= 65535 column-major,
 * d <= 65535 * 256 row-major. */
int mckl_b200_weighted_estimate(size_t n, size_t d, int col_major, const double *u_dev, const double *W_dev,
                                double *result_dev, void *stream);

/* ---- PMCMC: PMCMCMutation (algorithm/pmcmc.hpp:72-165) ----------------
 * C particle marginal Metropolis-Hastings chains of the AR(1) model, one
 * batched filter per chain and iteration.  Chain c starts at theta0[3c..]
 * = (phi, sx, sy), proposes theta + step * z (z standard normal, symmetric
 * random walk) and accepts when log(U01) < -prior(theta) - logL(theta) +
 * prior(theta') + logL(theta'), the reference's order of terms.  `prior`
 * returns the log prior density (-inf outside the support; proposals with
 * |phi| >= 1 or a non-positive scale are rejected without a filter run).
 * Randomness: proposals and uniforms from Philox4x32 key (seed, c) at
 * counters 2i and 2i + 1; filter keys (c, mix(seed, 2i)) and
 * (c, mix(seed, 2i + 1)).  Outputs (HOST): theta_out iters x C x 3,
 * loglik_out iters x C (state after each iteration; iteration 0 is the
 * start), accepted C.  fp64: 0 FP32 moves (the chosen form), 1 FP64. */
typedef double (*mckl_b200_log_prior_t)(const double *theta, void *user);
int mckl_b200_pmcmc_ar1(size_t C, const size_t *N, size_t T, const double *y, const double *theta0,
                        const double *step, mckl_b200_log_prior_t prior, void *user, size_t iters, uint32_t seed,
                        int fp64, double threshold, double *theta_out, double *loglik_out, uint32_t *accepted,
                        void *stream);

/* The same chains with the proposal as a hook: PMCMCMutation's `update`
 * evaluations (algorithm/pmcmc.hpp:116-145, the sum at :141-145), each of
 * which takes the chain's RNG and a copy of the parameters, changes the copy
 * and returns its log proposal ratio.  `proposal(c, i, words, theta, user)`
 * is called for chain c at iteration i >= 1 with four Philox4x32 words
 * (key (seed, c), counter 2i: the randomness the built-in random walk turns
 * into its three normals) and theta = a copy of the chain's (phi, sx, sy) to
 * change in place; it returns log q(theta | theta') - log q(theta' | theta)
 * (0 for a symmetric proposal; a non-finite value rejects the proposal), which
 * enters the acceptance sum where the reference adds its evaluations.
 * mckl_b200_pmcmc_ar1 is this call with the Gaussian random walk. */
typedef double (*mckl_b200_proposal_t)(size_t chain, size_t iter, const uint32_t words[4], double *theta,
                                       void *user);
int mckl_b200_pmcmc_ar1_proposal(size_t C, const size_t *N, size_t T, const double *y, const double *theta0,
                                 mckl_b200_proposal_t proposal, void *proposal_user, mckl_b200_log_prior_t prior,
                                 void *user, size_t iters, uint32_t seed, int fp64, double threshold,
                                 double *theta_out, double *loglik_out, uint32_t *accepted, void *stream);

/* ---- diagnostics (no counterpart in the reference) ----------------------
 * The library's double-double log (fn 0), exp (fn 1) and sin/cos (fn 2; cos
 * into y2_dev when non-null) element-wise, for checking against a host libm. */
int mckl_b200_math_f64(int fn, size_t n, const double *x_dev, double *y_dev, double *y2_dev, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MCKL_B200_H */
