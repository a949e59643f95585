/* oracle.h -- plain-C restatement of MCKL's counter-based RNG / SMC hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the CPU checker that the CUDA path is compared
 * against (tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg).
 * Nothing in the mckl_b200 package links or calls it.
 *
 * Parity is pinned: tests/test_oracle_pins.py checks every function here
 * against the reference's own known-answer files (example/random/random_<engine>.data,
 * first 1000 outputs of each seed-1 engine) and against the reference itself
 * compiled by oracle/Makefile (oracle/_ref/libmckl_ref.so), and the fixtures
 * in tests/golden/ were produced by the compiled reference.
 */
#ifndef MCKL_B200_ORACLE_H
#define MCKL_B200_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as mckl_b200_engine_t (include/mckl_b200.h). */
typedef struct orc_engine {
    uint64_t ctr[4];   /* counter of the last generated block */
    uint64_t key[4];   /* Philox4x32: 2 x u32, ARS: 4 x u32, Threefry4x64: 4 x u64 */
    uint64_t tweak[2]; /* Threefry4x64 tweak */
    uint32_t index;    /* words of that block already used; >= words/block: none buffered */
    uint32_t kind;     /* 1 Philox4x32, 2 Philox4x32_64, 3 Threefry4x64,
                          4 Threefry4x64_64, 5 ARS, 6 ARS_64 */
} orc_engine;

/* One generator block for counter `ctr` (16 bytes, 32 for Threefry4x64). */
int orc_block(const orc_engine *e, const uint64_t *ctr, void *out);

int orc_rand(orc_engine *e, size_t n, void *r);
int orc_u01(orc_engine *e, int variant, int is_f64, size_t n, void *r);
int orc_normal(orc_engine *e, int is_f64, size_t n, void *r, double mean, double sd);
int orc_exponential(orc_engine *e, int is_f64, size_t n, void *r, double lambda);
int orc_gamma(orc_engine *e, int is_f64, size_t n, void *r, double alpha, double beta);
int orc_gamma_blocks(const orc_engine *e, int is_f64, size_t nblocks, size_t block,
    const double *alpha, double beta, void *r, int nthreads);
int orc_gamma_blocks_from(const orc_engine *e, int is_f64, size_t first, size_t nblocks, size_t block,
    const double *alpha, double beta, void *r, int nthreads);

int orc_weight_set_log(size_t N, const double *v, double *W, double *ess);
int orc_weight_add_log(size_t N, double *W, const double *v, double *ess);

int orc_u01_sequence(int kind, orc_engine *e, size_t N, double *r);
int orc_u01_trans_sorted(size_t N, const double *u01, double *r);
int orc_rep_to_u01(size_t N, size_t M, const double *W, const double *u01seq, uint64_t *rep);
int orc_resample(int scheme, size_t N, size_t M, orc_engine *e, const double *W, uint64_t *rep);
int orc_rep_index(size_t N, size_t M, const uint64_t *rep, uint64_t *idx);
int orc_select_f64(size_t N, size_t dim, const uint64_t *idx, double *state);

int orc_simulate_ar1(size_t T, double phi, double sx, double sy, double sd0,
    const uint32_t key[2], double *x, double *y);
int orc_pf_ar1(size_t N, size_t T, const double *y, double phi, double sx, double sy,
    double sd0, const uint32_t mkey[2], const uint32_t rkey[2], int scheme,
    double threshold, double *loglik, double *ess_hist, uint8_t *resampled,
    uint64_t *anc, double *x_out, double *W_out);
int orc_weighted_estimate(size_t n, size_t d, int col_major, const double *u, const double *w, double *out);
int orc_fold(size_t n, const double *x, double s0, double *prefix, double *final_value);
int orc_math_f64(int fn, size_t n, const double *x, double *y, double *y2);
int orc_kalman_ar1(size_t T, const double *y, double phi, double sx, double sy,
    double *loglik, double *grad);

#ifdef __cplusplus
}
#endif

#endif
