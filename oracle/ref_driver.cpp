// ref_driver.cpp -- extern "C" wrappers around the MCKL reference headers.
//
// TEST INFRASTRUCTURE ONLY.  This file is compiled against the reference's own
// header-only sources (include/mckl/...) by oracle/Makefile into
// oracle/_ref/libmckl_ref.so.  It exists so that tests can (1) pin the plain-C
// restatement in oracle/oracle.c against the reference itself, (2) generate the
// golden fixtures under tests/golden/, and (3) time the reference's CPU path as
// the `cpu_baseline` / `--impl reference` arm of bench.py.  Nothing in the
// mckl_b200 package links or calls it.
//
// Every wrapper goes through the reference's public API:
//   engines        mckl::Philox4x32 / Threefry4x64 / ARS (+ _64)   random/{philox,threefry,aes}.hpp
//   raw words      mckl::rand(rng, n, r)                           random/counter.hpp:298-303
//   U01            mckl::u01_{canonical,cc,co,oc,oo}_distribution   random/u01_distribution.hpp:131-142
//   Normal         mckl::normal_distribution                        random/normal_distribution.hpp:83-101
//   Exponential    mckl::exponential_distribution                   random/exponential_distribution.hpp:59-60
//   Gamma          mckl::gamma_distribution                         random/gamma_distribution.hpp:277-302
//   Weight         mckl::Weight::{set_log,add_log,ess}              core/weight.hpp:123-148
//   resampling     mckl::Resample{Multinomial,...}                  algorithm/resample.hpp:569-593
//   rep -> index   mckl::resample_trans_rep_index                   algorithm/resample.hpp:416-466
//   SMC            mckl::SMCSampler + SMCSamplerEvalSMP<BackendSEQ> algorithm/smc.hpp:389-406
//
// Engine state crosses this boundary as `ref_engine`, the same POD layout as
// mckl_b200_engine_t in include/mckl_b200.h: the counter of the last generated
// block, the key, the Threefry tweak, and the number of words of that block
// already handed out (index == words per block means nothing is buffered).

#include <algorithm>
#include <cstring>
#include <mckl/algorithm/resample.hpp>
#include <mckl/algorithm/smc.hpp>
#include <mckl/core/state_matrix.hpp>
#include <mckl/random/aes.hpp>
#include <mckl/random/exponential_distribution.hpp>
#include <mckl/random/gamma_distribution.hpp>
#include <mckl/random/normal_distribution.hpp>
#include <mckl/random/philox.hpp>
#include <mckl/random/threefry.hpp>
#include <mckl/random/u01_distribution.hpp>
#include <mckl/smp.hpp>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <sstream>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

// The reference declares the Fortran BLAS dgemv_ for its SMCEstimator
// (internal/cblas.hpp:115-120) when no CBLAS is configured; no BLAS library is
// installed here, so a plain column-major dgemv is supplied.  None of the
// wrappers below registers an estimator, so it is only needed to link.
void dgemv_(const char *trans, const int *m, const int *n, const double *alpha,
    const double *a, const int *lda, const double *x, const int *incx,
    const double *beta, double *y, const int *incy)
{
    const bool t = (*trans == 'T' || *trans == 't' || *trans == 'C' ||
        *trans == 'c');
    const int leny = t ? *n : *m;
    const int lenx = t ? *m : *n;
    for (int i = 0; i != leny; ++i) {
        y[i * *incy] = (*beta == 0) ? 0.0 : *beta * y[i * *incy];
    }
    for (int j = 0; j != *n; ++j) {
        for (int i = 0; i != *m; ++i) {
            const double aij = a[i + static_cast<long>(j) * *lda];
            if (t) {
                y[j * *incy] += *alpha * aij * x[i * *incx];
            } else {
                y[i * *incy] += *alpha * aij * x[j * *incx];
            }
        }
    }
    (void) lenx;
}

struct ref_engine {
    std::uint64_t ctr[4];
    std::uint64_t key[4];
    std::uint64_t tweak[2];
    std::uint32_t index;
    std::uint32_t kind;
};

} // extern "C"

namespace {

enum Kind {
    kPhilox4x32 = 1,
    kPhilox4x32_64 = 2,
    kThreefry4x64 = 3,
    kThreefry4x64_64 = 4,
    kARS = 5,
    kARS_64 = 6
};

template <typename Eng>
constexpr unsigned words_per_block()
{
    return static_cast<unsigned>(
        Eng::generator_type::size() / sizeof(typename Eng::result_type));
}

template <typename C>
void ctr_decrement(C &c)
{
    for (auto &w : c) {
        if (w-- != 0) {
            return;
        }
    }
}

template <typename Eng>
void set_tweak(Eng &, const ref_engine *)
{
}

template <typename R>
void set_tweak(mckl::ThreefryEngine<R, std::uint64_t, 4> &eng,
    const ref_engine *s)
{
    if (s->tweak[0] != 0 || s->tweak[1] != 0) {
        eng.generator().tweak(s->tweak[0], s->tweak[1]);
    }
}

std::vector<unsigned long long> tokens_of(const std::string &str)
{
    std::istringstream is(str);
    std::vector<unsigned long long> t;
    unsigned long long v;
    while (is >> v) {
        t.push_back(v);
    }
    return t;
}

// Put `eng` into exactly the state described by `s`.
template <typename Eng>
void load(Eng &eng, const ref_engine *s)
{
    using key_type = typename Eng::key_type;
    using ctr_type = typename Eng::ctr_type;
    constexpr unsigned M = words_per_block<Eng>();

    key_type key;
    for (std::size_t i = 0; i != key.size(); ++i) {
        key[i] = static_cast<typename key_type::value_type>(s->key[i]);
    }
    eng.seed(key);
    set_tweak(eng, s);

    ctr_type c;
    for (std::size_t i = 0; i != c.size(); ++i) {
        c[i] = static_cast<typename ctr_type::value_type>(s->ctr[i]);
    }
    if (s->index >= M) {
        eng.ctr(c);
        return;
    }

    // Generate block c into the buffer, then rewrite the buffer index through
    // the engine's own text serialisation (random/counter.hpp:235-272).
    ctr_type cm = c;
    ctr_decrement(cm);
    eng.ctr(cm);
    (void) eng();
    std::ostringstream os;
    os << eng;
    std::vector<unsigned long long> t = tokens_of(os.str());
    t.back() = s->index;
    std::ostringstream rebuilt;
    for (std::size_t i = 0; i != t.size(); ++i) {
        rebuilt << (i == 0 ? "" : " ") << t[i];
    }
    std::istringstream is(rebuilt.str());
    is >> eng;
}

template <typename Eng>
void store(const Eng &eng, ref_engine *s)
{
    constexpr unsigned M = words_per_block<Eng>();
    std::ostringstream os;
    os << eng;
    std::vector<unsigned long long> t = tokens_of(os.str());
    // layout: M r_0..r_{M-1} Kc c_0..c_{Kc-1} <generator> index
    const std::size_t kc = static_cast<std::size_t>(t[M + 1]);
    for (std::size_t i = 0; i != 4; ++i) {
        s->ctr[i] = i < kc ? static_cast<std::uint64_t>(t[M + 2 + i]) : 0;
    }
    s->index = static_cast<std::uint32_t>(t.back());
}

// Run `f(engine)` on the engine type selected by s->kind, with load/store.
template <typename F>
int with_engine(ref_engine *s, F &&f)
{
    switch (s->kind) {
        case kPhilox4x32: {
            mckl::Philox4x32 e;
            load(e, s);
            f(e);
            store(e, s);
            return 0;
        }
        case kPhilox4x32_64: {
            mckl::Philox4x32_64 e;
            load(e, s);
            f(e);
            store(e, s);
            return 0;
        }
        case kThreefry4x64: {
            mckl::Threefry4x64 e;
            load(e, s);
            f(e);
            store(e, s);
            return 0;
        }
        case kThreefry4x64_64: {
            mckl::Threefry4x64_64 e;
            load(e, s);
            f(e);
            store(e, s);
            return 0;
        }
        case kARS: {
            mckl::ARS e;
            load(e, s);
            f(e);
            store(e, s);
            return 0;
        }
        case kARS_64: {
            mckl::ARS_64 e;
            load(e, s);
            f(e);
            store(e, s);
            return 0;
        }
        default:
            return -1;
    }
}

template <typename T>
struct U01Call {
    int variant;
    std::size_t n;
    T *r;
    template <typename Eng>
    void operator()(Eng &e) const
    {
        switch (variant) {
            case 0:
                mckl::u01_canonical_distribution(e, n, r);
                break;
            case 1:
                mckl::u01_cc_distribution(e, n, r);
                break;
            case 2:
                mckl::u01_co_distribution(e, n, r);
                break;
            case 3:
                mckl::u01_oc_distribution(e, n, r);
                break;
            case 4:
                mckl::u01_oo_distribution(e, n, r);
                break;
        }
    }
};

} // namespace

extern "C" {

int ref_rand(ref_engine *s, std::size_t n, void *r)
{
    return with_engine(s, [n, r](auto &e) {
        using R = typename std::remove_reference_t<decltype(e)>::result_type;
        mckl::rand(e, n, static_cast<R *>(r));
    });
}

int ref_u01(ref_engine *s, int variant, int is_f64, std::size_t n, void *r)
{
    if (variant < 0 || variant > 4) {
        return -2;
    }
    if (is_f64) {
        return with_engine(s, U01Call<double>{variant, n, static_cast<double *>(r)});
    }
    return with_engine(s, U01Call<float>{variant, n, static_cast<float *>(r)});
}

int ref_normal(ref_engine *s, int is_f64, std::size_t n, void *r, double mean,
    double sd)
{
    if (is_f64) {
        return with_engine(s, [=](auto &e) {
            mckl::normal_distribution(e, n, static_cast<double *>(r), mean, sd);
        });
    }
    return with_engine(s, [=](auto &e) {
        mckl::normal_distribution(e, n, static_cast<float *>(r),
            static_cast<float>(mean), static_cast<float>(sd));
    });
}

int ref_exponential(
    ref_engine *s, int is_f64, std::size_t n, void *r, double lambda)
{
    if (is_f64) {
        return with_engine(s, [=](auto &e) {
            mckl::exponential_distribution(e, n, static_cast<double *>(r), lambda);
        });
    }
    return with_engine(s, [=](auto &e) {
        mckl::exponential_distribution(
            e, n, static_cast<float *>(r), static_cast<float>(lambda));
    });
}

int ref_gamma(ref_engine *s, int is_f64, std::size_t n, void *r, double alpha,
    double beta)
{
    if (is_f64) {
        return with_engine(s, [=](auto &e) {
            mckl::gamma_distribution(e, n, static_cast<double *>(r), alpha, beta);
        });
    }
    return with_engine(s, [=](auto &e) {
        mckl::gamma_distribution(e, n, static_cast<float *>(r),
            static_cast<float>(alpha), static_cast<float>(beta));
    });
}

// Gamma over independent 4096-sample blocks: block b uses the engine in `s`
// with ctr[1] = b (ctr[0] = 0, nothing buffered) and shape alpha[b].
int ref_gamma_blocks(const ref_engine *s, int is_f64, std::size_t nblocks,
    std::size_t block, const double *alpha, double beta, void *r, int nthreads)
{
    int rc = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads > 0 ? nthreads : 1) reduction(| : rc)
#endif
    for (long long b = 0; b < static_cast<long long>(nblocks); ++b) {
        ref_engine e = *s;
        e.ctr[0] = 0;
        e.ctr[1] = static_cast<std::uint64_t>(b);
        e.ctr[2] = e.ctr[3] = 0;
        e.index = 0xFFFFFFFFu;
        if (is_f64) {
            rc |= ref_gamma(&e, 1, block,
                static_cast<double *>(r) + static_cast<std::size_t>(b) * block,
                alpha[b], beta);
        } else {
            rc |= ref_gamma(&e, 0, block,
                static_cast<float *>(r) + static_cast<std::size_t>(b) * block,
                alpha[b], beta);
        }
    }
    (void) nthreads;
    return rc;
}

int ref_weight_set_log(std::size_t N, const double *v, double *W, double *ess)
{
    mckl::Weight w(N);
    w.set_log(v);
    w.read(W);
    *ess = w.ess();
    return 0;
}

int ref_weight_add_log(std::size_t N, double *W, const double *v, double *ess)
{
    mckl::Weight w(N);
    w.set_exact(static_cast<double>(N), W);
    w.add_log(v);
    w.read(W);
    *ess = w.ess();
    return 0;
}

// scheme: 0 multinomial, 1 stratified, 2 systematic, 3 residual,
//         4 residual-stratified, 5 residual-systematic
int ref_resample(int scheme, std::size_t N, std::size_t M, ref_engine *s,
    const double *W, std::uint64_t *rep)
{
    std::vector<std::size_t> r(N);
    int rc = with_engine(s, [&](auto &e) {
        switch (scheme) {
            case 0:
                mckl::ResampleMultinomial()(N, M, e, W, r.data());
                break;
            case 1:
                mckl::ResampleStratified()(N, M, e, W, r.data());
                break;
            case 2:
                mckl::ResampleSystematic()(N, M, e, W, r.data());
                break;
            case 3:
                mckl::ResampleResidual()(N, M, e, W, r.data());
                break;
            case 4:
                mckl::ResampleResidualStratified()(N, M, e, W, r.data());
                break;
            case 5:
                mckl::ResampleResidualSystematic()(N, M, e, W, r.data());
                break;
        }
    });
    for (std::size_t i = 0; i != N; ++i) {
        rep[i] = r[i];
    }
    return rc;
}

// Sorted (0), stratified (1) and systematic (2) uniform sequences.
int ref_u01_sequence(int kind, ref_engine *s, std::size_t N, double *r)
{
    return with_engine(s, [=](auto &e) {
        switch (kind) {
            case 0:
                mckl::u01_rand_sorted(e, N, r);
                break;
            case 1:
                mckl::u01_rand_stratified(e, N, r);
                break;
            case 2:
                mckl::u01_rand_systematic(e, N, r);
                break;
        }
    });
}

int ref_u01_trans_sorted(std::size_t N, const double *u01, double *r)
{
    mckl::u01_trans_sorted(N, u01, r);
    return 0;
}

int ref_rep_to_u01(std::size_t N, std::size_t M, const double *W,
    const double *u01seq, std::uint64_t *rep)
{
    std::vector<std::size_t> r(N);
    mckl::resample_trans_u01_rep(N, M, W, u01seq, r.data());
    for (std::size_t i = 0; i != N; ++i) {
        rep[i] = r[i];
    }
    return 0;
}

int ref_rep_index(
    std::size_t N, std::size_t M, const std::uint64_t *rep, std::uint64_t *idx)
{
    std::vector<std::size_t> r(rep, rep + N);
    std::vector<std::size_t> x(M);
    mckl::resample_trans_rep_index(N, M, r.data(), x.data());
    for (std::size_t i = 0; i != M; ++i) {
        idx[i] = x[i];
    }
    return 0;
}

// The engine in state `s` written with the reference's operator<<
// (random/counter.hpp:235-250), and a state read with its operator>>
// (:252-272) into `s`.
int ref_engine_to_text(ref_engine *s, char *buf, std::size_t cap)
{
    std::string text;
    with_engine(s, [&](auto &e) {
        std::ostringstream os;
        os << e;
        text = os.str();
    });
    if (text.size() + 1 > cap) return 1;
    std::memcpy(buf, text.c_str(), text.size() + 1);
    return 0;
}

// Read `text` with operator>> and write the engine back with operator<<.
int ref_engine_text_roundtrip(ref_engine *s, const char *text, char *buf, std::size_t cap)
{
    int rc = 0;
    std::string out;
    with_engine(s, [&](auto &e) {
        std::istringstream is(text);
        is >> e;
        rc = is ? 0 : 1;
        std::ostringstream os;
        os << e;
        out = os.str();
    });
    if (rc || out.size() + 1 > cap) return 1;
    std::memcpy(buf, out.c_str(), out.size() + 1);
    return 0;
}

int ref_engine_from_text(ref_engine *s, const char *text)
{
    int rc = 0;
    with_engine(s, [&](auto &e) {
        std::istringstream is(text);
        is >> e;
        rc = is ? 0 : 1;
    });
    return rc;
}

// ResampleIndex (algorithm/resample.hpp:597-832): push R parent-index
// vectors of N entries, then read the ancestor matrix of iterations
// iter..iter_back (row- or column-major) and the single-particle trace
// index(id, iter_back, iter) for every id.
int ref_index_matrix(std::size_t N, std::size_t R, const std::uint64_t *idx, std::size_t iter_back,
    std::size_t iter, int col_major, std::uint64_t *out, std::uint64_t *trace)
{
    mckl::ResampleIndex<std::size_t> ri;
    for (std::size_t r = 0; r < R; ++r) {
        ri.push_back(N, idx + r * N);
    }
    ri.read_index_matrix(col_major ? mckl::ColMajor : mckl::RowMajor, out, iter_back, iter);
    if (trace) {
        for (std::size_t i = 0; i < N; ++i) trace[i] = ri.index(i, iter_back, iter);
    }
    return 0;
}

int ref_select_f64(std::size_t N, std::size_t dim, const std::uint64_t *idx,
    double *state)
{
    using SM = mckl::StateMatrix<mckl::ColMajor, double>;
    SM sm(N, dim);
    for (std::size_t d = 0; d != dim; ++d) {
        std::copy_n(state + d * N, N, sm.col_data(d));
    }
    std::vector<std::size_t> x(idx, idx + N);
    sm.select(N, x.data());
    for (std::size_t d = 0; d != dim; ++d) {
        std::copy_n(sm.col_data(d), N, state + d * N);
    }
    return 0;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Bootstrap particle filter for the AR(1) + Gaussian-noise model
//   x_0 ~ N(0, sd0^2),  x_t = phi x_{t-1} + sx eps_t,  y_t = x_t + sy eta_t
// run through mckl::SMCSampler.  Iteration 0 draws x_0 (no weighting);
// iteration t = 1..T propagates and weights with y_t.
// ---------------------------------------------------------------------------

namespace {

using AR1State = mckl::StateMatrix<mckl::ColMajor, double, 1>;

struct AR1Params {
    double phi, sx, sy, sd0;
    const double *y; // y[1..T] (y[0] unused)
    double lconst;   // -log(sy) - 0.5 log(2 pi)
    double hinv;     // 0.5 / (sy * sy)
};

template <typename Backend>
class AR1Selection
    : public mckl::SMCSamplerEvalSMP<AR1State, AR1Selection<Backend>, Backend>
{
  public:
    AR1Selection(const AR1Params &p, double *loglik) : p_(p), loglik_(loglik)
    {
    }

    void operator()(std::size_t iter, mckl::Particle<AR1State> &particle)
    {
        this->run(iter, particle, 1024);
    }

    void eval_first(std::size_t, mckl::Particle<AR1State> &particle)
    {
        ll_.resize(particle.size());
        eps_.resize(particle.size());
    }

    void eval_range(
        std::size_t iter, const mckl::ParticleRange<AR1State> &range)
    {
        auto rng = range.begin().rng();
        const std::size_t n = range.size();
        double *x = range.particle().state().col_data(0) + range.ibegin();
        double *ll = ll_.data() + range.ibegin();
        double *eps = eps_.data() + range.ibegin();
        if (iter == 0) {
            mckl::normal_distribution(rng, n, x, 0.0, p_.sd0);
        } else {
            mckl::normal_distribution(rng, n, eps, 0.0, 1.0);
            const double yt = p_.y[iter];
            for (std::size_t i = 0; i != n; ++i) {
                const double a = p_.phi * x[i];
                const double b = p_.sx * eps[i];
                x[i] = a + b;
                const double r = yt - x[i];
                const double r2 = r * r;
                ll[i] = p_.lconst - r2 * p_.hinv;
            }
        }
        range.begin().rng() = rng;
    }

    void eval_last(std::size_t iter, mckl::Particle<AR1State> &particle)
    {
        if (iter == 0) {
            return;
        }
        // log-likelihood increment: log sum_i W_{t-1,i} exp(ll_i), evaluated
        // as m + log sum_i W_i exp(ll_i - m) with the pre-update weights.
        const std::size_t N = particle.size();
        const double *W = particle.weight().data();
        double m = -std::numeric_limits<double>::infinity();
        for (std::size_t i = 0; i != N; ++i) {
            m = ll_[i] > m ? ll_[i] : m;
        }
        double s = 0;
        for (std::size_t i = 0; i != N; ++i) {
            s += W[i] * std::exp(ll_[i] - m);
        }
        *loglik_ += m + std::log(s);
        particle.weight().add_log(ll_.data());
    }

  private:
    AR1Params p_;
    double *loglik_;
    std::vector<double> ll_;
    std::vector<double> eps_;
};

template <typename Backend>
int pf_run(std::size_t N, std::size_t T, const AR1Params &p,
    const std::uint32_t mkey[2], const std::uint32_t rkey[2], int scheme,
    double threshold, double *loglik, double *ess_hist, std::uint8_t *resampled,
    std::uint64_t *anc, double *x_out, double *W_out, int record,
    std::uint64_t *digest = nullptr)
{
    mckl::SMCSampler<AR1State> sampler(N);
    std::array<std::uint32_t, 2> mk = {{mkey[0], mkey[1]}};
    std::array<std::uint32_t, 2> rk = {{rkey[0], rkey[1]}};
    sampler.particle().rng(0).seed(mk);
    sampler.particle().rng().seed(rk);
    *loglik = 0;
    sampler.selection(AR1Selection<Backend>(p, loglik));
    std::size_t rs_count = 0;
    if (record) {
        // Same three calls as mckl::ResampleEval::operator()
        // (algorithm/resample.hpp:494-507), recording the parent indices.
        sampler.resample([&, scheme](std::size_t iter,
                             mckl::Particle<AR1State> &particle) {
            const std::size_t n = particle.size();
            std::vector<std::size_t> rep(n), idx(n);
            switch (scheme) {
                case 0:
                    mckl::ResampleMultinomial()(
                        n, n, particle.rng(), particle.weight().data(), rep.data());
                    break;
                case 1:
                    mckl::ResampleStratified()(
                        n, n, particle.rng(), particle.weight().data(), rep.data());
                    break;
                case 2:
                    mckl::ResampleSystematic()(
                        n, n, particle.rng(), particle.weight().data(), rep.data());
                    break;
                default:
                    mckl::ResampleResidual()(
                        n, n, particle.rng(), particle.weight().data(), rep.data());
                    break;
            }
            mckl::resample_trans_rep_index(n, n, rep.data(), idx.data());
            if (anc != nullptr) {
                for (std::size_t i = 0; i != n; ++i) {
                    anc[iter * n + i] = idx[i];
                }
            }
            if (digest != nullptr) {
                // two exact integer sums of the parent vector (no wrap below
                // 2^31 particles): sum idx_i and sum idx_i (i + 1)
                std::uint64_t d1 = 0, d2 = 0;
                for (std::size_t i = 0; i != n; ++i) {
                    d1 += idx[i];
                    d2 += idx[i] * (i + 1);
                }
                digest[2 * iter] = d1;
                digest[2 * iter + 1] = d2;
            }
            if (resampled != nullptr) {
                resampled[iter] = 1;
            }
            ++rs_count;
            particle.select(n, idx.data());
        });
    } else {
        switch (scheme) {
            case 0:
                sampler.resample(mckl::Multinomial);
                break;
            case 1:
                sampler.resample(mckl::Stratified);
                break;
            case 2:
                sampler.resample(mckl::Systematic);
                break;
            default:
                sampler.resample(mckl::Residual);
                break;
        }
    }
    sampler.resample_threshold(threshold);
    sampler.iterate(T + 1);
    if (ess_hist != nullptr) {
        sampler.read_ess_history(ess_hist);
    }
    if (x_out != nullptr) {
        std::copy_n(sampler.particle().state().col_data(0), N, x_out);
    }
    if (W_out != nullptr) {
        sampler.particle().weight().read(W_out);
    }
    return 0;
}

} // namespace

extern "C" {

// backend: 0 = BackendSEQ (bit-comparable), 1 = BackendOMP (throughput only).
int ref_pf_ar1(std::size_t N, std::size_t T, const double *y, double phi,
    double sx, double sy, double sd0, const std::uint32_t mkey[2],
    const std::uint32_t rkey[2], int scheme, double threshold, int backend,
    double *loglik, double *ess_hist, std::uint8_t *resampled,
    std::uint64_t *anc, double *x_out, double *W_out, int record)
{
    AR1Params p;
    p.phi = phi;
    p.sx = sx;
    p.sy = sy;
    p.sd0 = sd0;
    p.y = y;
    p.lconst = -std::log(sy) - 0.5 * std::log(2 * 3.14159265358979323846);
    p.hinv = 0.5 / (sy * sy);
    if (backend == 1) {
        return pf_run<mckl::BackendOMP>(N, T, p, mkey, rkey, scheme, threshold,
            loglik, ess_hist, resampled, anc, x_out, W_out, record);
    }
    return pf_run<mckl::BackendSEQ>(N, T, p, mkey, rkey, scheme, threshold,
        loglik, ess_hist, resampled, anc, x_out, W_out, record);
}

// The same BackendSEQ run, recording per resampling iteration only two exact
// sums of its parent vector (digest[2 t], digest[2 t + 1]; zero where the
// iteration did not resample), so long runs at large N need no T x N record.
int ref_pf_ar1_digest(std::size_t N, std::size_t T, const double *y,
    double phi, double sx, double sy, double sd0, const std::uint32_t mkey[2],
    const std::uint32_t rkey[2], int scheme, double threshold, double *loglik,
    double *ess_hist, std::uint8_t *resampled, std::uint64_t *digest,
    double *x_out)
{
    AR1Params p;
    p.phi = phi;
    p.sx = sx;
    p.sy = sy;
    p.sd0 = sd0;
    p.y = y;
    p.lconst = -std::log(sy) - 0.5 * std::log(2 * 3.14159265358979323846);
    p.hinv = 0.5 / (sy * sy);
    std::fill_n(digest, 2 * (T + 1), std::uint64_t(0));
    return pf_run<mckl::BackendSEQ>(N, T, p, mkey, rkey, scheme, threshold,
        loglik, ess_hist, resampled, nullptr, x_out, nullptr, 1, digest);
}

// Many independent filters (one BackendSEQ sampler each), OpenMP over filters.
int ref_pf_ar1_batch(std::size_t F, const std::size_t *N, std::size_t T,
    const double *y /* F x (T+1) */, const double *phi, const double *sx,
    const double *sy, const std::uint32_t *mkeys /* F x 2 */,
    const std::uint32_t *rkeys /* F x 2 */, int scheme, double threshold,
    double *loglik, int nthreads)
{
    int rc = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1) reduction(| : rc)
#endif
    for (long long f = 0; f < static_cast<long long>(F); ++f) {
        const double sd0 = phi[f] * phi[f] < 1 ?
            sx[f] / std::sqrt(1 - phi[f] * phi[f]) :
            sx[f];
        rc |= ref_pf_ar1(N[f], T, y + f * (T + 1), phi[f], sx[f], sy[f], sd0,
            mkeys + 2 * f, rkeys + 2 * f, scheme, threshold, 0, loglik + f,
            nullptr, nullptr, nullptr, nullptr, nullptr, 0);
    }
    (void) nthreads;
    return rc;
}

// ---------------------------------------------------------------------------
// CPU throughput baselines: the reference's fills on `nthreads` host threads.
// Each thread positions its own engine at a block-aligned counter offset
// (rng.ctr(c), random/counter.hpp:129-133), so the words written are the same
// as one sequential stream.  Returns elapsed seconds (steady_clock).
// ---------------------------------------------------------------------------

double ref_fill_u32_parallel(const ref_engine *s, std::size_t nwords,
    std::uint32_t *r, int nthreads)
{
    const unsigned M = (s->kind == kThreefry4x64) ? 8 : 4;
    const std::size_t nblocks = nwords / M;
    auto t0 = std::chrono::steady_clock::now();
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
#endif
    {
        int tid = 0, nt = 1;
#ifdef _OPENMP
        tid = omp_get_thread_num();
        nt = omp_get_num_threads();
#endif
        const std::size_t b0 = nblocks * static_cast<std::size_t>(tid) / nt;
        const std::size_t b1 =
            nblocks * static_cast<std::size_t>(tid + 1) / nt;
        ref_engine e = *s;
        e.ctr[0] = s->ctr[0] + b0;
        e.index = 0xFFFFFFFFu;
        ref_rand(&e, (b1 - b0) * M, r + b0 * M);
    }
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

// Distribution fill over `nthreads` threads.  dist: 0..4 = U01 variants
// (canonical, cc, co, oc, oo), 5 = Normal(0,1), 6 = Exponential(1).  Each
// thread starts at a whole number of the reference's 8192-byte chunks, which
// is also a whole number of blocks, so outputs equal one sequential call.
double ref_dist_parallel(const ref_engine *s, int dist, int is_f64,
    std::size_t n, void *r, int nthreads)
{
    const std::size_t esz = is_f64 ? 8 : 4;
    const std::size_t K = 8192 / esz;
    const std::size_t nchunks = n / K;
    const unsigned M = (s->kind == kThreefry4x64) ? 8 : 4;
    const std::size_t words_per_elem = (dist == 0 && is_f64) ? 2 : 1;
    auto t0 = std::chrono::steady_clock::now();
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
#endif
    {
        int tid = 0, nt = 1;
#ifdef _OPENMP
        tid = omp_get_thread_num();
        nt = omp_get_num_threads();
#endif
        const std::size_t c0 = nchunks * static_cast<std::size_t>(tid) / nt;
        const std::size_t c1 =
            nchunks * static_cast<std::size_t>(tid + 1) / nt;
        std::size_t e0 = c0 * K;
        std::size_t e1 = (tid + 1 == nt) ? n : c1 * K;
        ref_engine e = *s;
        e.ctr[0] = s->ctr[0] + e0 * words_per_elem / M;
        e.index = 0xFFFFFFFFu;
        char *out = static_cast<char *>(r) + e0 * esz;
        if (dist <= 4) {
            ref_u01(&e, dist, is_f64, e1 - e0, out);
        } else if (dist == 5) {
            ref_normal(&e, is_f64, e1 - e0, out, 0.0, 1.0);
        } else {
            ref_exponential(&e, is_f64, e1 - e0, out, 1.0);
        }
    }
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

int ref_max_threads()
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

} // extern "C"
