// pmcmc.cu -- particle marginal Metropolis-Hastings for many chains at once.
//
// The reference's PMCMCMutation (algorithm/pmcmc.hpp:72-165) runs one chain:
// each iteration proposes new parameters (its `update` evaluations return the
// log proposal ratio), runs the particle filter with them, and accepts when
// log(U01) < -prior(old) - logL(old) + sum of evaluations + prior(new) +
// logL(new).  Here C chains of the AR(1) model advance together: the C
// filters of one iteration are one batched launch (one filter per chain), and
// the Metropolis-Hastings arithmetic, in the reference's order, runs on the
// host.  Proposals are Gaussian random walks (symmetric: the evaluations
// contribute 0).
//
// Randomness: chain c's proposal normals and acceptance uniform at iteration
// i come from Philox4x32-10 with key (seed, c) at counters 2i (three normals:
// Box-Muller on words (0, 1) and (2, 3)) and 2i + 1 (the uniform, word 0);
// the filters of iteration i use model key (c, mix(seed, 2i)) and resampling
// key (c, mix(seed, 2i + 1)), so every iteration draws fresh particles.
//
// The proposal is a hook: the reference's `update` evaluations take the
// chain's RNG and a copy of the parameters, change the copy and return their
// log proposal ratio (algorithm/pmcmc.hpp:116-145).  Here a proposal
// callback gets chain c's four words of counter 2i as its randomness, the
// copy of (phi, sx, sy) to change in place, and returns
// log q(theta | theta') - log q(theta' | theta); the built-in Gaussian random
// walk is the callback used when none is given (ratio 0).
#include <cmath>
#include <limits>
#include <vector>

#include "common.cuh"

namespace {

// Philox4x32-10 block for counter (ctr, 0): the same stream as the device
// generator.
void philox_host(uint32_t k0, uint32_t k1, uint64_t ctr, uint32_t out[4])
{
    uint32_t s0 = static_cast<uint32_t>(ctr), s1 = static_cast<uint32_t>(ctr >> 32), s2 = 0, s3 = 0;
    for (int r = 0; r < 10; ++r) {
        const uint64_t p2 = static_cast<uint64_t>(s2) * 0xCD9E8D57u;
        const uint64_t p0 = static_cast<uint64_t>(s0) * 0xD2511F53u;
        s0 = k0 ^ s1 ^ static_cast<uint32_t>(p2 >> 32);
        s1 = static_cast<uint32_t>(p2);
        s2 = k1 ^ s3 ^ static_cast<uint32_t>(p0 >> 32);
        s3 = static_cast<uint32_t>(p0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = s0;
    out[1] = s1;
    out[2] = s2;
    out[3] = s3;
}

// 32-bit finaliser of MurmurHash3 (a bijection): spreads (seed, iteration)
// over the key space
uint32_t mix32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x85EBCA6Bu;
    x ^= x >> 13;
    x *= 0xC2B2AE35u;
    x ^= x >> 16;
    return x;
}

constexpr double kTwoPi = 6.283185307179586476925286766559;

}  // namespace

namespace {

struct RandomWalk {
    const double *step;
};

// the built-in proposal: theta + step * (three standard normals by
// Box-Muller from the four words), symmetric
double random_walk(size_t, size_t, const uint32_t w[4], double *theta, void *user)
{
    const double *step = static_cast<const RandomWalk *>(user)->step;
    const double r0 = std::sqrt(-2.0 * std::log((w[0] + 1.0) * 0x1p-32));
    const double a0 = kTwoPi * (w[1] * 0x1p-32);
    const double r1 = std::sqrt(-2.0 * std::log((w[2] + 1.0) * 0x1p-32));
    const double a1 = kTwoPi * (w[3] * 0x1p-32);
    const double z[3] = {r0 * std::cos(a0), r0 * std::sin(a0), r1 * std::cos(a1)};
    for (int k = 0; k < 3; ++k) theta[k] = theta[k] + step[k] * z[k];
    return 0.0;
}

}  // namespace

extern "C" int mckl_b200_pmcmc_ar1(size_t C, const size_t *N, size_t T, const double *y, const double *theta0,
    const double *step, mckl_b200_log_prior_t prior, void *user, size_t iters, uint32_t seed, int fp64,
    double threshold, double *theta_out, double *loglik_out, uint32_t *accepted, void *stream)
{
    MB_CHECK_ARG(step != nullptr, "null step");
    RandomWalk rw{step};
    return mckl_b200_pmcmc_ar1_proposal(C, N, T, y, theta0, random_walk, &rw, prior, user, iters, seed, fp64,
        threshold, theta_out, loglik_out, accepted, stream);
}

extern "C" int mckl_b200_pmcmc_ar1_proposal(size_t C, const size_t *N, size_t T, const double *y,
    const double *theta0, mckl_b200_proposal_t proposal, void *proposal_user, mckl_b200_log_prior_t prior,
    void *user, size_t iters, uint32_t seed, int fp64, double threshold, double *theta_out, double *loglik_out,
    uint32_t *accepted, void *stream)
{
    using namespace mckl_b200;
    MB_CHECK_ARG(C > 0 && N && T > 0 && y && theta0 && proposal && prior && iters > 0, "bad arguments");
    MB_CHECK_ARG(theta_out && loglik_out && accepted, "null output");
    MB_CHECK_ARG(fp64 == 0 || fp64 == 1, "fp64: 0 (FP32 moves) or 1 (FP64)");
    std::vector<double> lq(C, 0.0);
    std::vector<double> phi(C), sx(C), sy(C), lp(C), ll(C), th(3 * C), thp(3 * C);
    std::vector<uint32_t> mk(2 * C), rk(2 * C), nres(C);
    std::vector<char> valid(C);
    auto keys = [&](size_t it) {
        for (size_t c = 0; c < C; ++c) {
            mk[2 * c] = static_cast<uint32_t>(c);
            mk[2 * c + 1] = mix32(seed ^ static_cast<uint32_t>(2 * it));
            rk[2 * c] = static_cast<uint32_t>(c);
            rk[2 * c + 1] = mix32(seed ^ static_cast<uint32_t>(2 * it + 1));
        }
    };
    for (size_t c = 0; c < C; ++c) {
        for (int k = 0; k < 3; ++k) th[3 * c + k] = theta0[3 * c + k];
        phi[c] = th[3 * c];
        sx[c] = th[3 * c + 1];
        sy[c] = th[3 * c + 2];
        lp[c] = prior(&th[3 * c], user);
        MB_CHECK_ARG(std::isfinite(lp[c]), "the prior density is zero at a starting point");
    }
    keys(0);
    mckl_b200_batched_t *b = nullptr;
    int rc = mckl_b200_batched_create(&b, C, N, T, y, phi.data(), sx.data(), sy.data(), mk.data(), rk.data(),
        threshold, fp64);
    if (rc != MCKL_B200_OK) return rc;
    auto run = [&]() {
        int r = mckl_b200_batched_run_graph(b, stream);
        if (r == MCKL_B200_OK) r = mckl_b200_batched_results(b, ll.data(), nres.data(), stream);
        return r;
    };
    // iteration 0: the filters at the starting points
    rc = run();
    std::vector<double> ll_cur(ll);
    for (size_t c = 0; c < C; ++c) accepted[c] = 0;
    for (size_t it = 0; rc == MCKL_B200_OK && it < iters; ++it) {
        if (it > 0) {
            for (size_t c = 0; c < C; ++c) {
                uint32_t w[4];
                philox_host(seed, static_cast<uint32_t>(c), 2 * it, w);
                for (int k = 0; k < 3; ++k) thp[3 * c + k] = th[3 * c + k];
                lq[c] = proposal(c, it, w, &thp[3 * c], proposal_user);
                const bool in_model = thp[3 * c] * thp[3 * c] < 1 && thp[3 * c + 1] > 0 && thp[3 * c + 2] > 0;
                lp[c] = in_model ? prior(&thp[3 * c], user) : -std::numeric_limits<double>::infinity();
                valid[c] = std::isfinite(lp[c]) && std::isfinite(lq[c]) ? 1 : 0;
                // a proposal outside the support is rejected without a filter
                // run: its filter reruns the current parameters
                const double *src = valid[c] ? &thp[3 * c] : &th[3 * c];
                phi[c] = src[0];
                sx[c] = src[1];
                sy[c] = src[2];
            }
            keys(it);
            rc = mckl_b200_batched_set_params(b, phi.data(), sx.data(), sy.data(), stream);
            if (rc == MCKL_B200_OK) rc = mckl_b200_batched_set_keys(b, mk.data(), rk.data(), stream);
            if (rc == MCKL_B200_OK) rc = run();
            if (rc != MCKL_B200_OK) break;
            for (size_t c = 0; c < C; ++c) {
                if (!valid[c]) continue;
                uint32_t w[4];
                philox_host(seed, static_cast<uint32_t>(c), 2 * it + 1, w);
                const double logu = std::log((w[0] + 0.5) * 0x1p-32);
                const double lp_old = prior(&th[3 * c], user);
                double prob = -lp_old - ll_cur[c];
                prob += lq[c];  // the proposal's log ratio (the reference's sum of evaluations)
                prob += lp[c];
                prob += ll[c];
                if (logu < prob) {
                    for (int k = 0; k < 3; ++k) th[3 * c + k] = thp[3 * c + k];
                    ll_cur[c] = ll[c];
                    ++accepted[c];
                }
            }
        }
        for (size_t c = 0; c < C; ++c) {
            for (int k = 0; k < 3; ++k) theta_out[(it * C + c) * 3 + k] = th[3 * c + k];
            loglik_out[it * C + c] = ll_cur[c];
        }
    }
    mckl_b200_batched_destroy(b);
    return rc;
}
