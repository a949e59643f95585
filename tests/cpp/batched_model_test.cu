// User models through the batched filters' model hook
// (include/mckl_b200_batched.cuh).
//
// `batched_model_test ar1 in out`: the AR(1) model written as a user would
// write it, run in FP32 and FP64; the test compares the log-likelihoods and
// resampling counts with the library's built-in AR(1) filters.  Input: int32
// F, int32 T, double threshold, uint64 n[F], double phi[F], sx[F], sy[F],
// uint32 mkey[2F], rkey[2F], double y[F (T + 1)].  Output: double
// loglik32[F], uint32 nres32[F], double loglik64[F], uint32 nres64[F].
//
// `batched_model_test offset in out`: a different model, x_0 ~ N(mu, sd0^2),
// x_t = mu + phi (x_{t-1} - mu) + sx e, y_t ~ N(x_t, sy^2), in FP64 on one
// filter; the test compares its log-likelihood with the exact (Kalman) one.
// Input: int32 T, uint32 mkey[2], rkey[2], uint64 N, double mu, phi, sx,
// sy, y[T + 1].  Output: double loglik, uint32 nres.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "mckl_b200_batched.cuh"

struct UserAr1 {
    struct Param {
        double phi, sx, sd0, lconst, hinv;
    };
    template <typename R>
    struct Dev {
        using M = mckl_b200::Math<R>;
        R phi, sx, sd0, lconst, hinv;
        __device__ Dev() {}
        __device__ explicit Dev(const Param &p)
            : phi(static_cast<R>(p.phi)), sx(static_cast<R>(p.sx)), sd0(static_cast<R>(p.sd0)),
              lconst(static_cast<R>(p.lconst)), hinv(static_cast<R>(p.hinv))
        {
        }
        __device__ R init(R e) const { return M::mul(sd0, e); }
        __device__ R move(R x, R e) const { return M::fma(phi, x, M::mul(sx, e)); }
        __device__ R log_density(R x, R y) const
        {
            const R r = M::sub(y, x);
            return M::fma(-M::mul(r, r), hinv, lconst);
        }
    };
};

struct OffsetAr1 {
    struct Param {
        double mu, phi, sx, sd0, lconst, hinv;
    };
    template <typename R>
    struct Dev {
        using M = mckl_b200::Math<R>;
        R mu, phi, sx, sd0, lconst, hinv;
        __device__ Dev() {}
        __device__ explicit Dev(const Param &p)
            : mu(static_cast<R>(p.mu)), phi(static_cast<R>(p.phi)), sx(static_cast<R>(p.sx)),
              sd0(static_cast<R>(p.sd0)), lconst(static_cast<R>(p.lconst)), hinv(static_cast<R>(p.hinv))
        {
        }
        __device__ R init(R e) const { return M::fma(sd0, e, mu); }
        __device__ R move(R x, R e) const { return M::add(mu, M::fma(phi, M::sub(x, mu), M::mul(sx, e))); }
        __device__ R log_density(R x, R y) const
        {
            const R r = M::sub(y, x);
            return M::fma(-M::mul(r, r), hinv, lconst);
        }
    };
};

template <typename T>
static bool get(FILE *f, T *p, size_t n)
{
    return fread(p, sizeof(T), n, f) == n;
}

static int offset_mode(const char *inp, const char *outp)
{
    FILE *in = fopen(inp, "rb");
    if (!in) return 3;
    int T = 0;
    uint32_t mkey[2], rkey[2];
    uint64_t N = 0;
    double v[4];
    if (!get(in, &T, 1) || !get(in, mkey, 2) || !get(in, rkey, 2) || !get(in, &N, 1) || !get(in, v, 4)) return 4;
    std::vector<double> y(T + 1);
    if (!get(in, y.data(), y.size())) return 5;
    fclose(in);
    const double mu = v[0], phi = v[1], sx = v[2], sy = v[3];
    OffsetAr1::Param par{mu, phi, sx, sx / std::sqrt(1 - phi * phi),
        -std::log(sy) - 0.5 * std::log(2 * 3.14159265358979323846), 0.5 / (sy * sy)};
    double ll = 0;
    uint32_t nr = 0;
    const cudaError_t e =
        mckl_b200::batched_run_model<OffsetAr1>(1, &N, &par, y.data(), T, mkey, rkey, 0.5, true, &ll, &nr);
    if (e != cudaSuccess) {
        fprintf(stderr, "batched_run_model: %s\n", cudaGetErrorString(e));
        return 6;
    }
    FILE *out = fopen(outp, "wb");
    if (!out) return 7;
    fwrite(&ll, sizeof(double), 1, out);
    fwrite(&nr, sizeof(uint32_t), 1, out);
    fclose(out);
    return 0;
}

int main(int argc, char **argv)
{
    if (argc != 4) return 2;
    if (std::string(argv[1]) == "offset") return offset_mode(argv[2], argv[3]);
    FILE *in = fopen(argv[2], "rb");
    if (!in) return 3;
    int F = 0, T = 0;
    double threshold = 0;
    if (!get(in, &F, 1) || !get(in, &T, 1) || !get(in, &threshold, 1)) return 4;
    std::vector<uint64_t> n(F);
    std::vector<double> phi(F), sx(F), sy(F), y(static_cast<size_t>(F) * (T + 1));
    std::vector<uint32_t> mkey(2 * F), rkey(2 * F);
    if (!get(in, n.data(), F) || !get(in, phi.data(), F) || !get(in, sx.data(), F) || !get(in, sy.data(), F) ||
        !get(in, mkey.data(), 2 * F) || !get(in, rkey.data(), 2 * F) || !get(in, y.data(), y.size()))
        return 5;
    fclose(in);
    // the parameters as the library's host code forms them for its AR(1) filters
    std::vector<UserAr1::Param> par(F);
    for (int f = 0; f < F; ++f)
        par[f] = {phi[f], sx[f], sx[f] / std::sqrt(1 - phi[f] * phi[f]),
            -std::log(sy[f]) - 0.5 * std::log(2 * 3.14159265358979323846), 0.5 / (sy[f] * sy[f])};
    std::vector<double> ll32(F), ll64(F);
    std::vector<uint32_t> nr32(F), nr64(F);
    cudaError_t e = mckl_b200::batched_run_model<UserAr1>(F, n.data(), par.data(), y.data(), T, mkey.data(),
        rkey.data(), threshold, false, ll32.data(), nr32.data());
    if (e == cudaSuccess)
        e = mckl_b200::batched_run_model<UserAr1>(F, n.data(), par.data(), y.data(), T, mkey.data(), rkey.data(),
            threshold, true, ll64.data(), nr64.data());
    if (e != cudaSuccess) {
        fprintf(stderr, "batched_run_model: %s\n", cudaGetErrorString(e));
        return 6;
    }
    FILE *out = fopen(argv[3], "wb");
    if (!out) return 7;
    fwrite(ll32.data(), sizeof(double), F, out);
    fwrite(nr32.data(), sizeof(uint32_t), F, out);
    fwrite(ll64.data(), sizeof(double), F, out);
    fwrite(nr64.data(), sizeof(uint32_t), F, out);
    fclose(out);
    return 0;
}
