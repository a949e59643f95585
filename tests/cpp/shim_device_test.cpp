// Device-side C++ API of include/mckl_b200.hpp: engines, distributions,
// Weight and resampling over device arrays.  tests/test_gpu_cpp.py compiles
// this file, runs it and compares what it writes (argv[1]) with the oracle.
#include <cstdio>
#include <vector>

#include "mckl_b200.hpp"

int main(int argc, char **argv)
{
    if (argc < 2) return 2;
    using namespace mckl_b200;
    FILE *f = std::fopen(argv[1], "wb");
    if (!f) return 2;
    try {
        Philox4x32 rng(42);
        DeviceBuffer<std::uint32_t> words(10000);
        rand(rng, 10000, words.data());
        std::vector<std::uint32_t> hw(10000);
        words.download(hw.data(), hw.size());
        std::fwrite(hw.data(), 4, hw.size(), f);

        DeviceBuffer<double> z(4097);
        normal_distribution(rng, 4097, z.data(), 0.0, 1.0);
        std::vector<double> hz(4097);
        z.download(hz.data(), hz.size());
        std::fwrite(hz.data(), 8, hz.size(), f);

        const std::size_t N = 3000;
        std::vector<double> v(N);
        for (std::size_t i = 0; i < N; ++i) v[i] = static_cast<double>((i * 7919) % 1000) / 100.0 - 5.0;
        DeviceBuffer<double> vd;
        vd.upload(v.data(), N);
        Weight w(N);
        w.set_log(vd.data());
        std::vector<double> hW(N);
        w.data();
        check_cuda(cudaMemcpy(hW.data(), w.data(), N * 8, cudaMemcpyDeviceToHost));
        std::fwrite(hW.data(), 8, N, f);

        Philox4x32 rrng(9);
        DeviceBuffer<std::uint64_t> rep(N), idx(N);
        ResampleSystematic()(N, N, rrng, w.data(), rep.data());
        resample_trans_rep_index(N, N, rep.data(), idx.data());
        std::vector<std::uint64_t> hi(N);
        idx.download(hi.data(), N);
        std::fwrite(hi.data(), 8, N, f);
        double ess = w.ess();
        std::fwrite(&ess, 8, 1, f);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    std::fclose(f);
    return 0;
}
