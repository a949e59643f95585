// The reference's own CounterEngine and distributions driven by the B200
// generators of include/mckl_b200.hpp, compared with the reference's own
// engines.  Built by oracle/Makefile (target shim) against the reference
// headers; run by tests/test_gpu_cpp.py.  Exit status 0 = all equal.
#include <mckl/random/aes.hpp>
#include <mckl/random/normal_distribution.hpp>
#include <mckl/random/philox.hpp>
#include <mckl/random/threefry.hpp>
#include <mckl/random/u01_distribution.hpp>

#include <cstdio>
#include <vector>

#include "mckl_b200.hpp"

template <typename RefEng, typename B200Eng>
int compare(const char *name, typename RefEng::key_type key)
{
    int bad = 0;
    RefEng a;
    B200Eng b;
    a.seed(key);
    b.seed(key);
    for (std::size_t n : {1ul, 3ul, 1000ul, 100000ul, 4000000ul}) {  // host and GPU fills
        std::vector<std::uint32_t> x(n), y(n);
        mckl::rand(a, n, x.data());
        mckl::rand(b, n, y.data());
        if (x != y) ++bad;
        std::vector<double> u(n), v(n);
        mckl::normal_distribution(a, n, u.data(), 0.5, 2.0);
        mckl::normal_distribution(b, n, v.data(), 0.5, 2.0);
        if (u != v) ++bad;
        mckl::u01_oo_distribution(a, n, u.data());
        mckl::u01_oo_distribution(b, n, v.data());
        if (u != v) ++bad;
        if (a() != b()) ++bad;
    }
    std::printf("%s: %s\n", name, bad ? "MISMATCH" : "equal");
    return bad;
}

int main()
{
    int bad = 0;
    bad += compare<mckl::Philox4x32, mckl::CounterEngine<std::uint32_t, mckl_b200::PhiloxGenerator4x32>>(
        "Philox4x32", {{42, 0}});
    bad += compare<mckl::Threefry4x64, mckl::CounterEngine<std::uint32_t, mckl_b200::Threefry4x64Generator>>(
        "Threefry4x64", {{42, 1, 2, 3}});
    bad += compare<mckl::ARS, mckl::CounterEngine<std::uint32_t, mckl_b200::ARSGenerator>>("ARS", {{42, 0, 0, 0}});
    return bad ? 1 : 0;
}
