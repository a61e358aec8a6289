// Host-only check (no GPU): the two-level Hilbert state table gives the same keys as the bitwise encoder.
// Built and run by tests/test_hilbert_table.py.
#include <cstdio>
#include <random>

#include "common.cuh"

using namespace ryo;

int main()
{
    constexpr HilbertLut L = makeHilbertLut();
    std::mt19937_64 rng(7);
    long bad = 0, n = 0;
    auto test = [&](unsigned x, unsigned y, unsigned z)
    {
        uint64_t a = hilbert3(x, y, z, kMaxLevel), b = hilbert3Lut(x, y, z, L.two, L.one);
        ++n;
        if (a != b && bad++ < 5)
            std::printf("mismatch %u %u %u: %llx %llx\n", x, y, z, (unsigned long long)a, (unsigned long long)b);
    };
    const unsigned M = (1u << kMaxLevel) - 1;
    const unsigned edge[] = {0, 1, 2, 3, M, M - 1, M / 2, M / 2 + 1, 1u << 20, (1u << 20) - 1};
    for (unsigned x : edge)
        for (unsigned y : edge)
            for (unsigned z : edge)
                test(x, y, z);
    for (int i = 0; i < 2000000; ++i)
        test(unsigned(rng()) & M, unsigned(rng()) & M, unsigned(rng()) & M);
    for (unsigned x = 0; x < 64; ++x) // every combination of the lowest six bits
        for (unsigned y = 0; y < 64; ++y)
            for (unsigned z = 0; z < 64; ++z)
                test(x, y, z);
    std::printf("checked %ld keys, %ld mismatches\n", n, bad);
    return bad != 0;
}
