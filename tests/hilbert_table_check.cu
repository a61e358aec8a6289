// Host-only check (no GPU): the two-level Hilbert state table gives the same keys as the bitwise encoder, and the
// top-down decoder gives the same node corners as the bitwise decoder.
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
    // the top-down decoder of node corners against the bitwise decoder, at every level
    const unsigned full[3] = {kMaxLevel, kMaxLevel, kMaxLevel};
    auto corner = [&](unsigned x, unsigned y, unsigned z)
    {
        uint64_t key = hilbert3(x, y, z, kMaxLevel);
        for (unsigned lvl = 0; lvl <= unsigned(kMaxLevel); ++lvl)
        {
            unsigned sh     = kMaxLevel - lvl;
            uint64_t start  = sh == unsigned(kMaxLevel) ? 0 : key & ~((uint64_t(1) << (3 * sh)) - 1);
            unsigned p[3], q[3];
            hilbertCorner(start, lvl, p);
            unhilbertKey(start, full, q);
            unsigned mask   = ~((1u << sh) - 1u);
            unsigned want[3] = {x & mask, y & mask, z & mask};
            ++n;
            bool ok = true;
            for (int d = 0; d < 3; ++d)
                ok = ok && p[d] == want[d] && (q[d] & mask) == want[d];
            if (!ok && bad++ < 5)
                std::printf("corner mismatch %u %u %u level %u: %u %u %u\n", x, y, z, lvl, p[0], p[1], p[2]);
        }
    };
    for (unsigned x : edge)
        for (unsigned y : edge)
            for (unsigned z : edge)
                corner(x, y, z);
    for (int i = 0; i < 200000; ++i)
        corner(unsigned(rng()) & M, unsigned(rng()) & M, unsigned(rng()) & M);
    std::printf("checked %ld keys, %ld mismatches\n", n, bad);
    return bad != 0;
}
