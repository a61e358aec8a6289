/*
 * ryoanji-b200: device-side building blocks shared by all kernels.
 *
 * Key arithmetic, the mixed-dimension Hilbert curve (encode and decode), the coordinate box and warp helpers.
 * Everything that feeds an integer output (keys, node boxes, MAC radii) keeps the reference's rounding points
 * exactly: products and sums are issued with explicit round-to-nearest intrinsics so that the compiler cannot
 * contract them into FMAs, which the reference CPU build does not do either.
 */
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/ryoanji_b200.h"

namespace ryo
{

constexpr int kMaxLevel    = 21;                     // 64-bit SFC keys: 21 octal digits
constexpr uint64_t kKeyEnd = uint64_t(1) << 63;      // end of the key range, also the "remove" marker key
constexpr int kWarp        = 32;

// ------------------------------------------------------------------------------------------------ error handling

struct CudaError
{
    cudaError_t err;
    const char* what;
};

#define RYO_CUDA(call)                                                                                                 \
    do                                                                                                                 \
    {                                                                                                                  \
        cudaError_t e_ = (call);                                                                                       \
        if (e_ != cudaSuccess) throw ::ryo::CudaError{e_, #call};                                                      \
    } while (0)

//! counts every kernel launch of the library (reported by ryo_kernel_launches)
uint64_t& launchCounter();

#define RYO_LAUNCH_CHECK()                                                                                             \
    do                                                                                                                 \
    {                                                                                                                  \
        ++::ryo::launchCounter();                                                                                      \
        RYO_CUDA(cudaGetLastError());                                                                                  \
    } while (0)

inline unsigned ceilDiv(size_t a, size_t b) { return unsigned((a + b - 1) / b); }

// ------------------------------------------------------------------------------------------------ key arithmetic

__host__ __device__ inline int clz64(uint64_t v)
{
#ifdef __CUDA_ARCH__
    return __clzll((long long)v);
#else
    return v ? __builtin_clzll(v) : 64;
#endif
}

//! key range covered by one node on @p level
__host__ __device__ inline uint64_t nodeRange(unsigned level) { return uint64_t(1) << (3 * (kMaxLevel - level)); }

//! level of a power-of-8 key range
__host__ __device__ inline unsigned rangeLevel(uint64_t range) { return unsigned(clz64(range - 1) - 1) / 3; }

//! number of leading key bits (excluding the unused top bit) shared by two keys
__host__ __device__ inline int commonBits(uint64_t a, uint64_t b) { return clz64(a ^ b) - 1; }

__host__ __device__ inline unsigned octalDigit(uint64_t key, unsigned level)
{
    return unsigned(key >> (3 * (kMaxLevel - level))) & 7u;
}

//! Warren-Salmon placeholder-bit prefix: the first @p len key bits behind a leading 1
__host__ __device__ inline uint64_t encodePrefix(uint64_t key, int len)
{
    return (key >> (63 - len)) | (uint64_t(1) << len);
}

__host__ __device__ inline int prefixLength(uint64_t prefix) { return 63 - clz64(prefix); }

__host__ __device__ inline uint64_t prefixStart(uint64_t prefix)
{
    int len = prefixLength(prefix);
    return (prefix ^ (uint64_t(1) << len)) << (63 - len);
}

//! position (level) of the last non-zero octal digit, kMaxLevel for 0
__host__ __device__ inline int lastNonZeroLevel(uint64_t key)
{
#ifdef __CUDA_ARCH__
    return key ? kMaxLevel - (__ffsll((long long)key) - 1) / 3 : kMaxLevel;
#else
    return key ? kMaxLevel - __builtin_ctzll(key) / 3 : kMaxLevel;
#endif
}

/*! @brief the minimal sequence of aligned octree nodes covering [a, b), written to @p out if not null
 *
 * Nodes grow while walking up from a's last non-zero digit to the first digit where a and b differ, then shrink
 * towards b. Returns the number of nodes. Same node sequence as cstone's spanSfcRange (cstone/sfc/common.hpp:412-451).
 */
__host__ __device__ inline int spanKeyRange(uint64_t a, uint64_t b, uint64_t* out)
{
    int num      = 0;
    int diffLvl  = (clz64(a ^ b) + 3 - 1) / 3;
    for (int lvl = lastNonZeroLevel(a); lvl > diffLvl; --lvl)
    {
        int reps = (8 - int(octalDigit(a, lvl))) % 8;
        for (int r = 0; r < reps; ++r)
        {
            if (out) out[num] = a;
            ++num;
            a += nodeRange(lvl);
        }
    }
    int bLast = lastNonZeroLevel(b);
    for (int lvl = diffLvl; lvl <= bLast; ++lvl)
    {
        int reps = int(octalDigit(b, lvl)) - int(octalDigit(a, lvl));
        for (int r = 0; r < reps; ++r)
        {
            if (out) out[num] = a;
            ++num;
            a += nodeRange(lvl);
        }
    }
    return num;
}

// ------------------------------------------------------------------------------------------------ Hilbert curve

/*! 3D Hilbert index of the @p order low bits of (px, py, pz). The digit of an octant and the re-orientation of the
 *  remaining bits per level define the curve of cstone/sfc/hilbert.hpp:43-94; the same curve is required for
 *  bit-identical keys. */
__host__ __device__ inline uint64_t hilbert3(unsigned px, unsigned py, unsigned pz, int order)
{
    // octant (x<<2|y<<1|z) -> Hilbert digit {0,1,3,2,7,6,4,5}, packed 3 bits per entry
    constexpr uint32_t digitOf = 0u | (1u << 3) | (3u << 6) | (2u << 9) | (7u << 12) | (6u << 15) | (4u << 18) |
                                 (5u << 21);
    uint64_t key = 0;
    for (int lvl = order - 1; lvl >= 0; --lvl)
    {
        unsigned bx = (px >> lvl) & 1u, by = (py >> lvl) & 1u, bz = (pz >> lvl) & 1u;
        unsigned oct = (bx << 2) | (by << 1) | bz;
        key          = (key << 3) | ((digitOf >> (3 * oct)) & 7u);
        unsigned nby = by ^ 1u, nbz = bz ^ 1u;
        px ^= 0u - (bx & (nby | bz));
        py ^= 0u - ((bx & (by | bz)) | (by & nbz));
        pz ^= 0u - ((bx & nby & nbz) | (by & nbz));
        if (bz)
        {
            unsigned t = px;
            px         = py;
            py         = pz;
            pz         = t;
        }
        else if (!by)
        {
            unsigned t = px;
            px         = pz;
            pz         = t;
        }
    }
    return key;
}

/*! hilbert3 as a state machine over 2 levels per step. The per-level update of hilbert3 is a signed permutation of
 *  the axes, so the transform accumulated down the levels is one of 48 states (axis permutation, flip bits). For
 *  every state and every pair of octants (original coordinate bits of two levels) the table holds the two Hilbert
 *  digits and the next state, generated at compile time by applying hilbert3's rules; the keys are therefore
 *  identical to hilbert3's. */
struct HilbertLut
{
    uint16_t two[48 * 64]; // (digit pair) | (next state << 6)
    uint16_t one[48 * 8];  // (digit) | (next state << 3)
};

constexpr int kHilbertPerms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

constexpr int hilbertPermIndex(int a, int b)
{
    for (int i = 0; i < 6; ++i)
        if (kHilbertPerms[i][0] == a && kHilbertPerms[i][1] == b) return i;
    return 0;
}

//! one level of hilbert3 for state @p state (perm index * 8 + flips x4 y2 z1) and original octant bits @p oct
constexpr void hilbertStep(int state, unsigned oct, unsigned& digit, int& next)
{
    const int* perm = kHilbertPerms[state / 8];
    unsigned fl[3]  = {unsigned(state >> 2) & 1u, unsigned(state >> 1) & 1u, unsigned(state) & 1u};
    unsigned ob[3]  = {(oct >> 2) & 1u, (oct >> 1) & 1u, oct & 1u};
    unsigned bx = ob[perm[0]] ^ fl[0], by = ob[perm[1]] ^ fl[1], bz = ob[perm[2]] ^ fl[2];
    constexpr unsigned digitOf[8] = {0, 1, 3, 2, 7, 6, 4, 5};
    digit        = digitOf[(bx << 2) | (by << 1) | bz];
    unsigned nby = by ^ 1u, nbz = bz ^ 1u;
    unsigned f[3] = {fl[0] ^ (bx & (nby | bz)), fl[1] ^ ((bx & (by | bz)) | (by & nbz)),
                     fl[2] ^ ((bx & nby & nbz) | (by & nbz))};
    int np[3]     = {perm[0], perm[1], perm[2]};
    unsigned nf[3] = {f[0], f[1], f[2]};
    if (bz)
    {
        np[0] = perm[1], np[1] = perm[2], np[2] = perm[0];
        nf[0] = f[1], nf[1] = f[2], nf[2] = f[0];
    }
    else if (!by)
    {
        np[0] = perm[2], np[2] = perm[0];
        nf[0] = f[2], nf[2] = f[0];
    }
    next = hilbertPermIndex(np[0], np[1]) * 8 + int((nf[0] << 2) | (nf[1] << 1) | nf[2]);
}

constexpr HilbertLut makeHilbertLut()
{
    HilbertLut t{};
    for (int st = 0; st < 48; ++st)
    {
        for (unsigned o = 0; o < 8; ++o)
        {
            unsigned d = 0;
            int nx     = 0;
            hilbertStep(st, o, d, nx);
            t.one[st * 8 + o] = uint16_t(d | (unsigned(nx) << 3));
        }
        for (unsigned o = 0; o < 64; ++o)
        {
            unsigned d1 = 0, d2 = 0;
            int s1 = 0, s2 = 0;
            hilbertStep(st, o >> 3, d1, s1);
            hilbertStep(s1, o & 7u, d2, s2);
            t.two[st * 64 + o] = uint16_t(((d1 << 3) | d2) | (unsigned(s2) << 6));
        }
    }
    return t;
}

/*! the inverse of the state table: for every state and Hilbert digit, the original octant bits and the next state.
 *  A key then decodes from its top level down, one lookup per level, and a node's corner needs only the node's own
 *  levels. */
struct HilbertDecodeLut
{
    uint16_t one[48 * 8]; // (octant bits x4 y2 z1) | (next state << 3)
};

constexpr HilbertDecodeLut makeHilbertDecodeLut()
{
    HilbertDecodeLut t{};
    for (int st = 0; st < 48; ++st)
        for (unsigned o = 0; o < 8; ++o)
        {
            unsigned d = 0;
            int nx     = 0;
            hilbertStep(st, o, d, nx);
            t.one[st * 8 + d] = uint16_t(o | (unsigned(nx) << 3));
        }
    return t;
}

#ifdef __CUDACC__
static __device__ const HilbertDecodeLut kHilbertDecodeDev = makeHilbertDecodeLut();
#endif

/*! integer coordinates of the lower corner of the node at octree level @p levels whose keys start at @p key, for a
 *  box whose three axes use all kMaxLevel levels: the top @p levels bits of each coordinate, lower bits zero */
__host__ __device__ inline void hilbertCorner(uint64_t key, unsigned levels, unsigned p[3])
{
#ifdef __CUDA_ARCH__
    const uint16_t* dec = kHilbertDecodeDev.one;
#else
    static constexpr HilbertDecodeLut host = makeHilbertDecodeLut();
    const uint16_t* dec = host.one;
#endif
    unsigned st = 0, x = 0, y = 0, z = 0;
    for (unsigned l = 0; l < levels; ++l)
    {
        unsigned e = dec[st * 8 + (unsigned(key >> (3 * (kMaxLevel - 1 - l))) & 7u)];
        x          = (x << 1) | ((e >> 2) & 1u);
        y          = (y << 1) | ((e >> 1) & 1u);
        z          = (z << 1) | (e & 1u);
        st         = e >> 3;
    }
    const unsigned sh = kMaxLevel - levels;
    p[0]              = x << sh;
    p[1]              = y << sh;
    p[2]              = z << sh;
}

//! bits 0..20 of v spread to every third bit (v_i at bit 3 i)
__host__ __device__ inline uint64_t spreadBits3(uint32_t v)
{
    uint64_t x = v & 0x1fffffu;
    x          = (x | (x << 32)) & 0x1f00000000ffffull;
    x          = (x | (x << 16)) & 0x1f0000ff0000ffull;
    x          = (x | (x << 8)) & 0x100f00f00f00f00full;
    x          = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x          = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

//! hilbert3(px, py, pz, kMaxLevel) through the tables (level 20 first, two levels per lookup, level 0 last)
__host__ __device__ inline uint64_t hilbert3Lut(unsigned px, unsigned py, unsigned pz, const uint16_t* two,
                                                const uint16_t* one)
{
    uint64_t m   = (spreadBits3(px) << 2) | (spreadBits3(py) << 1) | spreadBits3(pz);
    uint64_t key = 0;
    unsigned st  = 0;
#pragma unroll
    for (int lvl = kMaxLevel - 1; lvl >= 2; lvl -= 2)
    {
        unsigned e = two[st * 64 + (unsigned(m >> (3 * (lvl - 1))) & 63u)];
        key        = (key << 6) | (e & 63u);
        st         = e >> 6;
    }
    unsigned e = one[st * 8 + unsigned(m & 7u)];
    return (key << 3) | (e & 7u);
}

__host__ __device__ inline uint64_t hilbert2(unsigned px, unsigned py, int order)
{
    uint64_t key = 0;
    for (int lvl = order - 1; lvl >= 0; --lvl)
    {
        unsigned bx = (px >> lvl) & 1u, by = (py >> lvl) & 1u;
        if (by == 0)
        {
            unsigned t = px;
            px         = py ^ (0u - bx);
            py         = t ^ (0u - bx);
        }
        key = 4 * key + 2 * bx + (bx ^ by);
    }
    return key;
}

//! descending sort of the axis bit depths with the axis permutation (hilbert.hpp:128-157)
__host__ __device__ inline void sortAxes(unsigned b[3], int p[3])
{
    auto cswap = [&](int i, int j)
    {
        if (b[i] < b[j])
        {
            unsigned t = b[i];
            b[i]       = b[j];
            b[j]       = t;
            int tp     = p[i];
            p[i]       = p[j];
            p[j]       = tp;
        }
    };
    cswap(0, 1);
    cswap(0, 2);
    cswap(1, 2);
}

//! mixed-dimension Hilbert key for boxes whose axes have different bit depths (hilbert.hpp:117-244)
__host__ __device__ inline uint64_t hilbertKey(unsigned px, unsigned py, unsigned pz, const unsigned bits[3])
{
    if (bits[0] == kMaxLevel && bits[1] == kMaxLevel && bits[2] == kMaxLevel) { return hilbert3(px, py, pz, kMaxLevel); }
    unsigned b[3] = {bits[0], bits[1], bits[2]};
    int p[3]      = {0, 1, 2};
    sortAxes(b, p);
    uint64_t c[3] = {px, py, pz};
    uint64_t s[3] = {c[p[0]], c[p[1]], c[p[2]]};
    uint64_t key  = 0;
    if (b[0] > b[1])
    {
        int n = b[0] - b[1];
        for (int i = 0; i < n; ++i)
        {
            unsigned bit = b[0] - i - 1;
            key |= ((s[0] >> bit) & 1) << (3 * bit);
        }
        s[0] &= (uint64_t(1) << b[1]) - 1;
        b[0] -= n;
    }
    if (b[1] > b[2])
    {
        int n          = b[1] - b[2];
        uint64_t mask  = (uint64_t(1) << b[2]) - 1;
        uint64_t key2d = hilbert2(unsigned(s[0] >> b[2]), unsigned(s[1] >> b[2]), n);
        uint64_t lx = s[0] & mask, ly = s[1] & mask;
        for (int lvl = n - 1; lvl >= 0; --lvl)
        {
            unsigned q  = unsigned(key2d >> (2 * lvl)) & 3u;
            unsigned qx = (q >> 1) & 1u;
            unsigned qy = qx ^ (q & 1u);
            if (qy == 0)
            {
                uint64_t t = lx;
                lx         = ly;
                ly         = t;
                if (qx == 1)
                {
                    lx = mask - lx;
                    ly = mask - ly;
                }
            }
        }
        for (int i = 0; i < n; ++i)
            key |= ((key2d >> (2 * (n - 1 - i))) & 3) << (3 * (b[1] - 1 - i));
        s[0] = lx;
        s[1] = ly;
        b[0] -= n;
        b[1] -= n;
    }
    return key | hilbert3(unsigned(s[0]), unsigned(s[1]), unsigned(s[2]), b[2]);
}

__host__ __device__ inline void unhilbert3(uint64_t key, unsigned order, unsigned& ox, unsigned& oy, unsigned& oz)
{
    unsigned px = 0, py = 0, pz = 0;
    for (unsigned lvl = 0; lvl < order; ++lvl)
    {
        unsigned oct = unsigned(key >> (3 * lvl)) & 7u;
        unsigned bx = oct >> 2, by = (oct >> 1) & 1u, bz = oct & 1u;
        if (by ^ bz)
        {
            unsigned t = px;
            px         = pz;
            pz         = py;
            py         = t;
        }
        else if ((!bx && !by && !bz) || (bx && by && bz))
        {
            unsigned t = px;
            px         = pz;
            pz         = t;
        }
        unsigned mask = (1u << lvl) - 1;
        unsigned nbx = bx ^ 1u, nby = by ^ 1u, nbz = bz ^ 1u;
        px ^= mask & (0u - (bx & (by | bz)));
        py ^= mask & (0u - ((bx & (nby | nbz)) | (nbx & by & bz)));
        pz ^= mask & (0u - ((bx & nby & nbz) | (by & bz)));
        px |= bx << lvl;
        py |= (bx ^ by) << lvl;
        pz |= (by ^ bz) << lvl;
    }
    ox = px;
    oy = py;
    oz = pz;
}

__host__ __device__ inline void unhilbert2(uint64_t key, unsigned order, unsigned& ox, unsigned& oy)
{
    unsigned x = 0, y = 0;
    for (unsigned lvl = 0; lvl < 2 * order; lvl += 2)
    {
        unsigned sa = unsigned(key >> (lvl + 1)) & 1u;
        unsigned sb = unsigned(key >> lvl) & 1u;
        if ((sa ^ sb) == 0)
        {
            unsigned t = x;
            x          = y ^ (0u - sa);
            y          = t ^ (0u - sa);
        }
        x = (x >> 1) | (sa << 31);
        y = (y >> 1) | ((sa ^ sb) << 31);
    }
    ox = x >> (32 - order);
    oy = y >> (32 - order);
}

//! inverse of hilbertKey (hilbert.hpp:362-471)
__host__ __device__ inline void unhilbertKey(uint64_t key, const unsigned bits[3], unsigned out[3])
{
    unsigned b[3] = {bits[0], bits[1], bits[2]};
    int p[3]      = {0, 1, 2};
    sortAxes(b, p);
    uint64_t c[3] = {0, 0, 0};
    if (b[0] > b[1])
    {
        int n = b[0] - b[1];
        for (int i = 0; i < n; ++i)
        {
            unsigned bit = b[0] - 1 - i;
            c[0] |= ((key >> (3 * bit)) & 1) << bit;
        }
        key &= (uint64_t(1) << (3 * b[1])) - 1;
    }
    uint64_t key2d = 0;
    if (b[1] > b[2])
    {
        int n = b[1] - b[2];
        for (int i = 0; i < n; ++i)
            key2d |= ((key >> (3 * (b[1] - 1 - i))) & 3) << (2 * (n - 1 - i));
        unsigned ux, uy;
        unhilbert2(key2d, n, ux, uy);
        uint64_t nm = (uint64_t(1) << n) - 1;
        c[0] |= (uint64_t(ux) & nm) << b[2];
        c[1] |= (uint64_t(uy) & nm) << b[2];
        key &= (uint64_t(1) << (3 * b[2])) - 1;
    }
    unsigned shift = kMaxLevel - b[2];
    unsigned ux, uy, uz;
    unhilbert3(key << (3 * shift), kMaxLevel, ux, uy, uz);
    uint64_t x3 = ux >> shift, y3 = uy >> shift, z3 = uz >> shift;
    uint64_t maxc = (uint64_t(1) << b[2]) - 1;
    int n2        = b[1] > b[2] ? int(b[1] - b[2]) : 0;
    for (int i = 0; i < n2; ++i)
    {
        unsigned q  = unsigned(key2d >> (2 * i)) & 3u;
        unsigned qx = (q >> 1) & 1u;
        unsigned qy = qx ^ (q & 1u);
        if (qy == 0)
        {
            uint64_t t = x3;
            x3         = y3;
            y3         = t;
            if (qx == 1)
            {
                x3 = maxc - x3;
                y3 = maxc - y3;
            }
        }
    }
    c[0] |= x3;
    c[1] |= y3;
    c[2] |= z3;
    out[p[0]] = unsigned(c[0]);
    out[p[1]] = unsigned(c[1]);
    out[p[2]] = unsigned(c[2]);
}

//! digits above a short axis' depth may only use the axes present there (hilbert.hpp:516-552)
__host__ __device__ inline bool validMixDKey(uint64_t key, const unsigned bits[3])
{
    unsigned lo = bits[0], mid = bits[1], hi = bits[2];
    if (lo > mid) { unsigned t = lo; lo = mid; mid = t; }
    if (lo > hi) { unsigned t = lo; lo = hi; hi = t; }
    if (mid > hi) { unsigned t = mid; mid = hi; hi = t; }
    for (unsigned i = lo + 1; i <= unsigned(kMaxLevel); ++i)
    {
        unsigned d = unsigned(key >> (3 * (i - 1))) & 7u;
        if (i <= mid) { if (d > 3u) return false; }
        else if (i <= hi) { if (d > 1u) return false; }
    }
    return true;
}

// ------------------------------------------------------------------------------------------------ exact float ops

template<class T>
struct Fp;

template<>
struct Fp<float>
{
    __host__ __device__ static float mul(float a, float b)
    {
#ifdef __CUDA_ARCH__
        return __fmul_rn(a, b);
#else
        return a * b;
#endif
    }
    __host__ __device__ static float add(float a, float b)
    {
#ifdef __CUDA_ARCH__
        return __fadd_rn(a, b);
#else
        return a + b;
#endif
    }
    __host__ __device__ static float sub(float a, float b)
    {
#ifdef __CUDA_ARCH__
        return __fsub_rn(a, b);
#else
        return a - b;
#endif
    }
};

template<>
struct Fp<double>
{
    __host__ __device__ static double mul(double a, double b)
    {
#ifdef __CUDA_ARCH__
        return __dmul_rn(a, b);
#else
        return a * b;
#endif
    }
    __host__ __device__ static double add(double a, double b)
    {
#ifdef __CUDA_ARCH__
        return __dadd_rn(a, b);
#else
        return a + b;
#endif
    }
    __host__ __device__ static double sub(double a, double b)
    {
#ifdef __CUDA_ARCH__
        return __dsub_rn(a, b);
#else
        return a - b;
#endif
    }
};

//! x*x + (y*y + z*z), each product and sum rounded once (the reference's right-folded norm2)
template<class T>
__host__ __device__ inline T norm2Exact(T x, T y, T z)
{
    using F = Fp<T>;
    return F::add(F::mul(x, x), F::add(F::mul(y, y), F::mul(z, z)));
}

// ------------------------------------------------------------------------------------------------ coordinate box

/*! @brief the coordinate box in the form the kernels use (cstone/sfc/box.hpp:99-214)
 *
 * lo/len/inv follow Box<T>'s constructor; bits are the per-axis key depths of the mixed-dimension curve.
 */
template<class T>
struct DevBox
{
    T lo[3];
    T len[3];
    T inv[3];
    unsigned bits[3];
    int periodic;
};

template<class T>
inline DevBox<T> makeDevBox(const T* limits6, int periodic)
{
    DevBox<T> b;
    T maxDim = T(0);
    for (int d = 0; d < 3; ++d)
    {
        b.lo[d]  = limits6[2 * d];
        b.len[d] = limits6[2 * d + 1] - limits6[2 * d];
        b.inv[d] = T(1.) / (limits6[2 * d + 1] - limits6[2 * d]);
    }
    maxDim       = b.len[0] > b.len[1] ? b.len[0] : b.len[1];
    maxDim       = maxDim > b.len[2] ? maxDim : b.len[2];
    const T bias = T(0.5849625007211563); // 1 - log2(1 / 0.75): box.hpp:193
    for (int d = 0; d < 3; ++d)
    {
        T ratio   = maxDim / b.len[d];
        T l2      = sizeof(T) == 4 ? T(log2f(float(ratio))) : T(log2(double(ratio)));
        b.bits[d] = kMaxLevel - static_cast<unsigned>(floor(l2 + bias));
    }
    b.periodic = periodic;
    return b;
}

//! integer cell of x along one axis: floor(x*m) - floor(xmin*m) with exact fractional-part comparison (sfc.hpp:153-159)
template<class T>
__host__ __device__ inline int cellIndex(T x, T xmin, T m)
{
    using F = Fp<T>;
    T a = F::mul(x, m), b = F::mul(xmin, m);
    T fa = floor(a), fb = floor(b);
    return int(F::sub(fa, fb)) - int(F::sub(a, fa) < F::sub(b, fb));
}

//! integer cell coordinates of a point for its SFC key (sfc.hpp:161-207), clamped into the box
template<class T>
__host__ __device__ inline void pointCells(T x, T y, T z, const DevBox<T>& box, unsigned ic[3])
{
    const T v[3] = {x, y, z};
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
        T m   = Fp<T>::mul(T(1u << box.bits[d]), box.inv[d]);
        int c = cellIndex(v[d], box.lo[d], m);
        int cm = int((1u << box.bits[d]) - 1);
        c      = c < cm ? c : cm;
        ic[d]  = unsigned(c > 0 ? c : 0);
    }
}

//! SFC key of a point (sfc.hpp:161-207); coordinates outside the box are clamped into it
template<class T>
__host__ __device__ inline uint64_t pointKey(T x, T y, T z, const DevBox<T>& box)
{
    unsigned ic[3];
    pointCells(x, y, z, box, ic);
    return hilbertKey(ic[0], ic[1], ic[2], box.bits);
}

//! geometric centre and half size of the node with start key @p key on @p level (hilbert.hpp:562-585, box.hpp:357-381)
template<class T>
__host__ __device__ inline void nodeGeometry(uint64_t key, unsigned level, const DevBox<T>& box, T center[3], T size[3])
{
    using F = Fp<T>;
    if (!validMixDKey(key, box.bits))
    {
        for (int d = 0; d < 3; ++d)
        {
            center[d] = box.lo[d];
            size[d]   = T(0);
        }
        return;
    }
    unsigned fromRight = kMaxLevel - level;
    unsigned p[3];
    if (box.bits[0] == unsigned(kMaxLevel) && box.bits[1] == unsigned(kMaxLevel) && box.bits[2] == unsigned(kMaxLevel))
        hilbertCorner(key, level, p); // the node's levels only; the bits below are masked off next
    else
        unhilbertKey(key, box.bits, p);
    const T unit = T(1.) / T(1u << kMaxLevel);
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
        unsigned len = 1u << (box.bits[d] < fromRight ? box.bits[d] : fromRight);
        int i0       = int(p[d] & ~(len - 1));
        int i1       = i0 + int(len);
        T half       = F::mul(F::mul(F::mul(T(0.5), unit), box.len[d]), T(1u << (kMaxLevel - box.bits[d])));
        center[d]    = F::add(box.lo[d], F::mul(T(i1 + i0), half));
        size[d]      = F::mul(T(i1 - i0), half);
    }
}

//! squared MAC radius (2*max edge/theta + |com - geometric centre|)^2 of a node (macs.hpp:64-82)
template<class T>
__host__ __device__ inline T vecMacR2(uint64_t prefix, const T com[3], float invTheta, const DevBox<T>& box)
{
    using F      = Fp<T>;
    uint64_t key = prefixStart(prefix);
    unsigned lvl = unsigned(prefixLength(prefix)) / 3;
    T gc[3], gs[3];
    nodeGeometry(key, lvl, box, gc, gs);
    T s   = sqrt(norm2Exact(F::sub(com[0], gc[0]), F::sub(com[1], gc[1]), F::sub(com[2], gc[2])));
    T mx  = gs[0] > gs[1] ? gs[0] : gs[1];
    mx    = mx > gs[2] ? mx : gs[2];
    T l   = F::mul(T(2.0), mx);
    T mac = F::add(F::mul(l, T(invTheta)), s);
    return F::mul(mac, mac);
}

// ------------------------------------------------------------------------------------------------ warp helpers

//! order-preserving map of floats to unsigned integers (min/max by integer atomics)
__device__ __forceinline__ uint32_t orderedBits(float f)
{
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float orderedFloat(uint32_t u)
{
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ inline unsigned laneId() { return threadIdx.x & (kWarp - 1); }

__device__ inline unsigned lanemaskLt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template<class T>
__device__ inline T warpMin(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        T w = __shfl_xor_sync(0xffffffffu, v, o);
        v   = w < v ? w : v;
    }
    return v;
}

template<class T>
__device__ inline T warpMax(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        T w = __shfl_xor_sync(0xffffffffu, v, o);
        v   = w > v ? w : v;
    }
    return v;
}

template<class T>
__device__ inline T warpSum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

//! inclusive warp scan of ints
__device__ inline int warpInclusiveScan(int v)
{
    unsigned lane = laneId();
#pragma unroll
    for (int o = 1; o < kWarp; o <<= 1)
    {
        int w = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= unsigned(o)) v += w;
    }
    return v;
}

} // namespace ryo
