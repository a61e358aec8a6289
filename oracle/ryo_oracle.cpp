/*
 * TEST INFRASTRUCTURE ONLY — CPU oracle restating the reference algorithm of the single-GPU gravity path.
 * See ryo_oracle.h for the contract. Each function names the reference file:line it follows (paths relative to the
 * reference project root). Floating-point expressions keep the reference's evaluation order and rounding points,
 * and the file is compiled with -ffp-contract=off: the reference's default build has no FMA contraction.
 */
#include "ryo_oracle.h"

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

namespace
{

constexpr int kMaxLevel = 21;                         // 64-bit keys: 21 octal digits (cstone/tree/definitions.h:60-67)
constexpr uint64_t kKeyEnd = uint64_t(1) << 63;       // nodeRange(0)

// ------------------------------------------------------------------------------------------------ key arithmetic

inline int clz64(uint64_t v) { return v ? __builtin_clzll(v) : 64; }

//! octree level of a key range that is a power of 8 (cstone/sfc/common.hpp:146-151)
inline unsigned rangeLevel(uint64_t range) { return unsigned(clz64(range - 1) - 1) / 3; }

//! key range of a node on @p level (common.hpp:88-95)
inline uint64_t levelRange64(unsigned level) { return uint64_t(1) << (3 * (kMaxLevel - level)); }

//! octal digit of @p key on @p level, level 1 = most significant (common.hpp:288-292)
inline unsigned digitAt(uint64_t key, unsigned level) { return unsigned(key >> (3 * (kMaxLevel - level))) & 7u; }

//! Warren-Salmon placeholder-bit prefix of the first @p len key bits (common.hpp:162-170)
inline uint64_t toPrefix(uint64_t key, int len) { return (key >> (63 - len)) | (uint64_t(1) << len); }

inline int prefixLen(uint64_t prefix) { return 63 - clz64(prefix); }

inline uint64_t prefixKey(uint64_t prefix)
{
    int len = prefixLen(prefix);
    return (prefix ^ (uint64_t(1) << len)) << (63 - len);
}

// ------------------------------------------------------------------------------------------------ Hilbert curve

//! 3D Hilbert index of the @p order low bits of px, py, pz (cstone/sfc/hilbert.hpp:43-94)
uint64_t hilbert3(unsigned px, unsigned py, unsigned pz, int order)
{
    static const unsigned octantDigit[8] = {0, 1, 3, 2, 7, 6, 4, 5};
    uint64_t key                         = 0;
    for (int lvl = order - 1; lvl >= 0; --lvl)
    {
        unsigned bx = (px >> lvl) & 1u, by = (py >> lvl) & 1u, bz = (pz >> lvl) & 1u;
        key = (key << 3) | octantDigit[(bx << 2) | (by << 1) | bz];

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
        else if (!by) { std::swap(px, pz); }
    }
    return key;
}

//! 2D Hilbert index (hilbert.hpp:253-278)
uint64_t hilbert2(unsigned px, unsigned py, int order)
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

//! sort the three axis bit counts descending, tracking which axis went where (hilbert.hpp:128-157)
void sortAxes(unsigned b[3], int perm[3])
{
    auto cswap = [&](int i, int j)
    {
        if (b[i] < b[j])
        {
            std::swap(b[i], b[j]);
            std::swap(perm[i], perm[j]);
        }
    };
    cswap(0, 1);
    cswap(0, 2);
    cswap(1, 2);
}

//! mixed-dimension Hilbert key (hilbert.hpp:117-244)
uint64_t hilbertMixD(unsigned px, unsigned py, unsigned pz, unsigned bx, unsigned by, unsigned bz)
{
    unsigned b[3] = {bx, by, bz};
    int perm[3]   = {0, 1, 2};
    sortAxes(b, perm);
    uint64_t c[3] = {px, py, pz};
    uint64_t s[3] = {c[perm[0]], c[perm[1]], c[perm[2]]};
    uint64_t key  = 0;

    if (b[0] > b[1]) // one axis alone: one key bit per level
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
    if (b[1] > b[2]) // two axes: 2D Hilbert digits, then re-orient the low bits for the 3D part
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
                std::swap(lx, ly);
                if (qx == 1)
                {
                    lx = mask - lx;
                    ly = mask - ly;
                }
            }
        }
        for (int i = 0; i < n; ++i)
        {
            key |= ((key2d >> (2 * (n - 1 - i))) & 3) << (3 * (b[1] - 1 - i));
        }
        s[0] = lx;
        s[1] = ly;
        b[0] -= n;
        b[1] -= n;
    }
    return key | hilbert3(unsigned(s[0]), unsigned(s[1]), unsigned(s[2]), b[2]);
}

//! inverse of hilbert3 (hilbert.hpp:281-325)
void unhilbert3(uint64_t key, unsigned order, unsigned& ox, unsigned& oy, unsigned& oz)
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
        else if ((!bx && !by && !bz) || (bx && by && bz)) { std::swap(px, pz); }

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

//! inverse of hilbert2 (hilbert.hpp:328-359)
void unhilbert2(uint64_t key, unsigned order, unsigned& ox, unsigned& oy)
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

//! inverse of hilbertMixD (hilbert.hpp:362-471)
void unhilbertMixD(uint64_t key, unsigned bx, unsigned by, unsigned bz, uint64_t out[3])
{
    unsigned b[3] = {bx, by, bz};
    int perm[3]   = {0, 1, 2};
    sortAxes(b, perm);
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
        {
            key2d |= ((key >> (3 * (b[1] - 1 - i))) & 3) << (2 * (n - 1 - i));
        }
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
            std::swap(x3, y3);
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
    out[perm[0]] = c[0];
    out[perm[1]] = c[1];
    out[perm[2]] = c[2];
}

//! a key is a valid MixD key if the digits above the short axes' depths use only the present axes (hilbert.hpp:516-552)
bool validMixD(uint64_t key, unsigned bx, unsigned by, unsigned bz)
{
    unsigned b[3] = {bx, by, bz};
    std::sort(b, b + 3);
    for (unsigned i = b[0] + 1; i <= unsigned(kMaxLevel); ++i)
    {
        unsigned d = unsigned(key >> (3 * (i - 1))) & 7u;
        if (i <= b[1])
        {
            if (d > 3u) return false;
        }
        else if (i <= b[2])
        {
            if (d > 1u) return false;
        }
    }
    return true;
}

//! integer box of a node (hilbert.hpp:562-585)
std::array<int, 6> nodeIBox(uint64_t key, unsigned level, const unsigned bits[3])
{
    if (!validMixD(key, bits[0], bits[1], bits[2])) { return {0, 0, 0, 0, 0, 0}; }
    unsigned fromRight = kMaxLevel - level;
    unsigned lx = 1u << std::min(bits[0], fromRight), ly = 1u << std::min(bits[1], fromRight),
             lz = 1u << std::min(bits[2], fromRight);
    uint64_t p[3];
    unhilbertMixD(key, bits[0], bits[1], bits[2], p);
    unsigned ix = unsigned(p[0]) & ~(lx - 1), iy = unsigned(p[1]) & ~(ly - 1), iz = unsigned(p[2]) & ~(lz - 1);
    return {int(ix), int(ix + lx), int(iy), int(iy + ly), int(iz), int(iz + lz)};
}

// ------------------------------------------------------------------------------------------------ box and keys

template<class T>
struct BoxT
{
    T lo[3], len[3], inv[3];
    unsigned bits[3];
};

//! Box<T> constructor and computeBoxDimBits (cstone/sfc/box.hpp:113-128,190-198)
template<class T>
BoxT<T> makeBox(const T* b6)
{
    BoxT<T> b;
    for (int d = 0; d < 3; ++d)
    {
        b.lo[d]  = b6[2 * d];
        b.len[d] = b6[2 * d + 1] - b6[2 * d];
        b.inv[d] = T(1.) / (b6[2 * d + 1] - b6[2 * d]);
    }
    T maxDim   = std::max(std::max(b.len[0], b.len[1]), b.len[2]);
    const T bias = T(0.5849625007211563);
    for (int d = 0; d < 3; ++d)
    {
        unsigned red = static_cast<unsigned>(std::floor(std::log2(maxDim / b.len[d]) + bias));
        b.bits[d]    = kMaxLevel - red;
    }
    return b;
}

//! integer cell of x: floor(x*m) - floor(xmin*m) with the fractional parts compared (sfc.hpp:153-159)
template<class T>
int cellOf(T x, T xmin, T m)
{
    T a = x * m, b = xmin * m;
    T fa = std::floor(a), fb = std::floor(b);
    return int(fa - fb) - int(a - fa < b - fb);
}

//! sfc3D for Hilbert keys (sfc.hpp:161-207); out-of-box coordinates are clamped into the box
template<class T>
uint64_t keyOf(T x, T y, T z, const BoxT<T>& b)
{
    const T v[3] = {x, y, z};
    unsigned ic[3];
    for (int d = 0; d < 3; ++d)
    {
        T m    = T(1u << b.bits[d]) * b.inv[d];
        int c  = cellOf(v[d], b.lo[d], m);
        int cm = int((1u << b.bits[d]) - 1);
        c      = std::min(c, cm);
        ic[d]  = unsigned(std::max(c, 0));
    }
    return hilbertMixD(ic[0], ic[1], ic[2], b.bits[0], b.bits[1], b.bits[2]);
}

//! centre and half-size of an integer box (box.hpp:357-381)
template<class T>
void geoCenterSize(const std::array<int, 6>& ib, const BoxT<T>& b, T c[3], T s[3])
{
    const T unit = T(1.) / T(1u << kMaxLevel);
    for (int d = 0; d < 3; ++d)
    {
        T half = T(0.5) * unit * b.len[d] * T(1u << (kMaxLevel - b.bits[d]));
        c[d]   = b.lo[d] + T(ib[2 * d + 1] + ib[2 * d]) * half;
        s[d]   = T(ib[2 * d + 1] - ib[2 * d]) * half;
    }
}

//! (x*x) + ((y*y) + (z*z)): the reference's norm2 is a right fold (cstone/util/array.hpp:304-319)
template<class T>
inline T norm2(T x, T y, T z)
{
    return x * x + (y * y + z * z);
}

//! computeVecMacR2 (cstone/traversal/macs.hpp:64-82)
template<class T>
T vecMacR2(uint64_t prefix, const T com[3], float invTheta, const BoxT<T>& b)
{
    uint64_t key = prefixKey(prefix);
    unsigned lvl = unsigned(prefixLen(prefix)) / 3;
    auto ib      = nodeIBox(key, lvl, b.bits);
    T gc[3], gs[3];
    geoCenterSize(ib, b, gc, gs);
    T dx = com[0] - gc[0], dy = com[1] - gc[1], dz = com[2] - gc[2];
    T s   = std::sqrt(norm2(dx, dy, dz));
    T l   = T(2.0) * std::max(std::max(gs[0], gs[1]), gs[2]);
    T mac = l * invTheta + s;
    return mac * mac;
}

// ------------------------------------------------------------------------------------------------ cornerstone tree

uint32_t countIn(const uint64_t* k, size_t n, uint64_t a, uint64_t b)
{
    return uint32_t(std::lower_bound(k, k + n, b) - std::lower_bound(k, k + n, a));
}

//! split/merge decision of one leaf (cstone/tree/csarray.hpp:250-290)
int leafOp(const std::vector<uint64_t>& tree, size_t i, const std::vector<uint32_t>& counts, unsigned bucket)
{
    uint64_t node = tree[i];
    unsigned lvl  = rangeLevel(tree[i + 1] - node);
    int sib       = -1;
    if (lvl > 0)
    {
        sib = int(digitAt(node, lvl));
        if (tree[i - sib + 8] != tree[i - sib] + levelRange64(lvl - 1)) { sib = -1; }
    }
    if (sib > 0)
    {
        uint64_t parentCount = 0;
        for (int k = 0; k < 8; ++k)
            parentCount += counts[i - sib + k];
        if (parentCount <= bucket) { return 0; }
    }
    uint32_t c = counts[i];
    if (c > bucket * 512 && lvl + 3 < unsigned(kMaxLevel)) { return 4096; }
    if (c > bucket * 64 && lvl + 2 < unsigned(kMaxLevel)) { return 512; }
    if (c > bucket * 8 && lvl + 1 < unsigned(kMaxLevel)) { return 64; }
    if (c > bucket && lvl < unsigned(kMaxLevel)) { return 8; }
    return 1;
}

//! rebalance to the fixed point, starting from the root (csarray.hpp:331-440)
void buildLeaves(const uint64_t* keys, size_t n, unsigned bucket, std::vector<uint64_t>& tree,
                 std::vector<uint32_t>& counts)
{
    tree   = {0, kKeyEnd};
    counts = {uint32_t(n)};
    while (true)
    {
        size_t nn = tree.size() - 1;
        std::vector<int64_t> ops(nn + 1, 0);
        bool converged = true;
        for (size_t i = 0; i < nn; ++i)
        {
            ops[i] = leafOp(tree, i, counts, bucket);
            converged &= (ops[i] == 1);
        }
        std::exclusive_scan(ops.begin(), ops.end(), ops.begin(), int64_t(0));
        std::vector<uint64_t> next(size_t(ops[nn]) + 1);
        for (size_t i = 0; i < nn; ++i)
        {
            int64_t op   = ops[i + 1] - ops[i];
            uint64_t key = tree[i];
            unsigned lvl = rangeLevel(tree[i + 1] - key);
            if (op == 1) { next[ops[i]] = key; }
            else if (op > 1)
            {
                unsigned down = op == 8 ? 1 : op == 64 ? 2 : op == 512 ? 3 : 4;
                for (int64_t s = 0; s < op; ++s)
                    next[ops[i] + s] = key + uint64_t(s) * levelRange64(lvl + down);
            }
        }
        next.back() = tree.back();
        tree.swap(next);
        counts.resize(tree.size() - 1);
        for (size_t i = 0; i + 1 < tree.size(); ++i)
            counts[i] = countIn(keys, n, tree[i], tree[i + 1]);
        if (converged) { break; }
    }
}

//! digit weight for the binary-radix-tree to octree index map (cstone/sfc/common.hpp:307-312, octree.hpp:55-65)
int treeIndexWeight(uint64_t key, unsigned level)
{
    int w = 0;
    for (unsigned l = 1; l <= level + 1; ++l)
    {
        int d = int(digitAt(key, l));
        w += d >= 4 ? 7 - d : -d;
    }
    return w;
}

// ------------------------------------------------------------------------------------------------ multipoles

template<class T>
using Q8 = std::array<T, 8>;

//! P2M accumulate + finalize (ryoanji/nbody/cartesian_qpole.hpp:67-108)
template<class TA, class TX>
Q8<TA> p2m(const TX* x, const TX* y, const TX* z, const TX* m, size_t a, size_t b, const TA c[3])
{
    Q8<TA> q{};
    for (size_t i = a; i < b; ++i)
    {
        TA rx = TA(x[i]) - c[0], ry = TA(y[i]) - c[1], rz = TA(z[i]) - c[2];
        TA mi = TA(m[i]);
        q[0] += mi;
        q[1] += rx * rx * mi;
        q[2] += rx * ry * mi;
        q[3] += rx * rz * mi;
        q[4] += ry * ry * mi;
        q[5] += ry * rz * mi;
        q[6] += rz * rz * mi;
    }
    TA tr = q[1] + q[4] + q[6];
    q[7]  = tr;
    q[1]  = 3 * q[1] - tr;
    q[4]  = 3 * q[4] - tr;
    q[6]  = 3 * q[6] - tr;
    q[2] *= 3;
    q[3] *= 3;
    q[5] *= 3;
    return q;
}

//! parallel-axis shift of @p add by dX into @p out (cartesian_qpole.hpp:187-210)
template<class T>
void addShifted(Q8<T>& out, const T dX[3], const Q8<T>& add)
{
    T rx = dX[0], ry = dX[1], rz = dX[2];
    T rx2 = rx * rx, ry2 = ry * ry, rz2 = rz * rz;
    T r2  = T((rx2 + ry2 + rz2) * (1.0 / 3.0));
    T ml  = add[0] * 3;
    out[7] = out[7] + add[7] + ml * r2;
    out[0] += add[0];
    out[1] += add[1] + ml * (rx2 - r2);
    out[2] += add[2] + ml * rx * ry;
    out[3] += add[3] + ml * rx * rz;
    out[4] += add[4] + ml * (ry2 - r2);
    out[5] += add[5] + ml * ry * rz;
    out[6] += add[6] + ml * (rz2 - r2);
}

//! M2P (cartesian_qpole.hpp:152-176), in T, with 1/sqrt from @p rsq
template<class T, class R>
inline void m2p(T acc[4], const T t[3], const T c[3], const T* q, R rsq)
{
    T r[3]  = {t[0] - c[0], t[1] - c[1], t[2] - c[2]};
    T r2    = norm2(r[0], r[1], r[2]);
    T rm1   = rsq(r2);
    T rm2   = rm1 * rm1;
    T rm5   = rm2 * rm2 * rm1;
    T Qrx   = r[0] * q[1] + r[1] * q[2] + r[2] * q[3];
    T Qry   = r[0] * q[2] + r[1] * q[4] + r[2] * q[5];
    T Qrz   = r[0] * q[3] + r[1] * q[5] + r[2] * q[6];
    T rQr   = r[0] * Qrx + r[1] * Qry + r[2] * Qrz;
    T rQrAm = (T(-2.5) * rQr * rm5 - q[0] * rm1) * rm2;
    acc[0] += -(q[0] * rm1 + T(0.5) * rm5 * rQr);
    acc[1] += rm5 * Qrx + rQrAm * r[0];
    acc[2] += rm5 * Qry + rQrAm * r[1];
    acc[3] += rm5 * Qrz + rQrAm * r[2];
}

//! P2P (ryoanji/nbody/kernel.hpp:99-120), in T
template<class T, class R>
inline void p2p(T acc[4], const T ti[3], const T sj[3], T mj, T hi, T hj, R rsq)
{
    T dx = sj[0] - ti[0], dy = sj[1] - ti[1], dz = sj[2] - ti[2];
    T R2    = norm2(dx, dy, dz);
    T hij   = hi + hj;
    T hij2  = hij * hij;
    T R2eff = (R2 < hij2) ? hij2 : R2;
    T invR  = rsq(R2eff);
    T invR2 = invR * invR;
    T m3    = mj * invR * invR2;
    acc[0] -= m3 * R2;
    acc[1] += dx * m3;
    acc[2] += dy * m3;
    acc[3] += dz * m3;
}

const auto rsqF = [](float v) { return 1.0f / std::sqrt(v); };
const auto rsqD = [](double v) { return 1.0 / std::sqrt(v); };

// ------------------------------------------------------------------------------------------------ Ewald

struct EwaldK
{
    double h[3], hs[3], fc, fs;
};

struct EwaldParams
{
    double mroot[8];
    double center[3];
    int replicaShells, ewaldShells;
    double L, lCut, hCut, alphaScale, smallR;
    std::vector<EwaldK> ks;
};

//! ewaldEvalMultipoleComplete (ryoanji/nbody/ewald.hpp:90-115)
void ewaldEval(double acc[4], const double r[3], const double g[6], const double* M)
{
    double m   = M[0];
    double qxx = (M[1] + M[7]) / 3.0, qyy = (M[4] + M[7]) / 3.0, qzz = (M[6] + M[7]) / 3.0;
    double qxy = M[2] / 3.0, qxz = M[3] / 3.0, qyz = M[5] / 3.0;
    double Qr[3] = {r[0] * qxx + r[1] * qxy + r[2] * qxz, r[0] * qxy + r[1] * qyy + r[2] * qyz,
                    r[0] * qxz + r[1] * qyz + r[2] * qzz};
    double rQr = 0.5 * (r[0] * Qr[0] + r[1] * Qr[1] + r[2] * Qr[2]);
    double Qtr = 0.5 * M[7];
    double u   = -g[0] * m + g[1] * Qtr - g[2] * rQr;
    double f   = +g[1] * m - g[2] * Qtr + g[3] * rQr;
    acc[0] += u;
    for (int d = 0; d < 3; ++d)
        acc[d + 1] += g[2] * Qr[d] - r[d] * f;
}

//! ewaldInitParameters (ewald.hpp:133-198)
EwaldParams ewaldInit(const double* mroot, const double* center, int replicaShells, double L, double lCut,
                      double hCut, double alphaScale, double smallR)
{
    EwaldParams p{};
    std::copy(mroot, mroot + 8, p.mroot);
    std::copy(center, center + 3, p.center);
    if (lCut == 0 && hCut == 0 && alphaScale == 0) { replicaShells = 0; }
    p.replicaShells = replicaShells;
    p.ewaldShells   = std::max(int(std::ceil(lCut)), replicaShells);
    p.L             = L;
    p.lCut          = lCut;
    p.hCut          = hCut;
    p.alphaScale    = alphaScale;
    p.smallR        = smallR;
    if (p.ewaldShells == 0) { return p; }

    int hReps    = int(std::ceil(hCut));
    double alpha = alphaScale / L;
    double k4    = M_PI * M_PI / (alpha * alpha * L * L);
    for (int hx = -hReps; hx <= hReps; ++hx)
        for (int hy = -hReps; hy <= hReps; ++hy)
            for (int hz = -hReps; hz <= hReps; ++hz)
            {
                double hr[3] = {double(hx), double(hy), double(hz)};
                double h2    = norm2(hr[0], hr[1], hr[2]);
                if (h2 == 0 || h2 > hCut * hCut) { continue; }
                double g0 = std::exp(-k4 * h2) / (M_PI * h2 * L);
                double g1 = 2 * M_PI / L * g0;
                double g2 = -2 * M_PI / L * g1;
                double g3 = 2 * M_PI / L * g2;
                double g4 = -2 * M_PI / L * g3;
                double g5 = 2 * M_PI / L * g4;
                double gc[6] = {g0, 0.0, g2, 0.0, g4, 0.0};
                double gs[6] = {0.0, g1, 0.0, g3, 0.0, g5};
                double a1[4] = {0, 0, 0, 0}, a2[4] = {0, 0, 0, 0};
                ewaldEval(a1, hr, gc, mroot);
                ewaldEval(a2, hr, gs, mroot);
                EwaldK k;
                for (int d = 0; d < 3; ++d)
                {
                    k.h[d]  = hr[d];
                    k.hs[d] = 2 * M_PI / L * hr[d];
                }
                k.fc = a1[0];
                k.fs = a2[0];
                p.ks.push_back(k);
            }
    return p;
}

//! computeEwaldRealSpace + computeEwaldKSpace (ewald.hpp:200-327)
void ewaldTarget(const double pos[3], const EwaldParams& p, double acc[4])
{
    double L = p.L, alpha = p.alphaScale / L, alpha2 = alpha * alpha;
    double lCut2 = p.lCut * p.lCut * L * L;
    double k1    = M_PI / (alpha2 * L * L * L);
    double ka    = 2.0 * alpha / std::sqrt(M_PI);
    double smR2  = p.smallR * L * L;
    acc[0] += k1 * p.mroot[0];

    double r[3] = {pos[0] - p.center[0], pos[1] - p.center[1], pos[2] - p.center[2]};
    int S       = p.ewaldShells, Rs = p.replicaShells;
    for (int ix = -S; ix <= S; ++ix)
        for (int iy = -S; iy <= S; ++iy)
            for (int iz = -S; iz <= S; ++iz)
            {
                bool pre     = (-Rs <= ix && ix <= Rs) && (-Rs <= iy && iy <= Rs) && (-Rs <= iz && iz <= Rs);
                double R[3]  = {r[0] + ix * L, r[1] + iy * L, r[2] + iz * L};
                double R2    = norm2(R[0], R[1], R[2]);
                if (R2 > lCut2 && !pre) { continue; }
                double g[6];
                if (R2 < smR2 && ka > 0)
                {
                    double c0 = ka, a2 = R2 * alpha2;
                    g[0] = c0 * (a2 / 3.0 - 1.0);
                    c0 *= 2 * alpha2;
                    g[1] = c0 * (a2 / 5.0 - 1.0 / 3.0);
                    c0 *= 2 * alpha2;
                    g[2] = c0 * (a2 / 7.0 - 1.0 / 5.0);
                    c0 *= 2 * alpha2;
                    g[3] = c0 * (a2 / 9.0 - 1.0 / 7.0);
                    c0 *= 2 * alpha2;
                    g[4] = c0 * (a2 / 11.0 - 1.0 / 9.0);
                    c0 *= 2 * alpha2;
                    g[5] = c0 * (a2 / 13.0 - 1.0 / 11.0);
                }
                else
                {
                    double Rm = std::sqrt(R2), iR = 1.0 / Rm, iR2 = iR * iR;
                    double a   = std::exp(-R2 * alpha2) * ka * iR2;
                    double an  = 1.0;
                    double fn  = pre ? -std::erf(alpha * Rm) : std::erfc(alpha * Rm);
                    g[0] = fn * iR;
                    g[1] = g[0] * iR2 + a;
                    an *= 2 * alpha2;
                    g[2] = 3 * g[1] * iR2 + an * a;
                    an *= 2 * alpha2;
                    g[3] = 5 * g[2] * iR2 + an * a;
                    an *= 2 * alpha2;
                    g[4] = 7 * g[3] * iR2 + an * a;
                    an *= 2 * alpha2;
                    g[5] = 9 * g[4] * iR2 + an * a;
                }
                ewaldEval(acc, R, g, p.mroot);
            }

    for (const auto& k : p.ks)
    {
        double hx = k.hs[0] * r[0] + k.hs[1] * r[1] + k.hs[2] * r[2];
        double c = std::cos(hx), s = std::sin(hx);
        double sum  = k.fc * c + k.fs * s;
        double diff = k.fc * s - k.fs * c;
        acc[0] -= sum;
        acc[1] += diff * k.hs[0];
        acc[2] += diff * k.hs[1];
        acc[3] += diff * k.hs[2];
    }
}

} // namespace

// ==================================================================================================== C ABI

// ------------------------------------------------------------------------------------------------ target groups

/*! split bits of one window of G consecutive targets (findSplits, cstone/traversal/groups_gpu.cuh:39-73): bit i is
 *  set when the squared distance from target i to target i + 1 exceeds min(distCritSq, w_i^2); the last target of
 *  the window has no successor */
template<class T>
uint64_t findSplitsWindow(const T* pos4, int G, T distCritSq)
{
    uint64_t mask = 0;
    for (int i = 0; i + 1 < G; ++i)
    {
        const T* a = pos4 + 4 * i;
        const T* b = pos4 + 4 * (i + 1);
        T dx = b[0] - a[0], dy = b[1] - a[1], dz = b[2] - a[2];
        T d2 = norm2(dx, dy, dz);
        if (d2 > std::min(distCritSq, a[3] * a[3])) mask |= uint64_t(1) << i;
    }
    return mask;
}

/*! groupSplitsKernel (cstone/traversal/groups_gpu.cuh:148-265) for window w of G targets starting at first + w G:
 *  returns its split bits. Coordinates are in units of the longest box edge, leaf sizes in the unit box of the same
 *  aspect ratio; windows whose extent along an axis exceeds extentRatio * tolFactor * smallest leaf edge are also cut
 *  into equal power-of-two chunks. */
template<class Tc, class T>
uint64_t groupSplitsWindow(uint32_t first, uint32_t last, const Tc* x, const Tc* y, const Tc* z, const T* h,
                           const uint64_t* leaves, int numLeaves, const uint32_t* layout, const Tc* box6, int G,
                           float tolFactor, float extentRatio, uint32_t w)
{
    BoxT<Tc> box = makeBox(box6);
    unsigned bits[3] = {box.bits[0], box.bits[1], box.bits[2]};
    T unit6[6]       = {0, T(1) / T(1u << (kMaxLevel - bits[0])), 0, T(1) / T(1u << (kMaxLevel - bits[1])), 0,
                        T(1) / T(1u << (kMaxLevel - bits[2]))};
    BoxT<T> unitBox  = makeBox(unit6);
    std::vector<uint32_t> body(G);
    T nodeVolume = 1, leafEdge[3] = {1, 1, 1};
    for (int i = 0; i < G; ++i)
    {
        body[i]  = std::min<uint32_t>(first + w * uint32_t(G) + uint32_t(i), last - 1);
        int leaf = int(std::upper_bound(layout, layout + numLeaves, body[i]) - layout) - 1;
        uint64_t k0 = leaves[leaf], k1 = leaves[leaf + 1];
        auto ib     = nodeIBox(k0, rangeLevel(k1 - k0), unitBox.bits);
        T c[3], sz[3];
        geoCenterSize(ib, unitBox, c, sz);
        T vol      = 8 * sz[0] * sz[1] * sz[2];
        nodeVolume = vol > 0 ? std::min(vol, nodeVolume) : nodeVolume;
        for (int d = 0; d < 3; ++d)
            leafEdge[d] = std::min(leafEdge[d], T(2) * sz[d]);
    }
    Tc distCrit     = Tc(std::cbrt(nodeVolume) * tolFactor);
    Tc maxExtent    = std::max(std::max(box.len[0], box.len[1]), box.len[2]);
    Tc invMaxExtent = Tc(1) / maxExtent;
    std::vector<Tc> pos(4 * size_t(G));
    for (int i = 0; i < G; ++i)
    {
        uint32_t j     = body[i];
        pos[4 * i]     = x[j] * invMaxExtent;
        pos[4 * i + 1] = y[j] * invMaxExtent;
        pos[4 * i + 2] = z[j] * invMaxExtent;
        pos[4 * i + 3] = h ? Tc(2) * Tc(h[j]) * invMaxExtent : Tc(1);
    }
    uint64_t mask = findSplitsWindow<Tc>(pos.data(), G, distCrit * distCrit);

    Tc lo[3] = {pos[0], pos[1], pos[2]}, hi[3] = {lo[0], lo[1], lo[2]};
    for (int i = 0; i < G; ++i)
        for (int d = 0; d < 3; ++d)
        {
            lo[d] = std::min(lo[d], pos[4 * i + d]);
            hi[d] = std::max(hi[d], pos[4 * i + d]);
        }
    Tc ratio = 0;
    for (int d = 0; d < 3; ++d)
    {
        Tc allowed = Tc(tolFactor) * Tc(leafEdge[d]);
        Tc extent  = hi[d] - lo[d];
        if (allowed > 0) ratio = std::max(ratio, extent / allowed);
    }
    if (extentRatio > 0 && ratio > Tc(extentRatio))
    {
        unsigned chunk = unsigned(G);
        while (chunk > 1 && Tc(chunk) * ratio > Tc(G) * Tc(extentRatio))
            chunk /= 2;
        uint32_t inWindow = std::min<uint32_t>(uint32_t(G), last - (first + w * uint32_t(G)));
        for (int i = 0; i < G; ++i)
        {
            uint32_t next = uint32_t(i) + 1;
            if (next < inWindow && next % chunk == 0) mask |= uint64_t(1) << i;
        }
    }
    return mask;
}

template<class Tc, class T>
long groupSplits(uint32_t first, uint32_t last, const Tc* x, const Tc* y, const Tc* z, const T* h,
                 const uint64_t* leaves, int numLeaves, const uint32_t* layout, const Tc* box6, int G,
                 float tolFactor, float extentRatio, uint32_t* counts, uint32_t* groups, long capacity)
{
    uint32_t numWindows = (last - first + uint32_t(G) - 1) / uint32_t(G);
    std::vector<uint32_t> starts;
    for (uint32_t w = 0; w < numWindows; ++w)
    {
        uint64_t mask = groupSplitsWindow<Tc, T>(first, last, x, y, z, h, leaves, numLeaves, layout, box6, G,
                                                 tolFactor, extentRatio, w);
        if (counts) counts[w] = 1u + uint32_t(__builtin_popcountll(mask));
        uint32_t base = first + w * uint32_t(G);
        starts.push_back(base);
        for (int b = 0; b < G; ++b)
            if ((mask >> b) & 1u) starts.push_back(base + uint32_t(b) + 1);
    }
    long numGroups = long(starts.size());
    if (groups && numGroups + 1 <= capacity)
    {
        for (long i = 0; i < numGroups; ++i)
            groups[i] = starts[size_t(i)];
        groups[numGroups] = last;
    }
    return numGroups;
}

// ------------------------------------------------------------------------------------------------ MDQpole

/*! monopole + dipole + traceless quadrupole (12 values: mass, qxx, qxy, qxz, qyy, qyz, qzz, trace, px, py, pz, 0)
 *  about centre c (P2M_add / P2M_finalize, cartesian_qpole.hpp:237-303) */
template<class T>
void mdqP2M(const T* x, const T* y, const T* z, const T* m, size_t a, size_t b, const T c[3], T out[12])
{
    T g[12] = {};
    for (size_t i = a; i < b; ++i)
    {
        T rx = x[i] - c[0], ry = y[i] - c[1], rz = z[i] - c[2], mi = m[i];
        g[0] += mi;
        g[8] += mi * rx;
        g[9] += mi * ry;
        g[10] += mi * rz;
        g[1] += rx * rx * mi;
        g[2] += rx * ry * mi;
        g[3] += rx * rz * mi;
        g[4] += ry * ry * mi;
        g[5] += ry * rz * mi;
        g[6] += rz * rz * mi;
    }
    T tr = g[1] + g[4] + g[6];
    g[7] = tr;
    g[1] = 3 * g[1] - tr;
    g[4] = 3 * g[4] - tr;
    g[6] = 3 * g[6] - tr;
    g[2] *= 3;
    g[3] *= 3;
    g[5] *= 3;
    std::copy(g, g + 12, out);
}

//! add a child expansion at centre offset dX = parentCentre - childCentre (addQuadrupole, cartesian_qpole.hpp:352-398)
template<class T>
void mdqAdd(T out[12], const T dX[3], const T* a)
{
    T rx = dX[0], ry = dX[1], rz = dX[2];
    T rx2 = rx * rx, ry2 = ry * ry, rz2 = rz * rz;
    T r2  = (rx2 + ry2 + rz2) * (1.0 / 3.0);
    T ml  = a[0] * 3;
    T px = a[8], py = a[9], pz = a[10];
    T dip = rx * px + ry * py + rz * pz;
    out[7] = out[7] + a[7] + ml * r2 - 2.0 * dip;
    out[0] += a[0];
    out[8] += a[8] - a[0] * rx;
    out[9] += a[9] - a[0] * ry;
    out[10] += a[10] - a[0] * rz;
    out[1] += a[1] + ml * (rx2 - r2) - 6.0 * rx * px + 2.0 * dip;
    out[2] += a[2] + ml * rx * ry - 3.0 * (rx * py + ry * px);
    out[3] += a[3] + ml * rx * rz - 3.0 * (rx * pz + rz * px);
    out[4] += a[4] + ml * (ry2 - r2) - 6.0 * ry * py + 2.0 * dip;
    out[5] += a[5] + ml * ry * rz - 3.0 * (ry * pz + rz * py);
    out[6] += a[6] + ml * (rz2 - r2) - 6.0 * rz * pz + 2.0 * dip;
}

//! M2P of a CartesianMDQpole (cartesian_qpole.hpp:305-343), accumulating (u, ax, ay, az)
template<class T, class R>
void mdqM2P(T acc[4], const T t[3], const T c[3], const T* q, R rsq)
{
    T r[3] = {t[0] - c[0], t[1] - c[1], t[2] - c[2]};
    T r2   = norm2(r[0], r[1], r[2]);
    T rm1  = rsq(r2);
    T rm2  = rm1 * rm1;
    T rm5  = rm2 * rm2 * rm1;
    T Qrx  = r[0] * q[1] + r[1] * q[2] + r[2] * q[3];
    T Qry  = r[0] * q[2] + r[1] * q[4] + r[2] * q[5];
    T Qrz  = r[0] * q[3] + r[1] * q[5] + r[2] * q[6];
    T rQr  = r[0] * Qrx + r[1] * Qry + r[2] * Qrz;
    T qm   = (T(-2.5) * rQr * rm5 - q[0] * rm1) * rm2;
    T PR   = r[0] * q[8] + r[1] * q[9] + r[2] * q[10];
    T Px   = rm5 * (q[8] * r2 - T(3) * PR * r[0]);
    T Py   = rm5 * (q[9] * r2 - T(3) * PR * r[1]);
    T Pz   = rm5 * (q[10] * r2 - T(3) * PR * r[2]);
    acc[0] += (-q[0] - PR * rm2) * rm1 + T(-0.5) * rm5 * rQr;
    acc[1] += rm5 * Qrx + qm * r[0] + Px;
    acc[2] += rm5 * Qry + qm * r[1] + Py;
    acc[3] += rm5 * Qrz + qm * r[2] + Pz;
}

extern "C"
{

    void orc_box_dim_bits_f32(const float* box6, unsigned* bits3)
    {
        auto b = makeBox(box6);
        std::copy(b.bits, b.bits + 3, bits3);
    }

    void orc_box_dim_bits_f64(const double* box6, unsigned* bits3)
    {
        auto b = makeBox(box6);
        std::copy(b.bits, b.bits + 3, bits3);
    }

    void orc_sfc_keys_f32(const float* x, const float* y, const float* z, size_t n, const float* box6, uint64_t* keys)
    {
        auto b = makeBox(box6);
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < n; ++i)
            keys[i] = keyOf(x[i], y[i], z[i], b);
    }

    void orc_sfc_keys_f64(const double* x, const double* y, const double* z, size_t n, const double* box6,
                          uint64_t* keys)
    {
        auto b = makeBox(box6);
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < n; ++i)
            keys[i] = keyOf(x[i], y[i], z[i], b);
    }

    void orc_hilbert_ibox(uint64_t key, unsigned level, unsigned bx, unsigned by, unsigned bz, int* ibox6)
    {
        unsigned bits[3] = {bx, by, bz};
        auto b           = nodeIBox(key, level, bits);
        std::copy(b.begin(), b.end(), ibox6);
    }

    void orc_sort_keys(uint64_t* keys, uint32_t* order, size_t n)
    {
        std::vector<std::pair<uint64_t, uint32_t>> kv(n);
        for (size_t i = 0; i < n; ++i)
            kv[i] = {keys[i], uint32_t(i)};
        std::stable_sort(kv.begin(), kv.end(), [](auto& a, auto& b) { return a.first < b.first; });
        for (size_t i = 0; i < n; ++i)
        {
            keys[i]  = kv[i].first;
            order[i] = kv[i].second;
        }
    }

    long orc_octree_leaves(const uint64_t* sortedKeys, size_t n, unsigned bucket, uint64_t* leaves, uint32_t* counts,
                           long capacity)
    {
        std::vector<uint64_t> tree;
        std::vector<uint32_t> cnt;
        buildLeaves(sortedKeys, n, bucket, tree, cnt);
        long numLeaves = long(cnt.size());
        if (numLeaves <= capacity)
        {
            std::copy(tree.begin(), tree.end(), leaves);
            std::copy(cnt.begin(), cnt.end(), counts);
        }
        return numLeaves;
    }

    void orc_octree_link(const uint64_t* leaves, int numLeaves, uint64_t* prefixes, int* childOffsets, int* parents,
                         int* levelRange, int* internalToLeaf, int* leafToInternal)
    {
        // unsorted layout: internal nodes first (binary-radix-tree order), then the leaves (octree.hpp:77-100)
        int numInternal = (numLeaves - 1) / 7;
        int numNodes    = numLeaves + numInternal;
        std::vector<std::pair<uint64_t, int>> nodes(numNodes);
        for (int t = 0; t < numLeaves; ++t)
        {
            uint64_t key = leaves[t];
            unsigned lvl = rangeLevel(leaves[t + 1] - key);
            nodes[t + numInternal] = {toPrefix(key, 3 * lvl), t + numInternal};
            int common             = clz64(key ^ leaves[t + 1]) - 1;
            if (t < numLeaves - 1 && common % 3 == 0)
            {
                int at    = (t + treeIndexWeight(key, common / 3)) / 7;
                nodes[at] = {toPrefix(key, common), at};
            }
        }
        // level-major, SFC-minor order (octree.hpp:180-192); prefixes are unique
        std::stable_sort(nodes.begin(), nodes.end(), [](auto& a, auto& b) { return a.first < b.first; });
        for (int i = 0; i < numNodes; ++i)
        {
            prefixes[i]                     = nodes[i].first;
            leafToInternal[nodes[i].second] = i;
            internalToLeaf[i]               = nodes[i].second - numInternal;
        }
        for (int l = 0; l <= kMaxLevel; ++l)
            levelRange[l] = int(std::lower_bound(prefixes, prefixes + numNodes, toPrefix(0, 3 * l)) - prefixes);
        levelRange[kMaxLevel + 1] = numNodes;

        // link children and parents (octree.hpp:114-148)
        std::fill(childOffsets, childOffsets + numNodes, 0);
        for (int i = 0; i < numInternal; ++i)
        {
            int a         = leafToInternal[i];
            uint64_t pre  = prefixes[a];
            int len       = prefixLen(pre);
            unsigned lvl  = unsigned(len) / 3;
            uint64_t cpre = toPrefix(prefixKey(pre), len + 3);
            int lo = levelRange[lvl + 1], hi = levelRange[lvl + 2];
            int c = int(std::lower_bound(prefixes + lo, prefixes + hi, cpre) - prefixes);
            if (c != hi && prefixes[c] == cpre)
            {
                childOffsets[a]         = c;
                parents[(c - 1) / 8] = a;
            }
        }
    }

    void orc_upsweep_f32(int mode, const float* x, const float* y, const float* z, const float* m, int numLeaves,
                         const uint32_t* layout, const int* leafToInternal, const int* childOffsets,
                         const int* levelRange, const uint64_t* prefixes, int numNodes, float theta,
                         const float* box6, float* centers, float* multipoles)
    {
        auto box = makeBox(box6);
        std::fill(centers, centers + 4 * size_t(numNodes), 0.f);
        std::fill(multipoles, multipoles + 8 * size_t(numNodes), 0.f);
        if (mode == 0)
        {
            // float, reference CPU order (source_center.hpp:45-127, upsweep_cpu.hpp:41-74)
            auto addBody = [](float* c, float px, float py, float pz, float w)
            {
                w = std::abs(w);
                c[0] += w * px;
                c[1] += w * py;
                c[2] += w * pz;
                c[3] += w;
            };
            auto normalize = [](float* c)
            {
                float inv = (c[3] != 0.f) ? 1.f / c[3] : 1.f;
                c[0] *= inv;
                c[1] *= inv;
                c[2] *= inv;
            };
            for (int l = 0; l < numLeaves; ++l)
            {
                float* c = centers + 4 * size_t(leafToInternal[l]);
                for (uint32_t i = layout[l]; i < layout[l + 1]; ++i)
                    addBody(c, x[i], y[i], z[i], m[i]);
                normalize(c);
            }
            for (int lvl = kMaxLevel; lvl >= 0; --lvl)
                for (int i = levelRange[lvl]; i < levelRange[lvl + 1]; ++i)
                {
                    int fc = childOffsets[i];
                    if (!fc) continue;
                    float c[4] = {0, 0, 0, 0};
                    for (int k = fc; k < fc + 8; ++k)
                    {
                        const float* ck = centers + 4 * size_t(k);
                        addBody(c, ck[0], ck[1], ck[2], ck[3]);
                    }
                    normalize(c);
                    std::copy(c, c + 4, centers + 4 * size_t(i));
                }
            for (int l = 0; l < numLeaves; ++l)
            {
                int i    = leafToInternal[l];
                auto q   = p2m<float>(x, y, z, m, layout[l], layout[l + 1], centers + 4 * size_t(i));
                std::copy(q.begin(), q.end(), multipoles + 8 * size_t(i));
            }
            for (int lvl = kMaxLevel; lvl >= 0; --lvl)
                for (int i = levelRange[lvl]; i < levelRange[lvl + 1]; ++i)
                {
                    int fc = childOffsets[i];
                    if (!fc) continue;
                    Q8<float> q{};
                    const float* ci = centers + 4 * size_t(i);
                    for (int k = fc; k < fc + 8; ++k)
                    {
                        const float* ck = centers + 4 * size_t(k);
                        float d[3]      = {ci[0] - ck[0], ci[1] - ck[1], ci[2] - ck[2]};
                        Q8<float> a;
                        std::copy(multipoles + 8 * size_t(k), multipoles + 8 * size_t(k) + 8, a.begin());
                        addShifted(q, d, a);
                    }
                    std::copy(q.begin(), q.end(), multipoles + 8 * size_t(i));
                }
        }
        else
        {
            // double accumulation, one rounding to float per stored value
            std::vector<double> C(4 * size_t(numNodes), 0.0), Q(8 * size_t(numNodes), 0.0);
            for (int l = 0; l < numLeaves; ++l)
            {
                double* c = C.data() + 4 * size_t(leafToInternal[l]);
                for (uint32_t i = layout[l]; i < layout[l + 1]; ++i)
                {
                    double w = std::abs(double(m[i]));
                    c[0] += w * x[i];
                    c[1] += w * y[i];
                    c[2] += w * z[i];
                    c[3] += w;
                }
                double inv = c[3] != 0 ? 1.0 / c[3] : 1.0;
                c[0] *= inv;
                c[1] *= inv;
                c[2] *= inv;
                auto q = p2m<double>(x, y, z, m, layout[l], layout[l + 1], c);
                std::copy(q.begin(), q.end(), Q.data() + 8 * size_t(leafToInternal[l]));
            }
            for (int lvl = kMaxLevel; lvl >= 0; --lvl)
                for (int i = levelRange[lvl]; i < levelRange[lvl + 1]; ++i)
                {
                    int fc = childOffsets[i];
                    if (!fc) continue;
                    double* c = C.data() + 4 * size_t(i);
                    for (int k = fc; k < fc + 8; ++k)
                    {
                        const double* ck = C.data() + 4 * size_t(k);
                        double w         = std::abs(ck[3]);
                        c[0] += w * ck[0];
                        c[1] += w * ck[1];
                        c[2] += w * ck[2];
                        c[3] += w;
                    }
                    double inv = c[3] != 0 ? 1.0 / c[3] : 1.0;
                    c[0] *= inv;
                    c[1] *= inv;
                    c[2] *= inv;
                    Q8<double> q{};
                    for (int k = fc; k < fc + 8; ++k)
                    {
                        const double* ck = C.data() + 4 * size_t(k);
                        double d[3]      = {c[0] - ck[0], c[1] - ck[1], c[2] - ck[2]};
                        Q8<double> a;
                        std::copy(Q.data() + 8 * size_t(k), Q.data() + 8 * size_t(k) + 8, a.begin());
                        addShifted(q, d, a);
                    }
                    std::copy(q.begin(), q.end(), Q.data() + 8 * size_t(i));
                }
            for (size_t i = 0; i < 4 * size_t(numNodes); ++i)
                centers[i] = float(C[i]);
            for (size_t i = 0; i < 8 * size_t(numNodes); ++i)
                multipoles[i] = float(Q[i]);
        }
        // MAC radius from the float centre (source_center.hpp:129-143)
        float invTheta = 1.0f / theta;
        for (int i = 0; i < numNodes; ++i)
        {
            float* c  = centers + 4 * size_t(i);
            float mac = vecMacR2(prefixes[i], c, invTheta, box);
            c[3]      = (c[3] != 0.f) ? mac : 0.f;
        }
    }

    void orc_traverse_rule(int numGroups, const uint32_t* groupStart, const uint32_t* groupEnd, const float* xt,
                           const float* yt, const float* zt, const float* ht, const float* xs, const float* ys,
                           const float* zs, const float* ms, const float* hs, const int* childOffsets,
                           const int* internalToLeaf, const uint32_t* layout, const float* centers,
                           const float* multipoles, int initNodeIdx, int numShells, const float* boxL3,
                           uint32_t* m2pCount, uint32_t* p2pCount, double* acc4)
    {
        constexpr int kTargets = 64; // TravConfig::targetSize (traversal_gpu.cu:59-60)
#pragma omp parallel for schedule(dynamic, 16)
        for (int g = 0; g < numGroups; ++g)
        {
            int b = int(groupStart[g]), e = int(groupEnd[g]);
            // target positions as loaded by the warp: indices past the end repeat the last body (traversal_gpu.cu:448-453)
            float pos[kTargets][3];
            for (int k = 0; k < kTargets; ++k)
            {
                int i     = std::min(b + k, e - 1);
                pos[k][0] = xt[i];
                pos[k][1] = yt[i];
                pos[k][2] = zt[i];
            }
            float pos0[kTargets][3];
            std::memcpy(pos0, pos, sizeof(pos));
            float lo[3] = {pos[0][0], pos[0][1], pos[0][2]}, hi[3] = {lo[0], lo[1], lo[2]};
            for (int k = 1; k < kTargets; ++k)
                for (int d = 0; d < 3; ++d)
                {
                    lo[d] = std::min(lo[d], pos[k][d]);
                    hi[d] = std::max(hi[d], pos[k][d]);
                }
            float tc[3], ts[3];
            for (int d = 0; d < 3; ++d)
            {
                tc[d] = (hi[d] + lo[d]) * 0.5f;
                ts[d] = (hi[d] - lo[d]) * 0.5f;
            }

            uint32_t nM2P = 0, nP2P = 0;
            std::vector<double> acc(acc4 ? 4 * (e - b) : 0, 0.0);
            std::vector<int> stack;
            for (int iz = -numShells; iz <= numShells; ++iz)
                for (int iy = -numShells; iy <= numShells; ++iy)
                    for (int ix = -numShells; ix <= numShells; ++ix)
                    {
                        // the shift is added to and later subtracted from the float group centre, as in the
                        // reference (traversal_gpu.cu:484-505), so the MAC decisions are the reference's; the target
                        // positions are the original ones plus the shift. The reference shifts them back and forth
                        // too, which leaves rounding residues: a target then meets itself at a distance of about one
                        // float ulp of the box coordinates and, with a softening below that, gets a spurious force.
                        float sh[3] = {float(ix) * boxL3[0], float(iy) * boxL3[1], float(iz) * boxL3[2]};
                        for (int d = 0; d < 3; ++d)
                        {
                            tc[d] += sh[d];
                            for (int k = 0; k < kTargets; ++k)
                                pos[k][d] = pos0[k][d] + sh[d];
                        }

                        // interaction rule of traverseWarp (traversal_gpu.cu:210-237); order does not matter
                        stack.assign(1, initNodeIdx);
                        while (!stack.empty())
                        {
                            int first = stack.back();
                            stack.pop_back();
                            for (int cell = first; cell < first + 8; ++cell)
                            {
                                const float* mac = centers + 4 * size_t(cell);
                                float dx = std::abs(tc[0] - mac[0]) - ts[0];
                                float dy = std::abs(tc[1] - mac[1]) - ts[1];
                                float dz = std::abs(tc[2] - mac[2]) - ts[2];
                                dx = (dx + std::abs(dx)) * 0.5f;
                                dy = (dy + std::abs(dy)) * 0.5f;
                                dz = (dz + std::abs(dz)) * 0.5f;
                                bool close  = norm2(dx, dy, dz) < mac[3];
                                int child   = childOffsets[cell];
                                bool isNode = child != 0;
                                if (isNode && close) { stack.push_back(child); }
                                bool direct  = close && !isNode;
                                int leaf     = direct ? internalToLeaf[cell] : 0;
                                bool remote  = layout[leaf + 1] == layout[leaf] && mac[3] != 0.f;
                                bool approx  = !close || (!isNode && remote);
                                if (approx)
                                {
                                    ++nM2P;
                                    if (acc4)
                                    {
                                        double c3[3] = {mac[0], mac[1], mac[2]};
                                        double q[8];
                                        for (int k = 0; k < 8; ++k)
                                            q[k] = multipoles[8 * size_t(cell) + k];
                                        if (q[0] != 0.0 || q[7] != 0.0 || q[1] != 0.0 || q[2] != 0.0 ||
                                            q[3] != 0.0 || q[4] != 0.0 || q[5] != 0.0 || q[6] != 0.0)
                                            for (int k = 0; k < e - b; ++k)
                                            {
                                                double t3[3] = {pos[k][0], pos[k][1], pos[k][2]};
                                                m2p(&acc[4 * k], t3, c3, q, rsqD);
                                            }
                                    }
                                }
                                if (direct)
                                {
                                    uint32_t s0 = layout[leaf], s1 = layout[leaf + 1];
                                    nP2P += s1 - s0;
                                    if (acc4)
                                        for (int k = 0; k < e - b; ++k)
                                        {
                                            double t3[3] = {pos[k][0], pos[k][1], pos[k][2]};
                                            for (uint32_t s = s0; s < s1; ++s)
                                            {
                                                double s3[3] = {xs[s], ys[s], zs[s]};
                                                p2p(&acc[4 * k], t3, s3, double(ms[s]), double(ht[b + k]),
                                                    double(hs[s]), rsqD);
                                            }
                                        }
                                }
                            }
                        }

                        for (int d = 0; d < 3; ++d)
                            tc[d] -= sh[d];
                    }
            m2pCount[g] = nM2P;
            p2pCount[g] = nP2P;
            if (acc4)
                for (int k = 0; k < 4 * (e - b); ++k)
                    acc4[4 * size_t(b) + k] += acc[k];
        }
    }

    double orc_gravity_cpu_f32(const int* childOffsets, const int* parents, const int* internalToLeaf,
                               const float* centers, const float* multipoles, const uint32_t* layout, int numLeaves,
                               const float* x, const float* y, const float* z, const float* h, const float* m,
                               const float* box6, float G, int numShells, float* pot, float* ax, float* ay,
                               float* az)
    {
        constexpr int kGroup = 16; // traversal_cpu.hpp:180
        uint32_t first = layout[0], last = layout[numLeaves];
        float L[3]     = {box6[1] - box6[0], box6[3] - box6[2], box6[5] - box6[4]};
        double utot    = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : utot)
        for (long i0 = first; i0 < long(last); i0 += kGroup)
        {
            int valid = std::min<long>(kGroup, long(last) - i0);
            float tgt[kGroup][4];
            float acc[kGroup][4];
            for (int k = 0; k < kGroup; ++k)
            {
                // slots past the end repeat the last target (the reference leaves them unset)
                long i    = i0 + std::min(k, valid - 1);
                tgt[k][0] = x[i];
                tgt[k][1] = y[i];
                tgt[k][2] = z[i];
                tgt[k][3] = h[i];
                std::fill(acc[k], acc[k] + 4, 0.f);
            }
            for (int iz = -numShells; iz <= numShells; ++iz)
                for (int iy = -numShells; iy <= numShells; ++iy)
                    for (int ix = -numShells; ix <= numShells; ++ix)
                    {
                        float sh[3] = {ix * L[0], iy * L[1], iz * L[2]};
                        float t[kGroup][4];
                        for (int k = 0; k < kGroup; ++k)
                        {
                            for (int d = 0; d < 3; ++d)
                                t[k][d] = tgt[k][d] - sh[d];
                            t[k][3] = tgt[k][3];
                        }
                        float lo[3] = {t[0][0], t[0][1], t[0][2]}, hi[3] = {lo[0], lo[1], lo[2]};
                        for (int k = 1; k < kGroup; ++k)
                            for (int d = 0; d < 3; ++d)
                            {
                                lo[d] = std::min(t[k][d], lo[d]);
                                hi[d] = std::max(t[k][d], hi[d]);
                            }
                        float tc[3], ts[3];
                        for (int d = 0; d < 3; ++d)
                        {
                            tc[d] = (hi[d] + lo[d]) * 0.5f;
                            ts[d] = (hi[d] - lo[d]) * 0.5f;
                        }
                        // descendOrM2P (traversal_cpu.hpp:83-115)
                        auto descend = [&](int idx)
                        {
                            const float* com = centers + 4 * size_t(idx);
                            float dx = std::abs(tc[0] - com[0]) - ts[0];
                            float dy = std::abs(tc[1] - com[1]) - ts[1];
                            float dz = std::abs(tc[2] - com[2]) - ts[2];
                            dx += std::abs(dx);
                            dy += std::abs(dy);
                            dz += std::abs(dz);
                            dx *= 0.5f;
                            dy *= 0.5f;
                            dz *= 0.5f;
                            bool violates = norm2(dx, dy, dz) < std::abs(com[3]);
                            int leaf      = internalToLeaf[idx];
                            bool remote   = leaf >= 0 && layout[leaf] == layout[leaf + 1] && com[3] != 0.f;
                            if (!violates || remote)
                                for (int k = 0; k < kGroup; ++k)
                                    m2p(acc[k], t[k], com, multipoles + 8 * size_t(idx), rsqF);
                            return violates;
                        };
                        // leafP2P (traversal_cpu.hpp:123-138)
                        auto leafP2P = [&](int idx)
                        {
                            int leaf = internalToLeaf[idx];
                            for (int k = 0; k < kGroup; ++k)
                                for (uint32_t s = layout[leaf]; s < layout[leaf + 1]; ++s)
                                {
                                    float sj[3] = {x[s], y[s], z[s]};
                                    p2p(acc[k], t[k], sj, m[s], t[k][3], h[s], rsqF);
                                }
                        };
                        // stackless walk with parent links (cstone/traversal/traversal.hpp:26-69)
                        if (!descend(0)) { continue; }
                        if (childOffsets[0] == 0)
                        {
                            leafP2P(0);
                            continue;
                        }
                        int node       = childOffsets[0];
                        bool backtrack = false;
                        while (node != 0)
                        {
                            bool leaf = childOffsets[node] == 0;
                            bool down = !backtrack && descend(node);
                            if (leaf && down) { leafP2P(node); }
                            if (!leaf && down)
                            {
                                node      = childOffsets[node];
                                backtrack = false;
                            }
                            else if ((node - 1) % 8 < 7)
                            {
                                node++;
                                backtrack = false;
                            }
                            else
                            {
                                node      = parents[(node - 1) / 8];
                                backtrack = true;
                            }
                        }
                    }
            for (int k = 0; k < valid; ++k)
            {
                long i  = i0 + k;
                float u = G * m[i] * acc[k][0];
                utot += u;
                if (pot) pot[i] += u;
                ax[i] += G * acc[k][1];
                ay[i] += G * acc[k][2];
                az[i] += G * acc[k][3];
            }
        }
        return 0.5 * utot;
    }

    void orc_direct_f64(const float* x, const float* y, const float* z, const float* h, const float* m, size_t n,
                        const int64_t* targets, size_t numTargets, double G, const double* boxL3, int numShells,
                        double* pot, double* ax, double* ay, double* az)
    {
#pragma omp parallel for schedule(dynamic, 4)
        for (size_t t = 0; t < numTargets; ++t)
        {
            int64_t i      = targets[t];
            double acc[4]  = {0, 0, 0, 0};
            for (int iz = -numShells; iz <= numShells; ++iz)
                for (int iy = -numShells; iy <= numShells; ++iy)
                    for (int ix = -numShells; ix <= numShells; ++ix)
                    {
                        double ti[3] = {double(x[i]) + ix * boxL3[0], double(y[i]) + iy * boxL3[1],
                                        double(z[i]) + iz * boxL3[2]};
                        for (size_t s = 0; s < n; ++s)
                        {
                            double sj[3] = {x[s], y[s], z[s]};
                            p2p(acc, ti, sj, double(m[s]), double(h[i]), double(h[s]), rsqD);
                        }
                    }
            pot[t] = G * double(m[i]) * acc[0];
            ax[t]  = G * acc[1];
            ay[t]  = G * acc[2];
            az[t]  = G * acc[3];
        }
    }

    void orc_p2p_f64(const double* ti, const double* sj, double mj, double hi, double hj, double* acc4)
    {
        p2p(acc4, ti, sj, mj, hi, hj, rsqD);
    }

    void orc_p2m_f64(const double* x, const double* y, const double* z, const double* m, unsigned n, double* center4,
                     double* quad8)
    {
        double c[4] = {0, 0, 0, 0};
        for (unsigned i = 0; i < n; ++i)
        {
            double w = std::abs(m[i]);
            c[0] += w * x[i];
            c[1] += w * y[i];
            c[2] += w * z[i];
            c[3] += w;
        }
        double inv = c[3] != 0 ? 1.0 / c[3] : 1.0;
        for (int d = 0; d < 3; ++d)
            c[d] *= inv;
        auto q = p2m<double>(x, y, z, m, 0, n, c);
        std::copy(c, c + 4, center4);
        std::copy(q.begin(), q.end(), quad8);
    }

    void orc_m2p_f64(const double* target, const double* center, const double* quad8, double* acc4)
    {
        m2p(acc4, target, center, quad8, rsqD);
    }

    double orc_ewald_f64(const double* rootCenter3, const double* mroot8, const double* x, const double* y,
                         const double* z, const double* m, size_t n, const double* box6, double G, double* pot,
                         double* ax, double* ay, double* az, int numReplicaShells, double lCut, double hCut,
                         double alphaScale, double smallR)
    {
        double L = box6[1] - box6[0];
        auto p   = ewaldInit(mroot8, rootCenter3, numReplicaShells, L, lCut, hCut, alphaScale, smallR);
        if (p.ewaldShells == 0) { return 0.0; }
        double U = 0;
#pragma omp parallel for schedule(static) reduction(+ : U)
        for (size_t i = 0; i < n; ++i)
        {
            double pos[3] = {x[i], y[i], z[i]};
            double acc[4] = {0, 0, 0, 0};
            ewaldTarget(pos, p, acc);
            if (pot) pot[i] += G * acc[0] * m[i];
            U += acc[0] * m[i];
            ax[i] += G * acc[1];
            ay[i] += G * acc[2];
            az[i] += G * acc[3];
        }
        return 0.5 * G * U;
    }

    double orc_ewald_single_particle_energy(double m, unsigned N, double L, double G, double alphaScale)
    {
        double alpha = alphaScale / L, psi = 0;
        for (int hz = 0; hz < 10; ++hz)
            for (int hy = 0; hy < 10; ++hy)
                for (int hx = 0; hx < 10; ++hx)
                {
                    if (!(hx | hy | hz)) continue;
                    double h2 = hx * hx + hy * hy + hz * hz, hm = std::sqrt(h2);
                    psi += std::erfc(alpha * hm * L) / hm +
                           std::exp(-std::pow(M_PI * hm / (alpha * L), 2)) / (M_PI * h2);
                }
        double U = M_PI / (alpha * alpha * L * L * L) + 2 * alpha / std::sqrt(M_PI) - 1.0 / L * psi;
        return G / 2.0 * m * m * N * U;
    }

    double orc_solve_f32(float* x, float* y, float* z, float* m, float* h, size_t n, const float* box6,
                         unsigned bucket, float theta, float G, float* pot, float* ax, float* ay, float* az,
                         double* seconds)
    {
        using clock = std::chrono::steady_clock;
        auto t0     = clock::now();
        std::vector<uint64_t> keys(n);
        std::vector<uint32_t> order(n);
        orc_sfc_keys_f32(x, y, z, n, box6, keys.data());
        orc_sort_keys(keys.data(), order.data(), n);
        std::vector<float> tmp(n);
        for (float* a : {x, y, z, m, h})
        {
            for (size_t i = 0; i < n; ++i)
                tmp[i] = a[order[i]];
            std::copy(tmp.begin(), tmp.end(), a);
        }
        std::vector<uint64_t> leaves;
        std::vector<uint32_t> counts;
        buildLeaves(keys.data(), n, bucket, leaves, counts);
        int numLeaves   = int(counts.size());
        int numInternal = (numLeaves - 1) / 7, numNodes = numLeaves + numInternal;
        std::vector<uint64_t> prefixes(numNodes);
        std::vector<int> child(numNodes), parents(std::max(1, (numNodes - 1) / 8)), lr(23), i2l(numNodes),
            l2i(numNodes);
        orc_octree_link(leaves.data(), numLeaves, prefixes.data(), child.data(), parents.data(), lr.data(), i2l.data(),
                        l2i.data());
        std::vector<uint32_t> layout(numLeaves + 1, 0);
        std::inclusive_scan(counts.begin(), counts.end(), layout.begin() + 1);
        auto t1 = clock::now();
        std::vector<float> centers(4 * size_t(numNodes)), mp(8 * size_t(numNodes));
        orc_upsweep_f32(0, x, y, z, m, numLeaves, layout.data(), l2i.data() + numInternal, child.data(), lr.data(),
                        prefixes.data(), numNodes, theta, box6, centers.data(), mp.data());
        auto t2 = clock::now();
        std::fill(pot, pot + n, 0.f);
        std::fill(ax, ax + n, 0.f);
        std::fill(ay, ay + n, 0.f);
        std::fill(az, az + n, 0.f);
        double u = orc_gravity_cpu_f32(child.data(), parents.data(), i2l.data(), centers.data(), mp.data(),
                                       layout.data(), numLeaves, x, y, z, h, m, box6, G, 0, pot, ax, ay, az);
        auto t3 = clock::now();
        if (seconds)
        {
            seconds[0] = std::chrono::duration<double>(t1 - t0).count();
            seconds[1] = std::chrono::duration<double>(t2 - t1).count();
            seconds[2] = std::chrono::duration<double>(t3 - t2).count();
        }
        return u;
    }

    uint64_t orc_find_splits_f64(const double* pos4, int G, double distCritSq)
    {
        return findSplitsWindow<double>(pos4, G, distCritSq);
    }

    int orc_make_splits(uint64_t mask, int G, uint32_t* lengths)
    {
        // lengths of the runs ended by the 1-bits of a G-bit stream, then the remainder (makeSplits,
        // cstone/traversal/groups_gpu.cuh:86-110)
        int n = 0, run = 0;
        for (int b = 0; b < G; ++b)
        {
            ++run;
            if ((mask >> b) & 1u)
            {
                lengths[n++] = uint32_t(run);
                run          = 0;
            }
        }
        lengths[n++] = uint32_t(run);
        return n;
    }

    long orc_group_splits_f32(uint32_t first, uint32_t last, const float* x, const float* y, const float* z,
                              const float* h, const uint64_t* leaves, int numLeaves, const uint32_t* layout,
                              const float* box6, int groupSize, float tolFactor, float extentRatio, uint32_t* counts,
                              uint32_t* groups, long capacity)
    {
        return groupSplits<float, float>(first, last, x, y, z, h, leaves, numLeaves, layout, box6, groupSize,
                                         tolFactor, extentRatio, counts, groups, capacity);
    }

    long orc_group_splits_f64(uint32_t first, uint32_t last, const double* x, const double* y, const double* z,
                              const double* h, const uint64_t* leaves, int numLeaves, const uint32_t* layout,
                              const double* box6, int groupSize, float tolFactor, float extentRatio,
                              uint32_t* counts, uint32_t* groups, long capacity)
    {
        return groupSplits<double, double>(first, last, x, y, z, h, leaves, numLeaves, layout, box6, groupSize,
                                           tolFactor, extentRatio, counts, groups, capacity);
    }
    void orc_mdq_p2m_f64(const double* x, const double* y, const double* z, const double* m, unsigned n,
                         double* center4, double* mdq12)
    {
        double c[4] = {0, 0, 0, 0};
        for (unsigned i = 0; i < n; ++i)
        {
            double w = std::abs(m[i]);
            c[0] += w * x[i];
            c[1] += w * y[i];
            c[2] += w * z[i];
            c[3] += w;
        }
        double inv = c[3] != 0 ? 1.0 / c[3] : 1.0;
        for (int d = 0; d < 3; ++d)
            c[d] *= inv;
        mdqP2M<double>(x, y, z, m, 0, n, c, mdq12);
        std::copy(c, c + 4, center4);
    }

    void orc_mdq_m2m_f64(int numChildren, const double* centers4, const double* mdq12, const double* outCenter4,
                         double* out12)
    {
        std::fill(out12, out12 + 12, 0.0);
        for (int k = 0; k < numChildren; ++k)
        {
            double dX[3] = {outCenter4[0] - centers4[4 * k], outCenter4[1] - centers4[4 * k + 1],
                            outCenter4[2] - centers4[4 * k + 2]};
            mdqAdd<double>(out12, dX, mdq12 + 12 * k);
        }
    }

    void orc_mdq_m2p_f64(const double* target, const double* center, const double* mdq12, double* acc4)
    {
        // the reference's double inverseSquareRoot evaluates in single precision (kernel.hpp:38-52)
        mdqM2P<double>(acc4, target, center, mdq12, [](double v) { return double(1.0f / std::sqrt(float(v))); });
    }
} // extern "C"
