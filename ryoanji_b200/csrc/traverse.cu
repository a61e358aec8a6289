/*
 * ryoanji-b200: Barnes-Hut traversal with cartesian-quadrupole M2P and P2P on the FP32 pipe.
 *
 * Reference: ryoanji/src/ryoanji/nbody/traversal_gpu.cu:45-623 (warp per target group, MAC rule, overflow split).
 * The interaction rule per source cell is the reference's (traversal_gpu.cu:210-237): a cell that fails the MAC
 * against the group's bounding box is split if it has children and summed directly if it is a leaf; a cell that
 * passes, or an empty-bodied leaf with a non-zero MAC radius, is applied as a multipole. The per-group numbers of
 * approximated cells and direct bodies therefore equal the reference's whatever the traversal order.
 *
 * B200 design:
 *   - persistent warps pull 64-body target groups from a per-context work counter; each lane owns two targets;
 *   - depth-first traversal over a per-warp stack in shared memory (entries are the first of eight siblings;
 *     four entries, 32 cells, are tested per step), bounded by the stack capacity; a group that would exceed it is
 *     reported and split by the host, as the reference does with its global queue;
 *   - approximated cells and direct leaves are appended to per-warp lists in shared memory with ballot/popc
 *     compaction and evaluated in dense batches (64 bodies, 64 quadrupole cells or 32 dipole expansions, two per
 *     lane) whose data is staged in shared memory and read with broadcast loads, so the inner loops are FP32
 *     arithmetic plus one rsqrt per interaction;
 *   - the two targets of a lane are processed together with the packed f32x2 FMA/ADD/MUL of sm_100a, and the
 *     staged sources are stored pre-duplicated (s, s) so every source operand is a ready register pair: one
 *     instruction issues the work of two targets and the freed issue slots carry the rsqrt, shared-memory and
 *     traversal instructions (the kernel is issue-bound with scalar FP32);
 *   - a batch accumulates even and odd sources into two sets of fresh registers (two independent dependency
 *     chains per lane), and their sum is added to the per-target running sums with Kahan compensation; the running
 *     sums and compensations live in shared memory, which keeps the kernel at 96 registers (five blocks per SM);
 *   - the MAC test uses explicitly rounded single operations so that every decision is reproducible bit for bit.
 */
#include "internal.hpp"

namespace ryo
{

constexpr int kTravWarps    = 4;
constexpr int kTravThreads  = kTravWarps * kWarp;
constexpr int kM2PCap       = 64;  // pending approximated cells (flushed at 64, or 32 for dipole expansions)
constexpr int kLeafCap      = 64;  // pending direct leaves (flushed when more than 32 are pending)
constexpr int kP2PBatch     = 2 * kWarp; // direct bodies evaluated per staging round (two per lane)
constexpr int kRootOnly     = -2;  // stack marker: the root itself is the only cell (single-leaf tree); a marker
                                   // -(r + 2) stands for the single cell r

struct WarpSmem
{
    int m2p[kM2PCap + kWarp];
    int2 leaves[kLeafCap + kWarp];
    int leafScan[kLeafCap + kWarp];
    // staged sources, every value duplicated: M2P 5 x 16 bytes per cell for 64 quadrupoles (7 for 32 dipole
    // expansions), P2P 2 x 16 + 8 bytes per body for 64 bodies
    float4 stage[10 * kWarp];
    // per lane: Kahan running sums [0] and compensations [1] of (-phi, ax, ay, az), both targets packed
    unsigned long long sums[2][4][kWarp];
    // evaluation batches of the current walk: the next batch's number, and which of them this warp evaluates
    // (batch j when j % parts == part; parts is 1 outside the split second pass)
    int batchNext, part, parts, item;
    // 1 if every target and source of the launch has the softening of the group's targets (T.h0)
    int allUniform;
    // 1 if every source of the launch has the mass massU: the direct sums then apply it once per batch
    int uniformMass;
    float massU;
    int pad;
};

//! true if the walk's next evaluation batch belongs to this warp; counts the batch either way. Outside the split
//! second pass (kSplit false) every batch is the warp's own.
template<bool kSplit>
__device__ __forceinline__ bool ownBatch(WarpSmem& S)
{
    if constexpr (!kSplit) return true;
    int j = S.batchNext;
    __syncwarp();
    if (laneId() == 0) S.batchNext = j + 1;
    __syncwarp();
    return S.parts <= 1 || j % S.parts == S.part;
}

static_assert(2 * kP2PBatch + kP2PBatch / 2 <= 10 * kWarp, "a P2P batch must fit in the stage");
static_assert(5 * 2 * kWarp <= 10 * kWarp && 7 * kWarp <= 10 * kWarp, "an M2P batch must fit in the stage");
// an M2P flush leaves fewer than kWarp cells pending (at most 64 + 31 before it); one walk step adds at most kWarp
static_assert(2 * kWarp - 1 + kWarp <= kM2PCap + kWarp, "the pending cell list must hold a step's additions");
// a P2P evaluation leaves fewer than kP2PBatch bodies, so at most kP2PBatch - 1 leaves, pending; one walk step adds
// at most kWarp more
static_assert(kP2PBatch - 1 + kWarp <= kLeafCap + kWarp, "the pending leaf list must hold a step's additions");

// ------------------------------------------------------------------------------------------------ packed f32x2

using f2 = unsigned long long; // two floats: low half target 0, high half target 1

__device__ __forceinline__ f2 pk(float lo, float hi)
{
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void upk(f2 v, float& lo, float& hi) { asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v)); }
__device__ __forceinline__ f2 add2(f2 a, f2 b)
{
    f2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b)
{
    f2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b)
{
    f2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c)
{
    f2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}

__device__ __forceinline__ float rsqrtApprox(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ f2 rsqrt2(f2 v)
{
    float a, b;
    upk(v, a, b);
    return pk(rsqrtApprox(a), rsqrtApprox(b));
}

//! packed accumulators of a lane's two targets: P = -phi, X, Y, Z = acceleration
struct Acc2
{
    f2 p, x, y, z;
};

/*! M2P of one quadrupole (cartesian_qpole.hpp:152-176) for both targets; c* and q* are duplicated pairs.
 *  q = (qxx, qxy, qxz, qyy, qyz, qzz) traceless x3, m the mass. */
__device__ __forceinline__ void m2p2(Acc2& A, f2 tx, f2 ty, f2 tz, f2 cx, f2 cy, f2 cz, f2 m, f2 qxx, f2 qxy,
                                     f2 qxz, f2 qyy, f2 qyz, f2 qzz)
{
    const f2 kM25  = 0xC0200000C0200000ull; // (-2.5f, -2.5f)
    const f2 kHalf = 0x3F0000003F000000ull; // (0.5f, 0.5f)
    f2 rx  = sub2(tx, cx), ry = sub2(ty, cy), rz = sub2(tz, cz);
    f2 r2  = fma2(rx, rx, fma2(ry, ry, mul2(rz, rz)));
    f2 rm1 = rsqrt2(r2);
    f2 rm2 = mul2(rm1, rm1);
    f2 rm5 = mul2(mul2(rm2, rm2), rm1);
    f2 Qrx = fma2(rx, qxx, fma2(ry, qxy, mul2(rz, qxz)));
    f2 Qry = fma2(rx, qxy, fma2(ry, qyy, mul2(rz, qyz)));
    f2 Qrz = fma2(rx, qxz, fma2(ry, qyz, mul2(rz, qzz)));
    f2 rQr = fma2(rx, Qrx, fma2(ry, Qry, mul2(rz, Qrz)));
    f2 mr1 = mul2(m, rm1);
    f2 t   = mul2(rQr, rm5);
    f2 f   = mul2(sub2(mul2(t, kM25), mr1), rm2);
    A.p    = add2(A.p, fma2(t, kHalf, mr1));
    A.x    = fma2(rm5, Qrx, fma2(f, rx, A.x));
    A.y    = fma2(rm5, Qry, fma2(f, ry, A.y));
    A.z    = fma2(rm5, Qrz, fma2(f, rz, A.z));
}

/*! M2P of a monopole + dipole + quadrupole expansion (cartesian_qpole.hpp:305-343) for both targets: the
 *  quadrupole terms of m2p2 plus the dipole p: -phi += (p.r) / r^3, a += p / r^3 - 3 (p.r) r / r^5 */
__device__ __forceinline__ void m2p2mdq(Acc2& A, f2 tx, f2 ty, f2 tz, f2 cx, f2 cy, f2 cz, f2 m, f2 qxx, f2 qxy,
                                        f2 qxz, f2 qyy, f2 qyz, f2 qzz, f2 px, f2 py, f2 pz)
{
    const f2 kM25  = 0xC0200000C0200000ull; // (-2.5f, -2.5f)
    const f2 kHalf = 0x3F0000003F000000ull; // (0.5f, 0.5f)
    const f2 kM3   = 0xC0400000C0400000ull; // (-3f, -3f)
    f2 rx  = sub2(tx, cx), ry = sub2(ty, cy), rz = sub2(tz, cz);
    f2 r2  = fma2(rx, rx, fma2(ry, ry, mul2(rz, rz)));
    f2 rm1 = rsqrt2(r2);
    f2 rm2 = mul2(rm1, rm1);
    f2 rm3 = mul2(rm2, rm1);
    f2 rm5 = mul2(rm3, rm2);
    f2 Qrx = fma2(rx, qxx, fma2(ry, qxy, mul2(rz, qxz)));
    f2 Qry = fma2(rx, qxy, fma2(ry, qyy, mul2(rz, qyz)));
    f2 Qrz = fma2(rx, qxz, fma2(ry, qyz, mul2(rz, qzz)));
    f2 rQr = fma2(rx, Qrx, fma2(ry, Qry, mul2(rz, Qrz)));
    f2 PR  = fma2(rx, px, fma2(ry, py, mul2(rz, pz)));
    f2 mr1 = mul2(m, rm1);
    f2 t   = mul2(rQr, rm5);
    f2 f   = fma2(mul2(kM3, PR), rm5, mul2(sub2(mul2(t, kM25), mr1), rm2));
    A.p    = add2(A.p, fma2(PR, rm3, fma2(t, kHalf, mr1)));
    A.x    = fma2(rm5, Qrx, fma2(f, rx, fma2(px, rm3, A.x)));
    A.y    = fma2(rm5, Qry, fma2(f, ry, fma2(py, rm3, A.y)));
    A.z    = fma2(rm5, Qrz, fma2(f, rz, fma2(pz, rm3, A.z)));
}

/*! P2P with a softening floor hh = (h_i + h_j)^2 common to both targets and the source: the same arithmetic as
 *  p2p2 when every h is equal, without the two packed operations that form hh */
__device__ __forceinline__ void p2p2u(Acc2& A, f2 tx, f2 ty, f2 tz, float hh, f2 sx, f2 sy, f2 sz, f2 sm)
{
    f2 dx  = sub2(sx, tx), dy = sub2(sy, ty), dz = sub2(sz, tz);
    f2 r2  = fma2(dx, dx, fma2(dy, dy, mul2(dz, dz)));
    float r0, r1;
    upk(r2, r0, r1);
    f2 ir  = pk(rsqrtApprox(fmaxf(r0, hh)), rsqrtApprox(fmaxf(r1, hh)));
    f2 m3  = mul2(mul2(sm, ir), mul2(ir, ir));
    A.p    = fma2(m3, r2, A.p);
    A.x    = fma2(dx, m3, A.x);
    A.y    = fma2(dy, m3, A.y);
    A.z    = fma2(dz, m3, A.z);
}

/*! p2p2u for sources of one common mass, which the caller applies to the batch's sums: a packed multiply less
 *  per interaction */
__device__ __forceinline__ void p2p2um(Acc2& A, f2 tx, f2 ty, f2 tz, float hh, f2 sx, f2 sy, f2 sz)
{
    f2 dx  = sub2(sx, tx), dy = sub2(sy, ty), dz = sub2(sz, tz);
    f2 r2  = fma2(dx, dx, fma2(dy, dy, mul2(dz, dz)));
    float r0, r1;
    upk(r2, r0, r1);
    f2 ir  = pk(rsqrtApprox(fmaxf(r0, hh)), rsqrtApprox(fmaxf(r1, hh)));
    f2 i3  = mul2(ir, mul2(ir, ir));
    A.p    = fma2(i3, r2, A.p);
    A.x    = fma2(dx, i3, A.x);
    A.y    = fma2(dy, i3, A.y);
    A.z    = fma2(dz, i3, A.z);
}

/*! P2P (kernel.hpp:99-120) for both targets against one source; s* are duplicated pairs, th the targets' h */
__device__ __forceinline__ void p2p2(Acc2& A, f2 tx, f2 ty, f2 tz, f2 th, f2 sx, f2 sy, f2 sz, f2 sm, f2 sh)
{
    f2 dx  = sub2(sx, tx), dy = sub2(sy, ty), dz = sub2(sz, tz);
    f2 r2  = fma2(dx, dx, fma2(dy, dy, mul2(dz, dz)));
    f2 hij = add2(th, sh);
    f2 hh  = mul2(hij, hij);
    float r0, r1, h0, h1;
    upk(r2, r0, r1);
    upk(hh, h0, h1);
    f2 ir  = pk(rsqrtApprox(fmaxf(r0, h0)), rsqrtApprox(fmaxf(r1, h1)));
    f2 m3  = mul2(mul2(sm, ir), mul2(ir, ir));
    A.p    = fma2(m3, r2, A.p);
    A.x    = fma2(dx, m3, A.x);
    A.y    = fma2(dy, m3, A.y);
    A.z    = fma2(dz, m3, A.z);
}

struct TargetState
{
    f2 tx, ty, tz, th; // the lane's two targets (shifted by the current replica)
    float h0;          // the common smoothing length of the group's targets, if uniformH
    bool uniformH;
};

__device__ __forceinline__ void kahan2(f2& sum, f2& comp, f2 v)
{
    f2 y = sub2(v, comp);
    f2 t = add2(sum, y);
    comp = sub2(sub2(t, sum), y);
    sum  = t;
}

__device__ __forceinline__ Acc2 zero2()
{
    Acc2 a;
    a.p = a.x = a.y = a.z = 0ull;
    return a;
}

//! node data from the packed 64-byte records of the solver path
struct RecordNodes
{
    static constexpr bool kDipole = false;
    const NodeRecord* __restrict__ r;
    __device__ __forceinline__ void load(int cell, float4& c, int4& link) const
    {
        c    = __ldg(&r[cell].center);
        link = __ldg(&r[cell].link);
    }
    __device__ __forceinline__ void multipole(int cell, float4& c, float4& q0, float4& q1, float4& dp) const
    {
        c  = __ldg(&r[cell].center);
        q0 = __ldg(&r[cell].q0);
        q1 = __ldg(&r[cell].q1);
    }
};

//! the records plus node dipoles: monopole + dipole + quadrupole expansions (CartesianMDQpole)
struct RecordNodesMDQ : RecordNodes
{
    static constexpr bool kDipole = true;
    const float4* __restrict__ dip;
    __device__ __forceinline__ void multipole(int cell, float4& c, float4& q0, float4& q1, float4& dp) const
    {
        RecordNodes::multipole(cell, c, q0, q1, dp);
        dp = __ldg(dip + cell);
    }
};

//! node data from the reference's separate arrays (centres, multipoles, childOffsets, internalToLeaf, layout)
struct ArrayNodes
{
    static constexpr bool kDipole = false;
    const float4* __restrict__ centers;
    const float4* __restrict__ mpoles; // two float4 per node (three for CartesianMDQpole)
    const int* __restrict__ childOffsets;
    const int* __restrict__ internalToLeaf;
    const uint32_t* __restrict__ layout;
    __device__ __forceinline__ void load(int cell, float4& c, int4& link) const
    {
        c       = __ldg(centers + cell);
        int fc  = __ldg(childOffsets + cell);
        link    = make_int4(fc, 0, 0, 0);
        if (fc == 0)
        {
            int leaf = __ldg(internalToLeaf + cell);
            uint32_t a = __ldg(layout + leaf), b = __ldg(layout + leaf + 1);
            link.y     = int(a);
            link.z     = int(b - a);
        }
    }
    __device__ __forceinline__ void multipole(int cell, float4& c, float4& q0, float4& q1, float4& dp) const
    {
        c  = __ldg(centers + cell);
        q0 = __ldg(mpoles + 2 * cell);
        q1 = __ldg(mpoles + 2 * cell + 1);
    }
};

//! the reference's CartesianMDQpole arrays: 12 floats per node (mass, q x6, trace, px, py, pz, unused)
struct ArrayNodesMDQ : ArrayNodes
{
    static constexpr bool kDipole = true;
    __device__ __forceinline__ void multipole(int cell, float4& c, float4& q0, float4& q1, float4& dp) const
    {
        c  = __ldg(centers + cell);
        q0 = __ldg(mpoles + 3 * cell);
        q1 = __ldg(mpoles + 3 * cell + 1);
        dp = __ldg(mpoles + 3 * cell + 2);
    }
};

//! bodies as packed (x, y, z, w) plus one scalar array (solver path)
struct PackedBodies
{
    const float4* __restrict__ xyzw;
    const float* __restrict__ s;
    __device__ __forceinline__ float4 vec(int i) const { return __ldg(xyzw + i); }
    __device__ __forceinline__ float scalar(int i) const { return __ldg(s + i); }
};

//! bodies as the reference's separate arrays: vec = (x, y, z, w), scalar = s
struct SoABodies
{
    const float* __restrict__ x;
    const float* __restrict__ y;
    const float* __restrict__ z;
    const float* __restrict__ w;
    const float* __restrict__ s;
    __device__ __forceinline__ float4 vec(int i) const
    {
        return make_float4(__ldg(x + i), __ldg(y + i), __ldg(z + i), __ldg(w + i));
    }
    __device__ __forceinline__ float scalar(int i) const { return __ldg(s + i); }
};

__device__ __forceinline__ Acc2 sum2(const Acc2& a, const Acc2& b)
{
    Acc2 r;
    r.p = add2(a.p, b.p);
    r.x = add2(a.x, b.x);
    r.y = add2(a.y, b.y);
    r.z = add2(a.z, b.z);
    return r;
}
//! add one batch's partial sums to the lane's Kahan-compensated running sums in shared memory
__device__ __forceinline__ void addBatchS(WarpSmem& S, const Acc2& part)
{
    int lane = laneId();
    f2 v[4] = {part.p, part.x, part.y, part.z};
#pragma unroll
    for (int c = 0; c < 4; ++c)
    {
        f2 sum = S.sums[0][c][lane], comp = S.sums[1][c][lane];
        kahan2(sum, comp, v[c]);
        S.sums[0][c][lane] = sum;
        S.sums[1][c][lane] = comp;
    }
}

//! approximated cells per evaluation batch: 64 quadrupoles (5 staged float4 each), or 32 dipole expansions (7)
template<class Nodes>
__host__ __device__ constexpr int m2pBatch()
{
    return Nodes::kDipole ? kWarp : 2 * kWarp;
}

//! evaluate the first @p count (<= m2pBatch) pending cells
template<bool kSplit, class Nodes>
__device__ void evalM2P(WarpSmem& S, int count, const Nodes& nodes, TargetState& T)
{
    constexpr int kStride = Nodes::kDipole ? 7 : 5; // staged float4 per cell
    constexpr int kBatch  = m2pBatch<Nodes>();
    if (!ownBatch<kSplit>(S)) return;
    int lane = laneId();
#pragma unroll
    for (int half = 0; half < kBatch / kWarp; ++half)
    {
        int k = half * kWarp + lane;
        if (k < count)
        {
            float4 c, q0, q1, dp = make_float4(0.f, 0.f, 0.f, 0.f);
            nodes.multipole(S.m2p[k], c, q0, q1, dp);
            float4* st = S.stage + kStride * k;
            st[0]      = make_float4(c.x, c.x, c.y, c.y);
            st[1]      = make_float4(c.z, c.z, q0.x, q0.x);
            st[2]      = make_float4(q0.y, q0.y, q0.z, q0.z);
            st[3]      = make_float4(q0.w, q0.w, q1.x, q1.x);
            st[4]      = make_float4(q1.y, q1.y, q1.z, q1.z);
            if (Nodes::kDipole)
            {
                st[5 % kStride] = make_float4(dp.x, dp.x, dp.y, dp.y);
                st[6 % kStride] = make_float4(dp.z, dp.z, 0.f, 0.f);
            }
        }
    }
    __syncwarp();
    const ulonglong2* st = reinterpret_cast<const ulonglong2*>(S.stage);
    Acc2 pa = zero2(), pb = zero2();
    auto one = [&](Acc2& part, int j)
    {
        const ulonglong2* sj = st + kStride * j;
        ulonglong2 a = sj[0], b = sj[1], c = sj[2], d = sj[3], e = sj[4];
        if constexpr (Nodes::kDipole)
        {
            ulonglong2 f = sj[5 % kStride], g = sj[6 % kStride];
            m2p2mdq(part, T.tx, T.ty, T.tz, a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y, e.x, e.y, f.x, f.y, g.x);
        }
        else
            m2p2(part, T.tx, T.ty, T.tz, a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y, e.x, e.y);
    };
    if (count == kBatch)
    {
#pragma unroll 4
        for (int j = 0; j < kBatch; j += 2)
        {
            one(pa, j);
            one(pb, j + 1);
        }
    }
    else
    {
        int j = 0;
        for (; j + 1 < count; j += 2)
        {
            one(pa, j);
            one(pb, j + 1);
        }
        if (j < count) one(pa, j);
    }
    addBatchS(S, sum2(pa, pb));
    __syncwarp();
}

/*! evaluate pending direct leaves in batches of kP2PBatch bodies; with @p all == false only whole batches are evaluated
 *  and the remainder stays pending (the first pending leaf may be partly consumed). Returns the leaves left. */
template<bool kSplit, class Sources>
__device__ int evalP2P(WarpSmem& S, int numLeaves, bool all, const Sources& src, TargetState& T)
{
    int lane = laneId();
    // inclusive scan of the body counts over the pending leaves
    int total = 0;
    for (int base = 0; base < numLeaves; base += kWarp)
    {
        int i   = base + lane;
        int cnt = i < numLeaves ? S.leaves[i].y : 0;
        int inc = warpInclusiveScan(cnt) + total;
        if (i < numLeaves) S.leafScan[i] = inc;
        total = __shfl_sync(0xffffffffu, inc, kWarp - 1);
    }
    __syncwarp();
    int numBatches = all ? (total + kP2PBatch - 1) / kP2PBatch : total / kP2PBatch;
    // staged body k: positions and mass at stage[2 k], stage[2 k + 1], softening pair at sth[k]
    const ulonglong2* st = reinterpret_cast<const ulonglong2*>(S.stage);
    const f2* sth        = reinterpret_cast<const f2*>(S.stage + 2 * kP2PBatch);
    const bool allUniform = S.allUniform != 0; // no softening to stage or compare
    int first             = 0;                  // warp-uniform: the pending leaf that holds the batch's first body
    for (int b = 0; b < numBatches; ++b)
    {
        // where the next 64 leaves end relative to the batch start R0: bit q of ends is set if a leaf ends after
        // body R0 + q (its inclusive prefix is R0 + q + 1). A batch of 64 bodies meets at most 64 leaves.
        const int R0 = b * kP2PBatch;
        int t0 = first + lane, t1 = first + kWarp + lane;
        int p0 = t0 < numLeaves ? S.leafScan[t0] - R0 : kP2PBatch + 1;
        int p1 = t1 < numLeaves ? S.leafScan[t1] - R0 : kP2PBatch + 1;
        auto bitsIn = [](int p, int lo) { return p > lo && p <= lo + kWarp ? 1u << (p - lo - 1) : 0u; };
        unsigned endsLo = __reduce_or_sync(0xffffffffu, bitsIn(p0, 0) | bitsIn(p1, 0));
        unsigned endsHi = __reduce_or_sync(0xffffffffu, bitsIn(p0, kWarp) | bitsIn(p1, kWarp));
        const unsigned long long ends = (static_cast<unsigned long long>(endsHi) << 32) | endsLo;
        const int leafBase = first;
        first += __popcll(ends); // the leaves ending inside this batch come before the next batch's first body
        if (!ownBatch<kSplit>(S)) continue;
#pragma unroll
        for (int half = 0; half < 2; ++half)
        {
            int k = half * kWarp + lane;
            int r = R0 + k;
            if (r < total)
            {
                // body r lies in the leaf after the ones that end at or before it (ends bits 0 .. k - 1)
                int leaf  = leafBase + (k == 0 ? 0 : __popcll(ends & (~0ull >> (64 - k))));
                int2 lf   = S.leaves[leaf];
                int body  = lf.x + (r - (S.leafScan[leaf] - lf.y));
                float4 sj = src.vec(body);
                S.stage[2 * k]     = make_float4(sj.x, sj.x, sj.y, sj.y);
                S.stage[2 * k + 1] = make_float4(sj.z, sj.z, sj.w, sj.w);
                if (!allUniform)
                {
                    float hj = src.scalar(body);
                    reinterpret_cast<float2*>(S.stage + 2 * kP2PBatch)[k] = make_float2(hj, hj);
                }
            }
        }
        __syncwarp();
        int nvalid = min(kP2PBatch, total - b * kP2PBatch);
        Acc2 part  = zero2();
        // equal smoothing lengths for the targets and this batch's sources: hh is one constant
        if (T.uniformH)
        {
            float hj0 = T.h0;
            bool same = true;
            if (!allUniform)
            {
                float ha, hb, dup;
                upk(sth[0], hj0, dup);
                upk(sth[lane < nvalid ? lane : 0], ha, dup);
                upk(sth[kWarp + lane < nvalid ? kWarp + lane : 0], hb, dup);
                same = __all_sync(0xffffffffu, ha == hj0 && hb == hj0);
            }
            if (same)
            {
                float hij = __fadd_rn(T.h0, hj0);
                float hh  = __fmul_rn(hij, hij);
                Acc2 pb   = zero2();
                // two accumulation chains over the batch's sources
                auto batch = [&](auto&& oneU)
                {
                    if (nvalid == kP2PBatch)
                    {
#pragma unroll 8
                        for (int j = 0; j < kP2PBatch; j += 2)
                        {
                            oneU(part, j);
                            oneU(pb, j + 1);
                        }
                    }
                    else
                    {
                        int j = 0;
                        for (; j + 1 < nvalid; j += 2)
                        {
                            oneU(part, j);
                            oneU(pb, j + 1);
                        }
                        if (j < nvalid) oneU(part, j);
                    }
                };
                if (S.uniformMass)
                {
                    batch([&](Acc2& pp, int j)
                          {
                              ulonglong2 a = st[2 * j], c = st[2 * j + 1];
                              p2p2um(pp, T.tx, T.ty, T.tz, hh, a.x, a.y, c.x);
                          });
                    Acc2 sum = sum2(part, pb);
                    f2 mm    = pk(S.massU, S.massU);
                    sum.p    = mul2(sum.p, mm);
                    sum.x    = mul2(sum.x, mm);
                    sum.y    = mul2(sum.y, mm);
                    sum.z    = mul2(sum.z, mm);
                    addBatchS(S, sum);
                }
                else
                {
                    batch([&](Acc2& pp, int j)
                          {
                              ulonglong2 a = st[2 * j], c = st[2 * j + 1];
                              p2p2u(pp, T.tx, T.ty, T.tz, hh, a.x, a.y, c.x, c.y);
                          });
                    addBatchS(S, sum2(part, pb));
                }
                __syncwarp();
                continue;
            }
        }
        auto one = [&](int j)
        {
            ulonglong2 a = st[2 * j], c = st[2 * j + 1];
            p2p2(part, T.tx, T.ty, T.tz, T.th, a.x, a.y, c.x, c.y, sth[j]);
        };
        if (nvalid == kP2PBatch)
        {
#pragma unroll 8
            for (int j = 0; j < kP2PBatch; ++j)
                one(j);
        }
        else
        {
            for (int j = 0; j < nvalid; ++j)
                one(j);
        }
        addBatchS(S, part);
        __syncwarp();
    }
    if (all) return 0;
    // keep bodies [numBatches * kP2PBatch, total): drop fully consumed leaves, trim the first kept one
    int done = numBatches * kP2PBatch;
    int keepFrom = 0;
    {
        int lo = 0, hi = numLeaves; // first leaf with inclusive prefix > done
        while (lo < hi)
        {
            int mid = (lo + hi) >> 1;
            if (S.leafScan[mid] > done) hi = mid;
            else lo = mid + 1;
        }
        keepFrom = lo;
    }
    int keep = numLeaves - keepFrom;
    int2 tmp[(kLeafCap + kWarp + kWarp - 1) / kWarp];
    int nIter = (keep + kWarp - 1) / kWarp;
    for (int it = 0; it < nIter; ++it)
    {
        int i = keepFrom + it * kWarp + lane;
        if (i < numLeaves)
        {
            int2 lf = S.leaves[i];
            if (i == keepFrom)
            {
                int consumed = done - (S.leafScan[i] - lf.y);
                lf.x += consumed;
                lf.y -= consumed;
            }
            tmp[it] = lf;
        }
    }
    __syncwarp();
    for (int it = 0; it < nIter; ++it)
    {
        int i = it * kWarp + lane;
        if (keepFrom + i < numLeaves) S.leaves[i] = tmp[it];
    }
    __syncwarp();
    return keep;
}

__global__ void resetTraversal(Control* ctl, bool resetStats)
{
    if (threadIdx.x == 0)
    {
        ctl->workCounter = 0;
        ctl->failedCount = 0;
        ctl->heavyCount  = 0;
        if (resetStats)
        {
            for (int i = 0; i < 5; ++i)
                ctl->stats[i] = 0;
            ctl->potential = 0.0;
        }
    }
}

void launchTraversalReset(Control* ctl, bool resetStats, cudaStream_t s)
{
    resetTraversal<<<1, 32, 0, s>>>(ctl, resetStats);
    RYO_LAUNCH_CHECK();
}

/*! a target's G m phi and G a: added to the outputs (the reference's accumulation), or with P.overwrite stored as
 *  0 + value without reading them, which gives the bits an add to a zeroed output gives */
__device__ __forceinline__ void storeResult(const TraverseLaunch& P, int idx, float p, float x, float y, float z)
{
    const bool add = !P.overwrite;
    if (P.p) P.p[idx] = (add ? P.p[idx] : 0.f) + p;
    P.ax[idx] = (add ? P.ax[idx] : 0.f) + x;
    P.ay[idx] = (add ? P.ay[idx] : 0.f) + y;
    P.az[idx] = (add ? P.az[idx] : 0.f) + z;
}

//! one warp per queued group: add the parts' partial sums in part order (FP64) and write the group's results
__global__ void combineHeavyKernel(TraverseLaunch P, const float* __restrict__ mass)
{
    const unsigned w    = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
    const unsigned lane = laneId();
    if (w >= P.numHeavy) return; // whole warps leave together
    const unsigned g   = P.heavyGroups[w];
    const int K        = P.parts;
    const size_t item0 = size_t(w) * unsigned(K);
    bool failed        = false;
    for (int k = int(lane); k < K; k += kWarp)
        failed |= P.partStatus[item0 + k] != 0;
    if (__any_sync(0xffffffffu, failed))
    {
        if (lane == 0)
        {
            unsigned slotF = atomicAdd(&P.ctl->failedCount, 1u);
            if (slotF < P.failedCapacity) P.failedGroups[slotF] = g;
        }
        return;
    }
    const int b = int(P.groupStart[g]), e = int(P.groupEnd[g]);
    double pot  = 0.0;
#pragma unroll
    for (int t = 0; t < 2; ++t)
    {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        for (int k = 0; k < K; ++k)
        {
            float4 v = P.partials[(item0 + k) * (2 * kWarp) + t * kWarp + lane];
            s0 += v.x;
            s1 += v.y;
            s2 += v.z;
            s3 += v.w;
        }
        int idx = b + t * kWarp + int(lane);
        if (idx < e)
        {
            float phi = float(s0), gx = float(s1), gy = float(s2), gz = float(s3);
            float mi  = mass[idx];
            pot += double(mi) * double(phi);
            storeResult(P, idx, P.G * mi * phi, P.G * gx, P.G * gy, P.G * gz);
        }
    }
    pot = warpSum(pot);
    if (lane == 0)
    {
        atomicAdd(&P.ctl->potential, pot);
        if (P.sysPotential) atomicAdd(P.sysPotential + (P.groupSys ? P.groupSys[g] : 0u), pot);
    }
}

void launchCombineHeavy(const TraverseLaunch& t, const float* mass, cudaStream_t s)
{
    if (t.numHeavy == 0) return;
    combineHeavyKernel<<<ceilDiv(size_t(t.numHeavy) * kWarp, 256), 256, 0, s>>>(t, mass);
    RYO_LAUNCH_CHECK();
}

template<class Nodes, class Targets, class Sources, bool kSplit>
__global__ void __launch_bounds__(kTravThreads, 5)
    traverseKernel(TraverseLaunch P, Nodes nodes, Targets tgt, Sources src)
{
    extern __shared__ __align__(16) unsigned char smemRaw[];
    const int warp = threadIdx.x / kWarp, lane = laneId();
    int* stack     = reinterpret_cast<int*>(smemRaw) + warp * P.stackCapacity;
    WarpSmem& S    = reinterpret_cast<WarpSmem*>(smemRaw + sizeof(int) * kTravWarps * P.stackCapacity)[warp];
    const unsigned lt = lanemaskLt();

    const unsigned numItems = P.parts > 0 ? P.numHeavy * unsigned(P.parts) : unsigned(P.numGroups);
    while (true)
    {
        unsigned item = 0;
        if (lane == 0) item = atomicAdd(&P.ctl->workCounter, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= numItems) return;
        unsigned g = item;
        if (P.parts > 0) g = P.heavyGroups[item / unsigned(P.parts)];
        if (lane == 0)
        {
            S.batchNext = 0;
            S.part      = P.parts > 0 ? int(item % unsigned(P.parts)) : 0;
            S.parts     = P.parts > 0 ? P.parts : 1;
            S.item      = int(item);
        }

        const int b = int(P.groupStart[g]), e = int(P.groupEnd[g]);
        TargetState T;
        float4 t0 = tgt.vec(min(b + lane, e - 1));
        float4 t1 = tgt.vec(min(b + kWarp + lane, e - 1));
        T.tx      = pk(t0.x, t1.x);
        T.ty      = pk(t0.y, t1.y);
        T.tz      = pk(t0.z, t1.z);
        T.th      = pk(t0.w, t1.w);
        T.h0       = __shfl_sync(0xffffffffu, t0.w, 0);
        T.uniformH = __all_sync(0xffffffffu, t0.w == T.h0 && t1.w == T.h0);
        if (lane == 0)
        {
            S.allUniform = P.softeningRange && T.uniformH && P.softeningRange[0] == P.softeningRange[1] &&
                           orderedFloat(P.softeningRange[0]) == T.h0;
            S.uniformMass = P.massRange && !P.groupSys && P.massRange[0] == P.massRange[1];
            S.massU       = S.uniformMass ? orderedFloat(P.massRange[0]) : 0.f;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c)
            S.sums[0][c][lane] = S.sums[1][c][lane] = 0ull;
        float lo[3] = {fminf(t0.x, t1.x), fminf(t0.y, t1.y), fminf(t0.z, t1.z)};
        float hi[3] = {fmaxf(t0.x, t1.x), fmaxf(t0.y, t1.y), fmaxf(t0.z, t1.z)};
        float tc[3], ts[3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            float l = warpMin(lo[d]), h = warpMax(hi[d]);
            tc[d]   = __fmul_rn(__fadd_rn(h, l), 0.5f);
            ts[d]   = __fmul_rn(__fsub_rn(h, l), 0.5f);
        }

        // the group's tree root and periodic images: the launch's, or its system's in a batched solve
        int rootEntry = P.numNodes == 1 ? kRootOnly : P.initNode;
        int shells    = P.numShells;
        float boxL[3] = {P.boxL[0], P.boxL[1], P.boxL[2]};
        uint32_t sys  = 0;
        if (P.groupSys)
        {
            sys               = P.groupSys[g];
            const SysTrav& st = P.systems[sys];
            rootEntry         = st.entry;
            // a system's groups meet only its own bodies: its own softening range decides
            if (lane == 0)
            {
                S.allUniform  = T.uniformH && st.hLo == st.hHi && orderedFloat(st.hLo) == T.h0;
                S.uniformMass = st.mLo == st.mHi;
                S.massU       = S.uniformMass ? orderedFloat(st.mLo) : 0.f;
            }
            shells            = st.numShells;
            boxL[0]           = st.boxL[0];
            boxL[1]           = st.boxL[1];
            boxL[2]           = st.boxL[2];
        }

        unsigned nM2P = 0, nP2P = 0;
        int maxStack  = 0;
        bool overflow = false, heavy = false;
        const bool mayQueue = P.parts == 0 && P.heavyGroups != nullptr;
        for (int iz = -shells; iz <= shells && !overflow; ++iz)
            for (int iy = -shells; iy <= shells && !overflow; ++iy)
                for (int ix = -shells; ix <= shells && !overflow; ++ix)
                {
                    // the replica shift is added to and later subtracted from the group centre, as in the
                    // reference (traversal_gpu.cu:484-505), so the MAC decisions are the reference's. The targets
                    // are the original positions plus the shift: shifting them back and forth as the reference
                    // does leaves rounding residues, and a target then meets itself at about one float ulp of the
                    // box coordinates, which a softening below that turns into a large spurious force.
                    float sh[3] = {__fmul_rn(float(ix), boxL[0]), __fmul_rn(float(iy), boxL[1]),
                                   __fmul_rn(float(iz), boxL[2])};
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        tc[d] = __fadd_rn(tc[d], sh[d]);
                    if (shells > 0)
                    {
                        float4 u0 = tgt.vec(min(b + lane, e - 1));
                        float4 u1 = tgt.vec(min(b + kWarp + lane, e - 1));
                        T.tx      = add2(pk(u0.x, u1.x), pk(sh[0], sh[0]));
                        T.ty      = add2(pk(u0.y, u1.y), pk(sh[1], sh[1]));
                        T.tz      = add2(pk(u0.z, u1.z), pk(sh[2], sh[2]));
                    }

                    int sp = 1, nM = 0, nL = 0;
                    if (lane == 0) stack[0] = rootEntry;
                    __syncwarp();
                    while (sp > 0)
                    {
                        int k     = min(4, sp);
                        sp -= k;
                        int slot  = lane >> 3;
                        int entry = slot < k ? stack[sp + slot] : -1;
                        __syncwarp();
                        int cell = -1;
                        if (entry <= kRootOnly) cell = (lane & 7) == 0 ? kRootOnly - entry : -1;
                        else if (entry >= 0) cell = entry + (lane & 7);

                        bool valid = cell >= 0;
                        float4 c   = make_float4(0.f, 0.f, 0.f, 0.f);
                        int4 link  = make_int4(0, 0, 0, 0);
                        if (valid) nodes.load(cell, c, link);
                        bool close  = valid && macFails(c, tc, ts);
                        bool isNode = link.x != 0;
                        bool split  = close && isNode;
                        unsigned bs = __ballot_sync(0xffffffffu, split);
                        int nsplit  = __popc(bs);
                        if (sp + nsplit > P.stackCapacity)
                        {
                            overflow = true;
                            break;
                        }
                        if (split) stack[sp + __popc(bs & lt)] = link.x;
                        sp += nsplit;
                        maxStack = max(maxStack, sp);

                        bool direct = close && !isNode;
                        bool remote = direct && link.z == 0 && c.w != 0.f;
                        bool approx = valid && (!close || remote);
                        nM2P += __popc(__ballot_sync(0xffffffffu, approx));

                        bool evalM  = approx && c.w != 0.f; // massless cells contribute exactly zero
                        unsigned bm = __ballot_sync(0xffffffffu, evalM);
                        if (evalM) S.m2p[nM + __popc(bm & lt)] = cell;
                        nM += __popc(bm);

                        bool hasB   = direct && link.z > 0;
                        unsigned bl = __ballot_sync(0xffffffffu, hasB);
                        if (hasB) S.leaves[nL + __popc(bl & lt)] = make_int2(link.y, link.z);
                        nL += __popc(bl);
                        nP2P += __reduce_add_sync(0xffffffffu, hasB ? unsigned(link.z) : 0u);
                        __syncwarp();
                        if (mayQueue && nP2P + 2u * nM2P > P.heavyCost)
                        {
                            // too much for one warp: leave it to the split second pass
                            heavy    = true;
                            overflow = true;
                            break;
                        }

                        constexpr int kMB = m2pBatch<Nodes>();
                        while (nM >= kMB)
                        {
                            evalM2P<kSplit>(S, kMB, nodes, T);
                            nM -= kMB; // fewer than kWarp cells remain: one move per lane
                            if (lane < nM) S.m2p[lane] = S.m2p[kMB + lane];
                            __syncwarp();
                        }
                        if (nL > kLeafCap - kWarp) nL = evalP2P<kSplit>(S, nL, false, src, T);
                    }
                    if (!overflow)
                    {
                        if (nM > 0) evalM2P<kSplit>(S, nM, nodes, T);
                        if (nL > 0) evalP2P<kSplit>(S, nL, true, src, T);
                    }
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        tc[d] = __fsub_rn(tc[d], sh[d]);
                }

        if (heavy)
        {
            if (lane == 0)
            {
                unsigned slotH = atomicAdd(&P.ctl->heavyCount, 1u);
                if (slotH < P.heavyCapacity) P.heavyGroups[slotH] = g;
            }
            continue;
        }
        if (overflow)
        {
            // write nothing; the host splits the group and traverses the halves again (in the second pass the
            // combine step reports the group)
            if (P.parts > 0)
            {
                if (lane == 0) P.partStatus[S.item] = 1;
                if (S.part != 0) continue;
            }
            if (lane == 0)
            {
                if (P.parts == 0)
                {
                    unsigned slotF = atomicAdd(&P.ctl->failedCount, 1u);
                    if (slotF < P.failedCapacity) P.failedGroups[slotF] = g;
                }
                atomicMax(&P.ctl->stats[kMaxStack], (unsigned long long)maxStack);
            }
            continue;
        }

        // Kahan: the compensated sum is acc - comp; acc.p holds -phi
        float phi[2], gx[2], gy[2], gz[2];
        upk(sub2(S.sums[1][0][lane], S.sums[0][0][lane]), phi[0], phi[1]);
        upk(sub2(S.sums[0][1][lane], S.sums[1][1][lane]), gx[0], gx[1]);
        upk(sub2(S.sums[0][2][lane], S.sums[1][2][lane]), gy[0], gy[1]);
        upk(sub2(S.sums[0][3][lane], S.sums[1][3][lane]), gz[0], gz[1]);
        double pot = 0.0;
        if (P.parts > 0)
        {
            // this part's share; the combine step adds the parts in order. Every part walked the whole group, so
            // part 0 reports the group's interaction counts.
            float4* out       = P.partials + size_t(S.item) * (2 * kWarp);
            out[lane]         = make_float4(phi[0], gx[0], gy[0], gz[0]);
            out[kWarp + lane] = make_float4(phi[1], gx[1], gy[1], gz[1]);
            if (lane == 0) P.partStatus[S.item] = 0;
            if (S.part != 0) continue;
        }
        else
        {
#pragma unroll
            for (int k = 0; k < 2; ++k)
            {
                int idx = b + k * kWarp + lane;
                if (idx < e)
                {
                    float mi = tgt.scalar(idx);
                    pot += double(mi) * double(phi[k]);
                    storeResult(P, idx, P.G * mi * phi[k], P.G * gx[k], P.G * gy[k], P.G * gz[k]);
                }
            }
            pot = warpSum(pot);
        }
        if (lane == 0)
        {
            unsigned long long size = (unsigned long long)(e - b);
            atomicMax(&P.ctl->stats[kMaxP2P], (unsigned long long)nP2P);
            atomicAdd(&P.ctl->stats[kSumP2P], (unsigned long long)nP2P * size);
            atomicMax(&P.ctl->stats[kMaxM2P], (unsigned long long)nM2P);
            atomicAdd(&P.ctl->stats[kSumM2P], (unsigned long long)nM2P * size);
            atomicMax(&P.ctl->stats[kMaxStack], (unsigned long long)maxStack);
            if (P.parts == 0)
            {
                atomicAdd(&P.ctl->potential, pot);
                if (P.sysPotential) atomicAdd(P.sysPotential + sys, pot);
            }
            if (P.groupM2P) P.groupM2P[g] = nM2P;
            if (P.groupP2P) P.groupP2P[g] = nP2P;
        }
    }
}

template<class Nodes, class Targets, class Sources>
static void launchTyped(const TraverseLaunch& t, const Nodes& nodes, const Targets& tgt, const Sources& src,
                        int smCount, cudaStream_t s)
{
    auto kernel = t.parts > 0 ? traverseKernel<Nodes, Targets, Sources, true>
                              : traverseKernel<Nodes, Targets, Sources, false>;
    size_t smem = sizeof(int) * kTravWarps * size_t(t.stackCapacity) + sizeof(WarpSmem) * kTravWarps;
    RYO_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int perSm = 0;
    RYO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, kTravThreads, smem));
    if (perSm < 1) perSm = 1;
    int items  = t.parts > 0 ? int(t.numHeavy) * t.parts : t.numGroups;
    int want   = (items + kTravWarps - 1) / kTravWarps;
    int blocks = min(want, perSm * smCount);
    kernel<<<blocks, kTravThreads, smem, s>>>(t, nodes, tgt, src);
    RYO_LAUNCH_CHECK();
}

void launchTraverse(const TraverseLaunch& t, int smCount, cudaStream_t s)
{
    if (t.numGroups <= 0 || (t.parts > 0 && t.numHeavy == 0)) return;
    if (t.precision != kPrecisionF32)
    {
        launchTraverse64(t, smCount, s);
        return;
    }
    if (t.nodes)
    {
        PackedBodies tgt{t.tgtXYZH, t.tgtM}, src{t.srcXYZM, t.srcH};
        if (t.dipoles)
        {
            RecordNodesMDQ nodes;
            nodes.r   = t.nodes;
            nodes.dip = t.dipoles;
            launchTyped(t, nodes, tgt, src, smCount, s);
        }
        else
            launchTyped(t, RecordNodes{t.nodes}, tgt, src, smCount, s);
    }
    else
    {
        ArrayNodes nodes{t.centers, reinterpret_cast<const float4*>(t.multipoles), t.childOffsets, t.internalToLeaf,
                         t.layout};
        SoABodies tgt{t.xt, t.yt, t.zt, t.ht, t.mt}, src{t.xs, t.ys, t.zs, t.ms, t.hs};
        if (t.mdqArrays)
        {
            ArrayNodesMDQ mdq;
            static_cast<ArrayNodes&>(mdq) = nodes;
            launchTyped(t, mdq, tgt, src, smCount, s);
        }
        else
            launchTyped(t, nodes, tgt, src, smCount, s);
    }
}

} // namespace ryo
