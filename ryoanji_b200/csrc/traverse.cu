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
 *     compaction and evaluated in dense batches of 32 cells or 32 bodies whose data is staged in shared memory and
 *     read with broadcast loads, so the inner loops are FP32 arithmetic plus one rsqrt per interaction;
 *   - each batch accumulates into fresh registers and is added to the per-target sums with Kahan compensation;
 *   - the MAC test uses explicitly rounded single operations so that every decision is reproducible bit for bit.
 */
#include "internal.hpp"

namespace ryo
{

constexpr int kTravWarps    = 4;
constexpr int kTravThreads  = kTravWarps * kWarp;
constexpr int kStackDefault = 1024;
constexpr int kM2PCap       = 64;  // pending approximated cells (flushed at 32)
constexpr int kLeafCap      = 64;  // pending direct leaves (flushed when more than 32 are pending)
constexpr int kRootOnly     = -2;  // stack marker: the root itself is the only cell (single-leaf tree)

struct WarpSmem
{
    int m2p[kM2PCap + kWarp];
    int2 leaves[kLeafCap + kWarp];
    int leafScan[kLeafCap + kWarp];
    float4 stage[3 * kWarp];
    float stageH[kWarp];
};

__device__ __forceinline__ float rsqrtApprox(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ void kahanAdd(float& sum, float& comp, float v)
{
    float y = __fsub_rn(v, comp);
    float t = __fadd_rn(sum, y);
    comp    = __fsub_rn(__fsub_rn(t, sum), y);
    sum     = t;
}

//! the reference's applyMAC (traversal_gpu.cu:77-84) with every operation rounded once
__device__ __forceinline__ bool macFails(float4 c, const float tc[3], const float ts[3])
{
    float dx = __fsub_rn(fabsf(__fsub_rn(tc[0], c.x)), ts[0]);
    float dy = __fsub_rn(fabsf(__fsub_rn(tc[1], c.y)), ts[1]);
    float dz = __fsub_rn(fabsf(__fsub_rn(tc[2], c.z)), ts[2]);
    dx       = __fmul_rn(__fadd_rn(dx, fabsf(dx)), 0.5f);
    dy       = __fmul_rn(__fadd_rn(dy, fabsf(dy)), 0.5f);
    dz       = __fmul_rn(__fadd_rn(dz, fabsf(dz)), 0.5f);
    return norm2Exact(dx, dy, dz) < c.w;
}

//! M2P of one quadrupole (cartesian_qpole.hpp:152-176) into acc = (pot, ax, ay, az)
__device__ __forceinline__ void m2p(float4& acc, float tx, float ty, float tz, float4 c, float4 q0, float4 q1)
{
    float rx = tx - c.x, ry = ty - c.y, rz = tz - c.z;
    float r2  = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
    float rm1 = rsqrtApprox(r2);
    float rm2 = rm1 * rm1;
    float rm5 = rm2 * rm2 * rm1;
    // q0 = (m, qxx, qxy, qxz), q1 = (qyy, qyz, qzz, trace)
    float Qrx = fmaf(rx, q0.y, fmaf(ry, q0.z, rz * q0.w));
    float Qry = fmaf(rx, q0.z, fmaf(ry, q1.x, rz * q1.y));
    float Qrz = fmaf(rx, q0.w, fmaf(ry, q1.y, rz * q1.z));
    float rQr = fmaf(rx, Qrx, fmaf(ry, Qry, rz * Qrz));
    float mr1 = q0.x * rm1;
    float f   = fmaf(-2.5f * rQr, rm5, -mr1) * rm2;
    acc.x -= fmaf(0.5f * rm5, rQr, mr1);
    acc.y = fmaf(rm5, Qrx, fmaf(f, rx, acc.y));
    acc.z = fmaf(rm5, Qry, fmaf(f, ry, acc.z));
    acc.w = fmaf(rm5, Qrz, fmaf(f, rz, acc.w));
}

//! P2P (kernel.hpp:99-120) into acc = (pot, ax, ay, az)
__device__ __forceinline__ void p2p(float4& acc, float4 ti, float4 sj, float hj)
{
    float dx   = sj.x - ti.x, dy = sj.y - ti.y, dz = sj.z - ti.z;
    float r2   = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    float hij  = ti.w + hj;
    float r2e  = fmaxf(r2, hij * hij);
    float invR = rsqrtApprox(r2e);
    float m3   = sj.w * invR * (invR * invR);
    acc.x      = fmaf(-m3, r2, acc.x);
    acc.y      = fmaf(dx, m3, acc.y);
    acc.z      = fmaf(dy, m3, acc.z);
    acc.w      = fmaf(dz, m3, acc.w);
}

struct TargetState
{
    float4 ti[2];   // x, y, z, h of the two targets of this lane (shifted by the current replica)
    float4 acc[2];  // pot, ax, ay, az
    float4 comp[2]; // Kahan compensation
};

//! node data from the packed 64-byte records of the solver path
struct RecordNodes
{
    const NodeRecord* __restrict__ r;
    __device__ __forceinline__ void load(int cell, float4& c, int4& link) const
    {
        c    = __ldg(&r[cell].center);
        link = __ldg(&r[cell].link);
    }
    __device__ __forceinline__ void multipole(int cell, float4& c, float4& q0, float4& q1) const
    {
        c  = __ldg(&r[cell].center);
        q0 = __ldg(&r[cell].q0);
        q1 = __ldg(&r[cell].q1);
    }
};

//! node data from the reference's separate arrays (centres, multipoles, childOffsets, internalToLeaf, layout)
struct ArrayNodes
{
    const float4* __restrict__ centers;
    const float4* __restrict__ mpoles; // two float4 per node
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
    __device__ __forceinline__ void multipole(int cell, float4& c, float4& q0, float4& q1) const
    {
        c  = __ldg(centers + cell);
        q0 = __ldg(mpoles + 2 * cell);
        q1 = __ldg(mpoles + 2 * cell + 1);
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

__device__ __forceinline__ void addBatch(TargetState& T, const float4 part[2])
{
#pragma unroll
    for (int k = 0; k < 2; ++k)
    {
        kahanAdd(T.acc[k].x, T.comp[k].x, part[k].x);
        kahanAdd(T.acc[k].y, T.comp[k].y, part[k].y);
        kahanAdd(T.acc[k].z, T.comp[k].z, part[k].z);
        kahanAdd(T.acc[k].w, T.comp[k].w, part[k].w);
    }
}

//! evaluate the first @p count (<= 32) pending cells
template<class Nodes>
__device__ void evalM2P(WarpSmem& S, int count, const Nodes& nodes, TargetState& T)
{
    int lane = laneId();
    if (lane < count)
    {
        float4 c, q0, q1;
        nodes.multipole(S.m2p[lane], c, q0, q1);
        S.stage[3 * lane]     = c;
        S.stage[3 * lane + 1] = q0;
        S.stage[3 * lane + 2] = q1;
    }
    __syncwarp();
    float4 part[2] = {make_float4(0.f, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f)};
    if (count == kWarp)
    {
#pragma unroll 4
        for (int j = 0; j < kWarp; ++j)
        {
            float4 c = S.stage[3 * j], q0 = S.stage[3 * j + 1], q1 = S.stage[3 * j + 2];
            m2p(part[0], T.ti[0].x, T.ti[0].y, T.ti[0].z, c, q0, q1);
            m2p(part[1], T.ti[1].x, T.ti[1].y, T.ti[1].z, c, q0, q1);
        }
    }
    else
    {
        for (int j = 0; j < count; ++j)
        {
            float4 c = S.stage[3 * j], q0 = S.stage[3 * j + 1], q1 = S.stage[3 * j + 2];
            m2p(part[0], T.ti[0].x, T.ti[0].y, T.ti[0].z, c, q0, q1);
            m2p(part[1], T.ti[1].x, T.ti[1].y, T.ti[1].z, c, q0, q1);
        }
    }
    addBatch(T, part);
    __syncwarp();
}

/*! evaluate pending direct leaves in batches of 32 bodies; with @p all == false only whole batches are evaluated
 *  and the remainder stays pending (the first pending leaf may be partly consumed). Returns the leaves left. */
template<class Sources>
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
    int numBatches = all ? (total + kWarp - 1) / kWarp : total / kWarp;
    for (int b = 0; b < numBatches; ++b)
    {
        int r = b * kWarp + lane;
        if (r < total)
        {
            // first leaf whose inclusive prefix exceeds r
            int lo = 0, hi = numLeaves - 1;
            while (lo < hi)
            {
                int mid = (lo + hi) >> 1;
                if (S.leafScan[mid] > r) hi = mid;
                else lo = mid + 1;
            }
            int2 lf    = S.leaves[lo];
            int body   = lf.x + (r - (S.leafScan[lo] - lf.y));
            S.stage[lane]  = src.vec(body);
            S.stageH[lane] = src.scalar(body);
        }
        __syncwarp();
        int nvalid     = min(kWarp, total - b * kWarp);
        float4 part[2] = {make_float4(0.f, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f)};
        if (nvalid == kWarp)
        {
#pragma unroll 8
            for (int j = 0; j < kWarp; ++j)
            {
                float4 sj = S.stage[j];
                float hj  = S.stageH[j];
                p2p(part[0], T.ti[0], sj, hj);
                p2p(part[1], T.ti[1], sj, hj);
            }
        }
        else
        {
            for (int j = 0; j < nvalid; ++j)
            {
                float4 sj = S.stage[j];
                float hj  = S.stageH[j];
                p2p(part[0], T.ti[0], sj, hj);
                p2p(part[1], T.ti[1], sj, hj);
            }
        }
        addBatch(T, part);
        __syncwarp();
    }
    if (all) return 0;
    // keep bodies [numBatches * 32, total): drop fully consumed leaves, trim the first kept one
    int done = numBatches * kWarp;
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

template<class Nodes, class Targets, class Sources>
__global__ void __launch_bounds__(kTravThreads)
    traverseKernel(TraverseLaunch P, Nodes nodes, Targets tgt, Sources src)
{
    extern __shared__ __align__(16) unsigned char smemRaw[];
    const int warp = threadIdx.x / kWarp, lane = laneId();
    int* stack     = reinterpret_cast<int*>(smemRaw) + warp * P.stackCapacity;
    WarpSmem& S    = reinterpret_cast<WarpSmem*>(smemRaw + sizeof(int) * kTravWarps * P.stackCapacity)[warp];
    const unsigned lt = lanemaskLt();

    while (true)
    {
        unsigned g = 0;
        if (lane == 0) g = atomicAdd(&P.ctl->workCounter, 1u);
        g = __shfl_sync(0xffffffffu, g, 0);
        if (g >= unsigned(P.numGroups)) return;

        const int b = int(P.groupStart[g]), e = int(P.groupEnd[g]);
        TargetState T;
        float lo[3], hi[3];
#pragma unroll
        for (int k = 0; k < 2; ++k)
        {
            int idx  = min(b + k * kWarp + lane, e - 1);
            T.ti[k]  = tgt.vec(idx);
            T.acc[k]  = make_float4(0.f, 0.f, 0.f, 0.f);
            T.comp[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        lo[0] = fminf(T.ti[0].x, T.ti[1].x);
        lo[1] = fminf(T.ti[0].y, T.ti[1].y);
        lo[2] = fminf(T.ti[0].z, T.ti[1].z);
        hi[0] = fmaxf(T.ti[0].x, T.ti[1].x);
        hi[1] = fmaxf(T.ti[0].y, T.ti[1].y);
        hi[2] = fmaxf(T.ti[0].z, T.ti[1].z);
        float tc[3], ts[3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            float l = warpMin(lo[d]), h = warpMax(hi[d]);
            tc[d]   = __fmul_rn(__fadd_rn(h, l), 0.5f);
            ts[d]   = __fmul_rn(__fsub_rn(h, l), 0.5f);
        }

        unsigned nM2P = 0, nP2P = 0;
        int maxStack  = 0;
        bool overflow = false;
        for (int iz = -P.numShells; iz <= P.numShells && !overflow; ++iz)
            for (int iy = -P.numShells; iy <= P.numShells && !overflow; ++iy)
                for (int ix = -P.numShells; ix <= P.numShells && !overflow; ++ix)
                {
                    // the replica shift is added to and later subtracted from centre and targets (as in the reference)
                    float sh[3] = {__fmul_rn(float(ix), P.boxL[0]), __fmul_rn(float(iy), P.boxL[1]),
                                   __fmul_rn(float(iz), P.boxL[2])};
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        tc[d] = __fadd_rn(tc[d], sh[d]);
#pragma unroll
                    for (int k = 0; k < 2; ++k)
                    {
                        T.ti[k].x = __fadd_rn(T.ti[k].x, sh[0]);
                        T.ti[k].y = __fadd_rn(T.ti[k].y, sh[1]);
                        T.ti[k].z = __fadd_rn(T.ti[k].z, sh[2]);
                    }

                    int sp = 1, nM = 0, nL = 0;
                    if (lane == 0) stack[0] = P.numNodes == 1 ? kRootOnly : P.initNode;
                    __syncwarp();
                    while (sp > 0)
                    {
                        int k     = min(4, sp);
                        sp -= k;
                        int slot  = lane >> 3;
                        int entry = slot < k ? stack[sp + slot] : -1;
                        __syncwarp();
                        int cell = -1;
                        if (entry == kRootOnly) cell = (lane & 7) == 0 ? 0 : -1;
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

                        while (nM >= kWarp)
                        {
                            evalM2P(S, kWarp, nodes, T);
                            nM -= kWarp;
                            if (lane < nM) S.m2p[lane] = S.m2p[kWarp + lane];
                            __syncwarp();
                        }
                        if (nL > kLeafCap - kWarp) nL = evalP2P(S, nL, false, src, T);
                    }
                    if (!overflow)
                    {
                        if (nM > 0) evalM2P(S, nM, nodes, T);
                        if (nL > 0) evalP2P(S, nL, true, src, T);
                    }
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        tc[d] = __fsub_rn(tc[d], sh[d]);
#pragma unroll
                    for (int k = 0; k < 2; ++k)
                    {
                        T.ti[k].x = __fsub_rn(T.ti[k].x, sh[0]);
                        T.ti[k].y = __fsub_rn(T.ti[k].y, sh[1]);
                        T.ti[k].z = __fsub_rn(T.ti[k].z, sh[2]);
                    }
                }

        if (overflow)
        {
            // write nothing; the host splits the group and traverses the halves again
            if (lane == 0)
            {
                unsigned slotF = atomicAdd(&P.ctl->failedCount, 1u);
                if (slotF < P.failedCapacity) P.failedGroups[slotF] = g;
                atomicMax(&P.ctl->stats[kMaxStack], (unsigned long long)maxStack);
            }
            continue;
        }

        double pot = 0.0;
#pragma unroll
        for (int k = 0; k < 2; ++k)
        {
            int idx = b + k * kWarp + lane;
            if (idx < e)
            {
                // Kahan: the compensated sum is acc - comp
                float mi  = tgt.scalar(idx);
                float phi = __fsub_rn(T.acc[k].x, T.comp[k].x);
                pot += double(mi) * double(phi);
                if (P.p) P.p[idx] += P.G * mi * phi;
                P.ax[idx] += P.G * __fsub_rn(T.acc[k].y, T.comp[k].y);
                P.ay[idx] += P.G * __fsub_rn(T.acc[k].z, T.comp[k].z);
                P.az[idx] += P.G * __fsub_rn(T.acc[k].w, T.comp[k].w);
            }
        }
        pot = warpSum(pot);
        if (lane == 0)
        {
            unsigned long long size = (unsigned long long)(e - b);
            atomicMax(&P.ctl->stats[kMaxP2P], (unsigned long long)nP2P);
            atomicAdd(&P.ctl->stats[kSumP2P], (unsigned long long)nP2P * size);
            atomicMax(&P.ctl->stats[kMaxM2P], (unsigned long long)nM2P);
            atomicAdd(&P.ctl->stats[kSumM2P], (unsigned long long)nM2P * size);
            atomicMax(&P.ctl->stats[kMaxStack], (unsigned long long)maxStack);
            atomicAdd(&P.ctl->potential, pot);
            if (P.groupM2P) P.groupM2P[g] = nM2P;
            if (P.groupP2P) P.groupP2P[g] = nP2P;
        }
    }
}

template<class Nodes, class Targets, class Sources>
static void launchTyped(const TraverseLaunch& t, const Nodes& nodes, const Targets& tgt, const Sources& src,
                        int smCount, cudaStream_t s)
{
    auto kernel = traverseKernel<Nodes, Targets, Sources>;
    size_t smem = sizeof(int) * kTravWarps * size_t(t.stackCapacity) + sizeof(WarpSmem) * kTravWarps;
    RYO_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int perSm = 0;
    RYO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, kTravThreads, smem));
    if (perSm < 1) perSm = 1;
    int want   = (t.numGroups + kTravWarps - 1) / kTravWarps;
    int blocks = min(want, perSm * smCount);
    kernel<<<blocks, kTravThreads, smem, s>>>(t, nodes, tgt, src);
    RYO_LAUNCH_CHECK();
}

void launchTraverse(const TraverseLaunch& t, int smCount, cudaStream_t s)
{
    if (t.numGroups <= 0) return;
    if (t.nodes)
    {
        RecordNodes nodes{t.nodes};
        PackedBodies tgt{t.tgtXYZH, t.tgtM}, src{t.srcXYZM, t.srcH};
        launchTyped(t, nodes, tgt, src, smCount, s);
    }
    else
    {
        ArrayNodes nodes{t.centers, reinterpret_cast<const float4*>(t.multipoles), t.childOffsets, t.internalToLeaf,
                         t.layout};
        SoABodies tgt{t.xt, t.yt, t.zt, t.ht, t.mt}, src{t.xs, t.ys, t.zs, t.ms, t.hs};
        launchTyped(t, nodes, tgt, src, smCount, s);
    }
}

} // namespace ryo
