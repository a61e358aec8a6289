/*
 * ryoanji-b200: kernels of the batched solve (many independent systems, one launch per phase).
 *
 * The systems are concatenated: system s owns the bodies [first[s], first[s + 1]). Each body's key is its system
 * index in the top 3L bits (L = sysLevel octree levels) followed by the top 63 - 3L bits of its Hilbert key in the
 * system's own box. Sorting these keys sorts every system along its own curve and keeps the systems in place; the
 * cornerstone tree over them holds each system's tree below the level-L node of its prefix (leaves holding bodies
 * are forced to level >= L so no leaf spans two systems). A system's tree equals its stand-alone tree wherever
 * the stand-alone tree stops above level 21 - L.
 *
 * The reference solves one system per call (ryoanji/test/demo.cu:82-104); there is no batched counterpart.
 */
#include "internal.hpp"

namespace ryo
{

//! system of body i: the last s with first[s] <= i
__device__ __forceinline__ uint32_t systemOf(const uint64_t* __restrict__ first, uint32_t numSystems, uint64_t i)
{
    uint32_t lo = 0, hi = numSystems - 1;
    while (lo < hi)
    {
        uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(first + mid) <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

constexpr int kMinMaxChunk = 64;

//! per-system coordinate min/max: each thread scans a chunk of consecutive bodies and flushes at system changes
__global__ void batchMinMaxKernel(const float* __restrict__ x, const float* __restrict__ y,
                                  const float* __restrict__ z, size_t n, const uint64_t* __restrict__ first,
                                  uint32_t numSystems, uint32_t* __restrict__ mm)
{
    size_t c0 = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) * kMinMaxChunk;
    if (c0 >= n) return;
    size_t c1    = c0 + kMinMaxChunk < n ? c0 + kMinMaxChunk : n;
    uint32_t sys = systemOf(first, numSystems, c0);
    uint64_t end = __ldg(first + sys + 1);
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    auto flush = [&]()
    {
        uint32_t* m = mm + 6 * size_t(sys);
        for (int d = 0; d < 3; ++d)
        {
            atomicMin(m + 2 * d, orderedBits(lo[d]));
            atomicMax(m + 2 * d + 1, orderedBits(hi[d]));
            lo[d] = INFINITY;
            hi[d] = -INFINITY;
        }
    };
    for (size_t i = c0; i < c1; ++i)
    {
        if (i >= end)
        {
            flush();
            while (i >= end)
            {
                ++sys;
                end = __ldg(first + sys + 1);
            }
        }
        float v[3] = {x[i], y[i], z[i]};
        for (int d = 0; d < 3; ++d)
        {
            lo[d] = fminf(lo[d], v[d]);
            hi[d] = fmaxf(hi[d], v[d]);
        }
    }
    flush();
}

__global__ void batchMinMaxInit(uint32_t* mm, uint32_t numSystems)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 6 * numSystems) mm[i] = (i & 1) ? 0u : 0xffffffffu;
}

/*! the cube enclosing each system whose box is not given, as the single-system solve derives it: lower corner at the
 *  minimum, edge = largest extent (FP64), upper limit rounded up to cover the maximum */
__global__ void batchAutoBoxes(const uint32_t* __restrict__ mm, const int* __restrict__ useGiven, uint32_t numSystems,
                               DevBox<float>* __restrict__ boxes, float* __restrict__ limits)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= numSystems || useGiven[s]) return;
    float mn[3], mx[3];
    double ext = 0.0;
    for (int d = 0; d < 3; ++d)
    {
        mn[d] = orderedFloat(mm[6 * s + 2 * d]);
        mx[d] = orderedFloat(mm[6 * s + 2 * d + 1]);
        ext   = fmax(ext, double(mx[d]) - double(mn[d]));
    }
    if (!(ext > 0)) ext = 1.0;
    DevBox<float> b;
    for (int d = 0; d < 3; ++d)
    {
        float lo = mn[d];
        float hi = float(double(mn[d]) + ext);
        if (!(hi >= mx[d])) hi = nextafterf(mx[d], 3.4e38f);
        limits[6 * s + 2 * d]     = lo;
        limits[6 * s + 2 * d + 1] = hi;
        b.lo[d]                   = lo;
        b.len[d]                  = hi - lo;
        b.inv[d]                  = 1.f / (hi - lo);
        b.bits[d]                 = kMaxLevel; // a cube: no axis is reduced
    }
    b.periodic = 0;
    boxes[s]   = b;
}

//! the two-level Hilbert tables (identical keys to hilbert3), built at compile time
static __device__ const HilbertLut kBatchHilbertLut = makeHilbertLut();

__global__ void __launch_bounds__(256) batchKeysKernel(const float* __restrict__ x, const float* __restrict__ y,
                                                       const float* __restrict__ z, size_t n,
                                                       const uint64_t* __restrict__ first, uint32_t numSystems,
                                                       const DevBox<float>* __restrict__ boxes, int sysBits,
                                                       uint64_t* __restrict__ keys)
{
    __shared__ uint16_t two[48 * 64];
    __shared__ uint16_t one[48 * 8];
    for (int i = threadIdx.x; i < 48 * 64; i += blockDim.x)
        two[i] = kBatchHilbertLut.two[i];
    for (int i = threadIdx.x; i < 48 * 8; i += blockDim.x)
        one[i] = kBatchHilbertLut.one[i];
    __syncthreads();
    size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    {
        uint32_t s           = systemOf(first, numSystems, i);
        const DevBox<float>& b = boxes[s];
        unsigned ic[3];
        pointCells(x[i], y[i], z[i], b, ic);
        bool full  = b.bits[0] == unsigned(kMaxLevel) && b.bits[1] == unsigned(kMaxLevel) &&
                    b.bits[2] == unsigned(kMaxLevel);
        uint64_t k = full ? hilbert3Lut(ic[0], ic[1], ic[2], two, one) : hilbertKey(ic[0], ic[1], ic[2], b.bits);
        keys[i]    = (uint64_t(s) << (63 - sysBits)) | (k >> sysBits);
    }
}

/*! each system's root node (the level-L node of its prefix) and its first stack entry; flags a missing root */
__global__ void batchRootsKernel(uint32_t numSystems, const uint64_t* __restrict__ prefixes, int levelBegin,
                                 int levelEnd, const int* __restrict__ childOffsets, int sysLevel,
                                 const DevBox<float>* __restrict__ boxes, const int* __restrict__ numShells,
                                 SysTrav* __restrict__ out, int* __restrict__ rootNode, unsigned int* __restrict__ err)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= numSystems) return;
    int sysBits     = 3 * sysLevel;
    uint64_t target = encodePrefix(uint64_t(s) << (63 - sysBits), sysBits);
    int lo = levelBegin, hi = levelEnd;
    while (lo < hi)
    {
        int mid = (lo + hi) >> 1;
        if (prefixes[mid] < target) lo = mid + 1;
        else hi = mid;
    }
    SysTrav t;
    if (lo < levelEnd && prefixes[lo] == target)
    {
        int fc  = childOffsets[lo];
        t.entry = fc != 0 ? fc : -(lo + 2);
        if (rootNode) rootNode[s] = lo;
    }
    else
    {
        t.entry = -1; // nothing to traverse; reported as an error
        if (rootNode) rootNode[s] = -1;
        atomicExch(err, 1u);
    }
    t.numShells = numShells[s];
    t.boxL[0]   = boxes[s].len[0];
    t.boxL[1]   = boxes[s].len[1];
    t.boxL[2]   = boxes[s].len[2];
    t.hLo       = 0xffffffffu; // filled by batchSofteningRange
    t.hHi       = 0u;
    t.mLo       = 0xffffffffu;
    t.mHi       = 0u;
    out[s]      = t;
}

//! fixed groups of at most @p groupSize bodies inside every system
__global__ void batchGroupsKernel(uint32_t numGroups, const uint64_t* __restrict__ first,
                                  const uint32_t* __restrict__ groupOffset, uint32_t numSystems, uint32_t groupSize,
                                  uint32_t* __restrict__ start, uint32_t* __restrict__ end, uint32_t* __restrict__ sys)
{
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= numGroups) return;
    uint32_t lo = 0, hi = numSystems - 1;
    while (lo < hi)
    {
        uint32_t mid = (lo + hi + 1) >> 1;
        if (groupOffset[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    uint64_t b  = first[lo] + uint64_t(g - groupOffset[lo]) * groupSize;
    uint64_t e  = b + groupSize;
    uint64_t se = first[lo + 1];
    start[g]    = uint32_t(b);
    end[g]      = uint32_t(e < se ? e : se);
    sys[g]      = lo;
}

void launchBatchBoxes(const float* x, const float* y, const float* z, size_t n, const uint64_t* first,
                      uint32_t numSystems, const int* useGiven, uint32_t* mm, DevBox<float>* boxes, float* limits,
                      cudaStream_t s)
{
    batchMinMaxInit<<<ceilDiv(6 * numSystems, 256), 256, 0, s>>>(mm, numSystems);
    RYO_LAUNCH_CHECK();
    size_t threads = (n + kMinMaxChunk - 1) / kMinMaxChunk;
    batchMinMaxKernel<<<ceilDiv(threads, 256), 256, 0, s>>>(x, y, z, n, first, numSystems, mm);
    RYO_LAUNCH_CHECK();
    batchAutoBoxes<<<ceilDiv(numSystems, 128), 128, 0, s>>>(mm, useGiven, numSystems, boxes, limits);
    RYO_LAUNCH_CHECK();
}

void launchBatchKeys(const float* x, const float* y, const float* z, size_t n, const uint64_t* first,
                     uint32_t numSystems, const DevBox<float>* boxes, int sysLevel, uint64_t* keys, int smCount,
                     cudaStream_t s)
{
    size_t want = ceilDiv(n, 256);
    size_t cap  = size_t(smCount) * 16;
    batchKeysKernel<<<unsigned(want < cap ? want : cap), 256, 0, s>>>(x, y, z, n, first, numSystems, boxes,
                                                                      3 * sysLevel, keys);
    RYO_LAUNCH_CHECK();
}

//! one block per system: min and max softening and mass of its bodies (systems are contiguous runs of bodies)
__global__ void __launch_bounds__(256) batchSofteningRange(const float* __restrict__ h, const float* __restrict__ m,
                                                           const uint64_t* __restrict__ first, SysTrav* trav)
{
    __shared__ uint32_t sLo[2][8], sHi[2][8];
    const uint32_t s = blockIdx.x;
    uint32_t lo[2] = {0xffffffffu, 0xffffffffu}, hi[2] = {0u, 0u};
    for (uint64_t i = first[s] + threadIdx.x; i < first[s + 1]; i += blockDim.x)
    {
        uint32_t b = orderedBits(h[i]);
        lo[0]      = min(lo[0], b);
        hi[0]      = max(hi[0], b);
        if (m)
        {
            uint32_t c = orderedBits(m[i]);
            lo[1]      = min(lo[1], c);
            hi[1]      = max(hi[1], c);
        }
    }
    const unsigned warp = threadIdx.x / kWarp;
#pragma unroll
    for (int k = 0; k < 2; ++k)
    {
        lo[k] = __reduce_min_sync(0xffffffffu, lo[k]);
        hi[k] = __reduce_max_sync(0xffffffffu, hi[k]);
        if (laneId() == 0)
        {
            sLo[k][warp] = lo[k];
            sHi[k][warp] = hi[k];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        for (unsigned w = 1; w < blockDim.x / kWarp; ++w)
            for (int k = 0; k < 2; ++k)
            {
                lo[k] = min(lo[k], sLo[k][w]);
                hi[k] = max(hi[k], sHi[k][w]);
            }
        trav[s].hLo = lo[0];
        trav[s].hHi = hi[0];
        trav[s].mLo = lo[1];
        trav[s].mHi = hi[1];
    }
}

void launchBatchSofteningRange(const float* h, const float* m, const uint64_t* first, uint32_t numSystems,
                               SysTrav* trav, cudaStream_t s)
{
    if (numSystems == 0) return;
    batchSofteningRange<<<numSystems, 256, 0, s>>>(h, m, first, trav);
    RYO_LAUNCH_CHECK();
}

void launchBatchRoots(uint32_t numSystems, const uint64_t* prefixes, int levelBegin, int levelEnd,
                      const int* childOffsets, int sysLevel, const DevBox<float>* boxes, const int* numShells,
                      SysTrav* out, int* rootNode, unsigned int* err, cudaStream_t s)
{
    batchRootsKernel<<<ceilDiv(numSystems, 128), 128, 0, s>>>(numSystems, prefixes, levelBegin, levelEnd, childOffsets,
                                                               sysLevel, boxes, numShells, out, rootNode, err);
    RYO_LAUNCH_CHECK();
}

void launchBatchGroups(uint32_t numGroups, const uint64_t* first, const uint32_t* groupOffset, uint32_t numSystems,
                       uint32_t groupSize, uint32_t* start, uint32_t* end, uint32_t* sys, cudaStream_t s)
{
    if (numGroups == 0) return;
    batchGroupsKernel<<<ceilDiv(numGroups, 256), 256, 0, s>>>(numGroups, first, groupOffset, numSystems, groupSize,
                                                              start, end, sys);
    RYO_LAUNCH_CHECK();
}

} // namespace ryo
