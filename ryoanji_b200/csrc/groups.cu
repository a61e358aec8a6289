/*
 * ryoanji-b200: spatial target groups (cstone::computeGroupSplits, cstone/include/cstone/traversal/
 * groups_gpu.cuh:39-265 and groups_gpu.cu:60-151).
 *
 * The sorted targets are cut into fixed windows of 32 or 64; a window is split after target i when the next target
 * is farther than min(distCrit, 2 h_i) (distances in units of the longest box edge, distCrit = tolFactor times the
 * cube root of the smallest leaf volume met by the window, in the unit box of the same aspect ratio), and a window
 * whose extent along an axis exceeds extentRatio * tolFactor * its smallest leaf edge is also cut into equal
 * power-of-two chunks. The production caller of the reference (MultipoleHolder::computeSpatialGroups,
 * ryoanji/src/ryoanji/interface/multipole_holder.cu:36-53) uses tolFactor 2.
 *
 * B200 form: one warp per window, lane l holds targets l and l + 32 (the traversal's layout), split bits by
 * ballots, then one thread per window writes its subgroup starts at the offset given by a scan of the counts; no
 * host round trip between the two kernels apart from reading the group count.
 */
#include <cstdlib>

#include "internal.hpp"

namespace ryo
{

/*! The windows to split: fixed windows of G bodies over one range [first, last) of a single tree, or the windows
 *  of a batched solve (per-window bounds and system; each system's box; keys prefixed by the system index in the top
 *  3 * sysLevel bits, so a leaf's key and level within its system follow by dropping those bits). */
struct GroupWindows
{
    uint32_t first, last;      // single range, when start is null
    DevBox<float> unitBox;     // single range: the unit box of the box's aspect ratio
    float invMaxExtent;        // single range: 1 / the longest box edge
    const uint32_t* start;     // batch: window bounds and systems
    const uint32_t* end;
    const uint32_t* sys;
    const DevBox<float>* boxes; // batch: per-system boxes
    unsigned sysLevel;
};

//! bounds of window @p w, its system, and the system's unit box and inverse longest edge
__device__ inline void windowOf(const GroupWindows& W, uint32_t w, uint32_t G, uint32_t& wb, uint32_t& we,
                                uint32_t& sys, DevBox<float>& unitBox, float& invMaxExtent)
{
    if (!W.start)
    {
        wb           = W.first + w * G;
        we           = min(wb + G, W.last);
        sys          = 0;
        unitBox      = W.unitBox;
        invMaxExtent = W.invMaxExtent;
        return;
    }
    wb                  = W.start[w];
    we                  = W.end[w];
    sys                 = W.sys[w];
    const DevBox<float> b = W.boxes[sys];
    for (int d = 0; d < 3; ++d)
    {
        float len         = ldexpf(1.f, -int(kMaxLevel - b.bits[d])); // edge 2^-r for an axis reduced by r bits
        unitBox.lo[d]     = 0.f;
        unitBox.len[d]    = len;
        unitBox.inv[d]    = __frcp_rn(len);
        unitBox.bits[d]   = b.bits[d];
    }
    unitBox.periodic = 0;
    invMaxExtent     = __frcp_rn(fmaxf(fmaxf(b.len[0], b.len[1]), b.len[2]));
}

template<int NWT>
__global__ void __launch_bounds__(256)
    groupSplitsKernel(GroupWindows W, const float* __restrict__ x, const float* __restrict__ y,
                      const float* __restrict__ z, const float* __restrict__ h, const uint64_t* __restrict__ leaves,
                      int numLeaves, const uint32_t* __restrict__ layout, float tolFactor, float extentRatio,
                      uint32_t numWindows, unsigned long long* __restrict__ masks, uint32_t* __restrict__ counts)
{
    using F              = Fp<float>;
    constexpr uint32_t G = NWT * kWarp;
    const uint32_t w     = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
    const unsigned lane  = laneId();
    if (w >= numWindows) return; // whole warps leave together

    uint32_t wb, we, sys;
    DevBox<float> unitBox;
    float invMaxExtent;
    windowOf(W, w, G, wb, we, sys, unitBox, invMaxExtent);
    const unsigned sysBits = 3u * W.sysLevel;

    uint32_t body[NWT];
    float vol = 1.f, edge[3] = {1.f, 1.f, 1.f};
#pragma unroll
    for (int k = 0; k < NWT; ++k)
    {
        uint32_t b = wb + uint32_t(k) * kWarp + lane;
        body[k]    = b < we - 1 ? b : we - 1;
        // leaf holding the target: last leaf whose first body is <= it
        int lo = 0, hi = numLeaves; // upper_bound over layout[0, numLeaves)
        while (lo < hi)
        {
            int mid = (lo + hi) >> 1;
            if (layout[mid] <= body[k]) lo = mid + 1;
            else hi = mid;
        }
        int leaf    = lo - 1;
        uint64_t k0 = leaves[leaf], k1 = leaves[leaf + 1];
        unsigned lvl = unsigned(kMaxLevel) - unsigned(63 - clz64(k1 - k0)) / 3u - W.sysLevel;
        k0           = (k0 << sysBits) & ((1ull << 63) - 1ull); // the key within the system's own tree
        float c[3], s[3];
        nodeGeometry(k0, lvl, unitBox, c, s);
        float v = F::mul(F::mul(F::mul(8.f, s[0]), s[1]), s[2]);
        vol     = v > 0.f ? fminf(v, vol) : vol;
#pragma unroll
        for (int d = 0; d < 3; ++d)
            edge[d] = fminf(edge[d], F::mul(2.f, s[d]));
    }
    vol            = warpMin(vol);
    float distCrit = F::mul(cbrtf(vol), tolFactor);
    float dc2      = F::mul(distCrit, distCrit);

    float p[NWT][4];
#pragma unroll
    for (int k = 0; k < NWT; ++k)
    {
        uint32_t j = body[k];
        p[k][0]    = F::mul(x[j], invMaxExtent);
        p[k][1]    = F::mul(y[j], invMaxExtent);
        p[k][2]    = F::mul(z[j], invMaxExtent);
        p[k][3]    = h ? F::mul(F::mul(2.f, h[j]), invMaxExtent) : 1.f;
    }

    // split bits: distance from each target to the next one in the window
    unsigned mask[NWT];
#pragma unroll
    for (int k = 0; k < NWT; ++k)
    {
        float nx = __shfl_down_sync(0xffffffffu, p[k][0], 1);
        float ny = __shfl_down_sync(0xffffffffu, p[k][1], 1);
        float nz = __shfl_down_sync(0xffffffffu, p[k][2], 1);
        if (k + 1 < NWT)
        {
            float sx = __shfl_sync(0xffffffffu, p[k + 1 < NWT ? k + 1 : k][0], 0);
            float sy = __shfl_sync(0xffffffffu, p[k + 1 < NWT ? k + 1 : k][1], 0);
            float sz = __shfl_sync(0xffffffffu, p[k + 1 < NWT ? k + 1 : k][2], 0);
            if (lane == kWarp - 1)
            {
                nx = sx;
                ny = sy;
                nz = sz;
            }
        }
        float d2   = norm2Exact(F::sub(nx, p[k][0]), F::sub(ny, p[k][1]), F::sub(nz, p[k][2]));
        bool split = d2 > fminf(dc2, F::mul(p[k][3], p[k][3]));
        mask[k]    = __ballot_sync(0xffffffffu, split);
    }

    // windows much longer than their leaves along some axis: equal power-of-two chunks
    float ratio = 0.f;
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
        float lo = p[0][d], hi = p[0][d];
#pragma unroll
        for (int k = 1; k < NWT; ++k)
        {
            lo = fminf(lo, p[k][d]);
            hi = fmaxf(hi, p[k][d]);
        }
        float allowed = F::mul(tolFactor, warpMin(edge[d]));
        float extent  = F::sub(warpMax(hi), warpMin(lo));
        if (allowed > 0.f) ratio = fmaxf(ratio, __fdiv_rn(extent, allowed));
    }
    if (extentRatio > 0.f && ratio > extentRatio)
    {
        uint32_t chunk = G;
        while (chunk > 1 && F::mul(float(chunk), ratio) > F::mul(float(G), extentRatio))
            chunk >>= 1;
        uint32_t inWindow = we - wb;
#pragma unroll
        for (int k = 0; k < NWT; ++k)
        {
            uint32_t next = uint32_t(k) * kWarp + lane + 1;
            mask[k] |= __ballot_sync(0xffffffffu, next < inWindow && next % chunk == 0);
        }
    }
    if (lane == 0)
    {
        unsigned long long m = mask[0];
        if (NWT > 1) m |= (unsigned long long)(mask[NWT - 1]) << 32;
        masks[w]  = m;
        counts[w] = 1u + uint32_t(__popcll(m));
    }
}

//! subgroup starts of every window at the scanned offsets (and their systems, if @p groupSys); the final entry is
//! the end of the last window
__global__ void groupStartsKernel(GroupWindows W, uint32_t G, uint32_t numWindows,
                                  const unsigned long long* __restrict__ masks, const uint32_t* __restrict__ offsets,
                                  uint32_t* __restrict__ groups, uint32_t* __restrict__ groupSys)
{
    uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w > numWindows) return;
    if (w == numWindows)
    {
        groups[offsets[numWindows]] = W.start ? W.end[numWindows - 1] : W.last;
        return;
    }
    uint32_t base = W.start ? W.start[w] : W.first + w * G;
    uint32_t sys  = W.start ? W.sys[w] : 0u;
    uint32_t o    = offsets[w];
    if (groupSys) groupSys[o] = sys;
    groups[o++]          = base;
    unsigned long long m = masks[w];
    while (m)
    {
        int b = __ffsll(m) - 1;
        if (groupSys) groupSys[o] = sys;
        groups[o++] = base + uint32_t(b) + 1;
        m &= m - 1;
    }
}

float defaultExtentRatio()
{
    // the reference's default and its environment override (groups_gpu.cu:88-95)
    const char* v = std::getenv("CSTONE_GROUP_EXTENT_SPLIT");
    return v ? std::strtof(v, nullptr) : 8.0f;
}

namespace
{
uint32_t splitWindows(ryo_ctx* ctx, const GroupWindows& W, uint32_t numWindows, const float* x, const float* y,
                      const float* z, const float* h, const uint64_t* leaves, int numLeaves, const uint32_t* layout,
                      unsigned groupSize, float tolFactor, float extentRatio, uint32_t* groups, uint32_t* groupSys,
                      uint32_t capacity, cudaStream_t s)
{
    if (groupSize != 32 && groupSize != 64)
        throw CudaError{cudaErrorInvalidValue, "spatial groups: group size must be 32 or 64"};
    auto* masks     = ctx->scratch<unsigned long long>("grp.masks", numWindows, s);
    uint32_t* cnt   = ctx->scratch<uint32_t>("grp.counts", size_t(numWindows) + 1, s);
    uint32_t* offs  = ctx->scratch<uint32_t>("grp.offsets", size_t(numWindows) + 1, s);
    unsigned blocks = ceilDiv(size_t(numWindows) * kWarp, 256);
    if (groupSize == 64)
        groupSplitsKernel<2><<<blocks, 256, 0, s>>>(W, x, y, z, h, leaves, numLeaves, layout, tolFactor, extentRatio,
                                                    numWindows, masks, cnt);
    else
        groupSplitsKernel<1><<<blocks, 256, 0, s>>>(W, x, y, z, h, leaves, numLeaves, layout, tolFactor, extentRatio,
                                                    numWindows, masks, cnt);
    RYO_LAUNCH_CHECK();
    exclusiveScanU32(ctx, cnt, offs, numWindows, s);
    uint32_t numGroups = 0;
    RYO_CUDA(cudaMemcpyAsync(&numGroups, offs + numWindows, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    RYO_CUDA(cudaStreamSynchronize(s));
    if (groups && numGroups + 1 <= capacity)
    {
        groupStartsKernel<<<ceilDiv(size_t(numWindows) + 1, 256), 256, 0, s>>>(W, groupSize, numWindows, masks, offs,
                                                                                groups, groupSys);
        RYO_LAUNCH_CHECK();
    }
    return numGroups;
}
} // namespace

uint32_t computeGroupSplits(ryo_ctx* ctx, uint32_t first, uint32_t last, const float* x, const float* y,
                            const float* z, const float* h, const uint64_t* leaves, int numLeaves,
                            const uint32_t* layout, const DevBox<float>& box, unsigned groupSize, float tolFactor,
                            float extentRatio, uint32_t* groups, uint32_t capacity, cudaStream_t s)
{
    if (groupSize != 32 && groupSize != 64)
        throw CudaError{cudaErrorInvalidValue, "spatial groups: group size must be 32 or 64"};
    if (last <= first) return 0;
    uint32_t numWindows = (last - first + groupSize - 1) / groupSize;
    // the unit box of the same aspect ratio (edge 2^-r for an axis reduced by r bits)
    float unit6[6] = {0.f, 1.f / float(1u << (kMaxLevel - box.bits[0])), 0.f,
                      1.f / float(1u << (kMaxLevel - box.bits[1])), 0.f,
                      1.f / float(1u << (kMaxLevel - box.bits[2]))};
    GroupWindows W{};
    W.first           = first;
    W.last            = last;
    W.unitBox         = makeDevBox<float>(unit6, 0);
    float maxExtent   = std::max(std::max(box.len[0], box.len[1]), box.len[2]);
    W.invMaxExtent    = 1.f / maxExtent;
    return splitWindows(ctx, W, numWindows, x, y, z, h, leaves, numLeaves, layout, groupSize, tolFactor, extentRatio,
                        groups, nullptr, capacity, s);
}

uint32_t computeGroupSplitsBatch(ryo_ctx* ctx, const uint32_t* windowStart, const uint32_t* windowEnd,
                                 const uint32_t* windowSys, uint32_t numWindows, const DevBox<float>* sysBoxes,
                                 int sysLevel, const float* x, const float* y, const float* z,
                                 const uint64_t* leaves, int numLeaves, const uint32_t* layout, unsigned groupSize,
                                 float tolFactor, float extentRatio, uint32_t* groups, uint32_t* groupSys,
                                 uint32_t capacity, cudaStream_t s)
{
    if (numWindows == 0) return 0;
    GroupWindows W{};
    W.start    = windowStart;
    W.end      = windowEnd;
    W.sys      = windowSys;
    W.boxes    = sysBoxes;
    W.sysLevel = unsigned(sysLevel);
    return splitWindows(ctx, W, numWindows, x, y, z, nullptr, leaves, numLeaves, layout, groupSize, tolFactor,
                        extentRatio, groups, groupSys, capacity, s);
}

} // namespace ryo
