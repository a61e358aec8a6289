/*
 * ryoanji-b200: cornerstone leaf array, internal octree links and fixed target groups.
 *
 * Leaves. The reference converges a leaf array by repeated split/merge rounds with three host synchronisations
 * each (cstone/include/cstone/tree/csarray.hpp:266-440, csarray_gpu.cu:86-231). Its fixed point is unique: a node
 * is internal exactly when it holds more than bucketSize particles (and lies above level 21), and every child of
 * an internal node that is not itself internal is a leaf. Both facts follow from the rebalance rules (a node with
 * too many particles always splits; eight sibling leaves whose total fits always merge), so the fixed point can be
 * built directly from the sorted keys in one pass:
 *   - a node holds more than B particles iff it contains some window k[j], k[j+B] of B+1 consecutive sorted keys,
 *     so the deepest internal node containing particle i is the deepest common node of the windows covering i;
 *   - particle i lies in the child of that node containing it: the non-empty leaves;
 *   - the empty leaves are the minimal aligned node sequence filling the key gaps between non-empty leaves.
 * The result is bit-identical to the reference's converged leaves and counts.
 *
 * Links. The internal nodes and the level-sorted node order follow cstone/include/cstone/tree/octree.hpp:40-196
 * (the node numbering is part of the reference's output: internalToLeaf/leafToInternal are compared bit for bit).
 */
#include "internal.hpp"

namespace ryo
{

constexpr int kLeafBlock = 256;

/*! level of the leaf that contains each sorted particle, and where each particle starts a new non-empty leaf
 *
 * w[j] = min(commonLevel(k[j], k[j+B]), 20) is the level of the deepest internal node holding the window j; the
 * particle's leaf is one level below the deepest window level among the windows that contain it. The windows of
 * particle i are j in [i - B, i]; those outside [0, n - B) hold level 0 here, which leaves every maximum unchanged.
 * The maximum over B + 1 consecutive windows comes from a sparse table built by doubling in shared memory:
 * m_2P[t] = max(m_P[t], m_P[t + P]), and the window [a, a + K) is max(m_P[a], m_P[a + K - P]) for the largest power
 * of two P <= K. A block also computes the level of the particle before its first, so head[i] (1 where particle i
 * starts a non-empty leaf: its leaf's start differs from particle i - 1's) needs no second pass. blockHeads[b]
 * receives the number of heads in block b, whose scan places each block's leaves.
 */
__global__ void __launch_bounds__(kLeafBlock) leafLevels(const uint64_t* __restrict__ keys, uint32_t n,
                                                         uint32_t bucket, uint32_t minLevel,
                                                         uint8_t* __restrict__ level, uint8_t* __restrict__ head,
                                                         uint32_t* __restrict__ blockHeads)
{
    extern __shared__ unsigned char smem[];
    __shared__ uint8_t leafLvl[kLeafBlock + 1]; // particles i0 - 1 .. i0 + kLeafBlock - 1
    const uint32_t i0    = blockIdx.x * kLeafBlock;
    const uint32_t span  = kLeafBlock + bucket + 1;             // windows j in [i0 - B - 1, i0 + kLeafBlock)
    const int64_t jFirst = int64_t(i0) - int64_t(bucket) - 1;
    const int64_t numWin = int64_t(n) - int64_t(bucket);        // windows j in [0, n - B)
    uint8_t* src         = smem;
    uint8_t* dst         = smem + span;
    for (uint32_t t = threadIdx.x; t < span; t += kLeafBlock)
    {
        int64_t j = jFirst + t;
        uint8_t v = 0;
        if (j >= 0 && j < numWin)
        {
            int cb  = commonBits(keys[j], keys[j + bucket]);
            int lvl = cb / 3;
            v       = uint8_t(lvl < kMaxLevel - 1 ? lvl : kMaxLevel - 1);
        }
        src[t] = v;
    }
    __syncthreads();
    const uint32_t K = bucket + 1;
    uint32_t P       = 1;
    for (; 2 * P <= K; P *= 2)
    {
        for (uint32_t t = threadIdx.x; t + 2 * P <= span; t += kLeafBlock)
        {
            uint8_t a = src[t], b = src[t + P];
            dst[t]    = a > b ? a : b;
        }
        __syncthreads();
        uint8_t* tmp = src;
        src          = dst;
        dst          = tmp;
    }
    // particle i0 + tid covers the windows at [tid + 1, tid + 1 + K); the particle before the block, [0, K)
    auto leafLevel = [&](uint32_t a) -> uint32_t
    {
        uint8_t x = src[a], y = src[a + K - P];
        uint32_t lv = uint32_t(x > y ? x : y) + 1;
        return lv > minLevel ? lv : minLevel;
    };
    const uint32_t i = i0 + threadIdx.x;
    uint32_t lv      = leafLevel(threadIdx.x + 1);
    leafLvl[threadIdx.x + 1] = uint8_t(lv);
    if (threadIdx.x == 0) leafLvl[0] = uint8_t(leafLevel(0));
    __syncthreads();
    int h = 0;
    if (i < n)
    {
        h = 1;
        if (i > 0)
        {
            uint64_t st = keys[i] & ~(nodeRange(lv) - 1);
            uint64_t sp = keys[i - 1] & ~(nodeRange(leafLvl[threadIdx.x]) - 1);
            h           = sp != st;
        }
    }
    const int count = __syncthreads_count(h);
    if (threadIdx.x == 0) blockHeads[blockIdx.x] = uint32_t(count);
    if (i >= n) return;
    level[i] = uint8_t(lv);
    head[i]  = uint8_t(h);
}

/*! the start, level and first particle of every non-empty leaf, in particle order: block b of leafLevels' blocks
 *  writes its heads from blockOffset[b] on, ranked within the block by warp ballots */
__global__ void __launch_bounds__(kLeafBlock) leafCompact(const uint64_t* __restrict__ keys,
                                                          const uint8_t* __restrict__ level,
                                                          const uint8_t* __restrict__ head,
                                                          const uint32_t* __restrict__ blockOffset, uint32_t n,
                                                          uint64_t* __restrict__ leafStart,
                                                          uint8_t* __restrict__ leafLvl,
                                                          uint32_t* __restrict__ leafFirst)
{
    __shared__ uint32_t warpBase[kLeafBlock / kWarp];
    const uint32_t i      = blockIdx.x * kLeafBlock + threadIdx.x;
    const bool h          = i < n && head[i] != 0;
    const unsigned ballot = __ballot_sync(0xffffffffu, h);
    const unsigned warp   = threadIdx.x / kWarp;
    if (laneId() == 0) warpBase[warp] = __popc(ballot);
    __syncthreads();
    if (threadIdx.x == 0)
    {
        uint32_t run = 0;
        for (int w = 0; w < kLeafBlock / kWarp; ++w)
        {
            uint32_t c  = warpBase[w];
            warpBase[w] = run;
            run += c;
        }
    }
    __syncthreads();
    if (!h) return;
    const uint32_t q = blockOffset[blockIdx.x] + warpBase[warp] + __popc(ballot & lanemaskLt());
    leafStart[q]     = keys[i] & ~(nodeRange(level[i]) - 1);
    leafLvl[q]       = level[i];
    leafFirst[q]     = i;
}

//! number of output leaves contributed by non-empty leaf q: the gap before it plus itself (q == numNE: final gap)
__global__ void leafSlots(const uint64_t* __restrict__ leafStart, const uint8_t* __restrict__ leafLvl, uint32_t numNE,
                          uint32_t* __restrict__ slots)
{
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q > numNE) return;
    uint64_t prevEnd = q == 0 ? 0 : leafStart[q - 1] + nodeRange(leafLvl[q - 1]);
    uint64_t start   = q == numNE ? kKeyEnd : leafStart[q];
    slots[q]         = uint32_t(spanKeyRange(prevEnd, start, nullptr)) + (q < numNE ? 1u : 0u);
}

__global__ void leafWrite(const uint64_t* __restrict__ leafStart, const uint8_t* __restrict__ leafLvl,
                          const uint32_t* __restrict__ leafFirst, const uint32_t* __restrict__ offsets, uint32_t numNE,
                          uint32_t n, uint64_t* __restrict__ leaves, uint32_t* __restrict__ counts,
                          uint32_t* __restrict__ layout)
{
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q > numNE) return;
    uint64_t prevEnd = q == 0 ? 0 : leafStart[q - 1] + nodeRange(leafLvl[q - 1]);
    uint64_t start   = q == numNE ? kKeyEnd : leafStart[q];
    uint32_t o       = offsets[q];
    uint32_t first   = q == numNE ? n : leafFirst[q];
    int gap          = spanKeyRange(prevEnd, start, leaves + o);
    for (int g = 0; g < gap; ++g)
    {
        counts[o + g] = 0;
        if (layout) layout[o + g] = first;
    }
    if (q < numNE)
    {
        uint32_t last   = q + 1 < numNE ? leafFirst[q + 1] : n;
        leaves[o + gap] = start;
        counts[o + gap] = last - first;
        if (layout) layout[o + gap] = first;
    }
    else
    {
        leaves[o + gap] = kKeyEnd;
        if (layout) layout[o + gap] = n;
    }
}

__global__ void singleLeaf(uint64_t* leaves, uint32_t* counts, uint32_t* layout, uint32_t n)
{
    leaves[0] = 0;
    leaves[1] = kKeyEnd;
    counts[0] = n;
    if (layout)
    {
        layout[0] = 0;
        layout[1] = n;
    }
}

int buildLeaves(ryo_ctx* ctx, const uint64_t* keys, size_t n64, unsigned bucket, uint64_t* leaves, uint32_t* counts,
                uint32_t* layout, int capacity, cudaStream_t s, unsigned minLevel)
{
    uint32_t n = uint32_t(n64);
    if (minLevel > 0 && (n == 0 || minLevel > unsigned(kMaxLevel)))
        throw CudaError{cudaErrorInvalidValue, "leaf construction: no keys, or minimum level above 21"};
    if (n <= bucket && minLevel == 0)
    {
        if (capacity >= 1)
        {
            singleLeaf<<<1, 1, 0, s>>>(leaves, counts, layout, n);
            RYO_LAUNCH_CHECK();
        }
        return 1;
    }
    if (bucket > 16384) throw CudaError{cudaErrorInvalidValue, "bucket size above 16384 is not supported"};

    const uint32_t numBlocks = uint32_t(ceilDiv(n, kLeafBlock));
    uint8_t* level       = ctx->scratch<uint8_t>("leaf.level", n, s);
    uint8_t* head        = ctx->scratch<uint8_t>("leaf.head8", n, s);
    uint32_t* blockHeads = ctx->scratch<uint32_t>("leaf.blockHeads", size_t(numBlocks) + 1, s);
    size_t smemBytes = 2 * (size_t(kLeafBlock) + bucket + 1); // two window-level buffers of the sparse table
    if (smemBytes > 48 * 1024)
        RYO_CUDA(cudaFuncSetAttribute(leafLevels, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smemBytes)));
    leafLevels<<<numBlocks, kLeafBlock, smemBytes, s>>>(keys, n, bucket, minLevel, level, head, blockHeads);
    RYO_LAUNCH_CHECK();
    exclusiveScanU32(ctx, blockHeads, blockHeads, numBlocks, s);
    uint32_t numNE = 0;
    RYO_CUDA(cudaMemcpyAsync(&numNE, blockHeads + numBlocks, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    RYO_CUDA(cudaStreamSynchronize(s));

    uint64_t* leafStart = ctx->scratch<uint64_t>("leaf.start", numNE, s);
    uint8_t* leafLvl    = ctx->scratch<uint8_t>("leaf.lvl", numNE, s);
    uint32_t* leafFirst = ctx->scratch<uint32_t>("leaf.first", numNE, s);
    uint32_t* slots     = ctx->scratch<uint32_t>("leaf.slots", size_t(numNE) + 2, s);
    leafCompact<<<numBlocks, kLeafBlock, 0, s>>>(keys, level, head, blockHeads, n, leafStart, leafLvl, leafFirst);
    RYO_LAUNCH_CHECK();
    leafSlots<<<ceilDiv(numNE + 1, 256), 256, 0, s>>>(leafStart, leafLvl, numNE, slots);
    RYO_LAUNCH_CHECK();
    exclusiveScanU32(ctx, slots, slots, size_t(numNE) + 1, s);
    uint32_t numLeaves = 0;
    RYO_CUDA(cudaMemcpyAsync(&numLeaves, slots + numNE + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    RYO_CUDA(cudaStreamSynchronize(s));
    if (int64_t(numLeaves) <= int64_t(capacity))
    {
        leafWrite<<<ceilDiv(numNE + 1, 256), 256, 0, s>>>(leafStart, leafLvl, leafFirst, slots, numNE, n, leaves,
                                                           counts, layout);
        RYO_LAUNCH_CHECK();
    }
    return int(numLeaves);
}

// ------------------------------------------------------------------------------------------------ links

constexpr uint64_t kEmptySlot = 31; // sort key of a slot without a node: after every level (0 .. 21)
constexpr int kLevelBits      = 5;  // bits of a slot's sort key

//! weight of the digits on levels 1..level+1 in the binary-radix-tree to octree index map (octree.hpp:55-65)
__device__ inline int treeIndexWeight(uint64_t key, unsigned level)
{
    int w = 0;
    for (unsigned l = 1; l <= level + 1; ++l)
    {
        int d = int(octalDigit(key, l));
        w += d >= 4 ? 7 - d : -d;
    }
    return w;
}

/*! unsorted node layout: internal nodes first, numbered as in the reference's binary-radix-tree map (node of the
 *  leaf pair whose common prefix ends on a level boundary), then the leaves (octree_gpu.cu:41-64). Beside it, the
 *  sort slots of the level-major order: slot 2t holds the internal node of leaf pair t, if there is one, and slot
 *  2t + 1 leaf t; a slot's key is its node's level (31 for an empty slot) and its value the node's unsorted index.
 *  Nodes of one level appear in the slots in key order: two nodes of a level cover disjoint key ranges, and the leaf
 *  indices that stand for them (t for the node of pair t, which holds leaves t and t + 1; j for leaf j) are ordered
 *  as the ranges are. A stable sort of the slots by level is therefore the sort of the placeholder-bit prefixes. */
__global__ void unsortedLayout(const uint64_t* __restrict__ leaves, int numInternal, int numLeaves,
                               uint64_t* __restrict__ prefixes, uint64_t* __restrict__ slotLevel,
                               uint32_t* __restrict__ slotNode)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= numLeaves) return;
    uint64_t key              = leaves[t];
    uint64_t next             = leaves[t + 1];
    unsigned leafLevel        = rangeLevel(next - key);
    prefixes[t + numInternal] = encodePrefix(key, 3 * int(leafLevel));
    slotLevel[2 * t + 1]      = leafLevel;
    slotNode[2 * t + 1]       = uint32_t(numInternal + t);
    int common                = commonBits(key, next);
    if (t < numLeaves - 1 && common % 3 == 0)
    {
        int at           = (t + treeIndexWeight(key, common / 3)) / 7;
        prefixes[at]     = encodePrefix(key, common);
        slotLevel[2 * t] = uint64_t(common / 3);
        slotNode[2 * t]  = uint32_t(at);
    }
    else
    {
        slotLevel[2 * t] = kEmptySlot;
        slotNode[2 * t]  = 0;
    }
}

//! prefixes in the level-major order: sorted[i] = unsorted[order[i]]
__global__ void gatherPrefixes(const uint64_t* __restrict__ unsorted, const uint32_t* __restrict__ order, int numNodes,
                               uint64_t* __restrict__ sorted)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < numNodes) sorted[i] = unsorted[order[i]];
}

__global__ void invertOrder(const uint32_t* __restrict__ order, int numNodes, int numInternal,
                            int* __restrict__ internalToLeaf, int* __restrict__ leafToInternal)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= numNodes) return;
    int o             = int(order[i]);
    leafToInternal[o] = i;
    internalToLeaf[i] = o - numInternal;
}

__global__ void levelBounds(const uint64_t* __restrict__ prefixes, int numNodes, int* __restrict__ levelRange)
{
    int l = threadIdx.x;
    if (l > kMaxLevel + 1) return;
    if (l == kMaxLevel + 1)
    {
        levelRange[l] = numNodes;
        return;
    }
    uint64_t target = encodePrefix(0, 3 * l);
    int lo = 0, hi = numNodes;
    while (lo < hi)
    {
        int mid = (lo + hi) / 2;
        if (prefixes[mid] < target) lo = mid + 1;
        else hi = mid;
    }
    levelRange[l] = lo;
}

__global__ void linkNodes(const uint64_t* __restrict__ prefixes, int numInternal, const int* __restrict__ leafToInternal,
                          const int* __restrict__ levelRange, int* __restrict__ childOffsets, int* __restrict__ parents)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= numInternal) return;
    int a         = leafToInternal[t];
    uint64_t pre  = prefixes[a];
    int len       = prefixLength(pre);
    int lvl       = len / 3;
    uint64_t cpre = encodePrefix(prefixStart(pre), len + 3);
    int lo = levelRange[lvl + 1], hi = levelRange[lvl + 2];
    int end = hi;
    while (lo < hi)
    {
        int mid = (lo + hi) / 2;
        if (prefixes[mid] < cpre) lo = mid + 1;
        else hi = mid;
    }
    if (lo != end && prefixes[lo] == cpre)
    {
        childOffsets[a]       = lo;
        parents[(lo - 1) / 8] = a;
    }
}

void linkOctree(ryo_ctx* ctx, const uint64_t* leaves, int numLeaves, const OctreeArrays& out, int* hostLevelRange,
                cudaStream_t s)
{
    int numInternal = (numLeaves - 1) / 7;
    int numNodes    = numLeaves + numInternal;
    size_t slots    = 2 * size_t(numLeaves);
    uint64_t* pre   = ctx->scratch<uint64_t>("link.prefix", numNodes, s);
    uint64_t* lvl   = ctx->scratch<uint64_t>("link.slotLevel", slots, s);
    uint64_t* lvlB  = ctx->scratch<uint64_t>("link.slotLevelB", slots, s);
    uint32_t* ord   = ctx->scratch<uint32_t>("link.order", slots, s);
    uint32_t* ordB  = ctx->scratch<uint32_t>("link.orderB", slots, s);
    size_t tmpBytes = sortTempBytes(slots);
    void* tmp       = ctx->scratch<char>("link.sorttmp", tmpBytes, s);

    unsortedLayout<<<ceilDiv(numLeaves, 256), 256, 0, s>>>(leaves, numInternal, numLeaves, pre, lvl, ord);
    RYO_LAUNCH_CHECK();
    // one stable pass over the 5-bit levels; the empty slots sort behind the numNodes nodes
    bool alt              = radixSortPairs(lvl, ord, lvlB, ordB, slots, 0, kLevelBits, tmp, tmpBytes,
                                           &ctx->ctl->error, s, false);
    const uint32_t* order = alt ? ordB : ord;
    gatherPrefixes<<<ceilDiv(numNodes, 256), 256, 0, s>>>(pre, order, numNodes, out.prefixes);
    RYO_LAUNCH_CHECK();
    invertOrder<<<ceilDiv(numNodes, 256), 256, 0, s>>>(order, numNodes, numInternal, out.internalToLeaf,
                                                        out.leafToInternal);
    RYO_LAUNCH_CHECK();
    int* dlr = out.d_levelRange ? out.d_levelRange : ctx->scratch<int>("link.levelRange", kMaxLevel + 2, s);
    levelBounds<<<1, 32, 0, s>>>(out.prefixes, numNodes, dlr);
    RYO_LAUNCH_CHECK();
    RYO_CUDA(cudaMemsetAsync(out.childOffsets, 0, sizeof(int) * numNodes, s));
    int numParents = (numNodes - 1) / 8 > 1 ? (numNodes - 1) / 8 : 1;
    RYO_CUDA(cudaMemsetAsync(out.parents, 0, sizeof(int) * numParents, s));
    if (numInternal > 0)
    {
        linkNodes<<<ceilDiv(numInternal, 256), 256, 0, s>>>(out.prefixes, numInternal, out.leafToInternal, dlr,
                                                             out.childOffsets, out.parents);
        RYO_LAUNCH_CHECK();
    }
    RYO_CUDA(cudaMemcpyAsync(hostLevelRange, dlr, sizeof(int) * (kMaxLevel + 2), cudaMemcpyDeviceToHost, s));
    RYO_CUDA(cudaStreamSynchronize(s));
}

// ------------------------------------------------------------------------------------------------ groups

__global__ void fixedGroups(uint32_t first, uint32_t last, unsigned groupSize, uint32_t numGroups, uint32_t* groups)
{
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < numGroups) groups[g] = first + g * groupSize;
    if (g == numGroups) groups[g] = last;
}

void launchFixedGroups(uint32_t first, uint32_t last, unsigned groupSize, uint32_t* groups, cudaStream_t s)
{
    uint32_t numGroups = (last - first + groupSize - 1) / groupSize;
    fixedGroups<<<ceilDiv(numGroups + 1, 256), 256, 0, s>>>(first, last, groupSize, numGroups, groups);
    RYO_LAUNCH_CHECK();
}

} // namespace ryo
