/*
 * ryoanji-b200: the locally essential tree (LET) of the last solve for another rank's domain.
 *
 * Reference: the exchange of cstone's focused octrees between ranks (cstone/include/cstone/focus/
 * octree_focus_mpi.hpp:629, globalExchange, and the peer exchange it feeds), which gives every rank the multipoles
 * and the bodies of the other ranks' trees that its own targets need. Here a rank that has solved its own bodies
 * exports, for the bounding box of another rank's bodies, the part of its tree that any target group inside that box
 * can reach:
 *   - a node is kept iff every strict ancestor below the root fails the MAC against the box (the root is always
 *     opened, so its eight children are kept);
 *   - a kept internal node that fails the MAC keeps its children (all eight, contiguous); one that passes is sent as
 *     a multipole with no children;
 *   - a kept leaf that fails the MAC sends its bodies; one that passes is sent as a multipole with no bodies.
 * A target group inside the box has a distance to every cell at least the box's, so it opens no cell that the box
 * does not open; where float rounding of the two tests disagrees, a childless cell with a non-zero MAC radius is
 * still evaluated as a multipole by the traversal's rule for cells without bodies (traversal_gpu.cu:233-236).
 *
 * The export is one packed buffer of 32-bit words that the receiver traverses with ryo_traverse_f32 as the source
 * tree of its own targets: N kept nodes, L leaves with bodies, B bodies:
 *   [0, 4N) centres (x, y, z, MAC r^2) | [4N, 12N) multipoles (8 floats) | [12N, 13N) childOffsets |
 *   [13N, 14N) internalToLeaf | [14N, 14N + L + 2) layout (leaf L has no bodies; every childless cell without
 *   bodies points to it) | then x, y, z, m, h of the B bodies, B words each.
 */
#include "internal.hpp"

namespace ryo
{

//! flags per node of the last solve's tree: kept, kept leaf with bodies, and its body count
__global__ void letMarkKernel(const NodeRecord* __restrict__ nodes, const int* __restrict__ parents, int numNodes,
                              LetBox box, uint32_t* keep, uint32_t* leafFlag, uint32_t* bodyCount)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= numNodes) return;
    bool kept = true;
    for (int a = i; a > 0;)
    {
        int par = parents[(a - 1) / 8];
        if (par == 0) break; // the root is always opened
        if (!macFails(__ldg(&nodes[par].center), box.tc, box.ts))
        {
            kept = false;
            break;
        }
        a = par;
    }
    int4 link    = __ldg(&nodes[i].link);
    bool close   = macFails(__ldg(&nodes[i].center), box.tc, box.ts);
    bool direct  = kept && link.x == 0 && close && link.z > 0;
    keep[i]      = kept ? 1u : 0u;
    leafFlag[i]  = direct ? 1u : 0u;
    bodyCount[i] = direct ? uint32_t(link.z) : 0u;
}

//! writes the kept nodes, their links and the layout of the leaves with bodies into the packed buffer
__global__ void letNodesKernel(const NodeRecord* __restrict__ nodes, int numNodes, LetBox box,
                               const uint32_t* __restrict__ keepIdx, const uint32_t* __restrict__ leafIdx,
                               const uint32_t* __restrict__ bodyOff, LetLayout out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= numNodes) return;
    if (keepIdx[i + 1] == keepIdx[i]) return;
    uint32_t j     = keepIdx[i];
    NodeRecord r   = nodes[i];
    bool close     = macFails(r.center, box.tc, box.ts);
    bool isNode    = r.link.x != 0;
    bool opened    = isNode && (close || i == 0);
    bool direct    = leafIdx[i + 1] != leafIdx[i];
    reinterpret_cast<float4*>(out.centers)[j]            = r.center;
    reinterpret_cast<float4*>(out.multipoles)[2 * j]     = r.q0;
    reinterpret_cast<float4*>(out.multipoles)[2 * j + 1] = r.q1;
    out.childOffsets[j]   = opened ? int(keepIdx[r.link.x]) : 0;
    out.internalToLeaf[j] = opened ? -1 : int(direct ? leafIdx[i] : out.numLeaves);
    if (direct) out.layout[leafIdx[i]] = bodyOff[i];
    if (i == 0)
    {
        out.layout[out.numLeaves]     = out.numBodies;
        out.layout[out.numLeaves + 1] = out.numBodies;
    }
}

//! copies the bodies of the kept leaves with bodies, one warp per node
__global__ void letBodiesKernel(const NodeRecord* __restrict__ nodes, int numNodes, const float4* __restrict__ xyzm,
                                const float* __restrict__ h, const uint32_t* __restrict__ leafIdx,
                                const uint32_t* __restrict__ bodyOff, LetLayout out)
{
    int i    = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
    int lane = laneId();
    if (i >= numNodes || leafIdx[i + 1] == leafIdx[i]) return;
    int4 link  = __ldg(&nodes[i].link);
    uint32_t o = bodyOff[i];
    for (int k = lane; k < link.z; k += kWarp)
    {
        float4 b          = __ldg(xyzm + link.y + k);
        out.x[o + k]      = b.x;
        out.y[o + k]      = b.y;
        out.z[o + k]      = b.z;
        out.m[o + k]      = b.w;
        out.h[o + k]      = __ldg(h + link.y + k);
    }
}

LetCounts letSelect(ryo_ctx* ctx, const NodeRecord* nodes, const int* parents, int numNodes, const LetBox& box,
                    cudaStream_t s)
{
    size_t n           = size_t(numNodes);
    uint32_t* keep     = ctx->scratch<uint32_t>("let.keep", n, s);
    uint32_t* leafFlag = ctx->scratch<uint32_t>("let.leaf", n, s);
    uint32_t* bodies   = ctx->scratch<uint32_t>("let.bodies", n, s);
    uint32_t* keepIdx  = ctx->scratch<uint32_t>("let.keepIdx", n + 1, s);
    uint32_t* leafIdx  = ctx->scratch<uint32_t>("let.leafIdx", n + 1, s);
    uint32_t* bodyOff  = ctx->scratch<uint32_t>("let.bodyOff", n + 1, s);
    letMarkKernel<<<ceilDiv(n, 256), 256, 0, s>>>(nodes, parents, numNodes, box, keep, leafFlag, bodies);
    RYO_LAUNCH_CHECK();
    exclusiveScanU32(ctx, keep, keepIdx, n, s);
    exclusiveScanU32(ctx, leafFlag, leafIdx, n, s);
    exclusiveScanU32(ctx, bodies, bodyOff, n, s);
    uint32_t tot[3];
    RYO_CUDA(cudaMemcpyAsync(&tot[0], keepIdx + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    RYO_CUDA(cudaMemcpyAsync(&tot[1], leafIdx + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    RYO_CUDA(cudaMemcpyAsync(&tot[2], bodyOff + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    RYO_CUDA(cudaStreamSynchronize(s));
    LetCounts c;
    c.numNodes  = tot[0];
    c.numLeaves = tot[1];
    c.numBodies = tot[2];
    c.keepIdx   = keepIdx;
    c.leafIdx   = leafIdx;
    c.bodyOff   = bodyOff;
    return c;
}

void letWrite(const LetCounts& c, const NodeRecord* nodes, int numNodes, const float4* xyzm, const float* h,
              const LetBox& box, uint32_t* buffer, cudaStream_t s)
{
    size_t N = c.numNodes, L = c.numLeaves, B = c.numBodies;
    LetLayout out;
    out.numLeaves      = uint32_t(L);
    out.numBodies      = uint32_t(B);
    out.centers        = reinterpret_cast<float*>(buffer);
    out.multipoles     = reinterpret_cast<float*>(buffer + 4 * N);
    out.childOffsets   = reinterpret_cast<int*>(buffer + 12 * N);
    out.internalToLeaf = reinterpret_cast<int*>(buffer + 13 * N);
    out.layout         = buffer + 14 * N;
    float* bodies      = reinterpret_cast<float*>(buffer + 14 * N + L + 2);
    out.x              = bodies;
    out.y              = bodies + B;
    out.z              = bodies + 2 * B;
    out.m              = bodies + 3 * B;
    out.h              = bodies + 4 * B;
    letNodesKernel<<<ceilDiv(size_t(numNodes), 256), 256, 0, s>>>(nodes, numNodes, box, c.keepIdx, c.leafIdx,
                                                                   c.bodyOff, out);
    RYO_LAUNCH_CHECK();
    if (B > 0)
    {
        letBodiesKernel<<<ceilDiv(size_t(numNodes) * kWarp, 256), 256, 0, s>>>(nodes, numNodes, xyzm, h, c.leafIdx,
                                                                               c.bodyOff, out);
        RYO_LAUNCH_CHECK();
    }
}

} // namespace ryo
