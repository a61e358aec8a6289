/*
 * ryoanji-b200: host-side internals shared by the translation units (context, scratch memory, launchers).
 */
#pragma once

#include <algorithm>
#include <cmath>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.cuh"

namespace ryo
{

//! per-context device control block: work counters, statistics and error flags of the last calls
struct Control
{
    unsigned int workCounter;  // traversal work queue head
    unsigned int failedCount;  // groups that overflowed the traversal stack in the current pass
    unsigned int error;        // non-zero: a bounded device wait gave up
    unsigned int tileCounter;  // onesweep tile ticket of the current pass
    unsigned long long stats[5]; // sumP2P, maxP2P, sumM2P, maxM2P, maxStack
    double potential;          // sum m * phi of the traversal (no G)
    double ewaldPotential;     // sum m * phi of the Ewald correction (no G)
    unsigned int counters[8];  // scratch counters for other kernels
    unsigned int heavyCount;   // groups queued for the split second traversal pass
};

enum BhStat
{
    kSumP2P = 0,
    kMaxP2P,
    kSumM2P,
    kMaxM2P,
    kMaxStack
};

//! why the reference would refuse these Ewald settings, or nullptr: ceil(hCut) <= 3 (ryoanji/src/ryoanji/nbody/
//! ewald.hpp:52-60, which also bounds the wave-vector tables here), no negative value, and a positive alpha_scale
//! unless lCut, hCut and alpha_scale are all 0 (Ewald off)
inline const char* ewaldSettingsError(const ryo_ewald_settings& e)
{
    if (!(e.numReplicaShells >= 0 && e.lCut >= 0 && e.hCut >= 0 && e.alpha_scale >= 0 && e.small_R_scale_factor >= 0))
        return "ewald: settings must not be negative";
    if (!(std::ceil(e.hCut) <= 3)) return "ewald: hCut must be at most 3, as in the reference";
    bool off = e.lCut == 0 && e.hCut == 0 && e.alpha_scale == 0;
    if (!(off || e.alpha_scale > 0)) return "ewald: alpha_scale must be positive";
    return nullptr;
}

//! makes @p device the current device for its scope and restores the caller's afterwards, so that a context's calls
//! allocate and launch on the context's device whatever device the calling thread has current
class DeviceScope
{
public:
    explicit DeviceScope(int device)
    {
        if (cudaGetDevice(&prev_) == cudaSuccess && prev_ != device) switched_ = cudaSetDevice(device) == cudaSuccess;
    }
    ~DeviceScope()
    {
        if (switched_) cudaSetDevice(prev_);
    }
    DeviceScope(const DeviceScope&)            = delete;
    DeviceScope& operator=(const DeviceScope&) = delete;

private:
    int prev_      = 0;
    bool switched_ = false;
};

} // namespace ryo

struct ryo_ctx
{
    int device   = 0;
    int smCount  = 148;
    std::string lastError;
    ryo::Control* ctl = nullptr; // device
    unsigned long long hostStats[5] = {0, 0, 0, 0, 0};
    uint64_t retries                = 0;
    ryo_solve_arrays lastSolve      = {};
    //! what ryo_solve_targets_f32 needs of the last single-system solve (cleared by a batched solve, which reuses
    //! the same scratch buffers)
    struct SolveState
    {
        bool valid         = false;
        const void* nodes  = nullptr; // NodeRecord per node
        const void* xyzm   = nullptr; // float4 per source body
        const float* srcH  = nullptr; // the caller's h array of the solve (sorted)
        const void* dipoles = nullptr; // float4 per node for dipole expansions, else null
        const uint32_t* massRange = nullptr; // min and max source mass (ordered bits), null if not known
        int numNodes       = 0;
        unsigned groupSize = 64;
        float G            = 1.f;
        int periodic       = 0;
        int numShells      = 0;
        ryo_box_f32 box    = {};
        ryo_ewald_settings ewald = {};
        double root[11]    = {};
    } solveState;
    cudaEvent_t phaseEvents[7]      = {};
    cudaEvent_t pipeEvents[2]       = {};    // ordering between the solve and the copy stream of host solves
    cudaStream_t copyStream         = nullptr; // host solves: copies that overlap the solve

    struct Buffer
    {
        void* ptr    = nullptr;
        size_t bytes = 0;
    };
    std::unordered_map<std::string, Buffer> buffers;

    //! grow-only named scratch buffer of at least @p count elements
    template<class T>
    T* scratch(const std::string& name, size_t count, cudaStream_t s)
    {
        size_t bytes = count * sizeof(T);
        if (bytes == 0) bytes = 256;
        Buffer& b = buffers[name];
        if (b.bytes < bytes)
        {
            // growth is rare: wait for work that may still use the old buffer, then reallocate. A buffer that
            // grows again takes at least 1.5 times its old size, so a growing workload (a served stream)
            // reallocates O(log n) times.
            size_t old = b.bytes;
            if (b.ptr)
            {
                RYO_CUDA(cudaStreamSynchronize(s));
                RYO_CUDA(cudaFree(b.ptr));
                b.ptr   = nullptr;
                b.bytes = 0;
            }
            size_t grow = std::max(bytes + bytes / 8, old + old / 2);
            RYO_CUDA(cudaMalloc(&b.ptr, grow));
            b.bytes = grow;
        }
        return static_cast<T*>(b.ptr);
    }

    void releaseAll()
    {
        for (auto& e : phaseEvents)
            if (e) cudaEventDestroy(e);
        for (auto& e : pipeEvents)
            if (e) cudaEventDestroy(e);
        if (copyStream) cudaStreamDestroy(copyStream);
        copyStream = nullptr;
        for (auto& kv : buffers)
            if (kv.second.ptr) cudaFree(kv.second.ptr);
        buffers.clear();
    }
};

namespace ryo
{

// ---------------------------------------------------------------------------------------------------- sfc.cu
template<class T>
void launchKeys(const T* x, const T* y, const T* z, uint64_t* keys, size_t n, const DevBox<T>& box, bool keepRemoved,
                cudaStream_t s);
void launchBoundingBox(const float* x, const float* y, const float* z, size_t n, double* minmax6, cudaStream_t s);
void launchSequence(uint32_t* v, size_t n, uint32_t first, cudaStream_t s);
//! out[i] = in[order[i]] for float arrays
void launchGather(const uint32_t* order, const float* in, float* out, size_t n, cudaStream_t s);
template<class T>
void launchGatherT(const uint32_t* order, const T* in, T* out, size_t n, cudaStream_t s);
//! rec[2 i], rec[2 i + 1] = (x, y, z, m), (h, vx, vy, vz) of body i (null velocities give zeros)
void launchPackRecords(const float* x, const float* y, const float* z, const float* m, const float* h,
                       const float* vx, const float* vy, const float* vz, size_t n, float4* rec, cudaStream_t s);
//! body i of the output is record order[i]: the per-body arrays (null ones skipped) and xyzm / xyzh (may be null);
//! hRange (may be null, else 4 entries) receives the min and max softening, then the min and max mass, as ordered
//! bits (orderedBits)
void launchGatherRecords(const uint32_t* order, const float4* rec, size_t n, float* x, float* y, float* z, float* m,
                         float* h, float* vx, float* vy, float* vz, float4* xyzm, float4* xyzh, uint32_t* hRange,
                         cudaStream_t s);

// ---------------------------------------------------------------------------------------------------- scan / sort
//! out[i] = sum(in[0:i]) for i in [0, n]; out has n + 1 entries (out[n] = total); in-place allowed
void exclusiveScanU32(ryo_ctx* ctx, const uint32_t* in, uint32_t* out, size_t n, cudaStream_t s);

size_t staticSortMaxKeys();
//! sort of bits [0, 64) whose scratch is a fixed device array (no allocation); true if a look-back wait timed out
bool sortPairsStaticScratch(uint64_t* keys, uint32_t* values, uint64_t* keysAlt, uint32_t* valuesAlt, size_t n,
                            cudaStream_t s);
size_t sortTempBytes(size_t n);
/*! stable LSD sort of (keys, values) on bits [beginBit, endBit). Ping-pongs between (keys, values) and
 *  (keysAlt, valuesAlt), all four buffers of n elements; returns true if the result is in the Alt buffers.
 *  iotaValues: ignore the input values and sort (key, input index) pairs. */
bool radixSortPairs(uint64_t* keys, uint32_t* values, uint64_t* keysAlt, uint32_t* valuesAlt, size_t n, int beginBit,
                    int endBit, void* tmp, size_t tmpBytes, unsigned int* errorFlag, cudaStream_t s,
                    bool iotaValues = false);
//! runs one onesweep tile whose predecessor never publishes; true if its bounded look-back wait ran out and said so
bool sortWaitTimeoutSelfTest(cudaStream_t s);

// ---------------------------------------------------------------------------------------------------- octree.cu
//! cornerstone leaves of sorted keys; returns numLeaves (host), writes only if numLeaves <= capacity
//! cornerstone leaves of sorted keys; every leaf holding particles lies on level >= minLevel (0: the reference's
//! leaves; a batched solve uses the level of its system prefix so that no leaf spans two systems)
int buildLeaves(ryo_ctx* ctx, const uint64_t* sortedKeys, size_t n, unsigned bucket, uint64_t* leaves,
                uint32_t* counts, uint32_t* layout, int capacity, cudaStream_t s, unsigned minLevel = 0);

struct OctreeArrays
{
    uint64_t* prefixes;
    int* childOffsets;
    int* parents;
    int* internalToLeaf;
    int* leafToInternal;
    int* d_levelRange; // 23, device
};
//! internal octree of a leaf array; fills hostLevelRange[23]
void linkOctree(ryo_ctx* ctx, const uint64_t* leaves, int numLeaves, const OctreeArrays& out, int* hostLevelRange,
                cudaStream_t s);
void launchFixedGroups(uint32_t first, uint32_t last, unsigned groupSize, uint32_t* groups, cudaStream_t s);

// ---------------------------------------------------------------------------------------------------- upsweep.cu
// The reference-signature steps, for the reference's type sets: (Tc, Tm, Tf, Tmp) = (float, float, float, float),
// (double, double, double, double) and (double, float, double, float). Centres are 4 values of Tf per node,
// multipoles 8 (12 with mdq) values of Tmp per node.
template<class Tc, class Tm, class Tf>
void launchLeafCenters(const Tc* x, const Tc* y, const Tc* z, const Tm* m, const int* leafToInternal, int numLeaves,
                       const uint32_t* layout, Tf* centers, cudaStream_t s);
template<class Tf>
void launchUpsweepCenters(int first, int last, const int* childOffsets, Tf* centers, cudaStream_t s);
template<class Tc, class Tm, class Tf, class Tmp>
void launchLeafMultipoles(const Tc* x, const Tc* y, const Tc* z, const Tm* m, const int* leafToInternal,
                          int numLeaves, const uint32_t* layout, const Tf* centers, Tmp* multipoles, bool mdq,
                          cudaStream_t s);
template<class Tf, class Tmp>
void launchUpsweepMultipoles(int first, int last, const int* childOffsets, const Tf* centers, Tmp* multipoles, bool mdq,
                             cudaStream_t s);
template<class T>
void launchSetMac(const uint64_t* prefixes, int numNodes, T* centers, float invTheta, const DevBox<T>& box,
                  cudaStream_t s);

//! the reference's applyMAC (traversal_gpu.cu:77-84) with every operation rounded once: true if the cell of centre
//! c (MAC r^2 in c.w) is too close to the box of centre tc and half-size ts for its multipole
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

//! node record used by the traversal: 64 bytes, one cache line half per node
struct alignas(16) NodeRecord
{
    float4 center; // x, y, z, mac^2
    float4 q0;     // mass, qxx, qxy, qxz
    float4 q1;     // qyy, qyz, qzz, trace
    int4 link;     // child (global node index, 0 = leaf), first body, body count, unused
};

// ---------------------------------------------------------------------------------------------------- let.cu
//! a box as the traversal sees a target group: centre and half-size, rounded as the traversal rounds them
struct LetBox
{
    float tc[3], ts[3];
};
//! where the packed export buffer keeps each array
struct LetLayout
{
    float *centers, *multipoles;
    int *childOffsets, *internalToLeaf;
    uint32_t* layout;
    float *x, *y, *z, *m, *h;
    uint32_t numLeaves, numBodies;
};
//! sizes of one export and its per-node offsets (scratch of the context)
struct LetCounts
{
    uint32_t numNodes, numLeaves, numBodies;
    const uint32_t *keepIdx, *leafIdx, *bodyOff;
    size_t words() const { return 14 * size_t(numNodes) + numLeaves + 2 + 5 * size_t(numBodies); }
};
LetCounts letSelect(ryo_ctx* ctx, const NodeRecord* nodes, const int* parents, int numNodes, const LetBox& box,
                    cudaStream_t s);
void letWrite(const LetCounts& c, const NodeRecord* nodes, int numNodes, const float4* xyzm, const float* h,
              const LetBox& box, uint32_t* buffer, cudaStream_t s);

/*! upsweep of the solver path: per leaf FP64 centre of mass and P2M in one pass over the bodies, then M2M bottom-up
 *  (by last-arriving-child counters, or for large trees level by level from the deepest, one launch per level, with
 *  @p hostLevelRange the host copy of the level-major ranges), MAC radius, and the traversal node records. Also writes the reference-layout centers (4 floats) and multipoles (8
 *  floats) if not null. */
void launchFusedUpsweep(ryo_ctx* ctx, const float4* xyzm, int numLeaves, int numNodes, const uint32_t* layout,
                        const int* leafToInternal, const int* childOffsets, const int* parents,
                        const uint64_t* prefixes, float invTheta, const DevBox<float>& box, NodeRecord* records,
                        float4* centers, float* multipoles, double* rootCenterMultipole, cudaStream_t s,
                        const DevBox<float>* sysBoxes = nullptr, int sysLevel = 0, double* sysRoots = nullptr,
                        float4* dipoles = nullptr, uint32_t numSystems = 0, const int* hostLevelRange = nullptr);

//! pack reference-layout tree arrays into node records (for the reference-signature traverse)
void launchPackNodes(int numNodes, const float4* centers, const float* multipoles, const int* childOffsets,
                     const int* internalToLeaf, const uint32_t* layout, NodeRecord* records, cudaStream_t s);
void launchPackBodies(const float* x, const float* y, const float* z, const float* w, size_t n, float4* out,
                      cudaStream_t s);

// ---------------------------------------------------------------------------------------------------- traverse.cu
struct TraverseLaunch
{
    const uint32_t* groupStart;
    const uint32_t* groupEnd;
    int numGroups;
    int initNode;
    int numNodes; // 1 means the root is the only (leaf) node; any larger value otherwise
    // packed form (solver path): node records and (x,y,z,h) targets / (x,y,z,m) sources
    const NodeRecord* nodes;
    const float4* tgtXYZH;
    const float* tgtM;
    const float4* srcXYZM;
    const float* srcH;
    // reference form, used when nodes == nullptr
    const float4* centers;
    const float* multipoles;
    const int* childOffsets;
    const int* internalToLeaf;
    const uint32_t* layout;
    const float *xt, *yt, *zt, *mt, *ht;
    const float *xs, *ys, *zs, *ms, *hs;
    float G;
    int numShells;
    float boxL[3];
    float* p;
    float* ax;
    float* ay;
    float* az;
    uint32_t* groupM2P;
    uint32_t* groupP2P;
    uint32_t* failedGroups;
    uint32_t failedCapacity;
    int stackCapacity;
    Control* ctl;
    // monopole + dipole + quadrupole expansions: node dipoles beside the records (packed form), or 12-float
    // multipoles in the reference form
    const float4* dipoles;
    int mdqArrays;
    // batched systems (all optional): the system of every group, per-system traversal parameters and potentials
    const uint32_t* groupSys;
    const struct SysTrav* systems;
    double* sysPotential;
    // groups too costly for one warp. First pass (parts == 0, heavyGroups set): a group whose interaction count
    // (direct bodies + 2 x approximated cells) passes heavyCost stops and is queued in heavyGroups. Second pass
    // (parts > 0): item i walks group heavyGroups[i / parts] in full but evaluates only every parts-th batch,
    // starting at batch i % parts, and writes its compensated partial sums to partials[i][64] for the combine step.
    uint32_t balanceGroups; // group count the split threshold follows (0: the launch's); a solve traversed in several
                            // launches passes its total, so that its groups split as in one launch
    uint32_t* heavyGroups;
    uint32_t heavyCapacity;
    unsigned heavyCost;
    int parts;
    uint32_t numHeavy;  // second pass: queued groups
    float4* partials;   // second pass: (-phi, ax, ay, az) of the group's 64 targets, per item
    int* partStatus;    // second pass: per item, 1 if the walk overflowed the stack
    // min and max softening of every target and source as ordered bits (null: not known). Equal values let the
    // direct sums skip staging and comparing the sources' softening.
    const uint32_t* softeningRange;
    // min and max mass of every source as ordered bits (null: not known). Equal values let the direct sums apply
    // the mass once per batch instead of once per source.
    const uint32_t* massRange;
    // 1: p, ax, ay, az receive the group's results instead of adding them (0 + result, the same bits as an add to a
    // zeroed array) and are never read. The host-memory solve points them at the caller's mapped host arrays.
    int overwrite;
    // double coordinates (traverse64.cu): kPrecisionF64 (everything double) or kPrecisionMixed (double coordinates
    // and centres; float softenings, masses, multipoles and outputs). The float fields above are unused then; the
    // untyped pointers hold double (f64) or float (mixed) arrays.
    int precision;
    const double *xt64, *yt64, *zt64, *xs64, *ys64, *zs64;
    const void *mt64, *ht64, *ms64, *hs64;
    const double* centers64;   // 4 per node
    const void* multipoles64;  // 8 or 12 per node
    double G64;
    double boxL64[3];
    void *p64, *ax64, *ay64, *az64;
};

constexpr int kPrecisionF32   = 0;
constexpr int kPrecisionF64   = 1;
constexpr int kPrecisionMixed = 2;
void launchTraverse64(const TraverseLaunch& t, int smCount, cudaStream_t s);

//! per-system traversal parameters of a batched solve
struct SysTrav
{
    int entry;     // first stack entry: first child of the system's root, or -(root + 2) for a single-cell tree
    int numShells; // periodic replicas per dimension
    float boxL[3];
    uint32_t hLo, hHi; // min and max softening of the system's bodies as ordered bits (hLo > hHi: not known)
    uint32_t mLo, mHi; // min and max mass of the system's bodies as ordered bits (mLo > mHi: not known)
};
//! per-system softening and mass ranges of a batched solve into trav[s].hLo / hHi / mLo / mHi (one block per
//! system); m may be null (the mass range then stays unknown)
void launchBatchSofteningRange(const float* h, const float* m, const uint64_t* first, uint32_t numSystems,
                               SysTrav* trav, cudaStream_t s);
void launchTraverse(const TraverseLaunch& t, int smCount, cudaStream_t s);
/*! after a second pass: per queued group, the parts' partial sums added in part order into the outputs (and the
 *  potential); a group whose walk overflowed the stack goes to t.failedGroups instead. @p mass: target masses */
void launchCombineHeavy(const TraverseLaunch& t, const float* mass, cudaStream_t s);
void launchTraversalReset(Control* ctl, bool resetStats, cudaStream_t s);

// ---------------------------------------------------------------------------------------------------- groups.cu
//! the reference's default window-extent ratio (8, or CSTONE_GROUP_EXTENT_SPLIT)
float defaultExtentRatio();
/*! spatial target groups of the sorted targets [first, last): returns the group count; writes groups[count + 1]
 *  (starts, then last) when capacity >= count + 1 */
uint32_t computeGroupSplits(ryo_ctx* ctx, uint32_t first, uint32_t last, const float* x, const float* y,
                            const float* z, const float* h, const uint64_t* leaves, int numLeaves,
                            const uint32_t* layout, const DevBox<float>& box, unsigned groupSize, float tolFactor,
                            float extentRatio, uint32_t* groups, uint32_t capacity, cudaStream_t s);
/*! spatial groups of a batched solve: each fixed window [windowStart[w], windowEnd[w]) of system windowSys[w] is split
 *  with that system's box (no interaction radius); returns the group count and, when capacity >= count + 1, writes
 *  groups[count + 1] (starts, then the end of the last window) and groupSys[count] */
uint32_t computeGroupSplitsBatch(ryo_ctx* ctx, const uint32_t* windowStart, const uint32_t* windowEnd,
                                 const uint32_t* windowSys, uint32_t numWindows, const DevBox<float>* sysBoxes,
                                 int sysLevel, const float* x, const float* y, const float* z,
                                 const uint64_t* leaves, int numLeaves, const uint32_t* layout, unsigned groupSize,
                                 float tolFactor, float extentRatio, uint32_t* groups, uint32_t* groupSys,
                                 uint32_t capacity, cudaStream_t s);

// ---------------------------------------------------------------------------------------------------- batch.cu
void launchBatchBoxes(const float* x, const float* y, const float* z, size_t n, const uint64_t* first,
                      uint32_t numSystems, const int* useGiven, uint32_t* mm, DevBox<float>* boxes, float* limits,
                      cudaStream_t s);
void launchBatchKeys(const float* x, const float* y, const float* z, size_t n, const uint64_t* first,
                     uint32_t numSystems, const DevBox<float>* boxes, int sysLevel, uint64_t* keys, int smCount,
                     cudaStream_t s);
void launchBatchRoots(uint32_t numSystems, const uint64_t* prefixes, int levelBegin, int levelEnd,
                      const int* childOffsets, int sysLevel, const DevBox<float>* boxes, const int* numShells,
                      SysTrav* out, int* rootNode, unsigned int* err, cudaStream_t s);
void launchBatchGroups(uint32_t numGroups, const uint64_t* first, const uint32_t* groupOffset, uint32_t numSystems,
                       uint32_t groupSize, uint32_t* start, uint32_t* end, uint32_t* sys, cudaStream_t s);

// ---------------------------------------------------------------------------------------------------- ewald.cu
//! wave vectors of the k-space sum for ceil(hCut) <= 3: at most the 7^3 - 1 non-zero vectors of [-3, 3]^3
constexpr int kEwaldMaxK = 343;

struct EwaldHost
{
    double mroot[8];
    double center[3];
    int replicaShells, ewaldShells;
    double L, lCut, hCut, alphaScale, smallR;
    int numK;
    double kdata[kEwaldMaxK * 5]; // per k vector: hs[3], fc, fs
};
EwaldHost ewaldSetup(const double* mroot, const double* center, int replicaShells, double L, double lCut,
                     double hCut, double alphaScale, double smallR);
//! adds the FP64 particle-level Ewald correction (every source's monopole) to pot (G m phi), ax, ay, az of targets
void launchEwaldTargetsF64(ryo_ctx* ctx, const int64_t* targets, size_t numTargets, const float* x, const float* y,
                           const float* z, const float* m, size_t numBodies, double L, int replicaShells, double lCut,
                           double hCut, double alphaScale, double smallR, double G, double* pot, double* ax,
                           double* ay, double* az, cudaStream_t s);
void launchEwaldGroups(const EwaldHost& e, const uint32_t* groupStart, const uint32_t* groupEnd, uint32_t numGroups,
                       const float* x, const float* y, const float* z, const float* m, float G, float* ugrav,
                       float* ax, float* ay, float* az, double* potentialOut, cudaStream_t s);
//! the double-coordinate instantiations: all double, and double coordinates with float masses and outputs
void launchEwaldGroups(const EwaldHost& e, const uint32_t* groupStart, const uint32_t* groupEnd, uint32_t numGroups,
                       const double* x, const double* y, const double* z, const double* m, float G, double* ugrav,
                       double* ax, double* ay, double* az, double* potentialOut, cudaStream_t s);
void launchEwaldGroups(const EwaldHost& e, const uint32_t* groupStart, const uint32_t* groupEnd, uint32_t numGroups,
                       const double* x, const double* y, const double* z, const float* m, float G, float* ugrav,
                       float* ax, float* ay, float* az, double* potentialOut, cudaStream_t s);

// ---------------------------------------------------------------------------------------------------- probe.cu
void measurePeaks(int smCount, double* fp32, double* fp32x2, double* copyGBs, cudaStream_t s);

// ---------------------------------------------------------------------------------------------------- direct.cu
template<class T>
void launchDirect(size_t first, size_t last, size_t numBodies, const T* boxL, int numShells, const T* x, const T* y,
                  const T* z, const T* m, const T* h, T* p, T* ax, T* ay, T* az, cudaStream_t s);
void launchDirectTargets(const int64_t* targets, size_t numTargets, const float* x, const float* y, const float* z,
                         const float* m, const float* h, size_t numBodies, double G, const double* boxL,
                         int numShells, double* pot, double* ax, double* ay, double* az, cudaStream_t s);

} // namespace ryo
