/*
 * ryoanji-b200 — C ABI of the single-GPU Barnes-Hut gravity path for NVIDIA B200 (sm_100a).
 *
 * Plain pointers and sizes only. A function that takes a context (or a tree builder or engine made from one) runs
 * on the context's device, which it makes current for the call and restores afterwards; the others run on the
 * calling thread's current device. Every device array argument is memory of that device, and every stream one of
 * its streams, unless the comment says "host". Each entry point names the reference interface it replaces (paths
 * relative to the reference project root, tischwab0911/ryoanji). Functions return a ryo_status and never exit the
 * process.
 *
 * Conventions shared with the reference:
 *   - 64-bit Hilbert keys, 21 levels; keys equal to 2^63 mark removed particles.
 *   - cornerstone leaf arrays (numLeaves + 1 keys), Warren-Salmon placeholder-bit node prefixes, nodes sorted
 *     level-major; childOffsets is 0 for leaves; parents[(i - 1) / 8] is the parent of node i.
 *   - multipoles: 8 floats per node (mass, qxx, qxy, qxz, qyy, qyz, qzz, trace), traceless quadrupole times 3;
 *     source centres: 4 floats per node (x, y, z, squared MAC radius).
 *   - traversal outputs are ACCUMULATED into p, ax, ay, az.
 */
#ifndef RYOANJI_B200_H
#define RYOANJI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C"
{
#endif

#define RYO_API __attribute__((visibility("default")))

    typedef struct CUstream_st* ryo_stream_t; /* a cudaStream_t; NULL is the legacy default stream */

    typedef enum ryo_status
    {
        RYO_OK                              = 0,
        RYO_ERR_CUDA                        = 1, /* a CUDA call failed; see ryo_ctx_last_error */
        RYO_ERR_BAD_ARG                     = 2,
        RYO_ERR_OOM                         = 3,
        RYO_ERR_STACK_OVERFLOW_UNSPLITTABLE = 4, /* a single target still overflowed the traversal stack */
        RYO_ERR_TIMEOUT                     = 5, /* a bounded device wait gave up (error flag set by a kernel) */
        RYO_ERR_CAPACITY                    = 6, /* a caller-provided buffer is too small; see the size out-arg */
        RYO_ERR_NOT_CUBIC                   = 7, /* Ewald needs a cubic periodic box */
        RYO_ERR_NO_DEVICE                   = 8,
        RYO_ERR_INTERNAL                    = 9  /* an unexpected host-side failure inside the library (a C++ exception
                                                  that is no CUDA, argument or allocation error); see the last error */
    } ryo_status;

    /* cstone::BoundaryType (cstone/include/cstone/sfc/box.hpp:84-90) */
    enum
    {
        RYO_BOUNDARY_OPEN       = 0,
        RYO_BOUNDARY_PERIODIC   = 1,
        RYO_BOUNDARY_FIXED      = 2,
        RYO_BOUNDARY_CUBIC_OPEN = 3
    };

    /* cstone::Box<float> / Box<double> (cstone/include/cstone/sfc/box.hpp:99-214): xmin,xmax,ymin,ymax,zmin,zmax */
    typedef struct ryo_box_f32
    {
        float limits[6];
        int boundary[3];
    } ryo_box_f32;

    typedef struct ryo_box_f64
    {
        double limits[6];
        int boundary[3];
    } ryo_box_f64;

    /* cstone::GroupView (cstone/include/cstone/traversal/groups.hpp:28-35); groupStart/groupEnd are device arrays */
    typedef struct ryo_group_view
    {
        uint32_t firstBody, lastBody, numGroups;
        const uint32_t* groupStart;
        const uint32_t* groupEnd;
    } ryo_group_view;

    /* ryoanji::EwaldSettings (ryoanji/src/ryoanji/nbody/ewald.h:23-31). As in the reference, ceil(hCut) must be at
     * most 3 (ewald.hpp:52-60); no value may be negative, and alpha_scale must be positive unless lCut, hCut and
     * alpha_scale are all 0 (Ewald off). Other settings give RYO_ERR_BAD_ARG wherever a periodic box uses them. */
    typedef struct ryo_ewald_settings
    {
        int numReplicaShells;        /* 1 */
        double lCut;                 /* 2.6 */
        double hCut;                 /* 2.8 */
        double alpha_scale;          /* 2.0 */
        double small_R_scale_factor; /* 3.0e-3 */
    } ryo_ewald_settings;

    typedef struct ryo_ctx ryo_ctx_t;
    typedef struct ryo_treebuilder ryo_treebuilder_t;

    /* ------------------------------------------------------------------------------------------ context */

    RYO_API const char* ryo_status_string(ryo_status s);
    /* library version "major.minor.patch" */
    RYO_API const char* ryo_version(void);
    /* A context owns scratch memory, per-call counters and statistics on one device (no global device state, so
     * several contexts may run concurrently on different streams). A context is not locked: calls on one context
     * (and on the tree builders and engines made from it) must not overlap from several host threads; give each
     * thread its own context. */
    RYO_API ryo_status ryo_ctx_create(int device, ryo_ctx_t** out);
    RYO_API void ryo_ctx_destroy(ryo_ctx_t* ctx);
    /* the message of the context's last failed call; with NULL, that of the calling thread's last failed call of a
     * function that takes no context (and of a failed ryo_ctx_create) */
    RYO_API const char* ryo_ctx_last_error(const ryo_ctx_t* ctx);

    /* ------------------------------------------------------------------------------------------ cstone layer */

    /* cstone::computeSfcKeys (cstone/include/cstone/sfc/sfc_gpu.h:100-102, sfc_gpu.cu:35-44): Hilbert keys of
     * x, y, z in @p box; keys already equal to 2^63 are left unchanged. */
    RYO_API ryo_status ryo_compute_sfc_keys_f32(const float* x, const float* y, const float* z, uint64_t* keys,
                                                size_t n, const ryo_box_f32* box, ryo_stream_t stream);
    RYO_API ryo_status ryo_compute_sfc_keys_f64(const double* x, const double* y, const double* z, uint64_t* keys,
                                                size_t n, const ryo_box_f64* box, ryo_stream_t stream);

    /* bounding box of the coordinates (min/max per axis, exact), written to host @p limits6 */
    RYO_API ryo_status ryo_compute_bounding_box_f32(ryo_ctx_t* ctx, const float* x, const float* y, const float* z,
                                                    size_t n, float* limits6, ryo_stream_t stream);

    /* cstone::sequence (cstone/include/cstone/primitives/primitives_gpu.h): v[i] = first + i */
    RYO_API ryo_status ryo_sequence(uint32_t* v, size_t n, uint32_t first, ryo_stream_t stream);

    /* cstone::sortByKey with caller buffers (cstone/include/cstone/primitives/primitives_gpu.cu:311-356): stable
     * ascending sort of keys[0:n) carrying values along; keyBuf/valueBuf hold n elements each; tmp holds
     * ryo_sort_by_key_temp_bytes(n) bytes. Onesweep radix sort over bits [0, 64). n must be below 2^32 (the
     * sort's digit offsets are 32-bit); a larger n returns RYO_ERR_BAD_ARG. */
    RYO_API size_t ryo_sort_by_key_temp_bytes(size_t n);
    RYO_API ryo_status ryo_sort_by_key(uint64_t* keys, uint32_t* values, size_t n, uint64_t* keyBuf,
                                       uint32_t* valueBuf, void* tmp, size_t tmpBytes, ryo_stream_t stream);

    /* The sort of ryo_sort_by_key for callers that cannot allocate device memory (a host whose pool allocator holds
     * the free HBM, or a loop that cannot afford the device-wide wait of cudaFree). It has no counterpart in the
     * reference. Its scratch is one fixed device array per device, so it takes no tmp argument and allocates
     * nothing; n is at most RYO_SORT_STATIC_MAX_KEYS, a larger n returns RYO_ERR_CAPACITY and sorts nothing.
     * The first call on a device looks up that array's address (which may load the module): make it before any
     * stream capture. A cudaDeviceReset ends the context that held the array; the next call on that device finds it
     * again in the new context (and is then a first call). Calls on one device share the array: calls that overlap
     * in time race, so serialise them. */
#define RYO_SORT_STATIC_MAX_KEYS (1u << 24)
    RYO_API ryo_status ryo_sort_by_key_static(uint64_t* keys, uint32_t* values, size_t n, uint64_t* keyBuf,
                                              uint32_t* valueBuf, ryo_stream_t stream);

    /* Failure-detection self-test, no counterpart in the reference: one onesweep tile runs while the tile before it
     * never publishes its counts, so the tile's bounded look-back wait (2^22 polls, a few seconds) runs out. Returns
     * RYO_ERR_TIMEOUT, as a sort whose wait ran out does, and leaves the context usable; RYO_ERR_INTERNAL if the
     * wait did not report. Allocates and frees its own small buffers. */
    RYO_API ryo_status ryo_sort_wait_timeout_selftest(ryo_stream_t stream);

    /* cstone::computeOctree / updateOctreeGpu to convergence (cstone/include/cstone/tree/csarray.hpp:409-440,
     * update_gpu.cuh:43-68): the cornerstone leaf array of sorted keys with at most @p bucketSize particles per
     * leaf. Built in one pass (no host-synchronised rebalance loop); identical to the reference's fixed point.
     * Writes leaves[numLeaves + 1] and counts[numLeaves] if numLeaves <= capacity; *numLeaves (host) always.
     * n must be below 2^32. */
    RYO_API ryo_status ryo_compute_octree(ryo_ctx_t* ctx, const uint64_t* sortedKeys, size_t n, unsigned bucketSize,
                                          uint64_t* leaves, uint32_t* counts, int capacity, int* numLeaves,
                                          ryo_stream_t stream);

    /* cstone::buildOctreeGpu (cstone/include/cstone/tree/octree_gpu.cu:138-200): internal octree of a leaf array.
     * numNodes = numLeaves + (numLeaves - 1) / 7; parents holds max(1, (numNodes - 1) / 8) entries; levelRange is
     * HOST memory (23 entries), d_levelRange device memory (23 entries, may be NULL). */
    RYO_API ryo_status ryo_build_octree(ryo_ctx_t* ctx, const uint64_t* leaves, int numLeaves, uint64_t* prefixes,
                                        int* childOffsets, int* parents, int* levelRange, int* d_levelRange,
                                        int* internalToLeaf, int* leafToInternal, ryo_stream_t stream);

    /* cstone::computeFixedGroups (cstone/include/cstone/traversal/groups_gpu.cu:45-58): groups[0:numGroups+1] of
     * groupSize consecutive bodies in [first, last); groupStart = groups, groupEnd = groups + 1 */
    RYO_API ryo_status ryo_compute_fixed_groups(uint32_t first, uint32_t last, unsigned groupSize, uint32_t* groups,
                                                ryo_stream_t stream);

    /* cstone::computeGroupSplits (cstone/include/cstone/traversal/groups_gpu.cu:60-151, groups_gpu.cuh:39-265):
     * spatially compact target groups of at most groupSize (32 or 64) SFC-sorted bodies [first, last): fixed windows
     * split where consecutive bodies are farther apart than min(tolFactor * cbrt(smallest leaf volume), 2 h) and, when
     * a window is longer than extentRatio * tolFactor * its smallest leaf edge, into equal chunks. h may be NULL.
     * leaves/layout: the cornerstone leaf array and body layout of the same tree; box: the key box. extentRatio < 0
     * selects the reference default (8, or the environment variable CSTONE_GROUP_EXTENT_SPLIT). *numGroups (host)
     * always receives the count; groups[0:*numGroups + 1] are written if capacity allows (else RYO_ERR_CAPACITY). */
    RYO_API ryo_status ryo_compute_group_splits_f32(ryo_ctx_t* ctx, uint32_t first, uint32_t last, const float* x,
                                                    const float* y, const float* z, const float* h,
                                                    const uint64_t* leaves, int numLeaves, const uint32_t* layout,
                                                    const ryo_box_f32* box, unsigned groupSize, float tolFactor,
                                                    float extentRatio, uint32_t* groups, uint32_t capacity,
                                                    uint32_t* numGroups, ryo_stream_t stream);

    /* ------------------------------------------------------------------------------------------ upsweep
     * The individual steps of the reference's upward pass. Sums run in double precision on the device; stored
     * values are float. centers: 4 floats per node, multipoles: 8 floats per node. */

    /* cstone::computeLeafSourceCenterGpu (cstone/include/cstone/focus/source_center_gpu.h:65-80) */
    RYO_API ryo_status ryo_compute_leaf_source_center_f32(const float* x, const float* y, const float* z,
                                                          const float* m, const int* leafToInternal, int numLeaves,
                                                          const uint32_t* layout, float* centers,
                                                          ryo_stream_t stream);
    /* cstone::upsweepCentersGpu (source_center_gpu.h:82-92); levelRange is HOST memory */
    RYO_API ryo_status ryo_upsweep_centers_f32(int numLevels, const int* levelRange, const int* childOffsets,
                                               float* centers, ryo_stream_t stream);
    /* ryoanji::computeLeafMultipoles (ryoanji/src/ryoanji/nbody/upsweep_gpu.h:24-31) */
    RYO_API ryo_status ryo_compute_leaf_multipoles_f32(const float* x, const float* y, const float* z, const float* m,
                                                       const int* leafToInternal, int numLeaves,
                                                       const uint32_t* layout, const float* centers,
                                                       float* multipoles, ryo_stream_t stream);
    /* ryoanji::upsweepMultipoles (upsweep_gpu.h:33-41): M2M for cells [firstCell, lastCell) */
    RYO_API ryo_status ryo_upsweep_multipoles_f32(int firstCell, int lastCell, const int* childOffsets,
                                                  const float* centers, float* multipoles, ryo_stream_t stream);
    /* the same two steps for CartesianMDQpole (INSTANTIATE_MULTIPOLE(CartesianMDQpole), upsweep_gpu.cu:143):
     * 12 floats per node (mass, qxx, qxy, qxz, qyy, qyz, qzz, trace, px, py, pz, 0), FP64 sums */
    RYO_API ryo_status ryo_compute_leaf_multipoles_mdq_f32(const float* x, const float* y, const float* z,
                                                           const float* m, const int* leafToInternal, int numLeaves,
                                                           const uint32_t* layout, const float* centers,
                                                           float* multipoles, ryo_stream_t stream);
    RYO_API ryo_status ryo_upsweep_multipoles_mdq_f32(int firstCell, int lastCell, const int* childOffsets,
                                                      const float* centers, float* multipoles, ryo_stream_t stream);

    /* The steps above for the reference's other two type sets (COMPUTE_LEAF_SOURCE_CENTER_GPU,
     * source_center_gpu.cu:164-170; upsweepCentersGpu, :204-209; INSTANTIATE_MULTIPOLE, upsweep_gpu.cu:134-143;
     * SET_MAC_GPU, source_center_gpu.cu:312-319): _f64 takes double coordinates, masses, centres (4 doubles per
     * node) and multipoles (8 or 12 doubles per node); _mixed takes double coordinates and centres with float masses
     * and multipoles. The sums run in double as in _f32; stored values are rounded once to their type. */
    RYO_API ryo_status ryo_compute_leaf_source_center_f64(const double* x, const double* y, const double* z,
                                                          const double* m, const int* leafToInternal, int numLeaves,
                                                          const uint32_t* layout, double* centers,
                                                          ryo_stream_t stream);
    RYO_API ryo_status ryo_compute_leaf_source_center_mixed(const double* x, const double* y, const double* z,
                                                            const float* m, const int* leafToInternal, int numLeaves,
                                                            const uint32_t* layout, double* centers,
                                                            ryo_stream_t stream);
    RYO_API ryo_status ryo_upsweep_centers_f64(int numLevels, const int* levelRange, const int* childOffsets,
                                               double* centers, ryo_stream_t stream);
    RYO_API ryo_status ryo_compute_leaf_multipoles_f64(const double* x, const double* y, const double* z,
                                                       const double* m, const int* leafToInternal, int numLeaves,
                                                       const uint32_t* layout, const double* centers,
                                                       double* multipoles, ryo_stream_t stream);
    RYO_API ryo_status ryo_compute_leaf_multipoles_mixed(const double* x, const double* y, const double* z,
                                                         const float* m, const int* leafToInternal, int numLeaves,
                                                         const uint32_t* layout, const double* centers,
                                                         float* multipoles, ryo_stream_t stream);
    RYO_API ryo_status ryo_compute_leaf_multipoles_mdq_f64(const double* x, const double* y, const double* z,
                                                           const double* m, const int* leafToInternal, int numLeaves,
                                                           const uint32_t* layout, const double* centers,
                                                           double* multipoles, ryo_stream_t stream);
    RYO_API ryo_status ryo_compute_leaf_multipoles_mdq_mixed(const double* x, const double* y, const double* z,
                                                             const float* m, const int* leafToInternal, int numLeaves,
                                                             const uint32_t* layout, const double* centers,
                                                             float* multipoles, ryo_stream_t stream);
    RYO_API ryo_status ryo_upsweep_multipoles_f64(int firstCell, int lastCell, const int* childOffsets,
                                                  const double* centers, double* multipoles, ryo_stream_t stream);
    RYO_API ryo_status ryo_upsweep_multipoles_mixed(int firstCell, int lastCell, const int* childOffsets,
                                                    const double* centers, float* multipoles, ryo_stream_t stream);
    RYO_API ryo_status ryo_upsweep_multipoles_mdq_f64(int firstCell, int lastCell, const int* childOffsets,
                                                      const double* centers, double* multipoles, ryo_stream_t stream);
    RYO_API ryo_status ryo_upsweep_multipoles_mdq_mixed(int firstCell, int lastCell, const int* childOffsets,
                                                        const double* centers, float* multipoles,
                                                        ryo_stream_t stream);
    RYO_API ryo_status ryo_set_mac_f64(const uint64_t* prefixes, int numNodes, double* centers, float invTheta,
                                       const ryo_box_f64* box, ryo_stream_t stream);

    /* cstone::setMacGpu (source_center_gpu.h:104-116): centers[i][3] = squared vector-MAC radius, 0 if massless */
    RYO_API ryo_status ryo_set_mac_f32(const uint64_t* prefixes, int numNodes, float* centers, float invTheta,
                                       const ryo_box_f32* box, ryo_stream_t stream);

    /* ------------------------------------------------------------------------------------------ traversal */

    /* ryoanji::bhMaxTargetSize (ryoanji/src/ryoanji/nbody/traversal_gpu.h:58-59): 64 */
    RYO_API int ryo_bh_max_target_size(void);
    /* ryoanji::stackSize (traversal_gpu.h:61-62): size of the caller stack pool in ints. The B200 traversal keeps
     * its stacks in shared memory, so this is 0; a pool passed by a caller is not used. */
    RYO_API uint32_t ryo_stack_size(uint32_t numGroups);

    /* ryoanji::traverse (ryoanji/src/ryoanji/nbody/traversal_gpu.h:51-56), float instantiation: Barnes-Hut
     * accelerations of the targets grouped by @p grp from the tree of the sources. Starts with the 8 siblings at
     * initNodeIdx. numShells > 0 adds the (2 numShells + 1)^3 periodic replicas of edge boxL (3 floats, host).
     * Accumulates G m phi into p (if not NULL) and G a into ax, ay, az. *totalPotential (host, may be NULL)
     * receives 0.5 G sum(m phi) over the traversed targets. Groups whose traversal overflows the stack are split
     * and traversed again (ryoanji/src/ryoanji/nbody/traversal_gpu.cu:582-618). Every group must hold 1 to 64
     * targets within [firstBody, lastBody) (RYO_ERR_BAD_ARG otherwise; the call reads the group arrays back to check
     * them). The call synchronises its stream (the group check, the split passes, the statistics), so it cannot be
     * captured in a CUDA graph. */
    RYO_API ryo_status ryo_traverse_f32(ryo_ctx_t* ctx, const ryo_group_view* grp, int initNodeIdx, const float* xt,
                                        const float* yt, const float* zt, const float* mt, const float* ht,
                                        const float* xs, const float* ys, const float* zs, const float* ms,
                                        const float* hs, const int* childOffsets, const int* internalToLeaf,
                                        const uint32_t* layout, const float* sourceCenter, const float* multipoles,
                                        float G, int numShells, const float* boxL, float* p, float* ax, float* ay,
                                        float* az, double* totalPotential, ryo_stream_t stream);

    /* options of the extended traversal (not in the reference): per-group interaction counts and stack depth */
    typedef struct ryo_traverse_options
    {
        uint32_t* groupM2P; /* device, numGroups entries (may be NULL): approximated cells per group */
        uint32_t* groupP2P; /* device, numGroups entries (may be NULL): directly summed source bodies per group */
        int stackCapacity;  /* traversal stack entries per warp, 0 = default (512); small values force splits */
        int multipole;      /* RYO_MULTIPOLE_QUADRUPOLE: 8 floats per node in multipoles (default);
                               RYO_MULTIPOLE_MDQ: 12 floats per node (CartesianMDQpole, traversal_gpu.cu:641) */
    } ryo_traverse_options;

    RYO_API ryo_status ryo_traverse_ex_f32(ryo_ctx_t* ctx, const ryo_group_view* grp, int initNodeIdx,
                                           const float* xt, const float* yt, const float* zt, const float* mt,
                                           const float* ht, const float* xs, const float* ys, const float* zs,
                                           const float* ms, const float* hs, const int* childOffsets,
                                           const int* internalToLeaf, const uint32_t* layout,
                                           const float* sourceCenter, const float* multipoles, float G, int numShells,
                                           const float* boxL, float* p, float* ax, float* ay, float* az,
                                           double* totalPotential, const ryo_traverse_options* options,
                                           ryo_stream_t stream);

    /* ryoanji::traverse, the two double-coordinate instantiations (TRAVERSE_MPOLE, traversal_gpu.cu:635-641): _f64
     * is (double, double, double, double, double, multipoles of doubles); _mixed is (Tc = double, Th = Tm = Ta =
     * float, Tf = double, multipoles of floats), the caller side of codes whose particle positions are double. As in
     * the reference, the MAC and the sums run in double with the single-precision rsqrt of the double argument
     * (kernel.hpp:38-52). Centres are 4 doubles per node; multipoles 8 values per node, or 12 with options->multipole
     * = RYO_MULTIPOLE_MDQ. Semantics, checks and statistics are those of ryo_traverse_ex_f32 (options may be NULL).
     * A group too costly for one warp is evaluated by one warp here (no split second pass). */
    RYO_API ryo_status ryo_traverse_f64(ryo_ctx_t* ctx, const ryo_group_view* grp, int initNodeIdx, const double* xt,
                                        const double* yt, const double* zt, const double* mt, const double* ht,
                                        const double* xs, const double* ys, const double* zs, const double* ms,
                                        const double* hs, const int* childOffsets, const int* internalToLeaf,
                                        const uint32_t* layout, const double* sourceCenter, const double* multipoles,
                                        double G, int numShells, const double* boxL, double* p, double* ax,
                                        double* ay, double* az, double* totalPotential,
                                        const ryo_traverse_options* options, ryo_stream_t stream);
    RYO_API ryo_status ryo_traverse_mixed(ryo_ctx_t* ctx, const ryo_group_view* grp, int initNodeIdx, const double* xt,
                                          const double* yt, const double* zt, const float* mt, const float* ht,
                                          const double* xs, const double* ys, const double* zs, const float* ms,
                                          const float* hs, const int* childOffsets, const int* internalToLeaf,
                                          const uint32_t* layout, const double* sourceCenter,
                                          const float* multipoles, double G, int numShells, const double* boxL,
                                          float* p, float* ax, float* ay, float* az, double* totalPotential,
                                          const ryo_traverse_options* options, ryo_stream_t stream);

    /* The locally essential tree of the last ryo_solve_f32 on this context for another rank's domain, the exchange
     * step of a system spread over several GPUs (cstone/include/cstone/focus/octree_focus_mpi.hpp:629, globalExchange,
     * and the peer exchange it feeds). peerBox6 (host: xmin, xmax, ymin, ymax, zmin, zmax) bounds the other rank's
     * bodies. A node is exported iff every strict ancestor below the root fails the MAC against that box; a node
     * that fails it keeps its eight children (internal) or sends its bodies (leaf); one that passes is sent as a
     * multipole without children or bodies. The export is one packed buffer of 32-bit words (counts->words of them;
     * N nodes, L leaves with bodies, B bodies): centres [0, 4N), multipoles [4N, 12N) (8 floats), childOffsets
     * [12N, 13N), internalToLeaf [13N, 14N), layout [14N, 14N + L + 2), then x, y, z, m, h of the bodies (B each).
     * ryo_traverse_f32 evaluates it as the source tree of the other rank's targets (initNodeIdx 1, or 0 if N is 1).
     * Writes *counts always; RYO_ERR_CAPACITY (nothing written to @p buffer) if capacityWords is too small. Open
     * boundaries and quadrupole expansions only. The call synchronises its stream to read the sizes. Not in the
     * reference's single-GPU interface. */
    typedef struct ryo_let_counts
    {
        uint32_t numNodes, numLeaves, numBodies, pad;
        uint64_t words;
    } ryo_let_counts;
    RYO_API ryo_status ryo_let_export_f32(ryo_ctx_t* ctx, const float* peerBox6, uint32_t* buffer,
                                          size_t capacityWords, ryo_let_counts* counts, ryo_stream_t stream);

    /* ryoanji::readBhStats (traversal_gpu.h:64-65): {sumP2P, maxP2P, sumM2P, maxM2P, maxStack} of the last
     * traversal on this context; maxP2P is 0xFFFFFFFF if a single target could not be traversed */
    RYO_API ryo_status ryo_read_bh_stats(ryo_ctx_t* ctx, uint64_t* stats5);
    /* ryoanji::readTraversalRetries (traversal_gpu.h:67-68) */
    RYO_API uint64_t ryo_read_traversal_retries(ryo_ctx_t* ctx);

    /* ------------------------------------------------------------------------------------------ Ewald */

    /* ryoanji::computeGravityEwaldGpu (ryoanji/src/ryoanji/interface/ewald.cuh:24-27): root-multipole Ewald
     * correction of the targets in @p grp; rootCenter (3) and Mroot (8) are HOST arrays; *ugravTot (host) is
     * incremented by 0.5 G sum(m phi_ewald). The k-space sum runs in double precision. */
    RYO_API ryo_status ryo_compute_gravity_ewald_f32(ryo_ctx_t* ctx, const float* rootCenter, const float* Mroot,
                                                     const ryo_group_view* grp, const float* x, const float* y,
                                                     const float* z, const float* m, const ryo_box_f32* box, float G,
                                                     float* ugrav, float* ax, float* ay, float* az, double* ugravTot,
                                                     const ryo_ewald_settings* settings, ryo_stream_t stream);
    /* the double-coordinate instantiations (COMPUTE_GRAVITY_EWALD_GPU, ewald.cu:101-110): _f64 is
     * (CartesianQuadrupole<double or float>, double, double, double, double), the root expansion given as 8 doubles;
     * _mixed is (CartesianQuadrupole<float>, double, float, float, double). The real-space images run in double
     * there, as the reference's run in its coordinate type. */
    RYO_API ryo_status ryo_compute_gravity_ewald_f64(ryo_ctx_t* ctx, const double* rootCenter, const double* Mroot,
                                                     const ryo_group_view* grp, const double* x, const double* y,
                                                     const double* z, const double* m, const ryo_box_f64* box,
                                                     float G, double* ugrav, double* ax, double* ay, double* az,
                                                     double* ugravTot, const ryo_ewald_settings* settings,
                                                     ryo_stream_t stream);
    RYO_API ryo_status ryo_compute_gravity_ewald_mixed(ryo_ctx_t* ctx, const double* rootCenter, const float* Mroot,
                                                       const ryo_group_view* grp, const double* x, const double* y,
                                                       const double* z, const float* m, const ryo_box_f64* box,
                                                       float G, float* ugrav, float* ax, float* ay, float* az,
                                                       double* ugravTot, const ryo_ewald_settings* settings,
                                                       ryo_stream_t stream);

    /* ------------------------------------------------------------------------------------------ direct sums */

    /* ryoanji::directSum (ryoanji/src/ryoanji/nbody/direct.cuh:87-107): all-pairs sum for targets [first, last)
     * over numBodies sources with (2 numShells + 1)^3 replicas; adds m phi to p and a to ax, ay, az (no G).
     * first <= last <= numBodies, and replicas need boxL (RYO_ERR_BAD_ARG otherwise). */
    RYO_API ryo_status ryo_direct_sum_f32(size_t first, size_t last, size_t numBodies, const float* boxL,
                                          int numShells, const float* x, const float* y, const float* z,
                                          const float* m, const float* h, float* p, float* ax, float* ay, float* az,
                                          ryo_stream_t stream);
    RYO_API ryo_status ryo_direct_sum_f64(size_t first, size_t last, size_t numBodies, const double* boxL,
                                          int numShells, const double* x, const double* y, const double* z,
                                          const double* m, const double* h, double* p, double* ax, double* ay,
                                          double* az, ryo_stream_t stream);
    /* accuracy reference: double-precision direct sum for selected targets of float data, exact 1/sqrt
     * (the P2P<true> form, ryoanji/src/ryoanji/nbody/kernel.hpp:55-120); writes G m phi and G a per target. Every
     * target index must be a body (the call reads the indices back to check them, synchronising its stream;
     * RYO_ERR_BAD_ARG otherwise). */
    RYO_API ryo_status ryo_direct_targets_f64(const int64_t* targets, size_t numTargets, const float* x,
                                              const float* y, const float* z, const float* m, const float* h,
                                              size_t numBodies, double G, const double* boxL, int numShells,
                                              double* pot, double* ax, double* ay, double* az, ryo_stream_t stream);

    /* The periodic check (not in the reference): ADDS the FP64 particle-level Ewald correction to pot (G m phi), ax,
     * ay, az of the chosen targets, i.e. the reference's Ewald formulas (ryoanji/src/ryoanji/nbody/ewald.hpp:200-327)
     * with every source's monopole in place of the root multipole. After ryo_direct_targets_f64 with numShells =
     * settings->numReplicaShells over the same cubic box of edge L this gives the targets' periodic sum. */
    RYO_API ryo_status ryo_ewald_targets_f64(ryo_ctx_t* ctx, const int64_t* targets, size_t numTargets, const float* x,
                                             const float* y, const float* z, const float* m, size_t numBodies,
                                             double L, const ryo_ewald_settings* settings, double G, double* pot,
                                             double* ax, double* ay, double* az, ryo_stream_t stream);

    /* ------------------------------------------------------------------------------------------ TreeBuilder
     * ryoanji::TreeBuilder<uint64_t> (ryoanji/src/ryoanji/interface/treebuilder.cuh:34-125) */

    RYO_API ryo_status ryo_treebuilder_create(ryo_ctx_t* ctx, unsigned ncrit, ryo_treebuilder_t** out);
    RYO_API void ryo_treebuilder_destroy(ryo_treebuilder_t* tb);
    /* TreeBuilder::update: sorts x, y, z in place into SFC order and builds the tree; *numNodes (host) receives
     * the total node count. Like the reference, only x, y, z are permuted; ryo_treebuilder_order gives the
     * permutation for other per-particle arrays. */
    RYO_API ryo_status ryo_treebuilder_update_f32(ryo_treebuilder_t* tb, float* x, float* y, float* z, size_t n,
                                                  const ryo_box_f32* box, int* numNodes, ryo_stream_t stream);
    RYO_API ryo_status ryo_treebuilder_update_f64(ryo_treebuilder_t* tb, double* x, double* y, double* z, size_t n,
                                                  const ryo_box_f64* box, int* numNodes, ryo_stream_t stream);

    /* device arrays of the last update, valid until the next update (TreeBuilder accessors, treebuilder.cuh:103-112) */
    typedef struct ryo_tree_view
    {
        int numLeafNodes, numInternalNodes, numNodes;
        unsigned maxTreeLevel;        /* 21 */
        const uint32_t* layout;       /* numLeafNodes + 1 */
        const uint64_t* nodeKeys;     /* prefixes, numNodes */
        const int* childOffsets;      /* numNodes */
        const int* leafToInternal;    /* the leaf part: numLeafNodes entries */
        const int* internalToLeaf;    /* numNodes */
        const int* parents;           /* max(1, (numNodes - 1) / 8) */
        const uint64_t* leaves;       /* numLeafNodes + 1 */
        const uint32_t* order;        /* numBodies: original index of each sorted body */
        const uint64_t* sortedKeys;   /* numBodies */
        int levelRange[23];           /* host copy */
    } ryo_tree_view;
    RYO_API ryo_status ryo_treebuilder_view(const ryo_treebuilder_t* tb, ryo_tree_view* out);

    /* ------------------------------------------------------------------------------------------ fused solve
     * The B200 plain path for one system: keys, sort, gather, leaves, links, fused FP64 upsweep with MAC radii,
     * fixed groups, traversal, Ewald if periodic. Not in the reference; it composes the functions above with the
     * reference's semantics except that it permutes every per-particle array (TreeBuilder permutes only x, y, z). */
    /* multipole types of the reference (ryoanji/src/ryoanji/nbody/cartesian_qpole.hpp) */
    enum
    {
        RYO_MULTIPOLE_QUADRUPOLE = 0, /* CartesianQuadrupole: mass + traceless quadrupole (8 values) */
        RYO_MULTIPOLE_MDQ        = 1  /* CartesianMDQpole: mass + traceless quadrupole + dipole (12 values) */
    };

    typedef struct ryo_solve_params
    {
        unsigned bucketSize;         /* leaf capacity, reference ncrit (64) */
        unsigned groupSize;          /* target group size, <= 64 (64) */
        float theta;                 /* opening angle (0.5) */
        float G;                     /* gravitational constant (1) */
        int useBox;                  /* 1: use @p box; 0: bounding box of the data (open boundaries) */
        ryo_box_f32 box;             /* coordinate box; periodic boundary on all axes enables replicas + Ewald */
        int numShells;               /* periodic replica shells of the traversal when periodic, in [0, 4] (1) */
        ryo_ewald_settings ewald;    /* Ewald settings when periodic. As in the reference (the traverse and
                                        computeGravityEwaldGpu calls of MultipoleHolder take them separately),
                                        ewald.numReplicaShells, the shells the correction assumes the tree has
                                        summed, is not tied to numShells; a consistent periodic solve sets both to
                                        the same value. */
        int stackCapacity;           /* 0 = default */
        int timing;                  /* 1: record per-phase device times into ryo_solve_stats.ms */
        float groupTolerance;        /* > 0: spatial target groups (ryo_compute_group_splits_f32) with this
                                        tolFactor and no interaction radius (h is the softening here), groupSize
                                        32 or 64; 0: fixed groups, the reference demo's (0).
                                        The batched solve and the engine split each system's fixed windows
                                        with that system's box. */
        float groupExtentRatio;      /* window-extent ratio of the spatial groups; < 0: the reference default (-1) */
        int multipole;               /* RYO_MULTIPOLE_QUADRUPOLE (CartesianQuadrupole, default) or
                                        RYO_MULTIPOLE_MDQ (CartesianMDQpole: adds the dipole, for signed masses) */
    } ryo_solve_params;

    typedef struct ryo_solve_stats
    {
        int numLeaves, numNodes, numGroups;
        uint64_t sumP2P, maxP2P, sumM2P, maxM2P, maxStack, retries;
        double potentialEnergy; /* 0.5 G sum(m phi), tree + Ewald */
        float box[6];           /* the box used */
        /* with params.timing: device milliseconds of keys+sort+gather, leaves+links, upsweep, traversal (all
         * passes), Ewald, and the whole solve */
        float ms[6];
    } ryo_solve_stats;

    RYO_API void ryo_solve_params_default(ryo_solve_params* p);

    /* x, y, z, m, h: in any order on entry, SFC-sorted on return; vx, vy, vz (may be NULL) are permuted along;
     * p, ax, ay, az are overwritten with the potential (G m phi) and acceleration in sorted order; order (may be
     * NULL) receives the original index of each sorted body. stats (host, may be NULL). */
    RYO_API ryo_status ryo_solve_f32(ryo_ctx_t* ctx, const ryo_solve_params* params, float* x, float* y, float* z,
                                     float* m, float* h, float* vx, float* vy, float* vz, size_t n, float* p,
                                     float* ax, float* ay, float* az, uint32_t* order, ryo_solve_stats* stats,
                                     ryo_stream_t stream);

    /* The same solve from and to HOST memory (pinned memory copies fastest): x, y, z, m, h are read (not changed);
     * xs, ys, zs (may be NULL) receive the positions in SFC order, p, ax, ay, az the potential and acceleration in
     * that order, order (may be NULL) the original index of each sorted body. The copies overlap the solve: m and h
     * upload during the key sort and the leaf and link construction, the order downloads while the tree is built and
     * the sorted positions during the upsweep. For an open box, when p, ax, ay and az are page-locked and mapped
     * (cudaHostAlloc, cudaMallocHost, or cudaHostRegister with cudaHostRegisterMapped), the traversal stores its
     * results straight into them while it runs. Otherwise, for an open box with fixed groups the traversal runs in 8
     * launches whose results download while the next one runs.
     * Returns when every output is in host memory. Device buffers are context scratch. */
    RYO_API ryo_status ryo_solve_host_f32(ryo_ctx_t* ctx, const ryo_solve_params* params, const float* x,
                                          const float* y, const float* z, const float* m, const float* h, size_t n,
                                          float* xs, float* ys, float* zs, float* p, float* ax, float* ay, float* az,
                                          uint32_t* order, ryo_solve_stats* stats, ryo_stream_t stream);

    /* ------------------------------------------------------------------------------------------ batched solve
     * Many independent systems solved together, one launch per phase (not in the reference, which solves one system
     * per call). The body arrays are the systems' bodies concatenated: system s owns [firstBody, firstBody +
     * numBodies), in order and without gaps. Each system gets its own box (given, or the cube enclosing its bodies),
     * tree, groups, traversal and, for a periodic cubic box, Ewald correction; the results equal per-system calls of
     * ryo_solve_f32 with the same box and parameters wherever the system's tree stops above level 21 - L, where
     * L = ceil(log8(numSystems)) (at least 1) octree levels hold the system index. */
#define RYO_BATCH_MAX_SYSTEMS 4096
    typedef struct ryo_system
    {
        uint64_t firstBody;
        uint32_t numBodies; /* >= 1 */
        int useBox;         /* 0: the cube enclosing the system's bodies, open boundaries; 1: box below */
        ryo_box_f32 box;    /* with useBox; periodic boxes must be cubic */
        int numShells;      /* periodic replica shells of the traversal (periodic boxes only) */
    } ryo_system;

    /* params: bucketSize, groupSize, theta, G, ewald, stackCapacity and timing apply to every system (useBox, box and
     * numShells of params are ignored). Bodies are SFC-sorted within their system on return, vx, vy, vz (may be
     * NULL) permuted along; p, ax, ay, az overwritten; order (may be NULL) receives the original index of each
     * sorted body. energies (host, numSystems, may be NULL): 0.5 G sum(m phi) per system; boxes (host, 6 floats per
     * system, may be NULL): the box each system used. stats: totals over all systems. */
    RYO_API ryo_status ryo_solve_batch_f32(ryo_ctx_t* ctx, const ryo_solve_params* params, const ryo_system* systems,
                                           int numSystems, float* x, float* y, float* z, float* m, float* h, float* vx,
                                           float* vy, float* vz, size_t n, float* p, float* ax, float* ay, float* az,
                                           uint32_t* order, double* energies, float* boxes, ryo_solve_stats* stats,
                                           ryo_stream_t stream);

    /* ------------------------------------------------------------------------------------------ served stream
     * A request loop over the batched solve (not in the reference): requests (a particle set and K kick-drift-kick
     * leapfrog steps) are admitted in arrival order while the HBM budget and the system slots allow, stay resident
     * across their steps, and every ryo_engine_step advances all resident requests with one batched solve. A
     * request's first step evaluates its initial forces; it then takes numSteps steps of
     *     v += a dt/2;  x += v dt;  a = F(x);  v += a dt/2
     * (periodic systems wrap x into their box) and retires. Its host inputs must stay valid until it is admitted,
     * its host output until it retires. One engine belongs to one host thread; it uses its context's scratch. */
    typedef struct ryo_engine ryo_engine_t;
    typedef struct ryo_engine_params
    {
        ryo_solve_params solve; /* bucketSize, groupSize, theta, G, ewald, stackCapacity, timing */
        double hbmBudgetBytes;  /* admission budget (default 120e9) */
        double bytesPerBody;    /* device bytes charged per resident body (default 256) */
        int maxSystems;         /* resident requests at most (default and upper limit RYO_BATCH_MAX_SYSTEMS) */
        uint64_t reserveBodies; /* resident bodies the arenas hold from creation on (default 0: grown on demand,
                                   doubling, which waits for the device at each growth) */
        uint64_t maxStepBodies; /* bodies one step advances at most (default 7 x 2^20; 0: every resident request each
                                   step). Taken in the order of their remaining work (bodies x steps left, least
                                   first), the resident requests that still fit join the step (the first always
                                   does): short requests are not held to the pace of the long ones. The choice is
                                   renewed when requests are admitted or retire. */
    } ryo_engine_params;
    typedef struct ryo_engine_request
    {
        uint64_t tag;
        uint32_t numBodies;
        const float *x, *y, *z, *m, *h; /* host */
        const float *vx, *vy, *vz;      /* host, may be NULL (zero velocities) */
        int useBox;                     /* 0: the cube enclosing the bodies, recomputed every step */
        ryo_box_f32 box;
        int numShells;
        int numSteps; /* leapfrog steps after the initial force evaluation */
        float dt;
        float* out; /* host, may be NULL: on retirement 10 * numBodies floats, arrays of x, y, z, vx, vy, vz, ax,
                       ay, az, p in submission order (ax..p: G a and G m phi at the final positions) */
    } ryo_engine_request;
    typedef struct ryo_engine_step_info
    {
        int admitted, retired, resident, queued, solved, retries;
        uint64_t residentBodies;
        float ms[6]; /* phase times of the batched solve when params.solve.timing */
        /* interactions of the step's batched solve: sums over bodies and maxima over target groups */
        uint64_t sumP2P, maxP2P, sumM2P, maxM2P;
        /* host wall milliseconds of the step's parts: admission and arena rebuild, batched solve, kicks and
         * energies, retirement (results to the host) */
        float hostMs[4];
    } ryo_engine_step_info;
    typedef struct ryo_engine_result
    {
        uint64_t tag;
        uint32_t numBodies;
        int stepsDone;
        double kineticEnergy, potentialEnergy; /* at retirement */
        double initialEnergy;                  /* kinetic + potential after the initial force evaluation */
    } ryo_engine_result;

    RYO_API void ryo_engine_params_default(ryo_engine_params* p);
    RYO_API ryo_status ryo_engine_create(ryo_ctx_t* ctx, const ryo_engine_params* params, ryo_engine_t** out);
    RYO_API void ryo_engine_destroy(ryo_engine_t* engine);
    RYO_API const char* ryo_engine_last_error(const ryo_engine_t* engine);
    /* queue a request; RYO_ERR_CAPACITY if it alone exceeds the budget, RYO_ERR_NOT_CUBIC for a periodic box that is
     * not a cube and RYO_ERR_BAD_ARG for replica shells outside [0, 4] or, for a periodic request, Ewald settings
     * that the single-system solve refuses (refused here rather than at a later step; engine creation accepts any
     * Ewald settings, which open requests never use) */
    RYO_API ryo_status ryo_engine_submit(ryo_engine_t* engine, const ryo_engine_request* request);
    /* admit, kick-drift, one batched solve of every resident request, kick, retire the finished ones */
    RYO_API ryo_status ryo_engine_step(ryo_engine_t* engine, ryo_engine_step_info* info, ryo_stream_t stream);
    /* take up to capacity results of retired requests (oldest first); *count receives how many */
    RYO_API ryo_status ryo_engine_poll(ryo_engine_t* engine, ryo_engine_result* out, int capacity, int* count);
    RYO_API ryo_status ryo_engine_status(const ryo_engine_t* engine, int* queued, int* resident, double* bytesInUse);

    /* Field of the last ryo_solve_f32 on this context at separate targets: the reference's MultipoleHolder::compute
     * with distinct target and source arrays (ryoanji/src/ryoanji/interface/multipole_holder.cuh:64-77). The targets
     * (any order, any positions) are SFC-sorted internally and grouped in fixed groups of the solve's groupSize;
     * mt (may be NULL: unit masses) scales the potential, ht (may be NULL: 0) is the targets' softening. p (may be
     * NULL), ax, ay, az are OVERWRITTEN in the caller's order with G m phi and G a, Ewald included for a periodic
     * solve. The solve's tree and its source arrays (its x, y, z, m, h) must be unchanged since that solve; a
     * batched solve on the same context invalidates it. stats (may be NULL): interaction counts, energy. */
    RYO_API ryo_status ryo_solve_targets_f32(ryo_ctx_t* ctx, const float* xt, const float* yt, const float* zt,
                                             const float* mt, const float* ht, size_t n, float* p, float* ax,
                                             float* ay, float* az, ryo_solve_stats* stats, ryo_stream_t stream);

    /* device arrays of the last ryo_solve_f32 on this context (valid until the next solve on it): the sorted keys,
     * permutation, tree and the packed node records the traversal read (16 floats per node: centre x, y, z, squared
     * MAC radius; multipole mass, qxx, qxy, qxz, qyy, qyz, qzz, trace; then 4 ints: first child, first body, body
     * count, unused), plus the double-precision root expansion the Ewald correction used. */
    typedef struct ryo_solve_arrays
    {
        int numLeaves, numNodes, numGroups;
        const uint64_t* sortedKeys;
        const uint32_t* order;
        const uint64_t* leaves;
        const uint32_t* layout;
        const uint64_t* prefixes;
        const int* childOffsets;
        const int* internalToLeaf;
        const int* leafToInternal; /* full array: numNodes entries */
        const int* parents;
        const float* nodeData;
        const uint32_t* groups;
        const uint32_t* groupM2P; /* per target group: approximated cells (all replicas) */
        const uint32_t* groupP2P; /* per target group: directly summed source bodies */
        int levelRange[23];
        double rootCenter[3];
        double rootMultipole[8];
        const float* dipoles; /* RYO_MULTIPOLE_MDQ: 4 floats per node (px, py, pz, 0); NULL otherwise */
    } ryo_solve_arrays;
    RYO_API ryo_status ryo_solve_arrays_get(ryo_ctx_t* ctx, ryo_solve_arrays* out);

    /* ------------------------------------------------------------------------------------------ measurement */

    /* number of kernels this library has launched in the process so far (every launch is counted) */
    RYO_API uint64_t ryo_kernel_launches(void);
    /* calibration for roofline denominators (about 0.2 s): out3 = {FP32 FMA TFLOP/s, packed f32x2 FMA TFLOP/s,
     * streaming copy GB/s (read + write)} at the clocks of the call */
    RYO_API ryo_status ryo_measure_peaks(ryo_ctx_t* ctx, double* out3, ryo_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* RYOANJI_B200_H */
