/*
 * TEST INFRASTRUCTURE ONLY — the CPU oracle of the single-GPU gravity path.
 *
 * A plain C++ restatement of the reference algorithm (Cornerstone SFC keys and octree, Ryoanji upsweep, the GPU
 * traversal's interaction rule, the CPU tree walk, direct sums and the Ewald correction). Only tests/, the smoke
 * check and bench.py's cpu_baseline leg load it, as the checker; the product never does. Its correctness is pinned
 * against the reference's own CPU code (oracle/_ref) through committed golden fixtures (tests/golden/).
 *
 * All arrays are host memory. Coordinates are float unless a name ends in _f64. Tree conventions are the
 * reference's: cornerstone leaf keys (numLeaves + 1 entries), Warren-Salmon placeholder-bit prefixes, nodes sorted
 * level-major, childOffsets 0 for leaves, parents stored once per sibling group at (child - 1) / 8.
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C"
{
#endif

    /* ---- SFC keys (cstone/include/cstone/sfc/sfc.hpp:153-207, hilbert.hpp:43-244, box.hpp:160-197) ---- */
    void orc_box_dim_bits_f32(const float* box6, unsigned* bits3);
    void orc_box_dim_bits_f64(const double* box6, unsigned* bits3);
    void orc_sfc_keys_f32(const float* x, const float* y, const float* z, size_t n, const float* box6, uint64_t* keys);
    void orc_sfc_keys_f64(const double* x, const double* y, const double* z, size_t n, const double* box6,
                          uint64_t* keys);
    /* integer box of the node that starts at @p key on @p level (hilbert.hpp:562-585), ibox6 = x0,x1,y0,y1,z0,z1 */
    void orc_hilbert_ibox(uint64_t key, unsigned level, unsigned bx, unsigned by, unsigned bz, int* ibox6);

    /* ---- sorting (cstone/include/cstone/primitives/gather.hpp:43-66): stable ascending sort, order = permutation */
    void orc_sort_keys(uint64_t* keys, uint32_t* order, size_t n);

    /* ---- cornerstone leaf array by the reference's iterative rebalance (cstone/include/cstone/tree/csarray.hpp)
     * returns numLeaves; writes leaves (numLeaves + 1) and counts only if numLeaves <= capacity */
    long orc_octree_leaves(const uint64_t* sortedKeys, size_t n, unsigned bucket, uint64_t* leaves, uint32_t* counts,
                           long capacity);

    /* ---- linked octree (cstone/include/cstone/tree/octree.hpp:56-196); numNodes = numLeaves + (numLeaves-1)/7,
     * parents has max(1, (numNodes - 1) / 8) entries, levelRange 23 */
    void orc_octree_link(const uint64_t* leaves, int numLeaves, uint64_t* prefixes, int* childOffsets, int* parents,
                         int* levelRange, int* internalToLeaf, int* leafToInternal);

    /* ---- upsweep: centres, multipoles, MAC radii.
     * mode 0: float arithmetic in the reference's CPU order (source_center.hpp:45-143, upsweep_cpu.hpp:41-74,
     *         cartesian_qpole.hpp:67-235).
     * mode 1: the same quantities accumulated in double and rounded to float once at the end (the precision the
     *         GPU path uses). The MAC radius is computed in float from the float centre in both modes.
     * centers: 4 floats per node (x, y, z, mac^2), multipoles: 8 floats per node. */
    void orc_upsweep_f32(int mode, const float* x, const float* y, const float* z, const float* m, int numLeaves,
                         const uint32_t* layout, const int* leafToInternal, const int* childOffsets,
                         const int* levelRange, const uint64_t* prefixes, int numNodes, float theta,
                         const float* box6, float* centers, float* multipoles);

    /* ---- the GPU traversal's interaction rule (ryoanji/src/ryoanji/nbody/traversal_gpu.cu:197-313, 431-518):
     * per target group the number of approximated cells (M2P) and of directly summed source bodies (P2P), summed
     * over the 27 (numShells = 1) or 1 periodic replicas. If acc4 is not NULL, also evaluates those interactions in
     * double precision (exact 1/sqrt) and ADDS (pot, ax, ay, az) per target to acc4 (without G). */
    void orc_traverse_rule(int numGroups, const uint32_t* groupStart, const uint32_t* groupEnd, const float* xt,
                           const float* yt, const float* zt, const float* ht, const float* xs, const float* ys,
                           const float* zs, const float* ms, const float* hs, const int* childOffsets,
                           const int* internalToLeaf, const uint32_t* layout, const float* centers,
                           const float* multipoles, int initNodeIdx, int numShells, const float* boxL3,
                           uint32_t* m2pCount, uint32_t* p2pCount, double* acc4);

    /* ---- reference CPU tree walk (ryoanji/src/ryoanji/nbody/traversal_cpu.hpp:67-230), float, 16-body groups.
     * Adds G * m * pot, G * a to pot, ax, ay, az; returns the total potential energy 0.5 * G * sum(m * pot). */
    double orc_gravity_cpu_f32(const int* childOffsets, const int* parents, const int* internalToLeaf,
                               const float* centers, const float* multipoles, const uint32_t* layout, int numLeaves,
                               const float* x, const float* y, const float* z, const float* h, const float* m,
                               const float* box6, float G, int numShells, float* pot, float* ax, float* ay,
                               float* az);

    /* ---- direct sum in double (traversal_cpu.hpp:232-268 semantics, P2P<true>): for each of the numTargets
     * target indices, sum over all n sources and numShells replicas; writes (not adds) pot (= G*m*phi), ax, ay, az */
    void orc_direct_f64(const float* x, const float* y, const float* z, const float* h, const float* m, size_t n,
                        const int64_t* targets, size_t numTargets, double G, const double* boxL3, int numShells,
                        double* pot, double* ax, double* ay, double* az);

    /* ---- kernels with double arguments (kernel.hpp:99-120, cartesian_qpole.hpp:67-176) ---- */
    void orc_p2p_f64(const double* ti, const double* sj, double mj, double hi, double hj, double* acc4);
    void orc_p2m_f64(const double* x, const double* y, const double* z, const double* m, unsigned n, double* center4,
                     double* quad8);
    void orc_m2p_f64(const double* target, const double* center, const double* quad8, double* acc4);

    /* ---- Ewald root-multipole correction (ryoanji/src/ryoanji/nbody/ewald.hpp:133-389), double throughout.
     * Adds to pot/ax/ay/az (pot gets G*m*phi); returns 0.5 * G * sum(m * phi). */
    double orc_ewald_f64(const double* rootCenter3, const double* mroot8, const double* x, const double* y,
                         const double* z, const double* m, size_t n, const double* box6, double G, double* pot,
                         double* ax, double* ay, double* az, int numReplicaShells, double lCut, double hCut,
                         double alphaScale, double smallR);

    /* analytic total potential of one particle in a periodic cube (the reference test helper at
     * ryoanji/test/nbody/ewald_cpu.cpp:211-234) */
    double orc_ewald_single_particle_energy(double m, unsigned N, double L, double G, double alphaScale);

    /* ---- whole CPU path for the CPU baseline: keys, sort, gather, leaves, link, float upsweep, CPU walk.
     * Inputs are replaced by sorted copies; seconds[3] = {build, upsweep, gravity}; returns the energy. */
    double orc_solve_f32(float* x, float* y, float* z, float* m, float* h, size_t n, const float* box6,
                         unsigned bucket, float theta, float G, float* pot, float* ax, float* ay, float* az,
                         double* seconds);

    /* ---- spatial target groups (cstone/traversal/groups_gpu.cuh:39-265, groups_gpu.cu:60-118) */
    uint64_t orc_find_splits_f64(const double* pos4, int G, double distCritSq);
    int orc_make_splits(uint64_t mask, int G, uint32_t* lengths);
    /* writes counts[window] (1 + splits) and, if capacity allows, groups[numGroups + 1]; returns numGroups */
    long orc_group_splits_f32(uint32_t first, uint32_t last, const float* x, const float* y, const float* z,
                              const float* h, const uint64_t* leaves, int numLeaves, const uint32_t* layout,
                              const float* box6, int groupSize, float tolFactor, float extentRatio, uint32_t* counts,
                              uint32_t* groups, long capacity);
    long orc_group_splits_f64(uint32_t first, uint32_t last, const double* x, const double* y, const double* z,
                              const double* h, const uint64_t* leaves, int numLeaves, const uint32_t* layout,
                              const double* box6, int groupSize, float tolFactor, float extentRatio,
                              uint32_t* counts, uint32_t* groups, long capacity);

    /* ---- monopole + dipole + quadrupole expansions (cartesian_qpole.hpp:237-423), double; 12 values per expansion */
    void orc_mdq_p2m_f64(const double* x, const double* y, const double* z, const double* m, unsigned n,
                         double* center4, double* mdq12);
    void orc_mdq_m2m_f64(int numChildren, const double* centers4, const double* mdq12, const double* outCenter4,
                         double* out12);
    void orc_mdq_m2p_f64(const double* target, const double* center, const double* mdq12, double* acc4);

#ifdef __cplusplus
}
#endif
