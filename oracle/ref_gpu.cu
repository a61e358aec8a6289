/*
 * Test infrastructure only: a C-ABI wrapper around the reference's own single-GPU gravity path, compiled from the
 * reference sources in place into oracle/_ref (never committed, never linked by the product). The GPU tests run it
 * beside the B200 kernels on the same inputs to pin the traversal's interaction statistics and forces, and the
 * reference arm of bench.py times it as the reference's plain GPU path on the same box.
 *
 * The flow is the reference demo's (ryoanji/test/demo.cu:82-104, :171-190, :205-226):
 *   TreeBuilder<uint64_t>::update (keys, sort, x/y/z gather, updateOctreeGpu, buildOctreeGpu, layout)
 *   -> computeLeafSourceCenterGpu, upsweepCentersGpu, computeLeafMultipoles, upsweepMultipoles per level, setMacGpu
 *   -> computeFixedGroups(64) -> traverse -> readBhStats.
 * Device pointers in; host scalars out. Every function runs on the default stream and returns after the device has
 * finished, as the reference's functions do.
 */
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>
#include <thrust/device_vector.h>

#include "cstone/cuda/device_vector.h"
#include "cstone/focus/source_center_gpu.h"
#include "cstone/traversal/groups_gpu.h"
#include "ryoanji/interface/ewald.cuh"
#include "ryoanji/interface/treebuilder.cuh"
#include "ryoanji/nbody/cartesian_qpole.hpp"
#include "ryoanji/nbody/traversal_gpu.h"
#include "ryoanji/nbody/types.h"
#include "ryoanji/nbody/upsweep_gpu.h"

namespace
{
using Builder = ryoanji::TreeBuilder<uint64_t>;

struct RefTree
{
    explicit RefTree(unsigned bucket)
        : tb(bucket)
    {
    }
    Builder tb;
    int numNodes  = 0;
    int numLeaves = 0;
};

template<class T>
cstone::Box<T> makeBox(const T* b6)
{
    return cstone::Box<T>(b6[0], b6[1], b6[2], b6[3], b6[4], b6[5]);
}

//! the demo's upsweep (ryoanji/test/demo.cu:205-226) for coordinate type T, mass type Tm and multipole MType
template<class T, class Tm, class MType>
void upsweepFlow(RefTree& r, const T* x, const T* y, const T* z, const Tm* m, const cstone::Box<T>& box, float theta,
                 ryoanji::Vec4<T>* centers, MType* multipoles)
{
    const Builder& tb = r.tb;
    const int* levelRange = tb.levelRange();
    int numLevels         = tb.maxTreeLevel();
    auto exec             = cstone::execution::gpuDefaultStream;
    cstone::computeLeafSourceCenterGpu(exec, x, y, z, m, tb.leafToInternal(), r.numLeaves, tb.layout(), centers);
    cstone::upsweepCentersGpu(exec, cstone::maxTreeLevel<uint64_t>{}, levelRange, tb.childOffsets(), centers);
    ryoanji::computeLeafMultipoles(x, y, z, m, tb.leafToInternal(), r.numLeaves, tb.layout(), centers, multipoles);
    for (int level = numLevels - 1; level >= 1; level--)
        ryoanji::upsweepMultipoles(levelRange[level], levelRange[level + 1], tb.childOffsets(), centers, multipoles);
    cstone::setMacGpu(exec, tb.nodeKeys(), r.numNodes, centers, 1.f / theta, box);
    cudaDeviceSynchronize();
}

template<class Tc, class Th, class Tm, class Ta, class Tf, class MType>
double traverseFlow(uint32_t first, uint32_t last, uint32_t numGroups, const uint32_t* gStart, const uint32_t* gEnd,
                    int initNode, const Tc* xt, const Tc* yt, const Tc* zt, const Tm* mt, const Th* ht, const Tc* xs,
                    const Tc* ys, const Tc* zs, const Tm* ms, const Th* hs, const int* childOffsets,
                    const int* internalToLeaf, const uint32_t* layout, const Tf* centers, const void* multipoles,
                    Tc G, int numShells, const Tc* boxL3, Ta* p, Ta* ax, Ta* ay, Ta* az, uint64_t* stats5,
                    uint64_t* retries)
{
    cstone::GroupView grp{first, last, numGroups, gStart, gEnd};
    thrust::device_vector<int> pool(ryoanji::stackSize(numGroups));
    ryoanji::Vec3<Tc> boxL{boxL3[0], boxL3[1], boxL3[2]};
    double pot = ryoanji::traverse(grp, initNode, xt, yt, zt, mt, ht, xs, ys, zs, ms, hs, childOffsets,
                                   internalToLeaf, layout, reinterpret_cast<const ryoanji::Vec4<Tf>*>(centers),
                                   static_cast<const MType*>(multipoles), G, numShells, boxL, p, ax, ay, az,
                                   thrust::raw_pointer_cast(pool.data()));
    cudaDeviceSynchronize();
    auto s = ryoanji::readBhStats();
    for (int i = 0; i < 5; ++i)
        stats5[i] = s[i];
    if (retries) *retries = ryoanji::readTraversalRetries();
    return pot;
}

} // namespace

extern "C"
{
    //! the reference's TreeBuilder with leaf bucket size @p bucket
    void* ref_gpu_create(unsigned bucket) { return new RefTree(bucket); }
    void ref_gpu_destroy(void* h) { delete static_cast<RefTree*>(h); }

    /*! TreeBuilder::update (ryoanji/src/ryoanji/interface/treebuilder.cuh:56-101): sorts x, y, z in place along the
     *  Hilbert curve of the box (xmin, xmax, ymin, ymax, zmin, zmax, host) and builds the octree; returns the node
     *  count */
    int ref_gpu_build_f32(void* h, float* x, float* y, float* z, size_t n, const float* box6)
    {
        auto& r     = *static_cast<RefTree*>(h);
        r.numNodes  = r.tb.update(x, y, z, n, makeBox(box6));
        r.numLeaves = r.tb.numLeafNodes();
        cudaDeviceSynchronize();
        return r.numNodes;
    }
    int ref_gpu_build_f64(void* h, double* x, double* y, double* z, size_t n, const double* box6)
    {
        auto& r     = *static_cast<RefTree*>(h);
        r.numNodes  = r.tb.update(x, y, z, n, makeBox(box6));
        r.numLeaves = r.tb.numLeafNodes();
        cudaDeviceSynchronize();
        return r.numNodes;
    }

    /*! the last tree's leaf count and levelRange (host, 23 entries) */
    void ref_gpu_tree(void* h, int* levelRange23, int* numLeaves)
    {
        auto& r = *static_cast<RefTree*>(h);
        for (int i = 0; i < 23; ++i)
            levelRange23[i] = r.tb.levelRange()[i];
        *numLeaves = r.numLeaves;
    }

    /*! copies of the last tree's arrays into caller device buffers (any may be null): layout (leaves + 1), nodeKeys,
     *  childOffsets, leafToInternal (leaves) and internalToLeaf (nodes) */
    int ref_gpu_tree_copy(void* h, uint32_t* layout, uint64_t* prefixes, int* childOffsets, int* leafToInternal,
                          int* internalToLeaf)
    {
        auto& r       = *static_cast<RefTree*>(h);
        size_t nodes  = size_t(r.numNodes), leaves = size_t(r.numLeaves);
        auto copy     = [](void* dst, const void* src, size_t bytes)
        { return dst ? cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToDevice) : cudaSuccess; };
        cudaError_t e = copy(layout, r.tb.layout(), 4 * (leaves + 1));
        if (e == cudaSuccess) e = copy(prefixes, r.tb.nodeKeys(), 8 * nodes);
        if (e == cudaSuccess) e = copy(childOffsets, r.tb.childOffsets(), 4 * nodes);
        if (e == cudaSuccess) e = copy(leafToInternal, r.tb.leafToInternal(), 4 * leaves);
        if (e == cudaSuccess) e = copy(internalToLeaf, r.tb.internalToLeaf(), 4 * nodes);
        return int(e);
    }

    /*! the demo's upsweep on the last tree: centres (4 per node: com, MAC r^2) and multipoles (8 per node for the
     *  quadrupole, 12 with mdq != 0) in the coordinate type */
    void ref_gpu_upsweep_f32(void* h, const float* x, const float* y, const float* z, const float* m,
                             const float* box6, float theta, float* centers, float* multipoles, int mdq)
    {
        auto& r  = *static_cast<RefTree*>(h);
        auto box = makeBox(box6);
        auto* c  = reinterpret_cast<ryoanji::Vec4<float>*>(centers);
        if (mdq)
            upsweepFlow(r, x, y, z, m, box, theta, c, reinterpret_cast<ryoanji::CartesianMDQpole<float>*>(multipoles));
        else
            upsweepFlow(r, x, y, z, m, box, theta, c,
                        reinterpret_cast<ryoanji::CartesianQuadrupole<float>*>(multipoles));
    }
    void ref_gpu_upsweep_f64(void* h, const double* x, const double* y, const double* z, const double* m,
                             const double* box6, float theta, double* centers, double* multipoles, int mdq)
    {
        auto& r  = *static_cast<RefTree*>(h);
        auto box = makeBox(box6);
        auto* c  = reinterpret_cast<ryoanji::Vec4<double>*>(centers);
        if (mdq)
            upsweepFlow(r, x, y, z, m, box, theta, c,
                        reinterpret_cast<ryoanji::CartesianMDQpole<double>*>(multipoles));
        else
            upsweepFlow(r, x, y, z, m, box, theta, c,
                        reinterpret_cast<ryoanji::CartesianQuadrupole<double>*>(multipoles));
    }

    /*! the mixed type set: double coordinates and centres, float masses and multipoles */
    void ref_gpu_upsweep_mixed(void* h, const double* x, const double* y, const double* z, const float* m,
                               const double* box6, float theta, double* centers, float* multipoles, int mdq)
    {
        auto& r  = *static_cast<RefTree*>(h);
        auto box = makeBox(box6);
        auto* c  = reinterpret_cast<ryoanji::Vec4<double>*>(centers);
        if (mdq)
            upsweepFlow(r, x, y, z, m, box, theta, c, reinterpret_cast<ryoanji::CartesianMDQpole<float>*>(multipoles));
        else
            upsweepFlow(r, x, y, z, m, box, theta, c,
                        reinterpret_cast<ryoanji::CartesianQuadrupole<float>*>(multipoles));
    }

    /*! cstone::computeFixedGroups (cstone/include/cstone/traversal/groups_gpu.cu:45-58): writes the group boundaries
     *  (numGroups + 1, host) if they fit in @p capacity; returns the group count */
    long ref_gpu_fixed_groups(uint32_t first, uint32_t last, unsigned groupSize, uint32_t* groupsHost, long capacity)
    {
        cstone::GroupData<cstone::execution::Gpu> groups;
        cstone::computeFixedGroups(cstone::execution::gpuDefaultStream, first, last, groupSize, groups);
        cudaDeviceSynchronize();
        long ng = long(groups.numGroups);
        if (ng + 1 <= capacity)
        {
            std::vector<cstone::LocalIndex> s(ng), e(ng);
            cudaMemcpy(s.data(), groups.groupStart, sizeof(uint32_t) * ng, cudaMemcpyDeviceToHost);
            cudaMemcpy(e.data(), groups.groupEnd, sizeof(uint32_t) * ng, cudaMemcpyDeviceToHost);
            for (long i = 0; i < ng; ++i)
                groupsHost[i] = s[i];
            groupsHost[ng] = ng > 0 ? e[ng - 1] : first;
        }
        return ng;
    }

    /*! ryoanji::traverse (ryoanji/src/ryoanji/nbody/traversal_gpu.cu:535-623), float instantiation, with the groups
     *  [gStart[i], gEnd[i]) (device); returns the total potential, and readBhStats / readTraversalRetries */
    double ref_gpu_traverse_f32(uint32_t first, uint32_t last, uint32_t numGroups, const uint32_t* gStart,
                                const uint32_t* gEnd, int initNode, const float* xt, const float* yt, const float* zt,
                                const float* mt, const float* ht, const float* xs, const float* ys, const float* zs,
                                const float* ms, const float* hs, const int* childOffsets, const int* internalToLeaf,
                                const uint32_t* layout, const float* centers, const float* multipoles, float G,
                                int numShells, const float* boxL3, float* p, float* ax, float* ay, float* az,
                                uint64_t* stats5, uint64_t* retries, int mdq)
    {
        if (mdq)
            return traverseFlow<float, float, float, float, float, ryoanji::CartesianMDQpole<float>>(
                first, last, numGroups, gStart, gEnd, initNode, xt, yt, zt, mt, ht, xs, ys, zs, ms, hs, childOffsets,
                internalToLeaf, layout, centers, multipoles, G, numShells, boxL3, p, ax, ay, az, stats5, retries);
        return traverseFlow<float, float, float, float, float, ryoanji::CartesianQuadrupole<float>>(
            first, last, numGroups, gStart, gEnd, initNode, xt, yt, zt, mt, ht, xs, ys, zs, ms, hs, childOffsets,
            internalToLeaf, layout, centers, multipoles, G, numShells, boxL3, p, ax, ay, az, stats5, retries);
    }

    /*! ryoanji::traverse, the all-double instantiation (traversal_gpu.cu:637) */
    double ref_gpu_traverse_f64(uint32_t first, uint32_t last, uint32_t numGroups, const uint32_t* gStart,
                                const uint32_t* gEnd, int initNode, const double* xt, const double* yt,
                                const double* zt, const double* mt, const double* ht, const double* xs,
                                const double* ys, const double* zs, const double* ms, const double* hs,
                                const int* childOffsets, const int* internalToLeaf, const uint32_t* layout,
                                const double* centers, const double* multipoles, double G, int numShells,
                                const double* boxL3, double* p, double* ax, double* ay, double* az, uint64_t* stats5,
                                uint64_t* retries, int mdq)
    {
        if (mdq)
            return traverseFlow<double, double, double, double, double, ryoanji::CartesianMDQpole<double>>(
                first, last, numGroups, gStart, gEnd, initNode, xt, yt, zt, mt, ht, xs, ys, zs, ms, hs, childOffsets,
                internalToLeaf, layout, centers, multipoles, G, numShells, boxL3, p, ax, ay, az, stats5, retries);
        return traverseFlow<double, double, double, double, double, ryoanji::CartesianQuadrupole<double>>(
            first, last, numGroups, gStart, gEnd, initNode, xt, yt, zt, mt, ht, xs, ys, zs, ms, hs, childOffsets,
            internalToLeaf, layout, centers, multipoles, G, numShells, boxL3, p, ax, ay, az, stats5, retries);
    }

    /*! ryoanji::traverse, the mixed instantiation (traversal_gpu.cu:638): double coordinates and centres, float
     *  softenings, masses, outputs and multipoles */
    double ref_gpu_traverse_mixed(uint32_t first, uint32_t last, uint32_t numGroups, const uint32_t* gStart,
                                  const uint32_t* gEnd, int initNode, const double* xt, const double* yt,
                                  const double* zt, const float* mt, const float* ht, const double* xs,
                                  const double* ys, const double* zs, const float* ms, const float* hs,
                                  const int* childOffsets, const int* internalToLeaf, const uint32_t* layout,
                                  const double* centers, const float* multipoles, double G, int numShells,
                                  const double* boxL3, float* p, float* ax, float* ay, float* az, uint64_t* stats5,
                                  uint64_t* retries, int mdq)
    {
        if (mdq)
            return traverseFlow<double, float, float, float, double, ryoanji::CartesianMDQpole<float>>(
                first, last, numGroups, gStart, gEnd, initNode, xt, yt, zt, mt, ht, xs, ys, zs, ms, hs, childOffsets,
                internalToLeaf, layout, centers, multipoles, G, numShells, boxL3, p, ax, ay, az, stats5, retries);
        return traverseFlow<double, float, float, float, double, ryoanji::CartesianQuadrupole<float>>(
            first, last, numGroups, gStart, gEnd, initNode, xt, yt, zt, mt, ht, xs, ys, zs, ms, hs, childOffsets,
            internalToLeaf, layout, centers, multipoles, G, numShells, boxL3, p, ax, ay, az, stats5, retries);
    }

    /*! the reference's whole plain GPU path in one call, for timing (demo.cu:82-104 and :171-190): build (x, y, z
     *  sorted in place), upsweep, fixed groups of 64, traverse (accumulates into p, ax, ay, az). m and h are taken
     *  in the sorted order as given, as the demo does. Device times of the three parts in ms3 (host); returns the
     *  total potential and the statistics in stats5. */
    double ref_gpu_solve_f32(unsigned bucket, float theta, float* x, float* y, float* z, const float* m,
                             const float* h, size_t n, const float* box6, float G, float* p, float* ax, float* ay,
                             float* az, uint64_t* stats5, float* ms3)
    {
        cudaEvent_t ev[4];
        for (auto& e : ev)
            cudaEventCreate(&e);
        RefTree r(bucket);
        auto box = makeBox(box6);
        cudaEventRecord(ev[0]);
        r.numNodes  = r.tb.update(x, y, z, n, box);
        r.numLeaves = r.tb.numLeafNodes();
        cudaEventRecord(ev[1]);
        thrust::device_vector<ryoanji::Vec4<float>> centers(r.numNodes);
        thrust::device_vector<ryoanji::CartesianQuadrupole<float>> mpoles(r.numNodes);
        upsweepFlow(r, static_cast<const float*>(x), y, z, m, box, theta, thrust::raw_pointer_cast(centers.data()),
                    thrust::raw_pointer_cast(mpoles.data()));
        cudaEventRecord(ev[2]);
        cstone::GroupData<cstone::execution::Gpu> groups;
        cstone::computeFixedGroups(cstone::execution::gpuDefaultStream, 0, n, ryoanji::bhMaxTargetSize(), groups);
        thrust::device_vector<int> pool(ryoanji::stackSize(groups.numGroups));
        double pot = ryoanji::traverse(groups.view(), 1, static_cast<const float*>(x), y, z, m, h, x, y, z, m, h,
                                       r.tb.childOffsets(), r.tb.internalToLeaf(), r.tb.layout(),
                                       thrust::raw_pointer_cast(centers.data()),
                                       thrust::raw_pointer_cast(mpoles.data()), G, 0,
                                       ryoanji::Vec3<float>{box.lx(), box.ly(), box.lz()}, p, ax, ay, az,
                                       thrust::raw_pointer_cast(pool.data()));
        cudaEventRecord(ev[3]);
        cudaEventSynchronize(ev[3]);
        for (int i = 0; i < 3; ++i)
            cudaEventElapsedTime(ms3 + i, ev[i], ev[i + 1]);
        auto s = ryoanji::readBhStats();
        for (int i = 0; i < 5; ++i)
            stats5[i] = s[i];
        for (auto& e : ev)
            cudaEventDestroy(e);
        return pot;
    }

    /*! ryoanji::computeGravityEwaldGpu (ryoanji/src/ryoanji/interface/ewald.cu:64-99) over the groups [gStart, gEnd)
     *  (device) of a cubic box (box6 host); settings5 = numReplicaShells, lCut, hCut, alpha_scale,
     *  small_R_scale_factor; returns the increment of *ugravTot. kind 0: (Quad<float>, float, float, float, float);
     *  1: (Quad<double>, double, double, double, double); 2: (Quad<float>, double, float, float, double). Coordinates,
     *  masses and outputs follow the kind; rootCenter and Mroot are host doubles. */
    double ref_gpu_ewald(int kind, const double* rootCenter3, const double* mroot8, uint32_t first, uint32_t last,
                         uint32_t numGroups, const uint32_t* gStart, const uint32_t* gEnd, const void* x, const void* y,
                         const void* z, const void* m, const double* box6, float G, void* ugrav, void* ax, void* ay,
                         void* az, const double* settings5)
    {
        if (numGroups == 0) return 0.0;
        cstone::GroupView grp{first, last, numGroups, gStart, gEnd};
        ryoanji::EwaldSettings es{int(settings5[0]), settings5[1], settings5[2], settings5[3], settings5[4]};
        double total = 0;
        if (kind == 0)
        {
            cstone::Vec3<float> rc{float(rootCenter3[0]), float(rootCenter3[1]), float(rootCenter3[2])};
            ryoanji::CartesianQuadrupole<float> M;
            for (int i = 0; i < 8; ++i)
                M[i] = float(mroot8[i]);
            float tot = 0;
            cstone::Box<float> box(box6[0], box6[1], box6[2], box6[3], box6[4], box6[5]);
            ryoanji::computeGravityEwaldGpu(rc, M, grp, (const float*)x, (const float*)y, (const float*)z,
                                            (const float*)m, box, G, (float*)ugrav, (float*)ax, (float*)ay,
                                            (float*)az, &tot, es);
            total = tot;
        }
        else
        {
            cstone::Vec3<double> rc{rootCenter3[0], rootCenter3[1], rootCenter3[2]};
            cstone::Box<double> box(box6[0], box6[1], box6[2], box6[3], box6[4], box6[5]);
            if (kind == 1)
            {
                ryoanji::CartesianQuadrupole<double> M;
                for (int i = 0; i < 8; ++i)
                    M[i] = mroot8[i];
                ryoanji::computeGravityEwaldGpu(rc, M, grp, (const double*)x, (const double*)y, (const double*)z,
                                                (const double*)m, box, G, (double*)ugrav, (double*)ax, (double*)ay,
                                                (double*)az, &total, es);
            }
            else
            {
                ryoanji::CartesianQuadrupole<float> M;
                for (int i = 0; i < 8; ++i)
                    M[i] = float(mroot8[i]);
                ryoanji::computeGravityEwaldGpu(rc, M, grp, (const double*)x, (const double*)y, (const double*)z,
                                                (const float*)m, box, G, (float*)ugrav, (float*)ax, (float*)ay,
                                                (float*)az, &total, es);
            }
        }
        cudaDeviceSynchronize();
        return total;
    }

    //! the last CUDA error of this library's runtime (0 = none); clears it
    int ref_gpu_last_error() { return int(cudaGetLastError()); }
}
