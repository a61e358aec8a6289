/*
 * TEST INFRASTRUCTURE ONLY.
 *
 * C-ABI wrapper around the reference's own CPU path (Cornerstone + Ryoanji headers), compiled from the reference
 * sources where they lie by oracle/Makefile into oracle/_ref/libryo_ref.so. Nothing in the product links it: the
 * tests use it to pin the restated oracle (oracle/ryo_oracle.cpp) and to write golden fixtures, and bench.py times
 * it as the CPU baseline ("kind": "reference").
 *
 * Every entry point forwards to the reference function named beside it; the wrapper itself adds no arithmetic.
 */
#include <cstdint>
#include <cstring>
#include <chrono>
#include <numeric>
#include <span>
#include <vector>

#include "cstone/sfc/sfc.hpp"
#include "cstone/primitives/gather.hpp"
#include "cstone/tree/csarray.hpp"
#include "cstone/tree/octree.hpp"
#include "cstone/focus/source_center.hpp"
#include "ryoanji/nbody/upsweep_cpu.hpp"
#include "ryoanji/nbody/traversal_cpu.hpp"
#include "ryoanji/nbody/ewald.hpp"

using cstone::LocalIndex;
using cstone::TreeNodeIndex;

namespace
{
template<class T>
cstone::Box<T> makeBox(const T* b)
{
    return cstone::Box<T>(b[0], b[1], b[2], b[3], b[4], b[5]);
}

template<class T>
cstone::Box<T> makeBox(const T* b, int periodic)
{
    auto bt = periodic ? cstone::BoundaryType::periodic : cstone::BoundaryType::open;
    return cstone::Box<T>(b[0], b[1], b[2], b[3], b[4], b[5], bt, bt, bt);
}

using Quad = ryoanji::CartesianQuadrupole<float>;
using MDQ  = ryoanji::CartesianMDQpole<float>;
using Center = cstone::SourceCenterType<float>;
} // namespace

extern "C"
{

    //! cstone::computeSfcKeys (cstone/include/cstone/sfc/sfc.hpp:297-305), Hilbert, 64-bit
    int ref_sfc_keys_f32(const float* x, const float* y, const float* z, size_t n, const float* box, uint64_t* keys)
    {
        std::fill(keys, keys + n, 0);
        cstone::computeSfcKeys(x, y, z, cstone::sfcKindPointer(keys), n, makeBox(box));
        return 0;
    }

    int ref_sfc_keys_f64(const double* x, const double* y, const double* z, size_t n, const double* box,
                         uint64_t* keys)
    {
        std::fill(keys, keys + n, 0);
        cstone::computeSfcKeys(x, y, z, cstone::sfcKindPointer(keys), n, makeBox(box));
        return 0;
    }

    //! cstone::decodeHilbert / hilbertIBox (cstone/include/cstone/sfc/hilbert.hpp:362-471,562-585)
    void ref_hilbert_ibox(uint64_t key, unsigned level, unsigned bx, unsigned by, unsigned bz, int* ibox6)
    {
        auto b  = cstone::hilbertIBox<uint64_t>(key, level, bx, by, bz);
        ibox6[0] = b.xmin();
        ibox6[1] = b.xmax();
        ibox6[2] = b.ymin();
        ibox6[3] = b.ymax();
        ibox6[4] = b.zmin();
        ibox6[5] = b.zmax();
    }

    //! Box::getBoxDimBits (cstone/include/cstone/sfc/box.hpp:160-163)
    void ref_box_dim_bits_f32(const float* box, unsigned* bits3)
    {
        auto a   = makeBox(box).getBoxDimBits(21);
        bits3[0] = a[0];
        bits3[1] = a[1];
        bits3[2] = a[2];
    }

    //! cstone::sort_by_key (cstone/include/cstone/primitives/gather.hpp:43-66): std::stable_sort of (key, i)
    void ref_sort_keys(uint64_t* keys, uint32_t* order, size_t n)
    {
        std::iota(order, order + n, 0u);
        cstone::sort_by_key(keys, keys + n, order);
    }

    //! cstone::computeOctree (cstone/include/cstone/tree/csarray.hpp:429-440)
    long ref_octree_leaves(const uint64_t* keys, size_t n, unsigned bucket, uint64_t* leaves, uint32_t* counts,
                           long capacity)
    {
        auto [tree, cnt] = cstone::computeOctree<uint64_t>(std::span<const uint64_t>(keys, n), bucket);
        long numLeaves   = long(cnt.size());
        if (numLeaves <= capacity)
        {
            std::copy(tree.begin(), tree.end(), leaves);
            std::copy(cnt.begin(), cnt.end(), counts);
        }
        return numLeaves;
    }

    //! cstone::updateInternalTree / buildOctreeCpu (cstone/include/cstone/tree/octree.hpp:168-196,363-369)
    void ref_octree_link(const uint64_t* leaves, int numLeaves, uint64_t* prefixes, int* childOffsets, int* parents,
                         int* levelRange, int* internalToLeaf, int* leafToInternal)
    {
        cstone::OctreeData<uint64_t, cstone::execution::Cpu> o;
        o.resize(numLeaves);
        cstone::updateInternalTree<uint64_t>(std::span<const uint64_t>(leaves, size_t(numLeaves) + 1), o.data());
        int numNodes = o.numNodes;
        std::copy_n(o.prefixes.data(), numNodes, prefixes);
        std::copy_n(o.childOffsets.data(), numNodes, childOffsets);
        std::copy_n(o.parents.data(), o.parents.size(), parents);
        std::copy_n(o.levelRange.data(), 23, levelRange);
        std::copy_n(o.internalToLeaf.data(), numNodes, internalToLeaf);
        std::copy_n(o.leafToInternal.data(), numNodes, leafToInternal);
    }

    /*! @brief CPU upsweep in the order of the reference's single-GPU demo (ryoanji/test/demo.cu:319-346) with the
     *         CPU functions: computeLeafMassCenter + upsweep(CombineSourceCenter) (source_center.hpp:112-127,
     *         octree.hpp:377-396), computeLeafMultipoles + upsweepMultipoles (upsweep_cpu.hpp:41-74),
     *         setMac (source_center.hpp:129-143)
     */
    void ref_upsweep_f32(const float* x, const float* y, const float* z, const float* m, size_t n, int numLeaves,
                         const uint32_t* layout, const int* leafToInternalLeaves, const int* childOffsets,
                         const int* levelRange, const uint64_t* prefixes, int numNodes, float theta, const float* box,
                         float* centers, float* multipoles)
    {
        auto* c  = reinterpret_cast<Center*>(centers);
        auto* mp = reinterpret_cast<Quad*>(multipoles);
        std::fill(centers, centers + 4 * numNodes, 0.f);
        std::fill(multipoles, multipoles + 8 * numNodes, 0.f);
        std::span<const TreeNodeIndex> l2i(leafToInternalLeaves, numLeaves);
        cstone::computeLeafMassCenter<float, float, float>({x, n}, {y, n}, {z, n}, {m, n}, l2i, layout, c);
        std::span<const TreeNodeIndex> lr(levelRange, 23);
        cstone::upsweep(lr, childOffsets, c, cstone::CombineSourceCenter<float>{});
        ryoanji::computeLeafMultipoles(x, y, z, m, l2i, layout, c, mp);
        ryoanji::upsweepMultipoles(lr, childOffsets, c, mp);
        cstone::setMac<float, uint64_t>({prefixes, size_t(numNodes)}, {c, size_t(numNodes)}, 1.0f / theta,
                                        makeBox(box));
    }

    //! ryoanji::computeGravity (ryoanji/src/ryoanji/nbody/traversal_cpu.hpp:172-230)
    double ref_gravity_cpu_f32(const int* childOffsets, const int* parents, const int* internalToLeaf,
                               const float* centers, const float* multipoles, const uint32_t* layout, int numLeaves,
                               const float* x, const float* y, const float* z, const float* h, const float* m,
                               const float* box, int periodic, float G, int numShells, float* pot, float* ax, float* ay,
                               float* az)
    {
        float utot = 0;
        ryoanji::computeGravity(childOffsets, parents, internalToLeaf, reinterpret_cast<const Center*>(centers),
                                reinterpret_cast<const Quad*>(multipoles), layout, 0, numLeaves, x, y, z, h, m,
                                makeBox(box, periodic), G, pot, ax, ay, az, &utot, numShells);
        return utot;
    }

    //! ryoanji::directSum (ryoanji/src/ryoanji/nbody/traversal_cpu.hpp:232-268), double
    void ref_direct_f64(const double* x, const double* y, const double* z, const double* h, const double* m,
                        unsigned n, float G, const double* boxL, int numShells, double* ax, double* ay, double* az,
                        double* pot)
    {
        ryoanji::directSum(x, y, z, h, m, n, G, {boxL[0], boxL[1], boxL[2]}, numShells, ax, ay, az, pot);
    }

    //! ryoanji::P2P (ryoanji/src/ryoanji/nbody/kernel.hpp:99-120), double, accumulating into acc4
    void ref_p2p_f64(const double* ti, const double* sj, double mj, double hi, double hj, double* acc4)
    {
        cstone::Vec4<double> acc{acc4[0], acc4[1], acc4[2], acc4[3]};
        acc = ryoanji::P2P(acc, cstone::Vec3<double>{ti[0], ti[1], ti[2]}, cstone::Vec3<double>{sj[0], sj[1], sj[2]},
                           mj, hi, hj);
        for (int i = 0; i < 4; ++i)
            acc4[i] = acc[i];
    }

    //! ryoanji::P2M + M2P (ryoanji/src/ryoanji/nbody/cartesian_qpole.hpp:110-176), double
    void ref_p2m_f64(const double* x, const double* y, const double* z, const double* m, unsigned n, double* center4,
                     double* quad8)
    {
        auto c = cstone::massCenter<double>(x, y, z, m, 0, n);
        ryoanji::CartesianQuadrupole<double> q;
        ryoanji::P2M(x, y, z, m, 0, n, c, q);
        for (int i = 0; i < 4; ++i)
            center4[i] = c[i];
        for (int i = 0; i < 8; ++i)
            quad8[i] = q[i];
    }

    void ref_m2p_f64(const double* target, const double* center, const double* quad8, double* acc4)
    {
        ryoanji::CartesianQuadrupole<double> q;
        for (int i = 0; i < 8; ++i)
            q[i] = quad8[i];
        cstone::Vec4<double> acc{acc4[0], acc4[1], acc4[2], acc4[3]};
        acc = ryoanji::M2P(acc, cstone::Vec3<double>{target[0], target[1], target[2]},
                           cstone::Vec3<double>{center[0], center[1], center[2]}, q);
        for (int i = 0; i < 4; ++i)
            acc4[i] = acc[i];
    }

    //! ryoanji::computeGravityEwald (ryoanji/src/ryoanji/nbody/ewald.hpp:356-389), float coordinates
    double ref_ewald_f32(const float* rootCenter3, const float* mroot8, const float* x, const float* y, const float* z,
                         const float* m, unsigned n, const float* box, float G, float* pot, float* ax, float* ay,
                         float* az, int numReplicaShells, double lCut, double hCut, double alphaScale, double smallR)
    {
        Quad q;
        for (int i = 0; i < 8; ++i)
            q[i] = mroot8[i];
        ryoanji::EwaldSettings s{numReplicaShells, lCut, hCut, alphaScale, smallR};
        float utot = 0;
        ryoanji::computeGravityEwald(cstone::Vec3<float>{rootCenter3[0], rootCenter3[1], rootCenter3[2]}, q, 0, n, x,
                                     y, z, m, makeBox(box, 1), G, pot, ax, ay, az, &utot, s);
        return utot;
    }

    //! same, double coordinates and moments
    double ref_ewald_f64(const double* rootCenter3, const double* mroot8, const double* x, const double* y,
                         const double* z, const double* m, unsigned n, const double* box, float G, double* pot,
                         double* ax, double* ay, double* az, int numReplicaShells, double lCut, double hCut,
                         double alphaScale, double smallR)
    {
        ryoanji::CartesianQuadrupole<double> q;
        for (int i = 0; i < 8; ++i)
            q[i] = mroot8[i];
        ryoanji::EwaldSettings s{numReplicaShells, lCut, hCut, alphaScale, smallR};
        double utot = 0;
        ryoanji::computeGravityEwald(cstone::Vec3<double>{rootCenter3[0], rootCenter3[1], rootCenter3[2]}, q, 0, n,
                                     x, y, z, m, makeBox(box, 1), G, pot, ax, ay, az, &utot, s);
        return utot;
    }

    /*! @brief the whole reference CPU path for one float system, as timed for the CPU baseline
     *
     * computeSfcKeys -> sort_by_key -> gather x,y,z,m,h -> computeOctree -> updateInternalTree -> CPU upsweep ->
     * computeGravity (16-body groups). x,y,z,m,h are replaced by their SFC-sorted copies; outputs are in sorted
     * order. @p seconds receives {build, upsweep, gravity}. Returns the total potential energy.
     */
    double ref_solve_f32(float* x, float* y, float* z, float* m, float* h, size_t n, const float* box,
                         unsigned bucket, float theta, float G, float* pot, float* ax, float* ay, float* az,
                         double* seconds)
    {
        using clock = std::chrono::steady_clock;
        auto t0     = clock::now();
        std::vector<uint64_t> keys(n);
        std::vector<uint32_t> order(n);
        ref_sfc_keys_f32(x, y, z, n, box, keys.data());
        ref_sort_keys(keys.data(), order.data(), n);
        std::vector<float> tmp(n);
        for (float* a : {x, y, z, m, h})
        {
#pragma omp parallel for schedule(static)
            for (size_t i = 0; i < n; ++i)
                tmp[i] = a[order[i]];
            std::copy(tmp.begin(), tmp.end(), a);
        }
        auto [tree, counts] = cstone::computeOctree<uint64_t>(std::span<const uint64_t>(keys.data(), n), bucket);
        int numLeaves       = int(counts.size());
        cstone::OctreeData<uint64_t, cstone::execution::Cpu> o;
        o.resize(numLeaves);
        cstone::updateInternalTree<uint64_t>(tree, o.data());
        std::vector<LocalIndex> layout(numLeaves + 1, 0);
        std::inclusive_scan(counts.begin(), counts.end(), layout.begin() + 1);
        auto t1 = clock::now();

        std::vector<float> centers(4 * o.numNodes), mpoles(8 * o.numNodes);
        ref_upsweep_f32(x, y, z, m, n, numLeaves, layout.data(), o.leafToInternal.data() + o.numInternalNodes,
                        o.childOffsets.data(), o.levelRange.data(), o.prefixes.data(), o.numNodes, theta, box,
                        centers.data(), mpoles.data());
        auto t2 = clock::now();

        std::fill(pot, pot + n, 0.f);
        std::fill(ax, ax + n, 0.f);
        std::fill(ay, ay + n, 0.f);
        std::fill(az, az + n, 0.f);
        double u = ref_gravity_cpu_f32(o.childOffsets.data(), o.parents.data(), o.internalToLeaf.data(),
                                       centers.data(), mpoles.data(), layout.data(), numLeaves, x, y, z, h, m, box, 0,
                                       G, 0, pot, ax, ay, az);
        auto t3 = clock::now();
        if (seconds)
        {
            seconds[0] = std::chrono::duration<double>(t1 - t0).count();
            seconds[1] = std::chrono::duration<double>(t2 - t1).count();
            seconds[2] = std::chrono::duration<double>(t3 - t2).count();
        }
        return u;
    }

    // ---- monopole + dipole + quadrupole (CartesianMDQpole, ryoanji/src/ryoanji/nbody/cartesian_qpole.hpp:237-423)

    //! ryoanji::P2M for CartesianMDQpole about the |m|-weighted centre (cstone::massCenter), double
    void ref_mdq_p2m_f64(const double* x, const double* y, const double* z, const double* m, unsigned n,
                         double* center4, double* mdq12)
    {
        auto c = cstone::massCenter<double>(x, y, z, m, 0, n);
        ryoanji::CartesianMDQpole<double> q;
        ryoanji::P2M(x, y, z, m, 0, n, c, q);
        for (int i = 0; i < 4; ++i)
            center4[i] = c[i];
        for (int i = 0; i < 12; ++i)
            mdq12[i] = q[i];
    }

    //! ryoanji::M2M for CartesianMDQpole, double: children centres (4 each) and multipoles (12 each)
    void ref_mdq_m2m_f64(int numChildren, const double* centers4, const double* mdq12, const double* outCenter4,
                         double* out12)
    {
        std::vector<cstone::Vec4<double>> c(numChildren);
        std::vector<ryoanji::CartesianMDQpole<double>> q(numChildren);
        for (int k = 0; k < numChildren; ++k)
        {
            for (int i = 0; i < 4; ++i)
                c[k][i] = centers4[4 * k + i];
            for (int i = 0; i < 12; ++i)
                q[k][i] = mdq12[12 * k + i];
        }
        cstone::Vec4<double> oc{outCenter4[0], outCenter4[1], outCenter4[2], outCenter4[3]};
        ryoanji::CartesianMDQpole<double> out;
        ryoanji::M2M(0, numChildren, oc, c.data(), q.data(), out);
        for (int i = 0; i < 12; ++i)
            out12[i] = out[i];
    }

    //! ryoanji::M2P for CartesianMDQpole, double, accumulating into acc4
    void ref_mdq_m2p_f64(const double* target, const double* center, const double* mdq12, double* acc4)
    {
        ryoanji::CartesianMDQpole<double> q;
        for (int i = 0; i < 12; ++i)
            q[i] = mdq12[i];
        cstone::Vec4<double> acc{acc4[0], acc4[1], acc4[2], acc4[3]};
        acc = ryoanji::M2P(acc, cstone::Vec3<double>{target[0], target[1], target[2]},
                           cstone::Vec3<double>{center[0], center[1], center[2]}, q);
        for (int i = 0; i < 4; ++i)
            acc4[i] = acc[i];
    }

    //! the reference CPU upsweep (as ref_upsweep_f32) with CartesianMDQpole multipoles (12 floats per node)
    void ref_upsweep_mdq_f32(const float* x, const float* y, const float* z, const float* m, size_t n, int numLeaves,
                             const uint32_t* layout, const int* leafToInternalLeaves, const int* childOffsets,
                             const int* levelRange, const uint64_t* prefixes, int numNodes, float theta,
                             const float* box, float* centers, float* multipoles)
    {
        auto* c  = reinterpret_cast<Center*>(centers);
        auto* mp = reinterpret_cast<MDQ*>(multipoles);
        std::fill(centers, centers + 4 * numNodes, 0.f);
        std::fill(multipoles, multipoles + 12 * numNodes, 0.f);
        std::span<const TreeNodeIndex> l2i(leafToInternalLeaves, numLeaves);
        cstone::computeLeafMassCenter<float, float, float>({x, n}, {y, n}, {z, n}, {m, n}, l2i, layout, c);
        std::span<const TreeNodeIndex> lr(levelRange, 23);
        cstone::upsweep(lr, childOffsets, c, cstone::CombineSourceCenter<float>{});
        ryoanji::computeLeafMultipoles(x, y, z, m, l2i, layout, c, mp);
        ryoanji::upsweepMultipoles(lr, childOffsets, c, mp);
        cstone::setMac<float, uint64_t>({prefixes, size_t(numNodes)}, {c, size_t(numNodes)}, 1.0f / theta,
                                        makeBox(box));
    }

    //! ryoanji::computeGravity with CartesianMDQpole multipoles
    double ref_gravity_cpu_mdq_f32(const int* childOffsets, const int* parents, const int* internalToLeaf,
                                   const float* centers, const float* multipoles, const uint32_t* layout,
                                   int numLeaves, const float* x, const float* y, const float* z, const float* h,
                                   const float* m, const float* box, int periodic, float G, int numShells,
                                   float* pot, float* ax, float* ay, float* az)
    {
        float utot = 0;
        ryoanji::computeGravity(childOffsets, parents, internalToLeaf, reinterpret_cast<const Center*>(centers),
                                reinterpret_cast<const MDQ*>(multipoles), layout, 0, numLeaves, x, y, z, h, m,
                                makeBox(box, periodic), G, pot, ax, ay, az, &utot, numShells);
        return utot;
    }

} // extern "C"
