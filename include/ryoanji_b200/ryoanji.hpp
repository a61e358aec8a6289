/*
 * ryoanji-b200 — C++ drop-in surface over the C ABI (header only, C++17).
 *
 * Re-creates the template signatures that the reference's callers use (ryoanji/src/ryoanji/interface/
 * treebuilder.cuh:34-125, ryoanji/src/ryoanji/nbody/traversal_gpu.h:51-70, upsweep_gpu.h:24-41,
 * interface/ewald.cuh:24-27, and the cstone execution::Gpu functions) for the instantiations that the B200 library
 * implements: 64-bit keys and the reference's three type sets of the upward pass and the traversal: all float, all
 * double, and double coordinates and centres with float masses, softenings, multipoles and outputs (its "mixed"
 * instantiation). Multipoles are CartesianQuadrupole<T> (8 values per node) or CartesianMDQpole<T> (12), source
 * centres Vec4<T> (4 values per node). Device arrays are device pointers, as in the reference.
 *
 * Differences a caller sees:
 *   - everything lives in namespace ryo; ryoanji_b200/compat.hpp adds the reference's namespaces and spellings
 *     (cstone::, ryoanji::, execution::Gpu first arguments) on top of this header;
 *   - failures throw ryo::Error (status + message) instead of exiting the process;
 *   - each function takes an optional stream (last argument) and an optional ryo::Context; the default context
 *     is the current device's;
 *   - traverse ignores gmPool: the traversal stack lives in shared memory. stackSize() returns 0 so a caller that
 *     sizes gmPool from it allocates nothing.
 */
#ifndef RYOANJI_B200_RYOANJI_HPP
#define RYOANJI_B200_RYOANJI_HPP

#include <array>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>

#include "../ryoanji_b200.h"

namespace ryo
{

using TreeNodeIndex = int;
using LocalIndex    = uint32_t;

class Error : public std::runtime_error
{
public:
    Error(ryo_status s, const std::string& what)
        : std::runtime_error(what)
        , status(s)
    {
    }
    ryo_status status;
};

inline void check(ryo_status s, const ryo_ctx_t* ctx = nullptr)
{
    if (s != RYO_OK)
    {
        std::string msg = ryo_status_string(s);
        const char* detail = ryo_ctx_last_error(ctx);
        if (detail && *detail) msg += std::string(": ") + detail;
        throw Error(s, msg);
    }
}

//! owning handle of a ryo_ctx (per-device counters, statistics, scratch)
class Context
{
public:
    explicit Context(int device = 0)
    {
        ryo_ctx_t* h = nullptr;
        check(ryo_ctx_create(device, &h));
        h_.reset(h);
    }
    ryo_ctx_t* get() const { return h_.get(); }

private:
    struct Del
    {
        void operator()(ryo_ctx_t* c) const { ryo_ctx_destroy(c); }
    };
    std::unique_ptr<ryo_ctx_t, Del> h_;
};

inline Context& defaultContext()
{
    static Context ctx(0);
    return ctx;
}

//! the subset of cstone::Box<T> (cstone/include/cstone/sfc/box.hpp:99-213) that the gravity path reads
enum class BoundaryType : int
{
    open     = RYO_BOUNDARY_OPEN,
    periodic = RYO_BOUNDARY_PERIODIC,
    fixed    = RYO_BOUNDARY_FIXED,
};

template<class T>
class Box
{
public:
    Box(T xmin, T xmax, T ymin, T ymax, T zmin, T zmax, BoundaryType bx = BoundaryType::open,
        BoundaryType by = BoundaryType::open, BoundaryType bz = BoundaryType::open)
        : lim_{xmin, xmax, ymin, ymax, zmin, zmax}
        , bnd_{int(bx), int(by), int(bz)}
    {
    }
    Box(T lo, T hi, BoundaryType b = BoundaryType::open)
        : Box(lo, hi, lo, hi, lo, hi, b, b, b)
    {
    }
    T xmin() const { return lim_[0]; }
    T xmax() const { return lim_[1]; }
    T ymin() const { return lim_[2]; }
    T ymax() const { return lim_[3]; }
    T zmin() const { return lim_[4]; }
    T zmax() const { return lim_[5]; }
    T lx() const { return lim_[1] - lim_[0]; }
    T ly() const { return lim_[3] - lim_[2]; }
    T lz() const { return lim_[5] - lim_[4]; }
    BoundaryType boundaryX() const { return BoundaryType(bnd_[0]); }
    BoundaryType boundaryY() const { return BoundaryType(bnd_[1]); }
    BoundaryType boundaryZ() const { return BoundaryType(bnd_[2]); }

    ryo_box_f32 abiF32() const
    {
        ryo_box_f32 b{};
        for (int i = 0; i < 6; ++i)
            b.limits[i] = float(lim_[i]);
        for (int i = 0; i < 3; ++i)
            b.boundary[i] = bnd_[i];
        return b;
    }
    ryo_box_f64 abiF64() const
    {
        ryo_box_f64 b{};
        for (int i = 0; i < 6; ++i)
            b.limits[i] = double(lim_[i]);
        for (int i = 0; i < 3; ++i)
            b.boundary[i] = bnd_[i];
        return b;
    }

private:
    std::array<T, 6> lim_;
    std::array<int, 3> bnd_;
};

//! cstone::GroupView (cstone/include/cstone/traversal/groups.hpp:28-35)
struct GroupView
{
    LocalIndex firstBody, lastBody, numGroups;
    const LocalIndex* groupStart;
    const LocalIndex* groupEnd;

    ryo_group_view abi() const { return ryo_group_view{firstBody, lastBody, numGroups, groupStart, groupEnd}; }
};

template<class T>
struct Vec3
{
    T x, y, z;
};

//! the reference's multipole types (ryoanji/src/ryoanji/nbody/cartesian_qpole.hpp:24-48)
template<class T>
using CartesianQuadrupole = std::array<T, 8>;
template<class T>
using CartesianMDQpole = std::array<T, 12>;
//! a source centre: x, y, z and the squared MAC radius (cstone::SourceCenterType / Vec4<T>)
template<class T>
using Vec4 = std::array<T, 4>;

namespace detail
{
//! the value type of a multipole array element, and whether it is a CartesianMDQpole
template<class M>
struct Mpole
{
    using value                = M;
    static constexpr bool mdq  = false;
};
template<class T>
struct Mpole<std::array<T, 8>>
{
    using value               = T;
    static constexpr bool mdq = false;
};
template<class T>
struct Mpole<std::array<T, 12>>
{
    using value               = T;
    static constexpr bool mdq = true;
};
//! the value type of a centre array element (T or Vec4<T>)
template<class C>
struct Center
{
    using value = C;
};
template<class T>
struct Center<std::array<T, 4>>
{
    using value = T;
};
template<class Tc, class Tm>
inline constexpr bool isF32 = std::is_same_v<Tc, float> && std::is_same_v<Tm, float>;
template<class Tc, class Tm>
inline constexpr bool isF64 = std::is_same_v<Tc, double> && std::is_same_v<Tm, double>;
template<class Tc, class Tm>
inline constexpr bool isMixed = std::is_same_v<Tc, double> && std::is_same_v<Tm, float>;
template<class>
inline constexpr bool alwaysFalse = false;
} // namespace detail

//! ryoanji::TreeBuilder (ryoanji/src/ryoanji/interface/treebuilder.cuh:34-125); the returned pointers stay valid
//! until the next update
template<class KeyType>
class TreeBuilder
{
    static_assert(std::is_same_v<KeyType, uint64_t>, "the B200 library builds 64-bit key trees");

public:
    explicit TreeBuilder(unsigned ncrit, Context& ctx = defaultContext())
        : ctx_(&ctx)
    {
        ryo_treebuilder_t* h = nullptr;
        check(ryo_treebuilder_create(ctx.get(), ncrit, &h), ctx.get());
        h_.reset(h);
    }

    //! sorts x, y, z in place along the SFC, builds the tree, returns the total node count
    template<class T>
    int update(T* x, T* y, T* z, size_t numBodies, const Box<T>& box, ryo_stream_t stream = nullptr)
    {
        static_assert(std::is_same_v<T, float> || std::is_same_v<T, double>, "float or double coordinates");
        int numNodes = 0;
        if constexpr (std::is_same_v<T, float>)
        {
            ryo_box_f32 b = box.abiF32();
            check(ryo_treebuilder_update_f32(h_.get(), x, y, z, numBodies, &b, &numNodes, stream), ctx_->get());
        }
        else
        {
            ryo_box_f64 b = box.abiF64();
            check(ryo_treebuilder_update_f64(h_.get(), x, y, z, numBodies, &b, &numNodes, stream), ctx_->get());
        }
        check(ryo_treebuilder_view(h_.get(), &view_), ctx_->get());
        return numNodes;
    }

    const LocalIndex* layout() const { return view_.layout; }
    const KeyType* nodeKeys() const { return view_.nodeKeys; }
    const TreeNodeIndex* childOffsets() const { return view_.childOffsets; }
    const TreeNodeIndex* leafToInternal() const { return view_.leafToInternal; }
    const TreeNodeIndex* internalToLeaf() const { return view_.internalToLeaf; }
    const TreeNodeIndex* levelRange() const { return view_.levelRange; } // host pointer, as in the reference
    TreeNodeIndex numLeafNodes() const { return view_.numLeafNodes; }
    unsigned maxTreeLevel() const { return view_.maxTreeLevel; }
    //! not in the reference: the SFC permutation applied to x, y, z by the last update
    const LocalIndex* order() const { return view_.order; }

private:
    struct Del
    {
        void operator()(ryo_treebuilder_t* t) const { ryo_treebuilder_destroy(t); }
    };
    Context* ctx_;
    std::unique_ptr<ryo_treebuilder_t, Del> h_;
    ryo_tree_view view_{};
};

//! cstone::computeSfcKeys for the GPU (cstone/include/cstone/sfc/sfc_gpu.h)
template<class T>
void computeSfcKeys(const T* x, const T* y, const T* z, uint64_t* keys, size_t numKeys, const Box<T>& box,
                    ryo_stream_t stream = nullptr)
{
    if constexpr (std::is_same_v<T, float>)
    {
        ryo_box_f32 b = box.abiF32();
        check(ryo_compute_sfc_keys_f32(x, y, z, keys, numKeys, &b, stream));
    }
    else
    {
        ryo_box_f64 b = box.abiF64();
        check(ryo_compute_sfc_keys_f64(x, y, z, keys, numKeys, &b, stream));
    }
}

//! cstone::computeFixedGroups (cstone/include/cstone/traversal/groups_gpu.cuh): groups[0..] hold the starts and
//! the final end; ceil((last - first) / groupSize) + 1 entries
inline void computeFixedGroups(LocalIndex first, LocalIndex last, unsigned groupSize, LocalIndex* groups,
                               ryo_stream_t stream = nullptr)
{
    check(ryo_compute_fixed_groups(first, last, groupSize, groups, stream));
}

//! cstone::sequence (cstone/include/cstone/primitives/primitives_gpu.h:92): input[i] = init + i
inline void sequence(LocalIndex* input, size_t numElements, LocalIndex init, ryo_stream_t stream = nullptr)
{
    check(ryo_sequence(input, numElements, init, stream));
}

//! cstone::sortByKeyTempStorage (primitives_gpu.h:118-120) for 64-bit keys and 32-bit values, in bytes
template<class KeyType, class ValueType>
uint64_t sortByKeyTempStorage(uint64_t numElements)
{
    static_assert(std::is_same_v<KeyType, uint64_t> && sizeof(ValueType) == 4, "64-bit keys, 32-bit values");
    return ryo_sort_by_key_temp_bytes(numElements);
}

/*! cstone::sortByKey (primitives_gpu.h:122-130): stable ascending sort of the keys [first, last), carrying values
 *  along; keyBuf and valueBuf hold last - first elements, tmp sortByKeyTempStorage bytes. Fewer than 2^32 keys. */
template<class ValueType>
void sortByKey(uint64_t* first, uint64_t* last, ValueType* values, uint64_t* keyBuf, ValueType* valueBuf, void* tmp,
               uint64_t tmpBytes, ryo_stream_t stream = nullptr)
{
    static_assert(sizeof(ValueType) == 4, "32-bit values");
    check(ryo_sort_by_key(first, reinterpret_cast<uint32_t*>(values), size_t(last - first), keyBuf,
                          reinterpret_cast<uint32_t*>(valueBuf), tmp, tmpBytes, stream));
}

/*! cstone::computeOctree / updateOctreeGpu run to their fixed point (cstone/include/cstone/tree/csarray.hpp:409-440,
 *  update_gpu.cuh:43-68) for sorted 64-bit keys: the cornerstone leaves (numLeaves + 1 keys) and counts of at most
 *  @p bucketSize keys per leaf, in one pass. Returns numLeaves; when it exceeds @p capacity nothing is written, and
 *  a second call with that capacity writes the arrays. */
inline TreeNodeIndex computeOctreeGpu(const uint64_t* sortedKeys, size_t numKeys, unsigned bucketSize,
                                      uint64_t* leaves, LocalIndex* counts, TreeNodeIndex capacity,
                                      Context& ctx = defaultContext(), ryo_stream_t stream = nullptr)
{
    int numLeaves = 0;
    ryo_status s =
        ryo_compute_octree(ctx.get(), sortedKeys, numKeys, bucketSize, leaves, counts, capacity, &numLeaves, stream);
    if (s != RYO_ERR_CAPACITY) check(s, ctx.get());
    return numLeaves;
}

//! cstone::OctreeView (cstone/include/cstone/tree/octree.hpp:235-256) for 64-bit keys: where buildOctreeGpu writes
//! the linked octree. levelRange is host memory and d_levelRange device memory (may be null), as in the reference.
template<class KeyType>
struct OctreeView
{
    TreeNodeIndex numLeafNodes;
    TreeNodeIndex numInternalNodes;
    TreeNodeIndex numNodes;
    TreeNodeIndex numParents;

    KeyType* prefixes;
    TreeNodeIndex* childOffsets;
    TreeNodeIndex* parents;
    TreeNodeIndex* levelRange;
    TreeNodeIndex* d_levelRange;
    TreeNodeIndex* internalToLeaf;
    TreeNodeIndex* leafToInternal;
    KeyType* leaves{nullptr};
};

//! cstone::buildOctreeGpu (cstone/include/cstone/tree/octree_gpu.h:36) from the cornerstone leaves
template<class KeyType>
void buildOctreeGpu(const KeyType* cstoneTree, OctreeView<KeyType> d, Context& ctx = defaultContext(),
                    ryo_stream_t stream = nullptr)
{
    static_assert(std::is_same_v<KeyType, uint64_t>, "the B200 library builds 64-bit key trees");
    check(ryo_build_octree(ctx.get(), cstoneTree, d.numLeafNodes, d.prefixes, d.childOffsets, d.parents, d.levelRange,
                           d.d_levelRange, d.internalToLeaf, d.leafToInternal, stream),
          ctx.get());
}

/*! cstone::computeLeafSourceCenterGpu (cstone/include/cstone/focus/source_center_gpu.h:65-80) for the type sets
 *  (Tc, Tm, Tf) = (float, float, float), (double, double, double), (double, float, double); @p centers holds 4
 *  values per node (Tf or Vec4<Tf> elements) */
template<class Tc, class Tm, class C>
void computeLeafSourceCenterGpu(const Tc* x, const Tc* y, const Tc* z, const Tm* m,
                                const TreeNodeIndex* leafToInternal, TreeNodeIndex numLeaves,
                                const LocalIndex* layout, C* centers, ryo_stream_t stream = nullptr)
{
    using Tf = typename detail::Center<C>::value;
    auto* c  = reinterpret_cast<Tf*>(centers);
    if constexpr (detail::isF32<Tc, Tm> && std::is_same_v<Tf, float>)
        check(ryo_compute_leaf_source_center_f32(x, y, z, m, leafToInternal, numLeaves, layout, c, stream));
    else if constexpr (detail::isF64<Tc, Tm> && std::is_same_v<Tf, double>)
        check(ryo_compute_leaf_source_center_f64(x, y, z, m, leafToInternal, numLeaves, layout, c, stream));
    else if constexpr (detail::isMixed<Tc, Tm> && std::is_same_v<Tf, double>)
        check(ryo_compute_leaf_source_center_mixed(x, y, z, m, leafToInternal, numLeaves, layout, c, stream));
    else
        static_assert(detail::alwaysFalse<C>, "not an instantiated type set");
}

//! cstone::upsweepCentersGpu; levelRange is a host pointer as in the reference
template<class C>
void upsweepCentersGpu(int numLevels, const TreeNodeIndex* levelRange, const TreeNodeIndex* childOffsets, C* centers,
                       ryo_stream_t stream = nullptr)
{
    using Tf = typename detail::Center<C>::value;
    auto* c  = reinterpret_cast<Tf*>(centers);
    if constexpr (std::is_same_v<Tf, float>) check(ryo_upsweep_centers_f32(numLevels, levelRange, childOffsets, c, stream));
    else check(ryo_upsweep_centers_f64(numLevels, levelRange, childOffsets, c, stream));
}

//! cstone::setMacGpu with the vector MAC (float or double centres and box)
template<class C, class T>
void setMacGpu(const uint64_t* prefixes, TreeNodeIndex numNodes, C* centers, float invTheta, const Box<T>& box,
               ryo_stream_t stream = nullptr)
{
    using Tf = typename detail::Center<C>::value;
    static_assert(std::is_same_v<Tf, T>, "centres and box of one type");
    auto* c = reinterpret_cast<Tf*>(centers);
    if constexpr (std::is_same_v<T, float>)
    {
        ryo_box_f32 b = box.abiF32();
        check(ryo_set_mac_f32(prefixes, numNodes, c, invTheta, &b, stream));
    }
    else
    {
        ryo_box_f64 b = box.abiF64();
        check(ryo_set_mac_f64(prefixes, numNodes, c, invTheta, &b, stream));
    }
}

/*! ryoanji::computeLeafMultipoles (upsweep_gpu.h:24-31) for the type sets (Tc, Tm, Tf, MType) = (float, float,
 *  float, M<float>), (double, double, double, M<double>), (double, float, double, M<float>), M = CartesianQuadrupole
 *  or CartesianMDQpole; a plain value pointer means CartesianQuadrupole */
template<class Tc, class Tm, class C, class M>
void computeLeafMultipoles(const Tc* x, const Tc* y, const Tc* z, const Tm* m, const TreeNodeIndex* leafToInternal,
                           TreeNodeIndex numLeaves, const LocalIndex* layout, const C* centers, M* multipoles,
                           ryo_stream_t stream = nullptr)
{
    using Tf  = typename detail::Center<C>::value;
    using Tmp = typename detail::Mpole<M>::value;
    constexpr bool mdq = detail::Mpole<M>::mdq;
    const Tf* c        = reinterpret_cast<const Tf*>(centers);
    Tmp* q             = reinterpret_cast<Tmp*>(multipoles);
    if constexpr (detail::isF32<Tc, Tm> && std::is_same_v<Tf, float> && std::is_same_v<Tmp, float>)
        check(mdq ? ryo_compute_leaf_multipoles_mdq_f32(x, y, z, m, leafToInternal, numLeaves, layout, c, q, stream)
                  : ryo_compute_leaf_multipoles_f32(x, y, z, m, leafToInternal, numLeaves, layout, c, q, stream));
    else if constexpr (detail::isF64<Tc, Tm> && std::is_same_v<Tf, double> && std::is_same_v<Tmp, double>)
        check(mdq ? ryo_compute_leaf_multipoles_mdq_f64(x, y, z, m, leafToInternal, numLeaves, layout, c, q, stream)
                  : ryo_compute_leaf_multipoles_f64(x, y, z, m, leafToInternal, numLeaves, layout, c, q, stream));
    else if constexpr (detail::isMixed<Tc, Tm> && std::is_same_v<Tf, double> && std::is_same_v<Tmp, float>)
        check(mdq ? ryo_compute_leaf_multipoles_mdq_mixed(x, y, z, m, leafToInternal, numLeaves, layout, c, q, stream)
                  : ryo_compute_leaf_multipoles_mixed(x, y, z, m, leafToInternal, numLeaves, layout, c, q, stream));
    else
        static_assert(detail::alwaysFalse<M>, "not an instantiated type set");
}

//! ryoanji::upsweepMultipoles (upsweep_gpu.h:39-41) for cells [firstCell, lastCell) of one level
template<class C, class M>
void upsweepMultipoles(TreeNodeIndex firstCell, TreeNodeIndex lastCell, const TreeNodeIndex* childOffsets,
                       const C* centers, M* multipoles, ryo_stream_t stream = nullptr)
{
    using Tf  = typename detail::Center<C>::value;
    using Tmp = typename detail::Mpole<M>::value;
    constexpr bool mdq = detail::Mpole<M>::mdq;
    const Tf* c        = reinterpret_cast<const Tf*>(centers);
    Tmp* q             = reinterpret_cast<Tmp*>(multipoles);
    if constexpr (std::is_same_v<Tf, float> && std::is_same_v<Tmp, float>)
        check(mdq ? ryo_upsweep_multipoles_mdq_f32(firstCell, lastCell, childOffsets, c, q, stream)
                  : ryo_upsweep_multipoles_f32(firstCell, lastCell, childOffsets, c, q, stream));
    else if constexpr (std::is_same_v<Tf, double> && std::is_same_v<Tmp, double>)
        check(mdq ? ryo_upsweep_multipoles_mdq_f64(firstCell, lastCell, childOffsets, c, q, stream)
                  : ryo_upsweep_multipoles_f64(firstCell, lastCell, childOffsets, c, q, stream));
    else if constexpr (std::is_same_v<Tf, double> && std::is_same_v<Tmp, float>)
        check(mdq ? ryo_upsweep_multipoles_mdq_mixed(firstCell, lastCell, childOffsets, c, q, stream)
                  : ryo_upsweep_multipoles_mixed(firstCell, lastCell, childOffsets, c, q, stream));
    else
        static_assert(detail::alwaysFalse<M>, "not an instantiated type set");
}

/*! cstone::computeGroupSplits (groups_gpu.cu:60-151): spatial target groups of SFC-sorted bodies [first, last) into
 *  @p groups (capacity entries, at least last - first + 1); returns the group count. extentRatio < 0: the default. */
inline LocalIndex computeGroupSplits(LocalIndex first, LocalIndex last, const float* x, const float* y,
                                     const float* z, const float* h, const uint64_t* leaves, TreeNodeIndex numLeaves,
                                     const LocalIndex* layout, const Box<float>& box, unsigned groupSize,
                                     float tolFactor, LocalIndex* groups, LocalIndex capacity,
                                     float extentRatio = -1.f, Context& ctx = defaultContext(),
                                     ryo_stream_t stream = nullptr)
{
    ryo_box_f32 b  = box.abiF32();
    LocalIndex num = 0;
    check(ryo_compute_group_splits_f32(ctx.get(), first, last, x, y, z, h, leaves, numLeaves, layout, &b, groupSize,
                                       tolFactor, extentRatio, groups, capacity, &num, stream),
          ctx.get());
    return num;
}

inline int bhMaxTargetSize() { return ryo_bh_max_target_size(); }
inline LocalIndex stackSize(LocalIndex numGroups) { return ryo_stack_size(numGroups); }

/*! ryoanji::traverse (traversal_gpu.h:51-56) for the instantiated type sets (traversal_gpu.cu:635-641): (Tc, Th,
 *  Tm, Ta, Tf) = all float, all double, or (double, float, float, float, double); MType = CartesianQuadrupole or
 *  CartesianMDQpole of float (double in the all-double set), or a plain value pointer for CartesianQuadrupole.
 *  Accumulates into p (may be null), ax, ay, az and returns the total potential 0.5 G sum m phi. */
template<class Tc, class Th, class Tm, class Ta, class C, class M>
double traverse(GroupView grp, int initNodeIdx, const Tc* xt, const Tc* yt, const Tc* zt, const Tm* mt, const Th* ht,
                const Tc* xs, const Tc* ys, const Tc* zs, const Tm* ms, const Th* hs,
                const TreeNodeIndex* childOffsets, const TreeNodeIndex* internalToLeaf, const LocalIndex* layout,
                const C* sourceCenter, const M* multipoles, Tc G, int numShells, Vec3<Tc> boxL, Ta* p, Ta* ax, Ta* ay,
                Ta* az, int* /* gmPool: unused */, Context& ctx = defaultContext(), ryo_stream_t stream = nullptr)
{
    using Tf  = typename detail::Center<C>::value;
    using Tmp = typename detail::Mpole<M>::value;
    ryo_group_view g = grp.abi();
    double total     = 0;
    ryo_traverse_options opt{};
    opt.multipole = detail::Mpole<M>::mdq ? RYO_MULTIPOLE_MDQ : RYO_MULTIPOLE_QUADRUPOLE;
    const Tf* c   = reinterpret_cast<const Tf*>(sourceCenter);
    const Tmp* q  = reinterpret_cast<const Tmp*>(multipoles);
    Tc L[3]       = {boxL.x, boxL.y, boxL.z};
    constexpr bool f32 = detail::isF32<Tc, Tm> && std::is_same_v<Th, float> && std::is_same_v<Ta, float> &&
                         std::is_same_v<Tf, float> && std::is_same_v<Tmp, float>;
    constexpr bool f64 = detail::isF64<Tc, Tm> && std::is_same_v<Th, double> && std::is_same_v<Ta, double> &&
                         std::is_same_v<Tf, double> && std::is_same_v<Tmp, double>;
    constexpr bool mixed = detail::isMixed<Tc, Tm> && std::is_same_v<Th, float> && std::is_same_v<Ta, float> &&
                           std::is_same_v<Tf, double> && std::is_same_v<Tmp, float>;
    if constexpr (f32)
        check(ryo_traverse_ex_f32(ctx.get(), &g, initNodeIdx, xt, yt, zt, mt, ht, xs, ys, zs, ms, hs, childOffsets,
                                  internalToLeaf, layout, c, q, G, numShells, L, p, ax, ay, az, &total, &opt, stream),
              ctx.get());
    else if constexpr (f64)
        check(ryo_traverse_f64(ctx.get(), &g, initNodeIdx, xt, yt, zt, mt, ht, xs, ys, zs, ms, hs, childOffsets,
                               internalToLeaf, layout, c, q, G, numShells, L, p, ax, ay, az, &total, &opt, stream),
              ctx.get());
    else if constexpr (mixed)
        check(ryo_traverse_mixed(ctx.get(), &g, initNodeIdx, xt, yt, zt, mt, ht, xs, ys, zs, ms, hs, childOffsets,
                                 internalToLeaf, layout, c, q, G, numShells, L, p, ax, ay, az, &total, &opt, stream),
              ctx.get());
    else
        static_assert(detail::alwaysFalse<M>, "not an instantiated type set");
    return total;
}

/*! MultipoleHolder::compute with separate targets (multipole_holder.cuh:64-77) after a ryo_solve_f32 on @p ctx:
 *  overwrites p (may be null), ax, ay, az in the targets' order */
inline void computeTargets(const float* xt, const float* yt, const float* zt, const float* mt, const float* ht,
                           size_t numTargets, float* p, float* ax, float* ay, float* az,
                           Context& ctx = defaultContext(), ryo_stream_t stream = nullptr)
{
    check(ryo_solve_targets_f32(ctx.get(), xt, yt, zt, mt, ht, numTargets, p, ax, ay, az, nullptr, stream),
          ctx.get());
}

//! ryoanji::readBhStats (traversal_gpu.h:64-65): sumP2P, maxP2P, sumM2P, maxM2P, maxStack
inline std::array<uint64_t, 5> readBhStats(Context& ctx = defaultContext())
{
    std::array<uint64_t, 5> s{};
    check(ryo_read_bh_stats(ctx.get(), s.data()), ctx.get());
    return s;
}

inline uint64_t readTraversalRetries(Context& ctx = defaultContext()) { return ryo_read_traversal_retries(ctx.get()); }

//! ryoanji::EwaldSettings (ryoanji/src/ryoanji/nbody/ewald.h:23-31) with the reference defaults
inline ryo_ewald_settings defaultEwaldSettings()
{
    ryo_ewald_settings e{};
    e.numReplicaShells     = 1;
    e.lCut                 = 2.6;
    e.hCut                 = 2.8;
    e.alpha_scale          = 2.0;
    e.small_R_scale_factor = 3.0e-3;
    return e;
}

/*! ryoanji::computeGravityEwaldGpu (interface/ewald.cuh:24-27) for the instantiated sets (ewald.cu:101-110): float
 *  coordinates, masses and outputs with float Mroot; double everything (Mroot double or float); double coordinates
 *  with float masses and outputs and float Mroot. Mroot is the root's 8 multipole values (host). Adds the Ewald
 *  correction to ugrav, ax, ay, az and to *ugravTot. */
template<class Tc, class Tr, class Tm, class Ta>
void computeGravityEwaldGpu(const Vec3<Tc>& rootCenter, const Tr* Mroot, GroupView grp, const Tc* x, const Tc* y,
                            const Tc* z, const Tm* m, const Box<Tc>& box, float G, Ta* ugrav, Ta* ax, Ta* ay, Ta* az,
                            double* ugravTot, const ryo_ewald_settings& settings, Context& ctx = defaultContext(),
                            ryo_stream_t stream = nullptr)
{
    ryo_group_view g = grp.abi();
    Tc rc[3]         = {rootCenter.x, rootCenter.y, rootCenter.z};
    if constexpr (detail::isF32<Tc, Tm> && std::is_same_v<Ta, float> && std::is_same_v<Tr, float>)
    {
        ryo_box_f32 b = box.abiF32();
        check(ryo_compute_gravity_ewald_f32(ctx.get(), rc, Mroot, &g, x, y, z, m, &b, G, ugrav, ax, ay, az, ugravTot,
                                            &settings, stream),
              ctx.get());
    }
    else if constexpr (detail::isF64<Tc, Tm> && std::is_same_v<Ta, double>)
    {
        ryo_box_f64 b = box.abiF64();
        double mr[8];
        for (int i = 0; i < 8; ++i)
            mr[i] = double(Mroot[i]);
        check(ryo_compute_gravity_ewald_f64(ctx.get(), rc, mr, &g, x, y, z, m, &b, G, ugrav, ax, ay, az, ugravTot,
                                            &settings, stream),
              ctx.get());
    }
    else if constexpr (detail::isMixed<Tc, Tm> && std::is_same_v<Ta, float> && std::is_same_v<Tr, float>)
    {
        ryo_box_f64 b = box.abiF64();
        check(ryo_compute_gravity_ewald_mixed(ctx.get(), rc, Mroot, &g, x, y, z, m, &b, G, ugrav, ax, ay, az,
                                              ugravTot, &settings, stream),
              ctx.get());
    }
    else
        static_assert(detail::alwaysFalse<Tr>, "not an instantiated type set");
}

//! ryoanji::directSum (interface/multipole_holder.cuh:91-93): exact sums for targets [first, last)
inline void directSum(size_t first, size_t last, size_t numBodies, Vec3<float> boxL, int numShells, const float* x,
                      const float* y, const float* z, const float* m, const float* h, float* p, float* ax, float* ay,
                      float* az, ryo_stream_t stream = nullptr)
{
    float L[3] = {boxL.x, boxL.y, boxL.z};
    check(ryo_direct_sum_f32(first, last, numBodies, L, numShells, x, y, z, m, h, p, ax, ay, az, stream));
}

} // namespace ryo

#endif
