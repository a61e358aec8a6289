/*
 * ryoanji-b200 — the reference's namespaces and call signatures over ryoanji_b200/ryoanji.hpp (header only, C++17).
 *
 * A caller of the reference's single-GPU gravity path (the flow of ryoanji/test/demo.cu:82-104, :171-190, :205-226)
 * replaces its includes of cstone/ and ryoanji/ headers by this one and keeps its code: cstone::Box,
 * cstone::execution::Gpu / gpuDefaultStream / gpuStream, cstone::GroupData / GroupView / computeFixedGroups,
 * cstone::computeSfcKeys / sfcKindPointer / sequence / sortByKey, cstone::computeLeafSourceCenterGpu /
 * upsweepCentersGpu / setMacGpu / maxTreeLevel, and ryoanji::TreeBuilder / computeLeafMultipoles /
 * upsweepMultipoles / traverse / readBhStats / stackSize / bhMaxTargetSize / computeGravityEwaldGpu / directSum /
 * EwaldSettings / Vec3 / Vec4 / CartesianQuadrupole / CartesianMDQpole.
 *
 * Every call runs on the stream of its execution::Gpu argument (the reference's functions without one run on the
 * default stream, as there) and on the calling thread's default ryo::Context. GroupData owns its device array
 * (cudaMalloc / cudaFree), so this header needs the CUDA runtime, as the reference's headers do.
 */
#ifndef RYOANJI_B200_COMPAT_HPP
#define RYOANJI_B200_COMPAT_HPP

#include <cuda_runtime_api.h>

#include <utility>

#include "ryoanji.hpp"

namespace cstone
{

using LocalIndex    = ryo::LocalIndex;
using TreeNodeIndex = ryo::TreeNodeIndex;
using BoundaryType  = ryo::BoundaryType;
template<class T>
using Box = ryo::Box<T>;
template<class T>
using Vec3 = ryo::Vec3<T>;
template<class T>
using Vec4 = ryo::Vec4<T>;
template<class T>
using SourceCenterType = ryo::Vec4<T>;
using GroupView = ryo::GroupView;

namespace execution
{
//! cstone::execution::Gpu (cstone/include/cstone/execution.hpp:28-54): a stream
struct Gpu
{
    operator cudaStream_t() const { return stream; }
    cudaStream_t stream;
};
constexpr inline Gpu gpuStream(cudaStream_t s) noexcept { return Gpu{s}; }
constexpr inline Gpu gpuDefaultStream = Gpu{nullptr};
} // namespace execution

//! cstone::maxTreeLevel (cstone/include/cstone/tree/definitions.h:50-63) for 64-bit keys
template<class KeyType>
struct maxTreeLevel : std::integral_constant<unsigned, 21>
{
    static_assert(std::is_same_v<KeyType, uint64_t> || std::is_same_v<KeyType, unsigned long long>,
                  "64-bit keys");
};

//! cstone::sfcKindPointer (cstone/include/cstone/sfc/sfc.hpp:50-60): the keys are plain 64-bit Hilbert keys here
template<class KeyType>
KeyType* sfcKindPointer(KeyType* p)
{
    return p;
}
template<class KeyType>
const KeyType* sfcKindPointer(const KeyType* p)
{
    return p;
}

template<class T>
void computeSfcKeys(execution::Gpu exec, const T* x, const T* y, const T* z, uint64_t* keys, size_t numKeys,
                    const Box<T>& box)
{
    ryo::computeSfcKeys(x, y, z, keys, numKeys, box, exec.stream);
}

inline void sequence(execution::Gpu exec, LocalIndex* input, size_t numElements, LocalIndex init)
{
    ryo::sequence(input, numElements, init, exec.stream);
}

template<class KeyType, class ValueType>
uint64_t sortByKeyTempStorage(uint64_t numElements)
{
    return ryo::sortByKeyTempStorage<KeyType, ValueType>(numElements);
}

template<class ValueType>
void sortByKey(execution::Gpu exec, uint64_t* first, uint64_t* last, ValueType* values, uint64_t* keyBuf,
               ValueType* valueBuf, void* tmp, uint64_t tmpBytes)
{
    ryo::sortByKey(first, last, values, keyBuf, valueBuf, tmp, tmpBytes, exec.stream);
}

/*! cstone::GroupData<execution::Gpu> (cstone/include/cstone/traversal/groups.hpp:37-66): group boundaries in one
 *  device array, groupEnd = groupStart + 1 as in the reference's fixed groups */
template<class Exec>
class GroupData
{
    static_assert(std::is_same_v<Exec, execution::Gpu>, "device groups");

public:
    GroupData() = default;
    GroupData(const GroupData&) = delete;
    GroupData& operator=(const GroupData&) = delete;
    ~GroupData() { release(); }

    GroupView view() const { return {firstBody, lastBody, numGroups, groupStart, groupEnd}; }

    //! (re)size the device array to @p n boundaries
    LocalIndex* reserve(size_t n)
    {
        if (n > capacity_)
        {
            release();
            void* p = nullptr;
            if (cudaMalloc(&p, n * sizeof(LocalIndex)) != cudaSuccess)
                throw ryo::Error(RYO_ERR_OOM, "GroupData: cudaMalloc failed");
            data_     = static_cast<LocalIndex*>(p);
            capacity_ = n;
        }
        return data_;
    }

    LocalIndex firstBody = 0, lastBody = 0, numGroups = 0;
    LocalIndex* groupStart = nullptr;
    LocalIndex* groupEnd   = nullptr;

private:
    void release()
    {
        if (data_) cudaFree(data_);
        data_     = nullptr;
        capacity_ = 0;
    }
    LocalIndex* data_ = nullptr;
    size_t capacity_  = 0;
};

//! cstone::computeFixedGroups (cstone/include/cstone/traversal/groups_gpu.h:33-34)
inline void computeFixedGroups(execution::Gpu exec, LocalIndex first, LocalIndex last, unsigned groupSize,
                               GroupData<execution::Gpu>& groups)
{
    LocalIndex n     = last > first ? (last - first + groupSize - 1) / groupSize : 0;
    LocalIndex* data = groups.reserve(size_t(n) + 1);
    ryo::computeFixedGroups(first, last, groupSize, data, exec.stream);
    groups.firstBody  = first;
    groups.lastBody   = last;
    groups.numGroups  = n;
    groups.groupStart = data;
    groups.groupEnd   = data + 1;
}

template<class Tc, class Tm, class Tf>
void computeLeafSourceCenterGpu(execution::Gpu exec, const Tc* x, const Tc* y, const Tc* z, const Tm* m,
                                const TreeNodeIndex* leafToInternal, TreeNodeIndex numLeaves,
                                const LocalIndex* layout, Vec4<Tf>* centers)
{
    ryo::computeLeafSourceCenterGpu(x, y, z, m, leafToInternal, numLeaves, layout, centers, exec.stream);
}

template<class T>
void upsweepCentersGpu(execution::Gpu exec, int numLevels, const TreeNodeIndex* levelRange,
                       const TreeNodeIndex* childOffsets, Vec4<T>* centers)
{
    ryo::upsweepCentersGpu(numLevels, levelRange, childOffsets, centers, exec.stream);
}

template<class KeyType, class T>
void setMacGpu(execution::Gpu exec, const KeyType* prefixes, TreeNodeIndex numNodes, Vec4<T>* centers,
               float invTheta, const Box<T>& box)
{
    ryo::setMacGpu(reinterpret_cast<const uint64_t*>(prefixes), numNodes, centers, invTheta, box, exec.stream);
}

} // namespace cstone

namespace ryoanji
{

using cstone::LocalIndex;
using cstone::TreeNodeIndex;
template<class T>
using Vec3 = ryo::Vec3<T>;
template<class T>
using Vec4 = ryo::Vec4<T>;
template<class T>
using CartesianQuadrupole = ryo::CartesianQuadrupole<T>;
template<class T>
using CartesianMDQpole = ryo::CartesianMDQpole<T>;
template<class KeyType>
using TreeBuilder = ryo::TreeBuilder<KeyType>;

//! ryoanji::EwaldSettings (ryoanji/src/ryoanji/nbody/ewald.h:23-31), the reference's defaults
struct EwaldSettings
{
    int numReplicaShells        = 1;
    double lCut                 = 2.6;
    double hCut                 = 2.8;
    double alpha_scale          = 2.0;
    double small_R_scale_factor = 3.0e-3;
};

template<class Tc, class Tm, class Tf, class MType>
void computeLeafMultipoles(const Tc* x, const Tc* y, const Tc* z, const Tm* m, const TreeNodeIndex* leafToInternal,
                           TreeNodeIndex numLeaves, const LocalIndex* layout, const Vec4<Tf>* centers,
                           MType* multipoles)
{
    ryo::computeLeafMultipoles(x, y, z, m, leafToInternal, numLeaves, layout, centers, multipoles);
}

template<class T, class MType>
void upsweepMultipoles(TreeNodeIndex firstCell, TreeNodeIndex lastCell, const TreeNodeIndex* childOffsets,
                       const Vec4<T>* centers, MType* multipoles)
{
    ryo::upsweepMultipoles(firstCell, lastCell, childOffsets, centers, multipoles);
}

template<class Tc, class Th, class Tm, class Ta, class Tf, class MType>
double traverse(cstone::GroupView grp, int initNodeIdx, const Tc* xt, const Tc* yt, const Tc* zt, const Tm* mt,
                const Th* ht, const Tc* xs, const Tc* ys, const Tc* zs, const Tm* ms, const Th* hs,
                const TreeNodeIndex* childOffsets, const TreeNodeIndex* internalToLeaf, const LocalIndex* layout,
                const Vec4<Tf>* sourceCenter, const MType* multipoles, Tc G, int numShells, Vec3<Tc> boxL, Ta* p,
                Ta* ax, Ta* ay, Ta* az, int* gmPool)
{
    return ryo::traverse(grp, initNodeIdx, xt, yt, zt, mt, ht, xs, ys, zs, ms, hs, childOffsets, internalToLeaf,
                         layout, sourceCenter, multipoles, G, numShells, boxL, p, ax, ay, az, gmPool);
}

inline int bhMaxTargetSize() { return ryo::bhMaxTargetSize(); }
inline LocalIndex stackSize(LocalIndex numGroups) { return ryo::stackSize(numGroups); }
inline std::array<uint64_t, 5> readBhStats() { return ryo::readBhStats(); }
inline uint64_t readTraversalRetries() { return ryo::readTraversalRetries(); }

/*! ryoanji::computeGravityEwaldGpu (ryoanji/src/ryoanji/interface/ewald.cuh:24-27) for the reference's instantiated
 *  sets (ewald.cu:101-110) */
template<class MType, class Tc, class Ta, class Tm, class Tu>
void computeGravityEwaldGpu(const Vec3<Tc>& rootCenter, const MType& Mroot, cstone::GroupView grp, const Tc* x,
                            const Tc* y, const Tc* z, const Tm* m, const cstone::Box<Tc>& box, float G, Ta* ugrav,
                            Ta* ax, Ta* ay, Ta* az, Tu* ugravTot, EwaldSettings settings)
{
    ryo_ewald_settings s{settings.numReplicaShells, settings.lCut, settings.hCut, settings.alpha_scale,
                         settings.small_R_scale_factor};
    double total = 0;
    ryo::computeGravityEwaldGpu(rootCenter, Mroot.data(), grp, x, y, z, m, box, G, ugrav, ax, ay, az, &total, s);
    *ugravTot += Tu(total);
}

template<class T>
void directSum(size_t first, size_t last, size_t numBodies, Vec3<T> boxL, int numShells, const T* x, const T* y,
               const T* z, const T* m, const T* h, T* p, T* ax, T* ay, T* az)
{
    static_assert(std::is_same_v<T, float>, "the float direct sum; ryo_direct_sum_f64 for double");
    ryo::directSum(first, last, numBodies, boxL, numShells, x, y, z, m, h, p, ax, ay, az);
}

} // namespace ryoanji

#endif
