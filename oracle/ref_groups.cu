/*
 * Test infrastructure only: a C-ABI wrapper around the reference's own GPU target grouping
 * (cstone::computeGroupSplits, cstone/include/cstone/traversal/groups_gpu.cu:60-151), compiled from the reference
 * sources in place into oracle/_ref (never committed). Used by the GPU tests to pin the grouping restated in
 * ryo_oracle.cpp and implemented in ryoanji_b200/csrc/groups.cu. Device pointers in, host results out.
 */
#include <cstdint>
#include <vector>

#include "cstone/cuda/device_vector.h"
#include "cstone/traversal/groups_gpu.h"

extern "C" long ref_group_splits_f32(uint32_t first, uint32_t last, const float* x, const float* y, const float* z,
                                     const float* h, const uint64_t* leaves, int numLeaves, const uint32_t* layout,
                                     const float* box6, int groupSize, float tolFactor, uint32_t* groupsHost,
                                     long capacity)
{
    cstone::Box<float> box(box6[0], box6[1], box6[2], box6[3], box6[4], box6[5]);
    cstone::DeviceVector<cstone::LocalIndex> temp, groups;
    cstone::computeGroupSplits(cstone::execution::gpuDefaultStream, first, last, x, y, z, h, leaves, numLeaves,
                               layout, box, unsigned(groupSize), tolFactor, temp, groups);
    std::vector<cstone::LocalIndex> g(groups.size());
    cudaMemcpy(g.data(), groups.data(), sizeof(cstone::LocalIndex) * g.size(), cudaMemcpyDeviceToHost);
    long n = long(g.size()) - 1;
    if (n + 1 <= capacity)
        for (long i = 0; i <= n; ++i)
            groupsHost[i] = g[size_t(i)];
    return n;
}
