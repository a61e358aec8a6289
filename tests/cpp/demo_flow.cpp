// The reference demo's gravity flow (ryoanji/test/demo.cu:82-104, :171-190, :205-226) written in the reference's
// spellings, compiled against ryoanji_b200/compat.hpp instead of the reference's headers. Reads n float32 x, y, z
// from the file argv[1], runs build, upsweep, fixed groups and traverse for the three type sets (f32, f64, mixed)
// and prints one JSON line per set: readBhStats, the total potential and the sums of the accelerations, and writes
// ax, ay, az (in the sorted order, as float64) to argv[2].<set>.bin.
#include "ryoanji_b200/compat.hpp"

#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <vector>

using namespace ryoanji;

template<class T>
T* upload(const std::vector<T>& h)
{
    T* d = nullptr;
    cudaMalloc(&d, h.size() * sizeof(T));
    cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
    return d;
}

template<class Tc, class Th, class Tm, class Ta, class Tf, class MType>
int run(const char* name, const std::vector<float>& in, size_t n, const std::string& outPrefix)
{
    std::vector<Tc> hx(n), hy(n), hz(n);
    for (size_t i = 0; i < n; ++i)
    {
        hx[i] = in[i];
        hy[i] = in[n + i];
        hz[i] = in[2 * n + i];
    }
    Tc* x  = upload(hx);
    Tc* y  = upload(hy);
    Tc* z  = upload(hz);
    Tm* m  = upload(std::vector<Tm>(n, Tm(1.0 / n)));
    Th* h  = upload(std::vector<Th>(n, Th(0.005)));
    Ta* p  = upload(std::vector<Ta>(n, Ta(0)));
    Ta* ax = upload(std::vector<Ta>(n, Ta(0)));
    Ta* ay = upload(std::vector<Ta>(n, Ta(0)));
    Ta* az = upload(std::vector<Ta>(n, Ta(0)));
    float theta = 0.5f;
    Tc G        = 1;

    cstone::Box<Tc> box(-1, 1);
    TreeBuilder<uint64_t> treeBuilder(64);
    int numSources = treeBuilder.update(x, y, z, n, box);

    Vec4<Tf>* sourceCenter = nullptr;
    MType* multipole       = nullptr;
    cudaMalloc(&sourceCenter, sizeof(Vec4<Tf>) * numSources);
    cudaMalloc(&multipole, sizeof(MType) * numSources);
    const TreeNodeIndex* levelRange = treeBuilder.levelRange();
    cstone::computeLeafSourceCenterGpu(cstone::execution::gpuDefaultStream, x, y, z, m, treeBuilder.leafToInternal(),
                                       treeBuilder.numLeafNodes(), treeBuilder.layout(), sourceCenter);
    cstone::upsweepCentersGpu(cstone::execution::gpuDefaultStream, cstone::maxTreeLevel<uint64_t>{}, levelRange,
                              treeBuilder.childOffsets(), sourceCenter);
    computeLeafMultipoles(x, y, z, m, treeBuilder.leafToInternal(), treeBuilder.numLeafNodes(), treeBuilder.layout(),
                          sourceCenter, multipole);
    for (int level = treeBuilder.maxTreeLevel() - 1; level >= 1; level--)
        upsweepMultipoles(levelRange[level], levelRange[level + 1], treeBuilder.childOffsets(), sourceCenter,
                          multipole);
    cstone::setMacGpu(cstone::execution::gpuDefaultStream, treeBuilder.nodeKeys(), numSources, sourceCenter,
                      1.f / theta, box);

    cstone::GroupData<cstone::execution::Gpu> groups;
    cstone::computeFixedGroups(cstone::execution::gpuDefaultStream, 0, n, bhMaxTargetSize(), groups);
    int* globalPool = nullptr; // stackSize() is 0: the traversal keeps its stacks in shared memory
    double totalPotential = traverse(groups.view(), 1, x, y, z, m, h, x, y, z, m, h, treeBuilder.childOffsets(),
                                     treeBuilder.internalToLeaf(), treeBuilder.layout(), sourceCenter, multipole, G,
                                     0, {box.lx(), box.ly(), box.lz()}, p, ax, ay, az, globalPool);
    auto stats = readBhStats();

    std::vector<Ta> ha(n), hb(n), hc(n);
    cudaMemcpy(ha.data(), ax, n * sizeof(Ta), cudaMemcpyDeviceToHost);
    cudaMemcpy(hb.data(), ay, n * sizeof(Ta), cudaMemcpyDeviceToHost);
    cudaMemcpy(hc.data(), az, n * sizeof(Ta), cudaMemcpyDeviceToHost);
    std::vector<double> acc(3 * n);
    for (size_t i = 0; i < n; ++i)
    {
        acc[i]         = ha[i];
        acc[n + i]     = hb[i];
        acc[2 * n + i] = hc[i];
    }
    std::string path = outPrefix + "." + name + ".bin";
    FILE* f          = std::fopen(path.c_str(), "wb");
    std::fwrite(acc.data(), sizeof(double), acc.size(), f);
    std::fclose(f);
    std::printf("{\"set\": \"%s\", \"nodes\": %d, \"stats\": [%llu, %llu, %llu, %llu], \"potential\": %.17g}\n", name,
                numSources, (unsigned long long)stats[0], (unsigned long long)stats[1],
                (unsigned long long)stats[2], (unsigned long long)stats[3], totalPotential);
    for (void* ptr : {(void*)x, (void*)y, (void*)z, (void*)m, (void*)h, (void*)p, (void*)ax, (void*)ay, (void*)az,
                      (void*)sourceCenter, (void*)multipole})
        cudaFree(ptr);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int main(int argc, char** argv)
{
    if (argc < 3) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    std::vector<float> in;
    float v;
    while (std::fread(&v, sizeof(float), 1, f) == 1)
        in.push_back(v);
    std::fclose(f);
    size_t n = in.size() / 3;
    int rc   = 0;
    try
    {
        rc |= run<float, float, float, float, float, CartesianQuadrupole<float>>("f32", in, n, argv[2]);
        rc |= run<double, double, double, double, double, CartesianQuadrupole<double>>("f64", in, n, argv[2]);
        rc |= run<double, float, float, float, double, CartesianQuadrupole<float>>("mixed", in, n, argv[2]);
    }
    catch (const ryo::Error& e)
    {
        std::fprintf(stderr, "ryo::Error %d: %s\n", int(e.status), e.what());
        return 3;
    }
    return rc;
}
