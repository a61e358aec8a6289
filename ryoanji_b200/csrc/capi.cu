/*
 * ryoanji-b200: the C ABI (include/ryoanji_b200.h) over the kernels.
 *
 * Every entry point catches CUDA failures and turns them into a ryo_status with a message (the reference exits
 * the process instead, cstone/include/cstone/cuda/errorcheck.cuh:15-27). Scratch memory is owned by the context
 * (or the TreeBuilder) and grows on demand; nothing is kept in global device symbols, so contexts are independent.
 * The one exception is ryo_sort_by_key_static, whose scratch is a fixed device array shared by all its callers.
 */
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <stdexcept>

#include "internal.hpp"

using namespace ryo;

namespace
{
thread_local std::string tlsError;

struct ApiError
{
    ryo_status status;
    std::string what;
};

ryo_status fromCuda(const CudaError& e, std::string& msg)
{
    msg = std::string(e.what) + ": " + cudaGetErrorString(e.err);
    if (e.err == cudaErrorMemoryAllocation) return RYO_ERR_OOM;
    if (e.err == cudaErrorInvalidValue) return RYO_ERR_BAD_ARG;
    if (e.err == cudaErrorNoDevice || e.err == cudaErrorInvalidDevice) return RYO_ERR_NO_DEVICE;
    return RYO_ERR_CUDA;
}

template<class F>
ryo_status guarded(std::string& msg, F&& f)
{
    try
    {
        f();
        return RYO_OK;
    }
    catch (const CudaError& e)
    {
        return fromCuda(e, msg);
    }
    catch (const ApiError& e)
    {
        msg = e.what;
        return e.status;
    }
    catch (const std::bad_alloc&)
    {
        msg = "host allocation failed";
        return RYO_ERR_OOM;
    }
    catch (const std::exception& e)
    {
        // no exception may cross the C ABI: anything else becomes a status too
        msg = std::string("internal error: ") + e.what();
        return RYO_ERR_INTERNAL;
    }
    catch (...)
    {
        msg = "internal error";
        return RYO_ERR_INTERNAL;
    }
}

//! guarded, with the context's device current for the call
template<class F>
ryo_status guardedCtx(ryo_ctx* ctx, F&& f)
{
    DeviceScope device(ctx->device);
    return guarded(ctx->lastError, std::forward<F>(f));
}

#define REQUIRE(cond, msg)                                                                                             \
    do                                                                                                                 \
    {                                                                                                                  \
        if (!(cond)) throw ApiError{RYO_ERR_BAD_ARG, msg};                                                             \
    } while (0)

//! refuses the Ewald settings the reference refuses (ewaldSettingsError)
void checkEwald(const ryo_ewald_settings* e)
{
    REQUIRE(e, "ewald: null settings");
    if (const char* why = ewaldSettingsError(*e)) throw ApiError{RYO_ERR_BAD_ARG, why};
}

DevBox<float> boxOf(const ryo_box_f32* b)
{
    int periodic = b->boundary[0] == RYO_BOUNDARY_PERIODIC && b->boundary[1] == RYO_BOUNDARY_PERIODIC &&
                   b->boundary[2] == RYO_BOUNDARY_PERIODIC;
    return makeDevBox<float>(b->limits, periodic);
}

DevBox<double> boxOf(const ryo_box_f64* b)
{
    int periodic = b->boundary[0] == RYO_BOUNDARY_PERIODIC && b->boundary[1] == RYO_BOUNDARY_PERIODIC &&
                   b->boundary[2] == RYO_BOUNDARY_PERIODIC;
    return makeDevBox<double>(b->limits, periodic);
}

void checkBox(const float* l)
{
    for (int d = 0; d < 3; ++d)
        REQUIRE(l[2 * d + 1] > l[2 * d], "box: every axis needs max > min");
}

void checkBox(const double* l)
{
    for (int d = 0; d < 3; ++d)
        REQUIRE(l[2 * d + 1] > l[2 * d], "box: every axis needs max > min");
}

//! raise RYO_ERR_TIMEOUT if a kernel gave up a bounded wait
void checkDeviceError(ryo_ctx* ctx, cudaStream_t s)
{
    unsigned int err = 0;
    RYO_CUDA(cudaMemcpyAsync(&err, &ctx->ctl->error, sizeof(err), cudaMemcpyDeviceToHost, s));
    RYO_CUDA(cudaStreamSynchronize(s));
    if (err)
    {
        RYO_CUDA(cudaMemsetAsync(&ctx->ctl->error, 0, sizeof(unsigned int), s));
        throw ApiError{RYO_ERR_TIMEOUT, "a device-side bounded wait timed out"};
    }
}

} // namespace

// ==================================================================================================== context

extern "C" const char* ryo_status_string(ryo_status s)
{
    switch (s)
    {
        case RYO_OK: return "ok";
        case RYO_ERR_CUDA: return "CUDA error";
        case RYO_ERR_BAD_ARG: return "bad argument";
        case RYO_ERR_OOM: return "out of device memory";
        case RYO_ERR_STACK_OVERFLOW_UNSPLITTABLE: return "traversal stack overflow for a single target";
        case RYO_ERR_TIMEOUT: return "device wait timed out";
        case RYO_ERR_CAPACITY: return "buffer capacity too small";
        case RYO_ERR_NOT_CUBIC: return "Ewald needs a cubic periodic box";
        case RYO_ERR_NO_DEVICE: return "no CUDA device";
        case RYO_ERR_INTERNAL: return "internal error";
    }
    return "unknown status";
}

extern "C" const char* ryo_version(void) { return "0.1.0"; }

extern "C" ryo_status ryo_ctx_create(int device, ryo_ctx_t** out)
{
    if (!out) return RYO_ERR_BAD_ARG;
    *out         = nullptr;
    ryo_ctx* ctx = new (std::nothrow) ryo_ctx();
    if (!ctx)
    {
        tlsError = "ctx_create: host allocation failed";
        return RYO_ERR_OOM;
    }
    DeviceScope scope(device); // the caller's current device is restored on return
    ryo_status st = guarded(tlsError,
                            [&]
                            {
                                RYO_CUDA(cudaSetDevice(device));
                                ctx->device = device;
                                RYO_CUDA(cudaDeviceGetAttribute(&ctx->smCount, cudaDevAttrMultiProcessorCount, device));
                                RYO_CUDA(cudaMalloc(&ctx->ctl, sizeof(Control)));
                                RYO_CUDA(cudaMemset(ctx->ctl, 0, sizeof(Control)));
                            });
    if (st != RYO_OK)
    {
        delete ctx;
        return st;
    }
    *out = ctx;
    return RYO_OK;
}

extern "C" void ryo_ctx_destroy(ryo_ctx_t* ctx)
{
    if (!ctx) return;
    DeviceScope device(ctx->device);
    cudaDeviceSynchronize();
    ctx->releaseAll();
    if (ctx->ctl) cudaFree(ctx->ctl);
    delete ctx;
}

extern "C" const char* ryo_ctx_last_error(const ryo_ctx_t* ctx) { return ctx ? ctx->lastError.c_str() : tlsError.c_str(); }

// ==================================================================================================== cstone layer

extern "C" ryo_status ryo_compute_sfc_keys_f32(const float* x, const float* y, const float* z, uint64_t* keys,
                                               size_t n, const ryo_box_f32* box, ryo_stream_t stream)
{
    return guarded(tlsError,
                   [&]
                   {
                       REQUIRE(box && (n == 0 || (x && y && z && keys)), "compute_sfc_keys: null argument");
                       checkBox(box->limits);
                       launchKeys<float>(x, y, z, keys, n, boxOf(box), true, stream);
                   });
}

extern "C" ryo_status ryo_compute_sfc_keys_f64(const double* x, const double* y, const double* z, uint64_t* keys,
                                               size_t n, const ryo_box_f64* box, ryo_stream_t stream)
{
    return guarded(tlsError,
                   [&]
                   {
                       REQUIRE(box && (n == 0 || (x && y && z && keys)), "compute_sfc_keys: null argument");
                       checkBox(box->limits);
                       launchKeys<double>(x, y, z, keys, n, boxOf(box), true, stream);
                   });
}

extern "C" ryo_status ryo_compute_bounding_box_f32(ryo_ctx_t* ctx, const float* x, const float* y, const float* z,
                                                   size_t n, float* limits6, ryo_stream_t stream)
{
    if (!ctx) return RYO_ERR_BAD_ARG;
    return guardedCtx(ctx,
                   [&]
                   {
                       REQUIRE(limits6 && n > 0 && x && y && z, "compute_bounding_box: bad argument");
                       double* mm = ctx->scratch<double>("bbox", 6, stream);
                       launchBoundingBox(x, y, z, n, mm, stream);
                       double h[6];
                       RYO_CUDA(cudaMemcpyAsync(h, mm, sizeof(h), cudaMemcpyDeviceToHost, stream));
                       RYO_CUDA(cudaStreamSynchronize(stream));
                       for (int i = 0; i < 6; ++i)
                           limits6[i] = float(h[i]);
                   });
}

extern "C" ryo_status ryo_sequence(uint32_t* v, size_t n, uint32_t first, ryo_stream_t stream)
{
    return guarded(tlsError, [&] { launchSequence(v, n, first, stream); });
}

extern "C" size_t ryo_sort_by_key_temp_bytes(size_t n) { return sortTempBytes(n) + 64; }

namespace
{
__global__ void sortErrorFlagInit(unsigned int* f) { *f = 0; }
} // namespace

extern "C" ryo_status ryo_sort_by_key(uint64_t* keys, uint32_t* values, size_t n, uint64_t* keyBuf, uint32_t* valueBuf,
                                      void* tmp, size_t tmpBytes, ryo_stream_t stream)
{
    return guarded(tlsError,
                   [&]
                   {
                       if (n == 0) return;
                       REQUIRE(keys && values && keyBuf && valueBuf && tmp, "sort_by_key: null argument");
                       REQUIRE(n < (size_t(1) << 32), "sort_by_key: key count must be below 2^32");
                       if (tmpBytes < ryo_sort_by_key_temp_bytes(n))
                           throw ApiError{RYO_ERR_CAPACITY, "sort_by_key: temporary storage too small"};
                       // the last 64 bytes of tmp hold the wait-timeout flag
                       unsigned int* flag = reinterpret_cast<unsigned int*>(static_cast<char*>(tmp) + sortTempBytes(n));
                       sortErrorFlagInit<<<1, 1, 0, stream>>>(flag);
                       RYO_LAUNCH_CHECK();
                       bool alt = radixSortPairs(keys, values, keyBuf, valueBuf, n, 0, 64, tmp, sortTempBytes(n), flag,
                                                 stream, false);
                       if (alt)
                       {
                           RYO_CUDA(cudaMemcpyAsync(keys, keyBuf, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice,
                                                    stream));
                           RYO_CUDA(cudaMemcpyAsync(values, valueBuf, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                                                    stream));
                       }
                       unsigned int err = 0;
                       RYO_CUDA(cudaMemcpyAsync(&err, flag, sizeof(err), cudaMemcpyDeviceToHost, stream));
                       RYO_CUDA(cudaStreamSynchronize(stream));
                       if (err) throw ApiError{RYO_ERR_TIMEOUT, "sort_by_key: look-back wait timed out"};
                   });
}

extern "C" ryo_status ryo_sort_by_key_static(uint64_t* keys, uint32_t* values, size_t n, uint64_t* keyBuf,
                                             uint32_t* valueBuf, ryo_stream_t stream)
{
    return guarded(tlsError,
                   [&]
                   {
                       if (n == 0) return;
                       REQUIRE(keys && values && keyBuf && valueBuf, "sort_by_key_static: null argument");
                       if (n > staticSortMaxKeys())
                           throw ApiError{RYO_ERR_CAPACITY, "sort_by_key_static: more than RYO_SORT_STATIC_MAX_KEYS "
                                                            "keys; use ryo_sort_by_key with caller storage"};
                       if (sortPairsStaticScratch(keys, values, keyBuf, valueBuf, n, stream))
                           throw ApiError{RYO_ERR_TIMEOUT, "sort_by_key_static: look-back wait timed out"};
                   });
}

extern "C" ryo_status ryo_sort_wait_timeout_selftest(ryo_stream_t stream)
{
    return guarded(tlsError,
                   [&]
                   {
                       if (!sortWaitTimeoutSelfTest(stream))
                           throw ApiError{RYO_ERR_INTERNAL, "sort_wait_timeout_selftest: the look-back wait of a "
                                                            "tile whose predecessor never published did not report"};
                       throw ApiError{RYO_ERR_TIMEOUT, "sort_wait_timeout_selftest: look-back wait timed out"};
                   });
}

extern "C" ryo_status ryo_compute_octree(ryo_ctx_t* ctx, const uint64_t* sortedKeys, size_t n, unsigned bucketSize,
                                         uint64_t* leaves, uint32_t* counts, int capacity, int* numLeaves,
                                         ryo_stream_t stream)
{
    if (!ctx) return RYO_ERR_BAD_ARG;
    return guardedCtx(ctx,
                   [&]
                   {
                       REQUIRE(numLeaves && bucketSize > 0 && (n == 0 || sortedKeys), "compute_octree: bad argument");
                       REQUIRE(n < (size_t(1) << 32), "compute_octree: key count must be below 2^32");
                       int nl     = buildLeaves(ctx, sortedKeys, n, bucketSize, leaves, counts, nullptr, capacity,
                                                stream);
                       *numLeaves = nl;
                       RYO_CUDA(cudaStreamSynchronize(stream));
                       if (nl > capacity) throw ApiError{RYO_ERR_CAPACITY, "compute_octree: leaf capacity too small"};
                   });
}

extern "C" ryo_status ryo_build_octree(ryo_ctx_t* ctx, const uint64_t* leaves, int numLeaves, uint64_t* prefixes,
                                       int* childOffsets, int* parents, int* levelRange, int* d_levelRange,
                                       int* internalToLeaf, int* leafToInternal, ryo_stream_t stream)
{
    if (!ctx) return RYO_ERR_BAD_ARG;
    return guardedCtx(ctx,
                   [&]
                   {
                       REQUIRE(numLeaves >= 1 && leaves && prefixes && childOffsets && parents && levelRange &&
                                   internalToLeaf && leafToInternal,
                               "build_octree: bad argument");
                       OctreeArrays o{prefixes, childOffsets, parents, internalToLeaf, leafToInternal, d_levelRange};
                       linkOctree(ctx, leaves, numLeaves, o, levelRange, stream);
                       checkDeviceError(ctx, stream);
                   });
}

extern "C" ryo_status ryo_compute_fixed_groups(uint32_t first, uint32_t last, unsigned groupSize, uint32_t* groups,
                                               ryo_stream_t stream)
{
    return guarded(tlsError,
                   [&]
                   {
                       REQUIRE(groupSize > 0 && last >= first && groups, "compute_fixed_groups: bad argument");
                       launchFixedGroups(first, last, groupSize, groups, stream);
                   });
}

extern "C" ryo_status ryo_compute_group_splits_f32(ryo_ctx_t* ctx, uint32_t first, uint32_t last, const float* x,
                                                   const float* y, const float* z, const float* h,
                                                   const uint64_t* leaves, int numLeaves, const uint32_t* layout,
                                                   const ryo_box_f32* box, unsigned groupSize, float tolFactor,
                                                   float extentRatio, uint32_t* groups, uint32_t capacity,
                                                   uint32_t* numGroups, ryo_stream_t stream)
{
    if (!ctx) return RYO_ERR_BAD_ARG;
    return guardedCtx(ctx,
                   [&]
                   {
                       REQUIRE(numGroups && box && last >= first, "compute_group_splits: bad argument");
                       REQUIRE(groupSize == 32 || groupSize == 64, "compute_group_splits: groupSize must be 32 or 64");
                       REQUIRE(tolFactor > 0.f, "compute_group_splits: tolFactor must be positive");
                       REQUIRE(last == first || (x && y && z && leaves && layout && numLeaves >= 1),
                               "compute_group_splits: null argument");
                       checkBox(box->limits);
                       float ratio = extentRatio < 0.f ? defaultExtentRatio() : extentRatio;
                       uint32_t ng = computeGroupSplits(ctx, first, last, x, y, z, h, leaves, numLeaves, layout,
                                                        boxOf(box), groupSize, tolFactor, ratio, groups, capacity,
                                                        stream);
                       *numGroups = ng;
                       if (last > first && (!groups || ng + 1 > capacity))
                           throw ApiError{RYO_ERR_CAPACITY, "compute_group_splits: groups needs numGroups + 1 entries"};
                       RYO_CUDA(cudaStreamSynchronize(stream));
                   });
}

// ==================================================================================================== upsweep
//
// Each step exists for the reference's three type sets: _f32 (all float), _f64 (all double) and _mixed (double
// coordinates and centres, float masses and multipoles).

namespace
{
template<class Tc, class Tm, class Tf>
ryo_status leafSourceCenter(const Tc* x, const Tc* y, const Tc* z, const Tm* m, const int* leafToInternal,
                            int numLeaves, const uint32_t* layout, Tf* centers, ryo_stream_t stream)
{
    return guarded(tlsError,
                   [&]
                   {
                       REQUIRE(numLeaves == 0 || (x && y && z && m && leafToInternal && layout && centers),
                               "compute_leaf_source_center: null argument");
                       launchLeafCenters(x, y, z, m, leafToInternal, numLeaves, layout, centers, stream);
                   });
}

template<class Tf>
ryo_status upsweepCenters(int numLevels, const int* levelRange, const int* childOffsets, Tf* centers,
                          ryo_stream_t stream)
{
    return guarded(tlsError,
                   [&]
                   {
                       REQUIRE(levelRange && numLevels <= kMaxLevel + 1, "upsweep_centers: bad argument");
                       for (int level = numLevels - 1; level >= 0; --level)
                           launchUpsweepCenters(levelRange[level], levelRange[level + 1], childOffsets, centers,
                                                stream);
                   });
}

template<class Tc, class Tm, class Tf, class Tmp>
ryo_status leafMultipoles(const Tc* x, const Tc* y, const Tc* z, const Tm* m, const int* leafToInternal,
                          int numLeaves, const uint32_t* layout, const Tf* centers, Tmp* multipoles, bool mdq,
                          ryo_stream_t stream)
{
    return guarded(tlsError,
                   [&]
                   {
                       REQUIRE(numLeaves == 0 || (x && y && z && m && leafToInternal && layout && centers &&
                                                  multipoles),
                               "compute_leaf_multipoles: null argument");
                       launchLeafMultipoles(x, y, z, m, leafToInternal, numLeaves, layout, centers, multipoles, mdq,
                                            stream);
                   });
}

template<class Tf, class Tmp>
ryo_status upsweepMultipoles(int firstCell, int lastCell, const int* childOffsets, const Tf* centers, Tmp* multipoles,
                             bool mdq, ryo_stream_t stream)
{
    return guarded(tlsError,
                   [&]
                   {
                       REQUIRE(lastCell <= firstCell || (childOffsets && centers && multipoles),
                               "upsweep_multipoles: null argument");
                       launchUpsweepMultipoles(firstCell, lastCell, childOffsets, centers, multipoles, mdq, stream);
                   });
}

template<class T, class Box>
ryo_status setMac(const uint64_t* prefixes, int numNodes, T* centers, float invTheta, const Box* box,
                  ryo_stream_t stream)
{
    return guarded(tlsError,
                   [&]
                   {
                       REQUIRE(box, "set_mac: null box");
                       checkBox(box->limits);
                       launchSetMac(prefixes, numNodes, centers, invTheta, boxOf(box), stream);
                   });
}
} // namespace

extern "C" ryo_status ryo_compute_leaf_source_center_f32(const float* x, const float* y, const float* z,
                                                         const float* m, const int* leafToInternal, int numLeaves,
                                                         const uint32_t* layout, float* centers, ryo_stream_t stream)
{
    return leafSourceCenter(x, y, z, m, leafToInternal, numLeaves, layout, centers, stream);
}
extern "C" ryo_status ryo_compute_leaf_source_center_f64(const double* x, const double* y, const double* z,
                                                         const double* m, const int* leafToInternal, int numLeaves,
                                                         const uint32_t* layout, double* centers, ryo_stream_t stream)
{
    return leafSourceCenter(x, y, z, m, leafToInternal, numLeaves, layout, centers, stream);
}
extern "C" ryo_status ryo_compute_leaf_source_center_mixed(const double* x, const double* y, const double* z,
                                                           const float* m, const int* leafToInternal, int numLeaves,
                                                           const uint32_t* layout, double* centers,
                                                           ryo_stream_t stream)
{
    return leafSourceCenter(x, y, z, m, leafToInternal, numLeaves, layout, centers, stream);
}

extern "C" ryo_status ryo_upsweep_centers_f32(int numLevels, const int* levelRange, const int* childOffsets,
                                              float* centers, ryo_stream_t stream)
{
    return upsweepCenters(numLevels, levelRange, childOffsets, centers, stream);
}
extern "C" ryo_status ryo_upsweep_centers_f64(int numLevels, const int* levelRange, const int* childOffsets,
                                              double* centers, ryo_stream_t stream)
{
    return upsweepCenters(numLevels, levelRange, childOffsets, centers, stream);
}

#define RYO_LEAF_MULTIPOLES(NAME, Tc, Tm, Tf, Tmp, MDQ)                                                               \
    extern "C" ryo_status NAME(const Tc* x, const Tc* y, const Tc* z, const Tm* m, const int* leafToInternal,         \
                               int numLeaves, const uint32_t* layout, const Tf* centers, Tmp* multipoles,             \
                               ryo_stream_t stream)                                                                   \
    {                                                                                                                  \
        return leafMultipoles(x, y, z, m, leafToInternal, numLeaves, layout, centers, multipoles, MDQ, stream);      \
    }
RYO_LEAF_MULTIPOLES(ryo_compute_leaf_multipoles_f32, float, float, float, float, false)
RYO_LEAF_MULTIPOLES(ryo_compute_leaf_multipoles_f64, double, double, double, double, false)
RYO_LEAF_MULTIPOLES(ryo_compute_leaf_multipoles_mixed, double, float, double, float, false)
RYO_LEAF_MULTIPOLES(ryo_compute_leaf_multipoles_mdq_f32, float, float, float, float, true)
RYO_LEAF_MULTIPOLES(ryo_compute_leaf_multipoles_mdq_f64, double, double, double, double, true)
RYO_LEAF_MULTIPOLES(ryo_compute_leaf_multipoles_mdq_mixed, double, float, double, float, true)
#undef RYO_LEAF_MULTIPOLES

#define RYO_UPSWEEP_MULTIPOLES(NAME, Tf, Tmp, MDQ)                                                                    \
    extern "C" ryo_status NAME(int firstCell, int lastCell, const int* childOffsets, const Tf* centers,              \
                               Tmp* multipoles, ryo_stream_t stream)                                                  \
    {                                                                                                                  \
        return upsweepMultipoles(firstCell, lastCell, childOffsets, centers, multipoles, MDQ, stream);               \
    }
RYO_UPSWEEP_MULTIPOLES(ryo_upsweep_multipoles_f32, float, float, false)
RYO_UPSWEEP_MULTIPOLES(ryo_upsweep_multipoles_f64, double, double, false)
RYO_UPSWEEP_MULTIPOLES(ryo_upsweep_multipoles_mixed, double, float, false)
RYO_UPSWEEP_MULTIPOLES(ryo_upsweep_multipoles_mdq_f32, float, float, true)
RYO_UPSWEEP_MULTIPOLES(ryo_upsweep_multipoles_mdq_f64, double, double, true)
RYO_UPSWEEP_MULTIPOLES(ryo_upsweep_multipoles_mdq_mixed, double, float, true)
#undef RYO_UPSWEEP_MULTIPOLES

extern "C" ryo_status ryo_set_mac_f32(const uint64_t* prefixes, int numNodes, float* centers, float invTheta,
                                      const ryo_box_f32* box, ryo_stream_t stream)
{
    return setMac(prefixes, numNodes, centers, invTheta, box, stream);
}
extern "C" ryo_status ryo_set_mac_f64(const uint64_t* prefixes, int numNodes, double* centers, float invTheta,
                                      const ryo_box_f64* box, ryo_stream_t stream)
{
    return setMac(prefixes, numNodes, centers, invTheta, box, stream);
}

// ==================================================================================================== traversal

extern "C" int ryo_bh_max_target_size(void) { return 64; }
extern "C" uint32_t ryo_stack_size(uint32_t) { return 0; }

namespace
{

__global__ void splitGroupsKernel(const uint32_t* failed, uint32_t numFailed, const uint32_t* starts,
                                  const uint32_t* ends, const uint32_t* sys, uint32_t* newStart, uint32_t* newEnd,
                                  uint32_t* newSys, unsigned int* unsplit, unsigned int* numNew)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= numFailed) return;
    uint32_t g = failed[i];
    uint32_t a = starts[g], b = ends[g];
    if (b - a < 2)
    {
        atomicAdd(unsplit, 1u);
        return;
    }
    uint32_t mid  = a + (b - a) / 2;
    unsigned slot = atomicAdd(numNew, 2u);
    newStart[slot]     = a;
    newEnd[slot]       = mid;
    newStart[slot + 1] = mid;
    newEnd[slot + 1]   = b;
    if (sys) newSys[slot] = newSys[slot + 1] = sys[g];
}

/*! run a traversal to completion: groups that overflow the stack are split in two along the SFC and traversed
 *  again until none fails (traversal_gpu.cu:572-623); counts per group refer to the groups of @p t */
/*! the interaction count (direct bodies + 2 x approximated cells) past which a group is taken off its warp and
 *  split over several in a second pass. Uniform and Plummer groups stay well below it (at most about 17,000 at theta
 *  0.5); the groups that pass it are sparse outskirts whose bounding box reaches the dense centre, with up to a few
 *  hundred thousand direct bodies, which one warp would evaluate while the rest of the GPU idles. */
constexpr unsigned kHeavyCost      = 32768;
constexpr unsigned kWarpSlotsPerSm = 20;   // resident traversal warps per SM (5 blocks of 4)
constexpr unsigned kGroupsPerSlot  = 4;    // groups per warp slot from which a launch balances by itself
constexpr unsigned kMinHeavyCost   = 1024; // 16 evaluation batches

/*! the split threshold of a solve of @p numGroups groups. A solve with several groups per warp slot balances by
 *  itself and keeps kHeavyCost. A smaller one (a small system, or the last requests of a served stream) is bound by
 *  its slowest warps, so its threshold falls in proportion to its group count and more of its groups are spread
 *  over several warps: a 2^14-body Plummer sphere traverses in 0.38 ms instead of 0.86 ms. */
unsigned heavyCostFor(uint32_t numGroups, int smCount)
{
    const uint64_t full = uint64_t(smCount) * kWarpSlotsPerSm * kGroupsPerSlot;
    if (numGroups >= full) return kHeavyCost;
    return unsigned(std::max<uint64_t>(kMinHeavyCost, uint64_t(kHeavyCost) * numGroups / full));
}

//! warps per queued group: enough items to fill the GPU, at most 16 (each part repeats the group's walk)
int heavyParts(uint32_t numHeavy, int smCount)
{
    uint32_t want = (uint32_t(smCount) * kWarpSlotsPerSm + numHeavy - 1) / numHeavy;
    return int(std::max(2u, std::min(16u, want)));
}

/*! the groups of a traverse call are the caller's: each must hold 1 to 64 targets inside [firstBody, lastBody). A
 *  warp evaluates at most 64 targets, and an empty group would read before its start. The reference refuses
 *  unsupported group sizes too (cstone/traversal/groups_gpu.cu:150). The check reads the group arrays back, so the
 *  call synchronises its stream. */
void checkCallerGroups(const ryo_group_view* grp, cudaStream_t stream)
{
    if (grp->numGroups == 0) return;
    REQUIRE(grp->groupStart && grp->groupEnd, "traverse: null group arrays");
    std::vector<uint32_t> gs(grp->numGroups), ge(grp->numGroups);
    RYO_CUDA(cudaMemcpyAsync(gs.data(), grp->groupStart, gs.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                             stream));
    RYO_CUDA(cudaMemcpyAsync(ge.data(), grp->groupEnd, ge.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    RYO_CUDA(cudaStreamSynchronize(stream));
    for (size_t g = 0; g < gs.size(); ++g)
        REQUIRE(gs[g] >= grp->firstBody && ge[g] <= grp->lastBody && ge[g] > gs[g] && ge[g] - gs[g] <= 64,
                "traverse: every group needs 1 to 64 targets within [firstBody, lastBody)");
}

void runTraversal(ryo_ctx* ctx, TraverseLaunch t, cudaStream_t s, double* potentialOut)
{
    const uint32_t numGroups = uint32_t(t.numGroups);
    t.ctl                    = ctx->ctl;
    if (t.stackCapacity <= 0) t.stackCapacity = 512; // the deepest walks measured use about 110 entries
    launchTraversalReset(ctx->ctl, true, s);
    ctx->retries          = 0;
    bool unsplittable     = false;
    uint32_t* failed      = ctx->scratch<uint32_t>("trav.failed", std::max<uint32_t>(numGroups, 1), s);
    t.failedGroups        = failed;
    t.failedCapacity      = numGroups;
    int pass              = 0;
    bool flip             = false; // alternates the scratch buffers of successive split passes
    // one threshold for every pass, from the solve's group count: a group's split decision depends on its cost and
    // the solve's size, not on the launch or retry pass it falls in
    const unsigned heavyCost = heavyCostFor(t.balanceGroups ? t.balanceGroups : numGroups, ctx->smCount);
    while (t.numGroups > 0)
    {
        if (pass > 0) launchTraversalReset(ctx->ctl, false, s);
        ++pass;
        // first pass: groups too costly for one warp are queued; second pass: each queued group split over warps
        t.heavyGroups   = ctx->scratch<uint32_t>("trav.heavy", std::max(t.numGroups, 1), s);
        t.heavyCapacity = uint32_t(t.numGroups);
        t.heavyCost     = heavyCost;
        t.parts         = 0;
        t.numHeavy      = 0;
        launchTraverse(t, ctx->smCount, s);
        unsigned int counts[2] = {0, 0}; // failed, queued
        RYO_CUDA(cudaMemcpyAsync(&counts[0], &ctx->ctl->failedCount, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        RYO_CUDA(cudaMemcpyAsync(&counts[1], &ctx->ctl->heavyCount, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        RYO_CUDA(cudaStreamSynchronize(s));
        if (counts[1] > 0)
        {
            TraverseLaunch t2 = t;
            t2.numHeavy       = std::min(counts[1], t.heavyCapacity);
            t2.parts          = heavyParts(t2.numHeavy, ctx->smCount);
            size_t items      = size_t(t2.numHeavy) * size_t(t2.parts);
            t2.partials       = ctx->scratch<float4>("trav.partials", items * 2 * kWarp, s);
            t2.partStatus     = ctx->scratch<int>("trav.partStatus", items, s);
            RYO_CUDA(cudaMemsetAsync(&ctx->ctl->workCounter, 0, sizeof(unsigned), s));
            launchTraverse(t2, ctx->smCount, s);
            launchCombineHeavy(t2, t.nodes ? t.tgtM : t.mt, s);
            RYO_CUDA(cudaMemcpyAsync(&counts[0], &ctx->ctl->failedCount, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
            RYO_CUDA(cudaStreamSynchronize(s));
        }
        unsigned int numFailed = counts[0];
        if (numFailed == 0) break;
        ctx->retries += numFailed;
        // split the failed groups on the device: halves along the SFC
        uint32_t cap      = 2 * numFailed;
        uint32_t* nStart  = ctx->scratch<uint32_t>(flip ? "trav.splitB" : "trav.splitA", cap, s);
        uint32_t* nEnd    = ctx->scratch<uint32_t>(flip ? "trav.splitEndB" : "trav.splitEndA", cap, s);
        uint32_t* nSys    = t.groupSys ? ctx->scratch<uint32_t>(flip ? "trav.splitSysB" : "trav.splitSysA", cap, s)
                                       : nullptr;
        unsigned int* cnt = ctx->ctl->counters;
        RYO_CUDA(cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned int), s));
        splitGroupsKernel<<<ceilDiv(numFailed, 256), 256, 0, s>>>(failed, numFailed, t.groupStart, t.groupEnd,
                                                                   t.groupSys, nStart, nEnd, nSys, cnt + 1, cnt);
        RYO_LAUNCH_CHECK();
        unsigned int h[2];
        RYO_CUDA(cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, s));
        RYO_CUDA(cudaStreamSynchronize(s));
        if (h[1] > 0) unsplittable = true;
        // the new groups go to the buffer set not read by this pass
        uint32_t* keepStart = ctx->scratch<uint32_t>(flip ? "trav.curB" : "trav.curA", std::max(h[0], 1u), s);
        uint32_t* keepEnd   = ctx->scratch<uint32_t>(flip ? "trav.curEndB" : "trav.curEndA", std::max(h[0], 1u), s);
        RYO_CUDA(cudaMemcpyAsync(keepStart, nStart, h[0] * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        RYO_CUDA(cudaMemcpyAsync(keepEnd, nEnd, h[0] * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        if (t.groupSys)
        {
            uint32_t* keepSys = ctx->scratch<uint32_t>(flip ? "trav.curSysB" : "trav.curSysA", std::max(h[0], 1u), s);
            RYO_CUDA(cudaMemcpyAsync(keepSys, nSys, h[0] * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
            t.groupSys = keepSys;
        }
        t.groupStart = keepStart;
        t.groupEnd   = keepEnd;
        t.numGroups  = int(h[0]);
        t.groupM2P   = nullptr; // per-group counts are reported for unsplit groups only
        t.groupP2P   = nullptr;
        flip         = !flip;
        if (t.numGroups == 0) break;
        failed           = ctx->scratch<uint32_t>(flip ? "trav.failedB" : "trav.failedA", t.numGroups, s);
        t.failedGroups   = failed;
        t.failedCapacity = uint32_t(t.numGroups);
    }
    Control hc;
    RYO_CUDA(cudaMemcpyAsync(&hc, ctx->ctl, sizeof(Control), cudaMemcpyDeviceToHost, s));
    RYO_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < 5; ++i)
        ctx->hostStats[i] = hc.stats[i];
    if (unsplittable) ctx->hostStats[kMaxP2P] = 0xFFFFFFFFull;
    if (potentialOut) *potentialOut = hc.potential;
    if (hc.error) throw ApiError{RYO_ERR_TIMEOUT, "traversal: a device-side bounded wait timed out"};
}

} // namespace

extern "C" ryo_status ryo_traverse_ex_f32(ryo_ctx_t* ctx, const ryo_group_view* grp, int initNodeIdx, const float* xt,
                                          const float* yt, const float* zt, const float* mt, const float* ht,
                                          const float* xs, const float* ys, const float* zs, const float* ms,
                                          const float* hs, const int* childOffsets, const int* internalToLeaf,
                                          const uint32_t* layout, const float* sourceCenter, const float* multipoles,
                                          float G, int numShells, const float* boxL, float* p, float* ax, float* ay,
                                          float* az, double* totalPotential, const ryo_traverse_options* options,
                                          ryo_stream_t stream)
{
    if (!ctx) return RYO_ERR_BAD_ARG;
    return guardedCtx(ctx,
                   [&]
                   {
                       REQUIRE(grp && xt && yt && zt && mt && ht && xs && ys && zs && ms && hs && childOffsets &&
                                   internalToLeaf && layout && sourceCenter && multipoles && ax && ay && az,
                               "traverse: null argument");
                       REQUIRE(numShells >= 0 && (numShells == 0 || boxL), "traverse: replicas need boxL");
                       checkCallerGroups(grp, stream);
                       TraverseLaunch t{};
                       t.groupStart     = grp->groupStart;
                       t.groupEnd       = grp->groupEnd;
                       t.numGroups      = int(grp->numGroups);
                       t.initNode       = initNodeIdx;
                       t.numNodes       = initNodeIdx == 0 ? 1 : 2;
                       t.nodes          = nullptr;
                       t.centers        = reinterpret_cast<const float4*>(sourceCenter);
                       t.multipoles     = multipoles;
                       t.childOffsets   = childOffsets;
                       t.internalToLeaf = internalToLeaf;
                       t.layout         = layout;
                       t.xt = xt, t.yt = yt, t.zt = zt, t.mt = mt, t.ht = ht;
                       t.xs = xs, t.ys = ys, t.zs = zs, t.ms = ms, t.hs = hs;
                       t.G         = G;
                       t.numShells = numShells;
                       for (int d = 0; d < 3; ++d)
                           t.boxL[d] = numShells > 0 ? boxL[d] : 0.f;
                       t.p  = p;
                       t.ax = ax;
                       t.ay = ay;
                       t.az = az;
                       t.groupM2P      = options ? options->groupM2P : nullptr;
                       t.groupP2P      = options ? options->groupP2P : nullptr;
                       t.stackCapacity = options ? options->stackCapacity : 0;
                       t.mdqArrays     = options && options->multipole == RYO_MULTIPOLE_MDQ ? 1 : 0;
                       double pot      = 0;
                       runTraversal(ctx, t, stream, &pot);
                       if (totalPotential) *totalPotential = 0.5 * double(G) * pot;
                       if (ctx->hostStats[kMaxP2P] == 0xFFFFFFFFull)
                           throw ApiError{RYO_ERR_STACK_OVERFLOW_UNSPLITTABLE,
                                          "traverse: a single target overflowed the stack"};
                   });
}

extern "C" ryo_status ryo_traverse_f32(ryo_ctx_t* ctx, const ryo_group_view* grp, int initNodeIdx, const float* xt,
                                       const float* yt, const float* zt, const float* mt, const float* ht,
                                       const float* xs, const float* ys, const float* zs, const float* ms,
                                       const float* hs, const int* childOffsets, const int* internalToLeaf,
                                       const uint32_t* layout, const float* sourceCenter, const float* multipoles,
                                       float G, int numShells, const float* boxL, float* p, float* ax, float* ay,
                                       float* az, double* totalPotential, ryo_stream_t stream)
{
    return ryo_traverse_ex_f32(ctx, grp, initNodeIdx, xt, yt, zt, mt, ht, xs, ys, zs, ms, hs, childOffsets,
                               internalToLeaf, layout, sourceCenter, multipoles, G, numShells, boxL, p, ax, ay, az,
                               totalPotential, nullptr, stream);
}

namespace
{
//! the double-coordinate instantiations of traverse (traversal_gpu.cu:637-638): Th softenings, Tm masses, Ta
//! outputs, Tmp multipole values; centres are 4 doubles per node
template<class Th, class Tm, class Ta, class Tmp>
ryo_status traverseDouble(ryo_ctx_t* ctx, int precision, const ryo_group_view* grp, int initNodeIdx, const double* xt,
                          const double* yt, const double* zt, const Tm* mt, const Th* ht, const double* xs,
                          const double* ys, const double* zs, const Tm* ms, const Th* hs, const int* childOffsets,
                          const int* internalToLeaf, const uint32_t* layout, const double* sourceCenter,
                          const Tmp* multipoles, double G, int numShells, const double* boxL, Ta* p, Ta* ax, Ta* ay,
                          Ta* az, double* totalPotential, const ryo_traverse_options* options, ryo_stream_t stream)
{
    if (!ctx) return RYO_ERR_BAD_ARG;
    return guardedCtx(ctx,
                   [&]
                   {
                       REQUIRE(grp && xt && yt && zt && mt && ht && xs && ys && zs && ms && hs && childOffsets &&
                                   internalToLeaf && layout && sourceCenter && multipoles && ax && ay && az,
                               "traverse: null argument");
                       REQUIRE(numShells >= 0 && (numShells == 0 || boxL), "traverse: replicas need boxL");
                       checkCallerGroups(grp, stream);
                       TraverseLaunch t{};
                       t.precision      = precision;
                       t.groupStart     = grp->groupStart;
                       t.groupEnd       = grp->groupEnd;
                       t.numGroups      = int(grp->numGroups);
                       t.initNode       = initNodeIdx;
                       t.numNodes       = initNodeIdx == 0 ? 1 : 2;
                       t.childOffsets   = childOffsets;
                       t.internalToLeaf = internalToLeaf;
                       t.layout         = layout;
                       t.xt64 = xt, t.yt64 = yt, t.zt64 = zt, t.mt64 = mt, t.ht64 = ht;
                       t.xs64 = xs, t.ys64 = ys, t.zs64 = zs, t.ms64 = ms, t.hs64 = hs;
                       t.centers64    = sourceCenter;
                       t.multipoles64 = multipoles;
                       t.G64          = G;
                       t.G            = float(G);
                       t.numShells    = numShells;
                       for (int d = 0; d < 3; ++d)
                           t.boxL64[d] = numShells > 0 ? boxL[d] : 0.0;
                       t.p64 = p, t.ax64 = ax, t.ay64 = ay, t.az64 = az;
                       t.groupM2P      = options ? options->groupM2P : nullptr;
                       t.groupP2P      = options ? options->groupP2P : nullptr;
                       t.stackCapacity = options ? options->stackCapacity : 0;
                       t.mdqArrays     = options && options->multipole == RYO_MULTIPOLE_MDQ ? 1 : 0;
                       double pot      = 0;
                       runTraversal(ctx, t, stream, &pot);
                       if (totalPotential) *totalPotential = 0.5 * G * pot;
                       if (ctx->hostStats[kMaxP2P] == 0xFFFFFFFFull)
                           throw ApiError{RYO_ERR_STACK_OVERFLOW_UNSPLITTABLE,
                                          "traverse: a single target overflowed the stack"};
                   });
}
} // namespace

extern "C" ryo_status ryo_traverse_f64(ryo_ctx_t* ctx, const ryo_group_view* grp, int initNodeIdx, const double* xt,
                                       const double* yt, const double* zt, const double* mt, const double* ht,
                                       const double* xs, const double* ys, const double* zs, const double* ms,
                                       const double* hs, const int* childOffsets, const int* internalToLeaf,
                                       const uint32_t* layout, const double* sourceCenter, const double* multipoles,
                                       double G, int numShells, const double* boxL, double* p, double* ax, double* ay,
                                       double* az, double* totalPotential, const ryo_traverse_options* options,
                                       ryo_stream_t stream)
{
    return traverseDouble(ctx, kPrecisionF64, grp, initNodeIdx, xt, yt, zt, mt, ht, xs, ys, zs, ms, hs, childOffsets,
                          internalToLeaf, layout, sourceCenter, multipoles, G, numShells, boxL, p, ax, ay, az,
                          totalPotential, options, stream);
}

extern "C" ryo_status ryo_traverse_mixed(ryo_ctx_t* ctx, const ryo_group_view* grp, int initNodeIdx, const double* xt,
                                         const double* yt, const double* zt, const float* mt, const float* ht,
                                         const double* xs, const double* ys, const double* zs, const float* ms,
                                         const float* hs, const int* childOffsets, const int* internalToLeaf,
                                         const uint32_t* layout, const double* sourceCenter, const float* multipoles,
                                         double G, int numShells, const double* boxL, float* p, float* ax, float* ay,
                                         float* az, double* totalPotential, const ryo_traverse_options* options,
                                         ryo_stream_t stream)
{
    return traverseDouble(ctx, kPrecisionMixed, grp, initNodeIdx, xt, yt, zt, mt, ht, xs, ys, zs, ms, hs,
                          childOffsets, internalToLeaf, layout, sourceCenter, multipoles, G, numShells, boxL, p, ax,
                          ay, az, totalPotential, options, stream);
}

extern "C" ryo_status ryo_let_export_f32(ryo_ctx_t* ctx, const float* peerBox6, uint32_t* buffer,
                                         size_t capacityWords, ryo_let_counts* counts, ryo_stream_t stream)
{
    if (!ctx) return RYO_ERR_BAD_ARG;
    return guardedCtx(ctx,
                   [&]
                   {
                       const auto& S = ctx->solveState;
                       REQUIRE(peerBox6 && counts, "let_export: null argument");
                       REQUIRE(S.valid && S.nodes, "let_export: needs a preceding ryo_solve_f32 on this context");
                       REQUIRE(!S.periodic, "let_export: open boundaries only");
                       REQUIRE(!S.dipoles, "let_export: quadrupole expansions only");
                       for (int d = 0; d < 3; ++d)
                           REQUIRE(peerBox6[2 * d + 1] >= peerBox6[2 * d], "let_export: box max below min");
                       LetBox box;
                       for (int d = 0; d < 3; ++d)
                       {
                           float lo = peerBox6[2 * d], hi = peerBox6[2 * d + 1];
                           box.tc[d] = (hi + lo) * 0.5f; // the traversal's group box, rounded the same way
                           box.ts[d] = (hi - lo) * 0.5f;
                       }
                       const NodeRecord* nodes = static_cast<const NodeRecord*>(S.nodes);
                       LetCounts c = letSelect(ctx, nodes, ctx->lastSolve.parents, S.numNodes, box, stream);
                       counts->numNodes  = c.numNodes;
                       counts->numLeaves = c.numLeaves;
                       counts->numBodies = c.numBodies;
                       counts->words     = c.words();
                       if (!buffer || capacityWords < c.words())
                           throw ApiError{RYO_ERR_CAPACITY, "let_export: the buffer needs counts->words words"};
                       letWrite(c, nodes, S.numNodes, static_cast<const float4*>(S.xyzm), S.srcH, box, buffer,
                                stream);
                   });
}

extern "C" ryo_status ryo_read_bh_stats(ryo_ctx_t* ctx, uint64_t* stats5)
{
    if (!ctx || !stats5) return RYO_ERR_BAD_ARG;
    for (int i = 0; i < 5; ++i)
        stats5[i] = ctx->hostStats[i];
    return RYO_OK;
}

extern "C" uint64_t ryo_read_traversal_retries(ryo_ctx_t* ctx) { return ctx ? ctx->retries : 0; }

// ==================================================================================================== Ewald

namespace
{
//! computeGravityEwaldGpu for one type set: Tr the root expansion's values, Tc coordinates and box, Tm masses, Ta
//! outputs (ryoanji/src/ryoanji/interface/ewald.cu:31-110)
template<class Tr, class Tc, class Tm, class Ta, class Box>
ryo_status gravityEwald(ryo_ctx_t* ctx, const Tc* rootCenter, const Tr* Mroot, const ryo_group_view* grp, const Tc* x,
                        const Tc* y, const Tc* z, const Tm* m, const Box* box, float G, Ta* ugrav, Ta* ax, Ta* ay,
                        Ta* az, double* ugravTot, const ryo_ewald_settings* settings, ryo_stream_t stream)
{
    if (!ctx) return RYO_ERR_BAD_ARG;
    return guardedCtx(ctx,
                   [&]
                   {
                       checkEwald(settings);
                       REQUIRE(rootCenter && Mroot && grp && x && y && z && m && box && ax && ay && az && settings,
                               "compute_gravity_ewald: null argument");
                       Tc lx = box->limits[1] - box->limits[0], ly = box->limits[3] - box->limits[2],
                          lz = box->limits[5] - box->limits[4];
                       if (!(lx == ly && ly == lz)) throw ApiError{RYO_ERR_NOT_CUBIC, "Ewald needs a cubic box"};
                       double mr[8], c[3];
                       for (int i = 0; i < 8; ++i)
                           mr[i] = double(Mroot[i]);
                       for (int i = 0; i < 3; ++i)
                           c[i] = double(rootCenter[i]);
                       EwaldHost e = ewaldSetup(mr, c, settings->numReplicaShells, double(lx), settings->lCut,
                                                settings->hCut, settings->alpha_scale,
                                                settings->small_R_scale_factor);
                       double* pot = &ctx->ctl->ewaldPotential;
                       RYO_CUDA(cudaMemsetAsync(pot, 0, sizeof(double), stream));
                       launchEwaldGroups(e, grp->groupStart, grp->groupEnd, grp->numGroups, x, y, z, m, G, ugrav, ax,
                                         ay, az, pot, stream);
                       double h = 0;
                       RYO_CUDA(cudaMemcpyAsync(&h, pot, sizeof(double), cudaMemcpyDeviceToHost, stream));
                       RYO_CUDA(cudaStreamSynchronize(stream));
                       if (ugravTot) *ugravTot += 0.5 * double(G) * h;
                   });
}
} // namespace

extern "C" ryo_status ryo_compute_gravity_ewald_f32(ryo_ctx_t* ctx, const float* rootCenter, const float* Mroot,
                                                    const ryo_group_view* grp, const float* x, const float* y,
                                                    const float* z, const float* m, const ryo_box_f32* box, float G,
                                                    float* ugrav, float* ax, float* ay, float* az, double* ugravTot,
                                                    const ryo_ewald_settings* settings, ryo_stream_t stream)
{
    return gravityEwald(ctx, rootCenter, Mroot, grp, x, y, z, m, box, G, ugrav, ax, ay, az, ugravTot, settings,
                        stream);
}

extern "C" ryo_status ryo_compute_gravity_ewald_f64(ryo_ctx_t* ctx, const double* rootCenter, const double* Mroot,
                                                    const ryo_group_view* grp, const double* x, const double* y,
                                                    const double* z, const double* m, const ryo_box_f64* box, float G,
                                                    double* ugrav, double* ax, double* ay, double* az,
                                                    double* ugravTot, const ryo_ewald_settings* settings,
                                                    ryo_stream_t stream)
{
    return gravityEwald(ctx, rootCenter, Mroot, grp, x, y, z, m, box, G, ugrav, ax, ay, az, ugravTot, settings,
                        stream);
}

extern "C" ryo_status ryo_compute_gravity_ewald_mixed(ryo_ctx_t* ctx, const double* rootCenter, const float* Mroot,
                                                      const ryo_group_view* grp, const double* x, const double* y,
                                                      const double* z, const float* m, const ryo_box_f64* box,
                                                      float G, float* ugrav, float* ax, float* ay, float* az,
                                                      double* ugravTot, const ryo_ewald_settings* settings,
                                                      ryo_stream_t stream)
{
    return gravityEwald(ctx, rootCenter, Mroot, grp, x, y, z, m, box, G, ugrav, ax, ay, az, ugravTot, settings,
                        stream);
}

// ==================================================================================================== direct sums

extern "C" ryo_status ryo_direct_sum_f32(size_t first, size_t last, size_t numBodies, const float* boxL,
                                         int numShells, const float* x, const float* y, const float* z,
                                         const float* m, const float* h, float* p, float* ax, float* ay, float* az,
                                         ryo_stream_t stream)
{
    return guarded(tlsError,
                   [&]
                   {
                       REQUIRE(first <= last && last <= numBodies, "direct_sum: targets must be within the bodies");
                       REQUIRE(numShells >= 0 && (numShells == 0 || boxL), "direct_sum: replicas need boxL");
                       REQUIRE(last == first || (x && y && z && m && h && ax && ay && az),
                               "direct_sum: null argument");
                       launchDirect<float>(first, last, numBodies, boxL, numShells, x, y, z, m, h, p, ax, ay, az,
                                         stream);
                   });
}

extern "C" ryo_status ryo_direct_sum_f64(size_t first, size_t last, size_t numBodies, const double* boxL,
                                         int numShells, const double* x, const double* y, const double* z,
                                         const double* m, const double* h, double* p, double* ax, double* ay,
                                         double* az, ryo_stream_t stream)
{
    return guarded(tlsError,
                   [&]
                   {
                       REQUIRE(first <= last && last <= numBodies, "direct_sum: targets must be within the bodies");
                       REQUIRE(numShells >= 0 && (numShells == 0 || boxL), "direct_sum: replicas need boxL");
                       REQUIRE(last == first || (x && y && z && m && h && ax && ay && az),
                               "direct_sum: null argument");
                       launchDirect<double>(first, last, numBodies, boxL, numShells, x, y, z, m, h, p, ax, ay, az,
                                         stream);
                   });
}

extern "C" ryo_status ryo_direct_targets_f64(const int64_t* targets, size_t numTargets, const float* x, const float* y,
                                             const float* z, const float* m, const float* h, size_t numBodies,
                                             double G, const double* boxL, int numShells, double* pot, double* ax,
                                             double* ay, double* az, ryo_stream_t stream)
{
    return guarded(tlsError,
                   [&]
                   {
                       REQUIRE(numShells >= 0 && (numShells == 0 || boxL), "direct_targets: replicas need boxL");
                       if (numTargets == 0) return;
                       REQUIRE(targets && x && y && z && m && h && pot && ax && ay && az,
                               "direct_targets: null argument");
                       // every target must index a body: the kernel reads its position
                       std::vector<int64_t> t(numTargets);
                       RYO_CUDA(cudaMemcpyAsync(t.data(), targets, numTargets * sizeof(int64_t), cudaMemcpyDeviceToHost,
                                                stream));
                       RYO_CUDA(cudaStreamSynchronize(stream));
                       for (int64_t i : t)
                           REQUIRE(i >= 0 && uint64_t(i) < numBodies, "direct_targets: a target index is not a body");
                       launchDirectTargets(targets, numTargets, x, y, z, m, h, numBodies, G, boxL, numShells, pot, ax,
                                           ay, az, stream);
                   });
}

// ==================================================================================================== TreeBuilder

struct ryo_treebuilder
{
    ryo_ctx* ctx;
    unsigned ncrit;
    std::string tag;
    size_t numBodies = 0;
    int numLeaves = 0, numInternal = 0, numNodes = 0;
    int levelRange[kMaxLevel + 2] = {};
    uint64_t* sortedKeys = nullptr;
    uint32_t* order      = nullptr;
    uint64_t* leaves     = nullptr;
    uint32_t* counts     = nullptr;
    uint32_t* layout     = nullptr;
    OctreeArrays oct{};

    template<class T>
    T* buf(const char* name, size_t count, cudaStream_t s)
    {
        return ctx->scratch<T>(tag + name, count, s);
    }
};

namespace
{
template<class T>
void treebuilderUpdate(ryo_treebuilder* tb, T* x, T* y, T* z, size_t n, const DevBox<T>& box, cudaStream_t s)
{
    ryo_ctx* ctx = tb->ctx;
    REQUIRE(n > 0 && n < (size_t(1) << 32), "treebuilder: body count must be in [1, 2^32)");
    uint64_t* keys     = tb->buf<uint64_t>(".keys", n, s);
    uint64_t* keysAlt  = tb->buf<uint64_t>(".keysAlt", n, s);
    uint32_t* order    = tb->buf<uint32_t>(".order", n, s);
    uint32_t* orderAlt = tb->buf<uint32_t>(".orderAlt", n, s);
    size_t tmpBytes    = sortTempBytes(n);
    void* tmp          = tb->buf<char>(".sorttmp", tmpBytes, s);
    T* scratch         = tb->buf<T>(".coord", n, s);

    launchKeys<T>(x, y, z, keys, n, box, false, s);
    bool alt       = radixSortPairs(keys, order, keysAlt, orderAlt, n, 0, 64, tmp, tmpBytes, &ctx->ctl->error, s, true);
    tb->sortedKeys = alt ? keysAlt : keys;
    tb->order      = alt ? orderAlt : order;
    for (T* a : {x, y, z})
    {
        launchGatherT<T>(tb->order, a, scratch, n, s);
        RYO_CUDA(cudaMemcpyAsync(a, scratch, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
    }

    int cap     = int(std::min<size_t>(n / 2 + 64, size_t(1) << 30));
    tb->leaves  = tb->buf<uint64_t>(".leaves", size_t(cap) + 1, s);
    tb->counts  = tb->buf<uint32_t>(".counts", cap, s);
    tb->layout  = tb->buf<uint32_t>(".layout", size_t(cap) + 1, s);
    int nl      = buildLeaves(ctx, tb->sortedKeys, n, tb->ncrit, tb->leaves, tb->counts, tb->layout, cap, s);
    if (nl > cap)
    {
        cap        = nl;
        tb->leaves = tb->buf<uint64_t>(".leaves", size_t(cap) + 1, s);
        tb->counts = tb->buf<uint32_t>(".counts", cap, s);
        tb->layout = tb->buf<uint32_t>(".layout", size_t(cap) + 1, s);
        nl         = buildLeaves(ctx, tb->sortedKeys, n, tb->ncrit, tb->leaves, tb->counts, tb->layout, cap, s);
    }
    tb->numLeaves   = nl;
    tb->numInternal = (nl - 1) / 7;
    tb->numNodes    = nl + tb->numInternal;
    int nn          = tb->numNodes;
    tb->oct.prefixes       = tb->buf<uint64_t>(".prefixes", nn, s);
    tb->oct.childOffsets   = tb->buf<int>(".childOffsets", size_t(nn) + 1, s);
    tb->oct.parents        = tb->buf<int>(".parents", std::max(1, (nn - 1) / 8), s);
    tb->oct.internalToLeaf = tb->buf<int>(".internalToLeaf", nn, s);
    tb->oct.leafToInternal = tb->buf<int>(".leafToInternal", nn, s);
    tb->oct.d_levelRange   = tb->buf<int>(".levelRange", kMaxLevel + 2, s);
    linkOctree(ctx, tb->leaves, nl, tb->oct, tb->levelRange, s);
    tb->numBodies = n;
    checkDeviceError(ctx, s);
}
} // namespace

extern "C" ryo_status ryo_treebuilder_create(ryo_ctx_t* ctx, unsigned ncrit, ryo_treebuilder_t** out)
{
    if (!ctx || !out || ncrit == 0) return RYO_ERR_BAD_ARG;
    // the tag names the builder's buffers in the context: unique across threads
    static std::atomic<unsigned long long> counter{0};
    return guardedCtx(ctx,
                   [&]
                   {
                       auto tb   = std::make_unique<ryo_treebuilder>();
                       tb->ctx   = ctx;
                       tb->ncrit = ncrit;
                       tb->tag   = "tb" + std::to_string(++counter);
                       *out      = tb.release();
                   });
}

extern "C" void ryo_treebuilder_destroy(ryo_treebuilder_t* tb)
{
    if (!tb) return;
    DeviceScope device(tb->ctx->device);
    cudaDeviceSynchronize();
    for (auto it = tb->ctx->buffers.begin(); it != tb->ctx->buffers.end();)
    {
        if (it->first.rfind(tb->tag + ".", 0) == 0)
        {
            if (it->second.ptr) cudaFree(it->second.ptr);
            it = tb->ctx->buffers.erase(it);
        }
        else ++it;
    }
    delete tb;
}

extern "C" ryo_status ryo_treebuilder_update_f32(ryo_treebuilder_t* tb, float* x, float* y, float* z, size_t n,
                                                 const ryo_box_f32* box, int* numNodes, ryo_stream_t stream)
{
    if (!tb) return RYO_ERR_BAD_ARG;
    return guardedCtx(tb->ctx,
                   [&]
                   {
                       REQUIRE(x && y && z && box, "treebuilder_update: null argument");
                       checkBox(box->limits);
                       treebuilderUpdate<float>(tb, x, y, z, n, boxOf(box), stream);
                       if (numNodes) *numNodes = tb->numNodes;
                   });
}

extern "C" ryo_status ryo_treebuilder_update_f64(ryo_treebuilder_t* tb, double* x, double* y, double* z, size_t n,
                                                 const ryo_box_f64* box, int* numNodes, ryo_stream_t stream)
{
    if (!tb) return RYO_ERR_BAD_ARG;
    return guardedCtx(tb->ctx,
                   [&]
                   {
                       REQUIRE(x && y && z && box, "treebuilder_update: null argument");
                       checkBox(box->limits);
                       treebuilderUpdate<double>(tb, x, y, z, n, boxOf(box), stream);
                       if (numNodes) *numNodes = tb->numNodes;
                   });
}

extern "C" ryo_status ryo_treebuilder_view(const ryo_treebuilder_t* tb, ryo_tree_view* out)
{
    if (!tb || !out) return RYO_ERR_BAD_ARG;
    out->numLeafNodes     = tb->numLeaves;
    out->numInternalNodes = tb->numInternal;
    out->numNodes         = tb->numNodes;
    out->maxTreeLevel     = kMaxLevel;
    out->layout           = tb->layout;
    out->nodeKeys         = tb->oct.prefixes;
    out->childOffsets     = tb->oct.childOffsets;
    out->leafToInternal   = tb->oct.leafToInternal ? tb->oct.leafToInternal + tb->numInternal : nullptr;
    out->internalToLeaf   = tb->oct.internalToLeaf;
    out->parents          = tb->oct.parents;
    out->leaves           = tb->leaves;
    out->order            = tb->order;
    out->sortedKeys       = tb->sortedKeys;
    for (int i = 0; i < kMaxLevel + 2; ++i)
        out->levelRange[i] = tb->levelRange[i];
    return RYO_OK;
}

// ==================================================================================================== fused solve

extern "C" void ryo_solve_params_default(ryo_solve_params* p)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->bucketSize                 = 64;
    p->groupSize                  = 64;
    p->theta                      = 0.5f;
    p->G                          = 1.0f;
    p->useBox                     = 0;
    p->numShells                  = 1;
    p->ewald.numReplicaShells     = 1;
    p->ewald.lCut                 = 2.6;
    p->ewald.hCut                 = 2.8;
    p->ewald.alpha_scale          = 2.0;
    p->ewald.small_R_scale_factor = 3.0e-3;
    p->stackCapacity              = 0;
    p->groupTolerance             = 0.f;
    p->groupExtentRatio           = -1.f;
    p->multipole                  = RYO_MULTIPOLE_QUADRUPOLE;
}


namespace
{
//! phase marks of a timed solve: 0 start, 1 sorted, 2 tree, 3 upsweep, 4 traversal, 5 Ewald, 6 end
void mark(ryo_ctx* ctx, const ryo_solve_params* P, int i, cudaStream_t s)
{
    if (!P->timing) return;
    if (!ctx->phaseEvents[i]) RYO_CUDA(cudaEventCreate(&ctx->phaseEvents[i]));
    RYO_CUDA(cudaEventRecord(ctx->phaseEvents[i], s));
}
} // namespace

namespace
{
/*! host-memory pipeline of ryo_solve_host_f32: copies that overlap the solve on a second stream */
struct HostPipe
{
    cudaStream_t copy;       // the copy stream
    cudaEvent_t massReady;   // m and h on the device (recorded on the copy stream)
    float *hx, *hy, *hz;     // host: positions in SFC order (each may be null)
    float *hp, *hax, *hay, *haz;
    uint32_t* horder;        // host: original index of every sorted body (may be null)
    int chunks;              // traversal launches whose results are copied while the next one runs
};

//! record an event on @p from and make @p to wait for it
void streamAfter(ryo_ctx* ctx, cudaStream_t to, cudaStream_t from, int slot)
{
    if (!ctx->pipeEvents[slot]) RYO_CUDA(cudaEventCreateWithFlags(&ctx->pipeEvents[slot], cudaEventDisableTiming));
    RYO_CUDA(cudaEventRecord(ctx->pipeEvents[slot], from));
    RYO_CUDA(cudaStreamWaitEvent(to, ctx->pipeEvents[slot], 0));
}

void d2h(void* dst, const void* src, size_t bytes, cudaStream_t s)
{
    if (dst && bytes) RYO_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
}

/*! the device's address of the host array [@p h, @p h + n): non-null when the array is page-locked and mapped into
 *  this device's address space from its first to its last element, in one contiguous mapping */
float* mappedHostArray(float* h, size_t n)
{
    if (!h || n == 0) return nullptr;
    cudaPointerAttributes a0{}, a1{};
    cudaError_t e0 = cudaPointerGetAttributes(&a0, h);
    cudaError_t e1 = cudaPointerGetAttributes(&a1, h + (n - 1));
    if (e0 != cudaSuccess || e1 != cudaSuccess)
    {
        (void)cudaGetLastError(); // an address the runtime does not know is an answer here, not a failure
        return nullptr;
    }
    if (a0.type != cudaMemoryTypeHost || a1.type != cudaMemoryTypeHost || !a0.devicePointer || !a1.devicePointer)
        return nullptr;
    float* d0 = static_cast<float*>(a0.devicePointer);
    return static_cast<float*>(a1.devicePointer) == d0 + (n - 1) ? d0 : nullptr;
}

//! the device addresses of a host solve's four output arrays, if all four are mapped
bool mappedHostOutputs(const HostPipe* pipe, size_t n, float* out[4])
{
    float* h[4] = {pipe->hp, pipe->hax, pipe->hay, pipe->haz};
    for (int k = 0; k < 4; ++k)
        if (!(out[k] = mappedHostArray(h[k], n))) return false;
    return true;
}

/*! the fused single-system solve (ryo_solve_f32); with @p pipe, the host copies of ryo_solve_host_f32 are issued on
 *  its copy stream as soon as their data is final */
void solveSingle(ryo_ctx* ctx, const ryo_solve_params* P, float* x, float* y, float* z, float* m, float* h, float* vx,
                 float* vy, float* vz, size_t n, float* p, float* ax, float* ay, float* az, uint32_t* orderOut,
                 ryo_solve_stats* stats, cudaStream_t stream, const HostPipe* pipe)
{
    REQUIRE(x && y && z && m && h && p && ax && ay && az, "solve: null argument");
    REQUIRE(n > 0 && n < (size_t(1) << 32), "solve: body count must be in [1, 2^32)");
    REQUIRE(P->groupSize >= 1 && P->groupSize <= 64, "solve: groupSize must be in [1, 64]");
    REQUIRE(P->bucketSize >= 1 && P->theta > 0.f, "solve: bad bucketSize or theta");
    cudaStream_t s = stream;
    mark(ctx, P, 0, s);

    // box: given, or the cube enclosing the data (exact min/max)
    ryo_box_f32 box{};
    if (P->useBox) { box = P->box; }
    else
    {
        double* mm = ctx->scratch<double>("solve.bbox", 6, s);
        launchBoundingBox(x, y, z, n, mm, s);
        double hb[6];
        RYO_CUDA(cudaMemcpyAsync(hb, mm, sizeof(hb), cudaMemcpyDeviceToHost, s));
        RYO_CUDA(cudaStreamSynchronize(s));
        double ext = std::max({hb[1] - hb[0], hb[3] - hb[2], hb[5] - hb[4]});
        if (!(ext > 0)) ext = 1.0;
        for (int d = 0; d < 3; ++d)
        {
            box.limits[2 * d]     = float(hb[2 * d]);
            box.limits[2 * d + 1] = float(hb[2 * d] + ext);
            if (!(box.limits[2 * d + 1] >= float(hb[2 * d + 1])))
                box.limits[2 * d + 1] = std::nextafter(float(hb[2 * d + 1]), 3.4e38f);
            box.boundary[d] = RYO_BOUNDARY_OPEN;
        }
    }
    checkBox(box.limits);
    DevBox<float> dbox = boxOf(&box);
    bool periodic      = dbox.periodic;
    if (periodic)
    {
        checkEwald(&P->ewald);
        // the traversal's replica shells: a negative count would traverse nothing, and every further shell costs
        // (2 n + 1)^3 traversals (the batched solve and the engine refuse the same range)
        REQUIRE(P->numShells >= 0 && P->numShells <= 4, "solve: numShells must be in [0, 4] for a periodic box");
    }

    // keys and sort
    uint64_t* keys    = ctx->scratch<uint64_t>("solve.keys", n, s);
    uint64_t* keysAlt = ctx->scratch<uint64_t>("solve.keysAlt", n, s);
    uint32_t* ord     = ctx->scratch<uint32_t>("solve.order", n, s);
    uint32_t* ordAlt  = ctx->scratch<uint32_t>("solve.orderAlt", n, s);
    size_t tmpBytes   = sortTempBytes(n);
    void* tmp         = ctx->scratch<char>("solve.sorttmp", tmpBytes, s);
    launchKeys<float>(x, y, z, keys, n, dbox, false, s);
    bool alt = radixSortPairs(keys, ord, keysAlt, ordAlt, n, 0, 64, tmp, tmpBytes, &ctx->ctl->error,
                              s, true);
    const uint64_t* sorted = alt ? keysAlt : keys;
    const uint32_t* order  = alt ? ordAlt : ord;

    if (orderOut)
        RYO_CUDA(cudaMemcpyAsync(orderOut, order, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    // permute every per-particle array through 32-byte body records, writing the traversal's packed sources and
    // targets on the way. A host solve's masses and softenings arrive on the copy stream meanwhile: it builds the
    // leaves and links first, which need only the sorted keys, and permutes after them.
    float4* rec      = ctx->scratch<float4>("solve.bodyRecords", 2 * n, s);
    float4* xyzm     = ctx->scratch<float4>("solve.xyzm", n, s);
    float4* xyzh     = ctx->scratch<float4>("solve.xyzh", n, s);
    uint32_t* hRange = ctx->scratch<uint32_t>("solve.softeningRange", 4, s);
    auto permute     = [&]()
    {
        if (pipe) RYO_CUDA(cudaStreamWaitEvent(s, pipe->massReady, 0));
        launchPackRecords(x, y, z, m, h, vx, vy, vz, n, rec, s);
        launchGatherRecords(order, rec, n, x, y, z, m, h, vx, vy, vz, xyzm, xyzh, hRange, s);
        if (pipe)
        {
            // the sorted positions are final: copy them out while the upsweep and the traversal run
            streamAfter(ctx, pipe->copy, s, 0);
            d2h(pipe->hx, x, n * sizeof(float), pipe->copy);
            d2h(pipe->hy, y, n * sizeof(float), pipe->copy);
            d2h(pipe->hz, z, n * sizeof(float), pipe->copy);
        }
    };
    if (pipe)
    {
        // the permutation is final
        streamAfter(ctx, pipe->copy, s, 0);
        d2h(pipe->horder, order, n * sizeof(uint32_t), pipe->copy);
    }
    else permute();
    mark(ctx, P, 1, s);

    // leaves, links
    int cap           = int(std::min<size_t>(n / 2 + 64, size_t(1) << 30));
    uint64_t* leaves  = ctx->scratch<uint64_t>("solve.leaves", size_t(cap) + 1, s);
    uint32_t* counts  = ctx->scratch<uint32_t>("solve.counts", cap, s);
    uint32_t* layout  = ctx->scratch<uint32_t>("solve.layout", size_t(cap) + 1, s);
    int nl = buildLeaves(ctx, sorted, n, P->bucketSize, leaves, counts, layout, cap, s);
    if (nl > cap)
    {
        cap    = nl;
        leaves = ctx->scratch<uint64_t>("solve.leaves", size_t(cap) + 1, s);
        counts = ctx->scratch<uint32_t>("solve.counts", cap, s);
        layout = ctx->scratch<uint32_t>("solve.layout", size_t(cap) + 1, s);
        nl     = buildLeaves(ctx, sorted, n, P->bucketSize, leaves, counts, layout, cap, s);
    }
    int ni = (nl - 1) / 7, nn = nl + ni;
    OctreeArrays oct;
    oct.prefixes       = ctx->scratch<uint64_t>("solve.prefixes", nn, s);
    oct.childOffsets   = ctx->scratch<int>("solve.childOffsets", size_t(nn) + 1, s);
    oct.parents        = ctx->scratch<int>("solve.parents", std::max(1, (nn - 1) / 8), s);
    oct.internalToLeaf = ctx->scratch<int>("solve.internalToLeaf", nn, s);
    oct.leafToInternal = ctx->scratch<int>("solve.leafToInternal", nn, s);
    oct.d_levelRange   = ctx->scratch<int>("solve.levelRange", kMaxLevel + 2, s);
    int levelRange[kMaxLevel + 2];
    linkOctree(ctx, leaves, nl, oct, levelRange, s);
    if (pipe) permute();

    mark(ctx, P, 2, s);
    // fused upsweep: node records + FP64 root expansion
    REQUIRE(P->multipole == RYO_MULTIPOLE_QUADRUPOLE || P->multipole == RYO_MULTIPOLE_MDQ,
            "solve: unknown multipole type");
    NodeRecord* records = ctx->scratch<NodeRecord>("solve.records", nn, s);
    double* root        = ctx->scratch<double>("solve.root", 16, s);
    float4* dipoles     = P->multipole == RYO_MULTIPOLE_MDQ
                              ? ctx->scratch<float4>("solve.dipoles", nn, s)
                              : nullptr;
    launchFusedUpsweep(ctx, xyzm, nl, nn, layout, oct.leafToInternal + ni, oct.childOffsets,
                       oct.parents, oct.prefixes, 1.0f / P->theta, dbox, records, nullptr, nullptr,
                       root, s, nullptr, 0, nullptr, dipoles, 0, levelRange);

    mark(ctx, P, 3, s);
    // groups and traversal
    uint32_t numGroups = uint32_t((n + P->groupSize - 1) / P->groupSize);
    uint32_t* groups   = nullptr;
    if (P->groupTolerance > 0.f)
    {
        // spatial groups (the reference's production grouping); at most one group per body.
        // No interaction radius: h here is the gravitational softening, not the SPH smoothing
        // length the grouping's radius criterion was made for, and a tiny softening would split
        // every pair of bodies.
        REQUIRE(P->groupSize == 32 || P->groupSize == 64,
                "solve: spatial groups need groupSize 32 or 64");
        groups      = ctx->scratch<uint32_t>("solve.groups", n + 2, s);
        float ratio = P->groupExtentRatio < 0.f ? defaultExtentRatio() : P->groupExtentRatio;
        numGroups   = computeGroupSplits(ctx, 0, uint32_t(n), x, y, z, nullptr, leaves, nl, layout, dbox,
                                         P->groupSize, P->groupTolerance, ratio, groups,
                                         uint32_t(n + 2), s);
    }
    else
    {
        groups = ctx->scratch<uint32_t>("solve.groups", size_t(numGroups) + 1, s);
        launchFixedGroups(0, uint32_t(n), P->groupSize, groups, s);
    }
    // a host solve of an open system whose output arrays are page-locked and mapped stores the traversal's results
    // straight into them: the results cross the link while the traversal runs, and no download follows it
    float* mapped[4]  = {nullptr, nullptr, nullptr, nullptr};
    const bool direct = pipe && !periodic && mappedHostOutputs(pipe, n, mapped);
    if (!direct)
        for (float* a : {p, ax, ay, az})
            RYO_CUDA(cudaMemsetAsync(a, 0, n * sizeof(float), s));
    TraverseLaunch t{};
    t.groupStart    = groups;
    t.groupEnd      = groups + 1;
    t.numGroups     = int(numGroups);
    t.initNode      = nn == 1 ? 0 : 1;
    t.numNodes      = nn;
    t.nodes         = records;
    t.tgtXYZH       = xyzh;
    t.tgtM          = m;
    t.srcXYZM       = xyzm;
    t.srcH          = h;
    t.G             = P->G;
    t.numShells     = periodic ? P->numShells : 0;
    for (int d = 0; d < 3; ++d)
        t.boxL[d] = dbox.len[d];
    t.p  = direct ? mapped[0] : p;
    t.ax = direct ? mapped[1] : ax;
    t.ay = direct ? mapped[2] : ay;
    t.az = direct ? mapped[3] : az;
    t.overwrite     = direct ? 1 : 0;
    t.stackCapacity = P->stackCapacity;
    t.dipoles       = dipoles;
    t.softeningRange = hRange;
    t.massRange      = dipoles ? nullptr : hRange + 2; // signed-mass expansions keep the per-source mass
    uint32_t* gm2p  = ctx->scratch<uint32_t>("solve.groupM2P", numGroups, s);
    uint32_t* gp2p  = ctx->scratch<uint32_t>("solve.groupP2P", numGroups, s);
    RYO_CUDA(cudaMemsetAsync(gm2p, 0, sizeof(uint32_t) * numGroups, s));
    RYO_CUDA(cudaMemsetAsync(gp2p, 0, sizeof(uint32_t) * numGroups, s));
    t.groupM2P      = gm2p;
    t.groupP2P      = gp2p;
    double pot = 0;
    // otherwise, a host solve of an open system with fixed groups traverses in chunks of groups and copies each
    // chunk's results to the host while the next chunk runs
    const bool chunked = pipe && !direct && pipe->chunks > 1 && !periodic && !(P->groupTolerance > 0.f) &&
                         numGroups >= uint32_t(pipe->chunks);
    if (!chunked) runTraversal(ctx, t, s, &pot);
    else
    {
        unsigned long long acc[5] = {0, 0, 0, 0, 0};
        uint64_t retries          = 0;
        for (int c = 0; c < pipe->chunks; ++c)
        {
            uint32_t g0 = uint32_t(uint64_t(numGroups) * uint64_t(c) / uint64_t(pipe->chunks));
            uint32_t g1 = uint32_t(uint64_t(numGroups) * uint64_t(c + 1) / uint64_t(pipe->chunks));
            TraverseLaunch tc = t;
            tc.groupStart     = groups + g0;
            tc.groupEnd       = groups + g0 + 1;
            tc.numGroups      = int(g1 - g0);
            tc.groupM2P       = gm2p + g0;
            tc.groupP2P       = gp2p + g0;
            tc.balanceGroups  = numGroups;
            double cp         = 0;
            runTraversal(ctx, tc, s, &cp);
            pot += cp;
            acc[kSumP2P] += ctx->hostStats[kSumP2P];
            acc[kSumM2P] += ctx->hostStats[kSumM2P];
            for (int k : {int(kMaxP2P), int(kMaxM2P), int(kMaxStack)})
                acc[k] = std::max(acc[k], ctx->hostStats[k]);
            retries += ctx->retries;
            // fixed groups: group k holds bodies [k G, min((k + 1) G, n))
            size_t b0 = size_t(g0) * P->groupSize, b1 = std::min(size_t(g1) * P->groupSize, n);
            streamAfter(ctx, pipe->copy, s, 0);
            d2h(pipe->hp + b0, p + b0, (b1 - b0) * sizeof(float), pipe->copy);
            d2h(pipe->hax + b0, ax + b0, (b1 - b0) * sizeof(float), pipe->copy);
            d2h(pipe->hay + b0, ay + b0, (b1 - b0) * sizeof(float), pipe->copy);
            d2h(pipe->haz + b0, az + b0, (b1 - b0) * sizeof(float), pipe->copy);
        }
        for (int k = 0; k < 5; ++k)
            ctx->hostStats[k] = acc[k];
        ctx->retries = retries;
    }
    double energy = 0.5 * double(P->G) * pot;
    mark(ctx, P, 4, s);

    if (periodic)
    {
        if (!(dbox.len[0] == dbox.len[1] && dbox.len[1] == dbox.len[2]))
            throw ApiError{RYO_ERR_NOT_CUBIC, "solve: Ewald needs a cubic periodic box"};
        double hr[16];
        RYO_CUDA(cudaMemcpyAsync(hr, root, sizeof(double) * 11, cudaMemcpyDeviceToHost, s));
        RYO_CUDA(cudaStreamSynchronize(s));
        EwaldHost e = ewaldSetup(hr + 3, hr, P->ewald.numReplicaShells, double(dbox.len[0]),
                                 P->ewald.lCut, P->ewald.hCut, P->ewald.alpha_scale,
                                 P->ewald.small_R_scale_factor);
        double* ep = &ctx->ctl->ewaldPotential;
        RYO_CUDA(cudaMemsetAsync(ep, 0, sizeof(double), s));
        launchEwaldGroups(e, groups, groups + 1, numGroups, x, y, z, m, P->G, p, ax, ay, az, ep, s);
        double he = 0;
        RYO_CUDA(cudaMemcpyAsync(&he, ep, sizeof(double), cudaMemcpyDeviceToHost, s));
        RYO_CUDA(cudaStreamSynchronize(s));
        energy += 0.5 * double(P->G) * he;
    }
    if (pipe && !chunked && !direct)
    {
        streamAfter(ctx, pipe->copy, s, 0);
        d2h(pipe->hp, p, n * sizeof(float), pipe->copy);
        d2h(pipe->hax, ax, n * sizeof(float), pipe->copy);
        d2h(pipe->hay, ay, n * sizeof(float), pipe->copy);
        d2h(pipe->haz, az, n * sizeof(float), pipe->copy);
    }
    mark(ctx, P, 5, s);
    mark(ctx, P, 6, s);
    float ms[6] = {0, 0, 0, 0, 0, 0};
    if (P->timing)
    {
        RYO_CUDA(cudaEventSynchronize(ctx->phaseEvents[6]));
        for (int i = 0; i < 5; ++i)
            RYO_CUDA(cudaEventElapsedTime(&ms[i], ctx->phaseEvents[i], ctx->phaseEvents[i + 1]));
        RYO_CUDA(cudaEventElapsedTime(&ms[5], ctx->phaseEvents[0], ctx->phaseEvents[6]));
    }
    {
        auto& st      = ctx->solveState;
        st.valid      = true;
        st.nodes      = records;
        st.xyzm       = xyzm;
        st.srcH       = h;
        st.numNodes   = nn;
        st.groupSize  = P->groupSize;
        st.G          = P->G;
        st.periodic   = periodic ? 1 : 0;
        st.numShells  = periodic ? P->numShells : 0;
        st.box        = box;
        st.ewald      = P->ewald;
        st.dipoles    = dipoles;
        st.massRange  = dipoles ? nullptr : hRange + 2;
        ryo_solve_arrays& a = ctx->lastSolve;
        a.numLeaves         = nl;
        a.numNodes          = nn;
        a.numGroups         = int(numGroups);
        a.sortedKeys        = sorted;
        a.order             = order;
        a.leaves            = leaves;
        a.layout            = layout;
        a.prefixes          = oct.prefixes;
        a.childOffsets      = oct.childOffsets;
        a.internalToLeaf    = oct.internalToLeaf;
        a.leafToInternal    = oct.leafToInternal;
        a.parents           = oct.parents;
        a.nodeData          = reinterpret_cast<const float*>(records);
        a.groups            = groups;
        a.groupM2P          = gm2p;
        a.groupP2P          = gp2p;
        a.dipoles           = reinterpret_cast<const float*>(dipoles);
        for (int i = 0; i < kMaxLevel + 2; ++i)
            a.levelRange[i] = levelRange[i];
        double hr[11];
        RYO_CUDA(cudaMemcpyAsync(hr, root, sizeof(hr), cudaMemcpyDeviceToHost, s));
        RYO_CUDA(cudaStreamSynchronize(s));
        for (int i = 0; i < 3; ++i)
            a.rootCenter[i] = hr[i];
        for (int i = 0; i < 8; ++i)
            a.rootMultipole[i] = hr[3 + i];
        for (int i = 0; i < 11; ++i)
            st.root[i] = hr[i];
    }
    if (ctx->hostStats[kMaxP2P] == 0xFFFFFFFFull)
        throw ApiError{RYO_ERR_STACK_OVERFLOW_UNSPLITTABLE, "solve: a single target overflowed"};
    checkDeviceError(ctx, s);
    if (stats)
    {
        stats->numLeaves       = nl;
        stats->numNodes        = nn;
        stats->numGroups       = int(numGroups);
        stats->sumP2P          = ctx->hostStats[kSumP2P];
        stats->maxP2P          = ctx->hostStats[kMaxP2P];
        stats->sumM2P          = ctx->hostStats[kSumM2P];
        stats->maxM2P          = ctx->hostStats[kMaxM2P];
        stats->maxStack        = ctx->hostStats[kMaxStack];
        stats->retries         = ctx->retries;
        stats->potentialEnergy = energy;
        for (int i = 0; i < 6; ++i)
        {
            stats->box[i] = box.limits[i];
            stats->ms[i]  = ms[i];
        }
    }
}
} // namespace

extern "C" ryo_status ryo_solve_f32(ryo_ctx_t* ctx, const ryo_solve_params* P, float* x, float* y, float* z, float* m,
                                    float* h, float* vx, float* vy, float* vz, size_t n, float* p, float* ax,
                                    float* ay, float* az, uint32_t* orderOut, ryo_solve_stats* stats,
                                    ryo_stream_t stream)
{
    if (!ctx || !P) return RYO_ERR_BAD_ARG;
    return guardedCtx(ctx,
                   [&] { solveSingle(ctx, P, x, y, z, m, h, vx, vy, vz, n, p, ax, ay, az, orderOut, stats, stream,
                                     nullptr); });
}

extern "C" ryo_status ryo_solve_host_f32(ryo_ctx_t* ctx, const ryo_solve_params* P, const float* x, const float* y,
                                         const float* z, const float* m, const float* h, size_t n, float* xs,
                                         float* ys, float* zs, float* p, float* ax, float* ay, float* az,
                                         uint32_t* order, ryo_solve_stats* stats, ryo_stream_t stream)
{
    if (!ctx || !P) return RYO_ERR_BAD_ARG;
    return guardedCtx(ctx,
                   [&]
                   {
                       REQUIRE(x && y && z && m && h && p && ax && ay && az, "solve_host: null argument");
                       REQUIRE(n > 0 && n < (size_t(1) << 32), "solve_host: body count must be in [1, 2^32)");
                       cudaStream_t s = stream;
                       if (!ctx->copyStream)
                           RYO_CUDA(cudaStreamCreateWithFlags(&ctx->copyStream, cudaStreamNonBlocking));
                       float* d[9];
                       const char* names[9] = {"host.x", "host.y", "host.z", "host.m", "host.h",
                                               "host.p", "host.ax", "host.ay", "host.az"};
                       for (int k = 0; k < 9; ++k)
                           d[k] = ctx->scratch<float>(names[k], n, s);
                       // the copy stream starts after the work already queued on s, which may still use the buffers
                       streamAfter(ctx, ctx->copyStream, s, 1);
                       const size_t bytes = n * sizeof(float);
                       RYO_CUDA(cudaMemcpyAsync(d[0], x, bytes, cudaMemcpyHostToDevice, s));
                       RYO_CUDA(cudaMemcpyAsync(d[1], y, bytes, cudaMemcpyHostToDevice, s));
                       RYO_CUDA(cudaMemcpyAsync(d[2], z, bytes, cudaMemcpyHostToDevice, s));
                       RYO_CUDA(cudaMemcpyAsync(d[3], m, bytes, cudaMemcpyHostToDevice, ctx->copyStream));
                       RYO_CUDA(cudaMemcpyAsync(d[4], h, bytes, cudaMemcpyHostToDevice, ctx->copyStream));
                       RYO_CUDA(cudaEventRecord(ctx->pipeEvents[1], ctx->copyStream));
                       HostPipe pipe{ctx->copyStream, ctx->pipeEvents[1], xs, ys, zs, p, ax, ay, az, order, 8};
                       solveSingle(ctx, P, d[0], d[1], d[2], d[3], d[4], nullptr, nullptr, nullptr, n, d[5], d[6],
                                   d[7], d[8], nullptr, stats, s, &pipe);
                       RYO_CUDA(cudaStreamSynchronize(ctx->copyStream));
                       RYO_CUDA(cudaStreamSynchronize(s));
                   });
}

//! octree levels taken by the system index in batched keys: the smallest L >= 1 with 8^L >= numSystems
static int batchSystemLevel(int numSystems)
{
    int L = 1;
    while ((size_t(1) << (3 * L)) < size_t(numSystems))
        ++L;
    return L;
}

extern "C" ryo_status ryo_solve_batch_f32(ryo_ctx_t* ctx, const ryo_solve_params* P, const ryo_system* systems,
                                          int numSystems, float* x, float* y, float* z, float* m, float* h, float* vx,
                                          float* vy, float* vz, size_t n, float* p, float* ax, float* ay, float* az,
                                          uint32_t* orderOut, double* energies, float* boxesOut,
                                          ryo_solve_stats* stats, ryo_stream_t stream)
{
    if (!ctx || !P) return RYO_ERR_BAD_ARG;
    return guardedCtx(ctx,
                   [&]
                   {
                       REQUIRE(systems && numSystems >= 1 && numSystems <= RYO_BATCH_MAX_SYSTEMS,
                               "solve_batch: numSystems must be in [1, RYO_BATCH_MAX_SYSTEMS]");
                       REQUIRE(x && y && z && m && h && p && ax && ay && az, "solve_batch: null argument");
                       REQUIRE(n > 0 && n < (size_t(1) << 32), "solve_batch: body count must be in [1, 2^32)");
                       REQUIRE(P->groupSize >= 1 && P->groupSize <= 64, "solve_batch: groupSize must be in [1, 64]");
                       REQUIRE(P->bucketSize >= 1 && P->theta > 0.f, "solve_batch: bad bucketSize or theta");
                       cudaStream_t s      = stream;
                       const uint32_t ns   = uint32_t(numSystems);
                       const int sysLevel  = batchSystemLevel(numSystems);
                       ctx->solveState.valid = false; // the solve buffers are about to be reused
                       std::vector<uint64_t> first(ns + 1);
                       std::vector<int> useGiven(ns), shells(ns);
                       std::vector<DevBox<float>> hbox(ns);
                       std::vector<uint32_t> groupOffset(ns + 1);
                       uint64_t expect = 0, groups = 0;
                       for (uint32_t k = 0; k < ns; ++k)
                       {
                           const ryo_system& sy = systems[k];
                           REQUIRE(sy.firstBody == expect && sy.numBodies >= 1,
                                   "solve_batch: systems must tile the body arrays in order, none empty");
                           first[k]       = expect;
                           groupOffset[k] = uint32_t(groups);
                           expect += sy.numBodies;
                           groups += (sy.numBodies + P->groupSize - 1) / P->groupSize;
                           useGiven[k] = sy.useBox ? 1 : 0;
                           shells[k]   = 0;
                           if (sy.useBox)
                           {
                               checkBox(sy.box.limits);
                               hbox[k] = boxOf(&sy.box);
                               if (hbox[k].periodic)
                               {
                                   if (!(hbox[k].len[0] == hbox[k].len[1] && hbox[k].len[1] == hbox[k].len[2]))
                                       throw ApiError{RYO_ERR_NOT_CUBIC,
                                                      "solve_batch: Ewald needs a cubic periodic box"};
                                   REQUIRE(sy.numShells >= 0 && sy.numShells <= 4, "solve_batch: numShells in [0, 4]");
                                   checkEwald(&P->ewald);
                                   shells[k] = sy.numShells;
                               }
                           }
                       }
                       REQUIRE(expect == n, "solve_batch: the systems' bodies must add up to n");
                       first[ns]       = expect;
                       groupOffset[ns] = uint32_t(groups);
                       const uint32_t numGroups = uint32_t(groups);
                       mark(ctx, P, 0, s);

                       // per-system tables
                       uint64_t* dFirst   = ctx->scratch<uint64_t>("batch.first", ns + 1, s);
                       int* dUseGiven     = ctx->scratch<int>("batch.useGiven", ns, s);
                       int* dShells       = ctx->scratch<int>("batch.shells", ns, s);
                       DevBox<float>* dBx = ctx->scratch<DevBox<float>>("batch.boxes", ns, s);
                       uint32_t* dGOff    = ctx->scratch<uint32_t>("batch.groupOffset", ns + 1, s);
                       uint32_t* dMM      = ctx->scratch<uint32_t>("batch.minmax", 6 * size_t(ns), s);
                       float* dLimits     = ctx->scratch<float>("batch.limits", 6 * size_t(ns), s);
                       RYO_CUDA(cudaMemcpyAsync(dFirst, first.data(), sizeof(uint64_t) * (ns + 1),
                                                cudaMemcpyHostToDevice, s));
                       RYO_CUDA(cudaMemcpyAsync(dUseGiven, useGiven.data(), sizeof(int) * ns, cudaMemcpyHostToDevice,
                                                s));
                       RYO_CUDA(cudaMemcpyAsync(dShells, shells.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, s));
                       RYO_CUDA(cudaMemcpyAsync(dBx, hbox.data(), sizeof(DevBox<float>) * ns, cudaMemcpyHostToDevice,
                                                s));
                       RYO_CUDA(cudaMemcpyAsync(dGOff, groupOffset.data(), sizeof(uint32_t) * (ns + 1),
                                                cudaMemcpyHostToDevice, s));
                       launchBatchBoxes(x, y, z, n, dFirst, ns, dUseGiven, dMM, dBx, dLimits, s);

                       // system-prefixed keys, one sort for all systems, permute every per-body array
                       uint64_t* keys    = ctx->scratch<uint64_t>("solve.keys", n, s);
                       uint64_t* keysAlt = ctx->scratch<uint64_t>("solve.keysAlt", n, s);
                       uint32_t* ord     = ctx->scratch<uint32_t>("solve.order", n, s);
                       uint32_t* ordAlt  = ctx->scratch<uint32_t>("solve.orderAlt", n, s);
                       size_t tmpBytes   = sortTempBytes(n);
                       void* tmp         = ctx->scratch<char>("solve.sorttmp", tmpBytes, s);
                       launchBatchKeys(x, y, z, n, dFirst, ns, dBx, sysLevel, keys, ctx->smCount, s);
                       bool alt = radixSortPairs(keys, ord, keysAlt, ordAlt, n, 0, 64, tmp, tmpBytes, &ctx->ctl->error,
                                                 s, true);
                       const uint64_t* sorted = alt ? keysAlt : keys;
                       const uint32_t* order  = alt ? ordAlt : ord;
                       float4* rec            = ctx->scratch<float4>("solve.bodyRecords", 2 * n, s);
                       float4* xyzm           = ctx->scratch<float4>("solve.xyzm", n, s);
                       float4* xyzh           = ctx->scratch<float4>("solve.xyzh", n, s);
                       launchPackRecords(x, y, z, m, h, vx, vy, vz, n, rec, s);
                       uint32_t* hRange       = ctx->scratch<uint32_t>("solve.softeningRange", 4, s);
                       launchGatherRecords(order, rec, n, x, y, z, m, h, vx, vy, vz, xyzm, xyzh, hRange, s);
                       if (orderOut)
                           RYO_CUDA(cudaMemcpyAsync(orderOut, order, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
                       mark(ctx, P, 1, s);

                       // one tree over all systems: leaves holding bodies lie at or below the system level
                       int cap          = int(std::min<size_t>(n / 2 + 64 + 8 * size_t(ns), size_t(1) << 30));
                       uint64_t* leaves = ctx->scratch<uint64_t>("solve.leaves", size_t(cap) + 1, s);
                       uint32_t* counts = ctx->scratch<uint32_t>("solve.counts", cap, s);
                       uint32_t* layout = ctx->scratch<uint32_t>("solve.layout", size_t(cap) + 1, s);
                       int nl = buildLeaves(ctx, sorted, n, P->bucketSize, leaves, counts, layout, cap, s,
                                            unsigned(sysLevel));
                       if (nl > cap)
                       {
                           cap    = nl;
                           leaves = ctx->scratch<uint64_t>("solve.leaves", size_t(cap) + 1, s);
                           counts = ctx->scratch<uint32_t>("solve.counts", cap, s);
                           layout = ctx->scratch<uint32_t>("solve.layout", size_t(cap) + 1, s);
                           nl     = buildLeaves(ctx, sorted, n, P->bucketSize, leaves, counts, layout, cap, s,
                                                unsigned(sysLevel));
                       }
                       int ni = (nl - 1) / 7, nn = nl + ni;
                       OctreeArrays oct;
                       oct.prefixes       = ctx->scratch<uint64_t>("solve.prefixes", nn, s);
                       oct.childOffsets   = ctx->scratch<int>("solve.childOffsets", size_t(nn) + 1, s);
                       oct.parents        = ctx->scratch<int>("solve.parents", std::max(1, (nn - 1) / 8), s);
                       oct.internalToLeaf = ctx->scratch<int>("solve.internalToLeaf", nn, s);
                       oct.leafToInternal = ctx->scratch<int>("solve.leafToInternal", nn, s);
                       oct.d_levelRange   = ctx->scratch<int>("solve.levelRange", kMaxLevel + 2, s);
                       int levelRange[kMaxLevel + 2];
                       linkOctree(ctx, leaves, nl, oct, levelRange, s);
                       mark(ctx, P, 2, s);

                       // fused upsweep with each system's box; FP64 expansions of the system roots
                       REQUIRE(P->multipole == RYO_MULTIPOLE_QUADRUPOLE || P->multipole == RYO_MULTIPOLE_MDQ,
                               "solve_batch: unknown multipole type");
                       NodeRecord* records = ctx->scratch<NodeRecord>("solve.records", nn, s);
                       double* sysRoots    = ctx->scratch<double>("batch.roots", 11 * size_t(ns), s);
                       float4* dipoles     = P->multipole == RYO_MULTIPOLE_MDQ
                                                 ? ctx->scratch<float4>("solve.dipoles", nn, s)
                                                 : nullptr;
                       DevBox<float> unused = hbox[0];
                       launchFusedUpsweep(ctx, xyzm, nl, nn, layout, oct.leafToInternal + ni, oct.childOffsets,
                                          oct.parents, oct.prefixes, 1.0f / P->theta, unused, records, nullptr, nullptr,
                                          nullptr, s, dBx, sysLevel, sysRoots, dipoles, ns, levelRange);
                       mark(ctx, P, 3, s);

                       // groups inside systems, system roots, traversal
                       uint32_t* gStart = ctx->scratch<uint32_t>("batch.gstart", std::max(numGroups, 1u), s);
                       uint32_t* gEnd   = ctx->scratch<uint32_t>("batch.gend", std::max(numGroups, 1u), s);
                       uint32_t* gSys   = ctx->scratch<uint32_t>("batch.gsys", std::max(numGroups, 1u), s);
                       launchBatchGroups(numGroups, dFirst, dGOff, ns, P->groupSize, gStart, gEnd, gSys, s);
                       // traversal groups: the fixed windows, or their spatial splits within each system
                       uint32_t travGroups = numGroups;
                       uint32_t* tStart    = gStart;
                       uint32_t* tEnd      = gEnd;
                       uint32_t* tSys      = gSys;
                       if (P->groupTolerance > 0.f)
                       {
                           REQUIRE(P->groupSize == 32 || P->groupSize == 64,
                                   "solve_batch: spatial groups need groupSize 32 or 64");
                           uint32_t* sg   = ctx->scratch<uint32_t>("batch.sgroups", n + 2, s);
                           uint32_t* sSys = ctx->scratch<uint32_t>("batch.sgsys", n + 1, s);
                           float ratio    = P->groupExtentRatio < 0.f ? defaultExtentRatio() : P->groupExtentRatio;
                           travGroups = computeGroupSplitsBatch(ctx, gStart, gEnd, gSys, numGroups, dBx, sysLevel, x, y,
                                                                z, leaves, nl, layout, P->groupSize,
                                                                P->groupTolerance, ratio, sg, sSys, uint32_t(n + 2), s);
                           tStart = sg;
                           tEnd   = sg + 1;
                           tSys   = sSys;
                       }
                       SysTrav* dTrav   = ctx->scratch<SysTrav>("batch.trav", ns, s);
                       int* dRootNode   = ctx->scratch<int>("batch.rootNode", ns, s);
                       unsigned int* rootErr = ctx->ctl->counters + 4;
                       RYO_CUDA(cudaMemsetAsync(rootErr, 0, sizeof(unsigned int), s));
                       launchBatchRoots(ns, oct.prefixes, levelRange[sysLevel], levelRange[sysLevel + 1],
                                        oct.childOffsets, sysLevel, dBx, dShells, dTrav, dRootNode, rootErr, s);
                       // the mass range only where quadrupoles are summed (signed-mass expansions keep the
                       // per-source mass)
                       launchBatchSofteningRange(h, dipoles ? nullptr : m, dFirst, ns, dTrav, s);
                       double* sysPot = ctx->scratch<double>("batch.pot", 2 * size_t(ns), s); // tree, Ewald
                       RYO_CUDA(cudaMemsetAsync(sysPot, 0, sizeof(double) * 2 * ns, s));
                       for (float* a : {p, ax, ay, az})
                           RYO_CUDA(cudaMemsetAsync(a, 0, n * sizeof(float), s));
                       TraverseLaunch t{};
                       t.groupStart    = tStart;
                       t.groupEnd      = tEnd;
                       t.numGroups     = int(travGroups);
                       t.initNode      = 1;
                       t.numNodes      = nn;
                       t.nodes         = records;
                       t.tgtXYZH       = xyzh;
                       t.tgtM          = m;
                       t.srcXYZM       = xyzm;
                       t.srcH          = h;
                       t.G             = P->G;
                       t.p             = p;
                       t.ax            = ax;
                       t.ay            = ay;
                       t.az            = az;
                       t.stackCapacity = P->stackCapacity;
                       t.groupSys      = tSys;
                       t.dipoles       = dipoles;
                       t.softeningRange = hRange;
                       t.systems       = dTrav;
                       t.sysPotential  = sysPot;
                       double pot      = 0;
                       runTraversal(ctx, t, s, &pot);
                       mark(ctx, P, 4, s);

                       // Ewald for the periodic systems, one launch per periodic system
                       std::vector<double> hroots;
                       for (uint32_t k = 0; k < ns; ++k)
                       {
                           if (!(useGiven[k] && hbox[k].periodic)) continue;
                           if (hroots.empty())
                           {
                               hroots.resize(11 * size_t(ns));
                               RYO_CUDA(cudaMemcpyAsync(hroots.data(), sysRoots, sizeof(double) * 11 * ns,
                                                        cudaMemcpyDeviceToHost, s));
                               RYO_CUDA(cudaStreamSynchronize(s));
                           }
                           const double* r = hroots.data() + 11 * size_t(k);
                           EwaldHost e = ewaldSetup(r + 3, r, P->ewald.numReplicaShells, double(hbox[k].len[0]),
                                                    P->ewald.lCut, P->ewald.hCut, P->ewald.alpha_scale,
                                                    P->ewald.small_R_scale_factor);
                           uint32_t g0 = groupOffset[k], g1 = groupOffset[k + 1];
                           launchEwaldGroups(e, gStart + g0, gEnd + g0, g1 - g0, x, y, z, m, P->G, p, ax, ay, az,
                                             sysPot + ns + k, s);
                       }
                       mark(ctx, P, 5, s);
                       mark(ctx, P, 6, s);

                       std::vector<double> hp(2 * size_t(ns));
                       RYO_CUDA(cudaMemcpyAsync(hp.data(), sysPot, sizeof(double) * 2 * ns, cudaMemcpyDeviceToHost, s));
                       unsigned int herr = 0;
                       RYO_CUDA(cudaMemcpyAsync(&herr, rootErr, sizeof(herr), cudaMemcpyDeviceToHost, s));
                       std::vector<float> hl;
                       if (boxesOut)
                       {
                           hl.resize(6 * size_t(ns));
                           RYO_CUDA(cudaMemcpyAsync(hl.data(), dLimits, sizeof(float) * 6 * ns, cudaMemcpyDeviceToHost,
                                                    s));
                       }
                       RYO_CUDA(cudaStreamSynchronize(s));
                       if (herr) throw ApiError{RYO_ERR_CUDA, "solve_batch: a system root is missing from the tree"};
                       double total = 0;
                       for (uint32_t k = 0; k < ns; ++k)
                       {
                           double e = 0.5 * double(P->G) * (hp[k] + hp[ns + k]);
                           total += e;
                           if (energies) energies[k] = e;
                           if (boxesOut)
                               for (int d = 0; d < 6; ++d)
                                   boxesOut[6 * k + d] = useGiven[k] ? systems[k].box.limits[d] : hl[6 * k + d];
                       }
                       float ms[6] = {0, 0, 0, 0, 0, 0};
                       if (P->timing)
                       {
                           RYO_CUDA(cudaEventSynchronize(ctx->phaseEvents[6]));
                           for (int i = 0; i < 5; ++i)
                               RYO_CUDA(cudaEventElapsedTime(&ms[i], ctx->phaseEvents[i], ctx->phaseEvents[i + 1]));
                           RYO_CUDA(cudaEventElapsedTime(&ms[5], ctx->phaseEvents[0], ctx->phaseEvents[6]));
                       }
                       if (stats)
                       {
                           stats->numLeaves       = nl;
                           stats->numNodes        = nn;
                           stats->numGroups       = int(travGroups);
                           stats->sumP2P          = ctx->hostStats[kSumP2P];
                           stats->maxP2P          = ctx->hostStats[kMaxP2P];
                           stats->sumM2P          = ctx->hostStats[kSumM2P];
                           stats->maxM2P          = ctx->hostStats[kMaxM2P];
                           stats->maxStack        = ctx->hostStats[kMaxStack];
                           stats->retries         = ctx->retries;
                           stats->potentialEnergy = total;
                           for (int d = 0; d < 6; ++d)
                               stats->box[d] = 0.f;
                           for (int i = 0; i < 6; ++i)
                               stats->ms[i] = ms[i];
                       }
                   });
}

extern "C" ryo_status ryo_ewald_targets_f64(ryo_ctx_t* ctx, const int64_t* targets, size_t numTargets,
                                            const float* x, const float* y, const float* z, const float* m,
                                            size_t numBodies, double L, const ryo_ewald_settings* settings, double G,
                                            double* pot, double* ax, double* ay, double* az, ryo_stream_t stream)
{
    if (!ctx) return RYO_ERR_BAD_ARG;
    return guardedCtx(ctx,
                   [&]
                   {
                       checkEwald(settings);
                       REQUIRE(L > 0, "ewald_targets: bad box");
                       REQUIRE(numTargets == 0 || (targets && x && y && z && m && pot && ax && ay && az),
                               "ewald_targets: null argument");
                       launchEwaldTargetsF64(ctx, targets, numTargets, x, y, z, m, numBodies, L,
                                             settings->numReplicaShells, settings->lCut, settings->hCut,
                                             settings->alpha_scale, settings->small_R_scale_factor, G, pot, ax, ay, az,
                                             stream);
                   });
}

namespace
{
//! sorted target copies: packed (x, y, z, h), mass, and x, y, z, m again as separate arrays for the Ewald kernel
__global__ void packTargets(const uint32_t* __restrict__ order, const float* __restrict__ x,
                            const float* __restrict__ y, const float* __restrict__ z, const float* __restrict__ m,
                            const float* __restrict__ h, size_t n, float4* __restrict__ xyzh, float* __restrict__ sx,
                            float* __restrict__ sy, float* __restrict__ sz, float* __restrict__ sm)
{
    size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    {
        uint32_t j = order[i];
        float vx = x[j], vy = y[j], vz = z[j];
        float vm = m ? m[j] : 1.f;
        float vh = h ? h[j] : 0.f;
        xyzh[i]  = make_float4(vx, vy, vz, vh);
        sx[i]    = vx;
        sy[i]    = vy;
        sz[i]    = vz;
        sm[i]    = vm;
    }
}

//! results back to the caller's order: out[order[i]] = in[i] for the four arrays
__global__ void scatterTargets(const uint32_t* __restrict__ order, const float* __restrict__ in, size_t n,
                               float* __restrict__ p, float* __restrict__ ax, float* __restrict__ ay,
                               float* __restrict__ az)
{
    size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    {
        uint32_t j = order[i];
        if (p) p[j] = in[i];
        ax[j] = in[n + i];
        ay[j] = in[2 * n + i];
        az[j] = in[3 * n + i];
    }
}
} // namespace

extern "C" ryo_status ryo_solve_targets_f32(ryo_ctx_t* ctx, const float* xt, const float* yt, const float* zt,
                                           const float* mt, const float* ht, size_t n, float* p, float* ax,
                                           float* ay, float* az, ryo_solve_stats* stats, ryo_stream_t stream)
{
    if (!ctx) return RYO_ERR_BAD_ARG;
    return guardedCtx(ctx,
                   [&]
                   {
                       const auto& S = ctx->solveState;
                       REQUIRE(S.valid, "solve_targets: needs a preceding ryo_solve_f32 on this context");
                       REQUIRE(n > 0 && n < (size_t(1) << 32) && xt && yt && zt && ax && ay && az,
                               "solve_targets: bad argument");
                       cudaStream_t s      = stream;
                       DevBox<float> dbox  = boxOf(&S.box);
                       uint64_t* keys      = ctx->scratch<uint64_t>("tgt.keys", n, s);
                       uint64_t* keysAlt   = ctx->scratch<uint64_t>("tgt.keysAlt", n, s);
                       uint32_t* ord       = ctx->scratch<uint32_t>("tgt.order", n, s);
                       uint32_t* ordAlt    = ctx->scratch<uint32_t>("tgt.orderAlt", n, s);
                       size_t tmpBytes     = sortTempBytes(n);
                       void* tmp           = ctx->scratch<char>("tgt.sorttmp", tmpBytes, s);
                       // targets in SFC order of the solve's box, so that fixed groups are compact
                       launchKeys<float>(xt, yt, zt, keys, n, dbox, false, s);
                       bool alt = radixSortPairs(keys, ord, keysAlt, ordAlt, n, 0, 64, tmp, tmpBytes,
                                                 &ctx->ctl->error, s, true);
                       const uint32_t* order = alt ? ordAlt : ord;
                       float4* xyzh = ctx->scratch<float4>("tgt.xyzh", n, s);
                       float* sorted = ctx->scratch<float>("tgt.sorted", 8 * n, s); // x y z m | p ax ay az
                       unsigned grid = ceilDiv(n, 256) < unsigned(ctx->smCount * 16) ? ceilDiv(n, 256)
                                                                                    : unsigned(ctx->smCount * 16);
                       packTargets<<<grid, 256, 0, s>>>(order, xt, yt, zt, mt, ht, n, xyzh, sorted, sorted + n,
                                                        sorted + 2 * n, sorted + 3 * n);
                       RYO_LAUNCH_CHECK();
                       float* out = sorted + 4 * n;
                       RYO_CUDA(cudaMemsetAsync(out, 0, 4 * n * sizeof(float), s));
                       uint32_t numGroups = uint32_t((n + S.groupSize - 1) / S.groupSize);
                       uint32_t* groups   = ctx->scratch<uint32_t>("tgt.groups", size_t(numGroups) + 1, s);
                       launchFixedGroups(0, uint32_t(n), S.groupSize, groups, s);

                       TraverseLaunch t{};
                       t.groupStart    = groups;
                       t.groupEnd      = groups + 1;
                       t.numGroups     = int(numGroups);
                       t.initNode      = S.numNodes == 1 ? 0 : 1;
                       t.numNodes      = S.numNodes;
                       t.nodes         = static_cast<const NodeRecord*>(S.nodes);
                       t.dipoles       = static_cast<const float4*>(S.dipoles);
                       t.tgtXYZH       = xyzh;
                       t.tgtM          = sorted + 3 * n;
                       t.srcXYZM       = static_cast<const float4*>(S.xyzm);
                       t.srcH          = S.srcH;
                       t.massRange     = S.massRange; // the solve's sources: the same direct-sum arithmetic
                       t.G             = S.G;
                       t.numShells     = S.numShells;
                       for (int d = 0; d < 3; ++d)
                           t.boxL[d] = dbox.len[d];
                       t.p             = out;
                       t.ax            = out + n;
                       t.ay            = out + 2 * n;
                       t.az            = out + 3 * n;
                       double pot      = 0;
                       runTraversal(ctx, t, s, &pot);
                       double energy = 0.5 * double(S.G) * pot;
                       if (S.periodic)
                       {
                           EwaldHost e = ewaldSetup(S.root + 3, S.root, S.ewald.numReplicaShells, double(dbox.len[0]),
                                                    S.ewald.lCut, S.ewald.hCut, S.ewald.alpha_scale,
                                                    S.ewald.small_R_scale_factor);
                           double* ep = &ctx->ctl->ewaldPotential;
                           RYO_CUDA(cudaMemsetAsync(ep, 0, sizeof(double), s));
                           launchEwaldGroups(e, groups, groups + 1, numGroups, sorted, sorted + n, sorted + 2 * n,
                                             sorted + 3 * n, S.G, out, out + n, out + 2 * n, out + 3 * n, ep, s);
                           double he = 0;
                           RYO_CUDA(cudaMemcpyAsync(&he, ep, sizeof(double), cudaMemcpyDeviceToHost, s));
                           RYO_CUDA(cudaStreamSynchronize(s));
                           energy += 0.5 * double(S.G) * he;
                       }
                       scatterTargets<<<grid, 256, 0, s>>>(order, out, n, p, ax, ay, az);
                       RYO_LAUNCH_CHECK();
                       if (ctx->hostStats[kMaxP2P] == 0xFFFFFFFFull)
                           throw ApiError{RYO_ERR_STACK_OVERFLOW_UNSPLITTABLE, "solve_targets: a target overflowed"};
                       checkDeviceError(ctx, s);
                       if (stats)
                       {
                           *stats                 = ryo_solve_stats{};
                           stats->numGroups       = int(numGroups);
                           stats->numNodes        = S.numNodes;
                           stats->sumP2P          = ctx->hostStats[kSumP2P];
                           stats->maxP2P          = ctx->hostStats[kMaxP2P];
                           stats->sumM2P          = ctx->hostStats[kSumM2P];
                           stats->maxM2P          = ctx->hostStats[kMaxM2P];
                           stats->maxStack        = ctx->hostStats[kMaxStack];
                           stats->retries         = ctx->retries;
                           stats->potentialEnergy = energy;
                           for (int i = 0; i < 6; ++i)
                               stats->box[i] = S.box.limits[i];
                       }
                   });
}

extern "C" ryo_status ryo_solve_arrays_get(ryo_ctx_t* ctx, ryo_solve_arrays* out)
{
    if (!ctx || !out) return RYO_ERR_BAD_ARG;
    *out = ctx->lastSolve;
    return RYO_OK;
}

// ==================================================================================================== measurement

uint64_t& ryo::launchCounter()
{
    static uint64_t counter = 0;
    return counter;
}

extern "C" uint64_t ryo_kernel_launches(void) { return ryo::launchCounter(); }

extern "C" ryo_status ryo_measure_peaks(ryo_ctx_t* ctx, double* out3, ryo_stream_t stream)
{
    if (!ctx || !out3) return RYO_ERR_BAD_ARG;
    return guardedCtx(ctx, [&] { measurePeaks(ctx->smCount, out3, out3 + 1, out3 + 2, stream); });
}
