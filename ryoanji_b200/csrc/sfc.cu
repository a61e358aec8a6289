/*
 * ryoanji-b200: SFC keys, bounding box, sequences and gathers.
 *
 * computeSfcKeys (reference cstone/include/cstone/sfc/sfc_gpu.cu:23-44) is HBM-light and integer-heavy: each key
 * costs 21 Hilbert levels of bit arithmetic on 12 input bytes. Threads process four consecutive points with 128-bit
 * loads when the arrays allow it; the grid is a multiple of the SM count and strides over the data.
 */
#include <initializer_list>

#include "internal.hpp"

namespace ryo
{

template<class T>
__global__ void keysKernel(const T* __restrict__ x, const T* __restrict__ y, const T* __restrict__ z,
                           uint64_t* __restrict__ keys, size_t n, DevBox<T> box, bool keepRemoved)
{
    size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    {
        if (keepRemoved && keys[i] == kKeyEnd) continue;
        keys[i] = pointKey(x[i], y[i], z[i], box);
    }
}

//! four points per thread with 16-byte loads, keys written as two 16-byte stores
__global__ void keysKernelVec4(const float4* __restrict__ x, const float4* __restrict__ y,
                               const float4* __restrict__ z, ulonglong2* __restrict__ keys, size_t n4,
                               DevBox<float> box)
{
    size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n4; i += stride)
    {
        float4 px = x[i], py = y[i], pz = z[i];
        ulonglong2 a, b;
        a.x         = pointKey(px.x, py.x, pz.x, box);
        a.y         = pointKey(px.y, py.y, pz.y, box);
        b.x         = pointKey(px.z, py.z, pz.z, box);
        b.y         = pointKey(px.w, py.w, pz.w, box);
        keys[2 * i]     = a;
        keys[2 * i + 1] = b;
    }
}

//! the two-level Hilbert tables (identical keys to hilbert3), built at compile time
__device__ const HilbertLut kHilbertLut = makeHilbertLut();

//! keysKernelVec4 for boxes whose three axes use all 21 levels: the Hilbert index through the tables in shared
//! memory (two levels per lookup instead of bit arithmetic per level)
__global__ void __launch_bounds__(256) keysKernelVec4Lut(const float4* __restrict__ x, const float4* __restrict__ y,
                                                         const float4* __restrict__ z, ulonglong2* __restrict__ keys,
                                                         size_t n4, DevBox<float> box)
{
    __shared__ uint16_t two[48 * 64];
    __shared__ uint16_t one[48 * 8];
    for (int i = threadIdx.x; i < 48 * 64; i += blockDim.x)
        two[i] = kHilbertLut.two[i];
    for (int i = threadIdx.x; i < 48 * 8; i += blockDim.x)
        one[i] = kHilbertLut.one[i];
    __syncthreads();
    auto key = [&](float px, float py, float pz)
    {
        unsigned ic[3];
        pointCells(px, py, pz, box, ic);
        return hilbert3Lut(ic[0], ic[1], ic[2], two, one);
    };
    size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n4; i += stride)
    {
        float4 px = x[i], py = y[i], pz = z[i];
        ulonglong2 a, b;
        a.x             = key(px.x, py.x, pz.x);
        a.y             = key(px.y, py.y, pz.y);
        b.x             = key(px.z, py.z, pz.z);
        b.y             = key(px.w, py.w, pz.w);
        keys[2 * i]     = a;
        keys[2 * i + 1] = b;
    }
}

static unsigned streamGrid(size_t work, unsigned block)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    size_t want = (work + block - 1) / block;
    size_t cap  = size_t(sms) * 8;
    return unsigned(want < cap ? (want ? want : 1) : cap);
}

template<class T>
void launchKeys(const T* x, const T* y, const T* z, uint64_t* keys, size_t n, const DevBox<T>& box, bool keepRemoved,
                cudaStream_t s)
{
    if (n == 0) return;
    constexpr unsigned block = 256;
    bool aligned = (reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y) |
                    reinterpret_cast<uintptr_t>(z) | reinterpret_cast<uintptr_t>(keys)) % 16 == 0;
    if constexpr (std::is_same_v<T, float>)
    {
        if (aligned && !keepRemoved && n >= 4)
        {
            size_t n4  = n / 4;
            bool full  = box.bits[0] == unsigned(kMaxLevel) && box.bits[1] == unsigned(kMaxLevel) &&
                        box.bits[2] == unsigned(kMaxLevel);
            auto* x4 = reinterpret_cast<const float4*>(x);
            auto* y4 = reinterpret_cast<const float4*>(y);
            auto* z4 = reinterpret_cast<const float4*>(z);
            auto* k2 = reinterpret_cast<ulonglong2*>(keys);
            if (full) keysKernelVec4Lut<<<streamGrid(n4, block), block, 0, s>>>(x4, y4, z4, k2, n4, box);
            else keysKernelVec4<<<streamGrid(n4, block), block, 0, s>>>(x4, y4, z4, k2, n4, box);
            RYO_LAUNCH_CHECK();
            size_t done = n4 * 4;
            if (done < n)
            {
                keysKernel<<<1, 32, 0, s>>>(x + done, y + done, z + done, keys + done, n - done, box, false);
                RYO_LAUNCH_CHECK();
            }
            return;
        }
    }
    keysKernel<<<streamGrid(n, block), block, 0, s>>>(x, y, z, keys, n, box, keepRemoved);
    RYO_LAUNCH_CHECK();
}

template void launchKeys<float>(const float*, const float*, const float*, uint64_t*, size_t, const DevBox<float>&,
                                bool, cudaStream_t);
template void launchKeys<double>(const double*, const double*, const double*, uint64_t*, size_t,
                                 const DevBox<double>&, bool, cudaStream_t);

// ------------------------------------------------------------------------------------------------ bounding box

__device__ inline void atomicMinDouble(double* addr, double v)
{
    unsigned long long* a = reinterpret_cast<unsigned long long*>(addr);
    unsigned long long old = *a;
    while (v < __longlong_as_double(old))
    {
        unsigned long long prev = atomicCAS(a, old, __double_as_longlong(v));
        if (prev == old) break;
        old = prev;
    }
}

__device__ inline void atomicMaxDouble(double* addr, double v)
{
    unsigned long long* a = reinterpret_cast<unsigned long long*>(addr);
    unsigned long long old = *a;
    while (v > __longlong_as_double(old))
    {
        unsigned long long prev = atomicCAS(a, old, __double_as_longlong(v));
        if (prev == old) break;
        old = prev;
    }
}

__global__ void bboxInit(double* mm)
{
    if (threadIdx.x < 3)
    {
        mm[2 * threadIdx.x]     = 1e300;
        mm[2 * threadIdx.x + 1] = -1e300;
    }
}

//! per-axis min and max (exact in any precision), reduced per block and combined with double atomics
__global__ void bboxKernel(const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
                           size_t n, double* mm)
{
    float lo[3] = {3.4e38f, 3.4e38f, 3.4e38f}, hi[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    {
        float v[3] = {x[i], y[i], z[i]};
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            lo[d] = fminf(lo[d], v[d]);
            hi[d] = fmaxf(hi[d], v[d]);
        }
    }
    __shared__ float slo[3][32], shi[3][32];
    int w = threadIdx.x / kWarp, l = laneId();
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
        lo[d] = warpMin(lo[d]);
        hi[d] = warpMax(hi[d]);
        if (l == 0)
        {
            slo[d][w] = lo[d];
            shi[d][w] = hi[d];
        }
    }
    __syncthreads();
    if (w == 0)
    {
        int nw = blockDim.x / kWarp;
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            float a = l < nw ? slo[d][l] : 3.4e38f, b = l < nw ? shi[d][l] : -3.4e38f;
            a = warpMin(a);
            b = warpMax(b);
            if (l == 0)
            {
                atomicMinDouble(mm + 2 * d, double(a));
                atomicMaxDouble(mm + 2 * d + 1, double(b));
            }
        }
    }
}

void launchBoundingBox(const float* x, const float* y, const float* z, size_t n, double* minmax6, cudaStream_t s)
{
    bboxInit<<<1, 32, 0, s>>>(minmax6);
    RYO_LAUNCH_CHECK();
    if (n == 0) return;
    bboxKernel<<<streamGrid(n, 256), 256, 0, s>>>(x, y, z, n, minmax6);
    RYO_LAUNCH_CHECK();
}

// ------------------------------------------------------------------------------------------------ sequences, gathers

__global__ void sequenceKernel(uint32_t* v, size_t n, uint32_t first)
{
    size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        v[i] = first + uint32_t(i);
}

void launchSequence(uint32_t* v, size_t n, uint32_t first, cudaStream_t s)
{
    if (n == 0) return;
    sequenceKernel<<<streamGrid(n, 256), 256, 0, s>>>(v, n, first);
    RYO_LAUNCH_CHECK();
}

template<class T>
__global__ void gatherKernel(const uint32_t* __restrict__ order, const T* __restrict__ in, T* __restrict__ out,
                             size_t n)
{
    size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = in[order[i]];
}

template<class T>
void launchGatherT(const uint32_t* order, const T* in, T* out, size_t n, cudaStream_t s)
{
    if (n == 0) return;
    gatherKernel<<<streamGrid(n, 256), 256, 0, s>>>(order, in, out, n);
    RYO_LAUNCH_CHECK();
}

void launchGather(const uint32_t* order, const float* in, float* out, size_t n, cudaStream_t s)
{
    launchGatherT<float>(order, in, out, n, s);
}

//! every body as one 32-byte record (x, y, z, m, h, vx, vy, vz; absent velocities are zero), so that the permutation
//! after the sort reads one sector per body instead of one per array
__global__ void packRecordsKernel(const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
                                  const float* __restrict__ m, const float* __restrict__ h,
                                  const float* __restrict__ vx, const float* __restrict__ vy,
                                  const float* __restrict__ vz, size_t n, float4* __restrict__ rec)
{
    size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    {
        rec[2 * i]     = make_float4(x[i], y[i], z[i], m[i]);
        rec[2 * i + 1] = make_float4(h[i], vx ? vx[i] : 0.f, vy ? vy[i] : 0.f, vz ? vz[i] : 0.f);
    }
}

//! the sorted bodies from their records: the per-body arrays (overwritten in sorted order) and the packed source
//! (x, y, z, m) and target (x, y, z, h) arrays of the traversal
//! fold a thread's softening range into hRange[0] (min) and hRange[1] (max), as ordered bits; whole warps call it
__device__ __forceinline__ void foldRange(uint32_t lo, uint32_t hi, uint32_t* hRange)
{
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    if (laneId() == 0 && lo <= hi)
    {
        atomicMin(hRange, lo);
        atomicMax(hRange + 1, hi);
    }
}

__global__ void gatherRecordsKernel(const uint32_t* __restrict__ order, const float4* __restrict__ rec, size_t n,
                                    float* __restrict__ x, float* __restrict__ y, float* __restrict__ z,
                                    float* __restrict__ m, float* __restrict__ h, float* __restrict__ vx,
                                    float* __restrict__ vy, float* __restrict__ vz, float4* __restrict__ xyzm,
                                    float4* __restrict__ xyzh, uint32_t* __restrict__ hRange)
{
    size_t stride = size_t(gridDim.x) * blockDim.x;
    uint32_t lo = 0xffffffffu, hi = 0u, mlo = 0xffffffffu, mhi = 0u;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    {
        size_t j = order[i];
        float4 a = rec[2 * j], b = rec[2 * j + 1]; // one 32-byte sector
        lo       = min(lo, orderedBits(b.x));
        hi       = max(hi, orderedBits(b.x));
        mlo      = min(mlo, orderedBits(a.w));
        mhi      = max(mhi, orderedBits(a.w));
        x[i]     = a.x;
        y[i]     = a.y;
        z[i]     = a.z;
        m[i]     = a.w;
        h[i]     = b.x;
        if (vx) vx[i] = b.y;
        if (vy) vy[i] = b.z;
        if (vz) vz[i] = b.w;
        if (xyzm) xyzm[i] = a;
        if (xyzh) xyzh[i] = make_float4(a.x, a.y, a.z, b.x);
    }
    if (hRange)
    {
        foldRange(lo, hi, hRange);
        foldRange(mlo, mhi, hRange + 2);
    }
}

//! gatherRecordsKernel for four consecutive sorted bodies per thread: one 16-byte load of their indices, 16-byte
//! stores of every output (arrays 16-byte aligned, n4 = n / 4)
__global__ void gatherRecordsKernel4(const uint4* __restrict__ order, const float4* __restrict__ rec, size_t n4,
                                     float4* __restrict__ x, float4* __restrict__ y, float4* __restrict__ z,
                                     float4* __restrict__ m, float4* __restrict__ h, float4* __restrict__ vx,
                                     float4* __restrict__ vy, float4* __restrict__ vz, float4* __restrict__ xyzm,
                                     float4* __restrict__ xyzh, uint32_t* __restrict__ hRange)
{
    size_t stride = size_t(gridDim.x) * blockDim.x;
    uint32_t lo = 0xffffffffu, hi = 0u, mlo = 0xffffffffu, mhi = 0u;
    for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < n4; t += stride)
    {
        uint4 j = order[t];
        float4 a0 = rec[2 * size_t(j.x)], b0 = rec[2 * size_t(j.x) + 1];
        float4 a1 = rec[2 * size_t(j.y)], b1 = rec[2 * size_t(j.y) + 1];
        float4 a2 = rec[2 * size_t(j.z)], b2 = rec[2 * size_t(j.z) + 1];
        float4 a3 = rec[2 * size_t(j.w)], b3 = rec[2 * size_t(j.w) + 1];
        lo = min(min(min(lo, orderedBits(b0.x)), orderedBits(b1.x)), min(orderedBits(b2.x), orderedBits(b3.x)));
        hi = max(max(max(hi, orderedBits(b0.x)), orderedBits(b1.x)), max(orderedBits(b2.x), orderedBits(b3.x)));
        mlo = min(min(min(mlo, orderedBits(a0.w)), orderedBits(a1.w)), min(orderedBits(a2.w), orderedBits(a3.w)));
        mhi = max(max(max(mhi, orderedBits(a0.w)), orderedBits(a1.w)), max(orderedBits(a2.w), orderedBits(a3.w)));
        x[t] = make_float4(a0.x, a1.x, a2.x, a3.x);
        y[t] = make_float4(a0.y, a1.y, a2.y, a3.y);
        z[t] = make_float4(a0.z, a1.z, a2.z, a3.z);
        m[t] = make_float4(a0.w, a1.w, a2.w, a3.w);
        h[t] = make_float4(b0.x, b1.x, b2.x, b3.x);
        if (vx) vx[t] = make_float4(b0.y, b1.y, b2.y, b3.y);
        if (vy) vy[t] = make_float4(b0.z, b1.z, b2.z, b3.z);
        if (vz) vz[t] = make_float4(b0.w, b1.w, b2.w, b3.w);
        if (xyzm)
        {
            float4* o = xyzm + 4 * t;
            o[0] = a0;
            o[1] = a1;
            o[2] = a2;
            o[3] = a3;
        }
        if (xyzh)
        {
            float4* o = xyzh + 4 * t;
            o[0] = make_float4(a0.x, a0.y, a0.z, b0.x);
            o[1] = make_float4(a1.x, a1.y, a1.z, b1.x);
            o[2] = make_float4(a2.x, a2.y, a2.z, b2.x);
            o[3] = make_float4(a3.x, a3.y, a3.z, b3.x);
        }
    }
    if (hRange)
    {
        foldRange(lo, hi, hRange);
        foldRange(mlo, mhi, hRange + 2);
    }
}

namespace
{
bool aligned16(std::initializer_list<const void*> ptrs)
{
    for (const void* p : ptrs)
        if (reinterpret_cast<uintptr_t>(p) % 16 != 0) return false;
    return true;
}
} // namespace

void launchPackRecords(const float* x, const float* y, const float* z, const float* m, const float* h,
                       const float* vx, const float* vy, const float* vz, size_t n, float4* rec, cudaStream_t s)
{
    // one body per thread: coalesced 4-byte loads, and each warp's record stores cover whole 32-byte sectors
    // (four bodies per thread with 16-byte loads measured 2x slower: a lane's 128 contiguous output bytes spread
    // every store instruction over 32 lines)
    if (n == 0) return;
    packRecordsKernel<<<streamGrid(n, 256), 256, 0, s>>>(x, y, z, m, h, vx, vy, vz, n, rec);
    RYO_LAUNCH_CHECK();
}

void launchGatherRecords(const uint32_t* order, const float4* rec, size_t n, float* x, float* y, float* z, float* m,
                         float* h, float* vx, float* vy, float* vz, float4* xyzm, float4* xyzh, uint32_t* hRange,
                         cudaStream_t s)
{
    if (hRange)
    {
        // softening (min, max), then mass (min, max)
        RYO_CUDA(cudaMemsetAsync(hRange, 0xff, sizeof(uint32_t), s));
        RYO_CUDA(cudaMemsetAsync(hRange + 1, 0, sizeof(uint32_t), s));
        RYO_CUDA(cudaMemsetAsync(hRange + 2, 0xff, sizeof(uint32_t), s));
        RYO_CUDA(cudaMemsetAsync(hRange + 3, 0, sizeof(uint32_t), s));
    }
    if (n == 0) return;
    size_t done = 0;
    if (n >= 4 && aligned16({order, x, y, z, m, h, vx, vy, vz, xyzm, xyzh}))
    {
        size_t n4 = n / 4;
        auto f4   = [](float* a) { return reinterpret_cast<float4*>(a); };
        gatherRecordsKernel4<<<streamGrid(n4, 256), 256, 0, s>>>(reinterpret_cast<const uint4*>(order), rec, n4,
                                                                 f4(x), f4(y), f4(z), f4(m), f4(h), f4(vx), f4(vy),
                                                                 f4(vz), xyzm, xyzh, hRange);
        RYO_LAUNCH_CHECK();
        done = 4 * n4;
    }
    if (done == n) return;
    auto off  = [&](float* a) { return a ? a + done : nullptr; };
    auto off4 = [&](float4* a) { return a ? a + done : nullptr; };
    gatherRecordsKernel<<<streamGrid(n - done, 256), 256, 0, s>>>(order + done, rec, n - done, off(x), off(y), off(z),
                                                                  off(m), off(h), off(vx), off(vy), off(vz), off4(xyzm),
                                                                  off4(xyzh), hRange);
    RYO_LAUNCH_CHECK();
}

template void launchGatherT<float>(const uint32_t*, const float*, float*, size_t, cudaStream_t);
template void launchGatherT<double>(const uint32_t*, const double*, double*, size_t, cudaStream_t);
template void launchGatherT<float4>(const uint32_t*, const float4*, float4*, size_t, cudaStream_t);
template void launchGatherT<uint64_t>(const uint32_t*, const uint64_t*, uint64_t*, size_t, cudaStream_t);

} // namespace ryo
