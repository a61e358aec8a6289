/*
 * ryoanji-b200: device-wide exclusive scan and the onesweep LSD radix sort.
 *
 * Replaces the CUB DeviceRadixSort::SortPairs call of the reference (cstone/include/cstone/primitives/
 * primitives_gpu.cu:311-356). One upfront pass histograms every digit position; each 8-bit digit pass then reads
 * the keys once and writes them once: tiles rank their keys with one warp ballot per digit bit, publish per-digit tile counts
 * with decoupled look-back (bounded waits), stage the tile in shared memory in digit order and write coalesced runs.
 * The sort is stable (keys and payload indices keep their input order within equal keys), as the reference needs.
 */
#include <mutex>

#include "internal.hpp"

namespace ryo
{

// ------------------------------------------------------------------------------------------------ scan

constexpr int kScanBlock = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile  = kScanBlock * kScanItems;

//! inclusive block scan of one value per thread (blockDim.x <= 1024, multiple of 32)
template<class T>
__device__ T blockInclusiveScan(T v, T* sWarp, T* total)
{
    int lane = laneId(), warp = threadIdx.x / kWarp, nw = blockDim.x / kWarp;
#pragma unroll
    for (int o = 1; o < kWarp; o <<= 1)
    {
        T w = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += w;
    }
    if (lane == kWarp - 1) sWarp[warp] = v;
    __syncthreads();
    if (warp == 0)
    {
        T s = lane < nw ? sWarp[lane] : T(0);
#pragma unroll
        for (int o = 1; o < kWarp; o <<= 1)
        {
            T w = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += w;
        }
        if (lane < nw) sWarp[lane] = s;
    }
    __syncthreads();
    if (warp > 0) v += sWarp[warp - 1];
    if (total) *total = sWarp[nw - 1];
    __syncthreads();
    return v;
}

__global__ void __launch_bounds__(kScanBlock) scanTileSums(const uint32_t* __restrict__ in, size_t n,
                                                           uint32_t* __restrict__ tileSums)
{
    __shared__ uint32_t sWarp[32];
    size_t base  = size_t(blockIdx.x) * kScanTile + size_t(threadIdx.x) * kScanItems;
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i)
        if (base + i < n) sum += in[base + i];
    uint32_t tot;
    blockInclusiveScan(sum, sWarp, &tot);
    if (threadIdx.x == 0) tileSums[blockIdx.x] = tot;
}

//! exclusive scan of the tile sums in one block; tileSums[numTiles] receives the grand total
__global__ void __launch_bounds__(1024) scanTileOffsets(uint32_t* tileSums, uint32_t numTiles)
{
    __shared__ uint32_t sWarp[32];
    uint32_t carry = 0;
    for (uint32_t b = 0; b < numTiles; b += blockDim.x)
    {
        uint32_t i = b + threadIdx.x;
        uint32_t v = i < numTiles ? tileSums[i] : 0;
        uint32_t tot;
        uint32_t incl = blockInclusiveScan(v, sWarp, &tot);
        if (i < numTiles) tileSums[i] = carry + incl - v;
        carry += tot;
    }
    if (threadIdx.x == 0) tileSums[numTiles] = carry;
}

__global__ void __launch_bounds__(kScanBlock) scanApply(const uint32_t* in, size_t n,
                                                        const uint32_t* __restrict__ tileOffsets, uint32_t* out,
                                                        uint32_t numTiles)
{
    __shared__ uint32_t sWarp[32];
    size_t base = size_t(blockIdx.x) * kScanTile + size_t(threadIdx.x) * kScanItems;
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i)
    {
        v[i] = base + i < n ? in[base + i] : 0;
        sum += v[i];
    }
    uint32_t incl = blockInclusiveScan(sum, sWarp, (uint32_t*)nullptr);
    uint32_t run  = tileOffsets[blockIdx.x] + incl - sum;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i)
    {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = tileOffsets[numTiles];
}

void exclusiveScanU32(ryo_ctx* ctx, const uint32_t* in, uint32_t* out, size_t n, cudaStream_t s)
{
    uint32_t numTiles = uint32_t((n + kScanTile - 1) / kScanTile);
    if (numTiles == 0)
    {
        RYO_CUDA(cudaMemsetAsync(out, 0, sizeof(uint32_t), s));
        return;
    }
    uint32_t* sums = ctx->scratch<uint32_t>("scan.sums", numTiles + 1, s);
    scanTileSums<<<numTiles, kScanBlock, 0, s>>>(in, n, sums);
    RYO_LAUNCH_CHECK();
    scanTileOffsets<<<1, 1024, 0, s>>>(sums, numTiles);
    RYO_LAUNCH_CHECK();
    scanApply<<<numTiles, kScanBlock, 0, s>>>(in, n, sums, out, numTiles);
    RYO_LAUNCH_CHECK();
}

// ------------------------------------------------------------------------------------------------ radix sort

constexpr int kSortBlock  = 256;
constexpr int kSortWarps  = kSortBlock / kWarp;
constexpr int kSortItems  = 12;
constexpr int kSortTile   = kSortBlock * kSortItems;
constexpr int kDigits     = 256;
constexpr int kMaxPasses  = 8;
constexpr unsigned long long kFlagAggregate = 1ull << 62;
constexpr unsigned long long kFlagInclusive = 2ull << 62;
constexpr int kSpinLimit  = 1 << 22;

struct SortTemp
{
    uint32_t* hist;     // kMaxPasses x 256
    uint32_t* base;     // kMaxPasses x 256
    unsigned int* tile; // kMaxPasses tile tickets
    unsigned long long* status;
    size_t headBytes;
    size_t numTiles;
};

static SortTemp sortLayout(void* tmp, size_t n)
{
    SortTemp t;
    t.numTiles   = (n + kSortTile - 1) / kSortTile;
    char* p      = static_cast<char*>(tmp);
    t.hist       = reinterpret_cast<uint32_t*>(p);
    t.base       = t.hist + kMaxPasses * kDigits;
    t.tile       = reinterpret_cast<unsigned int*>(t.base + kMaxPasses * kDigits);
    t.headBytes  = 2 * kMaxPasses * kDigits * sizeof(uint32_t) + 256;
    t.status     = reinterpret_cast<unsigned long long*>(p + t.headBytes);
    return t;
}

size_t sortTempBytes(size_t n)
{
    size_t tiles = (n + kSortTile - 1) / kSortTile;
    return 2 * kMaxPasses * kDigits * sizeof(uint32_t) + 256 + (tiles + 1) * kDigits * sizeof(unsigned long long);
}

constexpr int kHistKeys = 4; // keys per thread and round of the histogram, loaded before any is counted

//! all digit histograms in one read of the keys: two shared-memory copies per block (each shared by four warps),
//! plain shared atomics, and one aggregated add when a whole warp holds the same digit (top digits of clustered or
//! presorted keys). A round loads kHistKeys keys per thread before counting them, so that enough loads are in
//! flight to cover the memory latency.
__global__ void __launch_bounds__(256) digitHistogram(const uint64_t* __restrict__ keys, size_t n, int beginBit,
                                                      int numPasses, uint32_t* hist)
{
    __shared__ uint32_t sh[2][kMaxPasses][kDigits];
    for (int i = threadIdx.x; i < 2 * kMaxPasses * kDigits; i += blockDim.x)
        (&sh[0][0][0])[i] = 0;
    __syncthreads();
    uint32_t(*mine)[kDigits] = sh[(threadIdx.x >> 7) & 1];
    const unsigned lane      = laneId();
    const size_t round       = size_t(blockDim.x) * kHistKeys;
    const size_t stride      = size_t(gridDim.x) * round;
    for (size_t i0 = size_t(blockIdx.x) * round; i0 < n; i0 += stride)
    {
        uint64_t key[kHistKeys];
#pragma unroll
        for (int k = 0; k < kHistKeys; ++k)
        {
            size_t i = i0 + size_t(k) * blockDim.x + threadIdx.x;
            key[k]   = i < n ? keys[i] : 0;
        }
#pragma unroll
        for (int k = 0; k < kHistKeys; ++k)
        {
            bool valid     = i0 + size_t(k) * blockDim.x + threadIdx.x < n;
            unsigned vmask = __ballot_sync(0xffffffffu, valid);
            if (vmask == 0) continue;
            int lead = __ffs(vmask) - 1;
            for (int p = 0; p < numPasses; ++p)
            {
                unsigned d  = unsigned(key[k] >> (beginBit + 8 * p)) & 255u;
                unsigned d0 = __shfl_sync(0xffffffffu, d, lead);
                if (__all_sync(0xffffffffu, !valid || d == d0))
                {
                    if (lane == unsigned(lead)) atomicAdd(&mine[p][d0], __popc(vmask));
                }
                else if (valid)
                    atomicAdd(&mine[p][d], 1u);
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < numPasses * kDigits; i += blockDim.x)
    {
        uint32_t c = (&sh[0][0][0])[i] + (&sh[1][0][0])[i];
        if (c) atomicAdd(hist + i, c);
    }
}

__global__ void digitBases(const uint32_t* hist, uint32_t* base, int numPasses)
{
    __shared__ uint32_t sWarp[32];
    for (int p = 0; p < numPasses; ++p)
    {
        uint32_t v    = hist[p * kDigits + threadIdx.x];
        uint32_t incl = blockInclusiveScan(v, sWarp, (uint32_t*)nullptr);
        base[p * kDigits + threadIdx.x] = incl - v;
    }
}

__global__ void __launch_bounds__(kSortBlock, 4) onesweepPass(const uint64_t* __restrict__ keysIn,
                                                           const uint32_t* __restrict__ valsIn,
                                                           uint64_t* __restrict__ keysOut,
                                                           uint32_t* __restrict__ valsOut, size_t n, int shift,
                                                           int nbits, const uint32_t* __restrict__ digitBase,
                                                           unsigned long long* status, unsigned int* tileTicket,
                                                           uint32_t epoch, unsigned int* errorFlag)
{
    __shared__ uint32_t sTile;
    __shared__ uint32_t sHist[kSortWarps][kDigits];
    __shared__ uint32_t sStart[kDigits];
    __shared__ uint32_t sGlobal[kDigits];
    __shared__ uint32_t sWarp[32];
    __shared__ uint64_t sKeys[kSortTile];
    __shared__ uint8_t sDig[kSortTile];

    const int tid = threadIdx.x, lane = laneId(), warp = tid / kWarp;
    for (int i = tid; i < kSortWarps * kDigits; i += kSortBlock)
        (&sHist[0][0])[i] = 0;
    if (tid == 0) sTile = atomicAdd(tileTicket, 1u);
    __syncthreads();

    const uint32_t tile  = sTile;
    const size_t base    = size_t(tile) * kSortTile;
    const uint32_t dmask = (1u << nbits) - 1;
    const size_t wbase   = base + size_t(warp) * (kSortItems * kWarp);

    // keys now, values only once the keys are staged (fewer live registers, more tiles in flight per SM); a padding
    // item past n has digit kDigits
    uint64_t k[kSortItems];
    uint32_t r[kSortItems];
#pragma unroll
    for (int i = 0; i < kSortItems; ++i)
    {
        size_t idx = wbase + size_t(i) * kWarp + lane;
        k[i]       = idx < n ? keysIn[idx] : 0;
    }
    auto digitOf = [&](int i) -> uint32_t
    {
        size_t idx = wbase + size_t(i) * kWarp + lane;
        return idx < n ? uint32_t(k[i] >> shift) & dmask : uint32_t(kDigits);
    };

    // rank within the warp: items in (item, lane) order, which is this warp's input order. The lanes holding the
    // same digit are found with one ballot per digit bit (plus one for the padding items past n).
    const unsigned lt = lanemaskLt();
#pragma unroll
    for (int i = 0; i < kSortItems; ++i)
    {
        const uint32_t di = digitOf(i);
        const bool valid  = di < kDigits;
        const unsigned vm = __ballot_sync(0xffffffffu, valid);
        unsigned peers    = valid ? vm : ~vm;
#pragma unroll
        for (int b = 0; b < 8; ++b)
        {
            if (b >= nbits) break; // uniform across the warp
            const bool bit    = (di >> b) & 1u;
            const unsigned bv = __ballot_sync(0xffffffffu, bit);
            peers &= bit ? bv : ~bv;
        }
        int leader     = __ffs(peers) - 1;
        uint32_t before = 0;
        if (lane == leader && valid)
        {
            before          = sHist[warp][di];
            sHist[warp][di] = before + __popc(peers);
        }
        before = __shfl_sync(0xffffffffu, before, leader);
        r[i]   = before + __popc(peers & lt);
    }
    __syncthreads();

    // digit tid: warp-exclusive offsets and the tile count
    uint32_t total = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w)
    {
        uint32_t c   = sHist[w][tid];
        sHist[w][tid] = total;
        total += c;
    }

    // decoupled look-back over earlier tiles for digit tid
    const unsigned long long tag = (unsigned long long)epoch << 32;
    volatile unsigned long long* mine = status + size_t(tile) * kDigits + tid;
    uint32_t excl = 0;
    if (tile == 0) { *mine = kFlagInclusive | tag | total; }
    else
    {
        *mine = kFlagAggregate | tag | total;
        long t    = long(tile) - 1;
        int spins = 0;
        while (t >= 0)
        {
            unsigned long long s = *(volatile unsigned long long*)(status + size_t(t) * kDigits + tid);
            unsigned long long flag = s & (3ull << 62);
            if (flag == 0 || uint32_t((s >> 32) & 0x3FFFFFFFu) != epoch)
            {
                if (++spins > kSpinLimit)
                {
                    atomicExch(errorFlag, 1u);
                    break;
                }
                __nanosleep(32);
                continue;
            }
            excl += uint32_t(s);
            if (flag == kFlagInclusive) break;
            --t;
        }
        *mine = kFlagInclusive | tag | uint32_t(excl + total);
    }
    sGlobal[tid] = digitBase[tid] + excl;
    uint32_t incl = blockInclusiveScan(total, sWarp, (uint32_t*)nullptr);
    sStart[tid]   = incl - total;
    __syncthreads();

    // stage the tile in digit order
#pragma unroll
    for (int i = 0; i < kSortItems; ++i)
    {
        const uint32_t di = digitOf(i);
        if (di < kDigits)
        {
            uint32_t pos = sStart[di] + sHist[warp][di] + r[i];
            sKeys[pos]   = k[i];
            r[i]         = pos;
        }
    }
    // the values, whose loads overlap the key writes below
    uint32_t v[kSortItems];
#pragma unroll
    for (int i = 0; i < kSortItems; ++i)
    {
        size_t idx = wbase + size_t(i) * kWarp + lane;
        v[i]       = idx < n ? (valsIn ? valsIn[idx] : uint32_t(idx)) : 0u;
    }
    __syncthreads();
    const uint32_t count = uint32_t(n - base < size_t(kSortTile) ? n - base : size_t(kSortTile));
    for (uint32_t p = tid; p < count; p += kSortBlock)
    {
        uint64_t key = sKeys[p];
        uint32_t dig = uint32_t(key >> shift) & dmask;
        sDig[p]      = uint8_t(dig);
        keysOut[sGlobal[dig] + (p - sStart[dig])] = key;
    }
    __syncthreads();
    uint32_t* sVals = reinterpret_cast<uint32_t*>(sKeys);
#pragma unroll
    for (int i = 0; i < kSortItems; ++i)
        if (wbase + size_t(i) * kWarp + lane < n) sVals[r[i]] = v[i];
    __syncthreads();
    for (uint32_t p = tid; p < count; p += kSortBlock)
    {
        uint32_t dig = sDig[p];
        valsOut[sGlobal[dig] + (p - sStart[dig])] = sVals[p];
    }
}

bool radixSortPairs(uint64_t* keys, uint32_t* values, uint64_t* keysAlt, uint32_t* valuesAlt, size_t n, int beginBit,
                    int endBit, void* tmp, size_t tmpBytes, unsigned int* errorFlag, cudaStream_t s, bool iotaValues)
{
    if (n == 0) return false;
    if (tmpBytes < sortTempBytes(n)) throw CudaError{cudaErrorInvalidValue, "radix sort: temporary storage too small"};
    int numPasses = (endBit - beginBit + 7) / 8;
    SortTemp t    = sortLayout(tmp, n);
    RYO_CUDA(cudaMemsetAsync(tmp, 0, t.headBytes, s));
    RYO_CUDA(cudaMemsetAsync(t.status, 0, t.numTiles * kDigits * sizeof(unsigned long long), s));

    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    size_t hb = (n + 256 * kHistKeys - 1) / (256 * kHistKeys);
    unsigned histBlocks = unsigned(hb < size_t(sms) * 4 ? hb : size_t(sms) * 4);
    digitHistogram<<<histBlocks, 256, 0, s>>>(keys, n, beginBit, numPasses, t.hist);
    RYO_LAUNCH_CHECK();
    digitBases<<<1, kDigits, 0, s>>>(t.hist, t.base, numPasses);
    RYO_LAUNCH_CHECK();

    // the whole shared memory as carveout, so that registers (four tiles per SM), not the L1 split, limit residency
    RYO_CUDA(cudaFuncSetAttribute(onesweepPass, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  int(cudaSharedmemCarveoutMaxShared)));
    // pass p reads buffer set p % 2 and writes the other
    bool inAlt = false;
    for (int p = 0; p < numPasses; ++p)
    {
        int shift          = beginBit + 8 * p;
        int nbits          = endBit - shift < 8 ? endBit - shift : 8;
        uint64_t* kin      = inAlt ? keysAlt : keys;
        uint64_t* kout     = inAlt ? keys : keysAlt;
        const uint32_t* vin = (p == 0 && iotaValues) ? nullptr : (inAlt ? valuesAlt : values);
        uint32_t* vout     = inAlt ? values : valuesAlt;
        onesweepPass<<<unsigned(t.numTiles), kSortBlock, 0, s>>>(kin, vin, kout, vout, n, shift, nbits,
                                                                  t.base + p * kDigits, t.status, t.tile + p,
                                                                  uint32_t(p + 1), errorFlag);
        RYO_LAUNCH_CHECK();
        inAlt = !inAlt;
    }
    return inAlt;
}

/*! failure-detection self-test of the look-back wait. One pass over two tiles of zero keys is launched with a single
 *  block whose tile ticket starts at 1: the block takes tile 1, and tile 0's status words are never published, so
 *  each digit thread's bounded wait runs out after kSpinLimit polls and raises the flag. The accesses stay inside the
 *  buffers: every key has digit 0 (base 0), so the lone tile scatters to positions [0, kSortTile) of the 2 x
 *  kSortTile outputs. Returns whether the flag was raised. */
bool sortWaitTimeoutSelfTest(cudaStream_t s)
{
    const size_t n = 2 * size_t(kSortTile);
    struct Buffers
    {
        void* p[5] = {};
        ~Buffers()
        {
            for (void* q : p)
                if (q) cudaFree(q);
        }
    } b;
    const size_t bytes[5] = {n * sizeof(uint64_t), n * sizeof(uint64_t), n * sizeof(uint32_t), sortTempBytes(n),
                             sizeof(unsigned int)};
    for (int i = 0; i < 5; ++i)
        RYO_CUDA(cudaMalloc(&b.p[i], bytes[i]));
    auto* keys = static_cast<uint64_t*>(b.p[0]);
    auto* kout = static_cast<uint64_t*>(b.p[1]);
    auto* vout = static_cast<uint32_t*>(b.p[2]);
    auto* flag = static_cast<unsigned int*>(b.p[4]);
    SortTemp t = sortLayout(b.p[3], n);
    RYO_CUDA(cudaMemsetAsync(keys, 0, bytes[0], s));
    RYO_CUDA(cudaMemsetAsync(b.p[3], 0, bytes[3], s));
    RYO_CUDA(cudaMemsetAsync(flag, 0, sizeof(unsigned int), s));
    const unsigned int one = 1;
    RYO_CUDA(cudaMemcpyAsync(t.tile, &one, sizeof(one), cudaMemcpyHostToDevice, s));
    digitHistogram<<<1, 256, 0, s>>>(keys, n, 0, 1, t.hist);
    RYO_LAUNCH_CHECK();
    digitBases<<<1, kDigits, 0, s>>>(t.hist, t.base, 1);
    RYO_LAUNCH_CHECK();
    onesweepPass<<<1, kSortBlock, 0, s>>>(keys, nullptr, kout, vout, n, 0, 8, t.base, t.status, t.tile, 1u, flag);
    RYO_LAUNCH_CHECK();
    unsigned int raised = 0;
    RYO_CUDA(cudaMemcpyAsync(&raised, flag, sizeof(raised), cudaMemcpyDeviceToHost, s));
    RYO_CUDA(cudaStreamSynchronize(s));
    return raised != 0;
}


// ------------------------------------------------------------------------------------------------ fixed scratch

/*
 * Scratch for the sort entry point that takes no temporary-storage argument. Some callers cannot allocate device
 * memory for a sort: a host whose pool allocator has already reserved the free HBM has nothing left for cudaMalloc,
 * and cudaFree waits for the whole device, which a caller sorting inside a latency-bound loop cannot afford. For them
 * the digit histograms, tile tickets, look-back status words and the wait-timeout flag live in this one array,
 * sized for kStaticSortMaxKeys keys. Its storage is created with the module on each device; no call allocates.
 * Every call clears what must start at zero (histograms, tickets, status words, flag) on its stream before the
 * first pass reads it. All calls on a device share the array, so calls that overlap in time race and corrupt each
 * other's results: callers serialise them (one stream, or their own ordering between streams and threads).
 */
constexpr size_t kStaticSortMaxKeys = size_t(1) << 24;
constexpr size_t kStaticSortBytes   = size_t(12) << 20;

static __device__ __align__(256) unsigned char staticSortScratch[kStaticSortBytes];

size_t staticSortMaxKeys() { return kStaticSortMaxKeys; }

//! the current CUDA context (the driver's handle), looked up through the runtime so that the library needs no link
//! to the driver library; null if the driver does not offer the call
static void* currentContext()
{
    using GetCtx = int (*)(void**);
    static GetCtx fn = []
    {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<GetCtx>(f);
    }();
    void* c = nullptr;
    if (fn && fn(&c) != 0) c = nullptr;
    return c;
}

//! the array's device address on the current device. It is looked up (cudaGetSymbolAddress) on the first call for
//! that device and again whenever the device's context has changed since: a cudaDeviceReset by the caller ends the
//! context that held the array, and the next call on that device then finds it in the new one.
static void* staticSortScratchAddress()
{
    constexpr int kMaxDevices = 64;
    static std::mutex lock;
    static void* address[kMaxDevices] = {};
    static void* context[kMaxDevices] = {};
    int dev = 0;
    RYO_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw CudaError{cudaErrorInvalidDevice, "static sort: device ordinal"};
    void* ctxNow = currentContext();
    std::lock_guard<std::mutex> guard(lock);
    if (!address[dev] || context[dev] != ctxNow)
    {
        void* p = nullptr;
        RYO_CUDA(cudaGetSymbolAddress(&p, staticSortScratch)); // also makes the device's context current
        if (!p) throw CudaError{cudaErrorInvalidSymbol, "static sort: scratch symbol has no address"};
        address[dev] = p;
        context[dev] = currentContext();
    }
    return address[dev];
}

bool sortPairsStaticScratch(uint64_t* keys, uint32_t* values, uint64_t* keysAlt, uint32_t* valuesAlt, size_t n,
                            cudaStream_t s)
{
    if (n > kStaticSortMaxKeys) throw CudaError{cudaErrorInvalidValue, "static sort: too many keys"};
    size_t need = sortTempBytes(n);
    if (need + 64 > kStaticSortBytes) throw CudaError{cudaErrorInvalidValue, "static sort: scratch too small"};
    char* base         = static_cast<char*>(staticSortScratchAddress());
    unsigned int* flag = reinterpret_cast<unsigned int*>(base + kStaticSortBytes - 64);
    RYO_CUDA(cudaMemsetAsync(flag, 0, sizeof(unsigned int), s));
    bool alt = radixSortPairs(keys, values, keysAlt, valuesAlt, n, 0, 64, base, need, flag, s, false);
    if (alt)
    {
        RYO_CUDA(cudaMemcpyAsync(keys, keysAlt, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
        RYO_CUDA(cudaMemcpyAsync(values, valuesAlt, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    }
    unsigned int err = 0;
    RYO_CUDA(cudaMemcpyAsync(&err, flag, sizeof(err), cudaMemcpyDeviceToHost, s));
    RYO_CUDA(cudaStreamSynchronize(s));
    return err != 0;
}

} // namespace ryo
