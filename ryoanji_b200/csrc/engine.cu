/*
 * ryoanji-b200: the served stream. Requests (a particle set plus K kick-drift-kick leapfrog steps) are admitted
 * under an HBM budget, stay resident on the device across their steps, and every engine step advances all resident
 * requests together with one batched solve. Requests that arrive while others are being stepped join at the next
 * step; finished ones leave and free their share of the budget (continuous batching).
 *
 * The reference has no serving layer; each step's physics is the reference path (one force evaluation per system
 * with the single-system solve's semantics, see batch.cu), and the leapfrog is the standard KDK scheme:
 *   v += a dt/2;  x += v dt;  a = F(x);  v += a dt/2.
 * A request's first engine step only evaluates its initial forces.
 *
 * Resident layout: one arena of per-body arrays (x, y, z, m, h, vx, vy, vz, ax, ay, az, p, id) with the requests
 * in consecutive ranges; id is the body's index in its request so results go back in submission order. When the
 * set of resident requests changes, one kernel compacts the survivors into the second arena and the admitted
 * requests are copied in behind them.
 */
#include <algorithm>
#include <chrono>
#include <deque>
#include <functional>

#include "internal.hpp"

namespace ryo
{

constexpr int kArenaArrays = 12; // x y z m h vx vy vz ax ay az p (floats); ids are separate

struct Arena
{
    float* a[kArenaArrays] = {};
    uint32_t* id           = nullptr;
    size_t capacity        = 0;
    void* block            = nullptr; // all arrays in one allocation

    //! room for at least @p n bodies; growth doubles, so a growing stream reallocates O(log n) times (each
    //! reallocation frees, which waits for the device)
    void ensure(size_t n)
    {
        if (n <= capacity) return;
        release_();
        size_t cap = std::max<size_t>(n, 2 * capacity);
        cap        = (cap + 63) / 64 * 64; // every array starts on a 256-byte boundary
        RYO_CUDA(cudaMalloc(&block, (kArenaArrays + 1) * cap * sizeof(float)));
        for (int k = 0; k < kArenaArrays; ++k)
            a[k] = static_cast<float*>(block) + size_t(k) * cap;
        id       = reinterpret_cast<uint32_t*>(static_cast<float*>(block) + size_t(kArenaArrays) * cap);
        capacity = cap;
    }
    void release()
    {
        release_();
        capacity = 0;
    }

private:
    void release_()
    {
        if (block) cudaFree(block);
        block = nullptr;
        for (int k = 0; k < kArenaArrays; ++k)
            a[k] = nullptr;
        id = nullptr;
    }
};

struct ArenaPtrs
{
    float* a[kArenaArrays];
    uint32_t* id;
};

/*! copy the bodies of the surviving requests: request r's bodies are the range [virtFirst[r], virtFirst[r + 1]) of
 *  the survivors taken in their new order; they move from srcFirst[r] to dstFirst[r] (newly admitted requests may
 *  sit between the destination ranges) */
__global__ void engineCompact(ArenaPtrs src, ArenaPtrs dst, const uint64_t* __restrict__ virtFirst,
                              const uint64_t* __restrict__ dstFirst, const uint64_t* __restrict__ srcFirst,
                              uint32_t numReq, uint64_t total)
{
    size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x; v < total; v += stride)
    {
        uint32_t lo = 0, hi = numReq - 1;
        while (lo < hi)
        {
            uint32_t mid = (lo + hi + 1) >> 1;
            if (virtFirst[mid] <= v) lo = mid;
            else hi = mid - 1;
        }
        size_t off = v - virtFirst[lo];
        size_t j   = srcFirst[lo] + off;
        size_t i   = dstFirst[lo] + off;
#pragma unroll
        for (int k = 0; k < kArenaArrays; ++k)
            dst.a[k][i] = src.a[k][j];
        dst.id[i] = src.id[j];
    }
}

__global__ void engineIota(uint32_t* id, uint64_t first, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) id[first + i] = i;
}

struct EngineSys
{
    float halfDt, dt;
    int stepping; // 1: this step kicks and drifts the system
    int periodic;
    float lo[3], len[3];
};

__device__ __forceinline__ uint32_t engineSystemOf(const uint64_t* __restrict__ first, uint32_t numSystems, uint64_t i)
{
    uint32_t lo = 0, hi = numSystems - 1;
    while (lo < hi)
    {
        uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(first + mid) <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

//! first half kick and drift of the stepping systems; periodic systems wrap back into their box
__global__ void engineKickDrift(ArenaPtrs A, uint64_t n, const uint64_t* __restrict__ first, uint32_t numSystems,
                                const EngineSys* __restrict__ sys)
{
    size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    {
        const EngineSys& S = sys[engineSystemOf(first, numSystems, i)];
        if (!S.stepping) continue;
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            float v  = A.a[5 + d][i] + S.halfDt * A.a[8 + d][i];
            float x  = A.a[d][i] + S.dt * v;
            if (S.periodic)
            {
                float r = x - S.lo[d];
                r -= S.len[d] * floorf(r / S.len[d]);
                if (!(r < S.len[d])) r = 0.f; // rounding can land exactly on the upper face
                x = S.lo[d] + r;
            }
            A.a[5 + d][i] = v;
            A.a[d][i]     = x;
        }
    }
}

//! second half kick of the stepping systems, then per-system kinetic energy (FP64)
__global__ void engineKick(ArenaPtrs A, uint64_t n, const uint64_t* __restrict__ first, uint32_t numSystems,
                           const EngineSys* __restrict__ sys, double* __restrict__ kinetic)
{
    size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    {
        uint32_t s         = engineSystemOf(first, numSystems, i);
        const EngineSys& S = sys[s];
        double v2          = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            float v = A.a[5 + d][i];
            if (S.stepping) v += S.halfDt * A.a[8 + d][i];
            A.a[5 + d][i] = v;
            v2 += double(v) * v;
        }
        double ke = 0.5 * double(A.a[3][i]) * v2;
        // neighbouring threads usually share the system: reduce over the warp's runs of equal s
        unsigned peers = __match_any_sync(__activemask(), s);
        int leader     = __ffs(peers) - 1;
        for (int o = 16; o > 0; o >>= 1)
        {
            double other = __shfl_down_sync(__activemask(), ke, o);
            int src      = int(threadIdx.x & 31) + o;
            if (src < 32 && ((peers >> src) & 1u)) ke += other;
        }
        if (int(threadIdx.x & 31) == leader) atomicAdd(kinetic + s, ke);
    }
}

//! gather ids by the permutation of the solve (order[i] = previous index of body i)
__global__ void engineGatherIds(const uint32_t* __restrict__ order, const uint32_t* __restrict__ in,
                                uint32_t* __restrict__ out, uint64_t n)
{
    size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = in[order[i]];
}

//! final state of one request in submission order: out[k][id[i]] = arena[k][first + i] for x y z vx vy vz ax ay az p
__global__ void engineScatterResult(ArenaPtrs A, uint64_t first, uint32_t n, float* __restrict__ out)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t j      = A.id[first + i];
    const int k[10] = {0, 1, 2, 5, 6, 7, 8, 9, 10, 11};
#pragma unroll
    for (int c = 0; c < 10; ++c)
        out[size_t(c) * n + j] = A.a[k[c]][first + i];
}

} // namespace ryo

using namespace ryo;

namespace
{

struct Request
{
    uint64_t tag;
    uint32_t n;
    ryo_system sys;
    int stepsLeft, stepsDone;
    float dt;
    bool haveForces;
    const float* in[8]; // host x y z m h vx vy vz (vx..vz may be null)
    float* out;         // host, 10 * n floats (may be null)
    double bytes;
    double e0;          // total energy after the initial forces
    uint64_t arenaFirst;
};

struct Arenas
{
    Arena buf[2];
    int cur = 0;
};

} // namespace

struct ryo_engine
{
    ryo_ctx* ctx;
    ryo_solve_params solve;
    double budget;
    double bytesPerBody;
    int maxSystems;
    uint64_t maxStepBodies = 0; // 0: every resident request steps every step
    uint32_t stepping      = 0; // with a cap: the resident requests (a prefix of the arena) the steps advance
    double used = 0;
    std::deque<Request> queue;
    std::vector<Request> resident;
    std::vector<ryo_engine_result> done;
    Arenas arenas;
    uint64_t residentBodies = 0;
    bool changed            = false;
    uint64_t solves         = 0;
    std::string lastError;

    ~ryo_engine()
    {
        arenas.buf[0].release();
        arenas.buf[1].release();
    }
};

namespace
{
ArenaPtrs ptrsOf(const Arena& a)
{
    ArenaPtrs p;
    for (int k = 0; k < kArenaArrays; ++k)
        p.a[k] = a.a[k];
    p.id = a.id;
    return p;
}

unsigned gridFor(size_t n, int sms)
{
    size_t want = (n + 255) / 256;
    size_t cap  = size_t(sms) * 16;
    return unsigned(std::max<size_t>(1, std::min(want, cap)));
}

//! the work a request has left: bodies times the force evaluations still to come
double remainingWork(const Request& q) { return double(q.n) * double(q.stepsLeft + (q.haveForces ? 0 : 1)); }

/*! rebuild the arena with the survivors and the newly admitted requests in one order. When steps are capped, the
 *  requests the next steps advance come first: taken in the order of their remaining work (least first), each one
 *  that still fits the cap joins (the first always does); the rest follow. Without a cap: survivors first, then the
 *  admitted in arrival order. Survivors are compacted on the device, admitted ones copied in. */
void rebuildArena(ryo_engine* E, std::vector<Request>& admitted, cudaStream_t s)
{
    Arena& src = E->arenas.buf[E->arenas.cur];
    Arena& dst = E->arenas.buf[1 - E->arenas.cur];
    std::vector<std::pair<Request, bool>> all; // (request, admitted now)
    for (auto& r : E->resident)
        all.emplace_back(r, false);
    for (auto& r : admitted)
        all.emplace_back(r, true);
    E->stepping = uint32_t(all.size());
    if (E->maxStepBodies > 0)
    {
        std::stable_sort(all.begin(), all.end(), [](const auto& a, const auto& b)
                         { return remainingWork(a.first) < remainingWork(b.first); });
        std::vector<char> take(all.size(), 0);
        uint64_t bodies = 0;
        for (size_t k = 0; k < all.size(); ++k)
            if (k == 0 || bodies + all[k].first.n <= E->maxStepBodies)
            {
                take[k] = 1;
                bodies += all[k].first.n;
            }
        std::vector<std::pair<Request, bool>> ordered;
        for (int pass = 1; pass >= 0; --pass)
            for (size_t k = 0; k < all.size(); ++k)
                if (take[k] == pass) ordered.push_back(all[k]);
        all.swap(ordered);
        E->stepping = uint32_t(std::count(take.begin(), take.end(), 1));
    }
    uint64_t total = 0;
    for (auto& r : all)
        total += r.first.n;
    dst.ensure(std::max<uint64_t>(total, 1));
    std::vector<uint64_t> vf, df, sf; // survivors: virtual, destination and source offsets
    uint64_t o = 0, survivors = 0;
    for (auto& [q, fresh] : all)
    {
        if (!fresh)
        {
            vf.push_back(survivors);
            df.push_back(o);
            sf.push_back(q.arenaFirst);
            survivors += q.n;
        }
        q.arenaFirst = o;
        o += q.n;
    }
    if (survivors > 0)
    {
        size_t k     = vf.size();
        uint64_t* d = E->ctx->scratch<uint64_t>("eng.compact", 3 * k, s);
        RYO_CUDA(cudaMemcpyAsync(d, vf.data(), k * 8, cudaMemcpyHostToDevice, s));
        RYO_CUDA(cudaMemcpyAsync(d + k, df.data(), k * 8, cudaMemcpyHostToDevice, s));
        RYO_CUDA(cudaMemcpyAsync(d + 2 * k, sf.data(), k * 8, cudaMemcpyHostToDevice, s));
        engineCompact<<<gridFor(survivors, E->ctx->smCount), 256, 0, s>>>(ptrsOf(src), ptrsOf(dst), d, d + k,
                                                                         d + 2 * k, uint32_t(k), survivors);
        RYO_LAUNCH_CHECK();
    }
    for (auto& [r, fresh] : all)
    {
        if (!fresh) continue;
        for (int k = 0; k < 8; ++k)
        {
            if (r.in[k])
                RYO_CUDA(cudaMemcpyAsync(dst.a[k] + r.arenaFirst, r.in[k], r.n * sizeof(float),
                                         cudaMemcpyHostToDevice, s));
            else
                RYO_CUDA(cudaMemsetAsync(dst.a[k] + r.arenaFirst, 0, r.n * sizeof(float), s));
        }
        engineIota<<<ceilDiv(r.n, 256), 256, 0, s>>>(dst.id, r.arenaFirst, r.n);
        RYO_LAUNCH_CHECK();
    }
    E->resident.clear();
    for (auto& r : all)
        E->resident.push_back(r.first);
    E->arenas.cur     = 1 - E->arenas.cur;
    E->residentBodies = total;
}

//! a failed batched solve inside a step: its status and the context's message
struct SolveFailed
{
    ryo_status status;
    std::string msg;
};

ryo_status engineGuard(ryo_engine* E, const std::function<void()>& f)
{
    DeviceScope device(E->ctx->device);
    try
    {
        f();
        return RYO_OK;
    }
    catch (const SolveFailed& e)
    {
        E->lastError = e.msg;
        return e.status;
    }
    catch (const CudaError& e)
    {
        E->lastError = std::string(e.what) + ": " + cudaGetErrorString(e.err);
        return e.err == cudaErrorMemoryAllocation ? RYO_ERR_OOM : RYO_ERR_CUDA;
    }
    catch (const std::bad_alloc&)
    {
        E->lastError = "host allocation failed";
        return RYO_ERR_OOM;
    }
    catch (const std::exception& e)
    {
        // no exception may cross the C ABI
        E->lastError = std::string("internal error: ") + e.what();
        return RYO_ERR_INTERNAL;
    }
    catch (...)
    {
        E->lastError = "internal error";
        return RYO_ERR_INTERNAL;
    }
}
} // namespace

extern "C" void ryo_engine_params_default(ryo_engine_params* p)
{
    if (!p) return;
    *p = ryo_engine_params{};
    ryo_solve_params_default(&p->solve);
    p->hbmBudgetBytes = 120e9;
    p->bytesPerBody   = 256.0;
    p->maxSystems     = RYO_BATCH_MAX_SYSTEMS;
    p->reserveBodies  = 0;
    p->maxStepBodies  = uint64_t(7) << 20;
}

extern "C" ryo_status ryo_engine_create(ryo_ctx_t* ctx, const ryo_engine_params* p, ryo_engine_t** out)
{
    if (!ctx || !p || !out) return RYO_ERR_BAD_ARG;
    if (!(p->hbmBudgetBytes > 0) || !(p->bytesPerBody > 0) || p->maxSystems < 1 ||
        p->maxSystems > RYO_BATCH_MAX_SYSTEMS)
        return RYO_ERR_BAD_ARG;
    ryo_engine* E = nullptr;
    DeviceScope device(ctx->device);
    try
    {
        E               = new ryo_engine();
        E->ctx          = ctx;
        E->solve        = p->solve;
        E->budget       = p->hbmBudgetBytes;
        E->bytesPerBody = p->bytesPerBody;
        E->maxSystems   = p->maxSystems;
        E->maxStepBodies = p->maxStepBodies;
        if (p->reserveBodies > 0)
        {
            E->arenas.buf[0].ensure(p->reserveBodies);
            E->arenas.buf[1].ensure(p->reserveBodies);
        }
        *out = E;
        return RYO_OK;
    }
    catch (const std::bad_alloc&)
    {
        delete E;
        return RYO_ERR_OOM;
    }
    catch (const CudaError& e)
    {
        ctx->lastError = std::string("engine_create: ") + e.what + ": " + cudaGetErrorString(e.err);
        delete E;
        return e.err == cudaErrorMemoryAllocation ? RYO_ERR_OOM : RYO_ERR_CUDA;
    }
    catch (...)
    {
        ctx->lastError = "engine_create: internal error";
        delete E;
        return RYO_ERR_INTERNAL;
    }
}

extern "C" void ryo_engine_destroy(ryo_engine_t* E)
{
    if (!E) return;
    DeviceScope device(E->ctx->device);
    cudaDeviceSynchronize();
    delete E;
}

extern "C" const char* ryo_engine_last_error(const ryo_engine_t* E) { return E ? E->lastError.c_str() : ""; }

extern "C" ryo_status ryo_engine_submit(ryo_engine_t* E, const ryo_engine_request* r)
{
    if (!E || !r) return RYO_ERR_BAD_ARG;
    if (!r->x || !r->y || !r->z || !r->m || !r->h || r->numBodies < 1 || r->numSteps < 0 || !(r->dt >= 0.f))
    {
        E->lastError = "engine_submit: bad request";
        return RYO_ERR_BAD_ARG;
    }
    if (r->useBox)
    {
        const float* l = r->box.limits;
        for (int d = 0; d < 3; ++d)
            if (!(l[2 * d + 1] > l[2 * d]))
            {
                E->lastError = "engine_submit: every box axis needs max > min";
                return RYO_ERR_BAD_ARG;
            }
        // the batched solve's checks of a periodic system, made here so that one bad request cannot fail every
        // step of the requests resident beside it
        const int* b = r->box.boundary;
        if (b[0] == RYO_BOUNDARY_PERIODIC && b[1] == RYO_BOUNDARY_PERIODIC && b[2] == RYO_BOUNDARY_PERIODIC)
        {
            DevBox<float> box = makeDevBox<float>(l, 1);
            if (!(box.len[0] == box.len[1] && box.len[1] == box.len[2]))
            {
                E->lastError = "engine_submit: Ewald needs a cubic periodic box";
                return RYO_ERR_NOT_CUBIC;
            }
            if (r->numShells < 0 || r->numShells > 4)
            {
                E->lastError = "engine_submit: numShells in [0, 4]";
                return RYO_ERR_BAD_ARG;
            }
            // the engine's Ewald settings apply to periodic requests only, as in the single-system solve
            if (const char* why = ewaldSettingsError(E->solve.ewald))
            {
                E->lastError = std::string("engine_submit: ") + why;
                return RYO_ERR_BAD_ARG;
            }
        }
    }
    Request q{};
    q.tag                = r->tag;
    q.n                  = r->numBodies;
    q.sys.numBodies      = r->numBodies;
    q.sys.useBox         = r->useBox;
    q.sys.box            = r->box;
    q.sys.numShells      = r->numShells;
    q.stepsLeft          = r->numSteps;
    q.dt                 = r->dt;
    const float* in[8]   = {r->x, r->y, r->z, r->m, r->h, r->vx, r->vy, r->vz};
    for (int k = 0; k < 8; ++k)
        q.in[k] = in[k];
    q.out   = r->out;
    q.bytes = E->bytesPerBody * double(r->numBodies);
    if (q.bytes > E->budget)
    {
        E->lastError = "engine_submit: the request alone exceeds the HBM budget";
        return RYO_ERR_CAPACITY;
    }
    try
    {
        E->queue.push_back(q);
    }
    catch (const std::bad_alloc&)
    {
        E->lastError = "engine_submit: host allocation failed";
        return RYO_ERR_OOM;
    }
    return RYO_OK;
}

extern "C" ryo_status ryo_engine_step(ryo_engine_t* E, ryo_engine_step_info* info, ryo_stream_t stream)
{
    if (!E) return RYO_ERR_BAD_ARG;
    return engineGuard(E,
                       [&]
                       {
                           cudaStream_t s = stream;
                           ryo_engine_step_info st{};
                           using Clock = std::chrono::steady_clock;
                           auto since  = [](Clock::time_point t0)
                           { return float(std::chrono::duration<double, std::milli>(Clock::now() - t0).count()); };
                           auto t0 = Clock::now();
                           // admission: arrival order, while the budget and the system slots allow
                           std::vector<Request> admitted;
                           while (!E->queue.empty() &&
                                  int(E->resident.size() + admitted.size()) < E->maxSystems &&
                                  E->used + E->queue.front().bytes <= E->budget)
                           {
                               E->used += E->queue.front().bytes;
                               admitted.push_back(E->queue.front());
                               E->queue.pop_front();
                           }
                           st.admitted = int(admitted.size());
                           if (!admitted.empty() || E->changed) rebuildArena(E, admitted, s);
                           E->changed = false;
                           st.resident       = int(E->resident.size());
                           st.residentBodies = E->residentBodies;
                           st.queued         = int(E->queue.size());
                           if (E->resident.empty())
                           {
                               if (info) *info = st;
                               return;
                           }
                           // the requests this step advances: all, or those the last rebuild chose (the arena's
                           // first E->stepping requests; while none of them retires the choice stands)
                           const uint32_t nsAll = uint32_t(E->resident.size());
                           uint32_t ns          = nsAll;
                           uint64_t n           = E->residentBodies;
                           if (E->maxStepBodies > 0)
                           {
                               ns = std::min(E->stepping, nsAll);
                               n  = 0;
                               for (uint32_t k = 0; k < ns; ++k)
                                   n += E->resident[k].n;
                           }
                           Arena& A    = E->arenas.buf[E->arenas.cur];
                           ArenaPtrs P = ptrsOf(A);

                           std::vector<ryo_system> sys(ns);
                           std::vector<EngineSys> es(ns);
                           std::vector<uint64_t> first(ns + 1);
                           for (uint32_t k = 0; k < ns; ++k)
                           {
                               Request& q          = E->resident[k];
                               sys[k]              = q.sys;
                               sys[k].firstBody    = q.arenaFirst;
                               first[k]            = q.arenaFirst;
                               EngineSys& e        = es[k];
                               e.dt                = q.dt;
                               e.halfDt            = 0.5f * q.dt;
                               e.stepping          = q.haveForces ? 1 : 0;
                               bool periodic       = q.sys.useBox && q.sys.box.boundary[0] == RYO_BOUNDARY_PERIODIC &&
                                               q.sys.box.boundary[1] == RYO_BOUNDARY_PERIODIC &&
                                               q.sys.box.boundary[2] == RYO_BOUNDARY_PERIODIC;
                               e.periodic          = periodic ? 1 : 0;
                               for (int d = 0; d < 3; ++d)
                               {
                                   e.lo[d]  = q.sys.box.limits[2 * d];
                                   e.len[d] = q.sys.box.limits[2 * d + 1] - q.sys.box.limits[2 * d];
                               }
                           }
                           first[ns]          = n;
                           uint64_t* dFirst   = E->ctx->scratch<uint64_t>("eng.first", ns + 1, s);
                           EngineSys* dSys    = E->ctx->scratch<EngineSys>("eng.sys", ns, s);
                           double* dKin       = E->ctx->scratch<double>("eng.kinetic", ns, s);
                           RYO_CUDA(cudaMemcpyAsync(dFirst, first.data(), 8 * (ns + 1), cudaMemcpyHostToDevice, s));
                           RYO_CUDA(cudaMemcpyAsync(dSys, es.data(), sizeof(EngineSys) * ns, cudaMemcpyHostToDevice,
                                                    s));
                           RYO_CUDA(cudaMemsetAsync(dKin, 0, sizeof(double) * ns, s));
                           engineKickDrift<<<gridFor(n, E->ctx->smCount), 256, 0, s>>>(P, n, dFirst, ns, dSys);
                           RYO_LAUNCH_CHECK();
                           st.hostMs[0] = since(t0);
                           auto t1      = Clock::now();

                           uint32_t* order = E->ctx->scratch<uint32_t>("eng.order", n, s);
                           std::vector<double> pe(ns);
                           ryo_solve_stats ss{};
                           ryo_status rs = ryo_solve_batch_f32(E->ctx, &E->solve, sys.data(), int(ns), P.a[0], P.a[1],
                                                               P.a[2], P.a[3], P.a[4], P.a[5], P.a[6], P.a[7], n,
                                                               P.a[11], P.a[8], P.a[9], P.a[10], order, pe.data(),
                                                               nullptr, &ss, s);
                           if (rs != RYO_OK)
                               throw SolveFailed{rs, "engine_step: batched solve failed: " + E->ctx->lastError};
                           st.hostMs[1] = since(t1);
                           auto t2      = Clock::now();
                           E->solves += ns;
                           uint32_t* idTmp = E->ctx->scratch<uint32_t>("eng.idtmp", n, s);
                           engineGatherIds<<<gridFor(n, E->ctx->smCount), 256, 0, s>>>(order, A.id, idTmp, n);
                           RYO_LAUNCH_CHECK();
                           RYO_CUDA(cudaMemcpyAsync(A.id, idTmp, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
                           engineKick<<<gridFor(n, E->ctx->smCount), 256, 0, s>>>(P, n, dFirst, ns, dSys, dKin);
                           RYO_LAUNCH_CHECK();
                           std::vector<double> ke(ns);
                           RYO_CUDA(cudaMemcpyAsync(ke.data(), dKin, sizeof(double) * ns, cudaMemcpyDeviceToHost, s));
                           RYO_CUDA(cudaStreamSynchronize(s));
                           st.hostMs[2] = since(t2);
                           auto t3      = Clock::now();

                           // advance the requests; retire the finished ones. Their final states are gathered into
                           // one device buffer and copied out with a single wait at the end of the step.
                           std::vector<Request> keep;
                           size_t outFloats = 0;
                           for (uint32_t k = 0; k < ns; ++k)
                           {
                               const Request& q = E->resident[k];
                               bool last        = q.haveForces ? q.stepsLeft <= 1 : q.stepsLeft <= 0;
                               if (last && q.out) outFloats += 10 * size_t(q.n);
                           }
                           float* results = outFloats ? E->ctx->scratch<float>("eng.result", outFloats, s) : nullptr;
                           size_t outAt   = 0;
                           for (uint32_t k = 0; k < ns; ++k)
                           {
                               Request& q = E->resident[k];
                               if (!q.haveForces)
                               {
                                   q.haveForces = true;
                                   q.e0         = ke[k] + pe[k];
                               }
                               else
                               {
                                   --q.stepsLeft;
                                   ++q.stepsDone;
                               }
                               if (q.stepsLeft > 0)
                               {
                                   keep.push_back(q);
                                   continue;
                               }
                               if (q.out)
                               {
                                   float* tmp = results + outAt;
                                   outAt += 10 * size_t(q.n);
                                   engineScatterResult<<<ceilDiv(q.n, 256), 256, 0, s>>>(P, q.arenaFirst, q.n, tmp);
                                   RYO_LAUNCH_CHECK();
                                   RYO_CUDA(cudaMemcpyAsync(q.out, tmp, 10 * size_t(q.n) * sizeof(float),
                                                            cudaMemcpyDeviceToHost, s));
                               }
                               ryo_engine_result res{};
                               res.tag             = q.tag;
                               res.numBodies       = q.n;
                               res.stepsDone       = q.stepsDone;
                               res.kineticEnergy   = ke[k];
                               res.potentialEnergy = pe[k];
                               res.initialEnergy   = q.e0;
                               E->done.push_back(res);
                               E->used -= q.bytes;
                               ++st.retired;
                               E->changed = true;
                           }
                           for (uint32_t k = ns; k < nsAll; ++k)
                               keep.push_back(E->resident[k]); // not advanced this step
                           if (outAt) RYO_CUDA(cudaStreamSynchronize(s));
                           E->resident.swap(keep);
                           st.hostMs[3] = since(t3);
                           st.solved    = int(ns);
                           st.retries   = int(ss.retries);
                           st.sumP2P    = ss.sumP2P;
                           st.maxP2P    = ss.maxP2P;
                           st.sumM2P    = ss.sumM2P;
                           st.maxM2P    = ss.maxM2P;
                           for (int i = 0; i < 6; ++i)
                               st.ms[i] = ss.ms[i];
                           if (info) *info = st;
                       });
}

extern "C" ryo_status ryo_engine_poll(ryo_engine_t* E, ryo_engine_result* out, int capacity, int* count)
{
    if (!E || !count || capacity < 0 || (capacity > 0 && !out)) return RYO_ERR_BAD_ARG;
    int c = std::min<int>(capacity, int(E->done.size()));
    for (int i = 0; i < c; ++i)
        out[i] = E->done[i];
    E->done.erase(E->done.begin(), E->done.begin() + c);
    *count = c;
    return RYO_OK;
}

extern "C" ryo_status ryo_engine_status(const ryo_engine_t* E, int* queued, int* resident, double* bytesInUse)
{
    if (!E) return RYO_ERR_BAD_ARG;
    if (queued) *queued = int(E->queue.size());
    if (resident) *resident = int(E->resident.size());
    if (bytesInUse) *bytesInUse = E->used;
    return RYO_OK;
}
