/*
 * ryoanji-b200: Barnes-Hut traversal for double coordinates.
 *
 * Reference: the two double instantiations of ryoanji::traverse (ryoanji/src/ryoanji/nbody/traversal_gpu.cu:635-641):
 *   "f64"   (Tc, Th, Tm, Ta, Tf) = (double, double, double, double, double), multipoles in double;
 *   "mixed" (double, float, float, float, double), multipoles in float
 * (the caller side of OPAL-X / IPPL, whose particle positions are double), each with the quadrupole and the
 * monopole + dipole + quadrupole expansion. As in the reference, the MAC, the group box and the interaction sums
 * run in double and 1/sqrt is the single-precision rsqrt of the double argument (kernel.hpp:38-52); softenings
 * combine in Th and masses enter as Tm.
 *
 * The walk and the interaction rule are those of the float kernel (traverse.cu): persistent warps pull 64-body
 * groups, a depth-first stack of first-children in shared memory (4 entries, 32 cells, per step), split iff node and
 * close, approximate iff not close or (leaf, no bodies, non-zero MAC radius), direct iff close leaf; so the per-group
 * counts equal the reference's. Evaluation stages 32 sources (one per lane) in shared memory as doubles and each
 * lane sums them for its two targets in FP64 registers; the FP64 pipe is half the FP32 rate on B200, and this path
 * trades that rate for the callers' precision.
 */
#include "internal.hpp"

namespace ryo
{

constexpr int kT64Warps   = 4;
constexpr int kT64Threads = kT64Warps * kWarp;
constexpr int kT64M2PCap  = 2 * kWarp; // pending approximated cells (evaluated in rounds of 32)
constexpr int kT64LeafCap = 2 * kWarp; // pending direct leaves (evaluated when more than 32 are pending)
constexpr int kT64Stride  = 16;        // staged doubles per source: x, y, z, then 12 multipole values or m, h
constexpr int kT64Root    = -2;        // stack marker of a single-node tree

struct WarpSmem64
{
    int m2p[kT64M2PCap + kWarp];
    int2 leaves[kT64LeafCap + kWarp];
    int leafScan[kT64LeafCap + kWarp];
    double stage[kWarp * kT64Stride];
};

//! the reference's applyMAC (traversal_gpu.cu:77-84) in double with every operation rounded once
__device__ __forceinline__ bool macFails64(const double c[4], const double tc[3], const double ts[3])
{
    double d[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        double v = __dsub_rn(fabs(__dsub_rn(tc[k], c[k])), ts[k]);
        d[k]     = __dmul_rn(__dadd_rn(v, fabs(v)), 0.5);
    }
    return norm2Exact(d[0], d[1], d[2]) < c[3];
}

//! the reference's inverseSquareRoot(double): rsqrt.approx.ftz of the argument rounded to float
__device__ __forceinline__ double rsqrt64(double x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(float(x)));
    return double(y);
}

struct Acc64
{
    double phi, x, y, z;
};

//! P2P (kernel.hpp:99-120) in double, softening combined in Th
template<class Th>
__device__ __forceinline__ void p2p64(Acc64& a, double tx, double ty, double tz, Th th, double sx, double sy, double sz,
                                      double sm, Th sh)
{
    double dx = sx - tx, dy = sy - ty, dz = sz - tz;
    double r2 = dx * dx + dy * dy + dz * dz;
    Th hij    = th + sh;
    Th hh     = hij * hij;
    double re = r2 < double(hh) ? double(hh) : r2;
    double ir = rsqrt64(re);
    double m3 = sm * ir * (ir * ir);
    a.phi -= m3 * r2;
    a.x += dx * m3;
    a.y += dy * m3;
    a.z += dz * m3;
}

//! M2P (cartesian_qpole.hpp:152-176, and :321-348 for the dipole terms) in double; q holds 12 values
template<bool kDipole>
__device__ __forceinline__ void m2p64(Acc64& a, double tx, double ty, double tz, const double* s)
{
    double rx = tx - s[0], ry = ty - s[1], rz = tz - s[2];
    const double* q = s + 3; // mass, qxx, qxy, qxz, qyy, qyz, qzz, trace, px, py, pz
    double r2  = rx * rx + ry * ry + rz * rz;
    double rm1 = rsqrt64(r2);
    double rm2 = rm1 * rm1;
    double rm5 = rm2 * rm2 * rm1;
    double Qrx = rx * q[1] + ry * q[2] + rz * q[3];
    double Qry = rx * q[2] + ry * q[4] + rz * q[5];
    double Qrz = rx * q[3] + ry * q[5] + rz * q[6];
    double rQr = rx * Qrx + ry * Qry + rz * Qrz;
    double f   = (-2.5 * rQr * rm5 - q[0] * rm1) * rm2;
    if constexpr (!kDipole)
    {
        a.phi -= q[0] * rm1 + 0.5 * rm5 * rQr;
        a.x += rm5 * Qrx + f * rx;
        a.y += rm5 * Qry + f * ry;
        a.z += rm5 * Qrz + f * rz;
    }
    else
    {
        double PR = rx * q[8] + ry * q[9] + rz * q[10];
        a.phi += (-q[0] - PR * rm2) * rm1 - 0.5 * rm5 * rQr;
        a.x += rm5 * Qrx + f * rx + rm5 * (q[8] * r2 - 3.0 * PR * rx);
        a.y += rm5 * Qry + f * ry + rm5 * (q[9] * r2 - 3.0 * PR * ry);
        a.z += rm5 * Qrz + f * rz + rm5 * (q[10] * r2 - 3.0 * PR * rz);
    }
}

template<class Th, class Tm, class Ta, class Tmp>
struct Trav64
{
    const double *xt, *yt, *zt, *xs, *ys, *zs;
    const Tm *mt, *ms;
    const Th *ht, *hs;
    const double* centers; // 4 per node: x, y, z, MAC r^2
    const Tmp* multipoles; // 8 or 12 per node
    Ta *p, *ax, *ay, *az;
};

//! evaluate the first @p count (<= 32) pending cells
template<bool kDipole, class Th, class Tm, class Ta, class Tmp>
__device__ void evalM2P64(WarpSmem64& S, int count, const Trav64<Th, Tm, Ta, Tmp>& A, const double tx[2],
                          const double ty[2], const double tz[2], Acc64 acc[2])
{
    constexpr int kVals = kDipole ? 12 : 8;
    const int lane      = laneId();
    if (lane < count)
    {
        int cell  = S.m2p[lane];
        double* s = S.stage + lane * kT64Stride;
        s[0]      = A.centers[4 * size_t(cell)];
        s[1]      = A.centers[4 * size_t(cell) + 1];
        s[2]      = A.centers[4 * size_t(cell) + 2];
#pragma unroll
        for (int k = 0; k < kVals; ++k)
            s[3 + k] = double(A.multipoles[kVals * size_t(cell) + k]);
    }
    __syncwarp();
    for (int j = 0; j < count; ++j)
    {
        const double* s = S.stage + j * kT64Stride;
#pragma unroll
        for (int t = 0; t < 2; ++t)
            m2p64<kDipole>(acc[t], tx[t], ty[t], tz[t], s);
    }
    __syncwarp();
}

//! evaluate every body of the @p numLeaves pending direct leaves, 32 per staging round
template<class Th, class Tm, class Ta, class Tmp>
__device__ void evalP2P64(WarpSmem64& S, int numLeaves, const Trav64<Th, Tm, Ta, Tmp>& A, const double tx[2],
                          const double ty[2], const double tz[2], const Th th[2], Acc64 acc[2])
{
    const int lane = laneId();
    int total      = 0;
    for (int base = 0; base < numLeaves; base += kWarp)
    {
        int i   = base + lane;
        int cnt = i < numLeaves ? S.leaves[i].y : 0;
        int inc = warpInclusiveScan(cnt) + total;
        if (i < numLeaves) S.leafScan[i] = inc;
        total = __shfl_sync(0xffffffffu, inc, kWarp - 1);
    }
    __syncwarp();
    for (int r0 = 0; r0 < total; r0 += kWarp)
    {
        int r = r0 + lane;
        if (r < total)
        {
            int lo = 0, hi = numLeaves - 1; // the first leaf whose inclusive prefix passes r
            while (lo < hi)
            {
                int mid = (lo + hi) >> 1;
                if (S.leafScan[mid] > r) hi = mid;
                else lo = mid + 1;
            }
            int2 lf   = S.leaves[lo];
            int body  = lf.x + (r - (S.leafScan[lo] - lf.y));
            double* s = S.stage + lane * kT64Stride;
            s[0]      = A.xs[body];
            s[1]      = A.ys[body];
            s[2]      = A.zs[body];
            s[3]      = double(A.ms[body]);
            reinterpret_cast<Th*>(s + 4)[0] = A.hs[body];
        }
        __syncwarp();
        int n = min(kWarp, total - r0);
        for (int j = 0; j < n; ++j)
        {
            const double* s = S.stage + j * kT64Stride;
            Th sh           = reinterpret_cast<const Th*>(s + 4)[0];
#pragma unroll
            for (int t = 0; t < 2; ++t)
                p2p64(acc[t], tx[t], ty[t], tz[t], th[t], s[0], s[1], s[2], s[3], sh);
        }
        __syncwarp();
    }
}

template<bool kDipole, class Th, class Tm, class Ta, class Tmp>
__global__ void __launch_bounds__(kT64Threads) traverseKernel64(TraverseLaunch P, Trav64<Th, Tm, Ta, Tmp> A)
{
    extern __shared__ __align__(16) unsigned char smemRaw[];
    const int warp = threadIdx.x / kWarp, lane = laneId();
    WarpSmem64& S  = reinterpret_cast<WarpSmem64*>(smemRaw)[warp];
    int* stack     = reinterpret_cast<int*>(smemRaw + sizeof(WarpSmem64) * kT64Warps) + warp * P.stackCapacity;
    const unsigned lt = lanemaskLt();

    while (true)
    {
        unsigned g = 0;
        if (lane == 0) g = atomicAdd(&P.ctl->workCounter, 1u);
        g = __shfl_sync(0xffffffffu, g, 0);
        if (g >= unsigned(P.numGroups)) return;
        const int b = int(P.groupStart[g]), e = int(P.groupEnd[g]);

        double px[2], py[2], pz[2];
        Th th[2];
#pragma unroll
        for (int t = 0; t < 2; ++t)
        {
            int i = min(b + t * kWarp + lane, e - 1);
            px[t] = A.xt[i];
            py[t] = A.yt[i];
            pz[t] = A.zt[i];
            th[t] = A.ht[i];
        }
        double tc[3], ts[3];
        {
            double lo[3] = {fmin(px[0], px[1]), fmin(py[0], py[1]), fmin(pz[0], pz[1])};
            double hi[3] = {fmax(px[0], px[1]), fmax(py[0], py[1]), fmax(pz[0], pz[1])};
#pragma unroll
            for (int d = 0; d < 3; ++d)
            {
                double l = warpMin(lo[d]), h = warpMax(hi[d]);
                tc[d]    = (h + l) * 0.5;
                ts[d]    = (h - l) * 0.5;
            }
        }
        Acc64 acc[2] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
        unsigned nM2P = 0, nP2P = 0;
        int maxStack  = 0;
        bool overflow = false;
        const int shells = P.numShells;
        for (int iz = -shells; iz <= shells && !overflow; ++iz)
            for (int iy = -shells; iy <= shells && !overflow; ++iy)
                for (int ix = -shells; ix <= shells && !overflow; ++ix)
                {
                    // as the float kernel: the group centre follows the reference's add/subtract sequence, the
                    // targets are the original positions plus the shift
                    double sh[3] = {ix * P.boxL64[0], iy * P.boxL64[1], iz * P.boxL64[2]};
                    double tx[2], ty[2], tz[2];
#pragma unroll
                    for (int t = 0; t < 2; ++t)
                    {
                        tx[t] = px[t] + sh[0];
                        ty[t] = py[t] + sh[1];
                        tz[t] = pz[t] + sh[2];
                    }
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        tc[d] += sh[d];

                    int sp = 1, nM = 0, nL = 0;
                    if (lane == 0) stack[0] = P.numNodes == 1 ? kT64Root : P.initNode;
                    __syncwarp();
                    while (sp > 0)
                    {
                        int k     = min(4, sp);
                        sp -= k;
                        int slot  = lane >> 3;
                        int entry = slot < k ? stack[sp + slot] : -1;
                        __syncwarp();
                        int cell = -1;
                        if (entry == kT64Root) cell = (lane & 7) == 0 ? 0 : -1;
                        else if (entry >= 0) cell = entry + (lane & 7);

                        bool valid   = cell >= 0;
                        double c[4]  = {0, 0, 0, 0};
                        int child = 0, first = 0, count = 0;
                        if (valid)
                        {
                            const double* cp = A.centers + 4 * size_t(cell);
                            c[0]             = cp[0];
                            c[1]             = cp[1];
                            c[2]             = cp[2];
                            c[3]             = cp[3];
                            child            = __ldg(P.childOffsets + cell);
                            if (child == 0)
                            {
                                int leaf = __ldg(P.internalToLeaf + cell);
                                first    = int(__ldg(P.layout + leaf));
                                count    = int(__ldg(P.layout + leaf + 1)) - first;
                            }
                        }
                        bool close  = valid && macFails64(c, tc, ts);
                        bool isNode = child != 0;
                        bool split  = close && isNode;
                        unsigned bs = __ballot_sync(0xffffffffu, split);
                        int nsplit  = __popc(bs);
                        if (sp + nsplit > P.stackCapacity)
                        {
                            overflow = true;
                            break;
                        }
                        if (split) stack[sp + __popc(bs & lt)] = child;
                        sp += nsplit;
                        maxStack = max(maxStack, sp);

                        bool direct = close && !isNode;
                        bool remote = direct && count == 0 && c[3] != 0.0;
                        bool approx = valid && (!close || remote);
                        nM2P += __popc(__ballot_sync(0xffffffffu, approx));
                        bool evalM  = approx && c[3] != 0.0;
                        unsigned bm = __ballot_sync(0xffffffffu, evalM);
                        if (evalM) S.m2p[nM + __popc(bm & lt)] = cell;
                        nM += __popc(bm);
                        bool hasB   = direct && count > 0;
                        unsigned bl = __ballot_sync(0xffffffffu, hasB);
                        if (hasB) S.leaves[nL + __popc(bl & lt)] = make_int2(first, count);
                        nL += __popc(bl);
                        nP2P += __reduce_add_sync(0xffffffffu, hasB ? unsigned(count) : 0u);
                        __syncwarp();
                        while (nM >= kWarp)
                        {
                            evalM2P64<kDipole>(S, kWarp, A, tx, ty, tz, acc);
                            nM -= kWarp;
                            if (lane < nM) S.m2p[lane] = S.m2p[kWarp + lane];
                            __syncwarp();
                        }
                        if (nL > kT64LeafCap - kWarp)
                        {
                            evalP2P64(S, nL, A, tx, ty, tz, th, acc);
                            nL = 0;
                        }
                    }
                    if (!overflow)
                    {
                        if (nM > 0) evalM2P64<kDipole>(S, nM, A, tx, ty, tz, acc);
                        if (nL > 0) evalP2P64(S, nL, A, tx, ty, tz, th, acc);
                    }
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        tc[d] -= sh[d];
                }

        if (overflow)
        {
            // write nothing; the host splits the group and traverses the halves again
            if (lane == 0)
            {
                unsigned slot = atomicAdd(&P.ctl->failedCount, 1u);
                if (slot < P.failedCapacity) P.failedGroups[slot] = g;
                atomicMax(&P.ctl->stats[kMaxStack], (unsigned long long)maxStack);
            }
            continue;
        }
        double pot = 0.0;
#pragma unroll
        for (int t = 0; t < 2; ++t)
        {
            int idx = b + t * kWarp + lane;
            if (idx < e)
            {
                double mi = double(A.mt[idx]);
                pot += mi * acc[t].phi;
                if (A.p) A.p[idx] += Ta(P.G64 * mi * acc[t].phi);
                A.ax[idx] += Ta(P.G64 * acc[t].x);
                A.ay[idx] += Ta(P.G64 * acc[t].y);
                A.az[idx] += Ta(P.G64 * acc[t].z);
            }
        }
        pot = warpSum(pot);
        if (lane == 0)
        {
            unsigned long long size = (unsigned long long)(e - b);
            atomicMax(&P.ctl->stats[kMaxP2P], (unsigned long long)nP2P);
            atomicAdd(&P.ctl->stats[kSumP2P], (unsigned long long)nP2P * size);
            atomicMax(&P.ctl->stats[kMaxM2P], (unsigned long long)nM2P);
            atomicAdd(&P.ctl->stats[kSumM2P], (unsigned long long)nM2P * size);
            atomicMax(&P.ctl->stats[kMaxStack], (unsigned long long)maxStack);
            atomicAdd(&P.ctl->potential, pot);
            if (P.groupM2P) P.groupM2P[g] = nM2P;
            if (P.groupP2P) P.groupP2P[g] = nP2P;
        }
    }
}

template<class Th, class Tm, class Ta, class Tmp>
static void launchTyped64(const TraverseLaunch& t, int smCount, cudaStream_t s)
{
    Trav64<Th, Tm, Ta, Tmp> A;
    A.xt = t.xt64, A.yt = t.yt64, A.zt = t.zt64, A.xs = t.xs64, A.ys = t.ys64, A.zs = t.zs64;
    A.mt = static_cast<const Tm*>(t.mt64), A.ms = static_cast<const Tm*>(t.ms64);
    A.ht = static_cast<const Th*>(t.ht64), A.hs = static_cast<const Th*>(t.hs64);
    A.centers    = t.centers64;
    A.multipoles = static_cast<const Tmp*>(t.multipoles64);
    A.p = static_cast<Ta*>(t.p64), A.ax = static_cast<Ta*>(t.ax64), A.ay = static_cast<Ta*>(t.ay64);
    A.az = static_cast<Ta*>(t.az64);
    auto kernel = t.mdqArrays ? traverseKernel64<true, Th, Tm, Ta, Tmp> : traverseKernel64<false, Th, Tm, Ta, Tmp>;
    size_t smem = sizeof(WarpSmem64) * kT64Warps + sizeof(int) * kT64Warps * size_t(t.stackCapacity);
    RYO_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int perSm = 0;
    RYO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, kT64Threads, smem));
    if (perSm < 1) perSm = 1;
    int want   = (t.numGroups + kT64Warps - 1) / kT64Warps;
    int blocks = min(want, perSm * smCount);
    kernel<<<blocks, kT64Threads, smem, s>>>(t, A);
    RYO_LAUNCH_CHECK();
}

void launchTraverse64(const TraverseLaunch& t, int smCount, cudaStream_t s)
{
    if (t.numGroups <= 0) return;
    if (t.precision == kPrecisionF64) launchTyped64<double, double, double, double>(t, smCount, s);
    else launchTyped64<float, float, float, float>(t, smCount, s);
}

} // namespace ryo
