/*
 * ryoanji-b200: upward pass — centres of mass, cartesian quadrupoles, MAC radii, traversal node records.
 *
 * Reference: cstone/include/cstone/focus/source_center_gpu.cu:103-310 (centres, setMac) and
 * ryoanji/src/ryoanji/nbody/upsweep_gpu.cu:33-128 (P2M, M2M), with the formulas of
 * ryoanji/src/ryoanji/nbody/cartesian_qpole.hpp:67-235. Sums run in double precision and are rounded to float once
 * per stored value; the MAC radius is computed in float from the stored float centre, as the reference does.
 *
 * The solver path uses one fused pass: eight lanes per leaf read the leaf's bodies once and accumulate, relative to
 * the leaf's first body, the fourteen sums that give both the centre of mass (weights |m|) and the second moments
 * about it; the last of eight siblings to finish combines them into the parent (parallel-axis theorem in double)
 * and climbs on, so the whole tree is reduced in one launch without per-level host loops.
 */
#include "internal.hpp"

namespace ryo
{

constexpr int kTpl = 8; // lanes per leaf

template<class T>
__device__ inline T groupSum8(T v)
{
#pragma unroll
    for (int o = 1; o < kTpl; o <<= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ------------------------------------------------------------------------------------------------ reference steps
//
// The reference instantiates its step functions for three type sets (coordinates Tc, masses Tm, centres Tf,
// multipole values Tmp): all float, all double, and double coordinates and centres with float masses and multipoles
// (cstone/include/cstone/focus/source_center_gpu.cu:164-170, ryoanji/src/ryoanji/nbody/upsweep_gpu.cu:134-143). The
// kernels below take the same sets; their sums run in double in every set and are rounded once per stored value.

//! a node centre (x, y, z, |m| or MAC r^2) of type T: float4 for float, four aligned doubles otherwise
template<class T>
struct alignas(4 * sizeof(T)) Center4
{
    T x, y, z, w;
};
template<class T>
using CenterOf = std::conditional_t<std::is_same_v<T, float>, float4, Center4<T>>;

template<class T>
__device__ __forceinline__ CenterOf<T> makeCenter(double x, double y, double z, double w)
{
    return CenterOf<T>{T(x), T(y), T(z), T(w)};
}

template<class Tc, class Tm, class Tf>
__global__ void leafCentersKernel(const Tc* __restrict__ x, const Tc* __restrict__ y, const Tc* __restrict__ z,
                                  const Tm* __restrict__ m, const int* __restrict__ leafToInternal, int numLeaves,
                                  const uint32_t* __restrict__ layout, CenterOf<Tf>* __restrict__ centers)
{
    int tid  = blockIdx.x * blockDim.x + threadIdx.x;
    int leaf = tid / kTpl;
    double c[4] = {0, 0, 0, 0};
    if (leaf < numLeaves)
    {
        for (uint32_t i = layout[leaf] + tid % kTpl; i < layout[leaf + 1]; i += kTpl)
        {
            double w = fabs(double(m[i]));
            c[0] += w * x[i];
            c[1] += w * y[i];
            c[2] += w * z[i];
            c[3] += w;
        }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
        c[k] = groupSum8(c[k]);
    if (leaf < numLeaves && tid % kTpl == 0)
    {
        double inv = c[3] != 0.0 ? 1.0 / c[3] : 1.0;
        centers[leafToInternal[leaf]] = makeCenter<Tf>(c[0] * inv, c[1] * inv, c[2] * inv, c[3]);
    }
}

template<class Tf>
__global__ void upsweepCentersKernel(int first, int last, const int* __restrict__ childOffsets, CenterOf<Tf>* centers)
{
    int i = first + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= last) return;
    int fc = childOffsets[i];
    if (!fc) return;
    double c[4] = {0, 0, 0, 0};
    for (int k = fc; k < fc + 8; ++k)
    {
        CenterOf<Tf> ck = centers[k];
        double w        = fabs(double(ck.w));
        c[0] += w * ck.x;
        c[1] += w * ck.y;
        c[2] += w * ck.z;
        c[3] += w;
    }
    double inv = c[3] != 0.0 ? 1.0 / c[3] : 1.0;
    centers[i] = makeCenter<Tf>(c[0] * inv, c[1] * inv, c[2] * inv, c[3]);
}

//! traceless x3 form with the trace in the last slot (cartesian_qpole.hpp:92-108)
template<class Tmp>
__device__ inline void finalizeQuad(const double raw[7], Tmp* out)
{
    double tr = raw[1] + raw[4] + raw[6];
    out[0]    = Tmp(raw[0]);
    out[1]    = Tmp(3 * raw[1] - tr);
    out[2]    = Tmp(3 * raw[2]);
    out[3]    = Tmp(3 * raw[3]);
    out[4]    = Tmp(3 * raw[4] - tr);
    out[5]    = Tmp(3 * raw[5]);
    out[6]    = Tmp(3 * raw[6] - tr);
    out[7]    = Tmp(tr);
}

//! leaf expansions (P2M_add / P2M_finalize, cartesian_qpole.hpp:67-108; with kMDQ the dipole of :237-303 too)
template<class Tc, class Tm, class Tf, class Tmp, bool kMDQ>
__global__ void leafMultipolesKernel(const Tc* __restrict__ x, const Tc* __restrict__ y, const Tc* __restrict__ z,
                                     const Tm* __restrict__ m, const int* __restrict__ leafToInternal, int numLeaves,
                                     const uint32_t* __restrict__ layout, const CenterOf<Tf>* __restrict__ centers,
                                     Tmp* __restrict__ multipoles)
{
    constexpr int kTerms = kMDQ ? 10 : 7; // mass, xx, xy, xz, yy, yz, zz (, px, py, pz)
    int tid  = blockIdx.x * blockDim.x + threadIdx.x;
    int leaf = tid / kTpl;
    double q[kTerms] = {};
    int node         = 0;
    if (leaf < numLeaves)
    {
        node           = leafToInternal[leaf];
        CenterOf<Tf> c = centers[node];
        for (uint32_t i = layout[leaf] + tid % kTpl; i < layout[leaf + 1]; i += kTpl)
        {
            double rx = double(x[i]) - c.x, ry = double(y[i]) - c.y, rz = double(z[i]) - c.z, mi = m[i];
            q[0] += mi;
            q[1] += rx * rx * mi;
            q[2] += rx * ry * mi;
            q[3] += rx * rz * mi;
            q[4] += ry * ry * mi;
            q[5] += ry * rz * mi;
            q[6] += rz * rz * mi;
            if constexpr (kMDQ)
            {
                q[7] += mi * rx;
                q[8] += mi * ry;
                q[9] += mi * rz;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < kTerms; ++k)
        q[k] = groupSum8(q[k]);
    if (leaf < numLeaves && tid % kTpl == 0)
    {
        Tmp* o = multipoles + (kMDQ ? 12 : 8) * size_t(node);
        finalizeQuad(q, o);
        if constexpr (kMDQ)
        {
            o[8]  = Tmp(q[7]);
            o[9]  = Tmp(q[8]);
            o[10] = Tmp(q[9]);
            o[11] = Tmp(0);
        }
    }
}

/*! M2M of cells [first, last) from their eight children, double sums: the quadrupole's parallel-axis theorem
 *  (addQuadrupole, cartesian_qpole.hpp:187-235) and, with kMDQ, the dipole terms of cartesian_qpole.hpp:352-418 */
template<class Tf, class Tmp, bool kMDQ>
__global__ void upsweepMultipolesKernel(int first, int last, const int* __restrict__ childOffsets,
                                        const CenterOf<Tf>* __restrict__ centers, Tmp* multipoles)
{
    constexpr int kVals = kMDQ ? 12 : 8;
    int i = first + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= last) return;
    int fc = childOffsets[i];
    if (!fc) return;
    CenterOf<Tf> cp = centers[i];
    double acc[11]  = {};
    for (int k = fc; k < fc + 8; ++k)
    {
        CenterOf<Tf> ck = centers[k];
        const Tmp* a    = multipoles + kVals * size_t(k);
        double rx = double(cp.x) - ck.x, ry = double(cp.y) - ck.y, rz = double(cp.z) - ck.z;
        double r2 = (rx * rx + ry * ry + rz * rz) * (1.0 / 3.0);
        double ml = double(a[0]) * 3;
        if constexpr (!kMDQ)
        {
            acc[7] += a[7] + ml * r2;
            acc[0] += a[0];
            acc[1] += a[1] + ml * (rx * rx - r2);
            acc[2] += a[2] + ml * rx * ry;
            acc[3] += a[3] + ml * rx * rz;
            acc[4] += a[4] + ml * (ry * ry - r2);
            acc[5] += a[5] + ml * ry * rz;
            acc[6] += a[6] + ml * (rz * rz - r2);
        }
        else
        {
            double px = a[8], py = a[9], pz = a[10];
            double dip = rx * px + ry * py + rz * pz;
            acc[7] += a[7] + ml * r2 - 2.0 * dip;
            acc[0] += a[0];
            acc[8] += px - double(a[0]) * rx;
            acc[9] += py - double(a[0]) * ry;
            acc[10] += pz - double(a[0]) * rz;
            acc[1] += a[1] + ml * (rx * rx - r2) - 6.0 * rx * px + 2.0 * dip;
            acc[2] += a[2] + ml * rx * ry - 3.0 * (rx * py + ry * px);
            acc[3] += a[3] + ml * rx * rz - 3.0 * (rx * pz + rz * px);
            acc[4] += a[4] + ml * (ry * ry - r2) - 6.0 * ry * py + 2.0 * dip;
            acc[5] += a[5] + ml * ry * rz - 3.0 * (ry * pz + rz * py);
            acc[6] += a[6] + ml * (rz * rz - r2) - 6.0 * rz * pz + 2.0 * dip;
        }
    }
    Tmp* o = multipoles + kVals * size_t(i);
#pragma unroll
    for (int k = 0; k < (kMDQ ? 11 : 8); ++k)
        o[k] = Tmp(acc[k]);
    if constexpr (kMDQ) o[11] = Tmp(0);
}

template<class T>
__global__ void setMacKernel(const uint64_t* __restrict__ prefixes, int numNodes, CenterOf<T>* centers, float invTheta,
                             DevBox<T> box)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= numNodes) return;
    CenterOf<T> c = centers[i];
    T com[3]      = {c.x, c.y, c.z};
    T mac         = vecMacR2(prefixes[i], com, invTheta, box);
    centers[i].w  = (c.w != T(0)) ? mac : T(0);
}

template<class Tc, class Tm, class Tf>
void launchLeafCenters(const Tc* x, const Tc* y, const Tc* z, const Tm* m, const int* leafToInternal, int numLeaves,
                       const uint32_t* layout, Tf* centers, cudaStream_t s)
{
    if (numLeaves <= 0) return;
    leafCentersKernel<Tc, Tm, Tf><<<ceilDiv(size_t(numLeaves) * kTpl, 256), 256, 0, s>>>(
        x, y, z, m, leafToInternal, numLeaves, layout, reinterpret_cast<CenterOf<Tf>*>(centers));
    RYO_LAUNCH_CHECK();
}

template<class Tf>
void launchUpsweepCenters(int first, int last, const int* childOffsets, Tf* centers, cudaStream_t s)
{
    if (last <= first) return;
    upsweepCentersKernel<Tf><<<ceilDiv(last - first, 256), 256, 0, s>>>(first, last, childOffsets,
                                                                        reinterpret_cast<CenterOf<Tf>*>(centers));
    RYO_LAUNCH_CHECK();
}

template<class Tc, class Tm, class Tf, class Tmp>
void launchLeafMultipoles(const Tc* x, const Tc* y, const Tc* z, const Tm* m, const int* leafToInternal,
                          int numLeaves, const uint32_t* layout, const Tf* centers, Tmp* multipoles, bool mdq,
                          cudaStream_t s)
{
    if (numLeaves <= 0) return;
    auto kernel = mdq ? leafMultipolesKernel<Tc, Tm, Tf, Tmp, true> : leafMultipolesKernel<Tc, Tm, Tf, Tmp, false>;
    kernel<<<ceilDiv(size_t(numLeaves) * kTpl, 256), 256, 0, s>>>(
        x, y, z, m, leafToInternal, numLeaves, layout, reinterpret_cast<const CenterOf<Tf>*>(centers), multipoles);
    RYO_LAUNCH_CHECK();
}

template<class Tf, class Tmp>
void launchUpsweepMultipoles(int first, int last, const int* childOffsets, const Tf* centers, Tmp* multipoles, bool mdq,
                             cudaStream_t s)
{
    if (last <= first) return;
    auto kernel = mdq ? upsweepMultipolesKernel<Tf, Tmp, true> : upsweepMultipolesKernel<Tf, Tmp, false>;
    kernel<<<ceilDiv(last - first, 256), 256, 0, s>>>(first, last, childOffsets,
                                                      reinterpret_cast<const CenterOf<Tf>*>(centers), multipoles);
    RYO_LAUNCH_CHECK();
}

template<class T>
void launchSetMac(const uint64_t* prefixes, int numNodes, T* centers, float invTheta, const DevBox<T>& box,
                  cudaStream_t s)
{
    if (numNodes <= 0) return;
    setMacKernel<T><<<ceilDiv(numNodes, 256), 256, 0, s>>>(prefixes, numNodes,
                                                           reinterpret_cast<CenterOf<T>*>(centers), invTheta, box);
    RYO_LAUNCH_CHECK();
}

// the reference's three type sets (coordinates, masses, centres, multipole values)
template void launchLeafCenters(const float*, const float*, const float*, const float*, const int*, int,
                                const uint32_t*, float*, cudaStream_t);
template void launchLeafCenters(const double*, const double*, const double*, const double*, const int*, int,
                                const uint32_t*, double*, cudaStream_t);
template void launchLeafCenters(const double*, const double*, const double*, const float*, const int*, int,
                                const uint32_t*, double*, cudaStream_t);
template void launchUpsweepCenters(int, int, const int*, float*, cudaStream_t);
template void launchUpsweepCenters(int, int, const int*, double*, cudaStream_t);
template void launchLeafMultipoles(const float*, const float*, const float*, const float*, const int*, int,
                                   const uint32_t*, const float*, float*, bool, cudaStream_t);
template void launchLeafMultipoles(const double*, const double*, const double*, const double*, const int*, int,
                                   const uint32_t*, const double*, double*, bool, cudaStream_t);
template void launchLeafMultipoles(const double*, const double*, const double*, const float*, const int*, int,
                                   const uint32_t*, const double*, float*, bool, cudaStream_t);
template void launchUpsweepMultipoles(int, int, const int*, const float*, float*, bool, cudaStream_t);
template void launchUpsweepMultipoles(int, int, const int*, const double*, double*, bool, cudaStream_t);
template void launchUpsweepMultipoles(int, int, const int*, const double*, float*, bool, cudaStream_t);
template void launchSetMac(const uint64_t*, int, float*, float, const DevBox<float>&, cudaStream_t);
template void launchSetMac(const uint64_t*, int, double*, float, const DevBox<double>&, cudaStream_t);

// ------------------------------------------------------------------------------------------------ fused path

//! double-precision node summary kept during the fused upsweep (128 bytes, one line per node)
struct alignas(128) DNode
{
    double c[3]; // centre of mass (weights |m|)
    double w;    // sum |m|
    double m;    // sum m
    double q[6]; // second moments about c: xx, xy, xz, yy, yz, zz
    double p[3]; // dipole about c: sum m (x - c) (zero for positive masses; kept for signed ones)
    double pad[2];
};

__device__ inline void storeDNode(DNode* d, const double c[3], double w, double m, const double q[6],
                                  const double dp[3])
{
    double2* p = reinterpret_cast<double2*>(d);
    __stcg(p + 0, make_double2(c[0], c[1]));
    __stcg(p + 1, make_double2(c[2], w));
    __stcg(p + 2, make_double2(m, q[0]));
    __stcg(p + 3, make_double2(q[1], q[2]));
    __stcg(p + 4, make_double2(q[3], q[4]));
    __stcg(p + 5, make_double2(q[5], dp[0]));
    __stcg(p + 6, make_double2(dp[1], dp[2]));
}

__device__ inline void loadDNode(const DNode* d, double c[3], double& w, double& m, double q[6], double dp[3])
{
    const double2* p = reinterpret_cast<const double2*>(d);
    double2 a = __ldcg(p + 0), b = __ldcg(p + 1), e = __ldcg(p + 2), f = __ldcg(p + 3), g = __ldcg(p + 4),
            k = __ldcg(p + 5), l = __ldcg(p + 6);
    dp[0] = k.y;
    dp[1] = l.x;
    dp[2] = l.y;
    c[0] = a.x;
    c[1] = a.y;
    c[2] = b.x;
    w    = b.y;
    m    = e.x;
    q[0] = e.y;
    q[1] = f.x;
    q[2] = f.y;
    q[3] = g.x;
    q[4] = g.y;
    q[5] = k.x;
}

struct FusedArgs
{
    const float4* xyzm;
    const uint32_t* layout;
    const int* leafToInternal;
    const int* childOffsets;
    const int* parents;
    const uint64_t* prefixes;
    int numLeaves;
    int numNodes;
    float invTheta;
    DevBox<float> box;
    DNode* dn;
    NodeRecord* records;
    float4* centers;
    float* multipoles;
    double* root; // 11 doubles: centre (3) + finalized multipole (8)
    // internal nodes by the climb (arrival counters, non-null) or by level launches (null)
    unsigned int* arrivals;
    // batched systems: node keys carry a system prefix of sysLevel octree levels; sysBoxes[s] is the box of system
    // s, and sysRoots (11 doubles per system) receives the FP64 expansion of every system's root node
    const DevBox<float>* sysBoxes;
    int sysLevel;
    uint32_t numSystems; // system prefixes at or above this index belong to no system: their nodes are empty
    double* sysRoots;
    // monopole + dipole + quadrupole expansions: node dipoles (px, py, pz, 0) are written here when not null, and
    // the second moments are combined with the dipole terms of the parallel-axis theorem
    float4* dipoles;
};

//! FP64 centre and finalized quadrupole (11 doubles) of a node, as the Ewald setup reads them
__device__ inline void writeRootExpansion(double* out, const double c[3], const double raw[7])
{
    out[0]    = c[0];
    out[1]    = c[1];
    out[2]    = c[2];
    double tr = raw[1] + raw[4] + raw[6];
    out[3]    = raw[0];
    out[4]    = 3 * raw[1] - tr;
    out[5]    = 3 * raw[2];
    out[6]    = 3 * raw[3];
    out[7]    = 3 * raw[4] - tr;
    out[8]    = 3 * raw[5];
    out[9]    = 3 * raw[6] - tr;
    out[10]   = tr;
}

//! write the float outputs of a finished node; @p prefix is the node's, loaded by the caller ahead of its sums
__device__ void emitNode(const FusedArgs& A, int node, uint64_t prefix, const double c[3], double w, double m,
                         const double q[6], const double dp[3], int child, uint32_t firstBody, uint32_t count)
{
    if (A.dipoles) A.dipoles[node] = make_float4(float(dp[0]), float(dp[1]), float(dp[2]), 0.f);
    float com[3] = {float(c[0]), float(c[1]), float(c[2])};
    double raw[7] = {m, q[0], q[1], q[2], q[3], q[4], q[5]};
    float mac     = 0.f;
    if (!A.sysBoxes)
        mac = w != 0.0 && float(w) != 0.f ? vecMacR2(prefix, com, A.invTheta, A.box) : 0.f;
    else
    {
        // a node inside a system: its geometry is the system-local node (prefix without the system bits) in the
        // system's box; nodes above the system level mix systems and are never traversed
        int lvl         = prefixLength(prefix) / 3;
        if (lvl >= A.sysLevel)
        {
            uint64_t start    = prefixStart(prefix);
            int sysBits       = 3 * A.sysLevel;
            uint32_t sys      = uint32_t(start >> (63 - sysBits));
            uint64_t local    = (start << sysBits) & (kKeyEnd - 1);
            uint64_t localPre = encodePrefix(local, 3 * (lvl - A.sysLevel));
            // the tree holds all 8^sysLevel system-level nodes; those past the last system are empty leaves, and
            // sysBoxes and sysRoots have entries for real systems only
            if (sys < A.numSystems)
            {
                if (w != 0.0 && float(w) != 0.f) mac = vecMacR2(localPre, com, A.invTheta, A.sysBoxes[sys]);
                if (lvl == A.sysLevel && A.sysRoots) writeRootExpansion(A.sysRoots + 11 * size_t(sys), c, raw);
            }
        }
    }
    float qf[8];
    finalizeQuad(raw, qf);
    float4 cen = make_float4(com[0], com[1], com[2], mac);
    NodeRecord r;
    r.center = cen;
    r.q0     = make_float4(qf[0], qf[1], qf[2], qf[3]);
    r.q1     = make_float4(qf[4], qf[5], qf[6], qf[7]);
    r.link   = make_int4(child, int(firstBody), int(count), 0);
    A.records[node] = r;
    if (A.centers) A.centers[node] = cen;
    if (A.multipoles)
    {
        float4* mp = reinterpret_cast<float4*>(A.multipoles + 8 * size_t(node));
        mp[0]      = r.q0;
        mp[1]      = r.q1;
    }
    if (node == 0 && A.root) writeRootExpansion(A.root, c, raw);
}

//! sum over the eight lanes of a leaf group
__device__ __forceinline__ double groupSum8(double v, unsigned gmask)
{
#pragma unroll
    for (int o = 1; o < kTpl; o <<= 1)
        v += __shfl_xor_sync(gmask, v, o, kTpl);
    return v;
}

//! combine the eight children of @p node (parallel-axis theorem, double): lane @p sub of the group holds child sub
__device__ void combineChildren(const FusedArgs& A, int node, int fc, int sub, unsigned gmask)
{
    const uint64_t prefix = sub == 0 ? A.prefixes[node] : 0; // in flight with the children
    double cc[3], cw, cm, cq[6], cp[3];
    loadDNode(A.dn + fc + sub, cc, cw, cm, cq, cp);
    double w  = fabs(cw);
    double W  = groupSum8(w, gmask);
    double M  = groupSum8(cm, gmask);
    double sx = groupSum8(w * cc[0], gmask);
    double sy = groupSum8(w * cc[1], gmask);
    double sz = groupSum8(w * cc[2], gmask);
    double c[3];
    double inv = W != 0.0 ? 1.0 / W : 1.0;
    c[0]       = sx * inv;
    c[1]       = sy * inv;
    c[2]       = sz * inv;
    double dx = cc[0] - c[0], dy = cc[1] - c[1], dz = cc[2] - c[2];
    // dipole about the parent centre; the quadrupole-only expansion drops the dipole terms, as the reference's
    // 8-value M2M does (they vanish for positive masses)
    double px = cp[0], py = cp[1], pz = cp[2];
    if (!A.dipoles) px = py = pz = 0.0;
    double q[6], dp[3];
    q[0]  = groupSum8(cq[0] + cm * dx * dx + 2 * dx * px, gmask);
    q[1]  = groupSum8(cq[1] + cm * dx * dy + dx * py + dy * px, gmask);
    q[2]  = groupSum8(cq[2] + cm * dx * dz + dx * pz + dz * px, gmask);
    q[3]  = groupSum8(cq[3] + cm * dy * dy + 2 * dy * py, gmask);
    q[4]  = groupSum8(cq[4] + cm * dy * dz + dy * pz + dz * py, gmask);
    q[5]  = groupSum8(cq[5] + cm * dz * dz + 2 * dz * pz, gmask);
    dp[0] = groupSum8(cp[0] + cm * dx, gmask);
    dp[1] = groupSum8(cp[1] + cm * dy, gmask);
    dp[2] = groupSum8(cp[2] + cm * dz, gmask);
    if (sub == 0)
    {
        storeDNode(A.dn + node, c, W, M, q, dp);
        emitNode(A, node, prefix, c, W, M, q, dp, fc, 0, 0);
    }
}

/*! eight lanes per leaf: one pass over the bodies, P2M of the leaf (small register footprint, so many leaf groups
 *  stay resident per SM). The internal nodes follow by the climb (A.arrivals set: the group of the eighth sibling to
 *  arrive combines the parent, one child per lane, and goes on up) or level by level (levelCombineKernel). */
__global__ void __launch_bounds__(256, 4) fusedUpsweepKernel(FusedArgs A)
{
    int tid     = blockIdx.x * blockDim.x + threadIdx.x;
    int leaf    = tid / kTpl;
    int sub     = tid % kTpl;
    bool active = leaf < A.numLeaves;
    // two dependent rounds of loads: the leaf's range and node, then its bodies and the node's prefix. The sums are
    // taken relative to the leaf's first body, which lane 0 of the group loads as its own first body.
    uint32_t b0 = 0, b1 = 0;
    int node    = 0;
    if (active)
    {
        b0   = A.layout[leaf];
        b1   = A.layout[leaf + 1];
        node = A.leafToInternal[leaf];
    }
    const uint64_t prefix = active && sub == 0 ? A.prefixes[node] : 0;
    float4 b              = make_float4(0.f, 0.f, 0.f, 0.f);
    uint32_t i            = b0 + sub;
    if (i < b1) b = A.xyzm[i];
    float4 p0;
    p0.x = __shfl_sync(0xFFFFFFFFu, b.x, 0, kTpl);
    p0.y = __shfl_sync(0xFFFFFFFFu, b.y, 0, kTpl);
    p0.z = __shfl_sync(0xFFFFFFFFu, b.z, 0, kTpl);
    // sums relative to the first body: sum|m|, sum|m|d, sum m, sum m d, sum m d d^T
    double s[14] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (; i < b1; i += kTpl)
    {
        if (i != b0 + sub) b = A.xyzm[i];
        double dx = double(b.x) - p0.x, dy = double(b.y) - p0.y, dz = double(b.z) - p0.z;
        double mi = b.w, wi = fabs(mi);
        s[0] += wi;
        s[1] += wi * dx;
        s[2] += wi * dy;
        s[3] += wi * dz;
        s[4] += mi;
        s[5] += mi * dx;
        s[6] += mi * dy;
        s[7] += mi * dz;
        s[8] += mi * dx * dx;
        s[9] += mi * dx * dy;
        s[10] += mi * dx * dz;
        s[11] += mi * dy * dy;
        s[12] += mi * dy * dz;
        s[13] += mi * dz * dz;
    }
#pragma unroll
    for (int k = 0; k < 14; ++k)
        s[k] = groupSum8(s[k]);
    if (!active) return; // the eight lanes of a leaf group leave together

    double W = s[0], M = s[4];
    double c[3], q[6], dp[3];
    if (W != 0.0)
    {
        double inv = 1.0 / W;
        double ex = s[1] * inv, ey = s[2] * inv, ez = s[3] * inv; // centre relative to p0
        c[0] = double(p0.x) + ex;
        c[1] = double(p0.y) + ey;
        c[2] = double(p0.z) + ez;
        // sum m (d - e)(d - e)^T
        q[0] = s[8] - 2 * ex * s[5] + M * ex * ex;
        q[1] = s[9] - ex * s[6] - ey * s[5] + M * ex * ey;
        q[2] = s[10] - ex * s[7] - ez * s[5] + M * ex * ez;
        q[3] = s[11] - 2 * ey * s[6] + M * ey * ey;
        q[4] = s[12] - ey * s[7] - ez * s[6] + M * ey * ez;
        q[5] = s[13] - 2 * ez * s[7] + M * ez * ez;
        // sum m (d - e)
        dp[0] = s[5] - M * ex;
        dp[1] = s[6] - M * ey;
        dp[2] = s[7] - M * ez;
    }
    else
    {
        // zero total |m|: centre at the origin like the reference's normalisation; moments about it
        c[0] = c[1] = c[2] = 0.0;
        double ox = p0.x, oy = p0.y, oz = p0.z; // p0 - 0
        q[0] = s[8] + 2 * ox * s[5] + M * ox * ox;
        q[1] = s[9] + ox * s[6] + oy * s[5] + M * ox * oy;
        q[2] = s[10] + ox * s[7] + oz * s[5] + M * ox * oz;
        q[3] = s[11] + 2 * oy * s[6] + M * oy * oy;
        q[4] = s[12] + oy * s[7] + oz * s[6] + M * oy * oz;
        q[5] = s[13] + 2 * oz * s[7] + M * oz * oz;
        dp[0] = s[5] + M * ox;
        dp[1] = s[6] + M * oy;
        dp[2] = s[7] + M * oz;
    }
    if (sub == 0)
    {
        storeDNode(A.dn + node, c, W, M, q, dp);
        emitNode(A, node, prefix, c, W, M, q, dp, 0, b0, b1 - b0);
    }
    if (!A.arrivals) return;

    const unsigned gmask = 0xFFu << (threadIdx.x & 24u);
    while (node > 0)
    {
        int parent = A.parents[(node - 1) / 8];
        int last   = 0;
        if (sub == 0)
        {
            __threadfence();
            last = atomicAdd(A.arrivals + parent, 1u) == 7u;
        }
        last = __shfl_sync(gmask, last, 0, kTpl);
        if (!last) break;
        __threadfence();
        combineChildren(A, parent, A.childOffsets[parent], sub, gmask);
        node = parent;
    }
}

/*! the internal nodes of one tree level, [first, last) in the level-major order: eight lanes per node combine its
 *  eight children (one per lane), which the leaf pass or the previous (deeper) level wrote. Leaves of the level are
 *  skipped. */
__global__ void __launch_bounds__(256) levelCombineKernel(FusedArgs A, int first, int last)
{
    const int tid  = blockIdx.x * blockDim.x + threadIdx.x;
    const int node = first + tid / kTpl;
    const int sub  = tid % kTpl;
    if (node >= last) return;                // whole groups of eight leave together
    const int fc = A.childOffsets[node];
    if (fc == 0) return;                     // a leaf: written by the leaf pass
    const unsigned gmask = 0xFFu << (threadIdx.x & 24u);
    combineChildren(A, node, fc, sub, gmask);
}

//! trees of at least this many nodes combine their internal nodes level by level. A 2^22-body cube has 300k nodes, a
//! 2^20-body cube 37k: the levels took 0.144 and 0.051 ms there, the climb 0.194 and 0.047 ms. A 2^26-body cube has
//! about 5M.
constexpr int kLevelUpsweepNodes = 1 << 17;

void launchFusedUpsweep(ryo_ctx* ctx, const float4* xyzm, int numLeaves, int numNodes, const uint32_t* layout,
                        const int* leafToInternal, const int* childOffsets, const int* parents,
                        const uint64_t* prefixes, float invTheta, const DevBox<float>& box, NodeRecord* records,
                        float4* centers, float* multipoles, double* root, cudaStream_t s,
                        const DevBox<float>* sysBoxes, int sysLevel, double* sysRoots, float4* dipoles,
                        uint32_t numSystems, const int* hostLevelRange)
{
    FusedArgs A;
    A.dipoles        = dipoles;
    A.sysBoxes       = sysBoxes;
    A.sysLevel       = sysLevel;
    A.sysRoots       = sysRoots;
    A.numSystems     = numSystems;
    A.xyzm           = xyzm;
    A.layout         = layout;
    A.leafToInternal = leafToInternal;
    A.childOffsets   = childOffsets;
    A.parents        = parents;
    A.prefixes       = prefixes;
    A.numLeaves      = numLeaves;
    A.numNodes       = numNodes;
    A.invTheta       = invTheta;
    A.box            = box;
    A.dn             = ctx->scratch<DNode>("up.dnode", numNodes, s);
    // the climb leaves the other leaf groups of a climbing warp idle, which large trees pay for; each level launch
    // costs a few microseconds, which small and deep trees pay for. The results are the same either way.
    const bool byLevels = hostLevelRange && numNodes >= kLevelUpsweepNodes;
    A.arrivals          = byLevels ? nullptr : ctx->scratch<unsigned int>("up.arrivals", numNodes, s);
    A.records        = records;
    A.centers        = centers;
    A.multipoles     = multipoles;
    A.root           = root;
    if (A.arrivals) RYO_CUDA(cudaMemsetAsync(A.arrivals, 0, sizeof(unsigned int) * numNodes, s));
    fusedUpsweepKernel<<<ceilDiv(size_t(numLeaves) * kTpl, 256), 256, 0, s>>>(A);
    RYO_LAUNCH_CHECK();
    if (!byLevels) return;
    // internal nodes bottom-up, one launch per level that holds nodes (level-major order: level l is
    // [levelRange[l], levelRange[l + 1]))
    for (int l = kMaxLevel - 1; l >= 0; --l)
    {
        const int first = hostLevelRange[l], last = hostLevelRange[l + 1];
        if (last <= first) continue;
        levelCombineKernel<<<ceilDiv(size_t(last - first) * kTpl, 256), 256, 0, s>>>(A, first, last);
        RYO_LAUNCH_CHECK();
    }
}

// ------------------------------------------------------------------------------------------------ packing

__global__ void packNodesKernel(int numNodes, const float4* __restrict__ centers, const float* __restrict__ multipoles,
                                const int* __restrict__ childOffsets, const int* __restrict__ internalToLeaf,
                                const uint32_t* __restrict__ layout, NodeRecord* __restrict__ records)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= numNodes) return;
    const float4* mp = reinterpret_cast<const float4*>(multipoles + 8 * size_t(i));
    NodeRecord r;
    r.center = centers[i];
    r.q0     = mp[0];
    r.q1     = mp[1];
    int leaf = internalToLeaf[i];
    int fc   = childOffsets[i];
    uint32_t first = 0, count = 0;
    if (leaf >= 0)
    {
        first = layout[leaf];
        count = layout[leaf + 1] - first;
    }
    r.link     = make_int4(fc, int(first), int(count), leaf);
    records[i] = r;
}

void launchPackNodes(int numNodes, const float4* centers, const float* multipoles, const int* childOffsets,
                     const int* internalToLeaf, const uint32_t* layout, NodeRecord* records, cudaStream_t s)
{
    if (numNodes <= 0) return;
    packNodesKernel<<<ceilDiv(numNodes, 256), 256, 0, s>>>(numNodes, centers, multipoles, childOffsets,
                                                           internalToLeaf, layout, records);
    RYO_LAUNCH_CHECK();
}

__global__ void packBodiesKernel(const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
                                 const float* __restrict__ w, size_t n, float4* __restrict__ out)
{
    size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = make_float4(x[i], y[i], z[i], w[i]);
}

void launchPackBodies(const float* x, const float* y, const float* z, const float* w, size_t n, float4* out,
                      cudaStream_t s)
{
    if (n == 0) return;
    size_t blocks = (n + 255) / 256;
    packBodiesKernel<<<unsigned(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0, s>>>(x, y, z, w, n, out);
    RYO_LAUNCH_CHECK();
}

} // namespace ryo
