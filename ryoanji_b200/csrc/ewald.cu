/*
 * ryoanji-b200: Ewald correction for periodic boxes (root-multipole form).
 *
 * Reference: ryoanji/src/ryoanji/nbody/ewald.hpp:90-389 and ryoanji/src/ryoanji/interface/ewald.cu:31-99. The tree
 * traversal covers the (2 numReplicaShells + 1)^3 replica boxes; the correction adds, per target, the real-space
 * images of the root multipole with erfc weights (-erf inside the replicated region) and the reciprocal-space sum.
 *
 * B200 form: one warp per target group, lanes over its targets. Real space runs in float. The reciprocal sum runs in
 * double: per target the three phase factors exp(2 pi i dx_d / L) are computed once and every wave vector's
 * exp(i k.r) is a product of their integer powers, so no trigonometric call is made per wave vector.
 */
#include <cmath>

#include "internal.hpp"

namespace ryo
{

//! kernel constants; R is the real-space type (float for float coordinates, double otherwise)
template<class R>
struct EwaldKernelParams
{
    R mroot[8];
    R center[3];
    double centerD[3];
    R L, lCut2, alpha, alpha2, k1, ka, smallR2;
    int replicaShells, ewaldShells;
    int numK;
    double twoPiOverL;
    signed char h[kEwaldMaxK][3];
    double fc[kEwaldMaxK];
    double fs[kEwaldMaxK];
};

//! ewaldEvalMultipoleComplete (ewald.hpp:90-115)
template<class T>
__host__ __device__ inline void ewaldEval(T acc[4], const T r[3], const T g[6], const T* M)
{
    T m   = M[0];
    T qxx = (M[1] + M[7]) / T(3), qyy = (M[4] + M[7]) / T(3), qzz = (M[6] + M[7]) / T(3);
    T qxy = M[2] / T(3), qxz = M[3] / T(3), qyz = M[5] / T(3);
    T Qr[3] = {r[0] * qxx + r[1] * qxy + r[2] * qxz, r[0] * qxy + r[1] * qyy + r[2] * qyz,
               r[0] * qxz + r[1] * qyz + r[2] * qzz};
    T rQr = T(0.5) * (r[0] * Qr[0] + r[1] * Qr[1] + r[2] * Qr[2]);
    T Qtr = T(0.5) * M[7];
    T u   = -g[0] * m + g[1] * Qtr - g[2] * rQr;
    T f   = g[1] * m - g[2] * Qtr + g[3] * rQr;
    acc[0] += u;
    for (int d = 0; d < 3; ++d)
        acc[d + 1] += g[2] * Qr[d] - r[d] * f;
}

EwaldHost ewaldSetup(const double* mroot, const double* center, int replicaShells, double L, double lCut, double hCut,
                     double alphaScale, double smallR)
{
    EwaldHost e{};
    for (int i = 0; i < 8; ++i)
        e.mroot[i] = mroot[i];
    for (int i = 0; i < 3; ++i)
        e.center[i] = center[i];
    if (lCut == 0 && hCut == 0 && alphaScale == 0) replicaShells = 0;
    e.replicaShells = replicaShells;
    e.ewaldShells   = std::max(int(std::ceil(lCut)), replicaShells);
    e.L             = L;
    e.lCut          = lCut;
    e.hCut          = hCut;
    e.alphaScale    = alphaScale;
    e.smallR        = smallR;
    e.numK          = 0;
    if (e.ewaldShells == 0) return e;
    // ewaldInitParameters (ewald.hpp:133-198)
    int hReps    = int(std::ceil(hCut));
    double alpha = alphaScale / L;
    double k4    = M_PI * M_PI / (alpha * alpha * L * L);
    for (int hx = -hReps; hx <= hReps; ++hx)
        for (int hy = -hReps; hy <= hReps; ++hy)
            for (int hz = -hReps; hz <= hReps; ++hz)
            {
                double hr[3] = {double(hx), double(hy), double(hz)};
                double h2    = hr[0] * hr[0] + (hr[1] * hr[1] + hr[2] * hr[2]);
                if (h2 == 0 || h2 > hCut * hCut) continue;
                if (e.numK >= kEwaldMaxK) // callers check hCut first; this keeps the tables in bounds regardless
                    throw CudaError{cudaErrorInvalidValue, "ewald: more wave vectors than hCut <= 3 gives"};
                double g0 = std::exp(-k4 * h2) / (M_PI * h2 * L);
                double g1 = 2 * M_PI / L * g0;
                double g2 = -2 * M_PI / L * g1;
                double g3 = 2 * M_PI / L * g2;
                double g4 = -2 * M_PI / L * g3;
                double g5 = 2 * M_PI / L * g4;
                double gc[6] = {g0, 0.0, g2, 0.0, g4, 0.0};
                double gs[6] = {0.0, g1, 0.0, g3, 0.0, g5};
                double a1[4] = {0, 0, 0, 0}, a2[4] = {0, 0, 0, 0};
                ewaldEval<double>(a1, hr, gc, mroot);
                ewaldEval<double>(a2, hr, gs, mroot);
                double* k = e.kdata + 5 * e.numK;
                k[0]      = hx;
                k[1]      = hy;
                k[2]      = hz;
                k[3]      = a1[0];
                k[4]      = a2[0];
                e.numK++;
            }
    return e;
}

__device__ inline double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

// the real-space functions in the real-space type
__device__ inline float rsSqrt(float v) { return sqrtf(v); }
__device__ inline double rsSqrt(double v) { return sqrt(v); }
__device__ inline float rsExp(float v) { return expf(v); }
__device__ inline double rsExp(double v) { return exp(v); }
__device__ inline float rsErf(float v) { return erff(v); }
__device__ inline double rsErf(double v) { return erf(v); }
__device__ inline float rsErfc(float v) { return erfcf(v); }
__device__ inline double rsErfc(double v) { return erfc(v); }

/*! one warp per target group. R is the real-space type: float for the reference's float instantiation, double for its
 *  double-coordinate ones (ryoanji/src/ryoanji/interface/ewald.cu:101-110), where the reference's real space runs in
 *  its coordinate type; the reciprocal sum is double in every set. Tc, Tm, Ta: coordinates, masses, outputs. */
template<class R, class Tc, class Tm, class Ta>
__global__ void ewaldKernel(const __grid_constant__ EwaldKernelParams<R> E, const uint32_t* __restrict__ groupStart,
                            const uint32_t* __restrict__ groupEnd, uint32_t numGroups, const Tc* __restrict__ x,
                            const Tc* __restrict__ y, const Tc* __restrict__ z, const Tm* __restrict__ m, float G,
                            Ta* ugrav, Ta* ax, Ta* ay, Ta* az, double* potential)
{
    int warpGlobal = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
    int lane       = laneId();
    double upot    = 0.0;
    if (warpGlobal < int(numGroups))
    {
        uint32_t b = groupStart[warpGlobal], e = groupEnd[warpGlobal];
        for (uint32_t i = b + lane; i < e; i += kWarp)
        {
            R pos[3]  = {R(x[i]), R(y[i]), R(z[i])};
            R acc[4]  = {E.k1 * E.mroot[0], R(0), R(0), R(0)};
            R r[3]    = {pos[0] - E.center[0], pos[1] - E.center[1], pos[2] - E.center[2]};
            int S     = E.ewaldShells, Rs = E.replicaShells;
            // real space (ewald.hpp:200-301)
            for (int ix = -S; ix <= S; ++ix)
                for (int iy = -S; iy <= S; ++iy)
                    for (int iz = -S; iz <= S; ++iz)
                    {
                        bool pre = (-Rs <= ix && ix <= Rs) && (-Rs <= iy && iy <= Rs) && (-Rs <= iz && iz <= Rs);
                        R Rv[3]  = {r[0] + ix * E.L, r[1] + iy * E.L, r[2] + iz * E.L};
                        R R2     = Rv[0] * Rv[0] + (Rv[1] * Rv[1] + Rv[2] * Rv[2]);
                        if (R2 > E.lCut2 && !pre) continue;
                        R g[6];
                        if (R2 < E.smallR2 && E.ka > R(0))
                        {
                            R c0 = E.ka, a2 = R2 * E.alpha2;
                            g[0] = c0 * (a2 / R(3) - R(1));
                            c0 *= 2 * E.alpha2;
                            g[1] = c0 * (a2 / R(5) - R(1) / R(3));
                            c0 *= 2 * E.alpha2;
                            g[2] = c0 * (a2 / R(7) - R(1) / R(5));
                            c0 *= 2 * E.alpha2;
                            g[3] = c0 * (a2 / R(9) - R(1) / R(7));
                            c0 *= 2 * E.alpha2;
                            g[4] = c0 * (a2 / R(11) - R(1) / R(9));
                            c0 *= 2 * E.alpha2;
                            g[5] = c0 * (a2 / R(13) - R(1) / R(11));
                        }
                        else
                        {
                            R Rm = rsSqrt(R2), iR = R(1) / Rm, iR2 = iR * iR;
                            R a  = rsExp(-R2 * E.alpha2) * E.ka * iR2;
                            R an = R(1);
                            R fn = pre ? -rsErf(E.alpha * Rm) : rsErfc(E.alpha * Rm);
                            g[0] = fn * iR;
                            g[1] = g[0] * iR2 + a;
                            an *= 2 * E.alpha2;
                            g[2] = 3 * g[1] * iR2 + an * a;
                            an *= 2 * E.alpha2;
                            g[3] = 5 * g[2] * iR2 + an * a;
                            an *= 2 * E.alpha2;
                            g[4] = 7 * g[3] * iR2 + an * a;
                            an *= 2 * E.alpha2;
                            g[5] = 9 * g[4] * iR2 + an * a;
                        }
                        ewaldEval<R>(acc, Rv, g, E.mroot);
                    }
            // reciprocal space (ewald.hpp:303-327), double, exp(i k.r) from powers of the per-axis phases
            double dr[3] = {double(pos[0]) - E.centerD[0], double(pos[1]) - E.centerD[1],
                            double(pos[2]) - E.centerD[2]};
            double2 pw[3][7];
#pragma unroll
            for (int d = 0; d < 3; ++d)
            {
                double sn, cs;
                sincos(E.twoPiOverL * dr[d], &sn, &cs);
                double2 e1 = make_double2(cs, sn), e1c = make_double2(cs, -sn);
                pw[d][3]   = make_double2(1.0, 0.0);
                pw[d][4]   = e1;
                pw[d][2]   = e1c;
                pw[d][5]   = cmul(e1, e1);
                pw[d][1]   = cmul(e1c, e1c);
                pw[d][6]   = cmul(pw[d][5], e1);
                pw[d][0]   = cmul(pw[d][1], e1c);
            }
            double kp = 0.0, ka3[3] = {0.0, 0.0, 0.0};
            for (int q = 0; q < E.numK; ++q)
            {
                int hx = E.h[q][0], hy = E.h[q][1], hz = E.h[q][2];
                double2 w = cmul(cmul(pw[0][hx + 3], pw[1][hy + 3]), pw[2][hz + 3]);
                double c = w.x, s = w.y;
                double sum  = E.fc[q] * c + E.fs[q] * s;
                double diff = E.fc[q] * s - E.fs[q] * c;
                kp -= sum;
                ka3[0] += diff * (E.twoPiOverL * hx);
                ka3[1] += diff * (E.twoPiOverL * hy);
                ka3[2] += diff * (E.twoPiOverL * hz);
            }
            double phi = double(acc[0]) + kp;
            double mi  = m[i];
            upot += phi * mi;
            if (ugrav) ugrav[i] += Ta(G * phi * mi);
            ax[i] += Ta(G * (double(acc[1]) + ka3[0]));
            ay[i] += Ta(G * (double(acc[2]) + ka3[1]));
            az[i] += Ta(G * (double(acc[3]) + ka3[2]));
        }
    }
    upot = warpSum(upot);
    if (lane == 0 && upot != 0.0) atomicAdd(potential, upot);
}

template<class R, class Tc, class Tm, class Ta>
static void launchEwaldTyped(const EwaldHost& h, const uint32_t* groupStart, const uint32_t* groupEnd,
                             uint32_t numGroups, const Tc* x, const Tc* y, const Tc* z, const Tm* m, float G, Ta* ugrav,
                             Ta* ax, Ta* ay, Ta* az, double* potentialOut, cudaStream_t s)
{
    if (h.ewaldShells == 0 || numGroups == 0) return;
    EwaldKernelParams<R> E{};
    for (int i = 0; i < 8; ++i)
        E.mroot[i] = R(h.mroot[i]);
    for (int i = 0; i < 3; ++i)
    {
        E.center[i]  = R(h.center[i]);
        E.centerD[i] = h.center[i];
    }
    double alpha    = h.alphaScale / h.L;
    E.L             = R(h.L);
    E.lCut2         = R(h.lCut * h.lCut * h.L * h.L);
    E.alpha         = R(alpha);
    E.alpha2        = R(alpha * alpha);
    E.k1            = R(M_PI / (alpha * alpha * h.L * h.L * h.L));
    E.ka            = R(2.0 * alpha / std::sqrt(M_PI));
    E.smallR2       = R(h.smallR * h.L * h.L);
    E.replicaShells = h.replicaShells;
    E.ewaldShells   = h.ewaldShells;
    E.numK          = h.numK;
    E.twoPiOverL    = 2 * M_PI / h.L;
    for (int q = 0; q < h.numK; ++q)
    {
        for (int d = 0; d < 3; ++d)
            E.h[q][d] = (signed char)h.kdata[5 * q + d];
        E.fc[q] = h.kdata[5 * q + 3];
        E.fs[q] = h.kdata[5 * q + 4];
    }
    unsigned threads = 128;
    unsigned blocks  = ceilDiv(size_t(numGroups) * kWarp, threads);
    ewaldKernel<R, Tc, Tm, Ta><<<blocks, threads, 0, s>>>(E, groupStart, groupEnd, numGroups, x, y, z, m, G, ugrav,
                                                           ax, ay, az, potentialOut);
    RYO_LAUNCH_CHECK();
}

void launchEwaldGroups(const EwaldHost& h, const uint32_t* groupStart, const uint32_t* groupEnd, uint32_t numGroups,
                       const float* x, const float* y, const float* z, const float* m, float G, float* ugrav,
                       float* ax, float* ay, float* az, double* potentialOut, cudaStream_t s)
{
    launchEwaldTyped<float>(h, groupStart, groupEnd, numGroups, x, y, z, m, G, ugrav, ax, ay, az, potentialOut, s);
}

void launchEwaldGroups(const EwaldHost& h, const uint32_t* groupStart, const uint32_t* groupEnd, uint32_t numGroups,
                       const double* x, const double* y, const double* z, const double* m, float G, double* ugrav,
                       double* ax, double* ay, double* az, double* potentialOut, cudaStream_t s)
{
    launchEwaldTyped<double>(h, groupStart, groupEnd, numGroups, x, y, z, m, G, ugrav, ax, ay, az, potentialOut, s);
}

void launchEwaldGroups(const EwaldHost& h, const uint32_t* groupStart, const uint32_t* groupEnd, uint32_t numGroups,
                       const double* x, const double* y, const double* z, const float* m, float G, float* ugrav,
                       float* ax, float* ay, float* az, double* potentialOut, cudaStream_t s)
{
    launchEwaldTyped<double>(h, groupStart, groupEnd, numGroups, x, y, z, m, G, ugrav, ax, ay, az, potentialOut, s);
}

// ------------------------------------------------------------------------------------------------ FP64 oracle

/*
 * Particle-level Ewald sum in FP64 for chosen targets, the check of the periodic solve: the same real-space and
 * reciprocal-space formulas as the correction above with every source's own monopole in place of the root
 * multipole. Added to the FP64 direct sum over the (2 numReplicaShells + 1)^3 replica boxes it gives each target's
 * periodic potential and acceleration without the tree's multipole approximation of the far replicas.
 */
struct EwaldParticleParams
{
    double L, lCut2, alpha, alpha2, ka, k1, smallR2;
    int replicaShells, ewaldShells;
};

constexpr int kEwaldOracleThreads = 256;

__device__ inline double blockSumD(double v, double* sh)
{
    v = warpSum(v);
    if (laneId() == 0) sh[threadIdx.x / kWarp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x < kWarp)
    {
        t = threadIdx.x < blockDim.x / kWarp ? sh[threadIdx.x] : 0.0;
        t = warpSum(t);
    }
    __syncthreads();
    return t;
}

//! real-space images of every source's monopole for one target per block; adds G m_i phi and G a
__global__ void __launch_bounds__(kEwaldOracleThreads)
    ewaldRealTargetsKernel(const int64_t* __restrict__ targets, const float* __restrict__ x,
                           const float* __restrict__ y, const float* __restrict__ z, const float* __restrict__ m,
                           size_t numBodies, EwaldParticleParams P, double G, double* pot, double* ax, double* ay,
                           double* az)
{
    __shared__ double sh[kEwaldOracleThreads / kWarp];
    int64_t i      = targets[blockIdx.x];
    double xi[3]   = {x[i], y[i], z[i]};
    double acc[4]  = {0, 0, 0, 0};
    const int S = P.ewaldShells, Rs = P.replicaShells;
    for (size_t j = threadIdx.x; j < numBodies; j += blockDim.x)
    {
        double mj   = m[j];
        double r[3] = {xi[0] - double(x[j]), xi[1] - double(y[j]), xi[2] - double(z[j])};
        for (int ix = -S; ix <= S; ++ix)
            for (int iy = -S; iy <= S; ++iy)
                for (int iz = -S; iz <= S; ++iz)
                {
                    bool pre    = (-Rs <= ix && ix <= Rs) && (-Rs <= iy && iy <= Rs) && (-Rs <= iz && iz <= Rs);
                    double R[3] = {r[0] + ix * P.L, r[1] + iy * P.L, r[2] + iz * P.L};
                    double R2   = R[0] * R[0] + (R[1] * R[1] + R[2] * R[2]);
                    if (R2 > P.lCut2 && !pre) continue;
                    double g0, g1;
                    if (R2 < P.smallR2 && P.ka > 0.0)
                    {
                        double a2 = R2 * P.alpha2;
                        g0        = P.ka * (a2 / 3.0 - 1.0);
                        g1        = P.ka * 2 * P.alpha2 * (a2 / 5.0 - 1.0 / 3.0);
                    }
                    else
                    {
                        double Rm = sqrt(R2), iR = 1.0 / Rm, iR2 = iR * iR;
                        double a  = exp(-R2 * P.alpha2) * P.ka * iR2;
                        double fn = pre ? -erf(P.alpha * Rm) : erfc(P.alpha * Rm);
                        g0        = fn * iR;
                        g1        = g0 * iR2 + a;
                    }
                    acc[0] -= g0 * mj;
                    double f = g1 * mj;
                    acc[1] -= R[0] * f;
                    acc[2] -= R[1] * f;
                    acc[3] -= R[2] * f;
                }
    }
    for (int k = 0; k < 4; ++k)
        acc[k] = blockSumD(acc[k], sh);
    if (threadIdx.x == 0)
    {
        pot[blockIdx.x] += G * double(m[i]) * acc[0];
        ax[blockIdx.x] += G * acc[1];
        ay[blockIdx.x] += G * acc[2];
        az[blockIdx.x] += G * acc[3];
    }
}

//! structure factors S(k) = sum_j m_j exp(i k . x_j), one block per wave vector
__global__ void __launch_bounds__(kEwaldOracleThreads)
    structureFactorKernel(const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
                          const float* __restrict__ m, size_t numBodies, const int* __restrict__ hvec,
                          double twoPiOverL, double* S)
{
    __shared__ double sh[kEwaldOracleThreads / kWarp];
    int hx = hvec[3 * blockIdx.x], hy = hvec[3 * blockIdx.x + 1], hz = hvec[3 * blockIdx.x + 2];
    double re = 0.0, im = 0.0;
    for (size_t j = threadIdx.x; j < numBodies; j += blockDim.x)
    {
        double ph = twoPiOverL * (hx * double(x[j]) + hy * double(y[j]) + hz * double(z[j]));
        double sn, cs;
        sincos(ph, &sn, &cs);
        re += double(m[j]) * cs;
        im += double(m[j]) * sn;
    }
    re = blockSumD(re, sh);
    im = blockSumD(im, sh);
    if (threadIdx.x == 0)
    {
        S[2 * blockIdx.x]     = re;
        S[2 * blockIdx.x + 1] = im;
    }
}

//! reciprocal-space sum and the neutralising constant for each target
__global__ void ewaldKspaceTargetsKernel(const int64_t* __restrict__ targets, size_t numTargets,
                                         const float* __restrict__ x, const float* __restrict__ y,
                                         const float* __restrict__ z, const float* __restrict__ m,
                                         const int* __restrict__ hvec, const double* __restrict__ g0,
                                         const double* __restrict__ S, int numK, double twoPiOverL, double k1M,
                                         double G, double* pot, double* ax, double* ay, double* az)
{
    size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= numTargets) return;
    int64_t i = targets[t];
    double xi[3] = {x[i], y[i], z[i]};
    double phi = k1M, a[3] = {0, 0, 0};
    for (int q = 0; q < numK; ++q)
    {
        int h[3]  = {hvec[3 * q], hvec[3 * q + 1], hvec[3 * q + 2]};
        double ph = twoPiOverL * (h[0] * xi[0] + h[1] * xi[1] + h[2] * xi[2]);
        double sn, cs;
        sincos(ph, &sn, &cs);
        double c = cs * S[2 * q] + sn * S[2 * q + 1]; // sum_j m_j cos(k.(x_i - x_j))
        double s = sn * S[2 * q] - cs * S[2 * q + 1]; // sum_j m_j sin(k.(x_i - x_j))
        phi += g0[q] * c;
        for (int d = 0; d < 3; ++d)
            a[d] -= g0[q] * s * (twoPiOverL * h[d]);
    }
    pot[t] += G * double(m[i]) * phi;
    ax[t] += G * a[0];
    ay[t] += G * a[1];
    az[t] += G * a[2];
}

void launchEwaldTargetsF64(ryo_ctx* ctx, const int64_t* targets, size_t numTargets, const float* x, const float* y,
                           const float* z, const float* m, size_t numBodies, double L, int replicaShells, double lCut,
                           double hCut, double alphaScale, double smallR, double G, double* pot, double* ax,
                           double* ay, double* az, cudaStream_t s)
{
    if (numTargets == 0 || numBodies == 0) return;
    EwaldParticleParams P{};
    double alpha    = alphaScale / L;
    P.L             = L;
    P.lCut2         = lCut * lCut * L * L;
    P.alpha         = alpha;
    P.alpha2        = alpha * alpha;
    P.ka            = 2.0 * alpha / std::sqrt(M_PI);
    P.k1            = M_PI / (alpha * alpha * L * L * L);
    P.smallR2       = smallR * L * L;
    P.replicaShells = replicaShells;
    P.ewaldShells   = std::max(int(std::ceil(lCut)), replicaShells);
    ewaldRealTargetsKernel<<<unsigned(numTargets), kEwaldOracleThreads, 0, s>>>(targets, x, y, z, m, numBodies, P, G,
                                                                               pot, ax, ay, az);
    RYO_LAUNCH_CHECK();
    // wave vectors and their coefficients as in ewaldSetup, for a unit monopole
    std::vector<int> hv;
    std::vector<double> g0;
    int hReps = int(std::ceil(hCut));
    double k4 = M_PI * M_PI / (alpha * alpha * L * L);
    for (int hx = -hReps; hx <= hReps; ++hx)
        for (int hy = -hReps; hy <= hReps; ++hy)
            for (int hz = -hReps; hz <= hReps; ++hz)
            {
                double h2 = double(hx) * hx + (double(hy) * hy + double(hz) * hz);
                if (h2 == 0 || h2 > hCut * hCut) continue;
                hv.insert(hv.end(), {hx, hy, hz});
                g0.push_back(std::exp(-k4 * h2) / (M_PI * h2 * L));
            }
    int numK = int(g0.size());
    // total mass for the neutralising constant
    std::vector<float> hm(numBodies);
    RYO_CUDA(cudaMemcpyAsync(hm.data(), m, numBodies * sizeof(float), cudaMemcpyDeviceToHost, s));
    int* dh    = ctx->scratch<int>("ew.hvec", std::max<size_t>(3 * size_t(numK), 1), s);
    double* dg = ctx->scratch<double>("ew.g0", std::max(numK, 1), s);
    double* dS = ctx->scratch<double>("ew.S", std::max<size_t>(2 * size_t(numK), 1), s);
    if (numK > 0)
    {
        RYO_CUDA(cudaMemcpyAsync(dh, hv.data(), sizeof(int) * hv.size(), cudaMemcpyHostToDevice, s));
        RYO_CUDA(cudaMemcpyAsync(dg, g0.data(), sizeof(double) * g0.size(), cudaMemcpyHostToDevice, s));
        structureFactorKernel<<<unsigned(numK), kEwaldOracleThreads, 0, s>>>(x, y, z, m, numBodies, dh,
                                                                            2 * M_PI / L, dS);
        RYO_LAUNCH_CHECK();
    }
    RYO_CUDA(cudaStreamSynchronize(s));
    double M = 0;
    for (float v : hm)
        M += v;
    ewaldKspaceTargetsKernel<<<ceilDiv(numTargets, 128), 128, 0, s>>>(targets, numTargets, x, y, z, m, dh, dg, dS,
                                                                       numK, 2 * M_PI / L, P.k1 * M, G, pot, ax, ay,
                                                                       az);
    RYO_LAUNCH_CHECK();
}

} // namespace ryo
