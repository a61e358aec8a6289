/*
 * ryoanji-b200: direct sums.
 *
 * ryo_direct_sum_* follow ryoanji/src/ryoanji/nbody/direct.cuh:36-107 (tiled all-pairs, P2P with the exact
 * 1/sqrt of the type, no G, p += m phi). The accuracy reference (launchDirectTargets) evaluates chosen targets of
 * float data entirely in double precision, the FP64 oracle that tree errors are quoted against; sources are staged
 * through shared memory in tiles and every thread owns one target.
 */
#include "internal.hpp"

namespace ryo
{

constexpr int kDirectThreads = 256;

template<class T>
__device__ inline T exactRsqrt(T v);
template<>
__device__ inline float exactRsqrt<float>(float v)
{
    return rsqrtf(v);
}
template<>
__device__ inline double exactRsqrt<double>(double v)
{
    return rsqrt(v);
}

template<class T>
__device__ inline void p2pExact(T acc[4], const T ti[3], const T sj[3], T mj, T hi, T hj)
{
    T dx = sj[0] - ti[0], dy = sj[1] - ti[1], dz = sj[2] - ti[2];
    T R2    = dx * dx + (dy * dy + dz * dz);
    T hij   = hi + hj;
    T hij2  = hij * hij;
    T R2eff = (R2 < hij2) ? hij2 : R2;
    T invR  = exactRsqrt(R2eff);
    T m3    = mj * invR * (invR * invR);
    acc[0] -= m3 * R2;
    acc[1] += dx * m3;
    acc[2] += dy * m3;
    acc[3] += dz * m3;
}

template<class T>
__global__ void __launch_bounds__(kDirectThreads) directKernel(size_t first, size_t last, size_t numSource,
                                                               T sx, T sy, T sz, int numShells,
                                                               const T* __restrict__ x, const T* __restrict__ y,
                                                               const T* __restrict__ z, const T* __restrict__ m,
                                                               const T* __restrict__ h, T* p, T* ax, T* ay, T* az)
{
    __shared__ T tile[kDirectThreads][5];
    size_t t  = first + size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    T pos[3]  = {T(0), T(0), T(0)};
    T hi      = T(1);
    if (t < last)
    {
        pos[0] = x[t];
        pos[1] = y[t];
        pos[2] = z[t];
        hi     = h[t];
    }
    T acc[4] = {T(0), T(0), T(0), T(0)};
    for (int iz = -numShells; iz <= numShells; ++iz)
        for (int iy = -numShells; iy <= numShells; ++iy)
            for (int ix = -numShells; ix <= numShells; ++ix)
            {
                T ti[3] = {pos[0] + ix * sx, pos[1] + iy * sy, pos[2] + iz * sz};
                for (size_t s0 = 0; s0 < numSource; s0 += kDirectThreads)
                {
                    size_t j = s0 + threadIdx.x;
                    if (j < numSource)
                    {
                        tile[threadIdx.x][0] = x[j];
                        tile[threadIdx.x][1] = y[j];
                        tile[threadIdx.x][2] = z[j];
                        tile[threadIdx.x][3] = m[j];
                        tile[threadIdx.x][4] = h[j];
                    }
                    else
                    {
                        tile[threadIdx.x][0] = tile[threadIdx.x][1] = tile[threadIdx.x][2] = T(0);
                        tile[threadIdx.x][3] = T(0);
                        tile[threadIdx.x][4] = T(1);
                    }
                    __syncthreads();
                    for (int k = 0; k < kDirectThreads; ++k)
                    {
                        T sj[3] = {tile[k][0], tile[k][1], tile[k][2]};
                        p2pExact(acc, ti, sj, tile[k][3], hi, tile[k][4]);
                    }
                    __syncthreads();
                }
            }
    if (t < last)
    {
        p[t] += m[t] * acc[0];
        ax[t] += acc[1];
        ay[t] += acc[2];
        az[t] += acc[3];
    }
}

template<class T>
void launchDirect(size_t first, size_t last, size_t numBodies, const T* boxL, int numShells, const T* x, const T* y,
                  const T* z, const T* m, const T* h, T* p, T* ax, T* ay, T* az, cudaStream_t s)
{
    if (last <= first) return;
    T L[3] = {boxL ? boxL[0] : T(0), boxL ? boxL[1] : T(0), boxL ? boxL[2] : T(0)};
    directKernel<T><<<ceilDiv(last - first, kDirectThreads), kDirectThreads, 0, s>>>(
        first, last, numBodies, L[0], L[1], L[2], numShells, x, y, z, m, h, p, ax, ay, az);
    RYO_LAUNCH_CHECK();
}

template void launchDirect<float>(size_t, size_t, size_t, const float*, int, const float*, const float*,
                                  const float*, const float*, const float*, float*, float*, float*, float*,
                                  cudaStream_t);
template void launchDirect<double>(size_t, size_t, size_t, const double*, int, const double*, const double*,
                                   const double*, const double*, const double*, double*, double*, double*, double*,
                                   cudaStream_t);

//! double-precision reference for chosen targets; sources in float are staged as float4 + h
__global__ void __launch_bounds__(kDirectThreads) directTargetsKernel(const int64_t* __restrict__ targets,
                                                                      size_t numTargets, const float* __restrict__ x,
                                                                      const float* __restrict__ y,
                                                                      const float* __restrict__ z,
                                                                      const float* __restrict__ m,
                                                                      const float* __restrict__ h, size_t numBodies,
                                                                      double G, double Lx, double Ly, double Lz,
                                                                      int numShells, double* pot, double* ax,
                                                                      double* ay, double* az)
{
    __shared__ float4 tile[kDirectThreads];
    __shared__ float tileH[kDirectThreads];
    size_t t  = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    int64_t i = t < numTargets ? targets[t] : 0;
    double pos[3] = {double(x[i]), double(y[i]), double(z[i])};
    double hi     = h[i];
    double acc[4] = {0, 0, 0, 0};
    for (int iz = -numShells; iz <= numShells; ++iz)
        for (int iy = -numShells; iy <= numShells; ++iy)
            for (int ix = -numShells; ix <= numShells; ++ix)
            {
                double ti[3] = {pos[0] + ix * Lx, pos[1] + iy * Ly, pos[2] + iz * Lz};
                for (size_t s0 = 0; s0 < numBodies; s0 += kDirectThreads)
                {
                    size_t j = s0 + threadIdx.x;
                    if (j < numBodies)
                    {
                        tile[threadIdx.x]  = make_float4(x[j], y[j], z[j], m[j]);
                        tileH[threadIdx.x] = h[j];
                    }
                    else
                    {
                        tile[threadIdx.x]  = make_float4(0.f, 0.f, 0.f, 0.f);
                        tileH[threadIdx.x] = 1.f;
                    }
                    __syncthreads();
                    int cnt = int(numBodies - s0 < size_t(kDirectThreads) ? numBodies - s0 : kDirectThreads);
                    for (int k = 0; k < cnt; ++k)
                    {
                        float4 sj4   = tile[k];
                        double sj[3] = {sj4.x, sj4.y, sj4.z};
                        p2pExact<double>(acc, ti, sj, double(sj4.w), hi, double(tileH[k]));
                    }
                    __syncthreads();
                }
            }
    if (t < numTargets)
    {
        pot[t] = G * double(m[i]) * acc[0];
        ax[t]  = G * acc[1];
        ay[t]  = G * acc[2];
        az[t]  = G * acc[3];
    }
}

void launchDirectTargets(const int64_t* targets, size_t numTargets, const float* x, const float* y, const float* z,
                         const float* m, const float* h, size_t numBodies, double G, const double* boxL,
                         int numShells, double* pot, double* ax, double* ay, double* az, cudaStream_t s)
{
    if (numTargets == 0) return;
    double L[3] = {boxL ? boxL[0] : 0.0, boxL ? boxL[1] : 0.0, boxL ? boxL[2] : 0.0};
    directTargetsKernel<<<ceilDiv(numTargets, kDirectThreads), kDirectThreads, 0, s>>>(
        targets, numTargets, x, y, z, m, h, numBodies, G, L[0], L[1], L[2], numShells, pot, ax, ay, az);
    RYO_LAUNCH_CHECK();
}

} // namespace ryo
