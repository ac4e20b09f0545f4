// gb_io.cuh -- device-side conversion between the host layouts of the ABI
// (Transform3 buffers of 12 doubles, Kinematics/Torce pairs of 3-vectors, one
// record per particle) and the engine's structure-of-arrays state.  The host
// only copies raw bytes; transposes and quaternion extraction run here.
#pragma once

#include "gb_dem.cuh"

namespace gb
{

// 12 doubles per particle -> positions + basis (FP64 modes) or unit
// quaternion (mixed mode, Quaternion::setQuaternion(Matrix3) then normalised,
// kept as a compensated FP32 pair)
template <typename St>
__global__ void k_set_transforms(int n, const double* __restrict__ tr, double* __restrict__ pos,
                                 St* __restrict__ rot, int quat)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n)
        return;
    const double* t = tr + 12 * (size_t)i;
#pragma unroll
    for(int k = 0; k < 3; ++k)
        pos[(size_t)k * n + i] = t[9 + k];
    if(!quat)
    {
#pragma unroll
        for(int k = 0; k < 9; ++k)
            rot[(size_t)k * n + i] = (St)t[k];
        return;
    }
    M3<double> R;
#pragma unroll
    for(int k = 0; k < 9; ++k)
        R.m[k] = t[k];
    Quat<double> q  = quat_from_basis(R);
    const double nq = sqrt(q.w * q.w + q.v.x * q.v.x + q.v.y * q.v.y + q.v.z * q.v.z);
    const double c[4] = {q.w / nq, q.v.x / nq, q.v.y / nq, q.v.z / nq};
    // a compensated pair: the FP32 value in rot[0..3] and its FP32 remainder
    // in rot[4..7], so that hi + lo carries the FP64 orientation
#pragma unroll
    for(int k = 0; k < 4; ++k)
    {
        const St hi                  = (St)c[k];
        rot[(size_t)k * n + i]       = hi;
        rot[(size_t)(4 + k) * n + i] = (St)(c[k] - (double)hi);
    }
}

template <typename St>
__global__ void k_get_transforms(int n, double* __restrict__ tr, const double* __restrict__ pos,
                                 const St* __restrict__ rot, int quat)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n)
        return;
    double* t = tr + 12 * (size_t)i;
#pragma unroll
    for(int k = 0; k < 3; ++k)
        t[9 + k] = pos[(size_t)k * n + i];
    if(!quat)
    {
#pragma unroll
        for(int k = 0; k < 9; ++k)
            t[k] = (double)rot[(size_t)k * n + i];
        return;
    }
    double q[4];
#pragma unroll
    for(int k = 0; k < 4; ++k)
        q[k] = (double)rot[(size_t)k * n + i] + (double)rot[(size_t)(4 + k) * n + i];
    const M3<double> R = quat_to_matrix<double>(q[0], q[1], q[2], q[3]);
#pragma unroll
    for(int k = 0; k < 9; ++k)
        t[k] = R.m[k];
}

// 6 doubles per particle <-> two SoA 3-vectors (velocity/omega, force/torque)
template <typename St>
__global__ void k_set_pairs3(int n, const double* __restrict__ in, St* __restrict__ a,
                             St* __restrict__ b)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n)
        return;
    const double* r = in + 6 * (size_t)i;
#pragma unroll
    for(int k = 0; k < 3; ++k)
    {
        a[(size_t)k * n + i] = (St)r[k];
        b[(size_t)k * n + i] = (St)r[3 + k];
    }
}

template <typename St>
__global__ void k_get_pairs3(int n, double* __restrict__ out, const St* __restrict__ a,
                             const St* __restrict__ b)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n)
        return;
    double* r = out + 6 * (size_t)i;
#pragma unroll
    for(int k = 0; k < 3; ++k)
    {
        r[k]     = (double)a[(size_t)k * n + i];
        r[3 + k] = (double)b[(size_t)k * n + i];
    }
}

} // namespace gb
