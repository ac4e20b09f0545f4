// gb_rawdata.cuh -- the RawData post-processing writer
// (RawDataPostProcessingWriter.cpp:63-210): one text file per component
// (position, translational and angular velocity, x/y/z), one line per save
// time: the time, then every particle's value, then every obstacle's (its
// origin; obstacle velocities are written as zeros).  Values are printed as
// the reference's realToString(ios::scientific, 6, v) does
// (GrainsUtils.hh:33-44): "%.6e", or the stream's default "0" / "-0" for a
// zero.  The coordination-number file gets an empty line per save (the
// reference's per-particle output is commented out, :149), or, with
// GB_RAW_COORDINATION_NUMBER, the time and each particle's particle-contact
// count of the last detect.  particleType.dat is rewritten at every save
// holding one empty line, as the reference leaves it.
//
// A save does not stall the step loop: one kernel on the engine's stream
// gathers the state into a device snapshot (after every step launched
// before it), a copy stream moves the snapshot to pinned host memory, and a
// host thread formats and writes the files while the next steps run.  The
// next save (or close) first waits for that thread.
#pragma once

#include <cmath>
#include <cstdio>
#include <string>
#include <thread>

namespace gb
{

template <typename St>
__global__ void __launch_bounds__(kBlock)
    k_raw_snapshot(int n, const double* __restrict__ pos, const St* __restrict__ vel,
                   const St* __restrict__ omg, const uint32_t* __restrict__ off,
                   const uint8_t* __restrict__ contact, double* __restrict__ snap,
                   uint32_t* __restrict__ coordination)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n)
        return;
#pragma unroll
    for(int k = 0; k < 3; ++k)
    {
        snap[(size_t)k * n + i]       = pos[(size_t)k * n + i];
        snap[(size_t)(3 + k) * n + i] = (double)vel[(size_t)k * n + i];
        snap[(size_t)(6 + k) * n + i] = (double)omg[(size_t)k * n + i];
    }
    if(coordination)
    {
        uint32_t nc = 0;
        if(off)
            for(uint32_t p = off[i]; p < off[i + 1]; ++p)
                nc += contact[p] == kContactParticle;
        coordination[i] = nc;
    }
}

// realToString(ios::scientific, 6, v): a zero keeps the stream's default
// format ("0", or "-0" for a negative zero)
inline int raw_real(char* buf, size_t cap, double v)
{
    if(v == 0.0)
        return std::snprintf(buf, cap, "%s", std::signbit(v) ? "-0" : "0");
    return std::snprintf(buf, cap, "%.6e", v);
}

} // namespace gb
