// gb_static_sort.cu -- the linked-cell sort (cell hash, stable radix sort of
// (cell, particle id), cell-start table) for callers that cannot allocate
// device memory.
//
// Some callers cannot call cudaMalloc at the point where they need the
// broad phase: a host code whose device memory is wholly reserved by another
// allocator in the same process (a caching allocator owns the pool, so a
// driver allocation fails or forces that allocator to release memory), or a
// time loop that must not block on the implicit device synchronisation a
// cudaMalloc/cudaFree pair causes.  gb_linked_cell_sort_static runs the same
// kernels as gb_update_links, but its scratch -- the hashes, the radix
// sort's ping-pong buffers, histograms and scan partials -- lives in one
// file-scope __device__ array sized for kStaticMaxParticles particles.
//
// Costs of that choice: every GPU that loads the library holds the array
// (about 6.4 MB) until the process exits, and every call shares it, so calls
// whose work overlaps on the GPU (different streams, or different host
// threads on one device) race on the scratch and must be serialised by the
// caller.  The array keeps the last call's contents; what must start at
// zero (the domain-error flag) is cleared by each call.
#include <cstdint>
#include <cuda_runtime.h>
#include <mutex>

#include "../../include/grains_b200.h"

namespace
{
// the broad-phase kernels, with internal linkage in this translation unit
#include "gb_broadphase.cuh"

constexpr int    kStaticMaxParticles = 1 << 18; // 262,144
constexpr int    kStaticMaxTiles     = (kStaticMaxParticles + gb::kTile - 1) / gb::kTile;
constexpr size_t kN                  = kStaticMaxParticles;
constexpr size_t kHistWords          = 256 * (size_t)kStaticMaxTiles;
constexpr size_t kPartWords          = 1024;
// word offsets: hash, iota, keys[2], ids (one ping-pong slot; the last pass
// scatters ids straight into the caller's output), histogram, scan
// partials, flags
constexpr size_t kOffHash  = 0;
constexpr size_t kOffIota  = kN;
constexpr size_t kOffKey0  = 2 * kN;
constexpr size_t kOffKey1  = 3 * kN;
constexpr size_t kOffId0   = 4 * kN;
constexpr size_t kOffId1   = 5 * kN;
constexpr size_t kOffHist  = 6 * kN;
constexpr size_t kOffPart  = kOffHist + kHistWords;
constexpr size_t kOffFlags = kOffPart + kPartWords;
constexpr size_t kWords    = kOffFlags + 64;

__device__ __align__(256) uint32_t g_sort_scratch[kWords];

constexpr int kMaxDevices = 64;
std::mutex    g_setup_mutex;
uint32_t*     g_scratch_addr[kMaxDevices] = {};

// The device address of g_sort_scratch on the current device.  In host code
// the symbol names a host-side stand-in, not device memory; its device
// address comes from cudaGetSymbolAddress, once per device, with that device
// current.
int scratch_on_current_device(uint32_t** out)
{
    int dev = -1;
    if(cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return GB_E_NO_DEVICE;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if(!g_scratch_addr[dev])
    {
        void* p = nullptr;
        if(cudaGetSymbolAddress(&p, g_sort_scratch) != cudaSuccess || !p)
            return GB_E_CUDA;
        g_scratch_addr[dev] = (uint32_t*)p;
    }
    *out = g_scratch_addr[dev];
    return GB_OK;
}

int scan_static(uint32_t* buf, int64_t n, uint32_t* part, cudaStream_t s)
{
    const int nb = (int)((n + gb::kTile - 1) / gb::kTile);
    if(nb < 1 || (size_t)nb > kPartWords)
        return GB_E_CAPACITY;
    gb::k_scan_reduce<<<nb, gb::kBlock, 0, s>>>(buf, n, part);
    gb::k_scan_partials<<<1, 1024, 0, s>>>(part, nb, nullptr);
    gb::k_scan_apply<<<nb, gb::kBlock, 0, s>>>(buf, buf, n, part);
    return cudaGetLastError() == cudaSuccess ? GB_OK : GB_E_CUDA;
}

} // namespace

extern "C" int gb_linked_cell_sort_static(const double* pos, int32_t n, const double origin[3],
                                          double cell_size, const int32_t dims[3],
                                          uint32_t* sorted_ids, uint32_t* cell_start,
                                          void* stream)
{
    if(!pos || !origin || !dims || !sorted_ids || !cell_start || n < 1 || !(cell_size > 0.0))
        return GB_E_INVALID_ARG;
    if(n > kStaticMaxParticles)
        return GB_E_CAPACITY; // more particles than the static scratch holds
    if(dims[0] < 1 || dims[1] < 1 || dims[2] < 1)
        return GB_E_INVALID_ARG;
    const uint64_t ncells = (uint64_t)dims[0] * dims[1] * dims[2];
    if(ncells > gb::kMaxCells)
        return GB_E_INVALID_ARG;
    uint32_t* sc = nullptr;
    int       st = scratch_on_current_device(&sc);
    if(st != GB_OK)
        return st;
    cudaStream_t s     = (cudaStream_t)stream;
    int*         flags = (int*)(sc + kOffFlags);
    if(cudaMemsetAsync(flags, 0, sizeof(int), s) != cudaSuccess)
        return GB_E_CUDA;
    const int nb = (n + gb::kBlock - 1) / gb::kBlock;
    gb::k_hash<<<nb, gb::kBlock, 0, s>>>(n, pos, pos + n, pos + 2 * (size_t)n, origin[0],
                                         origin[1], origin[2], cell_size, (uint32_t)dims[0],
                                         (uint32_t)dims[1], (uint32_t)dims[2], sc + kOffHash,
                                         sc + kOffIota, flags);
    int key_bits = 0;
    while(key_bits < 32 && (1ull << key_bits) < ncells)
        ++key_bits;
    const int       passes   = key_bits == 0 ? 0 : (key_bits + 7) / 8;
    const int       bits_per = passes ? (key_bits + passes - 1) / passes : 0;
    const int       ntile    = (n + gb::kTile - 1) / gb::kTile;
    const uint32_t* src_k    = sc + kOffHash;
    const uint32_t* src_i    = sc + kOffIota;
    for(int p = 0; p < passes; ++p)
    {
        const int      shift = p * bits_per;
        const int      b     = bits_per < key_bits - shift ? bits_per : key_bits - shift;
        const uint32_t mask  = (1u << b) - 1u;
        const int64_t  hn    = (int64_t)(mask + 1) * ntile;
        uint32_t*      hist  = sc + kOffHist;
        uint32_t*      dk    = sc + ((p & 1) ? kOffKey1 : kOffKey0);
        uint32_t*      di    = p == passes - 1 ? sorted_ids : sc + ((p & 1) ? kOffId1 : kOffId0);
        gb::k_radix_hist<<<ntile, gb::kBlock, 0, s>>>(src_k, n, shift, mask, hist);
        if((st = scan_static(hist, hn, sc + kOffPart, s)) != GB_OK)
            return st;
        gb::k_radix_scatter<<<ntile, gb::kBlock, 0, s>>>(src_k, src_i, dk, di, n, shift, mask,
                                                         hist);
        src_k = dk;
        src_i = di;
    }
    if(passes == 0)
    {
        if(cudaMemcpyAsync(sorted_ids, sc + kOffIota, n * sizeof(uint32_t),
                           cudaMemcpyDeviceToDevice, s)
           != cudaSuccess)
            return GB_E_CUDA;
    }
    gb::k_cell_start<<<(int)((ncells + 1 + gb::kCellsPerBlock - 1) / gb::kCellsPerBlock),
                       gb::kBlock, 0, s>>>(src_k, (uint32_t)n, (uint32_t)ncells, cell_start);
    if(cudaGetLastError() != cudaSuccess)
        return GB_E_CUDA;
    int hflags = 0;
    if(cudaMemcpyAsync(&hflags, flags, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess
       || cudaStreamSynchronize(s) != cudaSuccess)
        return GB_E_CUDA;
    if(hflags & gb::kFlagNonFinite)
        return GB_E_NONFINITE;
    if(hflags & gb::kFlagOutOfDomain)
        return GB_E_OUT_OF_DOMAIN;
    return GB_OK;
}
