// gb_broadphase.cuh -- linked-cell broad phase on the GPU: cell hash per
// particle, a stable LSD radix sort of (cell, particle id), the cell-start
// table, and device-wide exclusive scans.  Integer work: HBM-bound, no atomics
// on the data path (only shared-memory histogram counters).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gb
{

constexpr int kBlock = 256;           // threads per block for the streaming kernels
constexpr int kItems = 8;             // elements per thread in sort/scan tiles
constexpr int kTile  = kBlock * kItems;
constexpr int kWarps = kBlock / 32;

// device status bits (bit i <-> GB_E_* == -i)
constexpr int kFlagOutOfDomain = 1 << 5;
constexpr int kFlagNonFinite   = 1 << 6;
constexpr int kFlagCapacity    = 1 << 8;
constexpr int kFlagCellCrowded = 1 << 9; // a cell too full for the counting sort's rank pass
// Either one aborts the step: the kernels that write pair lists or state
// return at entry once it is set, and the host replays the step.
constexpr int kFlagScanStall   = 1 << 10; // a one-pass scan gave up waiting (never expected)
// a step with any of these leaves the state untouched: every later kernel of
// the step returns at entry (a stalled scan's offsets are not to be used)
constexpr int kFlagAbort = kFlagCapacity | kFlagCellCrowded | kFlagScanStall;

// The flags a kernel checks at entry were set by earlier kernels, so a plain
// (L1-cached) load sees them; a volatile load from every thread of a
// million-thread launch would queue a million requests on one L2 line.
__device__ __forceinline__ bool step_aborted(const int* flags)
{
    return flags && (*flags & kFlagAbort);
}

// Programmatic dependent launch: the kernels of a step are launched with the
// stream-serialization attribute relaxed, so that one is scheduled while the
// stream's previous kernel drains.  Each of them calls this first: it waits
// until the previous kernel has completed and its writes are visible (and so
// all earlier work of the stream), then lets the next kernel launch in turn.
// It comes before every return path, so that a kernel's completion still
// implies its predecessor's.  Without the attribute both are no-ops.
__device__ __forceinline__ void grid_dep_sync()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ---- cell hash: LinkedCell::computeCellId / computeLinearCellHash
//      (Grains/Component/src/LinkedCell.cpp:117-159): floor((p - min)/extent)
//      in IEEE double, linear hash (z*ny + y)*nx + x.  Out-of-grid centres are
//      clamped to the grid and flagged (the reference indexes out of bounds).
__global__ void k_hash(int n, const double* __restrict__ px, const double* __restrict__ py,
                       const double* __restrict__ pz, double mnx, double mny, double mnz,
                       double cell, uint32_t nx, uint32_t ny, uint32_t nz,
                       uint32_t* __restrict__ keys, uint32_t* __restrict__ ids,
                       int* __restrict__ flags)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n)
        return;
    const double p[3]  = {px[i], py[i], pz[i]};
    const double mn[3] = {mnx, mny, mnz};
    const uint32_t dim[3] = {nx, ny, nz};
    uint32_t       c[3];
    int            bad = 0;
#pragma unroll
    for(int k = 0; k < 3; ++k)
    {
        const double f = floor(__ddiv_rn(__dsub_rn(p[k], mn[k]), cell));
        if(!(f >= 0.0))
        {
            c[k] = 0;
            bad |= (f != f) ? kFlagNonFinite : kFlagOutOfDomain;
        }
        else if(f >= (double)dim[k])
        {
            c[k] = dim[k] - 1;
            bad |= kFlagOutOfDomain;
        }
        else
            c[k] = (uint32_t)f;
    }
    keys[i] = (c[2] * ny + c[1]) * nx + c[0];
    ids[i]  = (uint32_t)i;
    if(bad)
        atomicOr(flags, bad);
}

// ---- counting sort by cell --------------------------------------------------
// The sort the linked cell needs is by cell key with ascending particle id
// inside a cell (the order in which ComponentManagerCPU::updateLinks appends
// particles to its cell lists, ComponentManagerCPU.cpp:278-296).  With the
// cell count as the number of buckets, the exclusive scan of the per-cell
// counts is the cell-start table itself:
//   k_hash_count:    key per particle and count[key] += 1 (atomics)
//   scan:            cstart = exclusive scan of count (C + 1 entries)
//   k_cell_scatter:  each particle into a free slot of its cell (any order)
//   k_cell_rank:     each particle's rank among its cell's ids puts it in
//                    ascending-id order, and writes the sorted key, id and
//                    positions (the gather of the pair search) in one pass.
// The rank pass costs O(m^2) per cell of m particles; cells of more than
// kRankMaxCell particles flag kFlagCellCrowded and the caller sorts with the
// radix kernels below instead.
constexpr uint32_t kRankMaxCell = 512;

__global__ void k_hash_count(int n, const double* __restrict__ px, const double* __restrict__ py,
                             const double* __restrict__ pz, double mnx, double mny, double mnz,
                             double cell, uint32_t nx, uint32_t ny, uint32_t nz,
                             uint32_t* __restrict__ keys, uint32_t* __restrict__ count,
                             int* __restrict__ flags)
{
    grid_dep_sync();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n)
        return;
    const double   p[3]   = {px[i], py[i], pz[i]};
    const double   mn[3]  = {mnx, mny, mnz};
    const uint32_t dim[3] = {nx, ny, nz};
    uint32_t       c[3];
    int            bad = 0;
#pragma unroll
    for(int k = 0; k < 3; ++k)
    {
        const double f = floor(__ddiv_rn(__dsub_rn(p[k], mn[k]), cell));
        if(!(f >= 0.0))
        {
            c[k] = 0;
            bad |= (f != f) ? kFlagNonFinite : kFlagOutOfDomain;
        }
        else if(f >= (double)dim[k])
        {
            c[k] = dim[k] - 1;
            bad |= kFlagOutOfDomain;
        }
        else
            c[k] = (uint32_t)f;
    }
    const uint32_t key = (c[2] * ny + c[1]) * nx + c[0];
    keys[i]            = key;
    atomicAdd(&count[key], 1u);
    if(bad)
        atomicOr(flags, bad);
}

// count[] holds the per-cell counts again after the scan; each particle takes
// one of its cell's slots by decrementing it
__global__ void k_cell_scatter(int n, const uint32_t* __restrict__ keys,
                               const uint32_t* __restrict__ cstart, uint32_t* __restrict__ count,
                               uint32_t* __restrict__ unordered, const int* abort_flags)
{
    grid_dep_sync();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n || step_aborted(abort_flags))
        return;
    const uint32_t key  = keys[i];
    const uint32_t slot = cstart[key] + atomicSub(&count[key], 1u) - 1u;
    unordered[slot]     = (uint32_t)i;
}

// Particle e's entry at sorted position s: position and bounding radius
// (double4) and, when out32 is given, an FP32 copy for a conservative
// candidate pre-test: its radius is inflated by 2^-19 (|x| + |y| + |z| + r) =
// 32 u (...), u = 2^-24, and rounded up.  The rounding of the FP32 coordinates,
// of their difference and of the FP32 sum of squares (FMA or not) moves |d| by
// less than 1.01 u (|xa|_1 + |xb|_1) + 1.74 u |d| + 2.1 u |d|, so an FP32 "no
// overlap" (|d|^2 >= (wA + wB)^2) implies |d| >= (rA + rB)(1 + 26 u) in exact
// arithmetic, which the FP64 test also rejects.
__device__ __forceinline__ void put_sorted(uint32_t s, uint32_t e, const double* __restrict__ px,
                                           const double* __restrict__ py,
                                           const double* __restrict__ pz,
                                           const uint32_t* __restrict__ rb_id,
                                           const double* __restrict__ rcirc,
                                           double4* __restrict__ out, float4* __restrict__ out32)
{
    const double4 p = make_double4(px[e], py[e], pz[e], rcirc[rb_id[e]]);
    out[s]          = p;
    if(out32)
    {
        const double slack = 0x1p-19 * (fabs(p.x) + fabs(p.y) + fabs(p.z) + p.w);
        out32[s] = make_float4((float)p.x, (float)p.y, (float)p.z, __double2float_ru(p.w + slack));
    }
}

// slot t of the unordered cell lists -> its place in ascending-id order, with
// the sorted key and the sorted positions (put_sorted)
__global__ void k_cell_rank(int n, const uint32_t* __restrict__ unordered,
                            const uint32_t* __restrict__ keys, const uint32_t* __restrict__ cstart,
                            uint32_t* __restrict__ skeys, uint32_t* __restrict__ sids,
                            const double* __restrict__ px, const double* __restrict__ py,
                            const double* __restrict__ pz, const uint32_t* __restrict__ rb_id,
                            const double* __restrict__ rcirc, double4* __restrict__ out,
                            float4* __restrict__ out32, uint32_t* __restrict__ sorted_of,
                            int* __restrict__ flags)
{
    grid_dep_sync();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= n || step_aborted(flags))
        return;
    const uint32_t e   = unordered[t];
    const uint32_t key = keys[e];
    const uint32_t lo = cstart[key], hi = cstart[key + 1];
    uint32_t       s  = (uint32_t)t;
    if(hi - lo > kRankMaxCell)
        atomicOr(flags, kFlagCellCrowded); // keep a valid permutation; the caller redoes the sort
    else
    {
        uint32_t rank = 0;
        for(uint32_t u = lo; u < hi; ++u)
            rank += unordered[u] < e;
        s = lo + rank;
    }
    skeys[s]     = key;
    sids[s]      = e;
    sorted_of[e] = s;
    put_sorted(s, e, px, py, pz, rb_id, rcirc, out, out32);
}

// ---- radix sort, pass 1: per-block digit histograms, digit-major layout
//      hist[d * nblocks + block] so that one exclusive scan gives every
//      block's scatter base for every digit.
__global__ void __launch_bounds__(kBlock) k_radix_hist(const uint32_t* __restrict__ keys,
                                                       int n, int shift, uint32_t mask,
                                                       uint32_t* __restrict__ hist)
{
    __shared__ uint32_t h[256];
    const int           nb = (int)mask + 1;
    for(int b = threadIdx.x; b < nb; b += kBlock)
        h[b] = 0;
    __syncthreads();
    const int base = blockIdx.x * kTile;
#pragma unroll
    for(int j = 0; j < kItems; ++j)
    {
        const int idx = base + j * kBlock + threadIdx.x;
        if(idx < n)
            atomicAdd(&h[(keys[idx] >> shift) & mask], 1u);
    }
    __syncthreads();
    for(int b = threadIdx.x; b < nb; b += kBlock)
        hist[(size_t)b * gridDim.x + blockIdx.x] = h[b];
}

// ---- radix sort, pass 2: stable scatter.  Warp w of a block owns the
//      contiguous chunk [base + 256 w, base + 256 (w+1)) of the tile, so warp
//      order is index order.  Each warp counts its digits (leader lanes of
//      __match_any_sync groups, warp-private rows), a per-digit scan across
//      the warps turns the counts into absolute output positions, and a
//      second walk scatters with in-warp ranks.  Equal keys keep input order.
__global__ void __launch_bounds__(kBlock)
    k_radix_scatter(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                    uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, int n,
                    int shift, uint32_t mask, const uint32_t* __restrict__ hist_scan)
{
    __shared__ uint32_t cnt[kWarps][256];
    const int           tid  = threadIdx.x;
    const int           w    = tid >> 5;
    const int           lane = tid & 31;
    const unsigned      lt   = (1u << lane) - 1u;
    const int           nb   = (int)mask + 1;
    for(int i = tid; i < kWarps * 256; i += kBlock)
        (&cnt[0][0])[i] = 0;
    __syncthreads();
    const int chunk = blockIdx.x * kTile + w * (32 * kItems);
    uint32_t  k[kItems], dg[kItems];
#pragma unroll
    for(int r = 0; r < kItems; ++r)
    {
        const int  idx = chunk + r * 32 + lane;
        const bool v   = idx < n;
        k[r]           = v ? keys_in[idx] : 0u;
        dg[r]          = v ? ((k[r] >> shift) & mask) : (256u + (uint32_t)lane);
        const unsigned peers = __match_any_sync(0xffffffffu, dg[r]);
        if(v && lane == __ffs(peers) - 1)
            cnt[w][dg[r]] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    if(tid < nb)
    {
        uint32_t run = hist_scan[(size_t)tid * gridDim.x + blockIdx.x];
#pragma unroll
        for(int ww = 0; ww < kWarps; ++ww)
        {
            const uint32_t t = cnt[ww][tid];
            cnt[ww][tid]     = run;
            run += t;
        }
    }
    __syncthreads();
#pragma unroll
    for(int r = 0; r < kItems; ++r)
    {
        const int      idx   = chunk + r * 32 + lane;
        const bool     v     = idx < n;
        const unsigned peers = __match_any_sync(0xffffffffu, dg[r]);
        const int      lead  = __ffs(peers) - 1;
        uint32_t       off   = 0;
        if(v)
            off = cnt[w][dg[r]];
        __syncwarp();
        if(v)
        {
            const uint32_t pos = off + __popc(peers & lt);
            keys_out[pos]      = k[r];
            vals_out[pos]      = vals_in[idx];
            if(lane == lead)
                cnt[w][dg[r]] = off + __popc(peers);
        }
        __syncwarp();
    }
}

// ---- exclusive scan of uint32 in three kernels, no inter-block waiting ------
// (the static-scratch sort's scan; the engine's scans use k_scan_onepass below)
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for(int o = 1; o < 32; o <<= 1)
    {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if(lane >= o)
            x += y;
    }
    return x;
}

// exclusive scan of one value per thread across the block; returns the
// exclusive prefix and writes the block total to *total
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t x, uint32_t* total)
{
    __shared__ uint32_t ws[32];
    const int           lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int           nw   = (blockDim.x + 31) >> 5;
    const uint32_t      inc  = warp_incl_scan(x);
    if(lane == 31)
        ws[w] = inc;
    __syncthreads();
    if(w == 0)
    {
        uint32_t s = lane < nw ? ws[lane] : 0u;
        s          = warp_incl_scan(s);
        ws[lane]   = s;
    }
    __syncthreads();
    const uint32_t before = w ? ws[w - 1] : 0u;
    if(total)
        *total = ws[nw - 1];
    __syncthreads();
    return before + inc - x;
}

__global__ void __launch_bounds__(kBlock) k_scan_reduce(const uint32_t* __restrict__ in,
                                                        int64_t n, uint32_t* __restrict__ partial)
{
    const int64_t base = (int64_t)blockIdx.x * kTile + (int64_t)threadIdx.x * kItems;
    uint32_t      s    = 0;
#pragma unroll
    for(int j = 0; j < kItems; ++j)
        if(base + j < n)
            s += in[base + j];
    uint32_t tot;
    block_excl_scan(s, &tot);
    if(threadIdx.x == 0)
        partial[blockIdx.x] = tot;
}

// single block: exclusive scan of the per-tile partial sums, in chunks
// abort_flags (optional): a scan whose output belongs to an aborted step
// (step_aborted) leaves its output untouched
__global__ void __launch_bounds__(1024) k_scan_partials(uint32_t* __restrict__ partial, int m,
                                                        uint32_t* __restrict__ grand_total,
                                                        const int* abort_flags = nullptr)
{
    if(step_aborted(abort_flags))
        return;
    uint32_t carry = 0;
    for(int c = 0; c < m; c += 1024)
    {
        const int      i = c + threadIdx.x;
        const uint32_t x = i < m ? partial[i] : 0u;
        uint32_t       tot;
        const uint32_t ex = block_excl_scan(x, &tot);
        if(i < m)
            partial[i] = carry + ex;
        carry += tot;
    }
    if(threadIdx.x == 0 && grand_total)
        *grand_total = carry;
}

__global__ void __launch_bounds__(kBlock) k_scan_apply(const uint32_t* __restrict__ in,
                                                       uint32_t* __restrict__ out, int64_t n,
                                                       const uint32_t* __restrict__ partial,
                                                       const int* abort_flags = nullptr)
{
    if(step_aborted(abort_flags))
        return;
    const int64_t base = (int64_t)blockIdx.x * kTile + (int64_t)threadIdx.x * kItems;
    uint32_t      v[kItems];
    uint32_t      s = 0;
#pragma unroll
    for(int j = 0; j < kItems; ++j)
    {
        v[j] = base + j < n ? in[base + j] : 0u;
        s += v[j];
    }
    uint32_t run = partial[blockIdx.x] + block_excl_scan(s, nullptr);
#pragma unroll
    for(int j = 0; j < kItems; ++j)
        if(base + j < n)
        {
            out[base + j] = run;
            run += v[j];
        }
}

// One-pass exclusive scan (decoupled look-back: Merrill and Garland, "Single-
// pass Parallel Prefix Scan with Decoupled Look-back", 2016).  Each tile
// publishes its aggregate, then its inclusive prefix, in one 64-bit word:
// value in bits 0-31, status in bits 32-33 (1 aggregate, 2 inclusive prefix),
// the scan's epoch in bits 34-63.  A tile's exclusive prefix is the sum over
// its predecessors' words back to the first inclusive prefix, read 32 at a
// time by one warp.  Tiles are
// numbered in the order their blocks start (a ticket counter that only grows;
// `ticket_base` is its value before this launch), so every predecessor of a
// tile is already running and the look-back ends; a bound on the wait still
// stops it and flags kFlagScanStall.  Words of earlier scans carry another
// epoch and read as unpublished, so the state needs no clearing between scans.
// In place (in == out) is allowed.  abort_flags as for k_scan_apply.
constexpr unsigned long long kScanAggregate = 1ull, kScanPrefix = 2ull;
constexpr uint32_t           kScanEpochMask = (1u << 30) - 1u;
constexpr uint32_t           kScanSpinLimit = 1u << 20; // the default bound of the wait

__global__ void __launch_bounds__(kBlock)
    k_scan_onepass(const uint32_t* in, uint32_t* out, int64_t n,
                   unsigned long long* __restrict__ tile_state,
                   unsigned long long* __restrict__ ticket, unsigned long long ticket_base,
                   uint32_t epoch, uint32_t* __restrict__ grand_total,
                   const int* abort_flags, int* __restrict__ flags,
                   uint32_t spin_limit = kScanSpinLimit)
{
    grid_dep_sync();
    __shared__ uint32_t s_tile, s_prefix;
    if(threadIdx.x == 0)
        s_tile = (uint32_t)(atomicAdd(ticket, 1ull) - ticket_base);
    __syncthreads();
    if(step_aborted(abort_flags)) // every block alike, after taking its ticket
        return;
    const uint32_t tile = s_tile;
    if(tile >= gridDim.x) // a ticket count out of step with the host's: never expected
    {
        if(threadIdx.x == 0)
            atomicOr(flags, kFlagScanStall);
        return;
    }
    const int64_t  base = (int64_t)tile * kTile + (int64_t)threadIdx.x * kItems;
    uint32_t       v[kItems];
    uint32_t       s = 0;
    // a thread's kItems (8) consecutive entries in two 16-byte loads where
    // they lie wholly in range and the arrays are 16-byte aligned
    const bool vec = kItems == 8 && base + kItems <= n
                     && ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15u)
                            == 0;
    if(vec)
    {
        const uint4 a = *reinterpret_cast<const uint4*>(in + base);
        const uint4 b = *reinterpret_cast<const uint4*>(in + base + 4);
        v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w;
        v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
    }
    else
    {
#pragma unroll
        for(int j = 0; j < kItems; ++j)
            v[j] = base + j < n ? in[base + j] : 0u;
    }
#pragma unroll
    for(int j = 0; j < kItems; ++j)
        s += v[j];
    uint32_t       agg;
    const uint32_t ex = block_excl_scan(s, &agg);
    // the first warp looks back over 32 predecessors at a time: lane l reads
    // tile - 1 - l - 32 r; once none of the window is unpublished, the sum up
    // to the nearest inclusive prefix (or over the whole window) is taken
    if(threadIdx.x < 32)
    {
        const unsigned           lane = threadIdx.x;
        const uint32_t           ep   = epoch & kScanEpochMask;
        const unsigned long long tag  = (unsigned long long)ep << 34;
        uint32_t                 prefix = 0;
        if(tile > 0)
        {
            if(lane == 0)
                atomicExch(tile_state + tile, tag | (kScanAggregate << 32) | agg);
            int64_t  top   = (int64_t)tile - 1; // the window's newest predecessor
            uint32_t spins = 0;
            bool     done  = false;
            while(!done)
            {
                const int64_t      p = top - (int64_t)lane;
                unsigned long long w = 0;
                unsigned long long st;
                while(true)
                {
                    if(p < 0)
                        st = kScanPrefix; // before the first tile: prefix 0
                    else
                    {
                        w  = *(volatile unsigned long long*)(tile_state + p);
                        st = (uint32_t)(w >> 34) == ep ? (w >> 32) & 3ull : 0ull;
                    }
                    if(!__any_sync(0xffffffffu, st == 0ull))
                        break;
                    if(++spins > spin_limit)
                        break;
                }
                if(spins > spin_limit)
                {
                    if(lane == 0)
                        atomicOr(flags, kFlagScanStall);
                    break;
                }
                const uint32_t v       = p < 0 ? 0u : (uint32_t)w;
                const unsigned pmask   = __ballot_sync(0xffffffffu, st == kScanPrefix);
                const int      nearest = pmask ? __ffs(pmask) - 1 : 31;
                uint32_t       part    = (int)lane <= nearest ? v : 0u;
#pragma unroll
                for(int o = 16; o > 0; o >>= 1)
                    part += __shfl_xor_sync(0xffffffffu, part, o);
                prefix += part;
                done = pmask != 0u;
                top -= 32;
            }
            if(lane == 0)
                atomicExch(tile_state + tile, tag | (kScanPrefix << 32) | (prefix + agg));
        }
        else if(lane == 0)
            atomicExch(tile_state + tile, tag | (kScanPrefix << 32) | agg);
        if(lane == 0)
        {
            s_prefix = prefix;
            if(grand_total && (int64_t)(tile + 1) * kTile >= n)
                *grand_total = prefix + agg;
        }
    }
    __syncthreads();
    uint32_t run = s_prefix + ex;
    if(vec)
    {
        uint32_t o[kItems];
#pragma unroll
        for(int j = 0; j < kItems; ++j)
        {
            o[j] = run;
            run += v[j];
        }
        *reinterpret_cast<uint4*>(out + base)     = make_uint4(o[0], o[1], o[2], o[3]);
        *reinterpret_cast<uint4*>(out + base + 4) = make_uint4(o[4], o[5], o[6], o[7]);
        return;
    }
#pragma unroll
    for(int j = 0; j < kItems; ++j)
        if(base + j < n)
        {
            out[base + j] = run;
            run += v[j];
        }
}

// ---- cell-start table: start[c] = first sorted index whose key >= c, for all
//      c in [0, ncells] (so cell c holds [start[c], start[c+1]); empty cells
//      get an empty range).  A block covers kCellsPerBlock consecutive cells:
//      it locates its key range with two binary searches, stages those sorted
//      keys in shared memory, and answers each cell from there.
constexpr int kCellsPerBlock = 1024;
// Largest cell count of a grid: cell keys and k_cell_start's cell indices
// (up to ncells + kCellsPerBlock) stay below 2^32.
constexpr uint64_t kMaxCells = 0xFFFFFFFFull - 2 * kCellsPerBlock;
constexpr int kStageCap      = 4096;

__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* a, uint32_t n, uint32_t key)
{
    uint32_t lo = 0, hi = n;
    while(lo < hi)
    {
        const uint32_t mid = (lo + hi) >> 1;
        if(a[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(kBlock) k_cell_start(const uint32_t* __restrict__ skeys,
                                                       uint32_t n, uint32_t ncells,
                                                       uint32_t* __restrict__ start)
{
    __shared__ uint32_t range[2];
    __shared__ uint32_t sk[kStageCap];
    const uint32_t      c0 = blockIdx.x * kCellsPerBlock;
    if(threadIdx.x < 2)
    {
        // the block's key range in 64 bits: the upper bound of the last block
        // may lie past 2^32 - 1, beyond every key (callers keep ncells below
        // kMaxCells, so c0 + kCellsPerBlock does not wrap either)
        const uint64_t b = (uint64_t)c0 + (uint64_t)threadIdx.x * kCellsPerBlock;
        range[threadIdx.x] = lower_bound_u32(skeys, n, b > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)b);
    }
    __syncthreads();
    const uint32_t lo = range[0], hi = range[1];
    const uint32_t m  = hi - lo;
    const bool     staged = m <= (uint32_t)kStageCap;
    if(staged)
        for(uint32_t i = threadIdx.x; i < m; i += kBlock)
            sk[i] = skeys[lo + i];
    __syncthreads();
    for(int j = threadIdx.x; j < kCellsPerBlock; j += kBlock)
    {
        const uint32_t c = c0 + j;
        if(c > ncells)
            break;
        const uint32_t r = staged ? lower_bound_u32(sk, m, c) : lower_bound_u32(skeys + lo, m, c);
        start[c]         = lo + r;
    }
}

// positions and bounding radii in sorted order (put_sorted), for contiguous
// neighbour reads, after the radix sort
__global__ void k_gather_sorted(int n, const uint32_t* __restrict__ sids,
                                const double* __restrict__ px, const double* __restrict__ py,
                                const double* __restrict__ pz, const uint32_t* __restrict__ rb_id,
                                const double* __restrict__ rcirc, double4* __restrict__ out,
                                float4* __restrict__ out32, uint32_t* __restrict__ sorted_of)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= n)
        return;
    const uint32_t e = sids[t];
    sorted_of[e]     = (uint32_t)t;
    put_sorted((uint32_t)t, e, px, py, pz, rb_id, rcirc, out, out32);
}

} // namespace gb
