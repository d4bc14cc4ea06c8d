// Device radix sort of (cell key, particle index) pairs and an exclusive scan.
//
// Replaces the reference's region bookkeeping (region AABB update, region-pair
// overlap search with a host-side inclusive scan in the middle of every step:
// spmacc/particles/regions/NeighbourRegions.hpp:140-222, RegionBoundsUpdate.hpp:39-215):
// particles are re-binned every step by a stable LSD radix sort on their cell
// key, with no host round trip.
//
// Layout: one pass per 8-bit digit.  A pass is (1) a per-tile digit histogram,
// (2) an exclusive scan of the digit-major [digit][tile] count table, (3) a
// stable scatter: every tile ranks its keys per digit in input order (warp
// __match_any_sync ranks, then a per-digit prefix over the warps of the block)
// and writes them at the scanned offset.  Tiles are 4096 keys (256 threads x
// 16 rounds); keys are read coalesced, once per kernel.
#include "sph_launch.hpp"

namespace sph
{
    namespace
    {
        constexpr int kThreads = 256;
        constexpr int kRounds = 16;
        constexpr int kTile = kThreads * kRounds;
        constexpr int kScanItems = 8;
        constexpr int kScanTile = kThreads * kScanItems;

        __global__ void __launch_bounds__(kThreads) kRadixHist(
            uint32_t const* __restrict__ keys,
            uint32_t n,
            int shift,
            uint32_t* __restrict__ tileHist,
            uint32_t ntile)
        {
            __shared__ uint32_t h[256];
            h[threadIdx.x] = 0;
            __syncthreads();
            uint32_t const base = blockIdx.x * uint32_t(kTile);
#pragma unroll 4
            for(int r = 0; r < kRounds; ++r)
            {
                uint32_t const i = base + uint32_t(r) * kThreads + threadIdx.x;
                if(i < n)
                    atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
            }
            __syncthreads();
            tileHist[threadIdx.x * ntile + blockIdx.x] = h[threadIdx.x];
        }

        __global__ void __launch_bounds__(kThreads) kRadixScatter(
            uint32_t const* __restrict__ keysIn,
            uint32_t const* __restrict__ valsIn,
            uint32_t* __restrict__ keysOut,
            uint32_t* __restrict__ valsOut,
            uint32_t n,
            int shift,
            uint32_t const* __restrict__ tileOffset,
            uint32_t ntile)
        {
            __shared__ uint32_t running[256];
            __shared__ uint32_t warpCnt[kThreads / 32][256];
            int const tid = threadIdx.x;
            int const warp = tid >> 5;
            int const lane = tid & 31;
            running[tid] = tileOffset[tid * ntile + blockIdx.x];
            uint32_t const lanesBelow = (1u << lane) - 1u;
            uint32_t const base = blockIdx.x * uint32_t(kTile);
            for(int r = 0; r < kRounds; ++r)
            {
                for(int w = 0; w < kThreads / 32; ++w)
                    warpCnt[w][tid] = 0;
                __syncthreads();
                uint32_t const i = base + uint32_t(r) * kThreads + tid;
                bool const valid = i < n;
                uint32_t key = 0, val = 0;
                if(valid)
                {
                    key = keysIn[i];
                    val = valsIn[i];
                }
                uint32_t const digit = (key >> shift) & 255u;
                // Invalid lanes get a value no valid lane can have, so they rank alone.
                uint32_t const peers = __match_any_sync(0xffffffffu, valid ? digit : 0x100u + uint32_t(lane));
                uint32_t const rank = __popc(peers & lanesBelow);
                bool const leader = (peers & lanesBelow) == 0u;
                if(valid && leader)
                    warpCnt[warp][digit] = __popc(peers);
                __syncthreads();
                {
                    uint32_t run = running[tid];
#pragma unroll
                    for(int w = 0; w < kThreads / 32; ++w)
                    {
                        uint32_t const c = warpCnt[w][tid];
                        warpCnt[w][tid] = run;
                        run += c;
                    }
                    running[tid] = run;
                }
                __syncthreads();
                if(valid)
                {
                    uint32_t const dst = warpCnt[warp][digit] + rank;
                    keysOut[dst] = key;
                    valsOut[dst] = val;
                }
                __syncthreads();
            }
        }

        //! Block-level exclusive scan of kScanTile items; writes each tile's total.
        __global__ void __launch_bounds__(kThreads) kScanTiles(
            uint32_t const* __restrict__ in,
            uint32_t* __restrict__ out,
            uint32_t m,
            uint32_t* __restrict__ tileSums)
        {
            __shared__ uint32_t warpTot[kThreads / 32];
            int const tid = threadIdx.x;
            int const lane = tid & 31;
            int const warp = tid >> 5;
            uint32_t const base = blockIdx.x * uint32_t(kScanTile) + uint32_t(tid) * kScanItems;
            uint32_t v[kScanItems];
            uint32_t sum = 0;
#pragma unroll
            for(int k = 0; k < kScanItems; ++k)
            {
                uint32_t const i = base + k;
                v[k] = i < m ? in[i] : 0u;
                sum += v[k];
            }
            uint32_t incl = sum;
#pragma unroll
            for(int d = 1; d < 32; d <<= 1)
            {
                uint32_t const o = __shfl_up_sync(0xffffffffu, incl, d);
                if(lane >= d)
                    incl += o;
            }
            if(lane == 31)
                warpTot[warp] = incl;
            __syncthreads();
            uint32_t warpBase = 0, blockTot = 0;
#pragma unroll
            for(int w = 0; w < kThreads / 32; ++w)
            {
                uint32_t const t = warpTot[w];
                if(w < warp)
                    warpBase += t;
                blockTot += t;
            }
            uint32_t run = warpBase + incl - sum;
#pragma unroll
            for(int k = 0; k < kScanItems; ++k)
            {
                uint32_t const i = base + k;
                if(i < m)
                    out[i] = run;
                run += v[k];
            }
            if(tid == 0 && tileSums)
                tileSums[blockIdx.x] = blockTot;
        }

        __global__ void kAddTileBase(uint32_t* __restrict__ out, uint32_t m, uint32_t const* __restrict__ tileBase)
        {
            uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
            if(i < m)
                out[i] += tileBase[i / kScanTile];
        }
    } // namespace

    size_t scanScratchWords(uint32_t m)
    {
        size_t words = 0;
        while(m > uint32_t(kScanTile))
        {
            m = (m + kScanTile - 1) / kScanTile;
            words += 2 * size_t(m);
        }
        return words + 2;
    }

    void exclusiveScan(uint32_t const* in, uint32_t* out, uint32_t m, uint32_t* scratch, cudaStream_t s)
    {
        if(m == 0)
            return;
        uint32_t const ntile = (m + kScanTile - 1) / kScanTile;
        if(ntile == 1)
        {
            kScanTiles<<<1, kThreads, 0, s>>>(in, out, m, nullptr);
            countLaunches(1);
            return;
        }
        uint32_t* sums = scratch;
        uint32_t* sumsScanned = scratch + ntile;
        kScanTiles<<<ntile, kThreads, 0, s>>>(in, out, m, sums);
        countLaunches(1);
        exclusiveScan(sums, sumsScanned, ntile, scratch + 2 * size_t(ntile), s);
        kAddTileBase<<<(m + 255) / 256, 256, 0, s>>>(out, m, sumsScanned);
        countLaunches(1);
    }

    size_t radixScratchWords(uint32_t n)
    {
        uint32_t const ntile = (n + kTile - 1) / kTile;
        size_t const hist = size_t(256) * ntile;
        return 2 * hist + scanScratchWords(uint32_t(hist));
    }

    bool radixSortPairs(
        uint32_t* keysA,
        uint32_t* valsA,
        uint32_t* keysB,
        uint32_t* valsB,
        uint32_t n,
        int bits,
        uint32_t* scratch,
        cudaStream_t s)
    {
        bool inB = false;
        if(n == 0)
            return inB;
        uint32_t const ntile = (n + kTile - 1) / kTile;
        size_t const hist = size_t(256) * ntile;
        uint32_t* tileHist = scratch;
        uint32_t* tileOff = scratch + hist;
        uint32_t* scanScr = scratch + 2 * hist;
        for(int shift = 0; shift < bits; shift += 8)
        {
            uint32_t const* kin = inB ? keysB : keysA;
            uint32_t const* vin = inB ? valsB : valsA;
            uint32_t* kout = inB ? keysA : keysB;
            uint32_t* vout = inB ? valsA : valsB;
            kRadixHist<<<ntile, kThreads, 0, s>>>(kin, n, shift, tileHist, ntile);
            countLaunches(1);
            exclusiveScan(tileHist, tileOff, uint32_t(hist), scanScr, s);
            kRadixScatter<<<ntile, kThreads, 0, s>>>(kin, vin, kout, vout, n, shift, tileOff, ntile);
            countLaunches(1);
            inB = !inB;
        }
        return inB;
    }
} // namespace sph
