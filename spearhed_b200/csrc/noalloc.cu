// sph_density_noalloc: density summation on caller-owned device arrays, with no
// device allocation at all.
//
// Who needs it: code that must not call cudaMalloc/cudaFree while it runs — a
// host framework that owns every byte of device memory through its own pool
// (and would see foreign allocations as leaks or fragmentation), a solver that
// calls in from a phase where allocation would synchronise the device, or a
// plugin inside another program that forbids the CUDA allocator.  The regular
// entry points allocate their buffers inside the context (sph_create /
// sph_set_species / first compute call); this one uses a fixed scratch area
// instead.
//
// Scratch: one file-scope device array of kScratchBytes (32 MiB), present on
// every GPU that loads this library for as long as the process lives.  It holds
// the cell keys and particle indices of the radix sort (two copies each), the
// sort's tile histograms, the cell ranges and the packed positions of the
// sorted particles.  Limits: at most kMaxParticles particles and kMaxCells cells,
// and the layout must fit the array; larger calls return SPH_ERR_INVALID.
//
// Every call shares the one array, and it keeps the previous call's contents:
// everything that must start at zero (the cell ranges) is cleared by each call.
// Calls whose device work overlaps (two host threads, or two streams, without
// ordering between them) race on the array and give wrong results.
//
// Set-up: the first call on each device looks up the array's device address
// with cudaGetSymbolAddress while that device is current; that first call
// should be made before any stream capture begins.  The address is kept for
// the life of the process, so the entry point must not be called on a device
// after cudaDeviceReset() on it (the reset unloads the module that holds the
// array; a later call would write through the stale address).
//
// Inputs are checked on the device as in sph_set_species: a non-finite
// position, or a mass or h that is not finite and positive, returns
// SPH_ERR_NONFINITE; a finite position outside the box returns SPH_ERR_OUTSIDE.
// Those inputs are found by the same launch sequence that computes rho, so
// on either return rho holds values that must not be used.  Every call waits
// for its own work on `stream` before it returns.
#include "sph_launch.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

namespace sph
{
    int recordError(int code, std::string msg); // context.cu: sets sph_last_error_string()
}

namespace
{
    constexpr size_t kScratchBytes = size_t(32) << 20;
    constexpr uint32_t kMaxParticles = 1u << 18;
    constexpr uint32_t kMaxCells = 1u << 18;
    constexpr int kMaxDevices = 64;

    static __device__ __align__(256) unsigned char g_noallocScratch[kScratchBytes];

    std::mutex g_addrLock;
    void* g_scratchAddr[kMaxDevices] = {};

    int failNoAlloc(int code, std::string msg)
    {
        return sph::recordError(code, std::move(msg));
    }

    //! Device address of the scratch array on the current device (looked up once per device).
    int scratchAddress(int device, void** out)
    {
        std::lock_guard<std::mutex> g(g_addrLock);
        if(!g_scratchAddr[device])
        {
            void* p = nullptr;
            cudaError_t const e = cudaGetSymbolAddress(&p, g_noallocScratch);
            if(e != cudaSuccess || !p)
                return failNoAlloc(SPH_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_scratchAddr[device] = p;
        }
        *out = g_scratchAddr[device];
        return SPH_OK;
    }

    //! Bump allocator over the scratch array (256-byte aligned slices).
    struct Carve
    {
        unsigned char* base;
        size_t used = 0;
        template<typename T>
        T* take(size_t count)
        {
            used = (used + 255) & ~size_t(255);
            T* p = reinterpret_cast<T*>(base + used);
            used += count * sizeof(T);
            return p;
        }
    };

    constexpr int kThreads = 256;
    constexpr int kWarps = 4;

    //! Cell key of every particle (input order); one box, every particle a target.
    //! status[0] counts finite positions outside the box (on every axis,
    //! periodic ones included), status[1] non-finite positions and masses or
    //! smoothing lengths that are not finite and positive.
    __global__ void kKeysInput(
        sph::BoxDev const* __restrict__ box,
        uint32_t n,
        double const* __restrict__ x,
        double const* __restrict__ y,
        double const* __restrict__ z,
        double const* __restrict__ m,
        double const* __restrict__ h,
        uint32_t* __restrict__ keys,
        uint32_t* __restrict__ vals,
        uint32_t* __restrict__ status)
    {
        uint32_t const p = blockIdx.x * blockDim.x + threadIdx.x;
        if(p >= n)
            return;
        sph::BoxDev const& B = *box;
        double const pos[3] = {x[p], y[p], z[p]};
        double const mp = m[p], hp = h[p];
        bool nonfinite = !(isfinite(mp) && mp > 0.0) || !(isfinite(hp) && hp > 0.0);
        bool outside = false;
        for(int a = 0; a < 3; ++a)
        {
            nonfinite = nonfinite || !isfinite(pos[a]);
            outside = outside || pos[a] < B.lo[a] || pos[a] > B.lo[a] + B.L[a];
        }
        if(nonfinite)
            atomicAdd(&status[1], 1u);
        else if(outside)
            atomicAdd(&status[0], 1u);
        int const cx = sph::cellCoord(B, 0, isfinite(pos[0]) ? pos[0] : B.lo[0]);
        int const cy = sph::cellCoord(B, 1, isfinite(pos[1]) ? pos[1] : B.lo[1]);
        int const cz = sph::cellCoord(B, 2, isfinite(pos[2]) ? pos[2] : B.lo[2]);
        keys[p] = 2u * ((uint32_t(cz) * uint32_t(B.n[1]) + uint32_t(cy)) * uint32_t(B.n[0]) + uint32_t(cx));
        vals[p] = p;
    }

    template<typename V4, typename T>
    __global__ void kPackSorted(
        sph::BoxDev const* __restrict__ box,
        uint32_t n,
        uint32_t const* __restrict__ perm,
        double const* __restrict__ x,
        double const* __restrict__ y,
        double const* __restrict__ z,
        double const* __restrict__ m,
        double const* __restrict__ h,
        V4* __restrict__ pm,
        T* __restrict__ hc)
    {
        uint32_t const p = blockIdx.x * blockDim.x + threadIdx.x;
        if(p >= n)
            return;
        uint32_t const q = perm[p];
        sph::BoxDev const& B = *box;
        double const pos[3] = {x[q], y[q], z[q]};
        double rel[3];
        for(int a = 0; a < 3; ++a)
        {
            int const ca = sph::cellCoord(B, a, pos[a]);
            rel[a] = __dsub_rn(pos[a], cellOrigin(B, a, ca));
        }
        pm[p] = sph::mk4<V4>(rel[0], rel[1], rel[2], m[q]);
        hc[p] = T(h[q]);
    }

    __device__ __forceinline__ float mulRn(float a, float b)
    {
        return __fmul_rn(a, b);
    }
    __device__ __forceinline__ float addRn(float a, float b)
    {
        return __fadd_rn(a, b);
    }
    __device__ __forceinline__ double mulRn(double a, double b)
    {
        return __dmul_rn(a, b);
    }
    __device__ __forceinline__ double addRn(double a, double b)
    {
        return __dadd_rn(a, b);
    }

    template<typename T>
    __device__ __forceinline__ T edgeT(sph::BoxDev const& B, int a);
    template<>
    __device__ __forceinline__ float edgeT<float>(sph::BoxDev const& B, int a)
    {
        return B.edgef[a];
    }
    template<>
    __device__ __forceinline__ double edgeT<double>(sph::BoxDev const& B, int a)
    {
        return B.edge[a];
    }

    //! Density with the accumulation inside the cull (no neighbour list):
    //! one warp per cell, each lane one target, candidates read straight from
    //! the sorted records.  Same acceptance rule and summation order as the
    //! list-based kernel; the FP32 variant folds blocks of 8 accepted terms
    //! into a TwoSum-compensated sum.  rho is written in input order.
    template<int K, typename V4, typename T>
    __global__ void __launch_bounds__(kWarps * 32) kDensityInline(
        sph::BoxDev const* __restrict__ box,
        sph::Cells cells,
        uint32_t const* __restrict__ perm,
        V4 const* __restrict__ pm,
        T const* __restrict__ hc,
        double h0,
        double* __restrict__ rhoOut)
    {
        sph::BoxDev const& B = *box;
        int const warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        T const sup = T(sph::Kern<K>::support);
        T const Rg = mulRn(sup, T(h0));
        T const R2g = mulRn(Rg, Rg);
        for(uint32_t cell = blockIdx.x * kWarps + warp; cell < cells.ncells; cell += gridDim.x * kWarps)
        {
            uint32_t const tBeg = cells.start[cell], tEnd = cells.mid[cell];
            if(tBeg >= tEnd)
                continue;
            int const cc[3] = {int(cell % uint32_t(B.n[0])), int((cell / uint32_t(B.n[0])) % uint32_t(B.n[1])),
                               int(cell / (uint32_t(B.n[0]) * uint32_t(B.n[1])))};
            for(uint32_t tc = tBeg; tc < tEnd; tc += 32)
            {
                uint32_t const t = tc + uint32_t(lane);
                if(t >= tEnd)
                    continue;
                V4 const own = sph::ld4(pm + t);
                T const hi = hc[t];
                sph::HConst<T> const hk = sph::hconst<K, T>(hi);
                T acc = own.w * sph::kernelW<K, T>(T(0), hk);
                sph::CompAcc comp;
                T part = T(0);
                int inBlock = 0;
                for(int sl = 0; sl < 27; ++sl)
                {
                    int nc[3];
                    bool ok = true;
                    T sh[3];
                    for(int a = 0; a < 3; ++a)
                    {
                        int const o = sph::stencilOff(sl, a);
                        nc[a] = cc[a] + o;
                        if(nc[a] < 0 || nc[a] >= B.n[a])
                        {
                            if(B.periodic[a])
                                nc[a] = (nc[a] + B.n[a]) % B.n[a];
                            else
                                ok = false;
                        }
                        sh[a] = T(o) * edgeT<T>(B, a);
                    }
                    if(!ok)
                        continue;
                    uint32_t const ncell = (uint32_t(nc[2]) * uint32_t(B.n[1]) + uint32_t(nc[1])) * uint32_t(B.n[0])
                                           + uint32_t(nc[0]);
                    uint32_t const s = cells.start[ncell], e = cells.end[ncell];
                    for(uint32_t j = s; j < e; ++j)
                    {
                        if(sl == sph::kCentreSlot && j == t)
                            continue;
                        V4 const pj = sph::ld4(pm + j);
                        T const qx = pj.x + sh[0], qy = pj.y + sh[1], qz = pj.z + sh[2];
                        T const dx = own.x - qx, dy = own.y - qy, dz = own.z - qz;
                        // unfused, x then y then z: the acceptance test of the list-based kernel
                        T const r2 = addRn(addRn(mulRn(dx, dx), mulRn(dy, dy)), mulRn(dz, dz));
                        if(r2 < R2g)
                        {
                            T const r = r2 > T(0) ? r2 * (T(1) / sqrt(r2)) : T(0);
                            T const term = pj.w * sph::kernelW<K, T>(r, hk);
                            if constexpr(sizeof(T) == 4)
                            {
                                part += term;
                                if(++inBlock == 8)
                                {
                                    comp.fold(float(part));
                                    part = T(0);
                                    inBlock = 0;
                                }
                            }
                            else
                                acc += term;
                        }
                    }
                }
                double value;
                if constexpr(sizeof(T) == 4)
                {
                    comp.fold(float(part));
                    comp.fold(float(acc));
                    value = comp.value();
                }
                else
                    value = double(acc);
                rhoOut[perm[t]] = value;
            }
        }
    }

    template<int K, typename V4, typename T>
    void launchInline(
        sph::BoxDev const* box,
        sph::Cells const& cells,
        uint32_t const* perm,
        V4 const* pm,
        T const* hc,
        SphParams const& p,
        double* rho,
        cudaStream_t s)
    {
        uint32_t blocks = (cells.ncells + kWarps - 1) / kWarps;
        blocks = blocks > 148u * 32u ? 148u * 32u : blocks;
        // the global cull radius only: pair-max calls are refused before any launch
        kDensityInline<K, V4, T><<<blocks, kWarps * 32, 0, s>>>(box, cells, perm, pm, hc, p.h0, rho);
        sph::countLaunches(1);
    }

    template<typename V4, typename T>
    void launchInlineK(
        sph::BoxDev const* box,
        sph::Cells const& cells,
        uint32_t const* perm,
        V4 const* pm,
        T const* hc,
        SphParams const& p,
        double* rho,
        cudaStream_t s)
    {
        if(p.kernel == SPH_KERNEL_QUINTIC)
            launchInline<SPH_KERNEL_QUINTIC>(box, cells, perm, pm, hc, p, rho, s);
        else if(p.kernel == SPH_KERNEL_WENDLAND_C2)
            launchInline<SPH_KERNEL_WENDLAND_C2>(box, cells, perm, pm, hc, p, rho, s);
        else
            launchInline<SPH_KERNEL_CUBIC>(box, cells, perm, pm, hc, p, rho, s);
    }
} // namespace

extern "C" {

int sph_density_noalloc(
    SphParams const* params,
    SphBox const* box,
    int64_t n,
    double const* x,
    double const* y,
    double const* z,
    double const* mass,
    double const* h,
    double* rho,
    void* stream)
{
    if(!params || !box || n < 0 || (n > 0 && (!x || !y || !z || !mass || !h || !rho)))
        return failNoAlloc(SPH_ERR_INVALID, "sph_density_noalloc: null argument");
    SphParams const& p = *params;
    if(p.kernel < SPH_KERNEL_CUBIC || p.kernel > SPH_KERNEL_WENDLAND_C2 || !(p.h0 > 0.0)
       || (p.precision != SPH_PREC_FP64 && p.precision != SPH_PREC_FP32_COMP)
       || (p.cull != SPH_CULL_GLOBAL && p.cull != SPH_CULL_PAIR_MAX))
        return failNoAlloc(SPH_ERR_INVALID, "sph_density_noalloc: bad params");
    if(n == 0)
        return SPH_OK;
    if(uint64_t(n) > kMaxParticles)
        return failNoAlloc(
            SPH_ERR_INVALID,
            "sph_density_noalloc: " + std::to_string(n) + " particles exceed the fixed scratch limit of "
                + std::to_string(kMaxParticles));
    if(p.cull == SPH_CULL_PAIR_MAX)
        return failNoAlloc(
            SPH_ERR_UNSUPPORTED,
            "sph_density_noalloc: the global cull radius (SPH_CULL_GLOBAL) is required: the cell size cannot "
            "be derived from device-resident smoothing lengths without a host round trip");
    int device = 0;
    if(cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
        return failNoAlloc(SPH_ERR_CUDA, "sph_density_noalloc: no current CUDA device");
    // Cell grid of the box (same rule as the context path: edge >= support * h0).
    int const sup = p.kernel == SPH_KERNEL_QUINTIC ? 3 : 2;
    double const r64 = double(sup) * p.h0, r32 = double(float(sup) * float(p.h0));
    double const rc = (r64 > r32 ? r64 : r32) * (1.0 + 1.0 / 1048576.0);
    sph::BoxDev bd{};
    uint64_t ncells = 1;
    for(int a = 0; a < 3; ++a)
    {
        bd.lo[a] = box->lo[a];
        bd.L[a] = box->hi[a] - box->lo[a];
        if(!(bd.L[a] > 0.0) || !std::isfinite(bd.L[a]))
            return failNoAlloc(SPH_ERR_INVALID, "sph_density_noalloc: empty or non-finite box");
        bd.periodic[a] = box->periodic[a] ? 1 : 0;
        double const nd = std::floor(bd.L[a] / rc);
        bd.n[a] = nd < 1.0 ? 1 : (nd > 1.0e6 ? 1000000 : int32_t(nd));
        bd.edge[a] = bd.L[a] / bd.n[a];
        bd.edgef[a] = float(bd.edge[a]);
        if(bd.periodic[a] && bd.L[a] < rc)
            return failNoAlloc(SPH_ERR_UNSUPPORTED, "sph_density_noalloc: periodic box thinner than the radius");
        ncells *= uint64_t(bd.n[a]);
    }
    if(ncells > kMaxCells)
        return failNoAlloc(
            SPH_ERR_INVALID,
            "sph_density_noalloc: " + std::to_string(ncells) + " cells exceed the fixed scratch limit of "
                + std::to_string(kMaxCells));
    bd.cellBase = 0;
    bd.ncells = uint32_t(ncells);
    void* base = nullptr;
    int st = scratchAddress(device, &base);
    if(st)
        return st;
    uint32_t const nn = uint32_t(n);
    bool const fp64 = p.precision == SPH_PREC_FP64;
    Carve cv{static_cast<unsigned char*>(base)};
    sph::BoxDev* dBox = cv.take<sph::BoxDev>(1);
    uint32_t* status = cv.take<uint32_t>(4);
    uint32_t* keysA = cv.take<uint32_t>(nn);
    uint32_t* valsA = cv.take<uint32_t>(nn);
    uint32_t* keysB = cv.take<uint32_t>(nn);
    uint32_t* valsB = cv.take<uint32_t>(nn);
    uint32_t* sortScr = cv.take<uint32_t>(sph::radixScratchWords(nn));
    sph::Cells cells{};
    cells.ncells = uint32_t(ncells);
    cells.start = cv.take<uint32_t>(ncells);
    cells.mid = cv.take<uint32_t>(ncells);
    cells.end = cv.take<uint32_t>(ncells);
    sph::D4* pm64 = nullptr;
    double* hc64 = nullptr;
    float4* pm32 = nullptr;
    float* hc32 = nullptr;
    if(fp64)
    {
        pm64 = cv.take<sph::D4>(nn);
        hc64 = cv.take<double>(nn);
    }
    else
    {
        pm32 = cv.take<float4>(nn);
        hc32 = cv.take<float>(nn);
    }
    if(cv.used > kScratchBytes)
        return failNoAlloc(
            SPH_ERR_INVALID,
            "sph_density_noalloc: needs " + std::to_string(cv.used) + " bytes of scratch, the fixed array holds "
                + std::to_string(kScratchBytes));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // A launch error left pending by earlier, unrelated work on this thread
    // would otherwise be reported as this call's failure: clear it first.
    (void)cudaGetLastError();
    // Everything below is stream-ordered; nothing that must start at zero is
    // assumed to be zero from an earlier call.
    if(cudaMemcpyAsync(dBox, &bd, sizeof(bd), cudaMemcpyHostToDevice, s) != cudaSuccess
       || cudaMemsetAsync(status, 0, 4 * sizeof(uint32_t), s) != cudaSuccess)
        return failNoAlloc(SPH_ERR_CUDA, "sph_density_noalloc: stream operation failed");
    auto launched = [](char const* what) -> int
    {
        // launch configuration errors and failed memsets of the launchers
        cudaError_t const e = cudaGetLastError();
        if(e == cudaSuccess)
            return SPH_OK;
        return failNoAlloc(SPH_ERR_CUDA, std::string("sph_density_noalloc: ") + what + ": " + cudaGetErrorString(e));
    };
    unsigned const g = (nn + kThreads - 1) / kThreads;
    kKeysInput<<<g, kThreads, 0, s>>>(dBox, nn, x, y, z, mass, h, keysA, valsA, status);
    sph::countLaunches(1);
    if((st = launched("cell keys")))
        return st;
    int bits = 1;
    while((uint64_t(1) << bits) <= ncells * 2)
        ++bits;
    bool const inB = sph::radixSortPairs(keysA, valsA, keysB, valsB, nn, bits, sortScr, s);
    if((st = launched("radix sort")))
        return st;
    uint32_t const* keys = inB ? keysB : keysA;
    uint32_t const* perm = inB ? valsB : valsA;
    sph::DevCtx dc{};
    dc.n = nn;
    dc.cells = cells;
    sph::launchCellRanges(dc, keys, s); // clears start/mid/end, then fills them
    if((st = launched("cell ranges")))
        return st;
    if(fp64)
    {
        kPackSorted<sph::D4, double><<<g, kThreads, 0, s>>>(dBox, nn, perm, x, y, z, mass, h, pm64, hc64);
        sph::countLaunches(1);
        if((st = launched("packing")))
            return st;
        launchInlineK<sph::D4, double>(dBox, cells, perm, pm64, hc64, p, rho, s);
    }
    else
    {
        kPackSorted<float4, float><<<g, kThreads, 0, s>>>(dBox, nn, perm, x, y, z, mass, h, pm32, hc32);
        sph::countLaunches(1);
        if((st = launched("packing")))
            return st;
        launchInlineK<float4, float>(dBox, cells, perm, pm32, hc32, p, rho, s);
    }
    if((st = launched("density")))
        return st;
    // Bad inputs are only known after the work ran, so the density kernel is
    // told nothing; rho is written but must not be used on an error return.
    uint32_t bad[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(bad, status, sizeof(bad), cudaMemcpyDeviceToHost, s);
    if(e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if(e != cudaSuccess)
        return failNoAlloc(SPH_ERR_CUDA, std::string("sph_density_noalloc: ") + cudaGetErrorString(e));
    if(bad[1])
        return failNoAlloc(
            SPH_ERR_NONFINITE,
            "sph_density_noalloc: " + std::to_string(bad[1])
                + " particles with a non-finite position or a mass or h that is not finite and positive");
    if(bad[0])
        return failNoAlloc(
            SPH_ERR_OUTSIDE, "sph_density_noalloc: " + std::to_string(bad[0]) + " particles outside the box");
    return SPH_OK;
}
}
