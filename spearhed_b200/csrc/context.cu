// Host runtime and C ABI of the B200 SPH step (include/spearhed_b200.h).
//
// One sph_ctx owns one CUDA stream and all device memory of a run.  A step is
// a fixed sequence of launches on that stream with every scalar it needs (dt,
// time, c_h, the CFL minimum) kept in device memory, so a step never waits for
// the host and pairs of steps are captured into CUDA graphs on request.  This
// takes the place of the reference's runOneStep sender graph and of its two
// host round trips per step (NeighbourRegions.hpp:186-191, FrameIndex.hpp:209-280).
//
// Data flow: sph_set_species keeps a host mirror until the first compute call
// allocates the device state; after that, a species of unchanged size is
// copied straight from the caller's columns (pinned memory makes these copies
// asynchronous) into a staging column and gathered into the sorted state.
#include "sph_launch.hpp"

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

namespace
{
    thread_local std::string g_lastError;

    int fail(int code, std::string msg)
    {
        g_lastError = std::move(msg);
        return code;
    }

#define SPH_CUDA_TRY(expr)                                                                                             \
    do                                                                                                                 \
    {                                                                                                                  \
        cudaError_t const e_ = (expr);                                                                                 \
        if(e_ != cudaSuccess)                                                                                          \
            return fail(                                                                                               \
                e_ == cudaErrorMemoryAllocation ? SPH_ERR_NOMEM : SPH_ERR_CUDA,                                        \
                std::string(#expr) + ": " + cudaGetErrorString(e_));                                                   \
    } while(0)

    // Host columns of a species, in the order of the master state.
    constexpr int kHostCols = 14;
    enum
    {
        cX = 0,
        cY,
        cZ,
        cVX,
        cVY,
        cVZ,
        cU,
        cM,
        cH,
        cRho,
        cBX,
        cBY,
        cBZ,
        cPsi
    };

    struct HostSpecies
    {
        bool declared = false; //!< sph_set_species was called, possibly with no particles
        bool set = false;
        uint32_t roles = 0;
        int64_t n = 0;
        std::vector<double> col[kHostCols];
        std::vector<int32_t> box;
        uint32_t offset = 0;
    };

    int supportOf(int kernel)
    {
        return kernel == SPH_KERNEL_QUINTIC ? 3 : 2;
    }

    //! Smallest admissible cell edge for cull radius support*h: the larger of
    //! the FP64 and FP32 radius, widened by 2^-20 (same rule as the oracle).
    double cellRadius(int sup, double h)
    {
        double const r64 = double(sup) * h;
        double const r32 = double(float(sup) * float(h));
        return (r64 > r32 ? r64 : r32) * (1.0 + 1.0 / 1048576.0);
    }

    //! Input pointer of host column c in a view (nullptr when absent).
    double const* viewCol(SphSoAView const* v, int c)
    {
        if(!v)
            return nullptr;
        switch(c)
        {
        case cX:
        case cY:
        case cZ:
            return v->pos[c - cX];
        case cVX:
        case cVY:
        case cVZ:
            return v->vel[c - cVX];
        case cU:
            return v->u;
        case cM:
            return v->mass;
        case cH:
            return v->h;
        case cRho:
            return v->density;
        case cBX:
        case cBY:
        case cBZ:
            return v->B[c - cBX];
        case cPsi:
            return v->psi;
        }
        return nullptr;
    }

    int validateParams(SphParams const& p)
    {
        if(p.kernel < SPH_KERNEL_CUBIC || p.kernel > SPH_KERNEL_WENDLAND_C2)
            return fail(SPH_ERR_INVALID, "unknown kernel");
        if(p.precision != SPH_PREC_FP64 && p.precision != SPH_PREC_FP32_COMP)
            return fail(SPH_ERR_INVALID, "unknown precision");
        if(p.cull != SPH_CULL_GLOBAL && p.cull != SPH_CULL_PAIR_MAX)
            return fail(SPH_ERR_INVALID, "unknown cull mode");
        if(!(p.h0 > 0.0) || !std::isfinite(p.h0))
            return fail(SPH_ERR_INVALID, "h0 must be positive");
        if(!(p.gamma > 1.0))
            return fail(SPH_ERR_INVALID, "gamma must be > 1");
        if((p.physics & SPH_PHYS_DEDNER) && !(p.physics & SPH_PHYS_MHD))
            return fail(SPH_ERR_INVALID, "Dedner cleaning needs SPH_PHYS_MHD");
        if(p.max_neighbours < 0)
            return fail(SPH_ERR_INVALID, "max_neighbours must be >= 0");
        if((p.physics & SPH_PHYS_ADAPTIVE_H) && (p.cull != SPH_CULL_PAIR_MAX || !(p.hfact > 0.0)))
            return fail(SPH_ERR_INVALID, "adaptive h needs SPH_CULL_PAIR_MAX and hfact > 0");
        if(p.h_max < 0.0 || !std::isfinite(p.h_max))
            return fail(SPH_ERR_INVALID, "h_max must be >= 0");
        return SPH_OK;
    }
} // namespace

namespace sph
{
    //! NVTX range over a host scope (the launches of one pass, or one public
    //! call): profilers show the passes by name; without a tool attached a
    //! push/pop costs a branch.
    struct NvtxRange
    {
        explicit NvtxRange(char const* name)
        {
            nvtxRangePushA(name);
        }
        ~NvtxRange()
        {
            nvtxRangePop();
        }
        NvtxRange(NvtxRange const&) = delete;
        NvtxRange& operator=(NvtxRange const&) = delete;
    };

    //! Test hook (sphx_fail_alloc_after): device allocations left before the
    //! next one is refused with SPH_ERR_NOMEM; negative = no injection.
    std::atomic<long long> g_allocFailAfter{-1};

    //! True when the injection hook refuses this allocation (it then disarms).
    bool allocRefused()
    {
        long long k = g_allocFailAfter.load();
        while(k >= 0)
        {
            if(g_allocFailAfter.compare_exchange_weak(k, k - 1))
                return k == 0;
        }
        return false;
    }

    //! Records the message sph_last_error_string() returns on this thread.
    int recordError(int code, std::string msg)
    {
        return fail(code, std::move(msg));
    }
} // namespace sph

struct sph_ctx
{
    SphParams p{};
    cudaStream_t stream = nullptr;
    std::vector<SphBox> boxes;
    HostSpecies sp[SPH_NUM_SPECIES];
    bool allocated = false;     //!< device buffers exist for (allocN, allocCells, allocBoxes)
    bool deviceCurrent = false; //!< the device state holds the latest species data
    bool mirrorStale = false;   //!< the host mirror is older than the device state
    bool densityValid = false;
    bool forceValid = false;
    uint32_t n = 0, ncells = 0, activeCells = 0;
    uint32_t allocN = 0, allocCells = 0, allocBoxes = 0;
    std::vector<sph::BoxDev> boxDesc;
    sph::DevCtx dc{};
    sph::PhysArgs pa{};
    std::vector<void*> allocs;
    double* boxOut = nullptr;
    double* boxScratch = nullptr;
    std::vector<double*> staging;
    bool useGraph = false;
    cudaGraphExec_t graphs[2] = {nullptr, nullptr};
    unsigned graphKernels[2] = {0, 0}; //!< kernels in each captured two-step graph
    // Each captured graph records the stage-boundary events of its two steps; before
    // every replay its event-record nodes are pointed at that replay's own events,
    // so graph steps are timed per stage like eager ones.
    cudaGraph_t graphRaw[2] = {nullptr, nullptr};
    cudaEvent_t graphEv[2][10] = {};
    cudaGraphNode_t graphEvNode[2][10] = {};
    int parity = 0;
    std::vector<cudaEvent_t> events;
    cudaEvent_t eCall = nullptr; //!< start of a step call (before its snapshot)
    // Host<->device column copies run on their own stream so the copy engine
    // works while the gather / unpermute kernels of other columns run.
    cudaStream_t copyStream = nullptr;
    cudaEvent_t eCopy = nullptr, eCompute = nullptr;
    double timings[5] = {0, 0, 0, 0, 0};
    // State a step call starts from, restored when a neighbour list overflowed
    // in any of its steps: the call then regrows the lists and runs again.
    int densityVariant = 0, forceVariant = 0; //!< launch shapes (sph_autotune / sph_set_tuning)
    int64_t replays = 0;                      //!< step calls re-run after a list overflow
    // A context whose species hold no particles steps as a no-op, as the
    // reference's runOneStep does on an empty setup; its clock lives here.
    int64_t emptySteps = 0;
    double emptyTime = 0.0;
    bool empty() const
    {
        for(auto const& s : sp)
            if(s.set)
                return false;
        return true;
    }
    bool anyTwoLevel = false;                 //!< some box allocates level-1 cells
    uint32_t lastStat[sph::kStatWords] = {};  //!< status words of the last checkStatus
    // Bounded waits (sph_set_wait_timeout): a compute call whose device work
    // has not finished within waitLimit seconds returns SPH_ERR_TIMEOUT and
    // leaves its checks pending; sph_wait or the next call completes them.
    double waitLimit = 0.0;  //!< 0: wait without a limit
    bool boundedWait = false; //!< the running public call honours waitLimit
    cudaEvent_t eWait = nullptr;
    enum Pending
    {
        kPendNone = 0,
        kPendStep,
        kPendDensity,
        kPendForce
    };
    int pending = kPendNone;
    int32_t pendingSteps = 0;
    SphTuning tuning{};
    bool haveSnap = false;
    sph::Master snap{};
    sph::BoxScalars snapBs{};
    sph::StepScalars* snapScal = nullptr;

    ~sph_ctx()
    {
        release();
        for(cudaEvent_t e : events)
            cudaEventDestroy(e);
        for(auto& row : graphEv)
            for(cudaEvent_t e : row)
                if(e)
                    cudaEventDestroy(e);
        if(eCall)
            cudaEventDestroy(eCall);
        if(eWait)
            cudaEventDestroy(eWait);
        if(eCopy)
            cudaEventDestroy(eCopy);
        if(eCompute)
            cudaEventDestroy(eCompute);
        if(copyStream)
            cudaStreamDestroy(copyStream);
        if(stream)
            cudaStreamDestroy(stream);
    }

    //! The copy stream and its two hand-off events, created on first use.
    int ensureCopyStream()
    {
        if(!copyStream)
            SPH_CUDA_TRY(cudaStreamCreateWithFlags(&copyStream, cudaStreamNonBlocking));
        if(!eCopy)
            SPH_CUDA_TRY(cudaEventCreateWithFlags(&eCopy, cudaEventDisableTiming));
        if(!eCompute)
            SPH_CUDA_TRY(cudaEventCreateWithFlags(&eCompute, cudaEventDisableTiming));
        return SPH_OK;
    }

    void dropGraphs()
    {
        for(auto& g : graphs)
            if(g)
            {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
        for(auto& r : graphRaw)
            if(r)
            {
                cudaGraphDestroy(r);
                r = nullptr;
            }
    }

    void release()
    {
        dropGraphs();
        if(stream)
            cudaStreamSynchronize(stream);
        for(void* a : allocs)
            cudaFree(a);
        allocs.clear();
        staging.clear();
        dc = sph::DevCtx{};
        boxOut = nullptr;
        boxScratch = nullptr;
        haveSnap = false;
        snap = sph::Master{};
        snapBs = sph::BoxScalars{};
        snapScal = nullptr;
        allocated = false;
        deviceCurrent = false;
        densityValid = false;
        forceValid = false;
        parity = 0;
    }

    template<typename T>
    int alloc(T*& out, size_t count)
    {
        out = nullptr;
        if(count == 0)
            count = 1;
        void* ptr = nullptr;
        if(sph::allocRefused())
            return fail(SPH_ERR_NOMEM, "cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes: refused (injected)");
        cudaError_t const e = cudaMalloc(&ptr, count * sizeof(T));
        if(e != cudaSuccess)
            return fail(
                SPH_ERR_NOMEM,
                std::string("cudaMalloc of ") + std::to_string(count * sizeof(T)) + " bytes: " + cudaGetErrorString(e));
        allocs.push_back(ptr);
        out = static_cast<T*>(ptr);
        return SPH_OK;
    }

    int allocMaster(sph::Master& m)
    {
        int st = SPH_OK;
        for(int a = 0; a < 3 && !st; ++a)
            st = alloc(m.x[a], n);
        for(int a = 0; a < 3 && !st; ++a)
            st = alloc(m.v[a], n);
        for(int a = 0; a < 3 && !st; ++a)
            st = alloc(m.B[a], n);
        if(!st)
            st = alloc(m.u, n);
        if(!st)
            st = alloc(m.m, n);
        if(!st)
            st = alloc(m.h, n);
        if(!st)
            st = alloc(m.rho, n);
        if(!st)
            st = alloc(m.psi, n);
        if(!st)
            st = alloc(m.id, n);
        if(!st)
            st = alloc(m.box, n);
        if(!st)
            st = alloc(m.role, n);
        return st;
    }

    static double* masterCol(sph::Master const& m, int c)
    {
        switch(c)
        {
        case cX:
        case cY:
        case cZ:
            return m.x[c - cX];
        case cVX:
        case cVY:
        case cVZ:
            return m.v[c - cVX];
        case cU:
            return m.u;
        case cM:
            return m.m;
        case cH:
            return m.h;
        case cRho:
            return m.rho;
        case cBX:
        case cBY:
        case cBZ:
            return m.B[c - cBX];
        case cPsi:
            return m.psi;
        }
        return nullptr;
    }

    double colDefault(int c) const
    {
        return c == cH ? p.h0 : 0.0;
    }

    void physArgs()
    {
        pa.gamma = p.gamma;
        pa.alpha = p.alpha;
        pa.beta = p.beta;
        pa.avEps = p.av_eps;
        pa.mu0 = p.mu0 > 0 ? p.mu0 : 1.0;
        pa.cfl = p.cfl;
        pa.cflForce = p.cfl_force;
        pa.sigma = p.dedner_sigma;
        pa.h0 = p.h0;
        pa.hfact = p.hfact;
        pa.physics = p.physics;
        pa.cull = p.cull;
    }

    int stagingCols(size_t k)
    {
        while(staging.size() < k)
        {
            double* s = nullptr;
            int st = alloc(s, n);
            if(st)
                return st;
            staging.push_back(s);
        }
        return SPH_OK;
    }

    int layout();
    int allocate();
    int uploadMirror();
    int downloadMirror();
    int ensureDevice();
    int probeListCapacity();
    int growLists(uint32_t need, bool bestEffort = false);
    int build(bool drift);
    int clearStatus();
    int waitStream(char const* where);
    int evalStatus(char const* where);
    int checkStatus(char const* where);
    int completePending();
    void collectTimings(int32_t nsteps);
    int snapshot(bool restore);
    int runSteps(int32_t nsteps);
    int autotune(int32_t stepsPerTrial);
    int prepareGraph();
    void describeTuning();
    int densityPass();
    int forcePass();
    int stepOnce(cudaEvent_t const* ev, bool capture = false);
    int steps(int32_t nsteps, double dt);
    int setSpeciesFast(int32_t id, SphSoAView const* v);
};

//! Species offsets, host-side validation and the cell grid of every box.
int sph_ctx::layout()
{
    uint64_t total = 0;
    for(auto& s : sp)
        if(s.set)
        {
            s.offset = uint32_t(total);
            total += uint64_t(s.n);
        }
    if(total == 0)
        return fail(SPH_ERR_STATE, "no particles: call sph_set_species first");
    if(total >= sph::kMaxParticles)
        return fail(SPH_ERR_UNSUPPORTED, "more than 2^27 particles in one context");
    n = uint32_t(total);
    int const sup = supportOf(p.kernel);
    if(boxes.empty())
    {
        // Default domain: the particles' bounding box plus one radius, open.
        SphBox b{};
        double hmax = p.h0;
        for(int a = 0; a < 3; ++a)
        {
            b.lo[a] = 1e300;
            b.hi[a] = -1e300;
        }
        for(auto& s : sp)
            for(int64_t i = 0; s.set && i < s.n; ++i)
            {
                for(int a = 0; a < 3; ++a)
                {
                    b.lo[a] = std::min(b.lo[a], s.col[cX + a][i]);
                    b.hi[a] = std::max(b.hi[a], s.col[cX + a][i]);
                }
                hmax = std::max(hmax, s.col[cH][i]);
            }
        double const m = cellRadius(sup, hmax);
        for(int a = 0; a < 3; ++a)
        {
            b.lo[a] -= m;
            b.hi[a] += m;
        }
        boxes.push_back(b);
    }
    int32_t const nbox = int32_t(boxes.size());
    std::vector<double> hmax(nbox, p.cull == SPH_CULL_PAIR_MAX ? 0.0 : p.h0);
    std::vector<double> hmin(nbox, 1e300);
    for(auto& s : sp)
    {
        if(!s.set)
            continue;
        for(int64_t i = 0; i < s.n; ++i)
        {
            int32_t const b = s.box[i];
            if(b < 0 || b >= nbox)
                return fail(SPH_ERR_INVALID, "box_id out of range");
            SphBox const& B = boxes[b];
            for(int a = 0; a < 3; ++a)
            {
                double const x = s.col[cX + a][i];
                if(!std::isfinite(x))
                    return fail(SPH_ERR_NONFINITE, "non-finite position in the input");
                // periodic axes too: the cell search covers [lo, hi]; the drift
                // wraps movable particles back into it every step
                if(x < B.lo[a] || x > B.hi[a])
                    return fail(SPH_ERR_OUTSIDE, B.periodic[a] ? "particle outside its box along a periodic axis"
                                                              : "particle outside a non-periodic box axis");
            }
            if(!(s.col[cH][i] > 0.0) || !std::isfinite(s.col[cH][i]))
                return fail(SPH_ERR_NONFINITE, "smoothing length must be positive and finite");
            if((s.roles & SPH_ROLE_SOURCE) && !(s.col[cM][i] > 0.0))
                return fail(SPH_ERR_NONFINITE, "source particle mass must be positive");
            if(p.cull == SPH_CULL_PAIR_MAX)
            {
                hmax[b] = std::max(hmax[b], s.col[cH][i]);
                hmin[b] = std::min(hmin[b], s.col[cH][i]);
            }

        }
    }
    boxDesc.assign(nbox, sph::BoxDev{});
    uint64_t cellBase = 0, activeBase = 0;
    anyTwoLevel = false;
    bool const dynamic = p.cull == SPH_CULL_PAIR_MAX;
    for(int32_t b = 0; b < nbox; ++b)
    {
        SphBox const& B = boxes[b];
        // The grid follows the largest h of the box (global cull: h0).  With the
        // pair-max cull it is re-derived every step from the current h, within an
        // allocation that admits h shrinking by half on every axis.
        double const hgrid = hmax[b];
        if(dynamic && p.h_max > 0.0 && p.h_max < hmax[b])
            return fail(SPH_ERR_INVALID, "an input h exceeds params.h_max");
        // Boxes whose h spans a factor of 1.6 or more also allocate level-1 cells
        // (m0 x m1 x m2 per level-0 cell, each m in 1..4) for the particles whose
        // cull radius fits a level-1 edge; the grid update decides each step
        // whether they are used and how finely, with the level-0 edge covering
        // both the largest radius and twice the smallest.
        bool const two = dynamic && hmin[b] < 1e300
                         && 2.0 * cellRadius(sup, hmin[b]) <= sph::kTwoLevelSlack * cellRadius(sup, hgrid);
        double const rc = two ? std::max(cellRadius(sup, hgrid), 2.0 * cellRadius(sup, hmin[b])) : cellRadius(sup, hgrid);
        double const rAlloc = cellRadius(sup, hgrid);
        sph::BoxDev& d = boxDesc[b];
        uint64_t cells = 1, cellsMax = 1;
        // adaptive h is capped by h_max, else by what the periodic axes admit
        double hcap = p.h_max > 0.0 ? p.h_max : 1e300;
        for(int a = 0; a < 3; ++a)
        {
            d.lo[a] = B.lo[a];
            d.L[a] = B.hi[a] - B.lo[a];
            if(!(d.L[a] > 0.0))
                return fail(SPH_ERR_INVALID, "box with non-positive extent");
            d.periodic[a] = B.periodic[a] ? 1 : 0;
            double const nd = std::floor(d.L[a] / rc);
            d.n[a] = nd < 1.0 ? 1 : (nd > 1.0e6 ? 1000000 : int32_t(nd));
            double const ndMax = dynamic ? std::floor(d.L[a] / (0.5 * rAlloc)) : nd;
            d.nMax[a] = std::max(d.n[a], ndMax < 1.0 ? 1 : (ndMax > 1.0e6 ? 1000000 : int32_t(ndMax)));
            d.edge[a] = d.L[a] / d.n[a];
            d.edgef[a] = float(d.edge[a]);
            if(d.periodic[a] && d.L[a] < rAlloc)
                return fail(SPH_ERR_UNSUPPORTED, "periodic box thinner than the interaction radius");
            if(d.periodic[a] && p.h_max <= 0.0 && (p.physics & SPH_PHYS_ADAPTIVE_H))
            {
                double lim = d.L[a] / (double(sup) * (1.0 + 1.0 / 262144.0));
                while(lim > hmax[b] && cellRadius(sup, lim) > d.L[a])
                    lim = std::nextafter(lim, 0.0);
                hcap = std::min(hcap, std::max(lim, hmax[b]));
            }
            cells *= uint64_t(d.n[a]);
            cellsMax *= uint64_t(d.nMax[a]);
        }
        // Level-1 cells: up to 2 x 2 x 2 per allocated level-0 cell.  The grid
        // update chooses the splits each step; until it runs the box has one level.
        d.levelsAlloc = two ? 2 : 1;
        uint64_t const perCell = two ? 8 : 0;
        d.cells1Alloc = uint32_t(perCell * cellsMax);
        d.levels = 1;
        d.m[0] = d.m[1] = d.m[2] = 1;
        d.msub = 1;
        d.e1 = 0.0;
        d.cellBase = uint32_t(cellBase);
        d.ncells = uint32_t(cells);
        d.ncellsMax = uint32_t(cellsMax);
        d.nItems = uint32_t(cells);
        d.activeBase = uint32_t(activeBase);
        d.hcap = hcap;
        cellBase += cellsMax + perCell * cellsMax;
        anyTwoLevel = anyTwoLevel || two;
        activeBase += d.nItems;
        if(cellBase * 2 + 1 >= (1ull << 32))
            return fail(SPH_ERR_UNSUPPORTED, "too many cells (2^31)");
    }
    activeCells = uint32_t(activeBase);
    ncells = uint32_t(cellBase);
    return SPH_OK;
}

int sph_ctx::allocate()
{
    release();
    physArgs();
    uint32_t const nbox = uint32_t(boxDesc.size());
    dc.n = n;
    dc.nbox = nbox;
    dc.support = supportOf(p.kernel);
    int st = SPH_OK;
    if((st = alloc(dc.boxes, nbox)) || (st = alloc(dc.shift32, size_t(nbox) * 32))
       || (st = alloc(dc.shift64, size_t(nbox) * 32)) || (st = allocMaster(dc.cur)) || (st = allocMaster(dc.alt)))
        return st;
    for(int a = 0; a < 3 && !st; ++a)
        st = alloc(dc.d.dvdt[a], n);
    for(int a = 0; a < 3 && !st; ++a)
        st = alloc(dc.d.dBdt[a], n);
    if(st || (st = alloc(dc.d.dudt, n)) || (st = alloc(dc.d.dpsidt, n)) || (st = alloc(dc.d.divB, n)))
        return st;
    if(p.precision == SPH_PREC_FP64)
    {
        if((st = alloc(dc.r64.pm, n)) || (st = alloc(dc.r64.hc, n)) || (st = alloc(dc.r64.fv, n))
           || (st = alloc(dc.r64.ft, n)) || (st = alloc(dc.r64.fb, n)))
            return st;
    }
    else
    {
        if((st = alloc(dc.r32.pm, n)) || (st = alloc(dc.r32.hc, n)) || (st = alloc(dc.r32.fv, n))
           || (st = alloc(dc.r32.ft, n)) || (st = alloc(dc.r32.fb, n)))
            return st;
    }
    dc.cells.ncells = ncells;
    if((st = alloc(dc.cells.start, ncells)) || (st = alloc(dc.cells.mid, ncells)) || (st = alloc(dc.cells.end, ncells))
       || (st = alloc(dc.cells.bstart, ncells)) || (st = alloc(dc.cells.bend, ncells)))
        return st;
    if((st = alloc(dc.keysA, n)) || (st = alloc(dc.valsA, n)) || (st = alloc(dc.keysB, n)) || (st = alloc(dc.valsB, n))
       || (st = alloc(dc.sortScratch, sph::radixScratchWords(n))))
        return st;
    if((st = alloc(dc.status, sph::kStatWords)) || (st = alloc(dc.scal, 1)) || (st = alloc(dc.diag, sph::kDiagWords))
       || (st = alloc(dc.work, 1)) || (st = alloc(dc.kickDone, 1)))
        return st;
    SPH_CUDA_TRY(cudaMemsetAsync(dc.kickDone, 0, sizeof(uint32_t), stream));
    if((st = alloc(dc.bs.dt, nbox)) || (st = alloc(dc.bs.time, nbox)) || (st = alloc(dc.bs.lastDt, nbox))
       || (st = alloc(dc.bs.dtBits, nbox)) || (st = alloc(dc.bs.chBits, nbox)) || (st = alloc(dc.bs.hmaxBits, nbox))
       || (st = alloc(dc.bs.hminBits, nbox)) || (st = alloc(dc.activeTotal, 1)))
        return st;
    dc.nPartialBlocks = sph::partialBlocks(n);
    if((st = alloc(dc.partials, size_t(dc.nPartialBlocks) * sph::kDiagWords))
       || (st = alloc(boxOut, size_t(nbox) * sph::kDiagWords))
       || (st = alloc(boxScratch, sph::boxReduceScratchDoubles(nbox))) || (st = alloc(dc.lists.count, n)))
        return st;
    SPH_CUDA_TRY(cudaMemsetAsync(dc.diag, 0, sizeof(double) * sph::kDiagWords, stream));
    dc.keyBits = 1;
    while((uint64_t(1) << dc.keyBits) <= uint64_t(ncells) * 2)
        ++dc.keyBits;
    dc.lists.cap = 0;
    dc.lists.list = nullptr;
    sph::configurePairKernels();
    allocN = n;
    allocCells = ncells;
    allocBoxes = nbox;
    allocated = true;
    return SPH_OK;
}

//! Host mirror -> device state in input order (id[p] = p).
int sph_ctx::uploadMirror()
{
    std::vector<double> buf(n);
    for(int c = 0; c < kHostCols; ++c)
    {
        for(auto& s : sp)
            if(s.set)
                std::copy(s.col[c].begin(), s.col[c].end(), buf.begin() + s.offset);
        SPH_CUDA_TRY(cudaMemcpyAsync(masterCol(dc.cur, c), buf.data(), size_t(n) * 8, cudaMemcpyHostToDevice, stream));
        SPH_CUDA_TRY(cudaStreamSynchronize(stream));
    }
    std::vector<uint32_t> ids(n);
    std::vector<int32_t> bx(n);
    std::vector<uint8_t> roles(n);
    for(auto& s : sp)
        if(s.set)
            for(int64_t i = 0; i < s.n; ++i)
            {
                ids[s.offset + i] = uint32_t(s.offset + i);
                bx[s.offset + i] = s.box[i];
                roles[s.offset + i] = uint8_t(s.roles);
            }
    SPH_CUDA_TRY(cudaMemcpyAsync(dc.cur.id, ids.data(), size_t(n) * 4, cudaMemcpyHostToDevice, stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(dc.cur.box, bx.data(), size_t(n) * 4, cudaMemcpyHostToDevice, stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(dc.cur.role, roles.data(), size_t(n), cudaMemcpyHostToDevice, stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(
        dc.boxes,
        boxDesc.data(),
        sizeof(sph::BoxDev) * boxDesc.size(),
        cudaMemcpyHostToDevice,
        stream));
    std::vector<float4> sh32(boxDesc.size() * 32, float4{0.f, 0.f, 0.f, 0.f});
    std::vector<sph::D4> sh64(boxDesc.size() * 32, sph::D4{0.0, 0.0, 0.0, 0.0});
    for(size_t b = 0; b < boxDesc.size(); ++b)
        for(int sl = 0; sl < 27; ++sl)
        {
            sph::BoxDev const& d = boxDesc[b];
            int const o[3] = {sph::stencilOff(sl, 0), sph::stencilOff(sl, 1), sph::stencilOff(sl, 2)};
            sh32[b * 32 + sl] = float4{float(o[0]) * d.edgef[0], float(o[1]) * d.edgef[1], float(o[2]) * d.edgef[2], 0.f};
            sh64[b * 32 + sl] = sph::D4{double(o[0]) * d.edge[0], double(o[1]) * d.edge[1], double(o[2]) * d.edge[2], 0.0};
        }
    SPH_CUDA_TRY(cudaMemcpyAsync(dc.activeTotal, &activeCells, sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(dc.shift32, sh32.data(), sizeof(float4) * sh32.size(), cudaMemcpyHostToDevice, stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(dc.shift64, sh64.data(), sizeof(sph::D4) * sh64.size(), cudaMemcpyHostToDevice, stream));
    sph::StepScalars sc{};
    SPH_CUDA_TRY(cudaMemcpyAsync(dc.scal, &sc, sizeof(sc), cudaMemcpyHostToDevice, stream));
    std::vector<double> dts(boxDesc.size(), p.dt);
    SPH_CUDA_TRY(cudaMemcpyAsync(dc.bs.dt, dts.data(), 8 * dts.size(), cudaMemcpyHostToDevice, stream));
    SPH_CUDA_TRY(cudaMemsetAsync(dc.bs.time, 0, 8 * dts.size(), stream));
    SPH_CUDA_TRY(cudaMemsetAsync(dc.bs.lastDt, 0, 8 * dts.size(), stream));
    SPH_CUDA_TRY(cudaMemsetAsync(dc.bs.chBits, 0, 8 * dts.size(), stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(stream));
    mirrorStale = false;
    deviceCurrent = true;
    densityValid = false;
    forceValid = false;
    return SPH_OK;
}

//! Device state -> host mirror (input order), before a re-layout.
int sph_ctx::downloadMirror()
{
    int st = stagingCols(1);
    if(st)
        return st;
    for(auto& s : sp)
    {
        if(!s.set)
            continue;
        for(int c = 0; c < kHostCols; ++c)
        {
            sph::launchUnpermute(n, dc.cur.id, masterCol(dc.cur, c), staging[0], stream);
            SPH_CUDA_TRY(cudaMemcpyAsync(
                s.col[c].data(),
                staging[0] + s.offset,
                size_t(s.n) * 8,
                cudaMemcpyDeviceToHost,
                stream));
            SPH_CUDA_TRY(cudaStreamSynchronize(stream));
        }
    }
    mirrorStale = false;
    return SPH_OK;
}

int sph_ctx::probeListCapacity()
{
    uint32_t capN = uint32_t(p.max_neighbours);
    if(capN == 0)
    {
        int st = clearStatus();
        if(st || (st = build(false)))
            return st;
        sph::launchDensity(dc, pa, p.kernel, p.precision, true, densityVariant, stream);
        uint32_t stat[sph::kStatWords];
        SPH_CUDA_TRY(cudaMemcpyAsync(stat, dc.status, sizeof(stat), cudaMemcpyDeviceToHost, stream));
        SPH_CUDA_TRY(cudaStreamSynchronize(stream));
        capN = uint32_t(double(stat[sph::kStatMaxCount]) * 1.25) + 16;
    }
    return growLists(capN);
}

//! (Re)allocates the neighbour lists with room for `need` entries per target.
int sph_ctx::growLists(uint32_t need, bool bestEffort)
{
    uint32_t const capN = std::max<uint32_t>(32, (need + 7) & ~7u);
    SPH_CUDA_TRY(cudaStreamSynchronize(stream));
    uint32_t* list = nullptr;
    if(bestEffort)
    {
        // headroom only: the new rows are allocated beside the old ones, and a
        // context that cannot have them keeps the lists it has
        if(alloc(list, size_t(n) * capN) != SPH_OK)
        {
            cudaGetLastError();
            return SPH_OK;
        }
    }
    if(dc.lists.list)
    {
        auto it = std::find(allocs.begin(), allocs.end(), static_cast<void*>(dc.lists.list));
        if(it != allocs.end())
        {
            cudaFree(*it);
            allocs.erase(it);
        }
        dc.lists.list = nullptr;
    }
    if(!list)
    {
        int const st = alloc(list, size_t(n) * capN);
        if(st)
            return st;
    }
    dc.lists.list = list;
    dc.lists.cap = capN;
    dropGraphs();
    densityValid = false;
    forceValid = false;
    return SPH_OK;
}

int sph_ctx::ensureDevice()
{
    if(deviceCurrent)
        return SPH_OK;
    if(allocated && mirrorStale)
    {
        int st = downloadMirror();
        if(st)
            return st;
    }
    int st = layout();
    if(st)
        return st;
    bool const fresh = !allocated || n != allocN || ncells != allocCells || boxDesc.size() != allocBoxes;
    if(fresh && (st = allocate()))
        return st;
    physArgs();
    if((st = uploadMirror()))
        return st;
    if(fresh && (st = probeListCapacity()))
        return st;
    return SPH_OK;
}

//! Drift (optional) + cell keys + sort + cell ranges + permute/pack.
int sph_ctx::build(bool drift)
{
    sph::NvtxRange const range(drift ? "drift + cell sort" : "cell sort");
    SPH_CUDA_TRY(cudaMemsetAsync(&dc.scal->pairs, 0, sizeof(unsigned long long), stream));
    SPH_CUDA_TRY(cudaMemsetAsync(&dc.scal->candidates, 0, sizeof(unsigned long long), stream));
    SPH_CUDA_TRY(cudaMemsetAsync(dc.bs.chBits, 0, sizeof(unsigned long long) * dc.nbox, stream));
    if(p.cull == SPH_CULL_PAIR_MAX)
        sph::launchGridUpdate(dc, supportOf(p.kernel), stream);
    sph::launchDriftKeys(dc, drift, stream);
    bool const inB = sph::radixSortPairs(dc.keysA, dc.valsA, dc.keysB, dc.valsB, n, dc.keyBits, dc.sortScratch, stream);
    uint32_t const* keys = inB ? dc.keysB : dc.keysA;
    uint32_t const* perm = inB ? dc.valsB : dc.valsA;
    sph::launchCellRanges(dc, keys, stream);
    if(anyTwoLevel)
        sph::launchSubBlocks(dc, ncells, stream);
    sph::launchPermute(dc, perm, pa, p.precision, stream);
    std::swap(dc.cur, dc.alt);
    parity ^= 1;
    return SPH_OK;
}

int sph_ctx::densityPass()
{
    sph::NvtxRange const range("density pass");
    SPH_CUDA_TRY(cudaMemsetAsync(dc.lists.count, 0xff, size_t(n) * 4, stream));
    sph::launchDensity(dc, pa, p.kernel, p.precision, false, densityVariant, stream);
    return SPH_OK;
}

int sph_ctx::forcePass()
{
    sph::NvtxRange const range("force pass");
    SPH_CUDA_TRY(cudaMemsetAsync(dc.bs.dtBits, 0x7f, sizeof(unsigned long long) * dc.nbox, stream));
    sph::launchForce(dc, pa, p.kernel, p.precision, forceVariant, stream);
    return SPH_OK;
}

//! Zeroes the status words once per call: non-finite and escaped particles,
//! list overflow and the largest neighbour count then accumulate over every
//! step of the call, so a condition raised by any step is reported.
int sph_ctx::clearStatus()
{
    SPH_CUDA_TRY(cudaMemsetAsync(dc.status, 0, sizeof(uint32_t) * sph::kStatWords, stream));
    return SPH_OK;
}

//! Saves (restore = false) or restores (restore = true) the state a step call
//! starts from: every master column of the current buffer, the per-box clock
//! and CFL/Dedner words, and the step scalars.  The snapshot is allocated on
//! the first step call and freed with the context.
int sph_ctx::snapshot(bool restore)
{
    uint32_t const nb = dc.nbox;
    if(!haveSnap)
    {
        if(restore)
            return fail(SPH_ERR_STATE, "no step snapshot to restore");
        int st = allocMaster(snap);
        if(st || (st = alloc(snapBs.dt, nb)) || (st = alloc(snapBs.time, nb)) || (st = alloc(snapBs.lastDt, nb))
           || (st = alloc(snapBs.dtBits, nb)) || (st = alloc(snapBs.chBits, nb)) || (st = alloc(snapScal, 1)))
            return st;
        haveSnap = true;
    }
    sph::Master const& from = restore ? snap : dc.cur;
    sph::Master const& to = restore ? dc.cur : snap;
    sph::BoxScalars const& bf = restore ? snapBs : dc.bs;
    sph::BoxScalars const& bt = restore ? dc.bs : snapBs;
    sph::launchCopyMaster(to, from, n, stream);
    auto const d2d = cudaMemcpyDeviceToDevice;
    SPH_CUDA_TRY(cudaMemcpyAsync(bt.dt, bf.dt, 8 * size_t(nb), d2d, stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(bt.time, bf.time, 8 * size_t(nb), d2d, stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(bt.lastDt, bf.lastDt, 8 * size_t(nb), d2d, stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(bt.dtBits, bf.dtBits, 8 * size_t(nb), d2d, stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(bt.chBits, bf.chBits, 8 * size_t(nb), d2d, stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(
        restore ? dc.scal : snapScal,
        restore ? snapScal : dc.scal,
        sizeof(sph::StepScalars),
        d2d,
        stream));
    return SPH_OK;
}

//! Waits for everything queued on the context's stream.  Inside a public call
//! that honours the limit (sph_step, sph_density, sph_hydro, sph_mhd, sph_wait
//! and the completion of a pending call), the wait polls an event against the
//! deadline instead of blocking, and returns SPH_ERR_TIMEOUT when it passes
//! (the work keeps running; nothing is cancelled).
int sph_ctx::waitStream(char const* where)
{
    if(!boundedWait || !(waitLimit > 0.0))
    {
        SPH_CUDA_TRY(cudaStreamSynchronize(stream));
        return SPH_OK;
    }
    if(!eWait)
        SPH_CUDA_TRY(cudaEventCreateWithFlags(&eWait, cudaEventDisableTiming));
    SPH_CUDA_TRY(cudaEventRecord(eWait, stream));
    auto const t0 = std::chrono::steady_clock::now();
    std::chrono::microseconds nap(10);
    for(;;)
    {
        cudaError_t const q = cudaEventQuery(eWait);
        if(q == cudaSuccess)
        {
            // a "not ready" answer of the poll is not an error of this call
            if(cudaPeekAtLastError() == cudaErrorNotReady)
                cudaGetLastError();
            return SPH_OK;
        }
        if(q != cudaErrorNotReady)
            return fail(SPH_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(q));
        double const el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if(el >= waitLimit)
        {
            if(cudaPeekAtLastError() == cudaErrorNotReady)
                cudaGetLastError();
            return fail(
                SPH_ERR_TIMEOUT,
                std::string(where) + ": the device work did not finish within " + std::to_string(waitLimit)
                    + " s; it keeps running, and sph_wait (or the next call on this context) completes the call");
        }
        std::this_thread::sleep_for(nap);
        nap = std::min(nap * 2, std::chrono::microseconds(1000));
    }
}

int sph_ctx::checkStatus(char const* where)
{
    int const w = waitStream(where);
    if(w)
        return w;
    SPH_CUDA_TRY(cudaMemcpyAsync(lastStat, dc.status, sizeof(lastStat), cudaMemcpyDeviceToHost, stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(stream));
    SPH_CUDA_TRY(cudaGetLastError());
    return evalStatus(where);
}

//! The status words of lastStat as a status code (and error message).
int sph_ctx::evalStatus(char const* where)
{
    uint32_t const* const stat = lastStat;
    if(stat[sph::kStatNonFinite])
        return fail(
            SPH_ERR_NONFINITE,
            std::string(where) + ": " + std::to_string(stat[sph::kStatNonFinite]) + " particles with non-finite positions");
    if(stat[sph::kStatOutside])
        return fail(
            SPH_ERR_OUTSIDE,
            std::string(where) + ": " + std::to_string(stat[sph::kStatOutside])
                + " particles outside their box (a non-periodic axis, or a periodic one they were not wrapped on)");
    if(stat[sph::kStatCheck])
    {
        char bits[16];
        std::snprintf(bits, sizeof(bits), "0x%x", stat[sph::kStatCheck]);
        return fail(
            SPH_ERR_STATE,
            std::string(where) + ": a device bounds check failed (sites " + bits
                + "; the access was skipped and the results are not valid)");
    }
    if(stat[sph::kStatOverflow])
        return fail(
            SPH_ERR_OVERFLOW,
            std::string(where) + ": a neighbour list needed " + std::to_string(stat[sph::kStatOverflow])
                + " entries, capacity " + std::to_string(dc.lists.cap));
    return SPH_OK;
}

//! One runOneStep; ev (5 events or null) brackets build / density / force / kick.
//! Under stream capture the events are recorded as external events, so they
//! become event-record nodes of the graph (retargeted before each replay).
int sph_ctx::stepOnce(cudaEvent_t const* ev, bool capture)
{
    auto recordStage = [&](cudaEvent_t e, bool cap)
    {
        return cap ? cudaEventRecordWithFlags(e, stream, cudaEventRecordExternal) : cudaEventRecord(e, stream);
    };
    int st;
    if(ev)
        SPH_CUDA_TRY(recordStage(ev[0], capture));
    if((st = build(true)))
        return st;
    if(ev)
        SPH_CUDA_TRY(recordStage(ev[1], capture));
    if((st = densityPass()))
        return st;
    if(ev)
        SPH_CUDA_TRY(recordStage(ev[2], capture));
    if((st = forcePass()))
        return st;
    if(ev)
        SPH_CUDA_TRY(recordStage(ev[3], capture));
    {
        sph::NvtxRange const range("kick + reductions");
        sph::launchKick(dc, pa, (p.physics & SPH_PHYS_CFL) != 0, stream);
    }
    if(ev)
        SPH_CUDA_TRY(recordStage(ev[4], capture));
    return SPH_OK;
}

//! n_steps of runOneStep.  The call is transactional with respect to the
//! neighbour-list capacity: the state it starts from is saved first, and if a
//! list overflowed in any step (steps run without host round trips, so this is
//! seen only at the end), the lists grow, the state is restored and the steps
//! run again.  timings[4] spans the whole call, replays included; the per-stage
//! times are those of the run that is kept.
int sph_ctx::steps(int32_t nsteps, double dt)
{
    int st = ensureDevice();
    if(st)
        return st;
    if(!eCall)
        SPH_CUDA_TRY(cudaEventCreate(&eCall));
    SPH_CUDA_TRY(cudaEventRecord(eCall, stream));
    if(dt > 0.0)
        sph::launchFill(dc.bs.dt, dc.nbox, dt, stream);
    if((st = snapshot(false)))
        return st;
    constexpr int kMaxReplays = 8;
    for(int attempt = 0;; ++attempt)
    {
        st = runSteps(nsteps);
        if(st == SPH_ERR_TIMEOUT)
        {
            pending = kPendStep;
            pendingSteps = nsteps;
            densityValid = forceValid = false;
            return st;
        }
        if(st == SPH_ERR_OVERFLOW && attempt == kMaxReplays)
        {
            // give up with the state the call started from
            int const rs = snapshot(true);
            if(rs)
                return rs;
            SPH_CUDA_TRY(cudaStreamSynchronize(stream));
            break;
        }
        if(st != SPH_ERR_OVERFLOW)
            break;
        ++replays;
        uint32_t stat[sph::kStatWords];
        SPH_CUDA_TRY(cudaMemcpy(stat, dc.status, sizeof(stat), cudaMemcpyDeviceToHost));
        int const g = growLists(uint32_t(double(stat[sph::kStatOverflow]) * 1.25) + 16);
        if(g)
            return g;
        if((st = snapshot(true)))
            return st;
    }
    float ms = 0.f;
    if(cudaEventElapsedTime(&ms, eCall, events[1]) == cudaSuccess)
        timings[4] = ms;
    densityValid = st == SPH_OK;
    forceValid = st == SPH_OK;
    // Headroom: a call whose largest list came within 10% of the capacity grows
    // the lists now (after its timed events), so slowly rising neighbour counts
    // do not make a later call overflow and run again.  The derivatives stay
    // valid; the lists of this state are gone, so the density pass is not.
    uint32_t const maxCount = lastStat[sph::kStatMaxCount];
    if(st == SPH_OK && uint64_t(maxCount) * 10 > uint64_t(dc.lists.cap) * 9)
    {
        int const g = growLists(uint32_t(double(maxCount) * 1.25) + 16, true);
        if(g)
            return g;
        forceValid = true;
    }
    return st;
}

//! Captures the two-step graph of the current buffer parity by running two
//! steps from a snapshot, then puts the state (particles, clocks, counters)
//! back: the next sph_step replays the graph from the state it would have
//! started from anyway.  List overflows during the capture steps regrow the
//! lists as in a step call.
int sph_ctx::prepareGraph()
{
    int st = ensureDevice();
    if(st || (st = snapshot(false)))
        return st;
    for(int attempt = 0; attempt < 8; ++attempt)
    {
        st = runSteps(2);
        int const rs = snapshot(true);
        if(rs)
            return rs;
        if(st != SPH_ERR_OVERFLOW)
            break;
        uint32_t stat[sph::kStatWords];
        SPH_CUDA_TRY(cudaMemcpy(stat, dc.status, sizeof(stat), cudaMemcpyDeviceToHost));
        if((st = growLists(uint32_t(double(stat[sph::kStatOverflow]) * 1.25) + 16)))
            return st;
    }
    densityValid = false;
    forceValid = false;
    return st;
}

//! Fills `tuning` with the current shapes.
void sph_ctx::describeTuning()
{
    tuning.density_variant = densityVariant;
    tuning.force_variant = forceVariant;
    sph::densityShape(p.precision, densityVariant, &tuning.staging_depth, &tuning.density_blocks_per_sm,
                      &tuning.cull_unroll);
    tuning.force_blocks_per_sm = sph::forceBlocksPerSm(p.precision, int(p.physics), forceVariant);
    tuning.n_density_variants = sph::densityVariants(p.precision);
    tuning.n_force_variants = sph::forceVariants(p.precision);
}

//! Times every density and force launch shape over stepsPerTrial eager steps
//! from the same saved state (restored after each trial, and at the end) and
//! keeps the fastest of each.  Density and force shapes are independent, so
//! each kernel's trials vary its own shape with the other at its default.
int sph_ctx::autotune(int32_t stepsPerTrial)
{
    if(stepsPerTrial < 1)
        return fail(SPH_ERR_INVALID, "sph_autotune: steps_per_trial must be >= 1");
    int st = ensureDevice();
    if(st || (st = snapshot(false)))
        return st;
    bool const graph = useGraph;
    useGraph = false;
    dropGraphs();
    int const nd = sph::densityVariants(p.precision), nf = sph::forceVariants(p.precision);
    tuning = SphTuning{};
    for(int k = 0; k < 8; ++k)
        tuning.density_ms[k] = tuning.force_ms[k] = 0.0;
    int const d0 = densityVariant, f0 = forceVariant;
    auto trial = [&](int dv, int fv, double& dms, double& fms) -> int
    {
        densityVariant = dv;
        forceVariant = fv;
        // one untimed step first (a kernel's first launch also loads its module)
        int r = runSteps(1);
        int const rs0 = snapshot(true);
        if(rs0)
            return rs0;
        if(r != SPH_OK && r != SPH_ERR_OVERFLOW)
            return r;
        r = SPH_ERR_OVERFLOW;
        for(int attempt = 0; attempt < 8 && r == SPH_ERR_OVERFLOW; ++attempt)
        {
            r = runSteps(stepsPerTrial);
            if(r == SPH_ERR_OVERFLOW)
            {
                uint32_t stat[sph::kStatWords];
                SPH_CUDA_TRY(cudaMemcpy(stat, dc.status, sizeof(stat), cudaMemcpyDeviceToHost));
                int const g = growLists(uint32_t(double(stat[sph::kStatOverflow]) * 1.25) + 16);
                if(g)
                    return g;
            }
            int const rs = snapshot(true);
            if(rs)
                return rs;
        }
        dms = timings[1] / stepsPerTrial;
        fms = timings[2] / stepsPerTrial;
        return r;
    };
    double unused = 0.0;
    int bestD = 0, bestF = 0;
    for(int v = 0; v < nd && !st; ++v)
    {
        st = trial(v, 0, tuning.density_ms[v], unused);
        if(!st && tuning.density_ms[v] < tuning.density_ms[bestD])
            bestD = v;
    }
    for(int v = 0; v < nf && !st; ++v)
    {
        st = trial(0, v, unused, tuning.force_ms[v]);
        if(!st && tuning.force_ms[v] < tuning.force_ms[bestF])
            bestF = v;
    }
    useGraph = graph;
    if(st)
    {
        densityVariant = d0;
        forceVariant = f0;
        return st;
    }
    densityVariant = bestD;
    forceVariant = bestF;
    // the particles are back where they were; the derivatives are a trial's
    densityValid = false;
    forceValid = false;
    describeTuning();
    tuning.steps_per_trial = stepsPerTrial;
    return SPH_OK;
}

//! One attempt of a step call: the steps (pairs of them as CUDA graphs when
//! enabled), then the status check.
int sph_ctx::runSteps(int32_t nsteps)
{
    int st = clearStatus();
    if(st)
        return st;
    for(double& t : timings)
        t = 0.0;
    bool const graph = useGraph && nsteps >= 2;
    size_t const nev = size_t(nsteps) * 5 + 2;
    while(events.size() < nev)
    {
        cudaEvent_t e;
        SPH_CUDA_TRY(cudaEventCreate(&e));
        events.push_back(e);
    }
    cudaEvent_t const eBeg = events[0], eEnd = events[1];
    SPH_CUDA_TRY(cudaEventRecord(eBeg, stream));
    int32_t done = 0;
    if(graph)
    {
        while(nsteps - done >= 2)
        {
            cudaGraphExec_t& g = graphs[parity];
            if(!g)
            {
                cudaEvent_t* const gev = graphEv[parity];
                for(int k = 0; k < 10; ++k)
                    if(!gev[k])
                        SPH_CUDA_TRY(cudaEventCreate(&gev[k]));
                cudaGraph_t raw = nullptr;
                unsigned long long const before = sph::launchesSoFar();
                SPH_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
                int const s1 = stepOnce(gev, true);
                int const s2 = s1 ? s1 : stepOnce(gev + 5, true);
                cudaError_t const ce = cudaStreamEndCapture(stream, &raw);
                // the captured launches ran nothing yet: they count when the graph runs
                unsigned long long const recorded = sph::launchesSoFar() - before;
                sph::uncountLaunches(recorded);
                graphKernels[parity] = unsigned(recorded);
                if(s2)
                {
                    if(raw)
                        cudaGraphDestroy(raw);
                    return s2;
                }
                SPH_CUDA_TRY(ce);
                // find the event-record node of each captured stage event
                size_t nn = 0;
                SPH_CUDA_TRY(cudaGraphGetNodes(raw, nullptr, &nn));
                std::vector<cudaGraphNode_t> nodes(nn);
                SPH_CUDA_TRY(cudaGraphGetNodes(raw, nodes.data(), &nn));
                int found = 0;
                for(cudaGraphNode_t nd : nodes)
                {
                    cudaGraphNodeType ty;
                    SPH_CUDA_TRY(cudaGraphNodeGetType(nd, &ty));
                    if(ty != cudaGraphNodeTypeEventRecord)
                        continue;
                    cudaEvent_t ev = nullptr;
                    SPH_CUDA_TRY(cudaGraphEventRecordNodeGetEvent(nd, &ev));
                    for(int k = 0; k < 10; ++k)
                        if(ev == gev[k])
                        {
                            graphEvNode[parity][k] = nd;
                            ++found;
                        }
                }
                cudaError_t const ie = cudaGraphInstantiate(&g, raw, 0);
                if(ie != cudaSuccess || found != 10)
                {
                    cudaGraphDestroy(raw);
                    if(ie == cudaSuccess)
                    {
                        cudaGraphExecDestroy(g);
                        g = nullptr;
                    }
                    SPH_CUDA_TRY(ie);
                    return fail(SPH_ERR_CUDA, "sph_step: captured graph lacks its stage events");
                }
                graphRaw[parity] = raw;
            }
            // this replay's stage events
            for(int i = 0; i < 2; ++i)
                for(int k = 0; k < 5; ++k)
                    SPH_CUDA_TRY(cudaGraphExecEventRecordNodeSetEvent(
                        g, graphEvNode[parity][i * 5 + k], events[2 + size_t(done + i) * 5 + k]));
            SPH_CUDA_TRY(cudaGraphLaunch(g, stream));
            sph::countLaunches(graphKernels[parity]);
            done += 2;
        }
    }
    for(; done < nsteps; ++done)
        if((st = stepOnce(&events[2 + size_t(done) * 5])))
            return st;
    SPH_CUDA_TRY(cudaEventRecord(eEnd, stream));
    st = checkStatus("sph_step");
    if(st != SPH_ERR_TIMEOUT)
        collectTimings(nsteps);
    return st;
}

//! Per-stage and whole-run times of the last runSteps (its events have completed).
void sph_ctx::collectTimings(int32_t nsteps)
{
    float ms = 0.f;
    for(double& t : timings)
        t = 0.0;
    cudaEventElapsedTime(&ms, events[0], events[1]);
    timings[4] = ms;
    for(int32_t s = 0; s < nsteps; ++s)
        for(int k = 0; k < 4; ++k)
        {
            cudaEventElapsedTime(&ms, events[2 + size_t(s) * 5 + k], events[2 + size_t(s) * 5 + k + 1]);
            timings[k] += ms;
        }
}

//! Completes a call that returned SPH_ERR_TIMEOUT: waits (bounded) for its
//! work, then runs the checks it skipped.  A step call whose checks fail is
//! rolled back to the state it started from (its lists grown after an
//! overflow) and returns their status; a density call that overflowed grows
//! the lists.  Returns SPH_ERR_TIMEOUT while the work is still running.
int sph_ctx::completePending()
{
    if(pending == kPendNone)
        return SPH_OK;
    SPH_CUDA_TRY(cudaSetDevice(p.device));
    bool const bw = boundedWait;
    boundedWait = true;
    char const* const where = pending == kPendStep ? "sph_step" : (pending == kPendDensity ? "sph_density" : "sph_hydro");
    int st = checkStatus(where);
    boundedWait = bw;
    if(st == SPH_ERR_TIMEOUT)
        return st;
    int const kind = pending;
    pending = kPendNone;
    if(st == SPH_ERR_OVERFLOW && kind != kPendForce)
    {
        int const g = growLists(uint32_t(double(lastStat[sph::kStatOverflow]) * 1.25) + 16);
        if(g)
            return g;
        st = fail(SPH_ERR_OVERFLOW,
                  std::string(where) + ": a neighbour list overflowed; the lists have grown, run the call again");
    }
    if(kind == kPendStep)
    {
        if(st == SPH_OK)
        {
            collectTimings(pendingSteps);
            float ms = 0.f;
            if(eCall && cudaEventElapsedTime(&ms, eCall, events[1]) == cudaSuccess)
                timings[4] = ms;
            densityValid = forceValid = true;
            return SPH_OK;
        }
        // the call's checks failed: back to the state it started from
        int const rs = snapshot(true);
        if(rs)
            return rs;
        SPH_CUDA_TRY(cudaStreamSynchronize(stream));
        densityValid = forceValid = false;
        return st;
    }
    if(kind == kPendDensity)
    {
        densityValid = st == SPH_OK;
        forceValid = false;
        return st;
    }
    forceValid = st == SPH_OK;
    return st;
}

//! Species of unchanged size on an allocated context: caller columns -> staging
//! (input order) -> gather into the sorted state by particle id.
int sph_ctx::setSpeciesFast(int32_t id, SphSoAView const* v)
{
    HostSpecies& s = sp[id];
    int st = stagingCols(kHostCols);
    if(st || (st = ensureCopyStream()))
        return st;
    // h and source masses are checked on the device as they are gathered
    SPH_CUDA_TRY(cudaMemsetAsync(dc.status + sph::kStatBadInput, 0, sizeof(uint32_t), stream));
    // Column c's copy (copy stream) hands over to its gather (context stream)
    // through eCopy, so copy c + 1 runs under gather c.  The copies start after
    // everything already queued on the context's stream.
    SPH_CUDA_TRY(cudaEventRecord(eCompute, stream));
    SPH_CUDA_TRY(cudaStreamWaitEvent(copyStream, eCompute, 0));
    for(int c = 0; c < kHostCols; ++c)
    {
        double const* src = viewCol(v, c);
        double* stage = staging[c];
        if(src)
        {
            SPH_CUDA_TRY(
                cudaMemcpyAsync(stage + s.offset, src, size_t(s.n) * 8, cudaMemcpyHostToDevice, copyStream));
            SPH_CUDA_TRY(cudaEventRecord(eCopy, copyStream));
            SPH_CUDA_TRY(cudaStreamWaitEvent(stream, eCopy, 0));
        }
        bool const mustBePositive = c == cH || (c == cM && (s.roles & SPH_ROLE_SOURCE));
        sph::launchGatherSpecies(
            n,
            dc.cur.id,
            s.offset,
            uint32_t(s.n),
            src ? stage : nullptr,
            colDefault(c),
            masterCol(dc.cur, c),
            mustBePositive ? dc.status + sph::kStatBadInput : nullptr,
            stream);
    }
    if(v && v->box_id)
    {
        for(int64_t i = 0; i < s.n; ++i)
            if(v->box_id[i] < 0 || uint32_t(v->box_id[i]) >= allocBoxes)
                return fail(SPH_ERR_INVALID, "box_id out of range");
        int32_t* stage = reinterpret_cast<int32_t*>(staging[0]);
        SPH_CUDA_TRY(cudaStreamSynchronize(stream));
        SPH_CUDA_TRY(cudaMemcpyAsync(stage + s.offset, v->box_id, size_t(s.n) * 4, cudaMemcpyHostToDevice, stream));
        sph::launchGatherSpeciesInt(n, dc.cur.id, s.offset, uint32_t(s.n), stage, dc.cur.box, stream);
    }
    uint32_t bad = 0;
    SPH_CUDA_TRY(cudaMemcpyAsync(&bad, dc.status + sph::kStatBadInput, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(stream));
    mirrorStale = true;
    if(bad)
        return fail(
            SPH_ERR_NONFINITE,
            std::to_string(bad)
                + " smoothing lengths or source masses are not positive and finite; the species holds them until it "
                  "is set again");
    densityValid = false;
    forceValid = false;
    return SPH_OK;
}

// ============================================================== C ABI
namespace
{
    //! Device buffers of one sph_init_lattice call, freed on every exit.
    struct InitScratch
    {
        std::vector<void*> ptrs;
        ~InitScratch()
        {
            for(void* p : ptrs)
                cudaFree(p);
        }
        template<typename T>
        cudaError_t take(T*& out, size_t count)
        {
            void* p = nullptr;
            if(sph::allocRefused())
                return cudaErrorMemoryAllocation;
            cudaError_t const e = cudaMalloc(&p, (count ? count : 1) * sizeof(T));
            if(e == cudaSuccess)
                ptrs.push_back(p);
            out = static_cast<T*>(p);
            return e;
        }
    };
} // namespace

namespace
{
    //! Marks a public compute call whose waits honour the context's limit.
    struct BoundedCall
    {
        sph_ctx* c;
        explicit BoundedCall(sph_ctx* ctx) : c(ctx)
        {
            c->boundedWait = true;
        }
        ~BoundedCall()
        {
            c->boundedWait = false;
        }
    };
} // namespace

//! Every public call that touches a context's device state first completes a
//! call of that context that returned SPH_ERR_TIMEOUT (see sph_wait).
#define SPH_COMPLETE_PENDING(ctx)                                                                                      \
    do                                                                                                                 \
    {                                                                                                                  \
        int const pst_ = (ctx)->completePending();                                                                     \
        if(pst_)                                                                                                       \
            return pst_;                                                                                               \
    } while(0)

extern "C" {

int sph_default_params(SphParams* p)
{
    if(!p)
        return fail(SPH_ERR_INVALID, "null params");
    *p = SphParams{};
    p->kernel = SPH_KERNEL_CUBIC;
    p->precision = SPH_PREC_FP32_COMP;
    p->cull = SPH_CULL_GLOBAL;
    p->physics = 0;
    p->gamma = 5.0 / 3.0;
    p->h0 = 0.05;
    p->dt = 0.01;
    p->alpha = 1.0;
    p->beta = 2.0;
    p->av_eps = 0.01;
    p->cfl = 0.3;
    p->cfl_force = 0.25;
    p->dedner_sigma = 1.0;
    p->mu0 = 1.0;
    p->max_neighbours = 0;
    p->device = 0;
    return SPH_OK;
}

int sph_create(SphParams const* params, sph_ctx** out)
{
    if(!params || !out)
        return fail(SPH_ERR_INVALID, "null argument");
    *out = nullptr;
    int st = validateParams(*params);
    if(st)
        return st;
    SPH_CUDA_TRY(cudaSetDevice(params->device));
    sph_ctx* c = new(std::nothrow) sph_ctx();
    if(!c)
        return fail(SPH_ERR_NOMEM, "host allocation failed");
    c->p = *params;
    cudaError_t const e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if(e != cudaSuccess)
    {
        delete c;
        return fail(SPH_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    }
    *out = c;
    return SPH_OK;
}

int sph_destroy(sph_ctx* ctx)
{
    if(!ctx)
        return fail(SPH_ERR_INVALID, "null context");
    cudaSetDevice(ctx->p.device);
    delete ctx;
    return SPH_OK;
}

int sph_set_boxes(sph_ctx* ctx, int32_t nbox, SphBox const* boxes)
{
    if(!ctx || nbox < 1 || !boxes)
        return fail(SPH_ERR_INVALID, "sph_set_boxes: bad arguments");
    SPH_COMPLETE_PENDING(ctx);
    for(int32_t b = 0; b < nbox; ++b)
        for(int a = 0; a < 3; ++a)
            if(!(boxes[b].hi[a] > boxes[b].lo[a]) || !std::isfinite(boxes[b].lo[a]) || !std::isfinite(boxes[b].hi[a]))
                return fail(SPH_ERR_INVALID, "sph_set_boxes: empty or non-finite box");
    SPH_CUDA_TRY(cudaSetDevice(ctx->p.device));
    if(ctx->allocated && ctx->mirrorStale)
    {
        int st = ctx->downloadMirror();
        if(st)
            return st;
    }
    ctx->boxes.assign(boxes, boxes + nbox);
    ctx->deviceCurrent = false;
    return SPH_OK;
}

int sph_set_species(sph_ctx* ctx, int32_t species_id, uint32_t roles, int64_t n, SphSoAView const* v)
{
    if(!ctx || species_id < 0 || species_id >= SPH_NUM_SPECIES || n < 0 || (n > 0 && !v))
        return fail(SPH_ERR_INVALID, "sph_set_species: bad arguments");
    SPH_COMPLETE_PENDING(ctx);
    if(n > 0 && (!v->pos[0] || !v->pos[1] || !v->pos[2]))
        return fail(SPH_ERR_INVALID, "sph_set_species: positions are required");
    if((roles & SPH_ROLE_SOURCE) && n > 0 && !v->mass)
        return fail(SPH_ERR_INVALID, "sph_set_species: source species need masses");
    SPH_CUDA_TRY(cudaSetDevice(ctx->p.device));
    HostSpecies& s = ctx->sp[species_id];
    s.declared = true;
    if(ctx->allocated && ctx->deviceCurrent && s.set && s.n == n && s.roles == roles)
        return ctx->setSpeciesFast(species_id, v);
    if(ctx->allocated && ctx->mirrorStale)
    {
        int st = ctx->downloadMirror();
        if(st)
            return st;
    }
    s.set = n > 0;
    s.roles = roles;
    s.n = n;
    for(int c = 0; c < kHostCols; ++c)
    {
        double const* src = viewCol(v, c);
        s.col[c].assign(size_t(n), ctx->colDefault(c));
        if(src)
            std::copy(src, src + n, s.col[c].begin());
    }
    s.box.assign(size_t(n), 0);
    if(v && v->box_id)
        std::copy(v->box_id, v->box_id + n, s.box.begin());
    ctx->deviceCurrent = false;
    return SPH_OK;
}

int sph_density(sph_ctx* ctx)
{
    if(!ctx)
        return fail(SPH_ERR_INVALID, "null context");
    SPH_COMPLETE_PENDING(ctx);
    if(ctx->empty())
        return SPH_OK;
    SPH_CUDA_TRY(cudaSetDevice(ctx->p.device));
    BoundedCall const bounded(ctx);
    int st = ctx->ensureDevice();
    if(st || (st = ctx->clearStatus()) || (st = ctx->build(false)) || (st = ctx->densityPass()))
        return st;
    st = ctx->checkStatus("sph_density");
    if(st == SPH_ERR_TIMEOUT)
    {
        ctx->pending = sph_ctx::kPendDensity;
        ctx->densityValid = ctx->forceValid = false;
        return st;
    }
    if(st == SPH_ERR_OVERFLOW)
    {
        uint32_t stat[sph::kStatWords];
        SPH_CUDA_TRY(cudaMemcpy(stat, ctx->dc.status, sizeof(stat), cudaMemcpyDeviceToHost));
        if((st = ctx->growLists(uint32_t(double(stat[sph::kStatOverflow]) * 1.25) + 16)))
            return st;
        SPH_CUDA_TRY(cudaMemsetAsync(ctx->dc.status, 0, sizeof(uint32_t) * sph::kStatWords, ctx->stream));
        SPH_CUDA_TRY(cudaMemsetAsync(&ctx->dc.scal->pairs, 0, sizeof(unsigned long long), ctx->stream));
        SPH_CUDA_TRY(cudaMemsetAsync(&ctx->dc.scal->candidates, 0, sizeof(unsigned long long), ctx->stream));
        SPH_CUDA_TRY(cudaMemsetAsync(ctx->dc.bs.chBits, 0, sizeof(unsigned long long) * ctx->dc.nbox, ctx->stream));
        if((st = ctx->densityPass()) || (st = ctx->checkStatus("sph_density")))
        {
            if(st == SPH_ERR_TIMEOUT)
            {
                ctx->pending = sph_ctx::kPendDensity;
                ctx->densityValid = ctx->forceValid = false;
            }
            return st;
        }
    }
    else if(st)
        return st;
    ctx->densityValid = true;
    ctx->forceValid = false;
    return SPH_OK;
}

int sph_hydro(sph_ctx* ctx)
{
    if(!ctx)
        return fail(SPH_ERR_INVALID, "null context");
    SPH_COMPLETE_PENDING(ctx);
    if(ctx->empty())
        return SPH_OK;
    if(!ctx->densityValid)
        return fail(SPH_ERR_STATE, "sph_hydro needs the density of the current state (call sph_density first)");
    SPH_CUDA_TRY(cudaSetDevice(ctx->p.device));
    BoundedCall const bounded(ctx);
    int st = ctx->forcePass();
    if(st || (st = ctx->checkStatus("sph_hydro")))
    {
        if(st == SPH_ERR_TIMEOUT)
        {
            ctx->pending = sph_ctx::kPendForce;
            ctx->forceValid = false;
        }
        return st;
    }
    ctx->forceValid = true;
    return SPH_OK;
}

int sph_mhd(sph_ctx* ctx)
{
    if(!ctx)
        return fail(SPH_ERR_INVALID, "null context");
    if(!(ctx->p.physics & SPH_PHYS_MHD))
        return fail(SPH_ERR_STATE, "sph_mhd needs SPH_PHYS_MHD in the context's params");
    return sph_hydro(ctx);
}

int sph_step(sph_ctx* ctx, int32_t n_steps, double dt)
{
    if(!ctx || n_steps < 0 || !std::isfinite(dt))
        return fail(SPH_ERR_INVALID, "sph_step: bad arguments");
    SPH_COMPLETE_PENDING(ctx);
    if(ctx->empty())
    {
        ctx->emptySteps += n_steps;
        ctx->emptyTime += double(n_steps) * (dt > 0.0 ? dt : ctx->p.dt);
        return SPH_OK;
    }
    SPH_CUDA_TRY(cudaSetDevice(ctx->p.device));
    BoundedCall const bounded(ctx);
    sph::NvtxRange const range("sph_step");
    return ctx->steps(n_steps, dt);
}

int sphx_box_grid(sph_ctx* ctx, int32_t box, double* out)
{
    if(!ctx || !out || box < 0 || uint32_t(box) >= ctx->dc.nbox || !ctx->allocated)
        return fail(SPH_ERR_INVALID, "sphx_box_grid: bad arguments");
    SPH_CUDA_TRY(cudaSetDevice(ctx->p.device));
    SPH_COMPLETE_PENDING(ctx);
    sph::BoxDev b{};
    SPH_CUDA_TRY(cudaMemcpyAsync(&b, ctx->dc.boxes + box, sizeof(b), cudaMemcpyDeviceToHost, ctx->stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for(int a = 0; a < 3; ++a)
    {
        out[a] = double(b.n[a]);
        out[3 + a] = b.edge[a];
        out[6 + a] = double(b.m[a]);
    }
    out[9] = double(b.levels);
    out[10] = b.e1;
    out[11] = b.hcap;
    return SPH_OK;
}

int sphx_get_pair_records(sph_ctx* ctx, int32_t species_id, float* pm)
{
    if(!ctx || !pm || species_id < 0 || species_id >= SPH_NUM_SPECIES || !ctx->allocated
       || ctx->p.precision != SPH_PREC_FP32_COMP)
        return fail(SPH_ERR_INVALID, "sphx_get_pair_records: bad arguments (FP32 contexts only)");
    SPH_CUDA_TRY(cudaSetDevice(ctx->p.device));
    SPH_COMPLETE_PENDING(ctx);
    HostSpecies const& s = ctx->sp[species_id];
    uint32_t const n = ctx->n;
    std::vector<float4> rec(n);
    std::vector<uint32_t> id(n);
    SPH_CUDA_TRY(cudaMemcpyAsync(rec.data(), ctx->dc.r32.pm, size_t(n) * sizeof(float4), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(id.data(), ctx->dc.cur.id, size_t(n) * 4, cudaMemcpyDeviceToHost, ctx->stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for(uint32_t p = 0; p < n; ++p)
    {
        int64_t const k = int64_t(id[p]) - s.offset;
        if(k < 0 || k >= s.n)
            continue;
        pm[4 * k + 0] = rec[p].x;
        pm[4 * k + 1] = rec[p].y;
        pm[4 * k + 2] = rec[p].z;
        pm[4 * k + 3] = rec[p].w;
    }
    return SPH_OK;
}

long long sphx_fail_alloc_after(long long after)
{
    return sph::g_allocFailAfter.exchange(after < 0 ? -1 : after);
}

int sph_set_wait_timeout(sph_ctx* ctx, double seconds)
{
    if(!ctx || !(seconds >= 0.0) || !std::isfinite(seconds))
        return fail(SPH_ERR_INVALID, "sph_set_wait_timeout: bad arguments");
    ctx->waitLimit = seconds;
    return SPH_OK;
}

int sph_wait(sph_ctx* ctx)
{
    if(!ctx)
        return fail(SPH_ERR_INVALID, "null context");
    return ctx->completePending();
}

int sph_get_species(sph_ctx* ctx, int32_t species_id, SphSoAView* v)
{
    if(!ctx || !v || species_id < 0 || species_id >= SPH_NUM_SPECIES)
        return fail(SPH_ERR_INVALID, "sph_get_species: bad arguments");
    SPH_COMPLETE_PENDING(ctx);
    HostSpecies const& s = ctx->sp[species_id];
    if(s.declared && s.n == 0)
        return SPH_OK; // nothing to copy
    if(!s.set)
        return fail(SPH_ERR_STATE, "sph_get_species: species not set");
    SPH_CUDA_TRY(cudaSetDevice(ctx->p.device));
    int st = ctx->ensureDevice();
    if(st)
        return st;
    sph::DevCtx& d = ctx->dc;
    // (device column, host destination) pairs; every column is unpermuted into
    // its own staging column, then all copies run back to back.
    std::vector<std::pair<double const*, double*>> cols;
    for(int a = 0; a < 3; ++a)
    {
        cols.push_back({d.cur.x[a], v->pos[a]});
        cols.push_back({d.cur.v[a], v->vel[a]});
        cols.push_back({d.cur.B[a], v->B[a]});
    }
    cols.push_back({d.cur.m, v->mass});
    cols.push_back({d.cur.h, v->h});
    cols.push_back({d.cur.rho, v->density});
    cols.push_back({d.cur.u, v->u});
    cols.push_back({d.cur.psi, v->psi});
    if(ctx->forceValid)
    {
        for(int a = 0; a < 3; ++a)
            cols.push_back({d.d.dvdt[a], v->dvdt[a]});
        cols.push_back({d.d.dudt, v->dudt});
        if(ctx->p.physics & SPH_PHYS_MHD)
        {
            for(int a = 0; a < 3; ++a)
                cols.push_back({d.d.dBdt[a], v->dBdt[a]});
            cols.push_back({d.d.dpsidt, v->dpsidt});
            cols.push_back({d.d.divB, v->divB});
        }
    }
    size_t k = 0;
    for(auto const& c : cols)
        k += c.second ? 1 : 0;
    if((st = ctx->stagingCols(k + 1)) || (st = ctx->ensureCopyStream()))
        return st;
    // Column k's unpermute (context stream) hands over to its copy (copy
    // stream) through eCompute, so copy k runs under unpermute k + 1.
    k = 0;
    for(auto const& c : cols)
    {
        if(!c.second)
            continue;
        double* stage = ctx->staging[k++];
        sph::launchUnpermute(ctx->n, d.cur.id, c.first, stage, ctx->stream);
        SPH_CUDA_TRY(cudaEventRecord(ctx->eCompute, ctx->stream));
        SPH_CUDA_TRY(cudaStreamWaitEvent(ctx->copyStream, ctx->eCompute, 0));
        SPH_CUDA_TRY(
            cudaMemcpyAsync(c.second, stage + s.offset, size_t(s.n) * 8, cudaMemcpyDeviceToHost, ctx->copyStream));
    }
    if(v->box_id)
    {
        int32_t* istage = reinterpret_cast<int32_t*>(ctx->staging[k]);
        sph::launchUnpermuteInt(ctx->n, d.cur.id, reinterpret_cast<uint32_t const*>(d.cur.box), istage, ctx->stream);
        SPH_CUDA_TRY(cudaEventRecord(ctx->eCompute, ctx->stream));
        SPH_CUDA_TRY(cudaStreamWaitEvent(ctx->copyStream, ctx->eCompute, 0));
        SPH_CUDA_TRY(
            cudaMemcpyAsync(v->box_id, istage + s.offset, size_t(s.n) * 4, cudaMemcpyDeviceToHost, ctx->copyStream));
    }
    // every unpermute precedes a copy the copy stream waited for
    SPH_CUDA_TRY(cudaStreamSynchronize(ctx->copyStream));
    SPH_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return SPH_OK;
}

int sph_get_neighbour_counts(sph_ctx* ctx, int32_t species_id, int32_t* counts)
{
    if(!ctx || !counts || species_id < 0 || species_id >= SPH_NUM_SPECIES)
        return fail(SPH_ERR_INVALID, "sph_get_neighbour_counts: bad arguments");
    SPH_COMPLETE_PENDING(ctx);
    HostSpecies const& s = ctx->sp[species_id];
    if(s.declared && s.n == 0)
        return SPH_OK;
    if(!s.set)
        return fail(SPH_ERR_STATE, "species not set");
    if(!ctx->densityValid)
        return fail(SPH_ERR_STATE, "no neighbour build yet (call sph_density or sph_step)");
    SPH_CUDA_TRY(cudaSetDevice(ctx->p.device));
    int st = ctx->stagingCols(1);
    if(st)
        return st;
    int32_t* istage = reinterpret_cast<int32_t*>(ctx->staging[0]);
    sph::launchUnpermuteInt(ctx->n, ctx->dc.cur.id, ctx->dc.lists.count, istage, ctx->stream);
    SPH_CUDA_TRY(cudaMemcpyAsync(counts, istage + s.offset, size_t(s.n) * 4, cudaMemcpyDeviceToHost, ctx->stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return SPH_OK;
}

namespace
{
    //! Per-box step state copied back to the host.
    struct HostBoxState
    {
        std::vector<double> dt, time, lastDt;
        std::vector<unsigned long long> ch;
    };

    int reduceBoxes(sph_ctx* ctx, std::vector<double>& perBox, sph::StepScalars& sc, HostBoxState& hb)
    {
        int st = ctx->ensureDevice();
        if(st)
            return st;
        uint32_t const nbox = ctx->dc.nbox;
        sph::launchBoxReduce(ctx->dc, ctx->pa, ctx->boxOut, ctx->boxScratch, ctx->stream);
        perBox.resize(size_t(nbox) * sph::kDiagWords);
        hb.dt.resize(nbox);
        hb.time.resize(nbox);
        hb.lastDt.resize(nbox);
        hb.ch.resize(nbox);
        SPH_CUDA_TRY(cudaMemcpyAsync(perBox.data(), ctx->boxOut, perBox.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
        SPH_CUDA_TRY(cudaMemcpyAsync(&sc, ctx->dc.scal, sizeof(sc), cudaMemcpyDeviceToHost, ctx->stream));
        SPH_CUDA_TRY(cudaMemcpyAsync(hb.dt.data(), ctx->dc.bs.dt, 8 * nbox, cudaMemcpyDeviceToHost, ctx->stream));
        SPH_CUDA_TRY(cudaMemcpyAsync(hb.time.data(), ctx->dc.bs.time, 8 * nbox, cudaMemcpyDeviceToHost, ctx->stream));
        SPH_CUDA_TRY(cudaMemcpyAsync(hb.lastDt.data(), ctx->dc.bs.lastDt, 8 * nbox, cudaMemcpyDeviceToHost, ctx->stream));
        SPH_CUDA_TRY(cudaMemcpyAsync(hb.ch.data(), ctx->dc.bs.chBits, 8 * nbox, cudaMemcpyDeviceToHost, ctx->stream));
        SPH_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        return SPH_OK;
    }

    void fillDiag(SphDiag& o, double const* a, sph::StepScalars const& sc, HostBoxState const& hb, uint32_t b)
    {
        o.e_kin = a[0];
        o.e_int = a[1];
        o.e_mag = a[2];
        o.mom[0] = a[3];
        o.mom[1] = a[4];
        o.mom[2] = a[5];
        o.divb_mean = a[7] > 0 ? a[6] / a[7] : 0.0;
        o.divb_max = a[8];
        o.n_targets = int64_t(a[9]);
        o.time = hb.time[b];
        o.dt = hb.lastDt[b];
        o.dt_next = hb.dt[b];
        o.c_h = __builtin_bit_cast(double, hb.ch[b]);
        o.pairs = double(sc.pairs);
        o.steps = sc.steps;
        o.pairs_total = sc.pairsAccum;
        o.candidates = double(sc.candidates);
    }
} // namespace

int sph_reduce(sph_ctx* ctx, SphDiag* out)
{
    if(!ctx || !out)
        return fail(SPH_ERR_INVALID, "sph_reduce: bad arguments");
    SPH_COMPLETE_PENDING(ctx);
    if(ctx->empty())
    {
        *out = SphDiag{};
        out->steps = ctx->emptySteps;
        out->time = ctx->emptyTime;
        out->dt = out->dt_next = ctx->p.dt;
        return SPH_OK;
    }
    SPH_CUDA_TRY(cudaSetDevice(ctx->p.device));
    std::vector<double> pb;
    sph::StepScalars sc{};
    HostBoxState hb;
    int st = reduceBoxes(ctx, pb, sc, hb);
    if(st)
        return st;
    double a[sph::kDiagWords] = {};
    for(uint32_t b = 0; b < ctx->dc.nbox; ++b)
        for(int k = 0; k < sph::kDiagWords; ++k)
        {
            double const v = pb[size_t(b) * sph::kDiagWords + k];
            a[k] = (k == 8) ? std::max(a[k], v) : a[k] + v;
        }
    *out = SphDiag{};
    fillDiag(*out, a, sc, hb, 0);
    out->replays = ctx->replays;
    out->list_capacity = ctx->dc.lists.cap;
    // an ensemble reports the largest c_h and the smallest next dt over its boxes
    for(uint32_t b = 1; b < ctx->dc.nbox; ++b)
    {
        out->c_h = std::max(out->c_h, __builtin_bit_cast(double, hb.ch[b]));
        out->dt_next = std::min(out->dt_next, hb.dt[b]);
    }
    return SPH_OK;
}

int sph_ensemble_reduce(sph_ctx* ctx, int32_t nbox, SphDiag* out)
{
    if(!ctx || !out || nbox < 1)
        return fail(SPH_ERR_INVALID, "sph_ensemble_reduce: bad arguments");
    SPH_COMPLETE_PENDING(ctx);
    if(ctx->empty())
    {
        if(size_t(nbox) != std::max<size_t>(1, ctx->boxes.size()))
            return fail(SPH_ERR_INVALID, "sph_ensemble_reduce: nbox differs from the context's box count");
        for(int32_t b = 0; b < nbox; ++b)
        {
            out[b] = SphDiag{};
            out[b].steps = ctx->emptySteps;
            out[b].time = ctx->emptyTime;
            out[b].dt = out[b].dt_next = ctx->p.dt;
        }
        return SPH_OK;
    }
    SPH_CUDA_TRY(cudaSetDevice(ctx->p.device));
    std::vector<double> pb;
    sph::StepScalars sc{};
    HostBoxState hb;
    int st = reduceBoxes(ctx, pb, sc, hb);
    if(st)
        return st;
    if(uint32_t(nbox) != ctx->dc.nbox)
        return fail(SPH_ERR_INVALID, "sph_ensemble_reduce: nbox differs from the context's box count");
    for(int32_t b = 0; b < nbox; ++b)
    {
        out[b] = SphDiag{};
        fillDiag(out[b], &pb[size_t(b) * sph::kDiagWords], sc, hb, uint32_t(b));
        out[b].replays = ctx->replays;
        out[b].list_capacity = ctx->dc.lists.cap;
    }
    return SPH_OK;
}

int sph_get_clock(sph_ctx* ctx, int32_t nbox, double* time, double* dt_next)
{
    if(!ctx || nbox < 1 || !time || !dt_next)
        return fail(SPH_ERR_INVALID, "sph_get_clock: bad arguments");
    SPH_COMPLETE_PENDING(ctx);
    SPH_CUDA_TRY(cudaSetDevice(ctx->p.device));
    int st = ctx->ensureDevice();
    if(st)
        return st;
    if(uint32_t(nbox) != ctx->dc.nbox)
        return fail(SPH_ERR_INVALID, "sph_get_clock: nbox differs from the context's box count");
    SPH_CUDA_TRY(cudaMemcpyAsync(time, ctx->dc.bs.time, 8 * size_t(nbox), cudaMemcpyDeviceToHost, ctx->stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(dt_next, ctx->dc.bs.dt, 8 * size_t(nbox), cudaMemcpyDeviceToHost, ctx->stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return SPH_OK;
}

int sph_set_clock(sph_ctx* ctx, int32_t nbox, double const* time, double const* dt_next)
{
    if(!ctx || nbox < 1 || !time || !dt_next)
        return fail(SPH_ERR_INVALID, "sph_set_clock: bad arguments");
    SPH_COMPLETE_PENDING(ctx);
    for(int32_t b = 0; b < nbox; ++b)
        if(!std::isfinite(time[b]) || !(dt_next[b] > 0.0) || !std::isfinite(dt_next[b]))
            return fail(SPH_ERR_INVALID, "sph_set_clock: time must be finite and dt positive");
    SPH_CUDA_TRY(cudaSetDevice(ctx->p.device));
    int st = ctx->ensureDevice();
    if(st)
        return st;
    if(uint32_t(nbox) != ctx->dc.nbox)
        return fail(SPH_ERR_INVALID, "sph_set_clock: nbox differs from the context's box count");
    SPH_CUDA_TRY(cudaMemcpyAsync(ctx->dc.bs.time, time, 8 * size_t(nbox), cudaMemcpyHostToDevice, ctx->stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(ctx->dc.bs.dt, dt_next, 8 * size_t(nbox), cudaMemcpyHostToDevice, ctx->stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return SPH_OK;
}

int sph_get_timings(sph_ctx* ctx, int32_t n, double* ms)
{
    if(!ctx || !ms || n < 0)
        return fail(SPH_ERR_INVALID, "sph_get_timings: bad arguments");
    for(int32_t i = 0; i < n && i < 5; ++i)
        ms[i] = ctx->timings[i];
    return SPH_OK;
}

int sph_use_graph(sph_ctx* ctx, int32_t on)
{
    if(!ctx)
        return fail(SPH_ERR_INVALID, "null context");
    ctx->useGraph = on != 0;
    return SPH_OK;
}

int sph_prepare_graph(sph_ctx* ctx)
{
    if(!ctx)
        return fail(SPH_ERR_INVALID, "null context");
    SPH_COMPLETE_PENDING(ctx);
    if(!ctx->useGraph || ctx->empty())
        return SPH_OK;
    SPH_CUDA_TRY(cudaSetDevice(ctx->p.device));
    return ctx->prepareGraph();
}


int sph_init_lattice(
    sph_ctx* ctx,
    int32_t species_id,
    uint32_t roles,
    int32_t nblocks,
    const SphLatticeBlock* blocks,
    const SphInitProfile* profile,
    int64_t* n_out)
{
    if(!ctx || species_id < 0 || species_id >= SPH_NUM_SPECIES || nblocks < 0 || (nblocks > 0 && !blocks))
        return fail(SPH_ERR_INVALID, "sph_init_lattice: bad arguments");
    SPH_COMPLETE_PENDING(ctx);
    SphInitProfile prof{};
    if(profile)
        prof = *profile;
    if(prof.kind < SPH_PROFILE_CONSTANT || prof.kind > SPH_PROFILE_ROTOR)
        return fail(SPH_ERR_INVALID, "sph_init_lattice: unknown profile");
    // per-block lattice counts and site offsets; jitter groups of consecutive blocks
    std::vector<sph::LatticeBlockDev> hb(static_cast<size_t>(nblocks));
    std::vector<int> groupFirstBlock;
    unsigned long long sites = 0;
    for(int32_t b = 0; b < nblocks; ++b)
    {
        SphLatticeBlock const& B = blocks[b];
        sph::LatticeBlockDev& d = hb[size_t(b)];
        uint32_t n[3];
        bool const given = B.counts[0] > 0 || B.counts[1] > 0 || B.counts[2] > 0;
        for(int a = 0; a < 3; ++a)
            if(!std::isfinite(B.lo[a]) || !std::isfinite(B.hi[a]) || !(B.hi[a] >= B.lo[a]))
                return fail(SPH_ERR_INVALID, "sph_init_lattice: block with an invalid region");
        if(given)
        {
            for(int a = 0; a < 3; ++a)
            {
                if(B.counts[a] <= 0)
                    return fail(SPH_ERR_INVALID, "sph_init_lattice: counts must all be positive (or all 0)");
                n[a] = uint32_t(B.counts[a]);
            }
        }
        else
        {
            if(!(B.spacing > 0.0) || !std::isfinite(B.spacing))
                return fail(SPH_ERR_INVALID, "sph_init_lattice: block needs counts or a positive spacing");
            sph::latticeCounts(B.lo, B.hi, B.spacing, n);
        }
        if(B.mask < SPH_MASK_NONE || B.mask > SPH_MASK_OUTSIDE_DISC_XY)
            return fail(SPH_ERR_INVALID, "sph_init_lattice: unknown mask");
        if(B.box_id < 0)
            return fail(SPH_ERR_INVALID, "sph_init_lattice: negative box id");
        if(!(B.jitter >= 0.0) || !std::isfinite(B.jitter))
            return fail(SPH_ERR_INVALID, "sph_init_lattice: jitter must be >= 0");
        if(b == 0 || B.jitter_group != blocks[b - 1].jitter_group)
            groupFirstBlock.push_back(b);
        else if(B.jitter != blocks[b - 1].jitter || B.seed != blocks[b - 1].seed)
            return fail(SPH_ERR_INVALID, "sph_init_lattice: blocks of one jitter group need one amplitude and seed");
        for(int a = 0; a < 3; ++a)
        {
            d.lo[a] = B.lo[a];
            d.n[a] = n[a];
            d.d[a] = (B.hi[a] - B.lo[a]) / double(n[a]);
            d.vel[a] = B.vel[a];
            d.B[a] = B.B[a];
        }
        d.siteBase = sites;
        d.mask = B.mask;
        d.maskCentre[0] = B.mask_centre[0];
        d.maskCentre[1] = B.mask_centre[1];
        d.maskRadius = B.mask_radius;
        d.box = B.box_id;
        d.group = int32_t(groupFirstBlock.size() - 1);
        d.mass = B.mass;
        d.h = B.h;
        d.density = B.density;
        d.u = B.u;
        d.psi = B.psi;
        sites += (unsigned long long) n[0] * n[1] * n[2];
    }
    if(sites >= (1ull << 32))
        return fail(SPH_ERR_UNSUPPORTED, "sph_init_lattice: more than 2^32 lattice sites");
    SPH_CUDA_TRY(cudaSetDevice(ctx->p.device));
    if(!ctx->stream)
        SPH_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    cudaStream_t const s = ctx->stream;
    uint32_t total = 0;
    std::vector<uint32_t> first(size_t(nblocks) + 1, 0);
    InitScratch scr;
    sph::LatticeBlockDev* dBlocks = nullptr;
    uint32_t *flags = nullptr, *ranks = nullptr, *scanScratch = nullptr, *dFirst = nullptr;
    if(sites > 0)
    {
        SPH_CUDA_TRY(scr.take(dBlocks, hb.size()));
        SPH_CUDA_TRY(scr.take(flags, sites));
        SPH_CUDA_TRY(scr.take(ranks, sites));
        SPH_CUDA_TRY(scr.take(scanScratch, sph::scanScratchWords(uint32_t(sites))));
        SPH_CUDA_TRY(scr.take(dFirst, first.size()));
        SPH_CUDA_TRY(cudaMemcpyAsync(dBlocks, hb.data(), sizeof(hb[0]) * hb.size(), cudaMemcpyHostToDevice, s));
        sph::launchLatticeFlags(dBlocks, nblocks, sites, flags, s);
        sph::exclusiveScan(flags, ranks, uint32_t(sites), scanScratch, s);
        sph::launchBlockFirstRanks(dBlocks, nblocks, sites, flags, ranks, dFirst, s);
        SPH_CUDA_TRY(cudaMemcpyAsync(first.data(), dFirst, 4 * first.size(), cudaMemcpyDeviceToHost, s));
        SPH_CUDA_TRY(cudaStreamSynchronize(s));
        total = first[size_t(nblocks)];
    }
    // jitter groups: particle range of each group
    std::vector<sph::JitterGroupDev> groups(groupFirstBlock.size());
    for(size_t g = 0; g < groups.size(); ++g)
    {
        int const b0 = groupFirstBlock[g];
        int const b1 = g + 1 < groups.size() ? groupFirstBlock[g + 1] : nblocks;
        groups[g].amplitude = blocks[b0].jitter;
        groups[g].seed = blocks[b0].seed;
        groups[g].first = first[size_t(b0)];
        groups[g].count = first[size_t(b1)] - first[size_t(b0)];
    }
    // columns in species order, generated on the device
    std::vector<std::vector<double>> host(kHostCols);
    std::vector<int32_t> hostBox(total);
    if(total > 0)
    {
        sph::InitColumns col{};
        double* dcol[kHostCols];
        for(int c = 0; c < kHostCols; ++c)
            SPH_CUDA_TRY(scr.take(dcol[c], total));
        for(int a = 0; a < 3; ++a)
        {
            col.x[a] = dcol[cX + a];
            col.v[a] = dcol[cVX + a];
            col.B[a] = dcol[cBX + a];
        }
        col.u = dcol[cU];
        col.m = dcol[cM];
        col.h = dcol[cH];
        col.rho = dcol[cRho];
        col.psi = dcol[cPsi];
        SPH_CUDA_TRY(scr.take(col.box, total));
        SPH_CUDA_TRY(scr.take(col.group, total));
        sph::JitterGroupDev* dGroups = nullptr;
        SPH_CUDA_TRY(scr.take(dGroups, groups.size()));
        SPH_CUDA_TRY(
            cudaMemcpyAsync(dGroups, groups.data(), sizeof(groups[0]) * groups.size(), cudaMemcpyHostToDevice, s));
        sph::launchLatticePlace(dBlocks, nblocks, sites, flags, ranks, col, s);
        sph::InitProfileDev pd{};
        pd.kind = prof.kind;
        for(int k = 0; k < 8; ++k)
            pd.p[k] = prof.p[k];
        for(int a = 0; a < 3; ++a)
        {
            pd.wrap[a] = prof.wrap[a];
            pd.wrapLo[a] = prof.wrap_lo[a];
            pd.wrapHi[a] = prof.wrap_hi[a];
        }
        sph::launchJitterProfile(col, total, dGroups, pd, s);
        SPH_CUDA_TRY(cudaGetLastError());
        for(int c = 0; c < kHostCols; ++c)
        {
            host[size_t(c)].resize(total);
            SPH_CUDA_TRY(cudaMemcpyAsync(host[size_t(c)].data(), dcol[c], 8 * size_t(total), cudaMemcpyDeviceToHost, s));
        }
        SPH_CUDA_TRY(cudaMemcpyAsync(hostBox.data(), col.box, 4 * size_t(total), cudaMemcpyDeviceToHost, s));
        SPH_CUDA_TRY(cudaStreamSynchronize(s));
    }
    SphSoAView v{};
    for(int a = 0; a < 3; ++a)
    {
        v.pos[a] = host[size_t(cX + a)].data();
        v.vel[a] = host[size_t(cVX + a)].data();
        v.B[a] = host[size_t(cBX + a)].data();
    }
    v.mass = host[cM].data();
    v.h = host[cH].data();
    v.density = host[cRho].data();
    v.u = host[cU].data();
    v.psi = host[cPsi].data();
    v.box_id = hostBox.data();
    if(n_out)
        *n_out = int64_t(total);
    return sph_set_species(ctx, species_id, roles, int64_t(total), total > 0 ? &v : nullptr);
}

int sph_autotune(sph_ctx* ctx, int32_t steps_per_trial, SphTuning* out)
{
    if(!ctx)
        return fail(SPH_ERR_INVALID, "null context");
    SPH_COMPLETE_PENDING(ctx);
    SPH_CUDA_TRY(cudaSetDevice(ctx->p.device));
    int const st = ctx->autotune(steps_per_trial);
    if(st)
        return st;
    if(out)
        *out = ctx->tuning;
    return SPH_OK;
}

int sph_set_tuning(sph_ctx* ctx, int32_t density_variant, int32_t force_variant)
{
    if(!ctx)
        return fail(SPH_ERR_INVALID, "null context");
    if(density_variant < 0 || density_variant >= sph::densityVariants(ctx->p.precision) || force_variant < 0
       || force_variant >= sph::forceVariants(ctx->p.precision))
        return fail(SPH_ERR_INVALID, "sph_set_tuning: no such launch shape for this precision");
    if(ctx->densityVariant != density_variant || ctx->forceVariant != force_variant)
        ctx->dropGraphs();
    ctx->densityVariant = density_variant;
    ctx->forceVariant = force_variant;
    ctx->tuning.steps_per_trial = 0;
    return SPH_OK;
}

int sph_get_tuning(sph_ctx* ctx, SphTuning* out)
{
    if(!ctx || !out)
        return fail(SPH_ERR_INVALID, "sph_get_tuning: bad arguments");
    int32_t const spt = ctx->tuning.steps_per_trial;
    ctx->describeTuning();
    *out = ctx->tuning;
    out->steps_per_trial = spt;
    return SPH_OK;
}

const char* sph_last_error_string(void)
{
    return g_lastError.c_str();
}
} // extern "C"
