// Internal: device state of one context and the launchers of every kernel.
#pragma once

#include "sph_common.cuh"

#include <cstddef>

namespace sph
{
    //! 32-byte FP64 quadruple (two 16-byte loads).
    struct alignas(32) D4
    {
        double x, y, z, w;
    };

    //! Master particle state in the current sorted order (FP64 integration state).
    struct Master
    {
        double* x[3];
        double* v[3];
        double* u;
        double* m;
        double* h;
        double* rho;
        double* B[3];
        double* psi;
        uint32_t* id;   //!< input index (species offset + index within the species)
        int32_t* box;
        uint8_t* role;
    };

    //! Time derivatives and per-particle outputs of the force pass (sorted order).
    struct Derivs
    {
        double* dvdt[3];
        double* dudt;
        double* dBdt[3];
        double* dpsidt;
        double* divB;
    };

    //! Packed records the pair kernels read, in sorted order.  V4 is float4
    //! (FP32 path) or D4 (FP64 path).
    //!   pm: position relative to the lower corner of its cell (x, y, z) and mass
    //!   hc: smoothing length in the pair precision (the cull radius uses it)
    //!   fv: velocity (x, y, z) and h
    //!   ft: rho, (P + B^2/(2 mu0))/rho^2, signal speed c, 1/(mu0 rho^2)
    //!   fb: B (x, y, z) and psi/rho^2
    template<typename V4, typename T>
    struct Records
    {
        V4* pm;
        T* hc;
        V4* fv;
        V4* ft;
        V4* fb;
    };

    //! Physics constants the kernels need (one copy per launch, by value).
    struct PhysArgs
    {
        double gamma, alpha, beta, avEps, mu0, cfl, cflForce, sigma, h0, hfact;
        uint32_t physics;
        int32_t cull;
    };

    //! Derived per-particle quantities the force pass reads for a source:
    //! ft = (rho, (P + B^2/(2 mu0))/rho^2, c, 1/(mu0 rho^2)), fb = (B, psi/rho^2).
    //! c is the sound speed, or the fast speed sqrt(c_s^2 + B^2/(mu0 rho)) with MHD.
    __device__ __forceinline__ void derivedRecord(
        double rho,
        double u,
        double const B[3],
        double psi,
        PhysArgs const& pa,
        double ft[4],
        double fb[4])
    {
        bool const mhd = pa.physics & SPH_PHYS_MHD;
        double const P = (pa.gamma - 1.0) * rho * u;
        double const inv2 = 1.0 / (rho * rho);
        double const cs2 = pa.gamma * P / rho;
        double B2 = 0.0;
        if(mhd)
            B2 = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
        ft[0] = rho;
        ft[1] = (P + (mhd ? 0.5 * B2 / pa.mu0 : 0.0)) * inv2;
        ft[2] = sqrt(cs2 + (mhd ? B2 / (pa.mu0 * rho) : 0.0));
        ft[3] = inv2 / pa.mu0;
        fb[0] = mhd ? B[0] : 0.0;
        fb[1] = mhd ? B[1] : 0.0;
        fb[2] = mhd ? B[2] : 0.0;
        fb[3] = mhd ? psi * inv2 : 0.0;
    }

    //! Box of a density work item (boxes are sorted by activeBase).
    __device__ __forceinline__ int boxOfWork(BoxDev const* boxes, uint32_t nbox, uint32_t q)
    {
        int lo = 0, hi = int(nbox) - 1;
        while(lo < hi)
        {
            int const mid = (lo + hi + 1) >> 1;
            if(boxes[mid].activeBase <= q)
                lo = mid;
            else
                hi = mid - 1;
        }
        return lo;
    }

    //! Box of a global cell id (boxes are sorted by cellBase).
    __device__ __forceinline__ int boxOfCell(BoxDev const* boxes, uint32_t nbox, uint32_t cell)
    {
        int lo = 0, hi = int(nbox) - 1;
        while(lo < hi)
        {
            int const mid = (lo + hi + 1) >> 1;
            if(boxes[mid].cellBase <= cell)
                lo = mid;
            else
                hi = mid - 1;
        }
        return lo;
    }

    template<typename V4>
    __device__ __forceinline__ V4 mk4(double a, double b, double c, double d);
    template<>
    __device__ __forceinline__ float4 mk4<float4>(double a, double b, double c, double d)
    {
        return make_float4(float(a), float(b), float(c), float(d));
    }
    template<>
    __device__ __forceinline__ D4 mk4<D4>(double a, double b, double c, double d)
    {
        return D4{a, b, c, d};
    }

    //! Read-only 16/32-byte record loads.
    __device__ __forceinline__ float4 ld4(float4 const* p)
    {
        return __ldg(p);
    }
    __device__ __forceinline__ D4 ld4(D4 const* p)
    {
        double2 const a = __ldg(reinterpret_cast<double2 const*>(p));
        double2 const b = __ldg(reinterpret_cast<double2 const*>(p) + 1);
        return D4{a.x, a.y, b.x, b.y};
    }

    //! Cell index ranges in sorted order: [start, mid) targets, [mid, end) other sources.
    struct Cells
    {
        uint32_t* start;
        uint32_t* mid;
        uint32_t* end;
        uint32_t ncells;
        //! Two-level boxes: the sorted range of all level-1 sub-cells of level-0
        //! cell c (contiguous, parent-major numbering), at the level-0 cell id.
        uint32_t* bstart;
        uint32_t* bend;
    };

    //! Neighbour lists: row t (sorted target index) holds count[t] entries of
    //! packEntry(j, stencil slot) at list[t * cap + k].
    struct Lists
    {
        uint32_t* list;
        uint32_t* count;
        uint32_t cap;
    };

    //! Scalars the step keeps on the device so a step never waits for the host.
    struct StepScalars
    {
        unsigned long long pairs;  //!< accepted ordered pairs of the last neighbour build
        double pairsAccum;         //!< accepted pairs summed over the steps taken
        long long steps;
        unsigned long long candidates; //!< (target, staged source) pairs tested by the last cull
    };

    //! Per-box step state (structure of arrays, nbox entries each).  Boxes of an
    //! ensemble are independent: each has its own dt, time, CFL minimum and
    //! Dedner cleaning speed.
    struct BoxScalars
    {
        double* dt;                  //!< dt of the current step
        double* time;                //!< simulated time
        double* lastDt;              //!< dt of the last completed step
        unsigned long long* dtBits;  //!< min CFL dt over the box's targets (ordered bits)
        unsigned long long* chBits;  //!< max signal speed of the box's targets (ordered bits)
        unsigned long long* hmaxBits; //!< max h of the box's particles (ordered bits; the grid follows it)
        unsigned long long* hminBits; //!< min h of the box's particles (ordered bits; two levels when small enough)
    };

    struct DevCtx
    {
        uint32_t n;
        uint32_t nbox;
        BoxDev* boxes;
        //! Per box, 32 entries: stencil slot s -> image shift (o_x e_x, o_y e_y, o_z e_z, 0)
        //! with o = the slot's offsets in {-1, 0, 1} and e = the cell edges (exact products).
        float4* shift32;
        D4* shift64;
        Master cur, alt;
        Derivs d;
        Cells cells;
        Lists lists;
        Records<float4, float> r32;
        Records<D4, double> r64;
        uint32_t* keysA;
        uint32_t* valsA;
        uint32_t* keysB;
        uint32_t* valsB;
        uint32_t* sortScratch;
        uint32_t* status; //!< kStatWords words
        uint32_t* work;   //!< density work queue: next cell to hand out (zeroed before each launch)
        uint32_t* kickDone; //!< kick blocks finished; the last one finalises the step and resets it
        uint32_t* activeTotal; //!< work items of all boxes (their current cells, both levels)
        int32_t support;       //!< kernel support in units of h
        StepScalars* scal;
        BoxScalars bs;
        double* partials; //!< per-block diagnostics partial sums
        double* diag;     //!< finalized diagnostics (kDiagWords)
        uint32_t nPartialBlocks;
        int keyBits;
    };

    constexpr int kDiagWords = 12; // e_kin e_int e_mag mom3 divb_sum divb_cnt divb_max n_targets dt time

    //! Adds k to the library's kernel-launch counter (measure.cu).
    void countLaunches(unsigned k);
    //! The counter's value; and taking back launches that were only recorded
    //! into a CUDA graph (a graph's kernels count each time it is launched).
    unsigned long long launchesSoFar();
    void uncountLaunches(unsigned long long k);

    // ---- sort.cu
    size_t scanScratchWords(uint32_t m);
    void exclusiveScan(uint32_t const* in, uint32_t* out, uint32_t m, uint32_t* scratch, cudaStream_t s);
    size_t radixScratchWords(uint32_t n);
    //! Sorts (keysA, valsA) by the low `bits` bits of the key, stably; returns true
    //! when the result ended in (keysB, valsB).
    bool radixSortPairs(
        uint32_t* keysA,
        uint32_t* valsA,
        uint32_t* keysB,
        uint32_t* valsB,
        uint32_t n,
        int bits,
        uint32_t* scratch,
        cudaStream_t s);

    // ---- step_kernels.cu
    void launchDriftKeys(DevCtx const& c, bool drift, cudaStream_t s);
    void launchCellRanges(DevCtx const& c, uint32_t const* sortedKeys, cudaStream_t s);
    void launchPermute(DevCtx const& c, uint32_t const* perm, PhysArgs const& pa, int precision, cudaStream_t s);
    //! Kick, adaptive h and the block partials of the conserved sums; the last
    //! block to finish also finalises the step (sums, clock, next CFL dt).
    void launchKick(DevCtx const& c, PhysArgs const& pa, bool cfl, cudaStream_t s);
    void launchFinalize(DevCtx const& c, bool cfl, cudaStream_t s);
    void launchUnpermute(uint32_t n, uint32_t const* id, double const* src, double* dst, cudaStream_t s);
    void launchUnpermuteInt(uint32_t n, uint32_t const* id, uint32_t const* src, int32_t* dst, cudaStream_t s);
    //! Per-box conserved sums into out[nbox][kDiagWords]; scratch holds
    //! boxReduceScratchDoubles(nbox) doubles.
    void launchBoxReduce(DevCtx const& c, PhysArgs const& pa, double* out, double* scratch, cudaStream_t s);
    size_t boxReduceScratchDoubles(uint32_t nbox);
    void launchFill(double* p, size_t n, double v, cudaStream_t s);
    // ---- init.cu: device initialiser of lattice blocks
    //! One lattice block on the device (sites x-fastest, site s of the block at
    //! lo + (i + 0.5) * d per axis).
    struct LatticeBlockDev
    {
        double lo[3];
        double d[3];
        unsigned long long n[3];
        unsigned long long siteBase; //!< first global site index of the block
        int32_t mask;
        double maskCentre[2];
        double maskRadius;
        int32_t box;
        int32_t group; //!< jitter group
        double mass, h, density, u, psi;
        double vel[3], B[3];
    };
    struct JitterGroupDev
    {
        double amplitude;       //!< uniform displacement amplitude (length)
        unsigned long long seed;
        uint32_t first;         //!< first particle of the group
        uint32_t count;         //!< particles in the group
    };
    struct InitProfileDev
    {
        int32_t kind;
        double p[8];
        int32_t wrap[3];
        double wrapLo[3], wrapHi[3];
    };
    struct InitColumns
    {
        double* x[3];
        double* v[3];
        double* B[3];
        double* m;
        double* h;
        double* rho;
        double* u;
        double* psi;
        int32_t* box;
        int32_t* group;
    };
    void latticeCounts(double const lo[3], double const hi[3], double spacing, uint32_t n[3]);
    void launchLatticeFlags(LatticeBlockDev const* blocks, int nb, unsigned long long sites, uint32_t* flags, cudaStream_t s);
    void launchLatticePlace(
        LatticeBlockDev const* blocks,
        int nb,
        unsigned long long sites,
        uint32_t const* flags,
        uint32_t const* ranks,
        InitColumns const& out,
        cudaStream_t s);
    //! first[b] = compacted index of block b's first kept site; first[nb] = total kept.
    void launchBlockFirstRanks(
        LatticeBlockDev const* blocks,
        int nb,
        unsigned long long sites,
        uint32_t const* flags,
        uint32_t const* ranks,
        uint32_t* first,
        cudaStream_t s);
    void launchJitterProfile(
        InitColumns const& out,
        uint32_t n,
        JitterGroupDev const* groups,
        InitProfileDev const& prof,
        cudaStream_t s);

    //! Grid of every box from its particles' current largest h (pair-max cull):
    //! n = floor(L / cellRadius(support, hmax)) clamped to [1, nMax], the
    //! stencil shift tables, the active-cell prefix and total.
    //! Level-1 block range (bstart/bend) of every level-0 cell of the boxes
    //! that run two levels this step; totalCells bounds the work items.
    void launchSubBlocks(DevCtx const& c, uint32_t totalCells, cudaStream_t s);
    void launchGridUpdate(DevCtx const& c, int support, cudaStream_t s);

    //! dst <- src for every master column (n particles).
    void launchCopyMaster(Master const& dst, Master const& src, uint32_t n, cudaStream_t s);
    //! master[p] = src[id[p]] for one species; badCount (or null) counts values
    //! that are not positive and finite.
    void launchGatherSpecies(
        uint32_t n,
        uint32_t const* id,
        uint32_t off,
        uint32_t cnt,
        double const* src,
        double dflt,
        double* master,
        uint32_t* badCount,
        cudaStream_t s);
    void launchGatherSpeciesInt(
        uint32_t n,
        uint32_t const* id,
        uint32_t off,
        uint32_t cnt,
        int32_t const* src,
        int32_t* master,
        cudaStream_t s);
    uint32_t partialBlocks(uint32_t n);

    // ---- pair_kernels.cu
    //! Neighbour build + density (+ records for the force pass); countOnly only counts.
    //! Pair-kernel launches; `variant` picks the launch shape (0 = default,
    //! see densityVariants / forceVariants).
    void launchDensity(
        DevCtx const& c,
        PhysArgs const& pa,
        int kernel,
        int precision,
        bool countOnly,
        int variant,
        cudaStream_t s);
    void launchForce(DevCtx const& c, PhysArgs const& pa, int kernel, int precision, int variant, cudaStream_t s);
    int densityVariants(int precision);
    int forceVariants(int precision);
    void densityShape(int precision, int variant, int* stagingDepth, int* blocksPerSm, int* cullUnroll);
    int forceBlocksPerSm(int precision, int physics, int variant);
    //! Sets the shared-memory attributes of every pair-kernel instantiation
    //! (once, before any launch, so no attribute call happens during a graph capture).
    void configurePairKernels();
} // namespace sph
