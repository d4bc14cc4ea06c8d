// Per-particle kernels of the step: drift + cell keys, cell ranges, permute +
// record packing, kick + conserved-quantity partial sums, finalisation.
//
// These replace the reference's per-particle launches (launchForEach over
// PushVelocity / EulerIntegrate, spmacc/particles/algorithms/LaunchForEach.hpp:129-160;
// include/spearhed/particles/pusher/PushVelocity.hpp:38-41, EulerIntegrate.hpp:45-51)
// and its region bookkeeping.  All are HBM-streaming kernels: coalesced FP64
// columns in, coalesced columns out.
#include "sph_launch.hpp"

#include <algorithm>
#include <cfloat>

namespace sph
{
    namespace
    {
        constexpr int kThreads = 256;

        //! Drift (Movable): x += v dt with periodic wrap; then the cell key.  The
        //! product and the sum are rounded separately, as the reference's CPU
        //! path evaluates PushVelocity (PushVelocity.hpp:38-41), so the FP64
        //! positions equal the oracle's bit for bit.
        //! Key = 2 * global cell + (0 for targets, 1 for other sources); particles
        //! that are no source sort behind every cell (key 2 * ncells).
        __global__ void __launch_bounds__(kThreads) kDriftKeys(DevCtx c, bool drift)
        {
            uint32_t const p = blockIdx.x * blockDim.x + threadIdx.x;
            if(p >= c.n)
                return;
            uint8_t const role = c.cur.role[p];
            int32_t const bx = c.cur.box[p];
            BoxDev const& B = c.boxes[bx];
            double const dt = c.bs.dt[bx];
            double x[3];
            bool finite = true;
#pragma unroll
            for(int a = 0; a < 3; ++a)
            {
                x[a] = c.cur.x[a][p];
                if(drift && (role & SPH_ROLE_MOVABLE))
                {
                    x[a] = __dadd_rn(x[a], __dmul_rn(c.cur.v[a][p], dt));
                    if(B.periodic[a])
                    {
                        double const hiEdge = B.lo[a] + B.L[a];
                        for(int it = 0; it < 4 && x[a] >= hiEdge; ++it)
                            x[a] -= B.L[a];
                        for(int it = 0; it < 4 && x[a] < B.lo[a]; ++it)
                            x[a] += B.L[a];
                    }
                    c.cur.x[a][p] = x[a];
                }
                finite = finite && isfinite(x[a]);
            }
            uint32_t key = 2u * c.cells.ncells;
            if(!finite)
            {
                atomicAdd(&c.status[kStatNonFinite], 1u);
            }
            else
            {
                // every axis: a drifted particle was wrapped on its periodic axes;
                // one that was not (frozen, a density-only call, the same-size
                // species path) must lie in [lo, hi] for the cell search
                bool outside = false;
#pragma unroll
                for(int a = 0; a < 3; ++a)
                    if(x[a] < B.lo[a] || x[a] > B.lo[a] + B.L[a])
                        outside = true;
                if(outside)
                    atomicAdd(&c.status[kStatOutside], 1u);
                if(isSource(role))
                {
                    int cc[3];
#pragma unroll
                    for(int a = 0; a < 3; ++a)
                        cc[a] = cellCoord(B, a, x[a]);
                    uint32_t cell = B.cellBase + (uint32_t(cc[2]) * uint32_t(B.n[1]) + uint32_t(cc[1])) * uint32_t(B.n[0])
                                    + uint32_t(cc[0]);
                    if(B.levels == 2 && cellRadiusDev(c.support, c.cur.h[p]) <= B.e1)
                    {
                        // level 1: the sub-cell of the level-0 cell, from the position
                        // relative to the cell corner (as the permute computes it);
                        // sub-cells of one level-0 cell are numbered together
                        uint32_t sub = 0, stride = 1;
#pragma unroll
                        for(int a = 0; a < 3; ++a)
                        {
                            double const rel = __dsub_rn(x[a], cellOrigin(B, a, cc[a]));
                            uint32_t const s = B.m[a] == 2 && rel >= 0.5 * B.edge[a] ? 1u : 0u;
                            sub += s * stride;
                            stride *= uint32_t(B.m[a]);
                        }
                        cell = B.cellBase + B.ncellsMax + (cell - B.cellBase) * B.msub + sub;
                    }
                    if(checkIndex(cell < c.cells.ncells, c.status, kChkDriftCell))
                        key = 2u * cell + (isTarget(role) ? 0u : 1u);
                }
            }
            c.keysA[p] = key;
            c.valsA[p] = p;
        }

        __global__ void __launch_bounds__(kThreads) kCellRanges(uint32_t const* __restrict__ keys, uint32_t n, Cells cells)
        {
            uint32_t const p = blockIdx.x * blockDim.x + threadIdx.x;
            if(p >= n)
                return;
            uint32_t const k = keys[p];
            uint32_t const cell = k >> 1;
            if(cell >= cells.ncells)
                return;
            uint32_t const other = k & 1u;
            uint32_t const kp = p > 0 ? keys[p - 1] : 0xffffffffu;
            uint32_t const kn = p + 1 < n ? keys[p + 1] : 0xffffffffu;
            bool const firstOfCell = p == 0 || (kp >> 1) != cell;
            bool const lastOfCell = p + 1 == n || (kn >> 1) != cell;
            if(firstOfCell)
                cells.start[cell] = p;
            if(other && (p == 0 || kp != k))
                cells.mid[cell] = p;
            if(lastOfCell)
            {
                cells.end[cell] = p + 1;
                if(!other)
                    cells.mid[cell] = p + 1;
            }
        }

        template<typename V4, typename T>
        __global__ void __launch_bounds__(kThreads)
            kPermute(DevCtx c, uint32_t const* __restrict__ perm, PhysArgs pa, Records<V4, T> rec)
        {
            uint32_t const p = blockIdx.x * blockDim.x + threadIdx.x;
            if(p >= c.n)
                return;
            uint32_t const q = perm[p];
            if(!checkIndex(q < c.n, c.status, kChkPermute))
                return;
            double x[3], v[3], Bv[3];
#pragma unroll
            for(int a = 0; a < 3; ++a)
            {
                x[a] = c.cur.x[a][q];
                v[a] = c.cur.v[a][q];
                Bv[a] = c.cur.B[a][q];
                c.alt.x[a][p] = x[a];
                c.alt.v[a][p] = v[a];
                c.alt.B[a][p] = Bv[a];
            }
            double const u = c.cur.u[q], m = c.cur.m[q], h = c.cur.h[q], rho = c.cur.rho[q], psi = c.cur.psi[q];
            c.alt.u[p] = u;
            c.alt.m[p] = m;
            c.alt.h[p] = h;
            c.alt.rho[p] = rho;
            c.alt.psi[p] = psi;
            c.alt.id[p] = c.cur.id[q];
            int32_t const b = c.cur.box[q];
            c.alt.box[p] = b;
            uint8_t const role = c.cur.role[q];
            c.alt.role[p] = role;
            if(!isSource(role))
                return;
            BoxDev const& B = c.boxes[b];
            double rel[3];
#pragma unroll
            for(int a = 0; a < 3; ++a)
            {
                int const ca = cellCoord(B, a, x[a]);
                rel[a] = __dsub_rn(x[a], cellOrigin(B, a, ca));
            }
            rec.pm[p] = mk4<V4>(rel[0], rel[1], rel[2], m);
            rec.hc[p] = T(h);
            rec.fv[p] = mk4<V4>(v[0], v[1], v[2], h);
            if(!isTarget(role))
            {
                // Frozen source (Boundary species): rho and u keep their initial values.
                double ft[4], fb[4];
                derivedRecord(rho, u, Bv, psi, pa, ft, fb);
                rec.ft[p] = mk4<V4>(ft[0], ft[1], ft[2], ft[3]);
                rec.fb[p] = mk4<V4>(fb[0], fb[1], fb[2], fb[3]);
            }
        }

        __device__ __forceinline__ double warpSum(double v)
        {
#pragma unroll
            for(int o = 16; o > 0; o >>= 1)
                v += __shfl_down_sync(0xffffffffu, v, o);
            return v;
        }
        __device__ __forceinline__ double warpMax(double v)
        {
#pragma unroll
            for(int o = 16; o > 0; o >>= 1)
                v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
            return v;
        }

        //! Kick (Movable & Thermodynamic): v += dvdt dt, u += dudt dt, and with MHD
        //! B += dBdt dt, psi += dpsidt dt; then FP64 block partial sums of the
        //! conserved quantities of the new state (deterministic: fixed order).
        //! Step epilogue of one block: the block partials of the conserved sums
        //! in a fixed order (read through L2: other blocks wrote them), the step
        //! counters, and every box's clock and next dt.  red holds one row per warp.
        __device__ void finalizeStep(DevCtx const& c, bool cfl, double (*red)[kDiagWords])
        {
            double acc[kDiagWords];
#pragma unroll
            for(int k = 0; k < kDiagWords; ++k)
                acc[k] = 0.0;
            for(uint32_t b = threadIdx.x; b < c.nPartialBlocks; b += blockDim.x)
#pragma unroll
                for(int k = 0; k < kDiagWords; ++k)
                {
                    double const v = __ldcg(&c.partials[size_t(b) * kDiagWords + k]);
                    acc[k] = (k == 8) ? fmax(acc[k], v) : acc[k] + v;
                }
            int const lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            __syncthreads(); // red is free again
#pragma unroll
            for(int k = 0; k < kDiagWords; ++k)
            {
                double const r = (k == 8) ? warpMax(acc[k]) : warpSum(acc[k]);
                if(lane == 0)
                    red[warp][k] = r;
            }
            __syncthreads();
            if(threadIdx.x == 0)
            {
                double tot[kDiagWords];
#pragma unroll
                for(int k = 0; k < kDiagWords; ++k)
                {
                    tot[k] = 0.0;
                    for(int w = 0; w < int(blockDim.x / 32); ++w)
                        tot[k] = (k == 8) ? fmax(tot[k], red[w][k]) : tot[k] + red[w][k];
                }
                StepScalars& S = *c.scal;
                S.steps += 1;
                S.pairsAccum += double(S.pairs);
#pragma unroll
                for(int k = 0; k < 10; ++k)
                    c.diag[k] = tot[k];
                c.diag[10] = c.bs.dt[0];
                c.diag[11] = c.bs.time[0] + c.bs.dt[0];
            }
            // every box advances by its own dt; with CFL its next dt is its own minimum
            for(uint32_t b = threadIdx.x; b < c.nbox; b += blockDim.x)
            {
                double const dt = c.bs.dt[b];
                c.bs.time[b] += dt;
                c.bs.lastDt[b] = dt;
                if(cfl)
                {
                    double const dtn = __longlong_as_double(static_cast<long long>(c.bs.dtBits[b]));
                    if(dtn > 0.0 && dtn < 1e300)
                        c.bs.dt[b] = dtn;
                }
            }
        }

        __global__ void __launch_bounds__(kThreads) kKick(DevCtx c, PhysArgs pa, bool cfl)
        {
            __shared__ double red[kThreads / 32][kDiagWords];
            double acc[kDiagWords];
#pragma unroll
            for(int k = 0; k < kDiagWords; ++k)
                acc[k] = 0.0;
            bool const mhd = pa.physics & SPH_PHYS_MHD;
            // grid-stride: at most a few blocks per SM, so the step's epilogue
            // sums few block partials
            for(uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < c.n; p += gridDim.x * blockDim.x)
            {
                if(!isTarget(c.cur.role[p]))
                    continue;
                double const dt = c.bs.dt[c.cur.box[p]];
                double const m = c.cur.m[p];
                double v2 = 0.0, B2 = 0.0;
#pragma unroll
                for(int a = 0; a < 3; ++a)
                {
                    // unfused, as EulerIntegrate.hpp:45-51 on the reference's CPU path
                    double const va = __dadd_rn(c.cur.v[a][p], __dmul_rn(c.d.dvdt[a][p], dt));
                    c.cur.v[a][p] = va;
                    v2 += va * va;
                    acc[3 + a] += m * va;
                }
                double const u = __dadd_rn(c.cur.u[p], __dmul_rn(c.d.dudt[p], dt));
                c.cur.u[p] = u;
                if(mhd)
                {
#pragma unroll
                    for(int a = 0; a < 3; ++a)
                    {
                        double const Ba = __dadd_rn(c.cur.B[a][p], __dmul_rn(c.d.dBdt[a][p], dt));
                        c.cur.B[a][p] = Ba;
                        B2 += Ba * Ba;
                    }
                    c.cur.psi[p] = __dadd_rn(c.cur.psi[p], __dmul_rn(c.d.dpsidt[p], dt));
                }
                acc[0] += 0.5 * m * v2;
                acc[1] += m * u;
                double const rho = c.cur.rho[p];
                if(pa.physics & SPH_PHYS_ADAPTIVE_H)
                {
                    // h for the next step from this step's density, capped by the box's h cap
                    double const hn = pa.hfact * cbrt(m / rho);
                    double const cap = c.boxes[c.cur.box[p]].hcap;
                    c.cur.h[p] = hn < cap ? hn : cap;
                }
                if(mhd && rho > 0.0)
                    acc[2] += 0.5 * m * B2 / (pa.mu0 * rho);
                if(mhd && B2 > 0.0)
                {
                    double const e = fabs(c.d.divB[p]) * c.cur.h[p] / sqrt(B2);
                    acc[6] += e;
                    acc[7] += 1.0;
                    acc[8] = fmax(acc[8], e);
                }
                acc[9] += 1.0;
            }
            int const lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
            for(int k = 0; k < kDiagWords; ++k)
            {
                double const r = (k == 8) ? warpMax(acc[k]) : warpSum(acc[k]);
                if(lane == 0)
                    red[warp][k] = r;
            }
            __syncthreads();
            if(threadIdx.x < kDiagWords)
            {
                int const k = threadIdx.x;
                double r = 0.0;
                for(int w = 0; w < kThreads / 32; ++w)
                    r = (k == 8) ? fmax(r, red[w][k]) : r + red[w][k];
                c.partials[size_t(blockIdx.x) * kDiagWords + k] = r;
            }
            // the last block to finish finalises the step (no block waits for another)
            __shared__ bool last;
            __threadfence();
            __syncthreads();
            if(threadIdx.x == 0)
                last = atomicAdd(c.kickDone, 1u) == gridDim.x - 1;
            __syncthreads();
            if(last)
            {
                finalizeStep(c, cfl, red);
                if(threadIdx.x == 0)
                    *c.kickDone = 0;
            }
        }

        //! The step epilogue on its own (a step with no particle to kick).
        __global__ void __launch_bounds__(kThreads) kFinalize(DevCtx c, bool cfl)
        {
            __shared__ double red[kThreads / 32][kDiagWords];
            finalizeStep(c, cfl, red);
        }

        __global__ void kUnpermute(uint32_t n, uint32_t const* __restrict__ id, double const* __restrict__ src, double* __restrict__ dst)
        {
            uint32_t const p = blockIdx.x * blockDim.x + threadIdx.x;
            if(p < n)
                dst[id[p]] = src[p];
        }
        __global__ void kUnpermuteInt(uint32_t n, uint32_t const* __restrict__ id, uint32_t const* __restrict__ src, int32_t* __restrict__ dst)
        {
            uint32_t const p = blockIdx.x * blockDim.x + threadIdx.x;
            if(p < n)
                dst[id[p]] = int32_t(src[p]);
        }
        //! master[p] = src[id[p]] (or dflt) for the particles of one species
        //! (ids in [off, off + cnt)); src is in input order.
        __global__ void kGatherSpecies(
            uint32_t n,
            uint32_t const* __restrict__ id,
            uint32_t off,
            uint32_t cnt,
            double const* __restrict__ src,
            double dflt,
            double* __restrict__ master,
            uint32_t* __restrict__ badCount)
        {
            uint32_t const p = blockIdx.x * blockDim.x + threadIdx.x;
            if(p >= n)
                return;
            uint32_t const i = id[p];
            if(i - off < cnt)
            {
                double const v = src ? src[i] : dflt;
                // columns that must be positive and finite (h, source masses) pass a counter
                if(badCount && !(v > 0.0 && isfinite(v)))
                    atomicAdd(badCount, 1u);
                master[p] = v;
            }
        }
        __global__ void kGatherSpeciesInt(
            uint32_t n,
            uint32_t const* __restrict__ id,
            uint32_t off,
            uint32_t cnt,
            int32_t const* __restrict__ src,
            int32_t* __restrict__ master)
        {
            uint32_t const p = blockIdx.x * blockDim.x + threadIdx.x;
            if(p >= n)
                return;
            uint32_t const i = id[p];
            if(i - off < cnt)
                master[p] = src[i];
        }
        __global__ void kFill(double* p, size_t n, double v)
        {
            size_t const i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if(i < n)
                p[i] = v;
        }

        //! Largest and smallest h of each box's particles, as ordered bits.  A
        //! warp walks kHmaxRun consecutive groups of 32 particles (each group one
        //! coalesced load) and keeps a running maximum and minimum while every
        //! particle of a group is in the warp's current box.  After the first
        //! neighbour build the particles are box-sorted, so one pair of atomics
        //! serves a whole run instead of every group: the boxes' 512 addresses
        //! otherwise serialise about 2 n / 32 atomics in L2.  A group that spans
        //! boxes falls back to per-particle atomics.
        constexpr int kHmaxRun = 16;
        __global__ void __launch_bounds__(kThreads) kBoxHmax(DevCtx c)
        {
            int const lane = threadIdx.x & 31;
            uint32_t const base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * (32u * kHmaxRun);
            int cur = -1; // warp-uniform: the box the running extrema belong to
            double m = 0.0, mn = 1e300;
            auto flush = [&]()
            {
                if(cur < 0)
                    return;
#pragma unroll
                for(int o = 16; o > 0; o >>= 1)
                {
                    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
                    mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
                }
                if(lane == 0)
                {
                    atomicMax(&c.bs.hmaxBits[cur], orderedBits(m));
                    atomicMin(&c.bs.hminBits[cur], orderedBits(mn));
                }
                cur = -1;
                m = 0.0;
                mn = 1e300;
            };
            for(int it = 0; it < kHmaxRun; ++it)
            {
                uint32_t const g = base + uint32_t(it) * 32u;
                if(g >= c.n)
                    break;
                uint32_t const p = g + uint32_t(lane);
                int const box = p < c.n ? c.cur.box[p] : -1;
                double const h = p < c.n ? c.cur.h[p] : 0.0;
                int const box0 = __shfl_sync(0xffffffffu, box, 0);
                bool const uniform = __all_sync(0xffffffffu, box == box0 || box < 0);
                if(uniform && box0 == cur)
                {
                    if(box >= 0)
                    {
                        m = fmax(m, h);
                        mn = fmin(mn, h);
                    }
                    continue;
                }
                flush();
                if(uniform)
                {
                    cur = box0;
                    if(box >= 0)
                    {
                        m = h;
                        mn = h;
                    }
                }
                else if(box >= 0)
                {
                    atomicMax(&c.bs.hmaxBits[box], orderedBits(h));
                    atomicMin(&c.bs.hminBits[box], orderedBits(h));
                }
            }
            flush();
        }

        //! Current grid of every box from its largest h (one block): cell counts
        //! clamped to the allocation, edges, stencil shifts; then the prefix of
        //! active cells over boxes (the density pass's work items).
        __global__ void kGrid(DevCtx c, int sup)
        {
            for(uint32_t b = threadIdx.x; b < c.nbox; b += blockDim.x)
            {
                BoxDev& B = c.boxes[b];
                double const h = __longlong_as_double(static_cast<long long>(c.bs.hmaxBits[b]));
                double const hmin = __longlong_as_double(static_cast<long long>(c.bs.hminBits[b]));
                // Two levels pay once the smallest radius is under 1/1.6 of the
                // largest: the level-0 edge then also covers twice the smallest
                // radius (at most 1.25x the largest), so the small-h particles
                // always fit a level-1 sub-cell, also when the range hovers at 2.
                bool const two = B.levelsAlloc == 2 && h > 0.0 && hmin > 0.0 && hmin < 1e300
                                 && 2.0 * cellRadiusDev(sup, hmin) <= kTwoLevelSlack * cellRadiusDev(sup, h);
                if(h > 0.0)
                {
                    double const rc = two ? fmax(cellRadiusDev(sup, h), 2.0 * cellRadiusDev(sup, hmin))
                                          : cellRadiusDev(sup, h);
                    uint32_t cells = 1;
                    for(int a = 0; a < 3; ++a)
                    {
                        double const nd = floor(B.L[a] / rc);
                        int n = nd < 1.0 ? 1 : (nd > double(B.nMax[a]) ? B.nMax[a] : int(nd));
                        B.n[a] = n;
                        B.edge[a] = B.L[a] / double(n);
                        B.edgef[a] = float(B.edge[a]);
                        cells *= uint32_t(n);
                    }
                    B.ncells = cells;
                }
                // Level-1 split: halves on every axis whose edge holds twice the
                // smallest cull radius (finer splits leave too few targets per
                // sub-cell, and a split sized by the smallest h alone misses the
                // bulk of the small-h particles); reduced until the sub-cells fit
                // the allocation.  Two levels need at least two sub-cells.
                int m[3] = {1, 1, 1};
                if(two)
                {
                    double const rmin = cellRadiusDev(sup, hmin);
                    for(int a = 0; a < 3; ++a)
                        m[a] = B.edge[a] >= 2.0 * rmin ? 2 : 1;
                    while(uint64_t(m[0] * m[1] * m[2]) * B.ncells > B.cells1Alloc && m[0] * m[1] * m[2] > 1)
                    {
                        int const a = (m[0] >= m[1] && m[0] >= m[2]) ? 0 : (m[1] >= m[2] ? 1 : 2);
                        --m[a];
                    }
                }
                uint32_t const msub = uint32_t(m[0] * m[1] * m[2]);
                B.levels = two && msub >= 2 ? 2 : 1;
                double e1 = 0.0;
                if(B.levels == 2)
                {
                    e1 = B.edge[0] / double(m[0]);
                    e1 = fmin(e1, B.edge[1] / double(m[1]));
                    e1 = fmin(e1, B.edge[2] / double(m[2]));
                }
                else
                    m[0] = m[1] = m[2] = 1;
#pragma unroll
                for(int a = 0; a < 3; ++a)
                    B.m[a] = m[a];
                B.msub = B.levels == 2 ? msub : 1u;
                B.e1 = e1;
                B.nItems = B.levels == 2 ? B.ncells * (1u + msub) : B.ncells;
                for(int sl = 0; sl < 32; ++sl)
                {
                    int const o[3] = {stencilOff(sl, 0), stencilOff(sl, 1), stencilOff(sl, 2)};
                    bool const used = sl < 27;
                    c.shift32[size_t(b) * 32 + sl] = used ? make_float4(
                                                                float(o[0]) * B.edgef[0],
                                                                float(o[1]) * B.edgef[1],
                                                                float(o[2]) * B.edgef[2],
                                                                0.f)
                                                          : make_float4(0.f, 0.f, 0.f, 0.f);
                    c.shift64[size_t(b) * 32 + sl] = used ? D4{double(o[0]) * B.edge[0], double(o[1]) * B.edge[1],
                                                                double(o[2]) * B.edge[2], 0.0}
                                                          : D4{0.0, 0.0, 0.0, 0.0};
                }
            }
            __syncthreads();
            if(threadIdx.x == 0)
            {
                uint32_t base = 0;
                for(uint32_t b = 0; b < c.nbox; ++b)
                {
                    c.boxes[b].activeBase = base;
                    base += c.boxes[b].nItems;
                }
                *c.activeTotal = base;
            }
        }

        //! Level-1 block range of each level-0 cell of a two-level box: the union
        //! of its sub-cells' sorted ranges, which are contiguous because the
        //! sub-cells of one level-0 cell are numbered together.  One thread per
        //! work item; level-1 items and one-level boxes have nothing to do.
        __global__ void __launch_bounds__(kThreads) kSubBlocks(DevCtx c)
        {
            uint32_t const q = blockIdx.x * blockDim.x + threadIdx.x;
            if(q >= *c.activeTotal)
                return;
            int const box = boxOfWork(c.boxes, c.nbox, q);
            BoxDev const& B = c.boxes[box];
            uint32_t const l = q - B.activeBase;
            if(B.levels != 2 || l >= B.ncells)
                return;
            uint32_t const first = B.cellBase + B.ncellsMax + l * B.msub;
            uint32_t lo = 0xffffffffu, hi = 0;
            for(uint32_t sc = 0; sc < B.msub; ++sc)
            {
                uint32_t const s = c.cells.start[first + sc], e = c.cells.end[first + sc];
                if(e > s)
                {
                    lo = min(lo, s);
                    hi = max(hi, e);
                }
            }
            c.cells.bstart[B.cellBase + l] = hi > 0 ? lo : 0u;
            c.cells.bend[B.cellBase + l] = hi;
        }

        //! Copy of every master column (the state a step call starts from).
        __global__ void kCopyMaster(Master dst, Master src, uint32_t n)
        {
            for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
#pragma unroll
                for(int a = 0; a < 3; ++a)
                {
                    dst.x[a][i] = src.x[a][i];
                    dst.v[a][i] = src.v[a][i];
                    dst.B[a][i] = src.B[a][i];
                }
                dst.u[i] = src.u[i];
                dst.m[i] = src.m[i];
                dst.h[i] = src.h[i];
                dst.rho[i] = src.rho[i];
                dst.psi[i] = src.psi[i];
                dst.id[i] = src.id[i];
                dst.box[i] = src.box[i];
                dst.role[i] = src.role[i];
            }
        }

        //! Sorted-particle range [first, last) of every box's sources: one block
        //! per box takes the min start / max end over the box's non-empty cells.
        __global__ void __launch_bounds__(kThreads) kBoxRange(DevCtx c, uint32_t* range)
        {
            __shared__ uint32_t lo[kThreads], hi[kThreads];
            BoxDev const& B = c.boxes[blockIdx.x];
            uint32_t l = 0xffffffffu, h = 0;
            for(uint32_t lc = threadIdx.x; lc < B.nItems; lc += kThreads)
            {
                uint32_t const cell = B.cellBase + (lc < B.ncells ? lc : B.ncellsMax + (lc - B.ncells));
                uint32_t const s = c.cells.start[cell], e = c.cells.end[cell];
                if(e > s)
                {
                    l = min(l, s);
                    h = max(h, e);
                }
            }
            lo[threadIdx.x] = l;
            hi[threadIdx.x] = h;
            __syncthreads();
            for(int k = kThreads / 2; k > 0; k >>= 1)
            {
                if(int(threadIdx.x) < k)
                {
                    lo[threadIdx.x] = min(lo[threadIdx.x], lo[threadIdx.x + k]);
                    hi[threadIdx.x] = max(hi[threadIdx.x], hi[threadIdx.x + k]);
                }
                __syncthreads();
            }
            if(threadIdx.x == 0)
            {
                range[2 * blockIdx.x] = lo[0] == 0xffffffffu ? 0u : lo[0];
                range[2 * blockIdx.x + 1] = hi[0];
            }
        }

        //! Conserved-sum partials of box blockIdx.x, slice blockIdx.y of kBoxSlices:
        //! each block strides over its box's sorted range in a fixed order.
        __global__ void __launch_bounds__(kThreads)
            kBoxPartials(DevCtx c, PhysArgs pa, uint32_t const* range, double* partials)
        {
            __shared__ double red[kThreads / 32][kDiagWords];
            bool const mhd = pa.physics & SPH_PHYS_MHD;
            uint32_t const first = range[2 * blockIdx.x], last = range[2 * blockIdx.x + 1];
            double acc[kDiagWords];
#pragma unroll
            for(int k = 0; k < kDiagWords; ++k)
                acc[k] = 0.0;
            for(uint32_t p = first + blockIdx.y * kThreads + threadIdx.x; p < last; p += gridDim.y * kThreads)
            {
                if(!isTarget(c.cur.role[p]))
                    continue;
                double const m = c.cur.m[p];
                double v2 = 0.0, B2 = 0.0;
                for(int a = 0; a < 3; ++a)
                {
                    double const va = c.cur.v[a][p];
                    v2 += va * va;
                    acc[3 + a] += m * va;
                    if(mhd)
                        B2 += c.cur.B[a][p] * c.cur.B[a][p];
                }
                acc[0] += 0.5 * m * v2;
                acc[1] += m * c.cur.u[p];
                if(mhd && c.cur.rho[p] > 0.0)
                    acc[2] += 0.5 * m * B2 / (pa.mu0 * c.cur.rho[p]);
                if(mhd && B2 > 0.0)
                {
                    double const e2 = fabs(c.d.divB[p]) * c.cur.h[p] / sqrt(B2);
                    acc[6] += e2;
                    acc[7] += 1.0;
                    acc[8] = fmax(acc[8], e2);
                }
                acc[9] += 1.0;
            }
            int const lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
            for(int k = 0; k < kDiagWords; ++k)
            {
                double const r = (k == 8) ? warpMax(acc[k]) : warpSum(acc[k]);
                if(lane == 0)
                    red[warp][k] = r;
            }
            __syncthreads();
            if(threadIdx.x < kDiagWords)
            {
                int const k = threadIdx.x;
                double r = 0.0;
                for(int w = 0; w < kThreads / 32; ++w)
                    r = (k == 8) ? fmax(r, red[w][k]) : r + red[w][k];
                partials[(size_t(blockIdx.x) * gridDim.y + blockIdx.y) * kDiagWords + k] = r;
            }
        }

        //! Per box: the slices' partials summed in slice order.
        __global__ void kBoxFinal(uint32_t nbox, uint32_t slices, double const* partials, double* out)
        {
            uint32_t const b = blockIdx.x * blockDim.x + threadIdx.x;
            if(b >= nbox)
                return;
            for(int k = 0; k < kDiagWords; ++k)
            {
                double r = 0.0;
                for(uint32_t sl = 0; sl < slices; ++sl)
                {
                    double const v = partials[(size_t(b) * slices + sl) * kDiagWords + k];
                    r = (k == 8) ? fmax(r, v) : r + v;
                }
                out[size_t(b) * kDiagWords + k] = r;
            }
        }
    } // namespace

    uint32_t partialBlocks(uint32_t n)
    {
        uint32_t const b = (n + kThreads - 1) / kThreads;
        return b < 148u * 8u ? b : 148u * 8u;
    }

    void launchDriftKeys(DevCtx const& c, bool drift, cudaStream_t s)
    {
        if(c.n)
        {
            kDriftKeys<<<(c.n + kThreads - 1) / kThreads, kThreads, 0, s>>>(c, drift);
            countLaunches(1);
        }
    }

    void launchCellRanges(DevCtx const& c, uint32_t const* sortedKeys, cudaStream_t s)
    {
        cudaMemsetAsync(c.cells.start, 0, size_t(c.cells.ncells) * 4, s);
        cudaMemsetAsync(c.cells.mid, 0, size_t(c.cells.ncells) * 4, s);
        cudaMemsetAsync(c.cells.end, 0, size_t(c.cells.ncells) * 4, s);
        if(c.n)
        {
            kCellRanges<<<(c.n + kThreads - 1) / kThreads, kThreads, 0, s>>>(sortedKeys, c.n, c.cells);
            countLaunches(1);
        }
    }

    void launchPermute(DevCtx const& c, uint32_t const* perm, PhysArgs const& pa, int precision, cudaStream_t s)
    {
        if(!c.n)
            return;
        unsigned const g = (c.n + kThreads - 1) / kThreads;
        if(precision == SPH_PREC_FP64)
        {
            kPermute<D4, double><<<g, kThreads, 0, s>>>(c, perm, pa, c.r64);
            countLaunches(1);
        }
        else
        {
            kPermute<float4, float><<<g, kThreads, 0, s>>>(c, perm, pa, c.r32);
            countLaunches(1);
        }
    }

    void launchKick(DevCtx const& c, PhysArgs const& pa, bool cfl, cudaStream_t s)
    {
        if(c.n)
        {
            kKick<<<partialBlocks(c.n), kThreads, 0, s>>>(c, pa, cfl);
            countLaunches(1);
        }
        else
            launchFinalize(c, cfl, s);
    }

    void launchFinalize(DevCtx const& c, bool cfl, cudaStream_t s)
    {
        kFinalize<<<1, kThreads, 0, s>>>(c, cfl);
        countLaunches(1);
    }

    void launchUnpermute(uint32_t n, uint32_t const* id, double const* src, double* dst, cudaStream_t s)
    {
        if(n)
        {
            kUnpermute<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(n, id, src, dst);
            countLaunches(1);
        }
    }

    void launchUnpermuteInt(uint32_t n, uint32_t const* id, uint32_t const* src, int32_t* dst, cudaStream_t s)
    {
        if(n)
        {
            kUnpermuteInt<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(n, id, src, dst);
            countLaunches(1);
        }
    }

    void launchBoxReduce(DevCtx const& c, PhysArgs const& pa, double* out, double* scratch, cudaStream_t s)
    {
        // scratch: 2*nbox range words (as doubles' storage) + nbox*slices*kDiagWords partials
        uint32_t const slices = c.nbox == 1 ? 256u : (c.nbox < 64 ? 16u : 2u);
        uint32_t* range = reinterpret_cast<uint32_t*>(scratch);
        double* partials = scratch + c.nbox;
        kBoxRange<<<c.nbox, kThreads, 0, s>>>(c, range);
        countLaunches(1);
        kBoxPartials<<<dim3(c.nbox, slices), kThreads, 0, s>>>(c, pa, range, partials);
        countLaunches(1);
        kBoxFinal<<<(c.nbox + 127) / 128, 128, 0, s>>>(c.nbox, slices, partials, out);
        countLaunches(1);
    }

    size_t boxReduceScratchDoubles(uint32_t nbox)
    {
        uint32_t const slices = nbox == 1 ? 256u : (nbox < 64 ? 16u : 2u);
        return size_t(nbox) + size_t(nbox) * slices * kDiagWords;
    }

    void launchGatherSpecies(
        uint32_t n,
        uint32_t const* id,
        uint32_t off,
        uint32_t cnt,
        double const* src,
        double dflt,
        double* master,
        uint32_t* badCount,
        cudaStream_t s)
    {
        if(n)
        {
            kGatherSpecies<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(
                n, id, off, cnt, src, dflt, master, badCount);
            countLaunches(1);
        }
    }

    void launchGatherSpeciesInt(
        uint32_t n,
        uint32_t const* id,
        uint32_t off,
        uint32_t cnt,
        int32_t const* src,
        int32_t* master,
        cudaStream_t s)
    {
        if(n)
        {
            kGatherSpeciesInt<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(n, id, off, cnt, src, master);
            countLaunches(1);
        }
    }

    void launchSubBlocks(DevCtx const& c, uint32_t totalCells, cudaStream_t s)
    {
        if(totalCells)
        {
            kSubBlocks<<<(totalCells + kThreads - 1) / kThreads, kThreads, 0, s>>>(c);
            countLaunches(1);
        }
    }

    void launchGridUpdate(DevCtx const& c, int support, cudaStream_t s)
    {
        cudaMemsetAsync(c.bs.hmaxBits, 0, sizeof(unsigned long long) * c.nbox, s);
        cudaMemsetAsync(c.bs.hminBits, 0xff, sizeof(unsigned long long) * c.nbox, s);
        if(c.n)
        {
            uint32_t const perBlock = uint32_t(kThreads / 32) * 32u * uint32_t(kHmaxRun);
            kBoxHmax<<<(c.n + perBlock - 1) / perBlock, kThreads, 0, s>>>(c);
            countLaunches(1);
        }
        kGrid<<<1, 256, 0, s>>>(c, support);
        countLaunches(1);
    }

    void launchCopyMaster(Master const& dst, Master const& src, uint32_t n, cudaStream_t s)
    {
        if(n)
        {
            unsigned const blocks = unsigned(std::min<uint32_t>((n + 255) / 256, 148u * 16u));
            kCopyMaster<<<blocks, 256, 0, s>>>(dst, src, n);
            countLaunches(1);
        }
    }

    void launchFill(double* p, size_t n, double v, cudaStream_t s)
    {
        if(n)
        {
            kFill<<<unsigned((n + 255) / 256), 256, 0, s>>>(p, n, v);
            countLaunches(1);
        }
    }
} // namespace sph
