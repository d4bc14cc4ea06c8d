/* Oracle harness around the reference's own SPH physics headers.
 *
 * TEST INFRASTRUCTURE ONLY: this file is compiled (by oracle/Makefile, target
 * `ref`) against the unmodified reference headers where they lie in the
 * reference checkout, plus the host-only shims in oracle/ref_shim/ that stand
 * in for alpaka.  Output goes to oracle/_ref/.  Only tests/, the smoke check
 * and bench.py's CPU baseline may load the result.
 *
 * Compiled from the reference (not restated here):
 *   - CubicSplineKernel::{W,dWdr,gradWScalar}  include/spearhed/sph/CubicSplineKernel.hpp:49-140
 *   - QuinticSplineKernel::{W,dWdr,gradWScalar} include/spearhed/sph/QuinticSplineKernel.hpp:47-164
 *   - pressure / soundSpeed                     include/spearhed/sph/EquationOfState.hpp:32-47
 *   - DensityInitSelf, AccumulateDensity        include/spearhed/particles/density/DensitySummation.hpp:50-94
 *   - ZeroDerivatives, HydroInteraction         include/spearhed/sph/HydroForces.hpp:51-176
 *   - PairContext                               spmacc/particles/algorithms/InteractionContext.hpp:52-65
 *
 * Restated here (the reference's version needs alpaka):
 *   - the per-pair sweep of interactWithNeighbourFrame
 *     (spmacc/particles/algorithms/ParticleParticleInteraction.hpp:236-313):
 *     staged position = pos_j + shift, d = own - staged in x, y, z order,
 *     r2 accumulated in the same order, strict cull r2 < radius^2,
 *     invR = rsqrt(r2) and r = r2 * invR only when r2 > 0 (else both 0),
 *     isSelf = same particle and same image; stage() once per neighbour,
 *     prepare() once per own particle, accumulators seeded from the
 *     particle's current value and stored once.
 * The candidate list (which j to sweep for which i) is the caller's; for the
 * reference's semantics it must be a superset of the accepted pairs, which the
 * cull then filters exactly as the reference does.
 */
#include <spearhed/particles/density/DensitySummation.hpp>
#include <spearhed/sph/CubicSplineKernel.hpp>
#include <spearhed/sph/EquationOfState.hpp>
#include <spearhed/sph/HydroForces.hpp>
#include <spearhed/sph/QuinticSplineKernel.hpp>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <limits>
#include <vector>

#ifdef _OPENMP
#    include <omp.h>
#endif

#ifndef REF_SUFFIX
#    define REF_SUFFIX f32
#endif
#define REF_CAT2(a, b) a##_##b
#define REF_CAT(a, b) REF_CAT2(a, b)
#define REF_FN(name) REF_CAT(name, REF_SUFFIX)

namespace
{
    using T = spearhed::Real;
    using CS = spearhed::CS;
    namespace st = spearhed::tags;
    namespace pt = pmacc::spearhed::tags;

    //! Three-component view onto plain arrays, indexed by the reference's axis tags.
    struct Axes
    {
        T* p;
        T& operator[](pt::x_t) const
        {
            return p[0];
        }
        T& operator[](pt::y_t) const
        {
            return p[1];
        }
        T& operator[](pt::z_t) const
        {
            return p[2];
        }
    };

    //! A particle record addressed by the reference's attribute tags.  Plays the
    //! part of the own-read sub-record, the staged neighbour record and the
    //! accumulator sub-record; every field is plain storage.
    struct Rec
    {
        T mass = 0, h = 0, rho = 0, u = 0, dudt = 0, pOverRho2 = 0;
        T vel[3] = {0, 0, 0};
        T dvdt[3] = {0, 0, 0};

        T& operator[](st::mass_t)
        {
            return mass;
        }
        T const& operator[](st::mass_t) const
        {
            return mass;
        }
        T& operator[](st::smoothingLength_t)
        {
            return h;
        }
        T const& operator[](st::smoothingLength_t) const
        {
            return h;
        }
        T& operator[](st::density_t)
        {
            return rho;
        }
        T const& operator[](st::density_t) const
        {
            return rho;
        }
        T& operator[](st::internalEnergy_t)
        {
            return u;
        }
        T const& operator[](st::internalEnergy_t) const
        {
            return u;
        }
        T& operator[](st::dudt_t)
        {
            return dudt;
        }
        T const& operator[](st::dudt_t) const
        {
            return dudt;
        }
        T& operator[](st::pOverRho2_t)
        {
            return pOverRho2;
        }
        T const& operator[](st::pOverRho2_t) const
        {
            return pOverRho2;
        }
        Axes operator[](st::vel_t)
        {
            return Axes{vel};
        }
        Axes operator[](st::vel_t) const
        {
            return Axes{const_cast<T*>(vel)};
        }
        Axes operator[](st::dvdt_t)
        {
            return Axes{dvdt};
        }
        Axes operator[](st::dvdt_t) const
        {
            return Axes{const_cast<T*>(dvdt)};
        }
    };

    //! Staged-record handle: stage() takes its destination by value.
    struct RecRef
    {
        Rec* r;
        template<typename Tag>
        decltype(auto) operator[](Tag t) const
        {
            return (*r)[t];
        }
    };

    struct Worker
    {
    };

    using Vec = pmacc::spearhed::Vec<CS, pmacc::spearhed::ValueStorage<CS>>;

    //! Geometry of one candidate pair, following the reference sweep (see file header).
    inline bool pairContext(
        T const* own,
        T const* nb,
        T const* shift,
        T radius2,
        bool sameParticle,
        pmacc::spearhed::PairContext<CS>& ctx)
    {
        Vec rVec;
        T r2{0};
        int a = 0;
        pmacc::spearhed::for_each_tag<CS>(
            [&](auto tag)
            {
                T const staged = nb[a] + (shift ? shift[a] : T{0});
                T const d = own[a] - staged;
                rVec[tag] = d;
                r2 += d * d;
                ++a;
            });
        if(!(r2 < radius2))
            return false;
        T invR{0};
        T r{0};
        if(r2 > T{0})
        {
            invR = pmacc::math::rsqrt(r2);
            r = r2 * invR;
        }
        bool const zeroShift = !shift || (shift[0] == T{0} && shift[1] == T{0} && shift[2] == T{0});
        ctx = pmacc::spearhed::PairContext<CS>{rVec, r2, r, invR, sameParticle && zeroShift};
        return true;
    }

    template<typename K>
    void densityImpl(
        int ntarget,
        int const* targets,
        T const* pos,
        T const* mass,
        T const* h,
        int64_t const* candOff,
        int const* candIdx,
        T const* candShift,
        T radius,
        T* rhoOut)
    {
        T const radius2 = radius * radius;
        spearhed::DensityInitSelf<K> initSelf{};
        spearhed::AccumulateDensity<K> fn{};
        Worker w;
        for(int t = 0; t < ntarget; ++t)
        {
            int const i = targets[t];
            Rec own;
            own.mass = mass[i];
            own.h = h[i];
            // DensityInitSelf seeds the accumulator with the self term.
            initSelf(w, own);
            for(int64_t c = candOff[t]; c < candOff[t + 1]; ++c)
            {
                int const j = candIdx[c];
                pmacc::spearhed::PairContext<CS> ctx{};
                if(!pairContext(&pos[3 * i], &pos[3 * j], candShift ? &candShift[3 * c] : nullptr, radius2, i == j, ctx))
                    continue;
                Rec nb;
                nb.mass = mass[j];
                fn(w, own, nb, ctx, own);
            }
            rhoOut[t] = own.rho;
        }
    }

    template<typename K>
    void hydroImpl(
        int ntarget,
        int const* targets,
        T const* pos,
        T const* mass,
        T const* h,
        T const* rho,
        T const* u,
        T const* vel,
        int64_t const* candOff,
        int const* candIdx,
        T const* candShift,
        T gamma,
        T radius,
        T* dvdtOut,
        T* dudtOut)
    {
        T const radius2 = radius * radius;
        spearhed::HydroInteraction<K> fn{gamma};
        spearhed::ZeroDerivatives zero{};
        Worker w;
        for(int t = 0; t < ntarget; ++t)
        {
            int const i = targets[t];
            Rec own;
            own.mass = mass[i];
            own.h = h[i];
            own.rho = rho[i];
            own.u = u[i];
            for(int a = 0; a < 3; ++a)
                own.vel[a] = vel[3 * i + a];
            zero(w, own);
            auto const prep = fn.prepare(own);
            for(int64_t c = candOff[t]; c < candOff[t + 1]; ++c)
            {
                int const j = candIdx[c];
                pmacc::spearhed::PairContext<CS> ctx{};
                if(!pairContext(&pos[3 * i], &pos[3 * j], candShift ? &candShift[3 * c] : nullptr, radius2, i == j, ctx))
                    continue;
                Rec src;
                src.mass = mass[j];
                src.h = h[j];
                src.rho = rho[j];
                src.u = u[j];
                for(int a = 0; a < 3; ++a)
                    src.vel[a] = vel[3 * j + a];
                Rec staged;
                fn.stage(src, RecRef{&staged});
                fn(w, own, prep, staged, ctx, own);
            }
            for(int a = 0; a < 3; ++a)
                dvdtOut[3 * t + a] = own.dvdt[a];
            dudtOut[t] = own.dudt;
        }
    }
} // namespace


namespace
{
    // ---------------------------------------------------------------------
    // The reference's region/frame pair engine, restated for the CPU baseline
    // (the reference's own version is an alpaka kernel):
    //   - particles live in regions (axis-aligned boxes); a region holds its
    //     particles in frames of 64 slots (param/memory.param:35, numFrameSlots);
    //   - region bounds are the tight AABB of their particles
    //     (spmacc/particles/regions/RegionBoundsUpdate.hpp:63-103);
    //   - the neighbour regions of a target region are the regions whose AABB
    //     intersects the target AABB expanded by the radius
    //     (NeighbourRegions.hpp:78-133, AABB.hpp:79-119);
    //   - for each target frame, each neighbour region and each of its frames,
    //     the 64 slots are staged with the origin shift (dead slots get the
    //     sentinel max/4) and swept against every live own slot
    //     (ParticleParticleInteraction.hpp:236-313, :483-612).
    // ---------------------------------------------------------------------
    constexpr int kSlots = 64;

    struct Region
    {
        T origin[3];
        T lo[3], hi[3]; // tight bounds, absolute
        std::vector<int> frames; // frame ids
    };

    struct Frame
    {
        int region;
        int live;
        int idx[kSlots];
    };

    struct RegionSet
    {
        std::vector<Region> regions;
        std::vector<Frame> frames;
        std::vector<std::vector<int>> nbRegions;
    };

    RegionSet makeRegions(int n, T const* pos, T const* boxLo, T const* boxHi, T side, T radius)
    {
        RegionSet rs;
        int nr[3];
        for(int a = 0; a < 3; ++a)
            nr[a] = std::max(1, int((boxHi[a] - boxLo[a]) / side));
        rs.regions.resize(size_t(nr[0]) * nr[1] * nr[2]);
        std::vector<std::vector<int>> members(rs.regions.size());
        for(int i = 0; i < n; ++i)
        {
            int c[3];
            for(int a = 0; a < 3; ++a)
            {
                T const e = (boxHi[a] - boxLo[a]) / T(nr[a]);
                c[a] = std::min(nr[a] - 1, std::max(0, int((pos[3 * i + a] - boxLo[a]) / e)));
            }
            members[(size_t(c[2]) * nr[1] + c[1]) * nr[0] + c[0]].push_back(i);
        }
        for(size_t r = 0; r < rs.regions.size(); ++r)
        {
            Region& R = rs.regions[r];
            size_t const cz = r / (size_t(nr[0]) * nr[1]), cy = (r / nr[0]) % nr[1], cx = r % nr[0];
            size_t const cc[3] = {cx, cy, cz};
            for(int a = 0; a < 3; ++a)
            {
                T const e = (boxHi[a] - boxLo[a]) / T(nr[a]);
                R.origin[a] = boxLo[a] + T(cc[a]) * e;
                R.lo[a] = std::numeric_limits<T>::max();
                R.hi[a] = std::numeric_limits<T>::lowest();
            }
            for(size_t k = 0; k < members[r].size(); ++k)
            {
                if(k % kSlots == 0)
                {
                    Frame f{};
                    f.region = int(r);
                    f.live = 0;
                    rs.frames.push_back(f);
                    R.frames.push_back(int(rs.frames.size()) - 1);
                }
                Frame& f = rs.frames.back();
                int const i = members[r][k];
                f.idx[f.live++] = i;
                for(int a = 0; a < 3; ++a)
                {
                    R.lo[a] = std::min(R.lo[a], pos[3 * i + a]);
                    R.hi[a] = std::max(R.hi[a], pos[3 * i + a]);
                }
            }
        }
        rs.nbRegions.resize(rs.regions.size());
#pragma omp parallel for schedule(dynamic, 64)
        for(size_t t = 0; t < rs.regions.size(); ++t)
        {
            Region const& A = rs.regions[t];
            if(A.frames.empty())
                continue;
            for(size_t q = 0; q < rs.regions.size(); ++q)
            {
                Region const& B = rs.regions[q];
                if(B.frames.empty())
                    continue;
                bool hit = true;
                for(int a = 0; a < 3; ++a)
                    if((A.lo[a] - radius) > B.hi[a] || (A.hi[a] + radius) < B.lo[a])
                        hit = false;
                if(hit)
                    rs.nbRegions[t].push_back(int(q));
            }
        }
        return rs;
    }

    //! One pass over target frame tf: stage each neighbour frame, sweep, call fn.
    //! Returns the accepted non-self pairs.
    template<typename Fn, typename Stage, typename Own, typename Call>
    int64_t sweepFrame(
        RegionSet const& rs,
        int tf,
        T const* pos,
        T radius2,
        Own&& loadOwn,
        Stage&& stage,
        Call&& call)
    {
        Frame const& F = rs.frames[tf];
        Region const& RA = rs.regions[F.region];
        T ownRel[kSlots][3];
        for(int s = 0; s < F.live; ++s)
        {
            for(int a = 0; a < 3; ++a)
                ownRel[s][a] = pos[3 * F.idx[s] + a] - RA.origin[a];
            loadOwn(s, F.idx[s]);
        }
        T sentinel = std::numeric_limits<T>::max() / T{4};
        T staged[kSlots][3];
        int64_t pairs = 0;
        for(int nr : rs.nbRegions[F.region])
        {
            Region const& RB = rs.regions[nr];
            T shift[3];
            for(int a = 0; a < 3; ++a)
                shift[a] = RB.origin[a] - RA.origin[a];
            for(int gf : RB.frames)
            {
                Frame const& G = rs.frames[gf];
                for(int s = 0; s < kSlots; ++s)
                {
                    if(s < G.live)
                    {
                        stage(s, G.idx[s]);
                        for(int a = 0; a < 3; ++a)
                            staged[s][a] = (pos[3 * G.idx[s] + a] - RB.origin[a]) + shift[a];
                    }
                    else
                        for(int a = 0; a < 3; ++a)
                            staged[s][a] = sentinel;
                }
                bool const selfFrame = gf == tf;
                for(int i = 0; i < F.live; ++i)
                    for(int j = 0; j < kSlots; ++j)
                    {
                        T r2{0};
                        T d[3];
                        for(int a = 0; a < 3; ++a)
                        {
                            d[a] = ownRel[i][a] - staged[j][a];
                            r2 += d[a] * d[a];
                        }
                        if(r2 < radius2)
                        {
                            T invR{0}, r{0};
                            if(r2 > T{0})
                            {
                                invR = pmacc::math::rsqrt(r2);
                                r = r2 * invR;
                            }
                            bool const isSelf = selfFrame && j == i;
                            pairs += isSelf ? 0 : 1;
                            call(i, j, d, r2, r, invR, isSelf);
                        }
                    }
            }
        }
        return pairs;
    }
} // namespace

extern "C"
{
    T REF_FN(ref_cubic_W)(T r, T h)
    {
        return spearhed::CubicSplineKernel::W(r, h);
    }
    T REF_FN(ref_cubic_dWdr)(T r, T h)
    {
        return spearhed::CubicSplineKernel::dWdr(r, h);
    }
    T REF_FN(ref_cubic_gradWScalar)(T r, T invR, T h)
    {
        return spearhed::CubicSplineKernel::gradWScalar(r, invR, h);
    }
    T REF_FN(ref_quintic_W)(T r, T h)
    {
        return spearhed::QuinticSplineKernel::W(r, h);
    }
    T REF_FN(ref_quintic_dWdr)(T r, T h)
    {
        return spearhed::QuinticSplineKernel::dWdr(r, h);
    }
    T REF_FN(ref_quintic_gradWScalar)(T r, T invR, T h)
    {
        return spearhed::QuinticSplineKernel::gradWScalar(r, invR, h);
    }
    T REF_FN(ref_pressure)(T gamma, T rho, T u)
    {
        return spearhed::pressure(gamma, rho, u);
    }
    T REF_FN(ref_sound_speed)(T gamma, T p, T rho)
    {
        return spearhed::soundSpeed(gamma, p, rho);
    }


    /** CPU baseline: the reference's density pass then hydro pass (its own
     *  functors) over target frames of a region/frame decomposition of the
     *  input (regions of edge `side`), processed in order until `limit_s`
     *  seconds have passed or every frame is done; OpenMP over target frames.
     *  Returns accepted non-self pairs of each pass, the frames processed,
     *  and the seconds of the two passes. */
    int REF_FN(ref_region_bench)(
        int kernel,
        int n,
        T const* pos,
        T const* mass,
        T const* h,
        T* rho,
        T const* u,
        T const* vel,
        T const* boxLo,
        T const* boxHi,
        T side,
        T radius,
        T gamma,
        double limit_s,
        int64_t* pairsDensity,
        int64_t* pairsHydro,
        int* framesDone,
        int* framesTotal,
        double* seconds)
    {
        if(kernel != 0)
            return 9;
        using K = spearhed::CubicSplineKernel;
        RegionSet const rs = makeRegions(n, pos, boxLo, boxHi, side, radius);
        T const radius2 = radius * radius;
        int const nf = int(rs.frames.size());
        *framesTotal = nf;
        int64_t pd = 0, ph = 0;
        int done = 0;
        auto const t0 = std::chrono::steady_clock::now();
        int const batch = 256;
        while(done < nf)
        {
            int const end = std::min(nf, done + batch);
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : pd, ph)
            for(int tf = done; tf < end; ++tf)
            {
                Worker w;
                // density pass: DensityInitSelf + AccumulateDensity
                spearhed::DensityInitSelf<K> initSelf{};
                spearhed::AccumulateDensity<K> dfn{};
                Rec own[kSlots];
                Rec nb[kSlots];
                Frame const& F = rs.frames[tf];
                pd += sweepFrame<void>(
                    rs,
                    tf,
                    pos,
                    radius2,
                    [&](int s, int i)
                    {
                        own[s] = Rec{};
                        own[s].mass = mass[i];
                        own[s].h = h[i];
                        initSelf(w, own[s]);
                    },
                    [&](int s, int j) { nb[s].mass = mass[j]; },
                    [&](int i, int j, T const* d, T r2, T r, T invR, bool self)
                    {
                        Vec rv;
                        rv[pt::x_t{}] = d[0];
                        rv[pt::y_t{}] = d[1];
                        rv[pt::z_t{}] = d[2];
                        pmacc::spearhed::PairContext<CS> const ctx{rv, r2, r, invR, self};
                        dfn(w, own[i], nb[j], ctx, own[i]);
                    });
                for(int s = 0; s < F.live; ++s)
                    rho[F.idx[s]] = own[s].rho;
            }
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : pd, ph)
            for(int tf = done; tf < end; ++tf)
            {
                Worker w;
                spearhed::HydroInteraction<K> hfn{gamma};
                spearhed::ZeroDerivatives zero{};
                Rec own[kSlots];
                Rec staged[kSlots];
                decltype(hfn.prepare(own[0])) prep[kSlots];
                ph += sweepFrame<void>(
                    rs,
                    tf,
                    pos,
                    radius2,
                    [&](int s, int i)
                    {
                        own[s] = Rec{};
                        own[s].mass = mass[i];
                        own[s].h = h[i];
                        own[s].rho = rho[i];
                        own[s].u = u[i];
                        for(int a = 0; a < 3; ++a)
                            own[s].vel[a] = vel[3 * i + a];
                        zero(w, own[s]);
                        prep[s] = hfn.prepare(own[s]);
                    },
                    [&](int s, int j)
                    {
                        Rec src;
                        src.mass = mass[j];
                        src.h = h[j];
                        src.rho = rho[j];
                        src.u = u[j];
                        for(int a = 0; a < 3; ++a)
                            src.vel[a] = vel[3 * j + a];
                        hfn.stage(src, RecRef{&staged[s]});
                    },
                    [&](int i, int j, T const* d, T r2, T r, T invR, bool self)
                    {
                        Vec rv;
                        rv[pt::x_t{}] = d[0];
                        rv[pt::y_t{}] = d[1];
                        rv[pt::z_t{}] = d[2];
                        pmacc::spearhed::PairContext<CS> const ctx{rv, r2, r, invR, self};
                        hfn(w, own[i], prep[i], staged[j], ctx, own[i]);
                    });
            }
            done = end;
            double const el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if(el > limit_s)
                break;
        }
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        *pairsDensity = pd;
        *pairsHydro = ph;
        *framesDone = done;
        return 0;
    }

    //! kernel: 0 = cubic spline (support 2h), 1 = quintic spline (support 3h).
    void REF_FN(ref_density)(
        int kernel,
        int ntarget,
        int const* targets,
        T const* pos,
        T const* mass,
        T const* h,
        int64_t const* candOff,
        int const* candIdx,
        T const* candShift,
        T radius,
        T* rhoOut)
    {
        if(kernel == 1)
            densityImpl<spearhed::QuinticSplineKernel>(
                ntarget, targets, pos, mass, h, candOff, candIdx, candShift, radius, rhoOut);
        else
            densityImpl<spearhed::CubicSplineKernel>(
                ntarget, targets, pos, mass, h, candOff, candIdx, candShift, radius, rhoOut);
    }

    void REF_FN(ref_hydro)(
        int kernel,
        int ntarget,
        int const* targets,
        T const* pos,
        T const* mass,
        T const* h,
        T const* rho,
        T const* u,
        T const* vel,
        int64_t const* candOff,
        int const* candIdx,
        T const* candShift,
        T gamma,
        T radius,
        T* dvdtOut,
        T* dudtOut)
    {
        if(kernel == 1)
            hydroImpl<spearhed::QuinticSplineKernel>(
                ntarget, targets, pos, mass, h, rho, u, vel, candOff, candIdx, candShift, gamma, radius, dvdtOut, dudtOut);
        else
            hydroImpl<spearhed::CubicSplineKernel>(
                ntarget, targets, pos, mass, h, rho, u, vel, candOff, candIdx, candShift, gamma, radius, dvdtOut, dudtOut);
    }
}
