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

#include <cstdint>

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
