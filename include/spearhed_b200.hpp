/* spearhed_b200.hpp — header-only C++ shim over the C ABI (spearhed_b200.h)
 * that keeps the reference's stage-functor call shapes:
 *
 *   reference (include/spearhed/control/Simulation.x.cpp:278-296)      this shim
 *   UpdateDensity<K>{}(bundle, target, index, h0)                      UpdateDensity<K>{}(ctx)
 *   UpdateHydroForces<K>{gamma}(bundle, target, index, h0)             UpdateHydroForces<K>{}(ctx)
 *   launchForEach(..., EulerIntegrate{}, dt) after the passes          runOneStep(ctx, n, dt)
 *
 * The neighbour bundle, target buffer and frame index of the reference are
 * owned by the context here (cell-sorted arrays rebuilt on the device), so the
 * functors take the context only.  The kernel tag is checked against the
 * context's run-time kernel.  Arbitrary user functors cannot cross a C ABI;
 * the built-in physics are selected by SphParams.physics.
 *
 * Errors: the C ABI returns status codes; this shim turns them into
 * std::runtime_error, as the reference's host code throws
 * (PMACC_VERIFY_MSG / std::runtime_error, Simulation.x.cpp:204-206).
 */
#pragma once

#include "spearhed_b200.h"

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace spearhed_b200
{
    //! Kernel tags with the reference's static supportRadius (SphKernel concept,
    //! include/spearhed/sph/SphKernel.hpp:45-51).
    struct CubicSplineKernel
    {
        static constexpr int id = SPH_KERNEL_CUBIC;
        static constexpr int supportRadius = 2;
    };
    struct QuinticSplineKernel
    {
        static constexpr int id = SPH_KERNEL_QUINTIC;
        static constexpr int supportRadius = 3;
    };
    struct WendlandC2Kernel
    {
        static constexpr int id = SPH_KERNEL_WENDLAND_C2;
        static constexpr int supportRadius = 2;
    };

    inline void check(int status, char const* what)
    {
        if(status != SPH_OK)
            throw std::runtime_error(std::string(what) + ": " + sph_last_error_string());
    }

    //! Owns one sph_ctx (one CUDA stream, library-owned device memory).
    class Context
    {
    public:
        explicit Context(SphParams const& p) : params_(p)
        {
            check(sph_create(&p, &ctx_), "sph_create");
        }
        Context(SphParams const& p, std::vector<SphBox> const& boxes) : Context(p)
        {
            check(sph_set_boxes(ctx_, int32_t(boxes.size()), boxes.data()), "sph_set_boxes");
        }
        Context(Context const&) = delete;
        Context& operator=(Context const&) = delete;
        Context(Context&& o) noexcept : ctx_(std::exchange(o.ctx_, nullptr)), params_(o.params_)
        {
        }
        ~Context()
        {
            if(ctx_)
                sph_destroy(ctx_);
        }

        sph_ctx* get() const
        {
            return ctx_;
        }
        SphParams const& params() const
        {
            return params_;
        }

        //! InitParticles for one species (its roles follow speciesDefinition.param:56-88).
        void setSpecies(int32_t species, int64_t n, SphSoAView const& view, uint32_t roles = 0)
        {
            if(roles == 0)
                roles = species == SPH_SPECIES_BOUNDARY ? SPH_ROLES_BOUNDARY
                                                        : (species == SPH_SPECIES_TRACER ? SPH_ROLES_TRACER
                                                                                          : SPH_ROLES_DEFAULT);
            check(sph_set_species(ctx_, species, roles, n, &view), "sph_set_species");
        }
        void getSpecies(int32_t species, SphSoAView& view)
        {
            check(sph_get_species(ctx_, species, &view), "sph_get_species");
        }
        SphDiag reduce()
        {
            SphDiag d{};
            check(sph_reduce(ctx_, &d), "sph_reduce");
            return d;
        }
        //! Picks the fastest launch shapes on the current particles (state kept).
        SphTuning autotune(int32_t stepsPerTrial = 2)
        {
            SphTuning t{};
            check(sph_autotune(ctx_, stepsPerTrial, &t), "sph_autotune");
            return t;
        }

    private:
        sph_ctx* ctx_ = nullptr;
        SphParams params_;
    };

    template<typename K>
    void requireKernel(Context const& ctx)
    {
        if(ctx.params().kernel != K::id)
            throw std::invalid_argument("stage functor kernel differs from the context's SphParams.kernel");
    }

    //! UpdateDensity<K> (include/spearhed/particles/density/DensitySummation.hpp:104-138):
    //! self term m_i W(0, h_i) plus the gather over accepted neighbours.
    template<typename K>
    struct UpdateDensity
    {
        void operator()(Context& ctx) const
        {
            requireKernel<K>(ctx);
            check(sph_density(ctx.get()), "UpdateDensity");
        }
    };

    //! UpdateHydroForces<K> (include/spearhed/sph/HydroForces.hpp:183-214):
    //! zeroed derivatives, then the symmetric pressure force and P dV work (plus
    //! viscosity / SPMHD when SphParams.physics asks for them).
    template<typename K>
    struct UpdateHydroForces
    {
        void operator()(Context& ctx) const
        {
            requireKernel<K>(ctx);
            check(sph_hydro(ctx.get()), "UpdateHydroForces");
        }
    };

    //! Simulation::runOneStep repeated n times (control/Simulation.x.cpp:196-310).
    inline void runOneStep(Context& ctx, int32_t n = 1, double dt = 0.0)
    {
        check(sph_step(ctx.get(), n, dt), "runOneStep");
    }
} // namespace spearhed_b200
