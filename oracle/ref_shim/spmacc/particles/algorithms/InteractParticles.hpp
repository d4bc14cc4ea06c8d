/* Declarations only: the reference's stage functors (UpdateDensity,
 * UpdateHydroForces) name these in uninstantiated template bodies.  The
 * oracle never calls the stage functors; it drives the pair functors itself. */
#pragma once
#include <spmacc/particles/algorithms/InteractionContext.hpp>
namespace pmacc::spearhed
{
    namespace roles
    {
        struct Source
        {
        };
    } // namespace roles
    template<typename T>
    concept IsNeighbourBundle = true;
    struct UnusedSender
    {
        template<typename T>
        friend UnusedSender operator|(UnusedSender, T&&)
        {
            return {};
        }
    };
    template<typename... A>
    UnusedSender interact(A&&...)
    {
        return {};
    }
} // namespace pmacc::spearhed
namespace caravan::alpaka
{
    template<typename... A>
    pmacc::spearhed::UnusedSender sequence(A&&...)
    {
        return {};
    }
} // namespace caravan::alpaka
