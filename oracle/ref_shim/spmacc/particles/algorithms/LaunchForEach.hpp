/* Declarations only (see InteractParticles.hpp in this directory). */
#pragma once
#include <spmacc/particles/algorithms/InteractParticles.hpp>
namespace pmacc::spearhed
{
    namespace levels
    {
        inline constexpr int particle = 0;
    } // namespace levels
    template<typename... A>
    UnusedSender launchForEach(A&&...)
    {
        return {};
    }
} // namespace pmacc::spearhed
