/* Compile-time parameters for building the reference's physics headers on
 * the host.  Mirrors the names the reference's param files export
 * (Real, CS, T_dt, dt, h0, gamma_eos) with the 3D defaults; Real is chosen
 * per translation unit through SPH_REF_REAL (float or double). */
#pragma once
#include <cstdint>
#include <spmacc/topology/Cartesian.hpp>
#include <spmacc/topology/CoordinateSystem.hpp>

#ifndef SPH_REF_REAL
#    define SPH_REF_REAL float
#endif

namespace spearhed
{
    using Real = SPH_REF_REAL;
    using T_Dim = pmacc::spearhed::T_Dim;
    constexpr T_Dim simDim = 3;
    using CS = pmacc::spearhed::Cartesian<Real, simDim>;
    using T_dt = Real;
    constexpr T_dt dt = T_dt{0.01f};
    constexpr Real h0 = Real{0.05f};
    constexpr Real gamma_eos = Real{5} / Real{3};
    constexpr Real cflFactor = Real{0.3f};
} // namespace spearhed
