/* Host-only stand-in for the reference's alpaka-backed math functions
 * (packages/pmacc/include/pmacc/math/functions/Pow.hpp): pow. */
#pragma once
#include "Root.hpp"
namespace pmacc::math
{
    using std::pow;
} // namespace pmacc::math
