/* Host-only stand-in for the reference's alpaka-backed math functions
 * (packages/pmacc/include/pmacc/math/functions/Abs.hpp): abs. */
#pragma once
#include "Root.hpp"
namespace pmacc::math
{
    using std::abs;
} // namespace pmacc::math
