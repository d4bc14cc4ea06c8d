/* Host-only stand-in for the reference's alpaka-backed math functions
 * (packages/pmacc/include/pmacc/math/functions/Root.hpp): sqrt and rsqrt. */
#pragma once
#include <cmath>
namespace pmacc::math
{
    using std::sqrt;
    //! 1/sqrt(x) in the argument's own precision: the same expression oracle.cpp uses for
    //! invR (alpaka's Rsqrt, which pmacc::math::rsqrt forwards to, is not vendored).
    template<typename T>
    inline T rsqrt(T x)
    {
        return T(1) / std::sqrt(x);
    }
} // namespace pmacc::math
