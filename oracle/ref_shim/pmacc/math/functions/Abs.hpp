/* Host-only stand-in for the reference's alpaka-backed math functions. */
#pragma once
#include <cmath>
namespace pmacc::math
{
    using std::abs;
    using std::pow;
    using std::sqrt;
    //! 1/sqrt(x) in the argument's own precision (the oracle's rsqrt, see oracle.hpp).
    template<typename T>
    inline T rsqrt(T x)
    {
        return T(1) / std::sqrt(x);
    }
} // namespace pmacc::math
