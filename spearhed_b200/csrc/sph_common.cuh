// Shared device definitions of the B200 SPH step: box/cell-grid descriptors,
// SPH kernel functions, equation of state, compensated accumulation.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/spearhed_b200.h"

namespace sph
{
    // ------------------------------------------------------------------ grid
    //! One box of the run: the cell grid the neighbour search bins it into.
    //! Cell edge >= the cull radius on every axis, so the 27-cell stencil holds
    //! every neighbour (and, on periodic axes, every image within the radius).
    struct BoxDev
    {
        double lo[3];
        double L[3];
        double edge[3];
        float edgef[3];
        int32_t n[3];
        int32_t periodic[3];
        uint32_t cellBase; //!< first global cell id of this box (in the allocation)
        uint32_t ncells;   //!< cells of the current grid (n[0] n[1] n[2])
        double hcap;       //!< cap on adaptive h (params.h_max, else what the periodic axes admit)
        int32_t nMax[3];   //!< allocated cells per axis: the current grid never exceeds them
        uint32_t ncellsMax; //!< allocated level-0 cells; the cells1Alloc level-1 cells follow them
        uint32_t activeBase; //!< first work item of this box (prefix of items over boxes)
        uint32_t nItems;     //!< work items: ncells, plus ncells * msub with two levels
        int32_t levelsAlloc; //!< 2 when level-1 cells are allocated
        int32_t levels;      //!< 2 when this step bins small-h particles into level-1 cells
        double e1;           //!< smallest level-1 edge: a particle whose cell radius fits it is level 1
        int32_t m[3];        //!< level-1 sub-cells per level-0 cell along each axis (1 or 2)
        uint32_t msub;       //!< m[0] m[1] m[2]; level-1 cell of level-0 cell l, sub-cell s: l * msub + s
        uint32_t cells1Alloc; //!< allocated level-1 cells
    };

    //! Roles (include/spearhed_b200.h, SPH_ROLE_*).
    __host__ __device__ inline bool isTarget(uint8_t r)
    {
        return (r & SPH_ROLE_MOVABLE) && (r & SPH_ROLE_THERMODYNAMIC);
    }
    __host__ __device__ inline bool isSource(uint8_t r)
    {
        return r & SPH_ROLE_SOURCE;
    }

    //! Cell coordinate along one axis: floor((x - lo)/edge) clamped to [0, n-1].
    //! Cell edge for cull radius support * h: the larger of the FP64 and FP32
    //! radius widened by 2^-20 (the host's cellRadius, same rounding).
    __device__ __forceinline__ double cellRadiusDev(int sup, double h)
    {
        double const r64 = __dmul_rn(double(sup), h);
        double const r32 = double(__fmul_rn(float(sup), float(h)));
        return __dmul_rn(r64 > r32 ? r64 : r32, 1.0 + 1.0 / 1048576.0);
    }

    __device__ __forceinline__ int cellCoord(BoxDev const& b, int a, double x)
    {
        double const f = floor((x - b.lo[a]) / b.edge[a]);
        return f < 0.0 ? 0 : (f >= double(b.n[a]) ? b.n[a] - 1 : int(f));
    }

    //! Lower corner of cell c on axis a, lo + c * edge with the product and the
    //! sum rounded separately (no contraction), as the oracle computes it: the
    //! FP32 cell-relative positions then round from the same FP64 values.
    __device__ __forceinline__ double cellOrigin(BoxDev const& b, int a, int c)
    {
        return __dadd_rn(b.lo[a], __dmul_rn(double(c), b.edge[a]));
    }

    //! Stencil slot 0..26 <-> offset (ox, oy, oz), x fastest; slot 13 is the centre.
    __host__ __device__ __forceinline__ int stencilOff(int slot, int a)
    {
        return a == 0 ? (slot % 3) - 1 : (a == 1 ? ((slot / 3) % 3) - 1 : (slot / 9) - 1);
    }
    constexpr int kCentreSlot = 13;

    //! Stencil offsets of a slot with integer ops only (no division).
    __host__ __device__ __forceinline__ void slotOffsets(uint32_t slot, int& ox, int& oy, int& oz)
    {
        uint32_t const z = (slot * 57u) >> 9;       // slot / 9 for slot < 27
        uint32_t const rem = slot - 9u * z;
        uint32_t const y = (rem * 11u) >> 5;        // rem / 3 for rem < 9
        ox = int(rem - 3u * y) - 1;
        oy = int(y) - 1;
        oz = int(z) - 1;
    }

    //! A neighbour-list entry: sorted source index (27 bits) and stencil slot (5 bits).
    //! A box runs two cell levels while twice its smallest cull radius is at
    //! most this factor times its largest (h range >= 1.6); its level-0 edge
    //! then covers both radii.
    constexpr double kTwoLevelSlack = 1.25;

    __host__ __device__ __forceinline__ uint32_t packEntry(uint32_t j, uint32_t slot)
    {
        return (j << 5) | slot;
    }
    constexpr uint32_t kMaxParticles = 1u << 27;

    // --------------------------------------------------------------- kernels
    // Kernel functions follow the reference's formulas
    // (include/spearhed/sph/CubicSplineKernel.hpp:49-140,
    // QuinticSplineKernel.hpp:47-164); the Wendland C2 kernel (support 2h,
    // W = 21/(16 pi h^3) (1-q/2)^4 (1+2q)) is not in the reference.  Each takes
    // the reciprocal smoothing length so the pair loop divides nowhere.
    template<int K>
    struct Kern;

    template<>
    struct Kern<SPH_KERNEL_CUBIC>
    {
        static constexpr int support = 2;
        template<typename T>
        __device__ __forceinline__ static T norm()
        {
            return T(0.318309886183790671537767526745028724); // 1/pi
        }
        //! W(r,h) h^3 / sigma as a function of x = r/h.
        template<typename T>
        __device__ __forceinline__ static T shapeW(T x)
        {
            if(x < T(1))
                return T(1) - T(1.5) * x * x + T(0.75) * x * x * x;
            if(x < T(2))
            {
                T const t = T(2) - x;
                return T(0.25) * t * t * t;
            }
            return T(0);
        }
        //! (dW/dr) h^4 / sigma as a function of x = r/h.
        template<typename T>
        __device__ __forceinline__ static T shapeDW(T x)
        {
            if(x < T(1))
                return (T(2.25) * x - T(3)) * x;
            if(x < T(2))
            {
                T const t = T(2) - x;
                return T(-0.75) * t * t;
            }
            return T(0);
        }
    };

    template<>
    struct Kern<SPH_KERNEL_QUINTIC>
    {
        static constexpr int support = 3;
        template<typename T>
        __device__ __forceinline__ static T norm()
        {
            return T(0.00265258238486492226281472938954190604); // 1/(120 pi)
        }
        template<typename T>
        __device__ __forceinline__ static T shapeW(T x)
        {
            T const a = T(3) - x, b = T(2) - x, c = T(1) - x;
            T const a2 = a * a, b2 = b * b, c2 = c * c;
            if(x < T(1))
                return a2 * a2 * a - T(6) * b2 * b2 * b + T(15) * c2 * c2 * c;
            if(x < T(2))
                return a2 * a2 * a - T(6) * b2 * b2 * b;
            if(x < T(3))
                return a2 * a2 * a;
            return T(0);
        }
        template<typename T>
        __device__ __forceinline__ static T shapeDW(T x)
        {
            T const a = T(3) - x, b = T(2) - x, c = T(1) - x;
            T const a2 = a * a, b2 = b * b, c2 = c * c;
            if(x < T(1))
                return T(-5) * a2 * a2 + T(30) * b2 * b2 - T(75) * c2 * c2;
            if(x < T(2))
                return T(-5) * a2 * a2 + T(30) * b2 * b2;
            if(x < T(3))
                return T(-5) * a2 * a2;
            return T(0);
        }
    };

    template<>
    struct Kern<SPH_KERNEL_WENDLAND_C2>
    {
        static constexpr int support = 2;
        template<typename T>
        __device__ __forceinline__ static T norm()
        {
            return T(0.417781725616225256392384879024100200); // 21/(16 pi)
        }
        template<typename T>
        __device__ __forceinline__ static T shapeW(T x)
        {
            if(x < T(2))
            {
                T const t = T(1) - T(0.5) * x;
                T const t2 = t * t;
                return t2 * t2 * (T(1) + T(2) * x);
            }
            return T(0);
        }
        //! dW/dr h^4 / sigma = -5 x (1-x/2)^3.
        template<typename T>
        __device__ __forceinline__ static T shapeDW(T x)
        {
            if(x < T(2))
            {
                T const t = T(1) - T(0.5) * x;
                return T(-5) * x * t * t * t;
            }
            return T(0);
        }
    };

    //! Per-particle kernel constants: 1/h, sigma/h^3, sigma/h^4.
    template<typename T>
    struct HConst
    {
        T invh, wnorm, dwnorm;
    };
    template<int K, typename T>
    __device__ __forceinline__ HConst<T> hconstFromInv(T ih)
    {
        T const ih3 = ih * ih * ih;
        T const w = Kern<K>::template norm<T>() * ih3;
        return HConst<T>{ih, w, w * ih};
    }
    template<int K, typename T>
    __device__ __forceinline__ HConst<T> hconst(T h)
    {
        return hconstFromInv<K, T>(T(1) / h);
    }

    //! W(r, h).
    template<int K, typename T>
    __device__ __forceinline__ T kernelW(T r, HConst<T> const& c)
    {
        return c.wnorm * Kern<K>::shapeW(r * c.invh);
    }

    //! gradWScalar(r, invR, h) = dW/dr(r, h) * invR: zero when r is not > 0 or
    //! r >= support h (CubicSplineKernel.hpp:183-192).
    template<int K, typename T>
    __device__ __forceinline__ T gradWScalar(T r, T invR, HConst<T> const& c)
    {
        T const x = r * c.invh;
        if(!(r > T(0)) || x >= T(Kern<K>::support))
            return T(0);
        return c.dwnorm * Kern<K>::shapeDW(x) * invR;
    }

    // ------------------------------------------------------------------- EOS
    //! P = (gamma - 1) rho u (EquationOfState.hpp:32-35).
    template<typename T>
    __device__ __forceinline__ T pressure(T gamma, T rho, T u)
    {
        return (gamma - T(1)) * rho * u;
    }

    // -------------------------------------------------- compensated summation
    //! Knuth's TwoSum: s + e == a + b exactly.
    __device__ __forceinline__ void twoSum(float a, float b, float& s, float& e)
    {
        s = __fadd_rn(a, b);
        float const bb = __fsub_rn(s, a);
        e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
    }

    //! FP32 accumulator with a running compensation term.  Terms are summed
    //! plainly into a short block partial, and each block partial is folded
    //! into (hi, lo) with TwoSum, so the error no longer grows with the
    //! neighbour count (a block of up to 8 terms costs one FP32 rounding each).
    struct CompAcc
    {
        float hi = 0.f, lo = 0.f;
        __device__ __forceinline__ void fold(float part)
        {
            float s, e;
            twoSum(hi, part, s, e);
            hi = s;
            lo += e;
        }
        __device__ __forceinline__ double value() const
        {
            return double(hi) + double(lo);
        }
    };

    //! Ordered-integer view of a non-negative double, for atomicMax/atomicMin.
    __device__ __forceinline__ unsigned long long orderedBits(double x)
    {
        return static_cast<unsigned long long>(__double_as_longlong(x));
    }

    // ----------------------------------------------------------- status word
    //! Device status words the host reads after every call.
    enum StatusWord
    {
        kStatOverflow = 0,   //!< largest neighbour count that did not fit the list
        kStatOutside = 1,    //!< particles found outside a non-periodic box
        kStatNonFinite = 2,  //!< non-finite positions
        kStatMaxCount = 3,   //!< largest neighbour count seen (list sizing)
        kStatBadInput = 4,   //!< gathered h / source masses that are not positive and finite
        kStatCheck = 5,      //!< bounds-checked builds: bit s set when the check at site s failed
        kStatWords = 8
    };

    //! Sites of the device bounds checks (bits of the kStatCheck word).
    enum CheckSite
    {
        kChkCell = 0,       //!< a stencil cell id within the cell arrays
        kChkRange = 1,      //!< a cell's source range within the particles
        kChkStaged = 2,     //!< a staged candidate's particle index
        kChkTargets = 3,    //!< a target cell's range within the particles
        kChkRowEntry = 4,   //!< a list entry read back (particle index and stencil slot)
        kChkPermute = 5,    //!< a permutation index
        kChkKey = 6,        //!< a sorted cell key within the cells
        kChkDriftCell = 7   //!< a particle's cell id from the drift
    };

    //! Bounds-checked builds (compiled with -DSPH_CHECK): a failed check sets
    //! its site's bit in status[kStatCheck] and returns false, and the caller
    //! skips the access, so a bad index is reported, never dereferenced.  In
    //! the normal build every check is `true` and costs nothing.
    __device__ __forceinline__ bool checkIndex(bool ok, uint32_t* status, int site)
    {
#ifdef SPH_CHECK
        if(!ok)
            atomicOr(&status[kStatCheck], 1u << site);
        return ok;
#else
        (void)ok;
        (void)status;
        (void)site;
        return true;
#endif
    }
} // namespace sph
