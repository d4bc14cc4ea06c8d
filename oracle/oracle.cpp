/* CPU oracle for the SPH(-MHD) step — TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * Only tests/, the smoke check and bench.py's CPU-baseline leg load this
 * library (oracle/_build/liboracle.so).  The product path never calls it.
 *
 * What it restates, and from where (reference paths are relative to the
 * spearHED checkout):
 *   - Cubic / quintic spline kernels: include/spearhed/sph/CubicSplineKernel.hpp:49-140,
 *     QuinticSplineKernel.hpp:47-164 (same branch structure, same operation
 *     order, same h-power loop).  Pinned bit-for-bit against the reference's
 *     own headers compiled in oracle/ref_functors.cpp.
 *   - Ideal-gas EOS: include/spearhed/sph/EquationOfState.hpp:32-47 (sound
 *     speed evaluated in double, then cast).
 *   - Density gather with self term: include/spearhed/particles/density/
 *     DensitySummation.hpp:57-93 (rho_i = m_i W(0,h_i) + sum_{j!=i} m_j W(r,h_i)).
 *   - Inviscid hydro + P dV: include/spearhed/sph/HydroForces.hpp:112-175.
 *   - Pair geometry: spmacc/particles/algorithms/ParticleParticleInteraction.hpp:236-313
 *     (staged = pos_j + origin shift; d = own - staged in x,y,z order; r2
 *     summed unfused in that order; strict cull r2 < R^2; invR = 1/sqrt(r2),
 *     r = r2*invR only when r2 > 0, else both 0; isSelf = same particle and
 *     same image).
 *   - Step order: include/spearhed/control/Simulation.x.cpp:233-300 (drift of
 *     Movable species, neighbour search, density, forces, kick of
 *     Movable&Thermodynamic species; Boundary species are sources with frozen
 *     rho and u).  Drift/kick: particles/pusher/PushVelocity.hpp:38-41,
 *     EulerIntegrate.hpp:45-51.
 * Terms the reference does not have, written from the published methods
 * (parity for these is defined by this file, not by the reference):
 *   - Wendland C2 kernel (Wendland 1995; Dehnen & Aly 2012 normalisation,
 *     support 2h): W = 21/(16 pi h^3) (1-q/2)^4 (1+2q).
 *   - Artificial viscosity of Monaghan (1992, ARA&A 30, 543):
 *     mu = hbar v.r/(r^2 + eps hbar^2) for v.r < 0, Pi = (-alpha cbar mu + beta mu^2)/rhobar,
 *     applied with the mean kernel gradient; heating 1/2 m_j Pi v.gradW.
 *   - SPMHD (Price & Monaghan 2005; Price 2012, JCP 231, 759): Maxwell stress
 *     force, induction dB/dt = -(1/rho_i) sum m_j s_i [v_ij (B_i.r) - B_i (v_ij.r)],
 *     Borve et al. (2001) tensile correction -B_i sum m_j (B_i s_i/rho_i^2 + B_j s_j/rho_j^2).r.
 *   - Dedner cleaning in the constrained form of Tricco & Price (2012):
 *     dB/dt -= grad psi (symmetric), dpsi/dt = -c_h^2 divB - psi sigma c_h/h - psi divv/2,
 *     c_h = max fast speed.
 *   - CFL: dt_i = C h_i / max_j vsig_ij with vsig_ij = c_i + c_j - beta min(0, v_ij.r/|r|),
 *     and the force criterion C_f sqrt(h_i/|a_i|); dt = min over particles.
 *   - Periodic boxes through a cell stencil that enumerates every image
 *     within the radius (valid while the box is at least one radius wide).
 *
 * The cell geometry here is the one the CUDA path uses (cell edge >= the cull
 * radius, positions relative to the lower corner of their cell, stencil shift
 * o*edge added to the neighbour position), so that in the FP32 geometry mode
 * the accepted pair set is bit-identical to the GPU's.
 */
#include "../include/spearhed_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numbers>
#include <vector>

#ifdef _OPENMP
#    include <omp.h>
#endif

namespace orc
{
    // ---------------------------------------------------------------- kernels
    template<typename T>
    struct Cubic
    {
        static constexpr int support = 2;
        static T W(T r, T h)
        {
            T const x = r / h;
            T const sigma = T{1} / std::numbers::pi_v<T>;
            T kv{0};
            if(x < T{1})
                kv = T{1} - T{1.5} * x * x + T{0.75} * x * x * x;
            else if(x < T{2})
                kv = T{0.25} * (T{2} - x) * (T{2} - x) * (T{2} - x);
            T hp{1};
            for(int i = 0; i < 3; ++i)
                hp *= h;
            return sigma / hp * kv;
        }
        static T dWdr(T r, T h)
        {
            T const x = r / h;
            T const sigma = T{1} / std::numbers::pi_v<T>;
            T kv{0};
            if(x >= T{0} && x < T{1})
                kv = T{2.25} * x * x - T{3} * x;
            else if(x < T{2})
                kv = -T{0.75} * (T{2} - x) * (T{2} - x);
            T hp{1};
            for(int i = 0; i <= 3; ++i)
                hp *= h;
            return sigma / hp * kv;
        }
    };

    template<typename T>
    struct Quintic
    {
        static constexpr int support = 3;
        static T W(T r, T h)
        {
            T const x = r / h;
            T const sigma = T{1} / (T{120} * std::numbers::pi_v<T>);
            T kv{0};
            if(x < T{1})
            {
                T const a = T{3} - x, b = T{2} - x, c = T{1} - x;
                kv = a * a * a * a * a - T{6} * b * b * b * b * b + T{15} * c * c * c * c * c;
            }
            else if(x < T{2})
            {
                T const a = T{3} - x, b = T{2} - x;
                kv = a * a * a * a * a - T{6} * b * b * b * b * b;
            }
            else if(x < T{3})
            {
                T const a = T{3} - x;
                kv = a * a * a * a * a;
            }
            T hp{1};
            for(int i = 0; i < 3; ++i)
                hp *= h;
            return sigma / hp * kv;
        }
        static T dWdr(T r, T h)
        {
            T const x = r / h;
            T const sigma = T{1} / (T{120} * std::numbers::pi_v<T>);
            T kv{0};
            if(x < T{1})
            {
                T const a = T{3} - x, b = T{2} - x, c = T{1} - x;
                kv = -T{5} * a * a * a * a + T{30} * b * b * b * b - T{75} * c * c * c * c;
            }
            else if(x < T{2})
            {
                T const a = T{3} - x, b = T{2} - x;
                kv = -T{5} * a * a * a * a + T{30} * b * b * b * b;
            }
            else if(x < T{3})
            {
                T const a = T{3} - x;
                kv = -T{5} * a * a * a * a;
            }
            T hp{1};
            for(int i = 0; i <= 3; ++i)
                hp *= h;
            return sigma / hp * kv;
        }
    };

    //! Wendland C2 in 3D with support 2h (Dehnen & Aly 2012, H = 2h).
    template<typename T>
    struct WendlandC2
    {
        static constexpr int support = 2;
        static T W(T r, T h)
        {
            T const q = r / h;
            T const sigma = T{21} / (T{16} * std::numbers::pi_v<T>);
            T kv{0};
            if(q < T{2})
            {
                T const t = T{1} - T{0.5} * q;
                T const t2 = t * t;
                kv = t2 * t2 * (T{1} + T{2} * q);
            }
            return sigma / (h * h * h) * kv;
        }
        static T dWdr(T r, T h)
        {
            T const q = r / h;
            T const sigma = T{21} / (T{16} * std::numbers::pi_v<T>);
            T kv{0};
            if(q >= T{0} && q < T{2})
            {
                T const t = T{1} - T{0.5} * q;
                kv = T{-5} * q * t * t * t;
            }
            return sigma / (h * h * h * h) * kv;
        }
    };

    template<typename K, typename T>
    T gradWScalar(T r, T invR, T h)
    {
        if(!(r > T{0}) || r >= static_cast<T>(K::support) * h)
            return T{0};
        return K::dWdr(r, h) * invR;
    }

    template<typename T>
    T pressure(T gamma, T rho, T u)
    {
        return (gamma - T{1}) * rho * u;
    }
    template<typename T>
    T soundSpeed(T gamma, T p, T rho)
    {
        return static_cast<T>(std::sqrt(static_cast<double>(gamma * p / rho)));
    }

    inline int supportOf(int kernel)
    {
        return kernel == SPH_KERNEL_QUINTIC ? 3 : 2;
    }

    // ------------------------------------------------------------ cell grid
    struct Grid
    {
        double lo[3], L[3], edge[3];
        int n[3];
        int periodic[3];
        int64_t base; // first cell id of this box in the global cell numbering
        int64_t ncells() const
        {
            return int64_t(n[0]) * n[1] * n[2];
        }
    };

    //! Cell edge >= rcell on every axis; n = floor(L / rcell), at least 1 and
    //! at most nMax[a] when given.
    inline int makeGrid(SphBox const& b, double rcell, Grid& g, int const* nMax = nullptr)
    {
        for(int a = 0; a < 3; ++a)
        {
            g.lo[a] = b.lo[a];
            g.L[a] = b.hi[a] - b.lo[a];
            g.periodic[a] = b.periodic[a] ? 1 : 0;
            if(!(g.L[a] > 0.0))
                return SPH_ERR_INVALID;
            double const nd = std::floor(g.L[a] / rcell);
            g.n[a] = nd < 1.0 ? 1 : (nd > 1.0e6 ? 1000000 : int(nd));
            if(nMax && g.n[a] > nMax[a])
                g.n[a] = nMax[a];
            g.edge[a] = g.L[a] / g.n[a];
            if(g.periodic[a] && g.L[a] < rcell)
                return SPH_ERR_UNSUPPORTED; // images beyond the nearest would be needed
        }
        return SPH_OK;
    }

    /** Smallest admissible cell edge for cull radius support*h: the larger of the
     *  FP64 and FP32 values of support*h, widened by 2^-20 so that a radius
     *  rounded up in FP32 never exceeds the edge. */
    inline double cellRadius(int sup, double h)
    {
        double const r64 = double(sup) * h;
        double const r32 = double(float(sup) * float(h));
        return (r64 > r32 ? r64 : r32) * (1.0 + 1.0 / 1048576.0);
    }

    inline int cellCoord(Grid const& g, int a, double x)
    {
        double const f = std::floor((x - g.lo[a]) / g.edge[a]);
        int c = f < 0.0 ? 0 : (f >= g.n[a] ? g.n[a] - 1 : int(f));
        return c;
    }

    // ------------------------------------------------------------- the system
    struct System
    {
        SphParams p{};
        int nbox = 1;
        std::vector<SphBox> boxes;
        std::vector<Grid> grids;
        int64_t n = 0;
        uint8_t const* roles = nullptr;
        SphSoAView* v = nullptr;
        std::vector<int32_t> boxOf;
        std::vector<int> cx, cy, cz;
        std::vector<int64_t> cellOf; // global cell id, -1 for non-sources
        std::vector<int64_t> cellStart; // CSR over global cells (sources only)
        std::vector<int64_t> cellItems;
        std::vector<double> hcap;
        std::vector<int> nMax; // allocation of the first grid, per box and axis
        int64_t ncellTotal = 0;

        bool isTarget(int64_t i) const
        {
            return (roles[i] & SPH_ROLE_MOVABLE) && (roles[i] & SPH_ROLE_THERMODYNAMIC);
        }
        bool isSource(int64_t i) const
        {
            return roles[i] & SPH_ROLE_SOURCE;
        }
    };

    inline double col(double const* a, int64_t i, double dflt = 0.0)
    {
        return a ? a[i] : dflt;
    }

    //! Bin the sources into cells (stable: ascending particle index within a cell).
    inline int buildCells(System& s)
    {
        int const sup = supportOf(s.p.kernel);
        // cull radius upper bound per box
        std::vector<double> hmax(s.nbox, s.p.h0);
        if(s.p.cull == SPH_CULL_PAIR_MAX)
        {
            std::fill(hmax.begin(), hmax.end(), 0.0);
            for(int64_t i = 0; i < s.n; ++i)
            {
                double const hi = col(s.v->h, i, s.p.h0);
                hmax[s.boxOf[i]] = std::max(hmax[s.boxOf[i]], hi);
            }
        }
        s.grids.resize(s.nbox);
        bool const first = s.nMax.empty();
        bool const dynamic = s.p.cull == SPH_CULL_PAIR_MAX;
        if(first)
        {
            s.nMax.assign(size_t(s.nbox) * 3, 1);
            s.hcap.assign(s.nbox, 0.0);
        }
        int64_t base = 0;
        for(int b = 0; b < s.nbox; ++b)
        {
            // Same rule as the CUDA path: the grid follows the box's current
            // largest h (global cull: h0), its cell counts clamped to what the
            // first grid allocates (room for h halving on every axis).  Adaptive
            // h is capped by h_max, else by what the periodic axes admit.
            if(dynamic && s.p.h_max > 0.0 && s.p.h_max < hmax[b])
                return SPH_ERR_INVALID;
            double const rc = cellRadius(sup, hmax[b]);
            if(first)
            {
                double hcap = s.p.h_max > 0.0 ? s.p.h_max : 1e300;
                for(int a = 0; a < 3; ++a)
                {
                    double const L = s.boxes[b].hi[a] - s.boxes[b].lo[a];
                    double const nd = std::floor(L / rc);
                    int const n0 = nd < 1.0 ? 1 : (nd > 1.0e6 ? 1000000 : int(nd));
                    double const ndMax = dynamic ? std::floor(L / (0.5 * rc)) : nd;
                    s.nMax[size_t(b) * 3 + a]
                        = std::max(n0, ndMax < 1.0 ? 1 : (ndMax > 1.0e6 ? 1000000 : int(ndMax)));
                    if(s.boxes[b].periodic[a] && s.p.h_max <= 0.0 && (s.p.physics & SPH_PHYS_ADAPTIVE_H))
                    {
                        double lim = L / (double(sup) * (1.0 + 1.0 / 262144.0));
                        while(lim > hmax[b] && cellRadius(sup, lim) > L)
                            lim = std::nextafter(lim, 0.0);
                        hcap = std::min(hcap, std::max(lim, hmax[b]));
                    }
                }
                s.hcap[b] = hcap;
            }
            int const st = makeGrid(s.boxes[b], rc, s.grids[b], &s.nMax[size_t(b) * 3]);
            if(st != SPH_OK)
                return st;
            s.grids[b].base = base;
            base += s.grids[b].ncells();
        }
        s.ncellTotal = base;
        s.cx.assign(s.n, 0);
        s.cy.assign(s.n, 0);
        s.cz.assign(s.n, 0);
        s.cellOf.assign(s.n, -1);
        std::vector<int64_t> count(base + 1, 0);
        for(int64_t i = 0; i < s.n; ++i)
        {
            Grid const& g = s.grids[s.boxOf[i]];
            double const x[3] = {s.v->pos[0][i], s.v->pos[1][i], s.v->pos[2][i]};
            for(int a = 0; a < 3; ++a)
            {
                if(!std::isfinite(x[a]))
                    return SPH_ERR_NONFINITE;
                // every axis (the drift has wrapped movable particles on periodic ones)
                if(x[a] < g.lo[a] || x[a] > g.lo[a] + g.L[a])
                    return SPH_ERR_OUTSIDE;
            }
            s.cx[i] = cellCoord(g, 0, x[0]);
            s.cy[i] = cellCoord(g, 1, x[1]);
            s.cz[i] = cellCoord(g, 2, x[2]);
            int64_t const c = g.base + (int64_t(s.cz[i]) * g.n[1] + s.cy[i]) * g.n[0] + s.cx[i];
            if(s.isSource(i))
            {
                s.cellOf[i] = c;
                ++count[c + 1];
            }
        }
        for(int64_t c = 0; c < base; ++c)
            count[c + 1] += count[c];
        s.cellStart = count;
        s.cellItems.assign(count[base], 0);
        std::vector<int64_t> cursor(count.begin(), count.end() - 1);
        for(int64_t i = 0; i < s.n; ++i)
            if(s.cellOf[i] >= 0)
                s.cellItems[cursor[s.cellOf[i]]++] = i;
        return SPH_OK;
    }

    //! Position of particle i relative to the lower corner of its cell, in T.
    template<typename T>
    inline void relPos(System const& s, int64_t i, T out[3])
    {
        Grid const& g = s.grids[s.boxOf[i]];
        int const c[3] = {s.cx[i], s.cy[i], s.cz[i]};
        for(int a = 0; a < 3; ++a)
        {
            double const origin = g.lo[a] + double(c[a]) * g.edge[a];
            out[a] = static_cast<T>(s.v->pos[a][i] - origin);
        }
    }

    struct Pair
    {
        int64_t j;
        int8_t o[3];
    };

    //! Accepted neighbours of target i (i != j or a non-zero image), in stencil
    //! order z, y, x (x fastest), then ascending index inside a cell.
    //! Geometry in T exactly as the CUDA path computes it.
    template<typename T>
    inline void neighbours(System const& s, int64_t i, std::vector<Pair>& out)
    {
        out.clear();
        Grid const& g = s.grids[s.boxOf[i]];
        int const sup = supportOf(s.p.kernel);
        T pi[3];
        relPos<T>(s, i, pi);
        T const edge[3] = {static_cast<T>(g.edge[0]), static_cast<T>(g.edge[1]), static_cast<T>(g.edge[2])};
        T const hi = static_cast<T>(col(s.v->h, i, s.p.h0));
        T const h0 = static_cast<T>(s.p.h0);
        int const c[3] = {s.cx[i], s.cy[i], s.cz[i]};
        for(int oz = -1; oz <= 1; ++oz)
            for(int oy = -1; oy <= 1; ++oy)
                for(int ox = -1; ox <= 1; ++ox)
                {
                    int const o[3] = {ox, oy, oz};
                    int nc[3];
                    bool skip = false;
                    for(int a = 0; a < 3; ++a)
                    {
                        nc[a] = c[a] + o[a];
                        if(nc[a] < 0 || nc[a] >= g.n[a])
                        {
                            if(!g.periodic[a])
                            {
                                skip = true;
                                break;
                            }
                            nc[a] = (nc[a] + g.n[a]) % g.n[a];
                        }
                    }
                    if(skip)
                        continue;
                    int64_t const cell = g.base + (int64_t(nc[2]) * g.n[1] + nc[1]) * g.n[0] + nc[0];
                    T const sh[3] = {T(o[0]) * edge[0], T(o[1]) * edge[1], T(o[2]) * edge[2]};
                    for(int64_t q = s.cellStart[cell]; q < s.cellStart[cell + 1]; ++q)
                    {
                        int64_t const j = s.cellItems[q];
                        bool const self = (j == i) && ox == 0 && oy == 0 && oz == 0;
                        if(self)
                            continue;
                        T pj[3];
                        relPos<T>(s, j, pj);
                        T r2{0};
                        for(int a = 0; a < 3; ++a)
                        {
                            T const staged = pj[a] + sh[a];
                            T const d = pi[a] - staged;
                            r2 = r2 + d * d;
                        }
                        T hc = h0;
                        if(s.p.cull == SPH_CULL_PAIR_MAX)
                        {
                            T const hj = static_cast<T>(col(s.v->h, j, s.p.h0));
                            hc = hi > hj ? hi : hj;
                        }
                        T const R = static_cast<T>(sup) * hc;
                        if(r2 < R * R)
                            out.push_back(Pair{j, {int8_t(ox), int8_t(oy), int8_t(oz)}});
                    }
                }
    }

    //! FP64 displacement r_i - r_j of an accepted pair (the oracle's physics is FP64).
    inline void displacement(System const& s, int64_t i, Pair const& pr, double d[3])
    {
        double pi[3], pj[3];
        relPos<double>(s, i, pi);
        relPos<double>(s, pr.j, pj);
        Grid const& g = s.grids[s.boxOf[i]];
        for(int a = 0; a < 3; ++a)
            d[a] = pi[a] - (pj[a] + double(pr.o[a]) * g.edge[a]);
    }

    template<typename K>
    void densityPass(System& s, bool fp32geom)
    {
#pragma omp parallel
        {
            std::vector<Pair> nb;
#pragma omp for schedule(dynamic, 256)
            for(int64_t i = 0; i < s.n; ++i)
            {
                if(!s.isTarget(i))
                    continue;
                if(fp32geom)
                    neighbours<float>(s, i, nb);
                else
                    neighbours<double>(s, i, nb);
                double const hi = col(s.v->h, i, s.p.h0);
                double rho = s.v->mass[i] * K::W(0.0, hi);
                for(auto const& pr : nb)
                {
                    double d[3];
                    displacement(s, i, pr, d);
                    double const r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                    double r = 0.0;
                    if(r2 > 0.0)
                        r = r2 * (1.0 / std::sqrt(r2));
                    rho += s.v->mass[pr.j] * K::W(r, hi);
                }
                s.v->density[i] = rho;
            }
        }
    }

    struct Derived
    {
        double P, pOverRho2, pTotOverRho2, c, rho;
    };

    inline Derived derived(System const& s, int64_t i)
    {
        bool const mhd = s.p.physics & SPH_PHYS_MHD;
        double const rho = s.v->density[i];
        double const u = col(s.v->u, i);
        Derived d{};
        d.rho = rho;
        d.P = pressure(s.p.gamma, rho, u);
        d.pOverRho2 = d.P / (rho * rho);
        double const cs = soundSpeed(s.p.gamma, d.P, rho);
        if(mhd)
        {
            double B2 = 0;
            for(int a = 0; a < 3; ++a)
                B2 += col(s.v->B[a], i) * col(s.v->B[a], i);
            d.c = std::sqrt(cs * cs + B2 / (s.p.mu0 * rho));
            d.pTotOverRho2 = (d.P + 0.5 * B2 / s.p.mu0) / (rho * rho);
        }
        else
        {
            d.c = cs;
            d.pTotOverRho2 = d.pOverRho2;
        }
        return d;
    }

    //! Per box: the Dedner speed used and the CFL minimum; accepted pairs in total.
    struct ForceOut
    {
        std::vector<double> ch;
        std::vector<double> dtmin;
        double pairs = 0.0;
    };

    template<typename K>
    ForceOut forcePass(System& s, bool fp32geom)
    {
        SphParams const& p = s.p;
        bool const av = p.physics & SPH_PHYS_AV;
        bool const mhd = p.physics & SPH_PHYS_MHD;
        bool const dedner = mhd && (p.physics & SPH_PHYS_DEDNER);
        bool const tensile = mhd && (p.physics & SPH_PHYS_TENSILE);
        double const mu0 = p.mu0 > 0 ? p.mu0 : 1.0;
        std::vector<Derived> der(s.n);
        // each box of an ensemble has its own cleaning speed and CFL minimum
        std::vector<double> chBox(s.nbox, 0.0);
        for(int64_t i = 0; i < s.n; ++i)
            if(s.isSource(i) || s.isTarget(i))
            {
                der[i] = derived(s, i);
                if(s.isTarget(i))
                    chBox[s.boxOf[i]] = std::max(chBox[s.boxOf[i]], der[i].c);
            }
        std::vector<double> dtBox(s.nbox, 1e300);
        double pairs = 0.0;
#pragma omp parallel reduction(+ : pairs)
        {
            std::vector<double> dtLocal(s.nbox, 1e300);
            std::vector<Pair> nb;
#pragma omp for schedule(dynamic, 256)
            for(int64_t i = 0; i < s.n; ++i)
            {
                if(!s.isTarget(i))
                    continue;
                if(fp32geom)
                    neighbours<float>(s, i, nb);
                else
                    neighbours<double>(s, i, nb);
                pairs += double(nb.size());
                Derived const& di = der[i];
                double const ch = chBox[s.boxOf[i]];
                double const hi = col(s.v->h, i, p.h0);
                double const vi[3] = {col(s.v->vel[0], i), col(s.v->vel[1], i), col(s.v->vel[2], i)};
                double const Bi[3] = {col(s.v->B[0], i), col(s.v->B[1], i), col(s.v->B[2], i)};
                double const psii = col(s.v->psi, i);
                double a[3] = {0, 0, 0}, du = 0, duav = 0;
                double T3[3] = {0, 0, 0}, D = 0, divB = 0, gpsi[3] = {0, 0, 0};
                double aniso[3] = {0, 0, 0}, tens = 0;
                double vsig = di.c;
                for(auto const& pr : nb)
                {
                    int64_t const j = pr.j;
                    Derived const& dj = der[j];
                    double rv[3];
                    displacement(s, i, pr, rv);
                    double const r2 = rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2];
                    double invR = 0, r = 0;
                    if(r2 > 0.0)
                    {
                        invR = 1.0 / std::sqrt(r2);
                        r = r2 * invR;
                    }
                    double const hj = col(s.v->h, j, p.h0);
                    double const si = gradWScalar<K>(r, invR, hi);
                    double const sj = gradWScalar<K>(r, invR, hj);
                    double const mj = s.v->mass[j];
                    double const vj[3] = {col(s.v->vel[0], j), col(s.v->vel[1], j), col(s.v->vel[2], j)};
                    double const vij[3] = {vi[0] - vj[0], vi[1] - vj[1], vi[2] - vj[2]};
                    double const vr = vij[0] * rv[0] + vij[1] * rv[1] + vij[2] * rv[2];
                    // pressure gradient (HydroForces.hpp:155-166), total pressure with MHD
                    double const ti = mj * di.pTotOverRho2, tj = mj * dj.pTotOverRho2;
                    double const fiso = ti * si + tj * sj;
                    for(int q = 0; q < 3; ++q)
                        a[q] -= fiso * rv[q];
                    // P dV (HydroForces.hpp:168-173), thermal pressure only
                    du += mj * di.pOverRho2 * si * vr;
                    D += mj * si * vr;
                    if(av && vr < 0.0)
                    {
                        double const hb = 0.5 * (hi + hj);
                        double const mu = hb * vr / (r2 + p.av_eps * hb * hb);
                        double const cb = 0.5 * (di.c + dj.c);
                        double const rb = 0.5 * (di.rho + dj.rho);
                        double const Pi = (-p.alpha * cb * mu + p.beta * mu * mu) / rb;
                        double const gb = 0.5 * (si + sj);
                        for(int q = 0; q < 3; ++q)
                            a[q] -= mj * Pi * gb * rv[q];
                        duav += 0.5 * mj * Pi * gb * vr;
                    }
                    double const w = (r > 0.0) ? vr * invR : 0.0;
                    vsig = std::max(vsig, di.c + dj.c - p.beta * std::min(0.0, w));
                    if(mhd)
                    {
                        double const Bj[3] = {col(s.v->B[0], j), col(s.v->B[1], j), col(s.v->B[2], j)};
                        double const Bir = Bi[0] * rv[0] + Bi[1] * rv[1] + Bi[2] * rv[2];
                        double const Bjr = Bj[0] * rv[0] + Bj[1] * rv[1] + Bj[2] * rv[2];
                        double const ci = mj * si * Bir / (mu0 * di.rho * di.rho);
                        double const cj = mj * sj * Bjr / (mu0 * dj.rho * dj.rho);
                        for(int q = 0; q < 3; ++q)
                            aniso[q] += ci * Bi[q] + cj * Bj[q];
                        tens += ci + cj;
                        // induction: sum m_j s_i v_ij (B_i.r); the B_i (v_ij.r) part uses D
                        for(int q = 0; q < 3; ++q)
                            T3[q] += mj * si * Bir * vij[q];
                        divB += mj * si * (Bir - Bjr);
                        if(dedner)
                        {
                            double const psij = col(s.v->psi, j);
                            double const g = mj
                                             * (psii / (di.rho * di.rho) * si
                                                + psij / (dj.rho * dj.rho) * sj);
                            for(int q = 0; q < 3; ++q)
                                gpsi[q] += g * rv[q];
                        }
                    }
                }
                if(mhd)
                {
                    for(int q = 0; q < 3; ++q)
                    {
                        a[q] += aniso[q];
                        if(tensile)
                            a[q] -= Bi[q] * tens;
                    }
                }
                for(int q = 0; q < 3; ++q)
                    s.v->dvdt[q][i] = a[q];
                s.v->dudt[i] = du + duav;
                double const invRho = 1.0 / di.rho;
                double const divv = -invRho * D;
                double const dB = -invRho;
                double divBi = -invRho * divB;
                if(mhd)
                {
                    for(int q = 0; q < 3; ++q)
                    {
                        double v = dB * (T3[q] - Bi[q] * D);
                        if(dedner)
                            v -= di.rho * gpsi[q];
                        if(s.v->dBdt[q])
                            s.v->dBdt[q][i] = v;
                    }
                    if(s.v->dpsidt)
                        s.v->dpsidt[i] = dedner ? (-ch * ch * divBi - psii * p.dedner_sigma * ch / hi - 0.5 * psii * divv) : 0.0;
                    if(s.v->divB)
                        s.v->divB[i] = divBi;
                }
                double dt = p.cfl * hi / vsig;
                double const amag = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
                if(amag > 0.0 && p.cfl_force > 0.0)
                    dt = std::min(dt, p.cfl_force * std::sqrt(hi / amag));
                dtLocal[s.boxOf[i]] = std::min(dtLocal[s.boxOf[i]], dt);
            }
#pragma omp critical
            for(int b = 0; b < s.nbox; ++b)
                dtBox[b] = std::min(dtBox[b], dtLocal[b]);
        }
        ForceOut fo;
        fo.ch = chBox;
        fo.dtmin = dtBox;
        fo.pairs = pairs;
        return fo;
    }

    template<typename F>
    auto withKernel(int kernel, F&& f)
    {
        if(kernel == SPH_KERNEL_QUINTIC)
            return f(Quintic<double>{});
        if(kernel == SPH_KERNEL_WENDLAND_C2)
            return f(WendlandC2<double>{});
        return f(Cubic<double>{});
    }

    inline int setup(
        System& s,
        SphParams const* p,
        int32_t nbox,
        SphBox const* boxes,
        int64_t n,
        uint8_t const* roles,
        SphSoAView* v)
    {
        if(!p || !boxes || nbox < 1 || n < 0 || !roles || !v || !v->mass || !v->density)
            return SPH_ERR_INVALID;
        s.p = *p;
        if(s.p.mu0 <= 0)
            s.p.mu0 = 1.0;
        s.nbox = nbox;
        s.boxes.assign(boxes, boxes + nbox);
        s.n = n;
        s.roles = roles;
        s.v = v;
        s.boxOf.assign(n, 0);
        for(int64_t i = 0; i < n; ++i)
        {
            s.boxOf[i] = v->box_id ? v->box_id[i] : 0;
            if(s.boxOf[i] < 0 || s.boxOf[i] >= nbox)
                return SPH_ERR_INVALID;
        }
        return buildCells(s);
    }

    inline void diagnostics(System const& s, SphDiag& d)
    {
        double ek = 0, ei = 0, em = 0, m3[3] = {0, 0, 0}, dsum = 0, dmax = 0;
        int64_t nt = 0, nd = 0;
        double const mu0 = s.p.mu0 > 0 ? s.p.mu0 : 1.0;
        for(int64_t i = 0; i < s.n; ++i)
        {
            if(!s.isTarget(i))
                continue;
            double const m = s.v->mass[i];
            double v2 = 0, B2 = 0;
            for(int a = 0; a < 3; ++a)
            {
                double const va = col(s.v->vel[a], i);
                v2 += va * va;
                m3[a] += m * va;
                double const Ba = col(s.v->B[a], i);
                B2 += Ba * Ba;
            }
            ek += 0.5 * m * v2;
            ei += m * col(s.v->u, i);
            double const rho = s.v->density[i];
            if(rho > 0)
                em += 0.5 * m * B2 / (mu0 * rho);
            if(B2 > 0 && s.v->divB)
            {
                double const e = std::fabs(s.v->divB[i]) * col(s.v->h, i, s.p.h0) / std::sqrt(B2);
                dsum += e;
                dmax = std::max(dmax, e);
                ++nd;
            }
            ++nt;
        }
        d.e_kin = ek;
        d.e_int = ei;
        d.e_mag = em;
        for(int a = 0; a < 3; ++a)
            d.mom[a] = m3[a];
        d.divb_mean = nd ? dsum / double(nd) : 0.0;
        d.divb_max = dmax;
        d.n_targets = nt;
    }
} // namespace orc

extern "C"
{
    //! The oracle's kernel functions, for pinning tests (prec 0: double, 1: float).
    double orc_kernel_W(int kernel, int prec, double r, double h)
    {
        using namespace orc;
        if(prec)
        {
            float const rf = float(r), hf = float(h);
            if(kernel == SPH_KERNEL_QUINTIC)
                return Quintic<float>::W(rf, hf);
            if(kernel == SPH_KERNEL_WENDLAND_C2)
                return WendlandC2<float>::W(rf, hf);
            return Cubic<float>::W(rf, hf);
        }
        return withKernel(kernel, [&](auto k) { return decltype(k)::W(r, h); });
    }
    double orc_kernel_dWdr(int kernel, int prec, double r, double h)
    {
        using namespace orc;
        if(prec)
        {
            float const rf = float(r), hf = float(h);
            if(kernel == SPH_KERNEL_QUINTIC)
                return Quintic<float>::dWdr(rf, hf);
            if(kernel == SPH_KERNEL_WENDLAND_C2)
                return WendlandC2<float>::dWdr(rf, hf);
            return Cubic<float>::dWdr(rf, hf);
        }
        return withKernel(kernel, [&](auto k) { return decltype(k)::dWdr(r, h); });
    }
    double orc_kernel_gradWScalar(int kernel, int prec, double r, double invR, double h)
    {
        using namespace orc;
        if(prec)
        {
            float const rf = float(r), ivf = float(invR), hf = float(h);
            if(kernel == SPH_KERNEL_QUINTIC)
                return gradWScalar<Quintic<float>>(rf, ivf, hf);
            if(kernel == SPH_KERNEL_WENDLAND_C2)
                return gradWScalar<WendlandC2<float>>(rf, ivf, hf);
            return gradWScalar<Cubic<float>>(rf, ivf, hf);
        }
        return withKernel(kernel, [&](auto k) { return gradWScalar<decltype(k)>(r, invR, h); });
    }
    double orc_pressure(int prec, double gamma, double rho, double u)
    {
        return prec ? double(orc::pressure<float>(float(gamma), float(rho), float(u))) : orc::pressure(gamma, rho, u);
    }
    double orc_sound_speed(int prec, double gamma, double P, double rho)
    {
        return prec ? double(orc::soundSpeed<float>(float(gamma), float(P), float(rho)))
                    : orc::soundSpeed(gamma, P, rho);
    }

    //! Accepted neighbours (i != j or a non-zero image) per target; -1 for non-targets.
    //! geom_fp32 selects the FP32 geometry of the FP32 pair kernels.
    int orc_neighbour_counts(
        SphParams const* p,
        int32_t nbox,
        SphBox const* boxes,
        int64_t n,
        uint8_t const* roles,
        SphSoAView* v,
        int32_t geom_fp32,
        int32_t* counts,
        double* pairs)
    {
        orc::System s;
        int st = orc::setup(s, p, nbox, boxes, n, roles, v);
        if(st)
            return st;
        double total = 0;
#pragma omp parallel reduction(+ : total)
        {
            std::vector<orc::Pair> nb;
#pragma omp for schedule(dynamic, 256)
            for(int64_t i = 0; i < n; ++i)
            {
                if(!s.isTarget(i))
                {
                    counts[i] = -1;
                    continue;
                }
                if(geom_fp32)
                    orc::neighbours<float>(s, i, nb);
                else
                    orc::neighbours<double>(s, i, nb);
                counts[i] = int32_t(nb.size());
                total += double(nb.size());
            }
        }
        if(pairs)
            *pairs = total;
        return SPH_OK;
    }

    //! Neighbour list of one target particle: up to cap entries (j, ox, oy, oz).
    int orc_neighbour_list(
        SphParams const* p,
        int32_t nbox,
        SphBox const* boxes,
        int64_t n,
        uint8_t const* roles,
        SphSoAView* v,
        int32_t geom_fp32,
        int64_t i,
        int32_t cap,
        int64_t* js,
        int8_t* offs,
        int32_t* count)
    {
        orc::System s;
        int st = orc::setup(s, p, nbox, boxes, n, roles, v);
        if(st)
            return st;
        if(i < 0 || i >= n)
            return SPH_ERR_INVALID;
        std::vector<orc::Pair> nb;
        if(geom_fp32)
            orc::neighbours<float>(s, i, nb);
        else
            orc::neighbours<double>(s, i, nb);
        *count = int32_t(nb.size());
        for(int32_t k = 0; k < int32_t(nb.size()) && k < cap; ++k)
        {
            js[k] = nb[k].j;
            for(int a = 0; a < 3; ++a)
                offs[3 * k + a] = nb[k].o[a];
        }
        return SPH_OK;
    }

    /** Full neighbour lists of every target in CSR form (non-targets get an empty
     *  row): off[n+1], js[total], offs[3*total] (stencil image of each entry).
     *  Fails with SPH_ERR_OVERFLOW (and sets *total) when cap is too small. */
    int orc_neighbour_csr(
        SphParams const* p,
        int32_t nbox,
        SphBox const* boxes,
        int64_t n,
        uint8_t const* roles,
        SphSoAView* v,
        int32_t geom_fp32,
        int64_t cap,
        int64_t* off,
        int64_t* js,
        int8_t* offs,
        int64_t* total)
    {
        orc::System s;
        int st = orc::setup(s, p, nbox, boxes, n, roles, v);
        if(st)
            return st;
        std::vector<std::vector<orc::Pair>> all(n);
#pragma omp parallel for schedule(dynamic, 256)
        for(int64_t i = 0; i < n; ++i)
        {
            if(!s.isTarget(i))
                continue;
            if(geom_fp32)
                orc::neighbours<float>(s, i, all[i]);
            else
                orc::neighbours<double>(s, i, all[i]);
        }
        off[0] = 0;
        for(int64_t i = 0; i < n; ++i)
            off[i + 1] = off[i] + int64_t(all[i].size());
        *total = off[n];
        if(off[n] > cap)
            return SPH_ERR_OVERFLOW;
        for(int64_t i = 0; i < n; ++i)
            for(size_t k = 0; k < all[i].size(); ++k)
            {
                js[off[i] + k] = all[i][k].j;
                for(int a = 0; a < 3; ++a)
                    offs[3 * (off[i] + k) + a] = all[i][k].o[a];
            }
        return SPH_OK;
    }

    /** Positions relative to the lower corner of each particle's cell (FP64),
     *  rel[3*i+a], and the cell edges of every box, edge[3*b+a]. */
    int orc_relpos(
        SphParams const* p,
        int32_t nbox,
        SphBox const* boxes,
        int64_t n,
        uint8_t const* roles,
        SphSoAView* v,
        double* rel,
        double* edge,
        int32_t* ncell)
    {
        orc::System s;
        int st = orc::setup(s, p, nbox, boxes, n, roles, v);
        if(st)
            return st;
        for(int64_t i = 0; i < n; ++i)
            orc::relPos<double>(s, i, &rel[3 * i]);
        for(int b = 0; b < nbox; ++b)
            for(int a = 0; a < 3; ++a)
            {
                edge[3 * b + a] = s.grids[b].edge[a];
                ncell[3 * b + a] = s.grids[b].n[a];
            }
        return SPH_OK;
    }

    //! UpdateDensity: rho of every target (FP64).
    int orc_density(
        SphParams const* p,
        int32_t nbox,
        SphBox const* boxes,
        int64_t n,
        uint8_t const* roles,
        SphSoAView* v,
        int32_t geom_fp32)
    {
        orc::System s;
        int st = orc::setup(s, p, nbox, boxes, n, roles, v);
        if(st)
            return st;
        orc::withKernel(
            s.p.kernel,
            [&](auto k)
            {
                orc::densityPass<decltype(k)>(s, geom_fp32 != 0);
                return 0;
            });
        return SPH_OK;
    }

    //! Force pass (hydro + AV + MHD + Dedner per params.physics) on the current density.
    int orc_force(
        SphParams const* p,
        int32_t nbox,
        SphBox const* boxes,
        int64_t n,
        uint8_t const* roles,
        SphSoAView* v,
        int32_t geom_fp32,
        double* ch,
        double* dtmin)
    {
        orc::System s;
        int st = orc::setup(s, p, nbox, boxes, n, roles, v);
        if(st)
            return st;
        orc::ForceOut fo = orc::withKernel(
            s.p.kernel,
            [&](auto k) { return orc::forcePass<decltype(k)>(s, geom_fp32 != 0); });
        for(int b = 0; b < nbox; ++b)
        {
            if(ch)
                ch[b] = fo.ch[b];
            if(dtmin)
                dtmin[b] = fo.dtmin[b];
        }
        return SPH_OK;
    }

    //! Conserved-quantity sums of the current state.
    int orc_reduce(
        SphParams const* p,
        int32_t nbox,
        SphBox const* boxes,
        int64_t n,
        uint8_t const* roles,
        SphSoAView* v,
        SphDiag* out)
    {
        orc::System s;
        if(!p || !out || !v)
            return SPH_ERR_INVALID;
        s.p = *p;
        s.n = n;
        s.roles = roles;
        s.v = v;
        s.nbox = nbox;
        (void) boxes;
        orc::diagnostics(s, *out);
        return SPH_OK;
    }

    /** Simulation::runOneStep, n_steps times (Simulation.x.cpp:233-300):
     *  drift (Movable), density, forces, kick (Movable & Thermodynamic).
     *  dt_state[b] holds box b's dt of the next step (updated from the box's CFL
     *  minimum when SPH_PHYS_CFL is set); time[b] accumulates its simulated time. */
    int orc_step(
        SphParams const* p,
        int32_t nbox,
        SphBox const* boxes,
        int64_t n,
        uint8_t const* roles,
        SphSoAView* v,
        int32_t geom_fp32,
        int32_t n_steps,
        double* dt_state,
        double* time,
        SphDiag* diag)
    {
        if(!p || !dt_state || !time)
            return SPH_ERR_INVALID;
        std::vector<double> dtUsed(nbox);
        for(int32_t step = 0; step < n_steps; ++step)
        {
            for(int b = 0; b < nbox; ++b)
                dtUsed[b] = dt_state[b];
            // drift: r += v dt (PushVelocity.hpp:38-41); periodic wrap into [lo, hi)
            for(int64_t i = 0; i < n; ++i)
            {
                if(!(roles[i] & SPH_ROLE_MOVABLE))
                    continue;
                int const b = v->box_id ? v->box_id[i] : 0;
                double const dt = dtUsed[b];
                for(int a = 0; a < 3; ++a)
                {
                    double x = v->pos[a][i] + orc::col(v->vel[a], i) * dt;
                    if(boxes[b].periodic[a])
                    {
                        double const L = boxes[b].hi[a] - boxes[b].lo[a];
                        if(x >= boxes[b].hi[a])
                            x -= L;
                        else if(x < boxes[b].lo[a])
                            x += L;
                    }
                    v->pos[a][i] = x;
                }
            }
            orc::System s;
            int st = orc::setup(s, p, nbox, boxes, n, roles, v);
            if(st)
                return st;
            orc::withKernel(
                s.p.kernel,
                [&](auto k)
                {
                    orc::densityPass<decltype(k)>(s, geom_fp32 != 0);
                    return 0;
                });
            orc::ForceOut fo = orc::withKernel(
                s.p.kernel,
                [&](auto k) { return orc::forcePass<decltype(k)>(s, geom_fp32 != 0); });
            // kick: v += dvdt dt, u += dudt dt (EulerIntegrate.hpp:45-51); B, psi likewise
            bool const mhd = p->physics & SPH_PHYS_MHD;
            for(int64_t i = 0; i < n; ++i)
            {
                if(!s.isTarget(i))
                    continue;
                double const dt = dtUsed[s.boxOf[i]];
                for(int a = 0; a < 3; ++a)
                    v->vel[a][i] += v->dvdt[a][i] * dt;
                v->u[i] += v->dudt[i] * dt;
                if((p->physics & SPH_PHYS_ADAPTIVE_H) && v->h)
                {
                    // h for the next step: hfact (m/rho)^(1/3), capped by the cell size
                    double const hn = p->hfact * std::cbrt(v->mass[i] / v->density[i]);
                    double const cap = s.hcap[s.boxOf[i]];
                    v->h[i] = hn < cap ? hn : cap;
                }
                if(mhd)
                {
                    for(int a = 0; a < 3; ++a)
                        v->B[a][i] += v->dBdt[a][i] * dt;
                    if(v->psi && v->dpsidt)
                        v->psi[i] += v->dpsidt[i] * dt;
                }
            }
            for(int b = 0; b < nbox; ++b)
            {
                time[b] += dtUsed[b];
                if((p->physics & SPH_PHYS_CFL) && fo.dtmin[b] < 1e300)
                    dt_state[b] = fo.dtmin[b];
            }
            if(diag)
            {
                orc::diagnostics(s, *diag);
                diag->time = time[0];
                diag->dt = dtUsed[0];
                diag->dt_next = dt_state[0];
                diag->c_h = fo.ch[0];
                diag->pairs = fo.pairs;
                diag->steps = step + 1;
            }
        }
        return SPH_OK;
    }
}
