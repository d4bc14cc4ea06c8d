// Device initialiser of lattice particle blocks.
//
// Replaces the reference's set-up path: setups made of blocks, each block a
// list of region volumes filled by a count recipe and a placement recipe
// (include/spearhed/particles/initialization/SetupInterface.hpp:34-113), the
// driver that counts, scans and places per region on the device
// (InitParticles.hpp:284-433), and the simple-cubic placement at cell centres
// with its per-axis count rule (spmacc/particles/initialization/SC.hpp:38-200).
// A C ABI cannot take the reference's recipe functors, so a block carries its
// state as data and the analytic fields of the validation setups are built-in
// profiles; a keep-mask (inside / outside a disc) selects lattice sites.
//
// Order and arithmetic: sites of a block are numbered x-fastest (the reference's
// mixed-radix decomposition); a site sits at lo + (i + 0.5) * (extent / n) with
// the product and sum rounded separately; kept sites are compacted in site
// order.  Jitter draws Philox4x64-10 (Salmon et al. 2011) uniforms in [-1, 1)
// per jitter group, value a * n_group + i for axis a of the group's particle i,
// the stream of numpy's Philox(key=seed).uniform(-1, 1, (3, n_group)).
#include "sph_launch.hpp"

#include <cmath>
#include <cstdint>
#include <limits>

namespace sph
{
    namespace
    {
        constexpr int kInitThreads = 256;

        //! Truncation of a positive quotient that snaps round-off just below an
        //! integer up to it (SC.hpp:49-58: four epsilons of the quotient).
        template<typename S>
        uint32_t truncateNearInteger(S value)
        {
            uint32_t const truncated = static_cast<uint32_t>(value);
            S const scale = value > S(1) ? value : S(1);
            S const tolerance = S(4) * std::numeric_limits<S>::epsilon() * scale;
            S const distanceToNext = static_cast<S>(truncated + 1u) - value;
            return (distanceToNext >= S(0) && distanceToNext <= tolerance) ? truncated + 1u : truncated;
        }

        template<typename S>
        void scCounts(S const lo[3], S const hi[3], S spacing, uint32_t n[3])
        {
            // axis 0 truncates (with the round-off snap); transverse axes round
            n[0] = truncateNearInteger((hi[0] - lo[0]) / spacing);
            n[0] = n[0] == 0u ? 1u : n[0];
            for(int a = 1; a < 3; ++a)
            {
                uint32_t const v = static_cast<uint32_t>((hi[a] - lo[a]) / spacing + S(0.5));
                n[a] = v == 0u ? 1u : v;
            }
        }

        // ---- Philox4x64-10 (Random123 constants: multipliers and Weyl key bumps)
        struct U64x4
        {
            unsigned long long v[4];
        };

        __device__ __forceinline__ U64x4 philox4x64(U64x4 c, unsigned long long k0, unsigned long long k1)
        {
            constexpr unsigned long long M0 = 0xD2E7470EE14C6C93ull, M1 = 0xCA5A826395121157ull;
            constexpr unsigned long long W0 = 0x9E3779B97F4A7C15ull, W1 = 0xBB67AE8584CAA73Bull;
#pragma unroll
            for(int r = 0; r < 10; ++r)
            {
                unsigned long long const hi0 = __umul64hi(M0, c.v[0]), lo0 = M0 * c.v[0];
                unsigned long long const hi1 = __umul64hi(M1, c.v[2]), lo1 = M1 * c.v[2];
                c = U64x4{{hi1 ^ c.v[1] ^ k0, lo1, hi0 ^ c.v[3] ^ k1, lo0}};
                k0 += W0;
                k1 += W1;
            }
            return c;
        }

        //! Value `index` of the uniform [-1, 1) stream keyed by `seed`: the
        //! counter runs from 1, four 64-bit words per counter, 53-bit mantissa.
        __device__ __forceinline__ double philoxUniform(unsigned long long seed, unsigned long long index)
        {
            U64x4 const r = philox4x64(U64x4{{index / 4 + 1, 0ull, 0ull, 0ull}}, seed, 0ull);
            unsigned long long const w = r.v[index % 4];
            double const d = __dmul_rn(double(w >> 11), 1.0 / 9007199254740992.0);
            return __dadd_rn(-1.0, __dmul_rn(2.0, d));
        }

        __device__ __forceinline__ int blockOfSite(LatticeBlockDev const* b, int nb, unsigned long long s)
        {
            int lo = 0, hi = nb - 1;
            while(lo < hi)
            {
                int const mid = (lo + hi + 1) >> 1;
                if(b[mid].siteBase <= s)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            return lo;
        }

        __device__ __forceinline__ void sitePosition(LatticeBlockDev const& b, unsigned long long local, double x[3])
        {
            unsigned long long accum = 1;
#pragma unroll
            for(int a = 0; a < 3; ++a)
            {
                unsigned long long const ik = (local / accum) % b.n[a];
                accum *= b.n[a];
                x[a] = __dadd_rn(b.lo[a], __dmul_rn(double(ik) + 0.5, b.d[a]));
            }
        }

        __device__ __forceinline__ bool keepSite(LatticeBlockDev const& b, double const x[3])
        {
            if(b.mask == SPH_MASK_NONE)
                return true;
            double const r = hypot(x[0] - b.maskCentre[0], x[1] - b.maskCentre[1]);
            return b.mask == SPH_MASK_INSIDE_DISC_XY ? r < b.maskRadius : r >= b.maskRadius;
        }

        __global__ void kLatticeFlags(LatticeBlockDev const* blocks, int nb, unsigned long long sites, uint32_t* flags)
        {
            for(unsigned long long s = blockIdx.x * blockDim.x + threadIdx.x; s < sites;
                s += static_cast<unsigned long long>(gridDim.x) * blockDim.x)
            {
                int const bi = blockOfSite(blocks, nb, s);
                double x[3];
                sitePosition(blocks[bi], s - blocks[bi].siteBase, x);
                flags[s] = keepSite(blocks[bi], x) ? 1u : 0u;
            }
        }

        __global__ void kLatticePlace(
            LatticeBlockDev const* blocks,
            int nb,
            unsigned long long sites,
            uint32_t const* flags,
            uint32_t const* ranks,
            InitColumns out)
        {
            for(unsigned long long s = blockIdx.x * blockDim.x + threadIdx.x; s < sites;
                s += static_cast<unsigned long long>(gridDim.x) * blockDim.x)
            {
                if(!flags[s])
                    continue;
                int const bi = blockOfSite(blocks, nb, s);
                LatticeBlockDev const& b = blocks[bi];
                double x[3];
                sitePosition(b, s - b.siteBase, x);
                uint32_t const i = ranks[s];
#pragma unroll
                for(int a = 0; a < 3; ++a)
                {
                    out.x[a][i] = x[a];
                    out.v[a][i] = b.vel[a];
                    out.B[a][i] = b.B[a];
                }
                out.m[i] = b.mass;
                out.h[i] = b.h;
                out.rho[i] = b.density;
                out.u[i] = b.u;
                out.psi[i] = b.psi;
                out.box[i] = b.box;
                out.group[i] = b.group;
            }
        }

        __global__ void kJitterProfile(InitColumns out, uint32_t n, JitterGroupDev const* groups, InitProfileDev prof)
        {
            for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                double x[3] = {out.x[0][i], out.x[1][i], out.x[2][i]};
                JitterGroupDev const& g = groups[out.group[i]];
                if(g.amplitude != 0.0)
                {
                    unsigned long long const k = i - g.first;
#pragma unroll
                    for(int a = 0; a < 3; ++a)
                        x[a] = __dadd_rn(x[a], __dmul_rn(g.amplitude, philoxUniform(g.seed, a * g.count + k)));
                }
#pragma unroll
                for(int a = 0; a < 3; ++a)
                    if(prof.wrap[a])
                    {
                        // Python-style modulo into [lo, lo + L)
                        double const L = prof.wrapHi[a] - prof.wrapLo[a];
                        double m = fmod(x[a] - prof.wrapLo[a], L);
                        if(m < 0.0)
                            m += L;
                        x[a] = prof.wrapLo[a] + m;
                    }
                double const pi2 = 2.0 * 3.141592653589793;
                if(prof.kind == SPH_PROFILE_ORSZAG_TANG)
                {
                    double const b0 = prof.p[0];
                    out.v[0][i] = -sin(pi2 * x[1]);
                    out.v[1][i] = sin(pi2 * x[0]);
                    out.B[0][i] = -b0 * sin(pi2 * x[1]);
                    out.B[1][i] = b0 * sin(2.0 * pi2 * x[0]);
                }
                else if(prof.kind == SPH_PROFILE_KH_PERTURBATION)
                    out.v[1][i] = prof.p[0] * sin(2.0 * pi2 * x[0]);
                else if(prof.kind == SPH_PROFILE_ROTOR)
                {
                    double const xc = prof.p[0], yc = prof.p[1], omega = prof.p[2], r0 = prof.p[3], r1 = prof.p[4];
                    double const width = prof.p[5]; // taper width (r1 - r0 as the setup states it)
                    double const r = hypot(x[0] - xc, x[1] - yc);
                    double const taper = fmin(fmax((r1 - r) / width, 0.0), 1.0);
                    double const w = r < r0 ? omega : omega * taper;
                    out.v[0][i] = -w * (x[1] - yc);
                    out.v[1][i] = w * (x[0] - xc);
                }
                for(int a = 0; a < 3; ++a)
                    out.x[a][i] = x[a];
            }
        }

        __global__ void kBlockFirstRanks(
            LatticeBlockDev const* blocks,
            int nb,
            unsigned long long sites,
            uint32_t const* flags,
            uint32_t const* ranks,
            uint32_t* first)
        {
            int const b = blockIdx.x * blockDim.x + threadIdx.x;
            if(b < nb)
                first[b] = blocks[b].siteBase < sites ? ranks[blocks[b].siteBase] : ranks[sites - 1] + flags[sites - 1];
            else if(b == nb)
                first[nb] = ranks[sites - 1] + flags[sites - 1];
        }

        unsigned gridFor(unsigned long long n)
        {
            unsigned long long const b = (n + kInitThreads - 1) / kInitThreads;
            return unsigned(b > 148ull * 64ull ? 148ull * 64ull : (b == 0 ? 1ull : b));
        }
    } // namespace

    void latticeCounts(double const lo[3], double const hi[3], double spacing, uint32_t n[3])
    {
        scCounts<double>(lo, hi, spacing, n);
    }

    void launchLatticeFlags(LatticeBlockDev const* blocks, int nb, unsigned long long sites, uint32_t* flags, cudaStream_t s)
    {
        kLatticeFlags<<<gridFor(sites), kInitThreads, 0, s>>>(blocks, nb, sites, flags);
        countLaunches(1);
    }

    void launchLatticePlace(
        LatticeBlockDev const* blocks,
        int nb,
        unsigned long long sites,
        uint32_t const* flags,
        uint32_t const* ranks,
        InitColumns const& out,
        cudaStream_t s)
    {
        kLatticePlace<<<gridFor(sites), kInitThreads, 0, s>>>(blocks, nb, sites, flags, ranks, out);
        countLaunches(1);
    }

    void launchBlockFirstRanks(
        LatticeBlockDev const* blocks,
        int nb,
        unsigned long long sites,
        uint32_t const* flags,
        uint32_t const* ranks,
        uint32_t* first,
        cudaStream_t s)
    {
        kBlockFirstRanks<<<unsigned((nb + 1 + 255) / 256), 256, 0, s>>>(blocks, nb, sites, flags, ranks, first);
        countLaunches(1);
    }

    void launchJitterProfile(
        InitColumns const& out,
        uint32_t n,
        JitterGroupDev const* groups,
        InitProfileDev const& prof,
        cudaStream_t s)
    {
        kJitterProfile<<<gridFor(n), kInitThreads, 0, s>>>(out, n, groups, prof);
        countLaunches(1);
    }
} // namespace sph

extern "C" int sph_sc_cell_counts(const double* lo, const double* hi, double spacing, uint32_t* counts)
{
    if(!lo || !hi || !counts || !(spacing > 0.0) || !std::isfinite(spacing))
        return SPH_ERR_INVALID;
    for(int a = 0; a < 3; ++a)
        if(!(hi[a] >= lo[a]))
            return SPH_ERR_INVALID;
    sph::scCounts<double>(lo, hi, spacing, counts);
    return SPH_OK;
}

extern "C" int sph_sc_cell_counts_f32(const float* lo, const float* hi, float spacing, uint32_t* counts)
{
    if(!lo || !hi || !counts || !(spacing > 0.0f) || !std::isfinite(spacing))
        return SPH_ERR_INVALID;
    for(int a = 0; a < 3; ++a)
        if(!(hi[a] >= lo[a]))
            return SPH_ERR_INVALID;
    sph::scCounts<float>(lo, hi, spacing, counts);
    return SPH_OK;
}
