// Pair kernels: neighbour build + density summation, and the force pass.
//
// Replaces the reference's pair engine (interact() -> FrameInteractionKernel /
// UnifiedFrameInteractionKernel, spmacc/particles/algorithms/InteractParticles.hpp:140-199,
// ParticleParticleInteraction.hpp:219-612) and the functors it drives
// (AccumulateDensity, DensitySummation.hpp:50-74; HydroInteraction,
// HydroForces.hpp:86-176), plus the viscosity, SPMHD and Dedner terms the
// reference lacks.
//
// Density kernel: one warp per target cell (cell edge >= cull radius).  The
// warp stages the 27-cell stencil's sources into shared memory with the
// stencil shift already added (the reference's origin-shifted staging,
// ParticleParticleInteraction.hpp:241-265), each lane owns one target and
// sweeps the staged candidates with broadcast reads, culling with r^2
// evaluated unfused in x, y, z order exactly as the reference's CPU path does.
// Accepted pairs are written to the target's neighbour-list row (sorted source
// index + stencil slot); the density sum then runs over the compact row, so
// the kernel arithmetic runs on accepted pairs only, with every lane busy.
// The epilogue writes rho (FP64) and the target's derived record for the force
// pass.
//
// Force kernel: one thread per sorted target, over its list row, gathering the
// neighbours' 64-byte (FP32) or 128-byte (FP64) records through L1.
//
// Precision: FP32 kernels accumulate every per-particle sum with CompAcc
// (blocks of 8 terms folded by TwoSum); FP64 kernels sum plainly.
#include "sph_launch.hpp"

namespace sph
{
    namespace
    {
        constexpr int kDensWarps = 4;
        constexpr int kForceThreads = 128;
        constexpr int kBlock = 8; //!< terms per compensated block

        template<typename T>
        struct PairCfg;
        template<>
        struct PairCfg<float>
        {
            using V4 = float4;
            static constexpr int kStageBatch = 2; //!< staged positions per lane with loads in flight
        };
        template<>
        struct PairCfg<double>
        {
            using V4 = D4;
            static constexpr int kStageBatch = 2;
        };

        template<typename T>
        __device__ __forceinline__ Records<typename PairCfg<T>::V4, T> records(DevCtx const& c);
        template<>
        __device__ __forceinline__ Records<float4, float> records<float>(DevCtx const& c)
        {
            return c.r32;
        }
        template<>
        __device__ __forceinline__ Records<D4, double> records<double>(DevCtx const& c)
        {
            return c.r64;
        }

        template<typename T>
        __device__ __forceinline__ typename PairCfg<T>::V4 const* shiftTable(DevCtx const& c, int box);
        template<>
        __device__ __forceinline__ float4 const* shiftTable<float>(DevCtx const& c, int box)
        {
            return c.shift32 + size_t(box) * 32;
        }
        template<>
        __device__ __forceinline__ D4 const* shiftTable<double>(DevCtx const& c, int box)
        {
            return c.shift64 + size_t(box) * 32;
        }

        //! Paired FP32 arithmetic (sm_100 f32x2) that rounds like the reference's
        //! unfused scalar x, y, z sum.  A paired multiply feeding a paired add is
        //! contracted into a fused multiply-add even when both are written in
        //! PTX with an explicit .rn (measured on sm_100a: r^2 then differs from
        //! the scalar __fmul_rn/__fadd_rn sum by one ulp, which moves pairs at
        //! r^2 = R^2 across the cull).  Squares are therefore formed as
        //! fma.rn(a, a, zero) with a zero the compiler cannot see (one computed
        //! from a kernel argument): that is round(a^2) exactly, and an add of
        //! two fused results has nothing left to contract.
        __device__ __forceinline__ float2 add2Rn(float2 a, float2 b)
        {
            unsigned long long r;
            asm("add.rn.f32x2 %0, %1, %2;"
                : "=l"(r)
                : "l"(*reinterpret_cast<unsigned long long const*>(&a)),
                  "l"(*reinterpret_cast<unsigned long long const*>(&b)));
            return *reinterpret_cast<float2 const*>(&r);
        }
        __device__ __forceinline__ float2 sq2Rn(float2 a, float2 zero)
        {
            unsigned long long r;
            asm("fma.rn.f32x2 %0, %1, %1, %2;"
                : "=l"(r)
                : "l"(*reinterpret_cast<unsigned long long const*>(&a)),
                  "l"(*reinterpret_cast<unsigned long long const*>(&zero)));
            return *reinterpret_cast<float2 const*>(&r);
        }
        //! A run-time zero: R * 0 with R a finite kernel argument.  IEEE
        //! arithmetic does not let the compiler fold it (R could be NaN or
        //! infinite), so it stays opaque to contraction.
        __device__ __forceinline__ float2 opaqueZero2(float R)
        {
            float const z = __fmul_rn(R, 0.0f);
            return make_float2(z, z);
        }

        // Unfused arithmetic: the reference's CPU evaluation of the pair geometry.
        __device__ __forceinline__ float mulRn(float a, float b)
        {
            return __fmul_rn(a, b);
        }
        __device__ __forceinline__ float addRn(float a, float b)
        {
            return __fadd_rn(a, b);
        }
        __device__ __forceinline__ double mulRn(double a, double b)
        {
            return __dmul_rn(a, b);
        }
        __device__ __forceinline__ double addRn(double a, double b)
        {
            return __dadd_rn(a, b);
        }
        __device__ __forceinline__ float rsqrtT(float x)
        {
            return rsqrtf(x);
        }
        __device__ __forceinline__ double rsqrtT(double x)
        {
            return rsqrt(x);
        }
        __device__ __forceinline__ float rcpT(float x)
        {
            return __fdividef(1.0f, x);
        }
        __device__ __forceinline__ double rcpT(double x)
        {
            return 1.0 / x;
        }

        //! Division in the pair precision: fast in FP32 (the pair terms carry no
        //! tighter requirement), IEEE in FP64.
        __device__ __forceinline__ float divT(float a, float b)
        {
            return __fdividef(a, b);
        }
        __device__ __forceinline__ double divT(double a, double b)
        {
            return a / b;
        }

        template<typename T>
        __device__ __forceinline__ T edgeOf(BoxDev const& B, int a);
        template<>
        __device__ __forceinline__ float edgeOf<float>(BoxDev const& B, int a)
        {
            return B.edgef[a];
        }
        template<>
        __device__ __forceinline__ double edgeOf<double>(BoxDev const& B, int a)
        {
            return B.edge[a];
        }

        //! Accumulator: FP32 compensated (CompAcc + block partial) or FP64 plain.
        template<typename T>
        struct Acc;
        template<>
        struct Acc<float>
        {
            CompAcc c;
            float part = 0.f;
            __device__ __forceinline__ void add(float x)
            {
                part += x;
            }
            __device__ __forceinline__ void fold()
            {
                c.fold(part);
                part = 0.f;
            }
            __device__ __forceinline__ double value() const
            {
                return c.value();
            }
        };
        template<>
        struct Acc<double>
        {
            double s = 0.0;
            __device__ __forceinline__ void add(double x)
            {
                s += x;
            }
            __device__ __forceinline__ void fold()
            {
            }
            __device__ __forceinline__ double value() const
            {
                return s;
            }
        };

        __device__ __forceinline__ uint32_t warpMaxU(uint32_t v)
        {
#pragma unroll
            for(int o = 16; o > 0; o >>= 1)
                v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
            return v;
        }
        __device__ __forceinline__ unsigned long long warpSumU64(unsigned long long v)
        {
#pragma unroll
            for(int o = 16; o > 0; o >>= 1)
                v += __shfl_xor_sync(0xffffffffu, v, o);
            return v;
        }
        __device__ __forceinline__ double warpMaxD(double v)
        {
#pragma unroll
            for(int o = 16; o > 0; o >>= 1)
                v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
            return v;
        }
        __device__ __forceinline__ double warpMinD(double v)
        {
#pragma unroll
            for(int o = 16; o > 0; o >>= 1)
                v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
            return v;
        }

        template<typename T>
        __device__ __forceinline__ T warpMinT(T v)
        {
#pragma unroll
            for(int o = 16; o > 0; o >>= 1)
            {
                T const w = __shfl_xor_sync(0xffffffffu, v, o);
                v = w < v ? w : v;
            }
            return v;
        }
        template<typename T>
        __device__ __forceinline__ T warpMaxT(T v)
        {
#pragma unroll
            for(int o = 16; o > 0; o >>= 1)
            {
                T const w = __shfl_xor_sync(0xffffffffu, v, o);
                v = w > v ? w : v;
            }
            return v;
        }

        //! Lanes per target for a chunk of nt targets (power of two, nt * S <= 32):
        //! a full chunk gives every lane its own target; a short chunk spreads each
        //! target over S lanes that take consecutive blocks of four candidates.
        __device__ __forceinline__ int subLanes(uint32_t nt)
        {
            return nt > 16 ? 1 : (nt > 8 ? 2 : (nt > 4 ? 4 : (nt > 2 ? 8 : (nt > 1 ? 16 : 32))));
        }

        //! Compensated-sum combine of two (hi, lo) partials (TwoSum on the heads).
        __device__ __forceinline__ void combineComp(float& hi, float& lo, float ohi, float olo)
        {
            float s, e;
            twoSum(hi, ohi, s, e);
            hi = s;
            lo = lo + olo + e;
        }

        //! Far coordinate written into the staged tail past the last candidate:
        //! its r^2 overflows (FP32) or dwarfs any cull radius (FP64).
        constexpr float kFar = 1e30f;

        //! Acceptance mask of 32 staged candidates X/Y/Z[0..31] (negated, shifted
        //! source positions) for one target: bit 31-u set when candidate u has
        //! r^2 < R^2.  r^2 is the unfused x, y, z sum of the reference's CPU path;
        //! the test reads the sign of the exactly rounded r^2 - R^2, which is
        //! negative exactly when r^2 < R^2, and funnels it into the mask.
        //! FP32: two candidates per instruction with the paired f32x2 arithmetic
        //! of sm_100 (round-to-nearest per element, the scalar rounding).
        //! UNR: how many of the eight 4-candidate groups the compiler unrolls
        //! (8 = all; 2 keeps the hot code small where warps run several phases
        //! at once and the instruction caches become the bound).
        template<bool PAIRMAX, int UNR>
        __device__ __forceinline__ uint32_t cullMask32(
            float4 const& own,
            float nRi2,
            float const* X,
            float const* Y,
            float const* Z,
            float const* H,
            float supT,
            float R2g)
        {
            float2 const ox = make_float2(own.x, own.x);
            float2 const oy = make_float2(own.y, own.y);
            float2 const oz = make_float2(own.z, own.z);
            float2 const nR2 = make_float2(-R2g, -R2g);
            float2 const zero = opaqueZero2(supT);
            uint32_t mask = 0;
#pragma unroll UNR
            for(int q = 0; q < 32; q += 4)
            {
                float4 const xv = *reinterpret_cast<float4 const*>(X + q);
                float4 const yv = *reinterpret_cast<float4 const*>(Y + q);
                float4 const zv = *reinterpret_cast<float4 const*>(Z + q);
                float4 hv{};
                if constexpr(PAIRMAX)
                    hv = *reinterpret_cast<float4 const*>(H + q);
#pragma unroll
                for(int p = 0; p < 2; ++p)
                {
                    float2 const dx = add2Rn(ox, p ? make_float2(xv.z, xv.w) : make_float2(xv.x, xv.y));
                    float2 const dy = add2Rn(oy, p ? make_float2(yv.z, yv.w) : make_float2(yv.x, yv.y));
                    float2 const dz = add2Rn(oz, p ? make_float2(zv.z, zv.w) : make_float2(zv.x, zv.y));
                    float2 const r2 = add2Rn(add2Rn(sq2Rn(dx, zero), sq2Rn(dy, zero)), sq2Rn(dz, zero));
                    float2 nr = nR2;
                    if constexpr(PAIRMAX)
                    {
                        // -(supT max(h_i, h_j))^2 = min(-(supT h_i)^2, -(supT h_j)^2):
                        // the rounded product and square are monotone in h
                        float const n0 = p ? hv.z : hv.x, n1 = p ? hv.w : hv.y;
                        nr = make_float2(fminf(nRi2, n0), fminf(nRi2, n1));
                    }
                    float2 const d = add2Rn(r2, nr);
                    mask = __funnelshift_l(__float_as_uint(d.x), mask, 1);
                    mask = __funnelshift_l(__float_as_uint(d.y), mask, 1);
                }
            }
            return mask;
        }

        template<bool PAIRMAX, int UNR>
        __device__ __forceinline__ uint32_t cullMask32(
            D4 const& own,
            double nRi2,
            double const* X,
            double const* Y,
            double const* Z,
            double const* H,
            double supT,
            double R2g)
        {
            uint32_t mask = 0;
#pragma unroll 4
            for(int q = 0; q < 32; q += 2)
            {
                double2 const xv = *reinterpret_cast<double2 const*>(X + q);
                double2 const yv = *reinterpret_cast<double2 const*>(Y + q);
                double2 const zv = *reinterpret_cast<double2 const*>(Z + q);
#pragma unroll
                for(int p = 0; p < 2; ++p)
                {
                    double const dx = __dadd_rn(own.x, p ? xv.y : xv.x);
                    double const dy = __dadd_rn(own.y, p ? yv.y : yv.x);
                    double const dz = __dadd_rn(own.z, p ? zv.y : zv.x);
                    double const r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                    double nR2 = -R2g;
                    if constexpr(PAIRMAX)
                        nR2 = fmin(nRi2, H[q + p]);
                    double const d = __dadd_rn(r2, nR2);
                    mask = __funnelshift_l(uint32_t(__double2hiint(d)), mask, 1);
                }
            }
            return mask;
        }

        //! Staged columns are laid out in 32-candidate slabs, each followed by 16
        //! bytes of padding: the sub-lanes of a short chunk read the same offset
        //! of different slabs at once, and the skew puts up to eight such slabs
        //! on different shared-memory banks.  skewed(q) is the column index of
        //! window position q; a slab's 32 candidates stay contiguous.
        __device__ __forceinline__ uint32_t skewed(uint32_t q)
        {
            return q + ((q >> 5) << 2);
        }
        template<int CAP>
        constexpr int colLen()
        {
            return CAP + CAP / 8;
        }

        //! Per-lane state of one chunk of up to 32 targets of a cell.
        template<typename V4, typename T>
        struct TargetChunk
        {
            V4 own;
            T hi;
            T nR2;             //!< -(supT h_i)^2, the target's side of the pair-max cull radius
            uint32_t t;        //!< sorted target index
            uint32_t nl;       //!< accepted so far (same on every lane of the target's group)
            uint4 buf;         //!< full chunks: the last (nl mod 4) accepted entries, newest in w
            int S, sub;
            bool act;
        };

        template<typename V4, typename T>
        __device__ __forceinline__ void initChunk(
            TargetChunk<V4, T>& ch,
            Records<V4, T> const& rec,
            uint32_t tc,
            uint32_t tEnd,
            int lane,
            T supT)
        {
            uint32_t const nt = tc < tEnd ? min(32u, tEnd - tc) : 0u;
            ch.S = subLanes(nt == 0 ? 32u : nt);
            ch.sub = lane & (ch.S - 1);
            uint32_t const tt = uint32_t(lane) / uint32_t(ch.S);
            ch.act = tt < nt;
            ch.t = tc + tt;
            ch.nl = 0;
            ch.buf = make_uint4(0, 0, 0, 0);
            ch.own = V4{};
            ch.hi = T(1);
            if(ch.act)
            {
                ch.own = ld4(rec.pm + ch.t);
                ch.hi = rec.hc[ch.t];
            }
            T const Ri = mulRn(supT, ch.hi);
            ch.nR2 = -mulRn(Ri, Ri);
        }

        //! Cull the staged candidates [0, m) against one target chunk and append
        //! the accepted entries, in candidate order, to each target's list row.
        //! The staging holds negated shifted positions (sNX, sNY, sNZ), so
        //! dx = x_i + (-x_j) is the reference's x_i - x_j, rounding included; the
        //! window is padded with far candidates up to a multiple of 32.
        template<typename V4, typename T, bool PAIRMAX, int UNR>
        __device__ __forceinline__ void cullChunk(
            TargetChunk<V4, T>& ch,
            T const* sNX,
            T const* sNY,
            T const* sNZ,
            T const* sH,
            uint32_t const* sEnt,
            uint32_t const* sSelf,
            uint32_t tc,
            uint32_t m,
            T supT,
            T R2g,
            uint32_t* list,
            uint32_t cap,
            bool countOnly)
        {
            uint32_t* const row = list + size_t(ch.t) * cap;
            // The window is far-padded to whole 32-candidate slabs.  A target has
            // S lanes (S = 1 for a full chunk); in round r sub-lane s builds the
            // acceptance mask of slab r S + s (all lanes of a full chunk read the
            // same candidates: shared-memory broadcast) and clears the bit of the
            // target's own entry (its window position, recorded at staging).  One
            // call site of the mask cull serves both kinds of chunk, which keeps
            // the kernel's hot code small.
            int const S = ch.S;
            uint32_t const selfq = ch.act ? sSelf[ch.t - tc] : ~0u;
            uint32_t const nSlab = (m + 31u) >> 5;
            for(uint32_t g0 = 0; g0 < nSlab; g0 += uint32_t(S))
            {
                uint32_t const g = g0 + uint32_t(ch.sub);
                uint32_t const q0 = g << 5;
                uint32_t mask = 0;
                if(g < nSlab)
                {
                    uint32_t const c0 = skewed(q0);
                    mask = cullMask32<PAIRMAX, UNR>(ch.own, ch.nR2, sNX + c0, sNY + c0, sNZ + c0, sH + c0, supT, R2g);
                    if(!ch.act)
                        mask = 0;
                    if(selfq - q0 < 32u)
                        mask &= ~(0x80000000u >> (selfq - q0));
                }
                uint32_t const cnt = uint32_t(__popc(mask));
                if(S == 1)
                {
                    // full chunk: the lane's row grows by its own entries, four at
                    // a time (16-byte stores; rows are 32-byte aligned and cap is a
                    // multiple of 8)
                    if(countOnly)
                    {
                        ch.nl += cnt;
                        continue;
                    }
                    while(mask)
                    {
                        uint32_t const u = uint32_t(__clz(mask));
                        mask &= 0x7fffffffu >> u;
                        ch.buf = make_uint4(ch.buf.y, ch.buf.z, ch.buf.w, sEnt[q0 + u]);
                        ++ch.nl;
                        if((ch.nl & 3u) == 0 && ch.nl <= cap)
                            *reinterpret_cast<uint4*>(row + (ch.nl - 4)) = ch.buf;
                    }
                    continue;
                }
                // short chunk: an exclusive scan of the accepted counts over the
                // target's S lanes places each slab's entries in candidate order
                uint32_t incl = cnt;
                for(int d = 1; d < S; d <<= 1)
                {
                    uint32_t const o = __shfl_up_sync(0xffffffffu, incl, d, S);
                    if(ch.sub >= d)
                        incl += o;
                }
                uint32_t const total = __shfl_sync(0xffffffffu, incl, S - 1, S);
                if(!countOnly)
                {
                    uint32_t k = ch.nl + incl - cnt;
                    while(mask)
                    {
                        uint32_t const u = uint32_t(__clz(mask));
                        mask &= 0x7fffffffu >> u;
                        if(k < cap)
                            row[k] = sEnt[q0 + u];
                        ++k;
                    }
                }
                ch.nl += total;
            }
        }

        //! Writes a full chunk's buffered tail (the last nl mod 4 entries).
        template<typename V4, typename T>
        __device__ __forceinline__ void flushChunk(TargetChunk<V4, T> const& ch, uint32_t* list, uint32_t cap)
        {
            if(!ch.act || ch.S != 1)
                return;
            uint32_t const r = ch.nl & 3u;
            uint32_t const base = ch.nl - r;
            uint32_t* const row = list + size_t(ch.t) * cap;
            // buffered entries base .. base+r-1 sit in buf's last r components
            uint32_t const e[3] = {r == 3 ? ch.buf.y : (r == 2 ? ch.buf.z : ch.buf.w), r == 3 ? ch.buf.z : ch.buf.w, ch.buf.w};
#pragma unroll
            for(uint32_t i = 0; i < 3; ++i)
                if(i < r && base + i < cap)
                    row[base + i] = e[i];
        }

        //! Density of one target chunk over its list rows; writes rho, the
        //! count and the force-pass records.  Returns the chunk's max c.
        template<int K, typename V4, typename T>
        __device__ __forceinline__ double densityChunk(
            TargetChunk<V4, T> const& ch,
            DevCtx const& c,
            Records<V4, T> const& rec,
            PhysArgs const& pa,
            V4 const* stab,
            uint32_t cap)
        {
            bool const lead = ch.act && ch.sub == 0;
            uint32_t const n = ch.act ? min(ch.nl, cap) : 0u;
            uint32_t const* row = c.lists.list + size_t(ch.t) * cap;
            HConst<T> const hk = hconst<K, T>(ch.hi);
            Acc<T> rho;
            if(lead)
                rho.add(ch.own.w * kernelW<K, T>(T(0), hk));
            int const S = ch.S;
            auto term = [&](V4 const& pj, V4 const& o)
            {
                T const dx = ch.own.x - (pj.x + o.x);
                T const dy = ch.own.y - (pj.y + o.y);
                T const dz = ch.own.z - (pj.z + o.z);
                T const r2 = dx * dx + dy * dy + dz * dz;
                T const y = rsqrtT(r2);
                T const r = r2 > T(0) ? r2 * y : T(0);
                rho.add(pj.w * kernelW<K, T>(r, hk));
            };
            if(S == 1)
            {
                // Full chunk: the row four entries at a time, the next source's
                // record in flight; blocks of 8 terms as below.
                uint4 const* row4 = reinterpret_cast<uint4 const*>(row);
                V4 npm{};
                uint32_t nslot = 0;
                auto fetch = [&](uint32_t e)
                {
                    if(!checkIndex((e >> 5) < c.n, c.status, kChkRowEntry))
                        e = 0;
                    nslot = e & 31u;
                    npm = ld4(rec.pm + (e >> 5));
                };
                auto step = [&](uint32_t next)
                {
                    V4 const pj = npm;
                    V4 const o = ld4(stab + nslot);
                    fetch(next);
                    term(pj, o);
                };
                uint4 qc = make_uint4(0, 0, 0, 0);
                if(n > 0)
                {
                    qc = row4[0];
                    fetch(qc.x);
                }
                uint32_t const nFull = n & ~3u;
                for(uint32_t k0 = 0; k0 < nFull; k0 += 4)
                {
                    step(qc.y);
                    step(qc.z);
                    step(qc.w);
                    bool const more = k0 + 4 < n;
                    uint4 const qn = more ? row4[(k0 >> 2) + 1] : qc;
                    step(more ? qn.x : qc.w);
                    if(k0 & 4u)
                        rho.fold();
                    qc = qn;
                }
                // the last 1-3 entries (qc.x already fetched); a loop that is not
                // unrolled keeps one copy of the term, and the fetch after the
                // last entry re-reads qc.x, a valid entry
                uint32_t const tail = n - nFull;
#pragma unroll 1
                for(uint32_t i = 0; i < tail; ++i)
                    step(i + 1 < tail ? (i == 0 ? qc.y : qc.z) : qc.x);
            }
            uint32_t k = S == 1 ? n : uint32_t(ch.sub);
            while(k < n)
            {
                for(int b = 0; b < kBlock && k < n; ++b, k += uint32_t(S))
                {
                    uint32_t e = row[k];
                    if(!checkIndex((e >> 5) < c.n, c.status, kChkRowEntry))
                        e = 0;
                    term(ld4(rec.pm + (e >> 5)), ld4(stab + (e & 31u)));
                }
                rho.fold();
            }
            rho.fold();
            double rhoD;
            if constexpr(sizeof(T) == 4)
            {
                float rh = rho.c.hi, rl = rho.c.lo;
                for(int off = S >> 1; off > 0; off >>= 1)
                {
                    float const oh = __shfl_down_sync(0xffffffffu, rh, off, S);
                    float const ol = __shfl_down_sync(0xffffffffu, rl, off, S);
                    combineComp(rh, rl, oh, ol);
                }
                rhoD = double(rh) + double(rl);
            }
            else
            {
                double v = rho.value();
                for(int off = S >> 1; off > 0; off >>= 1)
                    v += __shfl_down_sync(0xffffffffu, v, off, S);
                rhoD = v;
            }
            if(!lead)
                return 0.0;
            uint32_t const t = ch.t;
            c.cur.rho[t] = rhoD;
            c.lists.count[t] = ch.nl;
            double Bv[3] = {c.cur.B[0][t], c.cur.B[1][t], c.cur.B[2][t]};
            double ft[4], fb[4];
            derivedRecord(rhoD, c.cur.u[t], Bv, c.cur.psi[t], pa, ft, fb);
            rec.ft[t] = mk4<V4>(ft[0], ft[1], ft[2], ft[3]);
            rec.fb[t] = mk4<V4>(fb[0], fb[1], fb[2], fb[3]);
            return ft[2];
        }

        //! Tunable launch shapes (picked per context by sph_autotune): CAP is the
        //! staging depth (candidates per shared-memory window), MINB the blocks
        //! per SM the register allocation must admit, CU the unroll depth of the
        //! FP32 mask cull (8 or 2; the FP64 cull ignores it).
        template<int K, typename T, bool PAIRMAX, int CAP, int MINB, int CU>
        __global__ void __launch_bounds__(kDensWarps * 32, MINB) kDensity(DevCtx c, PhysArgs pa, bool countOnly)
        {
            using V4 = typename PairCfg<T>::V4;
            extern __shared__ __align__(32) unsigned char smem[];
            int const warp = threadIdx.x >> 5;
            int const lane = threadIdx.x & 31;
            // per warp: negated shifted x, y, z, (pair-max cull) smoothing length, list entry
            constexpr int kCols = PAIRMAX ? 4 : 3;
            // (columns in skewed slabs, see skewed())
            constexpr int kCol = colLen<CAP>();
            T* const sNX = reinterpret_cast<T*>(smem) + warp * kCol;
            T* const sNY = sNX + kDensWarps * kCol;
            T* const sNZ = sNY + kDensWarps * kCol;
            T* const sH = sNZ + kDensWarps * kCol; // only with PAIRMAX: -(supT h_j)^2
            uint32_t* const sEnt = reinterpret_cast<uint32_t*>(reinterpret_cast<T*>(smem) + kCols * kDensWarps * kCol)
                                   + warp * CAP;
            // per warp: window position of each target's own entry (up to 64
            // targets of the chunk pair; ~0 = not in this window)
            uint32_t* const sSelf = reinterpret_cast<uint32_t*>(reinterpret_cast<T*>(smem) + kCols * kDensWarps * kCol)
                                    + kDensWarps * CAP + warp * 64;
            Records<V4, T> const rec = records<T>(c);
            T const supT = T(Kern<K>::support);
            T const Rg = mulRn(supT, T(pa.h0));
            T const R2g = mulRn(Rg, Rg);
            uint32_t const cap = c.lists.cap;
            uint32_t maxCount = 0;
            unsigned long long pairs = 0;
            unsigned long long cand = 0; // warp-uniform: staged sources x targets culled
            double chMax = 0.0;
            int chBox = -1; // box whose c_h maximum chMax holds (warp-uniform)

            // Work queue over the cells of the boxes' current grids: each warp
            // takes its next item from a counter; the fetch for the next item is
            // issued first and read at the loop's end.  Item q is cell
            // q - activeBase of the box whose range holds it.
            uint32_t const nWork = *c.activeTotal;
            uint32_t pending = 0;
            if(lane == 0)
                pending = atomicAdd(c.work, 1u);
            for(uint32_t q = __shfl_sync(0xffffffffu, pending, 0); q < nWork; q = __shfl_sync(0xffffffffu, pending, 0))
            {
                if(lane == 0)
                    pending = atomicAdd(c.work, 1u);
                int const box = boxOfWork(c.boxes, c.nbox, q);
                // item -> cell: the box's level-0 cells first, then its level-1 cells
                uint32_t const l = q - c.boxes[box].activeBase;
                uint32_t const nc0 = c.boxes[box].ncells;
                uint32_t const cell = c.boxes[box].cellBase + (l < nc0 ? l : c.boxes[box].ncellsMax + (l - nc0));
                if(!checkIndex(cell < c.cells.ncells, c.status, kChkCell))
                    continue;
                uint32_t const tBeg = c.cells.start[cell];
                uint32_t const tEnd = c.cells.mid[cell];
                if(tBeg >= tEnd || !checkIndex(tEnd <= c.n, c.status, kChkTargets))
                    continue;
                if(box != chBox)
                {
                    // flush the previous box's signal-speed maximum
                    double const m = warpMaxD(chMax);
                    if(lane == 0 && chBox >= 0 && !countOnly)
                        atomicMax(&c.bs.chBits[chBox], orderedBits(m));
                    chMax = 0.0;
                    chBox = box;
                }
                BoxDev const& B = c.boxes[box];
                // Target cell: level 0 (the grid) or level 1 (one of the m0 x m1 x m2
                // sub-cells of a level-0 cell, numbered parent-major), its level-0
                // parent c0 and, for level 1, its coordinates ct on the fine grid
                // (m_a n_a cells per axis).
                int const lt = l < B.ncells ? 0 : 1;
                int ct[3], c0[3];
                {
                    uint32_t const li = lt ? l - B.ncells : l;
                    uint32_t const par = lt ? li / B.msub : li;
                    uint32_t const n0 = uint32_t(B.n[0]), n1 = uint32_t(B.n[1]);
                    c0[0] = int(par % n0);
                    c0[1] = int((par / n0) % n1);
                    c0[2] = int(par / (n0 * n1));
                    uint32_t sub = lt ? li - par * B.msub : 0u;
#pragma unroll
                    for(int a = 0; a < 3; ++a)
                    {
                        uint32_t const sh = uint32_t(B.m[a] - 1); // splits are 1 or 2
                        ct[a] = (c0[a] << sh) + int(sub & sh);
                        sub >>= sh;
                    }
                }
                // Candidate descriptors: the 27 level-0 cells around the parent, then
                // with two levels either the 27 level-1 cells around a level-1 target
                // or, for a level-0 target, the level-1 block (all sub-cells) of each
                // of those 27 cells.  Each carries its source range and the level-0
                // stencil slot of its image.
                int const nDesc = 27 + (B.levels == 2 ? 27 : 0);
                auto describe = [&](int d, uint32_t& sBeg, uint32_t& sCnt, uint32_t& slot, T sh[3])
                {
                    sBeg = 0;
                    sCnt = 0;
                    slot = 0;
                    sh[0] = sh[1] = sh[2] = T(0);
                    if(d >= nDesc)
                        return;
                    int o[3], f[3];
                    bool ok = true;
                    bool const fine = d >= 27;
                    int const k = fine ? d - 27 : d;
                    bool const fineCell = fine && lt; // a level-1 neighbour of a level-1 target
#pragma unroll
                    for(int a = 0; a < 3; ++a)
                    {
                        int const n0 = B.n[a];
                        if(fineCell)
                        {
                            // fine-grid neighbour; its level-0 parent (image-aware) gives o
                            int const sh = B.m[a] - 1; // splits are 1 or 2
                            int const n1 = n0 << sh;
                            int const fa = ct[a] + stencilOff(k, a);
                            o[a] = (fa >> sh) - c0[a];
                            f[a] = fa < 0 || fa >= n1 ? (B.periodic[a] ? (fa + n1) % n1 : -1) : fa;
                            ok = ok && f[a] >= 0;
                        }
                        else
                        {
                            o[a] = stencilOff(k, a);
                            int ca = c0[a] + o[a];
                            if(ca < 0 || ca >= n0)
                            {
                                if(B.periodic[a])
                                    ca = (ca + n0) % n0;
                                else
                                    ok = false;
                            }
                            f[a] = ca;
                        }
                    }
                    slot = uint32_t((o[0] + 1) + 3 * (o[1] + 1) + 9 * (o[2] + 1));
#pragma unroll
                    for(int a = 0; a < 3; ++a)
                        sh[a] = T(o[a]) * edgeOf<T>(B, a);
                    if(!ok)
                        return;
                    if(fineCell)
                    {
                        int p[3];
                        uint32_t subc = 0, stride = 1;
#pragma unroll
                        for(int a = 0; a < 3; ++a)
                        {
                            int const sh = B.m[a] - 1;
                            p[a] = f[a] >> sh;
                            subc += uint32_t(f[a] & sh) * stride;
                            stride <<= sh;
                        }
                        uint32_t const par = (uint32_t(p[2]) * uint32_t(B.n[1]) + uint32_t(p[1])) * uint32_t(B.n[0])
                                             + uint32_t(p[0]);
                        uint32_t const cellId = B.cellBase + B.ncellsMax + par * B.msub + subc;
                        if(!checkIndex(cellId < c.cells.ncells, c.status, kChkCell))
                            return;
                        sBeg = c.cells.start[cellId];
                        sCnt = c.cells.end[cellId] - sBeg;
                        if(!checkIndex(sBeg <= c.n && sCnt <= c.n - sBeg, c.status, kChkRange))
                            sCnt = 0;
                        return;
                    }
                    uint32_t const cellId
                        = B.cellBase + (uint32_t(f[2]) * uint32_t(B.n[1]) + uint32_t(f[1])) * uint32_t(B.n[0]) + uint32_t(f[0]);
                    if(!checkIndex(cellId < c.cells.ncells, c.status, kChkCell))
                        return;
                    if(fine)
                    {
                        // all level-1 sub-cells of a level-0 neighbour, as one range
                        sBeg = c.cells.bstart[cellId];
                        sCnt = c.cells.bend[cellId] - sBeg;
                    }
                    else
                    {
                        sBeg = c.cells.start[cellId];
                        sCnt = c.cells.end[cellId] - sBeg;
                    }
                    if(!checkIndex(sBeg <= c.n && sCnt <= c.n - sBeg, c.status, kChkRange))
                        sCnt = 0;
                };

                // exclusive prefix of the page's source counts and the page total
                auto scan = [&](uint32_t cnt, uint32_t& pre, uint32_t& total)
                {
                    uint32_t incl = cnt;
#pragma unroll
                    for(int d = 1; d < 32; d <<= 1)
                    {
                        uint32_t const o = __shfl_up_sync(0xffffffffu, incl, d);
                        if(lane >= d)
                            incl += o;
                    }
                    pre = incl - cnt;
                    total = __shfl_sync(0xffffffffu, incl, 31);
                };
                // Page 0 (all of a single-level box's 27 slots) is described once per
                // cell; later pages once per target chunk.
                uint32_t sBeg0, sCnt0, slot0, pre0, total0;
                T sh0[3];
                describe(lane, sBeg0, sCnt0, slot0, sh0);
                scan(sCnt0, pre0, total0);

                // Two target chunks (up to 64 targets) share every staged window.
                for(uint32_t tc = tBeg; tc < tEnd; tc += 64)
                {
                    TargetChunk<V4, T> A, Bc;
                    initChunk(A, rec, tc, tEnd, lane, supT);
                    bool const twoChunks = tc + 32 < tEnd;
                    initChunk(Bc, rec, tc + 32, tEnd, lane, supT);
                    uint32_t const nTargets = min(32u, tEnd - tc) + (twoChunks ? min(32u, tEnd - tc - 32) : 0u);
                    // Bounding box of the two chunks' targets and their largest cull
                    // radius: staging keeps only candidates within that radius of the
                    // box.  For a target x_i in [lo, hi] and a staged -x_j, rounding
                    // is monotone, so |x_i - x_j| (rounded) >= max(lo - x_j, x_j - hi,
                    // 0) (rounded) on each axis; with the radius widened by 2^-10 the
                    // box test passes every candidate the exact cull accepts.
                    T bLo[3], bHi[3];
                    {
                        T const inf = T(kFar);
                        T const ax[3] = {A.own.x, A.own.y, A.own.z}, bx[3] = {Bc.own.x, Bc.own.y, Bc.own.z};
#pragma unroll
                        for(int a = 0; a < 3; ++a)
                        {
                            T const l0 = A.act ? ax[a] : inf, l1 = Bc.act ? bx[a] : inf;
                            T const h0 = A.act ? ax[a] : -inf, h1 = Bc.act ? bx[a] : -inf;
                            bLo[a] = warpMinT<T>(l0 < l1 ? l0 : l1);
                            bHi[a] = warpMaxT<T>(h0 > h1 ? h0 : h1);
                        }
                    }
                    T const widen = T(1) + T(1.0 / 1024.0);
                    // PAIRMAX: the pair radius is max(R_i, R_j); nRt = -(max_i R_i)^2
                    T nRt = -R2g;
                    if constexpr(PAIRMAX)
                    {
                        T const nA = A.act ? A.nR2 : T(0), nB = Bc.act ? Bc.nR2 : T(0);
                        nRt = warpMinT<T>(nA < nB ? nA : nB);
                    }
                    for(int page = 0; page * 32 < nDesc; ++page)
                    {
                    uint32_t sBeg = sBeg0, sCnt = sCnt0, slotD = slot0, pre = pre0, total = total0;
                    T sh[3] = {sh0[0], sh0[1], sh0[2]};
                    if(page > 0)
                    {
                        describe(page * 32 + lane, sBeg, sCnt, slotD, sh);
                        scan(sCnt, pre, total);
                    }
                    // entry of staged position q: eBase of q's descriptor + (q << 5)
                    // (j = sBeg + q - pre, packed as (j << 5) | slot)
                    uint32_t const eBase = ((sBeg - pre) << 5) | slotD;
                    for(uint32_t cb = 0; cb < total; cb += CAP)
                    {
                        uint32_t const ce = min(total, cb + uint32_t(CAP));
                        __syncwarp();
                        sSelf[lane] = ~0u;
                        sSelf[lane + 32] = ~0u;
                        // Flat staging: lane l reads window positions l, l + 32, ...; the
                        // descriptor of position q is the last one whose prefix is <= q
                        // (a shuffle binary search over the page's prefixes; empty
                        // descriptors share the next one's prefix and are passed over).
                        // kStageBatch positions' records are in flight at once.  The
                        // candidates that pass the box test are staged in order at
                        // 0 .. m-1.
                        constexpr int KB = PairCfg<T>::kStageBatch;
                        uint32_t mW = 0; // staged so far (warp-uniform)
#pragma unroll 1
                        for(uint32_t k0 = 0; cb + 32u * k0 < ce; k0 += KB)
                        {
                            uint32_t ent[KB];
                            int dsc[KB];
                            V4 pj[KB];
                            T hj[KB];
#pragma unroll
                            for(int k = 0; k < KB; ++k)
                            {
                                uint32_t const q = cb + uint32_t(lane) + 32u * (k0 + uint32_t(k));
                                int sd = 0;
#pragma unroll
                                for(int step = 16; step >= 1; step >>= 1)
                                {
                                    uint32_t const v = __shfl_sync(0xffffffffu, pre, sd + step);
                                    if(v <= q)
                                        sd += step;
                                }
                                dsc[k] = sd;
                                ent[k] = __shfl_sync(0xffffffffu, eBase, sd) + (q << 5);
                                if(q < ce && checkIndex((ent[k] >> 5) < c.n, c.status, kChkStaged))
                                {
                                    pj[k] = ld4(rec.pm + (ent[k] >> 5));
                                    if constexpr(PAIRMAX)
                                        hj[k] = rec.hc[ent[k] >> 5];
                                }
                            }
#pragma unroll
                            for(int k = 0; k < KB; ++k)
                            {
                                bool const in = cb + uint32_t(lane) + 32u * (k0 + uint32_t(k)) < ce;
                                T const sx = __shfl_sync(0xffffffffu, sh[0], dsc[k]);
                                T const sy = __shfl_sync(0xffffffffu, sh[1], dsc[k]);
                                T const sz = __shfl_sync(0xffffffffu, sh[2], dsc[k]);
                                T const nx = in ? -addRn(pj[k].x, sx) : T(kFar);
                                T const ny = in ? -addRn(pj[k].y, sy) : T(kFar);
                                T const nz = in ? -addRn(pj[k].z, sz) : T(kFar);
                                T nRj = T(0);
                                if constexpr(PAIRMAX)
                                {
                                    T const Rj = mulRn(supT, in ? hj[k] : T(0));
                                    nRj = -mulRn(Rj, Rj);
                                }
                                T const dx = fmax(fmax(addRn(bLo[0], nx), -addRn(bHi[0], nx)), T(0));
                                T const dy = fmax(fmax(addRn(bLo[1], ny), -addRn(bHi[1], ny)), T(0));
                                T const dz = fmax(fmax(addRn(bLo[2], nz), -addRn(bHi[2], nz)), T(0));
                                T const nR = (nRj < nRt ? nRj : nRt) * widen;
                                bool const pass = in && dx * dx + dy * dy + dz * dz + nR < T(0);
                                uint32_t const passMask = __ballot_sync(0xffffffffu, pass);
                                if(pass)
                                {
                                    uint32_t const w = mW + uint32_t(__popc(passMask & ((1u << lane) - 1u)));
                                    uint32_t const ws = skewed(w);
                                    sNX[ws] = nx;
                                    sNY[ws] = ny;
                                    sNZ[ws] = nz;
                                    sEnt[w] = ent[k];
                                    if constexpr(PAIRMAX)
                                        sH[ws] = nRj;
                                    // a target's own entry: centre slot, index among the pair's targets
                                    uint32_t const jr = (ent[k] >> 5) - tc;
                                    if((ent[k] & 31u) == kCentreSlot && jr < nTargets)
                                        sSelf[jr] = w;
                                }
                                mW += uint32_t(__popc(passMask));
                            }
                        }
                        uint32_t const m = mW;
                        // far candidates up to the next multiple of 32
                        for(uint32_t q = m + uint32_t(lane); q < ((m + 31u) & ~31u); q += 32)
                        {
                            uint32_t const qs = skewed(q);
                            sNX[qs] = T(kFar);
                            sNY[qs] = T(kFar);
                            sNZ[qs] = T(kFar);
                            if constexpr(PAIRMAX)
                                sH[qs] = T(0);
                        }
                        __syncwarp();
                        // One copy of the cull serves both chunks (a loop that is not
                        // unrolled): the kernel's hot code stays small enough for the
                        // instruction caches when warps run different phases at once.
#pragma unroll 1
                        for(int w = 0; w < (twoChunks ? 2 : 1); ++w)
                        {
                            TargetChunk<V4, T> ch = w ? Bc : A;
                            cullChunk<V4, T, PAIRMAX, CU>(
                                ch, sNX, sNY, sNZ, sH, sEnt, sSelf, tc, m, supT, R2g, c.lists.list, cap, countOnly);
                            if(w)
                                Bc = ch;
                            else
                                A = ch;
                        }
                        cand += uint64_t(m) * nTargets;
                    }
                    }
                    bool const leadA = A.act && A.sub == 0, leadB = twoChunks && Bc.act && Bc.sub == 0;
                    maxCount = max(maxCount, max(leadA ? A.nl : 0u, leadB ? Bc.nl : 0u));
                    pairs += (leadA ? A.nl : 0u) + (leadB ? Bc.nl : 0u);
                    if(countOnly)
                        continue;
                    flushChunk(A, c.lists.list, cap);
                    if(twoChunks)
                        flushChunk(Bc, c.lists.list, cap);
                    __syncwarp();
                    V4 const* const stab = shiftTable<T>(c, box);
                    // one copy of the density sum and its epilogue for both chunks
#pragma unroll 1
                    for(int w = 0; w < (twoChunks ? 2 : 1); ++w)
                    {
                        TargetChunk<V4, T> const ch = w ? Bc : A;
                        chMax = fmax(chMax, densityChunk<K>(ch, c, rec, pa, stab, cap));
                    }
                }
            }
            maxCount = warpMaxU(maxCount);
            pairs = warpSumU64(pairs);
            chMax = warpMaxD(chMax);
            if(lane == 0)
            {
                if(maxCount > cap)
                    atomicMax(&c.status[kStatOverflow], maxCount);
                atomicMax(&c.status[kStatMaxCount], maxCount);
                atomicAdd(&c.scal->pairs, pairs);
                atomicAdd(&c.scal->candidates, cand);
                if(!countOnly && chBox >= 0)
                    atomicMax(&c.bs.chBits[chBox], orderedBits(chMax));
            }
        }

        //! Physics variants compiled separately: 0 = the reference's inviscid
        //! hydro, 1 = hydro + viscosity, 2 = SPMHD with viscosity, Dedner and the
        //! tensile correction switched at run time, 3 = SPMHD with all three on.
        //!
        //! Accumulators (compensated in FP32): a (pressure, viscosity and magnetic
        //! force together), D = sum m_j s_i v_ij.r (P dV work, div v and the
        //! induction's B_i term), the viscous heating, T = sum m_j s_i (B_i.r) v_ij
        //! + rho_i^2 (Dedner gradient term) for the induction, and the div B sum.
        //! With the tensile correction the Maxwell-stress force and the Borve term
        //! combine to sum m_j s_j (B_j.r)/(mu0 rho_j^2) (B_j - B_i).
        //!
        //! The row is read 16 bytes (four entries) at a time; the records of the
        //! next entry are in flight while the current one is used.  Entries run in
        //! row order and the compensated blocks hold 8 terms, as in the density
        //! pass.
        template<typename V4, typename T>
        struct ForceAcc
        {
            Acc<T> ax, ay, az, D, duav, tx, ty, tz, divb;
            T vsig;
            __device__ __forceinline__ void fold()
            {
                ax.fold();
                ay.fold();
                az.fold();
                D.fold();
                duav.fold();
                tx.fold();
                ty.fold();
                tz.fold();
                divb.fold();
            }
        };

        //! Target-side data of the force pass.
        template<typename V4, typename T>
        struct OwnTarget
        {
            V4 pi, vi, ti, bi;
            HConst<T> hk;
            T alpha, beta, eps, rho2i;
            bool av, dedner, tensile;
        };

        template<int K, typename T, int PH, typename V4>
        __device__ __forceinline__ OwnTarget<V4, T> loadOwn(
            Records<V4, T> const& rec,
            PhysArgs const& pa,
            uint32_t t)
        {
            OwnTarget<V4, T> o;
            o.av = (PH == 1) || (PH == 3) || (PH == 2 && (pa.physics & SPH_PHYS_AV));
            o.dedner = (PH == 3) || (PH == 2 && (pa.physics & SPH_PHYS_DEDNER));
            o.tensile = (PH == 3) || (PH == 2 && (pa.physics & SPH_PHYS_TENSILE));
            o.pi = ld4(rec.pm + t);
            o.vi = ld4(rec.fv + t);
            o.ti = ld4(rec.ft + t);
            o.bi = V4{};
            if constexpr(PH >= 2)
                o.bi = ld4(rec.fb + t);
            o.hk = hconst<K, T>(o.vi.w);
            o.alpha = T(pa.alpha);
            o.beta = T(pa.beta);
            o.eps = T(pa.avEps);
            o.rho2i = o.ti.x * o.ti.x;
            return o;
        }

        //! One pair term of the force pass: source records pj, vj, tj, bj and
        //! the source's stencil image shift sh.
        template<int K, typename T, int PH, typename V4>
        __device__ __forceinline__ void pairTerm(
            OwnTarget<V4, T> const& ow,
            ForceAcc<V4, T>& A,
            V4 const& pj,
            V4 const& vj,
            V4 const& tj,
            V4 const& bj,
            V4 const& sh)
        {
            V4 const& pi = ow.pi;
            V4 const& vi = ow.vi;
            V4 const& ti = ow.ti;
            V4 const& bi = ow.bi;
            T const rx = pi.x - (pj.x + sh.x);
            T const ry = pi.y - (pj.y + sh.y);
            T const rz = pi.z - (pj.z + sh.z);
            T const r2 = rx * rx + ry * ry + rz * rz;
            T const y = rsqrtT(r2);
            T const invR = r2 > T(0) ? y : T(0);
            T const r = r2 * invR;
            T const si = gradWScalar<K, T>(r, invR, ow.hk);
            T sj = si; // equal smoothing lengths give the same factor
            if(vj.w != vi.w)
                sj = gradWScalar<K, T>(r, invR, hconstFromInv<K, T>(rcpT(vj.w)));
            T const mj = pj.w;
            T const vx = vi.x - vj.x, vy = vi.y - vj.y, vz = vi.z - vj.z;
            T const vr = vx * rx + vy * ry + vz * rz;
            T const msi = mj * si;
            // Isotropic pressure gradient (HydroForces.hpp:155-166).
            T f = -mj * (ti.y * si + tj.y * sj);
            if(ow.av)
            {
                // branch-free: mu = 0 (no viscosity) for receding pairs
                T const vn = vr < T(0) ? vr : T(0);
                T const hb = T(0.5) * (vi.w + vj.w);
                T const mu = divT(hb * vn, r2 + ow.eps * hb * hb);
                T const cb = T(0.5) * (ti.z + tj.z);
                T const rb = T(0.5) * (ti.x + tj.x);
                T const Pi = divT(-ow.alpha * cb * mu + ow.beta * mu * mu, rb);
                T const g = mj * Pi * T(0.5) * (si + sj);
                f -= g;
                A.duav.add(T(0.5) * g * vr);
            }
            T fx = f * rx, fy = f * ry, fz = f * rz;
            A.D.add(msi * vr);
            T const w = vr * invR;
            T const vs = ti.z + tj.z - ow.beta * (w < T(0) ? w : T(0));
            A.vsig = vs > A.vsig ? vs : A.vsig;
            if constexpr(PH >= 2)
            {
                T const Bir = bi.x * rx + bi.y * ry + bi.z * rz;
                T const Bjr = bj.x * rx + bj.y * ry + bj.z * rz;
                T const cj = mj * sj * Bjr * tj.w;
                if(ow.tensile)
                {
                    // stress + Borve: c_i B_i + c_j B_j - B_i (c_i + c_j) = c_j (B_j - B_i)
                    fx += cj * (bj.x - bi.x);
                    fy += cj * (bj.y - bi.y);
                    fz += cj * (bj.z - bi.z);
                }
                else
                {
                    T const ci = msi * Bir * ti.w;
                    fx += ci * bi.x + cj * bj.x;
                    fy += ci * bi.y + cj * bj.y;
                    fz += ci * bi.z + cj * bj.z;
                }
                T const wB = msi * Bir;
                T gx = wB * vx, gy = wB * vy, gz = wB * vz;
                if(ow.dedner)
                {
                    // rho_i^2 * m_j (psi_i/rho_i^2 s_i + psi_j/rho_j^2 s_j) r
                    T const g = ow.rho2i * mj * (bi.w * si + bj.w * sj);
                    gx += g * rx;
                    gy += g * ry;
                    gz += g * rz;
                }
                A.tx.add(gx);
                A.ty.add(gy);
                A.tz.add(gz);
                A.divb.add(msi * (Bir - Bjr));
            }
            A.ax.add(fx);
            A.ay.add(fy);
            A.az.add(fz);
        }

        //! FP64 epilogue of one target: derivatives and its CFL time step.
        template<typename T, int PH, typename V4>
        __device__ __forceinline__ double forceEpilogue(
            DevCtx const& c,
            PhysArgs const& pa,
            uint32_t t,
            int box,
            ForceAcc<V4, T> const& A,
            bool dedner)
        {
            double const rho = c.cur.rho[t];
            double const h = c.cur.h[t];
            double const pr2 = (pa.gamma - 1.0) * c.cur.u[t] / rho; // P_i / rho_i^2
            double const a[3] = {A.ax.value(), A.ay.value(), A.az.value()};
            double const Dv = A.D.value();
            c.d.dudt[t] = pr2 * Dv + A.duav.value();
            if constexpr(PH >= 2)
            {
                double const Bi[3] = {c.cur.B[0][t], c.cur.B[1][t], c.cur.B[2][t]};
                double const psi = c.cur.psi[t];
                double const tv[3] = {A.tx.value(), A.ty.value(), A.tz.value()};
                double const invRho = 1.0 / rho;
                double const divB = -invRho * A.divb.value();
                double const divv = -invRho * Dv;
                double const ch = __longlong_as_double(static_cast<long long>(c.bs.chBits[box]));
                // dB/dt = -(1/rho)(T_induction - B_i D) - rho grad(psi); T carries rho^2 grad(psi)/rho.
#pragma unroll
                for(int q = 0; q < 3; ++q)
                    c.d.dBdt[q][t] = -invRho * (tv[q] - Bi[q] * Dv);
                c.d.divB[t] = divB;
                c.d.dpsidt[t] = dedner ? (-ch * ch * divB - psi * pa.sigma * ch / h - 0.5 * psi * divv) : 0.0;
            }
#pragma unroll
            for(int q = 0; q < 3; ++q)
                c.d.dvdt[q][t] = a[q];
            double dt = pa.cfl * h / double(A.vsig);
            double const amag = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
            if(amag > 0.0 && pa.cflForce > 0.0)
                dt = fmin(dt, pa.cflForce * sqrt(h / amag));
            return dt;
        }

        //! Physics variants compiled separately: 0 = the reference's inviscid
        //! hydro, 1 = hydro + viscosity, 2 = SPMHD with viscosity, Dedner and the
        //! tensile correction switched at run time, 3 = SPMHD with all three on.
        //!
        //! Accumulators (compensated in FP32): a (pressure, viscosity and magnetic
        //! force together), D = sum m_j s_i v_ij.r (P dV work, div v and the
        //! induction's B_i term), the viscous heating, T = sum m_j s_i (B_i.r) v_ij
        //! + rho_i^2 (Dedner gradient term) for the induction, and the div B sum.
        //! With the tensile correction the Maxwell-stress force and the Borve term
        //! combine to sum m_j s_j (B_j.r)/(mu0 rho_j^2) (B_j - B_i).
        //!
        //! kForce: one thread per target.  The row is read 16 bytes (four
        //! entries) at a time; the records of the next entry are in flight while
        //! the current one is used.  Entries run in row order and the compensated
        //! blocks hold 8 terms, as in the density pass.
        template<int K, typename T, int PH, int MINB>
        __global__ void __launch_bounds__(kForceThreads, MINB) kForce(DevCtx c, PhysArgs pa)
        {
            using V4 = typename PairCfg<T>::V4;
            constexpr bool kMhd = PH >= 2;
            Records<V4, T> const rec = records<T>(c);
            uint32_t const t = blockIdx.x * blockDim.x + threadIdx.x;
            bool const act = t < c.n && isTarget(c.cur.role[t]);
            double dtLocal = 1e300;
            int const myBox = t < c.n ? c.cur.box[t] : -1;
            if(act)
            {
                OwnTarget<V4, T> const own = loadOwn<K, T, PH>(rec, pa, t);
                V4 const* const stab = shiftTable<T>(c, myBox);
                ForceAcc<V4, T> A;
                A.vsig = own.ti.z;
                uint32_t const n = min(c.lists.count[t], c.lists.cap);
                // rows are 32-byte aligned and hold a multiple of 8 entries
                uint4 const* row4 = reinterpret_cast<uint4 const*>(c.lists.list + size_t(t) * c.lists.cap);
                V4 npm{}, nfv{}, nft{}, nfb{};
                uint32_t nslot = 0;
                auto fetch = [&](uint32_t e)
                {
                    if(!checkIndex((e >> 5) < c.n, c.status, kChkRowEntry))
                        e = 0;
                    uint32_t const j = e >> 5;
                    nslot = e & 31u;
                    npm = ld4(rec.pm + j);
                    nfv = ld4(rec.fv + j);
                    nft = ld4(rec.ft + j);
                    if constexpr(kMhd)
                        nfb = ld4(rec.fb + j);
                };
                // one entry: take the fetched records, start fetching `next`
                auto step = [&](uint32_t next)
                {
                    V4 const pj = npm, vj = nfv, tj = nft, bj = nfb;
                    V4 const o = ld4(stab + nslot);
                    fetch(next);
                    pairTerm<K, T, PH>(own, A, pj, vj, tj, bj, o);
                };
                uint4 qc = make_uint4(0, 0, 0, 0);
                if(n > 0)
                {
                    qc = row4[0];
                    fetch(qc.x);
                }
                uint32_t const nFull = n & ~3u;
                uint32_t k0 = 0;
                for(; k0 < nFull; k0 += 4)
                {
                    step(qc.y);
                    step(qc.z);
                    step(qc.w);
                    // the next quad starts inside the row when k0 + 4 < n
                    bool const more = k0 + 4 < n;
                    uint4 const qn = more ? row4[(k0 >> 2) + 1] : qc;
                    step(more ? qn.x : qc.w); // a valid index either way
                    if(k0 & 4u)
                        A.fold();
                    qc = qn;
                }
                // the last 1-3 entries (qc.x already fetched); a loop that is not
                // unrolled keeps one copy of the pair term, and the fetch after
                // the last entry re-reads qc.x, a valid entry
                uint32_t const tail = n - nFull;
#pragma unroll 1
                for(uint32_t i = 0; i < tail; ++i)
                    step(i + 1 < tail ? (i == 0 ? qc.y : qc.z) : qc.x);
                A.fold();
                dtLocal = forceEpilogue<T, PH>(c, pa, t, myBox, A, own.dedner);
            }
            // CFL minimum per box: one atomic per warp when the warp is in one box
            int const box0 = __shfl_sync(0xffffffffu, myBox, 0);
            if(__all_sync(0xffffffffu, myBox == box0 || dtLocal >= 1e300))
            {
                dtLocal = warpMinD(dtLocal);
                if((threadIdx.x & 31) == 0 && dtLocal < 1e300)
                    atomicMin(&c.bs.dtBits[box0], orderedBits(dtLocal));
            }
            else if(dtLocal < 1e300)
                atomicMin(&c.bs.dtBits[myBox], orderedBits(dtLocal));
        }

        template<typename T, bool PM, int CAP>
        constexpr size_t densitySmem()
        {
            return size_t(kDensWarps)
                   * (colLen<CAP>() * (PM ? 4 : 3) * sizeof(T) + CAP * sizeof(uint32_t) + 64 * sizeof(uint32_t));
        }

        // ---- launch-shape variants -------------------------------------------
        // density FP32: (CAP, blocks/SM) = (256, 6), (256, 5), (128, 6), (128, 5),
        // each with the mask cull fully unrolled and unrolled twice;
        // density FP64: (256, 4), (128, 4).  force FP32: 4 or 5 blocks/SM (SPMHD
        // default 4, hydro default 5); force FP64: 3.  Variant 0 is the default.
        constexpr int kDensVariants32 = 8, kDensVariants64 = 2, kForceVariants32 = 2, kForceVariants64 = 1;
        constexpr int kDensCap32[kDensVariants32] = {256, 256, 128, 128, 256, 256, 128, 128};
        constexpr int kDensBlk32[kDensVariants32] = {6, 5, 6, 5, 6, 5, 6, 5};
        constexpr int kDensUnr32[kDensVariants32] = {8, 8, 8, 8, 2, 2, 2, 2};
        constexpr int kDensCap64[kDensVariants64] = {256, 128};

        //! Shared-memory carve-out (percent of the maximum) that fits `blocks`
        //! blocks of `smem` bytes; the rest of the unified array stays L1 for
        //! the list gathers.
        int carveout(size_t smem, int blocks)
        {
            size_t const need = size_t(blocks) * (smem + 1024);
            size_t const maxSmem = 228 * 1024;
            int pct = int((need * 100 + maxSmem - 1) / maxSmem);
            return pct > 100 ? 100 : pct;
        }

        template<int K, typename T, bool PM, int CAP, int MINB, int CU = 8>
        void configureDensity()
        {
            auto f = kDensity<K, T, PM, CAP, MINB, CU>;
            size_t const smem = densitySmem<T, PM, CAP>();
            cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
            cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, carveout(smem, MINB));
        }

        template<int K, typename T, int PH, int MINB>
        void configureForce()
        {
            cudaFuncSetAttribute(kForce<K, T, PH, MINB>, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
        }

        template<int K, typename T, bool PM, int CAP, int MINB, int CU = 8>
        void densityLaunch(DevCtx const& c, PhysArgs const& pa, bool countOnly, cudaStream_t s)
        {
            size_t const smem = densitySmem<T, PM, CAP>();
            // persistent grid: enough resident blocks to fill every SM; cells come
            // from the work queue
            uint32_t blocks = (c.cells.ncells + kDensWarps - 1) / kDensWarps;
            uint32_t const resident = 148u * uint32_t(MINB);
            blocks = blocks > resident ? resident : blocks;
            if(blocks)
            {
                cudaMemsetAsync(c.work, 0, sizeof(uint32_t), s);
                kDensity<K, T, PM, CAP, MINB, CU><<<blocks, kDensWarps * 32, smem, s>>>(c, pa, countOnly);
                countLaunches(1);
            }
        }

        template<int K, typename T, bool PM>
        void densityOne(DevCtx const& c, PhysArgs const& pa, bool countOnly, int variant, cudaStream_t s)
        {
            if constexpr(sizeof(T) == 4)
            {
                switch(variant)
                {
#define SPH_DENS32(v) densityLaunch<K, T, PM, kDensCap32[v], kDensBlk32[v], kDensUnr32[v]>(c, pa, countOnly, s)
                case 1: SPH_DENS32(1); break;
                case 2: SPH_DENS32(2); break;
                case 3: SPH_DENS32(3); break;
                case 4: SPH_DENS32(4); break;
                case 5: SPH_DENS32(5); break;
                case 6: SPH_DENS32(6); break;
                case 7: SPH_DENS32(7); break;
                default: SPH_DENS32(0); break;
#undef SPH_DENS32
                }
            }
            else
            {
                if(variant == 1)
                    densityLaunch<K, T, PM, kDensCap64[1], 4>(c, pa, countOnly, s);
                else
                    densityLaunch<K, T, PM, kDensCap64[0], 4>(c, pa, countOnly, s);
            }
        }

        template<int K, typename T>
        void densityPM(DevCtx const& c, PhysArgs const& pa, bool countOnly, int variant, cudaStream_t s)
        {
            if(pa.cull == SPH_CULL_PAIR_MAX)
                densityOne<K, T, true>(c, pa, countOnly, variant, s);
            else
                densityOne<K, T, false>(c, pa, countOnly, variant, s);
        }

        template<int K, typename T, int PH>
        void forceLaunch(DevCtx const& c, PhysArgs const& pa, int variant, cudaStream_t s)
        {
            unsigned const g = (c.n + kForceThreads - 1) / kForceThreads;
            if(!g)
                return;
            if constexpr(sizeof(T) == 4)
            {
                // variant 0: SPMHD 4 blocks/SM (128 registers), hydro 5; variant 1 the other
                constexpr int a = PH >= 2 ? 4 : 5, b = PH >= 2 ? 5 : 4;
                if(variant == 1)
                    kForce<K, T, PH, b><<<g, kForceThreads, 0, s>>>(c, pa);
                else
                    kForce<K, T, PH, a><<<g, kForceThreads, 0, s>>>(c, pa);
            }
            else
                kForce<K, T, PH, 3><<<g, kForceThreads, 0, s>>>(c, pa);
            countLaunches(1);
        }

        template<int K, typename T>
        void forceOne(DevCtx const& c, PhysArgs const& pa, int variant, cudaStream_t s)
        {
            uint32_t const full = SPH_PHYS_MHD | SPH_PHYS_AV | SPH_PHYS_DEDNER | SPH_PHYS_TENSILE;
            if((pa.physics & full) == full)
                forceLaunch<K, T, 3>(c, pa, variant, s);
            else if(pa.physics & SPH_PHYS_MHD)
                forceLaunch<K, T, 2>(c, pa, variant, s);
            else if(pa.physics & SPH_PHYS_AV)
                forceLaunch<K, T, 1>(c, pa, variant, s);
            else
                forceLaunch<K, T, 0>(c, pa, variant, s);
        }

        template<typename T>
        void densityK(DevCtx const& c, PhysArgs const& pa, int kernel, bool countOnly, int variant, cudaStream_t s)
        {
            if(kernel == SPH_KERNEL_QUINTIC)
                densityPM<SPH_KERNEL_QUINTIC, T>(c, pa, countOnly, variant, s);
            else if(kernel == SPH_KERNEL_WENDLAND_C2)
                densityPM<SPH_KERNEL_WENDLAND_C2, T>(c, pa, countOnly, variant, s);
            else
                densityPM<SPH_KERNEL_CUBIC, T>(c, pa, countOnly, variant, s);
        }

        template<typename T>
        void forceK(DevCtx const& c, PhysArgs const& pa, int kernel, int variant, cudaStream_t s)
        {
            if(kernel == SPH_KERNEL_QUINTIC)
                forceOne<SPH_KERNEL_QUINTIC, T>(c, pa, variant, s);
            else if(kernel == SPH_KERNEL_WENDLAND_C2)
                forceOne<SPH_KERNEL_WENDLAND_C2, T>(c, pa, variant, s);
            else
                forceOne<SPH_KERNEL_CUBIC, T>(c, pa, variant, s);
        }

        template<int K, bool PM>
        void configureDensityK()
        {
#define SPH_CONF32(v) configureDensity<K, float, PM, kDensCap32[v], kDensBlk32[v], kDensUnr32[v]>()
            SPH_CONF32(0);
            SPH_CONF32(1);
            SPH_CONF32(2);
            SPH_CONF32(3);
            SPH_CONF32(4);
            SPH_CONF32(5);
            SPH_CONF32(6);
            SPH_CONF32(7);
#undef SPH_CONF32
            configureDensity<K, double, PM, kDensCap64[0], 4>();
            configureDensity<K, double, PM, kDensCap64[1], 4>();
        }

        template<int K, int PH>
        void configureForceK()
        {
            constexpr int a = PH >= 2 ? 4 : 5, b = PH >= 2 ? 5 : 4;
            configureForce<K, float, PH, a>();
            configureForce<K, float, PH, b>();
            configureForce<K, double, PH, 3>();
        }

        template<int K>
        void configureK()
        {
            configureDensityK<K, true>();
            configureDensityK<K, false>();
            configureForceK<K, 0>();
            configureForceK<K, 1>();
            configureForceK<K, 2>();
            configureForceK<K, 3>();
        }
    } // namespace

    void configurePairKernels()
    {
        static bool done = false;
        if(done)
            return;
        configureK<SPH_KERNEL_CUBIC>();
        configureK<SPH_KERNEL_QUINTIC>();
        configureK<SPH_KERNEL_WENDLAND_C2>();
        done = true;
    }

    int densityVariants(int precision)
    {
        return precision == SPH_PREC_FP64 ? kDensVariants64 : kDensVariants32;
    }

    int forceVariants(int precision)
    {
        return precision == SPH_PREC_FP64 ? kForceVariants64 : kForceVariants32;
    }

    void densityShape(int precision, int variant, int* stagingDepth, int* blocksPerSm, int* cullUnroll)
    {
        bool const f64 = precision == SPH_PREC_FP64;
        int const v = variant < 0 || variant >= densityVariants(precision) ? 0 : variant;
        *stagingDepth = f64 ? kDensCap64[v] : kDensCap32[v];
        *blocksPerSm = f64 ? 4 : kDensBlk32[v];
        *cullUnroll = f64 ? 0 : kDensUnr32[v];
    }

    int forceBlocksPerSm(int precision, int physics, int variant)
    {
        if(precision == SPH_PREC_FP64)
            return 3;
        bool const mhd = physics & SPH_PHYS_MHD;
        return (variant == 1) == mhd ? 5 : 4;
    }


    void launchDensity(
        DevCtx const& c,
        PhysArgs const& pa,
        int kernel,
        int precision,
        bool countOnly,
        int variant,
        cudaStream_t s)
    {
        if(precision == SPH_PREC_FP64)
            densityK<double>(c, pa, kernel, countOnly, variant, s);
        else
            densityK<float>(c, pa, kernel, countOnly, variant, s);
    }

    void launchForce(DevCtx const& c, PhysArgs const& pa, int kernel, int precision, int variant, cudaStream_t s)
    {
        if(precision == SPH_PREC_FP64)
            forceK<double>(c, pa, kernel, variant, s);
        else
            forceK<float>(c, pa, kernel, variant, s);
    }
} // namespace sph
