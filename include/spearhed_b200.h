/* spearhed_b200 — C ABI for the B200-native SPH(-MHD) step.
 *
 * The step this library replaces is spearHED's neighbour-region SPH step as
 * composed by Simulation::runOneStep (include/spearhed/control/Simulation.x.cpp:196-310):
 * drift -> neighbour search -> UpdateDensity -> UpdateHydroForces -> EulerIntegrate.
 * It adds the terms the SPH-MHD step needs on top of the reference's
 * inviscid hydro: artificial viscosity, SPMHD induction and magnetic stress,
 * Dedner divergence cleaning, a CFL time step and FP64 conserved-quantity sums.
 *
 * Conventions
 *  - Every entry point returns an int status (SPH_OK == 0).  No C++ exception
 *    crosses this boundary.  sph_last_error_string() describes the last failure
 *    on the calling thread.
 *  - Host arrays are caller-owned and are copied in (sph_set_species) and out
 *    (sph_get_species).  Device memory is owned by the context.  Each context
 *    owns one CUDA stream; a context is not thread-safe, distinct contexts on
 *    distinct threads are.
 *  - All host columns are FP64 ("double"), one array per attribute component
 *    (structure of arrays), named after the reference's attribute tags
 *    (include/spearhed/param/speciesDefinition.param:100-110): position, vel,
 *    mass, smoothingLength (h), density, internalEnergy (u), dvdt, dudt, plus
 *    the MHD columns B, psi, dBdt, dpsidt that the reference does not carry.
 */
#ifndef SPEARHED_B200_H
#define SPEARHED_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum
{
    SPH_OK = 0,
    SPH_ERR_INVALID = 1,       /* bad argument (null pointer, bad enum, n < 0 ...)          */
    SPH_ERR_CUDA = 2,          /* a CUDA runtime call failed                                */
    SPH_ERR_NOMEM = 3,         /* device allocation failed                                  */
    SPH_ERR_OUTSIDE = 4,       /* a particle outside its box (see SphBox)                    */
    SPH_ERR_NONFINITE = 5,     /* NaN/Inf position, h <= 0 or mass <= 0 in the input        */
    SPH_ERR_OVERFLOW = 6,      /* a neighbour list exceeded its capacity (retry is automatic) */
    SPH_ERR_STATE = 7,         /* call out of order (e.g. hydro before density)             */
    SPH_ERR_TIMEOUT = 8,       /* a bounded wait on the device gave up                      */
    SPH_ERR_UNSUPPORTED = 9    /* configuration the library does not implement              */
};

/* ---- kernels (SphKernel models, include/spearhed/sph/SphKernel.hpp:45-51) -- */
enum
{
    SPH_KERNEL_CUBIC = 0,      /* M4 cubic spline, support 2h (CubicSplineKernel.hpp:40)      */
    SPH_KERNEL_QUINTIC = 1,    /* M5 quintic spline, support 3h (QuinticSplineKernel.hpp:39)  */
    SPH_KERNEL_WENDLAND_C2 = 2 /* Wendland C2, support 2h (not in the reference)              */
};

/* ---- physics switches (SphParams.physics bit mask) --------------------- */
enum
{
    SPH_PHYS_AV = 1u << 0,       /* Monaghan artificial viscosity (alpha, beta)              */
    SPH_PHYS_MHD = 1u << 1,      /* SPMHD induction + Maxwell stress                         */
    SPH_PHYS_DEDNER = 1u << 2,   /* Dedner/Tricco-Price hyperbolic divergence cleaning       */
    SPH_PHYS_TENSILE = 1u << 3,  /* Borve tensile-instability correction of the stress       */
    SPH_PHYS_CFL = 1u << 4,      /* adaptive dt from the CFL/force criteria (FP64 min)       */
    SPH_PHYS_ADAPTIVE_H = 1u << 5 /* h = hfact (m/rho)^(1/3) after every kick (needs SPH_CULL_PAIR_MAX) */
};

/* ---- precision of the pair kernels -------------------------------------- */
enum
{
    SPH_PREC_FP64 = 0,         /* FP64 plain pair kernels                                    */
    SPH_PREC_FP32_COMP = 1     /* FP32 pair kernels with compensated (two-sum) accumulation  */
};

/* ---- neighbour acceptance radius ---------------------------------------- */
enum
{
    SPH_CULL_GLOBAL = 0,       /* r^2 < (support*h0)^2: the reference's interact() radius    */
    SPH_CULL_PAIR_MAX = 1      /* r^2 < (support*max(h_i,h_j))^2: variable h                 */
};

/* ---- species and roles (include/spearhed/param/speciesDefinition.param:56-88,
 *      spmacc/particles/regions/RegionRole.hpp:42-62) ---------------------- */
enum
{
    SPH_SPECIES_DEFAULT = 0,   /* Interior|Movable|Source|Thermodynamic */
    SPH_SPECIES_BOUNDARY = 1,  /* Frozen|Source|Thermodynamic           */
    SPH_SPECIES_TRACER = 2,    /* Movable                               */
    SPH_NUM_SPECIES = 3
};
enum
{
    SPH_ROLE_MOVABLE = 1u << 0,
    SPH_ROLE_SOURCE = 1u << 1,
    SPH_ROLE_THERMODYNAMIC = 1u << 2,
    SPH_ROLE_FROZEN = 1u << 3,
    SPH_ROLE_INTERIOR = 1u << 4
};
#define SPH_ROLES_DEFAULT (SPH_ROLE_INTERIOR | SPH_ROLE_MOVABLE | SPH_ROLE_SOURCE | SPH_ROLE_THERMODYNAMIC)
#define SPH_ROLES_BOUNDARY (SPH_ROLE_FROZEN | SPH_ROLE_SOURCE | SPH_ROLE_THERMODYNAMIC)
#define SPH_ROLES_TRACER (SPH_ROLE_MOVABLE)

/* ---- run-time parameters (replace the reference's compile-time .param
 *      files: include/spearhed/param/sph.param:26-34, dimension.param:28-35) */
typedef struct SphParams
{
    int32_t kernel;        /* SPH_KERNEL_*                                                  */
    int32_t precision;     /* SPH_PREC_*                                                    */
    int32_t cull;          /* SPH_CULL_*                                                    */
    uint32_t physics;      /* SPH_PHYS_* mask; 0 = the reference's inviscid hydro           */
    double gamma;          /* adiabatic index (gamma_eos)                                   */
    double h0;             /* smoothing length used for the global cull radius (h0)         */
    double dt;             /* fixed time step, or the first step's dt when SPH_PHYS_CFL      */
    double alpha, beta;    /* artificial viscosity (Monaghan 1992), e.g. 1 and 2             */
    double av_eps;         /* eta^2 regulariser in mu_ij, 0.01                              */
    double cfl;            /* Courant factor for SPH_PHYS_CFL, e.g. 0.3                      */
    double cfl_force;      /* factor of the force criterion sqrt(h/|a|), e.g. 0.25          */
    double dedner_sigma;   /* Dedner damping constant sigma (tau = h/(sigma c_h)), e.g. 1    */
    double mu0;            /* magnetic permeability in code units (1)                        */
    int32_t max_neighbours;/* per-particle neighbour-list capacity; 0 = library default      */
    int32_t device;        /* CUDA device ordinal                                           */
    double hfact;          /* eta of SPH_PHYS_ADAPTIVE_H: h = hfact * (m/rho)^(1/3), e.g. 1.2 */
    double h_max;          /* largest h the run may reach: sets the cell size and caps adaptive h;
                              0 = the largest input h (times 1.5 with SPH_PHYS_ADAPTIVE_H)    */
} SphParams;

/* A particle box: the reference's fluid/wall domain (an AABB, spmacc/particles/regions/AABB.hpp:38-127).
 * Particles must lie inside [lo, hi] on every axis when they are set.  Along a periodic axis the
 * drift wraps movable particles back into [lo, hi) every step; a particle that leaves a
 * non-periodic axis, or lies outside a periodic one it was not wrapped on, is SPH_ERR_OUTSIDE. */
typedef struct SphBox
{
    double lo[3];
    double hi[3];
    int32_t periodic[3];
} SphBox;

/* Column pointers for one species (host, FP64, length n).  Any pointer may be
 * NULL: on input the attribute is then zero (h defaults to params.h0); on
 * output it is skipped.  box_id (int32) selects the ensemble box (NULL = 0). */
typedef struct SphSoAView
{
    double* pos[3];
    double* vel[3];
    double* mass;
    double* h;
    double* density;
    double* u;
    double* dvdt[3];
    double* dudt;
    double* B[3];
    double* psi;
    double* dBdt[3];
    double* dpsidt;
    double* divB;
    int32_t* box_id;
} SphSoAView;

/* Conserved quantities and step diagnostics, FP64 sums over the
 * Movable & Thermodynamic particles (block-then-grid reductions on the device). */
typedef struct SphDiag
{
    double time;           /* simulated time                                                */
    double dt;             /* dt of the last step                                           */
    double dt_next;        /* dt the next step will use                                     */
    double e_kin;          /* sum 1/2 m v^2                                                 */
    double e_int;          /* sum m u                                                       */
    double e_mag;          /* sum 1/2 m B^2 / (mu0 rho)                                     */
    double mom[3];         /* sum m v                                                       */
    double divb_mean;      /* mean of |divB| h / |B| (|B| > 0)                              */
    double divb_max;       /* max of |divB| h / |B|                                         */
    double c_h;            /* Dedner cleaning speed of the last force pass                  */
    double pairs;          /* ordered accepted pairs (i != j) of the last neighbour build   */
    int64_t steps;         /* steps taken by this context                                   */
    int64_t n_targets;     /* particles in the sums                                         */
    double pairs_total;    /* accepted ordered pairs summed over every step's neighbour build */
    double candidates;     /* (target, staged source) pairs the cull tested in the last build
                              (sources that passed the staging box test)                     */
    int64_t replays;       /* step calls this context re-ran after a neighbour-list overflow */
    int64_t list_capacity; /* neighbour-list entries per particle currently allocated      */
} SphDiag;

typedef struct sph_ctx sph_ctx;

/* Fill *p with the library defaults (cubic kernel, FP32-compensated, global
 * cull, inviscid hydro, gamma 5/3, h0 0.05, dt 0.01 — the reference's param files). */
int sph_default_params(SphParams* p);

/* Replaces: Simulation::init / pluginLoad device and heap setup
 * (include/spearhed/control/Simulation.x.cpp:129-169, 312-352). */
int sph_create(const SphParams* params, sph_ctx** out);
int sph_destroy(sph_ctx* ctx);

/* Replaces: the setup's domain AABB and region list
 * (share/spearhed/ValidationSetups/SodShockTube.hpp:442-467, InitRegions.hpp:47-104).
 * nbox > 1 makes an ensemble of independent boxes (particles select theirs by box_id). */
int sph_set_boxes(sph_ctx* ctx, int32_t nbox, const SphBox* boxes);

/* Replaces: InitParticles filling a species' ParticleRegionBuffer
 * (include/spearhed/particles/initialization/InitParticles.hpp:284-433). */
int sph_set_species(sph_ctx* ctx, int32_t species_id, uint32_t roles, int64_t n, const SphSoAView* view);

/* Replaces: ParticleRegionBuffer::deviceToHost + frame iteration in the tests
 * (tests/spearhed/unit/DensitySummation/DensitySummation.cpp:258-276).  Copies the
 * species back in the order it was given to sph_set_species. */
int sph_get_species(sph_ctx* ctx, int32_t species_id, SphSoAView* view);

/* Replaces: UpdateDensity<K>{}(bundle, target, index, h0)
 * (include/spearhed/particles/density/DensitySummation.hpp:104-138), including the
 * neighbour search it relies on (calculateNeighboursSender, NeighbourRegions.hpp:233-255). */
int sph_density(sph_ctx* ctx);

/* Replaces: UpdateHydroForces<K>{gamma}(bundle, target, index, h0)
 * (include/spearhed/sph/HydroForces.hpp:183-214).  Uses the density of the last
 * sph_density call.  With SPH_PHYS_AV the viscosity terms are added. */
int sph_hydro(sph_ctx* ctx);

/* The SPMHD pass (induction, Maxwell stress, Dedner): no reference counterpart.
 * Runs the full force pass with the MHD terms enabled in params.physics. */
int sph_mhd(sph_ctx* ctx);

/* Replaces: Simulation::runOneStep repeated n_steps times
 * (include/spearhed/control/Simulation.x.cpp:196-310): drift, neighbour search,
 * density, forces, kick.  dt > 0 overrides params.dt for these steps; dt <= 0
 * keeps params.dt (or the CFL dt when SPH_PHYS_CFL is set).  A context whose
 * species hold no particles steps as a no-op that only advances its clock, as
 * runOneStep accepts an empty setup (tests/spearhed/unit/SimulationTimestep/
 * SimulationTimestep.cpp:365-400); sph_density / sph_hydro then do nothing and
 * sph_reduce reports zero sums. */
int sph_step(sph_ctx* ctx, int32_t n_steps, double dt);

/* Bounded waits (no reference counterpart: its host waits are unbounded
 * syncWait calls, include/spearhed/control/Simulation.x.cpp:303-307).  With a
 * limit of `seconds` > 0, sph_step, sph_density, sph_hydro and sph_mhd wait at
 * most that long for their device work (polling an event; 0, the default,
 * waits without a limit).  When the limit passes the call returns
 * SPH_ERR_TIMEOUT; its work keeps running and nothing is cancelled, and the
 * call's checks (non-finite or escaped particles, list overflow) are still
 * owed.  sph_wait completes them, and so does the next call on the context
 * (every call that touches its device state, except sph_destroy, which waits
 * without a limit); until then that next call returns SPH_ERR_TIMEOUT too.
 * A completed call's results stand; a step call whose checks fail is rolled
 * back to the state it started from and sph_wait returns the check's status
 * (after a list overflow the lists have grown: run the call again). */
int sph_set_wait_timeout(sph_ctx* ctx, double seconds);
int sph_wait(sph_ctx* ctx);

/* Conserved-quantity reductions of the current state (no reference counterpart;
 * PMacc's device::Reduce, packages/pmacc/include/pmacc/device/Reduce.hpp:41, is unused there). */
int sph_reduce(sph_ctx* ctx, SphDiag* out);

/* Per-box diagnostics of an ensemble: out[nbox]. */
int sph_ensemble_reduce(sph_ctx* ctx, int32_t nbox, SphDiag* out);

/* Per-particle accepted-neighbour counts (i != j) of the last neighbour build, for
 * one species in its input order (int32, length n).  Used to prove that the
 * accepted pair set equals the oracle's. */
int sph_get_neighbour_counts(sph_ctx* ctx, int32_t species_id, int32_t* counts);

/* Device time of the last sph_step / sph_density / sph_hydro call per stage,
 * in milliseconds: [0] sort+permute, [1] density, [2] force, [3] integrate+reduce,
 * [4] whole call.  n is the array length (<= 5). */
int sph_get_timings(sph_ctx* ctx, int32_t n, double* ms);

/* Per-box simulated time and the dt the next step will use (nbox entries each):
 * the clock a checkpoint must save and restore.  No reference counterpart (the
 * reference's checkpointing is disabled, include/spearhed/control/Simulation.hpp:54-61). */
int sph_get_clock(sph_ctx* ctx, int32_t nbox, double* time, double* dt_next);
int sph_set_clock(sph_ctx* ctx, int32_t nbox, const double* time, const double* dt_next);

/* Capture each later sph_step's per-step launch sequence in a CUDA graph and
 * replay it (on = 1) or launch the kernels one by one (on = 0, the default). */
int sph_use_graph(sph_ctx* ctx, int32_t on);

/* With graph replay on: capture the graph the next sph_step will replay by
 * running two steps from a snapshot and restoring it, so the capture costs no
 * simulated time and no later step call pays for it (no reference counterpart). */
int sph_prepare_graph(sph_ctx* ctx);

/* Launch shapes of the two pair kernels (no reference counterpart; the
 * reference's frame size and threads per frame are compile-time constants,
 * spmacc/Frame.hpp:49-132).  density: staging depth (candidates per shared-memory
 * window), register cap (blocks per SM) and, in FP32, the unroll depth of the
 * mask cull; force: register cap.  Every shape gives identical bits. */
typedef struct SphTuning
{
    int32_t density_variant;      /* index into the density shapes (0 = default)          */
    int32_t force_variant;        /* index into the force shapes (0 = default)            */
    int32_t staging_depth;        /* density candidates per shared-memory window          */
    int32_t density_blocks_per_sm;
    int32_t force_blocks_per_sm;
    int32_t n_density_variants;   /* shapes available for this precision                 */
    int32_t n_force_variants;
    int32_t steps_per_trial;      /* steps timed per shape by sph_autotune (0: not tuned)  */
    double density_ms[8];         /* per-step density time of each shape (sph_autotune)   */
    double force_ms[8];           /* per-step force time of each shape (sph_autotune)     */
    int32_t cull_unroll;          /* FP32 density: 4-candidate groups of the 32-candidate
                                     mask cull unrolled (8 = all, 2); 0 in FP64          */
} SphTuning;

/* Times every launch shape of the density and force kernels on this context's
 * current particles (steps_per_trial steps each, the state restored after every
 * trial) and keeps the fastest of each.  The particles, clock and diagnostics are
 * left as they were.  *out (may be NULL) receives the choice and the timings. */
int sph_autotune(sph_ctx* ctx, int32_t steps_per_trial, SphTuning* out);

/* Sets the launch shapes explicitly (e.g. the choice of an earlier sph_autotune). */
int sph_set_tuning(sph_ctx* ctx, int32_t density_variant, int32_t force_variant);
int sph_get_tuning(sph_ctx* ctx, SphTuning* out);

/* ---- Device initialiser of particle species from lattice blocks ----
 * Replaces: the setup blocks (regions per species with a count and a placement
 * recipe, include/spearhed/particles/initialization/SetupInterface.hpp:34-113),
 * the init driver that counts, scans and places them on the device
 * (InitParticles.hpp:284-433) and simple-cubic placement at cell centres
 * (spmacc/particles/initialization/SC.hpp:118-200).  A block is a region filled by
 * an SC lattice, with constant state; a profile adds the analytic fields of the
 * validation setups after an optional per-group jitter and periodic wrap. */
enum
{
    SPH_MASK_NONE = 0,
    SPH_MASK_INSIDE_DISC_XY = 1,  /* keep sites with hypot(x - cx, y - cy) <  radius */
    SPH_MASK_OUTSIDE_DISC_XY = 2  /* keep sites with hypot(x - cx, y - cy) >= radius */
};
enum
{
    SPH_PROFILE_CONSTANT = 0,
    SPH_PROFILE_ORSZAG_TANG = 1,       /* v = (-sin 2pi y, sin 2pi x, 0), B = p0 (-sin 2pi y, sin 4pi x, 0) */
    SPH_PROFILE_KH_PERTURBATION = 2,   /* v_y = p0 sin(4 pi x) */
    SPH_PROFILE_ROTOR = 3              /* rotation p2 about (p0, p1) for r < p3, times clip((p4 - r) / p5, 0, 1) beyond */
};

typedef struct SphLatticeBlock
{
    double lo[3], hi[3];       /* region volume                                                   */
    int32_t counts[3];         /* lattice sites per axis; all 0: from spacing (sph_sc_cell_counts) */
    int32_t mask;              /* SPH_MASK_*                                                      */
    double spacing;
    double mask_centre[2];
    double mask_radius;
    int32_t box_id;
    int32_t jitter_group;      /* consecutive blocks with one id share one jitter stream           */
    double jitter;             /* the group's uniform displacement amplitude per axis (length)     */
    uint64_t seed;             /* the group's Philox4x64-10 key                                    */
    double mass, h, density, u, psi;
    double vel[3], B[3];
} SphLatticeBlock;

typedef struct SphInitProfile
{
    int32_t kind;              /* SPH_PROFILE_*                                                   */
    int32_t wrap[3];           /* wrap positions periodically into [wrap_lo, wrap_hi) per axis    */
    double wrap_lo[3], wrap_hi[3];
    double p[8];               /* profile parameters                                              */
} SphInitProfile;

/* Generates the species on the device from nblocks lattice blocks (kept sites in
 * block order, each block's sites x-fastest) and sets it as sph_set_species would;
 * *n_out (may be NULL) receives the particle count.  profile may be NULL. */
int sph_init_lattice(sph_ctx* ctx, int32_t species_id, uint32_t roles, int32_t nblocks,
                     const SphLatticeBlock* blocks, const SphInitProfile* profile, int64_t* n_out);

/* Replaces: computeSCCellCounts (spmacc/particles/initialization/SC.hpp:98-132):
 * SC sites per axis of the box lo..hi at `spacing` (axis 0 truncated with a
 * round-off snap, transverse axes rounded, each at least 1), in double or float. */
int sph_sc_cell_counts(const double* lo, const double* hi, double spacing, uint32_t* counts);
int sph_sc_cell_counts_f32(const float* lo, const float* hi, float spacing, uint32_t* counts);

/* Density summation that allocates no device memory, for callers that cannot
 * call cudaMalloc (no counterpart in the reference).
 *
 * Some callers cannot allocate: a host framework that owns all device memory
 * through its own pool, code running where an allocation would synchronise the
 * device, or a plugin hosted by a program that forbids the CUDA allocator.  This
 * entry point takes caller-owned DEVICE arrays (positions, mass, h; length n) and
 * writes rho (device, length n, input order); its scratch is one fixed 32 MiB
 * device array inside this library (held on every GPU that loads it until the
 * process exits).  Limits: n <= 262144 particles, <= 262144 cells, one box.
 * Every Default-species rule applies (all particles are targets and sources).
 * The work runs on `stream` (a cudaStream_t, NULL = legacy default stream) and
 * the call synchronizes that stream before it returns.  Calls share the scratch
 * array: calls whose device work overlaps (other threads or unordered streams)
 * race and give wrong results.  The first call on a device looks up the array's
 * address (cudaGetSymbolAddress) and keeps it for the process; make that first
 * call before any stream capture, and make no call on a device after
 * cudaDeviceReset() on it.
 * Returns:
 *   SPH_OK               rho written;
 *   SPH_ERR_INVALID      a null pointer, bad enums or h0, an empty or non-finite box,
 *                        n or the cell count above the limits, or a layout that does
 *                        not fit the scratch array (nothing launched);
 *   SPH_ERR_UNSUPPORTED  params->cull == SPH_CULL_PAIR_MAX, or a periodic axis
 *                        shorter than the cull radius (nothing launched);
 *   SPH_ERR_NONFINITE    a non-finite position, or a mass or h that is not finite
 *                        and positive (found on the device; rho must not be used);
 *   SPH_ERR_OUTSIDE      a finite position outside [lo, hi] on any axis, periodic
 *                        axes included (found on the device; rho must not be used);
 *   SPH_ERR_CUDA         no current device, the scratch address lookup failed, or
 *                        a CUDA call or launch of this entry point failed. */
int sph_density_noalloc(const SphParams* params, const SphBox* box, int64_t n, const double* x, const double* y,
                        const double* z, const double* mass, const double* h, double* rho, void* stream);

const char* sph_last_error_string(void);

/* Test hook (no reference counterpart): the device allocation `after` places
 * from now (0 = the next one) inside this library's contexts is refused with
 * SPH_ERR_NOMEM, once; a negative value disarms it.  Used to check that every
 * allocation point fails cleanly and leaves the context destroyable and
 * usable again.  Returns the previous setting. */
long long sphx_fail_alloc_after(long long after);

/* Diagnostic hook (no reference counterpart): the cell grid box `box` ran its
 * last neighbour build on, out[12] = cells per axis (3), cell edges (3),
 * level-1 splits per axis (3), levels, the smallest level-1 edge, the h cap. */
int sphx_box_grid(sph_ctx* ctx, int32_t box, double* out);

/* Diagnostic hook (no reference counterpart): the FP32 pair records of one
 * species as the last neighbour build made them, pm[4 n] in input order:
 * position relative to the lower corner of its cell (x, y, z) and mass.
 * FP32-compensated contexts only. */
int sphx_get_pair_records(sph_ctx* ctx, int32_t species_id, float* pm);

#ifdef __cplusplus
}
#endif
#endif /* SPEARHED_B200_H */
