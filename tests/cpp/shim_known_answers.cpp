// The reference's known-answer unit tests, driven through the header-only C++
// shim (include/spearhed_b200.hpp) with its reference-shaped call sites:
//
//   density_colocated  tests/spearhed/unit/DensitySummation/DensitySummation.cpp:232-280
//                      4 co-located particles, m = 1, h = 0.5: rho = 4 m W(0, h)
//   density_line       DensitySummation.cpp:283-344
//                      3 particles in a line, dx = 1.5, h = 1, m = 1.5:
//                      edges m (W(0) + W(dx)), middle m (W(0) + 2 W(dx))
//   hydro_pair         tests/spearhed/unit/HydroForces/HydroForces.cpp:159-239
//                      2 particles at rest, d = 0.4, h = 0.5, m = rho = u = 1:
//                      dvdt_x = -/+ m 2 P/rho^2 dWdr(d, h), dudt = 0
//   timestep           tests/spearhed/unit/SimulationTimestep/SimulationTimestep.cpp:272-330
//                      2 Default (x 0.45, v 0.01), 1 Boundary (x 0.525), 1 Tracer
//                      (x 0.35, v 0.02), dt 0.01: runOneStep x 3 in one call against
//                      three single-step calls
//
// Usage: shim_known_answers <test> <fp64|fp32>.  Prints one line per particle,
// "<test> <species> <i> key=value ...", for the test to compare with the
// expected values (computed from the oracle's kernel functions and the
// oracle's run); exits non-zero when a shim call throws.
#include "spearhed_b200.hpp"

#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

namespace sb = spearhed_b200;

namespace
{
    struct Columns
    {
        std::vector<double> pos[3], vel[3], mass, h, rho, u, dvdt[3], dudt;

        explicit Columns(size_t n)
        {
            for(int a = 0; a < 3; ++a)
            {
                pos[a].assign(n, 0.0);
                vel[a].assign(n, 0.0);
                dvdt[a].assign(n, 0.0);
            }
            mass.assign(n, 0.0);
            h.assign(n, 0.0);
            rho.assign(n, 0.0);
            u.assign(n, 0.0);
            dudt.assign(n, 0.0);
        }
        size_t size() const
        {
            return mass.size();
        }
        SphSoAView view()
        {
            SphSoAView v{};
            for(int a = 0; a < 3; ++a)
            {
                v.pos[a] = pos[a].data();
                v.vel[a] = vel[a].data();
                v.dvdt[a] = dvdt[a].data();
            }
            v.mass = mass.data();
            v.h = h.data();
            v.density = rho.data();
            v.u = u.data();
            v.dudt = dudt.data();
            return v;
        }
    };

    void print(char const* test, char const* species, Columns const& c)
    {
        for(size_t i = 0; i < c.size(); ++i)
            std::printf(
                "%s %s %zu x=%.17g y=%.17g z=%.17g vx=%.17g vy=%.17g vz=%.17g rho=%.17g u=%.17g ax=%.17g ay=%.17g "
                "az=%.17g dudt=%.17g\n",
                test,
                species,
                i,
                c.pos[0][i],
                c.pos[1][i],
                c.pos[2][i],
                c.vel[0][i],
                c.vel[1][i],
                c.vel[2][i],
                c.rho[i],
                c.u[i],
                c.dvdt[0][i],
                c.dvdt[1][i],
                c.dvdt[2][i],
                c.dudt[i]);
    }

    SphParams params(int precision, double h0)
    {
        SphParams p;
        sph_default_params(&p);
        p.kernel = SPH_KERNEL_CUBIC;
        p.precision = precision;
        p.h0 = h0;
        return p;
    }

    void densityColocated(int precision)
    {
        Columns c(4);
        for(size_t i = 0; i < c.size(); ++i)
        {
            c.mass[i] = 1.0;
            c.h[i] = 0.5;
        }
        sb::Context ctx(params(precision, 0.5));
        SphSoAView v = c.view();
        ctx.setSpecies(SPH_SPECIES_DEFAULT, int64_t(c.size()), v);
        sb::UpdateDensity<sb::CubicSplineKernel>{}(ctx);
        ctx.getSpecies(SPH_SPECIES_DEFAULT, v);
        print("density_colocated", "default", c);
    }

    void densityLine(int precision)
    {
        Columns c(3);
        for(size_t i = 0; i < c.size(); ++i)
        {
            c.pos[0][i] = 1.5 * double(i);
            c.mass[i] = 1.5;
            c.h[i] = 1.0;
        }
        sb::Context ctx(params(precision, 1.0));
        SphSoAView v = c.view();
        ctx.setSpecies(SPH_SPECIES_DEFAULT, int64_t(c.size()), v);
        sb::UpdateDensity<sb::CubicSplineKernel>{}(ctx);
        ctx.getSpecies(SPH_SPECIES_DEFAULT, v);
        print("density_line", "default", c);
    }

    void hydroPair(int precision)
    {
        Columns c(2);
        c.pos[0][0] = -0.2;
        c.pos[0][1] = 0.2;
        for(size_t i = 0; i < c.size(); ++i)
        {
            c.mass[i] = 1.0;
            c.h[i] = 0.5;
            c.rho[i] = 1.0;
            c.u[i] = 1.0;
        }
        sb::Context ctx(params(precision, 0.5));
        SphSoAView v = c.view();
        ctx.setSpecies(SPH_SPECIES_DEFAULT, int64_t(c.size()), v);
        sb::UpdateDensity<sb::CubicSplineKernel>{}(ctx);
        sb::UpdateHydroForces<sb::CubicSplineKernel>{}(ctx);
        ctx.getSpecies(SPH_SPECIES_DEFAULT, v);
        print("hydro_pair", "default", c);
    }

    //! The tiny three-species setup of SimulationTimestep.cpp (TinySetupFor<2, 1, 1>).
    struct Tiny
    {
        Columns fluid{2}, wall{1}, tracer{1};
        Tiny()
        {
            auto place = [](Columns& c, double x, double v, bool thermo)
            {
                for(size_t i = 0; i < c.size(); ++i)
                {
                    c.pos[0][i] = x;
                    c.pos[1][i] = 0.45;
                    c.pos[2][i] = 0.45;
                    for(int a = 0; a < 3; ++a)
                        c.vel[a][i] = v;
                    c.mass[i] = 1.0;
                    c.h[i] = 0.05;
                    c.rho[i] = thermo ? 1.0 : 0.0;
                    c.u[i] = thermo ? 1.0 : 0.0;
                }
            };
            place(fluid, 0.45, 0.01, true);
            place(wall, 0.525, 0.0, true);
            place(tracer, 0.35, 0.02, false);
        }
    };

    void runTiny(int precision, bool oneCall, Tiny& t)
    {
        SphParams p = params(precision, 0.05);
        p.dt = 0.01;
        p.gamma = 5.0 / 3.0;
        sb::Context ctx(p, {SphBox{{-1, -1, -1}, {1, 1, 1}, {0, 0, 0}}});
        SphSoAView vf = t.fluid.view(), vw = t.wall.view(), vt = t.tracer.view();
        ctx.setSpecies(SPH_SPECIES_DEFAULT, int64_t(t.fluid.size()), vf);
        ctx.setSpecies(SPH_SPECIES_BOUNDARY, int64_t(t.wall.size()), vw);
        ctx.setSpecies(SPH_SPECIES_TRACER, int64_t(t.tracer.size()), vt);
        if(oneCall)
            sb::runOneStep(ctx, 3);
        else
            for(int s = 0; s < 3; ++s)
                sb::runOneStep(ctx, 1);
        ctx.getSpecies(SPH_SPECIES_DEFAULT, vf);
        ctx.getSpecies(SPH_SPECIES_BOUNDARY, vw);
        ctx.getSpecies(SPH_SPECIES_TRACER, vt);
        if(ctx.reduce().steps != 3)
            throw std::runtime_error("step count");
    }

    void timestep(int precision)
    {
        Tiny composed, sequential;
        runTiny(precision, true, composed);
        runTiny(precision, false, sequential);
        print("timestep_composed", "default", composed.fluid);
        print("timestep_composed", "boundary", composed.wall);
        print("timestep_composed", "tracer", composed.tracer);
        print("timestep_sequential", "default", sequential.fluid);
        print("timestep_sequential", "boundary", sequential.wall);
        print("timestep_sequential", "tracer", sequential.tracer);
    }
} // namespace

int main(int argc, char** argv)
{
    if(argc < 3)
    {
        std::fprintf(stderr, "usage: %s <density_colocated|density_line|hydro_pair|timestep> <fp64|fp32>\n", argv[0]);
        return 2;
    }
    int const precision = std::strcmp(argv[2], "fp32") == 0 ? SPH_PREC_FP32_COMP : SPH_PREC_FP64;
    std::string const test = argv[1];
    try
    {
        if(test == "density_colocated")
            densityColocated(precision);
        else if(test == "density_line")
            densityLine(precision);
        else if(test == "hydro_pair")
            hydroPair(precision);
        else if(test == "timestep")
            timestep(precision);
        else
        {
            std::fprintf(stderr, "unknown test %s\n", test.c_str());
            return 2;
        }
    }
    catch(std::exception const& e)
    {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
