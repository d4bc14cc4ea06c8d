"""Default, Boundary and Tracer species stepped together (the reference's
SimulationTimestep and BoundaryConditions tests: Default + Boundary + Tracer,
walls frozen, interior confined).

A fluid slab between two frozen wall slabs (Boundary = Frozen|Source|
Thermodynamic) with drift-only tracers (Tracer = Movable), three full steps:

- the walls keep their positions, velocities, densities and energies bit for bit;
- tracers keep their velocities and move by v t (they are not sources);
- the fluid matches the oracle run of the same three species (FP64 to
  round-off, FP32 within 1e-4 density and 1e-3 velocity) and stays inside the walls;
- taking the tracers away changes no bit of the fluid.
"""
import numpy as np
import pytest

from spearhed_b200 import abi, setups

pytestmark = pytest.mark.gpu

DX = 0.025


def _slab(x0, x1, ny=10):
    nx = int(round((x1 - x0) / DX))
    return setups.lattice((x0, 0.0, 0.0), (x1, ny * DX, ny * DX), (nx, ny, ny))


def _species(pos, vel=None, u=1.5):
    n = pos.shape[1]
    s = abi.Species(n)
    s.pos[:] = pos
    s.vel[:] = 0.0 if vel is None else vel
    s.mass[:] = DX ** 3
    s.h[:] = 1.2 * DX
    s.density[:] = 1.0
    s.u[:] = u
    return s


def _setup(prec, tracers=True):
    fluid = _slab(0.2, 0.8)
    vel = np.zeros_like(fluid)
    vel[0] = 0.2 * np.sin(2 * np.pi * (fluid[0] - 0.2) / 0.6)
    walls = np.concatenate([_slab(0.1, 0.2), _slab(0.8, 0.9)], axis=1)
    species = {abi.SPECIES_DEFAULT: _species(fluid, vel), abi.SPECIES_BOUNDARY: _species(walls)}
    if tracers:
        rng = np.random.default_rng(7)
        tp = rng.uniform((0.3, 0.02, 0.02), (0.7, 0.23, 0.23), size=(64, 3)).T.copy()
        species[abi.SPECIES_TRACER] = _species(tp, rng.normal(scale=0.05, size=(3, 64)))
    params = abi.default_params(kernel=abi.KERNEL_CUBIC, precision=prec, physics=abi.PHYS_AV | abi.PHYS_CFL,
                                h0=1.2 * DX, gamma=1.4, dt=1e-3)
    box = abi.make_box((0.0, 0.0, 0.0), (1.0, 10 * DX, 10 * DX), (0, 1, 1))
    return params, [box], species


def _run(params, boxes, species, steps):
    import spearhed_b200 as sb
    ctx = sb.Context(params, boxes)
    for sid, s in species.items():
        ctx.set_species(sid, s.copy())
    ctx.step(steps)
    out = {sid: ctx.get_species(sid) for sid in species}
    d = ctx.reduce()
    ctx.close()
    return out, d


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32_COMP])
def test_walls_frozen_tracers_drift_fluid_matches_oracle(oracle, prec):
    params, boxes, species = _setup(prec)
    got, d = _run(params, boxes, species, 3)
    t = d["time"]
    assert d["steps"] == 3 and t > 0
    walls, w0 = got[abi.SPECIES_BOUNDARY], species[abi.SPECIES_BOUNDARY]
    for f in ("pos", "vel", "density", "u", "h"):
        assert np.array_equal(getattr(walls, f), getattr(w0, f)), f
    tr, t0 = got[abi.SPECIES_TRACER], species[abi.SPECIES_TRACER]
    assert np.array_equal(tr.vel, t0.vel)
    assert np.max(np.abs(tr.pos - (t0.pos + t0.vel * t))) <= 1e-13
    fluid = got[abi.SPECIES_DEFAULT]
    assert fluid.pos[0].min() > 0.1 and fluid.pos[0].max() < 0.9

    parts, roles = [], []
    for sid in sorted(species):
        parts.append(species[sid].copy())
        roles.append(np.full(species[sid].n, abi.SPECIES_ROLES[sid], dtype=np.uint8))
    p64 = abi.default_params(kernel=abi.KERNEL_CUBIC, precision=abi.PREC_FP64, physics=params.physics,
                             h0=params.h0, gamma=params.gamma, dt=params.dt)
    orc = oracle.System(p64, boxes, abi.Species.concat(parts), np.concatenate(roles))
    _, t_orc, _ = orc.step(3, params.dt)
    nf = fluid.n
    ref = orc.s
    if prec == abi.PREC_FP64:
        assert t == pytest.approx(t_orc, rel=1e-12)
        assert np.max(np.abs(fluid.pos - ref.pos[:, :nf])) <= 1e-12
        assert np.max(np.abs(fluid.density / ref.density[:nf] - 1)) <= 1e-10
        vel = ref.vel[:, :nf]
        assert np.max(np.abs(fluid.vel - vel)) / np.max(np.abs(vel)) <= 1e-9
    else:
        assert t == pytest.approx(t_orc, rel=1e-4)
        assert np.max(np.abs(fluid.density / ref.density[:nf] - 1)) <= 1e-4
        vel = ref.vel[:, :nf]
        assert np.max(np.abs(fluid.vel - vel)) / np.max(np.abs(vel)) <= 1e-3


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32_COMP])
def test_tracers_do_not_touch_the_fluid(prec):
    with_t, _ = _run(*_setup(prec, tracers=True), 3)
    without, _ = _run(*_setup(prec, tracers=False), 3)
    for f in ("pos", "vel", "density", "u", "h"):
        assert np.array_equal(getattr(with_t[abi.SPECIES_DEFAULT], f), getattr(without[abi.SPECIES_DEFAULT], f)), f


@pytest.mark.parametrize("sids", [(abi.SPECIES_DEFAULT,), (abi.SPECIES_DEFAULT, abi.SPECIES_BOUNDARY, abi.SPECIES_TRACER)])
def test_empty_setup_steps(sids):
    """An empty Default-only or all-species setup steps without error (the
    reference's runOneStep on an empty setup): the clock advances, the sums
    are zero and reading the empty species back gives nothing."""
    import spearhed_b200 as sb
    params = abi.default_params(dt=2e-3)
    ctx = sb.Context(params, [abi.make_box((0, 0, 0), (1, 1, 1))])
    for sid in sids:
        ctx.set_species(sid, abi.Species(0))
    ctx.step(3)
    ctx.density()
    d = ctx.reduce()
    assert d["steps"] == 3 and d["time"] == pytest.approx(6e-3)
    assert d["e_kin"] == d["e_int"] == d["pairs"] == 0 and d["n_targets"] == 0
    for sid in sids:
        assert ctx.get_species(sid).n == 0
    ctx.close()


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32_COMP])
def test_resetting_species_matches_a_fresh_context(prec):
    """Setting a species again on a used context (the reference's frame-index
    cache: fast path for the same particle count, rebuild when the topology
    changes) gives what a fresh context gives: bit for bit after a rebuild; to
    round-off on the fast path, which keeps the particles in their current
    sorted order (a stable sort then orders each cell differently from the
    input order, and so does the summation)."""
    import spearhed_b200 as sb
    params, boxes, species = _setup(prec, tracers=False)
    fluid = species[abi.SPECIES_DEFAULT]
    walls = species[abi.SPECIES_BOUNDARY]

    def fresh(s_fluid):
        out, _ = _run(params, boxes, {abi.SPECIES_DEFAULT: s_fluid, abi.SPECIES_BOUNDARY: walls}, 2)
        return out[abi.SPECIES_DEFAULT]

    ctx = sb.Context(params, boxes)
    ctx.set_species(abi.SPECIES_DEFAULT, fluid.copy())
    ctx.set_species(abi.SPECIES_BOUNDARY, walls.copy())
    ctx.step(2)
    # same count: new values through the fast path
    moved = fluid.copy()
    moved.vel[0] *= -1.0
    ctx.set_species(abi.SPECIES_DEFAULT, moved.copy())
    ctx.set_clock(0.0, params.dt)
    ctx.step(2)
    a = ctx.get_species(abi.SPECIES_DEFAULT)
    # changed count: the layout is rebuilt
    keep = np.arange(fluid.n) % 7 != 0
    fewer = abi.Species(int(keep.sum()))
    for c in abi.COLUMNS:
        getattr(fewer, c)[...] = getattr(fluid, c)[..., keep]
    fewer.box_id[:] = 0
    ctx.set_species(abi.SPECIES_DEFAULT, fewer.copy())
    ctx.set_clock(0.0, params.dt)
    ctx.step(2)
    b = ctx.get_species(abi.SPECIES_DEFAULT)
    ctx.close()
    ra, rb = fresh(moved), fresh(fewer)
    for f in ("pos", "vel", "density", "u"):
        assert np.array_equal(getattr(b, f), getattr(rb, f)), ("fewer", f)
    tol = 1e-12 if prec == abi.PREC_FP64 else 1e-5
    assert np.max(np.abs(a.pos - ra.pos)) <= tol
    assert np.max(np.abs(a.density / ra.density - 1)) <= tol
    assert np.max(np.abs(a.vel - ra.vel)) / np.max(np.abs(ra.vel)) <= 10 * tol
