"""GPU parity: the CUDA path, called through the C ABI, against the CPU oracle.

Tolerances (written here, per field):
  - accepted pair sets: exact (per-particle neighbour counts equal the oracle's
    in the same precision's geometry);
  - FP64 plain: density rel 1e-12, accelerations / du/dt normwise 1e-10;
  - FP32 compensated vs the FP64 oracle: density rel 1e-5, accelerations and
    du/dt normwise 1e-4 (max |err| / max |reference|), dB/dt normwise 1e-4.
"""
import numpy as np
import pytest

from spearhed_b200 import abi, setups

pytestmark = pytest.mark.gpu

CUBIC, QUINTIC, WENDLAND = abi.KERNEL_CUBIC, abi.KERNEL_QUINTIC, abi.KERNEL_WENDLAND_C2
PRECS = [abi.PREC_FP64, abi.PREC_FP32_COMP]
TOL = {abi.PREC_FP64: dict(rho=1e-12, acc=1e-10), abi.PREC_FP32_COMP: dict(rho=1e-5, acc=1e-4)}


def _ctx(params, boxes, species):
    import spearhed_b200 as sb
    ctx = sb.Context(params, boxes)
    for sid, s in species.items():
        ctx.set_species(sid, s)
    return ctx


def _oracle(oracle, params, boxes, species):
    parts, roles = [], []
    for sid in sorted(species):
        parts.append(species[sid].copy())
        roles.append(np.full(species[sid].n, abi.SPECIES_ROLES[sid], dtype=np.uint8))
    s = abi.Species.concat(parts)
    return oracle.System(params, boxes, s, np.concatenate(roles))


def _normwise(got, ref):
    scale = np.max(np.abs(ref))
    return np.max(np.abs(got - ref)) / (scale if scale > 0 else 1.0)


# ---- the reference's known answers, through the ABI ----------------------
@pytest.mark.parametrize("prec", PRECS)
def test_colocated_density(oracle, prec):
    n, h, m = 4, 0.5, 1.0
    s = abi.Species(n)
    s.mass[:] = m
    s.h[:] = h
    p = abi.default_params(precision=prec, h0=h)
    ctx = _ctx(p, None, {abi.SPECIES_DEFAULT: s})
    ctx.density()
    rho = ctx.get_species(abi.SPECIES_DEFAULT).density
    expected = n * m * oracle.orc().orc_kernel_W(CUBIC, 1, 0.0, h)
    assert np.allclose(rho, expected, rtol=1e-5)
    assert np.array_equal(ctx.neighbour_counts(abi.SPECIES_DEFAULT), np.full(n, n - 1))


@pytest.mark.parametrize("prec", PRECS)
def test_three_in_a_line_density(oracle, prec):
    dx, h, m = 1.5, 1.0, 1.5
    s = abi.Species(3)
    s.pos[0] = [0.0, dx, 2 * dx]
    s.mass[:] = m
    s.h[:] = h
    p = abi.default_params(precision=prec, h0=h)
    ctx = _ctx(p, None, {abi.SPECIES_DEFAULT: s})
    ctx.density()
    rho = ctx.get_species(abi.SPECIES_DEFAULT).density
    o = oracle.orc()
    w0, w1 = o.orc_kernel_W(CUBIC, 1, 0.0, h), o.orc_kernel_W(CUBIC, 1, dx, h)
    assert rho[0] == pytest.approx(m * (w0 + w1), rel=1e-5)
    assert rho[2] == pytest.approx(m * (w0 + w1), rel=1e-5)
    assert rho[1] == pytest.approx(m * (w0 + 2 * w1), rel=1e-5)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("cull", [abi.CULL_GLOBAL, abi.CULL_PAIR_MAX])
@pytest.mark.parametrize("n", [33, 200])
def test_every_pair_in_reach(oracle, prec, cull, n):
    """ParticleParticleInteraction.cpp:134-207: with every particle in every
    other's reach, the accepted pairs are all n(n-1) ordered pairs, self
    excluded.  n particles in [0.4, 0.6]^3 with h = 0.5 (cull radius 1, above
    the cloud's diameter) in a non-periodic unit box: one cell holds them all,
    every acceptance mask is full, and the cell runs full chunks plus a short
    tail chunk (n = 33: one target on 32 sub-lanes; n = 200: eight targets on
    four).  The densities are the oracle's."""
    rng = np.random.default_rng(7)
    s = abi.Species(n)
    s.pos[:] = 0.4 + 0.2 * rng.random((3, n))
    s.mass[:] = 1.0 / n
    s.h[:] = 0.5
    p = abi.default_params(precision=prec, h0=0.5, cull=cull)
    boxes = [abi.make_box((0.0, 0.0, 0.0), (1.0, 1.0, 1.0))]
    ctx = _ctx(p, boxes, {abi.SPECIES_DEFAULT: s})
    ctx.density()
    counts = ctx.neighbour_counts(abi.SPECIES_DEFAULT)
    rho = ctx.get_species(abi.SPECIES_DEFAULT).density
    ctx.close()
    assert np.array_equal(counts, np.full(n, n - 1))
    orc = _oracle(oracle, p, boxes, {abi.SPECIES_DEFAULT: s})
    orc.density()
    rel = np.max(np.abs(rho / orc.s.density - 1.0))
    assert rel <= TOL[prec]["rho"], rel


@pytest.mark.parametrize("prec", PRECS)
def test_two_particles_at_rest_repel(oracle, prec):
    d, h = 0.4, 0.5
    s = abi.Species(2)
    s.pos[0] = [-d / 2, d / 2]
    s.mass[:] = 1.0
    s.h[:] = h
    s.density[:] = 1.0
    s.u[:] = 1.0
    p = abi.default_params(precision=prec, h0=h)
    ctx = _ctx(p, None, {abi.SPECIES_DEFAULT: s})
    ctx.density()
    # The reference test drives the hydro functor on the initial rho = 1.
    out = ctx.get_species(abi.SPECIES_DEFAULT)
    s2 = s.copy()
    s2.density[:] = 1.0
    ctx2 = _ctx(p, None, {abi.SPECIES_DEFAULT: s2})
    ctx2.density()
    ctx2.hydro()
    got = ctx2.get_species(abi.SPECIES_DEFAULT)
    # expected from the density the pass itself computed
    o = oracle.orc()
    rho = got.density[0]
    P = o.orc_pressure(0, 5 / 3, rho, 1.0)
    exp_left = 2 * P / (rho * rho) * o.orc_kernel_dWdr(CUBIC, 0, d, h)
    assert got.dvdt[0, 0] == pytest.approx(exp_left, rel=1e-4)
    assert got.dvdt[0, 1] == pytest.approx(-exp_left, rel=1e-4)
    assert np.allclose(got.dvdt[1:], 0.0, atol=1e-6)
    assert np.allclose(got.dudt, 0.0, atol=1e-6)
    assert out.density[0] == pytest.approx(rho)


# ---- random clouds: pair sets, density, forces ----------------------------
def _cloud(kernel, prec, n=3000, seed=5, periodic=(0, 1, 1), physics=0, cull=abi.CULL_GLOBAL, vary_h=False,
           h_lo=0.6):
    rng = np.random.default_rng(seed)
    s = abi.Species(n)
    s.pos[:] = rng.uniform(0.0, 1.0, size=(3, n))
    h0 = 0.07 if kernel != QUINTIC else 0.05
    s.h[:] = h0 * (rng.uniform(h_lo, 1.0, n) if vary_h else 1.0)
    s.mass[:] = rng.uniform(0.5, 1.5, n) * 1e-3
    s.u[:] = rng.uniform(0.5, 2.0, n)
    s.vel[:] = rng.normal(size=(3, n)) * 0.3
    p = abi.default_params(kernel=kernel, precision=prec, physics=physics, cull=cull, h0=h0, gamma=1.4)
    box = abi.make_box((0, 0, 0), (1, 1, 1), periodic)
    return p, [box], {abi.SPECIES_DEFAULT: s}


@pytest.mark.parametrize("kernel", [CUBIC, QUINTIC, WENDLAND])
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("cull,vary", [(abi.CULL_GLOBAL, False), (abi.CULL_PAIR_MAX, True)])
def test_density_and_pairs_match_oracle(oracle, kernel, prec, cull, vary):
    p, boxes, sp = _cloud(kernel, prec, cull=cull, vary_h=vary)
    ctx = _ctx(p, boxes, sp)
    ctx.density()
    got = ctx.get_species(abi.SPECIES_DEFAULT)
    counts = ctx.neighbour_counts(abi.SPECIES_DEFAULT)
    orc = _oracle(oracle, p, boxes, sp)
    ocounts, _ = orc.neighbour_counts(fp32_geometry=(prec == abi.PREC_FP32_COMP))
    assert np.array_equal(counts, ocounts)
    orc.density()
    rel = np.max(np.abs(got.density / orc.s.density - 1.0))
    assert rel <= TOL[prec]["rho"], rel


@pytest.mark.parametrize("kernel", [CUBIC, QUINTIC, WENDLAND])
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("h_lo,n", [(0.25, 6000), (0.4, 4000)])
def test_two_level_grid_pairs_match_oracle(oracle, kernel, prec, h_lo, n):
    """Smoothing lengths spanning 4x and 2.5x under the pair-max cull: the box
    runs two cell levels, the level-0 cells split in two along the axes their
    edge allows (the oracle searches one level); the accepted pair sets are the
    same and the densities agree to round-off."""
    p, boxes, sp = _cloud(kernel, prec, n=n, cull=abi.CULL_PAIR_MAX, vary_h=True, h_lo=h_lo)
    ctx = _ctx(p, boxes, sp)
    ctx.density()
    got = ctx.get_species(abi.SPECIES_DEFAULT)
    counts = ctx.neighbour_counts(abi.SPECIES_DEFAULT)
    orc = _oracle(oracle, p, boxes, sp)
    ocounts, _ = orc.neighbour_counts(fp32_geometry=(prec == abi.PREC_FP32_COMP))
    assert np.array_equal(counts, ocounts)
    orc.density()
    rel = np.max(np.abs(got.density / orc.s.density - 1.0))
    assert rel <= TOL[prec]["rho"], rel


@pytest.mark.parametrize("kernel", [CUBIC, WENDLAND])
@pytest.mark.parametrize("prec", PRECS)
def test_pairs_at_the_cull_radius_match_oracle(oracle, kernel, prec):
    """A dyadic lattice (spacing 1/16, 10 points per periodic axis) whose cull
    radius is exactly two spacings.  The cell edge is the radius widened by
    2^-20, so each axis holds four cells of 2.5 spacings (5/32): cell corners,
    cell-relative positions and every distance are exact.  Pairs at r = R and
    beyond are rejected (strict r^2 < R^2) and the 26 offsets with
    i^2 + j^2 + k^2 <= 3 are accepted, through the staging box test, in cells
    of 8 to 27 targets (short and full chunks)."""
    dx = 1.0 / 16.0
    g = np.arange(10) * dx
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    n = X.size
    s = abi.Species(n)
    s.pos[:] = np.stack([X.ravel(), Y.ravel(), Z.ravel()])
    s.h[:] = dx  # support 2h = 2 dx
    s.mass[:] = 1e-3
    s.u[:] = 1.0
    p = abi.default_params(kernel=kernel, precision=prec, h0=dx)
    boxes = [abi.make_box((0, 0, 0), (10 * dx,) * 3, (1, 1, 1))]
    sp = {abi.SPECIES_DEFAULT: s}
    ctx = _ctx(p, boxes, sp)
    ctx.density()
    got = ctx.get_species(abi.SPECIES_DEFAULT)
    counts = ctx.neighbour_counts(abi.SPECIES_DEFAULT)
    assert np.all(counts == 26)
    orc = _oracle(oracle, p, boxes, sp)
    ocounts, _ = orc.neighbour_counts(fp32_geometry=(prec == abi.PREC_FP32_COMP))
    assert np.array_equal(counts, ocounts)
    orc.density()
    rel = np.max(np.abs(got.density / orc.s.density - 1.0))
    assert rel <= TOL[prec]["rho"], rel
    ctx.close()


@pytest.mark.parametrize("kernel", [CUBIC, WENDLAND])
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("cull,vary", [(abi.CULL_GLOBAL, False), (abi.CULL_PAIR_MAX, True)])
def test_dense_cluster_matches_oracle(oracle, kernel, prec, cull, vary):
    """A tenth of the box's particles in a ball of radius 0.04 inside a uniform
    cloud: the cluster's cells hold hundreds of targets, so a cell runs many
    64-target chunk pairs, each with its own staging box, plus a short tail
    chunk; the accepted pair sets are the oracle's and the densities agree."""
    p, boxes, sp = _cloud(kernel, prec, n=3000, cull=cull, vary_h=vary)
    s = sp[abi.SPECIES_DEFAULT]
    rng = np.random.default_rng(11)
    k = 300
    d = rng.normal(size=(3, k))
    d *= 0.04 * rng.uniform(0.0, 1.0, k) ** (1 / 3) / np.linalg.norm(d, axis=0)
    s.pos[:, :k] = 0.5 + d
    ctx = _ctx(p, boxes, sp)
    ctx.density()
    got = ctx.get_species(abi.SPECIES_DEFAULT)
    counts = ctx.neighbour_counts(abi.SPECIES_DEFAULT)
    assert counts[:k].min() >= k - 1  # the whole cluster is in every member's reach
    orc = _oracle(oracle, p, boxes, sp)
    ocounts, _ = orc.neighbour_counts(fp32_geometry=(prec == abi.PREC_FP32_COMP))
    assert np.array_equal(counts, ocounts)
    orc.density()
    rel = np.max(np.abs(got.density / orc.s.density - 1.0))
    assert rel <= TOL[prec]["rho"], rel
    ctx.close()


@pytest.mark.parametrize("kernel", [CUBIC, QUINTIC, WENDLAND])
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("physics", [0, abi.PHYS_AV])
def test_hydro_matches_oracle(oracle, kernel, prec, physics):
    p, boxes, sp = _cloud(kernel, prec, physics=physics)
    ctx = _ctx(p, boxes, sp)
    ctx.density()
    ctx.hydro()
    got = ctx.get_species(abi.SPECIES_DEFAULT)
    orc = _oracle(oracle, p, boxes, sp)
    orc.density()
    orc.force()
    assert _normwise(got.dvdt, orc.s.dvdt) <= TOL[prec]["acc"]
    assert _normwise(got.dudt, orc.s.dudt) <= TOL[prec]["acc"]


@pytest.mark.parametrize("prec", PRECS)
def test_mhd_orszag_tang_small_matches_oracle(oracle, prec):
    # Jittered lattice: on the exact lattice div B is round-off (~1e-15) and
    # comparing it would compare noise with noise.
    w = setups.orszag_tang(nx=32, nz=4, precision=prec, jitter=0.1)
    ctx = _ctx(w.params, w.boxes, w.species)
    ctx.density()
    ctx.mhd()
    got = ctx.get_species(abi.SPECIES_DEFAULT)
    orc = _oracle(oracle, w.params, w.boxes, w.species)
    ocounts, _ = orc.neighbour_counts(fp32_geometry=(prec == abi.PREC_FP32_COMP))
    assert np.array_equal(ctx.neighbour_counts(abi.SPECIES_DEFAULT), ocounts)
    orc.density()
    orc.force()
    assert np.max(np.abs(got.density / orc.s.density - 1)) <= TOL[prec]["rho"]
    for f in ("dvdt", "dudt", "dBdt"):
        err = _normwise(getattr(got, f), getattr(orc.s, f))
        assert err <= TOL[prec]["acc"], (f, err)
    # div B and dpsi/dt are differences of O(|B|/h) terms: scale by that.
    ch, _ = orc.force()
    scale = np.max(np.linalg.norm(orc.s.B, axis=0)) / w.params.h0
    assert np.max(np.abs(got.divB - orc.s.divB)) / scale <= TOL[prec]["acc"]
    assert np.max(np.abs(got.dpsidt - orc.s.dpsidt)) / (ch * ch * scale) <= TOL[prec]["acc"]
    assert np.max(np.abs(orc.s.divB)) > 1e-3 * scale  # the jitter makes div B non-trivial


@pytest.mark.parametrize("prec", PRECS)
def test_sod_steps_match_oracle(oracle, prec):
    """Five full steps (drift, neighbours, density, forces with AV, kick, CFL dt)."""
    w = setups.sod_small(precision=prec, scale=0.5)
    ctx = _ctx(w.params, w.boxes, w.species)
    ctx.step(5)
    got = ctx.get_species(abi.SPECIES_DEFAULT)
    dg = ctx.reduce()
    orc = _oracle(oracle, w.params, w.boxes, w.species)
    dt, t, d = orc.step(5, w.params.dt)
    assert dg["time"] == pytest.approx(t, rel=1e-9 if prec == abi.PREC_FP64 else 1e-4)
    if prec == abi.PREC_FP64:
        assert np.max(np.abs(got.pos - orc.s.pos)) <= 1e-12
        assert _normwise(got.vel, orc.s.vel) <= 1e-9
        assert np.max(np.abs(got.u / orc.s.u - 1)) <= 1e-10
        assert np.max(np.abs(got.density / orc.s.density - 1)) <= 1e-10
    else:
        assert np.max(np.abs(got.density / orc.s.density - 1)) <= 1e-4
        assert _normwise(got.vel, orc.s.vel) <= 1e-3
    assert dg["e_kin"] + dg["e_int"] == pytest.approx(d.e_kin + d.e_int, rel=1e-6)


def test_sod_one_step_fp32_errors_within_target_bounds(oracle):
    """After one step: density rel <= 1e-5, acceleration normwise <= 1e-4 (FP32 vs FP64 oracle)."""
    w = setups.sod_small(precision=abi.PREC_FP32_COMP, scale=0.5)
    ctx = _ctx(w.params, w.boxes, w.species)
    ctx.step(1)
    got = ctx.get_species(abi.SPECIES_DEFAULT)
    orc = _oracle(oracle, w.params, w.boxes, w.species)
    orc.step(1, w.params.dt)
    assert np.max(np.abs(got.density / orc.s.density - 1)) <= 1e-5
    assert _normwise(got.dvdt, orc.s.dvdt) <= 1e-4
