"""Error statuses of the C ABI, raised through the host and the kernels' status
words (no GPU fault is involved: the kernels count bad particles, the host
reads the counts and returns a status).

- set-up: non-finite positions, h <= 0, non-positive source masses and
  particles outside their box (on any axis, periodic ones included) are refused;
- stepping: a particle driven out of a non-periodic box is reported by the
  drift kernel (SPH_ERR_OUTSIDE);
- the same-size fast path of sph_set_species checks h and masses on the device.
"""
import numpy as np
import pytest

from spearhed_b200 import abi

pytestmark = pytest.mark.gpu


def _cloud(n=400, seed=3):
    rng = np.random.default_rng(seed)
    s = abi.Species(n)
    s.pos[:] = rng.uniform(0.2, 0.8, size=(3, n))
    s.h[:] = 0.08
    s.mass[:] = 1e-3
    s.density[:] = 1.0
    s.u[:] = 1.0
    return s


def _ctx(s, periodic=(0, 0, 0)):
    import spearhed_b200 as sb
    ctx = sb.Context(abi.default_params(h0=0.08), [abi.make_box((0, 0, 0), (1, 1, 1), periodic)])
    ctx.set_species(abi.SPECIES_DEFAULT, s)
    return ctx


def _code(fn):
    with pytest.raises(abi.SphError) as e:
        fn()
    return e.value.code


@pytest.mark.parametrize("field,value,code", [
    ("pos", np.nan, abi.SPH_ERR_NONFINITE),
    ("h", 0.0, abi.SPH_ERR_NONFINITE),
    ("mass", -1.0, abi.SPH_ERR_NONFINITE),
    ("pos", 1.5, abi.SPH_ERR_OUTSIDE),
])
def test_bad_input_is_refused(field, value, code):
    s = _cloud()
    getattr(s, field)[..., 7] = value
    ctx = _ctx(s)
    assert _code(lambda: ctx.step(1)) == code
    ctx.close()


def test_particle_leaving_a_closed_box_is_reported():
    s = _cloud()
    s.vel[0, 11] = 1e3  # crosses x = 1 within the first drift
    ctx = _ctx(s)
    assert _code(lambda: ctx.step(2, 1e-3)) == abi.SPH_ERR_OUTSIDE
    ctx.close()


def test_outside_a_periodic_axis_is_refused_at_set_up():
    s = _cloud()
    s.pos[0, 7] = 1.5  # periodic axis, but outside [lo, hi]: the cell search would miss pairs
    ctx = _ctx(s, periodic=(1, 1, 1))
    assert _code(lambda: ctx.step(1)) == abi.SPH_ERR_OUTSIDE
    ctx.close()


def test_upper_face_of_a_periodic_axis_is_the_lower_face():
    """x = hi is accepted on a periodic axis and is the same place as x = lo:
    every density agrees to round-off (the positions relative to the cells differ)."""
    import spearhed_b200 as sb
    rng = np.random.default_rng(4)
    n = 600
    s = abi.Species(n)
    s.pos[:] = rng.uniform(0.0, 1.0, size=(3, n))
    s.pos[0, :40] = 0.0
    s.h[:] = 0.08
    s.mass[:] = 1e-3
    s.u[:] = 1.0
    p = abi.default_params(h0=0.08, precision=abi.PREC_FP64)
    box = [abi.make_box((0, 0, 0), (1, 1, 1), (1, 1, 1))]
    rho = []
    for x0 in (0.0, 1.0):
        t = s.copy()
        t.pos[0, :40] = x0
        ctx = sb.Context(p, box)
        ctx.set_species(abi.SPECIES_DEFAULT, t)
        ctx.density()
        rho.append(ctx.get_species(abi.SPECIES_DEFAULT).density.copy())
        ctx.close()
    assert np.max(np.abs(rho[1] / rho[0] - 1.0)) < 1e-12


def test_periodic_axis_wraps_instead():
    s = _cloud()
    s.vel[0, 11] = 1e3
    ctx = _ctx(s, periodic=(1, 1, 1))
    ctx.step(2, 1e-3)
    got = ctx.get_species(abi.SPECIES_DEFAULT)
    assert 0.0 <= got.pos[0, 11] < 1.0
    ctx.close()


def test_fast_path_checks_smoothing_lengths_on_the_device():
    s = _cloud()
    ctx = _ctx(s)
    ctx.step(1)
    bad = ctx.get_species(abi.SPECIES_DEFAULT)
    bad.h[5] = -1.0  # same count: the values go straight to the device
    assert _code(lambda: ctx.set_species(abi.SPECIES_DEFAULT, bad)) == abi.SPH_ERR_NONFINITE
    ok = ctx.get_species(abi.SPECIES_DEFAULT)
    ok.h[:] = 0.08
    ctx.set_species(abi.SPECIES_DEFAULT, ok)
    ctx.step(1)
    ctx.close()


# ---- bounded waits (sph_set_wait_timeout / sph_wait) ----------------------
FIELDS = ("pos", "vel", "density", "u", "h", "B", "psi")


def _same(a, b):
    for f in FIELDS:
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


def test_step_past_its_wait_limit_times_out_and_completes_later():
    """Six steps of a 262,144-particle slab take milliseconds on the device; with
    a limit of 1 us the call returns SPH_ERR_TIMEOUT while its work runs on.
    sph_wait (no limit now) completes it, and the result is the one a call
    without a limit gives, bit for bit.  No kernel waits on anything: the
    work ends by itself, only the host stops waiting early."""
    import spearhed_b200 as sb
    from spearhed_b200 import setups
    w = setups.orszag_tang(nx=256, nz=4, precision=abi.PREC_FP32_COMP)
    s = w.species[abi.SPECIES_DEFAULT]
    ref = sb.Context(w.params, w.boxes)
    ref.set_species(abi.SPECIES_DEFAULT, s)
    ref.step(1)
    ref.step(6)
    want = ref.get_species(abi.SPECIES_DEFAULT)
    ref.close()
    ctx = sb.Context(w.params, w.boxes)
    ctx.set_species(abi.SPECIES_DEFAULT, s)
    ctx.step(1)
    ctx.set_wait_timeout(1e-6)
    assert _code(lambda: ctx.step(6)) == abi.SPH_ERR_TIMEOUT
    ctx.set_wait_timeout(0.0)
    ctx.wait()
    assert ctx.reduce()["steps"] == 7
    _same(ctx.get_species(abi.SPECIES_DEFAULT), want)
    ctx.close()


def test_timed_out_step_that_overflows_is_rolled_back():
    """A step call that times out and whose lists then turn out to have
    overflowed (capacity forced to 32 entries for ~92 neighbours) is rolled
    back when sph_wait runs its checks: SPH_ERR_OVERFLOW, the particles and the
    clock are those the call started from, the lists have grown, and the call
    run again gives the result of a run that never overflowed, bit for bit."""
    import spearhed_b200 as sb
    from spearhed_b200 import setups
    w = setups.orszag_tang(nx=192, nz=4, precision=abi.PREC_FP32_COMP, jitter=0.1)
    s = w.species[abi.SPECIES_DEFAULT]
    w.params.max_neighbours = 256
    ref = sb.Context(w.params, w.boxes)
    ref.set_species(abi.SPECIES_DEFAULT, s)
    ref.step(4)
    want = ref.get_species(abi.SPECIES_DEFAULT)
    ref.close()
    w.params.max_neighbours = 32
    ctx = sb.Context(w.params, w.boxes)
    ctx.set_species(abi.SPECIES_DEFAULT, s)
    before = ctx.get_species(abi.SPECIES_DEFAULT)
    ctx.set_wait_timeout(1e-6)
    assert _code(lambda: ctx.step(4)) == abi.SPH_ERR_TIMEOUT
    ctx.set_wait_timeout(0.0)
    assert _code(ctx.wait) == abi.SPH_ERR_OVERFLOW
    d = ctx.reduce()
    assert d["steps"] == 0 and d["time"] == 0.0 and d["list_capacity"] > 32
    _same(ctx.get_species(abi.SPECIES_DEFAULT), before)
    ctx.step(4)
    _same(ctx.get_species(abi.SPECIES_DEFAULT), want)
    ctx.close()


# ---- allocation failures (sphx_fail_alloc_after) --------------------------
def test_every_allocation_point_fails_cleanly_and_the_context_recovers():
    """The k-th device allocation is refused, for k = 0, 1, 2, ... until a run
    makes fewer allocations than k.  Each refusal surfaces as SPH_ERR_NOMEM
    from the call that needed the memory, or is absorbed where the memory was
    only headroom (the lists' growth ahead of need); the context is then used
    again as it is (the species and the clock set again, the steps run) and
    gives the result of a clean run, and it is destroyed without error."""
    import spearhed_b200 as sb
    from spearhed_b200 import setups
    L = abi.lib()
    w = setups.orszag_tang(nx=32, nz=4, precision=abi.PREC_FP64, jitter=0.1)
    s = w.species[abi.SPECIES_DEFAULT]

    def run(ctx):
        ctx.set_species(abi.SPECIES_DEFAULT, s)
        ctx.set_clock(0.0, w.params.dt)  # a refused call may have taken steps already
        ctx.step(3)
        return ctx.get_species(abi.SPECIES_DEFAULT)

    ref = sb.Context(w.params, w.boxes)
    want = run(ref)
    ref.close()
    refused = 0
    try:
        for k in range(400):
            L.sphx_fail_alloc_after(k)
            ctx = None
            try:
                ctx = sb.Context(w.params, w.boxes)
                got = run(ctx)
            except abi.SphError as e:
                assert e.code == abi.SPH_ERR_NOMEM, (k, e)
                refused += 1
                L.sphx_fail_alloc_after(-1)
                if ctx is not None:
                    got = run(ctx)  # the same context, used again
                else:
                    continue
            finally:
                armed = L.sphx_fail_alloc_after(-1)
            for f in FIELDS:
                assert np.allclose(getattr(got, f), getattr(want, f), rtol=1e-12, atol=1e-14), (k, f)
            ctx.close()
            if armed >= 0:
                break  # this run made fewer than k + 1 allocations: every point was covered
        else:
            pytest.fail("more than 400 allocations")
    finally:
        L.sphx_fail_alloc_after(-1)
    assert refused >= 20  # master columns, records, cells, sort, lists, snapshot, ...
