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
