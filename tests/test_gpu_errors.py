"""Error statuses of the C ABI, raised through the host and the kernels' status
words (no GPU fault is involved: the kernels count bad particles, the host
reads the counts and returns a status).

- set-up: non-finite positions, h <= 0, non-positive source masses and
  particles outside a non-periodic box axis are refused;
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
