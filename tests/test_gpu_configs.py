"""The remaining benchmark configurations at small sizes, against the oracle, and
the FP32 path's energy drift against the FP64 path's.

- Magnetised Kelvin-Helmholtz (two lattices, 2:1 density, jitter, adaptive h,
  pair-max cull) and the MHD rotor (10:1 density disc, rotation, adaptive h):
  two full steps match the oracle; FP64 to round-off, FP32 within the
  target error bounds after one step (density 1e-5, accelerations 1e-4).
- Energy drift: 100 steps of the jittered Orszag-Tang slab, FP32-compensated
  versus FP64 plain; the FP32 run's relative drift of the total energy
  (kinetic + internal + magnetic) stays within 2% of the FP64 run's drift (or
  1e-7 absolute), i.e. FP32 pair kernels add no drift of their own.
"""
import numpy as np
import pytest

from spearhed_b200 import abi, setups

pytestmark = pytest.mark.gpu


def _normwise(got, ref):
    return float(np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-300))


def _run(w, steps):
    import spearhed_b200 as sb
    ctx = sb.context_for(w)
    ctx.step(steps)
    out = ctx.get_species(abi.SPECIES_DEFAULT)
    d = ctx.reduce()
    ctx.close()
    return out, d


def _oracle_run(oracle, w, steps):
    s = w.species[abi.SPECIES_DEFAULT].copy()
    orc = oracle.System(w.params, w.boxes, s, np.full(s.n, abi.ROLES_DEFAULT, dtype=np.uint8))
    dts, t, d = orc.step(steps, w.params.dt)
    return orc, t, d


CONFIGS = {
    "kelvin_helmholtz": lambda prec: setups.kelvin_helmholtz(n_outer=32, n_band=40, precision=prec),
    "mhd_rotor": lambda prec: setups.mhd_rotor(nxy=64, nz=4, precision=prec),
}


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_config_fp64_two_steps_match_oracle(oracle, name):
    w = CONFIGS[name](abi.PREC_FP64)
    got, dg = _run(w, 2)
    orc, t, d = _oracle_run(oracle, w, 2)
    assert dg["time"] == pytest.approx(t, rel=1e-12)
    assert np.max(np.abs(got.pos - orc.s.pos)) <= 1e-12
    assert _normwise(got.vel, orc.s.vel) <= 1e-9
    assert np.max(np.abs(got.density / orc.s.density - 1)) <= 1e-10
    assert np.max(np.abs(got.h / orc.s.h - 1)) <= 1e-10
    assert _normwise(got.B, orc.s.B) <= 1e-9
    assert dg["e_kin"] + dg["e_int"] + dg["e_mag"] == pytest.approx(d.e_kin + d.e_int + d.e_mag, rel=1e-10)


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_config_fp32_one_step_within_target_bounds(oracle, name):
    import spearhed_b200 as sb
    w = CONFIGS[name](abi.PREC_FP32_COMP)
    ctx = sb.context_for(w)
    ctx.step(1)
    got = ctx.get_species(abi.SPECIES_DEFAULT)
    ctx.close()
    orc, _, _ = _oracle_run(oracle, CONFIGS[name](abi.PREC_FP64), 1)
    assert np.max(np.abs(got.density / orc.s.density - 1)) <= 1e-5
    assert _normwise(got.dvdt, orc.s.dvdt) <= 1e-4
    assert _normwise(got.dBdt, orc.s.dBdt) <= 1e-4


def test_fp32_energy_drift_matches_fp64():
    import spearhed_b200 as sb
    drift = {}
    for prec in (abi.PREC_FP64, abi.PREC_FP32_COMP):
        w = setups.orszag_tang(nx=64, nz=4, precision=prec, jitter=0.1)
        ctx = sb.context_for(w)
        ctx.step(1)
        d0 = ctx.reduce()
        ctx.step(100)
        d1 = ctx.reduce()
        ctx.close()
        e0 = d0["e_kin"] + d0["e_int"] + d0["e_mag"]
        e1 = d1["e_kin"] + d1["e_int"] + d1["e_mag"]
        drift[prec] = (e1 - e0) / e0
    d64, d32 = drift[abi.PREC_FP64], drift[abi.PREC_FP32_COMP]
    assert abs(d32 - d64) <= 0.02 * abs(d64) + 1e-7, drift
