"""Launch-shape tuning of the pair kernels.

- Every shape (staging depth, register caps, cull unroll) gives the same bits as the
  default: the shapes change windows and register allocation, not arithmetic
  or summation order.
- sph_autotune leaves the particles, the clock and the step count as they were,
  and reports a time for every shape it tried.
"""
import numpy as np
import pytest

from spearhed_b200 import abi, setups

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "vel", "u", "density", "h", "B", "psi", "dvdt", "dBdt")


def _steps(w, dv, fv, n=3):
    import spearhed_b200 as sb
    ctx = sb.context_for(w)
    ctx.set_tuning(dv, fv)
    ctx.step(n)
    out = ctx.get_species(abi.SPECIES_DEFAULT)
    ctx.close()
    return out


# OT: one level, global cull, mostly full chunks.  Rotor and a small Brio-Wu
# ensemble: two cell levels, the pair-max cull and cells of few targets, so the
# short chunks' slab cull, the skewed staging slabs and the own-entry positions
# run in every shape.
SHAPE_CASES = {
    "orszag_tang": lambda prec: setups.orszag_tang(nx=32, nz=4, precision=prec, jitter=0.1),
    "mhd_rotor": lambda prec: setups.mhd_rotor(nxy=64, precision=prec),
    "brio_wu_ensemble": lambda prec: setups.brio_wu_ensemble(nbox=6, n_lo=4096, n_hi=16384, precision=prec),
}


@pytest.mark.parametrize("prec", [abi.PREC_FP32_COMP, abi.PREC_FP64])
@pytest.mark.parametrize("case", list(SHAPE_CASES))
def test_every_shape_gives_the_same_bits(prec, case):
    import spearhed_b200 as sb
    w = SHAPE_CASES[case](prec)
    probe = sb.context_for(w)
    t = probe.tuning()
    probe.close()
    ref = _steps(w, 0, 0)
    for dv in range(t["n_density_variants"]):
        for fv in range(t["n_force_variants"]):
            if dv == 0 and fv == 0:
                continue
            got = _steps(w, dv, fv)
            for f in FIELDS:
                assert np.array_equal(getattr(got, f), getattr(ref, f)), (dv, fv, f)


def test_autotune_keeps_the_state():
    import spearhed_b200 as sb
    w = setups.sod_small(precision=abi.PREC_FP32_COMP, scale=0.5)
    ctx = sb.context_for(w)
    ctx.step(2)
    before = ctx.get_species(abi.SPECIES_DEFAULT)
    clock0 = ctx.clock()
    d0 = ctx.reduce()
    t = ctx.autotune(2)
    after = ctx.get_species(abi.SPECIES_DEFAULT)
    clock1 = ctx.clock()
    d1 = ctx.reduce()
    for f in ("pos", "vel", "u", "density", "h"):
        assert np.array_equal(getattr(after, f), getattr(before, f)), f
    assert np.array_equal(clock0[0], clock1[0]) and np.array_equal(clock0[1], clock1[1])
    assert d1["steps"] == d0["steps"] == 2
    assert len(t["density_ms"]) == t["n_density_variants"] >= 2
    assert all(x > 0 for x in t["density_ms"] + t["force_ms"])
    assert 0 <= t["density_variant"] < t["n_density_variants"]
    assert t["staging_depth"] in (128, 256)
    assert t["cull_unroll"] in ((8, 2) if t["n_density_variants"] == 8 else (0,))
    # the context keeps stepping with the chosen shapes
    ctx.step(1)
    assert ctx.reduce()["steps"] == 3
    ctx.close()
