"""Ensembles of independent boxes, CUDA-graph replay, and FP64 reproducibility.

- An ensemble (several boxes in one context) gives every box exactly the state
  it gets when run alone: same neighbour lists, same summation order, its own
  time step and Dedner speed (bitwise equal, FP64 and FP32).
- An ensemble matches the oracle run box by box (FP64).
- Replaying the step as a CUDA graph gives the same bits as launching it.
- Two FP64 runs of the same input give the same bits (fixed summation order).
"""
import numpy as np
import pytest

from spearhed_b200 import abi, setups

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "vel", "u", "density", "h", "B", "psi")


def _ensemble(sizes, prec, h_max=0.0):
    boxes, parts = [], []
    params = None
    for b, n in enumerate(sizes):
        p, box, s = setups.brio_wu_box(n, precision=prec, box_id=b)
        boxes.append(box)
        parts.append(s)
        params = p
    params.h_max = h_max
    return params, boxes, parts


def _run(params, boxes, species, steps, graph=False):
    import spearhed_b200 as sb
    ctx = sb.Context(params, boxes)
    ctx.set_species(abi.SPECIES_DEFAULT, species)
    if graph:
        ctx.use_graph(True)
    ctx.step(steps)
    out = ctx.get_species(abi.SPECIES_DEFAULT)
    diag = ctx.ensemble_reduce(len(boxes)) if len(boxes) > 1 else [ctx.reduce()]
    ctx.close()
    return out, diag


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32_COMP])
def test_ensemble_equals_independent_boxes(prec):
    params, boxes, parts = _ensemble([2000, 5200, 3100], prec)
    ens, dens = _run(params, boxes, abi.Species.concat(parts), 4)
    off = 0
    for b, s in enumerate(parts):
        one = s.copy()
        one.box_id[:] = 0
        alone, dal = _run(params, [boxes[b]], one, 4)
        for f in FIELDS:
            got = getattr(ens, f)[..., off:off + s.n]
            assert np.array_equal(got, getattr(alone, f)), (b, f)
        assert dens[b]["time"] == dal[0]["time"]
        assert dens[b]["dt_next"] == dal[0]["dt_next"]
        assert dens[b]["e_kin"] == pytest.approx(dal[0]["e_kin"], rel=1e-12)
        off += s.n
    # the boxes really have different time steps
    assert len({d["dt_next"] for d in dens}) == len(parts)


def test_ensemble_matches_oracle(oracle):
    # fixed h here: each box's cell size then follows from its own largest h on
    # both sides (under adaptive h the oracle re-derives the grid every step)
    params, boxes, parts = _ensemble([1500, 2600], abi.PREC_FP64)
    params.physics &= ~abi.PHYS_ADAPTIVE_H
    species = abi.Species.concat(parts)
    got, dg = _run(params, boxes, species, 3)
    orc = oracle.System(params, boxes, species.copy(), np.full(species.n, abi.ROLES_DEFAULT, dtype=np.uint8))
    dts, t, _ = orc.step(3, params.dt)
    for b in range(len(boxes)):
        assert dg[b]["time"] == pytest.approx(t[b], rel=1e-12)
        assert dg[b]["dt_next"] == pytest.approx(dts[b], rel=1e-9)
    assert np.max(np.abs(got.pos - orc.s.pos)) <= 1e-12
    assert np.max(np.abs(got.vel - orc.s.vel)) <= 1e-9 * max(1.0, np.max(np.abs(orc.s.vel)))
    assert np.max(np.abs(got.B - orc.s.B)) <= 1e-9
    assert np.max(np.abs(got.density / orc.s.density - 1)) <= 1e-10


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32_COMP])
def test_graph_replay_matches_eager(prec):
    w = setups.orszag_tang(nx=32, nz=4, precision=prec, jitter=0.1)
    s = w.species[abi.SPECIES_DEFAULT]
    eager, de = _run(w.params, w.boxes, s.copy(), 7)
    graph, dg = _run(w.params, w.boxes, s.copy(), 7, graph=True)
    for f in FIELDS:
        assert np.array_equal(getattr(eager, f), getattr(graph, f)), f
    assert de[0]["time"] == dg[0]["time"]


def test_fp64_runs_are_bit_reproducible():
    w = setups.sod_small(precision=abi.PREC_FP64, scale=0.5)
    s = w.species[abi.SPECIES_DEFAULT]
    a, _ = _run(w.params, w.boxes, s.copy(), 5)
    b, _ = _run(w.params, w.boxes, s.copy(), 5)
    for f in FIELDS:
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32_COMP])
def test_list_overflow_in_a_step_call_replays_from_its_start(prec):
    """A step call whose lists overflow (capacity forced to 32 entries for 92
    neighbours) restores the state it started from, regrows the lists and runs
    again: the result equals a run with large enough lists, bit for bit.  Both
    contexts get a fixed capacity, so neither runs the sizing pass (which sorts
    the particles once and so changes the summation order inside cells)."""
    import spearhed_b200 as sb
    w = setups.orszag_tang(nx=32, nz=4, precision=prec, jitter=0.1)
    s = w.species[abi.SPECIES_DEFAULT]
    w.params.max_neighbours = 256
    ref, dref = _run(w.params, w.boxes, s.copy(), 5)
    w.params.max_neighbours = 32
    ctx = sb.Context(w.params, w.boxes)
    ctx.set_species(abi.SPECIES_DEFAULT, s.copy())
    ctx.step(5)
    got = ctx.get_species(abi.SPECIES_DEFAULT)
    dg = ctx.reduce()
    assert int(np.max(ctx.neighbour_counts(abi.SPECIES_DEFAULT))) > 32
    ctx.close()
    for f in FIELDS:
        assert np.array_equal(getattr(got, f), getattr(ref, f)), f
    assert dg["time"] == dref[0]["time"]
    assert dg["steps"] == dref[0]["steps"] == 5
    # the call ran again once its lists had grown; the reference run never did
    assert dg["replays"] >= 1 and dref[0]["replays"] == 0
    assert dg["list_capacity"] > 32 and dref[0]["list_capacity"] == 256


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32_COMP])
def test_prepared_graph_leaves_the_state_and_replays_like_eager(prec):
    """sph_prepare_graph captures the next graph from a snapshot it restores:
    the clock and step count do not move, and the following steps (replayed)
    give the bits of eager steps from the same start."""
    import spearhed_b200 as sb
    w = setups.orszag_tang(nx=32, nz=4, precision=prec, jitter=0.1)
    eager = sb.context_for(w)
    eager.step(2)
    eager.step(4)
    ref = eager.get_species(abi.SPECIES_DEFAULT)
    dref = eager.reduce()
    eager.close()
    g = sb.context_for(w)
    g.use_graph(True)
    g.step(2)
    d0 = g.reduce()
    g.prepare_graph()
    d1 = g.reduce()
    assert d1["steps"] == d0["steps"] == 2 and d1["time"] == d0["time"]
    g.step(4)
    got = g.get_species(abi.SPECIES_DEFAULT)
    d = g.reduce()
    g.close()
    assert d["steps"] == dref["steps"] == 6 and d["time"] == dref["time"]
    for f in FIELDS:
        assert np.array_equal(getattr(got, f), getattr(ref, f)), f
