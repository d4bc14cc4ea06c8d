"""Snapshots (openPMD record names, raw binary + JSON) and checkpoint/resume."""
import numpy as np
import pytest

from spearhed_b200 import abi, io, setups


def test_snapshot_roundtrip(tmp_path):
    p, box, s = setups.brio_wu_box(3000)
    s.density[:] = np.linspace(0.1, 1.0, s.n)
    s.psi[:] = np.linspace(-1, 1, s.n)
    s.box_id[:] = 3
    tracer = abi.Species(7)
    tracer.pos[:] = 0.25
    path = str(tmp_path / "snap")
    io.write_snapshot(path, {abi.SPECIES_DEFAULT: s, abi.SPECIES_TRACER: tracer}, step=12, time=0.5, dt=1e-3)
    back, header = io.read_snapshot(path)
    assert header["step"] == 12 and header["time"] == 0.5
    assert set(back) == {abi.SPECIES_DEFAULT, abi.SPECIES_TRACER}
    for c in ("pos", "vel", "mass", "density", "u", "h", "B", "psi"):
        assert np.array_equal(getattr(back[abi.SPECIES_DEFAULT], c), getattr(s, c)), c
    assert np.array_equal(back[abi.SPECIES_DEFAULT].box_id, s.box_id)
    assert np.array_equal(back[abi.SPECIES_TRACER].pos, tracer.pos)
    # the record names a validate_sod.py-style reader looks for
    recs = header["species"]["Default"]["records"]
    for name in ("position/x", "velocity/x", "mass_density", "specific_internal_energy", "mass", "id"):
        assert name in recs


@pytest.mark.gpu
def test_checkpoint_resume_continues_the_run(tmp_path):
    import spearhed_b200 as sb
    w = setups.orszag_tang(nx=32, nz=4, precision=abi.PREC_FP64, jitter=0.1)
    s = w.species[abi.SPECIES_DEFAULT]
    straight = sb.Context(w.params, w.boxes)
    straight.set_species(abi.SPECIES_DEFAULT, s.copy())
    straight.step(6)
    ref = straight.get_species(abi.SPECIES_DEFAULT)
    t_ref, _ = straight.clock()

    first = sb.Context(w.params, w.boxes)
    first.set_species(abi.SPECIES_DEFAULT, s.copy())
    first.step(3)
    path = str(tmp_path / "ck")
    io.save_checkpoint(first, path, w.boxes)
    first.close()
    ctx, ck = io.resume(path)
    assert ck.steps == 3
    ctx.step(3)
    got = ctx.get_species(abi.SPECIES_DEFAULT)
    t, _ = ctx.clock()
    assert t[0] == pytest.approx(t_ref[0], rel=1e-12)
    # only the order of sums inside cells differs after a restart
    assert np.max(np.abs(got.pos - ref.pos)) <= 1e-12
    assert np.max(np.abs(got.vel - ref.vel)) <= 1e-10
    assert np.max(np.abs(got.B - ref.B)) <= 1e-10


class _FakeContext:
    """Stands in for a Context on the host: a clock and sums that move per step."""

    def __init__(self):
        self.steps = 0

    def step(self, k, dt=0.0):
        self.steps += k

    def reduce(self):
        n = self.steps
        return {"steps": n, "time": 0.01 * n, "dt": 0.01, "dt_next": 0.01, "e_kin": 1.0 + n, "e_int": 2.0,
                "e_mag": 0.5, "mom": [0.0, 1e-3 * n, 0.0], "divb_mean": 1e-4, "divb_max": 1e-3, "c_h": 2.0,
                "pairs": 1000.0 * n, "replays": 0}

    def timings(self):
        return [0.1, 0.2, 0.3, 0.05, 0.7]


def test_diagnostics_log_lines(tmp_path):
    path = str(tmp_path / "diag.jsonl")
    rows = io.run_logged(_FakeContext(), 7, path, every=3, meta={"workload": "fake"})
    assert [r["step"] for r in rows] == [3, 6, 7]
    header, back = io.read_diagnostics(path)
    assert header["format"] == io.DIAG_FORMAT and header["workload"] == "fake"
    assert back == rows
    r = back[-1]
    assert r["e_tot"] == pytest.approx(8.0 + 2.0 + 0.5)
    assert r["mom"] == [0.0, 0.007, 0.0]
    assert r["density_ms"] == 0.2 and r["call_ms"] == 0.7
    with pytest.raises(ValueError):
        (tmp_path / "bad.jsonl").write_text('{"format": "other"}\n')
        io.read_diagnostics(str(tmp_path / "bad.jsonl"))


@pytest.mark.gpu
def test_diagnostics_log_of_a_run(tmp_path):
    import spearhed_b200 as sb
    w = setups.sod_small(scale=0.5)
    ctx = sb.context_for(w)
    rows = io.run_logged(ctx, 6, str(tmp_path / "sod.jsonl"), every=2)
    ctx.close()
    assert [r["step"] for r in rows] == [2, 4, 6]
    assert all(r["pairs"] > 0 and r["call_ms"] > 0 for r in rows)
    assert rows[-1]["time"] > rows[0]["time"] > 0
