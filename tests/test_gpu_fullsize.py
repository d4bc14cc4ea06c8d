"""The benchmark configurations at their full sizes, through the C ABI, against
the CPU oracle (FP64).

One step of each configuration at the size it is benchmarked at:
  - Orszag-Tang slab 512 x 512 x 4 (1,048,576 particles, Wendland C2, SPMHD);
  - MHD rotor 1024 x 1024 x 4 (5.4 M, adaptive h, two cell levels);
  - magnetised Kelvin-Helmholtz 256^3 (16.8 M, jitter, adaptive h);
  - the Brio-Wu ensemble, all 512 boxes (31.3 M, cubic spline, per-box dt).
For each, in FP64-plain and in FP32-compensated:
  - the accepted pair set of the step's neighbour build equals the oracle's
    (per-particle counts, exact, in the precision's own geometry);
  - FP64: positions <= 1e-12 absolute, density rel <= 1e-10, velocities,
    accelerations, du/dt and dB/dt normwise <= 1e-9;
  - FP32: density rel <= 1e-5, accelerations, du/dt and dB/dt normwise <= 1e-4
    (the one-step bounds the FP32 path is built to), div B normwise <= 1e-4
    of |B|/h;
  - the conserved-quantity reductions of sph_reduce (total energy, momentum,
    <|div B| h/|B|> and max |div B| h/|B|) against the oracle's.
And the Sod shock tube at its full 18,432 particles for all 50 steps, the
oracle being the same run in FP64: the GPU FP64 run tracks it (time, positions,
density), and the FP32 run, given the oracle's time steps, stays within the
density bound; both runs' total-energy drift matches the oracle's drift.

The oracle runs on every host core (OpenMP); the whole file takes a few
minutes, most of it the oracle on the 16.8 M and 31.3 M particle inputs.
"""
import numpy as np
import pytest

from spearhed_b200 import abi, setups

pytestmark = [pytest.mark.gpu, pytest.mark.fullsize]

FP64, FP32 = abi.PREC_FP64, abi.PREC_FP32_COMP

FULL = {
    "orszag_tang": lambda prec: setups.orszag_tang(precision=prec),
    "mhd_rotor": lambda prec: setups.mhd_rotor(precision=prec),
    "kelvin_helmholtz": lambda prec: setups.kelvin_helmholtz(precision=prec),
    "brio_wu_ensemble": lambda prec: setups.brio_wu_ensemble(precision=prec),
}
# one configuration's oracle results are cached at a time, so both precisions
# of a configuration run back to back
CASES = [(name, prec) for name in FULL for prec in (FP64, FP32)]


def _normwise(got, ref):
    scale = float(np.max(np.abs(ref)))
    return float(np.max(np.abs(got - ref)) / scale) if scale > 0 else float(np.max(np.abs(got)))


def _energy(d):
    return d["e_kin"] + d["e_int"] + d["e_mag"]


def _diag(d):
    return {"e_kin": d.e_kin, "e_int": d.e_int, "e_mag": d.e_mag, "mom": list(d.mom),
            "divb_mean": d.divb_mean, "divb_max": d.divb_max}


@pytest.fixture(scope="module")
def oracle_step(oracle):
    cache = {}

    def get(name):
        if name not in cache:
            cache.clear()
            w = FULL[name](FP64)
            s0 = w.species[abi.SPECIES_DEFAULT]
            roles = np.full(s0.n, abi.ROLES_DEFAULT, dtype=np.uint8)
            orc = oracle.System(w.params, w.boxes, s0.copy(), roles)
            orc.step(1, w.params.dt)
            # Step 1's neighbour build sees the drifted positions (the kick
            # moves no particle) and the initial smoothing lengths (the kick
            # sets the new ones): count the pairs at that state.
            probe = s0.copy()
            probe.pos[:] = orc.s.pos
            po = oracle.System(w.params, w.boxes, probe, roles)
            counts = {FP64: po.neighbour_counts(False)[0], FP32: po.neighbour_counts(True)[0]}
            del po, probe
            s = orc.s
            cache[name] = {"s": s, "diag": _diag(orc.reduce()), "counts": counts, "h0": w.params.h0,
                           "momentum_scale": float(np.sum(s.mass * np.linalg.norm(s.vel, axis=0)))}
        return cache[name]

    return get


@pytest.mark.parametrize("name,prec", CASES, ids=[f"{n}-{'fp64' if p == FP64 else 'fp32'}" for n, p in CASES])
def test_full_size_step_matches_oracle(oracle_step, name, prec):
    import spearhed_b200 as sb
    ref = oracle_step(name)
    w = FULL[name](prec)
    ctx = sb.context_for(w)
    del w
    ctx.step(1)
    got = ctx.get_species(abi.SPECIES_DEFAULT)
    counts = ctx.neighbour_counts(abi.SPECIES_DEFAULT)
    dg = ctx.reduce()
    ctx.close()
    o = ref["s"]
    # the accepted pair set of the step's neighbour build
    mism = int(np.count_nonzero(counts != ref["counts"][prec]))
    assert mism == 0, f"{mism} particles with a different accepted-neighbour count"
    errs = {
        "density": float(np.max(np.abs(got.density / o.density - 1.0))),
        "dvdt": _normwise(got.dvdt, o.dvdt),
        "dudt": _normwise(got.dudt, o.dudt),
    }
    bmag = np.linalg.norm(o.B, axis=0)
    mhd = float(np.max(bmag)) > 0
    if mhd:
        errs["dBdt"] = _normwise(got.dBdt, o.dBdt)
        # div B is a difference of O(|B|/h) terms: scale by that
        scale = float(np.max(bmag)) / float(np.min(o.h))
        errs["divB"] = float(np.max(np.abs(got.divB - o.divB))) / scale
    if prec == FP64:
        errs["pos"] = float(np.max(np.abs(got.pos - o.pos)))
        errs["vel"] = _normwise(got.vel, o.vel)
        errs["h"] = float(np.max(np.abs(got.h / o.h - 1.0)))
        bound = {"density": 1e-10, "dvdt": 1e-9, "dudt": 1e-9, "dBdt": 1e-9, "divB": 1e-9, "pos": 1e-12,
                 "vel": 1e-9, "h": 1e-10}
    else:
        bound = {"density": 1e-5, "dvdt": 1e-4, "dudt": 1e-4, "dBdt": 1e-4, "divB": 1e-4}
    bad = {k: v for k, v in errs.items() if not v <= bound[k]}
    assert not bad, (bad, errs)
    # conserved-quantity reductions (sph_reduce) against the oracle's
    od = ref["diag"]
    e_ref = od["e_kin"] + od["e_int"] + od["e_mag"]
    assert _energy(dg) == pytest.approx(e_ref, rel=1e-10 if prec == FP64 else 1e-6)
    for k in ("e_kin", "e_int", "e_mag"):
        assert dg[k] == pytest.approx(od[k], rel=1e-9 if prec == FP64 else 1e-5, abs=1e-14 * abs(e_ref))
    mom_tol = (1e-12 if prec == FP64 else 1e-6) * ref["momentum_scale"]
    assert np.max(np.abs(np.asarray(dg["mom"]) - np.asarray(od["mom"]))) <= mom_tol
    if mhd:
        # dimensionless <|div B| h/|B|> and its maximum: relative where div B is
        # resolved, absolute at the round-off floor of an exact lattice
        rel, floor = (1e-8, 1e-12) if prec == FP64 else (1e-3, 1e-4)
        for k in ("divb_mean", "divb_max"):
            assert abs(dg[k] - od[k]) <= rel * abs(od[k]) + floor, (k, dg[k], od[k])


def _sod_oracle_run(oracle, steps):
    """The FP64 oracle Sod run, one step per call: (system, times, energies)."""
    w = setups.sod_small(precision=FP64)
    s = w.species[abi.SPECIES_DEFAULT].copy()
    orc = oracle.System(w.params, w.boxes, s, np.full(s.n, abi.ROLES_DEFAULT, dtype=np.uint8))
    d0 = orc.reduce()
    energies = [d0.e_kin + d0.e_int + d0.e_mag]
    times = [0.0]
    dt_state, t = w.params.dt, 0.0
    for _ in range(steps):
        dt_state, t, d = orc.step(1, dt_state, t)
        times.append(t)
        energies.append(d.e_kin + d.e_int + d.e_mag)
    return orc, np.asarray(times), np.asarray(energies)


@pytest.fixture(scope="module")
def sod_oracle(oracle):
    return _sod_oracle_run(oracle, 50)


def test_sod_full_size_50_steps_fp64_matches_oracle_run(sod_oracle):
    import spearhed_b200 as sb
    orc, times, energies = sod_oracle
    w = setups.sod_small(precision=FP64)
    assert w.n == 18432
    ctx = sb.context_for(w)
    e0 = _energy(ctx.reduce())
    ctx.step(50)
    got = ctx.get_species(abi.SPECIES_DEFAULT)
    dg = ctx.reduce()
    ctx.close()
    errs = {"time": abs(dg["time"] / times[-1] - 1.0),
            "pos": float(np.max(np.abs(got.pos - orc.s.pos))),
            "density": float(np.max(np.abs(got.density / orc.s.density - 1.0))),
            "vel": _normwise(got.vel, orc.s.vel),
            "u": float(np.max(np.abs(got.u / orc.s.u - 1.0)))}
    bound = {"time": 1e-9, "pos": 1e-10, "density": 1e-8, "vel": 1e-7, "u": 1e-8}
    bad = {k: v for k, v in errs.items() if not v <= bound[k]}
    assert not bad, (bad, errs)
    drift_orc = (energies[-1] - energies[0]) / energies[0]
    drift_gpu = (_energy(dg) - e0) / e0
    assert abs(drift_gpu - drift_orc) <= 1e-6 * abs(drift_orc) + 1e-12, (drift_gpu, drift_orc)


def test_sod_full_size_50_steps_fp32_on_the_oracle_time_steps(sod_oracle):
    """FP32-compensated pair kernels over the oracle's own dt sequence (CFL off,
    dt given), so both runs reach the same times: density within 1e-5 of the
    FP64 oracle after 50 steps, and the FP32 run's energy drift within 1% of
    the oracle's FP64 drift (FP32 pair sums add no drift of their own)."""
    import spearhed_b200 as sb
    orc, times, energies = sod_oracle
    w = setups.sod_small(precision=FP32)
    w.params.physics &= ~abi.PHYS_CFL
    ctx = sb.context_for(w)
    e0 = _energy(ctx.reduce())
    for dt in np.diff(times):
        ctx.step(1, float(dt))
    got = ctx.get_species(abi.SPECIES_DEFAULT)
    dg = ctx.reduce()
    ctx.close()
    assert dg["time"] == pytest.approx(times[-1], rel=1e-12)
    rho_err = float(np.max(np.abs(got.density / orc.s.density - 1.0)))
    assert rho_err <= 1e-5, rho_err
    drift_orc = (energies[-1] - energies[0]) / energies[0]
    drift_gpu = (_energy(dg) - e0) / e0
    assert abs(drift_gpu - drift_orc) <= 0.01 * abs(drift_orc), (drift_gpu, drift_orc)
