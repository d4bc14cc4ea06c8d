"""The header-only C++ shim (include/spearhed_b200.hpp) against the reference's
known answers.

tests/cpp/shim_known_answers.cpp ports four of the reference's unit tests to
the shim's reference-shaped call sites (UpdateDensity<K>{}(ctx),
UpdateHydroForces<K>{}(ctx), runOneStep(ctx, n)):
  - DensitySummation.cpp:232-280: 4 co-located particles, rho = 4 m W(0, h),
    rel 1e-5;
  - DensitySummation.cpp:283-344: 3 particles in a line, edge and middle
    densities, rel 1e-5;
  - HydroForces.cpp:159-239: two particles at rest repel along x with
    |dvdt_x| = m 2 P/rho^2 |dWdr(d, h)| (rel 1e-4), dvdt_y = dvdt_z = dudt = 0
    (margin 1e-6);
  - SimulationTimestep.cpp:272-330: three steps composed in one runOneStep call
    equal three single-step calls within the reference's margin 2e-5, and match
    the oracle's three-step run (FP64 1e-12, FP32 2e-5 relative).
Expected values come from the oracle's kernel functions, which are pinned bit
for bit to the reference's own headers (tests/test_oracle_pins.py).

Without a GPU the program is only built and linked, and run without arguments
(usage exit, no CUDA call).
"""
import os
import subprocess

import numpy as np
import pytest

from spearhed_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "shim_known_answers.cpp")
CUBIC = abi.KERNEL_CUBIC


@pytest.fixture(scope="module")
def shim_exe(tmp_path_factory):
    exe = tmp_path_factory.mktemp("shim") / "shim_known_answers"
    lib = os.path.join(ROOT, "spearhed_b200", "_lib")
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
                        "-L", lib, "-lspearhed_b200", f"-Wl,-rpath,{lib}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return str(exe)


def test_shim_program_compiles_and_links(shim_exe):
    # no arguments: the usage message, before any library call
    r = subprocess.run([shim_exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


def _run(exe, test, prec):
    r = subprocess.run([exe, test, "fp64" if prec == abi.PREC_FP64 else "fp32"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    rows = {}
    for line in r.stdout.splitlines():
        f = line.split()
        rec = {k: float(v) for k, v in (kv.split("=") for kv in f[3:])}
        rows.setdefault((f[0], f[1]), []).append(rec)
    return rows


PRECS = [abi.PREC_FP64, abi.PREC_FP32_COMP]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", PRECS)
def test_shim_density_colocated(shim_exe, oracle, prec):
    rows = _run(shim_exe, "density_colocated", prec)[("density_colocated", "default")]
    expected = 4 * 1.0 * oracle.orc().orc_kernel_W(CUBIC, 1, 0.0, 0.5)
    assert len(rows) == 4
    for r in rows:
        assert r["rho"] == pytest.approx(expected, rel=1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", PRECS)
def test_shim_density_line(shim_exe, oracle, prec):
    rows = _run(shim_exe, "density_line", prec)[("density_line", "default")]
    o = oracle.orc()
    w0, w1 = o.orc_kernel_W(CUBIC, 1, 0.0, 1.0), o.orc_kernel_W(CUBIC, 1, 1.5, 1.0)
    edge, mid = 1.5 * (w0 + w1), 1.5 * (w0 + 2 * w1)
    rho = sorted(r["rho"] for r in rows)
    assert rho[0] == pytest.approx(edge, rel=1e-5)
    assert rho[1] == pytest.approx(edge, rel=1e-5)
    assert rho[2] == pytest.approx(mid, rel=1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", PRECS)
def test_shim_hydro_pair_repels(shim_exe, oracle, prec):
    rows = _run(shim_exe, "hydro_pair", prec)[("hydro_pair", "default")]
    o = oracle.orc()
    for r in rows:
        # the force uses the density the shim's UpdateDensity computed
        P = o.orc_pressure(0, 5.0 / 3.0, r["rho"], 1.0)
        expected_left = 1.0 * 2 * P / (r["rho"] ** 2) * o.orc_kernel_dWdr(CUBIC, 0, 0.4, 0.5)
        expected = expected_left if r["x"] < 0 else -expected_left
        assert r["ax"] == pytest.approx(expected, rel=1e-4)
        assert abs(r["ay"]) <= 1e-6 and abs(r["az"]) <= 1e-6
        assert abs(r["dudt"]) <= 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("prec", PRECS)
def test_shim_timestep_composed_equals_sequential_and_oracle(shim_exe, oracle, prec):
    rows = _run(shim_exe, "timestep", prec)
    keys = ("x", "y", "z", "vx", "vy", "vz", "rho", "u")
    for sp in ("default", "boundary", "tracer"):
        a, b = rows[("timestep_composed", sp)], rows[("timestep_sequential", sp)]
        assert len(a) == len(b)
        for ra, rb in zip(a, b):
            for k in keys:
                assert ra[k] == pytest.approx(rb[k], abs=2e-5), (sp, k)
    # the oracle's three steps of the same setup (all species, their roles)
    parts, roles = [], []
    for sid, x, v, thermo, n in ((abi.SPECIES_DEFAULT, 0.45, 0.01, True, 2),
                                 (abi.SPECIES_BOUNDARY, 0.525, 0.0, True, 1),
                                 (abi.SPECIES_TRACER, 0.35, 0.02, False, 1)):
        s = abi.Species(n)
        s.pos[0] = x
        s.pos[1:] = 0.45
        s.vel[:] = v
        s.mass[:] = 1.0
        s.h[:] = 0.05
        s.density[:] = 1.0 if thermo else 0.0
        s.u[:] = 1.0 if thermo else 0.0
        parts.append(s)
        roles.append(np.full(n, abi.SPECIES_ROLES[sid], dtype=np.uint8))
    p = abi.default_params(kernel=CUBIC, precision=abi.PREC_FP64, h0=0.05, dt=0.01, gamma=5.0 / 3.0)
    box = abi.make_box((-1, -1, -1), (1, 1, 1))
    orc = oracle.System(p, [box], abi.Species.concat(parts), np.concatenate(roles))
    orc.step(3, 0.01)
    # FP64 to round-off; FP32 pair sums against the FP64 oracle within 2e-5
    # relative (the wall repels the fluid to |v| ~ 64 in three steps)
    tol = 1e-12 if prec == abi.PREC_FP64 else 2e-5
    got = rows[("timestep_composed", "default")] + rows[("timestep_composed", "boundary")] + \
        rows[("timestep_composed", "tracer")]
    for i, r in enumerate(got):
        assert r["x"] == pytest.approx(orc.s.pos[0, i], rel=tol, abs=tol)
        assert r["vx"] == pytest.approx(orc.s.vel[0, i], rel=tol, abs=tol)
        if i < 3:  # Default and Boundary carry rho and u
            assert r["rho"] == pytest.approx(orc.s.density[i], rel=tol, abs=tol)
            assert r["u"] == pytest.approx(orc.s.u[i], rel=tol, abs=tol)
