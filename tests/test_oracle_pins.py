"""Pins the CPU oracle to the reference.

1. Bit-for-bit against the reference's own physics headers, compiled from the
   reference checkout by oracle/Makefile (`make ref`): kernel functions
   (CubicSplineKernel.hpp, QuinticSplineKernel.hpp), EOS (EquationOfState.hpp),
   and the density / hydro pair functors (DensitySummation.hpp, HydroForces.hpp)
   driven over the oracle's own neighbour lists.
2. The reference's known-answer tests, restated on the oracle:
   tests/spearhed/unit/Kernels/Kernels.cpp:73-130,
   tests/spearhed/unit/DensitySummation/DensitySummation.cpp:230-345,
   tests/spearhed/unit/HydroForces/HydroForces.cpp:159-239.
"""
import ctypes as C
import math

import numpy as np
import pytest

from spearhed_b200 import abi

CUBIC, QUINTIC, WENDLAND = abi.KERNEL_CUBIC, abi.KERNEL_QUINTIC, abi.KERNEL_WENDLAND_C2


def _f32(x):
    return float(np.float32(x))


@pytest.mark.parametrize("kernel,name", [(CUBIC, "cubic"), (QUINTIC, "quintic")])
@pytest.mark.parametrize("prec,suf", [(0, "f64"), (1, "f32")])
def test_kernel_functions_bitwise_equal_reference(oracle, reflib, kernel, name, prec, suf):
    o = oracle.orc()
    W = getattr(reflib, f"ref_{name}_W_{suf}")
    dW = getattr(reflib, f"ref_{name}_dWdr_{suf}")
    gW = getattr(reflib, f"ref_{name}_gradWScalar_{suf}")
    sup = 3 if kernel == QUINTIC else 2
    rng = np.random.default_rng(7)
    for h in (0.05, 0.0078125, 0.5, 1.0, 0.009375, 1.0 / 30.0):
        rs = np.concatenate([np.linspace(0.0, 1.1 * sup * h, 401), rng.uniform(0, 1.05 * sup * h, 200),
                             [h, 2 * h, sup * h, sup * h * (1 - 1e-7)]])
        for r in rs:
            if prec:
                r, hh = _f32(r), _f32(h)
                inv = _f32(1.0 / r) if r > 0 else 0.0
            else:
                hh = h
                inv = 1.0 / r if r > 0 else 0.0
            assert o.orc_kernel_W(kernel, prec, r, hh) == W(r, hh), (r, hh)
            assert o.orc_kernel_dWdr(kernel, prec, r, hh) == dW(r, hh), (r, hh)
            assert o.orc_kernel_gradWScalar(kernel, prec, r, inv, hh) == gW(r, inv, hh), (r, hh)


@pytest.mark.parametrize("prec,suf", [(0, "f64"), (1, "f32")])
def test_eos_bitwise_equal_reference(oracle, reflib, prec, suf):
    o = oracle.orc()
    P = getattr(reflib, f"ref_pressure_{suf}")
    cs = getattr(reflib, f"ref_sound_speed_{suf}")
    rng = np.random.default_rng(3)
    for _ in range(500):
        g, rho, u = rng.choice([1.4, 5 / 3, 2.0]), rng.uniform(0.01, 10), rng.uniform(0.01, 10)
        if prec:
            g, rho, u = _f32(g), _f32(rho), _f32(u)
        p = o.orc_pressure(prec, g, rho, u)
        assert p == P(g, rho, u)
        assert o.orc_sound_speed(prec, g, p, rho) == cs(g, p, rho)


# ---- Kernels.cpp:73-130 --------------------------------------------------
@pytest.mark.parametrize("kernel", [CUBIC, QUINTIC, WENDLAND])
def test_kernel_zero_outside_support(oracle, kernel):
    o = oracle.orc()
    h = 0.5
    sup = 3 if kernel == QUINTIC else 2
    for prec in (0, 1):
        assert abs(o.orc_kernel_W(kernel, prec, sup * h, h)) <= 1e-7
        assert abs(o.orc_kernel_W(kernel, prec, sup * h + 0.1, h)) <= 1e-7
        assert o.orc_kernel_W(kernel, prec, 0.0, h) > 0.0


@pytest.mark.parametrize("kernel", [CUBIC, QUINTIC, WENDLAND])
def test_kernel_gradient_antisymmetric(oracle, kernel):
    o = oracle.orc()
    h = 0.5
    rv = np.array([0.4, -0.3, 0.2], dtype=np.float32)
    r = float(np.float32(math.sqrt(0.4 * 0.4 + 0.3 * 0.3 + 0.2 * 0.2)))
    s = o.orc_kernel_gradWScalar(kernel, 1, r, 1.0 / r, h)
    gp = s * rv
    gn = s * (-rv)
    assert np.allclose(gp, -gn, atol=1e-6)
    assert s < 0.0  # kernels decrease outward


@pytest.mark.parametrize("kernel", [CUBIC, QUINTIC, WENDLAND])
def test_kernel_radial_integral_is_one(oracle, kernel):
    """3D normalisation: 4 pi int W r^2 dr = 1 within 1% (Real = float evaluation)."""
    o = oracle.orc()
    h = 0.5
    sup = 3 if kernel == QUINTIC else 2
    n = 10000
    dr = sup * h / n
    acc = 0.0
    for i in range(n):
        r = (i + 0.5) * dr
        acc += o.orc_kernel_W(kernel, 1, r, h) * 4.0 * math.pi * r * r * dr
    assert acc == pytest.approx(1.0, rel=1e-2)


# ---- DensitySummation.cpp / HydroForces.cpp known answers --------------
def _system(oracle, pos, mass, h, rho, u, vel=None, h0=None, kernel=CUBIC, gamma=5 / 3, box=None):
    n = pos.shape[1]
    s = abi.Species(n)
    s.pos[:] = pos
    s.mass[:] = mass
    s.h[:] = h
    s.density[:] = rho
    s.u[:] = u
    if vel is not None:
        s.vel[:] = vel
    p = abi.default_params(kernel=kernel, precision=abi.PREC_FP64, cull=abi.CULL_GLOBAL, physics=0,
                           gamma=gamma, h0=h0 if h0 is not None else float(np.max(h)))
    box = box or abi.make_box((-5, -5, -5), (5, 5, 5))
    roles = np.full(n, abi.ROLES_DEFAULT, dtype=np.uint8)
    return oracle.System(p, [box], s, roles)


def test_density_colocated(oracle):
    """N = 4 co-located particles: rho = N m W(0, h) (DensitySummation.cpp:265-276)."""
    o = oracle.orc()
    n, h, m = 4, 0.5, 1.0
    sysm = _system(oracle, np.zeros((3, n)), m, h, 0.0, 0.0)
    sysm.density()
    expected = n * m * o.orc_kernel_W(CUBIC, 1, 0.0, h)
    assert np.allclose(sysm.s.density, expected, rtol=1e-5)


def test_density_three_in_a_line(oracle):
    """Particles at x = 0, 1.5, 3 with h = 1, m = 1.5 (DensitySummation.cpp:316-343)."""
    o = oracle.orc()
    dx, h, m = 1.5, 1.0, 1.5
    pos = np.zeros((3, 3))
    pos[0] = [0.0, dx, 2 * dx]
    sysm = _system(oracle, pos, m, h, 0.0, 0.0)
    sysm.density()
    w0 = o.orc_kernel_W(CUBIC, 1, 0.0, h)
    w1 = o.orc_kernel_W(CUBIC, 1, dx, h)
    edge, mid = m * (w0 + w1), m * (w0 + 2 * w1)
    rho = sysm.s.density
    assert rho[0] == pytest.approx(edge, rel=1e-5)
    assert rho[2] == pytest.approx(edge, rel=1e-5)
    assert rho[1] == pytest.approx(mid, rel=1e-5)


def test_hydro_two_particles_at_rest(oracle):
    """d = 0.4, h = 0.5, rho = u = m = 1: dvdt_x = -+ 2 m P/rho^2 dWdr(d, h), dudt = 0
    (HydroForces.cpp:205-232)."""
    o = oracle.orc()
    d, h = 0.4, 0.5
    pos = np.zeros((3, 2))
    pos[0] = [-d / 2, d / 2]
    sysm = _system(oracle, pos, 1.0, h, 1.0, 1.0)
    sysm.force()
    P = o.orc_pressure(0, 5 / 3, 1.0, 1.0)
    expected_left = 1.0 * 2 * P * o.orc_kernel_dWdr(CUBIC, 1, d, h)
    dv = sysm.s.dvdt
    assert dv[0, 0] == pytest.approx(expected_left, rel=1e-4)
    assert dv[0, 1] == pytest.approx(-expected_left, rel=1e-4)
    assert np.allclose(dv[1:], 0.0, atol=1e-6)
    assert np.allclose(sysm.s.dudt, 0.0, atol=1e-6)


def test_position_outside_a_periodic_axis_is_refused(oracle):
    """The cell search covers [lo, hi] on every axis: a particle outside it is
    SPH_ERR_OUTSIDE on periodic axes too, while x = hi is accepted."""
    rng = np.random.default_rng(2)
    pos = rng.uniform(0.0, 1.0, size=(3, 200))
    box = abi.make_box((0, 0, 0), (1, 1, 1), (1, 1, 1))
    pos[0, 3] = 1.0
    _system(oracle, pos, 1e-3, 0.08, 0.0, 1.0, box=box).density()
    pos[0, 3] = 1.5
    with pytest.raises(RuntimeError, match=f"oracle error {abi.SPH_ERR_OUTSIDE}"):
        _system(oracle, pos, 1e-3, 0.08, 0.0, 1.0, box=box).density()


# ---- the oracle's FP64 passes are the reference functors, bit for bit ----
def _random_cloud(oracle, kernel, n=1500, seed=11, periodic=(0, 1, 0)):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, 1.0, size=(3, n))
    h = 0.08 if kernel != QUINTIC else 0.055
    sysm = _system(oracle, pos, rng.uniform(0.5, 1.5, n) * 1e-3, h, 0.0, rng.uniform(0.5, 2.0, n),
                   vel=rng.normal(size=(3, n)), h0=h, kernel=kernel,
                   box=abi.make_box((0, 0, 0), (1, 1, 1), periodic))
    return sysm


@pytest.mark.parametrize("kernel", [CUBIC, QUINTIC])
def test_density_and_hydro_bitwise_equal_reference_functors(oracle, reflib, kernel):
    sysm = _random_cloud(oracle, kernel)
    n = sysm.s.n
    sysm.density()
    sysm.force()
    off, js, offs = sysm.neighbour_csr()
    rel, edge, _ = sysm.relpos()
    # The reference harness receives the oracle's own candidate lists plus the
    # self pair (its functors skip isSelf), with the stencil shift of each entry.
    cand_off = np.zeros(n + 1, dtype=np.int64)
    cand, shifts = [], []
    for i in range(n):
        cand.append(np.concatenate([[i], js[off[i]:off[i + 1]]]))
        shifts.append(np.concatenate([np.zeros((1, 3)), offs[off[i]:off[i + 1]] * edge[0]]))
        cand_off[i + 1] = cand_off[i] + len(cand[-1])
    cand = np.ascontiguousarray(np.concatenate(cand).astype(np.int32))
    shifts = np.ascontiguousarray(np.concatenate(shifts).ravel())
    targets = np.arange(n, dtype=np.int32)
    relf = np.ascontiguousarray(rel.ravel())
    D = C.POINTER(C.c_double)

    def p(a, t=D):
        return a.ctypes.data_as(t)

    R = (3 if kernel == QUINTIC else 2) * sysm.params.h0
    rho = np.zeros(n)
    reflib.ref_density_f64(kernel, n, p(targets, C.POINTER(C.c_int)), p(relf), p(sysm.s.mass), p(sysm.s.h),
                           p(cand_off, C.POINTER(C.c_int64)), p(cand, C.POINTER(C.c_int)), p(shifts), R, p(rho))
    assert np.array_equal(rho, sysm.s.density)
    vel = np.ascontiguousarray(sysm.s.vel.T.ravel())
    dv = np.zeros(3 * n)
    du = np.zeros(n)
    reflib.ref_hydro_f64(kernel, n, p(targets, C.POINTER(C.c_int)), p(relf), p(sysm.s.mass), p(sysm.s.h),
                         p(sysm.s.density), p(sysm.s.u), p(vel), p(cand_off, C.POINTER(C.c_int64)),
                         p(cand, C.POINTER(C.c_int)), p(shifts), sysm.params.gamma, R, p(dv), p(du))
    assert np.array_equal(dv.reshape(n, 3).T, sysm.s.dvdt)
    assert np.array_equal(du, sysm.s.dudt)


def test_neighbour_counts_match_brute_force(oracle):
    """Cell-stencil neighbour sets equal an O(N^2) minimum-image enumeration."""
    sysm = _random_cloud(oracle, CUBIC, n=800, periodic=(1, 1, 0))
    counts, pairs = sysm.neighbour_counts()
    pos = sysm.s.pos.T
    d = pos[:, None, :] - pos[None, :, :]
    for a, per in enumerate((1, 1, 0)):
        if per:
            d[..., a] -= np.round(d[..., a])
    r2 = (d ** 2).sum(-1)
    R = 2 * sysm.params.h0
    np.fill_diagonal(r2, np.inf)
    brute = (r2 < R * R).sum(1)
    assert np.array_equal(counts, brute)
    assert pairs == brute.sum()
