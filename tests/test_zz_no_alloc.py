"""sph_density_noalloc: the density entry point for callers that cannot allocate.

Such callers (a framework that owns all device memory through its own pool,
code that runs where an allocation would synchronise the device, a plugin in
a program that forbids the CUDA allocator) pass their own device arrays in and
out; the library works in a fixed scratch array instead of calling cudaMalloc.

Checked here through the C ABI: two calls in a row, on different inputs, each
equal to what the context-based entry point (sph_density) computes and to the
CPU oracle, within the tolerances the other GPU tests use (FP64 rel 1e-12,
FP32 compensated rel 1e-5); a call beyond the fixed size limit is refused with
SPH_ERR_INVALID; bad inputs (a position outside a closed box, a NaN position,
h = 0, a negative mass) are refused with SPH_ERR_OUTSIDE / SPH_ERR_NONFINITE,
and the next valid call still matches sph_density (the scratch keeps nothing a
refused call left behind).
This file is collected last so a run that stops at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from spearhed_b200 import abi, setups

pytestmark = pytest.mark.gpu

TOL = {abi.PREC_FP64: 1e-12, abi.PREC_FP32_COMP: 1e-5}


def _noalloc():
    L = abi.lib()
    f = L.sph_density_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(abi.SphParams), C.POINTER(abi.SphBox), C.c_int64] + [C.c_void_p] * 6 + [C.c_void_p]
    return f


def _context_density(params, box, species):
    import spearhed_b200 as sb
    ctx = sb.Context(params, [box])
    ctx.set_species(abi.SPECIES_DEFAULT, species)
    ctx.density()
    rho = ctx.get_species(abi.SPECIES_DEFAULT).density
    ctx.close()
    return rho


def _noalloc_call(params, box, species):
    """(status, rho) of one call on device copies of the species' columns."""
    import torch
    dev = torch.device("cuda:0")
    cols = [torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
            for a in (species.pos[0], species.pos[1], species.pos[2], species.mass, species.h)]
    rho = torch.full((species.n,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = _noalloc()(C.byref(params), C.byref(box), species.n, *[c.data_ptr() for c in cols], rho.data_ptr(),
                    stream)
    return st, rho.cpu().numpy()


def _noalloc_density(params, box, species):
    st, rho = _noalloc_call(params, box, species)
    assert st == abi.SPH_OK, abi.lib().sph_last_error_string()
    return rho


def _oracle_density(oracle, params, box, species):
    s = species.copy()
    orc = oracle.System(params, [box], s, np.full(s.n, abi.ROLES_DEFAULT, dtype=np.uint8))
    orc.density()
    return orc.s.density


def _cloud(kernel, prec, n, seed):
    rng = np.random.default_rng(seed)
    s = abi.Species(n)
    s.pos[:] = rng.uniform(0.0, 1.0, size=(3, n))
    h0 = 0.07 if kernel != abi.KERNEL_QUINTIC else 0.05
    s.h[:] = h0
    s.mass[:] = rng.uniform(0.5, 1.5, n) * 1e-3
    p = abi.default_params(kernel=kernel, precision=prec, h0=h0)
    return p, abi.make_box((0, 0, 0), (1, 1, 1), (0, 1, 1)), s


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32_COMP])
def test_two_calls_in_a_row_match_the_context_entry_point(prec, oracle):
    # call 1: a random cloud, cubic spline, periodic in y and z
    p1, b1, s1 = _cloud(abi.KERNEL_CUBIC, prec, 3000, seed=21)
    # call 2: a different size and kernel (jittered Orszag-Tang slab, Wendland C2)
    w = setups.orszag_tang(nx=48, nz=4, precision=prec, jitter=0.1)
    p2, b2, s2 = w.params, w.boxes[0], w.species[abi.SPECIES_DEFAULT]
    got1 = _noalloc_density(p1, b1, s1)
    got2 = _noalloc_density(p2, b2, s2)
    ref1 = _context_density(p1, b1, s1)
    ref2 = _context_density(p2, b2, s2)
    assert np.max(np.abs(got1 / ref1 - 1.0)) <= TOL[prec]
    assert np.max(np.abs(got2 / ref2 - 1.0)) <= TOL[prec]
    # both calls against the CPU oracle (FP64 restatement of the reference's
    # DensityInitSelf + AccumulateDensity over the exact neighbour set)
    p1o, p2o = abi.SphParams.from_buffer_copy(p1), abi.SphParams.from_buffer_copy(p2)
    p1o.precision = p2o.precision = abi.PREC_FP64
    orc1 = _oracle_density(oracle, p1o, b1, s1)
    orc2 = _oracle_density(oracle, p2o, b2, s2)
    assert np.max(np.abs(got1 / orc1 - 1.0)) <= TOL[prec]
    assert np.max(np.abs(got2 / orc2 - 1.0)) <= TOL[prec]
    # and the first input again, after the scratch held the second call's data
    again = _noalloc_density(p1, b1, s1)
    assert np.max(np.abs(again / ref1 - 1.0)) <= TOL[prec]


@pytest.mark.parametrize("case,status", [
    ("outside_closed_axis", abi.SPH_ERR_OUTSIDE),
    ("nan_position", abi.SPH_ERR_NONFINITE),
    ("zero_h", abi.SPH_ERR_NONFINITE),
    ("negative_mass", abi.SPH_ERR_NONFINITE),
])
def test_bad_inputs_are_refused_and_the_next_call_is_clean(case, status):
    p, b, s = _cloud(abi.KERNEL_CUBIC, abi.PREC_FP64, 2000, seed=33)
    bad = s.copy()
    if case == "outside_closed_axis":
        bad.pos[0, 17] = 1.25  # x is not periodic in this box
    elif case == "nan_position":
        bad.pos[1, 5] = float("nan")
    elif case == "zero_h":
        bad.h[9] = 0.0
    else:
        bad.mass[3] = -1e-3
    st, _ = _noalloc_call(p, b, bad)
    assert st == status, abi.lib().sph_last_error_string()
    got = _noalloc_density(p, b, s)
    ref = _context_density(p, b, s)
    assert np.max(np.abs(got / ref - 1.0)) <= TOL[abi.PREC_FP64]


def test_size_beyond_the_fixed_scratch_is_refused():
    import torch
    n = (1 << 18) + 1
    p = abi.default_params(h0=0.05)
    box = abi.make_box((0, 0, 0), (1, 1, 1))
    buf = torch.zeros(n, dtype=torch.float64, device="cuda:0")
    st = _noalloc()(C.byref(p), C.byref(box), n, *([buf.data_ptr()] * 6), 0)
    assert st == abi.SPH_ERR_INVALID
    assert b"scratch limit" in abi.lib().sph_last_error_string()
