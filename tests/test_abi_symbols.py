"""The C-ABI library loads without a GPU and exports every entry point the
public header declares; argument validation happens on the host."""
import ctypes as C
import os
import re

from spearhed_b200 import abi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "spearhed_b200.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(sph_\w+)\(", src, re.M)))


def test_header_declares_the_boundary():
    names = declared()
    for must in ("sph_create", "sph_destroy", "sph_set_species", "sph_get_species", "sph_density", "sph_hydro",
                 "sph_mhd", "sph_step", "sph_reduce", "sph_last_error_string", "sph_ensemble_reduce"):
        assert must in names


def test_library_exports_every_declared_symbol():
    L = abi.lib()
    for name in declared():
        assert hasattr(L, name), name


def test_default_params_and_host_validation():
    L = abi.lib()
    p = abi.SphParams()
    assert L.sph_default_params(C.byref(p)) == abi.SPH_OK
    assert p.kernel == abi.KERNEL_CUBIC and abs(p.gamma - 5 / 3) < 1e-15 and p.h0 == 0.05 and p.dt == 0.01
    ctx = C.c_void_p()
    bad = abi.default_params(kernel=7)
    assert L.sph_create(C.byref(bad), C.byref(ctx)) == abi.SPH_ERR_INVALID
    assert b"kernel" in L.sph_last_error_string()
    bad = abi.default_params(h0=-1.0)
    assert L.sph_create(C.byref(bad), C.byref(ctx)) == abi.SPH_ERR_INVALID
    bad = abi.default_params(physics=abi.PHYS_DEDNER)
    assert L.sph_create(C.byref(bad), C.byref(ctx)) == abi.SPH_ERR_INVALID
    assert L.sph_destroy(None) == abi.SPH_ERR_INVALID
    assert L.sph_step(None, 1, 0.0) == abi.SPH_ERR_INVALID
