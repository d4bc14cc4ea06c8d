"""The FP32 neighbour geometry against the oracle's, at the sizes where a
one-ulp difference in the cull's r^2 first showed.

The FP32 path culls on cell-relative FP32 positions: the FP64 position minus
its cell's lower corner (lo + c * edge, both unfused), rounded once to FP32.
A pair is accepted when the rounded, unfused x, y, z sum r^2 = dx^2 + dy^2 +
dz^2 is below R^2 (strict), as the reference evaluates it on the CPU.  On the
MHD rotor at 128^2 x 4 (84 k particles, two cell levels) and on the magnetised
Kelvin-Helmholtz lattice with 64 outer / 80 band layers (387 k, jittered),
some pairs sit at r^2 = R^2 to within one FP32 ulp, so a cull whose r^2 is
contracted into fused multiply-adds accepts or rejects them differently.

For both inputs, after one neighbour build (UpdateDensity):
  - the grid of each box (sphx_box_grid) has the oracle's cell counts and
    edges;
  - the FP32 pair records (sphx_get_pair_records) hold the oracle's FP32
    cell-relative positions and the FP32 masses, bit for bit;
  - every per-particle accepted-neighbour count equals the oracle's in FP32
    geometry, and the FP64 context's equal the oracle's in FP64 geometry.
"""
import ctypes as C

import numpy as np
import pytest

from spearhed_b200 import abi, setups

CASES = {
    "rotor128": lambda prec: setups.mhd_rotor(nxy=128, precision=prec),
    "kh64": lambda prec: setups.kelvin_helmholtz(n_outer=64, n_band=80, precision=prec),
}


@pytest.fixture(scope="module")
def oracle_geometry(oracle):
    cache = {}

    def get(name):
        if name not in cache:
            w = CASES[name](abi.PREC_FP64)
            s0 = w.species[abi.SPECIES_DEFAULT]
            po = oracle.System(w.params, w.boxes, s0.copy(), np.full(s0.n, abi.ROLES_DEFAULT, dtype=np.uint8))
            rel, edge, ncell = po.relpos()
            cache[name] = {"rel32": rel.astype(np.float32), "edge": edge, "ncell": ncell,
                           "mass32": s0.mass.astype(np.float32),
                           abi.PREC_FP32_COMP: po.neighbour_counts(True)[0],
                           abi.PREC_FP64: po.neighbour_counts(False)[0]}
        return cache[name]

    return get


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_fp32_records_and_grid_equal_the_oracle(oracle_geometry, name):
    import spearhed_b200 as sb
    ref = oracle_geometry(name)
    w = CASES[name](abi.PREC_FP32_COMP)
    n = w.species[abi.SPECIES_DEFAULT].n
    ctx = sb.context_for(w)
    ctx.density()
    L = abi.lib()
    grid = np.zeros(12)
    for b in range(len(w.boxes)):
        abi.check(L.sphx_box_grid(ctx._p, b, grid.ctypes.data_as(C.POINTER(C.c_double))))
        assert grid[0:3].astype(np.int32).tolist() == ref["ncell"][b].tolist()
        assert grid[3:6].tolist() == ref["edge"][b].tolist()
        assert grid[9] in (1.0, 2.0)
    pm = np.zeros(4 * n, dtype=np.float32)
    abi.check(L.sphx_get_pair_records(ctx._p, abi.SPECIES_DEFAULT, pm.ctypes.data_as(C.POINTER(C.c_float))))
    ctx.close()
    pm = pm.reshape(-1, 4)
    differ = int(np.count_nonzero(np.any(pm[:, :3] != ref["rel32"], axis=1)))
    assert differ == 0, f"{differ} FP32 cell-relative positions differ from the oracle's"
    assert np.array_equal(pm[:, 3], ref["mass32"])


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [abi.PREC_FP32_COMP, abi.PREC_FP64], ids=["fp32", "fp64"])
@pytest.mark.parametrize("name", list(CASES))
def test_borderline_pair_sets_equal_the_oracle(oracle_geometry, name, prec):
    import spearhed_b200 as sb
    ref = oracle_geometry(name)
    ctx = sb.context_for(CASES[name](prec))
    ctx.density()
    counts = ctx.neighbour_counts(abi.SPECIES_DEFAULT)
    ctx.close()
    bad = np.flatnonzero(counts != ref[prec])
    assert bad.size == 0, (bad.size, (counts[bad] - ref[prec][bad])[:10].tolist())


def test_geometry_hooks_refuse_a_null_context():
    # argument checks only, before any CUDA call
    L = abi.lib()
    pm = np.zeros(4, dtype=np.float32)
    rc = L.sphx_get_pair_records(None, 0, pm.ctypes.data_as(C.POINTER(C.c_float)))
    assert rc == abi.SPH_ERR_INVALID
    grid = np.zeros(12)
    assert L.sphx_box_grid(None, 0, grid.ctypes.data_as(C.POINTER(C.c_double))) == abi.SPH_ERR_INVALID
