"""spearhed_b200.validate on a small Orszag-Tang slab and a small MHD rotor: the FP32 run takes the
FP64 run's time steps, ends at the same simulated time, and stays within the
target bounds of it (density 1e-5 relative after one step grows slowly;
here 30 steps are held to 1e-4, and the energy drifts agree)."""
import pytest

from spearhed_b200 import setups, validate

pytestmark = pytest.mark.gpu


SMALL = {
    "small_ot": lambda prec: setups.orszag_tang(nx=32, nz=4, precision=prec, jitter=0.1),
    # two cell levels (10:1 disc), adaptive h, rotation
    "small_rotor": lambda prec: setups.mhd_rotor(nxy=64, nz=4, precision=prec),
}


@pytest.mark.parametrize("name", sorted(SMALL))
def test_fp32_follows_fp64_over_a_run(monkeypatch, name):
    monkeypatch.setitem(validate.WORKLOADS, name, SMALL[name])
    r = validate.run(name, 30)
    assert r["steps"] == 30 and r["time"] == r["time_fp32"] > 0
    assert r["density_rel_max"] <= 1e-4
    assert r["velocity_normwise"] <= 1e-3 and r["B_normwise"] <= 1e-3
    assert abs(r["energy_drift_difference"]) <= 0.02 * abs(r["energy_drift_fp64"]) + 1e-7
