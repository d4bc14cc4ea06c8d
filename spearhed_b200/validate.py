"""FP32-compensated against FP64-plain over a whole run of one workload.

    python -m spearhed_b200.validate --workload orszag_tang --steps 200

The FP64 run steps with its CFL time step, one step per call, and records each
dt; the FP32 run then takes exactly those steps (CFL off, dt given), so both
reach the same simulated times.  Printed as one JSON object:

* the relative drift of the total energy (kinetic + internal + magnetic) of
  each run and their difference;
* after the last step, the FP32 run's largest and median relative density
  error and its normwise velocity, internal-energy and B errors against FP64;
* both runs' mean and largest |div B| h / |B|.

Single-box workloads only (an ensemble's boxes each have their own dt).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import abi, context_for, setups

WORKLOADS = {
    "orszag_tang": lambda prec: setups.orszag_tang(precision=prec),
    "kelvin_helmholtz": lambda prec: setups.kelvin_helmholtz(precision=prec),
    "mhd_rotor": lambda prec: setups.mhd_rotor(precision=prec),
    "sod_small": lambda prec: setups.sod_small(precision=prec),
}


def _energy(d):
    return d["e_kin"] + d["e_int"] + d["e_mag"]


def _normwise(got, ref):
    scale = float(np.max(np.abs(ref)))
    return float(np.max(np.abs(got - ref)) / scale) if scale > 0 else 0.0


def run(workload: str, steps: int) -> dict:
    w64 = WORKLOADS[workload](abi.PREC_FP64)
    c64 = context_for(w64)
    e0 = _energy(c64.reduce())
    dts = []
    t0 = time.perf_counter()
    for _ in range(steps):
        c64.step(1)
        dts.append(c64.reduce()["dt"])
    t64 = time.perf_counter() - t0
    d64 = c64.reduce()
    s64 = c64.get_species(abi.SPECIES_DEFAULT)
    c64.close()

    w32 = WORKLOADS[workload](abi.PREC_FP32_COMP)
    w32.params.physics &= ~abi.PHYS_CFL
    c32 = context_for(w32)
    e0_32 = _energy(c32.reduce())
    t0 = time.perf_counter()
    for dt in dts:
        c32.step(1, dt)
    t32 = time.perf_counter() - t0
    d32 = c32.reduce()
    s32 = c32.get_species(abi.SPECIES_DEFAULT)
    c32.close()

    rel_rho = np.abs(s32.density / s64.density - 1.0)
    drift64 = (_energy(d64) - e0) / e0
    drift32 = (_energy(d32) - e0_32) / e0_32
    return {
        "workload": workload, "particles": int(s64.n), "steps": steps,
        "time": d64["time"], "time_fp32": d32["time"],
        "energy_drift_fp64": drift64, "energy_drift_fp32": drift32,
        "energy_drift_difference": drift32 - drift64,
        "density_rel_max": float(rel_rho.max()), "density_rel_median": float(np.median(rel_rho)),
        "velocity_normwise": _normwise(s32.vel, s64.vel),
        "u_normwise": _normwise(s32.u, s64.u),
        "B_normwise": _normwise(s32.B, s64.B),
        "divb_mean_fp64": d64["divb_mean"], "divb_max_fp64": d64["divb_max"],
        "divb_mean_fp32": d32["divb_mean"], "divb_max_fp32": d32["divb_max"],
        "wall_s_fp64": t64, "wall_s_fp32": t32,
    }


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--workload", default="orszag_tang", choices=sorted(WORKLOADS))
    ap.add_argument("--steps", type=int, default=200)
    a = ap.parse_args(argv)
    print(json.dumps(run(a.workload, a.steps)), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
