"""spearhed_b200 — B200-native SPH(-MHD) step behind spearHED's species/functor interface.

Python host API over the C ABI (include/spearhed_b200.h).  The compute path is
the CUDA library spearhed_b200/_lib/libspearhed_b200.so; there is no CPU
fallback (:func:`spearhed_b200.abi.lib` raises when the library is missing).

The stage-functor names mirror the reference's call sites
(include/spearhed/particles/density/DensitySummation.hpp:104-138,
include/spearhed/sph/HydroForces.hpp:183-214, control/Simulation.x.cpp:196-310):

    ctx = Context(params, boxes)
    ctx.set_species(SPECIES_DEFAULT, species)
    UpdateDensity(ctx)          # density summation (self term + gather)
    UpdateHydroForces(ctx)      # pressure force + P dV (+ viscosity / MHD per params)
    ctx.step(n)                 # runOneStep x n: drift, density, forces, kick
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .abi import (  # noqa: F401  (re-exported names)
    CULL_GLOBAL, CULL_PAIR_MAX, KERNEL_CUBIC, KERNEL_QUINTIC, KERNEL_WENDLAND_C2, PHYS_ADAPTIVE_H, PHYS_AV, PHYS_CFL,
    PHYS_DEDNER, PHYS_MHD, PHYS_TENSILE, PREC_FP32_COMP, PREC_FP64, ROLES_BOUNDARY, ROLES_DEFAULT,
    ROLES_TRACER, SPECIES_BOUNDARY, SPECIES_DEFAULT, SPECIES_ROLES, SPECIES_TRACER, SphBox, SphDiag,
    SphError, SphParams, Species, default_params, make_box,
)


class Context:
    """One simulation context (one CUDA stream, library-owned device memory)."""

    def __init__(self, params: SphParams, boxes=None):
        L = abi.lib()
        self._L = L
        self._p = C.c_void_p()
        self.params = params
        abi.check(L.sph_create(C.byref(params), C.byref(self._p)))
        self.nbox = 0
        if boxes:
            self.set_boxes(boxes)
        self._n = {}

    def set_boxes(self, boxes):
        arr = (SphBox * len(boxes))(*boxes)
        abi.check(self._L.sph_set_boxes(self._p, len(boxes), arr))
        self.nbox = len(boxes)

    def set_species(self, sid: int, species: Species, roles: int | None = None):
        roles = abi.SPECIES_ROLES[sid] if roles is None else roles
        v = species.view()
        abi.check(self._L.sph_set_species(self._p, sid, roles, species.n, C.byref(v)))
        self._n[sid] = species.n

    def get_species(self, sid: int) -> Species:
        s = Species(self._n[sid])
        v = s.view()
        abi.check(self._L.sph_get_species(self._p, sid, C.byref(v)))
        return s

    def density(self):
        abi.check(self._L.sph_density(self._p))

    def hydro(self):
        abi.check(self._L.sph_hydro(self._p))

    def mhd(self):
        abi.check(self._L.sph_mhd(self._p))

    def step(self, n_steps: int = 1, dt: float = 0.0):
        abi.check(self._L.sph_step(self._p, int(n_steps), float(dt)))

    def reduce(self) -> dict:
        d = SphDiag()
        abi.check(self._L.sph_reduce(self._p, C.byref(d)))
        return d.as_dict()

    def ensemble_reduce(self, nbox: int) -> list:
        arr = (SphDiag * nbox)()
        abi.check(self._L.sph_ensemble_reduce(self._p, nbox, arr))
        return [a.as_dict() for a in arr]

    def neighbour_counts(self, sid: int) -> np.ndarray:
        out = np.zeros(self._n[sid], dtype=np.int32)
        abi.check(self._L.sph_get_neighbour_counts(self._p, sid, out.ctypes.data_as(C.POINTER(C.c_int32))))
        return out

    def timings(self) -> list:
        ms = (C.c_double * 5)()
        abi.check(self._L.sph_get_timings(self._p, 5, ms))
        return list(ms)

    def clock(self):
        """(time, dt_next) per box."""
        n = max(self.nbox, 1)
        t = np.zeros(n)
        d = np.zeros(n)
        P = C.POINTER(C.c_double)
        abi.check(self._L.sph_get_clock(self._p, n, t.ctypes.data_as(P), d.ctypes.data_as(P)))
        return t, d

    def set_clock(self, time, dt_next):
        n = max(self.nbox, 1)
        t = np.ascontiguousarray(np.broadcast_to(np.asarray(time, dtype=np.float64), (n,)))
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt_next, dtype=np.float64), (n,)))
        P = C.POINTER(C.c_double)
        abi.check(self._L.sph_set_clock(self._p, n, t.ctypes.data_as(P), d.ctypes.data_as(P)))

    def set_wait_timeout(self, seconds: float):
        """Bound the wait of the compute calls (0 = no limit); see sph_set_wait_timeout."""
        abi.check(self._L.sph_set_wait_timeout(self._p, float(seconds)))

    def wait(self):
        """Complete a call that returned SPH_ERR_TIMEOUT (sph_wait)."""
        abi.check(self._L.sph_wait(self._p))

    def use_graph(self, on: bool = True):
        abi.check(self._L.sph_use_graph(self._p, int(bool(on))))

    def prepare_graph(self):
        """Capture the graph the next step call replays, from a snapshot that is
        then restored (no simulated time passes)."""
        abi.check(self._L.sph_prepare_graph(self._p))

    def init_lattice(self, species_id: int, init, roles: int | None = None) -> int:
        """Generates a species on the device from a setups.LatticeInit (lattice
        blocks + profile) and sets it; returns its particle count."""
        blocks, nb, prof = init.to_abi()
        n = C.c_int64(0)
        r = abi.SPECIES_ROLES[species_id] if roles is None else roles
        abi.check(self._L.sph_init_lattice(self._p, int(species_id), int(r), int(nb), blocks, C.byref(prof),
                                           C.byref(n)))
        self._n[species_id] = int(n.value)
        return int(n.value)

    def autotune(self, steps_per_trial: int = 2) -> dict:
        """Times every launch shape of the pair kernels on the current particles
        (the state is restored after each trial) and keeps the fastest."""
        t = abi.SphTuning()
        abi.check(self._L.sph_autotune(self._p, int(steps_per_trial), C.byref(t)))
        return t.as_dict()

    def set_tuning(self, density_variant: int, force_variant: int):
        abi.check(self._L.sph_set_tuning(self._p, int(density_variant), int(force_variant)))

    def tuning(self) -> dict:
        t = abi.SphTuning()
        abi.check(self._L.sph_get_tuning(self._p, C.byref(t)))
        return t.as_dict()

    def close(self):
        if self._p:
            abi.check(self._L.sph_destroy(self._p))
            self._p = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- reference-shaped stage functors -------------------------------------
def UpdateDensity(ctx: Context):
    """UpdateDensity<K>{}(bundle, target, index, h0) (DensitySummation.hpp:104-138)."""
    ctx.density()


def UpdateHydroForces(ctx: Context):
    """UpdateHydroForces<K>{gamma}(bundle, target, index, h0) (HydroForces.hpp:183-214)."""
    ctx.hydro()


def run_one_step(ctx: Context, n_steps: int = 1, dt: float = 0.0):
    """Simulation::runOneStep (control/Simulation.x.cpp:196-310), n_steps times."""
    ctx.step(n_steps, dt)


def context_for(workload, device_init: bool = False) -> Context:
    """A context holding every species of a :class:`spearhed_b200.setups.Workload`;
    with ``device_init`` the species are generated on the device from the
    workload's lattice blocks (sph_init_lattice) instead of copied from the host."""
    ctx = Context(workload.params, workload.boxes)
    for sid, s in workload.species.items():
        if device_init and sid in workload.init:
            ctx.init_lattice(sid, workload.init[sid])
        else:
            ctx.set_species(sid, s)
    return ctx
