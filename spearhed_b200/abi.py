"""ctypes mirror of include/spearhed_b200.h and the loader for the CUDA library.

The library is ``spearhed_b200/_lib/libspearhed_b200.so`` built in-tree by
``spearhed_b200.build``.  There is no CPU fallback: if the shared library is
missing or fails to load, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# SPEARHED_B200_VARIANT=check loads the bounds-checked build (device index
# checks that report SPH_ERR_STATE instead of reading out of range)
VARIANT = os.environ.get("SPEARHED_B200_VARIANT", "")
LIB_PATH = os.path.join(HERE, "_lib", "libspearhed_b200_check.so" if VARIANT == "check" else "libspearhed_b200.so")

# status codes
SPH_OK = 0
SPH_ERR_INVALID = 1
SPH_ERR_CUDA = 2
SPH_ERR_NOMEM = 3
SPH_ERR_OUTSIDE = 4
SPH_ERR_NONFINITE = 5
SPH_ERR_OVERFLOW = 6
SPH_ERR_STATE = 7
SPH_ERR_TIMEOUT = 8
SPH_ERR_UNSUPPORTED = 9

KERNEL_CUBIC, KERNEL_QUINTIC, KERNEL_WENDLAND_C2 = 0, 1, 2
PHYS_AV, PHYS_MHD, PHYS_DEDNER, PHYS_TENSILE, PHYS_CFL, PHYS_ADAPTIVE_H = 1, 2, 4, 8, 16, 32
PREC_FP64, PREC_FP32_COMP = 0, 1
CULL_GLOBAL, CULL_PAIR_MAX = 0, 1
SPECIES_DEFAULT, SPECIES_BOUNDARY, SPECIES_TRACER = 0, 1, 2
ROLE_MOVABLE, ROLE_SOURCE, ROLE_THERMODYNAMIC, ROLE_FROZEN, ROLE_INTERIOR = 1, 2, 4, 8, 16
ROLES_DEFAULT = ROLE_INTERIOR | ROLE_MOVABLE | ROLE_SOURCE | ROLE_THERMODYNAMIC
ROLES_BOUNDARY = ROLE_FROZEN | ROLE_SOURCE | ROLE_THERMODYNAMIC
ROLES_TRACER = ROLE_MOVABLE
SPECIES_ROLES = {SPECIES_DEFAULT: ROLES_DEFAULT, SPECIES_BOUNDARY: ROLES_BOUNDARY, SPECIES_TRACER: ROLES_TRACER}

_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int32)


class SphParams(C.Structure):
    _fields_ = [
        ("kernel", C.c_int32),
        ("precision", C.c_int32),
        ("cull", C.c_int32),
        ("physics", C.c_uint32),
        ("gamma", C.c_double),
        ("h0", C.c_double),
        ("dt", C.c_double),
        ("alpha", C.c_double),
        ("beta", C.c_double),
        ("av_eps", C.c_double),
        ("cfl", C.c_double),
        ("cfl_force", C.c_double),
        ("dedner_sigma", C.c_double),
        ("mu0", C.c_double),
        ("max_neighbours", C.c_int32),
        ("device", C.c_int32),
        ("hfact", C.c_double),
        ("h_max", C.c_double),
    ]


class SphBox(C.Structure):
    _fields_ = [("lo", C.c_double * 3), ("hi", C.c_double * 3), ("periodic", C.c_int32 * 3)]


class SphSoAView(C.Structure):
    _fields_ = [
        ("pos", _DP * 3),
        ("vel", _DP * 3),
        ("mass", _DP),
        ("h", _DP),
        ("density", _DP),
        ("u", _DP),
        ("dvdt", _DP * 3),
        ("dudt", _DP),
        ("B", _DP * 3),
        ("psi", _DP),
        ("dBdt", _DP * 3),
        ("dpsidt", _DP),
        ("divB", _DP),
        ("box_id", _IP),
    ]


class SphDiag(C.Structure):
    _fields_ = [
        ("time", C.c_double),
        ("dt", C.c_double),
        ("dt_next", C.c_double),
        ("e_kin", C.c_double),
        ("e_int", C.c_double),
        ("e_mag", C.c_double),
        ("mom", C.c_double * 3),
        ("divb_mean", C.c_double),
        ("divb_max", C.c_double),
        ("c_h", C.c_double),
        ("pairs", C.c_double),
        ("steps", C.c_int64),
        ("n_targets", C.c_int64),
        ("pairs_total", C.c_double),
        ("candidates", C.c_double),
        ("replays", C.c_int64),
        ("list_capacity", C.c_int64),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "mom"}
        d["mom"] = [self.mom[0], self.mom[1], self.mom[2]]
        return d


def default_params(**kw) -> SphParams:
    """Library defaults (the reference's param files), overridden by keyword."""
    p = SphParams(
        kernel=KERNEL_CUBIC, precision=PREC_FP32_COMP, cull=CULL_GLOBAL, physics=0,
        gamma=5.0 / 3.0, h0=0.05, dt=0.01, alpha=1.0, beta=2.0, av_eps=0.01, cfl=0.3,
        cfl_force=0.25, dedner_sigma=1.0, mu0=1.0, max_neighbours=0, device=0, hfact=1.2, h_max=0.0,
    )
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def make_box(lo, hi, periodic=(0, 0, 0)) -> SphBox:
    b = SphBox()
    for a in range(3):
        b.lo[a] = float(lo[a])
        b.hi[a] = float(hi[a])
        b.periodic[a] = int(bool(periodic[a]))
    return b


COLUMNS = ("pos", "vel", "mass", "h", "density", "u", "dvdt", "dudt", "B", "psi", "dBdt", "dpsidt", "divB")
VECTOR_COLUMNS = ("pos", "vel", "dvdt", "B", "dBdt")


class Species:
    """Host SoA of one species: FP64 numpy columns named after the reference's tags.

    Vector attributes are (3, n) arrays.  ``view()`` returns the SphSoAView that
    points into these arrays (the arrays must outlive the view's use).
    """

    def __init__(self, n: int):
        self.n = int(n)
        for c in COLUMNS:
            shape = (3, self.n) if c in VECTOR_COLUMNS else (self.n,)
            setattr(self, c, np.zeros(shape, dtype=np.float64))
        self.box_id = np.zeros(self.n, dtype=np.int32)

    def copy(self) -> "Species":
        s = Species(self.n)
        for c in COLUMNS:
            setattr(s, c, getattr(self, c).copy())
        s.box_id = self.box_id.copy()
        return s

    def view(self) -> SphSoAView:
        v = SphSoAView()
        for c in COLUMNS:
            arr = getattr(self, c)
            assert arr.dtype == np.float64 and arr.flags.c_contiguous
            if c in VECTOR_COLUMNS:
                ptrs = getattr(v, c)
                for a in range(3):
                    ptrs[a] = arr[a].ctypes.data_as(_DP)
            else:
                setattr(v, c, arr.ctypes.data_as(_DP))
        v.box_id = self.box_id.ctypes.data_as(_IP)
        return v

    @staticmethod
    def concat(parts):
        n = sum(p.n for p in parts)
        out = Species(n)
        for c in COLUMNS:
            arrs = [getattr(p, c) for p in parts]
            setattr(out, c, np.ascontiguousarray(np.concatenate(arrs, axis=-1)))
        out.box_id = np.ascontiguousarray(np.concatenate([p.box_id for p in parts]))
        return out


MASK_NONE, MASK_INSIDE_DISC_XY, MASK_OUTSIDE_DISC_XY = 0, 1, 2
PROFILE_CONSTANT, PROFILE_ORSZAG_TANG, PROFILE_KH_PERTURBATION, PROFILE_ROTOR = 0, 1, 2, 3


class SphLatticeBlock(C.Structure):
    _fields_ = [
        ("lo", C.c_double * 3),
        ("hi", C.c_double * 3),
        ("counts", C.c_int32 * 3),
        ("mask", C.c_int32),
        ("spacing", C.c_double),
        ("mask_centre", C.c_double * 2),
        ("mask_radius", C.c_double),
        ("box_id", C.c_int32),
        ("jitter_group", C.c_int32),
        ("jitter", C.c_double),
        ("seed", C.c_uint64),
        ("mass", C.c_double),
        ("h", C.c_double),
        ("density", C.c_double),
        ("u", C.c_double),
        ("psi", C.c_double),
        ("vel", C.c_double * 3),
        ("B", C.c_double * 3),
    ]


class SphInitProfile(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("wrap", C.c_int32 * 3),
        ("wrap_lo", C.c_double * 3),
        ("wrap_hi", C.c_double * 3),
        ("p", C.c_double * 8),
    ]


class SphTuning(C.Structure):
    _fields_ = [
        ("density_variant", C.c_int32),
        ("force_variant", C.c_int32),
        ("staging_depth", C.c_int32),
        ("density_blocks_per_sm", C.c_int32),
        ("force_blocks_per_sm", C.c_int32),
        ("n_density_variants", C.c_int32),
        ("n_force_variants", C.c_int32),
        ("steps_per_trial", C.c_int32),
        ("density_ms", C.c_double * 8),
        ("force_ms", C.c_double * 8),
        ("cull_unroll", C.c_int32),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if not k.endswith("_ms")}
        d["density_ms"] = [self.density_ms[i] for i in range(self.n_density_variants)]
        d["force_ms"] = [self.force_ms[i] for i in range(self.n_force_variants)]
        return d


_LIB = None


def lib():
    """Load the CUDA library; raise if it is absent (there is no fallback)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"spearhed_b200 CUDA library not built: {LIB_PATH} is missing "
            "(run `python -m spearhed_b200.build`)")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    ctx_p = C.c_void_p
    sig = {
        "sph_default_params": (C.c_int, [P(SphParams)]),
        "sph_create": (C.c_int, [P(SphParams), P(ctx_p)]),
        "sph_destroy": (C.c_int, [ctx_p]),
        "sph_set_boxes": (C.c_int, [ctx_p, C.c_int32, P(SphBox)]),
        "sph_set_species": (C.c_int, [ctx_p, C.c_int32, C.c_uint32, C.c_int64, P(SphSoAView)]),
        "sph_get_species": (C.c_int, [ctx_p, C.c_int32, P(SphSoAView)]),
        "sph_density": (C.c_int, [ctx_p]),
        "sph_hydro": (C.c_int, [ctx_p]),
        "sph_mhd": (C.c_int, [ctx_p]),
        "sph_step": (C.c_int, [ctx_p, C.c_int32, C.c_double]),
        "sph_reduce": (C.c_int, [ctx_p, P(SphDiag)]),
        "sph_ensemble_reduce": (C.c_int, [ctx_p, C.c_int32, P(SphDiag)]),
        "sph_get_neighbour_counts": (C.c_int, [ctx_p, C.c_int32, P(C.c_int32)]),
        "sph_get_timings": (C.c_int, [ctx_p, C.c_int32, P(C.c_double)]),
        "sph_use_graph": (C.c_int, [ctx_p, C.c_int32]),
        "sph_prepare_graph": (C.c_int, [ctx_p]),
        "sph_get_clock": (C.c_int, [ctx_p, C.c_int32, P(C.c_double), P(C.c_double)]),
        "sph_set_clock": (C.c_int, [ctx_p, C.c_int32, P(C.c_double), P(C.c_double)]),
        "sph_autotune": (C.c_int, [ctx_p, C.c_int32, P(SphTuning)]),
        "sph_init_lattice": (C.c_int, [ctx_p, C.c_int32, C.c_uint32, C.c_int32, P(SphLatticeBlock),
                                       P(SphInitProfile), P(C.c_int64)]),
        "sph_sc_cell_counts": (C.c_int, [P(C.c_double), P(C.c_double), C.c_double, P(C.c_uint32)]),
        "sph_sc_cell_counts_f32": (C.c_int, [P(C.c_float), P(C.c_float), C.c_float, P(C.c_uint32)]),
        "sph_set_tuning": (C.c_int, [ctx_p, C.c_int32, C.c_int32]),
        "sph_get_tuning": (C.c_int, [ctx_p, P(SphTuning)]),
        "sph_last_error_string": (C.c_char_p, []),
        "sph_set_wait_timeout": (C.c_int, [ctx_p, C.c_double]),
        "sph_wait": (C.c_int, [ctx_p]),
        "sph_density_noalloc": (C.c_int, [P(SphParams), P(SphBox), C.c_int64] + [C.c_void_p] * 7),
        "sphx_fail_alloc_after": (C.c_longlong, [C.c_longlong]),
        "sphx_box_grid": (C.c_int, [ctx_p, C.c_int32, P(C.c_double)]),
        "sphx_get_pair_records": (C.c_int, [ctx_p, C.c_int32, P(C.c_float)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _LIB = L
    return L


class SphError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"spearhed_b200 error {code}: {msg}")
        self.code = code


def check(code: int):
    if code != SPH_OK:
        msg = lib().sph_last_error_string()
        raise SphError(code, msg.decode() if msg else "")
    return code
