"""ctypes wrapper of the CPU oracle — TEST INFRASTRUCTURE ONLY.

Loads oracle/_build/liboracle.so (the FP64/FP32 restatement in oracle.cpp) and,
when present, oracle/_ref/libspearhed_ref.so (the reference's own physics
headers compiled by ``make ref``).  Only tests/, the smoke check and bench.py's
CPU-baseline leg may import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from spearhed_b200.abi import SphBox, SphDiag, SphParams, SphSoAView

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libspearhed_ref.so")

_ORC = None
_REF = None


def build(ref: bool = True, ref_root: str | None = None):
    """Compile the oracle, and the reference harness when a reference checkout
    is given (``ref_root`` or the REF_ROOT environment variable) and exists;
    without one the harness is left as it is (prebuilt, or absent)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    root = ref_root or os.environ.get("REF_ROOT")
    if ref and root and os.path.isdir(root):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_ROOT={root}"], check=True)


def _stale() -> bool:
    """The library is missing or older than a source it is built from."""
    if not os.path.exists(ORACLE_SO):
        return True
    built = os.path.getmtime(ORACLE_SO)
    srcs = [os.path.join(HERE, "oracle.cpp"), os.path.join(HERE, "Makefile"),
            os.path.join(os.path.dirname(HERE), "include", "spearhed_b200.h")]
    return any(os.path.exists(f) and os.path.getmtime(f) > built for f in srcs)


def orc():
    global _ORC
    if _ORC is None:
        if _stale():
            build(ref=False)
        L = C.CDLL(ORACLE_SO)
        P = C.POINTER
        common = [P(SphParams), C.c_int32, P(SphBox), C.c_int64, P(C.c_uint8), P(SphSoAView)]
        L.orc_kernel_W.restype = C.c_double
        L.orc_kernel_W.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double]
        L.orc_kernel_dWdr.restype = C.c_double
        L.orc_kernel_dWdr.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double]
        L.orc_kernel_gradWScalar.restype = C.c_double
        L.orc_kernel_gradWScalar.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]
        L.orc_pressure.restype = C.c_double
        L.orc_pressure.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double]
        L.orc_sound_speed.restype = C.c_double
        L.orc_sound_speed.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double]
        L.orc_neighbour_counts.restype = C.c_int
        L.orc_neighbour_counts.argtypes = common + [C.c_int32, P(C.c_int32), P(C.c_double)]
        L.orc_neighbour_list.restype = C.c_int
        L.orc_neighbour_list.argtypes = common + [C.c_int32, C.c_int64, C.c_int32, P(C.c_int64), P(C.c_int8), P(C.c_int32)]
        L.orc_neighbour_csr.restype = C.c_int
        L.orc_neighbour_csr.argtypes = common + [C.c_int32, C.c_int64, P(C.c_int64), P(C.c_int64), P(C.c_int8),
                                                 P(C.c_int64)]
        L.orc_relpos.restype = C.c_int
        L.orc_relpos.argtypes = common + [P(C.c_double), P(C.c_double), P(C.c_int32)]
        L.orc_density.restype = C.c_int
        L.orc_density.argtypes = common + [C.c_int32]
        L.orc_force.restype = C.c_int
        L.orc_force.argtypes = common + [C.c_int32, P(C.c_double), P(C.c_double)]
        L.orc_reduce.restype = C.c_int
        L.orc_reduce.argtypes = common + [P(SphDiag)]
        L.orc_step.restype = C.c_int
        L.orc_step.argtypes = common + [C.c_int32, C.c_int32, P(C.c_double), P(C.c_double), P(SphDiag)]
        _ORC = L
    return _ORC


def ref():
    """The reference-compiled harness, or None when it was not built."""
    global _REF
    if _REF is None and os.path.exists(REF_SO):
        L = C.CDLL(REF_SO)
        for suf, T in (("f32", C.c_float), ("f64", C.c_double)):
            for name in ("ref_cubic_W", "ref_cubic_dWdr", "ref_quintic_W", "ref_quintic_dWdr"):
                f = getattr(L, f"{name}_{suf}")
                f.restype = T
                f.argtypes = [T, T]
            for name in ("ref_cubic_gradWScalar", "ref_quintic_gradWScalar"):
                f = getattr(L, f"{name}_{suf}")
                f.restype = T
                f.argtypes = [T, T, T]
            f = getattr(L, f"ref_pressure_{suf}")
            f.restype = T
            f.argtypes = [T, T, T]
            f = getattr(L, f"ref_sound_speed_{suf}")
            f.restype = T
            f.argtypes = [T, T, T]
            TP = C.POINTER(T)
            f = getattr(L, f"ref_density_{suf}")
            f.restype = None
            f.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), TP, TP, TP, C.POINTER(C.c_int64),
                          C.POINTER(C.c_int), TP, T, TP]
            f = getattr(L, f"ref_region_bench_{suf}")
            f.restype = C.c_int
            f.argtypes = [C.c_int, C.c_int, TP, TP, TP, TP, TP, TP, TP, TP, T, T, T, C.c_double,
                          C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int), C.POINTER(C.c_int),
                          C.POINTER(C.c_double)]
            f = getattr(L, f"ref_hydro_{suf}")
            f.restype = None
            f.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), TP, TP, TP, TP, TP, TP, C.POINTER(C.c_int64),
                          C.POINTER(C.c_int), TP, T, T, TP, TP]
        _REF = L
    return _REF


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class System:
    """Particles of all species in one set of FP64 arrays, plus their roles."""

    def __init__(self, params: SphParams, boxes, species, roles):
        self.params = params
        self.boxes = (SphBox * len(boxes))(*boxes)
        self.nbox = len(boxes)
        self.s = species
        self.roles = np.ascontiguousarray(roles, dtype=np.uint8)
        self.view = species.view()

    def _common(self):
        return (C.byref(self.params), self.nbox, self.boxes, self.s.n,
                _ptr(self.roles, C.c_uint8), C.byref(self.view))

    def neighbour_counts(self, fp32_geometry=False):
        counts = np.zeros(self.s.n, dtype=np.int32)
        pairs = C.c_double(0)
        st = orc().orc_neighbour_counts(*self._common(), int(fp32_geometry), _ptr(counts, C.c_int32), C.byref(pairs))
        _check(st)
        return counts, pairs.value

    def neighbour_list(self, i, fp32_geometry=False, cap=4096):
        js = np.zeros(cap, dtype=np.int64)
        offs = np.zeros(3 * cap, dtype=np.int8)
        cnt = C.c_int32(0)
        _check(orc().orc_neighbour_list(*self._common(), int(fp32_geometry), int(i), cap, _ptr(js, C.c_int64),
                                         _ptr(offs, C.c_int8), C.byref(cnt)))
        k = min(cnt.value, cap)
        return js[:k], offs[:3 * k].reshape(k, 3)

    def neighbour_csr(self, fp32_geometry=False):
        """(off[n+1], js, offs[k,3]) of every target's accepted neighbours."""
        off = np.zeros(self.s.n + 1, dtype=np.int64)
        total = C.c_int64(0)
        cap = 0
        js = np.zeros(1, dtype=np.int64)
        offs = np.zeros(3, dtype=np.int8)
        st = orc().orc_neighbour_csr(*self._common(), int(fp32_geometry), cap, _ptr(off, C.c_int64),
                                     _ptr(js, C.c_int64), _ptr(offs, C.c_int8), C.byref(total))
        if st not in (0, 6):
            _check(st)
        cap = max(total.value, 1)
        js = np.zeros(cap, dtype=np.int64)
        offs = np.zeros(3 * cap, dtype=np.int8)
        _check(orc().orc_neighbour_csr(*self._common(), int(fp32_geometry), cap, _ptr(off, C.c_int64),
                                       _ptr(js, C.c_int64), _ptr(offs, C.c_int8), C.byref(total)))
        return off, js[:total.value], offs[:3 * total.value].reshape(-1, 3)

    def relpos(self):
        """Cell-relative FP64 positions (n,3), cell edges (nbox,3), cell counts (nbox,3)."""
        rel = np.zeros(3 * self.s.n, dtype=np.float64)
        edge = np.zeros(3 * self.nbox, dtype=np.float64)
        ncell = np.zeros(3 * self.nbox, dtype=np.int32)
        _check(orc().orc_relpos(*self._common(), _ptr(rel, C.c_double), _ptr(edge, C.c_double),
                                _ptr(ncell, C.c_int32)))
        return rel.reshape(-1, 3), edge.reshape(-1, 3), ncell.reshape(-1, 3)

    def density(self, fp32_geometry=False):
        _check(orc().orc_density(*self._common(), int(fp32_geometry)))

    def force(self, fp32_geometry=False):
        """Runs the force pass; returns (c_h, CFL minimum) — per box for an ensemble."""
        ch = np.zeros(self.nbox)
        dtm = np.zeros(self.nbox)
        _check(orc().orc_force(*self._common(), int(fp32_geometry), _ptr(ch, C.c_double), _ptr(dtm, C.c_double)))
        if self.nbox == 1:
            return float(ch[0]), float(dtm[0])
        return ch, dtm

    def reduce(self):
        d = SphDiag()
        _check(orc().orc_reduce(*self._common(), C.byref(d)))
        return d

    def step(self, n_steps, dt_state, time=0.0, fp32_geometry=False):
        """n_steps of the full step; dt_state and time are per box (scalars for one box)."""
        dts = np.ascontiguousarray(np.broadcast_to(np.asarray(dt_state, dtype=np.float64), (self.nbox,)))
        t = np.ascontiguousarray(np.broadcast_to(np.asarray(time, dtype=np.float64), (self.nbox,)))
        d = SphDiag()
        _check(orc().orc_step(*self._common(), int(fp32_geometry), int(n_steps), _ptr(dts, C.c_double),
                              _ptr(t, C.c_double), C.byref(d)))
        if self.nbox == 1:
            return float(dts[0]), float(t[0]), d
        return dts, t, d


def _check(st):
    if st != 0:
        raise RuntimeError(f"oracle error {st}")


def region_bench(species, params, box_lo, box_hi, side, limit_s=20.0, dtype=np.float32):
    """Time the reference's density + hydro functors (compiled from its sources)
    under its region/frame engine on the host cores: regions of edge `side`,
    64-slot frames, cubic spline with the radius 2*h0 of `params`.  Target
    frames run in order until `limit_s` has passed.  Returns a cpu_baseline dict."""
    L = ref()
    T = C.c_float if dtype == np.float32 else C.c_double
    suf = "f32" if dtype == np.float32 else "f64"
    n = species.n

    def arr(a):
        return np.ascontiguousarray(a, dtype=dtype)
    pos = arr(species.pos.T.ravel())
    vel = arr(species.vel.T.ravel())
    mass, h, u = arr(species.mass), arr(species.h), arr(species.u)
    rho = arr(species.density).copy()
    lo, hi = arr(box_lo), arr(box_hi)
    P = lambda a: a.ctypes.data_as(C.POINTER(T))  # noqa: E731
    pd, ph = C.c_int64(0), C.c_int64(0)
    fd, ft = C.c_int(0), C.c_int(0)
    sec = C.c_double(0)
    st = getattr(L, f"ref_region_bench_{suf}")(
        0, n, P(pos), P(mass), P(h), P(rho), P(u), P(vel), P(lo), P(hi), side, 2.0 * params.h0, params.gamma,
        limit_s, C.byref(pd), C.byref(ph), C.byref(fd), C.byref(ft), C.byref(sec))
    _check(st)
    value = (pd.value + ph.value) / sec.value
    return {"value": value, "unit": "pair-interactions/s", "kind": "reference",
            "pairs_density": pd.value, "pairs_hydro": ph.value, "seconds": sec.value,
            "frames": [fd.value, ft.value],
            "sample": (f"{fd.value} of {ft.value} target frames of the {n}-particle input: the reference's own "
                       "DensityInitSelf/AccumulateDensity and HydroInteraction functors (compiled from its "
                       "headers, FP32) under its region/frame engine (64-slot frames, AABB region search), "
                       "cubic spline at the same 2h radius, no periodic images (the reference has none); "
                       "2 pair passes (density, hydro)")}
