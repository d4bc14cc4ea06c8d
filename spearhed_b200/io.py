"""Particle snapshots and checkpoints: raw binary columns + a JSON header.

Snapshot layout.  The record names follow the reference's openPMD particle
output (include/spearhed/plugins/openPMD/OpenPMDOutput.hpp:53-160;
validate_sod.py reads position/x, velocity/x, mass_density and
specific_internal_energy).  HDF5 and openPMD-api are not available, so the
records are stored as one little-endian binary file per snapshot with a JSON
header naming every record, its offset, dtype and shape:

    <path>.json   {"format": "spearhed_b200.snapshot/1", "step", "time", "dt", "species": {...}}
    <path>.bin    the columns, back to back, 8-byte aligned

A checkpoint is a snapshot of every species plus what a restart needs: the
per-box clock (time, next dt), the boxes and the run parameters.  Restoring
it into a new context and continuing gives the same run up to the
summation order inside cells (the restored particles start in input order).
"""
from __future__ import annotations

import dataclasses
import json
import os

import numpy as np

from . import abi

FORMAT = "spearhed_b200.snapshot/1"

# record name -> (Species column, component or None)
RECORDS = [
    ("position/x", "pos", 0), ("position/y", "pos", 1), ("position/z", "pos", 2),
    ("velocity/x", "vel", 0), ("velocity/y", "vel", 1), ("velocity/z", "vel", 2),
    ("mass", "mass", None), ("mass_density", "density", None),
    ("specific_internal_energy", "u", None), ("smoothing_length", "h", None),
    ("magnetic_field/x", "B", 0), ("magnetic_field/y", "B", 1), ("magnetic_field/z", "B", 2),
    ("divergence_cleaning_psi", "psi", None),
]
SPECIES_NAMES = {abi.SPECIES_DEFAULT: "Default", abi.SPECIES_BOUNDARY: "Boundary", abi.SPECIES_TRACER: "Tracer"}


def write_snapshot(path, species: dict, step=0, time=0.0, dt=0.0, extra=None):
    """Write every species (id -> abi.Species) to <path>.bin / <path>.json."""
    header = {"format": FORMAT, "step": int(step), "time": float(time), "dt": float(dt), "species": {},
              "extra": extra or {}}
    off = 0
    with open(path + ".bin", "wb") as f:
        for sid, s in sorted(species.items()):
            recs = {}
            for name, col, comp in RECORDS:
                a = getattr(s, col)
                a = a[comp] if comp is not None else a
                buf = np.ascontiguousarray(a, dtype="<f8").tobytes()
                f.write(buf)
                recs[name] = {"offset": off, "dtype": "<f8", "shape": [s.n]}
                off += len(buf)
            ids = np.arange(s.n, dtype="<i8").tobytes()
            f.write(ids)
            recs["id"] = {"offset": off, "dtype": "<i8", "shape": [s.n]}
            off += len(ids)
            boxes = np.ascontiguousarray(s.box_id, dtype="<i4").tobytes()
            f.write(boxes)
            f.write(b"\0" * ((8 - len(boxes) % 8) % 8))
            recs["box_id"] = {"offset": off, "dtype": "<i4", "shape": [s.n]}
            off += len(boxes) + (8 - len(boxes) % 8) % 8
            header["species"][SPECIES_NAMES[sid]] = {"species_id": sid, "n": s.n, "records": recs}
    with open(path + ".json", "w") as f:
        json.dump(header, f, indent=1)
    return header


def read_snapshot(path):
    """(species dict id -> abi.Species, header) of a snapshot written by write_snapshot."""
    with open(path + ".json") as f:
        header = json.load(f)
    if header.get("format") != FORMAT:
        raise ValueError(f"{path}.json is not a {FORMAT} snapshot")
    raw = np.fromfile(path + ".bin", dtype=np.uint8)
    out = {}
    for info in header["species"].values():
        s = abi.Species(info["n"])
        recs = info["records"]

        def rec(name):
            r = recs[name]
            n = int(np.prod(r["shape"]))
            return np.frombuffer(raw, dtype=r["dtype"], count=n, offset=r["offset"])

        for name, col, comp in RECORDS:
            if comp is None:
                setattr(s, col, rec(name).astype(np.float64).copy())
            else:
                getattr(s, col)[comp] = rec(name)
        s.box_id = rec("box_id").astype(np.int32).copy()
        out[info["species_id"]] = s
    return out, header


def _params_dict(p: abi.SphParams):
    return {name: getattr(p, name) for name, _ in p._fields_}


def _params_from(d):
    return abi.SphParams(**{k: v for k, v in d.items() if k in dict(abi.SphParams._fields_)})


def _box_dict(b: abi.SphBox):
    return {"lo": list(b.lo), "hi": list(b.hi), "periodic": list(b.periodic)}


def save_checkpoint(ctx, path, boxes):
    """Snapshot of every species of `ctx` plus its clock, boxes and parameters."""
    species = {sid: ctx.get_species(sid) for sid in sorted(ctx._n)}
    t, dt = ctx.clock()
    d = ctx.reduce()
    extra = {"params": _params_dict(ctx.params), "boxes": [_box_dict(b) for b in boxes],
             "clock_time": t.tolist(), "clock_dt": dt.tolist(), "steps": int(d["steps"])}
    return write_snapshot(path, species, step=d["steps"], time=float(t[0]), dt=float(dt[0]), extra=extra)


@dataclasses.dataclass
class Checkpoint:
    params: abi.SphParams
    boxes: list
    species: dict
    time: np.ndarray
    dt: np.ndarray
    steps: int


def load_checkpoint(path) -> Checkpoint:
    species, header = read_snapshot(path)
    x = header["extra"]
    boxes = [abi.make_box(b["lo"], b["hi"], b["periodic"]) for b in x["boxes"]]
    return Checkpoint(_params_from(x["params"]), boxes, species, np.array(x["clock_time"]),
                      np.array(x["clock_dt"]), int(x["steps"]))


def resume(path):
    """A new context holding the checkpoint's particles and clock."""
    import spearhed_b200 as sb
    ck = load_checkpoint(path)
    ctx = sb.Context(ck.params, ck.boxes)
    for sid, s in ck.species.items():
        ctx.set_species(sid, s)
    ctx.set_clock(ck.time, ck.dt)
    return ctx, ck


# ---------------------------------------------------------------- diagnostics
DIAG_FORMAT = "spearhed_b200.diagnostics/1"


class DiagnosticsLog:
    """Per-step diagnostics as JSON lines (one object per record() call).

    Each line holds the step count and simulated time, the dt of the last step
    and the next one, the conserved quantities of sph_reduce (kinetic, internal,
    magnetic and total energy, momentum, <|div B| h/|B|> and its maximum, the
    Dedner speed), the accepted pairs of the last pass and the device time of
    the last call per stage (sph_get_timings: sort+permute, density, force,
    integrate+reduce, whole call).  The first line is a header with the format
    name.  The reference logs progress to stdout only
    (pmacc/simulationControl/SimulationHelper.cpp:89-108)."""

    STAGES = ("sort_permute_ms", "density_ms", "force_ms", "kick_reduce_ms", "call_ms")

    def __init__(self, path, meta=None):
        self.path = path
        self._f = open(path, "w")
        self._f.write(json.dumps({"format": DIAG_FORMAT, **(meta or {})}) + "\n")
        self._f.flush()

    def record(self, ctx, extra=None):
        d = ctx.reduce()
        tm = ctx.timings()
        row = {"step": int(d["steps"]), "time": d["time"], "dt": d["dt"], "dt_next": d["dt_next"],
               "e_kin": d["e_kin"], "e_int": d["e_int"], "e_mag": d["e_mag"],
               "e_tot": d["e_kin"] + d["e_int"] + d["e_mag"], "mom": list(d["mom"]),
               "divb_mean": d["divb_mean"], "divb_max": d["divb_max"], "c_h": d["c_h"],
               "pairs": d["pairs"], "replays": int(d["replays"])}
        row.update({k: float(v) for k, v in zip(self.STAGES, tm)})
        if extra:
            row.update(extra)
        self._f.write(json.dumps(row) + "\n")
        self._f.flush()
        return row

    def close(self):
        if self._f:
            self._f.close()
            self._f = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def run_logged(ctx, n_steps, path, every=1, dt=0.0, meta=None):
    """Steps `ctx` n_steps times, `every` steps per call, and logs one
    diagnostics line per call to `path` (JSON lines).  Returns the rows."""
    rows = []
    with DiagnosticsLog(path, meta) as log:
        done = 0
        while done < n_steps:
            k = min(every, n_steps - done)
            ctx.step(k, dt)
            done += k
            rows.append(log.record(ctx))
    return rows


def read_diagnostics(path):
    """(header, rows) of a diagnostics log."""
    with open(path) as f:
        lines = [json.loads(x) for x in f if x.strip()]
    if not lines or lines[0].get("format") != DIAG_FORMAT:
        raise ValueError(f"{path}: not a {DIAG_FORMAT} log")
    return lines[0], lines[1:]
