"""Host-side initial conditions for the benchmark and test workloads.

These play the part of the reference's setup blocks (SetupInterface +
InitParticles + the SC lattice: include/spearhed/particles/initialization/
InitParticles.hpp:284-433, spmacc/particles/initialization/SC.hpp:118-200,
share/spearhed/ValidationSetups/SodShockTube.hpp:128-176): they place particles
on simple-cubic lattices at cell centres, with equal masses, u = P/((gamma-1) rho).
Jitter, where a workload asks for it, comes from numpy's Philox4x32-10
counter-based generator keyed by the workload's seed.

Each generator returns a :class:`Workload`.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import abi


@dataclasses.dataclass
class Workload:
    name: str
    params: abi.SphParams
    boxes: list
    species: dict  # species id -> abi.Species
    steps: int = 1
    meta: dict = dataclasses.field(default_factory=dict)

    @property
    def n(self):
        return sum(s.n for s in self.species.values())

    def combined(self):
        """All species concatenated (Default, Boundary, Tracer order) with their roles."""
        parts, roles = [], []
        for sid in sorted(self.species):
            s = self.species[sid]
            parts.append(s)
            roles.append(np.full(s.n, abi.SPECIES_ROLES[sid], dtype=np.uint8))
        return abi.Species.concat(parts), np.concatenate(roles)

    def split(self, combined):
        """Inverse of :meth:`combined` for a state array set of the same layout."""
        out, off = {}, 0
        for sid in sorted(self.species):
            n = self.species[sid].n
            s = abi.Species(n)
            for c in abi.COLUMNS:
                setattr(s, c, np.ascontiguousarray(getattr(combined, c)[..., off:off + n]))
            s.box_id = np.ascontiguousarray(combined.box_id[off:off + n])
            out[sid] = s
            off += n
        return out


def lattice(lo, hi, counts):
    """Simple-cubic lattice at cell centres of the box lo..hi (SC.hpp:118-200)."""
    axes = [lo[a] + (np.arange(counts[a]) + 0.5) * (hi[a] - lo[a]) / counts[a] for a in range(3)]
    z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel()])


def philox_uniform(seed, shape):
    return np.random.Generator(np.random.Philox(key=seed)).uniform(-1.0, 1.0, size=shape)


def sod_small(precision=abi.PREC_FP32_COMP, scale=1, reference_physics=False, hfact=1.2):
    """3D Sod shock tube, gamma 1.4, periodic in y and z.

    Left x in [-0.5, 0): rho 1, P 1 on a (64 s)x(16 s)x(16 s) lattice; right
    x in [0, 0.5): rho 0.125, P 0.1 on (32 s)x(8 s)x(8 s); s = ``scale`` (1 gives
    N = 18432).  Equal masses; h = 1.2 x local spacing (56 lattice neighbours);
    cubic spline; artificial viscosity alpha 1, beta 2; CFL 0.3.  x is open: the
    box extends 0.25 beyond each end.  ``scale`` < 1 is allowed as a fraction
    (e.g. 0.5 halves every lattice count).
    """
    gamma = 1.4
    nl = (int(64 * scale), int(16 * scale), int(16 * scale))
    nr = (int(32 * scale), int(8 * scale), int(8 * scale))
    Ly = 0.125
    left = lattice((-0.5, 0.0, 0.0), (0.0, Ly, Ly), nl)
    right = lattice((0.0, 0.0, 0.0), (0.5, Ly, Ly), nr)
    dxl, dxr = 0.5 / nl[0], 0.5 / nr[0]
    m = 1.0 * dxl ** 3
    n = left.shape[1] + right.shape[1]
    s = abi.Species(n)
    s.pos[:] = np.concatenate([left, right], axis=1)
    s.mass[:] = m
    s.h[:] = np.concatenate([np.full(left.shape[1], hfact * dxl), np.full(right.shape[1], hfact * dxr)])
    rho = np.concatenate([np.full(left.shape[1], 1.0), np.full(right.shape[1], 0.125)])
    P = np.concatenate([np.full(left.shape[1], 1.0), np.full(right.shape[1], 0.1)])
    s.density[:] = rho
    s.u[:] = P / ((gamma - 1.0) * rho)
    physics = 0 if reference_physics else (abi.PHYS_AV | abi.PHYS_CFL | abi.PHYS_ADAPTIVE_H)
    params = abi.default_params(kernel=abi.KERNEL_CUBIC, precision=precision, cull=abi.CULL_PAIR_MAX,
                                physics=physics, gamma=gamma, h0=hfact * dxr, dt=1e-4, alpha=1.0, beta=2.0,
                                cfl=0.3, hfact=hfact, h_max=1.5 * hfact * dxr)
    box = abi.make_box((-0.75, 0.0, 0.0), (0.75, Ly, Ly), (0, 1, 1))
    return Workload("sod_small", params, [box], {abi.SPECIES_DEFAULT: s}, steps=50,
                    meta={"n_left": left.shape[1], "n_right": right.shape[1], "dx_left": dxl, "dx_right": dxr})


def orszag_tang(nx=512, nz=4, precision=abi.PREC_FP32_COMP, hfact=1.45, jitter=0.0, seed=2):
    """Orszag-Tang vortex in a thin periodic slab [0,1]^2 x [0, nz/nx].

    nx x nx x nz lattice of equal-mass particles; rho = 25/(36 pi), P = 5/(12 pi),
    gamma = 5/3, v = (-sin 2 pi y, sin 2 pi x, 0), B = (-sin 2 pi y, sin 4 pi x, 0)/sqrt(4 pi).
    Wendland C2 with h = hfact x spacing (hfact 1.45: 92 lattice neighbours,
    ~102 in the continuum), AV, SPMHD with Dedner cleaning and the tensile
    correction, CFL time step.  nx = 512, nz = 4 gives N = 1,048,576.
    ``jitter`` > 0 displaces every particle uniformly by up to jitter x spacing
    per axis (Philox, key ``seed``); the benchmark workload uses none.
    """
    gamma = 5.0 / 3.0
    dx = 1.0 / nx
    Lz = nz * dx
    pos = lattice((0.0, 0.0, 0.0), (1.0, 1.0, Lz), (nx, nx, nz))
    if jitter > 0.0:
        pos = pos + jitter * dx * philox_uniform(seed, pos.shape)
        pos[0] %= 1.0
        pos[1] %= 1.0
        pos[2] %= Lz
    n = pos.shape[1]
    s = abi.Species(n)
    s.pos[:] = pos
    rho0 = 25.0 / (36.0 * math.pi)
    P0 = 5.0 / (12.0 * math.pi)
    s.mass[:] = rho0 * dx ** 3
    s.h[:] = hfact * dx
    s.density[:] = rho0
    s.u[:] = P0 / ((gamma - 1.0) * rho0)
    x, y = pos[0], pos[1]
    s.vel[0] = -np.sin(2 * math.pi * y)
    s.vel[1] = np.sin(2 * math.pi * x)
    b0 = 1.0 / math.sqrt(4 * math.pi)
    s.B[0] = -b0 * np.sin(2 * math.pi * y)
    s.B[1] = b0 * np.sin(4 * math.pi * x)
    physics = abi.PHYS_AV | abi.PHYS_MHD | abi.PHYS_DEDNER | abi.PHYS_TENSILE | abi.PHYS_CFL
    params = abi.default_params(kernel=abi.KERNEL_WENDLAND_C2, precision=precision, cull=abi.CULL_GLOBAL,
                                physics=physics, gamma=gamma, h0=hfact * dx, dt=2e-4, alpha=1.0, beta=2.0,
                                cfl=0.3, dedner_sigma=1.0)
    box = abi.make_box((0.0, 0.0, 0.0), (1.0, 1.0, Lz), (1, 1, 1))
    return Workload("orszag_tang", params, [box], {abi.SPECIES_DEFAULT: s}, steps=200,
                    meta={"nx": nx, "nz": nz, "dx": dx})


def brio_wu_box(n_target=8192, precision=abi.PREC_FP32_COMP, nt=8, box_id=0):
    """One 3D Brio-Wu MHD shock tube (gamma 2, Bx 0.75).

    Left x in [-0.5, 0): rho 1, P 1, By +1; right x in [0, 0.5): rho 0.125, P 0.1,
    By -1.  Equal masses: the right lattice spacing is twice the left.  The tube
    is nt left lattice layers thick in y and z (periodic); its length is chosen
    so the box holds about n_target particles.  x is open (the box extends 0.25
    beyond each end).  Cubic spline, AV, SPMHD with Dedner cleaning and the
    tensile correction, adaptive h (hfact 1.2), CFL 0.3.
    """
    gamma = 2.0
    nxl = max(8, int(round(n_target / (nt * nt * 1.125))))
    nxl += nxl % 2
    dxl = 0.5 / nxl
    L = nt * dxl
    left = lattice((-0.5, 0.0, 0.0), (0.0, L, L), (nxl, nt, nt))
    right = lattice((0.0, 0.0, 0.0), (0.5, L, L), (nxl // 2, nt // 2, nt // 2))
    n = left.shape[1] + right.shape[1]
    s = abi.Species(n)
    s.pos[:] = np.concatenate([left, right], axis=1)
    m = dxl ** 3
    s.mass[:] = m
    isl = np.concatenate([np.ones(left.shape[1], bool), np.zeros(right.shape[1], bool)])
    rho = np.where(isl, 1.0, 0.125)
    P = np.where(isl, 1.0, 0.1)
    s.density[:] = rho
    s.u[:] = P / ((gamma - 1.0) * rho)
    s.h[:] = np.where(isl, 1.2 * dxl, 2.4 * dxl)
    s.B[0] = 0.75
    s.B[1] = np.where(isl, 1.0, -1.0)
    s.box_id[:] = box_id
    physics = (abi.PHYS_AV | abi.PHYS_MHD | abi.PHYS_DEDNER | abi.PHYS_TENSILE | abi.PHYS_CFL
               | abi.PHYS_ADAPTIVE_H)
    params = abi.default_params(kernel=abi.KERNEL_CUBIC, precision=precision, cull=abi.CULL_PAIR_MAX,
                                physics=physics, gamma=gamma, h0=2.4 * dxl, dt=1e-5, alpha=1.0, beta=2.0,
                                cfl=0.3, hfact=1.2, h_max=3.6 * dxl)
    box = abi.make_box((-0.75, 0.0, 0.0), (0.75, L, L), (0, 1, 1))
    return params, box, s


def brio_wu_ensemble(nbox=512, precision=abi.PREC_FP32_COMP, seed=5, n_lo=4096, n_hi=262144):
    """An ensemble of independent Brio-Wu tubes with particle counts drawn
    log-uniform in [n_lo, n_hi] (numpy Philox, key ``seed``).  With the default
    512 boxes this is about 31 M particles.  Every box keeps its own time step.
    The ensemble-wide h_max is the largest box's (it sets no cell size: each box
    has its own grid from its own h)."""
    rng = np.random.Generator(np.random.Philox(key=seed))
    sizes = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), size=nbox)).astype(int)
    boxes, parts, params = [], [], None
    hmax = 0.0
    for b, nb in enumerate(sizes):
        p, box, s = brio_wu_box(int(nb), precision=precision, box_id=b)
        boxes.append(box)
        parts.append(s)
        hmax = max(hmax, p.h_max)
        params = p
    species = abi.Species.concat(parts)
    # boxes differ in resolution; h_max = 0 lets each box size its grid from its own
    # largest h (x1.5 under adaptive h)
    params.h_max = 0.0
    return Workload("brio_wu_ensemble", params, boxes, {abi.SPECIES_DEFAULT: species}, steps=100,
                    meta={"sizes": sizes.tolist(), "seed": seed})


def kelvin_helmholtz(n_outer=224, n_band=282, precision=abi.PREC_FP32_COMP, hfact=1.45, seed=3):
    """Magnetised Kelvin-Helmholtz in the periodic unit cube.

    Band |y - 0.5| < 0.25: rho 2, vx +0.5; outside: rho 1, vx -0.5.  Each region
    is a lattice whose spacing follows its density (n_band/n_outer ~ 2^(1/3);
    n_outer = 224, n_band = 282 give 5.62 M + 11.21 M = 16.8 M particles, masses
    within 0.5% of each other).  Uniform jitter of 0.05 spacing (Philox, key
    ``seed``), vy = 0.01 sin(4 pi x), P = 2.5, gamma 5/3, Bx = 0.1.  Wendland C2,
    h = hfact x local spacing (adaptive), AV, SPMHD with Dedner cleaning, CFL.
    """
    gamma = 5.0 / 3.0
    if n_outer % 4 or n_band % 2:
        raise ValueError("n_outer must be a multiple of 4 and n_band even (whole layers per slab)")
    lo1 = lattice((0.0, 0.0, 0.0), (1.0, 0.25, 1.0), (n_outer, n_outer // 4, n_outer))
    lo2 = lattice((0.0, 0.75, 0.0), (1.0, 1.0, 1.0), (n_outer, n_outer // 4, n_outer))
    band = lattice((0.0, 0.25, 0.0), (1.0, 0.75, 1.0), (n_band, n_band // 2, n_band))
    d_o, d_b = 1.0 / n_outer, 1.0 / n_band
    pos_o = np.concatenate([lo1, lo2], axis=1)
    pos_o = pos_o + 0.05 * d_o * philox_uniform(seed, pos_o.shape)
    pos_b = band + 0.05 * d_b * philox_uniform(seed + 1000, band.shape)
    pos = np.concatenate([pos_o, pos_b], axis=1) % 1.0
    n_o, n = pos_o.shape[1], pos_o.shape[1] + pos_b.shape[1]
    s = abi.Species(n)
    s.pos[:] = pos
    isb = np.arange(n) >= n_o
    s.mass[:] = np.where(isb, 2.0 * d_b ** 3, 1.0 * d_o ** 3)
    s.density[:] = np.where(isb, 2.0, 1.0)
    s.u[:] = 2.5 / ((gamma - 1.0) * s.density)
    s.h[:] = hfact * np.where(isb, d_b, d_o)
    s.vel[0] = np.where(isb, 0.5, -0.5)
    s.vel[1] = 0.01 * np.sin(4 * math.pi * pos[0])
    s.B[0] = 0.1
    physics = (abi.PHYS_AV | abi.PHYS_MHD | abi.PHYS_DEDNER | abi.PHYS_TENSILE | abi.PHYS_CFL
               | abi.PHYS_ADAPTIVE_H)
    params = abi.default_params(kernel=abi.KERNEL_WENDLAND_C2, precision=precision, cull=abi.CULL_PAIR_MAX,
                                physics=physics, gamma=gamma, h0=hfact * d_o, dt=1e-4, cfl=0.3, hfact=hfact,
                                h_max=1.5 * hfact * d_o)
    box = abi.make_box((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (1, 1, 1))
    return Workload("kelvin_helmholtz", params, [box], {abi.SPECIES_DEFAULT: s}, steps=100,
                    meta={"n_outer": n_outer, "n_band": n_band})


def mhd_rotor(nxy=1024, nz=4, precision=abi.PREC_FP32_COMP, hfact=1.45, seed=4):
    """MHD rotor in a thin periodic slab [0,1]^2 x [0, nz/nxy].

    Ambient: rho 1 on an nxy x nxy x nz lattice.  Disc r < 0.1 (centre 0.5, 0.5):
    rho 10 on a finer lattice (9 layers per nz = 4 ambient layers in z, and the
    in-plane spacing that makes the number density ten times the ambient one),
    rigid rotation omega 20, linearly tapered to rest between r = 0.1 and 0.115.
    P = 1, Bx = 5/sqrt(4 pi), gamma 1.4; jitter 0.05 spacing (Philox, key seed).
    Equal masses; Wendland C2 with adaptive h (h = hfact (m/rho)^(1/3)), so the
    neighbour count is even in number but the cell sizes vary tenfold in
    density: the load-imbalance case.  nxy = 1024 gives about 5.4 M particles.
    """
    gamma = 1.4
    Lz = nz / nxy
    dxa = 1.0 / nxy
    amb = lattice((0.0, 0.0, 0.0), (1.0, 1.0, Lz), (nxy, nxy, nz))
    rr = np.hypot(amb[0] - 0.5, amb[1] - 0.5)
    amb = amb[:, rr >= 0.1]
    nzd = int(round(nz * 10 ** (1.0 / 3.0)))
    nzd += 1 if nzd == nz * 2 else 0
    # in-plane lattice count per unit length giving ten times the ambient number density
    nd = int(round(np.sqrt(10.0 * nxy ** 3 * Lz / nzd)))
    sq = lattice((0.4, 0.4, 0.0), (0.6, 0.6, Lz), (int(round(0.2 * nd)), int(round(0.2 * nd)), nzd))
    disc = sq[:, np.hypot(sq[0] - 0.5, sq[1] - 0.5) < 0.1]
    pos = np.concatenate([amb, disc], axis=1)
    pos = pos + 0.05 * dxa * philox_uniform(seed, pos.shape)
    pos[0] %= 1.0
    pos[1] %= 1.0
    pos[2] %= Lz
    n = pos.shape[1]
    s = abi.Species(n)
    s.pos[:] = pos
    m = dxa ** 2 * (Lz / nz)  # ambient mass: rho 1 times the ambient cell volume
    s.mass[:] = m
    isd = np.arange(n) >= amb.shape[1]
    s.density[:] = np.where(isd, 10.0, 1.0)
    s.u[:] = 1.0 / ((gamma - 1.0) * s.density)
    s.h[:] = hfact * np.cbrt(m / s.density)
    r = np.hypot(pos[0] - 0.5, pos[1] - 0.5)
    taper = np.clip((0.115 - r) / 0.015, 0.0, 1.0)
    omega = np.where(r < 0.1, 20.0, 20.0 * taper)
    s.vel[0] = -omega * (pos[1] - 0.5)
    s.vel[1] = omega * (pos[0] - 0.5)
    s.B[0] = 5.0 / math.sqrt(4 * math.pi)
    physics = (abi.PHYS_AV | abi.PHYS_MHD | abi.PHYS_DEDNER | abi.PHYS_TENSILE | abi.PHYS_CFL
               | abi.PHYS_ADAPTIVE_H)
    params = abi.default_params(kernel=abi.KERNEL_WENDLAND_C2, precision=precision, cull=abi.CULL_PAIR_MAX,
                                physics=physics, gamma=gamma, h0=hfact * dxa, dt=1e-5, cfl=0.3, hfact=hfact,
                                h_max=1.3 * hfact * dxa)
    box = abi.make_box((0.0, 0.0, 0.0), (1.0, 1.0, Lz), (1, 1, 1))
    return Workload("mhd_rotor", params, [box], {abi.SPECIES_DEFAULT: s}, steps=150,
                    meta={"nxy": nxy, "nz": nz, "n_disc": int(isd.sum())})
