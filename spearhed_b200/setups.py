"""Initial conditions for the benchmark and test workloads, as lattice blocks.

These play the part of the reference's setup blocks (SetupInterface +
InitParticles + the SC lattice: include/spearhed/particles/initialization/
SetupInterface.hpp:34-113, InitParticles.hpp:284-433,
spmacc/particles/initialization/SC.hpp:118-200,
share/spearhed/ValidationSetups/SodShockTube.hpp:128-176).  Every workload is a
list of :class:`LatticeBlock` (a region filled by a simple-cubic lattice at cell
centres, with constant state and an optional keep-mask) plus a profile of
analytic fields, a :class:`LatticeInit`.  The same description is generated two
ways with the same arithmetic: on the host here (:meth:`LatticeInit.generate`,
numpy) and on the device by ``sph_init_lattice`` (csrc/init.cu), which
:func:`spearhed_b200.context_for` uses with ``device_init=True``.

Jitter draws numpy's Philox4x64-10 (``Philox(key=seed).uniform(-1, 1)``) per
jitter group: axis a of the group's particle i takes value a * n_group + i.

Each generator returns a :class:`Workload`.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import abi


@dataclasses.dataclass
class LatticeBlock:
    """One region filled by an SC lattice (sites x-fastest, at lo + (i + 0.5) * ((hi - lo) / n))."""
    lo: tuple
    hi: tuple
    counts: tuple = (0, 0, 0)   # sites per axis; all 0: from `spacing` (sc_counts)
    spacing: float = 0.0
    mask: int = abi.MASK_NONE
    mask_centre: tuple = (0.0, 0.0)
    mask_radius: float = 0.0
    box_id: int = 0
    group: int = 0              # consecutive blocks of a group share one jitter stream
    jitter: float = 0.0         # uniform displacement amplitude (length) of the group
    seed: int = 0
    mass: float = 0.0
    h: float = 0.0
    density: float = 0.0
    u: float = 0.0
    psi: float = 0.0
    vel: tuple = (0.0, 0.0, 0.0)
    B: tuple = (0.0, 0.0, 0.0)

    def lattice_counts(self):
        if any(c > 0 for c in self.counts):
            return tuple(int(c) for c in self.counts)
        return sc_counts(self.lo, self.hi, self.spacing)


@dataclasses.dataclass
class LatticeInit:
    """A species as lattice blocks plus a profile (abi.PROFILE_*, parameters, periodic wrap)."""
    blocks: list
    profile: int = abi.PROFILE_CONSTANT
    params: tuple = ()
    wrap: tuple = (0, 0, 0)
    wrap_lo: tuple = (0.0, 0.0, 0.0)
    wrap_hi: tuple = (0.0, 0.0, 0.0)

    def to_abi(self):
        arr = (abi.SphLatticeBlock * max(len(self.blocks), 1))()
        for k, b in enumerate(self.blocks):
            d = arr[k]
            d.lo[:] = b.lo
            d.hi[:] = b.hi
            d.counts[:] = [int(c) for c in b.counts]
            d.spacing = b.spacing
            d.mask = b.mask
            d.mask_centre[:] = b.mask_centre
            d.mask_radius = b.mask_radius
            d.box_id = b.box_id
            d.jitter_group = b.group
            d.jitter = b.jitter
            d.seed = b.seed
            d.mass, d.h, d.density, d.u, d.psi = b.mass, b.h, b.density, b.u, b.psi
            d.vel[:] = b.vel
            d.B[:] = b.B
        prof = abi.SphInitProfile()
        prof.kind = self.profile
        prof.wrap[:] = list(self.wrap)
        prof.wrap_lo[:] = list(self.wrap_lo)
        prof.wrap_hi[:] = list(self.wrap_hi)
        for k, v in enumerate(self.params):
            prof.p[k] = v
        return arr, len(self.blocks), prof

    def generate(self) -> abi.Species:
        """Host generation with the device initialiser's arithmetic and order."""
        pos, state, groups = [], [], []
        for b in self.blocks:
            n = b.lattice_counts()
            x = lattice(b.lo, b.hi, n)
            if b.mask != abi.MASK_NONE:
                r = np.hypot(x[0] - b.mask_centre[0], x[1] - b.mask_centre[1])
                x = x[:, r < b.mask_radius] if b.mask == abi.MASK_INSIDE_DISC_XY else x[:, r >= b.mask_radius]
            pos.append(x)
            state.append((b, x.shape[1]))
        x = np.concatenate(pos, axis=1) if pos else np.zeros((3, 0))
        # jitter per group of consecutive blocks
        off, k = 0, 0
        while k < len(self.blocks):
            g = self.blocks[k].group
            kk, cnt = k, 0
            while kk < len(self.blocks) and self.blocks[kk].group == g:
                cnt += state[kk][1]
                kk += 1
            b0 = self.blocks[k]
            if b0.jitter != 0.0 and cnt:
                x[:, off:off + cnt] = x[:, off:off + cnt] + b0.jitter * philox_uniform(b0.seed, (3, cnt))
            off += cnt
            k = kk
        for a in range(3):
            if self.wrap[a]:
                L = self.wrap_hi[a] - self.wrap_lo[a]
                x[a] = self.wrap_lo[a] + (x[a] - self.wrap_lo[a]) % L
        n = x.shape[1]
        s = abi.Species(n)
        s.pos[:] = x
        off = 0
        for b, cnt in state:
            sl = slice(off, off + cnt)
            s.mass[sl], s.h[sl], s.density[sl], s.u[sl], s.psi[sl] = b.mass, b.h, b.density, b.u, b.psi
            for a in range(3):
                s.vel[a, sl] = b.vel[a]
                s.B[a, sl] = b.B[a]
            s.box_id[sl] = b.box_id
            off += cnt
        p = self.params
        if self.profile == abi.PROFILE_ORSZAG_TANG:
            s.vel[0] = -np.sin(2 * math.pi * x[1])
            s.vel[1] = np.sin(2 * math.pi * x[0])
            s.B[0] = -p[0] * np.sin(2 * math.pi * x[1])
            s.B[1] = p[0] * np.sin(4 * math.pi * x[0])
        elif self.profile == abi.PROFILE_KH_PERTURBATION:
            s.vel[1] = p[0] * np.sin(4 * math.pi * x[0])
        elif self.profile == abi.PROFILE_ROTOR:
            xc, yc, omega, r0, r1, width = p[:6]
            r = np.hypot(x[0] - xc, x[1] - yc)
            taper = np.clip((r1 - r) / width, 0.0, 1.0)
            w = np.where(r < r0, omega, omega * taper)
            s.vel[0] = -w * (x[1] - yc)
            s.vel[1] = w * (x[0] - xc)
        return s


def _trunc_near_integer(v, eps):
    """Truncation that snaps round-off just below an integer up (SC.hpp:49-58)."""
    t = int(v)
    tol = 4.0 * eps * (v if v > 1.0 else 1.0)
    dist = float(t + 1) - v
    return t + 1 if 0.0 <= dist <= tol else t


def sc_counts(lo, hi, spacing):
    """SC sites per axis (computeSCCellCounts, SC.hpp:98-132): axis 0 truncated
    with a round-off snap, transverse axes rounded, each at least 1 (double)."""
    n0 = _trunc_near_integer((hi[0] - lo[0]) / spacing, np.finfo(np.float64).eps)
    out = [max(n0, 1)]
    for a in (1, 2):
        out.append(max(int((hi[a] - lo[a]) / spacing + 0.5), 1))
    return tuple(out)


@dataclasses.dataclass
class Workload:
    name: str
    params: abi.SphParams
    boxes: list
    species: dict  # species id -> abi.Species
    steps: int = 1
    meta: dict = dataclasses.field(default_factory=dict)
    init: dict = dataclasses.field(default_factory=dict)  # species id -> LatticeInit (device initialiser input)

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


def _workload(name, params, boxes, inits, steps, meta):
    """A workload whose species are generated on the host from their lattice blocks."""
    return Workload(name, params, boxes, {sid: li.generate() for sid, li in inits.items()}, steps=steps,
                    meta=meta, init=inits)


def lattice(lo, hi, counts):
    """Simple-cubic lattice at cell centres of the box lo..hi, x fastest
    (SC.hpp:118-200: lo + (i + 0.5) * ((hi - lo) / n), each step rounded)."""
    axes = [lo[a] + (np.arange(counts[a]) + 0.5) * ((hi[a] - lo[a]) / counts[a]) for a in range(3)]
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
    dxl, dxr = 0.5 / nl[0], 0.5 / nr[0]
    m = 1.0 * dxl ** 3
    left = LatticeBlock((-0.5, 0.0, 0.0), (0.0, Ly, Ly), counts=nl, mass=m, h=hfact * dxl, density=1.0,
                        u=1.0 / ((gamma - 1.0) * 1.0))
    right = LatticeBlock((0.0, 0.0, 0.0), (0.5, Ly, Ly), counts=nr, mass=m, h=hfact * dxr, density=0.125,
                         u=0.1 / ((gamma - 1.0) * 0.125))
    physics = 0 if reference_physics else (abi.PHYS_AV | abi.PHYS_CFL | abi.PHYS_ADAPTIVE_H)
    params = abi.default_params(kernel=abi.KERNEL_CUBIC, precision=precision, cull=abi.CULL_PAIR_MAX,
                                physics=physics, gamma=gamma, h0=hfact * dxr, dt=1e-4, alpha=1.0, beta=2.0,
                                cfl=0.3, hfact=hfact, h_max=1.5 * hfact * dxr)
    box = abi.make_box((-0.75, 0.0, 0.0), (0.75, Ly, Ly), (0, 1, 1))
    return _workload("sod_small", params, [box], {abi.SPECIES_DEFAULT: LatticeInit([left, right])}, 50,
                     {"n_left": int(np.prod(nl)), "n_right": int(np.prod(nr)), "dx_left": dxl, "dx_right": dxr})


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
    rho0 = 25.0 / (36.0 * math.pi)
    P0 = 5.0 / (12.0 * math.pi)
    block = LatticeBlock((0.0, 0.0, 0.0), (1.0, 1.0, Lz), counts=(nx, nx, nz), jitter=jitter * dx if jitter > 0 else 0.0,
                         seed=seed, mass=rho0 * dx ** 3, h=hfact * dx, density=rho0, u=P0 / ((gamma - 1.0) * rho0))
    b0 = 1.0 / math.sqrt(4 * math.pi)
    wrap = (1, 1, 1) if jitter > 0 else (0, 0, 0)
    init = LatticeInit([block], abi.PROFILE_ORSZAG_TANG, (b0,), wrap=wrap, wrap_hi=(1.0, 1.0, Lz))
    physics = abi.PHYS_AV | abi.PHYS_MHD | abi.PHYS_DEDNER | abi.PHYS_TENSILE | abi.PHYS_CFL
    params = abi.default_params(kernel=abi.KERNEL_WENDLAND_C2, precision=precision, cull=abi.CULL_GLOBAL,
                                physics=physics, gamma=gamma, h0=hfact * dx, dt=2e-4, alpha=1.0, beta=2.0,
                                cfl=0.3, dedner_sigma=1.0)
    box = abi.make_box((0.0, 0.0, 0.0), (1.0, 1.0, Lz), (1, 1, 1))
    return _workload("orszag_tang", params, [box], {abi.SPECIES_DEFAULT: init}, 200, {"nx": nx, "nz": nz, "dx": dx})


def _brio_wu_blocks(n_target, precision, nt, box_id, reference_physics=False):
    gamma = 2.0
    nxl = max(8, int(round(n_target / (nt * nt * 1.125))))
    nxl += nxl % 2
    dxl = 0.5 / nxl
    L = nt * dxl
    m = dxl ** 3
    # reference physics: one constant h per box (the reference's h0 is both the
    # cull radius / 2 and every particle's h), here the left state's 1.2 dxl
    hr = 1.2 * dxl if reference_physics else 2.4 * dxl
    left = LatticeBlock((-0.5, 0.0, 0.0), (0.0, L, L), counts=(nxl, nt, nt), box_id=box_id, mass=m, h=1.2 * dxl,
                        density=1.0, u=1.0 / ((gamma - 1.0) * 1.0), B=(0.75, 1.0, 0.0))
    right = LatticeBlock((0.0, 0.0, 0.0), (0.5, L, L), counts=(nxl // 2, nt // 2, nt // 2), box_id=box_id, mass=m,
                         h=hr, density=0.125, u=0.1 / ((gamma - 1.0) * 0.125), B=(0.75, -1.0, 0.0))
    if reference_physics:
        # the reference's step: inviscid hydro, constant h and dt, no periodic
        # images (its region search has none); the pair-max cull with one h per
        # box is the reference's global radius 2 h0 box by box.  The tube's free
        # y and z surfaces expand, so the closed box leaves a tube width of room
        # on each side.
        params = abi.default_params(kernel=abi.KERNEL_CUBIC, precision=precision, cull=abi.CULL_PAIR_MAX,
                                    physics=0, gamma=gamma, h0=1.2 * dxl, dt=1e-5)
        box = abi.make_box((-0.75, -L, -L), (0.75, 2.0 * L, 2.0 * L), (0, 0, 0))
        return params, box, [left, right]
    physics = (abi.PHYS_AV | abi.PHYS_MHD | abi.PHYS_DEDNER | abi.PHYS_TENSILE | abi.PHYS_CFL
               | abi.PHYS_ADAPTIVE_H)
    params = abi.default_params(kernel=abi.KERNEL_CUBIC, precision=precision, cull=abi.CULL_PAIR_MAX,
                                physics=physics, gamma=gamma, h0=2.4 * dxl, dt=1e-5, alpha=1.0, beta=2.0,
                                cfl=0.3, hfact=1.2, h_max=3.6 * dxl)
    box = abi.make_box((-0.75, 0.0, 0.0), (0.75, L, L), (0, 1, 1))
    return params, box, [left, right]


def brio_wu_box(n_target=8192, precision=abi.PREC_FP32_COMP, nt=8, box_id=0):
    """One 3D Brio-Wu MHD shock tube (gamma 2, Bx 0.75).

    Left x in [-0.5, 0): rho 1, P 1, By +1; right x in [0, 0.5): rho 0.125, P 0.1,
    By -1.  Equal masses: the right lattice spacing is twice the left.  The tube
    is nt left lattice layers thick in y and z (periodic); its length is chosen
    so the box holds about n_target particles.  x is open (the box extends 0.25
    beyond each end).  Cubic spline, AV, SPMHD with Dedner cleaning and the
    tensile correction, adaptive h (hfact 1.2), CFL 0.3.
    """
    params, box, blocks = _brio_wu_blocks(n_target, precision, nt, box_id)
    return params, box, LatticeInit(blocks).generate()


def brio_wu_sizes(nbox=512, seed=5, n_lo=4096, n_hi=262144):
    """Target particle counts of the ensemble's boxes: log-uniform in
    [n_lo, n_hi] (numpy Philox, key ``seed``)."""
    rng = np.random.Generator(np.random.Philox(key=seed))
    return np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), size=nbox)).astype(int)


def brio_wu_ensemble(nbox=512, precision=abi.PREC_FP32_COMP, seed=5, n_lo=4096, n_hi=262144, rank=0, world=1,
                     reference_physics=False, boxes=None):
    """An ensemble of independent Brio-Wu tubes with particle counts drawn
    log-uniform in [n_lo, n_hi] (numpy Philox, key ``seed``).  With the default
    512 boxes this is about 31 M particles.  Every box keeps its own time step.
    The ensemble-wide h_max is 0, so each box sizes its grid from its own
    largest h (x1.5 under adaptive h, within its periodic extent).

    With ``world`` > 1 only the boxes that longest-processing-time assigns to
    ``rank`` are built (renumbered from 0; their global ids are in
    ``meta["global_boxes"]``), so each rank generates only its own particles.

    ``reference_physics`` builds the same particles under the reference's own
    step (inviscid hydro, one constant h per box, constant dt, no periodic
    images); ``boxes`` (global ids) builds only those boxes."""
    from .ensemble import lpt_partition
    sizes = brio_wu_sizes(nbox, seed, n_lo, n_hi)
    mine = np.arange(nbox) if world <= 1 else np.flatnonzero(lpt_partition(sizes, world) == rank)
    if boxes is not None:
        mine = np.asarray(boxes, dtype=np.int64)
    blist, blocks, params = [], [], None
    for local, b in enumerate(mine):
        p, box, bl = _brio_wu_blocks(int(sizes[b]), precision, 8, local, reference_physics)
        blist.append(box)
        blocks.extend(bl)
        params = p
    if params is None:  # a rank with no boxes
        params, _, _ = _brio_wu_blocks(int(n_lo), precision, 8, 0, reference_physics)
    params.h_max = 0.0
    return _workload("brio_wu_ensemble", params, blist, {abi.SPECIES_DEFAULT: LatticeInit(blocks)}, 100,
                     {"sizes": sizes.tolist(), "seed": seed, "global_boxes": mine.tolist(),
                      "reference_physics": bool(reference_physics)})


def kelvin_helmholtz(n_outer=224, n_band=282, precision=abi.PREC_FP32_COMP, hfact=1.45, seed=3):
    """Magnetised Kelvin-Helmholtz in the periodic unit cube.

    Band |y - 0.5| < 0.25: rho 2, vx +0.5; outside: rho 1, vx -0.5.  Each region
    is a lattice whose spacing follows its density (n_band/n_outer ~ 2^(1/3);
    n_outer = 224, n_band = 282 give 5.62 M + 11.21 M = 16.8 M particles, masses
    within 0.5% of each other).  Uniform jitter of 0.05 spacing (Philox, key
    ``seed`` outside, ``seed`` + 1000 in the band), vy = 0.01 sin(4 pi x), P = 2.5,
    gamma 5/3, Bx = 0.1.  Wendland C2, h = hfact x local spacing (adaptive), AV,
    SPMHD with Dedner cleaning, CFL.
    """
    gamma = 5.0 / 3.0
    if n_outer % 4 or n_band % 2:
        raise ValueError("n_outer must be a multiple of 4 and n_band even (whole layers per slab)")
    d_o, d_b = 1.0 / n_outer, 1.0 / n_band
    outer = dict(group=0, jitter=0.05 * d_o, seed=seed, mass=1.0 * d_o ** 3, h=hfact * d_o, density=1.0,
                 u=2.5 / ((gamma - 1.0) * 1.0), vel=(-0.5, 0.0, 0.0), B=(0.1, 0.0, 0.0))
    blocks = [
        LatticeBlock((0.0, 0.0, 0.0), (1.0, 0.25, 1.0), counts=(n_outer, n_outer // 4, n_outer), **outer),
        LatticeBlock((0.0, 0.75, 0.0), (1.0, 1.0, 1.0), counts=(n_outer, n_outer // 4, n_outer), **outer),
        LatticeBlock((0.0, 0.25, 0.0), (1.0, 0.75, 1.0), counts=(n_band, n_band // 2, n_band), group=1,
                     jitter=0.05 * d_b, seed=seed + 1000, mass=2.0 * d_b ** 3, h=hfact * d_b, density=2.0,
                     u=2.5 / ((gamma - 1.0) * 2.0), vel=(0.5, 0.0, 0.0), B=(0.1, 0.0, 0.0)),
    ]
    init = LatticeInit(blocks, abi.PROFILE_KH_PERTURBATION, (0.01,), wrap=(1, 1, 1), wrap_hi=(1.0, 1.0, 1.0))
    physics = (abi.PHYS_AV | abi.PHYS_MHD | abi.PHYS_DEDNER | abi.PHYS_TENSILE | abi.PHYS_CFL
               | abi.PHYS_ADAPTIVE_H)
    params = abi.default_params(kernel=abi.KERNEL_WENDLAND_C2, precision=precision, cull=abi.CULL_PAIR_MAX,
                                physics=physics, gamma=gamma, h0=hfact * d_o, dt=1e-4, cfl=0.3, hfact=hfact,
                                h_max=1.5 * hfact * d_o)
    box = abi.make_box((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (1, 1, 1))
    return _workload("kelvin_helmholtz", params, [box], {abi.SPECIES_DEFAULT: init}, 100,
                     {"n_outer": n_outer, "n_band": n_band})


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
    nzd = int(round(nz * 10 ** (1.0 / 3.0)))
    nzd += 1 if nzd == nz * 2 else 0
    # in-plane lattice count per unit length giving ten times the ambient number density
    nd = int(round(np.sqrt(10.0 * nxy ** 3 * Lz / nzd)))
    m = dxa ** 2 * (Lz / nz)  # ambient mass: rho 1 times the ambient cell volume
    Bx = 5.0 / math.sqrt(4 * math.pi)
    common = dict(group=0, jitter=0.05 * dxa, seed=seed, mass=m, B=(Bx, 0.0, 0.0), mask_centre=(0.5, 0.5),
                  mask_radius=0.1)
    blocks = [
        LatticeBlock((0.0, 0.0, 0.0), (1.0, 1.0, Lz), counts=(nxy, nxy, nz), mask=abi.MASK_OUTSIDE_DISC_XY,
                     density=1.0, u=1.0 / ((gamma - 1.0) * 1.0), h=float(hfact * np.cbrt(m / 1.0)), **common),
        LatticeBlock((0.4, 0.4, 0.0), (0.6, 0.6, Lz), counts=(int(round(0.2 * nd)), int(round(0.2 * nd)), nzd),
                     mask=abi.MASK_INSIDE_DISC_XY, density=10.0, u=1.0 / ((gamma - 1.0) * 10.0),
                     h=float(hfact * np.cbrt(m / 10.0)), **common),
    ]
    init = LatticeInit(blocks, abi.PROFILE_ROTOR, (0.5, 0.5, 20.0, 0.1, 0.115, 0.015), wrap=(1, 1, 1),
                       wrap_hi=(1.0, 1.0, Lz))
    physics = (abi.PHYS_AV | abi.PHYS_MHD | abi.PHYS_DEDNER | abi.PHYS_TENSILE | abi.PHYS_CFL
               | abi.PHYS_ADAPTIVE_H)
    params = abi.default_params(kernel=abi.KERNEL_WENDLAND_C2, precision=precision, cull=abi.CULL_PAIR_MAX,
                                physics=physics, gamma=gamma, h0=hfact * dxa, dt=1e-5, cfl=0.3, hfact=hfact,
                                h_max=1.3 * hfact * dxa)
    box = abi.make_box((0.0, 0.0, 0.0), (1.0, 1.0, Lz), (1, 1, 1))
    w = _workload("mhd_rotor", params, [box], {abi.SPECIES_DEFAULT: init}, 150, {"nxy": nxy, "nz": nz})
    w.meta["n_disc"] = int(np.sum(w.species[abi.SPECIES_DEFAULT].density == 10.0))
    return w
