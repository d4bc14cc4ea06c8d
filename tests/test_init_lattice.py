"""Lattice initialisation on the host: the SC count rule and placement pinned to
the reference's known answers (tests/spearhed/unit/ParticleInit/ParticleInit.cpp),
and the Philox4x64-10 stream the device initialiser draws, restated here the way
csrc/init.cu computes it, against numpy's Philox generator."""
import ctypes as C

import numpy as np

from spearhed_b200 import abi, setups


def _counts_c(lo, hi, spacing, f32=False):
    L = abi.lib()
    out = (C.c_uint32 * 3)()
    if f32:
        rc = L.sph_sc_cell_counts_f32((C.c_float * 3)(*lo), (C.c_float * 3)(*hi), C.c_float(spacing), out)
    else:
        rc = L.sph_sc_cell_counts((C.c_double * 3)(*lo), (C.c_double * 3)(*hi), C.c_double(spacing), out)
    assert rc == abi.SPH_OK
    return tuple(out)


def test_sc_counts_tolerate_roundoff_at_an_integral_ratio():
    # ParticleInit.cpp:108-119: the 3D Sod spacing 2 * (1/30) in float gives 15
    # cells on a unit axis; a 14.75-long axis at spacing 1 gives 14
    sod_right = float(np.float32(2.0) * (np.float32(1.0) / np.float32(30.0)))
    assert _counts_c((0, 0, 0), (1, 1, 1), sod_right, f32=True)[0] == 15
    assert _counts_c((0, 0, 0), (14.75, 1, 1), 1.0, f32=True)[0] == 14
    assert _counts_c((0, 0, 0), (1, 1, 1), 2.0 * (1.0 / 30.0))[0] == 15
    assert _counts_c((0, 0, 0), (14.75, 1, 1), 1.0)[0] == 14


def test_sc_counts_of_a_non_cubic_box_and_their_sites():
    # ParticleInit.cpp:324-361: [0,3] x [0,1] x [0,0.5] at spacing 1 -> (3, 1, 1),
    # sites (0.5, 0.5, 0.25), (1.5, 0.5, 0.25), (2.5, 0.5, 0.25)
    n = _counts_c((0, 0, 0), (3, 1, 0.5), 1.0)
    assert n == (3, 1, 1) == setups.sc_counts((0, 0, 0), (3, 1, 0.5), 1.0)
    x = setups.lattice((0, 0, 0), (3, 1, 0.5), n)
    assert np.array_equal(x.T, [[0.5, 0.5, 0.25], [1.5, 0.5, 0.25], [2.5, 0.5, 0.25]])


def test_sc_lattice_of_eight_sites():
    # ParticleInit.cpp:277-300: 2 x 2 x 2 in the unit cube, every axis sums to 4
    x = setups.lattice((0, 0, 0), (1, 1, 1), (2, 2, 2))
    assert np.array_equal(np.sort(np.unique(x)), [0.25, 0.75])
    assert np.all(x.sum(axis=1) == 4.0)


def test_python_count_rule_equals_the_library_rule():
    rng = np.random.default_rng(7)
    for _ in range(500):
        lo = rng.uniform(-1, 1, 3)
        hi = lo + rng.uniform(0.01, 3, 3)
        sp = rng.uniform(0.003, 0.5)
        assert setups.sc_counts(lo, hi, sp) == _counts_c(lo, hi, sp)


def _philox4x64(ctr, key):
    M0, M1 = 0xD2E7470EE14C6C93, 0xCA5A826395121157
    W0, W1 = 0x9E3779B97F4A7C15, 0xBB67AE8584CAA73B
    mask = (1 << 64) - 1
    c, k = list(ctr), list(key)
    for _ in range(10):
        p0, p1 = M0 * c[0], M1 * c[2]
        c = [(p1 >> 64) ^ c[1] ^ k[0], p1 & mask, (p0 >> 64) ^ c[3] ^ k[1], p0 & mask]
        k = [(k[0] + W0) & mask, (k[1] + W1) & mask]
    return c


def test_device_philox_stream_is_numpys():
    for seed in (2, 3, 4, 1003):
        want = setups.philox_uniform(seed, (3, 7)).ravel()
        got = []
        for index in range(21):
            w = _philox4x64([index // 4 + 1, 0, 0, 0], [seed, 0])[index % 4]
            got.append(-1.0 + 2.0 * ((w >> 11) * (1.0 / 9007199254740992.0)))
        assert np.array_equal(np.array(got), want), seed


def test_lattice_init_keeps_block_order_masks_and_groups():
    w = setups.mhd_rotor(nxy=64, nz=4)
    s = w.species[abi.SPECIES_DEFAULT]
    li = w.init[abi.SPECIES_DEFAULT]
    r = np.hypot(s.pos[0] - 0.5, s.pos[1] - 0.5)
    disc = s.density == 10.0
    assert w.meta["n_disc"] == int(disc.sum()) > 0
    assert np.all(np.diff(disc.astype(int)) >= 0)      # ambient block first, then the disc
    assert r[disc].max() < 0.1 + 0.1 * (1.0 / 64)      # disc sites inside 0.1 before jitter
    assert len(li.blocks) == 2 and li.blocks[0].group == li.blocks[1].group
