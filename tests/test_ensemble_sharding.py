"""Ensemble sharding across ranks (host logic, CPU): LPT partition, shards that
cover every box exactly once, and the host-side gather of per-box diagnostics
over a world-size-2 gloo group.  The per-rank stepping is replaced by a fake
context here; on GPUs each rank steps its shard with the CUDA library."""
import os
import socket

import numpy as np
import pytest

from spearhed_b200 import abi, ensemble, setups


def test_lpt_is_balanced_and_deterministic():
    rng = np.random.default_rng(0)
    costs = np.exp(rng.uniform(np.log(4e3), np.log(2.6e5), 512))
    for world in (1, 2, 4, 8):
        owner = ensemble.lpt_partition(costs, world)
        assert np.array_equal(owner, ensemble.lpt_partition(costs, world))
        loads = np.bincount(owner, weights=costs, minlength=world)
        # LPT bound: makespan <= (4/3 - 1/(3m)) OPT and OPT >= mean load, >= max item
        opt_lb = max(costs.sum() / world, costs.max())
        assert loads.max() <= (4.0 / 3.0) * opt_lb + 1e-9


def test_shards_cover_every_box_once():
    w = setups.brio_wu_ensemble(nbox=24, n_lo=500, n_hi=4000)
    s = w.species[abi.SPECIES_DEFAULT]
    seen = []
    total = 0
    for rank in range(3):
        boxes, sub, mine = ensemble.shard(w, rank, 3)
        assert len(boxes) == len(mine)
        assert set(np.unique(sub.box_id)) <= set(range(len(mine)))
        seen.extend(mine.tolist())
        total += sub.n
        # particle data of a shard is the original data of its boxes, in order
        for k, b in enumerate(mine):
            assert np.array_equal(sub.pos[:, sub.box_id == k], s.pos[:, s.box_id == b])
    assert sorted(seen) == list(range(24))
    assert total == s.n


class FakeContext:
    """Stands in for the CUDA context: 'steps' every box and reports its count."""

    def __init__(self, params, boxes):
        self.nbox = len(boxes)

    def set_species(self, sid, s):
        self.counts = np.bincount(s.box_id, minlength=self.nbox)

    def step(self, n):
        self.n = n

    def ensemble_reduce(self, nbox):
        return [{"n_targets": int(c), "steps": self.n} for c in self.counts]

    def close(self):
        pass


def _worker(rank, world, port, result_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    w = setups.brio_wu_ensemble(nbox=16, n_lo=500, n_hi=3000)
    mine, diags = ensemble.run_shard(w, rank, world, steps=3, make_context=FakeContext)
    merged = ensemble.gather_diagnostics(diags, mine, len(w.boxes))
    if rank == 0:
        counts = np.bincount(w.species[abi.SPECIES_DEFAULT].box_id, minlength=len(w.boxes))
        ok = all(merged[b] is not None and merged[b]["n_targets"] == counts[b] and merged[b]["steps"] == 3
                 for b in range(len(w.boxes)))
        with open(result_path, "w") as f:
            f.write("ok" if ok else "bad")
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_run_gathers_every_box_over_gloo(tmp_path):
    import torch.multiprocessing as mp
    out = tmp_path / "result.txt"
    mp.start_processes(_worker, args=(2, _free_port(), str(out)), nprocs=2, start_method="spawn")
    assert out.read_text() == "ok"


def test_ensemble_setup_builds_only_the_ranks_boxes():
    """setups.brio_wu_ensemble(rank, world) builds exactly the boxes the LPT
    partition gives that rank; together the ranks cover the ensemble once."""
    from spearhed_b200 import setups
    full = setups.brio_wu_ensemble(nbox=12, n_lo=512, n_hi=2048)
    seen = []
    total = 0
    for r in range(3):
        w = setups.brio_wu_ensemble(nbox=12, n_lo=512, n_hi=2048, rank=r, world=3)
        g = w.meta["global_boxes"]
        seen += g
        s = w.species[abi.SPECIES_DEFAULT]
        assert len(w.boxes) == len(g) and set(np.unique(s.box_id)) <= set(range(len(g)))
        total += s.n
    assert sorted(seen) == list(range(12))
    assert total == full.species[abi.SPECIES_DEFAULT].n
