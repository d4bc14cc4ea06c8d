"""bench.job_totals, the whole-job reduction of a multi-rank bench run (host
logic, CPU): over a world-size-2 gloo group the job's time is the slowest
rank's and its pairs and copied bytes are the ranks' sums.  On GPUs bench.py
runs the same call over NCCL for the timed steps and the end-to-end leg."""
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, result_path):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    # rank r: time 10 + 5 r ms, 1000 (r + 1) pairs, 3 + r GB in, 2 + r GB out
    slow, summed = bench.job_totals([10.0 + 5 * rank], [1000.0 * (rank + 1), 3e9 + 1e9 * rank, 2e9 + 1e9 * rank],
                                    "cpu")
    if rank == 0:
        ok = slow == [15.0] and summed == [3000.0, 7e9, 5e9]
        with open(result_path, "w") as f:
            f.write("ok" if ok else f"bad {slow} {summed}")
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_job_totals_take_the_slowest_rank_and_sum_the_rest(tmp_path):
    import torch.multiprocessing as mp
    out = tmp_path / "result.txt"
    mp.start_processes(_worker, args=(2, _free_port(), str(out)), nprocs=2, start_method="spawn")
    assert out.read_text() == "ok"
