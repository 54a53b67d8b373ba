"""The multi-GPU path of bench.py is independent replicas: the host logic
(maximum of the per-rank times over the process group, whole-job
throughput) runs here on CPU with the gloo backend and two ranks; the
reference arm's ranks other than 0 exit without work."""
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = bench.max_over_ranks(10.0 + 5.0 * rank)
    e2e = bench.max_over_ranks(2.0 + rank)
    comb = bench.combine_replicas(ms, e2e, world, 1000, 3)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ms, e2e, comb))


def _free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_replica_timing_is_the_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, e2e, comb in res:
        assert ms == 15.0 and e2e == 3.0
        work = 2 * 1000 * 100 * 3
        assert comb["value"] == pytest.approx(work / 15e-3)
        assert comb["ms_per_step"] == pytest.approx(5.0)
        assert comb["e2e_value"] == pytest.approx(work / 3.0)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
