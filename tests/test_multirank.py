"""The multi-rank bench logic on CPU: world size 2 over gloo. Envs are
sharded by rank (weak scaling, no collective in the step), timings are the
max over ranks, and the reference arm runs on rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    sys.path.insert(0, ROOT)
    import numpy as np

    import bench
    from pippin_b200 import mjcf, scenes
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        m = mjcf.load_string(scenes.ant_xml())
        q, v, _ = bench.initial_state(m, 8, bench.shard_seeds(rank)["state"])
        # this rank's (made-up) timed totals: rank 1 is the slow one
        mine = [10.0 + 5.0 * rank, 20.0 - 5.0 * rank, 30.0]
        mx, rates = bench.whole_job(mine, 4096, 100, ws)
        out[rank] = (mx, rates, float(q.sum()), float(v.sum()))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_envs_and_take_the_slowest():
    ws, port = 2, _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_rank_main, args=(ws, port, out), nprocs=ws, join=True)
        res = dict(out)
    assert set(res) == {0, 1}
    for r in (0, 1):
        mx, rates, _, _ = res[r]
        assert mx == [15.0, 20.0, 30.0]  # element-wise max over the ranks
        total = 4096 * ws * 100
        assert rates == pytest.approx([total / (t * 1e-3) for t in mx])
    # each rank steps its own, different envs
    assert res[0][2] != res[1][2] and res[0][3] != res[1][3]


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "3", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
