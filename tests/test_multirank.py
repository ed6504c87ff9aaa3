"""The N > 1 path of bench.py on CPU: two gloo ranks shard the energy grid
without overlap and agree on the max-over-ranks job time."""

import datetime
import json
import multiprocessing
import os
import socket

import numpy as np


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, outdir):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    E = bench.shard_energies(8, world, rank)
    t = bench.max_over_ranks(1.5 + rank, dist, "cpu")
    with open(os.path.join(outdir, "rank%d.json" % rank), "w") as f:
        json.dump({"E": E.tolist(), "t": t}, f)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce(tmp_path):
    world = 2
    port = _free_port()
    ctx = multiprocessing.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = [json.load(open(os.path.join(str(tmp_path), "rank%d.json" % r))) for r in range(world)]
    assert res[0]["t"] == res[1]["t"] == 2.5  # the slowest rank's time
    e0, e1 = res[0]["E"], res[1]["E"]
    assert len(set(e0) & set(e1)) == 0
    assert np.allclose(np.array(e0 + e1), np.linspace(-1.0, 1.0, 16))


def test_gpus_flag_spawns_ranks_itself():
    """bench.py --gpus 2 without a launcher starts two ranks through
    torch.distributed.run (the reference arm runs on CPU: rank 0 prints the one
    JSON line, rank 1 exits without work)."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0", "--cpu-budget-s", "0.5", "--npl", "3", "--b", "8",
                        "--ne", "4"], capture_output=True, text=True, timeout=300, env=env, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout
    assert lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2
