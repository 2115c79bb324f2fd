"""bench.py runs N independent replicas (one tank per GPU, no data
exchange); its only collectives are the barrier and the max/sum of the
per-rank timings.  Checked here with world_size 2 over gloo on CPU."""
import os
import pathlib
import socket
import sys

import torch.multiprocessing as mp

ROOT = pathlib.Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import bench
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t_max, units = bench.combine_ranks(0.5 + rank, 1000 * (rank + 1), device=None)
    q.put((rank, t_max, units))
    dist.destroy_process_group()


def test_two_rank_combination():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == [(0, 1.5, 3000), (1, 1.5, 3000)]
