"""Table-gradient all-reduce across ranks (gloo, two processes on the CPU)."""
import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        from agama_gpu_b200.integrate import allreduce_table_grads

        class Comp:                      # stands in for a Multipole (only its order matters)
            def __init__(self, k):
                self._sync_order = k
        a, b = Comp(0), Comp(1)
        # insertion order differs between ranks; the reduction order must not
        tg = {b: torch.full((2, 3), 10.0 * (rank + 1)), a: torch.arange(4.0) * (rank + 1)}
        if rank == 1:
            tg = {a: tg[a], b: tg[b]}
        out = allreduce_table_grads(tg)
        q.put((rank, out[a].tolist(), out[b].tolist()))
    finally:
        dist.destroy_process_group()


def test_table_gradients_summed_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, a, b in res:
        assert a == [0.0, 3.0, 6.0, 9.0]
        assert b == [[30.0] * 3] * 2


def test_single_process_is_a_no_op():
    from agama_gpu_b200.integrate import allreduce_table_grads
    t = {"x": torch.ones(3)}
    assert allreduce_table_grads(t) is t and torch.equal(t["x"], torch.ones(3))
