"""Field sharding across ranks: LPT balance and the gather of
log-likelihoods and gradients, with two gloo ranks on CPU (the per-field
evaluation is a stand-in here; tests/test_gpu_sharding.py runs real batches)."""
import os
import socket

import numpy as np


def test_lpt_partition_balances_cubic_costs():
    from exageostat_b200.sharding import lpt_partition

    rng = np.random.default_rng(0)
    n = rng.integers(500, 6001, size=512)
    parts = lpt_partition(n.astype(float) ** 3, 8)
    assert sorted(i for p in parts for i in p) == list(range(512))
    loads = [sum(float(n[i]) ** 3 for i in p) for p in parts]
    assert max(loads) / min(loads) < 1.02


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, sizes, thetas, q):
    import torch.distributed as dist

    from exageostat_b200.sharding import sharded_batch_loglik

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        evaluate = lambda idx, th: [sizes[i] * 1000.0 + th[j][0] for j, i in enumerate(idx)]
        out = sharded_batch_loglik(sizes, thetas, evaluate)
        q.put((rank, out.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_returns_every_field_on_every_rank():
    import torch.multiprocessing as mp

    sizes = [520, 5900, 1200, 3000, 800, 4100, 2600]
    thetas = [[0.1 * i, 0.1, 0.5] for i in range(len(sizes))]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, thetas, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    expect = [s * 1000.0 + t[0] for s, t in zip(sizes, thetas)]
    for _, out in res:
        assert np.allclose(out, expect)


def _worker_grad(rank, world, port, sizes, thetas, q):
    import torch.distributed as dist

    from exageostat_b200.sharding import sharded_batch_loglik

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        def evaluate(idx, th):
            ll = [sizes[i] * 1000.0 + th[j][0] for j, i in enumerate(idx)]
            g = [[sizes[i], th[j][1], -th[j][2]] for j, i in enumerate(idx)]
            return ll, g

        ll, g = sharded_batch_loglik(sizes, thetas, evaluate, grad=True)
        q.put((rank, ll.tolist(), g.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_of_loglik_and_gradients():
    import torch.multiprocessing as mp

    sizes = [520, 5900, 1200, 3000, 800, 4100, 2600, 700]
    thetas = [[0.1 * i, 0.2 + i, 0.5 * i] for i in range(len(sizes))]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_grad, args=(r, 2, port, sizes, thetas, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    for _, ll, g in res:
        assert np.allclose(ll, [s * 1000.0 + t[0] for s, t in zip(sizes, thetas)])
        assert np.allclose(g, [[s, t[1], -t[2]] for s, t in zip(sizes, thetas)])
