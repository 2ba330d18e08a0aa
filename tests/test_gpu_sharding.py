"""Sharded batches with real fields: two ranks (gloo, spawned processes)
each build an exageostat_b200.Batch of their LPT share of the fields on the
one GPU of this box and gather every field's log-likelihood and gradient; the
result must equal one process evaluating the whole batch.  The ranks'
kernels never wait on one another (the only exchange is the host-side gather
after each rank's evaluation), so sharing one GPU is safe."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _fields(seed, nfields):
    rng = np.random.default_rng(seed)
    xs, ys, zs, th = [], [], [], []
    for _ in range(nfields):
        n = int(rng.integers(300, 1800))
        xs.append(rng.random(n)), ys.append(rng.random(n)), zs.append(rng.standard_normal(n))
        th.append([rng.uniform(0.5, 2.0), rng.uniform(0.02, 0.1), rng.uniform(0.3, 1.0)])
    return xs, ys, zs, np.array(th)


def _rank(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ.setdefault("EXAGEOSTAT_B200_SILENT", "1")
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import exageostat_b200 as xg
        from exageostat_b200.sharding import ShardedBatch

        xg.init(0)
        xs, ys, zs, th = _fields(3, 11)
        with ShardedBatch(xs, ys, zs, ts=256) as sb:
            ll, g = sb.loglik(th, grad=True)
            q.put((rank, len(sb.mine), ll.tolist(), g.tolist()))
    except Exception as e:  # reported to the parent
        q.put((rank, -1, repr(e), None))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_real_batches(gpu):
    import torch.multiprocessing as mp

    xs, ys, zs, th = _fields(3, 11)
    with gpu.Batch(xs, ys, zs, ts=256) as b:
        ll_ref, g_ref = b.loglik(th, grad=True)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in procs]
    for p in procs:
        p.join(timeout=120)
    assert sum(r[1] for r in res) == 11, res
    for _, nmine, ll, g in res:
        assert nmine > 0
        assert np.allclose(ll, ll_ref, rtol=1e-13, atol=0)
        assert np.allclose(g, g_ref, rtol=1e-10, atol=1e-10 * np.abs(g_ref).max())
