"""Row sharding of the torus exchange (esthera_b200.sharding) as 2 and 4 gloo
ranks on CPU: every rank's exchanged sub-filters equal the single-process
exchange of the whole torus (the oracle's routing)."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _full_exchange(O, N, m, t, S, seed):
    rng = np.random.default_rng(seed)
    keys = -np.sort(-rng.standard_normal((N, m)).astype(np.float32), axis=1).reshape(-1)
    state = rng.standard_normal((S, N * m)).astype(np.float32)
    src = O.exchange_sources(2, N, m, t)  # torus
    return state, keys, state[:, src], keys[src]


def _rank(rank, world, port, N, m, t, S, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
        import sys
        sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
        import oracle as O
        from esthera_b200.sharding import TorusShard, halo_exchange
        state, keys, want_state, want_keys = _full_exchange(O, N, m, t, S, 7)
        sh = TorusShard(N, m, t, world, rank)
        lo, hi = sh.first_subfilter * m, (sh.first_subfilter + sh.num_subfilters) * m
        ls, lk = state[:, lo:hi], keys[lo:hi]
        up, down = sh.halos_out(ls, lk)
        tt = lambda h: (torch.from_numpy(np.ascontiguousarray(h[0])), torch.from_numpy(np.ascontiguousarray(h[1])))
        fu, fd = halo_exchange(dist, sh, tt(up), tt(down))
        got_s, got_k = sh.apply_exchange(ls, lk, (fu[0].numpy(), fu[1].numpy()), (fd[0].numpy(), fd[1].numpy()))
        ok = np.array_equal(got_s, want_state[:, lo:hi]) and np.array_equal(got_k, want_keys[lo:hi])
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, ok))
    except Exception as e:  # report, never hang the parent
        q.put((rank, repr(e)))


@pytest.mark.parametrize("world,N,t", [(2, 64, 2), (4, 128, 1), (2, 8, 1)])
def test_sharded_torus_exchange_matches_single(world, N, t):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    m, S = 16, 3
    procs = [ctx.Process(target=_rank, args=(r, world, port, N, m, t, S, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert all(v is True for v in res.values()), res


def test_single_rank_shard_is_whole_torus(O):
    from esthera_b200.sharding import TorusShard
    N, m, t, S = 32, 16, 2, 3
    state, keys, want_state, want_keys = _full_exchange(O, N, m, t, S, 3)
    sh = TorusShard(N, m, t, 1, 0)
    up, down = sh.halos_out(state, keys)
    got_s, got_k = sh.apply_exchange(state, keys, down, up)
    assert np.array_equal(got_s, want_state) and np.array_equal(got_k, want_keys)
    with pytest.raises(ValueError):
        TorusShard(2048, 512, 2, 3, 0)  # 64 rows over 3 ranks
