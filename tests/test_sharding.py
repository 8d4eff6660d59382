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


def _fake_snapshot(model, particles, m, seed):
    """A buffer in pf_server_snapshot's layout (header + random body)."""
    from esthera_b200.sharding import SNAPSHOT_MAGIC
    body = np.random.default_rng(seed).integers(0, 256, 3 * 4 * particles + 351 * 4 * (particles // m) + 4,
                                                dtype=np.uint8)
    hdr = np.array([SNAPSHOT_MAGIC, model, particles, particles // m], np.int64)
    return hdr.tobytes() + body.tobytes()


def test_plan_moves_balances_particles():
    from esthera_b200.sharding import plan_moves
    loads = [[(1, 4096), (2, 2048), (3, 1024), (4, 1024)], [(5, 256)], []]
    moves = plan_moves(loads)
    per = [dict(l) for l in loads]
    for src, dst, fid in moves:
        per[dst][fid] = per[src].pop(fid)
    tot = [sum(p.values()) for p in per]
    assert max(tot) == 4096 and sum(tot) == 8448  # the largest filter bounds the maximum
    assert all(len(set(p)) == len(p) for p in per)
    assert plan_moves([[(1, 100)], [(2, 90)]]) == []  # no move lowers the maximum
    assert plan_moves([[(1, 10), (2, 10)]]) == []      # one rank


def test_snapshot_header():
    from esthera_b200.sharding import snapshot_header
    snap = _fake_snapshot(3, 4096, 512, 1)
    assert snapshot_header(snap) == (3, 4096, 8)
    with pytest.raises(ValueError):
        snapshot_header(b"\0" * 64)


def _mover(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
        from esthera_b200.sharding import plan_moves, recv_filter, send_filter, snapshot_header
        filters = {10: (0, 2048), 11: (3, 4096), 12: (1, 1024), 13: (4, 512)}  # id: (model, particles)
        loads = [[(f, n) for f, (_, n) in filters.items()], []]
        moves = plan_moves(loads)
        ok = bool(moves)
        for src, dst, fid in moves:
            model, n = filters[fid]
            want = _fake_snapshot(model, n, 256, fid)
            if rank == src:
                send_filter(dist, want, dst)
            elif rank == dst:
                got = recv_filter(dist, src)
                ok = ok and got == want and snapshot_header(got) == (model, n, n // 256)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, ok))
    except Exception as e:  # report, never hang the parent
        q.put((rank, repr(e)))


def test_move_filters_between_ranks():
    """Rebalancing plan + snapshot transport over 2 gloo ranks: every moved
    filter's snapshot arrives byte for byte with its header intact."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_mover, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert all(v is True for v in res.values()), res


def _oracle_shard_rank(rank, world, port, N, m, t, res, steps, q):
    """One rank of the oracle filter split by rows: its own sub-filters with
    their whole-filter streams, the halos of the neighbouring ranks through
    halo_exchange, the exchange applied to its sorted copy, then resampling."""
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
        import workload as Wk
        from esthera_b200.sharding import TorusShard, halo_exchange
        p = Wk.params(0, 5)
        control, meas, _, _ = Wk.make_trace(0, p, 5, steps)
        md = O.model_from_params(0, p)
        sh = TorusShard(N, m, t, world, rank)
        f = O.Filter(md, m, sh.num_subfilters, t, O.EXCH_NONE, res, O.RNG_SUBFILTER, 96, 4, 1, 1.0, 0xF000000D, 0,
                     np.array(p.init_state[:3], np.float32))
        f.set_stream_offset(sh.first_subfilter)
        tt = lambda h: (torch.from_numpy(np.ascontiguousarray(h[0])), torch.from_numpy(np.ascontiguousarray(h[1])))
        for k in range(steps):
            f.sample(control[k], meas[k], threads=1)
            s, kk = f.sorted()
            up, down = sh.halos_out(s, kk)
            fu, fd = halo_exchange(dist, sh, tt(up), tt(down))
            es, ek = sh.apply_exchange(s, kk, (fu[0].numpy(), fu[1].numpy()), (fd[0].numpy(), fd[1].numpy()))
            f.set_sorted(es, ek)
            f.resample(threads=1)
        out = (rank, sh.first_subfilter, f.state())
        f.close()
        dist.barrier()
        dist.destroy_process_group()
        q.put(out)
    except Exception as e:  # report, never hang the parent
        q.put((rank, repr(e), None))


@pytest.mark.parametrize("world,N,t,res", [(2, 64, 2, 1), (2, 128, 1, 2), (4, 128, 1, 0)])
def test_sharded_oracle_filter_matches_whole(world, N, t, res):
    """The row-sharded step (per-rank streams at their whole-filter offsets,
    halo rows between neighbouring ranks, no collective over particles) gives
    the whole filter's particles bit for bit, through gloo ranks on CPU."""
    import multiprocessing as mp
    import oracle as O
    import workload as Wk
    m, steps = 64, 4
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_oracle_shard_rank, args=(r, world, port, N, m, t, res, steps, q))
             for r in range(world)]
    for pr in procs:
        pr.start()
    got = [q.get(timeout=240) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
    for g in got:
        assert g[2] is not None, g[1]
    p = Wk.params(0, 5)
    control, meas, _, _ = Wk.make_trace(0, p, 5, steps)
    md = O.model_from_params(0, p)
    f = O.Filter(md, m, N, t, O.EXCH_TORUS, res, O.RNG_SUBFILTER, 96, 4, 1, 1.0, 0xF000000D, 0,
                 np.array(p.init_state[:3], np.float32))
    for k in range(steps):
        f.step(control[k], meas[k], threads=1)
    whole = f.state()
    f.close()
    for rank, b0, st in got:
        assert np.array_equal(st, whole[:, b0 * m:b0 * m + st.shape[1]]), rank
