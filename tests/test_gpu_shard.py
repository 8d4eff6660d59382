"""A filter's torus rows spread over shards (pf_shard_*) step exactly like the
whole filter on one GPU: particles, sorted copies and estimates bit for bit,
for every resampler, through the device halo copy and through host buffers,
and with the shards as two gloo ranks (esthera_b200.sharding.ShardedFilter)."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UNI, ARM, BEACON = 0, 1, 3


def _setup(E, model, seed=3, steps=6):
    if model == UNI:
        p = E.unicycle_params(seed)
    elif model == ARM:
        p = E.dharm_params(seed)
    else:
        p = E.beacon_params()
    inputs, _ = E.make_trace(model, p, seed, steps)
    return p, inputs


def _cfg(E, res, m=128, N=128, t=2, **kw):
    return E.default_config(particles_per_subfilter=m, num_subfilters=N, num_transfer=t, exchange=E.EXCHANGE_TORUS,
                            resampler=res, rng=E.RNG_SUBFILTER, pipeline=E.PIPELINE_SPLIT, seed=17, **kw)


def _same_estimate(a, b):
    return (np.array_equal(a["mean"], b["mean"]) and a["log_norm"] == b["log_norm"]
            and np.array_equal(a["best"], b["best"]) and a["best_key"] == b["best_key"]
            and a["best_subfilter"] == b["best_subfilter"] and a["step"] == b["step"])


def _check_against_whole(E, whole, shards, m):
    P = whole.particles()
    s_all, k_all = whole.sorted()
    for s in shards:
        lo = s.first_subfilter * m
        hi = lo + s.N * m
        assert np.array_equal(s.particles(), P[:, lo:hi])
        ss, ks = s.sorted()
        assert np.array_equal(ss, s_all[:, lo:hi]) and np.array_equal(ks, k_all[lo:hi])


@pytest.mark.parametrize("model", [UNI, ARM, BEACON])
@pytest.mark.parametrize("res", [0, 1, 2])
def test_two_shards_equal_the_whole_filter(gpu, model, res):
    E = gpu
    p, inputs = _setup(E, model)
    cfg = _cfg(E, res)
    whole = E.ParticleFilter(model, p, config=cfg)
    dx, dy = whole.info()["torus"]
    assert (dx, dy) == (8, 16)
    shards = [E.FilterShard(model, p, 0, 8, config=cfg), E.FilterShard(model, p, 8, 16, config=cfg)]
    assert [s.first_subfilter for s in shards] == [0, 64] and shards[0].num_groups == 2
    for k in range(len(inputs)):
        want = whole.step(inputs[k])
        got = E.shard_step(shards, inputs[k])
        assert _same_estimate(got, want), (k, got, want)
        _check_against_whole(E, whole, shards, 128)


def test_three_uneven_shards_and_host_halos(gpu):
    """Rows [0,4) [4,12) [12,16): the 32-sub-filter shards' halo rows come from
    both neighbours; the host-buffer route equals the device copy."""
    E = gpu
    p, inputs = _setup(E, UNI, seed=5, steps=5)
    cfg = _cfg(E, 1, t=3)
    whole = E.ParticleFilter(UNI, p, config=cfg)
    a = [E.FilterShard(UNI, p, r0, r1, config=cfg) for r0, r1 in ((0, 4), (4, 12), (12, 16))]
    b = [E.FilterShard(UNI, p, r0, r1, config=cfg) for r0, r1 in ((0, 4), (4, 12), (12, 16))]
    for k in range(len(inputs)):
        want = whole.step(inputs[k])
        got_a = E.shard_step(a, inputs[k])
        # the same step through host buffers (as between processes)
        for s in b:
            s.sample(inputs[k])
        out = [(s.halo_out(0), s.halo_out(1)) for s in b]
        n = len(b)
        for i, s in enumerate(b):
            s.halo_in(0, out[(i - 1) % n][0])  # the upper neighbour's last row
            s.halo_in(1, out[(i + 1) % n][1])  # the lower neighbour's first row
        for s in b:
            s.resample()
        parts = [s.group_rows() for s in b]
        got_b = b[1].estimate(np.concatenate([q[0] for q in parts]), np.concatenate([q[1] for q in parts]))
        assert _same_estimate(got_a, want) and _same_estimate(got_b, want)
        _check_against_whole(E, whole, a, 128)
        _check_against_whole(E, whole, b, 128)


def test_shard_arguments(gpu):
    E = gpu
    p, inputs = _setup(E, UNI, steps=1)
    cfg = _cfg(E, 1)
    with pytest.raises(E.PFError) as e:
        E.FilterShard(UNI, p, 0, 16, config=cfg)  # every row: the whole filter
    assert e.value.status == E.PF_ERR_INVALID
    with pytest.raises(E.PFError) as e:
        E.FilterShard(UNI, p, 1, 8, config=cfg)  # starts at sub-filter 8
    assert e.value.status == E.PF_ERR_UNSUPPORTED
    with pytest.raises(E.PFError):
        E.FilterShard(UNI, p, 0, 8, config=_cfg(E, 1, exchange_period=2))
    ring = _cfg(E, 1)
    ring.exchange = E.EXCHANGE_RING
    with pytest.raises(E.PFError) as e:
        E.FilterShard(UNI, p, 0, 8, config=ring)
    assert e.value.status == E.PF_ERR_UNSUPPORTED
    a, b, c = (E.FilterShard(UNI, p, r0, r1, config=cfg) for r0, r1 in ((0, 4), (4, 8), (8, 16)))
    with pytest.raises(E.PFError) as e:
        a.step(inputs[0])  # a shard has no whole step
    assert e.value.status == E.PF_ERR_INVALID
    a.sample(inputs[0])
    with pytest.raises(E.PFError):
        a.send_halo(0, c)  # c is not below a
    a.send_halo(0, b)
    a.send_halo(1, c)  # c's last row (15) wraps to a's first row
    with pytest.raises(ValueError):
        a.halo_in(0, np.zeros(3, np.uint8))
    with pytest.raises(E.PFError):
        a.estimate(np.zeros((2, E.SHARD_ROW)), np.zeros((2, 3), np.float32))  # needs all 4 groups


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, res, steps, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
        import esthera_b200 as E
        from esthera_b200.sharding import ShardedFilter
        p, inputs = _setup(E, UNI, seed=9, steps=steps)
        f = ShardedFilter(dist, UNI, p, config=_cfg(E, res))
        ests = [f.step(inputs[k]) for k in range(steps)]
        out = (rank, f.shard.first_subfilter, f.particles(), np.array(ests))
        f.close()
        dist.barrier()
        dist.destroy_process_group()
        q.put(out)
    except Exception as e:  # report, never hang the parent
        q.put((rank, repr(e), None, None))


@pytest.mark.parametrize("res", [1, 2])
def test_two_gloo_ranks_equal_the_whole_filter(gpu, res):
    """Two processes, each one shard (on the same GPU: no kernel waits on
    another process), halos and group rows over gloo."""
    import multiprocessing as mp
    E = gpu
    steps = 4
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, res, steps, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    got = [q.get(timeout=300) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
    for g in got:
        assert g[2] is not None, g[1]
    p, inputs = _setup(E, UNI, seed=9, steps=steps)
    whole = E.ParticleFilter(UNI, p, config=_cfg(E, res))
    want = [whole.step(inputs[k]) for k in range(steps)]
    P = whole.particles()
    for rank, b0, parts, ests in got:
        assert np.array_equal(parts, P[:, b0 * 128:b0 * 128 + parts.shape[1]])
        for x, y in zip(ests, want):
            assert _same_estimate(x, y)
