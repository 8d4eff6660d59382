"""The serving form (pf_server_*) on the GPU through the C ABI: continuous
batching of updates from many resident filters of mixed models and sizes.
Every filter's results are the same alone and in the mix, and the same as a
pf_filter with that seed; admission follows the HBM budget."""
import numpy as np
import pytest

UNI, ARM = 0, 1
CFG = dict(particles_per_subfilter=256, particles_per_thread=4, num_transfer=2, exchange=1)


def trace(E, model, seed, steps):
    p = E.unicycle_params(seed) if model == UNI else E.dharm_params(seed)
    inputs, truth = E.make_trace(model, p, seed, steps)
    return p, inputs, truth


def run_alone(E, model, p, n, seed, inputs):
    srv = E.Server(1 << 30, 4, **CFG)
    fid = srv.open(model, p, n, seed)
    out = []
    for k in range(len(inputs)):
        srv.update(fid, inputs[k], tag=k)
        assert srv.launch() == 1
        r = srv.poll()
        assert len(r) == 1 and r[0]["filter"] == fid and r[0]["tag"] == k and r[0]["step"] == k + 1
        out.append(r[0]["estimate"])
    a, s, keys = srv.particles(fid, n)
    srv.close()
    return out, a


def same(x, y):
    return (np.array_equal(x["mean"], y["mean"]) and x["log_norm"] == y["log_norm"] and
            np.array_equal(x["best"], y["best"]) and x["best_key"] == y["best_key"] and
            x["best_subfilter"] == y["best_subfilter"])


@pytest.mark.gpu
def test_server_filter_equals_pf_filter(gpu):
    """A served filter == pf_create with the same seed (split pipeline)."""
    E = gpu
    for model, n, seed in [(UNI, 4096, 11), (ARM, 2048, 12)]:
        p, inputs, _ = trace(E, model, seed, 6)
        served, parts = run_alone(E, model, p, n, seed, inputs)
        f = E.ParticleFilter(model, p, pipeline=E.PIPELINE_SPLIT, num_subfilters=n // 256, seed=seed, **CFG)
        for k in range(6):
            assert same(served[k], f.step(inputs[k])), (model, k)
        assert np.array_equal(parts, f.particles())


@pytest.mark.gpu
def test_server_same_alone_and_in_mix(gpu):
    """Filter X's updates interleaved with other filters' (both models, uneven
    sizes, filters opened and closed meanwhile) give X's results alone."""
    E = gpu
    steps = 8
    px, inx, _ = trace(E, UNI, 101, steps)
    alone, parts_alone = run_alone(E, UNI, px, 3072, 101, inx)

    srv = E.Server(1 << 30, 16, **CFG)
    rng = np.random.default_rng(5)
    others = []
    for j, (model, n) in enumerate([(ARM, 1024), (UNI, 8192), (ARM, 4096), (UNI, 256)]):
        p, inp, _ = trace(E, model, 200 + j, 40)
        others.append([srv.open(model, p, n, 200 + j), inp, 0])
    x = srv.open(UNI, px, 3072, 101)
    got = {}
    k = 0
    late = None
    while len(got) < steps:
        if k < steps:
            srv.update(x, inx[k], tag=1000 + k)
            k += 1
        for o in others:
            for _ in range(int(rng.integers(0, 3))):  # 0-2 queued updates per round
                if o[2] < 40:
                    srv.update(o[0], o[1][o[2]], tag=o[2])
                    o[2] += 1
        if late is None and k == 4:  # a filter admitted mid-run
            p, inp, _ = trace(E, ARM, 300, 10)
            late = srv.open(ARM, p, 2048, 300)
            for q in range(5):
                srv.update(late, inp[q])
        srv.launch()
        for r in srv.poll():
            if r["filter"] == x:
                got[int(r["tag"]) - 1000] = r["estimate"]
        if k == 6 and others[0] is not None and srv.stats()["in_flight"] == 0:
            srv.close_filter(others[0][0])  # closed while others keep running
            others = others[1:]
    # drain
    while srv.stats()["queued_updates"] > 0:
        srv.launch()
        srv.poll()
    for q in range(steps):
        assert same(got[q], alone[q]), q
    a, _, _ = srv.particles(x, 3072)
    assert np.array_equal(a, parts_alone)


@pytest.mark.gpu
def test_server_admission_by_budget(gpu):
    E = gpu
    srv = E.Server(1, 1, **CFG)  # footprint query only
    fp = srv.footprint(UNI, 65536)
    srv.close()
    assert fp > 65536 * 3 * 4 * 2
    srv = E.Server(int(fp * 2.5), 8, **CFG)
    p = E.unicycle_params(3)
    a = srv.open(UNI, p, 65536, 1)
    b = srv.open(UNI, p, 65536, 2)
    with pytest.raises(E.PFError) as ei:
        srv.open(UNI, p, 65536, 3)
    assert ei.value.status == E.PF_ERR_ADMISSION
    assert srv.stats()["bytes_in_use"] == 2 * fp
    srv.close_filter(a)
    c = srv.open(UNI, p, 65536, 3)
    assert c >= 0 and srv.stats()["open_filters"] == 2
    with pytest.raises(E.PFError) as ei:
        srv.open(UNI, p, 1000, 4)  # not a multiple of m
    assert ei.value.status == E.PF_ERR_INVALID


@pytest.mark.gpu
def test_server_one_update_per_filter_per_batch(gpu):
    E = gpu
    srv = E.Server(1 << 30, 4, **CFG)
    p, inp, _ = trace(E, UNI, 9, 5)
    a = srv.open(UNI, p, 1024, 9)
    b = srv.open(UNI, p, 2048, 10)
    for k in range(3):
        srv.update(a, inp[k], tag=k)
    srv.update(b, inp[0], tag=7)
    assert srv.launch() == 2
    assert srv.launch() == 0  # a batch is in flight
    r = srv.poll()
    assert sorted((int(x["filter"]), int(x["tag"])) for x in r) == sorted([(a, 0), (b, 7)])
    assert srv.stats()["queued_updates"] == 2
    assert srv.launch() == 1
    r = srv.poll()
    assert len(r) == 1 and r[0]["tag"] == 1 and r[0]["step"] == 2


@pytest.mark.gpu
def test_server_normalisation_vs_fp64(gpu):
    E = gpu
    srv = E.Server(1 << 30, 4, **CFG)
    for model, n, seed in [(UNI, 16384, 21), (ARM, 4096, 22)]:
        p, inp, _ = trace(E, model, seed, 3)
        fid = srv.open(model, p, n, seed)
        for k in range(3):
            srv.update(fid, inp[k])
            srv.launch()
            r = srv.poll()
        _, _, keys = srv.particles(fid, n)
        kk = keys.astype(np.float64)
        mx = kk.max()
        ln = mx + np.log(np.sum(np.exp(kk - mx)))
        assert abs(r[0]["estimate"]["log_norm"] - ln) <= 1e-6 * max(1.0, abs(ln))


@pytest.mark.gpu
def test_server_snapshot_restore_moves_a_filter(gpu):
    """A filter snapshotted after 3 updates and restored into a filter of another
    server (same model, parameters and count, different seed and slot) gives
    the source's next results bit for bit; busy and mismatched filters are refused."""
    E = gpu
    p, inputs, _ = trace(E, UNI, 77, 7)
    src = E.Server(1 << 30, 4, **CFG)
    a = src.open(UNI, p, 2048, 77)
    for k in range(3):
        src.update(a, inputs[k], tag=k)
        src.launch()
        src.poll()
    snap = src.snapshot(a)
    src.update(a, inputs[3], tag=3)
    with pytest.raises(E.PFError) as ei:
        src.snapshot(a)  # an update queued
    assert ei.value.status == E.PF_ERR_BUSY
    want = []
    for k in range(3, 7):
        if k > 3:
            src.update(a, inputs[k], tag=k)
        src.launch()
        want.append(src.poll()[0])
    dst = E.Server(1 << 30, 4, **CFG)
    dst.open(ARM, E.dharm_params(3), 1024, 5)  # another slot in use first
    b = dst.open(UNI, p, 2048, 991)
    small = dst.open(UNI, p, 1024, 991)
    with pytest.raises(E.PFError) as ei:
        dst.restore(small, snap)
    assert ei.value.status == E.PF_ERR_INVALID
    with pytest.raises(E.PFError) as ei:
        dst.restore(b, snap[: len(snap) // 2])  # a truncated transfer is refused before it is read
    assert ei.value.status == E.PF_ERR_INVALID
    dst.restore(b, snap)
    for k in range(3, 7):
        dst.update(b, inputs[k], tag=k)
        dst.launch()
        r = dst.poll()[0]
        w = want[k - 3]
        assert r["step"] == w["step"] == k + 1
        assert same(r["estimate"], w["estimate"]), k
    assert np.array_equal(dst.particles(b, 2048)[0], src.particles(a, 2048)[0])
    src.close()
    dst.close()


@pytest.mark.gpu
def test_server_cancel_queued_updates(gpu):
    """A request cancelled on the host: closing a filter drops its queued
    updates (no result comes back for them), is refused while one of its
    updates is on the GPU, leaves the other filters' results unchanged, and
    its slot serves a new filter from a clean state."""
    E = gpu
    p, inputs, _ = trace(E, UNI, 61, 4)
    q, qin, _ = trace(E, UNI, 62, 4)
    alone, _ = run_alone(E, UNI, q, 1024, 62, qin)
    srv = E.Server(1 << 30, 4, **CFG)
    a = srv.open(UNI, p, 2048, 61)
    b = srv.open(UNI, q, 1024, 62)
    srv.update(a, inputs[0], tag=0)
    srv.update(b, qin[0], tag=100)
    assert srv.launch() == 2
    with pytest.raises(E.PFError) as ei:
        srv.close_filter(a)  # its update is on the GPU
    assert ei.value.status == E.PF_ERR_BUSY
    got_b = {}
    for r in srv.poll():
        if r["filter"] == b:
            got_b[int(r["tag"]) - 100] = r["estimate"]
    for k in (1, 2, 3):
        srv.update(a, inputs[k], tag=k)
    assert srv.stats()["queued_updates"] == 3
    srv.close_filter(a)  # cancels its three queued updates
    assert srv.stats()["queued_updates"] == 0 and srv.stats()["open_filters"] == 1
    for k in (1, 2, 3):
        srv.update(b, qin[k], tag=100 + k)
        assert srv.launch() == 1
        rs = srv.poll()
        assert len(rs) == 1 and rs[0]["filter"] == b
        got_b[k] = rs[0]["estimate"]
    for k in range(4):
        assert same(got_b[k], alone[k]), k
    # the freed slot serves a new filter from its initial state
    c = srv.open(UNI, p, 2048, 61)
    srv.update(c, inputs[0], tag=7)
    srv.launch()
    rc = srv.poll()[0]
    assert rc["filter"] == c and rc["step"] == 1
    first, _ = run_alone(E, UNI, p, 2048, 61, inputs[:1])
    assert same(rc["estimate"], first[0])
    srv.close()
