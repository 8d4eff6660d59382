"""Batched filters of uneven particle counts (pf_batch_*) on the GPU through the
C ABI: every filter of a batch reproduces, bit for bit, the same filter run
alone (pf_create with the filter's stream offset) -- host-stepped and
graph-replayed, with exchange every step or every few steps, ring or torus."""
import numpy as np
import pytest

UNI = 0


def batch_setup(E, counts, steps, seed0=4):
    params = [E.unicycle_params(seed0 + i) for i in range(len(counts))]
    traces = [E.make_trace(UNI, p, seed0 + i, steps) for i, p in enumerate(params)]
    inputs = np.stack([t[0] for t in traces])          # [F, steps]
    truth = np.stack([t[1] for t in traces])           # [F, steps, S]
    return params, inputs, truth


def single(E, p, cfg, stream_offset, n, m):
    return E.ParticleFilter(UNI, p, pipeline=E.PIPELINE_SPLIT, particles_per_subfilter=m, num_subfilters=n // m,
                            stream_offset=stream_offset, **cfg)


def same_estimate(x, y):
    return (np.array_equal(x["mean"], y["mean"]) and x["log_norm"] == y["log_norm"] and
            np.array_equal(x["best"], y["best"]) and x["best_key"] == y["best_key"] and
            x["best_subfilter"] == y["best_subfilter"] and x["step"] == y["step"])


CASES = [
    # m, ppt, exchange, t, period, resampler, counts
    (256, 2, 1, 2, 1, 1, [256, 512, 1024, 256, 768, 2304]),
    (128, 4, 1, 3, 2, 0, [128, 640, 384, 1024]),
    (256, 4, 2, 2, 1, 2, [1024, 2048, 512, 4096]),   # torus: N = 4, 8, 2, 16
    (256, 2, 2, 1, 4, 1, [1536, 256, 4096]),          # N = 6 (2x3), 1, 16
]


@pytest.mark.gpu
@pytest.mark.parametrize("m,ppt,exch,t,period,res,counts", CASES)
def test_batch_equals_single_filters(gpu, m, ppt, exch, t, period, res, counts):
    E = gpu
    steps = 7
    params, inputs, _ = batch_setup(E, counts, steps)
    cfg = dict(num_transfer=t, exchange=exch, resampler=res, exchange_period=period, particles_per_thread=ppt)
    B = E.FilterBatch(UNI, params, counts, particles_per_subfilter=m, **cfg)
    info = B.info()
    assert info["num_filters"] == len(counts) and info["total_particles"] == sum(counts)
    best = [B.step(inputs[:, k]) for k in range(steps)]
    for f, n in enumerate(counts):
        fi = B.filter_info(f)
        assert fi["num_subfilters"] == n // m
        s = single(E, params[f], cfg, fi["stream_offset"], n, m)
        for k in range(steps):
            e = s.step(inputs[f, k])
            assert same_estimate(best[k][f], e), (f, k)
        assert np.array_equal(B.particles(f), s.particles()), f


@pytest.mark.gpu
@pytest.mark.parametrize("m,exch,t,res", [(1024, 1, 2, 1), (512, 2, 1, 2), (1024, 0, 0, 0)])
def test_mixed_subfilter_sizes_equal_single_filters(gpu, m, exch, t, res):
    """m is an upper bound: each filter runs the largest power-of-two
    sub-filter size that divides its count (and fits the torus), in one launch
    group per size, and still equals the same filter run alone."""
    E = gpu
    counts = [256, 768, 1536, 4096, 5120, 96, 1024]
    steps = 5
    params, inputs, _ = batch_setup(E, counts, steps)
    cfg = dict(num_transfer=t, exchange=exch, resampler=res, particles_per_thread=4)
    B = E.FilterBatch(UNI, params, counts, particles_per_subfilter=m, **cfg)
    shapes = [B.filter_shape(f) for f in range(len(counts))]
    for n, (mf, ppt) in zip(counts, shapes):
        assert mf <= m and n % mf == 0 and (2 * mf > m or n % (2 * mf) != 0 or exch == 2)
    assert len({mf for mf, _ in shapes}) >= 3
    best = [B.step(inputs[:, k]) for k in range(steps)]
    for f, n in enumerate(counts):
        mf, ppt = shapes[f]
        fi = B.filter_info(f)
        assert fi["num_subfilters"] == n // mf
        c = dict(cfg, particles_per_thread=ppt)
        s = single(E, params[f], c, fi["stream_offset"], n, mf)
        for k in range(steps):
            assert same_estimate(best[k][f], s.step(inputs[f, k])), (f, k)
        assert np.array_equal(B.particles(f), s.particles()), f


@pytest.mark.gpu
@pytest.mark.parametrize("period", [1, 2])
def test_batch_graph_equals_host_steps(gpu, period):
    """pf_batch_submit (graph of many steps, device counter) == pf_batch_step."""
    import torch
    E = gpu
    counts = [256, 1280, 512, 3072, 256]
    steps = 9
    params, inputs, _ = batch_setup(E, counts, steps)
    cfg = dict(particles_per_subfilter=256, num_transfer=2, exchange=1, exchange_period=period)
    A = E.FilterBatch(UNI, params, counts, **cfg)
    ea = [A.step(inputs[:, k]) for k in range(steps)]
    B = E.FilterBatch(UNI, params, counts, **cfg)
    cap = steps
    d_in = torch.from_numpy(np.ascontiguousarray(inputs).view(np.uint8).reshape(-1).copy()).cuda()
    d_est = torch.zeros(len(counts) * cap * E.ESTIMATE_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    # two submissions: 5 steps (one 5-step graph) then 4 more would restart the
    # counter, so run all 9 at once and also check the poll/synchronize calls
    B.submit(d_in.data_ptr(), d_est.data_ptr(), cap, steps)
    B.synchronize()
    assert B.poll()
    est = d_est.cpu().numpy().view(E.ESTIMATE_DTYPE).reshape(len(counts), cap)
    for f in range(len(counts)):
        assert np.array_equal(A.particles(f), B.particles(f)), f
        for k in range(steps):
            x, y = est[f, k], ea[k][f]
            assert np.array_equal(x["mean"], y["mean"]) and x["best_key"] == y["best_key"], (f, k)
            assert x["step"] == k + 1


@pytest.mark.gpu
def test_batch_submit_split_into_graphs(gpu):
    """A run longer than one captured graph (300 steps: a 256-step graph plus
    single-step replays) matches host stepping at the end."""
    import torch
    E = gpu
    counts = [256, 512]
    steps = 300
    params, inputs, _ = batch_setup(E, counts, steps)
    cfg = dict(particles_per_subfilter=128, num_transfer=1, exchange=1, exchange_period=4)
    A = E.FilterBatch(UNI, params, counts, **cfg)
    for k in range(steps):
        ea = A.step(inputs[:, k])
    B = E.FilterBatch(UNI, params, counts, **cfg)
    d_in = torch.from_numpy(np.ascontiguousarray(inputs).view(np.uint8).reshape(-1).copy()).cuda()
    d_est = torch.zeros(len(counts) * steps * E.ESTIMATE_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    B.submit(d_in.data_ptr(), d_est.data_ptr(), steps, steps)
    B.synchronize()
    est = d_est.cpu().numpy().view(E.ESTIMATE_DTYPE).reshape(len(counts), steps)
    for f in range(len(counts)):
        assert np.array_equal(A.particles(f), B.particles(f))
        assert np.array_equal(est[f, -1]["mean"], ea[f]["mean"])


@pytest.mark.gpu
def test_batch_tracks(gpu):
    """Every filter of a mixed-size batch tracks its own seeded trajectory."""
    E = gpu
    counts = [256, 512, 2048, 8192]
    steps = 60
    params, inputs, truth = batch_setup(E, counts, steps, seed0=40)
    B = E.FilterBatch(UNI, params, counts, particles_per_subfilter=256, num_transfer=2, exchange=1)
    est = np.stack([B.step(inputs[:, k])["mean"][:, :2] for k in range(steps)], 1)  # [F, steps, 2]
    err = np.sqrt(((est[:, 10:] - truth[:, 10:, :2]) ** 2).sum(-1).mean(-1))
    assert np.all(err < 0.5), err


def test_batch_rejects_bad_shapes(E):
    import esthera_b200 as EB
    p = [EB.UnicycleParams() for _ in range(2)]
    for x in p:
        x.num_landmarks = 4
        x.sigma_range = 0.2
        x.sigma_bearing = 0.05
    with pytest.raises(EB.PFError) as ei:
        EB.FilterBatch(UNI, p, [256, 300], particles_per_subfilter=256)
    assert ei.value.status == EB.PF_ERR_INVALID
    with pytest.raises(EB.PFError) as ei:
        EB.FilterBatch(UNI, p, [256, 512], particles_per_subfilter=256, exchange=3)
    assert ei.value.status == EB.PF_ERR_UNSUPPORTED
    with pytest.raises(EB.PFError) as ei:
        EB.FilterBatch(UNI, p, [256, 5 * 32], particles_per_subfilter=256, exchange=2)  # 5 sub-filters of 32
    assert ei.value.status == EB.PF_ERR_INVALID


@pytest.mark.gpu
def test_batch_autotune(gpu):
    """The autotuner runs every buildable candidate, reports the others with
    their status, and picks the fastest accepted one."""
    E = gpu
    counts = [256, 768, 1536, 512]
    steps = 12
    params, inputs, truth = batch_setup(E, counts, steps)
    best, rows = E.batch_autotune(UNI, params, counts, inputs, truth, m_list=(128, 256, 512, 1024), ppt_list=(2, 4),
                                  tpp_list=(1, 2), period_list=(1, 2), burn_in=2, rmse_tol=0.5, num_transfer=1,
                                  exchange=1)
    assert len(rows) == 4 * 2 * 2 * 2
    for r in rows:  # m = 512 / 1024 cap each filter's sub-filters at a size dividing its count
        assert r["status"] == E.PF_OK and r["ms_per_step"] > 0 and np.isfinite(r["rmse"])
    ok = [r for r in rows if r["accepted"]]
    pick = max(ok, key=lambda r: r["particle_steps_per_s"])
    assert (best.particles_per_subfilter, best.particles_per_thread, best.threads_per_particle,
            best.exchange_period) == (pick["particles_per_subfilter"], pick["particles_per_thread"],
                                      pick["threads_per_particle"], pick["exchange_period"])


@pytest.mark.gpu
def test_batch_normalisation_vs_fp64(gpu):
    """Each filter's log normalisation (FP64 accumulation of FP32 weights)
    against an FP64 log-sum-exp of the same sorted keys on the host."""
    E = gpu
    counts = [256, 4096, 1280, 65536]
    params, inputs, _ = batch_setup(E, counts, 3)
    B = E.FilterBatch(UNI, params, counts, particles_per_subfilter=256, num_transfer=2, exchange=1)
    for k in range(3):
        est = B.step(inputs[:, k])
    for f in range(len(counts)):
        _, keys = B.sorted(f)
        kk = keys.astype(np.float64)
        mx = kk.max()
        ln = mx + np.log(np.sum(np.exp(kk - mx)))
        assert abs(est[f]["log_norm"] - ln) <= 1e-6 * max(1.0, abs(ln)), (f, est[f]["log_norm"], ln)


@pytest.mark.gpu
def test_batch_rmse_vs_fp64_oracle(gpu, O):
    """Tracking error of batched filters against the oracle's FP64 run of the
    same filters (same streams: each filter's oracle starts at its batch
    stream offset): the mean RMSE over the filters agrees within 5 % + 0.005.
    The batched results equal the plain path's bit for bit, so the plain path
    has the same error."""
    E = gpu
    counts = [2048, 4096, 8192, 2048, 4096, 8192]
    steps = 60
    params, inputs, truth = batch_setup(E, counts, steps, seed0=21)
    cfg = dict(num_transfer=2, exchange=1, resampler=1, particles_per_thread=4)
    B = E.FilterBatch(UNI, params, counts, particles_per_subfilter=256, **cfg)
    est = np.stack([B.step(inputs[:, k]) for k in range(steps)], axis=1)  # [F, steps]
    seed = B.config.seed
    g, o = [], []
    for f, n in enumerate(counts):
        mf, ppt = B.filter_shape(f)
        md = O.model_from_params(UNI, params[f])
        of = O.Filter(md, mf, n // mf, 2, O.EXCH_RING, 1, O.RNG_SUBFILTER, 96, ppt, 1, 1.0, seed, 0,
                      np.array(params[f].init_state[:3], np.float32))
        of.set_stream_offset(B.filter_info(f)["stream_offset"])
        om = np.array([of.step(inputs[f, k]["control"], inputs[f, k]["meas"])[0].mean[:2] for k in range(steps)])
        of.close()
        gm = np.array([e["mean"][:2] for e in est[f]])
        g.append(np.sqrt(np.mean(np.sum((gm[10:] - truth[f, 10:, :2]) ** 2, axis=1))))
        o.append(np.sqrt(np.mean(np.sum((om[10:] - truth[f, 10:, :2]) ** 2, axis=1))))
    g, o = float(np.mean(g)), float(np.mean(o))
    assert abs(g - o) <= 0.05 * o + 0.005, (g, o)
