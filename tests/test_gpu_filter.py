"""The whole filter step on the GPU through the C ABI: phased (one kernel per
reference phase) vs fused pipelines, CUDA-graph replay vs host stepping, the
oracle's whole-filter restatement, tracking accuracy (RMSE against the seeded
ground truth) and size-independent properties at the 2^20-particle shape."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UNI, ARM, REF = 0, 1, 2


def uni_setup(seed=1, steps=100):
    import esthera_b200 as E
    p = E.unicycle_params(seed)
    inputs, truth = E.make_trace(UNI, p, seed, steps)
    return p, inputs, truth


def run(E, model, params, inputs, steps=None, **cfg):
    f = E.ParticleFilter(model, params, **cfg)
    ests = [f.step(inputs[k]) for k in range(steps or len(inputs))]
    return f, ests


@pytest.mark.parametrize("res", [0, 1, 2])
@pytest.mark.parametrize("exch,t", [(0, 0), (1, 3), (2, 2), (3, 4)])
def test_phased_equals_split(gpu, res, exch, t):
    """One kernel per reference phase vs the two-kernel split pipeline (reference RNG layout)."""
    E = gpu
    p, inputs, _ = uni_setup()
    common = dict(particles_per_subfilter=256, num_subfilters=16, num_transfer=t, exchange=exch, resampler=res,
                  rng=E.RNG_REFLAYOUT, mtgp_streams=96)
    fa, ea = run(E, UNI, p, inputs, 6, pipeline=E.PIPELINE_PHASED, **common)
    fb, eb = run(E, UNI, p, inputs, 6, pipeline=E.PIPELINE_SPLIT, **common)
    assert fa.info()["pipeline"] == E.PIPELINE_PHASED and fb.info()["pipeline"] == E.PIPELINE_SPLIT
    assert np.array_equal(fa.particles(), fb.particles())
    for x, y in zip(ea, eb):
        assert x["best_subfilter"] == y["best_subfilter"] and x["best_key"] == y["best_key"]
        assert np.allclose(x["mean"], y["mean"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("m,ppt", [(128, 4), (256, 8), (512, 16), (512, 4), (256, 4), (256, 2), (64, 2)])
@pytest.mark.parametrize("res", [0, 1, 2])
@pytest.mark.parametrize("exch,t", [(0, 0), (1, 3), (2, 2), (3, 4)])
def test_fused_equals_split(gpu, m, ppt, res, exch, t):
    """The single-kernel step (one CTA per sub-filter, resampling deferred to the
    next launch) against the split pipeline with the same particles per thread."""
    E = gpu
    p, inputs, _ = uni_setup()
    common = dict(particles_per_subfilter=m, num_subfilters=16, num_transfer=t, exchange=exch, resampler=res,
                  particles_per_thread=ppt)
    fa, ea = run(E, UNI, p, inputs, 6, pipeline=E.PIPELINE_SPLIT, **common)
    fb, eb = run(E, UNI, p, inputs, 6, pipeline=E.PIPELINE_FUSED, **common)
    assert fb.info()["pipeline"] == E.PIPELINE_FUSED and fa.info()["pipeline"] == E.PIPELINE_SPLIT
    sa, ka = fa.sorted()
    sb, kb = fb.sorted()
    assert np.array_equal(ka, kb) and np.array_equal(sa, sb)
    assert np.array_equal(fa.particles(), fb.particles())
    for x, y in zip(ea, eb):
        assert x["best_subfilter"] == y["best_subfilter"] and x["best_key"] == y["best_key"]
        assert np.array_equal(x["best"], y["best"])
        assert np.allclose(x["mean"], y["mean"], rtol=1e-12, atol=1e-12)
        assert abs(x["log_norm"] - y["log_norm"]) <= 1e-12 * abs(x["log_norm"])


@pytest.mark.parametrize("model,m,N,ppt", [(ARM, 256, 4096, 2), (UNI, 512, 16384, 4)])
def test_fused_equals_split_many_groups(gpu, model, m, N, ppt):
    """More groups of 32 sub-filters than the resampling kernel stages in one
    round (the DH arm's 128 group rows against 64 per round at m = 256, the
    unicycle's 512 against 256 at m = 512): the split pipeline's final combine
    reads them in several windows, the single-kernel step's in chunks from
    global memory; the estimates agree to the last bit of the FP64 sums."""
    E = gpu
    if model == UNI:
        p, inputs, _ = uni_setup(steps=3)
    else:
        p = E.dharm_params(3)
        inputs, _ = E.make_trace(ARM, p, 3, 3)
    common = dict(particles_per_subfilter=m, num_subfilters=N, num_transfer=1, exchange=E.EXCHANGE_TORUS,
                  resampler=E.RESAMPLE_SYSTEMATIC, particles_per_thread=ppt)
    fa, ea = run(E, model, p, inputs, 3, pipeline=E.PIPELINE_SPLIT, **common)
    fb, eb = run(E, model, p, inputs, 3, pipeline=E.PIPELINE_FUSED, **common)
    assert fb.info()["pipeline"] == E.PIPELINE_FUSED and fa.info()["pipeline"] == E.PIPELINE_SPLIT
    assert np.array_equal(fa.particles(), fb.particles())
    for x, y in zip(ea, eb):
        assert x["best_subfilter"] == y["best_subfilter"] and x["best_key"] == y["best_key"]
        assert np.array_equal(x["best"], y["best"])
        assert np.array_equal(x["mean"], y["mean"]) and x["log_norm"] == y["log_norm"]
    fa.close()
    fb.close()


@pytest.mark.parametrize("rng_mode", [0, 1])
@pytest.mark.parametrize("res", [0, 1, 2])
def test_first_step_vs_oracle(gpu, O, rng_mode, res):
    E = gpu
    p, inputs, _ = uni_setup()
    m, N, t = 256, 16, 2
    f = E.ParticleFilter(UNI, p, particles_per_subfilter=m, num_subfilters=N, num_transfer=t, exchange=2,
                         resampler=res, rng=rng_mode, mtgp_streams=96)
    f.record_selection(True)
    ppt = f.info()["particles_per_thread"]
    md = O.model_from_params(UNI, p)
    orng = O.RNG_SUBFILTER if rng_mode == E.RNG_SUBFILTER else O.RNG_REFLAYOUT
    of = O.Filter(md, m, N, t, O.EXCH_TORUS, res, orng, 96, ppt, 1, 1.0, 0xF000000D, 0, np.zeros(3, np.float32))
    for k in range(3):
        if k > 0:  # continue both from the same particles so every step is compared on equal inputs
            f.set_particles(of.state())
        ge = f.step(inputs[k])
        oe, osel = of.step(inputs["control"][k], inputs["meas"][k], want_sel=True)
        gs, gk = f.sorted()
        os_, ok = of.sorted()
        # log-weights: FP32 device math vs FP64 oracle
        assert np.all(np.abs(gk - ok) <= 1e-4 * np.abs(ok) + 2e-3)
        # propagated state, sorted: identical random numbers, FP32 vs FP64 propagation
        same = np.flatnonzero(np.abs(gk - ok) <= 1e-4 * np.abs(ok) + 2e-3)
        d = np.abs(gs - os_)
        d[2] = np.abs(np.angle(np.exp(1j * (gs[2].astype(np.float64) - os_[2]))))
        frac_equal_order = np.mean(d.max(axis=0) < 1e-4)
        assert frac_equal_order > 0.97, frac_equal_order  # near-ties may swap sorted positions
        assert abs(ge["log_norm"] - oe.log_norm) < 1e-3 * abs(oe.log_norm) + 1e-3
        assert np.allclose(ge["mean"][:2], oe.mean[:2], atol=2e-3)
        gsel = f.selection()
        assert np.mean(gsel == osel) > 0.97


def test_graph_replay_equals_host_steps(gpu):
    import torch
    E = gpu
    p, inputs, _ = uni_setup(steps=12)
    cfg = dict(particles_per_subfilter=512, num_subfilters=32, num_transfer=2, exchange=2)
    fa, ea = run(E, UNI, p, inputs, 12, **cfg)
    fb = E.ParticleFilter(UNI, p, **cfg)
    d_in = torch.from_numpy(inputs.view(np.uint8).copy()).cuda()
    d_est = torch.zeros(12 * E.ESTIMATE_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    fb.run_device(d_in.data_ptr(), d_est.data_ptr(), 12, 12)
    fb.synchronize()
    est = d_est.cpu().numpy().view(E.ESTIMATE_DTYPE)
    assert np.array_equal(fa.particles(), fb.particles())
    for k in range(12):
        assert np.array_equal(est[k]["mean"], ea[k]["mean"]) and est[k]["best_key"] == ea[k]["best_key"]
        assert est[k]["step"] == k + 1


@pytest.mark.parametrize("period", [2, 3])
def test_graph_replay_exchange_period(gpu, period):
    """Graph replay with an exchange period: every resampling CTA reads the
    device step counter, which must not advance before all of them did."""
    import torch
    E = gpu
    steps = 9
    p, inputs, _ = uni_setup(steps=steps)
    cfg = dict(particles_per_subfilter=128, num_subfilters=2048, num_transfer=1, exchange=2,
               exchange_period=period, pipeline=E.PIPELINE_SPLIT)
    fa, ea = run(E, UNI, p, inputs, steps, **cfg)
    fb = E.ParticleFilter(UNI, p, **cfg)
    d_in = torch.from_numpy(inputs.view(np.uint8).copy()).cuda()
    d_est = torch.zeros(steps * E.ESTIMATE_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    fb.run_device(d_in.data_ptr(), d_est.data_ptr(), steps, steps)
    fb.synchronize()
    est = d_est.cpu().numpy().view(E.ESTIMATE_DTYPE)
    assert np.array_equal(fa.particles(), fb.particles())
    for k in range(steps):
        assert np.array_equal(est[k]["mean"], ea[k]["mean"]) and est[k]["step"] == k + 1


@pytest.mark.parametrize("pipe,period", [(0, 1), (2, 1), (2, 2)])
def test_submit_collect_equals_step(gpu, pipe, period):
    """Pipelined submit / collect against synchronous pf_step on the same
    inputs, past the ring depth, with a synchronous step and a
    re-initialisation in between."""
    E = gpu
    steps = 150
    p, inputs, _ = uni_setup(steps=steps)
    cfg = dict(particles_per_subfilter=256, num_subfilters=64, num_transfer=2, exchange=2, pipeline=pipe,
               exchange_period=period)
    fa, ea = run(E, UNI, p, inputs, steps, **cfg)
    fb = E.ParticleFilter(UNI, p, **cfg)
    got = []
    for k in range(E.QUEUE_DEPTH):
        fb.submit(inputs[k])
    with pytest.raises(E.PFError) as ei:
        fb.submit(inputs[E.QUEUE_DEPTH])
    assert ei.value.status == E.PF_ERR_BUSY
    got += list(fb.collect(10))
    k = E.QUEUE_DEPTH
    while k < 100:
        fb.submit(inputs[k])
        k += 1
        got += list(fb.collect(wait=False))
    got += list(fb.collect())
    assert len(got) == 100 and len(fb.collect(5, wait=False)) == 0
    got.append(fb.step(inputs[100]))  # a synchronous step in between
    for k in range(101, steps):
        fb.submit(inputs[k])
    got += list(fb.collect())
    assert len(got) == steps
    for k in range(steps):
        assert got[k]["step"] == ea[k]["step"] == k + 1
        assert np.array_equal(got[k]["mean"], ea[k]["mean"]) and got[k]["best_key"] == ea[k]["best_key"]
    assert np.array_equal(fa.particles(), fb.particles())
    # restart from the initial state: the queue re-reads the step counter
    init = np.zeros(3, np.float32)
    fa.set_initial_state(init)
    fb.set_initial_state(init)
    a = [fa.step(inputs[k]) for k in range(5)]
    for k in range(5):
        fb.submit(inputs[k])
    b = fb.collect(5)
    assert all(np.array_equal(x["mean"], y["mean"]) and x["step"] == y["step"] for x, y in zip(a, b))


def test_submit_collect_across_counter_wrap(gpu):
    """The pipelined queue indexes its rings with the device step counter; a
    filter restored with a step count just below 2^31 keeps stepping correctly
    past the wrap (same estimates as synchronous steps from the same state)."""
    E = gpu
    p, inputs, _ = uni_setup(steps=12)
    cfg = dict(particles_per_subfilter=128, num_subfilters=32, num_transfer=1, exchange=2)
    fa = E.ParticleFilter(UNI, p, **cfg)
    for k in range(2):
        fa.step(inputs[k])
    snap = fa.snapshot()
    snap[-4:] = np.array([2 ** 31 - 3], np.int32).view(np.uint8)  # the step count, stored last
    fb = E.ParticleFilter(UNI, p, **cfg)
    fa.restore(snap)
    fb.restore(snap)
    a = [fa.step(inputs[k]) for k in range(2, 10)]
    for k in range(2, 10):
        fb.submit(inputs[k])
    b = fb.collect(8)
    assert len(b) == 8
    for x, y in zip(a, b):
        assert np.array_equal(x["mean"], y["mean"]) and x["best_key"] == y["best_key"]
    assert np.array_equal(fa.particles(), fb.particles())


def test_snapshot_restore(gpu):
    E = gpu
    p, inputs, _ = uni_setup(steps=10)
    f = E.ParticleFilter(UNI, p, particles_per_subfilter=128, num_subfilters=8, num_transfer=1)
    for k in range(4):
        f.step(inputs[k])
    snap = f.snapshot()
    a = [f.step(inputs[k]) for k in range(4, 8)]
    pa = f.particles()
    with pytest.raises(E.PFError) as ei:
        f.restore(snap[:-4])  # truncated: refused before it is read
    assert ei.value.status == E.PF_ERR_INVALID
    f.restore(snap)
    b = [f.step(inputs[k]) for k in range(4, 8)]
    assert np.array_equal(pa, f.particles())
    assert all(np.array_equal(x["mean"], y["mean"]) for x, y in zip(a, b))


@pytest.mark.parametrize("m", [64, 128])
def test_skipped_subfilters_keep_propagated_state(gpu, O, m):
    E = gpu
    p, inputs, _ = uni_setup(steps=3)
    f = E.ParticleFilter(UNI, p, particles_per_subfilter=m, num_subfilters=64, num_transfer=1, exchange=1,
                         resampling_freq=0.5)
    f.record_selection(True)
    for k in range(2):
        f.step(inputs[k])
        sel = f.selection().reshape(64, m)
        skipped = np.all(sel == -1, axis=1)
        assert 10 < skipped.sum() < 54  # about half of the sub-filters skip at freq 0.5
        assert np.all((sel[~skipped] >= 0) & (sel[~skipped] < m))
        st = f.particles().reshape(3, 64, m)
        srt, _ = f.sorted()
        srt = srt.reshape(3, 64, m)
        for b in np.flatnonzero(skipped):  # unsorted propagated particles = a permutation of the sorted ones
            assert np.array_equal(np.sort(st[0, b]), np.sort(srt[0, b]))


@pytest.mark.parametrize("pipe", [0, 1, 2])
@pytest.mark.parametrize("res", [0, 1, 2])
def test_ess_gate_vs_oracle(gpu, O, pipe, res):
    """ESS-gated resampling on a torus with exchange: the engine's per
    sub-filter decisions and selections against the oracle on the same
    particles (decisions within 1e-5 of the threshold may differ: FP32 exp)."""
    E = gpu
    p, inputs, _ = uni_setup()
    m, N, t = 256, 64, 2
    rng = E.RNG_REFLAYOUT if pipe == E.PIPELINE_PHASED else E.RNG_SUBFILTER
    orng = O.RNG_REFLAYOUT if rng == E.RNG_REFLAYOUT else O.RNG_SUBFILTER
    md = O.model_from_params(UNI, p)
    probe = O.Filter(md, m, 32, 0, O.EXCH_NONE, res, O.RNG_SUBFILTER, 96, 2, 1, 1.0, 0xF000000D, 0,
                     np.zeros(3, np.float32))
    probe.step(inputs["control"][0], inputs["meas"][0])
    k = probe.sorted()[1].reshape(32, m).astype(np.float64)
    w = np.exp(k - k.max(axis=1, keepdims=True))
    frac = float(np.median(w.sum(axis=1) ** 2 / (w * w).sum(axis=1) / m))
    f = E.ParticleFilter(UNI, p, particles_per_subfilter=m, num_subfilters=N, num_transfer=t, exchange=2,
                         resampler=res, rng=rng, mtgp_streams=96, pipeline=pipe, ess_fraction=frac)
    assert f.info()["pipeline"] == pipe
    f.record_selection(True)
    of = O.Filter(md, m, N, t, O.EXCH_TORUS, res, orng, 96, f.info()["particles_per_thread"], 1, 1.0, 0xF000000D,
                  0, np.zeros(3, np.float32))
    of.f.ess_frac = frac
    mixed = 0
    for k in range(3):
        if k > 0:
            f.set_particles(of.state())
        f.step(inputs[k])
        _, osel = of.step(inputs["control"][k], inputs["meas"][k], want_sel=True)
        gsel, osel = f.selection().reshape(N, m), osel.reshape(N, m)
        gskip, oskip = np.all(gsel == -1, axis=1), np.all(osel == -1, axis=1)
        assert np.mean(gskip == oskip) > 0.95, (gskip.sum(), oskip.sum())
        both = ~gskip & ~oskip
        assert np.all((gsel[both] >= 0) & (gsel[both] < m))
        assert np.mean(gsel[both] == osel[both]) > 0.97
        mixed += 0 < oskip.sum() < N
    assert mixed >= 1


def rmse_xy(ests, truth):
    m = np.array([e["mean"][:2] for e in ests])
    return float(np.sqrt(np.mean(np.sum((m - truth[:, :2]) ** 2, axis=1))))


def test_unicycle_4096_rmse_matches_oracle(gpu, O):
    """Plain unicycle filter: 4096 = 8 x 512, systematic every step, no exchange, 100 steps, seed 1."""
    E = gpu
    p, inputs, truth = uni_setup(1, 100)
    f, ests = run(E, UNI, p, inputs, particles_per_subfilter=512, num_subfilters=8, num_transfer=0, exchange=0)
    g = rmse_xy(ests, truth)
    md = O.model_from_params(UNI, p)
    of = O.Filter(md, 512, 8, 0, 0, 1, O.RNG_SUBFILTER, 96, f.info()["particles_per_thread"], 1, 1.0, 0xF000000D, 0,
                  np.zeros(3, np.float32))
    oes = [of.step(inputs["control"][k], inputs["meas"][k])[0] for k in range(100)]
    o = float(np.sqrt(np.mean([(e.mean[0] - truth[k, 0]) ** 2 + (e.mean[1] - truth[k, 1]) ** 2
                               for k, e in enumerate(oes)])))
    assert g < 0.25 and o < 0.25
    assert abs(g - o) <= 0.05 * o + 0.005, (g, o)


def test_unicycle_2p20_torus_shape_properties(gpu):
    """2^20 particles = 2048 x 512 on a 32 x 64 torus, t = 2: sortedness, routing
    bounds, systematic monotone selections, finite estimates (size-independent checks)."""
    E = gpu
    p, inputs, truth = uni_setup(2, 4)
    f = E.ParticleFilter(UNI, p, particles_per_subfilter=512, num_subfilters=2048, num_transfer=2, exchange=2)
    assert f.info()["torus"] == (32, 64)
    f.record_selection(True)
    for k in range(4):
        e = f.step(inputs[k])
        assert e["flags"] == 0 and np.all(np.isfinite(e["mean"][:3]))
        _, keys = f.sorted()
        kk = keys.reshape(2048, 512)
        assert np.all(kk[:, :-1] >= kk[:, 1:])
        assert e["best_key"] == kk.max() and e["best_subfilter"] == int(np.argmax(kk[:, 0]))
        sel = f.selection().reshape(2048, 512)
        assert np.all((sel >= 0) & (sel < 512)) and np.all(np.diff(sel, axis=1) >= 0)
    assert np.hypot(*(e["mean"][:2] - truth[3, :2])) < 0.5


@pytest.mark.parametrize("res", [1, 2])
def test_unicycle_torus_256x512_tracks(gpu, res):
    E = gpu
    p, inputs, truth = uni_setup(2, 200)
    f, ests = run(E, UNI, p, inputs, particles_per_subfilter=512, num_subfilters=256, num_transfer=2, exchange=2,
                  resampler=res)
    assert rmse_xy(ests, truth) < 0.2


def test_dharm_tracks(gpu):
    E = gpu
    p = E.dharm_params(3)
    inputs, truth = E.make_trace(ARM, p, 3, 100)
    f, ests = run(E, ARM, p, inputs, particles_per_subfilter=256, num_subfilters=64, num_transfer=1, exchange=2)
    q = np.array([e["mean"][:6] for e in ests])
    err = np.angle(np.exp(1j * (q - truth[:, :6])))
    assert np.sqrt(np.mean(err[20:] ** 2)) < 0.05


def test_reference_driver_on_trace(gpu, tmp_path):
    E = gpu
    rng = np.random.default_rng(0)
    lines = []
    ang = np.full(5, 0.75 * np.pi)
    x, y = 7.0, 0.0
    for k in range(20):
        rate = rng.normal(0, 0.05, 5)
        ang = ang + rate
        x, y = x + 0.1, y + 0.05
        meas = ang + rng.normal(0, 0.02, 5)
        lines.append(" ".join("%.6f" % v for v in [x, y, *meas, *rate, 1.0, x, y, *ang]))
    fn = tmp_path / "arm_trace"
    fn.write_text("\n".join(lines) + "\n")
    e = E.particle_filter(256, 16, 1, 1.0, fn)
    assert np.isfinite(e) and e >= 0
