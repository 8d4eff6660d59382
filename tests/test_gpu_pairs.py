"""Two threads per particle (pf_config.threads_per_particle = 2): lane pairs
share each particle's propagate + weight and sort together.  Models without a
split (the reference's camera arm, the linear-Gaussian plugin) give the
one-thread results bit for bit; the split models (unicycle landmarks, beacon
ranges, the DH arm's kinematic chain) match the FP64 oracle like the one-thread
path does; batches with pairs equal their filters run alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UNI, ARM, REF, BEACON = 0, 1, 2, 3


def _same_particles(a, b):
    sa, ka = a.sorted()
    sb, kb = b.sorted()
    return np.array_equal(a.particles(), b.particles()) and np.array_equal(sa, sb) and np.array_equal(ka, kb)


@pytest.mark.parametrize("res", [0, 1, 2])
def test_pairs_equal_one_thread_for_unsplit_models(gpu, res):
    E = gpu
    prm = E.LinGaussParams(0.1, 0.5, 0.3, (0.0, 1.0))
    steps = 6
    inp = np.zeros(steps, E.STEP_INPUT_DTYPE)
    inp["dt"] = prm.dt
    inp["meas"][:, 0] = np.linspace(0.1, 0.6, steps)
    cfg = dict(particles_per_subfilter=256, num_subfilters=64, num_transfer=2, exchange=E.EXCHANGE_TORUS,
               resampler=res, pipeline=E.PIPELINE_SPLIT)
    a = E.ParticleFilter(E.MODEL_LINGAUSS, prm, threads_per_particle=1, **cfg)
    b = E.ParticleFilter(E.MODEL_LINGAUSS, prm, threads_per_particle=2, **cfg)
    for k in range(steps):
        ea, eb = a.step(inp[k]), b.step(inp[k])
        assert _same_particles(a, b), k
        assert ea["best_key"] == eb["best_key"] and ea["best_subfilter"] == eb["best_subfilter"]
        assert np.allclose(ea["mean"], eb["mean"], rtol=1e-12, atol=1e-12)


def _setup(E, model, seed, steps):
    if model == UNI:
        p = E.unicycle_params(seed)
    elif model == ARM:
        p = E.dharm_params(seed)
    else:
        p = E.beacon_params()
    inputs, _ = E.make_trace(model, p, seed, steps)
    return p, inputs


def _same_as_oracle(gs, os_, m, N, model):
    """Fraction of particles equal (1e-4, angles wrapped) with each
    sub-filter's particles in the order of a coordinate without ties (x, or a
    joint velocity of the arm): resampled duplicates share keys exactly, so
    sorted positions of ties may differ where FP32 and FP64 order near-ties
    differently."""
    S = gs.shape[0]
    col = 6 if model == ARM else 0
    angles = list(range(6)) if model == ARM else [2]
    g = gs.reshape(S, N, m).astype(np.float64)
    o = os_.reshape(S, N, m).astype(np.float64)
    g = np.take_along_axis(g, np.argsort(g[col], axis=1, kind="stable")[None], axis=2)
    o = np.take_along_axis(o, np.argsort(o[col], axis=1, kind="stable")[None], axis=2)
    d = np.abs(g - o)
    for v in angles:
        d[v] = np.abs(np.angle(np.exp(1j * (g[v] - o[v]))))
    return float((d.max(axis=0) < 1e-4).mean())


@pytest.mark.parametrize("model", [UNI, BEACON, ARM])
@pytest.mark.parametrize("res", [1, 2])
def test_pairs_steps_vs_oracle(gpu, O, model, res):
    """The split models with pairs against the FP64 oracle, every step from the
    oracle's particles: FP32 keys within tolerance, propagated particles equal,
    and the oracle's exchange + resampling run on the engine's sorted copy
    select the engine's slots and particles bit for bit."""
    E = gpu
    p, inputs = _setup(E, model, 3, 3)
    m, N, t = 256, 16, 2
    f = E.ParticleFilter(model, p, particles_per_subfilter=m, num_subfilters=N, num_transfer=t, exchange=2,
                         resampler=res, pipeline=E.PIPELINE_SPLIT, threads_per_particle=2)
    f.record_selection(True)
    ppt = f.info()["particles_per_thread"]
    md = O.model_from_params(model, p)
    S = f.num_state
    init = np.array(p.init_state[:S], np.float32)
    f.set_initial_state(init)
    of = O.Filter(md, m, N, t, O.EXCH_TORUS, res, O.RNG_SUBFILTER, 96, ppt, 1, 1.0, 0xF000000D, 0, init)
    katol = 5e-3 if model == ARM else 2e-3
    for k in range(3):
        if k > 0:
            f.set_particles(of.state())
        ge = f.step(inputs[k])
        oe = of.sample(inputs["control"][k], inputs["meas"][k])
        gs, gk = f.sorted()
        os_, ok = of.sorted()
        assert np.all(np.abs(gk - ok) <= 1e-4 * np.abs(ok) + katol), np.max(np.abs(gk - ok))
        same = _same_as_oracle(gs, os_, m, N, model)
        assert same > 0.99, same
        assert abs(ge["log_norm"] - oe.log_norm) < 1e-3 * abs(oe.log_norm) + 1e-3
        of.set_sorted(gs, gk)
        osel = of.resample()
        assert np.array_equal(f.selection(), osel)
        assert np.array_equal(f.particles(), of.state())


@pytest.mark.parametrize("m,ppt", [(256, 4), (512, 2), (128, 2)])
def test_pair_batch_equals_single_filters(gpu, m, ppt):
    E = gpu
    counts = [256, 1024, 768, 2048]
    steps = 5
    params = [E.unicycle_params(4 + i) for i in range(len(counts))]
    traces = [E.make_trace(UNI, q, 4 + i, steps) for i, q in enumerate(params)]
    inputs = np.stack([tr[0] for tr in traces])
    cfg = dict(num_transfer=1, exchange=1, resampler=1, particles_per_thread=ppt, threads_per_particle=2)
    B = E.FilterBatch(UNI, params, counts, particles_per_subfilter=m, **cfg)
    best = [B.step(inputs[:, k]) for k in range(steps)]
    for f, n in enumerate(counts):
        mf, e = B.filter_shape(f)
        fi = B.filter_info(f)
        s = E.ParticleFilter(UNI, params[f], pipeline=E.PIPELINE_SPLIT, particles_per_subfilter=mf,
                             num_subfilters=n // mf, stream_offset=fi["stream_offset"],
                             **dict(cfg, particles_per_thread=e))
        for k in range(steps):
            e1, e2 = best[k][f], s.step(inputs[f, k])
            assert np.array_equal(e1["mean"], e2["mean"]) and e1["best_key"] == e2["best_key"], (f, k)
        assert np.array_equal(B.particles(f), s.particles()), f


def test_pair_arguments(gpu):
    E = gpu
    p = E.unicycle_params(1)
    cfg = dict(particles_per_subfilter=256, num_subfilters=4)
    with pytest.raises(E.PFError) as e:
        E.ParticleFilter(UNI, p, threads_per_particle=3, **cfg)
    assert e.value.status == E.PF_ERR_INVALID
    with pytest.raises(E.PFError) as e:
        E.ParticleFilter(UNI, p, threads_per_particle=2, rng=E.RNG_REFLAYOUT, **cfg)
    assert e.value.status == E.PF_ERR_UNSUPPORTED
    f = E.ParticleFilter(UNI, p, threads_per_particle=2, pipeline=E.PIPELINE_FUSED, **cfg)
    assert f.info()["pipeline"] == E.PIPELINE_SPLIT  # the single-kernel step has no pair form
