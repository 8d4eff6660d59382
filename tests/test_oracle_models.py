"""The oracle's model restatements against numpy formulas, and the oracle
filter tracking the seeded ground truth (the CPU side of the RMSE check)."""
import numpy as np
import pytest


def test_unicycle_model_formula(O, E):
    p = E.unicycle_params(1)
    md = O.model_from_params(E.MODEL_UNICYCLE, p)
    rng = np.random.default_rng(0)
    n = 64
    st = np.stack([rng.normal(0, 3, n), rng.normal(0, 3, n), rng.uniform(-3, 3, n)]).astype(np.float32)
    nz = rng.standard_normal((3, n)).astype(np.float32)
    v, w, dt = 1.0, 0.2, 0.1
    z = np.concatenate([rng.uniform(1, 10, 4), rng.uniform(-3, 3, 4)]).astype(np.float32)
    new, ll = O.model_step(md, st, nz, [v, w], z)
    x, y, th = st.astype(np.float64)
    ex = x + v / w * (np.sin(th + w * dt) - np.sin(th)) + 0.05 * nz[0]
    ey = y - v / w * (np.cos(th + w * dt) - np.cos(th)) + 0.05 * nz[1]
    et = np.angle(np.exp(1j * (th + w * dt + 0.01 * nz[2])))
    assert np.allclose(new[0], ex, atol=1e-5) and np.allclose(new[1], ey, atol=1e-5)
    assert np.allclose(np.angle(np.exp(1j * (new[2] - et))), 0, atol=1e-6)
    lm = np.array([[p.landmarks[j][0], p.landmarks[j][1]] for j in range(4)])
    X, Y, TH = new.astype(np.float64)
    acc = 0
    for j in range(4):
        r = np.hypot(lm[j, 0] - X, lm[j, 1] - Y)
        b = np.arctan2(lm[j, 1] - Y, lm[j, 0] - X) - TH
        acc = acc + ((z[j] - r) / 0.2) ** 2 + (np.angle(np.exp(1j * (z[4 + j] - b))) / 0.05) ** 2
    assert np.allclose(ll, -0.5 * acc, rtol=1e-6, atol=1e-6)


def test_unicycle_straight_line_limit(O, E):
    md = O.model_from_params(E.MODEL_UNICYCLE, E.unicycle_params(1))
    st = np.array([[1.0], [2.0], [0.5]], np.float32)
    new, _ = O.model_step(md, st, np.zeros((3, 1), np.float32), [1.0, 0.0], np.ones(8, np.float32))
    assert np.allclose(new[:, 0], [1 + 0.1 * np.cos(0.5), 2 + 0.1 * np.sin(0.5), 0.5], atol=1e-7)


def _dh_fk(p, q):
    T = np.eye(4)
    for i in range(6):
        ct, st, ca, sa = np.cos(q[i]), np.sin(q[i]), np.cos(p.alpha[i]), np.sin(p.alpha[i])
        A = np.array([[ct, -st * ca, st * sa, p.a[i] * ct], [st, ct * ca, -ct * sa, p.a[i] * st],
                      [0, sa, ca, p.d[i]], [0, 0, 0, 1]])
        T = T @ A
    R = T[:3, :3]
    ypr = [np.arctan2(R[1, 0], R[0, 0]), np.arctan2(-R[2, 0], np.hypot(R[2, 1], R[2, 2])),
           np.arctan2(R[2, 1], R[2, 2])]
    return T[:3, 3], np.array(ypr)


def test_dharm_model_fk(O, E):
    p = E.dharm_params(3)
    md = O.model_from_params(E.MODEL_DHARM, p)
    rng = np.random.default_rng(1)
    n = 16
    st = np.concatenate([rng.uniform(-3, 3, (6, n)), rng.normal(0, 0.5, (6, n))]).astype(np.float32)
    nz = rng.standard_normal((6, n)).astype(np.float32)
    z = np.concatenate([rng.normal(0, 0.5, 3), rng.uniform(-3, 3, 3)]).astype(np.float32)
    new, ll = O.model_step(md, st, nz, [], z)
    for i in range(n):
        q = np.angle(np.exp(1j * (st[:6, i].astype(np.float64) + st[6:, i] * 0.01)))
        assert np.allclose(np.angle(np.exp(1j * (new[:6, i] - q))), 0, atol=1e-6)
        assert np.allclose(new[6:, i], st[6:, i] + 0.01 * nz[:, i], atol=1e-6)
        pos, ypr = _dh_fk(p, new[:6, i].astype(np.float64))
        e = np.sum(((z[:3] - pos) / 0.005) ** 2) + np.sum((np.angle(np.exp(1j * (z[3:] - ypr))) / 0.02) ** 2)
        assert np.isclose(ll[i], -0.5 * e, rtol=1e-6)


def test_refarm_model_reference_formula(O, E):
    md = O.model_from_params(E.MODEL_REFARM, E.refarm_params(1.0))
    rng = np.random.default_rng(2)
    st = np.concatenate([np.full((5, 4), 0.75 * np.pi), [[7] * 4, [0] * 4, [0] * 4, [0] * 4]]).astype(np.float32)
    nz = rng.standard_normal((9, 4)).astype(np.float32)
    c = rng.normal(0, 0.05, 5).astype(np.float32)
    z = np.concatenate([rng.uniform(2, 3, 5), [0.5, 1.5]]).astype(np.float32)
    new, ll = O.model_step(md, st, nz, c, z)
    for i in range(4):
        x = 7 + nz[5, i] * 0.2
        y = 0 + nz[6, i] * 0.2
        ang = 0.75 * np.pi + c * 1.0 + nz[:5, i] * 0.2
        cx, cy, cz = x * np.cos(ang[0]) + y * np.sin(ang[0]), -x * np.sin(ang[0]) + y * np.cos(ang[0]), 0.0
        for k in range(1, 5):
            cy, cz = cy * np.cos(ang[k]) - cz * np.sin(ang[k]), cy * np.sin(ang[k]) + cz * np.cos(ang[k]) - 3.0
        val = np.sum((ang - z[:5]) ** 2 * 0.1) + (cx - z[5]) ** 2 * 0.1 + (cy - z[6]) ** 2 * 0.1
        assert np.isclose(ll[i], -val, rtol=1e-5)


@pytest.mark.parametrize("rng_mode", [0, 1])
def test_oracle_filter_tracks_unicycle(O, E, rng_mode):
    p = E.unicycle_params(1)
    inputs, truth = E.make_trace(E.MODEL_UNICYCLE, p, 1, 100)
    md = O.model_from_params(E.MODEL_UNICYCLE, p)
    f = O.Filter(md, 512, 8, 0, O.EXCH_NONE, O.RES_SYSTEMATIC, rng_mode, 96, 2, 1, 1.0, 0xF000000D, 0,
                 np.zeros(3, np.float32))
    err = []
    for k in range(100):
        e, _ = f.step(inputs["control"][k], inputs["meas"][k])
        err.append((e.mean[0] - truth[k, 0]) ** 2 + (e.mean[1] - truth[k, 1]) ** 2)
    rmse = np.sqrt(np.mean(err))
    assert rmse < 0.25, rmse


def ess_ratio(keys, m, log_weights=True):
    """Per sub-filter effective sample size / m of sorted keys (FP64)."""
    k = keys.reshape(-1, m).astype(np.float64)
    w = np.exp(k - k.max(axis=1, keepdims=True)) if log_weights else k
    return w.sum(axis=1) ** 2 / (w * w).sum(axis=1) / m


@pytest.mark.parametrize("res", [0, 1, 2])
def test_oracle_ess_gate(O, E, res):
    """ESS-gated resampling in the oracle: a sub-filter resamples iff
    (sum w)^2 / sum w^2 < f * m; f -> 0 never resamples, and the sub-filters
    that do resample select exactly what the ungated filter selects."""
    p = E.unicycle_params(1)
    inputs, _ = E.make_trace(E.MODEL_UNICYCLE, p, 1, 3)
    md = O.model_from_params(E.MODEL_UNICYCLE, p)
    m, N = 128, 32

    def mk(frac):
        f = O.Filter(md, m, N, 0, O.EXCH_NONE, res, O.RNG_SUBFILTER, 96, 2, 1, 1.0, 0xF000000D, 0,
                     np.zeros(3, np.float32))
        f.f.ess_frac = frac
        return f

    base, never = mk(0.0), mk(1e-9)
    _, sel0 = base.step(inputs["control"][0], inputs["meas"][0], want_sel=True)
    _, seln = never.step(inputs["control"][0], inputs["meas"][0], want_sel=True)
    assert np.all(seln == -1) and np.all(sel0 >= 0)
    ratio = ess_ratio(base.sorted()[1], m)
    frac = float(np.median(ratio))
    gated = mk(frac)
    _, sel = gated.step(inputs["control"][0], inputs["meas"][0], want_sel=True)
    sel, sel0 = sel.reshape(N, m), sel0.reshape(N, m)
    skipped = np.all(sel == -1, axis=1)
    near = np.abs(ratio / frac - 1.0) < 1e-6
    assert np.array_equal(skipped[~near], (ratio >= frac)[~near])
    assert 0 < skipped.sum() < N
    assert np.array_equal(sel[~skipped], sel0[~skipped])
    # skipped sub-filters keep the propagated (unsorted) particles
    st, srt = gated.state().reshape(3, N, m), gated.sorted()[0].reshape(3, N, m)
    for b in np.flatnonzero(skipped):
        assert np.array_equal(np.sort(st[0, b]), np.sort(srt[0, b]))


def test_oracle_step_equals_sample_then_resample(O, E):
    """orc_filter_step is orc_filter_sample followed by orc_filter_resample, and
    handing the resampler its own sorted copy back changes nothing."""
    p = E.unicycle_params(2)
    inputs, _ = E.make_trace(0, p, 2, 3)
    md = O.model_from_params(0, p)
    for res in (0, 1, 2):
        a = O.Filter(md, 128, 16, 2, O.EXCH_TORUS, res, O.RNG_SUBFILTER, 96, 4, 1, 1.0, 0xF000000D, 0,
                     np.zeros(3, np.float32))
        b = O.Filter(md, 128, 16, 2, O.EXCH_TORUS, res, O.RNG_SUBFILTER, 96, 4, 1, 1.0, 0xF000000D, 0,
                     np.zeros(3, np.float32))
        for k in range(3):
            ea, sa = a.step(inputs["control"][k], inputs["meas"][k], want_sel=True)
            eb = b.sample(inputs["control"][k], inputs["meas"][k])
            s, kk = b.sorted()
            b.set_sorted(s, kk)
            sb = b.resample()
            assert np.array_equal(sa, sb) and np.array_equal(a.state(), b.state())
            assert ea.log_norm == eb.log_norm and list(ea.mean) == list(eb.mean)
