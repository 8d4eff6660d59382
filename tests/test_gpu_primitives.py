"""CUDA kernels through the C ABI against the reference's generator (golden
KATs) and the oracle: bit-exact for integer/index work, stated tolerances for
floating point."""
import numpy as np
import pytest

from golden.make_golden import KAT_CASES, KAT_N

pytestmark = pytest.mark.gpu

ME = [(32, 1), (64, 2), (128, 2), (128, 4), (256, 2), (256, 4), (512, 2), (512, 4), (1024, 2), (1024, 4)]


def test_mtgp_block_layout_matches_reference(gpu, golden):
    got = gpu.mtgp_generate(96, 0xF000000D, 768, kind=1, calls=2)
    assert np.array_equal(got, golden["blocks_G96_f32"])


@pytest.mark.parametrize("set_,seed", KAT_CASES)
@pytest.mark.parametrize("kind", [0, 1])
def test_mtgp_stream_kat(gpu, golden, set_, seed, kind):
    # stream g is seeded with base + g + 1: pick base so stream `set_` gets `seed`
    base = (seed - set_ - 1) & 0xFFFFFFFF
    out = gpu.mtgp_generate(set_ + 1, base, KAT_N, kind=kind).reshape(set_ + 1, KAT_N)
    key = "kat_%s_%d_%d" % ("u32" if kind == 0 else "f32", set_, seed)
    assert np.array_equal(out[set_], golden[key])


@pytest.mark.parametrize("per", [1, 255, 300, 1000])
def test_mtgp_state_continues_across_launches(gpu, O, per):
    out = gpu.mtgp_generate(3, 41, per, kind=1, calls=4).reshape(4, 3, per)
    for g in range(3):
        assert np.array_equal(out[:, g, :].reshape(-1), O.mtgp_stream(g, 41 + g + 1, 4 * per))


def test_mtgp_cuda_reference_mask(gpu, golden):
    out = gpu.mtgp_generate(1, 0, KAT_N, kind=1, mask=gpu.MTGP_MASK_CUDA_REF)
    assert np.array_equal(out, golden["cudamask_f32_0_1"])


def test_boxmuller_vs_oracle(gpu, O):
    rng = np.random.default_rng(7)
    u = (1 + rng.random(100001)).astype(np.float32)
    u[:4] = [1.0, 1.0, np.float32(1.9999999), np.float32(1.9999999)]
    n = 100001  # odd: the last pair reads one float past n, as the reference does
    g = gpu.boxmuller(np.concatenate([u, [np.float32(1.5)]]), n)
    o = O.boxmuller(np.concatenate([u, [np.float32(1.5)]]), n)
    # tolerance: FP32 logf/sqrtf/sincospif vs double, |z| <= 6
    assert np.max(np.abs(g[:n + 1] - o[:n + 1])) < 4e-6
    assert np.all(np.isfinite(g))


@pytest.mark.parametrize("m,ppt", ME)
def test_sort_bit_exact(gpu, O, golden, m, ppt):
    if m in (32, 64, 256, 512):
        keys = golden["sort_in_%d" % m]
        k, i = gpu.bitonic_sort(keys, m, ppt)
        assert np.array_equal(k, golden["sort_key_%d" % m]) and np.array_equal(i, golden["sort_idx_%d" % m])
    rng = np.random.default_rng(m * 10 + ppt)
    keys = np.round(rng.standard_normal(16 * m) * 3).astype(np.float32)
    keys[:m] = 0.0
    k, i = gpu.bitonic_sort(keys, m, ppt)
    ok, oi = O.bitonic_sort(keys, m)
    assert np.array_equal(k, ok) and np.array_equal(i, oi)


@pytest.mark.parametrize("m", [32, 64, 256, 512])
def test_resample_reference_bit_exact(gpu, golden, m):
    for ppt in [e for (mm, e) in ME if mm == m]:
        sel = gpu.resample(gpu.RESAMPLE_REFERENCE, golden["res_w_%d" % m], golden["res_uref_%d" % m], m, ppt)
        assert np.array_equal(sel, golden["res_ref_%d" % m])


@pytest.mark.parametrize("m,ppt", [(32, 1), (64, 2), (256, 2), (256, 4), (512, 2), (512, 4)])
def test_resample_systematic_bit_exact(gpu, golden, m, ppt):
    sel = gpu.resample(gpu.RESAMPLE_SYSTEMATIC, golden["res_w_%d" % m], golden["res_usys_%d" % m], m, ppt)
    assert np.array_equal(sel, golden["res_sys_%d_%d" % (m, ppt)])


@pytest.mark.parametrize("m", [32, 64, 256, 512])
def test_vose_bit_exact(gpu, golden, m):
    for ppt in [e for (mm, e) in ME if mm == m]:
        p, a = gpu.vose_build(golden["res_w_%d" % m], m, ppt)
        assert np.array_equal(p, golden["vose_prob_%d" % m]) and np.array_equal(a, golden["vose_alias_%d" % m])
        sel = gpu.resample(gpu.RESAMPLE_VOSE, golden["res_w_%d" % m], golden["res_uvose_%d" % m], m, ppt)
        assert np.array_equal(sel, golden["res_vose_%d" % m])


@pytest.mark.parametrize("m,ppt", [(128, 2), (128, 4), (1024, 2), (1024, 4)])
def test_resamplers_vs_oracle_other_sizes(gpu, O, m, ppt):
    rng = np.random.default_rng(m + ppt)
    w = (rng.exponential(1, 8 * m) ** 4).astype(np.float32)
    w[:m] = 0
    u = (1 + rng.random(8 * m)).astype(np.float32)
    assert np.array_equal(gpu.resample(0, w, u, m, ppt), O.resample(0, w, u, m, ppt))
    us = rng.random(8).astype(np.float32)
    assert np.array_equal(gpu.resample(1, w, us, m, ppt), O.resample(1, w, us, m, ppt))
    uv = rng.random(16 * m).astype(np.float32)
    assert np.array_equal(gpu.resample(2, w, uv, m, ppt), O.resample(2, w, uv, m, ppt))


@pytest.mark.parametrize("m,ppt", [(64, 2), (256, 8), (512, 4), (512, 16), (1024, 4)])
def test_systematic_search_jumps(gpu, O, m, ppt):
    """Systematic selection where a thread's consecutive positions cross many
    cumulative-sum entries (spikes among zeros, geometric and heavy-tailed
    weights) or none (all weight on one particle)."""
    rng = np.random.default_rng(7 * m + ppt)
    w = np.zeros((7, m), np.float32)
    w[0, rng.choice(m, 3, replace=False)] = [1.0, 5.0, 0.5]
    w[1] = 0.5 ** np.arange(m, dtype=np.float64)
    w[2, m // 2] = 1.0
    w[3] = 1.0
    w[4] = rng.exponential(1, m) ** 8
    w[5, -1] = 1e-30
    w[6, ::17] = rng.random(len(w[6, ::17]))
    us = rng.random(7).astype(np.float32)
    assert np.array_equal(gpu.resample(1, w.ravel(), us, m, ppt), O.resample(1, w.ravel(), us, m, ppt))


@pytest.mark.parametrize("tag", ["1_8_32_3", "2_2048_512_2", "2_1024_256_1", "2_12_64_4", "3_16_64_5"])
def test_exchange_routing_bit_exact(gpu, golden, tag):
    mode, N, m, t = map(int, tag.split("_"))
    keys = golden.get("exch_keys_" + tag)
    src = gpu.exchange_sources(mode, N, m, t, keys).reshape(N, m)
    nx = 4 * t if mode == 2 else t
    assert np.array_equal(src[:, m - nx:], golden["exch_src_" + tag])
    assert np.array_equal(src[:, :m - nx], np.arange(N * m).reshape(N, m)[:, :m - nx])


def _angle_close(a, b, atol):
    return np.all(np.abs(np.angle(np.exp(1j * (a.astype(np.float64) - b)))) < atol)


@pytest.mark.parametrize("model", [0, 1, 2])
def test_model_step_vs_oracle(gpu, O, model):
    rng = np.random.default_rng(model)
    n = 4096
    if model == 0:
        p = gpu.unicycle_params(1)
        st = np.stack([rng.normal(0, 3, n), rng.normal(0, 3, n), rng.uniform(-3.1, 3.1, n)]).astype(np.float32)
        inp, _ = gpu.make_trace(0, p, 1, 30)
        rec = inp[29]
    elif model == 1:
        p = gpu.dharm_params(3)
        st = np.concatenate([rng.uniform(-3, 3, (6, n)), rng.normal(0, 0.5, (6, n))]).astype(np.float32)
        inp, tr = gpu.make_trace(1, p, 3, 30)
        rec = inp[29]
        st[:, : n // 2] = (tr[28][:, None] + rng.normal(0, 0.01, (12, n // 2))).astype(np.float32)
    else:
        p = gpu.refarm_params(1.0)
        st = np.concatenate([np.full((5, n), 0.75 * np.pi) + rng.normal(0, 0.1, (5, n)),
                             rng.normal(7, 0.3, (1, n)), rng.normal(0, 0.3, (3, n))]).astype(np.float32)
        rec = np.zeros(1, gpu.STEP_INPUT_DTYPE)[0]
        rec["dt"] = 1.0
        rec["control"][:5] = rng.normal(0, 0.05, 5)
        rec["meas"][:7] = np.concatenate([np.full(5, 0.75 * np.pi), [7.0, 0.0]])
    S, K, Cn, Z = gpu.model_info(model)
    nz = rng.standard_normal((K, n)).astype(np.float32)
    gs, gl = gpu.model_step(model, p, rec, st, nz)
    md = O.model_from_params(model, p)
    os_, ol = O.model_step(md, st, nz, rec["control"][:max(Cn, 1)], rec["meas"][:Z], dt=float(rec["dt"]))
    ang = {0: [2], 1: list(range(6)), 2: list(range(5))}[model]
    for v in range(S):
        if v in ang:
            assert _angle_close(gs[v], os_[v], 2e-5), v
        else:
            assert np.allclose(gs[v], os_[v], atol=2e-5, rtol=1e-5), v
    # FP32 log-likelihood vs FP64 oracle: relative 1e-4 plus an absolute floor
    assert np.all(np.abs(gl - ol) <= 1e-4 * np.abs(ol) + 5e-3), np.max(np.abs(gl - ol) / (np.abs(ol) + 1))


@pytest.mark.parametrize("log_weights", [1, 0])
def test_estimate_entry_point_vs_fp64(gpu, log_weights):
    rng = np.random.default_rng(21 + log_weights)
    m, nsub, S = 256, 37, 3
    T = m * nsub
    st = np.stack([rng.normal(0, 2, T), rng.normal(1, 3, T), rng.uniform(-np.pi, np.pi, T)]).astype(np.float32)
    keys = (rng.normal(-50, 20, T) if log_weights else rng.exponential(1, T)).astype(np.float32)
    keys[5 * m + 17] = keys.max() + 1  # unique winner
    e = gpu.estimate(keys, st, m, angle_mask=0b100, log_weights=log_weights)
    w = np.exp(keys.astype(np.float64) - keys.max()) if log_weights else keys.astype(np.float64)
    W = w.sum()
    assert np.allclose(e["mean"][:2], (w[None] * st[:2]).sum(1) / W, rtol=1e-6, atol=1e-6)
    th = np.arctan2((w * np.sin(st[2])).sum(), (w * np.cos(st[2])).sum())
    assert abs(np.angle(np.exp(1j * (e["mean"][2] - th)))) < 1e-5
    ln = (keys.max() + np.log(W)) if log_weights else np.log(W)
    assert abs(e["log_norm"] - ln) < 1e-5 * abs(ln) + 1e-5
    assert e["best_subfilter"] == 5 and np.array_equal(e["best"][:3], st[:, 5 * m + 17])


def test_bounded_wait_reports_timeout_and_context_survives(gpu):
    """A kernel's bounded wait on an mbarrier phase that nothing completes gives
    up, reports the timeout bit, and the context stays usable afterwards."""
    assert gpu.bounded_wait_test(2000) == 1
    keys = np.arange(512, dtype=np.float32)[::-1].copy()
    k, i = gpu.bitonic_sort(keys[::-1].copy(), 512, 4)
    assert np.array_equal(k, keys) and np.array_equal(i, np.arange(512)[::-1])


@pytest.mark.parametrize("nthreads,give_up", [(128, [5]), (256, [0, 31, 200]), (512, list(range(0, 512, 2)))])
def test_bounded_wait_is_cta_wide_with_copies_in_flight(gpu, nthreads, give_up):
    """Some threads' waits run out (poll limit 0, set on the host) while the
    others see the bulk copy land: every thread must take the same branch, and
    the copy must have landed in shared memory before the block went on."""
    limits = np.full(nthreads, 1 << 18, np.int32)
    limits[give_up] = 0
    out, copied = gpu.bounded_wait_mixed_test(limits)
    assert np.all(out == out[0]), np.unique(out)
    assert out[0] == 0 and copied == 1
    # no thread gives up: the first wait succeeds everywhere
    out, copied = gpu.bounded_wait_mixed_test(np.full(nthreads, 1 << 18, np.int32))
    assert np.all(out == 1) and copied == 1
    # the context is still usable
    keys = np.arange(256, dtype=np.float32)
    k, _ = gpu.bitonic_sort(keys, 256, 4)
    assert np.array_equal(k, keys[::-1])
