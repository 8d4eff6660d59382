"""The oracle's sub-filter primitives: committed golden vectors (the sort,
multinomial and ring vectors pinned to the reference's own CUDA kernels) and
independent pure-Python restatements of the reference loops."""
from pathlib import Path

import numpy as np
import pytest

import refpy


@pytest.mark.parametrize("m", [32, 64, 256, 512])
def test_sort_golden(O, golden, m):
    k, i = O.bitonic_sort(golden["sort_in_%d" % m], m)
    assert np.array_equal(k, golden["sort_key_%d" % m])
    assert np.array_equal(i, golden["sort_idx_%d" % m])
    for b in range(4):
        kb = k[b * m:(b + 1) * m]
        assert np.all(kb[:-1] >= kb[1:])
        assert np.array_equal(np.sort(i[b * m:(b + 1) * m]), np.arange(m))
        assert np.array_equal(golden["sort_in_%d" % m][b * m:(b + 1) * m][i[b * m:(b + 1) * m]], kb)


@pytest.mark.parametrize("m", [2, 4, 8, 32, 64])
def test_sort_matches_python_network(O, m):
    rng = np.random.default_rng(m)
    for trial in range(6):
        keys = rng.integers(0, 4, m).astype(np.float32)  # heavy ties exercise the swap-on-equal rule
        pk, pi = refpy.bitonic_desc(keys)
        ok, oi = O.bitonic_sort(keys, m)
        assert np.array_equal(pk, ok) and np.array_equal(pi, oi)


def test_sort_swaps_equal_keys(O):
    # dir = 0 swaps when !(a > b): all-equal input is NOT left in place
    k, i = O.bitonic_sort(np.ones(8, np.float32), 8)
    pk, pi = refpy.bitonic_desc(np.ones(8))
    assert np.array_equal(i, pi)
    assert not np.array_equal(i, np.arange(8))


@pytest.mark.parametrize("m", [4, 32, 64])
def test_blelloch_matches_python(O, m):
    rng = np.random.default_rng(m + 1)
    w = rng.exponential(1, m).astype(np.float32)
    e, t = O.blelloch(w)
    pe, pt = refpy.blelloch(w)
    assert np.array_equal(e, pe) and np.float32(t) == pt


def test_blelloch_known_answer(O):
    e, t = O.blelloch(np.array([1, 2, 3, 4], np.float32))
    assert list(e) == [0, 1, 3, 6] and t == 10


@pytest.mark.parametrize("m", [32, 64, 256, 512])
def test_resample_ref_golden(O, golden, m):
    sel = O.resample(O.RES_REF, golden["res_w_%d" % m], golden["res_uref_%d" % m], m, 2)
    assert np.array_equal(sel, golden["res_ref_%d" % m])
    if m <= 64:
        w, u = golden["res_w_%d" % m], golden["res_uref_%d" % m]
        py = np.concatenate([refpy.resample_ref(w[b * m:(b + 1) * m], u[b * m:(b + 1) * m]) for b in range(4)])
        assert np.array_equal(sel, py)


@pytest.mark.parametrize("m,ept", [(32, 1), (64, 2), (256, 2), (256, 4), (512, 2), (512, 4)])
def test_resample_systematic_golden(O, golden, m, ept):
    w, u = golden["res_w_%d" % m], golden["res_usys_%d" % m]
    sel = O.resample(O.RES_SYSTEMATIC, w, u, m, ept)
    assert np.array_equal(sel, golden["res_sys_%d_%d" % (m, ept)])
    if m <= 64:
        py = np.concatenate([refpy.resample_systematic(w[b * m:(b + 1) * m], u[b], ept) for b in range(4)])
        assert np.array_equal(sel, py)


def test_scan_f64_matches_python(O):
    rng = np.random.default_rng(3)
    for m, ept in [(32, 1), (64, 2), (256, 4), (1024, 2)]:
        w = rng.exponential(1, m).astype(np.float32)
        cum, tot = O.scan_f64(w, m, ept)
        assert list(cum) == refpy.scan_f64(w, ept)
        assert abs(tot - float(np.sum(w.astype(np.float64)))) < 1e-9 * m


def test_systematic_offspring_counts(O):
    # systematic property: offspring count of slot j is floor or ceil of m * w_j / W
    rng = np.random.default_rng(9)
    m = 512
    w = rng.exponential(1, m).astype(np.float32)
    sel = O.resample(O.RES_SYSTEMATIC, w, rng.random(1).astype(np.float32), m, 2)
    cnt = np.bincount(sel, minlength=m)
    e = m * w.astype(np.float64) / w.astype(np.float64).sum()
    assert np.all(cnt >= np.floor(e) - 1e-9) and np.all(cnt <= np.ceil(e) + 1e-9)


@pytest.mark.parametrize("m", [32, 64, 256, 512])
def test_vose_golden(O, golden, m):
    w = golden["res_w_%d" % m]
    p, a = O.vose_build(w, m)
    assert np.array_equal(p, golden["vose_prob_%d" % m]) and np.array_equal(a, golden["vose_alias_%d" % m])
    sel = O.resample(O.RES_VOSE, w, golden["res_uvose_%d" % m], m, 2)
    assert np.array_equal(sel, golden["res_vose_%d" % m])
    if m <= 64:
        for b in range(4):
            pp, pa = refpy.vose_build(w[b * m:(b + 1) * m])
            assert np.array_equal(pp, p[b * m:(b + 1) * m]) and np.array_equal(pa, a[b * m:(b + 1) * m])


def test_vose_reproduces_distribution(O):
    # alias table: P(select j) = (prob_j + sum_{i: alias_i = j, i != j} (1 - prob_i)) / m
    rng = np.random.default_rng(11)
    m = 256
    w = rng.exponential(1, m).astype(np.float32) ** 3
    p, a = O.vose_build(w, m)
    pc = np.clip(p.astype(np.float64), 0, 1)
    mass = pc.copy()
    for i in range(m):
        if a[i] != i:
            mass[a[i]] += 1 - pc[i]
    assert np.allclose(mass / m, w / w.sum(), atol=2e-6)


def test_vose_uniform_fallback(O):
    p, a = O.vose_build(np.zeros(64, np.float32), 64)
    assert np.all(p == 1.0) and np.array_equal(a, np.arange(64))


@pytest.mark.parametrize("tag", ["1_8_32_3", "2_2048_512_2", "2_1024_256_1", "2_12_64_4", "3_16_64_5"])
def test_exchange_golden(O, golden, tag):
    mode, N, m, t = map(int, tag.split("_"))
    keys = golden.get("exch_keys_" + tag)
    src = O.exchange_sources(mode, N, m, t, keys).reshape(N, m)
    nx = 4 * t if mode == 2 else t
    assert np.array_equal(src[:, m - nx:], golden["exch_src_" + tag])
    assert np.array_equal(src[:, :m - nx], np.arange(N * m).reshape(N, m)[:, :m - nx])
    if N * m <= 4096:
        assert np.array_equal(src.reshape(-1), refpy.exchange_sources(mode, N, m, t, keys))


def test_torus_dims_reference_formula(O):
    # dx = 2^floor(log2 sqrt N), dy = N / dx (pf_generic.cu:682-683)
    for N in (1, 2, 8, 16, 1024, 2048, 4096, 12):
        dx = int(2 ** np.floor(np.log2(np.sqrt(N))))
        assert O.torus_dims(N) == (dx, N // dx) == refpy.torus_dims(N)
    assert O.torus_dims(2048) == (32, 64) and O.torus_dims(1024) == (32, 32)


def test_boxmuller_formula(O):
    rng = np.random.default_rng(5)
    u = (1 + rng.random(1000)).astype(np.float32)
    z = O.boxmuller(u)
    u1 = 2.0 - u[0::2].astype(np.float64)
    u2 = 2.0 - u[1::2].astype(np.float64)
    r = np.sqrt(-2 * np.log(u1))
    assert np.allclose(z[0::2], r * np.cos(2 * np.pi * u2), atol=1e-6)
    assert np.allclose(z[1::2], r * np.sin(2 * np.pi * u2), atol=1e-6)


@pytest.mark.parametrize("m", [32, 64, 256, 512])
def test_golden_pinned_to_reference_kernels(golden, m):
    """The committed sort / multinomial golden vectors equal what the
    reference's own CUDA kernels (block_sort, resampling) produced on the same
    inputs (tests/golden/make_ref_kernel_golden.py, run on a GPU)."""
    ref = np.load(Path(__file__).resolve().parent / "golden" / "ref_kernels.npz")
    assert np.array_equal(golden["sort_key_%d" % m], ref["sort_key_%d" % m])
    assert np.array_equal(golden["sort_idx_%d" % m], ref["sort_idx_%d" % m])
    assert np.array_equal(golden["res_ref_%d" % m], ref["res_ref_%d" % m])


def test_ring_golden_pinned_to_reference_kernel(golden):
    ref = np.load(Path(__file__).resolve().parent / "golden" / "ref_kernels.npz")
    assert np.array_equal(golden["exch_src_1_8_32_3"], ref["exch_src_1_8_32_3"])


def test_oracle_expneg_accuracy(O):
    """orc_expneg (the resampling weights' exponential, bit-identical to the
    engine's) is within 2 ulp of exp on [-87, 0], 0 below, NaN for NaN."""
    rng = np.random.default_rng(5)
    x = np.concatenate([-rng.exponential(3.0, 20000), -rng.uniform(0, 87, 20000), [0.0, -1e-30, -87.0]])
    x = x.astype(np.float32)
    got = O.expneg(x).astype(np.float64)
    ref = np.exp(x.astype(np.float64))
    assert np.max(np.abs(got - ref) / np.spacing(ref.astype(np.float32))) <= 2.0
    e = O.expneg(np.float32([-87.5, -100.0, -np.inf, np.nan]))
    assert np.all(e[:3] == 0) and np.isnan(e[3])


def test_exp_fit_script_checks_pass():
    import importlib.util
    from pathlib import Path
    spec = importlib.util.spec_from_file_location(
        "fit_exp", Path(__file__).resolve().parents[1] / "esthera_b200" / "csrc" / "fit_exp.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    assert m.main([]) == 0
