"""The engine's CUDA sort, multinomial resampling, ring routing and Vose alias
build -- and the CPU oracle -- against the reference's OWN kernels: the CUDA
block_sort with its bitonic network, resampling with prefix_sum +
binary_search and exchange_ring (pf_generic_soa.cu / bitonic-sort.cu, built
into oracle/_ref/libref_kernels.so by oracle/build_ref_kernels.sh) and the
OpenCL Vose resampler (resampling-valias.cl, compiled as CUDA into
oracle/_ref/libref_valias.so by oracle/build_ref_valias.sh), run on the same
GPU.  Inputs: seeded random keys with heavy ties, positive weights with zeros,
MTGP-style uniforms in [1, 2)."""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent.parent / "oracle"))
import ref_kernels as R  # noqa: E402

pytestmark = pytest.mark.gpu


def _require(built, lib, recipe):
    """The reference's own kernels are the strongest parity evidence: a missing
    library fails the test instead of skipping it (build() makes them wherever
    the Esthera tree is present, and the built files travel with the tree)."""
    if not built:
        pytest.fail("oracle/_ref/%s is missing: run oracle/%s (needs the Esthera tree)" % (lib, recipe))


@pytest.fixture(autouse=True)
def _reference_kernels_built():
    _require(R.available(), "libref_kernels.so", "build_ref_kernels.sh")

PPT = {32: [1], 64: [2], 128: [2, 4], 256: [2, 4, 8], 512: [2, 4, 16], 1024: [2, 4]}


def _uniforms_1_2(rng, n):
    return (1.0 + rng.integers(0, 1 << 23, n) / float(1 << 23)).astype(np.float32)  # exact in FP32


@pytest.mark.parametrize("m", [32, 64, 128, 256, 512, 1024])
def test_sort_equals_reference_kernel(gpu, O, m):
    E = gpu
    rng = np.random.default_rng(100 + m)
    nsub = 6
    keys = np.round(rng.standard_normal(nsub * m) * 3).astype(np.float32) / 3  # ties
    keys[::7] = -np.inf
    rk, rp = R.block_sort(keys, m)
    ok, op = O.bitonic_sort(keys, m)
    assert np.array_equal(rk, ok) and np.array_equal(rp, op)
    for ppt in PPT[m]:
        k, p = E.bitonic_sort(keys, m, ppt)
        assert np.array_equal(k, rk) and np.array_equal(p, rp), ppt


@pytest.mark.parametrize("m", [32, 64, 128, 256, 512, 1024])
def test_rank_sort_equals_reference_kernel(gpu, m):
    """The sampling kernels' sort for small-state models (keys-only network +
    rank, falling back to the full network on ties) against the reference's
    block_sort: distinct keys (no fallback), and sub-filters with ties, -inf,
    +0/-0 and NaN (every one of them falls back)."""
    E = gpu
    rng = np.random.default_rng(300 + m)
    nsub = 8
    keys = ((rng.permutation(nsub * m) - 0.5 * nsub * m) * 0.013).astype(np.float32)  # distinct
    b = keys.reshape(nsub, m)
    b[1, 5] = b[1, 9]                     # a tie
    b[2, ::3] = -np.inf                   # repeated -inf
    b[3, 0], b[3, 1] = 0.0, -0.0          # +0 / -0
    b[4, 7] = np.nan                      # NaN
    b[5, :] = np.round(b[5, :])           # many ties
    rk, rp = R.block_sort(keys, m)
    for ppt in PPT[m]:
        k, p, fb = E.rank_sort(keys, m, ppt)
        assert fb == 5, (ppt, fb)
        assert np.array_equal(k.view(np.uint32), rk.view(np.uint32)) and np.array_equal(p, rp), ppt
    # all distinct: no sub-filter falls back
    d = (rng.permutation(nsub * m).astype(np.float32) - 7.5) * 0.37
    rk, rp = R.block_sort(d, m)
    for ppt in PPT[m]:
        k, p, fb = E.rank_sort(d, m, ppt)
        assert fb == 0 and np.array_equal(k, rk) and np.array_equal(p, rp), ppt


@pytest.mark.parametrize("m", [32, 64, 128, 256, 512, 1024])
def test_multinomial_equals_reference_kernel(gpu, O, m):
    E = gpu
    rng = np.random.default_rng(200 + m)
    nsub = 6
    w = rng.exponential(1.0, nsub * m).astype(np.float32)
    w[rng.random(nsub * m) < 0.3] = 0.0
    u = _uniforms_1_2(rng, nsub * m)
    ref = R.resampling(w, u, m)
    assert np.array_equal(O.resample(O.RES_REF, w, u, m, 2), ref)
    for ppt in PPT[m]:
        assert np.array_equal(E.resample(E.RESAMPLE_REFERENCE, w, u, m, ppt), ref), ppt


def test_multinomial_skip_rule_of_reference_kernel(gpu):
    """A sub-filter whose decision uniform exceeds resampling_freq is left alone
    (pf_generic_soa.cu:423-429): -1 here, as the engine records it."""
    rng = np.random.default_rng(3)
    m, nsub = 64, 4
    w = rng.exponential(1.0, nsub * m).astype(np.float32)
    u = _uniforms_1_2(rng, nsub * m)
    dec = np.array([1.1, 1.9, 1.5, 1.2], np.float32)
    sel = R.resampling(w, u, m, dec, freq=0.5).reshape(nsub, m)
    assert np.all(sel[1] == -1) and np.all(sel[[0, 2, 3]] >= 0)


@pytest.mark.parametrize("N,m,t", [(8, 32, 3), (16, 256, 2), (5, 64, 32)])
def test_ring_routing_equals_reference_kernel(gpu, O, N, m, t):
    E = gpu
    keys = -np.sort(-np.random.default_rng(N + m).standard_normal((N, m)).astype(np.float32), axis=1).reshape(-1)
    rk, rsrc = R.exchange_ring(keys, m, t)
    assert np.array_equal(E.exchange_sources(E.EXCHANGE_RING, N, m, t), rsrc)
    assert np.array_equal(O.exchange_sources(O.EXCH_RING, N, m, t), rsrc)
    assert np.array_equal(rk, keys[rsrc])


def test_refarm_model_equals_reference_kernel(gpu):
    """The engine's reference-arm model (propagate + log-likelihood) against the
    reference's sampling_importance / sampling_iw on the same particles, normals,
    controls and measurements: states within 2e-5, log-likelihoods within
    1e-4 relative + 5e-3 absolute (FP32, different operation order)."""
    E = gpu
    rng = np.random.default_rng(11)
    n = 2048
    p = E.refarm_params(1.0)
    st = np.zeros((9, n), np.float32)
    st[:5] = (0.75 * np.pi + 0.3 * rng.standard_normal((5, n))).astype(np.float32)
    st[5] = (7.0 + rng.standard_normal(n)).astype(np.float32)
    st[6] = rng.standard_normal(n).astype(np.float32)
    st[7:] = rng.standard_normal((2, n)).astype(np.float32)
    nz = rng.standard_normal((9, n)).astype(np.float32)
    inp = np.zeros(1, E.STEP_INPUT_DTYPE)[0]
    inp["dt"] = 0.1
    inp["control"][:5] = rng.uniform(-0.5, 0.5, 5)
    inp["meas"][:5] = (0.75 * np.pi + 0.2 * rng.standard_normal(5)).astype(np.float32)
    inp["meas"][5:7] = [7.0, 0.5]
    so, ll = E.model_step(E.MODEL_REFARM, p, inp, st, nz)
    sr, w = R.sampling_importance(st, nz, inp["control"], inp["meas"], 0.1)
    assert np.allclose(so, sr, atol=2e-5, rtol=0)
    ok = w > 1e-30
    assert ok.mean() > 0.5
    lr = np.log(w[ok].astype(np.float64))
    assert np.allclose(ll[ok], lr, rtol=1e-4, atol=5e-3)


@pytest.mark.parametrize("w0,dt", [(0.2, 1.0), (-0.6, 0.5), (1.5, 1.0)])
def test_beacon_model_equals_reference_kernel(gpu, w0, dt):
    """The engine's beacon model against the reference unicycle program's own
    sampling_importance (sampling + importance_weight, particle_filter.cu:314-455)
    on the same particles, normals, controls and ranges.  States: within 2e-5
    plus the reference's own FP32 rounding of v/w (sin(th + w dt) - sin th),
    16 |v/w| 2^-24 (its argument th + w dt rounded to FP32, |th + w dt| < 8,
    and one ulp of each sine; the engine evaluates the arc without that
    difference); log-likelihoods within 1e-4 relative + 5e-3 absolute of
    log(weight)."""
    _require(R.unicycle_available(), "libref_unicycle.so", "build_ref_unicycle.sh")
    E = gpu
    rng = np.random.default_rng(int(100 * abs(w0)) + int(10 * dt))
    n = 4096
    p = E.beacon_params()
    # a cloud around (17, 30) tight enough that the weights stay representable
    st = np.stack([rng.normal(17, 0.5, n), rng.normal(30, 0.5, n), rng.uniform(-3.1, 3.1, n)]).astype(np.float32)
    nz = rng.standard_normal((3, n)).astype(np.float32)
    inp = np.zeros(1, E.STEP_INPUT_DTYPE)[0]
    inp["dt"] = dt
    inp["control"][:2] = [0.3, w0]
    bx = np.array([p.beacons[j][0] for j in range(10)], np.float64)
    by = np.array([p.beacons[j][1] for j in range(10)], np.float64)
    inp["meas"][:10] = np.sqrt((17 - bx) ** 2 + (30 - by) ** 2 + 9) + rng.normal(0, 0.5, 10)
    so, ll = E.model_step(E.MODEL_BEACON, p, inp, st, nz)
    sr, wt = R.unicycle_sampling(st, nz, 0.3, w0, dt, inp["meas"][:10])
    v = 0.3 + 0.5 * nz[0].astype(np.float64)
    w = w0 + 0.1 * nz[1].astype(np.float64)
    tol = 2e-5 + 16.0 * np.abs(v / w) * 2.0 ** -24
    assert np.all(np.abs(so[0] - sr[0]) <= tol) and np.all(np.abs(so[1] - sr[1]) <= tol)
    # the engine wraps the heading to [-pi, pi); the program does not
    assert np.all(np.abs(np.angle(np.exp(1j * (so[2].astype(np.float64) - sr[2])))) < 2e-5)
    ok = wt > 1e-30
    assert ok.mean() > 0.5
    lr = np.log(wt[ok].astype(np.float64))
    assert np.allclose(ll[ok], lr, rtol=1e-4, atol=5e-3)


@pytest.mark.parametrize("ang", [1.2, 2.0])
def test_camarm_model_equals_reference_kernel(gpu, O, ang):
    """The engine's camera-arm model against the reference's own pinhole-camera
    sampling_iw (pf_model_soa_packed_code.cuh:61-145) on the same particles,
    normals, controls and pixel measurements: states within 2e-5,
    log-likelihoods within 1e-4 relative + 5e-3 absolute of log(weight)."""
    _require(R.camarm_available(), "libref_camarm.so", "build_ref_camarm.sh")
    import test_camarm as T
    E = gpu
    p = E.camarm_params()
    rng = np.random.default_rng(int(ang * 100))
    n = 4096
    # a cloud tight enough that most weights exp(-value) stay above FP32 underflow
    st = T.cloud(rng, n, ang, 0.01)
    nz = (0.02 * rng.standard_normal((9, n))).astype(np.float32)
    inp = np.zeros(1, E.STEP_INPUT_DTYPE)[0]
    inp["dt"] = 1.0
    inp["control"][:5] = rng.normal(0, 0.002, 5)
    inp["meas"][:7] = T.measurement(O, p, ang)
    so, ll = E.model_step(E.MODEL_CAMARM, p, inp, st, nz)
    sr, wt = R.camarm_sampling(st, nz, inp["control"], inp["meas"], 1.0)
    assert np.allclose(so, sr, atol=2e-5, rtol=0)
    ok = wt > 1e-30
    assert ok.mean() > 0.5
    lr = np.log(wt[ok].astype(np.float64))
    assert np.allclose(ll[ok], lr, rtol=1e-4, atol=5e-3)


@pytest.mark.parametrize("m", [32, 64, 128, 256, 512, 1024])
def test_vose_pinned_to_reference_kernel(gpu, O, m):
    """The engine's Vose alias build and the oracle's against the reference's own
    resampling-valias.cl (run on this GPU through oracle/build_ref_valias.sh).
    The reference fills its work lists with atomics, so its tables' order is
    the hardware's; compared are the parts that do not depend on it:
    (1) the normalised, scaled starting probabilities, bit for bit (and the
    engine's final probabilities of the slots that start small, which the
    pairing never changes); (2) each slot's selection probability implied by
    the finished tables, within FP32 rounding; (3) the draw rule on the
    reference's own tables, bit for bit."""
    _require(R.valias_available(), "libref_valias.so", "build_ref_valias.sh")
    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    import make_ref_valias_golden as G
    E = gpu
    w, u2 = G.inputs(m, 1900 + m)
    scaled, rprob, ralias, rsel = R.valias(w, u2, m)
    # (1)
    assert np.array_equal(scaled.view(np.uint32), O.vose_scaled(w, m).view(np.uint32))
    for ppt in PPT[m]:
        eprob, ealias = E.vose_build(w, m, ppt)
        small = scaled <= 1.0
        assert np.array_equal(eprob[small], scaled[small]), ppt
        # (2)
        ri = O.implied_selection(rprob, ralias, m)
        ei = O.implied_selection(eprob, ealias, m)
        assert np.all(np.abs(ri - ei) <= 1e-6 + 1e-4 * ri), (ppt, np.max(np.abs(ri - ei)))
    wn = w.reshape(-1, m).astype(np.float64)
    tot = wn.sum(axis=1, keepdims=True)
    target = np.where(tot > 0, wn / np.where(tot > 0, tot, 1.0), 1.0 / m).reshape(-1)
    assert np.all(np.abs(ri - target) <= 1e-6 + 1e-4 * target)
    # (3)
    assert np.array_equal(O.vose_draws(rprob, ralias, u2, m), rsel)
