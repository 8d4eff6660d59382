"""The camera-arm model: the reference's pinhole-camera variant of the robot
arm (src/models/robotarm/cuda/pf_model_soa_packed_code.cuh:33-145: the
refarm chain, the cart's camera coordinates projected, distorted and mapped
to pixels) as a compiled-in model.

CPU: the oracle's restatement against numpy of the reference's formula, the
default calibration, and the trace reader (the robot-arm format,
pf_model_soa_packed_code.c:57-82).  GPU (through the C ABI): the model step
against the oracle, and the pipelines against each other.  The model against
the reference's own sampling_iw is in test_gpu_reference_kernels.py."""
import ctypes as C

import numpy as np
import pytest

CAM = 4


def cloud(rng, n, ang=1.2, spread=0.05):
    """Particles around angles `ang`, cart (7, 0), cart speed ~ spread: the
    camera sees the cart at a finite depth (cz away from 0)."""
    st = np.zeros((9, n), np.float32)
    st[:5] = ang + spread * rng.standard_normal((5, n))
    st[5] = 7 + 2 * spread * rng.standard_normal(n)
    st[6] = 2 * spread * rng.standard_normal(n)
    st[7:] = spread * rng.standard_normal((2, n))
    return st


def ref_formula(p, st, nz, c, z, dt):
    """The reference's sampling_iw in FP64 (states rounded to FP32 where it stores them)."""
    s = st.astype(np.float64)
    nz = np.asarray(nz, np.float64)
    x = (s[5] + s[7] * dt + nz[5] * 0.2).astype(np.float32).astype(np.float64)
    y = (s[6] + s[8] * dt + nz[6] * 0.2).astype(np.float32).astype(np.float64)
    ang = (s[:5] + np.asarray(c[:5], np.float64)[:, None] * dt + nz[:5] * 0.2).astype(np.float32).astype(np.float64)
    cx = x * np.cos(ang[0]) + y * np.sin(ang[0])
    cy = -x * np.sin(ang[0]) + y * np.cos(ang[0])
    cz = np.zeros_like(cx)
    for i in range(1, 5):
        cy, cz = cy * np.cos(ang[i]) - cz * np.sin(ang[i]), cy * np.sin(ang[i]) + cz * np.cos(ang[i]) - 3.0
    xn, yn = cx / cz, cy / cz
    k1, k2, k3, k4 = [np.float64(v) for v in p.kc]
    r2 = xn * xn + yn * yn
    dxx = 2 * k3 * xn * yn + k4 * (3 * xn * xn + yn * yn)
    dxy = k3 * (3 * yn * yn + xn * xn) + 2 * k4 * xn * yn
    xp = p.fc[0] * ((1 + k1 * r2 + k2 * r2 * r2) * xn + dxx) + p.cc[0]
    yp = p.fc[1] * ((1 + k1 * r2 + k2 * r2 * r2) * yn + dxy) + p.cc[1]
    val = np.sum((ang - np.asarray(z[:5], np.float64)[:, None]) ** 2 * 0.1, axis=0)
    val += (xp - z[5]) ** 2 * 0.1 + (yp - z[6]) ** 2 * 0.1
    return ang, x, y, -val


def measurement(O, p, ang=1.2):
    """Pixel coordinates of the cloud's centre (oracle, no noise), angles = ang."""
    md = O.model_from_params(CAM, p)
    st = np.array([ang] * 5 + [7, 0, 0, 0], np.float32)[:, None]
    z = np.zeros(7, np.float32)
    _, ll0 = O.model_step(md, st, np.zeros((9, 1), np.float32), np.zeros(5, np.float32), z)
    # recover the pixels from the oracle's own formula by probing: ll(z) = -0.1 |z - p|^2 - angle part
    ex = []
    for k in (5, 6):
        z1 = z.copy()
        z1[k] = 1.0
        _, ll1 = O.model_step(md, st.copy(), np.zeros((9, 1), np.float32), np.zeros(5, np.float32), z1)
        ex.append((ll1[0] - ll0[0] + 0.1) / 0.2)  # -0.1 (1 - p)^2 + 0.1 p^2 = 0.2 p - 0.1
    return np.array([ang] * 5 + ex, np.float32)


def test_camarm_default_calibration(E):
    p = E.camarm_params()
    assert E.model_info(CAM) == (9, 9, 5, 7)
    assert np.allclose(list(p.fc), [408.65831, 409.69059]) and np.allclose(list(p.cc), [166.32611, 108.93539])
    assert np.allclose(list(p.kc), [-0.21561, 1.60704, -0.01291, 0.00007])
    assert np.allclose(list(p.init_state), [0.75 * np.pi] * 5 + [7, 0, 0, 0]) and p.dt == 1.0


def test_camarm_oracle_reference_formula(O, E):
    p = E.camarm_params()
    md = O.model_from_params(CAM, p)
    rng = np.random.default_rng(4)
    n = 64
    st = cloud(rng, n)
    nz = (0.1 * rng.standard_normal((9, n))).astype(np.float32)
    c = rng.normal(0, 0.02, 5).astype(np.float32)
    z = measurement(O, p)
    new, ll = O.model_step(md, st, nz, c, z)
    ang, x, y, el = ref_formula(p, st, nz, c, z, 1.0)
    assert np.allclose(new[:5], ang, atol=1e-6) and np.allclose(new[5], x, atol=1e-6)
    assert np.allclose(new[6], y, atol=1e-6)
    assert np.allclose(ll, el, rtol=1e-9, atol=1e-9)


def test_camarm_trace_reader(E, tmp_path):
    vals = [150.5, 99.25] + [1.0, 1.1, 1.2, 1.3, 1.4] + [0.01, -0.02, 0.03, -0.04, 0.05] + [1, 0.7, 0.8] + \
           [1.01, 1.11, 1.21, 1.31, 1.41]
    fn = tmp_path / "trace"
    fn.write_text(" ".join(map(str, vals)) + "\n")
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    fp = libc.fopen(str(fn).encode(), b"r")
    inp = E.StepInput()
    act = np.zeros(16, np.float32)
    assert E.lib().pf_read_trace_line(fp, CAM, C.byref(inp), act.ctypes.data_as(C.POINTER(C.c_float))) == 0
    libc.fclose(fp)
    assert np.allclose(inp.meas[:7], [1.0, 1.1, 1.2, 1.3, 1.4, 150.5, 99.25])
    assert np.allclose(inp.control[:5], [0.01, -0.02, 0.03, -0.04, 0.05]) and inp.dt == 1.0


@pytest.mark.gpu
@pytest.mark.parametrize("ang", [1.2, 2.0])
def test_camarm_model_step_vs_oracle(gpu, O, ang):
    E = gpu
    p = E.camarm_params()
    rng = np.random.default_rng(int(ang * 10))
    n = 4096
    st = cloud(rng, n, ang)
    nz = (0.1 * rng.standard_normal((9, n))).astype(np.float32)
    rec = np.zeros(1, E.STEP_INPUT_DTYPE)[0]
    rec["dt"] = 1.0
    rec["control"][:5] = rng.normal(0, 0.02, 5)
    rec["meas"][:7] = measurement(O, p, ang)
    gs, gl = E.model_step(CAM, p, rec, st, nz)
    os_, ol = O.model_step(O.model_from_params(CAM, p), st, nz, rec["control"][:5], rec["meas"][:7], dt=1.0)
    assert np.all(np.abs(np.angle(np.exp(1j * (gs[:5].astype(np.float64) - os_[:5])))) < 2e-5)
    assert np.allclose(gs[5:], os_[5:], atol=2e-5, rtol=1e-6)
    # FP32 log-likelihood vs the FP64 oracle: relative 1e-4 plus an absolute floor
    assert np.all(np.abs(gl - ol) <= 1e-4 * np.abs(ol) + 5e-3), np.max(np.abs(gl - ol))


@pytest.mark.gpu
@pytest.mark.parametrize("res", [0, 1, 2])
def test_camarm_pipelines_agree(gpu, O, res):
    """Single-kernel and split pipelines bit for bit; phased and split on the
    reference random layout likewise; every estimate finite."""
    E = gpu
    p = E.camarm_params()
    for i in range(5):
        p.init_state[i] = 1.2
    z = measurement(O, p)
    rec = np.zeros(4, E.STEP_INPUT_DTYPE)
    rec["dt"] = 1.0
    rec["meas"][:, :7] = z
    common = dict(particles_per_subfilter=256, num_subfilters=16, num_transfer=1, exchange=1, resampler=res,
                  log_weights=1)
    a = E.ParticleFilter(CAM, p, pipeline=E.PIPELINE_FUSED, **common)
    b = E.ParticleFilter(CAM, p, pipeline=E.PIPELINE_SPLIT, **common)
    c = E.ParticleFilter(CAM, p, pipeline=E.PIPELINE_SPLIT, rng=E.RNG_REFLAYOUT, mtgp_streams=96, **common)
    d = E.ParticleFilter(CAM, p, pipeline=E.PIPELINE_PHASED, rng=E.RNG_REFLAYOUT, mtgp_streams=96, **common)
    for k in range(4):
        x, y = a.step(rec[k]), b.step(rec[k])
        assert x["flags"] == 0 and np.all(np.isfinite(x["mean"][:9]))
        assert np.array_equal(x["mean"], y["mean"]) and x["log_norm"] == y["log_norm"], k
        assert np.array_equal(x["best"], y["best"]) and x["best_subfilter"] == y["best_subfilter"], k
        u, w = c.step(rec[k]), d.step(rec[k])
        assert np.array_equal(u["best"], w["best"]) and u["best_subfilter"] == w["best_subfilter"], k
        assert np.allclose(u["mean"], w["mean"], rtol=1e-12, atol=1e-12), k
    assert np.array_equal(a.particles(), b.particles())


@pytest.mark.gpu
def test_camarm_batch_and_server_equal_single_filters(gpu, O):
    """Camera-arm filters in a batch and in the server reproduce pf_filter bit for bit."""
    E = gpu
    p = E.camarm_params()
    for i in range(5):
        p.init_state[i] = 2.0
    rec = np.zeros(4, E.STEP_INPUT_DTYPE)
    rec["dt"] = 1.0
    rec["meas"][:, :7] = measurement(O, p, 2.0)
    counts = [512, 256]
    cfg = dict(num_transfer=1, exchange=1, resampler=1, particles_per_thread=4)
    B = E.FilterBatch(CAM, [p, p], counts, particles_per_subfilter=256, **cfg)
    best = [B.step(np.stack([rec[k], rec[k]])) for k in range(4)]
    for f, n in enumerate(counts):
        s = E.ParticleFilter(CAM, p, pipeline=E.PIPELINE_SPLIT, particles_per_subfilter=256, num_subfilters=n // 256,
                             stream_offset=B.filter_info(f)["stream_offset"], **cfg)
        for k in range(4):
            e = s.step(rec[k])
            assert np.array_equal(best[k][f]["mean"], e["mean"]) and best[k][f]["log_norm"] == e["log_norm"], (f, k)
    srv = E.Server(1 << 30, 4, particles_per_subfilter=256, particles_per_thread=4, num_transfer=1, exchange=1)
    fid = srv.open(CAM, p, 512, 9)
    s = E.ParticleFilter(CAM, p, pipeline=E.PIPELINE_SPLIT, particles_per_subfilter=256, num_subfilters=2, seed=9,
                         particles_per_thread=4, num_transfer=1, exchange=1)
    for k in range(4):
        srv.update(fid, rec[k], tag=k)
        srv.launch()
        r = srv.poll()[0]["estimate"]
        e = s.step(rec[k])
        assert np.array_equal(r["mean"], e["mean"]) and r["log_norm"] == e["log_norm"], k
    srv.close()
