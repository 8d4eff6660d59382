"""The beacon model: the reference's unicycle program (src/models/unicycle/
particle_filter.cu:314-359, noisy velocity and turn rate, arc motion, weight
from the ranges to ten fixed 3-D beacons) as a compiled-in model.

CPU: the oracle's restatement against numpy of the reference's own difference
form, the default constants, the trace format of the program's reader
(particle_filter.cu:756-772) and its error (:1044), and the oracle filter
tracking a seeded trace.  GPU (through the C ABI): the model step against the
oracle, the first filter step against the oracle, the pipelines against each
other, RMSE against the oracle's, the program's drop-in loop, batches and the
server."""
import ctypes as C

import numpy as np
import pytest

BEACON = 3
BX = [12, 12, 13, 14, 16, 16, 18, 20, 20, 20]
BY = [12, 37, 25, 18, 12, 37, 30, 12, 25, 37]


def ref_formula(st, nz, v0, w0, dt, noise, z, beacons, sigma):
    """The reference's sampling + importance_weight in FP64, heading wrapped."""
    x, y, th = st.astype(np.float64)
    v = v0 + noise[0] * nz[0].astype(np.float64)
    w = w0 + noise[1] * nz[1].astype(np.float64)
    g = noise[2] * nz[2].astype(np.float64)
    nx = x + v / w * (np.sin(th + w * dt) - np.sin(th))
    ny = y - v / w * (np.cos(th + w * dt) - np.cos(th))
    nt = np.angle(np.exp(1j * (th + w * dt + g * dt)))
    X, Y = nx.astype(np.float32).astype(np.float64), ny.astype(np.float32).astype(np.float64)
    acc = 0.0
    for j, (bx, by, bz) in enumerate(beacons):
        e = np.sqrt((X - bx) ** 2 + (Y - by) ** 2 + bz * bz) - z[j]
        acc = acc + e * e
    L = len(beacons)
    ll = np.log(1e5) - (L // 2) * np.log(2 * np.pi) - acc / (2 * sigma * sigma)
    return nx, ny, nt, ll


def beacons_of(p):
    return [(p.beacons[j][0], p.beacons[j][1], p.beacons[j][2]) for j in range(p.num_beacons)]


def test_beacon_default_params_are_the_programs_constants(E):
    p = E.beacon_params()
    assert E.model_info(BEACON) == (3, 3, 2, 16)
    assert p.num_beacons == 10 and p.dt == 1.0
    assert [p.beacons[j][0] for j in range(10)] == BX and [p.beacons[j][1] for j in range(10)] == BY
    assert all(p.beacons[j][2] == 3.0 for j in range(10))
    assert np.allclose(list(p.noise), [0.5, 0.1, 0.01])
    assert np.isclose(p.sigma_range, np.sqrt(0.5))  # exp(-sum e^2) as a Gaussian
    assert np.allclose(list(p.init_state), [20, 40, -np.pi / 2])


def test_beacon_oracle_reference_formula(O, E):
    p = E.beacon_params()
    md = O.model_from_params(BEACON, p)
    rng = np.random.default_rng(3)
    n = 64
    st = np.stack([rng.uniform(10, 25, n), rng.uniform(10, 40, n), rng.uniform(-3, 3, n)]).astype(np.float32)
    nz = rng.standard_normal((3, n)).astype(np.float32)
    z = rng.uniform(2, 30, 10).astype(np.float32)
    v0, w0 = 0.3, 0.2
    new, ll = O.model_step(md, st, nz, [v0, w0], z)
    ex, ey, et, el = ref_formula(st, nz, v0, w0, 1.0, [0.5, 0.1, 0.01], z, beacons_of(p), np.float64(p.sigma_range))
    assert np.allclose(new[0], ex, atol=2e-6) and np.allclose(new[1], ey, atol=2e-6)
    assert np.all(np.abs(np.angle(np.exp(1j * (new[2] - et)))) < 1e-6)
    assert np.allclose(ll, el, rtol=1e-9, atol=1e-9)


def test_beacon_oracle_straight_line_limit(O, E):
    p = E.beacon_params()
    p.noise[0] = p.noise[1] = p.noise[2] = 0.0
    md = O.model_from_params(BEACON, p)
    st = np.array([[20.0], [40.0], [0.5]], np.float32)
    new, _ = O.model_step(md, st, np.zeros((3, 1), np.float32), [0.3, 0.0], np.ones(10, np.float32))
    assert np.allclose(new[:, 0], [20 + 0.3 * np.cos(0.5), 40 + 0.3 * np.sin(0.5), 0.5], atol=2e-6)


def test_half_angle_arc_equals_the_programs_difference_form():
    """The device's arc, v dt sinc(w dt / 2) (cos, sin)(th + w dt / 2), is the
    program's v/w (sin(th + w dt) - sin th, -(cos(th + w dt) - cos th)) (FP64;
    the identities sin a - sin b = 2 cos((a+b)/2) sin((a-b)/2) and
    cos a - cos b = -2 sin((a+b)/2) sin((a-b)/2)), and stays finite as w -> 0."""
    rng = np.random.default_rng(8)
    th = rng.uniform(-np.pi, np.pi, 1000)
    v = rng.uniform(0.0, 2.0, 1000)
    w = rng.uniform(-3.0, 3.0, 1000)
    dt = rng.uniform(0.05, 1.0, 1000)
    h = 0.5 * w * dt
    k = v * dt * np.sinc(h / np.pi)  # numpy's sinc is sin(pi x) / (pi x)
    assert np.allclose(k * np.cos(th + h), v / w * (np.sin(th + w * dt) - np.sin(th)), rtol=0, atol=1e-12)
    assert np.allclose(k * np.sin(th + h), -v / w * (np.cos(th + w * dt) - np.cos(th)), rtol=0, atol=1e-12)
    assert np.isclose(1.0 * 1.0 * np.sinc(0.0), 1.0)


def write_trace(path, inputs, truth):
    """The unicycle program's trace format: ranges[10] v omega dt x y theta."""
    rows = []
    for k in range(len(inputs)):
        vals = list(inputs["meas"][k][:10]) + [inputs["control"][k][0], inputs["control"][k][1], inputs["dt"][k]] + \
            list(truth[k])
        rows.append(" ".join("%.9g" % float(v) for v in vals))
    path.write_text("\n".join(rows) + "\n")


def read_trace(E, path, model=BEACON):
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    fp = libc.fopen(str(path).encode(), b"r")
    out = []
    while True:
        inp = E.StepInput()
        act = np.zeros(16, np.float32)
        if E.lib().pf_read_trace_line(fp, model, C.byref(inp), act.ctypes.data_as(C.POINTER(C.c_float))) != 0:
            break
        rec = np.zeros(1, E.STEP_INPUT_DTYPE)
        C.memmove(rec.ctypes.data, C.byref(inp), 128)
        out.append((rec[0], act[:3].copy()))
    libc.fclose(fp)
    return out


def test_beacon_trace_reader_and_error(E, tmp_path):
    p = E.beacon_params()
    inputs, truth = E.make_trace(BEACON, p, 9, 12)
    assert np.all(inputs["control"][:, 0] >= 0) and np.all(np.isfinite(inputs["meas"][:, :10]))
    fn = tmp_path / "unicycle_trace"
    write_trace(fn, inputs, truth)
    got = read_trace(E, fn)
    assert len(got) == 12
    for k, (rec, act) in enumerate(got):
        assert np.array_equal(rec["meas"][:10], inputs["meas"][k][:10])
        assert np.array_equal(rec["control"][:2], inputs["control"][k][:2]) and rec["dt"] == inputs["dt"][k]
        assert np.all(rec["meas"][10:] == 0) and np.all(rec["control"][2:] == 0)
        assert np.array_equal(act, truth[k])
    est = truth[3].copy()
    est[0] += 3.0
    est[1] -= 4.0
    f32 = C.POINTER(C.c_float)
    e = E.lib().pf_beacon_estimate_error(est.ctypes.data_as(f32), truth[3].copy().ctypes.data_as(f32))
    assert abs(e - 5.0) < 1e-5
    # a truncated line ends the trace
    fn.write_text(" ".join(["1.0"] * 15) + "\n")
    assert read_trace(E, fn) == []


def test_beacon_oracle_filter_tracks(O, E):
    p = E.beacon_params()
    inputs, truth = E.make_trace(BEACON, p, 1, 60)
    md = O.model_from_params(BEACON, p)
    f = O.Filter(md, 512, 4, 0, O.EXCH_NONE, O.RES_SYSTEMATIC, O.RNG_SUBFILTER, 96, 4, 1, 1.0, 0xF000000D, 0,
                 np.array(p.init_state[:], np.float32))
    err = []
    for k in range(60):
        e, _ = f.step(inputs["control"][k], inputs["meas"][k])
        err.append((e.mean[0] - truth[k, 0]) ** 2 + (e.mean[1] - truth[k, 1]) ** 2)
    rmse = float(np.sqrt(np.mean(err[5:])))
    assert rmse < 0.5, rmse


@pytest.mark.parametrize("log_weights", [0, 1])
def test_beacon_oracle_program_loop(O, E, log_weights):
    """The drop-in loop's configuration on the oracle: ring exchange, the
    reference's multinomial resampling (FP32 Blelloch scan) every step, the
    best particle of the best sub-filter as the estimate (linear weights as
    the program keeps them, and log weights)."""
    p = E.beacon_params()
    inputs, truth = E.make_trace(BEACON, p, 6, 40)
    f = O.Filter(O.model_from_params(BEACON, p), 256, 16, 1, O.EXCH_RING, O.RES_REF, O.RNG_SUBFILTER, 96, 4,
                 log_weights, 1.0, 0xF000000D, 0, np.array(p.init_state[:], np.float32))
    err = []
    for k in range(40):
        e, _ = f.step(inputs["control"][k], inputs["meas"][k])
        assert 0 <= e.best_sub < 16 and np.isfinite(e.best_key)
        err.append(np.hypot(e.best[0] - truth[k, 0], e.best[1] - truth[k, 1]))
    assert np.mean(err) < 2.0, np.mean(err)


# ---------------------------------------------------------------- GPU
def _angle_close(a, b, atol):
    return np.all(np.abs(np.angle(np.exp(1j * (a.astype(np.float64) - b)))) < atol)


@pytest.mark.gpu
@pytest.mark.parametrize("w0,wn", [(0.2, 0.1), (0.0, 1e-3), (0.0, 0.0), (2.5, 0.1)])
def test_beacon_model_step_vs_oracle(gpu, O, w0, wn):
    E = gpu
    p = E.beacon_params()
    p.noise[1] = wn
    rng = np.random.default_rng(int(w0 * 10) + int(wn * 1e4))
    n = 4096
    st = np.stack([rng.uniform(5, 30, n), rng.uniform(5, 45, n), rng.uniform(-3.1, 3.1, n)]).astype(np.float32)
    nz = rng.standard_normal((3, n)).astype(np.float32)
    rec = np.zeros(1, E.STEP_INPUT_DTYPE)[0]
    rec["dt"] = 1.0
    rec["control"][:2] = [0.3, w0]
    rec["meas"][:10] = rng.uniform(2, 35, 10)
    gs, gl = E.model_step(BEACON, p, rec, st, nz)
    os_, ol = O.model_step(O.model_from_params(BEACON, p), st, nz, rec["control"][:2], rec["meas"][:16], dt=1.0)
    assert np.allclose(gs[0], os_[0], atol=2e-5, rtol=1e-6) and np.allclose(gs[1], os_[1], atol=2e-5, rtol=1e-6)
    assert _angle_close(gs[2], os_[2], 2e-5)
    # FP32 log-likelihood vs the FP64 oracle: relative 1e-4 plus an absolute floor
    assert np.all(np.abs(gl - ol) <= 1e-4 * np.abs(ol) + 5e-3), np.max(np.abs(gl - ol))


@pytest.mark.gpu
@pytest.mark.parametrize("res", [0, 1, 2])
def test_beacon_first_steps_vs_oracle(gpu, O, res):
    E = gpu
    p = E.beacon_params()
    inputs, _ = E.make_trace(BEACON, p, 2, 3)
    m, N, t = 256, 16, 2
    f = E.ParticleFilter(BEACON, p, particles_per_subfilter=m, num_subfilters=N, num_transfer=t, exchange=2,
                         resampler=res)
    f.record_selection(True)
    ppt = f.info()["particles_per_thread"]
    of = O.Filter(O.model_from_params(BEACON, p), m, N, t, O.EXCH_TORUS, res, O.RNG_SUBFILTER, 96, ppt, 1, 1.0,
                  0xF000000D, 0, np.array(p.init_state[:], np.float32))
    for k in range(3):
        if k > 0:  # both continue from the same particles: every step compared on equal inputs
            f.set_particles(of.state())
        ge = f.step(inputs[k])
        oe, osel = of.step(inputs["control"][k], inputs["meas"][k], want_sel=True)
        gs, gk = f.sorted()
        os_, ok = of.sorted()
        assert np.all(np.abs(gk - ok) <= 1e-4 * np.abs(ok) + 2e-3)
        d = np.abs(gs - os_)
        d[2] = np.abs(np.angle(np.exp(1j * (gs[2].astype(np.float64) - os_[2]))))
        assert np.mean(d.max(axis=0) < 1e-4) > 0.97  # near-ties may swap sorted positions
        assert abs(ge["log_norm"] - oe.log_norm) < 1e-3 * abs(oe.log_norm) + 1e-3
        assert np.allclose(ge["mean"][:2], oe.mean[:2], atol=2e-3)
        assert np.mean(f.selection() == osel) > 0.97


@pytest.mark.gpu
@pytest.mark.parametrize("res", [0, 1, 2])
@pytest.mark.parametrize("exch,t", [(1, 2), (2, 1)])
def test_beacon_pipelines_agree(gpu, res, exch, t):
    """Single-kernel, split and phased (same random layout) pipelines: bit for bit."""
    E = gpu
    p = E.beacon_params()
    inputs, _ = E.make_trace(BEACON, p, 3, 5)
    common = dict(particles_per_subfilter=256, num_subfilters=16, num_transfer=t, exchange=exch, resampler=res)
    a = E.ParticleFilter(BEACON, p, pipeline=E.PIPELINE_FUSED, **common)
    b = E.ParticleFilter(BEACON, p, pipeline=E.PIPELINE_SPLIT, **common)
    c = E.ParticleFilter(BEACON, p, pipeline=E.PIPELINE_SPLIT, rng=E.RNG_REFLAYOUT, mtgp_streams=96, **common)
    d = E.ParticleFilter(BEACON, p, pipeline=E.PIPELINE_PHASED, rng=E.RNG_REFLAYOUT, mtgp_streams=96, **common)
    for k in range(5):
        x, y = a.step(inputs[k]), b.step(inputs[k])
        assert np.array_equal(x["mean"], y["mean"]) and x["log_norm"] == y["log_norm"], k
        assert np.array_equal(x["best"], y["best"]) and x["best_subfilter"] == y["best_subfilter"], k
        u, w = c.step(inputs[k]), d.step(inputs[k])
        assert np.array_equal(u["best"], w["best"]) and u["best_subfilter"] == w["best_subfilter"], k
        assert np.allclose(u["mean"], w["mean"], rtol=1e-12, atol=1e-12), k
    assert np.array_equal(a.particles(), b.particles())


@pytest.mark.gpu
def test_beacon_rmse_matches_oracle(gpu, O):
    E = gpu
    p = E.beacon_params()
    steps = 60
    inputs, truth = E.make_trace(BEACON, p, 1, steps)
    f = E.ParticleFilter(BEACON, p, particles_per_subfilter=512, num_subfilters=8, num_transfer=0, exchange=0)
    g = [f.step(inputs[k]) for k in range(steps)]
    of = O.Filter(O.model_from_params(BEACON, p), 512, 8, 0, O.EXCH_NONE, O.RES_SYSTEMATIC, O.RNG_SUBFILTER, 96,
                  f.info()["particles_per_thread"], 1, 1.0, 0xF000000D, 0, np.array(p.init_state[:], np.float32))
    o = [of.step(inputs["control"][k], inputs["meas"][k])[0] for k in range(steps)]

    def rmse(ms):
        return float(np.sqrt(np.mean([(ms[k][0] - truth[k, 0]) ** 2 + (ms[k][1] - truth[k, 1]) ** 2
                                      for k in range(5, steps)])))

    rg, ro = rmse([e["mean"] for e in g]), rmse([e.mean for e in o])
    assert rg < 0.5 and ro < 0.5, (rg, ro)
    assert abs(rg - ro) <= 0.05 * ro + 0.005, (rg, ro)


@pytest.mark.gpu
def test_beacon_program_loop_on_trace(gpu, tmp_path):
    """pf_beacon_particle_filter == the same loop written against pf_step."""
    E = gpu
    p = E.beacon_params()
    inputs, truth = E.make_trace(BEACON, p, 4, 40)
    fn = tmp_path / "unicycle_trace"
    write_trace(fn, inputs, truth)
    got = E.beacon_particle_filter(256, 16, 1, fn)
    f = E.ParticleFilter(BEACON, p, particles_per_subfilter=256, num_subfilters=16, num_transfer=1, exchange=1,
                         resampler=E.RESAMPLE_REFERENCE, pipeline=E.PIPELINE_SPLIT)
    errs = []
    for rec, act in read_trace(E, fn):
        e = f.step(rec)
        errs.append(np.float32(np.hypot(np.float64(e["best"][0]) - act[0], np.float64(e["best"][1]) - act[1])))
    assert np.isfinite(got) and abs(got - np.mean(np.float64(errs))) <= 1e-5 * max(1.0, got)
    assert got < 2.0, got


@pytest.mark.gpu
def test_beacon_batch_equals_single_filters(gpu):
    E = gpu
    counts = [512, 1024, 256]
    params = []
    for i in range(3):
        q = E.beacon_params()
        q.init_state[0] += i
        params.append(q)
    traces = [E.make_trace(BEACON, q, 20 + i, 5) for i, q in enumerate(params)]
    inputs = np.stack([t[0] for t in traces])
    cfg = dict(num_transfer=2, exchange=1, resampler=1, particles_per_thread=2)
    B = E.FilterBatch(BEACON, params, counts, particles_per_subfilter=256, **cfg)
    best = [B.step(inputs[:, k]) for k in range(5)]
    for f, n in enumerate(counts):
        s = E.ParticleFilter(BEACON, params[f], pipeline=E.PIPELINE_SPLIT, particles_per_subfilter=256,
                             num_subfilters=n // 256, stream_offset=B.filter_info(f)["stream_offset"], **cfg)
        for k in range(5):
            e = s.step(inputs[f, k])
            assert np.array_equal(best[k][f]["mean"], e["mean"]) and best[k][f]["log_norm"] == e["log_norm"], (f, k)
        assert np.array_equal(B.particles(f), s.particles()), f


@pytest.mark.gpu
def test_beacon_server_same_alone_and_in_mix(gpu):
    """A served beacon filter gives its results alone whether or not unicycle
    and arm filters' updates share its batches."""
    E = gpu
    cfg = dict(particles_per_subfilter=256, particles_per_thread=4, num_transfer=2, exchange=1)
    p = E.beacon_params()
    steps = 6
    inputs, _ = E.make_trace(BEACON, p, 31, steps)

    def serve(mix):
        srv = E.Server(1 << 30, 8, **cfg)
        others = []
        if mix:
            for j, (model, n) in enumerate([(0, 2048), (1, 1024)]):
                q = E.unicycle_params(40 + j) if model == 0 else E.dharm_params(40 + j)
                others.append((srv.open(model, q, n, 40 + j), E.make_trace(model, q, 40 + j, steps)[0]))
        x = srv.open(BEACON, p, 2048, 31)
        out = {}
        for k in range(steps):
            srv.update(x, inputs[k], tag=k)
            for oid, oin in others:
                srv.update(oid, oin[k], tag=100 + k)
            srv.launch()
            for r in srv.poll(wait=True):
                if r["filter"] == x:
                    out[int(r["tag"])] = r["estimate"]
        while len(out) < steps:
            srv.launch()
            for r in srv.poll(wait=True):
                if r["filter"] == x:
                    out[int(r["tag"])] = r["estimate"]
        parts = srv.particles(x, 2048)[0]
        srv.close()
        return out, parts

    alone, pa = serve(False)
    mixed, pm = serve(True)
    for k in range(steps):
        a, b = alone[k], mixed[k]
        assert np.array_equal(a["mean"], b["mean"]) and a["log_norm"] == b["log_norm"], k
        assert np.array_equal(a["best"], b["best"]) and a["best_subfilter"] == b["best_subfilter"], k
    assert np.array_equal(pa, pm)


@pytest.mark.gpu
def test_beacon_cli(gpu, tmp_path):
    """pf_cli -M unicycle prints the drop-in loop's mean error for each run."""
    import subprocess
    from pathlib import Path
    E = gpu
    p = E.beacon_params()
    inputs, truth = E.make_trace(BEACON, p, 5, 20)
    fn = tmp_path / "unicycle_trace"
    write_trace(fn, inputs, truth)
    cli = Path(E.__file__).resolve().parent / "pf_cli"
    out = subprocess.run([str(cli), "-M", "unicycle", "-m", "128", "-N", "8", "-t", "1", str(fn)], check=True,
                         capture_output=True, text=True).stdout.split("\n")
    assert out[0] == "N m t e"
    n, m, t, e = out[1].split()
    assert (int(n), int(m), int(t)) == (8, 128, 1)
    assert abs(float(e) - E.beacon_particle_filter(128, 8, 1, fn)) <= 1e-6 * max(1.0, float(e))
