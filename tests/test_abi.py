"""The C-ABI library: loads without a GPU, exports every symbol declared in
include/*.h, validates configurations on the host, and has no CPU path."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(pf[a-z]*_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_every_declared_symbol_is_exported(E):
    L = E.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    assert len(declared_functions()) > 30


def test_version_and_status_strings(E):
    assert E.lib().pf_version() >= 100
    assert E.status_string(E.PF_ERR_ADMISSION) == "admission rejected"


def test_default_config(E):
    c = E.default_config()
    assert (c.particles_per_subfilter, c.resampler, c.rng, c.log_weights) == (512, E.RESAMPLE_SYSTEMATIC,
                                                                               E.RNG_SUBFILTER, 1)
    assert c.seed == 0xF000000D


def test_model_info(E):
    assert E.model_info(E.MODEL_UNICYCLE) == (3, 3, 2, 16)
    assert E.model_info(E.MODEL_DHARM) == (12, 6, 0, 6)
    assert E.model_info(E.MODEL_REFARM) == (9, 9, 5, 7)
    assert E.model_info(E.MODEL_BEACON) == (3, 3, 2, 16)
    assert E.model_info(E.MODEL_CAMARM) == (9, 9, 5, 7)
    with pytest.raises(E.PFError):
        E.model_info(5)


def test_model_params_validated_on_the_host(E):
    """Bad model parameters are refused before any GPU work (on a GPU-less
    host the valid ones then fail with PF_ERR_CUDA: no CPU path)."""
    b = E.beacon_params()
    for field, val in [("num_beacons", 0), ("num_beacons", 17), ("sigma_range", 0.0)]:
        q = E.BeaconParams.from_buffer_copy(b)
        setattr(q, field, val)
        with pytest.raises(E.PFError) as ei:
            E.ParticleFilter(E.MODEL_BEACON, q, num_subfilters=8)
        assert ei.value.status == E.PF_ERR_INVALID, field
    # a params struct of the wrong model is refused by its size
    with pytest.raises(E.PFError) as ei:
        E.ParticleFilter(E.MODEL_CAMARM, b, num_subfilters=8)
    assert ei.value.status == E.PF_ERR_INVALID
    if E.device_count() == 0:
        for model, params in [(E.MODEL_BEACON, b), (E.MODEL_CAMARM, E.camarm_params())]:
            with pytest.raises(E.PFError) as ei:
                E.ParticleFilter(model, params, num_subfilters=8)
            assert ei.value.status == E.PF_ERR_CUDA


@pytest.mark.parametrize("kw,msg", [
    (dict(particles_per_subfilter=48), "power of two"),
    (dict(particles_per_subfilter=2048), "power of two"),
    (dict(exchange=2, num_subfilters=2048, num_transfer=103), "5*t"),
    (dict(exchange=2, num_subfilters=7, num_transfer=1), "dx*dy"),
    (dict(exchange=1, num_transfer=300), "2*t"),
    (dict(resampling_freq=1.5), "resampling_freq"),
    (dict(ess_fraction=-0.1), "ess_fraction"),
    (dict(pipeline=1, rng=0), "phased"),
    (dict(rng=1, mtgp_streams=201), "mtgp_streams"),
    (dict(particles_per_thread=3), "not built"),
])
def test_config_validation(E, kw, msg):
    p = E.unicycle_params(1)
    with pytest.raises(E.PFError) as ei:
        E.ParticleFilter(E.MODEL_UNICYCLE, p, **kw)
    assert msg in str(ei.value)


def test_bounded_wait_argument_checks(E):
    with pytest.raises(E.PFError):
        E.bounded_wait_test(0)
    for lim in (np.zeros(48, np.int32), np.zeros(2048, np.int32), np.full(64, -1, np.int32)):
        with pytest.raises(E.PFError) as ei:
            E.bounded_wait_mixed_test(lim)
        assert ei.value.status == E.PF_ERR_INVALID


def test_no_cpu_fallback(E):
    if E.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(E.PFError) as ei:
        E.ParticleFilter(E.MODEL_UNICYCLE, E.unicycle_params(1), num_subfilters=8)
    assert ei.value.status == E.PF_ERR_CUDA
    with pytest.raises(E.PFError):
        E.bitonic_sort(np.zeros(64, np.float32), 64)


def test_trace_generator_deterministic(E):
    p = E.unicycle_params(1)
    assert p.num_landmarks == 4
    lm = np.array([[p.landmarks[j][0], p.landmarks[j][1]] for j in range(4)])
    assert np.all(np.abs(lm) <= 10)
    a, ta = E.make_trace(E.MODEL_UNICYCLE, p, 1, 100)
    b, tb = E.make_trace(E.MODEL_UNICYCLE, p, 1, 100)
    c, tc = E.make_trace(E.MODEL_UNICYCLE, p, 2, 100)
    assert np.array_equal(ta, tb) and not np.array_equal(ta, tc)
    assert np.allclose(a["dt"], 0.1) and np.allclose(a["control"][:, 0], 1.0)
    assert np.allclose(a["control"][:, 1], 0.3 * np.sin(0.05 * 0.1 * np.arange(100)), atol=1e-6)
    # measurements are noisy ranges/bearings of the truth
    dx = lm[None, :, 0] - ta[:, None, 0]
    dy = lm[None, :, 1] - ta[:, None, 1]
    r = np.hypot(dx, dy)
    assert np.std(a["meas"][:, :4] - r) < 0.3
    d = np.angle(np.exp(1j * (a["meas"][:, 4:8] - (np.arctan2(dy, dx) - ta[:, None, 2]))))
    assert np.std(d) < 0.08


def test_dharm_params_from_seed(E):
    p = E.dharm_params(3)
    a = np.array(p.a[:])
    assert np.all((a >= 0.2) & (a <= 0.6))
    al = np.array(p.alpha[:])
    assert np.all(np.isclose(np.abs(al), np.pi / 2, atol=1e-6) | (al == 0))
    inp, tr = E.make_trace(E.MODEL_DHARM, p, 3, 50)
    assert tr.shape == (50, 12) and np.all(np.isfinite(inp["meas"][:, :6]))


def test_read_trace_line_reference_format(E, tmp_path):
    # robot-arm trace format of pf_model_soa.cuh:276-301
    vals = [0.5, 1.5] + [2.0, 2.1, 2.2, 2.3, 2.4] + [0.01, -0.02, 0.03, -0.04, 0.05] + [1, 0.7, 0.8] + \
           [2.01, 2.11, 2.21, 2.31, 2.41]
    f = tmp_path / "trace"
    f.write_text(" ".join(map(str, vals)) + "\n" + " ".join(map(str, vals)) + "\n")
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    fp = libc.fopen(str(f).encode(), b"r")
    inp = E.StepInput()
    act = np.zeros(16, np.float32)
    n = 0
    while E.lib().pf_read_trace_line(fp, E.MODEL_REFARM, C.byref(inp), act.ctypes.data_as(C.POINTER(C.c_float))) == 0:
        n += 1
    libc.fclose(fp)
    assert n == 2
    assert np.allclose(inp.meas[:7], [2.0, 2.1, 2.2, 2.3, 2.4, 0.5, 1.5])
    assert np.allclose(inp.control[:5], [0.01, -0.02, 0.03, -0.04, 0.05]) and inp.dt == 1.0
    assert np.allclose(act[:9], [2.01, 2.11, 2.21, 2.31, 2.41, 0.7, 0.8, 0, 0])
    est = act.copy()
    est[5] += 1.0
    assert abs(E.lib().pf_refarm_estimate_error(est.ctypes.data_as(C.POINTER(C.c_float)),
                                                act.ctypes.data_as(C.POINTER(C.c_float))) - 0.1) < 1e-6


def test_cli_binary_built():
    assert (ROOT / "esthera_b200" / "pf_cli").exists()


def test_driver_trace_errors_on_the_host(E, tmp_path):
    """Malformed or missing traces fail with PF_ERR_IO before any GPU work (no
    exit(), unlike the reference's drivers); an unknown model's trace is
    PF_ERR_UNSUPPORTED."""
    assert E.lib().pf_particle_filter(64, 2, 1, 1.0, str(tmp_path / "absent").encode(), None) == E.PF_ERR_IO
    assert E.lib().pf_beacon_particle_filter(64, 2, 1, str(tmp_path / "absent").encode(), None) == E.PF_ERR_IO
    fn = tmp_path / "bad"
    fn.write_text("0.5 1.5 2.0 2.1 oops 2.3 2.4\n")
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    inp = E.StepInput()
    act = np.zeros(16, np.float32)
    fp = libc.fopen(str(fn).encode(), b"r")
    for model, want in [(E.MODEL_REFARM, E.PF_ERR_IO), (E.MODEL_UNICYCLE, E.PF_ERR_UNSUPPORTED)]:
        got = E.lib().pf_read_trace_line(fp, model, C.byref(inp), act.ctypes.data_as(C.POINTER(C.c_float)))
        assert got == want, (model, got)
    libc.fclose(fp)
    assert E.lib().pf_read_trace_line(None, E.MODEL_REFARM, C.byref(inp),
                                      act.ctypes.data_as(C.POINTER(C.c_float))) == E.PF_ERR_INVALID


def test_cli_rejects_unknown_model_and_missing_trace(tmp_path):
    import subprocess
    cli = ROOT / "esthera_b200" / "pf_cli"
    r = subprocess.run([str(cli), "-M", "bogus", str(tmp_path / "t")], capture_output=True, text=True)
    assert r.returncode == 1 and "unknown model" in r.stderr
    r = subprocess.run([str(cli), "-M", "unicycle"], capture_output=True, text=True)
    assert r.returncode == 1 and "no input file" in r.stderr
    r = subprocess.run([str(cli), "-M", "unicycle", "-m", "64", "-N", "2", str(tmp_path / "absent")],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "error" in r.stderr  # PF_ERR_IO before any GPU work


def test_model_registry(E):
    """Every model registers itself at load time: the five built-in ones and the
    linear-Gaussian example added with PF_MODEL in one file."""
    ids = E.model_list()
    assert set(ids) >= {0, 1, 2, 3, 4, E.MODEL_LINGAUSS}
    assert [E.model_name(i) for i in range(5)] == ["unicycle", "dharm", "refarm", "beacon", "camarm"]
    assert E.model_name(E.MODEL_LINGAUSS) == "lingauss" and E.model_name(63) is None
    assert E.model_info(E.MODEL_LINGAUSS) == (2, 1, 0, 1)
    with pytest.raises(E.PFError) as ei:
        E.model_info(63)
    assert ei.value.status == E.PF_ERR_INVALID
    if E.device_count() == 0:  # no CPU path for a registered model either
        with pytest.raises(E.PFError) as ei:
            E.ParticleFilter(E.MODEL_LINGAUSS, E.LinGaussParams(0.1, 0.2, 0.5, (0.0, 1.0)), num_subfilters=4)
        assert ei.value.status == E.PF_ERR_CUDA
