"""A model added in one file (esthera_b200/csrc/pf_model_lingauss.cu, through
include/esthera_b200_model.cuh's PF_MODEL) runs through pf_create like a
built-in one, and the whole engine -- MTGP32 draws, the model, the sort, the
exchange, each resampler, the FP64 estimate -- tracks the exact posterior of
the linear-Gaussian model, the Kalman filter's, within Monte-Carlo error."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def kalman(params, z, dt):
    """FP64 Kalman filter of the model: x = (p, v), p' = p + v dt, v' = v +
    sigma_v n, z = p' + sigma_z e, starting from the point mass init_state."""
    x = np.array(params.init_state[:2], np.float64)
    P = np.zeros((2, 2))
    F = np.array([[1.0, dt], [0.0, 1.0]])
    Q = np.diag([0.0, params.sigma_v ** 2])
    H = np.array([[1.0, 0.0]])
    R = params.sigma_z ** 2
    means, sds = [], []
    for zk in z:
        x = F @ x
        P = F @ P @ F.T + Q
        S = (H @ P @ H.T)[0, 0] + R
        K = (P @ H.T)[:, 0] / S
        x = x + K * (zk - x[0])
        P = P - np.outer(K, H @ P)
        means.append(x.copy())
        sds.append(np.sqrt(np.maximum(np.diag(P), 0.0)))
    return np.array(means), np.array(sds)


def trace(params, steps, seed):
    rng = np.random.default_rng(seed)
    p, v = float(params.init_state[0]), float(params.init_state[1])
    z = np.zeros(steps)
    for k in range(steps):
        p = p + v * params.dt
        v = v + params.sigma_v * rng.standard_normal()
        z[k] = p + params.sigma_z * rng.standard_normal()
    return z


@pytest.mark.parametrize("res", [0, 1, 2])
def test_plugin_model_tracks_the_kalman_posterior(gpu, res):
    E = gpu
    prm = E.LinGaussParams(0.1, 0.5, 0.3, (0.0, 1.0))
    steps = 60
    z = trace(prm, steps, 11 + res)
    km, ks = kalman(prm, z, prm.dt)
    f = E.ParticleFilter(E.MODEL_LINGAUSS, prm, particles_per_subfilter=256, num_subfilters=256, num_transfer=2,
                         exchange=E.EXCHANGE_RING, resampler=res)
    inp = np.zeros(steps, E.STEP_INPUT_DTYPE)
    inp["dt"] = prm.dt
    inp["meas"][:, 0] = z
    est = np.array([f.step(inp[k])["mean"][:2] for k in range(steps)])
    # 256 sub-filters of 256 particles, each resampling on its own (the
    # reference's distributed filter: no weights carried across sub-filters),
    # so the Monte-Carlo error is that of 256-particle filters averaged: well
    # under a quarter of a posterior standard deviation
    tol = 0.25 * ks + 1e-3
    assert np.all(np.abs(est - km) <= tol), np.max(np.abs(est - km) / tol)
    rms = np.sqrt(np.mean(((est - km) / np.maximum(ks, 1e-3))[5:] ** 2))
    assert rms < 0.1, rms


def test_plugin_model_in_a_batch_equals_single_filters(gpu):
    """Batches take registered models too: each filter equals its single-filter run."""
    E = gpu
    prms = [E.LinGaussParams(0.1, 0.5, 0.3, (float(i), 1.0)) for i in range(3)]
    counts = [512, 1024, 256]
    steps = 6
    inputs = np.zeros((3, steps), E.STEP_INPUT_DTYPE)
    for i, p in enumerate(prms):
        inputs[i]["dt"] = p.dt
        inputs[i]["meas"][:, 0] = trace(p, steps, 40 + i)
    cfg = dict(num_transfer=1, exchange=E.EXCHANGE_RING, resampler=E.RESAMPLE_SYSTEMATIC)
    B = E.FilterBatch(E.MODEL_LINGAUSS, prms, counts, particles_per_subfilter=256, **cfg)
    best = [B.step(inputs[:, k]) for k in range(steps)]
    for i, n in enumerate(counts):
        s = E.ParticleFilter(E.MODEL_LINGAUSS, prms[i], pipeline=E.PIPELINE_SPLIT, particles_per_subfilter=256,
                             num_subfilters=n // 256, stream_offset=B.filter_info(i)["stream_offset"], **cfg)
        for k in range(steps):
            e = s.step(inputs[i, k])
            assert np.array_equal(best[k][i]["mean"], e["mean"]) and best[k][i]["log_norm"] == e["log_norm"], (i, k)
