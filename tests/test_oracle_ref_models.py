"""The oracle's FP64 model restatements against outputs of the reference's own
model kernels (the unicycle program's sampling_importance and the
pinhole-camera arm's sampling_iw), stored in tests/golden/ref_models.npz by
tests/golden/make_ref_model_golden.py on a GPU.  Tolerances: the reference
computes in FP32, the oracle in FP64 -- states within 2e-5 plus, for the
unicycle program's arc, its own FP32 cancellation 16 |v/w| 2^-24; log
weights within 1e-4 relative + 5e-3 of log(weight)."""
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_models.npz"
pytestmark = pytest.mark.skipif(not GOLDEN.exists(), reason="tests/golden/ref_models.npz not generated")


@pytest.fixture(scope="module")
def G():
    return dict(np.load(GOLDEN))


def test_oracle_beacon_equals_reference_kernel_outputs(O, E, G):
    p = E.beacon_params()
    v, w, dt = (float(x) for x in G["beacon_ctl"])
    p.dt = dt
    md = O.model_from_params(3, p)
    so, ll = O.model_step(md, G["beacon_state"], G["beacon_noise"], [v, w], G["beacon_meas"])
    sr, wt = G["beacon_state_out"], G["beacon_weight"]
    nz = G["beacon_noise"].astype(np.float64)
    tol = 2e-5 + 16.0 * np.abs((v + 0.5 * nz[0]) / (w + 0.1 * nz[1])) * 2.0 ** -24
    assert np.all(np.abs(so[0] - sr[0]) <= tol) and np.all(np.abs(so[1] - sr[1]) <= tol)
    assert np.all(np.abs(np.angle(np.exp(1j * (so[2].astype(np.float64) - sr[2])))) < 2e-5)
    ok = wt > 1e-30
    assert ok.mean() > 0.5
    assert np.allclose(ll[ok], np.log(wt[ok].astype(np.float64)), rtol=1e-4, atol=5e-3)


def test_oracle_camarm_equals_reference_kernel_outputs(O, E, G):
    md = O.model_from_params(4, E.camarm_params())
    so, ll = O.model_step(md, G["camarm_state"], G["camarm_noise"], G["camarm_control"], G["camarm_meas"])
    assert np.allclose(so, G["camarm_state_out"], atol=2e-5, rtol=0)
    wt = G["camarm_weight"]
    ok = wt > 1e-30
    assert ok.mean() > 0.5
    assert np.allclose(ll[ok], np.log(wt[ok].astype(np.float64)), rtol=1e-4, atol=5e-3)
