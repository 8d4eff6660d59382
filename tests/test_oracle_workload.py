"""The oracle's restatement of the seeded workloads (oracle/workload.py, used
by the bench's CPU arms so that they never load the engine) gives the same
parameters, inputs and ground truth as the engine's own generator."""
import numpy as np
import pytest


@pytest.mark.parametrize("model,seed", [(0, 1), (0, 2), (0, 7), (1, 3), (1, 11), (3, 0)])
def test_workload_equals_engine_generator(E, model, seed):
    import workload as Wk
    steps = 300
    if model == 0:
        pe, po = E.unicycle_params(seed), Wk.unicycle_params(seed)
        assert np.array_equal(np.array(pe.landmarks, np.float32), np.array(po.landmarks, np.float32))
        assert pe.dt == po.dt and list(pe.sigma_q) == po.sigma_q
    elif model == 1:
        pe, po = E.dharm_params(seed), Wk.dharm_params(seed)
        for k in ("a", "alpha", "d", "init_state"):
            assert np.array_equal(np.array(getattr(pe, k), np.float32), np.array(getattr(po, k), np.float32)), k
    else:
        pe, po = E.beacon_params(), Wk.beacon_params()
        assert np.array_equal(np.array(pe.beacons, np.float32), np.array(po.beacons, np.float32))
    inputs, truth = E.make_trace(model, pe, seed, steps)
    c, z, dt, tr = Wk.make_trace(model, po, seed, steps)
    assert np.array_equal(inputs["control"], c)
    assert np.array_equal(inputs["meas"], z)
    assert np.array_equal(inputs["dt"], dt)
    assert np.array_equal(truth, tr)


def test_oracle_model_from_workload_params(O, E):
    """model_from_params accepts the restated parameters and gives the same oracle model."""
    import workload as Wk
    a = O.model_from_params(0, E.unicycle_params(2))
    b = O.model_from_params(0, Wk.unicycle_params(2))
    assert bytes(a) == bytes(b)
    a = O.model_from_params(1, E.dharm_params(3))
    b = O.model_from_params(1, Wk.dharm_params(3))
    assert bytes(a) == bytes(b)
