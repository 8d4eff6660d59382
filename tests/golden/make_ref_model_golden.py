"""Run the reference's own model kernels -- the unicycle program's
sampling_importance (oracle/_ref/libref_unicycle.so, built by
oracle/build_ref_unicycle.sh) and the pinhole-camera arm's sampling_iw
(oracle/_ref/libref_camarm.so, oracle/build_ref_camarm.sh) -- on seeded
inputs and store inputs and outputs in ref_models.npz beside this script.
Needs a GPU (run it on one; the libraries travel with the repository
snapshot).  The CPU tests then check the oracle's FP64 model restatements
against these reference outputs."""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE.parent.parent / "oracle"))
sys.path.insert(0, str(HERE.parent))
import ref_kernels as R  # noqa: E402


def main():
    import esthera_b200 as E
    import oracle as O
    import test_camarm as T
    out = {}
    rng = np.random.default_rng(2024)
    n = 256
    # beacon: a cloud around (17, 30), the program's default constants
    st = np.stack([rng.normal(17, 0.5, n), rng.normal(30, 0.5, n), rng.uniform(-3.1, 3.1, n)]).astype(np.float32)
    nz = rng.standard_normal((3, n)).astype(np.float32)
    bx = np.array([12, 12, 13, 14, 16, 16, 18, 20, 20, 20], np.float64)
    by = np.array([12, 37, 25, 18, 12, 37, 30, 12, 25, 37], np.float64)
    z = (np.sqrt((17 - bx) ** 2 + (30 - by) ** 2 + 9) + rng.normal(0, 0.5, 10)).astype(np.float32)
    ctl = np.array([0.3, 0.2, 1.0], np.float32)  # v, omega, dt
    so, wt = R.unicycle_sampling(st, nz, float(ctl[0]), float(ctl[1]), float(ctl[2]), z)
    out.update(beacon_state=st, beacon_noise=nz, beacon_meas=z, beacon_ctl=ctl, beacon_state_out=so,
               beacon_weight=wt)
    # camera arm: a tight cloud around angles 2.0, the reference calibration
    p = E.camarm_params()
    st = T.cloud(rng, n, 2.0, 0.01)
    nz = (0.02 * rng.standard_normal((9, n))).astype(np.float32)
    c = rng.normal(0, 0.002, 5).astype(np.float32)
    zc = T.measurement(O, p, 2.0)
    so, wt = R.camarm_sampling(st, nz, c, zc, 1.0)
    out.update(camarm_state=st, camarm_noise=nz, camarm_control=c, camarm_meas=zc, camarm_state_out=so,
               camarm_weight=wt)
    dest = Path(sys.argv[1]) if len(sys.argv) > 1 else HERE / "ref_models.npz"
    np.savez_compressed(dest, **out)
    print("wrote", dest, sorted(out))


if __name__ == "__main__":
    main()
